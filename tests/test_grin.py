"""GRIN multimode setup (index profile, scalar mode solver, β(f) finite
differences, D(ω), γ) -- CPU only.

Checked against textbook facts the reference's own pipeline relies on: the
fused-silica Sellmeier index, central finite-difference weights, the 5-point
operator built independently, the harmonic-oscillator mode groups of a
parabolic core (degeneracies 1, 2, 3 and equal β² spacing 2 k NA / a), the
Gaussian-mode estimate of γ, and silica's material dispersion at 1030 nm.
"""
import math

import numpy as np
import pytest

from fiberlab_gpu import grin as G
from fiberlab_gpu import problem as P
from oracle import oracle as O


def test_central_fd_weights_known_answers():
    assert np.allclose(G.central_fd_weights(3, 2), [1, -2, 1], atol=1e-14)
    assert np.allclose(G.central_fd_weights(5, 1), [1 / 12, -2 / 3, 0, 2 / 3, -1 / 12], atol=1e-14)
    assert np.allclose(G.central_fd_weights(7, 3), [1 / 8, -1, 13 / 8, 0, -13 / 8, 1, -1 / 8],
                       atol=1e-13)
    with pytest.raises(P.ArgumentError):
        G.central_fd_weights(4, 1)


def test_silica_index():
    assert G.silica_index(1.55) == pytest.approx(1.44402, abs=2e-5)
    assert G.silica_index(0.5876) == pytest.approx(1.45846, abs=5e-5)   # d line


def test_mode_operator_matches_a_dense_build():
    nx, dx, lam = 6, 0.7, 1.03
    eps = 1 + np.random.default_rng(0).random((nx, nx))
    A = G.mode_operator(lam, dx, eps).toarray()
    ref = np.zeros((nx * nx, nx * nx))
    k2 = (2 * math.pi / lam) ** 2
    for j in range(nx):
        for i in range(nx):
            p = i + nx * j
            ref[p, p] = eps[i, j] * k2 - 4 / dx ** 2
            for ii, jj in ((i - 1, j), (i + 1, j), (i, j - 1), (i, j + 1)):
                if 0 <= ii < nx and 0 <= jj < nx:
                    ref[p, ii + nx * jj] = 1 / dx ** 2
    assert np.allclose(A, ref, rtol=1e-15, atol=0)


def test_parabolic_core_mode_groups():
    lam, a, na = 1.03, 25.0, 0.2
    eps, x, dx = G.build_grin(lam, 96, 100.0, a, na, 2.0)
    d, v, neff = G.solve_fiber_modes(lam, 6, dx, eps)
    assert np.all(np.diff(d) <= 0) and np.allclose(np.linalg.norm(v, axis=0), 1.0)
    # groups of 1, 2, 3 nearly degenerate modes, equally spaced in β²
    gaps = -np.diff(d)
    within = max(gaps[1], gaps[3], gaps[4])
    between = min(gaps[0], gaps[2])
    assert within < 0.02 * between
    k = 2 * math.pi / lam
    assert gaps[0] == pytest.approx(2 * k * na / a, rel=0.03)
    assert gaps[2] == pytest.approx(2 * k * na / a, rel=0.03)


def test_grin_params_reference_frame_dispersion_and_gamma():
    sim = P.get_disp_sim_params(1030e-9, 6, 256, 10.0, 3)
    g = G.grin_params(sim, 64, 100.0, 25.0, 0.2, 2.0)
    betas, D, gam = g["betas"], g["D"], g["gamma"]
    assert betas.shape == (4, 6) and D.shape == (6, 256)
    # mode 1 is the reference frame: zero β0 and β1
    assert betas[0, 0] == 0 and betas[1, 0] == 0 and D[0, 0] == 0
    # the LP11 pair shares its propagation constant
    assert betas[0, 1] == pytest.approx(betas[0, 2], rel=1e-6)
    # silica's material GVD at 1030 nm (~19 ps²/km) dominates β2
    assert 1.7e-26 < betas[2, 0] < 2.1e-26
    assert P.gamma_symmetric(gam) and gam[0, 0, 0, 0] > 0
    # γ of the fundamental against a Gaussian of w0² = a λ / (π NA)
    w0 = math.sqrt(25e-6 * 1030e-9 / (math.pi * 0.2))
    gauss = P.N2_SILICA * 2 * math.pi * sim["f0"] * 1e12 / (P.C0 * math.pi * w0 ** 2)
    assert gam[0, 0, 0, 0] == pytest.approx(gauss, rel=0.05)
    modes = g["modes"]
    assert np.allclose(np.sum(modes ** 2, axis=(0, 1)), 1.0)


def test_grin_problem_runs_through_the_oracle():
    fp = G.grin_problem(3, 256, 5.0, 0.05, 2e-9, 200e-15, nx=40,
                        weights=[0.8, 0.5, 0.33], raman_threshold_thz=-5.0)
    fp.validate()
    out, st, _ = O.forward(fp)
    n0, n1 = P.photon_number(out[0], fp.sim), P.photon_number(out[-1], fp.sim)
    assert st["naccept"] > 0 and abs(n1 / n0 - 1) < 1e-6
