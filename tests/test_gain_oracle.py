"""Pump-gain single-mode propagation (disp_gain_smf!, solve_disp_gain_smf;
YDFA rate equations) in the FP64 oracle and the host gain setup -- CPU only.

Pinned on the reference's own test (test/core/test_numerical_kernels.jl:5-25:
YDFA initialisation and a pumped propagation that succeeds with a finite
field), on closed forms (constant gain with no nonlinearity or dispersion;
the rate-equation limits of no light and of a saturating pump) and on a
literal restatement of the right-hand side.
"""
import math
import os

import numpy as np
import pytest

from fiberlab_gpu import gain as G
from fiberlab_gpu import problem as P
from oracle import oracle as O

# A checkout of the reference project, when one is available: its Yb
# cross-section data (src/gain_simulation/Yb_*.npz) then drives the
# "reference" case; without it that case is skipped.
REF_ROOT = os.environ.get("FIBERLAB_REFERENCE_ROOT", "")
REF_DATA = os.path.join(REF_ROOT, "src", "gain_simulation") if REF_ROOT else ""


def _synthetic_sections():
    # smooth Yb-like shapes (a 976 nm absorption peak, emission red of it)
    wl = np.linspace(900e-9, 1150e-9, 60)
    sa = 2.5e-24 * np.exp(-((wl - 976e-9) / 8e-9) ** 2) + 6e-26 * np.exp(-((wl - 1030e-9) / 20e-9) ** 2)
    se = 2.5e-24 * np.exp(-((wl - 976e-9) / 8e-9) ** 2) + 6e-25 * np.exp(-((wl - 1030e-9) / 25e-9) ** 2)
    return (wl, sa), (wl, se)


def _reference_sections():
    ab, em = (os.path.join(REF_DATA, f) for f in ("Yb_absorption.npz", "Yb_emission.npz"))
    if not (REF_DATA and os.path.exists(ab) and os.path.exists(em)):
        pytest.skip("the reference's Yb cross-section data is not present "
                    "(set FIBERLAB_REFERENCE_ROOT to a reference checkout)")
    a, e = np.load(ab), np.load(em)
    # get_ydfa_cross_sections: wavelength in nm, intensity x 1e-27 m²
    return (a["wavelength"] * 1e-9, a["intensity"] * 1e-27), (e["wavelength"] * 1e-9,
                                                               e["intensity"] * 1e-27)


def _kat_problem(**kw):
    # get_disp_sim_params(1030e-9, 1, 32, 5.0, 2); launch gauss 1e-4 W, 300 fs,
    # 80 MHz; user-defined fiber L = 1e-5 m, fR = 0, γ = 0, β = [0]
    return P.single_mode_problem(nt=32, time_window_ps=5.0, L=1e-5, power_w=1e-4,
                                 fwhm_s=300e-15, rep_rate_hz=80e6, gamma=0.0, betas=(0.0,),
                                 beta_order=2, fR=0.0, wavelength_m=1030e-9, pulse="gauss",
                                 reltol=1e-5, **kw)


@pytest.mark.parametrize("sections", ["reference", "synthetic"])
def test_ydfa_initialisation_and_pumped_propagation(sections):
    # test_numerical_kernels.jl:5-25
    ab, em = _reference_sections() if sections == "reference" else _synthetic_sections()
    fp = _kat_problem()
    p = G.ydfa_params(fp.sim, ab, em)
    for s in (p.sigma_as, p.sigma_es):
        assert len(s) == fp.nt and np.all(np.isfinite(s)) and np.all(s >= 0)
    out, pumps, st = O.forward_gain(fp, p, 0.05)
    assert st["z_end"] == fp.L and np.all(np.isfinite(out[-1])) and np.isfinite(pumps[-1])
    assert pumps[0] == 0.05 and np.array_equal(out[0], fp.uw0)


def test_constant_gain_closed_form():
    # no nonlinearity, no dispersion: u(L) = u0 e^{gL/2}; the constant model's
    # pump gain is -1 (the reference's placeholder): P(L) = P0 e^{-L}
    fp = P.single_mode_problem(nt=64, time_window_ps=3.0, L=0.5, power_w=1e-3, rep_rate_hz=80e6,
                               gamma=0.0, betas=(0.0,), beta_order=2, fR=0.0, reltol=1e-10,
                               abstol=1e-12)
    zs = [0.0, 0.17, 0.31, fp.L]
    out, pumps, _ = O.forward_gain(fp, 0.8, 0.05, zsave=zs)
    for z, u, pz in zip(zs, out, pumps):
        # the dense output at interior positions holds to the interpolant's order
        assert np.linalg.norm(u - fp.uw0 * math.exp(0.4 * z)) <= 1e-9 * np.linalg.norm(u)
        assert pz == pytest.approx(0.05 * math.exp(-z), rel=1e-9)


def test_gain_rhs_matches_literal_restatement():
    # disp_gain_smf! = disp_mmf! + g(ω)/2 ũ, dP/dz = g_P P, with the YDFA gain
    # of the lab-frame field e^{iDz} ũ and the pump power
    fp = P.single_mode_problem(nt=128, time_window_ps=3.0, L=0.3, power_w=0.1, rep_rate_hz=80e6,
                               wavelength_m=1030e-9)
    ab, em = _synthetic_sections()
    p = G.ydfa_params(fp.sim, ab, em)
    rng = np.random.default_rng(4)
    u = fp.uw0 * np.exp(0.3j * rng.standard_normal(fp.nt))[None, :]
    z, pump = 0.137, 0.3
    dP, du = O.rhs_gain(fp, p, z, pump, u)
    g, gp = G.ydfa_gain(p, np.exp(1j * fp.D[0] * z) * u[0], pump)
    ref = O.rhs_forward(fp, z, u) + 0.5 * g[None, :] * u
    assert np.linalg.norm(du - ref) <= 1e-12 * np.linalg.norm(ref)
    assert abs(dP - gp * pump) <= 1e-14 * abs(gp * pump)


def test_rate_equation_limits():
    sim = P.get_disp_sim_params(1030e-9, 1, 64, 5.0, 2)
    ab, em = _synthetic_sections()
    p = G.ydfa_params(sim, ab, em)
    a = G.gain_struct_arrays(p)
    # no light at all: every ion in the ground state (n2 = 0)
    g, gp = G.ydfa_gain(p, np.zeros(sim["Nt"]), 0.0)
    assert np.allclose(g, -a["gamma_s"] * a["sigma_as"] * p.rho, rtol=1e-14, atol=0)
    assert gp == pytest.approx(-a["gamma_p"] * p.sigma_ap * p.rho, rel=1e-14)
    # a saturating pump: n2 -> σap / (σap + σep) (1/2 for equal cross sections)
    g, gp = G.ydfa_gain(p, np.zeros(sim["Nt"]), 1e9)
    assert np.allclose(g, a["gamma_s"] * (a["sigma_es"] - a["sigma_as"]) * 0.5 * p.rho,
                       rtol=1e-6, atol=1e-12)
    assert abs(gp) < 1e-6 * a["gamma_p"] * p.sigma_ap * p.rho


def test_marcuse_overlap_and_defaults():
    # the default pump channel: V = 2π a NA / λ = 2.0924..., w = a (0.616 +
    # 1.66 V^-1.5 + 0.987 V^-6), Γ = 1 - exp(-2 a²/w²)
    a, na, lam = 2.5e-6, 0.13, 976e-9
    V = 2 * math.pi * a * na / lam
    w = a * (0.616 + 1.66 / V ** 1.5 + 0.987 / V ** 6)
    assert G.marcuse_overlap(a, na, lam) == pytest.approx(1 - math.exp(-2 * a * a / (w * w)),
                                                         rel=1e-15)
    sim = P.get_disp_sim_params(1030e-9, 1, 32, 5.0, 2)
    p = G.YDFAParams(fs=sim["fs"], dt_ps=sim["Δt"], nt=32)
    assert p.df == pytest.approx(1 / (32 * sim["Δt"] * 1e-12))
    assert 0 < p.gamma_s < p.gamma_p < 1
    with pytest.raises(P.ArgumentError):
        G.interpolate_cross_sections(sim["fs"], [1e-6], [1e-25])
