"""Objective epilogues (Raman band, fundamental mode, worst mode, spectral
peak, temporal width; dB form) -- CPU only.

The cost/seed restatements are pinned on the reference's own known-answer
tests (test/core/test_numerical_kernels.jl:275-294,
test/core/test_fiberlab_api.jl:2215-2230), each seed is checked as the
Wirtinger gradient of its cost by central differences, and the seeds are
driven through the FP64 oracle's adjoint against central differences of the
oracle's forward cost (the chain rule the GPU path uses).
"""
import numpy as np
import pytest

from fiberlab_gpu import objectives as Ob
from fiberlab_gpu import problem as P
from oracle import oracle as O


def _sim(nt=64):
    return P.get_disp_sim_params(1550e-9, 1, nt, 10.0, 2)


def _directional(cost, seed, u, d, h):
    fd = (cost(u + h * d) - cost(u - h * d)) / (2 * h)
    return fd, 2.0 * float(np.real(np.sum(np.conj(seed) * d)))


def test_temporal_width_known_answers():
    # test_numerical_kernels.jl:275-294
    nt = 64
    sim = _sim(nt)
    centred = np.zeros((1, nt), complex)
    centred[0, nt // 2] = 1
    edge = np.zeros((1, nt), complex)
    edge[0, 0] = 1
    assert Ob.temporal_width_cost(np.fft.ifft(centred, axis=1), sim)[0] < 1e-30
    assert Ob.temporal_width_cost(np.fft.ifft(edge, axis=1), sim)[0] == 1.0
    field = np.exp(0.17j * np.arange(1, nt + 1))[None, :]
    direction = np.exp(0.31j * np.arange(1, nt + 1))[None, :]
    _, seed = Ob.temporal_width_cost(field, sim)
    fd, adj = _directional(lambda u: Ob.temporal_width_cost(u, sim)[0], seed, field, direction,
                           1e-6)
    assert abs(fd - adj) <= 1e-6 * abs(adj) + 1e-8


def test_worst_mode_known_answers():
    # test_fiberlab_api.jl:2215-2230 (modes as rows here)
    mask = np.array([True, True, False, False])
    field = np.zeros((3, 4), complex)
    field[0, 0] = 1
    field[1, 2] = 1
    cost, seed = Ob.worst_mode_band_cost(field, mask, tau=50.0)
    assert 1 - np.log(2) / 50 <= cost <= 1
    assert np.all(seed[2] == 0)
    unit, _ = Ob.worst_mode_band_cost(field[[0, 2]], mask, tau=50.0)
    assert unit == 1.0
    with pytest.raises(P.ArgumentError):
        Ob.worst_mode_band_cost(np.zeros((2, 4), complex), mask)
    with pytest.raises(P.ArgumentError):
        Ob.worst_mode_band_cost(field, mask, tau=0.0)


def test_fundamental_seed_only_on_mode_one():
    rng = np.random.default_rng(1)
    u = rng.standard_normal((3, 32)) + 1j * rng.standard_normal((3, 32))
    mask = np.arange(32) < 9
    J, seed = Ob.fundamental_band_cost(u, mask)
    assert J == pytest.approx(np.sum(np.abs(u[0, :9]) ** 2) / np.sum(np.abs(u[0]) ** 2), rel=1e-15)
    assert np.all(seed[1:] == 0)


def test_band_objective_is_the_mode_sum():
    rng = np.random.default_rng(2)
    u = rng.standard_normal((2, 32)) + 1j * rng.standard_normal((2, 32))
    mask = np.arange(32) >= 20
    for name in ("raman_band", "mode_sum", "mmf_sum"):
        J, seed = Ob.cost_and_seed(name, u, mask)
        J0, seed0 = P.band_cost_and_seed(u, mask)
        assert J == J0 and np.array_equal(seed, seed0)
    with pytest.raises(P.ArgumentError):
        Ob.objective("no_such_objective", mask)
    with pytest.raises(P.ArgumentError):
        Ob.spectral_peak_cost(u, np.zeros(32, bool))


@pytest.mark.parametrize("name", ["raman_band", "fundamental_mode", "worst_mode", "raman_peak",
                                  "temporal_width"])
@pytest.mark.parametrize("log_cost", [False, True])
def test_seed_is_the_gradient_of_the_cost(name, log_cost):
    nt = 64
    sim = _sim(nt)
    rng = np.random.default_rng(7)
    u = rng.standard_normal((3, nt)) + 1j * rng.standard_normal((3, nt))
    mask = P.fftfreq(nt, 1 / sim["Δt"]) < -0.5
    J, seed = Ob.cost_and_seed(name, u, mask, sim, log_cost, worst_mode_tau=5.0)

    def cost(x):
        return Ob.cost_and_seed(name, x, mask, sim, log_cost, worst_mode_tau=5.0)[0]
    for _ in range(3):
        d = rng.standard_normal(u.shape) + 1j * rng.standard_normal(u.shape)
        fd, adj = _directional(cost, seed, u, d / np.linalg.norm(d), 1e-6)
        assert abs(fd - adj) <= 1e-6 * abs(adj) + 1e-9


@pytest.mark.parametrize("name", ["fundamental_mode", "worst_mode", "raman_peak",
                                  "temporal_width"])
def test_objective_seed_through_the_oracle_adjoint(name):
    # ∂J/∂φ = 2 Re(conj(λ0) i u_shaped) summed over modes, λ0 from the oracle
    # adjoint seeded by the objective, against central differences of the
    # oracle forward cost (tight tolerances so both sides resolve 1e-3)
    fp = P.multimode_problem(1, 32, 256, 5.0, 0.3, 5e-9, 200e-15, seed=3,
                             raman_threshold_thz=-3.0)
    fp.reltol, fp.abstol = 1e-11, 1e-11
    rng = np.random.default_rng(5)
    phi = 0.3 * rng.standard_normal(fp.nt)

    def shaped(ph):
        return fp.uw0 * np.exp(1j * ph)[None, :]

    def cost(ph):
        out, _, _ = O.forward(fp, u0=shaped(ph))
        return Ob.cost_and_seed(name, out[-1], fp.mask, fp.sim)[0]
    out, _, dense = O.forward(fp, u0=shaped(phi), keep_dense=True)
    J, seed = Ob.cost_and_seed(name, out[-1], fp.mask, fp.sim)
    lam0, _ = O.adjoint(fp, dense, seed)
    g = np.sum(2 * np.real(np.conj(lam0) * 1j * shaped(phi)), axis=0)
    for _ in range(2):
        d = rng.standard_normal(fp.nt)
        d /= np.linalg.norm(d)
        h = 1e-4
        fd = (cost(phi + h * d) - cost(phi - h * d)) / (2 * h)
        assert abs(fd - g @ d) <= 1e-3 * abs(fd) + 1e-12
