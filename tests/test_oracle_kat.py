"""Pins the FP64 CPU oracle against the reference's own known-answer tests
and published numbers (CPU only).

Each test restates one reference test or published figure:
  test/core/test_numerical_kernels.jl, test/core/test_propagation.jl,
  test/core/test_scalar_crosscheck.jl,
  docs/research/counterfactual-raman-benchmark.md.
"""
import numpy as np
import pytest

from fiberlab_gpu import problem as P
from oracle import oracle as O


def _custom(nt, L, D, gamma, hR, one_m_fR, launch, sim, reltol=1e-8, abstol=1e-6, mask=None):
    return P.FiberProblem(sim=sim, D=D, gamma=gamma, hR=hR, one_m_fR=one_m_fR, L=L,
                          uw0=launch, reltol=reltol, abstol=abstol, mask=mask)


def test_tsit5_tableau_order_conditions():
    # Tsitouras (2011) tableau and free interpolant: order conditions hold
    for th in (0.13, 0.5, 0.91, 1.0):
        assert np.max(np.abs(O.tsit5_order_residuals(th))) < 1e-13


def test_fft_conventions():
    # test_numerical_kernels.jl:259-265: fft(ifft(x)) == x and Parseval with N
    nt = 64
    temporal = np.exp(2j * np.pi * np.arange(nt) / nt)
    spectrum = O.fft(temporal, inverse=True)
    assert np.allclose(O.fft(spectrum), temporal, rtol=1e-14, atol=1e-14)
    assert abs(nt * np.sum(np.abs(spectrum) ** 2) - np.sum(np.abs(temporal) ** 2)) < 1e-12
    x = np.random.default_rng(0).standard_normal(256) + 1j
    assert np.allclose(O.fft(x), np.fft.fft(x), rtol=1e-13, atol=1e-12)
    assert np.allclose(O.fft(x, inverse=True), np.fft.ifft(x), rtol=1e-13, atol=1e-14)


def test_analytic_cw_kerr():
    # test_numerical_kernels.jl:329-353
    nt, L, pw, g = 64, 5.0, 2.0, 0.73
    sim = P.get_disp_sim_params(1550e-9, 1, nt, 10.0, 2)
    launch = np.fft.ifft(np.full((1, nt), np.sqrt(pw), complex), axis=1)
    base = dict(nt=nt, L=L, D=np.zeros((1, nt)), gamma=np.full((1, 1, 1, 1), g),
                hR=np.zeros(nt, complex), one_m_fR=1.0, launch=launch, sim=sim)
    expected = launch * np.exp(1j * g * pw * L)
    loose = O.forward(_custom(**base, reltol=1e-4, abstol=1e-6))[0][-1]
    tight = O.forward(_custom(**base, reltol=1e-10, abstol=1e-12))[0][-1]
    le = np.linalg.norm(loose - expected) / np.linalg.norm(expected)
    te = np.linalg.norm(tight - expected) / np.linalg.norm(expected)
    assert te < 1e-8
    assert te < 1e-3 * le


def test_exact_linear_multimode():
    # test_propagation.jl:124-150
    nt, modes, L = 32, 2, 0.1
    sim = P.get_disp_sim_params(1550e-9, modes, nt, 5.0, 2)
    t = sim["ts"] * 1e12
    env = np.exp(-0.5 * (t / 0.4) ** 2)
    second = (0.4 + 0.2j) * np.exp(-0.5 * ((t - 0.25) / 0.25) ** 2)
    launch = np.fft.ifft(np.stack([env, second]).astype(complex), axis=1)
    off = P.fftfreq(nt, 1 / sim["Δt"])
    D = np.stack([0.02 * off ** 2, -0.015 * off ** 2])
    fp = _custom(nt, L, D, np.zeros((2, 2, 2, 2)), np.zeros(nt, complex), 1.0, launch, sim)
    zs = [0.0, L / 3, L]
    out, _, _ = O.forward(fp, zsave=zs)
    for i, z in enumerate(zs):
        exp = np.exp(1j * D * z) * launch
        assert np.linalg.norm(out[i] - exp) / np.linalg.norm(exp) < 1e-12


def test_raman_response_formula():
    # test_numerical_kernels.jl:65-95
    fraction, t1, t2 = 0.18, 12.2e-3, 32.0e-3
    for nt in (64, 128, 256, 512):
        sim = P.get_disp_sim_params(1550e-9, 1, nt, 3.0, 2)
        r = P.single_oscillator_raman_fields(sim, fraction, 1e3 * t1, 1e3 * t2)
        om = 2 * np.pi * P.fftfreq(nt, 1 / sim["Δt"])
        amp = (t1 ** 2 + t2 ** 2) / (t1 * t2 ** 2)
        resp = fraction * amp * (1 / t1) / ((1 / t2 + 1j * om) ** 2 + (1 / t1) ** 2)
        cen = np.exp(-1j * om * sim["time_window"] / 2) * resp
        cen[nt // 2] = cen[nt // 2].real
        assert np.allclose(r["hRω"], cen, rtol=5e-14, atol=5e-14)
        assert abs(r["hRω"][0].real - fraction) < 5e-14 * fraction
        assert r["hRω"][nt // 2].imag == 0
        assert np.allclose(r["hRω"][1:nt // 2], np.conj(r["hRω"][nt // 2 + 1:][::-1]))
        assert P.real_response_spectrum(r["hRω"])
    bad = r["hRω"].copy()
    bad[1] += 0.1j
    assert not P.real_response_spectrum(bad)


def test_grid_validation_message():
    # test_numerical_kernels.jl:38-63
    with pytest.raises(P.ArgumentError, match="use at least 21.178 ps"):
        P.get_disp_sim_params(1550e-9, 1, 8192, 12.0, 2)
    for bad in ((-1550e-9, 1, 64, 3.0, 2), (1550e-9, 0, 64, 3.0, 2), (1550e-9, 1, 63, 3.0, 2),
                (1550e-9, 1, 2, 3.0, 2), (1550e-9, 1, 64, -3.0, 2), (1550e-9, 1, 64, 3.0, 1)):
        with pytest.raises(P.ArgumentError):
            P.get_disp_sim_params(*bad)


def test_published_counterfactual_centroid_shift():
    # counterfactual-raman-benchmark.md:43-52, :77: ΔC(neutral) = -0.717087 THz
    def prob(fR):
        return P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                                     fwhm_s=185e-15, rep_rate_hz=80.5e6, fR=fR)
    on, off = prob(0.18), prob(0.0)
    yon = O.forward(on)[0][-1]
    yoff = O.forward(off)[0][-1]
    dC = P.centroid_thz(yon, on.sim) - P.centroid_thz(yoff, off.sim)
    assert round(dC, 6) == -0.717087
    # within the published numerical envelope (:93, 5.95e-6 relative)
    assert abs(dC - (-0.717087)) / 0.717087 < 5.95e-6


def test_stokes_sign_and_photon_drift():
    # test_numerical_kernels.jl:204-221 (HNLF_zero_disp preset, 0.02 m, 0.05 W)
    fp = P.single_mode_problem(nt=256, time_window_ps=3.0, L=0.02, power_w=0.05,
                               gamma=10.0e-3, betas=(-0.1e-26, 3.0e-40), rep_rate_hz=80.5e6)
    out = O.forward(fp)[0]
    shift = P.centroid_thz(out[-1], fp.sim) - P.centroid_thz(out[0], fp.sim)
    assert shift < -1e-3
    n0, n1 = P.photon_number(out[0], fp.sim), P.photon_number(out[-1], fp.sim)
    assert abs(n1 / n0 - 1) < 1e-6


def test_rk4_crosscheck_against_tsit5():
    # test_scalar_crosscheck.jl:58-75: strict Tsit5 vs 128-step RK4
    base = P.single_mode_problem(nt=128, time_window_ps=4.0, L=0.02, power_w=0.02,
                                 rep_rate_hz=80.5e6)
    for fR in (0.18, 0.0):
        fp = P.single_mode_problem(nt=128, time_window_ps=4.0, L=0.02, power_w=0.02,
                                   rep_rate_hz=80.5e6, fR=fR, reltol=1e-11, abstol=1e-12)
        canon = O.forward(fp)[0][-1]
        ref = O.rk4_scalar(fp, 128)
        assert np.linalg.norm(ref - canon) / np.linalg.norm(canon) < 1e-7
    # linear RK4 is exact (:27-37)
    lin = P.single_mode_problem(nt=128, time_window_ps=4.0, L=0.02, power_w=0.02, gamma=0.0)
    out = O.rk4_scalar(lin, 4)
    assert np.allclose(out, np.exp(1j * lin.D * lin.L) * lin.uw0, rtol=2e-15, atol=2e-15)
    del base


def test_rk4_fourth_order_on_cw():
    # test_scalar_crosscheck.jl:39-56
    sim = P.get_disp_sim_params(1550e-9, 1, 64, 2.0, 2)
    raman = P.single_oscillator_raman_fields(sim, 0.0)
    launch = np.fft.ifft(np.full((1, 64), np.sqrt(5.0), complex), axis=1)
    fp = _custom(64, 2.0, P.dispersion_from_betas(sim, [0.0])[None, :], np.ones((1, 1, 1, 1)),
                 raman["hRω"], raman["one_m_fR"], launch, sim)
    exact = launch * np.exp(1j * 1.0 * 5.0 * 2.0)
    errs = [np.linalg.norm(O.rk4_scalar(fp, s) - exact) for s in (32, 64, 128)]
    assert np.log2(errs[0] / errs[1]) > 3.5
    assert np.log2(errs[1] / errs[2]) > 3.5
    assert errs[-1] / np.linalg.norm(exact) < 1e-4


def _weighted_gradient(fp, weights, phase):
    """Gradient of Σ w|u(L)|² w.r.t. the launch phase via the oracle adjoint."""
    us = fp.uw0 * np.exp(1j * phase)[None, :]
    out, _, dense = O.forward(fp, u0=us, keep_dense=True)
    lamL = weights * out[-1]
    lam0, _ = O.adjoint(fp, dense, lamL)
    return np.sum(2 * np.real(np.conj(lam0) * 1j * us), axis=0)


def test_adjoint_nyquist_seam():
    # test_numerical_kernels.jl:133-164
    nt = 64
    sim = P.get_disp_sim_params(1550e-9, 1, nt, 3.0, 2)
    t = sim["ts"] * 1e12
    temporal = (np.exp(-0.5 * (t / 0.07) ** 2) * np.exp(8j * (t / 0.07) ** 2))[None, :]
    launch = np.fft.ifft(temporal, axis=1)
    raman = P.single_oscillator_raman_fields(sim, 0.18)
    fp = _custom(nt, 0.05, P.dispersion_from_betas(sim, [0.0])[None, :],
                 np.full((1, 1, 1, 1), 2.0), raman["hRω"], raman["one_m_fR"], launch, sim)
    w = np.linspace(0.3, 1.7, nt)[None, :]
    phase = np.zeros(nt)
    g = _weighted_gradient(fp, w, phase)

    def cost(ph):
        y = O.forward(fp, u0=fp.uw0 * np.exp(1j * ph)[None, :])[0][-1]
        return float(np.sum(w * np.abs(y) ** 2))
    h = 1e-6
    rel = []
    for k in (1, nt // 2 - 1, nt // 2, nt - 1):
        e = np.zeros(nt)
        e[k] = h
        fd = (cost(phase + e) - cost(phase - e)) / (2 * h)
        assert abs(g[k] - fd) <= 1e-12 + 1e-4 * abs(fd)
        rel.append(abs(g[k] - fd) / abs(fd))
    assert max(rel) < 2e-5


def test_band_gradient_matches_central_differences():
    # band objective gradient vs central FD along random directions
    # (the reference's Taylor/FD checks, test/tier_slow.jl:36-53)
    fp = P.single_mode_problem(nt=256, time_window_ps=3.0, L=0.3, power_w=0.1,
                               rep_rate_hz=80.5e6, raman_threshold_thz=-4.0)
    rng = np.random.default_rng(0)
    phi = 0.3 * rng.standard_normal(fp.nt)
    J, g, _ = O.phase_gradient(fp, phi)

    def cost(ph):
        y = O.forward(fp, u0=fp.uw0 * np.exp(1j * ph)[None, :])[0][-1]
        return P.band_cost_and_seed(y, fp.mask)[0]
    assert abs(cost(phi) - J) < 1e-14
    for _ in range(4):
        d = rng.standard_normal(fp.nt)
        d /= np.linalg.norm(d)
        h = 1e-4
        fd = (cost(phi + h * d) - cost(phi - h * d)) / (2 * h)
        assert abs(fd - g @ d) <= 1e-3 * abs(fd)


def test_adjoint_rejects_nonsymmetric_gamma():
    # test_propagation.jl:178-192: forward accepts, adjoint rejects
    nt, modes = 32, 2
    sim = P.get_disp_sim_params(1550e-9, modes, nt, 5.0, 2)
    gam = np.zeros((2, 2, 2, 2))
    gam[0, 0, 0, 1] = 0.1
    launch = np.fft.ifft(np.ones((2, nt), complex), axis=1)
    fp = _custom(nt, 0.1, np.zeros((2, nt)), gam, np.zeros(nt, complex), 1.0, launch, sim)
    out, _, dense = O.forward(fp, keep_dense=True)
    assert np.all(np.isfinite(out))
    with pytest.raises(O.OracleError) as e:
        O.adjoint(fp, dense, np.ones((2, nt), complex))
    assert e.value.rc == 6
    assert not P.gamma_symmetric(gam)


def test_adjoint_scale_invariance():
    # test_numerical_kernels.jl:166-202: scaled seed gives the scaled gradient
    fp = P.single_mode_problem(nt=64, time_window_ps=3.0, L=0.3, power_w=0.1, rep_rate_hz=80.5e6)
    out, _, dense = O.forward(fp, keep_dense=True)
    seed = out[-1] * np.linspace(0.5, 1.5, fp.nt)[None, :]
    l1, _ = O.adjoint(fp, dense, seed)
    l2, _ = O.adjoint(fp, dense, -1e-4 * seed)
    assert np.allclose(l2, -1e-4 * l1, rtol=5e-4, atol=1e-12)
