"""GPU parity tests: the CUDA stepper through the C-ABI against the FP64
oracle (field ≤ 1e-5 relative L2 in FP32 mode, ≤ 1e-10 in FP64 mode; Raman
band fraction within 0.01 dB; gradients ≤ 1e-3 relative to the oracle
adjoint and to central differences)."""
import numpy as np
import pytest

from fiberlab_gpu import problem as P
from fiberlab_gpu._capi import Context, FiberLabGPUError, GPUProblem
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELD_TOL_FP32 = 1e-5
FIELD_TOL_FP64 = 1e-10
GRAD_TOL = 1e-3
DB_TOL = 0.01


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cfg0(nt=8192, T=10.0, **kw):
    return P.single_mode_problem(nt=nt, time_window_ps=T, L=0.5, power_w=0.1,
                                 rep_rate_hz=80e6, validate_grid=False, **kw)


@pytest.mark.parametrize("nt", [64, 256, 1024, 8192, 16384, 32768])
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_rhs_matches_oracle(gpu_ctx, nt, precision):
    # FP64 mode beyond 2^13 and both modes at 2^15 run on the multimode
    # runtime's kernels (2^15 through a 4-CTA cluster transform)
    fp = P.single_mode_problem(nt=nt, time_window_ps=10.0 if nt >= 1024 else 3.0, L=0.5,
                               power_w=0.1, rep_rate_hz=80.5e6, validate_grid=False)
    rng = np.random.default_rng(nt)
    u = fp.uw0 * np.exp(0.3j * rng.standard_normal(fp.nt))[None, :]
    lam = (rng.standard_normal(fp.nt) + 1j * rng.standard_normal(fp.nt))[None, :] * 1e-3
    gp = GPUProblem(gpu_ctx, fp, precision)
    z = 0.3217
    # forward RHS in the mode's precision; the adjoint RHS is FP64 in both modes
    tol = 2e-6 if precision == "fp32" else FIELD_TOL_FP64
    assert rel(gp.rhs(z, u), O.rhs_forward(fp, z, u)) < tol
    # The random λ fills every bin, and at the band edge the dispersion phase
    # D(ω)z reaches ~7e6 rad on the 2^15 / 10 ps grid: one FP64 rounding of
    # that argument is ~1e-9 rad, in the oracle as in the GPU.  Two FP64
    # evaluations agree to about that floor, 2 eps max|D z|.
    floor = 2 * np.finfo(float).eps * float(np.max(np.abs(fp.D))) * z
    assert rel(gp.rhs(z, lam, u), O.rhs_adjoint(fp, z, lam, u)) < max(FIELD_TOL_FP64, floor)


def test_forward_large_grids_against_tight_solution(gpu_ctx):
    # Nt = 2^14 and 2^15 over 10 ps.  At the default tolerances (reltol 1e-8,
    # abstol 1e-6) the RMS error norm is diluted over the mostly empty grid,
    # and the oracle's own answer is 2e-5 (2^14) and 5e-5 (2^15) from the
    # tight-tolerance solution; at 2^15 it moves by 1e-4 when reltol changes
    # by one part in 10^7.  So the GPU solves are held against the tight
    # solution (oracle, reltol = abstol = 1e-12), with bounds set by the
    # oracle's own default-tolerance error there: FP64 mode within 3x of it;
    # FP32 mode (whose FFT round-off floor enters the error norm in the empty
    # bins and adds steps) within 10x.
    for nt in (16384, 32768):
        fp = P.single_mode_problem(nt=nt, time_window_ps=10.0, L=0.3, power_w=0.1,
                                   rep_rate_hz=80.5e6, validate_grid=False)
        ref, _, _ = O.forward(fp)
        tight = P.FiberProblem(**{**fp.__dict__})
        tight.reltol = tight.abstol = 1e-12
        truth, _, _ = O.forward(tight)
        e_ref = rel(ref[-1], truth[-1])
        out64, _ = GPUProblem(gpu_ctx, fp, "fp64").forward() if nt == 32768 else (None, None)
        out32, st = GPUProblem(gpu_ctx, fp).forward()
        assert st["status"] == 0 and st["z_end"] == fp.L
        assert rel(out32[-1], truth[-1]) < max(10 * e_ref, FIELD_TOL_FP32)
        if out64 is not None:
            assert rel(out64[-1], truth[-1]) < 3 * e_ref


@pytest.mark.parametrize("nt,T", [(256, 3.0), (1024, 10.0), (2048, 10.0), (4096, 10.0)])
def test_forward_matches_oracle(gpu_ctx, nt, T):
    fp = P.single_mode_problem(nt=nt, time_window_ps=T, L=0.3, power_w=0.1,
                               rep_rate_hz=80.5e6, validate_grid=False)
    out, st = GPUProblem(gpu_ctx, fp).forward()
    ref, rst, _ = O.forward(fp)
    assert rel(out[-1], ref[-1]) < FIELD_TOL_FP32
    assert st["status"] == 0 and st["z_end"] == fp.L
    assert st["nf"] == 3 + 6 * (st["naccept"] + st["nreject"])


def test_forward_config0_shape(gpu_ctx):
    # Nt = 2^13 over 10 ps, SMF-28, 0.5 m, 0.1 W / 80 MHz, 185 fs sech²
    fp = cfg0()
    out, st = GPUProblem(gpu_ctx, fp).forward()
    ref, rst, _ = O.forward(fp)
    assert rel(out[-1], ref[-1]) < FIELD_TOL_FP32
    Jg = P.band_cost_and_seed(out[-1], fp.mask)[0]
    Jo = P.band_cost_and_seed(ref[-1], fp.mask)[0]
    assert abs(10 * np.log10(Jg) - 10 * np.log10(Jo)) < DB_TOL
    n0, n1 = P.photon_number(out[0], fp.sim), P.photon_number(out[-1], fp.sim)
    assert abs(n1 / n0 - 1) < 1e-5


def test_analytic_cw_kerr_gpu(gpu_ctx):
    nt, L, pw, g = 64, 5.0, 2.0, 0.73
    sim = P.get_disp_sim_params(1550e-9, 1, nt, 10.0, 2)
    launch = np.fft.ifft(np.full((1, nt), np.sqrt(pw), complex), axis=1)
    fp = P.FiberProblem(sim=sim, D=np.zeros((1, nt)), gamma=np.full((1, 1, 1, 1), g),
                        hR=np.zeros(nt, complex), one_m_fR=1.0, L=L, uw0=launch,
                        reltol=1e-10, abstol=1e-12)
    expected = launch * np.exp(1j * g * pw * L)
    out64, _ = GPUProblem(gpu_ctx, fp, "fp64").forward()
    assert rel(out64[-1], expected) < 1e-8
    # FP32 mode at the default tolerances (FP32 cannot meet abstol 1e-12)
    fp.reltol, fp.abstol = 1e-8, 1e-6
    out32, _ = GPUProblem(gpu_ctx, fp, "fp32").forward()
    assert rel(out32[-1], expected) < 1e-5


@pytest.mark.parametrize("nt,T", [(256, 3.0), (2048, 10.0)])
def test_fp64_mode_matches_oracle(gpu_ctx, nt, T):
    fp = P.single_mode_problem(nt=nt, time_window_ps=T, L=0.3, power_w=0.1,
                               rep_rate_hz=80.5e6, validate_grid=False)
    out, st = GPUProblem(gpu_ctx, fp, "fp64").forward()
    ref, rst, _ = O.forward(fp)
    assert rel(out[-1], ref[-1]) < FIELD_TOL_FP64
    assert st["naccept"] == rst["naccept"]


@pytest.mark.parametrize("nt", [16384, 32768])
def test_fp64_mode_large_grids(gpu_ctx, nt):
    # FP64 mode beyond one CTA's transform: the same steps as the oracle
    # (equal accepted count) and the field to FP64 round-off over 5 cm
    fp = P.single_mode_problem(nt=nt, time_window_ps=10.0, L=0.05, power_w=0.1,
                               rep_rate_hz=80.5e6, validate_grid=False)
    out, st = GPUProblem(gpu_ctx, fp, "fp64").forward()
    ref, rst, _ = O.forward(fp)
    assert st["status"] == 0 and st["z_end"] == fp.L
    assert st["naccept"] == rst["naccept"]
    assert rel(out[-1], ref[-1]) < 1e-9


def test_saveat_dense_output(gpu_ctx):
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                               rep_rate_hz=80.5e6)
    zs = [0.0, 0.1, 0.2345, 0.4, 0.5]
    out, _ = GPUProblem(gpu_ctx, fp).forward(saveat=zs)
    ref, _, _ = O.forward(fp, zsave=zs)
    for i in range(len(zs)):
        assert rel(out[i], ref[i]) < FIELD_TOL_FP32


def test_save_on_interior_step_end(gpu_ctx):
    # a save position exactly on the end of an accepted interior step is taken
    # from that step's dense output (not skipped): sol.t of a first forward
    # gives the step ends, the second forward with a save on one of them
    # takes the same steps and matches the oracle's dense output there and
    # the saves one ulp to either side
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                               rep_rate_hz=80.5e6)
    gp = GPUProblem(gpu_ctx, fp)
    gp.forward()
    t = gp.forward_times()
    assert t[0] == 0.0 and t[-1] == fp.L and np.all(np.diff(t) > 0)
    zk = float(t[len(t) // 2])
    zs = [0.0, np.nextafter(zk, 0.0), zk, np.nextafter(zk, 1.0), fp.L]
    out, st = gp.forward(saveat=zs)
    assert st["status"] == 0
    np.testing.assert_array_equal(gp.forward_times(), t)
    ref, _, _ = O.forward(fp, zsave=zs)
    for i in range(len(zs)):
        assert rel(out[i], ref[i]) < FIELD_TOL_FP32, (i, rel(out[i], ref[i]))
    assert rel(out[1], out[2]) < 1e-6 and rel(out[3], out[2]) < 1e-6


def test_seeded_adjoint_matches_oracle(gpu_ctx):
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                               rep_rate_hz=80.5e6)
    gp = GPUProblem(gpu_ctx, fp)
    out, _ = gp.forward()
    ref, _, dense = O.forward(fp, keep_dense=True)
    seed = ref[-1] * np.linspace(0.2, 1.8, fp.nt)[None, :]
    lam0, st = gp.adjoint(seed)
    lref, _ = O.adjoint(fp, dense, seed)
    assert rel(lam0, lref) < GRAD_TOL
    assert st["adj_naccept"] > 0
    # a second adjoint from the same forward checkpoints
    lam0b, _ = gp.adjoint(2.0 * seed)
    assert rel(lam0b, 2.0 * lref) < GRAD_TOL


@pytest.mark.parametrize("log_cost", [False, True])
def test_band_gradient_config1(gpu_ctx, log_cost):
    # config 1: Nt=2^13, φ ~ N(0, 0.5²) seed 0, Raman band < -13 THz, 32 checkpoints
    fp = cfg0()
    phi = 0.5 * np.random.default_rng(0).standard_normal(fp.nt)
    J, g, st = GPUProblem(gpu_ctx, fp).phase_gradient_batch(phi[None, :], log_cost=log_cost)
    Jo, go, _ = O.phase_gradient(fp, phi)
    if log_cost:
        assert abs(J[0] - 10 * np.log10(Jo)) < DB_TOL
        go = go * 10 / (np.log(10) * Jo)
    else:
        assert abs(10 * np.log10(J[0]) - 10 * np.log10(Jo)) < DB_TOL
    assert rel(g[0], go) < GRAD_TOL
    assert st[0]["checkpoints_used"] <= 32


def test_band_gradient_2p15(gpu_ctx):
    # Nt = 2^15 over 10 ps (the serving mix's largest grid) through the
    # cluster transform: forward, band objective, adjoint and gradient
    # (0.1 m; phase N(0, 0.5²) windowed to the pulse band: a white phase at
    # this grid spreads energy over ±1640 THz and the solves take thousands
    # of steps in the oracle)
    fp = P.single_mode_problem(nt=32768, time_window_ps=10.0, L=0.1, power_w=0.1,
                               rep_rate_hz=80e6, validate_grid=False, raman_threshold_thz=-5.0)
    f = P.fftfreq(fp.nt, 1 / fp.sim["Δt"])
    phi = 0.5 * np.random.default_rng(15).standard_normal(fp.nt) * np.exp(-(f / 4.0) ** 2)
    J, g, st = GPUProblem(gpu_ctx, fp).phase_gradient_batch(phi[None, :])
    Jo, go, _ = O.phase_gradient(fp, phi)
    assert abs(10 * np.log10(J[0]) - 10 * np.log10(Jo)) < DB_TOL
    assert rel(g[0], go) < GRAD_TOL
    assert st[0]["status"] == 0


def test_gradient_central_differences(gpu_ctx):
    # gradient vs central FD (h = 1e-4) along random unit directions, with the
    # FD costs from FP64 GPU forward solves
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                               rep_rate_hz=80.5e6, raman_threshold_thz=-5.0)
    rng = np.random.default_rng(3)
    phi = 0.5 * rng.standard_normal(fp.nt)
    J, g, _ = GPUProblem(gpu_ctx, fp).phase_gradient_batch(phi[None, :])
    gp64 = GPUProblem(gpu_ctx, fp, "fp64")

    def cost(ph):
        out, _ = gp64.forward(fp.uw0 * np.exp(1j * ph)[None, :])
        return P.band_cost_and_seed(out[-1], fp.mask)[0]
    for _ in range(8):
        d = rng.standard_normal(fp.nt)
        d /= np.linalg.norm(d)
        h = 1e-4
        fd = (cost(phi + h * d) - cost(phi - h * d)) / (2 * h)
        assert abs(fd - g[0] @ d) <= GRAD_TOL * abs(fd) + 1e-12


def test_gradient_central_differences_config1(gpu_ctx):
    # config 1 itself (Nt = 2^13 over 10 ps, 0.5 m, 0.1 W at 80 MHz, band
    # < -13 THz, phase N(0, 0.5²) seed 0): the FP32 product gradient against
    # central differences (h = 1e-4) along 8 random unit directions, with no
    # bias toward the gradient.  The 16 FD costs come from one batched
    # FP64-mode launch.
    fp = cfg0()
    rng = np.random.default_rng(0)
    phi = 0.5 * rng.standard_normal(fp.nt)
    J, g, _ = GPUProblem(gpu_ctx, fp).phase_gradient_batch(phi[None, :])
    drng = np.random.default_rng(8)
    d = drng.standard_normal((8, fp.nt))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    h = 1e-4
    probes = np.concatenate([phi + h * d, phi - h * d])
    Jp, _, _ = GPUProblem(gpu_ctx, fp, "fp64").phase_gradient_batch(probes)
    fd = (Jp[:8] - Jp[8:]) / (2 * h)
    ad = d @ g[0]
    err = np.abs(fd - ad) / np.abs(fd)
    assert np.all(err <= GRAD_TOL), (err, fd, ad)


def test_batch_results_equal_alone_and_in_mix(gpu_ctx):
    fp = P.single_mode_problem(nt=2048, time_window_ps=10.0, L=0.5, power_w=0.1,
                               rep_rate_hz=80.5e6)
    rng = np.random.default_rng(7)
    phis = 0.5 * rng.standard_normal((12, fp.nt))
    gp = GPUProblem(gpu_ctx, fp)
    Jb, gb, _ = gp.phase_gradient_batch(phis)
    for b in (0, 5, 11):
        Ja, ga, _ = GPUProblem(gpu_ctx, fp).phase_gradient_batch(phis[b:b + 1])
        assert Ja[0] == Jb[b]
        assert np.array_equal(ga[0], gb[b])


def test_status_codes_without_a_fault(gpu_ctx):
    # host-side injections, no GPU fault: non-Hermitian hR is rejected at
    # upload; a huge γ overflows the field -> FL_NONFINITE; a tiny iteration
    # cap -> FL_MAXITERS; a step log smaller than the solve -> FL_ECAPACITY
    fp = P.single_mode_problem(nt=256, time_window_ps=3.0, L=0.3, power_w=0.1,
                               rep_rate_hz=80.5e6)
    bad = P.FiberProblem(**{**fp.__dict__})
    bad.hR = fp.hR.copy()
    bad.hR[1] += 0.1j
    with pytest.raises(FiberLabGPUError) as e:
        GPUProblem(gpu_ctx, bad)
    assert e.value.status == 1
    huge = P.FiberProblem(**{**fp.__dict__})
    huge.gamma = np.full((1, 1, 1, 1), 1e30)
    with pytest.raises(FiberLabGPUError) as e:
        GPUProblem(gpu_ctx, huge).forward()
    assert e.value.status in (2, 3)
    with pytest.raises(FiberLabGPUError) as e:
        GPUProblem(Context(0, max_iters=3), fp).forward()
    assert e.value.status == 4
    long = P.single_mode_problem(nt=256, time_window_ps=3.0, L=3.0, power_w=0.3,
                                 rep_rate_hz=80.5e6)
    with pytest.raises(FiberLabGPUError) as e:
        GPUProblem(Context(0, step_log=4), long).phase_gradient_batch(np.zeros((1, long.nt)))
    assert e.value.status == 9
    # objective codes and the worst-mode smoothness are checked at the boundary
    from fiberlab_gpu._capi import load
    gp = GPUProblem(gpu_ctx, fp)
    for code, tau in ((7, 50.0), (-1, 50.0), (2, 0.0), (2, float("nan"))):
        with pytest.raises(FiberLabGPUError) as e:
            gp.ctx.check(load().fl_problem_set_objective(gp.h, code, tau))
        assert e.value.status == 1


@pytest.mark.parametrize("caps", [(2, 1), (4, 3), (4, 7)])
def test_adjoint_beyond_checkpoint_capacity(gpu_ctx, caps):
    # more accepted steps than checkpoints x segment_steps: each checkpoint
    # segment is replayed once per sub-segment of segment_steps steps (no
    # FL_ECAPACITY); the gradient matches the oracle and the default layout
    K, seg = caps
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                               rep_rate_hz=80.5e6, raman_threshold_thz=-5.0)
    phi = 0.5 * np.random.default_rng(31).standard_normal(fp.nt)
    J, g, st = GPUProblem(Context(0, checkpoints=K, segment_steps=seg), fp).phase_gradient_batch(
        phi[None, :])
    assert st[0]["status"] == 0 and st[0]["naccept"] > K * seg
    Jd, gd, _ = GPUProblem(gpu_ctx, fp).phase_gradient_batch(phi[None, :])
    Jo, go, _ = O.phase_gradient(fp, phi)
    assert J[0] == Jd[0]                      # the forward is the same solve
    assert rel(g[0], go) < GRAD_TOL and rel(g[0], gd[0]) < GRAD_TOL


def test_physical_gradient_phase_amplitude_energy(gpu_ctx):
    # spectral_shaper_model's physical gradient (physics_models.jl:1021-1081):
    # phase (vector), amplitude (vector) and energy controls of a 3-mode
    # problem against the same chain rule applied to the oracle's λ0
    from fiberlab_gpu import solve as S
    fp = P.multimode_problem(1, 32, 512, 5.0, 0.4, 5e-9, 200e-15, seed=2,
                             raman_threshold_thz=-5.0)
    rng = np.random.default_rng(21)
    control = {"phase": 0.3 * rng.standard_normal(fp.nt),
               "amplitude": 1.0 + 0.1 * rng.standard_normal(fp.nt) ** 2,
               "energy": 1.3}
    J, g = S.physical_gradient(fp, control, ctx=gpu_ctx)
    alpha = np.sqrt(control["energy"])
    ph = np.repeat(control["phase"][None, :], fp.M, axis=0)
    am = np.repeat(control["amplitude"][None, :], fp.M, axis=0)
    shaped = alpha * am * np.exp(1j * ph) * fp.uw0
    out, _, dense = O.forward(fp, u0=shaped, keep_dense=True)
    Jo, seed = P.band_cost_and_seed(out[-1], fp.mask)
    lam0, _ = O.adjoint(fp, dense, seed)
    gp = (2 * np.real(np.conj(lam0) * 1j * shaped)).sum(axis=0)
    ga = (2 * alpha * np.real(np.conj(lam0) * np.exp(1j * ph) * fp.uw0)).sum(axis=0)
    ge = np.real(np.sum(np.conj(lam0) * shaped)) / control["energy"]
    assert abs(10 * np.log10(J) - 10 * np.log10(Jo)) < DB_TOL
    assert rel(g["phase"], gp) < GRAD_TOL
    assert rel(g["amplitude"], ga) < GRAD_TOL
    assert abs(g["energy"][0] - ge) <= GRAD_TOL * abs(ge)
    with pytest.raises(P.ArgumentError):
        S.physical_gradient(fp, {"amplitude": -1.0}, ctx=gpu_ctx)


@pytest.mark.parametrize("objective", ["fundamental_mode", "worst_mode", "raman_peak",
                                       "temporal_width"])
def test_physical_gradient_objectives(gpu_ctx, objective):
    # the other field objectives of the reference registry
    # (physics_helpers.jl:234-318): GPU forward, host seed, GPU adjoint,
    # against the same seed through the oracle's forward and adjoint
    from fiberlab_gpu import objectives as Ob
    from fiberlab_gpu import solve as S
    fp = P.multimode_problem(1, 32, 512, 5.0, 0.4, 5e-9, 200e-15, seed=2,
                             raman_threshold_thz=-3.0)
    phi = 0.3 * np.random.default_rng(31).standard_normal(fp.nt)
    J, g = S.physical_gradient(fp, {"phase": phi}, ctx=gpu_ctx, objective=objective)
    shaped = np.exp(1j * phi)[None, :] * fp.uw0
    out, _, dense = O.forward(fp, u0=shaped, keep_dense=True)
    Jo, seed = Ob.cost_and_seed(objective, out[-1], fp.mask, fp.sim)
    lam0, _ = O.adjoint(fp, dense, seed)
    go = (2 * np.real(np.conj(lam0) * 1j * shaped)).sum(axis=0)
    assert abs(J - Jo) <= 1e-4 * abs(Jo)
    assert rel(g["phase"], go) < GRAD_TOL


def test_propagate_metrics_and_verify(gpu_ctx):
    # propagate(problem; saveat) on the GPU, then metrics/verify evidence
    # (propagation.jl:176-304) on the test_propagation.jl:19-111 shape; the
    # evidence matches the same reductions over the oracle's spectra
    from fiberlab_gpu import solve as S
    fp = P.single_mode_problem(nt=128, time_window_ps=3.0, L=1e-4, power_w=1e-5,
                               fwhm_s=250e-15, rep_rate_hz=50e6, pulse="gauss",
                               betas=(-2.17e-26,), beta_order=2)
    zs = [0.0, 0.5e-4, 1e-4]
    ref, _, _ = O.forward(fp, zsave=zs)
    for precision, drift in (("fp64", 1e-8), ("fp32", 1e-5)):
        res = S.propagate(fp, zs, precision=precision, ctx=gpu_ctx)
        ev = S.metrics(res)
        assert ev["max_photon_number_drift"] < drift
        assert ev["input_energy_pj"] == pytest.approx(0.2, rel=1e-5)
        for i in range(len(zs)):
            m, mo = S.field_metrics(res.spectra[i], fp.sim), S.field_metrics(ref[i], fp.sim)
            assert m["energy_pj"] == pytest.approx(mo["energy_pj"], rel=1e-6)
            assert m["peak_power_w"] == pytest.approx(mo["peak_power_w"], rel=1e-5)
        v = S.verify(res)
        assert v["pass"] and v["integrity_ok"] and v["launch_sampling_ok"]
        assert not S.verify(res, min_launch_samples_per_fwhm=16)["pass"]


@pytest.mark.parametrize("shape", ["sm1024", "sm16384", "sm32768", "mm3x512"])
def test_device_evidence_matches_host_reductions(gpu_ctx, shape):
    # fl_forward_evidence: the FP64 reductions behind metrics/verify run on
    # the device over the saved spectra (one CTA per save position, a 4-CTA
    # cluster at 2^15); the host restatement of propagation.jl:176-202 over
    # the same spectra is the check
    from fiberlab_gpu import solve as S
    if shape.startswith("sm"):
        nt = int(shape[2:])
        fp = P.single_mode_problem(nt=nt, time_window_ps=10.0, L=0.2, power_w=0.1,
                                   rep_rate_hz=80e6, validate_grid=False)
    else:
        fp = P.multimode_problem(1, 32, 512, 5.0, 0.3, 4e-9, 200e-15, seed=1,
                                 raman_threshold_thz=-5.0)
    zs = [0.0, 0.37 * fp.L, fp.L]
    res = S.propagate(fp, zs, ctx=gpu_ctx)
    assert res.device_evidence.shape == (3, 6 + fp.M)
    for i in range(3):
        dev = S.device_field_metrics(res.device_evidence[i], fp.sim)
        host = S.field_metrics(res.spectra[i], fp.sim)
        for key in ("energy_pj", "peak_power_w", "photon_number"):
            assert dev[key] == pytest.approx(host[key], rel=1e-12), key
        np.testing.assert_allclose(dev["mode_energy_pj"], host["mode_energy_pj"], rtol=1e-12)
        for key in ("temporal_edge_fraction", "spectral_edge_fraction"):
            assert dev[key] == pytest.approx(host[key], rel=1e-9, abs=1e-18), key
    # metrics from the device sums and from the host reductions agree
    host_res = S.PropagationResult(**{**res.__dict__, "device_evidence": None})
    a, b = S.metrics(res), S.metrics(host_res)
    for key in ("max_photon_number_drift", "max_temporal_edge_fraction", "output_energy_pj"):
        assert a[key] == pytest.approx(b[key], rel=1e-9, abs=1e-12), key


def test_dense_forward_adjoint_needs_no_recompute(gpu_ctx):
    # a solve of at most segment_steps accepted steps keeps every step's
    # interpolant during the forward: its adjoint recomputes nothing and
    # integrates 0 <- L without checkpoint stops; a small segment buffer
    # forces the checkpoint recompute; both match the oracle
    fp = cfg0(raman_threshold_thz=-13.0)
    phi = 0.5 * np.random.default_rng(0).standard_normal(fp.nt)
    Jd, gd, sd = GPUProblem(Context(0, segment_steps=64), fp).phase_gradient_batch(phi[None, :])
    Jr, gr, sr = GPUProblem(Context(0, segment_steps=4), fp).phase_gradient_batch(phi[None, :])
    assert sd[0]["recompute_steps"] == 0 and sd[0]["naccept"] <= 64
    assert sr[0]["recompute_steps"] >= sr[0]["naccept"]
    assert Jd[0] == Jr[0]                     # the same forward solve
    Jo, go, _ = O.phase_gradient(fp, phi)
    assert rel(gd[0], go) < GRAD_TOL and rel(gr[0], go) < GRAD_TOL


def test_lbfgs_batched_inverse_design(gpu_ctx):
    # optimize_spectral_phase (raman_optimization.jl:183-246) for two starts
    # in lockstep: every line search is one batched forward + adjoint launch
    # over 2 x 4 trial phases; the dB objective with the GDD regulariser
    import torch
    from fiberlab_gpu import optimize as OP
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                               rep_rate_hz=80.5e6, raman_threshold_thz=-5.0)
    gp = GPUProblem(gpu_ctx, fp)
    obj = OP.BandPhaseObjective(gp, log_cost=True, lambda_gdd=1e-4)
    x0 = 0.5 * np.random.default_rng(4).standard_normal((2, fp.nt))
    J0, g0 = obj(torch.from_numpy(x0).to(obj.device))
    Jb, gb, _ = gp.phase_gradient_batch(x0)
    Jr, gr = OP.gdd_penalty(torch.from_numpy(x0), fp.sim["Δt"], 1e-4)
    Jl = torch.from_numpy(Jb) + Jr
    assert np.allclose(J0.cpu().numpy(), 10 * np.log10(Jl.numpy()), rtol=0, atol=1e-9)
    ref_g = (torch.from_numpy(gb) + gr) * (10 / (np.log(10) * Jl))[:, None]
    assert rel(g0.cpu().numpy(), ref_g.numpy()) < 1e-12
    res = OP.optimize_spectral_phase(gp, x0, max_iter=6, lambda_gdd=1e-4, probes=4)
    tr = torch.stack([J0.cpu()] + [t.cpu() for t in res.trace])
    assert torch.all(tr[1:] <= tr[:-1] + 1e-12)
    assert torch.all(res.J.cpu() < J0.cpu() - 0.1)
    assert res.iterations.min() >= 1 and res.solves >= 2 * 4 * res.iterations.max()


@pytest.mark.parametrize("objective", ["fundamental_mode", "worst_mode", "raman_peak"])
def test_device_objective_seeds_single_mode(gpu_ctx, objective):
    # fl_problem_set_objective: the batched call computes J and the seed on
    # the device; against the oracle's forward and adjoint with the host seed
    from fiberlab_gpu import objectives as Ob
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                               rep_rate_hz=80.5e6, raman_threshold_thz=-5.0)
    phi = 0.5 * np.random.default_rng(8).standard_normal(fp.nt)
    gp = GPUProblem(gpu_ctx, fp)
    Jband, _, _ = gp.phase_gradient_batch(phi[None, :])
    gp.set_objective(objective)
    J, g, _ = gp.phase_gradient_batch(phi[None, :])
    shaped = fp.uw0 * np.exp(1j * phi)[None, :]
    out, _, dense = O.forward(fp, u0=shaped, keep_dense=True)
    Jo, seed = Ob.cost_and_seed(objective, out[-1], fp.mask, fp.sim)
    lam0, _ = O.adjoint(fp, dense, seed)
    go = (2 * np.real(np.conj(lam0) * 1j * shaped)).sum(axis=0)
    assert abs(J[0] - Jo) <= 1e-4 * abs(Jo)
    assert rel(g[0], go) < GRAD_TOL
    if objective != "raman_peak":   # one mode: the band objective itself
        assert J[0] == Jband[0]
    gp.set_objective("raman_band")
    assert gp.phase_gradient_batch(phi[None, :])[0][0] == Jband[0]
    with pytest.raises(ValueError):
        gp.set_objective("temporal_width")


def test_boundary_rejects_bad_input(gpu_ctx):
    # the C-ABI's input checks (the reference's ArgumentError cases,
    # propagation.jl:41-70, physics_helpers.jl:222-232): each call fails with
    # a status and a message, launches nothing, and the context stays usable
    fp = P.single_mode_problem(nt=256, time_window_ps=3.0, L=0.3, power_w=0.1,
                               rep_rate_hz=80.5e6)
    gp = GPUProblem(gpu_ctx, fp)

    def status(fn):
        with pytest.raises(FiberLabGPUError) as e:
            fn()
        return e.value.status
    # shapes that are not built: Nt beyond 2^15 or below 2^6, more than 10 modes
    for nt in (65536, 32):
        big = P.single_mode_problem(nt=nt, time_window_ps=10.0 if nt > 256 else 3.0, L=0.1,
                                    power_w=0.1, rep_rate_hz=80.5e6, validate_grid=False)
        assert status(lambda: GPUProblem(gpu_ctx, big)) == 10
    M = 11
    many = P.FiberProblem(sim=dict(fp.sim, M=M), D=np.zeros((M, fp.nt)),
                          gamma=np.full((M, M, M, M), 1e-3), hR=fp.hR, one_m_fR=fp.one_m_fR,
                          L=fp.L, uw0=np.repeat(fp.uw0, M, axis=0) / np.sqrt(M))
    assert status(lambda: GPUProblem(gpu_ctx, many)) == 10
    # an adjoint needs a preceding forward
    assert status(lambda: gp.adjoint(fp.uw0)) == 1
    # save positions: sorted, unique, from 0 to L
    for zs in ([0.0, 0.2, 0.1, fp.L], [0.0, 0.1, 0.1, fp.L], [0.0, 0.1], [0.05, fp.L],
               [0.0, float("nan"), fp.L]):
        assert status(lambda: gp.forward(saveat=zs)) == 1
    # launch spectra: finite and nonzero
    bad = fp.uw0.copy()
    bad[0, 3] = np.nan
    assert status(lambda: gp.forward(bad)) == 1
    assert status(lambda: gp.forward(np.zeros_like(fp.uw0))) == 1
    # band objective: a nonempty mask and finite phases
    phi = np.zeros((2, fp.nt))
    assert status(lambda: gp.phase_gradient_batch(phi, np.zeros(fp.nt, bool))) == 1
    phi[1, 7] = np.inf
    assert status(lambda: gp.phase_gradient_batch(phi)) == 1
    # the context is still usable
    out, st = gp.forward()
    assert st["status"] == 0 and np.all(np.isfinite(out))


def test_nonfinite_phase_in_a_large_batch(gpu_ctx):
    # a batch of at least 2^20 phase values is scanned on a host thread while
    # the GPU runs it; a non-finite phase still fails the call with FL_EINVAL
    fp = P.single_mode_problem(nt=2048, time_window_ps=10.0, L=0.1, power_w=0.1,
                               rep_rate_hz=80.5e6)
    gp = GPUProblem(gpu_ctx, fp)
    phi = np.zeros((512, fp.nt))  # 2^20 values
    phi[397, 1000] = np.nan
    with pytest.raises(FiberLabGPUError) as e:
        gp.phase_gradient_batch(phi)
    assert e.value.status == 1
    phi[397, 1000] = 0.0
    J, g, st = gp.phase_gradient_batch(phi)
    assert all(s["status"] == 0 for s in st) and np.all(np.isfinite(g))


def test_reference_dict_interface(gpu_ctx):
    # solve_disp_mmf(uω0, fiber, sim) / solve_adjoint_disp_mmf(λωL, sol, fiber,
    # sim) as the reference's callers use them (propagation.jl:35-53,
    # physics_models.jl:1035-1041): sol(z) at stored positions, "uω_z" and
    # "ut_z" at fiber["zsave"], destats, and sol_adj(0) = λ(0)
    from fiberlab_gpu import solve as S
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                               rep_rate_hz=80.5e6)
    zs = [0.1, 0.25]
    fiber = {"Dω": fp.D, "γ": fp.gamma, "hRω": fp.hR, "one_m_fR": fp.one_m_fR, "L": fp.L,
             "zsave": zs}
    res = S.solve_disp_mmf(fp.uw0, fiber, fp.sim, ctx=gpu_ctx)
    sol = res["ode_sol"]
    assert sol.retcode == "Success" and sol.destats.naccept > 0
    assert sol.destats.nf == 3 + 6 * (sol.destats.naccept + sol.destats.nreject)
    ref, _, dense = O.forward(fp, zsave=[0.0] + zs + [fp.L], keep_dense=True)
    for i in range(len(zs)):
        assert rel(res["uω_z"][i], ref[1 + i]) < FIELD_TOL_FP32
    assert np.allclose(res["ut_z"], np.fft.fft(res["uω_z"], axis=-1), rtol=0, atol=0)
    uL = np.exp(1j * fp.D * fp.L) * sol(fp.L)   # lab frame from the interaction frame
    assert rel(uL, ref[-1]) < FIELD_TOL_FP32
    with pytest.raises(P.ArgumentError):
        sol(0.3)
    _, seed = P.band_cost_and_seed(uL, fp.mask)
    sol_adj = S.solve_adjoint_disp_mmf(seed, sol, fiber, fp.sim)
    lref, _ = O.adjoint(fp, dense, seed)
    assert rel(sol_adj(0.0), lref) < GRAD_TOL
    assert sol_adj.destats.naccept > 0


def _synthetic_yb_sections():
    # smooth Yb-like shapes: a 976 nm absorption peak, emission red of it
    wl = np.linspace(900e-9, 1150e-9, 60)
    sa = 2.5e-24 * np.exp(-((wl - 976e-9) / 8e-9) ** 2) + 6e-26 * np.exp(-((wl - 1030e-9) / 20e-9) ** 2)
    se = 2.5e-24 * np.exp(-((wl - 976e-9) / 8e-9) ** 2) + 6e-25 * np.exp(-((wl - 1030e-9) / 25e-9) ** 2)
    return (wl, sa), (wl, se)


@pytest.mark.parametrize("model", ["constant", "ydfa"])
def test_gain_propagation_matches_oracle(gpu_ctx, model):
    # fl_forward_gain (solve_disp_gain_smf, simulate_disp_gain_mmf.jl:204-239):
    # the state [P_pump; ũ] with the constant or the rate-equation gain
    # against the oracle's restatement
    from fiberlab_gpu import gain as G
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.05,
                               rep_rate_hz=80e6, wavelength_m=1030e-9)
    gain = 0.8 if model == "constant" else G.ydfa_params(fp.sim, *_synthetic_yb_sections())
    zs = [0.0, 0.1, 0.25, fp.L]
    out, pumps, st = GPUProblem(gpu_ctx, fp).forward_gain(gain, 0.05, saveat=zs)
    ref, pumps_ref, rst = O.forward_gain(fp, gain, 0.05, zsave=zs)
    assert st["status"] == 0 and st["z_end"] == fp.L
    for i in range(len(zs)):
        assert rel(out[i], ref[i]) < FIELD_TOL_FP32
        assert pumps[i] == pytest.approx(pumps_ref[i], rel=1e-6)
    assert st["nf"] == 3 + 6 * (st["naccept"] + st["nreject"])
    assert abs(st["naccept"] - rst["naccept"]) <= 2


def test_gain_reference_shape_and_limits(gpu_ctx):
    # test_numerical_kernels.jl:5-25 at the smallest built grid (2^6): 1030 nm,
    # 300 fs Gaussian 1e-4 W at 80 MHz, no nonlinearity or dispersion, 1e-5 m,
    # 0.05 W pump, reltol 1e-5: succeeds with a finite field
    from fiberlab_gpu import gain as G
    fp = P.single_mode_problem(nt=64, time_window_ps=5.0, L=1e-5, power_w=1e-4, fwhm_s=300e-15,
                               rep_rate_hz=80e6, gamma=0.0, betas=(0.0,), beta_order=2, fR=0.0,
                               wavelength_m=1030e-9, pulse="gauss", reltol=1e-5)
    gain = G.ydfa_params(fp.sim, *_synthetic_yb_sections())
    gp = GPUProblem(gpu_ctx, fp)
    out, pumps, st = gp.forward_gain(gain, 0.05)
    ref, pumps_ref, _ = O.forward_gain(fp, gain, 0.05)
    assert st["status"] == 0 and np.all(np.isfinite(out)) and np.all(np.isfinite(pumps))
    assert rel(out[-1], ref[-1]) < FIELD_TOL_FP32
    with pytest.raises(FiberLabGPUError) as e:
        gp.forward_gain(gain, 0.05, saveat=[0.0, 0.5e-5])      # must end at L
    assert e.value.status == 1
    # built for M = 1, FP32 mode, Nt <= 2^13
    with pytest.raises(FiberLabGPUError) as e:
        GPUProblem(gpu_ctx, fp, "fp64").forward_gain(0.5, 0.05)
    assert e.value.status == 10
