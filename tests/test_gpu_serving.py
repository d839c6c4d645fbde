"""GPU tests of the continuous-batching server (fl_server_*).

Each request runs the same stepper as the one-problem-per-call path alone in
its slot, so a request's result must not depend on what else is in flight:
the same request alone and inside a mixed stream give bit-identical outputs,
and both agree with the plain fl_forward / fl_phase_gradient_batch path
(forward fields bit-identical; gradients within the 1e-3 gradient tolerance,
since the server keeps more z-checkpoints and so splits the adjoint at other
positions).  Admission follows the HBM budget; waits time out without fault.
"""
import numpy as np
import pytest

from fiberlab_gpu import problem as P
from fiberlab_gpu._capi import FiberLabGPUError, GPUProblem
from fiberlab_gpu.serving import Server

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-3


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _mix(gpu_ctx, n, seed, L_range=(0.05, 0.4), p_range=(0.02, 0.15)):
    reqs = P.serving_mix(n, seed=seed, log2_nt=(11, 15), L_range=L_range, p_range=p_range)
    probs = {}
    for r in reqs:
        if r.nt not in probs:
            fp = P.serving_grid_problem(r.nt)
            probs[r.nt] = (fp, GPUProblem(gpu_ctx, fp))
    return reqs, probs


def _submit(srv, r, probs):
    fp, gp = probs[r.nt]
    u0 = P.serving_launch(fp, r.power_w)
    if r.kind == 0:
        return srv.submit_forward(gp, u0=u0, L=r.L)
    return srv.submit_band_gradient(gp, r.phase, u0=u0, L=r.L)


def test_serving_alone_equals_in_mix(gpu_ctx):
    reqs, probs = _mix(gpu_ctx, 24, seed=5)
    srv = Server(gpu_ctx)
    handles = [_submit(srv, r, probs) for r in reqs]
    for h in handles:
        srv.wait(h)
    info = srv.info()
    assert info["completed"] == len(reqs) and info["in_flight"] == 0
    srv.close()
    for i in (0, 3, 7, 11, 19, 23):
        alone = Server(gpu_ctx)
        a = alone.wait(_submit(alone, reqs[i], probs))
        alone.close()
        h = handles[i]
        if reqs[i].kind == 0:
            assert np.array_equal(a.out_field, h.out_field)
        else:
            assert a.J == h.J and np.array_equal(a.out_grad, h.out_grad)
        assert a.stats["naccept"] == h.stats["naccept"]


def test_serving_matches_plain_path(gpu_ctx):
    reqs, probs = _mix(gpu_ctx, 8, seed=9)
    srv = Server(gpu_ctx)
    handles = [_submit(srv, r, probs) for r in reqs]
    for r, h in zip(reqs, handles):
        srv.wait(h)
        fp0, _ = probs[r.nt]
        fp = P.FiberProblem(**{**fp0.__dict__})
        fp.L = r.L
        u0 = P.serving_launch(fp0, r.power_w)
        gp = GPUProblem(gpu_ctx, fp)
        if r.kind == 0:
            out, st = gp.forward(u0)
            assert np.array_equal(out[-1], h.out_field)
        else:
            J, g, _ = gp.phase_gradient_batch(r.phase[None, :], u0=u0)
            assert abs(J[0] - h.J) <= 1e-9 * abs(J[0])
            assert rel(h.out_grad, g[0]) < GRAD_TOL
        assert h.latency_ms > 0
    srv.close()


def test_serving_admission_by_hbm_budget(gpu_ctx):
    fp = P.serving_grid_problem(4096)
    gp = GPUProblem(gpu_ctx, fp)
    tiny = Server(gpu_ctx, hbm_budget_bytes=1 << 20)
    with pytest.raises(FiberLabGPUError) as e:
        tiny.submit_forward(gp, L=0.1)
    assert e.value.status == 11  # FL_OOM_ADMISSION
    tiny.close()
    # room for a few slots: every request still completes, through slot reuse
    small = Server(gpu_ctx, hbm_budget_bytes=3 * 40 << 20)
    hs = [small.submit_forward(gp, u0=P.serving_launch(fp, 0.05 + 0.01 * k), L=0.1)
          for k in range(10)]
    for h in hs:
        small.wait(h)
    info = small.info()
    assert info["completed"] == 10 and info["hbm_bytes"] <= 3 * 40 << 20
    assert 1 <= info["slots"] < 10
    small.close()


def test_serving_wait_timeout_then_result(gpu_ctx):
    fp = P.serving_grid_problem(8192)
    gp = GPUProblem(gpu_ctx, fp)
    srv = Server(gpu_ctx)
    h = srv.submit_band_gradient(gp, 0.5 * np.random.default_rng(1).standard_normal(fp.nt),
                                 u0=P.serving_launch(fp, 0.3), L=2.0)
    with pytest.raises(TimeoutError):
        srv.wait(h, timeout_ms=0.0)
    srv.wait(h)
    assert h.status == 0 and h.stats["adj_naccept"] > 0
    srv.close()


def test_serving_multimode_requests(gpu_ctx):
    # a 3-mode forward and band gradient beside a single-mode forward in one
    # server: the multimode requests run on the mode-parallel kernels in
    # their own bucket, with the same answers as the plain entry points
    fp = P.multimode_problem(1, 32, 512, 5.0, 0.3, 4e-9, 200e-15, seed=4,
                             raman_threshold_thz=-5.0)
    gp = GPUProblem(gpu_ctx, fp)
    sm = P.serving_grid_problem(2048)
    gsm = GPUProblem(gpu_ctx, sm)
    phi = 0.4 * np.random.default_rng(2).standard_normal(fp.nt)
    srv = Server(gpu_ctx)
    hf = srv.submit_forward(gp, L=0.2)
    hg = srv.submit_band_gradient(gp, phi, L=0.2)
    hs = srv.submit_forward(gsm, u0=P.serving_launch(sm, 0.1), L=0.3)
    for h in (hf, hg, hs):
        srv.wait(h)
        assert h.status == 0
    short = P.FiberProblem(**{**fp.__dict__})
    short.L = 0.2
    gshort = GPUProblem(gpu_ctx, short)
    out, _ = gshort.forward()
    assert np.array_equal(out[-1], hf.out_field)
    J, g, _ = gshort.phase_gradient_batch(phi[None, :])
    assert abs(J[0] - hg.J) <= 1e-9 * abs(J[0])
    assert rel(hg.out_grad, g[0]) < GRAD_TOL
    smL = P.FiberProblem(**{**sm.__dict__})
    smL.L = 0.3
    out_sm, _ = GPUProblem(gpu_ctx, smL).forward(P.serving_launch(sm, 0.1))
    assert np.array_equal(out_sm[-1], hs.out_field)
    srv.close()


def test_serving_request_keeps_objective_of_submission(gpu_ctx):
    # a band-gradient request computes the objective its problem had when it
    # was submitted (fl_problem_set_objective), on the device, as the plain
    # batched call does
    fp = P.serving_grid_problem(2048)
    gp = GPUProblem(gpu_ctx, fp)
    phi = 0.4 * np.random.default_rng(6).standard_normal(fp.nt)
    u0 = P.serving_launch(fp, 0.2)
    short = P.FiberProblem(**{**fp.__dict__})
    short.L = 0.3
    ref = GPUProblem(gpu_ctx, short)
    ref.set_objective("raman_peak")
    Jp, gpk, _ = ref.phase_gradient_batch(phi[None, :], u0=u0)
    srv = Server(gpu_ctx)
    gp.set_objective("raman_peak")
    h = srv.submit_band_gradient(gp, phi, u0=u0, L=0.3)
    gp.set_objective("raman_band")      # later changes do not reach the request
    srv.wait(h)
    assert h.status == 0
    assert abs(h.J - Jp[0]) <= 1e-9 * abs(Jp[0])
    assert rel(h.out_grad, gpk[0]) < GRAD_TOL
    srv.close()
