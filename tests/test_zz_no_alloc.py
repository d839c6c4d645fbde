"""The allocation-free forward entry point, checked against fl_forward.

fl_forward_noalloc is for callers that cannot call cudaMalloc (a host runtime
whose device memory belongs to its own pool allocator, or a request loop that
must not take cudaMalloc's device synchronisation): it runs on device buffers
the caller owns and keeps its own state in a fixed 2 MiB device array (its
only limit is Nt <= 2^13: being forward-only it keeps no step log).  This
file is collected last so that a failure here comes after every other test.
"""
import numpy as np
import pytest

from fiberlab_gpu import problem as P
from fiberlab_gpu._capi import Context, GPUProblem, forward_noalloc

pytestmark = pytest.mark.gpu

FIELD_TOL_FP32 = 1e-5


def _device_inputs(torch, fp, zs):
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    bufs = dict(D=t(fp.D[0].astype(np.float64)),
                hR=t(np.ascontiguousarray(fp.hR).view(np.float64)),
                ss=t(fp.selfsteep.astype(np.float64)),
                u0=t(np.ascontiguousarray(fp.uw0[0]).view(np.float64)),
                zs=t(np.asarray(zs, dtype=np.float64)))
    bufs["out"] = torch.empty(2 * fp.nt * len(zs), dtype=torch.float64, device=dev)
    return bufs


def _run(b, fp, zs):
    return forward_noalloc(0, fp.nt, b["D"].data_ptr(), float(fp.gamma[0, 0, 0, 0]),
                           b["hR"].data_ptr(), b["ss"].data_ptr(), float(fp.one_m_fR),
                           float(fp.L), float(fp.reltol), float(fp.abstol), b["u0"].data_ptr(),
                           b["zs"].data_ptr(), len(zs), b["out"].data_ptr())


def test_forward_noalloc_matches_forward(gpu_ctx):
    torch = pytest.importorskip("torch")
    cases = [
        (P.single_mode_problem(nt=8192, time_window_ps=10.0, L=0.5, power_w=0.1, rep_rate_hz=80e6,
                               validate_grid=False), [0.0, 0.2, 0.5]),
        (P.single_mode_problem(nt=2048, time_window_ps=10.0, L=0.3, power_w=0.05,
                               rep_rate_hz=80.5e6), [0.0, 0.3]),
    ]
    # two calls in a row on the shared scratch array, each against fl_forward
    for fp, zs in cases:
        ref, rst = GPUProblem(gpu_ctx, fp).forward(saveat=zs)
        b = _device_inputs(torch, fp, zs)
        rc, st = _run(b, fp, zs)
        assert rc == 0, rc
        out = b["out"].cpu().numpy().view(np.complex128).reshape(len(zs), 1, fp.nt)
        for i in range(len(zs)):
            err = np.linalg.norm(out[i] - ref[i]) / np.linalg.norm(ref[i])
            assert err < FIELD_TOL_FP32, (fp.nt, zs[i], err)
        assert st["z_end"] == fp.L and st["naccept"] > 0


def test_forward_noalloc_long_solve_has_no_step_limit():
    # a forward-only solve keeps no step log: 1 W (5.9 kW peak) over 3 m of
    # SMF-28 on 2^11 points takes about 10^4 accepted steps, more than a
    # fixed step log of 8192 entries would hold, and still matches fl_forward
    # (run here with a step log large enough for its adjoint checkpoints)
    torch = pytest.importorskip("torch")
    fp = P.single_mode_problem(nt=2048, time_window_ps=10.0, L=3.0, power_w=1.0, rep_rate_hz=80e6,
                               validate_grid=False)
    zs = [0.0, 1.5, 3.0]
    ref, rst = GPUProblem(Context(0, step_log=1 << 16), fp).forward(saveat=zs)
    b = _device_inputs(torch, fp, zs)
    rc, st = _run(b, fp, zs)
    assert rc == 0, rc
    assert st["naccept"] > 8192 and rst["naccept"] > 8192, (st, rst)
    out = b["out"].cpu().numpy().view(np.complex128).reshape(len(zs), 1, fp.nt)
    for i in range(len(zs)):
        err = np.linalg.norm(out[i] - ref[i]) / np.linalg.norm(ref[i])
        assert err < FIELD_TOL_FP32, (zs[i], err)


def test_forward_noalloc_rejects_oversize_and_bad_input(gpu_ctx):
    torch = pytest.importorskip("torch")
    big = P.single_mode_problem(nt=16384, time_window_ps=10.0, L=0.1, power_w=0.05,
                                rep_rate_hz=80.5e6, validate_grid=False)
    b = _device_inputs(torch, big, [0.0, big.L])
    rc, _ = _run(b, big, [0.0, big.L])
    assert rc == 10  # FL_EUNSUPPORTED: beyond the 2^13 scratch limit, checked on the host
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.3, power_w=0.05,
                               rep_rate_hz=80.5e6)
    b = _device_inputs(torch, fp, [0.0, 0.1])  # does not end at L
    rc, _ = _run(b, fp, [0.0, 0.1])
    assert rc == 1  # FL_EINVAL
