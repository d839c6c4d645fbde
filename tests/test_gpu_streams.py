"""Caller-supplied CUDA streams (fl_ctx_set_stream).

The drop-in boundary runs on the caller's stream: work the caller queued on
that stream before a call is ordered before it, and two contexts on two
streams (one per host thread, the reference's concurrency rule: one solve
with its own state per thread, agent-docs/current-agent-context/NUMERICS.md:35-37)
give the same results as one context on its private stream.
"""
import threading

import numpy as np
import pytest

from fiberlab_gpu import problem as P
from fiberlab_gpu._capi import Context, GPUProblem

pytestmark = pytest.mark.gpu


def _problem():
    return P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                                 rep_rate_hz=80.5e6, raman_threshold_thz=-5.0)


def test_device_call_is_ordered_on_the_caller_stream():
    torch = pytest.importorskip("torch")
    fp = _problem()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(21)
    old, new = 0.5 * rng.standard_normal((2, 4, fp.nt))
    ctx = Context(0)
    gp = GPUProblem(ctx, fp)
    J_ref, g_ref, _ = gp.phase_gradient_batch(new)   # private stream, host buffers
    d_u0 = torch.from_numpy(np.ascontiguousarray(fp.uw0).view(np.float64).copy()).to(dev)
    d_m = torch.from_numpy(fp.mask.astype(np.uint8)).to(dev)
    d_ph = torch.from_numpy(old).to(dev)
    src = torch.from_numpy(new).pin_memory()
    d_J = torch.empty(4, dtype=torch.float64, device=dev)
    d_g = torch.empty((4, fp.nt), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    s = torch.cuda.Stream(device=dev)
    ctx.set_stream(s)
    assert ctx.stream == s.cuda_stream
    with torch.cuda.stream(s):
        torch.cuda._sleep(20_000_000)          # keep the stream busy ...
        d_ph.copy_(src, non_blocking=True)     # ... then overwrite the phases on it
    # no host synchronisation: the call must see the new phases
    gp.phase_gradient_batch_device(d_u0.data_ptr(), 4, d_ph.data_ptr(), d_m.data_ptr(),
                                   d_J.data_ptr(), d_g.data_ptr())
    np.testing.assert_array_equal(d_J.cpu().numpy(), J_ref)
    np.testing.assert_array_equal(d_g.cpu().numpy(), g_ref)
    ctx.set_stream(None)
    assert ctx.stream != s.cuda_stream


def test_two_contexts_on_two_caller_streams_match_private_stream():
    torch = pytest.importorskip("torch")
    fp = _problem()
    rng = np.random.default_rng(22)
    phs = [0.5 * rng.standard_normal((3, fp.nt)) for _ in range(2)]
    base = Context(0)
    ref = [GPUProblem(base, fp).phase_gradient_batch(p)[:2] for p in phs]
    fwd_ref, _ = GPUProblem(base, fp).forward(saveat=[0.0, 0.2, fp.L])
    out = [None, None]
    errs = []

    def worker(i):
        try:
            ctx = Context(0)
            s = torch.cuda.Stream(device=0)
            ctx.set_stream(s)
            gp = GPUProblem(ctx, fp)
            J, g, _ = gp.phase_gradient_batch(phs[i])
            f, _ = gp.forward(saveat=[0.0, 0.2, fp.L])
            out[i] = (J, g, f)
        except Exception as e:  # reported below
            errs.append(e)

    th = [threading.Thread(target=worker, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for i in range(2):
        np.testing.assert_array_equal(out[i][0], ref[i][0])
        np.testing.assert_array_equal(out[i][1], ref[i][1])
        np.testing.assert_array_equal(out[i][2], fwd_ref)


def test_multimode_graph_replays_on_the_caller_stream():
    # the multimode runtime captures its evaluation batch as a CUDA graph on
    # the context's private stream and launches it on the current stream:
    # torch's default (legacy) stream included
    torch = pytest.importorskip("torch")
    fp = P.multimode_problem(1, 32, 256, 5.0, 0.3, 4e-9, 200e-15, seed=0,
                             raman_threshold_thz=-5.0)
    ctx = Context(0)
    ref, _ = GPUProblem(ctx, fp).forward()
    ctx2 = Context(0)
    ctx2.set_stream(torch.cuda.default_stream(0))
    out, st = GPUProblem(ctx2, fp).forward()
    assert st["status"] == 0
    np.testing.assert_array_equal(out, ref)
