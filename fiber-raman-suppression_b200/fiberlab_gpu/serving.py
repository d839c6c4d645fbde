"""Continuous-batching server over the C-ABI (fl_server_*).

Requests -- forward propagations and forward + band-objective + adjoint
phase gradients of differing grid size, fiber length and launch -- are
queued, admitted into device slots as memory and slots free up, advanced a
bounded number of right-hand-side evaluations per launch alongside each
other, and retired with their outputs copied back.  Each request runs the
same stepper as the one-problem-per-call entry points (src/fiberlab/
propagation.jl:89 propagate, physics_models.jl:1033-1046 physical gradient),
alone in its slot, so its result does not depend on what else is running.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from ._capi import (FL_OK, FiberLabGPUError, FlRequest, FlServerInfo, FlServerOpts, FlStats,
                    GPUProblem, load)

FL_REQ_FORWARD = 0
FL_REQ_BAND_GRADIENT = 1
FL_EBUSY = 12
FL_TIMEOUT = 13


@dataclass
class Request:
    """One submitted solve; outputs are filled when it completes."""
    id: int
    kind: int
    problem: GPUProblem
    L: float
    out_field: Optional[np.ndarray] = None
    out_grad: Optional[np.ndarray] = None
    keep: list = field(default_factory=list)   # host buffers the C side copies from/to
    status: Optional[int] = None
    stats: Optional[dict] = None
    J: Optional[float] = None
    latency_ms: Optional[float] = None


class Server:
    def __init__(self, ctx, hbm_budget_bytes: int = 0, evals_per_launch: int = 0,
                 checkpoints: int = 0, segment_steps: int = 0, max_active_ctas: int = 0):
        self.ctx = ctx
        opts = FlServerOpts(hbm_budget_bytes, evals_per_launch, checkpoints, segment_steps,
                            max_active_ctas)
        h = C.c_void_p()
        ctx.check(load().fl_server_create(ctx.h, C.byref(opts), C.byref(h)))
        self.h = h

    def submit_forward(self, gp: GPUProblem, u0=None, L: float = 0.0) -> Request:
        fp = gp.fp
        u0 = np.ascontiguousarray(fp.uw0 if u0 is None else u0, dtype=np.complex128)
        out = np.empty((fp.M, fp.nt), dtype=np.complex128)
        req = FlRequest(gp.h.value, FL_REQ_FORWARD, float(L), u0.ctypes.data, None, None, 0,
                        out.ctypes.data, None)
        return self._submit(req, gp, L, out_field=out, keep=[u0])

    def submit_band_gradient(self, gp: GPUProblem, phase, mask=None, u0=None, L: float = 0.0,
                             log_cost: bool = False) -> Request:
        fp = gp.fp
        u0 = np.ascontiguousarray(fp.uw0 if u0 is None else u0, dtype=np.complex128)
        ph = np.ascontiguousarray(phase, dtype=np.float64)
        m = np.ascontiguousarray(fp.mask if mask is None else mask, dtype=np.uint8)
        g = np.empty(fp.nt)
        req = FlRequest(gp.h.value, FL_REQ_BAND_GRADIENT, float(L), u0.ctypes.data,
                        ph.ctypes.data, m.ctypes.data, int(log_cost), None, g.ctypes.data)
        return self._submit(req, gp, L, out_grad=g, keep=[u0, ph, m])

    def _submit(self, req, gp, L, out_field=None, out_grad=None, keep=()):
        i = C.c_long()
        self.ctx.check(load().fl_server_submit(self.h, C.byref(req), C.byref(i)))
        return Request(i.value, req.kind, gp, L or gp.fp.L, out_field, out_grad, list(keep))

    def _finish(self, r: Request, rc: int, st: FlStats, J, lat):
        r.status, r.stats, r.J, r.latency_ms = rc, st.as_dict(), J.value, lat.value
        if rc != FL_OK:
            raise FiberLabGPUError(rc, f"request {r.id} failed")
        return r

    def poll(self, r: Request) -> bool:
        st, J, lat = FlStats(), C.c_double(), C.c_double()
        rc = load().fl_server_poll(self.h, r.id, C.byref(st), C.byref(J), C.byref(lat))
        if rc == FL_EBUSY:
            return False
        self._finish(r, rc, st, J, lat)
        return True

    def wait(self, r: Request, timeout_ms: float = 600e3) -> Request:
        st, J, lat = FlStats(), C.c_double(), C.c_double()
        rc = load().fl_server_wait(self.h, r.id, float(timeout_ms), C.byref(st), C.byref(J),
                                   C.byref(lat))
        if rc == FL_TIMEOUT:
            raise TimeoutError(f"request {r.id} not finished after {timeout_ms} ms")
        return self._finish(r, rc, st, J, lat)

    def info(self) -> dict:
        inf = FlServerInfo()
        self.ctx.check(load().fl_server_info_get(self.h, C.byref(inf)))
        return inf.as_dict()

    def close(self):
        if getattr(self, "h", None):
            load().fl_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
