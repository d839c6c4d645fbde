"""ctypes binding of the C-ABI declared in include/fiberlab_gpu.h.

The shared library is built in-tree (fiberlab_gpu/libfiberlab_gpu.so).  There
is no CPU fallback: loading fails loudly when the library is missing, and the
calls fail with FL_ENODEV when no CUDA device is present.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# FIBERLAB_GPU_LIB selects another in-tree build of the same C-ABI, e.g. the
# bounds-checked libfiberlab_gpu_checked.so
LIB_PATH = os.environ.get("FIBERLAB_GPU_LIB") or os.path.join(_HERE, "libfiberlab_gpu.so")
CHECKED_LIB_PATH = os.path.join(_HERE, "libfiberlab_gpu_checked.so")

FL_OK = 0
STATUS = {0: "FL_OK", 1: "FL_EINVAL", 2: "FL_NONFINITE", 3: "FL_DT_UNDERFLOW", 4: "FL_MAXITERS",
          5: "FL_ENOMEM", 6: "FL_NONSYMMETRIC", 7: "FL_ENODEV", 8: "FL_ECUDA", 9: "FL_ECAPACITY",
          10: "FL_EUNSUPPORTED", 11: "FL_OOM_ADMISSION", 12: "FL_EBUSY", 13: "FL_TIMEOUT",
          14: "FL_ECHECK"}
PRECISION = {"fp32": 0, "fp64": 1}

# every exported symbol of include/fiberlab_gpu.h (checked by the CPU tests)
EXPORTS = ("fl_version", "fl_status_string", "fl_ctx_create", "fl_ctx_destroy",
           "fl_last_error", "fl_ctx_launch_count", "fl_ctx_synchronize", "fl_problem_create",
           "fl_problem_destroy", "fl_forward", "fl_adjoint", "fl_phase_gradient_batch",
           "fl_phase_gradient_batch_device", "fl_rhs_eval", "fl_ctx_timing",
           "fl_forward_noalloc", "fl_mode_phase_gradient_batch",
           "fl_mode_phase_gradient_batch_device", "fl_server_create", "fl_server_destroy",
           "fl_server_submit", "fl_server_poll", "fl_server_wait", "fl_server_info_get",
           "fl_problem_set_objective", "fl_forward_gain", "fl_ctx_set_stream",
           "fl_ctx_get_stream", "fl_forward_times",
           "fl_forward_evidence")

# device objectives (FL_OBJ_*) by the reference's objective names
# (physics_models.jl:947-962); temporal_width runs with a host seed
OBJECTIVE = {"raman_band": 0, "mode_sum": 0, "mmf_sum": 0, "fundamental_mode": 1,
             "mmf_fundamental": 1, "worst_mode": 2, "mmf_worst_mode": 2, "raman_peak": 3}


class FlCtxOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("checkpoints", C.c_int),
                ("segment_steps", C.c_int), ("step_log", C.c_int), ("max_iters", C.c_long)]


class FlGain(C.Structure):
    """fl_gain: the gain model of fl_forward_gain."""
    _fields_ = [("kind", C.c_int), ("g_const", C.c_double), ("gamma_p", C.c_double),
                ("sigma_ap", C.c_double), ("sigma_ep", C.c_double), ("h_nu_p", C.c_double),
                ("gamma_s", C.c_double), ("area", C.c_double), ("rho", C.c_double),
                ("tau21", C.c_double), ("psd_scale", C.c_double), ("df", C.c_double),
                ("sigma_as", C.c_void_p), ("sigma_es", C.c_void_p), ("h_nu_s", C.c_void_p)]


class FlStats(C.Structure):
    _fields_ = [("naccept", C.c_long), ("nreject", C.c_long), ("nf", C.c_long),
                ("adj_naccept", C.c_long), ("adj_nreject", C.c_long), ("adj_nf", C.c_long),
                ("status", C.c_int), ("checkpoints_used", C.c_int), ("J", C.c_double),
                ("z_end", C.c_double), ("recompute_steps", C.c_long)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class FlServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("evals_per_launch", C.c_int),
                ("checkpoints", C.c_int), ("segment_steps", C.c_int),
                ("max_active_ctas", C.c_int)]


class FlRequest(C.Structure):
    _fields_ = [("prob", C.c_void_p), ("kind", C.c_int), ("L", C.c_double), ("u0", C.c_void_p),
                ("phase", C.c_void_p), ("mask", C.c_void_p), ("log_cost", C.c_int),
                ("out_field", C.c_void_p), ("out_grad", C.c_void_p)]


class FlServerInfo(C.Structure):
    _fields_ = [("submitted", C.c_long), ("completed", C.c_long), ("in_flight", C.c_long),
                ("queued", C.c_long), ("slots", C.c_int), ("chunks", C.c_int),
                ("hbm_bytes", C.c_size_t), ("launches", C.c_long)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class FiberLabGPUError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


_lib = None


def load() -> C.CDLL:
    """Load the CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FiberLabGPUError(7, f"CUDA library not built: {LIB_PATH} is missing "
                                      "(run __graft_entry__.build())")
        lib = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.c_int, C.c_double
        lib.fl_version.restype = C.c_char_p
        lib.fl_status_string.restype = C.c_char_p
        lib.fl_status_string.argtypes = [ip]
        lib.fl_last_error.restype = C.c_char_p
        lib.fl_last_error.argtypes = [vp]
        lib.fl_ctx_create.argtypes = [ip, C.POINTER(FlCtxOpts), C.POINTER(vp)]
        lib.fl_ctx_destroy.argtypes = [vp]
        lib.fl_ctx_launch_count.restype = C.c_long
        lib.fl_ctx_launch_count.argtypes = [vp]
        lib.fl_ctx_synchronize.argtypes = [vp]
        lib.fl_ctx_set_stream.argtypes = [vp, vp]
        lib.fl_ctx_get_stream.restype = vp
        lib.fl_ctx_get_stream.argtypes = [vp]
        lib.fl_problem_create.argtypes = [vp, ip, ip, vp, vp, vp, vp, dp, dp, dp, dp, ip,
                                          C.POINTER(vp)]
        lib.fl_problem_destroy.argtypes = [vp]
        lib.fl_problem_set_objective.argtypes = [vp, ip, dp]
        lib.fl_forward_gain.argtypes = [vp, C.POINTER(FlGain), dp, vp, vp, ip, vp, vp,
                                        C.POINTER(FlStats)]
        lib.fl_forward.argtypes = [vp, vp, vp, ip, vp, C.POINTER(FlStats)]
        lib.fl_adjoint.argtypes = [vp, vp, vp, C.POINTER(FlStats)]
        lib.fl_phase_gradient_batch.argtypes = [vp, vp, ip, vp, vp, ip, vp, vp, vp]
        lib.fl_phase_gradient_batch_device.argtypes = [vp, vp, ip, vp, vp, ip, vp, vp, vp]
        lib.fl_mode_phase_gradient_batch.argtypes = [vp, vp, ip, vp, vp, ip, vp, vp, vp]
        lib.fl_mode_phase_gradient_batch_device.argtypes = [vp, vp, ip, vp, vp, ip, vp, vp, vp]
        lib.fl_rhs_eval.argtypes = [vp, ip, dp, vp, vp, vp]
        lib.fl_forward_times.argtypes = [vp, vp, C.c_long, C.POINTER(C.c_long)]
        lib.fl_forward_evidence.argtypes = [vp, ip, vp]
        lib.fl_ctx_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.fl_server_create.argtypes = [vp, C.POINTER(FlServerOpts), C.POINTER(vp)]
        lib.fl_server_destroy.argtypes = [vp]
        lib.fl_server_submit.argtypes = [vp, C.POINTER(FlRequest), C.POINTER(C.c_long)]
        lib.fl_server_poll.argtypes = [vp, C.c_long, C.POINTER(FlStats), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double)]
        lib.fl_server_wait.argtypes = [vp, C.c_long, C.c_double, C.POINTER(FlStats),
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.fl_server_info_get.argtypes = [vp, C.POINTER(FlServerInfo)]
        lib.fl_forward_noalloc.argtypes = [ip, ip, vp, dp, vp, vp, dp, dp, dp, dp, vp, vp, ip,
                                           vp, vp, C.POINTER(FlStats)]
        _lib = lib
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def forward_noalloc(device: int, nt: int, d_D: int, gamma: float, d_hR: int, d_selfsteep: int,
                    one_m_fR: float, L: float, reltol: float, abstol: float, d_u0: int,
                    d_saveat: int, nsave: int, d_out: int, stream: int = 0):
    """fl_forward_noalloc on caller-owned device buffers (integer device
    addresses); returns (status, stats dict).  The call allocates nothing."""
    st = FlStats()
    rc = load().fl_forward_noalloc(device, nt, d_D, gamma, d_hR, d_selfsteep, one_m_fR, L,
                                   reltol, abstol, d_u0, d_saveat, nsave, d_out, stream,
                                   C.byref(st))
    return rc, st.as_dict()


class Context:
    """fl_ctx on one device (one per host thread)."""

    def __init__(self, device: int = 0, checkpoints: int = 32, segment_steps: int = 64,
                 step_log: int = 0, max_iters: int = 100000, hbm_budget_bytes: int = 0):
        lib = load()
        self.opts = FlCtxOpts(hbm_budget_bytes, checkpoints, segment_steps, step_log, max_iters)
        h = C.c_void_p()
        rc = lib.fl_ctx_create(device, C.byref(self.opts), C.byref(h))
        if rc:
            raise FiberLabGPUError(rc, lib.fl_status_string(rc).decode())
        self.h = h
        self.device = int(device)

    def check(self, rc: int):
        if rc != FL_OK:
            raise FiberLabGPUError(rc, load().fl_last_error(self.h).decode())

    @property
    def launches(self) -> int:
        return load().fl_ctx_launch_count(self.h)

    def timing(self):
        """(last call ms, last stepper-kernel ms), CUDA events on the context stream."""
        a, b = C.c_double(), C.c_double()
        self.check(load().fl_ctx_timing(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def synchronize(self):
        self.check(load().fl_ctx_synchronize(self.h))

    def set_stream(self, stream=None):
        """Run this context's calls on a caller stream (fl_ctx_set_stream):
        a torch.cuda.Stream, a raw cudaStream_t handle (int), or None for the
        context's private stream.  Handle 0 (torch's default stream) is the
        legacy default stream and is passed as cudaStreamLegacy."""
        h = getattr(stream, "cuda_stream", stream)
        if stream is not None and h == 0:
            h = 1  # cudaStreamLegacy
        self.check(load().fl_ctx_set_stream(self.h, None if stream is None else int(h)))

    @property
    def stream(self) -> int:
        """The raw handle of the stream the context's calls run on."""
        return int(load().fl_ctx_get_stream(self.h) or 0)

    def close(self):
        if getattr(self, "h", None):
            load().fl_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GPUProblem:
    """fl_problem: device-resident tables of one resolved problem."""

    def __init__(self, ctx: Context, fp, precision: str = "fp32"):
        self.ctx, self.fp = ctx, fp
        nt, M = fp.nt, fp.M
        self._D = np.ascontiguousarray(fp.D, dtype=np.float64)
        self._g = np.ascontiguousarray(fp.gamma_ref_order(), dtype=np.float64)
        self._h = np.ascontiguousarray(fp.hR, dtype=np.complex128)
        self._s = np.ascontiguousarray(fp.selfsteep, dtype=np.float64)
        h = C.c_void_p()
        ctx.check(load().fl_problem_create(ctx.h, nt, M, _ptr(self._D), _ptr(self._g),
                                           _ptr(self._h), _ptr(self._s), float(fp.one_m_fR),
                                           float(fp.L), float(fp.reltol), float(fp.abstol),
                                           PRECISION[precision], C.byref(h)))
        self.h = h
        self.objective = "raman_band"

    def set_objective(self, name: str, worst_mode_tau: float = 50.0):
        """Objective of the batched gradient calls and band-gradient server
        requests of this problem (fl_problem_set_objective)."""
        if name not in OBJECTIVE:
            raise ValueError(f"objective {name!r} has no device seed; device objectives: "
                             f"{', '.join(sorted(OBJECTIVE))}")
        self.ctx.check(load().fl_problem_set_objective(self.h, OBJECTIVE[name],
                                                       float(worst_mode_tau)))
        self.objective = name

    def forward_gain(self, gain, pump_power: float, u0=None, saveat=None):
        """Pump-gain forward solve (fl_forward_gain): gain is a constant gain
        [1/m] or a fiberlab_gpu.gain.YDFAParams; returns the lab-frame spectra
        (nsave, 1, Nt) and pump powers (nsave,) at saveat (default [0, L]),
        and the stats."""
        from . import gain as G
        fp = self.fp
        u0 = np.ascontiguousarray(fp.uw0 if u0 is None else u0, dtype=np.complex128)
        g = FlGain()
        keep = []
        if isinstance(gain, (int, float)):
            g.kind, g.g_const = 0, float(gain)
        else:
            a = G.gain_struct_arrays(gain)
            g.kind = 1
            for k in ("gamma_p", "sigma_ap", "sigma_ep", "h_nu_p", "gamma_s", "area", "rho",
                      "tau21", "psd_scale", "df"):
                setattr(g, k, float(a[k]))
            for k in ("sigma_as", "sigma_es", "h_nu_s"):
                arr = np.ascontiguousarray(a[k], dtype=np.float64)
                keep.append(arr)
                setattr(g, k, arr.ctypes.data)
        z = np.ascontiguousarray([0.0, fp.L] if saveat is None else saveat, dtype=np.float64)
        out = np.empty((len(z), 1, fp.nt), dtype=np.complex128)
        pumps = np.empty(len(z))
        st = FlStats()
        self.ctx.check(load().fl_forward_gain(self.h, C.byref(g), float(pump_power), _ptr(u0),
                                              _ptr(z), len(z), _ptr(out), _ptr(pumps),
                                              C.byref(st)))
        return out, pumps, st.as_dict()

    def forward(self, u0=None, saveat=None):
        fp = self.fp
        u0 = np.ascontiguousarray(fp.uw0 if u0 is None else u0, dtype=np.complex128)
        z = np.ascontiguousarray([0.0, fp.L] if saveat is None else saveat, dtype=np.float64)
        out = np.empty((len(z), fp.M, fp.nt), dtype=np.complex128)
        st = FlStats()
        self.ctx.check(load().fl_forward(self.h, _ptr(u0), _ptr(z), len(z), _ptr(out),
                                         C.byref(st)))
        return out, st.as_dict()

    def forward_times(self) -> np.ndarray:
        """sol.t of the last forward: 0, every accepted step end, L."""
        n = C.c_long()
        self.ctx.check(load().fl_forward_times(self.h, None, 0, C.byref(n)))
        t = np.empty(n.value)
        self.ctx.check(load().fl_forward_times(self.h, _ptr(t), n.value, C.byref(n)))
        return t

    def forward_evidence(self, nsave: int) -> np.ndarray:
        """Device FP64 evidence sums of the last forward's nsave saved
        spectra (fl_forward_evidence): rows of [Σ P(t), max P(t), P at the
        temporal edges, Σ S(ω), S at the spectral edges, Σ |u|²/|selfsteep|,
        then Σ_t |fft(u_m)|² per mode]."""
        ev = np.empty((int(nsave), 6 + self.fp.M))
        self.ctx.check(load().fl_forward_evidence(self.h, int(nsave), _ptr(ev)))
        return ev

    def adjoint(self, lambdaL):
        lam = np.ascontiguousarray(lambdaL, dtype=np.complex128)
        out = np.empty_like(lam)
        st = FlStats()
        self.ctx.check(load().fl_adjoint(self.h, _ptr(lam), _ptr(out), C.byref(st)))
        return out, st.as_dict()

    def rhs(self, z, u, ufwd=None):
        """One forward (ufwd None) or adjoint RHS evaluation on the GPU."""
        u = np.ascontiguousarray(u, dtype=np.complex128)
        out = np.empty_like(u)
        uf = None if ufwd is None else np.ascontiguousarray(ufwd, dtype=np.complex128)
        self.ctx.check(load().fl_rhs_eval(self.h, int(uf is not None), float(z), _ptr(u),
                                          None if uf is None else _ptr(uf), _ptr(out)))
        return out

    def phase_gradient_batch(self, phases, mask=None, u0=None, log_cost=False, out=None):
        """Host-buffer batch: phases (B, Nt) -> J (B,), grad (B, Nt).  out =
        (J, grad) reuses caller arrays (page-locked ones make the library's
        copies direct transfers)."""
        fp = self.fp
        ph = np.ascontiguousarray(np.atleast_2d(phases), dtype=np.float64)
        B = ph.shape[0]
        u0 = np.ascontiguousarray(fp.uw0 if u0 is None else u0, dtype=np.complex128)
        m = np.ascontiguousarray(fp.mask if mask is None else mask, dtype=np.uint8)
        if out is None:
            J, g = np.empty(B), np.empty((B, fp.nt))
        else:
            J, g = out
            if J.shape != (B,) or g.shape != (B, fp.nt) or J.dtype != np.float64 or \
                    g.dtype != np.float64 or not (J.flags.c_contiguous and g.flags.c_contiguous):
                raise ValueError("out must be contiguous float64 arrays of shapes (B,), (B, Nt)")
        st = (FlStats * B)()
        self.ctx.check(load().fl_phase_gradient_batch(self.h, _ptr(u0), B, _ptr(ph), _ptr(m),
                                                      int(log_cost), _ptr(J), _ptr(g), st))
        return J, g, [s.as_dict() for s in st]

    def mode_phase_gradient_batch(self, phases, mask=None, u0=None, log_cost=False):
        """One phase per (mode, time bin): phases (B, M, Nt) -> J (B,), grad (B, M, Nt)."""
        fp = self.fp
        ph = np.ascontiguousarray(phases, dtype=np.float64).reshape(-1, fp.M, fp.nt)
        B = ph.shape[0]
        u0 = np.ascontiguousarray(fp.uw0 if u0 is None else u0, dtype=np.complex128)
        m = np.ascontiguousarray(fp.mask if mask is None else mask, dtype=np.uint8)
        J = np.empty(B)
        g = np.empty((B, fp.M, fp.nt))
        st = (FlStats * B)()
        self.ctx.check(load().fl_mode_phase_gradient_batch(self.h, _ptr(u0), B, _ptr(ph), _ptr(m),
                                                           int(log_cost), _ptr(J), _ptr(g), st))
        return J, g, [s.as_dict() for s in st]

    def phase_gradient_batch_device(self, d_u0: int, B: int, d_phases: int, d_mask: int,
                                    d_J: int, d_grad: int, log_cost=False, with_stats=True):
        st = (FlStats * B)() if with_stats else None
        self.ctx.check(load().fl_phase_gradient_batch_device(
            self.h, d_u0, B, d_phases, d_mask, int(log_cost), d_J, d_grad, st))
        return [s.as_dict() for s in st] if with_stats else None

    def mode_phase_gradient_batch_device(self, d_u0: int, B: int, d_phases: int, d_mask: int,
                                         d_J: int, d_grad: int, log_cost=False,
                                         with_stats=True):
        """Per-mode phases (B, M, Nt) and gradients on device buffers."""
        st = (FlStats * B)() if with_stats else None
        self.ctx.check(load().fl_mode_phase_gradient_batch_device(
            self.h, d_u0, B, d_phases, d_mask, int(log_cost), d_J, d_grad, st))
        return [s.as_dict() for s in st] if with_stats else None

    def close(self):
        if getattr(self, "h", None):
            load().fl_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
