"""ctypes front end of the FP64 CPU oracle (libfl_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py's CPU-baseline leg.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class OrcProblem(C.Structure):
    _fields_ = [("nt", C.c_int), ("m", C.c_int), ("D", C.c_void_p), ("gamma", C.c_void_p),
                ("hR", C.c_void_p), ("selfsteep", C.c_void_p), ("one_m_fR", C.c_double),
                ("L", C.c_double), ("reltol", C.c_double), ("abstol", C.c_double)]


class OrcStats(C.Structure):
    _fields_ = [("naccept", C.c_long), ("nreject", C.c_long), ("nf", C.c_long),
                ("retcode", C.c_int), ("z_end", C.c_double)]


RETCODES = {0: "ok", 1: "invalid argument", 2: "non-finite value", 3: "dt underflow",
            4: "maxiters", 5: "out of memory", 6: "gamma not permutation-symmetric"}


class OrcGain(C.Structure):
    _fields_ = [("kind", C.c_int), ("g_const", C.c_double), ("gamma_p", C.c_double),
                ("sigma_ap", C.c_double), ("sigma_ep", C.c_double), ("h_nu_p", C.c_double),
                ("gamma_s", C.c_double), ("area", C.c_double), ("rho", C.c_double),
                ("tau21", C.c_double), ("psd_scale", C.c_double), ("df", C.c_double),
                ("sigma_as", C.c_void_p), ("sigma_es", C.c_void_p), ("h_nu_s", C.c_void_p)]


class OracleError(RuntimeError):
    def __init__(self, rc):
        super().__init__(f"oracle error {rc}: {RETCODES.get(rc, '?')}")
        self.rc = rc


def build() -> str:
    path = os.path.join(_HERE, "libfl_oracle.so")
    src = os.path.join(_HERE, "fl_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return path


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        _LIB.orc_dense_steps.restype = C.c_long
    return _LIB


class Problem:
    """Holds the contiguous FP64 tables behind an orc_problem struct."""

    def __init__(self, fp):
        self.fp = fp
        self.D = np.ascontiguousarray(fp.D, dtype=np.float64)
        self.gamma = fp.gamma_ref_order().astype(np.float64)
        self.hR = np.ascontiguousarray(fp.hR, dtype=np.complex128)
        self.ss = np.ascontiguousarray(fp.selfsteep, dtype=np.float64)
        self.s = OrcProblem(fp.nt, fp.M, self.D.ctypes.data, self.gamma.ctypes.data,
                            self.hR.ctypes.data, self.ss.ctypes.data, float(fp.one_m_fR),
                            float(fp.L), float(fp.reltol), float(fp.abstol))

    def ref(self):
        return C.byref(self.s)


def _c(a, dtype=np.complex128):
    return np.ascontiguousarray(a, dtype=dtype)


def fft(x, inverse=False):
    x = _c(x).copy()
    nt = x.shape[-1]
    ncols = x.size // nt
    rc = lib().orc_fft(C.c_void_p(x.ctypes.data), nt, ncols, int(inverse))
    if rc:
        raise OracleError(rc)
    return x


def rhs_forward(fp, z, u):
    P = Problem(fp)
    u = _c(u)
    du = np.empty_like(u)
    rc = lib().orc_rhs_forward(P.ref(), C.c_double(z), C.c_void_p(u.ctypes.data),
                               C.c_void_p(du.ctypes.data))
    if rc:
        raise OracleError(rc)
    return du


def rhs_adjoint(fp, z, lam, ufwd):
    P = Problem(fp)
    lam, ufwd = _c(lam), _c(ufwd)
    out = np.empty_like(lam)
    rc = lib().orc_rhs_adjoint(P.ref(), C.c_double(z), C.c_void_p(lam.ctypes.data),
                               C.c_void_p(ufwd.ctypes.data), C.c_void_p(out.ctypes.data))
    if rc:
        raise OracleError(rc)
    return out


class Dense:
    def __init__(self, ptr, fp):
        self.ptr = ptr
        self.fp = fp

    def __del__(self):
        if self.ptr:
            lib().orc_dense_free(C.c_void_p(self.ptr))
            self.ptr = None

    def __call__(self, z):
        out = np.empty((self.fp.M, self.fp.nt), dtype=np.complex128)
        rc = lib().orc_dense_eval(C.c_void_p(self.ptr), C.c_double(z), C.c_void_p(out.ctypes.data))
        if rc:
            raise OracleError(rc)
        return out

    @property
    def t(self):
        n = lib().orc_dense_steps(C.c_void_p(self.ptr))
        out = np.empty(n + 1)
        lib().orc_dense_times(C.c_void_p(self.ptr), C.c_void_p(out.ctypes.data))
        return out


def forward(fp, u0=None, zsave=None, keep_dense=False):
    """Returns (lab spectra (nsave, M, Nt), stats dict, Dense or None)."""
    P = Problem(fp)
    u0 = _c(fp.uw0 if u0 is None else u0)
    zs = np.ascontiguousarray([0.0, fp.L] if zsave is None else zsave, dtype=np.float64)
    out = np.empty((len(zs), fp.M, fp.nt), dtype=np.complex128)
    st = OrcStats()
    dptr = C.c_void_p()
    rc = lib().orc_forward(P.ref(), C.c_void_p(u0.ctypes.data), len(zs),
                           C.c_void_p(zs.ctypes.data), C.c_void_p(out.ctypes.data),
                           C.byref(st), C.byref(dptr) if keep_dense else None)
    if rc:
        raise OracleError(rc)
    stats = dict(naccept=st.naccept, nreject=st.nreject, nf=st.nf)
    return out, stats, (Dense(dptr.value, fp) if keep_dense else None)


def adjoint(fp, dense, lambdaL):
    P = Problem(fp)
    lam = _c(lambdaL)
    out = np.empty_like(lam)
    st = OrcStats()
    rc = lib().orc_adjoint(P.ref(), C.c_void_p(dense.ptr), C.c_void_p(lam.ctypes.data),
                           C.c_void_p(out.ctypes.data), C.byref(st))
    if rc:
        raise OracleError(rc)
    return out, dict(naccept=st.naccept, nreject=st.nreject, nf=st.nf)


def rk4_scalar(fp, steps, u0=None):
    P = Problem(fp)
    u0 = _c(fp.uw0 if u0 is None else u0)
    out = np.empty_like(u0)
    rc = lib().orc_rk4_scalar(P.ref(), C.c_void_p(u0.ctypes.data), int(steps),
                              C.c_void_p(out.ctypes.data))
    if rc:
        raise OracleError(rc)
    return out


def tsit5_order_residuals(theta):
    res = np.zeros(16)
    n = lib().orc_tsit5_order_residuals(C.c_double(theta), C.c_void_p(res.ctypes.data), 16)
    return res[:n]


def batch_phase_gradient(fp, phases, mask, nthreads=0):
    """phases (B, Nt).  Returns (J (B,), grad (B, Nt), steps (B,), failed)."""
    P = Problem(fp)
    ph = _c(phases, np.float64)
    B = ph.shape[0]
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    J = np.zeros(B)
    g = np.zeros((B, fp.nt))
    ns = np.zeros(B, dtype=np.int64)
    u0 = _c(fp.uw0)
    failed = lib().orc_batch_phase_gradient(P.ref(), C.c_void_p(u0.ctypes.data),
                                            C.c_void_p(ph.ctypes.data), B,
                                            C.c_void_p(m.ctypes.data), C.c_void_p(J.ctypes.data),
                                            C.c_void_p(g.ctypes.data), C.c_void_p(ns.ctypes.data),
                                            int(nthreads))
    return J, g, ns, failed


def phase_gradient(fp, phase):
    """Single problem: J and ∂J/∂φ (vector phase, summed over modes)."""
    J, g, ns, failed = batch_phase_gradient(fp, np.asarray(phase)[None, :], fp.mask, 1)
    if failed:
        raise OracleError(2)
    return float(J[0]), g[0], int(ns[0])


def _gain_struct(gain):
    """orc_gain from a constant gain [1/m] or a YDFAParams (the arrays are
    kept alive on the returned holder)."""
    from fiberlab_gpu import gain as G
    g = OrcGain()
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
    return g, keep


def rhs_gain(fp, gain, z, pump, u):
    """One pump-gain RHS evaluation (orc_rhs_gain): returns (dP/dz, du~/dz)."""
    pr = Problem(fp)
    g, keep = _gain_struct(gain)
    st = _c(np.concatenate([[complex(pump)], np.asarray(u, np.complex128).reshape(-1)]))
    out = np.empty_like(st)
    rc = lib().orc_rhs_gain(C.byref(pr.s), C.byref(g), C.c_double(z),
                            C.c_void_p(st.ctypes.data), C.c_void_p(out.ctypes.data))
    if rc:
        raise OracleError(rc)
    return out[0], out[1:].reshape(1, -1)


def forward_gain(fp, gain, pump0, u0=None, zsave=None):
    """Pump-gain solve 0 -> L (orc_forward_gain): lab-frame spectra at zsave
    ((nsave, 1, Nt); default [0, L]), the pump powers there, and stats."""
    pr = Problem(fp)
    g, keep = _gain_struct(gain)
    u0 = _c(fp.uw0 if u0 is None else u0)
    zs = np.ascontiguousarray([0.0, fp.L] if zsave is None else zsave, dtype=np.float64)
    out = np.empty((len(zs), 1, fp.nt), np.complex128)
    pumps = np.empty(len(zs))
    st = OrcStats()
    rc = lib().orc_forward_gain(C.byref(pr.s), C.byref(g), C.c_double(pump0),
                                C.c_void_p(u0.ctypes.data), len(zs), C.c_void_p(zs.ctypes.data),
                                C.c_void_p(out.ctypes.data), C.c_void_p(pumps.ctypes.data),
                                C.byref(st))
    if rc:
        raise OracleError(rc)
    return out, pumps, {"naccept": st.naccept, "nreject": st.nreject, "nf": st.nf,
                        "z_end": st.z_end}
