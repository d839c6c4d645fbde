"""The bounds-checked build (libfiberlab_gpu_checked.so, -DFL_CHECKED).

Its solver state-index checks (stage, buffer parities, step log, checkpoint
segment and sub-segment, save position) must not change any result: the
same solves through the checked library -- loaded in a child process via
FIBERLAB_GPU_LIB -- give bit-identical outputs to the default library,
including solves that recompute in sub-segments and a multimode solve.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from fiberlab_gpu import _capi
from fiberlab_gpu import problem as P
from fiberlab_gpu._capi import Context, GPUProblem

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _solves(ctx_small):
    """(J, grad) of a single-mode gradient (dense forward), the same with a
    recompute in sub-segments, and a 3-mode gradient."""
    out = {}
    fp = P.single_mode_problem(nt=1024, time_window_ps=10.0, L=0.5, power_w=0.1,
                               rep_rate_hz=80.5e6, raman_threshold_thz=-5.0)
    phi = 0.5 * np.random.default_rng(41).standard_normal((2, fp.nt))
    out["sm_J"], out["sm_g"], _ = GPUProblem(Context(0), fp).phase_gradient_batch(phi)
    out["sub_J"], out["sub_g"], _ = GPUProblem(ctx_small, fp).phase_gradient_batch(phi)
    mp = P.multimode_problem(1, 32, 256, 5.0, 0.3, 4e-9, 200e-15, seed=0,
                             raman_threshold_thz=-5.0)
    mphi = 0.3 * np.random.default_rng(42).standard_normal((1, mp.nt))
    out["mm_J"], out["mm_g"], _ = GPUProblem(ctx_small, mp).phase_gradient_batch(mphi)
    return out


_CHILD = """
import sys, numpy as np
sys.path[:0] = [{root!r}, {pkg!r}, {tests!r}]
from fiberlab_gpu._capi import Context
import test_gpu_checked as T
np.savez({out!r}, **T._solves(Context(0, checkpoints=2, segment_steps=3)))
"""


def test_checked_build_gives_identical_results():
    if not os.path.exists(_capi.CHECKED_LIB_PATH):
        pytest.fail("the checked library is not built (run __graft_entry__.build())")
    ref = _solves(Context(0, checkpoints=2, segment_steps=3))
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "checked.npz")
        code = _CHILD.format(root=ROOT, pkg=os.path.join(ROOT, "fiber-raman-suppression_b200"),
                             tests=os.path.join(ROOT, "tests"), out=out)
        env = dict(os.environ, FIBERLAB_GPU_LIB=_capi.CHECKED_LIB_PATH)
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        got = np.load(out)
        for k, v in ref.items():
            np.testing.assert_array_equal(got[k], v, err_msg=k)
