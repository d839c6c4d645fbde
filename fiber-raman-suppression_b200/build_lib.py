"""Build recipe of the CUDA library (sm_100a only).

Compiles every translation unit under csrc/ in parallel with nvcc
(-gencode arch=compute_100a,code=sm_100a) and links
fiberlab_gpu/libfiberlab_gpu.so in-tree.  Objects are cached under _build/
and rebuilt when their source or any header changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "fiberlab_gpu", "libfiberlab_gpu.so")
# the checked build: -DFL_CHECKED adds the solver state-index checks
# (FL_ECHECK instead of an out-of-bounds access); no -lineinfo, to keep it small
BUILD_CHECKED = os.path.join(HERE, "_build_checked")
OUT_CHECKED = os.path.join(HERE, "fiberlab_gpu", "libfiberlab_gpu_checked.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA library cannot be built")


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src: str, obj: str, verbose: bool, checked: bool = False) -> str:
    flags = [f for f in FLAGS if f != "-lineinfo"] + ["-DFL_CHECKED"] if checked else FLAGS
    cmd = [nvcc()] + ARCH + flags + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stderr}")
    return r.stderr


def build(jobs: int | None = None, verbose: bool = False, force: bool = False,
          checked: bool = False) -> str:
    bdir, out = (BUILD_CHECKED, OUT_CHECKED) if checked else (BUILD, OUT)
    os.makedirs(bdir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hmt = _headers_mtime()
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(bdir, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hmt):
            todo.append((s, o))
    logs = {}
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            futs = {ex.submit(_compile, s, o, verbose, checked): s for s, o in todo}
            for f in cf.as_completed(futs):
                logs[futs[f]] = f.result()
    if todo or not os.path.exists(out):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", out] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    if verbose:
        for s, l in sorted(logs.items()):
            print(f"== {os.path.basename(s)}\n{l}")
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv, checked="--checked" in sys.argv))
