#!/usr/bin/env python
"""Generate the multimode gradient fixtures from the FP64 CPU oracle.

TEST INFRASTRUCTURE: runs the oracle (oracle/libfl_oracle.so, the FP64 C
restatement of simulate_disp_mmf.jl:25-60 / sensitivity_disp_mmf.jl:32-215,
309-332) once on the CPU and writes what the GPU tests compare against:

* config 2 (mm_config2.npz): M = 6 HG(m+n<=2) on a 64x64 grid, Nt = 2^12
  over 5 ps, L = 1 m, 2 nJ 200 fs sech², Dirichlet(1) launch weights with
  random phases (seed 0); per-mode spectral phase control φ[m, t] ~
  N(0, 0.5²) (seed 2); band objective on the red side beyond 2 THz (the
  -13 THz band holds only round-off at 2 nJ).  Stored: J, the per-mode
  gradient ∂J/∂φ[m, t] (physics_models.jl:1042 without the mode sum), the
  lab-frame output field and the oracle's step counts.
* config 4 (mm_config4.npz): M = 10 HG(m+n<=3) on a 96x96 grid, Nt = 2^14
  over 10 ps, L = 2 m, 5 nJ; 4 candidates of per-mode phases φ ~ N(0, 1)
  (seeds 4000..4003); band beyond 2 THz.  Stored: J per candidate, the
  gradient on the bins where the launch spectrum is not negligible (the
  gradient is 2 Re(conj(λ0) i u_shaped), so it vanishes with the launch;
  the norm dropped outside is recorded and is below 1e-9 of the total),
  candidate 0's output field (complex64) and the step counts.

Usage: python tests/golden/make_multimode_fixtures.py [config2|config4|all]
Config 4 takes about ten minutes per candidate on one core (the candidates
run in parallel processes).
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _p in (ROOT, os.path.join(ROOT, "fiber-raman-suppression_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

C4_SEEDS = (4000, 4001, 4002, 4003)
SUPPORT_REL = 1e-24  # launch bins kept: |u0|² summed over modes > this × max


def config2_problem():
    from fiberlab_gpu import problem as P
    return P.multimode_problem(2, 64, 4096, 5.0, 1.0, 2e-9, 200e-15, seed=0,
                               raman_threshold_thz=-2.0)


def config2_phases(fp):
    return 0.5 * np.random.default_rng(2).standard_normal((fp.M, fp.nt))


def config4_problem():
    from fiberlab_gpu import problem as P
    return P.multimode_problem(3, 96, 16384, 10.0, 2.0, 5e-9, 200e-15, seed=0,
                               raman_threshold_thz=-2.0)


def config4_phases(fp, seed):
    return np.random.default_rng(seed).standard_normal((fp.M, fp.nt))


def support(fp):
    """Bins where the launch spectrum (summed over modes) is not negligible."""
    e = np.sum(np.abs(fp.uw0) ** 2, axis=0)
    return np.nonzero(e > SUPPORT_REL * e.max())[0]


def oracle_mode_gradient(fp, phases):
    """J and ∂J/∂φ[m, t] of the band objective: oracle forward (dense
    output kept), band cost and seed (physics_helpers.jl:222-232), oracle
    adjoint, 2 Re(conj(λ0) i u_shaped)."""
    from fiberlab_gpu import problem as P
    from oracle import oracle as O
    us = fp.uw0 * np.exp(1j * phases)
    out, fst, dense = O.forward(fp, u0=us, keep_dense=True)
    J, seed = P.band_cost_and_seed(out[-1], fp.mask)
    lam0, ast = O.adjoint(fp, dense, seed)
    g = 2 * np.real(np.conj(lam0) * 1j * us)
    return J, g, out[-1], fst, ast


def _c4_worker(seed):
    t = time.time()
    fp = config4_problem()
    J, g, uL, fst, ast = oracle_mode_gradient(fp, config4_phases(fp, seed))
    return seed, J, g, uL, fst, ast, time.time() - t


def make_config2():
    t = time.time()
    fp = config2_problem()
    J, g, uL, fst, ast = oracle_mode_gradient(fp, config2_phases(fp))
    path = os.path.join(HERE, "mm_config2.npz")
    np.savez_compressed(path, J=J, grad=g, uL=uL, fwd_naccept=fst["naccept"],
                        adj_naccept=ast["naccept"], nt=fp.nt, M=fp.M)
    print(f"config 2: J={J:.6e}, fwd {fst['naccept']} / adj {ast['naccept']} steps, "
          f"{time.time() - t:.1f} s -> {path}")


def make_config4():
    fp = config4_problem()
    idx = support(fp)
    with mp.get_context("spawn").Pool(len(C4_SEEDS)) as pool:
        res = sorted(pool.map(_c4_worker, C4_SEEDS))
    Js, gs, drop, fna, ana = [], [], [], [], []
    uL0 = None
    for seed, J, g, uL, fst, ast, dt in res:
        mask = np.ones(fp.nt, bool)
        mask[idx] = False
        dropped = float(np.linalg.norm(g[:, mask]) / np.linalg.norm(g))
        assert dropped < 1e-9, (seed, dropped)
        Js.append(J)
        gs.append(g[:, idx].astype(np.float32))
        drop.append(dropped)
        fna.append(fst["naccept"])
        ana.append(ast["naccept"])
        if seed == C4_SEEDS[0]:
            uL0 = uL.astype(np.complex64)
        print(f"config 4 seed {seed}: J={J:.6e}, fwd {fst['naccept']} / adj {ast['naccept']} "
              f"steps, {dt:.0f} s, dropped gradient norm {dropped:.1e}")
    path = os.path.join(HERE, "mm_config4.npz")
    np.savez_compressed(path, seeds=np.array(C4_SEEDS), J=np.array(Js), idx=idx.astype(np.int32),
                        grad=np.stack(gs), dropped=np.array(drop), uL0=uL0,
                        fwd_naccept=np.array(fna), adj_naccept=np.array(ana), nt=fp.nt, M=fp.M)
    print(f"-> {path} ({os.path.getsize(path) / 1e6:.2f} MB, {len(idx)} support bins)")


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("config2", "all"):
        make_config2()
    if what in ("config4", "all"):
        make_config4()
