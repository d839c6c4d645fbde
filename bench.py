#!/usr/bin/env python
"""Headline benchmark: batched FP32 forward+adjoint band-gradient solves on B200.

Workload (one "step"): B independent single-mode inverse-design problems of
the Nt = 2^13 / 10 ps / SMF-28 / 0.5 m / 0.1 W / 185 fs sech² shape, each
with its own launch phase φ_b ~ N(0, 0.5²) (seeded), run forward, Raman-band
objective (< -13 THz), adjoint with z-checkpoints (32 slots) + recompute,
and phase gradient, all on the GPU in one batched call.  Metric: fwd+adjoint
solves/s (higher is better), whole job over all ranks.  The plain
one-at-a-time path (the same solve, one problem per call) and its latency
quantiles are reported beside it.

Multi-GPU: replicas only (independent problems per rank, no collective on
the data path; a barrier brackets the timed region and the time is the max
over ranks).  `--impl reference` times the CPU reference arm: the FP64 C
restatement of the reference solver on all host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "fiber-raman-suppression_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "fwd+adjoint solves/s"
UNIT = "solves/s"
NT, T_PS, L_M, P_W, REP = 8192, 10.0, 0.5, 0.1, 80e6
BYTES_FWD_STEP = 336  # per point per attempted forward step (FP32 complex field passes)
BYTES_ADJ_STEP = 384  # per point per attempted adjoint step
ORACLE_FFT = "radix-4 Stockham FP64 FFT in C, x86-64-v3 build (FFTW is not available)"


def workload_problem():
    from fiberlab_gpu import problem as P
    return P.single_mode_problem(nt=NT, time_window_ps=T_PS, L=L_M, power_w=P_W,
                                 rep_rate_hz=REP, raman_threshold_thz=-13.0,
                                 validate_grid=False)


def phases(rank: int, B: int, nt: int) -> np.ndarray:
    rng = np.random.default_rng(1000 + rank)
    return 0.5 * rng.standard_normal((B, nt))


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def config(B, world, extra=None,
           precision="FP32 bulk; FP64 phase/state/error norm/reductions; FP64 adjoint"):
    c = {"workload": f"single-mode inverse-design batch: Nt=2^13 over 10 ps, SMF-28, L=0.5 m, "
                     f"0.1 W/80 MHz 185 fs sech², phase N(0,0.5²), Raman band < -13 THz, "
                     f"fwd+adjoint, 32 z-checkpoints / 64 dense-output steps",
         "batch_per_gpu": B, "global_batch": B * world, "nt": NT, "modes": 1,
         "precision": precision,
         "parallelism": f"replicas x{world}", "l2": "inputs and per-slot workspaces > L2 (126 MB)"}
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per attempted (forward or adjoint) step from the committed
    ncu capture of the stepper (profiles/sm_advance_traffic.json); the bench
    scales it to its own launch by the attempted steps of that launch."""
    p = os.path.join(ROOT, "profiles", "sm_advance_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def cpu_baseline(fp, nthreads: int, nprob: int):
    from oracle import oracle as O
    ph = phases(999, nprob, fp.nt)
    t0 = time.perf_counter()
    J, g, ns, failed = O.batch_phase_gradient(fp, ph, fp.mask, nthreads)
    dt = time.perf_counter() - t0
    return nprob / dt, dt


SERVE_MIX = ("config 3: Poisson 2000/s, Nt 2^11..2^15 over 10 ps, L U(0.1,5) m, P U(0.02,0.3) W, "
             "half fwd / half fwd+adjoint (phase N(0,0.5^2)), FP32, seed 3")


def _quantiles(lat):
    return ({"latency_ms_p50": float(np.percentile(lat, 50)),
             "latency_ms_p99": float(np.percentile(lat, 99))} if lat else
            {"latency_ms_p50": None, "latency_ms_p99": None})


def _plain_worker(q, stop, dev_index, n, seed, window_s):
    """The plain one-at-a-time drop-in over the config-3 stream, in a child
    process: request i starts when it has arrived and request i-1 has
    finished, through the plain entry points with a problem per request
    (the reference builds its tables per solve).  Reports each completion
    (time since the stream's start, latency from arrival); stops starting
    requests when asked or after the window."""
    for _p in (ROOT, PKG):
        if _p not in sys.path:
            sys.path.insert(0, _p)
    from fiberlab_gpu import problem as P
    from fiberlab_gpu._capi import Context, FiberLabGPUError, GPUProblem
    reqs = P.serving_mix(n, seed=seed)
    grids = {nt: P.serving_grid_problem(nt) for nt in sorted({r.nt for r in reqs})}
    ctx = Context(dev_index, checkpoints=256, segment_steps=128, max_iters=400000)
    # one small solve per grid outside the stream (module load, first launches)
    for fp0 in grids.values():
        fp = P.FiberProblem(**{**fp0.__dict__})
        fp.L = 1e-3
        GPUProblem(ctx, fp).forward(P.serving_launch(fp0, 0.02))
    q.put(("start",))
    t0 = time.perf_counter()
    for i, r in enumerate(reqs):
        now = time.perf_counter() - t0
        if stop.is_set() or now > window_s:
            break
        if now < r.arrival_s:
            time.sleep(r.arrival_s - now)
        fp0 = grids[r.nt]
        u0 = P.serving_launch(fp0, r.power_w)
        status = 0
        try:
            fp = P.FiberProblem(**{**fp0.__dict__})
            fp.L = r.L
            gp = GPUProblem(ctx, fp)
            if r.kind == 0:
                gp.forward(u0)
            else:
                gp.phase_gradient_batch(r.phase[None, :], u0=u0)
        except FiberLabGPUError as e:
            status = e.status
        fin = time.perf_counter() - t0
        q.put(("done", i, status, fin, fin - r.arrival_s))
    q.put(("end",))


def serving_measure(ctx_cls, dev_index, n, window_s, plain_window_s, seed=3):
    """Config-3 stream (n requests, Poisson arrivals at 2000/s, log2 Nt
    uniform on 11..15 over 10 ps, L ~ U(0.1, 5) m, P ~ U(0.02, 0.3) W, half
    forward-only and half forward + band gradient with phase N(0, 0.5²)),
    taken by both paths in arrival order over a bounded window: the
    continuous-batching server (requests submitted as they arrive) for
    window_s seconds, then the plain one-at-a-time path for plain_window_s
    seconds.  Each path reports the requests completed inside its window,
    solves/s, p50/p99 latency (arrival to result) of those, the requests
    arrived but unfinished at the window's end and failures by status."""
    import multiprocessing as mp
    from fiberlab_gpu import problem as P
    from fiberlab_gpu._capi import FiberLabGPUError, GPUProblem
    from fiberlab_gpu.serving import Server
    ctx = ctx_cls(dev_index)
    reqs = P.serving_mix(n, seed=seed)
    grids = {}
    for r in reqs:
        if r.nt not in grids:
            fp = P.serving_grid_problem(r.nt)
            grids[r.nt] = (fp, GPUProblem(ctx, fp))
    srv = Server(ctx)
    # allocate each shape's first chunk outside the measured stream
    for nt, (fp, gp) in sorted(grids.items()):
        srv.wait(srv.submit_forward(gp, u0=P.serving_launch(fp, 0.02), L=1e-3))
    statuses, lat = {}, []
    t0 = time.perf_counter()
    i, outstanding = 0, []
    while True:
        now = time.perf_counter() - t0
        if now > window_s or (i >= n and not outstanding):
            break
        while i < n and reqs[i].arrival_s <= now:
            r = reqs[i]
            fp, gp = grids[r.nt]
            u0 = P.serving_launch(fp, r.power_w)
            h = (srv.submit_forward(gp, u0=u0, L=r.L) if r.kind == 0 else
                 srv.submit_band_gradient(gp, r.phase, u0=u0, L=r.L))
            outstanding.append(h)
            i += 1
        still = []
        for h in outstanding:
            try:
                if not srv.poll(h):
                    still.append(h)
                    continue
                statuses[0] = statuses.get(0, 0) + 1
                lat.append(h.latency_ms)
            except FiberLabGPUError as e:
                statuses[e.status] = statuses.get(e.status, 0) + 1
        outstanding = still
        time.sleep(0.0005)
    wall = min(time.perf_counter() - t0, window_s)
    info = srv.info()
    srv.close()
    done = statuses.get(0, 0)
    served = {"window_s": window_s, "completed": done, "solves_per_s": done / wall,
              **_quantiles(lat), "unfinished": i - sum(statuses.values()),
              "failed_by_status": {str(k): v for k, v in statuses.items() if k != 0},
              "slots": info["slots"], "hbm_bytes": info["hbm_bytes"]}

    # the plain path in a child process, stopped between requests at the
    # window's end (a request still running then is waited for, up to a bound)
    mpc = mp.get_context("spawn")
    q, stop = mpc.Queue(), mpc.Event()
    child = mpc.Process(target=_plain_worker, args=(q, stop, dev_index, n, seed, plain_window_s),
                        daemon=True)
    child.start()
    pst, plat = {}, []
    try:
        q.get(timeout=600)                         # the child's "start"
        ended = False
    except Exception:
        ended = True                               # the child did not start: no plain number
    t_start = time.perf_counter()
    while not ended:
        left = plain_window_s - (time.perf_counter() - t_start)
        if left <= 0 and not stop.is_set():
            stop.set()
        try:
            msg = q.get(timeout=max(0.05, min(left, 1.0)) if left > 0 else 60.0)
        except Exception:                          # nothing finished meanwhile
            if left > 0:
                continue
            break                                  # a request outlived the grace period
        if msg[0] == "end":
            ended = True
        elif msg[0] == "done":
            _, idx, status, fin, latency = msg
            if fin <= plain_window_s:
                pst[status] = pst.get(status, 0) + 1
                if status == 0:
                    plat.append(1e3 * latency)
    if child.is_alive():
        child.join(timeout=5)
    if child.is_alive():
        child.terminate()
        child.join(timeout=30)
    arrived = sum(1 for r in reqs if r.arrival_s <= plain_window_s)
    pdone = pst.get(0, 0)
    plain = {"window_s": plain_window_s, "completed": pdone,
             "solves_per_s": pdone / plain_window_s, **_quantiles(plat),
             "unfinished": arrived - sum(pst.values()),
             "failed_by_status": {str(k): v for k, v in pst.items() if k != 0}}
    return {"requests": n, "mix": SERVE_MIX, "served": served, "plain_one_at_a_time": plain,
            "served_over_plain": (served["solves_per_s"] / plain["solves_per_s"]
                                  if plain["solves_per_s"] > 0 else None)}


def optimizer_measure(ctx, B, probes, iters):
    """The inverse-design consumer of the batched gradient: B independent
    L-BFGS optimisations of the headline problem's phase (dB band objective
    with the reference's default GDD weight 1e-4), each line search one
    batched forward + adjoint launch over B x probes trial phases.  Reports
    accepted iterations per second over all B problems, the cost/gradient
    evaluations per second behind them, and the median improvement."""
    import torch
    from fiberlab_gpu import optimize as OP
    from fiberlab_gpu._capi import GPUProblem
    fp = workload_problem()
    gp = GPUProblem(ctx, fp)
    x0 = phases(77, B, fp.nt)
    obj = OP.BandPhaseObjective(gp, log_cost=True, lambda_gdd=1e-4)
    # warm-up at the line-search batch size (workspace allocation outside the timing)
    obj(torch.from_numpy(np.repeat(x0, probes, axis=0)).to(obj.device))
    solves0 = obj.solves
    J0, _ = obj(torch.from_numpy(x0).to(obj.device))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = OP.lbfgs(obj, torch.from_numpy(x0).to(obj.device), max_iter=iters, f_abstol=None,
                   probes=probes)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    gain = (J0 - res.J).cpu().numpy()
    return {"workload": f"{B} L-BFGS optimisations of the headline problem (dB band + GDD 1e-4),"
                        f" {probes} trial steps per line search, {iters} iterations",
            "iterations_per_s": float(res.iterations.sum()) / dt,
            "solves_per_s": (obj.solves - solves0 - B) / dt,
            "ms_per_iteration": 1e3 * dt / max(1, int(res.iterations.max())),
            "median_db_improvement": float(np.median(gain)),
            "line_search_launches": int(res.evaluations - 1)}


def multimode_measure(ctx, dev, B, steps, warmup):
    """Config 4: B per-mode phase candidates φ ~ N(0, 1) (seeded) of the M = 10
    HG(m+n<=3) problem on a 96x96 grid, Nt = 2^14 over 10 ps, L = 2 m, 5 nJ,
    forward + band objective (red side beyond 2 THz) + adjoint + per-mode
    gradient, one batched call on device buffers; and config 2 (M = 6,
    Nt = 2^12 over 5 ps, 1 m, 2 nJ), one forward + adjoint."""
    import torch
    from fiberlab_gpu import problem as P
    from fiberlab_gpu._capi import Context, GPUProblem
    out = {}
    fp = P.multimode_problem(3, 96, 16384, 10.0, 2.0, 5e-9, 200e-15, seed=0,
                             raman_threshold_thz=-2.0)
    # a dense-output buffer of 160 steps holds these solves (~120 forward
    # steps) whole: the adjoint recomputes nothing (820 MB per candidate)
    ctx = Context(ctx.device, checkpoints=32, segment_steps=160)
    gp = GPUProblem(ctx, fp)
    ph = np.random.default_rng(4).standard_normal((B, fp.M, fp.nt))
    d_u0 = torch.from_numpy(np.ascontiguousarray(fp.uw0).view(np.float64).copy()).to(dev)
    d_ph = torch.from_numpy(ph).to(dev)
    d_m = torch.from_numpy(fp.mask.astype(np.uint8)).to(dev)
    d_J = torch.empty(B, dtype=torch.float64, device=dev)
    d_g = torch.empty((B, fp.M, fp.nt), dtype=torch.float64, device=dev)
    run = lambda: gp.mode_phase_gradient_batch_device(d_u0.data_ptr(), B, d_ph.data_ptr(),
                                                     d_m.data_ptr(), d_J.data_ptr(),
                                                     d_g.data_ptr())
    for _ in range(warmup):
        run()
    ms, st = [], None
    for _ in range(steps):
        st = run()
        ms.append(ctx.timing()[0])
    M, N = fp.M, fp.nt
    fwd_att = sum(s["naccept"] + s["nreject"] for s in st)
    rec = sum(s["recompute_steps"] for s in st)
    adj_att = sum(s["adj_naccept"] + s["adj_nreject"] for s in st)
    t_batch = float(np.mean(ms)) / 1e3
    # roofline bytes per attempted step: 336 N M (forward and recompute), 384 N M (adjoint)
    alg_bytes = (BYTES_FWD_STEP * (fwd_att + rec) + BYTES_ADJ_STEP * adj_att) * N * M
    peak, peak_kind = measured_peak()
    # tensor-pipe work on tcgen05 kind::tf32 (unpadded GEMM flops, 6 RHS per
    # attempted step), with the rank r of the overlap Gram matrix (the library
    # drops eigenvalues below 1e-12 of the largest): per forward RHS the
    # reduction Z = Vᵀ P (2 NP r N) and the contraction U S̃ over all M² rows
    # (2 M² r N); per adjoint RHS the reductions of Y, D' = U S̃', C = U Cz
    # (2 NP r N each) and W = G w (2 * 2 NP² N)
    NP = M * (M + 1) // 2
    pairs = [(k, l) for k in range(M) for l in range(k, M)]
    gam = np.array([[fp.gamma[i, j, k, l] for (k, l) in pairs] for (i, j) in pairs])
    ev = np.abs(np.linalg.eigvalsh(gam))
    r = int(np.sum(ev > 1e-12 * ev.max()))
    tc_flops = ((2 * NP * r + 2 * M * M * r) * N * 6 * (fwd_att + rec)
                + (3 * 2 * NP * r + 4 * NP * NP) * N * 6 * adj_att)
    out["config4"] = {
        "workload": f"config 4: M=10 HG(m+n<=3), Nt=2^14 over 10 ps, L=2 m, 5 nJ, {B} per-mode "
                    "phase candidates N(0,1), fwd+adjoint, 160 dense-output steps",
        "solves_per_s": B * steps / (sum(ms) / 1e3), "ms_per_batch": float(np.mean(ms)),
        "steps_per_solve": {"forward": fwd_att / B, "adjoint": adj_att / B,
                            "recomputed": rec / B},
        "roofline": {"bound": "hbm", "achieved": alg_bytes / t_batch / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": alg_bytes / t_batch / 1e9 / peak,
                     "peak_source": peak_kind, "alg_bytes_per_batch": alg_bytes,
                     "scope": "whole batch (all multimode kernels) over its call time"},
        "tensor": {"flops_per_batch": tc_flops,
                   "achieved_tflops_over_batch": tc_flops / t_batch / 1e12,
                   "gram_rank": r,
                   "note": "the low-rank reductions and contractions and the adjoint's W GEMMs "
                           "(unpadded flops); 3 tf32 MMAs per product (3xTF32 split)"},
        "precision": "FP32 forward; mixed adjoint: lambda, its transforms and the sums over "
                     "modes FP64, the forward field's transform and pair products FP32, "
                     "per-point contractions 3xTF32",
        "contraction": "tcgen05 kind::tf32 (3xTF32), low-rank form G = U V^T of the overlap "
                       "Gram matrix: Z = V^T P, D = U S~, the adjoint's D', C = U Cz and "
                       "W = G u_k u_l on the symmetric pair image"}
    fp2 = P.multimode_problem(2, 64, 4096, 5.0, 1.0, 2e-9, 200e-15, seed=0,
                              raman_threshold_thz=-2.0)
    gp2 = GPUProblem(ctx, fp2)
    lat = []
    for i in range(4):
        t = time.perf_counter()
        gp2.phase_gradient_batch(np.zeros((1, fp2.nt)))
        if i:
            lat.append(1e3 * (time.perf_counter() - t))
    out["config2"] = {"workload": "config 2: M=6 HG(m+n<=2), Nt=2^12 over 5 ps, L=1 m, 2 nJ, "
                                  "one fwd+adjoint per call (host buffers)",
                      "latency_ms_p50": float(np.median(lat))}
    return out


def max_over_ranks(value: float, device=None) -> float:
    """The job's time: the maximum of a per-rank value over all ranks (one
    all-reduce; the identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def init_dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args):
    world, rank, local = init_dist()
    if rank != 0:
        return
    fp = workload_problem()
    cores = os.cpu_count() or 1
    nprob = max(cores, 8)
    for _ in range(args.warmup):
        cpu_baseline(fp, cores, cores)
    times, done = [], 0
    for _ in range(args.steps):
        _, dt = cpu_baseline(fp, cores, nprob)
        times.append(dt)
        done += nprob
    value = done / sum(times)
    sample = f"{nprob} problems per step (one per thread, {cores} threads)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(nprob, 1, {"implementation": "FP64 C restatement of the reference "
                                        "Julia solver (Julia is not installed), OpenMP over "
                                        "independent problems"},
                             precision="FP64 throughout"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample, "cpu_model": cpu_model(),
                             "fft": ORACLE_FFT},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    world, rank, local = init_dist()
    import torch
    import torch.distributed as dist
    from fiberlab_gpu._capi import Context, GPUProblem

    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = Context(local, checkpoints=32, segment_steps=64)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    B = args.batch or 4 * sms
    fp = workload_problem()
    gp = GPUProblem(ctx, fp, "fp32")
    ph_host = phases(rank, B, fp.nt)
    d_u0 = torch.from_numpy(np.ascontiguousarray(fp.uw0).view(np.float64).copy()).to(dev)
    d_ph = torch.from_numpy(ph_host).to(dev)
    d_mask = torch.from_numpy(fp.mask.astype(np.uint8)).to(dev)
    d_J = torch.empty(B, dtype=torch.float64, device=dev)
    d_g = torch.empty((B, fp.nt), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        return gp.phase_gradient_batch_device(d_u0.data_ptr(), B, d_ph.data_ptr(),
                                              d_mask.data_ptr(), d_J.data_ptr(), d_g.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    launches0 = ctx.launches
    call_ms, kern_ms, stats_all = [], [], []
    for _ in range(args.steps):
        flush.zero_()                      # L2 flush between timed iterations (not timed)
        torch.cuda.synchronize(dev)
        st = step()                        # synchronises the context stream
        c, k = ctx.timing()
        call_ms.append(c)
        kern_ms.append(k)
        stats_all.append(st)
    torch.cuda.synchronize(dev)
    launches = ctx.launches - launches0
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    t_rank = sum(call_ms)
    t_job = max_over_ranks(t_rank, dev)
    value = B * args.steps * world / (t_job / 1e3)

    # roofline of the stepper kernel: algorithmic bytes per launch / launch time
    st = stats_all[-1]
    fwd_att = sum(s["naccept"] + s["nreject"] for s in st)
    rec = sum(s["recompute_steps"] for s in st)   # forward steps the adjoint recomputed
    adj_att = sum(s["adj_naccept"] + s["adj_nreject"] for s in st)
    alg_bytes = (BYTES_FWD_STEP * (fwd_att + rec) + BYTES_ADJ_STEP * adj_att) * fp.nt
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / (kern_ms[-1] / 1e3) / 1e9
    tr = profiled_traffic()
    traffic = None
    if tr and tr.get("bytes_per_attempted_step"):
        traffic = tr["bytes_per_attempted_step"] * (fwd_att + adj_att)

    # end to end through the public host API: page-locked host buffers,
    # the library's host->device and device->host copies inside the call
    pin_ph = torch.from_numpy(ph_host).pin_memory()
    pin_J = torch.empty(B, dtype=torch.float64).pin_memory()
    pin_g = torch.empty((B, fp.nt), dtype=torch.float64).pin_memory()
    gp.phase_gradient_batch(pin_ph.numpy(), fp.mask, fp.uw0,
                            out=(pin_J.numpy(), pin_g.numpy()))   # warm-up (staging area)
    e2e_t = []
    for _ in range(args.steps):
        flush.zero_()                      # L2 flush between timed iterations (not timed)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        gp.phase_gradient_batch(pin_ph.numpy(), fp.mask, fp.uw0,
                                out=(pin_J.numpy(), pin_g.numpy()))
        e2e_t.append(time.perf_counter() - t0)
    e2e_value = B * world / max(np.mean(e2e_t), 1e-12)
    h2d = ph_host.nbytes + fp.uw0.nbytes + fp.mask.nbytes
    d2h = B * 8 + B * fp.nt * 8

    # plain one-at-a-time drop-in (same solve, one problem per call)
    plain_lat = []
    for b in range(args.plain):
        t0 = time.perf_counter()
        gp.phase_gradient_batch(ph_host[b:b + 1], fp.mask, fp.uw0)
        plain_lat.append(time.perf_counter() - t0)
    plain = {"solves_per_s": 1.0 / float(np.mean(plain_lat)),
             "latency_ms_p50": 1e3 * float(np.percentile(plain_lat, 50)),
             "latency_ms_p99": 1e3 * float(np.percentile(plain_lat, 99))}
    batched_lat = {"latency_ms_p50": float(np.percentile(call_ms, 50)),
                   "latency_ms_p99": float(np.percentile(call_ms, 99))}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = os.cpu_count() or 1
        v, dt = cpu_baseline(fp, cores, cores)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{cores} problems of this workload, one per thread ({dt:.1f} s)",
               "cpu_model": cpu_model(), "fft": ORACLE_FFT}

    multimode = None
    if args.mm_batch and rank == 0 and world == 1:
        multimode = multimode_measure(ctx, dev, args.mm_batch, min(args.steps, 3), 1)

    optimizer = None
    if args.opt_batch and rank == 0 and world == 1:
        optimizer = optimizer_measure(ctx, args.opt_batch, args.opt_probes, args.opt_iters)

    serving = None
    if args.serve and rank == 0 and world == 1:
        serving = serving_measure(Context, local, args.serve, args.serve_window,
                                  args.serve_plain_window)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": t_job / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config(B, world),
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h)},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                             "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                             "peak_source": peak_kind,
                             "kernel": "sm_advance_kernel<float,13,4>",
                             "alg_bytes_per_launch": alg_bytes},
                "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clocks,
                "plain_one_at_a_time": plain, "batched": batched_lat,
                "steps_per_solve": {"forward": fwd_att / B, "adjoint": adj_att / B,
                                    "recomputed": rec / B}}
        if multimode is not None:
            line.update(multimode)
        if optimizer is not None:
            line["inverse_design"] = optimizer
        if serving is not None:
            line["serving"] = serving
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=0, help="problems per GPU (default 4 x SMs)")
    ap.add_argument("--plain", type=int, default=32, help="one-at-a-time solves timed")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mm-batch", type=int, default=64,
                    help="config-4 candidates per batch reported beside the headline (0: off)")
    ap.add_argument("--opt-batch", type=int, default=148,
                    help="L-BFGS optimisations run in lockstep beside the headline (0: off)")
    ap.add_argument("--opt-probes", type=int, default=4, help="trial steps per line search")
    ap.add_argument("--opt-iters", type=int, default=3, help="L-BFGS iterations timed")
    ap.add_argument("--serve", type=int, default=4096,
                    help="requests of the config-3 serving stream (0: off)")
    ap.add_argument("--serve-window", type=float, default=30.0,
                    help="seconds the server takes the stream for")
    ap.add_argument("--serve-plain-window", type=float, default=60.0,
                    help="seconds the plain one-at-a-time path takes the same stream for")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
