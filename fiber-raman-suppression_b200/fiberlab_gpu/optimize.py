"""Spectral-phase inverse design: L-BFGS over the GPU cost and gradient.

The reference optimises one phase at a time with Optim.jl's L-BFGS around
`cost_and_gradient` (scripts/lib/raman_optimization.jl:102-246: shaped launch,
forward, Raman-band cost, adjoint, ∂J/∂φ, then the GDD and boundary
regularisers of scripts/lib/regularizers.jl:28-142 and the dB surface).

Here B independent optimisations run in lockstep with their state on the
device: the phases, gradients and L-BFGS history are (B, ...) device tensors,
and every iteration evaluates P trial step lengths per problem along its
search direction as ONE batched forward + adjoint call over B·P problems
(`fl_phase_gradient_batch_device`), so a line search costs one launch of the
stepper instead of a sequence of solves.  The vector algebra of the two-loop
recursion and the step selection are batched tensor operations.

Line search: the P trial lengths are a0·ρ^k (k = 0..P-1, ρ = 1/4).  The
longest trial satisfying the strong Wolfe conditions (Armijo c1 = 1e-4,
curvature c2 = 0.9) is taken; failing that, the lowest-cost trial that
satisfies Armijo; failing that, the next P shorter lengths are tried (up to
`retries` times) before the problem stops with `line_search_failed`.  a0 is 1
after the first iteration (the history scales the direction by s·y / y·y),
and 1/‖g‖₂ on the first.  Stopping follows the reference's options: f_abstol
on the change of J (0.01 dB with the dB surface, 1e-10 linear), g_abstol on
‖g‖∞ (1e-8), and max_iter.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np
import torch

from . import problem as P
from ._capi import GPUProblem

# ---------------------------------------------------------------------------
# Regularisers (scripts/lib/regularizers.jl), batched over leading axes; the
# time/frequency axis is the last one (the reference's rows).


def gdd_penalty(phi: torch.Tensor, dt: float, lam: float):
    """Σ λ (φ[i+1] - 2φ[i] + φ[i-1])² / Δω³ over the interior of the
    fftshift-ed (centred) phase, Δω = 2π / (Nt Δt) (regularizers.jl:28-60).
    phi (..., Nt) -> (J (...), ∂J/∂φ (..., Nt))."""
    if lam <= 0:
        return phi.new_zeros(phi.shape[:-1]), torch.zeros_like(phi)
    if not (math.isfinite(dt) and dt > 0):
        raise P.ArgumentError("Δt must be positive and finite")
    nt = phi.shape[-1]
    inv_dw3 = 1.0 / (2 * math.pi / (nt * dt)) ** 3
    c = torch.fft.fftshift(phi, dim=-1)
    d2 = c[..., 2:] - 2 * c[..., 1:-1] + c[..., :-2]
    J = lam * inv_dw3 * torch.sum(d2 * d2, dim=-1)
    coeff = 2 * lam * inv_dw3 * d2
    g = torch.zeros_like(c)
    g[..., :-2] += coeff
    g[..., 1:-1] -= 2 * coeff
    g[..., 2:] += coeff
    return J, torch.fft.ifftshift(g, dim=-1)


def boundary_phase_penalty(u_shaped: torch.Tensor, lam: float, shared: bool = True,
                           floor: float = 1e-8):
    """λ × (energy of the shaped input in the first and last max(1, Nt÷20)
    time samples) / (total), with its gradient with respect to the phase
    (regularizers.jl:72-130).  u_shaped (..., M, Nt) complex; the gradient is
    (..., Nt) summed over modes when shared (one phase for all modes), else
    (..., M, Nt).  Zero below the edge-fraction floor."""
    lead = u_shaped.shape[:-2]
    nt = u_shaped.shape[-1]
    gshape = lead + ((nt,) if shared else u_shaped.shape[-2:])
    zeroJ = torch.zeros(lead, dtype=torch.float64, device=u_shaped.device)
    if lam <= 0:
        return zeroJ, torch.zeros(gshape, dtype=torch.float64, device=u_shaped.device)
    n_edge = max(1, nt // 20)
    ut = torch.fft.fft(u_shaped, dim=-1)
    mask = torch.zeros(nt, dtype=torch.float64, device=u_shaped.device)
    mask[:n_edge] = 1.0
    mask[nt - n_edge:] = 1.0
    p = ut.real ** 2 + ut.imag ** 2
    total = torch.clamp(torch.sum(p, dim=(-2, -1)), min=float(np.finfo(float).eps))
    frac = torch.sum(p * mask, dim=(-2, -1)) / total
    coeff = (2 * lam * nt / total)[..., None, None]
    g = coeff * torch.imag(torch.conj(u_shaped) * torch.fft.ifft(ut * mask, dim=-1))
    on = frac > floor
    g = g * on[..., None, None]
    if shared:
        g = torch.sum(g, dim=-2)
    return lam * frac * on, g


def apply_log_surface(J: torch.Tensor, grad: torch.Tensor):
    """10 log10(max(J, 1e-15)) and the gradient scaled by its derivative
    (regularizers.jl:132-142)."""
    Jc = torch.clamp(J, min=1e-15)
    return 10.0 * torch.log10(Jc), grad * (10.0 / (Jc * math.log(10.0)))[..., None]


# ---------------------------------------------------------------------------
# The batched objective on the device


class BandPhaseObjective:
    """Regularised field objective of one problem for a batch of shared
    phases: phis (K, Nt) float64 on the device -> J (K,), ∂J/∂φ (K, Nt), with
    every forward + adjoint of the K phases in one batched launch
    (cost_and_gradient, raman_optimization.jl:102-177).  The objective is the
    Raman band by default, or any objective with a device seed
    (GPUProblem.set_objective: fundamental_mode, worst_mode, raman_peak);
    constructing it sets that objective on the problem."""

    def __init__(self, gp: GPUProblem, *, log_cost: bool = True, lambda_gdd: float = 0.0,
                 lambda_boundary: float = 0.0, device=None, objective: str = "raman_band",
                 worst_mode_tau: float = 50.0):
        fp = gp.fp
        if fp.mask is None or not np.any(fp.mask):
            raise P.ArgumentError("band mask must contain at least one bin")
        for name, v in (("lambda_gdd", lambda_gdd), ("lambda_boundary", lambda_boundary)):
            if not (math.isfinite(v) and v >= 0):
                raise P.ArgumentError(f"regularizer `{name}` lambda must be nonnegative and finite")
        self.gp, self.fp = gp, fp
        gp.set_objective(objective, worst_mode_tau)
        self.log_cost = log_cost
        self.lambda_gdd, self.lambda_boundary = float(lambda_gdd), float(lambda_boundary)
        self.device = torch.device(device or f"cuda:{gp.ctx.device}")
        self.u0 = torch.from_numpy(np.ascontiguousarray(fp.uw0)).to(self.device)
        self.u0_real = torch.view_as_real(self.u0).contiguous()
        self.mask = torch.from_numpy(fp.mask.astype(np.uint8)).to(self.device)
        self.calls = 0
        self.solves = 0

    def __call__(self, phis: torch.Tensor):
        K, nt = phis.shape
        phis = phis.contiguous()
        J = torch.empty(K, dtype=torch.float64, device=self.device)
        g = torch.empty((K, nt), dtype=torch.float64, device=self.device)
        # the library runs on its own stream: order it after torch's writes
        # and torch's reads after it
        torch.cuda.current_stream(self.device).synchronize()
        self.gp.phase_gradient_batch_device(self.u0_real.data_ptr(), K, phis.data_ptr(),
                                            self.mask.data_ptr(), J.data_ptr(), g.data_ptr(),
                                            log_cost=False, with_stats=False)
        self.gp.ctx.synchronize()
        self.calls += 1
        self.solves += K
        if self.lambda_gdd > 0:
            Jr, gr = gdd_penalty(phis, float(self.fp.sim["Δt"]), self.lambda_gdd)
            J, g = J + Jr, g + gr
        if self.lambda_boundary > 0:
            shaped = self.u0[None] * torch.exp(1j * phis)[:, None, :]
            Jr, gr = boundary_phase_penalty(shaped, self.lambda_boundary, shared=True)
            J, g = J + Jr, g + gr
        if self.log_cost:
            J, g = apply_log_surface(J, g)
        return J, g


# ---------------------------------------------------------------------------
# Batched L-BFGS


@dataclass
class LBFGSResult:
    x: torch.Tensor                 # (B, N) final phases
    J: torch.Tensor                 # (B,) final costs
    g: torch.Tensor                 # (B, N) final gradients
    iterations: np.ndarray          # (B,) accepted iterations
    status: list                    # per problem: converged_f / converged_g / max_iter / line_search_failed
    trace: list = field(default_factory=list)   # J (B,) after every iteration
    evaluations: int = 0            # batched objective calls
    solves: int = 0                 # cost/gradient evaluations (problems x probes)


def lbfgs(fg: Callable, x0: torch.Tensor, *, max_iter: int = 50, f_abstol: float = 0.01,
          g_abstol: float = 1e-8, memory: int = 10, probes: int = 8, shrink: float = 0.25,
          c1: float = 1e-4, c2: float = 0.9, retries: int = 3) -> LBFGSResult:
    """Minimise B independent objectives in lockstep.  fg maps a (K, N)
    tensor of points to (J (K,), g (K, N)); every call evaluates all active
    problems' trial points at once."""
    if max_iter < 1:
        raise P.ArgumentError("max_iter must be positive")
    if probes < 1 or not (0 < shrink < 1):
        raise P.ArgumentError("probes must be >= 1 and shrink in (0, 1)")
    x = x0.detach().clone().to(torch.float64)
    B, N = x.shape
    dev = x.device
    J, g = fg(x)
    calls, solves = 1, B
    S = torch.zeros((memory, B, N), dtype=torch.float64, device=dev)
    Y = torch.zeros_like(S)
    rho = torch.zeros((memory, B), dtype=torch.float64, device=dev)
    used = torch.zeros(B, dtype=torch.long, device=dev)     # history entries per problem
    head = 0                                                 # ring position (shared)
    iters = np.zeros(B, dtype=np.int64)
    status = [None] * B
    active = torch.ones(B, dtype=torch.bool, device=dev)
    trace = []
    if g_abstol is not None:
        for b in torch.nonzero(torch.amax(torch.abs(g), dim=1) <= g_abstol).flatten().tolist():
            status[b], active[b] = "converged_g", False
    ks = shrink ** torch.arange(probes, dtype=torch.float64, device=dev)
    for _ in range(max_iter):
        idx = torch.nonzero(active).flatten()
        if idx.numel() == 0:
            break
        A = idx.numel()
        xa, ga, Ja = x[idx], g[idx], J[idx]
        # two-loop recursion over the ring (newest first); entries a problem
        # has not filled have rho = 0 and drop out
        q = -ga.clone()
        alphas = []
        for j in range(memory):
            r = (head - 1 - j) % memory
            a = rho[r, idx] * torch.sum(S[r, idx] * q, dim=1)
            q -= a[:, None] * Y[r, idx]
            alphas.append((r, a))
        # initial inverse-Hessian scale s·y / y·y from the newest pair (1
        # where the newest slot holds none for a problem)
        rn = (head - 1) % memory
        sy = torch.sum(S[rn, idx] * Y[rn, idx], dim=1)
        yy = torch.sum(Y[rn, idx] * Y[rn, idx], dim=1)
        gamma = torch.where(rho[rn, idx] > 0, sy / torch.clamp(yy, min=1e-300),
                            torch.ones_like(sy))
        q *= gamma[:, None]
        for r, a in reversed(alphas):
            bcoef = rho[r, idx] * torch.sum(Y[r, idx] * q, dim=1)
            q += (a - bcoef)[:, None] * S[r, idx]
        d = q
        slope = torch.sum(ga * d, dim=1)
        # not a descent direction (round-off in the history): restart from -g
        bad = slope >= 0
        if torch.any(bad):
            d[bad] = -ga[bad]
            slope = torch.sum(ga * d, dim=1)
            used[idx[bad]] = 0
            rho[:, idx[bad]] = 0
        a0 = torch.where(used[idx] > 0, torch.ones_like(slope),
                         1.0 / torch.clamp(torch.linalg.vector_norm(ga, dim=1), min=1e-300))
        chosen = torch.full((A,), -1, dtype=torch.long, device=dev)
        xn, Jn, gn = xa.clone(), Ja.clone(), ga.clone()
        pending = torch.ones(A, dtype=torch.bool, device=dev)
        for _t in range(retries + 1):
            pidx = torch.nonzero(pending).flatten()
            if pidx.numel() == 0:
                break
            alpha = a0[pidx, None] * ks[None, :]                         # (A', P)
            trial = xa[pidx, None, :] + alpha[..., None] * d[pidx, None, :]
            Jt, gt = fg(trial.reshape(-1, N))
            calls += 1
            solves += trial.shape[0] * probes
            Jt = Jt.reshape(-1, probes)
            gt = gt.reshape(-1, probes, N)
            s0 = slope[pidx, None]
            armijo = torch.isfinite(Jt) & (Jt <= Ja[pidx, None] + c1 * alpha * s0)
            wolfe = armijo & (torch.abs(torch.sum(gt * d[pidx, None, :], dim=2)) <= c2 * torch.abs(s0))
            # the longest Wolfe trial, else the lowest-cost Armijo trial
            kw = torch.argmax(wolfe.to(torch.int8), dim=1)       # first True (longest step)
            ka = torch.argmin(torch.where(armijo, Jt, torch.full_like(Jt, math.inf)), dim=1)
            k = torch.where(wolfe.any(dim=1), kw, ka)
            got = armijo.any(dim=1)
            rows = torch.arange(pidx.numel(), device=dev)
            sel = pidx[got]
            chosen[sel] = k[got]
            xn[sel] = trial[rows[got], k[got]]
            Jn[sel] = Jt[rows[got], k[got]]
            gn[sel] = gt[rows[got], k[got]]
            pending[sel] = False
            a0[pidx] = a0[pidx] * shrink ** probes
        ok = chosen >= 0
        # history update (shared ring slot; problems that did not move keep rho = 0 there)
        s_new = xn - xa
        y_new = gn - ga
        sy_new = torch.sum(s_new * y_new, dim=1)
        keep = ok & (sy_new > 1e-12 * torch.linalg.vector_norm(s_new, dim=1)
                     * torch.linalg.vector_norm(y_new, dim=1))
        S[head, idx] = torch.where(keep[:, None], s_new, torch.zeros_like(s_new))
        Y[head, idx] = torch.where(keep[:, None], y_new, torch.zeros_like(y_new))
        rho[head, idx] = torch.where(keep, 1.0 / torch.where(keep, sy_new, torch.ones_like(sy_new)),
                                     torch.zeros_like(sy_new))
        used[idx] = torch.where(keep, torch.clamp(used[idx] + 1, max=memory), used[idx])
        head = (head + 1) % memory
        x[idx], g[idx] = xn, gn
        dJ = torch.abs(Jn - Ja)
        J[idx] = Jn
        for i, b in enumerate(idx.tolist()):
            if not bool(ok[i]):
                status[b], active[b] = "line_search_failed", False
                continue
            iters[b] += 1
            if f_abstol is not None and float(dJ[i]) <= f_abstol:
                status[b], active[b] = "converged_f", False
            elif g_abstol is not None and float(torch.amax(torch.abs(gn[i]))) <= g_abstol:
                status[b], active[b] = "converged_g", False
        trace.append(J.detach().clone())
    for b in range(B):
        if status[b] is None:
            status[b] = "max_iter"
    return LBFGSResult(x=x, J=J, g=g, iterations=iters, status=status, trace=trace,
                       evaluations=calls, solves=solves)


def optimize_spectral_phase(gp: GPUProblem, phi0=None, *, batch: int = 1, max_iter: int = 50,
                            log_cost: bool = True, lambda_gdd: float = 0.0,
                            lambda_boundary: float = 0.0, f_abstol=None, g_abstol=1e-8,
                            probes: int = 8, memory: int = 10, seed: Optional[int] = None):
    """optimize_spectral_phase (raman_optimization.jl:183-246) for `batch`
    independent starting phases at once.  phi0: (batch, Nt) or (Nt,) or None
    (zero phase; with batch > 1 and a seed, N(0, 0.5²) starts for the others).
    f_abstol defaults to the reference's 0.01 dB (log_cost) or 1e-10 (linear)."""
    fp = gp.fp
    obj = BandPhaseObjective(gp, log_cost=log_cost, lambda_gdd=lambda_gdd,
                             lambda_boundary=lambda_boundary)
    if phi0 is None:
        x0 = np.zeros((batch, fp.nt))
        if seed is not None and batch > 1:
            x0[1:] = 0.5 * np.random.default_rng(seed).standard_normal((batch - 1, fp.nt))
    else:
        x0 = np.atleast_2d(np.asarray(phi0, dtype=np.float64))
        if x0.shape[1] != fp.nt:
            raise P.ArgumentError(f"phase length {x0.shape[1]} does not match Nt={fp.nt}")
    if not np.all(np.isfinite(x0)):
        raise P.ArgumentError("phase contains NaN/Inf")
    if f_abstol is None:
        f_abstol = 0.01 if log_cost else 1e-10
    res = lbfgs(obj, torch.from_numpy(x0).to(obj.device), max_iter=max_iter, f_abstol=f_abstol,
                g_abstol=g_abstol, memory=memory, probes=probes)
    res.solves = obj.solves
    return res
