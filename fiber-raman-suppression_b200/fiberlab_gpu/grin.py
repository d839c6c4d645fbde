"""Graded-index (GRIN) multimode fiber setup: index profile, scalar mode
solver, dispersion from finite differences of β(f) and the Kerr tensor from
the mode overlaps.  One-time host setup (FP64) whose outputs -- D (M, Nt) and
γ (M, M, M, M) -- are the tables a multimode problem hands to the GPU.

Restated from src/simulation/fibers.jl:1-222 (build_GRIN, get_params,
solve_for_fiber_modes, compute_overlap_tensor) and the GRIN branch of
get_disp_fiber_params (src/helpers/helpers.jl:181-214).  The reference's
eigen solver is ARPACK (`eigs(A; which=:LR)`) and its finite-difference
weights come from FiniteDifferences.jl's `central_fdm`; both are third-party
and restated here from their published definitions (the largest eigenpairs
of the symmetric 5-point operator; the weights of the unique polynomial
rule on the symmetric stencil).  Modes within a degenerate group (LP11a/b
and the like) are any orthonormal basis of that group, in the reference as
here, so the eigenvalues, β(f) and basis-invariant sums are what compare.
"""
from __future__ import annotations

import math

import numpy as np

from . import problem as P

SELLMEIER_SILICA = ((0.6961663, 0.0684043), (0.4079426, 0.1162414), (0.8974794, 9.896161))


def silica_index(lam_um: float) -> float:
    """Fused-silica refractive index from the three-term Sellmeier equation
    (fibers.jl:28-54)."""
    l2 = lam_um * lam_um
    return math.sqrt(1 + sum(a * l2 / (l2 - b * b) for a, b in SELLMEIER_SILICA))


def build_grin(lam_um: float, nx: int, window_um: float, radius_um: float, core_na: float,
               alpha: float):
    """ε = n² of n(r) = max(n_cl, n_co - (n_co - n_cl)(r/a)^α) on an nx × nx
    grid, x = (-nx/2 .. nx/2-1)·dx (fibers.jl:28-54).  Returns (eps, x, dx)."""
    nco = silica_index(lam_um)
    ncl = math.sqrt(nco * nco - core_na * core_na)
    dx = window_um / nx
    x = np.arange(-nx / 2, nx / 2) * dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    r = np.sqrt(X * X + Y * Y)
    eps = np.maximum(ncl, nco - (nco - ncl) * (r / radius_um) ** alpha) ** 2
    return eps, x, dx


def mode_operator(lam_um: float, dx: float, eps: np.ndarray):
    """The sparse 5-point operator A = ∇² + ε k² (Dirichlet outside the grid)
    of the scalar wave equation A ψ = β² ψ (fibers.jl:159-197), with the
    unknowns in column-major order (index i + nx·j)."""
    import scipy.sparse as sp
    nx, ny = eps.shape
    k2 = (2 * math.pi / lam_um) ** 2
    c = 1.0 / (dx * dx)
    ex = sp.diags([np.full(nx - 1, c), np.full(nx - 1, c)], [-1, 1], shape=(nx, nx))
    ey = sp.diags([np.full(ny - 1, c), np.full(ny - 1, c)], [-1, 1], shape=(ny, ny))
    off = sp.kron(sp.identity(ny), ex) + sp.kron(ey, sp.identity(nx))
    diag = eps.reshape(-1, order="F") * k2 - 4 * c
    return (off + sp.diags(diag)).tocsr()


def solve_fiber_modes(lam_um: float, nmodes: int, dx: float, eps: np.ndarray):
    """The nmodes most-bound scalar modes (largest β²) of the GRIN profile
    (solve_for_fiber_modes, fibers.jl:159-197): returns (β² [µm⁻²],
    unit-norm profiles (nx·ny, nmodes) in column-major order, neff), sorted by
    decreasing β²."""
    from scipy.sparse.linalg import eigsh
    A = mode_operator(lam_um, dx, eps)
    n = A.shape[0]
    if not (1 <= nmodes < n - 1):
        raise P.ArgumentError("number of modes must be at least 1 and below the grid size")
    d, v = eigsh(A, k=nmodes, which="LA", tol=1e-13, maxiter=100000)
    order = np.argsort(-d)
    d, v = d[order], v[:, order]
    return d, v, lam_um * np.sqrt(d) / (2 * math.pi)


def central_fd_weights(points: int, order: int) -> np.ndarray:
    """Weights c_k, k = -(p-1)/2 .. (p-1)/2, of the order-th derivative at 0
    from the unique degree-(p-1) polynomial through the symmetric stencil of
    unit spacing: Σ c_k k^m = m! δ(m, order), m = 0 .. p-1."""
    if points % 2 == 0 or points <= order:
        raise P.ArgumentError("central stencil needs an odd number of points above the order")
    k = np.arange(points) - (points - 1) // 2
    V = np.vander(k, points, increasing=True).T.astype(np.float64)
    rhs = np.zeros(points)
    rhs[order] = math.factorial(order)
    return np.linalg.solve(V, rhs)


def grin_params(sim: dict, nx: int, window_um: float, radius_um: float, core_na: float,
                alpha: float, df_thz: float = 1.0):
    """get_params (fibers.jl:91-132): β(f) of the M modes on the stencil
    f0 + Δf·(-β_order .. β_order), their central-difference derivatives, the
    dispersion referenced to mode 1 (β0 and β1 of mode 1 removed), D(ω) =
    Σ_n β_n ω^n / n! and γ = S n2 ω0 / c from the modes at f0.  Returns a
    dict with "betas" (β_order+1, M), "D" (M, Nt), "gamma", "modes" (nx, nx,
    M), "x" [µm] and "neff" at f0."""
    f0, c0 = float(sim["f0"]), float(sim["c0"])
    M, nt, order = int(sim["M"]), int(sim["Nt"]), int(sim["β_order"])
    points = 2 * order + 1
    offsets = np.arange(points) - order
    beta_f = np.zeros((points, M))
    for i, off in enumerate(offsets):
        lam = c0 / ((f0 + df_thz * off) * 1e12) * 1e6
        eps, _, dx = build_grin(lam, nx, window_um, radius_um, core_na, alpha)
        _, _, neff = solve_fiber_modes(lam, M, dx, eps)
        beta_f[i] = 2 * math.pi * neff / (lam * 1e-6)
    deriv = np.zeros((order, M))
    for n in range(1, order + 1):
        deriv[n - 1] = central_fd_weights(points, n) @ beta_f / (2 * math.pi * df_thz / 1e-12) ** n
    betas = np.vstack([beta_f[order] - beta_f[order, 0], deriv[0] - deriv[0, 0], deriv[1:]])
    w = 2 * math.pi * P.fftfreq(nt, 1 / sim["Δt"]) * 1e12
    powers = np.stack([w ** n / math.factorial(n) for n in range(order + 1)], axis=1)
    D = (powers @ betas).T
    lam0 = c0 / f0 / 1e12 * 1e6
    eps, x, dx = build_grin(lam0, nx, window_um, radius_um, core_na, alpha)
    _, v, neff = solve_fiber_modes(lam0, M, dx, eps)
    modes = v.reshape(nx, nx, M, order="F")
    gamma = P.gamma_from_overlap(P.overlap_tensor(modes, dx * 1e-6), sim)
    return {"betas": betas, "D": np.ascontiguousarray(D), "gamma": gamma, "modes": modes,
            "x": x, "neff": neff}


def grin_problem(M: int, nt: int, time_window_ps: float, L: float, energy_j: float,
                 fwhm_s: float, *, nx: int = 48, window_um: float = 100.0,
                 radius_um: float = 25.0, core_na: float = 0.2, alpha: float = 2.0,
                 weights=None, beta_order: int = 3, fR: float = 0.18,
                 wavelength_m: float = 1030e-9, raman_threshold_thz: float = -13.0,
                 reltol: float = 1e-8, abstol: float = 1e-6, validate_grid: bool = True,
                 df_thz: float = 1.0) -> P.FiberProblem:
    """A GRIN multimode problem (get_disp_fiber_params, helpers.jl:181-214,
    with the sech² launch of simulate_disp_mmf.jl:140-159): M modes of a
    parabolic (α = 2) 25 µm / NA 0.2 core by default, launch split by
    `weights` (all in mode 1 when None)."""
    sim = P.get_disp_sim_params(wavelength_m, M, nt, time_window_ps, beta_order,
                                validate=validate_grid)
    g = grin_params(sim, nx, window_um, radius_um, core_na, alpha, df_thz)
    raman = P.single_oscillator_raman_fields(sim, fR)
    w = np.zeros(M, complex) if weights is None else np.asarray(weights, dtype=complex)
    if weights is None:
        w[0] = 1.0
    _, uw0 = P.get_initial_state(w / np.linalg.norm(w), energy_j, fwhm_s, 1.0, "sech_sq", sim)
    return P.FiberProblem(sim=sim, D=g["D"], gamma=g["gamma"], hR=raman["hRω"],
                          one_m_fR=raman["one_m_fR"], L=float(L), uw0=uw0, reltol=reltol,
                          abstol=abstol, mask=P.band_mask(sim, raman_threshold_thz),
                          meta=dict(kind="grin", neff=g["neff"], betas=g["betas"],
                                    fwhm_s=fwhm_s))
