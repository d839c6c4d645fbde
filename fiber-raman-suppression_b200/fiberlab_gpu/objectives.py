"""Terminal objectives of the inverse-design path and their adjoint seeds.

Each objective maps the lab-frame output spectrum u(L) (shape (M, Nt): the
reference's column-major (Nt, M) array) to a cost J and the terminal seed
∂J/∂conj(u(L)), the λ(L) handed to the adjoint solve, so that a change δu
moves the cost by 2 Re Σ conj(seed) δu.  Restated from
src/fiberlab/physics_helpers.jl:222-326 (the legacy twins in
src/mmf_cost.jl:49-166 compute the same values), with the objective names of
the registry at src/fiberlab/physics_models.jl:851-964.

These are FP64 reductions over one output field; they run on the host
between the GPU forward solve and the GPU adjoint solve.
"""
from __future__ import annotations

import math

import numpy as np

from .problem import ArgumentError, band_cost_and_seed, maybe_log_cost


def _check_mask(u: np.ndarray, mask: np.ndarray) -> np.ndarray:
    mask = np.asarray(mask, dtype=bool)
    if u.shape[-1] != mask.shape[0]:
        raise ArgumentError(f"field rows {u.shape[-1]} do not match band mask length {mask.shape[0]}")
    if not np.any(mask):
        raise ArgumentError("band mask must contain at least one bin")
    return mask


def spectral_band_cost(u: np.ndarray, mask: np.ndarray):
    """Mode-summed band fraction (_field_spectral_band_cost,
    physics_helpers.jl:222-232)."""
    u = np.atleast_2d(u)
    return band_cost_and_seed(u, _check_mask(u, mask))


def fundamental_band_cost(u: np.ndarray, mask: np.ndarray):
    """Band fraction of mode 1 alone; the seed is zero on the other modes
    (_field_fundamental_band_cost, physics_helpers.jl:234-247)."""
    u = np.atleast_2d(u)
    mask = _check_mask(u, mask)
    u1 = u[0]
    total = float(np.sum(np.abs(u1) ** 2))
    if not total > 0:
        raise ArgumentError("fundamental mode must have nonzero spectral energy")
    cost = float(np.sum(np.abs(u1[mask]) ** 2)) / total
    terminal = np.zeros_like(u, dtype=np.complex128)
    terminal[0] = u1 * (mask.astype(np.float64) - cost) / total
    return cost, terminal


def worst_mode_band_cost(u: np.ndarray, mask: np.ndarray, tau: float = 50.0):
    """Normalised log-sum-exp of the per-mode band fractions r_m over the
    modes with nonzero energy (_field_worst_mode_band_cost,
    physics_helpers.jl:249-286):

        J = max r + (log Σ exp(τ (r - max r)) - log K) / τ,
        seed_m = w_m u_m (mask - r_m) / E_m,   w = softmax(τ r),

    so max r - log(K)/τ <= J <= max r."""
    u = np.atleast_2d(u)
    mask = _check_mask(u, mask)
    tau = float(tau)
    if not (math.isfinite(tau) and tau > 0):
        raise ArgumentError("worst-mode smoothness τ must be positive and finite")
    totals = np.sum(np.abs(u) ** 2, axis=1)
    active = np.flatnonzero(totals > 0)
    if active.size == 0:
        raise ArgumentError("worst-mode cost requires a nonzero-energy mode")
    ratios = np.zeros(u.shape[0])
    ratios[active] = np.sum(np.abs(u[active][:, mask]) ** 2, axis=1) / totals[active]
    rmax = float(np.max(ratios[active]))
    shifted = tau * (ratios[active] - rmax)
    denom = float(np.sum(np.exp(shifted)))
    cost = rmax + (math.log(denom) - math.log(active.size)) / tau
    weights = np.exp(shifted) / denom
    terminal = np.zeros_like(u, dtype=np.complex128)
    m = mask.astype(np.float64)
    for w, mode in zip(weights, active):
        terminal[mode] = w * u[mode] * (m - ratios[mode]) / totals[mode]
    if not (0.0 <= cost <= 1.0):
        raise ArgumentError("worst-mode smooth proxy left the [0,1] leakage scale")
    return float(cost), terminal


def spectral_peak_cost(u: np.ndarray, mask: np.ndarray):
    """Energy of the strongest in-band bin (summed over modes) over the total
    (_field_spectral_peak_cost, physics_helpers.jl:288-302).  The first
    maximum wins a tie, as Julia's argmax does."""
    u = np.atleast_2d(u)
    mask = _check_mask(u, mask)
    total = float(np.sum(np.abs(u) ** 2))
    if not total > 0:
        raise ArgumentError("field must have nonzero spectral energy")
    band = np.flatnonzero(mask)
    bins = np.sum(np.abs(u) ** 2, axis=0)
    peak = int(band[np.argmax(bins[band])])
    cost = float(bins[peak]) / total
    pm = np.zeros(u.shape[1])
    pm[peak] = 1.0
    return cost, u * (pm - cost) / total


def temporal_width_cost(u: np.ndarray, sim: dict):
    """Normalised second moment of the temporal intensity about the window
    centre (_field_temporal_width_cost, physics_helpers.jl:304-318): with
    u_t = fft(u) along time and s_k = (k - floor(Nt/2)) Δt / (Nt Δt / 2),

        J = Σ s² |u_t|² / Σ |u_t|²,   seed = Nt ifft(u_t (s² - J) / Σ|u_t|²)."""
    u = np.atleast_2d(u)
    nt = int(sim["Nt"])
    if u.shape[1] != nt:
        raise ArgumentError(f"field rows {u.shape[1]} do not match Nt={nt}")
    ut = np.fft.fft(u, axis=1)
    total = float(np.sum(np.abs(ut) ** 2))
    if not total > 0:
        raise ArgumentError("field must have nonzero temporal energy")
    dt = float(sim["Δt"])
    half = max(dt * nt / 2, np.finfo(float).eps)
    s = (np.arange(nt) - nt // 2) * dt / half
    w = (s * s)[None, :]
    cost = float(np.sum(w * np.abs(ut) ** 2)) / total
    return cost, nt * np.fft.ifft(ut * (w - cost) / total, axis=1)


# objective names of the reference registry (physics_models.jl:947-964)
_BAND = {"raman_band", "mode_sum", "mmf_sum"}
_FUNDAMENTAL = {"fundamental_mode", "mmf_fundamental"}
_WORST = {"worst_mode", "mmf_worst_mode"}
NAMES = sorted(_BAND | _FUNDAMENTAL | _WORST | {"raman_peak", "temporal_width"})


def objective(name: str, mask=None, sim=None, worst_mode_tau: float = 50.0):
    """The cost-and-seed function of a named objective: field -> (J, seed)."""
    if name in _BAND:
        return lambda u: spectral_band_cost(u, mask)
    if name in _FUNDAMENTAL:
        return lambda u: fundamental_band_cost(u, mask)
    if name in _WORST:
        return lambda u: worst_mode_band_cost(u, mask, worst_mode_tau)
    if name == "raman_peak":
        return lambda u: spectral_peak_cost(u, mask)
    if name == "temporal_width":
        if sim is None:
            raise ArgumentError("temporal_width objective needs the sim grid")
        return lambda u: temporal_width_cost(u, sim)
    raise ArgumentError(f"unknown field objective {name!r}; known: {', '.join(NAMES)}")


def cost_and_seed(name: str, u: np.ndarray, mask=None, sim=None, log_cost: bool = False,
                  worst_mode_tau: float = 50.0):
    """(J, seed) of a named objective, in dB when log_cost (physics_helpers.jl:320-326)."""
    J, seed = objective(name, mask, sim, worst_mode_tau)(u)
    return maybe_log_cost(J, seed, log_cost)
