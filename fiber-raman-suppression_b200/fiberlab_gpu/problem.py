"""Host-side problem construction for the GMMNLSE stepper.

FP64 numpy restatement of FiberLab's setup layer, which runs once per problem
above the C-ABI (the CUDA library receives the finished tables):

  get_disp_sim_params                   src/helpers/helpers.jl:56-84
  _validate_positive_frequency_grid     src/helpers/helpers.jl:14-22
  _single_oscillator_raman_fields       src/helpers/helpers.jl:97-130
  get_disp_fiber_params_user_defined    src/helpers/helpers.jl:245-281
  get_initial_state                     src/simulation/simulate_disp_mmf.jl:140-159
  selfsteep = fftshift(ωs/ω0)           src/simulation/simulate_disp_mmf.jl:89
  _real_response_spectrum (hR check)    src/fiberlab/physics_models.jl:438-449
  band mask fftfreq < threshold         src/fiberlab/physics_models.jl:561
  γ = S·n2·ω0/c, S = Σψ⁴/dx²            src/simulation/fibers.jl:127-129, 214-222
  multimode launch normalisation        src/fiberlab/physics_models.jl:289-297

Layout follows the reference's column-major (Nt, M) arrays: a field is a numpy
array of shape (M, Nt), C-contiguous, so element (t, i) sits at t + Nt*i; the
gamma tensor is passed in the reference's element order γ[i,j,k,l] at
i + M(j + M(k + M l)) (``gamma.ravel(order="F")``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

C0 = 2.99792458e8          # m/s
H_PLANCK = 6.62607e-34      # J s
N2_SILICA = 2.3e-20         # m^2/W

SMF28 = dict(gamma=1.1e-3, betas=(-2.17e-26, 1.2e-40), fR=0.18)
RAMAN_TAU1_FS = 12.2
RAMAN_TAU2_FS = 32.0


class ArgumentError(ValueError):
    """Raised where the reference throws ArgumentError."""


def fftfreq(n: int, sample_rate: float) -> np.ndarray:
    """FFTW.fftfreq(n, fs): (0..n/2-1, -n/2..-1) * fs/n."""
    k = np.arange(n, dtype=np.float64)
    k[n // 2:] -= n
    return k * (sample_rate / n)


def minimum_time_window_ps(wavelength_m: float, nt: int) -> float:
    f0 = C0 / wavelength_m / 1e12
    return nt / (2 * f0)


def validate_positive_frequency_grid(wavelength_m: float, nt: int, time_window_ps: float) -> None:
    """helpers.jl:14-22 (same message text)."""
    minimum_window = minimum_time_window_ps(wavelength_m, nt)
    safe_window = (math.floor(minimum_window * 1000) + 1) / 1000
    if not time_window_ps > minimum_window:
        raise ArgumentError(
            "simulation bandwidth reaches nonpositive absolute optical frequencies: "
            f"Nt={nt} at λ0={wavelength_m * 1e9:.4g} nm requires time_window > "
            f"{minimum_window:.9g} ps (use at least {safe_window:.3f} ps); increase the "
            "window or use fewer samples")


def get_disp_sim_params(wavelength_m: float, M: int, nt: int, time_window_ps: float,
                        beta_order: int, *, validate: bool = True) -> dict:
    """helpers.jl:56-84.  ``validate=False`` builds grids below the
    positive-frequency limit with the same formulas (used by the benchmark
    shapes whose windows are narrower than the limit)."""
    if not (np.isfinite(wavelength_m) and wavelength_m > 0):
        raise ArgumentError("λ0 must be positive and finite")
    if not (isinstance(M, (int, np.integer)) and M > 0):
        raise ArgumentError("M must be a positive integer")
    if not (isinstance(nt, (int, np.integer)) and nt >= 4 and (nt & (nt - 1)) == 0):
        raise ArgumentError("Nt must be a power of two ≥ 4")
    if not (np.isfinite(time_window_ps) and time_window_ps > 0):
        raise ArgumentError("time_window must be positive and finite")
    if not (isinstance(beta_order, (int, np.integer)) and beta_order >= 2):
        raise ArgumentError("β_order must be an integer ≥ 2")
    f0 = C0 / wavelength_m / 1e12
    if validate:
        validate_positive_frequency_grid(wavelength_m, nt, time_window_ps)
    dt = time_window_ps / nt
    ts = 1e-12 * (-time_window_ps / 2 + np.arange(nt) * dt)
    fs = f0 + np.fft.fftshift(fftfreq(nt, 1 / dt))
    if validate and not np.all(fs > 0):
        raise ArgumentError(
            "simulation frequency construction violated the positive-frequency grid invariant")
    w0 = 2 * math.pi * f0
    ws = 2 * math.pi * fs
    eps = 1e-12 * dt / (H_PLANCK * 1e12 * f0)
    return {"λ0": float(wavelength_m), "f0": f0, "M": int(M), "Nt": int(nt),
            "time_window": float(time_window_ps), "Δt": dt, "ts": ts, "fs": fs,
            "ω0": w0, "ωs": ws, "c0": C0, "h": H_PLANCK, "ε": eps,
            "β_order": int(beta_order)}


def selfsteep(sim: dict) -> np.ndarray:
    """fftshift(ωs/ω0) (simulate_disp_mmf.jl:89)."""
    return np.fft.fftshift(sim["ωs"] / sim["ω0"])


def single_oscillator_raman_fields(sim: dict, fR: float = 0.18, tau1_fs: float = RAMAN_TAU1_FS,
                                   tau2_fs: float = RAMAN_TAU2_FS) -> dict:
    """helpers.jl:97-130."""
    fraction, t1, t2 = float(fR), float(tau1_fs), float(tau2_fs)
    if not (np.isfinite(fraction) and 0 <= fraction <= 1):
        raise ArgumentError("fR must be finite and lie in [0, 1]")
    if not (np.isfinite(t1) and t1 > 0):
        raise ArgumentError("τ1 must be positive and finite")
    if not (np.isfinite(t2) and t2 > 0):
        raise ArgumentError("τ2 must be positive and finite")
    nt, dt = int(sim["Nt"]), float(sim["Δt"])
    if not (nt >= 4 and (nt & (nt - 1)) == 0):
        raise ArgumentError("simulation Nt must be a power of two ≥ 4")
    if not (np.isfinite(dt) and dt > 0):
        raise ArgumentError("simulation Δt must be positive and finite")
    omega = 2 * math.pi * fftfreq(nt, 1 / dt)
    decay, resonance = 1e3 / t2, 1e3 / t1
    if not (np.isfinite(decay) and np.isfinite(resonance)):
        raise ArgumentError("Raman time constants are outside the supported Float64 range")
    with np.errstate(over="ignore", invalid="ignore"):
        response = fraction * (decay ** 2 + resonance ** 2) / (
            (decay + 1j * omega) ** 2 + resonance ** 2)
        centered = np.exp(-1j * omega * nt * dt / 2) * response
    centered[nt // 2] = centered[nt // 2].real
    if not np.all(np.isfinite(centered)):
        raise ArgumentError("Raman response is not finite for the requested parameters")
    return {"hRω": centered, "one_m_fR": 1 - fraction,
            "raman_response_model": "blow_wood_single_damped_oscillator_v1",
            "raman_fraction": fraction, "raman_tau1_fs": t1, "raman_tau2_fs": t2}


def real_response_spectrum(response: np.ndarray) -> bool:
    """physics_models.jl:438-449: the Raman spectrum must be Hermitian."""
    nt = len(response)
    scale = max(1.0, float(np.max(np.abs(response))))
    tol = 1e-12 * scale
    if abs(response[0].imag) > tol or abs(response[nt // 2].imag) > tol:
        return False
    a = response[1:nt // 2]
    b = np.conj(response[nt - 1:nt // 2:-1])
    return bool(np.all(np.abs(a - b) <= np.maximum(tol, 1e-12 * np.maximum(np.abs(a), np.abs(b)))))


def dispersion_from_betas(sim: dict, betas: Sequence[float], beta0: float = 0.0,
                          beta1: float = 0.0) -> np.ndarray:
    """D(ω) = Σ_n β_n/n! (2π·fftfreq·1e12)^n (helpers.jl:271-273); the reference
    uses β0 = β1 = 0, the multimode benchmark shapes add per-mode offsets."""
    nt, dt, order = sim["Nt"], sim["Δt"], sim["β_order"]
    if len(betas) > order - 1:
        raise ArgumentError(
            f"betas_user length must be ≤ β_order-1 ({order - 1}); got {len(betas)}")
    coeffs = [beta0, beta1] + list(betas) + [0.0] * (order - 1 - len(betas))
    w = 2 * math.pi * fftfreq(nt, 1 / dt) * 1e12
    D = np.zeros(nt)
    for n, b in enumerate(coeffs):
        D = D + (w ** n / math.factorial(n)) * b
    return D


def get_initial_state(u0_modes: np.ndarray, p_cont: float, fwhm: float, rep_rate: float,
                      pulse_form: str, sim: dict):
    """simulate_disp_mmf.jl:140-159.  Returns (ut0, uω0) of shape (M, Nt)."""
    M, nt, ts = sim["M"], sim["Nt"], sim["ts"]
    if pulse_form == "gauss":
        sigma = fwhm / 1.66511
        env = np.exp(-ts ** 2 / 2 / sigma ** 2)
        p_peak = 0.939437 * p_cont / fwhm / rep_rate
    elif pulse_form == "sech_sq":
        tau = fwhm / 1.7627
        env = 1.0 / np.cosh(-ts / tau)
        p_peak = 0.881374 * p_cont / fwhm / rep_rate
    else:
        raise ArgumentError(f'unsupported pulse_form="{pulse_form}"; expected "gauss" or "sech_sq"')
    modes = np.asarray(u0_modes, dtype=np.complex128).reshape(M)
    u0 = env[None, :].astype(np.complex128) * np.conj(modes)[:, None]   # u0_norm .*= u0_modes'
    u0 = u0 / math.sqrt(np.max(np.sum(np.abs(u0) ** 2, axis=0)))
    ut0 = u0 * math.sqrt(p_peak)
    uw0 = np.fft.ifft(ut0, axis=1)
    return ut0, uw0


def band_mask(sim: dict, threshold_thz: float) -> np.ndarray:
    """fftfreq(Nt, 1/Δt) < threshold (physics_models.jl:561)."""
    return fftfreq(sim["Nt"], 1 / sim["Δt"]) < threshold_thz


# ---------------------------------------------------------------------------
# Hermite-Gauss modes and the Kerr overlap tensor (multimode shapes)
# ---------------------------------------------------------------------------

def hg_mode_list(max_order: int):
    """(m, n) with m + n <= max_order, grouped by m + n."""
    return [(g - n, n) for g in range(max_order + 1) for n in range(g + 1)]


def hermite_gauss_modes(max_order: int, nx: int, w0_m: float, window_m: float):
    """Unit-norm discrete HG(m,n) profiles on an nx×nx grid; returns (modes
    (nx, nx, M), dx, [(m, n)])."""
    from numpy.polynomial.hermite import hermval
    x = (np.arange(nx) - (nx - 1) / 2) * (window_m / nx)
    dx = window_m / nx
    X, Y = np.meshgrid(x, x, indexing="ij")
    out = []
    idx = hg_mode_list(max_order)
    for (m, n) in idx:
        cm = np.zeros(m + 1); cm[m] = 1.0
        cn = np.zeros(n + 1); cn[n] = 1.0
        psi = hermval(math.sqrt(2) * X / w0_m, cm) * hermval(math.sqrt(2) * Y / w0_m, cn) * \
            np.exp(-(X ** 2 + Y ** 2) / w0_m ** 2)
        psi = psi / math.sqrt(np.sum(psi ** 2))
        out.append(psi)
    return np.stack(out, axis=-1), dx, idx


def overlap_tensor(modes: np.ndarray, dx_m: float) -> np.ndarray:
    """S_ijkl = Σ ψiψjψkψl / dx² (fibers.jl:214-222)."""
    M = modes.shape[-1]
    P = modes.reshape(-1, M)
    return np.einsum("pi,pj,pk,pl->ijkl", P, P, P, P) / dx_m ** 2


def gamma_from_overlap(S: np.ndarray, sim: dict, n2: float = N2_SILICA) -> np.ndarray:
    """γ = S·n2·ω0/c with ω0 in rad/s (fibers.jl:127-129)."""
    w0 = 2 * math.pi * sim["f0"] * 1e12
    return S * n2 * w0 / C0


# ---------------------------------------------------------------------------
# Problem object (the data a solve needs: fiber tables + sim grid + launch)
# ---------------------------------------------------------------------------

@dataclass
class FiberProblem:
    """Resolved propagation problem: the `fiber`/`sim` dictionaries the
    reference passes to solve_disp_mmf, reduced to the tables the stepper
    reads (simulate_disp_mmf.jl:183-187, physics_models.jl:463-465)."""
    sim: dict
    D: np.ndarray                 # (M, Nt) rad/m
    gamma: np.ndarray             # (M, M, M, M), gamma[i,j,k,l] = γ[i,j,k,l]
    hR: np.ndarray                # (Nt,) complex
    one_m_fR: float
    L: float
    uw0: np.ndarray               # (M, Nt) complex launch spectrum
    reltol: float = 1e-8
    abstol: float = 1e-6
    mask: Optional[np.ndarray] = None     # (Nt,) bool Raman band
    meta: dict = field(default_factory=dict)

    @property
    def nt(self) -> int:
        return int(self.sim["Nt"])

    @property
    def M(self) -> int:
        return int(self.sim["M"])

    @property
    def selfsteep(self) -> np.ndarray:
        return selfsteep(self.sim)

    def gamma_ref_order(self) -> np.ndarray:
        """γ flattened in the reference's element order (column-major)."""
        return np.ascontiguousarray(self.gamma.ravel(order="F"))

    def validate(self) -> None:
        nt, M = self.nt, self.M
        if self.D.shape != (M, nt):
            raise ArgumentError(f"dispersion size {self.D.shape[::-1]} does not match ({nt}, {M})")
        if self.gamma.shape != (M, M, M, M):
            raise ArgumentError("gamma tensor size does not match (M, M, M, M)")
        if not np.isrealobj(self.gamma):
            raise ArgumentError("gamma tensor must use real-valued storage")
        if not np.all(np.isfinite(self.gamma)):
            raise ArgumentError("gamma tensor must be finite")
        if self.hR.shape != (nt,):
            raise ArgumentError("Raman response must contain one value per frequency sample")
        if not real_response_spectrum(self.hR):
            raise ArgumentError("Raman response spectrum must be Hermitian (real time response)")
        if self.uw0.shape != (M, nt) or not np.all(np.isfinite(self.uw0)):
            raise ArgumentError("launch field must be finite with size (Nt, M)")
        if not (np.isfinite(self.L) and self.L > 0):
            raise ArgumentError("fiber length must be positive and finite")
        for name, v in (("reltol", self.reltol), ("abstol", self.abstol)):
            if not (np.isfinite(v) and v > 0):
                raise ArgumentError(f"{name} must be positive and finite")


def gamma_symmetric(gamma: np.ndarray) -> bool:
    """_adjoint_gamma_symmetric (sensitivity_disp_mmf.jl:103-112)."""
    tol = 1e-12 * max(1.0, float(np.max(np.abs(gamma))))

    def close(a, b):
        return np.all(np.abs(a - b) <= np.maximum(tol, 1e-12 * np.maximum(np.abs(a), np.abs(b))))
    return bool(close(gamma, gamma.transpose(1, 0, 2, 3)) and
                close(gamma, gamma.transpose(0, 2, 1, 3)) and
                close(gamma, gamma.transpose(0, 1, 3, 2)))


def single_mode_problem(nt: int = 8192, time_window_ps: float = 10.0, L: float = 0.5,
                        power_w: float = 0.1, fwhm_s: float = 185e-15,
                        rep_rate_hz: float = 80e6, gamma: float = SMF28["gamma"],
                        betas: Sequence[float] = SMF28["betas"], beta_order: int = 3,
                        fR: float = 0.18, wavelength_m: float = 1550e-9,
                        pulse: str = "sech_sq", raman_threshold_thz: float = -13.0,
                        reltol: float = 1e-8, abstol: float = 1e-6,
                        validate_grid: bool = True) -> FiberProblem:
    """_single_mode_low_level_setup (physics_models.jl:120-160) for a preset
    single-mode fiber; SMF-28 numbers from physics_helpers.jl:2-7."""
    sim = get_disp_sim_params(wavelength_m, 1, nt, time_window_ps, beta_order,
                              validate=validate_grid)
    raman = single_oscillator_raman_fields(sim, fR)
    D = dispersion_from_betas(sim, betas)[None, :]
    _, uw0 = get_initial_state(np.ones(1), power_w, fwhm_s, rep_rate_hz, pulse, sim)
    return FiberProblem(sim=sim, D=D, gamma=np.full((1, 1, 1, 1), float(gamma)),
                        hR=raman["hRω"], one_m_fR=raman["one_m_fR"], L=float(L), uw0=uw0,
                        reltol=reltol, abstol=abstol,
                        mask=band_mask(sim, raman_threshold_thz),
                        meta=dict(kind="single_mode", power_w=power_w, fwhm_s=fwhm_s,
                                  rep_rate_hz=rep_rate_hz))


def hg_group(m: int, n: int) -> int:
    return m + n


def multimode_problem(max_order: int, nx: int, nt: int, time_window_ps: float, L: float,
                      energy_j: float, fwhm_s: float, seed: int, *, w0_m: float = 15e-6,
                      window_factor: float = 8.0, beta0_by_group: Sequence[float] = (0, 50, 100, 150),
                      beta1_by_group: Sequence[float] = (0.0, 1e-13, -1e-13, 1e-13),
                      betas: Sequence[float] = SMF28["betas"], beta_order: int = 3,
                      fR: float = 0.18, wavelength_m: float = 1550e-9,
                      raman_threshold_thz: float = -13.0, reltol: float = 1e-8,
                      abstol: float = 1e-6, validate_grid: bool = False) -> FiberProblem:
    """Hermite-Gauss multimode problem (the fiber_problem explicit-physics
    path, physics_models.jl:330-423): HG(m,n), m+n <= max_order, unit-norm on
    an nx×nx grid spanning window_factor·w0; γ from the 4-overlaps; per-mode
    D = β0_g + β1_g ω + β2 ω²/2 + β3 ω³/6 by mode group g = m+n; launch split
    by sqrt(Dirichlet(1)) amplitudes with U(0, 2π) phases (seeded)."""
    modes, dx, idx = hermite_gauss_modes(max_order, nx, w0_m, window_factor * w0_m)
    M = len(idx)
    sim = get_disp_sim_params(wavelength_m, M, nt, time_window_ps, beta_order,
                              validate=validate_grid)
    S = overlap_tensor(modes, dx)
    gam = gamma_from_overlap(S, sim)
    D = np.stack([dispersion_from_betas(sim, betas, beta0=float(beta0_by_group[hg_group(*mn)]),
                                        beta1=float(beta1_by_group[hg_group(*mn)]))
                  for mn in idx])
    rng = np.random.default_rng(seed)
    w = rng.dirichlet(np.ones(M))
    ph = rng.uniform(0, 2 * math.pi, M)
    launch = np.sqrt(w) * np.exp(1j * ph)
    launch = launch / np.linalg.norm(launch)
    raman = single_oscillator_raman_fields(sim, fR)
    # energy per pulse E = P_cont / rep_rate: use rep_rate = 1 Hz
    _, uw0 = get_initial_state(launch, energy_j, fwhm_s, 1.0, "sech_sq", sim)
    return FiberProblem(sim=sim, D=D, gamma=gam, hR=raman["hRω"],
                        one_m_fR=raman["one_m_fR"], L=float(L), uw0=uw0, reltol=reltol,
                        abstol=abstol, mask=band_mask(sim, raman_threshold_thz),
                        meta=dict(kind="multimode", modes=idx, launch=launch, dx=dx,
                                  fwhm_s=fwhm_s))


# ---------------------------------------------------------------------------
# Objective, seed and gradient chain rule (host-side FP64 references)
# ---------------------------------------------------------------------------

def band_cost_and_seed(uwL: np.ndarray, mask: np.ndarray):
    """_field_spectral_band_cost (physics_helpers.jl:222-232)."""
    if not np.any(mask):
        raise ArgumentError("band mask must contain at least one bin")
    total = float(np.sum(np.abs(uwL) ** 2))
    if not total > 0:
        raise ArgumentError("field must have nonzero spectral energy")
    band = float(np.sum(np.abs(uwL[:, mask]) ** 2))
    cost = band / total
    terminal = uwL * (mask.astype(np.float64)[None, :] - cost) / total
    return cost, terminal


def maybe_log_cost(cost: float, terminal: np.ndarray, log_cost: bool):
    """_maybe_log_cost (physics_helpers.jl:320-326)."""
    if not log_cost:
        return cost, terminal
    floor = 1e-15
    scaled = 10.0 * math.log10(max(cost, floor))
    scale = 0.0 if cost <= floor else 10.0 / (math.log(10.0) * cost)
    return scaled, scale * terminal


def photon_number(spectrum: np.ndarray, sim: dict) -> float:
    """_photon_number (propagation.jl:184-187)."""
    omega = np.fft.fftshift(np.abs(sim["ωs"]))
    return float(sim["Δt"] * np.sum(np.abs(spectrum) ** 2 / omega[None, :]))


def centroid_thz(spectrum: np.ndarray, sim: dict) -> float:
    """Energy-weighted FFT-offset centroid (scientific_metrics.jl:275-285)."""
    f = fftfreq(sim["Nt"], 1 / sim["Δt"])
    e = np.sum(np.abs(spectrum) ** 2, axis=0)
    return float(np.sum(f * e) / np.sum(e))


# ---------------------------------------------------------------------------
# Serving request mix (synthetic, seeded)
# ---------------------------------------------------------------------------

@dataclass
class ServeRequest:
    arrival_s: float
    nt: int
    L: float
    power_w: float
    kind: int            # 0 forward, 1 forward + band gradient
    phase: Optional[np.ndarray] = None


def serving_grid_problem(nt: int, time_window_ps: float = 10.0) -> FiberProblem:
    """The per-grid tables of the serving mix: SMF-28, 185 fs sech² at
    80 MHz, band < -13 THz (lengths and powers vary per request)."""
    return single_mode_problem(nt=nt, time_window_ps=time_window_ps, L=1.0, power_w=0.1,
                               rep_rate_hz=80e6, raman_threshold_thz=-13.0,
                               validate_grid=False)


def serving_launch(fp: FiberProblem, power_w: float) -> np.ndarray:
    """Launch spectrum of the serving grid at an average power (the sech²
    pulse of get_initial_state scaled to P_avg)."""
    return fp.uw0 * math.sqrt(power_w / 0.1)


def serving_mix(n: int, seed: int = 0, rate_hz: float = 2000.0, log2_nt=(11, 15),
                L_range=(0.1, 5.0), p_range=(0.02, 0.3)) -> list:
    """n requests with exponential inter-arrival gaps (Poisson arrivals at
    rate_hz), log2 Nt uniform on log2_nt, L ~ U(L_range) m, P ~ U(p_range) W,
    half forward-only and half forward + band gradient with a launch phase
    N(0, 0.5²) per bin."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n))
    out = []
    for i in range(n):
        nt = 1 << int(rng.integers(log2_nt[0], log2_nt[1] + 1))
        L = float(rng.uniform(*L_range))
        P = float(rng.uniform(*p_range))
        kind = int(rng.integers(0, 2))
        ph = 0.5 * rng.standard_normal(nt) if kind == 1 else None
        out.append(ServeRequest(float(t[i]), nt, L, P, kind, ph))
    return out
