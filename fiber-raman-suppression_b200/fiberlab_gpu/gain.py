"""Gain models of the pump-gain single-mode propagation: host setup.

Restates the Yb-doped fiber amplifier parameters of
src/gain_simulation/gain.jl:25-68 (geometry and dopant defaults, pump and
signal channels, Marcuse mode-field overlaps), the cross-section
interpolation of :80-108 (linear in wavelength, flat outside the data) and
the YDFA branch of compute_gain (src/simulation/simulate_disp_gain_mmf.jl:
92-102).  The launch and fiber of the gain solver are those of any
single-mode problem (problem.single_mode_problem).  The cross-section
spectra are inputs: the caller passes
(wavelength, cross section) samples, e.g. those the reference keeps next to
gain.jl.  `gain_struct_arrays` gives the per-bin arrays in FFT bin order that
the solver's right-hand side consumes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
import numpy as np

from .problem import ArgumentError, C0

H_PLANCK_J = 6.62607015e-34   # the value calculate_gain_YDFA uses (gain.jl:151)


def marcuse_overlap(core_radius: float, na: float, wavelength: float) -> float:
    """Γ = 1 - exp(-2a²/w²) with w = a (0.616 + 1.66/V^1.5 + 0.987/V^6),
    V = 2π a NA / λ (gain.jl:58-66)."""
    V = 2 * math.pi * core_radius * na / wavelength
    w = core_radius * (0.616 + 1.66 / V ** 1.5 + 0.987 / V ** 6)
    return 1.0 - math.exp(-2 * core_radius ** 2 / w ** 2)


@dataclass
class YDFAParams:
    """YDFAParams (gain.jl:25-68): fs [THz] is the simulation's physical-order
    frequency grid, dt_ps its step; cross sections [m²] on fs."""
    fs: np.ndarray
    dt_ps: float
    nt: int
    L: float = 2.5
    core_radius: float = 2.5e-6
    NA: float = 0.13
    rho: float = 1e25
    tau21: float = 1.4e-3
    lambda_p: float = 976e-9
    sigma_ap: float = 2.5e-24
    sigma_ep: float = 2.5e-24
    lambda_s0: float = 1030e-9
    pulse_rep_rate: float = 80e6
    sigma_as: np.ndarray = field(default=None)
    sigma_es: np.ndarray = field(default=None)

    def __post_init__(self):
        self.fs = np.asarray(self.fs, dtype=np.float64)
        if self.sigma_as is None:
            self.sigma_as = np.zeros_like(self.fs)
        if self.sigma_es is None:
            self.sigma_es = np.zeros_like(self.fs)

    @property
    def area(self) -> float:
        return math.pi * self.core_radius ** 2

    @property
    def nu_p(self) -> float:
        return C0 / self.lambda_p

    @property
    def nus(self) -> np.ndarray:
        return self.fs * 1e12

    @property
    def dt(self) -> float:
        return self.dt_ps * 1e-12

    @property
    def df(self) -> float:
        return 1.0 / (self.nt * self.dt)

    @property
    def gamma_p(self) -> float:
        return marcuse_overlap(self.core_radius, self.NA, self.lambda_p)

    @property
    def gamma_s(self) -> float:
        return marcuse_overlap(self.core_radius, self.NA, self.lambda_s0)


def interpolate_cross_sections(fs_thz: np.ndarray, wavelength_m: np.ndarray,
                               sigma_m2: np.ndarray) -> np.ndarray:
    """Cross section on the simulation grid: linear in wavelength through the
    samples, the end values outside them (get_ydfa_cross_sections,
    gain.jl:80-108, with its Flat extrapolation)."""
    wl = np.asarray(wavelength_m, dtype=np.float64)
    sig = np.asarray(sigma_m2, dtype=np.float64)
    if wl.ndim != 1 or wl.shape != sig.shape or wl.size < 2:
        raise ArgumentError("cross sections need matching wavelength and value samples")
    order = np.argsort(wl)
    target = C0 / (np.asarray(fs_thz, dtype=np.float64) * 1e12)
    return np.interp(target, wl[order], sig[order])


def ydfa_params(sim: dict, absorption, emission, **overrides) -> YDFAParams:
    """get_YDFAParams (gain.jl:175-182) with the cross sections given as
    (wavelength [m], σ [m²]) sample pairs for absorption and emission."""
    p = YDFAParams(fs=sim["fs"], dt_ps=float(sim["Δt"]), nt=int(sim["Nt"]), **overrides)
    p.sigma_as = interpolate_cross_sections(p.fs, *absorption)
    p.sigma_es = interpolate_cross_sections(p.fs, *emission)
    return p


def gain_struct_arrays(p: YDFAParams) -> dict:
    """The scalars and FFT-order per-bin arrays of the solver's gain model
    (psd_from_uω's scale (Nt dt)² × repetition rate, h ν, cross sections)."""
    return {"gamma_p": p.gamma_p, "sigma_ap": p.sigma_ap, "sigma_ep": p.sigma_ep,
            "h_nu_p": H_PLANCK_J * p.nu_p, "gamma_s": p.gamma_s, "area": p.area,
            "rho": p.rho, "tau21": p.tau21,
            "psd_scale": (p.nt * p.dt) ** 2 * p.pulse_rep_rate, "df": p.df,
            "sigma_as": np.ascontiguousarray(np.fft.ifftshift(p.sigma_as)),
            "sigma_es": np.ascontiguousarray(np.fft.ifftshift(p.sigma_es)),
            "h_nu_s": np.ascontiguousarray(np.fft.ifftshift(H_PLANCK_J * p.nus))}


def ydfa_gain(p: YDFAParams, uw: np.ndarray, pump_w: float):
    """compute_gain for the YDFA model (simulate_disp_gain_mmf.jl:92-102 with
    calculate_gain_YDFA, gain.jl:150-166): the spectral gain g(ω) [1/m] in
    FFT bin order for the lab-frame spectrum uw (Nt,), and the pump gain."""
    a = gain_struct_arrays(p)
    ps = np.abs(np.asarray(uw).reshape(-1)) ** 2 * a["psd_scale"]
    w12 = np.sum(a["gamma_s"] * a["sigma_as"] * ps * a["df"] / (a["h_nu_s"] * a["area"]))
    w21 = np.sum(a["gamma_s"] * a["sigma_es"] * ps * a["df"] / (a["h_nu_s"] * a["area"]))
    r12 = a["gamma_p"] * a["sigma_ap"] * pump_w / (a["h_nu_p"] * a["area"])
    r21 = a["gamma_p"] * a["sigma_ep"] * pump_w / (a["h_nu_p"] * a["area"])
    n2 = (r12 + w12) / (r12 + r21 + w12 + w21 + 1.0 / a["tau21"])
    n1 = 1.0 - n2
    g = a["gamma_s"] * (a["sigma_es"] * n2 - a["sigma_as"] * n1) * a["rho"]
    gp = a["gamma_p"] * (a["sigma_ep"] * n2 - a["sigma_ap"] * n1) * a["rho"]
    return g, float(gp)
