"""Reference-shaped entry points over the CUDA stepper.

Mirrors FiberLab's solver boundary with the same names, argument meaning and
error behaviour:

  solve_disp_mmf(uω0, fiber, sim)            src/simulation/simulate_disp_mmf.jl:183-207
  solve_adjoint_disp_mmf(λωL, ũω, fiber, sim) src/simulation/sensitivity_disp_mmf.jl:309-332
  solve_disp_gain_smf(uω0, fiber, sim)       src/simulation/simulate_disp_gain_mmf.jl:204-239
  propagate(problem; saveat)                 src/fiberlab/propagation.jl:89-123
  metrics(result), verify(result; ...)       src/fiberlab/propagation.jl:176-304
  physical phase gradient                    src/fiberlab/physics_models.jl:1033-1046

`fiber` and `sim` are the reference's dictionaries (keys "Dω", "γ", "hRω",
"one_m_fR", "L", "zsave", optional "reltol"/"abstol"; "Nt", "M", "ωs", "ω0",
"Δt").  Fields are numpy arrays of shape (M, Nt) -- the memory layout of the
reference's column-major (Nt, M) arrays.  Every solve runs on the GPU; there
is no CPU path.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import objectives as O
from . import problem as P
from ._capi import Context, GPUProblem

_DEFAULT_CTX: Optional[Context] = None


def default_context() -> Context:
    global _DEFAULT_CTX
    if _DEFAULT_CTX is None:
        _DEFAULT_CTX = Context(0)
    return _DEFAULT_CTX


def problem_from_dicts(uw0, fiber: dict, sim: dict) -> P.FiberProblem:
    """The reference's (uω0, fiber, sim) triple as a FiberProblem
    (required keys physics_models.jl:463-465)."""
    for key in ("Nt", "M", "ωs", "ω0", "Δt"):
        if key not in sim:
            raise P.ArgumentError(f"sim is missing required key {key!r}")
    for key in ("Dω", "γ", "hRω", "one_m_fR", "L"):
        if key not in fiber:
            raise P.ArgumentError(f"fiber is missing required key {key!r}")
    gamma = np.asarray(fiber["γ"])
    if not np.isrealobj(gamma):
        raise P.ArgumentError("gamma tensor must use real-valued storage")
    fp = P.FiberProblem(sim=sim, D=np.asarray(fiber["Dω"], dtype=np.float64),
                        gamma=np.asarray(gamma, dtype=np.float64),
                        hR=np.asarray(fiber["hRω"], dtype=np.complex128),
                        one_m_fR=float(fiber["one_m_fR"]), L=float(fiber["L"]),
                        uw0=np.asarray(uw0, dtype=np.complex128),
                        reltol=float(fiber.get("reltol", 1e-8)),
                        abstol=float(fiber.get("abstol", 1e-6)))
    fp.validate()
    return fp


@dataclass
class DEStats:
    naccept: int
    nreject: int
    nf: int


class GPUSolution:
    """Stands in for the ODESolution of the reference solves: `sol(z)` at the
    stored positions (interaction frame), `t`, `retcode`, `destats`.  The
    forward keeps its z-checkpoints on the device for a following adjoint."""

    def __init__(self, gp: GPUProblem, t, u, stats, frame="interaction", D=None):
        self._gp = gp
        self.t = np.asarray(t, dtype=np.float64)
        self.u = u
        self.retcode = "Success"
        self.stats = stats
        if frame == "adjoint":
            self.destats = DEStats(stats["adj_naccept"], stats["adj_nreject"], stats["adj_nf"])
        else:
            self.destats = DEStats(stats["naccept"], stats["nreject"], stats["nf"])

    def __call__(self, z: float):
        idx = np.nonzero(self.t == z)[0]
        if len(idx) == 0:
            raise P.ArgumentError(
                f"z={z} is not a stored position; pass it in saveat/zsave")
        return self.u[idx[0]]


def solve_disp_mmf(uw0, fiber: dict, sim: dict, *, precision="fp32", ctx: Context = None,
                   saveat=None) -> dict:
    """Forward solve 0 -> L (simulate_disp_mmf.jl:183-207).  Returns
    {"ode_sol": GPUSolution} and, when fiber["zsave"] is set, the lab-frame
    "uω_z" (Nz, M, Nt) and time-domain "ut_z" (fft along time)."""
    fp = problem_from_dicts(uw0, fiber, sim)
    ctx = ctx or default_context()
    gp = GPUProblem(ctx, fp, precision)
    zsave = fiber.get("zsave")
    zs = [0.0, fp.L]
    if zsave is not None:
        zs = sorted(set([0.0, fp.L] + [float(z) for z in zsave]))
    if saveat is not None:
        zs = sorted(set(zs + [float(z) for z in saveat]))
    lab, stats = gp.forward(fp.uw0, zs)
    # interaction frame: ũ(z) = e^{-iDz} u(z)
    inter = np.stack([np.exp(-1j * fp.D * z) * lab[i] for i, z in enumerate(zs)])
    out = {"ode_sol": GPUSolution(gp, zs, inter, stats)}
    if zsave is not None:
        sel = [zs.index(float(z)) for z in zsave]
        out["uω_z"] = lab[sel]
        out["ut_z"] = np.fft.fft(lab[sel], axis=-1)
    return out


def solve_adjoint_disp_mmf(lamL, sol: GPUSolution, fiber: dict, sim: dict) -> GPUSolution:
    """Adjoint solve L -> 0 (sensitivity_disp_mmf.jl:309-332); `sol(0)` is λ(0)."""
    reltol = float(fiber.get("reltol", 1e-8))
    abstol = float(fiber.get("abstol", 1e-6))
    if not (np.isfinite(reltol) and reltol > 0):
        raise P.ArgumentError("adjoint reltol must be positive and finite")
    if not (np.isfinite(abstol) and abstol > 0):
        raise P.ArgumentError("adjoint abstol must be positive and finite")
    lam = np.asarray(lamL, dtype=np.complex128)
    if not np.all(np.isfinite(lam)):
        raise P.ArgumentError("adjoint terminal condition must be finite")
    if not P.gamma_symmetric(np.asarray(fiber["γ"], dtype=np.float64)):
        raise P.ArgumentError("fiber adjoint requires a fully permutation-symmetric gamma tensor")
    lam0, stats = sol._gp.adjoint(lam)
    L = float(fiber["L"])
    return GPUSolution(sol._gp, [0.0, L], np.stack([lam0, np.exp(-1j * np.asarray(fiber["Dω"]) * L) * lam]),
                       stats, frame="adjoint")


def solve_disp_gain_smf(uw0, fiber: dict, sim: dict, *, pump_power: float = 0.0,
                        ctx: Context = None) -> dict:
    """solve_disp_gain_smf (simulate_disp_gain_mmf.jl:204-239) on the GPU
    (fl_forward_gain).  Single mode only; fiber["gain_parameters"] is a
    constant gain [1/m] or a gain.YDFAParams (default 0.0, :210); the solve
    uses the reference's reltol = 1e-5 with the default abstol (:214-216).
    Returns {"ode_sol": GPUSolution} (its `pump` holds P at the stored
    positions) and, when fiber["zsave"] is set, the lab-frame "uω_z"
    (Nz, 1, Nt), "ut_z" (fft along time) and "Ppz" (Nz, 1) (:222-236)."""
    if int(sim.get("M", 0)) != 1:
        raise P.ArgumentError("disp_gain_smf is single mode only, requires M = 1 "
                              f"(got M = {sim.get('M')})")
    gain = fiber.get("gain_parameters", 0.0)
    fp = problem_from_dicts(uw0, fiber, sim)
    fp.reltol, fp.abstol = 1e-5, 1e-6
    zsave = fiber.get("zsave")
    zs = [0.0, fp.L]
    if zsave is not None:
        zs = sorted(set(zs + [float(z) for z in zsave]))
    gp = GPUProblem(ctx or default_context(), fp)
    lab, pumps, stats = gp.forward_gain(gain, float(pump_power), fp.uw0, zs)
    inter = np.stack([np.exp(-1j * fp.D * z) * lab[i] for i, z in enumerate(zs)])
    sol = GPUSolution(gp, zs, inter, stats)
    sol.pump = np.asarray(pumps)
    out = {"ode_sol": sol}
    if zsave is not None:
        sel = [zs.index(float(z)) for z in zsave]
        out["uω_z"] = lab[sel]
        out["ut_z"] = np.fft.fft(lab[sel], axis=-1)
        out["Ppz"] = np.asarray(pumps)[sel][:, None]
    return out


@dataclass
class PropagationResult:
    """Lab-frame samples of one run (propagation.jl:5-23); spectra (Nz, M, Nt)."""
    z_m: np.ndarray
    spectra: np.ndarray
    input_spectrum: np.ndarray
    output_spectrum: np.ndarray
    accepted_steps: int
    rhs_evaluations: int
    problem: Optional[P.FiberProblem] = None
    # per save position, the device's FP64 evidence sums (fl_forward_evidence)
    device_evidence: Optional[np.ndarray] = None


def save_positions(saveat, length_m: float) -> np.ndarray:
    """_save_positions (propagation.jl:60-70)."""
    if saveat is None:
        return np.array([0.0, length_m])
    z = np.asarray(saveat, dtype=np.float64)
    if z.ndim != 1:
        raise P.ArgumentError("saveat must be a vector of distances")
    if len(z) < 2:
        raise P.ArgumentError("saveat must include 0 and the fiber length")
    if not np.all(np.isfinite(z)):
        raise P.ArgumentError("saveat distances must be finite")
    if not np.all(np.diff(z) > 0):
        raise P.ArgumentError("saveat distances must be sorted and unique")
    if not (z[0] == 0.0 and z[-1] == length_m):
        raise P.ArgumentError(f"saveat must start at 0 and end at the fiber length {length_m}")
    return z


def propagate(fp: P.FiberProblem, saveat=None, *, precision="fp32",
              ctx: Context = None) -> PropagationResult:
    """propagate(problem; saveat) (propagation.jl:89-123)."""
    fp.validate()
    z = save_positions(saveat, fp.L)
    gp = GPUProblem(ctx or default_context(), fp, precision)
    spectra, stats = gp.forward(fp.uw0, z)
    return PropagationResult(z_m=z, spectra=spectra, input_spectrum=spectra[0].copy(),
                             output_spectrum=spectra[-1].copy(),
                             accepted_steps=stats["naccept"], rhs_evaluations=stats["nf"],
                             problem=fp, device_evidence=gp.forward_evidence(len(z)))


# ---------------------------------------------------------------------------
# Evidence over the saved spectra (propagation.jl:176-304).  A GPU result
# carries the FP64 reductions the device ran over its saved spectra
# (fl_forward_evidence, device_field_metrics); field_metrics restates the
# same reductions on the host for results made elsewhere (and checks the
# device sums in the tests).

def edge_fraction(power: np.ndarray) -> float:
    """_edge_fraction (propagation.jl:176-182): power in the first and last
    max(1, floor(0.05 n)) samples over the total."""
    power = np.asarray(power, dtype=np.float64)
    k = max(1, int(np.floor(0.05 * power.shape[0])))
    total = float(np.sum(power))
    if not total > 0:
        raise P.ArgumentError("field power must be nonzero")
    return float((np.sum(power[:k]) + np.sum(power[-k:])) / total)


def field_metrics(spectrum: np.ndarray, sim: dict) -> dict:
    """_field_metrics (propagation.jl:189-202) of one (M, Nt) spectrum: the
    time-domain field is fft along time (the reference's convention)."""
    u = np.atleast_2d(np.asarray(spectrum, dtype=np.complex128))
    temporal = np.fft.fft(u, axis=1)
    tpow = np.sum(np.abs(temporal) ** 2, axis=0)
    mode_energy = np.sum(np.abs(temporal) ** 2, axis=1) * float(sim["Δt"])
    spow = np.fft.fftshift(np.sum(np.abs(u) ** 2, axis=0))
    return {"energy_pj": float(np.sum(mode_energy)), "mode_energy_pj": mode_energy,
            "peak_power_w": float(np.max(tpow)),
            "temporal_edge_fraction": edge_fraction(tpow),
            "spectral_edge_fraction": edge_fraction(spow),
            "photon_number": P.photon_number(u, sim)}


def device_field_metrics(ev: np.ndarray, sim: dict) -> dict:
    """field_metrics of one save position from the device's FP64 sums
    (fl_forward_evidence): the reductions ran on the GPU; only the grid
    constants Δt and ω0 are applied here."""
    dt = float(sim["Δt"])
    mode_energy = np.asarray(ev[6:], dtype=np.float64) * dt
    return {"energy_pj": float(ev[0] * dt), "mode_energy_pj": mode_energy,
            "peak_power_w": float(ev[1]),
            "temporal_edge_fraction": float(ev[2] / ev[0]),
            "spectral_edge_fraction": float(ev[4] / ev[3]),
            "photon_number": float(ev[5] * dt / float(sim["ω0"]))}


def _integrity(result: PropagationResult) -> bool:
    """The structural part of _propagation_integrity (propagation.jl:125-145):
    sizes, ordered finite positions from 0 to L, and the input/output samples
    matching the first/last spectra and the problem's launch.  (The
    reference's SHA-256 evidence seal is provenance bookkeeping outside the
    solver path.)"""
    try:
        fp = result.problem
        z = np.asarray(result.z_m, dtype=np.float64)
        return (fp is not None and z.ndim == 1 and len(z) >= 2 and
                result.spectra.shape == (len(z), fp.M, fp.nt) and
                bool(np.all(np.isfinite(z))) and bool(np.all(np.diff(z) > 0)) and
                z[0] == 0.0 and z[-1] == float(fp.L) and
                np.array_equal(result.input_spectrum, fp.uw0) and
                np.array_equal(result.input_spectrum, result.spectra[0]) and
                np.array_equal(result.output_spectrum, result.spectra[-1]) and
                result.accepted_steps >= 0 and result.rhs_evaluations >= 0)
    except (AttributeError, TypeError, ValueError):
        return False


def _propagation_metrics(result: PropagationResult) -> dict:
    """_propagation_metrics (propagation.jl:204-237)."""
    fp = result.problem
    ev = result.device_evidence
    if ev is not None and np.shape(ev) == (len(result.z_m), 6 + fp.M):
        samples = [device_field_metrics(ev[i], fp.sim) for i in range(len(result.z_m))]
    else:  # a result that did not come from the GPU (no device sums)
        samples = [field_metrics(result.spectra[i], fp.sim) for i in range(len(result.z_m))]
    inp, out = samples[0], samples[-1]
    energy_drift = np.array([s["energy_pj"] / inp["energy_pj"] - 1 for s in samples])
    photon_drift = np.array([s["photon_number"] / inp["photon_number"] - 1 for s in samples])
    fwhm = fp.meta.get("fwhm_s") if fp.meta else None
    launch = None if fwhm is None else fwhm * 1e12 / float(fp.sim["Δt"])
    return {
        "samples": fp.nt, "modes": fp.M, "saved_positions": len(result.z_m),
        "length_m": float(fp.L), "time_window_ps": float(fp.sim["time_window"]),
        "delta_t_ps": float(fp.sim["Δt"]),
        "frequency_spacing_thz": 1.0 / float(fp.sim["time_window"]),
        "input_energy_pj": inp["energy_pj"], "output_energy_pj": out["energy_pj"],
        "input_mode_energy_pj": inp["mode_energy_pj"],
        "output_mode_energy_pj": out["mode_energy_pj"],
        "relative_energy_change": float(energy_drift[-1]),
        "max_relative_energy_change": float(np.max(np.abs(energy_drift))),
        "input_peak_power_w": inp["peak_power_w"], "output_peak_power_w": out["peak_power_w"],
        "max_temporal_edge_fraction": max(s["temporal_edge_fraction"] for s in samples),
        "max_spectral_edge_fraction": max(s["spectral_edge_fraction"] for s in samples),
        "max_photon_number_drift": float(np.max(np.abs(photon_drift))),
        "launch_samples_per_fwhm": launch, "retcode": "Success",
        "accepted_steps": result.accepted_steps, "rhs_evaluations": result.rhs_evaluations,
    }


def metrics(result: PropagationResult) -> dict:
    """metrics(result) (propagation.jl:239-242)."""
    if not _integrity(result):
        raise P.ArgumentError("propagation result was mutated")
    return _propagation_metrics(result)


def verify(result: PropagationResult, *, temporal_edge_limit=1e-3, spectral_edge_limit=1e-3,
           min_launch_samples_per_fwhm=8.0, require_launch_sampling=False,
           photon_drift_limit=1e-4, energy_drift_limit=None) -> dict:
    """verify(result; ...) (propagation.jl:244-304); None stands for the
    reference's `missing`."""
    if not (np.isfinite(temporal_edge_limit) and 0 <= temporal_edge_limit <= 1):
        raise P.ArgumentError("temporal_edge_limit must be finite and lie in [0, 1]")
    if not (np.isfinite(spectral_edge_limit) and 0 <= spectral_edge_limit <= 1):
        raise P.ArgumentError("spectral_edge_limit must be finite and lie in [0, 1]")
    if not (np.isfinite(min_launch_samples_per_fwhm) and min_launch_samples_per_fwhm > 0):
        raise P.ArgumentError("min_launch_samples_per_fwhm must be positive and finite")
    if photon_drift_limit is not None and not (np.isfinite(photon_drift_limit) and
                                               photon_drift_limit >= 0):
        raise P.ArgumentError("photon_drift_limit must be nonnegative and finite")
    if energy_drift_limit is not None and not (np.isfinite(energy_drift_limit) and
                                               energy_drift_limit >= 0):
        raise P.ArgumentError("energy_drift_limit must be nonnegative and finite")
    keys = ("pass", "integrity_ok", "solver_success", "finite_fields",
            "temporal_edges_contained", "spectral_edges_contained", "launch_sampling_ok",
            "photon_number_conserved", "energy_change_acceptable", "max_temporal_edge_fraction",
            "max_spectral_edge_fraction", "launch_samples_per_fwhm", "max_photon_number_drift",
            "max_relative_energy_change")
    if not _integrity(result):
        out = dict.fromkeys(keys)
        out.update({"pass": False, "integrity_ok": False})
        return out
    ev = _propagation_metrics(result)
    finite = bool(np.all(np.isfinite(result.spectra)))
    temporal_ok = ev["max_temporal_edge_fraction"] <= temporal_edge_limit
    spectral_ok = ev["max_spectral_edge_fraction"] <= spectral_edge_limit
    launch = ev["launch_samples_per_fwhm"]
    sampling_ok = None if launch is None else launch >= min_launch_samples_per_fwhm
    sampling_gate = sampling_ok is not False and (not require_launch_sampling or
                                                  sampling_ok is True)
    photon_ok = None if photon_drift_limit is None else \
        ev["max_photon_number_drift"] <= photon_drift_limit
    energy_ok = None if energy_drift_limit is None else \
        ev["max_relative_energy_change"] <= energy_drift_limit
    passed = (finite and temporal_ok and spectral_ok and sampling_gate and
              photon_ok is not False and energy_ok is not False)
    return {"pass": bool(passed), "integrity_ok": True, "solver_success": True,
            "finite_fields": finite, "temporal_edges_contained": bool(temporal_ok),
            "spectral_edges_contained": bool(spectral_ok), "launch_sampling_ok": sampling_ok,
            "photon_number_conserved": photon_ok, "energy_change_acceptable": energy_ok,
            "max_temporal_edge_fraction": ev["max_temporal_edge_fraction"],
            "max_spectral_edge_fraction": ev["max_spectral_edge_fraction"],
            "launch_samples_per_fwhm": launch,
            "max_photon_number_drift": ev["max_photon_number_drift"],
            "max_relative_energy_change": ev["max_relative_energy_change"]}


def phase_gradient(fp: P.FiberProblem, phases, *, log_cost=False, precision="fp32",
                   ctx: Context = None):
    """Raman-band cost J and ∂J/∂φ for one or more vector phases
    (physics_models.jl:1033-1046 with physics_helpers.jl:222-232)."""
    if fp.mask is None or not np.any(fp.mask):
        raise P.ArgumentError("band mask must contain at least one bin")
    if not P.gamma_symmetric(fp.gamma):
        raise P.ArgumentError("fiber adjoint requires a fully permutation-symmetric gamma tensor")
    gp = GPUProblem(ctx or default_context(), fp, precision)
    return gp.phase_gradient_batch(phases, fp.mask, fp.uw0, log_cost)


def _field_matrix(value, fp: P.FiberProblem, label: str):
    """_field_matrix / _phase_matrix (physics_models.jl:685-731): a scalar, an
    Nt vector (shared by the modes) or an (M, Nt) matrix, as (M, Nt) + shape."""
    nt, M = fp.nt, fp.M
    a = np.asarray(value, dtype=np.float64)
    if a.ndim == 0:
        if label == "phase":
            raise P.ArgumentError("fiber field physics requires a vector or matrix decoded phase")
        out, shape = np.full((M, nt), float(a)), "scalar"
    elif a.ndim == 1:
        if a.shape[0] != nt:
            raise P.ArgumentError(f"{label} vector length {a.shape[0]} does not match Nt={nt}")
        out, shape = np.repeat(a[None, :], M, axis=0), "vector"
    elif a.ndim == 2:
        if a.shape != (M, nt):
            raise P.ArgumentError(f"{label} matrix size {a.shape[::-1]} does not match ({nt}, {M})")
        out, shape = a.copy(), "matrix"
    else:
        raise P.ArgumentError(f"{label} must be a real scalar, vector, or matrix")
    if not np.all(np.isfinite(out)):
        raise P.ArgumentError(f"{label} values must be finite")
    return out, shape


def _for_shape(gradient: np.ndarray, shape: str):
    """_physical_gradient_for_shape (physics_models.jl:732-737)."""
    if shape == "scalar":
        return np.array([gradient.sum()])
    if shape == "vector":
        return gradient.sum(axis=0)
    return gradient


def physical_gradient(fp: P.FiberProblem, control: dict, *, log_cost=False, precision="fp32",
                      ctx: Context = None, objective: str = "raman_band",
                      worst_mode_tau: float = 50.0):
    """Objective cost and the spectral-shaper physical gradient
    (spectral_shaper_model, physics_models.jl:1021-1081): the launch
    u_shaped = sqrt(energy) · amplitude · cis(phase) · uω0 (:791-797) runs
    forward on the GPU, the named field objective (objectives.NAMES: the
    Raman band by default, physics_helpers.jl:222-318, dB form :320-326)
    gives J and the seed λ(L) on the host, the adjoint runs on the GPU, and
    from λ0 = λ(0)

        ∂J/∂phase     = 2 Re(conj(λ0) i u_shaped)
        ∂J/∂amplitude = 2 sqrt(energy) Re(conj(λ0) cis(phase) uω0)
        ∂J/∂energy    = Re(Σ conj(λ0) u_shaped) / energy

    each reduced to the shape of its control.  control may hold "phase",
    "amplitude" and "energy"; returns (J, {name: gradient}) for those given."""
    fp.validate()
    cost_fn = O.objective(objective, fp.mask, fp.sim, worst_mode_tau)
    if objective != "temporal_width" and (fp.mask is None or not np.any(fp.mask)):
        raise P.ArgumentError("band mask must contain at least one bin")
    if not P.gamma_symmetric(fp.gamma):
        raise P.ArgumentError("fiber adjoint requires a fully permutation-symmetric gamma tensor; "
                              "use propagate(problem) for forward-only nonsymmetric models")
    phase, phase_shape = _field_matrix(control.get("phase", np.zeros(fp.nt)), fp, "phase")
    amplitude, amp_shape = _field_matrix(control.get("amplitude", 1.0), fp, "amplitude")
    if not np.all(amplitude > 0):
        raise P.ArgumentError("fiber field amplitude control must be strictly positive")
    energy = float(control.get("energy", 1.0))
    if not (np.isfinite(energy) and energy > 0):
        raise P.ArgumentError("fiber field energy control must be positive and finite")
    alpha = np.sqrt(energy)
    shaped = alpha * amplitude * np.exp(1j * phase) * fp.uw0
    if not (np.all(np.isfinite(shaped)) and np.linalg.norm(shaped) > 0):
        raise P.ArgumentError("decoded controls must produce a finite, nonzero launch field")
    gp = GPUProblem(ctx or default_context(), fp, precision)
    out, _ = gp.forward(shaped)
    J, seed = P.maybe_log_cost(*cost_fn(out[-1]), log_cost)
    lam0, _ = gp.adjoint(seed)
    grads = {}
    if "phase" in control:
        grads["phase"] = _for_shape(2.0 * np.real(np.conj(lam0) * 1j * shaped), phase_shape)
    if "amplitude" in control:
        g = 2.0 * alpha * np.real(np.conj(lam0) * np.exp(1j * phase) * fp.uw0)
        grads["amplitude"] = _for_shape(g, amp_shape)
    if "energy" in control:
        grads["energy"] = np.array([np.real(np.sum(np.conj(lam0) * shaped)) / energy])
    for k, v in grads.items():
        if not np.all(np.isfinite(v)):
            raise P.ArgumentError(f"fiber field {k} physical gradient contains non-finite values")
    return J, grads
