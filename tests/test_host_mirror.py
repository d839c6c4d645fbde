"""Argument checks of the reference-named host mirror (solve.py) that run
before any device work -- CPU only: the (uω0, fiber, sim) dictionaries
(physics_models.jl:463-465, simulate_disp_mmf.jl:62-67), save positions
(propagation.jl:60-70) and the adjoint's terminal condition
(sensitivity_disp_mmf.jl:318-327).  tests/test_gpu_parity.py runs the same
functions through the GPU against the oracle."""
import numpy as np
import pytest

from fiberlab_gpu import problem as P
from fiberlab_gpu import solve as S


def _dicts(fp):
    fiber = {"Dω": fp.D, "γ": fp.gamma, "hRω": fp.hR, "one_m_fR": fp.one_m_fR, "L": fp.L,
             "zsave": None}
    return fiber, dict(fp.sim)


@pytest.fixture
def fp():
    return P.single_mode_problem(nt=128, time_window_ps=3.0, L=0.3, power_w=0.1,
                                 rep_rate_hz=80.5e6)


def test_problem_from_dicts_round_trip(fp):
    fiber, sim = _dicts(fp)
    fiber["reltol"], fiber["abstol"] = 1e-9, 1e-7
    q = S.problem_from_dicts(fp.uw0, fiber, sim)
    assert np.array_equal(q.D, fp.D) and np.array_equal(q.gamma, fp.gamma)
    assert q.reltol == 1e-9 and q.abstol == 1e-7 and q.L == fp.L


@pytest.mark.parametrize("where,key", [("sim", k) for k in ("Nt", "M", "ωs", "ω0", "Δt")] +
                         [("fiber", k) for k in ("Dω", "γ", "hRω", "one_m_fR", "L")])
def test_problem_from_dicts_missing_keys(fp, where, key):
    fiber, sim = _dicts(fp)
    del (sim if where == "sim" else fiber)[key]
    with pytest.raises(P.ArgumentError, match=key):
        S.problem_from_dicts(fp.uw0, fiber, sim)


def test_problem_from_dicts_rejects_bad_tables(fp):
    fiber, sim = _dicts(fp)
    with pytest.raises(P.ArgumentError, match="real-valued"):
        S.problem_from_dicts(fp.uw0, dict(fiber, **{"γ": fp.gamma.astype(complex)}), sim)
    with pytest.raises(P.ArgumentError, match="dispersion size"):
        S.problem_from_dicts(fp.uw0, dict(fiber, **{"Dω": fp.D[:, :64]}), sim)
    bad = fp.hR.copy()
    bad[1] += 0.5j
    with pytest.raises(P.ArgumentError, match="Hermitian"):
        S.problem_from_dicts(fp.uw0, dict(fiber, **{"hRω": bad}), sim)
    with pytest.raises(P.ArgumentError, match="fiber length"):
        S.problem_from_dicts(fp.uw0, dict(fiber, L=-1.0), sim)
    launch = fp.uw0.copy()
    launch[0, 0] = np.nan
    with pytest.raises(P.ArgumentError, match="launch field"):
        S.problem_from_dicts(launch, fiber, sim)


def test_save_positions():
    assert np.array_equal(S.save_positions(None, 0.5), [0.0, 0.5])
    assert np.array_equal(S.save_positions([0.0, 0.2, 0.5], 0.5), [0.0, 0.2, 0.5])
    for bad, msg in (([0.0, 0.3, 0.2, 0.5], "sorted"), ([0.0, 0.2, 0.2, 0.5], "sorted"),
                     ([0.1, 0.5], "start at 0"), ([0.0, 0.4], "start at 0"),
                     ([0.0], "include 0"), ([[0.0, 0.5]], "vector"),
                     ([0.0, np.inf, 0.5], "finite")):
        with pytest.raises(P.ArgumentError, match=msg):
            S.save_positions(bad, 0.5)


def test_adjoint_terminal_condition_checks(fp):
    # checked before the device is touched (no solution object needed)
    fiber, sim = _dicts(fp)
    lam = fp.uw0.copy()
    lam[0, 3] = np.inf
    with pytest.raises(P.ArgumentError, match="terminal condition"):
        S.solve_adjoint_disp_mmf(lam, None, fiber, sim)
    with pytest.raises(P.ArgumentError, match="reltol"):
        S.solve_adjoint_disp_mmf(fp.uw0, None, dict(fiber, reltol=0.0), sim)
    with pytest.raises(P.ArgumentError, match="abstol"):
        S.solve_adjoint_disp_mmf(fp.uw0, None, dict(fiber, abstol=np.nan), sim)
    g = np.zeros((2, 2, 2, 2))
    g[0, 0, 1, 1] = 1.0
    with pytest.raises(P.ArgumentError, match="symmetric"):
        S.solve_adjoint_disp_mmf(fp.uw0, None, dict(fiber, **{"γ": g}), sim)


def test_solve_disp_gain_smf_assembly(monkeypatch):
    # the dictionary interface and output assembly of solve_disp_gain_smf
    # (simulate_disp_gain_mmf.jl:204-239) around a stand-in for the device
    # call that returns the closed form of a constant gain with no
    # nonlinearity or dispersion (the GPU path itself is checked in
    # tests/test_gpu_parity.py::test_gain_propagation_matches_oracle)
    seen = {}

    class ClosedForm:
        def __init__(self, ctx, fp, precision="fp32"):
            self.fp = fp
            seen["tol"] = (fp.reltol, fp.abstol)

        def forward_gain(self, gain, pump, u0, saveat):
            z = np.asarray(saveat)
            out = np.stack([u0 * np.exp(0.5 * gain * zz) for zz in z])
            return out, pump * np.exp(-z), {"naccept": 3, "nreject": 0, "nf": 21,
                                            "adj_naccept": 0, "adj_nreject": 0, "adj_nf": 0}
    monkeypatch.setattr(S, "GPUProblem", ClosedForm)
    monkeypatch.setattr(S, "default_context", lambda: None)
    fp = P.single_mode_problem(nt=64, time_window_ps=3.0, L=0.2, power_w=1e-3, rep_rate_hz=80e6,
                               gamma=0.0, betas=(0.0,), beta_order=2, fR=0.0)
    fiber, sim = _dicts(fp)
    fiber["gain_parameters"] = 0.6
    fiber["zsave"] = [0.05, 0.2]
    res = S.solve_disp_gain_smf(fp.uw0, fiber, sim, pump_power=0.05)
    assert seen["tol"] == (1e-5, 1e-6)       # the reference's fixed reltol, default abstol
    assert res["uω_z"].shape == (2, 1, fp.nt) and res["Ppz"].shape == (2, 1)
    assert np.allclose(res["uω_z"][1], fp.uw0 * np.exp(0.3 * 0.2), rtol=1e-14)
    assert np.allclose(res["Ppz"][:, 0], 0.05 * np.exp(-np.array([0.05, 0.2])), rtol=1e-14)
    assert np.array_equal(res["ut_z"], np.fft.fft(res["uω_z"], axis=-1))
    sol = res["ode_sol"]
    assert list(sol.t) == [0.0, 0.05, 0.2] and sol.pump[0] == 0.05
    assert sol.destats.naccept == 3 and sol.retcode == "Success"
    assert np.allclose(sol(0.2), np.exp(-1j * fp.D * 0.2) * res["uω_z"][1])
    del fiber["zsave"]
    assert set(S.solve_disp_gain_smf(fp.uw0, fiber, sim, pump_power=0.05)) == {"ode_sol"}
    with pytest.raises(P.ArgumentError, match="single mode only"):
        S.solve_disp_gain_smf(fp.uw0, fiber, dict(sim, M=2))
