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
