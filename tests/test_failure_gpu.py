"""The failure paths of the solve and the step, made on the host without
any fault of the GPU.

* The reference's fault switch (YUZEN_FAULT_AMGCL=k:m,
  LinearSolverBackend.cpp:630-645) on the device solver and on the CPU oracle
  alike: the chosen solve breaks down before it iterates -- return 2, the
  caller's x untouched, the iteration count and residual the oracle's.
* A NaN in the right-hand side: return 2, x untouched.  An iteration cap of
  one: return 1.
* The whole step under the switch, against the reference's own run under it
  (tests/golden/fault_*.npz): a single broken-down Newton solve (the attempt
  fails and is repeated without the extrapolated start) and two in a row
  (that repeat fails too, and the time-step control cuts the step) end on the
  reference's film and clock.  The switch counts the film's Newton solves
  on both sides (the reference's set-up solves of the boundary rows run on
  its eigen backend, which the switch does not count).
* At a fixed step a Newton iteration that cannot converge is status -3 with
  the reference's FatalError text (FailedFixedStep, ImplicitSolver.cpp:
  192-201), and the step is usable again after yz_step_set_fields.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import _oracle
import _systems
import stateio
import yuzen_b200 as yz
from yuzen_b200 import step as ys

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(autouse=True)
def _switch_off():
    yz.fault_inject(0, 0)
    _oracle.fault_inject(0, 0)
    yield
    yz.fault_inject(0, 0)
    _oracle.fault_inject(0, 0)


def _gpu(d, x0, **over):
    s = yz.LinearSolverSettings(int(over.get("precondition", d["precondition"])), bool(d["scaling"]),
                                int(over.get("max_iteration", d["max_iteration"])), float(d["epsilon"]), False)
    pat = yz.CrsPattern(d["rowptr"], d["col"], d["sorted_col"], d["sorted_src"])
    x = np.array(x0, dtype=np.float64, copy=True)
    ret, it, res = yz.B200Backend().Solve(s, pat, over.get("values", d["values"]), over.get("rhs", d["rhs"]), x)
    return ret, it, res, x


@pytest.mark.parametrize("precondition", [2, 1])
def test_injected_breakdown_matches_the_oracle(precondition):
    """Three solves in a row with the switch on the second: each the
    oracle's to the bit (return, iterations, residual, x); the second a
    breakdown that leaves x as given."""
    d = _systems.film_system(64, seed=3, stiff=2.0)
    x0 = np.random.default_rng(0).standard_normal(d["n"]) * 1e-6
    yz.fault_inject(2, 1)
    _oracle.fault_inject(2, 1)
    for k in range(3):
        g = _gpu(d, x0, precondition=precondition, max_iteration=400)
        o = _oracle.OracleSolver().solve(d, precondition=precondition, x0=x0, max_iteration=400)
        assert (g[0], g[1], g[2]) == (o[0], o[1], o[2]), k
        assert np.array_equal(g[3], o[3]), k
        if k == 1:
            assert g[0] == 2 and np.array_equal(g[3], x0)


def test_nan_rhs_is_a_breakdown():
    d = _systems.film_system(40, seed=1)
    rhs = np.array(d["rhs"], copy=True)
    rhs[100] = np.nan
    x0 = np.full(d["n"], 0.25)
    ret, it, res, x = _gpu(d, x0, rhs=rhs)
    o = _oracle.OracleSolver().solve({**d, "rhs": rhs}, x0=x0)
    assert ret == 2 and o[0] == 2
    assert np.array_equal(x, x0)


def test_iteration_cap_returns_one():
    d = _systems.film_system(64, seed=2, stiff=2.0)
    ret, it, res, _ = _gpu(d, np.zeros(d["n"]), max_iteration=1)
    o = _oracle.OracleSolver().solve(d, max_iteration=1)
    assert ret == 1 and o[0] == 1 and it == o[1] == 1 and res == o[2]


@pytest.mark.parametrize("name", ["fault_adaptive_40", "fault2_adaptive_40"])
def test_step_under_the_fault_switch(name):
    d = stateio.load_npz(GOLDEN / f"{name}.npz")
    clean = ys.Step(ys.params_from_state(d), d["field_h0"], d["field_c0"], d["field_s0"])
    s_clean = clean.advance(int(d["steps_done"]))
    yz.fault_inject(int(d["fault_at"]), int(d["fault_count"]))
    st = ys.Step(ys.params_from_state(d), d["field_h0"], d["field_c0"], d["field_s0"])
    s = st.advance(int(d["steps_done"]))
    h, _ = st.fields()
    assert np.linalg.norm(h - d["field_h1"]) / np.linalg.norm(d["field_h1"]) <= 1e-10
    assert abs(s["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"])
    # the broken-down solves cost Newton passes (and, two in a row, a retry)
    assert s["newton_iterations"] > s_clean["newton_iterations"]


def test_fixed_step_failure_is_status_minus_3():
    d = stateio.load_npz(GOLDEN / "step_upwind_48.npz")
    st = ys.Step(ys.params_from_state(d), d["field_h0"], d["field_c0"], d["field_s0"])
    yz.fault_inject(1, 1000)
    with pytest.raises(yz.StepFailedError) as e:
        st.advance(1)
    assert e.value.status == -3
    assert "did not converge at the fixed step" in str(e.value)
    yz.fault_inject(0, 0)
    st.set_fields(d["field_h0"], d["field_c0"])
    s = st.advance(int(d["steps_done"]))
    h, _ = st.fields()
    assert np.isfinite(h).all() and s["steps"] == int(d["steps_done"])
