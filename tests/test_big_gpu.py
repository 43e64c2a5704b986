"""Parity of the device step at the measured workloads' sizes: the 224^2
spinodal film (periodic edges, adaptive dt, 5 steps) and the 512^2
all-physics film (every term, the concentration solved, 2 steps at
dt = 1e-5 s), against the reference's own time loop on the same seeded
case (tests/golden/big_*.npz).

Bars, as for the small step fixtures: the CRS patterns of the film and of
the concentration bit for bit (hashes); h and c after the steps within 1e-10
relative L2 on the FP64 drop-in path and the clock to 1e-12; the faster
forms (the FP32 V-cycle, with the AMG hierarchy reused, with the FP32
matrix) within 1e-8 of the reference's FP64 run.  On the 512^2 film the
linear solve of the first Newton system is also checked against the CPU
oracle solver at full size: answer, iteration count, residual and every
level of the AMG hierarchy bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import _big
import _oracle
import _systems
import yuzen_b200 as yz
from yuzen_b200 import step as ys

pytestmark = pytest.mark.gpu
IDS = [f.stem for f in _big.BIG]
#  arm: (precision, AMG hierarchy reuse)
FORMS = {"fp32_cycle": (1, 0), "fp32_reuse": (1, 64), "fp32m_reuse": (2, 64)}


def _rel(a, b) -> float:
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _run(d, state, precision=0, reuse=0):
    st = ys.Step(ys.params_from_state(state), state["field_h0"], state["field_c0"], state["field_s0"])
    st.set_precision(precision)
    st.set_amg_reuse(reuse)
    stats = st.advance(int(d["steps_done"]))
    h, c = st.fields()
    return st, stats, h, c


@pytest.mark.parametrize("f", _big.BIG, ids=IDS)
def test_big_patterns_bitwise(f):
    d, state = _big.load(f)
    st = ys.Step(ys.params_from_state(state), state["field_h0"], state["field_c0"], state["field_s0"])
    rowptr, col, bc = st.pattern()
    assert _big.field_hash(rowptr) == d["sha_rowptr"] and _big.field_hash(col) == d["sha_col"]
    assert _big.field_hash(bc) == d["sha_bc"]
    crow, ccol = st.conc_pattern()
    assert _big.field_hash(crow) == d["sha_rowptr_c"] and _big.field_hash(ccol) == d["sha_col_c"]


@pytest.mark.parametrize("f", _big.BIG, ids=IDS)
def test_big_fields_fp64(f):
    d, state = _big.load(f)
    _, stats, h, c = _run(d, state)
    assert stats["steps"] == d["steps_done"]
    assert _rel(h, d["field_h1"]) <= 1e-10, _rel(h, d["field_h1"])
    if "field_c1" in d:
        assert _rel(c, d["field_c1"]) <= 1e-10, _rel(c, d["field_c1"])
    assert abs(stats["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"])


@pytest.mark.parametrize("form", list(FORMS))
@pytest.mark.parametrize("f", _big.BIG, ids=IDS)
def test_big_fields_fp32_forms(f, form):
    d, state = _big.load(f)
    _, stats, h, c = _run(d, state, *FORMS[form])
    assert _rel(h, d["field_h1"]) <= 1e-8, _rel(h, d["field_h1"])
    if "field_c1" in d:
        assert _rel(c, d["field_c1"]) <= 1e-8, _rel(c, d["field_c1"])
    assert abs(stats["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"])


def test_big_first_solve_bitwise_at_512():
    """The first Newton system of the 512^2 film (as the device assembles it)
    solved by the device and by the CPU oracle: bit for bit, hierarchy
    included."""
    f = [p for p in _big.BIG if p.stem == "big_allphys_512"][0]
    d, state = _big.load(f)
    st = ys.Step(ys.params_from_state(state), state["field_h0"], state["field_c0"], state["field_s0"])
    rowptr, col, _ = st.pattern()
    ia, rhs = st.system(state["field_h0"], state["field_h0"], state["dt"])
    scol, ssrc = _systems.sorted_mirror(rowptr, col)
    sysd = {"rowptr": rowptr, "col": col, "sorted_col": scol, "sorted_src": ssrc, "values": ia, "rhs": rhs,
            "x0": np.zeros(rhs.size), "precondition": state["lin_precond"], "scaling": state["lin_scaling"],
            "max_iteration": state["lin_maxit"], "epsilon": state["lin_eps"], "conc": 0, "n": rhs.size}
    be = yz.B200Backend()
    s = yz.LinearSolverSettings(int(sysd["precondition"]), bool(sysd["scaling"]), int(sysd["max_iteration"]),
                                float(sysd["epsilon"]), False)
    x = np.zeros(rhs.size)
    ret, it, res = be.Solve(s, yz.CrsPattern(rowptr, col, scol, ssrc), ia, rhs, x)
    o = _oracle.OracleSolver()
    o_ret, o_it, o_res, o_x = o.solve(sysd)
    assert (ret, it, res) == (o_ret, o_it, o_res), ((ret, it, res), (o_ret, o_it, o_res))
    assert np.array_equal(x, o_x)
    gl, ol = be.levels(), o.levels()
    assert len(gl) == len(ol) and len(gl) > 2
    for a, b in zip(gl, ol):
        assert (a["rows"], a["nnz_a"], a["nnz_p"], a["direct"]) == (b["rows"], b["nnz_a"], b["nnz_p"], b["direct"])
        assert np.array_equal(a["a_ptr"], b["a_ptr"]) and np.array_equal(a["a_col"], b["a_col"])
        assert np.array_equal(a["a_val"], b["a_val"])
        if not a["direct"]:
            assert np.array_equal(a["agg"], b["agg"])
            assert np.array_equal(a["p_ptr"], b["p_ptr"]) and np.array_equal(a["p_col"], b["p_col"])
            assert np.array_equal(a["p_val"], b["p_val"])
