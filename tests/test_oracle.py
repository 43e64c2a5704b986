"""The CPU oracle of the linear solve, pinned before it is trusted.

* The golden fixtures were written by the reference's own sources (compiled by
  oracle/Makefile) solving with this oracle inside them; the standalone
  oracle library must give the same answers to the bit.
* The properties the reference's test_linear_solver.cpp pins for a backend
  (analytic 1-D Poisson, second order, determinism, zero right-hand side,
  inputs untouched) hold for the AMG flavour as well.
* When the reference-built oracle is present, the reference's own unit tests
  (yuzen/tests, 93 cases) pass with it.
"""
import subprocess

import numpy as np
import pytest

import _oracle
import _systems
import dumpio
from pathlib import Path

GOLDEN = sorted(Path(__file__).parent.joinpath("golden").glob("solve_*.npz"))


def _cases():
    for f in GOLDEN:
        for j, d in enumerate(dumpio.load_npz(f)):
            yield pytest.param(d, id=f"{f.stem}-{j}")


@pytest.mark.parametrize("d", list(_cases()))
def test_oracle_reproduces_reference_run(d):
    o = _oracle.OracleSolver(int(d["flavour"]))
    ret, it, res, x = o.solve(d)
    assert ret == d["ret"]
    assert it == d["iter"]
    assert res == d["resid"]
    assert np.array_equal(x, d["x"])


@pytest.mark.parametrize("d", list(_cases()))
def test_oracle_solution_solves_the_system(d):
    o = _oracle.OracleSolver(int(d["flavour"]))
    ret, it, res, x = o.solve(d)
    assert ret == 0
    # residual of the unscaled system: the tolerance holds on the row-scaled
    # system, up to the rounding floor eps |A| |x| of a fourth-order stencil
    y = _oracle.spmv(d["rowptr"], d["col"], d["values"], x)
    r = np.linalg.norm(y - d["rhs"])
    b = np.linalg.norm(d["rhs"])
    absA = np.zeros(d["n"])
    np.add.at(absA, np.repeat(np.arange(d["n"]), np.diff(d["rowptr"])), np.abs(d["values"]))
    # and the recursive-residual floor of BiCGStab, eps |b - A x0|: the initial
    # guess is the last Newton correction, which can be far larger than b
    r0 = np.linalg.norm(_oracle.spmv(d["rowptr"], d["col"], d["values"], d["x0"]) - d["rhs"])
    floor = 1e-13 * (absA.max() * np.abs(x).max() * np.sqrt(d["n"]) + r0)
    diag = np.abs(d["values"][d["rowptr"][:-1]])
    slack = diag.max() / max(diag.min(), 1e-300)
    assert r <= 10 * d["epsilon"] * b * slack + floor


@pytest.mark.parametrize("pre", [0, 1, 2])
def test_poisson_matches_analytic(pre):
    """test_linear_solver.cpp:87-116, through the AMG flavour."""
    p = _systems.poisson1d(202)
    o = _oracle.OracleSolver(_oracle.YZO_AMG)
    ret, it, res, x = o.solve(p, precondition=pre)
    assert ret == 0 and res < 1e-11
    err = np.max(np.abs(x[1:-1] - p["exact"][1:-1]))
    assert err < 1e-4


def test_poisson_second_order():
    """test_linear_solver.cpp:118-143 (the AMG flavour needs n > 3000 to coarsen)."""
    prev = None
    for n in (52, 102, 202, 402, 802, 1602, 3202, 6402):
        p = _systems.poisson1d(n)
        ret, it, res, x = _oracle.OracleSolver(_oracle.YZO_AMG).solve(p, max_iteration=20000)
        assert ret == 0
        err = np.max(np.abs(x[1:-1] - p["exact"][1:-1]))
        if prev is not None and n <= 1602:
            assert err < prev * 0.5
        prev = err


def test_same_answer_twice():
    p = _systems.film_system(60, seed=3)
    a = _oracle.OracleSolver().solve(p)
    b = _oracle.OracleSolver().solve(p)
    assert a[:3] == b[:3] and np.array_equal(a[3], b[3])


def test_zero_rhs_gives_zero():
    p = _systems.poisson1d(52)
    p["rhs"] = np.zeros(52)
    ret, it, res, x = _oracle.OracleSolver().solve(p)
    assert ret == 0 and np.all(x == 0)


def test_inputs_untouched():
    p = _systems.film_system(40, seed=1)
    v0, r0 = p["values"].copy(), p["rhs"].copy()
    _oracle.OracleSolver().solve(p)
    assert np.array_equal(v0, p["values"]) and np.array_equal(r0, p["rhs"])


def test_hierarchy_structure():
    p = _systems.film_system(96, seed=2)
    o = _oracle.OracleSolver()
    ret, it, res, x = o.solve(p)
    assert ret == 0
    lv = o.levels()
    assert len(lv) >= 2 and lv[-1]["direct"] and lv[-1]["rows"] <= 500
    for a, b in zip(lv, lv[1:]):
        assert b["rows"] < a["rows"]
        agg = a["agg"]
        assert agg.max() == b["rows"] - 1
        # every aggregate is non-empty
        assert np.all(np.bincount(agg[agg >= 0], minlength=b["rows"]) > 0)


def test_backoff_memory_roundtrip():
    """TryBackoff (LinearSolverBackend.cpp:262-270): a failed SPAI0 try is
    skipped for 16 solves, then 32; Memory() carries it."""
    p = _systems.film_system(40, seed=5, stiff=1e6)
    o = _oracle.OracleSolver()
    ret, it, res, x = o.solve(p, conc=1, max_iteration=2)
    assert o.memory() == [16.0, 32.0]


def test_reference_unit_tests_pass_with_oracle():
    if not _oracle.REF_TESTS.exists():
        pytest.skip("reference-built oracle not present (make -C oracle ref)")
    r = subprocess.run([str(_oracle.REF_TESTS)], capture_output=True, text=True, timeout=900,
                       env={"OMP_NUM_THREADS": "4", "PATH": "/usr/bin:/bin"})
    assert r.returncode == 0, r.stdout[-3000:]
    assert "Status: SUCCESS" in r.stdout


def test_oracle_fault_switch():
    """The oracle's copy of the reference's YUZEN_FAULT_AMGCL switch: the
    chosen solve returns 2 before iterating and leaves x as given."""
    import _systems
    d = _systems.film_system(40, seed=7)
    x0 = np.full(d["n"], 0.5)
    _oracle.fault_inject(1, 1)
    try:
        ret, it, res, x = _oracle.OracleSolver().solve(d, x0=x0)
        assert ret == 2 and it == 0 and np.array_equal(x, x0)
        assert _oracle.OracleSolver().solve(d, x0=x0)[0] == 0
    finally:
        _oracle.fault_inject(0, 0)


_THREADS_CHILD = r"""
import sys
sys.path[:0] = [sys.argv[1] + "/tests", sys.argv[1] + "/tests/golden"]
import hashlib
import numpy as np
import _oracle, _systems
p = _systems.film_system(120, seed=5)
r = _oracle.OracleSolver().solve(p)
print(r[0], r[1], repr(r[2]), hashlib.sha256(np.ascontiguousarray(r[3]).tobytes()).hexdigest())
"""


def test_oracle_thread_count_invariant():
    """The oracle's vector loops run on OpenMP threads over the fixed
    reduction tree, so one thread and eight give the same return code,
    iteration count, residual and x to the bit (the reference's
    test_linear_solver.cpp asks a backend for the same)."""
    import os
    import sys
    root = Path(__file__).resolve().parents[1]
    outs = []
    for t in ("1", "8"):
        r = subprocess.run([sys.executable, "-c", _THREADS_CHILD, str(root)], capture_output=True, text=True,
                           env=dict(os.environ, OMP_NUM_THREADS=t), timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(r.stdout.strip().splitlines()[-1])
    assert outs[0] == outs[1], outs
