"""Parity of the CUDA linear solve with the CPU oracle.

The FP64 solve is specified operation for operation by the oracle
(oracle/solver/yzo_solver.cpp), so the bar is bit equality: the answer x, the
iteration count, the reported residual, the return code, and the AMG
hierarchy (every level's matrix, prolongation and aggregate map).
"""
from pathlib import Path

import numpy as np
import pytest

import _oracle
import _systems
import dumpio
import yuzen_b200 as yz

pytestmark = pytest.mark.gpu
GOLDEN = sorted(Path(__file__).parent.joinpath("golden").glob("solve_*.npz"))


def _amg_cases():
    for f in GOLDEN:
        for j, d in enumerate(dumpio.load_npz(f)):
            if int(d["flavour"]) == _oracle.YZO_AMG:
                yield pytest.param(d, id=f"{f.stem}-{j}")


def gpu_solve(d, backend=None, **over):
    s = yz.LinearSolverSettings(precondition=int(over.get("precondition", d["precondition"])),
                                scaling=bool(over.get("scaling", d["scaling"])),
                                maxIteration=int(over.get("max_iteration", d["max_iteration"])),
                                epsilon=float(over.get("epsilon", d["epsilon"])),
                                conc=bool(over.get("conc", d["conc"])))
    be = backend or yz.B200Backend()
    pat = yz.CrsPattern(d["rowptr"], d["col"], d["sorted_col"], d["sorted_src"])
    x = np.array(d["x0"], dtype=np.float64, copy=True)
    ret, it, res = be.Solve(s, pat, d["values"], d["rhs"], x)
    return ret, it, res, x, be


def assert_same(a, b):
    assert a[0] == b[0], ("ret", a[0], b[0])
    assert a[1] == b[1], ("iter", a[1], b[1])
    assert a[2] == b[2], ("resid", a[2], b[2])
    assert np.array_equal(a[3], b[3]), np.max(np.abs(a[3] - b[3]))


@pytest.mark.parametrize("n", [0, 1, 255, 4095, 4096, 4097, 300001, 1 << 20])
def test_dot_bitwise(n):
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n) * 1e3
    assert yz.dot(x, y) == _oracle.dot(x, y)


@pytest.mark.parametrize("d", list(_amg_cases()))
def test_spmv_bitwise(d):
    x = np.random.default_rng(1).standard_normal(d["n"])
    assert np.array_equal(yz.spmv(d["rowptr"], d["col"], d["values"], x),
                          _oracle.spmv(d["rowptr"], d["col"], d["values"], x))


@pytest.mark.parametrize("d", list(_amg_cases()))
def test_golden_solve_bitwise(d):
    g = gpu_solve(d)
    o = _oracle.OracleSolver().solve(d)
    assert_same(g[:4], o)
    # and the oracle's answer inside the reference run
    assert g[0] == d["ret"] and g[1] == d["iter"] and g[2] == d["resid"]
    assert np.array_equal(g[3], d["x"])


def _levels_equal(gl, ol):
    assert len(gl) == len(ol)
    for a, b in zip(gl, ol):
        assert (a["rows"], a["nnz_a"], a["nnz_p"], a["direct"]) == (b["rows"], b["nnz_a"], b["nnz_p"], b["direct"])
        assert np.array_equal(a["a_ptr"], b["a_ptr"]) and np.array_equal(a["a_col"], b["a_col"])
        assert np.array_equal(a["a_val"], b["a_val"])
        if not a["direct"]:
            assert np.array_equal(a["agg"], b["agg"])
            if a["nnz_p"]:
                assert np.array_equal(a["p_ptr"], b["p_ptr"]) and np.array_equal(a["p_col"], b["p_col"])
                assert np.array_equal(a["p_val"], b["p_val"])


@pytest.mark.parametrize("d", [c for c in _amg_cases() if not c.values[0]["conc"]])
def test_hierarchy_bitwise(d):
    g = gpu_solve(d)
    o = _oracle.OracleSolver()
    o.solve(d)
    _levels_equal(g[4].levels(), o.levels())


@pytest.mark.parametrize("N,seed,periodic", [(96, 2, False), (200, 7, True), (384, 11, False)])
def test_synthetic_film_bitwise(N, seed, periodic):
    d = _systems.film_system(N, seed=seed, periodic=periodic)
    g = gpu_solve(d)
    o = _oracle.OracleSolver()
    assert_same(g[:4], o.solve(d))
    assert g[0] == 0
    _levels_equal(g[4].levels(), o.levels())


@pytest.mark.parametrize("pre,scaling,conc", [(0, 1, 0), (1, 1, 0), (2, 0, 0), (2, 1, 1)])
def test_settings_variants_bitwise(pre, scaling, conc):
    d = _systems.film_system(80, seed=4)
    g = gpu_solve(d, precondition=pre, scaling=scaling, conc=conc)
    o = _oracle.OracleSolver().solve(d, precondition=pre, scaling=scaling, conc=conc)
    assert_same(g[:4], o)


def test_backoff_sequence_matches_oracle():
    """A SPAI0 try that fails backs off for 16 solves (TryBackoff); the GPU
    context carries the same counters across a sequence of solves."""
    d = _systems.film_system(48, seed=5, stiff=30.0)
    be = yz.B200Backend()
    o = _oracle.OracleSolver()
    for k in range(3):
        g = gpu_solve(d, backend=be, conc=1, max_iteration=40)
        r = o.solve(d, conc=1, max_iteration=40)
        assert_same(g[:4], r)
        assert be.Memory() == o.memory()
    be.SetMemory([0.0, 16.0])
    assert be.Memory() == [0.0, 16.0]


def test_poisson_analytic_through_gpu():
    p = _systems.poisson1d(202)
    ret, it, res, x, _ = gpu_solve(p)
    assert ret == 0 and res < 1e-11
    assert np.max(np.abs(x[1:-1] - p["exact"][1:-1])) < 1e-4


def test_zero_rhs_and_untouched_inputs():
    d = _systems.film_system(40, seed=9)
    d["rhs"] = np.zeros(d["n"])
    v0 = d["values"].copy()
    ret, it, res, x, _ = gpu_solve(d)
    assert ret == 0 and np.all(x == 0) and np.array_equal(v0, d["values"])


def test_usage_errors_are_reported():
    be = yz.B200Backend()
    bad = yz.CrsPattern(np.array([0, 0], np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    with pytest.raises(yz.YzError):
        be.SetPattern(bad)
    x = np.zeros(1)
    with pytest.raises(yz.YzError):
        be.SolveDevice(yz.LinearSolverSettings(), 1, 1, 1)


def test_kernels_actually_launch():
    d = _systems.film_system(64, seed=1)
    g = gpu_solve(d)
    assert g[4].launches() > 50


_GRAPH_CHILD = r"""
import sys
sys.path[:0] = [sys.argv[1], sys.argv[1] + '/tests', sys.argv[1] + '/tests/golden']
import numpy as np
import _oracle, _systems
import yuzen_b200 as yz
d = _systems.film_system(200, seed=7, periodic=True)
s = yz.LinearSolverSettings(int(d['precondition']), bool(d['scaling']), int(d['max_iteration']),
                            float(d['epsilon']), bool(d['conc']))
be = yz.B200Backend()
pat = yz.CrsPattern(d['rowptr'], d['col'], d['sorted_col'], d['sorted_src'])
x = np.array(d['x0'], copy=True)
ret, it, res = be.Solve(s, pat, d['values'], d['rhs'], x)
o = _oracle.OracleSolver().solve(d)
assert (ret, it, res) == tuple(o[:3]), ((ret, it, res), o[:3])
assert np.array_equal(x, o[3])
print('ok', it)
"""


def test_stream_loop_bitwise():
    """The iterations launched from the stream (YZ_GRAPH=0: one iteration kept
    in flight, the form kernel timing uses) give the oracle's answer to the
    bit, as the default CUDA-graph form (a conditional while node whose body
    is one BiCGStab iteration) does."""
    import os
    import subprocess
    import sys
    repo = str(Path(__file__).resolve().parents[1])
    r = subprocess.run([sys.executable, "-c", _GRAPH_CHILD, repo], env=dict(os.environ, YZ_GRAPH="0"),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]


def _true_residual(d, x):
    """|b - A x| / |b| of the row-scaled system (the one the solve's
    tolerance is on), in numpy FP64"""
    n, rp, col, val = d["n"], d["rowptr"], d["col"], d["values"]
    rows = np.repeat(np.arange(n), np.diff(rp))
    r = np.asarray(d["rhs"], np.float64) - np.bincount(rows, weights=val * x[col], minlength=n)
    b = np.asarray(d["rhs"], np.float64).copy()
    if int(d["scaling"]):
        dia = val[rp[:-1]]              # the diagonal is stored first
        ok = np.abs(dia) >= 1e-30
        r[ok] /= dia[ok]
        b[ok] /= dia[ok]
    return np.linalg.norm(r) / np.linalg.norm(b)


def _abs_product(d, x):
    """| |A| |x| | / |b| of the row-scaled system: the size of the change
    that rounding the matrix's entries by a relative 1 can make in A x"""
    n, rp, col, val = d["n"], d["rowptr"], d["col"], d["values"]
    rows = np.repeat(np.arange(n), np.diff(rp))
    ax = np.bincount(rows, weights=np.abs(val) * np.abs(x[col]), minlength=n)
    b = np.asarray(d["rhs"], np.float64).copy()
    if int(d["scaling"]):
        dia = np.abs(val[rp[:-1]])
        ok = dia >= 1e-30
        ax[ok] /= dia[ok]
        b[ok] /= dia[ok]
    return np.linalg.norm(ax) / np.linalg.norm(b)


_FP32_CASES = [c for c in _amg_cases() if not c.values[0]["conc"]] + [
    pytest.param(_systems.film_system(200, seed=7, periodic=True), id="film200-periodic"),
    pytest.param(_systems.film_system(384, seed=11), id="film384")]


@pytest.mark.parametrize("d", _FP32_CASES)
def test_fp32_cycle_meets_the_tolerance(d):
    """The V-cycle in float (PREC_FP32_CYCLE) changes the preconditioner only:
    the hierarchy is the FP64 set-up's (the oracle's to the bit), and the
    FP64 BiCGStab around the cycle converges to the same tolerance in about
    as many iterations.  Its x has the true residual of the oracle's x (the
    recurrence's residual drifts from the true one by about the same amount
    in both, far above the tolerance where the start was far off) and lies
    within what that residual allows of the oracle's x."""
    be = yz.B200Backend()
    be.SetPrecision(yz.PREC_FP32_CYCLE)
    g = gpu_solve(d, backend=be)
    o = _oracle.OracleSolver()
    r = o.solve(d)
    _levels_equal(be.levels(), o.levels())
    assert g[0] == r[0] == 0, (g[:3], r[:3])
    eps = float(d["epsilon"])
    assert g[2] <= eps
    tg, to = _true_residual(d, g[3]), _true_residual(d, r[3])
    assert tg <= max(2.0 * eps, 4.0 * to), (tg, to, eps)
    assert g[1] <= r[1] + max(2, r[1] // 4), (g[1], r[1])
    assert np.linalg.norm(g[3] - r[3]) <= 1e4 * max(eps, to) * np.linalg.norm(r[3]) + 1e-300, \
        (np.linalg.norm(g[3] - r[3]) / np.linalg.norm(r[3]), eps, to)


def test_precision_usage_errors():
    be = yz.B200Backend()
    with pytest.raises(yz.YzError):
        be.SetPrecision(7)
    be.SetPrecision(yz.PREC_FP32_CYCLE)
    be.SetPrecision(yz.PREC_FP64)


def _height_sequences():
    """the film's solves of each golden run, in the order the reference made
    them (one pattern per run)"""
    for f in GOLDEN:
        seq = [d for d in dumpio.load_npz(f) if int(d["flavour"]) == _oracle.YZO_AMG and not d["conc"]]
        if len(seq) >= 2:
            yield pytest.param(seq, id=f.stem)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32cycle"])
@pytest.mark.parametrize("seq", list(_height_sequences()))
def test_amg_reuse_meets_the_tolerance(seq, precision):
    """With hierarchy reuse on, the solves after the first run on the first
    solve's hierarchy (fewer launches: no set-up) and the FP64 BiCGStab still
    meets each solve's tolerance, with the true residual of the oracle's own
    answer."""
    fresh, reused = yz.B200Backend(), yz.B200Backend()
    for be in (fresh, reused):
        be.SetPrecision(precision)
    reused.SetAmgReuse(8)
    n_fresh, n_reused = [], []
    d0 = seq[0]
    pat = yz.CrsPattern(d0["rowptr"], d0["col"], d0["sorted_col"], d0["sorted_src"])
    for d in seq:
        assert np.array_equal(d["rowptr"], d0["rowptr"]) and np.array_equal(d["col"], d0["col"])
        s = yz.LinearSolverSettings(int(d["precondition"]), bool(d["scaling"]), int(d["max_iteration"]),
                                    float(d["epsilon"]), bool(d["conc"]))
        for be, counts in ((fresh, n_fresh), (reused, n_reused)):
            l0 = be.launches()
            x = np.array(d["x0"], dtype=np.float64, copy=True)
            g = be.Solve(s, pat, d["values"], d["rhs"], x) + (x,)
            counts.append(be.launches() - l0)
            r = _oracle.OracleSolver().solve(d)
            assert g[0] == 0, g[:3]
            tg, to = _true_residual(d, g[3]), _true_residual(d, r[3])
            assert tg <= max(2.0 * float(d["epsilon"]), 4.0 * to), (tg, to, d["epsilon"])
    #  the second and later solves skipped the set-up (while the iteration
    #  counts stayed near the first solve's)
    assert any(b < a for a, b in zip(n_fresh[1:], n_reused[1:])), (n_fresh, n_reused)


def test_amg_reuse_usage_errors():
    be = yz.B200Backend()
    with pytest.raises(yz.YzError):
        be.SetAmgReuse(-1)
    be.SetAmgReuse(0)


def test_amg_reuse_failure_sets_up_afresh():
    """A solve on a reused hierarchy that fails is repeated from the caller's
    guess on a new set-up.  The second system is far from the first (another
    mobility field, 3 times stiffer: 814 iterations against 38) and its cap is
    the iteration count the oracle needs with a new set-up: when the stale
    hierarchy misses the cap, the repeat is the oracle's solve to the bit (its
    iterations come on top of the failed ones); when it does not, the answer
    meets the tolerance."""
    a = _systems.film_system(96, seed=2)
    b = _systems.film_system(96, seed=9, stiff=3.0)
    o = _oracle.OracleSolver().solve(b)
    assert o[0] == 0
    be = yz.B200Backend()
    be.SetAmgReuse(8)
    pat = yz.CrsPattern(a["rowptr"], a["col"], a["sorted_col"], a["sorted_src"])
    for d, cap in ((a, int(a["max_iteration"])), (b, int(o[1]))):
        s = yz.LinearSolverSettings(int(d["precondition"]), bool(d["scaling"]), cap, float(d["epsilon"]),
                                    bool(d["conc"]))
        x = np.array(d["x0"], dtype=np.float64, copy=True)
        ret, it, res = be.Solve(s, pat, d["values"], d["rhs"], x)
        assert ret == 0, (ret, it, res)
    if it > o[1]:
        assert res == o[2] and np.array_equal(x, o[3])
    else:
        assert res <= float(b["epsilon"])


@pytest.mark.parametrize("d", _FP32_CASES)
def test_fp32_matrix_solves_the_rounded_system(d):
    """PREC_FP32_MATRIX: the BiCGStab's SpMVs read the matrix rounded to
    float.  The solve converges to its tolerance on that system; measured on
    the FP64 system its residual is within what rounding the matrix to float
    can change it by, 2^-24 |A| |x| (a few times that, against the norm of
    b; large on the ill-conditioned 1-D fourth-order systems), and the
    hierarchy is still the FP64 set-up's."""
    be = yz.B200Backend()
    be.SetPrecision(yz.PREC_FP32_MATRIX)
    g = gpu_solve(d, backend=be)
    o = _oracle.OracleSolver()
    r = o.solve(d)
    _levels_equal(be.levels(), o.levels())
    assert g[0] == 0, g[:3]
    assert g[2] <= float(d["epsilon"])
    tg, to = _true_residual(d, g[3]), _true_residual(d, r[3])
    rounding = 4.0 * 2.0 ** -24 * _abs_product(d, g[3])
    assert tg <= max(2.0 * float(d["epsilon"]), 4.0 * to) + rounding, (tg, to, rounding)


_FUSE_CHILD = r"""
import json, sys
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/tests", sys.argv[1] + "/tests/golden"]
import numpy as np
import _systems
import yuzen_b200 as yz
import test_solver_gpu as t
d = _systems.film_system(384, seed=11)
be = yz.B200Backend()
be.SetPrecision(int(sys.argv[2]))
g = t.gpu_solve(d, backend=be)
print(json.dumps({"ret": g[0], "it": g[1], "res": g[2], "true": t._true_residual(d, g[3]), "levels": len(be.levels()),
                  "x": float(np.linalg.norm(g[3]))}))
"""


@pytest.mark.parametrize("precision", [yz.PREC_FP32_CYCLE, yz.PREC_FP32_MATRIX])
def test_fused_coarse_levels_match_the_separate_kernels(precision):
    """The FP32 cycle's coarse levels with their way down (pre-smoothing,
    residual, restriction) and way up (prolongation, post-smoothing) each in
    one launch (YZ_FUSE_FROM=1: every level below the finest; the default
    fuses from level 2), against the same cycle with every phase a kernel of
    its own (YZ_FUSE_FROM=0): the same preconditioner up to float
    rounding, so both solves of a 384^2 film (a hierarchy of several levels)
    meet the tolerance with true residuals alike and iteration counts within
    a tenth (float rounding alone moves a count by a few)."""
    import json
    import os
    import subprocess
    import sys
    root = Path(__file__).resolve().parents[1]
    out = {}
    for key, val in (("fused", "1"), ("separate", "0")):
        env = dict(os.environ)
        env.pop("YZ_FUSE_FROM", None)
        if val is not None:
            env["YZ_FUSE_FROM"] = val
        r = subprocess.run([sys.executable, "-c", _FUSE_CHILD, str(root), str(precision)], capture_output=True,
                           text=True, env=env, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[key] = json.loads(r.stdout.strip().splitlines()[-1])
    a, b = out["fused"], out["separate"]
    assert a["levels"] == b["levels"] >= 3, (a, b)
    assert a["ret"] == b["ret"] == 0, (a, b)
    assert abs(a["it"] - b["it"]) <= max(3, b["it"] // 10), (a, b)
    assert a["true"] <= 4.0 * max(b["true"], 1e-300) + 1e-14, (a, b)
    assert abs(a["x"] - b["x"]) <= 1e-6 * b["x"], (a, b)


def test_tuning_shapes_and_sweeps():
    """yz_solver_set_tuning: out-of-range shapes are usage errors; every shape
    solves the 384^2 film to the tolerance in the FP32 cycle, and the finest
    level's five default sweeps take fewer iterations than the reference's
    one."""
    d = _systems.film_system(384, seed=11)
    be = yz.B200Backend()
    for bad in ((-2, 0, 0), (2, 3, 0), (2, 0, 9)):
        with pytest.raises(yz.YzError):
            be.SetTuning(*bad)
    its = {}
    for shape in ((-1, 0, 1), (-1, 0, 0), (0, 8, 0), (1, 4, 3)):
        be = yz.B200Backend()
        be.SetPrecision(yz.PREC_FP32_CYCLE)
        be.SetTuning(*shape)
        g = gpu_solve(d, backend=be)
        assert g[0] == 0 and g[2] <= float(d["epsilon"]), (shape, g[:3])
        its[shape] = g[1]
    assert its[(-1, 0, 0)] < its[(-1, 0, 1)], its
