"""The ConcZ model without a device: the oracle's fixtures (the reference's
own runs of its CZ model, oracle/probe/yz_probe_cz.cpp, made by
tests/golden/make_golden.py) pinned by the properties the model holds --
the solute of a closed film conserved while its solvent evaporates, the
film's volume losing exactly what evaporated -- and the library's patterns of
both matrices against the reference's storage order."""
from pathlib import Path

import numpy as np
import pytest

import stateio

GOLD = Path(__file__).resolve().parent / "golden"
CASES = ["cz_sym_16", "cz_per_koren_16", "cz_spin_fixed_18", "cz_sym_64", "cz_min_4", "cz_vanleer_per_20"]


def load(name):
    return stateio.load_npz(GOLD / f"{name}.npz")


def solute(d, h, c):
    """sum over the real columns of h times the mean c of the real levels"""
    nx, ny, nz = d["nx"], d["ny"], d["nz"]
    H = h.reshape(ny, nx)[2:-2, 2:-2]
    C = c.reshape(nz, ny, nx)[2:-2, 2:-2, 2:-2]
    return float((H * C.mean(axis=0)).sum())


@pytest.mark.parametrize("name", CASES)
def test_reference_run_conserves_solute(name):
    """The reference's CZ step conserves the solute of a closed film (its
    conservative form on the moving zeta grid, CZ_ConcEquation_2D.cpp:84-130)
    while the solvent evaporates: the oracle's run holds it to rounding."""
    d = load(name)
    s0, s1 = solute(d, d["h0"], d["c0"]), solute(d, d["h1"], d["c1"])
    assert abs(s1 - s0) <= 1e-11 * abs(s0), (s0, s1)
    if d["on_evap"]:
        nx, ny = d["nx"], d["ny"]
        v0 = d["h0"].reshape(ny, nx)[2:-2, 2:-2].sum()
        v1 = d["h1"].reshape(ny, nx)[2:-2, 2:-2].sum()
        assert v1 < v0


@pytest.mark.parametrize("name", CASES)
def test_patterns_match_the_reference(name):
    from yuzen_b200 import cz
    d = load(name)
    p = cz.params_from_record(d)
    for which, pre in ((0, "h"), (1, "c")):
        rowptr, col, bc = cz.build_pattern(p, which)
        assert np.array_equal(rowptr, d[pre + "_rowptr"])
        assert np.array_equal(col, d[pre + "_col"])
        assert np.array_equal(bc, d[pre + "_bc"])


@pytest.mark.parametrize("kind", [2, 3, 4])
def test_edges_the_reference_refuses_are_refused(kind):
    """CheckParameters.cpp:340-353: the CZ model implements Symmetry and
    Periodic edges only."""
    from yuzen_b200 import YzError, cz
    p = cz.params_from_record(load("cz_sym_16"))
    p.bc[1] = kind
    with pytest.raises(YzError, match="Symmetry and Periodic"):
        cz.build_pattern(p, 0)


def test_unpaired_periodic_edge_is_refused():
    from yuzen_b200 import YzError, cz
    p = cz.params_from_record(load("cz_sym_16"))
    p.bc[0] = 1
    with pytest.raises(YzError, match="opposite edge"):
        cz.build_pattern(p, 1)


def test_fixture_covers_the_paths():
    """What the fixtures exercise: the coupling passes (Marangoni), the
    concentration's own two stages with the limited scheme, the LTE control's
    cuts, a fixed step, more than one AMG level."""
    a, b, c, big = (load(n) for n in CASES[:4])
    assert a["on_sc"] == 1 and a["coupling_passes"] > 0 and a["dt_control"] == 1 and a["dt_end"] < a["dt"]
    assert b["on_sc"] == 0 and b["c_scheme"] == 7 and b["bc"][0] == 1 and b["on_vg"] == 1 and b["on_hg"] == 1
    assert c["dt_control"] == 0 and c["on_cf"] == 1
    assert (big["nx"] - 4) * (big["ny"] - 4) > 3000


def test_bench_size_builder_matches_the_fixture():
    """The seeded 256^2 x 16 film of yuzen_b200.cases.cz_bumps is the one the
    reference ran for tests/golden/czbig_256.npz (make_golden checked every
    parameter against the reference's set-up when it was made)."""
    from yuzen_b200 import cases
    ref = stateio.load_npz(GOLD / "czbig_256.npz")
    rec = cases.cz_bumps(N=256, Nz=16, steps=3).record()
    assert np.array_equal(rec["h0"], ref["h0"])
    assert (rec["nx"], rec["ny"], rec["nz"]) == (ref["nx"], ref["ny"], ref["nz"])
