"""Parity of the device implicit step with the reference.

Each fixture holds a case as the reference's own model built it (the
whole-step probe), the system of its first Newton pass as the reference
solved it, and the state after N steps of the reference's time loop.

Bars: the CRS pattern bit for bit; the first pass's I + theta dt J entry by
entry within 1e-12 of its row's largest entry and the right-hand side within
1e-9 of its largest entry (the device's exp/pow/log1p may differ from the
host's in the last place, and A h is a difference of terms ~1/dx^4 larger);
h after N steps within 1e-10 relative L2, and the clock to 1e-12.
"""
from pathlib import Path

import numpy as np
import pytest

import stateio
from yuzen_b200 import step as ys

pytestmark = pytest.mark.gpu
STEPS = sorted(Path(__file__).parent.joinpath("golden").glob("step_*.npz"))
IDS = [f.stem for f in STEPS]


def make(d):
    return ys.Step(ys.params_from_state(d), d["field_h0"], d["field_c0"], d["field_s0"])


@pytest.mark.parametrize("f", STEPS, ids=IDS)
def test_pattern_bitwise(f):
    d = stateio.load_npz(f)
    rowptr, col, bc = make(d).pattern()
    assert np.array_equal(rowptr, d["rowptr"]) and np.array_equal(col, d["col"]) and np.array_equal(bc, d["bc"])


@pytest.mark.parametrize("f", STEPS, ids=IDS)
def test_first_newton_system(f):
    d = stateio.load_npz(f)
    st = make(d)
    ia, rhs = st.system(d["field_h0"], d["field_h0"], d["dt"])
    ref_ia, ref_rhs = d["sys_values"], d["sys_rhs"]
    rp = d["rowptr"]
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    rowmax = np.zeros(rp.size - 1)
    np.maximum.at(rowmax, rows, np.abs(ref_ia))
    err = np.abs(ia - ref_ia) / rowmax[rows]
    assert err.max() <= 1e-12, err.max()
    scale = np.abs(ref_rhs).max()
    assert np.abs(rhs - ref_rhs).max() <= 1e-9 * scale + 1e-300, (np.abs(rhs - ref_rhs).max(), scale)


@pytest.mark.parametrize("f", STEPS, ids=IDS)
def test_fields_after_steps(f):
    d = stateio.load_npz(f)
    st = make(d)
    stats = st.advance(d["steps_done"])
    h, c = st.fields()
    ref = d["field_h1"]
    rel = np.linalg.norm(h - ref) / np.linalg.norm(ref)
    assert rel <= 1e-10, rel
    assert abs(stats["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"]), (stats["time"], d["t_end"])
    assert np.array_equal(c, d["field_c1"])
