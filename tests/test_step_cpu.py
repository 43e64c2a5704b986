"""Host side of the whole-step seam, without a device: the CRS pattern of
I + theta dt J is the reference's to the bit (the whole-step probe dumps the
pattern C_ImplicitSolver::Alloc fixed, ImplicitSolver.cpp:60-81), and the
parameter block carries the probe's state."""
from pathlib import Path

import numpy as np
import pytest

import stateio
from yuzen_b200 import step as ys

STEPS = sorted(Path(__file__).parent.joinpath("golden").glob("step_*.npz"))


@pytest.mark.parametrize("f", STEPS, ids=[f.stem for f in STEPS])
def test_pattern_bitwise(f):
    d = stateio.load_npz(f)
    rowptr, col, bc = ys.pattern_2d(ys.params_from_state(d))
    assert np.array_equal(rowptr, d["rowptr"])
    assert np.array_equal(col, d["col"])
    assert np.array_equal(bc, d["bc"])


@pytest.mark.parametrize("f", STEPS, ids=[f.stem for f in STEPS])
def test_params_from_state(f):
    d = stateio.load_npz(f)
    p = ys.params_from_state(d)
    assert (p.nx, p.ny) == (d["nx"], d["ny"])
    assert p.dx == d["dx"] and p.Dp == d["Dp"] and p.dt == d["dt"]
    assert p.lin.epsilon == d["lin_eps"]


def test_unsupported_edges_are_refused():
    d = stateio.load_npz(STEPS[0])
    p = ys.params_from_state(d)
    p.bc[0] = 4  # Outlet
    with pytest.raises(Exception):
        ys.pattern_2d(p)
