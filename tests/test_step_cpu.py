"""Host side of the whole-step seam, without a device: the CRS pattern of
I + theta dt J is the reference's to the bit (the whole-step probe dumps the
pattern C_ImplicitSolver::Alloc fixed, ImplicitSolver.cpp:60-81), and the
parameter block carries the probe's state."""
from pathlib import Path

import numpy as np
import pytest

import stateio
from yuzen_b200 import step as ys

GOLDEN = Path(__file__).parent.joinpath("golden")
STEPS = sorted(GOLDEN.glob("step_*.npz"))


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


@pytest.mark.parametrize("bc,why", [
    ((2, 0, 4, 0), "Pinning next to an Outlet"),        # BC: Pinning-Outlet, not implemented in the reference
    ((3, 0, 2, 0), "FreshInlet next to a Pinning"),     # BC: Inlet-Pinning
    ((2, 0, 2, 0), "two Pinning edges meeting"),        # three corner rows left without a condition
    ((7, 0, 0, 0), "an unknown kind"),
])
def test_refused_edges(bc, why):
    d = stateio.load_npz(GOLDEN / "step_upwind_48.npz")
    p = ys.params_from_state(d)
    for e in range(4):
        p.bc[e] = bc[e]
    with pytest.raises(Exception):
        ys.pattern_2d(p)
