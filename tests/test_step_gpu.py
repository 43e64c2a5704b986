"""Parity of the device implicit step with the reference.

Each fixture holds a case as the reference's own model built it (the
whole-step probe), the system of its first Newton pass as the reference
solved it, and the state after N steps of the reference's time loop.

Bars: the CRS pattern bit for bit; the first pass's I + theta dt J entry by
entry within 1e-12 of its row's largest entry and the right-hand side within
1e-9 of its largest entry (the device's exp/pow/log1p may differ from the
host's in the last place, and A h is a difference of terms ~1/dx^4 larger);
h after N steps within 1e-10 relative L2, and the clock to 1e-12.  With
the well-mixed concentration solved in every Newton pass: its pattern bit for
bit, its first system as the film's, c after N steps within 1e-10 relative L2
and its change over the steps within 1e-6.
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
    st = make(d)
    rowptr, col, bc = st.pattern()
    assert np.array_equal(rowptr, d["rowptr"]) and np.array_equal(col, d["col"]) and np.array_equal(bc, d["bc"])
    #  the concentration equation's pattern (ConcField = WM only)
    crow, ccol = st.conc_pattern()
    assert np.array_equal(crow, d.get("rowptr_c", np.zeros(0, np.int32)))
    assert np.array_equal(ccol, d.get("col_c", np.zeros(0, np.int32)))


@pytest.mark.parametrize("f", STEPS, ids=IDS)
def test_first_newton_system(f):
    d = stateio.load_npz(f)
    if "sys_values" not in d:
        pytest.skip("the first Newton pass solves the concentration first (test_first_conc_system)")
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
def test_first_conc_system(f):
    """The concentration system of the first Newton pass (ConcEquationBase.h:
    302-369) entry by entry within 1e-12 of its row's largest entry, the
    right-hand side within 1e-10 of its largest entry."""
    d = stateio.load_npz(f)
    if "csys_values" not in d:
        pytest.skip("no concentration equation in this case")
    st = make(d)
    val, rhs = st.conc_system(d["field_h0"], d["field_c0"], d["dt"])
    ref_val, ref_rhs = d["csys_values"], d["csys_rhs"]
    rp = d["rowptr_c"]
    rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
    rowmax = np.zeros(rp.size - 1)
    np.maximum.at(rowmax, rows, np.abs(ref_val))
    err = np.abs(val - ref_val) / rowmax[rows]
    assert err.max() <= 1e-12, err.max()
    scale = np.abs(ref_rhs).max()
    assert np.abs(rhs - ref_rhs).max() <= 1e-10 * scale + 1e-300, (np.abs(rhs - ref_rhs).max(), scale)


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
    if not d["conc_field"]:
        assert np.array_equal(c, d["field_c1"])
        return
    #  the concentration: within 1e-10 relative L2, and its change over the
    #  steps (small next to c itself) within 1e-6 of the reference's change
    cref = d["field_c1"]
    assert np.linalg.norm(c - cref) / np.linalg.norm(cref) <= 1e-10
    dref = cref - d["field_c0"]
    assert np.linalg.norm((c - d["field_c0"]) - dref) <= 1e-6 * np.linalg.norm(dref), \
        (np.linalg.norm((c - d["field_c0"]) - dref), np.linalg.norm(dref))


@pytest.mark.parametrize("f", STEPS, ids=IDS)
def test_fields_after_steps_fp32_cycle(f):
    """The step with its solves' V-cycles in float (PREC_FP32_CYCLE): the
    FP64 BiCGStab meets the same tolerances, so h after N steps stays within
    1e-8 relative L2 of the reference's FP64 run (the error bar the FP32 arm
    is held to) and the clock is the same."""
    d = stateio.load_npz(f)
    st = make(d)
    st.set_precision(1)
    stats = st.advance(d["steps_done"])
    h, c = st.fields()
    ref = d["field_h1"]
    rel = np.linalg.norm(h - ref) / np.linalg.norm(ref)
    assert rel <= 1e-8, rel
    assert abs(stats["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"]), (stats["time"], d["t_end"])
    if d["conc_field"]:
        cref = d["field_c1"]
        assert np.linalg.norm(c - cref) / np.linalg.norm(cref) <= 1e-8


@pytest.mark.parametrize("f", STEPS, ids=IDS)
def test_fields_after_steps_fp32_cycle_amg_reuse(f):
    """The fast form of the step: V-cycles in float and each AMG set-up
    serving several solves.  The FP64 Newton iteration and BiCGStab meet the
    same tolerances, so h stays within 1e-8 relative L2 of the reference's
    FP64 run."""
    d = stateio.load_npz(f)
    st = make(d)
    st.set_precision(1)
    st.set_amg_reuse(8)
    stats = st.advance(d["steps_done"])
    h, c = st.fields()
    ref = d["field_h1"]
    rel = np.linalg.norm(h - ref) / np.linalg.norm(ref)
    assert rel <= 1e-8, rel
    assert abs(stats["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"]), (stats["time"], d["t_end"])
    if d["conc_field"]:
        cref = d["field_c1"]
        assert np.linalg.norm(c - cref) / np.linalg.norm(cref) <= 1e-8


@pytest.mark.parametrize("f", STEPS, ids=IDS)
def test_energy_budget(f):
    """The free energy F and the flux power D (the reference's EnergyEval)
    of the film the case starts from and of the film after N steps.  On the
    start film, which both sides hold to the bit, they differ by the order
    of the sums and pow's last place: 1e-13 relative (measured: at most
    5.5e-15).  On the end film they also carry the films' own difference,
    which is far below the 1e-10 the fields are held to: 1e-12 relative
    (measured: at most 1.4e-14)."""
    d = stateio.load_npz(f)
    st = make(d)
    F0, D0 = st.energy()
    st.advance(d["steps_done"])
    F1, D1 = st.energy()
    for name, mine, ref, rel in (("F0", F0, d["energy_F0"], 1e-13), ("D0", D0, d["energy_D0"], 1e-13),
                                 ("F1", F1, d["energy_F1"], 1e-12), ("D1", D1, d["energy_D1"], 1e-12)):
        scale = max(abs(ref), abs(d["energy_D0"] if name[0] == "D" else d["energy_F0"]) * 1e-3, 1e-300)
        assert abs(mine - ref) <= rel * scale, (name, mine, ref, abs(mine - ref) / scale)


@pytest.mark.parametrize("f", STEPS, ids=IDS)
def test_fields_after_steps_fp32_matrix_amg_reuse(f):
    """The FP32 form of the step: the BiCGStab's SpMVs on the matrix rounded
    to float and the V-cycles in float, each AMG set-up serving several
    solves; vectors, dot products and recurrences FP64, and the Newton
    residual assembled in FP64, which corrects the ~6e-8 change of the
    linear system.  h stays within 1e-8 relative L2 of the reference's FP64
    run (the metric's equal-error bar), and the clock is the same."""
    d = stateio.load_npz(f)
    st = make(d)
    st.set_precision(2)
    st.set_amg_reuse(8)
    stats = st.advance(d["steps_done"])
    h, c = st.fields()
    ref = d["field_h1"]
    rel = np.linalg.norm(h - ref) / np.linalg.norm(ref)
    assert rel <= 1e-8, rel
    assert abs(stats["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"]), (stats["time"], d["t_end"])
    if d["conc_field"]:
        cref = d["field_c1"]
        assert np.linalg.norm(c - cref) / np.linalg.norm(cref) <= 1e-8


@pytest.mark.parametrize("f", STEPS, ids=IDS)
def test_energy_history(f):
    """The energy history (Output.Energy) over the fixture's steps against
    the reference's own: the budget of the film the run ends on, the energy
    dissipated over the run (the trapezoid of the flux power over every
    step's dt) to 1e-12 relative, and the balance of the last step, a
    difference of energies over dt that is near 0 when the scheme is
    consistent, to 1e-9 of the flux power."""
    d = stateio.load_npz(f)
    st = make(d)
    st.set_energy(True)
    s = st.advance(d["steps_done"])
    scale_d = max(abs(d["energy_D0"]), abs(d["energy_D1"]), 1e-300)
    assert abs(s["energy_F"] - d["energy_F1"]) <= 1e-12 * abs(d["energy_F1"]), (s["energy_F"], d["energy_F1"])
    assert abs(s["energy_D"] - d["energy_D1"]) <= 1e-12 * scale_d, (s["energy_D"], d["energy_D1"])
    assert abs(s["energy_dissipated"] - d["energy_dissipated"]) <= 1e-12 * abs(d["energy_dissipated"]) + 1e-300, \
        (s["energy_dissipated"], d["energy_dissipated"])
    assert abs(s["energy_balance"] - d["energy_balance"]) <= 1e-9 * scale_d, (s["energy_balance"], d["energy_balance"])


def test_precision_switch_mid_run():
    """The arithmetic of the solves switched between steps, with hierarchy
    reuse on: the hierarchy set up in FP64 is not reused by the FP32 cycle
    (a change of precision sets up afresh), and the run still ends within
    the 1e-8 bar of the reference's."""
    f = [p for p in STEPS if p.stem == "step_allphys_64"][0]
    d = stateio.load_npz(f)
    st = make(d)
    st.set_amg_reuse(8)
    n = int(d["steps_done"])
    assert n >= 3
    first = st.advance(1)
    assert first["amg_setups"] >= 1
    st.set_precision(1)
    # the first step after the switch sets up afresh, a later one reuses
    assert st.advance(1)["amg_setups"] >= 1
    if n > 3:
        later = st.advance(n - 3)
        assert later["amg_setups"] < later["newton_iterations"], later
    st.set_precision(0)
    stats = st.advance(1)
    assert stats["amg_setups"] >= 1
    h, _ = st.fields()
    ref = d["field_h1"]
    assert np.linalg.norm(h - ref) / np.linalg.norm(ref) <= 1e-8
    assert abs(stats["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"])
