"""The compact fixtures at the workloads' sizes (224^2 spinodal, 512^2
all-physics) against the seeded builder, on the CPU: the builder's start
state -- every header value and the fields h, c, s -- is the one the
reference's whole-step probe started from (values equal, field hashes
equal), and the host-built CRS pattern of the step is the reference's
(hash of rowptr, col and the boundary flags)."""
from __future__ import annotations

import numpy as np
import pytest

import _big
from yuzen_b200 import step as ys

#  header values the builder does not restate (run results, the reference's
#  own bookkeeping), as in test_cases.py
SKIP = {"steps_done", "diverged", "run_seconds", "t_end", "jacobi_interval", "max_steps", "on_source", "Pe",
        "ev_e0", "Mr", "energy_F0", "energy_D0", "energy_F1", "energy_D1", "energy_dissipated", "energy_balance"}
CONC_KEYS = {"conv_conc", "conc_conv", "conc_diff", "lin_c_precond", "lin_c_scaling", "lin_c_maxit", "lin_c_eps",
             "lin_c_conc", "theta_c"}
DTC_KEYS = {"dt_change_factor", "dt_criterion", "dt_scale_floor", "dt_keep_steps"}


@pytest.mark.parametrize("f", _big.BIG, ids=[f.stem for f in _big.BIG])
def test_big_start_state_is_the_references(f):
    d, state = _big.load(f)
    for k, v in state.items():
        if isinstance(v, np.ndarray) or k in SKIP or k not in d:
            continue
        if (k in CONC_KEYS and not state["conc_field"]) or (k in DTC_KEYS and not state["dt_control"]):
            continue
        assert v == d[k], (k, v, d[k])
    for k in ("field_h0", "field_c0", "field_s0"):
        assert _big.field_hash(state[k]) == d["sha_" + k], k


@pytest.mark.parametrize("f", _big.BIG, ids=[f.stem for f in _big.BIG])
def test_big_pattern_is_the_references(f):
    d, state = _big.load(f)
    rowptr, col, bc = ys.pattern_2d(ys.params_from_state(state))
    assert _big.field_hash(rowptr) == d["sha_rowptr"]
    assert _big.field_hash(col) == d["sha_col"]
    assert _big.field_hash(bc) == d["sha_bc"]


REF = sorted(_big.GOLDEN.glob("ref_*.npz"))


@pytest.mark.parametrize("f", REF, ids=[f.stem for f in REF])
def test_reference_case_restated(f):
    """The builder's restatement of one of the reference's own benchmark cases
    (cases/scaling/bench2d_n0512.toml: the film and substrate of its shape
    library) against the start state the reference's set-up builds from that
    TOML: every header value equal (the step count and the unused step-control
    factor aside), h and c equal to the bit, the substrate s to rounding."""
    d, state = _big.load(f)
    for k, v in state.items():
        if isinstance(v, np.ndarray) or k in SKIP or k not in d or k in DTC_KEYS:
            continue
        assert v == d[k], (k, v, d[k])
    assert _big.field_hash(state["field_h0"]) == d["sha_field_h0"]
    assert _big.field_hash(state["field_c0"]) == d["sha_field_c0"]
    assert np.abs(state["field_s0"] - d["field_s0"]).max() <= 1e-15
