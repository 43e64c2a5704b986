"""The step's film solves with the learned preconditioner (yz_step_set_learned)
on the all-physics film of the step fixtures: the first SA-AMG solves collect
the network's (residual, V-cycle) pairs, the solve after them trains it on
the device, and the later solves try the network's flexible BiCGStab first.
The film and the concentration after the reference's steps are held to the
same 1e-8 of the reference's FP64 run as the other faster forms, the clock
to 1e-12; the stats show the collection, the training and the network's
solves (or its fall-backs to SA-AMG)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import stateio
from yuzen_b200 import learned as yl
from yuzen_b200 import step as ys

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("precision,reuse", [(0, 0), (2, 64)], ids=["fp64", "fp32m_reuse"])
def test_learned_step_meets_the_bar(precision, reuse):
    d = stateio.load_npz(GOLDEN / "step_allphys_64.npz")
    st = ys.Step(ys.params_from_state(d), d["field_h0"], d["field_c0"], d["field_s0"])
    st.set_precision(precision)
    st.set_amg_reuse(reuse)
    st.set_learned(yl.default_config(collect_solves=4, samples_per_solve=8, capacity=32, train_iters=150,
                                     batch=4, holdout=2, cap_factor=2.0))
    s = st.advance(int(d["steps_done"]))
    h, c = st.fields()
    assert np.linalg.norm(h - d["field_h1"]) / np.linalg.norm(d["field_h1"]) <= 1e-8
    assert np.linalg.norm(c - d["field_c1"]) / np.linalg.norm(d["field_c1"]) <= 1e-8
    assert abs(s["time"] - d["t_end"]) <= 1e-12 * abs(d["t_end"])
    assert s["learned_samples"] >= 8
    assert s["learned_train_ms"] > 0 and s["learned_loss"] >= 0
    assert s["learned_solves"] + s["learned_fallbacks"] >= 1


def test_learned_off_again():
    d = stateio.load_npz(GOLDEN / "step_allphys_64.npz")
    st = ys.Step(ys.params_from_state(d), d["field_h0"], d["field_c0"], d["field_s0"])
    st.set_learned(yl.default_config(collect_solves=2, capacity=8, train_iters=10, holdout=1))
    st.advance(1)
    st.set_learned(None)
    s = st.advance(int(d["steps_done"]) - 1)
    assert s["learned_solves"] == 0 and s["learned_fallbacks"] == 0 and s["learned_samples"] == 0
    h, _ = st.fields()
    assert np.linalg.norm(h - d["field_h1"]) / np.linalg.norm(d["field_h1"]) <= 1e-8
