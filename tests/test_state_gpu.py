"""The step's state and its field files.

* yz_step_get_state / yz_step_set_state (the reference's RestartState,
  IO/RestartState.h:57): a step resumed from the state taken after k steps
  ends, after more steps, on the film, concentration, clock and Newton count
  of the step that ran straight through -- to the bit on the FP64 path.
* The field file the step writes (the reference's ASCII restart format,
  Output.cpp:902-912): the reference's own time loop restarted from it ends
  within 1e-10 of a device step started from the same film.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import stateio
from yuzen_b200 import cases
from yuzen_b200 import step as ys

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
PROBE = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "yz_probe"


@pytest.mark.parametrize("name", ["step_allphys_64", "step_adaptive_40", "step_wm_slip_adaptive_40"])
def test_state_roundtrip_bitwise(name):
    d = stateio.load_npz(GOLDEN / f"{name}.npz")
    mk = lambda: ys.Step(ys.params_from_state(d), d["field_h0"], d["field_c0"], d["field_s0"])
    a = mk()
    a.advance(1)
    saved = a.state()
    ra = a.advance(2)
    ha, ca = a.fields()
    b = mk()
    b.set_state(saved)
    rb = b.advance(2)
    hb, cb = b.fields()
    assert np.array_equal(ha, hb) and np.array_equal(ca, cb)
    assert ra["time"] == rb["time"] and ra["dt"] == rb["dt"]
    assert ra["newton_iterations"] == rb["newton_iterations"]
    assert ra["linear_iterations"] == rb["linear_iterations"]


def test_state_rejects_another_grid():
    d = stateio.load_npz(GOLDEN / "step_allphys_64.npz")
    e = stateio.load_npz(GOLDEN / "step_adaptive_40.npz")
    a = ys.Step(ys.params_from_state(d), d["field_h0"], d["field_c0"], d["field_s0"])
    b = ys.Step(ys.params_from_state(e), e["field_h0"], e["field_c0"], e["field_s0"])
    import yuzen_b200 as yz
    with pytest.raises(yz.YzError):
        b.set_state(a.state())


@pytest.mark.skipif(not PROBE.exists(), reason="the whole-step probe is not built")
def test_field_file_restarts_the_reference(tmp_path):
    case = cases.allphys(N=48, steps=2)
    state = case.state()
    params = ys.params_from_state(state)
    first = ys.Step(params, state["field_h0"], state["field_c0"], state["field_s0"])
    first.advance(2)
    h, c = first.fields()
    # the reference's time loop from the file the step writes
    case.write_reference(tmp_path)
    first.write_field(tmp_path / "init.dat", case)
    res = subprocess.run([str(PROBE), "case.toml", "out.bin"], cwd=tmp_path, capture_output=True, text=True,
                         timeout=600, env=dict(os.environ, OMP_NUM_THREADS="4"))
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    ref = stateio.read_state(tmp_path / "out.bin")
    assert np.array_equal(ref["field_h0"], h) and np.array_equal(ref["field_c0"], c)
    # a device step started from the same film
    second = ys.Step(params, h, c, state["field_s0"])
    s = second.advance(int(ref["steps_done"]))
    h2, c2 = second.fields()
    assert np.linalg.norm(h2 - ref["field_h1"]) / np.linalg.norm(ref["field_h1"]) <= 1e-10
    assert np.linalg.norm(c2 - ref["field_c1"]) / np.linalg.norm(ref["field_c1"]) <= 1e-10
    assert abs(s["time"] - ref["t_end"]) <= 1e-12 * abs(ref["t_end"])
