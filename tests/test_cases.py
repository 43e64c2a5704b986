"""The seeded case builders (yuzen_b200/cases.py: the spinodal film, the
all-physics film, an instance of the batched ensemble) against the
reference's own set-up: the case is written in the reference's format, the whole-step probe
(the reference's C_Yuzen driver, oracle/probe/yz_probe.cpp) builds it, and
the non-dimensional state it hands the step -- every header value and the
fields h, c, s -- must equal the builder's to the bit.  Needs the probe
binary built by oracle/Makefile; skipped where it is absent."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import stateio
from yuzen_b200 import cases

PROBE = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "yz_probe"
pytestmark = pytest.mark.skipif(not PROBE.exists(), reason="the whole-step probe is not built")

#  header values the builder does not restate (run results, the reference's
#  own bookkeeping)
SKIP = {"steps_done", "diverged", "run_seconds", "t_end", "jacobi_interval", "max_steps", "on_source", "Pe",
        "ev_e0", "Mr"}


def _probe(case: cases.Case, work: Path) -> dict:
    case.steps = 1
    case.write_reference(work)
    env = dict(os.environ, OMP_NUM_THREADS="2")
    res = subprocess.run([str(PROBE), "case.toml", "out.bin"], cwd=work, env=env, capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    return stateio.read_state(work / "out.bin")


@pytest.mark.parametrize("make", [lambda: cases.spinodal_224(N=24, steps=1),
                                  lambda: cases.allphys(N=24, steps=1),
                                  lambda: cases.dewetting(24, theta_e=13.7, amp=3e-3, seed=5, steps=1)],
                         ids=["spinodal_24", "allphys_24", "dewetting_24"])
def test_state_bitwise(make, tmp_path):
    case = make()
    ref = _probe(case, tmp_path)
    mine = case.state()
    #  without ConcField = WM the concentration equation is not built: its
    #  scheme and solver settings are whatever its constructor left
    conc_keys = {"conv_conc", "conc_conv", "conc_diff", "lin_c_precond", "lin_c_scaling", "lin_c_maxit", "lin_c_eps",
                 "lin_c_conc", "theta_c"}
    #  likewise the step-control settings without Numerics.TimeStepControl
    dtc_keys = {"dt_change_factor", "dt_criterion", "dt_scale_floor", "dt_keep_steps"}
    for k, v in mine.items():
        if k in SKIP or k not in ref or (k in conc_keys and not mine["conc_field"]) or \
                (k in dtc_keys and not mine["dt_control"]):
            continue
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, ref[k]), k
        else:
            assert v == ref[k], (k, v, ref[k])
