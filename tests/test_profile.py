"""The profile table: the reference's YUZEN_PROF scopes (util/Profile.h:1-127)
on the device path.

* CPU: the entry points load; with YUZEN_PROFILE unset the table is empty
  and the switch reads 0.
* GPU: a process with YUZEN_PROFILE=1 that runs an all-physics step with the
  concentration fills the table with the reference's names (every solve
  under h.linsolve / c.linsolve, its set-up under lin.precond, its
  iterations under lin.iterate), the device seconds of a scope are no more
  than those of the scope that holds it, and at exit standard error carries
  the reference's lines "[profile] name calls seconds".  Without the switch
  the same process prints none.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

import yuzen_b200 as yz

ROOT = Path(__file__).resolve().parents[1]

_CHILD = r"""
import json, sys
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/tests", sys.argv[1] + "/tests/golden"]
import stateio
import yuzen_b200 as yz
from yuzen_b200 import step as ys
d = stateio.load_npz(sys.argv[1] + "/tests/golden/step_wm_allphys_48.npz")
s = ys.Step(ys.params_from_state(d), d["field_h0"], d["field_c0"], d["field_s0"])
r = s.advance(3)
print(json.dumps({"table": yz.profile_table(), "enabled": yz.lib().yz_profile_enabled(),
                  "newton": r["newton_iterations"], "steps": r["steps"]}))
"""


def test_profile_entry_points_on_cpu():
    if os.environ.get("YUZEN_PROFILE", "0") not in ("", "0"):
        pytest.skip("YUZEN_PROFILE is set in this process")
    L = yz.lib()
    for sym in ("yz_profile_enabled", "yz_profile_entry", "yz_profile_reset"):
        assert hasattr(L, sym)
    assert L.yz_profile_enabled() == 0
    assert yz.profile_table() == {}
    yz.profile_reset()


def _run(env_value):
    env = dict(os.environ)
    env.pop("YUZEN_PROFILE", None)
    if env_value is not None:
        env["YUZEN_PROFILE"] = env_value
    res = subprocess.run([sys.executable, "-c", _CHILD, str(ROOT)], capture_output=True, text=True, env=env,
                         timeout=600)
    assert res.returncode == 0, res.stderr[-3000:]
    import json
    out = json.loads(res.stdout.strip().splitlines()[-1])
    return out, res.stderr


@pytest.mark.gpu
def test_profile_table_on_device():
    out, err = _run("1")
    t = out["table"]
    assert out["enabled"] == 1
    for name in ("step", "h.assemble", "h.linsolve", "lin.prepare", "lin.precond", "lin.iterate", "h.couple",
                 "c.linsolve", "h.after"):
        assert name in t and t[name][0] > 0 and t[name][1] > 0.0, (name, t)
    assert t["step"][0] == out["steps"]
    # at most one film solve per Newton pass; one assembly per pass and one
    # at each attempt's start
    assert out["steps"] <= t["h.linsolve"][0] <= out["newton"]
    assert t["h.assemble"][0] >= t["h.linsolve"][0] + out["steps"]
    # inclusive times: a part is no longer than what holds it
    slack = 1e-4
    assert t["lin.iterate"][1] <= t["h.linsolve"][1] + t["c.linsolve"][1] + slack
    assert t["h.linsolve"][1] <= t["step"][1] + slack
    # the reference's exit lines
    lines = [ln for ln in err.splitlines() if ln.startswith("[profile]")]
    assert lines and lines[0].startswith("[profile] threads ")
    pat = re.compile(r"^\[profile\] (\S+)\s+(\d+)\s+([0-9.]+)$")
    names = {}
    for ln in lines[1:]:
        m = pat.match(ln)
        assert m, ln
        names[m.group(1)] = (int(m.group(2)), float(m.group(3)))
    assert set(names) == set(t)
    assert names["h.linsolve"][0] == t["h.linsolve"][0]


@pytest.mark.gpu
def test_profile_off_prints_nothing():
    out, err = _run(None)
    assert out["enabled"] == 0 and out["table"] == {}
    assert "[profile]" not in err


_CHILD_CZ = r"""
import json, sys
sys.path[:0] = [sys.argv[1], sys.argv[1] + "/tests", sys.argv[1] + "/tests/golden"]
import stateio
import yuzen_b200 as yz
from yuzen_b200 import cz
d = stateio.load_npz(sys.argv[1] + "/tests/golden/cz_sym_16.npz")
m = cz.CzModel(cz.params_from_record(d), d["xc"], d["xf"], d["yc"], d["yf"], d["h0"], d["s"], d["c0"])
r = m.advance(int(d["steps_done"]))
m.close()
print(json.dumps({"table": yz.profile_table(), "steps": r["steps"], "solves": r["solves"]}))
"""


@pytest.mark.gpu
def test_profile_table_of_the_concz_step():
    """The ConcZ step's scopes carry the reference's CZ labels (YUZEN_PROF in
    CZ_HeightEquation_2D.cpp and CZ_ConcEquation_2D.cpp): the film's
    assembly, right-hand side and solve, the velocity, the concentration's
    step and its solves."""
    env = dict(os.environ, YUZEN_PROFILE="1")
    res = subprocess.run([sys.executable, "-c", _CHILD_CZ, str(ROOT)], capture_output=True, text=True, env=env,
                         timeout=600)
    assert res.returncode == 0, res.stderr[-3000:]
    import json
    out = json.loads(res.stdout.strip().splitlines()[-1])
    t = out["table"]
    for name in ("step", "h.assemble", "h.rhs", "h.linsolve", "velocity", "c.solve", "c.linsolve", "lin.iterate"):
        assert name in t and t[name][0] > 0 and t[name][1] > 0.0, (name, t)
    assert t["step"][0] == out["steps"]
    assert t["h.linsolve"][0] + t["c.linsolve"][0] == out["solves"]
    assert t["h.linsolve"][1] <= t["step"][1] + 1e-4
