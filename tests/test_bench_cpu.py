"""bench.py's reference arm on CPU: the reference's own CPU solver (oracle/_ref,
built by oracle/Makefile) on a short run of a workload, printing the one JSON
line the measurement contract asks for."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
pytestmark = pytest.mark.skipif(not (REPO / "oracle" / "_ref" / "yuzen_oracle").exists(),
                                reason="the reference's driver is not built")


@pytest.mark.parametrize("config", ["spinodal_224"])
def test_reference_arm_line(config):
    r = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--config", config,
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=900, cwd=REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["config"]["workload"] == config
