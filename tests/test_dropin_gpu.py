"""The drop-in: the reference's own driver and model (oracle/_ref/yz_probe_b200,
built by `make -C oracle b200`) with the B200 linear solve behind its
ILinearSolverBackend seam (yuzen_b200/host/yz_backend_adapter.cpp), against
the same driver with the CPU oracle backend (oracle/_ref/yz_probe).

The GPU solve is specified to the bit by the oracle, so the two runs of the
reference's whole time loop -- its assembly, Newton iteration, concentration
equation, boundary rows and dt control, with every height and concentration
solve on the device -- end on the same film and concentration, bit for bit."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import stateio

pytestmark = pytest.mark.gpu
REPO = Path(__file__).resolve().parents[1]
PROBE = REPO / "oracle" / "_ref" / "yz_probe"
PROBE_B200 = REPO / "oracle" / "_ref" / "yz_probe_b200"
CASES = sorted((REPO / "tests" / "golden" / "cases").glob("dropin_*.toml"))


def run(exe: Path, case: Path, work: Path, env_extra: dict) -> dict:
    work.mkdir(parents=True, exist_ok=True)
    (work / case.name).write_text(case.read_text())
    env = dict(os.environ, OMP_NUM_THREADS="4", **env_extra)
    r = subprocess.run([str(exe), case.name, "out.bin"], cwd=work, env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return stateio.read_state(work / "out.bin")


@pytest.mark.parametrize("case", CASES, ids=[c.stem for c in CASES])
def test_reference_run_identical_with_b200_backend(case, tmp_path):
    if not (PROBE.exists() and PROBE_B200.exists()):
        pytest.skip("reference-built probes not present (make -C oracle ref b200)")
    cpu = run(PROBE, case, tmp_path / "cpu", {})
    gpu = run(PROBE_B200, case, tmp_path / "gpu", {"YZ_BACKEND": "b200"})
    assert gpu["steps_done"] == cpu["steps_done"] and gpu["t_end"] == cpu["t_end"]
    assert np.array_equal(gpu["field_h1"], cpu["field_h1"])
    assert np.array_equal(gpu["field_c1"], cpu["field_c1"])
