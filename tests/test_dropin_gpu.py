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


STEP_B200 = REPO / "oracle" / "_ref" / "yuzen_b200_step"


def read_seam2(path: Path) -> dict:
    """The record yuzen_b200_step writes: magic, nx, ny, steps, Newton passes,
    the clock, the wall time, linear iterations, then h and c (IL order)."""
    raw = path.read_bytes()
    assert raw[:8] == b"YZSEAM21"
    nx, ny, steps, newton = np.frombuffer(raw, "<i4", 4, 8)
    t_end, wall, linear = np.frombuffer(raw, "<f8", 3, 24)
    m = int(nx) * int(ny)
    h = np.frombuffer(raw, "<f8", m, 48).copy()
    c = np.frombuffer(raw, "<f8", m, 48 + 8 * m).copy()
    return {"steps": int(steps), "newton": int(newton), "t_end": float(t_end), "h": h, "c": c}


@pytest.mark.parametrize("case", CASES, ids=[c.stem for c in CASES])
def test_reference_driver_with_the_step_on_the_device(case, tmp_path):
    """Seam 2: the reference's own set-up of a TOML case (C_Yuzen) with its
    time loop replaced by the device step (yuzen_b200/host/yz_step_adapter.cpp,
    the parameters, film and concentration read out of the reference's
    objects and the result written back into them) against the reference's
    whole run of the same case: the same steps, the clock to 1e-12, h and c
    within 1e-10 relative L2."""
    if not (PROBE.exists() and STEP_B200.exists()):
        pytest.skip("reference-built binaries not present (make -C oracle ref b200)")
    cpu = run(PROBE, case, tmp_path / "cpu", {})
    work = tmp_path / "seam2"
    work.mkdir()
    (work / case.name).write_text(case.read_text())
    r = subprocess.run([str(STEP_B200), case.name, "out.bin"], cwd=work, capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, OMP_NUM_THREADS="4"))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    gpu = read_seam2(work / "out.bin")
    assert gpu["steps"] == cpu["steps_done"]
    assert abs(gpu["t_end"] - cpu["t_end"]) <= 1e-12 * abs(cpu["t_end"])
    assert np.linalg.norm(gpu["h"] - cpu["field_h1"]) / np.linalg.norm(cpu["field_h1"]) <= 1e-10
    assert np.linalg.norm(gpu["c"] - cpu["field_c1"]) / np.linalg.norm(cpu["field_c1"]) <= 1e-10


PROBE_CZ = REPO / "oracle" / "_ref" / "yz_probe_cz"
CZ_B200 = REPO / "oracle" / "_ref" / "yuzen_b200_cz"
CZ_CASES = sorted((REPO / "tests" / "golden" / "cases").glob("czdropin_*.toml"))


def read_seam3(path: Path) -> dict:
    """The record yuzen_b200_cz writes: magic, nx, ny, nz, steps, linear
    iterations, coupling passes, the clock, dt, the wall time, then h
    (nx*ny) and c (nx*ny*nz)."""
    raw = path.read_bytes()
    assert raw[:8] == b"YZSEAM31"
    nx, ny, nz, steps, linear, coupling = (int(v) for v in np.frombuffer(raw, "<i4", 6, 8))
    t_end, dt, wall = np.frombuffer(raw, "<f8", 3, 32)
    m2, m3 = nx * ny, nx * ny * nz
    h = np.frombuffer(raw, "<f8", m2, 56).copy()
    c = np.frombuffer(raw, "<f8", m3, 56 + 8 * m2).copy()
    return {"steps": steps, "linear": linear, "coupling": coupling, "t_end": float(t_end), "dt": float(dt),
            "h": h, "c": c}


@pytest.mark.parametrize("case", CZ_CASES, ids=[c.stem for c in CZ_CASES])
def test_reference_driver_with_the_cz_step_on_the_device(case, tmp_path):
    """Seam 3: the reference's own set-up of a ConcZ case (C_Yuzen) with its
    time loop replaced by the device step (yuzen_b200/host/yz_cz_adapter.cpp)
    against the reference's whole run of the same case (yz_probe_cz): the
    same steps, linear iterations and coupling passes, the clock to 1e-12,
    h and c within 1e-10 relative L2."""
    if not (PROBE_CZ.exists() and CZ_B200.exists()):
        pytest.skip("reference-built binaries not present (make -C oracle ref b200)")
    work = tmp_path / "ref"
    work.mkdir()
    (work / case.name).write_text(case.read_text())
    r = subprocess.run([str(PROBE_CZ), case.name, "out.bin"], cwd=work, capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, OMP_NUM_THREADS="4"))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    ref = stateio.read_records(work / "out.bin")
    work = tmp_path / "seam3"
    work.mkdir()
    (work / case.name).write_text(case.read_text())
    r = subprocess.run([str(CZ_B200), case.name, "out.bin"], cwd=work, capture_output=True, text=True, timeout=900,
                       env=dict(os.environ, OMP_NUM_THREADS="4"))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    gpu = read_seam3(work / "out.bin")
    assert gpu["steps"] == ref["steps_done"]
    assert gpu["linear"] == ref["linear_iterations"] and gpu["coupling"] == ref["coupling_passes"]
    assert abs(gpu["t_end"] - ref["t_end"]) <= 1e-12 * abs(ref["t_end"])
    eh = np.linalg.norm(gpu["h"] - ref["h1"]) / np.linalg.norm(ref["h1"])
    ec = np.linalg.norm(gpu["c"] - ref["c1"]) / np.linalg.norm(ref["c1"])
    assert eh <= 1e-10 and ec <= 1e-10, (eh, ec)
