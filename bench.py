#!/usr/bin/env python
"""bench.py -- time steps per second of the implicit step of the well-mixed
film-height equation on B200, next to the reference's CPU solver.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME]
    python bench.py --impl reference ...      # the reference's CPU solver

A step is one time step of the case (C_NewtonKantorovich::TimeAdvance and
the clock, NewtonKantorovich.cpp:424-486): assembly, Newton passes, one
BiCGStab + SA-AMG(SPAI0) solve of the film and one of the well-mixed
concentration per pass, all on the device.  The default workload is the
512 x 512 all-physics film (yuzen_b200.cases.allphys: capillary, disjoining,
vertical and in-plane gravity, rotation, Marangoni, evaporation, slip, the
concentration solved); the case is a seeded synthetic input built by
yuzen_b200.cases (the reference reads the same film through its ASCII
restart).  Four arms run from the same start: the plain FP64 path (the
drop-in), the FP32 V-cycle (the AMG preconditioner in float inside the FP64
BiCGStab), the FP32 V-cycle with each AMG set-up serving several solves
and the BiCGStab loop replayed as a cached CUDA graph, and that with the
BiCGStab's SpMVs on the float copy of the matrix.  Every arm's first steps
are checked against the reference's own run of the same case (the fixture
tests/golden/big_<workload>.npz: h and c after its steps); the headline is
the fastest arm whose film there is within 1e-8 (relative L2) of the
reference's.  Timing: per arm W untimed steps (the checked ones among them),
then K steps, each timed with CUDA events on the library's stream, the L2
cache (126 MB) flushed by writing a 256 MiB buffer between steps (outside the
timed region).  The same K steps are also timed end to end on the host clock
around the public calls (the film uploaded from pinned host memory, the step,
the film read back).  Under torchrun every rank runs an independent replica
and the time is the maximum over ranks.  One JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "steps/s at 512² all-physics: learned-precond FP32 vs plain FP64 GPU, equal h-error"
UNIT = "steps/s"

#  The kernel whose roofline is reported (the finest level's SpMV of the
#  BiCGStab iteration) and its algorithmic bytes per launch:
#  v = A p with alpha = rho / (rh . v): matrix values and columns (12 B per
#  entry), row pointers (4 B per row), p read once, rh read, v written
#  (8 B each per row).
ROOFLINE_KERNEL = "KSpmvAlpha"

#  DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
#  the reported kernels, from one ncu capture of each on its workload (a
#  single-kernel capture, cold L2, --clock-control none), by kernel and
#  workload: what roofline.traffic reports.  A kernel or workload without a
#  capture reports null.
NCU_TRAFFIC = {
    ("KSpmvAlpha", "allphys_512"): 33880064,
    # a Newton pass's assembly: KAssemble (180,615,424 B) + KUpwindFaces
    # (50,359,808 B); the pass's two smaller kernels (KFaceProps, KCellPi) were
    # not captured
    ("assembly", "allphys_512"): 180615424 + 50359808,
    # the ConcZ concentration assembly (one capture of its fourth launch on cz_256)
    ("KCzAssembleC", "cz_256"): 41707776 + 136976896,
}


PATHS = {
    "fp64": "plain FP64 (the drop-in path)",
    "fp32_cycle": "FP32 V-cycle inside the FP64 BiCGStab (AMG set-up, Krylov vectors, SpMVs and tests FP64)",
    "fp32_reuse": "FP32 V-cycle inside the FP64 BiCGStab, each AMG set-up serving several solves, the "
                  "BiCGStab loop replayed as a cached CUDA graph",
    "fp32m_reuse": "FP32 V-cycle and FP32 matrix values in the BiCGStab's SpMVs (vectors, dot products and "
                   "recurrences FP64; the Newton residual FP64), each AMG set-up serving several solves, the "
                   "BiCGStab loop replayed as a cached CUDA graph",
    "learned": "the learned preconditioner: a U-Net (BF16 tcgen05 convolutions, FP32 accumulation) trained on the "
               "device during the warm-up steps on the (residual, V-cycle) pairs of the first film solves, tried "
               "first in a flexible BiCGStab on every film solve, SA-AMG (the fp32m_reuse form) as its fallback "
               "and yardstick",
}
DTYPES = {"fp64": "f64", "fp32_cycle": "f64 (V-cycle f32)", "fp32_reuse": "f64 (V-cycle f32)",
          "fp32m_reuse": "f64 Newton / f32 matrix and V-cycle in an f64 Krylov",
          "learned": "f64 Newton / bf16 network (f32 accumulation), f32 matrix and V-cycle fallback in an f64 Krylov"}
#  arm -> (arithmetic of the solve, AMG hierarchy reuse on, learned preconditioner on)
ARMS = {"fp64": (0, False, False), "fp32_cycle": (1, False, False), "fp32_reuse": (1, True, False),
        "fp32m_reuse": (2, True, False), "learned": (2, True, True)}


def learned_config():
    """The learned arm's settings: the first six film solves (two steps)
    collect up to eight pairs each, the solve after them trains the network
    (200 Adam steps of four pairs, four held out), and every later film solve
    tries it first within three times the last SA-AMG solve's iterations."""
    from yuzen_b200 import learned
    return learned.default_config(collect_solves=6, samples_per_solve=8, capacity=48, train_iters=200, batch=4,
                                  holdout=4, cap_factor=3.0, seed=1, activation=0)


def cz_learned_config():
    """The ConcZ learned arm's settings: the first four film solves (the
    predictor and corrector of two steps) collect up to eight pairs each, the
    film solve after them (the third step's predictor, inside the steps
    checked against the reference) trains the network (200 Adam steps of four
    pairs, four held out), and every later film solve tries it first within
    three times the last SA-AMG solve's iterations."""
    from yuzen_b200 import learned
    return learned.default_config(collect_solves=4, samples_per_solve=8, capacity=32, train_iters=200, batch=4,
                                  holdout=4, cap_factor=3.0, seed=1, activation=0)


def spmv_alpha_bytes(n: int, nnz: int) -> int:
    return 12 * nnz + 4 * (n + 1) + 3 * 8 * n


def assembly_bytes(n: int, nnz: int) -> int:
    """Algorithmic bytes of one Newton pass's assembly (A, J, I + theta dt J
    and the right-hand side in one pass): read h, c, s, h^n and A(h^n) h^n
    (8 B each per row), write the I + theta dt J values and the A values kept
    for the explicit half (8 B per entry each) and the right-hand side."""
    return 5 * 8 * n + 2 * 8 * nnz + 8 * n


def oracle_fixture(workload: str):
    """The reference's own run of the workload's first steps (h and c after
    them), the fixture the parity tests hold the device to, or None."""
    p = REPO / "tests" / "golden" / f"big_{workload}.npz"
    if not p.exists():
        return None
    import numpy as np
    z = np.load(p)
    return {"steps": int(z["steps_done"]), "h": z["field_h1"], "c": z["field_c1"] if "field_c1" in z.files else None,
            "t_end": float(z["t_end"])}


def measured_peaks() -> dict:
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.TemporaryFile(mode="w+")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        self.out.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.out.read())) if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(k)
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": float(rows[0][2]),
                "samples": len(rows), "reasons": sorted(reasons)}


def make_case(name: str, steps: int):
    from yuzen_b200 import cases
    return cases.CONFIGS[name](steps=steps)


# ----------------------------------------------------------------------
#  the reference's CPU solver (the reference's sources compiled by
#  oracle/Makefile with the CPU restatement of its AMGCL backend)
# ----------------------------------------------------------------------
def reference_run(name: str, steps: int, threads: int, case=None) -> dict:
    exe = REPO / "oracle" / "_ref" / "yuzen_oracle"
    if not exe.exists():
        return {"unavailable": f"{exe.relative_to(REPO)} is not built (make -C oracle ref)"}
    cfg = case if case is not None else make_case(name, steps)
    with tempfile.TemporaryDirectory() as tmp:
        cfg.write_reference(tmp)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), YUZEN_THREAD_CAP="0", OMP_PROC_BIND="close")
        r = subprocess.run([str(exe), "case.toml"], cwd=tmp, env=env, capture_output=True, text=True, timeout=3600)
        info = Path(tmp) / cfg.name / "JobInfo.txt"
        if r.returncode != 0 or not info.exists():
            return {"unavailable": f"reference run failed (exit {r.returncode})"}
        text = info.read_text()
    loop = float(re.search(r"Time loop \[s\]\s*:\s*([0-9.eE+-]+)", text).group(1))
    nsteps = int(re.search(r"Time steps\s*:\s*([0-9]+)", text).group(1))
    newton = int(re.search(r"Newton iterations\s*:\s*([0-9]+)", text).group(1))
    linear = int(re.search(r"Linear iterations\s*:\s*([0-9]+)", text).group(1))
    return {"value": nsteps / loop, "loop_s": loop, "steps": nsteps, "newton": newton, "linear": linear,
            "threads": threads}


def ensemble_reference(a, threads: int) -> dict:
    """The reference's CPU solver on a bounded sample of the ensemble: the
    first a.ref_instances instances (one size each where the batch has it),
    a.steps steps each, one after the other with all host threads."""
    from yuzen_b200 import cases
    batch = cases.batch(256, steps=a.steps)
    seen, sample = set(), []
    for c in batch:
        if c.Nx not in seen:
            seen.add(c.Nx)
            sample.append(c)
    sample = sample[:a.ref_instances]
    loop, steps = 0.0, 0
    for c in sample:
        r = reference_run("", a.steps, threads, case=c)
        if "unavailable" in r:
            return r
        loop += r["loop_s"]
        steps += r["steps"]
    cells = sum(c.Nx * c.Ny for c in sample)
    #  instance-steps/s of the sample, scaled to the batch's mean instance
    mean_cells = sum(c.Nx * c.Ny for c in batch) / len(batch)
    return {"value": steps / loop * (cells / len(sample)) / mean_cells, "loop_s": loop, "steps": steps,
            "sample": f"{len(sample)} instances ({', '.join(str(c.Nx) for c in sample)} cells a side), "
                      f"{a.steps} steps each, scaled by cells to the batch's mean instance"}


def run_reference_arm(a) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if a.config == "cz_256":
        r = cz_reference_run(a.steps, threads)
        if "unavailable" in r:
            print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}))
            return
        print(json.dumps({
            "impl": "reference", "metric": CZ_METRIC, "value": r["value"], "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 / r["value"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": a.config, "linear_iterations": r["linear"]},
            "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": r["sample"]},
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    if a.config == "batch_256":
        r = ensemble_reference(a, threads)
        if "unavailable" in r:
            print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}))
            return
        print(json.dumps({
            "impl": "reference", "metric": ENSEMBLE_METRIC, "value": r["value"], "unit": ENSEMBLE_UNIT,
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "config": {"workload": a.config},
            "cpu_baseline": {"value": r["value"], "unit": ENSEMBLE_UNIT, "cores": threads, "kind": "reference",
                             "sample": r["sample"]},
            "e2e": {"value": r["value"], "unit": ENSEMBLE_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    r = reference_run(a.config, a.steps, threads)
    if "unavailable" in r:
        print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}))
        return
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 / r["value"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": a.config, "newton_iterations": r["newton"], "linear_iterations": r["linear"]},
        "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{r['steps']} steps of {a.config} (the reference's sources with the CPU "
                                   f"restatement of its AMGCL backend, {threads} OpenMP threads)"},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ----------------------------------------------------------------------
#  the device arm
# ----------------------------------------------------------------------
def run_device_arm(a) -> None:
    import numpy as np
    import torch

    import yuzen_b200 as yz
    from yuzen_b200 import step as ys

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)

    cfg = make_case(a.config, a.steps)
    state = cfg.state()
    params = ys.params_from_state(state)
    n = params.nx * params.ny
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    fx = oracle_fixture(a.config)
    hpin = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    cpin = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()

    def rel(x, y) -> float:
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))

    def timed_arm(name: str) -> dict:
        """On a fresh step of the case: the fixture's steps (checked against
        the reference's run), the rest of the W untimed steps, then K steps
        each timed on the device (CUDA events inside the step) and, around the
        same calls, end to end on the host clock: the film uploaded from
        pinned host memory, the step, the film read back"""
        precision, reuse, learn = ARMS[name]
        st = ys.Step(params, state["field_h0"], state["field_c0"], state["field_s0"], device=local)
        st.set_precision(precision)
        st.set_amg_reuse(a.amg_reuse if reuse else 0)
        if learn:
            st.set_learned(learned_config())
        out = {"total_ms": 0.0, "wall_s": 0.0, "newton": 0, "linear": 0, "launches": 0, "conc_solves": 0,
               "conc_iters": 0, "per_step": [], "per_setup": [], "warmup": 0,
               "parts": {"setup_ms": 0.0, "solve_ms": 0.0, "assemble_ms": 0.0},
               "learned": {"solves": 0, "fallbacks": 0, "iterations": 0, "train_ms": 0.0, "val_err": None,
                           "samples": 0, "warmup_solves": 0, "warmup_fallbacks": 0}}
        done = 0
        def note_learned(r, timed):
            L = out["learned"]
            if timed:
                L["solves"] += r["learned_solves"]
                L["fallbacks"] += r["learned_fallbacks"]
                L["iterations"] += r["learned_iterations"]
            else:
                L["warmup_solves"] += r["learned_solves"]
                L["warmup_fallbacks"] += r["learned_fallbacks"]
            L["train_ms"] += r["learned_train_ms"]
            L["val_err"] = r["learned_val_err"]
            L["samples"] = r["learned_samples"]
        if fx is not None:
            r = st.advance(fx["steps"])
            note_learned(r, False)
            done = fx["steps"]
            h, c = st.fields()
            out["h_err_vs_oracle"] = rel(h, fx["h"])
            out["c_err_vs_oracle"] = rel(c, fx["c"]) if fx["c"] is not None else None
            out["t_err_vs_oracle"] = abs(r["time"] - fx["t_end"]) / abs(fx["t_end"])
        if a.warmup > done:
            note_learned(st.advance(a.warmup - done), False)
            done = a.warmup
        out["warmup"] = done
        st.fields_into(hpin, cpin)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(a.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st.set_fields(hpin, cpin)
            r = st.advance(1)
            st.fields_into(hpin, cpin)
            out["wall_s"] += time.perf_counter() - t0
            out["total_ms"] += r["device_ms"]
            out["per_step"].append(round(r["device_ms"], 2))
            out["per_setup"].append(round(r["setup_ms"], 2))
            out["newton"] += r["newton_iterations"]
            out["linear"] += r["linear_iterations"]
            out["launches"] += r["launches"]
            out["conc_solves"] += r["conc_solves"]
            out["conc_iters"] += r["conc_iterations"]
            note_learned(r, True)
            for k in out["parts"]:
                out["parts"][k] += r[k]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t = torch.tensor([out["total_ms"], out["wall_s"]], dtype=torch.float64, device=f"cuda:{local}")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out["max_ms"] = float(t[0].item())
        out["max_wall_s"] = float(t[1].item())
        out["value"] = world * a.steps / (out["max_ms"] / 1e3)
        out["e2e"] = world * a.steps / max(out["max_wall_s"], 1e-9)
        out["finite"] = bool(np.isfinite(hpin).all())
        out["step"] = st
        return out

    names = [x for x in a.arms.split(",") if x]
    for x in names:
        if x not in ARMS:
            raise SystemExit(f"unknown arm {x}: {', '.join(ARMS)}")
    arms = {}
    with Clocks(local) as clk:
        for x in names:
            arms[x] = timed_arm(x)
    #  the headline: the fastest arm within 1e-8 of the reference's run (of
    #  its h, and c where the case solves it); without a fixture, of the FP64
    #  arm's h after the timed steps
    def qualifies(x) -> bool:
        v = arms[x]
        if fx is not None:
            return v["h_err_vs_oracle"] <= 1e-8 and (v["c_err_vs_oracle"] is None or v["c_err_vs_oracle"] <= 1e-8)
        return x == "fp64"
    qualified = [x for x in names if qualifies(x)]
    head_name = max(qualified or names[:1], key=lambda x: arms[x]["value"])
    head = arms[head_name]
    max_ms, value = head["max_ms"], head["value"]

    #  the roofline kernel (the finest level's FP64 SpMV + dot, the same
    #  kernel in every arm), every launch bracketed by CUDA events on the
    #  library's stream, over further steps of the first arm: timing single
    #  launches needs the iterations launched from the stream, so this runs
    #  apart from the arms' timed steps (where the loop may run as a graph)
    rstep = arms[names[0]]["step"]
    yz.time_kernel(ROOFLINE_KERNEL)
    for _ in range(a.roofline_steps):
        flush.zero_()
        torch.cuda.synchronize()
        rstep.advance(1)
    torch.cuda.synchronize()
    kern_ms, kern_n = yz.kernel_time()
    yz.time_kernel(None)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    nnz = int(ys.pattern_2d(params)[1].size)
    peaks = measured_peaks()
    roof = None
    if kern_n > 0:
        bytes_ = spmv_alpha_bytes(n, nnz)
        achieved = bytes_ / (kern_ms / kern_n / 1e3) / 1e9
        roof = {"kernel": ROOFLINE_KERNEL, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                "peak_source": peaks["source"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                "traffic": NCU_TRAFFIC.get((ROOFLINE_KERNEL, a.config)), "bytes_per_launch": bytes_,
                "launches": kern_n,
                "timed_over": f"{a.roofline_steps} further steps of the {names[0]} arm, L2 flushed between steps",
                "avg_launch_us": kern_ms / kern_n * 1e3}
    #  the assembly of a Newton pass (every term's A and J, I + theta dt J and
    #  the right-hand side), timed with CUDA events around it in every pass
    #  of the headline arm's timed steps
    asm = None
    if head["newton"] > 0 and head["parts"]["assemble_ms"] > 0:
        ab = assembly_bytes(n, nnz)
        per_pass_ms = head["parts"]["assemble_ms"] / head["newton"]
        ach = ab / (per_pass_ms / 1e3) / 1e9
        asm = {"kernel": "assembly of a Newton pass", "bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"],
               "peak_source": peaks["source"], "unit": "GB/s", "frac": ach / peaks["hbm_gbs"],
               "traffic": NCU_TRAFFIC.get(("assembly", a.config)), "bytes_per_launch": ab, "passes": head["newton"],
               "avg_pass_us": per_pass_ms * 1e3}
    cpu = None
    if world == 1 and not a.no_cpu_baseline:
        threads = os.cpu_count() or 1
        r = reference_run(a.config, a.cpu_steps, threads)
        if "unavailable" not in r:
            cpu = {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"{r['steps']} steps of {a.config}: the reference's sources with the CPU "
                             f"restatement of its AMGCL backend (linear solve and assembly on {threads} "
                             f"OpenMP threads)"}
        else:
            cpu = {"unavailable": r["unavailable"]}
    cfg_line = {"workload": a.config, "grid": [cfg.Nx, cfg.Ny], "rows": n, "nnz": nnz,
                "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                "l2": "flushed between steps (256 MiB write)",
                "path": PATHS[head_name], "arm": head_name,
                "amg_reuse": a.amg_reuse if ARMS[head_name][1] else 0,
                "learned_preconditioner": head_name == "learned",
                "warmup_steps": head["warmup"]}
    if fx is not None:
        cfg_line.update({
            "oracle_steps": fx["steps"],
            "h_err_vs_oracle": head["h_err_vs_oracle"], "c_err_vs_oracle": head["c_err_vs_oracle"],
            "h_err_vs_oracle_fp64": arms["fp64"]["h_err_vs_oracle"] if "fp64" in arms else None,
            "c_err_vs_oracle_fp64": arms["fp64"]["c_err_vs_oracle"] if "fp64" in arms else None})
    if "fp64" in arms:
        cfg_line["fp64_steps_per_s"] = arms["fp64"]["value"]
        cfg_line["speedup_vs_fp64"] = value / arms["fp64"]["value"]
    cfg_line["arms"] = {k: {"steps_per_s": v["value"], "e2e_steps_per_s": v["e2e"],
                            "ms_per_step": v["max_ms"] / a.steps,
                            "h_err_vs_oracle": v.get("h_err_vs_oracle"), "c_err_vs_oracle": v.get("c_err_vs_oracle"),
                            "newton_iterations": v["newton"], "linear_iterations": v["linear"],
                            "conc_solves": v["conc_solves"], "conc_iterations": v["conc_iters"],
                            "device_ms": {q: round(w, 3) for q, w in v["parts"].items()},
                            "step_ms": v["per_step"], "setup_ms_per_step": v["per_setup"],
                            "gpu_launches": v["launches"],
                            **({"learned": v["learned"]} if ARMS[k][2] else {})} for k, v in arms.items()}
    if "learned" in arms:
        L = arms["learned"]
        cfg_line["learned_steps_per_s"] = L["value"]
        cfg_line["learned_vs_fp64"] = L["value"] / arms["fp64"]["value"] if "fp64" in arms else None
        cfg_line["learned_h_err_vs_oracle"] = L.get("h_err_vs_oracle")
        cfg_line["learned_solves"] = L["learned"]["solves"]
        cfg_line["learned_fallbacks"] = L["learned"]["fallbacks"]
        cfg_line["learned_val_err"] = L["learned"]["val_err"]
        cfg_line["learned_train_ms"] = L["learned"]["train_ms"]
    cfg_line["finite"] = all(v["finite"] for v in arms.values())
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": max_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPES[head_name],
        "data": "synthetic (seeded, yuzen_b200.cases)",
        "config": cfg_line,
        "e2e": {"value": head["e2e"], "unit": UNIT, "h2d_bytes_per_step": 2 * 8 * n, "d2h_bytes_per_step": 2 * 8 * n,
                "steps": a.steps, "timed": "the same K steps as value, host clock around set_fields + advance + "
                                          "fields_into, L2 flushed between steps"},
        "gpu_launches": head["launches"],
        "roofline": roof,
        "roofline_assembly": asm,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


ENSEMBLE_METRIC = "instance-steps/s of the 256-instance dewetting and levelling ensemble (64²-256²)"
ENSEMBLE_UNIT = "instance-steps/s"


def run_ensemble_arm(a) -> None:
    """The batched ensemble (yuzen_b200.ensemble): 256 seeded dewetting and
    levelling instances, the FP32 arms' coarse launch shapes tuned per size
    (yuzen_b200.autotune, before the timed steps), partitioned over the ranks by cost, each rank advancing its
    instances concurrently on its GPU; a step is one step of every instance.
    Timed with CUDA events between device-wide synchronisations (the
    instances run on streams of their own), the maximum over ranks."""
    import numpy as np
    import torch

    import yuzen_b200 as yz
    from yuzen_b200 import cases, ensemble
    from yuzen_b200 import step as ys

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    batch = cases.batch(256, steps=a.steps)
    parts = ensemble.partition([ensemble.instance_cost(c) for c in batch], world)
    mine = parts[rank]
    arms = {}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    tunings = {}
    for name in [x for x in a.arms.split(",") if x]:
        prec, reuse, learn = ARMS[name]
        if learn:
            continue        # the ensemble has no learned arm
        #  the coarse levels' launch shapes per instance size, measured on one
        #  instance of each size (untimed; the FP64 cycle has none)
        tuning = {}
        if not a.no_autotune:
            from yuzen_b200 import autotune
            tuning = autotune.tune([batch[k] for k in mine], prec, amg_reuse=a.amg_reuse if reuse else 0,
                                   device=local)
            tunings[name] = autotune.summary(tuning)
        ens = ensemble.Ensemble([batch[k] for k in mine], device=local, precision=prec,
                                amg_reuse=a.amg_reuse if reuse else 0, workers=a.workers,
                                graph_loop=None if a.ensemble_graph < 0 else bool(a.ensemble_graph), tuning=tuning)
        if a.warmup > 0:
            ens.advance(a.warmup)
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        total_ms, launches = 0.0, 0
        for _ in range(a.steps):
            flush.zero_()
            torch.cuda.synchronize()
            l0 = ys.launch_count()
            e0.record()
            ens.advance(1)
            torch.cuda.synchronize()
            e1.record()
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            launches += ys.launch_count() - l0
        t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{local}")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        max_ms = float(t.item())
        h = {mine[j]: ensemble.checksum(ens.fields(j)[0]) for j in range(len(mine))}
        arms[name] = {"value": len(batch) * a.steps / (max_ms / 1e3), "max_ms": max_ms, "launches": launches,
                      "checksums": ensemble.gather_results(h, world, dist), "ens": ens}
    names = list(arms)
    head_name = names[-1]
    head = arms[head_name]
    #  end to end through the step's public calls with host buffers: every
    #  instance's film uploaded from pinned memory, one step, read back
    ens = head["ens"]
    pins = []
    for j in range(len(ens)):
        nn = ens.steps[j].n
        hp = torch.empty(nn, dtype=torch.float64, pin_memory=True).numpy()
        cp = torch.empty(nn, dtype=torch.float64, pin_memory=True).numpy()
        ens.steps[j].fields_into(hp, cp)
        pins.append((hp, cp))

    def e2e_one(j):
        st = ens.steps[j]
        st.set_fields(*pins[j])
        st.advance(1)
        st.fields_into(*pins[j])

    e2e_steps = max(0, min(a.steps, a.e2e_steps))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        list(ens._pool.map(e2e_one, range(len(ens))))
    e2e_s = max(time.perf_counter() - t0, 1e-9)
    et = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
    if dist:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    bytes_step = sum(2 * 8 * ens.steps[j].n for j in range(len(ens)))
    diff = None
    if "fp64" in arms and head_name != "fp64":
        a64, ah = arms["fp64"]["checksums"], head["checksums"]
        diff = max(abs(ah[k] - a64[k]) / max(abs(a64[k]), 1e-300) for k in a64)
    if rank == 0:
        line = {
            "metric": ENSEMBLE_METRIC, "value": head["value"], "unit": ENSEMBLE_UNIT, "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": head["max_ms"] / a.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": DTYPES[head_name], "data": "synthetic (seeded, cases.batch)",
            "config": {"workload": a.config, "instances": len(batch), "instances_rank0": len(mine),
                       "sizes": sorted({c.Nx for c in batch}), "path": PATHS[head_name],
                       "parallelism": f"instances partitioned over {world} GPUs" if world > 1 else "1 GPU",
                       "l2": "flushed between steps (256 MiB write)", "workers": ens.workers,
                       "graph_loop": "with hierarchy reuse" if a.ensemble_graph < 0 else bool(a.ensemble_graph),
                       "arms": {k: {"instance_steps_per_s": v["value"], "ms_per_step": v["max_ms"] / a.steps,
                                    "gpu_launches": v["launches"]} for k, v in arms.items()},
                       "checksum_rel_diff_vs_fp64": diff,
                       "autotune": tunings.get(head_name) if tunings else "off",
                       "kinds": {"dewetting": sum(1 for c in batch if c.name.startswith("dewetting")),
                                 "levelling": sum(1 for c in batch if c.name.startswith("levelling"))}},
            "e2e": {"value": len(batch) * e2e_steps / float(et.item()) if e2e_steps else None, "unit": ENSEMBLE_UNIT,
                    "h2d_bytes_per_step": bytes_step, "d2h_bytes_per_step": bytes_step, "steps": e2e_steps},
            "gpu_launches": head["launches"],
            "roofline": None,
            "cpu_baseline": None,
        }
        print(json.dumps(line))
    for v in arms.values():
        v["ens"].close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------------------------
#  the ConcZ workload (config 5): the film and its concentration through
#  the thickness at 256^2 x 16 levels (yuzen_b200.cases.cz_bumps)
# ----------------------------------------------------------------------
CZ_METRIC = "steps/s of the ConcZ evaporating film, 256² x 16 levels (semi-implicit film + zeta-grid concentration)"
CZ_ROOFLINE_KERNEL = "KCzAssembleC"


def cz_assembly_bytes(nr: int) -> int:
    """Algorithmic bytes of one concentration assembly (KCzAssembleC) over nr
    real cells: read c, the three volume fluxes (8 B each per cell), write the
    row's 21 values, B and the free-surface term (8 B each)."""
    return nr * (4 * 8 + 23 * 8)


def cz_reference_run(steps: int, threads: int) -> dict:
    #  the reference exactly as it builds (the libm's exp), for its timing
    exe = REPO / "oracle" / "_ref" / "yz_probe_cz_libm"
    if not exe.exists():
        return {"unavailable": f"{exe.relative_to(REPO)} is not built (make -C oracle ref)"}
    from yuzen_b200 import cases
    case = cases.cz_bumps(steps=steps)
    with tempfile.TemporaryDirectory() as tmp:
        case.write_reference(tmp)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), YUZEN_THREAD_CAP="0", OMP_PROC_BIND="close")
        r = subprocess.run([str(exe), "case.toml", "out.bin", "init=init.bin"], cwd=tmp, env=env, capture_output=True,
                           text=True, timeout=3600)
        if r.returncode != 0:
            return {"unavailable": "the reference's CZ run failed: " + (r.stdout + r.stderr)[-300:].replace("\n", " ")}
        sys.path.insert(0, str(REPO / "tests" / "golden"))
        import stateio
        d = stateio.read_records(Path(tmp) / "out.bin")
    return {"value": d["steps_done"] / d["wall"], "steps": d["steps_done"], "linear": d["linear_iterations"],
            "sample": f"{d['steps_done']} steps of cz_256 (the reference's CZ model from its sources, the CPU "
                      f"restatement of its AMGCL backend, {threads} OpenMP threads)"}


def run_cz_arm(a) -> None:
    import numpy as np
    import torch

    import yuzen_b200 as yz
    from yuzen_b200 import cases, cz

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)
    rec = cases.cz_bumps(steps=a.steps).record()
    params = cz.params_from_record(rec)
    n2, n3 = params.nx * params.ny, params.nx * params.ny * params.nz
    nr = (params.nx - 4) * (params.ny - 4) * (params.nz - 4)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    fxp = REPO / "tests" / "golden" / "czbig_256.npz"
    fx = dict(np.load(fxp)) if fxp.exists() else None
    hpin = torch.empty(n2, dtype=torch.float64, pin_memory=True).numpy()
    cpin = torch.empty(n3, dtype=torch.float64, pin_memory=True).numpy()
    #  arm -> (arithmetic of the solves, AMG hierarchy reuse); the learned
    #  arm is fp32_reuse with the network tried first on the film's solves
    arms_cz = {"fp64": (0, 0), "fp32_reuse": (1, 64), "fp32m_reuse": (2, 64), "learned": (1, 64)}
    names = [x for x in a.arms.split(",") if x in arms_cz] or ["fp64", "fp32_reuse"]

    def rel(x, y) -> float:
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))

    def timed_arm(name: str) -> dict:
        prec, reuse = arms_cz[name]
        m = cz.CzModel(params, rec["xc"], rec["xf"], rec["yc"], rec["yf"], rec["h0"], rec["s"], rec["c0"],
                       device=local)
        m.set_precision(prec)
        m.set_amg_reuse(reuse)
        if name == "learned":
            m.set_learned(cz_learned_config())
        out = {"total_ms": 0.0, "wall_s": 0.0, "linear": 0, "conc_iters": 0, "coupling": 0, "launches": 0,
               "per_step": []}
        L = {"solves": 0, "fallbacks": 0, "iterations": 0, "train_ms": 0.0, "warmup_solves": 0,
             "warmup_fallbacks": 0}

        def note_learned(r, timed):
            if name != "learned":
                return
            pre = "" if timed else "warmup_"
            L[pre + "solves"] += r["learned_solves"]
            L[pre + "fallbacks"] += r["learned_fallbacks"]
            if timed:
                L["iterations"] += r["learned_iterations"]
            L["train_ms"] += r["learned_train_ms"]
            L["val_err"], L["samples"] = r["learned_val_err"], r["learned_samples"]
        done = 0
        if fx is not None:
            r = m.advance(int(fx["steps_done"]))
            note_learned(r, False)
            done = int(fx["steps_done"])
            h, c = m.fields()
            nx, ny, nz = params.nx, params.ny, params.nz
            out["h_err_vs_oracle"] = rel(h, fx["h1"])
            out["c_colsum_err_vs_oracle"] = rel(c.reshape(nz, ny, nx)[2:-2].sum(axis=0).ravel(), fx["c1_colsum"])
            out["t_err_vs_oracle"] = abs(r["time"] - float(fx["t_end"])) / float(fx["t_end"])
        if a.warmup > done:
            note_learned(m.advance(a.warmup - done), False)
            done = a.warmup
        out["warmup"] = done
        m.fields_into(hpin, cpin)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for _ in range(a.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            m.set_fields(hpin, cpin)
            r = m.advance(1)
            m.fields_into(hpin, cpin)
            out["wall_s"] += time.perf_counter() - t0
            out["total_ms"] += r["device_ms"]
            out["per_step"].append(round(r["device_ms"], 2))
            out["linear"] += r["linear_iterations"]
            out["conc_iters"] += r["conc_iterations"]
            out["coupling"] += r["coupling_passes"]
            out["launches"] += r["launches"]
            note_learned(r, True)
        if name == "learned":
            out["learned"] = L
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t = torch.tensor([out["total_ms"], out["wall_s"]], dtype=torch.float64, device=f"cuda:{local}")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out["max_ms"], out["max_wall_s"] = float(t[0].item()), float(t[1].item())
        out["value"] = world * a.steps / (out["max_ms"] / 1e3)
        out["e2e"] = world * a.steps / max(out["max_wall_s"], 1e-9)
        out["finite"] = bool(np.isfinite(hpin).all() and np.isfinite(cpin).all())
        out["model"] = m
        return out

    arms, failed = {}, {}
    with Clocks(local) as clk:
        for x in names:
            try:
                arms[x] = timed_arm(x)
            except yz.StepFailedError as e:
                #  an arm whose solve does not converge at the fixed step
                #  (the FP32 matrix on the concentration's stiff zeta
                #  diffusion) is reported, not timed
                failed[x] = str(e)[:200]
    names = [x for x in names if x in arms]

    def qualifies(x) -> bool:
        v = arms[x]
        if fx is None:
            return x == "fp64"
        return v["h_err_vs_oracle"] <= 1e-8 and v["c_colsum_err_vs_oracle"] <= 1e-8
    qualified = [x for x in names if qualifies(x)]
    head_name = max(qualified or names[:1], key=lambda x: arms[x]["value"])
    head = arms[head_name]
    #  the concentration's assembly, every launch timed with CUDA events on the
    #  model's stream, over further steps of the first arm
    m0 = arms[names[0]]["model"]
    yz.time_kernel(CZ_ROOFLINE_KERNEL)
    for _ in range(max(1, a.roofline_steps)):
        flush.zero_()
        torch.cuda.synchronize()
        m0.advance(1)
    torch.cuda.synchronize()
    kern_ms, kern_n = yz.kernel_time()
    yz.time_kernel(None)
    peaks = measured_peaks()
    roof = None
    if kern_n:
        per = kern_ms / kern_n
        ach = cz_assembly_bytes(nr) / (per * 1e-3) / 1e9
        roof = {"kernel": CZ_ROOFLINE_KERNEL, "bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": ach / peaks["hbm_gbs"],
                "traffic": NCU_TRAFFIC.get((CZ_ROOFLINE_KERNEL, "cz_256")), "launches_timed": kern_n,
                "avg_launch_us": per * 1e3, "algorithmic_bytes_per_launch": cz_assembly_bytes(nr),
                "peak_source": peaks["source"]}
    cpu = None
    if rank == 0 and not a.no_cpu_baseline:
        r = cz_reference_run(a.cpu_steps, os.cpu_count() or 1)
        if "unavailable" not in r:
            cpu = {"value": r["value"], "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "reference",
                   "sample": r["sample"]}
    if rank == 0:
        line = {
            "metric": CZ_METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": head["max_ms"] / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"fp64": "f64", "learned": "f64 (V-cycle f32, bf16 network with f32 "
                                                               "accumulation)"}.get(head_name, "f64 (V-cycle f32)"),
            "data": "synthetic (seeded: yuzen_b200.cases.cz_bumps)",
            "config": {"workload": "cz_256", "grid": [256, 256, 16], "arm": head_name, "l2": "flushed (256 MiB)",
                       "arms": {x: {k: v for k, v in arms[x].items() if k != "model"} | {"steps_per_s": arms[x]["value"]}
                                for x in names}, "arms_failed": failed},
            "e2e": {"value": head["e2e"], "unit": UNIT, "h2d_bytes_per_step": 8 * (n2 + n3),
                    "d2h_bytes_per_step": 8 * (n2 + n3)},
            "gpu_launches": head["launches"], "clocks": clk.summary(), "roofline": roof, "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    for v in arms.values():
        v["model"].close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="allphys_512")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=6, help="steps of the ensemble's end-to-end measurement")
    ap.add_argument("--arms", default="fp64,fp32_cycle,fp32_reuse,fp32m_reuse,learned",
                    help="the arms timed, in order (fp64, fp32_cycle, fp32_reuse, fp32m_reuse, learned); headline: "
                         "the fastest one whose film is within 1e-8 of the reference's run")
    ap.add_argument("--amg-reuse", type=int, default=64, help="solves an AMG set-up serves in the fp32_reuse arm")
    ap.add_argument("--roofline-steps", type=int, default=3, help="steps over which the roofline kernel is timed")
    ap.add_argument("--workers", type=int, default=64, help="host threads advancing the ensemble's instances")
    ap.add_argument("--no-autotune", action="store_true", help="the ensemble's default launch shapes, untuned")
    ap.add_argument("--ref-instances", type=int, default=3, help="ensemble instances the reference arm samples")
    ap.add_argument("--ensemble-graph", type=int, default=-1,
                    help="the ensemble's BiCGStab loops as CUDA graphs (1) or from the streams (0); -1: graphs "
                         "where the AMG hierarchy is reused")
    a = ap.parse_args()
    if a.warmup < 3 and a.impl == "b200":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if a.impl == "reference":
        run_reference_arm(a)
    elif a.config == "batch_256":
        run_ensemble_arm(a)
    elif a.config == "cz_256":
        run_cz_arm(a)
    else:
        run_device_arm(a)


if __name__ == "__main__":
    main()
