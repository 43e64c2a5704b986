"""The batched ensemble: many independent instances of the implicit step
(each a yuzen_b200.step.Step with its own CUDA stream and device buffers)
advanced together on one GPU, and partitioned over the GPUs of a node.

On one GPU the instances run concurrently: a pool of host threads advances
them, each call into the library releasing the interpreter, so that the
kernels of different instances overlap on the device.  The instances share
nothing, so every instance's film is the one it would have alone.  Over
several GPUs (one process per GPU) the instances are partitioned by their
cost with no data-path exchange; per-instance results (steps, time,
iteration counts) are gathered to rank 0 when asked.
"""
from __future__ import annotations

import concurrent.futures
import os

import numpy as np

from . import PREC_FP64
from . import step as ys


def instance_cost(case) -> float:
    """The cost estimate the partition balances: the instance's cells (the
    step's work grows with the rows; the iteration counts of these films do
    not depend much on the size)."""
    return float(case.Nx * case.Ny)


def partition(costs, world: int) -> list:
    """Longest-processing-time partition of the instances over world ranks:
    instances by falling cost (ties by index), each to the rank with the
    least cost so far (ties to the lower rank).  Deterministic, so every rank
    computes the same partition on its own."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += float(costs[k])
    return [sorted(p) for p in parts]


class Ensemble:
    """Ensemble(cases, device, precision, amg_reuse, workers, graph_loop,
    tuning): one Step per case, each with the launch shapes tuning (from
    yuzen_b200.autotune.tune) gives its size; advance(n) advances every
    instance n steps concurrently."""

    def __init__(self, cases, device: int = 0, precision: int = PREC_FP64, amg_reuse: int = 0,
                 workers: int | None = None, graph_loop: bool | None = None, tuning: dict | None = None):
        self.cases = list(cases)
        self.steps = []
        #  the loop graphs pay when a hierarchy serves several solves (a
        #  graph kept for them); with a new set-up every solve each solve
        #  would capture anew, from many threads at once
        if graph_loop is None:
            graph_loop = amg_reuse > 0
        for c in self.cases:
            st0 = c.state()
            st = ys.Step(ys.params_from_state(st0), st0["field_h0"], st0["field_c0"], st0["field_s0"], device=device)
            st.set_precision(precision)
            st.set_amg_reuse(amg_reuse)
            #  each context captures its loop graph from its own thread in
            #  thread-local mode; graph_loop False launches from the stream
            st.set_graph_loop(bool(graph_loop))
            #  the launch shapes the autotuner chose for the instance's size
            t = (tuning or {}).get((c.Nx, c.Ny))
            if t is not None:
                st.set_tuning(t["fuse_from"], t["coarse_lanes"], t.get("fine_sweeps", 0))
            self.steps.append(st)
        self.workers = workers or min(len(self.steps), max(1, 2 * (os.cpu_count() or 1)))
        self._pool = concurrent.futures.ThreadPoolExecutor(max_workers=self.workers) if self.steps else None

    def __len__(self) -> int:
        return len(self.steps)

    def advance(self, nsteps: int = 1) -> list:
        """Advance every instance nsteps steps; the per-instance stats."""
        if not self.steps:
            return []
        futs = [self._pool.submit(st.advance, nsteps) for st in self.steps]
        return [f.result() for f in futs]

    def fields(self, k: int):
        return self.steps[k].fields()

    def close(self) -> None:
        if self._pool is not None:
            self._pool.shutdown(wait=True)
            self._pool = None
        for st in self.steps:
            st.close()
        self.steps = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gather_results(local: dict, world: int, dist=None) -> dict:
    """Per-instance results of every rank on every rank ({instance: value});
    a plain copy without torch.distributed."""
    if dist is None or world == 1:
        return dict(local)
    out = [None] * world
    dist.all_gather_object(out, local)
    merged = {}
    for part in out:
        merged.update(part)
    return merged


def checksum(h: np.ndarray) -> float:
    """A position-weighted sum of a film, for comparing runs cheaply."""
    w = np.arange(1, h.size + 1, dtype=np.float64)
    return float(np.dot(h.ravel(), w) / w.sum())
