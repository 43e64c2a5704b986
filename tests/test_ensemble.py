"""The batched ensemble's host logic on CPU: the seeded batch, the cost
partition over ranks, and the gather of per-instance results over a
world-size-2 gloo process group (the N-GPU path of the ensemble, whose
instances share no data)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from yuzen_b200 import cases, ensemble


def test_batch_is_seeded_and_in_range():
    a, b = cases.batch(64), cases.batch(64)
    key = lambda c: (c.name, c.Nx, c.disjoining, float(c.h_init[3, 5]))
    assert [key(c) for c in a] == [key(c) for c in b]
    assert {c.Nx for c in a} <= {64, 96, 128, 192, 256}
    kinds = {"dewetting": 0, "levelling": 0}
    for c in a:
        assert c.Nx == c.Ny and c.dt_control
        if c.name.startswith("dewetting"):
            kinds["dewetting"] += 1
            assert c.bc == ("Periodic",) * 4 and 5.0 <= c.disjoining[0] <= 20.0
            amp = np.max(np.abs(c.h_init - 1.0))
            assert amp <= 1e-2 and amp > 1e-4 * 0.5
        else:
            kinds["levelling"] += 1
            assert c.name.startswith("levelling") and c.bc == ("Symmetry",) * 4
            assert c.disjoining is None and c.vgrav is not None
            amp = np.max(np.abs(c.h_init - 1.0))
            assert 1e-2 * 0.5 < amp <= 1.1e-1
    assert kinds["dewetting"] > 16 and kinds["levelling"] > 16
    assert len({c.Nx for c in cases.batch(256)}) == 5


def test_autotune_classes_and_summary():
    from yuzen_b200 import PREC_FP64, autotune
    batch = cases.batch(32)
    cls = autotune.size_classes(batch)
    assert set(cls) == {(c.Nx, c.Ny) for c in batch}
    assert all(batch[k].Nx == s[0] for s, k in cls.items())
    assert all(min(j for j, c in enumerate(batch) if (c.Nx, c.Ny) == s) == k for s, k in cls.items())
    assert autotune.tune(batch, PREC_FP64) == {}          # nothing to tune on the FP64 cycle
    t = {(64, 64): {"fuse_from": 2, "coarse_lanes": 4, "fine_sweeps": 3, "ms_per_step": 1.0,
                    "default_ms_per_step": 1.5, "trials": {"-1,0,0": 1.5, "2,4,3": 1.0}}}
    assert autotune.summary(t) == {"64x64": {"fuse_from": 2, "coarse_lanes": 4, "fine_sweeps": 3, "ms_per_step": 1.0,
                                             "default_ms_per_step": 1.5}}
    assert all(len(c) == 3 for c in autotune.CANDIDATES) and autotune.CANDIDATES[0] == (-1, 0, 0)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_covers_balances_and_is_deterministic(world):
    costs = [ensemble.instance_cost(c) for c in cases.batch(256)]
    parts = ensemble.partition(costs, world)
    assert parts == ensemble.partition(costs, world)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[k] for k in p) for p in parts]
    #  LPT: no rank carries more than the lightest one plus one instance
    assert max(loads) - min(loads) <= max(costs)


def test_partition_edge_cases():
    assert ensemble.partition([], 2) == [[], []]
    assert ensemble.partition([5.0], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        ensemble.partition([1.0], 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        batch = cases.batch(16, sizes=(16, 24, 32))
        parts = ensemble.partition([ensemble.instance_cost(c) for c in batch], world)
        #  the rank's instances: a per-instance result computed locally (the
        #  initial film's checksum stands in for a run's result on CPU)
        local = {k: ensemble.checksum(batch[k].h_init) for k in parts[rank]}
        merged = ensemble.gather_results(local, world, dist)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"),
                np.array([merged[k] for k in range(len(batch))]))
    finally:
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    expect = np.array([ensemble.checksum(c.h_init) for c in cases.batch(16, sizes=(16, 24, 32))])
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"rank{r}.npy"), expect)
