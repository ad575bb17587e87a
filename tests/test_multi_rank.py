"""Multi-GPU layout on the host, as two gloo ranks on the CPU: the batched ensemble and the served trace shard whole
scenes (requests) across ranks with no collective on the data path; the only exchange is the max / sum of the timing
and work figures that bench.py reports.  Checked here: every scene lands on exactly one rank, the ranks' cell counts
are balanced, every rank derives the same assignment without communication, and the reductions bench.py uses give the
max over ranks and the sum of their work."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "heatflow-mpm_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from heatflow_mpm.batch import ensemble, shard_scenarios
        from heatflow_mpm.serve import poisson_trace
        scs = ensemble(count=64, seed=0)
        mine = shard_scenarios(scs, rank, world)
        ids = [s.tag["index"] for s in mine]
        trace = [r.rid for r in poisson_trace(rate=20, duration=5, seed=0) if r.rid % world == rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, {"ids": ids, "cells": sum(s.n ** 3 for s in mine), "trace": trace})
        elapsed = 1.0 + rank                      # a rank-dependent "time" and "work"
        t_max = bench.reduce_max(elapsed, "cpu", world)
        w_sum = bench.reduce_sum(10.0 * (rank + 1), "cpu", world)
        if rank == 0:
            out.put({"gathered": gathered, "t_max": t_max, "w_sum": w_sum})
    finally:
        dist.destroy_process_group()


def test_scene_sharding_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    res = out.get(timeout=60)
    g = res["gathered"]
    all_ids = sorted(i for r in g for i in r["ids"])
    assert all_ids == list(range(64))                              # every scene exactly once
    cells = [r["cells"] for r in g]
    assert max(cells) <= 1.1 * min(cells)                          # largest-first greedy balances the cells
    trace = sorted(i for r in g for i in r["trace"])
    assert trace == list(range(len(trace))) and len(trace) > 50    # every request exactly once
    assert res["t_max"] == 2.0 and res["w_sum"] == 30.0            # max over ranks; sum of work


def test_shard_assignment_is_deterministic():
    from heatflow_mpm.batch import ensemble, shard_scenarios
    scs = ensemble(count=64, seed=3)
    for world in (1, 2, 4, 8):
        parts = [shard_scenarios(scs, r, world) for r in range(world)]
        assert sorted(s.tag["index"] for p in parts for s in p) == list(range(64))
        assert parts == [shard_scenarios(scs, r, world) for r in range(world)]
