"""Multi-GPU replica logic, exercised as two ``gloo`` ranks on the CPU.

The replicas share no data path: each rank serves its share of the request
stream (computed identically on every rank) and the bench reduces only its
timings (max over ranks) and gathers summaries.  These tests run those steps
with world_size 2 over 127.0.0.1.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from gridfoam_b200.serving import poisson_stream  # noqa: E402
from gridfoam_b200.serving.shard import merge_summaries, shard_stream  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = poisson_stream(50, rate=50.0, seed=0)
        mine = shard_stream(reqs, world, rank)
        ids = [None] * world
        dist.all_gather_object(ids, [r.id for r in mine])
        # timing reduction used by the bench: max over ranks
        t = torch.tensor([10.0 + rank])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        lat = [None] * world
        dist.all_gather_object(lat, [0.1 * (rank + 1)] * len(mine))
        if rank == 0:
            out.put((ids, float(t.item()), lat))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_stream_sharding_and_reductions():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ids, tmax, lat = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    all_ids = sorted(ids[0] + ids[1])
    assert all_ids == list(range(50)) and not set(ids[0]) & set(ids[1])
    reqs = poisson_stream(50, rate=50.0, seed=0)
    work = [sum(r.cells for r in reqs if r.id in set(part)) for part in ids]
    assert max(work) <= 1.5 * min(work)
    assert tmax == 11.0
    s = merge_summaries(lat, [0.0, 0.0], [1.0, 2.0])
    assert s["completed"] == 50 and s["solves_per_s"] == pytest.approx(25.0)


def test_shard_is_a_partition_for_any_world():
    reqs = poisson_stream(40, rate=50.0, seed=3)
    for world in (1, 3, 8):
        parts = [shard_stream(reqs, world, r) for r in range(world)]
        got = sorted(x.id for p in parts for x in p)
        assert got == list(range(40))
    with pytest.raises(ValueError):
        shard_stream(reqs, 2, 2)
    assert np.isclose(merge_summaries([[1.0, 3.0]], [0.0], [2.0])["p50_latency_s"], 2.0)
