"""Sharding independent problems across ranks (gloo, world size 2, CPU).

Each rank derives the same partition from the problems' work estimates,
solves nothing (no GPU here) and reports its share; the shares are gathered
and must cover every problem exactly once with balanced work, and the
max-over-ranks reduction used for timing must see both ranks.
"""

from __future__ import annotations

import os

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from torchls_b200 import synthetic
from torchls_b200.batched import partition_problems


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        datas = synthetic.batched_bundle_adjustment(64, first_seed=0)
        work = [d.num_observations for d in datas]
        mine = partition_problems(work, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = torch.tensor([float(sum(work[j] for j in mine))])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            out.put((gathered, float(t), work))
    finally:
        dist.destroy_process_group()


def test_partition_covers_all_problems_with_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, max_load, work = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    flat = sorted(j for part in gathered for j in part)
    assert flat == list(range(64))
    total = sum(work)
    assert max_load <= total / 2 + max(work)  # LPT bound
    assert max_load == max(sum(work[j] for j in part) for part in gathered)


def test_partition_is_deterministic_and_balanced():
    work = [5, 1, 9, 3, 3, 7, 2, 8]
    a = partition_problems(work, 3)
    assert a == partition_problems(work, 3)
    loads = [sum(work[j] for j in p) for p in a]
    assert max(loads) - min(loads) <= max(work)
