"""Multi-process replica plumbing on CPU ranks (gloo, world size 2): the cross-rank timing
reduction bench.py uses over NCCL, the per-rank seeds and the job sharding.  No GPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from labeling_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, lr = replicas.rank_info()
        # rank k took 10 + k ms for (k + 1) * 1000 units
        t, u = replicas.combine(10.0 + rank, 1000.0 * (rank + 1), device="cpu")
        jobs = list(range(11))
        mine = list(replicas.shard(jobs, rank, world))
        everyone = [None] * world
        dist.all_gather_object(everyone, mine)
        q.put((rank, r, w, lr, t, u, replicas.replica_seed(10, rank), everyone))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_combine_shard_and_seeds_over_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    seeds = set()
    for rank, r, w, lr, t, u, seed, everyone in out:
        assert (r, w, lr) == (rank, world, rank)
        assert t == pytest.approx(11.0)           # the slowest rank's time
        assert u == pytest.approx(3000.0)         # all ranks' units
        seeds.add(seed)
        flat = sorted(x for part in everyone for x in part)
        assert flat == list(range(11))            # shards are disjoint and cover the jobs
    assert len(seeds) == world                    # every replica labels different images


def test_combine_is_identity_without_a_process_group():
    assert not dist.is_initialized()
    assert replicas.combine(3.5, 42.0) == (3.5, 42.0)
