"""Replica plumbing for multi-GPU runs: one process per GPU, each labeling its own images.

Block-equivalence labeling of one image does not shard (the largest configuration, a 512^3 volume
with int32 labels, fits one GPU many times over), so N GPUs run N independent replicas with no
collective on the data path.  The only cross-rank steps are the ones a measurement needs: a
barrier before and after the timed region, the slowest rank's time and the total work.  These
helpers keep that logic in one place so that it is tested on CPU ranks (gloo) as well as used by
bench.py over NCCL.
"""
from __future__ import annotations

import os
from typing import Sequence, Tuple, TypeVar

T = TypeVar("T")


def rank_info() -> Tuple[int, int, int]:
    """(rank, world size, local rank) from the torch.distributed launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base: int, rank: int) -> int:
    """Seed of a rank's synthetic inputs: every replica labels different images of one shape."""
    return base + 17 * rank


def shard(items: Sequence[T], rank: int, world: int) -> Sequence[T]:
    """The rank's share of a list of independent jobs (round robin; disjoint, covering)."""
    return items[rank::world]


def combine(elapsed_ms: float, units: float, device=None) -> Tuple[float, float]:
    """Whole-job timing over the ranks: (max elapsed ms, total units).  A no-op with one process.

    `device` is where the reduction tensors live: the rank's CUDA device for NCCL, the CPU for
    gloo.  Every rank must call this the same number of times, in the same order."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(elapsed_ms), float(units)
    t = torch.tensor([float(elapsed_ms)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())
