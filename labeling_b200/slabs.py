"""Slab split of one image: each slab labeled on its own, then one exchange step.

A 2D image is cut into bands of rows, a volume into bands of planes along d0 (its slowest
dimension).  Each slab is labeled by ``be_label2d`` / ``be_label3d`` on its own GPU (one process
per GPU, one slab per rank) or, on one GPU, one after another.  The exchange step moves only each
slab's first and last row (plane) of labels and its component count: every rank gathers them
(``all_gather`` over the process group -- NCCL for CUDA tensors, gloo on CPU), runs the same host
merge (``be_slab_merge``) and maps its own slab's labels in place (``be_slab_relabel``).  The
result equals labeling the whole image at once, canonical numbering included.

The reference labels one image on one device (Labeling2015/src/LabelingAlgs.cpp:989-1084); this
split is for images larger than one GPU's memory.  It has one collective: an all_gather of each
slab's border rows with its count packed in the same tensor.  The relabel scratch is sized before
the slabs are labeled (``slab_reserve``), so the exchange and relabel allocate nothing.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from . import Context, SlabMerge, label2d, label3d, slab_merge, slab_relabel, slab_reserve


def slab_bounds(n: int, parts: int) -> List[Tuple[int, int]]:
    """``parts`` bands of ``n`` rows (planes), sizes differing by at most one, in order."""
    if parts < 1 or parts > n:
        raise ValueError(f"cannot cut {n} rows into {parts} non-empty slabs")
    q, r = divmod(n, parts)
    out, a = [], 0
    for k in range(parts):
        b = a + q + (1 if k < r else 0)
        out.append((a, b))
        a = b
    return out


def _reserve(ctx: Context, slab_shape, n_slabs: int = 1) -> None:
    """Relabel scratch for a slab of this shape: at most one component per two pixels (plus one),
    at most every label of both border rows (planes) of every slab joined."""
    n = 1
    for d in slab_shape:
        n *= int(d)
    plane = n // int(slab_shape[0])
    slab_reserve(ctx, n // 2 + 1, 2 * plane * n_slabs)


def label_slabs(ctx: Context, img, out, parts: int, threshold: int = 0, stream=None) -> int:
    """Labels a 2D image [rows, cols] or a volume [d0, d1, d2] (CUDA tensors; ``out`` int32 of the
    same shape, contiguous rows) as ``parts`` slabs on this one GPU, one after another, and joins
    them.  Returns the component count of the whole image."""
    import torch

    bounds = slab_bounds(int(img.shape[0]), parts)
    _reserve(ctx, (bounds[0][1] - bounds[0][0],) + tuple(img.shape[1:]), parts)
    counts = []
    for a, b in bounds:
        if img.dim() == 3:
            counts.append(label3d(ctx, img[a:b], out[a:b], threshold=threshold, stream=stream))
        else:
            counts.append(label2d(ctx, img[a:b], out[a:b], threshold=threshold, stream=stream))
    # Every slab's first and last row in one device-to-host copy.
    rows = torch.stack([out[i] for a, b in bounds for i in (a, b - 1)]).cpu().numpy()
    m = slab_merge(counts, rows[0::2], rows[1::2])
    for s, (a, b) in enumerate(bounds):
        slab_relabel(ctx, out[a:b], counts[s], int(m.offsets[s]), m.joined_labels[s], m.joined_targets[s],
                     stream=stream)
    return m.total


def exchange_and_merge(top, bottom, count: int, group=None) -> Tuple[int, SlabMerge]:
    """The exchange step of rank k, which holds slab k of ``world_size`` slabs in rank order:
    gathers every slab's border rows (``top`` / ``bottom``, int32 tensors on the group's device)
    and count, and merges them on the host.  Returns (this rank's slab index, the merge)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = top.device
    # Top row, bottom row and the count (a label count fits int32: images have < 2^31 pixels)
    # travel in one tensor: one collective.
    n = top.numel()
    both = torch.cat([top.contiguous().reshape(-1), bottom.contiguous().reshape(-1),
                      torch.tensor([int(count)], dtype=torch.int32, device=dev)])
    gathered = [torch.empty_like(both) for _ in range(world)]
    dist.all_gather(gathered, both, group=group)
    g = torch.stack(gathered).cpu().numpy()
    shape = (world,) + tuple(top.shape)
    m = slab_merge(g[:, 2 * n].astype(np.int64), g[:, :n].reshape(shape), g[:, n:2 * n].reshape(shape))
    return rank, m


def label_distributed(ctx: Context, slab, out, threshold: int = 0, group=None, stream=None) -> int:
    """Rank k labels slab k (2D rows or 3D planes, on its own GPU), takes part in the exchange and
    maps its labels to the whole image's.  Every rank must call it, with slabs in rank order and
    equal border sizes.  Returns the component count of the whole image."""
    import torch.distributed as dist
    _reserve(ctx, tuple(slab.shape), dist.get_world_size(group))
    if slab.dim() == 3:
        count = label3d(ctx, slab, out, threshold=threshold, stream=stream)
    else:
        count = label2d(ctx, slab, out, threshold=threshold, stream=stream)
    k, m = exchange_and_merge(out[0], out[-1], count, group=group)
    slab_relabel(ctx, out, count, int(m.offsets[k]), m.joined_labels[k], m.joined_targets[k], stream=stream)
    return m.total
