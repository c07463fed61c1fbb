"""The canonical numbering of the union-find pipelines, restated on the CPU (labeling_b200/csrc:
the tile kernels count each segment's component roots, the scan takes their exclusive prefix over
segments in launch order, the write kernels label a root 1 + its segment's prefix + its rank
among the roots of its segment).  A segment is one image row inside one tile, numbered
row * tiles_x + tile column (2D) or voxel row * tiles_d2 + tile index along d2 (3D).  Given the
oracle's first pixel of every component, this numbering must give the oracle's canonical labels:
components ordered by their first pixel in raster order."""
import numpy as np
import pytest

from labeling_b200 import workloads as W
from oracle import oracle as O


def first_pixels(lab):
    flat = lab.ravel()
    k = int(flat.max())
    firsts = np.full(k + 1, -1, np.int64)
    idx = np.flatnonzero(flat)
    vals = flat[idx]
    order = np.argsort(vals, kind="stable")      # stable: first occurrence of each label first
    v_sorted, i_sorted = vals[order], idx[order]
    starts = np.flatnonzero(np.r_[True, v_sorted[1:] != v_sorted[:-1]])
    firsts[v_sorted[starts]] = i_sorted[starts]
    return firsts[1:]


def labels_by_segments(first, seg_of, n_segs):
    """1 + exclusive prefix of the per-segment root counts + rank within the segment."""
    segs = np.array([seg_of(int(p)) for p in first], np.int64)
    counts = np.bincount(segs, minlength=n_segs)
    prefix = np.concatenate([[0], np.cumsum(counts)[:-1]])
    order = np.lexsort((first, segs))            # within a segment: by position
    rank = np.empty(len(first), np.int64)
    seen = {}
    for i in order:
        s = int(segs[i])
        rank[i] = seen.get(s, 0)
        seen[s] = rank[i] + 1
    return 1 + prefix[segs] + rank


@pytest.mark.parametrize("seed", range(30))
def test_2d_segment_numbering_is_canonical(seed):
    rng = np.random.default_rng(seed)
    h, w = int(rng.integers(1, 300)), int(rng.integers(1, 700))
    img = W.bernoulli((h, w), float(rng.uniform(0.05, 0.7)), seed)
    lab, k = O.ccl2d(img)
    if k == 0:
        return
    TH, TW = 64, 256                              # the default tile
    tiles_x = (w + TW - 1) // TW
    first = first_pixels(lab)
    got = labels_by_segments(first, lambda p: (p // w) * tiles_x + (p % w) // TW, h * tiles_x)
    assert np.array_equal(got, lab.ravel()[first])
    assert np.array_equal(got, np.arange(1, k + 1))


@pytest.mark.parametrize("seed", range(20))
def test_3d_segment_numbering_is_canonical(seed):
    rng = np.random.default_rng(seed + 100)
    d0, d1, d2 = (int(x) for x in rng.integers(1, 40, size=3))
    d2 = int(rng.integers(1, 150))
    vol = W.bernoulli((d0, d1, d2), float(rng.uniform(0.05, 0.4)), seed)
    lab, k = O.ccl3d(vol)
    if k == 0:
        return
    TZ = 64                                       # tile extent along d2
    t2 = (d2 + TZ - 1) // TZ
    first = first_pixels(lab)
    got = labels_by_segments(first, lambda p: (p // d2) * t2 + (p % d2) // TZ, d0 * d1 * t2)
    assert np.array_equal(got, np.arange(1, k + 1))
