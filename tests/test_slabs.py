"""Slab split of one image (one exchange of border rows).

CPU: the host merge (``be_slab_merge``) joins slabs that the oracle labeled on their own, and the
mapped labels must equal the oracle's labels of the whole image bit for bit (integer work: exact),
with the component count; the exchange runs over two and three gloo ranks.  GPU: the one-GPU slab
path (``label_slabs``) against ``be_label2d`` / ``be_label3d`` on the whole image and the oracle.
"""
import os
import socket

import numpy as np
import pytest

from oracle import oracle as O


def _lib_or_skip():
    import labeling_b200 as be
    if not os.path.exists(be.LIB_PATH):
        pytest.skip("libbe_b200.so not built")
    return be


def _bounds(n, parts):
    from labeling_b200.slabs import slab_bounds
    return slab_bounds(n, parts)


def _join_on_host(be, img, parts, label):
    """Oracle-labels every slab on its own, merges the borders, applies the maps in numpy."""
    pieces, counts = [], []
    for a, b in _bounds(img.shape[0], parts):
        lab, k = label(img[a:b])
        pieces.append(lab)
        counts.append(k)
    m = be.slab_merge(counts, np.stack([p[0] for p in pieces]), np.stack([p[-1] for p in pieces]))
    out = np.concatenate([m.lut(s, counts[s])[p] for s, p in enumerate(pieces)]).astype(np.int32)
    return out, m.total


def _images2d():
    rng = np.random.default_rng(7)
    yield "bern0.5", (rng.random((97, 131)) < 0.5).astype(np.uint8) * 255
    yield "bern0.3", (rng.random((64, 64)) < 0.3).astype(np.uint8) * 255
    yield "empty", np.zeros((40, 33), np.uint8)
    yield "full", np.full((41, 17), 255, np.uint8)
    # Vertical serpentine: columns joined alternately at the top and the bottom, so pieces of one
    # component meet only through later slabs.
    s = np.zeros((60, 61), np.uint8)
    s[:, ::2] = 255
    for c in range(1, 61, 2):
        s[0 if (c // 2) % 2 else 59, c] = 255
    yield "serpentine", s
    # Diagonal chains: joined across every border only through the corner neighbours.
    d = np.zeros((50, 50), np.uint8)
    for k in range(0, 50, 5):
        for i in range(50):
            if 0 <= i + k < 50:
                d[i, i + k] = 255
    yield "diagonals", d


@pytest.mark.parametrize("parts", [1, 2, 3, 7, 40])
def test_merge_2d_equals_whole_image(parts):
    be = _lib_or_skip()
    for name, img in _images2d():
        if parts > img.shape[0]:
            continue
        ref, k = O.ccl2d(img, 0, True)
        got, total = _join_on_host(be, img, parts, lambda x: O.ccl2d(x, 0, True))
        assert total == k, (name, parts)
        np.testing.assert_array_equal(got, ref, err_msg=f"{name} parts={parts}")


@pytest.mark.parametrize("parts", [1, 2, 5, 16])
def test_merge_3d_equals_whole_volume(parts):
    be = _lib_or_skip()
    rng = np.random.default_rng(11)
    vols = {"bern0.2": (rng.random((16, 19, 23)) < 0.2).astype(np.uint8) * 255,
            "bern0.5": (rng.random((17, 12, 9)) < 0.5).astype(np.uint8) * 255,
            "empty": np.zeros((16, 5, 6), np.uint8)}
    # a corner-only chain through the planes: (i, i, i)
    ch = np.zeros((16, 16, 16), np.uint8)
    for i in range(16):
        ch[i, i, i] = ch[i, 15 - i, i] = 255
    vols["corners"] = ch
    for name, vol in vols.items():
        ref, k = O.ccl3d(vol, 0, True)
        got, total = _join_on_host(be, vol, parts, lambda x: O.ccl3d(x, 0, True))
        assert total == k, (name, parts)
        np.testing.assert_array_equal(got, ref, err_msg=f"{name} parts={parts}")


def test_merge_random_sweep():
    """Seeded sweep: random sizes, densities and slab counts, 2D and 3D, against the oracle."""
    be = _lib_or_skip()
    rng = np.random.default_rng(2024)
    for it in range(60):
        if it % 2 == 0:
            shape = (int(rng.integers(1, 80)), int(rng.integers(1, 80)))
            label = lambda x: O.ccl2d(x, 0, True)
        else:
            shape = tuple(int(v) for v in rng.integers(1, 14, size=3))
            label = lambda x: O.ccl3d(x, 0, True)
        img = (rng.random(shape) < rng.uniform(0.05, 0.95)).astype(np.uint8) * 255
        parts = int(rng.integers(1, shape[0] + 1))
        ref, k = label(img)
        got, total = _join_on_host(be, img, parts, label)
        assert total == k, (it, shape, parts)
        np.testing.assert_array_equal(got, ref, err_msg=f"case {it} shape={shape} parts={parts}")


def test_merge_rejects_bad_borders():
    be = _lib_or_skip()
    t = np.array([[1, 0, 3]], np.int32)   # label 3 > count 2
    with pytest.raises(be.BEError):
        be.slab_merge([2], t, t)
    with pytest.raises(be.BEError):
        be.slab_merge([1], -t, -t)


def test_merge_rejects_a_short_joined_capacity():
    import ctypes
    be = _lib_or_skip()
    # Two one-row slabs whose single components join: slab 1's piece is joined under slab 0's.
    tops = np.array([[1, 0], [1, 0]], np.int32)
    counts = np.array([1, 1], np.int64)
    offsets = np.zeros(2, np.int64)
    start = np.zeros(3, np.int64)
    total = ctypes.c_int64(0)
    jl = np.zeros(4, np.int32)
    jt = np.zeros(4, np.int32)
    lib = be.lib()
    args = (2, 1, 2, counts.ctypes.data, tops.ctypes.data, tops.ctypes.data, offsets.ctypes.data,
            ctypes.byref(total), jl.ctypes.data, jt.ctypes.data, start.ctypes.data)
    assert lib.be_slab_merge(*args, 0) == 1          # BE_ERR_INVALID: one joined piece, no room
    assert lib.be_slab_merge(*args, 1) == 0
    assert total.value == 1 and list(start) == [0, 0, 1] and jl[0] == 1 and jt[0] == 1


def test_slab_bounds():
    assert _bounds(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert _bounds(5, 5) == [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5)]
    with pytest.raises(ValueError):
        _bounds(3, 4)


# ---- the exchange over gloo ranks (CPU) -----------------------------------------------------

def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, img, q):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from labeling_b200.slabs import exchange_and_merge, slab_bounds
        a, b = slab_bounds(img.shape[0], world)[rank]
        lab, k = O.ccl2d(img[a:b], 0, True)
        t = torch.from_numpy(lab)
        idx, m = exchange_and_merge(t[0], t[-1], k)
        q.put((rank, idx, m.total, m.lut(idx, k)[lab].astype(np.int32)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def _worker3d(rank, world, port, vol, q):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from labeling_b200.slabs import exchange_and_merge, slab_bounds
        a, b = slab_bounds(vol.shape[0], world)[rank]
        lab, k = O.ccl3d(vol[a:b], 0, True)
        t = torch.from_numpy(lab)
        idx, m = exchange_and_merge(t[0], t[-1], k)
        q.put((rank, idx, m.total, m.lut(idx, k)[lab].astype(np.int32)))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_exchange_3d_over_two_gloo_ranks():
    _lib_or_skip()
    import torch.multiprocessing as mp
    rng = np.random.default_rng(5)
    vol = (rng.random((13, 17, 11)) < 0.3).astype(np.uint8) * 255
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker3d, args=(r, 2, port, vol, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref, k = O.ccl3d(vol, 0, True)
    assert all(r[1] == r[0] and r[2] == k for r in res)
    np.testing.assert_array_equal(np.concatenate([r[3] for r in res]), ref)


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_over_gloo_ranks(world):
    _lib_or_skip()
    import torch.multiprocessing as mp
    rng = np.random.default_rng(3)
    img = (rng.random((45, 70)) < 0.5).astype(np.uint8) * 255
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, img, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref, k = O.ccl2d(img, 0, True)
    assert all(r[1] == r[0] and r[2] == k for r in res)
    np.testing.assert_array_equal(np.concatenate([r[3] for r in res]), ref)


# ---- the one-GPU slab path ------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("parts", [1, 2, 3, 7])
def test_gpu_label_slabs_2d(ctx, parts):
    import torch
    import labeling_b200 as be
    from labeling_b200.slabs import label_slabs
    rng = np.random.default_rng(21 + parts)
    for img in [(rng.random((515, 1029)) < 0.5).astype(np.uint8) * 255,
                (rng.random((301, 64)) < 0.3).astype(np.uint8) * 255,
                next(v for n, v in _images2d() if n == "serpentine")]:
        d = torch.from_numpy(img).cuda()
        whole = torch.zeros(img.shape, dtype=torch.int32, device="cuda")
        k = be.label2d(ctx, d, whole)
        out = torch.full(img.shape, -5, dtype=torch.int32, device="cuda")
        total = label_slabs(ctx, d, out, parts)
        torch.cuda.synchronize()
        assert total == k
        np.testing.assert_array_equal(out.cpu().numpy(), whole.cpu().numpy())
        ref, kr = O.ccl2d(img, 0, True)
        assert kr == k
        np.testing.assert_array_equal(out.cpu().numpy(), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("parts", [2, 5])
def test_gpu_label_slabs_3d(ctx, parts):
    import torch
    import labeling_b200 as be
    from labeling_b200.slabs import label_slabs
    rng = np.random.default_rng(40 + parts)
    vol = (rng.random((67, 45, 38)) < 0.3).astype(np.uint8) * 255
    d = torch.from_numpy(vol).cuda()
    whole = torch.zeros(vol.shape, dtype=torch.int32, device="cuda")
    k = be.label3d(ctx, d, whole)
    out = torch.full(vol.shape, -5, dtype=torch.int32, device="cuda")
    total = label_slabs(ctx, d, out, parts)
    torch.cuda.synchronize()
    assert total == k
    np.testing.assert_array_equal(out.cpu().numpy(), whole.cpu().numpy())


@pytest.mark.gpu
def test_gpu_slab_relabel_odd_pitch_and_offset_only(ctx):
    import torch
    import labeling_b200 as be
    lab = torch.tensor([[0, 1, 2], [2, 0, 3]], dtype=torch.int32, device="cuda")
    be.slab_relabel(ctx, lab, 3, 10, np.array([], np.int32), np.array([], np.int32))
    torch.cuda.synchronize()
    assert lab.cpu().tolist() == [[0, 11, 12], [12, 0, 13]]
    base = torch.zeros((2, 5), dtype=torch.int32, device="cuda")
    view = base[:, 1:4]
    view.copy_(torch.tensor([[0, 1, 2], [2, 0, 3]], dtype=torch.int32))
    be.slab_relabel(ctx, view, 3, 4, np.array([2], np.int32), np.array([1], np.int32))
    torch.cuda.synchronize()
    assert base.cpu().tolist() == [[0, 0, 5, 1, 0], [0, 1, 0, 6, 0]]


@pytest.mark.gpu
def test_gpu_label_distributed_one_rank(ctx):
    """label_distributed over a one-rank NCCL group on one GPU: the packed all_gather of border
    rows and count on CUDA tensors, the host merge and the relabel call in stream order, against
    whole-image labels (2D and 3D).  Several ranks need several GPUs."""
    import socket
    import torch
    import torch.distributed as dist
    from labeling_b200 import workloads as W
    from labeling_b200.slabs import label_distributed
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        for img in (W.bernoulli((777, 1301), 0.5, seed=41), W.bernoulli((40, 50, 61), 0.3, seed=42)):
            ref, k = O.ccl2d(img) if img.ndim == 2 else O.ccl3d(img)
            d = torch.from_numpy(img).cuda()
            out = torch.full(img.shape, -1, dtype=torch.int32, device="cuda")
            total = label_distributed(ctx, d, out)
            assert total == k
            assert np.array_equal(out.cpu().numpy(), ref)
    finally:
        dist.destroy_process_group()
