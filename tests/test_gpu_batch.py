"""Batched labeling (one CUDA graph over many uneven 2D images and 3D volumes) and the
autotuner: every image of a batch must equal its own plain-call result and the oracle exactly."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _uneven_batch(seed, n2d=40, n3d=6):
    from labeling_b200 import workloads as W
    rng = np.random.default_rng(seed)
    items = []
    for (h, w) in W.log_uniform_sides(n2d, 17, 700, seed):
        items.append(W.bernoulli((h, w), float(rng.uniform(0.2, 0.8)), int(rng.integers(1 << 30))))
    for (a, b, c) in W.log_uniform_sides(n3d, 5, 70, seed + 1, dims=3):
        items.append(W.bernoulli((a, b, c), float(rng.uniform(0.05, 0.4)), int(rng.integers(1 << 30))))
    return items


@pytest.mark.parametrize("flags", [0, 0x100])
def test_batch_matches_oracle_and_plain(ctx, flags):
    import torch
    import labeling_b200 as be
    imgs = _uneven_batch(5)
    d_in = [torch.from_numpy(a).cuda() for a in imgs]
    d_out = [torch.full(a.shape, -3, dtype=torch.int32, device="cuda") for a in imgs]
    b = be.Batch(ctx, list(zip(d_in, d_out)), flags)
    b.run()
    counts = b.counts()
    for i, a in enumerate(imgs):
        ref, k = O.ccl2d(a) if a.ndim == 2 else O.ccl3d(a)
        assert counts[i] == k, i
        assert np.array_equal(d_out[i].cpu().numpy(), ref), i
    # run again (graph replay) after scribbling over the outputs
    for o in d_out:
        o.fill_(-5)
    b.run()
    assert b.counts() == counts
    ref0, _ = O.ccl2d(imgs[0])
    assert np.array_equal(d_out[0].cpu().numpy(), ref0)
    b.close()


def test_batch_tune_keeps_results(ctx):
    import torch
    import labeling_b200 as be
    imgs = _uneven_batch(9, n2d=25, n3d=3)
    d_in = [torch.from_numpy(a).cuda() for a in imgs]
    d_out = [torch.zeros(a.shape, dtype=torch.int32, device="cuda") for a in imgs]
    b = be.Batch(ctx, list(zip(d_in, d_out)))
    choice = b.tune()
    assert 0 <= (choice & 0xFF) < 3
    b.run()
    counts = b.counts()
    for i, a in enumerate(imgs):
        ref, k = O.ccl2d(a) if a.ndim == 2 else O.ccl3d(a)
        assert counts[i] == k and np.array_equal(d_out[i].cpu().numpy(), ref), i
    b.close()


def test_autotune_forms_agree_and_are_used(ctx, tmp_path):
    import torch
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    img = W.bernoulli((1500, 1700), 0.5, seed=3)
    d = torch.from_numpy(img).cuda()
    o = torch.zeros(img.shape, dtype=torch.int32, device="cuda")
    choice = be.autotune2d(ctx, d, o)            # checks internally that every form agrees
    assert choice in (0, 1, 2, 16)
    ref, k = O.ccl2d(img)
    assert np.array_equal(o.cpu().numpy(), ref)
    o.zero_()
    assert be.label2d(ctx, d, o) == k and np.array_equal(o.cpu().numpy(), ref)
    path = str(tmp_path / "tune.txt")
    ctx.tune_save(path)
    c2 = be.Context(0)
    c2.tune_load(path)
    o.zero_()
    assert be.label2d(c2, d, o) == k and np.array_equal(o.cpu().numpy(), ref)
    c2.close()
    vol = W.bernoulli((60, 70, 80), 0.2, seed=4)
    v = torch.from_numpy(vol).cuda()
    ov = torch.zeros(vol.shape, dtype=torch.int32, device="cuda")
    assert be.autotune3d(ctx, v, ov) in (0, 16)
    assert np.array_equal(ov.cpu().numpy(), O.ccl3d(vol)[0])


@pytest.mark.parametrize("shape", [0, 1, 2])
def test_each_tile_shape_exact(ctx, shape):
    """Route the plain 2D call to each tile shape through a loaded tuning table."""
    import os
    import tempfile
    import torch
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    rng = np.random.default_rng(shape)
    for _ in range(4):
        h, w = int(rng.integers(1, 900)), int(rng.integers(1, 1300))
        img = W.bernoulli((h, w), float(rng.uniform(0.1, 0.9)), int(rng.integers(1 << 20)))
        c = be.Context(0)
        cls = (2 << 16) | (int(np.floor(np.log2(h))) << 8) | int(np.floor(np.log2(w)))
        with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
            f.write(f"{cls} 1 {shape} 1.0\n")
        c.tune_load(f.name)
        os.unlink(f.name)
        d = torch.from_numpy(img).cuda()
        o = torch.zeros(img.shape, dtype=torch.int32, device="cuda")
        ref, k = O.ccl2d(img)
        assert be.label2d(c, d, o) == k and np.array_equal(o.cpu().numpy(), ref), (h, w, shape)
        c.close()
