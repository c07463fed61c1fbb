"""Parity at the benchmark configurations' own sizes: every label map the benchmark times must
equal the oracle's canonical labels bit for bit, with the same component count.

* 2D: the seven 8192 x 8192 families with the benchmark's seeds (Bernoulli p = 0.1 / 0.4 / 0.6 /
  0.9, 2000 disks over p = 0.05 noise, serpentine, spiral);
* 3D: the five 512^3 volumes with the benchmark's seeds (Bernoulli p = 0.1 / 0.3 / 0.5, Gaussian
  random field sigma 4 thresholded at its 50th and 80th percentiles);
* batch: 4096 images with sides log-uniform in [64, 2048] and densities U[0.2, 0.8] in one batch
  launch -- every image equal to its plain call, a seeded sample of 64 equal to the oracle;
* served: a mixed stream with 2D sides up to 8192 and 3D sides up to 384, every result equal to
  the oracle.

The oracle runs in threads (the C oracle releases the GIL through ctypes and keeps no state
between calls), one image at a time per thread.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

_POOL = 8


def _ref(img):
    return O.ccl2d(img) if img.ndim == 2 else O.ccl3d(img)


def _check_all(items):
    """items: list of (name, image, labels numpy, count).  Compares all of them against the
    oracle in parallel threads; returns the list of mismatching names."""
    def one(it):
        name, img, lab, n = it
        ref, k = _ref(img)
        return None if (n == k and np.array_equal(lab, ref)) else (name, n, k, int((lab != ref).sum()))
    with ThreadPoolExecutor(_POOL) as ex:
        return [r for r in ex.map(one, items) if r is not None]


def test_2d_8192_seven_families(ctx):
    import torch
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    items = []
    for i, fam in enumerate(W.FAMILIES_8192):
        img = W.family_8192(fam, seed=10 + i)       # the benchmark's image for this family
        d_in = torch.from_numpy(img).cuda()
        d_out = torch.full(img.shape, -1, dtype=torch.int32, device="cuda")
        n = be.label2d(ctx, d_in, d_out)
        # a second labeling of the same image must give the same map (schedule independence)
        d_out2 = torch.full(img.shape, -2, dtype=torch.int32, device="cuda")
        assert be.label2d(ctx, d_in, d_out2) == n
        assert torch.equal(d_out, d_out2), fam
        items.append((fam, img, d_out.cpu().numpy(), n))
        del d_in, d_out, d_out2
    assert _check_all(items) == []


def test_3d_512_five_volumes(ctx):
    import torch
    import labeling_b200 as be
    import bench
    vols = bench.make_3d_inputs(512, seed=100)      # the benchmark's volumes
    assert [n for n, _ in vols] == ["bern0.1", "bern0.3", "bern0.5", "grf50", "grf80"]
    items = []
    for name, vol in vols:
        d_in = torch.from_numpy(vol).cuda()
        d_out = torch.full(vol.shape, -1, dtype=torch.int32, device="cuda")
        n = be.label3d(ctx, d_in, d_out)
        items.append((name, vol, d_out.cpu().numpy(), n))
        del d_in, d_out
    torch.cuda.empty_cache()
    assert _check_all(items) == []


def test_batch_4096_uneven_images():
    import torch
    import labeling_b200 as be
    import bench
    c = be.Context(0)
    sides, d_in = bench.make_batch_inputs(4096, rank=0, dev=torch.device("cuda", 0))
    d_out = [torch.full((h, w), -3, dtype=torch.int32, device="cuda") for h, w in sides]
    b = be.Batch(c, list(zip(d_in, d_out)))
    b.tune()
    b.run()
    counts = b.counts()
    # every image equals its own plain call
    scratch = {}
    bad = []
    for i, ((h, w), x) in enumerate(zip(sides, d_in)):
        o = scratch.get((h, w))
        if o is None:
            o = scratch[(h, w)] = torch.empty((h, w), dtype=torch.int32, device="cuda")
        n = be.label2d(c, x, o)
        if n != counts[i] or not torch.equal(o, d_out[i]):
            bad.append(i)
    assert bad == []
    # a seeded sample against the oracle
    pick = np.random.default_rng(77).choice(len(sides), 64, replace=False)
    items = [(int(i), d_in[i].cpu().numpy(), d_out[i].cpu().numpy(), counts[i]) for i in pick]
    assert _check_all(items) == []
    b.close()
    c.close()


def test_served_mix_up_to_8192():
    import torch
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    rng = np.random.default_rng(31)
    imgs = [W.bernoulli((8192, 8192), 0.45, seed=32)]            # the largest 2D side
    for i in range(23):
        if rng.random() < 0.8:
            s = int(np.exp(rng.uniform(np.log(256), np.log(8192))))
            imgs.append(W.bernoulli((s, s), float(rng.uniform(0.2, 0.8)), int(rng.integers(1 << 30))))
        else:
            s = int(np.exp(rng.uniform(np.log(64), np.log(384))))
            imgs.append(W.grf((s, s, s), 4.0, 60, int(rng.integers(1 << 30)), device="cuda"))
    h_in = [torch.from_numpy(a).pin_memory() for a in imgs]
    h_out = [torch.full(a.shape, -1, dtype=torch.int32).pin_memory() for a in imgs]
    srv = be.Server(lanes=2, max_batch=16)
    ids = [srv.submit(a.numpy(), o.numpy()) for a, o in zip(h_in, h_out)]
    res = [srv.wait(i) for i in ids]
    srv.close()
    assert all(r[0] == 0 for r in res)
    items = [(i, imgs[i], h_out[i].numpy(), res[i][1]) for i in range(len(imgs))]
    assert _check_all(items) == []
