"""2D parity on the GPU: every label map must equal the oracle's canonical labels bit for bit
(integer work: the tolerance is exact) and the component count must match."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ALGOS = [1, 2]   # BE_ALGO_UF, BE_ALGO_ITER


def run2d(ctx, img, thr=0, algo=1, pitch_pad=0, offset=0):
    import torch
    import labeling_b200 as be
    h, w = img.shape
    buf = torch.zeros(h * (w + pitch_pad) + offset + 64, dtype=torch.uint8, device="cuda")
    view = buf[offset:offset + h * (w + pitch_pad)].view(h, w + pitch_pad)[:, :w]
    view.copy_(torch.from_numpy(img).cuda())
    out = torch.full((h, w + pitch_pad), -7, dtype=torch.int32, device="cuda")[:, :w]
    n = be.label2d(ctx, view, out, threshold=thr, algo=algo)
    torch.cuda.synchronize()
    return out.cpu().numpy(), n


@pytest.mark.parametrize("algo", ALGOS)
def test_golden_cases(ctx, golden, algo):
    for (dim, name), c in golden.items():
        if dim != "2d":
            continue
        lab, n = run2d(ctx, c["img"], int(c["thr"]), algo)
        assert np.array_equal(lab, c["canon"]), (name, algo)
        assert n == int(c["k"]), (name, algo)


@pytest.mark.parametrize("seed", range(12))
def test_random_shapes_uf_vs_oracle(ctx, seed):
    rng = np.random.default_rng(1000 + seed)
    h = int(rng.choice([1, 2, 3, 63, 64, 65, 127, 129, 200, 511, 700]))
    w = int(rng.choice([1, 2, 5, 255, 256, 257, 300, 513, 1000, 1023]))
    p = float(rng.uniform(0.05, 0.95))
    img = ((rng.random((h, w)) < p) * 255).astype(np.uint8)
    ref, k = O.ccl2d(img)
    lab, n = run2d(ctx, img, 0, 1)
    assert np.array_equal(lab, ref) and n == k


@pytest.mark.parametrize("p", [0.1, 0.4, 0.5, 0.6, 0.9])
def test_2048_bernoulli_both_forms(ctx, p):
    from labeling_b200 import workloads as W
    img = W.bernoulli((2048, 2048), p, seed=int(p * 100))
    ref, k = O.ccl2d(img)
    for algo in ALGOS:
        lab, n = run2d(ctx, img, 0, algo)
        assert n == k and np.array_equal(lab, ref), algo


@pytest.mark.parametrize("family", ["serpentine", "spiral", "disks"])
def test_worst_case_paths(ctx, family):
    from labeling_b200 import workloads as W
    img = W.family_8192(family, seed=3, side=1536)
    ref, k = O.ccl2d(img)
    for algo in ALGOS:
        lab, n = run2d(ctx, img, 0, algo)
        assert n == k and np.array_equal(lab, ref), algo


def test_pitch_offset_threshold(ctx):
    rng = np.random.default_rng(7)
    img = rng.integers(0, 256, (333, 517)).astype(np.uint8)
    for thr in (0, 8, 128, 254):
        ref, k = O.ccl2d(img, thr)
        for pad, off in ((0, 0), (11, 3), (64, 16)):
            lab, n = run2d(ctx, img, thr, 1, pad, off)
            assert n == k and np.array_equal(lab, ref), (thr, pad, off)


def test_edge_shapes(ctx):
    for img in (np.zeros((1, 1), np.uint8), np.full((1, 1), 255, np.uint8),
                np.full((1, 4097), 255, np.uint8), np.full((4097, 1), 255, np.uint8),
                np.zeros((300, 300), np.uint8), np.full((300, 301), 255, np.uint8),
                (np.indices((256, 256)).sum(0) % 2 * 255).astype(np.uint8)):
        ref, k = O.ccl2d(img)
        for algo in ALGOS:
            lab, n = run2d(ctx, img, 0, algo)
            assert n == k and np.array_equal(lab, ref), (img.shape, algo)


def test_repeat_is_deterministic(ctx):
    from labeling_b200 import workloads as W
    img = W.bernoulli((1111, 2222), 0.45, seed=9)
    a, na = run2d(ctx, img)
    b, nb = run2d(ctx, img)
    assert na == nb and np.array_equal(a, b)


def test_host_api_and_reference_interface(ctx):
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    img = W.bernoulli((777, 555), 0.5, seed=11)
    ref, k = O.ccl2d(img)
    lab, n, us = be.label2d_host(ctx, img)
    assert n == k and np.array_equal(lab, ref) and us > 0
    lab2, us2 = be.make_labeler("bleq", gpu=True).Label(img)
    assert np.array_equal(lab2, ref) and us2 > 0
    with pytest.raises(be.BEError):
        be.label2d_host(ctx, img, coh=be.COH_4)


@pytest.mark.parametrize("p", [0.41, 0.45, 0.6])
def test_large_image_repeated(ctx, p):
    """4096^2 near the 8-connectivity percolation threshold, three runs, each exact."""
    from labeling_b200 import workloads as W
    img = W.bernoulli((4096, 4100), p, seed=int(p * 1000))
    ref, k = O.ccl2d(img)
    for _ in range(3):
        lab, n = run2d(ctx, img)
        assert n == k and np.array_equal(lab, ref)


@pytest.mark.parametrize("conn8", [False, True])
def test_pixel_label_equivalence_lbeq(ctx, golden, conn8):
    """-a lbeq -g: pixel-level label equivalence, 4-connectivity by default (the reference's
    COH_DEFAULT) and 8 with -c 8.  Canonical labels equal the union-find oracle with the same
    connectivity, and the reference's own lbeq labels (golden) after canonicalisation, except where
    the reference's pixel-(0,0) quirk applies."""
    import labeling_b200 as be
    coh = be.COH_8 if conn8 else be.COH_DEFAULT
    for (dim, name), c in golden.items():
        if dim != "2d":
            continue
        img, thr = c["img"], int(c["thr"])
        lab, n, _ = be.label2d_host(ctx, img, thr, be.ALGO_PIXEL, coh)
        ref, k = O.ccl2d(img, thr, conn8=conn8)
        assert n == k and np.array_equal(lab, ref), name
        if img[0, 0] <= thr:
            gold, _ = O.canon(c["distr8" if conn8 else "distr4"])
            assert np.array_equal(lab, gold), name
    from labeling_b200 import workloads as W
    for p in (0.3, 0.55, 0.8):
        img = W.bernoulli((700, 900), p, seed=int(100 * p))
        lab, n, _ = be.label2d_host(ctx, img, 0, be.ALGO_PIXEL, coh)
        ref, k = O.ccl2d(img, 0, conn8=conn8)
        assert n == k and np.array_equal(lab, ref)


def test_run_equivalence_slot_matches_reference_kernels(ctx, golden):
    """-a runeq -g: the reference's run kernels (golden outputs) give 4-connected components; the
    slot labels them with the run-equivalence form, 4-connected, and rejects COH_4 as the
    reference does."""
    import labeling_b200 as be
    for (dim, name), c in golden.items():
        if dim != "2d":
            continue
        lab, n, _ = be.label2d_host(ctx, c["img"], int(c["thr"]), be.ALGO_RUNS, be.COH_4)
        want, k = O.canon(c["runeq"])
        assert n == k and np.array_equal(lab, want), name
    lab_alg = be.make_labeler("runeq")
    img = (np.random.default_rng(4).random((90, 130)) < 0.5).astype(np.uint8) * 255
    labels, _ = lab_alg.Label(img)
    assert np.array_equal(labels, O.ccl2d(img, 8, False)[0])
    with pytest.raises(ValueError):
        lab_alg.Label(img, coh=be.COH_4)
    with pytest.raises(ValueError):
        be.make_labeler("runeq", three_d=True)


def test_iterative_graph_cache_reuse(ctx):
    """The iterative and pixel forms keep their instantiated graph per size: a call with a new
    image, new buffers or a new threshold at the same size reuses it (only the image arguments
    change), a new size rebuilds it.  Every result exact, in both directions of the switch."""
    import torch
    import labeling_b200 as be
    rng = np.random.default_rng(99)
    for (h, w), thr in [((300, 400), 0), ((300, 400), 100), ((301, 400), 0), ((300, 400), 0), ((300, 400), 7)]:
        img = rng.integers(0, 256, (h, w)).astype(np.uint8)
        ref, k = O.ccl2d(img, thr)
        lab, n = run2d(ctx, img, thr, algo=2)
        assert n == k and np.array_equal(lab, ref), (h, w, thr)
        lab, n = run2d(ctx, img, thr, algo=3)          # pixel form, 4-connected by default
        ref4, k4 = O.ccl2d(img, thr, False)
        assert n == k4 and np.array_equal(lab, ref4), (h, w, thr, "pixel 4")
        d = torch.from_numpy(img).cuda()
        out = torch.empty((h, w), dtype=torch.int32, device="cuda")
        n8 = be.label2d(ctx, d, out, threshold=thr, algo=be.ALGO_PIXEL, coh=be.COH_8)
        assert n8 == k and np.array_equal(out.cpu().numpy(), ref), (h, w, thr, "pixel")
    for shape, thr in [((20, 30, 40), 0), ((20, 30, 40), 50), ((21, 30, 40), 0)]:
        vol = rng.integers(0, 256, shape).astype(np.uint8)
        ref, k = O.ccl3d(vol, thr)
        d = torch.from_numpy(vol).cuda()
        out = torch.empty(shape, dtype=torch.int32, device="cuda")
        assert be.label3d(ctx, d, out, threshold=thr, algo=be.ALGO_ITER) == k
        assert np.array_equal(out.cpu().numpy(), ref), (shape, thr)


@pytest.mark.parametrize("seed", range(8))
def test_run_equivalence_form_vs_oracle(ctx, seed):
    """The run-equivalence form (runs per row, overlap ranges, Scan / Analyze) on random shapes,
    pitches and thresholds: 4-connectivity (BE_COH_4 and the default) and 8 (BE_COH_8), exact."""
    import labeling_b200 as be
    rng = np.random.default_rng(300 + seed)
    h = int(rng.choice([1, 2, 3, 31, 32, 33, 100, 257]))
    w = int(rng.choice([1, 2, 31, 32, 33, 63, 64, 65, 500, 1025]))
    img = rng.integers(0, 256, (h, w)).astype(np.uint8)
    thr = int(rng.choice([0, 100, 200]))
    for coh, conn8 in ((be.COH_4, False), (be.COH_DEFAULT, False), (be.COH_8, True)):
        ref, k = O.ccl2d(img, thr, conn8)
        for pad, off in ((0, 0), (7, 5)):
            import torch
            buf = torch.zeros(h * (w + pad) + off + 64, dtype=torch.uint8, device="cuda")
            view = buf[off:off + h * (w + pad)].view(h, w + pad)[:, :w]
            view.copy_(torch.from_numpy(img).cuda())
            out = torch.full((h, w + pad), -7, dtype=torch.int32, device="cuda")[:, :w]
            n = be.label2d(ctx, view, out, threshold=thr, algo=be.ALGO_RUNS, coh=coh)
            assert n == k and np.array_equal(out.cpu().numpy(), ref), (h, w, thr, coh, pad, off)


@pytest.mark.parametrize("family", ["serpentine", "spiral", "bern0.5"])
def test_run_equivalence_long_paths(ctx, family):
    """Paths that need many Scan / Analyze rounds (one serpentine or spiral run chain) and dense
    noise, 2048 x 2048, both connectivities, exact; full-size images are in test_gpu_full.py."""
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    img = W.family_8192(family, seed=5, side=2048)
    for coh, conn8 in ((be.COH_4, False), (be.COH_8, True)):
        ref, k = O.ccl2d(img, 0, conn8)
        lab, n = run2d(ctx, img, 0, algo=be.ALGO_RUNS) if coh == be.COH_4 else (None, None)
        if coh == be.COH_8:
            import torch
            d = torch.from_numpy(img).cuda()
            o = torch.empty(img.shape, dtype=torch.int32, device="cuda")
            n = be.label2d(ctx, d, o, algo=be.ALGO_RUNS, coh=be.COH_8)
            lab = o.cpu().numpy()
        assert n == k and np.array_equal(lab, ref), (family, coh)


def test_run_equivalence_rejects_3d(ctx):
    import torch
    import labeling_b200 as be
    v = torch.zeros((4, 5, 6), dtype=torch.uint8, device="cuda")
    o = torch.zeros((4, 5, 6), dtype=torch.int32, device="cuda")
    with pytest.raises(be.BEError):
        be.label3d(ctx, v, o, algo=be.ALGO_RUNS)
