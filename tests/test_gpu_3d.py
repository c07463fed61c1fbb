"""3D parity on the GPU (26-connectivity), exact."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ALGOS = [1, 2]


def run3d(ctx, vol, thr=0, algo=1):
    import torch
    import labeling_b200 as be
    v = torch.from_numpy(np.ascontiguousarray(vol)).cuda()
    out = torch.full(vol.shape, -7, dtype=torch.int32, device="cuda")
    n = be.label3d(ctx, v, out, threshold=thr, algo=algo)
    torch.cuda.synchronize()
    return out.cpu().numpy(), n


@pytest.mark.parametrize("algo", ALGOS)
def test_golden_cases(ctx, golden, algo):
    for (dim, name), c in golden.items():
        if dim != "3d":
            continue
        lab, n = run3d(ctx, c["img"], 0, algo)
        assert np.array_equal(lab, c["canon"]), (name, algo)
        assert n == int(c["k"]), (name, algo)


@pytest.mark.parametrize("seed", range(10))
def test_random_shapes(ctx, seed):
    rng = np.random.default_rng(2000 + seed)
    shape = tuple(int(rng.choice([1, 2, 15, 16, 17, 31, 33, 40, 63, 65, 70])) for _ in range(3))
    p = float(rng.uniform(0.02, 0.6))
    vol = ((rng.random(shape) < p) * 255).astype(np.uint8)
    ref, k = O.ccl3d(vol)
    for algo in ALGOS:
        lab, n = run3d(ctx, vol, 0, algo)
        assert n == k and np.array_equal(lab, ref), (shape, algo)


@pytest.mark.parametrize("p", [0.1, 0.3, 0.5])
def test_128_cube_bernoulli(ctx, p):
    from labeling_b200 import workloads as W
    vol = W.bernoulli((128, 130, 129), p, seed=int(p * 10))
    ref, k = O.ccl3d(vol)
    for algo in ALGOS:
        lab, n = run3d(ctx, vol, 0, algo)
        assert n == k and np.array_equal(lab, ref), algo


@pytest.mark.parametrize("pct", [50, 80])
def test_grf(ctx, pct):
    from labeling_b200 import workloads as W
    vol = W.grf((96, 96, 96), 4.0, pct, seed=pct)
    ref, k = O.ccl3d(vol)
    lab, n = run3d(ctx, vol)
    assert n == k and np.array_equal(lab, ref)


def test_host_api_and_reference_interface(ctx):
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    vol = W.bernoulli((40, 50, 60), 0.25, seed=5)
    ref, k = O.ccl3d(vol)
    lab, n, us = be.label3d_host(ctx, vol)
    assert n == k and np.array_equal(lab, ref)
    lab2, _ = be.make_labeler("bleq", gpu=True, three_d=True).Label(vol)
    assert np.array_equal(lab2, ref)
    with pytest.raises(ValueError):
        be.make_labeler("bleq", gpu=True, three_d=True).Label(vol, coh=be.COH_8)


@pytest.mark.parametrize("p", [0.1, 0.12, 0.3])
def test_large_volume_repeated(ctx, p):
    """Large volumes near the 26-connectivity percolation threshold, labeled three times: each run
    must equal the oracle (catches schedule-dependent races)."""
    from labeling_b200 import workloads as W
    vol = W.bernoulli((384, 384, 320), p, seed=int(p * 1000))
    ref, k = O.ccl3d(vol)
    for _ in range(3):
        lab, n = run3d(ctx, vol)
        assert n == k and np.array_equal(lab, ref)


def test_pixel_label_equivalence_lbeq_3d(ctx, golden):
    """-a lbeq -3 -g: voxel-level label equivalence, 26-connectivity; equals the reference's own
    LBEQ3D labels (golden) after canonicalisation."""
    import labeling_b200 as be
    for (dim, name), c in golden.items():
        if dim != "3d":
            continue
        lab, n, _ = be.label3d_host(ctx, c["img"], 0, be.ALGO_PIXEL)
        gold, k = O.canon(c["lbeq"])
        assert n == k and np.array_equal(lab, gold), name
    from labeling_b200 import workloads as W
    vol = W.bernoulli((70, 80, 90), 0.2, seed=12)
    lab, n, _ = be.label3d_host(ctx, vol, 0, be.ALGO_PIXEL)
    ref, k = O.ccl3d(vol)
    assert n == k and np.array_equal(lab, ref)
