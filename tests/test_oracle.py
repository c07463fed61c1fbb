"""The oracle (test infrastructure) against the golden fixtures made by the reference's own code,
and against independent labelers.  CPU only."""
import numpy as np
import pytest
import scipy.ndimage as ndi

from oracle import oracle as O


def test_be2d_restatement_matches_reference_labels(golden):
    """The C restatement reproduces the reference LBEQ2_* label VALUES, not only the partition."""
    n = 0
    for (dim, name), c in golden.items():
        if dim != "2d":
            continue
        raw = O.be2d_raw(c["img"], int(c["thr"]))
        assert np.array_equal(raw, c["raw"]), name
        can, k = O.canon(raw)
        assert np.array_equal(can, c["canon"]) and k == int(c["k"]), name
        n += 1
    assert n >= 20


def test_be3d_restatement_matches_reference_labels(golden):
    n = 0
    for (dim, name), c in golden.items():
        if dim != "3d":
            continue
        raw = O.be3d_raw(c["img"], 0)
        assert np.array_equal(raw, c["raw"]), name
        n += 1
    assert n >= 7


def test_lbeq_restatement_matches_reference(golden):
    for (dim, name), c in golden.items():
        if dim == "2d":
            thr = int(c["thr"])
            assert np.array_equal(O.lbeq2d_raw(c["img"], thr, conn8=False), c["distr4"]), name
            assert np.array_equal(O.lbeq2d_raw(c["img"], thr, conn8=True), c["distr8"]), name
        else:
            assert np.array_equal(O.lbeq3d_raw(c["img"], 0), c["lbeq"]), name


def test_union_find_oracle_agrees_with_golden(golden):
    for (dim, name), c in golden.items():
        if dim == "2d":
            can, k = O.ccl2d(c["img"], int(c["thr"]))
        else:
            can, k = O.ccl3d(c["img"], 0)
        assert np.array_equal(can, c["canon"]) and k == int(c["k"]), name


def test_grana_golden_is_the_same_partition(golden):
    for (dim, name), c in golden.items():
        if dim != "2d":
            continue
        g, _ = O.canon(c["grana"].astype(np.uint32))
        assert np.array_equal(g, c["canon"]), name


@pytest.mark.parametrize("seed", range(6))
def test_oracles_agree_with_scipy(seed):
    rng = np.random.default_rng(seed)
    h, w = rng.integers(1, 120, 2)
    img = ((rng.random((h, w)) < rng.uniform(0.05, 0.95)) * 255).astype(np.uint8)
    lab, k = ndi.label(img > 0, structure=np.ones((3, 3)))
    s, ks = O.canon(lab.astype(np.uint32))
    a, ka = O.be2d(img)
    b, kb = O.ccl2d(img)
    assert np.array_equal(a, s) and np.array_equal(b, s) and ka == kb == ks
    vol = ((rng.random(tuple(rng.integers(1, 24, 3))) < rng.uniform(0.05, 0.5)) * 255).astype(np.uint8)
    lab3, _ = ndi.label(vol > 0, structure=np.ones((3, 3, 3)))
    s3, _ = O.canon(lab3.astype(np.uint32))
    assert np.array_equal(O.be3d(vol)[0], s3) and np.array_equal(O.ccl3d(vol)[0], s3)


def test_reference_quirks_are_reproduced(golden):
    """-a lbeq -g in 2D: COH_DEFAULT is 4-connectivity and a foreground pixel at (0, 0) keeps label
    0 (LabelingAlgs.cl:37, 48-50, 68); both behaviours are in the golden data."""
    c = golden[("2d", "corners_10x12")]
    assert c["distr4"][0, 0] == 0 and c["img"][0, 0] == 255
    c = golden[("2d", "checker_40")]
    k4 = len(np.unique(c["distr4"])) - 1
    assert k4 > 1 and int(c["k"]) == 1
