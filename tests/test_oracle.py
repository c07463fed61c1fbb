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


# --- the reference's own CPU code (oracle/_ref), present only where it was built ---------------

needs_ref_cpu = pytest.mark.skipif(O.cpu_lib() is None, reason="oracle/_ref/libref_cpu.so not built")
needs_ref_kernels = pytest.mark.skipif(O.ref_lib() is None, reason="oracle/_ref/libref_be.so not built")


@needs_ref_cpu
@pytest.mark.parametrize("seed", range(4))
def test_reference_cpu_bleq_matches_oracle_with_one_background_row_and_column(seed):
    """The reference's OpenMP block labeler (TLabelEquivalenceX2, the CPU baseline) gives the
    oracle's partition once its border probes cannot wrap: one background row and column
    appended (how the baseline is run), any size, odd or even."""
    rng = np.random.default_rng(seed)
    for _ in range(25):
        h, w = rng.integers(1, 90, 2)
        img = ((rng.random((h, w)) < rng.uniform(0.2, 0.8)) * 255).astype(np.uint8)
        raw, us = O.ref_cpu_bleq(img)
        assert np.array_equal(O.canon(raw)[0], O.ccl2d(img)[0]) and us >= 0


@needs_ref_cpu
def test_reference_cpu_bleq_right_border_wrap_is_the_references():
    """At the right border the reference's CPU block labeler reads the next row's first pixels
    (RemoveBorderBlocks compares pixel coordinates with the image size, LabelingAlgs.cpp:366-374):
    in this 4 x 4 image the pixel at (0, 3) "touches" (1, 0) through the wrap, and the two
    components come out as one.  With the background row and column the baseline appends, the
    labels are exact.  The GPU path follows the reference's GPU kernels, which pad the image and
    do not wrap."""
    img = np.zeros((4, 4), np.uint8)
    img[0, 3] = img[1, 0] = img[2, 0] = 255
    raw, _ = O.ref_cpu_bleq(img, pad=False)
    assert O.canon(raw)[1] == 1 and O.ccl2d(img)[1] == 2
    assert O.canon(O.ref_cpu_bleq(img)[0])[1] == 2


@needs_ref_kernels
def test_reference_3d_kernels_threaded_match_serial():
    """The reference's 3D kernels on the host over OpenMP threads (the 3D CPU baseline) give the
    serial sweep's partition and the oracle's."""
    rng = np.random.default_rng(11)
    for shape, p in [((21, 34, 47), 0.3), ((64, 64, 64), 0.25)]:
        vol = ((rng.random(shape) < p) * 255).astype(np.uint8)
        serial, _ = O.ref_be3d_timed(vol, 0, 1)
        threaded, _ = O.ref_be3d_timed(vol, 0, 0)
        ref = O.ccl3d(vol)[0]
        assert np.array_equal(O.canon(serial)[0], ref) and np.array_equal(O.canon(threaded)[0], ref)


def test_reference_run_equivalence_kernels_are_4_connected(golden):
    """The reference's GPU run equivalence (RE* kernels, golden outputs) joins runs that overlap in
    a column: its labels are exactly the 4-connected components, which is what the runeq slot of
    this package returns."""
    for (dim, name), c in golden.items():
        if dim != "2d":
            continue
        assert np.array_equal(O.canon(c["runeq"])[0], O.ccl2d(c["img"], int(c["thr"]), False)[0]), name
