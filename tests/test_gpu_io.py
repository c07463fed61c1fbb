"""Ingest and egress on the device against numpy restatements of the reference's host steps
(exact: byte work).  RGB2Gray (LabelingTools.cpp:39-49), Read3DImage's slice stacking
(main.cpp:172-212), LabelsToRGB / Write3DLabels (main.cpp:248-305, with a deterministic colour
map in place of std::rand)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def gray_ref(img: np.ndarray, binarize: bool = True, rgb: bool = False, opencv4: bool = False) -> np.ndarray:
    """cv::COLOR_RGB2GRAY on 8-bit data, then threshold 8.  OpenCV 3.0.0 (the reference's version)
    rounds 0.299 / 0.587 / 0.114 with 14-bit weights; OpenCV 4 with 15-bit weights summing to
    2^15 (tests/test_io_restatement.py pins the latter to the cv2 in this image)."""
    if rgb:
        r, g, b = (img[..., k].astype(np.uint32) for k in range(3))
        if opencv4:
            y = (r * 9798 + g * 19235 + b * 3735 + (1 << 14)) >> 15
        else:
            y = (r * 4899 + g * 9617 + b * 1868 + (1 << 13)) >> 14
    else:
        y = img.astype(np.uint32)
    return np.where(y > 8, 255, 0).astype(np.uint8) if binarize else y.astype(np.uint8)


def colour_ref(labels: np.ndarray, seed: int) -> np.ndarray:
    """Background black; label l -> low 3 bytes of the MurmurHash3 finalizer of l ^ (seed * phi)."""
    l = labels.astype(np.uint32)
    with np.errstate(over="ignore"):
        h = l ^ np.uint32((seed * 0x9E3779B9) & 0xFFFFFFFF)
        h ^= h >> np.uint32(16)
        h *= np.uint32(0x85EBCA6B)
        h ^= h >> np.uint32(13)
        h *= np.uint32(0xC2B2AE35)
        h ^= h >> np.uint32(16)
    h = np.where(labels == 0, np.uint32(0), h & np.uint32(0xFFFFFF))
    return np.stack([(h >> np.uint32(8 * k)) & np.uint32(255) for k in range(3)], -1).astype(np.uint8)


@pytest.mark.parametrize("channels", [1, 3])
def test_to_gray_matches_rgb2gray(ctx, channels):
    import torch
    import labeling_b200 as be
    rng = np.random.default_rng(3)
    shape = (333, 517, 3) if channels == 3 else (333, 517)
    img = rng.integers(0, 40, shape, dtype=np.uint8)   # values around the threshold of 8
    d = torch.from_numpy(img).cuda()
    for binarize in (True, False):
        out = torch.empty((333, 517), dtype=torch.uint8, device="cuda")
        be.to_gray(ctx, d, out, binarize=binarize)
        assert np.array_equal(out.cpu().numpy(), gray_ref(img, binarize, channels == 3))


@pytest.mark.parametrize("channels", [1, 3])
def test_to_gray_matches_opencv(ctx, channels):
    """Pinned to OpenCV itself: the reference's RGB2Gray is cv::cvtColor(COLOR_RGB2GRAY) for
    colour input, then cv::threshold(img, img, cv::THRESH_OTSU, 255, CV_8UC1) -- THRESH_OTSU (8)
    passed as the threshold value and CV_8UC1 (0) as the type, THRESH_BINARY
    (LabelingTools.cpp:39-49)."""
    import cv2
    import torch
    import labeling_b200 as be
    rng = np.random.default_rng(11 + channels)
    shape = (301, 419, 3) if channels == 3 else (301, 419)
    for hi in (40, 256):
        img = rng.integers(0, hi, shape, dtype=np.uint8)
        gray = cv2.cvtColor(img, cv2.COLOR_RGB2GRAY) if channels == 3 else img
        _, want = cv2.threshold(gray, cv2.THRESH_OTSU, 255, cv2.THRESH_BINARY)
        d = torch.from_numpy(img).cuda()
        out = torch.empty(shape[:2], dtype=torch.uint8, device="cuda")
        # the cv2 in this image is OpenCV 4: its weights, bit for bit
        be.to_gray(ctx, d, out, binarize=True, opencv4=True)
        assert np.array_equal(out.cpu().numpy(), want)
        be.to_gray(ctx, d, out, binarize=False, opencv4=True)
        assert np.array_equal(out.cpu().numpy(), gray)
        # the default (OpenCV 3.0.0's weights) stays within one gray level of it
        be.to_gray(ctx, d, out, binarize=False)
        diff = np.abs(out.cpu().numpy().astype(np.int32) - gray.astype(np.int32))
        assert diff.max() <= 1 and (channels == 3 or diff.max() == 0)


@pytest.mark.parametrize("channels,shape", [(1, (70, 45, 33)), (3, (40, 37, 65)), (1, (1, 1, 1))])
def test_stack_slices_then_label(ctx, channels, shape):
    """Slices -> volume with the slice index fastest, then 3D BE on it, equals the oracle on the
    numpy-stacked volume."""
    import torch
    import labeling_b200 as be
    planes, rows, cols = shape
    rng = np.random.default_rng(planes)
    sl = rng.integers(0, 20, shape + ((3,) if channels == 3 else ()), dtype=np.uint8)
    ref_vol = np.ascontiguousarray(np.transpose(gray_ref(sl, True, channels == 3), (1, 2, 0)))
    d = torch.from_numpy(sl).cuda()
    vol = torch.empty((rows, cols, planes), dtype=torch.uint8, device="cuda")
    be.stack_slices(ctx, d, vol)
    assert np.array_equal(vol.cpu().numpy(), ref_vol)
    out = torch.empty(vol.shape, dtype=torch.int32, device="cuda")
    n = be.label3d(ctx, vol, out)
    ref, k = O.ccl3d(ref_vol)
    assert n == k and np.array_equal(out.cpu().numpy(), ref)


def test_colour_maps(ctx):
    import torch
    import labeling_b200 as be
    rng = np.random.default_rng(9)
    lab = rng.integers(0, 5000, (123, 77), dtype=np.int32)
    lab[::7] = 0
    d = torch.from_numpy(lab).cuda()
    rgb = torch.empty((123, 77, 3), dtype=torch.uint8, device="cuda")
    be.labels_to_rgb(ctx, d, rgb, seed=5)
    want = colour_ref(lab, 5)
    assert np.array_equal(rgb.cpu().numpy(), want)
    assert (want[lab == 0] == 0).all() and len({tuple(c) for c in want[lab > 0][:500]}) > 400
    vol = rng.integers(0, 300, (9, 40, 70), dtype=np.int32)
    dv = torch.from_numpy(vol).cuda()
    planes = torch.empty((70, 9, 40, 3), dtype=torch.uint8, device="cuda")
    be.volume_to_rgb_planes(ctx, dv, planes, seed=5)
    assert np.array_equal(planes.cpu().numpy(), np.transpose(colour_ref(vol, 5), (2, 0, 1, 3)))


def test_bad_arguments_are_rejected(ctx):
    import torch
    import labeling_b200 as be
    img = torch.zeros((8, 8, 2), dtype=torch.uint8, device="cuda")   # two channels: not supported
    out = torch.empty((8, 8), dtype=torch.uint8, device="cuda")
    with pytest.raises(be.BEError):
        be.to_gray(ctx, img, out)
