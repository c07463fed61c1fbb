"""The numpy restatement of the reference's RGB2Gray used by the device ingest tests, pinned to
OpenCV itself on the CPU (LabelingTools.cpp:39-49: cv::cvtColor(COLOR_RGB2GRAY), then
cv::threshold with the value 8 and THRESH_BINARY).

The reference builds against OpenCV 3.0.0, whose 8-bit RGB -> gray uses 14-bit weights
(4899, 9617, 1868); the cv2 in this image is OpenCV 4, whose weights are 15-bit (9798, 19235,
3735).  The OpenCV 4 form is pinned here bit for bit against cv2; the 3.0.0 form, the device
default, is the same rounding one bit coarser and stays within one gray level of it."""
import numpy as np
import pytest

from test_gpu_io import gray_ref


@pytest.mark.parametrize("channels", [1, 3])
def test_gray_restatement_equals_opencv(channels):
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(5 + channels)
    shape = (257, 383, 3) if channels == 3 else (257, 383)
    img = rng.integers(0, 256, shape, dtype=np.uint8)
    gray = cv2.cvtColor(img, cv2.COLOR_RGB2GRAY) if channels == 3 else img
    _, want = cv2.threshold(gray, 8, 255, cv2.THRESH_BINARY)
    assert cv2.THRESH_OTSU == 8   # the value the reference passes as its threshold
    assert np.array_equal(gray_ref(img, False, channels == 3, opencv4=True), gray)
    assert np.array_equal(gray_ref(img, True, channels == 3, opencv4=True), want)
    d = np.abs(gray_ref(img, False, channels == 3).astype(np.int32) - gray.astype(np.int32))
    assert d.max() <= 1


def test_gray_weights_are_the_published_fractions():
    """Both fixed-point forms round 0.299 / 0.587 / 0.114 to their scale, with the weights
    summing to the scale (white stays 255)."""
    for w, scale in (((4899, 9617, 1868), 1 << 14), ((9798, 19235, 3735), 1 << 15)):
        assert sum(w) == scale
        for wi, f in zip(w, (0.299, 0.587, 0.114)):
            assert abs(wi - f * scale) <= 1
        assert (255 * sum(w) + scale // 2) // scale == 255
