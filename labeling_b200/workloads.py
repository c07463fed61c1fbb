"""Seeded synthetic inputs for the labeling workloads (numpy; optional torch for large volumes).

Image families of the benchmark configurations:
  * ``bernoulli``   i.i.d. foreground with probability p (0/255 pixels);
  * ``disks``       filled disks (centres uniform, radius U[rmin, rmax]) over Bernoulli noise;
  * ``serpentine``  one 1-pixel-wide path: full rows on every second line, joined at
                    alternating ends (a single component whose propagation distance is ~N/2);
  * ``spiral``      one 1-pixel-wide square spiral with 1-pixel gaps between its arms;
  * ``grf``         Gaussian random field (white noise smoothed by a Gaussian of std sigma),
                    thresholded at a percentile (3D volumes);
  * uneven batches of images whose sides are log-uniform.
All generators take an explicit seed; the same seed gives the same array.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np


def bernoulli(shape, p: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return ((rng.random(shape, dtype=np.float32) < p) * 255).astype(np.uint8)


def disks(h: int, w: int, n: int = 2000, rmin: float = 4, rmax: float = 200, p_noise: float = 0.05,
          seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    img = (rng.random((h, w), dtype=np.float32) < p_noise)
    cy = rng.uniform(0, h, n)
    cx = rng.uniform(0, w, n)
    rr = rng.uniform(rmin, rmax, n)
    for y, x, r in zip(cy, cx, rr):
        y0, y1 = max(0, int(y - r)), min(h, int(y + r) + 1)
        x0, x1 = max(0, int(x - r)), min(w, int(x + r) + 1)
        if y0 >= y1 or x0 >= x1:
            continue
        yy = np.arange(y0, y1, dtype=np.float32)[:, None] - y
        xx = np.arange(x0, x1, dtype=np.float32)[None, :] - x
        img[y0:y1, x0:x1] |= (yy * yy + xx * xx) <= r * r
    return (img * 255).astype(np.uint8)


def serpentine(h: int, w: int) -> np.ndarray:
    img = np.zeros((h, w), np.uint8)
    img[0::2, :] = 255
    for y in range(1, h, 2):
        x = w - 1 if (y // 2) % 2 == 0 else 0
        img[y, x] = 255
    return img


def spiral(h: int, w: int) -> np.ndarray:
    """Clockwise square spiral from the top-left corner inward, arms 2 pixels apart."""
    img = np.zeros((h, w), np.uint8)
    top, left, bottom, right = 0, 0, h - 1, w - 1
    while top <= bottom and left <= right:
        img[top, left:right + 1] = 255                       # right along the top
        if top + 1 > bottom:
            break
        img[top:bottom + 1, right] = 255                     # down the right side
        if right - 1 < left:
            break
        img[bottom, left:right + 1] = 255                    # left along the bottom
        if bottom - 2 < top + 2:
            break
        img[top + 2:bottom + 1, left] = 255                  # up the left side, stop 2 short
        if left + 2 > right - 2:
            break
        img[top + 2, left:left + 3] = 255                    # step inward to the next arm
        top, left, bottom, right = top + 2, left + 2, bottom - 2, right - 2
    return img


def grf(shape, sigma: float, percentile: float, seed: int, device: str = "cpu") -> np.ndarray:
    """Gaussian random field thresholded so that (100 - percentile)% of voxels are foreground."""
    try:
        import torch
    except ImportError:  # pragma: no cover
        torch = None
    if torch is not None and (device != "cpu" or np.prod(shape) > (1 << 22)):
        dev = device if device != "cpu" or not torch.cuda.is_available() else "cuda"
        g = torch.Generator(device="cpu").manual_seed(seed)
        noise = torch.randn(tuple(shape), generator=g, dtype=torch.float32).to(dev)
        f = torch.fft.rfftn(noise)
        freqs = [torch.fft.fftfreq(n, device=dev) for n in shape[:-1]] + [torch.fft.rfftfreq(shape[-1], device=dev)]
        k2 = sum(fr.reshape([-1 if i == j else 1 for j in range(len(shape))]) ** 2
                 for i, fr in enumerate(freqs))
        field = torch.fft.irfftn(f * torch.exp(-2 * (math.pi ** 2) * (sigma ** 2) * k2), s=tuple(shape))
        flat = field.flatten()
        k = int(round(flat.numel() * percentile / 100.0))
        k = min(max(k, 1), flat.numel())
        thr = flat.kthvalue(k).values
        return ((field > thr).to(torch.uint8) * 255).cpu().numpy()
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    field = gaussian_filter(rng.standard_normal(shape).astype(np.float32), sigma, mode="wrap")
    thr = np.percentile(field, percentile)
    return ((field > thr) * 255).astype(np.uint8)


def log_uniform_sides(n: int, lo: int, hi: int, seed: int, dims: int = 2) -> List[Tuple[int, ...]]:
    rng = np.random.default_rng(seed)
    v = np.exp(rng.uniform(math.log(lo), math.log(hi), (n, dims)))
    return [tuple(int(round(x)) for x in row) for row in v]


def family_8192(name: str, seed: int = 0, side: int = 8192) -> np.ndarray:
    """The 8192^2 families: bern0.1 / bern0.4 / bern0.6 / bern0.9 / disks / serpentine / spiral."""
    if name.startswith("bern"):
        return bernoulli((side, side), float(name[4:]), seed)
    if name == "disks":
        return disks(side, side, 2000, 4, 200, 0.05, seed)
    if name == "serpentine":
        return serpentine(side, side)
    if name == "spiral":
        return spiral(side, side)
    raise ValueError(name)


FAMILIES_8192 = ["bern0.1", "bern0.4", "bern0.6", "bern0.9", "disks", "serpentine", "spiral"]
