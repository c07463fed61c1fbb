"""Generates the golden fixtures of tests/golden/ by running the reference's own code.

The reference's kernels (Labeling2015/src/LabelingAlgs.cl) and Grana labeler
(Labeling2015/src/cvlabeling_imagelab.cpp) are compiled from the reference tree by oracle/Makefile
(`make -C oracle ref`) into oracle/_ref/; this script drives them on small seeded inputs and stores
inputs and outputs as .npz files.  It needs the reference sources only when it runs; the fixtures
it writes are what the tests read.

    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402


def cases_2d(rng):
    out = []
    shapes = [(1, 1), (1, 17), (19, 1), (2, 2), (3, 3), (4, 4), (7, 5), (31, 33), (32, 32),
              (33, 31), (63, 65), (64, 256), (65, 257), (97, 130), (128, 300), (200, 199)]
    for i, (h, w) in enumerate(shapes):
        p = [0.1, 0.3, 0.5, 0.7, 0.9][i % 5]
        img = ((rng.random((h, w)) < p) * 255).astype(np.uint8)
        out.append((f"bern_{h}x{w}_p{p}", img))
    # a checkerboard (every pixel its own 4-component, one 8-component), all-zero, all-one,
    # single corner pixels, and a grey-level image for the threshold
    cb = ((np.indices((40, 40)).sum(0) % 2) * 255).astype(np.uint8)
    out.append(("checker_40", cb))
    out.append(("zeros_20x30", np.zeros((20, 30), np.uint8)))
    out.append(("ones_21x29", np.full((21, 29), 255, np.uint8)))
    px = np.zeros((10, 12), np.uint8); px[0, 0] = 255; px[9, 11] = 255; px[0, 11] = 255
    out.append(("corners_10x12", px))
    dots = np.zeros((24, 24), np.uint8); dots[::2, ::2] = 255
    out.append(("dots_24", dots))
    grey = rng.integers(0, 256, (50, 70)).astype(np.uint8)
    out.append(("grey_50x70", grey))
    return out


def cases_3d(rng):
    out = []
    shapes = [(1, 1, 1), (2, 2, 2), (3, 4, 5), (8, 8, 8), (5, 9, 17), (12, 10, 33), (17, 16, 15)]
    for i, (a, b, c) in enumerate(shapes):
        p = [0.05, 0.1, 0.2, 0.3, 0.5][i % 5]
        vol = ((rng.random((a, b, c)) < p) * 255).astype(np.uint8)
        out.append((f"bern3_{a}x{b}x{c}_p{p}", vol))
    d = np.zeros((6, 6, 6), np.uint8); d[::2, ::2, ::2] = 255
    out.append(("dots3_6", d))
    return out


def main():
    if O.ref_lib() is None or O.grana_lib() is None:
        raise SystemExit("build the reference oracle first: make -C oracle ref")
    rng = np.random.default_rng(20161)
    data = {}
    for name, img in cases_2d(rng):
        thr = 100 if name.startswith("grey") else 0
        raw = O.ref_be2d_raw(img, thr)                   # reference LBEQ2_* label values
        can, k = O.canon(raw)
        g, kg = O.ref_grana(img, thr)                    # reference Grana labels + numLabels
        assert O.canon(g.astype(np.uint32))[1] == k == kg, name
        d4 = O.ref_distr2d_raw(img, thr, 2)              # reference -a lbeq -g (COH_DEFAULT)
        d8 = O.ref_distr2d_raw(img, thr, 1)              # reference -a lbeq -g -c 8
        re = O.ref_runeq2d_raw(img, thr)                 # reference -a runeq -g (RE* kernels)
        data[f"2d/{name}/img"] = img
        data[f"2d/{name}/thr"] = np.array(thr)
        data[f"2d/{name}/raw"] = raw
        data[f"2d/{name}/canon"] = can
        data[f"2d/{name}/k"] = np.array(k)
        data[f"2d/{name}/grana"] = g
        data[f"2d/{name}/distr4"] = d4
        data[f"2d/{name}/distr8"] = d8
        data[f"2d/{name}/runeq"] = re
    for name, vol in cases_3d(rng):
        raw = O.ref_be3d_raw(vol, 0)                     # reference BLEQ3D_* label values
        can, k = O.canon(raw)
        lb3 = O.ref_lbeq3d_raw(vol, 0)                   # reference -a lbeq -3 -g
        data[f"3d/{name}/img"] = vol
        data[f"3d/{name}/raw"] = raw
        data[f"3d/{name}/canon"] = can
        data[f"3d/{name}/k"] = np.array(k)
        data[f"3d/{name}/lbeq"] = lb3
    path = os.path.join(HERE, "be_golden.npz")
    np.savez_compressed(path, **data)
    print(f"wrote {path}: {len(data)} arrays, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
