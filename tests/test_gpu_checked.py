"""The bounds-checked build (-DBE_BOUNDS_CHECK, libbe_b200_check.so) on the union-find pipelines:
every guarded index of the tile, merge, scan/node and write kernels is checked and a failure is
recorded (and the access skipped) instead of touching memory out of bounds.  A child process loads
that build (the package binds one library per process, chosen by BE_B200_LIB), labels 2D images
and 3D volumes chosen to reach the kernels' edge paths -- shapes that end inside a tile, pitched
views, the deepest in-tile chains (spiral, serpentine), dense and sparse noise -- and checks that
no index check failed and that every label map equals the oracle's."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
sys.path.insert(0, ROOT)
import numpy as np, torch
import labeling_b200 as be
from labeling_b200 import workloads as W
from oracle import oracle as O
ctx = be.Context(0)
bad = []
cases2 = [("bern0.5", W.bernoulli((1000, 1500), 0.5, seed=3)),
          ("bern0.1", W.bernoulli((777, 1031), 0.1, seed=4)),
          ("bern0.9", W.bernoulli((513, 2049), 0.9, seed=5)),
          ("spiral", W.spiral(1024, 1024)),
          ("serpentine", W.serpentine(1030, 770)),
          ("disks", W.disks(1200, 900, 60, 4, 80, 0.05, seed=6))]
for name, img in cases2:
    d_in = torch.from_numpy(img).cuda()
    d_out = torch.full(img.shape, -1, dtype=torch.int32, device="cuda")
    n = be.label2d(ctx, d_in, d_out)
    site, val = ctx.check_status(2)
    ref, k = O.ccl2d(img)
    if site or n != k or not np.array_equal(d_out.cpu().numpy(), ref):
        bad.append((name, site, val, n, k))
# a pitched view (rows of 1536 bytes, 1000 columns used)
base = W.bernoulli((600, 1536), 0.45, seed=7)
view = torch.from_numpy(base).cuda()[:, 17:1017]
out = torch.full((600, 1000), -1, dtype=torch.int32, device="cuda")
n = be.label2d(ctx, view, out)
site, val = ctx.check_status(2)
ref, k = O.ccl2d(np.ascontiguousarray(base[:, 17:1017]))
if site or n != k or not np.array_equal(out.cpu().numpy(), ref):
    bad.append(("pitched", site, val, n, k))
cases3 = [("bern0.3", W.bernoulli((70, 90, 130), 0.3, seed=8)),
          ("bern0.1", W.bernoulli((33, 65, 97), 0.1, seed=9)),
          ("bern0.5", W.bernoulli((48, 64, 64), 0.5, seed=10)),
          ("grf", W.grf((80, 80, 80), 4.0, 60, 11, device="cuda"))]
for name, vol in cases3:
    v_in = torch.from_numpy(vol).cuda()
    v_out = torch.full(vol.shape, -1, dtype=torch.int32, device="cuda")
    n = be.label3d(ctx, v_in, v_out)
    site, val = ctx.check_status(3)
    ref, k = O.ccl3d(vol)
    if site or n != k or not np.array_equal(v_out.cpu().numpy(), ref):
        bad.append((name, site, val, n, k))
ctx.close()
print("RESULT", json.dumps(bad))
""".replace("ROOT", repr(ROOT))


def _checked_lib() -> str:
    from labeling_b200 import build
    if not os.path.exists(build.LIB_CHECK):
        build.build(checked=True)
    return build.LIB_CHECK


def test_checked_build_no_index_failures():
    lib = _checked_lib()
    env = dict(os.environ, BE_B200_LIB=lib)
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("RESULT ")]
    assert line, r.stdout[-2000:] + r.stderr[-2000:]
    assert json.loads(line[0][7:]) == []
