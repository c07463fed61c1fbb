"""The `labeling` command line (the reference demo's flags, main.cpp:399-447)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "labeling_b200", "labeling")


def run(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=120).stdout


def test_help_lists_gpu_algorithms():
    out = run("-h")
    assert "bleq" in out and "lbeq" in out and "-3" in out


def test_rejects_unknown_key_and_cpu_modes():
    assert "unknown key -x" in run("-x")
    assert "doesn't support" in run("-a", "bleq", "-u", "-i", "nothing.pgm")
    assert "doesn't support" in run("-a", "bleq", "-i", "nothing.pgm")   # CPU slot is empty
    assert "No labeling algorithm" in run("-a", "nope", "-g", "-i", "x.pgm")


def _write_pgm(path, img):
    with open(path, "wb") as f:
        f.write(b"P5\n%d %d\n255\n" % (img.shape[1], img.shape[0]))
        f.write(img.tobytes())


@pytest.mark.gpu
def test_cli_labels_2d_dir_and_3d_volume(tmp_path):
    from labeling_b200 import workloads as W
    src = tmp_path / "in"
    src.mkdir()
    for i in range(3):
        _write_pgm(str(src / f"im{i}.pgm"), W.bernoulli((100 + i, 130), 0.5, i))
    out = tmp_path / "out"
    out.mkdir()
    txt = run("-a", "bleq", "-g", "-i", str(src), "-o", str(out), "-l", "3")
    assert "Avg processing time" in txt, txt
    assert sorted(os.listdir(out)) == ["im0.pgm.ppm", "im1.pgm.ppm", "im2.pgm.ppm"]
    vol = W.bernoulli((20, 30, 40), 0.2, 5)
    np.save(str(tmp_path / "vol.npy"), vol)
    out3 = tmp_path / "out3"
    out3.mkdir()
    txt = run("-a", "bleq", "-3", "-g", "-i", str(tmp_path / "vol.npy"), "-o", str(out3))
    assert "Processing time" in txt, txt
    assert len(os.listdir(out3)) == 40
    assert "Only default coherence" in run("-a", "bleq", "-3", "-g", "-c", "8", "-i", str(tmp_path / "vol.npy"))
    # 4-connectivity is refused by block equivalence, as in the reference
    assert "4-connectivity" in run("-a", "bleq", "-g", "-c", "4", "-i", str(src / "im0.pgm"))
