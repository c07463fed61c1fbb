"""ctypes access to the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
bench.py import this module; the product path (``labeling_b200``) never does.

* ``liboracle.so`` -- the C restatement of the reference BE path (``be_oracle.c``).
* ``_ref/libref_be.so`` -- the reference's own ``LabelingAlgs.cl`` kernels compiled as C++ and run
  serially with the reference's host flow (``ref_driver.cpp``); present when the reference sources
  were available at build time.
* ``_ref/libref_grana.so`` -- the reference's vendored Grana labeler (``ref_grana.cpp``).
* ``_ref/libref_cpu.so`` -- the reference's OpenMP CPU labelers (``ref_cpu.cpp``).
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64 = ctypes.c_int64
_long = ctypes.c_long

_libs: dict = {}


def _load(name: str) -> Optional[ctypes.CDLL]:
    if name in _libs:
        return _libs[name]
    path = os.path.join(HERE, name)
    lib = ctypes.CDLL(path) if os.path.exists(path) else None
    _libs[name] = lib
    return lib


def lib() -> ctypes.CDLL:
    l = _load("liboracle.so")
    if l is None:
        raise RuntimeError("oracle/liboracle.so is not built (run `make -C oracle`)")
    l.orc_be2d_raw.argtypes = [_u8p, _i64, _i64, _i64, ctypes.c_int, _u32p]
    l.orc_be3d_raw.argtypes = [_u8p, _i64, _i64, _i64, ctypes.c_int, _u32p]
    l.orc_lbeq2d_raw.argtypes = [_u8p, _i64, _i64, _i64, ctypes.c_int, ctypes.c_int, _u32p]
    l.orc_lbeq3d_raw.argtypes = [_u8p, _i64, _i64, _i64, ctypes.c_int, _u32p]
    l.orc_canon.argtypes = [_u32p, _i64, _i32p]
    l.orc_canon.restype = _i64
    l.orc_ccl2d.argtypes = [_u8p, _i64, _i64, _i64, ctypes.c_int, ctypes.c_int, _i32p]
    l.orc_ccl2d.restype = _i64
    l.orc_ccl3d.argtypes = [_u8p, _i64, _i64, _i64, ctypes.c_int, ctypes.c_int, _i32p]
    l.orc_ccl3d.restype = _i64
    return l


def ref_lib() -> Optional[ctypes.CDLL]:
    l = _load(os.path.join("_ref", "libref_be.so"))
    if l is not None:
        l.ref_lbeq2_raw.argtypes = [_u8p, _long, _long, _long, ctypes.c_int, _u32p]
        l.ref_bleq3d_raw.argtypes = [_u8p, _long, _long, _long, ctypes.c_int, _u32p]
        l.ref_distr2d_raw.argtypes = [_u8p, _long, _long, _long, ctypes.c_int, ctypes.c_int, _u32p]
        l.ref_lbeq3d_raw.argtypes = [_u8p, _long, _long, _long, ctypes.c_int, _u32p]
        l.ref_bleq3d_timed.argtypes = [_u8p, _long, _long, _long, ctypes.c_int, _u32p,
                                       ctypes.POINTER(ctypes.c_double)]
        l.ref_runeq2d_raw.argtypes = [_u8p, _long, _long, _long, ctypes.c_int, _u32p]
        l.ref_set_threads.argtypes = [ctypes.c_int]
        l.ref_set_threads.restype = ctypes.c_int
    return l


def grana_lib() -> Optional[ctypes.CDLL]:
    l = _load(os.path.join("_ref", "libref_grana.so"))
    if l is not None:
        l.ref_grana.argtypes = [_u8p, _long, _long, _long, ctypes.c_int, _i32p,
                                ctypes.POINTER(ctypes.c_int)]
    return l


def cpu_lib() -> Optional[ctypes.CDLL]:
    """The reference's OpenMP CPU labelers (LabelingAlgs.cpp), compiled by `make -C oracle ref`."""
    l = _load(os.path.join("_ref", "libref_cpu.so"))
    if l is not None:
        l.ref_cpu_label2d.argtypes = [ctypes.c_char_p, _u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, _i32p, ctypes.POINTER(ctypes.c_double)]
        l.ref_cpu_max_threads.restype = ctypes.c_int
    return l


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _u8(img: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(img, dtype=np.uint8)


def canon(raw: np.ndarray) -> Tuple[np.ndarray, int]:
    """Canonical relabeling of any label map (0 = background)."""
    raw = np.ascontiguousarray(raw).astype(np.uint32, copy=False)
    out = np.empty(raw.shape, np.int32)
    k = lib().orc_canon(_p(raw, _u32p), raw.size, _p(out, _i32p))
    if k < 0:
        raise MemoryError("orc_canon failed")
    return out, int(k)


def be2d_raw(img: np.ndarray, thr: int = 0) -> np.ndarray:
    img = _u8(img)
    out = np.empty(img.shape, np.uint32)
    rc = lib().orc_be2d_raw(_p(img, _u8p), img.shape[0], img.shape[1], img.shape[1], thr,
                            _p(out, _u32p))
    if rc:
        raise RuntimeError(f"orc_be2d_raw rc={rc}")
    return out


def be3d_raw(vol: np.ndarray, thr: int = 0) -> np.ndarray:
    vol = _u8(vol)
    out = np.empty(vol.shape, np.uint32)
    rc = lib().orc_be3d_raw(_p(vol, _u8p), *vol.shape, thr, _p(out, _u32p))
    if rc:
        raise RuntimeError(f"orc_be3d_raw rc={rc}")
    return out


def lbeq2d_raw(img: np.ndarray, thr: int = 0, conn8: bool = False) -> np.ndarray:
    img = _u8(img)
    out = np.empty(img.shape, np.uint32)
    rc = lib().orc_lbeq2d_raw(_p(img, _u8p), img.shape[0], img.shape[1], img.shape[1], thr,
                              int(conn8), _p(out, _u32p))
    if rc:
        raise RuntimeError(f"orc_lbeq2d_raw rc={rc}")
    return out


def lbeq3d_raw(vol: np.ndarray, thr: int = 0) -> np.ndarray:
    vol = _u8(vol)
    out = np.empty(vol.shape, np.uint32)
    rc = lib().orc_lbeq3d_raw(_p(vol, _u8p), *vol.shape, thr, _p(out, _u32p))
    if rc:
        raise RuntimeError(f"orc_lbeq3d_raw rc={rc}")
    return out


def be2d(img: np.ndarray, thr: int = 0) -> Tuple[np.ndarray, int]:
    """Canonical labels of the reference BE restatement (2D, 8-connectivity)."""
    return canon(be2d_raw(img, thr))


def be3d(vol: np.ndarray, thr: int = 0) -> Tuple[np.ndarray, int]:
    """Canonical labels of the reference BE restatement (3D, 26-connectivity)."""
    return canon(be3d_raw(vol, thr))


def ccl2d(img: np.ndarray, thr: int = 0, conn8: bool = True) -> Tuple[np.ndarray, int]:
    """Canonical labels from the independent union-find oracle (fast)."""
    img = _u8(img)
    out = np.empty(img.shape, np.int32)
    k = lib().orc_ccl2d(_p(img, _u8p), img.shape[0], img.shape[1], img.shape[1], thr, int(conn8),
                        _p(out, _i32p))
    if k < 0:
        raise RuntimeError(f"orc_ccl2d rc={k}")
    return out, int(k)


def ccl3d(vol: np.ndarray, thr: int = 0, conn26: bool = True) -> Tuple[np.ndarray, int]:
    vol = _u8(vol)
    out = np.empty(vol.shape, np.int32)
    k = lib().orc_ccl3d(_p(vol, _u8p), *vol.shape, thr, int(conn26), _p(out, _i32p))
    if k < 0:
        raise RuntimeError(f"orc_ccl3d rc={k}")
    return out, int(k)


# --- the reference's own code, compiled from its sources (present only when built) -----------

def ref_be2d_raw(img: np.ndarray, thr: int = 0) -> np.ndarray:
    l = ref_lib()
    if l is None:
        raise RuntimeError("oracle/_ref/libref_be.so is not built")
    img = _u8(img)
    out = np.empty(img.shape, np.uint32)
    if l.ref_lbeq2_raw(_p(img, _u8p), img.shape[0], img.shape[1], img.shape[1], thr,
                       _p(out, _u32p)):
        raise RuntimeError("ref_lbeq2_raw failed")
    return out


def ref_be3d_raw(vol: np.ndarray, thr: int = 0) -> np.ndarray:
    l = ref_lib()
    if l is None:
        raise RuntimeError("oracle/_ref/libref_be.so is not built")
    vol = _u8(vol)
    out = np.empty(vol.shape, np.uint32)
    if l.ref_bleq3d_raw(_p(vol, _u8p), *vol.shape, thr, _p(out, _u32p)):
        raise RuntimeError("ref_bleq3d_raw failed")
    return out


def ref_be3d_timed(vol: np.ndarray, thr: int = 0, threads: int = 1) -> Tuple[np.ndarray, float]:
    """The reference's 3D block-equivalence kernels (TOCLBlockEquivalence3D) run on the host with
    `threads` work-item threads (0 = all); returns the raw labels and the time of the kernel
    sequence in microseconds."""
    l = ref_lib()
    if l is None:
        raise RuntimeError("oracle/_ref/libref_be.so is not built")
    vol = _u8(vol)
    out = np.empty(vol.shape, np.uint32)
    us = ctypes.c_double(0.0)
    l.ref_set_threads(threads)
    try:
        if l.ref_bleq3d_timed(_p(vol, _u8p), *vol.shape, thr, _p(out, _u32p), ctypes.byref(us)):
            raise RuntimeError("ref_bleq3d_timed failed")
    finally:
        l.ref_set_threads(1)
    return out, float(us.value)


def ref_distr2d_raw(img: np.ndarray, thr: int = 0, coh: int = 2) -> np.ndarray:
    l = ref_lib()
    if l is None:
        raise RuntimeError("oracle/_ref/libref_be.so is not built")
    img = _u8(img)
    out = np.empty(img.shape, np.uint32)
    if l.ref_distr2d_raw(_p(img, _u8p), img.shape[0], img.shape[1], img.shape[1], thr, coh,
                         _p(out, _u32p)):
        raise RuntimeError("ref_distr2d_raw failed")
    return out


def ref_runeq2d_raw(img: np.ndarray, thr: int = 0) -> np.ndarray:
    """The reference's GPU run-equivalence kernels (RE*, LabelingAlgs.cl:325-616) with its host
    flow (TOCLRunEquivLabeling, LabelingAlgs.cpp:1090-1268), serially on the host."""
    l = ref_lib()
    if l is None:
        raise RuntimeError("oracle/_ref/libref_be.so is not built")
    img = _u8(img)
    out = np.empty(img.shape, np.uint32)
    if l.ref_runeq2d_raw(_p(img, _u8p), img.shape[0], img.shape[1], img.shape[1], thr, _p(out, _u32p)):
        raise RuntimeError("ref_runeq2d_raw failed")
    return out


def ref_lbeq3d_raw(vol: np.ndarray, thr: int = 0) -> np.ndarray:
    l = ref_lib()
    if l is None:
        raise RuntimeError("oracle/_ref/libref_be.so is not built")
    vol = _u8(vol)
    out = np.empty(vol.shape, np.uint32)
    if l.ref_lbeq3d_raw(_p(vol, _u8p), *vol.shape, thr, _p(out, _u32p)):
        raise RuntimeError("ref_lbeq3d_raw failed")
    return out


def ref_cpu_label2d(img: np.ndarray, alg: str = "bleq", thr: int = 0, threads: int = 0,
                    coh: int = 1) -> Tuple[np.ndarray, float]:
    """One of the reference's CPU labelers ("bleq" = TLabelEquivalenceX2, "lbeq" =
    TLabelDistribution, "runeq" = TRunEqivLabeling, "gr-block" = Grana), run through
    ILabeling::Label (LabelingTools.cpp:19-36) with `threads` OpenMP threads (0 = all).  Returns
    the reference's raw labels and its own stopwatch time in microseconds.  The reference CPU
    block labeler mis-connects blocks at an even-width right border (RemoveBorderBlocks compares
    pixel coordinates with the image size, LabelingAlgs.cpp:366-374, so px == w - 1 never holds
    and the x + 2 probes wrap into the next row), and TLabelDistribution leaves a foreground
    pixel at (0, 0) unlabeled; both are the reference's behaviour, kept here as it is."""
    l = cpu_lib()
    if l is None:
        raise RuntimeError("oracle/_ref/libref_cpu.so is not built")
    img = _u8(img)
    out = np.empty(img.shape, np.int32)
    us = ctypes.c_double(0.0)
    rc = l.ref_cpu_label2d(alg.encode(), _p(img, _u8p), img.shape[0], img.shape[1], thr, threads, coh,
                           _p(out, _i32p), ctypes.byref(us))
    if rc:
        raise RuntimeError(f"ref_cpu_label2d({alg}) failed: {rc}")
    return out, float(us.value)


def ref_cpu_bleq(img: np.ndarray, thr: int = 0, threads: int = 0, pad: bool = True) -> Tuple[np.ndarray, float]:
    """The reference's CPU block-equivalence labeler (the `bleq` CPU slot, main.cpp:122-126).

    With `pad` (the default) the image gets one background row and column at its end before the
    call and the labels are cropped back: that keeps the labeler's right- and bottom-border
    probes inside background, and its labels are then exact (the padding is outside the
    reference's stopwatch, which covers DoLabel only)."""
    img = _u8(img)
    if not pad:
        return ref_cpu_label2d(img, "bleq", thr, threads, 1)
    h, w = img.shape
    padded = np.zeros((h + 1, w + 1), np.uint8)
    padded[:h, :w] = img
    lab, us = ref_cpu_label2d(padded, "bleq", thr, threads, 1)
    return np.ascontiguousarray(lab[:h, :w]), us


def ref_grana(img: np.ndarray, thr: int = 0) -> Tuple[np.ndarray, int]:
    """The reference's Grana labeler; returns its own labels and its numLabels."""
    l = grana_lib()
    if l is None:
        raise RuntimeError("oracle/_ref/libref_grana.so is not built")
    img = _u8(img)
    out = np.empty(img.shape, np.int32)
    n = ctypes.c_int(0)
    if l.ref_grana(_p(img, _u8p), img.shape[0], img.shape[1], img.shape[1], thr, _p(out, _i32p),
                   ctypes.byref(n)):
        raise RuntimeError("ref_grana failed")
    return out, int(n.value)
