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
    return l


def grana_lib() -> Optional[ctypes.CDLL]:
    l = _load(os.path.join("_ref", "libref_grana.so"))
    if l is not None:
        l.ref_grana.argtypes = [_u8p, _long, _long, _long, ctypes.c_int, _i32p,
                                ctypes.POINTER(ctypes.c_int)]
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


def ref_lbeq3d_raw(vol: np.ndarray, thr: int = 0) -> np.ndarray:
    l = ref_lib()
    if l is None:
        raise RuntimeError("oracle/_ref/libref_be.so is not built")
    vol = _u8(vol)
    out = np.empty(vol.shape, np.uint32)
    if l.ref_lbeq3d_raw(_p(vol, _u8p), *vol.shape, thr, _p(out, _u32p)):
        raise RuntimeError("ref_lbeq3d_raw failed")
    return out


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
