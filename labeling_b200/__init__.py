"""B200-native Block-Equivalence connected-component labeling.

Python access to ``libbe_b200.so`` (the CUDA kernels behind the C ABI of ``include/be.h``)
through ctypes, plus a mirror of the reference's labeler interface:

* :class:`Context` -- one CUDA context's labeler state (``be_create`` / ``be_destroy``).
* :func:`label2d` / :func:`label3d` -- device buffers (torch CUDA tensors or raw pointers) in,
  int32 canonical labels out (``be_label2d`` / ``be_label3d``).
* :func:`label2d_host` / :func:`label3d_host` -- numpy in, numpy out.
* :class:`Labeling` / :class:`Labeling3D` -- ``Label(pixels, threads, coh) -> (labels, µs)``, the
  shape of ``ILabeling::Label`` (Labeling2015/src/LabelingTools.hpp:58-73), selected through
  :func:`make_labeler` with the reference's algorithm names (``bleq``, ``lbeq``).

There is no CPU fallback: if the library is missing or no GPU is present, every call raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# BE_B200_LIB selects another build of the same ABI (e.g. the bounds-checked
# libbe_b200_check.so made by `python -m labeling_b200.build --checked`).
LIB_PATH = os.environ.get("BE_B200_LIB") or os.path.join(_HERE, "libbe_b200.so")

BE_OK = 0
STATUS = {0: "BE_OK", 1: "BE_ERR_INVALID", 2: "BE_ERR_OOM", 3: "BE_ERR_NO_CONVERGENCE",
          4: "BE_ERR_CUDA", 5: "BE_ERR_TIMEOUT", 6: "BE_ERR_BUSY", 7: "BE_ERR_CANCELLED",
          8: "BE_ERR_TOO_LARGE"}
ALGO_AUTO, ALGO_UF, ALGO_ITER, ALGO_PIXEL, ALGO_RUNS = 0, 1, 2, 3, 4
COH_4, COH_8, COH_DEFAULT = 0, 1, 2

_lib = None
BATCH_ONE_CTA_PER_TILE = 0x100


class BEImage(ctypes.Structure):
    """``be_image`` of include/be.h: one image (dims = (rows, cols, 0)) or volume of a batch."""
    _fields_ = [("in_", ctypes.c_void_p), ("out", ctypes.c_void_p), ("in_pitch", ctypes.c_int64),
                ("out_pitch", ctypes.c_int64), ("dims", ctypes.c_int32 * 3),
                ("threshold", ctypes.c_int32)]


class BERequest(ctypes.Structure):
    _fields_ = [("in_", ctypes.c_void_p), ("out", ctypes.c_void_p), ("dims", ctypes.c_int32 * 3),
                ("threshold", ctypes.c_int32), ("flags", ctypes.c_int32)]


class BEResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("n_components", ctypes.c_int64),
                ("latency_us", ctypes.c_double)]


class BEServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("max_device_bytes", ctypes.c_int64),
                ("lanes", ctypes.c_int32), ("max_batch", ctypes.c_int32),
                ("inject_alloc_failure_every", ctypes.c_int32)]


class BEServeStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int64), ("rejected", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("batches", ctypes.c_int64), ("pixels", ctypes.c_int64), ("p50_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double), ("wall_s", ctypes.c_double),
                ("device_bytes_in_use", ctypes.c_int64), ("device_bytes_budget", ctypes.c_int64)]


REQ_DEVICE_BUFFERS = 1


class BEError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """The loaded C-ABI library (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m labeling_b200.build`")
    l = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, c_int = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_int
    p64 = ctypes.POINTER(ctypes.c_int64)
    pdbl = ctypes.POINTER(ctypes.c_double)
    l.be_version.restype = ctypes.c_char_p
    l.be_create.argtypes = [ctypes.POINTER(vp), c_int]
    l.be_destroy.argtypes = [vp]
    l.be_last_error.argtypes = [vp]
    l.be_last_error.restype = ctypes.c_char_p
    l.be_label2d.argtypes = [vp, vp, i64, i32, i32, c_int, c_int, c_int, vp, i64, p64, vp]
    l.be_label3d.argtypes = [vp, vp, i32, i32, i32, c_int, c_int, vp, p64, vp]
    l.be_label2d_host.argtypes = [vp, vp, i64, i32, i32, c_int, c_int, c_int, vp, i64, p64, pdbl]
    l.be_label3d_host.argtypes = [vp, vp, i32, i32, i32, c_int, c_int, vp, p64, pdbl]
    l.be_autotune2d.argtypes = [vp, vp, i64, i32, i32, c_int, vp, i64, ctypes.POINTER(c_int), vp]
    l.be_autotune3d.argtypes = [vp, vp, i32, i32, i32, c_int, vp, ctypes.POINTER(c_int), vp]
    l.be_tune_save.argtypes = [vp, ctypes.c_char_p]
    l.be_tune_load.argtypes = [vp, ctypes.c_char_p]
    l.be_batch_create.argtypes = [vp, ctypes.POINTER(BEImage), c_int, c_int, ctypes.POINTER(vp)]
    l.be_batch_run.argtypes = [vp, vp]
    l.be_batch_counts.argtypes = [vp, p64, vp]
    l.be_batch_tune.argtypes = [vp, vp, ctypes.POINTER(c_int)]
    l.be_batch_destroy.argtypes = [vp]
    l.be_server_default_config.argtypes = [ctypes.POINTER(BEServerConfig)]
    l.be_server_create.argtypes = [ctypes.POINTER(BEServerConfig), ctypes.POINTER(vp)]
    l.be_server_submit.argtypes = [vp, ctypes.POINTER(BERequest), ctypes.POINTER(ctypes.c_uint64)]
    l.be_server_wait.argtypes = [vp, ctypes.c_uint64, i64, ctypes.POINTER(BEResult)]
    l.be_server_cancel.argtypes = [vp, ctypes.c_uint64]
    l.be_server_stats.argtypes = [vp, ctypes.POINTER(BEServeStats)]
    l.be_server_reset_stats.argtypes = [vp]
    l.be_server_destroy.argtypes = [vp]
    l.be_set_stage_timing.argtypes = [vp, c_int]
    l.be_check_status.argtypes = [vp, c_int, ctypes.POINTER(ctypes.c_uint32)]
    l.be_stage_times.argtypes = [vp, ctypes.POINTER(ctypes.c_float), c_int, ctypes.POINTER(c_int)]
    l.be_to_gray.argtypes = [vp, vp, i64, c_int, i32, i32, c_int, vp, i64, vp]
    l.be_stack_slices.argtypes = [vp, vp, c_int, i32, i32, i32, vp, vp]
    l.be_labels_to_rgb.argtypes = [vp, vp, i64, ctypes.c_uint32, vp, vp]
    l.be_volume_to_rgb_planes.argtypes = [vp, vp, i32, i32, i32, ctypes.c_uint32, vp, vp]
    l.be_slab_merge.argtypes = [i32, i32, i32, vp, vp, vp, vp, p64, vp, vp, vp, i64]
    l.be_slab_relabel.argtypes = [vp, vp, i64, i32, i64, i64, i64, vp, vp, i32, vp]
    l.be_slab_reserve.argtypes = [vp, i64, i64]
    _lib = l
    return l


def version() -> str:
    return lib().be_version().decode()


class Context:
    """Labeler state on one CUDA device; not thread-safe (one per host thread)."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        rc = lib().be_create(ctypes.byref(self._h), int(device))
        if rc:
            raise BEError(rc, f"be_create(device={device}) failed")
        self.device = device

    @property
    def handle(self) -> ctypes.c_void_p:
        if not self._h:
            raise RuntimeError("context is closed")
        return self._h

    def check(self, rc: int) -> None:
        if rc:
            raise BEError(rc, lib().be_last_error(self._h).decode())

    def check_status(self, dims: int):
        """(site, value) of the first failed index check of the last call (checked builds)."""
        out = (ctypes.c_uint32 * 3)()
        self.check(lib().be_check_status(self.handle, dims, out))
        return int(out[0]), int(out[1]) | (int(out[2]) << 32)

    def tune_save(self, path: str) -> None:
        self.check(lib().be_tune_save(self.handle, path.encode()))

    def tune_load(self, path: str) -> None:
        self.check(lib().be_tune_load(self.handle, path.encode()))

    def set_stage_timing(self, on: bool) -> None:
        self.check(lib().be_set_stage_timing(self.handle, int(on)))

    def stage_times(self):
        """Device ms of each launch of the last plain call (stage timing must be on)."""
        ms = (ctypes.c_float * 16)()
        n = ctypes.c_int(0)
        self.check(lib().be_stage_times(self.handle, ms, 16, ctypes.byref(n)))
        return [float(ms[i]) for i in range(n.value)]

    def close(self) -> None:
        if self._h:
            lib().be_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(x) -> int:
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    return int(x)


def _stream(stream) -> Optional[int]:
    if stream is None:
        try:
            import torch
            return int(torch.cuda.current_stream().cuda_stream)
        except Exception:
            return None
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    return int(stream)


def label2d(ctx: Context, img, out, threshold: int = 0, algo: int = ALGO_AUTO,
            coh: int = COH_DEFAULT, want_count: bool = True, stream=None,
            in_pitch: Optional[int] = None, out_pitch: Optional[int] = None,
            rows: Optional[int] = None, cols: Optional[int] = None) -> Optional[int]:
    """Labels a device image.  ``img``: uint8 CUDA tensor [rows, cols] (or a pointer with
    rows/cols/in_pitch); ``out``: int32 CUDA tensor of the same shape.  Returns the component
    count (synchronizing) when ``want_count``."""
    if hasattr(img, "shape"):
        rows, cols = int(img.shape[0]), int(img.shape[1])
        in_pitch = int(img.stride(0)) if in_pitch is None else in_pitch
        out_pitch = int(out.stride(0)) if out_pitch is None else out_pitch
    n = ctypes.c_int64(0)
    ctx.check(lib().be_label2d(ctx.handle, _ptr(img), in_pitch, rows, cols, threshold, coh, algo,
                               _ptr(out), out_pitch, ctypes.byref(n) if want_count else None,
                               _stream(stream)))
    return int(n.value) if want_count else None


def label3d(ctx: Context, vol, out, threshold: int = 0, algo: int = ALGO_AUTO,
            want_count: bool = True, stream=None, dims=None) -> Optional[int]:
    """Labels a dense device volume [d0, d1, d2] (d2 fastest) into int32 ``out``."""
    d0, d1, d2 = (int(s) for s in (vol.shape if dims is None else dims))
    n = ctypes.c_int64(0)
    ctx.check(lib().be_label3d(ctx.handle, _ptr(vol), d0, d1, d2, threshold, algo, _ptr(out),
                               ctypes.byref(n) if want_count else None, _stream(stream)))
    return int(n.value) if want_count else None


# ---- ingest and egress on the device (RGB2Gray, Read3DImage, LabelsToRGB, Write3DLabels) -----

GRAY_BINARIZE, GRAY_OPENCV4 = 1, 2


def to_gray(ctx: Context, img, out, binarize: bool = True, opencv4: bool = False, stream=None) -> None:
    """uint8 CUDA tensor [rows, cols] or [rows, cols, 3] (RGB) -> uint8 [rows, cols]: gray as
    cv::COLOR_RGB2GRAY, then (binarize) the reference's fixed threshold, gray > 8 ? 255 : 0.
    The gray weights are OpenCV 3.0.0's (the reference's OpenCV), or OpenCV 4's with opencv4."""
    channels = int(img.shape[2]) if img.dim() == 3 else 1
    rows, cols = int(img.shape[0]), int(img.shape[1])
    flags = (GRAY_BINARIZE if binarize else 0) | (GRAY_OPENCV4 if opencv4 else 0)
    ctx.check(lib().be_to_gray(ctx.handle, _ptr(img), int(img.stride(0)), channels, rows, cols,
                               flags, _ptr(out), int(out.stride(0)), _stream(stream)))


def stack_slices(ctx: Context, slices, out, stream=None) -> None:
    """Contiguous uint8 CUDA tensor of slices [planes, rows, cols] (or [..., 3] RGB) -> binarized
    volume ``out`` [rows, cols, planes], the slice index fastest (Read3DImage's layout)."""
    channels = int(slices.shape[3]) if slices.dim() == 4 else 1
    planes, rows, cols = (int(x) for x in slices.shape[:3])
    assert slices.is_contiguous() and out.is_contiguous() and tuple(out.shape) == (rows, cols, planes)
    ctx.check(lib().be_stack_slices(ctx.handle, _ptr(slices), channels, rows, cols, planes, _ptr(out),
                                    _stream(stream)))


def labels_to_rgb(ctx: Context, labels, out, seed: int = 0, stream=None) -> None:
    """Contiguous int32 labels (any shape) -> uint8 ``out`` of shape labels.shape + (3,): the
    background black, every label a colour hashed from (label, seed)."""
    assert labels.is_contiguous() and out.is_contiguous() and out.numel() == 3 * labels.numel()
    ctx.check(lib().be_labels_to_rgb(ctx.handle, _ptr(labels), int(labels.numel()), seed & 0xFFFFFFFF,
                                     _ptr(out), _stream(stream)))


def volume_to_rgb_planes(ctx: Context, labels, out, seed: int = 0, stream=None) -> None:
    """int32 label volume [d0, d1, d2] -> uint8 ``out`` [d2, d0, d1, 3]: one colour image per index
    of the last dimension (Write3DLabels's planes)."""
    d0, d1, d2 = (int(x) for x in labels.shape)
    assert labels.is_contiguous() and out.is_contiguous() and tuple(out.shape) == (d2, d0, d1, 3)
    ctx.check(lib().be_volume_to_rgb_planes(ctx.handle, _ptr(labels), d0, d1, d2, seed & 0xFFFFFFFF,
                                            _ptr(out), _stream(stream)))


# ---- slab split of one image (one exchange of border rows; see labeling_b200.slabs) --------

class SlabMerge:
    """Result of :func:`slab_merge`: ``offsets[s]``, ``total`` and, per slab, the ascending local
    labels joined under an earlier piece (``joined_labels[s]``) with their final labels
    (``joined_targets[s]``)."""

    def __init__(self, offsets, total, joined_labels, joined_targets):
        self.offsets = offsets
        self.total = total
        self.joined_labels = joined_labels
        self.joined_targets = joined_targets

    def lut(self, s: int, count: int) -> np.ndarray:
        """Slab s's label map as a dense array (index = local label), for checks on the host."""
        m = np.zeros(count + 1, np.int64)
        loc = np.arange(1, count + 1)
        jl = self.joined_labels[s]
        m[1:] = self.offsets[s] + loc - np.searchsorted(jl, loc, side="left")
        m[jl] = self.joined_targets[s]
        return m


def slab_merge(counts, tops: np.ndarray, bottoms: np.ndarray) -> SlabMerge:
    """Joins slabs labeled on their own (``be_slab_merge``; host only, no GPU).  ``counts``: the
    slabs' component counts; ``tops`` / ``bottoms``: int32 [n_slabs, cols] (2D) or
    [n_slabs, d1, d2] (3D), each slab's first and last row (plane) of local labels."""
    counts = np.ascontiguousarray(counts, np.int64)
    tops = np.ascontiguousarray(tops, np.int32)
    bottoms = np.ascontiguousarray(bottoms, np.int32)
    n = int(counts.shape[0])
    assert tops.shape == bottoms.shape and tops.shape[0] == n and tops.ndim in (2, 3)
    prow, pcol = (1, int(tops.shape[1])) if tops.ndim == 2 else (int(tops.shape[1]), int(tops.shape[2]))
    cap = 2 * prow * pcol * n
    offsets = np.zeros(n, np.int64)
    total = ctypes.c_int64(0)
    jl = np.zeros(max(cap, 1), np.int32)
    jt = np.zeros(max(cap, 1), np.int32)
    start = np.zeros(n + 1, np.int64)
    rc = lib().be_slab_merge(n, prow, pcol, counts.ctypes.data, tops.ctypes.data, bottoms.ctypes.data,
                             offsets.ctypes.data, ctypes.byref(total), jl.ctypes.data, jt.ctypes.data,
                             start.ctypes.data, cap)
    if rc != BE_OK:
        raise BEError(rc, "be_slab_merge: bad slab borders or counts")
    return SlabMerge(offsets, int(total.value), [jl[start[s]:start[s + 1]].copy() for s in range(n)],
                     [jt[start[s]:start[s + 1]].copy() for s in range(n)])


def slab_reserve(ctx: Context, max_count: int, max_joined: int) -> None:
    """Sizes the context's slab scratch so that later :func:`slab_relabel` calls of up to
    ``max_count`` local labels and ``max_joined`` joined labels allocate nothing
    (``be_slab_reserve``)."""
    ctx.check(lib().be_slab_reserve(ctx.handle, int(max_count), int(max_joined)))


def slab_relabel(ctx: Context, labels, count: int, offset: int, joined_labels: np.ndarray,
                 joined_targets: np.ndarray, stream=None) -> None:
    """Maps one slab's local labels (int32 CUDA tensor, 2D [rows, cols] or contiguous 3D
    [planes, d1, d2]) to the whole image's labels in place (``be_slab_relabel``)."""
    jl = np.ascontiguousarray(joined_labels, np.int32)
    jt = np.ascontiguousarray(joined_targets, np.int32)
    if labels.dim() == 3:
        assert labels.is_contiguous()
        rows, cols, pitch = int(labels.shape[0]) * int(labels.shape[1]), int(labels.shape[2]), int(labels.shape[2])
    else:
        rows, cols, pitch = int(labels.shape[0]), int(labels.shape[1]), int(labels.stride(0))
    ctx.check(lib().be_slab_relabel(ctx.handle, _ptr(labels), rows, cols, pitch, int(count), int(offset),
                                    jl.ctypes.data if jl.size else None, jt.ctypes.data if jt.size else None,
                                    int(jl.size), _stream(stream)))


def label2d_host(ctx: Context, img: np.ndarray, threshold: int = 0, algo: int = ALGO_AUTO,
                 coh: int = COH_DEFAULT, out: Optional[np.ndarray] = None) -> Tuple[np.ndarray, int, float]:
    """numpy uint8 [rows, cols] -> (int32 labels, component count, device µs).  Pass page-locked
    arrays (e.g. numpy views of pinned torch tensors) for full-speed copies."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    rows, cols = img.shape
    if out is None:
        out = np.empty((rows, cols), np.int32)
    assert out.shape == (rows, cols) and out.dtype == np.int32 and out.flags.c_contiguous
    n, us = ctypes.c_int64(0), ctypes.c_double(0)
    ctx.check(lib().be_label2d_host(ctx.handle, img.ctypes.data, cols, rows, cols, threshold, coh,
                                    algo, out.ctypes.data, cols, ctypes.byref(n), ctypes.byref(us)))
    return out, int(n.value), float(us.value)


def label3d_host(ctx: Context, vol: np.ndarray, threshold: int = 0, algo: int = ALGO_AUTO,
                 out: Optional[np.ndarray] = None) -> Tuple[np.ndarray, int, float]:
    vol = np.ascontiguousarray(vol, dtype=np.uint8)
    if out is None:
        out = np.empty(vol.shape, np.int32)
    assert out.shape == vol.shape and out.dtype == np.int32 and out.flags.c_contiguous
    n, us = ctypes.c_int64(0), ctypes.c_double(0)
    ctx.check(lib().be_label3d_host(ctx.handle, vol.ctypes.data, *vol.shape, threshold, algo,
                                    out.ctypes.data, ctypes.byref(n), ctypes.byref(us)))
    return out, int(n.value), float(us.value)


def autotune2d(ctx: Context, img, out, threshold: int = 0, stream=None) -> int:
    """Times every 2D form on this device image, keeps the fastest for its size class; returns
    the choice (0..2 = union-find tile shape, 16 = iterative form)."""
    ch = ctypes.c_int(-1)
    ctx.check(lib().be_autotune2d(ctx.handle, _ptr(img), int(img.stride(0)), int(img.shape[0]),
                                  int(img.shape[1]), threshold, _ptr(out), int(out.stride(0)),
                                  ctypes.byref(ch), _stream(stream)))
    return ch.value


def autotune3d(ctx: Context, vol, out, threshold: int = 0, stream=None) -> int:
    ch = ctypes.c_int(-1)
    ctx.check(lib().be_autotune3d(ctx.handle, _ptr(vol), *(int(x) for x in vol.shape), threshold,
                                  _ptr(out), ctypes.byref(ch), _stream(stream)))
    return ch.value


class Batch:
    """A fixed list of device images / volumes labeled by one CUDA-graph launch (be_batch_*).
    ``items``: sequence of (in_tensor, out_tensor[, threshold]); 2D tensors are images, 3D tensors
    dense volumes.  The tensors must outlive the batch."""

    def __init__(self, ctx: Context, items, flags: int = 0):
        self.ctx = ctx
        arr = (BEImage * len(items))()
        self._keep = []
        for i, it in enumerate(items):
            t_in, t_out = it[0], it[1]
            thr = it[2] if len(it) > 2 else 0
            e = arr[i]
            e.in_, e.out, e.threshold = _ptr(t_in), _ptr(t_out), int(thr)
            if t_in.dim() == 2:
                e.dims[0], e.dims[1], e.dims[2] = int(t_in.shape[0]), int(t_in.shape[1]), 0
                e.in_pitch, e.out_pitch = int(t_in.stride(0)), int(t_out.stride(0))
            else:
                e.dims[0], e.dims[1], e.dims[2] = (int(x) for x in t_in.shape)
                e.in_pitch = e.out_pitch = 0
            self._keep.append((t_in, t_out))
        self.n = len(items)
        self._h = ctypes.c_void_p()
        ctx.check(lib().be_batch_create(ctx.handle, arr, len(items), flags, ctypes.byref(self._h)))

    def run(self, stream=None) -> None:
        self.ctx.check(lib().be_batch_run(self._h, _stream(stream)))

    def counts(self, stream=None):
        out = (ctypes.c_int64 * self.n)()
        self.ctx.check(lib().be_batch_counts(self._h, out, _stream(stream)))
        return [int(x) for x in out]

    def tune(self, stream=None) -> int:
        ch = ctypes.c_int(-1)
        self.ctx.check(lib().be_batch_tune(self._h, _stream(stream), ctypes.byref(ch)))
        return ch.value

    def close(self) -> None:
        if self._h:
            lib().be_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching labeling server (be_server_*).  ``submit`` takes numpy arrays (host
    requests; page-locked arrays give asynchronous copies) or CUDA tensors with device=True; the
    arrays must stay alive until ``wait`` returns."""

    def __init__(self, device: int = 0, lanes: int = 2, max_batch: int = 256,
                 max_device_bytes: int = 0, inject_alloc_failure_every: int = 0):
        cfg = BEServerConfig()
        lib().be_server_default_config(ctypes.byref(cfg))
        cfg.device, cfg.lanes, cfg.max_batch = device, lanes, max_batch
        cfg.max_device_bytes, cfg.inject_alloc_failure_every = max_device_bytes, inject_alloc_failure_every
        self._h = ctypes.c_void_p()
        rc = lib().be_server_create(ctypes.byref(cfg), ctypes.byref(self._h))
        if rc:
            raise BEError(rc, "be_server_create failed")

    def submit(self, img, out, threshold: int = 0, device: bool = False) -> int:
        r = BERequest()
        if device:
            r.in_, r.out = _ptr(img), _ptr(out)
        else:
            assert img.flags.c_contiguous and out.flags.c_contiguous and out.dtype == np.int32
            r.in_, r.out = img.ctypes.data, out.ctypes.data
        shp = tuple(int(x) for x in img.shape)
        r.dims[0], r.dims[1], r.dims[2] = shp[0], shp[1], shp[2] if len(shp) == 3 else 0
        r.threshold, r.flags = threshold, REQ_DEVICE_BUFFERS if device else 0
        i = ctypes.c_uint64(0)
        rc = lib().be_server_submit(self._h, ctypes.byref(r), ctypes.byref(i))
        if rc:
            raise BEError(rc, "be_server_submit failed")
        return int(i.value)

    def wait(self, rid: int, timeout_us: int = -1):
        """(status, n_components, latency_us); status BE_ERR_TIMEOUT leaves the request pending."""
        res = BEResult()
        st = lib().be_server_wait(self._h, rid, timeout_us, ctypes.byref(res))
        if st == 5:
            return 5, None, None
        return int(res.status), int(res.n_components), float(res.latency_us)

    def cancel(self, rid: int) -> int:
        return lib().be_server_cancel(self._h, rid)

    def stats(self) -> dict:
        st = BEServeStats()
        lib().be_server_stats(self._h, ctypes.byref(st))
        return {f: getattr(st, f) for f, _ in BEServeStats._fields_}

    def reset_stats(self) -> None:
        lib().be_server_reset_stats(self._h)

    def close(self) -> None:
        if self._h:
            lib().be_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --- the reference's labeler interface (ILabeling / IOCLLabeling3D shape) --------------------

class Labeling:
    """2D labeler with the call shape of ``ILabeling::Label``: binarizes with threshold 8 (the
    reference's ``RGB2Gray``, LabelingTools.cpp:39-49), labels on the GPU and returns
    ``(labels, time_us)``; ``time_us`` covers the labeling only, like the reference's ``watch_``.
    ``threads`` is accepted for interface parity and ignored (OpenMP thread count)."""

    threshold = 8

    def __init__(self, algo: int = ALGO_AUTO, device: int = 0):
        self.ctx = Context(device)
        self.algo = algo

    def Label(self, pixels: np.ndarray, threads: int = 0, coh: int = COH_DEFAULT):
        if pixels.size == 0:
            raise ValueError("Labeling.Label : Input image is empty")
        if pixels.ndim == 3:   # colour input: cv::cvtColor(COLOR_RGB2GRAY), 14-bit fixed point
            r, g, b = (pixels[..., k].astype(np.uint32) for k in range(3))
            pixels = ((r * 4899 + g * 9617 + b * 1868 + (1 << 13)) >> 14).astype(np.uint8)
        labels, _, us = label2d_host(self.ctx, pixels, self.threshold, self.algo, coh)
        return labels, us


class RunEquivalence(Labeling):
    """The ``runeq -g`` slot (TOCLRunEquivLabeling, LabelingAlgs.cpp:1090-1268): the reference's
    run kernels join runs that overlap in a column -- 4-connectivity -- whatever coherence is
    asked for, and reject COH_4 themselves; so does this: COH_4 raises, anything else labels
    4-connected with the run-equivalence form (ALGO_RUNS)."""

    def __init__(self, device: int = 0):
        super().__init__(ALGO_RUNS, device)

    def Label(self, pixels: np.ndarray, threads: int = 0, coh: int = COH_DEFAULT):
        if coh == COH_4:
            raise ValueError("RunEquivalence.Label : 4x connectivity is not implemented for this method")
        return super().Label(pixels, threads, COH_4)


class Labeling3D:
    """3D labeler with the call shape of ``IOCLLabeling3D::Label`` (LabelingTools.cpp:180-221):
    only the default connectivity is accepted; the input volume is used as is (``Read3DImage``
    already binarized its slices)."""

    threshold = 0

    def __init__(self, algo: int = ALGO_AUTO, device: int = 0):
        self.ctx = Context(device)
        self.algo = algo

    def Label(self, pixels: np.ndarray, threads: int = 0, coh: int = COH_DEFAULT):
        if pixels.size == 0:
            raise ValueError("Labeling3D.Label : Input image is empty")
        if pixels.ndim != 3:
            raise ValueError("Labeling3D.Label : Input image is not a 3D image")
        if coh != COH_DEFAULT:
            raise ValueError("Labeling3D.Label : Only default coherence is supported for 3D labeling")
        labels, _, us = label3d_host(self.ctx, pixels, self.threshold, self.algo)
        return labels, us


ALGORITHMS = {
    "bleq": ("Block equivalence by Zavalishin et.al. 2016", ALGO_AUTO),
    "lbeq": ("Label equivalence by Kalentev et.al. 2012 (pixel level)", ALGO_PIXEL),
    "runeq": ("Run equivalence by Bekhtin et.al. 2015 (4-connected, 2D only)", ALGO_RUNS),
}


def make_labeler(name: str, gpu: bool = True, three_d: bool = False, device: int = 0):
    """The reference's algorithm registry (main.cpp:101-131, SetLabelingAlg :373-395) for the GPU
    slots this package fills: ``-a bleq|lbeq [-3] -g``.  CPU slots are not provided."""
    if name not in ALGORITHMS:
        raise ValueError("No labeling algorithm specified" if not name else
                         f"Chosen algorithm '{name}' is not provided by the GPU labeler")
    if not gpu:
        raise ValueError("Chosen algorithm doesn't support specified capabilities (CPU mode)")
    algo = ALGORITHMS[name][1]
    if name == "runeq":
        if three_d:   # the reference has no 3D run equivalence (main.cpp:127-130)
            raise ValueError("Chosen algorithm doesn't support specified capabilities (3D)")
        return RunEquivalence(device)
    return Labeling3D(algo, device) if three_d else Labeling(algo, device)
