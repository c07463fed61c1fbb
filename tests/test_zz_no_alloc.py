"""be_label2d_noalloc: the 2D entry point for callers that cannot allocate device memory (a
framework that owns the device memory pool, a loop that must not stall on cudaMalloc, a plugin
host that forbids allocation).  Its scratch is a fixed array inside the library, so this test
checks that two calls in a row give exactly what be_label2d gives (labels are integers: the
tolerance is exact), and that an image beyond the fixed limit is refused.  Collected last on
purpose; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc():
    import labeling_b200 as be
    f = be.lib().be_label2d_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    return f


def test_noalloc_matches_label2d_on_two_calls():
    import torch
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    f = _noalloc()
    ctx = be.Context(0)
    images = [W.bernoulli((1000, 1500), 0.5, seed=21), W.disks(2048, 3000, 300, 4, 60, 0.05, seed=22)]
    for img in images:
        d_in = torch.from_numpy(img).cuda()
        ref = torch.empty(img.shape, dtype=torch.int32, device="cuda")
        k_ref = be.label2d(ctx, d_in, ref)
        out = torch.full(img.shape, -1, dtype=torch.int32, device="cuda")
        k = ctypes.c_int64(-1)
        stream = torch.cuda.current_stream().cuda_stream
        rc = f(d_in.data_ptr(), img.shape[1], img.shape[0], img.shape[1], 0, out.data_ptr(),
               img.shape[1], ctypes.byref(k), stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert k.value == k_ref
        assert torch.equal(out, ref)
    ctx.close()


@pytest.mark.parametrize("shape", [(4096, 4096), (65536, 256)])
def test_noalloc_at_its_limits(shape):
    """Images that fill the fixed scratch exactly: 4096 x 4096 is 1024 tiles, 65536 x 256 is 1024
    tiles and 65536 segments (one per row).  Labels and count must equal be_label2d's; one call
    passes no count pointer and is followed by a stream synchronization."""
    import torch
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    f = _noalloc()
    ctx = be.Context(0)
    img = W.bernoulli(shape, 0.45, seed=shape[0] % 97)
    d_in = torch.from_numpy(img).cuda()
    ref = torch.empty(img.shape, dtype=torch.int32, device="cuda")
    k_ref = be.label2d(ctx, d_in, ref)
    stream = torch.cuda.current_stream()
    for want_count in (True, False):
        out = torch.full(img.shape, -1, dtype=torch.int32, device="cuda")
        k = ctypes.c_int64(-1)
        rc = f(d_in.data_ptr(), img.shape[1], img.shape[0], img.shape[1], 0, out.data_ptr(),
               img.shape[1], ctypes.byref(k) if want_count else None, stream.cuda_stream)
        assert rc == 0
        stream.synchronize()
        if want_count:
            assert k.value == k_ref
        assert torch.equal(out, ref)
    ctx.close()


def test_noalloc_refuses_images_beyond_its_scratch():
    import torch
    f = _noalloc()
    rows, cols = 4097, 4096   # 65 tile rows x 16 tile columns > 1024 tiles
    d_in = torch.zeros(1, dtype=torch.uint8, device="cuda")
    d_out = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = f(d_in.data_ptr(), cols, rows, cols, 0, d_out.data_ptr(), cols, None, None)
    assert rc == 8   # BE_ERR_TOO_LARGE, before anything is launched
