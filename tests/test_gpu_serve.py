"""The serving loop: continuous batching of mixed 2D / 3D requests.  Every result must equal the
same image labeled alone (exact), whatever else was in flight; admission, injected allocation
failures, cancellation and timeouts are exercised on the host side (no GPU fault)."""
import threading

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mixed(seed, n=30):
    from labeling_b200 import workloads as W
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if rng.random() < 0.8:
            h, w = (int(x) for x in np.exp(rng.uniform(np.log(16), np.log(1500), 2)))
            out.append(W.bernoulli((h, w), float(rng.uniform(0.2, 0.8)), int(rng.integers(1 << 30))))
        else:
            d = tuple(int(x) for x in np.exp(rng.uniform(np.log(8), np.log(90), 3)))
            out.append(W.bernoulli(d, float(rng.uniform(0.05, 0.35)), int(rng.integers(1 << 30))))
    return out


def _ref(img):
    return O.ccl2d(img) if img.ndim == 2 else O.ccl3d(img)


def test_mixed_stream_two_threads_equals_alone(ctx):
    import labeling_b200 as be
    imgs = _mixed(1, 40)
    outs = [np.full(a.shape, -1, np.int32) for a in imgs]
    srv = be.Server(lanes=2, max_batch=8)
    ids = [None] * len(imgs)

    def producer(part):
        for i in part:
            ids[i] = srv.submit(imgs[i], outs[i])

    th = [threading.Thread(target=producer, args=(range(k, len(imgs), 2),)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i, rid in enumerate(ids):
        st, k, lat = srv.wait(rid)
        ref, kr = _ref(imgs[i])
        assert st == 0 and k == kr and lat > 0, i
        assert np.array_equal(outs[i], ref), i
    # the same images labeled alone through the plain entry points
    for i in (0, 1, len(imgs) - 1):
        alone = (be.label2d_host if imgs[i].ndim == 2 else be.label3d_host)(ctx, imgs[i])[0]
        assert np.array_equal(alone, outs[i])
    s = srv.stats()
    assert s["completed"] == len(imgs) and s["batches"] >= 2 and s["p99_us"] >= s["p50_us"] > 0
    srv.close()


def test_admission_refuses_what_can_never_fit():
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    srv = be.Server(max_device_bytes=32 << 20)
    big = W.bernoulli((4096, 4096), 0.5, 1)       # needs ~117 MB
    small = W.bernoulli((300, 400), 0.5, 2)
    ob, os_ = np.zeros(big.shape, np.int32), np.zeros(small.shape, np.int32)
    rb, rs = srv.submit(big, ob), srv.submit(small, os_)
    assert srv.wait(rb)[0] == 6                    # BE_ERR_BUSY
    st, k, _ = srv.wait(rs)
    assert st == 0 and np.array_equal(os_, O.ccl2d(small)[0])
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_injected_allocation_failures_do_not_stop_the_server():
    import labeling_b200 as be
    imgs = _mixed(2, 24)
    outs = [np.zeros(a.shape, np.int32) for a in imgs]
    srv = be.Server(lanes=1, max_batch=1, inject_alloc_failure_every=5)
    ids = [srv.submit(a, o) for a, o in zip(imgs, outs)]
    failed = ok = 0
    for a, o, rid in zip(imgs, outs, ids):
        st, k, _ = srv.wait(rid)
        if st == 2:                                # BE_ERR_OOM from the injected failure
            failed += 1
        else:
            assert st == 0 and np.array_equal(o, _ref(a)[0])
            ok += 1
    assert failed > 0 and ok > 0
    srv.close()


def test_cancel_and_timeout():
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    srv = be.Server(lanes=1, max_batch=1)
    imgs = [W.bernoulli((2048, 2048), 0.5, s) for s in range(6)]
    outs = [np.zeros(a.shape, np.int32) for a in imgs]
    ids = [srv.submit(a, o) for a, o in zip(imgs, outs)]
    assert srv.cancel(ids[-1]) == 0
    r0 = srv.wait(ids[0], timeout_us=0)             # done already, or BE_ERR_TIMEOUT (pending)
    if r0[0] == 5:
        r0 = srv.wait(ids[0])
    assert r0[0] == 0 and np.array_equal(outs[0], O.ccl2d(imgs[0])[0])
    for a, o, rid in zip(imgs[1:-1], outs[1:-1], ids[1:-1]):
        st, k, _ = srv.wait(rid)
        assert st == 0 and np.array_equal(o, O.ccl2d(a)[0])
    assert srv.wait(ids[-1])[0] == 7                # BE_ERR_CANCELLED
    srv.close()


def test_device_resident_requests():
    import torch
    import labeling_b200 as be
    imgs = _mixed(3, 12)
    d_in = [torch.from_numpy(a).cuda() for a in imgs]
    d_out = [torch.zeros(a.shape, dtype=torch.int32, device="cuda") for a in imgs]
    srv = be.Server(lanes=2, max_batch=4)
    ids = [srv.submit(x, y, device=True) for x, y in zip(d_in, d_out)]
    for a, y, rid in zip(imgs, d_out, ids):
        st, k, _ = srv.wait(rid)
        ref, kr = _ref(a)
        assert st == 0 and k == kr and np.array_equal(y.cpu().numpy(), ref)
    srv.close()


def test_admission_sees_memory_taken_after_creation():
    """Admission reads the device's free memory when it forms a batch, not only the budget fixed
    at creation: memory another user of the GPU takes later holds a request back (it stays
    pending, no failure) until that memory is released."""
    import torch
    import labeling_b200 as be
    from labeling_b200 import workloads as W
    torch.cuda.empty_cache()
    srv = be.Server(lanes=1, max_batch=1)          # budget: 80% of the free memory now
    img = W.bernoulli((4096, 4096), 0.5, 3)         # needs ~117 MB of device memory
    out = np.zeros(img.shape, np.int32)
    free, _ = torch.cuda.mem_get_info()
    hog = torch.empty(max(free - (48 << 20), 0), dtype=torch.uint8, device="cuda")   # leaves ~48 MB
    try:
        rid = srv.submit(img, out)
        st, _, _ = srv.wait(rid, timeout_us=300_000)
        assert st == 5                              # BE_ERR_TIMEOUT: still waiting for memory
    finally:
        del hog
        torch.cuda.empty_cache()
    st, k, _ = srv.wait(rid)
    ref, kr = O.ccl2d(img)
    assert st == 0 and k == kr and np.array_equal(out, ref)
    srv.close()
