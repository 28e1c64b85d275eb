"""knnag_forward_noalloc: the forward for callers that cannot allocate device
memory (allocator-free serving sections, plugins whose host framework owns
all device allocations).  Its scratch is a fixed array inside the library,
so it must give the same results as knnag_forward -- on consecutive calls,
whatever the previous call left in that shared array.

Tolerances as in the other parity tests: idxs and dists exact, w_out and
f_out within 1e-5 relative to the tensor's max.  After every call the
array's device status word is read back (knnag_noalloc_read_device_status)
and must be clear.  The cases cover each layout the array can hold: FP32
with the spatial search index (K <= 32), FP32 with K > 32 (exact kernel
only), FP64 (larger records, no index), and an FP32 shape whose scratch is
just under the array's size.  The file name sorts last so a run that stops
at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_err

FWD_TOL = 1e-5


def lib_and_capi():
    from cuda_knn_aggregate import capi

    L = capi.lib()
    V, I = ctypes.c_void_p, ctypes.c_int
    fn = L.knnag_forward_noalloc
    fn.argtypes = [V] * 5 + [I] * 6 + [V] * 4 + [V]
    fn.restype = I
    return fn, capi


def run_noalloc(fn, capi, q, p, f, sigma, R, K):
    B, Q, P, F = q.shape[0], q.shape[1], p.shape[1], f.shape[2]
    o = dict(dtype=q.dtype, device=q.device)
    f_out, w_out, dists = torch.empty(B, Q, F, **o), torch.empty(B, Q, K, **o), torch.empty(B, Q, K, **o)
    idxs = torch.empty(B, Q, K, dtype=torch.int64, device=q.device)
    rc = fn(*[capi._p(t) for t in (q, p, f, sigma, R)], B, Q, P, F, K, capi._dtype(q),
            *[capi._p(t) for t in (f_out, w_out, dists, idxs)], capi._stream(q.device))
    assert rc == 0, capi.lib().knnag_status_string(rc).decode()
    return f_out, w_out, dists, idxs


def assert_same(a, b):
    f0, w0, d0, i0 = [x.cpu().numpy() for x in a]
    f1, w1, d1, i1 = [x.cpu().numpy() for x in b]
    assert np.array_equal(i0, i1)
    assert np.array_equal(d0.view(np.uint8), d1.view(np.uint8))
    assert rel_err(w0, w1) < FWD_TOL
    assert rel_err(f0, f1) < FWD_TOL


@pytest.mark.gpu
def test_noalloc_matches_forward_on_consecutive_calls():
    from cuda_knn_aggregate import workloads as W

    fn, capi = lib_and_capi()
    dev = torch.device("cuda:0")
    # two different problems back to back: the second call must not see the
    # first one's leftovers in the shared scratch
    cases = [W.make("small", B=2, Q=1000, P=500, F=32, K=12, seed=31),
             W.make("small", B=1, Q=700, P=2300, F=20, K=16, seed=32)]
    for shape, t in cases + cases:
        x = [a.to(dev) for a in t]
        got = run_noalloc(fn, capi, *x, shape.K)
        assert capi.noalloc_device_status(dev) == 0
        want = capi.forward(*x, shape.K)
        torch.cuda.synchronize()
        assert_same(got, want)


@pytest.mark.gpu
def test_noalloc_other_layouts_and_the_size_limit():
    """FP64, K > 32 and a shape whose scratch is just under the fixed array
    (and one point more, which must be refused), each twice in a row."""
    from cuda_knn_aggregate import workloads as W

    fn, capi = lib_and_capi()
    dev = torch.device("cuda:0")
    lim = 8 << 20
    L = capi.lib()
    # FP32, K=16, Q=512: the largest P whose scratch fits (bisection on the
    # library's own workspace size)
    lo, hi = 1, 1 << 20
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if L.knnag_forward_workspace_bytes(1, 512, mid, 8, 16, capi.F32) <= lim:
            lo = mid
        else:
            hi = mid - 1
    near_P = lo
    assert 25000 < near_P < 40000  # about 276 bytes per point
    assert L.knnag_forward_workspace_bytes(1, 512, near_P, 8, 16, capi.F32) <= lim
    assert L.knnag_forward_workspace_bytes(1, 512, near_P + 1, 8, 16, capi.F32) > lim
    cases = [W.make("small", B=2, Q=300, P=400, F=6, K=9, seed=33, dtype=torch.float64),
             W.make("small", B=1, Q=200, P=300, F=8, K=40, seed=34),
             W.make("small", B=1, Q=512, P=near_P, F=8, K=16, seed=35)]
    for shape, t in cases + cases:
        x = [a.to(dev) for a in t]
        got = run_noalloc(fn, capi, *x, shape.K)
        assert capi.noalloc_device_status(dev) == 0
        want = capi.forward(*x, shape.K)
        torch.cuda.synchronize()
        assert_same(got, want)
    _, t = W.make("small", B=1, Q=512, P=near_P + 1, F=8, K=16, seed=36)
    x = [a.to(dev) for a in t]
    with pytest.raises(RuntimeError, match="scratch"):
        capi.forward_noalloc(*x, 16)


@pytest.mark.gpu
def test_noalloc_rejects_sizes_beyond_its_scratch():
    fn, capi = lib_and_capi()
    dev = torch.device("cuda:0")
    B, Q, P, F, K = 1, 4, 1 << 20, 4, 8  # records alone would need 64 MiB
    q = torch.zeros(B, Q, 3, device=dev)
    small = torch.zeros(16, device=dev)  # never read: the size check comes first
    ptr = capi._p(small)
    out = torch.zeros(64, device=dev)
    rc = fn(capi._p(q), ptr, ptr, ptr, ptr, B, Q, P, F, K, 0, capi._p(out), capi._p(out), capi._p(out),
            capi._p(out), capi._stream(dev))
    assert rc == 8
    assert b"scratch" in capi.lib().knnag_status_string(rc)
