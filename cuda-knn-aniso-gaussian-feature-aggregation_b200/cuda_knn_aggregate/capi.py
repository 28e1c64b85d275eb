"""ctypes binding of the C ABI in ``include/knn_aniso.h`` (libknn_aniso.so).

This is the binding a host program without the torch extension would use:
plain device pointers, sizes, a stream handle and an int status.  Torch is
used here only to allocate device memory and to name the current stream.
Every function raises ``RuntimeError`` with the library's status text when
the status is not ``KNNAG_OK``.
"""
from __future__ import annotations

import ctypes
import os
import re

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libknn_aniso.so")
HEADER = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include", "knn_aniso.h")

F32, F64 = 0, 1
NEED_DQ, NEED_DP, NEED_DF, NEED_DSIGMA, NEED_DR, NEED_DGFO = 1, 2, 4, 8, 16, 32
NEED_ALL = 63

_V = ctypes.c_void_p
_I = ctypes.c_int
_S = ctypes.c_size_t

_SIGS = {
    "knnag_status_string": ([_I], ctypes.c_char_p),
    "knnag_version": ([], _I),
    "knnag_forward_workspace_bytes": ([_I, _I, _I, _I, _I, _I], _S),
    "knnag_forward": ([_V] * 5 + [_I] * 6 + [_V] * 4 + [_V, _V, _S, _V], _I),
    "knnag_forward_noalloc": ([_V] * 5 + [_I] * 6 + [_V] * 4 + [_V], _I),
    "knnag_noalloc_read_device_status": ([_V], _I),
    "knnag_variant_workspace_bytes": ([_I, _I, _I, _I], _S),
    "knnag_forward_precomputed": ([_V] * 6 + [_I] * 6 + [_V] * 3 + [_V, _S, _V], _I),
    "knnag_forward_lookup": ([_V] * 6 + [_I] * 7 + [_V] * 4 + [_V, _S, _V], _I),
    "knnag_forward_isotropic": ([_V] * 4 + [_I] * 7 + [_V] * 4 + [_V], _I),
    "knnag_cloudset_bytes": ([_I, _V], _S),
    "knnag_cloudset_build_workspace_bytes": ([_I, _V], _S),
    "knnag_cloudset_init": ([_I, _V, _V, _S, _V], _I),
    "knnag_cloudset_build": ([_V, _V, _V, _I, _V, _V, _S, _V, _S, _V], _I),
    "knnag_segments_bytes": ([_I], _S),
    "knnag_segments_encode": ([_I, _V, _V, _V, _V, _I, _V, _I, _V, _S], _I),
    "knnag_ragged_workspace_bytes": ([_I, ctypes.c_longlong], _S),
    "knnag_ragged_forward": ([_V, _V, _V, _V, _I, _I, ctypes.c_longlong, ctypes.c_longlong, _I, _I, _I]
                             + [_V] * 4 + [_V, _S, _V], _I),
    "knnag_ragged_grad_q": ([_V, _V, _V, _V, _I, _V, _V, _V, _I, ctypes.c_longlong, ctypes.c_longlong, _I, _I, _V,
                             _V, _S, _V], _I),
    "knnag_feature_row_sums": ([_V, ctypes.c_longlong, _I, _I, _V, _V], _I),
    "knnag_points_bytes": ([_I, _I, _I], _S),
    "knnag_pack_points": ([_V, _V, _V, _I, _I, _I, _V, _V], _I),
    "knnag_adjacency_bytes": ([_I, _I, _I, _I], _S),
    "knnag_build_adjacency": ([_V, _I, _I, _I, _I, _V, _V], _I),
    "knnag_forward_counted": ([_V] * 5 + [_I] * 6 + [_V] * 4 + [_V, _V, _V, _S, _V], _I),
    "knnag_build_adjacency_counted": ([_V, _I, _I, _I, _I, _V, _V], _I),
    "knnag_backward_workspace_bytes": ([_I, _I, _I, _I, _I, _I], _S),
    "knnag_backward": ([_V] * 9 + [_I] * 7 + [_V, _V] + [_V] * 6 + [_V, _S, _V], _I),
    "knnag_backward_2nd": ([_V] * 10 + [_I] * 7 + [_V, _V, _V] + [_V] * 6 + [_V, _S, _V], _I),
    "knnag_read_device_status": ([_V, _V], _I),
    "knnag_set_profile_events": ([_V, _V], None),
    "knnag_launch_count": ([], ctypes.c_longlong),
    "knnag_fp32_peak_probe": ([_V, _I, _I, _V], _I),
    "knnag_set_search_splits": ([_I], _I),
    "knnag_get_search_splits": ([], _I),
    "knnag_debug_set_search_stall": ([_I, _I], _I),
}

_lib = None


def lib():
    """Load libknn_aniso.so and declare every exported signature."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python build.py`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def header_functions():
    """Names of the functions declared in include/knn_aniso.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+char\*|int|size_t|void|long\s+long)\s+(knnag_\w+)\s*\(",
                                 text, re.M)))


def _p(t):
    if t is None:
        return None
    if not t.is_contiguous():
        raise ValueError("the C ABI takes dense row-major arrays: pass contiguous tensors")
    return ctypes.c_void_p(t.data_ptr())


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _dtype(t):
    if t.dtype == torch.float32:
        return F32
    if t.dtype == torch.float64:
        return F64
    raise TypeError("float32 or float64 only")


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().knnag_status_string(rc).decode())


def forward(q, p, f, sigma, R, K, points=None):
    """knnag_forward: returns (f_out, w_out, dists, idxs)."""
    B, Q, P, F = q.shape[0], q.shape[1], p.shape[1], f.shape[2]
    dt = _dtype(q)
    f_out = torch.empty(B, Q, F, dtype=q.dtype, device=q.device)
    w_out = torch.empty(B, Q, K, dtype=q.dtype, device=q.device)
    dists = torch.empty(B, Q, K, dtype=q.dtype, device=q.device)
    idxs = torch.empty(B, Q, K, dtype=torch.int64, device=q.device)
    nb = lib().knnag_forward_workspace_bytes(B, Q, P, F, K, dt)
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=q.device)
    _check(lib().knnag_forward(_p(q), _p(p), _p(f), _p(sigma), _p(R), B, Q, P, F, K, dt, _p(f_out), _p(w_out),
                               _p(dists), _p(idxs), _p(points), _p(ws), nb, _stream(q.device)))
    return f_out, w_out, dists, idxs


def forward_noalloc(q, p, f, sigma, R, K):
    """knnag_forward_noalloc (scratch in the library's fixed device array):
    returns (f_out, w_out, dists, idxs).  Read its device status with
    noalloc_device_status() before the next call."""
    B, Q, P, F = q.shape[0], q.shape[1], p.shape[1], f.shape[2]
    o = dict(dtype=q.dtype, device=q.device)
    f_out, w_out, dists = torch.empty(B, Q, F, **o), torch.empty(B, Q, K, **o), torch.empty(B, Q, K, **o)
    idxs = torch.empty(B, Q, K, dtype=torch.int64, device=q.device)
    _check(lib().knnag_forward_noalloc(_p(q), _p(p), _p(f), _p(sigma), _p(R), B, Q, P, F, K, _dtype(q), _p(f_out),
                                       _p(w_out), _p(dists), _p(idxs), _stream(q.device)))
    return f_out, w_out, dists, idxs


def noalloc_device_status(device):
    """knnag_noalloc_read_device_status on `device`: 0 (ok) or 7 (an error
    latched on the device); synchronises the current stream."""
    with torch.cuda.device(device):
        return int(lib().knnag_noalloc_read_device_status(_stream(device)))


def forward_precomputed(q, p, f, sigma, R, knn_idxs):
    """knnag_forward_precomputed: returns (f_out, w_out, dists)."""
    B, Q, P, F, K = q.shape[0], q.shape[1], p.shape[1], f.shape[2], knn_idxs.shape[2]
    dt = _dtype(q)
    o = dict(dtype=q.dtype, device=q.device)
    f_out, w_out, dists = torch.empty(B, Q, F, **o), torch.empty(B, Q, K, **o), torch.empty(B, Q, K, **o)
    nb = lib().knnag_variant_workspace_bytes(B, Q, P, dt)
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=q.device)
    _check(lib().knnag_forward_precomputed(_p(q), _p(p), _p(f), _p(sigma), _p(R), _p(knn_idxs), B, Q, P, F, K, dt,
                                           _p(f_out), _p(w_out), _p(dists), _p(ws), nb, _stream(q.device)))
    return f_out, w_out, dists


def forward_lookup(q, p, f, sigma, R, knn_table, K):
    """knnag_forward_lookup: returns (f_out, w_out, dists, idxs)."""
    B, Q, P, F = q.shape[0], q.shape[1], p.shape[1], f.shape[2]
    dt = _dtype(q)
    o = dict(dtype=q.dtype, device=q.device)
    f_out, w_out, dists = torch.empty(B, Q, F, **o), torch.empty(B, Q, K, **o), torch.empty(B, Q, K, **o)
    idxs = torch.empty(B, Q, K, dtype=torch.int64, device=q.device)
    nb = lib().knnag_variant_workspace_bytes(B, Q, P, dt)
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=q.device)
    _check(lib().knnag_forward_lookup(_p(q), _p(p), _p(f), _p(sigma), _p(R), _p(knn_table), knn_table.shape[1], B, Q,
                                      P, F, K, dt, _p(f_out), _p(w_out), _p(dists), _p(idxs), _p(ws), nb,
                                      _stream(q.device)))
    return f_out, w_out, dists, idxs


def forward_isotropic(q, p, f, sigma, K):
    """knnag_forward_isotropic: returns (f_out, w_sum [B,Q,1], dists, idxs)."""
    B, Q, P, F = q.shape[0], q.shape[1], p.shape[1], f.shape[2]
    dt = _dtype(q)
    o = dict(dtype=q.dtype, device=q.device)
    f_out, w_sum, dists = torch.empty(B, Q, F, **o), torch.empty(B, Q, 1, **o), torch.empty(B, Q, K, **o)
    idxs = torch.empty(B, Q, K, dtype=torch.int64, device=q.device)
    _check(lib().knnag_forward_isotropic(_p(q), _p(p), _p(f), _p(sigma), sigma.shape[2], B, Q, P, F, K, dt,
                                         _p(f_out), _p(w_sum), _p(dists), _p(idxs), _stream(q.device)))
    return f_out, w_sum, dists, idxs


def pack_points(p, sigma, R):
    B, P = p.shape[0], p.shape[1]
    out = torch.empty(B, P, 16, dtype=p.dtype, device=p.device)
    _check(lib().knnag_pack_points(_p(p), _p(sigma), _p(R), B, P, _dtype(p), _p(out), _stream(p.device)))
    return out


def build_adjacency(idxs, P):
    B, Q, K = idxs.shape
    nb = lib().knnag_adjacency_bytes(B, Q, P, K)
    adj = torch.empty(max(nb, 1), dtype=torch.uint8, device=idxs.device)
    _check(lib().knnag_build_adjacency(_p(idxs), B, Q, P, K, _p(adj), _stream(idxs.device)))
    return adj


def forward_counted(q, p, f, sigma, R, K):
    """knnag_forward_counted, then knnag_build_adjacency_counted: returns
    (f_out, w_out, dists, idxs, adjacency)."""
    B, Q, P, F = q.shape[0], q.shape[1], p.shape[1], f.shape[2]
    dt = _dtype(q)
    o = dict(dtype=q.dtype, device=q.device)
    f_out, w_out, dists = torch.empty(B, Q, F, **o), torch.empty(B, Q, K, **o), torch.empty(B, Q, K, **o)
    idxs = torch.empty(B, Q, K, dtype=torch.int64, device=q.device)
    nb = lib().knnag_forward_workspace_bytes(B, Q, P, F, K, dt)
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=q.device)
    na = lib().knnag_adjacency_bytes(B, Q, P, K)
    adj = torch.empty(max(na, 1), dtype=torch.uint8, device=q.device)
    st = _stream(q.device)
    _check(lib().knnag_forward_counted(_p(q), _p(p), _p(f), _p(sigma), _p(R), B, Q, P, F, K, dt, _p(f_out), _p(w_out),
                                       _p(dists), _p(idxs), None, _p(adj), _p(ws), nb, st))
    _check(lib().knnag_build_adjacency_counted(_p(idxs), B, Q, P, K, _p(adj), st))
    return f_out, w_out, dists, idxs, adj


def adjacency_arrays(adj, B, Q, P, K):
    """(rowptr [B*P+1], entries [B*Q*K]) int32 views of an adjacency buffer."""
    rows, n = B * P, B * Q * K
    r256 = lambda x: (x + 255) // 256 * 256
    i32 = adj.view(torch.int32)
    off = (r256((rows + 1) * 4) + r256(rows * 4) + r256(n * 4)) // 4
    return i32[: rows + 1], i32[off: off + n]


def backward(gfo, q, p, f, sigma, R, idxs, w_out=None, needs=NEED_ALL & ~NEED_DGFO, points=None, adjacency=None,
             want_coef=False):
    """knnag_backward: returns (dq, dp, df, dsigma, dR, coef) (None where not requested)."""
    B, Q, P, F, K = q.shape[0], q.shape[1], p.shape[1], f.shape[2], idxs.shape[2]
    dt = _dtype(q)
    mk = lambda bit, *shape: torch.empty(*shape, dtype=q.dtype, device=q.device) if needs & bit else None
    dq, dp, df = mk(NEED_DQ, B, Q, 3), mk(NEED_DP, B, P, 3), mk(NEED_DF, B, P, F)
    ds, dR = mk(NEED_DSIGMA, B, P, 3), mk(NEED_DR, B, P, 3, 3)
    coef = torch.empty(B, Q, K, dtype=q.dtype, device=q.device) if want_coef else None
    nb = lib().knnag_backward_workspace_bytes(B, Q, P, F, K, dt)
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=q.device)
    _check(lib().knnag_backward(_p(gfo), None, _p(q), _p(p), _p(f), _p(sigma), _p(R), _p(w_out), _p(idxs), B, Q, P,
                                F, K, dt, needs, _p(points), _p(adjacency), _p(dq), _p(dp), _p(df), _p(ds), _p(dR),
                                _p(coef), _p(ws), nb, _stream(q.device)))
    return dq, dp, df, ds, dR, coef


def backward_2nd(ggq, gfo, q, p, f, sigma, R, idxs, w_out=None, needs=NEED_ALL, points=None, adjacency=None,
                 coef=None):
    """knnag_backward_2nd: returns (dgfo, dq, dp, df, dsigma, dR)."""
    B, Q, P, F, K = q.shape[0], q.shape[1], p.shape[1], f.shape[2], idxs.shape[2]
    dt = _dtype(q)
    mk = lambda bit, *shape: torch.empty(*shape, dtype=q.dtype, device=q.device) if needs & bit else None
    dgfo, dq, dp = mk(NEED_DGFO, B, Q, F), mk(NEED_DQ, B, Q, 3), mk(NEED_DP, B, P, 3)
    df, ds, dR = mk(NEED_DF, B, P, F), mk(NEED_DSIGMA, B, P, 3), mk(NEED_DR, B, P, 3, 3)
    nb = lib().knnag_backward_workspace_bytes(B, Q, P, F, K, dt)
    ws = torch.empty(max(nb, 1), dtype=torch.uint8, device=q.device)
    _check(lib().knnag_backward_2nd(_p(ggq), _p(gfo), None, _p(q), _p(p), _p(f), _p(sigma), _p(R), _p(w_out),
                                    _p(idxs), B, Q, P, F, K, dt, needs, _p(points), _p(adjacency), _p(coef),
                                    _p(dgfo), _p(dq), _p(dp), _p(df), _p(ds), _p(dR), _p(ws), nb,
                                    _stream(q.device)))
    return dgfo, dq, dp, df, ds, dR


def set_profile_events(ev_begin, ev_end):
    """Record torch.cuda.Event pair around every later forward's search kernel
    (None, None switches it off).  The events must have been recorded once so
    their CUDA handles exist."""
    h = lambda e: ctypes.c_void_p(e.cuda_event) if e is not None else None
    lib().knnag_set_profile_events(h(ev_begin), h(ev_end))


def launch_count():
    return int(lib().knnag_launch_count())


def fp32_peak_probe(out, blocks, iters):
    _check(lib().knnag_fp32_peak_probe(_p(out), blocks, iters, _stream(out.device)))


def set_search_splits(splits):
    """Process-wide split count of the uniform search (0: automatic)."""
    _check(lib().knnag_set_search_splits(int(splits)))


def search_splits():
    return int(lib().knnag_get_search_splits())


def debug_set_search_stall(visit, wait_spins=0):
    """Test hook of the search's bounded waits (knnag_debug_set_search_stall):
    visit >= 0 never issues that visit's tile copy, so the waits time out;
    (-1, 0) restores normal operation."""
    _check(lib().knnag_debug_set_search_stall(int(visit), int(wait_spins)))


def read_device_status(workspace, device):
    """knnag_read_device_status of a workspace: 0 or 7 (KNNAG_ERR_DEVICE)."""
    with torch.cuda.device(device):
        return int(lib().knnag_read_device_status(_p(workspace), _stream(device)))
