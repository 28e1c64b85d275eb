"""Autotuner of the uniform op's search split (warps per 32-query group).

Each candidate (1, 2, 4) runs the forward on the caller's inputs; the
fastest median of CUDA-event timings wins and is cached per shape bucket
(batch size, log2 of Q and P, K register bucket).  ``use_tuned`` applies the
cached choice process-wide through the C ABI (``knnag_set_search_splits``);
results never depend on it, only the time.  The ragged path has its own
tuner (``ragged.autotune_splits``).
"""
from __future__ import annotations

import torch

from . import capi

_CACHE: dict = {}


def shape_bucket(B, Q, P, K):
    kb = 8 if K <= 8 else 16 if K <= 16 else 32 if K <= 32 else 64
    return (int(B), int(Q).bit_length(), int(P).bit_length(), kb)


def autotune_search_splits(q, p, f, sigma, R, K, reps=5, cache=True):
    """Best split for inputs shaped like these (CUDA tensors of the op)."""
    from . import _C

    key = shape_bucket(q.shape[0], q.shape[1], p.shape[1], K)
    if cache and key in _CACHE:
        return _CACHE[key]
    prev = capi.search_splits()
    times = {}
    try:
        for g in (1, 2, 4):
            capi.set_search_splits(g)
            with torch.no_grad():
                for _ in range(2):
                    _C.knn_aggregate_aniso_forward(q, p, f, sigma, R, int(K))
                ts = []
                for _ in range(reps):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    _C.knn_aggregate_aniso_forward(q, p, f, sigma, R, int(K))
                    e1.record()
                    e1.synchronize()
                    ts.append(e0.elapsed_time(e1))
            times[g] = sorted(ts)[len(ts) // 2]
    finally:
        capi.set_search_splits(prev)
    best = min(times, key=times.get)
    _CACHE[key] = best
    return best


def use_tuned(q, p, K):
    """Apply the cached split of this shape bucket (automatic if none)."""
    capi.set_search_splits(_CACHE.get(shape_bucket(q.shape[0], q.shape[1], p.shape[1], K), 0))


def tune_cache():
    return dict(_CACHE)
