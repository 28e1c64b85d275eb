"""Autotuner of the search's launch shape, cached per shape bucket on disk.

The tuned knobs change only the time, never a result:

* ``splits``, the search launch shape (the C ABI's
  ``knnag_set_search_splits``): 1, 2, 4 -> 4, 2, 1 warps of 32 queries per
  CTA; 8 -> 2 warps of 16 queries; 16 -> 4 warps of 8; 32 -> 1 warp of 16;
  64 -> 1 warp of 8 -- queries per CTA and per warp; 128 -> the tensor-core
  filtered search (128 queries per CTA, two threads per query);
* the K register layout: the list length is the K bucket (8, 16, 32) --
  part of the shape bucket, not a free knob.

``autotune_search(...)`` times every candidate on the caller's inputs (the
median of CUDA-event timings of the forward) and keeps the fastest, keyed by
``shape_bucket`` -- batch size, log2 of Q and P, and the K bucket -- under
the device name and the library version.  Choices are kept in memory and
in a JSON file: ``$KNNAG_TUNE_CACHE`` if set, else
``~/.cache/cuda_knn_aggregate/tune.json``.  A later process with the same
device, library and bucket reads the choice from the file and times
nothing.  ``use_tuned`` applies the cached choice process-wide.

The ragged path has its own tuner (``ragged.autotune_splits``), keyed by its
own bucket, sharing the file.
"""
from __future__ import annotations

import json
import os
import tempfile

import torch

from . import capi

SPLITS = (1, 2, 4, 8, 16, 32, 64, 128)
_CACHE: dict = {}      # in-memory: full key -> choice dict
_LOADED: set = set()   # files already read into _CACHE
TIMED = {"runs": 0}    # number of candidate timings made in this process


def cache_path() -> str:
    env = os.environ.get("KNNAG_TUNE_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "cuda_knn_aggregate", "tune.json")


def _device_tag(device=None) -> str:
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    return f"{torch.cuda.get_device_name(dev)}|lib{capi.lib().knnag_version()}"


def shape_bucket(B, Q, P, K):
    kb = 8 if K <= 8 else 16 if K <= 16 else 32 if K <= 32 else 64
    return (int(B), int(Q).bit_length(), int(P).bit_length(), kb)


def _key(kind, bucket, device=None) -> str:
    return f"{_device_tag(device)}|{kind}|{','.join(str(x) for x in bucket)}"


def _load(path=None):
    path = path or cache_path()
    if path in _LOADED:
        return
    _LOADED.add(path)
    try:
        with open(path) as fh:
            data = json.load(fh)
        if isinstance(data, dict):
            for k, v in data.items():
                _CACHE.setdefault(k, v)
    except (OSError, ValueError):
        pass


def _store(key, choice, path=None):
    """Record a choice in memory and merge it into the JSON file (written
    atomically: a temporary file renamed over the old one)."""
    path = path or cache_path()
    _CACHE[key] = choice
    try:
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        try:
            with open(path) as fh:
                data = json.load(fh)
            if not isinstance(data, dict):
                data = {}
        except (OSError, ValueError):
            data = {}
        data[key] = choice
        fd, tmp = tempfile.mkstemp(dir=os.path.dirname(path) or ".", prefix=".tune.")
        with os.fdopen(fd, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # an unwritable cache location costs a re-tune later, nothing else


def lookup(kind, bucket, device=None):
    """The cached choice for (kind, bucket) on this device, or None."""
    _load()
    return _CACHE.get(_key(kind, bucket, device))


def record(kind, bucket, choice, device=None):
    _store(_key(kind, bucket, device), choice)


def _median_ms(fn, reps):
    for _ in range(2):
        fn()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    TIMED["runs"] += 1
    return sorted(ts)[len(ts) // 2]


def autotune_search(q, p, f, sigma, R, K, reps=5, cache=True):
    """Best launch shape {"splits": s} for inputs shaped like these (CUDA
    tensors of the op): read from the cache when this bucket was tuned on
    this device before, else timed and recorded."""
    from . import _C

    bucket = shape_bucket(q.shape[0], q.shape[1], p.shape[1], K)
    if cache:
        hit = lookup("uniform", bucket, q.device)
        if hit is not None:
            return dict(hit)
    prev = capi.search_splits()
    times = {}
    try:
        with torch.no_grad():
            for g in SPLITS:
                capi.set_search_splits(g)
                times[g] = _median_ms(lambda: _C.knn_aggregate_aniso_forward(q, p, f, sigma, R, int(K)), reps)
    finally:
        capi.set_search_splits(prev)
    best = {"splits": min(times, key=times.get), "ms": {str(g): t for g, t in times.items()}}
    record("uniform", bucket, best, q.device)
    return dict(best)


def autotune_search_splits(q, p, f, sigma, R, K, reps=5, cache=True):
    """The tuned ``splits`` alone (see autotune_search)."""
    return int(autotune_search(q, p, f, sigma, R, K, reps, cache)["splits"])


def use_tuned(q, p, K):
    """Apply the cached choice of this shape bucket process-wide (the
    automatic choice if the bucket was never tuned)."""
    hit = lookup("uniform", shape_bucket(q.shape[0], q.shape[1], p.shape[1], K), q.device)
    capi.set_search_splits(int(hit["splits"]) if hit else 0)


def tune_cache():
    """Every choice known to this process: {key: choice}."""
    _load()
    return dict(_CACHE)
