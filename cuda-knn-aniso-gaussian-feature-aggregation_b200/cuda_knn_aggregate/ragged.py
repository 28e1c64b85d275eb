"""Ragged batches over resident point clouds (FP32), through the C ABI.

The reference op takes one uniform batch per call
(``cuda_knn_aggregate/__init__.py:6-32``), so clouds of different sizes are a
host loop of calls.  Here:

* ``CloudSet`` keeps C clouds (p, sigma, R, f concatenated in cloud order)
  resident on the device together with their search index (packed records,
  Hilbert-sorted tiles, tile key bounds) and the per-point row sums of f,
  built once and rebuilt in place when the geometry or the features change.
* A segment table lists the query sets of one call: segment s has Q_s queries
  against cloud ``cloud_s`` with K_s neighbours.  ``ragged_forward`` runs all
  of them in one launch sequence; per segment the result is bit-identical to
  the uniform op on that cloud and query set.
* ``RaggedExecutor`` is a fixed-capacity step (forward, optionally grad_q)
  captured once in a CUDA graph and replayed on any table within its
  capacity; only the query rows and the table are copied in per step.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import capi

# search launch shapes (the C ABI's `splits` code): 1, 2, 4 -> 4, 2, 1 warps of
# 32 queries per CTA; 8 -> 2 warps of 16; 16 -> 4 warps of 8; 32 -> 1 warp of
# 16; 64 -> 1 warp of 8
_SPLITS = (1, 2, 4, 8, 16, 32, 64)


def _i32(xs):
    xs = [int(x) for x in xs]
    return (ctypes.c_int * len(xs))(*xs)


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _check(rc):
    if rc != 0:
        raise RuntimeError(capi.lib().knnag_status_string(rc).decode())


def _f32(t, name, shape_tail):
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if t.dtype != torch.float32:
        raise TypeError(f"{name} must be float32 (ragged calls are FP32)")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")
    if tuple(t.shape[1:]) != tuple(shape_tail):
        raise ValueError(f"{name} must have shape [N, {', '.join(map(str, shape_tail))}]")
    return t


class CloudSet:
    """C resident clouds and their search index.

    ``p [sum P, 3]``, ``sigma [sum P, 3]``, ``R [sum P, 3, 3]``, ``f [sum P, F]``
    (FP32, contiguous, one device), cloud c = rows ``offsets[c]:offsets[c+1]``.
    The tensors are kept by reference: after changing p, sigma or R in place,
    call ``build()`` (kernels only, capturable in a CUDA graph)."""

    def __init__(self, p, sigma, R, f, sizes):
        sizes = [int(s) for s in sizes]
        if not sizes or min(sizes) < 1:
            raise ValueError("every cloud needs at least one point")
        n = sum(sizes)
        self.p = _f32(p, "p", (3,))
        self.sigma = _f32(sigma, "sigma", (3,))
        self.R = _f32(R, "R", (3, 3))
        if f.dim() != 2:
            raise ValueError("f must have shape [sum P, F]")
        self.f = _f32(f, "f", (f.shape[1],))
        for t, name in ((p, "p"), (sigma, "sigma"), (R, "R"), (f, "f")):
            if t.shape[0] != n:
                raise ValueError(f"{name} must have sum(sizes) = {n} rows")
            if t.device != p.device:
                raise RuntimeError("all tensors must be on one device")
        self.device = p.device
        self.sizes = sizes
        self.C = len(sizes)
        self.F = int(f.shape[1])
        self.max_points = max(sizes)
        self.offsets = [0]
        for s in sizes:
            self.offsets.append(self.offsets[-1] + s)
        self._P = _i32(sizes)
        L = capi.lib()
        nb = L.knnag_cloudset_bytes(self.C, self._P)
        if nb == 0:
            raise ValueError("cloud set too large for 32-bit point indexing")
        self.buf = torch.empty(nb, dtype=torch.uint8, device=self.device)
        self._ws = torch.empty(max(1, L.knnag_cloudset_build_workspace_bytes(self.C, self._P)), dtype=torch.uint8,
                               device=self.device)
        self.f_row_sums = torch.empty(n, device=self.device)
        with torch.cuda.device(self.device):
            _check(L.knnag_cloudset_init(self.C, self._P, _ptr(self.buf), nb, _stream(self.device)))
            self.build()
            self.features_changed()

    @classmethod
    def from_clouds(cls, clouds):
        """From a list of (p [P,3], sigma [P,3], R [P,3,3], f [P,F]) device tensors."""
        cat = [torch.cat([c[i].float() for c in clouds]).contiguous() for i in range(4)]
        return cls(*cat, [c[0].shape[0] for c in clouds])

    def build(self):
        """(Re)build the records and the search index from p, sigma, R."""
        _check(capi.lib().knnag_cloudset_build(_ptr(self.p), _ptr(self.sigma), _ptr(self.R), self.C, self._P,
                                               _ptr(self.buf), self.buf.numel(), _ptr(self._ws), self._ws.numel(),
                                               _stream(self.device)))

    def features_changed(self):
        """Recompute the per-point feature row sums d(sum f_out)/dq uses
        (call after changing f in place; capturable)."""
        _check(capi.lib().knnag_feature_row_sums(_ptr(self.f), self.f.shape[0], self.F, capi.F32,
                                                 _ptr(self.f_row_sums), _stream(self.device)))

    def cloud(self, c):
        """(p, sigma, R, f) views of cloud c."""
        a, b = self.offsets[c], self.offsets[c + 1]
        return self.p[a:b], self.sigma[a:b], self.R[a:b], self.f[a:b]

    def nbytes(self):
        return self.buf.numel() + sum(t.numel() * 4 for t in (self.p, self.sigma, self.R, self.f))


def default_splits(total_queries, device=None):
    """Search launch shape by the warps the queries give at 32 per warp (the
    uniform op's rule): many -> 128-query CTAs; few -> fewer queries per
    warp, for more warps."""
    sms = torch.cuda.get_device_properties(device or torch.cuda.current_device()).multi_processor_count \
        if torch.cuda.is_available() else 148
    warps32 = (int(total_queries) + 31) // 32
    if warps32 >= 16 * sms:
        return 1
    if warps32 >= 4 * sms:
        return 8
    return 16


class SegmentTable:
    """Host encoding (pinned) of a segment table and its device copy, for up
    to ``cap_segments`` segments."""

    def __init__(self, cap_segments, device):
        self.cap = int(cap_segments)
        nb = capi.lib().knnag_segments_bytes(self.cap)
        self.host = torch.empty(nb, dtype=torch.uint8, pin_memory=torch.cuda.is_available())
        self.dev = torch.empty(nb, dtype=torch.uint8, device=device)
        self.nseg = 0
        self.nbytes = 0

    def encode(self, cloudset, clouds, Qs, Ks, want_grad=None, splits=1):
        n = len(clouds)
        if n < 1 or n > self.cap or len(Qs) != n or len(Ks) != n:
            raise ValueError(f"1..{self.cap} segments with one Q and one K each")
        wg = None if want_grad is None else _i32([1 if w else 0 for w in want_grad])
        _check(capi.lib().knnag_segments_encode(n, _i32(clouds), _i32(Qs), _i32(Ks), wg, cloudset.C, cloudset._P,
                                                int(splits), _ptr(self.host), self.host.numel()))
        self.nseg = n
        self.nbytes = capi.lib().knnag_segments_bytes(n)

    def upload(self):
        """Copy the encoded bytes to the device on the current stream (the
        pinned host buffer must not be re-encoded until the copy has run)."""
        self.dev[: self.nbytes].copy_(self.host[: self.nbytes], non_blocking=True)


@dataclass
class RaggedResult:
    """Outputs of a ragged call: f_out [sum Q, F] and w_out / dists / idxs
    flat [sum Q K] (segment s at ``e_off[s]``, row-major [Q_s, K_s]); dq
    [sum Q, 3] where computed."""
    f_out: torch.Tensor
    w_out: torch.Tensor
    dists: torch.Tensor
    idxs: torch.Tensor
    Qs: list
    Ks: list
    q_off: list
    e_off: list
    dq: torch.Tensor | None = None

    def segment(self, s):
        """(f_out [Q,F], w_out [Q,K], dists [Q,K], idxs [Q,K]) of segment s."""
        a, Q, K, e = self.q_off[s], self.Qs[s], self.Ks[s], self.e_off[s]
        v = lambda t: t[e: e + Q * K].view(Q, K)
        return self.f_out[a: a + Q], v(self.w_out), v(self.dists), v(self.idxs)


def _offsets(Qs, Ks):
    q_off, e_off, a, e = [], [], 0, 0
    for Q, K in zip(Qs, Ks):
        q_off.append(a)
        e_off.append(e)
        a += Q
        e += Q * K
    return q_off, e_off, a, e


def ragged_forward(cloudset: CloudSet, q, clouds, Qs, Ks, splits=None, grad_q=None, grad_f_out=None):
    """Forward of every segment (eager).  q [sum Q, 3] FP32 on the cloud
    set's device, segment s = rows ``q_off[s]:q_off[s]+Qs[s]`` against cloud
    ``clouds[s]`` with ``Ks[s]`` neighbours.  ``grad_q`` (list of bools, the
    True ones first) also computes dq = d<grad_f_out, f_out>/dq for those
    segments (grad_f_out None: all ones)."""
    Qs, Ks, clouds = [int(x) for x in Qs], [int(x) for x in Ks], [int(c) for c in clouds]
    q_off, e_off, total_q, total_e = _offsets(Qs, Ks)
    _f32(q, "q", (3,))
    if q.shape[0] != total_q:
        raise ValueError(f"q must have sum(Qs) = {total_q} rows")
    dev = cloudset.device
    splits = splits or default_splits(total_q, dev)
    table = SegmentTable(len(clouds), dev)
    table.encode(cloudset, clouds, Qs, Ks, grad_q, splits)
    F = cloudset.F
    f_out = torch.empty(max(total_q, 1), F, device=dev)[:total_q]
    w_out = torch.empty(max(total_e, 1), device=dev)[:total_e]
    dists = torch.empty(max(total_e, 1), device=dev)[:total_e]
    idxs = torch.empty(max(total_e, 1), dtype=torch.int64, device=dev)[:total_e]
    L = capi.lib()
    cap_q = max(total_q, 1)
    ws = torch.empty(L.knnag_ragged_workspace_bytes(len(clouds), cap_q), dtype=torch.uint8, device=dev)
    max_k = max(Ks)
    with torch.cuda.device(dev):
        table.upload()
        st = _stream(dev)
        qp = q if total_q else torch.empty(1, 3, device=dev)
        _check(L.knnag_ragged_forward(_ptr(cloudset.buf), _ptr(table.dev), _ptr(qp), _ptr(cloudset.f), F, len(clouds),
                                      cap_q, max(total_e, 1), max_k, cloudset.max_points, splits, _ptr(f_out),
                                      _ptr(w_out), _ptr(dists), _ptr(idxs), _ptr(ws), ws.numel(), st))
        res = RaggedResult(f_out, w_out, dists, idxs, Qs, Ks, q_off, e_off)
        if grad_q is not None and any(grad_q):
            dq = torch.zeros(max(total_q, 1), 3, device=dev)[:total_q]
            gws = torch.empty(256, dtype=torch.uint8, device=dev)
            _check(L.knnag_ragged_grad_q(_ptr(cloudset.buf), _ptr(table.dev), _ptr(qp), _ptr(cloudset.f), F,
                                         _ptr(grad_f_out), None if grad_f_out is not None else _ptr(cloudset.f_row_sums),
                                         _ptr(idxs), len(clouds), cap_q, max(total_e, 1), max_k,
                                         cloudset.max_points, _ptr(dq), _ptr(gws), gws.numel(), st))
            res.dq = dq
        # the pinned table must outlive the asynchronous copy
        torch.cuda.current_stream(dev).synchronize()
        rc = L.knnag_read_device_status(_ptr(ws), st)
        _check(rc)
    return res


# ---------------------------------------------------------------- autotuner


def shape_bucket(cloudset: CloudSet, Qs, Ks):
    """Shape bucket of a ragged step: log2 of the largest cloud, of the step's
    total queries and of its mean segment size, and the K register bucket."""
    total = max(1, sum(int(q) for q in Qs))
    kmax = max(int(k) for k in Ks)
    kb = 8 if kmax <= 8 else 16 if kmax <= 16 else 32 if kmax <= 32 else 64
    return (int(cloudset.max_points).bit_length(), total.bit_length(), max(1, total // len(Qs)).bit_length(), kb)


def autotune_splits(cloudset: CloudSet, clouds, qs, Ks, reps=3, cache=True):
    """Search launch shape (queries per CTA and per warp, the ``splits`` codes
    1, 2, 4, 8, 16, 32, 64) for steps shaped like this one: each candidate runs the step as a captured graph
    ``reps`` times (after a warm-up) and the fastest median wins.  Cached per
    ``shape_bucket`` in memory and in the tuner's JSON file
    (``tuning.cache_path()``), so a later process reuses the choice."""
    from . import tuning

    Qs = [int(x.shape[0]) for x in qs]
    bucket = shape_bucket(cloudset, Qs, Ks)
    dev = cloudset.buf.device
    if cache:
        hit = tuning.lookup("ragged", bucket, dev)
        if hit is not None:
            return int(hit["splits"])
    times = {}
    for g in _SPLITS:
        ex = RaggedExecutor(cloudset, len(clouds), sum(Qs), max(Ks), splits=g, copy_out=False)
        ex.submit(clouds, qs, Ks)
        ex.result()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(ex.stream):
                e0.record()
                ex.graph.replay()
                e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        times[g] = sorted(ts)[len(ts) // 2]
        tuning.TIMED["runs"] += 1
        del ex
    best = min(times, key=times.get)
    tuning.record("ragged", bucket, {"splits": best, "ms": {str(g): t for g, t in times.items()}}, dev)
    return best


def tune_cache():
    """The autotuner's choices known to this process (both tuners)."""
    from . import tuning

    return tuning.tune_cache()


class RaggedExecutor:
    """Fixed-capacity ragged step (forward, and dq for the segments that ask)
    captured in a CUDA graph on its own stream.

    ``submit(clouds, qs, Ks, want_grad)`` stages the query rows (host or
    device tensors) and the encoded table, replays the step and starts the
    device-to-host copies of f_out (and dq); ``done()`` polls and
    ``result()`` waits.  Capacities: ``cap_segments`` segments, ``cap_queries``
    queries, ``max_k`` neighbours per query."""

    def __init__(self, cloudset: CloudSet, cap_segments, cap_queries, max_k, splits=None, graph=True,
                 copy_out=True):
        self.cs = cloudset
        dev = cloudset.device
        self.dev = dev
        self.cap_segments, self.cap_q, self.max_k = int(cap_segments), int(cap_queries), int(max_k)
        self.cap_e = self.cap_q * self.max_k
        self.splits = splits or default_splits(self.cap_q, dev)
        F = cloudset.F
        L = capi.lib()
        pin = torch.cuda.is_available()
        self.q_host = torch.empty(self.cap_q, 3, pin_memory=pin)
        self.q_dev = torch.empty(self.cap_q, 3, device=dev)
        self.f_out = torch.empty(self.cap_q, F, device=dev)
        self.w_out = torch.empty(self.cap_e, device=dev)
        self.dists = torch.empty(self.cap_e, device=dev)
        self.idxs = torch.empty(self.cap_e, dtype=torch.int64, device=dev)
        self.dq = torch.zeros(self.cap_q, 3, device=dev)
        self.copy_out = copy_out
        self.f_host = torch.empty(self.cap_q, F, pin_memory=pin) if copy_out else None
        self.dq_host = torch.empty(self.cap_q, 3, pin_memory=pin) if copy_out else None
        self.table = SegmentTable(self.cap_segments, dev)
        self.ws = torch.empty(L.knnag_ragged_workspace_bytes(self.cap_segments, self.cap_q), dtype=torch.uint8,
                              device=dev)
        self.gws = torch.empty(256, dtype=torch.uint8, device=dev)
        self.stream = torch.cuda.Stream(dev)
        self.event = torch.cuda.Event()
        self.graph = None
        self.pending = None
        self.launches_per_step = None
        # a valid table for warm-up and capture: one segment of one query
        self._encode([0], [1], [min(self.max_k, cloudset.sizes[0])], [True])
        self.q_dev.zero_()
        with torch.cuda.device(dev), torch.cuda.stream(self.stream):
            self.table.upload()
            for _ in range(2):
                self._kernels()
        self.stream.synchronize()
        if graph:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.device(dev), torch.cuda.graph(g, stream=self.stream):
                c0 = capi.launch_count()
                self._kernels()
                self.launches_per_step = capi.launch_count() - c0
            self.graph = g
        self.stream.synchronize()

    def _encode(self, clouds, Qs, Ks, want_grad):
        self.table.encode(self.cs, clouds, Qs, Ks, want_grad, self.splits)
        self.meta = (list(Qs), list(Ks)) + _offsets(Qs, Ks)[:2]

    def _kernels(self):
        L = capi.lib()
        st = ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)
        _check(L.knnag_ragged_forward(_ptr(self.cs.buf), _ptr(self.table.dev), _ptr(self.q_dev), _ptr(self.cs.f),
                                      self.cs.F, self.cap_segments, self.cap_q, self.cap_e, self.max_k,
                                      self.cs.max_points, self.splits, _ptr(self.f_out), _ptr(self.w_out),
                                      _ptr(self.dists), _ptr(self.idxs), _ptr(self.ws), self.ws.numel(), st))
        _check(L.knnag_ragged_grad_q(_ptr(self.cs.buf), _ptr(self.table.dev), _ptr(self.q_dev), _ptr(self.cs.f),
                                     self.cs.F, None, _ptr(self.cs.f_row_sums), _ptr(self.idxs), self.cap_segments,
                                     self.cap_q, self.cap_e,
                                     self.max_k, self.cs.max_points, _ptr(self.dq), _ptr(self.gws), self.gws.numel(),
                                     st))

    def submit(self, clouds, qs, Ks, want_grad=None, outs=None):
        """Start one step.  Segments wanting dq are moved first; ``order``
        (returned by result) maps table position -> caller's index.  ``outs``
        (optional, caller's order): per segment a pair of host tensors
        (f_dst [Q, F], dq_dst [Q, 3] or None) that receive the segment's
        f_out / dq by device-to-host copies inside the step; without it the
        whole f_out (and dq) range is copied to f_host / dq_host."""
        if self.pending is not None:
            raise RuntimeError("previous step not collected")
        n = len(clouds)
        wg = [bool(w) for w in (want_grad or [False] * n)]
        # segments wanting dq first (the table's dq prefix); within each
        # group the heaviest (cloud size x K) first, so the persistent search
        # starts the long work items early and the tail is short
        sizes = self.cs.sizes
        order = sorted(range(n), key=lambda i: (not wg[i], -sizes[int(clouds[i])] * int(Ks[i])))
        clouds = [int(clouds[i]) for i in order]
        qs = [qs[i] for i in order]
        Ks = [int(Ks[i]) for i in order]
        wg = [wg[i] for i in order]
        outs = None if outs is None else [outs[i] for i in order]
        Qs = [int(x.shape[0]) for x in qs]
        total = sum(Qs)
        if total > self.cap_q or n > self.cap_segments or max(Ks) > self.max_k:
            raise ValueError("step exceeds the executor's capacity")
        self._encode(clouds, Qs, Ks, wg)
        q_off = self.meta[2]
        with torch.cuda.stream(self.stream):
            # device or pinned sources go straight to the device; pageable
            # ones through the pinned staging buffer
            on_host = [not x.is_cuda and not x.is_pinned() for x in qs]
            for i, x in enumerate(qs):
                rows = slice(q_off[i], q_off[i] + Qs[i])
                if on_host[i]:
                    self.q_host[rows].copy_(x)
                else:
                    self.q_dev[rows].copy_(x, non_blocking=True)
            if all(on_host):
                self.q_dev[:total].copy_(self.q_host[:total], non_blocking=True)
            elif any(on_host):
                for i in (i for i in range(n) if on_host[i]):
                    rows = slice(q_off[i], q_off[i] + Qs[i])
                    self.q_dev[rows].copy_(self.q_host[rows], non_blocking=True)
            self.table.upload()
            if self.graph is not None:
                self.graph.replay()
            else:
                self._kernels()
            if outs is not None:
                for i, (fd, dd) in enumerate(outs):
                    rows = slice(q_off[i], q_off[i] + Qs[i])
                    if fd is not None:
                        fd.copy_(self.f_out[rows], non_blocking=True)
                    if dd is not None and wg[i]:
                        dd.copy_(self.dq[rows], non_blocking=True)
            elif self.copy_out:
                self.f_host[:total].copy_(self.f_out[:total], non_blocking=True)
                g = sum(Q for Q, w in zip(Qs, wg) if w)
                if g:
                    self.dq_host[:g].copy_(self.dq[:g], non_blocking=True)
            self.event.record(self.stream)
        self.pending = (order, wg)
        return self

    def done(self):
        return self.pending is None or self.event.query()

    def result(self):
        """Wait for the step; returns (order, RaggedResult) with device
        outputs (and, when copy_out, host copies f_host / dq_host)."""
        self.event.synchronize()
        order, wg = self.pending
        self.pending = None
        Qs, Ks, q_off, e_off = self.meta
        t = sum(Qs)
        e = sum(Q * K for Q, K in zip(Qs, Ks))
        res = RaggedResult(self.f_out[:t], self.w_out[:e], self.dists[:e], self.idxs[:e], Qs, Ks, q_off, e_off,
                           self.dq[:t])
        return order, wg, res

    def check_status(self):
        """Raise if the device latched an error (validation or a timed-out wait)."""
        with torch.cuda.device(self.dev):
            _check(capi.lib().knnag_read_device_status(_ptr(self.ws), _stream(self.dev)))
            _check(capi.lib().knnag_read_device_status(_ptr(self.gws), _stream(self.dev)))
