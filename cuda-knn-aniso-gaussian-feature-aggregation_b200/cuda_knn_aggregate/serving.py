"""Continuous-batching request loop over resident clouds.

Requests (a query set against one resident cloud, K neighbours, optionally
d(sum f_out)/dq) arrive over time.  The server owns ``inflight`` ragged
executors (each a captured CUDA graph on its own stream, ``ragged.py``);
whenever one is free it takes the queued work first-come first-served --
as many request chunks as fit its query and segment capacity -- and
launches it, while the steps already launched keep running on the device.
A request larger than one step is split into chunks; it completes when its
last chunk's outputs have reached its host buffers.  Memory is admitted
against budgets: on the device, the resident clouds plus every executor's
buffers must fit the HBM budget, which fixes the step capacity; on the host,
request outputs live in a pinned ring of fixed size, and an arrived request
waits until the ring has room for its outputs (space comes back as requests
complete and their outputs are released).

Latency of a request = completion time (its last chunk's step observed done
by the host loop, outputs already copied to host memory) - arrival time.
"""
from __future__ import annotations

import collections
import math
import statistics
import time
from dataclasses import dataclass, field

import torch

from .ragged import CloudSet, RaggedExecutor, autotune_splits


class PinnedRing:
    """FIFO arena of pinned host memory: ``alloc`` takes the next free run
    (wrapping at the end), ``free`` releases in any order and the space is
    reclaimed from the oldest allocation on.  Returns None when full."""

    def __init__(self, nbytes):
        self.cap = int(nbytes)
        self.buf = torch.empty(self.cap, dtype=torch.uint8, pin_memory=torch.cuda.is_available())
        self.live = collections.deque()  # [offset, size, freed]
        self.head = 0                    # next offset to hand out

    def alloc(self, nbytes):
        n = (int(nbytes) + 255) // 256 * 256
        if n > self.cap:
            return None
        if not self.live:
            self.head = 0
            off = 0
        else:
            tail = self.live[0][0]
            wrapped = self.live[-1][0] < tail  # the newest run lies below the oldest
            if not wrapped:              # free space: [head, cap) and [0, tail)
                if self.head + n <= self.cap:
                    off = self.head
                elif n <= tail:
                    off = 0
                else:
                    return None
            else:                        # free space: [head, tail)
                if self.head + n <= tail:
                    off = self.head
                else:
                    return None
        self.live.append([off, n, False])
        self.head = off + n
        return off

    def free(self, off):
        for e in self.live:
            if e[0] == off and not e[2]:
                e[2] = True
                break
        while self.live and self.live[0][2]:
            self.live.popleft()

    def view(self, off, shape):
        n = 4
        for d in shape:
            n *= d
        return self.buf[off: off + n].view(torch.float32).view(*shape)


@dataclass
class Request:
    cloud: int
    q: torch.Tensor          # [Q, 3] float32 (host; pinned is faster)
    K: int = 16
    want_grad: bool = False
    arrival: float = 0.0     # seconds after the run starts
    done: float | None = None
    f_out: torch.Tensor | None = None   # [Q, F] host, filled on completion
    dq: torch.Tensor | None = None      # [Q, 3] host when want_grad
    chunks_left: int = 0

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival


@dataclass
class ServeStats:
    n_requests: int
    queries: int
    seconds: float
    latencies_ms: list = field(repr=False)
    steps: int = 0
    mean_segments_per_step: float = 0.0
    mean_queries_per_step: float = 0.0

    @property
    def throughput(self):
        return self.queries / self.seconds if self.seconds > 0 else 0.0

    def pct(self, p):
        xs = sorted(self.latencies_ms)
        if not xs:
            return None
        i = min(len(xs) - 1, max(0, math.ceil(p / 100.0 * len(xs)) - 1))
        return xs[i]

    def summary(self):
        return {"requests": self.n_requests, "queries": self.queries, "seconds": self.seconds,
                "throughput_qps": self.throughput, "p50_ms": self.pct(50), "p99_ms": self.pct(99),
                "mean_ms": statistics.mean(self.latencies_ms) if self.latencies_ms else None,
                "steps": self.steps, "mean_segments_per_step": self.mean_segments_per_step,
                "mean_queries_per_step": self.mean_queries_per_step}


def step_bytes_per_query(F, max_k):
    """Device bytes one query of step capacity costs: q, f_out, dq, w_out,
    dists, idxs, and the forward workspace (flag list, query order, cells)."""
    return 12 + 4 * F + 12 + max_k * (4 + 4 + 8) + 4 + 4 + 8


class Server:
    def __init__(self, cloudset: CloudSet, hbm_budget_bytes=40e9, max_k=16, step_queries=1 << 20, inflight=3,
                 cap_segments=256, splits=None, graph=True, host_budget_bytes=2e9, tune_requests=None):
        """``splits``: the search launch shape (1, 2, 4, 8, 16; see ``tuning``), or
        "auto" to let the autotuner time the candidates on one step packed
        from ``tune_requests``."""
        self.cs = cloudset
        self.max_k = int(max_k)
        per_q = step_bytes_per_query(cloudset.F, self.max_k)
        room = int(hbm_budget_bytes) - cloudset.nbytes()
        fit = room // (inflight * per_q)
        if fit < 1024:
            raise ValueError("the HBM budget does not hold the resident clouds plus the step buffers")
        self.step_queries = int(min(step_queries, fit))
        self.cap_segments = int(cap_segments)
        if splits == "auto":
            if not tune_requests:
                raise ValueError("splits='auto' needs tune_requests")
            take, tot = [], 0
            for r in tune_requests:
                Q = int(min(r.q.shape[0], self.step_queries - tot))
                if Q < 1 or len(take) == self.cap_segments:
                    break
                take.append((r, Q))
                tot += Q
            splits = autotune_splits(cloudset, [r.cloud for r, _ in take],
                                     [r.q[:Q].to(cloudset.device) for r, Q in take], [r.K for r, _ in take])
        self.splits = splits
        self.execs = [RaggedExecutor(cloudset, cap_segments, self.step_queries, self.max_k, splits=splits,
                                     graph=graph, copy_out=False) for _ in range(inflight)]
        self.splits = self.execs[0].splits
        self.device_bytes = cloudset.nbytes() + inflight * per_q * self.step_queries
        self.ring = PinnedRing(host_budget_bytes)

    def run(self, requests, keep_outputs=True, clock=time.perf_counter, time_limit=None):
        """Serve ``requests`` (sorted by arrival) in real time; returns ServeStats.
        With keep_outputs False, each request's host buffers are released once
        it completes (only its latency is kept)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        F = self.cs.F
        pin = torch.cuda.is_available()
        queue = collections.deque()           # (request, row0, row1)
        busy = {}                             # executor index -> list of chunks
        slots = {}                            # request id -> ring offsets of its outputs
        nxt = 0
        done_count = 0
        lat = []
        steps = segs = qsum = 0
        t0 = clock()
        last_done = t0
        while done_count < len(reqs):
            now = clock() - t0
            if time_limit is not None and now > time_limit:
                break
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                r = reqs[nxt]
                Q = int(r.q.shape[0])
                if keep_outputs:
                    r.f_out = torch.empty(Q, F, pin_memory=pin)
                    r.dq = torch.empty(Q, 3, pin_memory=pin) if r.want_grad else None
                else:
                    # outputs in the pinned ring; wait for room (admission)
                    fo = self.ring.alloc(Q * F * 4)
                    go = self.ring.alloc(Q * 12) if (fo is not None and r.want_grad) else None
                    if fo is None or (r.want_grad and go is None):
                        if fo is not None:
                            self.ring.free(fo)
                        break
                    slots[id(r)] = (fo, go)
                    r.f_out = self.ring.view(fo, (Q, F))
                    r.dq = self.ring.view(go, (Q, 3)) if r.want_grad else None
                n_chunks = max(1, -(-Q // self.step_queries))
                r.chunks_left = n_chunks
                for c in range(n_chunks):
                    queue.append((r, c * self.step_queries, min(Q, (c + 1) * self.step_queries)))
                nxt += 1
            progressed = False
            # completions
            for i in list(busy):
                ex = self.execs[i]
                if ex.done():
                    ex.result()
                    tdone = clock()
                    for (r, a, b) in busy.pop(i):
                        r.chunks_left -= 1
                        if r.chunks_left == 0:
                            r.done = tdone - t0
                            lat.append((r.done - r.arrival) * 1e3)
                            done_count += 1
                            last_done = tdone
                            if not keep_outputs:
                                r.f_out = r.dq = None
                                for off in slots.pop(id(r)):
                                    if off is not None:
                                        self.ring.free(off)
                    progressed = True
            # admissions: every free executor takes what fits, FIFO
            for i, ex in enumerate(self.execs):
                if i in busy or not queue:
                    continue
                take, total = [], 0
                while queue and len(take) < self.cap_segments:
                    r, a, b = queue[0]
                    if total + (b - a) > self.step_queries:
                        break
                    take.append(queue.popleft())
                    total += b - a
                if not take:
                    continue
                ex.submit([r.cloud for r, _, _ in take], [r.q[a:b] for r, a, b in take], [r.K for r, _, _ in take],
                          [r.want_grad for r, _, _ in take],
                          outs=[(r.f_out[a:b], r.dq[a:b] if r.want_grad else None) for r, a, b in take])
                busy[i] = take
                steps += 1
                segs += len(take)
                qsum += total
                progressed = True
            if not progressed:
                if not busy and not queue and nxt < len(reqs):
                    wait = reqs[nxt].arrival - (clock() - t0)
                    if wait > 2e-4:
                        time.sleep(wait - 1e-4)
                else:
                    time.sleep(2e-5)
        for i in list(busy):
            self.execs[i].result()
        first = reqs[0].arrival if reqs else 0.0
        seconds = (last_done - t0) - first
        return ServeStats(n_requests=done_count, queries=sum(int(r.q.shape[0]) for r in reqs if r.done is not None),
                          seconds=seconds, latencies_ms=lat, steps=steps,
                          mean_segments_per_step=segs / steps if steps else 0.0,
                          mean_queries_per_step=qsum / steps if steps else 0.0)
