"""Benchmark of the knn_aggregate_aniso training step.

One step = forward (fused kNN search + aggregation), dq = d(sum f_out)/dq
with create_graph, Eikonal loss mean((|dq| - 1)^2), backward into q, p, f,
sigma and R -- the forward + first- + second-order path.  Workload: the
reference README's timing-table shape, B=2, Q=12288, P=4096, F=64, K=16,
FP32, seeded synthetic uniform-cube inputs.  One unit = one query.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference|reference-ext]

--impl ours (default): the CUDA path, steps replayed from a CUDA graph with
    inputs resident in HBM, L2 flushed between steps (inputs are smaller than
    L2).  Prints one JSON line with value, e2e (public API with host buffers
    and copies in the timed region), roofline of the search kernel, the CPU
    baseline, clocks and launch counts.
--impl reference: the reference path on this machine's host cores (the
    reference ships no CPU implementation, so the plain-PyTorch CPU
    formulation of the op is timed -- all threads -- on a bounded sample of the
    same workload).
--impl reference-ext: the reference CUDA extension, compiled from its own
    sources, on the same GPU through autograd wiring equivalent to the
    reference's package (eager; it launches on the legacy default stream).

Under torchrun each rank runs its own batch (independent clouds: no
collective on the data path, weak scaling); rank 0 prints the line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "cuda-knn-aniso-gaussian-feature-aggregation_b200")
sys.path.insert(0, PKG_DIR)

METRIC = "fwd+1st+2nd-order queries/s"
UNIT = "queries/s"
WORKLOAD = dict(name="table", B=2, Q=12288, P=4096, F=64, K=16)
FLOP_PER_PAIR = 26          # 3 sub, 3x(1 mul + 2 fma), 3 squares, 1 mul + 2 fma
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, local, backend):
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))


def max_over_ranks(x: float, ws: int, device) -> float:
    if ws == 1:
        return x
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        loaded = [x for x in sm if mx and x > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def workloads_module():
    """cuda_knn_aggregate/workloads.py loaded by file path: it needs only
    torch, and importing it through the package would load the package's
    CUDA extension (which the reference arm must not touch)."""
    import importlib.util

    name = "knnag_bench_workloads"
    if name not in sys.modules:
        path = os.path.join(PKG_DIR, "cuda_knn_aggregate", "workloads.py")
        spec = importlib.util.spec_from_file_location(name, path)
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def make_inputs(rank, device):
    shape, t = workloads_module().make(WORKLOAD["name"], seed=1001 + 7919 * rank)
    return shape, t


def eikonal_step_fn(op, ins, K):
    def step():
        for a in ins:
            a.grad = None
        f_out = op(*ins, K)[0]
        (gq,) = torch.autograd.grad(f_out.sum(), ins[0], create_graph=True)
        loss = ((gq.norm(dim=-1) - 1.0) ** 2).mean()
        loss.backward()
        return loss.detach()

    return step

# ---------------------------------------------------------------- CPU side

def cpu_step_rate(q_per_batch: int, min_seconds: float = 0.0, iters: int | None = None):
    """Plain-PyTorch FP32 formulation of the step on the host cores (all
    threads), on the first q_per_batch queries of each batch element of the
    workload, for exactly `iters` iterations or, when iters is None, until
    min_seconds have passed (at least 2); returns (queries/s, iterations,
    seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    torch.set_num_threads(os.cpu_count() or 1)
    shape, t = make_inputs(0, "cpu")
    q = t[0][:, :q_per_batch].contiguous()
    base = [q] + [x.clone() for x in t[1:]]
    fwd = lambda *a: O.plain_forward(*a, chunk=256)
    n, t0 = 0, time.perf_counter()
    while True:
        ins = [x.clone().requires_grad_(True) for x in base]
        O.eikonal_step(*ins, shape.K, forward=fwd)
        n += 1
        el = time.perf_counter() - t0
        if (iters is not None and n >= iters) or (iters is None and el >= min_seconds and n >= 2):
            break
    return shape.B * q_per_batch * n / el, n, el, torch.get_num_threads()


def cpu_baseline_block(seconds=12.0, q_per_batch=2048):
    rate, n, el, thr = cpu_step_rate(q_per_batch, seconds)
    return {"value": rate, "unit": UNIT, "cores": thr, "kind": "port",
            "sample": f"plain-PyTorch FP32 step (oracle/oracle.py) on {q_per_batch} of 12288 queries per batch "
                      f"element, full P=4096, {n} iterations in {el:.1f} s"}


# ------------------------------------------------------------ reference ext

def ref_ext():
    """The reference extension (compiled from its own sources) with the
    reference package's autograd wiring: (module, op) or (None, reason)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_ext as RX

    mod, why = RX.load()
    if mod is None:
        return None, why
    return mod, RX.op(mod)


def load_reference_ext():
    mod, why = ref_ext()
    return (mod, None) if mod is not None else (None, why)


def e2e_times(op, host, K, device, steps, warmup, flush):
    """Per-step ms of the Eikonal step through `op` from pinned host inputs:
    H2D copies, the step, and the D2H read of the loss inside each timed
    region (CUDA events on the current stream)."""
    loss_h = torch.empty((), dtype=torch.float32).pin_memory()
    out = []
    for i in range(warmup + steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dev_in = [x.to(device, non_blocking=True).requires_grad_(True) for x in host]
        f_out = op(*dev_in, K)[0]
        (gq,) = torch.autograd.grad(f_out.sum(), dev_in[0], create_graph=True)
        loss = ((gq.norm(dim=-1) - 1.0) ** 2).mean()
        loss.backward()
        loss_h.copy_(loss.detach(), non_blocking=True)
        e1.record()
        e1.synchronize()
        if i >= warmup:
            out.append(e0.elapsed_time(e1))
    return out, loss_h.element_size()


def time_reference_ext(device, steps, warmup, host=None):
    """The reference extension's Eikonal step on this GPU: device-resident
    inputs (eager; it cannot be graph-captured: it launches on the legacy
    default stream), and, when `host` inputs are given, end to end from
    pinned host buffers as our e2e figure is taken."""
    mod, op = ref_ext()
    if mod is None:
        return {"unavailable": op}
    shape, t = make_inputs(0, device)
    ins = [x.to(device).requires_grad_(True) for x in t]
    step = eikonal_step_fn(op, ins, shape.K)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = statistics.mean(times)
    out = {"value": shape.B * shape.Q / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": steps,
           "how": "reference extension compiled from its own sources (sm_100), reference autograd wiring, eager"}
    if host is not None:
        e2e, _ = e2e_times(op, host, shape.K, device, steps, 1, flush)
        out["e2e_ms_per_step"] = statistics.mean(e2e)
    return out


# ------------------------------------------------------------ ragged / served

def _events():
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def ragged_block(device, steps=10, ref_steps=2, with_reference=True):
    """Ragged batch of 64 clouds (P ~ logU[1024, 32768], Q ~ logU[2048,
    65536], K in {8, 16, 32}, F=64, Gaussian-mixture clouds): one captured
    graph of cloud-set build + ragged forward, against a per-cloud loop of
    the uniform op (one eager call per cloud) and a per-cloud loop of the
    reference extension.  Forward only; L2 flushed between steps."""
    from cuda_knn_aggregate import capi, knn_aggregate_aniso
    from cuda_knn_aggregate import workloads as W
    from cuda_knn_aggregate.ragged import CloudSet, RaggedExecutor, autotune_splits

    rb = W.ragged_batch()
    C = len(rb.sizes)
    p, sigma, R, f, q = [t.to(device) for t in (rb.p, rb.sigma, rb.R, rb.f, rb.q)]
    cs = CloudSet(p, sigma, R, f, rb.sizes)
    total_q = sum(rb.Qs)
    qsegs = [q[a:a + n] for a, n in zip(_prefix(rb.Qs), rb.Qs)]
    splits = autotune_splits(cs, list(range(C)), qsegs, rb.Ks)
    ex = RaggedExecutor(cs, cap_segments=C, cap_queries=total_q, max_k=max(rb.Ks), splits=splits, graph=False,
                        copy_out=False)
    ex.submit(list(range(C)), qsegs, rb.Ks)
    order = ex.result()[0]  # table position -> cloud (the executor sorts heaviest first)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)

    def ragged_step():
        cs.build()
        ex._kernels()

    side = torch.cuda.Stream(device)
    side.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(side):
        ragged_step()
    torch.cuda.current_stream(device).wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        c0 = capi.launch_count()
        ragged_step()
        launches = capi.launch_count() - c0
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    t_graph = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = _events()
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        t_graph.append(e0.elapsed_time(e1))
    ex.check_status()
    pos_of = {c: i for i, c in enumerate(order)}
    q_off_tab = _prefix([rb.Qs[c] for c in order])
    res_f = [ex.f_out[q_off_tab[pos_of[c]]: q_off_tab[pos_of[c]] + rb.Qs[c]].clone() for c in range(C)]

    clouds = [[t.contiguous() for t in cs.cloud(c)] for c in range(C)]
    qs = [q[a:a + n].contiguous() for a, n in zip(_prefix(rb.Qs), rb.Qs)]

    def loop(op):
        outs = []
        with torch.no_grad():
            for c in range(C):
                pc, sc, Rc, fc = clouds[c]
                outs.append(op(qs[c][None], pc[None], fc[None], sc[None], Rc[None], rb.Ks[c])[0])
        return outs

    for _ in range(2):
        loop(knn_aggregate_aniso)
    torch.cuda.synchronize()
    t_loop = []
    for _ in range(max(3, steps // 2)):
        flush.zero_()
        e0, e1 = _events()
        e0.record()
        outs = loop(knn_aggregate_aniso)
        e1.record()
        e1.synchronize()
        t_loop.append(e0.elapsed_time(e1))
    same = all(torch.equal(outs[c][0], res_f[c]) for c in range(C))
    ms, ms_loop = statistics.median(t_graph), statistics.median(t_loop)
    pairs = sum(a * b for a, b in zip(rb.Qs, rb.sizes))
    out = {"workload": "ragged: 64 clouds, P~logU[1024,32768], Q~logU[2048,65536], K in {8,16,32}, F=64, "
                       "8-Gaussian mixtures; forward (cloud-set build + ragged search/aggregation)",
           "clouds": C, "queries": total_q, "points": sum(rb.sizes), "pairs": pairs,
           "ms_per_step": ms, "value": total_q / (ms / 1e3), "unit": UNIT, "execution": "one CUDA graph",
           "gpu_launches_per_step": launches, "splits": splits,
           "per_cloud_loop": {"ms_per_step": ms_loop, "value": total_q / (ms_loop / 1e3),
                              "how": "eager loop of knn_aggregate_aniso, one call per cloud"},
           "speedup_vs_loop": ms_loop / ms, "f_out_identical_to_loop": bool(same)}
    ref, why = load_reference_ext() if with_reference else (None, "skipped (--no-reference-ext)")
    if ref is None:
        out["reference_ext_loop"] = {"unavailable": why}
    else:
        rop = lambda *a: ref.knn_aggregate_aniso_forward(*a)
        loop(rop)
        torch.cuda.synchronize()
        t_ref = []
        for _ in range(ref_steps):
            flush.zero_()
            e0, e1 = _events()
            e0.record()
            loop(rop)
            e1.record()
            e1.synchronize()
            t_ref.append(e0.elapsed_time(e1))
        mr = statistics.median(t_ref)
        out["reference_ext_loop"] = {"ms_per_step": mr, "value": total_q / (mr / 1e3),
                                     "how": "reference extension forward, one call per cloud"}
        out["speedup_vs_reference_loop"] = mr / ms
    return out


def sphere_block(device, steps=5, ref_steps=1, with_reference=True, sample=256):
    """Large single cloud: B=1, P=131072 sphere-surface points (surface-aligned
    Gaussians), Q=524288 near-surface queries, F=128, K=16; the Eikonal
    training step (forward, dq with create_graph, backward), graphed, L2
    flushed; the reference extension's step beside it; idxs/dists of the
    first ``sample`` queries checked bit for bit against the CPU oracle."""
    from cuda_knn_aggregate import knn_aggregate_aniso
    from cuda_knn_aggregate import workloads as W

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    shape, t = W.make("sphere")
    ins = [x.to(device).requires_grad_(True) for x in t]
    step = eikonal_step_fn(knn_aggregate_aniso, ins, shape.K)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)
    side = torch.cuda.Stream(device)
    side.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(side):
        for _ in range(2):
            step()
    torch.cuda.current_stream(device).wait_stream(side)
    for a in ins:
        a.grad = None
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        step()
    g.replay()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = _events()
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms = statistics.median(ts)
    units = shape.B * shape.Q
    with torch.no_grad():
        _, _, d, i = knn_aggregate_aniso(*[x.detach() for x in ins], shape.K)
    q, p, f, sg, R = t
    _, _, d_or, i_or = O.forward_f32(q[:, :sample], p, f, sg, R, shape.K, with_features=False)
    match = bool((i[:, :sample].cpu().numpy() == i_or).all() and
                 (d[:, :sample].cpu().numpy().view("int32") == d_or.view("int32")).all())
    out = {"workload": "sphere: B=1 P=131072 sphere surface (radial noise 0.01, R third column = normal, "
                       "sigma (0.02,0.02,0.005)), Q=524288 surface + N(0,0.05) queries, F=128, K=16; "
                       "fwd + dq(create_graph) + Eikonal backward",
           "ms_per_step": ms, "value": units / (ms / 1e3), "unit": UNIT, "execution": "CUDA graph replay",
           "pairs": shape.B * shape.Q * shape.P, "idxs_dists_bit_exact_vs_oracle_sample": match,
           "oracle_sample_queries": sample}
    del g
    ref, rop = ref_ext() if with_reference else (None, "skipped (--no-reference-ext)")
    if ref is None:
        out["reference_ext"] = {"unavailable": rop}
    else:
        rstep = eikonal_step_fn(rop, ins, shape.K)
        rstep()
        torch.cuda.synchronize()
        tr = []
        for _ in range(ref_steps):
            flush.zero_()
            e0, e1 = _events()
            e0.record()
            rstep()
            e1.record()
            e1.synchronize()
            tr.append(e0.elapsed_time(e1))
        mr = statistics.median(tr)
        out["reference_ext"] = {"ms_per_step": mr, "value": units / (mr / 1e3), "steps": ref_steps}
        out["speedup_vs_reference"] = mr / ms
    return out


def _prefix(xs):
    a, o = 0, []
    for x in xs:
        o.append(a)
        a += x
    return o


def served_block(device, seconds_per_rate=2.0, loads=(0.5, 0.8, 0.95)):
    """Serving over 16 resident sphere-layout clouds (P cycling 16384 /
    65536 / 131072, F=64): requests with Q ~ logU[256, 65536] against a random
    cloud, K=16, 30% also asking d(sum f_out)/dq, host query buffers in and
    host outputs out.  Saturated throughput (every request queued at t=0),
    then Poisson arrivals at fractions of it with p50/p99 latency; beside it
    the same requests served by a per-request loop of the uniform op."""
    from cuda_knn_aggregate import knn_aggregate_aniso
    from cuda_knn_aggregate import workloads as W
    from cuda_knn_aggregate.ragged import CloudSet
    from cuda_knn_aggregate.serving import Request, Server

    p, sigma, R, f, sizes = W.serving_clouds()
    cs = CloudSet(p.to(device), sigma.to(device), R.to(device), f.to(device), sizes)

    def requests(n, rate, seed):
        raw = W.serving_requests(n, rate, seed=seed)
        return [Request(cloud=r["cloud"], q=r["q"].pin_memory(), K=r["K"], want_grad=r["want_grad"],
                        arrival=r["arrival"]) for r in raw]

    warm = requests(40, None, 7)
    srv = Server(cs, hbm_budget_bytes=40e9, max_k=16, step_queries=1 << 18, inflight=3, cap_segments=256,
                 splits="auto", tune_requests=warm, host_budget_bytes=2e9)
    srv.run(warm, keep_outputs=False)  # warm-up
    sat = srv.run(requests(300, None, 8), keep_outputs=False)
    mean_q = sat.queries / max(1, sat.n_requests)
    sat_rps = sat.throughput / mean_q
    out = {"workload": "served: 16 resident sphere clouds (P 16384/65536/131072, F=64), Q~logU[256,65536], K=16, "
                       "30% fwd + d(sum f_out)/dq, pinned host queries in, host f_out/dq out",
           "hbm_budget_gb": 40, "device_bytes": srv.device_bytes, "step_queries": srv.step_queries,
           "inflight_steps": len(srv.execs), "splits": srv.splits, "host_ring_gb": srv.ring.cap / 1e9,
           "saturated": {**sat.summary(), "requests_per_s": sat_rps}, "rates": []}
    for i, frac in enumerate(loads):
        rate = frac * sat_rps
        n = max(20, int(rate * seconds_per_rate))
        st = srv.run(requests(n, rate, 100 + i), keep_outputs=False)
        out["rates"].append({"load": frac, "rate_rps": rate, **st.summary()})
    mid = out["rates"][len(out["rates"]) // 2] if out["rates"] else None
    if mid:
        out["p50_ms"], out["p99_ms"], out["at_load"] = mid["p50_ms"], mid["p99_ms"], mid["load"]

    # per-request plain loop of the uniform op (same requests, saturated)
    reqs = requests(60, None, 9)
    clouds = [[t.contiguous() for t in cs.cloud(c)] for c in range(cs.C)]
    qmax = max(int(r.q.shape[0]) for r in reqs)
    fo_host = torch.empty(qmax, cs.F, pin_memory=True)  # preallocated pinned outputs, as the server's ring
    dq_host = torch.empty(qmax, 3, pin_memory=True)

    def plain(r):
        pc, sc, Rc, fc = clouds[r.cloud]
        Q = int(r.q.shape[0])
        qd = r.q.to(device, non_blocking=True)[None]
        if r.want_grad:
            qd.requires_grad_(True)
            fo = knn_aggregate_aniso(qd, pc[None], fc[None], sc[None], Rc[None], r.K)[0]
            dq = torch.autograd.grad(fo.sum(), qd)[0]
            dq_host[:Q].copy_(dq[0], non_blocking=True)
        else:
            with torch.no_grad():
                fo = knn_aggregate_aniso(qd, pc[None], fc[None], sc[None], Rc[None], r.K)[0]
        fo_host[:Q].copy_(fo[0].detach(), non_blocking=True)

    for r in reqs:  # warm-up pass over every request shape
        plain(r)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in reqs:
        plain(r)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    qn = sum(int(r.q.shape[0]) for r in reqs)
    out["per_request_loop"] = {"throughput_qps": qn / el, "requests": len(reqs),
                               "how": "eager loop of knn_aggregate_aniso (+autograd dq), one call per request"}
    out["speedup_vs_loop"] = out["saturated"]["throughput_qps"] / (qn / el)
    return out


# ------------------------------------------------------------------- arms

def fp32_peak_tflops(device):
    from cuda_knn_aggregate import capi

    blocks, iters = 148 * 8, 8192
    out = torch.empty(blocks * 256, dtype=torch.float32, device=device)
    for _ in range(2):
        capi.fp32_peak_probe(out, blocks, iters)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(3):
        e0.record()
        capi.fp32_peak_probe(out, blocks, iters)
        e1.record()
        e1.synchronize()
        best = max(best, blocks * 256 * iters * 32 / (e0.elapsed_time(e1) / 1e3) / 1e12)
    return best


# DRAM bytes (read + write) of one search_f32_kernel<16,2,16> launch at the
# table workload, from the ncu capture summarised in
# profiles/search_f32_table.md (dram__bytes_read.sum + dram__bytes_write.sum
# of one launch); update it with that summary whenever the search kernel
# changes.
SEARCH_TRAFFIC_BYTES = 3230720
SEARCH_TRAFFIC_SOURCE = "ncu capture of one search_f32_kernel<16,2,16> launch (profiles/search_f32_table.md)"

CONFIG = {"workload": "table: B=2 Q=12288 P=4096 F=64 K=16, fwd + dq(create_graph) + Eikonal backward",
          "l2": "flushed between timed steps (256 MiB write)"}


def compact(block, keys):
    """The named figures of a workload block (the full block: --workload NAME)."""
    return {k: block[k] for k in keys if k in block}


def run_ours(args):
    ws, rank, local = dist_env()
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    init_dist(ws, local, "nccl")
    from cuda_knn_aggregate import capi, knn_aggregate_aniso

    shape, t = make_inputs(rank, device)
    K, units = shape.K, shape.B * shape.Q
    ins = [x.to(device).requires_grad_(True) for x in t]
    step = eikonal_step_fn(knn_aggregate_aniso, ins, K)

    ev_sb, ev_se = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev_sb.record()
    ev_se.record()
    torch.cuda.synchronize()
    capi.set_profile_events(ev_sb, ev_se)

    c0 = capi.launch_count()
    step()
    torch.cuda.synchronize()
    launches_per_step = capi.launch_count() - c0

    # eager timing (for reference; the headline uses the captured step)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)
    eager = []
    for _ in range(max(3, args.warmup)):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        e1.synchronize()
        eager.append(e0.elapsed_time(e1))

    side = torch.cuda.Stream(device)
    side.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(side):
        for _ in range(3):
            step()
    torch.cuda.current_stream(device).wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    for a in ins:
        a.grad = None
    with torch.cuda.graph(graph):
        step()
    for _ in range(args.warmup):
        flush.zero_()
        graph.replay()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    barrier(ws)
    torch.cuda.synchronize()
    step_ms, search_ms = [], []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        graph.replay()
        e1.record()
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        search_ms.append(ev_sb.elapsed_time(ev_se))
    torch.cuda.synchronize()
    barrier(ws)
    clocks = sampler.stop()
    capi.set_profile_events(None, None)

    ms = max_over_ranks(statistics.mean(step_ms), ws, device)
    value = ws * units / (ms / 1e3)

    # end to end through the public API: host inputs in pinned memory,
    # H2D copies + step + D2H of the loss inside the timed region
    host = [x.detach().cpu().pin_memory() for x in t]
    h2d = sum(x.numel() * x.element_size() for x in host)
    e2e, d2h = e2e_times(knn_aggregate_aniso, host, K, device, args.steps, args.warmup, flush)
    e2e_ms = max_over_ranks(statistics.mean(e2e), ws, device)

    if rank != 0:
        barrier(ws)
        return None

    search_s = statistics.median(search_ms) / 1e3
    pairs = shape.B * shape.Q * shape.P
    peak = fp32_peak_tflops(device)
    achieved = FLOP_PER_PAIR * pairs / search_s / 1e12
    roofline = {"bound": "fp32", "kernel": "search_f32_kernel", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": "measured: FFMA-bound probe kernel in bench.py (MEASURED_PEAKS.json has no FP32 figure)",
                "algorithmic": f"{FLOP_PER_PAIR} FLOP x {pairs} (q,p) pairs per launch",
                "launch_ms": search_s * 1e3, "traffic": SEARCH_TRAFFIC_BYTES, "traffic_source": SEARCH_TRAFFIC_SOURCE}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded uniform cube, README timing-table shape)",
        "config": {**CONFIG, "queries_per_gpu": units, "parallelism": f"independent batches per rank x{ws}",
                   "execution": "CUDA graph replay"},
        "e2e": {"value": ws * units / (e2e_ms / 1e3), "unit": UNIT, "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "how": "public API knn_aggregate_aniso + autograd, eager, pinned host inputs"},
        "roofline": roofline,
        "clocks": clocks,
        "gpu_launches": launches_per_step * args.steps,
        "gpu_launches_per_step": launches_per_step,
        "eager_ms_per_step": statistics.mean(eager),
    }
    if ws == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_block()
    if ws == 1 and not args.no_ragged:
        rb = ragged_block(device, with_reference=not args.no_reference_ext)
        out["ragged"] = compact(rb, ("clouds", "queries", "ms_per_step", "value", "speedup_vs_loop",
                                     "f_out_identical_to_loop", "speedup_vs_reference_loop"))
    if ws == 1 and not args.no_sphere:
        sb = sphere_block(device, with_reference=not args.no_reference_ext)
        out["sphere"] = compact(sb, ("ms_per_step", "value", "idxs_dists_bit_exact_vs_oracle_sample",
                                     "speedup_vs_reference"))
        if "reference_ext" in sb and "ms_per_step" in sb["reference_ext"]:
            out["sphere"]["reference_ext_ms_per_step"] = sb["reference_ext"]["ms_per_step"]
    if ws == 1 and not args.no_served:
        sv = served_block(device)
        out["served"] = {"saturated_qps": sv["saturated"]["throughput_qps"], "at_load": sv.get("at_load"),
                         "speedup_vs_per_request_loop": sv.get("speedup_vs_loop")}
        out["served_p50_ms"] = sv.get("p50_ms")
        out["served_p99_ms"] = sv.get("p99_ms")
    # the north-star comparator last, so it is in any tail of the line: the
    # reference extension's step on this GPU, device-resident and end to end
    if ws == 1 and not args.no_reference_ext:
        r = time_reference_ext(device, min(args.steps, 10), 2, host=host)
        if "ms_per_step" in r:
            out["reference_ext_ms_per_step"] = r["ms_per_step"]
            out["reference_ext_e2e_ms_per_step"] = r.get("e2e_ms_per_step")
            out["speedup_vs_reference_ext"] = r["ms_per_step"] / ms
            if r.get("e2e_ms_per_step"):
                out["e2e_speedup_vs_reference_ext"] = r["e2e_ms_per_step"] / e2e_ms
        else:
            out["reference_ext"] = r
    print(json.dumps(out), flush=True)
    barrier(ws)
    return out


def run_reference_cpu(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return None
    q_per_batch = 2048
    cpu_step_rate(q_per_batch, iters=args.warmup)
    rate, n, el, thr = cpu_step_rate(q_per_batch, iters=args.steps)
    ms = el / n * 1e3
    block = {"value": rate, "unit": UNIT, "cores": thr, "kind": "port",
             "sample": f"plain-PyTorch FP32 step (oracle/oracle.py) on {q_per_batch} of 12288 queries per batch "
                       f"element of the table workload, full P=4096; {n} steps"}
    out = {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "impl": "reference", "data": "synthetic (seeded uniform cube, README timing-table shape)",
           "config": {**CONFIG, "queries_per_gpu": 24576, "parallelism": "host cores",
                      "execution": "plain-PyTorch CPU formulation (the reference ships no CPU implementation), "
                                   "timed on a bounded query sample per step (see cpu_baseline.sample)"},
           "cpu_baseline": block,
           "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return out


def run_reference_ext(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return None
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    r = time_reference_ext(device, args.steps, args.warmup)
    out = {"metric": METRIC, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "impl": "reference-ext", "dtype": "f32", **r}
    print(json.dumps(out), flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-ext"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-ext", action="store_true")
    ap.add_argument("--no-ragged", action="store_true", help="skip the ragged-batch block")
    ap.add_argument("--no-served", action="store_true", help="skip the serving block")
    ap.add_argument("--no-sphere", action="store_true", help="skip the large single-cloud block")
    ap.add_argument("--workload", default="table", choices=["table", "ragged", "served", "sphere"],
                    help="table: the headline line (with the ragged and served blocks attached); ragged / "
                         "served: only that block, as its own JSON line (for profiling)")
    ap.add_argument("--search-splits", type=int, default=0,
                    help="launch shape of the uniform search (knnag_set_search_splits; 0: automatic, "
                         "128: the tensor-core search), for profiling one kernel")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.search_splits and args.impl == "ours":
        from cuda_knn_aggregate import capi

        capi.set_search_splits(args.search_splits)
    if args.workload != "table" and args.impl == "ours":
        device = torch.device("cuda", 0)
        torch.cuda.set_device(device)
        if args.workload == "ragged":
            blk = ragged_block(device, with_reference=not args.no_reference_ext)
        elif args.workload == "sphere":
            blk = sphere_block(device, with_reference=not args.no_reference_ext)
        else:
            blk = served_block(device)
        print(json.dumps(blk), flush=True)
        return
    if args.impl == "reference":
        run_reference_cpu(args)
    elif args.impl == "reference-ext":
        run_reference_ext(args)
    else:
        run_ours(args)
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1 and args.impl == "ours":
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
