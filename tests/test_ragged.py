"""Ragged batches over resident clouds (cuda_knn_aggregate.ragged).

CPU: the segment-table encoder and cloud-set sizing of the C ABI (host-only
functions).  GPU: every segment of a ragged call equals the uniform op on
that cloud and query set bit for bit (idxs, dists, w_out, f_out, dq), also
through a captured graph replayed on new tables, and each request's result is
the same alone and in a mixed step; an invalid table latches a device error
and writes nothing.
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_err
import oracle as O

I = lambda xs: (ctypes.c_int * len(xs))(*xs)


def _lib():
    from cuda_knn_aggregate import capi

    return capi.lib()


def _encode(clouds, Qs, Ks, want=None, P=(1000, 200, 50000), splits=1):
    L = _lib()
    n = len(clouds)
    nb = L.knnag_segments_bytes(n)
    buf = np.zeros(nb, np.uint8)
    rc = L.knnag_segments_encode(n, I(clouds), I(Qs), I(Ks), None if want is None else I(want), len(P), I(P), splits,
                                 ctypes.c_void_p(buf.ctypes.data), nb)
    return rc, buf


def _header(buf):
    i32 = buf[:16].view(np.int32)
    i64 = buf[16:64].view(np.int64)
    return dict(magic=int(i32[0]), nseg=int(i32[1]), kmax=int(i32[2]), qpc=int(i32[3]), total_q=int(i64[0]),
                total_e=int(i64[1]), n_items=int(buf[32:36].view(np.int32)[0]),
                total_qcells=int(buf[36:40].view(np.int32)[0]), bigk_q=int(i64[3]), grad_rows=int(i64[4]))


def _descs(buf, n):
    out = []
    for s in range(n):
        d = buf[64 + 48 * s: 64 + 48 * (s + 1)]
        a = d[:24].view(np.int64)
        b = d[24:48].view(np.int32)
        out.append(dict(q_off=int(a[0]), e_off=int(a[1]), bigk_off=int(a[2]), cloud=int(b[0]), Q=int(b[1]),
                        K=int(b[2]), qbits=int(b[3]), qcell_off=int(b[4]), item_off=int(b[5])))
    return out


# ------------------------------------------------------------------- CPU


def test_segment_encoder_offsets():
    clouds, Qs, Ks = [0, 2, 1, 2, 0], [300, 5000, 0, 40, 129], [8, 16, 5, 40, 32]
    rc, buf = _encode(clouds, Qs, Ks, want=[1, 1, 0, 0, 0], splits=1)
    assert rc == 0
    h = _header(buf)
    assert h["nseg"] == 5 and h["kmax"] == 40 and h["qpc"] == 128
    assert h["total_q"] == sum(Qs) and h["total_e"] == sum(q * k for q, k in zip(Qs, Ks))
    assert h["grad_rows"] == 5300 and h["bigk_q"] == 40
    # K > 32 segments get no search items; the others ceil(Q / qpc)
    assert h["n_items"] == 3 + 40 + 0 + 0 + 2
    d = _descs(buf, 5)
    q = e = it = bk = cells = 0
    for s in range(5):
        assert (d[s]["q_off"], d[s]["e_off"], d[s]["item_off"], d[s]["bigk_off"], d[s]["qcell_off"]) == (q, e, it, bk,
                                                                                                          cells)
        q += Qs[s]
        e += Qs[s] * Ks[s]
        it += 0 if Ks[s] > 32 else -(-Qs[s] // 128)
        bk += Qs[s] if Ks[s] > 32 else 0
        cells += 8 ** d[s]["qbits"]
        assert 8 ** d[s]["qbits"] <= max(8, Qs[s])  # the workspace bound cap_q + 8 * cap_segments
    assert h["total_qcells"] == cells


@pytest.mark.parametrize("splits,qpc", [(1, 128), (2, 64), (4, 32)])
def test_segment_encoder_splits(splits, qpc):
    rc, buf = _encode([0], [1000], [16], splits=splits)
    assert rc == 0 and _header(buf)["qpc"] == qpc and _header(buf)["n_items"] == -(-1000 // qpc)


def test_segment_encoder_errors():
    assert _encode([0, 1], [10, 10], [8, 8], want=[0, 1])[0] == 1       # dq segments must come first
    assert _encode([0], [10], [201], P=(200,))[0] == 2                  # K > P
    assert _encode([0], [10], [0])[0] == 2                              # K < 1
    assert _encode([3], [10], [8])[0] == 1                              # cloud out of range
    assert _encode([0], [-1], [8])[0] == 1                              # negative Q
    assert _encode([0], [10], [8], splits=3)[0] == 1                    # splits not 1, 2, 4
    h = _header(_encode([0, 1], [10, 20], [4, 4])[1])
    assert h["grad_rows"] == 30                                         # no want_grad: every row


def test_cloudset_sizes():
    L = _lib()
    assert L.knnag_cloudset_bytes(2, I([100, 0])) == 0
    assert L.knnag_cloudset_bytes(0, I([1])) == 0
    a = L.knnag_cloudset_bytes(2, I([100, 300]))
    b = L.knnag_cloudset_bytes(2, I([100, 30000]))
    assert 0 < a < b
    # records (64 B) + search tiles (64 B per padded point) dominate
    assert b >= (100 + 30000) * 64 + (128 + 30080) * 64


# ------------------------------------------------------------------- GPU


def _clouds(sizes, F, seed):
    g = torch.Generator().manual_seed(seed)
    out = []
    for P in sizes:
        p = torch.rand(P, 3, generator=g)
        A = torch.randn(P, 3, 3, generator=g, dtype=torch.float64)
        R = torch.linalg.qr(A)[0].float().contiguous()
        sigma = 5.0 + 50.0 * torch.rand(P, 3, generator=g)
        f = torch.rand(P, F, generator=g)
        out.append((p, sigma, R, f))
    return out


def _queries(Q, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.rand(Q, 3, generator=g) * 1.1 - 0.05


SIZES = [4096, 1, 300, 20000, 128, 1000]
SEGS = [  # (cloud, Q, K, want dq)
    (0, 3000, 16, True), (3, 12288, 8, True), (1, 50, 1, False), (2, 700, 32, False), (3, 0, 16, False),
    (5, 257, 40, False), (4, 999, 128, False), (0, 129, 3, False), (3, 4000, 24, False)]


def _uniform(cl, q, K, want_dq):
    import cuda_knn_aggregate as C

    p, s, R, f = [t.cuda() for t in cl]
    qq = q.cuda()[None].requires_grad_(want_dq)
    f_out, w, d, i = C.knn_aggregate_aniso(qq, p[None], f[None], s[None], R[None], K)
    dq = torch.autograd.grad(f_out.sum(), qq)[0][0] if want_dq else None
    return f_out[0].detach(), w[0], d[0], i[0], dq


@pytest.mark.gpu
def test_ragged_forward_matches_uniform_op():
    from cuda_knn_aggregate.ragged import CloudSet, ragged_forward

    F = 12
    clouds = _clouds(SIZES, F, seed=1)
    cs = CloudSet.from_clouds([[t.cuda() for t in c] for c in clouds])
    qs = [_queries(Q, seed=10 + i) for i, (_, Q, _, _) in enumerate(SEGS)]
    res = ragged_forward(cs, torch.cat(qs).cuda(), [s[0] for s in SEGS], [s[1] for s in SEGS], [s[2] for s in SEGS],
                         grad_q=[s[3] for s in SEGS])
    for i, (c, Q, K, want) in enumerate(SEGS):
        if Q == 0:
            continue
        f_out, w, d, idx = res.segment(i)
        uf, uw, ud, ui, udq = _uniform(clouds[c], qs[i], K, want)
        assert torch.equal(idx, ui), i
        assert torch.equal(d, ud), i
        assert torch.equal(w, uw), i
        assert torch.equal(f_out, uf), i
        if want:
            a = res.q_off[i]
            assert torch.equal(res.dq[a: a + Q], udq), i


@pytest.mark.gpu
def test_ragged_forward_vs_oracle():
    from cuda_knn_aggregate.ragged import CloudSet, ragged_forward

    clouds = _clouds([3000, 700], 8, seed=2)
    cs = CloudSet.from_clouds([[t.cuda() for t in c] for c in clouds])
    qs = [_queries(2000, 5), _queries(900, 6)]
    segs = [(1, 2000, 16), (0, 900, 9)]
    res = ragged_forward(cs, torch.cat(qs).cuda(), [s[0] for s in segs], [s[1] for s in segs], [s[2] for s in segs])
    for i, (c, Q, K) in enumerate(segs):
        p, s, R, f = clouds[c]
        fo, w, d, idx = O.forward_f32(qs[i][None], p[None], f[None], s[None], R[None], K)
        f_out, ww, dd, ii = res.segment(i)
        assert np.array_equal(ii.cpu().numpy(), idx[0])
        assert np.array_equal(dd.cpu().numpy().view(np.int32), d[0].view(np.int32))
        assert rel_err(ww.cpu().numpy(), w[0]) < 1e-5
        assert rel_err(f_out.cpu().numpy(), fo[0]) < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("splits", [1, 4])
def test_executor_graph_replays_and_alone_vs_mixed(splits):
    """One captured graph, replayed on different tables: every request's
    outputs are identical alone (one-segment step) and in a mixed step."""
    from cuda_knn_aggregate.ragged import CloudSet, RaggedExecutor

    F = 16
    clouds = _clouds([5000, 800, 20000], F, seed=3)
    cs = CloudSet.from_clouds([[t.cuda() for t in c] for c in clouds])
    ex = RaggedExecutor(cs, cap_segments=8, cap_queries=30000, max_k=32, splits=splits)
    assert ex.graph is not None
    reqs = [(0, _queries(4000, 20), 16, True), (2, _queries(9000, 21), 8, False), (1, _queries(300, 22), 32, True),
            (2, _queries(1, 23), 1, False), (0, _queries(7000, 24), 16, False)]
    alone = []
    for c, q, K, g in reqs:
        ex.submit([c], [q], [K], [g])
        order, wg, r = ex.result()
        ex.check_status()
        alone.append([t.clone() for t in r.segment(0)] + [r.dq[: q.shape[0]].clone() if g else None])
    # mixed, in two different orders (dq segments are moved first inside)
    for perm in ([0, 1, 2, 3, 4], [4, 3, 1, 2, 0]):
        ex.submit([reqs[i][0] for i in perm], [reqs[i][1] for i in perm], [reqs[i][2] for i in perm],
                  [reqs[i][3] for i in perm])
        order, wg, r = ex.result()
        ex.check_status()
        for pos, src in enumerate(order):
            rid = perm[src]
            seg = r.segment(pos)
            for a, b in zip(seg, alone[rid][:4]):
                assert torch.equal(a, b), rid
            if reqs[rid][3]:
                a = r.q_off[pos]
                assert torch.equal(r.dq[a: a + reqs[rid][1].shape[0]], alone[rid][4]), rid
                assert torch.equal(ex.f_host[a: a + reqs[rid][1].shape[0]], alone[rid][0].cpu())


@pytest.mark.gpu
def test_invalid_table_latches_and_writes_nothing():
    """A table beyond the call's capacities fails the device-side validation:
    the status word latches and the outputs stay untouched."""
    from cuda_knn_aggregate import capi
    from cuda_knn_aggregate.ragged import CloudSet, SegmentTable, _ptr

    clouds = _clouds([1000], 4, seed=4)
    cs = CloudSet.from_clouds([[t.cuda() for t in c] for c in clouds])
    L = capi.lib()
    t = SegmentTable(2, cs.device)
    t.encode(cs, [0, 0], [600, 600], [8, 8])
    t.upload()
    cap_q = 1000  # the table holds 1200 queries
    q = torch.rand(1200, 3, device="cuda")
    f_out = torch.full((cap_q, 4), 7.0, device="cuda")
    w = torch.full((cap_q * 8,), 7.0, device="cuda")
    d = torch.full((cap_q * 8,), 7.0, device="cuda")
    i = torch.full((cap_q * 8,), 7, dtype=torch.int64, device="cuda")
    ws = torch.empty(L.knnag_ragged_workspace_bytes(2, cap_q), dtype=torch.uint8, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.knnag_ragged_forward(_ptr(cs.buf), _ptr(t.dev), _ptr(q), _ptr(cs.f), 4, 2, cap_q, cap_q * 8, 8, 1000, 1,
                                _ptr(f_out), _ptr(w), _ptr(d), _ptr(i), _ptr(ws), ws.numel(), st)
    assert rc == 0
    assert L.knnag_read_device_status(_ptr(ws), st) == 7  # KNNAG_ERR_DEVICE
    assert bool((f_out == 7).all()) and bool((w == 7).all()) and bool((i == 7).all())
    # the same call with room for the table succeeds (the buffers are held in
    # names: a temporary passed as _ptr(torch.empty(...)) is freed at once and
    # its memory handed to the next one)
    f2, w2, d2 = torch.empty(1200, 4, device="cuda"), torch.empty(9600, device="cuda"), torch.empty(9600, device="cuda")
    i2 = torch.empty(9600, dtype=torch.int64, device="cuda")
    ws2 = torch.empty(L.knnag_ragged_workspace_bytes(2, 1200), dtype=torch.uint8, device="cuda")
    rc = L.knnag_ragged_forward(_ptr(cs.buf), _ptr(t.dev), _ptr(q), _ptr(cs.f), 4, 2, 1200, 9600, 8, 1000, 1,
                                _ptr(f2), _ptr(w2), _ptr(d2), _ptr(i2), _ptr(ws2), ws2.numel(), st)
    assert rc == 0
    assert L.knnag_read_device_status(_ptr(ws2), st) == 0
    assert bool((i2 >= 0).all()) and bool((i2 < 1000).all())


@pytest.mark.gpu
def test_cloudset_rebuild_after_geometry_change():
    """build() after moving the points in place gives the uniform op's result
    on the new geometry."""
    from cuda_knn_aggregate.ragged import CloudSet, ragged_forward

    clouds = _clouds([2000, 3000], 8, seed=5)
    cs = CloudSet.from_clouds([[t.cuda() for t in c] for c in clouds])
    q = _queries(1500, 9)
    cs.p.mul_(0.5).add_(0.25)
    cs.build()
    res = ragged_forward(cs, q.cuda(), [1], [1500], [16])
    moved = [t.clone() for t in clouds[1]]
    moved[0] = moved[0] * 0.5 + 0.25
    uf, uw, ud, ui, _ = _uniform(moved, q, 16, False)
    f_out, w, d, idx = res.segment(0)
    assert torch.equal(idx, ui) and torch.equal(d, ud) and torch.equal(f_out, uf)


@pytest.mark.gpu
def test_server_results_match_uniform_op():
    """Requests served under continuous batching (Poisson arrivals, several
    steps in flight, large requests split into chunks) get exactly the
    uniform op's f_out and d(sum f_out)/dq."""
    from cuda_knn_aggregate import workloads as W
    from cuda_knn_aggregate.ragged import CloudSet
    from cuda_knn_aggregate.serving import Request, Server

    p, sigma, R, f, sizes = W.serving_clouds(n_clouds=4, F=16, sizes=(3000, 9000))
    cs = CloudSet(p.cuda(), sigma.cuda(), R.cuda(), f.cuda(), sizes)
    srv = Server(cs, hbm_budget_bytes=4e9, max_k=16, step_queries=6000, inflight=3, cap_segments=16)
    raw = W.serving_requests(40, rate_hz=400.0, n_clouds=4, q_range=(64, 9000), seed=11)
    reqs = [Request(cloud=r["cloud"], q=r["q"], K=r["K"], want_grad=r["want_grad"], arrival=r["arrival"]) for r in raw]
    stats = srv.run(reqs)
    assert stats.n_requests == 40 and len(stats.latencies_ms) == 40
    assert stats.steps >= 2 and stats.pct(99) >= stats.pct(50) > 0
    assert any(r.q.shape[0] > 6000 for r in reqs)  # some requests were chunked
    for r in reqs:
        uf, _, _, _, udq = _uniform(cs_cloud(cs, r.cloud), r.q, r.K, r.want_grad)
        assert torch.equal(r.f_out, uf.cpu())
        if r.want_grad:
            assert torch.equal(r.dq, udq.cpu())


def cs_cloud(cs, c):
    return [t.cpu() for t in cs.cloud(c)]


@pytest.mark.gpu
@pytest.mark.parametrize("rows", [32768, 32769, 100003, 1 << 20])
def test_adjacency_long_scan(rows):
    """Point->entry adjacency over more rows than one scan CTA covers (the
    three-pass scan): row pointers equal the exclusive prefix of a numpy
    histogram, every row holds exactly its entries in ascending order."""
    from cuda_knn_aggregate import capi

    g = torch.Generator().manual_seed(rows)
    Q, K = 20000, 8
    idxs = torch.randint(0, rows, (1, Q, K), generator=g)
    adj = capi.build_adjacency(idxs.cuda(), rows)
    rowptr, entries = capi.adjacency_arrays(adj, 1, Q, rows, K)
    torch.cuda.synchronize()
    counts = np.bincount(idxs.numpy().ravel(), minlength=rows)
    ref = np.concatenate([[0], np.cumsum(counts)])
    assert np.array_equal(rowptr.cpu().numpy(), ref)
    e = entries.cpu().numpy()
    flat = idxs.numpy().ravel()
    order = np.argsort(flat, kind="stable")
    assert np.array_equal(e, order)


@pytest.mark.gpu
def test_adjacency_row_lengths():
    """Rows of every length class the row sort distinguishes (register
    networks up to 32/64/128/256 entries, shared memory up to 1024, the
    ranking loop beyond), each at and one past its limit, in shuffled
    order: every row holds its entry ids ascending."""
    from cuda_knn_aggregate import capi

    lengths = [0, 1, 2, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512, 513, 1023, 1024, 1025, 2500]
    rows = len(lengths) + 5  # a few empty rows at the end
    K = 4
    flat = np.concatenate([np.full(n, r, dtype=np.int64) for r, n in enumerate(lengths)])
    flat = np.concatenate([flat, np.zeros((-len(flat)) % K, dtype=np.int64)])  # pad to whole queries (row 0)
    rng = np.random.default_rng(7)
    rng.shuffle(flat)
    Q = len(flat) // K
    idxs = torch.from_numpy(flat.reshape(1, Q, K))
    adj = capi.build_adjacency(idxs.cuda(), rows)
    rowptr, entries = capi.adjacency_arrays(adj, 1, Q, rows, K)
    torch.cuda.synchronize()
    counts = np.bincount(flat, minlength=rows)
    assert np.array_equal(rowptr.cpu().numpy(), np.concatenate([[0], np.cumsum(counts)]))
    assert np.array_equal(entries.cpu().numpy(), np.argsort(flat, kind="stable"))


@pytest.mark.gpu
def test_ragged_long_query_scan():
    """A ragged call whose query-cell array needs the multi-CTA scan."""
    from cuda_knn_aggregate.ragged import CloudSet, ragged_forward

    clouds = _clouds([6000, 2500], 8, seed=12)
    cs = CloudSet.from_clouds([[t.cuda() for t in c] for c in clouds])
    qs = [_queries(50000, 40), _queries(30000, 41)]
    res = ragged_forward(cs, torch.cat(qs).cuda(), [0, 1], [50000, 30000], [16, 8])
    for i, (c, K) in enumerate([(0, 16), (1, 8)]):
        uf, uw, ud, ui, _ = _uniform(clouds[c], qs[i], K, False)
        f_out, w, d, idx = res.segment(i)
        assert torch.equal(idx, ui) and torch.equal(d, ud) and torch.equal(f_out, uf)
