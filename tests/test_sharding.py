"""Query sharding of one cloud across ranks, on CPU (gloo, world_size 2).

Each rank holds a replica of p, f, sigma, R, runs the Eikonal training step
on its contiguous share of the queries (an odd count, so the shares differ
by one) with the loss's mean taken over all ranks' queries, then sums the
point-side gradients in one all-reduce.  The op is the plain-PyTorch oracle
in FP64 (no GPU here).  Checked: every rank's point gradients equal the
single-process step's, the ranks' query-side results (f_out rows and dL/dq)
concatenate to the single-process ones, the shares tile [0, Q), and the
gradient exchange is a single collective.
"""
import os
import socket
import sys

import numpy as np
import torch
import torch.multiprocessing as mp

from conftest import ROOT, PKG_DIR

WS = 2
SHAPE = dict(B=2, Q=301, P=200, F=8, K=6)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs():
    from cuda_knn_aggregate import workloads as W

    kw = dict(SHAPE)
    K = kw.pop("K")
    _, t = W.make("small", K=K, seed=57, dtype=torch.float64, **kw)
    return t, K


def _worker(rank, port, out_dir):
    for p in (ROOT, PKG_DIR, os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import torch.distributed as dist

    import oracle as O
    from cuda_knn_aggregate import sharding as S

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=WS)
    try:
        (q, p, f, sigma, R), K = _inputs()
        leaves = [x.clone().requires_grad_(True) for x in (p, f, sigma, R)]
        cloud = S.QueryShardedCloud(*leaves, op=O.plain_forward)
        assert (cloud.rank, cloud.world) == (rank, WS)
        ql = cloud.queries(q).requires_grad_(True)
        f_out = cloud(ql, K)[0]
        (gq,) = torch.autograd.grad(f_out.sum(), ql, create_graph=True)
        loss = S.global_mean(((gq.norm(dim=-1) - 1.0) ** 2).sum(), gq.shape[0] * gq.shape[1])
        loss.backward()
        calls = []
        real = dist.all_reduce

        def counting(*a, **k):
            calls.append(1)
            return real(*a, **k)

        dist.all_reduce = counting
        try:
            cloud.reduce_grads()
        finally:
            dist.all_reduce = real
        a, b = S.query_range(q.shape[1], rank, WS)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), start=a, stop=b, f_out=f_out.detach().numpy(),
                 dq=ql.grad.numpy(), gq=gq.detach().numpy(), n_collectives=len(calls),
                 **{n: x.grad.numpy() for n, x in zip(("p", "f", "sigma", "R"), leaves)})
    finally:
        dist.destroy_process_group()


def test_query_range_tiles_the_queries():
    from cuda_knn_aggregate.sharding import query_range

    for Q in (0, 1, 7, 301, 12288):
        for world in (1, 2, 3, 8):
            ranges = [query_range(Q, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == Q
            assert all(ranges[i][1] == ranges[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1


def test_two_rank_query_sharding_matches_single_process(tmp_path):
    import oracle as O

    port = _free_port()
    mp.start_processes(_worker, args=(port, str(tmp_path)), nprocs=WS, join=True, start_method="spawn")
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(WS)]

    (q, p, f, sigma, R), K = _inputs()
    qq = q.clone().requires_grad_(True)
    leaves = [x.clone().requires_grad_(True) for x in (p, f, sigma, R)]
    f_out = O.plain_forward(qq, *leaves, K)[0]
    (gq,) = torch.autograd.grad(f_out.sum(), qq, create_graph=True)
    ((gq.norm(dim=-1) - 1.0) ** 2).mean().backward()

    assert [int(r["start"]) for r in res] == [0, int(res[0]["stop"])] and int(res[-1]["stop"]) == q.shape[1]
    cat = lambda k: np.concatenate([r[k] for r in res], axis=1)
    np.testing.assert_array_equal(cat("f_out"), f_out.detach().numpy())
    np.testing.assert_array_equal(cat("gq"), gq.detach().numpy())
    np.testing.assert_allclose(cat("dq"), qq.grad.numpy(), rtol=1e-12, atol=1e-15)
    for r in res:
        assert int(r["n_collectives"]) == 1
        for n, x in zip(("p", "f", "sigma", "R"), leaves):
            np.testing.assert_allclose(r[n], x.grad.numpy(), rtol=1e-10, atol=1e-13)
