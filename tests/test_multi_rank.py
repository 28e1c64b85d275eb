"""Multi-rank host logic of bench.py on CPU (gloo, world_size 2).

The op shards by batch element (whole clouds per rank, no collective on the
data path): each rank draws its own seeded batch, runs the op on it, and the
only cross-rank steps are the barriers around the timed region and the max
over ranks of the step time.  Here the op is the CPU oracle (no GPU), and the
test checks that (1) the ranks' batches differ, (2) each rank's result equals
what a single process computes for that batch, (3) max_over_ranks returns the
slowest rank's time on every rank and (4) the whole-job value is
world_size x units / max time.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import ROOT

WS = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard_slice(t, n=64, P=256):
    """First n queries and P points of a batch element (keeps the oracle fast)."""
    q, p, f, sigma, R = t
    return q[:, :n].contiguous(), p[:, :P].contiguous(), f[:, :P].contiguous(), sigma[:, :P].contiguous(), \
        R[:, :P].contiguous()


def _worker(rank, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(WS),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bench
    import oracle as O
    import torch.distributed as dist

    ws, r, local = bench.dist_env()
    assert (ws, r, local) == (WS, rank, rank)
    bench.init_dist(ws, local, "gloo")
    try:
        shape, t = bench.make_inputs(rank, torch.device("cpu"))
        q, p, f, sigma, R = _shard_slice(t)
        fo, w, d, idx = O.forward_f32(q, p, f, sigma, R, shape.K)
        bench.barrier(ws)
        my_ms = 10.0 + 5.0 * rank
        slowest = bench.max_over_ranks(my_ms, ws, torch.device("cpu"))
        units = q.shape[0] * q.shape[1]
        value = ws * units / (slowest / 1e3)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), q=q.numpy(), idx=idx, fo=fo, slowest=slowest, value=value,
                 units=units)
        bench.barrier(ws)
    finally:
        dist.destroy_process_group()


def test_two_rank_weak_scaling_host_path(tmp_path):
    import oracle as O
    import bench

    port = _free_port()
    mp.start_processes(_worker, args=(port, str(tmp_path)), nprocs=WS, join=True, start_method="spawn")
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(WS)]
    # (1) independent batches per rank
    assert not np.array_equal(res[0]["q"], res[1]["q"])
    # (2) each rank's result is the single-process result for its batch
    for r in range(WS):
        shape, t = bench.make_inputs(r, torch.device("cpu"))
        q, p, f, sigma, R = _shard_slice(t)
        fo, w, d, idx = O.forward_f32(q, p, f, sigma, R, shape.K)
        assert np.array_equal(idx, res[r]["idx"])
        assert np.array_equal(fo, res[r]["fo"])
    # (3) every rank saw the slowest rank's time; (4) whole-job value
    for r in range(WS):
        assert float(res[r]["slowest"]) == 15.0
        assert float(res[r]["value"]) == pytest.approx(WS * int(res[r]["units"]) / 0.015)
