"""Query sharding of one cloud across ranks (one process per GPU).

The reference runs one cloud on one GPU: its backward scatters the
point-side gradients of every (query, neighbour) entry into dL/dp, dL/df,
dL/dsigma and dL/dR with float atomics (``csrc/backward.cu:91, 102-119``
first order, ``:291, 308-326`` second order).  When one cloud's query set is
split across ranks that scatter becomes a cross-rank sum, and that is the
only exchange the path has:

* every rank holds a replica of the cloud -- p, f, sigma, R (316 bytes per
  point at F = 64);
* rank r takes the contiguous range ``query_range(Q, r, world)`` of every
  batch element's queries (contiguous ranges keep the spatial order the
  search exploits, and the ranges differ in size by at most one query);
* the forward, the first-order and the second-order backward run locally:
  no query-side value depends on another rank's queries, so f_out, w_out,
  dists, idxs and dL/dq of a query are those of the unsharded op;
* after the local backward, ``all_reduce_point_grads`` sums the replicas'
  ``.grad`` of p, f, sigma and R over the ranks in ONE collective (the four
  gradients flattened into one bucket; NCCL over NVLink between GPUs, gloo
  on CPU).

A loss that is a mean over all queries must divide by the global query
count on every rank (``global_mean``), so that the summed point gradients
equal the single-process ones.  Nothing here issues a TMA load or reads
another GPU's memory: the only cross-GPU traffic is the collective.
"""
from __future__ import annotations

import torch


def query_range(Q: int, rank: int, world: int):
    """[start, stop) of the queries of `rank` when Q queries are split over
    `world` ranks in contiguous ranges whose sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(Q, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_queries(q: torch.Tensor, rank: int, world: int) -> torch.Tensor:
    """This rank's contiguous share of q [B, Q, 3] (a contiguous copy)."""
    a, b = query_range(q.shape[1], rank, world)
    return q[:, a:b].contiguous()


def global_mean(local_sum: torch.Tensor, n_local: int, group=None) -> torch.Tensor:
    """local_sum / (total count over the ranks): the rank's share of a mean
    over every rank's items (its gradient is the rank's share of the
    gradient of that mean).  One all-reduce of the counts."""
    import torch.distributed as dist

    n = torch.tensor([n_local], dtype=torch.float64, device=local_sum.device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(n, group=group)
    return local_sum / n.to(local_sum.dtype)


def all_reduce_point_grads(tensors, group=None) -> None:
    """Sum the ``.grad`` of the replicated point-side tensors (p, f, sigma,
    R) over the ranks, in place, with one all-reduce of a flat bucket.  A
    tensor without a gradient on this rank contributes zeros (every rank
    takes part in the same collective with the same bucket layout)."""
    import torch.distributed as dist

    tensors = list(tensors)
    if not tensors:
        return
    grads = [t.grad if t.grad is not None else torch.zeros_like(t) for t in tensors]
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat, group=group)
    off = 0
    for t, g in zip(tensors, grads):
        n = g.numel()
        summed = flat[off:off + n].view_as(g)
        if t.grad is None:
            t.grad = summed.clone()
        else:
            t.grad.copy_(summed)
        off += n


class QueryShardedCloud:
    """One cloud replicated on every rank, its queries split across ranks.

    ``op`` is the aggregation op (default: ``knn_aggregate_aniso``).
    ``cloud(q_local, K)`` runs it on this rank's queries against the
    replica; after the local ``backward()`` of a loss built with
    ``global_mean``, ``reduce_grads()`` makes every rank's point gradients
    equal those of the unsharded step.
    """

    def __init__(self, p, f, sigma, R, group=None, op=None):
        import torch.distributed as dist

        self.p, self.f, self.sigma, self.R = p, f, sigma, R
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.rank, self.world = 0, 1
        if op is None:
            from . import knn_aggregate_aniso as op
        self.op = op

    def queries(self, q: torch.Tensor) -> torch.Tensor:
        return shard_queries(q, self.rank, self.world)

    def __call__(self, q_local: torch.Tensor, K: int):
        return self.op(q_local, self.p, self.f, self.sigma, self.R, K)

    def reduce_grads(self) -> None:
        if self.world > 1:
            all_reduce_point_grads((self.p, self.f, self.sigma, self.R), self.group)
