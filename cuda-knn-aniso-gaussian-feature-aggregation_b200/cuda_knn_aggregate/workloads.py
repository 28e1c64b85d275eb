"""Seeded synthetic point clouds and query sets for the kNN aggregation workloads.

The reference project publishes no dataset; its timing table
(``README.md:47-55``) and usage snippet (``README.md:26-45``) only fix shapes.
These generators produce inputs with those shapes and the value
distributions stated for each workload, on the CPU with a seeded
``torch.Generator`` (seed ``1000 + n`` for workload ``n``) so every run --
tests, fixtures, benchmarks -- sees the same bytes.

Layout of every tensor matches the reference op (``__init__.py:6-31``):
``q [B,Q,3]``, ``p [B,P,3]``, ``f [B,P,F]``, ``sigma [B,P,3]`` (a precision:
it multiplies the squared rotated offset), ``R [B,P,3,3]`` row-major whose
rows are the Gaussian's axes.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch


@dataclass(frozen=True)
class Shape:
    B: int
    Q: int
    P: int
    F: int
    K: int


# name -> (shape, seed); "small" is the README usage case, "table" the README timing table shape
SHAPES = {
    "small": (Shape(B=2, Q=1000, P=500, F=32, K=12), 1000),
    "table": (Shape(B=2, Q=12288, P=4096, F=64, K=16), 1001),
    "sphere": (Shape(B=1, Q=524288, P=131072, F=128, K=16), 1002),
}


def random_rotations(n: int, g: torch.Generator, dtype=torch.float32) -> torch.Tensor:
    """Orthonormal 3x3 matrices: Q factor of QR of a standard-normal matrix,
    with each column's sign fixed by the sign of the matching diagonal of R."""
    a = torch.randn(n, 3, 3, generator=g, dtype=torch.float64)
    qm, rm = torch.linalg.qr(a)
    d = torch.sign(torch.diagonal(rm, dim1=-2, dim2=-1))
    d[d == 0] = 1.0
    qm = qm * d.unsqueeze(-2)
    return qm.to(dtype).contiguous()


def uniform_cloud(shape: Shape, seed: int, dtype=torch.float32):
    """Uniform-cube workload: q, p ~ U[0,1)^3, f ~ U[0,1), sigma ~ U[0.05,0.2]^3,
    R random orthonormal per point."""
    g = torch.Generator().manual_seed(seed)
    B, Q, P, F = shape.B, shape.Q, shape.P, shape.F
    q = torch.rand(B, Q, 3, generator=g, dtype=dtype)
    p = torch.rand(B, P, 3, generator=g, dtype=dtype)
    f = torch.rand(B, P, F, generator=g, dtype=dtype)
    sigma = 0.05 + 0.15 * torch.rand(B, P, 3, generator=g, dtype=dtype)
    R = random_rotations(B * P, g, dtype).reshape(B, P, 3, 3)
    return tuple(t.contiguous() for t in (q, p, f, sigma, R))


def readme_cloud(B, Q, P, F, seed: int, dtype=torch.float32):
    """Inputs as in the reference's usage snippet (``README.md:35-39``):
    every tensor ``torch.rand``, so R is neither orthonormal nor symmetric."""
    g = torch.Generator().manual_seed(seed)
    q = torch.rand(B, Q, 3, generator=g, dtype=dtype)
    p = torch.rand(B, P, 3, generator=g, dtype=dtype)
    f = torch.rand(B, P, F, generator=g, dtype=dtype)
    sigma = torch.rand(B, P, 3, generator=g, dtype=dtype)
    R = torch.rand(B, P, 3, 3, generator=g, dtype=dtype)
    return q, p, f, sigma, R


def _tangent_frames(n: torch.Tensor) -> torch.Tensor:
    """[N,3,3] with columns (t1, t2, n): an orthonormal frame whose third column
    is the unit normal ``n``."""
    helper = torch.zeros_like(n)
    use_x = n[:, 0].abs() < 0.9
    helper[use_x, 0] = 1.0
    helper[~use_x, 1] = 1.0
    t1 = torch.linalg.cross(helper, n)
    t1 = t1 / t1.norm(dim=-1, keepdim=True)
    t2 = torch.linalg.cross(n, t1)
    return torch.stack([t1, t2, n], dim=-1)


def sphere_cloud(shape: Shape, seed: int, dtype=torch.float32,
                 radial_std: float = 0.01, query_std: float = 0.05):
    """Large single-cloud workload: points on the unit sphere with N(0, radial_std)
    radial noise, queries = surface samples + N(0, query_std)^3 offsets,
    surface-aligned Gaussians (R's third column is the sphere normal),
    sigma = (0.02, 0.02, 0.005), f ~ U[0,1)."""
    g = torch.Generator().manual_seed(seed)
    B, Q, P, F = shape.B, shape.Q, shape.P, shape.F
    n = torch.randn(B * P, 3, generator=g, dtype=torch.float64)
    n = n / n.norm(dim=-1, keepdim=True)
    eps = radial_std * torch.randn(B * P, 1, generator=g, dtype=torch.float64)
    p = (n * (1.0 + eps)).reshape(B, P, 3)
    s = torch.randn(B * Q, 3, generator=g, dtype=torch.float64)
    s = s / s.norm(dim=-1, keepdim=True)
    q = (s + query_std * torch.randn(B * Q, 3, generator=g, dtype=torch.float64)).reshape(B, Q, 3)
    R = _tangent_frames(n).reshape(B, P, 3, 3)
    sigma = torch.tensor([0.02, 0.02, 0.005], dtype=torch.float64).expand(B, P, 3).clone()
    f = torch.rand(B, P, F, generator=g, dtype=torch.float64)
    return tuple(t.to(dtype).contiguous() for t in (q, p, f, sigma, R))


def make(name: str, dtype=torch.float32, **overrides):
    """Build a named workload; ``overrides`` may replace B/Q/P/F/K (and seed)."""
    shape, seed = SHAPES[name]
    seed = overrides.pop("seed", seed)
    if overrides:
        shape = Shape(**{**shape.__dict__, **overrides})
    if name == "sphere":
        t = sphere_cloud(shape, seed, dtype)
    else:
        t = uniform_cloud(shape, seed, dtype)
    return shape, t


def lattice_ties(B=1, n_side=4, Q=64, F=8, seed=7, dtype=torch.float32):
    """A tie-heavy case: points on an ``n_side``^3 lattice with spacing 0.25
    (some duplicated), identity R, unit sigma, and queries on lattice points
    and cell centres, so many keys are exactly equal in FP32."""
    g = torch.Generator().manual_seed(seed)
    ax = torch.arange(n_side, dtype=torch.float64) * 0.25
    grid = torch.stack(torch.meshgrid(ax, ax, ax, indexing="ij"), dim=-1).reshape(-1, 3)
    dup = grid[torch.randint(0, grid.shape[0], (grid.shape[0] // 4,), generator=g)]
    pts = torch.cat([grid, dup], 0)
    pts = pts[torch.randperm(pts.shape[0], generator=g)]
    P = pts.shape[0]
    qi = torch.randint(0, 2, (Q, 3), generator=g, dtype=torch.float64) * 0.125
    qb = grid[torch.randint(0, grid.shape[0], (Q,), generator=g)] + qi
    p = pts.expand(B, P, 3).clone()
    q = qb.expand(B, Q, 3).clone()
    f = torch.rand(B, P, F, generator=g, dtype=torch.float64)
    sigma = torch.ones(B, P, 3, dtype=torch.float64)
    R = torch.eye(3, dtype=torch.float64).expand(B, P, 3, 3).clone()
    return tuple(t.to(dtype).contiguous() for t in (q, p, f, sigma, R))


def pairs_count(shape: Shape) -> int:
    return shape.B * shape.Q * shape.P


def log_uniform_int(g: torch.Generator, lo: int, hi: int, n: int) -> torch.Tensor:
    u = torch.rand(n, generator=g, dtype=torch.float64)
    return torch.exp(math.log(lo) + u * (math.log(hi) - math.log(lo))).floor().long().clamp(lo, hi)


# ---------------------------------------------------------------- ragged


@dataclass
class RaggedBatch:
    """Clouds of different sizes, concatenated in cloud order (p, sigma, R,
    f [sum P, ...]); one query set per cloud (q [sum Q, 3], cloud c at rows
    q_off[c]:q_off[c]+Qs[c]) with its own K."""
    p: torch.Tensor
    sigma: torch.Tensor
    R: torch.Tensor
    f: torch.Tensor
    sizes: list
    q: torch.Tensor
    Qs: list
    Ks: list

    def cloud(self, c):
        a = sum(self.sizes[:c])
        b = a + self.sizes[c]
        return self.p[a:b], self.sigma[a:b], self.R[a:b], self.f[a:b]

    def queries(self, c):
        a = sum(self.Qs[:c])
        return self.q[a: a + self.Qs[c]]


def _mixture(g, centres, n, std, dtype):
    comp = torch.randint(0, centres.shape[0], (n,), generator=g)
    return (centres[comp] + std * torch.randn(n, 3, generator=g, dtype=torch.float64)).to(dtype)


def ragged_batch(n_clouds=64, seed=1003, F=64, p_range=(1024, 32768), q_range=(2048, 65536), ks=(8, 16, 32),
                 dtype=torch.float32):
    """Ragged-batch workload: P ~ logU[p_range], Q ~ logU[q_range], K drawn
    from ``ks`` per cloud; points and queries from a mixture of 8 isotropic
    Gaussians (centres U[0,1)^3, std 0.05) per cloud, R random orthonormal,
    sigma ~ U[0.01, 0.1]^3, f ~ U[0,1)."""
    g = torch.Generator().manual_seed(seed)
    sizes = log_uniform_int(g, *p_range, n_clouds).tolist()
    Qs = log_uniform_int(g, *q_range, n_clouds).tolist()
    Ks = [int(ks[i]) for i in torch.randint(0, len(ks), (n_clouds,), generator=g).tolist()]
    ps, qs = [], []
    for P, Q in zip(sizes, Qs):
        centres = torch.rand(8, 3, generator=g, dtype=torch.float64)
        ps.append(_mixture(g, centres, P, 0.05, dtype))
        qs.append(_mixture(g, centres, Q, 0.05, dtype))
    n = sum(sizes)
    p = torch.cat(ps).contiguous()
    R = random_rotations(n, g, dtype)
    sigma = (0.01 + 0.09 * torch.rand(n, 3, generator=g, dtype=torch.float64)).to(dtype)
    f = torch.rand(n, F, generator=g, dtype=torch.float64).to(dtype)
    return RaggedBatch(p, sigma.contiguous(), R, f.contiguous(), sizes, torch.cat(qs).contiguous(), Qs, Ks)


def serving_clouds(n_clouds=16, seed=1004, F=64, sizes=(16384, 65536, 131072), dtype=torch.float32):
    """Resident clouds of the serving workload: sizes cycle through ``sizes``;
    sphere-surface layout of the large single-cloud workload (unit sphere
    with N(0, 0.01) radial noise, R's third column the normal, sigma = (0.02,
    0.02, 0.005)), f ~ U[0,1)."""
    g = torch.Generator().manual_seed(seed)
    P = [int(sizes[i % len(sizes)]) for i in range(n_clouds)]
    ps, Rs, fs = [], [], []
    for n_pts in P:
        n = torch.randn(n_pts, 3, generator=g, dtype=torch.float64)
        n = n / n.norm(dim=-1, keepdim=True)
        eps = 0.01 * torch.randn(n_pts, 1, generator=g, dtype=torch.float64)
        ps.append(n * (1.0 + eps))
        Rs.append(_tangent_frames(n))
        fs.append(torch.rand(n_pts, F, generator=g, dtype=torch.float64))
    n = sum(P)
    sigma = torch.tensor([0.02, 0.02, 0.005], dtype=torch.float64).expand(n, 3)
    cat = lambda xs: torch.cat(xs).to(dtype).contiguous()
    return cat(ps), sigma.to(dtype).contiguous(), cat(Rs), cat(fs), P


def serving_requests(n_requests, rate_hz, n_clouds=16, seed=1005, q_range=(256, 65536), K=16, grad_fraction=0.3,
                     dtype=torch.float32):
    """Requests of the serving workload: Poisson arrivals at ``rate_hz``
    (exponential gaps; every arrival 0 when rate_hz is None), a uniformly
    random cloud, Q ~ logU[q_range] queries = unit-sphere samples + N(0,
    0.05)^3 offsets, K neighbours, and a ``grad_fraction`` chance of also
    asking for d(sum f_out)/dq.  Returns a list of dicts."""
    g = torch.Generator().manual_seed(seed)
    Qs = log_uniform_int(g, *q_range, n_requests).tolist()
    clouds = torch.randint(0, n_clouds, (n_requests,), generator=g).tolist()
    grads = (torch.rand(n_requests, generator=g) < grad_fraction).tolist()
    if rate_hz:
        gaps = -torch.log(1.0 - torch.rand(n_requests, generator=g, dtype=torch.float64)) / rate_hz
        t = torch.cumsum(gaps, 0).tolist()
    else:
        t = [0.0] * n_requests
    out = []
    for i in range(n_requests):
        s = torch.randn(Qs[i], 3, generator=g, dtype=torch.float64)
        s = s / s.norm(dim=-1, keepdim=True)
        q = (s + 0.05 * torch.randn(Qs[i], 3, generator=g, dtype=torch.float64)).to(dtype).contiguous()
        out.append(dict(cloud=clouds[i], q=q, K=K, want_grad=bool(grads[i]), arrival=t[i]))
    return out
