"""Host model of the tensor-core candidate filter's error bound (no GPU).

The tensor-core search (csrc/knn_search_tc.cu) admits a point as a candidate
when its approximate key -- phi(q - o) . psi(p - o) from one TF32 GEMM with
hi/lo-split features, o the tile's box centre -- is at most the query's
threshold + E(q, tile).  Exactness needs |approximate - exact FP32 key| <= E
for every pair.  This test restates, in numpy, the operands the kernels build
(knn_spatial.cu tc_tile_operand: psi in double rounded to FP32, hi = low 13
mantissa bits cleared, lo = psi - hi, the tile maxima; knn_search_tc.cu: phi
in FP32, the bound E) and emulates the tensor core's arithmetic pessimistically
(every operand truncated to TF32, products exact, FP32 accumulation in the
order 0..31 with round-to-nearest, and again with every partial sum rounded
toward zero), on inputs chosen to stress it: the uniform table cloud, the
reference README's non-orthonormal R, a thin sphere shell, a cloud offset by
1000, a cloud scaled by 1e-3, extreme anisotropy and negative precisions.  The
exact key is the oracle's FP32 key (the reference's contraction).  The bar:
|approximate - exact| <= E / 4 everywhere (a 4x margin on top of the bound's
own).
"""
import zlib

import numpy as np
import pytest
import torch

import oracle as O

TP = 128  # points per tile


def tf32(x):
    return (np.ascontiguousarray(x, dtype=np.float32).view(np.uint32) & np.uint32(0xFFFFE000)).view(np.float32)


def tile_operand(p, sigma, R):
    """B rows [n, 32] and the 16 bound terms of one tile (n <= 128 points),
    as tc_tile_operand writes them."""
    lo, hi = p.min(0).astype(np.float32), p.max(0).astype(np.float32)
    o = (np.float32(0.5) * lo + np.float32(0.5) * hi).astype(np.float32)
    pp = p.astype(np.float64) - o.astype(np.float64)
    Rd, sd = R.astype(np.float64), sigma.astype(np.float64)
    M = np.einsum("nam,na,nab->nmb", Rd, sd, Rd)
    mp = np.einsum("nmb,nb->nm", M, pp)
    pmp = np.einsum("nm,nm->n", pp, mp)
    psi = np.stack([M[:, 0, 0], M[:, 1, 1], M[:, 2, 2], 2 * M[:, 0, 1], 2 * M[:, 0, 2], 2 * M[:, 1, 2],
                    -2 * mp[:, 0], -2 * mp[:, 1], -2 * mp[:, 2], pmp], 1).astype(np.float32)
    h = tf32(psi)
    brow = np.concatenate([h, psi - h, h, np.zeros((len(p), 2), np.float32)], 1)
    nu = (np.abs(sd) * (Rd ** 2).sum(2)).sum(1) * (1 + 1e-6)
    lam = np.abs(M).sum((1, 2)) * (1 + 1e-6)
    p1 = np.abs(pp).sum(1) * (1 + 1e-6)
    info = np.concatenate([o, np.ldexp(np.abs(psi).max(0), -12), [1e-5 * nu.max(), p1.max(), np.ldexp(lam.max(), -20)]])
    return brow, info.astype(np.float32)


def query_rows(q, info):
    """A rows [m, 32] and the bound E [m] of queries against one tile."""
    x = (q - info[:3]).astype(np.float32)
    X, Y, Z = x[:, 0], x[:, 1], x[:, 2]
    ph = np.stack([X * X, Y * Y, Z * Z, X * Y, X * Z, Y * Z, X, Y, Z, np.ones_like(X)], 1).astype(np.float32)
    h = tf32(ph)
    arow = np.concatenate([h, h, ph - h, np.zeros((len(q), 2), np.float32)], 1)
    q1 = np.abs(x).sum(1, dtype=np.float32)
    e1 = (np.abs(ph) * info[3:13]).sum(1, dtype=np.float32)
    s1 = q1 + info[14]
    E = (e1 + info[13] * s1 * s1 + info[15] * q1 * s1 + np.float32(1e-30)) * np.float32(1.001)
    return arow, E.astype(np.float32)


def gemm_tf32(arow, brow, toward_zero):
    a, b = tf32(arow).astype(np.float64), tf32(brow).astype(np.float64)
    acc = np.zeros((len(a), len(b)), np.float32)
    for k in range(a.shape[1]):
        exact = acc.astype(np.float64) + np.outer(a[:, k], b[:, k])
        r = exact.astype(np.float32)
        if toward_zero:  # round the partial sum toward zero instead of to nearest
            away = np.abs(r.astype(np.float64)) > np.abs(exact)
            r = np.where(away, np.nextafter(r, np.float32(0)), r)
        acc = r
    return acc


def cloud(kind, rng, Q=256, P=384):
    q = rng.random((Q, 3), dtype=np.float32)
    p = rng.random((P, 3), dtype=np.float32)
    sigma = (0.05 + 0.15 * rng.random((P, 3))).astype(np.float32)
    R = np.linalg.qr(rng.standard_normal((P, 3, 3)))[0].astype(np.float32)
    if kind == "readme":
        sigma = rng.random((P, 3), dtype=np.float32)
        R = rng.random((P, 3, 3), dtype=np.float32)
    elif kind == "shell":
        n = rng.standard_normal((P, 3))
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        p = (n * (1 + 0.01 * rng.standard_normal((P, 1)))).astype(np.float32)
        s = rng.standard_normal((Q, 3))
        s /= np.linalg.norm(s, axis=1, keepdims=True)
        q = (s + 0.05 * rng.standard_normal((Q, 3))).astype(np.float32)
        sigma = np.tile(np.float32([0.02, 0.02, 0.005]), (P, 1))
    elif kind == "offset":
        q, p = (q + 1000).astype(np.float32), (p + 1000).astype(np.float32)
    elif kind == "tiny":
        q, p = (q * 1e-3).astype(np.float32), (p * 1e-3).astype(np.float32)
        sigma = (sigma * 1e6).astype(np.float32)
    elif kind == "aniso":
        sigma = (10.0 ** rng.uniform(-3, 3, (P, 3))).astype(np.float32)
    elif kind == "negative":
        sigma = rng.uniform(-0.2, 0.2, (P, 3)).astype(np.float32)
    return q, p, sigma, R


@pytest.mark.parametrize("kind", ["table", "readme", "shell", "offset", "tiny", "aniso", "negative"])
def test_approximate_keys_within_the_bound(kind):
    rng = np.random.default_rng(zlib.crc32(kind.encode()))
    q, p, sigma, R = cloud(kind, rng)
    exact = O.keys_f32(torch.from_numpy(q[None]), torch.from_numpy(p[None]), torch.from_numpy(sigma[None]),
                       torch.from_numpy(R[None]))[0].astype(np.float64)
    worst = 0.0
    for t0 in range(0, len(p), TP):
        sl = slice(t0, t0 + TP)
        brow, info = tile_operand(p[sl], sigma[sl], R[sl])
        arow, E = query_rows(q, info)
        for toward_zero in (False, True):
            approx = gemm_tf32(arow, brow, toward_zero).astype(np.float64)
            err = np.abs(approx - exact[:, sl])
            worst = max(worst, float((err / E[:, None].astype(np.float64)).max()))
    assert worst <= 0.25, f"approximation error reaches {worst:.3f} of the bound"


def test_padding_rows_are_never_candidates():
    """A padding row (psi = (0, .., 1e30)) gives an approximate key near 1e30:
    above every finite threshold + bound, so no padding point is examined."""
    rng = np.random.default_rng(7)
    q, p, sigma, R = cloud("table", rng, Q=64, P=100)
    brow, info = tile_operand(p, sigma, R)
    psi = np.zeros((1, 10), np.float32)
    psi[0, 9] = np.float32(1e30)
    h = tf32(psi)
    pad = np.concatenate([h, psi - h, h, np.zeros((1, 2), np.float32)], 1)
    arow, E = query_rows(q, info)
    approx = gemm_tf32(arow, pad, False)[:, 0]
    assert (approx > 1e29).all() and (E < 1e3).all()
