"""The reference's other forward ops: aggregation at precomputed indices
(csrc/forward.cu:186-230), the lookup variant (csrc/forward.cu:113-183) and
the isotropic kNN forward (csrc/forward.cu:5-53).

CPU tests pin the oracle's restatements against fixtures made by the
reference extension (tests/golden/make_golden.py); GPU tests hold this
library's ops, through both the torch extension and the C ABI, to the same
fixtures and to the oracle at larger sizes:

* ``idxs`` and ``dists`` bit for bit;
* ``w_out`` / ``f_out`` within 1e-5 relative to the tensor's max;
* gradients (precomputed / lookup share the main op's adjoint) within 1e-4
  relative to each tensor's max against FP64 autograd at the same indices.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN_DIR, rel_err
import oracle as O

FWD_TOL = 1e-5
GRAD_TOL = 1e-4


def load(name):
    return np.load(os.path.join(GOLDEN_DIR, f"ref_var_{name}.npz"))


def bits_equal(a, b):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    b = np.ascontiguousarray(np.asarray(b, dtype=np.float32))
    return a.shape == b.shape and np.array_equal(a.view(np.int32), b.view(np.int32))


# ----------------------------------------------------------------- CPU: oracle


def test_oracle_precomputed_vs_reference():
    z = load("pre")
    fo, w, d = O.precomputed_f32(z["q"], z["p"], z["f"], z["sigma"], z["R"], z["knn_idxs"])
    assert bits_equal(d, z["dists"])
    assert rel_err(w, z["w_out"]) < FWD_TOL
    assert rel_err(fo, z["f_out"]) < FWD_TOL


@pytest.mark.parametrize("name", ["lookup", "lookup_ties"])
def test_oracle_lookup_vs_reference(name):
    z = load(name)
    fo, w, d, idx = O.lookup_f32(z["q"], z["p"], z["f"], z["sigma"], z["R"], z["knn_table"])
    assert np.array_equal(idx, z["idxs"])
    assert bits_equal(d, z["dists"])
    assert rel_err(w, z["w_out"]) < FWD_TOL
    assert rel_err(fo, z["f_out"]) < FWD_TOL


@pytest.mark.parametrize("name", ["iso", "iso_kp", "iso_ties"])
def test_oracle_isotropic_vs_reference(name):
    z = load(name)
    K = int(z["K"])
    fo, ws, d, idx = O.iso_f32(z["q"], z["p"], z["f"], z["sigma"], K)
    assert np.array_equal(idx, z["idxs"])
    assert bits_equal(d, z["dists"])
    assert rel_err(ws, z["w_out"]) < FWD_TOL
    assert rel_err(fo, z["f_out"]) < FWD_TOL


def test_isotropic_contraction_is_pinned():
    """Of the three ways to contract x*x + y*y + z*z, only ISO_SQ_MODE gives
    the reference's distances on every fixture."""
    hits = []
    for mode in range(3):
        ok = True
        for name in ("iso", "iso_kp", "iso_ties"):
            z = load(name)
            _, _, d, _ = O.iso_f32(z["q"], z["p"], z["f"], z["sigma"], int(z["K"]), mode=mode)
            ok &= bits_equal(d, z["dists"])
        hits.append(ok)
    assert hits[O.ISO_SQ_MODE] and sum(hits) == 1


def test_lookup_contraction_is_pinned():
    """lookup_ties is built so that the three roundings of x*x + y*y + z*z
    pick different nearest points (six points per query at exactly equal
    squared distances in exact arithmetic): only LOOKUP_SQ_MODE reproduces
    the reference extension's nearest points, and each other mode differs
    on some query."""
    z = load("lookup_ties")
    hits = []
    for mode in range(3):
        _, _, d, idx = O.lookup_f32(z["q"], z["p"], z["f"], z["sigma"], z["R"], z["knn_table"], mode=mode)
        hits.append(np.array_equal(idx, z["idxs"]) and bits_equal(d, z["dists"]))
    assert hits[O.LOOKUP_SQ_MODE] and sum(hits) == 1


def test_isotropic_ties_fixture_has_ties():
    z = load("iso_ties")
    d = z["dists"]
    assert (np.diff(d, axis=-1) == 0).any(-1).mean() > 0.5


# ------------------------------------------------------------------ GPU: ops


def _cuda(z, *names):
    return [torch.from_numpy(np.ascontiguousarray(z[n])).cuda() for n in names]


def _check_fwd(outs, ref, names):
    for n, v in zip(names, outs):
        v = v.detach().cpu().numpy()
        if n == "idxs":
            assert np.array_equal(v, ref[n]), n
        elif n == "dists":
            assert bits_equal(v, ref[n]), n
        else:
            assert rel_err(v, ref[n]) < FWD_TOL, n


@pytest.mark.gpu
def test_precomputed_vs_reference_fixture():
    import cuda_knn_aggregate as C
    from cuda_knn_aggregate import capi

    z = load("pre")
    q, p, f, s, R, idx = _cuda(z, "q", "p", "f", "sigma", "R", "knn_idxs")
    K = int(z["K"])
    outs = C._C.knn_precomputed_aggregate_aniso_forward(q, p, f, s, R, idx, K)
    _check_fwd(outs, z, ("f_out", "w_out", "dists"))
    outs = capi.forward_precomputed(q, p, f, s, R, idx)
    torch.cuda.synchronize()
    _check_fwd(outs, z, ("f_out", "w_out", "dists"))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["lookup", "lookup_ties"])
def test_lookup_vs_reference_fixture(name):
    import cuda_knn_aggregate as C
    from cuda_knn_aggregate import capi

    z = load(name)
    q, p, f, s, R, table = _cuda(z, "q", "p", "f", "sigma", "R", "knn_table")
    K = int(z["K"])
    outs = C.knn_aggregate_aniso_lookup(q, p, f, s, R, table, K)
    _check_fwd(outs, z, ("f_out", "w_out", "dists", "idxs"))
    outs = capi.forward_lookup(q, p, f, s, R, table, K)
    torch.cuda.synchronize()
    _check_fwd(outs, z, ("f_out", "w_out", "dists", "idxs"))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["iso", "iso_kp", "iso_ties"])
def test_isotropic_vs_reference_fixture(name):
    import cuda_knn_aggregate as C
    from cuda_knn_aggregate import capi

    z = load(name)
    q, p, f, s = _cuda(z, "q", "p", "f", "sigma")
    K = int(z["K"])
    outs = C._C.knn_aggregate_forward(q, p, f, s, K)
    _check_fwd(outs, z, ("f_out", "w_out", "dists", "idxs"))
    outs = capi.forward_isotropic(q, p, f, s, K)
    torch.cuda.synchronize()
    _check_fwd(outs, z, ("f_out", "w_out", "dists", "idxs"))


def _cloud(B, Q, P, F, seed, S=3):
    g = torch.Generator().manual_seed(seed)
    q = torch.rand(B, Q, 3, generator=g) * 2 - 1
    p = torch.rand(B, P, 3, generator=g) * 2 - 1
    f = torch.randn(B, P, F, generator=g)
    sigma = 4.0 + 60.0 * torch.rand(B, P, S, generator=g)
    A = torch.randn(B, P, 3, 3, generator=g, dtype=torch.float64)
    R = torch.linalg.qr(A)[0].float().contiguous()
    return q, p, f, sigma, R


@pytest.mark.gpu
@pytest.mark.parametrize("B,Q,P,F,K", [(2, 20000, 6000, 16, 8), (1, 5000, 3000, 3, 32), (3, 777, 129, 1, 1)])
def test_precomputed_vs_oracle(B, Q, P, F, K):
    import cuda_knn_aggregate as C

    q, p, f, s, R = _cloud(B, Q, P, F, seed=B * 7 + K)
    g = torch.Generator().manual_seed(K)
    idx = torch.randint(0, P, (B, Q, K), generator=g)
    # indices outside [0, P) contribute nothing (dist = +inf, w = 0)
    idx[0, ::97, 0] = -1
    idx[-1, ::89, -1] = P + 3
    fo, w, d = O.precomputed_f32(q, p, f, s, R, idx)
    outs = C._C.knn_precomputed_aggregate_aniso_forward(*[t.cuda() for t in (q, p, f, s, R, idx)], K)
    _check_fwd(outs, dict(f_out=fo, w_out=w, dists=d), ("f_out", "w_out", "dists"))
    assert np.isinf(outs[2][0, ::97, 0].cpu().numpy()).all()


@pytest.mark.gpu
@pytest.mark.parametrize("B,Q,P,F,K,cols", [(2, 20000, 5000, 8, 8, 8), (1, 3000, 700, 4, 5, 16)])
def test_lookup_vs_oracle(B, Q, P, F, K, cols):
    import cuda_knn_aggregate as C

    q, p, f, s, R = _cloud(B, Q, P, F, seed=31 + K)
    g = torch.Generator().manual_seed(cols)
    table = torch.randint(0, P, (P, cols), generator=g)
    fo, w, d, idx = O.lookup_f32(q, p, f, s, R, table[:, :K].contiguous())
    outs = C.knn_aggregate_aniso_lookup(*[t.cuda() for t in (q, p, f, s, R, table)], K)
    _check_fwd(outs, dict(f_out=fo, w_out=w, dists=d, idxs=idx), ("f_out", "w_out", "dists", "idxs"))


@pytest.mark.gpu
@pytest.mark.parametrize("B,Q,P,F,K,S", [(2, 8000, 5000, 8, 16, 1), (1, 3000, 2000, 4, 48, 3), (2, 500, 7, 2, 7, 1)])
def test_isotropic_vs_oracle(B, Q, P, F, K, S):
    import cuda_knn_aggregate as C

    q, p, f, s, _ = _cloud(B, Q, P, F, seed=5 + K, S=S)
    s = (s / 60.0).contiguous()
    fo, ws, d, idx = O.iso_f32(q, p, f, s, K)
    outs = C._C.knn_aggregate_forward(*[t.cuda() for t in (q, p, f, s)], K)
    _check_fwd(outs, dict(f_out=fo, w_out=ws, dists=d, idxs=idx), ("f_out", "w_out", "dists", "idxs"))


@pytest.mark.gpu
def test_variants_float64():
    """FP64 inputs run the same kernels in double (exp in double)."""
    import cuda_knn_aggregate as C

    q, p, f, s, R = [t.double().cuda() for t in _cloud(1, 600, 300, 4, seed=9)]
    idx = torch.randint(0, 300, (1, 600, 6), generator=torch.Generator().manual_seed(3)).cuda()
    f_out, w_out, dists = C._C.knn_precomputed_aggregate_aniso_forward(q, p, f, s, R, idx, 6)
    ref = O.aggregate64(q.cpu(), p.cpu(), f.cpu(), s.cpu(), R.cpu(), idx.cpu())
    assert rel_err(f_out.cpu().numpy(), ref[0].numpy()) < 1e-12
    fo, ws, d, ix = C._C.knn_aggregate_forward(q, p, f, s[..., :1].contiguous(), 5)
    d64 = ((q.cpu()[0][:, None, :] - p.cpu()[0][None]) ** 2).sum(-1)
    top = torch.topk(d64, 5, dim=-1, largest=False).values
    assert torch.allclose(d.cpu()[0], top, rtol=1e-12, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["precomputed", "lookup"])
def test_variant_gradients(variant):
    """First- and second-order (Eikonal) gradients through the variants match
    FP64 autograd of the plain formula at the same indices."""
    import cuda_knn_aggregate as C

    B, Q, P, F, K = 2, 3000, 1500, 8, 8
    q, p, f, s, R = _cloud(B, Q, P, F, seed=77)
    g = torch.Generator().manual_seed(78)
    gfo = torch.randn(B, Q, F, generator=g)
    ggq = torch.randn(B, Q, 3, generator=g)
    dev = [t.cuda().requires_grad_(True) for t in (q, p, f, s, R)]
    if variant == "precomputed":
        idx = torch.randint(0, P, (B, Q, K), generator=g).cuda()
        f_out, _, _ = C.KNNPrecomputedAnisotropicAggregate.apply(*dev, idx, K)
    else:
        table = torch.randint(0, P, (P, K), generator=g).cuda()
        f_out, _, _, idx = C.KNNLookupAnisotropicAggregate.apply(*dev, table, K)
    grads = torch.autograd.grad(f_out, dev, gfo.cuda(), create_graph=True)
    (grads[0] * ggq.cuda()).sum().backward()
    first, second = O.grads64(*[t.double() for t in (q, p, f, s, R)], idx.cpu(), gfo.double(), ggq.double())
    for n, a, b in zip(("dq", "dp", "df", "dsigma", "dR"), grads, first):
        assert rel_err(a.detach().cpu().numpy(), b.numpy()) < GRAD_TOL, n
    for n, t, b in zip(("dq", "dp", "df", "dsigma", "dR"), dev, second[1:]):
        assert rel_err(t.grad.cpu().numpy(), b.numpy()) < GRAD_TOL, n
