"""GPU parity of the CUDA path against the reference extension's fixtures and
the CPU oracle.

Bars (stated per test): idxs and dists bit-exact; w_out / f_out within 1e-5
of the FP64 oracle (relative to the tensor's max); gradients within 1e-4 of
the FP64 oracle and of the reference's own backward.  Every forward /
backward here goes through the C ABI (cuda_knn_aggregate.capi) unless the
test is about the autograd layer.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN_CASES, GOLDEN_DIR, rel_err
import oracle as O

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-5
GRAD_TOL = 1e-4


def capi():
    from cuda_knn_aggregate import capi as C

    return C


def load(name):
    z = np.load(os.path.join(GOLDEN_DIR, f"ref_{name}.npz"))
    dev = torch.device("cuda:0")
    t = {k: torch.from_numpy(z[k]).to(dev) for k in ("q", "p", "f", "sigma", "R", "gfo", "ggq")}
    t["idxs"] = torch.from_numpy(z["idxs"].astype(np.int64)).to(dev)
    return z, t, int(z["K"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_forward_matches_reference_extension(name):
    z, t, K = load(name)
    f_out, w_out, dists, idxs = capi().forward(t["q"], t["p"], t["f"], t["sigma"], t["R"], K)
    torch.cuda.synchronize()
    assert np.array_equal(idxs.cpu().numpy(), z["idxs"].astype(np.int64))
    assert np.array_equal(dists.cpu().numpy().view(np.int32), z["dists"].view(np.int32))
    assert rel_err(w_out.cpu().numpy(), z["w_out"]) < FWD_TOL
    assert rel_err(f_out.cpu().numpy(), z["f_out"]) < FWD_TOL


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_forward_weights_and_features_bit_exact(name):
    """Same __expf and the same k-order fma accumulation as the reference."""
    z, t, K = load(name)
    f_out, w_out, _, _ = capi().forward(t["q"], t["p"], t["f"], t["sigma"], t["R"], K)
    torch.cuda.synchronize()
    assert np.array_equal(w_out.cpu().numpy().view(np.int32), z["w_out"].view(np.int32))
    assert np.array_equal(f_out.cpu().numpy().view(np.int32), z["f_out"].view(np.int32))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_backward_matches_reference_and_oracle(name):
    z, t, K = load(name)
    C = capi()
    args = (t["q"], t["p"], t["f"], t["sigma"], t["R"])
    dq, dp, df, ds, dR, coef = C.backward(t["gfo"], *args, t["idxs"], want_coef=True)
    dgfo, dq2, dp2, df2, ds2, dR2 = C.backward_2nd(t["ggq"], t["gfo"], *args, t["idxs"], coef=coef)
    torch.cuda.synchronize()
    tt = lambda k: torch.from_numpy(z[k]).double()
    first, second = O.grads64(tt("q"), tt("p"), tt("f"), tt("sigma"), tt("R"), torch.from_numpy(z["idxs"]).long(),
                              tt("gfo"), tt("ggq"))
    for got, n, ref in zip((dq, dp, df, ds, dR), ("dq", "dp", "df", "dsigma", "dR"), first):
        assert rel_err(got.cpu().numpy(), z["b1_" + n]) < GRAD_TOL, n
        assert rel_err(got.cpu().numpy(), ref.numpy()) < GRAD_TOL, n
    for got, n, ref in zip((dgfo, dq2, dp2, df2, ds2, dR2), ("dgfo", "dq", "dp", "df", "dsigma", "dR"), second):
        assert rel_err(got.cpu().numpy(), z["b2_" + n]) < GRAD_TOL, n
        assert rel_err(got.cpu().numpy(), ref.numpy()) < GRAD_TOL, n


def test_second_order_without_saved_coef_matches():
    z, t, K = load("small")
    C = capi()
    args = (t["q"], t["p"], t["f"], t["sigma"], t["R"])
    _, _, _, _, _, coef = C.backward(t["gfo"], *args, t["idxs"], want_coef=True)
    a = C.backward_2nd(t["ggq"], t["gfo"], *args, t["idxs"], coef=coef)
    b = C.backward_2nd(t["ggq"], t["gfo"], *args, t["idxs"], coef=None)
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_backward_is_deterministic():
    z, t, K = load("small")
    C = capi()
    args = (t["gfo"], t["q"], t["p"], t["f"], t["sigma"], t["R"], t["idxs"])
    r1 = C.backward(*args)
    r2 = C.backward(*args)
    for x, y in zip(r1[:5], r2[:5]):
        assert torch.equal(x, y)


@pytest.mark.parametrize("shape", [
    dict(B=2, Q=2048, P=4096, F=64, K=16),   # the timing-table point count
    dict(B=3, Q=333, P=1000, F=5, K=7),      # ragged tiles, F not a multiple of 4
    dict(B=1, Q=97, P=300, F=16, K=32),      # largest register list
    dict(B=1, Q=64, P=100, F=8, K=40),       # K > 32: exact MinK kernel for every query
    dict(B=2, Q=50, P=33, F=3, K=33),        # K == P
    dict(B=1, Q=4000, P=257, F=4, K=1),      # K = 1, one point past a tile
])
def test_forward_random_vs_oracle(shape):
    K = shape.pop("K")
    _, (q, p, f, sigma, R) = __import__("cuda_knn_aggregate").workloads.make("small", K=K, **shape, seed=77)
    fo64, w64, d_ref, i_ref = O.forward_f32(q, p, f, sigma, R, K)
    dev = torch.device("cuda:0")
    f_out, w_out, dists, idxs = capi().forward(*[x.to(dev) for x in (q, p, f, sigma, R)], K)
    torch.cuda.synchronize()
    assert np.array_equal(idxs.cpu().numpy(), i_ref)
    assert np.array_equal(dists.cpu().numpy().view(np.int32), d_ref.view(np.int32))
    assert rel_err(w_out.cpu().numpy(), w64) < FWD_TOL
    assert rel_err(f_out.cpu().numpy(), fo64) < FWD_TOL


def test_readme_inputs_sphere_inputs_vs_oracle():
    from cuda_knn_aggregate import workloads as W

    dev = torch.device("cuda:0")
    cases = [(W.readme_cloud(2, 1500, 700, 12, seed=3), 12),
             (W.make("sphere", Q=3000, P=5000, F=8)[1], 16)]
    for (q, p, f, sigma, R), K in cases:
        fo64, w64, d_ref, i_ref = O.forward_f32(q, p, f, sigma, R, K)
        f_out, w_out, dists, idxs = capi().forward(*[x.to(dev) for x in (q, p, f, sigma, R)], K)
        assert np.array_equal(idxs.cpu().numpy(), i_ref)
        assert np.array_equal(dists.cpu().numpy().view(np.int32), d_ref.view(np.int32))
        assert rel_err(f_out.cpu().numpy(), fo64) < FWD_TOL


def test_nan_in_fill_phase_follows_reference_rules():
    """A NaN key among points 0..K-1 is kept by MinK's fill phase; the exact
    replay must reproduce that (NaN is compared bitwise as a NaN)."""
    from cuda_knn_aggregate import workloads as W

    _, (q, p, f, sigma, R) = W.make("small", B=1, Q=64, P=200, F=4, seed=9)
    sigma[0, 3, 1] = float("nan")
    K = 8
    _, _, d_ref, i_ref = O.forward_f32(q, p, f, sigma, R, K, with_features=False)
    dev = torch.device("cuda:0")
    _, _, dists, idxs = capi().forward(*[x.to(dev) for x in (q, p, f, sigma, R)], K)
    assert np.array_equal(idxs.cpu().numpy(), i_ref)
    d = dists.cpu().numpy()
    assert np.array_equal(np.isnan(d), np.isnan(d_ref))
    assert np.array_equal(np.nan_to_num(d).view(np.int32), np.nan_to_num(d_ref).view(np.int32))


def test_float64_path():
    from cuda_knn_aggregate import workloads as W

    _, (q, p, f, sigma, R) = W.make("small", B=2, Q=300, P=400, F=6, seed=5, dtype=torch.float64)
    K = 9
    dev = torch.device("cuda:0")
    f_out, w_out, dists, idxs = capi().forward(*[x.to(dev) for x in (q, p, f, sigma, R)], K)
    ks = O.all_keys(q, p, sigma, R)
    ref = torch.topk(ks, K, dim=-1, largest=False, sorted=True)
    same = (ref.indices == idxs.cpu()).all(-1)
    assert same.float().mean() > 0.99
    fo, w = O.aggregate64(q, p, f, sigma, R, idxs.cpu())
    assert rel_err(f_out.cpu().numpy(), fo.numpy()) < 1e-12
    assert rel_err(w_out.cpu().numpy(), w.numpy()) < 1e-12


def test_capi_rejects_bad_arguments():
    C = capi()
    dev = torch.device("cuda:0")
    q = torch.rand(1, 4, 3, device=dev)
    p = torch.rand(1, 5, 3, device=dev)
    with pytest.raises(RuntimeError, match="K must satisfy"):
        C.forward(q, p, torch.rand(1, 5, 2, device=dev), torch.rand(1, 5, 3, device=dev),
                  torch.rand(1, 5, 3, 3, device=dev), 6)


@pytest.mark.gpu
def test_search_splits_setting_does_not_change_results():
    """The process-wide split setting (and the autotuner that picks it)
    changes only the time: every split gives identical outputs."""
    import cuda_knn_aggregate as C
    from cuda_knn_aggregate import capi, tuning
    from cuda_knn_aggregate import workloads as W

    _, t = W.make("table", Q=3000, P=2000, seed=77)
    ins = [x.cuda() for x in t]
    outs = []
    try:
        for g in (1, 2, 4, 8, 16, 32, 64, 0):
            capi.set_search_splits(g)
            outs.append(C._C.knn_aggregate_aniso_forward(*ins, 16))
        best = tuning.autotune_search_splits(*ins, 16)
        assert best in (1, 2, 4, 8, 16, 32, 64)
        tuning.use_tuned(ins[0], ins[1], 16)
        assert capi.search_splits() == best
        outs.append(C._C.knn_aggregate_aniso_forward(*ins, 16))
    finally:
        capi.set_search_splits(0)
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert torch.equal(a, b)
    with pytest.raises(RuntimeError):
        capi.set_search_splits(3)


@pytest.mark.parametrize("shape", [dict(B=2, Q=3000, P=2000, F=16, K=16), dict(B=1, Q=500, P=300, F=8, K=40),
                                   dict(B=2, Q=200, P=300, F=6, K=9, dtype=torch.float64)])
def test_counting_forward_gives_the_same_adjacency(shape):
    """knnag_forward_counted + knnag_build_adjacency_counted: the same outputs
    as knnag_forward and the same rowptr / sorted entries as a full
    knnag_build_adjacency, on the search path, the exact path (K > 32) and
    FP64."""
    from cuda_knn_aggregate import workloads as W

    shape = dict(shape)
    K = shape.pop("K")
    dtype = shape.pop("dtype", torch.float32)
    _, t = W.make("small", K=K, seed=61, dtype=dtype, **shape)
    x = [a.cuda() for a in t]
    C = capi()
    ref = C.forward(*x, K)
    *outs, adj = C.forward_counted(*x, K)
    for a, b in zip(ref, outs):
        assert torch.equal(a, b)
    B, Q, P = shape["B"], shape["Q"], shape["P"]
    full = C.build_adjacency(ref[3], P)
    torch.cuda.synchronize()
    r0, e0 = C.adjacency_arrays(full, B, Q, P, K)
    r1, e1 = C.adjacency_arrays(adj, B, Q, P, K)
    assert torch.equal(r0, r1) and torch.equal(e0, e1)
