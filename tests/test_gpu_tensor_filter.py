"""GPU parity of the tensor-core filtered search (launch shape code 128).

The tensor-core search (csrc/knn_search_tc.cu) replaces the key loop of the
reference's forward (csrc/forward.cu:83-95) with approximate keys from a
tcgen05 TF32 GEMM plus a rigorous error bound, and recomputes the exact FP32
key of every candidate.  Its results must equal the reference's bit for bit:
idxs / dists / w_out / f_out against the reference extension's fixtures and
the CPU oracle, and bit-identical to the CUDA-core search on the same inputs,
including inputs that stress the bound (README non-orthonormal R, a thin
sphere shell, a cloud offset by 1000, a cloud scaled by 1e-3, extreme
anisotropy, negative precisions), ties (every query tied), non-finite values,
every K bucket, the counting forward, and the bounded-wait timeout path.
Every call goes through the C ABI.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN_CASES, GOLDEN_DIR, rel_err
import oracle as O
from test_tensor_filter_bound import cloud

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
TC = 128
FWD_TOL = 1e-5


@pytest.fixture(autouse=True)
def _restore_setting():
    from cuda_knn_aggregate import capi

    yield
    capi.set_search_splits(0)


def _forward(t, K, splits):
    from cuda_knn_aggregate import capi

    capi.set_search_splits(splits)
    out = capi.forward(*t, K)
    torch.cuda.synchronize()
    return [o.cpu() for o in out]


def _bits(x):
    return x.view(torch.int32) if x.dtype == torch.float32 else x


def _identical(a, b):
    return all(torch.equal(_bits(x), _bits(y)) for x, y in zip(a, b))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_matches_reference_extension_fixtures(name):
    z = np.load(os.path.join(GOLDEN_DIR, f"ref_{name}.npz"))
    t = [torch.from_numpy(z[k]).to(DEV) for k in ("q", "p", "f", "sigma", "R")]
    K = int(z["K"])
    f_out, w_out, dists, idxs = _forward(t, K, TC)
    assert np.array_equal(idxs.numpy(), z["idxs"].astype(np.int64))
    assert np.array_equal(dists.numpy().view(np.int32), z["dists"].view(np.int32))
    assert np.array_equal(w_out.numpy().view(np.int32), z["w_out"].view(np.int32))
    assert np.array_equal(f_out.numpy().view(np.int32), z["f_out"].view(np.int32))


@pytest.mark.parametrize("kind", ["table", "readme", "shell", "offset", "tiny", "aniso", "negative"])
def test_stress_inputs_match_oracle_and_cuda_core(kind):
    import zlib

    rng = np.random.default_rng(zlib.crc32(kind.encode()) + 1)
    q, p, sigma, R = cloud(kind, rng, Q=3000, P=2500)
    f = rng.random((len(p), 12), dtype=np.float32)
    t = [torch.from_numpy(x[None].copy()) for x in (q, p, f, sigma, R)]
    K = 16
    got = _forward([x.to(DEV) for x in t], K, TC)
    fo64, w64, d_ref, i_ref = O.forward_f32(*t, K)
    assert np.array_equal(got[3].numpy(), i_ref)
    assert np.array_equal(got[2].numpy().view(np.int32), d_ref.view(np.int32))
    assert rel_err(got[0].numpy(), fo64) < FWD_TOL
    assert _identical(got, _forward([x.to(DEV) for x in t], K, 8))


@pytest.mark.parametrize("K", [1, 5, 8, 9, 16, 17, 32])
def test_every_k_bucket_matches_oracle(K):
    from cuda_knn_aggregate import workloads as W

    _, t = W.make("small", B=2, Q=1500, P=1200, F=16, K=K, seed=500 + K)
    got = _forward([x.to(DEV) for x in t], K, TC)
    _, _, d_ref, i_ref = O.forward_f32(*t, K, with_features=False)
    assert np.array_equal(got[3].numpy(), i_ref)
    assert np.array_equal(got[2].numpy().view(np.int32), d_ref.view(np.int32))


def test_table_and_sphere_sample_identical_to_cuda_core():
    from cuda_knn_aggregate import workloads as W

    for name, kw in (("table", {}), ("sphere", {"Q": 131072})):
        shape, t = W.make(name, **kw)
        x = [a.to(DEV) for a in t]
        assert _identical(_forward(x, shape.K, TC), _forward(x, shape.K, 8)), name


def test_non_finite_values_take_the_exact_replay():
    """A NaN record among points 0..K-1 (MinK's fill phase), an infinite
    sigma elsewhere and a NaN query: the affected queries are flagged and
    replayed, and every result equals the oracle's."""
    from cuda_knn_aggregate import workloads as W

    _, (q, p, f, sigma, R) = W.make("small", B=1, Q=700, P=900, F=8, K=12, seed=61)
    p[0, 3, 1] = float("nan")
    sigma[0, 500, 2] = float("inf")
    q[0, 10, 0] = float("nan")
    t = (q, p, f, sigma, R)
    x = [a.to(DEV) for a in t]
    got = _forward(x, 12, TC)
    _, _, d_ref, i_ref = O.forward_f32(*t, 12, with_features=False)
    assert np.array_equal(got[3].numpy(), i_ref)
    d = got[2].numpy()
    fin = ~np.isnan(d_ref)  # NaN keys: any NaN bit pattern (the host's and the GPU's differ)
    assert np.array_equal(np.isnan(d), ~fin)
    assert np.array_equal(d[fin].view(np.int32), d_ref[fin].view(np.int32))
    assert _identical(got, _forward(x, 12, 8))


def test_counting_forward_counts_the_same_rows():
    from cuda_knn_aggregate import capi, workloads as W

    shape, t = W.make("small", B=2, Q=2000, P=1500, F=8, K=16, seed=62)
    x = [a.to(DEV) for a in t]
    res = []
    for splits in (TC, 8):
        capi.set_search_splits(splits)
        *out, adj = capi.forward_counted(*x, shape.K)
        torch.cuda.synchronize()
        res.append((out[3].cpu(), capi.adjacency_arrays(adj, shape.B, shape.Q, shape.P, shape.K)[0].cpu()))
    assert torch.equal(res[0][0], res[1][0])
    assert torch.equal(res[0][1], res[1][1])


def test_wait_timeout_latches_error_and_writes_nothing():
    from cuda_knn_aggregate import capi
    from test_gpu_failure import STALL_SPINS, _forward_into, _inputs

    shape, t, x = _inputs(seed=63)
    B, Q, P, F, K = shape.B, shape.Q, shape.P, shape.F, shape.K
    outs = [torch.full((B, Q, F), -7.0, device=DEV), torch.full((B, Q, K), -7.0, device=DEV),
            torch.full((B, Q, K), -7.0, device=DEV), torch.full((B, Q, K), -7, dtype=torch.int64, device=DEV)]
    ws = torch.empty(capi.lib().knnag_forward_workspace_bytes(B, Q, P, F, K, capi.F32), dtype=torch.uint8, device=DEV)
    capi.set_search_splits(TC)
    capi.debug_set_search_stall(0, STALL_SPINS)
    try:
        assert _forward_into(capi, x, K, outs, ws) == 0
        torch.cuda.synchronize()
        assert capi.read_device_status(ws, DEV) == 7  # KNNAG_ERR_DEVICE
    finally:
        capi.debug_set_search_stall(-1, 0)
    for o in outs:
        assert bool((o == -7).all()), "a timed-out search CTA must not write outputs"
    assert _forward_into(capi, x, K, outs, ws) == 0
    assert capi.read_device_status(ws, DEV) == 0
    _, _, d_ref, i_ref = O.forward_f32(*t, K, with_features=False)
    assert np.array_equal(outs[3].cpu().numpy(), i_ref)
