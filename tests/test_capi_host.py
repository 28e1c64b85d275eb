"""Host-only checks of the C ABI and the package (no GPU needed): the library
loads and exports every function include/knn_aniso.h declares, sizes are
reported, and argument validation returns its status codes before any
device work."""
import ctypes

import pytest
import torch


def test_library_exports_every_header_symbol():
    from cuda_knn_aggregate import capi

    lib = capi.lib()
    names = capi.header_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
    assert lib.knnag_version() >= 10000


def test_status_strings():
    from cuda_knn_aggregate import capi

    lib = capi.lib()
    for code in range(8):
        assert lib.knnag_status_string(code)
    assert b"K" in lib.knnag_status_string(2)


def test_workspace_queries():
    from cuda_knn_aggregate import capi

    lib = capi.lib()
    a = lib.knnag_forward_workspace_bytes(2, 12288, 4096, 64, 16, capi.F32)
    b = lib.knnag_forward_workspace_bytes(2, 12288, 4096, 64, 40, capi.F32)
    assert a > b > 0  # K > 32 needs no pair tiles
    assert lib.knnag_points_bytes(2, 4096, capi.F32) == 2 * 4096 * 64
    assert lib.knnag_adjacency_bytes(2, 12288, 4096, 16) >= 2 * 2 * 12288 * 16 * 4
    assert lib.knnag_backward_workspace_bytes(2, 12288, 4096, 64, 16, capi.F64) > 0


def test_validation_before_device_work():
    from cuda_knn_aggregate import capi

    lib = capi.lib()
    V = ctypes.c_void_p
    one = V(16)  # never dereferenced: validation fails first
    ws = V(256)
    args = [one] * 5 + [1, 4, 8, 2, 9, 0] + [one] * 4 + [None, ws, 1 << 20, None]
    assert lib.knnag_forward(*args) == 2  # K > P
    args[9] = 4
    args[10] = 7
    assert lib.knnag_forward(*args) == 3  # dtype
    args[10] = 0
    args[0] = None
    assert lib.knnag_forward(*args) == 1  # null q
    args[0] = one
    args[17] = 16
    assert lib.knnag_forward(*args) == 4  # workspace too small
    args[5] = 0
    assert lib.knnag_forward(*args) == 0  # B = 0: nothing to do


def test_misaligned_record_buffers_rejected():
    """Packed records and cloud sets are read with 16-byte loads and bulk
    copies: a buffer that is not 16-byte aligned is refused before any
    device work."""
    from cuda_knn_aggregate import capi

    lib = capi.lib()
    V = ctypes.c_void_p
    one, odd = V(16), V(24)  # never dereferenced
    assert lib.knnag_pack_points(one, one, one, 1, 4, capi.F32, odd, None) == 1
    P = (ctypes.c_int * 1)(100)
    nb = lib.knnag_cloudset_bytes(1, P)
    assert lib.knnag_cloudset_init(1, P, odd, nb, None) == 1
    assert lib.knnag_cloudset_init(1, P, None, nb, None) == 1


def test_python_api_rejects_cpu_tensors():
    from cuda_knn_aggregate import knn_aggregate_aniso

    t = [torch.rand(1, 4, 3), torch.rand(1, 8, 3), torch.rand(1, 8, 2), torch.rand(1, 8, 3), torch.rand(1, 8, 3, 3)]
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        knn_aggregate_aniso(*t, 2)


def test_workload_generators():
    from cuda_knn_aggregate import workloads as W

    shape, (q, p, f, sigma, R) = W.make("small")
    assert q.shape == (2, 1000, 3) and f.shape == (2, 500, 32) and R.shape == (2, 500, 3, 3)
    eye = torch.eye(3).expand_as(R)
    assert torch.allclose(R @ R.transpose(-1, -2), eye, atol=1e-5)
    assert sigma.min() >= 0.05 and sigma.max() <= 0.2
    _, (q2, *_r) = W.make("small")
    assert torch.equal(q, q2)  # seeded
    _, (q, p, f, sigma, R) = W.make("sphere", Q=1000, P=2000, F=8)
    n = R[..., :, 2]
    assert torch.allclose((p / p.norm(dim=-1, keepdim=True) * n).sum(-1), torch.ones(1, 2000), atol=1e-5)
    assert torch.allclose(sigma[0, 0], torch.tensor([0.02, 0.02, 0.005]))
