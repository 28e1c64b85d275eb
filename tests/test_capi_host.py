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


def _header_prototypes():
    """{name: (return class, [parameter classes])} parsed from the header,
    classes being 'ptr', 'int', 'size', 'i64' or 'void'."""
    import re
    from cuda_knn_aggregate import capi

    text = re.sub(r"/\*.*?\*/", " ", open(capi.HEADER).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"(const\s+char\s*\*|int|size_t|void|long\s+long)\s+(knnag_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, params = m.group(1), m.group(2), m.group(3)

        def cls(decl):
            decl = decl.strip()
            if "*" in decl:
                return "ptr"
            if decl.startswith("size_t"):
                return "size"
            if decl.startswith("long long") or decl.startswith("int64_t"):
                return "i64"
            if decl.startswith("int"):
                return "int"
            return decl

        args = [] if params.strip() in ("", "void") else [cls(p) for p in params.split(",")]
        protos[name] = (cls(ret) if ret != "void" else "void", args)
    return protos


def test_ctypes_signatures_match_header():
    """Every signature the ctypes binding declares has the header's
    parameter count and kinds (pointer, int, size_t, 64-bit int) and return
    kind, so a change of the C ABI cannot leave the binding behind."""
    from cuda_knn_aggregate import capi

    kind = {ctypes.c_void_p: "ptr", ctypes.c_char_p: "ptr", ctypes.c_int: "int", ctypes.c_size_t: "size",
            ctypes.c_longlong: "i64", None: "void"}
    protos = _header_prototypes()
    assert len(protos) >= len(capi._SIGS)
    for name, (args, res) in capi._SIGS.items():
        assert name in protos, name
        ret, hargs = protos[name]
        assert [kind[a] for a in args] == hargs, name
        assert kind[res] == ret, name
