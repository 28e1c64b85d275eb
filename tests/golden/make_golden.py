"""Generate the golden fixtures in this directory by running the reference
extension itself.

Run on a machine with a CUDA GPU, after ``python oracle/build_ref.py`` has
compiled the reference's own ``csrc`` sources into ``oracle/_ref/knn_ref_C.so``:

    python tests/golden/make_golden.py --out tests/golden

Each case draws seeded inputs on the CPU, copies them to ``cuda:0``, calls the
reference ops ``knn_aggregate_aniso_forward`` (``csrc/forward.cu:286-338``),
``knn_aggregate_aniso_backward`` (``csrc/backward.cu:331-389``) and
``knn_aggregate_aniso_backward_2nd`` (``csrc/backward.cu:392-455``) exactly as
the reference's autograd Functions do (``cuda_knn_aggregate/__init__.py:88,
235, 276``, with a zero ``grad_w_out``), and stores inputs and outputs in one
compressed ``.npz`` per case.  The inputs are stored too, so the fixtures
stand alone: the CPU tests never regenerate them.
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "cuda-knn-aniso-gaussian-feature-aggregation_b200"))
from cuda_knn_aggregate import workloads as W  # noqa: E402


def load_ref():
    path = os.path.join(ROOT, "oracle", "_ref", "knn_ref_C.so")
    spec = importlib.util.spec_from_file_location("knn_ref_C", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cases():
    """(name, (q,p,f,sigma,R), K, seed for the incoming gradients)."""
    out = []
    shape, t = W.make("small")
    out.append(("small", t, shape.K))
    out.append(("readme", W.readme_cloud(2, 300, 200, 16, seed=11), 8))
    out.append(("ties", W.lattice_ties(B=2, n_side=4, Q=96, F=8, seed=7), 8))
    _, t = W.make("small", B=1, Q=128, P=16, F=8, seed=21)
    out.append(("k_eq_p", t, 16))
    _, t = W.make("small", B=2, Q=200, P=300, F=5, seed=22)
    out.append(("k1_f5", t, 1))
    _, t = W.make("small", B=1, Q=150, P=200, F=1, seed=23)
    out.append(("f1", t, 7))
    _, t = W.make("small", B=1, Q=256, P=128, F=4, seed=24)
    out.append(("allkeys", t, 128))
    _, t = W.make("small", B=1, Q=128, P=4096, F=8, seed=25)
    out.append(("table_slice", t, 16))
    return out


def run_case(ref, tensors, K, seed):
    q, p, f, sigma, R = [x.cuda().contiguous() for x in tensors]
    B, Q, F = q.shape[0], q.shape[1], f.shape[2]
    f_out, w_out, dists, idxs = ref.knn_aggregate_aniso_forward(q, p, f, sigma, R, K)
    g = torch.Generator().manual_seed(seed)
    gfo = torch.randn(B, Q, F, generator=g).cuda()
    ggq = torch.randn(B, Q, 3, generator=g).cuda()
    gwo = torch.zeros(B, Q, K, device="cuda")
    b1 = ref.knn_aggregate_aniso_backward(gfo, gwo, q, p, f, sigma, R, w_out, idxs)
    b2 = ref.knn_aggregate_aniso_backward_2nd(ggq, gfo, gwo, q, p, f, sigma, R, w_out, idxs)
    torch.cuda.synchronize()
    c = lambda x: x.detach().cpu().numpy()
    rec = dict(q=c(q), p=c(p), f=c(f), sigma=c(sigma), R=c(R), K=np.int64(K),
               f_out=c(f_out), w_out=c(w_out), dists=c(dists), idxs=c(idxs).astype(np.int32),
               gfo=c(gfo), ggq=c(ggq))
    for n, v in zip(("dq", "dp", "df", "dsigma", "dR"), b1):
        rec["b1_" + n] = c(v)
    for n, v in zip(("dgfo", "dq", "dp", "df", "dsigma", "dR"), b2):
        rec["b2_" + n] = c(v)
    return rec


def variant_cases():
    """Fixtures of the reference's other forward ops (csrc/forward.cu:5-53,
    113-183, 186-230): isotropic kNN, lookup through a neighbour table, and
    aggregation at precomputed indices."""
    out = []
    g = torch.Generator().manual_seed(600)
    _, t = W.make("small", B=2, Q=300, P=400, F=12, seed=41)
    q, p, f, sigma, R = t
    # precomputed: indices of the aniso kNN of another query set plus random ones
    idx = torch.randint(0, 400, (2, 300, 9), generator=g)
    out.append(("pre", dict(q=q, p=p, f=f, sigma=sigma, R=R, knn_idxs=idx, K=9)))
    # lookup: table = the 10 Euclidean nearest points of every point of batch 0
    d = ((p[0][:, None, :] - p[0][None, :, :]) ** 2).sum(-1)
    table = torch.topk(d, 10, dim=-1, largest=False).indices
    out.append(("lookup", dict(q=q, p=p, f=f, sigma=sigma, R=R, knn_table=table, K=10)))
    # isotropic: sigma [B,P,1]
    s1 = 0.5 + torch.rand(2, 400, 1, generator=g)
    out.append(("iso", dict(q=q, p=p, f=f, sigma=s1.contiguous(), K=12)))
    _, t = W.make("small", B=1, Q=200, P=64, F=4, seed=42)
    q, p, f, sigma, R = t
    out.append(("iso_kp", dict(q=q, p=p, f=f, sigma=sigma[..., :1].contiguous(), K=64)))
    lt = W.lattice_ties(B=1, n_side=4, Q=64, F=4, seed=8)
    out.append(("iso_ties", dict(q=lt[0], p=lt[1], f=lt[2], sigma=lt[3][..., :1].contiguous(), K=8)))
    q, p, f, sigma, R, table = lookup_ties()
    out.append(("lookup_ties", dict(q=q, p=p, f=f, sigma=sigma, R=R, knn_table=table, K=6)))
    return out


def lookup_ties(n_side=5, seed=607, F=4):
    """Lookup input whose nearest point depends on how x*x + y*y + z*z is
    rounded: every query q (a float in [1, 2)^3) has six points q - d for
    the six permutations d of one offset (a, b, c), each coordinate a
    multiple of 2^-23, so q - p is exact and the six squared distances are
    equal in exact arithmetic; their FP32 values differ only by the order
    of the rounded operations.  The clusters are 0.18 apart, so each
    query's nearest point is one of its own six."""
    import itertools

    g = torch.Generator().manual_seed(seed)
    ax = 1.05 + 0.18 * torch.arange(n_side, dtype=torch.float64)
    qc = torch.stack(torch.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
    qc = (qc + 0.02 * torch.rand(qc.shape, generator=g, dtype=torch.float64)).float().double()
    Q = qc.shape[0]
    k = torch.randint(100000, 160000, (Q, 3), generator=g).double() * 2.0 ** -23
    offs = torch.stack([k[:, list(pm)] for pm in itertools.permutations(range(3))], 1)
    pts = (qc[:, None, :] - offs).reshape(-1, 3)
    pts = pts[torch.randperm(pts.shape[0], generator=g)]
    P = pts.shape[0]
    q, p = qc.float()[None].contiguous(), pts.float()[None].contiguous()
    assert torch.equal(p.double()[0], pts), "points must be exact in FP32"
    f = torch.rand(1, P, F, generator=g)
    sigma = (0.05 + 0.15 * torch.rand(1, P, 3, generator=g)).contiguous()
    R = W.random_rotations(P, g).reshape(1, P, 3, 3).contiguous()
    d = ((pts[:, None, :] - pts[None, :, :]) ** 2).sum(-1)
    table = torch.topk(d, 6, dim=-1, largest=False).indices
    return q, p, f, sigma, R, table


def run_variant(ref, name, c):
    dev = lambda x: x.cuda().contiguous()
    rec = {k: (v.numpy() if isinstance(v, torch.Tensor) else np.int64(v)) for k, v in c.items()}
    if name == "pre":
        o = ref.knn_precomputed_aggregate_aniso_forward(*[dev(c[k]) for k in ("q", "p", "f", "sigma", "R", "knn_idxs")],
                                                        c["K"])
        names = ("f_out", "w_out", "dists")
    elif name.startswith("lookup"):
        o = ref.knn_lookup_aggregate_aniso_forward(*[dev(c[k]) for k in ("q", "p", "f", "sigma", "R", "knn_table")],
                                                   c["K"])
        names = ("f_out", "w_out", "dists", "idxs")
    else:
        o = ref.knn_aggregate_forward(*[dev(c[k]) for k in ("q", "p", "f", "sigma")], c["K"])
        names = ("f_out", "w_out", "dists", "idxs")
    torch.cuda.synchronize()
    for n, v in zip(names, o):
        rec[n] = v.detach().cpu().numpy()
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--only-variants", action="store_true")
    ap.add_argument("--only", default=None, help="generate this one variant case (e.g. lookup_ties)")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    ref = load_ref()
    for i, (name, t, K) in enumerate(cases()):
        if a.only_variants or a.only:
            break
        rec = run_case(ref, t, K, seed=500 + i)
        path = os.path.join(a.out, f"ref_{name}.npz")
        np.savez_compressed(path, **rec)
        print(f"{name}: {os.path.getsize(path)} bytes")
    for name, c in variant_cases():
        if a.only and name != a.only:
            continue
        rec = run_variant(ref, name, c)
        path = os.path.join(a.out, f"ref_var_{name}.npz")
        np.savez_compressed(path, **rec)
        print(f"var_{name}: {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
