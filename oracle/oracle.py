"""CPU oracle for ``knn_aggregate_aniso`` -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker or the timed CPU
baseline; the product never routes through it.

Two layers:

* ``forward_f32`` -- the C restatement in ``knn_oracle.c`` of the reference
  forward (``csrc/forward.cu:83-109`` with ``csrc/mink.cuh:60-112``): FP32 keys
  emulated bit-exactly in the reference compiler's contraction order
  (``KEY_MODE``, pinned against fixtures made by the reference extension), the
  reference's exact MinK insertion/eviction/sort rules, and FP64 weights and
  feature sums.  Gives bit-exact ``idxs``/``dists`` and FP64 ``w_out``/``f_out``.
* ``aggregate64`` / ``grads64`` / ``plain_forward`` -- the op restated in plain
  PyTorch (the formula of ``README.md:13-22``): ``f_out = sum_k exp(-s_k)
  f[idx_k]`` with ``s = sum_i sigma_i (R_i . (q - p))^2``.  Torch autograd on
  it gives first-order gradients (what ``csrc/backward.cu:5-121`` computes) and
  the second-order Eikonal gradients (``csrc/backward.cu:124-328``).  As in
  the reference (``cuda_knn_aggregate/__init__.py:93-117``), only ``f_out``
  carries gradient; ``w_out`` and ``dists`` are returned detached.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "liboracle.so")
SRC = os.path.join(HERE, "knn_oracle.c")

# Contraction order of the reference build's FP32 key (see knn_oracle.c
# row_dot/quad_form): 0,0 = j = fma(R2, z, fma(R0, x, R1*y)),
# s = fma(l*l, s2, fma(j*j, s0, (k*k)*s1)).  Pinned by tests/test_oracle_golden.py.
KEY_MODE = (0, 0)


def build_lib(force: bool = False) -> str:
    """Compile knn_oracle.c into oracle/_build/liboracle.so (gcc, no contraction)."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(SRC):
        tmp = LIB_PATH + f".tmp{os.getpid()}"
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
                               "-std=c11", SRC, "-lm", "-o", tmp])
        os.replace(tmp, LIB_PATH)
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(build_lib())
        P = ctypes.c_void_p
        I = ctypes.c_int
        L.oracle_keys_f32.argtypes = [P, P, P, P, I, I, I, I, I, P]
        L.oracle_forward_f32.argtypes = [P, P, P, P, P, I, I, I, I, I, I, I, P, P, P, P]
        L.oracle_num_threads.restype = I
        _LIB = L
    return _LIB


def _np32(t):
    if isinstance(t, torch.Tensor):
        t = t.detach().cpu().numpy()
    return np.ascontiguousarray(t, dtype=np.float32)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def keys_f32(q, p, sigma, R, mode=KEY_MODE):
    """Every pair's FP32 key, [B,Q,P] (csrc/forward.cu:85-92)."""
    q, p, sigma, R = map(_np32, (q, p, sigma, R))
    B, Q, P = q.shape[0], q.shape[1], p.shape[1]
    out = np.empty((B, Q, P), np.float32)
    lib().oracle_keys_f32(_ptr(q), _ptr(p), _ptr(sigma), _ptr(R), B, Q, P, mode[0], mode[1], _ptr(out))
    return out


def forward_f32(q, p, f, sigma, R, K, mode=KEY_MODE, with_features=True):
    """Reference forward on the CPU: (fout64, w64, dists f32, idxs int64)."""
    q, p, f, sigma, R = map(_np32, (q, p, f, sigma, R))
    B, Q, P, F = q.shape[0], q.shape[1], p.shape[1], f.shape[2]
    if not 1 <= K <= P:
        raise ValueError(f"oracle needs 1 <= K <= P (K={K}, P={P})")
    idxs = np.empty((B, Q, K), np.int64)
    dists = np.empty((B, Q, K), np.float32)
    w64 = np.empty((B, Q, K), np.float64)
    fo = np.empty((B, Q, F), np.float64) if with_features else None
    lib().oracle_forward_f32(_ptr(q), _ptr(p), _ptr(f), _ptr(sigma), _ptr(R), B, Q, P, F, K, mode[0], mode[1],
                             _ptr(idxs), _ptr(dists), _ptr(w64), _ptr(fo))
    return fo, w64, dists, idxs


# ----------------------------------------------------------------------------
# Plain PyTorch restatement (any dtype/device); differentiable in q,p,f,sigma,R
# ----------------------------------------------------------------------------

def _gather_points(x, idxs):
    """x [B,P,...] gathered at idxs [B,Q,K] -> [B,Q,K,...]."""
    B, Q, K = idxs.shape
    flat = idxs.reshape(B, Q * K)
    tail = x.shape[2:]
    ix = flat.reshape(B, Q * K, *([1] * len(tail))).expand(B, Q * K, *tail)
    return torch.gather(x, 1, ix).reshape(B, Q, K, *tail)


def keys_at(q, p, sigma, R, idxs):
    """s for the pairs named by idxs: [B,Q,K] (csrc/forward.cu:85-92)."""
    pk = _gather_points(p, idxs)
    Rk = _gather_points(R, idxs)
    sk = _gather_points(sigma, idxs)
    d = q.unsqueeze(2) - pk                              # [B,Q,K,3]
    u = torch.einsum("bqkim,bqkm->bqki", Rk, d)           # rows of R dotted with d
    return (sk * u * u).sum(-1)


def aggregate64(q, p, f, sigma, R, idxs):
    """(f_out, w) at fixed neighbour indices; f_out differentiable, w = exp(-s)."""
    s = keys_at(q, p, sigma, R, idxs)
    w = torch.exp(-s)
    fk = _gather_points(f, idxs)
    return (w.unsqueeze(-1) * fk).sum(2), w


def all_keys(q, p, sigma, R):
    """Every pair's key in the plain formulation, [B,Q,P]."""
    d = q.unsqueeze(2) - p.unsqueeze(1)                  # [B,Q,P,3]
    u = torch.einsum("bpim,bqpm->bqpi", R, d)
    return (sigma.unsqueeze(1) * u * u).sum(-1)


def plain_forward(q, p, f, sigma, R, K, chunk=1024):
    """The whole op in plain PyTorch: brute-force keys, top-K (torch.topk,
    ascending), weights and weighted sum.  Ties are ordered by torch, not by
    the reference's MinK rules.  Returns (f_out, w_out, dists, idxs)."""
    B, Q = q.shape[0], q.shape[1]
    with torch.no_grad():
        idx_chunks = []
        for s0 in range(0, Q, chunk):
            ks = all_keys(q[:, s0:s0 + chunk], p, sigma, R)
            idx_chunks.append(torch.topk(ks, K, dim=-1, largest=False, sorted=True).indices)
        idxs = torch.cat(idx_chunks, 1)
    s = keys_at(q, p, sigma, R, idxs)
    w = torch.exp(-s)
    f_out = (w.unsqueeze(-1) * _gather_points(f, idxs)).sum(2)
    return f_out, w.detach(), s.detach(), idxs


def grads64(q, p, f, sigma, R, idxs, gfo, ggq=None):
    """First-order gradients of <gfo, f_out> w.r.t. (q, p, f, sigma, R) at fixed
    idxs, and -- when ggq is given -- the second-order gradients of
    <ggq, dq> w.r.t. (gfo, q, p, f, sigma, R), i.e. what the reference's
    backward (csrc/backward.cu:5-121) and double backward
    (csrc/backward.cu:124-328) return.  Computed in the inputs' dtype."""
    ins = [t.detach().clone().requires_grad_(True) for t in (q, p, f, sigma, R)]
    g = gfo.detach().clone().requires_grad_(ggq is not None)
    f_out, _ = aggregate64(*ins, idxs)
    first = torch.autograd.grad(f_out, ins, grad_outputs=g, create_graph=ggq is not None)
    if ggq is None:
        return tuple(t.detach() for t in first), None
    second = torch.autograd.grad(first[0], [g] + ins, grad_outputs=ggq, allow_unused=True)
    second = tuple(torch.zeros_like(x) if s is None else s.detach() for s, x in zip(second, [g] + ins))
    return tuple(t.detach() for t in first), second


def eikonal_step(q, p, f, sigma, R, K, forward=plain_forward):
    """The timed training step: forward, dq = d(sum f_out)/dq with
    create_graph, Eikonal loss mean((|dq| - 1)^2), backward into every input.
    Returns (loss, f_out, idxs)."""
    f_out, w, d, idxs = forward(q, p, f, sigma, R, K)
    (gq,) = torch.autograd.grad(f_out.sum(), q, create_graph=True)
    loss = ((gq.norm(dim=-1) - 1.0) ** 2).mean()
    loss.backward()
    return loss.detach(), f_out.detach(), idxs


def eikonal_grads64(q, p, f, sigma, R, idxs, chunk=2048):
    """The timed step's gradients in FP64 at fixed idxs, chunked over the
    queries so that full-size workloads fit in host memory: dq = d(sum
    f_out)/dq per query, loss = mean((|dq| - 1)^2) over all B*Q queries, and
    d loss / d(q, p, f, sigma, R) -- each chunk's share of the loss is
    back-propagated on its own and the point-side gradients accumulate.
    Returns (loss, dq [B,Q,3], (grad_q, grad_p, grad_f, grad_sigma, grad_R))."""
    B, Q = q.shape[0], q.shape[1]
    pp, ff, ss, RR = [x.detach().double().clone().requires_grad_(True) for x in (p, f, sigma, R)]
    dq = torch.empty(B, Q, 3, dtype=torch.float64)
    gq = torch.empty(B, Q, 3, dtype=torch.float64)
    loss = 0.0
    for s0 in range(0, Q, chunk):
        qc = q[:, s0:s0 + chunk].detach().double().clone().requires_grad_(True)
        fo, _ = aggregate64(qc, pp, ff, ss, RR, idxs[:, s0:s0 + chunk])
        (g,) = torch.autograd.grad(fo.sum(), qc, create_graph=True)
        lc = ((g.norm(dim=-1) - 1.0) ** 2).sum() / (B * Q)
        lc.backward()
        dq[:, s0:s0 + chunk] = g.detach()
        gq[:, s0:s0 + chunk] = qc.grad
        loss += float(lc.detach())
    return loss, dq, (gq, pp.grad, ff.grad, ss.grad, RR.grad)


# ----------------------------------------------------------------------------
# Variants of the forward (reference csrc/forward.cu:5-53, 113-183, 186-230)
# ----------------------------------------------------------------------------

# Contraction order of the squared Euclidean distances of the lookup and
# isotropic kernels (knn_oracle.c sq_dist3), pinned by tests/test_oracle_golden.py.
LOOKUP_SQ_MODE = 0
ISO_SQ_MODE = 1


def _variant_lib():
    L = lib()
    if not hasattr(L, "_variants_ready"):
        P = ctypes.c_void_p
        I = ctypes.c_int
        L.oracle_precomputed_f32.argtypes = [P] * 6 + [I] * 5 + [P, P, P]
        L.oracle_lookup_f32.argtypes = [P] * 6 + [I] * 6 + [P, P, P, P]
        L.oracle_iso_f32.argtypes = [P] * 4 + [I] * 7 + [P, P, P, P]
        L._variants_ready = True
    return L


def precomputed_f32(q, p, f, sigma, R, idxs):
    """(fout64, w64, dists f32) at given neighbour indices [B,Q,K]."""
    q, p, f, sigma, R = map(_np32, (q, p, f, sigma, R))
    idxs = np.ascontiguousarray(idxs.cpu().numpy() if isinstance(idxs, torch.Tensor) else idxs, dtype=np.int64)
    B, Q, P, F = q.shape[0], q.shape[1], p.shape[1], f.shape[2]
    K = idxs.shape[2]
    d = np.empty((B, Q, K), np.float32)
    w = np.empty((B, Q, K), np.float64)
    fo = np.empty((B, Q, F), np.float64)
    _variant_lib().oracle_precomputed_f32(_ptr(q), _ptr(p), _ptr(f), _ptr(sigma), _ptr(R), _ptr(idxs), B, Q, P, F, K,
                                          _ptr(d), _ptr(w), _ptr(fo))
    return fo, w, d


def lookup_f32(q, p, f, sigma, R, table, mode=None):
    """(fout64, w64, dists f32, idxs int64) of the lookup variant."""
    q, p, f, sigma, R = map(_np32, (q, p, f, sigma, R))
    table = np.ascontiguousarray(table.cpu().numpy() if isinstance(table, torch.Tensor) else table, dtype=np.int64)
    B, Q, P, F = q.shape[0], q.shape[1], p.shape[1], f.shape[2]
    K = table.shape[1]
    idxs = np.empty((B, Q, K), np.int64)
    d = np.empty((B, Q, K), np.float32)
    w = np.empty((B, Q, K), np.float64)
    fo = np.empty((B, Q, F), np.float64)
    _variant_lib().oracle_lookup_f32(_ptr(q), _ptr(p), _ptr(f), _ptr(sigma), _ptr(R), _ptr(table), B, Q, P, F, K,
                                     LOOKUP_SQ_MODE if mode is None else mode, _ptr(idxs), _ptr(d), _ptr(w), _ptr(fo))
    return fo, w, d, idxs


def iso_f32(q, p, f, sigma, K, mode=None):
    """(fout64, wsum64 [B,Q,1], dists f32, idxs int64) of the isotropic forward;
    sigma [B,P,S], component 0 is used."""
    q, p, f, sigma = map(_np32, (q, p, f, sigma))
    B, Q, P, F, S = q.shape[0], q.shape[1], p.shape[1], f.shape[2], sigma.shape[2]
    idxs = np.empty((B, Q, K), np.int64)
    d = np.empty((B, Q, K), np.float32)
    ws = np.empty((B, Q, 1), np.float64)
    fo = np.empty((B, Q, F), np.float64)
    _variant_lib().oracle_iso_f32(_ptr(q), _ptr(p), _ptr(f), _ptr(sigma), B, Q, P, F, K, S,
                                  ISO_SQ_MODE if mode is None else mode, _ptr(idxs), _ptr(d), _ptr(ws), _ptr(fo))
    return fo, ws, d, idxs
