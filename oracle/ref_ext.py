"""The reference extension, run through the reference package's own autograd
wiring -- TEST AND COMPARISON INFRASTRUCTURE ONLY.

``oracle/_ref/knn_ref_C.so`` is the reference project's ``_C`` module compiled
from its own sources by ``oracle/build_ref.py``.  This module loads it and
wraps its three differentiable ops exactly as the reference's
``cuda_knn_aggregate/__init__.py`` does (``KNNAnisotropicAggregate``
``:64-117``: forward saves ``(q, p, f, sigma, R, w_out, idxs)``;
``KNNAnisotropicAggregateBackward`` ``:216-289``: its forward runs the
first-order op, its backward the second-order op with ``grad_grad_q``
only), so a training step on it is the reference's training step.  Used by
the parity tests as the bit-exact reference and by ``bench.py`` as the timed
north-star comparator; never by the product.
"""
from __future__ import annotations

import importlib.util
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "knn_ref_C.so")

_MOD = None


def load():
    """(module, None) or (None, reason) when the extension was not built."""
    global _MOD
    if _MOD is not None:
        return _MOD, None
    if not os.path.exists(REF_SO):
        return None, "reference extension not built (oracle/build_ref.py needs the reference checkout)"
    spec = importlib.util.spec_from_file_location("knn_ref_C", REF_SO)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    _MOD = mod
    return mod, None


def op(ref=None):
    """knn_aggregate_aniso of the reference package on the reference
    extension: ``op(q, p, f, sigma, R, K) -> (f_out, w_out, dists, idxs)``."""
    if ref is None:
        ref, why = load()
        if ref is None:
            raise RuntimeError(why)

    class RefBackward(torch.autograd.Function):
        @staticmethod
        def forward(ctx, gfo, gwo, q, p, f, sigma, R, w_out, idxs):
            outs = ref.knn_aggregate_aniso_backward(gfo, gwo, q, p, f, sigma, R, w_out, idxs)
            ctx.save_for_backward(gfo, gwo, q, p, f, sigma, R, w_out, idxs)
            return tuple(outs)

        @staticmethod
        def backward(ctx, ggq, ggp, ggf, ggs, ggR):
            gfo, gwo, q, p, f, sigma, R, w_out, idxs = ctx.saved_tensors
            o = ref.knn_aggregate_aniso_backward_2nd(ggq.contiguous(), gfo.contiguous(), gwo.contiguous(), q, p, f,
                                                     sigma, R, w_out, idxs)
            return o[0], None, o[1], o[2], o[3], o[4], o[5], None, None

    class RefAgg(torch.autograd.Function):
        @staticmethod
        def forward(ctx, q, p, f, sigma, R, K):
            f_out, w_out, dists, idxs = ref.knn_aggregate_aniso_forward(q, p, f, sigma, R, K)
            ctx.save_for_backward(q, p, f, sigma, R, w_out, idxs)
            return f_out, w_out, dists, idxs

        @staticmethod
        def backward(ctx, gfo, gwo, gd, gi):
            q, p, f, sigma, R, w_out, idxs = ctx.saved_tensors
            g = RefBackward.apply(gfo.contiguous(), gwo.contiguous(), q, p, f, sigma, R, w_out, idxs)
            return (*g, None)

    return RefAgg.apply
