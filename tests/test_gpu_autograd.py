"""The autograd layer on the GPU: the Eikonal training step against the FP64
oracle, FP64 gradcheck of the first- and second-order kernels against finite
differences, and the reference-compatible `_C` ops.

Tolerances: forward 1e-5, gradients 1e-4 (relative to each tensor's max).
"""
import numpy as np
import pytest
import torch

from conftest import rel_err
import oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def make(**kw):
    from cuda_knn_aggregate import workloads as W

    dtype = kw.pop("dtype", torch.float32)
    return W.make("small", dtype=dtype, **kw)


def test_eikonal_step_vs_fp64_oracle():
    from cuda_knn_aggregate import knn_aggregate_aniso

    shape, t = make(B=2, Q=1000, P=500, F=32, K=12)
    K = shape.K
    ins = [x.to(DEV).requires_grad_(True) for x in t]
    f_out, w_out, dists, idxs = knn_aggregate_aniso(*ins, K)
    (gq,) = torch.autograd.grad(f_out.sum(), ins[0], create_graph=True)
    loss = ((gq.norm(dim=-1) - 1.0) ** 2).mean()
    loss.backward()

    ref = [x.double().clone().requires_grad_(True) for x in t]
    fo, _ = O.aggregate64(*ref, idxs.cpu())
    (g64,) = torch.autograd.grad(fo.sum(), ref[0], create_graph=True)
    l64 = ((g64.norm(dim=-1) - 1.0) ** 2).mean()
    l64.backward()
    assert rel_err(f_out.detach().cpu().numpy(), fo.detach().numpy()) < 1e-5
    assert rel_err(gq.detach().cpu().numpy(), g64.detach().numpy()) < 1e-4
    assert abs(loss.item() - l64.item()) <= 1e-4 * abs(l64.item())
    for a, b in zip(ins, ref):
        assert rel_err(a.grad.cpu().numpy(), b.grad.numpy()) < 1e-4


def test_full_backward_vs_oracle():
    """loss = <v, f_out>: all first-order gradients through the autograd layer."""
    from cuda_knn_aggregate import knn_aggregate_aniso

    shape, t = make(B=2, Q=700, P=900, F=20, K=16, seed=3)
    ins = [x.to(DEV).requires_grad_(True) for x in t]
    f_out, _, _, idxs = knn_aggregate_aniso(*ins, shape.K)
    v = torch.randn_like(f_out)
    (f_out * v).sum().backward()
    ref = [x.double() for x in t]
    first, _ = O.grads64(*ref, idxs.cpu(), v.double().cpu())
    for a, g in zip(ins, first):
        assert rel_err(a.grad.cpu().numpy(), g.numpy()) < 1e-4


def test_gradients_of_w_out_and_dists_are_ignored():
    """As in the reference, only f_out carries gradient."""
    from cuda_knn_aggregate import knn_aggregate_aniso

    shape, t = make(B=1, Q=64, P=200, F=4, K=8, seed=4)
    ins = [x.to(DEV).requires_grad_(True) for x in t]
    f_out, w_out, dists, _ = knn_aggregate_aniso(*ins, shape.K)
    (w_out.sum() + dists.sum()).backward()
    for a in ins:
        assert a.grad is None or torch.count_nonzero(a.grad) == 0


def test_gradcheck_first_and_second_order_fp64():
    """FP64 finite-difference checks at Q=64, P=128 (F=8, K=4): f_out w.r.t.
    every input, and dL/dq (the Eikonal path) w.r.t. every input."""
    from cuda_knn_aggregate import knn_aggregate_aniso

    shape, t = make(B=1, Q=64, P=128, F=8, K=4, seed=11, dtype=torch.float64)
    K = shape.K
    ins = tuple(x.to(DEV).requires_grad_(True) for x in t)

    def fwd(q, p, f, sigma, R):
        return knn_aggregate_aniso(q, p, f, sigma, R, K)[0]

    assert torch.autograd.gradcheck(fwd, ins, eps=1e-6, atol=1e-7, rtol=1e-4)

    g = torch.Generator().manual_seed(0)
    v = torch.randn(1, 64, 8, generator=g, dtype=torch.float64).to(DEV)

    def dq(q, p, f, sigma, R):
        out = knn_aggregate_aniso(q, p, f, sigma, R, K)[0]
        return torch.autograd.grad((out * v).sum(), q, create_graph=True)[0]

    assert torch.autograd.gradcheck(dq, ins, eps=1e-6, atol=1e-7, rtol=1e-4)


def test_reference_compatible_ops():
    """_C keeps the reference's op names, argument lists and return lists."""
    from cuda_knn_aggregate import _C

    shape, t = make(B=2, Q=100, P=300, F=8, K=6, seed=12)
    q, p, f, sigma, R = [x.to(DEV) for x in t]
    f_out, w_out, dists, idxs = _C.knn_aggregate_aniso_forward(q, p, f, sigma, R, 6)
    gfo = torch.randn_like(f_out)
    gwo = torch.zeros_like(w_out)
    ggq = torch.randn_like(q)
    b1 = _C.knn_aggregate_aniso_backward(gfo, gwo, q, p, f, sigma, R, w_out, idxs)
    b2 = _C.knn_aggregate_aniso_backward_2nd(ggq, gfo, gwo, q, p, f, sigma, R, w_out, idxs)
    assert len(b1) == 5 and len(b2) == 6
    first, second = O.grads64(*[x.double().cpu() for x in (q, p, f, sigma, R)], idxs.cpu(), gfo.double().cpu(),
                              ggq.double().cpu())
    for a, r in zip(b1, first):
        assert rel_err(a.cpu().numpy(), r.numpy()) < 1e-4
    for a, r in zip(b2, second):
        assert rel_err(a.cpu().numpy(), r.numpy()) < 1e-4


def test_function_subclass_written_against_the_reference():
    """KNNAnisotropicAggregate is a torch.autograd.Function: a subclass in the
    reference's style (its own forward saving (q, p, f, sigma, R, w_out,
    idxs), the base class's backward) trains to the same gradients as the
    C++ autograd route of the base class, through both orders."""
    import cuda_knn_aggregate as C

    assert issubclass(C.KNNAnisotropicAggregate, torch.autograd.Function)
    assert issubclass(C.KNNLookupAnisotropicAggregate, C.KNNAnisotropicAggregate)
    assert issubclass(C.KNNPrecomputedAnisotropicAggregate, C.KNNAnisotropicAggregate)

    class Mine(C.KNNAnisotropicAggregate):
        @staticmethod
        def forward(ctx, q, p, f, sigma, R, K):
            f_out, w_out, dists, idxs = C._C.knn_aggregate_aniso_forward(q, p, f, sigma, R, K)
            ctx.save_for_backward(q, p, f, sigma, R, w_out, idxs)
            return f_out, w_out, dists, idxs

    shape, t = make(B=2, Q=300, P=400, F=8, K=8, seed=21)
    results = []
    for name, op in (("base", C.KNNAnisotropicAggregate.apply), ("subclass", Mine.apply),
                     ("precomputed", C.KNNPrecomputedAnisotropicAggregate.apply)):
        ins = [x.to(DEV).requires_grad_(True) for x in t]
        if name == "precomputed":
            idxs = C.knn_aggregate_aniso(*[x.detach() for x in ins], shape.K)[3]
            f_out = op(*ins, idxs, shape.K)[0]
        else:
            f_out = op(*ins, shape.K)[0]
        (gq,) = torch.autograd.grad(f_out.sum(), ins[0], create_graph=True)
        ((gq.norm(dim=-1) - 1.0) ** 2).mean().backward()
        results.append([f_out.detach(), gq.detach()] + [x.grad for x in ins])
    for other in results[1:]:
        for a, b in zip(results[0], other):
            assert rel_err(b.cpu().numpy(), a.cpu().numpy()) < 1e-5


def test_errors_follow_reference_wording():
    from cuda_knn_aggregate import knn_aggregate_aniso

    _, t = make(B=1, Q=8, P=16, F=4, K=4)
    q, p, f, sigma, R = [x.to(DEV) for x in t]
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        knn_aggregate_aniso(q.cpu(), p, f, sigma, R, 4)
    with pytest.raises(RuntimeError, match="must be contiguous"):
        knn_aggregate_aniso(q.transpose(0, 1).contiguous().transpose(0, 1)[:, ::2], p, f, sigma, R, 4)
    with pytest.raises(RuntimeError, match="K must satisfy"):
        knn_aggregate_aniso(q, p, f, sigma, R, 17)


def test_step_is_capturable_in_a_cuda_graph():
    """Forward + autograd.grad(create_graph) + backward replays in a graph with
    the same results as eager execution."""
    from cuda_knn_aggregate import knn_aggregate_aniso

    shape, t = make(B=2, Q=512, P=700, F=16, K=12, seed=13)
    ins = [x.to(DEV).requires_grad_(True) for x in t]

    def step():
        for a in ins:
            a.grad = None
        f_out, _, _, _ = knn_aggregate_aniso(*ins, shape.K)
        (gq,) = torch.autograd.grad(f_out.sum(), ins[0], create_graph=True)
        loss = ((gq.norm(dim=-1) - 1.0) ** 2).mean()
        loss.backward()
        return loss.detach()

    eager = step()
    eager_grads = [a.grad.clone() for a in ins]
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(2):
            step()
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    for a in ins:
        a.grad = None
    with torch.cuda.graph(g):
        out = step()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, eager)
    for a, e in zip(ins, eager_grads):
        assert torch.equal(a.grad, e)


@pytest.mark.gpu
def test_backward_computes_only_requested_gradients():
    """The autograd nodes ask the running graph task which gradients are
    used: autograd.grad(f_out.sum(), q) launches fewer kernels than a request
    for every input (no point-side kernels, no adjacency), with identical dq;
    the Eikonal second order then still gives every input's gradient."""
    import cuda_knn_aggregate as C
    from cuda_knn_aggregate import capi
    from cuda_knn_aggregate import workloads as W

    _, t = W.make("small", seed=5)
    ins = [x.cuda().requires_grad_(True) for x in t]
    f_out = C.knn_aggregate_aniso(*ins, 12)[0]
    c0 = capi.launch_count()
    (dq_only,) = torch.autograd.grad(f_out.sum(), ins[0], retain_graph=True)
    torch.cuda.synchronize()
    n_q = capi.launch_count() - c0
    c0 = capi.launch_count()
    grads_all = torch.autograd.grad(f_out.sum(), ins, retain_graph=True)
    torch.cuda.synchronize()
    n_all = capi.launch_count() - c0
    assert n_q < n_all
    assert torch.equal(dq_only, grads_all[0])
    # Eikonal step: every input gets a second-order gradient
    (gq,) = torch.autograd.grad(f_out.sum(), ins[0], create_graph=True)
    ((gq.norm(dim=-1) - 1.0) ** 2).mean().backward()
    for x in ins:
        assert x.grad is not None and torch.isfinite(x.grad).all()


@pytest.mark.gpu
@pytest.mark.parametrize("F", [1, 5, 64])
def test_broadcast_grad_f_out_matches_dense(F):
    """f_out.sum() hands the backward one value broadcast over [B,Q,F]; the
    kernels then use per-point row sums of f instead of grad_f_out rows.
    First- and second-order (Eikonal) gradients equal the ones computed
    with the same gradient materialised as a dense tensor."""
    import cuda_knn_aggregate as C
    from cuda_knn_aggregate import workloads as W

    _, t = W.make("small", F=F, seed=11)
    res = []
    for dense in (False, True):
        ins = [x.cuda().requires_grad_(True) for x in t]
        f_out = C.knn_aggregate_aniso(*ins, 12)[0]
        if dense:
            first = torch.autograd.grad(f_out, ins, torch.ones_like(f_out).contiguous(), create_graph=True)
        else:
            first = torch.autograd.grad(f_out.sum(), ins, create_graph=True)
        ((first[0].norm(dim=-1) - 1.0) ** 2).mean().backward()
        res.append([g.detach() for g in first] + [x.grad for x in ins])
    for a, b in zip(*res):
        assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < 1e-5
