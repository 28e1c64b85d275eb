"""Failure detection on the GPU without a fault: the search kernels' waits
on their tile copies are bounded, and one that runs out latches an error
the host reads back, while the kernel returns and the context stays usable.

The test hook knnag_debug_set_search_stall arms the mbarrier of one tile
visit but never issues its copy -- a phase that nothing completes -- with a
wait budget of a few hundred microseconds.  No kernel faults or traps.
"""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
STALL_SPINS = 2000  # x 256 ns sleeps: about half a millisecond per wait


def _inputs(seed=41):
    from cuda_knn_aggregate import workloads as W

    shape, t = W.make("small", B=1, Q=256, P=1000, F=8, K=8, seed=seed)
    return shape, t, [a.to(DEV) for a in t]


def _forward_into(capi, x, K, outs, ws):
    q, p, f, sigma, R = x
    B, Q, P, F = q.shape[0], q.shape[1], p.shape[1], f.shape[2]
    return capi.lib().knnag_forward(*[capi._p(a) for a in x], B, Q, P, F, K, capi.F32,
                                    *[capi._p(a) for a in outs], None, capi._p(ws), ws.numel(),
                                    capi._stream(DEV))


def test_search_wait_timeout_latches_error_and_writes_nothing():
    from cuda_knn_aggregate import capi

    shape, t, x = _inputs()
    B, Q, P, F, K = shape.B, shape.Q, shape.P, shape.F, shape.K
    outs = [torch.full((B, Q, F), -7.0, device=DEV), torch.full((B, Q, K), -7.0, device=DEV),
            torch.full((B, Q, K), -7.0, device=DEV), torch.full((B, Q, K), -7, dtype=torch.int64, device=DEV)]
    nb = capi.lib().knnag_forward_workspace_bytes(B, Q, P, F, K, capi.F32)
    ws = torch.empty(nb, dtype=torch.uint8, device=DEV)
    capi.debug_set_search_stall(0, STALL_SPINS)
    try:
        assert _forward_into(capi, x, K, outs, ws) == 0  # enqueued
        torch.cuda.synchronize()  # every kernel returned
        assert capi.read_device_status(ws, DEV) == 7  # KNNAG_ERR_DEVICE latched
    finally:
        capi.debug_set_search_stall(-1, 0)
    for o in outs:
        assert bool((o == -7).all()), "a timed-out search CTA must not write outputs"
    # the status word was cleared by the read; the context is still usable
    assert capi.read_device_status(ws, DEV) == 0
    assert _forward_into(capi, x, K, outs, ws) == 0
    assert capi.read_device_status(ws, DEV) == 0
    _, _, d_ref, i_ref = O.forward_f32(*t, K, with_features=False)
    assert np.array_equal(outs[3].cpu().numpy(), i_ref)
    assert np.array_equal(outs[2].cpu().numpy().view(np.int32), d_ref.view(np.int32))


def test_torch_path_reports_latched_errors_when_asked(monkeypatch):
    from cuda_knn_aggregate import capi, knn_aggregate_aniso

    shape, _, x = _inputs(seed=42)
    monkeypatch.setenv("KNNAG_CHECK_DEVICE_STATUS", "1")
    capi.debug_set_search_stall(0, STALL_SPINS)
    try:
        with pytest.raises(RuntimeError, match="latched on the device"):
            knn_aggregate_aniso(*x, shape.K)
    finally:
        capi.debug_set_search_stall(-1, 0)
    out = knn_aggregate_aniso(*x, shape.K)  # checked, and clean
    monkeypatch.setenv("KNNAG_CHECK_DEVICE_STATUS", "0")
    again = knn_aggregate_aniso(*x, shape.K)
    assert torch.equal(out[3], again[3])
