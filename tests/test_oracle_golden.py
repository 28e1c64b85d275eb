"""Pin the CPU oracle against fixtures produced by the reference extension.

The fixtures in tests/golden were made by tests/golden/make_golden.py, which
runs the reference's own CUDA ops (compiled from its sources by
oracle/build_ref.py) on a B200.  Here, with no GPU, the oracle must reproduce:

* ``idxs`` and ``dists`` bit for bit -- this fixes the FP32 contraction order
  of the key (csrc/forward.cu:88-92) and the MinK tie rules (csrc/mink.cuh);
* ``w_out`` and ``f_out`` within 1e-5 relative to the tensor's max;
* the first-order (csrc/backward.cu:5-121) and second-order
  (csrc/backward.cu:124-328) gradients within 1e-4 relative to each tensor's max.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN_CASES, GOLDEN_DIR, rel_err
import oracle as O

FWD_TOL = 1e-5
GRAD_TOL = 1e-4


def load(name):
    return np.load(os.path.join(GOLDEN_DIR, f"ref_{name}.npz"))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_forward_bit_exact(name):
    z = load(name)
    K = int(z["K"])
    fo, w, d, idx = O.forward_f32(z["q"], z["p"], z["f"], z["sigma"], z["R"], K)
    assert np.array_equal(idx, z["idxs"].astype(np.int64))
    assert np.array_equal(d.view(np.int32), z["dists"].view(np.int32))
    assert rel_err(w, z["w_out"]) < FWD_TOL
    assert rel_err(fo, z["f_out"]) < FWD_TOL


def test_ties_case_really_has_ties():
    """The lattice fixture must exercise MinK's history-dependent tie order:
    for these queries the reference order differs from (key, index) order."""
    z = load("ties")
    K = int(z["K"])
    keys = O.keys_f32(z["q"], z["p"], z["sigma"], z["R"])
    top = np.sort(keys, -1)[..., : K + 1]
    assert (np.diff(top, axis=-1) == 0).any(-1).all()
    order = np.argsort(keys, axis=-1, kind="stable")[..., :K]
    assert (order != z["idxs"]).any(-1).sum() > 0


def test_other_contractions_do_not_match():
    """Only the pinned contraction reproduces the reference's keys."""
    z = load("allkeys")
    K = int(z["K"])
    hits = []
    for jm in range(5):
        for sm in range(4):
            _, _, d, idx = O.forward_f32(z["q"], z["p"], z["f"], z["sigma"], z["R"], K, mode=(jm, sm),
                                         with_features=False)
            hits.append(np.array_equal(d.view(np.int32), z["dists"].view(np.int32)))
    assert hits[0] and sum(hits) == 1


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_gradients_vs_reference(name):
    z = load(name)
    t = lambda k: torch.from_numpy(z[k]).double()
    idx = torch.from_numpy(z["idxs"]).long()
    first, second = O.grads64(t("q"), t("p"), t("f"), t("sigma"), t("R"), idx, t("gfo"), t("ggq"))
    for n, g in zip(("dq", "dp", "df", "dsigma", "dR"), first):
        assert rel_err(g.numpy(), z["b1_" + n]) < GRAD_TOL, n
    for n, g in zip(("dgfo", "dq", "dp", "df", "dsigma", "dR"), second):
        assert rel_err(g.numpy(), z["b2_" + n]) < GRAD_TOL, n


def test_plain_forward_matches_oracle_small():
    """The plain-PyTorch formulation (FP64) agrees with the C oracle away from ties."""
    z = load("small")
    K = int(z["K"])
    t = lambda k: torch.from_numpy(z[k]).double()
    f_out, w, d, idx = O.plain_forward(t("q"), t("p"), t("f"), t("sigma"), t("R"), K)
    same = (idx.numpy() == z["idxs"]).all(-1)
    assert same.mean() > 0.99
    assert rel_err(f_out.numpy()[same], z["f_out"][same]) < FWD_TOL


def test_oracle_rejects_bad_k():
    z = load("k_eq_p")
    with pytest.raises(ValueError):
        O.forward_f32(z["q"], z["p"], z["f"], z["sigma"], z["R"], z["p"].shape[1] + 1)
