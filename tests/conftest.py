import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "cuda-knn-aniso-gaussian-feature-aggregation_b200")
for p in (ROOT, PKG_DIR, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")

# the tests' autotuner choices go to a private file, not the user's cache
if "KNNAG_TUNE_CACHE" not in os.environ:
    import tempfile

    os.environ["KNNAG_TUNE_CACHE"] = os.path.join(tempfile.mkdtemp(prefix="knnag_tune_"), "tune.json")
GOLDEN_CASES = ["small", "readme", "ties", "k_eq_p", "k1_f5", "f1", "allkeys"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200 / sm_100a)")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU on this machine")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def rel_err(a, b):
    """max |a - b| / max |b| (0 when both are zero)."""
    import numpy as np

    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max() if b.size else 0.0
    num = np.abs(a - b).max() if b.size else 0.0
    return 0.0 if num == 0 else num / max(den, 1e-300)
