"""The autotuner's on-disk cache: a process that tunes a shape bucket
writes its choice to the JSON file; a fresh process reads it back and picks
the same launch shape without timing anything, with results identical to
the untuned op (tuned knobs change only the time)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import PKG_DIR

pytestmark = pytest.mark.gpu

CHILD = r"""
import json, sys, torch
sys.path.insert(0, sys.argv[1])
from cuda_knn_aggregate import _C, capi, tuning, workloads as W
shape, t = W.make("table", Q=3000, P=2000, seed=91)
x = [a.cuda() for a in t]
ref = _C.knn_aggregate_aniso_forward(*x, shape.K)
choice = tuning.autotune_search(*x, shape.K, reps=3)
tuning.use_tuned(x[0], x[1], shape.K)
out = _C.knn_aggregate_aniso_forward(*x, shape.K)
same = all(torch.equal(a, b) for a, b in zip(ref, out))
capi.set_search_splits(0)
print(json.dumps({"splits": choice["splits"], "timed": tuning.TIMED["runs"], "same": same,
                  "applied": capi.search_splits()}))
"""


def _run(cache):
    env = dict(os.environ, KNNAG_TUNE_CACHE=str(cache))
    r = subprocess.run([sys.executable, "-c", CHILD, PKG_DIR], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_second_process_reuses_the_cached_choice(tmp_path):
    cache = tmp_path / "tune.json"
    first = _run(cache)
    assert first["timed"] == 8 and first["splits"] in (1, 2, 4, 8, 16, 32, 64, 128) and first["same"]
    data = json.loads(cache.read_text())
    assert any("|uniform|" in k and v["splits"] == first["splits"] for k, v in data.items())
    second = _run(cache)
    assert second["timed"] == 0, "the second process re-timed a cached bucket"
    assert second["splits"] == first["splits"] and second["same"]
