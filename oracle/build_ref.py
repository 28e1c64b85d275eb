"""Build recipe for the reference extension, compiled from its own sources.

Test infrastructure only.  This compiles the reference project's three
sources -- ``csrc/knn_aggregate.cpp``, ``csrc/forward.cu`` and
``csrc/backward.cu`` of LemonATsu/CUDA-kNN-Aniso-Gaussian-Feature-Aggregation --
where they lie in the read-only reference checkout, with nvcc/g++ directly
(the reference's own ``setup.py`` is not run), into one Python extension
module ``oracle/_ref/knn_ref_C.so`` that exports the reference's six ``_C``
ops unchanged.

Flags mirror the reference's ``setup.py:24-32`` (``-O2`` for both compilers,
no fast-math, so nvcc's default ``-fmad=true`` contraction applies) plus the
defines torch's ``BuildExtension`` adds; the arch is ``sm_100`` as torch would
pick on a B200.  The module is used on the GPU box as the bit-exact reference
for ``idxs``/``dists`` and as the timed reference extension.  Nothing here is
imported by the product.

Usage: ``python oracle/build_ref.py [--src DIR]``.  The checkout is ``--src``,
else the ``KNN_REFERENCE_SRC`` environment variable, else a directory named
``reference`` beside this repository's root.  Exits 0 without building when
the checkout is absent (as on a machine that only runs the prebuilt module).
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
MODULE = "knn_ref_C"
REPO_ROOT = os.path.dirname(HERE)


def default_src() -> str:
    """Location of the reference checkout: $KNN_REFERENCE_SRC, else
    ``<parent of the repository root>/reference``."""
    env = os.environ.get("KNN_REFERENCE_SRC")
    if env:
        return env
    return os.path.join(os.path.dirname(REPO_ROOT), "reference")


def _torch_paths():
    import torch  # noqa: F401
    from torch.utils import cpp_extension as ce

    incs = ce.include_paths(device_type="cuda")
    libs = ce.library_paths(device_type="cuda")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    return incs, libs, abi


def build(src_root: str | None = None, verbose: bool = True) -> str | None:
    csrc = os.path.join(src_root or default_src(), "csrc")
    if not os.path.isdir(csrc):
        if verbose:
            print(f"[build_ref] reference sources not found at {csrc}; skipping")
        return None
    os.makedirs(OUT_DIR, exist_ok=True)
    out = os.path.join(OUT_DIR, MODULE + ".so")
    srcs = [os.path.join(csrc, n) for n in ("knn_aggregate.cpp", "forward.cu", "backward.cu")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(s) for s in srcs):
        return out

    incs, libs, abi = _torch_paths()
    py_inc = sysconfig.get_paths()["include"]
    inc_flags = [f"-I{p}" for p in incs + [py_inc, csrc]]
    defs = [
        f"-DTORCH_EXTENSION_NAME={MODULE}",
        "-DTORCH_API_INCLUDE_EXTENSION_H",
        f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
    ]
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    objs = []
    for s in srcs:
        o = os.path.join(OUT_DIR, os.path.basename(s) + ".o")
        if s.endswith(".cu"):
            cmd = [nvcc, "-c", s, "-o", o, *inc_flags, *defs,
                   "-D__CUDA_NO_HALF_OPERATORS__", "-D__CUDA_NO_HALF_CONVERSIONS__",
                   "-D__CUDA_NO_BFLOAT16_CONVERSIONS__", "-D__CUDA_NO_HALF2_OPERATORS__",
                   "--expt-relaxed-constexpr", "-std=c++17", "-Xcompiler", "-fPIC",
                   "-O2", "-gencode", "arch=compute_100,code=sm_100"]
        else:
            cmd = ["g++", "-c", s, "-o", o, *inc_flags, *defs, "-std=c++17", "-fPIC", "-O2"]
        if verbose:
            print("[build_ref]", os.path.basename(s))
        subprocess.check_call(cmd)
        objs.append(o)
    link = ["g++", "-shared", "-o", out, *objs, *[f"-L{p}" for p in libs],
            *[f"-Wl,-rpath,{p}" for p in libs],
            "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python", "-lcudart"]
    subprocess.check_call(link)
    for o in objs:
        os.remove(o)
    if verbose:
        print("[build_ref] wrote", out)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=None, help="reference checkout (default: $KNN_REFERENCE_SRC or ../reference)")
    a = ap.parse_args()
    build(a.src)
    sys.exit(0)
