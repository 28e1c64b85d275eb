"""In-tree build of the CUDA library and its torch extension.

* ``cuda_knn_aggregate/libknn_aniso.so`` -- the C-ABI library
  (``include/knn_aniso.h``), built by nvcc for sm_100a from ``csrc/*.cu``
  (no fast-math: the key arithmetic must round exactly like the reference).
* ``cuda_knn_aggregate/_C.<abi>.so`` -- the torch extension
  (``csrc/torch_ext.cpp``), linked against the library with an ``$ORIGIN``
  rpath so both load from the package directory.

Usage: ``python build.py [--force] [--jobs N]``.  Sources are rebuilt only
when newer than their outputs.  Works without a GPU (nvcc cross-compiles).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
PKG = os.path.join(HERE, "cuda_knn_aggregate")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

CU_SOURCES = ["knn_search.cu", "knn_search_tc.cu", "knn_spatial.cu", "knn_adjoint.cu", "knn_capi.cu", "knn_noalloc.cu", "knn_variants.cu",
              "knn_ragged.cu"]
HEADERS = ["knn_common.cuh", "knn_internal.h", "knn_ragged.h", "knn_search_dev.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH

LIB = os.path.join(PKG, "libknn_aniso.so")
EXT = os.path.join(PKG, "_C" + sysconfig.get_config_var("EXT_SUFFIX"))


def _newer(out: str, deps) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print("[build]", " ".join(os.path.basename(c) if c.endswith((".cu", ".cpp")) else c for c in cmd[:3]), "...")
    subprocess.check_call(cmd)


def build_lib(force=False, jobs=3, verbose=True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "knn_aniso.h")]
    objs, cmds = [], []
    for s in CU_SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        if force or not _newer(obj, [src] + hdrs):
            cmds.append([NVCC, "-c", src, "-o", obj, f"-I{INCLUDE}", f"-I{CSRC}"] + NVCC_FLAGS)
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        list(ex.map(lambda c: _run(c, verbose), cmds))
    if force or cmds or not _newer(LIB, objs):
        tmp = LIB + f".tmp{os.getpid()}"
        _run([NVCC, "-shared", "-o", tmp, *objs, "-cudart", "static"] + ARCH, verbose)
        os.replace(tmp, LIB)
    return LIB


def build_ext(force=False, verbose=True) -> str:
    import torch
    from torch.utils import cpp_extension as ce

    src = os.path.join(CSRC, "torch_ext.cpp")
    deps = [src, os.path.join(INCLUDE, "knn_aniso.h"), LIB]
    if not force and _newer(EXT, deps):
        return EXT
    incs = ce.include_paths(device_type="cuda") + [sysconfig.get_paths()["include"], INCLUDE]
    libs = ce.library_paths(device_type="cuda")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    tmp = EXT + f".tmp{os.getpid()}"
    cmd = ["g++", "-shared", "-O2", "-std=c++17", "-fPIC", src, "-o", tmp,
           "-DTORCH_EXTENSION_NAME=_C", "-DTORCH_API_INCLUDE_EXTENSION_H", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           *[f"-I{p}" for p in incs], *[f"-L{p}" for p in libs], f"-L{PKG}",
           "-Wl,-rpath,$ORIGIN", *[f"-Wl,-rpath,{p}" for p in libs],
           "-lknn_aniso", "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python",
           "-lcudart"]
    _run(cmd, verbose)
    os.replace(tmp, EXT)
    return EXT


def build(force=False, jobs=3, verbose=True):
    build_lib(force, jobs, verbose)
    build_ext(force, verbose)
    return LIB, EXT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=3)
    a = ap.parse_args()
    build(a.force, a.jobs)
    sys.exit(0)
