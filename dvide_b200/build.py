"""Build recipe for the native parts of dvide_b200.

* libdvide_b200.so -- every CUDA kernel and the C ABI of include/dvide.h,
  compiled for sm_100a only, with -fmad=false so that the FP64 path rounds
  exactly like the CPU oracle (no fused multiply-add).
* libdvide_cxx.so -- the C++ System/Body/APGD/CollisionDetector classes
  (include/dvide/*.h) layered on the C ABI.

Outputs are written in-tree, next to this file, so they travel with the
repository snapshot.
"""
from __future__ import annotations

import os
import concurrent.futures
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

CUDA_SOURCES = ["dv_sort.cu", "dv_collide.cu", "dv_apgd.cu", "dv_pgj.cu", "dv_pgs.cu", "dv_engine.cu", "dv_diag.cu", "dv_scene.cu", "dv_batch.cu", "dv_server.cu", "dv_noalloc.cu", "dv_selftest.cu"]
CUDA_HEADERS = ["dv_common.cuh", "dv_internal.cuh", "dv_engine.h", "dv_solve.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden"]

LIB = os.path.join(HERE, "libdvide_b200.so")
CXX_LIB = os.path.join(HERE, "libdvide_cxx.so")
DRIVER = os.path.join(HERE, "drivers", "settle")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda(force=False, verbose=False):
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in CUDA_HEADERS] + [os.path.join(INCLUDE, "dvide.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    objs = [os.path.join(HERE, "_build", os.path.basename(s) + ".o") for s in srcs]
    cmds = [[_nvcc(), *ARCH, *NVCC_FLAGS, "-I", INCLUDE, "-c", s, "-o", o] for s, o in zip(srcs, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd))
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(cmds))) as ex:
        list(ex.map(subprocess.check_call, cmds))
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart_static"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


def build_cxx(force=False, verbose=False):
    """C++ System/Body/APGD/CollisionDetector layer and the settle driver."""
    src = os.path.join(CSRC, "cxx", "System.cpp")
    hdrs = [os.path.join(INCLUDE, "dvide", h) for h in os.listdir(os.path.join(INCLUDE, "dvide"))]
    inc = ["-I", INCLUDE, "-I", os.path.join(CUDA_HOME, "include")]
    rpath = "-Wl,-rpath,$ORIGIN"
    if force or _stale(CXX_LIB, [src, LIB] + hdrs):
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", *inc, src, "-o", CXX_LIB,
               "-L", HERE, "-ldvide_b200", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
               rpath]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    dsrc = os.path.join(HERE, "drivers", "settle.cpp")
    if force or _stale(DRIVER, [dsrc, CXX_LIB] + hdrs):
        cmd = ["g++", "-O2", "-std=c++17", *inc, dsrc, "-o", DRIVER, "-L", HERE, "-ldvide_cxx",
               "-ldvide_b200", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart",
               "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return [CXX_LIB, DRIVER]


def build(force=False, verbose=False):
    out = [build_cuda(force=force, verbose=verbose)]
    out += build_cxx(force=force, verbose=verbose)
    return out


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv, verbose=True):
        print(p)
