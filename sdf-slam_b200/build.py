"""Builds libsdfgpu.so (CUDA for sm_100a + host C++) in-tree.

assembly.cu is compiled with --fmad=false so that residuals, Jacobians, J^T J
and -J^T r round every product and sum separately (the reference's unfused
FP64 expressions); the factorization kernels keep fused multiply-adds.
"""
from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libsdfgpu.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++20", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]

SOURCES = {
    "assembly.cu": ["--fmad=false"],
    "cellsort.cu": [],
    "factor.cu": [],
    "engine.cu": [],
    "ldlt.cu": [],
    "noalloc.cu": [],
    "peak.cu": [],
    "schur_tc.cu": [],
    "dense_root.cu": [],
    "refine.cu": [],
    "problem_device.cu": [],
    "problem_build.cpp": ["-x", "cu"],
    "alloc.cpp": ["-x", "cu"],
    "host_pool.cpp": ["-x", "cu"],
    "symbolic.cpp": ["-x", "cu"],
    "capi.cpp": ["-x", "cu"],
    "incremental.cpp": ["-x", "cu"],
    "writers.cpp": ["-x", "cu"],
    "server.cpp": ["-x", "cu"],
    "kernel_timer.cpp": ["-x", "cu"],
}
HEADERS = ["internal.h", "device.cuh", "engine.h", "ldlt.h", "server.h", "host_pool.h", "incremental.h", "schur_tc.h", "kernel_timer.h", "dense_root.h", "front_ops.cuh",
           "trig.cuh"]


def _newest_header() -> float:
    paths = [os.path.join(CSRC, h) for h in HEADERS]
    paths.append(os.path.join(HERE, "..", "include", "sdfgpu.h"))
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def _compile(src: str, extra: list[str], force: bool) -> str:
    obj = os.path.join(BUILD_DIR, src + ".o")
    path = os.path.join(CSRC, src)
    if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
            and os.path.getmtime(obj) >= _newest_header()):
        return obj
    cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", path, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source for sm_100a and link lib/libsdfgpu.so."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    os.makedirs(OUT_DIR, exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        futs = {ex.submit(_compile, s, e, force): s for s, e in SOURCES.items()}
        objs = [f.result() for f in concurrent.futures.as_completed(futs)]
    objs.sort()
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs, "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
