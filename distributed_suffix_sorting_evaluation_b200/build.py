"""Builds the in-tree native artefacts for sm_100a:

  lib/libdcxgpu.so  -- the CUDA engine and its C ABI (include/dcx_gpu.h)
  lib/dcx_cli       -- the reference-compatible command line front end
  lib/libtextgen.so -- seeded synthetic text generators of the benchmark workloads

Run as ``python -m distributed_suffix_sorting_evaluation_b200.build``.
nvcc cross-compiles, so no GPU is needed to build.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
INC = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", f"-I{INC}"]
HOST_CXX = "/usr/bin/g++"

SOURCES = ["dcx.cu", "noalloc.cu"]
HEADERS = ["common.cuh", "radix.cuh", "keys.cuh", "segsort.cuh", "warpsort.cuh", "small_sa.cuh", "level_kernels.cuh", "lcp.cuh",
           "lcp_scatter.cuh", "bwt.cuh", "gsa.cuh", "serve.cuh"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    so = os.path.join(LIB, "libdcxgpu.so")
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INC, "dcx_gpu.h")]
    if force or _stale(so, deps):
        cmd = [_nvcc()] + NVCC_FLAGS + ["-shared", "-o", so] + [os.path.join(CSRC, f) for f in SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    cli = os.path.join(LIB, "dcx_cli")
    cli_src = os.path.join(CSRC, "cli.cpp")
    if os.path.exists(cli_src) and (force or _stale(cli, [cli_src, so, os.path.join(INC, "dcx_gpu.h")])):
        cuda_lib = "/usr/local/cuda/lib64"
        cmd = [HOST_CXX, "-O2", "-std=c++17", f"-I{INC}", "-o", cli, cli_src, f"-L{LIB}", "-ldcxgpu",
               f"-L{cuda_lib}", "-lcudart", "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{cuda_lib}", "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    gen = os.path.join(LIB, "libtextgen.so")
    gen_src = os.path.join(CSRC, "textgen.cpp")
    if force or _stale(gen, [gen_src]):
        cmd = [HOST_CXX, "-O2", "-std=c++17", "-fopenmp", "-shared", "-fPIC", "-o", gen, gen_src]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return so


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
