"""Builds the in-tree native artefacts of thesiscode_b200.

  thesiscode_b200/libmpgpu.so   CUDA kernels (sm_100a) + C ABI (include/mpgpu.h)
  thesiscode_b200/mpgpu_cli     scrimppp-compatible command line (C++ host code)

Usage: python -m thesiscode_b200.build [--force]
nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmpgpu.so")
CLI = os.path.join(HERE, "mpgpu_cli")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["mp_prep.cu", "mp_join_fp64.cu", "mp_join_fp32.cu", "mp_finalize.cu",
                "mp_capi.cu", "mp_calib.cu", "mp_batch.cu", "mp_noalloc.cu", "mp_prescrimp.cu",
                "mp_guard.cu", "mp_serve.cu"]
HOST_SOURCES = ["host/matprof_algo.cpp", "host/gpu_variants.cpp", "host/profile_io.cpp",
                "host/mp_server.cpp"]
CLI_SOURCES = ["host/main.cpp"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", *ARCH,
              f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}"]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}",
             f"-I{os.path.join(CUDA_HOME, 'include')}"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False) -> None:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    headers += [os.path.join(CSRC, "host", h) for h in os.listdir(os.path.join(CSRC, "host"))
                if h.endswith((".h", ".hpp"))]
    headers.append(os.path.join(ROOT, "include", "mpgpu.h"))
    objs = []
    for src in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        if force or _stale(o, [s, *headers]):
            _run([NVCC, *NVCC_FLAGS, "-c", s, "-o", o])
        objs.append(o)
    host_objs = []
    for src in HOST_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.basename(src).replace(".cpp", ".o"))
        if force or _stale(o, [s, *headers]):
            _run(["g++", *CXX_FLAGS, "-c", s, "-o", o])
        host_objs.append(o)
    if force or _stale(LIB, objs + host_objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs, *host_objs])
    cli_srcs = [os.path.join(CSRC, s) for s in CLI_SOURCES]
    if force or _stale(CLI, cli_srcs + [LIB, *headers]):
        _run(["g++", *CXX_FLAGS, "-o", CLI, *cli_srcs, f"-L{HERE}", "-lmpgpu",
              f"-Wl,-rpath,$ORIGIN", "-lpthread"])


if __name__ == "__main__":
    build(force="--force" in sys.argv)
