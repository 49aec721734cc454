"""Builds the engine in-tree: libcvl.so (sm_100a CUDA + host engine, C ABI)
and bin/CURVELET (the drop-in CLI), with nvcc/g++ directly.

    python -m curvelet_construction_on_gpu_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libcvl.so")
CLI = os.path.join(PKG, "bin", "CURVELET")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
              "-Xcompiler", "-fPIC,-O2", "-shared"]
LIB_SOURCES = ["cvl_engine.cu", "cvl_server.cpp", "cvl_io.cpp"]
LIB_DEPS = ["cvl_engine.cu", "cvl_server.cpp", "cvl_io.cpp", "cvl_internal.h", "cvl_pinned.h", "cvl_kernels.cuh", "cvl_path.cuh", "cvl_scan.cuh", "cvl_contours.cuh", "cvl_polyarcs.cuh"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    # the system g++ (an inherited CXX may point at a toolchain without the C++ runtime pieces)
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout, r.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, d) for d in LIB_DEPS] + [os.path.join(INCLUDE, "cvl.h")]
    if force or _stale(LIB, deps):
        cmd = [_nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-o", LIB + ".tmp",
               *[os.path.join(CSRC, s) for s in LIB_SOURCES]]
        if ptxas_verbose:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd, verbose)
        os.replace(LIB + ".tmp", LIB)
    cli_deps = [os.path.join(CSRC, "cvl_cli.cpp"), os.path.join(INCLUDE, "cvl.h"), LIB]
    if force or _stale(CLI, cli_deps):
        os.makedirs(os.path.dirname(CLI), exist_ok=True)
        cmd = [_cxx(), "-O2", "-std=c++17", "-I", INCLUDE, os.path.join(CSRC, "cvl_cli.cpp"), "-L", PKG, "-lcvl",
               "-Wl,-rpath,$ORIGIN/..", "-o", CLI]
        _run(cmd, verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
