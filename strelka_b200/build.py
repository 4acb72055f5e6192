"""Builds the in-tree CUDA/C++ library ``strelka_b200/libstrelka_b200.so``.

Every ``.cu`` file is compiled for sm_100a only with ``-fmad=false`` (no fused
multiply-add contraction: the kernels reproduce the host-side restatement of
the shader math bit for bit) and every ``.cpp`` file with
``-ffp-contract=off``.  The CUDA runtime is linked statically so the library
does not depend on which ``libcudart`` another module of the process loaded.

Usage: ``python -m strelka_b200.build [--force]``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libstrelka_b200.so")

NVCC = os.environ.get("STRELKA_NVCC", "/usr/local/cuda/bin/nvcc")
# The system compiler (an inherited $CXX may point at a wrapper without OpenMP).
HOST_CXX = os.environ.get("STRELKA_CXX", "/usr/bin/g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
    "-ccbin", HOST_CXX,
    "-Xcompiler", "-fPIC,-fopenmp,-ffp-contract=off",
    "-I", os.path.join(ROOT, "include"),
]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-Wall",
             "-Wno-unused-function", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include"]


def _headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(obj: str, src: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = _headers()
    objs = []
    relink = force or not os.path.exists(LIB)
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            if src.endswith(".cu"):
                cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
            else:
                cmd = [HOST_CXX] + CXX_FLAGS + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
            relink = True
    if not relink and any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        relink = True
    if relink:
        tmp = LIB + ".tmp"
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-ccbin", HOST_CXX,
                               "-Xcompiler", "-fopenmp", "-o", tmp] + objs + ["-lgomp"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
