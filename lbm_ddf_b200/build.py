"""Build recipe for the engine's native code (run by __graft_entry__.build()).

* ``liblbm_ddf.so``: the CUDA kernels and the C ABI of include/lbm_ddf.h,
  compiled for sm_100a only.
* ``rb3d``: the C++ host driver with the reference's run surface, linked
  against liblbm_ddf.so.

Both land in this package directory (in-tree), so they travel with the source.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "liblbm_ddf.so")
DRIVER = os.path.join(PKG, "rb3d")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Werror", "all-warnings"]  # a warning (e.g. the address of a temporary) fails the build
LIB_SOURCES = ["engine.cu", "batch.cu"]
HEADERS = ["lattice.cuh", "step.cuh", "bulk.cuh", "rowstep.cuh", "internal.h"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _sources(names):
    return [os.path.join(CSRC, n) for n in names if os.path.exists(os.path.join(CSRC, n))]


def build_lib(force: bool = False, verbose: bool = False) -> str:
    srcs = _sources(LIB_SOURCES)
    deps = srcs + _sources(HEADERS) + [os.path.join(ROOT, "include", "lbm_ddf.h"), __file__]
    if force or _newer(LIB, deps):
        cmd = ["nvcc"] + ARCH + NVCC_FLAGS + ["-shared", "-o", LIB] + srcs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def build_driver(force: bool = False, verbose: bool = False) -> str | None:
    src = os.path.join(CSRC, "rb3d_main.cpp")
    if not os.path.exists(src):
        return None
    if force or _newer(DRIVER, [src, LIB, os.path.join(ROOT, "include", "lbm_ddf.h")]):
        cmd = ["g++", "-O2", "-std=c++17", "-o", DRIVER, src, "-I" + os.path.join(ROOT, "include"),
               "-L" + PKG, "-llbm_ddf", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return DRIVER


def build(force: bool = False, verbose: bool = False) -> None:
    build_lib(force, verbose)
    build_driver(force, verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
