"""Builds the reference's own single-GPU program into oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  The reference (Summer536/LBM_DDF ``src/``) takes its
run surface as compile-time macros from ``src/parameters.h``.  That header is
include-guarded by ``PARAMETERS_H``, so predefining the guard and every macro
on the nvcc command line compiles the unmodified sources, where they lie, with
the grid, Rayleigh number, step counts and output cadences of one case.  The
flags are the reference Makefile's (``Makefile:3``) with the architecture
changed from sm_80 to sm_100a.

Each case becomes one binary ``oracle/_ref/rb3d_<case>``.  The binaries are
built here (nvcc cross-compiles) and run on a B200; the reference sources are
only needed at build time.  Nothing is copied from the reference tree.

Usage:  python oracle/build_ref.py [case ...]      (default: every case)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# The reference's src/ directory: LBM_REFERENCE_SRC, else a checkout of the
# reference project beside this repository (../reference/src).
REF_SRC = os.environ.get("LBM_REFERENCE_SRC") or os.path.normpath(
    os.path.join(HERE, "..", "..", "reference", "src"))
SOURCES = ["main.cu", "globals.cu", "initial.cu", "collision.cu", "streaming.cu",
           "macrovar.cu", "output.cu"]
NEVER = 1_000_000_000

sys.path.insert(0, HERE)
from ref_cases import REF_CASES  # noqa: E402


def binary(name: str) -> str:
    return os.path.join(OUT, "rb3d_" + name)


def defines(c: dict) -> list[str]:
    return [
        "-DPARAMETERS_H",
        f"-DCONTINUE_STEP={c['continue_step']}",
        f"-DLX={c['lx']}", f"-DLY={c['ly']}", f"-DLZ={c['lz']}",
        "-DLXYZ=(LX*LY*LZ)", "-DNPOP=27",
        f"-DNEND={c['nend']}",
        f"-DNDIAG={c.get('ndiag', NEVER)}",
        f"-DNFLOWOUT={c.get('nflowout', NEVER)}",
        f"-DNNUOUT={c.get('nnuout', NEVER)}",
        f"-DRAYLEIGH={c['rayleigh']!r}", f"-DPRANDTL={c['prandtl']!r}",
        "-DT_HOT=1.0", "-DT_COLD=0.0", "-DGRAVITY=1.0",
        # free-fall velocity 0.1: g*beta*dT*LY = 0.01
        "-DBETA=(0.01/(LY*1.0))",
        "-DBLOCK_X=8", "-DBLOCK_Y=8", "-DBLOCK_Z=4",
    ]


def build_case(name: str, force: bool = False) -> str:
    c = REF_CASES[name]
    out = binary(name)
    srcs = [os.path.join(REF_SRC, s) for s in SOURCES]
    if not force and os.path.exists(out):
        newest = max(os.path.getmtime(s) for s in srcs + [os.path.join(HERE, "ref_cases.py")])
        if os.path.getmtime(out) >= newest:
            return out
    os.makedirs(OUT, exist_ok=True)
    cmd = ["nvcc", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++14",
           "-rdc=true", "--use_fast_math", "-w"] + defines(c) + srcs + ["-o", out]
    subprocess.run(cmd, check=True)
    return out


def available() -> bool:
    return all(os.path.exists(os.path.join(REF_SRC, s)) for s in SOURCES)


def main(argv: list[str]) -> int:
    if not available():
        print(f"reference sources not found under {REF_SRC}; nothing built")
        return 0
    names = argv or list(REF_CASES)
    for n in names:
        print("building", binary(n), flush=True)
        build_case(n)
    return 0


if __name__ == "__main__":
    raise SystemExit(main(sys.argv[1:]))
