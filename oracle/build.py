"""Build recipe of the CPU oracle (test infrastructure): ``oracle/liboracle.so``.

The reference library itself cannot be compiled in this environment (it needs
the OpenCV, Eigen, Boost and oneTBB development packages, none of which is
installed), so there is no ``oracle/_ref`` build; the oracle is the C++
restatement in this directory.

Flags: ``-ffp-contract=off`` because the reference is built without FMA
contraction; ``-mavx2 -mfma`` so that the explicit ``std::fma`` of the
derivative chain (which mirrors OpenCV's filter2D) is a single instruction.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
# Only this directory's sources; from include/ the public C header (the
# parameter struct and status codes) and the FP64 fit cores of
# include/cctag_b200/portable/ (the arithmetic that stands in for Eigen).
SOURCES = sorted(HERE.glob("*.cpp"))
INCLUDE = HERE.parent / "include"
HEADERS = sorted(HERE.glob("*.h")) + sorted(HERE.glob("*.hpp")) + sorted(INCLUDE.rglob("*.h*"))
FLAGS = ["-O3", "-std=c++17", "-fPIC", "-shared", "-mavx2", "-mfma", "-ffp-contract=off", "-Wall", "-pthread"]


def build_oracle(force: bool = False, verbose: bool = False) -> Path:
    newest = max(p.stat().st_mtime for p in SOURCES + HEADERS + [Path(__file__)])
    if LIB.exists() and not force and LIB.stat().st_mtime >= newest:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["g++", *FLAGS, "-I", str(INCLUDE), "-I", "/usr/local/cuda/include", "-o", str(tmp), *map(str, SOURCES)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv, verbose=True))
