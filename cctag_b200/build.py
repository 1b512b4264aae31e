"""Build the in-tree shared library ``cctag_b200/libcctag_b200.so``.

CUDA sources are compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); host sources with g++.  The CUDA
runtime is linked statically so the library is self-contained.  Rebuilds only
when a source or header is newer than the library.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build" / "cctag_b200"
LIB = PKG / "libcctag_b200.so"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function", "-ffp-contract=off", "-mpopcnt"]
# Translation units whose float arithmetic must equal the host restatement's
# bit for bit: no contraction of a * b + c into a fused multiply-add.
NO_FMAD = {"loop_one", "grow", "outer_select"}


def _sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted(CSRC.glob("*.cpp"))
    hdr = sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.rglob("*.h")) + sorted(INCLUDE.rglob("*.hpp"))
    return cu, cpp, hdr


def _run(cmd, verbose):
    if verbose:
        print(" ".join(map(str, cmd)), file=sys.stderr)
    r = subprocess.run(list(map(str, cmd)), capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build command failed ({r.returncode}): {' '.join(map(str, cmd))}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, file=sys.stderr)
    return r


def build_library(force: bool = False, verbose: bool = False) -> Path:
    cu, cpp, hdr = _sources()
    newest = max(p.stat().st_mtime for p in cu + cpp + hdr + [Path(__file__)])
    if LIB.exists() and not force and LIB.stat().st_mtime >= newest:
        return LIB
    BUILD.mkdir(parents=True, exist_ok=True)
    inc = ["-I", INCLUDE, "-I", CSRC, "-I", CUDA_HOME / "include"]
    objs = []
    for src in cu:
        obj = BUILD / (src.stem + ".cu.o")
        extra = ["--fmad=false"] if src.stem in NO_FMAD else []
        _run([NVCC, *ARCH, *CUDA_FLAGS, *extra, *inc, "-c", src, "-o", obj], verbose)
        objs.append(obj)
    for src in cpp:
        obj = BUILD / (src.stem + ".o")
        _run(["g++", *CXX_FLAGS, *inc, "-c", src, "-o", obj], verbose)
        objs.append(obj)
    tmp = LIB.with_suffix(".so.tmp")
    _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lpthread"], verbose)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
