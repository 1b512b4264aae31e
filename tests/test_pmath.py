"""The portable transcendental functions shared by the host and GPU candidate
stage (include/cctag_b200/portable/pmath.hpp) are the correctly rounded float values of
sin, cos and atan2 (checked against libm's double precision, rounded once),
with IEEE signed-zero results; the PCG32 jump-ahead they use; and the
correctly rounded division by small integers of the GPU sample statistics."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_pmath_correctly_rounded(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    exe = tmp_path / "pmath"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", str(ROOT / "cctag_b200" / "csrc"), "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "pmath_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


def test_pcg_jump_ahead(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    exe = tmp_path / "pcg"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", str(ROOT / "cctag_b200" / "csrc"), "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "pcg_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


def test_div_small_exhaustive(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    exe = tmp_path / "div_small"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", str(ROOT / "cctag_b200" / "csrc"), "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "div_small_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
