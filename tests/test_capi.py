"""CPU tests of the C ABI: the library loads, exports every declared symbol,
and the calls that need no GPU behave."""
import ctypes as C
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").rglob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"^\s*(?:[\w\*\s]+?)\b(cctagb_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_symbol(built_library):
    lib = C.CDLL(str(built_library))
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol(built_library):
    from cctag_b200 import capi

    assert declared_symbols() <= set(capi.SIGNATURES)


def test_default_params_match_reference_defaults(built_library):
    from cctag_b200 import capi

    p = capi.default_params(3)
    # Params.hpp:27-66
    assert (p.distSearch, p.thrGradientMagInVote, p.nCrowns, p.nCircles) == (30, 2500, 3, 6)
    assert abs(p.cannyThrLow - 0.01) < 1e-9 and abs(p.cannyThrHigh - 0.04) < 1e-9
    assert (p.maximumNbSeeds, p.maximumNbCandidatesLoopTwo, p.minVotesToSelectCandidate) == (500, 40, 3)
    assert (p.nSamplesOuterEllipse, p.numCutsInIdentStep, p.sampleCutLength) == (150, 22, 100)
    assert p.imagedCenterNGridSample == 5 and abs(p.imagedCenterNeighbourSize - 0.2) < 1e-7
    assert abs(p.ellipseGrowingEllipticHullWidth - 2.3) < 1e-6


def test_status_strings_and_null_handles(built_library):
    from cctag_b200 import capi

    lib = capi.load()
    assert lib.cctagb_status_string(capi.OK) == b"ok"
    assert lib.cctagb_destroy(None) == capi.BAD_ARG
    n = C.c_int()
    assert lib.cctagb_detect(None, None, 1, 1, 1, 0, None, 0, C.byref(n), None) == capi.BAD_ARG
    assert lib.cctagb_create(None, 64, 64, 1, None) == capi.BAD_ARG


def build_shim_example(built_library, tmp_path):
    import subprocess

    exe = tmp_path / "shim_example"
    cmd = ["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / "shim_example.cpp"),
           "-o", str(exe), str(built_library), f"-Wl,-rpath,{built_library.parent}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_shim_compiles_and_links(built_library, tmp_path):
    """The header-only ICCTag.hpp shim compiles against the C ABI with no
    OpenCV/Boost/Eigen, using cv::Mat / ptr_list look-alike types."""
    assert build_shim_example(built_library, tmp_path).exists()


def test_binding_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of the ABI structs have the C compiler's sizes and
    field offsets."""
    import shutil
    import subprocess

    from cctag_b200 import capi

    if not shutil.which("gcc"):
        import pytest
        pytest.skip("gcc not available")
    root = Path(__file__).resolve().parents[1]
    checks = {
        "cctagb_params": (capi.Params, []),
        "cctagb_marker": (capi.Marker, ["outer", "homography", "quality", "scale"]),
        "cctagb_stats": (capi.Stats, ["ms_image_stage", "h2d_bytes", "kernel_launches", "ms_cut_selection"]),
        "cctagb_frame": (capi.Frame, ["pitch", "out", "n_out", "status", "stats"]),
        "cctagb_cut_task": (capi.CutTask, ["x0", "ncuts", "stop", "roi"]),
        "cctagb_ident_result": (capi.IdentResult, ["H", "residual", "nvalid", "iterations"]),
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cctag_b200.h"', "int main(void) {"]
    for cname, (_, fields) in checks.items():
        lines.append(f'printf("%zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'printf("%zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(root / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = []
    for _, (ct, fields) in checks.items():
        want.append(C.sizeof(ct))
        want += [getattr(ct, f).offset for f in fields]
    assert got == want
