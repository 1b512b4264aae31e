"""Regenerate the golden fixtures in this directory.

Sources:
  * the reference CCTag sources, read as text: the two thinning tables of
    ``src/cctag/filter/thinning.cpp:12-13``, the 3-crown bank of
    ``src/cctag/CCTagMarkersBank.cpp:120-152``, and the point sets and expected
    outcomes of the reference's ellipse-fit and ellipse-representation unit
    tests (``src/cctag/test/fitEllipse.cpp``,
    ``src/cctag/geometry/test/ellipse.cpp``);
  * OpenCV (``cv2``, the installed stand-in for the reference's OpenCV 4.5.3):
    ``cv2.filter2D`` with the reference's 9x9 derivative kernel and
    ``cv2.resize`` (INTER_LINEAR), on seeded images.

Usage:  python tests/golden/make_golden.py /path/to/reference
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF: Path = Path(".")

KERNEL_ROWS = """
-0.000000143284235 -0.000003558691641 -0.000028902492951 -0.000064765993382 0 0.000064765993382 0.000028902492951 0.000003558691641 0.000000143284235
-0.000004744922188 -0.000117847682078 -0.000957119116802 -0.002144755142391 0 0.002144755142391 0.000957119116802 0.000117847682078 0.000004744922188
-0.000057804985902 -0.001435678675203 -0.011660097860113 -0.026128466569370 0 0.026128466569370 0.011660097860113 0.001435678675203 0.000057804985902
-0.000259063973527 -0.006434265427174 -0.052256933138740 -0.117099663048638 0 0.117099663048638 0.052256933138740 0.006434265427174 0.000259063973527
-0.000427124283626 -0.010608310271112 -0.086157117207395 -0.193064705260108 0 0.193064705260108 0.086157117207395 0.010608310271112 0.000427124283626
-0.000259063973527 -0.006434265427174 -0.052256933138740 -0.117099663048638 0 0.117099663048638 0.052256933138740 0.006434265427174 0.000259063973527
-0.000057804985902 -0.001435678675203 -0.011660097860113 -0.026128466569370 0 0.026128466569370 0.011660097860113 0.001435678675203 0.000057804985902
-0.000004744922188 -0.000117847682078 -0.000957119116802 -0.002144755142391 0 0.002144755142391 0.000957119116802 0.000117847682078 0.000004744922188
-0.000000143284235 -0.000003558691641 -0.000028902492951 -0.000064765993382 0 0.000064765993382 0.000028902492951 0.000003558691641 0.000000143284235
"""


def kernel_dx() -> np.ndarray:
    return np.array([[float(t) for t in r.split()] for r in KERNEL_ROWS.strip().splitlines()], np.float32)


def reference_tables():
    src = (REF / "src/cctag/filter/thinning.cpp").read_text()
    tabs = dict(re.findall(r"lutthin(\d)\[512\] = \{([^}]*)\}", src))
    lut1 = np.array([int(v) for v in tabs["1"].split(",")], np.uint8)
    lut2 = np.array([int(v) for v in tabs["2"].split(",")], np.uint8)
    bank_src = (REF / "src/cctag/CCTagMarkersBank.cpp").read_text()
    body = bank_src.split("idThreeCrowns[32][5] =")[1].split(";")[0]
    vals = [float(v.rstrip("f")) for v in re.findall(r"[0-9]+\.[0-9]+f", body)]
    bank = np.array(vals, np.float32).reshape(32, 5)
    return lut1, lut2, bank


def opencv_cases():
    import cv2

    K = kernel_dx()
    rng = np.random.default_rng(20240601)
    cases = {}
    for i, (h, w) in enumerate([(64, 96), (37, 53), (9, 9), (3, 17), (120, 160)]):
        img = rng.integers(0, 256, (h, w), dtype=np.uint8)
        if i % 2 == 0 and min(h, w) > 8:
            img = cv2.GaussianBlur(img, (0, 0), 1.3)
        cases[f"deriv{i}_img"] = img
        cases[f"deriv{i}_dx"] = cv2.filter2D(img, cv2.CV_16S, K, borderType=cv2.BORDER_REPLICATE)
        cases[f"deriv{i}_dy"] = cv2.filter2D(img, cv2.CV_16S, np.ascontiguousarray(K.T),
                                             borderType=cv2.BORDER_REPLICATE)
    for i, (h, w) in enumerate([(64, 96), (135, 240), (101, 77), (31, 45)]):
        img = rng.integers(0, 256, (h, w), dtype=np.uint8)
        cases[f"resize{i}_img"] = img
        cases[f"resize{i}_out"] = cv2.resize(img, (w // 2, h // 2))
    return cases


def _points(body):
    return [[float(x), float(y)] for x, y in re.findall(r"emplace_back\(\s*([-0-9.]+)f?\s*,\s*([-0-9.]+)f?\s*\)", body)]


def reference_fit_cases():
    """The reference's fit known-answer tests: for each case its points and
    whether the fit must succeed with the points' mass center inside the
    ellipse ("inside") or throw std::domain_error ("throw")."""
    src = (REF / "src/cctag/test/fitEllipse.cpp").read_text()
    cases = []
    for name, body in re.findall(r"BOOST_AUTO_TEST_CASE\((\w+)\)\s*\{(.*?)\n\}", src, re.S):
        live = "\n".join(l for l in body.splitlines() if not l.strip().startswith("//"))
        if name == "test_throw_5points":  # 0 to 4 copies of (5, 0)
            for i in range(5):
                cases.append({"name": f"{name}_{i}", "points": [[5.0, 0.0]] * i, "expect": "throw"})
            continue
        if "fit_and_check_ellipse" in live:
            expect = "inside"
        elif "THROW" in live:
            expect = "throw"
        else:
            continue  # the case the reference disabled (its assertion is commented out)
        pts = _points(body)
        loop = re.search(r"for \(int j = 0; j < (\d+); \+\+j\)", live)
        if loop and len(pts) == 1:  # one point pushed in a loop
            pts = pts * int(loop.group(1))
        cases.append({"name": name, "points": pts, "expect": expect})
    ell = (REF / "src/cctag/geometry/test/ellipse.cpp").read_text()
    gt = {k: float(v) for k, v in re.findall(r"const float (\w+GT) = ([-0-9.]+)f;", ell)}
    return {"fit": cases, "representation": {"points": _points(ell), "aGT": gt["aGT"], "bGT": gt["bGT"],
                                             "cxGT": gt["cxGT"], "cyGT": gt["cyGT"], "numTrials": 10}}


def main():
    global REF
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    REF = Path(sys.argv[1])
    (HERE / "reference_geometry_cases.json").write_text(json.dumps(reference_fit_cases(), indent=1))
    lut1, lut2, bank = reference_tables()
    np.savez_compressed(HERE / "reference_tables.npz", lutthin1=lut1, lutthin2=lut2, idThreeCrowns=bank)
    np.savez_compressed(HERE / "opencv_cases.npz", **opencv_cases())
    print("wrote", HERE / "reference_tables.npz", HERE / "opencv_cases.npz", HERE / "reference_geometry_cases.json")


if __name__ == "__main__":
    main()
