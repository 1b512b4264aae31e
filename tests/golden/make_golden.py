"""Regenerate the golden fixtures in this directory.

Sources:
  * the reference CCTag sources (read as text, when present): the two thinning
    tables of ``src/cctag/filter/thinning.cpp:12-13`` and the 3-crown bank of
    ``src/cctag/CCTagMarkersBank.cpp:120-152``;
  * OpenCV (``cv2``, the installed stand-in for the reference's OpenCV 4.5.3):
    ``cv2.filter2D`` with the reference's 9x9 derivative kernel and
    ``cv2.resize`` (INTER_LINEAR), on seeded images.

Usage:  python tests/golden/make_golden.py [/path/to/reference]
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference")

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


def main():
    lut1, lut2, bank = reference_tables()
    np.savez_compressed(HERE / "reference_tables.npz", lutthin1=lut1, lutthin2=lut2, idThreeCrowns=bank)
    np.savez_compressed(HERE / "opencv_cases.npz", **opencv_cases())
    print("wrote", HERE / "reference_tables.npz", HERE / "opencv_cases.npz")


if __name__ == "__main__":
    main()
