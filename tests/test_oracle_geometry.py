"""CPU tests of the oracle's candidate-stage geometry: the reference's own unit
tests of the ellipse fit and of the ellipse representation (fixtures read
from the reference sources by tests/golden/make_golden.py), the FP64 fit core
against an independent float64 eigen solver, and the oracle's independence
from the library's sources."""
import ctypes as C
import json
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
CASES = json.loads((ROOT / "tests" / "golden" / "reference_geometry_cases.json").read_text())
_P = C.c_void_p
_F = C.c_float


@pytest.fixture(scope="module")
def geo(orc):
    lib = orc.load()
    lib.orc_fit_ellipse.argtypes = [_P, C.c_int, _P]
    lib.orc_fit_circle.argtypes = [_P, C.c_int, _P]
    lib.orc_ellipse_matrix.argtypes = [_F, _F, _F, _F, _F, _P]
    lib.orc_ellipse_params.argtypes = [_P, _P]
    for f in ("orc_fit_ellipse", "orc_fit_circle", "orc_ellipse_matrix", "orc_ellipse_params"):
        getattr(lib, f).restype = C.c_int
    return lib


def fit(lib, pts):
    xy = np.ascontiguousarray(np.asarray(pts, np.float32).reshape(-1, 2))
    out = np.zeros(5, np.float32)
    rc = lib.orc_fit_ellipse(xy.ctypes.data_as(_P), len(xy), out.ctypes.data_as(_P))
    return None if rc else out


def check_pt_in_ellipse(pt, e):
    """The reference test's check_pt_in_ellipse (test/fitEllipse.cpp:21-32)."""
    tx, ty = pt[0] - e[0], pt[1] - e[1]
    pa = np.arctan2(ty, tx)
    x = e[2] * np.cos(pa + e[4])
    y = e[3] * np.sin(pa + e[4])
    return np.hypot(tx, ty) < np.hypot(x, y)


@pytest.mark.parametrize("case", CASES["fit"], ids=[c["name"] for c in CASES["fit"]])
def test_reference_fit_cases(geo, case):
    """test/fitEllipse.cpp: fits whose points' mass center must lie inside the
    fitted ellipse, and degenerate point sets that must throw."""
    e = fit(geo, case["points"]) if case["points"] else fit(geo, np.zeros((0, 2)))
    if case["expect"] == "throw":
        assert e is None
    else:
        assert e is not None
        pts = np.asarray(case["points"], np.float32)
        assert check_pt_in_ellipse(pts.mean(axis=0), e)


def test_reference_ellipse_representation(geo):
    """geometry/test/ellipse.cpp: parameters -> conic -> parameters, and the
    rotated / translated points of x^2/25 + y^2/9 = 1 on the conic."""
    r = CASES["representation"]
    pts = np.asarray(r["points"], np.float32)
    a, b, cx, cy = r["aGT"], r["bGT"], r["cxGT"], r["cyGT"]
    step = np.float32(np.pi) / r["numTrials"]
    for i in range(r["numTrials"]):
        ang = np.float32(i) * step
        Q = np.zeros(9, np.float32)
        assert geo.orc_ellipse_matrix(cx, cy, a, b, ang, Q.ctypes.data_as(_P)) == 0
        Q = Q.reshape(3, 3).astype(np.float64)
        c, s = np.cos(ang), np.sin(ang)
        T = np.array([[c, -s, cx], [s, c, cy], [0, 0, 1]])
        for p in pts:
            v = T @ np.array([p[0], p[1], 1.0])
            assert abs(v @ Q @ v) < 1e-3
        par = np.zeros(5, np.float32)
        assert geo.orc_ellipse_params(np.ascontiguousarray(Q, np.float32).ctypes.data_as(_P),
                                      par.ctypes.data_as(_P)) == 0
        # the major axis comes back along y: a and b swap, the angle moves by pi/2
        assert abs(par[0] - cx) < 1e-3 and abs(par[1] - cy) < 1e-3
        assert abs(par[3] - a) < 1e-3 and abs(par[2] - b) < 1e-3
        assert abs(abs(par[4] - ang) - np.pi / 2) < 1e-3 or abs(par[4] - ang) < 1e-3


def _direct_fit_float64(pts):
    """Fitzgibbon / Halir-Flusser direct fit with numpy's general eigen solver."""
    p = np.asarray(pts, np.float64)
    p = p - p.mean(axis=0)
    x, y = p[:, 0], p[:, 1]
    D1 = np.stack([x * x, x * y, y * y], 1)
    D2 = np.stack([x, y, np.ones_like(x)], 1)
    S1, S2, S3 = D1.T @ D1, D1.T @ D2, D2.T @ D2
    T = -np.linalg.solve(S3, S2.T)
    M = S1 + S2 @ T
    M = np.array([M[2] / 2, -M[1], M[0] / 2])
    w, v = np.linalg.eig(M)
    v = v.real
    cond = 4 * v[0] * v[2] - v[1] ** 2
    k = int(np.argmin(np.where(cond > 0, cond, np.inf)))
    a1 = v[:, k]
    return np.concatenate([a1, T @ a1])


def _conic_of(e):
    cx, cy, a, b, t = map(float, e)
    c, s = np.cos(t), np.sin(t)
    Ri = np.array([[c, s, -(c * cx + s * cy)], [-s, c, s * cx - c * cy], [0, 0, 1]])
    return Ri.T @ np.diag([1 / a ** 2, 1 / b ** 2, -1]) @ Ri


def test_fit_core_against_float64_eigen(geo):
    """The FP64 fit core (cubic roots + cross-product eigenvectors) gives the
    conic of numpy's float64 eigen decomposition of the same reduced scatter
    matrix, on noisy arcs of random ellipses (short arcs included)."""
    rng = np.random.default_rng(7)
    worst = 0.0
    for _ in range(300):
        a, b = rng.uniform(5, 200, 2)
        t0, span = rng.uniform(0, 2 * np.pi), rng.uniform(0.8, 2 * np.pi)
        th = t0 + np.sort(rng.uniform(0, span, int(rng.integers(8, 200))))
        cx, cy, ang = rng.uniform(100, 1000), rng.uniform(100, 1000), rng.uniform(0, np.pi)
        x, y = a * np.cos(th), b * np.sin(th)
        pts = np.stack([cx + x * np.cos(ang) - y * np.sin(ang), cy + x * np.sin(ang) + y * np.cos(ang)], 1)
        pts = np.round(pts + rng.normal(0, 0.3, pts.shape)).astype(np.float32)
        e = fit(geo, pts)
        if e is None:
            continue
        off = pts.astype(np.float64).mean(axis=0)
        q = _direct_fit_float64(pts)
        # numpy's conic in uncentred coordinates, scaled and signed like the oracle's
        A, B, Cc, Dd, Ee, Ff = q
        Qc = np.array([[A, B / 2, Dd / 2], [B / 2, Cc, Ee / 2], [Dd / 2, Ee / 2, Ff]])
        Tm = np.array([[1, 0, -off[0]], [0, 1, -off[1]], [0, 0, 1]])
        Qr = Tm.T @ Qc @ Tm
        Qo = _conic_of(e)
        Qr = Qr * (np.abs(Qo).max() / np.abs(Qr).max()) * np.sign(Qr[0, 0] * Qo[0, 0])
        rel = np.abs(Qr - Qo).max() / np.abs(Qo).max()
        worst = max(worst, rel)
        assert rel < 2e-4, (rel, e)
    assert 0 < worst < 2e-4


def test_fit_circle_exact_circle(geo):
    th = np.linspace(0, 2 * np.pi, 40, endpoint=False)
    pts = np.stack([300 + 50 * np.cos(th), 200 + 50 * np.sin(th)], 1).astype(np.float32)
    out = np.zeros(3, np.float32)
    assert geo.orc_fit_circle(np.ascontiguousarray(pts).ctypes.data_as(_P), len(pts), out.ctypes.data_as(_P)) == 0
    np.testing.assert_allclose(out, [300, 200, 50], atol=1e-3)


def test_oracle_is_built_from_its_own_sources():
    """The oracle library compiles oracle/*.cpp only, and no oracle source
    includes a file of the library's package."""
    import oracle.build as ob

    assert all(Path(s).parent == ROOT / "oracle" for s in ob.SOURCES)
    for f in list((ROOT / "oracle").glob("*.cpp")) + list((ROOT / "oracle").glob("*.h*")):
        for inc in re.findall(r'#include\s+"([^"]+)"', f.read_text()):
            assert "cctag_b200/csrc" not in inc and not inc.startswith(".."), (f.name, inc)


def test_oracle_bank_equals_reference(golden_tables):
    src = (ROOT / "oracle" / "oracle_bank.hpp").read_text()
    vals = [float(v.rstrip("f")) for v in re.findall(r"[0-9]+\.[0-9]+f", src)]
    np.testing.assert_array_equal(np.array(vals, np.float32).reshape(32, 5), golden_tables["idThreeCrowns"])
