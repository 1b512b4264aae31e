"""TEST INFRASTRUCTURE ONLY -- ctypes binding of the CPU oracle (liboracle.so).

Imported by the test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` only, as the checker / the timed CPU restatement of the
reference path.  The product library never loads it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .build import LIB, build_oracle

_P = C.c_void_p
_I = C.c_int
_F = C.c_float


class VoteParams(C.Structure):
    _fields_ = [("distSearch", _I), ("thrGradientMagInVote", _I), ("angleVoting", _F), ("ratioVoting", _F),
                ("nCrowns", _I), ("minVotesToSelectCandidate", _I)]


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build_oracle()
        lib = C.CDLL(str(LIB))
        lib.orc_pyramid_down.argtypes = [_P, _I, _I, _P, _I, _I]
        lib.orc_derivatives.argtypes = [_P, _I, _I, _P, _P]
        lib.orc_canny.argtypes = [_P, _P, _I, _I, _F, _F, _P, _P]
        lib.orc_thin_lut.argtypes = [_I, _P]
        lib.orc_thin.argtypes = [_P, _I, _I]
        lib.orc_vote.argtypes = [_P, _P, _P, _I, _I, C.POINTER(VoteParams), _I] + [_P] * 14
        lib.orc_vote.restype = _I
        lib.orc_level.argtypes = [_P, _I, _I, _F, _F, _P, _P, _P]
        _extra_signatures(lib)
        _lib = lib
    return _lib


def _extra_signatures(lib):
    """Signatures of the identification / candidate entry points (oracle_ident.cpp)."""
    for name, (res, args) in IDENT_SIGNATURES.items():
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args


IDENT_SIGNATURES: dict = {}


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def pyramid(gray: np.ndarray, levels: int = 4):
    lib = load()
    out = [np.ascontiguousarray(gray, dtype=np.uint8)]
    for _ in range(1, levels):
        h, w = out[-1].shape
        d = np.empty((h // 2, w // 2), np.uint8)
        lib.orc_pyramid_down(_p(out[-1]), w, h, _p(d), w // 2, h // 2)
        out.append(d)
    return out


def derivatives(img: np.ndarray):
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape
    dx = np.empty((h, w), np.int16)
    dy = np.empty((h, w), np.int16)
    load().orc_derivatives(_p(img), w, h, _p(dx), _p(dy))
    return dx, dy


def canny(dx: np.ndarray, dy: np.ndarray, thr_low=0.01 * 256, thr_high=0.04 * 256, with_map=False):
    dx = np.ascontiguousarray(dx, dtype=np.int16)
    dy = np.ascontiguousarray(dy, dtype=np.int16)
    h, w = dx.shape
    e = np.empty((h, w), np.uint8)
    m = np.empty((h, w), np.uint8) if with_map else None
    load().orc_canny(_p(dx), _p(dy), w, h, np.float32(thr_low), np.float32(thr_high), _p(e), _p(m))
    return (e, m) if with_map else e


def thin_lut(pass_no: int) -> np.ndarray:
    lut = np.empty(512, np.uint8)
    load().orc_thin_lut(pass_no, _p(lut))
    return lut


def thin(edges: np.ndarray) -> np.ndarray:
    e = np.ascontiguousarray(edges, dtype=np.uint8).copy()
    h, w = e.shape
    load().orc_thin(_p(e), w, h)
    return e


def level(img: np.ndarray, thr_low=np.float32(0.01) * np.float32(256), thr_high=np.float32(0.04) * np.float32(256)):
    """Derivatives -> Canny -> thinning of one pyramid level."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape
    dx = np.empty((h, w), np.int16)
    dy = np.empty((h, w), np.int16)
    e = np.empty((h, w), np.uint8)
    load().orc_level(_p(img), w, h, np.float32(thr_low), np.float32(thr_high), _p(dx), _p(dy), _p(e))
    return dx, dy, e


def vote(edges, dx, dy, distSearch=30, thrGradient=2500, angleVoting=0.0, ratioVoting=4.0, nCrowns=3, minVotes=3):
    edges = np.ascontiguousarray(edges, dtype=np.uint8)
    dx = np.ascontiguousarray(dx, dtype=np.int16)
    dy = np.ascontiguousarray(dy, dtype=np.int16)
    h, w = edges.shape
    cap = int((edges == 255).sum()) + 1
    i32 = lambda n=cap: np.empty(n, np.int32)  # noqa: E731
    ex, ey, before, after, chosen = i32(), i32(), i32(), i32(), i32()
    total = np.empty(cap, np.float32)
    nvotes, is_max = i32(), i32()
    flow = np.empty(cap, np.float32)
    voff, vlist = i32(cap + 1), i32()
    spush, ssorted = i32(), i32()
    ns = np.zeros(1, np.int32)
    vp = VoteParams(distSearch, thrGradient, angleVoting, ratioVoting, nCrowns, minVotes)
    E = load().orc_vote(_p(edges), _p(dx), _p(dy), w, h, C.byref(vp), cap, _p(ex), _p(ey), _p(before), _p(after),
                        _p(chosen), _p(total), _p(nvotes), _p(is_max), _p(flow), _p(voff), _p(vlist), _p(spush),
                        _p(ssorted), _p(ns))
    if E < 0:
        raise RuntimeError("oracle vote: capacity exceeded")
    S = int(ns[0])
    return dict(x=ex[:E].copy(), y=ey[:E].copy(), before=before[:E].copy(), after=after[:E].copy(),
                chosen=chosen[:E].copy(), total=total[:E].copy(), nvotes=nvotes[:E].copy(),
                is_max=is_max[:E].copy(), flow=flow[:E].copy(), voff=voff[:E + 1].copy(),
                vlist=vlist[:voff[E]].copy(), seeds_push=spush[:S].copy(), seeds=ssorted[:S].copy())


class Marker(C.Structure):
    _fields_ = [("id", _I), ("status", _I), ("x", _F), ("y", _F), ("cx", _F), ("cy", _F), ("a", _F), ("b", _F),
                ("angle", _F), ("quality", _F), ("level", _I)]


def detect(gray: np.ndarray, params=None, fp64: bool = False, cap: int = 512):
    """Whole CPU detection (oracle image stage + candidate stage + oracle
    identification); returns a list of Marker records."""
    from cctag_b200.capi import Params  # the ctypes layout of cctagb_params only

    lib = load()
    lib.orc_detect.argtypes = [_P, _I, _I, C.POINTER(Params), _I, _P, _I]
    lib.orc_detect.restype = _I
    lib.orc_params_default.argtypes = [C.POINTER(Params), _I]
    if params is None:
        params = Params()
        lib.orc_params_default(C.byref(params), 3)
    p = params
    g = np.ascontiguousarray(gray, dtype=np.uint8)
    out = (Marker * cap)()
    n = lib.orc_detect(_p(g), g.shape[1], g.shape[0], C.byref(p), int(bool(fp64)), C.cast(out, C.c_void_p), cap)
    return [out[i] for i in range(min(n, cap))]


def cut_selection(gray: np.ndarray, params=None, cap: int = 512):
    """identify_step_1 of every candidate of a frame, in candidate order:
    a list of (status, stops) with stops an (ncuts, 2) float32 array of the
    selected cut ends (Identification.cpp:1172-1300)."""
    from cctag_b200.capi import Params

    lib = load()
    lib.orc_cut_selection.argtypes = [_P, _I, _I, C.POINTER(Params), _P, _P, _P, _I, _I]
    lib.orc_cut_selection.restype = _I
    lib.orc_params_default.argtypes = [C.POINTER(Params), _I]
    if params is None:
        params = Params()
        lib.orc_params_default(C.byref(params), 3)
    g = np.ascontiguousarray(gray, dtype=np.uint8)
    kc = 32
    status = np.zeros(cap, np.int32)
    ncuts = np.zeros(cap, np.int32)
    stops = np.zeros((cap, kc, 2), np.float32)
    n = lib.orc_cut_selection(_p(g), g.shape[1], g.shape[0], C.byref(params), _p(status), _p(ncuts), _p(stops), kc,
                              cap)
    return [(int(status[i]), stops[i, :ncuts[i]].copy()) for i in range(min(n, cap))]


def loop_two(gray: np.ndarray, level: int, params=None):
    """Loop 1 and the outlier removal of loop 2 (host restatement) for one
    level: (seed, score, keep, filtered) as Detector.level_loop_two."""
    from cctag_b200.capi import Params

    lib = load()
    lib.orc_loop_two.argtypes = [_P, _I, _I, C.POINTER(Params), _I, _I, _P, _P, _P, _P, _I, _P, C.POINTER(_I)]
    lib.orc_loop_two.restype = _I
    lib.orc_params_default.argtypes = [C.POINTER(Params), _I]
    if params is None:
        params = Params()
        lib.orc_params_default(C.byref(params), 3)
    g = np.ascontiguousarray(gray, dtype=np.uint8)
    cap, fcap = 4096, 1 << 22
    seed, score, keep, nflt = (np.zeros(cap, np.int32) for _ in range(4))
    flt = np.zeros(fcap, np.int32)
    nt = C.c_int()
    n = lib.orc_loop_two(_p(g), g.shape[1], g.shape[0], C.byref(params), level, cap, _p(seed), _p(score),
                         _p(keep), _p(nflt), fcap, _p(flt), C.byref(nt))
    if n < 0:
        raise ValueError("orc_loop_two failed")
    offs = np.concatenate([[0], np.cumsum(nflt[:n])])
    return seed[:n].copy(), score[:n].copy(), keep[:n].copy(), [flt[offs[i]:offs[i + 1]].copy() for i in range(n)]


# ------------------------------------------------ batched identification --
def _refine_sigs(lib):
    D = C.c_double
    lib.orc_cut_cost_h.argtypes = [_P, C.c_size_t, _P, _P, _I, D, _P, _P]
    lib.orc_cut_cost_h.restype = _I
    lib.orc_cut_cost.argtypes = [_P, C.c_size_t, _P, D, D, _I, D, _P, _P]
    lib.orc_cut_cost.restype = _I
    lib.orc_refine_grid.argtypes = [_P, C.c_size_t, _P, _I, D, _I, D, D, _P]
    lib.orc_refine_grid.restype = _I


def _begin_sig(n_crowns=3):
    return float(np.float32(1.0) - np.float32(2 * n_crowns - 1) * np.float32(0.15))


def cut_cost(img: np.ndarray, task, cx: float, cy: float, n_samples: int = 100, n_crowns: int = 3):
    """FP64 cost of a cctagb_cut_task at an imaged center: (cost, d_center[2],
    d_h[9], H[9]); cost is None when fewer than two cuts stay inside."""
    lib = load()
    _refine_sigs(lib)
    g = np.ascontiguousarray(img, dtype=np.uint8)
    out = np.zeros(12)
    H = np.zeros(9)
    ok = lib.orc_cut_cost(_p(g), g.shape[1], C.byref(task), cx, cy, n_samples, _begin_sig(n_crowns), _p(out), _p(H))
    return (out[0] if ok else None), out[1:3].copy(), out[3:12].copy(), H


def cut_cost_h(img: np.ndarray, task, H, n_samples: int = 100, n_crowns: int = 3):
    """FP64 cost of a task at a given homography and d cost / d H."""
    lib = load()
    _refine_sigs(lib)
    g = np.ascontiguousarray(img, dtype=np.uint8)
    Hd = np.ascontiguousarray(H, dtype=np.float64).reshape(9)
    cost = C.c_double()
    grad = np.zeros(9)
    ok = lib.orc_cut_cost_h(_p(g), g.shape[1], C.byref(task), _p(Hd), n_samples, _begin_sig(n_crowns), C.byref(cost),
                            _p(grad))
    return (cost.value if ok else None), grad


def refine_grid(img: np.ndarray, task, stop_width: float = 0.02, n_samples: int = 100, n_crowns: int = 3,
                grid_n: int = 5, neighbour_size: float = 0.2):
    """FP64 grid refinement of a task continued to `stop_width`: (x, y, cost) or None."""
    lib = load()
    _refine_sigs(lib)
    g = np.ascontiguousarray(img, dtype=np.uint8)
    out = np.zeros(3)
    ok = lib.orc_refine_grid(_p(g), g.shape[1], C.byref(task), n_samples, _begin_sig(n_crowns), grid_n,
                             neighbour_size, stop_width, _p(out))
    return (float(out[0]), float(out[1]), float(out[2])) if ok else None
