"""ctypes binding of the C ABI (``include/cctag_b200.h``).

Loading fails loudly: there is no CPU fallback behind this module.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libcctag_b200.so"

OK, BAD_ARG, CUDA_ERROR, NO_DEVICE = 0, 1, 2, 3
OVERFLOW_EDGES, OVERFLOW_SEEDS, OVERFLOW_VOTERS, HYST_NO_CONVERGE = 4, 5, 6, 7
TOO_LARGE, BANK_ERROR, INTERNAL = 8, 9, 10

REFINE_GRID, REFINE_GAUSS_NEWTON = 0, 1
IDENT_AUTO, IDENT_BLOCK = 0, 1
TUNE_MAX_TRIED = 16


class Params(C.Structure):
    """Mirror of ``cctagb_params`` (field names of cctag::Parameters)."""
    _fields_ = [
        ("cannyThrLow", C.c_float), ("cannyThrHigh", C.c_float), ("distSearch", C.c_int),
        ("thrGradientMagInVote", C.c_int), ("angleVoting", C.c_float), ("ratioVoting", C.c_float),
        ("averageVoteMin", C.c_float), ("thrMedianDistanceEllipse", C.c_float), ("maximumNbSeeds", C.c_int),
        ("maximumNbCandidatesLoopTwo", C.c_int), ("nCrowns", C.c_int), ("nCircles", C.c_int),
        ("minPointsSegmentCandidate", C.c_int), ("minVotesToSelectCandidate", C.c_int),
        ("threshRobustEstimationOfOuterEllipse", C.c_float), ("ellipseGrowingEllipticHullWidth", C.c_float),
        ("windowSizeOnInnerEllipticSegment", C.c_int), ("numberOfMultiresLayers", C.c_int),
        ("numberOfProcessedMultiresLayers", C.c_int), ("nSamplesOuterEllipse", C.c_int),
        ("numCutsInIdentStep", C.c_int), ("numSamplesOuterEdgePointsRefinement", C.c_int),
        ("cutsSelectionTrials", C.c_int), ("sampleCutLength", C.c_int), ("imagedCenterNGridSample", C.c_int),
        ("imagedCenterNeighbourSize", C.c_float), ("minIdentProba", C.c_float), ("useLMDif", C.c_int),
        ("searchForAnotherSegment", C.c_int), ("writeOutput", C.c_int), ("doIdentification", C.c_int),
        ("maxEdges", C.c_uint32), ("refineMode", C.c_int), ("gnIterations", C.c_int),
        ("gnCoarseRounds", C.c_int), ("edgeCapacityDivisor", C.c_int), ("hostThreads", C.c_int),
        ("gnCoarseGrid", C.c_int), ("gnCoarseNeighbourSize", C.c_float), ("batchWaveFrames", C.c_int),
        ("identLayout", C.c_int), ("hostSpinMicros", C.c_int), ("gpuEllipseGrowing", C.c_int),
        ("gpuGrowMaxPoints", C.c_int),
    ]


class TuneChoice(C.Structure):
    """Mirror of ``cctagb_tune_choice``."""
    _fields_ = [("batchWaveFrames", C.c_int), ("identLayout", C.c_int), ("ms_per_frame", C.c_float),
                ("from_cache", C.c_int), ("n_tried", C.c_int), ("tried_wave", C.c_int * TUNE_MAX_TRIED),
                ("tried_layout", C.c_int * TUNE_MAX_TRIED), ("tried_ms_per_frame", C.c_float * TUNE_MAX_TRIED),
                ("hostThreads", C.c_int), ("tried_threads", C.c_int * TUNE_MAX_TRIED)]


class Ellipse(C.Structure):
    _fields_ = [("cx", C.c_float), ("cy", C.c_float), ("a", C.c_float), ("b", C.c_float), ("angle", C.c_float),
                ("m", C.c_float * 9)]


class Marker(C.Structure):
    _fields_ = [("id", C.c_int), ("status", C.c_int), ("x", C.c_float), ("y", C.c_float), ("outer", Ellipse),
                ("homography", C.c_float * 9), ("quality", C.c_float), ("pyramidLevel", C.c_int),
                ("scale", C.c_float)]


class Stats(C.Structure):
    _fields_ = [("edge_points", C.c_int * 8), ("seeds", C.c_int * 8), ("candidates", C.c_int),
                ("markers", C.c_int), ("ms_image_stage", C.c_float), ("ms_host_candidates", C.c_float),
                ("ms_identify", C.c_float), ("ms_total", C.c_float), ("h2d_bytes", C.c_longlong),
                ("d2h_bytes", C.c_longlong), ("kernel_launches", C.c_int), ("ms_download", C.c_float),
                ("ms_cut_selection", C.c_float), ("grown_gpu", C.c_int), ("grown_host", C.c_int)]


class Frame(C.Structure):
    _fields_ = [("gray", C.c_void_p), ("w", C.c_int), ("h", C.c_int), ("pitch", C.c_size_t),
                ("frame_id", C.c_int), ("is_device", C.c_int), ("out", C.POINTER(Marker)), ("cap", C.c_int),
                ("n_out", C.c_int), ("status", C.c_int), ("stats", Stats)]


MAX_CUTS = 32


class CutTask(C.Structure):
    _fields_ = [("Q", C.c_float * 9), ("cx", C.c_float), ("cy", C.c_float), ("a", C.c_float), ("b", C.c_float),
                ("angle", C.c_float), ("x0", C.c_float), ("y0", C.c_float), ("ncuts", C.c_int),
                ("stop", (C.c_float * 2) * MAX_CUTS), ("roi", C.c_int * 4), ("local", C.c_int)]


class IdentResult(C.Structure):
    _fields_ = [("status", C.c_int), ("id", C.c_int), ("x", C.c_float), ("y", C.c_float), ("H", C.c_float * 9),
                ("residual", C.c_float), ("score", C.c_float), ("nvalid", C.c_int), ("iterations", C.c_int)]


# Every symbol declared in include/cctag_b200.h, with its signature.
_P = C.c_void_p
_I = C.c_int
_SZ = C.c_size_t
SIGNATURES = {
    "cctagb_params_default": (None, [C.POINTER(Params), _I]),
    "cctagb_status_string": (C.c_char_p, [_I]),
    "cctagb_create": (_I, [C.POINTER(Params), _I, _I, _I, C.POINTER(_P)]),
    "cctagb_destroy": (_I, [_P]),
    "cctagb_last_error_string": (C.c_char_p, [_P]),
    "cctagb_set_bank": (_I, [_P, _P, _I, _I]),
    "cctagb_detect": (_I, [_P, _P, _I, _I, _SZ, _I, _P, _I, C.POINTER(_I), _P]),
    "cctagb_detect_device": (_I, [_P, _P, _I, _I, _SZ, _I, _P, _I, C.POINTER(_I), _P]),
    "cctagb_detect_batch": (_I, [_P, _P, _I]),
    "cctagb_host_frames": (_I, [_P, _I, C.POINTER(_P)]),
    "cctagb_submit": (_I, [_P, _P, _I, _I, _SZ, _I, _I, C.POINTER(_I)]),
    "cctagb_wait": (_I, [_P, _I, _P, _I, C.POINTER(_I), _P]),
    "cctagb_last_tasks": (_I, [_P, _P, _I, C.POINTER(_I)]),
    "cctagb_identify_tasks": (_I, [_P, _P, _I, _I, _SZ, _P, _I, _I, _P]),
    "cctagb_cut_cost": (_I, [_P, _P, _I, _I, _SZ, _P, _I, _P, _P, _P, _P]),
    "cctagb_cut_cost_f64": (_I, [_P, _P, _I, _I, _SZ, _P, _I, _P, _P, _P, _P]),
    "cctagb_image_stage": (_I, [_P, _P, _I, _I, _SZ, _I]),
    "cctagb_level_size": (_I, [_P, _I, C.POINTER(_I), C.POINTER(_I)]),
    "cctagb_level_planes": (_I, [_P, _I, _P, _P, _P, _P]),
    "cctagb_level_edge_points": (_I, [_P, _I, _I, C.POINTER(_I), _P, _P]),
    "cctagb_level_links": (_I, [_P, _I, _I, _P, _P]),
    "cctagb_level_votes": (_I, [_P, _I, _I, _P, _P, _P, _P, _P, _I, _P]),
    "cctagb_level_seeds": (_I, [_P, _I, _I, _P, C.POINTER(_I)]),
    "cctagb_level_loop_two": (_I, [_P, _I, _I, _P, _P, _P, _P, C.POINTER(_I), _I, _P, C.POINTER(_I)]),
    "cctagb_canny_from_derivatives": (_I, [_P, _P, _P, _I, _I, _P]),
    "cctagb_get_stream": (_I, [_P, C.POINTER(_P)]),
    "cctagb_set_stage_timing": (_I, [_P, _I]),
    "cctagb_stage_times": (_I, [_P, _I, _P, C.POINTER(_I)]),
    "cctagb_stage_name": (C.c_char_p, [_I]),
    "cctagb_edges_noalloc": (_I, [_P, _I, _I, _SZ, C.c_float, C.c_float, _P, _P, _P, _P, _P]),
    "cctagb_autotune": (_I, [_P, _P, _I, C.c_char_p, _I, C.POINTER(TuneChoice)]),
    "cctagb_tune_key": (_I, [C.c_char_p, _I, _I, _I, _I, _I, C.c_char_p, _I]),
    "cctagb_tune_cache_get": (_I, [C.c_char_p, C.c_char_p, C.POINTER(TuneChoice)]),
    "cctagb_tune_cache_put": (_I, [C.c_char_p, C.c_char_p, C.POINTER(TuneChoice)]),
}

_lib = None


def load() -> C.CDLL:
    """Load the library (built by ``cctag_b200.build``); raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run cctag_b200/build.py (there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class CCTagError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


def default_params(n_crowns: int = 3) -> Params:
    p = Params()
    load().cctagb_params_default(C.byref(p), n_crowns)
    return p


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
