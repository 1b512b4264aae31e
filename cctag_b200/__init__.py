"""B200-native CCTag detection hot path.

Python view of the C ABI (``include/cctag_b200.h``) for tests, benchmarks and
scripting.  C++ callers use the header-only shim ``include/cctag_b200/ICCTag.hpp``
which mirrors the reference's ``ICCTag.hpp`` API.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import CCTagError, Params, default_params


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)

__all__ = ["Detector", "CCTagError", "Params", "default_params", "capi"]


class Detector:
    """One handle (device arena, stream, captured graphs).  Not thread-safe."""

    def __init__(self, params: Params | None = None, max_w: int = 1920, max_h: int = 1080, max_batch: int = 1):
        self._lib = capi.load()
        self.params = params if params is not None else default_params(3)
        h = C.c_void_p()
        st = self._lib.cctagb_create(C.byref(self.params), int(max_w), int(max_h), int(max_batch), C.byref(h))
        if st != capi.OK:
            raise CCTagError(st, f"cctagb_create failed: {self._lib.cctagb_status_string(st).decode()}")
        self._h = h
        self.max_w, self.max_h = int(max_w), int(max_h)
        self._tickets: dict = {}   # ticket -> key of the host frame kept alive until waited
        self._inflight: dict = {}

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.cctagb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int, what: str):
        if st != capi.OK:
            msg = self._lib.cctagb_last_error_string(self._h).decode()
            raise CCTagError(st, f"{what}: {msg}")

    # -- configuration -----------------------------------------------------
    def set_bank(self, ratios):
        a = np.ascontiguousarray(np.asarray(ratios, dtype=np.float32))
        if a.ndim != 2:
            raise ValueError("bank must be a 2-D array (ids x ratios)")
        self._check(self._lib.cctagb_set_bank(self._h, capi.ptr(a), a.shape[0], a.shape[1]), "set_bank")

    # -- image stage ---------------------------------------------------------
    def image_stage(self, gray: np.ndarray):
        g = np.ascontiguousarray(gray, dtype=np.uint8)
        H, W = g.shape
        self._check(self._lib.cctagb_image_stage(self._h, capi.ptr(g), W, H, W, 0), "image_stage")

    def image_stage_device(self, dptr: int, w: int, h: int, pitch: int):
        self._check(self._lib.cctagb_image_stage(self._h, C.c_void_p(dptr), w, h, pitch, 1), "image_stage")

    def level_size(self, level: int):
        w, h = C.c_int(), C.c_int()
        self._check(self._lib.cctagb_level_size(self._h, level, C.byref(w), C.byref(h)), "level_size")
        return w.value, h.value

    def level_planes(self, level: int):
        w, h = self.level_size(level)
        src = np.empty((h, w), np.uint8)
        dx = np.empty((h, w), np.int16)
        dy = np.empty((h, w), np.int16)
        edges = np.empty((h, w), np.uint8)
        self._check(self._lib.cctagb_level_planes(self._h, level, capi.ptr(src), capi.ptr(dx), capi.ptr(dy),
                                                  capi.ptr(edges)), "level_planes")
        return src, dx, dy, edges

    def edge_points(self, level: int):
        w, h = self.level_size(level)
        cap = w * h
        n = C.c_int()
        x = np.empty(cap, np.int32)
        y = np.empty(cap, np.int32)
        self._check(self._lib.cctagb_level_edge_points(self._h, level, cap, C.byref(n), capi.ptr(x), capi.ptr(y)),
                    "edge_points")
        return x[:n.value].copy(), y[:n.value].copy()

    def links(self, level: int):
        x, _ = self.edge_points(level)
        n = len(x)
        b = np.empty(max(n, 1), np.int32)
        a = np.empty(max(n, 1), np.int32)
        self._check(self._lib.cctagb_level_links(self._h, level, max(n, 1), capi.ptr(b), capi.ptr(a)), "links")
        return b[:n].copy(), a[:n].copy()

    def votes(self, level: int):
        x, _ = self.edge_points(level)
        n = len(x)
        cap = max(n, 1)
        chosen = np.empty(cap, np.int32)
        nvotes = np.empty(cap, np.int32)
        flow = np.empty(cap, np.float32)
        voff = np.empty(cap + 1, np.int32)
        vlist = np.empty(cap, np.int32)
        nv = np.zeros(1, np.int32)
        self._check(self._lib.cctagb_level_votes(self._h, level, cap, capi.ptr(chosen), capi.ptr(nvotes),
                                                 capi.ptr(flow), capi.ptr(voff), capi.ptr(vlist), cap,
                                                 capi.ptr(nv)), "votes")
        return dict(chosen=chosen[:n].copy(), nvotes=nvotes[:n].copy(), flow=flow[:n].copy(),
                    voff=voff[:n + 1].copy(), vlist=vlist[:nv[0]].copy())

    def seeds(self, level: int):
        x, _ = self.edge_points(level)
        cap = max(len(x), 1)
        s = np.empty(cap, np.int32)
        n = C.c_int()
        self._check(self._lib.cctagb_level_seeds(self._h, level, cap, capi.ptr(s), C.byref(n)), "seeds")
        return s[:n.value].copy()

    def canny_from_derivatives(self, dx: np.ndarray, dy: np.ndarray) -> np.ndarray:
        dx = np.ascontiguousarray(dx, dtype=np.int16)
        dy = np.ascontiguousarray(dy, dtype=np.int16)
        H, W = dx.shape
        out = np.empty((H, W), np.uint8)
        self._check(self._lib.cctagb_canny_from_derivatives(self._h, capi.ptr(dx), capi.ptr(dy), W, H,
                                                            capi.ptr(out)), "canny_from_derivatives")
        return out

    # -- timing --------------------------------------------------------------
    @property
    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self._lib.cctagb_get_stream(self._h, C.byref(s)), "get_stream")
        return s.value or 0

    def set_stage_timing(self, on: bool = True):
        self._check(self._lib.cctagb_set_stage_timing(self._h, int(bool(on))), "set_stage_timing")

    def stage_times(self) -> dict:
        ms = np.zeros(64, np.float32)
        n = C.c_int()
        self._check(self._lib.cctagb_stage_times(self._h, 64, capi.ptr(ms), C.byref(n)), "stage_times")
        return {self._lib.cctagb_stage_name(k).decode(): float(ms[k]) for k in range(n.value)}

    # -- detection -----------------------------------------------------------
    def detect_device(self, dptr: int, w: int, h: int, pitch: int, frame_id: int = 0, cap: int = 256):
        out = (capi.Marker * cap)()
        n = C.c_int()
        stats = capi.Stats()
        self._check(self._lib.cctagb_detect_device(self._h, C.c_void_p(dptr), w, h, pitch, frame_id, out, cap,
                                                   C.byref(n), C.byref(stats)), "detect_device")
        return [out[i] for i in range(n.value)], stats

    @staticmethod
    def _frame_array(frames, cap):
        """cctagb_frame array of uint8 numpy arrays (host) or ``(device_ptr,
        w, h, pitch)`` tuples (device memory), with the buffers it points to."""
        n = len(frames)
        fr = (capi.Frame * n)()
        outs = [(capi.Marker * cap)() for _ in range(n)]
        keep = []
        for i, f in enumerate(frames):
            if isinstance(f, np.ndarray):
                g = np.ascontiguousarray(f, dtype=np.uint8)
                keep.append(g)
                fr[i].gray, fr[i].h, fr[i].w = g.ctypes.data, g.shape[0], g.shape[1]
                fr[i].pitch, fr[i].is_device = g.shape[1], 0
            else:
                fr[i].gray, fr[i].w, fr[i].h, fr[i].pitch = f
                fr[i].is_device = 1
            fr[i].frame_id = i
            fr[i].out = C.cast(outs[i], C.POINTER(capi.Marker))
            fr[i].cap = cap
        return fr, outs, keep

    def detect_batch(self, frames, cap: int = 256):
        """Detection of several independent frames (cctagb_detect_batch).

        `frames` holds uint8 numpy arrays (host) or ``(device_ptr, w, h, pitch)``
        tuples (device memory).  Returns one ``(markers, stats)`` pair per frame.
        """
        fr, outs, _keep = self._frame_array(frames, cap)
        n = len(frames)
        self._check(self._lib.cctagb_detect_batch(self._h, fr, n), "detect_batch")
        return [([outs[i][k] for k in range(fr[i].n_out)], fr[i].stats) for i in range(n)]

    def autotune(self, frames, cache_path: str | None = None, reps: int = 3, cap: int = 256) -> dict:
        """Choose and set the batch configuration for these frames
        (cctagb_autotune): from the cache file when it holds the key, else
        measured on the frames and written to the cache file."""
        fr, _outs, _keep = self._frame_array(frames, cap)
        ch = capi.TuneChoice()
        path = None if cache_path is None else str(cache_path).encode()
        self._check(self._lib.cctagb_autotune(self._h, fr, len(frames), path, int(reps), C.byref(ch)), "autotune")
        self.params.batchWaveFrames = ch.batchWaveFrames
        self.params.identLayout = ch.identLayout
        self.params.hostThreads = ch.hostThreads
        return tune_choice_dict(ch)

    # -- streaming ingest --------------------------------------------------------
    def host_frames(self, n: int):
        """n pinned frame buffers owned by the handle, as (max_h, max_w) uint8 arrays."""
        ptrs = (C.c_void_p * n)()
        self._check(self._lib.cctagb_host_frames(self._h, n, ptrs), "host_frames")
        size = self.max_w * self.max_h
        return [np.ctypeslib.as_array((C.c_uint8 * size).from_address(p)).reshape(self.max_h, self.max_w)
                for p in ptrs]

    def submit(self, gray, frame_id: int = 0, w: int | None = None, h: int | None = None, pitch: int | None = None,
               is_device: bool = False) -> int:
        """cctagb_submit: a host numpy frame (kept alive until waited) or a
        device pointer with w/h/pitch; returns the ticket."""
        t = C.c_int()
        if isinstance(gray, np.ndarray):
            g = gray if gray.flags["C_CONTIGUOUS"] and gray.dtype == np.uint8 else np.ascontiguousarray(gray, np.uint8)
            hh, ww = g.shape
            ptr, pitch, is_device = g.ctypes.data, int(g.strides[0]), False
            self._inflight[id(g)] = g
        else:
            ptr, ww, hh = int(gray), int(w), int(h)
            pitch = int(pitch if pitch is not None else ww)
        self._check(self._lib.cctagb_submit(self._h, C.c_void_p(ptr), ww, hh, pitch, int(is_device), frame_id,
                                            C.byref(t)), "submit")
        if isinstance(gray, np.ndarray):
            self._tickets[t.value] = id(g)
        return t.value

    def wait(self, ticket: int, cap: int = 256):
        """cctagb_wait: (markers, stats) of a submitted frame."""
        out = (capi.Marker * cap)()
        n = C.c_int()
        stats = capi.Stats()
        try:
            self._check(self._lib.cctagb_wait(self._h, ticket, out, cap, C.byref(n), C.byref(stats)), "wait")
        finally:
            key = self._tickets.pop(ticket, None)
            if key is not None:
                self._inflight.pop(key, None)
        return [out[i] for i in range(n.value)], stats

    def level_loop_two(self, level: int):
        """Loop-two inputs of one level from the last detect (GPU loop 1 and
        outlier removal): (seed, score, keep, filtered) with filtered a list
        of int32 arrays (empty for candidates not kept)."""
        cap, fcap = 4096, 1 << 22
        seed = np.zeros(cap, np.int32)
        score = np.zeros(cap, np.int32)
        keep = np.zeros(cap, np.int32)
        nflt = np.zeros(cap, np.int32)
        flt = np.zeros(fcap, np.int32)
        n, nt = C.c_int(), C.c_int()
        self._check(self._lib.cctagb_level_loop_two(self._h, level, cap, _ptr(seed), _ptr(score), _ptr(keep),
                                                    _ptr(nflt), C.byref(n), fcap, _ptr(flt), C.byref(nt)),
                    "level_loop_two")
        k = n.value
        offs = np.concatenate([[0], np.cumsum(nflt[:k])])
        return seed[:k].copy(), score[:k].copy(), keep[:k].copy(), [flt[offs[i]:offs[i + 1]].copy() for i in range(k)]

    # -- identification of caller-given candidates ---------------------------
    def last_tasks(self):
        """Identification tasks of the last detect call (ctypes CutTask array)."""
        n = C.c_int()
        cap = 1024
        out = (capi.CutTask * cap)()
        self._check(self._lib.cctagb_last_tasks(self._h, out, cap, C.byref(n)), "last_tasks")
        return out[:n.value]

    def identify_tasks(self, dptr: int, w: int, h: int, pitch: int, tasks, refine_mode: int = capi.REFINE_GRID):
        """cctagb_identify_tasks on a device image; returns IdentResult list."""
        n = len(tasks)
        arr = (capi.CutTask * n)(*tasks)
        out = (capi.IdentResult * n)()
        self._check(self._lib.cctagb_identify_tasks(self._h, C.c_void_p(dptr), w, h, pitch, arr, n, refine_mode,
                                                    out), "identify_tasks")
        return list(out)

    def cut_cost(self, dptr: int, w: int, h: int, pitch: int, tasks, centers: np.ndarray, fp64: bool = False):
        """cctagb_cut_cost (or cctagb_cut_cost_f64): (cost[n], d_center[n,2], d_h[n,9])."""
        n = len(tasks)
        arr = (capi.CutTask * n)(*tasks)
        c = np.ascontiguousarray(centers, dtype=np.float32).reshape(n, 2)
        cost = np.zeros(n, np.float32)
        dc = np.zeros((n, 2), np.float32)
        dh = np.zeros((n, 9), np.float32)
        fn = self._lib.cctagb_cut_cost_f64 if fp64 else self._lib.cctagb_cut_cost
        self._check(fn(self._h, C.c_void_p(dptr), w, h, pitch, arr, n, capi.ptr(c), capi.ptr(cost), capi.ptr(dc),
                       capi.ptr(dh)), "cut_cost")
        return cost, dc, dh

    def detect(self, gray: np.ndarray, frame_id: int = 0, cap: int = 256):
        g = np.ascontiguousarray(gray, dtype=np.uint8)
        H, W = g.shape
        out = (capi.Marker * cap)()
        n = C.c_int()
        stats = capi.Stats()
        self._check(self._lib.cctagb_detect(self._h, capi.ptr(g), W, H, W, frame_id, out, cap, C.byref(n),
                                            C.byref(stats)), "detect")
        return [out[i] for i in range(n.value)], stats


def tune_choice_dict(ch: capi.TuneChoice) -> dict:
    return {"batchWaveFrames": ch.batchWaveFrames, "identLayout": ch.identLayout, "hostThreads": ch.hostThreads,
            "ms_per_frame": round(float(ch.ms_per_frame), 4), "from_cache": bool(ch.from_cache),
            "tried": [{"batchWaveFrames": ch.tried_wave[i], "identLayout": ch.tried_layout[i],
                       "hostThreads": ch.tried_threads[i],
                       "ms_per_frame": round(float(ch.tried_ms_per_frame[i]), 4)} for i in range(ch.n_tried)]}


def tune_key(gpu_name: str, sm_count: int, w: int, h: int, frames: int, n_crowns: int) -> str:
    """Cache key of a batch configuration (cctagb_tune_key)."""
    buf = C.create_string_buffer(512)
    st = capi.load().cctagb_tune_key(gpu_name.encode(), sm_count, w, h, frames, n_crowns, buf, len(buf))
    if st != capi.OK:
        raise CCTagError(st, "tune_key")
    return buf.value.decode()


def tune_cache_get(cache_path: str, key: str) -> dict | None:
    """The cache file's entry for `key` (cctagb_tune_cache_get), None if absent."""
    ch = capi.TuneChoice()
    st = capi.load().cctagb_tune_cache_get(str(cache_path).encode(), key.encode(), C.byref(ch))
    return tune_choice_dict(ch) if st == capi.OK else None


def tune_cache_put(cache_path: str, key: str, batch_wave_frames: int, ident_layout: int, ms_per_frame: float = 0.0,
                   host_threads: int = 0):
    """Add or replace the cache file's entry for `key` (cctagb_tune_cache_put)."""
    ch = capi.TuneChoice()
    ch.batchWaveFrames, ch.identLayout, ch.ms_per_frame = batch_wave_frames, ident_layout, ms_per_frame
    ch.hostThreads = host_threads
    st = capi.load().cctagb_tune_cache_put(str(cache_path).encode(), key.encode(), C.byref(ch))
    if st != capi.OK:
        raise CCTagError(st, "tune_cache_put")
