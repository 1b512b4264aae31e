"""Benchmark of the CCTag detection hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--config NAME]

One step = a batch of 16 synthetic 1920x1080 frames (12 markers each, noise,
motion blur, illumination gradient; seeded) through the whole detection:
pyramid, derivatives, Canny, thinning, edge points, vote and seeds on the GPU,
the candidate stage on the host, cut selection on the host, identification on
the GPU.  The batch goes through cctagb_detect_batch, whose slots overlap one
frame's host stage with other frames' GPU stages.  N > 1 runs one independent
replica per GPU on its own frames (no collective on the data path); `value` is
frames/s over all ranks, timed as the max over ranks.

`value`: frames/s with the frames already in device memory.
`e2e`: frames/s with the frames in pinned host memory (host->device copies and
every device->host download inside the timed region).
`plain`: the same frames one at a time through cctagb_detect_device /
cctagb_detect (single-frame latency path).
`c4_cameras`: 16 cameras per step at mixed resolutions (640x480 .. 3840x2160,
0-20 markers each) through cctagb_detect_batch, with per-frame p50/p99.
Between timed steps the L2 is flushed by writing a 256 MiB buffer (untimed);
each step is bracketed by CUDA events on the library's stream (every call is
synchronous, so the closing event follows all of the step's work).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "1080p frames/s + per-stage HBM GB/s; batched/adjoint vs plain at <=0.05 px"
UNIT = "frames/s"
BATCH = 16  # frames per step (distinct seeded frames)
SLOTS = 16  # detection slots of the batch handle (one wave of 16 frames per step)
N_FRAMES = BATCH


# ------------------------------------------------------------------ helpers --
def dist_setup(backend: str | None = None):
    """Rank, world size and local rank from the launcher's environment; the
    process group is NCCL on GPUs (gloo when there is no GPU, for tests)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    """The largest of every rank's x (device times: the job takes the slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def frame_seeds(rank, n):
    """Seeds of a rank's frames: replicas work on their own frames."""
    return [100 + i + 1000 * rank for i in range(n)]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([c.strip() for c in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(s):
            try:
                return float(s)
            except ValueError:
                return None

        sm = [v for v in (num(r[1]) for r in self.rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in self.rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def host_pool():
    """Process pool (spawn: safe after CUDA is initialised) to render the
    synthetic inputs over the host cores."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    return ProcessPoolExecutor(max_workers=os.cpu_count() or 1, mp_context=mp.get_context("spawn"))


def tune_cache_path():
    """The autotuner's JSON cache: $CCTAG_B200_TUNE_CACHE, else a file in the
    user's cache directory."""
    p = Path(os.environ.get("CCTAG_B200_TUNE_CACHE") or Path.home() / ".cache" / "cctag_b200" / "tune.json")
    p.parent.mkdir(parents=True, exist_ok=True)
    return p


def autotune(det, fr, reps=5):
    """Batch configuration of `det` for the frames of `fr` (cctagb_autotune)."""
    import cctag_b200
    from cctag_b200 import capi

    ch = capi.TuneChoice()
    det._check(det._lib.cctagb_autotune(det._h, fr, len(fr), str(tune_cache_path()).encode(), reps, C.byref(ch)),
               "autotune")
    return cctag_b200.tune_choice_dict(ch)


def make_frames(config, n=N_FRAMES, rank=0):
    from cctag_b200.synth import config_frame

    return [config_frame(config, seed=sd).image for sd in frame_seeds(rank, n)]


# -------------------------------------------------------- algorithmic bytes --
def stage_bytes(levels, E, S, V):
    """Algorithmic bytes per image-stage kernel group for one frame (n = level
    pixels, E = edge points, S = seeds, V = votes cast)."""
    n = [w * h for (w, h) in levels]
    nt = sum(n)
    Et, St, Vt = sum(E), sum(S), sum(V)
    return {
        "pyramid": n[0] + sum(n[1:]),                 # read level 0, write levels 1..3
        "deriv_nms": 6 * nt,                          # 1 B in, dx+dy 4 B + class map 1 B out
        "hyst_merge": 1 * nt,                         # class map in (tile bit planes are its own output)
        "hyst_compress": 3 * nt // 8,                 # two tile bit planes in, result bit plane out
        "final_thin": nt // 4,                        # result bit plane in, edge bitmap out
        "row_scan": 8 * sum(h for (_, h) in levels),
        # bitmap in, word + first-index plane out, dx/dy gathers, points, gradients, vote counters out
        "emit": nt // 8 + nt // 4 + 4 * Et + 16 * Et,
        "walk": 8 * Et + 8 * Et + nt // 8,            # points + gradients in, links out, bitmap once
        "vote": 8 * Et + 8 * Et,                      # links in, chosen + length out
        "voter_scan": 4 * Et + 4 * Et,
        "voter_fill": 4 * Et + 4 * Vt,
        "voter_sort": 8 * Vt + 4 * Et + 8 * St,
    }


def ident_flops(n_markers, rounds=10, trials=25, cuts=22, samples=100):
    """FP32 operations of the grid refinement (per candidate and round: 25
    trials x 22 cuts x 100 samples of homography + bilinear ~ 30 flop, plus the
    cost accumulation ~ 3 flop per sample)."""
    return n_markers * rounds * trials * cuts * samples * 33


def profiled_traffic(config):
    """DRAM bytes per launch of each image-stage kernel group (one launch over
    the 16 frames of a step), from the ncu summary of this workload under
    profiles/ (cold-cache capture; the `stage: bytes` lines of its last code
    block)."""
    name = {"c2_1080p": "dram_image_stage_c2_1080p_batch16.md"}.get(config)
    f = ROOT / "profiles" / name if name else None
    if not f or not f.exists():
        return {}
    blocks = f.read_text().split("```")
    out = {}
    for line in blocks[-2].splitlines() if len(blocks) >= 3 else []:
        k, _, v = line.partition(":")
        if v.strip().isdigit():
            out[k.strip()] = int(v)
    return out


# ------------------------------------------------------------ the b200 arm --
def run_b200(args, rank, world, local):
    import torch

    import cctag_b200
    from cctag_b200 import capi

    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    frames = make_frames(args.config, rank=rank)
    H, W = frames[0].shape
    det = cctag_b200.Detector(max_w=W, max_h=H, max_batch=SLOTS)
    stream = torch.cuda.ExternalStream(det.stream)
    # single-frame calls on a handle of their own (one slot: the whole host pool)
    det1 = cctag_b200.Detector(max_w=W, max_h=H)
    stream1 = torch.cuda.ExternalStream(det1.stream)
    d_frames = [torch.from_numpy(f).to(dev) for f in frames]
    h_frames = [torch.from_numpy(f).pin_memory() for f in frames]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    cap = 512
    outs = [(capi.Marker * cap)() for _ in range(BATCH)]

    def batch_struct(tensors, is_device):
        fr = (capi.Frame * len(tensors))()
        for i, t in enumerate(tensors):
            h, w = t.shape
            fr[i].gray, fr[i].w, fr[i].h, fr[i].pitch = t.data_ptr(), w, h, w
            fr[i].is_device, fr[i].frame_id = int(is_device), i
            fr[i].out = C.cast(outs[i], C.POINTER(capi.Marker))
            fr[i].cap = cap
        return fr

    fr_dev = batch_struct(d_frames, True)
    fr_host = batch_struct(h_frames, False)
    # wave size and identification layout for this GPU and workload
    tune = autotune(det, fr_dev)

    def step_batch(fr):
        def run(i):
            det._check(det._lib.cctagb_detect_batch(det._h, fr, len(fr)), "detect_batch")
            return fr
        return run

    out1 = (capi.Marker * cap)()

    def step_device(i):
        t = d_frames[i % len(d_frames)]
        return det1.detect_device(t.data_ptr(), W, H, W, frame_id=i)

    def step_host(i):
        t = h_frames[i % len(h_frames)]
        n = C.c_int()
        st = capi.Stats()
        det1._check(det1._lib.cctagb_detect(det1._h, C.c_void_p(t.data_ptr()), W, H, W, i, out1, cap, C.byref(n),
                                            C.byref(st)), "detect")
        return [out1[k] for k in range(n.value)], st

    def timed(step_fn, steps, stream=stream):
        total = 0.0
        last = None
        per = []
        for i in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            last = step_fn(i)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            per.append(ms)
            total += ms
        return total, last, per

    for i in range(args.warmup):
        step_batch(fr_dev)(i)
        step_batch(fr_host)(i)
        step_device(i)
        step_host(i)
    torch.cuda.synchronize()
    barrier(world)
    n_plain = max(args.steps, BATCH)
    with ClockSampler(local) as clk:
        ms_dev, fr_last, _ = timed(step_batch(fr_dev), args.steps)
        torch.cuda.synchronize()
        barrier(world)
        ms_e2e, fr_last_h, _ = timed(step_batch(fr_host), args.steps)
        torch.cuda.synchronize()
        barrier(world)
        ms_plain, (markers, stats), per_plain = timed(step_device, n_plain, stream1)
        ms_plain_h, (_, stats_h), _ = timed(step_host, n_plain, stream1)
    torch.cuda.synchronize()
    barrier(world)
    ms_dev = max_over_ranks(ms_dev, world)
    ms_e2e = max_over_ranks(ms_e2e, world)
    ms_plain = max_over_ranks(ms_plain, world)
    ms_plain_h = max_over_ranks(ms_plain_h, world)
    batch_frame_ms = [fr_last[i].stats.ms_total for i in range(BATCH)]
    launches_batch = sum(fr_last[i].stats.kernel_launches for i in range(BATCH))
    launches_batch_h = sum(fr_last_h[i].stats.kernel_launches for i in range(BATCH))
    h2d = sum(fr_last_h[i].stats.h2d_bytes for i in range(BATCH))
    d2h = sum(fr_last_h[i].stats.d2h_bytes for i in range(BATCH))
    # Batched and single-frame paths return the same markers for a frame.
    same = all(
        [(m.id, m.status, m.x, m.y) for m in det1.detect(frames[i])[0]]
        == [(outs[i][k].id, outs[i][k].status, outs[i][k].x, outs[i][k].y) for k in range(fr_last_h[i].n_out)]
        for i in range(min(4, BATCH)))

    # Per-stage device times of the batched image stage with the step's 16
    # frames in one wave (one launch per kernel over all of them; events
    # between the kernels, eager, nothing else running), separate pass.
    pt = cctag_b200.default_params(3)
    pt.batchWaveFrames = BATCH
    det_t = cctag_b200.Detector(pt, max_w=W, max_h=H, max_batch=BATCH)
    det_t.set_stage_timing(True)
    bacc = {}
    for i in range(max(3, min(args.steps, 10))):
        flush.zero_()
        torch.cuda.synchronize()
        det_t._check(det_t._lib.cctagb_detect_batch(det_t._h, fr_dev, BATCH), "detect_batch")
        for k, v in det_t.stage_times().items():
            bacc.setdefault(k, []).append(v)
    det_t.close()
    batch_stage_ms = {k: statistics.median(v) for k, v in bacc.items()}
    # per-frame edge points, seeds and votes of the batch's frames
    bE, bS, bV, blevels = [], [], [], []
    for i in range(BATCH):
        _, st_i = step_device(i)
        blevels.append([det1.level_size(l) for l in range(4)])
        bE.append([st_i.edge_points[l] for l in range(4)])
        bS.append([st_i.seeds[l] for l in range(4)])
        bV.append([int(len(det1.votes(l)["vlist"])) for l in range(4)])
    # Per-stage device times of one frame's image stage and the
    # identification kernel (single-frame path), separate pass.
    det1.set_stage_timing(True)
    acc = {}
    id_ms, host_ms, dl_ms, cut_ms = [], [], [], []
    for i in range(max(3, min(args.steps, 20))):
        flush.zero_()
        torch.cuda.synchronize()
        _, st = step_device(i)
        for k, v in det1.stage_times().items():
            acc.setdefault(k, []).append(v)
        id_ms.append(st.ms_identify)
        host_ms.append(st.ms_host_candidates)
        dl_ms.append(st.ms_download)
        cut_ms.append(st.ms_cut_selection)
    det1.set_stage_timing(False)
    stage_ms = {k: statistics.median(v) for k, v in acc.items()}

    levels = [det1.level_size(l) for l in range(4)]
    E = [stats.edge_points[l] for l in range(4)]
    S = [stats.seeds[l] for l in range(4)]
    V = [int(len(det1.votes(l)["vlist"])) for l in range(4)]
    sb = stage_bytes(levels, E, S, V)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    def stage_table(ms_by, bytes_by):
        return {k: {"ms": round(ms_by[k], 5), "bytes": bytes_by[k],
                    "GB_s": round(bytes_by[k] / (ms_by[k] * 1e-3) / 1e9, 1) if ms_by[k] > 0 else None,
                    "frac_of_measured_hbm": round(bytes_by[k] / (ms_by[k] * 1e-3) / 1e9 / peak, 4)
                    if ms_by[k] > 0 else None}
                for k in bytes_by}

    # algorithmic bytes of the batched launch: the sum over its frames
    bsb = {}
    for i in range(BATCH):
        for k, v in stage_bytes(blevels[i], bE[i], bS[i], bV[i]).items():
            bsb[k] = bsb.get(k, 0) + v
    stages = stage_table(batch_stage_ms, bsb)
    stages_single = stage_table(stage_ms, sb)
    n_ident = sum(1 for m in markers if m.status in (1, -4))
    idm = statistics.median(id_ms)
    stages_single["identify"] = {"ms": round(idm, 5), "markers": n_ident, "bound": "fp32 SIMT + L2 gathers",
                          "GFLOP_s": round(ident_flops(n_ident) / (idm * 1e-3) / 1e9, 1) if idm > 0 else None}
    stages_single["host_candidates"] = {"ms": round(statistics.median(host_ms), 4), "where": "host CPU (C++), includes the "
                                 "edge-point download"}
    stages_single["download"] = {"ms": round(statistics.median(dl_ms), 4), "where": "D2H of the edge-point collections"}
    stages_single["host_cut_setup"] = {"ms": round(statistics.median(cut_ms), 4), "where": "host CPU (C++): outer points and tasks staged for upload; the angular sort, subsampling and cut selection run on the GPU just before identification"}
    # Roofline object for the dominant HBM-class kernel group of the batched
    # image stage (one launch over the step's 16 frames).
    top = max(batch_stage_ms, key=lambda k: batch_stage_ms[k])
    traffic = profiled_traffic(args.config).get(top)
    ach = bsb[top] / (batch_stage_ms[top] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": top, "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": traffic, "peak_source": peak_src,
                "launch": f"one launch per kernel over the image stages of the {BATCH} frames of a step",
                "note": "achieved = algorithmic bytes of the launch / its CUDA-event time, frac of measured"}

    c3 = run_c3(args, flush, torch, peak, peak_src) if rank == 0 and not args.no_c3 else None
    c4 = run_c4(args, flush, torch) if rank == 0 and not args.no_c4 else None
    c5 = run_c5(args, torch) if rank == 0 and not args.no_c5 else None

    fps_dev = world * args.steps * BATCH / (ms_dev * 1e-3)
    fps_e2e = world * args.steps * BATCH / (ms_e2e * 1e-3)
    found = sorted(m.id for m in markers if m.status == 1)
    line = {
        "metric": METRIC, "value": round(fps_dev, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_dev / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8/i16/f32", "data": "synthetic",
        "config": {"workload": f"{args.config}: full detection (pyramid .. identification, 3 crowns) of a batch "
                               f"of {BATCH} frames per step through cctagb_detect_batch",
                   "frame": f"{W}x{H}", "frames_per_step": BATCH, "detection_slots": SLOTS,
                   "host_threads": os.cpu_count(), "levels": levels, "edge_points": E,
                   "seeds": S, "markers_reliable": len(found), "candidates": stats.candidates,
                   "l2": "flushed between steps (256 MiB write, untimed)", "parallelism": f"replicas x{world}",
                   "batch_frame_p50_ms": round(statistics.median(batch_frame_ms), 3),
                   "batch_frame_p99_ms": round(float(np.percentile(batch_frame_ms, 99)), 3),
                   "batched_equals_single": bool(same),
                   "batch_config": {"batchWaveFrames": tune["batchWaveFrames"],
                                    "identLayout": ["auto", "block"][tune["identLayout"]],
                                    "hostThreads": tune["hostThreads"] or "default"}},
        "autotune": tune,
        "e2e": {"value": round(fps_e2e, 2), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "plain": {"value": round(world * n_plain / (ms_plain * 1e-3), 2),
                  "e2e": round(world * n_plain / (ms_plain_h * 1e-3), 2), "unit": UNIT,
                  "p50_ms": round(statistics.median(per_plain), 3),
                  "p99_ms": round(float(np.percentile(per_plain, 99)), 3),
                  "note": "one frame per call (cctagb_detect_device / cctagb_detect)"},
        "stages": stages,
        "stages_single_frame": stages_single,
        "roofline": roofline,
        "gpu_launches": int(launches_batch + launches_batch_h) * args.steps
                        + int(stats.kernel_launches + stats_h.kernel_launches) * n_plain,
        "clocks": clk.summary(),
    }
    if c3 is not None:
        line["c3_clutter"] = c3
    if c4 is not None:
        line["c4_cameras"] = c4
    if c5 is not None:
        line["c5_refine"] = c5
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(frames[:2], budget_s=args.cpu_budget, threads=1)
    det.close()
    det1.close()
    return line


def run_batch_only(args, torch, local):
    """The step's 16 frames through cctagb_detect_batch in one wave (one
    batched image-stage launch per kernel), `steps` times, for profiling."""
    import cctag_b200
    from cctag_b200 import capi

    frames = make_frames(args.config)
    H, W = frames[0].shape
    p = cctag_b200.default_params(3)
    p.batchWaveFrames = BATCH
    det = cctag_b200.Detector(p, max_w=W, max_h=H, max_batch=BATCH)
    d = [torch.from_numpy(f).to(f"cuda:{local}") for f in frames]
    cap = 512
    outs = [(capi.Marker * cap)() for _ in frames]
    fr = (capi.Frame * len(frames))()
    for i, t in enumerate(d):
        fr[i].gray, fr[i].w, fr[i].h, fr[i].pitch, fr[i].is_device, fr[i].frame_id = t.data_ptr(), W, H, W, 1, i
        fr[i].out = C.cast(outs[i], C.POINTER(capi.Marker))
        fr[i].cap = cap
    for _ in range(args.warmup + args.steps):
        det._check(det._lib.cctagb_detect_batch(det._h, fr, len(frames)), "detect_batch")
    torch.cuda.synchronize()
    det.close()
    return {"frames_per_call": len(frames), "calls": args.warmup + args.steps, "frame": f"{W}x{H}"}


def run_plain(args, torch, local):
    """Single-frame detections of the configuration's frames, one per call
    (cctagb_detect_device), for profiling one frame's kernels."""
    import cctag_b200

    frames = make_frames(args.config, n=max(1, min(args.steps, N_FRAMES)))
    H, W = frames[0].shape
    det = cctag_b200.Detector(max_w=W, max_h=H)
    d = [torch.from_numpy(f).to(f"cuda:{local}") for f in frames]
    for i in range(args.warmup):
        det.detect_device(d[i % len(d)].data_ptr(), W, H, W)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        det.detect_device(d[i % len(d)].data_ptr(), W, H, W)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    det.close()
    return {"frames": args.steps, "ms_per_frame_wall": round(dt * 1e3 / args.steps, 3), "frame": f"{W}x{H}"}


def run_c5(args, torch):
    """Candidate refinement (C5): 4096 distinct candidates (crops r 8-150 px,
    tilt <= 70 deg, noise sigma 2-12) in one device atlas, identified per call
    with the reference's grid refinement and with Gauss-Newton, their center
    error against the FP64 oracle (grid continued to 1e-4 px), the cost
    adjoint's rate, and the adjoint's accuracy (FP64 kernel against central
    differences of the FP64 oracle cost)."""
    import cctag_b200
    import oracle
    from cctag_b200 import capi
    from cctag_b200.synth import cut_task_from_marker, refine_atlas

    with host_pool() as pool:
        atlas, crops = refine_atlas(seed=0, n_crops=args.c5_candidates,
                                    map_fn=lambda f, j: pool.map(f, j, chunksize=32))
    tasks = [cut_task_from_marker(m, roi, local=True) for m, roi in crops]
    n_total = len(tasks)
    H, W = atlas.shape
    det = cctag_b200.Detector(max_w=640, max_h=480)
    stream = torch.cuda.ExternalStream(det.stream)
    d = torch.from_numpy(atlas).to(torch.device("cuda", torch.cuda.current_device()))
    arr = (capi.CutTask * n_total)(*tasks)
    out = (capi.IdentResult * n_total)()
    centers = np.array([[t.x0, t.y0] for t in tasks], np.float32)
    cost = np.zeros(n_total, np.float32)
    dcen = np.zeros((n_total, 2), np.float32)
    dh = np.zeros((n_total, 9), np.float32)

    def ident(mode):
        det._check(det._lib.cctagb_identify_tasks(det._h, C.c_void_p(d.data_ptr()), W, H, W, arr, n_total, mode, out),
                   "identify_tasks")
        return [(r.status, r.id, r.x, r.y, r.iterations) for r in out]

    def adjoint():
        det._check(det._lib.cctagb_cut_cost(det._h, C.c_void_p(d.data_ptr()), W, H, W, arr, n_total,
                                            capi.ptr(centers), capi.ptr(cost), capi.ptr(dcen), capi.ptr(dh)),
                   "cut_cost")

    def timed(fn, steps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            r = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps, r

    steps = max(3, min(args.steps, 10))
    ms_grid, res_grid = timed(lambda: ident(capi.REFINE_GRID), steps)
    ms_gn, res_gn = timed(lambda: ident(capi.REFINE_GAUSS_NEWTON), steps)
    ms_adj, _ = timed(adjoint, steps)

    # centers against the FP64 oracle, on every candidate
    dense = [oracle.refine_grid(atlas, t, 1e-4) for t in tasks]

    def errs(res):
        return [float(np.hypot(r[2] - q[0], r[3] - q[1])) for r, q in zip(res, dense) if r[0] == 1 and q is not None]

    def stats(v):
        return {"median_px": round(float(np.median(v)), 4), "p95_px": round(float(np.percentile(v, 95)), 4),
                "max_px": round(float(np.max(v)), 4), "over_0.02_px": int(sum(x > 0.02 for x in v)),
                "n": len(v)} if v else None

    egn_grid = [float(np.hypot(a[2] - b[2], a[3] - b[3])) for a, b in zip(res_grid, res_gn)
                if a[0] == 1 and b[0] == 1]
    # adjoint accuracy: the FP64 kernel's center gradient against central
    # differences (h = 1e-6 px) of the FP64 oracle cost, and the FP32 kernel's
    # against the FP64 kernel's, on the first 256 candidates off their start.
    # A difference quotient that straddles a kink of the bilinear image (its
    # two step sizes disagree) is no derivative and is counted apart, as in
    # the GPU test.
    nb = min(256, n_total)
    cen = centers[:nb] + np.float32([0.6, -0.4])
    c64, g64, h64 = det.cut_cost(d.data_ptr(), W, H, W, tasks[:nb], cen, fp64=True)
    c32, g32, h32 = det.cut_cost(d.data_ptr(), W, H, W, tasks[:nb], cen)
    rel_fd, rel_32, kinks = [], [], 0
    for i, t in enumerate(tasks[:nb]):
        x, y = float(cen[i, 0]), float(cen[i, 1])
        fds = []
        for h in (1e-6, 2e-6):
            fd = []
            for ddx, ddy in ((h, 0.0), (0.0, h)):
                a = oracle.cut_cost(atlas, t, x + ddx, y + ddy)[0]
                b = oracle.cut_cost(atlas, t, x - ddx, y - ddy)[0]
                fd.append(None if a is None or b is None else (a - b) / (2 * h))
            fds.append(fd)
        if any(None in fd for fd in fds) or c64[i] >= np.finfo(np.float32).max:
            continue
        f1, f2 = np.array(fds[0]), np.array(fds[1])
        if np.linalg.norm(f1 - f2) > 1e-6 * np.linalg.norm(f1):
            kinks += 1
            continue
        rel_fd.append(float(np.linalg.norm(g64[i] - f1) / np.linalg.norm(f1)))
        rel_32.append(float(np.linalg.norm(g32[i] - g64[i]) / np.linalg.norm(g64[i])))
    det.close()

    ok_grid = sum(1 for r in res_grid if r[0] == 1)
    ok_gn = sum(1 for r in res_gn if r[0] == 1)
    same_id = sum(1 for a, b in zip(res_grid, res_gn) if a[0] == 1 and b[0] == 1 and a[1] == b[1])
    return {
        "candidates_per_call": n_total, "distinct": n_total, "atlas": f"{W}x{H}",
        "grid": {"candidates_per_s": round(n_total / (ms_grid * 1e-3), 1), "ms_per_call": round(ms_grid, 3),
                 "identified": ok_grid, "vs_fp64_oracle": stats(errs(res_grid)),
                 "mean_rounds": round(float(np.mean([r[4] for r in res_grid])), 2)},
        "gauss_newton": {"candidates_per_s": round(n_total / (ms_gn * 1e-3), 1), "ms_per_call": round(ms_gn, 3),
                         "identified": ok_gn, "vs_fp64_oracle": stats(errs(res_gn)), "vs_grid": stats(egn_grid),
                         "same_id_as_grid": same_id,
                         "mean_evaluations": round(float(np.mean([r[4] for r in res_gn])), 2)},
        "adjoint": {"candidates_per_s": round(n_total / (ms_adj * 1e-3), 1), "ms_per_call": round(ms_adj, 3),
                    "note": "cctagb_cut_cost: cost + d/dcenter + d/dH per candidate (FP32)",
                    "fp64_kernel_vs_central_differences": {
                        "median_rel": float(f"{np.median(rel_fd):.3g}"), "max_rel": float(f"{np.max(rel_fd):.3g}"),
                        "n": len(rel_fd), "h_px": 1e-6, "straddling_a_kink": kinks},
                    "fp32_kernel_vs_fp64_kernel": {"median_rel": float(f"{np.median(rel_32):.3g}"),
                                                   "max_rel": float(f"{np.max(rel_32):.3g}")}},
        "speedup_gn_vs_grid": round(ms_grid / ms_gn, 2),
        "note": "cctagb_identify_tasks on one device atlas of distinct rendered crops; tasks from the rendered "
                "outer ellipses (22 cuts), started at the ellipse center",
    }


def _c3_frame(seed):
    from cctag_b200.synth import config_frame

    return config_frame("c3_4k_clutter", seed=seed).image


def run_c3(args, flush, torch, peak, peak_src):
    """4K clutter (C3): 3840x2160 frames with 30 markers, 200 distractor
    ellipses, 300 line segments and a band-limited background texture (about
    1.7 M Canny edge points, 1.2 M on level 0).  Frames/s of a
    4-frame batch per call, the edge points and votes, per-stage GB/s and the
    roofline of the dominant image-stage kernel group, and the CPU baseline."""
    import cctag_b200
    from cctag_b200 import capi

    seeds = [300, 301, 302, 303]
    with host_pool() as pool:
        frames = list(pool.map(_c3_frame, seeds))
    H, W = frames[0].shape
    det = cctag_b200.Detector(max_w=W, max_h=H, max_batch=SLOTS)
    stream = torch.cuda.ExternalStream(det.stream)
    dev = torch.device("cuda", torch.cuda.current_device())
    d = [torch.from_numpy(f).to(dev) for f in frames]
    cap = 512
    outs = [(capi.Marker * cap)() for _ in frames]
    fr = (capi.Frame * len(frames))()
    for i, t in enumerate(d):
        fr[i].gray, fr[i].w, fr[i].h, fr[i].pitch, fr[i].is_device, fr[i].frame_id = t.data_ptr(), W, H, W, 1, i
        fr[i].out = C.cast(outs[i], C.POINTER(capi.Marker))
        fr[i].cap = cap
    tune = autotune(det, fr, reps=3)
    for _ in range(args.warmup):
        det._check(det._lib.cctagb_detect_batch(det._h, fr, len(frames)), "detect_batch")
    steps = max(5, min(args.steps, 20))
    total = 0.0
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        det._check(det._lib.cctagb_detect_batch(det._h, fr, len(frames)), "detect_batch")
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    fps = steps * len(frames) / (total * 1e-3)
    # per-stage device times of one frame's image stage (separate eager pass)
    det.set_stage_timing(True)
    acc = {}
    for i in range(max(3, min(args.steps, 10))):
        flush.zero_()
        torch.cuda.synchronize()
        _, st = det.detect_device(d[i % len(d)].data_ptr(), W, H, W)
        for k, v in det.stage_times().items():
            acc.setdefault(k, []).append(v)
    det.set_stage_timing(False)
    _, st = det.detect_device(d[0].data_ptr(), W, H, W)
    levels = [det.level_size(l) for l in range(4)]
    E = [st.edge_points[l] for l in range(4)]
    S = [st.seeds[l] for l in range(4)]
    V = [int(len(det.votes(l)["vlist"])) for l in range(4)]
    det.close()
    stage_ms = {k: statistics.median(v) for k, v in acc.items()}
    sb = stage_bytes(levels, E, S, V)
    stages = {k: {"ms": round(stage_ms[k], 5), "bytes": sb[k],
                  "GB_s": round(sb[k] / (stage_ms[k] * 1e-3) / 1e9, 1) if stage_ms[k] > 0 else None}
              for k in sb}
    top = max(stage_ms, key=lambda k: stage_ms[k])
    ach = sb[top] / (stage_ms[top] * 1e-3) / 1e9
    out = {"value": round(fps, 2), "unit": UNIT, "steps": steps, "frames_per_step": len(frames),
           "frame": f"{W}x{H}", "edge_points": E, "votes": V, "seeds": S,
           "markers": int(sum(fr[i].n_out for i in range(len(frames)))),
           "image_stage_ms": round(sum(stage_ms.values()), 4), "stages": stages,
           "roofline": {"bound": "hbm", "kernel": top, "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(ach / peak, 4), "peak_source": peak_src},
           "autotune": tune,
           "note": "cctagb_detect_batch of 4 distinct frames per call, frames in device memory; stages of one "
                   "frame's image stage (single-frame launch)"}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(frames[:2], budget_s=min(args.cpu_budget, 10.0), threads=1)
    return out


def run_c4(args, flush, torch):
    """Multi-camera step: 16 frames of mixed resolution per call, 1,000 timed
    steps (per-frame p50 / p99 over all of their frames)."""
    import cctag_b200
    from cctag_b200 import capi
    from cctag_b200.synth import camera_batch

    with host_pool() as pool:
        batches = [[f.image for f in camera_batch(seed=s, n=BATCH, map_fn=pool.map)] for s in range(2)]
    det = cctag_b200.Detector(max_w=3840, max_h=2160, max_batch=SLOTS)
    stream = torch.cuda.ExternalStream(det.stream)
    dev = torch.device("cuda", torch.cuda.current_device())
    cap = 512
    dev_batches, frs, outs = [], [], []
    for cams in batches:
        d = [torch.from_numpy(c).to(dev) for c in cams]
        o = [(capi.Marker * cap)() for _ in cams]
        fr = (capi.Frame * len(cams))()
        for i, t in enumerate(d):
            h, w = t.shape
            fr[i].gray, fr[i].w, fr[i].h, fr[i].pitch, fr[i].is_device, fr[i].frame_id = t.data_ptr(), w, h, w, 1, i
            fr[i].out = C.cast(o[i], C.POINTER(capi.Marker))
            fr[i].cap = cap
        dev_batches.append(d)
        frs.append(fr)
        outs.append(o)
    tune = autotune(det, frs[0])
    for k in range(args.warmup):
        for fr in frs:
            det._check(det._lib.cctagb_detect_batch(det._h, fr, BATCH), "detect_batch")
    steps = max(1000, args.steps)  # the multi-camera workload's 1,000 steps after warm-up
    total, per_frame, markers = 0.0, [], 0
    for k in range(steps):
        fr = frs[k % len(frs)]
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        det._check(det._lib.cctagb_detect_batch(det._h, fr, BATCH), "detect_batch")
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
        per_frame += [fr[i].stats.ms_total for i in range(BATCH)]
        markers += int(sum(fr[i].n_out for i in range(BATCH)))
    det.close()
    sizes = sorted({f"{c.shape[1]}x{c.shape[0]}" for cams in batches for c in cams})
    return {"value": round(steps * BATCH / (total * 1e-3), 2), "unit": UNIT, "steps": steps,
            "frames_per_step": BATCH, "distinct_frames": BATCH * len(batches), "resolutions": sizes,
            "markers_per_step": round(markers / steps, 1),
            "frame_p50_ms": round(statistics.median(per_frame), 3),
            "frame_p99_ms": round(float(np.percentile(per_frame, 99)), 3),
            "autotune": tune,
            "note": "cctagb_detect_batch, frames in device memory; per-frame latency = host wall time of the "
                    "frame's detection inside the batch"}


# ------------------------------------------------------ CPU (oracle) legs --
def oracle_frame(img):
    """The reference CPU path (C++ restatement): whole detection of one frame."""
    import oracle

    return oracle.detect(img)


def cpu_baseline(frames, budget_s=15.0, threads=1):
    import oracle

    oracle.load()
    oracle_frame(frames[0])  # warm
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < budget_s or n < 1:
        oracle_frame(frames[n % len(frames)])
        n += 1
    dt = time.perf_counter() - t0
    return {"value": round(n / dt, 3), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} frames of the same workload in {dt:.1f} s on 1 core (whole detection: C++ "
                      f"restatement of the reference CPU path)"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    frames = make_frames(args.config)
    threads = os.cpu_count() or 1
    import oracle

    oracle.load()
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(threads) as ex:
        for i in range(args.warmup):
            list(ex.map(oracle_frame, frames[:BATCH]))
        t0 = time.perf_counter()
        for s in range(args.steps):
            list(ex.map(oracle_frame, frames[:BATCH]))
        dt = time.perf_counter() - t0
    fps = args.steps * BATCH / dt
    H, W = frames[0].shape
    return {
        "impl": "reference", "metric": METRIC, "value": round(fps, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/i16/f32",
        "data": "synthetic",
        "config": {"workload": f"{args.config}: full detection (pyramid .. identification, 3 crowns) of a batch "
                               f"of {BATCH} frames per step", "frame": f"{W}x{H}", "frames_per_step": BATCH},
        "cpu_baseline": {"value": round(fps, 3), "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{BATCH} frames per step spread over {threads} host threads, one frame per "
                                   "thread at a time (C++ restatement of the reference CPU path; the reference "
                                   "itself cannot be built here)"},
        "e2e": {"value": round(fps, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="c2_1080p")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-c4", action="store_true", help="skip the multi-camera (mixed resolution) leg")
    ap.add_argument("--no-c5", action="store_true", help="skip the candidate-refinement leg")
    ap.add_argument("--no-c3", action="store_true", help="skip the 4K clutter leg")
    ap.add_argument("--c5-candidates", type=int, default=4096, help="distinct candidates of the refinement leg")
    ap.add_argument("--leg", default="all", choices=["all", "plain", "batch", "c3", "c4", "c5"],
                    help="run one secondary leg alone and print its object (for profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line))
        return
    rank, world, local = dist_setup()
    if args.leg != "all":
        import torch

        torch.cuda.set_device(local)
        if args.leg == "c5":
            print(json.dumps({"c5_refine": run_c5(args, torch)}))
        elif args.leg == "plain":
            print(json.dumps({"plain": run_plain(args, torch, local)}))
        elif args.leg == "batch":
            print(json.dumps({"batch": run_batch_only(args, torch, local)}))
        elif args.leg == "c3":
            flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
            peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) \
                if (ROOT / "MEASURED_PEAKS.json").exists() else {}
            print(json.dumps({"c3_clutter": run_c3(args, flush, torch, peaks.get("hbm_gbs", 6650.0),
                                                   "measured" if "hbm_gbs" in peaks else "fallback")}))
        else:
            flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
            print(json.dumps({"c4_cameras": run_c4(args, flush, torch)}))
        return
    line = run_b200(args, rank, world, local)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
