"""GPU ellipse growing (the candidates' growing half of completeFlowComponent,
Detection.cpp:190-267, and ellipseGrowing2, EllipseGrowing.cpp:459-551, in
k_grow) against the host code on the same frames: every marker field and
every selected cut end bit for bit, so the outer point lists (their order
included) and ellipses that leave the kernel are the host's."""
import numpy as np
import pytest

import cctag_b200
from cctag_b200.synth import camera_batch, config_frame, render_frame

pytestmark = pytest.mark.gpu


def _run(img, gpu):
    p = cctag_b200.default_params(3)
    p.gpuEllipseGrowing = int(gpu)
    with cctag_b200.Detector(p, max_w=img.shape[1], max_h=img.shape[0]) as det:
        markers, stats = det.detect(img)
        tasks = det.last_tasks()
    ms = [(m.id, m.status, m.pyramidLevel, np.float32(m.x).view(np.uint32), np.float32(m.y).view(np.uint32),
           np.array([m.outer.cx, m.outer.cy, m.outer.a, m.outer.b, m.outer.angle], np.float32).tobytes(),
           np.array(m.homography, np.float32).tobytes()) for m in markers]
    cuts = [np.array([[t.stop[k][0], t.stop[k][1]] for k in range(t.ncuts)], np.float32).tobytes() for t in tasks]
    return ms, cuts, stats


CASES = [("c1_720p", 1), ("c1_720p", 2), ("c1_720p", 3), ("c1_720p", 5), ("c2_1080p", 100), ("c2_1080p", 101),
         ("small", 4), ("small", 7), ("camera", 0), ("camera", 1), ("camera", 2), ("camera", 3), ("tilted", 9)]


def _frame(name, seed):
    if name == "camera":
        return camera_batch(seed=3, n=4)[seed].image
    if name == "tilted":
        return render_frame(1280, 720, 4, (40, 160), 70, seed=seed, noise_sigma=9.0).image
    return config_frame(name, seed=seed).image


@pytest.mark.parametrize("name,seed", CASES, ids=[f"{n}-{s}" for n, s in CASES])
def test_gpu_growing_equals_host(built_library, name, seed):
    img = _frame(name, seed)
    g_ms, g_cuts, g_stats = _run(img, True)
    h_ms, h_cuts, h_stats = _run(img, False)
    assert g_ms == h_ms
    assert g_cuts == h_cuts
    # every candidate grew on the GPU (none too large for the kernel)
    assert g_stats.grown_gpu > 0 and g_stats.grown_host == 0
    assert h_stats.grown_gpu == 0 and h_stats.grown_host == g_stats.grown_gpu


def test_candidates_over_the_capacity_grow_on_the_host(built_library):
    """With room for few outer points on the GPU, the larger candidates grow on
    the host and the rest on the GPU, with the host's results throughout."""
    img = config_frame("c1_720p", seed=2).image
    p = cctag_b200.default_params(3)
    p.gpuEllipseGrowing = 1
    p.gpuGrowMaxPoints = 120
    with cctag_b200.Detector(p, max_w=img.shape[1], max_h=img.shape[0]) as det:
        markers, stats = det.detect(img)
        got = [(m.id, m.status, m.x, m.y, m.outer.a) for m in markers]
    h_ms, _, h_stats = _run(img, False)
    assert got == [(m[0], m[1], np.uint32(m[3]).view(np.float32), np.uint32(m[4]).view(np.float32),
                    np.frombuffer(m[5], np.float32)[2]) for m in h_ms]
    assert stats.grown_gpu > 0 and stats.grown_host > 0
    assert stats.grown_gpu + stats.grown_host == h_stats.grown_host
