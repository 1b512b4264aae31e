"""Batched identification on the GPU (cctagb_identify_tasks, cctagb_cut_cost):
cost and adjoints against the FP64 oracle, the grid path against detection,
Gauss-Newton against the grid and the dense FP64 refinement, and candidate
rectangles inside a larger image."""
import ctypes as C

import numpy as np
import pytest

import cctag_b200
import oracle
from cctag_b200 import capi
from cctag_b200.synth import config_frame, cut_task_from_marker, render_frame

pytestmark = pytest.mark.gpu


def to_device(img):
    import torch

    return torch.from_numpy(np.ascontiguousarray(img)).cuda()


@pytest.fixture(scope="module")
def scene():
    f = render_frame(1280, 720, 4, (40, 120), 50, seed=21, noise_sigma=5.0)
    tasks = [cut_task_from_marker(m, (0, 0, 1280, 720)) for m in f.markers]
    return f, tasks


def test_cut_cost_matches_fp64_oracle(detector, scene):
    """Cost and both gradients within 1e-3 (relative; FP32 homography and
    sample positions against FP64, measured up to 3.3e-4) of the oracle, at
    the start and off-center."""
    f, tasks = scene
    d = to_device(f.image)
    for shift in [(0.0, 0.0), (0.8, -0.6)]:
        centers = np.array([[t.x0 + shift[0], t.y0 + shift[1]] for t in tasks], np.float32)
        cost, dc, dh = detector.cut_cost(d.data_ptr(), 1280, 720, 1280, tasks, centers)
        for i, t in enumerate(tasks):
            want, wdc, wdh, _ = oracle.cut_cost(f.image, t, float(centers[i, 0]), float(centers[i, 1]))
            assert want is not None
            assert abs(cost[i] - want) <= 1e-3 * want
            assert np.linalg.norm(dc[i] - wdc) <= 1e-3 * np.linalg.norm(wdc), (dc[i], wdc)
            assert np.linalg.norm(dh[i] - wdh) <= 1e-3 * np.linalg.norm(wdh), (dh[i], wdh)


def test_cut_cost_without_two_cuts_inside(detector, scene):
    f, tasks = scene
    t = tasks[0]
    small = capi.CutTask.from_buffer_copy(t)
    small.roi[0], small.roi[1], small.roi[2], small.roi[3] = int(t.cx) - 3, int(t.cy) - 3, 6, 6
    d = to_device(f.image)
    cost, dc, dh = detector.cut_cost(d.data_ptr(), 1280, 720, 1280, [small], np.array([[t.x0, t.y0]], np.float32))
    assert cost[0] == np.finfo(np.float32).max and not dc.any() and not dh.any()


def test_identify_tasks_grid_reproduces_detection(detector):
    """The detection's own tasks, run again through cctagb_identify_tasks on
    the same frame, give the detection's centers and IDs exactly."""
    fr = config_frame("c1_720p", seed=1)
    markers, _ = detector.detect(fr.image)
    tasks = detector.last_tasks()
    assert tasks
    d = to_device(fr.image)
    res = detector.identify_tasks(d.data_ptr(), 1280, 720, 1280, tasks, capi.REFINE_GRID)
    got = {(r.id, r.x, r.y) for r in res if r.status == 1}
    for m in markers:
        if m.status == 1:
            assert (m.id, m.x, m.y) in got


def test_gauss_newton_matches_grid_and_dense_oracle(detector, scene):
    """Gauss-Newton centers within 0.05 px of the grid's and of the FP64 grid
    continued to 1e-4 px; same IDs; fewer cost evaluations."""
    f, tasks = scene
    d = to_device(f.image)
    grid = detector.identify_tasks(d.data_ptr(), 1280, 720, 1280, tasks, capi.REFINE_GRID)
    gn = detector.identify_tasks(d.data_ptr(), 1280, 720, 1280, tasks, capi.REFINE_GAUSS_NEWTON)
    for t, m, a, b in zip(tasks, f.markers, grid, gn):
        assert a.status == 1 and b.status == 1
        assert a.id == b.id == m.id
        assert np.hypot(a.x - b.x, a.y - b.y) <= 0.05
        dense = oracle.refine_grid(f.image, t, 1e-4)
        assert np.hypot(b.x - dense[0], b.y - dense[1]) <= 0.05


def test_rectangles_inside_a_larger_image(detector, scene):
    """A frame pasted at an offset into a larger image (wider pitch), with the
    tasks moved and given the frame's rectangle, gives the same results."""
    f, tasks = scene
    ox, oy, W, H = 37, 53, 1400, 800
    big = np.full((H, W), 255, np.uint8)
    big[oy:oy + 720, ox:ox + 1280] = f.image
    moved = [cut_task_from_marker(m, (ox, oy, 1280, 720), offset=(ox, oy)) for m in f.markers]
    d0, d1 = to_device(f.image), to_device(big)
    a = detector.identify_tasks(d0.data_ptr(), 1280, 720, 1280, tasks, capi.REFINE_GRID)
    b = detector.identify_tasks(d1.data_ptr(), W, H, W, moved, capi.REFINE_GRID)
    for p, q in zip(a, b):
        assert p.status == q.status and p.id == q.id
        assert np.hypot(p.x + ox - q.x, p.y + oy - q.y) <= 2e-3


def test_task_outside_the_image_is_rejected(detector, scene):
    f, tasks = scene
    bad = capi.CutTask.from_buffer_copy(tasks[0])
    bad.roi[2] = 2000
    d = to_device(f.image)
    with pytest.raises(cctag_b200.CCTagError) as e:
        detector.identify_tasks(d.data_ptr(), 1280, 720, 1280, [bad], capi.REFINE_GRID)
    assert e.value.status == capi.BAD_ARG


@pytest.mark.parametrize("mode", [capi.REFINE_GRID, capi.REFINE_GAUSS_NEWTON])
def test_few_and_many_candidates_give_the_same_bits(detector, scene, mode):
    """A handful of candidates runs as clusters of blocks, thousands as one
    block each; both sum the same per-chunk terms in the same order."""
    f, tasks = scene
    d = to_device(f.image)
    few = detector.identify_tasks(d.data_ptr(), 1280, 720, 1280, tasks, mode)
    many = detector.identify_tasks(d.data_ptr(), 1280, 720, 1280, tasks * 64, mode)
    for i, a in enumerate(few):
        for b in many[i::len(tasks)]:
            assert (a.status, a.id, a.x, a.y, a.residual, a.iterations) == \
                (b.status, b.id, b.x, b.y, b.residual, b.iterations)
