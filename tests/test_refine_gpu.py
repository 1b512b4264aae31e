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
from cctag_b200.synth import config_frame, cut_task_from_marker, refine_atlas, render_frame

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


@pytest.fixture(scope="module")
def c5_crops():
    """64 crops of the candidate-refinement workload (r 8-150 px, tilt <= 70
    deg, noise sigma 2-12) in one atlas, as crop-local tasks."""
    atlas, crops = refine_atlas(seed=0, n_crops=64)
    return atlas, [cut_task_from_marker(m, roi, local=True) for m, roi in crops]


def test_fp64_adjoint_matches_central_differences(detector, c5_crops):
    """The adjoint of the cut sampling, evaluated in double precision on the
    GPU (cctagb_cut_cost_f64), against FP64 central differences of the FP64
    oracle cost: relative error <= 1e-4 on the center gradient, off the
    start on every crop.  Bilinear interpolation has kinks at pixel lines; a
    difference quotient that straddles one (its two step sizes disagree) is
    no derivative and is left out -- at most a few percent of the crops."""
    atlas, tasks = c5_crops
    H, W = atlas.shape
    d = to_device(atlas)
    cen = np.array([[t.x0 + 0.6, t.y0 - 0.4] for t in tasks], np.float32)
    cost, dc, dh = detector.cut_cost(d.data_ptr(), W, H, W, tasks, cen, fp64=True)
    checked = 0
    for i, t in enumerate(tasks):
        x, y = float(cen[i, 0]), float(cen[i, 1])
        want, _, wdh, _ = oracle.cut_cost(atlas, t, x, y)
        if want is None:
            continue
        assert abs(cost[i] - want) <= 1e-6 * want
        assert np.linalg.norm(dh[i] - wdh) <= 1e-6 * np.linalg.norm(wdh)
        fds = []
        for h in (1e-6, 2e-6):
            g = []
            for ex, ey in ((h, 0.0), (0.0, h)):
                a = oracle.cut_cost(atlas, t, x + ex, y + ey)[0]
                b = oracle.cut_cost(atlas, t, x - ex, y - ey)[0]
                g.append((a - b) / (2 * h))
            fds.append(np.array(g))
        if np.linalg.norm(fds[0] - fds[1]) > 1e-6 * np.linalg.norm(fds[0]):
            continue  # straddles a kink
        checked += 1
        assert np.linalg.norm(dc[i] - fds[0]) <= 1e-4 * np.linalg.norm(fds[0]), (i, dc[i], fds[0])
    assert checked >= 0.9 * len(tasks)


def test_gauss_newton_within_0_02_px_of_fp64_oracle(detector, c5_crops):
    """Gauss-Newton centers within 0.02 px of the FP64 grid refinement
    continued to 1e-4 px, with the grid's IDs, on the refinement workload's
    crops; and fewer cost evaluations than the grid's trials."""
    atlas, tasks = c5_crops
    H, W = atlas.shape
    d = to_device(atlas)
    grid = detector.identify_tasks(d.data_ptr(), W, H, W, tasks, capi.REFINE_GRID)
    gn = detector.identify_tasks(d.data_ptr(), W, H, W, tasks, capi.REFINE_GAUSS_NEWTON)
    n = 0
    for t, a, b in zip(tasks, grid, gn):
        assert a.status == b.status
        if b.status != 1:
            continue
        assert a.id == b.id
        dense = oracle.refine_grid(atlas, t, 1e-4)
        assert np.hypot(b.x - dense[0], b.y - dense[1]) <= 0.02
        n += 1
    assert n >= 0.85 * len(tasks)


def test_local_tasks_match_image_coordinates(detector, c5_crops):
    """Crop-local tasks give the results of the same tasks in image
    coordinates, moved by the crop corner: the same IDs, and centers within
    0.02 px (the FP32 inputs round differently at image coordinates of
    thousands of pixels, and the grid's discrete steps follow them)."""
    atlas, tasks = c5_crops
    H, W = atlas.shape
    d = to_device(atlas)
    moved = []
    for t in tasks:
        g = capi.CutTask.from_buffer_copy(t)
        ox, oy = t.roi[0], t.roi[1]
        T = np.array([[1, 0, -ox], [0, 1, -oy], [0, 0, 1.0]])
        Q = T.T @ np.array(t.Q[:], np.float64).reshape(3, 3) @ T
        Q = Q / np.abs(Q).max()
        for k in range(9):
            g.Q[k] = float(Q.flat[k])
        g.cx, g.cy, g.x0, g.y0 = t.cx + ox, t.cy + oy, t.x0 + ox, t.y0 + oy
        for c in range(t.ncuts):
            g.stop[c][0], g.stop[c][1] = t.stop[c][0] + ox, t.stop[c][1] + oy
        g.local = 0
        moved.append(g)
    a = detector.identify_tasks(d.data_ptr(), W, H, W, tasks, capi.REFINE_GRID)
    b = detector.identify_tasks(d.data_ptr(), W, H, W, moved, capi.REFINE_GRID)
    for t, p, q in zip(tasks, a, b):
        assert p.status == q.status and p.id == q.id
        if p.status == 1:
            assert np.hypot(p.x + t.roi[0] - q.x, p.y + t.roi[1] - q.y) <= 0.02


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
        assert np.hypot(b.x - dense[0], b.y - dense[1]) <= 0.02


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
