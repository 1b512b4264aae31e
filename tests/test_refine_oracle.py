"""FP64 oracle of the batched identification calls (CPU): its analytic
gradients against central differences, its scale invariance, and the dense
grid refinement against the rendered ground truth."""
import numpy as np
import pytest

import oracle
from cctag_b200.synth import cut_task_from_marker, render_frame


@pytest.fixture(scope="module")
def scene():
    f = render_frame(640, 480, 2, (60, 100), 50, seed=11, noise_sigma=5.0)
    return f, [cut_task_from_marker(m, (0, 0, 640, 480)) for m in f.markers]


def _center_fd(img, t, cx, cy, h):
    f = lambda x, y: oracle.cut_cost(img, t, x, y)[0]
    return np.array([(f(cx + h, cy) - f(cx - h, cy)) / (2 * h), (f(cx, cy + h) - f(cx, cy - h)) / (2 * h)])


def test_center_gradient_matches_central_differences(scene):
    """d cost / d center against central differences.  The image is bilinear
    between pixel centres, so the cost has kinks where a sample crosses a
    pixel row or column: with h = 1e-5 px hardly any sample crosses one and
    every case agrees to 1e-6; with h = 1e-3 px some do, and the median
    relative error over the cases is held to 1e-4."""
    f, tasks = scene
    errs = []
    for t in tasks:
        for (dx, dy) in [(0.0, 0.0), (0.7, -0.4), (-0.3, 0.9), (1.5, 1.1)]:
            cx, cy = t.x0 + dx, t.y0 + dy
            cost, dc, _, _ = oracle.cut_cost(f.image, t, cx, cy)
            assert cost is not None
            fd5 = _center_fd(f.image, t, cx, cy, 1e-5)
            assert np.linalg.norm(fd5 - dc) <= 1e-6 * np.linalg.norm(dc), (fd5, dc)
            fd3 = _center_fd(f.image, t, cx, cy, 1e-3)
            errs.append(np.linalg.norm(fd3 - dc) / np.linalg.norm(dc))
    assert np.median(errs) <= 1e-4, errs


def test_homography_gradient_matches_central_differences(scene):
    """d cost / d H against central differences (step 1e-7 of each entry)."""
    f, tasks = scene
    for t in tasks:
        _, _, _, H = oracle.cut_cost(f.image, t, t.x0, t.y0)
        _, g = oracle.cut_cost_h(f.image, t, H)
        fd = np.zeros(9)
        for j in range(9):
            h = 1e-7 * max(abs(H[j]), 1e-3 * np.abs(H).max())
            e = np.zeros(9)
            e[j] = h
            fd[j] = (oracle.cut_cost_h(f.image, t, H + e)[0] - oracle.cut_cost_h(f.image, t, H - e)[0]) / (2 * h)
        assert np.linalg.norm(fd - g) <= 1e-6 * np.linalg.norm(g)


def test_homography_gradient_is_orthogonal_to_h(scene):
    """The cost does not change when H is scaled, so sum(G * H) = 0."""
    f, tasks = scene
    for t in tasks:
        _, _, g, H = oracle.cut_cost(f.image, t, t.x0 + 0.3, t.y0)
        assert abs(np.dot(g, H)) <= 1e-9 * np.linalg.norm(g) * np.linalg.norm(H)


def test_dense_refinement_near_truth(scene):
    """Grid refinement continued to 1e-4 px lands near the rendered center,
    and the reference's 0.02 px stop lands near the dense result."""
    f, tasks = scene
    for t, m in zip(tasks, f.markers):
        dense = oracle.refine_grid(f.image, t, 1e-4)
        coarse = oracle.refine_grid(f.image, t, 0.02)
        assert dense is not None and coarse is not None
        assert np.hypot(dense[0] - m.center[0], dense[1] - m.center[1]) < 0.1
        assert np.hypot(dense[0] - coarse[0], dense[1] - coarse[1]) < 0.05
        assert dense[2] <= coarse[2] + 1e-9
