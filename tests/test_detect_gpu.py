"""End-to-end detection on the GPU: seeded synthetic frames with known marker
IDs and imaged centres (the renderer's ground truth)."""
import numpy as np
import pytest

import cctag_b200
from cctag_b200.synth import config_frame, render_frame

pytestmark = pytest.mark.gpu

CENTER_TOL_PX = 0.5   # vs the rendered ground truth (includes blur/quantisation bias)


def match(markers, truth):
    """Pair detected reliable markers with ground-truth markers by centre."""
    out = []
    for m in markers:
        if m.status != 1:
            continue
        d = [np.hypot(m.x - g.center[0], m.y - g.center[1]) for g in truth]
        j = int(np.argmin(d))
        out.append((m, truth[j], d[j]))
    return out


@pytest.mark.parametrize("name,seed", [("c1_720p", 1), ("c1_720p", 2), ("c1_720p", 3), ("small", 4)])
def test_detect_ids_and_centers(detector, name, seed):
    fr = config_frame(name, seed=seed)
    markers, stats = detector.detect(fr.image)
    pairs = match(markers, fr.markers)
    found = {id(g) for _, g, d in pairs if d < 3.0}
    assert len(found) >= max(1, len(fr.markers) - 1), (stats.candidates, [(m.id, m.status, m.x, m.y) for m in markers])
    for m, g, d in pairs:
        if d < 3.0:
            assert m.id == g.id, (m.id, g.id, d)
            assert d < CENTER_TOL_PX, d


def test_detect_1080p_runs(detector):
    fr = config_frame("c2_1080p", seed=1)
    markers, stats = detector.detect(fr.image)
    pairs = [(m, g, d) for m, g, d in match(markers, fr.markers) if d < 3.0]
    assert len(pairs) >= len(fr.markers) // 2
    assert all(m.id == g.id for m, g, _ in pairs)


def test_detect_blank_frame(detector):
    markers, stats = detector.detect(np.full((240, 320), 200, np.uint8))
    assert markers == [] and stats.candidates == 0


def test_detect_is_deterministic(detector):
    fr = config_frame("c1_720p", seed=5)
    a, _ = detector.detect(fr.image)
    b, _ = detector.detect(fr.image)
    assert [(m.id, m.status, m.x, m.y) for m in a] == [(m.id, m.status, m.x, m.y) for m in b]
