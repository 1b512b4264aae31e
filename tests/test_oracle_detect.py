"""CPU tests of the oracle's whole detection (image stage, candidate stage,
identification) against the renderer's ground truth, and of its FP32
(reference arithmetic) against its FP64 centre refinement."""
import numpy as np
import pytest

from cctag_b200.synth import config_frame


@pytest.mark.parametrize("name,seed", [("small", 4), ("c1_720p", 1), ("c1_720p", 2)])
def test_oracle_detects_ids_and_centers(orc, name, seed):
    fr = config_frame(name, seed=seed)
    ms = orc.detect(fr.image)
    ok = [m for m in ms if m.status == 1]
    assert len(ok) == len(fr.markers)
    for g in fr.markers:
        d = [np.hypot(m.x - g.center[0], m.y - g.center[1]) for m in ok]
        j = int(np.argmin(d))
        assert ok[j].id == g.id
        assert d[j] < 0.5


def test_oracle_fp32_matches_fp64_refinement(orc):
    fr = config_frame("c1_720p", seed=3)
    a = orc.detect(fr.image)
    b = orc.detect(fr.image, fp64=True)
    assert [m.id for m in a] == [m.id for m in b]
    for m, n in zip(a, b):
        assert np.hypot(m.x - n.x, m.y - n.y) < 0.05


def test_clutter_frames_have_the_workload_edge_density(orc):
    """The 4K clutter workload's frames carry 1-3 M Canny edge points over the
    pyramid (its stated range), most of them on level 0."""
    img = config_frame("c3_4k_clutter", seed=300).image
    counts = [int((orc.level(lv)[2] != 0).sum()) for lv in orc.pyramid(img, 4)]
    assert 1_000_000 <= sum(counts) <= 3_000_000, counts
    assert counts[0] >= 1_000_000, counts
