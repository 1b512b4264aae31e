"""Loop 1 (edge linking from the seeds) and the outlier removal of loop 2 on
the GPU against the host restatement of the oracle, bit for bit: the same
candidates in the same loop-one order, the same children counts, the same
keep decisions and the same filtered children, on every pyramid level."""
import numpy as np
import pytest

from cctag_b200.synth import config_frame

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,seed", [("c1_720p", 1), ("c1_720p", 3), ("c2_1080p", 2), ("c2_1080p", 100),
                                       ("small", 4)])
def test_loop_two_inputs_match_oracle(detector, orc, name, seed):
    fr = config_frame(name, seed=seed)
    detector.detect(fr.image)
    kept = 0
    for level in range(4):
        g_seed, g_score, g_keep, g_flt = detector.level_loop_two(level)
        w_seed, w_score, w_keep, w_flt = orc.loop_two(fr.image, level)
        assert np.array_equal(g_seed, w_seed), (level, g_seed[:10], w_seed[:10])
        assert np.array_equal(g_score, w_score), level
        assert np.array_equal(g_keep, w_keep), level
        for i, (a, b) in enumerate(zip(g_flt, w_flt)):
            assert np.array_equal(a, b), (level, i, len(a), len(b))
        kept += int(g_keep.sum())
    assert kept > 0


def test_loop_two_inputs_blank_frame(detector):
    detector.detect(np.full((240, 320), 90, np.uint8))
    for level in range(4):
        seed, score, keep, flt = detector.level_loop_two(level)
        assert len(seed) == 0 and len(flt) == 0
