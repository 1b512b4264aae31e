"""The reference's regression check between a log of this library's
detections and a log of the oracle's detections of the same frames (GPU)."""
import pytest

import oracle
from cctag_b200 import regression as rg
from cctag_b200.capi import default_params
from cctag_b200.synth import config_frame

pytestmark = pytest.mark.gpu


def test_library_log_passes_the_reference_checker_against_the_oracle(detector, tmp_path):
    frames = [config_frame("c1_720p", seed=s).image for s in (1, 2, 3)]
    params = default_params(3)
    ours = rg.detect_frames(detector, "c1_720p.avi", frames, params)
    ours.save(tmp_path / "test.xml")
    ref = rg.FileLog("c1_720p.avi", rg.parameters_of(params))
    for i, g in enumerate(frames):
        ref.frameLogs.append(rg.FrameLog(i, 0.0, [rg.DetectedTag(m.id, m.status, m.x, m.y, m.quality)
                                                   for m in oracle.detect(g, fp64=True)]))
    ref.save(tmp_path / "reference.xml")
    report = rg.compare(rg.FileLog.load(tmp_path / "reference.xml"), rg.FileLog.load(tmp_path / "test.xml"),
                        epsilon=0.05)
    assert report["elapsed_diff_mean"] > 0.0
