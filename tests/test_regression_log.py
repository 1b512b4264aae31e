"""Regression logs in the reference's Boost-XML FileLog layout (CPU)."""
import pytest

from cctag_b200 import regression as rg
from cctag_b200.capi import default_params


def _log(shift=0.0, quality=1.0):
    p = rg.parameters_of(default_params(3))
    tags = [rg.DetectedTag(3, 1, 10.5 + shift, 20.25, quality), rg.DetectedTag(7, 1, 100.0, 50.0, 2.0),
            rg.DetectedTag(-1, -3, 1.0, 2.0, 0.0)]
    return rg.FileLog("frames/cam0.png", p, [rg.FrameLog(0, 0.0125, tags), rg.FrameLog(1, 0.011, tags[:2])])


def test_archive_layout():
    x = _log().to_xml().splitlines()
    assert x[0].startswith('<?xml version="1.0"') and x[1] == "<!DOCTYPE boost_serialization>"
    assert x[2].startswith('<boost_serialization signature="serialization::archive"')
    assert x[3] == '<FileLog class_id="0" tracking_level="0" version="0">'
    body = "\n".join(x)
    # the Params.hpp serialize() order, first and last members
    assert body.index("<_cannyThrLow>0.01</_cannyThrLow>") < body.index("<_pinnedNearbyPoints>60</_pinnedNearbyPoints>")
    # class attributes only on the first element of each class
    assert body.count('class_id="3"') == 1 and body.count('class_id="5"') == 1
    assert "<count>2</count>" in body and "<item_version>0</item_version>" in body


def test_round_trip():
    a = _log()
    b = rg.FileLog.from_xml(a.to_xml())
    assert b.filename == a.filename and b.parameters == a.parameters
    assert [(f.frame, len(f.tags)) for f in b.frameLogs] == [(0, 3), (1, 2)]
    assert b.frameLogs[0].tags[0] == rg.DetectedTag(3, 1, 10.5, 20.25, 1.0)


def test_reader_accepts_archives_without_class_attributes():
    text = _log().to_xml()
    for attr in ('class_id="0" ', 'class_id="3" ', 'tracking_level="0" ', 'version="0"'):
        text = text.replace(attr, "")
    assert len(rg.FileLog.from_xml(text).frameLogs) == 2


def test_checker_rules():
    ref = _log()
    assert rg.compare(ref, _log(shift=0.4, quality=1.5), epsilon=0.5)["quality_diff_mean"] == pytest.approx(0.25)
    with pytest.raises(rg.CheckError, match="positions"):
        rg.compare(ref, _log(shift=0.6), epsilon=0.5)
    other = _log()
    other.frameLogs[0].tags[1] = rg.DetectedTag(8, 1, 100.0, 50.0, 2.0)
    with pytest.raises(rg.CheckError, match="IDs"):
        rg.compare(ref, other, epsilon=0.5)
    fewer = _log()
    fewer.frameLogs[0].tags.pop()
    with pytest.raises(rg.CheckError, match="# of tags"):
        rg.compare(ref, fewer, epsilon=0.5)
    dup = _log()
    dup.frameLogs[1].tags[1] = rg.DetectedTag(3, 1, 1.0, 1.0, 1.0)
    with pytest.raises(rg.CheckError, match="duplicate"):
        rg.compare(ref, dup, epsilon=0.5)
