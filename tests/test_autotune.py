"""CPU tests of the batch autotuner's cache (cctagb_tune_key / _cache_get /
_cache_put): keys, round trips, entries kept across writes, malformed and
foreign files, and a GPU test that cctagb_autotune measures once, then reads
its choice back from the cache, and that the identification layout it picks
does not change any marker."""
import json

import pytest

import cctag_b200
from cctag_b200 import capi


def test_key_names_gpu_size_frames_and_crowns(built_library):
    k = cctag_b200.tune_key("NVIDIA B200", 148, 1920, 1080, 16, 3)
    assert k == "NVIDIA B200|sm148|1920x1080|f16|c3"
    # separators and quotes in a device name cannot break the key or the file
    assert cctag_b200.tune_key('a|b"c', 1, 2, 3, 4, 5) == "a_b_c|sm1|2x3|f4|c5"


def test_put_then_get_round_trip(built_library, tmp_path):
    f = tmp_path / "tune.json"
    assert cctag_b200.tune_cache_get(f, "k1") is None  # no file yet
    cctag_b200.tune_cache_put(f, "k1", 8, capi.IDENT_BLOCK, 0.625)
    got = cctag_b200.tune_cache_get(f, "k1")
    assert got["batchWaveFrames"] == 8 and got["identLayout"] == capi.IDENT_BLOCK
    assert got["from_cache"] and abs(got["ms_per_frame"] - 0.625) < 1e-6
    doc = json.loads(f.read_text())
    assert doc["version"] == 2 and doc["entries"]["k1"]["batchWaveFrames"] == 8
    assert doc["entries"]["k1"]["hostThreads"] == 0


def test_other_entries_are_kept_and_replaced_in_place(built_library, tmp_path):
    f = tmp_path / "tune.json"
    cctag_b200.tune_cache_put(f, "gpu|sm148|1920x1080|f16|c3", 4, capi.IDENT_AUTO, 0.8)
    cctag_b200.tune_cache_put(f, "gpu|sm148|3840x2160|f4|c3", 2, capi.IDENT_BLOCK, 3.1)
    cctag_b200.tune_cache_put(f, "gpu|sm148|1920x1080|f16|c3", 16, capi.IDENT_BLOCK, 0.7)
    a = cctag_b200.tune_cache_get(f, "gpu|sm148|1920x1080|f16|c3")
    b = cctag_b200.tune_cache_get(f, "gpu|sm148|3840x2160|f4|c3")
    assert (a["batchWaveFrames"], a["identLayout"]) == (16, capi.IDENT_BLOCK)
    assert (b["batchWaveFrames"], b["identLayout"]) == (2, capi.IDENT_BLOCK)
    assert len(json.loads(f.read_text())["entries"]) == 2
    assert not list(tmp_path.glob("*.tmp.*"))  # the temporary file was renamed


@pytest.mark.parametrize("text", [
    "", "{", "[]",
    '{"version": 1, "entries": {"k": {"batchWaveFrames": 4, "identLayout": 0, "hostThreads": 0}}}',
    '{"version": 2, "entries": []}',
    '{"version": 2, "entries": {"k": {"batchWaveFrames": 0, "identLayout": 0, "hostThreads": 0}}}',
    '{"version": 2, "entries": {"k": {"batchWaveFrames": 17, "identLayout": 0, "hostThreads": 0}}}',
    '{"version": 2, "entries": {"k": {"batchWaveFrames": 4.5, "identLayout": 0, "hostThreads": 0}}}',
    '{"version": 2, "entries": {"k": {"batchWaveFrames": 4, "identLayout": 2, "hostThreads": 0}}}',
    '{"version": 2, "entries": {"k": {"batchWaveFrames": 4, "identLayout": 0, "hostThreads": 65}}}',
    '{"version": 2, "entries": {"k": {"batchWaveFrames": 4, "identLayout": 0}}}',
    '{"version": 2, "entries": {"k": {"batchWaveFrames": "4", "identLayout": 0, "hostThreads": 0}}}',
    '{"version": 2, "entries": {"k": {"identLayout": 0, "hostThreads": 0}}} trailing',
    "[" * 100 + "]" * 100,
])
def test_malformed_foreign_or_out_of_range_entries_are_misses(built_library, tmp_path, text):
    f = tmp_path / "tune.json"
    f.write_text(text)
    assert cctag_b200.tune_cache_get(f, "k") is None
    # a write over such a file starts a fresh cache
    cctag_b200.tune_cache_put(f, "k", 2, capi.IDENT_AUTO)
    assert cctag_b200.tune_cache_get(f, "k")["batchWaveFrames"] == 2


def test_escaped_keys_round_trip(built_library, tmp_path):
    f = tmp_path / "tune.json"
    key = 'odd "name" \\ with\ttab'
    cctag_b200.tune_cache_put(f, key, 4, capi.IDENT_BLOCK)
    assert cctag_b200.tune_cache_get(f, key)["identLayout"] == capi.IDENT_BLOCK
    assert json.loads(f.read_text())["entries"][key]["batchWaveFrames"] == 4


def test_put_rejects_out_of_range_choices(built_library, tmp_path):
    f = tmp_path / "tune.json"
    for wave, layout, threads in ((0, 0, 0), (17, 0, 0), (4, 2, 0), (4, -1, 0), (4, 0, -1), (4, 0, 65)):
        with pytest.raises(cctag_b200.CCTagError):
            cctag_b200.tune_cache_put(f, "k", wave, layout, host_threads=threads)
    assert not f.exists()
    with pytest.raises(cctag_b200.CCTagError):
        cctag_b200.tune_cache_put(tmp_path / "no_such_dir" / "tune.json", "k", 4, 0)


@pytest.mark.gpu
def test_autotune_measures_then_reads_the_cache(built_library, tmp_path):
    from cctag_b200.synth import config_frame

    frames = [config_frame("small", seed=30 + i).image for i in range(4)]
    h, w = frames[0].shape
    f = tmp_path / "tune.json"
    with cctag_b200.Detector(max_w=w, max_h=h, max_batch=4) as det:
        want = [[(m.id, m.status, m.x, m.y) for m in r[0]] for r in det.detect_batch(frames)]
        first = det.autotune(frames, cache_path=f, reps=2)
        # waves 1, 2, 4 x two layouts, then pool sizes at the best of those
        assert not first["from_cache"] and 6 < len(first["tried"]) <= 9
        assert (first["batchWaveFrames"], first["identLayout"], first["hostThreads"]) in \
            {(t["batchWaveFrames"], t["identLayout"], t["hostThreads"]) for t in first["tried"]}
        assert det.params.batchWaveFrames == first["batchWaveFrames"]
        assert det.params.hostThreads == first["hostThreads"]
        got = [[(m.id, m.status, m.x, m.y) for m in r[0]] for r in det.detect_batch(frames)]
        assert got == want
    with cctag_b200.Detector(max_w=w, max_h=h, max_batch=4) as det:
        second = det.autotune(frames, cache_path=f)
        assert second["from_cache"] and second["tried"] == []
        assert (second["batchWaveFrames"], second["identLayout"], second["hostThreads"]) == \
            (first["batchWaveFrames"], first["identLayout"], first["hostThreads"])
        got = [[(m.id, m.status, m.x, m.y) for m in r[0]] for r in det.detect_batch(frames)]
        assert got == want


@pytest.mark.gpu
def test_block_layout_gives_the_same_markers(built_library):
    from cctag_b200.synth import config_frame

    img = config_frame("c1_720p", seed=3).image
    res = []
    for layout in (capi.IDENT_AUTO, capi.IDENT_BLOCK):
        p = cctag_b200.default_params(3)
        p.identLayout = layout
        with cctag_b200.Detector(p, max_w=img.shape[1], max_h=img.shape[0]) as det:
            ms, _ = det.detect(img)
            res.append([(m.id, m.status, m.x, m.y, tuple(m.homography)) for m in ms])
    assert res[0] == res[1] and len(res[0]) > 0
