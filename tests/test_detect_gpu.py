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


@pytest.mark.parametrize("name,seed", [("c1_720p", 1), ("c1_720p", 3), ("c2_1080p", 2)])
def test_detect_matches_oracle(detector, orc, name, seed):
    """Same markers as the CPU oracle (same image-stage inputs, same candidate
    stage): IDs and statuses exact; centres within 0.05 px of the oracle's FP64
    refinement."""
    fr = config_frame(name, seed=seed)
    got, _ = detector.detect(fr.image)
    want = orc.detect(fr.image, fp64=True)
    assert [(m.id, m.status, m.pyramidLevel) for m in got] == [(m.id, m.status, m.level) for m in want]
    for g, w in zip(got, want):
        assert abs(g.outer.cx - w.cx) < 1e-3 and abs(g.outer.a - w.a) < 1e-3
        if g.status == 1:
            assert np.hypot(g.x - w.x, g.y - w.y) <= 0.05, (g.x, g.y, w.x, w.y)


@pytest.mark.parametrize("name,seed", [("c1_720p", 1), ("c1_720p", 3), ("c2_1080p", 2), ("small", 4)])
def test_cut_selection_matches_oracle_bits(detector, orc, name, seed):
    """Cut collection, outer-edge refinement and uniform selection on the GPU
    (identify_step_1 after the angular sort) select the same cut ends as the
    oracle's restatement, bit for bit, for every candidate it keeps."""
    fr = config_frame(name, seed=seed)
    detector.detect(fr.image)
    tasks = detector.last_tasks()
    want = [stops for st, stops in orc.cut_selection(fr.image) if st == 1]
    assert len(tasks) == len(want) and len(want) > 0
    for t, w in zip(tasks, want):
        got = np.array([[t.stop[k][0], t.stop[k][1]] for k in range(t.ncuts)], np.float32).reshape(-1, 2)
        assert got.shape == w.shape, (got.shape, w.shape)
        assert np.array_equal(got.view(np.uint32), w.view(np.uint32)), np.abs(got - w).max()


def test_cpp_shim_example_runs(built_library, tmp_path):
    """The C++ drop-in example (reference-style cctagDetection) finds the
    markers of a rendered frame."""
    import subprocess
    import sys

    sys.path.insert(0, str(__import__("pathlib").Path(__file__).parent))
    from test_capi import build_shim_example

    fr = config_frame("c1_720p", seed=2)
    raw = tmp_path / "frame.raw"
    raw.write_bytes(np.array(fr.image.shape[::-1], np.int32).tobytes() + fr.image.tobytes())
    exe = build_shim_example(built_library, tmp_path)
    r = subprocess.run([str(exe), str(raw)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    rows = [l.split() for l in r.stdout.strip().splitlines()]
    ids = sorted(int(x[0]) for x in rows if int(x[1]) == 1)
    assert ids == sorted(g.id for g in fr.markers)


def _key(markers):
    return [(m.id, m.status, m.x, m.y, m.outer.a, m.outer.b) for m in markers]


def test_detect_batch_matches_single_frames(built_library, detector):
    """Every frame of a mixed-resolution batch gives exactly what a single
    detect of that frame gives, whatever slot ran it."""
    from cctag_b200.synth import CAMERA_SIZES, render_frame
    frames = []
    for i, (w, h) in enumerate(CAMERA_SIZES[:3] * 2):
        frames.append(render_frame(w, h, 3 + i, (15.0, min(w, h) / 5.0), 50, seed=300 + i, noise_sigma=5.0).image)
    with cctag_b200.Detector(max_w=1920, max_h=1080, max_batch=4) as bd:
        got = bd.detect_batch(frames)
        again = bd.detect_batch(frames[::-1])[::-1]
    # two slots for six frames: each slot runs three in turn, and a single
    # call afterwards is unaffected
    with cctag_b200.Detector(max_w=1920, max_h=1080, max_batch=2) as bd2:
        turns = bd2.detect_batch(frames)
        after, _ = bd2.detect(frames[0])
    for f, (m, st), (m2, _), (m3, _) in zip(frames, got, again, turns):
        want, _ = detector.detect(f)
        assert _key(m) == _key(want)
        assert _key(m2) == _key(want)
        assert _key(m3) == _key(want)
        assert st.markers == len(m)
    assert _key(after) == _key(detector.detect(frames[0])[0])


def test_detect_batch_reports_the_failing_frame(built_library):
    """A frame larger than the handle fails alone; the others are detected."""
    small = config_frame("small", seed=4).image
    big = np.zeros((1080, 1920), np.uint8)
    with cctag_b200.Detector(max_w=1280, max_h=720, max_batch=2) as bd:
        with pytest.raises(cctag_b200.CCTagError) as e:
            bd.detect_batch([small, big, small])
        assert e.value.status == cctag_b200.capi.TOO_LARGE
        assert "frame 1" in str(e.value)
        ok = bd.detect_batch([small, small])
    assert len(ok) == 2 and _key(ok[0][0]) == _key(ok[1][0])


def test_streaming_submit_wait_matches_detect(built_library, detector):
    """Frames submitted to the streaming ingest (pinned buffers owned by the
    handle, several in flight) come back with exactly cctagb_detect's result,
    whatever order the tickets are waited in."""
    from cctag_b200.synth import render_frame
    frames = [render_frame(1280, 720, 3, (30.0, 90.0), 50, seed=600 + i, noise_sigma=5.0).image for i in range(6)]
    want = [_key(detector.detect(f)[0]) for f in frames]
    with cctag_b200.Detector(max_w=1280, max_h=720, max_batch=3) as sd:
        bufs = sd.host_frames(3)
        tickets = []
        for i, f in enumerate(frames[:3]):
            bufs[i][:, :] = f
            tickets.append(sd.submit(bufs[i], frame_id=i))
        tickets += [sd.submit(f, frame_id=3 + i) for i, f in enumerate(frames[3:])]
        # another detection call is refused while tickets are outstanding
        with pytest.raises(cctag_b200.CCTagError):
            sd.detect(frames[0])
        got = {t: _key(sd.wait(t)[0]) for t in reversed(tickets)}
        assert [got[t] for t in tickets] == want
        assert _key(sd.detect(frames[0])[0]) == want[0]   # usable again once drained
        with pytest.raises(cctag_b200.CCTagError):
            sd.wait(tickets[0])                           # a ticket is released by its wait
