"""GPU parity of the image stage and the vote, through the C ABI, against the
CPU oracle (bit-exact: planes, edge maps, edge order, links, votes, flow
lengths, voter lists and seed order)."""
import numpy as np
import pytest

import cctag_b200
from cctag_b200.synth import config_frame, render_frame

pytestmark = pytest.mark.gpu


def oracle_frame(orc, img, levels=4):
    out = []
    for lvl, src in enumerate(orc.pyramid(img, levels)):
        dx, dy, e = orc.level(src)
        v = orc.vote(e, dx, dy)
        out.append(dict(src=src, dx=dx, dy=dy, edges=e, vote=v))
    return out


def check_level(det, lvl, ref):
    src, dx, dy, edges = det.level_planes(lvl)
    np.testing.assert_array_equal(src, ref["src"], err_msg=f"level {lvl} src")
    np.testing.assert_array_equal(dx, ref["dx"], err_msg=f"level {lvl} dx")
    np.testing.assert_array_equal(dy, ref["dy"], err_msg=f"level {lvl} dy")
    np.testing.assert_array_equal(edges, ref["edges"], err_msg=f"level {lvl} edges")
    v = ref["vote"]
    x, y = det.edge_points(lvl)
    np.testing.assert_array_equal(x, v["x"])
    np.testing.assert_array_equal(y, v["y"])
    b, a = det.links(lvl)
    np.testing.assert_array_equal(b, v["before"], err_msg=f"level {lvl} before")
    np.testing.assert_array_equal(a, v["after"], err_msg=f"level {lvl} after")
    g = det.votes(lvl)
    np.testing.assert_array_equal(g["chosen"], v["chosen"], err_msg=f"level {lvl} chosen")
    np.testing.assert_array_equal(g["nvotes"], v["nvotes"], err_msg=f"level {lvl} nvotes")
    np.testing.assert_array_equal(g["voff"], v["voff"])
    np.testing.assert_array_equal(g["vlist"], v["vlist"])
    np.testing.assert_array_equal(g["flow"].view(np.int32), v["flow"].view(np.int32), err_msg=f"level {lvl} flow")
    np.testing.assert_array_equal(det.seeds(lvl), v["seeds"], err_msg=f"level {lvl} seeds")


@pytest.mark.parametrize("name,seed", [("small", 1), ("small", 2), ("small", 3), ("c1_720p", 1), ("c1_720p", 7)])
def test_image_stage_matches_oracle(detector, orc, name, seed):
    img = config_frame(name, seed=seed).image
    detector.image_stage(img)
    for lvl, ref in enumerate(oracle_frame(orc, img)):
        check_level(detector, lvl, ref)


def test_image_stage_1080p_matches_oracle(detector, orc):
    img = config_frame("c2_1080p", seed=1).image
    detector.image_stage(img)
    for lvl, ref in enumerate(oracle_frame(orc, img)):
        check_level(detector, lvl, ref)


@pytest.mark.parametrize("shape", [(181, 257), (99, 131), (16, 16), (8, 40)])
def test_odd_and_tiny_sizes(detector, orc, shape):
    rng = np.random.default_rng(shape[0] * 1000 + shape[1])
    img = render_frame(shape[1], shape[0], 1 if min(shape) > 90 else 0, (20, 40), 30, seed=int(rng.integers(1 << 30)),
                       noise_sigma=10.0)
    detector.image_stage(img.image)
    for lvl, ref in enumerate(oracle_frame(orc, img.image)):
        check_level(detector, lvl, ref)


def test_blank_frame_has_no_edges(detector):
    detector.image_stage(np.full((120, 160), 77, np.uint8))
    for lvl in range(4):
        x, _ = detector.edge_points(lvl)
        assert len(x) == 0
        assert len(detector.seeds(lvl)) == 0


def test_canny_from_opencv_derivatives(detector, orc, opencv_cases):
    """Parity when both sides are fed the same (OpenCV) derivative images."""
    for k in opencv_cases:
        if k.startswith("deriv") and k.endswith("_dx"):
            dx = opencv_cases[k]
            dy = opencv_cases[k[:-3] + "_dy"]
            got = detector.canny_from_derivatives(dx, dy)
            want = orc.thin(orc.canny(dx, dy))
            np.testing.assert_array_equal(got, want, err_msg=k)


def test_clutter_4k_vote_counts(detector, orc):
    """Clutter stress: 4K with distractor ellipses, lines and a textured
    background (about 1.7 M edge points), integer vote counts bit-exact at
    every level."""
    img = config_frame("c3_4k_clutter", seed=3).image
    detector.image_stage(img)
    for lvl, src in enumerate(orc.pyramid(img, 4)):
        dx, dy, e = orc.level(src)
        v = orc.vote(e, dx, dy)
        g = detector.votes(lvl)
        np.testing.assert_array_equal(g["nvotes"], v["nvotes"], err_msg=f"level {lvl}")
        np.testing.assert_array_equal(detector.seeds(lvl), v["seeds"], err_msg=f"level {lvl}")


def test_errors_are_status_codes(built_library):
    p = cctag_b200.default_params(3)
    with cctag_b200.Detector(p, max_w=64, max_h=64) as d:
        with pytest.raises(cctag_b200.CCTagError) as ei:
            d.image_stage(np.zeros((80, 80), np.uint8))
        assert ei.value.status == cctag_b200.capi.TOO_LARGE
        with pytest.raises(cctag_b200.CCTagError) as ei:
            d.image_stage(np.zeros((4, 4), np.uint8))
        assert ei.value.status == cctag_b200.capi.BAD_ARG
    p.edgeCapacityDivisor = 100000
    with cctag_b200.Detector(p, max_w=640, max_h=480) as d:
        with pytest.raises(cctag_b200.CCTagError) as ei:
            d.image_stage(config_frame("small", seed=1).image)
        assert ei.value.status == cctag_b200.capi.OVERFLOW_EDGES
        # the handle stays usable after an error
        d.image_stage(np.full((120, 160), 5, np.uint8))
    p = cctag_b200.default_params(3)
    p.distSearch = 1 << 20
    with pytest.raises(cctag_b200.CCTagError) as ei:
        cctag_b200.Detector(p, max_w=64, max_h=64)
    assert ei.value.status == cctag_b200.capi.BAD_ARG


def test_stage_timing_mode_gives_same_results(detector, orc):
    img = config_frame("small", seed=5).image
    detector.set_stage_timing(True)
    try:
        detector.image_stage(img)
        times = detector.stage_times()
    finally:
        detector.set_stage_timing(False)
    assert set(times) >= {"pyramid", "deriv_nms", "vote", "voter_sort"}
    assert all(v >= 0 for v in times.values()) and sum(times.values()) > 0
    ref = oracle_frame(orc, img)
    for lvl in range(4):
        check_level(detector, lvl, ref[lvl])
