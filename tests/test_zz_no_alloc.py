"""GPU test of cctagb_edges_noalloc, the edge stage for callers that cannot
allocate device memory (all memory given to their own pool, or a real-time
loop that forbids cudaMalloc/cudaFree after start-up).

The entry point is called through the C ABI on device buffers that this test
allocates itself, twice in a row on different frames (so the second call runs
on scratch left by the first), and its derivatives and edge map must equal,
bit for bit, those of the handle-based image stage (cctagb_image_stage) on the
same frames -- the exact tolerance the other image-stage tests use.

This file is named so that pytest collects it last."""
import ctypes as C

import numpy as np
import pytest

from cctag_b200.synth import config_frame, render_frame

pytestmark = pytest.mark.gpu


def _handle_edges(img):
    import cctag_b200

    with cctag_b200.Detector(max_w=img.shape[1], max_h=img.shape[0]) as det:
        det.image_stage(img)
        _, dx, dy, edges = det.level_planes(0)
    return dx, dy, edges


def _noalloc_edges(img, stream):
    import torch

    from cctag_b200 import capi

    lib = capi.load()
    h, w = img.shape
    d_gray = torch.from_numpy(np.ascontiguousarray(img)).cuda()
    d_dx = torch.empty((h, w), dtype=torch.int16, device="cuda")
    d_dy = torch.empty((h, w), dtype=torch.int16, device="cuda")
    d_edges = torch.empty((h, w), dtype=torch.uint8, device="cuda")
    d_status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    st = lib.cctagb_edges_noalloc(C.c_void_p(d_gray.data_ptr()), w, h, w, C.c_float(0.01), C.c_float(0.04),
                                  C.c_void_p(d_dx.data_ptr()), C.c_void_p(d_dy.data_ptr()),
                                  C.c_void_p(d_edges.data_ptr()), C.c_void_p(d_status.data_ptr()),
                                  C.c_void_p(stream.cuda_stream))
    assert st == capi.OK, lib.cctagb_status_string(st)
    stream.synchronize()
    assert int(d_status.item()) == 0
    return d_dx.cpu().numpy(), d_dy.cpu().numpy(), d_edges.cpu().numpy()


def test_edges_noalloc_matches_image_stage_twice(built_library):
    import torch

    frames = [config_frame("c1_720p", seed=11).image,
              render_frame(1000, 600, 3, (30, 90), 45, seed=12, noise_sigma=7.0).image]
    stream = torch.cuda.Stream()
    for img in frames:  # two calls in a row; the second reuses the scratch
        want = _handle_edges(img)
        got = _noalloc_edges(img, stream)
        for name, g, e in zip(("dx", "dy", "edges"), got, want):
            np.testing.assert_array_equal(g, e, err_msg=name)


def test_edges_noalloc_at_the_size_limits(built_library):
    """Frames of exactly the maximum pixel count with one side at the maximum
    (4096 x 256 and 256 x 4096), where the scratch array's bitmap words and
    row counts are at their bounds."""
    import torch

    stream = torch.cuda.Stream()
    for w, h in ((4096, 256), (256, 4096)):
        img = render_frame(w, h, 3, (20, 60), 45, seed=w + h, noise_sigma=6.0).image
        want = _handle_edges(img)
        got = _noalloc_edges(img, stream)
        for name, g, e in zip(("dx", "dy", "edges"), got, want):
            np.testing.assert_array_equal(g, e, err_msg=f"{w}x{h} {name}")


def test_edges_noalloc_rejects_oversized_frames(built_library):
    import torch

    from cctag_b200 import capi

    lib = capi.load()
    buf = torch.empty(16, dtype=torch.uint8, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    st = lib.cctagb_edges_noalloc(p, 2048, 1024, 2048, C.c_float(0.01), C.c_float(0.04), p, p, p, None, None)
    assert st == capi.TOO_LARGE
    st = lib.cctagb_edges_noalloc(p, 4097, 200, 4097, C.c_float(0.01), C.c_float(0.04), p, p, p, None, None)
    assert st == capi.TOO_LARGE
    st = lib.cctagb_edges_noalloc(p, 100, 100, 128, C.c_float(0.01), C.c_float(0.04), p, p, p, None, None)
    assert st == capi.BAD_ARG
