"""Seeded synthetic CCTag frames with ground truth.

The reference ships no test frames with expected outputs, so the test-suite and
the benchmark render their own.  A 3-crown marker is the stack of discs drawn by
``markersToPrint/generators/generate.py:80-95``: a black disc of radius 1, then
alternating white/black discs at the radii ``1/ratio`` of its bank row
(``CCTagMarkersBank.cpp:120-152``; e.g. ID 0 -> 0.9, 0.8, 0.7, 0.6, 0.5).  A
white paper margin out to radius ``margin`` surrounds it.

Each marker is mapped into the image by a pinhole homography (in-plane rotation,
tilt about a random in-plane axis, mild perspective).  Pixel (row i, col j) has
its centre at image coordinates (x=j, y=i), the convention of the reference's
bilinear sampler (``Identification.hpp:197-219``).  Coverage is supersampled,
then the frame gets a Gaussian blur, an optional linear motion blur, a linear
illumination gradient, Gaussian noise and 8-bit quantisation.

Ground truth per marker: id, imaged centre (image of the marker origin), the
homography H (marker plane -> image) and the outer ellipse (image of the unit
circle) as a conic matrix.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .bank import THREE_CROWNS

__all__ = ["Marker", "Frame", "render_frame", "config_frame", "marker_homography"]


@dataclass
class Marker:
    id: int
    center: tuple[float, float]
    radius_px: float
    H: np.ndarray          # 3x3, marker plane -> image
    outer_conic: np.ndarray  # 3x3 conic of the outer circle in the image


@dataclass
class Frame:
    image: np.ndarray
    markers: list[Marker] = field(default_factory=list)
    seed: int = 0


def marker_homography(rng, cx, cy, radius_px, max_tilt_deg, focal):
    """Plane -> image homography with the origin imaged at (cx, cy)."""
    rot = rng.uniform(0, 2 * np.pi)
    tilt = np.deg2rad(rng.uniform(0, max_tilt_deg))
    axis = rng.uniform(0, np.pi)
    cz, sz = np.cos(rot), np.sin(rot)
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1.0]])
    ca, sa = np.cos(axis), np.sin(axis)
    Ra = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1.0]])
    ct, st = np.cos(tilt), np.sin(tilt)
    Rx = np.array([[1, 0, 0], [0, ct, -st], [0, st, ct]])
    R = Ra @ Rx @ Ra.T @ Rz
    # Depth such that the marker (radius 1) spans ~radius_px pixels.
    Z = focal / radius_px
    K = np.array([[focal, 0, cx], [0, focal, cy], [0, 0, 1.0]])
    t = np.array([0.0, 0.0, Z])
    H = K @ np.column_stack([R[:, 0], R[:, 1], t])
    return H / H[2, 2]


def _outer_conic(H):
    Hi = np.linalg.inv(H)
    C = Hi.T @ np.diag([1.0, 1.0, -1.0]) @ Hi
    return C / np.linalg.norm(C)


def _ring_value(rho, radii, margin):
    """Intensity in [0, 1] (1 = white) of a 3-crown marker at plane radius rho."""
    # Outside-in: margin white, [r5..1] black, [r4..r5] white, ...
    out = np.full(rho.shape, np.nan, dtype=np.float32)
    out[rho <= margin] = 1.0
    out[rho <= 1.0] = 0.0
    color = 1.0
    for r in radii:  # descending radii: 0.9, 0.8, 0.7, 0.6, 0.5
        out[rho <= r] = color
        color = 1.0 - color
    return out


def _paint_marker(canvas, weight, H, radii, margin, white, black, ss):
    Hh, Ww = canvas.shape
    Hi = np.linalg.inv(H)
    # Bounding box of the margin circle in the image.
    th = np.linspace(0, 2 * np.pi, 256)
    pts = H @ np.vstack([margin * np.cos(th), margin * np.sin(th), np.ones_like(th)])
    px, py = pts[0] / pts[2], pts[1] / pts[2]
    x0, x1 = int(np.floor(px.min())) - 2, int(np.ceil(px.max())) + 2
    y0, y1 = int(np.floor(py.min())) - 2, int(np.ceil(py.max())) + 2
    x0, y0 = max(x0, 0), max(y0, 0)
    x1, y1 = min(x1, Ww - 1), min(y1, Hh - 1)
    if x1 < x0 or y1 < y0:
        return
    offs = (np.arange(ss) + 0.5) / ss - 0.5
    xs = np.arange(x0, x1 + 1, dtype=np.float64)
    ys = np.arange(y0, y1 + 1, dtype=np.float64)
    acc = np.zeros((len(ys), len(xs)), np.float32)
    cov = np.zeros((len(ys), len(xs)), np.float32)
    for oy in offs:
        for ox in offs:
            X = xs[None, :] + ox
            Y = ys[:, None] + oy
            u = Hi[0, 0] * X + Hi[0, 1] * Y + Hi[0, 2]
            v = Hi[1, 0] * X + Hi[1, 1] * Y + Hi[1, 2]
            w = Hi[2, 0] * X + Hi[2, 1] * Y + Hi[2, 2]
            rho = np.sqrt((u / w) ** 2 + (v / w) ** 2)
            val = _ring_value(rho, radii, margin)
            inside = ~np.isnan(val)
            acc += np.where(inside, black + (white - black) * np.nan_to_num(val), 0.0)
            cov += inside
    cov /= ss * ss
    acc /= ss * ss
    sl = canvas[y0:y1 + 1, x0:x1 + 1]
    canvas[y0:y1 + 1, x0:x1 + 1] = sl * (1.0 - cov) + acc


def _gauss_blur(img, sigma):
    if sigma <= 0:
        return img
    r = int(np.ceil(3 * sigma))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    k /= k.sum()
    pad = np.pad(img, ((0, 0), (r, r)), mode="edge")
    tmp = sum(k[i] * pad[:, i:i + img.shape[1]] for i in range(2 * r + 1))
    pad = np.pad(tmp, ((r, r), (0, 0)), mode="edge")
    return sum(k[i] * pad[i:i + img.shape[0], :] for i in range(2 * r + 1)).astype(np.float32)


def _motion_blur(img, length, angle):
    if length < 1.0:
        return img
    n = int(np.ceil(length)) * 2 + 1
    acc = np.zeros_like(img)
    for t in np.linspace(-length / 2, length / 2, n):
        dx, dy = t * np.cos(angle), t * np.sin(angle)
        ix, iy = int(np.floor(dx)), int(np.floor(dy))
        fx, fy = dx - ix, dy - iy
        sh = np.roll(np.roll(img, iy, axis=0), ix, axis=1)
        sh1 = np.roll(sh, 1, axis=1)
        sh2 = np.roll(sh, 1, axis=0)
        sh3 = np.roll(sh1, 1, axis=0)
        acc += (1 - fx) * (1 - fy) * sh + fx * (1 - fy) * sh1 + (1 - fx) * fy * sh2 + fx * fy * sh3
    return acc / n


def _draw_distractors(rng, canvas, n_ellipses, n_lines):
    Hh, Ww = canvas.shape
    yy, xx = np.mgrid[0:Hh, 0:Ww]
    for _ in range(n_ellipses):
        cx, cy = rng.uniform(0, Ww), rng.uniform(0, Hh)
        a = rng.uniform(8, 120)
        b = a * rng.uniform(0.3, 1.0)
        ang = rng.uniform(0, np.pi)
        val = rng.uniform(0, 255)
        width = rng.uniform(1.5, 6)
        rings = 1 if rng.uniform() < 0.5 else 2
        x0, x1 = int(max(cx - a - 8, 0)), int(min(cx + a + 8, Ww - 1))
        y0, y1 = int(max(cy - a - 8, 0)), int(min(cy + a + 8, Hh - 1))
        if x1 <= x0 or y1 <= y0:
            continue
        X = xx[y0:y1 + 1, x0:x1 + 1] - cx
        Y = yy[y0:y1 + 1, x0:x1 + 1] - cy
        c, s = np.cos(ang), np.sin(ang)
        u = c * X + s * Y
        v = -s * X + c * Y
        for k in range(rings):
            sc = 1.0 - 0.35 * k
            rr = np.sqrt((u / (a * sc)) ** 2 + (v / (b * sc)) ** 2)
            d = np.abs(rr - 1.0) * b * sc
            cov = np.clip(width / 2 - d + 0.5, 0, 1).astype(np.float32)
            sl = canvas[y0:y1 + 1, x0:x1 + 1]
            canvas[y0:y1 + 1, x0:x1 + 1] = sl * (1 - cov) + val * cov
    for _ in range(n_lines):
        x0f, y0f = rng.uniform(0, Ww), rng.uniform(0, Hh)
        L = rng.uniform(20, 300)
        ang = rng.uniform(0, 2 * np.pi)
        x1f, y1f = x0f + L * np.cos(ang), y0f + L * np.sin(ang)
        width = rng.uniform(1, 4)
        val = rng.uniform(0, 255)
        bx0 = int(max(min(x0f, x1f) - 4, 0)); bx1 = int(min(max(x0f, x1f) + 4, Ww - 1))
        by0 = int(max(min(y0f, y1f) - 4, 0)); by1 = int(min(max(y0f, y1f) + 4, Hh - 1))
        if bx1 <= bx0 or by1 <= by0:
            continue
        X = xx[by0:by1 + 1, bx0:bx1 + 1]
        Y = yy[by0:by1 + 1, bx0:bx1 + 1]
        dxl, dyl = x1f - x0f, y1f - y0f
        t = np.clip(((X - x0f) * dxl + (Y - y0f) * dyl) / (L * L), 0, 1)
        d = np.hypot(X - (x0f + t * dxl), Y - (y0f + t * dyl))
        cov = np.clip(width / 2 - d + 0.5, 0, 1).astype(np.float32)
        sl = canvas[by0:by1 + 1, bx0:bx1 + 1]
        canvas[by0:by1 + 1, bx0:bx1 + 1] = sl * (1 - cov) + val * cov


def render_frame(width, height, n_markers, radius_range, max_tilt_deg, *, seed, bg=128.0,
                 noise_sigma=4.0, blur_sigma=1.0, motion_len=0.0, motion_angle=0.0,
                 illum_grad=0.0, n_ellipses=0, n_lines=0, margin=1.3, ss=None,
                 bank=THREE_CROWNS, white=235.0, black=20.0, texture=(0.0, 0.0)) -> Frame:
    """Render one frame; markers do not overlap (rejection placement).
    texture = (amplitude, sigma): a band-limited background (white noise
    blurred by sigma px, scaled to that standard deviation) under the
    distractors and markers, for clutter with dense edges."""
    rng = np.random.default_rng(seed)
    canvas = np.full((height, width), bg, np.float32)
    if texture[0] > 0:
        t = _gauss_blur(rng.standard_normal((height, width)).astype(np.float32), texture[1])
        canvas += np.float32(texture[0]) * t / max(float(t.std()), 1e-6)
    if n_ellipses or n_lines:
        _draw_distractors(rng, canvas, n_ellipses, n_lines)
    focal = 1.2 * max(width, height)
    placed: list[tuple[float, float, float]] = []
    markers: list[Marker] = []
    tries = 0
    while len(markers) < n_markers and tries < 200 * max(1, n_markers):
        tries += 1
        r = rng.uniform(*radius_range)
        ext = r * margin * 1.6 + 4
        if 2 * ext >= min(width, height):
            continue
        cx = rng.uniform(ext, width - ext)
        cy = rng.uniform(ext, height - ext)
        if any((cx - px) ** 2 + (cy - py) ** 2 < (ext + pe) ** 2 for px, py, pe in placed):
            continue
        H = marker_homography(rng, cx, cy, r, max_tilt_deg, focal)
        mid = int(rng.integers(0, len(bank)))
        radii = sorted((1.0 / float(q) for q in bank[mid]), reverse=True)
        sub = ss if ss is not None else (8 if r <= 60 else 4)
        _paint_marker(canvas, None, H, radii, margin, white, black, sub)
        placed.append((cx, cy, ext))
        markers.append(Marker(mid, (cx, cy), r, H, _outer_conic(H)))
    img = _gauss_blur(canvas, blur_sigma)
    img = _motion_blur(img, motion_len, motion_angle)
    if illum_grad:
        ang = rng.uniform(0, 2 * np.pi)
        yy, xx = np.mgrid[0:height, 0:width]
        ramp = ((xx - width / 2) * np.cos(ang) + (yy - height / 2) * np.sin(ang))
        ramp = ramp / max(np.abs(ramp).max(), 1.0)
        img = img + illum_grad * ramp.astype(np.float32)
    if noise_sigma > 0:
        img = img + rng.normal(0.0, noise_sigma, img.shape).astype(np.float32)
    out = np.clip(np.rint(img), 0, 255).astype(np.uint8)
    return Frame(out, markers, seed)


def config_frame(name: str, seed: int = 0) -> Frame:
    """The benchmark configurations, by name."""
    rng = np.random.default_rng(seed + 1000)
    if name == "c1_720p":
        return render_frame(1280, 720, 4, (40, 120), 45, seed=seed, noise_sigma=4.0, blur_sigma=1.0)
    if name == "c2_1080p":
        return render_frame(1920, 1080, 12, (20, 200), 60, seed=seed, noise_sigma=8.0, blur_sigma=1.0,
                            motion_len=float(rng.uniform(0, 5)), motion_angle=float(rng.uniform(0, np.pi)),
                            illum_grad=40.0)
    if name == "c3_4k_clutter":
        # a band-limited background texture brings the Canny points into the
        # 1-3 M range of this workload (about 1.2 M on level 0)
        return render_frame(3840, 2160, 30, (15, 300), 60, seed=seed, noise_sigma=6.0, blur_sigma=1.0,
                            n_ellipses=200, n_lines=300, texture=(6.0, 2.0))
    if name == "small":
        return render_frame(320, 240, 1, (40, 60), 30, seed=seed, noise_sigma=3.0, blur_sigma=1.0)
    raise ValueError(f"unknown configuration {name!r}")


CAMERA_SIZES = ((640, 480), (1280, 720), (1920, 1080), (3840, 2160))


def _camera_frame(job):
    w, h, n_markers, rmax, seed, noise = job
    return render_frame(w, h, n_markers, (15.0, rmax), 60, seed=seed, noise_sigma=noise, blur_sigma=1.0)


def camera_batch(seed: int = 0, n: int = 16, map_fn=map) -> list:
    """Multi-camera step: n frames, each of a resolution drawn uniformly from
    CAMERA_SIZES, with 0-20 markers (outer radius up to a quarter of the
    shorter side), tilt <= 60 deg, noise sigma 4-8.  map_fn renders the frames
    (a process pool's map spreads them over the host cores; same result)."""
    rng = np.random.default_rng(seed + 7000)
    jobs = []
    for i in range(n):
        w, h = CAMERA_SIZES[int(rng.integers(len(CAMERA_SIZES)))]
        rmax = min(200.0, min(w, h) / 4.0)
        jobs.append((w, h, int(rng.integers(0, 21)), rmax, seed * 1000 + i, float(rng.uniform(4.0, 8.0))))
    return list(map_fn(_camera_frame, jobs))


def ellipse_of_conic(Q: np.ndarray):
    """(cx, cy, a, b, angle) of an ellipse conic x^T Q x = 0 (a along angle)."""
    Q = np.asarray(Q, np.float64)
    A, bvec = Q[:2, :2], Q[:2, 2]
    c = -np.linalg.solve(A, bvec)
    k = Q[2, 2] + bvec @ c
    w, V = np.linalg.eigh(A / -k)
    a, b = 1.0 / np.sqrt(w[0]), 1.0 / np.sqrt(w[1])
    ang = float(np.arctan2(V[1, 0], V[0, 0]))
    return float(c[0]), float(c[1]), float(a), float(b), ang


def cut_task_from_marker(m: Marker, roi, n_cuts: int = 22, offset=(0.0, 0.0), start=None, local=False):
    """A cctagb_cut_task for a rendered marker: its true outer ellipse, cut
    stops spread evenly on it, the ellipse center as the initial imaged center
    (as detection starts), all shifted by `offset` (an atlas placement);
    `roi` = (x, y, w, h) in the shifted image.  local: the geometry stays in
    the marker's own frame (the task's coordinates are relative to the roi
    corner; `offset` is then only the roi's placement)."""
    from .capi import CutTask

    ox, oy = (0.0, 0.0) if local else offset
    T = np.array([[1, 0, -ox], [0, 1, -oy], [0, 0, 1.0]])
    Q = T.T @ m.outer_conic @ T          # conic in shifted coordinates
    Q = Q / np.abs(Q).max()
    cx, cy, a, b, ang = ellipse_of_conic(Q)
    t = CutTask()
    for k in range(9):
        t.Q[k] = float(Q.flat[k])
    t.cx, t.cy, t.a, t.b, t.angle = cx, cy, a, b, ang
    t.x0, t.y0 = (cx, cy) if start is None else start
    t.ncuts = n_cuts
    ca, sa = np.cos(ang), np.sin(ang)
    for i in range(n_cuts):
        th = 2 * np.pi * i / n_cuts
        t.stop[i][0] = cx + a * np.cos(th) * ca - b * np.sin(th) * sa
        t.stop[i][1] = cy + a * np.cos(th) * sa + b * np.sin(th) * ca
    for k in range(4):
        t.roi[k] = int(roi[k])
    t.local = int(bool(local))
    return t


def _refine_crop(job):
    """One crop of refine_atlas (module level so that a process pool can run it)."""
    seed, i, r, noise = job
    s = int(np.ceil(4.2 * r + 12))
    return render_frame(s, s, 1, (r, r), 70, seed=seed * 100000 + i, noise_sigma=noise, blur_sigma=1.0)


def refine_atlas(seed: int = 0, n_crops: int = 256, width: int = 4096, map_fn=map):
    """Candidate-refinement workload: n_crops single-marker crops (outer radius
    8-150 px, tilt <= 70 deg, noise sigma 2-12) packed row by row into one
    atlas image.  Returns (atlas, [(marker in its crop's coordinates, roi)]), roi =
    (x, y, w, h) of the crop in the atlas.  map_fn renders the crops (a
    process pool's map spreads them over the host cores; same result)."""
    rng = np.random.default_rng(seed + 9000)
    jobs = []
    for i in range(n_crops):
        r = float(rng.uniform(8.0, 150.0))
        jobs.append((seed, i, r, float(rng.uniform(2.0, 12.0))))
    crops = [f for f in map_fn(_refine_crop, jobs) if f.markers]
    # shelf packing
    x = y = shelf = 0
    places = []
    for f in crops:
        h, w = f.image.shape
        if x + w > width:
            x, y, shelf = 0, y + shelf, 0
        places.append((x, y))
        x += w
        shelf = max(shelf, h)
    atlas = np.full((y + shelf, width), 128, np.uint8)
    out = []
    for f, (ox, oy) in zip(crops, places):
        h, w = f.image.shape
        atlas[oy:oy + h, ox:ox + w] = f.image
        m = f.markers[0]
        out.append((m, (ox, oy, w, h)))
    return atlas, out
