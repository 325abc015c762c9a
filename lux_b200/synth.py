"""Seeded synthetic stereo inputs for the benchmark workloads (no datasets or real captures are available offline).

A workload is a rectified pair (or a multi-camera capture) expressed in the reference's own input domain: RGBA8
"YUVA" images (grey = (Y, 128, 128, 255)) and CalibData with a pure horizontal baseline, so that plane k of the
plane sweep is disparity k (PlaneDensity 1, a far plane at 1e30 m, near = f·B/(D-1)):
  * texture: a 1/f-spectrum noise image, scaled to the full range of the bit depth;
  * ground truth: six seeded piecewise-planar disparity segments (Voronoi cells) in [0, D-1];
  * the other image: the reference warped by the disparity (nearest surface wins), holes filled by edge repeat,
    plus N(0, sigma^2) noise; 12-bit data is mapped to bytes with (v + 8) >> 4, saturated.
"""
from dataclasses import dataclass
from typing import List

import numpy as np

from .api import CalibData, StereoParams


def texture(h, w, seed, max_value=255.0):
    """1/f-spectrum texture in [0, max_value]."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((h, w)).astype(np.float32)
    spec = np.fft.rfft2(noise)
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.rfftfreq(w)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    f[0, 0] = 1.0
    spec = spec / f
    spec[0, 0] = 0.0
    img = np.fft.irfft2(spec, s=(h, w)).astype(np.float32)
    lo, hi = np.percentile(img, 0.5), np.percentile(img, 99.5)
    img = (img - lo) / max(hi - lo, 1e-6)
    return np.clip(img, 0.0, 1.0) * max_value


def planar_disparity(h, w, d_max, seed, segments=6):
    """Six seeded planar segments (Voronoi cells), values clamped to [0, d_max]."""
    rng = np.random.default_rng(seed + 7919)
    cy = rng.uniform(0, h, segments)
    cx = rng.uniform(0, w, segments)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    d2 = (yy[None] - cy[:, None, None]) ** 2 + (xx[None] - cx[:, None, None]) ** 2
    lab = np.argmin(d2, axis=0)
    disp = np.zeros((h, w), np.float32)
    for s in range(segments):
        base = rng.uniform(0.1, 0.9) * d_max
        gx = rng.uniform(-0.3, 0.3) * d_max / w
        gy = rng.uniform(-0.3, 0.3) * d_max / h
        m = lab == s
        disp[m] = base + gx * (xx[m] - cx[s]) + gy * (yy[m] - cy[s])
    return np.clip(disp, 0, d_max)


def warp_other(left, disp, seed, sigma, max_value):
    """The other view: right(x - d) = left(x), nearest surface (largest d) wins, holes by edge repeat, + noise."""
    h, w = left.shape
    d = np.rint(disp).astype(np.int64)
    xl = np.broadcast_to(np.arange(w), (h, w))
    xr = xl - d
    order = np.argsort(d, axis=1, kind="stable")  # ascending d: the largest d is written last and wins
    rows = np.arange(h)[:, None]
    xr_o = np.take_along_axis(xr, order, 1)
    val_o = np.take_along_axis(left, order, 1)
    ok = (xr_o >= 0) & (xr_o < w)
    right = np.full((h, w), np.nan, np.float32)
    rr = np.broadcast_to(rows, (h, w))[ok]
    right[rr, xr_o[ok]] = val_o[ok]
    # edge repeat: carry the last filled value to the right; leading holes take the first filled value
    filled = ~np.isnan(right)
    idx = np.where(filled, np.arange(w)[None, :], 0)
    np.maximum.accumulate(idx, axis=1, out=idx)
    right = np.take_along_axis(np.nan_to_num(right, nan=0.0), idx, 1)
    first = np.argmax(filled, axis=1)
    lead = np.arange(w)[None, :] < first[:, None]
    right = np.where(lead, np.take_along_axis(right, first[:, None], 1), right)
    rng = np.random.default_rng(seed + 104729)
    right = right + rng.standard_normal((h, w)).astype(np.float32) * sigma
    return np.clip(np.rint(right), 0, max_value)


def to_u8(img, bits):
    """Bytes in the reference's domain: 8-bit as is, 12-bit via (v + 8) >> 4 saturated."""
    v = np.asarray(img).astype(np.int64)
    if bits == 8:
        return np.clip(v, 0, 255).astype(np.uint8)
    return np.clip((v + 8) >> 4, 0, 255).astype(np.uint8)


def gray_rgba(y):
    """(Y, 128, 128, 255): a grey image as the reference's YUVA byte image."""
    h, w = y.shape
    out = np.empty((h, w, 4), np.uint8)
    out[..., 0] = y
    out[..., 1] = 128
    out[..., 2] = 128
    out[..., 3] = 255
    return out


def rectified_calibs(f, cx, cy, baseline):
    """Reference at the origin; the other camera shifted so that a point of disparity d is sampled at x - d."""
    K = np.array([f, 0, cx, 0, f, cy, 0, 0, 1], np.float32)
    R = np.eye(3, dtype=np.float32).reshape(9)
    return [CalibData(K.copy(), np.zeros(3, np.float32), R.copy()),
            CalibData(K.copy(), np.array([-baseline, 0, 0], np.float32), R.copy())]


@dataclass
class PairWorkload:
    images: List[np.ndarray]      # RGBA8 per camera (camera 0 = reference)
    gray: List[int]
    calibs: List[CalibData]
    near: float
    far: float
    params: StereoParams
    disparity: np.ndarray         # ground truth (reference grid)
    d: int
    samples: List[np.ndarray] = None  # the cameras' grey samples as uint16 (pairs of more than 8 bits), before the byte mapping

    @property
    def de(self):
        h, w = self.images[0].shape[:2]
        return w * h * self.d


def rectified_pair(w, h, d, seed=0, bits=8, noise_sigma=2.0, tile=64, f=1000.0, baseline=100.0):
    """One rectified grey pair with planes == integer disparities 0..d-1 (d a multiple of 8)."""
    maxv = 255.0 if bits == 8 else 4095.0
    left = np.rint(texture(h, w, seed, maxv))
    disp = planar_disparity(h, w, d - 1, seed)
    right = warp_other(left, disp, seed, noise_sigma, maxv)
    left = np.clip(left + np.random.default_rng(seed + 15485863).standard_normal((h, w)) * noise_sigma, 0, maxv)
    imgs = [gray_rgba(to_u8(np.rint(left), bits)), gray_rgba(to_u8(right, bits))]
    samples = [np.rint(left).astype(np.uint16), right.astype(np.uint16)] if bits > 8 else None
    near = np.float32(f * baseline / (d - 1))
    params = StereoParams(scale=1, tile=tile, skip_mode=0, plane_density=1.0)
    return PairWorkload(imgs, [1, 1], rectified_calibs(f, w / 2.0, h / 2.0, baseline), float(near), 1e30, params, disp, d,
                        samples)


@dataclass
class CaptureWorkload:
    images: List[np.ndarray]
    gray: List[int]
    calibs: List[CalibData]
    near: float
    far: float
    inv_depth: np.ndarray


def capture(w, h, n_cams, seed=0, f=None, baseline_mm=(8.0, 40.0), near=200.0, far=640000.0, colour=True):
    """A multi-camera capture in the L16 convention: reference camera 0 plus translated cameras (R = I), colour YUVA
    textures, a scene of planar patches at 0.4-6 m. Camera k's image is the reference resampled by the parallax
    f·t/Z (a backward warp on the reference grid)."""
    rng = np.random.default_rng(seed)
    f = f if f is not None else 0.75 * w
    z_inv = 1.0 / np.clip(planar_disparity(h, w, 1.0, seed) * 5600.0 + 400.0, 400.0, 6000.0)  # 1/mm
    chans = [texture(h, w, seed * 7 + c, 255.0) for c in range(3)]
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    imgs, cal = [], []
    K = np.array([f, 0, w / 2.0, 0, f, h / 2.0, 0, 0, 1], np.float32)
    R = np.eye(3, dtype=np.float32).reshape(9)
    for k in range(n_cams):
        if k == 0:
            t = np.zeros(3, np.float32)
        else:
            ang = rng.uniform(0, 2 * np.pi)
            b = rng.uniform(*baseline_mm)
            t = np.array([b * np.cos(ang), b * np.sin(ang), 0.0], np.float32)
        # camera k sees the reference point at x + f·t/Z: sample the reference at x - f·t·invZ
        sx = np.clip(np.rint(xx - f * t[0] * z_inv), 0, w - 1).astype(np.int64)
        sy = np.clip(np.rint(yy - f * t[1] * z_inv), 0, h - 1).astype(np.int64)
        img = np.empty((h, w, 4), np.uint8)
        for c in range(3):
            v = chans[c][sy, sx] + rng.standard_normal((h, w)) * 1.5
            img[..., c] = np.clip(np.rint(v), 0, 255)
        if not colour:
            img[..., 1] = 128
            img[..., 2] = 128
        img[..., 3] = 255
        imgs.append(img)
        cal.append(CalibData(K.copy(), (-t).astype(np.float32), R.copy()))
    gray = [0 if colour else 1] * n_cams
    return CaptureWorkload(imgs, gray, cal, near, far, z_inv)


@dataclass
class ModuleCapture(CaptureWorkload):
    """A capture of one reference module and several others, each with its own crop, focal scale and disparity range."""
    sizes: List[tuple]        # (w, h) per camera
    d_per_camera: List[int]   # the disparity range each other camera spans between near and the far plane
    params: StereoParams = None

    @property
    def de(self):
        h, w = self.images[0].shape[:2]
        return w * h * max(self.d_per_camera)


def module_capture(w, h, n_others=10, seed=0, crop_mp=(1.0, 6.0), ds=(64, 96, 128, 192), near=400.0, far=1e30,
                   size_scale=1.0, tile=64):
    """A batched full capture: reference camera 0 (w x h, focal 0.9 w) and n_others module cameras, half "wide" (focal
    scale 1.0-1.3) and half "tele" (2.2-2.7), each with a crop uniform in crop_mp megapixels (4:3, times size_scale in
    area) and a disparity range D_k drawn from ds, realised by its baseline B_k = D_k·near/f_k in a random direction
    (R = I). Grey u8 images (Y = texture, U = V = 128). The scene is the reference texture on six planar patches at
    near-6 m; camera k sees it through a backward warp (two fixed-point steps for the parallax). One layer over all
    cameras sums their costs (the reference's fusion) with n = max D_k planes (density 1)."""
    rng = np.random.default_rng(seed)
    f0 = 0.9 * w
    cx0, cy0 = (w - 1) / 2.0, (h - 1) / 2.0
    # the scene on a canvas three times the reference extent (wide cameras see beyond the reference crop)
    H3, W3 = 3 * h, 3 * w
    tex = texture(H3, W3, seed * 13 + 1, 255.0)
    z_inv = 1.0 / np.clip(planar_disparity(H3, W3, 1.0, seed) * (6000.0 - near) + near, near, 6000.0)

    def scene(x, y):  # reference-pixel coordinates -> (texture, 1/Z) by nearest sampling on the canvas
        xi = np.clip(np.rint(x + w), 0, W3 - 1).astype(np.int64)
        yi = np.clip(np.rint(y + h), 0, H3 - 1).astype(np.int64)
        return tex[yi, xi], z_inv[yi, xi]

    R = np.eye(3, dtype=np.float32).reshape(9)
    K0 = np.array([f0, 0, cx0, 0, f0, cy0, 0, 0, 1], np.float32)
    imgs, cal, sizes, dk = [], [], [], []
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    t0, _ = scene(xx, yy)
    imgs.append(gray_rgba(to_u8(np.rint(t0 + rng.standard_normal(t0.shape) * 1.5), 8)))
    cal.append(CalibData(K0.copy(), np.zeros(3, np.float32), R.copy()))
    sizes.append((w, h))
    for k in range(n_others):
        tele = k >= n_others // 2
        s = rng.uniform(2.2, 2.7) if tele else rng.uniform(1.0, 1.3)
        mp = rng.uniform(*crop_mp) * 1e6 * size_scale
        hk = max(8, int(round(np.sqrt(mp * 3.0 / 4.0))))
        wk = max(8, int(round(hk * 4.0 / 3.0)))
        fk = f0 * s
        d = int(rng.choice(ds))
        b = d * near / fk
        ang = rng.uniform(0, 2 * np.pi)
        t = np.array([b * np.cos(ang), b * np.sin(ang), 0.0], np.float32)
        cxk, cyk = (wk - 1) / 2.0, (hk - 1) / 2.0
        v, u = np.mgrid[0:hk, 0:wk].astype(np.float32)
        # camera k sees the scene point at reference (x, y) at u = cxk + fk·((x - cx0)/f0 + t_x/Z)
        x = cx0 + f0 * (u - cxk) / fk
        y = cy0 + f0 * (v - cyk) / fk
        for _ in range(2):
            _, zi = scene(x, y)
            x = cx0 + f0 * ((u - cxk) / fk - t[0] * zi)
            y = cy0 + f0 * ((v - cyk) / fk - t[1] * zi)
        tk, _ = scene(x, y)
        imgs.append(gray_rgba(to_u8(np.rint(tk + rng.standard_normal(tk.shape) * 1.5), 8)))
        K = np.array([fk, 0, cxk, 0, fk, cyk, 0, 0, 1], np.float32)
        cal.append(CalibData(K, (-t).astype(np.float32), R.copy()))
        sizes.append((wk, hk))
        dk.append(d)
    params = StereoParams(scale=1, tile=tile, skip_mode=0, plane_density=1.0)
    return ModuleCapture(imgs, [1] * (n_others + 1), cal, near, far, z_inv[h:2 * h, w:2 * w], sizes, dk, params)


def isp_image(w, h, seed=0):
    """A half-resolution ISP output as the stereo images take it: linear RGB in [0, 1] (1/f texture per channel, a
    colour cast), alpha 1; (h, w, 4) float32."""
    rng = np.random.default_rng(seed)
    out = np.empty((h, w, 4), np.float32)
    for c in range(3):
        out[..., c] = (texture(h, w, seed * 7 + c, max_value=1.0) * rng.uniform(0.4, 1.0)).astype(np.float32)
    out[..., 3] = 1.0
    return out


def aligned_calib(sw, sh, dw, dh, seed=0, angle_deg=0.6, focal_ratio=1.02, shift=(3.5, -2.25), lens=4e-9):
    """An aligned calibration of the stereo-image warp (the fields AlignedCalib.Build leaves): the rotation homography
    H = K_B·R·K_A^-1 of a dw x dh view onto a sw x sh module (a small rotation about the optical axis and a tilt, focal
    lengths in the given ratio, a shifted principal point), and a radial CRA lut lut[r] = 1 + lens·r^2 over 4096 radius
    steps with the scales putting the image corners near r = 3000. Values are float32 as the host computes them."""
    rng = np.random.default_rng(seed)
    f_a = 1.1 * dw
    Ka = np.array([[f_a, 0, dw / 2.0], [0, f_a, dh / 2.0], [0, 0, 1]])
    Kb = np.array([[f_a * focal_ratio, 0, sw / 2.0 + shift[0]], [0, f_a * focal_ratio, sh / 2.0 + shift[1]], [0, 0, 1]])
    a = np.deg2rad(angle_deg)
    t = np.deg2rad(rng.uniform(-0.3, 0.3, 2))
    Rz = np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])
    Rx = np.array([[1, 0, 0], [0, np.cos(t[0]), -np.sin(t[0])], [0, np.sin(t[0]), np.cos(t[0])]])
    Ry = np.array([[np.cos(t[1]), 0, np.sin(t[1])], [0, 1, 0], [-np.sin(t[1]), 0, np.cos(t[1])]])
    H = (Kb @ Rz @ Rx @ Ry @ np.linalg.inv(Ka)).astype(np.float32)
    r = np.arange(4096, dtype=np.float64)
    lut = (1.0 + lens * r * r).astype(np.float32)
    half_diag = 0.5 * np.hypot(sw, sh)
    s = np.float32(3000.0 / half_diag)
    from .api import AlignedCalib
    return AlignedCalib(H=H, lut=lut, cx=np.float32(sw / 2.0), cy=np.float32(sh / 2.0), sx=s, sy=s)


def census_capture(w, h, ds, seed=0, f=1000.0):
    """A capture for the census mode: one reference image and one other image per pair on the reference's grid, pair k
    seeing a scene whose disparities span 0..ds[k]-1 (its baseline B_k = ds[k] units, so fb[k] = f·B_k). Returns
    (reference (h, w) uint8, [others (h, w) uint8], fb float32 array)."""
    left = np.rint(texture(h, w, seed, 255.0))
    shape = planar_disparity(h, w, 1.0, seed)  # a common scene depth structure, scaled per pair
    others = []
    for k, d in enumerate(ds):
        others.append(warp_other(left, shape * (d - 1), seed + 31 * (k + 1), 2.0, 255.0).astype(np.uint8))
    ref = np.clip(left + np.random.default_rng(seed + 7).standard_normal((h, w)) * 2.0, 0, 255).round().astype(np.uint8)
    return ref, others, np.asarray([f * d for d in ds], np.float32)
