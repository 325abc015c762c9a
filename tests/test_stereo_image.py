"""Stereo-image formation after the ISP and the reference guide's 8-bit warp against the oracle, bit for bit.

StereoImage.Warp (6x6 Lanczos-3 taps through an aligned calibration, fill 0), ConvertToYUV + the 8-bit store
(StereoImageBuilder.Create after the ISP) and Rgba8Warp.Warp (every tap clamped). The host-side tables (the Lanczos taps
from Wine's sinf, the YUV rows) are checked on the CPU; the kernels on the GPU. The reference ships no vectors for these
functions: the oracle restates StereoImage.cs, ReferenceGuide.cs and WineCrt.cs.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def api():
    from lux_b200 import api
    return api


def _bits(a):
    a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    return np.ascontiguousarray(a).view(np.uint8)


def test_lanczos_table_host_matches_oracle(api):
    """The taps the library uploads (host code) equal the oracle's LanczosTable; every phase sums to 1 within rounding."""
    t = api.StereoImage.lanczos_table()
    assert np.array_equal(t.view(np.uint32), O.lanczos_table().view(np.uint32))
    assert np.all(np.abs(t.sum(1) - 1.0) < 1e-6)
    assert t[0, 2] == 1.0  # phase 0: the centre tap alone (up to the normalisation)


def test_wine_sinf_accuracy():
    """The oracle's Wine sinf against double-precision sin: within one float ulp over the Lanczos arguments."""
    xs = np.linspace(-3 * math.pi, 3 * math.pi, 40001).astype(np.float32)
    for x in xs:
        s = O.wine_sinf(x)
        assert abs(s - math.sin(float(x))) <= 1.2e-7 * max(1.0, abs(s)), x


@pytest.mark.parametrize("sensor", [2, 4])
def test_yuv_matrix_host_matches_oracle(api, sensor):
    for neutral in ([0.5, 1.0, 0.6], [0.42, 1.0, 0.73], [1.0, 1.0, 1.0]):
        got = api.StereoImage.yuv_matrix(sensor, neutral)
        assert np.array_equal(got.view(np.uint32), O.yuv_matrix(sensor, neutral).view(np.uint32))


def test_gamma_encode_tracks_power():
    """GammaEncode's polynomials stay within 0.1 % of 255·|m|^(1/2.2) over the ISP range."""
    for m in (1e-4, 0.01, 0.18, 0.5, 0.9, 1.0, -0.3):
        want = math.copysign(255.0 * abs(m) ** (1 / 2.2), m)
        assert abs(O.gamma_encode(m) - want) <= 1e-3 * abs(want)
    assert O.gamma_encode(0.0) == 0.0


CASES = [  # (sw, sh, dw, dh, seed, angle): destinations inside the source, and larger ones with fill and clamped borders
    (200, 150, 180, 140, 0, 0.6),
    (200, 150, 240, 180, 1, -1.5),
    (97, 61, 120, 77, 2, 3.0),
    (64, 48, 64, 48, 3, 0.0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("sw,sh,dw,dh,seed,angle", CASES)
@pytest.mark.parametrize("gain", [1.0, 1.37])
def test_warp_f32_matches_oracle(api, sw, sh, dw, dh, seed, angle, gain):
    from lux_b200 import synth
    src = synth.isp_image(sw, sh, seed)
    ac = synth.aligned_calib(sw, sh, dw, dh, seed=seed, angle_deg=angle)
    got = api.StereoImage.warp(src, dw, dh, ac, gain=gain)
    want = O.warp_f32(src, gain, dw, dh, ac)
    assert np.array_equal(_bits(got), _bits(want))
    if dw > sw:
        assert (want[..., 3] == 0).any()  # the fill region is exercised


@pytest.mark.gpu
@pytest.mark.parametrize("sw,sh,dw,dh,seed,angle", CASES)
@pytest.mark.parametrize("sensor,neutral,gain", [(2, (0.5, 1.0, 0.6), 1.0), (4, (0.42, 1.0, 0.73), 0.81)])
def test_stereo_image_matches_oracle(api, sw, sh, dw, dh, seed, angle, sensor, neutral, gain):
    """The 8-bit stereo image and the YUV floats of the reference branch (StereoImageBuilder.cs:61-69)."""
    from lux_b200 import synth
    src = synth.isp_image(sw, sh, seed + 10)
    ac = synth.aligned_calib(sw, sh, dw, dh, seed=seed, angle_deg=angle)
    rgba, yuv = api.StereoImage.create(src, dw, dh, ac, sensor, neutral, gain=gain, keep_yuv=True)
    w_rgba, w_yuv = O.stereo_image(src, gain, dw, dh, ac, sensor, neutral)
    assert np.array_equal(rgba, w_rgba)
    assert np.array_equal(_bits(yuv), _bits(w_yuv))


@pytest.mark.gpu
def test_stereo_image_on_device_feeds_the_solve(api):
    """Device in, device out: the stereo image stays in HBM (a CUDA tensor) and equals the host-path result."""
    import torch
    from lux_b200 import synth
    src = synth.isp_image(160, 120, 5)
    ac = synth.aligned_calib(160, 120, 160, 120, seed=5)
    host, _ = api.StereoImage.create(src, 160, 120, ac, 2, (0.5, 1.0, 0.6))
    dev, _ = api.StereoImage.create(torch.from_numpy(src).cuda(), 160, 120, ac, 2, (0.5, 1.0, 0.6))
    assert dev.is_cuda and np.array_equal(dev.cpu().numpy(), host)


@pytest.mark.gpu
@pytest.mark.parametrize("sw,sh,dw,dh,seed,angle", CASES)
def test_rgba8_warp_matches_oracle(api, sw, sh, dw, dh, seed, angle):
    from lux_b200 import synth
    rng = np.random.default_rng(seed)
    src = rng.integers(0, 256, (sh, sw, 4), dtype=np.uint8)
    ac = synth.aligned_calib(sw, sh, dw, dh, seed=seed, angle_deg=angle)
    assert np.array_equal(api.Rgba8Warp.warp(src, dw, dh, ac), O.warp_rgba8(src, dw, dh, ac))


@pytest.mark.gpu
def test_warp_errors(api):
    """A subnormal r2 makes the reference index the lut at -2^31 (IndexOutOfRangeException): LUX_ERR_INDEX, on the host
    path as in the oracle; an empty source is refused."""
    from lux_b200 import synth
    src = synth.isp_image(40, 30, 1)
    ac = synth.aligned_calib(40, 30, 40, 30, seed=1)
    ac.sx = ac.sy = np.float32(1e-22)
    with pytest.raises(O.OracleError) as e:
        O.warp_f32(src, 1.0, 40, 30, ac)
    assert e.value.code == 7
    with pytest.raises(api.LuxIndexError):
        api.StereoImage.warp(src, 40, 30, ac)
    ok = synth.aligned_calib(40, 30, 40, 30, seed=1)
    with pytest.raises(api.LuxError):
        api.Rgba8Warp.warp(np.zeros((0, 4, 4), np.uint8), 8, 8, ok)


def _views(dw, dh, angle_deg, shift):
    """The reference camera's view (calib2) and a module's view (calibA) of the colour transfer: a rotation about the
    optical axis and a principal-point shift between them."""
    from lux_b200 import api
    f = np.float32(1.1 * dw)
    K2 = np.array([f, 0, dw / 2.0, 0, f, dh / 2.0, 0, 0, 1], np.float32)
    KA = np.array([f * 1.01, 0, dw / 2.0 + shift[0], 0, f * 1.01, dh / 2.0 + shift[1], 0, 0, 1], np.float32)
    a = np.deg2rad(angle_deg)
    R = np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]], np.float32).reshape(9)
    return (api.CalibData(K2, np.zeros(3, np.float32), np.eye(3, dtype=np.float32).reshape(9)),
            api.CalibData(KA, np.array([-25.0, 3.0, 0.0], np.float32), R))


@pytest.mark.gpu
@pytest.mark.parametrize("dw,dh,angle,shift,device", [(180, 140, 2.0, (6.0, -4.0), False), (120, 77, -4.0, (-30.0, 12.0), True),
                                                      (64, 48, 0.0, (0.0, 0.0), False), (96, 70, 0.5, (400.0, 0.0), False)])
def test_stereo_image_transfer_matches_oracle(api, dw, dh, angle, shift, device):
    """The non-reference branch (StereoImageBuilder.cs:71-77): the reference's YUV floats from the reference branch, then
    the module's image colour-matched to its crop; the 8-bit image and the transfer F bit for bit. The last case's crop
    lies outside the reference image (an empty crop: the identity transfer)."""
    import torch
    from lux_b200 import synth
    sw, sh = dw + 20, dh + 10
    neutral = (0.5, 1.0, 0.6)
    ref_src, mod_src = synth.isp_image(sw, sh, 21), synth.isp_image(sw, sh, 22)
    ac_ref = synth.aligned_calib(sw, sh, dw, dh, seed=21)
    ac_mod = synth.aligned_calib(sw, sh, dw, dh, seed=22, angle_deg=angle)
    ref_view, view = _views(dw, dh, angle, shift)
    _, ref_yuv = api.StereoImage.create(ref_src, dw, dh, ac_ref, 2, neutral, keep_yuv=True)
    _, w_ref_yuv = O.stereo_image(ref_src, 1.0, dw, dh, ac_ref, 2, neutral)
    assert np.array_equal(_bits(ref_yuv), _bits(w_ref_yuv))
    src = torch.from_numpy(mod_src).cuda() if device else mod_src
    ry = torch.from_numpy(ref_yuv).cuda() if device else ref_yuv
    got, F = api.StereoImage.create_transfer(src, dw, dh, ac_mod, 2, neutral, ry, ref_view, view, gain=0.87)
    want, wF = O.stereo_image_transfer(mod_src, 0.87, dw, dh, ac_mod, 2, neutral, w_ref_yuv, ref_view, view)
    assert np.array_equal(F.view(np.uint32), wF.view(np.uint32))
    got = got.cpu().numpy() if hasattr(got, "cpu") else got
    assert np.array_equal(got, want)
    if shift[0] > 100:
        assert np.array_equal(F, np.eye(4, dtype=np.float32))
    else:
        assert not np.array_equal(F, np.eye(4, dtype=np.float32))


@pytest.mark.gpu
def test_stereo_image_transfer_needs_reference(api):
    from lux_b200 import synth
    src = synth.isp_image(40, 30, 1)
    ac = synth.aligned_calib(40, 30, 40, 30, seed=1)
    rv, v = _views(40, 30, 0.0, (0.0, 0.0))
    with pytest.raises(api.LuxError, match="Empty reference yuv"):
        api.L.load()  # the library is there; the call refuses the missing reference image
        ctx = api.default_context()
        c, lut = ac.to_c()
        n = np.ascontiguousarray(np.array([0.5, 1.0, 0.6], np.float32))
        out = np.empty((30, 40, 4), np.uint8)
        ctx.check(ctx.lib.lux_stereo_image_transfer(ctx.handle, src.ctypes.data, 40, 30, 0, 1.0, api.ctypes.byref(c), 40, 30, 2,
                                                    n.ctypes.data, None, 0, api.ctypes.byref(rv.to_c()), api.ctypes.byref(v.to_c()),
                                                    out.ctypes.data, 0, None))
