"""GPU parity: the CUDA path through the C ABI against the oracle, bit for bit (integer stages) and within 1e-5
relative (the float upsample; it is checked for exact equality as well)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from lux_b200 import api
    return api.Context(0)


def _filtered(oracle, images):
    return [oracle.box_filter3(im) for im in images]


@pytest.mark.parametrize("h,w", [(1, 1), (2, 2), (3, 7), (41, 67), (480, 640)])
def test_box_filter(ctx, oracle, h, w):
    from lux_b200 import api
    img = np.random.default_rng(h + w).integers(0, 256, (h, w, 4), dtype=np.uint8)
    assert np.array_equal(api.DenseStereo.box_filter3(img, ctx=ctx), oracle.box_filter3(img))


def _compare_layer(gl, ol, tag):
    assert (gl.W, gl.H, gl.n_planes, gl.MinLo, gl.MaxHi) == (ol["W"], ol["H"], ol["n_planes"], ol["MinLo"], ol["MaxHi"]), tag
    assert np.array_equal(gl.Planes, ol["Planes"]), tag
    assert np.array_equal(gl.Start, ol["Start"]) and np.array_equal(gl.Count, ol["Count"]), tag
    assert np.array_equal(gl.Cap, ol["Cap"]) and np.array_equal(gl.Skip, ol["Skip"]), tag
    assert np.array_equal(gl.Offsets, ol["Offsets"]), tag
    assert np.array_equal(gl.Guidance, ol["Guidance"]), tag
    comp = (ol["Skip"].reshape(-1) == 0)
    off, cap = ol["Offsets"][:-1], ol["Cap"].reshape(-1).astype(np.int64)
    mask = np.repeat(comp, cap)
    assert np.array_equal(gl.Raw[mask], ol["Raw"][mask]), tag + " raw"
    if ol["AggPass1"] is not None:
        assert np.array_equal(gl.AggPass1, ol["AggPass1"]), tag + " agg pass1"
    assert np.array_equal(gl.Agg, ol["Agg"]), tag + " agg"
    assert np.array_equal(gl.Depth.view(np.uint32), ol["Depth"].view(np.uint32)), tag + " depth"


# (W, H, D, T): K = T - ((W-1) mod T) revisit rows per band takes the values 1, T and in between; D covers the 2-, 4- and
# 8-plane lane widths with and without padding lanes; H covers partial last bands and partial last CTA bands.
UNIFORM_CASES = [(48, 40, 16, 8), (65, 49, 16, 4), (160, 120, 32, 16), (257, 93, 64, 64), (100, 77, 24, 8), (130, 70, 96, 16),
                 (200, 35, 136, 8), (71, 66, 256, 64), (33, 17, 40, 2), (64, 9, 192, 32)]


SGM_FORMS = {"fused": 1, "split": 2, "replay": 0, "wave": 3}  # kernel -> lux_layer_info.sgm_kernel


def _sgm_args(kernel):
    return dict(force_replay=True) if kernel == "replay" else dict(sgm=kernel)


@pytest.mark.parametrize("kernel", ["fused", "split", "wave", "replay"])
@pytest.mark.parametrize("w,h,d,tile", UNIFORM_CASES)
def test_uniform_layer_bit_exact(ctx, oracle, w, h, d, tile, kernel):
    from lux_b200 import api, synth
    wl = synth.rectified_pair(w, h, d, seed=w + h, tile=tile)
    filt = _filtered(oracle, wl.images)
    ol = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True)
    gl = api.DenseLayer.compute(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True, keep_agg=True,
                                ctx=ctx, **_sgm_args(kernel))
    try:
        assert gl.sgm_kernel == SGM_FORMS[kernel]
        assert gl.cost_kernel == (3 if d % 8 == 0 else 0)  # a rectified grey pair: the shared-column axis cost kernel
        _compare_layer(gl, ol, f"{w}x{h} D{d} T{tile} {kernel}")
    finally:
        gl.close()


@pytest.mark.parametrize("w,h,d,tile", [(50, 23, 24, 3), (41, 30, 16, 5), (150, 140, 16, 96)])
def test_replay_barrier_form_bit_exact(ctx, oracle, w, h, d, tile):
    """Tiles the row hand-over does not take (odd tiles, whose bands' boundary rows share a line-buffer half, and tiles
    past 64 rows) step with a block barrier: the exact replay, bit for bit."""
    from lux_b200 import api, synth
    wl = synth.rectified_pair(w, h, d, seed=w * h, tile=tile)
    filt = _filtered(oracle, wl.images)
    ol = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True)
    gl = api.DenseLayer.compute(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True, keep_agg=True,
                                ctx=ctx, force_replay=True)
    try:
        assert gl.sgm_kernel == SGM_FORMS["replay"]
        _compare_layer(gl, ol, f"{w}x{h} D{d} T{tile} replay")
    finally:
        gl.close()


@pytest.mark.parametrize("w,h,d,tile", [(600, 40, 264, 8), (520, 48, 400, 16), (700, 30, 552, 4), (300, 20, 768, 2)])
def test_wide_uniform_layer_fused_bit_exact(ctx, oracle, w, h, d, tile):
    """Uniform layers past 256 planes (the L16 pyramid's first layer has 552) on the fused fast kernel, a lane holding 16
    or 24 planes with the padding octets of the last lane masked; a chain or wave form asked for runs fused there."""
    from lux_b200 import api, synth
    wl = synth.rectified_pair(w, h, d, seed=d + tile, tile=tile)
    filt = _filtered(oracle, wl.images)
    ol = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True)
    for sgm in ("auto", "split"):
        gl = api.DenseLayer.compute(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True, keep_agg=True,
                                    sgm=sgm, ctx=ctx)
        try:
            assert gl.n_planes == d and gl.sgm_kernel == SGM_FORMS["fused"]
            _compare_layer(gl, ol, f"{w}x{h} D{d} T{tile} fused ({sgm})")
        finally:
            gl.close()


@pytest.mark.parametrize("w,h,d,tile", [(120, 90, 24, 20), (150, 100, 16, 34), (140, 130, 16, 50)])
def test_replay_partial_last_part_bit_exact(ctx, oracle, w, h, d, tile):
    """The row form splits a band into parts of min(8, T/2) rows; these tiles leave a shorter last part (T = 20: 8 + 8 +
    4; T = 34: four parts of 8 and one of 2; T = 50: six of 8 and one of 2), whose last row publishes to the next band."""
    from lux_b200 import api, synth
    wl = synth.rectified_pair(w, h, d, seed=w + h, tile=tile)
    filt = _filtered(oracle, wl.images)
    ol = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True)
    gl = api.DenseLayer.compute(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True, keep_agg=True,
                                ctx=ctx, force_replay=True)
    try:
        assert gl.sgm_kernel == SGM_FORMS["replay"]
        _compare_layer(gl, ol, f"{w}x{h} D{d} T{tile} replay")
    finally:
        gl.close()


@pytest.mark.parametrize("kernel", ["fused", "split", "wave"])
def test_uniform_fast_depth_without_kept_aggregates(ctx, oracle, kernel):
    """The production form (no Agg kept, WTA fused into the last kernel of pass -1) gives the same depth."""
    from lux_b200 import api, synth
    wl = synth.rectified_pair(300, 170, 64, seed=9, tile=64)
    filt = _filtered(oracle, wl.images)
    ol = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params)
    gl = api.DenseLayer.compute(wl.images, wl.gray, wl.calibs, wl.near, wl.far, wl.params, prefilter=True, sgm=kernel, ctx=ctx)
    try:
        assert gl.sgm_kernel == SGM_FORMS[kernel]
        assert np.array_equal(gl.Depth.view(np.uint32), ol["Depth"].view(np.uint32))
        with pytest.raises(api.LuxError):
            gl.Agg
    finally:
        gl.close()


def test_multicamera_colour_layer_bit_exact(ctx, oracle):
    """Three colour cameras, translated in x and y: the general projection with half-pixel resampling."""
    from lux_b200 import api, synth
    cap = synth.capture(120, 90, 3, seed=11, f=90.0, baseline_mm=(20.0, 60.0))
    filt = _filtered(oracle, cap.images)
    p = api.StereoParams(scale=1, tile=8, skip_mode=0, plane_density=2.0)
    ol = oracle.layer(filt, cap.gray, cap.calibs, cap.near, cap.far, p, keep_pass1=True)
    gl = api.DenseLayer.compute(filt, cap.gray, cap.calibs, cap.near, cap.far, p, keep_pass1=True, keep_agg=True, ctx=ctx)
    try:
        assert gl.cost_kernel == 1
        _compare_layer(gl, ol, "3cam")
    finally:
        gl.close()


@pytest.mark.parametrize("focal,skip,w", [(1.0, 0, 157), (1.0, 2, 211), (1.3, 0, 130), (0.77, 2, 97), (1.0, 0, 30),
                                           (1.0, 0, 124), (1.0, 2, 253), (1.3, 2, 125)])
def test_axis_pair_shared_columns(ctx, oracle, focal, skip, w):
    """The shared-column grey cost kernel: widths below, at and past its 62-pixel warp runs, skipped pixels,
    and a second camera with another focal length, where neighbouring target positions step by more (1.3) or less
    (0.77) than one pixel so that lanes compute their own block columns."""
    from lux_b200 import api, synth
    h, d = 61, 48
    wl = synth.rectified_pair(w, h, d, seed=w + 3, tile=8)
    f2 = np.float32(1000.0 * focal)
    cal = list(wl.calibs)
    cal[1] = api.CalibData(np.array([f2, 0, w / 2.0 + 1.5, 0, f2, h / 2.0 - 0.5, 0, 0, 1], np.float32),
                           np.array([-100.0, 0, 0], np.float32), np.eye(3, dtype=np.float32).reshape(9))
    p = api.StereoParams(scale=1, tile=8, skip_mode=skip, plane_density=1.0)
    filt = _filtered(oracle, wl.images)
    ol = oracle.layer(filt, wl.gray, cal, wl.near, wl.far, p, keep_pass1=True)
    gl = api.DenseLayer.compute(filt, wl.gray, cal, wl.near, wl.far, p, keep_pass1=True, keep_agg=True, ctx=ctx)
    try:
        assert gl.cost_kernel == (3 if gl.n_planes % 8 == 0 else 0)
        _compare_layer(gl, ol, f"shared columns f{focal} skip{skip} w{w}")
    finally:
        gl.close()


def test_axis_pair_scale2_grey(ctx, oracle):
    """A grey axis-aligned pair at scale 2 (blocks of neighbouring pixels do not overlap): the per-row axis kernel."""
    from lux_b200 import api, synth
    wl = synth.rectified_pair(180, 120, 64, seed=8, tile=8)
    p = api.StereoParams(scale=2, tile=8, skip_mode=0, plane_density=1.0)
    filt = _filtered(oracle, wl.images)
    ol = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, p, keep_pass1=True)
    gl = api.DenseLayer.compute(filt, wl.gray, wl.calibs, wl.near, wl.far, p, keep_pass1=True, keep_agg=True, ctx=ctx)
    try:
        assert gl.cost_kernel == (2 if gl.n_planes % 8 == 0 else 0)
        _compare_layer(gl, ol, "axis grey scale 2")
    finally:
        gl.close()


@pytest.mark.parametrize("kernel", ["fused", "split", "wave"])
def test_axis_pair_colour_bit_exact(ctx, oracle, kernel):
    """A rectified colour pair: the axis-aligned cost kernel with the colour block (the tests above are grey)."""
    from lux_b200 import api, synth
    wl = synth.rectified_pair(140, 90, 48, seed=41, tile=8)
    rng = np.random.default_rng(41)
    imgs = []
    for im in wl.images:
        im = im.copy()
        im[..., 1] = np.clip(im[..., 0].astype(np.int32) // 2 + rng.integers(0, 60, im.shape[:2]), 0, 255)
        im[..., 2] = np.clip(255 - im[..., 0].astype(np.int32) + rng.integers(0, 40, im.shape[:2]), 0, 255)
        imgs.append(im)
    gray = [0, 0]
    filt = _filtered(oracle, imgs)
    ol = oracle.layer(filt, gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True)
    gl = api.DenseLayer.compute(filt, gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True, keep_agg=True, sgm=kernel,
                                ctx=ctx)
    try:
        assert gl.sgm_kernel == SGM_FORMS[kernel]
        assert gl.cost_kernel == 2
        _compare_layer(gl, ol, "axis colour")
    finally:
        gl.close()


@pytest.mark.parametrize("kernel", ["fused", "split", "wave", "replay"])
def test_uniform_layer_with_skip_mask(ctx, oracle, kernel):
    """A first layer with SkipMode 2: skipped pixels aggregate raw 0 (DenseStereoSgm.cs:242)."""
    from lux_b200 import api, synth
    wl = synth.rectified_pair(150, 96, 32, seed=21, tile=16)
    p = api.StereoParams(**{**wl.params.__dict__, "skip_mode": 2})
    filt = _filtered(oracle, wl.images)
    ol = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, p, keep_pass1=True)
    gl = api.DenseLayer.compute(filt, wl.gray, wl.calibs, wl.near, wl.far, p, keep_pass1=True, keep_agg=True, ctx=ctx,
                                **_sgm_args(kernel))
    try:
        assert gl.Skip.any()
        assert gl.sgm_kernel == SGM_FORMS[kernel]
        _compare_layer(gl, ol, f"skip {kernel}")
    finally:
        gl.close()


@pytest.mark.parametrize("w,h", [(2080, 1560), (1040, 780), (191, 127), (127, 191), (95, 97), (33, 25)])
def test_skip_mask_on_the_device(ctx, oracle, w, h):
    """SkipMode 2's mask (DenseStereoSgm.cs:65-87), made on the device from the generator stream every 64x64 tile
    restarts: the pyramid's two finest layer sizes, last tiles that absorb a remainder of at most 32 pixels or stand on
    their own past it, and a layer smaller than one tile (eight planes, so the solve itself is cheap)."""
    from lux_b200 import api, synth
    wl = synth.rectified_pair(w, h, 8, seed=5, tile=8)
    p = api.StereoParams(**{**wl.params.__dict__, "skip_mode": 2})
    gl = api.DenseLayer.compute(wl.images, wl.gray, wl.calibs, wl.near, wl.far, p, prefilter=True, ctx=ctx)
    try:
        assert np.array_equal(gl.Skip.reshape(h, w), oracle.skip_mask(2, w, h).reshape(h, w))
    finally:
        gl.close()


@pytest.mark.parametrize("kernel", ["fused", "split", "wave"])
@pytest.mark.parametrize("n_cams,colour", [(4, False), (6, True), (6, False)])
def test_multicamera_layers_bit_exact(ctx, oracle, n_cams, colour, kernel):
    """Grey and colour layers with 3 and 5 other cameras (the per-camera cost loop with its camera count at run time)."""
    from lux_b200 import api, synth
    cap = synth.capture(96, 72, n_cams, seed=30 + n_cams, f=72.0, baseline_mm=(15.0, 50.0), colour=colour)
    filt = _filtered(oracle, cap.images)
    p = api.StereoParams(scale=1, tile=8, skip_mode=0, plane_density=2.0)
    ol = oracle.layer(filt, cap.gray, cap.calibs, cap.near, cap.far, p, keep_pass1=True)
    gl = api.DenseLayer.compute(filt, cap.gray, cap.calibs, cap.near, cap.far, p, keep_pass1=True, keep_agg=True, sgm=kernel,
                                ctx=ctx)
    try:
        assert gl.sgm_kernel == SGM_FORMS[kernel]
        assert gl.cost_kernel == 1  # lanes over pixels for any number of other cameras
        _compare_layer(gl, ol, f"{n_cams}cam colour={colour}")
    finally:
        gl.close()


@pytest.mark.parametrize("kernel", ["fused", "split", "wave"])
def test_module_capture_bit_exact(ctx, oracle, kernel):
    """A batched capture: 10 module cameras with their own crops, focal scales and disparity ranges, fused at cost level
    into one layer (the reference's multi-view sum, DenseStereo.cs:242-291)."""
    from lux_b200 import api, synth
    mc = synth.module_capture(96, 72, seed=3, size_scale=0.002, tile=8)
    assert len({s for s in mc.sizes}) > 5
    filt = _filtered(oracle, mc.images)
    ol = oracle.layer(filt, mc.gray, mc.calibs, mc.near, mc.far, mc.params, keep_pass1=True)
    gl = api.DenseLayer.compute(filt, mc.gray, mc.calibs, mc.near, mc.far, mc.params, keep_pass1=True, keep_agg=True, sgm=kernel,
                                ctx=ctx)
    try:
        assert gl.sgm_kernel == SGM_FORMS[kernel] and gl.cost_kernel == 1
        _compare_layer(gl, ol, f"module capture {kernel}")
    finally:
        gl.close()


@pytest.mark.parametrize("kernel", ["fused", "split", "wave"])
def test_pyramid_bit_exact(ctx, oracle, kernel):
    """DenseStereoPyramid.Run: six L16 layers (ragged ranges, skip masks, align choice) against the oracle."""
    from lux_b200 import api, synth
    cap = synth.capture(416, 312, 3, seed=5, f=330.0)
    ol = oracle.pyramid(cap.images, cap.gray, cap.calibs, cap.near, cap.far, keep_pass1=True)
    gls = api.DenseStereoPyramid.run(cap.images, cap.gray, cap.calibs, cap.near, cap.far, keep_pass1=True, keep_agg=True,
                                     sgm=kernel, ctx=ctx)
    try:
        assert gls[0].sgm_kernel == SGM_FORMS[kernel]  # the first layer is uniform; the others take the replay
        for i in range(6):
            _compare_layer(gls[i], ol[i], f"L{i}")
    finally:
        for g in gls:
            g.close()


@pytest.mark.parametrize("pw,ph", [(52, 39), (208, 156)])
def test_upsample(ctx, oracle, pw, ph):
    from lux_b200 import api
    rng = np.random.default_rng(pw)
    depth = rng.uniform(300.0, 6000.0, (ph, pw)).astype(np.float32)
    guide = rng.integers(0, 256, (2 * ph, 2 * pw, 4), dtype=np.uint8)
    conf = rng.uniform(0, 1, (ph, pw)).astype(np.float32)
    od, oc = oracle.upsample(depth, pw, ph, guide, pw, ph, prev_conf=conf)
    r = api.DenseUpsampleLayer.run(depth, pw, ph, guide, pw, ph, prev_confidence=conf, ctx=ctx)
    rel = np.abs(r.Depth - od) / np.abs(od)
    assert rel.max() <= 1e-5
    assert np.array_equal(r.Depth.view(np.uint32), od.view(np.uint32))
    assert np.array_equal(r.Confidence.view(np.uint32), oc.view(np.uint32))


def test_upsample_size_error(ctx):
    from lux_b200 import api
    depth = np.ones((10, 12), np.float32) * 1000
    guide = np.zeros((20, 24, 4), np.uint8)
    with pytest.raises(api.InvalidOperationError):
        api.DenseUpsampleLayer.run(depth, 12, 10, guide, 13, 10, ctx=ctx)


def test_layer_errors(ctx):
    from lux_b200 import api, synth
    wl = synth.rectified_pair(32, 24, 16, seed=1, tile=8)
    with pytest.raises(api.InvalidOperationError):
        api.DenseLayer.compute(wl.images, wl.gray, wl.calibs, 500.0, 100.0, wl.params, ctx=ctx)
    bad = api.StereoParams(scale=1, tile=8, skip_mode=3, plane_density=1.0)
    with pytest.raises(api.NotSupportedError):
        api.DenseLayer.compute(wl.images, wl.gray, wl.calibs, wl.near, wl.far, bad, ctx=ctx)


@pytest.mark.parametrize("bits,w,h,stride", [(12, 333, 47, 333), (12, 4160, 20, 4200), (10, 65, 9, 70), (16, 31, 5, 31)])
def test_image_from_grey16(ctx, bits, w, h, stride):
    """u16 grey samples made into the reference's byte domain on the GPU, host and device sources, equal to the mapping
    the 12-bit workloads apply on the host ((v + 8) >> 4 saturated for 12 bits)."""
    import torch
    from lux_b200 import api, synth
    rng = np.random.default_rng(bits * w)
    full = rng.integers(0, 1 << bits, (h, stride), dtype=np.uint16)
    full[0, : min(w, 8)] = [(1 << bits) - 1, 0, 7, 8, 4087, 4088, 4095, 1][: min(w, 8)]  # rounding and saturation edges
    sh = bits - 8
    want = synth.gray_rgba(np.clip((full[:, :w].astype(np.int64) + (1 << (sh - 1))) >> sh, 0, 255).astype(np.uint8))
    if bits == 12:
        assert np.array_equal(want, synth.gray_rgba(synth.to_u8(full[:, :w], 12)))
    host = api.image_from_grey16(np.ascontiguousarray(full[:, :w]), bits, ctx=ctx)
    ctx.check(ctx.lib.lux_sgm_sync(ctx.handle))
    assert np.array_equal(host.cpu().numpy(), want)
    dev = torch.from_numpy(full.view(np.int16)).cuda()[:, :w]  # a strided device view
    assert dev.stride(0) == stride
    out = api.image_from_grey16(dev, bits, ctx=ctx)
    ctx.check(ctx.lib.lux_sgm_sync(ctx.handle))
    assert np.array_equal(out.cpu().numpy(), want)


def test_pyramid_index_error_parity(ctx, oracle):
    """A capture whose finest layer makes the reference write past the end of its line buffer (a last-column pixel of
    the second half whose range spills beyond the buffer, DenseStereoSgm.cs:300-313, an IndexOutOfRangeException in the
    C#): the oracle and the GPU pyramid both report LUX_ERR_INDEX."""
    from lux_b200 import api, synth
    cap = synth.capture(520, 390, 5, seed=3)
    with pytest.raises(oracle.OracleError) as eo:
        oracle.pyramid(cap.images, cap.gray, cap.calibs, cap.near, cap.far, threads=4)
    assert eo.value.code == 7
    with pytest.raises(api.LuxIndexError):
        for g in api.DenseStereoPyramid.run(cap.images, cap.gray, cap.calibs, cap.near, cap.far, ctx=ctx):
            g.close()
