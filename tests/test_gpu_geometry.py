"""GPU parity at the geometry the benchmark measures, through the C ABI, bit for bit against the oracle.

* the 1040x780 D=64 pair (the reference's CPU-runnable case) as a full frame, every fast aggregation form;
* the 13 MP pair's kernel geometry: a 4160-wide strip of 600 rows of the 12-bit generator at D=256, tile 64, so the
  cost kernel runs 4160-wide rows and the aggregation its full-width launch shapes;
* the reference's align-2 memory-pressure mode (DenseStereoSgm.cs:339-344) on ragged layers that follow a previous
  layer (RangeFromPrevious, DenseStereoSgm.cs:91-142): its IndexOutOfRangeException where a cap is not a multiple of 8,
  and its line-buffer layout where every cap is.
Raw costs, both aggregate volumes and the depth are compared as bits; the production form (no aggregates kept, images
filtered on the GPU) is checked on the depth."""
import os

import numpy as np
import pytest

from test_gpu_parity import SGM_FORMS, _compare_layer

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1  # the oracle's cost prepass runs on every host core (its aggregation is serial)


@pytest.fixture(scope="module")
def ctx():
    from lux_b200 import api
    c = api.Context(0)
    yield c
    c.close()


def _solve_both_forms(ctx, oracle, wl, forms, tag, cost_kernel):
    from lux_b200 import api
    filt = [oracle.box_filter3(im) for im in wl.images]
    ol = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True, threads=THREADS)
    for kernel in forms:
        gl = api.DenseLayer.compute(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True, keep_agg=True,
                                    sgm=kernel, ctx=ctx)
        try:
            assert gl.sgm_kernel == SGM_FORMS[kernel]
            assert gl.cost_kernel == cost_kernel
            _compare_layer(gl, ol, f"{tag} {kernel}")
        finally:
            gl.close()
        # the production form: unfiltered images in, the depth only
        gp = api.DenseLayer.compute(wl.images, wl.gray, wl.calibs, wl.near, wl.far, wl.params, prefilter=True, sgm=kernel,
                                    ctx=ctx)
        try:
            assert np.array_equal(gp.Depth.view(np.uint32), ol["Depth"].view(np.uint32)), f"{tag} {kernel} production"
        finally:
            gp.close()


def test_pair_1040x780_d64_full_frame(ctx, oracle):
    from lux_b200 import synth
    wl = synth.rectified_pair(1040, 780, 64, seed=0, tile=64)
    _solve_both_forms(ctx, oracle, wl, ["fused", "split", "wave"], "1040x780 D64", cost_kernel=3)


def test_pair_13mp_geometry_strip(ctx, oracle):
    from lux_b200 import synth
    wl = synth.rectified_pair(4160, 600, 256, seed=1, bits=12, tile=64)
    _solve_both_forms(ctx, oracle, wl, ["split", "fused", "wave"], "4160x600 D256", cost_kernel=3)


def test_align2_ragged_layer_index_error(ctx, oracle):
    """With align 2 a ragged layer's caps are rounded to 2 planes, but the reference's Pixel still walks the aggregates
    in blocks of 8 (DenseStereoSgm.cs:300-313) and indexes past Agg[pi] for a cap that is not a multiple of 8: the C#
    throws IndexOutOfRangeException. The oracle and the library both report it (LUX_ERR_INDEX)."""
    from lux_b200 import api, synth
    cap = synth.capture(416, 312, 3, seed=12, f=330.0)
    filt = [oracle.box_filter3(im) for im in cap.images]
    params = api.StereoParams.l16_pyramid()
    ol0 = oracle.layer(filt, cap.gray, cap.calibs, cap.near, cap.far, params[0], index=0, threads=THREADS)
    gl0 = api.DenseLayer.compute(filt, cap.gray, cap.calibs, cap.near, cap.far, params[0], index=0, ctx=ctx)
    try:
        with pytest.raises(oracle.OracleError) as eo:
            oracle.layer(filt, cap.gray, cap.calibs, cap.near, cap.far, params[1], index=1, align=2, prev=ol0)
        assert eo.value.code == 7
        with pytest.raises(api.LuxIndexError):
            api.DenseLayer.compute(filt, cap.gray, cap.calibs, cap.near, cap.far, params[1], index=1, align=2, prev=gl0,
                                   ctx=ctx).close()
    finally:
        gl0.close()


@pytest.mark.parametrize("level,lo_hi", [(2, (2, 8)), (3, (5, 11)), (4, (3, 17))])
def test_align2_layout_bit_exact(ctx, oracle, level, lo_hi):
    """The align-2 layout where the reference runs through: a previous layer whose depth alternates between two planes in
    a checkerboard gives every pixel the same range (count a multiple of 8), so no cap overruns, while MaxHi is rounded
    to 2 instead of 8 and the exact replay's line buffer (4·MaxHi + 5 words a slot) and its initial RangeC (= align) take
    the align-2 values. The previous layer is resumed from the depth map (lux_layer_from_depth)."""
    from lux_b200 import api, synth
    cap = synth.capture(640, 480, 3, seed=20 + level, f=500.0)
    filt = [oracle.box_filter3(im) for im in cap.images]
    p = api.StereoParams.l16_pyramid()[level]
    max_hi = {}
    for align in (2, 8):
        planes = oracle.planes(cap.near, cap.far, cap.calibs, p.plane_density, align)
        pw, ph = (640 + 2 * p.scale - 1) // (2 * p.scale), (480 + 2 * p.scale - 1) // (2 * p.scale)
        yy, xx = np.mgrid[0:ph, 0:pw]
        depth = np.where((xx + yy) % 2 == 0, planes[lo_hi[0]], planes[lo_hi[1]]).astype(np.float32)
        skip = np.zeros((ph, pw), np.uint8)
        ol = oracle.layer(filt, cap.gray, cap.calibs, cap.near, cap.far, p, index=level, align=align,
                          prev={"W": pw, "H": ph, "Depth": depth, "Skip": skip}, keep_pass1=True, threads=THREADS)
        prev = api.DenseLayer.from_depth(depth, skip, ctx=ctx)
        gl = api.DenseLayer.compute(filt, cap.gray, cap.calibs, cap.near, cap.far, p, index=level, align=align, prev=prev,
                                    keep_pass1=True, keep_agg=True, ctx=ctx)
        try:
            assert gl.sgm_kernel == SGM_FORMS["replay"] and gl.Align == align
            assert np.all(ol["Cap"] % 8 == 0) and np.all(ol["Count"] == lo_hi[1] - lo_hi[0] + 2)
            _compare_layer(gl, ol, f"align {align} level {level}")
            max_hi[align] = gl.MaxHi
        finally:
            gl.close()
            prev.close()
    assert max_hi[2] != max_hi[8]  # the two layouts differ
