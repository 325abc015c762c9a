"""CPU checks of the oracle (the CPU restatement of the reference) and of its pins."""
import hashlib
import json
import os
import re
import struct

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _header_tables():
    src = open(os.path.join(ROOT, "lux_b200", "csrc", "intel_approx_tables.h")).read()
    out = {}
    for name, body in re.findall(r"static const uint32_t (\w+)\[4096\] = \{([^}]*)\}", src):
        out[name] = [int(v, 16) for v in re.findall(r"0x([0-9a-f]+)u", body)]
    return out


def test_intel_tables_match_reference_digests():
    """The regenerated rcpss/rsqrtss tables equal IntelApprox.Tables.cs (RcpTable, RsqrtOddTable = exponent 127,
    RsqrtEvenTable = exponent 128), compared by SHA-256 against the digests taken from the reference."""
    gold = json.load(open(os.path.join(GOLDEN, "intel_tables.json")))["tables"]
    mine = _header_tables()
    pairs = {"RcpTable": "lux_rcp_table", "RsqrtOddTable": "lux_rsqrt_table_e127", "RsqrtEvenTable": "lux_rsqrt_table_e128"}
    for ref_name, my_name in pairs.items():
        vals = mine[my_name]
        assert len(vals) == gold[ref_name]["count"] == 4096
        assert hashlib.sha256(struct.pack("<4096I", *vals)).hexdigest() == gold[ref_name]["sha256"], ref_name


def test_mt19937_known_answer(oracle):
    """std::mt19937 default seed: the 10000th output is 4123659995 (C++ standard, [rand.predef])."""
    s = oracle.mt19937_stream(5489, 10000)
    assert int(s[-1]) == 4123659995


@pytest.mark.parametrize("h,w", [(1, 1), (1, 5), (2, 2), (3, 7), (17, 9), (40, 33)])
def test_box_filter_vector_equals_scalar(oracle, h, w):
    """BoxFilter3's 8-lane form and its scalar twin (DenseStereo.cs:93-159) agree."""
    rng = np.random.default_rng(h * 100 + w)
    img = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    assert (oracle.box_filter3(img) == oracle.box_filter3(img, scalar=True)).all()


def test_oracle_regression_fixture(oracle):
    """The oracle reproduces its committed outputs for a small seeded pair (guards the restatement against drift)."""
    from lux_b200 import synth
    g = np.load(os.path.join(GOLDEN, "oracle_small.npz"))
    wl = synth.rectified_pair(48, 40, 16, seed=3, tile=8)
    assert (wl.images[0] == g["img0"]).all() and (wl.images[1] == g["img1"]).all()
    filt = [oracle.box_filter3(im) for im in wl.images]
    L = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True)
    for k in ("raw", "agg_pass1", "agg", "depth", "planes"):
        key = {"raw": "Raw", "agg_pass1": "AggPass1", "agg": "Agg", "depth": "Depth", "planes": "Planes"}[k]
        assert np.array_equal(L[key], g[k]), k


def test_oracle_depth_tracks_ground_truth(oracle):
    from lux_b200 import synth
    wl = synth.rectified_pair(160, 120, 32, seed=1, tile=16)
    filt = [oracle.box_filter3(im) for im in wl.images]
    L = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params)
    disp = 1000.0 * 100.0 / L["Depth"]
    assert (np.abs(disp - wl.disparity) < 1.5).mean() > 0.8


def test_planes_errors(oracle):
    from lux_b200 import synth
    c = synth.rectified_calibs(1000.0, 10.0, 10.0, 100.0)
    with pytest.raises(oracle.OracleError) as e:
        oracle.planes(500.0, 200.0, c, 1.0, 8)
    assert e.value.code == 1
    with pytest.raises(oracle.OracleError) as e:
        oracle.planes(-1.0, 200.0, c, 1.0, 8)
    assert e.value.code == 2
    same = [c[0], c[0]]
    with pytest.raises(oracle.OracleError) as e:
        oracle.planes(200.0, 640000.0, same, 1.0, 8)
    assert e.value.code == 3


def test_skip_mask_one_per_cell(oracle):
    m = oracle.skip_mask(2, 130, 70)
    cells = (m[:70, :130] == 0).reshape(35, 2, 65, 2).sum(axis=(1, 3))
    assert (cells == 1).all()


def _nearest16(scale, off, n_out, n_src):
    """ImageResample0's 16.16 source index (DepthCache.cs:42-51), int32 wrap-around, clamped to the source."""
    s16, o16 = int(scale * 65536.0), int(off * 65536.0)
    v = (np.arange(n_out, dtype=np.int64) * s16 + o16) & 0xFFFFFFFF
    v = np.where(v >= 1 << 31, v - (1 << 32), v) >> 16
    return np.clip(v, 0, n_src - 1)


def test_depth_cache_set_properties(oracle):
    """Set (DepthCache.cs:136-143): each cache pixel is its nearest source pixel after two rcpps round trips (each within
    1.5·2^-12 relative, so within 7.5e-4), clipped to 1e5; at equal dims the resample is the identity."""
    rng = np.random.default_rng(1)
    d = np.exp(rng.uniform(np.log(300.0), np.log(3e5), (57, 83))).astype(np.float32)
    same = oracle.depth_cache_set(d, 83, 57)
    assert np.all(np.abs(same - np.minimum(d, 1e5)) <= 7.5e-4 * np.minimum(d, 1e5))
    cw, ch = 130, 41
    got = oracle.depth_cache_set(d, cw, ch)
    ys, xs = _nearest16(57 / ch, 0.0, ch, 57), _nearest16(83 / cw, 0.0, cw, 83)
    near = np.minimum(d[np.ix_(ys, xs)], 1e5)
    assert np.all(np.abs(got - near) <= 7.5e-4 * near)
    assert got.max() <= 1e5
    with pytest.raises(oracle.OracleError) as e:
        oracle.depth_cache_set(d, 0, 5)
    assert e.value.code == 15


def test_depth_cache_fetch_properties(oracle):
    """Fetch (DepthCache.cs:161-239): the plain window at scale 1; elsewhere the nearest window pixel (offsets from
    ((float)x0 + 0.5f)·sx − ⌊x0·sx⌋) within 2 ulp after the reciprocal round trip; the reference's ROI checks."""
    rng = np.random.default_rng(2)
    img = rng.uniform(500.0, 9e4, (96, 128)).astype(np.float32)
    assert np.array_equal(oracle.depth_cache_fetch(img, (5, 7, 50, 60), (128, 96)), img[7:60, 5:50])
    for rect, dims in (((3, 2, 40, 30), (64, 48)), ((10, 11, 200, 150), (256, 192)), ((0, 0, 97, 71), (97, 71))):
        x0, y0, x1, y1 = rect
        sx, sy = 128 / dims[0], 96 / dims[1]
        wx0, wy0 = max(int(np.floor(x0 * sx)), 0), max(int(np.floor(y0 * sy)), 0)
        wx1, wy1 = min(int(np.ceil(x1 * sx)), 128), min(int(np.ceil(y1 * sy)), 96)
        offx = float(np.float32(x0) + np.float32(0.5)) * sx - wx0
        offy = float(np.float32(y0) + np.float32(0.5)) * sy - wy0
        xs = wx0 + _nearest16(sx, offx, x1 - x0, wx1 - wx0)
        ys = wy0 + _nearest16(sy, offy, y1 - y0, wy1 - wy0)
        got = oracle.depth_cache_fetch(img, rect, dims)
        want = img[np.ix_(ys, xs)]
        assert np.all(np.abs(got.view(np.int32) - want.view(np.int32)) <= 2), rect
    for rect in ((4, 4, 4, 8), (-1, 0, 3, 3), (0, 0, 129, 5)):
        with pytest.raises(oracle.OracleError) as e:
            oracle.depth_cache_fetch(img, rect, (128, 96))
        assert e.value.code == 14


def _rcp_bits_np(b, table):
    """IntelApprox.RcpBits (IntelApprox.cs:21-29) on uint32 arrays."""
    b = b.astype(np.uint64)
    sign, e, m = b & 0x80000000, (b >> 23) & 0xFF, b & 0x7FFFFF
    r = table[(m >> 11).astype(np.int64)].astype(np.uint64)
    re = ((r >> 23) & 0xFF).astype(np.int64) - (e.astype(np.int64) - 127)
    out = sign | (np.clip(re, 0, 255).astype(np.uint64) << 23) | (r & 0x7FFFFF)
    out = np.where(re <= 0, sign, out)
    out = np.where(e == 0, sign | 0x7F800000, out)
    out = np.where(e == 0xFF, np.where(m != 0, b | 0x400000, sign), out)
    return out.astype(np.uint32)


def test_depth_cache_composite_rcp():
    """The one-lookup rcpps(rcpps(v)) of the depth cache's Set kernel (comp[i] = (E(j) - E(i))·2^23 + M(j), j = M(i) >> 11,
    added to v's sign and exponent bits) equals the two table steps for every table index, sign and exponent 3..250."""
    t = np.array(_header_tables()["lux_rcp_table"], np.uint64)
    ti = t
    tj = t[((ti & 0x7FFFFF) >> 11).astype(np.int64)]
    comp = (((tj >> 23) & 0xFF).astype(np.int64) - ((ti >> 23) & 0xFF).astype(np.int64)) * (1 << 23) + (tj & 0x7FFFFF).astype(np.int64)
    rng = np.random.default_rng(4)
    i = np.tile(np.arange(4096, dtype=np.uint64), 248 * 2)
    e = np.repeat(np.arange(3, 251, dtype=np.uint64), 4096 * 2)
    s = np.tile(np.repeat(np.array([0, 1], np.uint64), 4096), 248)
    b = ((s << 31) | (e << 23) | (i << 11) | rng.integers(0, 2048, i.size).astype(np.uint64)).astype(np.uint32)
    two = _rcp_bits_np(_rcp_bits_np(b, t), t)
    one = ((b.astype(np.int64) & 0xFF800000) + comp[i.astype(np.int64)]) & 0xFFFFFFFF
    assert np.array_equal(one.astype(np.uint32), two)


def _layer_cases():
    """Uniform grey pairs (T 4-64, D 16-64), a colour multi-camera layer and ragged layers after a previous layer."""
    from lux_b200 import api, synth
    cases = []
    for (w, h, d, t) in [(48, 40, 16, 8), (65, 33, 32, 4), (70, 40, 64, 64)]:
        wl = synth.rectified_pair(w, h, d, seed=w + d, tile=t)
        cases.append((wl.images, wl.gray, wl.calibs, wl.near, wl.far, [wl.params]))
    cap = synth.capture(160, 120, 3, seed=4, f=130.0)
    cases.append((cap.images, cap.gray, cap.calibs, cap.near, cap.far, api.StereoParams.l16_pyramid()[:4]))
    return cases


def _run_chain(oracle, imgs, gray, calibs, near, far, plist, **kw):
    filt = [oracle.box_filter3(im) for im in imgs]
    out, prev = [], None
    for i, p in enumerate(plist):
        L = oracle.layer(filt, gray, calibs, near, far, p, index=i, prev=prev, keep_pass1=True, **kw)
        out.append(L)
        prev = L
    return out


def _same(a, b):
    for k in ("Raw", "AggPass1", "Agg", "Start", "Count", "Cap"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["Depth"].view(np.uint32), b["Depth"].view(np.uint32))


def test_vector_pixel_form_equals_scalar_form(oracle):
    """Pixel's 8-lane vector form (DenseStereoSgm.cs:280-299), where its guard lets the reference take it, gives the
    values of the scalar form (:300-313) that the oracle otherwise runs: both restated, compared on every layer output."""
    try:
        for case in _layer_cases():
            oracle.set_vector_form(False)
            scalar = _run_chain(oracle, *case)
            oracle.set_vector_form(True)
            vector = _run_chain(oracle, *case)
            assert oracle.vector_calls() > 0  # the guard held for some path blocks
            for a, b in zip(scalar, vector):
                _same(a, b)
    finally:
        oracle.set_vector_form(False)


def test_single_thread_form_equals_parallel_prepass(oracle):
    """The reference's guarantee that the thread count does not change the result (StereoAsyncApi.cs:44-47,
    DenseStereoSgm.cs:176-180): Threads == 1 (costs computed at each pass +1 visit) equals the row-parallel prepass on
    1 and on 4 workers."""
    for case in _layer_cases():
        one = _run_chain(oracle, *case, inline_cost=True)
        for threads in (1, 4):
            par = _run_chain(oracle, *case, threads=threads)
            for a, b in zip(one, par):
                _same(a, b)
