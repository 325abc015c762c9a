"""Dump and golden-file formats of the dense stage (StereoAsyncApi.cs:197-262) against the oracle's restatement of them.

The CPU tests write and read the float and RGBA8 image formats through the C ABI (host code, no GPU); the GPU test
dumps a solved six-layer pyramid and compares every file byte for byte with the files the oracle's layers give.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def api():
    from lux_b200 import api
    return api


def test_f32_round_trip(api, tmp_path):
    rng = np.random.default_rng(0)
    d = rng.standard_normal((37, 53)).astype(np.float32)
    p = tmp_path / "x_depth.f32"
    api.dump_f32(p, d)
    assert p.read_bytes() == O.f32_bytes(d)
    back = api.load_f32(p)
    assert back.shape == (37, 53) and np.array_equal(back.view(np.uint32), d.view(np.uint32))
    api.dump_f32(tmp_path / "empty.f32", np.zeros((0, 5), np.float32))
    assert api.load_f32(tmp_path / "empty.f32").shape == (0, 5)


def test_load_f32_errors(api, tmp_path):
    """LoadF32 (:257-261): a dump whose bytes per pixel is not 4 is refused; a missing file is an I/O error."""
    img = np.zeros((4, 6, 4), np.uint8)
    p = tmp_path / "img.u8"
    p.write_bytes(np.array([6, 4, 6, 1], "<i4").tobytes() + img[..., 0].tobytes())
    with pytest.raises(api.InvalidOperationError, match="expected a 4-byte float dump"):
        api.load_f32(p)
    with pytest.raises(api.LuxError) as e:
        api.load_f32(tmp_path / "missing.f32")
    assert e.value.code == 16


def test_rgba8_dump_strided(api, tmp_path):
    """DumpRgba8 (:217-223) writes w·4 bytes per row whatever the source stride."""
    rng = np.random.default_rng(1)
    big = rng.integers(0, 256, (20, 31, 4), dtype=np.uint8)
    from lux_b200 import _lib as L
    view = big[:, :23]
    ci = L.Img(big.ctypes.data, 23, 20, 31, 0)
    rc = api.L.load().lux_dump_rgba8(os.fsencode(tmp_path / "v.img"), ci)
    assert rc == 0
    assert (tmp_path / "v.img").read_bytes() == O.rgba8_bytes(view)
    api.dump_rgba8(tmp_path / "w.img", big)
    assert (tmp_path / "w.img").read_bytes() == O.rgba8_bytes(big)


@pytest.mark.gpu
def test_dense_dump_matches_oracle(api, tmp_path):
    """The dense dump of a six-layer pyramid (cost volumes of layers 0..2 with their pass-1 copies) equals, file for file,
    the dump the oracle's layers give."""
    from lux_b200 import synth
    cap = synth.capture(416, 312, 3, seed=5, f=330.0)
    ol = O.pyramid(cap.images, cap.gray, cap.calibs, cap.near, cap.far, keep_pass1=True)
    layers = api.DenseStereoPyramid.run(cap.images, cap.gray, cap.calibs, cap.near, cap.far, keep_pass1=True, keep_agg=True)
    try:
        prefix = str(tmp_path / "cap")
        api.dump_dense(prefix, layers, cap.images, cap.calibs, cv_max=2)
        want = O.dense_dump_bytes(ol, cap.images, [O.box_filter3(im) for im in cap.images], cap.calibs, cv_max=2)
        got = {f[len("cap"):]: (tmp_path / f).read_bytes() for f in os.listdir(tmp_path) if f.startswith("cap_")}
        assert sorted(got) == sorted(want)
        for name in want:
            assert got[name] == want[name], name
        d5 = api.load_f32(prefix + "_dense_L5_depth.f32")  # the file LUX_DENSE_OVERRIDE reads
        assert np.array_equal(d5, layers[5].Depth)
        with pytest.raises(api.LuxError):  # the final aggregates of a fast-kernel layer are only there with keep_agg
            plain = api.DenseStereoPyramid.run(cap.images, cap.gray, cap.calibs, cap.near, cap.far)
            try:
                plain[0].dump_cost_volume(prefix + "_plain")
            finally:
                for g in plain:
                    g.close()
    finally:
        for g in layers:
            g.close()
