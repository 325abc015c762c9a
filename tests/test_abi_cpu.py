"""The C-ABI library loads without a GPU, exports every symbol include/lux_sgm.h declares, and its host-only entry
points match the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "lux_sgm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lux_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from lux_b200 import _lib
    lib = _lib.load()
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert {n for n, _, _ in _lib.SIGNATURES} == set(names)


def test_host_planes_match_oracle(oracle):
    """lux_sgm_planes (host code of the library) equals the oracle's DenseStereo.Planes bit for bit."""
    from lux_b200 import api, synth
    for d, f, b in [(16, 1000.0, 100.0), (64, 3000.0, 12.5), (256, 2800.0, 40.0)]:
        wl_c = synth.rectified_calibs(f, 100.0, 80.0, b)
        near = float(np.float32(f * b / (d - 1)))
        a = api.DenseStereo.planes(near, 1e30, wl_c, 1.0, 8)
        o = oracle.planes(near, 1e30, wl_c, 1.0, 8)
        assert a.tobytes() == o.tobytes()
        assert len(a) == d
    # a multi-camera rig with rotations and the L16 near/far
    rng = np.random.default_rng(5)
    cal = []
    for k in range(5):
        th = rng.uniform(-0.05, 0.05)
        R = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]], np.float32).reshape(9)
        K = np.array([3000 + 50 * k, 0, 1040, 0, 3000 + 50 * k, 780, 0, 0, 1], np.float32)
        cal.append(api.CalibData(K, rng.uniform(-30, 30, 3).astype(np.float32), R))
    for align in (8, 2):
        a = api.DenseStereo.planes(200.0, 640000.0, cal, 2.0, align)
        o = oracle.planes(200.0, 640000.0, cal, 2.0, align)
        assert a.tobytes() == o.tobytes()


def test_host_planes_errors():
    from lux_b200 import api, synth
    c = synth.rectified_calibs(1000.0, 10.0, 10.0, 100.0)
    with pytest.raises(api.InvalidOperationError):
        api.DenseStereo.planes(500.0, 200.0, c, 1.0, 8)
    with pytest.raises(api.InvalidOperationError):
        api.DenseStereo.planes(0.0, 200.0, c, 1.0, 8)
    with pytest.raises(api.InvalidOperationError):
        api.DenseStereo.planes(200.0, 640000.0, [c[0], c[0]], 1.0, 8)


def test_l16_params_match_reference_defaults():
    from lux_b200 import _lib, api
    lib = _lib.load()
    arr = (_lib.Params * 6)()
    lib.lux_sgm_l16_pyramid(arr)
    py = api.StereoParams.l16_pyramid()
    for i in range(6):
        assert (arr[i].scale, arr[i].tile, arr[i].skip_mode) == (py[i].scale, py[i].tile, py[i].skip_mode)
        assert arr[i].p1 == 1 and arr[i].p2scale == 500.0 and arr[i].margin == 1
        assert [np.float32(v) for v in arr[i].guidance] == [np.float32(v) for v in py[i].guidance]
