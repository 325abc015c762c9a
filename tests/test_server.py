"""The request server (lux_server_*): a mix of requests of different sizes submitted together, under a budget that
admits several at once and under one that admits them one by one; every result equals the same request solved alone
through lux_sgm_layer, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests():
    from lux_b200 import api, synth
    reqs = []
    for k, (w, h, d, tile) in enumerate([(300, 170, 64, 64), (96, 80, 16, 8), (520, 390, 32, 64), (160, 120, 48, 16)]):
        wl = synth.rectified_pair(w, h, d, seed=50 + k, tile=tile)
        reqs.append((wl.images, wl.gray, wl.calibs, wl.near, wl.far, wl.params))
    cap = synth.capture(120, 90, 4, seed=57, f=90.0, baseline_mm=(20.0, 60.0))
    reqs.append((cap.images, cap.gray, cap.calibs, cap.near, cap.far,
                 api.StereoParams(scale=1, tile=8, skip_mode=0, plane_density=2.0)))
    mc = synth.module_capture(96, 72, seed=58, size_scale=0.002, tile=8)
    reqs.append((mc.images, mc.gray, mc.calibs, mc.near, mc.far, mc.params))
    return reqs


@pytest.mark.parametrize("budget", [0, 1])
def test_served_results_equal_solo(budget):
    from lux_b200 import api
    reqs = _requests()
    ctx = api.Context(0)
    solo = []
    for images, gray, calibs, near, far, params in reqs:
        L = api.DenseLayer.compute(images, gray, calibs, near, far, params, prefilter=True, ctx=ctx)
        solo.append(L.Depth.copy())
        L.close()
    ctx.close()
    srv = api.Server(0, hbm_budget_bytes=budget, slots=3)  # budget 1 byte: one request at a time
    try:
        tickets = [srv.submit(*r) for r in reqs * 2]  # every request twice, all in flight together
        results = [srv.wait(t) for t in tickets]
    finally:
        srv.close()
    for i, r in enumerate(results):
        assert r.status == 0
        ref = solo[i % len(reqs)]
        assert r.Depth.shape == ref.shape
        assert np.array_equal(r.Depth.view(np.uint32), ref.view(np.uint32)), i
        assert r.run_ms > 0 and r.queue_ms >= 0
