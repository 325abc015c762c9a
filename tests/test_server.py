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


def _heavy_and_light():
    from lux_b200 import synth
    heavy = [synth.rectified_pair(2080, 1560, 256, seed=60 + k, bits=12, tile=64) for k in range(2)]
    light = [synth.rectified_pair(300, 170, 64, seed=70 + k, tile=64) for k in range(4)]
    return [(w.images, w.gray, w.calibs, w.near, w.far, w.params) for w in heavy], \
           [(w.images, w.gray, w.calibs, w.near, w.far, w.params) for w in light]


def test_light_requests_pass_a_heavy_one_that_waits():
    """JobQueue.Dispatch (Lux.Library/Core/JobQueue.cs:496-521): with a budget that holds one heavy request (estimate above
    1.5 GiB) at a time, the second heavy request waits for memory and the light requests queued behind it start ahead
    of it; every result still equals the request solved alone."""
    import torch
    from lux_b200 import api
    heavy, light = _heavy_and_light()
    dev = lambda r: ([torch.from_numpy(im).cuda() for im in r[0]],) + tuple(r[1:])  # noqa: E731
    heavy, light = [dev(r) for r in heavy], [dev(r) for r in light]
    est_h = [api.Server.estimate(*r) for r in heavy]
    est_l = [api.Server.estimate(*r) for r in light]
    assert min(est_h) > 3 << 29 and max(est_l) <= 3 << 29  # heavy and light as the job queue draws the line
    ctx = api.Context(0)
    solo = []
    for r in heavy + light:
        L = api.DenseLayer.compute(*r, prefilter=True, ctx=ctx)
        solo.append(L.Depth.copy())
        L.close()
    ctx.close()
    srv = api.Server(0, hbm_budget_bytes=max(est_h) + sum(est_l), slots=3)
    try:
        tickets = [srv.submit(*r) for r in heavy + light]
        results = [srv.wait(t) for t in tickets]
        assert srv.passed >= 1
    finally:
        srv.close()
    for i, r in enumerate(results):
        assert r.status == 0
        assert np.array_equal(r.Depth.view(np.uint32), solo[i].view(np.uint32)), i
    # the second heavy request started after at least one light request that was queued behind it
    start_h2 = results[1].queue_ms
    assert any(r.queue_ms < start_h2 for r in results[2:])


def test_priority_order():
    """Waiting requests start by priority (lower first), then by arrival (JobQueue.cs:497)."""
    from lux_b200 import api
    heavy, light = _heavy_and_light()
    srv = api.Server(0, hbm_budget_bytes=0, slots=1)
    try:
        first = srv.submit(*heavy[0])  # occupies the only worker while the others queue
        t = [srv.submit(*light[k], priority=p) for k, p in enumerate([2, 0, 1, 0])]
        srv.wait(first)
        res = [srv.wait(x) for x in t]
    finally:
        srv.close()
    # start time relative to the common submission: priority 0 (second, fourth), then 1, then 2
    start = [r.queue_ms for r in res]
    assert start[1] < start[3] < start[2] < start[0]


def test_estimate_covers_the_device_high_water():
    """The server's per-request estimate is at least the device memory the solve really takes at its peak (the pool's
    high-water mark with nothing else allocated), for a preview pair, a 3 MP D=256 pair, a 13 MP D=128 pair and a
    module capture."""
    from lux_b200 import api, synth
    reqs = []
    for (w, h, d, bits) in [(520, 390, 32, 8), (2080, 1560, 256, 12), (4160, 3120, 128, 12)]:
        wl = synth.rectified_pair(w, h, d, seed=80 + d, bits=bits, tile=64)
        reqs.append((wl.images, wl.gray, wl.calibs, wl.near, wl.far, wl.params))
    mc = synth.module_capture(2080, 1560, seed=81, tile=64)
    reqs.append((mc.images, mc.gray, mc.calibs, mc.near, mc.far, mc.params))
    ctx = api.Context(0)
    try:
        for r in reqs:
            est = api.Server.estimate(*r)
            ctx.check(ctx.lib.lux_sgm_sync(ctx.handle))
            api.pool_high_water(0, reset=True)
            base = api.pool_high_water(0)
            L = api.DenseLayer.compute(*r, prefilter=True, ctx=ctx)
            _ = L.Depth
            L.close()
            ctx.check(ctx.lib.lux_sgm_sync(ctx.handle))
            peak = api.pool_high_water(0) - base
            assert peak > 0 and est >= peak, (r[0][0].shape, est, peak)
    finally:
        ctx.close()


def test_cancel_before_start():
    """A queued request canceled before it starts reports LUX_ERR_CANCELED (OperationCanceledException); a finished one
    is not changed (a started state of the reference runs to its end, StereoAsyncApi.cs:51-64); the rest run as if the
    canceled one had never been submitted."""
    from lux_b200 import api
    heavy, light = _heavy_and_light()
    ctx = api.Context(0)
    solo = []
    for r in light:
        L = api.DenseLayer.compute(*r, prefilter=True, ctx=ctx)
        solo.append(L.Depth.copy())
        L.close()
    ctx.close()
    srv = api.Server(0, hbm_budget_bytes=0, slots=1)
    try:
        first = srv.submit(*heavy[0])  # occupies the only worker while the others queue
        t = [srv.submit(*r) for r in light]
        assert srv.cancel(t[1])
        with pytest.raises(api.LuxError):
            srv.cancel(123456789)  # unknown ticket
        srv.wait(first)
        res = {k: srv.wait(x) for k, x in enumerate(t) if k != 0}
        assert not srv.cancel(t[0])  # finished (its wait not yet taken): left as it is
        res[0] = srv.wait(t[0])
    finally:
        srv.close()
    assert res[1].status == 13
    for k in range(len(light)):
        if k == 1:
            continue
        assert res[k].status == 0
        assert np.array_equal(res[k].Depth.view(np.uint32), solo[k].view(np.uint32)), k
