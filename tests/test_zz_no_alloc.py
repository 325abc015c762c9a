"""lux_sgm_upsample_noalloc, the upsample for hosts that cannot let this library allocate GPU memory (their HBM belongs to
another allocator, or their request loop must not synchronise on cudaMalloc / cudaFree), checked through the C ABI
against lux_sgm_upsample on two calls in a row with different sizes, plus its size limit. It has no counterpart in the
reference. The file name makes pytest collect it after the other test files."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from lux_b200 import api
    c = api.Context(0)
    yield c
    c.close()


def _inputs(pw, ph, seed):
    rng = np.random.default_rng(seed)
    depth = rng.uniform(300.0, 6000.0, (ph, pw)).astype(np.float32)
    guide = rng.integers(0, 256, (2 * ph, 2 * pw, 4), dtype=np.uint8)
    conf = rng.uniform(0, 1, (ph, pw)).astype(np.float32)
    return depth, guide, conf


def _noalloc(ctx, depth, guide, conf, pw, ph, set_w, set_h):
    import torch
    from lux_b200 import _lib
    dev = torch.device("cuda", 0)
    d_prev = torch.from_numpy(depth).to(dev)
    d_conf = torch.from_numpy(conf).to(dev)
    d_guide = torch.from_numpy(guide).to(dev)
    gh, gw = guide.shape[:2]
    d_out = torch.full((gh, gw), float("nan"), dtype=torch.float32, device=dev)
    d_oc = torch.full((gh, gw), float("nan"), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    img = _lib.Img(d_guide.data_ptr(), gw, gh, gw, 1)
    free0 = torch.cuda.mem_get_info(0)[0]
    rc = ctx.lib.lux_sgm_upsample_noalloc(ctx.handle, d_prev.data_ptr(), pw, ph, ctypes.byref(img), set_w, set_h, 12.0, 2,
                                          d_conf.data_ptr(), d_out.data_ptr(), d_oc.data_ptr())
    free1 = torch.cuda.mem_get_info(0)[0]
    return rc, d_out.cpu().numpy(), d_oc.cpu().numpy(), free0, free1


def test_noalloc_matches_upsample_twice(ctx):
    from lux_b200 import api
    results = []
    for k, (pw, ph) in enumerate([(208, 156), (52, 39)]):
        depth, guide, conf = _inputs(pw, ph, 100 + k)
        ref = api.DenseUpsampleLayer.run(depth, pw, ph, guide, pw, ph, prev_confidence=conf, ctx=ctx)
        before = ctx.lib.lux_sgm_kernel_launches()
        rc, d, c, free0, free1 = _noalloc(ctx, depth, guide, conf, pw, ph, pw, ph)
        ctx.check(rc)
        assert ctx.lib.lux_sgm_kernel_launches() - before == 3  # resample + bilateral of depth and of confidence
        assert np.array_equal(d.view(np.uint32), ref.Depth.view(np.uint32)), (pw, ph)
        assert np.array_equal(c.view(np.uint32), ref.Confidence.view(np.uint32)), (pw, ph)
        results.append((free0, free1))
    # the second call finds its scratch already set up and takes no device memory
    assert results[1][0] == results[1][1]


def test_noalloc_limits(ctx):
    from lux_b200 import _lib, api
    import torch
    dev = torch.device("cuda", 0)
    d_prev = torch.zeros(8, dtype=torch.float32, device=dev)
    d_guide = torch.zeros((4, 4, 4), dtype=torch.uint8, device=dev)
    d_out = torch.zeros(16, dtype=torch.float32, device=dev)
    img = _lib.Img(d_guide.data_ptr(), 4, 4, 4, 1)
    big = 1 << 12  # 4096 x 4096 > LUX_UPSAMPLE_NOALLOC_MAX_PIXELS: rejected before any launch
    rc = ctx.lib.lux_sgm_upsample_noalloc(ctx.handle, d_prev.data_ptr(), big, big, ctypes.byref(img), 2, 2, 12.0, 2, None,
                                          d_out.data_ptr(), None)
    assert rc == 9
    assert b"exceeds the static scratch" in ctx.lib.lux_sgm_last_error(ctx.handle)
    host_img = _lib.Img(np.zeros(64, np.uint8).ctypes.data, 4, 4, 4, 0)
    rc = ctx.lib.lux_sgm_upsample_noalloc(ctx.handle, d_prev.data_ptr(), 2, 2, ctypes.byref(host_img), 2, 2, 12.0, 2, None,
                                          d_out.data_ptr(), None)
    assert rc == 9
    # the reference's size check still applies after the computation
    d_prev2 = torch.full((2, 2), 1000.0, dtype=torch.float32, device=dev)
    rc = ctx.lib.lux_sgm_upsample_noalloc(ctx.handle, d_prev2.data_ptr(), 2, 2, ctypes.byref(img), 3, 2, 12.0, 2, None,
                                          d_out.data_ptr(), None)
    with pytest.raises(api.InvalidOperationError):
        ctx.check(rc)


def test_noalloc_inputs_ordered_by_an_event(ctx):
    """Inputs written on another stream reach the call through an event that the context's stream waits on, with no
    device-wide synchronisation: the result equals lux_sgm_upsample's."""
    import torch
    from lux_b200 import _lib, api
    pw, ph = 96, 64
    depth, guide, conf = _inputs(pw, ph, 7)
    ref = api.DenseUpsampleLayer.run(depth, pw, ph, guide, pw, ph, prev_confidence=conf, ctx=ctx)
    dev = torch.device("cuda", 0)
    h_prev = torch.from_numpy(depth).pin_memory()
    h_conf = torch.from_numpy(conf).pin_memory()
    h_guide = torch.from_numpy(guide).pin_memory()
    side = torch.cuda.Stream(dev)
    with torch.cuda.stream(side):
        d_prev = h_prev.to(dev, non_blocking=True)
        d_conf = h_conf.to(dev, non_blocking=True)
        d_guide = h_guide.to(dev, non_blocking=True)
        d_out = torch.empty((2 * ph, 2 * pw), dtype=torch.float32, device=dev)
        d_oc = torch.empty((2 * ph, 2 * pw), dtype=torch.float32, device=dev)
        written = torch.cuda.Event()
        written.record(side)
    lux_stream = torch.cuda.ExternalStream(ctx.lib.lux_sgm_stream(ctx.handle), device=dev)
    lux_stream.wait_event(written)
    img = _lib.Img(d_guide.data_ptr(), 2 * pw, 2 * ph, 2 * pw, 1)
    rc = ctx.lib.lux_sgm_upsample_noalloc(ctx.handle, d_prev.data_ptr(), pw, ph, ctypes.byref(img), pw, ph, 12.0, 2,
                                          d_conf.data_ptr(), d_out.data_ptr(), d_oc.data_ptr())
    ctx.check(rc)
    side.synchronize()
    assert np.array_equal(d_out.cpu().numpy().view(np.uint32), ref.Depth.view(np.uint32))
    assert np.array_equal(d_oc.cpu().numpy().view(np.uint32), ref.Confidence.view(np.uint32))
