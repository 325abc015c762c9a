"""The failure path of the bounded device waits, tested without a GPU fault.

Every wait of the aggregation kernels (a block waiting for the block above it, a warp for its neighbour) gives up after
the context's wait limit and the solve returns LUX_ERR_TIMEOUT. The test shortens the limit to 1 ms and makes one block
wait on a counter that nothing publishes (lux_sgm_debug_stall): the wait runs out, the kernels return, and the same
context then solves a layer bit for bit like the oracle. Nothing traps, faults or spins without a bound."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LUX_ERR_TIMEOUT = 11


def _compute(api, ctx, wl, filt, kernel):
    args = dict(force_replay=True) if kernel == "replay" else dict(sgm=kernel)
    return api.DenseLayer.compute(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True, keep_agg=True,
                                  ctx=ctx, **args)


@pytest.mark.parametrize("kernel", ["fused", "split", "wave", "replay"])
def test_stalled_block_times_out_and_context_recovers(oracle, kernel):
    from lux_b200 import api, synth
    ctx = api.Context(0)
    try:
        assert ctx.wait_limit_ns == 20_000_000_000
        wl = synth.rectified_pair(160, 120, 32, seed=17, tile=8)
        filt = [oracle.box_filter3(im) for im in wl.images]
        ol = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True)
        ctx.wait_limit_ns = 1_000_000
        ctx.debug_stall(1)
        with pytest.raises(api.LuxError) as e:
            _compute(api, ctx, wl, filt, kernel).close()
        assert e.value.code == LUX_ERR_TIMEOUT
        ctx.debug_stall(-1)
        ctx.wait_limit_ns = 0  # back to the default
        assert ctx.wait_limit_ns == 20_000_000_000
        gl = _compute(api, ctx, wl, filt, kernel)
        try:
            assert np.array_equal(gl.Agg, ol["Agg"])
            assert np.array_equal(gl.AggPass1, ol["AggPass1"])
            assert np.array_equal(gl.Depth.view(np.uint32), ol["Depth"].view(np.uint32))
        finally:
            gl.close()
    finally:
        ctx.close()


def test_debug_stall_arguments():
    from lux_b200 import api
    ctx = api.Context(0)
    try:
        with pytest.raises(api.LuxError):
            ctx.debug_stall(0)  # block 0 waits on nobody
        with pytest.raises(api.LuxError):
            ctx.debug_stall(-2)
    finally:
        ctx.close()
