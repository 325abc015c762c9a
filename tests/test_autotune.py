"""The autotuner of the fast aggregation form: the first solve of a layer shape times every form on its own cost volume
and keeps the fastest for later solves; whatever it picks, the layer is bit-identical to the oracle."""
import numpy as np
import pytest

from test_gpu_parity import _compare_layer

pytestmark = pytest.mark.gpu


def test_autotune_picks_keeps_and_can_be_overridden(oracle):
    from lux_b200 import api, synth
    W, H, D, T = 200, 150, 64, 16
    wl = synth.rectified_pair(W, H, D, seed=5, tile=T)
    filt = [oracle.box_filter3(im) for im in wl.images]
    ol = oracle.layer(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True)
    ctx = api.Context(0)

    def solve():
        return api.DenseLayer.compute(filt, wl.gray, wl.calibs, wl.near, wl.far, wl.params, keep_pass1=True, keep_agg=True,
                                      ctx=ctx)
    try:
        api.set_tuned_form(W, H, D, T, 0)  # forget any earlier choice for this shape
        ctx.set_autotune(True)
        n0 = api.kernel_launches()
        g1 = solve()
        n1 = api.kernel_launches()
        assert g1.tuned in (1, 2, 3) and api.tuned_form(W, H, D, T) == g1.tuned
        _compare_layer(g1, ol, "tuning solve")
        g1.close()
        g2 = solve()  # the cached choice: one form runs
        n2 = api.kernel_launches()
        assert g2.tuned == 0 and g2.sgm_kernel == api.tuned_form(W, H, D, T)
        assert n2 - n1 < n1 - n0
        _compare_layer(g2, ol, "tuned solve")
        g2.close()
        for f in (1, 2, 3):  # a choice set from outside (e.g. restored from an earlier process) is followed
            api.set_tuned_form(W, H, D, T, f)
            g = solve()
            assert g.sgm_kernel == f and g.tuned == 0
            assert np.array_equal(g.Depth.view(np.uint32), ol["Depth"].view(np.uint32))
            g.close()
        api.set_tuned_form(W, H, D, T, 0)
        ctx.set_autotune(False)  # untuned and not tuning: the size rule (the fused wavefront below 2 MP)
        g = solve()
        assert g.tuned == 0 and g.sgm_kernel == 1 and api.tuned_form(W, H, D, T) == 0
        g.close()
    finally:
        ctx.close()


def test_tuned_form_arguments():
    from lux_b200 import api
    with pytest.raises(api.LuxError):
        api.set_tuned_form(10, 10, 16, 8, 4)
    with pytest.raises(api.LuxError):
        api.set_tuned_form(0, 10, 16, 8, 1)
