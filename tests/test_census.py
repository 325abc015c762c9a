"""The opt-in census stereo mode (census, Hamming cost, 8-path SGM, WTA, subpixel, left/right check, fusion) against
oracle/census_oracle.py. The reference has no such stage, so parity is unpinned: the oracle restates the published method
with this library's conventions. Disparities and fused depths must match bit for bit (the float steps are single
IEEE operations in the same order, well within the 1e-5 relative tolerance allowed for the subpixel and fusion steps).
"""
import numpy as np
import pytest

from oracle import census_oracle as C


def _pair(w, h, d, seed):
    from lux_b200 import synth
    wl = synth.rectified_pair(w, h, max(8, (d + 7) // 8 * 8), seed=seed)
    return wl.images[0][..., 0].copy(), wl.images[1][..., 0].copy()


def test_census_oracle_properties():
    """A flat image has an all-zero census; a pixel against itself costs 0; the oracle tracks a synthetic pair's truth."""
    flat = np.full((20, 30), 77, np.uint8)
    assert not C.census(flat).any()
    img = np.random.default_rng(0).integers(0, 256, (20, 30), dtype=np.uint8)
    c = C.census(img)
    cost = C.hamming_cost(c, c, 4)
    assert (cost[:, :, 0] == 0).all() and (cost[:, :2, 3] == C.INVALID_COST).all()
    from lux_b200 import synth
    wl = synth.rectified_pair(96, 64, 16, seed=3)
    d = C.census_sgm(wl.images[0][..., 0], wl.images[1][..., 0], 16, 10, 120)
    ok = d >= 0
    assert ok.mean() > 0.8
    assert np.median(np.abs(d[ok] - wl.disparity[ok])) < 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,D,p1,p2", [(64, 48, 16, 10, 120), (97, 61, 40, 8, 96), (130, 70, 64, 10, 150), (160, 90, 128, 12, 200),
                                         (120, 40, 200, 5, 60), (50, 33, 256, 10, 120), (33, 17, 7, 3, 30)])
def test_census_sgm_matches_oracle(w, h, D, p1, p2):
    """Every lane width (1, 2, 4, 8 disparities a lane, with padding lanes), ragged sizes, disparity ranges wider than
    the image, subpixel and the left/right check."""
    from lux_b200 import api
    left, right = _pair(w, h, D, seed=w + D)
    got = api.CensusStereo.compute(left, right, D, p1, p2)
    want = C.census_sgm(left, right, D, p1, p2)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("subpixel,lr,diff", [(False, False, 1), (True, False, 1), (False, True, 0), (True, True, 3)])
def test_census_sgm_options(subpixel, lr, diff):
    from lux_b200 import api
    left, right = _pair(88, 52, 32, seed=4)
    got = api.CensusStereo.compute(left, right, 32, 10, 120, subpixel=subpixel, lr_check=lr, lr_max_diff=diff)
    want = C.census_sgm(left, right, 32, 10, 120, lr_max_diff=diff, subpixel=subpixel, lr_check=lr)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_census_device_images_and_fusion():
    """Device-resident RGBA images in and disparities out; then three pairs fused into one depth map (even and odd counts
    of valid depths, pixels with none)."""
    import torch
    from lux_b200 import api
    disps, fbs = [], []
    for k, D in enumerate((32, 48, 64)):
        left, right = _pair(72, 50, D, seed=20 + k)
        rgba = [torch.from_numpy(np.repeat(im[..., None], 4, axis=2)).cuda() for im in (left, right)]
        got = api.CensusStereo.compute(rgba[0], rgba[1], D, 10, 120)
        assert got.is_cuda
        want = C.census_sgm(left, right, D, 10, 120)
        assert np.array_equal(got.cpu().numpy().view(np.uint32), want.view(np.uint32))
        disps.append(want)
        fbs.append(1000.0 * (1.0 + 0.3 * k))
    disps[2][:10] = -1.0  # rows where only two pairs are valid
    disps[0][:5] = disps[1][:5] = -1.0  # rows with one or none
    fused = api.CensusStereo.fuse(disps, fbs)
    want = C.fuse(disps, fbs)
    assert np.array_equal(fused.view(np.uint32), want.view(np.uint32))
    dev = api.CensusStereo.fuse([torch.from_numpy(d).cuda() for d in disps], fbs)
    assert np.array_equal(dev.cpu().numpy().view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_census_errors():
    from lux_b200 import api
    left, right = _pair(40, 30, 16, seed=1)
    for kw in (dict(max_disparity=0), dict(max_disparity=257), dict(max_disparity=16, p2=9000)):
        d = kw.pop("max_disparity")
        with pytest.raises(api.LuxError):
            api.CensusStereo.compute(left, right, d, **kw)
    with pytest.raises(api.LuxError):
        api.CensusStereo.compute(left, right[:, :20].copy(), 16)


@pytest.mark.gpu
def test_census_capture_batch_matches_pairs():
    """A capture's pairs in one batch (one launch per stage over every pair, the reference's census made once) give each
    pair's disparities exactly as a solve of that pair alone, and the fused depth of the oracle."""
    from lux_b200 import api, synth
    ds = [64, 24, 40, 96]
    ref, others, fb = synth.census_capture(90, 56, ds, seed=5)
    depth, disps = api.CensusStereo.capture(ref, others, ds, fb)
    want = [C.census_sgm(ref, o, d, 10, 120) for o, d in zip(others, ds)]
    for k in range(len(ds)):
        assert np.array_equal(disps[k].view(np.uint32), want[k].view(np.uint32)), k
        alone = api.CensusStereo.compute(ref, others[k], ds[k])
        assert np.array_equal(alone.view(np.uint32), want[k].view(np.uint32)), k
    assert np.array_equal(depth.view(np.uint32), C.fuse(want, fb).view(np.uint32))
    assert (depth > 0).mean() > 0.5
