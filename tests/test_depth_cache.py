"""Depth image cache (DepthCache.cs:87-254) on the GPU against the oracle, bit for bit.

Set: inverse depth, nearest resample to the cache dims in 16.16 fixed point, min(rcp, 1e5). Fetch: the ROI check, the plain
view at scale 1, else the source window with its offsets, the reciprocal pass (rcpps + Newton below (vw/32)·32 columns,
division above), the nearest resample and the division back. The oracle restates both from the reference's code; the
reference ships no tests or vectors for this class, so the pin is the shared rcpps table (pinned by the table tests) and
the restated arithmetic.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bits(a):
    a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _depth(rng, h, w, specials=True):
    """Depth in millimetres as the upsample gives it (400 mm .. 200 m, with a far band above the 1e5 clip), plus the
    special values the reciprocal passes treat apart: zeros, infinities, NaN, negatives, subnormals."""
    d = np.exp(rng.uniform(np.log(400.0), np.log(2.0e5), (h, w))).astype(np.float32)
    if specials:
        n = max(1, h * w // 200)
        for v in (0.0, -0.0, np.inf, -np.inf, np.nan, -1234.5, 1e-40, 3.4e38):
            d.flat[rng.integers(0, h * w, n)] = np.float32(v)
    return d


@pytest.fixture(scope="module")
def api():
    from lux_b200 import api
    return api


SET_CASES = [
    (416, 312, 522, 392),   # the full-depth -> level-1 ratio of a 10432x7824 canvas (4160x3120 -> 5216x3912), scaled down
    (1000, 700, 333, 250),  # a downscale
    (37, 23, 64, 9),        # ragged, up in x and down in y
    (100, 80, 100, 80),     # same size
    (1, 1, 7, 5),           # one source pixel
    (5, 3, 1, 1),
]


@pytest.mark.parametrize("device", [False, True])
@pytest.mark.parametrize("w,h,cw,ch", SET_CASES)
def test_set_matches_oracle(api, w, h, cw, ch, device):
    import torch
    rng = np.random.default_rng(w * 7919 + h * 31 + cw)
    d = _depth(rng, h, w)
    c = api.DepthImageCache((cw, ch), device=device)
    c.Set(torch.from_numpy(d).cuda() if device else d)
    assert tuple(c.Current.shape) == (ch, cw)
    if device:
        assert c.Current.is_cuda
    ref = O.depth_cache_set(d, cw, ch)
    assert np.array_equal(_bits(c.Current), _bits(ref))


def test_set_every_exponent(api):
    """Every sign, exponent and rcpps table index (random low mantissa bits) through Set at equal dims: the one-lookup
    path for ordinary exponents and the two-step path for the rest give the oracle's bits."""
    rng = np.random.default_rng(9)
    e = np.repeat(np.arange(256, dtype=np.uint32), 4096 * 2)
    i = np.tile(np.arange(4096, dtype=np.uint32), 512)
    s = np.tile(np.repeat(np.array([0, 1], np.uint32), 4096), 256)
    b = (s << 31) | (e << 23) | (i << 11) | rng.integers(0, 2048, i.size).astype(np.uint32)
    d = b.view(np.float32).reshape(1024, 2048)
    c = api.DepthImageCache((2048, 1024))
    c.Set(d)
    assert np.array_equal(_bits(c.Current), _bits(O.depth_cache_set(d, 2048, 1024)))
    raw = api.DepthImageCache.fetch(d, (0, 0, 1024, 512), (1024, 512))
    assert np.array_equal(_bits(raw), _bits(O.depth_cache_fetch(d, (0, 0, 1024, 512), (1024, 512))))


def test_set_full_resolution(api):
    """FromFullDepth (:239-244): the 4160x3120 full depth into the 5216x3912 level-1 cache, on the device."""
    import torch
    rng = np.random.default_rng(5)
    d = _depth(rng, 3120, 4160)
    c = api.DepthImageCache((5216, 3912), device=True)
    c.Set(torch.from_numpy(d).cuda())
    ref = O.depth_cache_set(d, 5216, 3912)
    assert np.array_equal(_bits(c.Current), _bits(ref))
    assert float(c.Current.max()) <= 100000.0


def _rects(rng, dims, n):
    W, H = dims
    out = [(0, 0, W, H), (0, 0, 1, 1), (W - 1, H - 1, W, H), (W // 3, H // 4, W // 3 + 33, H // 4 + 17)]
    for _ in range(n):
        x0, x1 = sorted(rng.integers(0, W + 1, 2))
        y0, y1 = sorted(rng.integers(0, H + 1, 2))
        if x1 > x0 and y1 > y0:
            out.append((int(x0), int(y0), int(x1), int(y1)))
    return out


FETCH_DIMS = [(522, 392), (261, 196), (1044, 784), (163, 122), (2088, 1568), (500, 400)]


@pytest.mark.parametrize("device", [False, True])
@pytest.mark.parametrize("dims", FETCH_DIMS)
def test_fetch_matches_oracle(api, dims, device):
    """Fetch at the cache's own grid (the plain view), coarser and finer levels and a non-integer ratio; rects whose source
    windows are and are not multiples of 32 wide, so both halves of the reciprocal pass are read."""
    import torch
    rng = np.random.default_rng(dims[0] * 13 + dims[1])
    cache = O.depth_cache_set(_depth(rng, 312, 416), 522, 392)
    img = torch.from_numpy(cache).cuda() if device else cache
    for rect in _rects(rng, dims, 12):
        got = api.DepthImageCache.fetch(img, rect, dims)
        ref = O.depth_cache_fetch(cache, rect, dims)
        assert tuple(got.shape) == (rect[3] - rect[1], rect[2] - rect[0])
        assert np.array_equal(_bits(got), _bits(ref)), rect


def test_fetch_specials_and_unset_cache(api):
    """A zero-filled cache fetched before its first Set, and caches holding zeros, infinities and NaN: the NaN bits are
    the ones an SSE reciprocal pass leaves."""
    rng = np.random.default_rng(11)
    c = api.DepthImageCache((200, 150))
    for rect, dims in (((0, 0, 100, 75), (100, 75)), ((3, 5, 90, 60), (400, 300)), ((0, 0, 200, 150), (200, 150))):
        assert np.array_equal(_bits(c.Fetch(rect, dims)), _bits(O.depth_cache_fetch(c.Current, rect, dims)))
    raw = _depth(rng, 150, 200)
    for rect, dims in (((0, 0, 100, 75), (100, 75)), ((7, 1, 61, 70), (300, 301)), ((0, 0, 50, 50), (64, 64))):
        got = api.DepthImageCache.fetch(raw, rect, dims)
        assert np.array_equal(_bits(got), _bits(O.depth_cache_fetch(raw, rect, dims))), rect


def test_set_then_fetch_levels(api):
    """The export path: Set from a full depth, then Fetch every level of a six-level pipeline over the whole frame and a
    tile of it (FetchForExport, :248-253, shifts the rect by the level origin; origin 0 here)."""
    import torch
    rng = np.random.default_rng(3)
    d = _depth(rng, 624, 832, specials=False)
    c = api.DepthImageCache((1043, 782), device=True)
    c.Set(torch.from_numpy(d).cuda())
    host = c.Current.cpu().numpy()
    for lv in range(6):
        dims = (2086 >> lv, 1564 >> lv)
        for rect in ((0, 0) + dims, (dims[0] // 4, dims[1] // 4, dims[0] // 2 + 1, dims[1] // 2 + 3)):
            got = c.Fetch(rect, dims)
            assert np.array_equal(_bits(got), _bits(O.depth_cache_fetch(host, rect, dims))), (lv, rect)


@pytest.mark.parametrize("rect,dims", [
    ((5, 5, 5, 9), (20, 20)),     # zero width
    ((5, 5, 9, 5), (20, 20)),     # zero height
    ((9, 5, 5, 9), (20, 20)),     # x1 < x0
    ((-1, 0, 4, 4), (20, 20)),    # negative origin
    ((0, -3, 4, 4), (20, 20)),
    ((0, 0, 21, 4), (20, 20)),    # past the level's dims
    ((0, 0, 4, 21), (20, 20)),
    ((0, 0, 4, 4), (0, 0)),       # empty level
])
def test_fetch_invalid_roi(api, rect, dims):
    cache = np.ones((10, 10), np.float32)
    with pytest.raises(O.OracleError) as e:
        O.depth_cache_fetch(cache, rect, dims)
    assert e.value.code == 14
    with pytest.raises(api.InvalidOperationError, match="invalid ROI requested!"):
        api.DepthImageCache.fetch(cache, rect, dims)


def test_set_empty_image(api):
    c = api.DepthImageCache((0, 4))
    with pytest.raises(api.InvalidOperationError, match="empty image!"):
        c.Set(np.ones((3, 3), np.float32))
    with pytest.raises(O.OracleError) as e:
        O.depth_cache_set(np.ones((3, 3), np.float32), 0, 4)
    assert e.value.code == 15
