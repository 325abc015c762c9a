"""ctypes wrapper of the CPU oracle (oracle/lux_oracle.c) — TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker / baseline; never by the
product path. Parity unpinned against reference outputs (see lux_oracle.h).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liblux_oracle.so")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


class LoParams(ctypes.Structure):
    _fields_ = [("margin", ctypes.c_int), ("plane_density", ctypes.c_float), ("scale", ctypes.c_int), ("skip_mode", ctypes.c_int),
                ("p1", ctypes.c_uint16), ("p2scale", ctypes.c_float), ("guidance", ctypes.c_float * 4), ("tile", ctypes.c_int)]


class LoCalib(ctypes.Structure):
    _fields_ = [("K", ctypes.c_float * 9), ("T", ctypes.c_float * 3), ("R", ctypes.c_float * 9)]


class LoLayer(ctypes.Structure):
    _fields_ = [("p", LoParams), ("index", ctypes.c_int), ("align", ctypes.c_int), ("w", ctypes.c_int), ("h", ctypes.c_int),
                ("n_planes", ctypes.c_int), ("min_lo", ctypes.c_int), ("max_hi", ctypes.c_int),
                ("planes", ctypes.POINTER(ctypes.c_float)), ("guidance", ctypes.POINTER(ctypes.c_uint8)),
                ("skip", ctypes.POINTER(ctypes.c_uint8)), ("start", ctypes.POINTER(ctypes.c_uint16)),
                ("count", ctypes.POINTER(ctypes.c_uint16)), ("cap", ctypes.POINTER(ctypes.c_uint16)),
                ("off", ctypes.POINTER(ctypes.c_uint64)), ("agg", ctypes.POINTER(ctypes.c_uint16)),
                ("agg_pass1", ctypes.POINTER(ctypes.c_uint16)), ("raw", ctypes.POINTER(ctypes.c_uint8)),
                ("depth", ctypes.POINTER(ctypes.c_float)),
                ("n_cams", ctypes.c_int), ("images", ctypes.c_void_p), ("iw", ctypes.c_void_p), ("ih", ctypes.c_void_p),
                ("warps", ctypes.c_void_p), ("wq", ctypes.c_void_p),
                ("threads", ctypes.c_int), ("keep_pass1", ctypes.c_int), ("xsw", ctypes.c_int), ("inline_cost", ctypes.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        l = ctypes.CDLL(LIB)
        l.lo_planes.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.POINTER(LoCalib), ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)]
        l.lo_box_filter3.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        l.lo_box_filter3_scalar.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        l.lo_layer_init.argtypes = [ctypes.POINTER(LoLayer), ctypes.POINTER(LoParams), ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(LoCalib), ctypes.c_float,
                                    ctypes.c_float, ctypes.c_int, ctypes.POINTER(LoLayer)]
        l.lo_layer_compute.argtypes = [ctypes.POINTER(LoLayer)]
        l.lo_layer_free.argtypes = [ctypes.POINTER(LoLayer)]
        l.lo_pyramid_run.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.POINTER(LoCalib), ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(LoLayer)]
        l.lo_upsample.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p]
        l.lo_traversal_trace.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_long]
        l.lo_traversal_trace.restype = ctypes.c_long
        l.lo_set_vector_form.argtypes = [ctypes.c_int]
        l.lo_vector_calls.restype = ctypes.c_long
        l.lo_rcp_bits.argtypes = [ctypes.c_uint32]
        l.lo_rcp_bits.restype = ctypes.c_uint32
        l.lo_rsqrt_bits.argtypes = [ctypes.c_uint32]
        l.lo_rsqrt_bits.restype = ctypes.c_uint32
        l.lo_mt_seed.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        l.lo_mt_next.argtypes = [ctypes.c_void_p]
        l.lo_mt_next.restype = ctypes.c_uint32
        l.lo_skip_mask.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        l.lo_flow_matrix.argtypes = [ctypes.POINTER(LoCalib), ctypes.POINTER(LoCalib), ctypes.POINTER(ctypes.c_float)]
        l.lo_default_params.argtypes = [ctypes.POINTER(LoParams)]
        l.lo_l16_pyramid.argtypes = [ctypes.POINTER(LoParams)]
        l.lo_depth_cache_set.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        l.lo_depth_cache_fetch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        l.lo_wine_sinf.argtypes = [ctypes.c_float]
        l.lo_wine_sinf.restype = ctypes.c_float
        l.lo_gamma_encode.argtypes = [ctypes.c_float]
        l.lo_gamma_encode.restype = ctypes.c_float
        l.lo_lanczos_table.argtypes = [ctypes.c_void_p]
        l.lo_yuv_matrix.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        l.lo_warp_f32.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(LoAligned), ctypes.c_void_p]
        l.lo_convert_yuv.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        l.lo_to_rgba8.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        l.lo_warp_rgba8.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(LoAligned), ctypes.c_void_p]
        l.lo_crop_rect.argtypes = [ctypes.POINTER(LoCalib), ctypes.POINTER(LoCalib), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_void_p]
        l.lo_color_transfer.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(LoCalib), ctypes.POINTER(LoCalib), ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        _lib = l
    return _lib


class LoAligned(ctypes.Structure):
    _fields_ = [("H", ctypes.c_float * 9), ("lut", ctypes.c_void_p), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
                ("sx", ctypes.c_float), ("sy", ctypes.c_float)]


class OracleError(RuntimeError):
    def __init__(self, code, where):
        super().__init__(f"oracle error {code} in {where}")
        self.code = code


def _calibs(calibs):
    arr = (LoCalib * len(calibs))()
    for i, c in enumerate(calibs):
        for j, v in enumerate(np.asarray(c.K, np.float32).reshape(9)):
            arr[i].K[j] = float(v)
        for j, v in enumerate(np.asarray(c.T, np.float32).reshape(3)):
            arr[i].T[j] = float(v)
        for j, v in enumerate(np.asarray(c.R, np.float32).reshape(9)):
            arr[i].R[j] = float(v)
    return arr


def params_c(p):
    lp = LoParams()
    lp.margin, lp.plane_density, lp.scale, lp.skip_mode = p.margin, p.plane_density, p.scale, p.skip_mode
    lp.p1, lp.p2scale, lp.tile = p.p1, p.p2scale, p.tile
    for i in range(4):
        lp.guidance[i] = float(p.guidance[i])
    return lp


def planes(near, far, calibs, density, align):
    out = (ctypes.c_float * (4096 + align + 16))()
    n = ctypes.c_int()
    rc = lib().lo_planes(near, far, _calibs(calibs), len(calibs), density, align, out, ctypes.byref(n))
    if rc:
        raise OracleError(rc, "planes")
    return np.frombuffer(out, np.float32, n.value).copy()


def box_filter3(img, scalar=False):
    a = np.ascontiguousarray(img, np.uint8)
    h, w, _ = a.shape
    out = np.empty_like(a)
    (lib().lo_box_filter3_scalar if scalar else lib().lo_box_filter3)(a.ctypes.data, w, h, out.ctypes.data)
    return out


def _arr(ptr, dtype, n):
    if n == 0 or not ptr:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


def _extract(L):
    w, h = L.w, L.h
    npx = w * h
    vol = int(np.ctypeslib.as_array(L.off, shape=(npx + 1,))[npx])
    return {
        "W": w, "H": h, "n_planes": L.n_planes, "MinLo": L.min_lo, "MaxHi": L.max_hi, "Align": L.align,
        "Planes": _arr(L.planes, np.float32, L.n_planes),
        "Guidance": _arr(L.guidance, np.uint8, npx * 4).reshape(h, w, 4),
        "Skip": _arr(L.skip, np.uint8, npx).reshape(h, w),
        "Start": _arr(L.start, np.uint16, npx).reshape(h, w),
        "Count": _arr(L.count, np.uint16, npx).reshape(h, w),
        "Cap": _arr(L.cap, np.uint16, npx).reshape(h, w),
        "Offsets": _arr(L.off, np.uint64, npx + 1),
        "Agg": _arr(L.agg, np.uint16, vol),
        "AggPass1": _arr(L.agg_pass1, np.uint16, vol) if L.agg_pass1 else None,
        "Raw": _arr(L.raw, np.uint8, vol),
        "Depth": _arr(L.depth, np.float32, npx).reshape(h, w) if L.depth else None,
    }


def _images(images):
    imgs = [np.ascontiguousarray(im, np.uint8) for im in images]
    ptrs = (ctypes.c_void_p * len(imgs))(*[im.ctypes.data for im in imgs])
    iw = (ctypes.c_int * len(imgs))(*[im.shape[1] for im in imgs])
    ih = (ctypes.c_int * len(imgs))(*[im.shape[0] for im in imgs])
    return imgs, ptrs, iw, ih


def layer(filtered, gray, calibs, near, far, params, index=0, align=8, prev=None, keep_pass1=False, threads=1, xsw=False,
          inline_cost=False):
    """DenseLayer.Init + Compute on box-filtered images. prev: a dict from a previous call (needs its Depth and Skip).
    inline_cost: the reference's Threads == 1 form (costs computed at every pass +1 visit) instead of the row-parallel
    prepass on `threads` workers (its Threads > 1 form)."""
    imgs, ptrs, iw, ih = _images(filtered)
    g = np.ascontiguousarray(np.asarray(gray, np.uint8))
    cc = _calibs(calibs)
    L = LoLayer()
    prevL = None
    if prev is not None:
        prevL = LoLayer()
        prevL.w, prevL.h = prev["W"], prev["H"]
        pd = np.ascontiguousarray(prev["Depth"], np.float32)
        ps = np.ascontiguousarray(prev["Skip"], np.uint8)
        prevL.depth = pd.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        prevL.skip = ps.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
    lp = params_c(params)
    rc = lib().lo_layer_init(ctypes.byref(L), ctypes.byref(lp), index, len(imgs), ptrs, iw, ih, g.ctypes.data, cc, near, far, align,
                             ctypes.byref(prevL) if prevL is not None else None)
    try:
        if rc:
            raise OracleError(rc, "layer_init")
        L.threads, L.keep_pass1, L.xsw = threads, 1 if keep_pass1 else 0, 1 if xsw else 0
        L.inline_cost = 1 if inline_cost else 0
        rc = lib().lo_layer_compute(ctypes.byref(L))
        if rc:
            raise OracleError(rc, "layer_compute")
        return _extract(L)
    finally:
        lib().lo_layer_free(ctypes.byref(L))


def set_vector_form(on):
    """Pixel's 8-lane vector form where the reference takes it (True), or the scalar form only (False, the default)."""
    lib().lo_set_vector_form(1 if on else 0)


def vector_calls():
    """Path blocks that took the vector form since the last set_vector_form."""
    return int(lib().lo_vector_calls())


def pyramid(images, gray, calibs, near, far, threads=1, keep_pass1=False):
    """DenseStereoPyramid.Run on the raw camera images: six layer dicts."""
    imgs, ptrs, iw, ih = _images(images)
    g = np.ascontiguousarray(np.asarray(gray, np.uint8))
    cc = _calibs(calibs)
    Ls = (LoLayer * 6)()
    rc = lib().lo_pyramid_run(len(imgs), ptrs, iw, ih, g.ctypes.data, cc, near, far, threads, 1 if keep_pass1 else 0, Ls)
    try:
        if rc:
            raise OracleError(rc, "pyramid")
        return [_extract(Ls[i]) for i in range(6)]
    finally:
        for i in range(6):
            lib().lo_layer_free(ctypes.byref(Ls[i]))


def upsample(prev_depth, pw, ph, guide, set_w, set_h, sigma=12.0, scale=2, prev_conf=None):
    g = np.ascontiguousarray(guide, np.uint8)
    gh, gw, _ = g.shape
    pd = np.ascontiguousarray(np.asarray(prev_depth, np.float32).reshape(-1))
    out = np.empty(gw * gh, np.float32)
    conf = None
    if prev_conf is not None:
        pc = np.ascontiguousarray(np.asarray(prev_conf, np.float32).reshape(-1))
        conf = np.empty(gw * gh, np.float32)
    rc = lib().lo_upsample(pd.ctypes.data, pw, ph, g.ctypes.data, gw, gh, gw, set_w, set_h, sigma, scale,
                           pc.ctypes.data if prev_conf is not None else None, out.ctypes.data,
                           conf.ctypes.data if conf is not None else None)
    if rc:
        raise OracleError(rc, "upsample")
    return out.reshape(gh, gw), (conf.reshape(gh, gw) if conf is not None else None)


def depth_cache_set(depth, cw, ch):
    """DepthImageCache.Set (DepthCache.cs:137-143): the cache image (ch, cw) made from a depth map."""
    d = np.ascontiguousarray(np.asarray(depth, np.float32))
    h, w = d.shape
    out = np.empty((ch, cw), np.float32)
    rc = lib().lo_depth_cache_set(d.ctypes.data, w, h, cw, ch, out.ctypes.data)
    if rc:
        raise OracleError(rc, "depth_cache_set")
    return out


def depth_cache_fetch(cache, rect, dims):
    """DepthImageCache.Fetch (DepthCache.cs:160-183): rect = (x0, y0, x1, y1) against pipeline dims (w, h)."""
    c = np.ascontiguousarray(np.asarray(cache, np.float32))
    ih, iw = c.shape
    x0, y0, x1, y1 = rect
    out = np.empty((max(y1 - y0, 0), max(x1 - x0, 0)), np.float32)
    rc = lib().lo_depth_cache_fetch(c.ctypes.data, iw, ih, x0, y0, x1, y1, dims[0], dims[1], out.ctypes.data)
    if rc:
        raise OracleError(rc, "depth_cache_fetch")
    return out


def traversal_trace(w, h, tile, xsw=False):
    """Per Pixel() call of the reference traversal: (dir, x, y, r, is_revisit, src0..src3) as an (n, 9) int array."""
    cap = 2 * w * h * 2 + 64
    buf = np.empty(cap * 9, np.int32)
    n = lib().lo_traversal_trace(w, h, tile, 1 if xsw else 0, buf.ctypes.data, cap)
    if n < 0:
        raise OracleError(-1, "traversal_trace")
    return buf[: n * 9].reshape(n, 9).copy()


def skip_mask(mode, w, h):
    out = np.empty(w * h, np.uint8)
    rc = lib().lo_skip_mask(mode, w, h, out.ctypes.data)
    if rc:
        raise OracleError(rc, "skip_mask")
    return out.reshape(h, w)


def mt19937_stream(seed, n):
    st = ctypes.create_string_buffer(624 * 4 + 16)
    lib().lo_mt_seed(st, seed)
    return np.array([lib().lo_mt_next(st) for _ in range(n)], np.uint32)


# ---------------- dump formats (StereoAsyncApi.cs:197-262), restated for the tests ----------------

def _hdr(w, h, bpp):
    return np.array([w, h, w, bpp], "<i4").tobytes()


def f32_bytes(a):
    """DumpF32 (StereoAsyncApi.cs:252-256)."""
    a = np.ascontiguousarray(a, "<f4")
    return _hdr(a.shape[1], a.shape[0], 4) + a.tobytes()


def rgba8_bytes(img):
    """DumpRgba8 (StereoAsyncApi.cs:217-223)."""
    a = np.ascontiguousarray(img, np.uint8)
    return _hdr(a.shape[1], a.shape[0], 4) + a.tobytes()


def cost_volume_bytes(L):
    """DumpCostVolume (StereoAsyncApi.cs:227-250) of an oracle layer dict: {suffix: bytes} for _offsets.u32, _costvol.bin
    and, when the layer kept them, _costvol_pass1.bin."""
    w, h = L["W"], L["H"]
    start, count, cap, skip = (np.asarray(L[k]).reshape(-1) for k in ("Start", "Count", "Cap", "Skip"))
    off = L["Offsets"]
    sizes = 8 + cap.astype(np.int64) * np.where(skip == 0, 3, 2)
    boff = (np.concatenate([[0], np.cumsum(sizes)[:-1]]) & 0xFFFFFFFF).astype("<u4")
    out = {"_offsets.u32": _hdr(w, h, 4) + boff.tobytes()}

    def body(agg):
        parts = []
        for i in range(w * h):
            o, c = int(off[i]), int(cap[i])
            parts.append(np.array([start[i], count[i], 1, c], "<u2").tobytes())
            parts.append(np.ascontiguousarray(agg[o:o + c], "<u2").tobytes())
            if skip[i] == 0:
                parts.append(L["Raw"][o:o + c].tobytes())
        return b"".join(parts)

    out["_costvol.bin"] = body(L["Agg"])
    if L.get("AggPass1") is not None:
        out["_costvol_pass1.bin"] = body(L["AggPass1"])
    return out


def dense_dump_bytes(layers, images, filtered, calibs, cv_max=2):
    """The files of State4And5's dense dump (StereoAsyncApi.cs:197-214), as {name after the prefix: bytes}."""
    out = {}
    for i, L in enumerate(layers):
        p = f"_dense_L{i}"
        out[p + "_depth.f32"] = f32_bytes(L["Depth"])
        out[p + "_planes.f32"] = np.ascontiguousarray(L["Planes"], "<f4").tobytes()
        out[p + "_skip.u8"] = _hdr(L["W"], L["H"], 1) + np.ascontiguousarray(L["Skip"], np.uint8).tobytes()
        if i == 0:
            out[p + "_guidance.img"] = rgba8_bytes(L["Guidance"])
        if i <= cv_max:
            for k, v in cost_volume_bytes(L).items():
                out[p + k] = v
    cb = bytearray(len(calibs) * 0xA8)
    for c, cal in enumerate(calibs):
        cb[c * 0xA8:c * 0xA8 + 36] = np.asarray(cal.K, "<f4").reshape(9).tobytes()
        cb[c * 0xA8 + 0x24:c * 0xA8 + 0x30] = np.asarray(cal.T, "<f4").reshape(3).tobytes()
        cb[c * 0xA8 + 0x30:c * 0xA8 + 0x54] = np.asarray(cal.R, "<f4").reshape(9).tobytes()
    out["_dense_calibs.bin"] = bytes(cb)
    for k, (im, fi) in enumerate(zip(images, filtered)):
        out[f"_dense_img{k}.img"] = rgba8_bytes(im)
        out[f"_dense_filt{k}.img"] = rgba8_bytes(fi)
    return out


# ---------------- stereo-image formation after the ISP (StereoImage.cs, ReferenceGuide.cs) ----------------

def _aligned(ac):
    a = LoAligned()
    for i, v in enumerate(np.asarray(ac.H, np.float32).reshape(9)):
        a.H[i] = float(v)
    lut = np.ascontiguousarray(np.asarray(ac.lut, np.float32))
    assert lut.size == 4096
    a.lut = lut.ctypes.data
    a.cx, a.cy, a.sx, a.sy = float(ac.cx), float(ac.cy), float(ac.sx), float(ac.sy)
    return a, lut


def wine_sinf(x):
    return lib().lo_wine_sinf(float(np.float32(x)))


def gamma_encode(m):
    return np.float32(lib().lo_gamma_encode(float(np.float32(m))))


def lanczos_table():
    """StereoImage.LanczosTable (StereoImage.cs:212-237): (64, 6) float32."""
    t = np.empty(384, np.float32)
    lib().lo_lanczos_table(t.ctypes.data)
    return t.reshape(64, 6)


def yuv_matrix(sensor_type, neutral):
    """StereoImage.YuvMatrix (StereoImage.cs:140-160): (3, 4) float32 rows (v, u', t')."""
    n = np.ascontiguousarray(np.asarray(neutral, np.float32).reshape(3))
    M = np.empty((3, 4), np.float32)
    lib().lo_yuv_matrix(int(sensor_type), n.ctypes.data, M.ctypes.data)
    return M


def warp_f32(src, gain, dw, dh, ac):
    """StereoImage.Warp (StereoImage.cs:249-296) of an (sh, sw, 4) float32 image scaled by gain first."""
    s = np.ascontiguousarray(np.asarray(src, np.float32))
    sh, sw = s.shape[:2]
    a, keep = _aligned(ac)
    out = np.empty((dh, dw, 4), np.float32)
    rc = lib().lo_warp_f32(s.ctypes.data, sw, sh, float(np.float32(gain)), dw, dh, ctypes.byref(a), out.ctypes.data)
    if rc:
        raise OracleError(rc, "warp_f32")
    return out


def convert_yuv(rgba, M):
    """StereoImage.ConvertToYuv (StereoImage.cs:181-195) on a copy."""
    out = np.array(rgba, np.float32, copy=True, order="C")
    m = np.ascontiguousarray(M, np.float32)
    lib().lo_convert_yuv(out.ctypes.data, out.size // 4, m.ctypes.data)
    return out


def to_rgba8(rgba):
    """StereoImage.ToRgba8 (StereoImage.cs:198-209)."""
    r = np.ascontiguousarray(rgba, np.float32)
    out = np.empty(r.shape, np.uint8)
    lib().lo_to_rgba8(r.ctypes.data, r.size, out.ctypes.data)
    return out


def stereo_image(src, gain, dw, dh, ac, sensor_type, neutral):
    """StereoImageBuilder.Create, colour path after the ISP (StereoImageBuilder.cs:61-69, 78): gain, warp, YUV, 8 bits.
    Returns (rgba8, yuv float image)."""
    yuv = convert_yuv(warp_f32(src, gain, dw, dh, ac), yuv_matrix(sensor_type, neutral))
    return to_rgba8(yuv), yuv


def warp_rgba8(src, dw, dh, ac):
    """Rgba8Warp.Warp (ReferenceGuide.cs:108-156) of an (sh, sw, 4) uint8 image."""
    s = np.ascontiguousarray(np.asarray(src, np.uint8))
    sh, sw = s.shape[:2]
    a, keep = _aligned(ac)
    out = np.empty((dh, dw, 4), np.uint8)
    rc = lib().lo_warp_rgba8(s.ctypes.data, sw, sh, dw, dh, ctypes.byref(a), out.ctypes.data)
    if rc:
        raise OracleError(rc, "warp_rgba8")
    return out


def color_transfer(work, ref, calib2, calibA):
    """StereoColorTransfer.Transfer (StereoColorTransfer.cs:128-138): (out YUVA floats, F 4x4, crop rect, N work, N ref)."""
    wk = np.ascontiguousarray(np.asarray(work, np.float32))
    rf = np.ascontiguousarray(np.asarray(ref, np.float32))
    h, w = wk.shape[:2]
    rh, rw = rf.shape[:2]
    out = np.empty_like(wk)
    F = np.empty(16, np.float32)
    crop = np.empty(4, np.int32)
    nw, nr = ctypes.c_float(), ctypes.c_float()
    lib().lo_color_transfer(wk.ctypes.data, w, h, rf.ctypes.data, rw, rh, _calibs([calib2]), _calibs([calibA]), out.ctypes.data,
                            F.ctypes.data, crop.ctypes.data, ctypes.byref(nw), ctypes.byref(nr))
    return out, F.reshape(4, 4), tuple(int(v) for v in crop), nw.value, nr.value


def stereo_image_transfer(src, gain, dw, dh, ac, sensor_type, neutral, ref_yuv, ref_view, view):
    """StereoImageBuilder.Create for a non-reference module with the reference crop (StereoImageBuilder.cs:61-65, 71-77):
    (rgba8, F)."""
    yuv = convert_yuv(warp_f32(src, gain, dw, dh, ac), yuv_matrix(sensor_type, neutral))
    out, F, crop, nw, nr = color_transfer(yuv, ref_yuv, ref_view, view)
    return to_rgba8(out), F
