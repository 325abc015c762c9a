"""Host-side mirror of Lux.Engine's dense-stereo interface, backed by the CUDA library through its C ABI.

Names and argument meanings follow the reference:
  * StereoParams / StereoParams.l16_pyramid()      Lux.Engine/Pipeline/Registration/DenseStereo.cs:15-31
  * DenseStereo.planes(...)                        DenseStereo.cs:41-88
  * DenseStereo.box_filter3(...)                   DenseStereo.cs:93-123
  * DenseLayer (init + compute on the GPU)         DenseStereoSgm.cs:13-232
  * DenseStereoPyramid.run(...)                    DenseStereoSgm.cs:331-353
  * DenseUpsampleLayer.run(...)                    DenseUpsampleLayer.cs:35-48
Errors raise the exception class the reference throws (InvalidOperationError, NotSupportedError, IndexError), each
carrying the C status code.
"""
import ctypes
import os
import struct
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib as L


class LuxError(L.LuxError):
    pass


class InvalidOperationError(LuxError):
    """InvalidOperationException of the reference (planes, upsample size)."""


class NotSupportedError(LuxError):
    """NotSupportedException of the reference (skip mode, memory budget)."""


class LuxIndexError(LuxError, IndexError):
    """The reference indexes outside an array for these inputs (IndexOutOfRangeException)."""


class OperationCanceledError(LuxError):
    """OperationCanceledException of the reference: a request canceled before it started."""


_EXC = {1: InvalidOperationError, 2: InvalidOperationError, 3: InvalidOperationError, 6: InvalidOperationError,
        4: NotSupportedError, 5: NotSupportedError, 7: LuxIndexError, 13: OperationCanceledError, 14: InvalidOperationError,
        15: InvalidOperationError, 17: InvalidOperationError}


def _raise(code, msg):
    raise _EXC.get(code, LuxError)(code, msg)


def _f32bits(u):
    return struct.unpack("<f", struct.pack("<I", u))[0]


@dataclass
class StereoParams:
    """StereoParams (DenseStereo.cs:15-21), the fields the dense path reads."""
    margin: int = 1
    plane_density: float = 2.0
    scale: int = 32
    skip_mode: int = 0
    p1: int = 1
    p2scale: float = 500.0
    guidance: tuple = field(default_factory=lambda: (np.float32(_f32bits(0x3ef6384f)) / np.float32(6),
                                                     np.float32(_f32bits(0x3ef6384f)) / np.float32(16),
                                                     np.float32(_f32bits(0x3ef6384f)) / np.float32(16), np.float32(0)))
    tile: int = 4

    @staticmethod
    def l16_pyramid() -> List["StereoParams"]:
        """StereoParams.L16Pyramid(false) (DenseStereo.cs:24-30)."""
        scales, tiles = (32, 16, 8, 4, 2, 1), (4, 8, 16, 32, 64, 64)
        return [StereoParams(scale=scales[i], tile=tiles[i], skip_mode=2 if i >= 4 else 0) for i in range(6)]

    def to_c(self):
        p = L.Params()
        p.margin, p.plane_density, p.scale, p.skip_mode = self.margin, self.plane_density, self.scale, self.skip_mode
        p.p1, p.p2scale, p.tile = self.p1, self.p2scale, self.tile
        for i in range(4):
            p.guidance[i] = float(self.guidance[i])
        return p


@dataclass
class CalibData:
    """CalibData (Triangulator.cs:8-19): row-major K (3x3), T (3), R (3x3), X_cam = R·X + t."""
    K: np.ndarray
    T: np.ndarray
    R: np.ndarray

    def to_c(self):
        c = L.Calib()
        for i, v in enumerate(np.asarray(self.K, np.float32).reshape(9)):
            c.K[i] = float(v)
        for i, v in enumerate(np.asarray(self.T, np.float32).reshape(3)):
            c.T[i] = float(v)
        for i, v in enumerate(np.asarray(self.R, np.float32).reshape(9)):
            c.R[i] = float(v)
        return c


def _calibs_c(calibs):
    arr = (L.Calib * len(calibs))()
    for i, c in enumerate(calibs):
        arr[i] = c.to_c()
    return arr


def _img_c(img):
    """A C image from a numpy (H, W, 4) uint8 array or a CUDA torch uint8 tensor of that shape."""
    if hasattr(img, "data_ptr"):  # torch tensor
        h, w, c = img.shape
        assert c == 4 and img.is_contiguous()
        return L.Img(img.data_ptr(), w, h, w, 1 if img.is_cuda else 0), img
    a = np.ascontiguousarray(img, dtype=np.uint8)
    h, w, c = a.shape
    assert c == 4
    return L.Img(a.ctypes.data, w, h, w, 0), a


class Context:
    """One GPU, one stream, an HBM budget (0 = none). Layers created through it keep their state on the device."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.lib = L.load()
        h = ctypes.c_void_p()
        rc = self.lib.lux_sgm_create(device, hbm_budget_bytes, ctypes.byref(h))
        if rc:
            _raise(rc, "lux_sgm_create failed")
        self.handle = h
        self.device = device

    def check(self, rc):
        if rc:
            _raise(rc, self.lib.lux_sgm_last_error(self.handle).decode())

    @property
    def wait_limit_ns(self) -> int:
        """The bound of every device-side wait of the aggregation kernels (ns; default 20 s)."""
        return int(self.lib.lux_sgm_get_wait_limit(self.handle))

    @wait_limit_ns.setter
    def wait_limit_ns(self, ns: int):
        self.check(self.lib.lux_sgm_set_wait_limit(self.handle, int(ns)))

    def set_autotune(self, on: bool):
        """Untuned uniform layer shapes time every fast aggregation form on their first solve (the default) or not."""
        self.check(self.lib.lux_sgm_set_autotune(self.handle, 1 if on else 0))

    def debug_stall(self, block: int):
        """Failure-path tests only: aggregation block `block` (>= 1) waits on a counter nothing publishes (-1: off)."""
        self.check(self.lib.lux_sgm_debug_stall(self.handle, int(block)))

    def close(self):
        if self.handle:
            self.lib.lux_sgm_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def _flags(keep_pass1, keep_agg, prefilter, force_replay, sgm="auto"):
    if sgm not in ("auto", "fused", "split", "wave"):
        raise ValueError(f"sgm must be 'auto', 'fused', 'split' or 'wave', not {sgm!r}")
    return ((L.LAYER_KEEP_PASS1 if keep_pass1 else 0) | (L.LAYER_KEEP_AGG if keep_agg else 0) |
            (L.LAYER_PREFILTER if prefilter else 0) | (L.LAYER_FORCE_REPLAY if force_replay else 0) |
            (L.LAYER_SGM_FUSED if sgm == "fused" else 0) | (L.LAYER_SGM_SPLIT if sgm == "split" else 0) |
            (L.LAYER_SGM_WAVE if sgm == "wave" else 0))


def revisit_schedule(w, h, tile, second_pass):
    """The revisit schedule of the fast uniform kernel (diagnostic): (h, 7) int32 rows, pass +1's last odd row, and the
    (first, count) of the revisits the last row runs after its own visit."""
    out = np.zeros(7 * h + 2, np.int32)
    yb = ctypes.c_int32()
    rc = L.load().lux_sgm_revisit_schedule(w, h, tile, 1 if second_pass else 0, out.ctypes.data, ctypes.byref(yb))
    if rc:
        _raise(rc, "lux_sgm_revisit_schedule failed")
    return out[: 7 * h].reshape(h, 7), yb.value, (int(out[7 * h]), int(out[7 * h + 1]))


def kernel_launches() -> int:
    """Kernels the CUDA library has launched in this process."""
    return int(L.load().lux_sgm_kernel_launches())


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class DenseStereo:
    @staticmethod
    def planes(near, far, calibs: Sequence[CalibData], density, align) -> np.ndarray:
        """DenseStereo.Planes (DenseStereo.cs:41-88): metric plane depths, plane 0 = far .. n-1 = near."""
        lib = L.load()
        out = (ctypes.c_float * (4096 + max(int(align), 1) + 8))()
        n = ctypes.c_int32()
        cc = _calibs_c(calibs)
        rc = lib.lux_sgm_planes(near, far, cc, len(calibs), density, align, out, ctypes.byref(n))
        if rc:
            _raise(rc, {1: "The near end has to be smaller than the fard end!", 2: "Both the near and far end have to be positive!",
                        3: "Baseline too small, check calibration."}.get(rc, "planes failed"))
        return np.frombuffer(out, dtype=np.float32, count=n.value).copy()

    @staticmethod
    def box_filter3(img, ctx: Optional[Context] = None) -> np.ndarray:
        """DenseStereo.BoxFilter3 (DenseStereo.cs:93-123) on the GPU."""
        ctx = ctx or default_context()
        ci, keep = _img_c(img)
        out = np.empty((ci.h, ci.w, 4), np.uint8)
        ctx.check(ctx.lib.lux_sgm_box_filter3(ctx.handle, ctypes.byref(ci), out.ctypes.data))
        return out


def image_from_grey16(samples, bits: int = 12, ctx: Optional[Context] = None, out=None):
    """A grey camera image of `bits` bits per sample (uint16; a numpy array or a torch tensor, host or CUDA) made into the
    reference's grey Rgba8Image bytes (Y, 128, 128, 255), Y = (v + 2^(bits-9)) >> (bits - 8) saturated, on the GPU: a CUDA
    uint8 tensor (h, w, 4) usable as an on-device image of DenseLayer.compute. Host samples cross as 2 bytes a pixel."""
    import torch
    ctx = ctx or default_context()
    if hasattr(samples, "data_ptr"):
        h, w = samples.shape
        assert samples.element_size() == 2
        on_dev, ptr, stride = (1 if samples.is_cuda else 0), samples.data_ptr(), samples.stride(0)
        _torch_ready(samples)
    else:
        a = np.ascontiguousarray(samples, np.uint16)
        h, w = a.shape
        on_dev, ptr, stride = 0, a.ctypes.data, w
    if out is None:
        out = torch.empty((h, w, 4), dtype=torch.uint8, device=torch.device("cuda", ctx.device))
    ctx.check(ctx.lib.lux_image_from_grey16(ctx.handle, ptr, w, h, stride, on_dev, int(bits), out.data_ptr()))
    return out


class DenseLayer:
    """A computed DenseLayer (DenseStereoSgm.cs:13-232) whose state lives on the GPU until close()."""

    def __init__(self, ctx: Context, handle):
        self.ctx = ctx
        self.handle = handle
        info = L.LayerInfo()
        ctx.check(ctx.lib.lux_layer_get_info(handle, ctypes.byref(info)))
        self.W, self.H, self.Index, self.Align = info.w, info.h, info.index, info.align
        self.n_planes, self.MinLo, self.MaxHi, self.Tile = info.n_planes, info.min_lo, info.max_hi, info.tile
        self.volume = info.volume
        self.gpu_ms_cost, self.gpu_ms_sgm, self.gpu_ms_wta = info.gpu_ms_cost, info.gpu_ms_sgm, info.gpu_ms_wta
        self.sgm_kernel = info.sgm_kernel
        self.cost_kernel = info.cost_kernel
        self.tuned = info.tuned

    @staticmethod
    def compute(images, gray, calibs, near, far, params: StereoParams, index=0, align=8, prev: Optional["DenseLayer"] = None,
                keep_pass1=False, prefilter=False, keep_agg=False, force_replay=False, sgm="auto",
                ctx: Optional[Context] = None) -> "DenseLayer":
        """DenseLayer.Init + Compute (DenseStereoSgm.cs:34-62, 181-232). images: RGBA8 (camera 0 = reference), box-filtered
        already unless prefilter=True (then BoxFilter3 runs on the GPU first, as DenseStereoPyramid.Run does).
        keep_pass1 / keep_agg keep DenseLayer.AggPass1 / Agg readable (the depth needs neither); force_replay aggregates
        with the exact traversal replay kernel even where the fast uniform kernel applies; sgm picks the form of the fast
        kernel ("fused" four-path wavefront, "split" path-group chains, "auto" by size)."""
        ctx = ctx or default_context()
        arr = (L.Img * len(images))()
        keep = []
        for i, im in enumerate(images):
            ci, k = _img_c(im)
            arr[i] = ci
            keep.append(k)
        g = np.ascontiguousarray(np.asarray(gray, dtype=np.uint8))
        cc = _calibs_c(calibs)
        p = params.to_c()
        out = ctypes.c_void_p()
        rc = ctx.lib.lux_sgm_layer(ctx.handle, len(images), arr, g.ctypes.data, cc, near, far, ctypes.byref(p), index, align,
                                   prev.handle if prev is not None else None,
                                   _flags(keep_pass1, keep_agg, prefilter, force_replay, sgm), ctypes.byref(out))
        ctx.check(rc)
        return DenseLayer(ctx, out)

    @staticmethod
    def from_depth(depth, skip=None, ctx: Optional[Context] = None) -> "DenseLayer":
        """A previous layer made from a stored depth map (h, w) float32 and skip mask (0 = computed; None: all computed),
        for resuming a pyramid from a dumped layer: the next layer's RangeFromPrevious reads only these two fields."""
        ctx = ctx or default_context()
        d = np.ascontiguousarray(np.asarray(depth, np.float32))
        h, w = d.shape
        sk = None if skip is None else np.ascontiguousarray(np.asarray(skip, np.uint8).reshape(h, w))
        out = ctypes.c_void_p()
        ctx.check(ctx.lib.lux_layer_from_depth(ctx.handle, w, h, d.ctypes.data, None if sk is None else sk.ctypes.data,
                                               ctypes.byref(out)))
        return DenseLayer(ctx, out)

    def _read(self, field_id, dtype, count):
        out = np.empty(count, dtype=dtype)
        self.ctx.check(self.ctx.lib.lux_layer_read(self.handle, field_id, out.ctypes.data, out.nbytes))
        return out

    @property
    def Depth(self):
        return self._read(L.FIELD_DEPTH, np.float32, self.W * self.H).reshape(self.H, self.W)

    @property
    def Planes(self):
        return self._read(L.FIELD_PLANES, np.float32, self.n_planes)

    @property
    def Skip(self):
        return self._read(L.FIELD_SKIP, np.uint8, self.W * self.H).reshape(self.H, self.W)

    @property
    def Start(self):
        return self._read(L.FIELD_START, np.uint16, self.W * self.H).reshape(self.H, self.W)

    @property
    def Count(self):
        return self._read(L.FIELD_COUNT, np.uint16, self.W * self.H).reshape(self.H, self.W)

    @property
    def Cap(self):
        return self._read(L.FIELD_CAP, np.uint16, self.W * self.H).reshape(self.H, self.W)

    @property
    def Offsets(self):
        return self._read(L.FIELD_OFFSETS, np.uint64, self.W * self.H + 1)

    @property
    def Agg(self):
        """Final aggregates, CSR-flat: pixel i owns [Offsets[i], Offsets[i] + Cap[i])."""
        return self._read(L.FIELD_AGG, np.uint16, self.volume)

    @property
    def AggPass1(self):
        return self._read(L.FIELD_AGG_PASS1, np.uint16, self.volume)

    @property
    def Raw(self):
        return self._read(L.FIELD_RAW, np.uint8, self.volume)

    @property
    def Guidance(self):
        return self._read(L.FIELD_GUIDANCE, np.uint8, self.W * self.H * 4).reshape(self.H, self.W, 4)

    def dump_cost_volume(self, prefix):
        """DumpCostVolume (StereoAsyncApi.cs:227-250): <prefix>_offsets.u32, _costvol.bin, _costvol_pass1.bin (when kept).
        Needs the final aggregates (keep_agg=True on the fast kernels)."""
        self.ctx.check(self.ctx.lib.lux_dump_cost_volume(self.handle, os.fsencode(prefix)))

    def device_ptr(self, field_id):
        return self.ctx.lib.lux_layer_device_ptr(self.handle, field_id)

    def close(self):
        if self.handle:
            self.ctx.lib.lux_layer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DenseStereoPyramid:
    @staticmethod
    def run(images, gray, calibs, near=200.0, far=640000.0, keep_pass1=False, keep_agg=False, force_replay=False,
            sgm="auto", ctx: Optional[Context] = None) -> List[DenseLayer]:
        """DenseStereoPyramid.Run (DenseStereoSgm.cs:331-353): the raw (unfiltered) camera images in, six layers out."""
        ctx = ctx or default_context()
        arr = (L.Img * len(images))()
        keep = []
        for i, im in enumerate(images):
            ci, k = _img_c(im)
            arr[i] = ci
            keep.append(k)
        g = np.ascontiguousarray(np.asarray(gray, dtype=np.uint8))
        cc = _calibs_c(calibs)
        outs = (ctypes.c_void_p * 6)()
        ctx.check(ctx.lib.lux_sgm_pyramid(ctx.handle, len(images), arr, g.ctypes.data, cc, near, far,
                                          _flags(keep_pass1, keep_agg, False, force_replay, sgm), outs))
        return [DenseLayer(ctx, ctypes.c_void_p(outs[i])) for i in range(6)]


@dataclass
class UpsampleResult:
    Depth: np.ndarray
    W: int
    H: int
    Confidence: Optional[np.ndarray] = None


class DenseUpsampleLayer:
    Sigma = 12.0
    Scale = 2

    @staticmethod
    def run(prev_depth, pw, ph, guide, set_w, set_h, sigma=12.0, scale=2, prev_confidence=None,
            ctx: Optional[Context] = None) -> UpsampleResult:
        """DenseUpsampleLayer.Run (DenseUpsampleLayer.cs:35-48) on the GPU."""
        ctx = ctx or default_context()
        gi, gkeep = _img_c(guide)
        prev = np.ascontiguousarray(np.asarray(prev_depth, np.float32).reshape(-1))
        out = np.empty(gi.w * gi.h, np.float32)
        conf_out = None
        conf_ptr = None
        cin = None
        if prev_confidence is not None:
            cin = np.ascontiguousarray(np.asarray(prev_confidence, np.float32).reshape(-1))
            conf_out = np.empty(gi.w * gi.h, np.float32)
            conf_ptr = conf_out.ctypes.data
        rc = ctx.lib.lux_sgm_upsample(ctx.handle, prev.ctypes.data, pw, ph, 0, ctypes.byref(gi), set_w, set_h, sigma, scale,
                                      cin.ctypes.data if cin is not None else None, out.ctypes.data, conf_ptr)
        ctx.check(rc)
        return UpsampleResult(out.reshape(gi.h, gi.w), gi.w, gi.h,
                              conf_out.reshape(gi.h, gi.w) if conf_out is not None else None)


def dump_f32(path, data):
    """DumpF32 (StereoAsyncApi.cs:252-256): int32 {w, h, w, 4} then the rows of a 2-D float32 array."""
    d = np.ascontiguousarray(np.asarray(data, np.float32))
    h, w = d.shape
    rc = L.load().lux_dump_f32(os.fsencode(path), d.ctypes.data, w, h)
    if rc:
        _raise(rc, f"lux_dump_f32 {path}")


def load_f32(path):
    """LoadF32 (StereoAsyncApi.cs:257-261), as LUX_DENSE_OVERRIDE reads a layer-5 depth: the (h, w) float32 array."""
    lib = L.load()
    w, h = ctypes.c_int32(), ctypes.c_int32()
    rc = lib.lux_load_f32(os.fsencode(path), None, 0, ctypes.byref(w), ctypes.byref(h))
    if rc == 0:
        out = np.empty((h.value, w.value), np.float32)
        rc = lib.lux_load_f32(os.fsencode(path), out.ctypes.data, out.size, ctypes.byref(w), ctypes.byref(h))
    if rc:
        _raise(rc, {17: f"{path}: expected a 4-byte float dump"}.get(rc, f"lux_load_f32 {path}"))
    return out


def dump_rgba8(path, img):
    """DumpRgba8 (StereoAsyncApi.cs:217-223): int32 {w, h, w, 4} then the rows of an (h, w, 4) uint8 image."""
    ci, keep = _img_c(img)
    rc = L.load().lux_dump_rgba8(os.fsencode(path), ctypes.byref(ci))
    if rc:
        _raise(rc, f"lux_dump_rgba8 {path}")


def dump_dense(prefix, layers, images, calibs, cv_max=2, ctx: Optional[Context] = None):
    """The dense dump of State4And5 (StereoAsyncApi.cs:197-214) for solved layers and their raw input images:
    <prefix>_dense_L<i>_{depth.f32, planes.f32, skip.u8}, _dense_L0_guidance.img, _dense_calibs.bin,
    _dense_img<k>.img, _dense_filt<k>.img and the cost volumes of layers 0..cv_max."""
    ctx = ctx or default_context()
    arr = (L.Img * len(images))()
    keep = []
    for i, im in enumerate(images):
        ci, k = _img_c(im)
        arr[i] = ci
        keep.append(k)
    hs = (ctypes.c_void_p * len(layers))(*[l.handle.value if hasattr(l.handle, "value") else l.handle for l in layers])
    ctx.check(ctx.lib.lux_dump_dense(ctx.handle, hs, len(layers), len(images), arr, _calibs_c(calibs), os.fsencode(prefix),
                                     cv_max))


def _f32_image(a):
    """(pointer, on_device, keep-alive, (h, w)) of a 2-D float32 image: a numpy array or a contiguous CUDA torch tensor."""
    if hasattr(a, "data_ptr"):
        assert a.dim() == 2 and a.is_contiguous() and str(a.dtype) == "torch.float32"
        return a.data_ptr(), 1 if a.is_cuda else 0, a, tuple(a.shape)
    d = np.ascontiguousarray(np.asarray(a, np.float32))
    assert d.ndim == 2
    return d.ctypes.data, 0, d, d.shape


def _torch_ready(*arrays):
    """Work torch queued on its current stream for these CUDA tensors is done before the library's stream reads them."""
    for a in arrays:
        if hasattr(a, "is_cuda") and a.is_cuda:
            import torch
            torch.cuda.current_stream(a.device).synchronize()
            return


def _f32_like(ref, h, w):
    if hasattr(ref, "data_ptr"):
        import torch
        return torch.empty((h, w), dtype=torch.float32, device=ref.device)
    return np.empty((h, w), np.float32)


class DepthImageCache:
    """DepthImageCache (DepthCache.cs:87-254) on the GPU: the depth image the renderer and exporter read, made from the
    upsampled full-resolution depth. Current is a numpy array, or a CUDA torch tensor (device=True) that stays in HBM:
    Set and Fetch then read and write device memory only."""
    Clip = 100000.0

    def __init__(self, dims, device: bool = False, ctx: Optional[Context] = None):
        """The constructor (:96): a zero image at dims = (W, H)."""
        self.ctx = ctx or default_context()
        w, h = dims
        if device:
            import torch
            self.Current = torch.zeros((h, w), dtype=torch.float32, device=f"cuda:{self.ctx.device}")
        else:
            self.Current = np.zeros((h, w), np.float32)

    def Set(self, depth):
        """Set (:136-143): inverse depth, nearest resample to the cache dims, min(rcp, 1e5); the result is published."""
        ptr, on_dev, keep, (h, w) = _f32_image(depth)
        ch, cw = self.Current.shape
        out = _f32_like(self.Current, ch, cw)
        optr, oon, okeep, _ = _f32_image(out)
        _torch_ready(depth, out)
        self.ctx.check(self.ctx.lib.lux_depth_cache_set(self.ctx.handle, ptr, w, h, on_dev, cw, ch, optr, oon))
        self.ctx.check(self.ctx.lib.lux_sgm_sync(self.ctx.handle))  # device in and out: the call is asynchronous
        self.Current = out

    def Fetch(self, rect, dims):
        """Fetch (:146) on the published image."""
        return DepthImageCache.fetch(self.Current, rect, dims, self.ctx)

    @staticmethod
    def fetch(img, rect, dims, ctx: Optional[Context] = None):
        """Fetch(img, rect, dims) (:161-181): rect = (x0, y0, x1, y1) in the grid of dims = (W, H); the ROI at that grid
        as a (y1 - y0, x1 - x0) image of the same kind as img. Raises InvalidOperationError("invalid ROI requested!")."""
        ctx = ctx or default_context()
        ptr, on_dev, keep, (ch, cw) = _f32_image(img)
        x0, y0, x1, y1 = (int(v) for v in rect)
        out = _f32_like(img, max(y1 - y0, 0), max(x1 - x0, 0))
        optr, oon, okeep, _ = _f32_image(out)
        _torch_ready(img, out)
        ctx.check(ctx.lib.lux_depth_cache_fetch(ctx.handle, ptr, cw, ch, on_dev, x0, y0, x1, y1, int(dims[0]), int(dims[1]),
                                                optr, oon))
        ctx.check(ctx.lib.lux_sgm_sync(ctx.handle))
        return out


@dataclass
class AlignedCalib:
    """AlignedCalib (Lux.Engine/Pipeline/Geometry/AlignedCalibration.cs:149-178) as AlignedCalib.Build leaves it: the
    row-major homography H (view -> module), the 4096 CRA factors lut, the centre (Cx, Cy) and the scales (Sx, Sy)."""
    H: np.ndarray
    lut: np.ndarray
    cx: float
    cy: float
    sx: float
    sy: float

    def to_c(self):
        c = L.AlignedCalib()
        for i, v in enumerate(np.asarray(self.H, np.float32).reshape(9)):
            c.H[i] = float(v)
        lut = np.ascontiguousarray(np.asarray(self.lut, np.float32))
        if lut.size != 4096:
            raise ValueError("the CRA lut has 4096 entries")
        c.lut = lut.ctypes.data
        c.cx, c.cy, c.sx, c.sy = float(self.cx), float(self.cy), float(self.sx), float(self.sy)
        return c, lut


def _image_f32(a):
    """(pointer, on_device, keep-alive, (h, w)) of an (h, w, 4) float32 image: numpy or a contiguous CUDA torch tensor."""
    if hasattr(a, "data_ptr"):
        assert a.dim() == 3 and a.shape[2] == 4 and a.is_contiguous() and str(a.dtype) == "torch.float32"
        return a.data_ptr(), 1 if a.is_cuda else 0, a, tuple(a.shape[:2])
    d = np.ascontiguousarray(np.asarray(a, np.float32))
    assert d.ndim == 3 and d.shape[2] == 4
    return d.ctypes.data, 0, d, d.shape[:2]


def _empty_like_kind(ref, shape, dtype):
    if hasattr(ref, "data_ptr") and ref.is_cuda:
        import torch
        return torch.empty(shape, dtype={np.float32: torch.float32, np.uint8: torch.uint8}[dtype], device=ref.device)
    return np.empty(shape, dtype)


def _ptr(a):
    return (a.data_ptr(), 1 if a.is_cuda else 0) if hasattr(a, "data_ptr") else (a.ctypes.data, 0)


class StereoImage:
    """Stereo-image formation after the ISP (StereoImage.cs, StereoImageBuilder.cs:45-79, colour sensors) on the GPU.
    Images are numpy arrays or CUDA torch tensors; outputs are of the kind of the source."""

    @staticmethod
    def lanczos_table() -> np.ndarray:
        """LanczosTable (StereoImage.cs:212-237): (64, 6) float32."""
        out = np.empty(384, np.float32)
        L.load().lux_lanczos_table(out.ctypes.data)
        return out.reshape(64, 6)

    @staticmethod
    def yuv_matrix(sensor_type, neutral) -> np.ndarray:
        """YuvMatrix (StereoImage.cs:140-160): (3, 4) float32 rows (v, u', t')."""
        n = np.ascontiguousarray(np.asarray(neutral, np.float32).reshape(3))
        out = np.empty(12, np.float32)
        L.load().lux_yuv_matrix(int(sensor_type), n.ctypes.data, out.ctypes.data)
        return out.reshape(3, 4)

    @staticmethod
    def warp(src, dw, dh, ac: AlignedCalib, gain=1.0, ctx: Optional[Context] = None):
        """Warp (StereoImage.cs:249-296) of an (sh, sw, 4) float image scaled by gain first: (dh, dw, 4) float32."""
        ctx = ctx or default_context()
        ptr, on_dev, keep, (sh, sw) = _image_f32(src)
        out = _empty_like_kind(src, (dh, dw, 4), np.float32)
        optr, oon = _ptr(out)
        c, lut = ac.to_c()
        _torch_ready(src, out)
        ctx.check(ctx.lib.lux_warp_f32(ctx.handle, ptr, sw, sh, on_dev, float(gain), ctypes.byref(c), dw, dh, optr, oon))
        return out

    @staticmethod
    def create(src, dw, dh, ac: AlignedCalib, sensor_type, neutral, gain=1.0, keep_yuv=False, ctx: Optional[Context] = None):
        """StereoImageBuilder.Create after RunIspTiled (StereoImageBuilder.cs:61-69, 78): the (dh, dw, 4) uint8 stereo
        image and, with keep_yuv, its (dh, dw, 4) YUV floats (the reference camera's RefYuv), else None."""
        ctx = ctx or default_context()
        ptr, on_dev, keep, (sh, sw) = _image_f32(src)
        out = _empty_like_kind(src, (dh, dw, 4), np.uint8)
        yuv = _empty_like_kind(src, (dh, dw, 4), np.float32) if keep_yuv else None
        optr, oon = _ptr(out)
        yptr, yon = _ptr(yuv) if yuv is not None else (None, 0)
        n = np.ascontiguousarray(np.asarray(neutral, np.float32).reshape(3))
        c, lut = ac.to_c()
        _torch_ready(src, out, *(() if yuv is None else (yuv,)))
        ctx.check(ctx.lib.lux_stereo_image(ctx.handle, ptr, sw, sh, on_dev, float(gain), ctypes.byref(c), dw, dh, int(sensor_type),
                                           n.ctypes.data, optr, oon, yptr, yon))
        return out, yuv


    @staticmethod
    def create_transfer(src, dw, dh, ac: AlignedCalib, sensor_type, neutral, ref_yuv, ref_view: CalibData, view: CalibData,
                        gain=1.0, ctx: Optional[Context] = None):
        """StereoImageBuilder.Create for a non-reference module with the reference crop (StereoImageBuilder.cs:71-77): the
        (dh, dw, 4) uint8 stereo image colour-matched to the crop of ref_yuv (the reference's YUV floats, from create(...,
        keep_yuv=True)), and the (4, 4) float32 transfer. ref_view / view: the reference's and this module's views."""
        ctx = ctx or default_context()
        ptr, on_dev, keep, (sh, sw) = _image_f32(src)
        rptr, ron, rkeep, _ = _image_f32(ref_yuv)
        out = _empty_like_kind(src, (dh, dw, 4), np.uint8)
        optr, oon = _ptr(out)
        n = np.ascontiguousarray(np.asarray(neutral, np.float32).reshape(3))
        F = np.empty(16, np.float32)
        c, lut = ac.to_c()
        rv, vv = ref_view.to_c(), view.to_c()
        _torch_ready(src, ref_yuv, out)
        ctx.check(ctx.lib.lux_stereo_image_transfer(ctx.handle, ptr, sw, sh, on_dev, float(gain), ctypes.byref(c), dw, dh,
                                                    int(sensor_type), n.ctypes.data, rptr, ron, ctypes.byref(rv), ctypes.byref(vv),
                                                    optr, oon, F.ctypes.data))
        return out, F.reshape(4, 4)


class Rgba8Warp:
    @staticmethod
    def warp(src, dw, dh, ac: AlignedCalib, ctx: Optional[Context] = None):
        """Rgba8Warp.Warp (ReferenceGuide.cs:108-156): the reference guide's 8-bit warp of an (sh, sw, 4) uint8 image."""
        ctx = ctx or default_context()
        ci, keep = _img_c(src)
        out = _empty_like_kind(src, (dh, dw, 4), np.uint8)
        optr, oon = _ptr(out)
        c, lut = ac.to_c()
        _torch_ready(src, out)
        ctx.check(ctx.lib.lux_warp_rgba8(ctx.handle, ctypes.byref(ci), ctypes.byref(c), dw, dh, optr, oon))
        return out


class CensusStereo:
    """The opt-in census stereo mode of a rectified grey pair (no counterpart in the reference): census 9x7, Hamming cost,
    8-path SGM with constant P1/P2, first-minimum WTA, parabolic subpixel, left/right check (-1 where it fails)."""

    @staticmethod
    def compute(left, right, max_disparity, p1=10, p2=120, subpixel=True, lr_check=True, lr_max_diff=1,
                ctx: Optional[Context] = None):
        """left, right: (h, w, 4) uint8 (grey in channel 0) or (h, w) uint8. Returns (h, w) float32 disparities."""
        ctx = ctx or default_context()
        imgs = []
        for im in (left, right):
            if not hasattr(im, "data_ptr") and np.asarray(im).ndim == 2:
                im = np.repeat(np.asarray(im, np.uint8)[..., None], 4, axis=2)
            imgs.append(_img_c(im))
        (cl, kl), (cr, kr) = imgs
        prm = L.CensusParams(int(max_disparity), int(p1), int(p2), 1 if subpixel else 0, 1 if lr_check else 0, int(lr_max_diff))
        out = _empty_like_kind(left if hasattr(left, "data_ptr") else np.empty(0), (cl.h, cl.w), np.float32)
        optr, oon = _ptr(out)
        _torch_ready(left, right, out)
        ctx.check(ctx.lib.lux_census_sgm(ctx.handle, ctypes.byref(cl), ctypes.byref(cr), ctypes.byref(prm), optr, oon))
        return out

    @staticmethod
    def capture(ref, others, max_disparities, fbs, p1=10, p2=120, subpixel=True, lr_check=True, lr_max_diff=1,
                ctx: Optional[Context] = None):
        """A capture's pairs in one batch (the reference image against each other image, all on the reference's grid):
        (fused (h, w) float32 depth, (n, h, w) float32 disparities)."""
        ctx = ctx or default_context()

        def rgba(im):
            if not hasattr(im, "data_ptr") and np.asarray(im).ndim == 2:
                return np.repeat(np.asarray(im, np.uint8)[..., None], 4, axis=2)
            return im
        cr, kr = _img_c(rgba(ref))
        oth = (L.Img * len(others))()
        keep = []
        for i, im in enumerate(others):
            ci, k = _img_c(rgba(im))
            oth[i] = ci
            keep.append(k)
        ds = np.ascontiguousarray(np.asarray(max_disparities, np.int32))
        fb = np.ascontiguousarray(np.asarray(fbs, np.float32))
        prm = L.CensusParams(0, int(p1), int(p2), 1 if subpixel else 0, 1 if lr_check else 0, int(lr_max_diff))
        depth = np.empty((cr.h, cr.w), np.float32)
        disps = np.empty((len(others), cr.h, cr.w), np.float32)
        _torch_ready(ref, *others)
        ctx.check(ctx.lib.lux_census_capture(ctx.handle, len(others), ctypes.byref(cr), oth, ds.ctypes.data, fb.ctypes.data,
                                             ctypes.byref(prm), depth.ctypes.data, 0, disps.ctypes.data))
        return depth, disps

    @staticmethod
    def fuse(disps, fbs, ctx: Optional[Context] = None):
        """The median depth over the pairs' valid disparities (fB / d for d > 0), 0 where none is valid."""
        ctx = ctx or default_context()
        keep = [_f32_image(d) for d in disps]
        h, w = keep[0][3]
        on_dev = keep[0][1]
        ptrs = (ctypes.c_void_p * len(keep))(*[k[0] for k in keep])
        fb = np.ascontiguousarray(np.asarray(fbs, np.float32))
        out = _f32_like(disps[0], h, w)
        optr, oon, okeep, _ = _f32_image(out)
        _torch_ready(*disps, out)
        ctx.check(ctx.lib.lux_fuse_disparities(ctx.handle, ptrs, fb.ctypes.data, len(keep), w, h, on_dev, optr, oon))
        return out


@dataclass
class ServedResult:
    """One served request: its depth map (the layer grid) and the times it spent queued and running."""
    Depth: np.ndarray
    status: int
    n_planes: int
    queue_ms: float
    run_ms: float


SGM_FORM_NAMES = {1: "fused", 2: "split", 3: "wave"}


def tuned_form(w, h, n_planes, tile) -> int:
    """The fast aggregation form the autotuner chose for a layer shape (1 fused, 2 split, 3 wave), 0 if none yet."""
    return int(L.load().lux_sgm_tuned_form(w, h, n_planes, tile))


def set_tuned_form(w, h, n_planes, tile, form: int):
    """Sets (1-3) or clears (0) the autotuner's choice for a layer shape."""
    rc = L.load().lux_sgm_set_tuned_form(w, h, n_planes, tile, int(form))
    if rc:
        _raise(rc, "lux_sgm_set_tuned_form failed")


def pool_high_water(device: int = 0, reset: bool = False) -> int:
    """High-water mark (bytes) of the device memory pool this library allocates from; reset restarts it."""
    b = ctypes.c_uint64()
    rc = L.load().lux_sgm_pool_high_water(device, 1 if reset else 0, ctypes.byref(b))
    if rc:
        _raise(rc, "lux_sgm_pool_high_water failed")
    return int(b.value)


class Server:
    """The request server of the C ABI (lux_server_*; no counterpart in the reference): depth solves of mixed sizes
    admitted in arrival order against an HBM budget and run on `slots` worker contexts, overlapping on the GPU. A request
    is one layer solved from unfiltered images exactly as DenseLayer.compute(..., prefilter=True) solves it."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, slots: int = 2):
        self.lib = L.load()
        h = ctypes.c_void_p()
        rc = self.lib.lux_server_create(device, hbm_budget_bytes, slots, ctypes.byref(h))
        if rc:
            _raise(rc, "lux_server_create failed")
        self.handle = h
        self._pending = {}

    @staticmethod
    def _request(images, gray, calibs, near, far, params, flags, priority, out):
        arr = (L.Img * len(images))()
        keep = []
        for i, im in enumerate(images):
            ci, k = _img_c(im)
            arr[i] = ci
            keep.append(k)
        g = np.ascontiguousarray(np.asarray(gray, dtype=np.uint8))
        cc = _calibs_c(calibs)
        req = L.Request(len(images), ctypes.cast(arr, ctypes.c_void_p), g.ctypes.data, ctypes.cast(cc, ctypes.c_void_p), near, far,
                        params.to_c(), flags, out.ctypes.data if out is not None else None, out.nbytes if out is not None else 0,
                        int(priority))
        return req, (keep, arr, g, cc)

    @staticmethod
    def estimate(images, gray, calibs, near, far, params: StereoParams, flags: int = 0) -> int:
        """The device bytes the server reserves for this request against its budget."""
        req, _keep = Server._request(images, gray, calibs, near, far, params, flags, 0, None)
        b = ctypes.c_uint64()
        rc = L.load().lux_server_estimate(ctypes.byref(req), ctypes.byref(b))
        if rc:
            _raise(rc, "lux_server_estimate failed")
        return int(b.value)

    @property
    def passed(self) -> int:
        """Requests that started ahead of an earlier-queued one that had to wait for memory."""
        return int(self.lib.lux_server_passed(self.handle))

    def submit(self, images, gray, calibs, near, far, params: StereoParams, flags: int = 0, priority: int = 0) -> int:
        """Queues a request (lower priority values start first; equal ones in arrival order) and returns its ticket."""
        arr = (L.Img * len(images))()
        keep = []
        for i, im in enumerate(images):
            ci, k = _img_c(im)
            arr[i] = ci
            keep.append(k)
        g = np.ascontiguousarray(np.asarray(gray, dtype=np.uint8))
        cc = _calibs_c(calibs)
        h0, w0 = np.asarray(images[0]).shape[:2] if not hasattr(images[0], "data_ptr") else images[0].shape[:2]
        sc = max(1, int(params.scale))
        out = np.empty(((h0 + sc - 1) // sc, (w0 + sc - 1) // sc), np.float32)
        req = L.Request(len(images), ctypes.cast(arr, ctypes.c_void_p), g.ctypes.data, ctypes.cast(cc, ctypes.c_void_p), near, far,
                        params.to_c(), flags, out.ctypes.data, out.nbytes, int(priority))
        t = ctypes.c_uint64()
        rc = self.lib.lux_server_submit(self.handle, ctypes.byref(req), ctypes.byref(t))
        if rc:
            _raise(rc, self.lib.lux_server_last_error(self.handle).decode())
        self._pending[t.value] = (out, keep, arr, g, cc)  # the image data and the output stay alive until wait
        return t.value

    def cancel(self, ticket: int) -> bool:
        """Cancels a request that has not started (its wait then reports status 13, LUX_ERR_CANCELED); returns False
        when it has started already, which leaves it running to its end (a started state of the reference runs on)."""
        rc = self.lib.lux_server_cancel(self.handle, ticket)
        if rc == 13:
            return False
        if rc:
            _raise(rc, self.lib.lux_server_last_error(self.handle).decode())
        return True

    def wait(self, ticket: int, timeout_ns: int = 0) -> ServedResult:
        r = L.Result()
        rc = self.lib.lux_server_wait(self.handle, ticket, timeout_ns, ctypes.byref(r))
        if rc:
            _raise(rc, self.lib.lux_server_last_error(self.handle).decode())
        out = self._pending.pop(ticket)[0]
        return ServedResult(out, r.status, r.n_planes, r.queue_ms, r.run_ms)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.lux_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
