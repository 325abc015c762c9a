"""ctypes binding of liblux_sgm.so (include/lux_sgm.h).

The library is built in-tree by lux_b200/build.py. Loading fails loudly when it is missing: there is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblux_sgm.so")

LUX_OK = 0
ERRORS = {
    1: "LUX_ERR_NEAR_FAR", 2: "LUX_ERR_NONPOSITIVE", 3: "LUX_ERR_BASELINE", 4: "LUX_ERR_SKIPMODE", 5: "LUX_ERR_BUDGET",
    6: "LUX_ERR_UPSAMPLE_SIZE", 7: "LUX_ERR_INDEX", 8: "LUX_ERR_ALLOC", 9: "LUX_ERR_ARG", 10: "LUX_ERR_CUDA",
    11: "LUX_ERR_TIMEOUT", 12: "LUX_ERR_UNSUPPORTED", 13: "LUX_ERR_CANCELED", 14: "LUX_ERR_ROI", 15: "LUX_ERR_EMPTY_IMAGE",
    16: "LUX_ERR_IO", 17: "LUX_ERR_FORMAT",
}

FIELD_DEPTH, FIELD_PLANES, FIELD_SKIP, FIELD_START, FIELD_COUNT, FIELD_CAP = 0, 1, 2, 3, 4, 5
FIELD_OFFSETS, FIELD_AGG, FIELD_AGG_PASS1, FIELD_RAW, FIELD_GUIDANCE = 6, 7, 8, 9, 10

LAYER_KEEP_PASS1, LAYER_KEEP_AGG, LAYER_PREFILTER, LAYER_FORCE_REPLAY = 1, 2, 4, 8
LAYER_SGM_FUSED, LAYER_SGM_SPLIT, LAYER_SGM_WAVE = 16, 32, 64


class Img(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("w", ctypes.c_int32), ("h", ctypes.c_int32), ("stride", ctypes.c_int32),
                ("on_device", ctypes.c_int32)]


class Calib(ctypes.Structure):
    _fields_ = [("K", ctypes.c_float * 9), ("T", ctypes.c_float * 3), ("R", ctypes.c_float * 9)]


class Params(ctypes.Structure):
    _fields_ = [("margin", ctypes.c_int32), ("plane_density", ctypes.c_float), ("scale", ctypes.c_int32),
                ("skip_mode", ctypes.c_int32), ("p1", ctypes.c_uint16), ("reserved", ctypes.c_uint16),
                ("p2scale", ctypes.c_float), ("guidance", ctypes.c_float * 4), ("tile", ctypes.c_int32)]


class Request(ctypes.Structure):
    _fields_ = [("n_cams", ctypes.c_int32), ("images", ctypes.c_void_p), ("gray", ctypes.c_void_p), ("calibs", ctypes.c_void_p),
                ("near", ctypes.c_float), ("far", ctypes.c_float), ("params", Params), ("flags", ctypes.c_int32),
                ("out_depth", ctypes.c_void_p), ("out_bytes", ctypes.c_uint64), ("priority", ctypes.c_int32)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("w", ctypes.c_int32), ("h", ctypes.c_int32), ("n_planes", ctypes.c_int32),
                ("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double)]


class AlignedCalib(ctypes.Structure):
    _fields_ = [("H", ctypes.c_float * 9), ("lut", ctypes.c_void_p), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
                ("sx", ctypes.c_float), ("sy", ctypes.c_float)]


class CensusParams(ctypes.Structure):
    _fields_ = [("max_disparity", ctypes.c_int32), ("p1", ctypes.c_uint32), ("p2", ctypes.c_uint32), ("subpixel", ctypes.c_int32),
                ("lr_check", ctypes.c_int32), ("lr_max_diff", ctypes.c_int32)]


class LayerInfo(ctypes.Structure):
    _fields_ = [("w", ctypes.c_int32), ("h", ctypes.c_int32), ("index", ctypes.c_int32), ("align", ctypes.c_int32),
                ("n_planes", ctypes.c_int32), ("min_lo", ctypes.c_int32), ("max_hi", ctypes.c_int32), ("tile", ctypes.c_int32),
                ("volume", ctypes.c_uint64), ("gpu_ms_cost", ctypes.c_float), ("gpu_ms_sgm", ctypes.c_float),
                ("gpu_ms_wta", ctypes.c_float), ("sgm_kernel", ctypes.c_int32),
                ("cost_kernel", ctypes.c_int32), ("tuned", ctypes.c_int32)]


# every exported symbol with its signature: (name, restype, argtypes)
SIGNATURES = [
    ("lux_sgm_create", ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    ("lux_sgm_destroy", None, [ctypes.c_void_p]),
    ("lux_sgm_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("lux_sgm_sync", ctypes.c_int, [ctypes.c_void_p]),
    ("lux_sgm_kernel_launches", ctypes.c_uint64, []),
    ("lux_sgm_stream", ctypes.c_void_p, [ctypes.c_void_p]),
    ("lux_sgm_set_wait_limit", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    ("lux_sgm_set_autotune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ("lux_sgm_tuned_form", ctypes.c_int32, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    ("lux_sgm_set_tuned_form", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    ("lux_sgm_get_wait_limit", ctypes.c_uint64, [ctypes.c_void_p]),
    ("lux_sgm_debug_stall", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ("lux_sgm_revisit_schedule", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    ("lux_sgm_default_params", None, [ctypes.POINTER(Params)]),
    ("lux_sgm_l16_pyramid", None, [ctypes.POINTER(Params)]),
    ("lux_sgm_planes", ctypes.c_int, [ctypes.c_float, ctypes.c_float, ctypes.POINTER(Calib), ctypes.c_int32, ctypes.c_float,
                                      ctypes.c_int32, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int32)]),
    ("lux_sgm_box_filter3", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Img), ctypes.c_void_p]),
    ("lux_image_from_grey16", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    ("lux_sgm_layer", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(Img), ctypes.c_void_p, ctypes.POINTER(Calib),
                                     ctypes.c_float, ctypes.c_float, ctypes.POINTER(Params), ctypes.c_int32, ctypes.c_int32,
                                     ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    ("lux_sgm_pyramid", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(Img), ctypes.c_void_p, ctypes.POINTER(Calib),
                                       ctypes.c_float, ctypes.c_float, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    ("lux_layer_get_info", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(LayerInfo)]),
    ("lux_layer_read", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint64]),
    ("lux_layer_device_ptr", ctypes.c_void_p, [ctypes.c_void_p, ctypes.c_int32]),
    ("lux_layer_destroy", None, [ctypes.c_void_p]),
    ("lux_layer_from_depth", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    ("lux_sgm_upsample", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.POINTER(Img), ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.c_int32,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("lux_depth_cache_set", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32]),
    ("lux_depth_cache_fetch", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32]),
    ("lux_dump_f32", ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    ("lux_load_f32", ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_int32)]),
    ("lux_dump_rgba8", ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(Img)]),
    ("lux_dump_cost_volume", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    ("lux_dump_dense", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32, ctypes.c_int32,
                                      ctypes.POINTER(Img), ctypes.POINTER(Calib), ctypes.c_char_p, ctypes.c_int32]),
    ("lux_warp_f32", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                                    ctypes.POINTER(AlignedCalib), ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32]),
    ("lux_stereo_image", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_float, ctypes.POINTER(AlignedCalib), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32]),
    ("lux_stereo_image_transfer", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.c_float, ctypes.POINTER(AlignedCalib), ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(Calib),
                                                 ctypes.POINTER(Calib), ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ("lux_census_sgm", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Img), ctypes.POINTER(Img), ctypes.POINTER(CensusParams),
                                      ctypes.c_void_p, ctypes.c_int32]),
    ("lux_census_capture", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(Img), ctypes.POINTER(Img), ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.POINTER(CensusParams), ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    ("lux_fuse_disparities", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_int32,
                                            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32]),
    ("lux_warp_rgba8", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Img), ctypes.POINTER(AlignedCalib), ctypes.c_int32,
                                      ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32]),
    ("lux_lanczos_table", None, [ctypes.c_void_p]),
    ("lux_yuv_matrix", None, [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    ("lux_server_create", ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    ("lux_server_destroy", None, [ctypes.c_void_p]),
    ("lux_server_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("lux_server_submit", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]),
    ("lux_server_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(Result)]),
    ("lux_server_estimate", ctypes.c_int, [ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]),
    ("lux_server_passed", ctypes.c_uint64, [ctypes.c_void_p]),
    ("lux_server_cancel", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    ("lux_sgm_pool_high_water", ctypes.c_int, [ctypes.c_int, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64)]),
    ("lux_sgm_upsample_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                                ctypes.POINTER(Img), ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                                                ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
]

_lib = None


def load(path=LIB_PATH):
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m lux_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class LuxError(RuntimeError):
    """A non-zero status of the C ABI. `code` is the LUX_ERR_* value."""

    def __init__(self, code, message):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code
