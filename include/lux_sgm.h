/* lux_sgm.h — C ABI of the B200 dense-stereo depth stage (liblux_sgm.so).
 *
 * This library replaces the CPU dense-stereo stage of Lux.Engine (mprovenz/lux). A C# host binds it with P/Invoke
 * (`[LibraryImport]` or NativeLibrary.Load + `delegate* unmanaged`, as Lux.DepthModel/OnnxDepthNetwork.cs:52-55 does for
 * ONNX Runtime). Plain pointers and sizes only; every function returns a status (0 = ok) and records a message that
 * lux_sgm_last_error() returns. Status codes map onto the exceptions the reference throws (see LUX_ERR_*).
 *
 * Threading: a context serialises its own calls (internal mutex) and owns one CUDA stream; use one context per host
 * thread for concurrency. Results do not depend on the schedule (the reference's guarantee, StereoAsyncApi.cs:44-47).
 */
#ifndef LUX_SGM_H
#define LUX_SGM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define LUX_OK 0
#define LUX_ERR_NEAR_FAR 1      /* InvalidOperationException "The near end has to be smaller than the fard end!" (DenseStereo.cs:43) */
#define LUX_ERR_NONPOSITIVE 2   /* InvalidOperationException "Both the near and far end have to be positive!" (DenseStereo.cs:44) */
#define LUX_ERR_BASELINE 3      /* InvalidOperationException "Baseline too small, check calibration." (DenseStereo.cs:63) */
#define LUX_ERR_SKIPMODE 4      /* NotSupportedException "unrecognized sampling pattern" (DenseStereoSgm.cs:69) */
#define LUX_ERR_BUDGET 5        /* NotSupportedException "StereoLayer memory budget exceeded" (DenseStereoSgm.cs:343), or the HBM budget */
#define LUX_ERR_UPSAMPLE_SIZE 6 /* InvalidOperationException "Incorrect output depth size!" (DenseUpsampleLayer.cs:43) */
#define LUX_ERR_INDEX 7         /* the reference indexes outside an array for these inputs (IndexOutOfRangeException) */
#define LUX_ERR_ALLOC 8         /* device allocation failed */
#define LUX_ERR_ARG 9           /* invalid argument (null pointer, bad size) */
#define LUX_ERR_CUDA 10         /* a CUDA call failed */
#define LUX_ERR_TIMEOUT 11      /* a bounded device-side wait gave up (the kernel returned without finishing) */
#define LUX_ERR_UNSUPPORTED 12  /* inputs outside what this implementation supports (message says which) */
#define LUX_ERR_CANCELED 13     /* OperationCanceledException: the request was canceled before it started */
#define LUX_ERR_ROI 14          /* InvalidOperationException "invalid ROI requested!" (DepthCache.cs:164) */
#define LUX_ERR_EMPTY_IMAGE 15  /* InvalidOperationException "empty image!" (DepthCache.cs:62) */
#define LUX_ERR_IO 16           /* a dump file could not be opened, written or read (IOException) */
#define LUX_ERR_FORMAT 17       /* InvalidOperationException "expected a 4-byte float dump" (StereoAsyncApi.cs:258) */

/* Rgba8Image (Lux.Engine/Pipeline/Registration/SparseLnrMatch.cs:8-13): 8-bit RGBA ("YUVA"), stride in pixels.
 * on_device != 0: data is a device pointer of the context's GPU (no copy); else host memory. */
typedef struct {
  const uint8_t* data;
  int32_t w, h, stride;
  int32_t on_device;
} lux_img_rgba8;

/* CalibData (Lux.Engine/Pipeline/Registration/Triangulator.cs:8-19): row-major K, t, R, X_cam = R·X + t. */
typedef struct {
  float K[9], T[3], R[9];
} lux_calib;

/* StereoParams (Lux.Engine/Pipeline/Registration/DenseStereo.cs:15-21): the fields the dense path reads. */
typedef struct {
  int32_t margin;        /* Margin, 1 */
  float plane_density;   /* PlaneDensity, 2.0 */
  int32_t scale;         /* Scale, 32 */
  int32_t skip_mode;     /* SkipMode, 0 or 2 */
  uint16_t p1;           /* P1, 1 */
  uint16_t reserved;
  float p2scale;         /* P2Scale, 500 */
  float guidance[4];     /* Guidance weights */
  int32_t tile;          /* Tile T (even), 4 */
} lux_stereo_params;

typedef struct lux_sgm_ctx lux_sgm_ctx;
typedef struct lux_layer lux_layer;

/* Context: one GPU, one stream, an HBM budget that every request is admitted against (0 = no limit). */
int lux_sgm_create(int device, uint64_t hbm_budget_bytes, lux_sgm_ctx** out);
void lux_sgm_destroy(lux_sgm_ctx* ctx);
const char* lux_sgm_last_error(const lux_sgm_ctx* ctx);
/* Synchronises the context's stream. */
int lux_sgm_sync(lux_sgm_ctx* ctx);
/* The number of kernels this library has launched in this process (all contexts). */
uint64_t lux_sgm_kernel_launches(void);
/* The context's CUDA stream (a cudaStream_t), for callers that record events or order work against it. */
void* lux_sgm_stream(lux_sgm_ctx* ctx);

/* Failure detection (no counterpart in the reference, whose CPU loops cannot stall on another thread's progress). Every
 * device-side wait of the aggregation kernels (a block waiting for the block above it, a warp for its neighbour) is
 * bounded by this limit in ns of the GPU's global timer; when it passes, the kernel stops, the solve returns
 * LUX_ERR_TIMEOUT and the context stays usable. 0 restores the default (20 s). */
int lux_sgm_set_wait_limit(lux_sgm_ctx* ctx, uint64_t limit_ns);
uint64_t lux_sgm_get_wait_limit(const lux_sgm_ctx* ctx);
/* For tests of the failure path only: the aggregation block with ticket `block` (>= 1; -1 turns it off) waits for the
 * block before it on a counter that nothing publishes, so the wait runs out after the wait limit and the solve returns
 * LUX_ERR_TIMEOUT. Nothing faults; the other blocks see the error word and return. */
int lux_sgm_debug_stall(lux_sgm_ctx* ctx, int32_t block);

/* StereoParams defaults / L16Pyramid() (DenseStereo.cs:15-30). */
void lux_sgm_default_params(lux_stereo_params* p);
void lux_sgm_l16_pyramid(lux_stereo_params out[6]);

/* DenseStereo.Planes (DenseStereo.cs:41-88). out must hold 4096 + align floats. Host only. */
int lux_sgm_planes(float near_, float far_, const lux_calib* calibs, int32_t n_cams, float density, int32_t align, float* out,
                   int32_t* n_out);

/* A grey camera image of `bits` (9..16) bits per sample stored as uint16 (src: host, or device when src_on_device; stride
 * in samples) made into the reference's grey image domain on the GPU: Rgba8Image bytes (Y, 128, 128, 255) with
 * Y = (v + 2^(bits-9)) >> (bits - 8) saturated (12-bit: (v + 8) >> 4), the mapping every 12-bit input of this library
 * follows (the reference's only image type is Rgba8Image, SparseLnrMatch.cs:8-13). dst: a device buffer of w*h*4 bytes,
 * then usable as an on_device lux_img_rgba8 (stride w). From host memory the samples cross as 2 bytes a pixel; the call
 * returns once the host buffer has been read, and the result is ordered on the context's stream. */
int lux_image_from_grey16(lux_sgm_ctx* ctx, const uint16_t* src, int32_t w, int32_t h, int32_t stride, int32_t src_on_device,
                          int32_t bits, uint8_t* dst);

/* DenseStereo.BoxFilter3 (DenseStereo.cs:93-123) of one image; dst is host memory of w*h*4 bytes (dense). */
int lux_sgm_box_filter3(lux_sgm_ctx* ctx, const lux_img_rgba8* src, uint8_t* dst);

/* flags of lux_sgm_layer / lux_sgm_pyramid */
#define LUX_LAYER_KEEP_PASS1 1   /* keep the aggregates after pass +1 (DenseLayer.KeepPass1) */
#define LUX_LAYER_KEEP_AGG 2     /* keep the final aggregates (DenseLayer.Agg); the depth never needs them */
#define LUX_LAYER_PREFILTER 4    /* images are unfiltered: apply DenseStereo.BoxFilter3 on the device first */
#define LUX_LAYER_FORCE_REPLAY 8 /* aggregate with the exact traversal replay even where the fast uniform kernel applies */
/* The fast uniform aggregation has three forms with the same results: the four paths fused in one wavefront (faster on
 * small layers), the same in a lean form, and the path groups {0,1} / {2,3} as row and column chains (faster from about
 * 2 MP). It takes uniform layers of up to 768 planes; past 256 planes (the L16 pyramid's first layer has 552) only the
 * fused form runs them, whatever these flags ask. By default the library picks by timing (below); these flags force
 * one form (tuning and tests). */
#define LUX_LAYER_SGM_FUSED 16
#define LUX_LAYER_SGM_SPLIT 32
#define LUX_LAYER_SGM_WAVE 64    /* the fused wavefront in its lean form (progress counters, packed minima) */
/* Autotuning of the fast form (no counterpart in the reference, which has one CPU loop): with none of the three flags
 * above, a uniform layer of a shape (w, h, planes, tile) not seen before is aggregated once with every fast form on its
 * own cost volume, timed with CUDA events; the fastest is kept for later solves of that shape by every context of the
 * process (all forms give the same bits, so the result does not depend on the choice). Without autotuning, or for a
 * shape not yet tuned, the choice is by size. lux_sgm_set_tuned_form sets or (form 0) clears a choice, e.g. to restore
 * choices saved from an earlier process. */
int lux_sgm_set_autotune(lux_sgm_ctx* ctx, int32_t on);
int32_t lux_sgm_tuned_form(int32_t w, int32_t h, int32_t n_planes, int32_t tile);
int lux_sgm_set_tuned_form(int32_t w, int32_t h, int32_t n_planes, int32_t tile, int32_t form);

/* DenseLayer.Init + DenseLayer.Compute (DenseStereoSgm.cs:34-62, 181-232): one pyramid layer on the GPU.
 * images: n_cams camera images (camera 0 = reference), box-FILTERED already unless LUX_LAYER_PREFILTER (as
 * DenseStereoPyramid.Run filters them, DenseStereoSgm.cs:335); gray[k] selects the grey cost weights; prev = the
 * previous layer (NULL for a first layer: every pixel searches all planes). The layer object owns its device state
 * until lux_layer_destroy. LUX_ERR_UNSUPPORTED where the exact replay would need a line buffer (2·(w+2)·(4·MaxHi+5)
 * u16) past 2^31 - 2^16 elements, which it indexes with 32-bit integers (w beyond about 65,000 pixels). */
int lux_sgm_layer(lux_sgm_ctx* ctx, int32_t n_cams, const lux_img_rgba8* images, const uint8_t* gray, const lux_calib* calibs,
                  float near_, float far_, const lux_stereo_params* params, int32_t index, int32_t align, const lux_layer* prev,
                  int32_t flags, lux_layer** out);

/* DenseStereoPyramid.Run (DenseStereoSgm.cs:331-353): box filter, six L16 layers with the 1 GiB align-8/align-2 choice.
 * flags: LUX_LAYER_KEEP_PASS1 / KEEP_AGG / FORCE_REPLAY apply to every layer. out receives six layer objects. */
int lux_sgm_pyramid(lux_sgm_ctx* ctx, int32_t n_cams, const lux_img_rgba8* images, const uint8_t* gray, const lux_calib* calibs,
                    float near_, float far_, int32_t flags, lux_layer* out[6]);

/* Diagnostic (host only): the revisit schedule the fast uniform kernel replays for a w×h layer with tile T, one pass
 * (second_pass = pass -1), as 7 int32 per row: flags, batch_first, batch_count, src0, src1, src2, extra
 * (see lux_b200/csrc/revisit_schedule.h), then end_first and end_count: out holds 7*h + 2 int32. *y_b receives
 * pass +1's last odd row. */
int lux_sgm_revisit_schedule(int32_t w, int32_t h, int32_t tile, int32_t second_pass, int32_t* out, int32_t* y_b);

/* Layer facts (DenseLayer fields). */
typedef struct {
  int32_t w, h, index, align, n_planes, min_lo, max_hi, tile;
  uint64_t volume;       /* sum of per-pixel caps: the element count of agg / raw */
  float gpu_ms_cost;     /* device time of the matching-cost kernel (CUDA events on the context's stream) */
  float gpu_ms_sgm;      /* device time of the two aggregation passes */
  float gpu_ms_wta;      /* device time of the winner-take-all */
  int32_t sgm_kernel;    /* 0 = the exact traversal replay, 1 = fast, four paths fused, 2 = fast, path groups as chains,
                            3 = fast, four paths fused, lean wavefront */
  int32_t cost_kernel;   /* 0 = per-pixel warps (any layer), 1 = per-row warps (uniform layer), 2 = per-row warps of an axis-aligned
                            pair, 3 = the same with block columns shared between neighbouring pixels (grey, scale 1) */
  int32_t tuned;         /* the fast form the autotuner chose on this solve (it timed every form), 0 when it did not run */
} lux_layer_info;
int lux_layer_get_info(const lux_layer* layer, lux_layer_info* info);

/* Copies a layer field into host memory: bytes must equal the field's size.
 *   LUX_FIELD_DEPTH     float[w*h]        Depth (after WTA)
 *   LUX_FIELD_PLANES    float[n_planes]   Planes
 *   LUX_FIELD_SKIP      uint8[w*h]        Skip (0 computed, 0xff skipped)
 *   LUX_FIELD_START / COUNT / CAP  uint16[w*h]
 *   LUX_FIELD_OFFSETS   uint64[w*h+1]     CSR offsets of the ragged volume (pixel i: [off[i], off[i]+cap[i]))
 *   LUX_FIELD_AGG       uint16[volume]    Agg (final aggregates)
 *   LUX_FIELD_AGG_PASS1 uint16[volume]    AggPass1 (needs keep_pass1)
 *   LUX_FIELD_RAW       uint8[volume]     Raw (entries of skipped pixels are 0)
 *   LUX_FIELD_GUIDANCE  uint8[w*h*4]      Guidance */
enum {
  LUX_FIELD_DEPTH = 0,
  LUX_FIELD_PLANES = 1,
  LUX_FIELD_SKIP = 2,
  LUX_FIELD_START = 3,
  LUX_FIELD_COUNT = 4,
  LUX_FIELD_CAP = 5,
  LUX_FIELD_OFFSETS = 6,
  LUX_FIELD_AGG = 7,
  LUX_FIELD_AGG_PASS1 = 8,
  LUX_FIELD_RAW = 9,
  LUX_FIELD_GUIDANCE = 10,
};
int lux_layer_read(const lux_layer* layer, int32_t field, void* dst, uint64_t bytes);
/* The device pointer of a field (valid until lux_layer_destroy), or NULL. */
const void* lux_layer_device_ptr(const lux_layer* layer, int32_t field);
/* A previous layer made from a stored depth map (host w×h floats) and skip mask (host w×h bytes, 0 = computed; NULL: all
 * computed): the two DenseLayer fields the next layer's RangeFromPrevious reads (DenseStereoSgm.cs:91-142). It resumes a
 * pyramid from a dumped layer (lux_load_f32 of the reference's `_dense_L<i>_depth` dump, StereoAsyncApi.cs:197-214), so one
 * layer can be solved against the C# build's own previous layer. Only LUX_FIELD_DEPTH and LUX_FIELD_SKIP are readable. */
int lux_layer_from_depth(lux_sgm_ctx* ctx, int32_t w, int32_t h, const float* depth, const uint8_t* skip, lux_layer** out);
void lux_layer_destroy(lux_layer* layer);

/* DenseUpsampleLayer.Run (DenseUpsampleLayer.cs:35-48): prev depth pw×ph (host, or device when prev_on_device), guide RGBA8,
 * output depth guide.w×guide.h into out_depth (host). prev_conf / out_conf optional (NULL). */
int lux_sgm_upsample(lux_sgm_ctx* ctx, const float* prev_depth, int32_t pw, int32_t ph, int32_t prev_on_device,
                     const lux_img_rgba8* guide, int32_t set_w, int32_t set_h, float sigma, int32_t scale,
                     const float* prev_conf, float* out_depth, float* out_conf);

/* Dump and golden-file formats of the dense stage (StereoAsyncApi.cs:217-262; host code, no counterpart needed on the
 * GPU). Every image file starts with int32 {w, h, stride = w, bytes per pixel}.
 * lux_dump_f32 / lux_load_f32: DumpF32 / LoadF32 (:252-261), the format LUX_DENSE_OVERRIDE reads (ExportBuild.cs:89-96);
 *   lux_load_f32 with out = NULL only reports w and h; LUX_ERR_FORMAT when bytes per pixel != 4.
 * lux_dump_rgba8: DumpRgba8 (:217-223), host or device image.
 * lux_dump_cost_volume: DumpCostVolume (:227-250): <prefix>_offsets.u32, _costvol.bin and (when kept) _costvol_pass1.bin;
 *   the layer needs its final aggregates (LUX_LAYER_KEEP_AGG on the fast kernels).
 * lux_dump_dense: the dump of State4And5 (:197-214) for solved layers and their inputs under <prefix>_dense_*; cost
 *   volumes of layers 0..cv_max (the reference's LUX_DENSE_DUMP_CV, default 2). */
int lux_dump_f32(const char* path, const float* data, int32_t w, int32_t h);
int lux_load_f32(const char* path, float* out, uint64_t cap_floats, int32_t* w, int32_t* h);
int lux_dump_rgba8(const char* path, const lux_img_rgba8* img);
int lux_dump_cost_volume(const lux_layer* layer, const char* prefix);
int lux_dump_dense(lux_sgm_ctx* ctx, lux_layer* const* layers, int32_t n_layers, int32_t n_cams, const lux_img_rgba8* images,
                   const lux_calib* calibs, const char* prefix, int32_t cv_max);

/* AlignedCalib (Lux.Engine/Pipeline/Geometry/AlignedCalibration.cs:149-178), the geometry of the stereo-image and guide
 * warps as the host builds it (AlignedCalib.Build): H row-major, the 4096 CRA factors (host memory), centre and scales. */
typedef struct {
  float H[9];
  const float* lut;
  float cx, cy, sx, sy;
} lux_aligned_calib;

/* StereoImage.Warp (Lux.Engine/Pipeline/Registration/StereoImage.cs:249-296): dst (dw x dh RGBA floats) from src (sw x sh
 * RGBA floats, rows of sw pixels) scaled by gain first, 6x6 Lanczos-3 taps, 0 where no tap lands. */
int lux_warp_f32(lux_sgm_ctx* ctx, const float* src, int32_t sw, int32_t sh, int32_t src_on_device, float gain,
                 const lux_aligned_calib* ac, int32_t dw, int32_t dh, float* dst, int32_t dst_on_device);
/* StereoImageBuilder.Create (StereoImageBuilder.cs:61-69, 78), colour sensors after the ISP: the half-resolution ISP
 * output src scaled by the exposure gain, warped into dw x dh, ConvertToYUV with the sensor's luma basis over the neutral
 * (StereoImage.cs:140-195), the 8-bit store (:198-209) into out_rgba8 — the dense solve's input image, which can stay on
 * the device — and, when out_yuv is not NULL, the YUV floats (the reference camera's RefYuv). */
int lux_stereo_image(lux_sgm_ctx* ctx, const float* src, int32_t sw, int32_t sh, int32_t src_on_device, float gain,
                     const lux_aligned_calib* ac, int32_t dw, int32_t dh, int32_t sensor_type, const float* neutral,
                     uint8_t* out_rgba8, int32_t out_on_device, float* out_yuv, int32_t yuv_on_device);
/* StereoImageBuilder.Create for a non-reference module with the reference crop (StereoImageBuilder.cs:61-65, 71-77): the
 * stereo image as lux_stereo_image makes it, colour-matched to the crop of the reference camera's YUV image (ref_yuv,
 * dw x dh RGBA floats: lux_stereo_image's out_yuv of the reference) by StereoColorTransfer.Transfer
 * (StereoColorTransfer.cs:128-138): the crop rect from ref_view (calib2) and view (calibA), the statistics of both images,
 * the 4x4 transfer (written to out_F when not NULL, row-major), its application and the 8-bit store. The statistics run on
 * the host (a serial recurrence over the pixels), the rest on the GPU. "Empty reference yuv." is LUX_ERR_ARG. */
int lux_stereo_image_transfer(lux_sgm_ctx* ctx, const float* src, int32_t sw, int32_t sh, int32_t src_on_device, float gain,
                              const lux_aligned_calib* ac, int32_t dw, int32_t dh, int32_t sensor_type, const float* neutral,
                              const float* ref_yuv, int32_t ref_on_device, const lux_calib* ref_view, const lux_calib* view,
                              uint8_t* out_rgba8, int32_t out_on_device, float* out_F);
/* Rgba8Warp.Warp (ReferenceGuide.cs:108-156): the 8-bit warp that makes the upsample's guide from the ISP'd reference
 * image (every tap clamped to the image). "empty source image!" is LUX_ERR_ARG. */
int lux_warp_rgba8(lux_sgm_ctx* ctx, const lux_img_rgba8* src, const lux_aligned_calib* ac, int32_t dw, int32_t dh, uint8_t* dst,
                   int32_t dst_on_device);
/* StereoImage.LanczosTable (StereoImage.cs:212-237): the 64 x 6 taps the warps use. */
void lux_lanczos_table(float* out384);
/* StereoImage.YuvMatrix (StereoImage.cs:140-160): the 3 x 4 rows (v, u', t'). */
void lux_yuv_matrix(int32_t sensor_type, const float* neutral, float* out12);

/* The opt-in census stereo mode of a rectified pair (no counterpart in the reference, whose dense stage is the plane sweep
 * above; parity is with this library's own CPU restatement of the method). Census transform over a 9x7 window, Hamming
 * cost (62 where x - d leaves the image), eight-path semi-global aggregation with constant P1 and P2, the first disparity
 * of least cost, parabolic subpixel refinement, and a left/right check that marks inconsistent pixels -1. Grey values are
 * byte 0 of the RGBA8 images (same size). max_disparity 1..256; 8·(62 + p2) must fit 16 bits (p2 <= 8129). */
typedef struct {
  int32_t max_disparity;
  uint32_t p1, p2;
  int32_t subpixel;     /* nonzero: parabolic refinement */
  int32_t lr_check;     /* nonzero: left/right consistency */
  int32_t lr_max_diff;  /* the largest accepted |d_left - d_right| */
} lux_census_params;
int lux_census_sgm(lux_sgm_ctx* ctx, const lux_img_rgba8* left, const lux_img_rgba8* right, const lux_census_params* params,
                   float* out_disp, int32_t out_on_device);
/* The census mode over a capture's pairs in one batch: the reference image against others[0..n) (n <= 16, all the
 * reference's size, on its grid), pair k with disparity range max_disparity[k] and focal x baseline fb[k]; params gives P1,
 * P2 and the options (its max_disparity is ignored). Every stage is one launch over all pairs (the reference's census is
 * made once); the pairs' disparities are fused as lux_fuse_disparities fuses them into out_depth. out_disps, when not
 * NULL, receives the n disparity maps (host, n x w x h floats). */
int lux_census_capture(lux_sgm_ctx* ctx, int32_t n, const lux_img_rgba8* ref, const lux_img_rgba8* others, const int32_t* max_disparity,
                       const float* fb, const lux_census_params* params, float* out_depth, int32_t out_on_device, float* out_disps);
/* The fusion of a capture's pairs: per pair the depth fb[k] / disparity where the disparity is positive, per pixel the
 * median of the valid depths (the mean of the two middle ones for an even count), 0 where none is valid. disps: n <= 16
 * pointers to w x h disparity maps (device pointers when on_device, else host). */
int lux_fuse_disparities(lux_sgm_ctx* ctx, const float* const* disps, const float* fb, int32_t n, int32_t w, int32_t h,
                         int32_t on_device, float* out_depth, int32_t out_on_device);

/* DepthImageCache.Set (Lux.Engine/Pipeline/Export/DepthCache.cs:136-143, fed by FromFullDepth :239-244): the cache image
 * (cw x ch floats) made from a depth map (w x h): InverseDepth, the nearest 16.16 resample to the cache dims, then
 * min(rcpps(x), 1e5). depth / cache are device pointers of the context's GPU when *_on_device, else host memory.
 * LUX_ERR_EMPTY_IMAGE when cw or ch <= 0 ("empty image!", :62). With both on the device the call is asynchronous on the
 * context's stream (lux_sgm_stream / lux_sgm_sync order later work after it); with either on the host it returns when
 * the result is there. */
int lux_depth_cache_set(lux_sgm_ctx* ctx, const float* depth, int32_t w, int32_t h, int32_t depth_on_device, int32_t cw, int32_t ch,
                        float* cache, int32_t cache_on_device);
/* DepthImageCache.Fetch (DepthCache.cs:161-239): the ROI [x0, x1) x [y0, y1) of pipeline dims (dims_w, dims_h) read from a
 * cache image (cw x ch) into out ((x1-x0) x (y1-y0) floats): a plain copy when the scale is 1, else the reciprocal of
 * the source window, the nearest resample and the division back. LUX_ERR_ROI for an invalid ROI ("invalid ROI
 * requested!", :164). Synchronous or not as lux_depth_cache_set. */
int lux_depth_cache_fetch(lux_sgm_ctx* ctx, const float* cache, int32_t cw, int32_t ch, int32_t cache_on_device, int32_t x0, int32_t y0,
                          int32_t x1, int32_t y1, int32_t dims_w, int32_t dims_h, float* out, int32_t out_on_device);

/* ---- Request server: the serving form of the stage, admitted like Lux.Library's job queue
 * (Lux.Library/Core/JobQueue.cs:23-28, Dispatch :474-531). ----
 * Depth solves of mixed sizes wait in (priority, arrival) order, lower priority values first. Whenever one of the
 * `slots` worker contexts is free, the first waiting request whose host-side estimate of device memory fits what the
 * running requests leave of the HBM budget starts (0 = no limit; when nothing runs, the first request starts
 * regardless). A heavy request (estimate above 1.5 GiB, the queue's LightBytes) that does not fit holds back every heavy
 * request behind it (no overtaking), while light ones may pass it; one heavy request runs at a time (a heavy solve fills
 * the GPU, and two side by side only interleave their blocks). Each worker has its own CUDA stream, so requests
 * that arrive while others are on the GPU start as soon as a slot and memory are free and overlap on the device. A
 * request is one layer, solved exactly as lux_sgm_layer solves it from unfiltered images (LUX_LAYER_PREFILTER is
 * implied; prev = NULL, align 8), its depth map copied into out_depth (host, the layer's w*h floats, out_bytes long;
 * NULL: nothing copied). The server copies the request's small arrays at submit; the caller keeps the image data and
 * out_depth alive until lux_server_wait has returned for the ticket. Every result equals the same request solved alone.
 * The workers pick the aggregation form by size (path-group chains from about 2 MP, the fused wavefront below) unless
 * the request's flags name one: the autotuner's choices are timed on an idle GPU and need not be the best beside other
 * requests; the workers do not autotune either. */
typedef struct lux_server lux_server;
typedef struct {
  int32_t n_cams;
  const lux_img_rgba8* images;
  const uint8_t* gray;
  const lux_calib* calibs;
  float near_, far_;
  lux_stereo_params params;
  int32_t flags;
  float* out_depth;
  uint64_t out_bytes;
  int32_t priority;  /* JobInfo.Priority: lower values start first; equal values in arrival order */
} lux_request;
typedef struct {
  int32_t status;           /* LUX_OK or the status the solve returned */
  int32_t w, h, n_planes;   /* the layer's size and plane count */
  double queue_ms, run_ms;  /* submit -> start of the solve, start -> depth in out_depth */
} lux_result;
int lux_server_create(int device, uint64_t hbm_budget_bytes, int32_t slots, lux_server** out);
void lux_server_destroy(lux_server* server);  /* finishes the requests already submitted */
const char* lux_server_last_error(const lux_server* server);
int lux_server_submit(lux_server* server, const lux_request* req, uint64_t* ticket);
/* Waits for a ticket (timeout_ns 0: no limit; LUX_ERR_TIMEOUT when it passes) and releases it. */
int lux_server_wait(lux_server* server, uint64_t ticket, uint64_t timeout_ns, lux_result* out);
/* The device bytes the server reserves for a request against its budget (JobInfo.EstimatedMemoryBytes). */
int lux_server_estimate(const lux_request* req, uint64_t* bytes);
/* How many requests started ahead of an earlier-queued one that had to wait (light requests passing a heavy one). */
uint64_t lux_server_passed(const lux_server* server);
/* Cancels a request that has not started: its lux_server_wait then reports status LUX_ERR_CANCELED
 * (OperationCanceledException). The reference is cancelable between the states of a capture's registration, and a state
 * once started runs to its end (StereoAsyncApi.cs:51-64); here a request that has started runs to its end and the call
 * returns LUX_ERR_CANCELED without changing it. LUX_ERR_ARG for an unknown ticket. */
int lux_server_cancel(lux_server* server, uint64_t ticket);
/* The high-water mark of the device memory this library's allocations hold in the device's memory pool (the stream-
 * ordered pool every context allocates from), in bytes; reset != 0 resets it to the current use afterwards. */
int lux_sgm_pool_high_water(int device, int32_t reset, uint64_t* bytes);

/* No counterpart in the reference. lux_sgm_upsample without any device allocation, for hosts that cannot let this
 * library allocate GPU memory: a process whose HBM is already reserved by another allocator (an inference server or a
 * framework's caching pool holding nearly all of it), where a cudaMalloc here would fail or fragment that pool, and a
 * serving loop that must not pay the implicit device synchronisation of cudaMalloc / cudaFree on every request.
 * prev_depth (and prev_conf) are device arrays of pw×ph floats, guide a device image (on_device != 0, stride >= w), out_depth
 * (and out_conf) device arrays of guide.w×guide.h floats; results equal lux_sgm_upsample's. The one scratch buffer, the
 * resampled guidance (pw·ph RGBA8 pixels), is a static device array of LUX_UPSAMPLE_NOALLOC_MAX_PIXELS pixels (16 MiB)
 * that every GPU which loads this library holds until the process exits; a larger pw·ph returns LUX_ERR_ARG. Each call
 * writes every byte of it that it reads, so nothing has to start at zero. The first call on a device looks the array up
 * (cudaGetSymbolAddress, with the context's device current): make that first call before any stream capture. All calls
 * share the array and it keeps the last call's contents, so calls that overlap in time on one device (through different
 * contexts) race: serialise them. The work runs on the context's stream (lux_sgm_stream), a non-blocking stream that
 * nothing orders after the caller's own streams: prev_depth, prev_conf and the guide must be complete before the call
 * (synchronise the stream that wrote them, or make lux_sgm_stream wait on an event recorded after the writes).
 * Returns after the context's stream has finished the work. */
#define LUX_UPSAMPLE_NOALLOC_MAX_PIXELS (4u << 20)
int lux_sgm_upsample_noalloc(lux_sgm_ctx* ctx, const float* prev_depth, int32_t pw, int32_t ph, const lux_img_rgba8* guide,
                             int32_t set_w, int32_t set_h, float sigma, int32_t scale, const float* prev_conf,
                             float* out_depth, float* out_conf);

#ifdef __cplusplus
}
#endif
#endif
