/* CPU oracle for the dense-stereo depth stage of Lux.Engine — TEST INFRASTRUCTURE ONLY.
 *
 * A literal C restatement of Lux.Engine/Pipeline/Registration/DenseStereo.cs, DenseStereoSgm.cs and
 * DenseUpsampleLayer.cs (plus the IntelApprox, Mt19937, Mat4D and Homography.Sqrt helpers they use). It is the checker
 * for the CUDA path in lux_b200 and the CPU baseline of bench.py; no product code links it.
 *
 * Parity status: the reference's own test suite holds no golden vectors for this path, and the reference (C#/.NET 10)
 * cannot run in this environment, so the restatement as a whole is PARITY UNPINNED against reference outputs. Pinned
 * pieces: the rcp/rsqrt tables (equal to the reference's IntelApprox.Tables.cs, checked by hash), the MSVC mt19937
 * stream (C++ standard known answer), and the reference's own vector/scalar twins (both restated here and checked
 * against each other).
 *
 * Numerics: every float operation is a separate IEEE single rounding (build with -ffp-contract=off, no fast-math);
 * float->int casts follow .NET 9+ (truncate, saturate, NaN -> 0); Math.Min/Max follow .NET (NaN propagates).
 */
#pragma once
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  LO_OK = 0,
  LO_ERR_NEAR_FAR = 1,      /* "The near end has to be smaller than the fard end!"  DenseStereo.cs:43 */
  LO_ERR_NONPOSITIVE = 2,   /* "Both the near and far end have to be positive!"      DenseStereo.cs:44 */
  LO_ERR_BASELINE = 3,      /* "Baseline too small, check calibration."               DenseStereo.cs:63 */
  LO_ERR_SKIPMODE = 4,      /* NotSupported "unrecognized sampling pattern"           DenseStereoSgm.cs:69 */
  LO_ERR_BUDGET = 5,        /* NotSupported "StereoLayer memory budget exceeded"      DenseStereoSgm.cs:343 */
  LO_ERR_UPSAMPLE_SIZE = 6, /* "Incorrect output depth size!"                         DenseUpsampleLayer.cs:43 */
  LO_ERR_INDEX = 7,         /* an access the reference performs out of its arrays (IndexOutOfRangeException) */
  LO_ERR_ALLOC = 8,
  LO_ERR_ARG = 9,
  LO_ERR_ROI = 14,          /* "invalid ROI requested!"                               DepthCache.cs:164 */
  LO_ERR_EMPTY_IMAGE = 15,  /* "empty image!"                                         DepthCache.cs:62 */
};

typedef struct { float K[9], T[3], R[9]; } lo_calib; /* Triangulator.cs:8-19, row-major */

/* StereoParams (DenseStereo.cs:15-21): the fields the dense path reads. */
typedef struct {
  int margin;
  float plane_density;
  int scale;
  int skip_mode;
  uint16_t p1;
  float p2scale;
  float guidance[4];
  int tile;
} lo_params;

void lo_default_params(lo_params* p);             /* StereoParams defaults */
void lo_l16_pyramid(lo_params out[6]);             /* StereoParams.L16Pyramid(false), DenseStereo.cs:24-30 */

uint32_t lo_rcp_bits(uint32_t b);                  /* IntelApprox.RcpBits, IntelApprox.cs:21-29 */
uint32_t lo_rsqrt_bits(uint32_t b);                /* IntelApprox.RsqrtBits, IntelApprox.cs:32-45 */
float lo_rcp(float x);
float lo_homography_sqrt(float x);                 /* Homography.Sqrt, Homography.cs:18 */

typedef struct { uint32_t mt[624]; int idx; } lo_mt19937;  /* FundamentalMatrixFilter.cs:8-30 */
void lo_mt_seed(lo_mt19937* m, uint32_t seed);
uint32_t lo_mt_next(lo_mt19937* m);

void lo_flow_matrix(const lo_calib* a, const lo_calib* b, float out[16]);  /* Mat4D.FlowMatrix, ViewTransform.cs:126 */

/* DenseStereo.Planes (DenseStereo.cs:41-88). out must hold 4096 + align floats. */
int lo_planes(float near_, float far_, const lo_calib* calibs, int ncams, float density, int align, float* out, int* n_out);

void lo_box_filter3(const uint8_t* src, int w, int h, uint8_t* dst);        /* vector form, DenseStereo.cs:93-123 */
void lo_box_filter3_scalar(const uint8_t* src, int w, int h, uint8_t* dst); /* scalar twin, DenseStereo.cs:138-159 */
void lo_guidance(const uint8_t* img0, int w0, int h0, int w, int h, int scale, uint8_t* out); /* DenseStereo.cs:163-177 */

/* DenseStereo.CostContext / BuildContext (DenseStereo.cs:183-199). Images are dense RGBA8. */
typedef struct {
  const uint8_t* ref; int w, h;
  int n_others;
  const uint8_t* const* others; const int* ow; const int* oh;
  const float (*warps)[16];
  const uint16_t (*wq)[4];
  const float* planes; int n_planes;
} lo_costctx;

/* MatchingCost (vector form with its scalar fallback, DenseStereo.cs:217-292) and the scalar twin (:295-373). */
int lo_matching_cost(const lo_costctx* c, int x, int y, int start, int count, uint16_t* cost);
int lo_matching_cost_scalar(const lo_costctx* c, int x, int y, int start, int count, uint16_t* cost);
void lo_normalise(const uint16_t* cost, int count, int cap, int n_others, uint8_t* raw); /* DenseStereo.cs:376-381 */

int lo_skip_mask(int mode, int w, int h, uint8_t* m); /* DenseLayer.SkipMask, DenseStereoSgm.cs:65-87 */

/* One DenseLayer (DenseStereoSgm.cs:13-325). The ragged volume is stored CSR: pixel i owns agg[off[i] .. off[i]+cap[i]). */
typedef struct {
  lo_params p;
  int index, align, w, h, n_planes, min_lo, max_hi;
  float* planes;
  uint8_t* guidance;
  uint8_t* skip;
  uint16_t *start, *count, *cap;
  uint64_t* off;            /* w*h + 1 */
  uint16_t* agg;
  uint16_t* agg_pass1;      /* NULL unless keep_pass1 */
  uint8_t* raw;             /* raw costs (entries of skipped pixels stay 0) */
  float* depth;
  /* cost context */
  int n_cams; const uint8_t* const* images; const int* iw; const int* ih;
  float (*warps)[16]; uint16_t (*wq)[4];
  int threads; int keep_pass1; int xsw;  /* xsw = LUX_SGM_XSW=1 behaviour (DenseStereoSgm.cs:31) */
  /* inline_cost = 1: the reference's Threads == 1 form (DenseStereoSgm.cs:243-249): no prepass; every visit of pass +1
     computes its pixel's costs and stores them, and pass -1 reads the stored ones. 0: the Threads > 1 form, a row-parallel
     prepass on `threads` workers (:186-205), which the reference states gives the same values (:176-180). */
  int inline_cost;
} lo_layer;

/* Pixel's 8-lane vector form (DenseStereoSgm.cs:280-299) where its guard holds (on = 1), else the scalar form only (0,
   the default); lo_vector_calls: path blocks that took the vector form since the last lo_set_vector_form. */
void lo_set_vector_form(int on);
long lo_vector_calls(void);

/* DenseLayer.Init (DenseStereoSgm.cs:34-62). images are the box-filtered camera images (camera 0 = reference). */
int lo_layer_init(lo_layer* L, const lo_params* p, int index, int n_cams, const uint8_t* const* images, const int* iw, const int* ih,
                  const uint8_t* gray, const lo_calib* calibs, float near_, float far_, int align, const lo_layer* prev);
/* DenseLayer.Compute (DenseStereoSgm.cs:181-232): raw costs, pass +1, pass -1, WTA. */
int lo_layer_compute(lo_layer* L);
void lo_layer_free(lo_layer* L);
/* DenseLayer.MemoryEstimate (DenseStereoSgm.cs:144-156). */
int lo_memory_estimate(const lo_params* p, int n_cams, const int* iw, const int* ih, const lo_calib* calibs, float near_, float far_,
                       int align, const lo_layer* prev, int64_t* out);

/* DenseStereoPyramid.Run (DenseStereoSgm.cs:331-353): six L16 layers. layers[] receives the initialised+computed layers. */
int lo_pyramid_run(int n_cams, const uint8_t* const* images, const int* iw, const int* ih, const uint8_t* gray,
                   const lo_calib* calibs, float near_, float far_, int threads, int keep_pass1, lo_layer layers[6]);

/* DenseUpsampleLayer (DenseUpsampleLayer.cs:35-218). guide is RGBA8 with a stride in pixels. out: gw*gh floats. */
void lo_image_shift(const uint8_t* src, int w, int h, int stride, float sx, float sy, uint8_t* dst);
void lo_nearest_resize(const uint8_t* src, int sw, int sh, int sstride, int w, int h, uint8_t* dst);
void lo_inverse_depth(const float* src, size_t n, float* dst);
void lo_bilateral_upsample(const float* lo_, int lw, int lh, const uint8_t* guide, int gw, int gh, int gstride,
                           const uint8_t* g2, float sigma, float* out);
int lo_upsample(const float* prev_depth, int pw, int ph, const uint8_t* guide, int gw, int gh, int gstride, int set_w, int set_h,
                float sigma, int scale, const float* prev_conf, float* out_depth, float* out_conf);

/* Index-only replay of DenseLayer.Compute's traversal (DenseStereoSgm.cs:206-224): for every Pixel call in order, the
 * event id that last wrote each of the four neighbour line-buffer slots it reads (-1 = never written in this layer).
 * Event ids count Pixel calls in order over both passes. ev_out receives, per call, {dir, x, y, r, is_revisit, src0..src3}
 * (9 ints). Returns the number of calls, or -1 when max_events is too small. Used to check the GPU schedule. */
long lo_traversal_trace(int w, int h, int tile, int xsw, int* ev_out, long max_events);

/* Depth image cache (DepthCache.cs): Set into a cw x ch cache, Fetch of a ROI against pipeline dims (dw, dh). */
int lo_depth_cache_set(const float* src, int w, int h, int cw, int ch, float* out);
int lo_depth_cache_fetch(const float* img, int iw, int ih, int x0, int y0, int x1, int y1, int dw, int dh, float* out);

/* Stereo-image formation after the ISP (StereoImage.cs, ReferenceGuide.cs, WineCrt.cs). An aligned calibration is
 * the warp's geometry: H row-major, the 4096-entry CRA lut, the centre (cx, cy) and scales (sx, sy). */
typedef struct {
  float H[9];
  const float* lut;
  float cx, cy, sx, sy;
} lo_aligned;
float lo_wine_sinf(float x);                                       /* WineCrt.Sinf, WineCrt.cs:77-99 */
void lo_lanczos_table(float tbl[384]);                             /* StereoImage.LanczosTable, StereoImage.cs:212-237 */
float lo_gamma_encode(float m);                                    /* StereoImage.GammaEncode, StereoImage.cs:162-178 */
void lo_yuv_matrix(int sensor_type, const float neutral[3], float M[3][4]); /* StereoImage.YuvMatrix, StereoImage.cs:140-160 */
/* StereoImage.Warp (StereoImage.cs:249-296, the vector form's per-lane order): dst (dw x dh x 4 floats, zero-filled
 * where nothing is sampled) from src (sw x sh x 4 floats), src scaled by gain first (StereoImageBuilder.cs:62). */
int lo_warp_f32(const float* src, int sw, int sh, float gain, int dw, int dh, const lo_aligned* ac, float* dst);
void lo_convert_yuv(float* rgba, size_t npx, const float M[3][4]);  /* StereoImage.ConvertToYuv, StereoImage.cs:181-195 */
void lo_to_rgba8(const float* rgba, size_t n, uint8_t* out);       /* StereoImage.ToRgba8, StereoImage.cs:198-209 */
/* Rgba8Warp.Warp (ReferenceGuide.cs:108-156): the 8-bit warp of the reference guide. */
int lo_warp_rgba8(const uint8_t* src, int sw, int sh, int dw, int dh, const lo_aligned* ac, uint8_t* dst);

/* StereoColorTransfer.Transfer (StereoColorTransfer.cs:128-138) of a work YUVA image (w x h x 4 floats) onto the crop of
 * a reference YUVA image (rw x rh) given by calib2 (the reference view) and calibA (the work view): out (w x h x 4),
 * F the 4x4 row-major transfer, crop the clamped rect {X0, Y0, X1, Y1}, n_work / n_ref the gated pixel counts. */
void lo_crop_rect(const lo_calib* calib2, const lo_calib* calibA, int x0, int y0, int x1, int y1, int out[4]);
void lo_color_transfer(const float* work, int w, int h, const float* ref, int rw, int rh, const lo_calib* calib2,
                       const lo_calib* calibA, float* out, float F[16], int crop[4], float* n_work, float* n_ref);

#ifdef __cplusplus
}
#endif
