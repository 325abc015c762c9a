// Internal host-side interface between the C ABI (lux_sgm.cu) and the kernel files.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace lux {

constexpr int kMaxCams = 16;        // reference + up to 15 other cameras per layer (an L16 capture has 16 modules)
// Every launch_* wrapper counts its kernels here (reported through lux_sgm_kernel_launches).
void count_launches(int n);
uint64_t kernel_launches();

constexpr uint64_t kTimeoutNs = 20ull * 1000 * 1000 * 1000;  // bounded device waits: 20 s of %globaltimer (default)

// Layer geometry and per-pixel ranges, all device pointers.
struct LayerGeom {
  int W, H, n_planes, align, min_lo, max_hi, tile;
  const float* planes;
  const uchar4* guidance;
  const uint8_t* skip;
  const uint16_t* start;
  const uint16_t* count;
  const uint16_t* cap;
  const uint64_t* off;
  uint64_t volume;
  bool uniform;  // every pixel searches [0, n) with cap n (first layer)
  // Bounded device waits: every cross-block or cross-warp wait of the aggregation kernels gives up after timeout_ns of
  // %globaltimer (error 11). stall_block >= 0 (failure-path tests only): the block with that ticket waits for the block
  // before it on `never`, a zero counter that nothing publishes, so its wait runs out and the launch ends with error 11.
  uint64_t timeout_ns;
  int stall_block;
  const int* never;
};

struct CostArgs {
  const uint8_t* ref; int rw, rh;  // box-filtered reference image (dense RGBA8)
  int n_others;
  const uint8_t* other[kMaxCams];
  const uint32_t* phase[kMaxCams];  // per other camera: four half-pixel phase images, [4][oh][ow] of uint2 (grey) or u32
  int ow[kMaxCams], oh[kMaxCams];
  float warp[kMaxCams][16];
  uint16_t wq[kMaxCams][4];
  float norm;                       // 0x3d17b426 / nOthers
  int scale;
  int axis;                         // one other camera, axis-aligned flow matrix: zt.w holds 1/pz per plane
  int vcols;                        // axis, grey, scale 1: phase images as vertical triples, blocks from shared columns
  uint32_t one;                     // 1: a multiplier the compiler cannot fold, so that adds can issue on the FMA pipe
};

// prep.cu
void launch_box_filter3(const uint8_t* src, int w, int h, int stride, uint8_t* dst, cudaStream_t s);
// DenseLayer.SkipMask for SkipMode 0 or 2 (checked by the caller); bits: host_skip_stream_bits on the device.
void launch_skip_mask(int mode, int w, int h, const uint32_t* bits, uint8_t* m, cudaStream_t s);
void launch_guidance(const uint8_t* img0, int w0, int h0, int w, int h, int scale, uchar4* out, cudaStream_t s);
// b: the n plane-index boundaries (device); monotone: b is non-decreasing (bisection gives the scan's answer)
void launch_range_from_previous(const float* prev_depth, const uint8_t* prev_skip, int pw, int ph, const float* b, int monotone,
                                int n, const uint32_t* rcp_table, int W, int H, int margin, uint16_t* start, uint16_t* count,
                                int* minmax /* [0]=minLo [1]=maxHi, preset to INT_MAX, 0 */, void* scratch, cudaStream_t s);
size_t range_from_previous_scratch_bytes(int pw, int ph);
void launch_caps_offsets(const uint16_t* count, int npx, int align, uint16_t* cap, uint64_t* off, void* scratch, size_t scratch_bytes,
                         cudaStream_t s);
size_t caps_offsets_scratch_bytes(int npx);
void launch_estimate_terms(const uint16_t* count, const uint8_t* skip, int npx, int align, unsigned long long* out_cost,
                           cudaStream_t s);
void launch_check_caps(const uint16_t* cap, int npx, int* err, cudaStream_t s);
void launch_wta(const LayerGeom& g, const uint16_t* agg, float* depth, int* err, cudaStream_t s);
void launch_fill_u16(uint16_t* p, size_t n, uint16_t v, cudaStream_t s);
// grey u16 samples of `bits` (9..16) bits -> the reference's grey YUVA bytes, dense w x h RGBA8 (h <= 65535)
void launch_grey16_to_rgba8(const uint16_t* src, int w, int h, int stride, int bits, uint8_t* dst, cudaStream_t s);
void launch_uniform_ranges(uint16_t* start, uint16_t* count, uint16_t* cap, uint64_t* off, int npx, int n, cudaStream_t s);
// upsample chain (DenseUpsampleLayer.cs): g2 = NearestResize(ImageShift(guide)), then the bilateral upsample of 1/depth
void launch_upsample(const float* prev, int pw, int ph, const uint8_t* guide, int gw, int gh, int gstride, float sigma,
                     const uint32_t* rcp_table, uint8_t* g2, float* out_depth, const float* prev_conf, float* out_conf,
                     cudaStream_t s);

// depth_cache.cu: DepthImageCache.Set and Fetch (DepthCache.cs)
void launch_depth_cache_set(const float* src, int w, int h, int cw, int ch, const uint32_t* rcp, float* out, cudaStream_t s);
void launch_depth_cache_fetch(const float* img, int istride, int vx0, int vy0, int vw, int vh, double offx, double offy, double sx,
                              double sy, int rw, int rh, const uint32_t* rcp, float* out, cudaStream_t s);

// warp.cu: stereo-image formation after the ISP and the reference guide's 8-bit warp (StereoImage.cs, ReferenceGuide.cs)
struct WarpGeom {  // AlignedCalib (Lux.Engine/Pipeline/Geometry/AlignedCalibration.cs:149-178) with its lut on the device
  float h[9];
  float cx, cy, sx, sy;
  const float* lut;
  float neg_zero;  // -0.0f, given at run time (the packed products of the warp kernels add it)
};
struct YuvRows {  // the rows (v, u', t') of StereoImage.YuvMatrix
  float m[3][4];
};
// taps: the 384-float Lanczos table; rsq: the rsqrt tables for exponents 127 then 128 (4096 entries each).
// m == nullptr: the warped float image into out_f. Else the stereo image into out_u8 and, when out_f != nullptr, its
// YUV floats into out_f.
void launch_warp_f32(const float* src, int sw, int sh, float gain, const WarpGeom& g, const float* taps, const uint32_t* rsq,
                     int dw, int dh, const YuvRows* m, float* out_f, uint8_t* out_u8, int* err, cudaStream_t s);
void launch_warp_rgba8(const uint8_t* src, int sw, int sh, int sstride, const WarpGeom& g, const float* taps, const uint32_t* rsq,
                       int dw, int dh, uint8_t* out, int* err, cudaStream_t s);
struct ColourF {  // a row-major 4x4 colour transfer (StereoColorTransfer.Solve)
  float f[16];
};
// census_sgm.cu: the opt-in census stereo mode (census, Hamming cost, 8-path SGM, WTA, subpixel, left/right, fusion)
constexpr int kMaxFusePairs = 16;
int census_lpt(int D);  // disparities per lane: 1, 2, 4 or 8 for D up to 32, 64, 128, 256 (0: too large)
// One pair of a batch: the other image's census (W x H), its cost and path sums (W x H x 32·census_lpt(D)),
// its left and right integer disparities and its float disparities (W x H), and its disparity range D.
struct CensusPair {
  uint64_t* cr;
  uint8_t* cost;
  uint16_t* S;
  int *dl, *dr;
  float* disp;
  int D;
};
struct CensusPairs {
  CensusPair p[kMaxFusePairs];
};
// n pairs (<= kMaxFusePairs) of the reference image against others[k] (device pointers), all W x H; grey at byte 0 of
// every bpp bytes, rows stride pixels apart; pair k's buffers are laid out with 32·census_lpt(D_k) values a pixel; cl:
// the reference's census (W x H). One launch per stage covers every pair of the same lane width.
void launch_census_batch(const uint8_t* ref, const uint8_t* const* others, int n, int w, int h, int stride, int bpp, uint32_t P1,
                         uint32_t P2, int subpixel, int lr, int max_diff, uint64_t* cl, const CensusPairs& ps, cudaStream_t s);
// disps: a device array of n device pointers to W x H disparity maps (n <= kMaxFusePairs); fb: n focal x baseline products.
void launch_fuse(const float* const* disps, const float* fb, int n, int npx, float* out, cudaStream_t s);

// StereoColorTransfer.Apply of a YUVA float image and the 8-bit store of the result.
void launch_colour_apply(const float* yuv, int npx, const ColourF& F, uint8_t* out, cudaStream_t s);

// cost.cu
// The phase images of every other camera into a.phase (4·ow·oh u32 each); then the cost volume.
// zt: per other camera and plane, the plane-only projection terms (z·W[8] + W[12], z·W[9] + W[13], z·W[10] + W[14], 0),
// each product and sum rounded to float, as float4 × n_planes × n_others.
bool cost_all_grey(const CostArgs& a);
void launch_phases(const CostArgs& a, cudaStream_t s);
// Returns the kernel it used: 0 per-pixel warps, 1 per-row warps (uniform layers), 2 per-row warps of an axis-aligned pair.
// Small layers with many planes: the warp-per-pixel cost kernel (and horizontal phase images) instead of the row kernels.
bool cost_small_wide_layer(int W, int H, int n_planes);
int launch_cost(const CostArgs& a, const LayerGeom& g, const float4* zt, uint8_t* raw, int* err, cudaStream_t s);

// sgm_emulate.cu: the exact replay of the reference's sheared-tile traversal on its line-buffer layout (any layer)
struct EmuBuffers {
  uint16_t* L; size_t Llen;
  uint16_t* Min;
  uint16_t* RangeS;
  uint16_t* RangeC;
  float4* Pix;
  int* ticket;    // [2]
  int* progress;  // [2 * bands * kEmuParts]
};
constexpr int kEmuPartRows = 8;  // rows of a block (part) of the exact replay's row form: min(8, T/2)
constexpr int kEmuParts = 16;    // at most, blocks per band (parts of at least 4 rows, T <= 64)
size_t emu_line_buffer_elems(int W, int max_hi);
void emu_init_buffers(const EmuBuffers& b, int W, int max_hi, int align, int bands, cudaStream_t s);
void launch_sgm_emulate(const LayerGeom& g, const EmuBuffers& b, int dir, int xsw, uint16_t p1, float p2scale, const float gw[4],
                        const uint8_t* raw, uint16_t* agg, int* err, cudaStream_t s);

// sgm_uniform.cu: the fast aggregation of a uniform layer (every pixel searches all planes)
struct UniformBuffers {
  void* band_state;     // per CTA band: the last row's path states (boundary between CTA bands)
  int* band_progress;   // per CTA band
  int* ticket;          // [1]
  void* side;           // per-row states of the two revisit-adjacent columns
  void* edge_state;     // pass +1 final line-buffer row read by pass -1 (W+2 slots)
  void* events;         // host-built revisit schedule
};
size_t uniform_supported_planes();
// Layers past 256 planes: only the fused form (k_sgm_uniform, LPT 16 or 24) runs them.
bool uniform_wide_planes(int n_planes);
bool uniform_fast_supported(int W, int H, int n_planes, int tile, uint16_t p1, float p2scale);
size_t uniform_scratch_bytes(int W, int H, int n_planes, int tile);
// Both passes, WTA into depth. agg holds pass +1's aggregates afterwards, and the final ones when keep_agg.
// sgm_split.cu: the same aggregation by path groups {0, 1} (row chains) and {2, 3} (column chains)
size_t split_scratch_bytes(int W, int H, int n);
int run_sgm_split(const LayerGeom& g, int xsw, uint16_t p1, float p2scale, const float gw[4], const uint8_t* raw, uint16_t* agg,
                  uint16_t* agg_pass1, float* depth, int keep_agg, void* scratch, size_t scratch_bytes, int* err, cudaStream_t s);
// sgm_wave.cu: the fused four-path wavefront in its lean form (progress counters, packed minima, 16 rows a block)
size_t wave_scratch_bytes(int W, int H, int n);
int run_sgm_wave(const LayerGeom& g, int xsw, uint16_t p1, float p2scale, const float gw[4], const uint8_t* raw, uint16_t* agg,
                 uint16_t* agg_pass1, float* depth, int keep_agg, void* scratch, size_t scratch_bytes, int* err, cudaStream_t s);
int run_sgm_uniform(const LayerGeom& g, int xsw, uint16_t p1, float p2scale, const float gw[4], const uint8_t* raw, uint16_t* agg,
                    uint16_t* agg_pass1, float* depth, int keep_agg, void* scratch, size_t scratch_bytes, int* err,
                    cudaStream_t s);

}  // namespace lux
