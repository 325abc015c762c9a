// Box filter, guidance, plane ranges from the previous layer, CSR offsets, WTA and the upsample chain.
// Each kernel restates one reference function with its exact operation order (file:line in each comment).
#include <algorithm>
#include <atomic>
#include <cstring>

#include <cub/cub.cuh>

#include "common.cuh"
#include "internal.h"

namespace lux {

static std::atomic<uint64_t> g_launches{0};
void count_launches(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }
uint64_t kernel_launches() { return g_launches.load(); }

// ---- DenseStereo.BoxFilter3 (DenseStereo.cs:93-159): per channel float(Σ)·(1/(cols·rows)), RNE, saturated ----
// DenseLayer.SkipMask (DenseStereoSgm.cs:65-87), SkipMode 2: the image is cut into 64x64 tiles (the last tile of a row or
// column takes the remainder, nx = w/64 + (64 < 2·(w%64))), each drawing from a fresh default-seeded mt19937; its 2x2
// cells in row order take two draws each, dy then dx, and the cell's pixel (x + dx, y + dy) is computed (0), every
// other pixel skipped (0xff). Tiles start at multiples of 64, so a pixel's cell is (x & ~1, y & ~1) and it is the
// chosen one when its parities are (dx, dy). bits: the stream's low bits (host_skip_stream_bits).
__global__ void k_skip_mask(uint8_t* __restrict__ m, int w, int h, int nx, int ny, const uint32_t* __restrict__ bits) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= w || y >= h) return;
  const int i = min(x >> 6, nx - 1), j = min(y >> 6, ny - 1);
  const int x0 = 64 * i, x1 = min(w, x0 + (i == nx - 1 ? 128 : 64)), y0 = 64 * j;
  const int c = ((y - y0) >> 1) * ((x1 - x0 + 1) >> 1) + ((x - x0) >> 1);  // the cell's index in its tile
  const int k = 2 * c;
  const int dy = (__ldg(bits + (k >> 5)) >> (k & 31)) & 1, dx = (__ldg(bits + ((k + 1) >> 5)) >> ((k + 1) & 31)) & 1;
  m[(size_t)y * w + x] = ((x & 1) == dx && (y & 1) == dy) ? 0 : 0xff;
}

void launch_skip_mask(int mode, int w, int h, const uint32_t* bits, uint8_t* m, cudaStream_t s) {
  if (mode == 0) {
    cudaMemsetAsync(m, 0, (size_t)w * h, s);
    return;
  }
  int nx = w / 64 + (64 < 2 * (w % 64) ? 1 : 0), ny = h / 64 + (64 < 2 * (h % 64) ? 1 : 0);
  if (nx < 1) nx = 1;
  if (ny < 1) ny = 1;
  k_skip_mask<<<dim3((w + 255) / 256, h), 256, 0, s>>>(m, w, h, nx, ny, bits);
  count_launches(1);
}

__global__ void k_box_filter3(const uint8_t* __restrict__ src, int w, int h, int stride, uint8_t* __restrict__ dst) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= w) return;
  int y0 = max(y - 1, 0), y1 = min(y + 1, h - 1), x0 = max(x - 1, 0), x1 = min(x + 1, w - 1);
  int rows = y1 - y0 + 1, cols = x1 - x0 + 1;
  // vector form: 1/(2·rows) at the edge columns, 1/(3·rows) inside (:110); the scalar form gives the same divisors
  float inv = __fdiv_rn(1.0f, __fmul_rn((float)cols, (float)rows));
  int s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  for (int yy = y0; yy <= y1; yy++)
    for (int xx = x0; xx <= x1; xx++) {
      uchar4 p = __ldg(reinterpret_cast<const uchar4*>(src) + (size_t)yy * stride + xx);
      s0 += p.x; s1 += p.y; s2 += p.z; s3 += p.w;
    }
  auto q = [&](int s) {
    int v = __float2int_rn(__fmul_rn((float)s, inv));  // cvtps2dq
    return (unsigned char)min(max(v, 0), 255);           // packssdw + packuswb
  };
  reinterpret_cast<uchar4*>(dst)[(size_t)y * w + x] = make_uchar4(q(s0), q(s1), q(s2), q(s3));
}

void launch_box_filter3(const uint8_t* src, int w, int h, int stride, uint8_t* dst, cudaStream_t s) {
  dim3 grid((w + 127) / 128, h);
  k_box_filter3<<<grid, 128, 0, s>>>(src, w, h, stride, dst);
  count_launches(1);
}

// ---- DenseStereo.Guidance (DenseStereo.cs:163-177) ----
__global__ void k_guidance(const uchar4* __restrict__ img0, int w0, int h0, int w, int h, int scale, uchar4* __restrict__ out) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= w) return;
  int sx = x, sy = y;
  if (!(w0 == w && h0 == h)) {
    int half = (scale + (scale >> 31)) >> 1;
    sy = min(scale * y + half, h0 - 1);
    sx = min(scale * x + half, w0 - 1);
  }
  out[(size_t)y * w + x] = img0[(size_t)sy * w0 + sx];
}

void launch_guidance(const uint8_t* img0, int w0, int h0, int w, int h, int scale, uchar4* out, cudaStream_t s) {
  dim3 grid((w + 127) / 128, h);
  k_guidance<<<grid, 128, 0, s>>>(reinterpret_cast<const uchar4*>(img0), w0, h0, w, h, scale, out);
  count_launches(1);
}

// ---- DenseLayer.RangeFromPrevious (DenseStereoSgm.cs:91-140) ----
// scratch: idx[pw*ph], hmin, hmax (u16)
size_t range_from_previous_scratch_bytes(int pw, int ph) { return (size_t)pw * ph * 2 * 3 + 256; }

// plane index of every previous pixel: #{j : b[j] <= rcp(depth)} as the scan `while (c < n && b[c] <= v) c++` (:101)
__global__ void k_plane_index(const float* __restrict__ depth, int npx, const float* __restrict__ b, int n, int monotone,
                              const uint32_t* __restrict__ rcp_table, uint16_t* __restrict__ idx) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npx) return;
  float v = rcp_approx(depth[i], rcp_table);
  int c;
  if (monotone) {  // b non-decreasing: the first index with !(b[c] <= v) by bisection
    int lo = 0, hi = n;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (__ldg(b + mid) <= v) lo = mid + 1; else hi = mid;
    }
    c = lo;
  } else {
    c = 0;
    while (c < n && __ldg(b + c) <= v) c++;
  }
  idx[i] = (uint16_t)c;
}

// 4-wide horizontal min/max over computed pixels x-1..x+2 (clamped) (:105-117)
__global__ void k_hminmax(const uint16_t* __restrict__ idx, const uint8_t* __restrict__ skip, int pw, int ph, uint16_t* __restrict__ hmin,
                          uint16_t* __restrict__ hmax) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= pw) return;
  unsigned mn = 0xffff, mx = 0;
  for (int k = -1; k <= 2; k++) {
    int xx = min(max(x + k, 0), pw - 1);
    if (skip[(size_t)y * pw + xx] > 0) continue;
    unsigned v = idx[(size_t)y * pw + xx];
    mn = min(mn, v);
    mx = max(mx, v);
  }
  hmin[(size_t)y * pw + x] = (uint16_t)mn;
  hmax[(size_t)y * pw + x] = (uint16_t)mx;
}

// vertical 4-tall min/max (:118-125) sampled at the nearest previous pixel, margin, range (:126-138)
__global__ void k_ranges(const uint16_t* __restrict__ hmin, const uint16_t* __restrict__ hmax, int pw, int ph, int W, int H, float fx,
                         float fy, int n, int margin, uint16_t* __restrict__ start, uint16_t* __restrict__ count, int* minmax) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  int lo = 0x7fffffff, hi = 0;
  if (x < W) {
    int py = f2i(__fmul_rn((float)y, fy)), px = f2i(__fmul_rn((float)x, fx));
    py = min(max(py, 0), ph - 1);  // (float)y·fy never leaves [0, ph-1]; the clamp only guards the load
    px = min(max(px, 0), pw - 1);
    unsigned mn = 0xffff, mx = 0;
    for (int k = -1; k <= 2; k++) {
      int yy = min(max(py + k, 0), ph - 1);
      mn = min(mn, (unsigned)hmin[(size_t)yy * pw + px]);
      mx = max(mx, (unsigned)hmax[(size_t)yy * pw + px]);
    }
    lo = max(0, (int)mn - margin);
    hi = min(n - 1, (int)mx + 1);
    size_t i = (size_t)y * W + x;
    start[i] = (uint16_t)lo;
    count[i] = (uint16_t)(hi - lo);
    lo &= 0xffff;
    hi &= 0xffff;
  }
  // block reduction, then one atomic per block
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&minmax[0], lo);
    atomicMax(&minmax[1], hi);
  }
}

void launch_range_from_previous(const float* prev_depth, const uint8_t* prev_skip, int pw, int ph, const float* b, int monotone,
                                int n, const uint32_t* rcp_table, int W, int H, int margin, uint16_t* start, uint16_t* count,
                                int* minmax, void* scratch, cudaStream_t s) {
  uint16_t* idx = static_cast<uint16_t*>(scratch);
  uint16_t* hmin = idx + (size_t)pw * ph;
  uint16_t* hmax = hmin + (size_t)pw * ph;
  int npx = pw * ph;
  k_plane_index<<<(npx + 255) / 256, 256, 0, s>>>(prev_depth, npx, b, n, monotone, rcp_table, idx);
  count_launches(1);
  dim3 g1((pw + 127) / 128, std::min(ph, 65535));
  k_hminmax<<<g1, 128, 0, s>>>(idx, prev_skip, pw, ph, hmin, hmax);
  count_launches(1);
  float fy = (float)(ph - 1) / (float)(H - 1), fx = (float)(pw - 1) / (float)(W - 1);
  dim3 g2((W + 127) / 128, H);
  k_ranges<<<g2, 128, 0, s>>>(hmin, hmax, pw, ph, W, H, fx, fy, n, margin, start, count, minmax);
  count_launches(1);
}

// ---- caps and CSR offsets (DenseStereoSgm.cs:53-58): cap = count rounded up to align ----
__global__ void k_caps(const uint16_t* __restrict__ count, int npx, int align, uint16_t* __restrict__ cap, uint64_t* __restrict__ c64) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npx) return;
  int c = ((count[i] + align - 1) / align) * align;
  cap[i] = (uint16_t)c;
  c64[i] = (uint64_t)c;
}

size_t caps_offsets_scratch_bytes(int npx) {
  size_t tmp = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp, (const uint64_t*)nullptr, (uint64_t*)nullptr, npx + 1);
  return tmp + (size_t)(npx + 1) * 8 + 256;
}

void launch_caps_offsets(const uint16_t* count, int npx, int align, uint16_t* cap, uint64_t* off, void* scratch, size_t scratch_bytes,
                         cudaStream_t s) {
  uint64_t* c64 = static_cast<uint64_t*>(scratch);
  void* tmp = static_cast<char*>(scratch) + ((size_t)(npx + 1) * 8 + 255) / 256 * 256;
  size_t tmp_bytes = scratch_bytes - ((size_t)(npx + 1) * 8 + 255) / 256 * 256;
  cudaMemsetAsync(c64 + npx, 0, 8, s);
  k_caps<<<(npx + 255) / 256, 256, 0, s>>>(count, npx, align, cap, c64);
  count_launches(1);
  cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, c64, off, npx + 1, s);
}

// Σ (8 + cap·(skipped ? 2 : 3)) of DenseLayer.MemoryEstimate (DenseStereoSgm.cs:153)
__global__ void k_estimate(const uint16_t* __restrict__ count, const uint8_t* __restrict__ skip, int npx, int align,
                           unsigned long long* out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long v = 0;
  if (i < npx) {
    int c = ((count[i] + align - 1) / align) * align;
    v = 8ull + (unsigned long long)c * (skip[i] == 0 ? 3ull : 2ull);
  }
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(out, v);
}

void launch_estimate_terms(const uint16_t* count, const uint8_t* skip, int npx, int align, unsigned long long* out, cudaStream_t s) {
  k_estimate<<<(npx + 255) / 256, 256, 0, s>>>(count, skip, npx, align, out);
  count_launches(1);
}

// A pixel whose cap is not a multiple of 8 makes the reference's scalar SGM lanes write agg[cap] (DenseStereoSgm.cs:302-311).
__global__ void k_check_caps(const uint16_t* __restrict__ cap, int npx, int* err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < npx && cap[i] != 0 && (cap[i] & 7) != 0) atomicCAS(err, 0, 7 /* LUX_ERR_INDEX */);
}
void launch_check_caps(const uint16_t* cap, int npx, int* err, cudaStream_t s) {
  k_check_caps<<<(npx + 255) / 256, 256, 0, s>>>(cap, npx, err);
  count_launches(1);
}

// A grey image of `bits` per sample (9..16, u16) as the reference's grey YUVA bytes (Y, 128, 128, 255): Y = (v + half) >>
// (bits - 8) saturated at 255, half = 1 << (bits - 9) (12-bit: (v + 8) >> 4). Four pixels a thread.
__global__ void k_grey16_to_rgba8(const uint16_t* __restrict__ src, int w, int h, int stride, int bits, uchar4* __restrict__ dst) {
  const int shift = bits - 8, half = 1 << (shift - 1);
  const int x4 = (blockIdx.x * blockDim.x + threadIdx.x) * 4, y = blockIdx.y;
  if (x4 >= w || y >= h) return;
  const uint16_t* row = src + (size_t)y * stride;
  uchar4* out = dst + (size_t)y * w;
  for (int k = 0; k < 4 && x4 + k < w; k++) {
    const int v = min(255, ((int)row[x4 + k] + half) >> shift);
    out[x4 + k] = make_uchar4((unsigned char)v, 128, 128, 255);
  }
}
void launch_grey16_to_rgba8(const uint16_t* src, int w, int h, int stride, int bits, uint8_t* dst, cudaStream_t s) {
  dim3 grid((w + 4 * 128 - 1) / (4 * 128), h);
  k_grey16_to_rgba8<<<grid, 128, 0, s>>>(src, w, h, stride, bits, reinterpret_cast<uchar4*>(dst));
  count_launches(1);
}

__global__ void k_fill_u16(uint16_t* p, size_t n, uint16_t v) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (; i < n; i += stride) p[i] = v;
}
void launch_fill_u16(uint16_t* p, size_t n, uint16_t v, cudaStream_t s) {
  if (n == 0) return;
  size_t nb = (n + 255) / 256;
  int blocks = (int)(nb < 148 * 16 ? nb : 148 * 16);
  k_fill_u16<<<blocks, 256, 0, s>>>(p, n, v);
  count_launches(1);
}

// a first layer: Start 0, Count = Cap = n (DenseStereoSgm.cs:43-46)
__global__ void k_uniform_ranges(uint16_t* start, uint16_t* count, uint16_t* cap, uint64_t* off, int npx, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > npx) return;
  off[i] = (uint64_t)i * (uint64_t)n;
  if (i == npx) return;
  start[i] = 0;
  count[i] = (uint16_t)n;
  cap[i] = (uint16_t)n;
}
void launch_uniform_ranges(uint16_t* start, uint16_t* count, uint16_t* cap, uint64_t* off, int npx, int n, cudaStream_t s) {
  k_uniform_ranges<<<(npx + 1 + 255) / 256, 256, 0, s>>>(start, count, cap, off, npx, n);
  count_launches(1);
}

// ---- WTA (DenseStereoSgm.cs:225-231): first minimum of agg[0, count) -> Planes[(ushort)(Start + arg)] ----
__global__ void k_wta(const uint16_t* __restrict__ agg, const uint64_t* __restrict__ off, const uint16_t* __restrict__ start,
                      const uint16_t* __restrict__ count, const float* __restrict__ planes, int n, int npx, float* __restrict__ depth,
                      int* err) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= npx) return;
  const uint16_t* a = agg + off[warp];
  int cnt = count[warp];
  int best = 0xffff, arg = 0x7fffffff;
  for (int k = lane; k < cnt; k += 32) {
    int v = a[k];
    if (v < best) { best = v; arg = k; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    int ob = __shfl_xor_sync(0xffffffffu, best, o), oa = __shfl_xor_sync(0xffffffffu, arg, o);
    if (ob < best || (ob == best && oa < arg)) { best = ob; arg = oa; }
  }
  if (lane == 0) {
    if (arg == 0x7fffffff) arg = 0;
    int pl = (uint16_t)(start[warp] + arg);
    if (pl >= n) { atomicCAS(err, 0, 7); pl = 0; }
    depth[warp] = planes[pl];
  }
}

void launch_wta(const LayerGeom& g, const uint16_t* agg, float* depth, int* err, cudaStream_t s) {
  int npx = g.W * g.H;
  k_wta<<<(npx + 7) / 8, 256, 0, s>>>(agg, g.off, g.start, g.count, g.planes, g.n_planes, npx, depth, err);
  count_launches(1);
}

// ---- DenseUpsampleLayer (DenseUpsampleLayer.cs:35-218) ----
struct ShiftTaps {
  float kx[4], ky[4];
  int stepX, stepY;
};

// g2(x,y) = ImageShift(guide, 0.5, 0.5)(sx, sy) with the 16.16 nearest steps of NearestResize (:69-131): the shifted guide is
// only ever read at these positions, so only they are computed.
__global__ void k_shift_resize(const uint8_t* __restrict__ guide, int gw, int gh, int gstride, int pw, int ph, ShiftTaps t,
                               uint8_t* __restrict__ g2) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= pw) return;
  for (int y = blockIdx.y; y < ph; y += gridDim.y) {  // gridDim.y is capped at 65535 rows; taller images loop
  int sy = (int)((unsigned)y * (unsigned)t.stepY) >> 16;  // the accumulated yAcc (int, wraps like the reference's sum)
  int sx = (int)((unsigned)x * (unsigned)t.stepX) >> 16;
  int rows[4];
  for (int i = 0; i < 4; i++) { int ry = sy - 1 + i; rows[i] = ry < 0 ? 0 : ry >= gh ? gh - 1 : ry; }
  uint8_t outv[4];
  for (int ch = 0; ch < 4; ch++) {
    float v[4];
    for (int j = 0; j < 4; j++) {  // columns sx-1 .. sx+2 of the row buffer (clamp-to-edge)
      int c = sx - 1 + j;
      int cx = c < 0 ? 0 : c >= gw ? gw - 1 : c;
      float acc = __fmul_rn((float)guide[((size_t)rows[0] * gstride + cx) * 4 + ch], t.ky[0]);
      for (int i = 1; i < 4; i++) acc = __fadd_rn(__fmul_rn((float)guide[((size_t)rows[i] * gstride + cx) * 4 + ch], t.ky[i]), acc);
      v[j] = acc;
    }
    float s = __fadd_rn(__fadd_rn(__fmul_rn(v[3], t.kx[3]), __fmul_rn(v[2], t.kx[2])),
                        __fadd_rn(__fmul_rn(v[1], t.kx[1]), __fmul_rn(v[0], t.kx[0])));
    int q = __float2int_rn(s);
    outv[ch] = (uint8_t)(q < 0 ? 0 : q > 255 ? 255 : q);
  }
  *reinterpret_cast<uchar4*>(g2 + ((size_t)y * pw + x) * 4) = make_uchar4(outv[0], outv[1], outv[2], outv[3]);
  }
}

LUX_DEV float up_exp2(float t) {  // Exp2Fast (:151-159)
  const float C1 = __uint_as_float(0x3d9fcb52u), C2 = __uint_as_float(0x3e677e26u), C3 = __uint_as_float(0x3f322226u),
              C4 = __uint_as_float(0x3f7ffb19u);
  t = t < 128.0f ? t : 128.0f;
  t = t > -126.0f ? t : -126.0f;
  int n = f2i(t) + ((int)__float_as_uint(t) >> 31);
  float f = __fsub_rn(t, (float)n);
  float p = __fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(f, C1), C2), f), C3), f), C4);
  return __uint_as_float(__float_as_uint(p) + ((unsigned)n << 23));
}
LUX_DEV float spatial_w(float f, int i) {  // SpatialW (:212-217)
  float d = fabsf(__fsub_rn(f, (float)(i * 2)));
  d = d < 1.0f ? d : 1.0f;
  return f2i(d) == 0 ? 1.0f : __uint_as_float(0x3eaaaaabu);
}

// BilateralUpsampleFromCollapse (:166-209). inverse != 0: lo = rcp(prev) and out = rcp(V/S) (the InverseDepth steps).
__global__ void k_bilateral(const float* __restrict__ prev, int lw, int lh, const uint8_t* __restrict__ guide, int W, int H, int gstride,
                            const uint8_t* __restrict__ g2, float k, int inverse, const uint32_t* __restrict__ rcp_table,
                            float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= W) return;
  for (int y = blockIdx.y; y < H; y += gridDim.y) {  // gridDim.y is capped at 65535 rows; taller images loop
  const float eps = __uint_as_float(0x322bcc77u);
  int wm1 = lw - 1, hm1 = lh - 1;
  int iy0 = (y - 1) / 2;
  float fy = __fadd_rn((float)y, -0.5f);
  const uint8_t* o = guide + ((size_t)y * gstride + x) * 4;
  float hr = o[0], hg = o[1], hb = o[2];
  int ix0 = (x - 1) / 2;
  float fx = __fadd_rn((float)x, -0.5f);
  int ibx = ix0 < 0 ? 0 : ix0;
  if (ibx > wm1) ibx = wm1;
  float wx0 = spatial_w(fx, ibx);
  int ix1 = ix0 + 1;
  if (ix1 < 0) ix1 = 0;
  if (ix1 > wm1) ix1 = wm1;
  float wx1 = spatial_w(fx, ix1);
  float accV = 0.0f, accS = 0.0f;
  for (int j = 0; j < 2; j++) {
    int iy = iy0 + j;
    if (iy < 0) iy = 0;
    if (iy > hm1) iy = hm1;
    float wy = spatial_w(fy, iy);
    size_t lrow = (size_t)iy * lw;
    const uint8_t* q = g2 + (lrow + ibx) * 4;
    float d0 = __fsub_rn(hr, (float)q[0]), d1 = __fsub_rn(hg, (float)q[1]), d2 = __fsub_rn(hb, (float)q[2]);
    float s = __fadd_rn(__fmul_rn(d1, d1), __fadd_rn(__fmul_rn(d2, d2), __fmul_rn(d0, d0)));
    float t = -__fmul_rn(s, k);
    float w0 = __fmul_rn(__fadd_rn(up_exp2(t), eps), __fmul_rn(wy, wx0));
    q = g2 + (lrow + ix1) * 4;
    d0 = __fsub_rn(hr, (float)q[0]); d1 = __fsub_rn(hg, (float)q[1]); d2 = __fsub_rn(hb, (float)q[2]);
    s = __fadd_rn(__fmul_rn(d1, d1), __fadd_rn(__fmul_rn(d2, d2), __fmul_rn(d0, d0)));
    t = -__fmul_rn(s, k);
    float w1 = __fmul_rn(__fadd_rn(up_exp2(t), eps), __fmul_rn(wy, wx1));
    float l0 = prev[lrow + ibx], l1 = prev[lrow + ix1];
    if (inverse) { l0 = rcp_approx(l0, rcp_table); l1 = rcp_approx(l1, rcp_table); }
    float v0 = __fmul_rn(l0, w0), v1 = __fmul_rn(l1, w1);
    accV = __fadd_rn(v1, __fadd_rn(v0, accV));
    accS = __fadd_rn(w1, __fadd_rn(w0, accS));
  }
  float r = __fdiv_rn(accV, accS);
  out[(size_t)y * W + x] = inverse ? rcp_approx(r, rcp_table) : r;
  }
}

static float cubic_tap_host(float x) {  // CubicTap (:56-62)
  uint32_t u = 0x3e2aaaabu;
  float sixth;
  memcpy(&sixth, &u, 4);
  volatile float x2 = x * x, x3 = x2 * x;
  if (x < 1.0f) { volatile float a = x3 * 9.0f; volatile float b = x2 * (-15.0f); b = b + 6.0f; b = b + a; return b * sixth; }
  if (x < 2.0f) {
    volatile float a = x3 * (-3.0f); volatile float b = x2 * 15.0f; volatile float c = x * (-24.0f);
    c = c + 12.0f; c = c + b; c = c + a; return c * sixth;
  }
  return 0.0f;
}

void launch_upsample(const float* prev, int pw, int ph, const uint8_t* guide, int gw, int gh, int gstride, float sigma,
                     const uint32_t* rcp_table, uint8_t* g2, float* out_depth, const float* prev_conf, float* out_conf,
                     cudaStream_t s) {
  ShiftTaps t;
  float tx = 0.5f, ty = 0.5f;  // ImageShift(guide, 0.5f, 0.5f): floor 0, fraction 0.5
  t.kx[0] = cubic_tap_host(tx + 1.0f); t.kx[1] = cubic_tap_host(tx); t.kx[2] = cubic_tap_host(1.0f - tx); t.kx[3] = cubic_tap_host(2.0f - tx);
  t.ky[0] = cubic_tap_host(ty + 1.0f); t.ky[1] = cubic_tap_host(ty); t.ky[2] = cubic_tap_host(1.0f - ty); t.ky[3] = cubic_tap_host(2.0f - ty);
  double sy = (double)gh * 65536.0 / (double)ph, sx = (double)gw * 65536.0 / (double)pw;
  t.stepY = sy >= 2147483648.0 ? 0x7fffffff : (int)sy;
  t.stepX = sx >= 2147483648.0 ? 0x7fffffff : (int)sx;
  dim3 g1((pw + 127) / 128, std::min(ph, 65535));
  k_shift_resize<<<g1, 128, 0, s>>>(guide, gw, gh, gstride, pw, ph, t, g2);
  count_launches(1);
  volatile float ss = sigma * sigma;
  float k = 0.5f / ss;
  dim3 g3((gw + 127) / 128, std::min(gh, 65535));
  k_bilateral<<<g3, 128, 0, s>>>(prev, pw, ph, guide, gw, gh, gstride, g2, k, 1, rcp_table, out_depth);
  count_launches(1);
  if (prev_conf && out_conf) {
    k_bilateral<<<g3, 128, 0, s>>>(prev_conf, pw, ph, guide, gw, gh, gstride, g2, k, 0, rcp_table, out_conf);
    count_launches(1);
  }
}

}  // namespace lux
