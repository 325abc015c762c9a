// The depth image cache that the renderer and exporter read (Lux.Engine/Pipeline/Export/DepthCache.cs), fed by the
// upsampled full-resolution depth: Set (inverse depth, nearest resample to the cache dims, clipped inverse back) and
// Fetch (a ROI at another pipeline level: a reciprocal pass over the source window, nearest resample, division back).
// Every float step keeps the reference's operation and rounding (rcpps = IntelApprox.RcpBits on the table; one Newton
// step (1 - v·r)·r + r; IEEE division), so results are bit-identical.
#include <algorithm>
#include <atomic>

#include "common.cuh"
#include "internal.h"

namespace lux {

// ImageResample0 (DepthCache.cs:38-70): 16.16 fixed point with int32 wrap-around, clamped to [0, n-1]
LUX_DEV int nearest16(int s16, int o16, int i, int n) {
  const int v = (int)((unsigned)s16 * (unsigned)i + (unsigned)o16) >> 16;
  return v < 0 ? 0 : v > n - 1 ? n - 1 : v;
}

// The NaN an SSE reciprocal pass leaves: a NaN input propagates quieted; a NaN made from numbers (0·inf in the Newton
// step of a zero or infinite depth) is the x86 default NaN 0xffc00000. CUDA's arithmetic returns its canonical NaN
// instead, so a NaN result is rewritten to the x86 one (a zero-filled cache, fetched before its first Set, gives these).
LUX_DEV float x86_nan(float r, float v) {
  if (r == r) return r;
  return v != v ? __uint_as_float(__float_as_uint(v) | 0x00400000u) : __uint_as_float(0xffc00000u);
}

// Both kernels are persistent (a few blocks per SM looping over tiles), so the 16 KB rcpps table is copied into shared
// memory once per block: read from global memory, a warp's 32 table lookups would be 32 scattered L1 requests. A tile is
// kDcRows output rows x kDcCols·256 columns. A thread works out the tile's source rows once (the nearest resample maps
// consecutive output rows to non-decreasing source rows, so a row that samples the same source row as the row above
// reuses its value) and then takes its kDcCols columns (x, x + 256, ...) in turn, issuing the loads of all the column's
// rows before converting them.
constexpr int kDcThreads = 256, kDcRows = 8, kDcCols = 4, kDcTileW = kDcThreads * kDcCols;

LUX_DEV void load_table(uint32_t* tab, const uint32_t* __restrict__ g) {
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) reinterpret_cast<uint4*>(tab)[i] = __ldg(reinterpret_cast<const uint4*>(g) + i);
  __syncthreads();
}

LUX_DEV float rcp_s(float v, const uint32_t* tab) {
  const uint32_t b = __float_as_uint(v);
  return __uint_as_float(rcp_entry(b, tab[(b >> 11) & 0xfff]));
}

// Set's rcpps(rcpps(v)) by one lookup. Table entry i is 1/1.m (exponent E(i) of 126 or 127, mantissa M(i)); the first
// rcpps of v = 2^(e-127)·1.m gives exponent E(i) + 127 - e and mantissa M(i), so the second looks up j = M(i) >> 11 and
// gives exponent e + E(j) - E(i) and mantissa M(j). comp[i] = (E(j) - E(i))·2^23 + M(j) added to v's sign and exponent
// bits is the pair, exact while both steps stay normal: 3 <= e <= 250 is well inside. Other exponents (zeros, subnormals,
// infinities, NaN, the extremes) take the two table steps.
LUX_DEV void build_composite(int32_t* comp, const uint32_t* __restrict__ g) {
  for (int i = threadIdx.x; i < 4096; i += blockDim.x) {
    const uint32_t ti = __ldg(g + i), tj = __ldg(g + ((ti & 0x7fffffu) >> 11));
    comp[i] = ((int32_t)((tj >> 23) & 0xff) - (int32_t)((ti >> 23) & 0xff)) * (1 << 23) + (int32_t)(tj & 0x7fffffu);
  }
  __syncthreads();
}

LUX_DEV float rcp_rcp(float v, const int32_t* comp, const uint32_t* __restrict__ g) {
  const uint32_t b = __float_as_uint(v), e = (b >> 23) & 0xff;
  if (e - 3u <= 247u) return __uint_as_float((b & 0xff800000u) + (uint32_t)comp[(b >> 11) & 0xfff]);
  return rcp_approx(rcp_approx(v, g), g);
}

// Set: only the source pixels the nearest resample reads are inverted (InverseDepth is per pixel, so the values are
// those of inverting the whole image first); then minps(rcpps(x), 1e5).
__global__ void __launch_bounds__(kDcThreads) k_depth_cache_set(const float* __restrict__ src, int w, int h, int cw, int ch, int sx16,
                                                                int sy16, const uint32_t* __restrict__ rcp, float* __restrict__ out) {
  __shared__ int32_t comp[4096];
  build_composite(comp, rcp);
  const int col_tiles = (cw + kDcTileW - 1) / kDcTileW, tiles = col_tiles * ((ch + kDcRows - 1) / kDcRows);
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int xb = (t % col_tiles) * kDcTileW + threadIdx.x, y0 = (t / col_tiles) * kDcRows, nrows = min(kDcRows, ch - y0);
    const float* row[kDcRows];
    bool fresh[kDcRows];
#pragma unroll
    for (int i = 0, prev = -1; i < kDcRows; i++) {
      const int sy = nearest16(sy16, 0, y0 + i, h);
      fresh[i] = sy != prev && i < nrows;
      row[i] = src + (size_t)sy * w;
      prev = sy;
    }
#pragma unroll
    for (int k = 0; k < kDcCols; k++) {
      const int x = xb + k * kDcThreads;
      if (x >= cw) break;
      const int sx = nearest16(sx16, 0, x, w);
      float v[kDcRows];
#pragma unroll
      for (int i = 0; i < kDcRows; i++)
        if (fresh[i]) v[i] = __ldcs(row[i] + sx);
      float r = 0.f, *o = out + (size_t)y0 * cw + x;
#pragma unroll
      for (int i = 0; i < kDcRows; i++, o += cw) {
        if (i >= nrows) break;
        if (fresh[i]) {
          const float q = rcp_rcp(v[i], comp, rcp);
          r = q < 100000.0f ? q : 100000.0f;
        }
        __stcs(o, r);
      }
    }
  }
}

// Fetch (FetchFull / FetchSampled, DepthCache.cs:185-239): per output pixel the window pixel it samples, its reciprocal
// (columns below vec: rcpps + one Newton step, then x 1.0; the rest: division), and the division back. 1.0f / x is the
// correctly rounded reciprocal, which __frcp_rn computes for every input.
LUX_DEV float fetch_value(float v, bool newton, const uint32_t* tab) {
  float inv;
  if (newton) {
    const float r = rcp_s(v, tab);
    inv = __fmul_rn(__fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fmul_rn(v, r)), r), r), 1.0f);
  } else {
    inv = __frcp_rn(v);
  }
  return x86_nan(__frcp_rn(inv), v);
}

__global__ void __launch_bounds__(kDcThreads) k_depth_cache_fetch(const float* __restrict__ img, int istride, int vx0, int vy0, int vw,
                                                                  int vh, int vec, int sx16, int sy16, int ox16, int oy16, int rw, int rh,
                                                                  const uint32_t* __restrict__ rcp, float* __restrict__ out) {
  __shared__ uint32_t tab[4096];
  load_table(tab, rcp);
  const int col_tiles = (rw + kDcTileW - 1) / kDcTileW, tiles = col_tiles * ((rh + kDcRows - 1) / kDcRows);
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int xb = (t % col_tiles) * kDcTileW + threadIdx.x, y0 = (t / col_tiles) * kDcRows, nrows = min(kDcRows, rh - y0);
    const float* row[kDcRows];
    bool fresh[kDcRows];
#pragma unroll
    for (int i = 0, prev = -1; i < kDcRows; i++) {
      const int py = nearest16(sy16, oy16, y0 + i, vh);
      fresh[i] = py != prev && i < nrows;
      row[i] = img + (size_t)(vy0 + py) * istride + vx0;
      prev = py;
    }
#pragma unroll
    for (int k = 0; k < kDcCols; k++) {
      const int x = xb + k * kDcThreads;
      if (x >= rw) break;
      const int px = nearest16(sx16, ox16, x, vw);
      const bool newton = px < vec;
      float v[kDcRows];
#pragma unroll
      for (int i = 0; i < kDcRows; i++)
        if (fresh[i]) v[i] = __ldg(row[i] + px);
      float r = 0.f, *o = out + (size_t)y0 * rw + x;
#pragma unroll
      for (int i = 0; i < kDcRows; i++, o += rw) {
        if (i >= nrows) break;
        if (fresh[i]) r = fetch_value(v[i], newton, tab);
        __stcs(o, r);
      }
    }
  }
}

// Resident blocks of `kernel` on all SMs (at most `tiles`): the persistent grid. `cache` keeps the count for the process
// (every GPU it runs on is the same part).
template <class K>
int persistent_blocks(K kernel, int tiles, std::atomic<int>& cache) {
  int n = cache.load(std::memory_order_relaxed);
  if (n <= 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kDcThreads, 0) != cudaSuccess || per_sm <= 0) per_sm = 1;
    n = sms * per_sm;
    cache.store(n, std::memory_order_relaxed);
  }
  return std::max(1, std::min(tiles, n));
}
std::atomic<int> g_set_blocks{0}, g_fetch_blocks{0};

void launch_depth_cache_set(const float* src, int w, int h, int cw, int ch, const uint32_t* rcp, float* out, cudaStream_t s) {
  const int sx16 = (int)((double)w / cw * 65536.0), sy16 = (int)((double)h / ch * 65536.0);
  const int tiles = ((cw + kDcTileW - 1) / kDcTileW) * ((ch + kDcRows - 1) / kDcRows);
  k_depth_cache_set<<<persistent_blocks(k_depth_cache_set, tiles, g_set_blocks), kDcThreads, 0, s>>>(src, w, h, cw, ch, sx16,
                                                                                                     sy16, rcp, out);
  count_launches(1);
}

void launch_depth_cache_fetch(const float* img, int istride, int vx0, int vy0, int vw, int vh, double offx, double offy, double sx,
                              double sy, int rw, int rh, const uint32_t* rcp, float* out, cudaStream_t s) {
  const int ox16 = (int)(offx * 65536.0), oy16 = (int)(offy * 65536.0), sx16 = (int)(sx * 65536.0), sy16 = (int)(sy * 65536.0);
  const int tiles = ((rw + kDcTileW - 1) / kDcTileW) * ((rh + kDcRows - 1) / kDcRows);
  k_depth_cache_fetch<<<persistent_blocks(k_depth_cache_fetch, tiles, g_fetch_blocks), kDcThreads, 0, s>>>(
      img, istride, vx0, vy0, vw, vh, (vw / 32) * 32, sx16, sy16, ox16, oy16, rw, rh, rcp, out);
  count_launches(1);
}

}  // namespace lux
