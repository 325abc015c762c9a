// The depth image cache that the renderer and exporter read (Lux.Engine/Pipeline/Export/DepthCache.cs), fed by the
// upsampled full-resolution depth: Set (inverse depth, nearest resample to the cache dims, clipped inverse back) and
// Fetch (a ROI at another pipeline level: a reciprocal pass over the source window, nearest resample, division back).
// Every float step keeps the reference's operation and rounding (rcpps = IntelApprox.RcpBits on the table; one Newton
// step (1 - v·r)·r + r; IEEE division), so results are bit-identical.
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

// Set: only the source pixels the nearest resample reads are inverted (InverseDepth is per pixel, so the values are
// those of inverting the whole image first); then minps(rcpps(x), 1e5).
__global__ void k_depth_cache_set(const float* __restrict__ src, int w, int h, int cw, int ch, int sx16, int sy16,
                                  const uint32_t* __restrict__ rcp, float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= cw) return;
  const float v = src[(size_t)nearest16(sy16, 0, y, h) * w + nearest16(sx16, 0, x, w)];
  const float r = rcp_approx(rcp_approx(v, rcp), rcp);
  out[(size_t)y * cw + x] = r < 100000.0f ? r : 100000.0f;
}

// Fetch (FetchFull / FetchSampled, DepthCache.cs:185-239): per output pixel the window pixel it samples, its reciprocal
// (columns below vec: rcpps + one Newton step, then x 1.0; the rest: division), and the division back.
__global__ void k_depth_cache_fetch(const float* __restrict__ img, int istride, int vx0, int vy0, int vw, int vh, int vec, int sx16,
                                    int sy16, int ox16, int oy16, int rw, int rh, const uint32_t* __restrict__ rcp,
                                    float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= rw) return;
  const int px = nearest16(sx16, ox16, x, vw), py = nearest16(sy16, oy16, y, vh);
  const float v = img[(size_t)(vy0 + py) * istride + vx0 + px];
  float inv;
  if (px < vec) {
    const float r = rcp_approx(v, rcp);
    inv = __fmul_rn(__fadd_rn(__fmul_rn(__fsub_rn(1.0f, __fmul_rn(v, r)), r), r), 1.0f);
  } else {
    inv = __fdiv_rn(1.0f, v);
  }
  out[(size_t)y * rw + x] = x86_nan(__fdiv_rn(1.0f, inv), v);
}

void launch_depth_cache_set(const float* src, int w, int h, int cw, int ch, const uint32_t* rcp, float* out, cudaStream_t s) {
  const int sx16 = (int)((double)w / cw * 65536.0), sy16 = (int)((double)h / ch * 65536.0);
  k_depth_cache_set<<<dim3((cw + 127) / 128, ch), 128, 0, s>>>(src, w, h, cw, ch, sx16, sy16, rcp, out);
  count_launches(1);
}

void launch_depth_cache_fetch(const float* img, int istride, int vx0, int vy0, int vw, int vh, double offx, double offy, double sx,
                              double sy, int rw, int rh, const uint32_t* rcp, float* out, cudaStream_t s) {
  const int ox16 = (int)(offx * 65536.0), oy16 = (int)(offy * 65536.0), sx16 = (int)(sx * 65536.0), sy16 = (int)(sy * 65536.0);
  k_depth_cache_fetch<<<dim3((rw + 127) / 128, rh), 128, 0, s>>>(img, istride, vx0, vy0, vw, vh, (vw / 32) * 32, sx16, sy16, ox16,
                                                                  oy16, rw, rh, rcp, out);
  count_launches(1);
}

}  // namespace lux
