// The opt-in census stereo mode of a rectified grey pair (no counterpart in the reference, whose dense stage is the
// plane sweep): census transform, Hamming matching cost, eight-path semi-global aggregation with constant penalties P1 and
// P2, winner-take-all with parabolic subpixel refinement and a left/right consistency check, and the fusion of several
// pairs' disparities into one depth map. The method is Hirschmueller's semi-global matching (PAMI 2008) on the census
// transform of Zabih and Woodfill (ECCV 1994); the conventions (9x7 window, out-of-range cost 62, first minimum, the
// median fusion) are spelled out with each kernel.
//
// Layout in HBM: census images W x H uint64; the cost volume [pixel][Dp] uint8 and the path sums [pixel][Dp] uint16 with
// Dp = 32 x LPT >= D (disparities over the 32 lanes of a warp, LPT per lane).
#include "../../include/lux_sgm.h"
#include "common.cuh"
#include "internal.h"

namespace lux {

namespace {

constexpr int kCensusWX = 4, kCensusWY = 3;  // a 9x7 window: 62 bits
constexpr uint32_t kInvalidCost = 62;        // the cost where x - d leaves the image
constexpr uint32_t kBig = 1u << 20;          // disparities past D: never a minimum

// value i of a lane's LPT registers (i known only at run time)
template <int LPT>
LUX_DEV uint32_t pick(const uint32_t (&v)[LPT], int i) {
  uint32_t r = v[0];
#pragma unroll
  for (int k = 1; k < LPT; k++) r = i == k ? v[k] : r;
  return r;
}

// The first disparity with the least path sum S[0..D) of a pixel held by a warp (LPT a lane), with the parabolic subpixel
// correction (S[d-1] - S[d+1]) / (2 (S[d-1] - 2 S[d] + S[d+1])) where 0 < d < D - 1 and the denominator is positive.
template <int LPT>
LUX_DEV void wta_of(const uint32_t (&s)[LPT], int lane, int D, int subpixel, int& d_out, float& disp_out) {
  uint32_t best = kBig, arg = kBig;
#pragma unroll
  for (int i = 0; i < LPT; i++) {
    const int d = lane * LPT + i;
    const uint32_t v = d < D ? (s[i] & 0xffffu) : kBig;
    if (v < best) {
      best = v;
      arg = d;
    }
  }
  const uint32_t m = __reduce_min_sync(0xffffffffu, best);
  const int d = (int)__reduce_min_sync(0xffffffffu, best == m ? arg : kBig);
  const int dm = max(d - 1, 0), dp = min(d + 1, D - 1);
  const float a = (float)__shfl_sync(0xffffffffu, pick<LPT>(s, dm % LPT) & 0xffffu, dm / LPT);
  const float c = (float)__shfl_sync(0xffffffffu, pick<LPT>(s, dp % LPT) & 0xffffu, dp / LPT);
  float out = (float)d;
  if (subpixel && d > 0 && d < D - 1) {
    const float b = (float)m;
    const float den = __fmul_rn(2.0f, __fadd_rn(__fsub_rn(a, __fmul_rn(2.0f, b)), c));
    if (den > 0.0f) out = __fadd_rn(out, __fdiv_rn(__fsub_rn(a, c), den));
  }
  d_out = d;
  disp_out = out;
}

// Bit k (row-major over the window, centre skipped) is set when that neighbour, read at the clamped position, is darker
// than the centre.
__global__ void k_census(const uint8_t* __restrict__ img, int w, int h, int stride, int bpp, uint64_t* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  auto at = [&](int xx, int yy) { return (int)__ldg(img + ((size_t)min(max(yy, 0), h - 1) * stride + min(max(xx, 0), w - 1)) * bpp); };
  const int c = at(x, y);
  uint64_t v = 0;
  int bit = 0;
#pragma unroll
  for (int dy = -kCensusWY; dy <= kCensusWY; dy++)
#pragma unroll
    for (int dx = -kCensusWX; dx <= kCensusWX; dx++) {
      if (dx == 0 && dy == 0) continue;
      v |= (uint64_t)(at(x + dx, y + dy) < c) << bit;
      bit++;
    }
  out[(size_t)y * w + x] = v;
}

// C(x, y, d) = popcount(L(x, y) ^ R(x - d, y)), 62 where x - d < 0. A warp per pixel, lane j making disparities j, j + 32,
// ...: each load instruction reads 32 neighbouring right-image words and each store writes 32 consecutive cost bytes.
template <int LPT>
__global__ void __launch_bounds__(256) k_hamming(const uint64_t* __restrict__ cl, const CensusPairs ps, int w, int h) {
  constexpr int Dp = 32 * LPT;
  const CensusPair& pr = ps.p[blockIdx.y];  // one grid row per pair of the batch
  const uint64_t* __restrict__ cr = pr.cr;
  uint8_t* __restrict__ cost = pr.cost;
  const int D = pr.D;
  const int lane = threadIdx.x & 31;
  const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (p >= w * h) return;
  const int y = p / w, x = p - y * w;
  const uint64_t a = __ldg(cl + p);
  const uint64_t* row = cr + (size_t)y * w;
  uint8_t* out = cost + (size_t)p * Dp;
#pragma unroll
  for (int k = 0; k < LPT; k++) {
    const int d = lane + 32 * k;
    out[d] = (uint8_t)(d < D && x - d >= 0 ? __popcll(a ^ __ldg(row + x - d)) : kInvalidCost);
  }
}

// A lane's LPT cost bytes and LPT path sums as one vector access each.
template <int LPT>
struct LaneIO;
template <>
struct LaneIO<1> {
  static LUX_DEV void cost(const uint8_t* p, uint32_t (&c)[1]) { c[0] = *p; }
  static LUX_DEV void load(const uint16_t* p, uint32_t (&v)[1]) { v[0] = *p; }
  static LUX_DEV void store(uint16_t* p, const uint32_t (&v)[1]) { *p = (uint16_t)v[0]; }
};
template <>
struct LaneIO<2> {
  static LUX_DEV void cost(const uint8_t* p, uint32_t (&c)[2]) {
    const uint32_t w = *reinterpret_cast<const uint16_t*>(p);
    c[0] = w & 0xff;
    c[1] = w >> 8;
  }
  static LUX_DEV void load(const uint16_t* p, uint32_t (&v)[2]) {
    const uint32_t w = *reinterpret_cast<const uint32_t*>(p);
    v[0] = w & 0xffff;
    v[1] = w >> 16;
  }
  static LUX_DEV void store(uint16_t* p, const uint32_t (&v)[2]) { *reinterpret_cast<uint32_t*>(p) = v[0] | v[1] << 16; }
};
template <>
struct LaneIO<4> {
  static LUX_DEV void cost(const uint8_t* p, uint32_t (&c)[4]) {
    const uint32_t w = *reinterpret_cast<const uint32_t*>(p);
#pragma unroll
    for (int i = 0; i < 4; i++) c[i] = (w >> (8 * i)) & 0xff;
  }
  static LUX_DEV void load(const uint16_t* p, uint32_t (&v)[4]) {
    const uint2 w = *reinterpret_cast<const uint2*>(p);
    v[0] = w.x & 0xffff;
    v[1] = w.x >> 16;
    v[2] = w.y & 0xffff;
    v[3] = w.y >> 16;
  }
  static LUX_DEV void store(uint16_t* p, const uint32_t (&v)[4]) {
    *reinterpret_cast<uint2*>(p) = make_uint2(v[0] | v[1] << 16, v[2] | v[3] << 16);
  }
};
template <>
struct LaneIO<8> {
  static LUX_DEV void cost(const uint8_t* p, uint32_t (&c)[8]) {
    const uint2 w = *reinterpret_cast<const uint2*>(p);
#pragma unroll
    for (int i = 0; i < 4; i++) {
      c[i] = (w.x >> (8 * i)) & 0xff;
      c[4 + i] = (w.y >> (8 * i)) & 0xff;
    }
  }
  static LUX_DEV void load(const uint16_t* p, uint32_t (&v)[8]) {
    const uint4 w = *reinterpret_cast<const uint4*>(p);
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
      v[2 * i] = ws[i] & 0xffff;
      v[2 * i + 1] = ws[i] >> 16;
    }
  }
  static LUX_DEV void store(uint16_t* p, const uint32_t (&v)[8]) {
    *reinterpret_cast<uint4*>(p) = make_uint4(v[0] | v[1] << 16, v[2] | v[3] << 16, v[4] | v[5] << 16, v[6] | v[7] << 16);
  }
};

// One warp walks one scanline of direction (dx, dy):
//   L(p, d) = C(p, d) + min(L(q, d), L(q, d - 1) + P1, L(q, d + 1) + P1, m + P2) - m,  m = min_k L(q, k),
// with q the previous pixel (L = C at the first pixel), and adds L into the path sums (the first direction stores them).
// The scanline starts are the pixels whose previous pixel lies outside the image: a whole row for dy != 0, then a whole
// column (less the corner already counted) for dx != 0. The next pixel's cost and sums are loaded while this one is
// computed, so the HBM latency is off the recurrence.
template <int LPT, bool LAST>
__global__ void __launch_bounds__(128) k_census_path(const CensusPairs ps, int w, int h, int dx, int dy, uint32_t P1, uint32_t P2,
                                                     int first, int subpixel) {
  constexpr int Dp = 32 * LPT;
  const CensusPair& pr = ps.p[blockIdx.y];  // one grid row per pair of the batch
  const uint8_t* __restrict__ cost = pr.cost;
  uint16_t* __restrict__ S = pr.S;
  int* __restrict__ dl = pr.dl;
  float* __restrict__ disp = pr.disp;
  const int D = pr.D;
  using IO = LaneIO<LPT>;
  const int lane = threadIdx.x & 31;
  const int line = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int n_row = dy != 0 ? w : 0, n_col = dx != 0 ? h - (dy != 0 ? 1 : 0) : 0;
  if (line >= n_row + n_col) return;
  int x, y;
  if (line < n_row) {
    x = line;
    y = dy > 0 ? 0 : h - 1;
  } else {
    x = dx > 0 ? 0 : w - 1;
    const int k = line - n_row;
    y = dy == 0 ? k : (dy > 0 ? k + 1 : k);  // the corner row was started by the row starts
  }
  auto at = [&](int xx, int yy) { return ((size_t)yy * w + xx) * Dp + lane * LPT; };
  uint32_t L[LPT], c[LPT], sv[LPT];
  uint32_t m = 0;
  IO::cost(cost + at(x, y), c);
  if (!first) IO::load(S + at(x, y), sv);
  bool start = true;
  for (;;) {
    const int xn = x + dx, yn = y + dy;
    const bool more = xn >= 0 && xn < w && yn >= 0 && yn < h;
    uint32_t cn[LPT], sn[LPT];
    if (more) {
      IO::cost(cost + at(xn, yn), cn);
      if (!first) IO::load(S + at(xn, yn), sn);
    }
    uint32_t nl[LPT];
    if (start) {
#pragma unroll
      for (int i = 0; i < LPT; i++) nl[i] = lane * LPT + i < D ? c[i] : kBig;
      start = false;
    } else {
      const uint32_t left = __shfl_up_sync(0xffffffffu, L[LPT - 1], 1), right = __shfl_down_sync(0xffffffffu, L[0], 1);
#pragma unroll
      for (int i = 0; i < LPT; i++) {
        const uint32_t lm = i > 0 ? L[i - 1] : (lane > 0 ? left : kBig);
        const uint32_t lp = i < LPT - 1 ? L[i + 1] : (lane < 31 ? right : kBig);
        const uint32_t t = min(min(L[i], min(lm, lp) + P1), m + P2);
        nl[i] = lane * LPT + i < D ? c[i] + t - m : kBig;
      }
    }
    uint32_t lmin = kBig, out[LPT];
#pragma unroll
    for (int i = 0; i < LPT; i++) {
      L[i] = nl[i];
      lmin = min(lmin, nl[i]);
      out[i] = first ? nl[i] : sv[i] + nl[i];  // padding lanes store don't-care values (never read)
    }
    m = __reduce_min_sync(0xffffffffu, lmin);
    IO::store(S + at(x, y), out);
    if (LAST) {  // the path sums of this pixel are final: the winner-take-all here saves reading them again
      int d;
      float v;
      wta_of<LPT>(out, lane, D, subpixel, d, v);
      if (lane == 0) {
        dl[(size_t)y * w + x] = d;
        disp[(size_t)y * w + x] = v;
      }
    }
    if (!more) break;
    x = xn;
    y = yn;
#pragma unroll
    for (int i = 0; i < LPT; i++) {
      c[i] = cn[i];
      sv[i] = sn[i];
    }
  }
}

// The right image's first minimum over d of S(x + d, y, d), x + d < W (a warp per right-image pixel).
template <int LPT>
__global__ void __launch_bounds__(256) k_census_wta_right(const CensusPairs ps, int w, int h) {
  constexpr int Dp = 32 * LPT;
  const CensusPair& pr = ps.p[blockIdx.y];
  const uint16_t* __restrict__ S = pr.S;
  int* __restrict__ dr = pr.dr;
  const int D = pr.D;
  const int lane = threadIdx.x & 31;
  const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (p >= w * h) return;
  const int y = p / w, x = p - y * w;
  uint32_t best = kBig, arg = kBig;
#pragma unroll
  for (int i = 0; i < LPT; i++) {
    const int d = lane * LPT + i;
    const uint32_t v = d < D && x + d < w ? __ldg(S + ((size_t)y * w + x + d) * Dp + d) : kBig;
    if (v < best) {
      best = v;
      arg = d;
    }
  }
  const uint32_t m = __reduce_min_sync(0xffffffffu, best);
  const uint32_t d = __reduce_min_sync(0xffffffffu, best == m ? arg : kBig);
  if (lane == 0) dr[p] = (int)d;
}

// Left/right consistency: a pixel keeps its disparity when |d(x) - d_R(x - d(x))| <= max_diff, else -1.
__global__ void k_census_lr(const CensusPairs ps, int w, int h, int max_diff) {
  const CensusPair& pr = ps.p[blockIdx.y];
  const int* __restrict__ dl = pr.dl;
  const int* __restrict__ dr = pr.dr;
  float* __restrict__ disp = pr.disp;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= w * h) return;
  const int y = p / w, x = p - y * w, d = dl[p], xr = x - d;
  if (xr < 0 || abs(d - dr[(size_t)y * w + xr]) > max_diff) disp[p] = -1.0f;
}

// The median of a pixel's valid depths fB_k / d_k (d_k > 0) over the pairs (the mean of the two middle ones for an even
// count), 0 where none is valid.
__global__ void k_fuse(const float* const* __restrict__ disps, const float* __restrict__ fb, int n, int npx, float* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npx) return;
  float z[kMaxFusePairs];
  int k = 0;
  for (int i = 0; i < n; i++) {
    const float d = disps[i][p];
    if (d > 0.0f) {
      const float v = __fdiv_rn(fb[i], d);
      int j = k++;
      while (j > 0 && z[j - 1] > v) {  // insertion, ascending
        z[j] = z[j - 1];
        j--;
      }
      z[j] = v;
    }
  }
  out[p] = k == 0 ? 0.0f : (k & 1) ? z[k / 2] : __fmul_rn(__fadd_rn(z[k / 2 - 1], z[k / 2]), 0.5f);
}

template <int LPT>
void batch_stages(const uint64_t* cl, const CensusPairs& ps, int n, int w, int h, uint32_t P1, uint32_t P2, int subpixel, int lr,
                  int max_diff, cudaStream_t s) {
  const int npx = w * h;
  k_hamming<LPT><<<dim3((unsigned)((npx + 7) / 8), n), 256, 0, s>>>(cl, ps, w, h);
  static const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {1, -1}, {-1, 1}};
  for (int k = 0; k < 8; k++) {
    const int dx = dirs[k][0], dy = dirs[k][1];
    const int lines = (dy != 0 ? w : 0) + (dx != 0 ? h - (dy != 0 ? 1 : 0) : 0);
    const dim3 grid((lines + 3) / 4, n);
    if (k == 7) k_census_path<LPT, true><<<grid, 128, 0, s>>>(ps, w, h, dx, dy, P1, P2, 0, subpixel);
    else k_census_path<LPT, false><<<grid, 128, 0, s>>>(ps, w, h, dx, dy, P1, P2, k == 0 ? 1 : 0, subpixel);
  }
  count_launches(9);
  if (lr) {
    k_census_wta_right<LPT><<<dim3((npx + 7) / 8, n), 256, 0, s>>>(ps, w, h);
    k_census_lr<<<dim3((npx + 255) / 256, n), 256, 0, s>>>(ps, w, h, max_diff);
    count_launches(2);
  }
}

}  // namespace

int census_lpt(int D) { return D <= 32 ? 1 : D <= 64 ? 2 : D <= 128 ? 4 : D <= 256 ? 8 : 0; }

void launch_census_batch(const uint8_t* ref, const uint8_t* const* others, int n, int w, int h, int stride, int bpp, uint32_t P1,
                         uint32_t P2, int subpixel, int lr, int max_diff, uint64_t* cl, const CensusPairs& ps, cudaStream_t s) {
  const dim3 b2(32, 8), g2((w + 31) / 32, (h + 7) / 8);
  k_census<<<g2, b2, 0, s>>>(ref, w, h, stride, bpp, cl);  // the reference's census, shared by every pair
  for (int k = 0; k < n; k++) k_census<<<g2, b2, 0, s>>>(others[k], w, h, stride, bpp, ps.p[k].cr);
  count_launches(1 + n);
  // the pairs grouped by lane width (disparities a lane), one launch per stage and group
  for (const int lpt : {1, 2, 4, 8}) {
    CensusPairs grp{};
    int m = 0;
    for (int k = 0; k < n; k++)
      if (census_lpt(ps.p[k].D) == lpt) grp.p[m++] = ps.p[k];
    if (m == 0) continue;
    switch (lpt) {
      case 1: batch_stages<1>(cl, grp, m, w, h, P1, P2, subpixel, lr, max_diff, s); break;
      case 2: batch_stages<2>(cl, grp, m, w, h, P1, P2, subpixel, lr, max_diff, s); break;
      case 4: batch_stages<4>(cl, grp, m, w, h, P1, P2, subpixel, lr, max_diff, s); break;
      default: batch_stages<8>(cl, grp, m, w, h, P1, P2, subpixel, lr, max_diff, s); break;
    }
  }
}

void launch_fuse(const float* const* disps, const float* fb, int n, int npx, float* out, cudaStream_t s) {
  k_fuse<<<(npx + 255) / 256, 256, 0, s>>>(disps, fb, n, npx, out);
  count_launches(1);
}

}  // namespace lux
