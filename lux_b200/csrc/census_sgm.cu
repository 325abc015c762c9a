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

// C(x, y, d) = popcount(L(x, y) ^ R(x - d, y)), 62 where x - d < 0. A thread makes eight disparities of one pixel (one
// 8-byte store); threads of a warp take neighbouring pixels, so the right-image reads of a disparity are one coalesced row.
__global__ void k_hamming(const uint64_t* __restrict__ cl, const uint64_t* __restrict__ cr, int w, int h, int D, int Dp,
                          uint8_t* __restrict__ cost) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, g = blockIdx.z;
  if (x >= w) return;
  const uint64_t a = __ldg(cl + (size_t)y * w + x);
  uint32_t lo = 0, hi = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const int d = g * 8 + k;
    uint32_t c = kInvalidCost;
    if (d < D && x - d >= 0) c = (uint32_t)__popcll(a ^ __ldg(cr + (size_t)y * w + x - d));
    if (k < 4) lo |= c << (8 * k);
    else hi |= c << (8 * (k - 4));
  }
  *reinterpret_cast<uint2*>(cost + ((size_t)y * w + x) * Dp + g * 8) = make_uint2(lo, hi);
}

// One warp walks one scanline of direction (dx, dy):
//   L(p, d) = C(p, d) + min(L(q, d), L(q, d - 1) + P1, L(q, d + 1) + P1, m + P2) - m,  m = min_k L(q, k),
// with q the previous pixel (L = C at the first pixel), and adds L into the path sums (the first direction stores them).
// The scanline starts are the pixels whose previous pixel lies outside the image: a whole row for dy != 0, then a whole
// column (less the corner already counted) for dx != 0.
template <int LPT>
__global__ void __launch_bounds__(128) k_census_path(const uint8_t* __restrict__ cost, int w, int h, int D, int dx, int dy, uint32_t P1,
                                                     uint32_t P2, int first, uint16_t* __restrict__ S) {
  constexpr int Dp = 32 * LPT;
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
  uint32_t L[LPT];
  uint32_t m = 0;
  bool start = true;
  for (; x >= 0 && x < w && y >= 0 && y < h; x += dx, y += dy) {
    const size_t p = (size_t)y * w + x;
    uint32_t c[LPT];
    {
      const uint8_t* cp = cost + p * Dp + lane * LPT;
#pragma unroll
      for (int i = 0; i < LPT; i++) c[i] = cp[i];
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
    uint32_t lmin = kBig;
#pragma unroll
    for (int i = 0; i < LPT; i++) {
      L[i] = nl[i];
      lmin = min(lmin, nl[i]);
    }
    m = __reduce_min_sync(0xffffffffu, lmin);
    uint16_t* sp = S + p * Dp + lane * LPT;
#pragma unroll
    for (int i = 0; i < LPT; i++) {
      if (lane * LPT + i >= D) continue;
      sp[i] = (uint16_t)(first ? L[i] : sp[i] + L[i]);
    }
  }
}

// The first disparity with the least path sum of a pixel (a warp per pixel), with the parabolic subpixel correction
// (S[d-1] - S[d+1]) / (2 (S[d-1] - 2 S[d] + S[d+1])) where 0 < d < D - 1 and the denominator is positive.
template <int LPT>
__global__ void __launch_bounds__(256) k_census_wta(const uint16_t* __restrict__ S, int npx, int D, int subpixel, int* __restrict__ dl,
                                                    float* __restrict__ disp) {
  constexpr int Dp = 32 * LPT;
  const int lane = threadIdx.x & 31;
  const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (p >= npx) return;
  const uint16_t* sp = S + (size_t)p * Dp;
  uint32_t best = kBig, arg = kBig;
#pragma unroll
  for (int i = 0; i < LPT; i++) {
    const int d = lane * LPT + i;
    const uint32_t v = d < D ? sp[d] : kBig;
    if (v < best) {
      best = v;
      arg = d;
    }
  }
  const uint32_t m = __reduce_min_sync(0xffffffffu, best);
  const uint32_t d = __reduce_min_sync(0xffffffffu, best == m ? arg : kBig);
  if (lane == 0) {
    float out = (float)d;
    if (subpixel && d > 0 && (int)d < D - 1) {
      const float a = sp[d - 1], b = sp[d], c = sp[d + 1];
      const float den = __fmul_rn(2.0f, __fadd_rn(__fsub_rn(a, __fmul_rn(2.0f, b)), c));
      if (den > 0.0f) out = __fadd_rn(out, __fdiv_rn(__fsub_rn(a, c), den));
    }
    dl[p] = (int)d;
    disp[p] = out;
  }
}

// The right image's first minimum over d of S(x + d, y, d), x + d < W (a warp per right-image pixel).
template <int LPT>
__global__ void __launch_bounds__(256) k_census_wta_right(const uint16_t* __restrict__ S, int w, int h, int D, int* __restrict__ dr) {
  constexpr int Dp = 32 * LPT;
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
__global__ void k_census_lr(const int* __restrict__ dl, const int* __restrict__ dr, int w, int h, int max_diff, float* __restrict__ disp) {
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
void paths_and_wta(const uint8_t* cost, int w, int h, int D, uint32_t P1, uint32_t P2, int subpixel, int lr, int max_diff,
                   uint16_t* S, int* dl, int* dr, float* disp, cudaStream_t s) {
  static const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {1, -1}, {-1, 1}};
  for (int k = 0; k < 8; k++) {
    const int dx = dirs[k][0], dy = dirs[k][1];
    const int lines = (dy != 0 ? w : 0) + (dx != 0 ? h - (dy != 0 ? 1 : 0) : 0);
    k_census_path<LPT><<<(lines + 3) / 4, 128, 0, s>>>(cost, w, h, D, dx, dy, P1, P2, k == 0 ? 1 : 0, S);
  }
  const int npx = w * h;
  k_census_wta<LPT><<<(npx + 7) / 8, 256, 0, s>>>(S, npx, D, subpixel, dl, disp);
  count_launches(9);
  if (lr) {
    k_census_wta_right<LPT><<<(npx + 7) / 8, 256, 0, s>>>(S, w, h, D, dr);
    k_census_lr<<<(npx + 255) / 256, 256, 0, s>>>(dl, dr, w, h, max_diff, disp);
    count_launches(2);
  }
}

}  // namespace

int census_lpt(int D) { return D <= 32 ? 1 : D <= 64 ? 2 : D <= 128 ? 4 : D <= 256 ? 8 : 0; }

void launch_census_sgm(const uint8_t* left, const uint8_t* right, int w, int h, int stride, int bpp, int D, uint32_t P1, uint32_t P2,
                       int subpixel, int lr, int max_diff, uint64_t* cl, uint64_t* cr, uint8_t* cost, uint16_t* S, int* dl, int* dr,
                       float* disp, cudaStream_t s) {
  const int lpt = census_lpt(D), Dp = 32 * lpt;
  const dim3 b2(32, 8), g2((w + 31) / 32, (h + 7) / 8);
  k_census<<<g2, b2, 0, s>>>(left, w, h, stride, bpp, cl);
  k_census<<<g2, b2, 0, s>>>(right, w, h, stride, bpp, cr);
  k_hamming<<<dim3((w + 127) / 128, h, Dp / 8), 128, 0, s>>>(cl, cr, w, h, D, Dp, cost);
  count_launches(3);
  switch (lpt) {
    case 1: paths_and_wta<1>(cost, w, h, D, P1, P2, subpixel, lr, max_diff, S, dl, dr, disp, s); break;
    case 2: paths_and_wta<2>(cost, w, h, D, P1, P2, subpixel, lr, max_diff, S, dl, dr, disp, s); break;
    case 4: paths_and_wta<4>(cost, w, h, D, P1, P2, subpixel, lr, max_diff, S, dl, dr, disp, s); break;
    default: paths_and_wta<8>(cost, w, h, D, P1, P2, subpixel, lr, max_diff, S, dl, dr, disp, s); break;
  }
}

void launch_fuse(const float* const* disps, const float* fb, int n, int npx, float* out, cudaStream_t s) {
  k_fuse<<<(npx + 255) / 256, 256, 0, s>>>(disps, fb, n, npx, out);
  count_launches(1);
}

}  // namespace lux
