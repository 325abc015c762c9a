// Plane-sweep matching cost -> u8 raw volume: DenseStereo.MatchingCost + Normalise (DenseStereo.cs:217-292, 376-381).
//
// One warp per reference pixel, lanes over planes. Per other camera and plane: the projection through the flow matrix
// (no FMA, IEEE 1/pz; the plane-only terms z·W2 + W3 come from a per-layer table), the half-pixel `pavgb` resampling
// of the target block, capped |diff| of the 3x3 blocks, the fixed-point channel weights, and a u16 wrap-sum over
// cameras. A plane whose position repeats or leaves the valid rect reuses the last computed cost (:273-274): the warp
// finds that plane with a ballot and carries it across chunks of 32 planes.
//
// Half-pixel phases: the resampled block value at (x, y) with fractions (hx, hy) is pavgb over rows first, then over
// columns, of the 2x2 neighbourhood at (x, y) (:248-253); it depends on (x, y, hx, hy) only, so k_phase_* writes the four
// phase images of every other camera once per layer and a plane's 3x3 block is three row loads with no averaging:
//   grey camera (weights {12240, 0, 0, 0}, only Y contributes): per pixel and phase the Y bytes of columns x, x+1, x+2
//     as u16 pairs {x | x+2 << 16, x+1}, so a block row is one 8-byte load; |t - r| capped at 2 in u16x2 lanes;
//   colour camera: the RGBA word per pixel and phase; even bytes (Y, V) and odd bytes (U, A) as u16x2 lanes.
// Both are exact restatements of the reference's byte-lane sums (each channel sum is at most 9·6).
#include <climits>

#include "common.cuh"
#include "internal.h"

namespace lux {

LUX_DEV uint32_t vmin2c(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("min.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
LUX_DEV uint32_t vmax2c(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("max.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
LUX_DEV uint32_t absdiff2(uint32_t a, uint32_t b) { return vmax2c(a, b) - vmin2c(a, b); }  // per u16 lane, no borrow
LUX_DEV int avg_u8(int a, int b) { return (a + b + 1) >> 1; }                 // pavgb on one byte

// The phase-h value (h = 2·hy + hx) of byte channel `ch` at (x, y): rows averaged first, then columns. Only positions
// whose 2x2 neighbourhood lies in the image are ever read by the cost; the others are clamped.
LUX_DEV int phase_byte(const uint8_t* img, int iw, int ih, int x, int y, int h, int ch) {
  const int x1 = min(x + 1, iw - 1), y1 = min(y + 1, ih - 1);
  auto at = [&](int xx, int yy) { return (int)img[((size_t)yy * iw + xx) * 4 + ch]; };
  int a = at(x, y), b = at(x1, y);
  if (h & 2) {
    a = avg_u8(a, at(x, y1));
    b = avg_u8(b, at(x1, y1));
  }
  return (h & 1) ? avg_u8(a, b) : a;
}

// Grey: out[h][y][x] = the Y bytes of phase h at columns x, x+1, x+2 as u16 pairs: {x | x+2 << 16, x+1}.
__global__ void k_phase_grey(const uint8_t* __restrict__ img, int iw, int ih, uint2* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= iw) return;
#pragma unroll
  for (int h = 0; h < 4; h++) {
    const uint32_t p0 = phase_byte(img, iw, ih, x, y, h, 0), p1 = phase_byte(img, iw, ih, min(x + 1, iw - 1), y, h, 0),
                   p2 = phase_byte(img, iw, ih, min(x + 2, iw - 1), y, h, 0);
    out[((size_t)h * ih + y) * iw + x] = make_uint2(p0 | (p2 << 16), p1);
  }
}
// Grey, vertical triples (the shared-column axis kernel): out[h][y][x] = the Y bytes of phase h at rows y, y+1, y+2 of
// column x as u16 pairs: {y | y+2 << 16, y+1}.
__global__ void k_phase_grey_v(const uint8_t* __restrict__ img, int iw, int ih, uint2* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= iw) return;
#pragma unroll
  for (int h = 0; h < 4; h++) {
    const uint32_t p0 = phase_byte(img, iw, ih, x, y, h, 0), p1 = phase_byte(img, iw, ih, x, min(y + 1, ih - 1), h, 0),
                   p2 = phase_byte(img, iw, ih, x, min(y + 2, ih - 1), h, 0);
    out[((size_t)h * ih + y) * iw + x] = make_uint2(p0 | (p2 << 16), p1);
  }
}
// Colour: out[h][y][x] = the RGBA word of phase h.
__global__ void k_phase_colour(const uint8_t* __restrict__ img, int iw, int ih, uint32_t* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= iw) return;
#pragma unroll
  for (int h = 0; h < 4; h++) {
    uint32_t v = 0;
#pragma unroll
    for (int ch = 0; ch < 4; ch++) v |= (uint32_t)phase_byte(img, iw, ih, x, y, h, ch) << (8 * ch);
    out[((size_t)h * ih + y) * iw + x] = v;
  }
}

// Grey block: S0 = Σ min(|t - r|, 2) over the 3x3 Y block. Row r of the target is one 8-byte load {t0 | t2 << 16, t1}.
// In each u16 lane max(t + (256 - r), (256 + r) - t) = 256 + |t - r|, so min(., 258) - 256 is the capped difference
// with two adds and two min/max instead of three min/max and a subtract (the 256s are removed once, at the end); the
// unused upper lane of the odd word is capped at 256 (a zero term).
struct GreyRef {
  uint32_t ea[3], eb[3], oa[3], ob[3];  // per row: 256 - r and 256 + r for the lanes {r0, r2} and {r1, 0}
};
LUX_DEV GreyRef grey_ref(const uint32_t (&ge)[3], const uint32_t (&go)[3]) {
  GreyRef g;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    g.ea[r] = 0x01000100u - ge[r];
    g.eb[r] = 0x01000100u + ge[r];
    g.oa[r] = 0x01000100u - go[r];
    g.ob[r] = 0x01000100u + go[r];
  }
  return g;
}
LUX_DEV int grey_cost(const uint2* __restrict__ q, int iw, const GreyRef& g) {
  uint32_t s = 0;
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const uint2 t = __ldg(q + (size_t)r * iw);
    s += vmin2c(vmax2c(t.x + g.ea[r], g.eb[r] - t.x), 0x01020102u) + vmin2c(vmax2c(t.y + g.oa[r], g.ob[r] - t.y), 0x01000102u);
  }
  const int S0 = (int)((s & 0xffffu) + (s >> 16)) - 12 * 256;
  return (S0 * 12240 + 16) >> 5;
}

// Colour block: even bytes (Y, V) and odd bytes (U, A) as u16 pairs, caps {Y:2, V:6} and {U:6, A:0}.
LUX_DEV int colour_cost(const uint32_t* __restrict__ q, int iw, const uint32_t (&re)[3][3], const uint32_t (&ro)[3][3],
                        const uint16_t (&wq)[4]) {
  const uint32_t capE = 0x00060002u, capO = 0x00000006u;
  uint32_t se = 0, so = 0;
#pragma unroll
  for (int r = 0; r < 3; r++) {
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const uint32_t w = __ldg(q + (size_t)r * iw + p);
      se += vmin2c(absdiff2(w & 0x00ff00ffu, re[r][p]), capE);
      so += vmin2c(absdiff2((w >> 8) & 0x00ff00ffu, ro[r][p]), capO);
    }
  }
  const int S0 = se & 0xffff, S2 = se >> 16, S1 = so & 0xffff, S3 = so >> 16;
  const int cY = (S0 * wq[0] + 16) >> 5, cU = (S1 * wq[1] + 16) >> 5, cV = (S2 * wq[2] + 16) >> 5, cA = (S3 * wq[3] + 16) >> 5;
  return (cY + cU) + (cV + cA);  // at most 6885: MathF.Min(…, 65535) and the float round trip change nothing
}

template <bool GREY>
__global__ void __launch_bounds__(256) k_cost(const CostArgs a, const LayerGeom g, const float4* __restrict__ zt,
                                              uint8_t* __restrict__ raw, int* err) {
  __shared__ int s_carry[8][kMaxCams];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int npx = g.W * g.H;
  const int n = g.n_planes;
  const int half = (a.scale + (a.scale >> 31)) >> 1;
  const uint32_t* ref = reinterpret_cast<const uint32_t*>(a.ref);
  for (int pi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; pi < npx; pi += nwarps) {
    if (g.skip[pi]) {  // skipped pixels aggregate raw 0 and 255 past their count (DenseStereoSgm.cs:242)
      uint8_t* out = raw + g.off[pi];
      const int count = g.count[pi], cap = g.cap[pi];
      for (int d = lane; d < cap; d += 32) out[d] = d < count ? 0 : 255;
      continue;
    }
    const int x = pi % g.W, y = pi / g.W;
    const int xImg = min(a.scale * x + half, a.rw - 1), yImg = min(a.scale * y + half, a.rh - 1);
    const int start = g.start[pi], count = g.count[pi], cap = g.cap[pi];
    uint8_t* out = raw + g.off[pi];
    if (start + count > n) {  // MatchingCostScalar would index Planes past its end
      if (lane == 0) atomicCAS(err, 0, 7);
      continue;
    }
    // the reference 3x3 block, rows/columns clamped to the image
    uint32_t ge[3], go[3], re[3][3], ro[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
      const int yy = min(max(yImg + r - 1, 0), a.rh - 1);
      uint32_t yb[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const uint32_t w = __ldg(ref + (size_t)yy * a.rw + min(max(xImg + c - 1, 0), a.rw - 1));
        yb[c] = w & 0xffu;
        re[r][c] = w & 0x00ff00ffu;
        ro[r][c] = (w >> 8) & 0x00ff00ffu;
      }
      ge[r] = yb[0] | (yb[2] << 16);
      go[r] = yb[1];
    }
    const GreyRef gr = grey_ref(ge, go);
    const float xf = (float)xImg, yf = (float)yImg;
    for (int c0 = 0; c0 < count; c0 += 32) {
      const int d = c0 + lane;
      const bool valid = d < count;
      const int pl = valid ? start + d : start;
      const float z = __ldg(g.planes + pl);
      const int last = min(31, count - 1 - c0);
      const float xz = __fmul_rn(xf, z), yz = __fmul_rn(yf, z);  // (x·z)·1.0f: the product by one is exact
      uint32_t acc = 0;
      for (int k = 0; k < a.n_others; k++) {
        const float* Wm = a.warp[k];
        const int iw = a.ow[k], ih = a.oh[k];
        const int x0 = 1, y0 = 1, x1 = iw - 2, y1 = ih - 2;
        // p = ((z·W2 + W3) + xz·W0) + yz·W1 (:255-259), the first term from the table; then 1/pz and the +0.25 bias
        const float4 zk = __ldg(zt + (size_t)k * n + pl);
        const float px = __fadd_rn(__fadd_rn(zk.x, __fmul_rn(xz, Wm[0])), __fmul_rn(yz, Wm[4]));
        const float py = __fadd_rn(__fadd_rn(zk.y, __fmul_rn(xz, Wm[1])), __fmul_rn(yz, Wm[5]));
        const float pz = __fadd_rn(__fadd_rn(zk.z, __fmul_rn(xz, Wm[2])), __fmul_rn(yz, Wm[6]));
        const float inv = __frcp_rn(pz);  // the correctly rounded 1/pz, as the reference's division
        float fx = __fadd_rn(__fmul_rn(px, inv), 0.25f), fy = __fadd_rn(__fmul_rn(py, inv), 0.25f);
        if (d == 0) {  // the first plane is clamped into the rect (:263-269)
          fx = cs_minf(cs_maxf(fx, (float)x0), (float)(x1 - 1));
          fy = cs_minf(cs_maxf(fy, (float)y0), (float)(y1 - 1));
        }
        // (int)(2f) gives the integer part (>> 1) and the half-pixel bit (& 1) wherever the position can be in the rect
        // (f >= 1); elsewhere both forms fall outside it
        const int tx = f2i(__fadd_rn(fx, fx)), ty = f2i(__fadd_rn(fy, fy));
        const int ix = tx >> 1, iy = ty >> 1, h = ((ty & 1) << 1) | (tx & 1);
        bool inb = valid && !(ix < x0 || ix >= x1 || iy < y0 || iy >= y1);
        if (d == 0 && !inb) {  // the scalar fallback of the reference would read out of the image
          atomicCAS(err, 0, 7);
        }
        int costK = 0;
        if (inb) {
          const size_t qi = ((size_t)h * ih + (iy - 1)) * iw + (ix - 1);
          if (GREY) costK = grey_cost(reinterpret_cast<const uint2*>(a.phase[k]) + qi, iw, gr);
          else costK = colour_cost(a.phase[k] + qi, iw, re, ro, a.wq[k]);
        }
        const uint32_t m = __ballot_sync(0xffffffffu, inb);
        const uint32_t below = m & ((1u << lane) - 1u);
        const int src = below ? 31 - __clz(below) : 0;
        const int prevCost = __shfl_sync(0xffffffffu, costK, src);
        const int carry = c0 == 0 ? 0 : s_carry[wib][k];
        const int res = inb ? costK : (below ? prevCost : carry);
        __syncwarp();
        const int tail = __shfl_sync(0xffffffffu, res, last);
        if (lane == 0) s_carry[wib][k] = tail;
        __syncwarp();
        acc += (uint32_t)res;
      }
      if (valid) out[d] = (uint8_t)f2i(__fmul_rn((float)(acc & 0xffffu), a.norm));  // Normalise (:378-379)
    }
    for (int d = count + lane; d < cap; d += 32) out[d] = 255;  // padding planes (:380)
  }
}

// Uniform layers (every pixel searches planes [0, n), cap n, n % 8 == 0; 1 to 15 other cameras): lanes over 32
// neighbouring pixels of a row,
// each lane walking its pixel's planes in order like the reference's loop, so the last computed cost of a camera
// (:273-274) is a register, the plane terms are the same for the whole warp, and the camera constants stay in
// registers. Eight planes of u8 costs go out per 8-byte store. Skipped pixels get raw 0 (DenseStereoSgm.cs:242).
template <bool GREY, int NK>
__global__ void __launch_bounds__(256) k_cost_rows(const CostArgs a, const LayerGeom g, const float4* __restrict__ zt,
                                                   uint8_t* __restrict__ raw, int* err) {
  const int lane = threadIdx.x & 31;
  const int tiles_x = (g.W + 31) >> 5;
  const int ntiles = tiles_x * g.H;
  const int n = g.n_planes;
  const int half = (a.scale + (a.scale >> 31)) >> 1;
  const uint32_t* ref = reinterpret_cast<const uint32_t*>(a.ref);
  // NK cameras exactly (NK <= 4), or up to NK with a.n_others of them; the camera loops are unrolled, so the camera
  // constants are kernel-argument operands
  const int nk = NK <= 4 ? NK : a.n_others;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += (gridDim.x * blockDim.x) >> 5) {
    const int y = t / tiles_x, x = ((t - y * tiles_x) << 5) + lane;
    if (x >= g.W) continue;
    const size_t pi = (size_t)y * g.W + x;
    uint8_t* out = raw + pi * n;
    if (g.skip[pi]) {
      for (int d = 0; d < n; d += 8) *reinterpret_cast<uint2*>(out + d) = make_uint2(0u, 0u);
      continue;
    }
    const int xImg = min(a.scale * x + half, a.rw - 1), yImg = min(a.scale * y + half, a.rh - 1);
    uint32_t ge[3], go[3], re[3][3], ro[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++) {  // the reference 3x3 block, rows/columns clamped to the image
      const int yy = min(max(yImg + r - 1, 0), a.rh - 1);
      uint32_t yb[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const uint32_t w = __ldg(ref + (size_t)yy * a.rw + min(max(xImg + c - 1, 0), a.rw - 1));
        yb[c] = w & 0xffu;
        re[r][c] = w & 0x00ff00ffu;
        ro[r][c] = (w >> 8) & 0x00ff00ffu;
      }
      ge[r] = yb[0] | (yb[2] << 16);
      go[r] = yb[1];
    }
    const GreyRef gr = grey_ref(ge, go);
    const float xf = (float)xImg, yf = (float)yImg;
    int last[NK];
#pragma unroll
    for (int k = 0; k < NK; k++) last[k] = 0;
    uint32_t pk0 = 0, pk1 = 0;
    for (int d = 0; d < n; d++) {
      const float z = __ldg(g.planes + d);
      const float xz = __fmul_rn(xf, z), yz = __fmul_rn(yf, z);
      uint32_t acc = 0;
#pragma unroll
      for (int k = 0; k < NK; k++) {
        if (k >= nk) break;
        const float* Wm = a.warp[k];
        const int iwk = a.ow[k], ihk = a.oh[k];
        const float4 zk = __ldg(zt + (size_t)k * n + d);
        const float px = __fadd_rn(__fadd_rn(zk.x, __fmul_rn(xz, Wm[0])), __fmul_rn(yz, Wm[4]));
        const float py = __fadd_rn(__fadd_rn(zk.y, __fmul_rn(xz, Wm[1])), __fmul_rn(yz, Wm[5]));
        const float pz = __fadd_rn(__fadd_rn(zk.z, __fmul_rn(xz, Wm[2])), __fmul_rn(yz, Wm[6]));
        const float inv = __frcp_rn(pz);
        float fx = __fadd_rn(__fmul_rn(px, inv), 0.25f), fy = __fadd_rn(__fmul_rn(py, inv), 0.25f);
        const int x1 = iwk - 2, y1 = ihk - 2;
        if (d == 0) {  // the first plane is clamped into the rect (:263-269)
          fx = cs_minf(cs_maxf(fx, 1.0f), (float)(x1 - 1));
          fy = cs_minf(cs_maxf(fy, 1.0f), (float)(y1 - 1));
        }
        const int tx = f2i(__fadd_rn(fx, fx)), ty = f2i(__fadd_rn(fy, fy));
        const int ix = tx >> 1, iy = ty >> 1;
        if (ix >= 1 && ix < x1 && iy >= 1 && iy < y1) {
          const int h = ((ty & 1) << 1) | (tx & 1);
          const size_t qi = ((size_t)h * ihk + (iy - 1)) * iwk + (ix - 1);
          last[k] = GREY ? grey_cost(reinterpret_cast<const uint2*>(a.phase[k]) + qi, iwk, gr)
                         : colour_cost(a.phase[k] + qi, iwk, re, ro, a.wq[k]);
        } else if (d == 0) {  // the scalar fallback of the reference would read out of the image
          atomicCAS(err, 0, 7);
        }
        acc += (uint32_t)last[k];
      }
      const uint32_t b = (uint32_t)f2i(__fmul_rn((float)(acc & 0xffffu), a.norm)) & 0xffu;  // Normalise (:378-379)
      const int sh = (d & 3) * 8;
      if (d & 4) pk1 |= b << sh;
      else pk0 |= b << sh;
      if ((d & 7) == 7) {
        *reinterpret_cast<uint2*>(out + (d - 7)) = make_uint2(pk0, pk1);
        pk0 = pk1 = 0;
      }
    }
  }
}

// Uniform layers of one axis-aligned camera pair (flow-matrix terms W1 = W2 = W4 = W6 = 0, as for a rectified pair; the
// host checks them, that every plane term z·W10 + W14 is finite and non-zero and that x·z cannot overflow). Then, exactly:
//   pz = z·W10 + W14 (adding the ±0 products changes no non-zero value), so 1/pz is a per-plane constant (zt.w);
//   px = (z·W8 + W12) + x·z·W0, where the dropped ±0 term can only change the sign of a zero px, and a zero px gives
//     the same fx (0.25, or NaN with an infinite 1/pz) either way;
//   py = (z·W9 + W13) + y·z·W5 likewise, so the row and half-pixel bit of the target depend on (row, plane) only: lane j
//     of a warp computes them for plane d0 + j and the warp shuffles them to every pixel.
// The first plane (clamped into the rect) keeps the general projection.
template <bool GREY>
__global__ void __launch_bounds__(256) k_cost_axis(const CostArgs a, const LayerGeom g, const float4* __restrict__ zt,
                                                   uint8_t* __restrict__ raw, int* err) {
  const int lane = threadIdx.x & 31;
  const int tiles_x = (g.W + 31) >> 5;
  const int ntiles = tiles_x * g.H;
  const int n = g.n_planes;
  const int half = (a.scale + (a.scale >> 31)) >> 1;
  const uint32_t* ref = reinterpret_cast<const uint32_t*>(a.ref);
  const float* Wm = a.warp[0];
  const float w0 = Wm[0], w1 = Wm[1], w2 = Wm[2], w4 = Wm[4], w5 = Wm[5], w6 = Wm[6];
  const int iw = a.ow[0], ih = a.oh[0], x1 = iw - 2, y1 = ih - 2;
  const uint32_t* phase = a.phase[0];
  const int plane_stride = ih * iw;
  constexpr int kNoRow = INT_MIN;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += (gridDim.x * blockDim.x) >> 5) {
    const int y = t / tiles_x, xr = ((t - y * tiles_x) << 5) + lane;
    const int x = min(xr, g.W - 1);
    const size_t pi = (size_t)y * g.W + x;
    uint8_t* out = raw + pi * n;
    const bool skipped = g.skip[pi] != 0;
    const bool live = xr < g.W && !skipped;
    if (xr < g.W && skipped)
      for (int d = 0; d < n; d += 8) *reinterpret_cast<uint2*>(out + d) = make_uint2(0u, 0u);
    if (__ballot_sync(0xffffffffu, live) == 0) continue;
    const int xImg = min(a.scale * x + half, a.rw - 1), yImg = min(a.scale * y + half, a.rh - 1);
    uint32_t ge[3], go[3], re[3][3], ro[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++) {  // the reference 3x3 block, rows/columns clamped to the image
      const int yy = min(max(yImg + r - 1, 0), a.rh - 1);
      uint32_t yb[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const uint32_t w = __ldg(ref + (size_t)yy * a.rw + min(max(xImg + c - 1, 0), a.rw - 1));
        yb[c] = w & 0xffu;
        re[r][c] = w & 0x00ff00ffu;
        ro[r][c] = (w >> 8) & 0x00ff00ffu;
      }
      ge[r] = yb[0] | (yb[2] << 16);
      go[r] = yb[1];
    }
    const GreyRef gr = grey_ref(ge, go);
    const float xf = (float)xImg, yf = (float)yImg;
    int last = 0;
    uint32_t pk0 = 0, pk1 = 0;
    auto put = [&](int d, uint32_t acc) {  // Normalise (:378-379) and eight planes per store
      const uint32_t b = (uint32_t)f2i(__fmul_rn((float)(acc & 0xffffu), a.norm)) & 0xffu;
      const int sh = (d & 3) * 8;
      if (d & 4) pk1 |= b << sh;
      else pk0 |= b << sh;
      if ((d & 7) == 7) {
        if (live) *reinterpret_cast<uint2*>(out + (d - 7)) = make_uint2(pk0, pk1);
        pk0 = pk1 = 0;
      }
    };
    {  // plane 0: the general projection, clamped into the rect (:263-269)
      const float z = __ldg(g.planes);
      const float xz = __fmul_rn(xf, z), yz = __fmul_rn(yf, z);
      const float4 zk = __ldg(zt);
      const float px = __fadd_rn(__fadd_rn(zk.x, __fmul_rn(xz, w0)), __fmul_rn(yz, w4));
      const float py = __fadd_rn(__fadd_rn(zk.y, __fmul_rn(xz, w1)), __fmul_rn(yz, w5));
      const float pz = __fadd_rn(__fadd_rn(zk.z, __fmul_rn(xz, w2)), __fmul_rn(yz, w6));
      const float inv = __frcp_rn(pz);
      const float fx = cs_minf(cs_maxf(__fadd_rn(__fmul_rn(px, inv), 0.25f), 1.0f), (float)(x1 - 1));
      const float fy = cs_minf(cs_maxf(__fadd_rn(__fmul_rn(py, inv), 0.25f), 1.0f), (float)(y1 - 1));
      const int tx = f2i(__fadd_rn(fx, fx)), ty = f2i(__fadd_rn(fy, fy));
      const int ix = tx >> 1, iy = ty >> 1;
      if (ix >= 1 && ix < x1 && iy >= 1 && iy < y1) {
        if (live) {
          const size_t qi = ((size_t)(((ty & 1) << 1) | (tx & 1)) * ih + (iy - 1)) * iw + (ix - 1);
          last = GREY ? grey_cost(reinterpret_cast<const uint2*>(phase) + qi, iw, gr) : colour_cost(phase + qi, iw, re, ro, a.wq[0]);
        }
      } else if (live) {  // the scalar fallback of the reference would read out of the image
        atomicCAS(err, 0, 7);
      }
      put(0, (uint32_t)last);
    }
    for (int d0 = 0; d0 < n; d0 += 32) {
      // lane j: the target row offset of plane d0 + j (or kNoRow when the row leaves the rect)
      int rowoff;
      {
        const int dj = min(d0 + lane, n - 1);
        const float4 zj = __ldg(zt + dj);
        const float yz = __fmul_rn(yf, __ldg(g.planes + dj));
        const float fy = __fadd_rn(__fmul_rn(__fadd_rn(zj.y, __fmul_rn(yz, w5)), zj.w), 0.25f);
        const int ty = f2i(__fadd_rn(fy, fy)), iy = ty >> 1;
        rowoff = (iy >= 1 && iy < y1) ? ((((ty & 1) << 1) * ih) + iy - 1) * iw - 1 : kNoRow;
      }
      const int jend = min(32, n - d0);
      for (int j = (d0 == 0 ? 1 : 0); j < jend; j++) {
        const int d = d0 + j;
        const int ro_d = __shfl_sync(0xffffffffu, rowoff, j);
        if (ro_d != kNoRow && live) {
          const float4 zk = __ldg(zt + d);
          const float xz = __fmul_rn(xf, __ldg(g.planes + d));
          const float fx = __fadd_rn(__fmul_rn(__fadd_rn(zk.x, __fmul_rn(xz, w0)), zk.w), 0.25f);
          const int tx = f2i(__fadd_rn(fx, fx)), ix = tx >> 1;
          if (ix >= 1 && ix < x1) {
            const int qi = ro_d + (tx & 1) * plane_stride + ix;
            last = GREY ? grey_cost(reinterpret_cast<const uint2*>(phase) + qi, iw, gr) : colour_cost(phase + qi, iw, re, ro, a.wq[0]);
          }
        }
        put(d, (uint32_t)last);
      }
    }
  }
}

// One block column of the grey cost: the three capped differences of a target column triple t (vertical layout) against
// a reference column triple, in u16x2 lanes each offset by 256 (as grey_cost); three columns sum to S0 + 12·256.
struct ColRef {
  uint32_t ea, eb, oa, ob;
};
LUX_DEV ColRef col_ref(uint32_t even, uint32_t odd) { return ColRef{0x01000100u - even, 0x01000100u + even, 0x01000100u - odd, 0x01000100u + odd}; }
LUX_DEV uint32_t col_cost(uint2 t, const ColRef& c) {
  return vmin2c(vmax2c(t.x + c.ea, c.eb - t.x), 0x01020102u) + vmin2c(vmax2c(t.y + c.oa, c.ob - t.y), 0x01000102u);
}
// The same with the four adds as multiply-adds by one = 1 and neg = 0xffffffff (kernel-argument values, so they stay
// multiply-adds and issue on the FMA pipe; the ALU pipe bounds the kernel that uses this). Equal mod 2^32.
LUX_DEV uint32_t col_cost_m(uint2 t, const ColRef& c, uint32_t one, uint32_t neg) {
  return vmin2c(vmax2c(t.x * one + c.ea, t.x * neg + c.eb), 0x01020102u) +
         vmin2c(vmax2c(t.y * one + c.oa, t.y * neg + c.ob), 0x01000102u);
}

// Uniform layers of one axis-aligned grey pair at scale 1 (the plain stereo pair): the 3x3 blocks of neighbouring
// pixels overlap, and so do their target blocks wherever the target column advances by one whole pixel with the same
// half-pixel phase from one pixel to the next. A lane holds P neighbouring pixels of a row (slots 0..P-1) and a warp a
// run of 32·P - 2 pixels (slots 0 and 1 of lane 0 are the two pixels to the left of the run, computed and not stored).
// Per plane every slot computes only the right column of its block (reference column x + 1, clamped as the reference
// clamps its block, against target column ix + 1) and takes the middle and left columns from the two pixels to its left
// (the lane's own slots, or slots P-2 and P-1 of the lane to the left by shuffle) when their target positions are
// exactly 2 and 4 half-pixels to the left; a warp vote keeps the common case, where every slot that needs its block has
// it that way, free of per-slot branches. Elsewhere a slot computes the two columns itself. The terms, and so the sums,
// are the reference's (:222-246); only who computes a term changes. The plane terms, the target row and the neighbour
// exchange are shared by the lane's P pixels. Normalise (:378-379) of one camera's cost is a function of S0 (0..18), a
// 19-entry table. Two pixels a lane: 4 (79 registers) take more issue slots a DE, and staging each 32-plane group in
// shared memory (whole-sector stores) saves DRAM traffic the kernel is not bound by at the price of instructions it is.
constexpr int kAxPx = 2;                 // pixels a lane
constexpr int kAxRun = 32 * kAxPx - 2;  // pixels a warp stores

template <int P>
__global__ void __launch_bounds__(256, P > 2 ? 3 : 4)
    k_cost_axis_v(const CostArgs a, const LayerGeom g, const float4* __restrict__ zt, uint8_t* __restrict__ raw, int* err) {
  constexpr int kRun = 32 * P - 2;
  __shared__ uint8_t s_norm[32];
  if (threadIdx.x < 32)
    s_norm[threadIdx.x] =
        (uint8_t)(f2i(__fmul_rn((float)(((uint32_t)(min((int)threadIdx.x, 18) * 12240 + 16) >> 5) & 0xffffu), a.norm)) & 0xff);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int runs_x = (g.W + kRun - 1) / kRun;
  const int nruns = runs_x * g.H;
  const int n = g.n_planes;
  const uint8_t* ref8 = a.ref;
  const float* Wm = a.warp[0];
  const float w0 = Wm[0], w1 = Wm[1], w2 = Wm[2], w4 = Wm[4], w5 = Wm[5], w6 = Wm[6];
  const int iw = a.ow[0], ih = a.oh[0], x1 = iw - 2, y1 = ih - 2;
  const uint2* q = reinterpret_cast<const uint2*>(a.phase[0]);
  const int plane_stride = ih * iw;
  constexpr int kNoRow = INT_MIN;
  // (s · 0x10001) >> 16 is the sum of the two u16 lanes of a block sum s (each lane under 2^15, so nothing carries)
  const uint32_t one = a.one, neg = 0u - a.one, k10001 = 0x10001u * a.one;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nruns; t += (gridDim.x * blockDim.x) >> 5) {
    const int y = t / runs_x;
    const int x0 = (t - y * runs_x) * kRun - 2;  // x of slot 0 of lane 0
    const int xs = x0 + lane * P;                // x of this lane's slot 0
    const long long row0 = (long long)y * g.W;
    bool live[P];
    float xf[P];
    ColRef cr[P];
    const int ya = max(y - 1, 0), yb = min(y + 1, a.rh - 1);
    bool any = false;
#pragma unroll
    for (int j = 0; j < P; j++) {
      const int x = xs + j;
      const bool in_row = lane * P + j >= 2 && x < g.W;  // slots 0 and 1 of lane 0 belong to the run to the left
      const bool skipped = in_row && g.skip[row0 + x] != 0;
      live[j] = in_row && !skipped;
      any = any || live[j];
      if (skipped) {  // skipped pixels aggregate raw 0 (DenseStereoSgm.cs:242)
        uint8_t* out = raw + (row0 + x) * n;
        for (int d = 0; d < n; d += 8) *reinterpret_cast<uint2*>(out + d) = make_uint2(0u, 0u);
      }
      xf[j] = (float)min(x, a.rw - 1);  // scale 1: the reference grid is the layer grid
      // this slot's right reference column (rows y-1, y, y+1 and the column clamped like the reference's block)
      const int c = min(max(x + 1, 0), a.rw - 1);
      const uint32_t r0 = ref8[((size_t)ya * a.rw + c) * 4], r1 = ref8[((size_t)y * a.rw + c) * 4], r2 = ref8[((size_t)yb * a.rw + c) * 4];
      cr[j] = col_ref(r0 | (r2 << 16), r1);
    }
    if (__ballot_sync(0xffffffffu, any) == 0) continue;
    // slots P-2 and P-1 of the lane to the left. Slot j's left and middle block columns are entries j and j + 1 of
    // {left lane's P-2, left lane's P-1, own 0, ..., own P-1}, its right column entry j + 2.
    const ColRef lA{__shfl_up_sync(0xffffffffu, cr[P - 2].ea, 1), __shfl_up_sync(0xffffffffu, cr[P - 2].eb, 1),
                    __shfl_up_sync(0xffffffffu, cr[P - 2].oa, 1), __shfl_up_sync(0xffffffffu, cr[P - 2].ob, 1)};
    const ColRef lB{__shfl_up_sync(0xffffffffu, cr[P - 1].ea, 1), __shfl_up_sync(0xffffffffu, cr[P - 1].eb, 1),
                    __shfl_up_sync(0xffffffffu, cr[P - 1].oa, 1), __shfl_up_sync(0xffffffffu, cr[P - 1].ob, 1)};
    auto ext_ref = [&](int e) -> const ColRef& { return e == 0 ? lA : e == 1 ? lB : cr[e - 2]; };
    uint32_t last[P];  // the normalised cost of the last plane computed, per slot (:273-274)
    {  // plane 0: the general projection, clamped into the rect (:263-269)
      const float z = __ldg(g.planes);
      const float4 zk = __ldg(zt);
      const float yz = __fmul_rn((float)y, z);
#pragma unroll
      for (int j = 0; j < P; j++) {
        last[j] = 0;
        const float xz = __fmul_rn(xf[j], z);
        const float px = __fadd_rn(__fadd_rn(zk.x, __fmul_rn(xz, w0)), __fmul_rn(yz, w4));
        const float py = __fadd_rn(__fadd_rn(zk.y, __fmul_rn(xz, w1)), __fmul_rn(yz, w5));
        const float pz = __fadd_rn(__fadd_rn(zk.z, __fmul_rn(xz, w2)), __fmul_rn(yz, w6));
        const float inv = __frcp_rn(pz);
        const float fx = cs_minf(cs_maxf(__fadd_rn(__fmul_rn(px, inv), 0.25f), 1.0f), (float)(x1 - 1));
        const float fy = cs_minf(cs_maxf(__fadd_rn(__fmul_rn(py, inv), 0.25f), 1.0f), (float)(y1 - 1));
        const int tx = f2i(__fadd_rn(fx, fx)), ty = f2i(__fadd_rn(fy, fy));
        const int ix = tx >> 1, iy = ty >> 1;
        if (ix >= 1 && ix < x1 && iy >= 1 && iy < y1) {
          if (live[j]) {
            const size_t base = ((size_t)(((ty & 1) << 1) | (tx & 1)) * ih + (iy - 1)) * iw + (ix - 1);
            const uint32_t s = col_cost(__ldg(q + base), ext_ref(j)) + col_cost(__ldg(q + base + 1), ext_ref(j + 1)) +
                               col_cost(__ldg(q + base + 2), cr[j]);
            last[j] = s_norm[(s & 0xffffu) + (s >> 16) - 12 * 256];
          }
        } else if (live[j]) {  // the scalar fallback of the reference would read out of the image
          atomicCAS(err, 0, 7);
        }
      }
    }
    const float yf = (float)y;
    auto row_offset = [&](int d) {  // lane j: the offset of row iy - 1 of phase 2·hy of plane d + j (kNoRow: off the rect)
      const int dj = min(d + lane, n - 1);
      const float4 zj = __ldg(zt + dj);
      const float yz = __fmul_rn(yf, __ldg(g.planes + dj));
      const float fy = __fadd_rn(__fmul_rn(__fadd_rn(zj.y, __fmul_rn(yz, w5)), zj.w), 0.25f);
      const int ty = f2i(__fadd_rn(fy, fy)), iy = ty >> 1;
      return (iy >= 1 && iy < y1) ? (((ty & 1) << 1) * ih + iy - 1) * iw : kNoRow;
    };
    int rowoff = row_offset(0);
    // eight planes of u8 costs a slot as one 64-bit value {lo, hi}, plane d at byte d % 8: each plane shifts it right by
    // one byte and enters at the top
    uint32_t lo[P], hi[P];
#pragma unroll
    for (int j = 0; j < P; j++) {
      lo[j] = 0;
      hi[j] = last[j] << 24;
    }
    for (int d = 1; d < n; d++) {
      if ((d & 31) == 0) rowoff = row_offset(d);
      const int ro_d = __shfl_sync(0xffffffffu, rowoff, d & 31);
      if (ro_d != kNoRow) {  // the same for the whole warp
        const float4 zk = __ldg(zt + d);
        const float z = __ldg(g.planes + d);
        int tx[P], ix[P], rb[P];
        uint32_t c[P];
        bool inr[P];
#pragma unroll
        for (int j = 0; j < P; j++) {
          const float xz = __fmul_rn(xf[j], z);
          const float fx = __fadd_rn(__fmul_rn(__fadd_rn(zk.x, __fmul_rn(xz, w0)), zk.w), 0.25f);
          tx[j] = f2i(__fadd_rn(fx, fx));
          ix[j] = tx[j] >> 1;
          inr[j] = ix[j] >= 1 && ix[j] < x1;
          rb[j] = ro_d + (tx[j] & 1) * plane_stride;  // row iy - 1 of the slot's phase
          // column ix + 1, clamped only to stay in the image: a column a neighbour takes (ix + 1 of a slot whose right
          // neighbour is in the rect one pixel on) lies in [0, iw - 3] already, so a negative ix + 1 may map to iw - 1
          c[j] = col_cost_m(__ldg(q + rb[j] + min((uint32_t)(ix[j] + 1), (uint32_t)(iw - 1))), cr[j], one, neg);
        }
        // slots P-2 and P-1 of the lane to the left; slot P-1's target is sent as kNoRow unless slot P-2's is one pixel
        // left of it, so that one comparison checks both neighbours of slot 0. A neighbour pair found unequal (by this
        // or by the wrapping compares below) only sends a slot to its own columns, which is always exact.
        const int tl = (uint32_t)tx[P - 1] - (uint32_t)tx[P - 2] == 2u ? tx[P - 1] : kNoRow;
        const uint32_t cA = __shfl_up_sync(0xffffffffu, c[P - 2], 1), cB = __shfl_up_sync(0xffffffffu, c[P - 1], 1);
        const int tB = __shfl_up_sync(0xffffffffu, tl, 1);
        bool fast[P];
        bool pair[P];  // pair[j]: slot j's target is one pixel right of slot j-1's (j >= 1)
#pragma unroll
        for (int j = 1; j < P; j++) pair[j] = (uint32_t)tx[j] - (uint32_t)tx[j - 1] == 2u;
        fast[0] = (uint32_t)tx[0] - (uint32_t)tB == 2u;
#pragma unroll
        for (int j = 1; j < P; j++) fast[j] = pair[j] && (j == 1 ? fast[0] : pair[j - 1]);
        bool ok = true;  // every slot that needs its block has it from its neighbours
#pragma unroll
        for (int j = 0; j < P; j++) ok = ok && (fast[j] || !(live[j] && inr[j]));
        auto ext_c = [&](int e) { return e == 0 ? cA : e == 1 ? cB : c[e - 2]; };
        if (__all_sync(0xffffffffu, ok)) {
#pragma unroll
          for (int j = 0; j < P; j++) {
            const uint32_t sum = ext_c(j) + ext_c(j + 1) + c[j];
            if (inr[j]) last[j] = s_norm[((sum * k10001) >> 16) - 12 * 256];
          }
        } else {
#pragma unroll
          for (int j = 0; j < P; j++) {
            if (inr[j]) {
              uint32_t sum;
              if (fast[j]) sum = ext_c(j) + ext_c(j + 1) + c[j];
              else sum = col_cost(__ldg(q + rb[j] + ix[j] - 1), ext_ref(j)) + col_cost(__ldg(q + rb[j] + ix[j]), ext_ref(j + 1)) + c[j];
              last[j] = s_norm[(sum & 0xffffu) + (sum >> 16) - 12 * 256];
            }
          }
        }
      }
#pragma unroll
      for (int j = 0; j < P; j++) {
        lo[j] = __funnelshift_r(lo[j], hi[j], 8);
        hi[j] = __funnelshift_r(hi[j], last[j], 8);
      }
      if ((d & 7) == 7) {
        const int d0 = d - 7;
#pragma unroll
        for (int j = 0; j < P; j++)
          if (live[j]) *reinterpret_cast<uint2*>(raw + (row0 + xs + j) * n + d0) = make_uint2(lo[j], hi[j]);
      }
    }
  }
}

bool cost_all_grey(const CostArgs& a) {
  for (int k = 0; k < a.n_others; k++)
    if (!(a.wq[k][0] == 12240 && a.wq[k][1] == 0 && a.wq[k][2] == 0 && a.wq[k][3] == 0)) return false;
  return true;
}

void launch_phases(const CostArgs& a, cudaStream_t s) {
  const bool grey = cost_all_grey(a);
  for (int k = 0; k < a.n_others; k++) {
    dim3 grid((a.ow[k] + 127) / 128, a.oh[k]);
    uint32_t* out = const_cast<uint32_t*>(a.phase[k]);
    if (a.vcols) k_phase_grey_v<<<grid, 128, 0, s>>>(a.other[k], a.ow[k], a.oh[k], reinterpret_cast<uint2*>(out));
    else if (grey) k_phase_grey<<<grid, 128, 0, s>>>(a.other[k], a.ow[k], a.oh[k], reinterpret_cast<uint2*>(out));
    else k_phase_colour<<<grid, 128, 0, s>>>(a.other[k], a.ow[k], a.oh[k], out);
    count_launches(1);
  }
}

template <bool GREY>
static void launch_rows(int nk, int blocks, const CostArgs& a, const LayerGeom& g, const float4* zt, uint8_t* raw, int* err,
                        cudaStream_t s) {
  switch (nk) {
    case 1: k_cost_rows<GREY, 1><<<blocks, 256, 0, s>>>(a, g, zt, raw, err); break;
    case 2: k_cost_rows<GREY, 2><<<blocks, 256, 0, s>>>(a, g, zt, raw, err); break;
    case 3: k_cost_rows<GREY, 3><<<blocks, 256, 0, s>>>(a, g, zt, raw, err); break;
    case 4: k_cost_rows<GREY, 4><<<blocks, 256, 0, s>>>(a, g, zt, raw, err); break;
    default: k_cost_rows<GREY, kMaxCams - 1><<<blocks, 256, 0, s>>>(a, g, zt, raw, err); break;
  }
}

// The row kernels give a warp 32 pixels of a row and walk the planes in each lane: a small layer with many planes (the
// L16 pyramid's first layer: 65x49 pixels, 552 planes, 147 row tiles) leaves most SMs idle for a long walk, so it takes
// the warp-per-pixel kernel, lanes over planes (same bits), with the horizontal phase images that kernel reads.
bool cost_small_wide_layer(int W, int H, int n_planes) { return ((W + 31) / 32) * H < 148 * 4 && n_planes > 256; }

int launch_cost(const CostArgs& a, const LayerGeom& g, const float4* zt, uint8_t* raw, int* err, cudaStream_t s) {
  const int npx = g.W * g.H;
  const bool grey = cost_all_grey(a);
  int kind = 0;
  if (g.uniform && !cost_small_wide_layer(g.W, g.H, g.n_planes) && g.n_planes % 8 == 0 && a.n_others >= 1 &&
      a.n_others <= kMaxCams - 1) {
    const int tiles = ((g.W + 31) / 32) * g.H;
    int blocks = (tiles + 7) / 8;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (a.vcols) {
      const int vruns = ((g.W + kAxRun - 1) / kAxRun) * g.H;
      int vb = (vruns + 7) / 8;
      if (vb > 148 * 16) vb = 148 * 16;
      k_cost_axis_v<kAxPx><<<vb, 256, 0, s>>>(a, g, zt, raw, err);
      kind = 3;
    } else if (a.axis) {
      if (grey) k_cost_axis<true><<<blocks, 256, 0, s>>>(a, g, zt, raw, err);
      else k_cost_axis<false><<<blocks, 256, 0, s>>>(a, g, zt, raw, err);
      kind = 2;
    } else {
      if (grey) launch_rows<true>(a.n_others, blocks, a, g, zt, raw, err, s);
      else launch_rows<false>(a.n_others, blocks, a, g, zt, raw, err, s);
      kind = 1;
    }
  } else {
    int blocks = (npx + 7) / 8;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (grey) k_cost<true><<<blocks, 256, 0, s>>>(a, g, zt, raw, err);
    else k_cost<false><<<blocks, 256, 0, s>>>(a, g, zt, raw, err);
  }
  count_launches(1);
  return kind;
}

}  // namespace lux
