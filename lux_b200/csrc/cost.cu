// Plane-sweep matching cost -> u8 raw volume: DenseStereo.MatchingCost + Normalise (DenseStereo.cs:217-292, 376-381).
//
// One warp per reference pixel, lanes over planes. Per other camera and plane: the projection through the flow matrix
// (no FMA, IEEE 1/pz; the plane-only terms z·W2 + W3 come from a per-layer table), the half-pixel `pavgb` resampling
// of a 4x4 target block, capped |diff| of the 3x3 blocks, the fixed-point channel weights, and a u16 wrap-sum over
// cameras. A plane whose position repeats or leaves the valid rect reuses the last computed cost (:273-274): the warp
// finds that plane with a ballot and carries it across chunks of 32 planes.
//
// Byte arithmetic: a grey camera (weights {12240, 0, 0, 0}) only ever contributes its Y channel, so its block cost is
// nine scalar byte differences. A colour camera splits each RGBA word into two u16x2 lanes (Y|V and U|A) and uses
// min/max.u16x2 for |a-b| and the caps. Both are exact restatements of the byte-lane sums of the reference (each
// channel sum is at most 9·6, so nothing carries between lanes).
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
LUX_DEV int yb(uint32_t w) { return (int)(w & 0xffu); }
LUX_DEV int avg_u8(int a, int b) { return (a + b + 1) >> 1; }  // pavgb on one byte
// pavgb on the u16x2 lanes of byte values
LUX_DEV uint32_t avg_u16x2(uint32_t a, uint32_t b) { return ((a + b + 0x00010001u) >> 1) & 0x00ff00ffu; }

// Grey camera: S0 = Σ min(|t - r|, 2) over the 3x3 block of Y values (rows averaged first, then pixels).
template <int HX, int HY>
LUX_DEV int grey_block(const uint32_t* __restrict__ base, int iw, const int (&ry)[3][3]) {
  int s = 0;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    int row[4];
#pragma unroll
    for (int p = 0; p < 3 + HX; p++) {
      int v = yb(__ldg(base + (size_t)q * iw + p));
      if (HY) v = avg_u8(v, yb(__ldg(base + (size_t)(q + 1) * iw + p)));
      row[p] = v;
    }
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const int v = HX ? avg_u8(row[p], row[p + 1]) : row[p];
      s += min(abs(v - ry[q][p]), 2);
    }
  }
  return (s * 12240 + 16) >> 5;
}

// Colour camera: even bytes (Y, V) and odd bytes (U, A) as u16 pairs.
template <int HX, int HY>
LUX_DEV int colour_block(const uint32_t* __restrict__ base, int iw, const uint32_t (&re)[3][3], const uint32_t (&ro)[3][3],
                         const uint16_t (&wq)[4]) {
  const uint32_t capE = 0x00060002u, capO = 0x00000006u;  // {Y:2, V:6} and {U:6, A:0}
  uint32_t se = 0, so = 0;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    uint32_t e[4], o[4];
#pragma unroll
    for (int p = 0; p < 3 + HX; p++) {
      uint32_t w = __ldg(base + (size_t)q * iw + p);
      uint32_t ev = w & 0x00ff00ffu, od = (w >> 8) & 0x00ff00ffu;
      if (HY) {
        uint32_t w2 = __ldg(base + (size_t)(q + 1) * iw + p);
        ev = avg_u16x2(ev, w2 & 0x00ff00ffu);
        od = avg_u16x2(od, (w2 >> 8) & 0x00ff00ffu);
      }
      e[p] = ev;
      o[p] = od;
    }
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const uint32_t ve = HX ? avg_u16x2(e[p], e[p + 1]) : e[p];
      const uint32_t vo = HX ? avg_u16x2(o[p], o[p + 1]) : o[p];
      se += vmin2c(vmax2c(ve, re[q][p]) - vmin2c(ve, re[q][p]), capE);
      so += vmin2c(vmax2c(vo, ro[q][p]) - vmin2c(vo, ro[q][p]), capO);
    }
  }
  const int S0 = se & 0xffff, S2 = se >> 16, S1 = so & 0xffff, S3 = so >> 16;
  const int cY = (S0 * wq[0] + 16) >> 5, cU = (S1 * wq[1] + 16) >> 5, cV = (S2 * wq[2] + 16) >> 5, cA = (S3 * wq[3] + 16) >> 5;
  return (cY + cU) + (cV + cA);  // at most 6885: MathF.Min(…, 65535) and the float round trip change nothing
}

template <bool GREY>
__global__ void __launch_bounds__(256) k_cost(const CostArgs a, const LayerGeom g, const float* __restrict__ zt, uint8_t* __restrict__ raw,
                                              int* err) {
  __shared__ int s_carry[8][kMaxCams];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int npx = g.W * g.H;
  const int n = g.n_planes;
  const int half = (a.scale + (a.scale >> 31)) >> 1;
  const uint32_t* ref = reinterpret_cast<const uint32_t*>(a.ref);
  for (int pi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; pi < npx; pi += nwarps) {
    if (g.skip[pi]) continue;
    const int x = pi % g.W, y = pi / g.W;
    const int xImg = min(a.scale * x + half, a.rw - 1), yImg = min(a.scale * y + half, a.rh - 1);
    const int start = g.start[pi], count = g.count[pi], cap = g.cap[pi];
    uint8_t* out = raw + g.off[pi];
    if (start + count > n) {  // MatchingCostScalar would index Planes past its end
      if (lane == 0) atomicCAS(err, 0, 7);
      continue;
    }
    int ry[3][3];
    uint32_t re[3][3], ro[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++) {  // the reference 3x3 block, rows/columns clamped to the image
      const int yy = min(max(yImg + r - 1, 0), a.rh - 1);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const uint32_t w = __ldg(ref + (size_t)yy * a.rw + min(max(xImg + c - 1, 0), a.rw - 1));
        ry[r][c] = yb(w);
        re[r][c] = w & 0x00ff00ffu;
        ro[r][c] = (w >> 8) & 0x00ff00ffu;
      }
    }
    const float xf = (float)xImg, yf = (float)yImg;
    for (int c0 = 0; c0 < count; c0 += 32) {
      const int d = c0 + lane;
      const bool valid = d < count;
      const int pl = valid ? start + d : start;
      const float z = __ldg(g.planes + pl);
      const int last = min(31, count - 1 - c0);
      uint32_t acc = 0;
      for (int k = 0; k < a.n_others; k++) {
        const float* Wm = a.warp[k];
        const int iw = a.ow[k], ih = a.oh[k];
        const int x0 = 1, y0 = 1, x1 = iw - 2, y1 = ih - 2;
        // p = ((z·W2 + W3) + xz·W0) + yz·W1 (:255-259), the first term from the table; then 1/pz and the +0.25 bias
        const float* zk = zt + ((size_t)k * n + pl) * 3;
        const float xz = __fmul_rn(xf, z), yz = __fmul_rn(yf, z);  // (x·z)·1.0f: the product by one is exact
        const float px = __fadd_rn(__fadd_rn(__ldg(zk + 0), __fmul_rn(xz, Wm[0])), __fmul_rn(yz, Wm[4]));
        const float py = __fadd_rn(__fadd_rn(__ldg(zk + 1), __fmul_rn(xz, Wm[1])), __fmul_rn(yz, Wm[5]));
        const float pz = __fadd_rn(__fadd_rn(__ldg(zk + 2), __fmul_rn(xz, Wm[2])), __fmul_rn(yz, Wm[6]));
        const float inv = __fdiv_rn(1.0f, pz);
        const float fx = __fadd_rn(__fmul_rn(px, inv), 0.25f), fy = __fadd_rn(__fmul_rn(py, inv), 0.25f);
        int ix, iy, hx, hy;
        bool inb;
        if (d == 0) {  // the first plane is clamped into the rect (:263-269)
          const float cx = cs_minf(cs_maxf(fx, (float)x0), (float)(x1 - 1)), cy = cs_minf(cs_maxf(fy, (float)y0), (float)(y1 - 1));
          ix = f2i(cx); iy = f2i(cy); hx = f2i(__fadd_rn(cx, cx)) & 1; hy = f2i(__fadd_rn(cy, cy)) & 1;
          inb = true;
          if (ix < x0 || ix >= x1 || iy < y0 || iy >= y1) {  // the scalar fallback of the reference would read out of the image
            atomicCAS(err, 0, 7);
            inb = false;
          }
        } else {
          ix = f2i(fx); iy = f2i(fy); hx = f2i(__fadd_rn(fx, fx)) & 1; hy = f2i(__fadd_rn(fy, fy)) & 1;
          inb = valid && !(ix < x0 || ix >= x1 || iy < y0 || iy >= y1);
        }
        int costK = 0;
        if (inb) {
          const uint32_t* base = reinterpret_cast<const uint32_t*>(a.other[k]) + (size_t)(iy - 1) * iw + (ix - 1);
          if (GREY) {
            costK = hx ? (hy ? grey_block<1, 1>(base, iw, ry) : grey_block<1, 0>(base, iw, ry))
                       : (hy ? grey_block<0, 1>(base, iw, ry) : grey_block<0, 0>(base, iw, ry));
          } else {
            costK = hx ? (hy ? colour_block<1, 1>(base, iw, re, ro, a.wq[k]) : colour_block<1, 0>(base, iw, re, ro, a.wq[k]))
                       : (hy ? colour_block<0, 1>(base, iw, re, ro, a.wq[k]) : colour_block<0, 0>(base, iw, re, ro, a.wq[k]));
          }
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

void launch_cost(const CostArgs& a, const LayerGeom& g, const float* zt, uint8_t* raw, int* err, cudaStream_t s) {
  const int npx = g.W * g.H;
  int blocks = (npx + 7) / 8;
  if (blocks > 148 * 64) blocks = 148 * 64;
  bool grey = true;
  for (int k = 0; k < a.n_others; k++)
    if (!(a.wq[k][0] == 12240 && a.wq[k][1] == 0 && a.wq[k][2] == 0 && a.wq[k][3] == 0)) grey = false;
  if (grey) k_cost<true><<<blocks, 256, 0, s>>>(a, g, zt, raw, err);
  else k_cost<false><<<blocks, 256, 0, s>>>(a, g, zt, raw, err);
  count_launches(1);
}

}  // namespace lux
