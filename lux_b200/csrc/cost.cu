// Plane-sweep matching cost -> u8 raw volume: DenseStereo.MatchingCost + Normalise (DenseStereo.cs:217-292, 376-381).
//
// One warp per reference pixel, lanes over planes. Per other camera and plane: the projection through the flow matrix
// (no FMA, IEEE 1/pz), the half-pixel `pavgb` resampling of a 4x4 target block, per-channel capped |diff| of the 3x3
// blocks packed four bytes to a word, the fixed-point channel weights, and a u16 wrap-sum over cameras. A plane whose
// position repeats or leaves the valid rect reuses the last computed cost (:273-274): the warp finds that plane with a
// ballot, and carries it across chunks of 32 planes.
#include "common.cuh"
#include "internal.h"

namespace lux {

constexpr uint32_t kCapsPacked = 0x00060602u;  // CostContext.Caps {2, 6, 6, 0} (DenseStereo.cs:187), one byte per channel

// The capped SAD of one target position (DenseStereo.cs:276-287): rows averaged first (hy), then pixels (hx).
LUX_DEV int block_cost(const uint32_t* __restrict__ img, int iw, int ix, int iy, int hx, int hy, const uint32_t (&rb)[3][3],
                       const uint16_t (&wq)[4]) {
  const uint32_t* base = img + (size_t)(iy - 1) * iw + (ix - 1);
  uint32_t row[3][4];
#pragma unroll
  for (int q = 0; q < 3; q++) {
#pragma unroll
    for (int p = 0; p < 4; p++) {
      if (p == 3 && !hx) { row[q][p] = 0; continue; }
      uint32_t a = __ldg(base + (size_t)q * iw + p);
      if (hy) a = __vavgu4(a, __ldg(base + (size_t)(q + 1) * iw + p));  // pavgb with the next row
      row[q][p] = a;
    }
  }
  uint32_t s = 0;
#pragma unroll
  for (int q = 0; q < 3; q++)
#pragma unroll
    for (int p = 0; p < 3; p++) {
      uint32_t v = hx ? __vavgu4(row[q][p], row[q][p + 1]) : row[q][p];  // pavgb with the next pixel
      s += __vminu4(__vabsdiffu4(v, rb[q][p]), kCapsPacked);           // byte lanes stay below 256: 9 x 6
    }
  int S0 = s & 0xff, S1 = (s >> 8) & 0xff, S2 = (s >> 16) & 0xff, S3 = s >> 24;
  int cY = (S0 * wq[0] + 16) >> 5, cU = (S1 * wq[1] + 16) >> 5, cV = (S2 * wq[2] + 16) >> 5, cA = (S3 * wq[3] + 16) >> 5;
  int ck = (cY + cU) + (cV + cA);
  return f2i(fminf((float)ck, 65535.0f));  // ck is finite and non-negative: MathF.Min semantics do not matter here
}

__global__ void __launch_bounds__(256) k_cost(const CostArgs a, const LayerGeom g, uint8_t* __restrict__ raw, int* err) {
  __shared__ int s_carry[8][kMaxCams];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int npx = g.W * g.H;
  const int half = (a.scale + (a.scale >> 31)) >> 1;
  const uint32_t* ref = reinterpret_cast<const uint32_t*>(a.ref);
  for (int pi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; pi < npx; pi += nwarps) {
    if (g.skip[pi]) continue;
    const int x = pi % g.W, y = pi / g.W;
    const int xImg = min(a.scale * x + half, a.rw - 1), yImg = min(a.scale * y + half, a.rh - 1);
    const int start = g.start[pi], count = g.count[pi], cap = g.cap[pi];
    uint8_t* out = raw + g.off[pi];
    if (start + count > g.n_planes) {  // MatchingCostScalar would index Planes past its end
      if (lane == 0) atomicCAS(err, 0, 7);
      continue;
    }
    uint32_t rb[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
      int yy = min(max(yImg + r - 1, 0), a.rh - 1);
#pragma unroll
      for (int c = 0; c < 3; c++) rb[r][c] = __ldg(ref + (size_t)yy * a.rw + min(max(xImg + c - 1, 0), a.rw - 1));
    }
    const float xf = (float)xImg, yf = (float)yImg;
    for (int c0 = 0; c0 < count; c0 += 32) {
      const int d = c0 + lane;
      const bool valid = d < count;
      const float z = valid ? __ldg(g.planes + start + d) : 1.0f;
      const int last = min(31, count - 1 - c0);
      uint32_t acc = 0;
      for (int k = 0; k < a.n_others; k++) {
        const float* Wm = a.warp[k];
        const int iw = a.ow[k], ih = a.oh[k];
        const int x0 = 1, y0 = 1, x1 = iw - 2, y1 = ih - 2;
        // p = ((z·W2 + W3) + xz·W0) + yz·W1 (:255-259), then 1/pz and the +0.25 bias (:260-261)
        float xz = __fmul_rn(__fmul_rn(xf, z), 1.0f), yz = __fmul_rn(__fmul_rn(yf, z), 1.0f);
        float px = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(z, Wm[8]), Wm[12]), __fmul_rn(xz, Wm[0])), __fmul_rn(yz, Wm[4]));
        float py = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(z, Wm[9]), Wm[13]), __fmul_rn(xz, Wm[1])), __fmul_rn(yz, Wm[5]));
        float pz = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(z, Wm[10]), Wm[14]), __fmul_rn(xz, Wm[2])), __fmul_rn(yz, Wm[6]));
        float inv = __fdiv_rn(1.0f, pz);
        float fx = __fadd_rn(__fmul_rn(px, inv), 0.25f), fy = __fadd_rn(__fmul_rn(py, inv), 0.25f);
        int ix, iy, hx, hy;
        bool inb;
        if (d == 0) {  // the first plane is clamped into the rect (:263-269)
          float cx = cs_minf(cs_maxf(fx, (float)x0), (float)(x1 - 1)), cy = cs_minf(cs_maxf(fy, (float)y0), (float)(y1 - 1));
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
        int costK = inb ? block_cost(reinterpret_cast<const uint32_t*>(a.other[k]), iw, ix, iy, hx, hy, rb, a.wq[k]) : 0;
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

void launch_cost(const CostArgs& a, const LayerGeom& g, uint8_t* raw, int* err, cudaStream_t s) {
  int npx = g.W * g.H;
  int blocks = (npx + 7) / 8;
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_cost<<<blocks, 256, 0, s>>>(a, g, raw, err);
  count_launches(1);
}

}  // namespace lux
