// Stereo-image formation after the ISP (Lux.Engine/Pipeline/Registration/StereoImage.cs, StereoImageBuilder.cs) and the
// 8-bit warp of the reference guide (ReferenceGuide.cs:100-162): a 6x6-tap Lanczos-3 resample (64 phases) of a source
// image through an aligned calibration (a homography, then the lens CRA factor from a 4096-entry table indexed by the
// radius), followed for the stereo images by ConvertToYUV (luma basis over the neutral, gamma 1/2.2 by log2/exp2
// polynomials) and the 8-bit store. Every float step keeps the reference's operation and rounding order; division is
// the correctly rounded reciprocal (__frcp_rn, equal to 1.0f / x); rsqrtss is the reference's table model.
//
// One thread per destination pixel, 16x16 blocks so the 6x6 source windows of a block overlap in L1. The tap table sits
// in shared memory (its rows are indexed by each thread's own phase). The four channels of a pixel go through the tap
// sums as two pairs on Blackwell's packed f32x2 instructions: two correctly rounded single-precision operations per
// instruction, the same bits as the scalar ones, and half the issue slots of the 6x6x4 taps.
#include "../../include/lux_sgm.h"
#include "common.cuh"
#include "internal.h"

namespace lux {

namespace {

// IntelApprox.RsqrtBits (Lux.Engine/Imaging/IntelApprox.cs:32-45): rsqrtss on the tables for even and odd exponents.
LUX_DEV uint32_t rsqrt_bits(uint32_t b, const uint32_t* __restrict__ t127, const uint32_t* __restrict__ t128) {
  const uint32_t sign = b & 0x80000000u, e = (b >> 23) & 0xff, m = b & 0x7fffff;
  if (e == 0xff && m != 0) return b | 0x400000u;
  if (e == 0) return sign | 0x7f800000u;
  if (sign != 0) return 0xffc00000u;
  if (e == 0xff) return 0;
  const int k = (int)e - 127;
  const uint32_t r = (k & 1) == 0 ? __ldg(t127 + (m >> 11)) : __ldg(t128 + (m >> 11));
  const int re = (int)((r >> 23) & 0xff) - ((k & 1) == 0 ? k / 2 : (k - 1) / 2);
  if (re <= 0) return 0;
  return ((uint32_t)re << 23) | (r & 0x7fffff);
}

// The destination pixel (x, y) mapped to 64ths of a source pixel (StereoImage.cs:260-272, ReferenceGuide.cs:122-130).
// False where the reference would index the lut below 0 (a subnormal r2 gives r = -inf).
LUX_DEV bool warp_map(const WarpGeom& g, const uint32_t* rsq, int x, int y, int& px, int& py) {
  const float fx = (float)x, fy = (float)y;
  const float xn = __fadd_rn(g.h[2], __fadd_rn(__fmul_rn(g.h[0], fx), __fmul_rn(g.h[1], fy)));
  const float yn = __fadd_rn(g.h[5], __fadd_rn(__fmul_rn(g.h[3], fx), __fmul_rn(g.h[4], fy)));
  const float den = __fadd_rn(__fadd_rn(__fmul_rn(g.h[7], fy), __fmul_rn(g.h[6], fx)), g.h[8]);
  const float w = __frcp_rn(den);
  const float dx = __fsub_rn(__fmul_rn(w, xn), g.cx), dy = __fsub_rn(__fmul_rn(w, yn), g.cy);
  const float a = __fmul_rn(g.sy, dy), b = __fmul_rn(g.sx, dx);
  const float r2 = __fadd_rn(__fmul_rn(a, a), __fmul_rn(b, b));
  float r = 0.0f;
  if (r2 != 0.0f) {
    const float rs = __uint_as_float(rsqrt_bits(__float_as_uint(r2), rsq, rsq + 4096));
    const float S = __fmul_rn(r2, rs);
    r = __fmul_rn(__fadd_rn(__fmul_rn(S, rs), -3.0f), __fmul_rn(S, -0.5f));
  }
  int idx = f2i(r);
  if (idx >= 0x1000) idx = 0xfff;
  if (idx < 0) return false;
  const float lu = __ldg(g.lut + idx);
  px = f2i(__fmul_rn(__fadd_rn(__fadd_rn(g.cx, -2.0f), __fmul_rn(lu, dx)), 64.0f));
  py = f2i(__fmul_rn(__fadd_rn(__fadd_rn(g.cy, -2.0f), __fmul_rn(dy, lu)), 64.0f));
  return true;
}

// Two floats in one 64-bit register pair, and the packed f32x2 product and sum (sm_100a), each element rounded to nearest
// as __fmul_rn / __fadd_rn. The assembler fuses a packed multiply whose result feeds a packed add into one fused
// multiply-add (a single rounding) even with the rounding mode spelled out, so the product is made as fma(a, b, z) with
// z = -0.0 from a kernel argument: a·b + (-0) is a·b for every input, and a value the assembler cannot see is never
// folded away, so nothing is fused.
struct F2 {
  unsigned long long v;
};
LUX_DEV F2 f2(float a, float b) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
  return r;
}
LUX_DEV float2 unf2(F2 x) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(x.v));
  return r;
}
LUX_DEV F2 mul2(F2 a, F2 b, F2 z) {
  F2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(z.v));
  return d;
}
LUX_DEV F2 add2(F2 a, F2 b) {
  F2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
  return d;
}
struct Px {  // an RGBA pixel as the pairs (R, G) and (B, A)
  F2 lo, hi;
};
LUX_DEV Px px_mul(Px p, F2 s, F2 z) { return Px{mul2(p.lo, s, z), mul2(p.hi, s, z)}; }
LUX_DEV Px px_add(Px a, Px b) { return Px{add2(a.lo, b.lo), add2(a.hi, b.hi)}; }
LUX_DEV Px px_of(float4 v) { return Px{f2(v.x, v.y), f2(v.z, v.w)}; }
LUX_DEV float4 px_f4(Px p) {
  const float2 a = unf2(p.lo), b = unf2(p.hi);
  return make_float4(a.x, a.y, b.x, b.y);
}

// (c5·t5 + c4·t4) + ((c3·t3 + c2·t2) + (c1·t1 + c0·t0)): the pairing of both tap sums of the float warp and of the row
// combination of the 8-bit warp. t holds each tap twice (the pair (t, t)).
LUX_DEV Px tap6(const Px (&c)[6], const F2* t, F2 z) {
  return px_add(px_add(px_mul(c[5], t[5], z), px_mul(c[4], t[4], z)),
                px_add(px_add(px_mul(c[3], t[3], z), px_mul(c[2], t[2], z)), px_add(px_mul(c[1], t[1], z), px_mul(c[0], t[0], z))));
}

// StereoImage.GammaEncode (StereoImage.cs:162-178): 255·sign·|m|^(1/2.2) by the log2 and exp2 polynomials.
LUX_DEV float gamma_encode(float m) {
  const int bits = __float_as_int(m), a = bits & 0x7fffffff;
  const float f = __uint_as_float(((uint32_t)a & 0x007fffffu) | 0x3f800000u);
  const float e = (float)((int)((uint32_t)a + 0xc0800000u) >> 23);
  const float lg = __fadd_rn(
      __fmul_rn(__fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(f, __uint_as_float(0x3e511af3u)), __uint_as_float(0xbfa05375u)), f),
                          __uint_as_float(0x40552f75u)),
                f),
      __fadd_rn(e, __uint_as_float(0xc0121769u)));
  float l = __fmul_rn(lg, __uint_as_float(0x3ee8ba2eu));
  l = fminf(fmaxf(l, -126.0f), 128.0f);  // l is finite for every input
  const int i = f2i(l) + (__float_as_int(l) >> 31);
  const float fr = __fsub_rn(l, (float)i);
  const float p2 = __fadd_rn(
      __fmul_rn(__fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(fr, __uint_as_float(0x3d9fcb52u)), __uint_as_float(0x3e677e26u)), fr),
                          __uint_as_float(0x3f322226u)),
                fr),
      __uint_as_float(0x3f7ffb19u));
  const float pw = __uint_as_float(((uint32_t)i << 23) + __float_as_uint(p2));
  const float sgn = a == 0 ? 0.0f : __uint_as_float(((uint32_t)bits & 0x80000000u) | 0x3f800000u);
  return __fmul_rn(pw, __fmul_rn(sgn, 255.0f));
}

// cvtps2dq (round to nearest even; NaN and values outside int32 give 0x80000000), packssdw, packuswb.
LUX_DEV uint32_t store_u8(float v) {
  if (!(v >= -2147483648.0f && v < 2147483648.0f)) return 0;
  const int iv = __float2int_rn(v);
  return (uint32_t)(iv < 0 ? 0 : iv > 255 ? 255 : iv);
}
LUX_DEV uint32_t pack_u8(float4 v) { return store_u8(v.x) | store_u8(v.y) << 8 | store_u8(v.z) << 16 | store_u8(v.w) << 24; }

// The tap table in shared memory with every tap doubled into a pair.
LUX_DEV void load_taps(F2* tab, const float* __restrict__ g) {
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  for (int i = t; i < 384; i += blockDim.x * blockDim.y) {
    const float v = __ldg(g + i);
    tab[i] = f2(v, v);
  }
  __syncthreads();
}

// MODE 0: the warped float image (StereoImage.Warp). MODE 1: the stereo image (StereoImageBuilder.Create after the ISP):
// ConvertToYUV and the 8-bit store of the warped pixel, and its YUV floats when yuv is not null.
template <int MODE>
__global__ void __launch_bounds__(256, 4) k_warp_f32(const float4* __restrict__ src, int sw, int sh, float gain, const WarpGeom g,
                                                  const float* __restrict__ taps, const uint32_t* __restrict__ rsq, int dw, int dh,
                                                  YuvRows m, float4* __restrict__ out_f, uint32_t* __restrict__ out_u8, int* err) {
  __shared__ F2 tab[384];
  load_taps(tab, taps);
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dw || y >= dh) return;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  const F2 g2 = f2(gain, gain), z = f2(g.neg_zero, g.neg_zero);
  int px, py;
  if (!warp_map(g, rsq, x, y, px, py)) {
    atomicCAS(err, 0, LUX_ERR_INDEX);
  } else {
    const int i = px >> 6, j = py >> 6;
    const bool interior = i >= 0 && i <= sw - 6 && j >= 0 && j <= sh - 6;
    if (interior || (j < sh && j + 6 > 0 && i < sw && i + 6 > 0)) {  // else the fill value 0
      const F2 *ty = tab + (py & 63) * 6, *tx = tab + (px & 63) * 6;
      const float4* row[6];
#pragma unroll
      for (int k = 0; k < 6; k++) row[k] = src + (size_t)min(max(j + k, 0), sh - 1) * sw;
      Px c[6];
#pragma unroll
      for (int k = 0; k < 6; k++) {
        const int col = min(max(i + k, 0), sw - 1);
        Px p[6];
#pragma unroll
        for (int r = 0; r < 6; r++) {
          p[r] = px_of(__ldg(row[r] + col));
          if (gain != 1.0f) p[r] = px_mul(p[r], g2, z);  // the source scaled in place first (StereoImageBuilder.cs:62)
        }
        c[k] = tap6(p, ty, z);
      }
      acc = px_f4(tap6(c, tx, z));
    }
  }
  const size_t o = (size_t)y * dw + x;
  if (MODE == 0) {
    out_f[o] = acc;
    return;
  }
  // ConvertToYUV (StereoImage.cs:181-195): (w·m3 + z·m2) + (y·m1 + x·m0) per row, then gamma and the U/V offsets
  float yuv[3];
#pragma unroll
  for (int r = 0; r < 3; r++)
    yuv[r] = gamma_encode(__fadd_rn(__fadd_rn(__fmul_rn(acc.w, m.m[r][3]), __fmul_rn(acc.z, m.m[r][2])),
                                    __fadd_rn(__fmul_rn(acc.y, m.m[r][1]), __fmul_rn(acc.x, m.m[r][0]))));
  const float4 v = make_float4(__fadd_rn(yuv[0], 0.0f), __fadd_rn(yuv[1], 128.0f), __fadd_rn(yuv[2], 128.0f), 1.0f);
  out_u8[o] = pack_u8(v);
  if (out_f) out_f[o] = v;
}

// Rgba8Warp.Warp (ReferenceGuide.cs:108-156): every tap clamped to the image (no fill), the six column sums accumulated
// row by row from the bytes as floats, the row combination as the float warp, the 8-bit store.
__global__ void __launch_bounds__(256) k_warp_rgba8(const uchar4* __restrict__ src, int sw, int sh, int sstride, const WarpGeom g,
                                                    const float* __restrict__ taps, const uint32_t* __restrict__ rsq, int dw, int dh,
                                                    uint32_t* __restrict__ out, int* err) {
  __shared__ F2 tab[384];
  load_taps(tab, taps);
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dw || y >= dh) return;
  int px, py;
  if (!warp_map(g, rsq, x, y, px, py)) {
    atomicCAS(err, 0, LUX_ERR_INDEX);
    out[(size_t)y * dw + x] = 0;
    return;
  }
  // a byte b as a float, exactly: the bits 0x4b0000bb are 2^23 + b, less 2^23 (one byte permute and half a packed add)
  const F2 bias = f2(-8388608.0f, -8388608.0f), z = f2(g.neg_zero, g.neg_zero);
  const int i = px >> 6, j = py >> 6;
  const F2 *ty = tab + (py & 63) * 6, *tx = tab + (px & 63) * 6;
  const uint32_t* row[6];
#pragma unroll
  for (int k = 0; k < 6; k++) row[k] = reinterpret_cast<const uint32_t*>(src) + (size_t)min(max(j + k, 0), sh - 1) * sstride;
  Px c[6];
#pragma unroll
  for (int k = 0; k < 6; k++) {
    const int col = min(max(i + k, 0), sw - 1);
    Px s;
#pragma unroll
    for (int r = 0; r < 6; r++) {
      const uint32_t w = __ldg(row[r] + col);
      const Px v{add2(f2(__uint_as_float(__byte_perm(w, 0x4b000000u, 0x7540)), __uint_as_float(__byte_perm(w, 0x4b000000u, 0x7541))), bias),
                 add2(f2(__uint_as_float(__byte_perm(w, 0x4b000000u, 0x7542)), __uint_as_float(__byte_perm(w, 0x4b000000u, 0x7543))), bias)};
      const Px p = px_mul(v, ty[r], z);
      s = r == 0 ? p : px_add(s, p);
    }
    c[k] = s;
  }
  out[(size_t)y * dw + x] = pack_u8(px_f4(tap6(c, tx, z)));
}

// StereoColorTransfer.Apply (StereoColorTransfer.cs:112-125) and the 8-bit store: o = a·((1·c3 + z·c2) + (y·c1 + x·c0))
// per lane with c_j the columns of the row-major F, alpha kept.
__global__ void __launch_bounds__(256) k_colour_apply(const float4* __restrict__ yuv, int npx, const ColourF F, uint32_t* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npx) return;
  const float4 p = yuv[i];
  float o[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float acc = __fadd_rn(__fadd_rn(__fmul_rn(1.0f, F.f[4 * k + 3]), __fmul_rn(p.z, F.f[4 * k + 2])),
                                __fadd_rn(__fmul_rn(p.y, F.f[4 * k + 1]), __fmul_rn(p.x, F.f[4 * k])));
    o[k] = __fmul_rn(p.w, acc);
  }
  out[i] = pack_u8(make_float4(o[0], o[1], o[2], p.w));
}

}  // namespace

void launch_colour_apply(const float* yuv, int npx, const ColourF& F, uint8_t* out, cudaStream_t s) {
  k_colour_apply<<<(npx + 255) / 256, 256, 0, s>>>(reinterpret_cast<const float4*>(yuv), npx, F, reinterpret_cast<uint32_t*>(out));
  count_launches(1);
}

void launch_warp_f32(const float* src, int sw, int sh, float gain, const WarpGeom& g, const float* taps, const uint32_t* rsq,
                     int dw, int dh, const YuvRows* m, float* out_f, uint8_t* out_u8, int* err, cudaStream_t s) {
  const dim3 block(16, 16), grid((dw + 15) / 16, (dh + 15) / 16);
  const float4* s4 = reinterpret_cast<const float4*>(src);
  if (m)
    k_warp_f32<1><<<grid, block, 0, s>>>(s4, sw, sh, gain, g, taps, rsq, dw, dh, *m, reinterpret_cast<float4*>(out_f),
                                         reinterpret_cast<uint32_t*>(out_u8), err);
  else
    k_warp_f32<0><<<grid, block, 0, s>>>(s4, sw, sh, gain, g, taps, rsq, dw, dh, YuvRows{}, reinterpret_cast<float4*>(out_f), nullptr,
                                         err);
  count_launches(1);
}

void launch_warp_rgba8(const uint8_t* src, int sw, int sh, int sstride, const WarpGeom& g, const float* taps, const uint32_t* rsq,
                       int dw, int dh, uint8_t* out, int* err, cudaStream_t s) {
  const dim3 block(16, 16), grid((dw + 15) / 16, (dh + 15) / 16);
  k_warp_rgba8<<<grid, block, 0, s>>>(reinterpret_cast<const uchar4*>(src), sw, sh, sstride, g, taps, rsq, dw, dh,
                                      reinterpret_cast<uint32_t*>(out), err);
  count_launches(1);
}

}  // namespace lux
