// Host-side geometry of the dense stage (see host_geom.h). Compiled without FP contraction: each float operation rounds
// once, as in the .NET reference.
#include "host_geom.h"

#include <climits>
#include <cmath>
#include <cstring>

#include "intel_approx_tables.h"

namespace lux {
namespace {

inline uint32_t bits_of(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float float_of(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline int net_f2i(float f) {  // (int)f in .NET 9+
  if (f != f) return 0;
  if (f >= 2147483648.0f) return INT_MAX;
  if (f < -2147483648.0f) return INT_MIN;
  return (int)f;
}

// Homography.Sqrt (Homography.cs:18): rsqrt table + one Newton step, 0 for 0
float approx_sqrt(float x) {
  float r = float_of(host_rsqrt_bits(bits_of(x)));
  float A = x * r, B = A * (-0.5f), C = A * r, D = C + (-3.0f), s = D * B;
  return x == 0.0f ? 0.0f : s;
}

// RcpNr (DenseStereo.cs:37): rcp + one Newton step
float rcp_newton(float a) {
  float x0 = host_rcp(a);
  float t = a * x0;
  t = 1.0f - t;
  t = x0 * t;
  return x0 + t;
}

struct Twister {  // std::mt19937 as Lux's Mt19937 (FundamentalMatrixFilter.cs:8-30)
  uint32_t s[624];
  int i = 624;
  explicit Twister(uint32_t seed) {
    s[0] = seed;
    for (int k = 1; k < 624; k++) s[k] = 1812433253u * (s[k - 1] ^ (s[k - 1] >> 30)) + (uint32_t)k;
  }
  uint32_t next() {
    if (i >= 624) {
      for (int k = 0; k < 624; k++) {
        uint32_t y = (s[k] & 0x80000000u) | (s[(k + 1) % 624] & 0x7fffffffu);
        s[k] = s[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
      }
      i = 0;
    }
    uint32_t r = s[i++];
    r ^= r >> 11;
    r ^= (r << 7) & 0x9d2c5680u;
    r ^= (r << 15) & 0xefc60000u;
    r ^= r >> 18;
    return r;
  }
};

void mul4(const double* a, const double* b, double* o) {  // Mat4D.Mul (ViewTransform.cs:88-94)
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      o[4 * i + j] = ((a[4 * i + 3] * b[12 + j] + a[4 * i + 2] * b[8 + j]) + (a[4 * i + 1] * b[4 + j] + a[4 * i] * b[j]));
}

void inverse4(const double* m, double* o) {  // Mat4D.Inverse (ViewTransform.cs:96-120): adjugate over the determinant
  const double m00 = m[0], m01 = m[1], m02 = m[2], m03 = m[3], m10 = m[4], m11 = m[5], m12 = m[6], m13 = m[7];
  const double m20 = m[8], m21 = m[9], m22 = m[10], m23 = m[11], m30 = m[12], m31 = m[13], m32 = m[14], m33 = m[15];
  double c[16];
  c[0] = (m11 * (m22 * m33 - m23 * m32)) + ((m12 * (m23 * m31 - m33 * m21)) + (m13 * (m32 * m21 - m31 * m22)));
  c[1] = (m01 * (m23 * m32 - m22 * m33)) + ((m02 * (m33 * m21 - m23 * m31)) + (m03 * (m31 * m22 - m32 * m21)));
  c[2] = (((m02 * m13 - m12 * m03) * m31) + ((m12 * m01) * m33 + (m11 * m03) * m32)) - ((m01 * m13) * m32 + (m11 * m02) * m33);
  c[3] = ((m23 * (m11 * m02 - m12 * m01)) + (m21 * (m12 * m03 - m02 * m13))) + (m22 * (m01 * m13 - m11 * m03));
  c[4] = ((m12 * (m33 * m20 - m23 * m30)) + (m13 * (m22 * m30 - m32 * m20))) + (m10 * (m23 * m32 - m22 * m33));
  c[5] = (m00 * (m22 * m33 - m23 * m32)) + ((m02 * (m23 * m30 - m33 * m20)) + (m03 * (m32 * m20 - m22 * m30)));
  c[6] = (m33 * (m02 * m10 - m00 * m12)) + ((m30 * (m12 * m03 - m02 * m13)) + (m32 * (m00 * m13 - m03 * m10)));
  c[7] = (((m02 * m13 - m12 * m03) * m20) + ((m03 * m10) * m22 + (m00 * m12) * m23)) - (m23 * (m02 * m10) + (m00 * m13) * m22);
  c[8] = (m11 * (m23 * m30 - m33 * m20)) + ((m13 * (m31 * m20 - m21 * m30)) + (m10 * (m33 * m21 - m23 * m31)));
  c[9] = (m00 * (m23 * m31 - m33 * m21)) + (((m33 * m20 - m23 * m30) * m01) + (m03 * (m21 * m30 - m31 * m20)));
  c[10] = (((m01 * m13 - m11 * m03) * m30) + ((m00 * m11) * m33 + (m03 * m10) * m31)) - ((m00 * m13) * m31 + m33 * (m01 * m10));
  c[11] = (m23 * (m01 * m10 - m00 * m11)) + ((m20 * (m11 * m03 - m01 * m13)) + (m21 * (m00 * m13 - m03 * m10)));
  c[12] = (m11 * (m32 * m20 - m22 * m30)) + ((m12 * (m21 * m30 - m31 * m20)) + (m10 * (m31 * m22 - m32 * m21)));
  c[13] = (m00 * (m32 * m21 - m31 * m22)) + (((m22 * m30 - m32 * m20) * m01) + (m02 * (m31 * m20 - m21 * m30)));
  c[14] = (m32 * (m01 * m10 - m00 * m11)) + (((m11 * m02 - m12 * m01) * m30) + (m31 * (m00 * m12 - m02 * m10)));
  c[15] = (((m12 * m01 - m11 * m02) * m20) + ((m02 * m10) * m21 + (m00 * m11) * m22)) - ((m01 * m10) * m22 + (m00 * m12) * m21);
  const double det = ((c[12] * m03 + m02 * c[8]) + (c[4] * m01 + m00 * c[0]));
  const double rd = 1.0 / det;
  for (int k = 0; k < 16; k++) o[k] = c[k] * rd;
}

void k_matrix(const lux_calib& c, double* k) {
  std::memset(k, 0, 16 * sizeof(double));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) k[4 * i + j] = c.K[3 * i + j];
  k[15] = 1.0;
}
void e_matrix(const lux_calib& c, double* e) {
  std::memset(e, 0, 16 * sizeof(double));
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) e[4 * i + j] = c.R[3 * i + j];
    e[4 * i + 3] = c.T[i];
  }
  e[15] = 1.0;
}

}  // namespace

uint32_t host_rcp_bits(uint32_t b) {
  uint32_t sign = b & 0x80000000u, e = (b >> 23) & 0xff, m = b & 0x7fffff;
  if (e == 0xff) return m != 0 ? (b | 0x400000u) : sign;
  if (e == 0) return sign | 0x7f800000u;
  uint32_t r = lux_rcp_table[m >> 11];
  int re = (int)((r >> 23) & 0xff) - ((int)e - 127);
  if (re <= 0) return sign;
  return sign | ((uint32_t)re << 23) | (r & 0x7fffff);
}

uint32_t host_rsqrt_bits(uint32_t b) {
  uint32_t sign = b & 0x80000000u, e = (b >> 23) & 0xff, m = b & 0x7fffff;
  if (e == 0xff && m != 0) return b | 0x400000u;
  if (e == 0) return sign | 0x7f800000u;
  if (sign != 0) return 0xffc00000u;
  if (e == 0xff) return 0;
  int k = (int)e - 127;
  uint32_t r;
  int re;
  if ((k & 1) == 0) {
    r = lux_rsqrt_table_e127[m >> 11];
    re = (int)((r >> 23) & 0xff) - k / 2;
  } else {
    r = lux_rsqrt_table_e128[m >> 11];
    re = (int)((r >> 23) & 0xff) - (k - 1) / 2;
  }
  if (re <= 0) return 0;
  return ((uint32_t)re << 23) | (r & 0x7fffff);
}

float host_rcp(float x) { return float_of(host_rcp_bits(bits_of(x))); }
const uint32_t* host_rcp_table() { return lux_rcp_table; }
const uint32_t* host_rsqrt_table(bool e128) { return e128 ? lux_rsqrt_table_e128 : lux_rsqrt_table_e127; }
void host_mat4_mul(const double* a, const double* b, double* o) { mul4(a, b, o); }

namespace {

// sinf as Wine's ucrtbase evaluates it (Lux.Engine/Pipeline/WineCrt.cs:21-99): quadrant shifts by multiples of pi/2 in
// double, then the Taylor polynomials of sin and cos to degree 9 and 10 in double, rounded to float once. The Lanczos
// table only reaches |x| < 3·pi, inside the shifted ranges; the general reduction (n = rint(x·2/pi)) covers the rest.
float sin_poly(double x) {
  const double z = x * x;
  if (x > -0.007817583158612251 && 0.007817583158612251 > x) return (float)((z * -0.16666666666666666 + 1.0) * x);
  const double s = x * z, w = z * z;
  const double r = 2.7557319223985893e-06 * z - 0.0001984126984126984, q = z * 0.008333333333333333 - 0.16666666666666666;
  return (float)((w * s) * r + (q * s + x));
}
float cos_poly(double x) {
  const double z = x * x;
  if (x > -0.007816314697265625 && 0.007816314697265625 > x) return (float)(z * -0.5 + 1.0);
  double p = -2.755731922398589e-07 * z + 2.48015873015873e-05;
  p = p * z - 0.001388888888888889;
  p = p * z + 0.041666666666666664;
  p = p * z - 0.5;
  return (float)(p * z + 1.0);
}
float crt_sinf(float x) {
  const double half_pi = 1.5707963267948966, pi = 3.141592653589793, three_half_pi = 4.71238898038469, two_pi = 6.283185307179586;
  const uint32_t ax = bits_of(x) & 0x7fffffffu;
  const bool neg = (bits_of(x) >> 31) != 0;
  const double d = x;
  if (ax <= 0x3f490fdau) return ax < 0x39800000u ? x : sin_poly(d);                                      // |x| <= pi/4
  if (ax <= 0x4016cbe3u) return neg ? -cos_poly(d + half_pi) : cos_poly(d - half_pi);                   // <= 3pi/4
  if (ax <= 0x407b53d1u) return sin_poly(neg ? -(d + pi) : -(d - pi));                                  // <= 5pi/4
  if (ax <= 0x40afeddfu) return neg ? cos_poly(d + three_half_pi) : -cos_poly(d - three_half_pi);       // <= 7pi/4
  if (ax <= 0x40e231d5u) return sin_poly(neg ? d + two_pi : d - two_pi);                                // <= 9pi/4
  if (ax >= 0x7f800000u) return x - x;
  const double n = d * 6.36619772367581382433e-01 + 6755399441055744.0 - 6755399441055744.0;
  const double y = d - n * 1.57079631090164184570e+00 - n * 1.58932547735281966916e-08;
  switch ((int)n & 3) {
    case 0: return sin_poly(y);
    case 1: return cos_poly(y);
    case 2: return sin_poly(-y);
    default: return -cos_poly(y);
  }
}

}  // namespace

void host_lanczos_table(float out[384]) {
  const float pi = float_of(0x40490fdbu), pi_3 = float_of(0x3f860a92u), pi_sq = float_of(0x411de9e7u);
  for (int phase = 0; phase < 64; phase++) {
    const float p = (float)phase * 0.015625f;
    float sum = 0.0f;
    for (int tap = 0; tap < 6; tap++) {
      const float x = p - (float)(tap - 2);
      float w = 0.0f;
      if (x == 0.0f) w = 1.0f;
      else if (std::fabs(x) < 3.0f) w = (crt_sinf(x * pi_3) * (crt_sinf(x * pi) * 3.0f)) / ((x * x) * pi_sq);
      out[phase * 6 + tap] = w;
      sum = sum + w;
    }
    const float inv = 1.0f / sum;
    for (int tap = 0; tap < 6; tap++) out[phase * 6 + tap] *= inv;
  }
}

void host_yuv_matrix(int sensor_type, const float neutral[3], float out[12]) {
  // the luma basis per sensor type: AR1335 (types 2, 3) and the others (StereoImage.cs:135-136)
  static const uint32_t kAr1335[3] = {0x3e5cb924u, 0x3edd5758u, 0x3eb44c16u}, kOther[3] = {0x3e9e39b4u, 0x3e95ca4bu, 0x3ecbfc22u};
  const uint32_t* t = (sensor_type == 2 || sensor_type == 3) ? kAr1335 : kOther;
  const float a = float_of(t[0]), b = float_of(t[1]), c = float_of(t[2]);
  const float ix = 1.0f / neutral[0], iy = 1.0f / neutral[1], iz = 1.0f / neutral[2];
  const float s = c + a;
  const float u0 = (b * (-b) - s * c) * ix, u1 = ((a - c) * b) * iy, u2 = (s * a - b * (-b)) * iz;
  const float t0 = ix * (-b), t1 = iy * s, t2 = iz * (-b);
  // 1/|row| by rsqrtss and one Newton step, in the reference's operation order
  const float v2 = c * c + (b * b + a * a);
  const float rv = float_of(host_rsqrt_bits(bits_of(v2))), Sv = v2 * rv;
  const float kv = v2 == 0.0f ? 0.0f : (Sv * rv + (-3.0f)) * (Sv * (-0.5f));
  const float nu = u2 * u2 + (u1 * u1 + u0 * u0), ru = float_of(host_rsqrt_bits(bits_of(nu)));
  const float ku = ((ru * (-0.5f)) * kv) * ((nu * ru) * ru + (-3.0f));
  const float nt = t2 * t2 + (t1 * t1 + t0 * t0), rt = float_of(host_rsqrt_bits(bits_of(nt)));
  const float kt = ((rt * (-0.5f)) * kv) * ((nt * rt) * rt + (-3.0f));
  const float m[12] = {a, b, c, 0.0f, u0 * ku, u1 * ku, ku * u2, 0.0f, t0 * kt, t1 * kt, kt * t2, 0.0f};
  std::memcpy(out, m, sizeof m);
}

int host_planes(float near_, float far_, const lux_calib* calibs, int ncams, float density, int align, std::vector<float>& planes) {
  if (!(near_ < far_)) return LUX_ERR_NEAR_FAR;
  if (!(near_ > 0.0f && far_ > 0.0f)) return LUX_ERR_NONPOSITIVE;
  if (align <= 0 || ncams <= 0 || !calibs) return LUX_ERR_ARG;
  std::vector<float> C(3 * (size_t)ncams);
  for (int k = 0; k < ncams; k++) {  // camera centres t·R (DenseStereo.cs:46-50)
    const float *R = calibs[k].R, *t = calibs[k].T;
    C[3 * k + 0] = (t[0] * R[0] + t[1] * R[3]) + t[2] * R[6];
    C[3 * k + 1] = (t[0] * R[1] + t[1] * R[4]) + t[2] * R[7];
    C[3 * k + 2] = (t[0] * R[2] + t[1] * R[5]) + t[2] * R[8];
  }
  float B = 0.0f;  // the largest distance to the reference centre, MAXSS order (:51-58)
  for (int k = 0; k < ncams; k++) {
    float dx = C[0] - C[3 * k], dy = C[1] - C[3 * k + 1], dz = C[2] - C[3 * k + 2];
    float d2 = dz * dz + (dx * dx + dy * dy);
    float d = approx_sqrt(d2);
    if (!(d <= B)) B = d;
  }
  const float inv_near = rcp_newton(near_), inv_far = rcp_newton(far_);
  const float inv = inv_near - inv_far;
  int n = net_f2i(((inv * density) * B) * calibs[0].K[0]);
  if (n > 0x1000) n = 0x1000;
  if (n <= 0) return LUX_ERR_BASELINE;
  n = ((n + align - 1) / align) * align;
  planes.assign((size_t)n, 0.0f);
  const float step = (inv_near - inv_far) / (float)(n - 1), base = inv_far;
  if (n - 1 <= 7) {
    float v = base;
    for (int i = 0; i < n - 1; i++) { planes[i] = 1.0f / v; v += step; }
  } else {  // eight planes per iteration from two 4-lane RcpNr vectors (:71-85)
    const int m = (n - 1) & ~7;
    float lanes[4];
    const float d4 = 4.0f * step;
    for (int l = 0; l < 4; l++) lanes[l] = step * (float)l + base;
    for (int i = 0; i < m; i += 8) {
      float hi[4];
      for (int l = 0; l < 4; l++) hi[l] = lanes[l] + d4;
      for (int l = 0; l < 4; l++) {
        planes[i + l] = rcp_newton(lanes[l]);
        planes[i + 4 + l] = rcp_newton(hi[l]);
      }
      for (int l = 0; l < 4; l++) lanes[l] = hi[l] + d4;
    }
    float v = (float)m * step + base;
    for (int i = m; i < n - 1; i++) { planes[i] = 1.0f / v; v += step; }
  }
  planes[n - 1] = near_;
  return LUX_OK;
}

void host_flow_matrix(const lux_calib& a, const lux_calib& b, float out[16]) {
  double kb[16], eb[16], ka[16], ea[16], pb[16], pa[16], ia[16], M[16];
  k_matrix(b, kb); e_matrix(b, eb); mul4(kb, eb, pb);
  k_matrix(a, ka); e_matrix(a, ea); mul4(ka, ea, pa);
  inverse4(pa, ia);
  mul4(pb, ia, M);
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) out[4 * c + r] = (float)M[4 * r + c];
}

void host_skip_stream_bits(uint32_t out[256]) {
  Twister mt(5489u);  // the default seed, as every tile of DenseLayer.SkipMask uses (DenseStereoSgm.cs:74-84)
  for (int w = 0; w < 256; w++) out[w] = 0;
  for (int k = 0; k < 8192; k++) out[k >> 5] |= (mt.next() & 1u) << (k & 31);
}

bool host_range_bounds(const std::vector<float>& planes, std::vector<float>& b) {
  const size_t n = planes.size();
  b.assign(n, 0.0f);
  for (size_t i = 0; i + 1 < n; i++) b[i] = (host_rcp(planes[i + 1]) + host_rcp(planes[i])) * 0.5f;
  if (n) b[n - 1] = 3.40282347e+38f;  // float.MaxValue
  bool mono = true;
  for (size_t i = 0; i + 1 < n; i++)
    if (!(b[i] <= b[i + 1])) mono = false;
  return mono;
}

}  // namespace lux
