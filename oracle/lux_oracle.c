/* CPU oracle for the dense-stereo depth stage of Lux.Engine — TEST INFRASTRUCTURE ONLY (see lux_oracle.h).
 * Parity unpinned against reference outputs (no golden vectors exist for this path; the C# reference cannot run here).
 * Each function cites the reference file:line it restates. Build: -O2 -ffp-contract=off (no FMA, no fast-math). */
#include "lux_oracle.h"
#include "intel_approx_tables.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* ---------------- .NET scalar semantics ---------------- */
static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float ffrom(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
/* (int)f in .NET 9+: truncation, saturating, NaN -> 0 */
static inline int cs_f2i(float f) {
  if (f != f) return 0;
  if (f >= 2147483648.0f) return INT_MAX;
  if (f < -2147483648.0f) return INT_MIN;
  return (int)f;
}
/* Math.Max / Math.Min (float): NaN propagates, +0 > -0 */
static inline float cs_maxf(float a, float b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a == b) return signbit(a) ? b : a;
  return a > b ? a : b;
}
static inline float cs_minf(float a, float b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a == b) return signbit(a) ? a : b;
  return a < b ? a : b;
}
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int iclamp(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }

/* ---------------- StereoParams (DenseStereo.cs:15-31) ---------------- */
void lo_default_params(lo_params* p) {
  p->margin = 1;
  p->plane_density = 2.0f;
  p->scale = 32;
  p->skip_mode = 0;
  p->p1 = 1;
  p->p2scale = 500.0f;
  float g = ffrom(0x3ef6384fu);
  p->guidance[0] = g / 6.0f;
  p->guidance[1] = g / 16.0f;
  p->guidance[2] = g / 16.0f;
  p->guidance[3] = 0.0f;
  p->tile = 4;
}

void lo_l16_pyramid(lo_params out[6]) {
  static const int scales[6] = {32, 16, 8, 4, 2, 1}, tiles[6] = {4, 8, 16, 32, 64, 64};
  for (int i = 0; i < 6; i++) {
    lo_default_params(&out[i]);
    out[i].scale = scales[i];
    out[i].tile = tiles[i];
    out[i].skip_mode = i >= 4 ? 2 : 0;
    out[i].plane_density = 2.0f;
  }
}

/* ---------------- IntelApprox (IntelApprox.cs:21-45) ---------------- */
uint32_t lo_rcp_bits(uint32_t b) {
  uint32_t sign = b & 0x80000000u, e = (b >> 23) & 0xff, m = b & 0x7fffff;
  if (e == 0xff) return m != 0 ? (b | 0x400000u) : sign;
  if (e == 0) return sign | 0x7f800000u;
  uint32_t r = lux_rcp_table[m >> 11];
  int re = (int)((r >> 23) & 0xff) - ((int)e - 127);
  if (re <= 0) return sign;
  return sign | ((uint32_t)re << 23) | (r & 0x7fffff);
}

uint32_t lo_rsqrt_bits(uint32_t b) {
  uint32_t sign = b & 0x80000000u, e = (b >> 23) & 0xff, m = b & 0x7fffff;
  if (e == 0xff && m != 0) return b | 0x400000u;
  if (e == 0) return sign | 0x7f800000u;
  if (sign != 0) return 0xffc00000u;
  if (e == 0xff) return 0;
  int k = (int)e - 127;
  uint32_t r;
  int re;
  if ((k & 1) == 0) { r = lux_rsqrt_table_e127[m >> 11]; re = (int)((r >> 23) & 0xff) - k / 2; }
  else { r = lux_rsqrt_table_e128[m >> 11]; re = (int)((r >> 23) & 0xff) - (k - 1) / 2; }
  if (re <= 0) return 0;
  return ((uint32_t)re << 23) | (r & 0x7fffff);
}

float lo_rcp(float x) { return ffrom(lo_rcp_bits(fbits(x))); }
static float lo_rsqrt_raw(float x) { return ffrom(lo_rsqrt_bits(fbits(x))); }

/* Homography.Sqrt (Homography.cs:18) */
float lo_homography_sqrt(float x) {
  float r = lo_rsqrt_raw(x);
  float A = x * r, B = A * (-0.5f), C = A * r, D = C + (-3.0f), s = D * B;
  return x == 0.0f ? 0.0f : s;
}

/* RcpNr (DenseStereo.cs:37-38): rcp + one Newton step */
static float rcp_nr(float a) {
  float x0 = lo_rcp(a);
  float t = a * x0;
  t = 1.0f - t;
  t = x0 * t;
  return x0 + t;
}

/* ---------------- Mt19937 (FundamentalMatrixFilter.cs:8-30) ---------------- */
void lo_mt_seed(lo_mt19937* m, uint32_t seed) {
  m->mt[0] = seed;
  for (int i = 1; i < 624; i++) m->mt[i] = (uint32_t)(1812433253u * (m->mt[i - 1] ^ (m->mt[i - 1] >> 30)) + (uint32_t)i);
  m->idx = 624;
}

uint32_t lo_mt_next(lo_mt19937* m) {
  if (m->idx >= 624) {
    for (int i = 0; i < 624; i++) {
      uint32_t y = (m->mt[i] & 0x80000000u) | (m->mt[(i + 1) % 624] & 0x7fffffffu);
      m->mt[i] = m->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) != 0 ? 0x9908b0dfu : 0u);
    }
    m->idx = 0;
  }
  uint32_t r = m->mt[m->idx++];
  r ^= r >> 11;
  r ^= (r << 7) & 0x9d2c5680u;
  r ^= (r << 15) & 0xefc60000u;
  r ^= r >> 18;
  return r;
}

/* ---------------- Mat4D (ViewTransform.cs:86-133), double ---------------- */
static void mat4_mul(const double* a, const double* b, double* o) {
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      o[4 * i + j] = ((a[4 * i + 3] * b[12 + j] + a[4 * i + 2] * b[8 + j]) + (a[4 * i + 1] * b[4 + j] + a[4 * i] * b[j]));
}

static void mat4_inverse(const double* m, double* o) {
  double m00 = m[0], m01 = m[1], m02 = m[2], m03 = m[3], m10 = m[4], m11 = m[5], m12 = m[6], m13 = m[7];
  double m20 = m[8], m21 = m[9], m22 = m[10], m23 = m[11], m30 = m[12], m31 = m[13], m32 = m[14], m33 = m[15];
  double adj[16];
  adj[0] = (m11 * (m22 * m33 - m23 * m32)) + ((m12 * (m23 * m31 - m33 * m21)) + (m13 * (m32 * m21 - m31 * m22)));
  adj[1] = (m01 * (m23 * m32 - m22 * m33)) + ((m02 * (m33 * m21 - m23 * m31)) + (m03 * (m31 * m22 - m32 * m21)));
  adj[2] = (((m02 * m13 - m12 * m03) * m31) + ((m12 * m01) * m33 + (m11 * m03) * m32)) - ((m01 * m13) * m32 + (m11 * m02) * m33);
  adj[3] = ((m23 * (m11 * m02 - m12 * m01)) + (m21 * (m12 * m03 - m02 * m13))) + (m22 * (m01 * m13 - m11 * m03));
  adj[4] = ((m12 * (m33 * m20 - m23 * m30)) + (m13 * (m22 * m30 - m32 * m20))) + (m10 * (m23 * m32 - m22 * m33));
  adj[5] = (m00 * (m22 * m33 - m23 * m32)) + ((m02 * (m23 * m30 - m33 * m20)) + (m03 * (m32 * m20 - m22 * m30)));
  adj[6] = (m33 * (m02 * m10 - m00 * m12)) + ((m30 * (m12 * m03 - m02 * m13)) + (m32 * (m00 * m13 - m03 * m10)));
  adj[7] = (((m02 * m13 - m12 * m03) * m20) + ((m03 * m10) * m22 + (m00 * m12) * m23)) - (m23 * (m02 * m10) + (m00 * m13) * m22);
  adj[8] = (m11 * (m23 * m30 - m33 * m20)) + ((m13 * (m31 * m20 - m21 * m30)) + (m10 * (m33 * m21 - m23 * m31)));
  adj[9] = (m00 * (m23 * m31 - m33 * m21)) + (((m33 * m20 - m23 * m30) * m01) + (m03 * (m21 * m30 - m31 * m20)));
  adj[10] = (((m01 * m13 - m11 * m03) * m30) + ((m00 * m11) * m33 + (m03 * m10) * m31)) - ((m00 * m13) * m31 + m33 * (m01 * m10));
  adj[11] = (m23 * (m01 * m10 - m00 * m11)) + ((m20 * (m11 * m03 - m01 * m13)) + (m21 * (m00 * m13 - m03 * m10)));
  adj[12] = (m11 * (m32 * m20 - m22 * m30)) + ((m12 * (m21 * m30 - m31 * m20)) + (m10 * (m31 * m22 - m32 * m21)));
  adj[13] = (m00 * (m32 * m21 - m31 * m22)) + (((m22 * m30 - m32 * m20) * m01) + (m02 * (m31 * m20 - m21 * m30)));
  adj[14] = (m32 * (m01 * m10 - m00 * m11)) + (((m11 * m02 - m12 * m01) * m30) + (m31 * (m00 * m12 - m02 * m10)));
  adj[15] = (((m12 * m01 - m11 * m02) * m20) + ((m02 * m10) * m21 + (m00 * m11) * m22)) - ((m01 * m10) * m22 + (m00 * m12) * m21);
  double det = ((adj[12] * m03 + m02 * adj[8]) + (adj[4] * m01 + m00 * adj[0]));
  double rd = 1.0 / det;
  for (int k = 0; k < 16; k++) o[k] = adj[k] * rd;
}

static void kd(const lo_calib* c, double* k) {
  memset(k, 0, 16 * sizeof(double));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) k[4 * i + j] = c->K[3 * i + j];
  k[15] = 1.0;
}
static void ed(const lo_calib* c, double* e) {
  memset(e, 0, 16 * sizeof(double));
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) e[4 * i + j] = c->R[3 * i + j];
    e[4 * i + 3] = c->T[i];
  }
  e[15] = 1.0;
}

void lo_flow_matrix(const lo_calib* a, const lo_calib* b, float out[16]) {
  double ka[16], ea[16], kb[16], eb[16], p1[16], p2[16], inv[16], M[16];
  kd(b, kb); ed(b, eb); mat4_mul(kb, eb, p1);
  kd(a, ka); ed(a, ea); mat4_mul(ka, ea, p2);
  mat4_inverse(p2, inv);
  mat4_mul(p1, inv, M);
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) out[4 * c + r] = (float)M[4 * r + c];
}

/* ---------------- Planes (DenseStereo.cs:41-88) ---------------- */
int lo_planes(float near_, float far_, const lo_calib* calibs, int ncams, float density, int align, float* planes, int* n_out) {
  if (!(near_ < far_)) return LO_ERR_NEAR_FAR;
  if (!(near_ > 0.0f && far_ > 0.0f)) return LO_ERR_NONPOSITIVE;
  if (align <= 0 || ncams <= 0) return LO_ERR_ARG;
  float (*C)[3] = (float (*)[3])malloc(sizeof(float[3]) * (size_t)ncams);
  if (!C) return LO_ERR_ALLOC;
  for (int k = 0; k < ncams; k++) {
    const float *R = calibs[k].R, *t = calibs[k].T;
    C[k][0] = (t[0] * R[0] + t[1] * R[3]) + t[2] * R[6];
    C[k][1] = (t[0] * R[1] + t[1] * R[4]) + t[2] * R[7];
    C[k][2] = (t[0] * R[2] + t[1] * R[5]) + t[2] * R[8];
  }
  float B = 0.0f;
  for (int k = 0; k < ncams; k++) {
    float dx = C[0][0] - C[k][0], dy = C[0][1] - C[k][1], dz = C[0][2] - C[k][2];
    float d2 = dz * dz + (dx * dx + dy * dy);
    float d = lo_homography_sqrt(d2);
    if (!(d <= B)) B = d;
  }
  free(C);
  float x1_0 = rcp_nr(near_), x1_1 = rcp_nr(far_);
  float inv = x1_0 - x1_1;
  int n = cs_f2i(((inv * density) * B) * calibs[0].K[0]);
  if (n > 0x1000) n = 0x1000;
  if (n <= 0) return LO_ERR_BASELINE;
  n = ((n + align - 1) / align) * align;
  float step = (x1_0 - x1_1) / (float)(n - 1), bas = x1_1;
  if (n - 1 <= 7) {
    float v = bas;
    for (int i = 0; i < n - 1; i++) { planes[i] = 1.0f / v; v += step; }
  } else {
    int m = (n - 1) & ~7;
    float v4[4], d4 = 4.0f * step;
    for (int l = 0; l < 4; l++) v4[l] = step * (float)l + bas;
    for (int i = 0; i < m; i += 8) {
      float hi[4];
      for (int l = 0; l < 4; l++) hi[l] = v4[l] + d4;
      for (int l = 0; l < 4; l++) { planes[i + l] = rcp_nr(v4[l]); planes[i + 4 + l] = rcp_nr(hi[l]); }
      for (int l = 0; l < 4; l++) v4[l] = hi[l] + d4;
    }
    float v = (float)m * step + bas;
    for (int i = m; i < n - 1; i++) { planes[i] = 1.0f / v; v += step; }
  }
  planes[n - 1] = near_;
  *n_out = n;
  return LO_OK;
}

/* ---------------- BoxFilter3 (DenseStereo.cs:93-159) ---------------- */
static inline uint8_t sat_u8_rne(float v) {
  /* cvtps2dq (RNE; NaN/overflow -> INT_MIN) -> packssdw -> packuswb */
  int q;
  if (v != v || v >= 2147483648.0f || v < -2147483648.0f) q = INT_MIN;
  else q = (int)rintf(v);
  if (q < 0) return 0;
  if (q > 255) return 255;
  return (uint8_t)q;
}

void lo_box_filter3(const uint8_t* src, int W, int H, uint8_t* dst) {
  if (W < 2) { lo_box_filter3_scalar(src, W, H, dst); return; }
  /* row sums of three taps (RowSums3, :126-135), then the sum of up to three rows */
  uint16_t* sums = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)W * 4 * 3);
  for (int y = 0; y < H; y++) {
    int y0 = imax(y - 1, 0), y1 = imin(y + 1, H - 1);
    int rows = y1 - y0 + 1;
    for (int k = 0; k < rows; k++) {
      const uint8_t* row = src + (size_t)(y0 + k) * W * 4;
      uint16_t* s = sums + (size_t)k * W * 4;
      int last = (W - 1) * 4;
      for (int c = 0; c < 4; c++) {
        s[c] = (uint16_t)(row[c] + row[4 + c]);
        s[last + c] = (uint16_t)(row[last - 4 + c] + row[last + c]);
      }
      for (int i = 4; i < last; i++) s[i] = (uint16_t)(row[i - 4] + row[i] + row[i + 4]);
    }
    float invEdge = 1.0f / ((float)2 * (float)rows), invInner = 1.0f / ((float)3 * (float)rows);
    for (int x = 0; x < W; x++)
      for (int c = 0; c < 4; c++) {
        int sum = 0;
        for (int k = 0; k < rows; k++) sum += sums[(size_t)k * W * 4 + x * 4 + c];
        float v = (float)sum * ((x == 0 || x == W - 1) ? invEdge : invInner);
        dst[((size_t)y * W + x) * 4 + c] = sat_u8_rne(v);
      }
  }
  free(sums);
}

void lo_box_filter3_scalar(const uint8_t* src, int W, int H, uint8_t* dst) {
  for (int y = 0; y < H; y++) {
    int y0 = imax(y - 1, 0), y1 = imin(y + 1, H - 1);
    int rows = y1 - y0 + 1;
    for (int x = 0; x < W; x++) {
      int x0 = imax(x - 1, 0), x1 = imin(x + 1, W - 1);
      int cols = x1 - x0 + 1;
      float inv = 1.0f / ((float)cols * (float)rows);
      for (int c = 0; c < 4; c++) {
        int sum = 0;
        for (int yy = y0; yy <= y1; yy++)
          for (int xx = x0; xx <= x1; xx++) sum += src[((size_t)yy * W + xx) * 4 + c];
        float v = (float)sum * inv;
        int r = cs_f2i(rintf(v));
        dst[((size_t)y * W + x) * 4 + c] = (uint8_t)iclamp(r, 0, 255);
      }
    }
  }
}

/* ---------------- Guidance (DenseStereo.cs:163-177) ---------------- */
void lo_guidance(const uint8_t* img0, int W0, int H0, int w, int h, int scale, uint8_t* g) {
  if (W0 == w && H0 == h) { memcpy(g, img0, (size_t)w * h * 4); return; }
  int half = (scale + (scale >> 31)) >> 1;
  for (int y = 0; y < h; y++) {
    int sy = imin(scale * y + half, H0 - 1);
    for (int x = 0; x < w; x++) {
      int sx = imin(scale * x + half, W0 - 1);
      memcpy(g + ((size_t)y * w + x) * 4, img0 + ((size_t)sy * W0 + sx) * 4, 4);
    }
  }
}

/* ---------------- MatchingCost (DenseStereo.cs:217-373) ---------------- */
static const uint8_t kCaps[4] = {2, 6, 6, 0}; /* CostContext.Caps, DenseStereo.cs:187 */

static inline uint8_t pavgb(uint8_t a, uint8_t b) { return (uint8_t)((a + b + 1) >> 1); }

/* the per-(camera, plane) projection shared by both forms (DenseStereo.cs:254-266, :319-331) */
static inline void project(const float* Wm, float xf, float yf, float z, float* fx, float* fy) {
  float xz = (xf * z) * 1.0f, yz = (yf * z) * 1.0f;
  float px = ((z * Wm[8] + Wm[12]) + xz * Wm[0]) + yz * Wm[4];
  float py = ((z * Wm[9] + Wm[13]) + xz * Wm[1]) + yz * Wm[5];
  float pz = ((z * Wm[10] + Wm[14]) + xz * Wm[2]) + yz * Wm[6];
  float inv = 1.0f / pz;
  *fx = px * inv + 0.25f;
  *fy = py * inv + 0.25f;
}

static void ref_block(const lo_costctx* c, int x, int y, uint8_t rb[3][16]) {
  memset(rb, 0, 48);
  for (int r = -1; r <= 1; r++) {
    int yy = iclamp(y + r, 0, c->h - 1);
    for (int cc = -1; cc <= 1; cc++) {
      int xx = iclamp(x + cc, 0, c->w - 1);
      memcpy(&rb[r + 1][(cc + 1) * 4], c->ref + ((size_t)yy * c->w + xx) * 4, 4);
    }
  }
}

/* the block cost of one target position: the vector form's byte lanes (DenseStereo.cs:276-287) */
static int block_cost_vec(const uint8_t* img, int iw, int ix, int iy, int hx, int hy, const uint8_t rb[3][16], const uint16_t* wq) {
  uint8_t a[4][16];
  const uint8_t* t = img + ((size_t)(iy - 1) * iw + (ix - 1)) * 4;
  for (int q = 0; q < 4; q++) memcpy(a[q], t + (size_t)q * iw * 4, 16);
  uint8_t r[3][16];
  for (int q = 0; q < 3; q++)
    for (int b = 0; b < 16; b++) r[q][b] = hy ? pavgb(a[q][b], a[q + 1][b]) : a[q][b];
  if (hx)
    for (int q = 0; q < 3; q++) {
      uint8_t nx[16];
      for (int b = 0; b < 16; b++) nx[b] = r[q][(b < 12 ? b + 4 : b)]; /* NextPixel: pixels (1,2,3,3) */
      for (int b = 0; b < 16; b++) r[q][b] = pavgb(r[q][b], nx[b]);
    }
  uint8_t rowSum[16];
  for (int b = 0; b < 16; b++) {
    int s = 0;
    for (int q = 0; q < 3; q++) {
      int hi = r[q][b] > rb[q][b] ? r[q][b] : rb[q][b], lo = r[q][b] > rb[q][b] ? rb[q][b] : r[q][b];
      int d = (uint8_t)(hi - lo);
      s += d < kCaps[b & 3] ? d : kCaps[b & 3];
    }
    rowSum[b] = (uint8_t)s; /* byte lanes: at most 3·28 */
  }
  uint32_t e0, e1, e2;
  memcpy(&e0, rowSum, 4); memcpy(&e1, rowSum + 4, 4); memcpy(&e2, rowSum + 8, 4);
  uint32_t s = e0 + e1 + e2;
  int S0 = (int)(s & 0xff), S1 = (int)((s >> 8) & 0xff), S2 = (int)((s >> 16) & 0xff), S3 = (int)(s >> 24);
  int cY = (S0 * wq[0] + 16) >> 5, cU = (S1 * wq[1] + 16) >> 5, cV = (S2 * wq[2] + 16) >> 5, cA = (S3 * wq[3] + 16) >> 5;
  int ck = (cY + cU) + (cV + cA);
  float cf = cs_minf((float)ck, 65535.0f);
  return cs_f2i(cf);
}

int lo_matching_cost(const lo_costctx* c, int x, int y, int start, int count, uint16_t* cost) {
  if (start < 0 || count < 0 || start + count > c->n_planes) return lo_matching_cost_scalar(c, x, y, start, count, cost);
  memset(cost, 0, sizeof(uint16_t) * (size_t)count);
  uint8_t rb[3][16];
  ref_block(c, x, y, rb);
  float xf = (float)x, yf = (float)y;
  for (int k = 0; k < c->n_others; k++) {
    const uint8_t* img = c->others[k];
    const float* Wm = c->warps[k];
    const uint16_t* wq = c->wq[k];
    int iw = c->ow[k], ih = c->oh[k];
    int x0 = 1, y0 = 1, x1 = iw - 2, y1 = ih - 2;
    int lix = INT_MIN, liy = 0, lhx = 0, lhy = 0, lastCost = 0, haveLast = 0;
    for (int d = 0; d < count; d++) {
      float fx, fy;
      project(Wm, xf, yf, c->planes[start + d], &fx, &fy);
      int ix, iy, hx, hy;
      if (d == 0) {
        float cx = cs_minf(cs_maxf(fx, (float)x0), (float)(x1 - 1)), cy = cs_minf(cs_maxf(fy, (float)y0), (float)(y1 - 1));
        ix = cs_f2i(cx); iy = cs_f2i(cy); hx = cs_f2i(cx + cx) & 1; hy = cs_f2i(cy + cy) & 1;
        if (ix < x0 || ix >= x1 || iy < y0 || iy >= y1) return lo_matching_cost_scalar(c, x, y, start, count, cost);
      } else {
        ix = cs_f2i(fx); iy = cs_f2i(fy); hx = cs_f2i(fx + fx) & 1; hy = cs_f2i(fy + fy) & 1;
        if (haveLast && ix == lix && iy == liy && hx == lhx && hy == lhy) { cost[d] = (uint16_t)(cost[d] + lastCost); continue; }
        if (ix < x0 || ix >= x1 || iy < y0 || iy >= y1) { cost[d] = (uint16_t)(cost[d] + lastCost); continue; }
      }
      int costK = block_cost_vec(img, iw, ix, iy, hx, hy, rb, wq);
      cost[d] = (uint16_t)(cost[d] + costK);
      lix = ix; liy = iy; lhx = hx; lhy = hy; lastCost = costK; haveLast = 1;
    }
  }
  return LO_OK;
}

int lo_matching_cost_scalar(const lo_costctx* c, int x, int y, int start, int count, uint16_t* cost) {
  if (start < 0 || count < 0 || start + count > c->n_planes) return LO_ERR_INDEX;
  memset(cost, 0, sizeof(uint16_t) * (size_t)count);
  uint8_t refBlock[3 * 12];
  for (int r = -1; r <= 1; r++) {
    int yy = iclamp(y + r, 0, c->h - 1);
    for (int cc = -1; cc <= 1; cc++) {
      int xx = iclamp(x + cc, 0, c->w - 1);
      for (int ch = 0; ch < 4; ch++) refBlock[(r + 1) * 12 + (cc + 1) * 4 + ch] = c->ref[((size_t)yy * c->w + xx) * 4 + ch];
    }
  }
  for (int k = 0; k < c->n_others; k++) {
    const uint8_t* img = c->others[k];
    const float* Wm = c->warps[k];
    const uint16_t* wq = c->wq[k];
    int iw = c->ow[k], ih = c->oh[k];
    int x0 = 1, y0 = 1, x1 = iw - 2, y1 = ih - 2;
    int lix = INT_MIN, liy = 0, lhx = 0, lhy = 0, lastCost = 0, haveLast = 0;
    for (int d = 0; d < count; d++) {
      float fx, fy;
      project(Wm, (float)x, (float)y, c->planes[start + d], &fx, &fy);
      int ix, iy, hx, hy;
      if (d == 0) {
        float cx = cs_minf(cs_maxf(fx, (float)x0), (float)(x1 - 1)), cy = cs_minf(cs_maxf(fy, (float)y0), (float)(y1 - 1));
        ix = cs_f2i(cx); iy = cs_f2i(cy); hx = cs_f2i(cx + cx) & 1; hy = cs_f2i(cy + cy) & 1;
      } else {
        ix = cs_f2i(fx); iy = cs_f2i(fy); hx = cs_f2i(fx + fx) & 1; hy = cs_f2i(fy + fy) & 1;
        if (haveLast && ix == lix && iy == liy && hx == lhx && hy == lhy) { cost[d] = (uint16_t)(cost[d] + lastCost); continue; }
        if (ix < x0 || ix >= x1 || iy < y0 || iy >= y1) { cost[d] = (uint16_t)(cost[d] + lastCost); continue; }
      }
      uint8_t T[64];
      for (int q = 0; q < 4; q++) {
        int yy = iy - 1 + q;
        for (int pI = 0; pI < 4; pI++) {
          int xx = ix - 1 + pI;
          if (yy < 0 || yy >= ih || xx < 0 || xx >= iw) return LO_ERR_INDEX;
          for (int ch = 0; ch < 4; ch++) T[q * 16 + pI * 4 + ch] = img[((size_t)yy * iw + xx) * 4 + ch];
        }
      }
      int A[8] = {0}, Bw[8] = {0};
      for (int q = 0; q < 3; q++) {
        uint8_t row[16];
        for (int b = 0; b < 16; b++) row[b] = hy ? pavgb(T[q * 16 + b], T[(q + 1) * 16 + b]) : T[q * 16 + b];
        if (hx) {
          for (int b = 0; b < 12; b++) row[b] = pavgb(row[b], row[b + 4]);
          for (int b = 12; b < 16; b++) row[b] = pavgb(row[b], 0);
        }
        for (int b = 0; b < 16; b++) {
          int rbv = b < 12 ? refBlock[q * 12 + b] : 0;
          int diff = imax(row[b], rbv) - imin(row[b], rbv);
          int dd = imin(diff, (int)kCaps[b & 3]);
          if (b < 8) A[b] = imin(A[b] + dd, 65535); else Bw[b - 8] = imin(Bw[b - 8] + dd, 65535);
        }
      }
      int S[4];
      for (int ch = 0; ch < 4; ch++) {
        int s0 = imin(A[ch] + Bw[ch], 65535), s1 = imin(A[4 + ch] + 0, 65535);
        S[ch] = imin(s0 + s1, 65535);
      }
      int cY = (S[0] * wq[0] + 16) >> 5, cU = (S[1] * wq[1] + 16) >> 5, cV = (S[2] * wq[2] + 16) >> 5, cA = (S[3] * wq[3] + 16) >> 5;
      int ck = (cY + cU) + (cV + cA);
      float cf = cs_minf((float)ck, 65535.0f);
      int costK = cs_f2i(cf);
      cost[d] = (uint16_t)(cost[d] + costK);
      lix = ix; liy = iy; lhx = hx; lhy = hy; lastCost = costK; haveLast = 1;
    }
  }
  return LO_OK;
}

void lo_normalise(const uint16_t* cost, int count, int cap, int n_others, uint8_t* raw) {
  float f = ffrom(0x3d17b426u) / (float)n_others;
  for (int d = 0; d < count; d++) raw[d] = (uint8_t)cs_f2i((float)cost[d] * f);
  for (int d = count; d < cap; d++) raw[d] = 255;
}

/* ---------------- SkipMask (DenseStereoSgm.cs:65-87) ---------------- */
int lo_skip_mask(int mode, int w, int h, uint8_t* m) {
  memset(m, 0, (size_t)w * h);
  if (mode == 0) return LO_OK;
  if (mode != 2) return LO_ERR_SKIPMODE;
  memset(m, 0xff, (size_t)w * h);
  int nx = w / 64 + (64 < 2 * (w % 64) ? 1 : 0), ny = h / 64 + (64 < 2 * (h % 64) ? 1 : 0);
  if (nx < 1) nx = 1;
  if (ny < 1) ny = 1;
  lo_mt19937 mt;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      int x0 = 64 * i, x1 = imin(w, x0 + 64 * (i == nx - 1 ? 2 : 1)), y0 = 64 * j, y1 = imin(h, y0 + 64 * (j == ny - 1 ? 2 : 1));
      lo_mt_seed(&mt, 5489u);
      for (int y = y0; y < y1; y += 2)
        for (int x = x0; x < x1; x += 2) {
          int dy = (int)(lo_mt_next(&mt) & 1), dx = (int)(lo_mt_next(&mt) & 1);
          int yy = y + dy, xx = x + dx;
          if (xx >= 0 && xx < w && yy >= 0 && yy < h) m[(size_t)yy * w + xx] = 0;
        }
    }
  return LO_OK;
}

/* ---------------- RangeFromPrevious (DenseStereoSgm.cs:91-140) ---------------- */
static int range_from_previous(lo_layer* L, const lo_layer* prev) {
  int n = L->n_planes, pw = prev->w, ph = prev->h;
  float* b = (float*)malloc(sizeof(float) * (size_t)n);
  uint16_t* idx = (uint16_t*)malloc(sizeof(uint16_t) * (size_t)pw * ph);
  uint16_t *hmin = (uint16_t*)malloc(2 * (size_t)pw * ph), *hmax = (uint16_t*)malloc(2 * (size_t)pw * ph);
  uint16_t *vmin = (uint16_t*)malloc(2 * (size_t)pw * ph), *vmax = (uint16_t*)malloc(2 * (size_t)pw * ph);
  if (!b || !idx || !hmin || !hmax || !vmin || !vmax) { free(b); free(idx); free(hmin); free(hmax); free(vmin); free(vmax); return LO_ERR_ALLOC; }
  for (int i = 0; i < n - 1; i++) b[i] = (lo_rcp(L->planes[i + 1]) + lo_rcp(L->planes[i])) * 0.5f;
  b[n - 1] = 3.40282347e+38f;
  for (int i = 0; i < pw * ph; i++) {
    float v = lo_rcp(prev->depth[i]);
    int c = 0;
    while (c < n && b[c] <= v) c++;
    idx[i] = (uint16_t)c;
  }
  for (int y = 0; y < ph; y++)
    for (int x = 0; x < pw; x++) {
      uint16_t mn = 0xffff, mx = 0;
      for (int k = -1; k <= 2; k++) {
        int xx = iclamp(x + k, 0, pw - 1);
        if (prev->skip[y * pw + xx] > 0) continue; /* valid = computed pixels only */
        uint16_t v = idx[y * pw + xx];
        if (v < mn) mn = v;
        if (v > mx) mx = v;
      }
      hmin[y * pw + x] = mn; hmax[y * pw + x] = mx;
    }
  for (int y = 0; y < ph; y++)
    for (int x = 0; x < pw; x++) {
      uint16_t mn = 0xffff, mx = 0;
      for (int k = -1; k <= 2; k++) {
        int yy = iclamp(y + k, 0, ph - 1);
        uint16_t a = hmin[yy * pw + x], c = hmax[yy * pw + x];
        if (a < mn) mn = a;
        if (c > mx) mx = c;
      }
      vmin[y * pw + x] = mn; vmax[y * pw + x] = mx;
    }
  float fy = (float)(ph - 1) / (float)(L->h - 1), fx = (float)(pw - 1) / (float)(L->w - 1);
  int maxHi = 0, minLo = INT_MAX;
  for (int y = 0; y < L->h; y++) {
    int py = cs_f2i((float)y * fy);
    for (int x = 0; x < L->w; x++) {
      int px = cs_f2i((float)x * fx);
      if (py < 0 || py >= ph || px < 0 || px >= pw) { free(b); free(idx); free(hmin); free(hmax); free(vmin); free(vmax); return LO_ERR_INDEX; }
      int lo = imax(0, vmin[py * pw + px] - L->p.margin), hi = imin(n - 1, vmax[py * pw + px] + 1);
      int i = y * L->w + x;
      L->start[i] = (uint16_t)lo;
      L->count[i] = (uint16_t)(hi - lo);
      maxHi = imax(maxHi, hi & 0xffff);
      minLo = imin(minLo, lo & 0xffff);
    }
  }
  L->max_hi = maxHi;
  L->min_lo = minLo;
  free(b); free(idx); free(hmin); free(hmax); free(vmin); free(vmax);
  return LO_OK;
}

/* ---------------- DenseLayer.Init (DenseStereoSgm.cs:34-62) ---------------- */
int lo_layer_init(lo_layer* L, const lo_params* p, int index, int n_cams, const uint8_t* const* images, const int* iw, const int* ih,
                  const uint8_t* gray, const lo_calib* calibs, float near_, float far_, int align, const lo_layer* prev) {
  memset(L, 0, sizeof(*L));
  L->p = *p;
  L->index = index;
  L->align = align;
  L->w = (iw[0] + p->scale - 1) / p->scale;
  L->h = (ih[0] + p->scale - 1) / p->scale;
  L->planes = (float*)malloc(sizeof(float) * (4096 + (size_t)align + 8));
  int rc = lo_planes(near_, far_, calibs, n_cams, p->plane_density, align, L->planes, &L->n_planes);
  if (rc) return rc;
  int w = L->w, h = L->h, n = L->n_planes;
  size_t npx = (size_t)w * h;
  L->guidance = (uint8_t*)malloc(npx * 4);
  lo_guidance(images[0], iw[0], ih[0], w, h, p->scale, L->guidance);
  L->skip = (uint8_t*)malloc(npx);
  rc = lo_skip_mask(p->skip_mode, w, h, L->skip);
  if (rc) return rc;
  L->start = (uint16_t*)calloc(npx, 2);
  L->count = (uint16_t*)calloc(npx, 2);
  L->cap = (uint16_t*)calloc(npx, 2);
  if (!prev) {
    for (size_t i = 0; i < npx; i++) { L->start[i] = 0; L->count[i] = (uint16_t)n; L->cap[i] = (uint16_t)n; }
    L->min_lo = 0;
    L->max_hi = ((n + align - 1) / align) * align;
  } else {
    rc = range_from_previous(L, prev);
    if (rc) return rc;
    L->max_hi = ((L->max_hi + align - 1) / align) * align;
  }
  L->off = (uint64_t*)malloc(sizeof(uint64_t) * (npx + 1));
  uint64_t tot = 0;
  for (size_t i = 0; i < npx; i++) {
    int cap = ((L->count[i] + align - 1) / align) * align;
    L->cap[i] = (uint16_t)cap;
    L->off[i] = tot;
    tot += (uint64_t)cap;
  }
  L->off[npx] = tot;
  L->agg = (uint16_t*)calloc(tot + 1, 2);
  L->raw = (uint8_t*)calloc(tot + 1, 1);
  L->n_cams = n_cams;
  L->images = images; L->iw = iw; L->ih = ih;
  L->warps = (float (*)[16])malloc(sizeof(float[16]) * (size_t)(n_cams > 1 ? n_cams - 1 : 1));
  L->wq = (uint16_t (*)[4])malloc(sizeof(uint16_t[4]) * (size_t)(n_cams > 1 ? n_cams - 1 : 1));
  for (int k = 1; k < n_cams; k++) {
    lo_flow_matrix(&calibs[0], &calibs[k], L->warps[k - 1]);
    static const uint16_t wg[4] = {12240, 0, 0, 0}, wc[4] = {8160, 680, 680, 0};
    memcpy(L->wq[k - 1], gray[k] ? wg : wc, sizeof(wg));
  }
  if (!L->planes || !L->guidance || !L->skip || !L->start || !L->agg || !L->raw) return LO_ERR_ALLOC;
  return LO_OK;
}

void lo_layer_free(lo_layer* L) {
  free(L->planes); free(L->guidance); free(L->skip); free(L->start); free(L->count); free(L->cap); free(L->off);
  free(L->agg); free(L->agg_pass1); free(L->raw); free(L->depth); free(L->warps); free(L->wq);
  memset(L, 0, sizeof(*L));
}

/* ---------------- MemoryEstimate (DenseStereoSgm.cs:144-156) ---------------- */
int lo_memory_estimate(const lo_params* p, int n_cams, const int* iw, const int* ih, const lo_calib* calibs, float near_, float far_,
                       int align, const lo_layer* prev, int64_t* out) {
  lo_layer L;
  memset(&L, 0, sizeof(L));
  L.p = *p;
  L.align = align;
  L.w = (iw[0] + p->scale - 1) / p->scale;
  L.h = (ih[0] + p->scale - 1) / p->scale;
  float planes[4096 + 16];
  L.planes = planes;
  int rc = lo_planes(near_, far_, calibs, n_cams, p->plane_density, align, planes, &L.n_planes);
  if (rc) return rc;
  size_t npx = (size_t)L.w * L.h;
  uint8_t* skip = (uint8_t*)malloc(npx);
  rc = lo_skip_mask(p->skip_mode, L.w, L.h, skip);
  if (rc) { free(skip); return rc; }
  L.start = (uint16_t*)calloc(npx, 2);
  L.count = (uint16_t*)calloc(npx, 2);
  rc = range_from_previous(&L, prev);
  if (rc) { free(skip); free(L.start); free(L.count); return rc; }
  int64_t maxHi = ((L.max_hi + align - 1) / align) * align;
  int64_t cost = 0;
  for (size_t i = 0; i < npx; i++) {
    int cap = ((L.count[i] + align - 1) / align) * align;
    cost += 8 + (int64_t)cap * (skip[i] == 0 ? 3 : 2);
  }
  int64_t w = L.w, h = L.h, imgs = 0;
  for (int k = 0; k < n_cams; k++) imgs += (int64_t)ih[k] * iw[k] * 4;
  *out = cost + w * h * 4 + 20 * (2 * w + 4) + 2 * ((4LL * maxHi + 5) * (2 * w + 4) + 8 * w + 16) + imgs + w * h * 8;
  free(skip); free(L.start); free(L.count);
  return LO_OK;
}

/* ---------------- DenseLayer.Compute / Pixel (DenseStereoSgm.cs:158-324) ---------------- */
typedef struct {
  lo_layer* L;
  uint16_t* Lb; size_t Llen;   /* _L */
  uint16_t* Min;               /* _Min */
  uint16_t *RangeS, *RangeC;   /* _RangeS, _RangeC */
  float (*Pix)[4];             /* _Pix */
  int slotStride, halfL, halfM, halfR;
  uint8_t* rawTmp;             /* the shared scratch `raw` of Compute (n + 8 bytes) */
  int err;
  const lo_costctx* cctx;      /* inline_cost: the cost context and the `costTmp` scratch of Compute */
  uint16_t* costTmp;
} sgm_state;

static inline int lidx(const sgm_state* s, int half, int slot, int path) {
  return half * s->halfL + slot * s->slotStride + 1 + path * (s->L->max_hi + 1);
}
/* The reference runs Pixel's 8-lane vector form (DenseStereoSgm.cs:280-299) where its guard holds and the scalar form
   (:300-313) elsewhere; both give the same values there, since the guard keeps the block loads clear of the stores.
   The oracle takes the scalar form unless lo_set_vector_form(1), which restates the vector form too, so a test can
   check the two against each other; lo_vector_calls() counts the path blocks that took it. */
static int g_vector_form = 0;
static long g_vector_calls = 0;
void lo_set_vector_form(int on) { g_vector_form = on; g_vector_calls = 0; }
long lo_vector_calls(void) { return g_vector_calls; }
static inline int sat16(int v) { return v > 65535 ? 65535 : v; }

/* Rd (DenseStereoSgm.cs:324): before the buffer 2000, past its end 0 */
static inline int rd(const sgm_state* s, long i) { return i < 0 ? 2000 : (size_t)i < s->Llen ? s->Lb[i] : 0; }

static void pixel(sgm_state* s, int x, int y, int dir, int cur, int other) {
  lo_layer* L = s->L;
  int W = L->w;
  int pi = y * W + x, slot = x + 1;
  const uint8_t* gb = L->guidance + (size_t)pi * 4;
  float g[4] = {(float)gb[0], (float)gb[1], (float)gb[2], (float)gb[3]};
  memcpy(s->Pix[cur * s->halfR + slot], g, sizeof(g));
  int start = L->start[pi], count = L->count[pi], cap = L->cap[pi];
  uint8_t* raw = s->rawTmp;
  if (L->skip[pi] != 0) {
    memset(raw, 0, (size_t)cap);
    for (int k = count; k < cap; k++) raw[k] = 255;
  } else if (dir > 0 && s->cctx) { /* Threads == 1: pass +1 computes the costs at every visit and stores them (:243-249) */
    int W0 = L->iw[0], H0 = L->ih[0], sc = L->p.scale, hf = (sc + (sc >> 31)) >> 1;
    int xImg = imin(sc * x + hf, W0 - 1), yImg = imin(sc * y + hf, H0 - 1);
    int rc = lo_matching_cost(s->cctx, xImg, yImg, start, count, s->costTmp);
    if (rc) { s->err = rc; return; }
    lo_normalise(s->costTmp, count, cap, s->cctx->n_others, raw);
    memcpy(L->raw + L->off[pi], raw, (size_t)cap);
  } else {
    memcpy(raw, L->raw + L->off[pi], (size_t)cap); /* the stored costs (prepass == pass-1 costs, :176-180) */
  }
  int sp = s->RangeS[cur * s->halfR + slot], cp = s->RangeC[cur * s->halfR + slot];
  uint16_t* agg = L->agg + L->off[pi];
  int P1 = L->p.p1;
  float p2Base = (float)L->p.p1 * L->p.p2scale;
  const float* gw = L->p.guidance;
  const float E3 = ffrom(0x3d9fcb52u), E2 = ffrom(0x3e677e26u), E1 = ffrom(0x3f322226u), E0 = ffrom(0x3f7ffb19u);
  for (int p = 0; p < 4; p++) {
    int baseCur = lidx(s, cur, slot, p);
    {
      long q0 = sp - L->min_lo, k0 = q0 < 0 ? -q0 : 0;
      long k1 = cp < (long)s->Llen - baseCur - q0 ? cp : (long)s->Llen - baseCur - q0;
      for (long k = k0; k < k1; k++) s->Lb[baseCur + q0 + k] = 2000;
    }
    int ns = slot + (p == 2 ? 0 : p == 3 ? dir : -dir);
    int half = p == 0 ? cur : other;
    int minPrev = s->Min[half * s->halfM + ns * 4 + p];
    const float* pn = s->Pix[half * s->halfR + ns];
    float d0 = (g[0] - pn[0]) * gw[0], d1 = (g[1] - pn[1]) * gw[1], d2 = (g[2] - pn[2]) * gw[2];
    float S = (fabsf(d0) + fabsf(d2)) + fabsf(d1);
    float e = cs_maxf(cs_minf(-S, 128.0f), -126.0f);
    int ei = cs_f2i(e) + (e < 0.0f ? -1 : 0);
    float f = e - (float)ei;
    float poly = ((E3 * f + E2) * f + E1) * f + E0;
    float E = ffrom(fbits(poly) + ((uint32_t)ei << 23));
    int P2 = cs_f2i(p2Base * E);
    int P2p = imin(P2 + minPrev, 65535);
    if (cap == 0) { s->Min[cur * s->halfM + slot * 4 + p] = 0xffff; continue; }
    int nb = lidx(s, half, ns, p);
    int runMin = 0xffff;
    int q = start - L->min_lo;
    /* the 8-lane form (DenseStereoSgm.cs:280-299): whole blocks, every neighbour read and every write inside the buffer,
       the written range clear of the range read, a P2 term that fits 16 bits */
    if (g_vector_form && (cap & 7) == 0 && P2p >= 0 && (long)nb + q - 1 >= 0 && (size_t)((long)nb + q + cap + 1) <= s->Llen &&
        (long)baseCur + q >= 0 && (size_t)((long)baseCur + q + cap) <= s->Llen && labs((long)baseCur - nb) >= cap + 16) {
      const uint16_t* pn = s->Lb + nb + q;
      uint16_t* pw = s->Lb + baseCur + q;
      uint16_t vrun[8];
      for (int l = 0; l < 8; l++) vrun[l] = 0xffff;
      for (int b = 0; b < cap; b += 8) {
        uint16_t lm[8], l0[8], lp[8], lc[8];
        memcpy(lm, pn + b - 1, sizeof lm); /* Vector128.Load of the three neighbour blocks, before the block's store */
        memcpy(l0, pn + b, sizeof l0);
        memcpy(lp, pn + b + 1, sizeof lp);
        for (int l = 0; l < 8; l++) {
          int m = imin(imin(sat16(lm[l] + P1), l0[l]), imin(sat16(lp[l] + P1), P2p)); /* Min(Min(AddSat(Lm,P1),L0), Min(AddSat(Lp,P1),P2)) */
          int v = sat16(raw[b + l] + m) - minPrev;                                        /* SubtractSaturate(AddSaturate(r16, m), minPrev) */
          lc[l] = (uint16_t)(v < 0 ? 0 : v);
        }
        memcpy(pw + b, lc, sizeof lc);
        for (int l = 0; l < 8; l++) {
          if (lc[l] < vrun[l]) vrun[l] = lc[l];
          agg[b + l] = (uint16_t)sat16(agg[b + l] + lc[l]);
        }
      }
      for (int l = 0; l < 8; l++) runMin = imin(runMin, vrun[l]);
      g_vector_calls++;
      s->Min[cur * s->halfM + slot * 4 + p] = (uint16_t)runMin;
      continue;
    }
    /* the scalar form: every read through Rd, lanes in order (DenseStereoSgm.cs:300-313) */
    for (int b = 0; b < cap; b += 8)
      for (int l = 0; l < 8; l++) {
        long qi = (long)q + b + l;
        int Lm = rd(s, nb + qi - 1), Lp = rd(s, nb + qi + 1), L0 = rd(s, nb + qi);
        int m = imin(imin(imin(Lm + P1, 65535), L0), imin(imin(Lp + P1, 65535), P2p));
        int lc = imin(raw[b + l] + m, 65535) - minPrev;
        if (lc < 0) lc = 0;
        long wi = baseCur + qi;
        if (wi < 0 || (size_t)wi >= s->Llen) { s->err = LO_ERR_INDEX; return; }
        s->Lb[wi] = (uint16_t)lc;
        if (lc < runMin) runMin = lc;
        if (b + l >= cap) { s->err = LO_ERR_INDEX; return; } /* agg[b + l] past the pixel's cap */
        agg[b + l] = (uint16_t)imin(agg[b + l] + lc, 65535);
      }
    s->Min[cur * s->halfM + slot * 4 + p] = (uint16_t)runMin;
  }
  s->RangeS[cur * s->halfR + slot] = (uint16_t)start;
  s->RangeC[cur * s->halfR + slot] = (uint16_t)cap;
}

/* raw costs of every computed pixel, rows in parallel on `threads` workers (DenseStereoSgm.cs:186-205); pass 1 then reads
   them like pass 2 does, which the reference states gives the same values and aggregation order (:176-180) */
typedef struct {
  lo_layer* L;
  lo_costctx c;
  int next_row;
  int err;
  pthread_mutex_t mu;
} raw_job;

static void* raw_worker(void* arg) {
  raw_job* j = (raw_job*)arg;
  lo_layer* L = j->L;
  int W = L->w, H = L->h, W0 = L->iw[0], H0 = L->ih[0], sc = L->p.scale, half = (sc + (sc >> 31)) >> 1;
  uint16_t* cost = (uint16_t*)malloc(sizeof(uint16_t) * ((size_t)L->n_planes + 8));
  uint8_t* raw = (uint8_t*)malloc((size_t)L->n_planes + 8 + 65536);
  for (;;) {
    pthread_mutex_lock(&j->mu);
    int y = j->next_row++;
    pthread_mutex_unlock(&j->mu);
    if (y >= H) break;
    for (int x = 0; x < W; x++) {
      int pi = y * W + x;
      if (L->skip[pi] != 0) continue;
      int start = L->start[pi], count = L->count[pi], cap = L->cap[pi];
      int xImg = imin(sc * x + half, W0 - 1), yImg = imin(sc * y + half, H0 - 1);
      int rc = lo_matching_cost(&j->c, xImg, yImg, start, count, cost);
      if (rc) {
        pthread_mutex_lock(&j->mu);
        j->err = rc;
        pthread_mutex_unlock(&j->mu);
        continue;
      }
      lo_normalise(cost, count, cap, j->c.n_others, raw);
      memcpy(L->raw + L->off[pi], raw, (size_t)cap);
    }
  }
  free(cost);
  free(raw);
  return NULL;
}

static void compute_raw(lo_layer* L, int* err) {
  raw_job j;
  memset(&j, 0, sizeof(j));
  j.L = L;
  j.c.ref = L->images[0]; j.c.w = L->iw[0]; j.c.h = L->ih[0];
  j.c.n_others = L->n_cams - 1;
  j.c.others = L->images + 1; j.c.ow = L->iw + 1; j.c.oh = L->ih + 1;
  j.c.warps = (const float (*)[16])L->warps; j.c.wq = (const uint16_t (*)[4])L->wq;
  j.c.planes = L->planes; j.c.n_planes = L->n_planes;
  pthread_mutex_init(&j.mu, NULL);
  int nt = L->threads > 1 ? L->threads : 1;
  if (nt == 1) {
    raw_worker(&j);
  } else {
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nt);
    for (int t = 0; t < nt; t++) pthread_create(&th[t], NULL, raw_worker, &j);
    for (int t = 0; t < nt; t++) pthread_join(th[t], NULL);
    free(th);
  }
  pthread_mutex_destroy(&j.mu);
  if (j.err) *err = j.err;
}

int lo_layer_compute(lo_layer* L) {
  int err = 0;
  lo_costctx cctx;
  memset(&cctx, 0, sizeof(cctx));
  if (!L->inline_cost) {
    compute_raw(L, &err);
    if (err) return err;
  } else {
    cctx.ref = L->images[0]; cctx.w = L->iw[0]; cctx.h = L->ih[0];
    cctx.n_others = L->n_cams - 1;
    cctx.others = L->images + 1; cctx.ow = L->iw + 1; cctx.oh = L->ih + 1;
    cctx.warps = (const float (*)[16])L->warps; cctx.wq = (const uint16_t (*)[4])L->wq;
    cctx.planes = L->planes; cctx.n_planes = L->n_planes;
  }
  sgm_state s;
  memset(&s, 0, sizeof(s));
  s.L = L;
  if (L->inline_cost) {
    s.cctx = &cctx;
    s.costTmp = (uint16_t*)malloc(sizeof(uint16_t) * ((size_t)L->n_planes + 8));
  }
  int W = L->w, H = L->h, T = L->p.tile;
  int maxCnt = L->max_hi;
  s.slotStride = 4 * maxCnt + 5;
  int slots = W + 2;
  s.halfL = slots * s.slotStride;
  s.Llen = (size_t)2 * s.halfL;
  s.Lb = (uint16_t*)malloc(sizeof(uint16_t) * s.Llen);
  for (size_t i = 0; i < s.Llen; i++) s.Lb[i] = 2000;
  s.halfM = slots * 4;
  s.Min = (uint16_t*)malloc(sizeof(uint16_t) * 2 * (size_t)s.halfM);
  for (int i = 0; i < 2 * s.halfM; i++) s.Min[i] = 2000;
  s.halfR = slots;
  s.RangeS = (uint16_t*)calloc(2 * (size_t)slots, 2);
  s.RangeC = (uint16_t*)malloc(sizeof(uint16_t) * 2 * (size_t)slots);
  for (int i = 0; i < 2 * slots; i++) s.RangeC[i] = (uint16_t)L->align;
  s.Pix = (float (*)[4])calloc(2 * (size_t)slots, sizeof(float[4]));
  s.rawTmp = (uint8_t*)calloc((size_t)L->n_planes + 8 + 65536, 1);
  static const int dirs[2] = {1, -1};
  for (int di = 0; di < 2 && !s.err; di++) {
    int dir = dirs[di];
    int gwN = (W + T + T - 1) / T, ghN = (H + T - 1) / T;
    for (int j = 0; j < ghN && !s.err; j++)
      for (int i = 0; i < gwN && !s.err; i++) {
        int x0 = dir > 0 ? i * T : W - 1 - i * T, y0 = dir > 0 ? j * T : H - 1 - j * T;
        int yEnd = iclamp(y0 + dir * T, -1, H);
        for (int r = 0;; r++) {
          int y = y0 + dir * r;
          if (y == yEnd) break;
          int xs = iclamp(x0 - dir * r, 0, (L->xsw && dir > 0) ? W : W - 1), xe = iclamp(x0 + dir * (T - r), -1, W);
          if (xs == xe) continue;
          int cur = (r & 1) == 0 ? 1 : 0, other = 1 - cur;
          for (int x = xs; x != xe && !s.err; x += dir) pixel(&s, x, y, dir, cur, other);
        }
      }
    if (dir > 0 && L->keep_pass1) {
      L->agg_pass1 = (uint16_t*)malloc(sizeof(uint16_t) * (L->off[(size_t)W * H] + 1));
      memcpy(L->agg_pass1, L->agg, sizeof(uint16_t) * L->off[(size_t)W * H]);
    }
  }
  free(s.Lb); free(s.Min); free(s.RangeS); free(s.RangeC); free(s.Pix); free(s.rawTmp); free(s.costTmp);
  if (s.err) return s.err;
  /* WTA (DenseStereoSgm.cs:225-231) */
  L->depth = (float*)malloc(sizeof(float) * (size_t)W * H);
  for (size_t i = 0; i < (size_t)W * H; i++) {
    const uint16_t* agg = L->agg + L->off[i];
    int cnt = L->count[i];
    uint16_t best = 0xffff;
    int arg = 0;
    for (int k = 0; k < cnt; k++)
      if (agg[k] < best) { best = agg[k]; arg = k; }
    int pl = (uint16_t)(L->start[i] + arg);
    if (pl >= L->n_planes) return LO_ERR_INDEX;
    L->depth[i] = L->planes[pl];
  }
  return LO_OK;
}

/* ---------------- DenseStereoPyramid.Run (DenseStereoSgm.cs:331-353) ---------------- */
int lo_pyramid_run(int n_cams, const uint8_t* const* images, const int* iw, const int* ih, const uint8_t* gray,
                   const lo_calib* calibs, float near_, float far_, int threads, int keep_pass1, lo_layer layers[6]) {
  lo_params pars[6];
  lo_l16_pyramid(pars);
  uint8_t** filtered = (uint8_t**)calloc((size_t)n_cams, sizeof(uint8_t*));
  for (int k = 0; k < n_cams; k++) {
    filtered[k] = (uint8_t*)malloc((size_t)iw[k] * ih[k] * 4);
    lo_box_filter3(images[k], iw[k], ih[k], filtered[k]);
  }
  memset(layers, 0, sizeof(lo_layer) * 6);
  const lo_layer* prev = NULL;
  int rc = LO_OK;
  for (int i = 0; i < 6; i++) {
    int align = 8;
    if (prev) {
      int64_t est8, est2;
      rc = lo_memory_estimate(&pars[i], n_cams, iw, ih, calibs, near_, far_, 8, prev, &est8);
      if (rc) break;
      if (est8 >= 0x40000000LL) {
        rc = lo_memory_estimate(&pars[i], n_cams, iw, ih, calibs, near_, far_, 2, prev, &est2);
        if (rc) break;
        if (est2 >= 0x40000000LL) { rc = LO_ERR_BUDGET; break; }
        align = 2;
      }
    }
    rc = lo_layer_init(&layers[i], &pars[i], i, n_cams, (const uint8_t* const*)filtered, iw, ih, gray, calibs, near_, far_, align, prev);
    if (rc) break;
    layers[i].threads = threads;
    layers[i].keep_pass1 = keep_pass1;
    rc = lo_layer_compute(&layers[i]);
    if (rc) break;
    prev = &layers[i];
  }
  /* the filtered images are owned by the layers' lifetime in the reference; here the caller receives copies */
  for (int i = 0; i < 6; i++) { layers[i].images = NULL; layers[i].iw = NULL; layers[i].ih = NULL; }
  for (int k = 0; k < n_cams; k++) free(filtered[k]);
  free(filtered);
  return rc;
}

/* ---------------- DenseUpsampleLayer (DenseUpsampleLayer.cs:35-218) ---------------- */
static float cubic_tap(float x) {
  const float sixth = ffrom(0x3e2aaaabu);
  float x2 = x * x, x3 = x2 * x;
  if (x < 1.0f) { float a = x3 * 9.0f; float b = x2 * (-15.0f); b = b + 6.0f; b = b + a; return b * sixth; }
  if (x < 2.0f) { float a = x3 * (-3.0f); float b = x2 * 15.0f; float c = x * (-24.0f); c = c + 12.0f; c = c + b; c = c + a; return c * sixth; }
  return 0.0f;
}

void lo_image_shift(const uint8_t* src, int W, int H, int stride, float sx, float sy, uint8_t* dst) {
  int ix = cs_f2i(floorf(sx)), iy = cs_f2i(floorf(sy));
  float tx = sx - (float)ix, ty = sy - (float)iy;
  float kx[4] = {cubic_tap(tx + 1.0f), cubic_tap(tx), cubic_tap(1.0f - tx), cubic_tap(2.0f - tx)};
  float ky[4] = {cubic_tap(ty + 1.0f), cubic_tap(ty), cubic_tap(1.0f - ty), cubic_tap(2.0f - ty)};
  float* rowBuf = (float*)malloc(sizeof(float) * ((size_t)W + 4) * 4);
  for (int y = 0; y < H; y++) {
    int r0 = y + iy - 1;
    int rows[4];
    for (int i = 0; i < 4; i++) { int ry = r0 + i; rows[i] = ry < 0 ? 0 : ry >= H ? H - 1 : ry; }
    for (int c = -2; c < W + 2; c++) {
      int cx = c < 0 ? 0 : c >= W ? W - 1 : c;
      int ob = (c + 2) * 4;
      for (int ch = 0; ch < 4; ch++) {
        float acc = (float)src[((size_t)rows[0] * stride + cx) * 4 + ch] * ky[0];
        for (int i = 1; i < 4; i++) {
          float t = (float)src[((size_t)rows[i] * stride + cx) * 4 + ch] * ky[i];
          acc = t + acc;
        }
        rowBuf[ob + ch] = acc;
      }
    }
    for (int x = 0; x < W; x++) {
      int b = (x + ix - 1 + 2) * 4;
      for (int ch = 0; ch < 4; ch++) {
        float v0 = rowBuf[b + ch], v1 = rowBuf[b + 4 + ch], v2 = rowBuf[b + 8 + ch], v3 = rowBuf[b + 12 + ch];
        float p3 = v3 * kx[3], p2 = v2 * kx[2], p1 = v1 * kx[1], p0 = v0 * kx[0];
        float s = (p3 + p2) + (p1 + p0);
        int q = cs_f2i(rintf(s));
        dst[((size_t)y * W + x) * 4 + ch] = (uint8_t)(q < 0 ? 0 : q > 255 ? 255 : q);
      }
    }
  }
  free(rowBuf);
}

void lo_nearest_resize(const uint8_t* src, int sw, int sh, int sstride, int W, int H, uint8_t* dst) {
  memset(dst, 0, (size_t)W * H * 4);
  if (W > 0 && H > 0) {
    int stepY = (int)((double)sh * 65536.0 / (double)H);
    int stepX = (int)((double)sw * 65536.0 / (double)W);
    int yAcc = 0;
    for (int y = 0; y < H; y++) {
      int sy = yAcc >> 16, xAcc = 0;
      for (int x = 0; x < W; x++) {
        int sx = xAcc >> 16;
        memcpy(dst + ((size_t)y * W + x) * 4, src + ((size_t)sy * sstride + sx) * 4, 4);
        xAcc += stepX;
      }
      yAcc += stepY;
    }
  }
}

void lo_inverse_depth(const float* src, size_t n, float* dst) {
  for (size_t i = 0; i < n; i++) dst[i] = lo_rcp(src[i]);
}

static inline float exp2_fast(float t) {
  const float C1 = ffrom(0x3d9fcb52u), C2 = ffrom(0x3e677e26u), C3 = ffrom(0x3f322226u), C4 = ffrom(0x3f7ffb19u);
  t = t < 128.0f ? t : 128.0f;
  t = t > -126.0f ? t : -126.0f;
  int n = cs_f2i(t) + ((int32_t)fbits(t) >> 31);
  float f = t - (float)n;
  float p = ((f * C1 + C2) * f + C3) * f + C4;
  return ffrom(fbits(p) + ((uint32_t)n << 23));
}

static inline float spatial_w(float f, int i) {
  float d = fabsf(f - (float)(i * 2));
  d = d < 1.0f ? d : 1.0f;
  return cs_f2i(d) == 0 ? 1.0f : ffrom(0x3eaaaaabu);
}

void lo_bilateral_upsample(const float* lo_, int lw, int lh, const uint8_t* guide, int W, int H, int gstride, const uint8_t* g2,
                           float sigma, float* outp) {
  float k = 0.5f / (sigma * sigma);
  const float eps = ffrom(0x322bcc77u);
  int wm1 = lw - 1, hm1 = lh - 1;
  for (int y = 0; y < H; y++) {
    int iy0 = (y - 1) / 2;
    float fy = (float)y + (-0.5f);
    for (int x = 0; x < W; x++) {
      const uint8_t* o = guide + ((size_t)y * gstride + x) * 4;
      float hr = o[0], hg = o[1], hb = o[2];
      int ix0 = (x - 1) / 2;
      float fx = (float)x + (-0.5f);
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
        int lrow = iy * lw;
        const uint8_t* q = g2 + ((size_t)iy * lw + ibx) * 4;
        float d0 = hr - (float)q[0], d1 = hg - (float)q[1], d2 = hb - (float)q[2];
        float s = d1 * d1 + (d2 * d2 + d0 * d0);
        float t = -(s * k);
        float w0 = (exp2_fast(t) + eps) * (wy * wx0);
        q = g2 + ((size_t)iy * lw + ix1) * 4;
        d0 = hr - (float)q[0]; d1 = hg - (float)q[1]; d2 = hb - (float)q[2];
        s = d1 * d1 + (d2 * d2 + d0 * d0);
        t = -(s * k);
        float w1 = (exp2_fast(t) + eps) * (wy * wx1);
        float v0 = lo_[lrow + ibx] * w0, v1 = lo_[lrow + ix1] * w1;
        accV = v1 + (v0 + accV);
        accS = w1 + (w0 + accS);
      }
      outp[(size_t)y * W + x] = accV / accS;
    }
  }
}

int lo_upsample(const float* prev_depth, int pw, int ph, const uint8_t* guide, int gw, int gh, int gstride, int set_w, int set_h,
                float sigma, int scale, const float* prev_conf, float* out_depth, float* out_conf) {
  uint8_t* shifted = (uint8_t*)malloc((size_t)gw * gh * 4);
  uint8_t* g2 = (uint8_t*)malloc((size_t)pw * ph * 4 + 4);
  float* inv = (float*)malloc(sizeof(float) * (size_t)pw * ph + 4);
  float* u = (float*)malloc(sizeof(float) * (size_t)gw * gh);
  lo_image_shift(guide, gw, gh, gstride, 0.5f, 0.5f, shifted);
  lo_nearest_resize(shifted, gw, gh, gw, pw, ph, g2);
  lo_inverse_depth(prev_depth, (size_t)pw * ph, inv);
  lo_bilateral_upsample(inv, pw, ph, guide, gw, gh, gstride, g2, sigma, u);
  lo_inverse_depth(u, (size_t)gw * gh, out_depth);
  int rc = LO_OK;
  if (gw != set_w * scale || gh != set_h * scale) rc = LO_ERR_UPSAMPLE_SIZE;
  else if (prev_conf && pw > 0 && ph > 0 && out_conf) lo_bilateral_upsample(prev_conf, pw, ph, guide, gw, gh, gstride, g2, sigma, out_conf);
  free(shifted); free(g2); free(inv); free(u);
  return rc;
}

/* ---------------- traversal replay (DenseStereoSgm.cs:206-224) ---------------- */
long lo_traversal_trace(int W, int H, int T, int xsw, int* ev, long max_events) {
  int slots = W + 2;
  long* last = (long*)malloc(sizeof(long) * 2 * (size_t)slots);
  for (int i = 0; i < 2 * slots; i++) last[i] = -1;
  uint8_t* seen = (uint8_t*)calloc((size_t)W * H, 1);
  long n = 0;
  static const int dirs[2] = {1, -1};
  for (int di = 0; di < 2; di++) {
    int dir = dirs[di];
    memset(seen, 0, (size_t)W * H);
    int gwN = (W + T + T - 1) / T, ghN = (H + T - 1) / T;
    for (int j = 0; j < ghN; j++)
      for (int i = 0; i < gwN; i++) {
        int x0 = dir > 0 ? i * T : W - 1 - i * T, y0 = dir > 0 ? j * T : H - 1 - j * T;
        int yEnd = iclamp(y0 + dir * T, -1, H);
        for (int r = 0;; r++) {
          int y = y0 + dir * r;
          if (y == yEnd) break;
          int xs = iclamp(x0 - dir * r, 0, (xsw && dir > 0) ? W : W - 1), xe = iclamp(x0 + dir * (T - r), -1, W);
          if (xs == xe) continue;
          int cur = (r & 1) == 0 ? 1 : 0, other = 1 - cur;
          for (int x = xs; x != xe; x += dir) {
            if (n >= max_events) { free(last); free(seen); return -1; }
            int slot = x + 1;
            int* e = ev + 9 * n;
            e[0] = dir; e[1] = x; e[2] = y; e[3] = r; e[4] = seen[(size_t)y * W + x] ? 1 : 0;
            seen[(size_t)y * W + x] = 1;
            for (int p = 0; p < 4; p++) {
              int ns = slot + (p == 2 ? 0 : p == 3 ? dir : -dir);
              int half = p == 0 ? cur : other;
              e[5 + p] = (int)last[half * slots + ns];
            }
            last[cur * slots + slot] = n;
            n++;
          }
        }
      }
  }
  free(last); free(seen);
  return n;
}

/* ---------------- depth image cache (Lux.Engine/Pipeline/Export/DepthCache.cs) ---------------- */

/* ImageResample0 (DepthCache.cs:38-70): nearest neighbour in 16.16 fixed point, int32 wrap-around, clamped to [0, n-1]. */
static int lo_nearest(int s16, int o16, int i, int n) {
  int v = (int32_t)((uint32_t)s16 * (uint32_t)i + (uint32_t)o16) >> 16;
  return v < 0 ? 0 : v > n - 1 ? n - 1 : v;
}

/* DepthImageCache.Set (DepthCache.cs:137-143): InverseDepth (rcpps, no Newton step), the nearest resample to the cache
 * dims (scale = src / dst in double, offset 0), then InverseDepthClip: minps(rcpps(x), 1e5). */
int lo_depth_cache_set(const float* src, int w, int h, int cw, int ch, float* out) {
  if (cw <= 0 || ch <= 0) return LO_ERR_EMPTY_IMAGE; /* ImageResample0.Run (DepthCache.cs:62) */
  if (w <= 0 || h <= 0) return LO_ERR_INDEX;          /* the resample clamps to index -1 of an empty source */
  if (!src || !out) return LO_ERR_ARG;
  const int sx16 = (int)((double)w / cw * 65536.0), sy16 = (int)((double)h / ch * 65536.0);
  const float clip = 100000.0f;
  for (int y = 0; y < ch; y++) {
    const int sy = lo_nearest(sy16, 0, y, h);
    for (int x = 0; x < cw; x++) {
      const int sx = lo_nearest(sx16, 0, x, w);
      const float inv = lo_rcp(src[(size_t)sy * w + sx]);
      const float r = lo_rcp(inv);
      out[(size_t)y * cw + x] = r < clip ? r : clip; /* minps(a, b): a when a < b, else b */
    }
  }
  return LO_OK;
}

/* DepthImageCache.Fetch (DepthCache.cs:160-183) on a dense iw x ih image with a full valid rect: the ROI check, the
 * plain view when the scale is 1, else the source window, its reciprocal (rcpps + one Newton step for the first
 * (vw/32)·32 columns, division for the rest), the nearest resample with the window offset, and the division back
 * (FetchFull / FetchSampled, :185-239, which give the same pixels). out holds (x1-x0)·(y1-y0) floats. */
int lo_depth_cache_fetch(const float* img, int iw, int ih, int x0, int y0, int x1, int y1, int dw, int dh, float* out) {
  const int rw = x1 - x0, rh = y1 - y0;
  if (rw == 0 || x1 < x0 || rh == 0 || y1 < y0 || (y0 | x0) < 0 || x1 > dw || y1 > dh) return LO_ERR_ROI;
  const double sx = (double)iw / dw, sy = (double)ih / dh;
  if (sx == 1.0 && sy == 1.0) {
    for (int y = 0; y < rh; y++)
      for (int x = 0; x < rw; x++) out[(size_t)y * rw + x] = img[(size_t)(y0 + y) * iw + x0 + x];
    return LO_OK;
  }
  int sx0 = (int)floor(x0 * sx), sy0 = (int)floor(y0 * sy);
  if (sx0 < 0) sx0 = 0;
  if (sy0 < 0) sy0 = 0;
  int sx1 = (int)ceil((rw + (double)x0) * sx), sy1 = (int)ceil((rh + (double)y0) * sy);
  if (sx1 > iw) sx1 = iw;
  if (sy1 > ih) sy1 = ih;
  const double offX = (double)((float)x0 + 0.5f) * sx - sx0, offY = (double)((float)y0 + 0.5f) * sy - sy0;
  const int vx0 = sx0, vy0 = sy0, vx1 = sx1, vy1 = sy1;
  const int vw = vx1 <= vx0 || vy1 <= vy0 ? 0 : vx1 - vx0, vh = vw == 0 ? 0 : vy1 - vy0;
  if (vw == 0) return LO_ERR_INDEX; /* an empty source window: the reference's resample would index outside it */
  const int ox16 = (int)(offX * 65536.0), oy16 = (int)(offY * 65536.0), sx16 = (int)(sx * 65536.0), sy16 = (int)(sy * 65536.0);
  const int vec = (vw / 32) * 32;
  for (int y = 0; y < rh; y++) {
    const int py = lo_nearest(sy16, oy16, y, vh);
    for (int x = 0; x < rw; x++) {
      const int px = lo_nearest(sx16, ox16, x, vw);
      const float v = img[(size_t)(vy0 + py) * iw + vx0 + px];
      float inv;
      if (px < vec) {
        const float r = lo_rcp(v);
        inv = ((1.0f - v * r) * r + r) * 1.0f;
      } else {
        inv = 1.0f / v;
      }
      out[(size_t)y * rw + x] = 1.0f / inv;
    }
  }
  return LO_OK;
}

/* ---------------- stereo-image formation after the ISP (StereoImage.cs, ReferenceGuide.cs) ---------------- */

/* WineCrt.Sindf / Cosdf (WineCrt.cs:24-45): Wine's ucrtbase Taylor kernels on a double argument. */
static float wine_sindf(double x) {
  double z = x * x;
  if (x > -0.007817583158612251 && 0.007817583158612251 > x) return (float)((z * -0.16666666666666666 + 1.0) * x);
  double s = x * z, w = z * z;
  double r = 2.7557319223985893e-06 * z - 0.0001984126984126984, q = z * 0.008333333333333333 - 0.16666666666666666;
  return (float)((w * s) * r + (q * s + x));
}
static float wine_cosdf(double x) {
  double z = x * x;
  if (x > -0.007816314697265625 && 0.007816314697265625 > x) return (float)(z * -0.5 + 1.0);
  double p = -2.755731922398589e-07 * z + 2.48015873015873e-05;
  p = p * z - 0.001388888888888889;
  p = p * z + 0.041666666666666664;
  p = p * z - 0.5;
  return (float)(p * z + 1.0);
}

/* WineCrt.Sinf (WineCrt.cs:77-99) for |x| below 2^28·π/2 (the Lanczos table needs |x| < 3π). */
float lo_wine_sinf(float x) {
  const double pio2 = 1.5707963267948966, pi = 3.141592653589793, three_pio2 = 4.71238898038469, two_pi = 6.283185307179586;
  uint32_t ix = fbits(x);
  int sign = (int)(ix >> 31);
  ix &= 0x7fffffffu;
  if (ix <= 0x3f490fdau) return ix < 0x39800000u ? x : wine_sindf(x);
  if (ix <= 0x407b53d1u) {
    double d = x;
    if (ix <= 0x4016cbe3u) return sign ? -wine_cosdf(d + pio2) : wine_cosdf(d - pio2);
    return wine_sindf(sign ? -(d + pi) : -(d - pi));
  }
  if (ix <= 0x40e231d5u) {
    double d = x;
    if (ix <= 0x40afeddfu) return sign ? wine_cosdf(d + three_pio2) : -wine_cosdf(d - three_pio2);
    return wine_sindf(sign ? d + two_pi : d - two_pi);
  }
  if (ix >= 0x7f800000u) return x - x;
  {
    /* musl __rem_pio2f, medium path */
    double fn = (double)x * 6.36619772367581382433e-01 + 6755399441055744.0 - 6755399441055744.0;
    double y = x - fn * 1.57079631090164184570e+00 - fn * 1.58932547735281966916e-08;
    int n = (int)fn;
    switch (n & 3) {
      case 0: return wine_sindf(y);
      case 1: return wine_cosdf(y);
      case 2: return wine_sindf(-y);
      default: return -wine_cosdf(y);
    }
  }
}

/* StereoImage.LanczosTable (StereoImage.cs:212-237): 64 phases x 6 taps of sinc(x)·sinc(x/3), normalised by the
 * sequential sum. */
void lo_lanczos_table(float tbl[384]) {
  const float step = ffrom(0x3c800000u), pi3 = ffrom(0x3f860a92u), pi = ffrom(0x40490fdbu), pi2 = ffrom(0x411de9e7u), three = 3.0f;
  for (int k = 0; k < 64; k++) {
    float p = (float)k * step, sum = 0.0f;
    for (int j = 0; j < 6; j++) {
      float x = p - (float)(j - 2), w;
      if (x == 0.0f) w = 1.0f;
      else if (fabsf(x) < three) {
        float s1 = lo_wine_sinf(x * pi), t = s1 * three, s2 = lo_wine_sinf(x * pi3);
        w = (s2 * t) / ((x * x) * pi2);
      } else w = 0.0f;
      tbl[k * 6 + j] = w;
      sum = sum + w;
    }
    float inv = 1.0f / sum;
    for (int j = 0; j < 6; j++) tbl[k * 6 + j] *= inv;
  }
}

/* (int)f as .NET 9+ converts: truncation, saturating, NaN -> 0. */
static int net_int(float f) {
  if (f != f) return 0;
  if (f >= 2147483648.0f) return INT32_MAX;
  if (f <= -2147483648.0f) return INT32_MIN;
  return (int)f;
}

/* The map of one destination pixel through an aligned calibration (StereoImage.cs:260-272): 64ths of a source pixel.
 * Returns 0, or -1 where the reference would index the lut below 0 (a subnormal r2 makes r = -inf). */
static int warp_map(const lo_aligned* a, int x, int y, int* px, int* py) {
  const float* H = a->H;
  float fx = (float)x, fy = (float)y;
  float Xn = H[2] + (H[0] * fx + H[1] * fy), Yn = H[5] + (H[3] * fx + H[4] * fy);
  float den = (H[7] * fy + H[6] * fx) + H[8], w = 1.0f / den;
  float dx = w * Xn - a->cx, dy = w * Yn - a->cy;
  float r2 = (a->sy * dy) * (a->sy * dy) + (a->sx * dx) * (a->sx * dx);
  float r;
  if (r2 == 0.0f) r = 0.0f;
  else {
    float rs = ffrom(lo_rsqrt_bits(fbits(r2)));
    float S = r2 * rs;
    r = ((S * rs) + (-3.0f)) * (S * (-0.5f));
  }
  int idx = net_int(r);
  if (idx >= 0x1000) idx = 0xfff;
  if (idx < 0) return -1;
  float lu = a->lut[idx];
  *px = net_int(((a->cx + (-2.0f)) + lu * dx) * 64.0f);
  *py = net_int(((a->cy + (-2.0f)) + dy * lu) * 64.0f);
  return 0;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }

int lo_warp_f32(const float* src, int sw, int sh, float gain, int dw, int dh, const lo_aligned* ac, float* dst) {
  if (sw < 1 || sh < 1 || dw < 0 || dh < 0 || !ac || !ac->lut) return LO_ERR_ARG;
  float tbl[384];
  lo_lanczos_table(tbl);
  memset(dst, 0, (size_t)dw * dh * 16);
  for (int y = 0; y < dh; y++)
    for (int x = 0; x < dw; x++) {
      int px, py;
      if (warp_map(ac, x, y, &px, &py)) return LO_ERR_INDEX;
      int i = px >> 6, fx = px & 63, j = py >> 6, fy = py & 63;
      int interior = i >= 0 && i <= sw - 6 && j >= 0 && j <= sh - 6;
      if (!interior && !(j < sh && j + 6 > 0 && i < sw && i + 6 > 0)) continue; /* fill 0 */
      const float *ty = tbl + fy * 6, *tx = tbl + fx * 6;
      int ro[6], co[6];
      for (int k = 0; k < 6; k++) {
        ro[k] = interior ? j + k : clampi(j + k, 0, sh - 1);
        co[k] = interior ? i + k : clampi(i + k, 0, sw - 1);
      }
      for (int c = 0; c < 4; c++) {
        float C[6];
        for (int cc = 0; cc < 6; cc++) {
          float P[6];
          for (int rr = 0; rr < 6; rr++) {
            float v = src[((size_t)ro[rr] * sw + co[cc]) * 4 + c];
            P[rr] = gain != 1.0f ? v * gain : v; /* the source scaled in place before the warp */
          }
          C[cc] = (P[5] * ty[5] + P[4] * ty[4]) + ((P[3] * ty[3] + P[2] * ty[2]) + (P[1] * ty[1] + P[0] * ty[0]));
        }
        dst[((size_t)y * dw + x) * 4 + c] = (C[5] * tx[5] + C[4] * tx[4]) + ((C[3] * tx[3] + C[2] * tx[2]) + (C[1] * tx[1] + C[0] * tx[0]));
      }
    }
  return LO_OK;
}

/* StereoImage.GammaEncode (StereoImage.cs:162-178): 255·sign·|m|^(1/2.2) by the log2/exp2 polynomials. */
float lo_gamma_encode(float m) {
  int32_t bits = (int32_t)fbits(m);
  int32_t a = bits & 0x7fffffff;
  float f = ffrom(((uint32_t)a & 0x007fffffu) | 0x3f800000u);
  float e = (float)((int32_t)((uint32_t)a + 0xc0800000u) >> 23);
  float log2 = ((f * ffrom(0x3e511af3u) + ffrom(0xbfa05375u)) * f + ffrom(0x40552f75u)) * f + (e + ffrom(0xc0121769u));
  float l = log2 * ffrom(0x3ee8ba2eu);
  l = l < -126.0f ? -126.0f : l; /* MathF.Max(l, -126) then MathF.Min(., 128); l is never NaN here */
  l = l > 128.0f ? 128.0f : l;
  int i = (int)l + ((int32_t)fbits(l) >> 31);
  float fr = l - (float)i;
  float p2 = ((fr * ffrom(0x3d9fcb52u) + ffrom(0x3e677e26u)) * fr + ffrom(0x3f322226u)) * fr + ffrom(0x3f7ffb19u);
  float pw = ffrom(((uint32_t)i << 23) + fbits(p2)); /* int32 wrap-around sum */
  float sgn = a == 0 ? 0.0f : ffrom(((uint32_t)bits & 0x80000000u) | 0x3f800000u);
  return pw * (sgn * 255.0f);
}

/* StereoImage.YuvMatrix (StereoImage.cs:140-160): rows (v, u', t') for the sensor type and the AsShot neutral. */
void lo_yuv_matrix(int sensor_type, const float neutral[3], float M[3][4]) {
  static const uint32_t ar1335[4] = {0x3e5cb924u, 0x3edd5758u, 0x3eb44c16u, 0x40145fafu};
  static const uint32_t other[4] = {0x3e9e39b4u, 0x3e95ca4bu, 0x3ecbfc22u, 0x40351eb8u};
  const uint32_t* t = (sensor_type == 2 || sensor_type == 3) ? ar1335 : other;
  float a = ffrom(t[0]), b = ffrom(t[1]), c = ffrom(t[2]);
  float invx = 1.0f / neutral[0], invy = 1.0f / neutral[1], invz = 1.0f / neutral[2];
  float s = c + a;
  float u0 = (b * (-b) - s * c) * invx, u1 = ((a - c) * b) * invy, u2 = (s * a - b * (-b)) * invz;
  float t0 = invx * (-b), t1 = invy * s, t2 = invz * (-b);
  float v2 = c * c + (b * b + a * a);
  float rs = ffrom(lo_rsqrt_bits(fbits(v2)));
  float S = v2 * rs;
  float kv = ((S * rs + (-3.0f)) * (S * (-0.5f)));
  if (v2 == 0.0f) kv = 0.0f;
  float u2n = u2 * u2 + (u1 * u1 + u0 * u0);
  float rsu = ffrom(lo_rsqrt_bits(fbits(u2n)));
  float ku = ((rsu * (-0.5f)) * kv) * ((u2n * rsu) * rsu + (-3.0f));
  float t2n = t2 * t2 + (t1 * t1 + t0 * t0);
  float rst = ffrom(lo_rsqrt_bits(fbits(t2n)));
  float kt = ((rst * (-0.5f)) * kv) * ((t2n * rst) * rst + (-3.0f));
  M[0][0] = a; M[0][1] = b; M[0][2] = c; M[0][3] = 0.0f;
  M[1][0] = u0 * ku; M[1][1] = u1 * ku; M[1][2] = ku * u2; M[1][3] = 0.0f;
  M[2][0] = t0 * kt; M[2][1] = t1 * kt; M[2][2] = kt * t2; M[2][3] = 0.0f;
}

void lo_convert_yuv(float* px, size_t npx, const float M[3][4]) {
  for (size_t o = 0; o < npx * 4; o += 4) {
    float x = px[o], y = px[o + 1], z = px[o + 2], ww = px[o + 3];
    float my = (ww * M[0][3] + z * M[0][2]) + (y * M[0][1] + x * M[0][0]);
    float mu = (ww * M[1][3] + z * M[1][2]) + (y * M[1][1] + x * M[1][0]);
    float mv = (ww * M[2][3] + z * M[2][2]) + (y * M[2][1] + x * M[2][0]);
    px[o] = lo_gamma_encode(my) + 0.0f;
    px[o + 1] = lo_gamma_encode(mu) + 128.0f;
    px[o + 2] = lo_gamma_encode(mv) + 128.0f;
    px[o + 3] = 1.0f;
  }
}

/* cvtps2dq (round to nearest even; NaN and out-of-range -> 0x80000000), then packssdw and packuswb. */
static uint8_t store_u8(float v) {
  int iv;
  if (v != v || v >= 2147483648.0f || v < -2147483648.0f) iv = INT32_MIN;
  else iv = (int)nearbyintf(v);
  return (uint8_t)clampi(clampi(iv, -32768, 32767), 0, 255);
}

void lo_to_rgba8(const float* rgba, size_t n, uint8_t* out) {
  for (size_t i = 0; i < n; i++) out[i] = store_u8(rgba[i]);
}

int lo_warp_rgba8(const uint8_t* src, int sw, int sh, int dw, int dh, const lo_aligned* ac, uint8_t* dst) {
  if (sw < 1 || sh < 1) return LO_ERR_ARG; /* "empty source image!" */
  if (dw < 0 || dh < 0 || !ac || !ac->lut) return LO_ERR_ARG;
  float tbl[384];
  lo_lanczos_table(tbl);
  for (int y = 0; y < dh; y++)
    for (int x = 0; x < dw; x++) {
      int px, py;
      if (warp_map(ac, x, y, &px, &py)) return LO_ERR_INDEX;
      int i = px >> 6, fx = px & 63, j = py >> 6, fy = py & 63;
      int interior = i >= 0 && i <= sw - 6 && j >= 0 && j <= sh - 6;
      int ro[6], co[6];
      for (int k = 0; k < 6; k++) {
        ro[k] = interior ? j + k : clampi(j + k, 0, sh - 1);
        co[k] = interior ? i + k : clampi(i + k, 0, sw - 1);
      }
      const float *ty = tbl + fy * 6, *tx = tbl + fx * 6;
      for (int c = 0; c < 4; c++) {
        float C[6];
        for (int cc = 0; cc < 6; cc++) {
          float acc = (float)src[((size_t)ro[0] * sw + co[cc]) * 4 + c] * ty[0];
          for (int rr = 1; rr < 6; rr++) acc = acc + (float)src[((size_t)ro[rr] * sw + co[cc]) * 4 + c] * ty[rr];
          C[cc] = acc;
        }
        float v = (C[5] * tx[5] + C[4] * tx[4]) + ((C[3] * tx[3] + C[2] * tx[2]) + (C[1] * tx[1] + C[0] * tx[0]));
        dst[((size_t)y * dw + x) * 4 + c] = store_u8(v);
      }
    }
  return LO_OK;
}

/* ---------------- StereoColorTransfer (StereoColorTransfer.cs:15-148) ---------------- */

/* Inv3D (:21-28): the 3x3 double inverse, in its operation order. */
static void inv3d(const double* m, double* o) {
  double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
  double c00 = i * e - f * h, c10 = d * i - g * f, c20 = d * h - g * e;
  double det = ((c20 * c) + (c00 * a)) - (c10 * b);
  double inv = 1.0 / det;
  o[0] = c00 * inv; o[1] = (c * h - b * i) * inv; o[2] = (b * f - c * e) * inv;
  o[3] = -(c10 * inv); o[4] = (i * a - c * g) * inv; o[5] = (c * d - f * a) * inv;
  o[6] = c20 * inv; o[7] = (g * b - h * a) * inv; o[8] = (e * a - d * b) * inv;
}

/* CropRect (:32-51) */
void lo_crop_rect(const lo_calib* calib2, const lo_calib* calibA, int x0, int y0, int x1, int y1, int out[4]) {
  float xf[16];
  lo_flow_matrix(calib2, calibA, xf);
  double D[9], Di[9];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) D[3 * r + c] = xf[4 * c + r];
  inv3d(D, Di);
  const float cx[4] = {(float)x0, (float)x0, (float)x1, (float)x1}, cy[4] = {(float)y0, (float)y1, (float)y0, (float)y1};
  float minX = 0, minY = 0, maxX = 0, maxY = 0;
  for (int k = 0; k < 4; k++) {
    float X = cx[k], Y = cy[k];
    double w = Di[8] + (Di[7] * Y + Di[6] * X);
    float wf = (float)w;
    float r0 = lo_rcp(wf);
    float r = ((1.0f - wf * r0) * r0 + r0) * 1.0f;
    float x = (float)(Di[2] + (Di[1] * Y + Di[0] * X)) * r;
    float y = (float)(Di[5] + (Di[4] * Y + Di[3] * X)) * r;
    if (k == 0) {
      minX = maxX = x;
      minY = maxY = y;
    } else {
      if (x <= minX) minX = x;
      if (maxX <= x) maxX = x;
      if (y <= minY) minY = y;
      if (maxY <= y) maxY = y;
    }
  }
  out[0] = net_int(minX); out[1] = net_int(minY); out[2] = net_int(maxX); out[3] = net_int(maxY);
}

typedef struct {
  float mean[4], D[4], O[4], N;
} lo_cstats;

/* Accumulate (:56-75): Welford in float over the pixels with alpha > 0.95, lane by lane as the SSE vectors. */
static lo_cstats accumulate(const float* yuva, int w, int h, int stride, size_t offset) {
  static const float c0[4] = {1, 0, 0, 0}, c1[4] = {0, 1, 0, 0}, c2[4] = {0, 0, 1, 0}, e3[4] = {0, 0, 0, 1};
  lo_cstats s;
  memset(&s, 0, sizeof s);
  float n = 0.0f;
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const float* p = yuva + (offset + (size_t)y * stride + x) * 4;
      float px = p[0], py = p[1], pz = p[2], pw = p[3];
      if (!(pw > 0.95f)) continue;
      float n1 = n + 1.0f, r = 1.0f / n1;
      float d[4], t[4];
      for (int k = 0; k < 4; k++) d[k] = ((pz * c2[k] - s.mean[k]) + pw * e3[k]) + (py * c1[k] + px * c0[k]);
      for (int k = 0; k < 4; k++) {
        float rd = r * d[k];
        t[k] = n * rd;
        s.mean[k] = rd + s.mean[k];
        s.D[k] = t[k] * d[k] + s.D[k];
      }
      const float ds[4] = {d[1], d[2], d[0], d[3]};
      for (int k = 0; k < 4; k++) s.O[k] = ds[k] * t[k] + s.O[k];
      n = n1;
    }
  s.N = n;
  return s;
}

/* Chol (:77-84) of Cov (:86-91): L = U^T, row-major. */
static void chol_cov(const lo_cstats* st, double L[9]) {
  float inv = 1.0f / st->N, Dn[4], On[4];
  for (int k = 0; k < 4; k++) {
    Dn[k] = st->D[k] * inv;
    On[k] = st->O[k] * inv;
  }
  const float C[9] = {Dn[0], On[0], On[2], On[0], Dn[1], On[1], On[2], On[1], Dn[2]};
  const double tol = 0.001;
  double U00 = C[0] + tol, U01 = C[1], U02 = C[2], U11 = C[4] + tol, U12 = C[5], U22 = C[8] + tol;
  double d0 = U00;
  if (d0 > 0) {
    U00 = sqrt(d0);
    double q = 1.0 / U00;
    U01 *= q;
    U02 *= q;
    double d1 = U11 - U01 * U01;
    if (d1 > 0) {
      U11 = sqrt(d1);
      U12 = U12 - U02 * U01;
      q = 1.0 / U11;
      U12 *= q;
      double d2 = U22 - (U02 * U02 + U12 * U12);
      if (d2 > 0) U22 = sqrt(d2);
    }
  }
  L[0] = U00; L[1] = 0; L[2] = 0; L[3] = U01; L[4] = U11; L[5] = 0; L[6] = U02; L[7] = U12; L[8] = U22;
}

static void ident4(double* m) {
  memset(m, 0, 16 * sizeof(double));
  m[0] = m[5] = m[10] = m[15] = 1.0;
}

/* Solve (:94-108) */
static void color_solve(const lo_cstats* work, const lo_cstats* ref, float F[16]) {
  memset(F, 0, 16 * sizeof(float));
  F[0] = F[5] = F[10] = F[15] = 1.0f;
  if (net_int(work->N) < 100 || net_int(ref->N) < 100) return;
  double Lr[9], Lw[9], Li[9], A4[16], Tr[16], Tw[16], M4[16], Minv4[16], t1[16], t2[16], t3[16], X[16];
  chol_cov(ref, Lr);
  chol_cov(work, Lw);
  inv3d(Lw, Li);
  memset(A4, 0, sizeof A4);
  A4[15] = 1.0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) A4[4 * i + j] = (Lr[3 * i] * Li[j] + Lr[3 * i + 1] * Li[3 + j]) + Lr[3 * i + 2] * Li[6 + j];
  ident4(Tr);
  ident4(Tw);
  for (int k = 0; k < 3; k++) {
    Tr[4 * k + 3] = ref->mean[k];
    Tw[4 * k + 3] = -(double)work->mean[k];
  }
  ident4(M4);
  ident4(Minv4);
  Minv4[4] = -0.0;
  mat4_mul(Tr, A4, t1);
  mat4_mul(t1, Tw, t2);
  mat4_mul(Minv4, t2, t3);
  mat4_mul(t3, M4, X);
  for (int k = 0; k < 16; k++) F[k] = (float)X[k];
}

void lo_color_transfer(const float* work, int w, int h, const float* ref, int rw, int rh, const lo_calib* calib2,
                       const lo_calib* calibA, float* out, float F[16], int crop[4], float* n_work, float* n_ref) {
  int rect[4];
  lo_crop_rect(calib2, calibA, 0, 0, rw, rh, rect);
  int X0 = rect[0] > 0 ? rect[0] : 0, Y0 = rect[1] > 0 ? rect[1] : 0, X1 = rect[2] < rw ? rect[2] : rw, Y1 = rect[3] < rh ? rect[3] : rh;
  lo_cstats sw = accumulate(work, w, h, w, 0), sr;
  if (X1 - X0 <= 0 || Y1 - Y0 <= 0) memset(&sr, 0, sizeof sr);
  else sr = accumulate(ref, X1 - X0, Y1 - Y0, rw, (size_t)Y0 * rw + X0);
  color_solve(&sw, &sr, F);
  crop[0] = X0; crop[1] = Y0; crop[2] = X1; crop[3] = Y1;
  *n_work = sw.N;
  *n_ref = sr.N;
  /* Apply (:112-125): o = a·((1·c3 + z·c2) + (y·c1 + x·c0)), o.a = a, with c_j the columns of F */
  for (size_t p = 0; p < (size_t)w * h; p++) {
    const float x = work[p * 4], y = work[p * 4 + 1], z = work[p * 4 + 2], a = work[p * 4 + 3];
    for (int k = 0; k < 3; k++) {
      float acc = (1.0f * F[4 * k + 3] + z * F[4 * k + 2]) + (y * F[4 * k + 1] + x * F[4 * k]);
      out[p * 4 + k] = a * acc;
    }
    out[p * 4 + 3] = a;
  }
}
