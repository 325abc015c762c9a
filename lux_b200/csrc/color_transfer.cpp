// The colour transfer of a non-reference stereo image onto the reference camera's crop
// (Lux.Engine/Pipeline/Registration/StereoColorTransfer.cs:15-138): the crop rect, the per-image statistics and the 4x4
// transfer. Host code by design: the statistics are a Welford recurrence in float over the pixels in row order, whose
// every step depends on the one before, so no parallel order gives the reference's bits, and one core runs the 3.2
// million steps of a 2080x1560 image in about as long as one GPU thread would. The per-pixel apply and the 8-bit store
// that follow run on the GPU (warp.cu). Every float and double operation is the reference's, in its order.
#include <cmath>
#include <cstring>

#include "host_geom.h"

namespace lux {

namespace {

inline uint32_t bits_of_f(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
inline float float_of_b(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
inline int to_int(float f) {  // (int)f in .NET 9+: truncation, saturating, NaN -> 0
  if (f != f) return 0;
  if (f >= 2147483648.0f) return 2147483647;
  if (f <= -2147483648.0f) return (-2147483647 - 1);
  return (int)f;
}

// Inv3D (:21-28): the double 3x3 inverse by cofactors, in the reference's operation order.
void inverse3(const double* m, double* o) {
  const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
  const double c00 = i * e - f * h, c10 = d * i - g * f, c20 = d * h - g * e;
  const double inv = 1.0 / (((c20 * c) + (c00 * a)) - (c10 * b));
  const double r[9] = {c00 * inv,           (c * h - b * i) * inv, (b * f - c * e) * inv, -(c10 * inv),       (i * a - c * g) * inv,
                       (c * d - f * a) * inv, c20 * inv,            (g * b - h * a) * inv, (e * a - d * b) * inv};
  std::memcpy(o, r, sizeof r);
}

// Chol of Cov (:77-91): the covariance over the count in float, then the Cholesky factor in double with 0.001 added to the
// diagonal; a factor step whose pivot is not positive is skipped, as the reference leaves it. Returns L = U^T.
void cholesky_of(const ColourStats& st, double L[9]) {
  const float inv = 1.0f / st.N;
  float Dn[3], On[3];
  for (int k = 0; k < 3; k++) {
    Dn[k] = st.D[k] * inv;
    On[k] = st.O[k] * inv;
  }
  // the covariance rows {Dn0, On0, On2}, {On0, Dn1, On1}, {On2, On1, Dn2}; only the upper triangle is read
  const double tol = 0.001;
  double u00 = (double)Dn[0] + tol, u01 = On[0], u02 = On[2], u11 = (double)Dn[1] + tol, u12 = On[1], u22 = (double)Dn[2] + tol;
  if (u00 > 0) {
    u00 = std::sqrt(u00);
    const double q0 = 1.0 / u00;
    u01 *= q0;
    u02 *= q0;
    const double p1 = u11 - u01 * u01;
    if (p1 > 0) {
      u11 = std::sqrt(p1);
      u12 = u12 - u02 * u01;
      u12 *= 1.0 / u11;
      const double p2 = u22 - (u02 * u02 + u12 * u12);
      if (p2 > 0) u22 = std::sqrt(p2);
    }
  }
  const double l[9] = {u00, 0.0, 0.0, u01, u11, 0.0, u02, u12, u22};
  std::memcpy(L, l, sizeof l);
}

}  // namespace

void host_crop_rect(const lux_calib& ref_view, const lux_calib& view, int rw, int rh, int out[4]) {
  float xf[16];
  host_flow_matrix(ref_view, view, xf);  // (K_view·E_view)·(K_ref·E_ref)^-1, column-major
  double m[9], mi[9];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) m[3 * r + c] = xf[4 * c + r];
  inverse3(m, mi);
  // the four corners in the reference's order: (x0, y0), (x0, y1), (x1, y0), (x1, y1)
  const float xs[4] = {0.0f, 0.0f, (float)rw, (float)rw}, ys[4] = {0.0f, (float)rh, 0.0f, (float)rh};
  float lo_x = 0, lo_y = 0, hi_x = 0, hi_y = 0;
  for (int k = 0; k < 4; k++) {
    const float X = xs[k], Y = ys[k];
    const float wf = (float)(mi[8] + (mi[7] * Y + mi[6] * X));
    const float r0 = float_of_b(host_rcp_bits(bits_of_f(wf)));
    const float r = ((1.0f - wf * r0) * r0 + r0) * 1.0f;  // rcpps and one Newton step
    const float x = (float)(mi[2] + (mi[1] * Y + mi[0] * X)) * r, y = (float)(mi[5] + (mi[4] * Y + mi[3] * X)) * r;
    if (k == 0) {
      lo_x = hi_x = x;
      lo_y = hi_y = y;
      continue;
    }
    if (x <= lo_x) lo_x = x;
    if (hi_x <= x) hi_x = x;
    if (y <= lo_y) lo_y = y;
    if (hi_y <= y) hi_y = y;
  }
  out[0] = to_int(lo_x);
  out[1] = to_int(lo_y);
  out[2] = to_int(hi_x);
  out[3] = to_int(hi_y);
}

ColourStats host_colour_stats(const float* yuva, int w, int h, int stride, size_t offset) {
  // the reference keeps the mean, the squared deviations (D) and the rotated cross products (O) as four-lane vectors;
  // every lane is written out here with the lane's own basis factors (1 or 0) so each product and sum is the same
  static const float kX[4] = {1, 0, 0, 0}, kY[4] = {0, 1, 0, 0}, kZ[4] = {0, 0, 1, 0}, kW[4] = {0, 0, 0, 1};
  ColourStats s;
  std::memset(&s, 0, sizeof s);
  float n = 0.0f;
  for (int y = 0; y < h; y++) {
    const float* row = yuva + (offset + (size_t)y * stride) * 4;
    for (int x = 0; x < w; x++) {
      const float* p = row + (size_t)x * 4;
      if (!(p[3] > 0.95f)) continue;  // the alpha gate
      const float n1 = n + 1.0f, r = 1.0f / n1;
      float d[4], t[4];
      for (int k = 0; k < 4; k++) d[k] = ((p[2] * kZ[k] - s.mean[k]) + p[3] * kW[k]) + (p[1] * kY[k] + p[0] * kX[k]);
      for (int k = 0; k < 4; k++) {
        const float rd = r * d[k];
        t[k] = n * rd;
        s.mean[k] = rd + s.mean[k];
        s.D[k] = t[k] * d[k] + s.D[k];
      }
      s.O[0] = d[1] * t[0] + s.O[0];  // lanes rotated to (y, z, x, w)
      s.O[1] = d[2] * t[1] + s.O[1];
      s.O[2] = d[0] * t[2] + s.O[2];
      s.O[3] = d[3] * t[3] + s.O[3];
      n = n1;
    }
  }
  s.N = n;
  return s;
}

void host_colour_solve(const ColourStats& work, const ColourStats& ref, float F[16]) {
  std::memset(F, 0, 16 * sizeof(float));
  F[0] = F[5] = F[10] = F[15] = 1.0f;
  if (to_int(work.N) < 100 || to_int(ref.N) < 100) return;  // too few gated pixels: the identity
  double lr[9], lw[9], lwi[9];
  cholesky_of(ref, lr);
  cholesky_of(work, lw);
  inverse3(lw, lwi);
  double a4[16] = {0}, tr[16] = {0}, tw[16] = {0}, eye[16] = {0}, minv[16] = {0};
  a4[15] = 1.0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) a4[4 * i + j] = (lr[3 * i] * lwi[j] + lr[3 * i + 1] * lwi[3 + j]) + lr[3 * i + 2] * lwi[6 + j];
  for (int k = 0; k < 4; k++) tr[5 * k] = tw[5 * k] = eye[5 * k] = minv[5 * k] = 1.0;
  for (int k = 0; k < 3; k++) {
    tr[4 * k + 3] = ref.mean[k];
    tw[4 * k + 3] = -(double)work.mean[k];
  }
  minv[4] = -0.0;  // the inverse of the identity basis as the reference forms it: -0 at (1, 0)
  double t1[16], t2[16], t3[16], x[16];
  host_mat4_mul(tr, a4, t1);
  host_mat4_mul(t1, tw, t2);
  host_mat4_mul(minv, t2, t3);
  host_mat4_mul(t3, eye, x);
  for (int k = 0; k < 16; k++) F[k] = (float)x[k];
}

}  // namespace lux
