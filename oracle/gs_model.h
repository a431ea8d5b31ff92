// gs_model.h — the oracle's own statement of the 3D Gaussian model's
// per-primitive math (TEST INFRASTRUCTURE ONLY: included by nps_oracle_gs.cpp,
// never by the CUDA library, whose kernels carry their own copy of the model).
//
// Record layout (the trainer's parameter format, 64 floats = 256 B per
// Gaussian): mean 0-2, log-scales 3-5, quaternion (w, x, y, z) 6-9, opacity
// logit 10, pad 11, SH coefficients 12-59 (16 x rgb), 60-63 free.  A view
// record is 48 floats: view-projection (column-major), its inverse, camera
// position, pad.
//
// Colour: real spherical harmonics with the Condon-Shortley phase, basis
// index k = l^2 + l + m, evaluated at the unit direction from the camera to
// the mean.  Y_lm = K_lm * Q_lm(x, y, z) with K_lm the orthonormal factor
// sqrt((2l+1)/(4 pi) (l-|m|)!/(l+|m|)!) (times sqrt 2 for m != 0) and Q_lm
// the Cartesian form of P_l^|m|(z) cos / sin(|m| phi) on the unit sphere; the
// coefficient table below is built from those factors at start-up.
//
// Covariance: Sigma = M M^T with M = R(q / |q|) diag(exp(log-scales)); the
// 2D covariance is J Sigma J^T + lowpass I, with J the Jacobian of the pixel
// position (u, v) = ((ndc_x + 1) W/2 - 1/2, (1 - ndc_y) H/2 - 1/2) with
// respect to the mean, taken from the rows of the view-projection matrix.
#pragma once

#include <cmath>
#include <cstdint>

namespace orc_gm {

constexpr int kP = 64;
constexpr int kMean = 0, kLogScale = 3, kQuat = 6, kOpacity = 10, kSH = 12;
constexpr int kUsed = 60;
constexpr int kViewRec = 48;

// ---- real spherical harmonics up to degree 3

inline double factorial(int n) {
  double f = 1;
  for (int i = 2; i <= n; ++i) f *= i;
  return f;
}

// K_lm (sqrt 2 included for m != 0)
inline double sh_norm(int l, int m) {
  const double pi = 3.14159265358979323846;
  const int a = m < 0 ? -m : m;
  const double k = std::sqrt((2 * l + 1) / (4 * pi) * factorial(l - a) / factorial(l + a));
  return a ? std::sqrt(2.0) * k : k;
}

// Coefficient c_k with Y_k = c_k * poly_k(x, y, z), poly_k listed in real_sh.
// The leading factor of each polynomial is that of P_l^|m| (Condon-Shortley
// sign included) times the factor of the Cartesian form of cos / sin(|m| phi):
//   l=1: P_1^1 = -s                      -> -x, -y
//   l=2: P_2^1 = -3 z s, P_2^2 = 3 s^2     -> -3xz, -3yz; 3(x^2 - y^2), 3 * 2xy
//        P_2^0 = (3z^2 - 1)/2            -> (2z^2 - x^2 - y^2) / 2
//   l=3: P_3^1 = -3/2 (5z^2 - 1) s       -> -3/2 x(4z^2 - x^2 - y^2), same with y
//        P_3^2 = 15 z s^2                -> 15 z(x^2 - y^2), 15 * 2xyz
//        P_3^3 = -15 s^3                 -> -15 x(x^2 - 3y^2), -15 y(3x^2 - y^2)
//        P_3^0 = (5z^3 - 3z)/2           -> z(2z^2 - 3x^2 - 3y^2) / 2
// (s = sqrt(1 - z^2); on the unit sphere 1 = x^2 + y^2 + z^2.)
struct ShTable {
  double c[16];
  ShTable() {
    c[0] = sh_norm(0, 0);
    c[1] = -sh_norm(1, -1);
    c[2] = sh_norm(1, 0);
    c[3] = -sh_norm(1, 1);
    c[4] = 6 * sh_norm(2, -2);
    c[5] = -3 * sh_norm(2, -1);
    c[6] = 0.5 * sh_norm(2, 0);
    c[7] = -3 * sh_norm(2, 1);
    c[8] = 3 * sh_norm(2, 2);
    c[9] = -15 * sh_norm(3, -3);
    c[10] = 30 * sh_norm(3, -2);
    c[11] = -1.5 * sh_norm(3, -1);
    c[12] = 0.5 * sh_norm(3, 0);
    c[13] = -1.5 * sh_norm(3, 1);
    c[14] = 15 * sh_norm(3, 2);
    c[15] = -15 * sh_norm(3, 3);
  }
};

template <class T>
inline T sh_c(int k) {
  static const ShTable table;
  return (T)table.c[k];
}

// Basis values b[0 .. (deg+1)^2) at the unit direction (x, y, z).
template <class T>
void real_sh(int deg, T x, T y, T z, T* b) {
  b[0] = sh_c<T>(0);
  if (deg == 0) return;
  b[1] = sh_c<T>(1) * y;
  b[2] = sh_c<T>(2) * z;
  b[3] = sh_c<T>(3) * x;
  if (deg == 1) return;
  const T x2 = x * x, y2 = y * y, z2 = z * z;
  b[4] = sh_c<T>(4) * x * y;
  b[5] = sh_c<T>(5) * y * z;
  b[6] = sh_c<T>(6) * (2 * z2 - x2 - y2);
  b[7] = sh_c<T>(7) * x * z;
  b[8] = sh_c<T>(8) * (x2 - y2);
  if (deg == 2) return;
  b[9] = sh_c<T>(9) * y * (3 * x2 - y2);
  b[10] = sh_c<T>(10) * x * y * z;
  b[11] = sh_c<T>(11) * y * (4 * z2 - x2 - y2);
  b[12] = sh_c<T>(12) * z * (2 * z2 - 3 * x2 - 3 * y2);
  b[13] = sh_c<T>(13) * x * (4 * z2 - x2 - y2);
  b[14] = sh_c<T>(14) * z * (x2 - y2);
  b[15] = sh_c<T>(15) * x * (x2 - 3 * y2);
}

// Partial derivatives of each basis polynomial (as written in real_sh, i.e.
// of the ambient polynomial, not projected onto the sphere) in x, y and z.
template <class T>
void real_sh_grad(int deg, T x, T y, T z, T* gx, T* gy, T* gz) {
  for (int k = 0; k < 16; ++k) gx[k] = gy[k] = gz[k] = 0;
  if (deg == 0) return;
  gy[1] = sh_c<T>(1);
  gz[2] = sh_c<T>(2);
  gx[3] = sh_c<T>(3);
  if (deg == 1) return;
  const T x2 = x * x, y2 = y * y, z2 = z * z;
  // c xy
  gx[4] = sh_c<T>(4) * y;
  gy[4] = sh_c<T>(4) * x;
  // c yz
  gy[5] = sh_c<T>(5) * z;
  gz[5] = sh_c<T>(5) * y;
  // c (2z^2 - x^2 - y^2)
  gx[6] = -2 * sh_c<T>(6) * x;
  gy[6] = -2 * sh_c<T>(6) * y;
  gz[6] = 4 * sh_c<T>(6) * z;
  // c xz
  gx[7] = sh_c<T>(7) * z;
  gz[7] = sh_c<T>(7) * x;
  // c (x^2 - y^2)
  gx[8] = 2 * sh_c<T>(8) * x;
  gy[8] = -2 * sh_c<T>(8) * y;
  if (deg == 2) return;
  // c (3x^2 y - y^3)
  gx[9] = 6 * sh_c<T>(9) * x * y;
  gy[9] = sh_c<T>(9) * (3 * x2 - 3 * y2);
  // c xyz
  gx[10] = sh_c<T>(10) * y * z;
  gy[10] = sh_c<T>(10) * x * z;
  gz[10] = sh_c<T>(10) * x * y;
  // c (4yz^2 - x^2 y - y^3)
  gx[11] = -2 * sh_c<T>(11) * x * y;
  gy[11] = sh_c<T>(11) * (4 * z2 - x2 - 3 * y2);
  gz[11] = 8 * sh_c<T>(11) * y * z;
  // c (2z^3 - 3x^2 z - 3y^2 z)
  gx[12] = -6 * sh_c<T>(12) * x * z;
  gy[12] = -6 * sh_c<T>(12) * y * z;
  gz[12] = sh_c<T>(12) * (6 * z2 - 3 * x2 - 3 * y2);
  // c (4xz^2 - x^3 - xy^2)
  gx[13] = sh_c<T>(13) * (4 * z2 - 3 * x2 - y2);
  gy[13] = -2 * sh_c<T>(13) * x * y;
  gz[13] = 8 * sh_c<T>(13) * x * z;
  // c (x^2 z - y^2 z)
  gx[14] = 2 * sh_c<T>(14) * x * z;
  gy[14] = -2 * sh_c<T>(14) * y * z;
  gz[14] = sh_c<T>(14) * (x2 - y2);
  // c (x^3 - 3xy^2)
  gx[15] = sh_c<T>(15) * (3 * x2 - 3 * y2);
  gy[15] = -6 * sh_c<T>(15) * x * y;
}

// ---- rotation of a unit quaternion and its vector-Jacobian product

// R[r][c] (row-major) of the unit quaternion (w, x, y, z).
template <class T>
void quat_rotation(T w, T x, T y, T z, T R[3][3]) {
  R[0][0] = 1 - 2 * (y * y + z * z);
  R[0][1] = 2 * (x * y - w * z);
  R[0][2] = 2 * (x * z + w * y);
  R[1][0] = 2 * (x * y + w * z);
  R[1][1] = 1 - 2 * (x * x + z * z);
  R[1][2] = 2 * (y * z - w * x);
  R[2][0] = 2 * (x * z - w * y);
  R[2][1] = 2 * (y * z + w * x);
  R[2][2] = 1 - 2 * (x * x + y * y);
}

// dq_k = sum_rc G[r][c] dR[r][c]/dq_k, the partials of quat_rotation's
// entries (linear in the quaternion) written out per component.
template <class T>
void quat_rotation_vjp(T w, T x, T y, T z, const T G[3][3], T* dq) {
  const T dw[3][3] = {{0, -2 * z, 2 * y}, {2 * z, 0, -2 * x}, {-2 * y, 2 * x, 0}};
  const T dx[3][3] = {{0, 2 * y, 2 * z}, {2 * y, -4 * x, -2 * w}, {2 * z, 2 * w, -4 * x}};
  const T dy[3][3] = {{-4 * y, 2 * x, 2 * w}, {2 * x, 0, 2 * z}, {-2 * w, 2 * z, -4 * y}};
  const T dz[3][3] = {{-4 * z, -2 * w, 2 * x}, {2 * w, -4 * z, 2 * y}, {2 * x, 2 * y, 0}};
  const T(*D[4])[3] = {dw, dx, dy, dz};
  for (int k = 0; k < 4; ++k) {
    T s = 0;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        // entries of R that do not involve q_k: w is off the diagonal only,
        // x / y / z are absent from R[0][0] / R[1][1] / R[2][2]
        const bool independent = k == 0 ? r == c : (r == k - 1 && c == k - 1);
        if (!independent) s += G[r][c] * D[k][r][c];
      }
    dq[k] = s;
  }
}

// ---- projection of one Gaussian into one view

template <class T>
struct Footprint {
  T cx, cy, cw;      // clip-space x, y, w (w = view depth)
  T u, v;            // pixel position of the mean
  T J[2][3];         // d(u, v) / d(mean)
  T S[3][3];         // 3D covariance
  T M[3][3];         // R diag(scale)
  T R[3][3];
  T sc[3];           // scales
  T qn[4];           // normalised quaternion
  T qlen;            // |q| (clamped away from 0)
  T A, B, C;         // 2D covariance with the low-pass added
  T det;
  T ca, cb, cc;      // its inverse (the conic); zero when det <= 0
};

// `rec` is a parameter record (kP floats, or their widening to T); vp the
// view-projection, column-major: element (row r, column c) at vp[4c + r].
template <class T>
void project_gaussian(const float* vp, const T* rec, T W, T H, T lowpass, Footprint<T>& f) {
  const T* m = rec + kMean;
  T row[4][3];
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 3; ++c) row[r][c] = (T)vp[4 * c + r];
  f.cx = row[0][0] * m[0] + row[0][1] * m[1] + row[0][2] * m[2] + (T)vp[12];
  f.cy = row[1][0] * m[0] + row[1][1] * m[1] + row[1][2] * m[2] + (T)vp[13];
  f.cw = row[3][0] * m[0] + row[3][1] * m[1] + row[3][2] * m[2] + (T)vp[15];
  const T inv_w = (T)1 / f.cw;
  const T half_w = W * (T)0.5, half_h = H * (T)0.5;
  f.u = (f.cx * inv_w + 1) * half_w - (T)0.5;
  f.v = (1 - f.cy * inv_w) * half_h - (T)0.5;
  // d(cx / cw)/dm_k = (row0_k cw - cx row3_k) / cw^2, likewise for y
  const T inv_w2 = inv_w * inv_w;
  for (int k = 0; k < 3; ++k) {
    f.J[0][k] = half_w * (row[0][k] * f.cw - f.cx * row[3][k]) * inv_w2;
    f.J[1][k] = -half_h * (row[1][k] * f.cw - f.cy * row[3][k]) * inv_w2;
  }
  const T* q = rec + kQuat;
  T q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  if (!(q2 > (T)1e-24)) q2 = (T)1e-24;
  f.qlen = std::sqrt(q2);
  for (int k = 0; k < 4; ++k) f.qn[k] = q[k] / f.qlen;
  quat_rotation(f.qn[0], f.qn[1], f.qn[2], f.qn[3], f.R);
  for (int k = 0; k < 3; ++k) f.sc[k] = std::exp(rec[kLogScale + k]);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) f.M[r][c] = f.R[r][c] * f.sc[c];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) f.S[r][c] = f.M[r][0] * f.M[c][0] + f.M[r][1] * f.M[c][1] + f.M[r][2] * f.M[c][2];
  T JS[2][3];
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 3; ++c) JS[r][c] = f.J[r][0] * f.S[0][c] + f.J[r][1] * f.S[1][c] + f.J[r][2] * f.S[2][c];
  f.A = JS[0][0] * f.J[0][0] + JS[0][1] * f.J[0][1] + JS[0][2] * f.J[0][2] + lowpass;
  f.B = JS[0][0] * f.J[1][0] + JS[0][1] * f.J[1][1] + JS[0][2] * f.J[1][2];
  f.C = JS[1][0] * f.J[1][0] + JS[1][1] * f.J[1][1] + JS[1][2] * f.J[1][2] + lowpass;
  f.det = f.A * f.C - f.B * f.B;
  const T inv_det = f.det > 0 ? (T)1 / f.det : (T)0;
  f.ca = f.C * inv_det;
  f.cb = -f.B * inv_det;
  f.cc = f.A * inv_det;
}

// ---- split sampling of the threshold ADC
//
// The children's means are a pure function of (Gaussian index, seed, child):
// a counter-based integer hash (multiply / xor-shift rounds) gives two
// uniforms per axis, Box-Muller turns them into a standard normal z, and the
// child sits at mean + R (scale * z) with log-scales reduced by ln 1.6.

inline uint32_t split_hash(uint32_t a, uint32_t b) {
  uint32_t h = (a * 0x9E3779B1u) ^ ((b + 0x7F4A7C15u) * 0x85EBCA77u);
  h ^= h >> 15;
  h *= 0x2C1B3C6Du;
  h ^= h >> 12;
  h *= 0x297A2D39u;
  h ^= h >> 15;
  return h;
}

// top 24 bits, centred in their interval: (0, 1) exclusive
inline float split_uniform(uint32_t h) { return ((float)(h >> 8) + 0.5f) * (1.0f / 16777216.0f); }

inline void split_child(const float* rec, uint32_t i, uint32_t seed, uint32_t child, float mean[3], float ls[3]) {
  const float* q = rec + kQuat;
  float n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (!(n > 1e-12f)) n = 1e-12f;
  float R[3][3];
  quat_rotation<float>(q[0] / n, q[1] / n, q[2] / n, q[3] / n, R);
  float z[3];
  for (int k = 0; k < 3; ++k) {
    const uint32_t h1 = split_hash(i, seed * 8u + child * 4u + (uint32_t)k);
    const uint32_t h2 = split_hash(h1, 0x51ED270Bu);
    const float radius = std::sqrt(-2.0f * std::log(split_uniform(h1)));
    const float angle = 6.2831853f * split_uniform(h2);
    z[k] = radius * std::cos(angle) * std::exp(rec[kLogScale + k]);
  }
  for (int r = 0; r < 3; ++r) mean[r] = rec[kMean + r] + (R[r][0] * z[0] + R[r][1] * z[1] + R[r][2] * z[2]);
  const float ln_1_6 = 0.47000363f;
  for (int k = 0; k < 3; ++k) ls[k] = rec[kLogScale + k] - ln_1_6;
}

}  // namespace orc_gm
