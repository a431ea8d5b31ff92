// gs_math.cuh — math of the 3D Gaussian model (host + device).
//
// Model: per Gaussian a mean, log-scales, a rotation quaternion (w, x, y, z,
// normalised on use), an opacity logit and real spherical-harmonic colour
// coefficients up to degree 3.  Screen-space covariance by the EWA affine
// approximation, with the Jacobian of the pixel projection taken directly from
// the view-projection matrix (the same construction the reference uses for its
// projected axes, splat_backward.wgsl:52-58).  SH constants are the standard
// real-SH normalisations sqrt((2l+1)/(4 pi) * (l-|m|)!/(l+|m|)!) (times the
// usual sqrt(2) for m != 0), with the sign convention used by most splatting
// codes.
#pragma once
#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define GSM_HD __host__ __device__ __forceinline__
#else
#define GSM_HD inline
#endif

namespace nps {
namespace gsm {

// parameter record (floats per Gaussian, padded to 64 = 256 B)
constexpr int kP = 64;
constexpr int kMean = 0, kLogScale = 3, kQuat = 6, kOpacity = 10, kSH = 12;
constexpr int kUsed = 60;  // end of the used floats: 3 + 3 + 4 + 1 + pad + 48
constexpr int kViewRec = 48;  // floats per view: vp[16], vp_inv[16], cam_pos[3], pad

constexpr float SH_C0 = 0.28209479177387814f;
constexpr float SH_C1 = 0.4886025119029199f;
constexpr float SH_C2_0 = 1.0925484305920792f, SH_C2_1 = -1.0925484305920792f, SH_C2_2 = 0.31539156525252005f,
                SH_C2_3 = -1.0925484305920792f, SH_C2_4 = 0.5462742152960396f;
constexpr float SH_C3_0 = -0.5900435899266435f, SH_C3_1 = 2.890611442640554f, SH_C3_2 = -0.4570457994644658f,
                SH_C3_3 = 0.3731763325901154f, SH_C3_4 = -0.4570457994644658f, SH_C3_5 = 1.445305721320277f,
                SH_C3_6 = -0.5900435899266435f;

template <class T>
GSM_HD void sh_basis(int deg, T x, T y, T z, T* b) {
  b[0] = (T)SH_C0;
  if (deg < 1) return;
  b[1] = -(T)SH_C1 * y;
  b[2] = (T)SH_C1 * z;
  b[3] = -(T)SH_C1 * x;
  if (deg < 2) return;
  const T xx = x * x, yy = y * y, zz = z * z;
  b[4] = (T)SH_C2_0 * x * y;
  b[5] = (T)SH_C2_1 * y * z;
  b[6] = (T)SH_C2_2 * (2 * zz - xx - yy);
  b[7] = (T)SH_C2_3 * x * z;
  b[8] = (T)SH_C2_4 * (xx - yy);
  if (deg < 3) return;
  b[9] = (T)SH_C3_0 * y * (3 * xx - yy);
  b[10] = (T)SH_C3_1 * x * y * z;
  b[11] = (T)SH_C3_2 * y * (4 * zz - xx - yy);
  b[12] = (T)SH_C3_3 * z * (2 * zz - 3 * xx - 3 * yy);
  b[13] = (T)SH_C3_4 * x * (4 * zz - xx - yy);
  b[14] = (T)SH_C3_5 * z * (xx - yy);
  b[15] = (T)SH_C3_6 * x * (xx - 3 * yy);
}

// d basis_k / d(x, y, z), written into gx, gy, gz (k >= 1; basis 0 is constant)
template <class T>
GSM_HD void sh_basis_grad(int deg, T x, T y, T z, T* gx, T* gy, T* gz) {
  for (int k = 0; k < 16; ++k) gx[k] = gy[k] = gz[k] = 0;
  if (deg < 1) return;
  gy[1] = -(T)SH_C1;
  gz[2] = (T)SH_C1;
  gx[3] = -(T)SH_C1;
  if (deg < 2) return;
  const T xx = x * x, yy = y * y, zz = z * z;
  gx[4] = (T)SH_C2_0 * y; gy[4] = (T)SH_C2_0 * x;
  gy[5] = (T)SH_C2_1 * z; gz[5] = (T)SH_C2_1 * y;
  gx[6] = -2 * (T)SH_C2_2 * x; gy[6] = -2 * (T)SH_C2_2 * y; gz[6] = 4 * (T)SH_C2_2 * z;
  gx[7] = (T)SH_C2_3 * z; gz[7] = (T)SH_C2_3 * x;
  gx[8] = 2 * (T)SH_C2_4 * x; gy[8] = -2 * (T)SH_C2_4 * y;
  if (deg < 3) return;
  gx[9] = 6 * (T)SH_C3_0 * x * y; gy[9] = (T)SH_C3_0 * (3 * xx - 3 * yy);
  gx[10] = (T)SH_C3_1 * y * z; gy[10] = (T)SH_C3_1 * x * z; gz[10] = (T)SH_C3_1 * x * y;
  gx[11] = -2 * (T)SH_C3_2 * x * y; gy[11] = (T)SH_C3_2 * (4 * zz - xx - 3 * yy); gz[11] = 8 * (T)SH_C3_2 * y * z;
  gx[12] = -6 * (T)SH_C3_3 * x * z; gy[12] = -6 * (T)SH_C3_3 * y * z; gz[12] = (T)SH_C3_3 * (6 * zz - 3 * xx - 3 * yy);
  gx[13] = (T)SH_C3_4 * (4 * zz - 3 * xx - yy); gy[13] = -2 * (T)SH_C3_4 * x * y; gz[13] = 8 * (T)SH_C3_4 * x * z;
  gx[14] = 2 * (T)SH_C3_5 * x * z; gy[14] = -2 * (T)SH_C3_5 * y * z; gz[14] = (T)SH_C3_5 * (xx - yy);
  gx[15] = (T)SH_C3_6 * (3 * xx - 3 * yy); gy[15] = -6 * (T)SH_C3_6 * x * y;
}

// Rotation matrix (row-major R[r][c]) of a unit quaternion (w, x, y, z).
template <class T>
GSM_HD void quat_to_rot(T w, T x, T y, T z, T R[3][3]) {
  R[0][0] = 1 - 2 * (y * y + z * z); R[0][1] = 2 * (x * y - w * z); R[0][2] = 2 * (x * z + w * y);
  R[1][0] = 2 * (x * y + w * z); R[1][1] = 1 - 2 * (x * x + z * z); R[1][2] = 2 * (y * z - w * x);
  R[2][0] = 2 * (x * z - w * y); R[2][1] = 2 * (y * z + w * x); R[2][2] = 1 - 2 * (x * x + y * y);
}

// dL/dq for R(q) given dL/dR (q unit, before renormalisation chain)
template <class T>
GSM_HD void rot_grad_to_quat(T w, T x, T y, T z, const T G[3][3], T* dq) {
  dq[0] = G[0][1] * (-2 * z) + G[0][2] * (2 * y) + G[1][0] * (2 * z) + G[1][2] * (-2 * x) + G[2][0] * (-2 * y) +
          G[2][1] * (2 * x);
  dq[1] = G[0][1] * (2 * y) + G[0][2] * (2 * z) + G[1][0] * (2 * y) + G[1][1] * (-4 * x) + G[1][2] * (-2 * w) +
          G[2][0] * (2 * z) + G[2][1] * (2 * w) + G[2][2] * (-4 * x);
  dq[2] = G[0][0] * (-4 * y) + G[0][1] * (2 * x) + G[0][2] * (2 * w) + G[1][0] * (2 * x) + G[1][2] * (2 * z) +
          G[2][0] * (-2 * w) + G[2][1] * (2 * z) + G[2][2] * (-4 * y);
  dq[3] = G[0][0] * (-4 * z) + G[0][1] * (-2 * w) + G[0][2] * (2 * x) + G[1][0] * (2 * w) + G[1][1] * (-4 * z) +
          G[1][2] * (2 * y) + G[2][0] * (2 * x) + G[2][1] * (2 * y);
}

// Projection of one Gaussian into one view.  vp is column-major (element
// (row r, col c) at vp[4c + r]).  Pixel coordinates: x right, y down, pixel
// centres at integers, u = (ndc_x + 1) W/2 - 1/2, v = (1 - ndc_y) H/2 - 1/2.
template <class T>
struct Proj {
  T cx, cy, cw;      // clip x, y, w (w = view depth)
  T u, v;            // pixel position of the mean
  T J[2][3];         // d(u, v) / d(mean)
  T S[3][3];         // 3D covariance
  T M[3][3];         // R * diag(scale) (columns = scaled axes)
  T R[3][3];
  T sc[3];
  T qn[4];           // normalised quaternion
  T qlen;
  T A, B, C;         // 2D covariance (+ low-pass)
  T det;
  T ca, cb, cc;      // conic (inverse 2D covariance)
};

// a0 m0 + a1 m1 + a2 m2 + c with every product and sum rounded on its own
// (no fused multiply-add), left to right: the view depth that orders the
// tile lists is then the plain float evaluation bit for bit, so two Gaussians
// whose depths differ in the last place keep the order a plain evaluation
// gives them.
template <class T>
GSM_HD T dot3_plus_rounded(const T* a, const T* m, T c) {
#ifdef __CUDA_ARCH__
  if constexpr (sizeof(T) == sizeof(float))
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(a[0], m[0]), __fmul_rn(a[1], m[1])), __fmul_rn(a[2], m[2])), c);
#endif
  return a[0] * m[0] + a[1] * m[1] + a[2] * m[2] + c;
}

template <class T>
GSM_HD void project(const float* vp, const T* mean, const T* log_scale, const T* quat, T W, T H, T lowpass, Proj<T>& P) {
  const T r0[3] = {(T)vp[0], (T)vp[4], (T)vp[8]};
  const T r1[3] = {(T)vp[1], (T)vp[5], (T)vp[9]};
  const T r3[3] = {(T)vp[3], (T)vp[7], (T)vp[11]};
  P.cx = r0[0] * mean[0] + r0[1] * mean[1] + r0[2] * mean[2] + (T)vp[12];
  P.cy = r1[0] * mean[0] + r1[1] * mean[1] + r1[2] * mean[2] + (T)vp[13];
  P.cw = dot3_plus_rounded<T>(r3, mean, (T)vp[15]);
  const T iw = (T)1 / P.cw;
  const T a = W * (T)0.5, b = H * (T)0.5;
  P.u = (P.cx * iw + 1) * a - (T)0.5;
  P.v = (1 - P.cy * iw) * b - (T)0.5;
  const T iw2 = iw * iw;
  for (int k = 0; k < 3; ++k) {
    P.J[0][k] = a * (r0[k] * P.cw - P.cx * r3[k]) * iw2;
    P.J[1][k] = -b * (r1[k] * P.cw - P.cy * r3[k]) * iw2;
  }
  T ql = quat[0] * quat[0] + quat[1] * quat[1] + quat[2] * quat[2] + quat[3] * quat[3];
  ql = ql > (T)1e-24 ? ql : (T)1e-24;
#ifdef __CUDA_ARCH__
  P.qlen = sqrt(ql);
#else
  P.qlen = std::sqrt(ql);
#endif
  for (int k = 0; k < 4; ++k) P.qn[k] = quat[k] / P.qlen;
  quat_to_rot(P.qn[0], P.qn[1], P.qn[2], P.qn[3], P.R);
  for (int k = 0; k < 3; ++k) {
#ifdef __CUDA_ARCH__
    P.sc[k] = exp(log_scale[k]);
#else
    P.sc[k] = std::exp(log_scale[k]);
#endif
  }
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) P.M[r][c] = P.R[r][c] * P.sc[c];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) P.S[r][c] = P.M[r][0] * P.M[c][0] + P.M[r][1] * P.M[c][1] + P.M[r][2] * P.M[c][2];
  T JS[2][3];
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 3; ++c) JS[r][c] = P.J[r][0] * P.S[0][c] + P.J[r][1] * P.S[1][c] + P.J[r][2] * P.S[2][c];
  P.A = JS[0][0] * P.J[0][0] + JS[0][1] * P.J[0][1] + JS[0][2] * P.J[0][2] + lowpass;
  P.B = JS[0][0] * P.J[1][0] + JS[0][1] * P.J[1][1] + JS[0][2] * P.J[1][2];
  P.C = JS[1][0] * P.J[1][0] + JS[1][1] * P.J[1][1] + JS[1][2] * P.J[1][2] + lowpass;
  P.det = P.A * P.C - P.B * P.B;
  const T id = P.det > 0 ? (T)1 / P.det : (T)0;
  P.ca = P.C * id;
  P.cb = -P.B * id;
  P.cc = P.A * id;
}

// ---- ADC split sampling (shared by the kernel and the oracle)
// Counter-based hash: child means are a pure function of (index, seed, child).
GSM_HD uint32_t adc_hash(uint32_t a, uint32_t b) {
  uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u;
  h ^= h >> 15;
  h *= 0x2C1B3C6Du;
  h ^= h >> 12;
  h *= 0x297A2D39u;
  h ^= h >> 15;
  return h;
}
GSM_HD float adc_uniform(uint32_t h) { return ((float)(h >> 8) + 0.5f) * (1.0f / 16777216.0f); }

// Child `ch` (0 or 1) of a split: mean = parent mean + R (s * z), z ~ N(0, I)
// by Box-Muller from the hash; log-scales = parent - ln 1.6.
GSM_HD void adc_split_child(const float* P, uint32_t i, uint32_t seed, uint32_t ch, float mean[3], float ls[3]) {
  float qw = P[6], qx = P[7], qy = P[8], qz = P[9];
  float ql = sqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
  ql = ql > 1e-12f ? ql : 1e-12f;
  float R[3][3];
  quat_to_rot<float>(qw / ql, qx / ql, qy / ql, qz / ql, R);
  float z[3];
  for (int k = 0; k < 3; ++k) {
    const uint32_t h1 = adc_hash(i, seed * 8u + ch * 4u + (uint32_t)k);
    const uint32_t h2 = adc_hash(h1, 0x51ED270Bu);
    z[k] = sqrtf(-2.0f * logf(adc_uniform(h1))) * cosf(6.2831853f * adc_uniform(h2)) * expf(P[3 + k]);
  }
  for (int r = 0; r < 3; ++r) mean[r] = P[r] + (R[r][0] * z[0] + R[r][1] * z[1] + R[r][2] * z[2]);
  const float d = 0.47000363f;  // ln 1.6
  for (int k = 0; k < 3; ++k) ls[k] = P[3 + k] - d;
}

}  // namespace gsm
}  // namespace nps
