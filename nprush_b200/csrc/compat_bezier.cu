// compat_bezier.cu — cubic 3D Bezier stroke training step with the
// reference's semantics (GpuBezierOptimizerManager.dispatch(),
// GpuBezierOptimizerManager.ts:370-406):
//   k_bz_project  per (view, curve): projected control points
//                 (bezier_backward.wgsl:69-72), culling and hull box
//                 (:126-156) -> tile rectangle (binning.cuh), the per-control-
//                 point screen Jacobians of backproject_gradient (:74-88)
//   scan, emit, stable radix sort, ranges (as for splats; 1024 cap at :166)
//   k_bz_raster   one CTA per (tile, view): the 16-segment closest-point walk,
//                 pressure, analytic coverage, composite over the background
//                 (:196-269), luma / contrast / depth / edge loss (:271-320),
//                 reverse backward through the closest segment with the width,
//                 softness and direction-regulariser terms (:325-563),
//                 transmittance replayed exactly from per-28-curve
//                 checkpoints; i32 gradients reduced per warp and CTA before
//                 one global atomic; loss_accum and the pixel_loss map
//   k_bz_step     bezier_step.wgsl:50-189
//   k_bz_adc      bezier_adc.wgsl:75-315 (kill, split/clone, spawn, second
//                 split/clone, reset) in one CTA, serial-equivalent
// Compiled with --fmad=false (the reference's fp32 operation order).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "binning.cuh"
#include "common.cuh"
#include "context.h"

namespace nps {
namespace bz {

constexpr int kRecF = 20;      // forward record floats
constexpr int kRecB = 24;      // backward record floats (per control point: d screen / d world, 2 x 3)
constexpr uint32_t kCap = 1024;  // BEZIER_MAX_TILE_BEZIERS, constants.ts:20
constexpr int kChunk = 28;       // with the checkpoints in global memory, 3 CTAs per SM fit
constexpr int kMaxChunks = (kCap + kChunk - 1) / kChunk;  // transmittance checkpoints per pixel
constexpr int kThreads = 256;
constexpr uint32_t kNSeg = 16;   // bezier_backward.wgsl:52
constexpr float kKillAlpha = 0.005f;  // constants.ts:15
constexpr float kFpPos = 10000.0f, kFpCol = 100000.0f;  // constants.ts:18-19
constexpr uint32_t kPixelLossSize = 512u * 512u;        // constants.ts:10

__device__ __forceinline__ float clampf(float e, float lo, float hi) { return fminf(fmaxf(e, lo), hi); }
__device__ __forceinline__ float smoothstepf(float lo, float hi, float x) {
  const float t = clampf((x - lo) / (hi - lo), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ int32_t to_i32(float a) {
  // the conversion instruction truncates and clamps below at INT32_MIN by
  // itself (float-to-integer conversions saturate); WGSL's upper bound is the
  // largest float below 2^31
  if (a != a) return 0;
  return a >= 2147483520.0f ? 2147483520 : (int32_t)a;
}
__device__ __forceinline__ float4 mulv(const float* m, float x, float y, float z, float w) {
  float4 o;
  o.x = m[0] * x + m[4] * y + m[8] * z + m[12] * w;
  o.y = m[1] * x + m[5] * y + m[9] * z + m[13] * w;
  o.z = m[2] * x + m[6] * y + m[10] * z + m[14] * w;
  o.w = m[3] * x + m[7] * y + m[11] * z + m[15] * w;
  return o;
}
__device__ __forceinline__ float fractf(float x) { return x - floorf(x); }

// bezier_backward.wgsl:56-62
__device__ __forceinline__ float2 bezier_at(const float* q, float t) {
  const float omt = 1.0f - t;
  const float c0 = omt * omt * omt, c1 = 3.0f * omt * omt * t, c2 = 3.0f * omt * t * t, c3 = t * t * t;
  return make_float2(c0 * q[0] + c1 * q[2] + c2 * q[4] + c3 * q[6], c0 * q[1] + c1 * q[3] + c2 * q[5] + c3 * q[7]);
}
// bezier_backward.wgsl:64-67
__device__ __forceinline__ float4 bernstein(float t) {
  const float omt = 1.0f - t;
  return make_float4(omt * omt * omt, 3.0f * omt * omt * t, 3.0f * omt * t * t, t * t * t);
}

struct Uni {
  float mode, max_width, prune_alpha, prune_width, bg_penalty;
};

__global__ void __launch_bounds__(256) k_bz_project(const float* __restrict__ bz, uint32_t n,
                                                    const float* __restrict__ views, uint32_t nv, uint32_t w,
                                                    uint32_t h, const float* __restrict__ tabs, uint32_t tiles_x,
                                                    uint32_t tiles_y, float* __restrict__ fwd,
                                                    float* __restrict__ bwd, uint32_t* __restrict__ counts,
                                                    uint2* __restrict__ rects) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nv * n) return;
  const uint32_t v = g / n, i = g - v * n;
  const float* vp = views + 32 * (size_t)v;
  float b[20];
  const float4* b4 = reinterpret_cast<const float4*>(bz + 20 * (size_t)i);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const float4 t = b4[q];
    b[4 * q] = t.x; b[4 * q + 1] = t.y; b[4 * q + 2] = t.z; b[4 * q + 3] = t.w;
  }
  const float aspect = (float)w / (float)h;
  float px[4], py[4], pw[4];
  float jb[24];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float4 cl = mulv(vp, b[4 * c], b[4 * c + 1], b[4 * c + 2], 1.0f);
    px[c] = cl.x / cl.w * aspect;
    py[c] = cl.y / cl.w;
    pw[c] = cl.w;
    const float ww = cl.w, w2 = ww * ww;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const float v0 = vp[ax * 4 + 0], v1 = vp[ax * 4 + 1], v3 = vp[ax * 4 + 3];
      jb[6 * c + ax] = aspect * (v0 * ww - cl.x * v3) / w2;
      jb[6 * c + 3 + ax] = (v1 * ww - cl.y * v3) / w2;
    }
  }
  const float width = fmaxf(b[3], 0.001f), soft = fmaxf(b[7], 0.001f);
  float4* f4 = reinterpret_cast<float4*>(fwd + (size_t)g * kRecF);
  f4[0] = make_float4(px[0], py[0], px[1], py[1]);
  f4[1] = make_float4(px[2], py[2], px[3], py[3]);
  f4[2] = make_float4(pw[0], pw[1], pw[2], pw[3]);
  f4[3] = make_float4(width, soft, b[19], b[16]);
  f4[4] = make_float4(b[17], b[18], 0.0f, 0.0f);
  float4* j4 = reinterpret_cast<float4*>(bwd + (size_t)g * kRecB);
#pragma unroll
  for (int q = 0; q < 6; ++q) j4[q] = make_float4(jb[4 * q], jb[4 * q + 1], jb[4 * q + 2], jb[4 * q + 3]);
  uint32_t cnt = 0;
  uint2 rect = make_uint2(0u, 0u);
  if (!(b[19] < kKillAlpha) && !(pw[0] <= 0.0f || pw[1] <= 0.0f || pw[2] <= 0.0f || pw[3] <= 0.0f)) {
    const float oc = width + soft;
    const float mnx = fminf(fminf(px[0], px[1]), fminf(px[2], px[3])) - oc;
    const float mny = fminf(fminf(py[0], py[1]), fminf(py[2], py[3])) - oc;
    const float mxx = fmaxf(fmaxf(px[0], px[1]), fmaxf(px[2], px[3])) + oc;
    const float mxy = fmaxf(fmaxf(py[0], py[1]), fmaxf(py[2], py[3])) + oc;
    if (bin::tile_rect(tabs, tiles_x, tiles_y, mnx, mny, mxx, mxy, &rect))
      cnt = ((rect.x >> 16) - (rect.x & 0xffffu)) * ((rect.y >> 16) - (rect.y & 0xffffu));
  }
  counts[g] = cnt;
  rects[g] = rect;
}

struct RasterArgs {
  const float* fwd;
  const float* bwd;
  const uint32_t* vals;
  const uint32_t* rstart;
  const uint32_t* rend;
  const float* tgt_rgba;
  const float* tgt_depth;
  const float* bg_rgba;
  const float* bg_depth;
  const float* normal_rgba;
  int32_t* grads;
  float* loss_accum;
  int32_t* pixel_loss;
  float* out_rgbd;
  uint32_t n, w, h, tiles_x, num_tiles;
  Uni u;
  float* ckpt;  // per (view, tile): T of every pixel at the start of each chunk, [kMaxChunks][kThreads]
};

constexpr size_t kRasterSmem = sizeof(uint32_t) * kChunk + sizeof(float) * kChunk * (kRecF + kRecB) +
                               sizeof(float) * 2 * kChunk * kThreads +
                               kChunk * kThreads + sizeof(int32_t) * kChunk * 18 + sizeof(float) * kChunk;

// 16-segment closest-point walk (bezier_backward.wgsl:213-230)
__device__ __forceinline__ void walk(const float* q, float ppx, float ppy, float* min_d, uint32_t* min_k, float* min_u) {
  float md = 1e9f, mu = 0.0f;
  uint32_t mk = 1;
  float2 prev = make_float2(q[0], q[1]);
  for (uint32_t s = 1; s <= kNSeg; ++s) {
    const float2 cur = bezier_at(q, (float)s / (float)kNSeg);
    const float sx = cur.x - prev.x, sy = cur.y - prev.y;
    const float len2 = fmaxf(sx * sx + sy * sy, 1e-8f);
    const float u = clampf(((ppx - prev.x) * sx + (ppy - prev.y) * sy) / len2, 0.0f, 1.0f);
    const float prx = prev.x + u * sx, pry = prev.y + u * sy;
    const float dfx = ppx - prx, dfy = ppy - pry;
    const float d = sqrtf(dfx * dfx + dfy * dfy);
    if (d < md) { md = d; mk = s; mu = u; }
    prev = cur;
  }
  *min_d = md; *min_k = mk; *min_u = mu;
}

// True when the pixel is farther than |width| + |softness| (0.1% + 1e-6
// margin for rounding) from the bounding box of the four projected control
// points.  The curve lies in their convex hull, so every segment of the walk
// is farther still: the coverage smoothstep is exactly 1, alpha exactly 0,
// and the pair changes nothing at this pixel (it is skipped without the walk).
__device__ __forceinline__ bool bz_far(const float* f, float ppx, float ppy) {
  const float mnx = fminf(fminf(f[0], f[2]), fminf(f[4], f[6])), mxx = fmaxf(fmaxf(f[0], f[2]), fmaxf(f[4], f[6]));
  const float mny = fminf(fminf(f[1], f[3]), fminf(f[5], f[7])), mxy = fmaxf(fmaxf(f[1], f[3]), fmaxf(f[5], f[7]));
  const float dx = fmaxf(fmaxf(mnx - ppx, ppx - mxx), 0.0f), dy = fmaxf(fmaxf(mny - ppy, ppy - mxy), 0.0f);
  const float r = (fabsf(f[12]) + fabsf(f[13])) * 1.001f + 1e-6f;
  return dx * dx + dy * dy > r * r;
}

// alpha and segment of one (pixel, curve) pair (bezier_backward.wgsl:231-256)
__device__ __forceinline__ float bz_alpha(const float* f, float ppx, float ppy, uint32_t* kseg, float* dval) {
  float md, mu;
  uint32_t mk;
  walk(f, ppx, ppy, &md, &mk, &mu);
  const float t = ((float)(mk - 1) + mu) / (float)kNSeg;
  const float dt = t - 0.5f;
  const float pressure = 1.0f - 4.0f * dt * dt;
  const float lw = f[12] * pressure, ls = f[13] * pressure, lo = f[14] * pressure;
  const float a_geom = 1.0f - smoothstepf(lw - ls, lw + ls, md);
  const float a = clampf(a_geom * lo, 0.0f, 0.999f);
  const float4 B = bernstein(t);
  const float raw_w = B.x * f[8] + B.y * f[9] + B.z * f[10] + B.w * f[11];
  const float lin_w = fmaxf(raw_w, 0.1f);
  *dval = clampf(1.0f - 0.1f / lin_w, 0.0f, 1.0f);
  *kseg = mk;
  return a;
}

__device__ __forceinline__ float tex_dot(const float* rgba, int32_t x, int32_t y, uint32_t w, float kx, float ky,
                                         float kz) {
  const float4 t = reinterpret_cast<const float4*>(rgba)[(size_t)y * w + x];
  return t.x * kx + t.y * ky + t.z * kz;
}

__global__ void __launch_bounds__(kThreads, 3) k_bz_raster(RasterArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* ids = reinterpret_cast<uint32_t*>(smem);
  float* sf = reinterpret_cast<float*>(smem + sizeof(uint32_t) * kChunk);  // [kChunk][kRecF]
  float* sb = sf + kChunk * kRecF;                                          // [kChunk][kRecB]
  float* sA = sb + kChunk * kRecB;                                          // [kChunk][kThreads]
  float* sT = sA + kChunk * kThreads;
  uint8_t* sK = reinterpret_cast<uint8_t*>(sT + kChunk * kThreads);         // [kChunk][kThreads]
  int32_t* gacc = reinterpret_cast<int32_t*>(sK + kChunk * kThreads);       // [kChunk][18]
  float* lacc = reinterpret_cast<float*>(gacc + kChunk * 18);               // [kChunk]

  const uint32_t tx = blockIdx.x, ty = blockIdx.y, v = blockIdx.z;
  const uint32_t tid = threadIdx.x, lane = tid & 31;
  const uint32_t px = tx * 16 + (tid & 15), py = ty * 16 + (tid >> 4);
  const bool inside = px < A.w && py < A.h;
  const float aspect = (float)A.w / (float)A.h;
  const float ppx = bin::pixel_px(px, A.w, aspect), ppy = bin::pixel_py(py, A.h);
  const uint32_t key = v * A.num_tiles + ty * A.tiles_x + tx;
  // the checkpoints are this CTA's own (32 KB-scale, global memory kept in L2
  // between the forward's write and the backward's read; in shared memory they
  // held residency at two CTAs per SM, here three fit)
  float* ckpt = A.ckpt + (size_t)key * kMaxChunks * kThreads;
  const uint32_t start = A.rstart[key];
  const uint32_t len = min(A.rend[key] - start, kCap);
  const uint32_t nch = (len + kChunk - 1) / kChunk;
  const float* fwd_v = A.fwd + (size_t)v * A.n * kRecF;
  const float* bwd_v = A.bwd + (size_t)v * A.n * kRecB;
  const size_t plane = (size_t)A.w * A.h;
  const size_t pix_local = (size_t)(inside ? py : 0) * A.w + (inside ? px : 0);
  const size_t pix = (size_t)v * plane + pix_local;

  float T = 1.0f, Cr = 0.0f, Cg = 0.0f, Cb = 0.0f, D = 0.0f;
  for (uint32_t c = 0; c < nch; ++c) {
    const uint32_t cnt = min((uint32_t)kChunk, len - c * kChunk);
    __syncthreads();
    if (tid < cnt) ids[tid] = A.vals[start + c * kChunk + tid];
    __syncthreads();
    for (uint32_t e = tid; e < cnt * 5; e += kThreads) {
      const uint32_t k = e / 5, q = e - k * 5;
      reinterpret_cast<float4*>(sf)[k * 5 + q] = reinterpret_cast<const float4*>(fwd_v + (size_t)ids[k] * kRecF)[q];
    }
    ckpt[c * kThreads + tid] = T;
    __syncthreads();
    for (uint32_t k = 0; k < cnt; ++k) {
      const float* f = sf + k * kRecF;
      if (bz_far(f, ppx, ppy)) continue;  // alpha 0: nothing changes
      uint32_t kseg;
      float dv;
      const float a = bz_alpha(f, ppx, ppy, &kseg, &dv);
      Cr += T * a * f[15];
      Cg += T * a * f[16];
      Cb += T * a * f[17];
      D += T * a * dv;
      T = T * (1.0f - a);
    }
  }
  const bool color_mode = A.u.mode > 0.5f;
  float bgr = 0.0f, bgg = 0.0f, bgb = 0.0f, bgd = 1.0f;
  float4 tc = make_float4(0.f, 0.f, 0.f, 0.f);
  float td = 1.0f;
  if (inside) {
    if (color_mode) {
      const float4 bt = reinterpret_cast<const float4*>(A.bg_rgba)[pix];
      bgr = bt.x; bgg = bt.y; bgb = bt.z;
      bgd = A.bg_depth[pix];
    }
    tc = reinterpret_cast<const float4*>(A.tgt_rgba)[pix];
    td = A.tgt_depth[pix];
  }
  Cr += T * bgr; Cg += T * bgg; Cb += T * bgb;
  D += T * bgd;
  if (inside && A.out_rgbd) reinterpret_cast<float4*>(A.out_rgbd)[pix] = make_float4(Cr, Cg, Cb, D);
  // loss, bezier_backward.wgsl:271-320
  const float lw0 = 0.2126f, lw1 = 0.7152f, lw2 = 0.0722f;
  const float dCr_raw = 2.0f * (Cr - tc.x), dCg_raw = 2.0f * (Cg - tc.y), dCb_raw = 2.0f * (Cb - tc.z);
  const bool fgb = td < 0.99f;
  const float dD_total = (fgb && color_mode) ? 0.5f * 2.0f * (D - td) : 0.0f;
  const float luma_err = (dCr_raw * 0.5f) * lw0 + (dCg_raw * 0.5f) * lw1 + (dCb_raw * 0.5f) * lw2;
  const float* tgt_v = A.tgt_rgba + (size_t)v * plane * 4;
  const float* nrm_v = A.normal_rgba + (size_t)v * plane * 4;
  const int32_t ix = (int32_t)px, iy = (int32_t)py, W1 = (int32_t)A.w - 1, H1 = (int32_t)A.h - 1;
  float cw = 1.0f;
  if (inside) {
    const float luma_r = tex_dot(tgt_v, min(max(ix + 1, 0), W1), min(max(iy, 0), H1), A.w, lw0, lw1, lw2);
    const float luma_l = tex_dot(tgt_v, min(max(ix - 1, 0), W1), min(max(iy, 0), H1), A.w, lw0, lw1, lw2);
    const float luma_u = tex_dot(tgt_v, min(max(ix, 0), W1), min(max(iy + 1, 0), H1), A.w, lw0, lw1, lw2);
    const float luma_d = tex_dot(tgt_v, min(max(ix, 0), W1), min(max(iy - 1, 0), H1), A.w, lw0, lw1, lw2);
    const float contrast = sqrtf((luma_r - luma_l) * (luma_r - luma_l) + (luma_u - luma_d) * (luma_u - luma_d));
    cw = 1.0f + clampf(contrast * 8.0f, 0.0f, 3.0f);
  }
  const float dl0 = luma_err * lw0 * 6.0f, dl1 = luma_err * lw1 * 6.0f, dl2 = luma_err * lw2 * 6.0f;
  const float dr_dot = dCr_raw * lw0 + dCg_raw * lw1 + dCb_raw * lw2;
  const float dC0 = (dl0 + (dCr_raw - dr_dot * lw0)) * cw;
  const float dC1 = (dl1 + (dCg_raw - dr_dot * lw1)) * cw;
  const float dC2 = (dl2 + (dCb_raw - dr_dot * lw2)) * cw;
  float dT = (dC0 * bgr + dC1 * bgg + dC2 * bgb) + dD_total * bgd;
  const float coverage = 1.0f - T;
  const float d_cov = A.u.mode < 0.5f ? 2.0f * 2.0f * (coverage - tc.x) : 0.0f;
  dT += -d_cov;
  const float is_bg = (0.995f <= td) ? 1.0f : 0.0f;
  const bool is_fine = A.u.max_width > 0.0f;
  // direction-regulariser flow field (pair independent), bezier_backward.wgsl:449-476
  float fdx = 0.0f, fdy = 0.0f;
  bool has_flow = false;
  if (is_fine && inside) {
    const int32_t rx = min(max(ix + 2, 0), W1), lx = min(max(ix - 2, 0), W1);
    const int32_t uy = min(max(iy + 2, 0), H1), dy = min(max(iy - 2, 0), H1);
    const float cr = tex_dot(tgt_v, rx, iy, A.w, 0.333f, 0.333f, 0.333f);
    const float cl = tex_dot(tgt_v, lx, iy, A.w, 0.333f, 0.333f, 0.333f);
    const float cu = tex_dot(tgt_v, ix, uy, A.w, 0.333f, 0.333f, 0.333f);
    const float cd = tex_dot(tgt_v, ix, dy, A.w, 0.333f, 0.333f, 0.333f);
    const float gx = (cr - cl) * 0.25f * aspect, gy = -(cu - cd) * 0.25f;
    const float nr = tex_dot(nrm_v, rx, iy, A.w, 0.333f, 0.333f, 0.333f);
    const float nl = tex_dot(nrm_v, lx, iy, A.w, 0.333f, 0.333f, 0.333f);
    const float nu = tex_dot(nrm_v, ix, uy, A.w, 0.333f, 0.333f, 0.333f);
    const float nd = tex_dot(nrm_v, ix, dy, A.w, 0.333f, 0.333f, 0.333f);
    const float gnx = (nr - nl) * 0.25f * aspect, gny = -(nu - nd) * 0.25f;
    const float frx = gx + 2.0f * gnx, fry = gy + 2.0f * gny;
    const float flen = sqrtf(frx * frx + fry * fry);
    if (flen > 1e-4f) {
      has_flow = true;
      fdx = frx / flen;
      fdy = fry / flen;
    }
  }

  for (int c = (int)nch - 1; c >= 0; --c) {
    const uint32_t cnt = min((uint32_t)kChunk, len - (uint32_t)c * kChunk);
    __syncthreads();
    if (tid < cnt) ids[tid] = A.vals[start + c * kChunk + tid];
    for (uint32_t e = tid; e < kChunk * 18; e += kThreads) gacc[e] = 0;
    if (tid < kChunk) lacc[tid] = 0.0f;
    __syncthreads();
    for (uint32_t e = tid; e < cnt * 5; e += kThreads) {
      const uint32_t k = e / 5, q = e - k * 5;
      reinterpret_cast<float4*>(sf)[k * 5 + q] = reinterpret_cast<const float4*>(fwd_v + (size_t)ids[k] * kRecF)[q];
    }
    for (uint32_t e = tid; e < cnt * 6; e += kThreads) {
      const uint32_t k = e / 6, q = e - k * 6;
      reinterpret_cast<float4*>(sb)[k * 6 + q] = reinterpret_cast<const float4*>(bwd_v + (size_t)ids[k] * kRecB)[q];
    }
    __syncthreads();
    float Tc = ckpt[c * kThreads + tid];
    for (uint32_t k = 0; k < cnt; ++k) {
      uint32_t kseg = 1;
      float dv = 0.0f;
      const float a = bz_far(sf + k * kRecF, ppx, ppy) ? 0.0f : bz_alpha(sf + k * kRecF, ppx, ppy, &kseg, &dv);
      sA[k * kThreads + tid] = a;
      sT[k * kThreads + tid] = Tc;
      sK[k * kThreads + tid] = (uint8_t)kseg;
      Tc = Tc * (1.0f - a);
    }
    for (int k = (int)cnt - 1; k >= 0; --k) {
      const float a = sA[k * kThreads + tid];
      const bool valid = inside && !(a < 0.001f);
      if (!__any_sync(0xffffffffu, valid)) continue;
      int32_t q[18];
#pragma unroll
      for (int j = 0; j < 18; ++j) q[j] = 0;
      float clc = 0.0f;
      if (valid) {
        const float* f = sf + k * kRecF;
        const float* jb = sb + k * kRecB;
        const float width = f[12], soft = f[13], opacity = f[14];
        const float col0 = f[15], col1 = f[16], col2 = f[17];
        const float T_prev = sT[k * kThreads + tid];
        const uint32_t kseg = sK[k * kThreads + tid];
        const float t_prev = (float)(kseg - 1) / (float)kNSeg, t_curr = (float)kseg / (float)kNSeg;
        const float2 pp = bezier_at(f, t_prev), cp = bezier_at(f, t_curr);
        const float segx = cp.x - pp.x, segy = cp.y - pp.y;
        const float len2 = fmaxf(segx * segx + segy * segy, 1e-8f);
        const float u_c = clampf(((ppx - pp.x) * segx + (ppy - pp.y) * segy) / len2, 0.0f, 1.0f);
        const float prx = pp.x + u_c * segx, pry = pp.y + u_c * segy;
        const float dvx = ppx - prx, dvy = ppy - pry;
        const float d = fmaxf(sqrtf(dvx * dvx + dvy * dvy), 1e-6f);
        const float t_pix = ((float)(kseg - 1) + u_c) / (float)kNSeg;
        const float dtp = t_pix - 0.5f;
        const float pressure = 1.0f - 4.0f * dtp * dtp;
        const float4 Bp = bernstein(t_pix);
        // depth value of the pair: the forward's, recomputed (same t, same ops)
        const float raw_wf = Bp.x * f[8] + Bp.y * f[9] + Bp.z * f[10] + Bp.w * f[11];
        const float d_val = clampf(1.0f - 0.1f / fmaxf(raw_wf, 0.1f), 0.0f, 1.0f);
        const float TA = T_prev * a;
        const float dColor0 = dC0 * TA, dColor1 = dC1 * TA, dColor2 = dC2 * TA;
        const float tc0 = T_prev * col0, tc1 = T_prev * col1, tc2 = T_prev * col2;
        const float da = dT * (-T_prev) + (dC0 * tc0 + dC1 * tc1 + dC2 * tc2) + dD_total * (T_prev * d_val);
        const float ac0 = a * col0, ac1 = a * col1, ac2 = a * col2;
        dT = dT * (1.0f - a) + (dC0 * ac0 + dC1 * ac1 + dC2 * ac2) + dD_total * (a * d_val);
        const float lwid = width * pressure, lsoft = soft * pressure, lop = opacity * pressure;
        const float inner = lwid - lsoft, outer = lwid + lsoft;
        const float denom = fmaxf(outer - inner, 1e-6f);
        const float x_in = clampf((d - inner) / denom, 0.0f, 1.0f);
        const float ss_d = 6.0f * x_in * (1.0f - x_in) / denom;
        const bool in_band = (d > inner) && (d < outer);
        const float a_geom = 1.0f - smoothstepf(inner, outer, d);
        const float bg_pen = A.u.bg_penalty * is_bg;
        const float d_opacity = da * a_geom * pressure + bg_pen;
        const float da_eff = da * lop;
        const float dDd = in_band ? -da_eff * ss_d : 0.0f;
        const float dWidth = in_band ? da_eff * ss_d * pressure / denom : 0.0f;
        const float dmi = clampf(d - inner, 0.0f, denom);
        const float dx_ds = pressure * (denom - 2.0f * dmi) / fmaxf(denom * denom, 1e-12f);
        float dSoft = in_band ? -da_eff * ss_d * dx_ds : 0.0f;
        const float raw_w = Bp.x * f[8] + Bp.y * f[9] + Bp.z * f[10] + Bp.w * f[11];
        const float lin_w = fmaxf(raw_w, 0.1f);
        const float ddw = 0.1f / (lin_w * lin_w);
        const float kz = dD_total * (T_prev * a) * ddw;
        const float dZ[4] = {kz * Bp.x, kz * Bp.y, kz * Bp.z, kz * Bp.w};
        const float dprx = -dDd * dvx / d, dpry = -dDd * dvy / d;
        const float dPx = (1.0f - u_c) * dprx, dPy = (1.0f - u_c) * dpry;
        const float dQx = u_c * dprx, dQy = u_c * dpry;
        const float4 Bpv = bernstein(t_prev), Bcv = bernstein(t_curr);
        const float bpv[4] = {Bpv.x, Bpv.y, Bpv.z, Bpv.w}, bcv[4] = {Bcv.x, Bcv.y, Bcv.z, Bcv.w};
        dSoft += is_fine ? 5.0f * 2.0f * soft : 0.0f;
        if (is_fine && len2 > 1e-10f && has_flow) {
          const float sl = sqrtf(len2);
          const float tgx = segx / sl, tgy = segy / sl;
          const float tg = tgx * fdx + tgy * fdy;
          const float dld = 1.5f * 2.0f * tg;
          const float dtvx = dld * fdx, dtvy = dld * fdy;
          const float il = 1.0f / sqrtf(len2);
          const float tdot = dtvx * tgx + dtvy * tgy;
          const float dsx = (dtvx - tgx * tdot) * il, dsy = (dtvy - tgy * tdot) * il;
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) {
            const float ex = bpv[cc] * (-dsx) + bcv[cc] * dsx;
            const float ey = bpv[cc] * (-dsy) + bcv[cc] * dsy;
#pragma unroll
            for (int ax = 0; ax < 3; ++ax)
              q[3 * cc + ax] += to_i32((ex * jb[6 * cc + ax] + ey * jb[6 * cc + 3 + ax]) * kFpPos);
          }
        }
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          const float ex = bpv[cc] * dPx + bcv[cc] * dQx;
          const float ey = bpv[cc] * dPy + bcv[cc] * dQy;
          const float g0 = ex * jb[6 * cc + 0] + ey * jb[6 * cc + 3];
          const float g1 = ex * jb[6 * cc + 1] + ey * jb[6 * cc + 4];
          const float g2 = ex * jb[6 * cc + 2] + ey * jb[6 * cc + 5];
          q[3 * cc + 0] += to_i32(g0 * kFpPos);
          q[3 * cc + 1] += to_i32(g1 * kFpPos);
          q[3 * cc + 2] += to_i32((g2 + dZ[cc]) * kFpPos);
        }
        q[12] = to_i32(dColor0 * kFpCol);
        q[13] = to_i32(dColor1 * kFpCol);
        q[14] = to_i32(dColor2 * kFpCol);
        q[15] = to_i32(d_opacity * kFpCol);
        q[16] = to_i32(dWidth * kFpPos);
        q[17] = to_i32(dSoft * kFpPos);
        clc = (dC0 * dC0 * 1.0f + dC1 * dC1 * 1.0f + dC2 * dC2 * 1.0f) * (T_prev * a);
      }
#pragma unroll
      for (int j = 0; j < 18; ++j) {
        const int32_t r = __reduce_add_sync(0xffffffffu, q[j]);
        if (lane == 0 && r != 0) atomicAdd(&gacc[k * 18 + j], r);
      }
      float cl = clc;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) cl += __shfl_xor_sync(0xffffffffu, cl, o);
      if (lane == 0 && cl != 0.0f) atomicAdd(&lacc[k], cl);
    }
    __syncthreads();
    for (uint32_t e = tid; e < cnt * 18; e += kThreads) {
      const int32_t val = gacc[e];
      if (val != 0) atomicAdd(&A.grads[18 * (size_t)ids[e / 18] + (e % 18)], val);
    }
    if (tid < cnt && lacc[tid] != 0.0f) atomicAdd(&A.loss_accum[ids[tid]], lacc[tid]);
  }
  if (inside) {
    // per-pixel residual for ADC seeding (bezier_backward.wgsl:568-571); the
    // reference indexes y * W + x into a 512 x 512 buffer
    const float hr = dCr_raw * 0.5f, hg = dCg_raw * 0.5f, hb = dCb_raw * 0.5f;
    const float residual = (hr * hr + hg * hg + hb * hb) * T;
    const size_t idx = pix_local;
    if (idx < kPixelLossSize) atomicAdd(&A.pixel_loss[idx], to_i32(residual * 10000.0f));
  }
}

__constant__ float c_lr[18] = {0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f,
                               0.005f, 0.005f, 0.005f, 0.01f, 0.01f, 0.01f, 0.005f, 0.002f, 0.002f};
__constant__ float c_mu[18] = {0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f,
                               0.005f, 0.005f, 0.005f, 0.01f, 0.01f, 0.01f, 0.005f, 0.003f, 0.003f};
__constant__ int c_off[18] = {0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14, 16, 17, 18, 19, 3, 7};

struct StepArgs {
  float bc1, bc2, pixel_norm, no_kill, width_hi, alpha_thresh, width_thresh;
  float vp[16];
};

// bezier_step.wgsl:50-189, one thread per curve
__global__ void __launch_bounds__(128) k_bz_step(float* __restrict__ bz, int32_t* __restrict__ grads,
                                                 float* __restrict__ am, float* __restrict__ av,
                                                 float* __restrict__ gacc, uint32_t n, StepArgs s) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float b[20];
  float4* b4 = reinterpret_cast<float4*>(bz + 20 * (size_t)i);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const float4 t = b4[q];
    b[4 * q] = t.x; b[4 * q + 1] = t.y; b[4 * q + 2] = t.z; b[4 * q + 3] = t.w;
  }
  int2* g2 = reinterpret_cast<int2*>(grads + 18 * (size_t)i);
  if (b[19] < kKillAlpha) {
#pragma unroll
    for (int q = 0; q < 9; ++q) g2[q] = make_int2(0, 0);
    return;
  }
  int32_t g[18];
  float m[18], v[18];
  float2* m2 = reinterpret_cast<float2*>(am + 18 * (size_t)i);
  float2* v2 = reinterpret_cast<float2*>(av + 18 * (size_t)i);
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const int2 a = g2[q];
    const float2 mm = m2[q], vv = v2[q];
    g[2 * q] = a.x; g[2 * q + 1] = a.y;
    m[2 * q] = mm.x; m[2 * q + 1] = mm.y;
    v[2 * q] = vv.x; v[2 * q + 1] = vv.y;
  }
  const float B1 = 0.9f, B2 = 0.999f, EPS = 1e-8f;
  float pos_g2 = 0.0f;
#pragma unroll
  for (int k = 0; k < 18; ++k) {
    const float fps = (k >= 12 && k <= 15) ? kFpCol : kFpPos;
    const float gr = (float)g[k] / fps * s.pixel_norm;
    const float mm = B1 * m[k] + (1.0f - B1) * gr;
    const float vv = B2 * v[k] + (1.0f - B2) * gr * gr;
    m[k] = mm;
    v[k] = vv;
    const float m_hat = mm / s.bc1, v_hat = vv / s.bc2;
    const float raw_u = c_lr[k] * m_hat / (sqrtf(v_hat) + EPS);
    const float u = clampf(raw_u, -c_mu[k], c_mu[k]);
    const float lo = k < 12 ? -1e9f : (k < 16 ? 0.0f : 0.001f);
    const float hi = k < 12 ? 1e9f : (k < 15 ? 1.0f : (k == 15 ? 0.99f : (k == 16 ? s.width_hi : 0.03f)));
    b[c_off[k]] = clampf(b[c_off[k]] - u, lo, hi);
    if (k <= 11) pos_g2 += gr * gr;
  }
  gacc[i] = gacc[i] + sqrtf(pos_g2);
  if (b[19] < s.alpha_thresh || b[3] <= s.width_thresh) b[19] = 0.0f;
  if (b[19] > 0.0f && s.no_kill < 0.5f) {
    const float mg = 1.2f;  // BEZIER_OFFSCREEN_MARGIN, constants.ts:14
    bool L = true, R = true, Bo = true, Ab = true, Be = true;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const float4 cl = mulv(s.vp, b[4 * c], b[4 * c + 1], b[4 * c + 2], 1.0f);
      L = L && cl.x < -mg * cl.w;
      R = R && cl.x > mg * cl.w;
      Bo = Bo && cl.y < -mg * cl.w;
      Ab = Ab && cl.y > mg * cl.w;
      Be = Be && cl.w < 0.0f;
    }
    if (L || R || Bo || Ab || Be) b[19] = 0.0f;
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) b4[q] = make_float4(b[4 * q], b[4 * q + 1], b[4 * q + 2], b[4 * q + 3]);
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    g2[q] = make_int2(0, 0);
    m2[q] = make_float2(m[2 * q], m[2 * q + 1]);
    v2[q] = make_float2(v[2 * q], v[2 * q + 1]);
  }
}

constexpr int kAdcThreads = 1024;

__device__ __forceinline__ uint32_t block_scan_excl(uint32_t x, uint32_t* total) {
  __shared__ uint32_t warp_sums[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_sums[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    const uint32_t s0 = warp_sums[lane];
    uint32_t si = s0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += y;
    }
    warp_sums[lane] = si - s0;
    if (lane == 31) *total = si;
  }
  __syncthreads();
  const uint32_t r = warp_sums[wid] + inc - x;
  __syncthreads();
  return r;
}

struct AdcArgs {
  float adam_t, no_kill;
  float vp[16], vp_inv[16];
  uint32_t n;
};

// clone or split curve i into slot ni (bezier_adc.wgsl:323-370)
__device__ void clone_split(float* __restrict__ bz, float* __restrict__ am, float* __restrict__ av, uint32_t i,
                            uint32_t ni, float adam_t) {
  float b[20], nb[20];
  float4* b4 = reinterpret_cast<float4*>(bz + 20 * (size_t)i);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const float4 t = b4[q];
    b[4 * q] = t.x; b[4 * q + 1] = t.y; b[4 * q + 2] = t.z; b[4 * q + 3] = t.w;
  }
#pragma unroll
  for (int k = 0; k < 20; ++k) nb[k] = b[k];
  float p[4][3];
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int k = 0; k < 3; ++k) p[c][k] = b[4 * c + k];
  float mid[3], da[3], db[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    mid[k] = (p[0][k] + 3.0f * p[1][k] + 3.0f * p[2][k] + p[3][k]) * 0.125f;
    da[k] = mid[k] - p[0][k];
    db[k] = p[3][k] - mid[k];
  }
  const float la = sqrtf(da[0] * da[0] + da[1] * da[1] + da[2] * da[2]);
  const float lb = sqrtf(db[0] * db[0] + db[1] * db[1] + db[2] * db[2]);
  if (la + lb > 0.25f) {  // BEZIER_SPLIT_LEN_THRESHOLD, constants.ts:9
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float q0 = (p[0][k] + p[1][k]) * 0.5f, q1 = (p[1][k] + p[2][k]) * 0.5f, q2 = (p[2][k] + p[3][k]) * 0.5f;
      const float r0 = (q0 + q1) * 0.5f, r1 = (q1 + q2) * 0.5f, s = (r0 + r1) * 0.5f;
      b[0 + k] = p[0][k]; b[4 + k] = q0; b[8 + k] = r0; b[12 + k] = s;
      nb[0 + k] = s; nb[4 + k] = r1; nb[8 + k] = q2; nb[12 + k] = p[3][k];
    }
    b[11] = 0.0f; b[15] = 0.0f; nb[11] = 0.0f; nb[15] = 0.0f;
  } else {
    const float seed = (float)i * 3.14159f + adam_t;
    const float j[3] = {(fractf(sinf(seed * 12.9898f) * 43758.5453f) - 0.5f) * 0.001f,
                        (fractf(sinf(seed * 78.233f) * 43758.5453f) - 0.5f) * 0.001f,
                        (fractf(sinf(seed * 43.123f) * 43758.5453f) - 0.5f) * 0.001f};
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int k = 0; k < 3; ++k) nb[4 * c + k] = b[4 * c + k] + j[k];
    nb[11] = 0.0f; nb[15] = 0.0f;
  }
  float4* n4 = reinterpret_cast<float4*>(bz + 20 * (size_t)ni);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    b4[q] = make_float4(b[4 * q], b[4 * q + 1], b[4 * q + 2], b[4 * q + 3]);
    n4[q] = make_float4(nb[4 * q], nb[4 * q + 1], nb[4 * q + 2], nb[4 * q + 3]);
  }
  float2* mi = reinterpret_cast<float2*>(am + 18 * (size_t)i);
  float2* vi = reinterpret_cast<float2*>(av + 18 * (size_t)i);
  float2* mn = reinterpret_cast<float2*>(am + 18 * (size_t)ni);
  float2* vn = reinterpret_cast<float2*>(av + 18 * (size_t)ni);
  const float2 z = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int q = 0; q < 9; ++q) { mi[q] = z; vi[q] = z; mn[q] = z; vn[q] = z; }
}

__device__ __forceinline__ bool offscreen(const float* vp, const float* p3) {
  const float4 c = mulv(vp, p3[0], p3[1], p3[2], 1.0f);
  if (c.w < 0.0f) return true;
  const float iw = fmaxf(c.w, 1e-5f);
  const float nx = c.x / iw, ny = c.y / iw;
  return fabsf(nx) > 1.2f || fabsf(ny) > 1.2f;
}

// One clone/split pass (bezier_adc.wgsl:310-371 and :434-494) over the
// current state, serial semantics: the k-th candidate (ascending index) takes
// dead[dead_count - 1 - k].  A candidate whose slot lies ahead of it inside
// the 1024 window makes that slot alive (with its accumulator) before the
// serial loop reaches it: the window is committed up to that slot and
// restarted there.  Returns the new dead_count.
__device__ uint32_t clone_pass(float* __restrict__ bz, float* __restrict__ am, float* __restrict__ av,
                               const float* __restrict__ gacc, const uint32_t* __restrict__ dead,
                               uint32_t dead_count, const AdcArgs& a, uint32_t* s_total, uint32_t* s_min,
                               uint32_t* clones) {
  const float P = 50.0f, TAU_POS = 0.0002f;  // constants.ts:6-7 (the shader divides by the constant)
  uint32_t base = 0;
  const uint32_t tid = threadIdx.x;
  while (base < a.n) {
    const uint32_t i = base + tid;
    const bool inwin = i < a.n;
    bool cand = false;
    if (inwin) {
      const float op = bz[20 * (size_t)i + 19];
      cand = !(op < kKillAlpha) && !(gacc[i] / P <= TAU_POS);
    }
    const uint32_t r = block_scan_excl(cand ? 1u : 0u, s_total);
    const bool has_slot = cand && r < dead_count;
    const uint32_t d = has_slot ? dead[dead_count - 1 - r] : 0u;
    if (tid == 0) *s_min = 0xffffffffu;
    __syncthreads();
    if (has_slot && d > i && d < base + kAdcThreads) atomicMin(s_min, d);
    __syncthreads();
    const uint32_t commit_end = *s_min == 0xffffffffu ? base + kAdcThreads : *s_min;
    const bool commit = inwin && i < commit_end && has_slot;
    if (commit) clone_split(bz, am, av, i, d, a.adam_t);
    const uint32_t used = __syncthreads_count(commit);
    dead_count -= used;
    *clones += used;
    __threadfence_block();
    __syncthreads();
    base = commit_end;
  }
  return dead_count;
}

// bezier_adc.wgsl:75-315 in one CTA.
__global__ void __launch_bounds__(kAdcThreads) k_bz_adc(float* __restrict__ bz, float* __restrict__ am,
                                                        float* __restrict__ av, float* __restrict__ gacc,
                                                        float* __restrict__ lacc, int32_t* __restrict__ pixel_loss,
                                                        uint32_t* __restrict__ dead, uint32_t* __restrict__ stats,
                                                        AdcArgs a) {
  __shared__ uint32_t s_total, s_min;
  __shared__ int32_t s_bv[32];
  __shared__ uint32_t s_bp[32];
  const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const float P = 50.0f, TAU_POS = 0.0002f, TAU_LOSS = 0.001f;  // constants.ts:6-8
  // dead slots in index order (bezier_adc.wgsl:77-82)
  uint32_t dc = 0;
  for (uint32_t base = 0; base < a.n; base += kAdcThreads) {
    const uint32_t i = base + tid;
    const uint32_t f = (i < a.n && bz[20 * (size_t)i + 19] < kKillAlpha) ? 1u : 0u;
    const uint32_t r = block_scan_excl(f, &s_total);
    if (f) dead[dc + r] = i;
    dc += s_total;
    __syncthreads();
  }
  // pass 1: kill stuck + lossy and offscreen curves, appended in index order
  for (uint32_t base = 0; base < a.n; base += kAdcThreads) {
    const uint32_t i = base + tid;
    uint32_t kill = 0;
    if (i < a.n) {
      float* b = bz + 20 * (size_t)i;
      if (!(b[19] < kKillAlpha)) {
        const float gn = gacc[i] / P, ln = lacc[i] / P;
        if (a.no_kill < 0.5f && gn <= TAU_POS && ln > TAU_LOSS) kill = 1;
        else if (offscreen(a.vp, b) && offscreen(a.vp, b + 4) && offscreen(a.vp, b + 8) && offscreen(a.vp, b + 12))
          kill = 1;
        if (kill) b[19] = 0.0f;
      }
    }
    const uint32_t r = block_scan_excl(kill, &s_total);
    if (kill) dead[dc + r] = i;
    dc += s_total;
    __syncthreads();
  }
  uint32_t clones = 0;
  // pass 1.5
  dc = clone_pass(bz, am, av, gacc, dead, dc, a, &s_total, &s_min, &clones);
  // pass 2: spawn at the highest-loss pixels (strided scan, bezier_adc.wgsl:376-432)
  const uint32_t stride = max(1u, kPixelLossSize / 4096u);
  const uint32_t max_spawns = min(dc, 512u);
  uint32_t spawns = 0;
  for (uint32_t sp = 0; sp < max_spawns; ++sp) {
    if (dc == 0) break;
    const uint32_t start = (sp * 997u) % stride;
    int32_t bv = 0;
    uint32_t bp = 0xffffffffu;
    for (uint32_t k = tid; k * stride + start < kPixelLossSize; k += kAdcThreads) {
      const uint32_t px = start + k * stride;
      const int32_t v = pixel_loss[px];
      if (v > bv) { bv = v; bp = px; }
    }
    // block arg-max, first maximum in scan order (smallest pixel index)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const int32_t ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const uint32_t op = __shfl_xor_sync(0xffffffffu, bp, o);
      if (ov > bv || (ov == bv && op < bp)) { bv = ov; bp = op; }
    }
    if (lane == 0) { s_bv[wid] = bv; s_bp[wid] = bp; }
    __syncthreads();
    if (tid == 0) {
      int32_t best_val = 0;
      uint32_t best_px = 0xffffffffu;
      for (int w = 0; w < kAdcThreads / 32; ++w)
        if (s_bv[w] > best_val || (s_bv[w] == best_val && s_bv[w] > 0 && s_bp[w] < best_px)) {
          best_val = s_bv[w];
          best_px = s_bp[w];
        }
      uint32_t spawn_px;
      if (best_val <= 0) {
        const float sf = (float)sp * 1234.5678f + a.adam_t * 0.1f;
        const uint32_t rx = (uint32_t)fmaxf(0.0f, fractf(sinf(sf * 12.9898f) * 43758.5453f) * 256.0f);
        const uint32_t ry = (uint32_t)fmaxf(0.0f, fractf(sinf(sf * 78.233f) * 43758.5453f) * 256.0f);
        spawn_px = ry * 256u + rx;
      } else {
        spawn_px = best_px;
        pixel_loss[best_px] = 0;
      }
      dc -= 1;
      const uint32_t slot = dead[dc];
      // pixel_to_world at depth 0.5, bezier_adc.wgsl:52-65 (OPTIM 256 x 256)
      const uint32_t pxx = spawn_px % 256u, pyy = spawn_px / 256u;
      const float ux = ((float)pxx + 0.5f) / 256.0f, uy = ((float)pyy + 0.5f) / 256.0f;
      const float ndx = ux * 2.0f - 1.0f, ndy = 1.0f - uy * 2.0f;
      const float wv = 0.1f / fmaxf(1.0f - 0.5f, 1e-5f);
      const float4 wp = mulv(a.vp_inv, ndx * wv, ndy * wv, wv, wv);
      const float cx = wp.x / wp.w, cy = wp.y / wp.w, cz = wp.z / wp.w;
      const float seed = (float)spawn_px * 1.61803f + (float)sp * 2.71828f;
      const float ang = fractf(sinf(seed * 127.1f) * 43758.5453f) * 6.28318f;
      const float tgx = cosf(ang) * 0.025f, tgz = sinf(ang) * 0.025f;  // BEZIER_SPAWN_TANGENT_LEN
      float* nb = bz + 20 * (size_t)slot;
      nb[0] = cx - tgx; nb[1] = cy - 0.0f; nb[2] = cz - tgz; nb[3] = 0.015f;
      nb[4] = cx - tgx * 0.33f; nb[5] = cy - 0.0f * 0.33f; nb[6] = cz - tgz * 0.33f; nb[7] = 0.005f;
      nb[8] = cx + tgx * 0.33f; nb[9] = cy + 0.0f * 0.33f; nb[10] = cz + tgz * 0.33f; nb[11] = 0.0f;
      nb[12] = cx + tgx; nb[13] = cy + 0.0f; nb[14] = cz + tgz; nb[15] = 0.0f;
      nb[16] = 0.5f; nb[17] = 0.5f; nb[18] = 0.5f; nb[19] = 0.5f;
      for (int k = 0; k < 18; ++k) { am[18 * (size_t)slot + k] = 0.0f; av[18 * (size_t)slot + k] = 0.0f; }
      s_total = dc;
    }
    __syncthreads();
    dc = s_total;
    ++spawns;
    __threadfence_block();
    __syncthreads();
  }
  // pass 3
  if (dc > 0) dc = clone_pass(bz, am, av, gacc, dead, dc, a, &s_total, &s_min, &clones);
  __syncthreads();
  for (uint32_t k = tid; k < kPixelLossSize; k += kAdcThreads) pixel_loss[k] = 0;
  for (uint32_t k = tid; k < a.n; k += kAdcThreads) { gacc[k] = 0.0f; lacc[k] = 0.0f; }
  if (tid == 0 && stats) { stats[0] = clones; stats[1] = spawns; }
}


// ------------------------------------------------------------- display forward
// bezier_forward.wgsl:48-182 headless: each curve covers its hull box +-
// (width + softness), clamped to +-4 (SCREEN_BOUND) and culled if any control
// point has w <= 0; the fragment walks the 16 segments, applies pressure,
// coverage and (optionally) the brush alpha, and composites premultiplied,
// front to back with curve 0 in front (reverse instance order in the
// reference), over the given background.
constexpr int kBRend = 20;

__global__ void __launch_bounds__(256) k_bz_render_project(const float* __restrict__ bz, uint32_t n,
                                                           const float* __restrict__ vp, uint32_t w, uint32_t h,
                                                           const float* __restrict__ tabs, uint32_t tiles_x,
                                                           uint32_t tiles_y, float* __restrict__ rec,
                                                           uint32_t* __restrict__ counts, uint2* __restrict__ rects) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float b[20];
  const float4* b4 = reinterpret_cast<const float4*>(bz + 20 * (size_t)i);
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    const float4 t = b4[q];
    b[4 * q] = t.x; b[4 * q + 1] = t.y; b[4 * q + 2] = t.z; b[4 * q + 3] = t.w;
  }
  const float aspect = (float)w / (float)h;
  float px[4], py[4];
  bool ok = true;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float4 cl = mulv(vp, b[4 * c], b[4 * c + 1], b[4 * c + 2], 1.0f);
    px[c] = cl.x / cl.w * aspect;
    py[c] = cl.y / cl.w;
    ok = ok && !(cl.w <= 0.0f);
  }
  uint32_t cnt = 0;
  uint2 rect = make_uint2(0u, 0u);
  if (ok) {
    const float width = fmaxf(b[3], 0.0001f), soft = fmaxf(b[7], 0.0001f), pad = width + soft;
    const float SB = 4.0f;
    const float x0 = fmaxf(fminf(fminf(px[0], px[1]), fminf(px[2], px[3])) - pad, -SB);
    const float y0 = fmaxf(fminf(fminf(py[0], py[1]), fminf(py[2], py[3])) - pad, -SB);
    const float x1 = fminf(fmaxf(fmaxf(px[0], px[1]), fmaxf(px[2], px[3])) + pad, SB);
    const float y1 = fminf(fmaxf(fmaxf(py[0], py[1]), fmaxf(py[2], py[3])) + pad, SB);
    float4* r4 = reinterpret_cast<float4*>(rec + (size_t)i * kBRend);
    r4[0] = make_float4(px[0], py[0], px[1], py[1]);
    r4[1] = make_float4(px[2], py[2], px[3], py[3]);
    r4[2] = make_float4(x0, x1, y0, y1);
    r4[3] = make_float4(width, soft, b[19], b[16]);
    r4[4] = make_float4(b[17], b[18], 0.0f, 0.0f);
    if (bin::tile_rect(tabs, tiles_x, tiles_y, x0, y0, x1, y1, &rect))
      cnt = ((rect.x >> 16) - (rect.x & 0xffffu)) * ((rect.y >> 16) - (rect.y & 0xffffu));
  }
  counts[i] = cnt;
  rects[i] = rect;
}

__device__ __forceinline__ float brush_sample(const float* brush, uint32_t bw, uint32_t bh, float u, float v) {
  if (!brush) return 1.0f;
  const float x = u * (float)bw - 0.5f, y = v * (float)bh - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const float ax = x - fx, ay = y - fy;
  const int ix = (int)fx, iy = (int)fy;
  auto at = [&](int xx, int yy) {
    xx = ((xx % (int)bw) + (int)bw) % (int)bw;
    yy = min(max(yy, 0), (int)bh - 1);
    return brush[(size_t)yy * bw + xx];
  };
  return (1 - ay) * ((1 - ax) * at(ix, iy) + ax * at(ix + 1, iy)) + ay * ((1 - ax) * at(ix, iy + 1) + ax * at(ix + 1, iy + 1));
}

__global__ void __launch_bounds__(256) k_bz_render_raster(const float* __restrict__ rec,
                                                          const uint32_t* __restrict__ vals,
                                                          const uint32_t* __restrict__ rstart,
                                                          const uint32_t* __restrict__ rend, uint32_t w, uint32_t h,
                                                          uint32_t tiles_x, const float4* __restrict__ bg,
                                                          const float* __restrict__ brush, uint32_t bw, uint32_t bh,
                                                          float4* __restrict__ out) {
  __shared__ float sr[128][kBRend];
  const uint32_t tx = blockIdx.x, ty = blockIdx.y, tid = threadIdx.x;
  const uint32_t px = tx * 16 + (tid & 15), py = ty * 16 + (tid >> 4);
  const bool inside = px < w && py < h;
  const float aspect = (float)w / (float)h;
  const float ppx = bin::pixel_px(px, w, aspect), ppy = bin::pixel_py(py, h);
  const uint32_t key = ty * tiles_x + tx;
  const uint32_t start = rstart[key], end = rend[key];
  float T = 1.0f, C0 = 0.0f, C1 = 0.0f, C2 = 0.0f, C3 = 0.0f;
  for (uint32_t base = start; base < end; base += 128) {
    __syncthreads();
    const uint32_t nb = min(128u, end - base);
    for (uint32_t e = tid; e < nb * 5; e += 256) {
      const uint32_t k = e / 5, q = e - k * 5;
      reinterpret_cast<float4*>(&sr[k][0])[q] = reinterpret_cast<const float4*>(rec + (size_t)vals[base + k] * kBRend)[q];
    }
    __syncthreads();
    for (uint32_t j = 0; j < nb; ++j) {
      const float* f = sr[j];
      if (!(ppx >= f[8] && ppx < f[9] && ppy > f[10] && ppy <= f[11])) continue;
      if (bz_far(f, ppx, ppy)) continue;  // alpha 0
      float md = 1e9f, mu = 0.0f, cross = 0.0f;
      uint32_t mk = 1;
      float2 prev = make_float2(f[0], f[1]);
      for (uint32_t s = 1; s <= kNSeg; ++s) {
        const float2 cur = bezier_at(f, (float)s / (float)kNSeg);
        const float sx = cur.x - prev.x, sy = cur.y - prev.y;
        const float len2 = fmaxf(sx * sx + sy * sy, 1e-8f);
        const float u = clampf(((ppx - prev.x) * sx + (ppy - prev.y) * sy) / len2, 0.0f, 1.0f);
        const float prx = prev.x + u * sx, pry = prev.y + u * sy;
        const float dfx = ppx - prx, dfy = ppy - pry;
        const float d = sqrtf(dfx * dfx + dfy * dfy);
        if (d < md) {
          md = d; mk = s; mu = u;
          const float sl = sqrtf(len2);
          cross = dfx * (-(sy / sl)) + dfy * (sx / sl);
        }
        prev = cur;
      }
      const float t = ((float)(mk - 1) + mu) / (float)kNSeg;
      const float dt = t - 0.5f;
      const float pressure = 1.0f - 4.0f * dt * dt;
      const float lw = f[12] * pressure, ls = f[13] * pressure, lo = f[14] * pressure;
      const float a_geom = 1.0f - smoothstepf(lw - ls, lw + ls, md);
      const float bv = clampf(cross / fmaxf(lw + ls, 1e-6f) * 0.5f + 0.5f, 0.0f, 1.0f);
      const float a = clampf(a_geom * brush_sample(brush, bw, bh, t, bv) * lo, 0.0f, 0.999f);
      if (a < 0.001f) continue;
      C0 += T * f[15] * a;
      C1 += T * f[16] * a;
      C2 += T * f[17] * a;
      C3 += T * a;
      T *= (1.0f - a);
    }
  }
  if (inside) {
    const size_t pix = (size_t)py * w + px;
    const float4 g = bg ? bg[pix] : make_float4(0.f, 0.f, 0.f, 0.f);
    out[pix] = make_float4(C0 + T * g.x, C1 + T * g.y, C2 + T * g.z, C3 + T * g.w);
  }
}

}  // namespace bz
}  // namespace nps

// =================================================================== host side
using namespace nps;

struct nps_bezier_opt {
  nps_ctx* ctx = nullptr;
  uint32_t n = 0;
  DevBuf params, grads, am, av, gacc, lacc, pixel_loss, dead, stat;
  float adam_t = 0.0f;
  uint32_t step_count = 0, adc_period = 50;
  bz::Uni uni{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  float no_kill = 0.0f;
  uint32_t nv = 0;
  std::vector<float> views_host;  // nv * 32: vp, vp_inv
  DevBuf views;
  uint32_t w = 0, h = 0, tv = 0;
  DevBuf own[5];
  const float* tex[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // target, target depth, bg, bg depth, normal
  DevBuf fwd, bwd, counts, offsets, rects, total, keys, vals, ranges, tabs;
  DevBuf ckbuf;  // raster checkpoints per (view, tile)
  SortWork sw;
  uint32_t pair_cap = 0;
  nps_stats stats{};
  // display render work buffers
  DevBuf r_rec, r_counts, r_offsets, r_rects, r_total, r_cam, r_keys, r_vals, r_ranges, r_tabs;
  SortWork r_sw;
  uint32_t r_pair_cap = 0;
};

namespace {
int check_bz(nps_bezier_opt* o) {
  if (!o) {
    set_error("null Bezier optimizer");
    return NPS_ERR_INVALID;
  }
  return bind_device(o->ctx);
}
int copy_in_bz(void* dst, const void* src, size_t bytes, int mem, cudaStream_t s) {
  if (bytes == 0) return NPS_OK;
  if (!src) {
    set_error("null source pointer");
    return NPS_ERR_INVALID;
  }
  if (mem == NPS_MEM_HOST) {
    NPS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    NPS_CUDA(cudaStreamSynchronize(s));
  } else {
    NPS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
  }
  return NPS_OK;
}
}  // namespace

extern "C" {

int nps_bezier_opt_create(nps_ctx* ctx, uint32_t num_beziers, nps_bezier_opt** out) {
  if (!out || num_beziers == 0 || num_beziers > (1u << 25)) {
    set_error("nps_bezier_opt_create: bad arguments (num_beziers=%u)", num_beziers);
    return NPS_ERR_INVALID;
  }
  *out = nullptr;
  NPS_TRY(bind_device(ctx));
  nps_bezier_opt* o = new nps_bezier_opt();
  o->ctx = ctx;
  o->n = num_beziers;
  const size_t n = num_beziers;
  int rc = NPS_OK;
  if ((rc = o->params.ensure(sizeof(float) * 20 * n)) || (rc = o->grads.ensure(sizeof(int32_t) * 18 * n)) ||
      (rc = o->am.ensure(sizeof(float) * 18 * n)) || (rc = o->av.ensure(sizeof(float) * 18 * n)) ||
      (rc = o->gacc.ensure(sizeof(float) * n)) || (rc = o->lacc.ensure(sizeof(float) * n)) ||
      (rc = o->pixel_loss.ensure(sizeof(int32_t) * bz::kPixelLossSize)) || (rc = o->dead.ensure(sizeof(uint32_t) * n)) ||
      (rc = o->stat.ensure(64)) || (rc = o->total.ensure(16))) {
    delete o;
    return rc;
  }
  cudaStream_t s = ctx->stream;
  cudaMemsetAsync(o->params.p, 0, sizeof(float) * 20 * n, s);
  cudaMemsetAsync(o->grads.p, 0, sizeof(int32_t) * 18 * n, s);
  cudaMemsetAsync(o->am.p, 0, sizeof(float) * 18 * n, s);
  cudaMemsetAsync(o->av.p, 0, sizeof(float) * 18 * n, s);
  cudaMemsetAsync(o->gacc.p, 0, sizeof(float) * n, s);
  cudaMemsetAsync(o->lacc.p, 0, sizeof(float) * n, s);
  cudaMemsetAsync(o->pixel_loss.p, 0, sizeof(int32_t) * bz::kPixelLossSize, s);
  cudaMemsetAsync(o->stat.p, 0, 64, s);
  NPS_CUDA(cudaGetLastError());
  *out = o;
  return NPS_OK;
}

int nps_bezier_opt_destroy(nps_bezier_opt* o) {
  if (!o) return NPS_OK;
  cudaSetDevice(o->ctx->device);
  cudaStreamSynchronize(o->ctx->stream);
  for (DevBuf* b : {&o->params, &o->grads, &o->am, &o->av, &o->gacc, &o->lacc, &o->pixel_loss, &o->dead, &o->stat,
                    &o->views, &o->own[0], &o->own[1], &o->own[2], &o->own[3], &o->own[4], &o->fwd, &o->bwd, &o->ckbuf,
                    &o->counts, &o->offsets, &o->rects, &o->total, &o->keys, &o->vals, &o->ranges, &o->tabs,
                    &o->sw.hist, &o->sw.partial, &o->sw.lookback, &o->sw.keys_alt, &o->sw.vals_alt, &o->r_rec, &o->r_counts,
                    &o->r_offsets, &o->r_rects, &o->r_total, &o->r_cam, &o->r_keys, &o->r_vals, &o->r_ranges,
                    &o->r_tabs, &o->r_sw.hist, &o->r_sw.partial, &o->r_sw.lookback, &o->r_sw.keys_alt,
                    &o->r_sw.vals_alt})
    b->release();
  delete o;
  return NPS_OK;
}

int nps_bezier_opt_write_params(nps_bezier_opt* o, const float* bz, uint32_t first, uint32_t count, int mem) {
  NPS_TRY(check_bz(o));
  if ((uint64_t)first + count > o->n) {
    set_error("bezier write_params: range beyond %u curves", o->n);
    return NPS_ERR_INVALID;
  }
  return copy_in_bz(o->params.as<float>() + 20 * (size_t)first, bz, sizeof(float) * 20 * (size_t)count, mem,
                    o->ctx->stream);
}

int nps_bezier_opt_write_state(nps_bezier_opt* o, const int32_t* grads, const float* m, const float* v, float t,
                               const float* grad_accum, const float* loss_accum, const int32_t* pixel_loss, int mem) {
  NPS_TRY(check_bz(o));
  cudaStream_t s = o->ctx->stream;
  const size_t n = o->n;
  if (grads) NPS_TRY(copy_in_bz(o->grads.p, grads, sizeof(int32_t) * 18 * n, mem, s));
  if (m) NPS_TRY(copy_in_bz(o->am.p, m, sizeof(float) * 18 * n, mem, s));
  if (v) NPS_TRY(copy_in_bz(o->av.p, v, sizeof(float) * 18 * n, mem, s));
  if (grad_accum) NPS_TRY(copy_in_bz(o->gacc.p, grad_accum, sizeof(float) * n, mem, s));
  if (loss_accum) NPS_TRY(copy_in_bz(o->lacc.p, loss_accum, sizeof(float) * n, mem, s));
  if (pixel_loss) NPS_TRY(copy_in_bz(o->pixel_loss.p, pixel_loss, sizeof(int32_t) * bz::kPixelLossSize, mem, s));
  o->adam_t = t;
  return NPS_OK;
}

int nps_bezier_opt_read_state(nps_bezier_opt* o, float* bzp, int32_t* grads, float* m, float* v, float* t,
                              float* grad_accum, float* loss_accum, int32_t* pixel_loss) {
  NPS_TRY(check_bz(o));
  cudaStream_t s = o->ctx->stream;
  const size_t n = o->n;
  if (bzp) NPS_CUDA(cudaMemcpyAsync(bzp, o->params.p, sizeof(float) * 20 * n, cudaMemcpyDeviceToHost, s));
  if (grads) NPS_CUDA(cudaMemcpyAsync(grads, o->grads.p, sizeof(int32_t) * 18 * n, cudaMemcpyDeviceToHost, s));
  if (m) NPS_CUDA(cudaMemcpyAsync(m, o->am.p, sizeof(float) * 18 * n, cudaMemcpyDeviceToHost, s));
  if (v) NPS_CUDA(cudaMemcpyAsync(v, o->av.p, sizeof(float) * 18 * n, cudaMemcpyDeviceToHost, s));
  if (grad_accum) NPS_CUDA(cudaMemcpyAsync(grad_accum, o->gacc.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
  if (loss_accum) NPS_CUDA(cudaMemcpyAsync(loss_accum, o->lacc.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
  if (pixel_loss)
    NPS_CUDA(cudaMemcpyAsync(pixel_loss, o->pixel_loss.p, sizeof(int32_t) * bz::kPixelLossSize, cudaMemcpyDeviceToHost,
                             s));
  NPS_CUDA(cudaStreamSynchronize(s));
  if (t) *t = o->adam_t;
  return NPS_OK;
}

int nps_bezier_opt_write_vp(nps_bezier_opt* o, const float* vp, const float* vp_inv, uint32_t nv) {
  NPS_TRY(check_bz(o));
  if (!vp || !vp_inv || nv == 0 || nv > 4096) {
    set_error("bezier write_vp: bad arguments");
    return NPS_ERR_INVALID;
  }
  o->views_host.assign(32 * (size_t)nv, 0.0f);
  for (uint32_t v = 0; v < nv; ++v) {
    std::memcpy(&o->views_host[32 * v], vp + 16 * v, 64);
    std::memcpy(&o->views_host[32 * v + 16], vp_inv + 16 * v, 64);
  }
  NPS_TRY(o->views.ensure(sizeof(float) * o->views_host.size()));
  o->nv = nv;
  return copy_in_bz(o->views.p, o->views_host.data(), sizeof(float) * o->views_host.size(), NPS_MEM_HOST,
                    o->ctx->stream);
}

int nps_bezier_opt_write_mode(nps_bezier_opt* o, float mode) {
  NPS_TRY(check_bz(o));
  o->uni.mode = mode;
  return NPS_OK;
}
int nps_bezier_opt_write_bg_penalty(nps_bezier_opt* o, float w) {
  NPS_TRY(check_bz(o));
  o->uni.bg_penalty = w;
  return NPS_OK;
}
int nps_bezier_opt_write_max_width(nps_bezier_opt* o, float w) {
  NPS_TRY(check_bz(o));
  o->uni.max_width = w;
  return NPS_OK;
}
int nps_bezier_opt_write_kill_thresholds(nps_bezier_opt* o, float alpha, float width) {
  NPS_TRY(check_bz(o));
  o->uni.prune_alpha = alpha;
  o->uni.prune_width = width;
  return NPS_OK;
}
int nps_bezier_opt_set_adc_period(nps_bezier_opt* o, uint32_t period) {
  NPS_TRY(check_bz(o));
  if (period == 0) {
    set_error("bezier set_adc_period: period must be > 0");
    return NPS_ERR_INVALID;
  }
  o->adc_period = period;
  return NPS_OK;
}
int nps_bezier_opt_write_no_kill(nps_bezier_opt* o, int no_kill) {
  NPS_TRY(check_bz(o));
  o->no_kill = no_kill ? 1.0f : 0.0f;
  return NPS_OK;
}

int nps_bezier_opt_set_target(nps_bezier_opt* o, const float* target_rgba, const float* target_depth,
                              const float* bg_rgba, const float* bg_depth, const float* normal_rgba, uint32_t w,
                              uint32_t h, uint32_t nv, int mem) {
  NPS_TRY(check_bz(o));
  const float* src[5] = {target_rgba, target_depth, bg_rgba, bg_depth, normal_rgba};
  for (int k = 0; k < 5; ++k)
    if (!src[k]) {
      set_error("bezier set_target: null texture %d", k);
      return NPS_ERR_INVALID;
    }
  if (w == 0 || h == 0 || nv == 0 || w > 16 * 65535 || h > 16 * 65535) {
    set_error("bezier set_target: bad size");
    return NPS_ERR_INVALID;
  }
  const size_t px = (size_t)w * h * nv;
  const size_t bytes[5] = {16 * px, 4 * px, 16 * px, 4 * px, 16 * px};
  for (int k = 0; k < 5; ++k) {
    if (mem == NPS_MEM_DEVICE_BORROW) {
      if (((uintptr_t)src[k] & 15) != 0) {
        set_error("bezier set_target: borrowed textures must be 16-byte aligned");
        return NPS_ERR_INVALID;
      }
      o->tex[k] = src[k];
    } else {
      NPS_TRY(o->own[k].ensure(bytes[k]));
      NPS_TRY(copy_in_bz(o->own[k].p, src[k], bytes[k], mem, o->ctx->stream));
      o->tex[k] = o->own[k].as<float>();
    }
  }
  o->w = w;
  o->h = h;
  o->tv = nv;
  const uint32_t tx = div_up(w, 16), ty = div_up(h, 16);
  NPS_TRY(o->tabs.ensure(sizeof(float) * 2 * (tx + ty)));
  bin::k_tile_tables<<<1, 256, 0, o->ctx->stream>>>(o->tabs.as<float>(), tx, ty, w, h);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int nps_bezier_opt_backward(nps_bezier_opt* o, float* out_rgbd) {
  NPS_TRY(check_bz(o));
  if (!o->tex[0] || o->nv == 0) {
    set_error("bezier backward: set_target and write_vp first");
    return NPS_ERR_STATE;
  }
  if (o->tv != o->nv) {
    set_error("bezier backward: %u target views but %u cameras", o->tv, o->nv);
    return NPS_ERR_STATE;
  }
  cudaStream_t s = o->ctx->stream;
  const uint32_t n = o->n, nv = o->nv;
  const uint32_t tiles_x = div_up(o->w, 16), tiles_y = div_up(o->h, 16), num_tiles = tiles_x * tiles_y;
  const size_t g = (size_t)n * nv;
  if (g >= (1ull << 31) || (uint64_t)num_tiles * nv >= (1ull << 31)) {
    set_error("bezier backward: problem too large");
    return NPS_ERR_INVALID;
  }
  NPS_TRY(o->fwd.ensure(sizeof(float) * bz::kRecF * g));
  NPS_TRY(o->bwd.ensure(sizeof(float) * bz::kRecB * g));
  NPS_TRY(o->counts.ensure(sizeof(uint32_t) * g));
  NPS_TRY(o->offsets.ensure(sizeof(uint32_t) * g));
  NPS_TRY(o->rects.ensure(sizeof(uint2) * g));
  NPS_TRY(o->ranges.ensure(sizeof(uint32_t) * 2 * (size_t)num_tiles * nv));
  bz::k_bz_project<<<div_up(g, 256), 256, 0, s>>>(o->params.as<float>(), n, o->views.as<float>(), nv, o->w, o->h,
                                                   o->tabs.as<float>(), tiles_x, tiles_y, o->fwd.as<float>(),
                                                   o->bwd.as<float>(), o->counts.as<uint32_t>(), o->rects.as<uint2>());
  NPS_CHECK_LAUNCH();
  uint32_t* total = o->total.as<uint32_t>();
  NPS_TRY(exclusive_scan_u32(o->counts.as<uint32_t>(), o->offsets.as<uint32_t>(), (uint32_t)g, total, o->sw, s));
  uint32_t K = 0;
  NPS_CUDA(cudaMemcpyAsync(&K, total, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  if (K > o->pair_cap || o->pair_cap == 0) {
    const uint32_t cap = K + K / 4 + 4096;
    NPS_TRY(o->keys.ensure(sizeof(uint32_t) * (size_t)cap));
    NPS_TRY(o->vals.ensure(sizeof(uint32_t) * (size_t)cap));
    o->pair_cap = cap;
  }
  NPS_CUDA(cudaMemsetAsync(o->ranges.p, 0, sizeof(uint32_t) * 2 * (size_t)num_tiles * nv, s));
  uint32_t* rstart = o->ranges.as<uint32_t>();
  uint32_t* rend = rstart + (size_t)num_tiles * nv;
  const uint32_t* vs = o->vals.as<uint32_t>();
  if (K > 0) {
    bin::k_emit<<<div_up(g, 256), 256, 0, s>>>(o->counts.as<uint32_t>(), o->offsets.as<uint32_t>(),
                                                o->rects.as<uint2>(), n, nv, tiles_x, num_tiles, o->pair_cap,
                                                o->keys.as<uint32_t>(), o->vals.as<uint32_t>());
    NPS_CHECK_LAUNCH();
    int bits = 1;
    while ((1ull << bits) < (uint64_t)num_tiles * nv) ++bits;
    uint32_t *ks = nullptr, *vv = nullptr;
    NPS_TRY(radix_sort_u32(o->keys.as<uint32_t>(), o->vals.as<uint32_t>(), total, o->pair_cap, bits, o->sw, s, &ks,
                           &vv));
    bin::k_ranges<<<4 * kNumSMs, 256, 0, s>>>(ks, total, o->pair_cap, rstart, rend);
    NPS_CHECK_LAUNCH();
    vs = vv;
  }
  bz::RasterArgs ra;
  ra.fwd = o->fwd.as<float>();
  ra.bwd = o->bwd.as<float>();
  ra.vals = vs;
  ra.rstart = rstart;
  ra.rend = rend;
  ra.tgt_rgba = o->tex[0];
  ra.tgt_depth = o->tex[1];
  ra.bg_rgba = o->tex[2];
  ra.bg_depth = o->tex[3];
  ra.normal_rgba = o->tex[4];
  ra.grads = o->grads.as<int32_t>();
  ra.loss_accum = o->lacc.as<float>();
  ra.pixel_loss = o->pixel_loss.as<int32_t>();
  ra.out_rgbd = out_rgbd;
  ra.n = n;
  ra.w = o->w;
  ra.h = o->h;
  ra.tiles_x = tiles_x;
  ra.num_tiles = num_tiles;
  ra.u = o->uni;
  NPS_TRY(o->ckbuf.ensure(sizeof(float) * (size_t)tiles_x * tiles_y * nv * bz::kMaxChunks * bz::kThreads));
  ra.ckpt = o->ckbuf.as<float>();
  NPS_CUDA(cudaFuncSetAttribute(bz::k_bz_raster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bz::kRasterSmem));
  bz::k_bz_raster<<<dim3(tiles_x, tiles_y, nv), bz::kThreads, bz::kRasterSmem, s>>>(ra);
  NPS_CHECK_LAUNCH();
  o->stats.pairs = K;
  return NPS_OK;
}

int nps_bezier_opt_step(nps_bezier_opt* o) {
  NPS_TRY(check_bz(o));
  if (o->nv == 0) {
    set_error("bezier step: write_vp first (the offscreen kill uses the camera)");
    return NPS_ERR_STATE;
  }
  const float t = o->adam_t + 1.0f;
  bz::StepArgs a;
  a.bc1 = 1.0f - std::pow(0.9f, t);
  a.bc2 = 1.0f - std::pow(0.999f, t);
  const float pixel_count = (float)o->w * (float)o->h;  // GpuBezierOptimizerManager.ts:375-380
  a.pixel_norm = 1.0f / std::fmax(pixel_count, 1.0f);
  a.no_kill = o->no_kill;
  a.width_hi = o->uni.max_width > 0.0f ? o->uni.max_width : 0.1f;
  a.alpha_thresh = o->uni.prune_alpha > 0.0f ? o->uni.prune_alpha : 0.001f;
  a.width_thresh = o->uni.prune_width > 0.0f ? o->uni.prune_width : 0.001f;
  std::memcpy(a.vp, o->views_host.data(), 64);  // the uniform VP: the first camera
  bz::k_bz_step<<<div_up(o->n, 128), 128, 0, o->ctx->stream>>>(o->params.as<float>(), o->grads.as<int32_t>(),
                                                                o->am.as<float>(), o->av.as<float>(),
                                                                o->gacc.as<float>(), o->n, a);
  NPS_CHECK_LAUNCH();
  o->adam_t = t;
  return NPS_OK;
}

int nps_bezier_opt_adc(nps_bezier_opt* o) {
  NPS_TRY(check_bz(o));
  if (o->nv == 0) {
    set_error("bezier adc: write_vp first");
    return NPS_ERR_STATE;
  }
  bz::AdcArgs a;
  a.adam_t = o->adam_t;
  a.no_kill = o->no_kill;
  std::memcpy(a.vp, o->views_host.data(), 64);
  std::memcpy(a.vp_inv, o->views_host.data() + 16, 64);
  a.n = o->n;
  bz::k_bz_adc<<<1, bz::kAdcThreads, 0, o->ctx->stream>>>(o->params.as<float>(), o->am.as<float>(), o->av.as<float>(),
                                                          o->gacc.as<float>(), o->lacc.as<float>(),
                                                          o->pixel_loss.as<int32_t>(), o->dead.as<uint32_t>(),
                                                          o->stat.as<uint32_t>(), a);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int nps_bezier_opt_dispatch(nps_bezier_opt* o) {
  NPS_TRY(nps_bezier_opt_backward(o, nullptr));
  NPS_TRY(nps_bezier_opt_step(o));
  o->step_count++;
  if (o->step_count % o->adc_period == 0) NPS_TRY(nps_bezier_opt_adc(o));  // GpuBezierOptimizerManager.ts:398-404
  return NPS_OK;
}

int nps_bezier_opt_render(nps_bezier_opt* o, const float* vp, uint32_t w, uint32_t h, const float* bg_rgba,
                          const float* brush, uint32_t brush_w, uint32_t brush_h, float* out_rgba) {
  NPS_TRY(check_bz(o));
  if (!vp || !out_rgba || w == 0 || h == 0 || w > 16 * 65535 || h > 16 * 65535 || (brush && (!brush_w || !brush_h))) {
    set_error("bezier render: bad arguments");
    return NPS_ERR_INVALID;
  }
  cudaStream_t s = o->ctx->stream;
  const uint32_t n = o->n, tiles_x = div_up(w, 16), tiles_y = div_up(h, 16), num_tiles = tiles_x * tiles_y;
  NPS_TRY(o->r_rec.ensure(sizeof(float) * bz::kBRend * n));
  NPS_TRY(o->r_counts.ensure(sizeof(uint32_t) * n));
  NPS_TRY(o->r_offsets.ensure(sizeof(uint32_t) * n));
  NPS_TRY(o->r_rects.ensure(sizeof(uint2) * n));
  NPS_TRY(o->r_total.ensure(16));
  NPS_TRY(o->r_cam.ensure(64));
  NPS_TRY(o->r_ranges.ensure(sizeof(uint32_t) * 2 * num_tiles));
  NPS_TRY(o->r_tabs.ensure(sizeof(float) * 2 * (tiles_x + tiles_y)));
  NPS_TRY(copy_in_bz(o->r_cam.p, vp, 64, NPS_MEM_HOST, s));
  bin::k_tile_tables<<<1, 256, 0, s>>>(o->r_tabs.as<float>(), tiles_x, tiles_y, w, h);
  bz::k_bz_render_project<<<div_up(n, 256), 256, 0, s>>>(o->params.as<float>(), n, o->r_cam.as<float>(), w, h,
                                                          o->r_tabs.as<float>(), tiles_x, tiles_y,
                                                          o->r_rec.as<float>(), o->r_counts.as<uint32_t>(),
                                                          o->r_rects.as<uint2>());
  NPS_CHECK_LAUNCH();
  uint32_t* total = o->r_total.as<uint32_t>();
  NPS_TRY(exclusive_scan_u32(o->r_counts.as<uint32_t>(), o->r_offsets.as<uint32_t>(), n, total, o->r_sw, s));
  uint32_t K = 0;
  NPS_CUDA(cudaMemcpyAsync(&K, total, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  if (K > o->r_pair_cap || o->r_pair_cap == 0) {
    const uint32_t cap = K + K / 4 + 4096;
    NPS_TRY(o->r_keys.ensure(sizeof(uint32_t) * (size_t)cap));
    NPS_TRY(o->r_vals.ensure(sizeof(uint32_t) * (size_t)cap));
    o->r_pair_cap = cap;
  }
  uint32_t* rstart = o->r_ranges.as<uint32_t>();
  uint32_t* rend = rstart + num_tiles;
  NPS_CUDA(cudaMemsetAsync(rstart, 0, sizeof(uint32_t) * 2 * num_tiles, s));
  const uint32_t* vs = o->r_vals.as<uint32_t>();
  if (K > 0) {
    bin::k_emit<<<div_up(n, 256), 256, 0, s>>>(o->r_counts.as<uint32_t>(), o->r_offsets.as<uint32_t>(),
                                                o->r_rects.as<uint2>(), n, 1, tiles_x, num_tiles, o->r_pair_cap,
                                                o->r_keys.as<uint32_t>(), o->r_vals.as<uint32_t>());
    NPS_CHECK_LAUNCH();
    int bits = 1;
    while ((1ull << bits) < (uint64_t)num_tiles) ++bits;
    uint32_t *ks = nullptr, *vv = nullptr;
    NPS_TRY(radix_sort_u32(o->r_keys.as<uint32_t>(), o->r_vals.as<uint32_t>(), total, o->r_pair_cap, bits, o->r_sw, s,
                           &ks, &vv));
    bin::k_ranges<<<4 * kNumSMs, 256, 0, s>>>(ks, total, o->r_pair_cap, rstart, rend);
    NPS_CHECK_LAUNCH();
    vs = vv;
  }
  bz::k_bz_render_raster<<<dim3(tiles_x, tiles_y), 256, 0, s>>>(o->r_rec.as<float>(), vs, rstart, rend, w, h, tiles_x,
                                                                 (const float4*)bg_rgba, brush, brush_w, brush_h,
                                                                 (float4*)out_rgba);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int nps_bezier_opt_buffers(nps_bezier_opt* o, float** bzp, int32_t** grads, float** m, float** v, float** gacc,
                           float** lacc, int32_t** pixel_loss) {
  NPS_TRY(check_bz(o));
  if (bzp) *bzp = o->params.as<float>();
  if (grads) *grads = o->grads.as<int32_t>();
  if (m) *m = o->am.as<float>();
  if (v) *v = o->av.as<float>();
  if (gacc) *gacc = o->gacc.as<float>();
  if (lacc) *lacc = o->lacc.as<float>();
  if (pixel_loss) *pixel_loss = o->pixel_loss.as<int32_t>();
  return NPS_OK;
}

// the manager's stepCount (GpuBezierOptimizerManager.ts:398): dispatch() calls so far, which decide
// when ADC runs; restoring a checkpoint sets it back
int nps_bezier_opt_set_step_count(nps_bezier_opt* o, uint32_t count) {
  NPS_TRY(check_bz(o));
  o->step_count = count;
  return NPS_OK;
}

int nps_bezier_opt_stats(nps_bezier_opt* o, nps_stats* out) {
  NPS_TRY(check_bz(o));
  if (!out) return NPS_ERR_INVALID;
  uint32_t st[2] = {0, 0};
  NPS_CUDA(cudaMemcpyAsync(st, o->stat.p, sizeof(st), cudaMemcpyDeviceToHost, o->ctx->stream));
  NPS_CUDA(cudaStreamSynchronize(o->ctx->stream));
  o->stats.adc_clones = st[0];
  o->stats.reserved[0] = st[1];
  o->stats.step_count = o->step_count;
  *out = o->stats;
  return NPS_OK;
}

}  // extern "C"
