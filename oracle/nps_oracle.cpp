// nps_oracle.cpp — CPU oracle for the nprush hot path.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file;
// it is loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU
// baseline leg, always as the checker, never as the thing measured or shipped.
//
// Part 1 ("compat") restates the reference's WGSL compute shaders in plain C++:
//   splat_backward.wgsl:34-457   binning (index order, 1024 cap), fp32
//                                front-to-back composite, L2 + depth loss,
//                                reference backward with i32 fixed-point sums
//   splat_step.wgsl:32-106       Adam + clamps + prune + grad_accum
//   splat_adc.wgsl:28-87         serial clone / split into dead slots
//   bezier_backward.wgsl:56-572  Bezier binning, 16-segment walk, composite,
//                                luma/contrast loss, backward, loss maps
//   bezier_step.wgsl:50-189      Adam + clamps + prune + offscreen kill
//   bezier_adc.wgsl:52-315       kill / split / clone / spawn passes
// The per-operation float order matches the shaders so that, compiled with
// -ffp-contract=off, results are bit-identical to the reference's own shader
// code run on the host (oracle/_ref, built by oracle/build_ref.py).  That
// comparison is what pins this restatement (tests/test_oracle_pin.py).
//
// Part 2 ("gs") is the 3D Gaussian training model, which has no reference counterpart:
// standard 3D Gaussians (log-scales, logit opacity, SH up to degree 3), depth
// ordered compositing and L1 / L2 / D-SSIM losses, templated on the scalar so
// the double instantiation is the FP64 central-difference oracle.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ----------------------------------------------------------------- helpers
struct V2 { float x, y; };
struct V3 { float x, y, z; };
struct V4 { float x, y, z, w; };

inline V3 cross3(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
// column-major 4x4 times (x,y,z,w): sum over columns left to right (matches WGSL M*v)
inline V4 mulv(const float* m, float x, float y, float z, float w) {
  V4 o;
  o.x = m[0] * x + m[4] * y + m[8] * z + m[12] * w;
  o.y = m[1] * x + m[5] * y + m[9] * z + m[13] * w;
  o.z = m[2] * x + m[6] * y + m[10] * z + m[14] * w;
  o.w = m[3] * x + m[7] * y + m[11] * z + m[15] * w;
  return o;
}
inline float clampf(float e, float lo, float hi) { return std::fmin(std::fmax(e, lo), hi); }
inline float smoothstepf(float lo, float hi, float x) {
  float t = clampf((x - lo) / (hi - lo), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
// WGSL i32(f32): truncate toward zero, saturate
inline int32_t to_i32(float a) {
  if (std::isnan(a)) return 0;
  if (a >= 2147483520.0f) return 2147483520;
  if (a <= -2147483648.0f) return INT32_MIN;
  return (int32_t)a;
}
inline int32_t wrap_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
inline float fractf(float a) { return a - std::floor(a); }

// splat_backward.wgsl:34-40 pixel_to_p
inline V2 pixel_to_p(uint32_t px, uint32_t py, uint32_t w, uint32_t h, float aspect) {
  float ux = ((float)px + 0.5f) / (float)w;
  float uy = ((float)py + 0.5f) / (float)h;
  V2 p{ux * 2.0f - 1.0f, uy * 2.0f - 1.0f};
  p.y = -p.y;
  p.x = p.x * aspect;
  return p;
}
// splat_backward.wgsl:42-45 quat_rotate(q, v), q = (w, x, y, z)
inline V3 quat_rotate(V4 q, V3 v) {
  V3 u{q.y, q.z, q.w};
  V3 c = cross3(u, v);
  V3 t{2.0f * c.x, 2.0f * c.y, 2.0f * c.z};
  V3 c2 = cross3(u, t);
  return {v.x + q.x * t.x + c2.x, v.y + q.x * t.y + c2.y, v.z + q.x * t.z + c2.z};
}
// splat_backward.wgsl:52-58 project_axis
inline V2 project_axis(const float* vp, V3 ax, float cx, float cy, float w, float aspect) {
  V4 ac = mulv(vp, ax.x, ax.y, ax.z, 0.0f);
  return {(ac.x * w - cx * ac.w) / (w * w) * aspect, (ac.y * w - cy * ac.w) / (w * w)};
}

// ===================================================================== splats
constexpr uint32_t SPLAT_MAX_TILE = 1024;     // constants.ts:35
constexpr float SPLAT_FP_SCALE_POS = 10000.0f; // constants.ts:36
constexpr float SPLAT_FP_SCALE_COL = 100000.0f;// constants.ts:37
constexpr float SPLAT_OPACITY_KILL = 0.05f;    // constants.ts:32
constexpr float SPLAT_VOLUME_KILL = 1e-7f;     // constants.ts:34
constexpr float SPLAT_GRAD_THRESH = 0.00005f;  // constants.ts:31
constexpr float SPLAT_ADC_PERIOD = 25.0f;      // constants.ts:30
constexpr float ADAM_B1 = 0.9f, ADAM_B2 = 0.999f, ADAM_EPS = 1e-8f;  // constants.ts:7-9

// Pixel-independent part of eval_splat (splat_backward.wgsl:92-126) for one
// splat and one view.  Identical arithmetic, evaluated once instead of per pixel.
struct SplatProj {
  float sx, sy, sz;
  float clip_x, clip_y, w;
  float screen_x, screen_y;
  V2 ax, ay, az;
  float m0x, m0y, m1x, m1y, m2x, m2y;
  float A, B, C;
};
inline SplatProj splat_project(const float* s, const float* vp, float aspect, uint32_t h) {
  SplatProj P;
  V4 clip = mulv(vp, s[0], s[1], s[2], 1.0f);
  P.w = clip.w;
  P.clip_x = clip.x;
  P.clip_y = clip.y;
  P.screen_x = clip.x / clip.w * aspect;
  P.screen_y = clip.y / clip.w;
  V4 q{s[8], s[9], s[10], s[11]};
  P.sx = std::fmax(s[3], 0.0001f);
  P.sy = std::fmax(s[12], 0.0001f);
  P.sz = std::fmax(s[15], 0.0001f);
  V3 axw = quat_rotate(q, {1.0f, 0.0f, 0.0f});
  V3 ayw = quat_rotate(q, {0.0f, 1.0f, 0.0f});
  V3 azw = quat_rotate(q, {0.0f, 0.0f, 1.0f});
  P.ax = project_axis(vp, axw, P.clip_x, P.clip_y, P.w, aspect);
  P.ay = project_axis(vp, ayw, P.clip_x, P.clip_y, P.w, aspect);
  P.az = project_axis(vp, azw, P.clip_x, P.clip_y, P.w, aspect);
  P.m0x = P.ax.x * P.sx; P.m0y = P.ax.y * P.sx;
  P.m1x = P.ay.x * P.sy; P.m1y = P.ay.y * P.sy;
  P.m2x = P.az.x * P.sz; P.m2y = P.az.y * P.sz;
  float cov00 = P.m0x * P.m0x + P.m1x * P.m1x + P.m2x * P.m2x;
  float cov01 = P.m0x * P.m0y + P.m1x * P.m1y + P.m2x * P.m2y;
  float cov11 = P.m0y * P.m0y + P.m1y * P.m1y + P.m2y * P.m2y;
  float filter_std = 0.3f * (2.0f / (float)h);
  float filter2 = filter_std * filter_std;
  cov00 += filter2;
  cov11 += filter2;
  float det = cov00 * cov11 - cov01 * cov01;
  float inv_det = std::fabs(det) < 1e-10f ? 0.0f : 1.0f / det;
  P.A = cov11 * inv_det;
  P.B = -cov01 * inv_det;
  P.C = cov00 * inv_det;
  return P;
}

// Binning predicate, splat_backward.wgsl:155-195.  Returns false if culled,
// otherwise the screen-space AABB [smin, smax].
inline bool splat_aabb(const float* s, const float* vp, float aspect, uint32_t h, float* smin, float* smax) {
  if (s[7] < 0.005f) return false;
  V4 c0 = mulv(vp, s[0], s[1], s[2], 1.0f);
  float pz = c0.w;
  float px = c0.x / c0.w * aspect, py = c0.y / c0.w;
  if (pz < 0.0f) return false;
  float sx = std::fmax(s[3], 0.0001f), sy = std::fmax(s[12], 0.0001f), sz = std::fmax(s[15], 0.0001f);
  float safe_sb = std::fmax(s[14], 0.0001f);
  float R = std::pow(15.0f / safe_sb, 1.0f / s[13]);
  V4 q{s[8], s[9], s[10], s[11]};
  V3 axw = quat_rotate(q, {1.0f, 0.0f, 0.0f});
  V3 ayw = quat_rotate(q, {0.0f, 1.0f, 0.0f});
  V3 azw = quat_rotate(q, {0.0f, 0.0f, 1.0f});
  V4 clip = mulv(vp, s[0], s[1], s[2], 1.0f);
  V2 ax = project_axis(vp, axw, clip.x, clip.y, clip.w, aspect);
  V2 ay = project_axis(vp, ayw, clip.x, clip.y, clip.w, aspect);
  V2 az = project_axis(vp, azw, clip.x, clip.y, clip.w, aspect);
  float m0x = ax.x * sx, m0y = ax.y * sx, m1x = ay.x * sy, m1y = ay.y * sy, m2x = az.x * sz, m2y = az.y * sz;
  float cov00 = m0x * m0x + m1x * m1x + m2x * m2x;
  float cov11 = m0y * m0y + m1y * m1y + m2y * m2y;
  float filter_std = 0.3f * (2.0f / (float)h);
  float filter2 = filter_std * filter_std;
  cov00 += filter2;
  cov11 += filter2;
  float max_r = R * std::sqrt(std::fmax(std::fmax(cov00, cov11), 1e-9f));
  smin[0] = px - max_r; smin[1] = py - max_r;
  smax[0] = px + max_r; smax[1] = py + max_r;
  return true;
}

// Tile rectangle in aspect-corrected screen space, splat_backward.wgsl:148-153.
inline void tile_rect(uint32_t tx, uint32_t ty, uint32_t w, uint32_t h, float aspect, float* tmin, float* tmax) {
  uint32_t x0 = tx * 16u, y0 = ty * 16u;
  uint32_t x1 = std::min(x0 + 16u, w), y1 = std::min(y0 + 16u, h);
  V2 p00 = pixel_to_p(x0, y0, w, h, aspect);
  V2 p11 = pixel_to_p(x1, y1, w, h, aspect);
  tmin[0] = p00.x; tmin[1] = p11.y;
  tmax[0] = p11.x; tmax[1] = p00.y;
}

// Per-pixel quantities of eval_splat that depend on p (splat_backward.wgsl:98,127-132).
struct PixEval { float dx, dy, spx, spy, r; };
inline PixEval splat_pix(const SplatProj& P, V2 p) {
  PixEval e;
  e.dx = p.x - P.screen_x;
  e.dy = p.y - P.screen_y;
  e.spx = P.A * e.dx + P.B * e.dy;
  e.spy = P.B * e.dx + P.C * e.dy;
  float r2 = e.dx * e.spx + e.dy * e.spy;
  e.r = std::sqrt(std::fmax(r2, 0.0001f));
  return e;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// Splat forward + loss + backward for one view: splat_backward.wgsl:136-457.
//   splats      N x 16 floats, the reference's AoS record (pos_sx, color, quat, sy_shape)
//   vp, vpinv   column-major 4x4 (mat4x4f as uploaded by writeSplatVPMatrix)
//   tgt_rgba    H x W x 4 target colour (targetTex), tgt_depth H x W (targetDepthTex.r)
//   grads_q     N x 16 i32, ADDED to (the reference's atomicAdd of i32(g*scale))
//   grads_f     N x 16 f32 unquantised sums (may be null)
//   out_rgbd    H x W x 4: composited colour + reciprocal depth (may be null)
//   tile_count  tiles_y x tiles_x list lengths after the cap (may be null)
//   terms       N: ADDED the number of (pixel, splat) backward terms with
//               alpha >= 0.001 each splat's gradient sums (may be null; the
//               bound for the device's i32 sums, whose terms are truncated
//               one by one)
int orc_splat_backward(const float* splats, uint32_t n, const float* vp, const float* vpinv,
                       const float* tgt_rgba, const float* tgt_depth, uint32_t w, uint32_t h,
                       int32_t* grads_q, float* grads_f, float* out_rgbd, uint32_t* tile_count,
                       uint32_t* terms) {
  const float aspect = (float)w / (float)h;
  const uint32_t tiles_x = (w + 15) / 16, tiles_y = (h + 15) / 16;
  std::vector<SplatProj> proj(n);
  std::vector<uint8_t> live(n);
  std::vector<float> bb(4 * (size_t)n);
  for (uint32_t i = 0; i < n; ++i) {
    live[i] = splat_aabb(splats + 16 * (size_t)i, vp, aspect, h, &bb[4 * i], &bb[4 * i + 2]);
    proj[i] = splat_project(splats + 16 * (size_t)i, vp, aspect, h);
  }
  const float DEPTH_NEAR = 0.1f;
  std::vector<uint32_t> list;
  list.reserve(SPLAT_MAX_TILE);
  std::vector<float> alphas(SPLAT_MAX_TILE), Ts(SPLAT_MAX_TILE + 1);
  for (uint32_t ty = 0; ty < tiles_y; ++ty)
    for (uint32_t tx = 0; tx < tiles_x; ++tx) {
      float tmin[2], tmax[2];
      tile_rect(tx, ty, w, h, aspect, tmin, tmax);
      list.clear();
      for (uint32_t i = 0; i < n && list.size() < SPLAT_MAX_TILE; ++i) {
        if (!live[i]) continue;
        const float* b = &bb[4 * i];
        if (!(b[0] > tmax[0] || b[2] < tmin[0] || b[1] > tmax[1] || b[3] < tmin[1])) list.push_back(i);
      }
      if (tile_count) tile_count[ty * tiles_x + tx] = (uint32_t)list.size();
      const uint32_t cnt = (uint32_t)list.size();
      for (uint32_t py = ty * 16; py < std::min(ty * 16 + 16, h); ++py)
        for (uint32_t px = tx * 16; px < std::min(tx * 16 + 16, w); ++px) {
          V2 p = pixel_to_p(px, py, w, h, aspect);
          const float* tc = tgt_rgba + ((size_t)py * w + px) * 4;
          const float td = tgt_depth[(size_t)py * w + px];
          Ts[0] = 1.0f;
          float Cr = 0.0f, Cg = 0.0f, Cb = 0.0f, D = 0.0f;
          for (uint32_t k = 0; k < cnt; ++k) {
            const float* s = splats + 16 * (size_t)list[k];
            const SplatProj& P = proj[list[k]];
            PixEval e = splat_pix(P, p);
            float power = -s[14] * std::pow(e.r, s[13]);
            float a = clampf(power > -15.0f ? std::exp(power) * s[7] : 0.0f, 0.0f, 0.999f);
            alphas[k] = a;
            Cr += Ts[k] * a * s[4];
            Cg += Ts[k] * a * s[5];
            Cb += Ts[k] * a * s[6];
            float ld = std::fmax(P.w, DEPTH_NEAR);
            float depth = clampf(1.0f - DEPTH_NEAR / ld, 0.0f, 1.0f);
            D += Ts[k] * a * depth;
            Ts[k + 1] = Ts[k] * (1.0f - a);
          }
          const float bg = 0.05f;
          Cr += Ts[cnt] * bg; Cg += Ts[cnt] * bg; Cb += Ts[cnt] * bg;
          D += Ts[cnt] * 1.0f;
          if (out_rgbd) {
            float* o = out_rgbd + ((size_t)py * w + px) * 4;
            o[0] = Cr; o[1] = Cg; o[2] = Cb; o[3] = D;
          }
          // loss, splat_backward.wgsl:250-257
          float dCr = 2.0f * (Cr - tc[0]), dCg = 2.0f * (Cg - tc[1]), dCb = 2.0f * (Cb - tc[2]);
          bool fg = td < 0.99f;
          float dD = fg ? 2.0f * (D - td) : 0.0f;
          float dT_C = dCr * bg + dCg * bg + dCb * bg;
          float dT_D = dD * 1.0f;
          // reverse loop, splat_backward.wgsl:259-456
          for (uint32_t j = 0; j < cnt; ++j) {
            uint32_t idx = cnt - 1 - j;
            uint32_t i = list[idx];
            float a = alphas[idx];
            if (a < 0.001f) continue;
            if (terms) ++terms[i];
            const float* s = splats + 16 * (size_t)i;
            const SplatProj& P = proj[i];
            PixEval e = splat_pix(P, p);
            float cr = s[4], cg = s[5], cb = s[6], opacity = s[7];
            float T_prev = Ts[idx];
            float TA = T_prev * a;
            float dColr = dCr * TA, dColg = dCg * TA, dColb = dCb * TA;
            float ldb = std::fmax(P.w, DEPTH_NEAR);
            float depth = clampf(1.0f - DEPTH_NEAR / ldb, 0.0f, 1.0f);
            float tcr = T_prev * cr, tcg = T_prev * cg, tcb = T_prev * cb;
            float da_C = dT_C * (-T_prev) + (dCr * tcr + dCg * tcg + dCb * tcb);
            float da_D = dT_D * (-T_prev) + dD * T_prev * depth;
            float da = da_C + da_D;
            float acr = a * cr, acg = a * cg, acb = a * cb;
            dT_C = dT_C * (1.0f - a) + (dCr * acr + dCg * acg + dCb * acb);
            dT_D = dT_D * (1.0f - a) + dD * a * depth;
            float d_depth = dD * T_prev * a;
            float sx = P.sx, sy = P.sy, sz = P.sz;
            float shape_a = s[13], shape_b = s[14];
            float power = -shape_b * std::pow(e.r, shape_a);
            bool above = power > -15.0f;
            float a_un = above ? std::exp(power) : 0.0f;
            float d_opacity = above ? da * a_un : 0.0f;
            float d_power = above ? da * opacity * a_un : 0.0f;
            float r_pow_a = std::pow(e.r, shape_a);
            float r_pow_a_m2 = std::pow(e.r, shape_a - 2.0f);
            float d_shape_a = above ? d_power * (-shape_b * r_pow_a * std::log(e.r)) : 0.0f;
            float d_shape_b = above ? d_power * (-r_pow_a) : 0.0f;
            float kk = d_power * (-shape_b * shape_a * r_pow_a_m2);
            float ddx = above ? kk * e.spx : 0.0f, ddy = above ? kk * e.spy : 0.0f;
            float dsx_ = -ddx, dsy_ = -ddy;  // d_screen
            float sp0 = e.spx * P.m0x + e.spy * P.m0y;
            float sp1 = e.spx * P.m1x + e.spy * P.m1y;
            float sp2 = e.spx * P.m2x + e.spy * P.m2y;
            float dm0x = -sp0 * ddx, dm0y = -sp0 * ddy;
            float dm1x = -sp1 * ddx, dm1y = -sp1 * ddy;
            float dm2x = -sp2 * ddx, dm2y = -sp2 * ddy;
            V2 dax{dm0x * sx, dm0y * sx}, day{dm1x * sy, dm1y * sy}, daz{dm2x * sz, dm2y * sz};
            float d_sx = dm0x * P.ax.x + dm0y * P.ax.y;
            float d_sy = dm1x * P.ay.x + dm1y * P.ay.y;
            float d_sz = dm2x * P.az.x + dm2y * P.az.y;
            float ww = P.w, w2 = ww * ww;
            float d_pos[3];
            for (int ax = 0; ax < 3; ++ax) {
              float vp0 = vp[ax * 4 + 0], vp1 = vp[ax * 4 + 1], vp3 = vp[ax * 4 + 3];
              float ds_dx = aspect * (vp0 * ww - P.clip_x * vp3) / w2;
              float ds_dy = (vp1 * ww - P.clip_y * vp3) / w2;
              d_pos[ax] = dsx_ * ds_dx + dsy_ * ds_dy;
              float d_depth_d_w = DEPTH_NEAR / (ww * ww);
              d_pos[ax] += (P.w > DEPTH_NEAR) ? vp3 * d_depth_d_w * d_depth : 0.0f;
            }
            if (fg) {
              // reconstruct_world_pos, splat_backward.wgsl:64-75
              float wr = 0.1f / std::fmax(1.0f - td, 1e-5f);
              float ndx = p.x / aspect, ndy = p.y;
              V4 wp = mulv(vpinv, ndx * wr, ndy * wr, wr, wr);
              float surf[3] = {wp.x / wp.w, wp.y / wp.w, wp.z / wp.w};
              for (int ax = 0; ax < 3; ++ax) {
                float err = s[ax] - surf[ax];
                d_pos[ax] += 0.3f * 2.0f * err * (T_prev * a);
              }
            }
            float dax_w[3], day_w[3], daz_w[3];
            for (int ax = 0; ax < 3; ++ax) {
              float vp0 = vp[ax * 4 + 0], vp1 = vp[ax * 4 + 1], vp3 = vp[ax * 4 + 3];
              float j0 = aspect * (vp0 * ww - P.clip_x * vp3) / w2;
              float j1 = (vp1 * ww - P.clip_y * vp3) / w2;
              dax_w[ax] = dax.x * j0 + dax.y * j1;
              day_w[ax] = day.x * j0 + day.y * j1;
              daz_w[ax] = daz.x * j0 + daz.y * j1;
            }
            float qw = s[8], qx = s[9], qy = s[10], qz = s[11];
            // splat_backward.wgsl:410-426
            float d_qw = (dax_w[1] * 2.0f * qz - dax_w[2] * 2.0f * qy) + (-day_w[0] * 2.0f * qz + day_w[2] * 2.0f * qx) +
                         (daz_w[0] * 2.0f * qy - daz_w[1] * 2.0f * qx);
            float d_qx = (dax_w[1] * 2.0f * qy + dax_w[2] * 2.0f * qz) +
                         (day_w[0] * 2.0f * qy - day_w[1] * 4.0f * qx + day_w[2] * 2.0f * qw) +
                         (daz_w[0] * 2.0f * qz - daz_w[1] * 2.0f * qw - daz_w[2] * 4.0f * qx);
            float d_qy = (-dax_w[0] * 4.0f * qy + dax_w[1] * 2.0f * qx + dax_w[2] * (-2.0f * qw)) +
                         (day_w[0] * 2.0f * qx + day_w[2] * 2.0f * qz) +
                         (daz_w[0] * 2.0f * qw + daz_w[1] * 2.0f * qz - daz_w[2] * 4.0f * qy);
            float d_qz = (-dax_w[0] * 4.0f * qz + dax_w[1] * 2.0f * qw + dax_w[2] * 2.0f * qx) +
                         (-day_w[0] * 2.0f * qw - day_w[1] * 4.0f * qz + day_w[2] * 2.0f * qy) +
                         (daz_w[0] * 2.0f * qx + daz_w[1] * 2.0f * qy);
            d_shape_a += 0.005f * 2.0f * (shape_a - 6.0f);
            d_shape_b += 0.005f * 2.0f * (shape_b - 0.3f);
            const float g[16] = {d_pos[0], d_pos[1], d_pos[2], d_sx, dColr, dColg, dColb, d_opacity,
                                 d_qw, d_qx, d_qy, d_qz, d_sy, d_shape_a, d_shape_b, d_sz};
            int32_t* gq = grads_q + 16 * (size_t)i;
            for (int k = 0; k < 16; ++k) {
              float sc = (k >= 4 && k <= 7) ? SPLAT_FP_SCALE_COL : SPLAT_FP_SCALE_POS;
              gq[k] = wrap_add(gq[k], to_i32(g[k] * sc));
            }
            if (grads_f)
              for (int k = 0; k < 16; ++k) grads_f[16 * (size_t)i + k] += g[k];
          }
        }
    }
  return 0;
}

// Splat Adam step: splat_step.wgsl:32-106.  The step counter is passed by
// value: every splat uses t = *adam_t + 1 (the shader's intent; on the GPU its
// read/write of adam.t across workgroups is a race), then *adam_t is advanced.
int orc_splat_step(float* splats, int32_t* grads, float* m, float* v, float* adam_t, float* grad_accum,
                   uint32_t n) {
  static const float lr[16] = {0.0005f, 0.0005f, 0.0005f, 0.01f, 0.02f, 0.02f, 0.02f, 0.01f,
                               0.005f, 0.005f, 0.005f, 0.005f, 0.01f, 0.01f, 0.01f, 0.01f};
  static const float mu[16] = {0.005f, 0.005f, 0.005f, 0.005f, 0.001f, 0.001f, 0.001f, 0.0005f,
                               0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.05f, 0.05f, 0.005f};
  static const float lo[16] = {-1e9f, -1e9f, -1e9f, 0.001f, 0.05f, 0.05f, 0.05f, 0.01f,
                               -1e9f, -1e9f, -1e9f, -1e9f, 0.001f, 0.1f, 0.01f, 0.001f};
  static const float hi[16] = {1e9f, 1e9f, 1e9f, 2.0f, 1.0f, 1.0f, 1.0f, 0.99f,
                               1e9f, 1e9f, 1e9f, 1e9f, 2.0f, 10.0f, 5.0f, 2.0f};
  const float t = *adam_t + 1.0f;
  const float bc1 = 1.0f - std::pow(ADAM_B1, t), bc2 = 1.0f - std::pow(ADAM_B2, t);
  for (uint32_t i = 0; i < n; ++i) {
    float* s = splats + 16 * (size_t)i;
    float pos_g2 = 0.0f;
    for (int k = 0; k < 16; ++k) {
      size_t pi = 16 * (size_t)i + k;
      int32_t raw = grads[pi];
      grads[pi] = 0;
      float fps = (k >= 4 && k <= 7) ? SPLAT_FP_SCALE_COL : SPLAT_FP_SCALE_POS;
      float g = (float)raw / fps / 16384.0f;
      float mm = ADAM_B1 * m[pi] + (1.0f - ADAM_B1) * g;
      float vv = ADAM_B2 * v[pi] + (1.0f - ADAM_B2) * g * g;
      m[pi] = mm;
      v[pi] = vv;
      float m_hat = mm / bc1, v_hat = vv / bc2;
      float raw_u = lr[k] * m_hat / (std::sqrt(v_hat) + ADAM_EPS);
      float u = clampf(raw_u, -mu[k], mu[k]);
      s[k] = clampf(s[k] - u, lo[k], hi[k]);
      if (k <= 2) pos_g2 += g * g;
    }
    float ql = std::sqrt(s[8] * s[8] + s[9] * s[9] + s[10] * s[10] + s[11] * s[11]);
    ql = std::fmax(ql, 1e-8f);
    s[8] /= ql; s[9] /= ql; s[10] /= ql; s[11] /= ql;
    grad_accum[i] += std::sqrt(pos_g2);
    float vol = s[3] * s[12] * s[15];
    if (s[7] < SPLAT_OPACITY_KILL || vol < SPLAT_VOLUME_KILL) s[7] = 0.0f;
  }
  *adam_t = t;
  return 0;
}

// Splat ADC: splat_adc.wgsl:28-87 (serial reference semantics, including the
// re-visit of freshly filled slots that lie ahead of the cursor).
int orc_splat_adc(float* splats, float* m, float* v, float adam_t, float* grad_accum, uint32_t n) {
  uint32_t next_dead = 0;
  for (uint32_t i = 0; i < n; ++i) {
    float s[16];
    std::memcpy(s, splats + 16 * (size_t)i, sizeof(s));
    if (s[7] < SPLAT_OPACITY_KILL) continue;
    float ga = grad_accum[i] / SPLAT_ADC_PERIOD;
    grad_accum[i] = 0.0f;
    if (!(ga > SPLAT_GRAD_THRESH)) continue;
    float scale_norm = std::sqrt(s[3] * s[3] + s[12] * s[12] + s[15] * s[15]);
    bool found = false;
    uint32_t nidx = 0;
    for (uint32_t d = next_dead; d < n; ++d) {
      if (splats[16 * (size_t)d + 7] < SPLAT_OPACITY_KILL) { nidx = d; found = true; next_dead = d + 1; break; }
    }
    if (!found) next_dead = n;
    if (!found) continue;
    float ns[16];
    std::memcpy(ns, s, sizeof(s));
    if (scale_norm > 0.01f) {
      const float f = 0.625f;
      s[3] *= f; s[12] *= f; s[15] *= f;
      ns[3] *= f; ns[12] *= f; ns[15] *= f;
      s[0] -= s[3] * 0.05f;
      ns[0] += s[3] * 0.05f;
    } else {
      float seed = (float)i * 3.14159f + adam_t;
      ns[0] += (fractf(std::sin(seed * 12.9898f) * 43758.5453f) - 0.5f) * 0.002f;
      ns[1] += (fractf(std::sin(seed * 78.233f) * 43758.5453f) - 0.5f) * 0.002f;
    }
    std::memcpy(splats + 16 * (size_t)i, s, sizeof(s));
    std::memcpy(splats + 16 * (size_t)nidx, ns, sizeof(ns));
    for (int p = 0; p < 16; ++p) {
      m[16 * (size_t)i + p] = 0.0f; v[16 * (size_t)i + p] = 0.0f;
      m[16 * (size_t)nidx + p] = 0.0f; v[16 * (size_t)nidx + p] = 0.0f;
    }
  }
  return 0;
}

}  // extern "C"

// ==================================================================== Beziers
namespace {
constexpr uint32_t BEZ_MAX_TILE = 1024;        // constants.ts:20
constexpr float BEZ_FP_POS = 10000.0f, BEZ_FP_COL = 100000.0f;  // constants.ts:18-19
constexpr float BEZ_KILL_ALPHA = 0.005f;       // constants.ts:15
constexpr uint32_t N_SEG = 16;                 // bezier_backward.wgsl:52
constexpr float DEPTH_NEAR_BEZ = 0.1f;         // bezier_backward.wgsl:54

// bezier_backward.wgsl:56-62
inline V2 bezier_at(V2 p0, V2 p1, V2 p2, V2 p3, float t) {
  float omt = 1.0f - t;
  float c0 = omt * omt * omt, c1 = 3.0f * omt * omt * t, c2 = 3.0f * omt * t * t, c3 = t * t * t;
  return {c0 * p0.x + c1 * p1.x + c2 * p2.x + c3 * p3.x, c0 * p0.y + c1 * p1.y + c2 * p2.y + c3 * p3.y};
}
// bezier_backward.wgsl:64-67
inline V4 bernstein(float t) {
  float omt = 1.0f - t;
  return {omt * omt * omt, 3.0f * omt * omt * t, 3.0f * omt * t * t, t * t * t};
}
struct PC { float x, y, w; };
// bezier_backward.wgsl:69-72
inline PC project_center(const float* vp, const float* p3, float aspect) {
  V4 c = mulv(vp, p3[0], p3[1], p3[2], 1.0f);
  return {c.x / c.w * aspect, c.y / c.w, c.w};
}
// bezier_backward.wgsl:74-88
inline V3 backproject(const float* vp, const float* p3, float aspect, V2 d) {
  V4 c = mulv(vp, p3[0], p3[1], p3[2], 1.0f);
  float w = c.w, w2 = w * w;
  float o[3];
  for (int ax = 0; ax < 3; ++ax) {
    float v0 = vp[ax * 4 + 0], v1 = vp[ax * 4 + 1], v3 = vp[ax * 4 + 3];
    float dsx = aspect * (v0 * w - c.x * v3) / w2;
    float dsy = (v1 * w - c.y * v3) / w2;
    o[ax] = d.x * dsx + d.y * dsy;
  }
  return {o[0], o[1], o[2]};
}
inline float dot3v(const float* a, float x, float y, float z) { return a[0] * x + a[1] * y + a[2] * z; }
inline float tex_dot(const float* rgba, int32_t x, int32_t y, uint32_t w, float kx, float ky, float kz) {
  const float* t = rgba + ((size_t)y * w + x) * 4;
  return t[0] * kx + t[1] * ky + t[2] * kz;
}
inline int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return std::min(std::max(v, lo), hi); }
}  // namespace

extern "C" {

// Bezier forward + loss + backward for one view: bezier_backward.wgsl:103-572.
//   beziers N x 20 (p0.xyz width, p1.xyz softness, p2.xyz _, p3.xyz _, rgba)
//   uni[6] = {mode, max_width, prune_alpha, prune_width, bg_penalty, _}
//   textures H x W x 4 (target, background, normal); depths H x W (.r)
//   grads_q  N x 18 i32 (+=); grads_f N x 18 unquantised (+=, may be null)
//   loss_accum N (+=, the shader's non-atomic RMW), pixel_loss (+=, indexed y*W+x)
//   terms    N (+=, may be null): (pixel, curve) backward terms (alpha >= 0.001)
//            each curve's gradient sums
int orc_bezier_backward(const float* beziers, uint32_t n, const float* vp, const float* uni,
                        const float* tgt_rgba, const float* tgt_depth, const float* bg_rgba,
                        const float* bg_depth, const float* normal_rgba, uint32_t w, uint32_t h,
                        int32_t* grads_q, float* grads_f, float* loss_accum, int32_t* pixel_loss,
                        float* out_rgbd, uint32_t* tile_count, uint32_t* terms) {
  const float aspect = (float)w / (float)h;
  const uint32_t tiles_x = (w + 15) / 16, tiles_y = (h + 15) / 16;
  const float mode = uni[0], max_width = uni[1], bg_penalty = uni[4];
  const bool color_mode = mode > 0.5f;
  // per-curve projected control points (the shader recomputes them per pixel;
  // identical arithmetic)
  std::vector<PC> pcs(4 * (size_t)n);
  std::vector<uint8_t> live(n);
  std::vector<float> bb(4 * (size_t)n);
  for (uint32_t i = 0; i < n; ++i) {
    const float* b = beziers + 20 * (size_t)i;
    for (int k = 0; k < 4; ++k) pcs[4 * i + k] = project_center(vp, b + 4 * k, aspect);
    live[i] = 0;
    if (b[19] < BEZ_KILL_ALPHA) continue;
    float width = std::fmax(b[3], 0.001f), soft = std::fmax(b[7], 0.001f);
    const PC* q = &pcs[4 * i];
    if (q[0].w <= 0.0f || q[1].w <= 0.0f || q[2].w <= 0.0f || q[3].w <= 0.0f) continue;
    float oc = width + soft;
    float mnx = std::fmin(std::fmin(q[0].x, q[1].x), std::fmin(q[2].x, q[3].x)) - oc;
    float mny = std::fmin(std::fmin(q[0].y, q[1].y), std::fmin(q[2].y, q[3].y)) - oc;
    float mxx = std::fmax(std::fmax(q[0].x, q[1].x), std::fmax(q[2].x, q[3].x)) + oc;
    float mxy = std::fmax(std::fmax(q[0].y, q[1].y), std::fmax(q[2].y, q[3].y)) + oc;
    bb[4 * i] = mnx; bb[4 * i + 1] = mny; bb[4 * i + 2] = mxx; bb[4 * i + 3] = mxy;
    live[i] = 1;
  }
  std::vector<uint32_t> list;
  std::vector<float> alphas(BEZ_MAX_TILE), depths(BEZ_MAX_TILE), Ts(BEZ_MAX_TILE + 1);
  std::vector<uint32_t> min_seg(BEZ_MAX_TILE);
  const float lw[3] = {0.2126f, 0.7152f, 0.0722f};
  for (uint32_t ty = 0; ty < tiles_y; ++ty)
    for (uint32_t tx = 0; tx < tiles_x; ++tx) {
      float tmin[2], tmax[2];
      tile_rect(tx, ty, w, h, aspect, tmin, tmax);
      list.clear();
      for (uint32_t i = 0; i < n && list.size() < BEZ_MAX_TILE; ++i) {
        if (!live[i]) continue;
        const float* b = &bb[4 * i];
        if (!(b[0] > tmax[0] || b[2] < tmin[0] || b[1] > tmax[1] || b[3] < tmin[1])) list.push_back(i);
      }
      if (tile_count) tile_count[ty * tiles_x + tx] = (uint32_t)list.size();
      const uint32_t cnt = (uint32_t)list.size();
      for (uint32_t py = ty * 16; py < std::min(ty * 16 + 16, h); ++py)
        for (uint32_t px = tx * 16; px < std::min(tx * 16 + 16, w); ++px) {
          const size_t pix = (size_t)py * w + px;
          V2 p = pixel_to_p(px, py, w, h, aspect);
          const float* tc = tgt_rgba + pix * 4;
          const float td = tgt_depth[pix];
          Ts[0] = 1.0f;
          float Cr = 0, Cg = 0, Cb = 0, D = 0;
          for (uint32_t k = 0; k < cnt; ++k) {
            const float* b = beziers + 20 * (size_t)list[k];
            const PC* q = &pcs[4 * list[k]];
            float width = std::fmax(b[3], 0.001f), soft = std::fmax(b[7], 0.001f), opacity = b[19];
            V2 p0{q[0].x, q[0].y}, p1{q[1].x, q[1].y}, p2{q[2].x, q[2].y}, p3{q[3].x, q[3].y};
            float min_d = 1e9f, min_u = 0.0f;
            uint32_t min_k = 1;
            V2 prev = p0;
            for (uint32_t s = 1; s <= N_SEG; ++s) {
              V2 cur = bezier_at(p0, p1, p2, p3, (float)s / (float)N_SEG);
              V2 seg{cur.x - prev.x, cur.y - prev.y};
              float len2 = std::fmax(seg.x * seg.x + seg.y * seg.y, 1e-8f);
              float u = clampf(((p.x - prev.x) * seg.x + (p.y - prev.y) * seg.y) / len2, 0.0f, 1.0f);
              V2 pr{prev.x + u * seg.x, prev.y + u * seg.y};
              V2 df{p.x - pr.x, p.y - pr.y};
              float d = std::sqrt(df.x * df.x + df.y * df.y);
              if (d < min_d) { min_d = d; min_k = s; min_u = u; }
              prev = cur;
            }
            float t = ((float)(min_k - 1) + min_u) / (float)N_SEG;
            float dt = t - 0.5f;
            float pressure = 1.0f - 4.0f * dt * dt;
            float lwid = width * pressure, lsoft = soft * pressure, lop = opacity * pressure;
            float a_geom = 1.0f - smoothstepf(lwid - lsoft, lwid + lsoft, min_d);
            float a = clampf(a_geom * lop, 0.0f, 0.999f);
            V4 B = bernstein(t);
            float raw_w = B.x * q[0].w + B.y * q[1].w + B.z * q[2].w + B.w * q[3].w;
            float lin_w = std::fmax(raw_w, DEPTH_NEAR_BEZ);
            float dv = clampf(1.0f - DEPTH_NEAR_BEZ / lin_w, 0.0f, 1.0f);
            alphas[k] = a;
            min_seg[k] = min_k;
            depths[k] = dv;
            Cr += Ts[k] * a * b[16]; Cg += Ts[k] * a * b[17]; Cb += Ts[k] * a * b[18];
            D += Ts[k] * a * dv;
            Ts[k + 1] = Ts[k] * (1.0f - a);
          }
          float bgr = 0, bgg = 0, bgb = 0, bgd = 1.0f;
          if (color_mode) {
            const float* bt = bg_rgba + pix * 4;
            bgr = bt[0]; bgg = bt[1]; bgb = bt[2];
            bgd = bg_depth[pix];
          }
          Cr += Ts[cnt] * bgr; Cg += Ts[cnt] * bgg; Cb += Ts[cnt] * bgb;
          D += Ts[cnt] * bgd;
          if (out_rgbd) {
            float* o = out_rgbd + pix * 4;
            o[0] = Cr; o[1] = Cg; o[2] = Cb; o[3] = D;
          }
          // loss, bezier_backward.wgsl:271-320
          float dCr_raw = 2.0f * (Cr - tc[0]), dCg_raw = 2.0f * (Cg - tc[1]), dCb_raw = 2.0f * (Cb - tc[2]);
          bool fgb = td < 0.99f;
          float dD_total = (fgb && color_mode) ? 0.5f * 2.0f * (D - td) : 0.0f;
          float luma_err = (dCr_raw * 0.5f) * lw[0] + (dCg_raw * 0.5f) * lw[1] + (dCb_raw * 0.5f) * lw[2];
          int32_t ix = (int32_t)px, iy = (int32_t)py, W1 = (int32_t)w - 1, H1 = (int32_t)h - 1;
          float luma_r = tex_dot(tgt_rgba, clampi(ix + 1, 0, W1), clampi(iy, 0, H1), w, lw[0], lw[1], lw[2]);
          float luma_l = tex_dot(tgt_rgba, clampi(ix - 1, 0, W1), clampi(iy, 0, H1), w, lw[0], lw[1], lw[2]);
          float luma_u = tex_dot(tgt_rgba, clampi(ix, 0, W1), clampi(iy + 1, 0, H1), w, lw[0], lw[1], lw[2]);
          float luma_d = tex_dot(tgt_rgba, clampi(ix, 0, W1), clampi(iy - 1, 0, H1), w, lw[0], lw[1], lw[2]);
          float contrast = std::sqrt((luma_r - luma_l) * (luma_r - luma_l) + (luma_u - luma_d) * (luma_u - luma_d));
          float cw = 1.0f + clampf(contrast * 8.0f, 0.0f, 3.0f);
          float dl[3] = {luma_err * lw[0] * 6.0f, luma_err * lw[1] * 6.0f, luma_err * lw[2] * 6.0f};
          float dr_dot = dCr_raw * lw[0] + dCg_raw * lw[1] + dCb_raw * lw[2];
          float dch[3] = {dCr_raw - dr_dot * lw[0], dCg_raw - dr_dot * lw[1], dCb_raw - dr_dot * lw[2]};
          float dC[3] = {(dl[0] + dch[0]) * cw, (dl[1] + dch[1]) * cw, (dl[2] + dch[2]) * cw};
          float dT = (dC[0] * bgr + dC[1] * bgg + dC[2] * bgb) + dD_total * bgd;
          float coverage = 1.0f - Ts[cnt];
          float edge_target = tc[0];
          float d_cov = mode < 0.5f ? 2.0f * 2.0f * (coverage - edge_target) : 0.0f;
          dT += -d_cov;
          float is_bg = (0.995f <= td) ? 1.0f : 0.0f;
          for (uint32_t j = 0; j < cnt; ++j) {
            uint32_t idx = cnt - 1 - j;
            float a = alphas[idx];
            if (a < 0.001f) continue;
            uint32_t i = list[idx];
            if (terms) ++terms[i];
            const float* b = beziers + 20 * (size_t)i;
            const PC* q = &pcs[4 * i];
            float width = std::fmax(b[3], 0.001f), soft = std::fmax(b[7], 0.001f), opacity = b[19];
            float col[3] = {b[16], b[17], b[18]};
            V2 p0{q[0].x, q[0].y}, p1{q[1].x, q[1].y}, p2{q[2].x, q[2].y}, p3{q[3].x, q[3].y};
            float T_prev = Ts[idx];
            float d_val = depths[idx];
            float TA = T_prev * a;
            float dColor[3] = {dC[0] * TA, dC[1] * TA, dC[2] * TA};
            float tcol[3] = {T_prev * col[0], T_prev * col[1], T_prev * col[2]};
            float da = dT * (-T_prev) + (dC[0] * tcol[0] + dC[1] * tcol[1] + dC[2] * tcol[2]) + dD_total * (T_prev * d_val);
            float acol[3] = {a * col[0], a * col[1], a * col[2]};
            dT = dT * (1.0f - a) + (dC[0] * acol[0] + dC[1] * acol[1] + dC[2] * acol[2]) + dD_total * (a * d_val);
            uint32_t kseg = min_seg[idx];
            float t_prev = (float)(kseg - 1) / (float)N_SEG, t_curr = (float)kseg / (float)N_SEG;
            V2 pp = bezier_at(p0, p1, p2, p3, t_prev), cp = bezier_at(p0, p1, p2, p3, t_curr);
            V2 seg{cp.x - pp.x, cp.y - pp.y};
            float len2 = std::fmax(seg.x * seg.x + seg.y * seg.y, 1e-8f);
            float u_c = clampf(((p.x - pp.x) * seg.x + (p.y - pp.y) * seg.y) / len2, 0.0f, 1.0f);
            V2 pr{pp.x + u_c * seg.x, pp.y + u_c * seg.y};
            V2 dvv{p.x - pr.x, p.y - pr.y};
            float d = std::fmax(std::sqrt(dvv.x * dvv.x + dvv.y * dvv.y), 1e-6f);
            float t_pix = ((float)(kseg - 1) + u_c) / (float)N_SEG;
            float dtp = t_pix - 0.5f;
            float pressure = 1.0f - 4.0f * dtp * dtp;
            V4 Bp = bernstein(t_pix);
            float lwid = width * pressure, lsoft = soft * pressure, lop = opacity * pressure;
            float inner = lwid - lsoft, outer = lwid + lsoft;
            float denom = std::fmax(outer - inner, 1e-6f);
            float x_in = clampf((d - inner) / denom, 0.0f, 1.0f);
            float ss_d = 6.0f * x_in * (1.0f - x_in) / denom;
            bool in_band = (d > inner) && (d < outer);
            float a_geom = 1.0f - smoothstepf(inner, outer, d);
            float bg_pen = bg_penalty * is_bg;
            float d_opacity = da * a_geom * pressure + bg_pen;
            float da_eff = da * lop;
            float dDd = in_band ? -da_eff * ss_d : 0.0f;
            float dWidth = in_band ? da_eff * ss_d * pressure / denom : 0.0f;
            float dmi = clampf(d - inner, 0.0f, denom);
            float dx_ds = pressure * (denom - 2.0f * dmi) / std::fmax(denom * denom, 1e-12f);
            float dSoft = in_band ? -da_eff * ss_d * dx_ds : 0.0f;
            float w0 = project_center(vp, b + 0, aspect).w, w1 = project_center(vp, b + 4, aspect).w;
            float w2 = project_center(vp, b + 8, aspect).w, w3 = project_center(vp, b + 12, aspect).w;
            float raw_w = Bp.x * w0 + Bp.y * w1 + Bp.z * w2 + Bp.w * w3;
            float lin_w = std::fmax(raw_w, DEPTH_NEAR_BEZ);
            float ddw = DEPTH_NEAR_BEZ / (lin_w * lin_w);
            float kz = dD_total * (T_prev * a) * ddw;
            float dZ[4] = {kz * Bp.x, kz * Bp.y, kz * Bp.z, kz * Bp.w};
            float dprx = -dDd * dvv.x / d, dpry = -dDd * dvv.y / d;
            V2 dPrev{(1.0f - u_c) * dprx, (1.0f - u_c) * dpry};
            V2 dCurr{u_c * dprx, u_c * dpry};
            V4 Bpv = bernstein(t_prev), Bcv = bernstein(t_curr);
            bool is_fine = max_width > 0.0f;
            int32_t* gq = grads_q + 18 * (size_t)i;
            float* gf = grads_f ? grads_f + 18 * (size_t)i : nullptr;
            dSoft += is_fine ? 5.0f * 2.0f * soft : 0.0f;
            if (is_fine && len2 > 1e-10f) {
              float sl = std::sqrt(len2);
              V2 tang{seg.x / sl, seg.y / sl};
              int32_t rx = clampi(ix + 2, 0, W1), lx = clampi(ix - 2, 0, W1);
              int32_t uy = clampi(iy + 2, 0, H1), dy = clampi(iy - 2, 0, H1);
              float cr = tex_dot(tgt_rgba, rx, iy, w, 0.333f, 0.333f, 0.333f);
              float cl = tex_dot(tgt_rgba, lx, iy, w, 0.333f, 0.333f, 0.333f);
              float cu = tex_dot(tgt_rgba, ix, uy, w, 0.333f, 0.333f, 0.333f);
              float cd = tex_dot(tgt_rgba, ix, dy, w, 0.333f, 0.333f, 0.333f);
              float gx = (cr - cl) * 0.25f * aspect, gy = -(cu - cd) * 0.25f;
              float nr = tex_dot(normal_rgba, rx, iy, w, 0.333f, 0.333f, 0.333f);
              float nl = tex_dot(normal_rgba, lx, iy, w, 0.333f, 0.333f, 0.333f);
              float nu = tex_dot(normal_rgba, ix, uy, w, 0.333f, 0.333f, 0.333f);
              float nd = tex_dot(normal_rgba, ix, dy, w, 0.333f, 0.333f, 0.333f);
              float gnx = (nr - nl) * 0.25f * aspect, gny = -(nu - nd) * 0.25f;
              float frx = gx + 2.0f * gnx, fry = gy + 2.0f * gny;
              float flen = std::sqrt(frx * frx + fry * fry);
              if (flen > 1e-4f) {
                V2 fd{frx / flen, fry / flen};
                float tg = tang.x * fd.x + tang.y * fd.y;
                float dld = 1.5f * 2.0f * tg;
                V2 dtv{dld * fd.x, dld * fd.y};
                float il = 1.0f / std::sqrt(len2);
                float tdot = dtv.x * tang.x + dtv.y * tang.y;
                V2 dseg{(dtv.x - tang.x * tdot) * il, (dtv.y - tang.y * tdot) * il};
                V2 dPd{-dseg.x, -dseg.y}, dCd = dseg;
                V2 dP2d[4] = {{Bpv.x * dPd.x + Bcv.x * dCd.x, Bpv.x * dPd.y + Bcv.x * dCd.y},
                              {Bpv.y * dPd.x + Bcv.y * dCd.x, Bpv.y * dPd.y + Bcv.y * dCd.y},
                              {Bpv.z * dPd.x + Bcv.z * dCd.x, Bpv.z * dPd.y + Bcv.z * dCd.y},
                              {Bpv.w * dPd.x + Bcv.w * dCd.x, Bpv.w * dPd.y + Bcv.w * dCd.y}};
                for (int c = 0; c < 4; ++c) {
                  V3 d3 = backproject(vp, b + 4 * c, aspect, dP2d[c]);
                  float gg[3] = {d3.x, d3.y, d3.z};
                  for (int k = 0; k < 3; ++k) {
                    gq[3 * c + k] = wrap_add(gq[3 * c + k], to_i32(gg[k] * BEZ_FP_POS));
                    if (gf) gf[3 * c + k] += gg[k];
                  }
                }
              }
            }
            V2 dP[4] = {{Bpv.x * dPrev.x + Bcv.x * dCurr.x, Bpv.x * dPrev.y + Bcv.x * dCurr.y},
                        {Bpv.y * dPrev.x + Bcv.y * dCurr.x, Bpv.y * dPrev.y + Bcv.y * dCurr.y},
                        {Bpv.z * dPrev.x + Bcv.z * dCurr.x, Bpv.z * dPrev.y + Bcv.z * dCurr.y},
                        {Bpv.w * dPrev.x + Bcv.w * dCurr.x, Bpv.w * dPrev.y + Bcv.w * dCurr.y}};
            float g18[18];
            for (int c = 0; c < 4; ++c) {
              V3 d3 = backproject(vp, b + 4 * c, aspect, dP[c]);
              g18[3 * c + 0] = d3.x;
              g18[3 * c + 1] = d3.y;
              g18[3 * c + 2] = d3.z + dZ[c];
            }
            g18[12] = dColor[0]; g18[13] = dColor[1]; g18[14] = dColor[2]; g18[15] = d_opacity;
            g18[16] = dWidth; g18[17] = dSoft;
            for (int k = 0; k < 18; ++k) {
              float sc = (k >= 12 && k <= 15) ? BEZ_FP_COL : BEZ_FP_POS;
              gq[k] = wrap_add(gq[k], to_i32(g18[k] * sc));
              if (gf) gf[k] += g18[k];
            }
            float clc = (dC[0] * dC[0] * 1.0f + dC[1] * dC[1] * 1.0f + dC[2] * dC[2] * 1.0f) * (T_prev * a);
            loss_accum[i] += clc;
          }
          float hr = dCr_raw * 0.5f, hg = dCg_raw * 0.5f, hb = dCb_raw * 0.5f;
          float residual = (hr * hr + hg * hg + hb * hb) * Ts[cnt];
          pixel_loss[pix] = wrap_add(pixel_loss[pix], to_i32(residual * 10000.0f));
        }
    }
  return 0;
}

// Bezier Adam step: bezier_step.wgsl:50-189.  uni[6] as above; t by value.
int orc_bezier_step(float* beziers, int32_t* grads, float* m, float* v, float* adam_t, float pixel_count,
                    float no_kill, float* grad_accum, const float* vp, const float* uni, uint32_t n) {
  static const float lr[18] = {0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f,
                               0.005f, 0.005f, 0.005f, 0.01f, 0.01f, 0.01f, 0.005f, 0.002f, 0.002f};
  static const float mu[18] = {0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.005f,
                               0.005f, 0.005f, 0.005f, 0.01f, 0.01f, 0.01f, 0.005f, 0.003f, 0.003f};
  const float max_width = uni[1], pa = uni[2], pw = uni[3];
  const float t = *adam_t + 1.0f;
  for (uint32_t i = 0; i < n; ++i) {
    float* b = beziers + 20 * (size_t)i;
    if (b[19] < BEZ_KILL_ALPHA) {
      for (int k = 0; k < 18; ++k) grads[18 * (size_t)i + k] = 0;
      continue;
    }
    // flat parameter order of bezier_step.wgsl:132-139 -> record offsets
    static const int off[18] = {0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14, 16, 17, 18, 19, 3, 7};
    const float width_hi = max_width > 0.0f ? max_width : 0.1f;
    float pos_g2 = 0.0f;
    for (int k = 0; k < 18; ++k) {
      size_t pi = 18 * (size_t)i + k;
      int32_t raw = grads[pi];
      grads[pi] = 0;
      float fps = (k >= 12 && k <= 15) ? BEZ_FP_COL : BEZ_FP_POS;
      float pn = 1.0f / std::fmax(pixel_count, 1.0f);
      float g = (float)raw / fps * pn;
      float mm = ADAM_B1 * m[pi] + (1.0f - ADAM_B1) * g;
      float vv = ADAM_B2 * v[pi] + (1.0f - ADAM_B2) * g * g;
      m[pi] = mm;
      v[pi] = vv;
      float m_hat = mm / (1.0f - std::pow(ADAM_B1, t));
      float v_hat = vv / (1.0f - std::pow(ADAM_B2, t));
      float raw_u = lr[k] * m_hat / (std::sqrt(v_hat) + ADAM_EPS);
      float u = clampf(raw_u, -mu[k], mu[k]);
      float lo = k < 12 ? -1e9f : (k < 16 ? 0.0f : 0.001f);
      float hi = k < 12 ? 1e9f : (k < 15 ? 1.0f : (k == 15 ? 0.99f : (k == 16 ? width_hi : 0.03f)));
      b[off[k]] = clampf(b[off[k]] - u, lo, hi);
      if (k <= 11) pos_g2 += g * g;
    }
    grad_accum[i] += std::sqrt(pos_g2);
    float at = pa > 0.0f ? pa : 0.001f;
    float wt = pw > 0.0f ? pw : 0.001f;
    if (b[19] < at || b[3] <= wt) b[19] = 0.0f;
    if (b[19] > 0.0f && no_kill < 0.5f) {
      V4 c[4];
      for (int k = 0; k < 4; ++k) c[k] = mulv(vp, b[4 * k], b[4 * k + 1], b[4 * k + 2], 1.0f);
      const float mg = 1.2f;  // constants.ts:14
      bool L = true, R = true, Bo = true, A = true, Be = true;
      for (int k = 0; k < 4; ++k) {
        L = L && c[k].x < -mg * c[k].w;
        R = R && c[k].x > mg * c[k].w;
        Bo = Bo && c[k].y < -mg * c[k].w;
        A = A && c[k].y > mg * c[k].w;
        Be = Be && c[k].w < 0.0f;
      }
      if (L || R || Bo || A || Be) b[19] = 0.0f;
    }
  }
  *adam_t = t;
  return 0;
}

// Bezier ADC: bezier_adc.wgsl:75-315 (serial passes, reference order).
int orc_bezier_adc(float* beziers, float* m, float* v, float adam_t, float no_kill, float* grad_accum,
                   float* loss_accum, int32_t* pixel_loss, const float* vp, const float* vpinv, uint32_t n) {
  const float P = 50.0f, TAU_POS = 0.0002f, TAU_LOSS = 0.001f, SPLIT_LEN = 0.25f;  // constants.ts:6-9
  const uint32_t PLS = 512u * 512u, OW = 256u, OH = 256u;  // constants.ts:10; manager bakes 256x256
  std::vector<uint32_t> dead;
  dead.reserve(n);
  for (uint32_t i = 0; i < n; ++i)
    if (beziers[20 * (size_t)i + 19] < BEZ_KILL_ALPHA) dead.push_back(i);
  auto offscreen = [&](const float* p3) {
    V4 c = mulv(vp, p3[0], p3[1], p3[2], 1.0f);
    if (c.w < 0.0f) return true;
    float iw = std::fmax(c.w, 1e-5f);
    float nx = c.x / iw, ny = c.y / iw;
    return std::fabs(nx) > 1.2f || std::fabs(ny) > 1.2f;
  };
  // pass 1
  for (uint32_t i = 0; i < n; ++i) {
    float* b = beziers + 20 * (size_t)i;
    if (b[19] < BEZ_KILL_ALPHA) continue;
    float gn = grad_accum[i] / P, ln = loss_accum[i] / P;
    if (no_kill < 0.5f && gn <= TAU_POS && ln > TAU_LOSS) { b[19] = 0.0f; dead.push_back(i); continue; }
    if (offscreen(b) && offscreen(b + 4) && offscreen(b + 8) && offscreen(b + 12)) { b[19] = 0.0f; dead.push_back(i); }
  }
  auto clone_split = [&](uint32_t i, uint32_t ni) {
    float* b = beziers + 20 * (size_t)i;
    float nb[20];
    std::memcpy(nb, b, sizeof(nb));
    float p[4][3];
    for (int c = 0; c < 4; ++c) for (int k = 0; k < 3; ++k) p[c][k] = b[4 * c + k];
    float mid[3], len_a = 0, len_b = 0;
    for (int k = 0; k < 3; ++k) mid[k] = (p[0][k] + 3.0f * p[1][k] + 3.0f * p[2][k] + p[3][k]) * 0.125f;
    float da[3], db[3];
    for (int k = 0; k < 3; ++k) { da[k] = mid[k] - p[0][k]; db[k] = p[3][k] - mid[k]; }
    len_a = std::sqrt(da[0] * da[0] + da[1] * da[1] + da[2] * da[2]);
    len_b = std::sqrt(db[0] * db[0] + db[1] * db[1] + db[2] * db[2]);
    if (len_a + len_b > SPLIT_LEN) {
      float q0[3], q1[3], q2[3], r0[3], r1[3], s[3];
      for (int k = 0; k < 3; ++k) {
        q0[k] = (p[0][k] + p[1][k]) * 0.5f; q1[k] = (p[1][k] + p[2][k]) * 0.5f; q2[k] = (p[2][k] + p[3][k]) * 0.5f;
        r0[k] = (q0[k] + q1[k]) * 0.5f; r1[k] = (q1[k] + q2[k]) * 0.5f; s[k] = (r0[k] + r1[k]) * 0.5f;
      }
      for (int k = 0; k < 3; ++k) {
        b[0 + k] = p[0][k]; b[4 + k] = q0[k]; b[8 + k] = r0[k]; b[12 + k] = s[k];
        nb[0 + k] = s[k]; nb[4 + k] = r1[k]; nb[8 + k] = q2[k]; nb[12 + k] = p[3][k];
      }
      b[11] = 0.0f; b[15] = 0.0f; nb[11] = 0.0f; nb[15] = 0.0f;
    } else {
      float seed = (float)i * 3.14159f + adam_t;
      float j[3] = {(fractf(std::sin(seed * 12.9898f) * 43758.5453f) - 0.5f) * 0.001f,
                    (fractf(std::sin(seed * 78.233f) * 43758.5453f) - 0.5f) * 0.001f,
                    (fractf(std::sin(seed * 43.123f) * 43758.5453f) - 0.5f) * 0.001f};
      for (int c = 0; c < 4; ++c)
        for (int k = 0; k < 3; ++k) nb[4 * c + k] = b[4 * c + k] + j[k];
      nb[11] = 0.0f; nb[15] = 0.0f;
    }
    std::memcpy(beziers + 20 * (size_t)ni, nb, sizeof(nb));
    for (int k = 0; k < 18; ++k) {
      m[18 * (size_t)i + k] = 0; v[18 * (size_t)i + k] = 0;
      m[18 * (size_t)ni + k] = 0; v[18 * (size_t)ni + k] = 0;
    }
  };
  // pass 1.5
  for (uint32_t i = 0; i < n; ++i) {
    float* b = beziers + 20 * (size_t)i;
    if (b[19] < BEZ_KILL_ALPHA) continue;
    float gn = grad_accum[i] / P;
    if (gn <= TAU_POS) continue;
    if (dead.empty()) continue;
    uint32_t ni = dead.back();
    dead.pop_back();
    clone_split(i, ni);
  }
  // pass 2: spawn at pixel_loss maxima
  uint32_t max_sp = std::min<uint32_t>((uint32_t)dead.size(), 512u);
  uint32_t stride = std::max(1u, PLS / 4096u);
  for (uint32_t sp = 0; sp < max_sp; ++sp) {
    if (dead.empty()) break;
    uint32_t best_px = 0;
    int32_t best_val = 0;
    uint32_t start = (sp * 997u) % stride;
    for (uint32_t px = start; px < PLS; px += stride) {
      int32_t vv = pixel_loss[px];
      if (vv > best_val) { best_val = vv; best_px = px; }
    }
    uint32_t spx = best_px;
    if (best_val <= 0) {
      float sf = (float)sp * 1234.5678f + adam_t * 0.1f;
      uint32_t rx = (uint32_t)std::max(0.0f, fractf(std::sin(sf * 12.9898f) * 43758.5453f) * (float)OW);
      uint32_t ry = (uint32_t)std::max(0.0f, fractf(std::sin(sf * 78.233f) * 43758.5453f) * (float)OH);
      spx = ry * OW + rx;
    } else {
      pixel_loss[best_px] = 0;
    }
    uint32_t slot = dead.back();
    dead.pop_back();
    // pixel_to_world, bezier_adc.wgsl:52-65
    uint32_t pxx = spx % OW, pyy = spx / OW;
    float ux = ((float)pxx + 0.5f) / (float)OW, uy = ((float)pyy + 0.5f) / (float)OH;
    float ndx = ux * 2.0f - 1.0f, ndy = 1.0f - uy * 2.0f;
    float wv = 0.1f / std::fmax(1.0f - 0.5f, 1e-5f);
    V4 wp = mulv(vpinv, ndx * wv, ndy * wv, wv, wv);
    float ctr[3] = {wp.x / wp.w, wp.y / wp.w, wp.z / wp.w};
    float seed = (float)spx * 1.61803f + (float)sp * 2.71828f;
    float ang = fractf(std::sin(seed * 127.1f) * 43758.5453f) * 6.28318f;
    float tgx = std::cos(ang) * 0.025f, tgz = std::sin(ang) * 0.025f;  // constants.ts:11
    float* nb = beziers + 20 * (size_t)slot;
    nb[0] = ctr[0] - tgx; nb[1] = ctr[1] - 0.0f; nb[2] = ctr[2] - tgz; nb[3] = 0.015f;
    nb[4] = ctr[0] - tgx * 0.33f; nb[5] = ctr[1] - 0.0f * 0.33f; nb[6] = ctr[2] - tgz * 0.33f; nb[7] = 0.005f;
    nb[8] = ctr[0] + tgx * 0.33f; nb[9] = ctr[1] + 0.0f * 0.33f; nb[10] = ctr[2] + tgz * 0.33f; nb[11] = 0.0f;
    nb[12] = ctr[0] + tgx; nb[13] = ctr[1] + 0.0f; nb[14] = ctr[2] + tgz; nb[15] = 0.0f;
    nb[16] = 0.5f; nb[17] = 0.5f; nb[18] = 0.5f; nb[19] = 0.5f;
    for (int k = 0; k < 18; ++k) { m[18 * (size_t)slot + k] = 0; v[18 * (size_t)slot + k] = 0; }
  }
  // pass 3
  for (uint32_t i = 0; i < n; ++i) {
    if (dead.empty()) break;
    float* b = beziers + 20 * (size_t)i;
    if (b[19] < BEZ_KILL_ALPHA) continue;
    float gn = grad_accum[i] / P;
    if (gn <= TAU_POS) continue;
    uint32_t ni = dead.back();
    dead.pop_back();
    clone_split(i, ni);
  }
  std::memset(pixel_loss, 0, sizeof(int32_t) * PLS);
  for (uint32_t i = 0; i < n; ++i) { grad_accum[i] = 0; loss_accum[i] = 0; }
  return 0;
}

}  // extern "C"

// ============================================================ display forwards
namespace {
// Point-in-quad with the top-left rule: the quad is the axis-aligned screen
// rectangle [x0, x1] x [y0, y1] (aspect-corrected, y up); left and top edges
// are inside, right and bottom edges outside.
inline bool in_quad(V2 p, float x0, float x1, float y0, float y1) {
  return p.x >= x0 && p.x < x1 && p.y > y0 && p.y <= y1;
}
// Per-splat screen quad of splat_forward.wgsl's vertex stage (vert, :43-117):
// centre, extent rectangle, conic and encoded depth; ok = false when culled.
struct SplatQuad { bool ok; float cx, cy, x0, x1, y0, y1, A, B, C, depth; };

std::vector<SplatQuad> splat_quads(const float* splats, uint32_t n, const float* vp, uint32_t w, uint32_t h) {
  const float aspect = (float)w / (float)h;
  std::vector<SplatQuad> q(n);
  for (uint32_t i = 0; i < n; ++i) {
    const float* s = splats + 16 * (size_t)i;
    SplatQuad& o = q[i];
    o.ok = false;
    const float sx = std::fmax(s[3], 0.0001f), sy = std::fmax(s[12], 0.0001f), sz = std::fmax(s[15], 0.0001f);
    const float safe_b = std::fmax(s[14], 0.0001f);
    const float R = std::pow(15.0f / safe_b, 1.0f / s[13]);
    V4 clip = mulv(vp, s[0], s[1], s[2], 1.0f);
    const float W = clip.w;
    if (W < 0.1f) continue;
    // all six vertices carry the centre's clip z and w: clipping against
    // 0 <= z <= w keeps or drops the whole quad
    if (!(clip.z >= 0.0f && clip.z <= W)) continue;
    V4 qq{s[8], s[9], s[10], s[11]};
    V2 ax = project_axis(vp, quat_rotate(qq, {1, 0, 0}), clip.x, clip.y, W, aspect);
    V2 ay = project_axis(vp, quat_rotate(qq, {0, 1, 0}), clip.x, clip.y, W, aspect);
    V2 az = project_axis(vp, quat_rotate(qq, {0, 0, 1}), clip.x, clip.y, W, aspect);
    const float m0x = ax.x * sx, m0y = ax.y * sx, m1x = ay.x * sy, m1y = ay.y * sy, m2x = az.x * sz, m2y = az.y * sz;
    float cov00 = m0x * m0x + m1x * m1x + m2x * m2x;
    float cov01 = m0x * m0y + m1x * m1y + m2x * m2y;
    float cov11 = m0y * m0y + m1y * m1y + m2y * m2y;
    const float fs = 0.3f * (2.0f / (float)h);
    cov00 += fs * fs;
    cov11 += fs * fs;
    const float det = cov00 * cov11 - cov01 * cov01;
    const float inv_det = std::fabs(det) < 1e-10f ? 0.0f : 1.0f / det;
    o.A = cov11 * inv_det; o.B = -cov01 * inv_det; o.C = cov00 * inv_det;
    const float ex = R * std::sqrt(std::fmax(cov00, 1e-9f)), ey = R * std::sqrt(std::fmax(cov11, 1e-9f));
    o.cx = clip.x / W * aspect;
    o.cy = clip.y / W;
    o.x0 = o.cx - ex; o.x1 = o.cx + ex; o.y0 = o.cy - ey; o.y1 = o.cy + ey;
    const float ld = std::fmax(W, 0.1f);
    o.depth = clampf(1.0f - 0.1f / ld, 0.0f, 1.0f);
    o.ok = true;
  }
  return q;
}
}  // namespace

extern "C" {

// splat_forward.wgsl:42-156 with GpuSplatForwardPipelineManager.dispatch(clear)
// (GpuSplatForwardPipelineManager.ts:114-137), headless and in fp32: instances
// are drawn in reverse index order with src-alpha blending, which equals
// front-to-back compositing with splat 0 in front.  out_rgba / out_depth:
// H x W x 4 (colour rgb + alpha; encoded depth in rgb + alpha).
int orc_splat_render(const float* splats, uint32_t n, const float* vp, uint32_t w, uint32_t h, float* out_rgba,
                     float* out_depth) {
  const float aspect = (float)w / (float)h;
  const std::vector<SplatQuad> q = splat_quads(splats, n, vp, w, h);
#pragma omp parallel for schedule(dynamic, 8)
  for (long pl = 0; pl < (long)w * h; ++pl) {
    const uint32_t px = (uint32_t)(pl % w), py = (uint32_t)(pl / w);
    V2 p = pixel_to_p(px, py, w, h, aspect);
    float T = 1.0f, C[3] = {0, 0, 0}, D = 0.0f;
    for (uint32_t i = 0; i < n; ++i) {
      const SplatQuad& o = q[i];
      if (!o.ok || !in_quad(p, o.x0, o.x1, o.y0, o.y1)) continue;
      const float* s = splats + 16 * (size_t)i;
      const float dx = p.x - o.cx, dy = p.y - o.cy;
      const float r2 = o.A * dx * dx + 2.0f * o.B * dx * dy + o.C * dy * dy;
      const float r = std::sqrt(std::fmax(r2, 0.0001f));
      const float pw = -s[14] * std::pow(r, s[13]);
      float a = pw > -15.0f ? std::exp(pw) * s[7] : 0.0f;
      a = clampf(a, 0.0f, 0.999f);
      if (a < 0.001f) continue;
      for (int c = 0; c < 3; ++c) C[c] += T * a * s[4 + c];
      D += T * a * o.depth;
      T *= (1.0f - a);
    }
    float* oc = out_rgba + 4 * (size_t)pl;
    float* od = out_depth + 4 * (size_t)pl;
    for (int c = 0; c < 3; ++c) oc[c] = C[c] + T * 0.05f;
    oc[3] = 1.0f;
    od[0] = od[1] = od[2] = D + T * 1.0f;
    od[3] = 1.0f;
  }
  return 0;
}

// The same pass as the render pipeline runs it: instance ii draws splat
// n - 1 - ii (splat_forward.wgsl:44), and each fragment that survives the
// discard (alpha >= 0.001, :143-145) is blended over the attachment's current
// value with the pipeline's blend state (GpuSplatForwardPipelineManager.ts:64-77):
// rgb = src.rgb * a + dst.rgb * (1 - a), alpha = a + dst.a * (1 - a); colour
// src = (splat rgb, a), depth src = (enc, enc, enc, a) (:150-153).  rgba and
// depth hold the attachments' starting values (the clear colours, or the
// loaded contents) and receive the result; depth may be null.
int orc_splat_render_blend(const float* splats, uint32_t n, const float* vp, uint32_t w, uint32_t h, float* rgba,
                           float* depth) {
  const float aspect = (float)w / (float)h;
  const std::vector<SplatQuad> q = splat_quads(splats, n, vp, w, h);
#pragma omp parallel for schedule(dynamic, 8)
  for (long pl = 0; pl < (long)w * h; ++pl) {
    const uint32_t px = (uint32_t)(pl % w), py = (uint32_t)(pl / w);
    const V2 p = pixel_to_p(px, py, w, h, aspect);
    float* c = rgba + 4 * (size_t)pl;
    float* d = depth ? depth + 4 * (size_t)pl : nullptr;
    for (uint32_t ii = 0; ii < n; ++ii) {
      const uint32_t i = n - 1 - ii;
      const SplatQuad& o = q[i];
      if (!o.ok || !in_quad(p, o.x0, o.x1, o.y0, o.y1)) continue;
      const float* s = splats + 16 * (size_t)i;
      const float dx = p.x - o.cx, dy = p.y - o.cy;
      const float r2 = o.A * dx * dx + 2.0f * o.B * dx * dy + o.C * dy * dy;
      const float r = std::sqrt(std::fmax(r2, 0.0001f));
      const float pw = -s[14] * std::pow(r, s[13]);
      float a = pw > -15.0f ? std::exp(pw) * s[7] : 0.0f;
      a = clampf(a, 0.0f, 0.999f);
      if (a < 0.001f) continue;
      for (int k = 0; k < 3; ++k) c[k] = s[4 + k] * a + c[k] * (1.0f - a);
      c[3] = a + c[3] * (1.0f - a);
      if (d) {
        for (int k = 0; k < 3; ++k) d[k] = o.depth * a + d[k] * (1.0f - a);
        d[3] = a + d[3] * (1.0f - a);
      }
    }
  }
  return 0;
}

// bezier_forward.wgsl:48-182 with GpuBezierForwardPipelineManager.dispatch
// (GpuBezierForwardPipelineManager.ts:131-148), headless fp32, premultiplied
// one / one-minus-src-alpha blending over `bg_rgba` (H x W x 4; the cleared
// target is 0).  brush: optional single-channel texture bw x bh sampled
// bilinearly at level 0 with u repeat / v clamp; null = coverage only.
int orc_bezier_render(const float* bz, uint32_t n, const float* vp, uint32_t w, uint32_t h, const float* bg_rgba,
                      const float* brush, uint32_t bw, uint32_t bh, float* out_rgba) {
  const float aspect = (float)w / (float)h;
  struct Q { bool ok; float p[8]; float x0, x1, y0, y1; };
  std::vector<Q> q(n);
  for (uint32_t i = 0; i < n; ++i) {
    const float* b = bz + 20 * (size_t)i;
    Q& o = q[i];
    o.ok = false;
    PC c[4];
    for (int k = 0; k < 4; ++k) c[k] = project_center(vp, b + 4 * k, aspect);
    if (c[0].w <= 0.0f || c[1].w <= 0.0f || c[2].w <= 0.0f || c[3].w <= 0.0f) continue;
    for (int k = 0; k < 4; ++k) { o.p[2 * k] = c[k].x; o.p[2 * k + 1] = c[k].y; }
    const float width = std::fmax(b[3], 0.0001f), soft = std::fmax(b[7], 0.0001f), pad = width + soft;
    const float SB = 4.0f;
    o.x0 = std::fmax(std::fmin(std::fmin(c[0].x, c[1].x), std::fmin(c[2].x, c[3].x)) - pad, -SB);
    o.y0 = std::fmax(std::fmin(std::fmin(c[0].y, c[1].y), std::fmin(c[2].y, c[3].y)) - pad, -SB);
    o.x1 = std::fmin(std::fmax(std::fmax(c[0].x, c[1].x), std::fmax(c[2].x, c[3].x)) + pad, SB);
    o.y1 = std::fmin(std::fmax(std::fmax(c[0].y, c[1].y), std::fmax(c[2].y, c[3].y)) + pad, SB);
    o.ok = true;
  }
  auto brush_at = [&](float u, float v) -> float {
    if (!brush) return 1.0f;
    float x = u * (float)bw - 0.5f, y = v * (float)bh - 0.5f;
    float fx = std::floor(x), fy = std::floor(y);
    float ax = x - fx, ay = y - fy;
    auto at = [&](int ix, int iy) {
      ix = ((ix % (int)bw) + (int)bw) % (int)bw;
      iy = std::min(std::max(iy, 0), (int)bh - 1);
      return brush[(size_t)iy * bw + ix];
    };
    int ix = (int)fx, iy = (int)fy;
    return (1 - ay) * ((1 - ax) * at(ix, iy) + ax * at(ix + 1, iy)) + ay * ((1 - ax) * at(ix, iy + 1) + ax * at(ix + 1, iy + 1));
  };
#pragma omp parallel for schedule(dynamic, 8)
  for (long pl = 0; pl < (long)w * h; ++pl) {
    const uint32_t px = (uint32_t)(pl % w), py = (uint32_t)(pl / w);
    V2 p = pixel_to_p(px, py, w, h, aspect);
    float T = 1.0f, C[4] = {0, 0, 0, 0};
    for (uint32_t i = 0; i < n; ++i) {
      const Q& o = q[i];
      if (!o.ok || !in_quad(p, o.x0, o.x1, o.y0, o.y1)) continue;
      const float* b = bz + 20 * (size_t)i;
      V2 p0{o.p[0], o.p[1]}, p1{o.p[2], o.p[3]}, p2{o.p[4], o.p[5]}, p3{o.p[6], o.p[7]};
      float min_d = 1e9f, min_u = 0.0f, cross = 0.0f;
      uint32_t min_k = 1;
      V2 prev = p0;
      for (uint32_t s = 1; s <= N_SEG; ++s) {
        V2 cur = bezier_at(p0, p1, p2, p3, (float)s / (float)N_SEG);
        V2 seg{cur.x - prev.x, cur.y - prev.y};
        float len2 = std::fmax(seg.x * seg.x + seg.y * seg.y, 1e-8f);
        float u = clampf(((p.x - prev.x) * seg.x + (p.y - prev.y) * seg.y) / len2, 0.0f, 1.0f);
        V2 pr{prev.x + u * seg.x, prev.y + u * seg.y};
        V2 df{p.x - pr.x, p.y - pr.y};
        float d = std::sqrt(df.x * df.x + df.y * df.y);
        if (d < min_d) {
          min_d = d; min_k = s; min_u = u;
          float sl = std::sqrt(len2);
          cross = df.x * (-(seg.y / sl)) + df.y * (seg.x / sl);
        }
        prev = cur;
      }
      float t = ((float)(min_k - 1) + min_u) / (float)N_SEG;
      float dt = t - 0.5f;
      float pressure = 1.0f - 4.0f * dt * dt;
      float width = std::fmax(b[3], 0.0001f), soft = std::fmax(b[7], 0.0001f);
      float lw = width * pressure, ls = soft * pressure, lo = b[19] * pressure;
      float a_geom = 1.0f - smoothstepf(lw - ls, lw + ls, min_d);
      float bv = clampf(cross / std::fmax(lw + ls, 1e-6f) * 0.5f + 0.5f, 0.0f, 1.0f);
      float a = clampf(a_geom * brush_at(t, bv) * lo, 0.0f, 0.999f);
      if (a < 0.001f) continue;
      for (int c = 0; c < 3; ++c) C[c] += T * b[16 + c] * a;
      C[3] += T * a;
      T *= (1.0f - a);
    }
    const float* bgp = bg_rgba + 4 * (size_t)pl;
    float* o = out_rgba + 4 * (size_t)pl;
    for (int c = 0; c < 4; ++c) o[c] = C[c] + T * bgp[c];
  }
  return 0;
}

}  // extern "C"
