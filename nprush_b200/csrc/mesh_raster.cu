// mesh_raster.cu — the reference viewer's mesh render pass as CUDA kernels:
// the environment background (envmap.wgsl:36-52) and an indexed triangle mesh
// through mesh.wgsl's standard pipeline (vert :39-50, frag :52-70), with the
// fixed-function state of GpuMeshRenderPipelineManager.ts:84-112 (triangle
// list, back faces culled, counter-clockwise front, depth "less") and the
// clears of GpuRunner.svelte.ts:611-634.  It writes the two colour targets of
// that pass: the shaded colour and the reciprocal-encoded view depth
// 1 - 0.1 / max(w, 0.1) (mesh.wgsl:37-47) that the target preprocessing reads.
//
// Pipeline (one render):
//   k_mesh_vertex   one thread per vertex: clip position and varyings (80 B)
//   k_mesh_setup    one thread per triangle: clip against 0 <= z <= w and a
//                   guard band |x|, |y| <= 64 w (Sutherland-Hodgman, fan of
//                   <= 7 sub-triangles), project, snap to 1/256 pixel, cull
//                   back faces; rasterise small unclipped triangles (box of
//                   <= 32 pixels) itself, count 1024-pixel chunks of the
//                   other sub-triangles' pixel boxes
//   exclusive scan  chunk offsets
//   k_mesh_raster   one warp per chunk (32 pixels per lane): exact 64-bit
//                   edge functions at pixel centres (watertight, top-left
//                   rule), depth z/w, and a 64-bit atomicMin of (depth bits,
//                   sub-triangle id) per pixel — the smallest depth wins and,
//                   among equal depths, the earliest triangle, which is what
//                   "less" in draw order keeps
//   k_mesh_shade    one thread per pixel: perspective-correct varyings of the
//                   winner (recomputed from its triangle), the fragment stage,
//                   or the background
// Compiled with --fmad=false; every float operation is rounded separately in
// the order of the CPU restatement, so both draw the same pixels.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "context.h"

namespace nps {
namespace mr {

constexpr float kDepthNear = 0.1f;        // mesh.wgsl:37
constexpr float kPi = 3.14159265358979f;  // envmap.wgsl:33
constexpr uint32_t kChunk = 1024;         // pixels per raster task
constexpr int kRasterThreads = 256;
constexpr int kSubpix = 256;              // sub-pixel steps per pixel
constexpr float kGuard = 64.0f;           // guard band in units of w
constexpr int kPlanes = 6;
constexpr int kMaxSubs = 7;               // <= 9 vertices after 6 planes: <= 7 fan triangles
constexpr int kMaxPoly = 10;

struct Uniforms {  // the shared uniform buffer (GpuUniformsBufferManager.ts: 208 bytes)
  float vp[16], view[16], shading_mode, pad[3], inv_vp[16];
};

struct Tex {
  const float4* p;
  int w, h;
};

__device__ __forceinline__ int wrap(int i, int n, bool repeat) {
  if (repeat) {
    const int r = i % n;
    return r < 0 ? r + n : r;
  }
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}
// level-0 bilinear sample with exact float weights (WebGPU linear filtering)
__device__ __forceinline__ float3 sample(const Tex& t, float u, float v, bool rep_u, bool rep_v) {
  if (rep_u) u = u - floorf(u);
  if (rep_v) v = v - floorf(v);
  // bounded texel coordinates: the same taps for every finite input (beyond
  // the edges both taps clamp to the edge texel), defined for NaN
  const float fx = fminf(fmaxf(u * (float)t.w - 0.5f, -2.0f), (float)(t.w + 1));
  const float fy = fminf(fmaxf(v * (float)t.h - 0.5f, -2.0f), (float)(t.h + 1));
  const float x0f = floorf(fx), y0f = floorf(fy);
  const float ax = fx - x0f, ay = fy - y0f;
  const int xa = wrap((int)x0f, t.w, rep_u), xb = wrap((int)x0f + 1, t.w, rep_u);
  const int ya = wrap((int)y0f, t.h, rep_v), yb = wrap((int)y0f + 1, t.h, rep_v);
  const float4 a = __ldg(t.p + (size_t)ya * t.w + xa), b = __ldg(t.p + (size_t)ya * t.w + xb);
  const float4 c = __ldg(t.p + (size_t)yb * t.w + xa), d = __ldg(t.p + (size_t)yb * t.w + xb);
  const float tr = a.x + (b.x - a.x) * ax, br = c.x + (d.x - c.x) * ax;
  const float tg = a.y + (b.y - a.y) * ax, bg = c.y + (d.y - c.y) * ax;
  const float tb = a.z + (b.z - a.z) * ax, bb = c.z + (d.z - c.z) * ax;
  return make_float3(tr + (br - tr) * ay, tg + (bg - tg) * ay, tb + (bb - tb) * ay);
}
__device__ __forceinline__ float3 normalize3(float x, float y, float z) {
  const float s = 1.0f / sqrtf(x * x + y * y + z * z);
  return make_float3(x * s, y * s, z * s);
}
__device__ __forceinline__ float reinhard(float c) { return c / (c + 1.0f); }
__device__ __forceinline__ float unorm8(float x) { return rintf(fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f) / 255.0f; }
// WGSL M * v, column-major: ((c0 v0 + c1 v1) + c2 v2) + c3 v3
__device__ __forceinline__ float mrow(const float* m, int r, float a, float b, float c, float d) {
  return m[r] * a + m[4 + r] * b + m[8 + r] * c + m[12 + r] * d;
}

// ---- vertex stage (mesh.wgsl:39-50) -> 5 float4:
// [pos] [normal, viewDepth] [viewNormal, 0] [color] [uv, 0, 0]
__global__ void k_mesh_vertex(const float* __restrict__ verts, uint32_t n, Uniforms u, float4* __restrict__ vout) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* v = verts + (size_t)i * 12;
  const float px = v[0], py = v[1], pz = v[2], nx = v[3], ny = v[4], nz = v[5];
  float pos[4], vn[3];
#pragma unroll
  for (int r = 0; r < 4; ++r) pos[r] = mrow(u.vp, r, px, py, pz, 1.0f);
#pragma unroll
  for (int r = 0; r < 3; ++r) vn[r] = mrow(u.view, r, nx, ny, nz, 0.0f);
  const float lin = fmaxf(pos[3], kDepthNear);
  const float vd = fminf(fmaxf(1.0f - kDepthNear / lin, 0.0f), 1.0f);
  float4* o = vout + (size_t)i * 5;
  o[0] = make_float4(pos[0], pos[1], pos[2], pos[3]);
  o[1] = make_float4(nx, ny, nz, vd);
  o[2] = make_float4(vn[0], vn[1], vn[2], 0.0f);
  o[3] = make_float4(v[6], v[7], v[8], v[9]);
  o[4] = make_float4(v[10], v[11], 0.0f, 0.0f);
}

// ---- clipping against z >= 0, w - z >= 0 and the guard band
struct CV {
  float4 p;    // clip position
  float c[3];  // weights of the triangle's original vertices
};
__device__ __forceinline__ float plane_dist(const float4& p, int plane) {
  switch (plane) {
    case 0: return p.z;
    case 1: return p.w - p.z;
    case 2: return kGuard * p.w - p.x;
    case 3: return kGuard * p.w + p.x;
    case 4: return kGuard * p.w - p.y;
    default: return kGuard * p.w + p.y;
  }
}

// clipped polygon of triangle t (0 when nothing is left)
__device__ __forceinline__ int clip_triangle(const float4* __restrict__ vout, const uint32_t* __restrict__ idx,
                                             uint32_t t, CV poly[kMaxPoly]) {
  int n = 3;
  bool inside = true;
  for (int j = 0; j < 3; ++j) {
    poly[j].p = vout[(size_t)idx[3 * (size_t)t + j] * 5];
    poly[j].c[0] = poly[j].c[1] = poly[j].c[2] = 0.0f;
    poly[j].c[j] = 1.0f;
    for (int k = 0; k < kPlanes; ++k) inside = inside && plane_dist(poly[j].p, k) >= 0.0f;
  }
  if (inside) return 3;
  CV tmp[kMaxPoly];
  for (int plane = 0; plane < kPlanes; ++plane) {
    int m = 0;
    for (int i = 0; i < n; ++i) {
      const CV& a = poly[i];
      const CV& b = poly[(i + 1) % n];
      const float da = plane_dist(a.p, plane), db = plane_dist(b.p, plane);
      if (da >= 0.0f) tmp[m++] = a;
      if ((da >= 0.0f) != (db >= 0.0f)) {
        const float s = da / (da - db);
        CV q;
        q.p = make_float4(a.p.x + s * (b.p.x - a.p.x), a.p.y + s * (b.p.y - a.p.y), a.p.z + s * (b.p.z - a.p.z),
                          a.p.w + s * (b.p.w - a.p.w));
        for (int j = 0; j < 3; ++j) q.c[j] = a.c[j] + s * (b.c[j] - a.c[j]);
        tmp[m++] = q;
      }
    }
    n = m;
    for (int i = 0; i < n; ++i) poly[i] = tmp[i];
    if (n < 3) return 0;
  }
  return n;
}

struct Sub {
  float z[3], iw[3];
  long long X[3], Y[3];  // snapped to 1/256 pixel
  long long area;
  int bx0, bx1, by0, by1;
  float c[3][3];
};

__device__ __forceinline__ long long floor_div(long long a, long long b) {  // b > 0
  return a >= 0 ? a / b : -((-a + b - 1) / b);
}

// sub-triangle k of the polygon (a fan from its first vertex); false if culled
__device__ __forceinline__ bool setup_sub(const CV* poly, int n, int k, int W, int H, Sub& s) {
  if (n < k + 3) return false;
  const int id[3] = {0, k + 1, k + 2};
  for (int j = 0; j < 3; ++j) {
    const float4 p = poly[id[j]].p;
    if (!(p.w > 0.0f)) return false;
    const float nx = p.x / p.w, ny = p.y / p.w, nz = p.z / p.w;
    const float fx = (nx + 1.0f) * 0.5f * (float)W;
    const float fy = (1.0f - ny) * 0.5f * (float)H;
    s.z[j] = nz;
    s.iw[j] = 1.0f / p.w;
    if (!isfinite(fx) || !isfinite(fy) || !isfinite(nz) || !isfinite(s.iw[j])) return false;
    s.X[j] = (long long)rintf(fx * (float)kSubpix);
    s.Y[j] = (long long)rintf(fy * (float)kSubpix);
    for (int q = 0; q < 3; ++q) s.c[j][q] = poly[id[j]].c[q];
  }
  const long long A = (s.X[1] - s.X[0]) * (s.Y[2] - s.Y[0]) - (s.X[2] - s.X[0]) * (s.Y[1] - s.Y[0]);
  if (A >= 0) return false;  // counter-clockwise on screen is the front face
  s.area = -A;
  const long long half = kSubpix / 2;
  const long long minx = min(min(s.X[0], s.X[1]), s.X[2]), maxx = max(max(s.X[0], s.X[1]), s.X[2]);
  const long long miny = min(min(s.Y[0], s.Y[1]), s.Y[2]), maxy = max(max(s.Y[0], s.Y[1]), s.Y[2]);
  s.bx0 = (int)max(0ll, -floor_div(-(minx - half), kSubpix));
  s.bx1 = (int)min((long long)W - 1, floor_div(maxx - half, kSubpix));
  s.by0 = (int)max(0ll, -floor_div(-(miny - half), kSubpix));
  s.by1 = (int)min((long long)H - 1, floor_div(maxy - half, kSubpix));
  return s.bx0 <= s.bx1 && s.by0 <= s.by1;
}

__device__ __forceinline__ bool top_left(long long ax, long long ay, long long bx, long long by) {
  return by > ay || (by == ay && bx < ax);
}
// exact coverage of the pixel centre, screen barycentrics and clamped depth
__device__ __forceinline__ bool cover(const Sub& s, int px, int py, float l[3], float& z) {
  const long long cx = (long long)px * kSubpix + kSubpix / 2, cy = (long long)py * kSubpix + kSubpix / 2;
  const long long e0 = (s.Y[2] - s.Y[1]) * (cx - s.X[1]) - (s.X[2] - s.X[1]) * (cy - s.Y[1]);
  const long long e1 = (s.Y[0] - s.Y[2]) * (cx - s.X[2]) - (s.X[0] - s.X[2]) * (cy - s.Y[2]);
  const long long e2 = (s.Y[1] - s.Y[0]) * (cx - s.X[0]) - (s.X[1] - s.X[0]) * (cy - s.Y[0]);
  const bool in = (e0 > 0 || (e0 == 0 && top_left(s.X[1], s.Y[1], s.X[2], s.Y[2]))) &&
                  (e1 > 0 || (e1 == 0 && top_left(s.X[2], s.Y[2], s.X[0], s.Y[0]))) &&
                  (e2 > 0 || (e2 == 0 && top_left(s.X[0], s.Y[0], s.X[1], s.Y[1])));
  const float area = (float)s.area;
  l[0] = (float)e0 / area;
  l[1] = (float)e1 / area;
  l[2] = (float)e2 / area;
  z = fminf(fmaxf(l[0] * s.z[0] + l[1] * s.z[1] + l[2] * s.z[2], 0.0f), 1.0f);
  return in;
}

// depth test of one covered sample: "less" in draw order
__device__ __forceinline__ void depth_min(unsigned long long* zbuf, int W, int px, int py, float z, uint32_t sub) {
  const unsigned long long key = ((unsigned long long)__float_as_uint(z) << 32) | sub;
  atomicMin(zbuf + (size_t)py * W + px, key);
}

// Counts the 1024-pixel chunks of each sub-triangle for k_mesh_raster.  An
// unclipped triangle whose pixel box holds at most kSmallBox pixels (most
// triangles of a detailed mesh) is rasterised here by its own thread and
// gets no chunks: a warp task would spend more on finding and setting up the
// triangle than on its few pixels.
constexpr uint32_t kSmallBox = 32;
__global__ void k_mesh_setup(const float4* __restrict__ vout, const uint32_t* __restrict__ idx, uint32_t n_tris,
                             int W, int H, uint32_t* __restrict__ chunks, unsigned long long* __restrict__ zbuf) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tris) return;
  CV poly[kMaxPoly];
  const int n = clip_triangle(vout, idx, t, poly);
  for (int k = 0; k < kMaxSubs; ++k) {
    Sub s;
    uint32_t c = 0;
    if (setup_sub(poly, n, k, W, H, s)) {
      const uint32_t bw = (uint32_t)(s.bx1 - s.bx0 + 1), pixels = bw * (uint32_t)(s.by1 - s.by0 + 1);
      if (n == 3 && pixels <= kSmallBox) {
        const uint32_t sub = (uint32_t)kMaxSubs * t + k;
        for (uint32_t p = 0; p < pixels; ++p) {
          const int px = s.bx0 + (int)(p % bw), py = s.by0 + (int)(p / bw);
          float l[3], z;
          if (cover(s, px, py, l, z) && z < 1.0f) depth_min(zbuf, W, px, py, z, sub);
        }
      } else {
        c = (pixels + kChunk - 1) / kChunk;
      }
    }
    chunks[(size_t)kMaxSubs * t + k] = c;
  }
}

// last s with offsets[s] <= task (offsets ascending, offsets[0] = 0)
__device__ __forceinline__ uint32_t find_sub(const uint32_t* __restrict__ offsets, uint32_t n, uint32_t task) {
  uint32_t lo = 0, hi = n;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(offsets + mid) <= task) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kRasterThreads) k_mesh_raster(const float4* __restrict__ vout,
                                                                 const uint32_t* __restrict__ idx,
                                                                 const uint32_t* __restrict__ offsets,
                                                                 const uint32_t* __restrict__ total, uint32_t n_subs,
                                                                 int W, int H,
                                                                 unsigned long long* __restrict__ zbuf) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warps = gridDim.x * (kRasterThreads / 32);
  const uint32_t n_tasks = *total;
  for (uint32_t task = blockIdx.x * (kRasterThreads / 32) + (threadIdx.x >> 5); task < n_tasks; task += warps) {
    const uint32_t sub = find_sub(offsets, n_subs, task);
    const uint32_t chunk = task - __ldg(offsets + sub);
    CV poly[kMaxPoly];
    const int n = clip_triangle(vout, idx, sub / kMaxSubs, poly);
    Sub s;
    if (!setup_sub(poly, n, (int)(sub % kMaxSubs), W, H, s)) continue;  // cannot happen: it has chunks
    const uint32_t bw = (uint32_t)(s.bx1 - s.bx0 + 1), count = bw * (uint32_t)(s.by1 - s.by0 + 1);
    for (uint32_t i = 0; i < kChunk / 32u; ++i) {
      const uint32_t p = chunk * kChunk + i * 32u + lane;
      if (p >= count) break;
      const int px = s.bx0 + (int)(p % bw), py = s.by0 + (int)(p / bw);
      float l[3], z;
      if (cover(s, px, py, l, z) && z < 1.0f) depth_min(zbuf, W, px, py, z, sub);
    }
  }
}

__device__ __forceinline__ float3 cross3(const float3& a, const float3& b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// mesh.wgsl:87-121, the PBR stage of the ground (setPbrMesh): albedo and a
// tangent-space normal map sampled linearly with repeat, a TBN frame from the
// interpolated normal, the matcap lit by the perturbed view-space normal
__device__ __forceinline__ float3 frag_pbr(const Uniforms& u, const Tex& matcap, const Tex& albedo, const Tex& nmap,
                                           const float4& nrm, const float4& uv) {
  const float3 alb = sample(albedo, uv.x, uv.y, true, true);
  const float3 t3 = sample(nmap, uv.x, uv.y, true, true);
  const float tsx = t3.x * 2.0f - 1.0f, tsy = t3.y * 2.0f - 1.0f, tsz = t3.z * 2.0f - 1.0f;
  const float3 N = normalize3(nrm.x, nrm.y, nrm.z);
  float3 up = make_float3(0.0f, 0.0f, 1.0f);
  if (fabsf(N.x * up.x + N.y * up.y + N.z * up.z) > 0.99f) up = make_float3(1.0f, 0.0f, 0.0f);
  const float3 tc = cross3(up, N);
  const float3 T = normalize3(tc.x, tc.y, tc.z);
  const float3 B = cross3(N, T);
  const float3 wn = normalize3(T.x * tsx + B.x * tsy + N.x * tsz, T.y * tsx + B.y * tsy + N.y * tsz,
                               T.z * tsx + B.z * tsy + N.z * tsz);
  const float3 vn = normalize3(mrow(u.view, 0, wn.x, wn.y, wn.z, 0.0f), mrow(u.view, 1, wn.x, wn.y, wn.z, 0.0f),
                               mrow(u.view, 2, wn.x, wn.y, wn.z, 0.0f));
  if (u.shading_mode < 0.5f) return make_float3((wn.x + 1.0f) * 0.5f, (wn.y + 1.0f) * 0.5f, (wn.z + 1.0f) * 0.5f);
  const float mx = vn.x * 0.5f + 0.5f, my = vn.y * 0.5f + 0.5f;
  const float3 mc = sample(matcap, mx, 1.0f - my, false, false);
  return make_float3(mc.x * alb.x, mc.y * alb.y, mc.z * alb.z);
}

__global__ void k_mesh_shade(const float4* __restrict__ vout, const uint32_t* __restrict__ idx,
                             const unsigned long long* __restrict__ zbuf, int W, int H, Uniforms u, Tex matcap,
                             Tex env, Tex albedo, Tex nmap, uint32_t first_pbr, int draw_env, int quantize,
                             float4* __restrict__ color, float4* __restrict__ depth) {
  const int x = blockIdx.x * 16 + threadIdx.x, y = blockIdx.y * 16 + threadIdx.y;
  if (x >= W || y >= H) return;
  const size_t pix = (size_t)y * W + x;
  const unsigned long long key = zbuf[pix];
  float4 col, dep = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
  if (key == ~0ull) {
    if (draw_env) {  // envmap.wgsl:36-52 at the pixel centre's ndc
      const float ndx = ((float)x + 0.5f) / (float)W * 2.0f - 1.0f, ndy = 1.0f - ((float)y + 0.5f) / (float)H * 2.0f;
      float nh[4], fh[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        nh[r] = mrow(u.inv_vp, r, ndx, ndy, 0.0f, 1.0f);
        fh[r] = mrow(u.inv_vp, r, ndx, ndy, 1.0f, 1.0f);
      }
      const float3 d = normalize3(fh[0] / fh[3] - nh[0] / nh[3], fh[1] / fh[3] - nh[1] / nh[3],
                                  fh[2] / fh[3] - nh[2] / nh[3]);
      const float lon = atan2f(d.y, d.x), lat = asinf(fminf(fmaxf(d.z, -1.0f), 1.0f));
      const float uu = lon / (2.0f * kPi) + 0.5f, vv = 0.5f - lat / kPi;
      const float3 c = sample(env, uu, vv, true, false);
      col = make_float4(reinhard(c.x * 4.0f), reinhard(c.y * 4.0f), reinhard(c.z * 4.0f), 1.0f);
    } else {
      col = make_float4(0.05f, 0.05f, 0.05f, 1.0f);  // the pass's clear colour
    }
  } else {
    const uint32_t sub = (uint32_t)(key & 0xffffffffu), t = sub / kMaxSubs;
    CV poly[kMaxPoly];
    const int n = clip_triangle(vout, idx, t, poly);
    Sub s;
    setup_sub(poly, n, (int)(sub % kMaxSubs), W, H, s);
    float l[3], z;
    cover(s, x, y, l, z);
    const float q0 = l[0] * s.iw[0], q1 = l[1] * s.iw[1], q2 = l[2] * s.iw[2];
    const float qs = q0 + q1 + q2;
    const float b0 = q0 / qs, b1 = q1 / qs, b2 = q2 / qs;
    float wt[3];
    for (int j = 0; j < 3; ++j) wt[j] = b0 * s.c[0][j] + b1 * s.c[1][j] + b2 * s.c[2][j];
    const float4* v0 = vout + (size_t)idx[3 * (size_t)t] * 5;
    const float4* v1 = vout + (size_t)idx[3 * (size_t)t + 1] * 5;
    const float4* v2 = vout + (size_t)idx[3 * (size_t)t + 2] * 5;
    auto lerp4 = [&](int f) {
      const float4 a = v0[f], b = v1[f], c = v2[f];
      return make_float4(wt[0] * a.x + wt[1] * b.x + wt[2] * c.x, wt[0] * a.y + wt[1] * b.y + wt[2] * c.y,
                         wt[0] * a.z + wt[1] * b.z + wt[2] * c.z, wt[0] * a.w + wt[1] * b.w + wt[2] * c.w);
    };
    const float4 nrm_vd = lerp4(1), vnrm = lerp4(2), vcol = lerp4(3);
    float3 fin;
    if (t >= first_pbr) {
      fin = frag_pbr(u, matcap, albedo, nmap, nrm_vd, lerp4(4));
    } else if (u.shading_mode < 0.5f) {  // mesh.wgsl:52-70
      const float3 nn = normalize3(nrm_vd.x, nrm_vd.y, nrm_vd.z);
      fin = make_float3((nn.x + 1.0f) * 0.5f, (nn.y + 1.0f) * 0.5f, (nn.z + 1.0f) * 0.5f);
    } else {
      const float3 vn = normalize3(vnrm.x, vnrm.y, vnrm.z);
      const float uvx = vn.x * 0.5f + 0.5f, uvy = vn.y * 0.5f + 0.5f;
      const float3 mc = sample(matcap, uvx, 1.0f - uvy, false, false);
      fin = make_float3(mc.x * vcol.x, mc.y * vcol.y, mc.z * vcol.z);
    }
    col = make_float4(reinhard(fin.x * 4.0f), reinhard(fin.y * 4.0f), reinhard(fin.z * 4.0f), 1.0f);
    dep = make_float4(nrm_vd.w, nrm_vd.w, nrm_vd.w, 1.0f);
  }
  if (quantize) {
    col = make_float4(unorm8(col.x), unorm8(col.y), unorm8(col.z), 1.0f);
    dep = make_float4(unorm8(dep.x), unorm8(dep.y), unorm8(dep.z), 1.0f);
  }
  color[pix] = col;
  depth[pix] = dep;
}

}  // namespace mr
}  // namespace nps

using namespace nps;

struct nps_mesh {
  nps_ctx* ctx = nullptr;
  uint32_t n_verts = 0, n_tris = 0;
  DevBuf verts, idx, vout, chunks, offsets, total, zbuf, matcap, env, albedo, nmap;
  SortWork work;
  int matcap_w = 1, matcap_h = 1, env_w = 1, env_h = 1, albedo_w = 1, albedo_h = 1, nmap_w = 1, nmap_h = 1;
  uint32_t first_pbr = 0xffffffffu;  // triangles from here on use the PBR stage
  ~nps_mesh() {
    for (DevBuf* b : {&verts, &idx, &vout, &chunks, &offsets, &total, &zbuf, &matcap, &env, &albedo, &nmap, &work.hist,
                      &work.partial, &work.lookback, &work.keys_alt, &work.vals_alt})
      b->release();
  }
};

namespace {
int upload_tex(nps_mesh* o, DevBuf& buf, const float* rgba, uint32_t w, uint32_t h, int& ow, int& oh) {
  if (!rgba || w == 0 || h == 0 || w > 65536 || h > 65536) {
    set_error("nps_mesh texture: bad arguments");
    return NPS_ERR_INVALID;
  }
  NPS_TRY(bind_device(o->ctx));
  cudaStream_t s = o->ctx->stream;
  NPS_CUDA(cudaStreamSynchronize(s));  // a render in flight may read the old image
  NPS_TRY(buf.ensure((size_t)w * h * 16));
  NPS_CUDA(cudaMemcpyAsync(buf.p, rgba, (size_t)w * h * 16, cudaMemcpyDefault, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  ow = (int)w;
  oh = (int)h;
  return NPS_OK;
}
}  // namespace

extern "C" {

int nps_mesh_create(nps_ctx* ctx, const float* vertices, uint32_t n_vertices, const uint32_t* indices,
                    uint32_t n_tris, nps_mesh** out) {
  if (!ctx || !out || (n_vertices && !vertices) || (n_tris && !indices) || n_tris > (1u << 25) ||
      n_vertices > (1u << 27)) {
    set_error("nps_mesh_create: bad arguments");
    return NPS_ERR_INVALID;
  }
  *out = nullptr;
  for (size_t i = 0; i < (size_t)n_tris * 3; ++i)
    if (indices[i] >= n_vertices) {
      set_error("nps_mesh_create: index %u of triangle %zu is not below the vertex count %u", indices[i], i / 3,
                n_vertices);
      return NPS_ERR_INVALID;
    }
  NPS_TRY(bind_device(ctx));
  nps_mesh* o = new nps_mesh();
  o->ctx = ctx;
  o->n_verts = n_vertices;
  o->n_tris = n_tris;
  const float white[4] = {1.0f, 1.0f, 1.0f, 1.0f};
  int rc = NPS_OK;
  if ((rc = o->verts.ensure((size_t)n_vertices * 48 + 16)) || (rc = o->idx.ensure((size_t)n_tris * 12 + 16)) ||
      (rc = o->albedo.ensure(16)) || (rc = o->nmap.ensure(16)) ||
      (rc = o->vout.ensure((size_t)n_vertices * 80 + 16)) ||
      (rc = o->chunks.ensure((size_t)n_tris * 4 * mr::kMaxSubs + 16)) ||
      (rc = o->offsets.ensure((size_t)n_tris * 4 * mr::kMaxSubs + 16)) || (rc = o->total.ensure(16)) ||
      (rc = o->matcap.ensure(16)) || (rc = o->env.ensure(16))) {
    delete o;
    return rc;
  }
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaSuccess;
  if (n_vertices) e = cudaMemcpyAsync(o->verts.p, vertices, (size_t)n_vertices * 48, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && n_tris)
    e = cudaMemcpyAsync(o->idx.p, indices, (size_t)n_tris * 12, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(o->matcap.p, white, 16, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(o->env.p, white, 16, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(o->albedo.p, white, 16, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(o->nmap.p, white, 16, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_error("nps_mesh_create: upload failed: %s", cudaGetErrorString(e));
    delete o;
    return NPS_ERR_CUDA;
  }
  *out = o;
  return NPS_OK;
}

int nps_mesh_destroy(nps_mesh* o) {
  if (!o) return NPS_OK;
  cudaSetDevice(o->ctx->device);
  cudaStreamSynchronize(o->ctx->stream);
  delete o;
  return NPS_OK;
}

int nps_mesh_set_matcap(nps_mesh* o, const float* rgba, uint32_t w, uint32_t h) {
  if (!o) {
    set_error("nps_mesh_set_matcap: null handle");
    return NPS_ERR_INVALID;
  }
  return upload_tex(o, o->matcap, rgba, w, h, o->matcap_w, o->matcap_h);
}

int nps_mesh_set_env(nps_mesh* o, const float* rgba, uint32_t w, uint32_t h) {
  if (!o) {
    set_error("nps_mesh_set_env: null handle");
    return NPS_ERR_INVALID;
  }
  return upload_tex(o, o->env, rgba, w, h, o->env_w, o->env_h);
}

int nps_mesh_set_pbr(nps_mesh* o, uint32_t first_tri, const float* albedo_rgba, uint32_t aw, uint32_t ah, int srgb,
                     const float* normal_rgba, uint32_t nw, uint32_t nh) {
  if (!o || !albedo_rgba || !normal_rgba || aw == 0 || ah == 0 || nw == 0 || nh == 0 || aw > 65536 || ah > 65536 ||
      nw > 65536 || nh > 65536) {
    set_error("nps_mesh_set_pbr: bad arguments");
    return NPS_ERR_INVALID;
  }
  const float* alb = albedo_rgba;
  std::vector<float> lin;
  if (srgb) {  // an sRGB texture view: each texel decoded to linear before filtering
    lin.assign(albedo_rgba, albedo_rgba + (size_t)aw * ah * 4);
    for (size_t i = 0; i < lin.size(); ++i) {
      if (i % 4 == 3) continue;  // alpha is not encoded
      const float c = lin[i];
      lin[i] = c > 0.04045f ? std::pow((c + 0.055f) / 1.055f, 2.4f) : c / 12.92f;
    }
    alb = lin.data();
  }
  NPS_TRY(upload_tex(o, o->albedo, alb, aw, ah, o->albedo_w, o->albedo_h));
  NPS_TRY(upload_tex(o, o->nmap, normal_rgba, nw, nh, o->nmap_w, o->nmap_h));
  o->first_pbr = first_tri;
  return NPS_OK;
}

int nps_mesh_render(nps_mesh* o, const float* uniforms52, float* color_rgba, float* depth_rgba, uint32_t w,
                    uint32_t h, int draw_env, int quantize) {
  if (!o || !uniforms52 || !color_rgba || !depth_rgba || w == 0 || h == 0 || w > 16384 || h > 16384 ||
      color_rgba == depth_rgba || (((uintptr_t)color_rgba | (uintptr_t)depth_rgba) & 15) != 0) {
    set_error("nps_mesh_render: bad arguments (distinct 16-byte aligned float4 images, at most 16384 x 16384)");
    return NPS_ERR_INVALID;
  }
  NPS_TRY(bind_device(o->ctx));
  cudaStream_t s = o->ctx->stream;
  mr::Uniforms u;
  std::memcpy(&u, uniforms52, sizeof u);
  const size_t npx = (size_t)w * h;
  NPS_TRY(o->zbuf.ensure(npx * 8));
  NPS_CUDA(cudaMemsetAsync(o->zbuf.p, 0xFF, npx * 8, s));
  const float4* vout = o->vout.as<float4>();
  if (o->n_verts)
    mr::k_mesh_vertex<<<div_up(o->n_verts, 256), 256, 0, s>>>(o->verts.as<float>(), o->n_verts, u,
                                                               o->vout.as<float4>());
  if (o->n_tris) {
    const uint32_t n_subs = mr::kMaxSubs * o->n_tris;
    mr::k_mesh_setup<<<div_up(o->n_tris, 128), 128, 0, s>>>(vout, o->idx.as<uint32_t>(), o->n_tris, (int)w, (int)h,
                                                            o->chunks.as<uint32_t>(),
                                                            o->zbuf.as<unsigned long long>());
    NPS_CHECK_LAUNCH();
    NPS_TRY(exclusive_scan_u32(o->chunks.as<uint32_t>(), o->offsets.as<uint32_t>(), n_subs, o->total.as<uint32_t>(),
                               o->work, s));
    const int sms = o->ctx->sm_count > 0 ? o->ctx->sm_count : kNumSMs;
    mr::k_mesh_raster<<<sms * 8, mr::kRasterThreads, 0, s>>>(vout, o->idx.as<uint32_t>(), o->offsets.as<uint32_t>(),
                                                              o->total.as<uint32_t>(), n_subs, (int)w, (int)h,
                                                              o->zbuf.as<unsigned long long>());
    NPS_CHECK_LAUNCH();
  }
  const mr::Tex mt{o->matcap.as<float4>(), o->matcap_w, o->matcap_h}, et{o->env.as<float4>(), o->env_w, o->env_h};
  const mr::Tex at{o->albedo.as<float4>(), o->albedo_w, o->albedo_h}, nt{o->nmap.as<float4>(), o->nmap_w, o->nmap_h};
  const dim3 grid(div_up(w, 16), div_up(h, 16));
  mr::k_mesh_shade<<<grid, dim3(16, 16), 0, s>>>(vout, o->idx.as<uint32_t>(), o->zbuf.as<unsigned long long>(),
                                                 (int)w, (int)h, u, mt, et, at, nt, o->first_pbr, draw_env, quantize,
                                                 (float4*)color_rgba, (float4*)depth_rgba);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

}  // extern "C"
