// path_trace.cu — progressive path tracer used as a target generator: the SAH
// BVH built on the host (src/lib/gpu/bvh.ts:105-223) and the per-pixel
// diffuse / mirror path tracer over it (path_trace.wgsl:1-268) with its
// Reinhard resolve (path_trace_resolve.wgsl:20-30), as driven by
// GpuPathTracePipelineManager.ts:103-247.
//
// Layout on the device:
//   nodes    2 x float4 per node, the reference's 32-byte node
//            [min.xyz, data0 | max.xyz, data1] (data bits stored as floats)
//   tri_pos  3 x float4 per triangle in BVH order: the three corner positions
//            (v0.xyz v1.x | v1.yz v2.xy | v2.z) gathered so a leaf reads 48
//            contiguous bytes per triangle instead of three 48-byte vertices
//   tri_idx  3 x u32 per triangle in BVH order (the reference's bvh_tris)
//   verts    12 floats per vertex [pos, normal, rgba, uv] (shading at the hit)
//   env      H x W float4 environment image (equirectangular, z up)
// One thread per pixel, 128-thread blocks of four 8 x 4 warp tiles; the
// traversal stack (64 entries, the reference's size and overflow rule) lives
// in local memory.  A launch can run several frames: each frame's sample is
// computed exactly as one dispatch of the reference computes it and added to
// the pixel's running sums in frame order, so F frames in one launch equal F
// dispatches.  The shading of the closest hit (normal, colour) is computed
// once after traversal from the winning triangle's barycentrics, which gives
// the values the reference computes at every closer hit.
//
// Compiled with --fmad=false: every fp32 operation is rounded separately, in
// the reference's order, so the path up to the transcendental functions
// (atan2, asin, sin, cos) reproduces the WGSL arithmetic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "common.cuh"
#include "context.h"

namespace nps {
namespace pt {

constexpr uint32_t kLeafFlag = 0x80000000u;  // bvh.ts:15
constexpr int kMaxLeafTris = 4;               // bvh.ts:16
constexpr int kSahBins = 8;                   // bvh.ts:17
constexpr uint32_t kMaxStack = 64;            // path_trace.wgsl:16
constexpr int kBounces = 8;                   // path_trace.wgsl:243
constexpr float kPi = 3.14159265358979f;      // path_trace.wgsl:198

// ------------------------------------------------------------------ host BVH
// bvh.ts builds in JavaScript numbers (IEEE doubles) and writes the node
// bounds with setFloat32; this builder keeps every quantity in double and
// rounds only when writing a node, so its nodes are the reference's bit for
// bit.  The recursion is replaced by an explicit stack that visits nodes in
// the same pre-order (node, left subtree, right subtree), and partitions are
// stable, as the reference's array pushes are.
struct Box {
  double mn[3], mx[3];
};
static Box empty_box() {
  const double inf = std::numeric_limits<double>::infinity();
  return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
}
static void unite(Box& a, const Box& b) {
  for (int i = 0; i < 3; ++i) {
    a.mn[i] = std::min(a.mn[i], b.mn[i]);
    a.mx[i] = std::max(a.mx[i], b.mx[i]);
  }
}
static double surface_area(const Box& a) {  // bvh.ts:45-50
  const double dx = a.mx[0] - a.mn[0], dy = a.mx[1] - a.mn[1], dz = a.mx[2] - a.mn[2];
  return 2 * (dx * dy + dy * dz + dz * dx);
}
struct BuildTri {
  uint32_t i0, i1, i2;
  Box box;
  double c[3];
};

struct Bvh {
  std::vector<float> nodes;    // 8 per node (data words hold u32 bits)
  std::vector<uint32_t> tris;  // 3 per triangle, BVH order
};

static void put_bounds(Bvh& b, uint32_t idx, const Box& box) {
  float* n = b.nodes.data() + (size_t)idx * 8;
  for (int i = 0; i < 3; ++i) {
    n[i] = (float)box.mn[i];
    n[4 + i] = (float)box.mx[i];
  }
}
static void put_data(Bvh& b, uint32_t idx, uint32_t d0, uint32_t d1) {
  float* n = b.nodes.data() + (size_t)idx * 8;
  std::memcpy(n + 3, &d0, 4);
  std::memcpy(n + 7, &d1, 4);
}
static int bin_of(double c, double cmin, double cmax) {  // bvh.ts:147-148
  int b = (int)std::floor(((c - cmin) / (cmax - cmin)) * kSahBins);
  return std::min(b, kSahBins - 1);
}

static void build_bvh(const float* verts, const uint32_t* idx, uint32_t n_tris, Bvh& out) {
  std::vector<BuildTri> tris(n_tris);
  const double eps = 1e-4;                 // bvh.ts:66
  for (uint32_t t = 0; t < n_tris; ++t) {  // bvh.ts:208-216
    BuildTri& bt = tris[t];
    bt.i0 = idx[3 * (size_t)t];
    bt.i1 = idx[3 * (size_t)t + 1];
    bt.i2 = idx[3 * (size_t)t + 2];
    for (int k = 0; k < 3; ++k) {
      const double a = verts[(size_t)bt.i0 * 12 + k], b = verts[(size_t)bt.i1 * 12 + k],
                   c = verts[(size_t)bt.i2 * 12 + k];
      bt.box.mn[k] = std::min(std::min(a, b), c) - eps;
      bt.box.mx[k] = std::max(std::max(a, b), c) + eps;
      bt.c[k] = (bt.box.mn[k] + bt.box.mx[k]) * 0.5;
    }
  }
  out.nodes.clear();
  out.tris.clear();
  out.nodes.reserve((size_t)std::max<uint32_t>(1, 2 * n_tris) * 8);
  out.tris.reserve((size_t)n_tris * 3);
  std::vector<uint32_t> order(n_tris), scratch(n_tris);
  for (uint32_t i = 0; i < n_tris; ++i) order[i] = i;

  struct Job {
    uint32_t lo, hi;  // range of `order`
    int64_t parent;   // node index of the parent, -1 for the root
    bool right;       // which child of the parent this is
  };
  std::vector<Job> stack{{0u, n_tris, -1, false}};
  std::vector<uint32_t> left_of;  // per node: its left child (set when the left job runs)
  while (!stack.empty()) {
    const Job j = stack.back();
    stack.pop_back();
    Box bounds = empty_box(), cent = empty_box();
    for (uint32_t i = j.lo; i < j.hi; ++i) {
      const BuildTri& t = tris[order[i]];
      unite(bounds, t.box);
      const Box cb{{t.c[0], t.c[1], t.c[2]}, {t.c[0], t.c[1], t.c[2]}};
      unite(cent, cb);
    }
    const uint32_t node = (uint32_t)(out.nodes.size() / 8);
    out.nodes.resize(out.nodes.size() + 8, 0.0f);
    left_of.push_back(0);
    put_bounds(out, node, bounds);
    if (j.parent >= 0) {  // internal node data (left, right): the left child comes first
      if (!j.right) {
        left_of[(size_t)j.parent] = node;
      } else {
        put_data(out, (uint32_t)j.parent, left_of[(size_t)j.parent], node);
      }
    }
    const uint32_t n = j.hi - j.lo;
    if ((int)n <= kMaxLeafTris) {  // bvh.ts:130-135
      const uint32_t start = (uint32_t)(out.tris.size() / 3);
      for (uint32_t i = j.lo; i < j.hi; ++i) {
        const BuildTri& t = tris[order[i]];
        out.tris.push_back(t.i0);
        out.tris.push_back(t.i1);
        out.tris.push_back(t.i2);
      }
      put_data(out, node, start, (n | kLeafFlag));
      continue;
    }
    // SAH over 8 centroid bins per axis (bvh.ts:138-175)
    double best_cost = std::numeric_limits<double>::infinity();
    int best_axis = 0, best_split = 0;
    const double parent_sa = surface_area(bounds);
    for (int axis = 0; axis < 3; ++axis) {
      const double cmin = cent.mn[axis], cmax = cent.mx[axis];
      if (cmax - cmin < 1e-8) continue;
      Box bin_box[kSahBins];
      int bin_count[kSahBins] = {};
      for (int b = 0; b < kSahBins; ++b) bin_box[b] = empty_box();
      for (uint32_t i = j.lo; i < j.hi; ++i) {
        const BuildTri& t = tris[order[i]];
        const int b = bin_of(t.c[axis], cmin, cmax);
        unite(bin_box[b], t.box);
        bin_count[b]++;
      }
      Box left_box[kSahBins - 1];
      int left_count[kSahBins - 1];
      Box lb = empty_box();
      int lc = 0;
      for (int i = 0; i < kSahBins - 1; ++i) {
        unite(lb, bin_box[i]);
        lc += bin_count[i];
        left_box[i] = lb;
        left_count[i] = lc;
      }
      Box rb = empty_box();
      int rc = 0;
      for (int i = kSahBins - 2; i >= 0; --i) {
        unite(rb, bin_box[i + 1]);
        rc += bin_count[i + 1];
        // an empty side has infinite area; inf * 0 is NaN, which never wins
        const double cost = (surface_area(left_box[i]) * left_count[i] + surface_area(rb) * rc) / parent_sa;
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = axis;
          best_split = i;
        }
      }
    }
    const double cmin = cent.mn[best_axis], cmax = cent.mx[best_axis];
    uint32_t mid = j.lo + n / 2;  // median split of the current order (bvh.ts:180-183, 191-195)
    if (!(cmax - cmin < 1e-8 || best_cost >= (double)n)) {
      uint32_t nl = 0, nr = 0;
      for (uint32_t i = j.lo; i < j.hi; ++i) {
        const uint32_t ti = order[i];
        if (bin_of(tris[ti].c[best_axis], cmin, cmax) <= best_split) order[j.lo + nl++] = ti;
        else scratch[nr++] = ti;
      }
      // left stays in place, right follows it; when one side is empty the
      // order is unchanged and the median split stands
      std::copy(scratch.begin(), scratch.begin() + nr, order.begin() + j.lo + nl);
      if (nl != 0 && nr != 0) mid = j.lo + nl;
    }
    stack.push_back(Job{mid, j.hi, (int64_t)node, true});
    stack.push_back(Job{j.lo, mid, (int64_t)node, false});
  }
}

// ------------------------------------------------------------------ device
struct Scene {
  const float4* __restrict__ nodes;
  const float4* __restrict__ tri_pos;
  const uint32_t* __restrict__ tri_idx;
  const float* __restrict__ verts;
  const float4* __restrict__ env;
  int env_w, env_h;
  uint32_t n_nodes;
};

__device__ __forceinline__ uint32_t pcg(uint32_t v) {  // path_trace.wgsl:34-38
  const uint32_t s = v * 747796405u + 2891336453u;
  const uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}
__device__ __forceinline__ float2 rand2(uint32_t& seed) {  // path_trace.wgsl:39-43
  seed = pcg(seed);
  const uint32_t a = seed;
  seed = pcg(seed);
  const uint32_t b = seed;
  return make_float2((float)a / 4294967296.0f, (float)b / 4294967296.0f);
}

__device__ __forceinline__ float comp(const float3& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
__device__ __forceinline__ float dot3(const float3& a, const float3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 normalize3(const float3& a) {
  const float s = 1.0f / sqrtf(dot3(a, a));
  return make_float3(a.x * s, a.y * s, a.z * s);
}
__device__ __forceinline__ float3 cross3(const float3& a, const float3& b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// per-ray constants of the watertight test (path_trace.wgsl:63-82)
struct RayShear {
  int kx, ky, kz;
  float sx, sy, sz;
};
__device__ __forceinline__ RayShear shear_of(const float3& rd) {
  RayShear r;
  int kz = 0;
  const float ax = fabsf(rd.x), ay = fabsf(rd.y), az = fabsf(rd.z);
  if (ay > ax) kz = 1;
  if (az > fmaxf(ax, ay)) kz = 2;
  int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
  if (comp(rd, kz) < 0.0f) {
    const int tmp = kx;
    kx = ky;
    ky = tmp;
  }
  r.kx = kx;
  r.ky = ky;
  r.kz = kz;
  r.sz = 1.0f / comp(rd, kz);
  r.sx = comp(rd, kx) * r.sz;
  r.sy = comp(rd, ky) * r.sz;
  return r;
}

struct Hit {
  float t, u, v, w;
  uint32_t tri;  // BVH-order triangle index; ~0u = no hit
};

// path_trace.wgsl:60-131 without the shading (done once for the closest hit)
__device__ __forceinline__ void intersect(const float3& ro, const RayShear& s, const float3& p0, const float3& p1,
                                          const float3& p2, uint32_t tri, Hit& best) {
  const float3 A = make_float3(p0.x - ro.x, p0.y - ro.y, p0.z - ro.z);
  const float3 B = make_float3(p1.x - ro.x, p1.y - ro.y, p1.z - ro.z);
  const float3 C = make_float3(p2.x - ro.x, p2.y - ro.y, p2.z - ro.z);
  const float Akz = comp(A, s.kz), Bkz = comp(B, s.kz), Ckz = comp(C, s.kz);
  const float Ax = comp(A, s.kx) - s.sx * Akz, Ay = comp(A, s.ky) - s.sy * Akz;
  const float Bx = comp(B, s.kx) - s.sx * Bkz, By = comp(B, s.ky) - s.sy * Bkz;
  const float Cx = comp(C, s.kx) - s.sx * Ckz, Cy = comp(C, s.ky) - s.sy * Ckz;
  const float U = Cx * By - Cy * Bx;
  const float V = Ax * Cy - Ay * Cx;
  const float W = Bx * Ay - By * Ax;
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return;
  const float det = U + V + W;
  if (det == 0.0f) return;
  const float Az = s.sz * Akz, Bz = s.sz * Bkz, Cz = s.sz * Ckz;
  const float T = U * Az + V * Bz + W * Cz;
  const float inv_det = 1.0f / det;
  const float t = T * inv_det;
  if (t < 1e-4f || t >= best.t) return;
  best.t = t;
  best.u = U * inv_det;
  best.v = V * inv_det;
  best.w = W * inv_det;
  best.tri = tri;
}

// path_trace.wgsl:133-144
__device__ __forceinline__ bool aabb_hit(const float3& ro, const float3& inv_rd, const float4& lo, const float4& hi,
                                         float t_max) {
  const float t0x = (lo.x - ro.x) * inv_rd.x, t0y = (lo.y - ro.y) * inv_rd.y, t0z = (lo.z - ro.z) * inv_rd.z;
  const float t1x = (hi.x - ro.x) * inv_rd.x, t1y = (hi.y - ro.y) * inv_rd.y, t1z = (hi.z - ro.z) * inv_rd.z;
  const float tmin = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
  const float tmax = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
  return tmax >= 0.0f && tmax >= tmin && tmin < t_max;
}

// path_trace.wgsl:148-192: explicit-stack traversal, right child pushed first
__device__ __forceinline__ Hit scene_hit(const Scene& sc, const float3& ro, const float3& rd, uint32_t* overflow) {
  Hit best;
  best.t = 1e30f;
  best.tri = ~0u;
  best.u = best.v = best.w = 0.0f;
  const float3 inv_rd = make_float3(1.0f / rd.x, 1.0f / rd.y, 1.0f / rd.z);
  const RayShear sh = shear_of(rd);
  uint32_t stack[kMaxStack];
  uint32_t top = 0;
  stack[top++] = 0u;
  uint32_t visits = 0;  // a tree visits each node at most once per ray
  while (top > 0u) {
    if (++visits > sc.n_nodes) {
      atomicAdd(overflow, 1u);
      break;
    }
    const uint32_t node = stack[--top];
    const float4 lo = __ldg(sc.nodes + 2 * (size_t)node), hi = __ldg(sc.nodes + 2 * (size_t)node + 1);
    if (!aabb_hit(ro, inv_rd, lo, hi, best.t)) continue;
    const uint32_t d1 = __float_as_uint(hi.w);
    if (d1 & kLeafFlag) {
      const uint32_t first = __float_as_uint(lo.w), count = d1 & ~kLeafFlag;
      for (uint32_t k = 0; k < count; ++k) {
        const uint32_t tri = first + k;
        const float4 a = __ldg(sc.tri_pos + 3 * (size_t)tri), b = __ldg(sc.tri_pos + 3 * (size_t)tri + 1),
                     c = __ldg(sc.tri_pos + 3 * (size_t)tri + 2);
        intersect(ro, sh, make_float3(a.x, a.y, a.z), make_float3(a.w, b.x, b.y), make_float3(b.z, b.w, c.x), tri,
                  best);
      }
    } else {
      const uint32_t left = __float_as_uint(lo.w), right = d1;
      if (top + 1u < kMaxStack) stack[top++] = right;
      if (top < kMaxStack) stack[top++] = left;
    }
  }
  return best;
}

// shading of the closest hit (path_trace.wgsl:127-128)
__device__ __forceinline__ void shade(const Scene& sc, const Hit& h, float3& nrm, float4& col) {
  const uint32_t i0 = __ldg(sc.tri_idx + 3 * (size_t)h.tri), i1 = __ldg(sc.tri_idx + 3 * (size_t)h.tri + 1),
                 i2 = __ldg(sc.tri_idx + 3 * (size_t)h.tri + 2);
  const float* a = sc.verts + (size_t)i0 * 12;
  const float* b = sc.verts + (size_t)i1 * 12;
  const float* c = sc.verts + (size_t)i2 * 12;
  const float3 n = make_float3(h.u * __ldg(a + 3) + h.v * __ldg(b + 3) + h.w * __ldg(c + 3),
                               h.u * __ldg(a + 4) + h.v * __ldg(b + 4) + h.w * __ldg(c + 4),
                               h.u * __ldg(a + 5) + h.v * __ldg(b + 5) + h.w * __ldg(c + 5));
  nrm = normalize3(n);
  col = make_float4(h.u * __ldg(a + 6) + h.v * __ldg(b + 6) + h.w * __ldg(c + 6),
                    h.u * __ldg(a + 7) + h.v * __ldg(b + 7) + h.w * __ldg(c + 7),
                    h.u * __ldg(a + 8) + h.v * __ldg(b + 8) + h.w * __ldg(c + 8),
                    h.u * __ldg(a + 9) + h.v * __ldg(b + 9) + h.w * __ldg(c + 9));
}

// textureSampleLevel at level 0 with the path tracer's sampler
// (GpuPathTracePipelineManager.ts:204-208: linear, u repeat, v clamp-to-edge)
__device__ __forceinline__ int wrap_repeat(int i, int n) {
  const int r = i % n;
  return r < 0 ? r + n : r;
}
__device__ __forceinline__ int wrap_clamp(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }
__device__ __forceinline__ float3 sample_env(const Scene& sc, const float3& dir) {  // path_trace.wgsl:200-205
  const float u = atan2f(dir.y, dir.x) / (2.0f * kPi) + 0.5f;
  const float v = 0.5f - asinf(fminf(fmaxf(dir.z, -1.0f), 1.0f)) / kPi;
  const int w = sc.env_w, h = sc.env_h;
  const float fx = (u - floorf(u)) * (float)w - 0.5f, fy = v * (float)h - 0.5f;
  const float x0f = floorf(fx), y0f = floorf(fy);
  const float ax = fx - x0f, ay = fy - y0f;
  const int x0 = wrap_repeat((int)x0f, w), x1 = wrap_repeat((int)x0f + 1, w);
  const int y0 = wrap_clamp((int)y0f, h), y1 = wrap_clamp((int)y0f + 1, h);
  const float4 a = __ldg(sc.env + (size_t)y0 * w + x0), b = __ldg(sc.env + (size_t)y0 * w + x1);
  const float4 c = __ldg(sc.env + (size_t)y1 * w + x0), d = __ldg(sc.env + (size_t)y1 * w + x1);
  const float tr = a.x + (b.x - a.x) * ax, br = c.x + (d.x - c.x) * ax;
  const float tg = a.y + (b.y - a.y) * ax, bg = c.y + (d.y - c.y) * ax;
  const float tb = a.z + (b.z - a.z) * ax, bb = c.z + (d.z - c.z) * ax;
  return make_float3(tr + (br - tr) * ay, tg + (bg - tg) * ay, tb + (bb - tb) * ay);
}

// path_trace.wgsl:208-219
__device__ __forceinline__ float3 cosine_hemisphere(const float3& n, uint32_t& seed) {
  const float2 r = rand2(seed);
  const float phi = 2.0f * kPi * r.x;
  const float sr = sqrtf(r.y);
  const float x = cosf(phi) * sr, y = sinf(phi) * sr, z = sqrtf(fmaxf(0.0f, 1.0f - r.y));
  float3 up = make_float3(0.0f, 1.0f, 0.0f);
  if (fabsf(n.y) > 0.99f) up = make_float3(1.0f, 0.0f, 0.0f);
  const float3 t = normalize3(cross3(up, n));
  const float3 b = cross3(n, t);
  return normalize3(
      make_float3(t.x * x + b.x * y + n.x * z, t.y * x + b.y * y + n.y * z, t.z * x + b.z * y + n.z * z));
}

struct Camera {
  float m[16];  // inverse view-projection, column-major (WGSL mat4x4f)
};

// one sample of pixel (x, y) for `frame` (path_trace.wgsl:222-262)
__device__ __forceinline__ float3 trace_pixel(const Scene& sc, const Camera& cam, uint32_t x, uint32_t y, uint32_t w,
                                              uint32_t h, uint32_t frame, uint32_t* overflow) {
  const uint32_t pixel = y * w + x;
  uint32_t seed = pcg(pixel ^ (frame * 2654435761u));
  const float2 j = rand2(seed);
  const float jx = j.x - 0.5f, jy = j.y - 0.5f;
  const float ux = ((float)x + 0.5f + jx) / (float)w, uy = ((float)y + 0.5f + jy) / (float)h;
  const float nx = ux * 2.0f - 1.0f, ny = 1.0f - uy * 2.0f;
  const float* m = cam.m;
  float nh[4], fh[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    nh[r] = m[r] * nx + m[4 + r] * ny + m[8 + r] * 0.0f + m[12 + r] * 1.0f;
    fh[r] = m[r] * nx + m[4 + r] * ny + m[8 + r] * 1.0f + m[12 + r] * 1.0f;
  }
  const float3 ro = make_float3(nh[0] / nh[3], nh[1] / nh[3], nh[2] / nh[3]);
  const float3 rd = normalize3(make_float3(fh[0] / fh[3] - ro.x, fh[1] / fh[3] - ro.y, fh[2] / fh[3] - ro.z));
  float3 radiance = make_float3(0.0f, 0.0f, 0.0f), thr = make_float3(1.0f, 1.0f, 1.0f);
  float3 o = ro, d = rd;
  for (int bounce = 0; bounce < kBounces; ++bounce) {
    const Hit hit = scene_hit(sc, o, d, overflow);
    if (hit.tri == ~0u) {
      const float3 e = sample_env(sc, d);
      radiance = make_float3(radiance.x + thr.x * e.x, radiance.y + thr.y * e.y, radiance.z + thr.z * e.z);
      break;
    }
    float3 nrm;
    float4 col;
    shade(sc, hit, nrm, col);
    const float3 n = dot3(nrm, d) > 0.0f ? make_float3(-nrm.x, -nrm.y, -nrm.z) : nrm;
    o = make_float3(o.x + d.x * hit.t + n.x * 5e-4f, o.y + d.y * hit.t + n.y * 5e-4f, o.z + d.z * hit.t + n.z * 5e-4f);
    if (col.w < 0.5f) {  // perfect mirror
      const float k = 2.0f * dot3(n, d);
      d = make_float3(d.x - k * n.x, d.y - k * n.y, d.z - k * n.z);
    } else {
      thr = make_float3(thr.x * col.x, thr.y * col.y, thr.z * col.z);
      d = cosine_hemisphere(n, seed);
    }
  }
  return radiance;
}

__global__ void __launch_bounds__(128, 10) k_path_trace(Scene sc, Camera cam, float4* __restrict__ accum, uint32_t w,
                                                    uint32_t h, uint32_t frame0, uint32_t frames,
                                                    uint32_t* overflow) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t x = blockIdx.x * 16u + (warp & 1u) * 8u + (lane & 7u);
  const uint32_t y = blockIdx.y * 8u + (warp >> 1) * 4u + (lane >> 3);
  if (x >= w || y >= h) return;
  float4 acc = accum[(size_t)y * w + x];
  for (uint32_t f = 0; f < frames; ++f) {
    const float3 r = trace_pixel(sc, cam, x, y, w, h, frame0 + f, overflow);
    acc.x += r.x;
    acc.y += r.y;
    acc.z += r.z;
    acc.w += 1.0f;
  }
  accum[(size_t)y * w + x] = acc;
}

// path_trace_resolve.wgsl:20-30: mean radiance x 4 through c / (c + 1)
__device__ __forceinline__ float unorm8(float x) { return rintf(fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f) / 255.0f; }
__global__ void k_pt_resolve(const float4* __restrict__ accum, float4* __restrict__ out, uint32_t w, uint32_t h,
                             int quantize) {
  const uint32_t x = blockIdx.x * 16u + threadIdx.x, y = blockIdx.y * 16u + threadIdx.y;
  if (x >= w || y >= h) return;
  const float4 a = accum[(size_t)y * w + x];
  const float n = fmaxf(a.w, 1.0f);
  float r = (a.x / n) * 4.0f, g = (a.y / n) * 4.0f, b = (a.z / n) * 4.0f;
  r = r / (r + 1.0f);
  g = g / (g + 1.0f);
  b = b / (b + 1.0f);
  if (quantize) r = unorm8(r), g = unorm8(g), b = unorm8(b);
  out[(size_t)y * w + x] = make_float4(r, g, b, 1.0f);
}

int check_mesh(const char* fn, const float* vertices, uint32_t n_vertices, const uint32_t* indices, uint32_t n_tris) {
  if ((n_vertices && !vertices) || (n_tris && !indices) || n_tris > (1u << 26) || n_vertices > (1u << 27)) {
    set_error("%s: bad arguments", fn);
    return NPS_ERR_INVALID;
  }
  for (size_t i = 0; i < (size_t)n_tris * 3; ++i)
    if (indices[i] >= n_vertices) {
      set_error("%s: index %u of triangle %zu is not below the vertex count %u", fn, indices[i], i / 3, n_vertices);
      return NPS_ERR_INVALID;
    }
  for (size_t v = 0; v < n_vertices; ++v)
    for (int k = 0; k < 10; ++k)
      if (!std::isfinite(vertices[v * 12 + k])) {
        set_error("%s: vertex %zu has a non-finite position, normal or colour", fn, v);
        return NPS_ERR_INVALID;
      }
  return NPS_OK;
}

}  // namespace pt
}  // namespace nps

using namespace nps;

struct nps_pt {
  nps_ctx* ctx = nullptr;
  pt::Bvh bvh;
  uint32_t n_verts = 0, n_tris = 0;
  DevBuf nodes, tri_pos, tri_idx, verts, env, stats;
  int env_w = 0, env_h = 0;
  ~nps_pt() {
    for (DevBuf* b : {&nodes, &tri_pos, &tri_idx, &verts, &env, &stats}) b->release();
  }
};

extern "C" {

int nps_bvh_build(const float* vertices, uint32_t n_vertices, const uint32_t* indices, uint32_t n_tris,
                  float* nodes, uint32_t* tri_indices, uint32_t* n_nodes) {
  if (!nodes || !n_nodes || (n_tris && !tri_indices)) {
    set_error("nps_bvh_build: bad arguments");
    return NPS_ERR_INVALID;
  }
  NPS_TRY(pt::check_mesh("nps_bvh_build", vertices, n_vertices, indices, n_tris));
  pt::Bvh b;
  pt::build_bvh(vertices, indices, n_tris, b);
  std::memcpy(nodes, b.nodes.data(), b.nodes.size() * 4);
  if (n_tris) std::memcpy(tri_indices, b.tris.data(), (size_t)n_tris * 12);
  *n_nodes = (uint32_t)(b.nodes.size() / 8);
  return NPS_OK;
}

int nps_pt_create(nps_ctx* ctx, const float* vertices, uint32_t n_vertices, const uint32_t* indices, uint32_t n_tris,
                  nps_pt** out) {
  if (!ctx || !out) {
    set_error("nps_pt_create: bad arguments");
    return NPS_ERR_INVALID;
  }
  *out = nullptr;
  NPS_TRY(pt::check_mesh("nps_pt_create", vertices, n_vertices, indices, n_tris));
  NPS_TRY(bind_device(ctx));
  nps_pt* o = new nps_pt();
  o->ctx = ctx;
  o->n_verts = n_vertices;
  o->n_tris = n_tris;
  pt::build_bvh(vertices, indices, n_tris, o->bvh);
  const size_t n_nodes = o->bvh.nodes.size() / 8;
  std::vector<float> pos((size_t)n_tris * 12, 0.0f);
  for (size_t t = 0; t < n_tris; ++t)
    for (int c = 0; c < 3; ++c)
      for (int k = 0; k < 3; ++k) pos[t * 12 + c * 3 + k] = vertices[(size_t)o->bvh.tris[t * 3 + c] * 12 + k];
  const float white[4] = {1.0f, 1.0f, 1.0f, 1.0f};
  int rc = NPS_OK;
  if ((rc = o->nodes.ensure(n_nodes * 32)) || (rc = o->tri_pos.ensure(pos.size() * 4 + 16)) ||
      (rc = o->tri_idx.ensure((size_t)n_tris * 12 + 16)) || (rc = o->verts.ensure((size_t)n_vertices * 48 + 16)) ||
      (rc = o->env.ensure(16)) || (rc = o->stats.ensure(16))) {
    delete o;
    return rc;
  }
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(o->nodes.p, o->bvh.nodes.data(), n_nodes * 32, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && n_tris)
    e = cudaMemcpyAsync(o->tri_pos.p, pos.data(), pos.size() * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && n_tris)
    e = cudaMemcpyAsync(o->tri_idx.p, o->bvh.tris.data(), (size_t)n_tris * 12, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && n_vertices)
    e = cudaMemcpyAsync(o->verts.p, vertices, (size_t)n_vertices * 48, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(o->env.p, white, 16, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(o->stats.p, 0, 16, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host staging vectors go out of scope
  if (e != cudaSuccess) {
    set_error("nps_pt_create: upload failed: %s", cudaGetErrorString(e));
    delete o;
    return NPS_ERR_CUDA;
  }
  o->env_w = o->env_h = 1;
  *out = o;
  return NPS_OK;
}

int nps_pt_destroy(nps_pt* o) {
  if (!o) return NPS_OK;
  cudaSetDevice(o->ctx->device);
  cudaStreamSynchronize(o->ctx->stream);
  delete o;
  return NPS_OK;
}

int nps_pt_bvh_size(nps_pt* o, uint32_t* n_nodes, uint32_t* n_tris) {
  if (!o || !n_nodes || !n_tris) {
    set_error("nps_pt_bvh_size: bad arguments");
    return NPS_ERR_INVALID;
  }
  *n_nodes = (uint32_t)(o->bvh.nodes.size() / 8);
  *n_tris = o->n_tris;
  return NPS_OK;
}

int nps_pt_read_bvh(nps_pt* o, float* nodes, uint32_t* tri_indices) {
  if (!o || !nodes || (o->n_tris && !tri_indices)) {
    set_error("nps_pt_read_bvh: bad arguments");
    return NPS_ERR_INVALID;
  }
  std::memcpy(nodes, o->bvh.nodes.data(), o->bvh.nodes.size() * 4);
  if (o->n_tris) std::memcpy(tri_indices, o->bvh.tris.data(), (size_t)o->n_tris * 12);
  return NPS_OK;
}

int nps_pt_set_env(nps_pt* o, const float* rgba, uint32_t w, uint32_t h) {
  if (!o || !rgba || w == 0 || h == 0 || w > 65536 || h > 65536) {
    set_error("nps_pt_set_env: bad arguments");
    return NPS_ERR_INVALID;
  }
  NPS_TRY(bind_device(o->ctx));
  cudaStream_t s = o->ctx->stream;
  NPS_CUDA(cudaStreamSynchronize(s));  // a trace in flight may still read the old image
  NPS_TRY(o->env.ensure((size_t)w * h * 16));
  NPS_CUDA(cudaMemcpyAsync(o->env.p, rgba, (size_t)w * h * 16, cudaMemcpyDefault, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  o->env_w = (int)w;
  o->env_h = (int)h;
  return NPS_OK;
}

int nps_pt_trace(nps_pt* o, const float* inv_view_proj, uint32_t frame, uint32_t n_frames, float* accum_rgba,
                 uint32_t w, uint32_t h) {
  if (!o || !inv_view_proj || !accum_rgba || w == 0 || h == 0 || w > 65536 || h > 65536 || n_frames > 65536) {
    set_error("nps_pt_trace: bad arguments");
    return NPS_ERR_INVALID;
  }
  if (((uintptr_t)accum_rgba & 15) != 0) {
    set_error("nps_pt_trace: the accumulation image must be a 16-byte aligned float4 array");
    return NPS_ERR_INVALID;
  }
  NPS_TRY(bind_device(o->ctx));
  if (n_frames == 0) return NPS_OK;
  pt::Scene sc;
  sc.nodes = o->nodes.as<float4>();
  sc.tri_pos = o->tri_pos.as<float4>();
  sc.tri_idx = o->tri_idx.as<uint32_t>();
  sc.verts = o->verts.as<float>();
  sc.env = o->env.as<float4>();
  sc.env_w = o->env_w;
  sc.env_h = o->env_h;
  sc.n_nodes = (uint32_t)(o->bvh.nodes.size() / 8);
  pt::Camera cam;
  std::memcpy(cam.m, inv_view_proj, sizeof cam.m);
  const dim3 grid(div_up(w, 16), div_up(h, 8));
  pt::k_path_trace<<<grid, 128, 0, o->ctx->stream>>>(sc, cam, (float4*)accum_rgba, w, h, frame, n_frames,
                                                     o->stats.as<uint32_t>());
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int nps_pt_overflows(nps_pt* o, uint32_t* count) {
  if (!o || !count) {
    set_error("nps_pt_overflows: bad arguments");
    return NPS_ERR_INVALID;
  }
  NPS_TRY(bind_device(o->ctx));
  NPS_CUDA(cudaMemcpyAsync(count, o->stats.p, 4, cudaMemcpyDeviceToHost, o->ctx->stream));
  NPS_CUDA(cudaStreamSynchronize(o->ctx->stream));
  return NPS_OK;
}

int nps_pt_resolve(nps_ctx* ctx, const float* accum_rgba, float* out_rgba, uint32_t w, uint32_t h, int quantize) {
  if (!ctx || !accum_rgba || !out_rgba || w == 0 || h == 0 || w > 65536 || h > 65536 ||
      (((uintptr_t)accum_rgba | (uintptr_t)out_rgba) & 15) != 0) {
    set_error("nps_pt_resolve: bad arguments (16-byte aligned float4 images)");
    return NPS_ERR_INVALID;
  }
  NPS_TRY(bind_device(ctx));
  const dim3 grid(div_up(w, 16), div_up(h, 16));
  pt::k_pt_resolve<<<grid, dim3(16, 16), 0, ctx->stream>>>((const float4*)accum_rgba, (float4*)out_rgba, w, h,
                                                           quantize);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

}  // extern "C"
