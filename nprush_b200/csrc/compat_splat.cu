// compat_splat.cu — splat training step with the reference's semantics.
//
// Implements GpuSplatOptimizerManager.dispatch() (GpuSplatOptimizerManager.ts:
// 365-388) as B200 kernels instead of the reference's per-tile all-N scan:
//   k_project      per (view, splat): the pixel-independent part of eval_splat
//                  (splat_backward.wgsl:92-126) + the binning AABB
//                  (:155-195) turned into a tile rectangle (exact predicate,
//                  binary search over per-axis tile bounds)
//   scan + k_emit  one (view*tiles + tile, splat) pair per overlapped tile
//   radix sort     stable by key, so every tile list is in ascending splat
//                  index order, as the reference's bitmask compaction
//                  (:199-210) produces
//   k_raster       one CTA per (tile, view): first 1024 entries only (the cap
//                  at :205), fp32 front-to-back composite (:216-248), L2 +
//                  depth loss (:250-257), reverse backward (:259-456) with
//                  transmittance replayed exactly from per-32-splat
//                  checkpoints, per-pair i32 truncation, warp __reduce_add_sync
//                  and CTA shared-memory sums before one global atomic per
//                  (splat, param) per tile
//   k_step         splat_step.wgsl:32-106
//   k_adc          splat_adc.wgsl:28-87, same serial result, computed a
//                  1024-splat window at a time
// This file is compiled with --fmad=false: every float operation is rounded
// separately, in the reference's order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "binning.cuh"
#include "bulk.cuh"
#include "common.cuh"
#include "context.h"

namespace nps {
namespace compat {

constexpr int kFwd = 16;        // floats per forward record
constexpr int kBwd = 36;        // floats per backward record (144 B)
constexpr uint32_t kCap = 1024; // SPLAT_MAX_TILE_SPLATS, constants.ts:35
constexpr int kChunk = 32;
constexpr int kThreads = 256;
constexpr float kFpPos = 10000.0f, kFpCol = 100000.0f;  // constants.ts:36-37
constexpr float kOpacityKill = 0.05f, kVolumeKill = 1e-7f, kGradThresh = 0.00005f, kAdcPeriod = 25.0f;

__constant__ float c_lr[16] = {0.0005f, 0.0005f, 0.0005f, 0.01f, 0.02f, 0.02f, 0.02f, 0.01f,
                               0.005f, 0.005f, 0.005f, 0.005f, 0.01f, 0.01f, 0.01f, 0.01f};
__constant__ float c_mu[16] = {0.005f, 0.005f, 0.005f, 0.005f, 0.001f, 0.001f, 0.001f, 0.0005f,
                               0.005f, 0.005f, 0.005f, 0.005f, 0.005f, 0.05f, 0.05f, 0.005f};
__constant__ float c_lo[16] = {-1e9f, -1e9f, -1e9f, 0.001f, 0.05f, 0.05f, 0.05f, 0.01f,
                               -1e9f, -1e9f, -1e9f, -1e9f, 0.001f, 0.1f, 0.01f, 0.001f};
__constant__ float c_hi[16] = {1e9f, 1e9f, 1e9f, 2.0f, 1.0f, 1.0f, 1.0f, 0.99f,
                               1e9f, 1e9f, 1e9f, 1e9f, 2.0f, 10.0f, 5.0f, 2.0f};

__device__ __forceinline__ float clampf(float e, float lo, float hi) { return fminf(fmaxf(e, lo), hi); }

// WGSL i32(f32): truncate toward zero, saturate.
__device__ __forceinline__ int32_t to_i32(float a) {
  // the conversion instruction truncates and clamps below at INT32_MIN by
  // itself (float-to-integer conversions saturate); WGSL's upper bound is the
  // largest float below 2^31
  if (a != a) return 0;
  return a >= 2147483520.0f ? 2147483520 : (int32_t)a;
}

// WGSL M * vec4 with a column-major matrix, summed left to right.
__device__ __forceinline__ float4 mulv(const float* m, float x, float y, float z, float w) {
  float4 o;
  o.x = m[0] * x + m[4] * y + m[8] * z + m[12] * w;
  o.y = m[1] * x + m[5] * y + m[9] * z + m[13] * w;
  o.z = m[2] * x + m[6] * y + m[10] * z + m[14] * w;
  o.w = m[3] * x + m[7] * y + m[11] * z + m[15] * w;
  return o;
}

struct f3 { float x, y, z; };
__device__ __forceinline__ f3 cross3(f3 a, f3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
// splat_backward.wgsl:42-45
__device__ __forceinline__ f3 quat_rotate(float qw, float qx, float qy, float qz, f3 v) {
  f3 u{qx, qy, qz};
  f3 c = cross3(u, v);
  f3 t{2.0f * c.x, 2.0f * c.y, 2.0f * c.z};
  f3 c2 = cross3(u, t);
  return {v.x + qw * t.x + c2.x, v.y + qw * t.y + c2.y, v.z + qw * t.z + c2.z};
}
// splat_backward.wgsl:52-58
__device__ __forceinline__ float2 project_axis(const float* vp, f3 ax, float cx, float cy, float w, float aspect) {
  float4 ac = mulv(vp, ax.x, ax.y, ax.z, 0.0f);
  return make_float2((ac.x * w - cx * ac.w) / (w * w) * aspect, (ac.y * w - cy * ac.w) / (w * w));
}
// splat_backward.wgsl:34-40, one axis at a time
__device__ __forceinline__ float pixel_px(uint32_t px, uint32_t w, float aspect) {
  float u = ((float)px + 0.5f) / (float)w;
  return (u * 2.0f - 1.0f) * aspect;
}
__device__ __forceinline__ float pixel_py(uint32_t py, uint32_t h) {
  float u = ((float)py + 0.5f) / (float)h;
  return -(u * 2.0f - 1.0f);
}

// Tile bounds per axis, splat_backward.wgsl:148-153.
__global__ void k_tile_tables(float* tabs, uint32_t tiles_x, uint32_t tiles_y, uint32_t w, uint32_t h) {
  const float aspect = (float)w / (float)h;
  for (uint32_t t = threadIdx.x; t < tiles_x; t += blockDim.x) {
    tabs[t] = pixel_px(t * 16u, w, aspect);                            // tile_min_p.x
    tabs[tiles_x + t] = pixel_px(min(t * 16u + 16u, w), w, aspect);    // tile_max_p.x
  }
  for (uint32_t t = threadIdx.x; t < tiles_y; t += blockDim.x) {
    tabs[2 * tiles_x + t] = pixel_py(min(t * 16u + 16u, h), h);        // tile_min_p.y
    tabs[2 * tiles_x + tiles_y + t] = pixel_py(t * 16u, h);            // tile_max_p.y
  }
}

__global__ void __launch_bounds__(256) k_project(const float* __restrict__ splats, uint32_t n,
                                                 const float* __restrict__ views, uint32_t nv, uint32_t w, uint32_t h,
                                                 const float* __restrict__ tabs, uint32_t tiles_x, uint32_t tiles_y,
                                                 float* __restrict__ fwd, float* __restrict__ bwd,
                                                 uint32_t* __restrict__ counts, uint2* __restrict__ rects) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nv * n) return;
  const uint32_t v = g / n, i = g - v * n;
  const float* vp = views + 32 * (size_t)v;
  float s[16];
  const float4* sp4 = reinterpret_cast<const float4*>(splats + 16 * (size_t)i);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float4 t = sp4[q];
    s[4 * q] = t.x; s[4 * q + 1] = t.y; s[4 * q + 2] = t.z; s[4 * q + 3] = t.w;
  }
  const float aspect = (float)w / (float)h;
  // eval_splat, pixel-independent part (splat_backward.wgsl:94-126)
  float4 clip = mulv(vp, s[0], s[1], s[2], 1.0f);
  const float W = clip.w;
  const float scx = clip.x / clip.w * aspect, scy = clip.y / clip.w;
  const float sx = fmaxf(s[3], 0.0001f), sy = fmaxf(s[12], 0.0001f), sz = fmaxf(s[15], 0.0001f);
  f3 axw = quat_rotate(s[8], s[9], s[10], s[11], {1.0f, 0.0f, 0.0f});
  f3 ayw = quat_rotate(s[8], s[9], s[10], s[11], {0.0f, 1.0f, 0.0f});
  f3 azw = quat_rotate(s[8], s[9], s[10], s[11], {0.0f, 0.0f, 1.0f});
  float2 ax = project_axis(vp, axw, clip.x, clip.y, W, aspect);
  float2 ay = project_axis(vp, ayw, clip.x, clip.y, W, aspect);
  float2 az = project_axis(vp, azw, clip.x, clip.y, W, aspect);
  const float m0x = ax.x * sx, m0y = ax.y * sx, m1x = ay.x * sy, m1y = ay.y * sy, m2x = az.x * sz, m2y = az.y * sz;
  float cov00 = m0x * m0x + m1x * m1x + m2x * m2x;
  float cov01 = m0x * m0y + m1x * m1y + m2x * m2y;
  float cov11 = m0y * m0y + m1y * m1y + m2y * m2y;
  const float filter_std = 0.3f * (2.0f / (float)h);
  const float filter2 = filter_std * filter_std;
  cov00 += filter2;
  cov11 += filter2;
  const float det = cov00 * cov11 - cov01 * cov01;
  const float inv_det = fabsf(det) < 1e-10f ? 0.0f : 1.0f / det;
  const float A = cov11 * inv_det, B = -cov01 * inv_det, C = cov00 * inv_det;
  const float ld = fmaxf(W, 0.1f);
  const float depth = clampf(1.0f - 0.1f / ld, 0.0f, 1.0f);

  float4* f4 = reinterpret_cast<float4*>(fwd + (size_t)g * kFwd);
  f4[0] = make_float4(scx, scy, A, B);
  f4[1] = make_float4(C, s[13], s[14], s[7]);
  f4[2] = make_float4(s[4], s[5], s[6], depth);
  // a / 2 for pow(r, a) = 2^((a / 2) log2 r^2); the shape regularisers' gradients (splat_backward.wgsl:427-428)
  f4[3] = make_float4(0.5f * s[13], 0.005f * 2.0f * (s[13] - 6.0f), 0.005f * 2.0f * (s[14] - 0.3f), 0.0f);
  float4* b4 = reinterpret_cast<float4*>(bwd + (size_t)g * kBwd);
  // pixel-independent factors of the backward's screen-space chain rule
  // (splat_backward.wgsl:380-398), per world axis: d screen / d pos, and the
  // depth term's vp[ax][3] * DEPTH_NEAR / w^2 — the same expressions, in the
  // same order, as a per-pixel evaluation would give
  const float w2 = W * W;
  const float d_depth_d_w = 0.1f / (W * W);
  float dsx[3], dsy[3], kdep[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float vp0 = vp[k * 4 + 0], vp1 = vp[k * 4 + 1], vp3 = vp[k * 4 + 3];
    dsx[k] = aspect * (vp0 * W - clip.x * vp3) / w2;
    dsy[k] = (vp1 * W - clip.y * vp3) / w2;
    kdep[k] = vp3 * d_depth_d_w;
  }
  // the quaternion's doubles and quadruples (exact scalings) that the
  // rotation's gradient (splat_backward.wgsl:410-426) multiplies with
  b4[0] = make_float4(W, sx, sy, sz);
  b4[1] = make_float4(m0x, m0y, m1x, m1y);
  b4[2] = make_float4(m2x, m2y, ax.x, ax.y);
  b4[3] = make_float4(ay.x, ay.y, az.x, az.y);
  b4[4] = make_float4(s[0], s[1], s[2], 2.0f * s[8]);
  b4[5] = make_float4(2.0f * s[9], 2.0f * s[10], 2.0f * s[11], 4.0f * s[9]);
  b4[6] = make_float4(4.0f * s[10], 4.0f * s[11], dsx[0], dsx[1]);
  b4[7] = make_float4(dsx[2], dsy[0], dsy[1], dsy[2]);
  b4[8] = make_float4(kdep[0], kdep[1], kdep[2], 0.0f);

  // binning AABB, splat_backward.wgsl:157-190 (same arithmetic, cov00/cov11
  // recomputed there without cov01: identical values)
  uint32_t cnt = 0;
  uint2 rect = make_uint2(0u, 0u);
  if (!(s[7] < 0.005f) && !(W < 0.0f)) {
    const float safe_sb = fmaxf(s[14], 0.0001f);
    const float R = powf(15.0f / safe_sb, 1.0f / s[13]);
    const float max_r = R * sqrtf(fmaxf(fmaxf(cov00, cov11), 1e-9f));
    const float smin_x = scx - max_r, smin_y = scy - max_r, smax_x = scx + max_r, smax_y = scy + max_r;
    const float* tminx = tabs;
    const float* tmaxx = tabs + tiles_x;
    const float* tminy = tabs + 2 * tiles_x;
    const float* tmaxy = tabs + 2 * tiles_x + tiles_y;
    // first tx with !(smin.x > tile_max.x)
    uint32_t lo = 0, hi = tiles_x;
    while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (!(smin_x > tmaxx[m])) hi = m; else lo = m + 1; }
    const uint32_t x0 = lo;
    // first tx with (smax.x < tile_min.x) -> last overlapping = that - 1
    lo = 0; hi = tiles_x;
    while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (smax_x < tminx[m]) hi = m; else lo = m + 1; }
    const uint32_t x1 = lo;  // exclusive
    // rows: tile_max.y / tile_min.y decrease with ty
    lo = 0; hi = tiles_y;
    while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (!(smax_y < tminy[m])) hi = m; else lo = m + 1; }
    const uint32_t y0 = lo;
    lo = 0; hi = tiles_y;
    while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (smin_y > tmaxy[m]) hi = m; else lo = m + 1; }
    const uint32_t y1 = lo;  // exclusive
    if (x1 > x0 && y1 > y0) {
      cnt = (x1 - x0) * (y1 - y0);
      rect = make_uint2(x0 | (x1 << 16), y0 | (y1 << 16));
    }
  }
  counts[g] = cnt;
  rects[g] = rect;
}

// ---- cap-aware binning
// Only the first kCap entries of a tile list (in splat index order) are ever
// composited, and at 200k splats most of a scene's (tile, splat) overlaps lie
// beyond them.  The splats are cut into nb index blocks of bs splats:
// k_bin_diff adds every splat's tile rectangle to a 2D difference grid of its
// (view, block), k_bin_rows / k_bin_cols turn each grid into per-tile counts,
// k_bin_cutoff finds for every (view, tile) the block in which its running
// count reaches kCap (every later block lies beyond the cap) and the full list
// length, and k_bin_pairs counts, then writes, only the pairs whose splat
// block is at or before its tile's cutoff block.  Pairs are written in
// (view, splat) order, so the stable sort by tile key still gives every tile
// list in index order, and its first kCap entries are exactly those of the
// full list.  Without a cutoff array (nb = 1) every overlapped tile is kept.
__global__ void k_bin_diff(const uint2* __restrict__ rects, const uint32_t* __restrict__ counts, uint32_t n,
                           uint32_t nv, uint32_t bs, uint32_t nb, uint32_t gx, uint32_t gy, int32_t* __restrict__ grid) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nv * n || counts[g] == 0) return;
  const uint32_t v = g / n, i = g - v * n;
  const uint2 r = rects[g];
  const uint32_t x0 = r.x & 0xffffu, x1 = r.x >> 16, y0 = r.y & 0xffffu, y1 = r.y >> 16;
  int32_t* G = grid + ((size_t)v * nb + i / bs) * gx * gy;
  atomicAdd(G + y0 * gx + x0, 1);
  atomicAdd(G + y0 * gx + x1, -1);
  atomicAdd(G + y1 * gx + x0, -1);
  atomicAdd(G + y1 * gx + x1, 1);
}

// In-place inclusive prefix of every grid row (along x), one thread per row.
__global__ void k_bin_rows(int32_t* __restrict__ grid, uint32_t rows, uint32_t gx) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  int32_t* p = grid + (size_t)r * gx;
  int32_t acc = 0;
  for (uint32_t x = 0; x < gx; ++x) p[x] = acc += p[x];
}

// In-place inclusive prefix of every grid column (along y), one thread per
// (grid, column).
__global__ void k_bin_cols(int32_t* __restrict__ grid, uint32_t grids, uint32_t gx, uint32_t gy) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= grids * gx) return;
  const uint32_t gi = t / gx, x = t - gi * gx;
  int32_t* p = grid + (size_t)gi * gx * gy + x;
  int32_t acc = 0;
  for (uint32_t y = 0; y < gy; ++y) p[(size_t)y * gx] = acc += p[(size_t)y * gx];
}

// Per (view, tile): the last splat block its first kCap entries need, and the
// full list length.  Also sums the lengths (pairs overlapped) into *total.
__global__ void k_bin_cutoff(const int32_t* __restrict__ grid, uint32_t nv, uint32_t nb, uint32_t tiles_x,
                             uint32_t num_tiles, uint32_t gx, uint32_t gy, uint32_t* __restrict__ cutoff,
                             uint32_t* __restrict__ tile_len, unsigned long long* __restrict__ total) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t len = 0;
  if (t < nv * num_tiles) {
    const uint32_t v = t / num_tiles, tile = t - v * num_tiles;
    const uint32_t ty = tile / tiles_x, tx = tile - ty * tiles_x;
    const int32_t* G = grid + (size_t)v * nb * gx * gy + (size_t)ty * gx + tx;
    uint32_t cut = nb - 1;
    bool found = false;
    for (uint32_t b = 0; b < nb; ++b) {
      len += (uint32_t)G[(size_t)b * gx * gy];
      if (!found && len >= kCap) {
        cut = b;
        found = true;
      }
    }
    cutoff[t] = cut;
    tile_len[t] = len;
  }
  unsigned long long s = len;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s != 0) atomicAdd(total, s);
}

// One warp per (view, splat) item, its lanes over the item's tile rectangle:
// kWrite = false counts the kept pairs into out_counts, kWrite = true writes
// them at offsets[item] onwards (positions beyond cap are dropped).
template <bool kWrite>
__global__ void __launch_bounds__(256) k_bin_pairs(const uint2* __restrict__ rects, const uint32_t* __restrict__ counts,
                                                   const uint32_t* __restrict__ cutoff, uint32_t n, uint32_t nv,
                                                   uint32_t bs, uint32_t tiles_x, uint32_t num_tiles,
                                                   uint32_t* __restrict__ out_counts,
                                                   const uint32_t* __restrict__ offsets, uint32_t cap,
                                                   uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < nv * n; g += nw) {
    const uint32_t c = counts[g];
    if (c == 0) {
      if (!kWrite && lane == 0) out_counts[g] = 0;
      continue;
    }
    const uint32_t v = g / n, i = g - v * n, b = i / bs;
    const uint2 r = rects[g];
    const uint32_t x0 = r.x & 0xffffu, x1 = r.x >> 16, y0 = r.y & 0xffffu;
    const uint32_t w = x1 - x0;
    const uint32_t* cut = cutoff ? cutoff + (size_t)v * num_tiles : nullptr;
    uint32_t pos = kWrite ? offsets[g] : 0u;
    for (uint32_t base = 0; base < c; base += 32) {
      const uint32_t k = base + lane;
      uint32_t tile = 0;
      bool keep = false;
      if (k < c) {
        const uint32_t ry = k / w;
        tile = (y0 + ry) * tiles_x + x0 + (k - ry * w);
        keep = !cut || cut[tile] >= b;
      }
      const uint32_t m = __ballot_sync(0xffffffffu, keep);
      if (kWrite && keep) {
        const uint32_t p = pos + __popc(m & ((1u << lane) - 1u));
        if (p < cap) {
          keys[p] = v * num_tiles + tile;
          vals[p] = i;
        }
      }
      pos += __popc(m);
    }
    if (!kWrite && lane == 0) out_counts[g] = pos;
  }
}

// Statistics of the last backward's tile lists from their full lengths:
// out[0] += sum of min(length, kCap) (pairs composited), out[1] = longest.
__global__ void k_tile_stats(const uint32_t* __restrict__ tile_len, uint32_t m, unsigned long long* __restrict__ out) {
  unsigned long long sum = 0;
  uint32_t mx = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const uint32_t len = tile_len[i];
    sum += min(len, kCap);
    mx = max(mx, len);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out, sum);
    atomicMax(out + 1, (unsigned long long)mx);
  }
}

// Full list lengths when every pair was emitted (no cutoff): rend - rstart.
__global__ void k_range_len(const uint32_t* __restrict__ rstart, const uint32_t* __restrict__ rend, uint32_t m,
                            uint32_t* __restrict__ tile_len) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    tile_len[i] = rend[i] - rstart[i];
}

// Tile list bounds in the sorted key array.
__global__ void k_ranges(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ total, uint32_t cap,
                         uint32_t* __restrict__ rstart, uint32_t* __restrict__ rend) {
  const uint32_t K = min(*total, cap);
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < K; p += gridDim.x * blockDim.x) {
    const uint32_t k = keys[p];
    if (p == 0 || keys[p - 1] != k) rstart[k] = p;
    if (p == K - 1 || keys[p + 1] != k) rend[k] = p + 1;
  }
}

struct RasterArgs {
  const float* fwd;
  const float* bwd;
  const uint32_t* vals;
  const uint32_t* rstart;
  const uint32_t* rend;
  const float* views;
  const float* tgt_rgba;
  const float* tgt_depth;
  int32_t* grads;
  float* out_rgbd;
  uint32_t* err;  // bounded waits that gave up (the output of such a tile is not written)
  float* ckpt;    // per (view, tile): T of every pixel at the start of each chunk, [kNumChunks][kThreads]
  uint32_t spin_limit;   // polls of a staging mbarrier before the wait gives up
  uint32_t stall_batch;  // tests: the batch of tile 0 whose copies are never issued (0xffffffff = none)
  uint32_t n, w, h, tiles_x, num_tiles;
};

constexpr uint32_t kNumChunks = kCap / kChunk;
constexpr uint32_t kFwdBytes = sizeof(float) * kFwd, kBwdBytes = sizeof(float) * kBwd;

// Shared memory of one k_raster CTA (dynamic, ~50 KB: four CTAs per SM).
struct __align__(16) RasterSmem {
  float fwd[2][kChunk][kFwd];          // staged forward records (double-buffered)
  float bwd[2][kChunk][kBwd];          // staged backward records
  float tprev[kChunk][kThreads];       // T before each pair of the chunk being differentiated
  int32_t gacc[2][kChunk][16];         // per-chunk CTA sums of the i32 gradient terms
  uint32_t ids[3][kChunk];             // splat index of each staged record
  uint64_t bar[2];                     // one mbarrier per record buffer
  int abort;
};

// Approximate base-2 logarithm and exponential on the special-function unit.
// WGSL defines pow(x, y)'s accuracy as that of exp2(y * log2(x)), and exp's
// and log's by a few ULP: the reference's shaders are not bit-defined here.
__device__ __forceinline__ float lg2_approx(float x) {
  float y;
  asm("lg2.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kLog2e = 1.4426950408889634f;
constexpr float kHalfLn2 = 0.34657359027997264f;

// Per-pixel part of eval_splat (splat_backward.wgsl:127-132) for forward
// record f at pixel (ppx, ppy): r = sqrt(max(r2, 1e-4)), pow(r, a) evaluated
// as 2^((a / 2) log2 max(r2, 1e-4)) (f[12] = a / 2), exp(x) as 2^(x log2 e).
// Every caller evaluates the same instruction sequence, so the forward, its
// replay and the backward see bit-identical alphas.
struct PixEval {
  float spx, spy, r2c, lg, rpa, power, a_un, al;
  bool above;
};
__device__ __forceinline__ PixEval eval_px(const float* f, float ppx, float ppy) {
  PixEval e;
  const float dx = ppx - f[0], dy = ppy - f[1];
  e.spx = fmaf(f[2], dx, f[3] * dy);
  e.spy = fmaf(f[3], dx, f[4] * dy);
  e.r2c = fmaxf(fmaf(dx, e.spx, dy * e.spy), 0.0001f);
  e.lg = lg2_approx(e.r2c);
  e.rpa = ex2_approx(f[12] * e.lg);
  e.power = -f[6] * e.rpa;
  e.above = e.power > -15.0f;
  e.a_un = e.above ? ex2_approx(e.power * kLog2e) : 0.0f;
  e.al = clampf(e.above ? e.a_un * f[7] : 0.0f, 0.0f, 0.999f);
  return e;
}

// The part of one (pixel, splat) backward term (splat_backward.wgsl:259-330)
// that every valid pair evaluates: the carried dL/dT sums (updated in place),
// dL/dalpha, dL/dpower and the shape gradients with their regularisers.
struct PairCommon {
  float da, d_power, d_shape_a, d_shape_b;
};
__device__ __forceinline__ PairCommon pair_common(const float* f, const PixEval& e, float T_prev, float dCr,
                                                  float dCg, float dCb, float dD, float& dT_C, float& dT_D) {
  const float cr = f[8], cg = f[9], cb = f[10], opacity = f[7], depth = f[11];
  const float shape_b = f[6], al = e.al;
  const float tcr = T_prev * cr, tcg = T_prev * cg, tcb = T_prev * cb;
  const float da_C = dT_C * (-T_prev) + (dCr * tcr + dCg * tcg + dCb * tcb);
  const float da_D = dT_D * (-T_prev) + dD * T_prev * depth;
  PairCommon p;
  p.da = da_C + da_D;
  const float acr = al * cr, acg = al * cg, acb = al * cb;
  dT_C = dT_C * (1.0f - al) + (dCr * acr + dCg * acg + dCb * acb);
  dT_D = dT_D * (1.0f - al) + dD * al * depth;
  p.d_power = e.above ? p.da * opacity * e.a_un : 0.0f;
  const float logr = e.lg * kHalfLn2;
  p.d_shape_a = e.above ? p.d_power * (-shape_b * e.rpa * logr) : 0.0f;
  p.d_shape_b = e.above ? p.d_power * (-e.rpa) : 0.0f;
  p.d_shape_a += f[13];  // 0.005 * 2 * (shape_a - 6), per splat (k_project)
  p.d_shape_b += f[14];  // 0.005 * 2 * (shape_b - 0.3)
  return p;
}

// One CTA per (tile, view), one pixel per thread, each warp an 8 x 4 strip.
// Records are staged 32 at a time by warp 0 with bulk copies completing on
// an mbarrier, double-buffered (the next chunk lands while this one is
// composited); the forward stores T at every chunk start, and the backward
// walks the chunks in reverse, replaying each from its checkpoint.  The
// checkpoints (32 KB per CTA) live in global memory, where they stay in L2
// between the forward's write and the backward's read: kept in shared memory
// they held residency at two CTAs per SM, here four fit (64 registers).
//
// Exact skips (results identical to evaluating every pair):
//  * a warp whose 32 pixels all reached T == 0 stops compositing: a pair
//    then adds T * alpha * c = 0 and leaves T at 0 (for finite colours and
//    depths, which the step keeps inside their boxes);
//  * a chunk that starts at T == 0 for the whole warp is not replayed;
//  * a pair whose valid pixels (alpha >= 0.001) all have T_prev == 0 adds
//    only its shape regularisers: with T_prev == 0 every other term is a
//    product with a zero factor, which is 0 or NaN, and i32() maps both to 0;
//    so only dL/dT, d_shape_a and d_shape_b are evaluated and summed.
__global__ void __launch_bounds__(kThreads, 4) k_raster(RasterArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RasterSmem& S = *reinterpret_cast<RasterSmem*>(smem_raw);
  constexpr unsigned kFull = 0xffffffffu;

  const uint32_t tx = blockIdx.x, ty = blockIdx.y, v = blockIdx.z;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t px = tx * 16 + 8 * (warp & 1u) + (lane & 7u), py = ty * 16 + 4 * (warp >> 1) + (lane >> 3);
  const bool inside = px < a.w && py < a.h;
  const float aspect = (float)a.w / (float)a.h;
  const float ppx = pixel_px(px, a.w, aspect), ppy = pixel_py(py, a.h);
  const uint32_t key = v * a.num_tiles + ty * a.tiles_x + tx;
  const uint32_t start = a.rstart[key];
  const uint32_t len = min(a.rend[key] - start, kCap);
  const uint32_t nch = (len + kChunk - 1) / kChunk;
  const float* fwd_v = a.fwd + (size_t)v * a.n * kFwd;
  const float* bwd_v = a.bwd + (size_t)v * a.n * kBwd;
  float* ckpt = a.ckpt + (size_t)key * kNumChunks * kThreads;  // this CTA's own: written, then read back
  for (uint32_t e = tid; e < 2 * kChunk * 16; e += kThreads) (&S.gacc[0][0][0])[e] = 0;
  if (tid == 0) {
    bulk::mbar_init(&S.bar[0], 1);
    bulk::mbar_init(&S.bar[1], 1);
    S.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // Batch q (warp 0 stages it into record buffer q & 1, ids q % 3): for
  // q < nch the forward records of chunk q, else both records of chunk
  // 2 nch - 1 - q (the backward's order).
  auto stage = [&](uint32_t q) {
    const bool both = q >= nch;
    const uint32_t c = both ? 2 * nch - 1 - q : q;
    const uint32_t cnt = min((uint32_t)kChunk, len - c * kChunk);
    const uint32_t b = q & 1u;
    if (lane == 0) bulk::mbar_expect_tx(&S.bar[b], cnt * (both ? kFwdBytes + kBwdBytes : kFwdBytes));
    if (lane < cnt && !(key == 0 && q == a.stall_batch)) {
      bulk::fence_proxy_async();  // the buffer was last read through the generic proxy
      const uint32_t id = a.vals[start + c * kChunk + lane];
      S.ids[q % 3][lane] = id;
      bulk::bulk_g2s(&S.fwd[b][lane][0], fwd_v + (size_t)id * kFwd, kFwdBytes, &S.bar[b]);
      if (both) bulk::bulk_g2s(&S.bwd[b][lane][0], bwd_v + (size_t)id * kBwd, kBwdBytes, &S.bar[b]);
    }
  };
  auto wait_batch = [&](uint32_t q) {
    if (!bulk::mbar_wait(&S.bar[q & 1u], (q >> 1) & 1u, a.spin_limit) && lane == 0) {
      atomicAdd(a.err, 1u);
      S.abort = 1;
    }
  };
  uint32_t issued = 0;  // batches staged so far (CTA-uniform)
  if (nch > 0) {
    if (warp == 0) stage(0);
    issued = 1;
  }

  // ---- forward: front-to-back composite (splat_backward.wgsl:216-248)
  float T = 1.0f, Cr = 0.0f, Cg = 0.0f, Cb = 0.0f, D = 0.0f;
  bool wdone = false;
  uint32_t c = 0;
  for (; c < nch; ++c) {
    __syncthreads();  // every warp is done with batch c - 1: its buffers may be refilled
    if (S.abort) break;
    if (issued < 2 * nch) {
      if (warp == 0) stage(issued);
      ++issued;
    }
    wait_batch(c);
    ckpt[c * kThreads + tid] = T;
    if (!wdone) {
      const uint32_t cnt = min((uint32_t)kChunk, len - c * kChunk);
      const uint32_t b = c & 1u;
      for (uint32_t k = 0; k < cnt; ++k) {
        const float* f = S.fwd[b][k];
        const float al = eval_px(f, ppx, ppy).al;
        Cr += T * al * f[8];
        Cg += T * al * f[9];
        Cb += T * al * f[10];
        D += T * al * f[11];
        T = T * (1.0f - al);
      }
      wdone = __all_sync(kFull, T == 0.0f);
    }
  }
  const float bg = 0.05f;
  Cr += T * bg; Cg += T * bg; Cb += T * bg;
  D += T * 1.0f;
  const size_t pix = ((size_t)v * a.h + (inside ? py : 0)) * a.w + (inside ? px : 0);
  if (inside && a.out_rgbd && !S.abort) reinterpret_cast<float4*>(a.out_rgbd)[pix] = make_float4(Cr, Cg, Cb, D);
  // loss, splat_backward.wgsl:250-257
  const float4 tc = inside ? reinterpret_cast<const float4*>(a.tgt_rgba)[pix] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float td = inside ? a.tgt_depth[pix] : 1.0f;
  const float dCr = 2.0f * (Cr - tc.x), dCg = 2.0f * (Cg - tc.y), dCb = 2.0f * (Cb - tc.z);
  const bool fg = td < 0.99f;
  const float dD = fg ? 2.0f * (D - td) : 0.0f;
  float dT_C = dCr * bg + dCg * bg + dCb * bg;
  float dT_D = dD * 1.0f;
  // reconstruct_world_pos (splat_backward.wgsl:64-75): pair-independent
  float surf_x = 0.0f, surf_y = 0.0f, surf_z = 0.0f;
  if (fg) {
    const float* vpi = a.views + 32 * (size_t)v + 16;
    const float wr = 0.1f / fmaxf(1.0f - td, 1e-5f);
    const float ndx = ppx / aspect, ndy = ppy;
    float4 wp = mulv(vpi, ndx * wr, ndy * wr, wr, wr);
    surf_x = wp.x / wp.w; surf_y = wp.y / wp.w; surf_z = wp.z / wp.w;
  }
  const float DEPTH_NEAR = 0.1f;

  // ---- backward: reverse order (splat_backward.wgsl:259-456)
  auto flush = [&](uint32_t q) {  // batch q's CTA sums -> one global atomic per (splat, value)
    const uint32_t cc = 2 * nch - 1 - q;
    const uint32_t cnt = min((uint32_t)kChunk, len - cc * kChunk);
    int32_t* g = &S.gacc[q & 1u][0][0];
    for (uint32_t e = tid; e < cnt * 16; e += kThreads) {
      const int32_t val = g[e];
      if (val != 0) {
        atomicAdd(&a.grads[16 * (size_t)S.ids[q % 3][e >> 4] + (e & 15)], val);
        g[e] = 0;
      }
    }
  };
  uint32_t j = 0;
  for (; c == nch && j < nch; ++j) {
    const uint32_t q = nch + j, cc = nch - 1 - j, b = q & 1u;
    __syncthreads();  // batch q - 1 is done: its sums are complete and its buffers free
    if (S.abort) break;
    if (j > 0) flush(q - 1);
    if (issued < 2 * nch) {
      if (warp == 0) stage(issued);
      ++issued;
    }
    wait_batch(q);
    const uint32_t cnt = min((uint32_t)kChunk, len - cc * kChunk);
    // replay the chunk forward from its checkpoint: bit-identical Ts
    const float T0 = ckpt[cc * kThreads + tid];
    const bool zero_chunk = __all_sync(kFull, T0 == 0.0f);
    if (!zero_chunk) {
      float Tc = T0;
      for (uint32_t k = 0; k < cnt; ++k) {
        S.tprev[k][tid] = Tc;
        Tc = Tc * (1.0f - eval_px(S.fwd[b][k], ppx, ppy).al);
      }
    }
    int32_t* gacc = &S.gacc[b][0][0];
    for (int k = (int)cnt - 1; k >= 0; --k) {
      const float* f = S.fwd[b][k];
      const PixEval e = eval_px(f, ppx, ppy);
      const bool valid = inside && !(e.al < 0.001f);
      if (!__any_sync(kFull, valid)) continue;
      const float T_prev = zero_chunk ? 0.0f : S.tprev[k][tid];
      if (!__any_sync(kFull, valid && T_prev != 0.0f)) {
        // only the shape regularisers and the carried dL/dT sums (see above)
        int32_t q13 = 0, q14 = 0;
        if (valid) {
          const PairCommon p = pair_common(f, e, T_prev, dCr, dCg, dCb, dD, dT_C, dT_D);
          q13 = to_i32(p.d_shape_a * kFpPos);
          q14 = to_i32(p.d_shape_b * kFpPos);
        }
        const int32_t r13 = __reduce_add_sync(kFull, q13), r14 = __reduce_add_sync(kFull, q14);
        if (lane == 0) {
          if (r13 != 0) atomicAdd(&gacc[k * 16 + 13], r13);
          if (r14 != 0) atomicAdd(&gacc[k * 16 + 14], r14);
        }
        continue;
      }
      int32_t qv[16];
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) qv[jj] = 0;
      if (valid) {
        const float* bw = S.bwd[b][k];
        const float al = e.al;
        const float shape_a = f[5], shape_b = f[6];
        const float Wc = bw[0], sx = bw[1], sy = bw[2], sz = bw[3];
        const float m0x = bw[4], m0y = bw[5], m1x = bw[6], m1y = bw[7], m2x = bw[8], m2y = bw[9];
        const float axx = bw[10], axy = bw[11], ayx = bw[12], ayy = bw[13], azx = bw[14], azy = bw[15];
        const float pos0 = bw[16], pos1 = bw[17], pos2 = bw[18];
        // 2 q and 4 q: x * 2 * q == x * (2 q) exactly, the scaling by 2 or 4 being exact
        const float q2w = bw[19], q2x = bw[20], q2y = bw[21], q2z = bw[22];
        const float q4x = bw[23], q4y = bw[24], q4z = bw[25];
        const float TA = T_prev * al;
        const float dColr = dCr * TA, dColg = dCg * TA, dColb = dCb * TA;
        const float d_depth = dD * T_prev * al;
        const PairCommon p = pair_common(f, e, T_prev, dCr, dCg, dCb, dD, dT_C, dT_D);
        const float d_opacity = e.above ? p.da * e.a_un : 0.0f;
        const float r_pow_a_m2 = __fdividef(e.rpa, e.r2c);  // r^(a - 2) = r^a / r^2
        const float kk = p.d_power * (-shape_b * shape_a * r_pow_a_m2);
        const float ddx = e.above ? kk * e.spx : 0.0f, ddy = e.above ? kk * e.spy : 0.0f;
        const float dsx_ = -ddx, dsy_ = -ddy;
        const float sp0 = e.spx * m0x + e.spy * m0y;
        const float sp1 = e.spx * m1x + e.spy * m1y;
        const float sp2 = e.spx * m2x + e.spy * m2y;
        const float dm0x = -sp0 * ddx, dm0y = -sp0 * ddy;
        const float dm1x = -sp1 * ddx, dm1y = -sp1 * ddy;
        const float dm2x = -sp2 * ddx, dm2y = -sp2 * ddy;
        const float daxx = dm0x * sx, daxy = dm0y * sx, dayx = dm1x * sy, dayy = dm1y * sy, dazx = dm2x * sz,
                    dazy = dm2y * sz;
        const float d_sx = dm0x * axx + dm0y * axy;
        const float d_sy = dm1x * ayx + dm1y * ayy;
        const float d_sz = dm2x * azx + dm2y * azy;
        float dpos[3], daw[3], dbw[3], dcw[3];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          // d screen / d pos and vp[ax][3] DEPTH_NEAR / w^2 from the record (k_project)
          const float ds_dx = bw[26 + ax], ds_dy = bw[29 + ax];
          dpos[ax] = dsx_ * ds_dx + dsy_ * ds_dy;
          dpos[ax] += (Wc > DEPTH_NEAR) ? bw[32 + ax] * d_depth : 0.0f;
          daw[ax] = daxx * ds_dx + daxy * ds_dy;
          dbw[ax] = dayx * ds_dx + dayy * ds_dy;
          dcw[ax] = dazx * ds_dx + dazy * ds_dy;
        }
        if (fg) {
          dpos[0] += 0.3f * 2.0f * (pos0 - surf_x) * (T_prev * al);
          dpos[1] += 0.3f * 2.0f * (pos1 - surf_y) * (T_prev * al);
          dpos[2] += 0.3f * 2.0f * (pos2 - surf_z) * (T_prev * al);
        }
        // splat_backward.wgsl:410-426
        const float d_qw = (daw[1] * q2z - daw[2] * q2y) + (-dbw[0] * q2z + dbw[2] * q2x) +
                           (dcw[0] * q2y - dcw[1] * q2x);
        const float d_qx = (daw[1] * q2y + daw[2] * q2z) + (dbw[0] * q2y - dbw[1] * q4x + dbw[2] * q2w) +
                           (dcw[0] * q2z - dcw[1] * q2w - dcw[2] * q4x);
        const float d_qy = (-daw[0] * q4y + daw[1] * q2x + daw[2] * (-q2w)) + (dbw[0] * q2x + dbw[2] * q2z) +
                           (dcw[0] * q2w + dcw[1] * q2z - dcw[2] * q4y);
        const float d_qz = (-daw[0] * q4z + daw[1] * q2w + daw[2] * q2x) +
                           (-dbw[0] * q2w - dbw[1] * q4z + dbw[2] * q2y) + (dcw[0] * q2x + dcw[1] * q2y);
        qv[0] = to_i32(dpos[0] * kFpPos);
        qv[1] = to_i32(dpos[1] * kFpPos);
        qv[2] = to_i32(dpos[2] * kFpPos);
        qv[3] = to_i32(d_sx * kFpPos);
        qv[4] = to_i32(dColr * kFpCol);
        qv[5] = to_i32(dColg * kFpCol);
        qv[6] = to_i32(dColb * kFpCol);
        qv[7] = to_i32(d_opacity * kFpCol);
        qv[8] = to_i32(d_qw * kFpPos);
        qv[9] = to_i32(d_qx * kFpPos);
        qv[10] = to_i32(d_qy * kFpPos);
        qv[11] = to_i32(d_qz * kFpPos);
        qv[12] = to_i32(d_sy * kFpPos);
        qv[13] = to_i32(p.d_shape_a * kFpPos);
        qv[14] = to_i32(p.d_shape_b * kFpPos);
        qv[15] = to_i32(d_sz * kFpPos);
      }
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) {
        const int32_t r = __reduce_add_sync(kFull, qv[jj]);
        if (lane == 0 && r != 0) atomicAdd(&gacc[k * 16 + jj], r);
      }
    }
  }
  __syncthreads();
  if (!S.abort) {
    if (nch > 0) flush(2 * nch - 1);
    return;
  }
  // a bounded wait gave up: wait (bounded) for the batches still in flight
  // (at most the last two staged) before the CTA's shared memory is released
  if (tid == 0)
    for (uint32_t q = issued >= 2 ? issued - 2 : 0; q < issued; ++q)
      (void)bulk::mbar_wait(&S.bar[q & 1u], (q >> 1) & 1u, a.spin_limit);
}

// splat_step.wgsl:32-106, one thread per splat.
__global__ void __launch_bounds__(256) k_step(float* __restrict__ splats, int32_t* __restrict__ grads,
                                              float* __restrict__ am, float* __restrict__ av,
                                              float* __restrict__ gacc, uint32_t n, float bc1, float bc2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s[16], m[16], v[16];
  int32_t g[16];
  float4* s4 = reinterpret_cast<float4*>(splats + 16 * (size_t)i);
  float4* m4 = reinterpret_cast<float4*>(am + 16 * (size_t)i);
  float4* v4 = reinterpret_cast<float4*>(av + 16 * (size_t)i);
  int4* g4 = reinterpret_cast<int4*>(grads + 16 * (size_t)i);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float4 a = s4[q], b = m4[q], c = v4[q];
    int4 d = g4[q];
    s[4 * q] = a.x; s[4 * q + 1] = a.y; s[4 * q + 2] = a.z; s[4 * q + 3] = a.w;
    m[4 * q] = b.x; m[4 * q + 1] = b.y; m[4 * q + 2] = b.z; m[4 * q + 3] = b.w;
    v[4 * q] = c.x; v[4 * q + 1] = c.y; v[4 * q + 2] = c.z; v[4 * q + 3] = c.w;
    g[4 * q] = d.x; g[4 * q + 1] = d.y; g[4 * q + 2] = d.z; g[4 * q + 3] = d.w;
  }
  const float B1 = 0.9f, B2 = 0.999f, EPS = 1e-8f;
  float pos_g2 = 0.0f;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const float fps = (k >= 4 && k <= 7) ? kFpCol : kFpPos;
    const float gr = (float)g[k] / fps / 16384.0f;
    const float mm = B1 * m[k] + (1.0f - B1) * gr;
    const float vv = B2 * v[k] + (1.0f - B2) * gr * gr;
    m[k] = mm;
    v[k] = vv;
    const float m_hat = mm / bc1, v_hat = vv / bc2;
    const float raw_u = c_lr[k] * m_hat / (sqrtf(v_hat) + EPS);
    const float u = clampf(raw_u, -c_mu[k], c_mu[k]);
    s[k] = clampf(s[k] - u, c_lo[k], c_hi[k]);
    if (k <= 2) pos_g2 += gr * gr;
  }
  float ql = sqrtf(s[8] * s[8] + s[9] * s[9] + s[10] * s[10] + s[11] * s[11]);
  ql = fmaxf(ql, 1e-8f);
  s[8] = s[8] / ql; s[9] = s[9] / ql; s[10] = s[10] / ql; s[11] = s[11] / ql;
  gacc[i] = gacc[i] + sqrtf(pos_g2);
  const float vol = s[3] * s[12] * s[15];
  if (s[7] < kOpacityKill || vol < kVolumeKill) s[7] = 0.0f;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    s4[q] = make_float4(s[4 * q], s[4 * q + 1], s[4 * q + 2], s[4 * q + 3]);
    m4[q] = make_float4(m[4 * q], m[4 * q + 1], m[4 * q + 2], m[4 * q + 3]);
    v4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    g4[q] = make_int4(0, 0, 0, 0);
  }
}

constexpr int kAdcThreads = 1024;

// Exclusive scan of one value per thread over a 1024-thread block.
__device__ __forceinline__ uint32_t block_exclusive_scan_adc(uint32_t x, uint32_t* total) {
  __shared__ uint32_t warp_sums[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_sums[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = warp_sums[lane];
    uint32_t si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += y;
    }
    warp_sums[lane] = si - s;
    if (lane == 31) *total = si;
  }
  __syncthreads();
  uint32_t r = warp_sums[wid] + inc - x;
  __syncthreads();
  return r;
}

__device__ __forceinline__ float fractf(float x) { return x - floorf(x); }

// splat_adc.wgsl:28-87.  One CTA.  The serial loop is reproduced window by
// window: every splat of a 1024-wide window is classified in parallel, the
// k-th clone candidate takes the k-th unused dead slot, and the window is
// committed up to the first slot that a candidate fills AHEAD of itself inside
// the window (that slot is alive, with its stale accumulator, when the serial
// loop reaches it) — the window then restarts there.
__global__ void __launch_bounds__(kAdcThreads) k_adc(float* __restrict__ splats, float* __restrict__ am,
                                                     float* __restrict__ av, float* __restrict__ gacc,
                                                     uint32_t* __restrict__ dead, uint32_t n, float adam_t,
                                                     uint32_t* __restrict__ stats) {
  __shared__ uint32_t s_total;
  __shared__ uint32_t s_min;
  const uint32_t tid = threadIdx.x;
  // dead slots at entry, ascending (the serial search order)
  uint32_t nd = 0;
  for (uint32_t base = 0; base < n; base += kAdcThreads) {
    const uint32_t i = base + tid;
    const uint32_t f = (i < n && splats[16 * (size_t)i + 7] < kOpacityKill) ? 1u : 0u;
    const uint32_t r = block_exclusive_scan_adc(f, &s_total);
    if (f) dead[nd + r] = i;
    nd += s_total;
    __syncthreads();
  }
  uint32_t cursor = 0, clones = 0;
  uint32_t base = 0;
  while (base < n) {
    const uint32_t i = base + tid;
    const bool inwin = i < n;
    bool alive = false, cand = false;
    if (inwin) {
      const float op = splats[16 * (size_t)i + 7];
      alive = !(op < kOpacityKill);
      cand = alive && (gacc[i] / kAdcPeriod > kGradThresh);
    }
    const uint32_t r = block_exclusive_scan_adc(cand ? 1u : 0u, &s_total);
    const bool has_slot = cand && (cursor + r < nd);
    const uint32_t d = has_slot ? dead[cursor + r] : 0u;
    if (tid == 0) s_min = 0xffffffffu;
    __syncthreads();
    if (has_slot && d > i && d < base + kAdcThreads) atomicMin(&s_min, d);
    __syncthreads();
    const uint32_t commit_end = s_min == 0xffffffffu ? base + kAdcThreads : s_min;
    const bool commit = inwin && i < commit_end;
    if (commit && alive) gacc[i] = 0.0f;
    if (commit && has_slot) {
      float s[16], ns[16];
      float4* s4 = reinterpret_cast<float4*>(splats + 16 * (size_t)i);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float4 t = s4[q];
        s[4 * q] = t.x; s[4 * q + 1] = t.y; s[4 * q + 2] = t.z; s[4 * q + 3] = t.w;
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) ns[k] = s[k];
      const float scale_norm = sqrtf(s[3] * s[3] + s[12] * s[12] + s[15] * s[15]);
      if (scale_norm > 0.01f) {
        const float fct = 0.625f;
        s[3] *= fct; s[12] *= fct; s[15] *= fct;
        ns[3] *= fct; ns[12] *= fct; ns[15] *= fct;
        s[0] -= s[3] * 0.05f;
        ns[0] += s[3] * 0.05f;
      } else {
        const float seed = (float)i * 3.14159f + adam_t;
        ns[0] += (fractf(sinf(seed * 12.9898f) * 43758.5453f) - 0.5f) * 0.002f;
        ns[1] += (fractf(sinf(seed * 78.233f) * 43758.5453f) - 0.5f) * 0.002f;
      }
      float4* d4 = reinterpret_cast<float4*>(splats + 16 * (size_t)d);
      float4* mi = reinterpret_cast<float4*>(am + 16 * (size_t)i);
      float4* vi = reinterpret_cast<float4*>(av + 16 * (size_t)i);
      float4* md = reinterpret_cast<float4*>(am + 16 * (size_t)d);
      float4* vd = reinterpret_cast<float4*>(av + 16 * (size_t)d);
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        s4[q] = make_float4(s[4 * q], s[4 * q + 1], s[4 * q + 2], s[4 * q + 3]);
        d4[q] = make_float4(ns[4 * q], ns[4 * q + 1], ns[4 * q + 2], ns[4 * q + 3]);
        mi[q] = z; vi[q] = z; md[q] = z; vd[q] = z;
      }
    }
    const uint32_t used = __syncthreads_count(commit && has_slot);
    cursor += used;
    clones += used;
    __threadfence_block();
    __syncthreads();
    base = commit_end;
  }
  if (tid == 0 && stats) stats[0] = clones;
}


// ------------------------------------------------------------- display forward
// splat_forward.wgsl:42-156 (vertex quad, fragment alpha) headless: each splat
// covers the screen rectangle centre +- R sqrt(cov) (top-left rule); its
// fragments composite front to back with splat 0 in front (the reference
// draws instances in reverse order with src-alpha blending).
constexpr int kRend = 16;  // floats per render record

__global__ void __launch_bounds__(256) k_render_project(const float* __restrict__ splats, uint32_t n,
                                                        const float* __restrict__ vp, uint32_t w, uint32_t h,
                                                        const float* __restrict__ tabs, uint32_t tiles_x,
                                                        uint32_t tiles_y, float* __restrict__ rec,
                                                        uint32_t* __restrict__ counts, uint2* __restrict__ rects) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s[16];
  const float4* sp4 = reinterpret_cast<const float4*>(splats + 16 * (size_t)i);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float4 t = sp4[q];
    s[4 * q] = t.x; s[4 * q + 1] = t.y; s[4 * q + 2] = t.z; s[4 * q + 3] = t.w;
  }
  const float aspect = (float)w / (float)h;
  uint32_t cnt = 0;
  uint2 rect = make_uint2(0u, 0u);
  const float sx = fmaxf(s[3], 0.0001f), sy = fmaxf(s[12], 0.0001f), sz = fmaxf(s[15], 0.0001f);
  const float safe_b = fmaxf(s[14], 0.0001f);
  const float R = powf(15.0f / safe_b, 1.0f / s[13]);
  const float4 clip = mulv(vp, s[0], s[1], s[2], 1.0f);
  const float W = clip.w;
  float4* r4 = reinterpret_cast<float4*>(rec + (size_t)i * kRend);
  // the vertex stage collapses splats with w < 0.1 (splat_forward.wgsl:61-66); every vertex
  // of the quad has the centre's clip z and w, so the pipeline's clipping against
  // 0 <= z <= w keeps or drops the whole quad (a splat past the far plane is not drawn)
  if (!(W < 0.1f) && clip.z >= 0.0f && clip.z <= W) {
    f3 axw = quat_rotate(s[8], s[9], s[10], s[11], {1.0f, 0.0f, 0.0f});
    f3 ayw = quat_rotate(s[8], s[9], s[10], s[11], {0.0f, 1.0f, 0.0f});
    f3 azw = quat_rotate(s[8], s[9], s[10], s[11], {0.0f, 0.0f, 1.0f});
    const float2 ax = project_axis(vp, axw, clip.x, clip.y, W, aspect);
    const float2 ay = project_axis(vp, ayw, clip.x, clip.y, W, aspect);
    const float2 az = project_axis(vp, azw, clip.x, clip.y, W, aspect);
    const float m0x = ax.x * sx, m0y = ax.y * sx, m1x = ay.x * sy, m1y = ay.y * sy, m2x = az.x * sz, m2y = az.y * sz;
    float cov00 = m0x * m0x + m1x * m1x + m2x * m2x;
    const float cov01 = m0x * m0y + m1x * m1y + m2x * m2y;
    float cov11 = m0y * m0y + m1y * m1y + m2y * m2y;
    const float fs = 0.3f * (2.0f / (float)h);
    cov00 += fs * fs;
    cov11 += fs * fs;
    const float det = cov00 * cov11 - cov01 * cov01;
    const float inv_det = fabsf(det) < 1e-10f ? 0.0f : 1.0f / det;
    const float A = cov11 * inv_det, B = -cov01 * inv_det, C = cov00 * inv_det;
    const float ex = R * sqrtf(fmaxf(cov00, 1e-9f)), ey = R * sqrtf(fmaxf(cov11, 1e-9f));
    const float cx = clip.x / W * aspect, cy = clip.y / W;
    const float ld = fmaxf(W, 0.1f);
    const float depth = clampf(1.0f - 0.1f / ld, 0.0f, 1.0f);
    r4[0] = make_float4(cx, cy, cx - ex, cx + ex);
    r4[1] = make_float4(cy - ey, cy + ey, A, B);
    r4[2] = make_float4(C, s[13], s[14], s[7]);
    r4[3] = make_float4(s[4], s[5], s[6], depth);
    if (bin::tile_rect(tabs, tiles_x, tiles_y, cx - ex, cy - ey, cx + ex, cy + ey, &rect))
      cnt = ((rect.x >> 16) - (rect.x & 0xffffu)) * ((rect.y >> 16) - (rect.y & 0xffffu));
  }
  counts[i] = cnt;
  rects[i] = rect;
}

__global__ void __launch_bounds__(256) k_render_raster(const float* __restrict__ rec, const uint32_t* __restrict__ vals,
                                                       const uint32_t* __restrict__ rstart,
                                                       const uint32_t* __restrict__ rend, uint32_t w, uint32_t h,
                                                       uint32_t tiles_x, float4* __restrict__ out_rgba,
                                                       float4* __restrict__ out_depth, int load) {
  __shared__ float4 sr[256][4];
  const uint32_t tx = blockIdx.x, ty = blockIdx.y, tid = threadIdx.x;
  const uint32_t px = tx * 16 + (tid & 15), py = ty * 16 + (tid >> 4);
  const bool inside = px < w && py < h;
  const float aspect = (float)w / (float)h;
  const float ppx = pixel_px(px, w, aspect), ppy = pixel_py(py, h);
  const uint32_t key = ty * tiles_x + tx;
  const uint32_t start = rstart[key], end = rend[key];
  float T = 1.0f, C0 = 0.0f, C1 = 0.0f, C2 = 0.0f, D = 0.0f;
  for (uint32_t base = start; base < end; base += 256) {
    __syncthreads();
    if (base + tid < end) {
      const float4* src = reinterpret_cast<const float4*>(rec + (size_t)vals[base + tid] * kRend);
      sr[tid][0] = src[0]; sr[tid][1] = src[1]; sr[tid][2] = src[2]; sr[tid][3] = src[3];
    }
    __syncthreads();
    const uint32_t nb = min(256u, end - base);
    for (uint32_t j = 0; j < nb; ++j) {
      const float4 a = sr[j][0], b = sr[j][1];
      // pixel centre inside the quad (top-left rule)
      if (!(ppx >= a.z && ppx < a.w && ppy > b.x && ppy <= b.y)) continue;
      const float4 c = sr[j][2], d = sr[j][3];
      const float dx = ppx - a.x, dy = ppy - a.y;
      const float r2 = b.z * dx * dx + 2.0f * b.w * dx * dy + c.x * dy * dy;
      const float r = sqrtf(fmaxf(r2, 0.0001f));
      const float pw = -c.z * powf(r, c.y);
      float al = pw > -15.0f ? expf(pw) * c.w : 0.0f;
      al = clampf(al, 0.0f, 0.999f);
      if (al < 0.001f) continue;
      C0 += T * al * d.x;
      C1 += T * al * d.y;
      C2 += T * al * d.z;
      D += T * al * d.w;
      T *= (1.0f - al);
    }
  }
  if (inside) {
    const size_t pix = (size_t)py * w + px;
    if (!load) {  // attachments cleared to colour (0.05, 0.05, 0.05, 1), depth 1
      out_rgba[pix] = make_float4(C0 + T * 0.05f, C1 + T * 0.05f, C2 + T * 0.05f, 1.0f);
      const float dd = D + T * 1.0f;
      if (out_depth) out_depth[pix] = make_float4(dd, dd, dd, 1.0f);
    } else {  // over the attachments' current contents; alpha = a + dst.a (1 - a) per fragment
      const float4 c = out_rgba[pix];
      out_rgba[pix] = make_float4(C0 + T * c.x, C1 + T * c.y, C2 + T * c.z, (1.0f - T) + T * c.w);
      if (out_depth) {
        const float4 d = out_depth[pix];
        out_depth[pix] = make_float4(D + T * d.x, D + T * d.y, D + T * d.z, (1.0f - T) + T * d.w);
      }
    }
  }
}

}  // namespace compat
}  // namespace nps

// =================================================================== host side
using namespace nps;

// work buffers of the display render (kept by the optimiser, on its device)
struct RenderWork {
  DevBuf rec, counts, offsets, rects, total, cam, keys, vals, ranges, tabs;
  SortWork sw;
  uint32_t pair_cap = 0;
  void release() {
    for (DevBuf* b : {&rec, &counts, &offsets, &rects, &total, &cam, &keys, &vals, &ranges, &tabs, &sw.hist,
                      &sw.partial, &sw.lookback, &sw.keys_alt, &sw.vals_alt})
      b->release();
  }
};

struct nps_splat_opt {
  nps_ctx* ctx = nullptr;
  RenderWork* rw = nullptr;
  uint32_t n = 0;
  DevBuf params, grads, am, av, gacc;
  float adam_t = 0.0f;
  uint32_t step_count = 0;
  // cameras
  uint32_t nv = 0;
  DevBuf views;  // nv * 32 floats: vp, vp_inv
  // targets
  uint32_t w = 0, h = 0, tv = 0;
  DevBuf tgt_rgba_own, tgt_depth_own;
  const float* tgt_rgba = nullptr;
  const float* tgt_depth = nullptr;
  // work
  DevBuf fwd, bwd, counts, kept, offsets, rects, total, keys, vals, ranges, tabs, dead, stat, tstat;
  DevBuf grid, cutoff, tile_len;  // cap-aware binning
  DevBuf ckbuf;                   // raster checkpoints: 32 KB per (view, tile)
  SortWork sw;
  uint32_t pair_cap = 0;
  uint32_t last_ranges = 0;  // (view, tile) entries of the last backward's ranges
  uint32_t spin_limit = 1u << 22, stall_batch = 0xffffffffu;  // raster staging waits (nps_splat_opt_set_wait_guard)
  bool pairs_from_ranges = true;  // the last backward kept every overlapped pair
  uint32_t kept_pairs = 0;
  nps_stats stats{};
};

namespace {

int copy_in(void* dst, const void* src, size_t bytes, int mem, cudaStream_t s) {
  if (bytes == 0) return NPS_OK;
  if (!src) {
    set_error("null source pointer");
    return NPS_ERR_INVALID;
  }
  if (mem == NPS_MEM_HOST) {
    NPS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    NPS_CUDA(cudaStreamSynchronize(s));  // host buffer may be reused on return
  } else {
    NPS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
  }
  return NPS_OK;
}

int check_opt(nps_splat_opt* o) {
  if (!o) {
    set_error("null splat optimizer");
    return NPS_ERR_INVALID;
  }
  return bind_device(o->ctx);
}

}  // namespace

extern "C" {

int nps_splat_opt_create(nps_ctx* ctx, uint32_t num_splats, nps_splat_opt** out) {
  if (!out || num_splats == 0 || num_splats > (1u << 26)) {
    set_error("nps_splat_opt_create: bad arguments (num_splats=%u)", num_splats);
    return NPS_ERR_INVALID;
  }
  *out = nullptr;
  NPS_TRY(bind_device(ctx));
  nps_splat_opt* o = new nps_splat_opt();
  o->ctx = ctx;
  o->n = num_splats;
  const size_t p16 = sizeof(float) * 16 * (size_t)num_splats;
  int rc = NPS_OK;
  if ((rc = o->params.ensure(p16)) || (rc = o->grads.ensure(p16)) || (rc = o->am.ensure(p16)) ||
      (rc = o->av.ensure(p16)) || (rc = o->gacc.ensure(sizeof(float) * num_splats)) ||
      (rc = o->dead.ensure(sizeof(uint32_t) * num_splats)) || (rc = o->stat.ensure(64)) ||
      (rc = o->total.ensure(sizeof(uint32_t) * 4))) {
    delete o;
    return rc;
  }
  cudaStream_t s = ctx->stream;
  cudaMemsetAsync(o->params.p, 0, p16, s);
  cudaMemsetAsync(o->grads.p, 0, p16, s);
  cudaMemsetAsync(o->am.p, 0, p16, s);
  cudaMemsetAsync(o->av.p, 0, p16, s);
  cudaMemsetAsync(o->gacc.p, 0, sizeof(float) * num_splats, s);
  cudaMemsetAsync(o->stat.p, 0, 64, s);
  cudaMemsetAsync(o->total.p, 0, sizeof(uint32_t) * 4, s);
  NPS_CUDA(cudaGetLastError());
  *out = o;
  return NPS_OK;
}

int nps_splat_opt_destroy(nps_splat_opt* o) {
  if (!o) return NPS_OK;
  cudaSetDevice(o->ctx->device);
  cudaStreamSynchronize(o->ctx->stream);
  for (DevBuf* b : {&o->params, &o->grads, &o->am, &o->av, &o->gacc, &o->views, &o->tgt_rgba_own,
                    &o->tgt_depth_own, &o->fwd, &o->bwd, &o->counts, &o->kept, &o->offsets, &o->rects, &o->total,
                    &o->grid, &o->cutoff, &o->tile_len, &o->ckbuf,
                    &o->keys, &o->vals, &o->ranges, &o->tabs, &o->dead, &o->stat, &o->tstat, &o->sw.hist,
                    &o->sw.partial, &o->sw.lookback, &o->sw.keys_alt, &o->sw.vals_alt})
    b->release();
  if (o->rw) {
    o->rw->release();
    delete o->rw;
  }
  delete o;
  return NPS_OK;
}

int nps_splat_opt_write_params(nps_splat_opt* o, const float* splats, uint32_t first, uint32_t count, int mem) {
  NPS_TRY(check_opt(o));
  if ((uint64_t)first + count > o->n) {
    set_error("write_params: range [%u, %u) beyond %u splats", first, first + count, o->n);
    return NPS_ERR_INVALID;
  }
  return copy_in(o->params.as<float>() + 16 * (size_t)first, splats, sizeof(float) * 16 * (size_t)count, mem,
                 o->ctx->stream);
}

int nps_splat_opt_write_state(nps_splat_opt* o, const int32_t* grads, const float* m, const float* v, float t,
                              const float* gacc, int mem) {
  NPS_TRY(check_opt(o));
  const size_t p16 = sizeof(float) * 16 * (size_t)o->n;
  if (grads) NPS_TRY(copy_in(o->grads.p, grads, p16, mem, o->ctx->stream));
  if (m) NPS_TRY(copy_in(o->am.p, m, p16, mem, o->ctx->stream));
  if (v) NPS_TRY(copy_in(o->av.p, v, p16, mem, o->ctx->stream));
  if (gacc) NPS_TRY(copy_in(o->gacc.p, gacc, sizeof(float) * o->n, mem, o->ctx->stream));
  o->adam_t = t;
  return NPS_OK;
}

int nps_splat_opt_read_state(nps_splat_opt* o, float* splats, int32_t* grads, float* m, float* v, float* t,
                             float* gacc) {
  NPS_TRY(check_opt(o));
  cudaStream_t s = o->ctx->stream;
  const size_t p16 = sizeof(float) * 16 * (size_t)o->n;
  if (splats) NPS_CUDA(cudaMemcpyAsync(splats, o->params.p, p16, cudaMemcpyDeviceToHost, s));
  if (grads) NPS_CUDA(cudaMemcpyAsync(grads, o->grads.p, p16, cudaMemcpyDeviceToHost, s));
  if (m) NPS_CUDA(cudaMemcpyAsync(m, o->am.p, p16, cudaMemcpyDeviceToHost, s));
  if (v) NPS_CUDA(cudaMemcpyAsync(v, o->av.p, p16, cudaMemcpyDeviceToHost, s));
  if (gacc) NPS_CUDA(cudaMemcpyAsync(gacc, o->gacc.p, sizeof(float) * o->n, cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  if (t) *t = o->adam_t;
  return NPS_OK;
}

int nps_splat_opt_write_vp(nps_splat_opt* o, const float* vp, const float* vp_inv, uint32_t num_views, int blur) {
  (void)blur;
  NPS_TRY(check_opt(o));
  if (!vp || !vp_inv || num_views == 0 || num_views > 4096) {
    set_error("write_vp: bad arguments");
    return NPS_ERR_INVALID;
  }
  std::vector<float> host(32 * (size_t)num_views);
  for (uint32_t v = 0; v < num_views; ++v) {
    std::memcpy(&host[32 * v], vp + 16 * v, 64);
    std::memcpy(&host[32 * v + 16], vp_inv + 16 * v, 64);
  }
  NPS_TRY(o->views.ensure(sizeof(float) * host.size()));
  o->nv = num_views;
  return copy_in(o->views.p, host.data(), sizeof(float) * host.size(), NPS_MEM_HOST, o->ctx->stream);
}

int nps_splat_opt_set_target(nps_splat_opt* o, const float* rgba, const float* depth, uint32_t w, uint32_t h,
                             uint32_t nv, int mem) {
  NPS_TRY(check_opt(o));
  if (!rgba || !depth || w == 0 || h == 0 || nv == 0 || w > 16 * 65535 || h > 16 * 65535) {
    set_error("set_target: bad arguments");
    return NPS_ERR_INVALID;
  }
  const size_t px = (size_t)w * h * nv;
  if (mem == NPS_MEM_DEVICE_BORROW) {
    if (((uintptr_t)rgba & 15) != 0) {
      set_error("set_target: borrowed rgba must be 16-byte aligned");
      return NPS_ERR_INVALID;
    }
    o->tgt_rgba = rgba;
    o->tgt_depth = depth;
  } else {
    NPS_TRY(o->tgt_rgba_own.ensure(sizeof(float) * 4 * px));
    NPS_TRY(o->tgt_depth_own.ensure(sizeof(float) * px));
    NPS_TRY(copy_in(o->tgt_rgba_own.p, rgba, sizeof(float) * 4 * px, mem, o->ctx->stream));
    NPS_TRY(copy_in(o->tgt_depth_own.p, depth, sizeof(float) * px, mem, o->ctx->stream));
    o->tgt_rgba = o->tgt_rgba_own.as<float>();
    o->tgt_depth = o->tgt_depth_own.as<float>();
  }
  o->w = w;
  o->h = h;
  o->tv = nv;
  const uint32_t tx = div_up(w, 16), ty = div_up(h, 16);
  NPS_TRY(o->tabs.ensure(sizeof(float) * 2 * (tx + ty)));
  compat::k_tile_tables<<<1, 256, 0, o->ctx->stream>>>(o->tabs.as<float>(), tx, ty, w, h);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int nps_splat_opt_backward(nps_splat_opt* o, float* out_rgbd) {
  NPS_TRY(check_opt(o));
  if (!o->tgt_rgba || o->nv == 0) {
    set_error("backward: set_target and write_vp first");
    return NPS_ERR_STATE;
  }
  if (o->tv != o->nv) {
    set_error("backward: %u target views but %u cameras", o->tv, o->nv);
    return NPS_ERR_STATE;
  }
  cudaStream_t s = o->ctx->stream;
  const uint32_t n = o->n, nv = o->nv;
  const uint32_t tiles_x = div_up(o->w, 16), tiles_y = div_up(o->h, 16), num_tiles = tiles_x * tiles_y;
  const size_t g = (size_t)n * nv;
  if (g >= (1ull << 31) || (uint64_t)num_tiles * nv >= (1ull << 31)) {
    set_error("backward: problem too large");
    return NPS_ERR_INVALID;
  }
  NPS_TRY(o->fwd.ensure(sizeof(float) * compat::kFwd * g));
  NPS_TRY(o->bwd.ensure(sizeof(float) * compat::kBwd * g));
  NPS_TRY(o->counts.ensure(sizeof(uint32_t) * g));
  NPS_TRY(o->kept.ensure(sizeof(uint32_t) * g));
  NPS_TRY(o->offsets.ensure(sizeof(uint32_t) * g));
  NPS_TRY(o->rects.ensure(sizeof(uint2) * g));
  NPS_TRY(o->ranges.ensure(sizeof(uint32_t) * 2 * (size_t)num_tiles * nv));
  NPS_TRY(o->tile_len.ensure(sizeof(uint32_t) * (size_t)num_tiles * nv));
  uint32_t* total = o->total.as<uint32_t>();  // [0] pairs kept, [1] bounded waits that gave up, [2..3] u64 pairs
  unsigned long long* overlapped = reinterpret_cast<unsigned long long*>(total + 2);
  o->sw.err = total + 1;
  compat::k_project<<<div_up(g, 256), 256, 0, s>>>(o->params.as<float>(), n, o->views.as<float>(), nv, o->w, o->h,
                                                    o->tabs.as<float>(), tiles_x, tiles_y, o->fwd.as<float>(),
                                                    o->bwd.as<float>(), o->counts.as<uint32_t>(),
                                                    o->rects.as<uint2>());
  NPS_CHECK_LAUNCH();
  // splat blocks of the cap-aware binning: about 1024 splats each, at most
  // 256, and the (view, block) difference grids within 2^26 cells
  const uint32_t gx = tiles_x + 1, gy = tiles_y + 1;
  const uint64_t cells = (uint64_t)nv * gx * gy;
  uint32_t nb = std::min<uint32_t>(div_up(n, 1024), 256u);
  nb = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(nb, (1ull << 26) / cells));
  const uint32_t bs = div_up(n, nb);
  nb = div_up(n, bs);
  const uint32_t* cutoff = nullptr;
  NPS_CUDA(cudaMemsetAsync(overlapped, 0, sizeof(unsigned long long), s));
  if (nb > 1) {
    NPS_TRY(o->grid.ensure(sizeof(int32_t) * cells * nb));
    NPS_TRY(o->cutoff.ensure(sizeof(uint32_t) * (size_t)num_tiles * nv));
    int32_t* grid = o->grid.as<int32_t>();
    NPS_CUDA(cudaMemsetAsync(grid, 0, sizeof(int32_t) * cells * nb, s));
    compat::k_bin_diff<<<div_up(g, 256), 256, 0, s>>>(o->rects.as<uint2>(), o->counts.as<uint32_t>(), n, nv, bs, nb,
                                                       gx, gy, grid);
    const uint32_t grids = nv * nb;
    compat::k_bin_rows<<<div_up((size_t)grids * gy, 128), 128, 0, s>>>(grid, grids * gy, gx);
    compat::k_bin_cols<<<div_up((size_t)grids * gx, 128), 128, 0, s>>>(grid, grids, gx, gy);
    compat::k_bin_cutoff<<<div_up((size_t)num_tiles * nv, 128), 128, 0, s>>>(
        grid, nv, nb, tiles_x, num_tiles, gx, gy, o->cutoff.as<uint32_t>(), o->tile_len.as<uint32_t>(), overlapped);
    NPS_CHECK_LAUNCH();
    cutoff = o->cutoff.as<uint32_t>();
  }
  const uint32_t pair_grid = 8 * kNumSMs;  // 256-thread blocks of warps over the (view, splat) items
  compat::k_bin_pairs<false><<<pair_grid, 256, 0, s>>>(o->rects.as<uint2>(), o->counts.as<uint32_t>(), cutoff, n,
                                                       nv, bs, tiles_x, num_tiles, o->kept.as<uint32_t>(), nullptr, 0,
                                                       nullptr, nullptr);
  NPS_CHECK_LAUNCH();
  NPS_TRY(exclusive_scan_u32(o->kept.as<uint32_t>(), o->offsets.as<uint32_t>(), (uint32_t)g, total, o->sw, s));
  uint32_t hk[2] = {0, 0};  // pairs kept, bounded waits of the previous backward that gave up
  NPS_CUDA(cudaMemcpyAsync(hk, total, sizeof(hk), cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  const uint32_t K = hk[0];
  if (hk[1] != 0) {
    NPS_CUDA(cudaMemsetAsync(total + 1, 0, sizeof(uint32_t), s));
    o->stats.reserved[2] += hk[1];
    set_error("backward: %u bounded device waits of the previous backward gave up (its gradients are not valid)",
              hk[1]);
    return NPS_ERR_TIMEOUT;
  }
  if (K > o->pair_cap) {
    uint32_t cap = K + K / 4 + 4096;
    NPS_TRY(o->keys.ensure(sizeof(uint32_t) * (size_t)cap));
    NPS_TRY(o->vals.ensure(sizeof(uint32_t) * (size_t)cap));
    o->pair_cap = cap;
  }
  NPS_CUDA(cudaMemsetAsync(o->ranges.p, 0, sizeof(uint32_t) * 2 * (size_t)num_tiles * nv, s));
  uint32_t* rstart = o->ranges.as<uint32_t>();
  uint32_t* rend = rstart + (size_t)num_tiles * nv;
  compat::RasterArgs ra{};
  ra.fwd = o->fwd.as<float>();
  ra.bwd = o->bwd.as<float>();
  ra.vals = o->counts.as<uint32_t>();  // no pairs: never read
  ra.rstart = rstart;
  ra.rend = rend;
  ra.views = o->views.as<float>();
  ra.tgt_rgba = o->tgt_rgba;
  ra.tgt_depth = o->tgt_depth;
  ra.grads = o->grads.as<int32_t>();
  ra.out_rgbd = out_rgbd;
  ra.err = total + 1;
  NPS_TRY(o->ckbuf.ensure(sizeof(float) * (size_t)num_tiles * nv * compat::kNumChunks * compat::kThreads));
  ra.ckpt = o->ckbuf.as<float>();
  ra.spin_limit = o->spin_limit;
  ra.stall_batch = o->stall_batch;
  ra.n = n;
  ra.w = o->w;
  ra.h = o->h;
  ra.tiles_x = tiles_x;
  ra.num_tiles = num_tiles;
  if (K > 0) {
    compat::k_bin_pairs<true><<<pair_grid, 256, 0, s>>>(o->rects.as<uint2>(), o->counts.as<uint32_t>(), cutoff, n, nv,
                                                        bs, tiles_x, num_tiles, nullptr, o->offsets.as<uint32_t>(),
                                                        o->pair_cap, o->keys.as<uint32_t>(), o->vals.as<uint32_t>());
    NPS_CHECK_LAUNCH();
    int bits = 1;
    while ((1ull << bits) < (uint64_t)num_tiles * nv) ++bits;
    uint32_t *ks = nullptr, *vs = nullptr;
    NPS_TRY(radix_sort_u32(o->keys.as<uint32_t>(), o->vals.as<uint32_t>(), total, o->pair_cap, bits, o->sw, s, &ks,
                           &vs));
    compat::k_ranges<<<4 * kNumSMs, 256, 0, s>>>(ks, total, o->pair_cap, rstart, rend);
    NPS_CHECK_LAUNCH();
    ra.vals = vs;
  }
  if (!cutoff) {
    // every overlapped pair was kept: the lists are complete
    compat::k_range_len<<<4 * kNumSMs, 256, 0, s>>>(rstart, rend, num_tiles * nv, o->tile_len.as<uint32_t>());
    NPS_CHECK_LAUNCH();
  }
  NPS_CUDA(cudaFuncSetAttribute(compat::k_raster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(compat::RasterSmem)));
  compat::k_raster<<<dim3(tiles_x, tiles_y, nv), compat::kThreads, sizeof(compat::RasterSmem), s>>>(ra);
  NPS_CHECK_LAUNCH();
  o->pairs_from_ranges = cutoff == nullptr;
  o->kept_pairs = K;
  o->last_ranges = num_tiles * nv;
  return NPS_OK;
}

int nps_splat_opt_step(nps_splat_opt* o) {
  NPS_TRY(check_opt(o));
  const float t = o->adam_t + 1.0f;
  // 1 - pow(beta, t) in f32, as splat_step.wgsl:71-72 evaluates it
  const float bc1 = 1.0f - std::pow(0.9f, t), bc2 = 1.0f - std::pow(0.999f, t);
  compat::k_step<<<div_up(o->n, 256), 256, 0, o->ctx->stream>>>(o->params.as<float>(), o->grads.as<int32_t>(),
                                                                 o->am.as<float>(), o->av.as<float>(),
                                                                 o->gacc.as<float>(), o->n, bc1, bc2);
  NPS_CHECK_LAUNCH();
  o->adam_t = t;
  return NPS_OK;
}

int nps_splat_opt_adc(nps_splat_opt* o) {
  NPS_TRY(check_opt(o));
  compat::k_adc<<<1, compat::kAdcThreads, 0, o->ctx->stream>>>(o->params.as<float>(), o->am.as<float>(),
                                                                o->av.as<float>(), o->gacc.as<float>(),
                                                                o->dead.as<uint32_t>(), o->n, o->adam_t,
                                                                o->stat.as<uint32_t>());
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int nps_splat_opt_dispatch(nps_splat_opt* o) {
  NPS_TRY(nps_splat_opt_backward(o, nullptr));
  NPS_TRY(nps_splat_opt_step(o));
  o->step_count++;
  if (o->step_count % 25 == 0) NPS_TRY(nps_splat_opt_adc(o));  // GpuSplatOptimizerManager.ts:380-385
  return NPS_OK;
}

int nps_splat_opt_buffers(nps_splat_opt* o, float** splats, int32_t** grads, float** m, float** v, float** gacc) {
  NPS_TRY(check_opt(o));
  if (splats) *splats = o->params.as<float>();
  if (grads) *grads = o->grads.as<int32_t>();
  if (m) *m = o->am.as<float>();
  if (v) *v = o->av.as<float>();
  if (gacc) *gacc = o->gacc.as<float>();
  return NPS_OK;
}

// the manager's stepCount (GpuSplatOptimizerManager.ts:380): dispatch() calls so far, which decide
// when ADC runs; restoring a checkpoint sets it back
int nps_splat_opt_set_step_count(nps_splat_opt* o, uint32_t count) {
  NPS_TRY(check_opt(o));
  o->step_count = count;
  return NPS_OK;
}

int nps_splat_opt_set_wait_guard(nps_splat_opt* o, uint32_t spin_limit, uint32_t stall_batch) {
  NPS_TRY(check_opt(o));
  o->spin_limit = spin_limit ? spin_limit : 1u << 22;
  o->stall_batch = stall_batch;
  return NPS_OK;
}

int nps_splat_opt_stats(nps_splat_opt* o, nps_stats* out) {
  NPS_TRY(check_opt(o));
  if (!out) return NPS_ERR_INVALID;
  cudaStream_t s = o->ctx->stream;
  uint32_t clones = 0;
  uint64_t ts[2] = {0, 0};  // pairs composited (each tile list capped), longest list
  unsigned long long overlapped = 0;
  NPS_CUDA(cudaMemcpyAsync(&clones, o->stat.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  if (o->last_ranges > 0) {
    NPS_TRY(o->tstat.ensure(2 * sizeof(uint64_t)));
    NPS_CUDA(cudaMemsetAsync(o->tstat.p, 0, 2 * sizeof(uint64_t), s));
    compat::k_tile_stats<<<std::min(div_up(o->last_ranges, 256), 4u * kNumSMs), 256, 0, s>>>(
        o->tile_len.as<uint32_t>(), o->last_ranges, o->tstat.as<unsigned long long>());
    NPS_CHECK_LAUNCH();
    NPS_CUDA(cudaMemcpyAsync(ts, o->tstat.p, sizeof(ts), cudaMemcpyDeviceToHost, s));
    NPS_CUDA(cudaMemcpyAsync(&overlapped, o->total.as<uint32_t>() + 2, sizeof(overlapped), cudaMemcpyDeviceToHost, s));
  }
  NPS_CUDA(cudaStreamSynchronize(s));
  o->stats.reserved[1] = o->kept_pairs;  // pairs kept by the cap-aware binning and sorted
  o->stats.pairs = o->pairs_from_ranges ? o->kept_pairs : overlapped;
  o->stats.pairs_capped = ts[0];
  o->stats.max_tile_len = (uint32_t)ts[1];
  o->stats.adc_clones = clones;
  o->stats.step_count = o->step_count;
  *out = o->stats;
  return NPS_OK;
}

}  // extern "C"

// ================================================================ render
static int splat_render(nps_splat_opt* o, const float* vp, uint32_t w, uint32_t h, float* out_rgba, float* out_depth,
                        int load) {
  NPS_TRY(check_opt(o));
  if (!vp || !out_rgba || w == 0 || h == 0 || w > 16 * 65535 || h > 16 * 65535) {
    set_error("splat render: bad arguments");
    return NPS_ERR_INVALID;
  }
  if (!o->rw) o->rw = new RenderWork();
  RenderWork& rw = *o->rw;
  cudaStream_t s = o->ctx->stream;
  const uint32_t n = o->n, tiles_x = div_up(w, 16), tiles_y = div_up(h, 16), num_tiles = tiles_x * tiles_y;
  NPS_TRY(rw.rec.ensure(sizeof(float) * compat::kRend * n));
  NPS_TRY(rw.counts.ensure(sizeof(uint32_t) * n));
  NPS_TRY(rw.offsets.ensure(sizeof(uint32_t) * n));
  NPS_TRY(rw.rects.ensure(sizeof(uint2) * n));
  NPS_TRY(rw.total.ensure(16));
  NPS_TRY(rw.cam.ensure(64));
  NPS_TRY(rw.ranges.ensure(sizeof(uint32_t) * 2 * num_tiles));
  NPS_TRY(rw.tabs.ensure(sizeof(float) * 2 * (tiles_x + tiles_y)));
  NPS_TRY(copy_in(rw.cam.p, vp, 64, NPS_MEM_HOST, s));
  bin::k_tile_tables<<<1, 256, 0, s>>>(rw.tabs.as<float>(), tiles_x, tiles_y, w, h);
  compat::k_render_project<<<div_up(n, 256), 256, 0, s>>>(o->params.as<float>(), n, rw.cam.as<float>(), w, h,
                                                           rw.tabs.as<float>(), tiles_x, tiles_y, rw.rec.as<float>(),
                                                           rw.counts.as<uint32_t>(), rw.rects.as<uint2>());
  NPS_CHECK_LAUNCH();
  uint32_t* total = rw.total.as<uint32_t>();
  NPS_TRY(exclusive_scan_u32(rw.counts.as<uint32_t>(), rw.offsets.as<uint32_t>(), n, total, rw.sw, s));
  uint32_t K = 0;
  NPS_CUDA(cudaMemcpyAsync(&K, total, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  if (K > rw.pair_cap || rw.pair_cap == 0) {
    const uint32_t cap = K + K / 4 + 4096;
    NPS_TRY(rw.keys.ensure(sizeof(uint32_t) * (size_t)cap));
    NPS_TRY(rw.vals.ensure(sizeof(uint32_t) * (size_t)cap));
    rw.pair_cap = cap;
  }
  uint32_t* rstart = rw.ranges.as<uint32_t>();
  uint32_t* rend = rstart + num_tiles;
  NPS_CUDA(cudaMemsetAsync(rstart, 0, sizeof(uint32_t) * 2 * num_tiles, s));
  const uint32_t* vs = rw.vals.as<uint32_t>();
  if (K > 0) {
    bin::k_emit<<<div_up(n, 256), 256, 0, s>>>(rw.counts.as<uint32_t>(), rw.offsets.as<uint32_t>(),
                                                rw.rects.as<uint2>(), n, 1, tiles_x, num_tiles, rw.pair_cap,
                                                rw.keys.as<uint32_t>(), rw.vals.as<uint32_t>());
    NPS_CHECK_LAUNCH();
    int bits = 1;
    while ((1ull << bits) < (uint64_t)num_tiles) ++bits;
    uint32_t *ks = nullptr, *vv = nullptr;
    NPS_TRY(radix_sort_u32(rw.keys.as<uint32_t>(), rw.vals.as<uint32_t>(), total, rw.pair_cap, bits, rw.sw, s, &ks,
                           &vv));
    bin::k_ranges<<<4 * kNumSMs, 256, 0, s>>>(ks, total, rw.pair_cap, rstart, rend);
    NPS_CHECK_LAUNCH();
    vs = vv;
  }
  compat::k_render_raster<<<dim3(tiles_x, tiles_y), 256, 0, s>>>(rw.rec.as<float>(), vs, rstart, rend, w, h, tiles_x,
                                                                  (float4*)out_rgba, (float4*)out_depth, load);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

extern "C" int nps_splat_opt_render(nps_splat_opt* o, const float* vp, uint32_t w, uint32_t h, float* out_rgba,
                                    float* out_depth) {
  return splat_render(o, vp, w, h, out_rgba, out_depth, 0);
}

extern "C" int nps_splat_opt_render_load(nps_splat_opt* o, const float* vp, uint32_t w, uint32_t h, float* rgba,
                                         float* depth) {
  return splat_render(o, vp, w, h, rgba, depth, 1);
}

// ============================================ ADC without device allocation
// Some callers cannot let a library allocate device memory: an application
// that hands its whole device-memory budget to its own arena or pool (a
// cudaMalloc from the library would fail or break its accounting), or one that
// shares the GPU with latency-critical work such as a render loop, where
// cudaMalloc / cudaFree may synchronise the device and stall that work.
// nps_splat_adc_noalloc runs the splat ADC (splat_adc.wgsl:28-87) on buffers
// the caller owns, with the kernel's scratch (the dead-slot list and a result
// word) in a fixed array compiled into the library.

namespace {
constexpr uint32_t kNoAllocMaxSplats = 262144;  // 1 MiB of dead-slot list
// Scratch for nps_splat_adc_noalloc: [0, kNoAllocMaxSplats) dead-slot list,
// then 64 words of results.  Every GPU that loads the library holds it until
// exit.  Host code must not use this name as a device address (it is a host
// stand-in); the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint32_t g_adc_scratch[kNoAllocMaxSplats + 64];

constexpr int kMaxDevices = 64;
uint32_t* g_adc_scratch_dev[kMaxDevices] = {nullptr};
std::mutex g_adc_scratch_mu;

// The scratch array's device address on the current device (looked up once
// per device, with that device current).
int adc_scratch_address(uint32_t** out) {
  int dev = 0;
  NPS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("splat_adc_noalloc: device %d beyond %d supported", dev, kMaxDevices);
    return NPS_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_adc_scratch_mu);
  if (!g_adc_scratch_dev[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_adc_scratch);
    if (e != cudaSuccess || !p) {
      set_error("splat_adc_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev, cudaGetErrorString(e));
      return NPS_ERR_CUDA;
    }
    g_adc_scratch_dev[dev] = (uint32_t*)p;
  }
  *out = g_adc_scratch_dev[dev];
  return NPS_OK;
}
}  // namespace

extern "C" int nps_splat_adc_noalloc(float* splats, float* adam_m, float* adam_v, float* grad_accum, uint32_t n,
                                     float adam_t, void* cuda_stream, uint32_t* clones_host) {
  if (!splats || !adam_m || !adam_v || !grad_accum || n == 0) {
    set_error("splat_adc_noalloc: null buffer or zero splats");
    return NPS_ERR_INVALID;
  }
  if (n > kNoAllocMaxSplats) {
    set_error("splat_adc_noalloc: %u splats exceed the fixed scratch of %u (use nps_splat_opt_adc)", n,
              kNoAllocMaxSplats);
    return NPS_ERR_CAPACITY;
  }
  // the kernel moves whole records as float4 (16-byte loads and stores) and
  // the accumulators as floats: an offset view that breaks either alignment
  // is rejected here rather than faulting on the device
  if ((((uintptr_t)splats | (uintptr_t)adam_m | (uintptr_t)adam_v) & 15u) != 0 || ((uintptr_t)grad_accum & 3u) != 0) {
    set_error("splat_adc_noalloc: splats, adam_m and adam_v must be 16-byte aligned, grad_accum 4-byte aligned");
    return NPS_ERR_INVALID;
  }
  uint32_t* scratch = nullptr;
  NPS_TRY(adc_scratch_address(&scratch));
  cudaStream_t s = (cudaStream_t)cuda_stream;
  uint32_t* stats = scratch + kNoAllocMaxSplats;
  // no clearing needed: the kernel writes the dead-slot list before reading
  // it, and writes the result word at its end on every call
  compat::k_adc<<<1, compat::kAdcThreads, 0, s>>>(splats, adam_m, adam_v, grad_accum, scratch, n, adam_t, stats);
  NPS_CHECK_LAUNCH();
  if (clones_host) {
    NPS_CUDA(cudaMemcpyAsync(clones_host, stats, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    NPS_CUDA(cudaStreamSynchronize(s));
  }
  return NPS_OK;
}
