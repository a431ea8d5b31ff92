// gs.cu — batched multi-view 3D Gaussian trainer (forward, L1 + D-SSIM loss,
// backward, Adam) for sm_100a.
//
// One train step over V views is a fixed sequence of launches, each covering
// all views at once:
//   k_preprocess   (view, Gaussian): projection, EWA 2D covariance, conic,
//                  tile rectangle of the alpha >= 1/255 ellipse, SH colour,
//                  depth key
//   radix sort     32-bit depth keys of all (view, Gaussian) records
//   k_gather_counts + scan + k_emit: (view * tiles + tile, record) pairs
//                  written in depth order
//   radix sort     stable by tile key -> every tile list is depth ordered
//   k_ranges       tile list bounds
//   k_fwd          one CTA per (tile, view): records staged in shared memory
//                  256 at a time, warps skip records whose footprint misses
//                  their two pixel rows, front-to-back compositing with alpha
//                  clamp 0.99, 1/255 skip and early termination at T < 1e-4
//                  (block-wide vote ends the tile), final T and last
//                  contributor stored per pixel (O(pixels) state, no
//                  per-pair state)
//   k_ssim_fwd2 / k_ssim_bwd2 / k_loss_reduce: (1 - l) L1 + l (1 - SSIM), 11x11
//                  Gaussian window (sigma 1.5), l = 0.2, and dL/dimage
//   k_bwd2         reverse traversal replaying transmittance from the final
//                  T, two pixels per thread, per-Gaussian gradients summed
//                  over the warp by a 16-shuffle reduce-scatter, then over the
//                  CTA in shared memory, then one global atomic per (tile,
//                  Gaussian, value); k_bwd<true> + k_det_segsum: the
//                  deterministic two-pass variant
//   k_project_bwd  eight lanes per Gaussian over the views: screen-space
//                  gradients -> parameter gradients, ADC statistics
//   k_adam         fused Adam over the 59 parameters of every Gaussian
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bulk.cuh"
#include "common.cuh"
#include "context.h"
#include "gs_math.cuh"

namespace nps {
namespace gs {

using namespace gsm;

constexpr int kThreads = 256;
constexpr float kLowpass = 0.3f;       // px^2 added to the 2D covariance diagonal
constexpr float kNear = 0.2f;          // cull Gaussians closer than this (view depth)
constexpr float kAlphaMin = 1.0f / 255.0f;
constexpr float kAlphaMax = 0.99f;
constexpr float kTMin = 1e-4f;
constexpr int kG2 = 12;                // floats per screen-space gradient record
constexpr int kSsimWin = 11;
constexpr float kSsimC1 = 0.01f * 0.01f, kSsimC2 = 0.03f * 0.03f;

__constant__ float c_ssim_w[kSsimWin];

struct Rec {  // projected record, 3 x float4 = 48 B
  float4 a;   // u, v, conic a, conic b
  float4 b;   // conic c, opacity, r, g
  float4 c;   // b, level t2 of the alpha >= 1/255 ellipse (q(d) <= t2), half-extents (x, y) of its box
};

// True if the alpha >= 1/255 ellipse of the record misses the pixel-centre
// rectangle [x0, x0 + w] x [y0, y0 + h]: its box misses, or the smallest
// value of q(d) = ca dx^2 + 2 cb dx dy + cc dy^2 over the rectangle (offsets
// from the centre) exceeds the level t2.  A conservative skip test: the
// level carries the footprint's margin.
__device__ __forceinline__ bool rec_misses_box(const float4& a, float cc, const float4& c, float x0, float y0,
                                               float w, float h) {
  if ((a.x + c.z < x0) || (a.x - c.z > x0 + w) || (a.y + c.w < y0) || (a.y - c.w > y0 + h)) return true;
  const float lx = x0 - a.x, hx = x0 + w - a.x, ly = y0 - a.y, hy = y0 + h - a.y;
  if (lx <= 0.0f && hx >= 0.0f && ly <= 0.0f && hy >= 0.0f) return false;  // centre inside
  const float ca = a.z, cb = a.w;
  // the form's minimum on each edge (the other coordinate clamped to the edge)
  const float icc = cc > 0.0f ? 1.0f / cc : 0.0f, ica = ca > 0.0f ? 1.0f / ca : 0.0f;
  const float y_l = fminf(fmaxf(-cb * lx * icc, ly), hy), y_h = fminf(fmaxf(-cb * hx * icc, ly), hy);
  const float x_l = fminf(fmaxf(-cb * ly * ica, lx), hx), x_h = fminf(fmaxf(-cb * hy * ica, lx), hx);
  const float q1 = ca * lx * lx + 2.0f * cb * lx * y_l + cc * y_l * y_l;
  const float q2 = ca * hx * hx + 2.0f * cb * hx * y_h + cc * y_h * y_h;
  const float q3 = ca * x_l * x_l + 2.0f * cb * x_l * ly + cc * ly * ly;
  const float q4 = ca * x_h * x_h + 2.0f * cb * x_h * hy + cc * hy * hy;
  return fminf(fminf(q1, q2), fminf(q3, q4)) > c.y;
}

#ifndef NPS_GS_SOLO
#define NPS_GS_SOLO 0
#endif
#ifndef NPS_GS_STRIP_W
#define NPS_GS_STRIP_W 8
#endif
// Thread-to-pixel map of the 16 x 16 tile kernels (forms 0 and 2): thread tid
// shades PPT vertically adjacent pixels from (x, y) of the tile, and its warp
// covers a kW x kH strip at (wx, wy), the region its per-warp culling tests.
// NPS_GS_STRIP_W 8 (default): the strips closest to square, 8 x 4 (PPT 1),
// 8 x 8 (PPT 2) and 16 x 8 (PPT 4), so a small footprint meets fewer warps
// (backward -9%, forward -5% at 200k Gaussians, 800 x 800, 8 views, PPT 2,
// against 16 x 4); 16: full-width 16 x 2·PPT strips.
template <int PPT>
struct TileMap16 {
  static constexpr int kW = (NPS_GS_STRIP_W == 8 && PPT == 4) ? 16 : NPS_GS_STRIP_W, kH = 32 * PPT / kW;
  static constexpr int kWarpsX = 16 / kW;
  static_assert(kW == 16 || kW == 8, "strip width");
  __device__ static uint32_t wx(uint32_t tid) { return ((tid >> 5) % kWarpsX) * kW; }
  __device__ static uint32_t wy(uint32_t tid) { return ((tid >> 5) / kWarpsX) * kH; }
  __device__ static uint32_t x(uint32_t tid) { return wx(tid) + (tid & (kW - 1)); }
  __device__ static uint32_t y(uint32_t tid) { return wy(tid) + PPT * ((tid & 31) / kW); }
};

// Exponent of the Gaussian at offset d = (dx, dy) from its centre, -q(d) / 2
// with q(d) = dx u + dy w and (u, w) the conic (a.z, a.w; a.w, cc) times d.
// Every raster kernel evaluates it in this one order, so the forward and the
// backward take the same alpha >= 1/255 decisions; u and w are reused by the
// backward's mean gradient.
__device__ __forceinline__ float gs_power(const float4& a, float cc, float dx, float dy, float& u, float& w) {
  u = fmaf(a.w, dy, a.z * dx);
  w = fmaf(cc, dy, a.w * dx);
  return -0.5f * fmaf(dy, w, dx * u);
}

// true if the Gaussian's alpha >= 1/255 box misses the warp's pixels
// (rows y0, y0 + 1 and columns x0 .. x0 + 15)
__device__ __forceinline__ bool warp_misses(float u, float v, float ex, float ey, float x0, float y0) {
  return (u + ex < x0) || (u - ex > x0 + 15.0f) || (v + ey < y0) || (v - ey > y0 + 1.0f);
}

// Sum of 16 values over the warp by recursive halving (reduce-scatter): 16
// shuffles instead of 5 per value.  On return, lanes 2k and 2k+1 hold the
// warp total of value k.
__device__ __forceinline__ float warp_sum16(float (&v)[16], uint32_t lane) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float send = b4 ? v[j] : v[j + 8], keep = b4 ? v[j + 8] : v[j];
    v[j] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float send = b3 ? v[j] : v[j + 4], keep = b3 ? v[j + 4] : v[j];
    v[j] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const float send = b2 ? v[j] : v[j + 2], keep = b2 ? v[j + 2] : v[j];
    v[j] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  {
    const float send = b1 ? v[0] : v[1], keep = b1 ? v[1] : v[0];
    v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  }
  return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// Sum of 9 values over the warp by uneven recursive halving: at each level a
// lane keeps the first ceil(m/2) of its m partial values (lower half of the
// lane pair) or the rest (upper half, padded with a zero), 5 + 3 + 2 + 1 + 1
// = 12 shuffles.  On return, lanes 2q and 2q + 1 hold the warp total of value
// warp_sum9_index(lane) when that is below 9 (every value has one q).
__device__ __forceinline__ float warp_sum9(const float (&v)[9], uint32_t lane) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
  float w[5], x[3], y[2];
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    const float hi = j + 5 < 9 ? v[j + 5] : 0.0f;
    const float send = b4 ? v[j] : hi, keep = b4 ? hi : v[j];
    w[j] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const float hi = j + 3 < 5 ? w[j + 3] : 0.0f;
    const float send = b3 ? w[j] : hi, keep = b3 ? hi : w[j];
    x[j] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const float hi = j + 2 < 3 ? x[j + 2] : 0.0f;
    const float send = b2 ? x[j] : hi, keep = b2 ? hi : x[j];
    y[j] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
  const float send = b1 ? y[0] : y[1], keep = b1 ? y[1] : y[0];
  const float z = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  return z + __shfl_xor_sync(0xffffffffu, z, 1);
}

// The value whose total warp_sum9 leaves in this lane; 15 for a padding slot.
// Nibble q of the table is the index kept by lanes 2q, 2q + 1 (the
// partition above traced through its four uneven levels).
__device__ __forceinline__ uint32_t warp_sum9_index(uint32_t lane) {
  return (uint32_t)(0xfff8f765ff43f210ull >> (4u * ((lane >> 1) & 15u))) & 15u;
}

__device__ __forceinline__ float sigmoidf(float x) { return 1.0f / (1.0f + expf(-x)); }

// ------------------------------------------------------------ preprocess
template <int DEG>
__global__ void __launch_bounds__(256) k_preprocess(const float* __restrict__ params, uint32_t n,
                                                    const float* __restrict__ views, uint32_t nv, uint32_t W,
                                                    uint32_t H, uint32_t tiles_x, uint32_t tiles_y, float inv_tile,
                                                    Rec* __restrict__ recs, uint32_t* __restrict__ counts,
                                                    uint2* __restrict__ rects, uint32_t* __restrict__ dkeys,
                                                    uint32_t* __restrict__ dvals, uint32_t* __restrict__ ecounts,
                                                    uint32_t* __restrict__ tmasks) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nv * n) return;
  const uint32_t v = g / n, i = g - v * n;
  // the record in 16-byte loads (floats 0..11, then the SH coefficients if visible)
  const float4* p4 = reinterpret_cast<const float4*>(params + (size_t)i * kP);
  const float4 q0 = p4[0], q1 = p4[1], q2 = p4[2];
  const float* view = views + (size_t)v * kViewRec;
  float mean[3] = {q0.x, q0.y, q0.z};
  float ls[3] = {q0.w, q1.x, q1.y};
  float q[4] = {q1.z, q1.w, q2.x, q2.y};
  Proj<float> P;
  project<float>(view, mean, ls, q, (float)W, (float)H, kLowpass, P);
  uint32_t cnt = 0, ecnt = 0, tmask = 0;
  uint2 rect = make_uint2(0, 0);
  uint32_t key = 0xffffffffu;
  Rec r;
  r.a = make_float4(0, 0, 0, 0);
  r.b = make_float4(0, 0, 0, 0);
  r.c = make_float4(0, 0, 0, 0);
  const float op = sigmoidf(q2.z);  // opacity logit, float 10
  // A pixel contributes only where o * G >= 1/255, i.e. inside the ellipse
  // d^T Sigma^-1 d <= t2 = 2 ln(255 o).  Its axis-aligned box, centre +-
  // sqrt(t2 * Sigma_xx), +- sqrt(t2 * Sigma_yy), bounds the tile rectangle and
  // the per-warp culling (1% margin on t2 for rounding).
  if (P.cw > kNear && P.det > 0.0f && op * 255.0f > 1.0f) {
    const float t2 = 2.0f * logf(255.0f * op) * 1.01f;
    const float ex = sqrtf(t2 * P.A), ey = sqrtf(t2 * P.C);
    const int x0 = max(0, min((int)tiles_x, (int)floorf((P.u - ex) * inv_tile)));
    const int x1 = max(0, min((int)tiles_x, (int)floorf((P.u + ex) * inv_tile) + 1));
    const int y0 = max(0, min((int)tiles_y, (int)floorf((P.v - ey) * inv_tile)));
    const int y1 = max(0, min((int)tiles_y, (int)floorf((P.v + ey) * inv_tile) + 1));
    if (x1 > x0 && y1 > y0) {
      cnt = (uint32_t)((x1 - x0) * (y1 - y0));
      rect = make_uint2((uint32_t)x0 | ((uint32_t)x1 << 16), (uint32_t)y0 | ((uint32_t)y1 << 16));
      key = __float_as_uint(P.cw);  // positive floats order like their bit patterns
      // SH colour for the view direction
      const float dx = mean[0] - view[32], dy = mean[1] - view[33], dz = mean[2] - view[34];
      const float il = rsqrtf(fmaxf(dx * dx + dy * dy + dz * dz, 1e-20f));
      float basis[16];
      sh_basis<float>(DEG, dx * il, dy * il, dz * il, basis);
      constexpr int nb = (DEG + 1) * (DEG + 1);
      float sh[(3 * nb + 3) / 4 * 4];
#pragma unroll
      for (int k4 = 0; k4 < (3 * nb + 3) / 4; ++k4) {
        const float4 t = p4[3 + k4];
        sh[4 * k4] = t.x; sh[4 * k4 + 1] = t.y; sh[4 * k4 + 2] = t.z; sh[4 * k4 + 3] = t.w;
      }
      float col[3] = {0.5f, 0.5f, 0.5f};
#pragma unroll
      for (int k = 0; k < nb; ++k) {
        col[0] += basis[k] * sh[3 * k + 0];
        col[1] += basis[k] * sh[3 * k + 1];
        col[2] += basis[k] * sh[3 * k + 2];
      }
      r.a = make_float4(P.u, P.v, P.ca, P.cb);
      r.b = make_float4(P.cc, op, fmaxf(col[0], 0.0f), fmaxf(col[1], 0.0f));
      // c.y: the alpha >= 1/255 level of the conic form (same 1% margin), for exact per-warp culling
      r.c = make_float4(fmaxf(col[2], 0.0f), t2 + 1e-4f, ex, ey);
      // Pairs are emitted only for the tiles of the box whose pixel-centre
      // square the alpha >= 1/255 ellipse meets, for boxes of at most 32
      // tiles; a tile the ellipse misses gets no contribution from this
      // Gaussian, so the images are unchanged and the lists shorter.  Per tile
      // row, the ellipse's x-extent over the row's pixel-centre band
      // [y, y + T - 1] is exact: the left boundary x = k dy - hw(dy) (k =
      // Sigma_xy / Sigma_yy, hw^2 = (t2 - dy^2 / Sigma_yy) det / Sigma_yy) is
      // convex in dy with its minimum at the leftmost point dy = -Sigma_xy
      // sqrt(t2 / Sigma_xx), so the band's minimum is there clamped to the
      // band (the right boundary mirrors it); widened by 1e-3 px + 1e-6 |u|
      // for rounding.  The tiles of the row meeting that extent are set in a
      // 32-bit mask, row-major over the box.
      ecnt = cnt;
      if (cnt <= 32) {
        const float T = 1.0f / inv_tile, tm1 = T - 1.0f;
        const float kx = P.B / P.C, hw2 = P.det / P.C, ic = 1.0f / P.C;
        const float dyx = P.B * sqrtf(t2 / P.A), eps = 1e-3f + 1e-6f * fabsf(P.u);
        const uint32_t w = (uint32_t)(x1 - x0);
        for (int ty = y0; ty < y1; ++ty) {
          const float ly = fmaxf((float)ty * T - P.v, -ey), hy = fminf((float)ty * T + tm1 - P.v, ey);
          if (ly > hy) continue;
          const float dl = fminf(fmaxf(-dyx, ly), hy), dr = fminf(fmaxf(dyx, ly), hy);
          const float xl = P.u + kx * dl - sqrtf(fmaxf(t2 - dl * dl * ic, 0.0f) * hw2) - eps;
          const float xr = P.u + kx * dr + sqrtf(fmaxf(t2 - dr * dr * ic, 0.0f) * hw2) + eps;
          const int c0 = max(x0, (int)ceilf((xl - tm1) * inv_tile)), c1 = min(x1, (int)floorf(xr * inv_tile) + 1);
          if (c1 > c0) tmask |= ((c1 - c0 == 32) ? 0xffffffffu : ((1u << (c1 - c0)) - 1u))
                                << ((uint32_t)(ty - y0) * w + (uint32_t)(c0 - x0));
        }
        ecnt = (uint32_t)__popc(tmask);
      }
    }
  }
  recs[g] = r;
  counts[g] = cnt;
  ecounts[g] = ecnt;
  tmasks[g] = tmask;
  rects[g] = rect;
  dkeys[g] = key;
  dvals[g] = g;
}

__global__ void k_gather_counts(const uint32_t* __restrict__ sorted_g, const uint32_t* __restrict__ counts,
                                uint32_t m, uint32_t* __restrict__ out) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < m) out[j] = counts[sorted_g[j]];
}

// One warp per 32 consecutive depth-sorted (view, Gaussian) entries: their
// pairs are one contiguous output range, written 32 consecutive slots at a
// time (coalesced); each lane finds the entry owning its slot by a binary
// search over the warp's offsets (shuffles).  Output identical to writing
// each entry's tile rectangle row by row.
__global__ void __launch_bounds__(256) k_emit(const uint32_t* __restrict__ sorted_g,
                                              const uint32_t* __restrict__ ecounts,
                                              const uint32_t* __restrict__ offsets, const uint2* __restrict__ rects,
                                              const uint32_t* __restrict__ tmasks, uint32_t m, uint32_t n,
                                              uint32_t tiles_x, uint32_t num_tiles, uint32_t cap,
                                              uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31;
  if (__all_sync(0xffffffffu, j >= m)) return;
  uint32_t g = 0, c = 0, off = 0xffffffffu, x0 = 0, w = 1, y0 = 0, tm = 0;
  if (j < m) {
    g = sorted_g[j];
    c = ecounts[g];
    off = offsets[j];
    const uint2 r = rects[g];
    x0 = r.x & 0xffffu;
    w = max((r.x >> 16) - x0, 1u);
    y0 = r.y & 0xffffu;
    // boxes of at most 32 tiles emit only the tiles of their mask
    if (((r.y >> 16) - y0) * ((r.x >> 16) - x0) <= 32u) tm = tmasks[g];
    else tm = 0xffffffffu;
  }
  const uint32_t start = __shfl_sync(0xffffffffu, off, 0);
  const uint32_t end = __reduce_max_sync(0xffffffffu, j < m ? off + c : 0u);
  for (uint32_t base = start; base < end; base += 32) {
    const uint32_t sl = base + lane;
    // largest lane whose offset <= sl (lanes past m carry offset ~0u)
    uint32_t L = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1) {
      const uint32_t o2 = __shfl_sync(0xffffffffu, off, L + step);
      if (o2 <= sl) L += step;
    }
    const uint32_t gL = __shfl_sync(0xffffffffu, g, L), oL = __shfl_sync(0xffffffffu, off, L);
    const uint32_t x0L = __shfl_sync(0xffffffffu, x0, L), wL = __shfl_sync(0xffffffffu, w, L);
    const uint32_t y0L = __shfl_sync(0xffffffffu, y0, L), tmL = __shfl_sync(0xffffffffu, tm, L);
    if (sl < end && sl < cap) {
      uint32_t local = sl - oL;
      if (tmL != 0xffffffffu) {
        // the local-th set bit of the mask is the tile's index in the box
        uint32_t mk = tmL;
        for (uint32_t t = 0; t < local; ++t) mk &= mk - 1u;
        local = (uint32_t)(__ffs(mk) - 1);
      }
      const uint32_t ry = local / wL;
      keys[sl] = (gL / n) * num_tiles + (y0L + ry) * tiles_x + x0L + (local - ry * wL);
      vals[sl] = gL;
    }
  }
}

// Four consecutive sorted keys per thread from one 16-byte load (the key
// buffers are 256-byte aligned), with the neighbours on either side.
__global__ void k_ranges(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ total, uint32_t cap,
                         uint32_t* __restrict__ rstart, uint32_t* __restrict__ rend) {
  const uint32_t K = min(*total, cap);
  const uint32_t n4 = (K + 3) / 4;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += gridDim.x * blockDim.x) {
    const uint32_t p0 = 4 * q;
    uint32_t k[4];
    if (p0 + 3 < K) {
      const uint4 v = __ldg(reinterpret_cast<const uint4*>(keys) + q);
      k[0] = v.x; k[1] = v.y; k[2] = v.z; k[3] = v.w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) k[j] = p0 + j < K ? __ldg(keys + p0 + j) : 0u;
    }
    const uint32_t prev = p0 > 0 ? __ldg(keys + p0 - 1) : 0u;
    const uint32_t next = p0 + 4 < K ? __ldg(keys + p0 + 4) : 0u;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t p = p0 + j;
      if (p >= K) break;
      const uint32_t before = j == 0 ? prev : k[j - 1], after = j == 3 ? next : k[j + 1];
      if (p == 0 || before != k[j]) rstart[k[j]] = p;
      if (p == K - 1 || after != k[j]) rend[k[j]] = p + 1;
    }
  }
}

// ------------------------------------------------------------ forward raster
// ---- record staging with bulk asynchronous copies (double-buffered)
// Each staged record (48 B, 16-byte aligned in global and shared memory) is one
// cp.async.bulk global -> shared completing on the buffer's mbarrier; thread 0
// posts the batch's byte count.  Waits are bounded: on a timeout the kernel
// records it in *err and carries on (the batch is then undefined).
using namespace nps::bulk;
// stage records vals[b0 .. b0 + nb) into buf (thread t copies records t,
// t + blockDim.x, ...)
__device__ __forceinline__ void stage_batch(const Rec* __restrict__ recs, const uint32_t* __restrict__ vals,
                                            uint32_t b0, uint32_t nb, Rec* buf, uint64_t* bar, uint32_t* gidx) {
  if (threadIdx.x == 0) mbar_expect_tx(bar, nb * (uint32_t)sizeof(Rec));
  if (threadIdx.x < nb)
    // this buffer was last read through the generic proxy (before a barrier)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) {
    const uint32_t g = vals[b0 + i];
    if (gidx) gidx[i] = g;
    bulk_g2s(buf + i, recs + g, (uint32_t)sizeof(Rec), bar);
  }
}

// Forward raster, PPT vertically adjacent pixels per thread: 256 / PPT
// threads per 16 x 16 tile, a warp covers a 16 x 2·PPT strip, records staged
// SB = SPS · 256 / PPT at a time.  (PPT, SB) is the autotuned variant.
// kOrd: a 1D grid whose block b takes work item order[b] (longest tile
// lists first), else the grid is (tiles x, tiles y, views).  With 1 or 2
// pixels per thread at most 51 registers: ten 128-thread blocks per SM (the
// shared-memory limit) instead of nine.
template <int PPT, int SPS, bool kOrd>
__global__ void __launch_bounds__(256 / PPT, PPT <= 2 ? 1280 / (256 / PPT) : 1) k_fwd(const Rec* __restrict__ recs, const uint32_t* __restrict__ vals,
                                                   const uint32_t* __restrict__ rstart,
                                                   const uint32_t* __restrict__ rend, uint32_t W, uint32_t H,
                                                   uint32_t tiles_x, uint32_t num_tiles, float3 bg,
                                                   float4* __restrict__ img, uint32_t* __restrict__ ncontrib,
                                                   uint32_t* __restrict__ tile_last, uint32_t* __restrict__ err,
                                                   const uint32_t* __restrict__ order) {
  constexpr int NT = 256 / PPT, SB = NT * SPS;
  static_assert(SB <= 256, "staging buffers beyond the static shared-memory budget");
  __shared__ __align__(16) Rec s_rec[2][SB];
  __shared__ __align__(8) uint64_t s_bar[2];
  uint32_t tx = blockIdx.x, ty = blockIdx.y, v = blockIdx.z;
  if constexpr (kOrd) {
    const uint32_t it = order[blockIdx.x];
    v = it / num_tiles;
    const uint32_t tile = it - v * num_tiles;
    ty = tile / tiles_x;
    tx = tile - ty * tiles_x;
  }
  const uint32_t tid = threadIdx.x;
  using TM = TileMap16<PPT>;
  const uint32_t px = tx * 16 + TM::x(tid), py = ty * 16 + TM::y(tid);
  const float fx = (float)px;
  const float wx0 = (float)(tx * 16 + TM::wx(tid)), wy0 = (float)(ty * 16 + TM::wy(tid));
  constexpr float ww = (float)(TM::kW - 1), wh = (float)(TM::kH - 1);
  const uint32_t key = v * num_tiles + ty * tiles_x + tx;
  const uint32_t start = rstart[key], end = rend[key];
  float T[PPT], C0[PPT], C1[PPT], C2[PPT];
  uint32_t last[PPT];
  bool dn[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    T[k] = 1.0f; C0[k] = C1[k] = C2[k] = 0.0f; last[k] = 0;
    dn[k] = !(px < W && py + k < H);
  }
#define NPS_ALL_DONE(d)                      \
  do {                                       \
    d = true;                                \
    _Pragma("unroll") for (int k_ = 0; k_ < PPT; ++k_) d = d && dn[k_]; \
  } while (0)
  __shared__ uint32_t s_abort;
  if (tid == 0) {
    s_abort = 0u;
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const uint32_t nbatch = (end - start + SB - 1) / SB;
  if (nbatch > 0) stage_batch(recs, vals, start, min((uint32_t)SB, end - start), s_rec[0], &s_bar[0], nullptr);
  bool pending_next = false;
  for (uint32_t bi = 0; bi < nbatch; ++bi) {
    const uint32_t base = start + bi * SB, buf = bi & 1u;
    const uint32_t nb = min((uint32_t)SB, end - base);
    // prefetch the next batch into the other buffer (read two batches ago)
    pending_next = bi + 1 < nbatch;
    if (pending_next)
      stage_batch(recs, vals, base + SB, min((uint32_t)SB, end - base - SB), s_rec[buf ^ 1u], &s_bar[buf ^ 1u],
                  nullptr);
    if (!mbar_wait(&s_bar[buf], (bi >> 1) & 1u)) s_abort = 1u;  // the batch is undefined: end the tile below
    const Rec* sr = s_rec[buf];
    // staged pairs whose alpha >= 1/255 box meets the warp's strip (one lane
    // tests SB / 32 pairs; the warp then walks the set bits in order)
    uint32_t hit[SB / 32];
#pragma unroll
    for (int qq = 0; qq < SB / 32; ++qq) {
      const uint32_t jj = qq * 32 + (tid & 31);
      bool h = false;
      if (jj < nb) h = !rec_misses_box(sr[jj].a, sr[jj].b.x, sr[jj].c, wx0, wy0, ww, wh);
      hit[qq] = __ballot_sync(0xffffffffu, h);
    }
    bool done;
    NPS_ALL_DONE(done);
#pragma unroll
    for (int qq = 0; qq < SB / 32; ++qq)
    for (uint32_t m = hit[qq]; m != 0u && !done;) {
      const int bit = __ffs(m) - 1;
      m &= m - 1u;
      const uint32_t j = qq * 32 + bit;
      const float4 a = sr[j].a;
      const float4 c4 = sr[j].c;
      const float4 b = sr[j].b;
      const float dx = a.x - fx, pmin = -0.5f * c4.y;
#pragma unroll
      for (int k = 0; k < PPT; ++k) {
        if (dn[k]) continue;
        const float dy = a.y - (float)(py + k);
        float cu, cw;
        const float power = gs_power(a, b.x, dx, dy, cu, cw);
        if (power > 0.0f || power < pmin) continue;  // pmin: alpha < 1/255 below it (see pix_bwd_pair)
        const float alpha = fminf(kAlphaMax, b.y * __expf(power));
        if (alpha < kAlphaMin) continue;
        const float test_T = T[k] * (1.0f - alpha);
        if (test_T < kTMin) {
          dn[k] = true;
          continue;
        }
        const float w = alpha * T[k];
        C0[k] += b.z * w;
        C1[k] += b.w * w;
        C2[k] += c4.x * w;
        T[k] = test_T;
        last[k] = base - start + j + 1;
      }
      NPS_ALL_DONE(done);
    }
    // every pixel of the tile done: stop (after the prefetch in flight lands)
    NPS_ALL_DONE(done);
    if (__syncthreads_count(done) == NT || s_abort) {
      if (pending_next && !mbar_wait(&s_bar[buf ^ 1u], ((bi + 1) >> 1) & 1u)) s_abort = 1u;
      // a batch whose wait gave up may still have copies in flight: wait again (bounded)
      if (s_abort) (void)mbar_wait(&s_bar[buf], (bi >> 1) & 1u);
      break;
    }
  }
  __syncthreads();
  if (s_abort) {
    // a bounded wait gave up: the tile's outputs are not written (the step reports NPS_ERR_TIMEOUT)
    if (tid == 0) atomicAdd(err, 1u);
    return;
  }
  uint32_t wmax = 0;
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    if (px < W && py + k < H) {
      const size_t pix = ((size_t)v * H + py + k) * W + px;
      img[pix] = make_float4(C0[k] + T[k] * bg.x, C1[k] + T[k] * bg.y, C2[k] + T[k] * bg.z, T[k]);
      ncontrib[pix] = last[k];
    }
    wmax = max(wmax, last[k]);
  }
  // the tile's last contributor over its pixels (the backward's batch range)
  wmax = __reduce_max_sync(0xffffffffu, wmax);
  if ((tid & 31) == 0 && wmax > 0) atomicMax(tile_last + key, wmax);
#undef NPS_ALL_DONE
}

// ------------------------------------------------------------ loss
// (1 - l) * mean|x - y| + l * (1 - mean SSIM), averaged over views.
// k_ssim_fwd2 writes, per pixel and channel, the three maps whose Gaussian
// correlation gives dL/dx, plus per-block partial sums of |x - y| and SSIM;
// k_ssim_bwd2 correlates the maps and adds the L1 term.
//
// 32 x 32 output tiles (input span 42 x 42), zero padding outside the image,
// register-blocked separable window: the horizontal pass runs 4 consecutive
// outputs of a row from 14 inputs held in registers, the vertical pass 4
// consecutive rows of a column.  The gradient maps are planar (V x 9 x H x W)
// so the backward's halo loads are coalesced.
constexpr int kHalo = kSsimWin / 2;
constexpr int kLT = 32, kLI = kLT + 2 * kHalo, kLS = kLI + 1;  // 32, 42, row stride 43
constexpr int kHS = kLT + 1;                                    // row stride of the horizontal sums
constexpr size_t kSsimFwdSmem = sizeof(float) * (2 * 3 * kLI * kLS + 5 * kLI * kHS);
constexpr size_t kSsimBwdSmem = sizeof(float) * (3 * kLI * kLS + 3 * kLI * kHS);

__global__ void __launch_bounds__(256) k_ssim_fwd2(const float4* __restrict__ img, const float4* __restrict__ tgt,
                                                   const uint32_t* __restrict__ tgt_ids, uint32_t W, uint32_t H,
                                                   float lambda, float inv_norm, float* __restrict__ maps,
                                                   float* __restrict__ partial) {
  extern __shared__ float sm[];
  float* sx = sm;                        // [3][kLI][kLS]
  float* sy = sx + 3 * kLI * kLS;        // [3][kLI][kLS]
  float* hm = sy + 3 * kLI * kLS;        // [5][kLI][kHS]
  __shared__ float red[2][8];
  const uint32_t v = blockIdx.z, tid = threadIdx.x;
  const int ox = blockIdx.x * kLT - kHalo, oy = blockIdx.y * kLT - kHalo;
  const float4* im = img + (size_t)v * W * H;
  const float4* tg = tgt + (size_t)tgt_ids[v] * W * H;
  // staging in two halves, each issuing all its loads before its stores, so
  // the load latency is paid twice rather than once per element
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    constexpr int kIt = (kLI * kLI + 511) / 512;  // 4 elements per thread per half
    float4 a[kIt], b[kIt];
#pragma unroll
    for (int i = 0; i < kIt; ++i) {
      const int e = tid + (half * kIt + i) * 256;
      const int ly = e / kLI, lx = e - ly * kLI;
      const int gx = ox + lx, gy = oy + ly;
      a[i] = b[i] = make_float4(0, 0, 0, 0);
      if (e < kLI * kLI && gx >= 0 && gy >= 0 && gx < (int)W && gy < (int)H) {
        a[i] = im[(size_t)gy * W + gx];
        b[i] = tg[(size_t)gy * W + gx];
      }
    }
#pragma unroll
    for (int i = 0; i < kIt; ++i) {
      const int e = tid + (half * kIt + i) * 256;
      if (e >= kLI * kLI) continue;
      const int ly = e / kLI, lx = e - ly * kLI;
      const int o = ly * kLS + lx;
      sx[o] = a[i].x; sx[kLI * kLS + o] = a[i].y; sx[2 * kLI * kLS + o] = a[i].z;
      sy[o] = b[i].x; sy[kLI * kLS + o] = b[i].y; sy[2 * kLI * kLS + o] = b[i].z;
    }
  }
  __syncthreads();
  const int col = tid & 31, rg = tid >> 5;  // vertical pass: column, 4-row group
  const int px = blockIdx.x * kLT + col;
  float l1 = 0.0f, ss = 0.0f;
  for (int c = 0; c < 3; ++c) {
    const float* X = sx + c * kLI * kLS;
    const float* Y = sy + c * kLI * kLS;
    for (int r = tid; r < kLI * (kLT / 4); r += 256) {
      const int row = r >> 3, x0 = (r & 7) * 4;
      float xv[14], yv[14];
#pragma unroll
      for (int j = 0; j < 14; ++j) {
        xv[j] = X[row * kLS + x0 + j];
        yv[j] = Y[row * kLS + x0 + j];
      }
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        float m0 = 0, m1 = 0, m2 = 0, m3 = 0, m4 = 0;
#pragma unroll
        for (int k = 0; k < kSsimWin; ++k) {
          const float w = c_ssim_w[k], x = xv[o + k], y = yv[o + k];
          m0 += w * x; m1 += w * y; m2 += w * x * x; m3 += w * y * y; m4 += w * x * y;
        }
        const int q = row * kHS + x0 + o;
        hm[q] = m0; hm[kLI * kHS + q] = m1; hm[2 * kLI * kHS + q] = m2;
        hm[3 * kLI * kHS + q] = m3; hm[4 * kLI * kHS + q] = m4;
      }
    }
    __syncthreads();
    float mo[4][5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      float hv[14];
#pragma unroll
      for (int j = 0; j < 14; ++j) hv[j] = hm[q * kLI * kHS + (rg * 4 + j) * kHS + col];
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k < kSsimWin; ++k) acc += c_ssim_w[k] * hv[o + k];
        mo[o][q] = acc;
      }
    }
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      const int py = blockIdx.y * kLT + rg * 4 + o;
      if (px >= (int)W || py >= (int)H) continue;
      const float mx = mo[o][0], my = mo[o][1];
      const float sxx = mo[o][2] - mx * mx, syy = mo[o][3] - my * my, sxy = mo[o][4] - mx * my;
      const float A1 = 2.0f * mx * my + kSsimC1, A2 = 2.0f * sxy + kSsimC2;
      const float B1 = mx * mx + my * my + kSsimC1, B2 = sxx + syy + kSsimC2;
      // two fast reciprocals instead of five divisions (B1, B2 >= C1, C2 > 0)
      const float iB1 = __fdividef(1.0f, B1), iB2 = __fdividef(1.0f, B2), iB = iB1 * iB2;
      const float sv = (A1 * A2) * iB;
      ss += sv;
      const float dLds = -lambda * inv_norm;
      const float ds_dmx = (2.0f * my * A2) * iB - sv * 2.0f * mx * iB1;
      const float ds_dsxx = -sv * iB2;
      const float ds_dsxy = 2.0f * A1 * iB;
      const float dm = dLds * ds_dmx, d2 = dLds * ds_dsxx, dxy = dLds * ds_dsxy;
      const size_t plane = (size_t)W * H, pix = (size_t)py * W + px;
      float* mp = maps + ((size_t)v * 9 + 3 * c) * plane + pix;
      mp[0] = dm - 2.0f * mx * d2 - my * dxy;
      mp[plane] = d2;
      mp[2 * plane] = dxy;
      const int cy = rg * 4 + o + kHalo, cx = col + kHalo;
      l1 += fabsf(X[cy * kLS + cx] - Y[cy * kLS + cx]);
    }
    __syncthreads();  // before the next channel overwrites the horizontal sums
  }
  for (int o = 16; o > 0; o >>= 1) {
    l1 += __shfl_xor_sync(0xffffffffu, l1, o);
    ss += __shfl_xor_sync(0xffffffffu, ss, o);
  }
  if ((tid & 31) == 0) {
    red[0][tid >> 5] = l1;
    red[1][tid >> 5] = ss;
  }
  __syncthreads();
  if (tid == 0) {
    float a = 0, b = 0;
    for (int w = 0; w < 8; ++w) { a += red[0][w]; b += red[1][w]; }
    const size_t bi = ((size_t)v * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    partial[2 * bi] = a;
    partial[2 * bi + 1] = b;
  }
}

// four blocks per SM (at most 64 registers; five fit in shared memory)
__global__ void __launch_bounds__(256, 4) k_ssim_bwd2(const float4* __restrict__ img, const float4* __restrict__ tgt,
                                                   const uint32_t* __restrict__ tgt_ids,
                                                   const float* __restrict__ maps, uint32_t W, uint32_t H,
                                                   float lambda, float inv_norm, float4* __restrict__ dimg) {
  extern __shared__ float sm[];
  float* mp = sm;                    // [3][kLI][kLS]
  float* hm = mp + 3 * kLI * kLS;    // [3][kLI][kHS]
  const uint32_t v = blockIdx.z, tid = threadIdx.x;
  const int ox = blockIdx.x * kLT - kHalo, oy = blockIdx.y * kLT - kHalo;
  const size_t plane = (size_t)W * H;
  const int col = tid & 31, rg = tid >> 5;
  const int px = blockIdx.x * kLT + col;
  // the image and target are read per channel where they are used (they
  // come from L2), so no registers hold them across the kernel
  const float* imf = reinterpret_cast<const float*>(img + (size_t)v * plane);
  const float* tgf = reinterpret_cast<const float*>(tgt + (size_t)tgt_ids[v] * plane);
  const float l1w = (1.0f - lambda) * inv_norm;
  float d[4][3];
  for (int c = 0; c < 3; ++c) {
    const float* mv = maps + ((size_t)v * 9 + 3 * c) * plane;
    {  // stage the channel's three maps: every load issued before the stores
      constexpr int kIt = (kLI * kLI + 255) / 256;  // 7 elements per thread
      float m0[kIt], m1[kIt], m2[kIt];
#pragma unroll
      for (int i = 0; i < kIt; ++i) {
        const int e = tid + i * 256;
        const int ly = e / kLI, lx = e - ly * kLI;
        const int gx = ox + lx, gy = oy + ly;
        const bool ok = e < kLI * kLI && gx >= 0 && gy >= 0 && gx < (int)W && gy < (int)H;
        const size_t g = ok ? (size_t)gy * W + gx : 0;
        m0[i] = ok ? mv[g] : 0.0f;
        m1[i] = ok ? mv[plane + g] : 0.0f;
        m2[i] = ok ? mv[2 * plane + g] : 0.0f;
      }
#pragma unroll
      for (int i = 0; i < kIt; ++i) {
        const int e = tid + i * 256;
        if (e >= kLI * kLI) continue;
        const int ly = e / kLI, lx = e - ly * kLI;
        const int o = ly * kLS + lx;
        mp[o] = m0[i];
        mp[kLI * kLS + o] = m1[i];
        mp[2 * kLI * kLS + o] = m2[i];
      }
    }
    __syncthreads();
    for (int r = tid; r < 3 * kLI * (kLT / 4); r += 256) {
      const int q = r / (kLI * (kLT / 4)), rr = r - q * (kLI * (kLT / 4));
      const int row = rr >> 3, x0 = (rr & 7) * 4;
      float mvv[14];
#pragma unroll
      for (int j = 0; j < 14; ++j) mvv[j] = mp[q * kLI * kLS + row * kLS + x0 + j];
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k < kSsimWin; ++k) acc += c_ssim_w[k] * mvv[o + k];
        hm[q * kLI * kHS + row * kHS + x0 + o] = acc;
      }
    }
    __syncthreads();
    float cv[4][3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      float hv[14];
#pragma unroll
      for (int j = 0; j < 14; ++j) hv[j] = hm[q * kLI * kHS + (rg * 4 + j) * kHS + col];
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k < kSsimWin; ++k) acc += c_ssim_w[k] * hv[o + k];
        cv[o][q] = acc;
      }
    }
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      const int py = blockIdx.y * kLT + rg * 4 + o;
      const bool in = px < (int)W && py < (int)H;
      const size_t pix = in ? (size_t)py * W + px : 0;
      const float x = in ? __ldg(imf + 4 * pix + c) : 0.0f;
      const float y = in ? __ldg(tgf + 4 * pix + c) : 0.0f;
      const float diff = x - y;
      const float sgn = diff > 0.0f ? 1.0f : (diff < 0.0f ? -1.0f : 0.0f);
      d[o][c] = cv[o][0] + 2.0f * x * cv[o][1] + y * cv[o][2] + l1w * sgn;
    }
    __syncthreads();  // before the next channel overwrites the staged maps
  }
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    const int py = blockIdx.y * kLT + rg * 4 + o;
    if (px < (int)W && py < (int)H)
      dimg[(size_t)v * plane + (size_t)py * W + px] = make_float4(d[o][0], d[o][1], d[o][2], 0.0f);
  }
}

// Per-pixel losses without the SSIM term: mean |x - y| (KIND = kLossL1) or
// mean (x - y)^2 (KIND = kLossL2) over the colour channels.  A fixed grid of
// blocks per view strides over the view's pixels; each block writes its sums
// of |x - y| and (x - y)^2 to partial (in block order, so k_loss_reduce adds
// them in a fixed order), and every pixel its dL/dimage.
constexpr int kLossL1Dssim = 0, kLossL1 = 1, kLossL2 = 2;
constexpr uint32_t kPixLossBlocks = 128;  // per view
template <int KIND>
__global__ void __launch_bounds__(256) k_pix_loss(const float4* __restrict__ img, const float4* __restrict__ tgt,
                                                  const uint32_t* __restrict__ tgt_ids, uint32_t npix,
                                                  float inv_norm, float4* __restrict__ dimg,
                                                  float* __restrict__ partial) {
  __shared__ float red[2][8];
  const uint32_t v = blockIdx.y, tid = threadIdx.x;
  const float4* im = img + (size_t)v * npix;
  const float4* tg = tgt + (size_t)tgt_ids[v] * npix;
  float4* dm = dimg + (size_t)v * npix;
  float a = 0.0f, b = 0.0f;
  for (uint32_t i = blockIdx.x * 256 + tid; i < npix; i += gridDim.x * 256) {
    const float4 x = __ldg(im + i), y = __ldg(tg + i);
    const float d0 = x.x - y.x, d1 = x.y - y.y, d2 = x.z - y.z;
    a += fabsf(d0) + fabsf(d1) + fabsf(d2);
    b += d0 * d0 + d1 * d1 + d2 * d2;
    float4 g;
    if (KIND == kLossL2) {
      const float s = 2.0f * inv_norm;
      g = make_float4(s * d0, s * d1, s * d2, 0.0f);
    } else {
      auto sg = [](float d) { return d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f); };
      g = make_float4(sg(d0) * inv_norm, sg(d1) * inv_norm, sg(d2) * inv_norm, 0.0f);
    }
    dm[i] = g;
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((tid & 31) == 0) {
    red[0][tid >> 5] = a;
    red[1][tid >> 5] = b;
  }
  __syncthreads();
  if (tid == 0) {
    float sa = 0.0f, sb = 0.0f;
    for (int w = 0; w < 8; ++w) { sa += red[0][w]; sb += red[1][w]; }
    const size_t bi = (size_t)v * gridDim.x + blockIdx.x;
    partial[2 * bi] = sa;
    partial[2 * bi + 1] = sb;
  }
}

// Sums the per-block partials (|x - y| and SSIM sums for kind 0, |x - y| and
// (x - y)^2 sums otherwise) into loss[0..2] = (loss, mean L1, mean SSIM or
// mean squared error).
__global__ void k_loss_reduce(const float* __restrict__ partial, uint32_t nblocks, int kind, float lambda,
                              float inv_norm, float wconst, float* __restrict__ loss) {
  __shared__ float r0[kThreads], r1[kThreads];
  float a = 0, b = 0;
  for (uint32_t i = threadIdx.x; i < nblocks; i += kThreads) {
    a += partial[2 * i];
    b += partial[2 * i + 1];
  }
  r0[threadIdx.x] = a;
  r1[threadIdx.x] = b;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      r0[threadIdx.x] += r0[threadIdx.x + s];
      r1[threadIdx.x] += r1[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    // inv_norm = 1 / (3 H W V_loss); wconst = V / V_loss (this call's share of the loss)
    loss[0] = kind == kLossL1   ? r0[0] * inv_norm
              : kind == kLossL2 ? r1[0] * inv_norm
                                : (1.0f - lambda) * r0[0] * inv_norm + lambda * (wconst - r1[0] * inv_norm);
    loss[1] = r0[0] * inv_norm;  // mean L1
    loss[2] = r1[0] * inv_norm;  // mean SSIM (kind 0) or mean squared error
  }
}

// ------------------------------------------------------------ backward raster
// Reverse-order replay of the forward per pixel.  Default: the per-pair
// gradients of a warp are reduced by shuffles, summed over the CTA's warps with
// shared-memory atomics and added to the (view, Gaussian) records with global
// atomics.  kDet (deterministic two-pass mode): warps stage their sums in
// shared memory, which are folded in warp order, and each pair's tile sum is
// stored to `part` (no atomics); k_det_segsum then adds the pairs of each
// (view, Gaussian) record in sorted-pair order.
template <bool kDet>
__global__ void __launch_bounds__(kThreads) k_bwd(const Rec* __restrict__ recs, const uint32_t* __restrict__ vals,
                                                  const uint32_t* __restrict__ rstart,
                                                  const uint32_t* __restrict__ rend, uint32_t W, uint32_t H,
                                                  uint32_t tiles_x, uint32_t num_tiles, float3 bg,
                                                  const float4* __restrict__ img, const uint32_t* __restrict__ ncontrib,
                                                  const float4* __restrict__ dimg, float* __restrict__ g2,
                                                  float* __restrict__ part) {
  __shared__ float4 s_a[kThreads];
  __shared__ float4 s_b[kThreads];
  __shared__ float4 s_c[kThreads];
  __shared__ uint32_t s_g[kThreads];
  __shared__ float s_acc[kThreads][10];
  __shared__ float s_stage[kDet ? (kThreads / 32) * 320 : 1];
  __shared__ uint32_t s_max;
  const uint32_t tx = blockIdx.x, ty = blockIdx.y, v = blockIdx.z, tid = threadIdx.x, lane = tid & 31;
  const uint32_t warp = tid >> 5;
  const uint32_t px = tx * 16 + (tid & 15), py = ty * 16 + (tid >> 4);
  const bool inside = px < W && py < H;
  const float fx = (float)px, fy = (float)py;
  const float wx0 = (float)(tx * 16), wy0 = (float)(ty * 16 + 2 * (tid >> 5));
  const uint32_t key = v * num_tiles + ty * tiles_x + tx;
  const uint32_t start = rstart[key], end = rend[key];
  (void)end;
  float T = 1.0f, T_final = 1.0f;
  uint32_t last = 0;
  float dC[3] = {0, 0, 0};
  if (inside) {
    const size_t pix = ((size_t)v * H + py) * W + px;
    const float4 o = img[pix];
    T = o.w;
    T_final = o.w;
    last = ncontrib[pix];
    const float4 d = dimg[pix];
    dC[0] = d.x; dC[1] = d.y; dC[2] = d.z;
  }
  if (tid == 0) s_max = 0;
  __syncthreads();
  atomicMax(&s_max, last);
  __syncthreads();
  const uint32_t maxlast = s_max;
  const float bg_dot = bg.x * dC[0] + bg.y * dC[1] + bg.z * dC[2];
  float accum[3] = {0, 0, 0}, last_col[3] = {0, 0, 0};
  float last_alpha = 0.0f;

  // gradient of this pixel w.r.t. pair j of the staged batch (returns false if
  // the pair does not contribute here); advances the replay state
  auto pair_grad = [&](int j, uint32_t cur, float* gv) -> bool {
#pragma unroll
    for (int k = 0; k < 16; ++k) gv[k] = 0.0f;
    if (!(inside && cur < last)) return false;
    const float4 a = s_a[j];
    const float4 c4 = s_c[j];
    const float4 b = s_b[j];
    const float col[3] = {b.z, b.w, c4.x};
    const float dx = a.x - fx, dy = a.y - fy;
    float u, w;
    const float power = gs_power(a, b.x, dx, dy, u, w);
    if (power > 0.0f) return false;
    const float G = __expf(power);
    const float araw = b.y * G;
    const float alpha = fminf(kAlphaMax, araw);
    if (alpha < kAlphaMin) return false;
    T = T / (1.0f - alpha);
    const float wgt = alpha * T;
    float dL_dalpha = 0.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      accum[c] = last_alpha * last_col[c] + (1.0f - last_alpha) * accum[c];
      last_col[c] = col[c];
      dL_dalpha += (col[c] - accum[c]) * dC[c];
      gv[6 + c] = wgt * dC[c];
    }
    dL_dalpha *= T;
    last_alpha = alpha;
    dL_dalpha += (-T_final / (1.0f - alpha)) * bg_dot;
    if (araw <= kAlphaMax) {
      const float dL_dG = b.y * dL_dalpha;
      const float gdx = G * dx, gdy = G * dy;
      gv[0] = dL_dG * (-gdx * a.z - gdy * a.w);   // d/du
      gv[1] = dL_dG * (-gdy * b.x - gdx * a.w);   // d/dv
      gv[2] = -0.5f * gdx * dx * dL_dG;           // d/d conic a
      gv[3] = -gdx * dy * dL_dG;                  // d/d conic b
      gv[4] = -0.5f * gdy * dy * dL_dG;           // d/d conic c
      gv[5] = G * dL_dalpha;                      // d/d opacity
    }
    return true;
  };

  for (uint32_t bend = start + maxlast; bend > start;) {
    const uint32_t bstart = bend > start + kThreads ? bend - kThreads : start;
    const uint32_t nb = bend - bstart;
    __syncthreads();
    if (tid < nb) {
      const uint32_t gg = vals[bstart + tid];
      const Rec r = recs[gg];
      s_a[tid] = r.a;
      s_b[tid] = r.b;
      s_c[tid] = r.c;
      s_g[tid] = gg;
    }
#pragma unroll
    for (int k = 0; k < 10; ++k) s_acc[tid][k] = 0.0f;
    __syncthreads();
    if constexpr (!kDet) {
      for (int j = (int)nb - 1; j >= 0; --j) {
        const float4 a = s_a[j];
        const float4 c4 = s_c[j];
        if (warp_misses(a.x, a.y, c4.z, c4.w, wx0, wy0)) continue;  // warp-uniform
        float gv[16];
        const bool contrib = pair_grad(j, bstart + (uint32_t)j - start, gv);
        if (__any_sync(0xffffffffu, contrib)) {
          const float tot = warp_sum16(gv, lane);
          const uint32_t k = lane >> 1;
          if ((lane & 1) == 0 && k < 10) atomicAdd(&s_acc[j][k], tot);
        }
      }
    } else {
      // sub-batches of 32 pairs: warps stage, then one fixed-order fold
      for (int jhi = (int)nb - 1; jhi >= 0; jhi -= 32) {
        const int jlo = jhi >= 31 ? jhi - 31 : 0;
        float* st = s_stage + warp * 320;
        for (int k = (int)lane; k < 320; k += 32) st[k] = 0.0f;
        __syncwarp();
        for (int j = jhi; j >= jlo; --j) {
          const float4 a = s_a[j];
          const float4 c4 = s_c[j];
          if (warp_misses(a.x, a.y, c4.z, c4.w, wx0, wy0)) continue;  // warp-uniform
          float gv[16];
          const bool contrib = pair_grad(j, bstart + (uint32_t)j - start, gv);
          if (__any_sync(0xffffffffu, contrib)) {
            const float tot = warp_sum16(gv, lane);
            const uint32_t k = lane >> 1;
            if ((lane & 1) == 0 && k < 10) st[(j - jlo) * 10 + (int)k] = tot;
          }
        }
        __syncthreads();
        for (int t = (int)tid; t < 320; t += kThreads) {
          const int p = t / 10, k = t % 10;
          if (jlo + p <= jhi) {
            float sum = 0.0f;
#pragma unroll
            for (int w = 0; w < kThreads / 32; ++w) sum += s_stage[w * 320 + p * 10 + k];
            s_acc[jlo + p][k] = sum;
          }
        }
        __syncthreads();
      }
    }
    __syncthreads();
    if (tid < nb) {
      if constexpr (kDet) {
        float* dst = part + (size_t)(bstart + tid) * 10;
#pragma unroll
        for (int k = 0; k < 10; ++k) dst[k] = s_acc[tid][k];
      } else {
        float* dst = g2 + (size_t)s_g[tid] * kG2;
#pragma unroll
        for (int k = 0; k < 10; ++k) {
          const float x = s_acc[tid][k];
          if (x != 0.0f) atomicAdd(dst + k, x);
        }
      }
    }
    bend = bstart;
  }
}

// Per-pixel replay state of the backward.  The colour behind the current
// pair enters the gradient only through its dot product with dL/dpixel, so the
// replay carries that scalar (acc_dot) instead of the colour itself.
struct PixBwd {
  float T;          // transmittance in front of the pair being replayed
  float nbg;        // -T_final (background . dL/dpixel)
  float last_alpha, acc_dot, last_dot;
  float dC[3];
  float fx, fy;
  uint32_t last;    // contributors of the pixel; 0 outside the image
};

__device__ __forceinline__ void pix_bwd_init(PixBwd& s, uint32_t px, uint32_t py, uint32_t v, uint32_t W, uint32_t H,
                                             float3 bg, const float4* __restrict__ img,
                                             const uint32_t* __restrict__ ncontrib,
                                             const float4* __restrict__ dimg) {
  s.fx = (float)px;
  s.fy = (float)py;
  s.T = 1.0f;
  s.last = 0;
  s.dC[0] = s.dC[1] = s.dC[2] = 0.0f;
  if (px < W && py < H) {
    const size_t pix = ((size_t)v * H + py) * W + px;
    const float4 o = img[pix];
    s.T = o.w;
    s.last = ncontrib[pix];
    const float4 d = dimg[pix];
    s.dC[0] = d.x; s.dC[1] = d.y; s.dC[2] = d.z;
  }
  s.nbg = -s.T * (bg.x * s.dC[0] + bg.y * s.dC[1] + bg.z * s.dC[2]);
  s.last_alpha = s.acc_dot = s.last_dot = 0.0f;
}

// Scale of gradient term k that pix_bwd_pair leaves out of its per-pixel sums
// (applied once to the warp total): terms 0..4 are accumulated with their
// common factor -1 and terms 2 and 4 with twice their value.
__device__ __forceinline__ float bwd_term_scale(uint32_t k) {
  return k < 5u ? ((k == 2u || k == 4u) ? -0.5f : -1.0f) : 1.0f;
}

// adds this pixel's gradient w.r.t. the pair (a, b, c4) at sorted offset cur
// to gv[0..8] (terms 0..4 without their bwd_term_scale); returns whether the
// pair contributes here
__device__ __forceinline__ bool pix_bwd_pair(PixBwd& s, const float4& a, const float4& b, const float4& c4,
                                             uint32_t cur, float* gv) {
  if (cur >= s.last) return false;
  const float dx = a.x - s.fx, dy = a.y - s.fy;
  float u, w;
  const float power = gs_power(a, b.x, dx, dy, u, w);
  // power < -c4.y / 2 (outside the alpha >= 1/255 ellipse with its margin)
  // implies alpha < 1/255, so skipping those pixels before the exponential
  // leaves every decision of the alpha test below unchanged
  if (power > 0.0f || power < -0.5f * c4.y) return false;
  const float G = __expf(power);
  const float araw = b.y * G;
  const float alpha = fminf(kAlphaMax, araw);
  if (alpha < kAlphaMin) return false;
  // one reciprocal serves both divisions (approximate, ~2 ulp; alpha <= 0.99)
  const float inv1ma = __fdividef(1.0f, 1.0f - alpha);
  s.T = s.T * inv1ma;
  const float wgt = alpha * s.T;
  // colour behind this pair, dotted with dL/dpixel: last_alpha * last + (1 - last_alpha) * acc
  const float cdot = fmaf(c4.x, s.dC[2], fmaf(b.w, s.dC[1], b.z * s.dC[0]));
  s.acc_dot = fmaf(s.last_alpha, s.last_dot - s.acc_dot, s.acc_dot);
  s.last_dot = cdot;
  s.last_alpha = alpha;
  const float dL_dalpha = fmaf(s.nbg, inv1ma, (cdot - s.acc_dot) * s.T);
#pragma unroll
  for (int c = 0; c < 3; ++c) gv[6 + c] = fmaf(wgt, s.dC[c], gv[6 + c]);
  if (araw <= kAlphaMax) {
    // dL/dG = opacity dL/dalpha; h = G dL/dG
    const float h = araw * dL_dalpha, hx = h * dx, hy = h * dy;
    gv[0] = fmaf(h, u, gv[0]);     // d/du:  -h u
    gv[1] = fmaf(h, w, gv[1]);     // d/dv:  -h w
    gv[2] = fmaf(hx, dx, gv[2]);   // d/d conic a: -h dx dx / 2
    gv[3] = fmaf(hx, dy, gv[3]);   // d/d conic b: -h dx dy
    gv[4] = fmaf(hy, dy, gv[4]);   // d/d conic c: -h dy dy / 2
    gv[5] = fmaf(G, dL_dalpha, gv[5]);  // d/d opacity
  }
  return true;
}

// Backward raster, PPT vertically adjacent pixels per thread (256 / PPT
// threads per 16 x 16 tile, a warp covers a 16 x 2·PPT strip): one warp
// reduction serves 32·PPT pixels.  The warp first ballots the staged pairs
// that meet its strip and that some of its pixels reached, then walks them in
// reverse order.  Per-pair sums go to shared memory and then to the (view,
// Gaussian) records with global atomics.  PPT is the autotuned variant.
// With 1 or 2 pixels per thread at most 64 registers (1024 / (256 / PPT) blocks of 256 / PPT threads,
// 32 warps per SM): eight 128-thread blocks per SM instead of six cut the backward by 8% at the
// benchmark workload.  4 pixels per thread would spill under that bound and keep their registers.
template <int PPT, int SPS, bool kOrd>
__global__ void __launch_bounds__(256 / PPT, PPT <= 2 ? 1024 / (256 / PPT) : 1) k_bwd2(const Rec* __restrict__ recs, const uint32_t* __restrict__ vals,
                                                    const uint32_t* __restrict__ rstart,
                                                    const uint32_t* __restrict__ rend, uint32_t W, uint32_t H,
                                                    uint32_t tiles_x, uint32_t num_tiles, float3 bg,
                                                    const float4* __restrict__ img,
                                                    const uint32_t* __restrict__ ncontrib,
                                                    const float4* __restrict__ dimg, float* __restrict__ g2,
                                                    uint32_t* __restrict__ err, const uint32_t* __restrict__ order,
                                                    const uint32_t* __restrict__ qctl) {
  constexpr int NT = 256 / PPT, SB = NT * SPS;
  static_assert(SB <= 256, "staging buffers beyond the static shared-memory budget");
  __shared__ __align__(16) Rec s_rec[2][SB];
  __shared__ uint32_t s_g[3][SB];
  __shared__ float s_acc[2][SB][9];
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ uint32_t s_max;
  uint32_t tx = blockIdx.x, ty = blockIdx.y, v = blockIdx.z;
  if constexpr (kOrd) {
    // 1D grid over the items with contributors, longest first
    if (blockIdx.x >= qctl[0]) return;
    const uint32_t it = order[blockIdx.x];
    v = it / num_tiles;
    const uint32_t tile = it - v * num_tiles;
    ty = tile / tiles_x;
    tx = tile - ty * tiles_x;
  }
  const uint32_t tid = threadIdx.x, lane = tid & 31;
  using TM = TileMap16<PPT>;
  const uint32_t px = tx * 16 + TM::x(tid), py = ty * 16 + TM::y(tid);
  const float wx0 = (float)(tx * 16 + TM::wx(tid)), wy0 = (float)(ty * 16 + TM::wy(tid));
  constexpr float ww = (float)(TM::kW - 1), wh = (float)(TM::kH - 1);
  const uint32_t key = v * num_tiles + ty * tiles_x + tx;
  const uint32_t start = rstart[key];
  PixBwd p[PPT];
  uint32_t mylast = 0;
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    pix_bwd_init(p[k], px, py + k, v, W, H, bg, img, ncontrib, dimg);
    mylast = max(mylast, p[k].last);
  }
  __shared__ uint32_t s_abort;
  if (tid == 0) {
    s_max = 0;
    s_abort = 0u;
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (uint32_t r = tid; r < (uint32_t)(2 * SB * 9); r += NT) (&s_acc[0][0][0])[r] = 0.0f;
  __syncthreads();
  atomicMax(&s_max, mylast);
  __syncthreads();
  const uint32_t maxlast = s_max;
  uint32_t wlast = mylast;  // pairs at or beyond every pixel's last contributor are skipped
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) wlast = max(wlast, __shfl_xor_sync(0xffffffffu, wlast, o));
  // batches in reverse: batch i covers [max(start, top - (i+1) NT), top - i NT), top = start + maxlast
  const uint32_t nbatch = (maxlast + SB - 1) / SB;
  auto bstart_of = [&](uint32_t i) {
    const uint32_t hi = start + maxlast - i * SB;
    return hi > start + SB ? hi - SB : start;
  };
  if (nbatch > 0) {
    const uint32_t b0 = bstart_of(0);
    stage_batch(recs, vals, b0, start + maxlast - b0, s_rec[0], &s_bar[0], s_g[0]);
  }
  // One CTA barrier per batch: batch bi accumulates into s_acc[bi & 1]; after
  // the barrier each thread flushes and clears its rows of that buffer while
  // others may already walk batch bi + 1 into the other one.  The barrier also
  // orders the re-staging of s_rec[bi & 1] (issued at batch bi + 1, after the
  // barrier of batch bi) after every read of it, and the record ids rotate
  // through three buffers so that staging batch bi + 2 never overwrites the
  // ids the flush of batch bi is still reading.
  uint32_t gb = 0;  // bi % 3
  for (uint32_t bi = 0; bi < nbatch; ++bi) {
    const uint32_t buf = bi & 1u, gnext = gb == 2u ? 0u : gb + 1u;
    const uint32_t bend = start + maxlast - bi * SB, bstart = bstart_of(bi);
    const uint32_t nb = bend - bstart;
    if (bi + 1 < nbatch) {
      const uint32_t nbs = bstart_of(bi + 1);
      stage_batch(recs, vals, nbs, bstart - nbs, s_rec[buf ^ 1u], &s_bar[buf ^ 1u], s_g[gnext]);
    }
    if (!mbar_wait(&s_bar[buf], (bi >> 1) & 1u)) s_abort = 1u;  // the batch is undefined: end the tile below
    const Rec* sr = s_rec[buf];
    float(*acc)[9] = s_acc[buf];
    uint32_t hit[SB / 32];
#pragma unroll
    for (int qq = 0; qq < SB / 32; ++qq) {
      const uint32_t jj = qq * 32 + lane;
      bool h = false;
      if (jj < nb && bstart + jj - start < wlast)
        h = !rec_misses_box(sr[jj].a, sr[jj].b.x, sr[jj].c, wx0, wy0, ww, wh);
      hit[qq] = __ballot_sync(0xffffffffu, h);
    }
#pragma unroll
    for (int qq = SB / 32 - 1; qq >= 0; --qq)
    for (uint32_t m = hit[qq]; m != 0u;) {
      const int bit = 31 - __clz(m);
      m &= ~(1u << bit);
      const int j = qq * 32 + bit;  // descending within the batch
      const float4 a = sr[j].a;
      const float4 c4 = sr[j].c;
      const float4 b = sr[j].b;
      const uint32_t cur = bstart + (uint32_t)j - start;
      float gv[9];
#pragma unroll
      for (int k = 0; k < 9; ++k) gv[k] = 0.0f;
      bool any = false;
#pragma unroll
      for (int k = 0; k < PPT; ++k) any |= pix_bwd_pair(p[k], a, b, c4, cur, gv);
      const uint32_t cm = __ballot_sync(0xffffffffu, any);
#if NPS_GS_SOLO
      if (cm != 0u && (cm & (cm - 1u)) == 0u) {
        // one contributing lane: its values are the warp totals
        if (any) {
#pragma unroll
          for (int k = 0; k < 9; ++k) atomicAdd(&acc[j][k], gv[k] * bwd_term_scale((uint32_t)k));
        }
      } else
#endif
      if (cm != 0u) {
        const float tot = warp_sum9(gv, lane);
        const uint32_t k = warp_sum9_index(lane);
        if ((lane & 1) == 0 && k < 9) atomicAdd(&acc[j][k], tot * bwd_term_scale(k));
      }
    }
    __syncthreads();
    if (s_abort) {
      // a bounded wait gave up: no further sums leave the tile (the step reports NPS_ERR_TIMEOUT); the
      // batch staged for bi + 1 is waited for (bounded) before the CTA's shared memory is released
      if (tid == 0) {
        atomicAdd(err, 1u);
        (void)mbar_wait(&s_bar[buf], (bi >> 1) & 1u);  // the batch whose wait gave up, again (bounded)
        if (bi + 1 < nbatch) (void)mbar_wait(&s_bar[buf ^ 1u], ((bi + 1) >> 1) & 1u);
      }
      return;
    }
    for (uint32_t r = tid; r < nb; r += NT) {
      float* dst = g2 + (size_t)s_g[gb][r] * kG2;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const float x = acc[r][k];
        if (x != 0.0f) {
          atomicAdd(dst + k, x);
          acc[r][k] = 0.0f;
        }
      }
    }
    gb = gnext;
  }
}

#include "gs_raster_ws.cuh"

// deterministic mode: (record, sorted position) pairs to sort by record
__global__ void k_det_prep(const uint32_t* __restrict__ sorted_vals, const uint32_t* __restrict__ total, uint32_t cap,
                           uint32_t* __restrict__ keys, uint32_t* __restrict__ pos) {
  const uint32_t K = min(*total, cap);
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < K; p += gridDim.x * blockDim.x) {
    keys[p] = sorted_vals[p];
    pos[p] = p;
  }
}

// deterministic mode: each record's pair sums added in sorted-pair order
__global__ void k_det_segsum(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ pos,
                             const uint32_t* __restrict__ total, uint32_t cap, const float* __restrict__ part,
                             float* __restrict__ g2) {
  const uint32_t K = min(*total, cap);
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < K; p += gridDim.x * blockDim.x) {
    const uint32_t k = keys[p];
    if (p > 0 && keys[p - 1] == k) continue;  // not the first pair of this record
    float sum[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t q = p; q < K && keys[q] == k; ++q) {
      const float* src = part + (size_t)pos[q] * 10;
#pragma unroll
      for (int c = 0; c < 10; ++c) sum[c] += src[c];
    }
    float* dst = g2 + (size_t)k * kG2;
#pragma unroll
    for (int c = 0; c < 10; ++c) dst[c] = sum[c];
  }
}

// ------------------------------------------------------------ projection backward
// Eight lanes per Gaussian, each taking the views v = lane, lane + 8, ...: a
// lane accumulates its views' parameter gradients in record layout (64
// registers), then the eight partial records are summed by a reduce-scatter
// over the group (xor 4, 2, 1: 56 shuffles) and lane s writes floats
// 8s .. 8s + 7 of the Gaussian's gradient record.  The ADC statistic rides in
// the padding floats 60 and 61 through the reduction.
// ONE: at most eight views, so each lane has at most one view.  Its SH
// gradient is then basis[k] * dc[c] exactly (a sum of one term), which is
// formed just before the reduction instead of being accumulated through the
// view's projection arithmetic: 48 fewer live registers there.
template <int DEG, bool ONE>
__global__ void __launch_bounds__(128, ONE ? 4 : 1) k_project_bwd(const float* __restrict__ params, uint32_t n,
                                                     const float* __restrict__ views, uint32_t nv, uint32_t W,
                                                     uint32_t H, const uint32_t* __restrict__ counts,
                                                     const float* __restrict__ g2, float* __restrict__ grads,
                                                     float* __restrict__ adc_grad, float* __restrict__ adc_denom,
                                                     int accumulate, float adc_scale) {
  constexpr int nb = (DEG + 1) * (DEG + 1);
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t i = t >> 3, sub = t & 7;
  const bool live = i < n;  // whole groups are live or not (n * 8 threads, groups aligned)
  if (__all_sync(0xffffffffu, !live)) return;
  const float4* p4 = reinterpret_cast<const float4*>(params + (size_t)(live ? i : 0) * kP);
  const float4 q0 = p4[0], q1 = p4[1], q2 = p4[2];
  float mean[3] = {q0.x, q0.y, q0.z};
  float ls[3] = {q0.w, q1.x, q1.y};
  float q[4] = {q1.z, q1.w, q2.x, q2.y};
  const float op_logit = q2.z;
  float sh[(3 * nb + 3) / 4 * 4];
#pragma unroll
  for (int k4 = 0; k4 < (3 * nb + 3) / 4; ++k4) {
    const float4 t = p4[3 + k4];
    sh[4 * k4] = t.x; sh[4 * k4 + 1] = t.y; sh[4 * k4 + 2] = t.z; sh[4 * k4 + 3] = t.w;
  }
  float g[kP];
#pragma unroll
  for (int k = 0; k < kP; ++k) g[k] = 0.0f;
  float one_basis[ONE ? nb : 1], one_dc[3] = {0.0f, 0.0f, 0.0f};
  bool one_has = false;
  for (uint32_t v = sub; live && v < nv; v += 8) {
    const size_t gi = (size_t)v * n + i;
    if (counts[gi] == 0) continue;
    const float* gr = g2 + gi * kG2;
    const float du = gr[0], dv = gr[1], dca = gr[2], dcb = gr[3], dcc = gr[4], dop = gr[5];
    const float dcol[3] = {gr[6], gr[7], gr[8]};
    const float* view = views + (size_t)v * kViewRec;
    Proj<float> P;
    project<float>(view, mean, ls, q, (float)W, (float)H, kLowpass, P);
    // NDC-space gradient of this view's own loss (the loss is averaged over adc_scale views)
    g[60] += adc_scale * sqrtf((du * 0.5f * W) * (du * 0.5f * W) + (dv * 0.5f * H) * (dv * 0.5f * H));
    g[61] += 1.0f;
    g[kOpacity] += dop;
    const float ddx = mean[0] - view[32], ddy = mean[1] - view[33], ddz = mean[2] - view[34];
    const float l2 = fmaxf(ddx * ddx + ddy * ddy + ddz * ddz, 1e-20f);
    const float il = rsqrtf(l2);
    const float dir[3] = {ddx * il, ddy * il, ddz * il};
    float basis[16];
    sh_basis<float>(DEG, dir[0], dir[1], dir[2], basis);
    // the stored colour is clamped; recompute the unclamped value to test the clamp
    float dc[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float raw = 0.5f;
#pragma unroll
      for (int k = 0; k < nb; ++k) raw += basis[k] * sh[3 * k + c];
      dc[c] = raw < 0.0f ? 0.0f : dcol[c];
    }
    if constexpr (DEG > 0) {
      float bx[16], by[16], bz[16];
      sh_basis_grad<float>(DEG, dir[0], dir[1], dir[2], bx, by, bz);
      float ddir[3] = {0, 0, 0};
#pragma unroll
      for (int k = 1; k < nb; ++k) {
        const float s = sh[3 * k] * dc[0] + sh[3 * k + 1] * dc[1] + sh[3 * k + 2] * dc[2];
        ddir[0] += s * bx[k];
        ddir[1] += s * by[k];
        ddir[2] += s * bz[k];
      }
      const float dd = dir[0] * ddir[0] + dir[1] * ddir[1] + dir[2] * ddir[2];
#pragma unroll
      for (int c = 0; c < 3; ++c) g[c] += (ddir[c] - dir[c] * dd) * il;
    }
    if constexpr (ONE) {
#pragma unroll
      for (int k = 0; k < nb; ++k) one_basis[k] = basis[k];
#pragma unroll
      for (int c = 0; c < 3; ++c) one_dc[c] = dc[c];
      one_has = true;
    } else {
#pragma unroll
      for (int k = 0; k < nb; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) g[kSH + 3 * k + c] += basis[k] * dc[c];
    }
    // conic -> covariance: dL/dCov = -Inv H Inv, H = [[ga, gb/2], [gb/2, gc]]
    const float ia = P.ca, ib = P.cb, ic = P.cc;
    const float h00 = dca, h01 = 0.5f * dcb, h11 = dcc;
    const float x00 = h00 * ia + h01 * ib, x01 = h00 * ib + h01 * ic;
    const float x10 = h01 * ia + h11 * ib, x11 = h01 * ib + h11 * ic;
    const float G00 = -(ia * x00 + ib * x10);
    const float G01 = -(ia * x01 + ib * x11);
    const float G10 = -(ib * x00 + ic * x10);
    const float G11 = -(ib * x01 + ic * x11);
    const float Gs[2][2] = {{G00, 0.5f * (G01 + G10)}, {0.5f * (G01 + G10), G11}};
    // dL/dSigma = J^T Gs J ; dL/dJ = 2 Gs J Sigma
    float GJ[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) GJ[r][c] = Gs[r][0] * P.J[0][c] + Gs[r][1] * P.J[1][c];
    float dS[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) dS[r][c] = P.J[0][r] * GJ[0][c] + P.J[1][r] * GJ[1][c];
    float dJ[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        dJ[r][c] = 2.0f * (GJ[r][0] * P.S[0][c] + GJ[r][1] * P.S[1][c] + GJ[r][2] * P.S[2][c]);
    // J depends on the mean through clip (x, y, w)
    {
      const float r0[3] = {view[0], view[4], view[8]};
      const float r1[3] = {view[1], view[5], view[9]};
      const float r3[3] = {view[3], view[7], view[11]};
      const float a = 0.5f * W, b = 0.5f * H;
      const float iw = 1.0f / P.cw, iw2 = iw * iw, iw3 = iw2 * iw;
      const float d0r0 = dJ[0][0] * r0[0] + dJ[0][1] * r0[1] + dJ[0][2] * r0[2];
      const float d0r3 = dJ[0][0] * r3[0] + dJ[0][1] * r3[1] + dJ[0][2] * r3[2];
      const float d1r1 = dJ[1][0] * r1[0] + dJ[1][1] * r1[1] + dJ[1][2] * r1[2];
      const float d1r3 = dJ[1][0] * r3[0] + dJ[1][1] * r3[1] + dJ[1][2] * r3[2];
#pragma unroll
      for (int l = 0; l < 3; ++l) {
        g[l] += a * (-d0r0 * r3[l] * iw2 - d0r3 * r0[l] * iw2 + 2.0f * P.cx * d0r3 * r3[l] * iw3);
        g[l] += -b * (-d1r1 * r3[l] * iw2 - d1r3 * r1[l] * iw2 + 2.0f * P.cy * d1r3 * r3[l] * iw3);
        g[l] += P.J[0][l] * du + P.J[1][l] * dv;
      }
    }
    // Sigma = M M^T, M = R diag(s)
    float dM[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        dM[r][c] = 2.0f * (dS[r][0] * P.M[0][c] + dS[r][1] * P.M[1][c] + dS[r][2] * P.M[2][c]);
    float dR[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float ds = 0.0f;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        ds += dM[r][c] * P.R[r][c];
        dR[r][c] = dM[r][c] * P.sc[c];
      }
      g[kLogScale + c] += ds * P.sc[c];
    }
    float dqn[4];
    rot_grad_to_quat<float>(P.qn[0], P.qn[1], P.qn[2], P.qn[3], dR, dqn);
    const float qd = P.qn[0] * dqn[0] + P.qn[1] * dqn[1] + P.qn[2] * dqn[2] + P.qn[3] * dqn[3];
#pragma unroll
    for (int k = 0; k < 4; ++k) g[kQuat + k] += (dqn[k] - P.qn[k] * qd) / P.qlen;
    if constexpr (ONE) break;  // a lane's only view
  }
  if constexpr (ONE) {
    if (one_has) {
#pragma unroll
      for (int k = 0; k < nb; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) g[kSH + 3 * k + c] = one_basis[k] * one_dc[c];
    }
  }
  // reduce-scatter over the group's eight lanes
  const bool b2 = sub & 4, b1 = sub & 2, b0 = sub & 1;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const float send = b2 ? g[j] : g[j + 32], keep = b2 ? g[j + 32] : g[j];
    g[j] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float send = b1 ? g[j] : g[j + 16], keep = b1 ? g[j + 16] : g[j];
    g[j] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float send = b0 ? g[j] : g[j + 8], keep = b0 ? g[j + 8] : g[j];
    g[j] = keep + __shfl_xor_sync(0xffffffffu, send, 1);
  }
  if (!live) return;
  // this lane holds record floats 8 * sub .. 8 * sub + 7 in g[0..7]
  if (sub == 1) {
    const float op = sigmoidf(op_logit);
    g[kOpacity - 8] *= op * (1.0f - op);
    g[11 - 8] = 0.0f;
  }
  if (sub == 7) {
    adc_grad[i] += g[60 - 56];
    adc_denom[i] += g[61 - 56];
    g[4] = g[5] = g[6] = g[7] = 0.0f;
  }
  float4* out4 = reinterpret_cast<float4*>(grads + (size_t)i * kP + 8 * sub);
  float4 w0 = make_float4(g[0], g[1], g[2], g[3]), w1 = make_float4(g[4], g[5], g[6], g[7]);
  if (accumulate) {
    const float4 a0 = out4[0], a1 = out4[1];
    w0.x += a0.x; w0.y += a0.y; w0.z += a0.z; w0.w += a0.w;
    w1.x += a1.x; w1.y += a1.y; w1.z += a1.z; w1.w += a1.w;
  }
  out4[0] = w0;
  out4[1] = w1;
}

// ------------------------------------------------------------ Adam
struct AdamArgs {
  float lr[6];  // mean, log-scale, quat, opacity, SH DC, SH rest
  float b1, b2, eps;
};

// Step state in device memory (so that a captured graph advances it):
// [0] step counter, [1] skip flag, [2], [3] bias corrections (f32 bits),
// [4] steps skipped for pair overflow, [6] bounded device waits that gave up
// (raster staging, sort look-back), [7] the value of [6] the last Adam step saw.
// The step is skipped when the last forward produced more pairs than the
// pair buffers hold (only possible in a captured graph, whose capacity is
// fixed: parameters stay unchanged and the host grows the capacity), or when
// a bounded wait gave up since the last step (its results are incomplete).
__global__ void k_adam_prep(uint32_t* st, const uint32_t* total, uint32_t cap) {
  const bool overflow = *total > cap;
  const bool timed_out = st[6] != st[7];
  st[7] = st[6];
  st[1] = (overflow || timed_out) ? 1u : 0u;
  if (overflow) {
    st[4] += 1u;  // skipped steps so far (read by the host after graph replays)
    return;
  }
  if (timed_out) return;
  const uint32_t step = st[0] + 1;
  st[0] = step;
  st[2] = __float_as_uint((float)(1.0 - pow(0.9, (double)step)));
  st[3] = __float_as_uint((float)(1.0 - pow(0.999, (double)step)));
}

__device__ __forceinline__ float lr_of(const AdamArgs& a, int k) {
  return k < 3 ? a.lr[0] : k < 6 ? a.lr[1] : k < 10 ? a.lr[2] : k < 12 ? a.lr[3] : k < 15 ? a.lr[4] : a.lr[5];
}

// one thread per float4 of the parameter record (16 per Gaussian)
__global__ void __launch_bounds__(256) k_adam(float4* __restrict__ p, const float4* __restrict__ g,
                                              float4* __restrict__ m, float4* __restrict__ v, uint32_t n4,
                                              AdamArgs a, const uint32_t* __restrict__ st) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n4 || st[1] != 0u) return;
  if ((t & 15u) * 4u >= (uint32_t)kUsed) return;  // floats 60-63: nothing to update, nothing to move
  const float bc1 = __uint_as_float(st[2]), bc2 = __uint_as_float(st[3]);
  const int k0 = (int)(t & 15u) * 4;
  float4 pp = p[t], gg = g[t], mm = m[t], vv = v[t];
  float* pf = &pp.x;
  const float* gf = &gg.x;
  float* mf = &mm.x;
  float* vf = &vv.x;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int k = k0 + c;
    if (k == 11 || k >= kUsed) continue;
    const float gr = gf[c];
    mf[c] = a.b1 * mf[c] + (1.0f - a.b1) * gr;
    vf[c] = a.b2 * vf[c] + (1.0f - a.b2) * gr * gr;
    const float mh = mf[c] / bc1, vh = vf[c] / bc2;
    pf[c] -= lr_of(a, k) * mh / (sqrtf(vh) + a.eps);
  }
  p[t] = pp;
  m[t] = mm;
  v[t] = vv;
}


// ------------------------------------------------------------ ADC (densify / prune)
// Classify every Gaussian from its accumulated view-space gradient norm
// (average over the views that saw it): prune if opacity < prune_opacity;
// else densify if avg >= grad_thresh — split into two children (scales / 1.6,
// means drawn from the parent Gaussian) when its largest scale exceeds
// split_scale, otherwise clone it.  Outputs per Gaussian: 0 (pruned), 1 or 2.
struct AdcParams {
  float grad_thresh, split_scale, prune_opacity;
  uint32_t seed;
};

// flags: bit 0 keep, bit 1 densify candidate, bit 2 split (else clone)
__global__ void k_adc_classify(const float* __restrict__ params, const float* __restrict__ adc_grad,
                               const float* __restrict__ adc_denom, uint32_t n, AdcParams a,
                               uint32_t* __restrict__ flags, uint32_t* __restrict__ keep_cnt,
                               uint32_t* __restrict__ cand_cnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* p = params + (size_t)i * kP;
  const float op = 1.0f / (1.0f + expf(-p[kOpacity]));
  uint32_t f = 0;
  if (!(op < a.prune_opacity)) {
    f = 1;
    const float d = adc_denom[i];
    const float avg = d > 0.0f ? adc_grad[i] / d : 0.0f;
    if (avg >= a.grad_thresh) {
      f |= 2;
      const float ms = expf(fmaxf(fmaxf(p[3], p[4]), p[5]));
      if (ms > a.split_scale) f |= 4;
    }
  }
  flags[i] = f;
  keep_cnt[i] = f & 1u;
  cand_cnt[i] = (f >> 1) & 1u;
}

__global__ void k_adc_count(const uint32_t* __restrict__ flags, const uint32_t* __restrict__ cand_rank, uint32_t n,
                            uint32_t budget, uint32_t* __restrict__ out_cnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t f = flags[i];
  out_cnt[i] = (f & 1u) ? ((f & 2u) && cand_rank[i] < budget ? 2u : 1u) : 0u;
}

// ADC feature vector of each Gaussian (16 floats) for the learned policy, the
// plain rule's decision (0 keep, 1 clone, 2 split, 3 prune) and its lineage id
// (record float 63: copied to clones and split children, so a family shares it).
__global__ void k_adc_features(const float* __restrict__ params, const float* __restrict__ am,
                               const float* __restrict__ av, const float* __restrict__ adc_grad,
                               const float* __restrict__ adc_denom, uint32_t n, AdcParams a, float step_frac,
                               float* __restrict__ feat, uint8_t* __restrict__ plain, uint32_t* __restrict__ ids) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* p = params + (size_t)i * kP;
  const float op = 1.0f / (1.0f + expf(-p[kOpacity]));
  const float d = adc_denom[i];
  const float avg = d > 0.0f ? adc_grad[i] / d : 0.0f;
  float l0 = p[3], l1 = p[4], l2 = p[5];
  // sorted descending
  if (l0 < l1) { const float t = l0; l0 = l1; l1 = t; }
  if (l1 < l2) { const float t = l1; l1 = l2; l2 = t; }
  if (l0 < l1) { const float t = l0; l0 = l1; l1 = t; }
  const float* mm = am + (size_t)i * kP;
  const float* vv = av + (size_t)i * kP;
  float rest = 0.0f;
  for (int k = 15; k < 60; ++k) rest += p[k] * p[k];
  float f[16];
  f[0] = log10f(avg + 1e-10f) + 4.0f;
  f[1] = log1pf(d) * 0.25f;
  f[2] = op;
  f[3] = p[kOpacity] * 0.25f;
  f[4] = (l0 + 4.0f) * 0.5f;
  f[5] = (l1 + 4.0f) * 0.5f;
  f[6] = (l2 + 4.0f) * 0.5f;
  f[7] = (l0 - logf(a.split_scale)) * 0.4342945f;
  f[8] = sqrtf(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) * 0.5f;
  f[9] = sqrtf(p[12] * p[12] + p[13] * p[13] + p[14] * p[14]) * 0.28209479f;
  f[10] = sqrtf(rest);
  f[11] = step_frac;
  f[12] = log10f(sqrtf((vv[0] + vv[1] + vv[2]) * (1.0f / 3.0f)) + 1e-12f) + 6.0f;
  f[13] = log10f(fabsf(mm[kOpacity]) + 1e-10f) + 6.0f;
  f[14] = fminf(fmaxf(log10f((avg + 1e-12f) / a.grad_thresh), -3.0f), 3.0f) * (1.0f / 3.0f);
  f[15] = 1.0f;
  float4* o4 = reinterpret_cast<float4*>(feat + (size_t)i * 16);
  o4[0] = make_float4(f[0], f[1], f[2], f[3]);
  o4[1] = make_float4(f[4], f[5], f[6], f[7]);
  o4[2] = make_float4(f[8], f[9], f[10], f[11]);
  o4[3] = make_float4(f[12], f[13], f[14], f[15]);
  if (plain) {
    uint8_t dec = 0;
    if (op < a.prune_opacity) dec = 3;
    else if (avg >= a.grad_thresh) dec = expf(fmaxf(fmaxf(p[3], p[4]), p[5])) > a.split_scale ? 2 : 1;
    plain[i] = dec;
  }
  if (ids) ids[i] = __float_as_uint(p[63]);
}

// Policy decisions to ADC flags: argmax over {keep (0), clone, split, prune}
// logits; a row with non-finite logits falls back to the plain rule.
__global__ void k_adc_policy_flags(const float* __restrict__ logits, const float* __restrict__ params,
                                   const float* __restrict__ adc_grad, const float* __restrict__ adc_denom,
                                   uint32_t n, AdcParams a, uint32_t* __restrict__ flags,
                                   uint32_t* __restrict__ keep_cnt, uint32_t* __restrict__ cand_cnt,
                                   uint32_t* __restrict__ fallback, float keep_logit) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float z1 = logits[3 * (size_t)i], z2 = logits[3 * (size_t)i + 1], z3 = logits[3 * (size_t)i + 2];
  uint32_t f;
  if (isfinite(z1) && isfinite(z2) && isfinite(z3)) {
    int best = 0;
    float m = keep_logit;  // 0: plain argmax; > 0 favours keep (act only when confident)
    if (z1 > m) m = z1, best = 1;
    if (z2 > m) m = z2, best = 2;
    if (z3 > m) m = z3, best = 3;
    f = best == 0 ? 1u : best == 1 ? 3u : best == 2 ? 7u : 0u;
  } else {
    const float* p = params + (size_t)i * kP;
    const float op = 1.0f / (1.0f + expf(-p[kOpacity]));
    f = 0;
    if (!(op < a.prune_opacity)) {
      f = 1;
      const float d = adc_denom[i];
      const float avg = d > 0.0f ? adc_grad[i] / d : 0.0f;
      if (avg >= a.grad_thresh) f |= expf(fmaxf(fmaxf(p[3], p[4]), p[5])) > a.split_scale ? 6u : 2u;
    }
    atomicAdd(fallback, 1u);
  }
  flags[i] = f;
  keep_cnt[i] = f & 1u;
  cand_cnt[i] = (f >> 1) & 1u;
}

__global__ void k_assign_ids(float* __restrict__ params, uint32_t n, uint32_t base) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) params[(size_t)i * kP + 63] = __uint_as_float(base + i);
}

// one thread per (Gaussian, float4 of its record)
__global__ void k_adc_scatter(const float4* __restrict__ p_in, const float4* __restrict__ m_in,
                              const float4* __restrict__ v_in, const uint32_t* __restrict__ flags,
                              const uint32_t* __restrict__ out_cnt, const uint32_t* __restrict__ out_off, uint32_t n,
                              AdcParams a, float4* __restrict__ p_out, float4* __restrict__ m_out,
                              float4* __restrict__ v_out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * 16) return;
  const uint32_t i = t >> 4, q = t & 15;
  const uint32_t c = out_cnt[i];
  if (c == 0) return;
  const uint32_t o = out_off[i];
  const float4 pv = p_in[t];
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  if (c == 1) {
    p_out[(size_t)o * 16 + q] = pv;
    m_out[(size_t)o * 16 + q] = m_in[t];
    v_out[(size_t)o * 16 + q] = v_in[t];
    return;
  }
  const bool split = flags[i] & 4u;
  if (!split) {
    // clone: the original keeps its optimiser state, the copy starts at zero
    p_out[(size_t)o * 16 + q] = pv;
    m_out[(size_t)o * 16 + q] = m_in[t];
    v_out[(size_t)o * 16 + q] = v_in[t];
    p_out[(size_t)(o + 1) * 16 + q] = pv;
    m_out[(size_t)(o + 1) * 16 + q] = z;
    v_out[(size_t)(o + 1) * 16 + q] = z;
    return;
  }
  // split: two children, fresh optimiser state
  for (uint32_t ch = 0; ch < 2; ++ch) {
    float4 r = pv;
    if (q <= 1) {
      float mean[3], ls[3];
      gsm::adc_split_child(reinterpret_cast<const float*>(p_in + (size_t)i * 16), i, a.seed, ch, mean, ls);
      if (q == 0) r = make_float4(mean[0], mean[1], mean[2], ls[0]);
      else r = make_float4(ls[1], ls[2], pv.z, pv.w);
    }
    p_out[(size_t)(o + ch) * 16 + q] = r;
    m_out[(size_t)(o + ch) * 16 + q] = z;
    v_out[(size_t)(o + ch) * 16 + q] = z;
  }
}

// per-view squared error of the last forward against the targets
__global__ void k_sq_err(const float4* __restrict__ img, const float4* __restrict__ tgt,
                         const uint32_t* __restrict__ tids, uint32_t W, uint32_t H, double* __restrict__ acc) {
  const uint32_t v = blockIdx.y;
  const size_t np = (size_t)W * H;
  double sum = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
    const float4 a = img[(size_t)v * np + i], b = tgt[(size_t)tids[v] * np + i];
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    sum += (double)(dx * dx + dy * dy + dz * dz);
  }
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(acc + v, sum);
}

}  // namespace gs
}  // namespace nps

// =================================================================== host side
using namespace nps;

namespace {
__global__ void k_set_u32(uint32_t* p, uint32_t v) { *p = v; }
}  // namespace

struct nps_gs {
  nps_ctx* ctx = nullptr;
  uint32_t cap = 0, n = 0;
  int sh_deg = 3;
  DevBuf params, grads, am, av, adc_grad, adc_denom;
  uint32_t step = 0;
  float lr[6] = {1.6e-4f, 5e-3f, 1e-3f, 5e-2f, 2.5e-3f, 2.5e-3f / 20.0f};
  float lambda = 0.2f;
  int loss_kind = gs::kLossL1Dssim;  // NPS_GS_LOSS_*
  bool accumulate = false;   // backward adds to the gradients instead of replacing them
  bool deterministic = false;  // two-pass backward reduction (no float atomics)
  // raster variants: pixels per thread (1, 2, 4) and records staged per batch; see nps_gs_autotune
  int fwd_ppt = 1, bwd_ppt = 2, fwd_stage = 256, bwd_stage = 128;
  // raster form: 0 = one CTA per (tile, view), 1 = persistent warp-specialised kernel over a work queue
  int fwd_form = 0, bwd_form = 0;
  uint32_t tile = 16;  // tile edge in pixels (8, 16, 32); form 0 and the deterministic backward need 16
  DevBuf tile_last, ws_order_f, ws_order_b, ws_q;  // per-item last contributor, work queues, queue control
  DevBuf det_part, det_keys, det_pos;
  SortWork sw_det;
  uint32_t loss_views = 0;   // views the loss is averaged over (0: the views of each call)
  float bg[3] = {0.0f, 0.0f, 0.0f};
  // targets
  uint32_t w = 0, h = 0, nt = 0;
  DevBuf tgt_own;
  // overlapped target upload: host -> staging on a copy stream, staging -> targets in stream order
  DevBuf tgt_stage;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t stage_ready = nullptr, stage_free = nullptr;
  bool stage_used = false;
  const float4* tgt = nullptr;
  // views of the current step
  uint32_t nv = 0;
  DevBuf views, tids;
  // forward state
  DevBuf recs, counts, ecounts, tmasks, rects, dkeys, dvals, cnt_sorted, offsets, total, mcount, keys, vals, ranges;
  DevBuf img, ncontrib;
  DevBuf maps, partial, loss, dimg, g2;
  SortWork sw_depth, sw_tile;
  uint32_t pair_cap = 0;
  uint32_t K = 0;
  const uint32_t* sorted_vals = nullptr;
  bool fwd_valid = false, loss_valid = false;
  nps_stats stats{};
  // device step state (see k_adam_prep)
  DevBuf stepst;
  // ADC work: alternate parameter / optimiser buffers and flags
  DevBuf p_alt, m_alt, v_alt, aflags, akeep, acand, akeep_off, acand_off, acnt, aoff, atot, psnr_acc, afeat, alogits;
  uint32_t adc_seed = 0;
  float policy_margin = 0.0f;  // keep's logit in the policy's decision (0: argmax)
  // CUDA-graph capture of the whole train step
  bool graph_mode = false, capturing = false;
  cudaGraphExec_t gexec = nullptr;
  cudaEvent_t gdone = nullptr;   // recorded after the newest replay
  cudaEvent_t gprev = nullptr;   // recorded after the replay before it
  uint32_t skip_seen = 0;        // device skip count already accounted for
  // pinned staging for set_views (copies leave without a stream sync)
  struct Stage {
    void* host = nullptr;
    size_t bytes = 0;
    cudaEvent_t done = nullptr;
  } vstage[4];
  uint32_t vstage_next = 0;
  uint32_t* h_status = nullptr;  // pinned: pair count of the last graph replay
  uint64_t gkey = 0;
  uint32_t gcap = 0, skipped = 0;
  uint32_t graph_kernels = 0;  // kernel nodes of the captured step (launches per replay)
  uint32_t timeouts_seen = 0;  // bounded-wait timeouts already reported (device counter stepst[6])
  // optional per-stage timing with CUDA events on the context stream
  bool timing = false;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> gtimers;  // event nodes of the captured graph
  bool gpending = false;  // the last replay's timers are not collected yet
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_used;
  double stage_ms[16] = {0};
  uint64_t stage_calls[16] = {0};
};

namespace {
// stage ids reported by nps_gs_stage_times
enum { ST_PRE = 0, ST_DSORT, ST_EMIT, ST_TSORT, ST_RANGES, ST_FWD, ST_LOSS, ST_BWD, ST_PBWD, ST_ADAM, ST_COUNT };
cudaEvent_t ev_get(nps_gs* o) {
  if (o->ev_pool.empty()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  cudaEvent_t e = o->ev_pool.back();
  o->ev_pool.pop_back();
  return e;
}
struct StageTimer {
  nps_gs* o;
  int id;
  cudaEvent_t e0 = nullptr;
  StageTimer(nps_gs* oo, int i) : o(oo), id(i) {
    if (o->timing) {
      e0 = ev_get(o);
      // External: while capturing, a plain record would only mark a dependency
      cudaEventRecordWithFlags(e0, o->ctx->stream, o->capturing ? cudaEventRecordExternal : 0);
    }
  }
  ~StageTimer() {
    if (o->timing) {
      cudaEvent_t e1 = ev_get(o);
      cudaEventRecordWithFlags(e1, o->ctx->stream, o->capturing ? cudaEventRecordExternal : 0);
      if (o->capturing)
        o->gtimers.push_back({id, {e0, e1}});
      else
        o->ev_used.push_back({id, {e0, e1}});
    }
  }
};
}  // namespace

namespace {
int check_gs(nps_gs* o) {
  if (!o) {
    set_error("null Gaussian trainer");
    return NPS_ERR_INVALID;
  }
  return bind_device(o->ctx);
}
int copy_in_gs(void* dst, const void* src, size_t bytes, int mem, cudaStream_t s) {
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
bool g_ssim_w_set = false;
int ensure_ssim_weights() {
  if (g_ssim_w_set) return NPS_OK;
  float w[gs::kSsimWin];
  double s = 0;
  for (int k = 0; k < gs::kSsimWin; ++k) {
    double d = k - gs::kSsimWin / 2;
    w[k] = (float)std::exp(-d * d / (2.0 * 1.5 * 1.5));
    s += w[k];
  }
  for (int k = 0; k < gs::kSsimWin; ++k) w[k] = (float)(w[k] / s);
  NPS_CUDA(cudaMemcpyToSymbol(gs::c_ssim_w, w, sizeof(w)));
  g_ssim_w_set = true;
  return NPS_OK;
}
}  // namespace

extern "C" {

int nps_gs_create(nps_ctx* ctx, uint32_t capacity, uint32_t sh_degree, nps_gs** out) {
  if (!out || capacity == 0 || capacity > (1u << 26) || sh_degree > 3) {
    set_error("nps_gs_create: bad arguments (capacity=%u, sh_degree=%u)", capacity, sh_degree);
    return NPS_ERR_INVALID;
  }
  *out = nullptr;
  NPS_TRY(bind_device(ctx));
  NPS_TRY(ensure_ssim_weights());
  nps_gs* o = new nps_gs();
  o->ctx = ctx;
  o->cap = capacity;
  o->n = 0;
  // kernels with more than 48 KB of dynamic shared memory (set outside any capture)
  if (cudaFuncSetAttribute(gs::k_ssim_fwd2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gs::kSsimFwdSmem) !=
          cudaSuccess ||
      cudaFuncSetAttribute(gs::k_ssim_bwd2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gs::kSsimBwdSmem) !=
          cudaSuccess) {
    delete o;
    set_error("nps_gs_create: cannot raise the loss kernels' shared-memory limit");
    return NPS_ERR_CUDA;
  }
  o->sh_deg = (int)sh_degree;
  const size_t pb = sizeof(float) * gsm::kP * (size_t)capacity;
  int rc = NPS_OK;
  if ((rc = o->params.ensure(pb)) || (rc = o->grads.ensure(pb)) || (rc = o->am.ensure(pb)) ||
      (rc = o->av.ensure(pb)) || (rc = o->adc_grad.ensure(sizeof(float) * capacity)) ||
      (rc = o->adc_denom.ensure(sizeof(float) * capacity)) || (rc = o->total.ensure(16)) ||
      (rc = o->mcount.ensure(16)) || (rc = o->loss.ensure(64)) || (rc = o->stepst.ensure(32))) {
    delete o;
    return rc;
  }
  cudaStream_t s = ctx->stream;
  // the sorts' look-back timeouts count with the raster kernels' (reported as NPS_ERR_TIMEOUT)
  o->sw_depth.err = o->sw_tile.err = o->sw_det.err = o->stepst.as<uint32_t>() + 6;
  for (DevBuf* b : {&o->params, &o->grads, &o->am, &o->av}) cudaMemsetAsync(b->p, 0, pb, s);
  cudaMemsetAsync(o->adc_grad.p, 0, sizeof(float) * capacity, s);
  cudaMemsetAsync(o->adc_denom.p, 0, sizeof(float) * capacity, s);
  cudaMemsetAsync(o->loss.p, 0, 64, s);
  cudaMemsetAsync(o->stepst.p, 0, 32, s);
  cudaMemsetAsync(o->total.p, 0, 16, s);
  NPS_CUDA(cudaGetLastError());
  *out = o;
  return NPS_OK;
}

int nps_gs_destroy(nps_gs* o) {
  if (!o) return NPS_OK;
  cudaSetDevice(o->ctx->device);
  cudaStreamSynchronize(o->ctx->stream);
  if (o->gexec) cudaGraphExecDestroy(o->gexec);
  if (o->copy_stream) cudaStreamSynchronize(o->copy_stream), cudaStreamDestroy(o->copy_stream);
  if (o->stage_ready) cudaEventDestroy(o->stage_ready);
  if (o->stage_free) cudaEventDestroy(o->stage_free);
  o->tgt_stage.release();
  if (o->gdone) cudaEventDestroy(o->gdone);
  if (o->gprev) cudaEventDestroy(o->gprev);
  for (auto& st : o->vstage) {
    if (st.done) cudaEventSynchronize(st.done), cudaEventDestroy(st.done);
    if (st.host) cudaFreeHost(st.host);
  }
  if (o->h_status) cudaFreeHost(o->h_status);
  for (auto& u : o->ev_used) { cudaEventDestroy(u.second.first); cudaEventDestroy(u.second.second); }
  for (auto& u : o->gtimers) { cudaEventDestroy(u.second.first); cudaEventDestroy(u.second.second); }
  for (cudaEvent_t e : o->ev_pool) cudaEventDestroy(e);
  for (DevBuf* b : {&o->p_alt, &o->m_alt, &o->v_alt, &o->aflags, &o->akeep, &o->acand, &o->akeep_off, &o->acand_off,
                    &o->acnt, &o->aoff, &o->atot, &o->psnr_acc, &o->stepst, &o->afeat, &o->alogits,
                    &o->det_part, &o->det_keys, &o->det_pos, &o->sw_det.hist, &o->sw_det.partial,
                    &o->sw_det.lookback, &o->sw_det.keys_alt, &o->sw_det.vals_alt})
    b->release();
  for (DevBuf* b : {&o->tile_last, &o->ws_order_f, &o->ws_order_b, &o->ws_q}) b->release();
  for (DevBuf* b : {&o->params, &o->grads, &o->am, &o->av, &o->adc_grad, &o->adc_denom, &o->tgt_own, &o->views,
                    &o->tids, &o->recs, &o->counts, &o->ecounts, &o->tmasks, &o->rects, &o->dkeys, &o->dvals,
                    &o->cnt_sorted, &o->offsets, &o->total, &o->mcount, &o->keys, &o->vals, &o->ranges, &o->img,
                    &o->ncontrib, &o->maps,
                    &o->partial, &o->loss, &o->dimg, &o->g2, &o->sw_depth.hist, &o->sw_depth.partial,
                    &o->sw_depth.lookback, &o->sw_depth.keys_alt, &o->sw_depth.vals_alt, &o->sw_tile.hist,
                    &o->sw_tile.partial, &o->sw_tile.lookback, &o->sw_tile.keys_alt, &o->sw_tile.vals_alt})
    b->release();
  delete o;
  return NPS_OK;
}

int nps_gs_write_params(nps_gs* o, const float* params, uint32_t first, uint32_t count, int mem) {
  NPS_TRY(check_gs(o));
  if ((uint64_t)first + count > o->cap) {
    set_error("gs_write_params: range [%u, %u) beyond capacity %u", first, first + count, o->cap);
    return NPS_ERR_INVALID;
  }
  NPS_TRY(copy_in_gs(o->params.as<float>() + (size_t)gsm::kP * first, params, sizeof(float) * gsm::kP * count, mem,
                     o->ctx->stream));
  if (first + count > o->n) o->n = first + count;
  o->fwd_valid = false;
  return NPS_OK;
}

int nps_gs_set_count(nps_gs* o, uint32_t n) {
  NPS_TRY(check_gs(o));
  if (n > o->cap) {
    set_error("gs_set_count: %u beyond capacity %u", n, o->cap);
    return NPS_ERR_INVALID;
  }
  o->n = n;
  o->fwd_valid = false;
  return NPS_OK;
}

int nps_gs_write_state(nps_gs* o, const float* adam_m, const float* adam_v, uint32_t step, int mem) {
  NPS_TRY(check_gs(o));
  const size_t pb = sizeof(float) * gsm::kP * (size_t)o->n;
  if (adam_m) NPS_TRY(copy_in_gs(o->am.p, adam_m, pb, mem, o->ctx->stream));
  if (adam_v) NPS_TRY(copy_in_gs(o->av.p, adam_v, pb, mem, o->ctx->stream));
  o->step = step;
  const uint32_t st[4] = {step, 0u, 0u, 0u};
  NPS_TRY(copy_in_gs(o->stepst.p, st, sizeof(st), NPS_MEM_HOST, o->ctx->stream));
  return NPS_OK;
}

int nps_gs_write_adc_stats(nps_gs* o, const float* adc_grad, const float* adc_denom, int mem) {
  NPS_TRY(check_gs(o));
  const size_t b = sizeof(float) * (size_t)o->n;
  if (adc_grad) NPS_TRY(copy_in_gs(o->adc_grad.p, adc_grad, b, mem, o->ctx->stream));
  if (adc_denom) NPS_TRY(copy_in_gs(o->adc_denom.p, adc_denom, b, mem, o->ctx->stream));
  return NPS_OK;
}

int nps_gs_read_state(nps_gs* o, float* params, float* grads, float* adam_m, float* adam_v, float* adc_grad,
                      float* adc_denom) {
  NPS_TRY(check_gs(o));
  cudaStream_t s = o->ctx->stream;
  const size_t pb = sizeof(float) * gsm::kP * (size_t)o->n;
  if (params) NPS_CUDA(cudaMemcpyAsync(params, o->params.p, pb, cudaMemcpyDeviceToHost, s));
  if (grads) NPS_CUDA(cudaMemcpyAsync(grads, o->grads.p, pb, cudaMemcpyDeviceToHost, s));
  if (adam_m) NPS_CUDA(cudaMemcpyAsync(adam_m, o->am.p, pb, cudaMemcpyDeviceToHost, s));
  if (adam_v) NPS_CUDA(cudaMemcpyAsync(adam_v, o->av.p, pb, cudaMemcpyDeviceToHost, s));
  if (adc_grad) NPS_CUDA(cudaMemcpyAsync(adc_grad, o->adc_grad.p, sizeof(float) * o->n, cudaMemcpyDeviceToHost, s));
  if (adc_denom)
    NPS_CUDA(cudaMemcpyAsync(adc_denom, o->adc_denom.p, sizeof(float) * o->n, cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  return NPS_OK;
}

int nps_gs_set_lr(nps_gs* o, const float* lr6) {
  NPS_TRY(check_gs(o));
  if (!lr6) return NPS_ERR_INVALID;
  for (int k = 0; k < 6; ++k) o->lr[k] = lr6[k];
  return NPS_OK;
}

int nps_gs_set_background(nps_gs* o, float r, float g, float b) {
  NPS_TRY(check_gs(o));
  o->bg[0] = r; o->bg[1] = g; o->bg[2] = b;
  o->fwd_valid = false;
  return NPS_OK;
}

int nps_gs_set_targets(nps_gs* o, const float* rgba, uint32_t w, uint32_t h, uint32_t num_targets, int mem) {
  NPS_TRY(check_gs(o));
  if (!rgba || w == 0 || h == 0 || num_targets == 0 || w > 16 * 4096 || h > 16 * 4096) {
    set_error("gs_set_targets: bad arguments");
    return NPS_ERR_INVALID;
  }
  if (((uintptr_t)rgba & 15) != 0 && mem != NPS_MEM_HOST) {
    set_error("gs_set_targets: device targets must be 16-byte aligned");
    return NPS_ERR_INVALID;
  }
  const size_t bytes = sizeof(float) * 4 * (size_t)w * h * num_targets;
  if (mem == NPS_MEM_DEVICE_BORROW) {
    o->tgt = (const float4*)rgba;
  } else {
    NPS_TRY(o->tgt_own.ensure(bytes));
    NPS_TRY(copy_in_gs(o->tgt_own.p, rgba, bytes, mem, o->ctx->stream));
    o->tgt = o->tgt_own.as<float4>();
  }
  o->w = w;
  o->h = h;
  o->nt = num_targets;
  o->fwd_valid = false;
  return NPS_OK;
}

int nps_gs_upload_targets(nps_gs* o, const float* host_images, const uint32_t* ids, uint32_t n_ids, uint32_t w,
                          uint32_t h) {
  NPS_TRY(check_gs(o));
  if (!host_images || !ids || n_ids == 0 || w == 0 || h == 0 || w > 16 * 4096 || h > 16 * 4096) {
    set_error("gs_upload_targets: bad arguments");
    return NPS_ERR_INVALID;
  }
  cudaStream_t s = o->ctx->stream;
  const size_t ib = sizeof(float) * 4 * (size_t)w * h, bytes = ib * n_ids;
  if (!o->copy_stream) {
    NPS_CUDA(cudaStreamCreateWithFlags(&o->copy_stream, cudaStreamNonBlocking));
    NPS_CUDA(cudaEventCreateWithFlags(&o->stage_ready, cudaEventDisableTiming));
    NPS_CUDA(cudaEventCreateWithFlags(&o->stage_free, cudaEventDisableTiming));
  }
  if (o->tgt_stage.bytes < bytes || o->tgt_own.bytes < bytes) {
    NPS_CUDA(cudaStreamSynchronize(s));
    NPS_CUDA(cudaStreamSynchronize(o->copy_stream));
    NPS_TRY(o->tgt_stage.ensure(bytes));
    NPS_TRY(o->tgt_own.ensure(bytes));
  }
  // the staging buffer is free once the previous staging -> targets copy ran
  if (o->stage_used) NPS_CUDA(cudaStreamWaitEvent(o->copy_stream, o->stage_free, 0));
  for (uint32_t i = 0; i < n_ids; ++i)
    NPS_CUDA(cudaMemcpyAsync(o->tgt_stage.as<char>() + i * ib, reinterpret_cast<const char*>(host_images) + ids[i] * ib,
                             ib, cudaMemcpyHostToDevice, o->copy_stream));
  NPS_CUDA(cudaEventRecord(o->stage_ready, o->copy_stream));
  // in stream order: after every step queued so far has read the old targets
  NPS_CUDA(cudaStreamWaitEvent(s, o->stage_ready, 0));
  NPS_CUDA(cudaMemcpyAsync(o->tgt_own.p, o->tgt_stage.p, bytes, cudaMemcpyDeviceToDevice, s));
  NPS_CUDA(cudaEventRecord(o->stage_free, s));
  o->stage_used = true;
  o->tgt = o->tgt_own.as<float4>();
  o->w = w;
  o->h = h;
  o->nt = n_ids;
  o->fwd_valid = false;
  return NPS_OK;
}

int nps_gs_read_loss(nps_gs* o, float* loss3_host) {
  NPS_TRY(check_gs(o));
  if (!loss3_host) return NPS_ERR_INVALID;
  NPS_CUDA(cudaMemcpyAsync(loss3_host, o->loss.p, sizeof(float) * 3, cudaMemcpyDeviceToHost, o->ctx->stream));
  NPS_CUDA(cudaStreamSynchronize(o->ctx->stream));
  return NPS_OK;
}

int nps_gs_set_image_size(nps_gs* o, uint32_t w, uint32_t h) {
  NPS_TRY(check_gs(o));
  if (w == 0 || h == 0 || w > 16 * 4096 || h > 16 * 4096) {
    set_error("gs_set_image_size: bad size %ux%u", w, h);
    return NPS_ERR_INVALID;
  }
  if (o->tgt && (o->w != w || o->h != h)) {
    set_error("gs_set_image_size: %ux%u differs from the targets' %ux%u", w, h, o->w, o->h);
    return NPS_ERR_INVALID;
  }
  o->w = w;
  o->h = h;
  o->fwd_valid = false;
  return NPS_OK;
}

int nps_gs_set_views(nps_gs* o, const float* vp, const float* vp_inv, const uint32_t* target_ids, uint32_t nv) {
  NPS_TRY(check_gs(o));
  if (!vp || !vp_inv || nv == 0 || nv > 1024) {
    set_error("gs_set_views: bad arguments");
    return NPS_ERR_INVALID;
  }
  std::vector<float> host((size_t)gsm::kViewRec * nv, 0.0f);
  std::vector<uint32_t> ids(nv, 0);
  for (uint32_t v = 0; v < nv; ++v) {
    float* r = &host[(size_t)gsm::kViewRec * v];
    std::memcpy(r, vp + 16 * v, 64);
    std::memcpy(r + 16, vp_inv + 16 * v, 64);
    // camera centre: VP^-1 (0, 0, 1, 0), dehomogenised
    const float* iv = vp_inv + 16 * v;
    const double cw = iv[11];
    if (std::fabs(cw) < 1e-30) {
      set_error("gs_set_views: view %u has no finite camera centre", v);
      return NPS_ERR_INVALID;
    }
    r[32] = (float)(iv[8] / cw);
    r[33] = (float)(iv[9] / cw);
    r[34] = (float)(iv[10] / cw);
    ids[v] = target_ids ? target_ids[v] : v;
    if (o->nt && ids[v] >= o->nt) {
      set_error("gs_set_views: target id %u out of range (%u targets)", ids[v], o->nt);
      return NPS_ERR_INVALID;
    }
  }
  NPS_TRY(o->views.ensure(sizeof(float) * host.size()));
  NPS_TRY(o->tids.ensure(sizeof(uint32_t) * nv));
  cudaStream_t s = o->ctx->stream;
  // stage through a pinned slot so that the copies queue behind in-flight
  // work instead of waiting for it; a slot is reused once its copies are done
  nps_gs::Stage& sl = o->vstage[o->vstage_next];
  o->vstage_next = (o->vstage_next + 1) % 4;
  const size_t vb = sizeof(float) * host.size(), ib = sizeof(uint32_t) * nv;
  if (sl.done) NPS_CUDA(cudaEventSynchronize(sl.done));
  else NPS_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
  if (sl.bytes < vb + ib) {
    if (sl.host) NPS_CUDA(cudaFreeHost(sl.host));
    sl.host = nullptr;
    sl.bytes = 0;
    NPS_CUDA(cudaMallocHost(&sl.host, vb + ib));
    sl.bytes = vb + ib;
  }
  std::memcpy(sl.host, host.data(), vb);
  std::memcpy(static_cast<char*>(sl.host) + vb, ids.data(), ib);
  NPS_CUDA(cudaMemcpyAsync(o->views.p, sl.host, vb, cudaMemcpyHostToDevice, s));
  NPS_CUDA(cudaMemcpyAsync(o->tids.p, static_cast<char*>(sl.host) + vb, ib, cudaMemcpyHostToDevice, s));
  NPS_CUDA(cudaEventRecord(sl.done, s));
  o->nv = nv;
  o->fwd_valid = false;
  return NPS_OK;
}

}  // extern "C"

// Forward over all views.  Eager (capture == false): reads the pair count back
// and grows the pair buffers to fit.  Captured (capture == true): no host
// synchronisation; the pair buffers keep their capacity and the emit kernel
// drops pairs beyond it (Adam then skips the step, see k_adam_prep).
// Raster launches of the current forward state, by variant (pixels per thread).
// Raster variants: (form, pixels per thread, records staged per batch), for
// a tile edge T.  Form 0: one CTA per (tile, view), records double-buffered
// (k_fwd, k_bwd2), T = 16 only; form 1: persistent warp-specialised kernels
// over a longest-first work queue (k_fwd_ws, k_bwd_ws), a 3-slot ring of
// staged records, T = 8 (1 or 2 pixels per thread), 16 (1, 2, 4) or 32 (4);
// form 2: one CTA per work item, blocks taking the items longest first
// (k_fwd and k_bwd2 ordered), T = 16.
struct RasterVariant {
  int form, ppt, stage;
};
static bool valid_variant(uint32_t tile, int form, int ppt, int stage) {
  if (form == 0 || form == 2) {
    if (tile != 16 || (ppt != 1 && ppt != 2 && ppt != 4)) return false;
    return stage == 256 / ppt || (stage == 512 / ppt && stage <= 256);
  }
  if (form != 1 || (stage != 64 && stage != 128)) return false;
  if (tile == 8) return ppt == 1 || ppt == 2;
  if (tile == 16) return (ppt == 1 && stage == 128) || ppt == 2 || ppt == 4;
  if (tile == 32) return ppt == 4;
  return false;
}
constexpr RasterVariant kVariants[] = {{0, 1, 256}, {0, 2, 128}, {0, 2, 256}, {0, 4, 64}, {0, 4, 128}, {1, 1, 64},
                                       {1, 1, 128}, {1, 2, 64},  {1, 2, 128}, {1, 4, 64}, {1, 4, 128}, {2, 1, 256},
                                       {2, 2, 128}, {2, 2, 256}, {2, 4, 64},  {2, 4, 128}};
constexpr int kNumVariants = 16;
constexpr uint32_t kTiles[] = {8, 16, 32};
constexpr int kNumTiles = 3;
// per tile in the autotuner's times: binning, then the forward and backward time of each variant
constexpr int kTuneStride = 1 + 2 * kNumVariants;

// Resident CTAs of a persistent kernel on the device (queried once per kernel).
template <class K>
static int persistent_grid(nps_gs* o, K kernel, int threads, int* cache) {
  if (*cache == 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    *cache = per_sm * o->ctx->sm_count;
  }
  return *cache;
}

static int ensure_ws_buffers(nps_gs* o, uint32_t nitems) {
  NPS_TRY(o->tile_last.ensure(sizeof(uint32_t) * (size_t)nitems));
  NPS_TRY(o->ws_order_f.ensure(sizeof(uint32_t) * (size_t)nitems));
  NPS_TRY(o->ws_order_b.ensure(sizeof(uint32_t) * (size_t)nitems));
  NPS_TRY(o->ws_q.ensure(64));
  return NPS_OK;
}

// Raster launches of the current forward state, by variant.  Both forms
// write every tile's last contributor (tile_last), which orders and bounds
// the persistent backward whatever form the forward took.
static int launch_fwd_raster(nps_gs* o, int form, int ppt, int stage) {
  cudaStream_t s = o->ctx->stream;
  const uint32_t W = o->w, H = o->h, nv = o->nv;
  const uint32_t tiles_x = div_up(W, o->tile), tiles_y = div_up(H, o->tile), num_tiles = tiles_x * tiles_y;
  const uint32_t nitems = num_tiles * nv;
  const uint32_t* rstart = o->ranges.as<uint32_t>();
  const uint32_t* rend = rstart + (size_t)num_tiles * nv;
  const float3 bg = make_float3(o->bg[0], o->bg[1], o->bg[2]);
  NPS_TRY(ensure_ws_buffers(o, nitems));
  NPS_CUDA(cudaMemsetAsync(o->tile_last.p, 0, sizeof(uint32_t) * (size_t)nitems, s));
  uint32_t* err = o->stepst.as<uint32_t>() + 6;
  if (form == 1) {
    uint32_t* q = o->ws_q.as<uint32_t>();
    gs::k_order_items<false><<<1, 1024, 0, s>>>(rstart, rend, nullptr, nitems, o->ws_order_f.as<uint32_t>(), q);
    NPS_CHECK_LAUNCH();
#define NPS_FWD_WS(TS, PPT, SB)                                                                                \
  do {                                                                                                         \
    static int grid_cache = 0;                                                                                 \
    const int grid = persistent_grid(o, gs::k_fwd_ws<TS, PPT, SB>, TS * TS / PPT + 32, &grid_cache);           \
    gs::k_fwd_ws<TS, PPT, SB><<<grid, TS * TS / PPT + 32, 0, s>>>(                                             \
        o->recs.as<gs::Rec>(), o->sorted_vals, rstart, rend, o->ws_order_f.as<uint32_t>(), q, W, H, tiles_x,   \
        num_tiles, bg, o->img.as<float4>(), o->ncontrib.as<uint32_t>(), o->tile_last.as<uint32_t>(), err);     \
  } while (0)
    if (o->tile == 8) {
      if (ppt == 1 && stage == 64) NPS_FWD_WS(8, 1, 64);
      else if (ppt == 1) NPS_FWD_WS(8, 1, 128);
      else if (stage == 64) NPS_FWD_WS(8, 2, 64);
      else NPS_FWD_WS(8, 2, 128);
    } else if (o->tile == 32) {
      if (stage == 64) NPS_FWD_WS(32, 4, 64);
      else NPS_FWD_WS(32, 4, 128);
    } else {
      if (ppt == 1) NPS_FWD_WS(16, 1, 128);
      else if (ppt == 2 && stage == 64) NPS_FWD_WS(16, 2, 64);
      else if (ppt == 2) NPS_FWD_WS(16, 2, 128);
      else if (stage == 64) NPS_FWD_WS(16, 4, 64);
      else NPS_FWD_WS(16, 4, 128);
    }
#undef NPS_FWD_WS
    NPS_CHECK_LAUNCH();
    return NPS_OK;
  }
  if (o->tile != 16) {
    set_error("gs raster: the one-CTA-per-tile kernels need 16 x 16 tiles (tile is %u)", o->tile);
    return NPS_ERR_STATE;
  }
  const bool ord = form == 2;
  if (ord) {
    gs::k_order_items<false><<<1, 1024, 0, s>>>(rstart, rend, nullptr, nitems, o->ws_order_f.as<uint32_t>(),
                                                o->ws_q.as<uint32_t>());
    NPS_CHECK_LAUNCH();
  }
  const dim3 grid = ord ? dim3(nitems, 1, 1) : dim3(tiles_x, tiles_y, nv);
#define NPS_FWD(PPT, SPS)                                                                                     \
  do {                                                                                                        \
    if (ord)                                                                                                  \
      gs::k_fwd<PPT, SPS, true><<<grid, 256 / PPT, 0, s>>>(                                                   \
          o->recs.as<gs::Rec>(), o->sorted_vals, rstart, rend, W, H, tiles_x, num_tiles, bg, o->img.as<float4>(), \
          o->ncontrib.as<uint32_t>(), o->tile_last.as<uint32_t>(), err, o->ws_order_f.as<uint32_t>());        \
    else                                                                                                      \
      gs::k_fwd<PPT, SPS, false><<<grid, 256 / PPT, 0, s>>>(                                                  \
          o->recs.as<gs::Rec>(), o->sorted_vals, rstart, rend, W, H, tiles_x, num_tiles, bg, o->img.as<float4>(), \
          o->ncontrib.as<uint32_t>(), o->tile_last.as<uint32_t>(), err, nullptr);                             \
  } while (0)
  const int sps = stage * ppt / 256;
  if (ppt == 2 && sps == 2) NPS_FWD(2, 2);
  else if (ppt == 2) NPS_FWD(2, 1);
  else if (ppt == 4 && sps == 2) NPS_FWD(4, 2);
  else if (ppt == 4) NPS_FWD(4, 1);
  else NPS_FWD(1, 1);
#undef NPS_FWD
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

static int launch_bwd_raster(nps_gs* o, int form, int ppt, int stage, const float4* dimg) {
  cudaStream_t s = o->ctx->stream;
  const uint32_t W = o->w, H = o->h, nv = o->nv;
  const uint32_t tiles_x = div_up(W, o->tile), tiles_y = div_up(H, o->tile), num_tiles = tiles_x * tiles_y;
  const uint32_t nitems = num_tiles * nv;
  const uint32_t* rstart = o->ranges.as<uint32_t>();
  const uint32_t* rend = rstart + (size_t)num_tiles * nv;
  const float3 bg = make_float3(o->bg[0], o->bg[1], o->bg[2]);
  uint32_t* err = o->stepst.as<uint32_t>() + 6;
  if (form == 1) {
    NPS_TRY(ensure_ws_buffers(o, nitems));
    uint32_t* q = o->ws_q.as<uint32_t>() + 2;
    gs::k_order_items<true><<<1, 1024, 0, s>>>(nullptr, nullptr, o->tile_last.as<uint32_t>(), nitems,
                                               o->ws_order_b.as<uint32_t>(), q);
    NPS_CHECK_LAUNCH();
#define NPS_BWD_WS(TS, PPT, SB)                                                                                \
  do {                                                                                                         \
    static int grid_cache = 0;                                                                                 \
    const int grid = persistent_grid(o, gs::k_bwd_ws<TS, PPT, SB>, TS * TS / PPT + 32, &grid_cache);           \
    gs::k_bwd_ws<TS, PPT, SB><<<grid, TS * TS / PPT + 32, 0, s>>>(                                             \
        o->recs.as<gs::Rec>(), o->sorted_vals, rstart, o->tile_last.as<uint32_t>(),                            \
        o->ws_order_b.as<uint32_t>(), q, W, H, tiles_x, num_tiles, bg, o->img.as<float4>(),                    \
        o->ncontrib.as<uint32_t>(), dimg, o->g2.as<float>(), err);                                             \
  } while (0)
    if (o->tile == 8) {
      if (ppt == 1 && stage == 64) NPS_BWD_WS(8, 1, 64);
      else if (ppt == 1) NPS_BWD_WS(8, 1, 128);
      else if (stage == 64) NPS_BWD_WS(8, 2, 64);
      else NPS_BWD_WS(8, 2, 128);
    } else if (o->tile == 32) {
      if (stage == 64) NPS_BWD_WS(32, 4, 64);
      else NPS_BWD_WS(32, 4, 128);
    } else {
      if (ppt == 1) NPS_BWD_WS(16, 1, 128);
      else if (ppt == 2 && stage == 64) NPS_BWD_WS(16, 2, 64);
      else if (ppt == 2) NPS_BWD_WS(16, 2, 128);
      else if (stage == 64) NPS_BWD_WS(16, 4, 64);
      else NPS_BWD_WS(16, 4, 128);
    }
#undef NPS_BWD_WS
    NPS_CHECK_LAUNCH();
    return NPS_OK;
  }
  if (o->tile != 16) {
    set_error("gs raster: the one-CTA-per-tile kernels need 16 x 16 tiles (tile is %u)", o->tile);
    return NPS_ERR_STATE;
  }
  if (form == 2) {
    NPS_TRY(ensure_ws_buffers(o, nitems));
    uint32_t* q = o->ws_q.as<uint32_t>() + 2;
    gs::k_order_items<true><<<1, 1024, 0, s>>>(nullptr, nullptr, o->tile_last.as<uint32_t>(), nitems,
                                               o->ws_order_b.as<uint32_t>(), q);
    NPS_CHECK_LAUNCH();
#define NPS_BWD2O(PPT, SPS)                                                                                   \
  gs::k_bwd2<PPT, SPS, true><<<nitems, 256 / PPT, 0, s>>>(o->recs.as<gs::Rec>(), o->sorted_vals, rstart, rend, W, H, \
                                                        tiles_x, num_tiles, bg, o->img.as<float4>(),              \
                                                        o->ncontrib.as<uint32_t>(), dimg, o->g2.as<float>(), err, \
                                                        o->ws_order_b.as<uint32_t>(), q)
    const int sps2 = stage * ppt / 256;
    if (ppt == 1) NPS_BWD2O(1, 1);
    else if (ppt == 2 && sps2 == 2) NPS_BWD2O(2, 2);
    else if (ppt == 2) NPS_BWD2O(2, 1);
    else if (sps2 == 2) NPS_BWD2O(4, 2);
    else NPS_BWD2O(4, 1);
#undef NPS_BWD2O
    NPS_CHECK_LAUNCH();
    return NPS_OK;
  }
  const dim3 grid(tiles_x, tiles_y, nv);
#define NPS_BWD(PPT, SPS)                                                                                     \
  gs::k_bwd2<PPT, SPS, false><<<grid, 256 / PPT, 0, s>>>(o->recs.as<gs::Rec>(), o->sorted_vals, rstart, rend, W, H, \
                                                         tiles_x, num_tiles, bg, o->img.as<float4>(),             \
                                                         o->ncontrib.as<uint32_t>(), dimg, o->g2.as<float>(), err, \
                                                         nullptr, nullptr)
  const int sps = stage * ppt / 256;
  if (ppt == 1) NPS_BWD(1, 1);
  else if (ppt == 2 && sps == 2) NPS_BWD(2, 2);
  else if (ppt == 4 && sps == 2) NPS_BWD(4, 2);
  else if (ppt == 4) NPS_BWD(4, 1);
  else NPS_BWD(2, 1);
#undef NPS_BWD
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

static int gs_forward_impl(nps_gs* o, float* out_rgba, bool capture) {
  if (o->nv == 0 || o->w == 0) {
    set_error("gs_forward: set_views and set_targets (or set_image_size) first");
    return NPS_ERR_STATE;
  }
  cudaStream_t s = o->ctx->stream;
  const uint32_t n = o->n, nv = o->nv, W = o->w, H = o->h;
  const uint32_t tiles_x = div_up(W, o->tile), tiles_y = div_up(H, o->tile), num_tiles = tiles_x * tiles_y;
  const size_t M = (size_t)n * nv;
  const size_t npix = (size_t)W * H * nv;
  if (M >= (1ull << 31) || (uint64_t)num_tiles * nv >= (1ull << 31)) {
    set_error("gs_forward: problem too large");
    return NPS_ERR_INVALID;
  }
  NPS_TRY(o->recs.ensure(sizeof(gs::Rec) * (M + 1)));
  NPS_TRY(o->counts.ensure(sizeof(uint32_t) * (M + 1)));
  NPS_TRY(o->ecounts.ensure(sizeof(uint32_t) * (M + 1)));
  NPS_TRY(o->tmasks.ensure(sizeof(uint32_t) * (M + 1)));
  NPS_TRY(o->rects.ensure(sizeof(uint2) * (M + 1)));
  NPS_TRY(o->dkeys.ensure(sizeof(uint32_t) * (M + 1)));
  NPS_TRY(o->dvals.ensure(sizeof(uint32_t) * (M + 1)));
  NPS_TRY(o->cnt_sorted.ensure(sizeof(uint32_t) * (M + 1)));
  NPS_TRY(o->offsets.ensure(sizeof(uint32_t) * (M + 1)));
  NPS_TRY(o->ranges.ensure(sizeof(uint32_t) * 2 * (size_t)num_tiles * nv));
  NPS_TRY(o->img.ensure(sizeof(float4) * npix));
  NPS_TRY(o->ncontrib.ensure(sizeof(uint32_t) * npix));
  uint32_t* rstart = o->ranges.as<uint32_t>();
  uint32_t* rend = rstart + (size_t)num_tiles * nv;
  NPS_CUDA(cudaMemsetAsync(o->ranges.p, 0, sizeof(uint32_t) * 2 * (size_t)num_tiles * nv, s));
  uint32_t K = 0;
  const uint32_t* vs = o->counts.as<uint32_t>();
  if (M > 0) {
    { StageTimer t_pre(o, ST_PRE);
#define NPS_PRE(D)                                                                                          \
  gs::k_preprocess<D><<<div_up(M, 256), 256, 0, s>>>(o->params.as<float>(), n, o->views.as<float>(), nv, W, H, \
                                                      tiles_x, tiles_y, 1.0f / (float)o->tile,                  \
                                                      o->recs.as<gs::Rec>(),                                    \
                                                      o->counts.as<uint32_t>(), o->rects.as<uint2>(),           \
                                                      o->dkeys.as<uint32_t>(), o->dvals.as<uint32_t>(),         \
                                                      o->ecounts.as<uint32_t>(), o->tmasks.as<uint32_t>())
    switch (o->sh_deg) {
      case 0: NPS_PRE(0); break;
      case 1: NPS_PRE(1); break;
      case 2: NPS_PRE(2); break;
      default: NPS_PRE(3); break;
    }
#undef NPS_PRE
    NPS_CHECK_LAUNCH(); }
    k_set_u32<<<1, 1, 0, s>>>(o->mcount.as<uint32_t>(), (uint32_t)M);
    uint32_t *dk = nullptr, *dv = nullptr;
    { StageTimer t(o, ST_DSORT);
    NPS_TRY(radix_sort_u32(o->dkeys.as<uint32_t>(), o->dvals.as<uint32_t>(), o->mcount.as<uint32_t>(), (uint32_t)M, 32,
                           o->sw_depth, s, &dk, &dv)); }
    o->sorted_vals = dv;
    gs::k_gather_counts<<<div_up(M, 256), 256, 0, s>>>(dv, o->ecounts.as<uint32_t>(), (uint32_t)M,
                                                        o->cnt_sorted.as<uint32_t>());
    NPS_CHECK_LAUNCH();
    uint32_t* total = o->total.as<uint32_t>();
    NPS_TRY(exclusive_scan_u32(o->cnt_sorted.as<uint32_t>(), o->offsets.as<uint32_t>(), (uint32_t)M, total, o->sw_tile,
                               s));
    if (!capture) {
      uint32_t tmo = 0;
      NPS_CUDA(cudaMemcpyAsync(&K, total, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      NPS_CUDA(cudaMemcpyAsync(&tmo, o->stepst.as<uint32_t>() + 6, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      NPS_CUDA(cudaStreamSynchronize(s));
      if (tmo != o->timeouts_seen) {
        // reported here: the next Adam step must not skip for it again
        o->timeouts_seen = tmo;
        k_set_u32<<<1, 1, 0, s>>>(o->stepst.as<uint32_t>() + 7, tmo);
        set_error("gs_forward: a bounded device wait (sort look-back or raster staging) gave up in this or an "
                  "earlier call; its results were incomplete and no update used them");
        return NPS_ERR_TIMEOUT;
      }
      if (K > o->pair_cap || o->pair_cap == 0) {
        const uint32_t cap = K + K / 4 + 4096;
        NPS_TRY(o->keys.ensure(sizeof(uint32_t) * (size_t)cap));
        NPS_TRY(o->vals.ensure(sizeof(uint32_t) * (size_t)cap));
        o->pair_cap = cap;
      }
    }
    if (K > 0 || capture) {
      { StageTimer t(o, ST_EMIT);
      gs::k_emit<<<div_up(M, 256), 256, 0, s>>>(dv, o->ecounts.as<uint32_t>(), o->offsets.as<uint32_t>(),
                                                 o->rects.as<uint2>(), o->tmasks.as<uint32_t>(), (uint32_t)M, n,
                                                 tiles_x, num_tiles, o->pair_cap,
                                                 o->keys.as<uint32_t>(), o->vals.as<uint32_t>());
      NPS_CHECK_LAUNCH(); }
      int bits = 1;
      while ((1ull << bits) < (uint64_t)num_tiles * nv) ++bits;
      uint32_t *ks = nullptr, *vv = nullptr;
      { StageTimer t(o, ST_TSORT);
      NPS_TRY(radix_sort_u32(o->keys.as<uint32_t>(), o->vals.as<uint32_t>(), total, o->pair_cap, bits, o->sw_tile, s,
                             &ks, &vv)); }
      { StageTimer t(o, ST_RANGES);
      gs::k_ranges<<<16 * kNumSMs, 256, 0, s>>>(ks, total, o->pair_cap, rstart, rend);
      NPS_CHECK_LAUNCH(); }
      vs = vv;
    }
  }
  o->K = K;
  o->sorted_vals = vs;
  const float3 bg = make_float3(o->bg[0], o->bg[1], o->bg[2]);
  StageTimer t_fwd(o, ST_FWD);
  NPS_TRY(launch_fwd_raster(o, o->fwd_form, o->fwd_ppt, o->fwd_stage));
  NPS_CHECK_LAUNCH();
  if (out_rgba) NPS_CUDA(cudaMemcpyAsync(out_rgba, o->img.p, sizeof(float4) * npix, cudaMemcpyDeviceToDevice, s));
  o->fwd_valid = true;
  o->loss_valid = false;
  if (!capture) o->stats.pairs = K;
  return NPS_OK;
}

extern "C" {

int nps_gs_forward(nps_gs* o, float* out_rgba) {
  NPS_TRY(check_gs(o));
  return gs_forward_impl(o, out_rgba, false);
}

int nps_gs_loss(nps_gs* o, float* loss3_host) {
  NPS_TRY(check_gs(o));
  if (!o->fwd_valid || !o->tgt) {
    set_error("gs_loss: forward (and set_targets) first");
    return NPS_ERR_STATE;
  }
  cudaStream_t s = o->ctx->stream;
  const uint32_t W = o->w, H = o->h, nv = o->nv;
  const size_t npix = (size_t)W * H * nv;
  const uint32_t lv = o->loss_views ? o->loss_views : nv;
  const float inv_norm = (float)(1.0 / (3.0 * (double)W * H * lv));
  NPS_TRY(o->dimg.ensure(sizeof(float4) * npix));
  if (o->loss_kind != gs::kLossL1Dssim) {
    const dim3 grid(std::min(gs::kPixLossBlocks, div_up((size_t)W * H, 256)), nv);
    const uint32_t nblocks = grid.x * grid.y;
    NPS_TRY(o->partial.ensure(sizeof(float) * 2 * nblocks));
    StageTimer t(o, ST_LOSS);
    if (o->loss_kind == gs::kLossL2)
      gs::k_pix_loss<gs::kLossL2><<<grid, 256, 0, s>>>(o->img.as<float4>(), o->tgt, o->tids.as<uint32_t>(), W * H,
                                                       inv_norm, o->dimg.as<float4>(), o->partial.as<float>());
    else
      gs::k_pix_loss<gs::kLossL1><<<grid, 256, 0, s>>>(o->img.as<float4>(), o->tgt, o->tids.as<uint32_t>(), W * H,
                                                       inv_norm, o->dimg.as<float4>(), o->partial.as<float>());
    gs::k_loss_reduce<<<1, gs::kThreads, 0, s>>>(o->partial.as<float>(), nblocks, o->loss_kind, 0.0f, inv_norm,
                                                 (float)nv / (float)lv, o->loss.as<float>());
    NPS_CHECK_LAUNCH();
  } else {
    const dim3 grid(div_up(W, gs::kLT), div_up(H, gs::kLT), nv);
    const uint32_t nblocks = grid.x * grid.y * grid.z;
    NPS_TRY(o->maps.ensure(sizeof(float) * 9 * npix));
    NPS_TRY(o->partial.ensure(sizeof(float) * 2 * nblocks));
    StageTimer t(o, ST_LOSS);
    gs::k_ssim_fwd2<<<grid, 256, gs::kSsimFwdSmem, s>>>(o->img.as<float4>(), o->tgt, o->tids.as<uint32_t>(), W, H,
                                                       o->lambda, inv_norm, o->maps.as<float>(),
                                                       o->partial.as<float>());
    gs::k_ssim_bwd2<<<grid, 256, gs::kSsimBwdSmem, s>>>(o->img.as<float4>(), o->tgt, o->tids.as<uint32_t>(),
                                                       o->maps.as<float>(), W, H, o->lambda, inv_norm,
                                                       o->dimg.as<float4>());
    gs::k_loss_reduce<<<1, gs::kThreads, 0, s>>>(o->partial.as<float>(), nblocks, o->loss_kind, o->lambda,
                                                 inv_norm, (float)nv / (float)lv, o->loss.as<float>());
    NPS_CHECK_LAUNCH();
  }
  if (loss3_host) {
    NPS_CUDA(cudaMemcpyAsync(loss3_host, o->loss.p, sizeof(float) * 3, cudaMemcpyDeviceToHost, s));
    NPS_CUDA(cudaStreamSynchronize(s));
  }
  o->loss_valid = true;
  return NPS_OK;
}

int nps_gs_backward(nps_gs* o, const float* dl_dimg) {
  NPS_TRY(check_gs(o));
  if (!o->fwd_valid) {
    set_error("gs_backward: forward first");
    return NPS_ERR_STATE;
  }
  if (!dl_dimg && !o->loss_valid) {
    set_error("gs_backward: no image gradient given and no fused loss computed");
    return NPS_ERR_STATE;
  }
  cudaStream_t s = o->ctx->stream;
  const uint32_t n = o->n, nv = o->nv, W = o->w, H = o->h;
  const uint32_t tiles_x = div_up(W, o->tile), tiles_y = div_up(H, o->tile), num_tiles = tiles_x * tiles_y;
  const size_t M = (size_t)n * nv;
  NPS_TRY(o->g2.ensure(sizeof(float) * gs::kG2 * (M + 1)));
  NPS_CUDA(cudaMemsetAsync(o->g2.p, 0, sizeof(float) * gs::kG2 * M, s));
  const uint32_t* rstart = o->ranges.as<uint32_t>();
  const uint32_t* rend = rstart + (size_t)num_tiles * nv;
  const float3 bg = make_float3(o->bg[0], o->bg[1], o->bg[2]);
  const float4* dimg = dl_dimg ? (const float4*)dl_dimg : o->dimg.as<float4>();
  if (!o->deterministic) {
    StageTimer t(o, ST_BWD);
    NPS_TRY(launch_bwd_raster(o, o->bwd_form, o->bwd_ppt, o->bwd_stage, dimg));
    NPS_CHECK_LAUNCH();
  } else if (o->pair_cap > 0) {
    if (o->tile != 16) {
      set_error("gs_backward: the deterministic backward needs 16 x 16 tiles (tile is %u)", o->tile);
      return NPS_ERR_STATE;
    }
    StageTimer t(o, ST_BWD);
    const uint32_t cap = o->pair_cap;
    NPS_TRY(o->det_part.ensure(sizeof(float) * 10 * (size_t)cap));
    NPS_TRY(o->det_keys.ensure(sizeof(uint32_t) * (size_t)cap));
    NPS_TRY(o->det_pos.ensure(sizeof(uint32_t) * (size_t)cap));
    NPS_CUDA(cudaMemsetAsync(o->det_part.p, 0, sizeof(float) * 10 * (size_t)cap, s));
    gs::k_bwd<true><<<dim3(tiles_x, tiles_y, nv), gs::kThreads, 0, s>>>(
        o->recs.as<gs::Rec>(), o->sorted_vals, rstart, rend, W, H, tiles_x, num_tiles, bg, o->img.as<float4>(),
        o->ncontrib.as<uint32_t>(), dimg, nullptr, o->det_part.as<float>());
    NPS_CHECK_LAUNCH();
    const uint32_t* total = o->total.as<uint32_t>();
    gs::k_det_prep<<<4 * kNumSMs, 256, 0, s>>>(o->sorted_vals, total, cap, o->det_keys.as<uint32_t>(),
                                               o->det_pos.as<uint32_t>());
    NPS_CHECK_LAUNCH();
    int bits = 1;
    while (bits < 32 && ((uint64_t)1 << bits) < (uint64_t)M) ++bits;
    uint32_t *ko = nullptr, *vo = nullptr;
    NPS_TRY(radix_sort_u32(o->det_keys.as<uint32_t>(), o->det_pos.as<uint32_t>(), total, cap, bits, o->sw_det, s,
                           &ko, &vo));
    gs::k_det_segsum<<<4 * kNumSMs, 256, 0, s>>>(ko, vo, total, cap, o->det_part.as<float>(), o->g2.as<float>());
    NPS_CHECK_LAUNCH();
  }
  if (n > 0) {
    StageTimer t(o, ST_PBWD);
    const uint32_t blocks = div_up((size_t)n * 8, 128);
    const float adc_scale = (float)(o->loss_views ? o->loss_views : nv);
#define NPS_PBWD1(D, ONE)                                                                                        \
  gs::k_project_bwd<D, ONE><<<blocks, 128, 0, s>>>(o->params.as<float>(), n, o->views.as<float>(), nv, W, H,     \
                                                    o->counts.as<uint32_t>(), o->g2.as<float>(),                  \
                                                    o->grads.as<float>(), o->adc_grad.as<float>(),                \
                                                    o->adc_denom.as<float>(), o->accumulate ? 1 : 0, adc_scale)
#define NPS_PBWD(D)            \
  if (nv <= 8) {               \
    NPS_PBWD1(D, true);        \
  } else {                     \
    NPS_PBWD1(D, false);       \
  }
    switch (o->sh_deg) {
      case 0: NPS_PBWD(0); break;
      case 1: NPS_PBWD(1); break;
      case 2: NPS_PBWD(2); break;
      default: NPS_PBWD(3); break;
    }
#undef NPS_PBWD
    NPS_CHECK_LAUNCH();
  }
  return NPS_OK;
}

int nps_gs_backward_host(nps_gs* o, const float* dl_dimg_host) {
  NPS_TRY(check_gs(o));
  if (!dl_dimg_host) {
    set_error("gs_backward_host: null image gradient");
    return NPS_ERR_INVALID;
  }
  if (!o->fwd_valid) {
    set_error("gs_backward: forward first");
    return NPS_ERR_STATE;
  }
  const size_t bytes = sizeof(float4) * (size_t)o->w * o->h * o->nv;
  NPS_TRY(o->dimg.ensure(bytes));
  NPS_TRY(copy_in_gs(o->dimg.p, dl_dimg_host, bytes, NPS_MEM_HOST, o->ctx->stream));
  o->loss_valid = false;  // the stored gradient is no longer the fused loss's
  return nps_gs_backward(o, o->dimg.as<float>());
}

int nps_gs_adam(nps_gs* o) {
  NPS_TRY(check_gs(o));
  if (o->n == 0) return NPS_OK;
  o->step += 1;
  gs::AdamArgs a;
  for (int k = 0; k < 6; ++k) a.lr[k] = o->lr[k];
  a.b1 = 0.9f;
  a.b2 = 0.999f;
  a.eps = 1e-15f;
  const uint32_t n4 = o->n * 16;
  StageTimer t_adam(o, ST_ADAM);
  gs::k_adam_prep<<<1, 1, 0, o->ctx->stream>>>(o->stepst.as<uint32_t>(), o->total.as<uint32_t>(),
                                               o->pair_cap ? o->pair_cap : 0xffffffffu);
  gs::k_adam<<<div_up(n4, 256), 256, 0, o->ctx->stream>>>(o->params.as<float4>(), o->grads.as<float4>(),
                                                           o->am.as<float4>(), o->av.as<float4>(), n4, a,
                                                           o->stepst.as<uint32_t>());
  NPS_CHECK_LAUNCH();
  o->fwd_valid = false;
  return NPS_OK;
}

}  // extern "C"

static int gs_step_eager(nps_gs* o) {
  NPS_TRY(gs_forward_impl(o, nullptr, false));
  NPS_TRY(nps_gs_loss(o, nullptr));
  NPS_TRY(nps_gs_backward(o, nullptr));
  NPS_TRY(nps_gs_adam(o));
  return NPS_OK;
}

// Captures forward + loss + backward + Adam (no host synchronisation inside)
// and instantiates it.  All buffers already have their sizes from an eager
// step, so nothing is allocated while capturing.
// Adds the stage times of the last graph replay (waits for it to finish).
static int collect_graph_timers(nps_gs* o) {
  if (!o->gpending) return NPS_OK;
  o->gpending = false;
  NPS_CUDA(cudaEventSynchronize(o->gdone));
  for (auto& g : o->gtimers) {
    float t = 0.0f;
    NPS_CUDA(cudaEventElapsedTime(&t, g.second.first, g.second.second));
    o->stage_ms[g.first] += t;
    o->stage_calls[g.first] += 1;
  }
  return NPS_OK;
}

static int gs_capture(nps_gs* o) {
  cudaStream_t s = o->ctx->stream;
  NPS_TRY(collect_graph_timers(o));
  if (o->gexec) {
    cudaGraphExecDestroy(o->gexec);
    o->gexec = nullptr;
  }
  for (auto& g : o->gtimers) {
    o->ev_pool.push_back(g.second.first);
    o->ev_pool.push_back(g.second.second);
  }
  o->gtimers.clear();
  if (!o->h_status) {
    NPS_CUDA(cudaMallocHost((void**)&o->h_status, 16));
    std::memset(o->h_status, 0, 16);  // page-locked memory may be reused: no stale status words
  }
  if (!o->gdone) NPS_CUDA(cudaEventCreateWithFlags(&o->gdone, cudaEventDisableTiming));
  if (!o->gprev) NPS_CUDA(cudaEventCreateWithFlags(&o->gprev, cudaEventDisableTiming));
  NPS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  o->capturing = true;
  const uint32_t step_before = o->step;
  int rc = gs_forward_impl(o, nullptr, true);
  if (rc == NPS_OK) rc = nps_gs_loss(o, nullptr);
  if (rc == NPS_OK) rc = nps_gs_backward(o, nullptr);
  if (rc == NPS_OK) rc = nps_gs_adam(o);
  if (rc == NPS_OK) {
    cudaError_t e = cudaMemcpyAsync(o->h_status, o->total.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(o->h_status + 1, o->stepst.as<uint32_t>() + 4, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(o->h_status + 2, o->stepst.as<uint32_t>() + 6, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) {
      set_error("graph capture: %s", cudaGetErrorString(e));
      rc = NPS_ERR_CUDA;
    }
  }
  o->capturing = false;
  o->step = step_before;  // captured, not executed
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(s, &graph);
  if (rc != NPS_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ee != cudaSuccess) {
    set_error("graph capture failed: %s", cudaGetErrorString(ee));
    return NPS_ERR_CUDA;
  }
  // kernel launches per replay: the graph's kernel nodes
  size_t nn = 0;
  uint32_t nk = 0;
  if (cudaGraphGetNodes(graph, nullptr, &nn) == cudaSuccess && nn > 0) {
    std::vector<cudaGraphNode_t> nodes(nn);
    if (cudaGraphGetNodes(graph, nodes.data(), &nn) == cudaSuccess)
      for (size_t i = 0; i < nn; ++i) {
        cudaGraphNodeType ty;
        if (cudaGraphNodeGetType(nodes[i], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++nk;
      }
  }
  o->graph_kernels = nk;
  const cudaError_t ie = cudaGraphInstantiate(&o->gexec, graph, 0);
  cudaGraphDestroy(graph);
  if (ie != cudaSuccess) {
    o->gexec = nullptr;
    set_error("graph instantiate failed: %s", cudaGetErrorString(ie));
    return NPS_ERR_CUDA;
  }
  o->gcap = o->pair_cap;
  return NPS_OK;
}

extern "C" {

int nps_gs_set_graph(nps_gs* o, int enable) {
  NPS_TRY(check_gs(o));
  o->graph_mode = enable != 0;
  if (!o->graph_mode && o->gexec) {
    NPS_CUDA(cudaStreamSynchronize(o->ctx->stream));
    cudaGraphExecDestroy(o->gexec);
    o->gexec = nullptr;
  }
  return NPS_OK;
}

int nps_gs_train_step(nps_gs* o, float* loss3_host) {
  NPS_TRY(check_gs(o));
  cudaStream_t s = o->ctx->stream;
  if (!o->graph_mode) {
    NPS_TRY(gs_step_eager(o));
  } else {
    // shape of the captured step; anything else in it reads device memory
    const uint64_t key = ((uint64_t)o->n * 1000003ull) ^ ((uint64_t)o->nv << 40) ^ ((uint64_t)o->w << 20) ^
                         ((uint64_t)o->h << 4) ^ (uint64_t)o->sh_deg ^ ((uint64_t)(uintptr_t)o->tgt << 7) ^
                         ((uint64_t)__builtin_bit_cast(uint32_t, o->bg[0]) << 3) ^ (uint64_t)o->lambda * 131ull;
    if (o->gexec) {
      // at most two replays in flight (one while stage timers are read, since
      // their event nodes are shared by all replays)
      NPS_CUDA(cudaEventSynchronize(o->timing ? o->gdone : o->gprev));
      if (o->timing) NPS_TRY(collect_graph_timers(o));
      const uint32_t sk = o->h_status[1];
      if (sk != o->skip_seen) {
        // a replay overflowed its pair buffers and skipped its update
        o->skipped += sk - o->skip_seen;
        o->skip_seen = sk;
        o->gkey = 0;
      }
      if (o->h_status[2] != o->timeouts_seen) {
        o->timeouts_seen = o->h_status[2];
        set_error("gs_train_step: a bounded device wait (sort look-back or raster staging) gave up in an earlier "
                  "step (its update was skipped); this step was not run");
        return NPS_ERR_TIMEOUT;
      }
    }
    if (!o->gexec || key != o->gkey) {
      NPS_TRY(collect_graph_timers(o));
      NPS_TRY(gs_step_eager(o));  // sizes every buffer (and is this call's step)
      NPS_TRY(gs_capture(o));
      NPS_CUDA(cudaStreamSynchronize(s));
      o->skip_seen = o->h_status[1] = 0;
      o->h_status[2] = o->timeouts_seen;  // what the replays report until a wait gives up
      NPS_CUDA(cudaMemsetAsync(o->stepst.as<uint32_t>() + 4, 0, sizeof(uint32_t), s));
      o->gkey = key;
    } else {
      NPS_CUDA(cudaGraphLaunch(o->gexec, s));
      std::swap(o->gdone, o->gprev);
      NPS_CUDA(cudaEventRecord(o->gdone, s));
      o->step += 1;
      o->fwd_valid = false;
      // stage times are read at the next call (or by nps_gs_stage_times)
      o->gpending = o->timing && !o->gtimers.empty();
    }
  }
  if (loss3_host) {
    // the step's loss, read once the whole step (Adam included) has finished
    NPS_CUDA(cudaMemcpyAsync(loss3_host, o->loss.p, sizeof(float) * 3, cudaMemcpyDeviceToHost, s));
    NPS_CUDA(cudaStreamSynchronize(s));
  }
  return NPS_OK;
}

int nps_gs_read_image(nps_gs* o, float* rgba, float* dl_dimage) {
  NPS_TRY(check_gs(o));
  const size_t bytes = sizeof(float4) * (size_t)o->w * o->h * o->nv;
  cudaStream_t s = o->ctx->stream;
  if (rgba) {
    if (!o->fwd_valid) {
      set_error("gs_read_image: no forward state");
      return NPS_ERR_STATE;
    }
    NPS_CUDA(cudaMemcpyAsync(rgba, o->img.p, bytes, cudaMemcpyDeviceToHost, s));
  }
  if (dl_dimage) {
    if (!o->loss_valid) {
      set_error("gs_read_image: no loss gradient");
      return NPS_ERR_STATE;
    }
    NPS_CUDA(cudaMemcpyAsync(dl_dimage, o->dimg.p, bytes, cudaMemcpyDeviceToHost, s));
  }
  NPS_CUDA(cudaStreamSynchronize(s));
  return NPS_OK;
}

int nps_gs_buffers(nps_gs* o, float** params, float** grads, float** adam_m, float** adam_v, float** image,
                   float** dl_dimage) {
  NPS_TRY(check_gs(o));
  if (params) *params = o->params.as<float>();
  if (grads) *grads = o->grads.as<float>();
  if (adam_m) *adam_m = o->am.as<float>();
  if (adam_v) *adam_v = o->av.as<float>();
  if (image) *image = o->img.as<float>();
  if (dl_dimage) *dl_dimage = o->dimg.as<float>();
  return NPS_OK;
}

int nps_gs_adc_buffers(nps_gs* o, float** adc_grad, float** adc_denom) {
  NPS_TRY(check_gs(o));
  if (adc_grad) *adc_grad = o->adc_grad.as<float>();
  if (adc_denom) *adc_denom = o->adc_denom.as<float>();
  return NPS_OK;
}

}  // extern "C"

namespace {
int adc_prepare(nps_gs* o) {
  const uint32_t n = o->n;
  const size_t pb = sizeof(float) * gsm::kP * (size_t)o->cap;
  NPS_TRY(o->p_alt.ensure(pb));
  NPS_TRY(o->m_alt.ensure(pb));
  NPS_TRY(o->v_alt.ensure(pb));
  for (DevBuf* b : {&o->aflags, &o->akeep, &o->acand, &o->akeep_off, &o->acand_off, &o->acnt, &o->aoff})
    NPS_TRY(b->ensure(sizeof(uint32_t) * (n + 1)));
  NPS_TRY(o->atot.ensure(16));
  return NPS_OK;
}

// Applies the flags in o->aflags (with keep / candidate indicators in akeep /
// acand): densify the first candidates that fit the capacity, compact.
int adc_apply(nps_gs* o, const gs::AdcParams& a, uint32_t* counts4) {
  cudaStream_t s = o->ctx->stream;
  const uint32_t n = o->n;
  uint32_t* tot = o->atot.as<uint32_t>();
  NPS_TRY(exclusive_scan_u32(o->akeep.as<uint32_t>(), o->akeep_off.as<uint32_t>(), n, tot, o->sw_tile, s));
  NPS_TRY(exclusive_scan_u32(o->acand.as<uint32_t>(), o->acand_off.as<uint32_t>(), n, tot + 1, o->sw_tile, s));
  uint32_t h[2] = {0, 0};
  NPS_CUDA(cudaMemcpyAsync(h, tot, sizeof(h), cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  const uint32_t kept = h[0], cands = h[1];
  const uint32_t budget = o->cap > kept ? o->cap - kept : 0;
  gs::k_adc_count<<<div_up(n, 256), 256, 0, s>>>(o->aflags.as<uint32_t>(), o->acand_off.as<uint32_t>(), n, budget,
                                                 o->acnt.as<uint32_t>());
  NPS_TRY(exclusive_scan_u32(o->acnt.as<uint32_t>(), o->aoff.as<uint32_t>(), n, tot + 2, o->sw_tile, s));
  uint32_t nn = 0;
  NPS_CUDA(cudaMemcpyAsync(&nn, tot + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  gs::k_adc_scatter<<<div_up((size_t)n * 16, 256), 256, 0, s>>>(
      o->params.as<float4>(), o->am.as<float4>(), o->av.as<float4>(), o->aflags.as<uint32_t>(),
      o->acnt.as<uint32_t>(), o->aoff.as<uint32_t>(), n, a, o->p_alt.as<float4>(), o->m_alt.as<float4>(),
      o->v_alt.as<float4>());
  NPS_CHECK_LAUNCH();
  NPS_CUDA(cudaStreamSynchronize(s));
  std::swap(o->params, o->p_alt);
  std::swap(o->am, o->m_alt);
  std::swap(o->av, o->v_alt);
  o->gkey = 0;  // a captured step holds the old buffers and count
  NPS_CUDA(cudaMemsetAsync(o->adc_grad.p, 0, sizeof(float) * o->cap, s));
  NPS_CUDA(cudaMemsetAsync(o->adc_denom.p, 0, sizeof(float) * o->cap, s));
  if (counts4) {
    counts4[0] = n;
    counts4[1] = nn;
    counts4[2] = std::min(cands, budget);
    counts4[3] = n - kept;
  }
  o->n = nn;
  o->fwd_valid = false;
  return NPS_OK;
}
}  // namespace

extern "C" {

int nps_gs_adc(nps_gs* o, float grad_thresh, float split_scale, float prune_opacity, uint32_t* counts4) {
  NPS_TRY(check_gs(o));
  if (counts4) counts4[0] = counts4[1] = counts4[2] = counts4[3] = 0;
  const uint32_t n = o->n;
  if (n == 0) return NPS_OK;
  NPS_TRY(adc_prepare(o));
  gs::AdcParams a{grad_thresh, split_scale, prune_opacity, ++o->adc_seed};
  gs::k_adc_classify<<<div_up(n, 256), 256, 0, o->ctx->stream>>>(
      o->params.as<float>(), o->adc_grad.as<float>(), o->adc_denom.as<float>(), n, a, o->aflags.as<uint32_t>(),
      o->akeep.as<uint32_t>(), o->acand.as<uint32_t>());
  NPS_CHECK_LAUNCH();
  return adc_apply(o, a, counts4);
}

int nps_gs_adc_features(nps_gs* o, float step_frac, float grad_thresh, float split_scale, float prune_opacity,
                        float* features_dev, uint8_t* plain_dev, uint32_t* ids_dev) {
  NPS_TRY(check_gs(o));
  if (!features_dev) return NPS_ERR_INVALID;
  const uint32_t n = o->n;
  if (n == 0) return NPS_OK;
  gs::AdcParams a{grad_thresh, split_scale, prune_opacity, 0};
  gs::k_adc_features<<<div_up(n, 256), 256, 0, o->ctx->stream>>>(
      o->params.as<float>(), o->am.as<float>(), o->av.as<float>(), o->adc_grad.as<float>(), o->adc_denom.as<float>(),
      n, a, step_frac, features_dev, plain_dev, ids_dev);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int nps_gs_set_policy_margin(nps_gs* o, float margin) {
  NPS_TRY(check_gs(o));
  o->policy_margin = margin;
  return NPS_OK;
}

int nps_gs_assign_ids(nps_gs* o, uint32_t base) {
  NPS_TRY(check_gs(o));
  if (o->n == 0) return NPS_OK;
  gs::k_assign_ids<<<div_up(o->n, 256), 256, 0, o->ctx->stream>>>(o->params.as<float>(), o->n, base);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int nps_gs_adc_policy(nps_gs* o, nps_mlp* policy, float step_frac, float grad_thresh, float split_scale,
                      float prune_opacity, uint32_t* counts4, uint32_t* fallback_host) {
  NPS_TRY(check_gs(o));
  if (counts4) counts4[0] = counts4[1] = counts4[2] = counts4[3] = 0;
  if (fallback_host) *fallback_host = 0;
  if (!policy) {
    // no network: the plain threshold rule
    if (fallback_host) *fallback_host = o->n;
    return nps_gs_adc(o, grad_thresh, split_scale, prune_opacity, counts4);
  }
  const uint32_t n = o->n;
  if (n == 0) return NPS_OK;
  NPS_TRY(adc_prepare(o));
  cudaStream_t s = o->ctx->stream;
  NPS_TRY(o->afeat.ensure(sizeof(float) * 16 * (size_t)n));
  NPS_TRY(o->alogits.ensure(sizeof(float) * 3 * (size_t)n + 16));
  gs::AdcParams a{grad_thresh, split_scale, prune_opacity, ++o->adc_seed};
  gs::k_adc_features<<<div_up(n, 256), 256, 0, s>>>(o->params.as<float>(), o->am.as<float>(), o->av.as<float>(),
                                                    o->adc_grad.as<float>(), o->adc_denom.as<float>(), n, a,
                                                    step_frac, o->afeat.as<float>(), nullptr, nullptr);
  NPS_CHECK_LAUNCH();
  NPS_TRY(nps_mlp_forward(policy, o->afeat.as<float>(), n, o->alogits.as<float>()));
  uint32_t* fb = o->alogits.as<uint32_t>() + 3 * (size_t)n;
  NPS_CUDA(cudaMemsetAsync(fb, 0, 4, s));
  gs::k_adc_policy_flags<<<div_up(n, 256), 256, 0, s>>>(o->alogits.as<float>(), o->params.as<float>(),
                                                        o->adc_grad.as<float>(), o->adc_denom.as<float>(), n, a,
                                                        o->aflags.as<uint32_t>(), o->akeep.as<uint32_t>(),
                                                        o->acand.as<uint32_t>(), fb, o->policy_margin);
  NPS_CHECK_LAUNCH();
  if (fallback_host) NPS_CUDA(cudaMemcpyAsync(fallback_host, fb, 4, cudaMemcpyDeviceToHost, s));
  return adc_apply(o, a, counts4);
}

int nps_gs_psnr(nps_gs* o, float* psnr_host) {
  NPS_TRY(check_gs(o));
  if (!o->fwd_valid || !o->tgt || !psnr_host) {
    set_error("gs_psnr: forward (and set_targets) first");
    return NPS_ERR_STATE;
  }
  cudaStream_t s = o->ctx->stream;
  NPS_TRY(o->psnr_acc.ensure(sizeof(double) * o->nv));
  NPS_CUDA(cudaMemsetAsync(o->psnr_acc.p, 0, sizeof(double) * o->nv, s));
  gs::k_sq_err<<<dim3(2 * kNumSMs, o->nv), 256, 0, s>>>(o->img.as<float4>(), o->tgt, o->tids.as<uint32_t>(), o->w,
                                                        o->h, o->psnr_acc.as<double>());
  NPS_CHECK_LAUNCH();
  std::vector<double> acc(o->nv);
  NPS_CUDA(cudaMemcpyAsync(acc.data(), o->psnr_acc.p, sizeof(double) * o->nv, cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  for (uint32_t v = 0; v < o->nv; ++v) {
    const double mse = acc[v] / (3.0 * (double)o->w * o->h);
    psnr_host[v] = (float)(mse > 0 ? -10.0 * std::log10(mse) : 1e9);
  }
  return NPS_OK;
}

// ---- checkpoint: little-endian header + params, Adam m, v (n x 64 floats
// each) + ADC accumulators (n floats each)
namespace {
struct GsCkptHeader {
  char magic[8];
  uint32_t version, n, sh_deg, step, adc_seed, loss_views;
  float lr[6], bg[3], lambda;
  uint32_t reserved[8];
};
static_assert(sizeof(GsCkptHeader) == 104, "checkpoint header layout");
constexpr char kCkptMagic[8] = {'N', 'P', 'S', 'G', 'S', 'C', 'K', '1'};
}  // namespace

int nps_gs_count(nps_gs* o, uint32_t* count) {
  NPS_TRY(check_gs(o));
  if (!count) return NPS_ERR_INVALID;
  *count = o->n;
  return NPS_OK;
}

int nps_gs_save(nps_gs* o, const char* path) {
  NPS_TRY(check_gs(o));
  if (!path) return NPS_ERR_INVALID;
  cudaStream_t s = o->ctx->stream;
  const size_t n = o->n, pf = (size_t)gsm::kP * n;
  std::vector<float> buf(3 * pf + 2 * n);
  uint32_t st[8] = {0};
  if (n) {
    NPS_CUDA(cudaMemcpyAsync(buf.data(), o->params.p, sizeof(float) * pf, cudaMemcpyDeviceToHost, s));
    NPS_CUDA(cudaMemcpyAsync(buf.data() + pf, o->am.p, sizeof(float) * pf, cudaMemcpyDeviceToHost, s));
    NPS_CUDA(cudaMemcpyAsync(buf.data() + 2 * pf, o->av.p, sizeof(float) * pf, cudaMemcpyDeviceToHost, s));
    NPS_CUDA(cudaMemcpyAsync(buf.data() + 3 * pf, o->adc_grad.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
    NPS_CUDA(cudaMemcpyAsync(buf.data() + 3 * pf + n, o->adc_denom.p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
  }
  NPS_CUDA(cudaMemcpyAsync(st, o->stepst.p, 32, cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  GsCkptHeader h{};
  std::memcpy(h.magic, kCkptMagic, 8);
  h.version = 1;
  h.n = (uint32_t)n;
  h.sh_deg = (uint32_t)o->sh_deg;
  h.step = st[0];
  h.adc_seed = o->adc_seed;
  h.loss_views = o->loss_views;
  for (int k = 0; k < 6; ++k) h.lr[k] = o->lr[k];
  for (int k = 0; k < 3; ++k) h.bg[k] = o->bg[k];
  h.lambda = o->lambda;
  h.reserved[0] = (uint32_t)o->loss_kind;
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error("gs_save: cannot open %s", path);
    return NPS_ERR_INVALID;
  }
  const bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 &&
                  std::fwrite(buf.data(), sizeof(float), buf.size(), f) == buf.size();
  const bool closed = std::fclose(f) == 0;
  if (!ok || !closed) {
    set_error("gs_save: write to %s failed", path);
    return NPS_ERR_INVALID;
  }
  return NPS_OK;
}

int nps_gs_load(nps_gs* o, const char* path) {
  NPS_TRY(check_gs(o));
  if (!path) return NPS_ERR_INVALID;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("gs_load: cannot open %s", path);
    return NPS_ERR_INVALID;
  }
  GsCkptHeader h{};
  if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != 1) {
    std::fclose(f);
    set_error("gs_load: %s is not a Gaussian checkpoint", path);
    return NPS_ERR_INVALID;
  }
  if (h.n > o->cap || h.sh_deg != (uint32_t)o->sh_deg) {
    std::fclose(f);
    set_error("gs_load: checkpoint has %u Gaussians of SH degree %u (trainer: capacity %u, degree %d)", h.n,
              h.sh_deg, o->cap, o->sh_deg);
    return NPS_ERR_INVALID;
  }
  const size_t n = h.n, pf = (size_t)gsm::kP * n;
  std::vector<float> buf(3 * pf + 2 * n);
  const bool ok = std::fread(buf.data(), sizeof(float), buf.size(), f) == buf.size();
  std::fclose(f);
  if (!ok) {
    set_error("gs_load: %s is truncated", path);
    return NPS_ERR_INVALID;
  }
  cudaStream_t s = o->ctx->stream;
  if (n) {
    NPS_CUDA(cudaMemcpyAsync(o->params.p, buf.data(), sizeof(float) * pf, cudaMemcpyHostToDevice, s));
    NPS_CUDA(cudaMemcpyAsync(o->am.p, buf.data() + pf, sizeof(float) * pf, cudaMemcpyHostToDevice, s));
    NPS_CUDA(cudaMemcpyAsync(o->av.p, buf.data() + 2 * pf, sizeof(float) * pf, cudaMemcpyHostToDevice, s));
    NPS_CUDA(cudaMemcpyAsync(o->adc_grad.p, buf.data() + 3 * pf, sizeof(float) * n, cudaMemcpyHostToDevice, s));
    NPS_CUDA(cudaMemcpyAsync(o->adc_denom.p, buf.data() + 3 * pf + n, sizeof(float) * n, cudaMemcpyHostToDevice, s));
  }
  const uint32_t st[8] = {h.step, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
  NPS_CUDA(cudaMemcpyAsync(o->stepst.p, st, 32, cudaMemcpyHostToDevice, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  o->n = h.n;
  o->step = h.step;
  o->adc_seed = h.adc_seed;
  o->loss_views = h.loss_views;
  for (int k = 0; k < 6; ++k) o->lr[k] = h.lr[k];
  for (int k = 0; k < 3; ++k) o->bg[k] = h.bg[k];
  o->lambda = h.lambda;
  o->timeouts_seen = 0;
  o->loss_kind = h.reserved[0] <= (uint32_t)gs::kLossL2 ? (int)h.reserved[0] : gs::kLossL1Dssim;
  o->fwd_valid = o->loss_valid = false;
  o->gkey = 0;
  o->skip_seen = 0;
  if (o->h_status) o->h_status[1] = o->h_status[2] = 0;
  return NPS_OK;
}

int nps_gs_set_raster(nps_gs* o, int fwd_form, int fwd_ppt, int fwd_stage, int bwd_form, int bwd_ppt,
                      int bwd_stage) {
  NPS_TRY(check_gs(o));
  if (fwd_stage == 0) fwd_stage = fwd_form == 1 ? 128 : 256 / (fwd_ppt ? fwd_ppt : 1);
  if (bwd_stage == 0) bwd_stage = bwd_form == 1 ? 128 : 256 / (bwd_ppt ? bwd_ppt : 1);
  if (!valid_variant(o->tile, fwd_form, fwd_ppt, fwd_stage) || !valid_variant(o->tile, bwd_form, bwd_ppt, bwd_stage)) {
    set_error("gs_set_raster: (form, pixels per thread, records per stage) (%d, %d, %d) / (%d, %d, %d) is not a "
              "variant for %u x %u tiles: form 0 (tile 16) (1, 256), (2, 128), (2, 256), (4, 64), (4, 128); form 1 "
              "tile 8 (1 or 2, 64 or 128), tile 16 (1, 128), (2 or 4, 64 or 128), tile 32 (4, 64 or 128)",
              fwd_form, fwd_ppt, fwd_stage, bwd_form, bwd_ppt, bwd_stage, o->tile, o->tile);
    return NPS_ERR_INVALID;
  }
  o->fwd_form = fwd_form;
  o->fwd_ppt = fwd_ppt;
  o->fwd_stage = fwd_stage;
  o->bwd_form = bwd_form;
  o->bwd_ppt = bwd_ppt;
  o->bwd_stage = bwd_stage;
  o->gkey = 0;
  return NPS_OK;
}

int nps_gs_set_variant(nps_gs* o, int fwd_ppt, int fwd_stage, int bwd_ppt, int bwd_stage) {
  return nps_gs_set_raster(o, 0, fwd_ppt, fwd_stage, 0, bwd_ppt, bwd_stage);
}

int nps_gs_set_tile(nps_gs* o, uint32_t tile) {
  NPS_TRY(check_gs(o));
  if (tile != 8 && tile != 16 && tile != 32) {
    set_error("gs_set_tile: tile edge %u (8, 16 or 32)", tile);
    return NPS_ERR_INVALID;
  }
  if (tile != 16 && o->deterministic) {
    set_error("gs_set_tile: the deterministic backward needs 16 x 16 tiles");
    return NPS_ERR_STATE;
  }
  o->tile = tile;
  // keep the raster variants if they serve the new tile, else its default persistent ones
  const RasterVariant def = tile == 8 ? RasterVariant{1, 1, 128} : tile == 32 ? RasterVariant{1, 4, 128}
                                                                              : RasterVariant{1, 2, 128};
  if (!valid_variant(tile, o->fwd_form, o->fwd_ppt, o->fwd_stage))
    o->fwd_form = def.form, o->fwd_ppt = def.ppt, o->fwd_stage = def.stage;
  if (!valid_variant(tile, o->bwd_form, o->bwd_ppt, o->bwd_stage))
    o->bwd_form = def.form, o->bwd_ppt = def.ppt, o->bwd_stage = def.stage;
  o->fwd_valid = o->loss_valid = false;
  o->gkey = 0;
  return NPS_OK;
}

int nps_gs_get_raster(nps_gs* o, int* choice7) {
  NPS_TRY(check_gs(o));
  if (!choice7) return NPS_ERR_INVALID;
  choice7[0] = (int)o->tile;
  choice7[1] = o->fwd_form; choice7[2] = o->fwd_ppt; choice7[3] = o->fwd_stage;
  choice7[4] = o->bwd_form; choice7[5] = o->bwd_ppt; choice7[6] = o->bwd_stage;
  return NPS_OK;
}

// GPU time of the binning stages (projection, depth sort, pair emission, tile
// sort, ranges) of one eager forward at the current tile size, in ms.
static int binning_ms(nps_gs* o, float* ms) {
  const bool timing = o->timing;
  for (auto& u : o->ev_used) {
    o->ev_pool.push_back(u.second.first);
    o->ev_pool.push_back(u.second.second);
  }
  o->ev_used.clear();
  o->timing = true;
  int rc = gs_forward_impl(o, nullptr, false);
  o->timing = timing;
  NPS_TRY(rc);
  NPS_CUDA(cudaStreamSynchronize(o->ctx->stream));
  float tot = 0.0f;
  for (auto& u : o->ev_used) {
    if (u.first == ST_PRE || u.first == ST_DSORT || u.first == ST_EMIT || u.first == ST_TSORT ||
        u.first == ST_RANGES) {
      float t = 0.0f;
      NPS_CUDA(cudaEventElapsedTime(&t, u.second.first, u.second.second));
      tot += t;
    }
    o->ev_pool.push_back(u.second.first);
    o->ev_pool.push_back(u.second.second);
  }
  o->ev_used.clear();
  *ms = tot;
  return NPS_OK;
}

// The autotuner: for each tile edge (8, 16, 32; 16 only in deterministic
// mode) it bins the current views (timing the binning), then times every
// raster variant valid for that tile, forward and backward (three launches
// each after a warm-up launch), and keeps the tile whose binning + fastest
// forward + fastest backward is smallest, with those variants.  The choice
// is cached in a text file (one line per workload: key, tile and the six
// variant numbers) when cache_path is given.
int nps_gs_autotune_raster(nps_gs* o, const char* cache_path, int* choice7, float* times_ms99) {
  NPS_TRY(check_gs(o));
  if (!o->tgt || o->nv == 0) {
    set_error("gs_autotune: set views and targets first");
    return NPS_ERR_STATE;
  }
  cudaDeviceProp prop;
  NPS_CUDA(cudaGetDeviceProperties(&prop, o->ctx->device));
  // workload key: device, image, views, SH degree, Gaussian count (to ~19%), deterministic mode
  char key[256];
  const int nbucket = o->n ? (int)std::lround(4.0 * std::log2((double)o->n)) : 0;
  std::snprintf(key, sizeof(key), "%s|sm%d|%ux%u|v%u|sh%d|n%d|det%d", prop.name, prop.multiProcessorCount, o->w,
                o->h, o->nv, o->sh_deg, nbucket, o->deterministic ? 1 : 0);
  for (char* c = key; *c; ++c)
    if (*c == ' ') *c = '_';
  auto report = [&](bool timed) -> int {
    if (choice7) NPS_TRY(nps_gs_get_raster(o, choice7));
    if (times_ms99 && !timed)
      for (int i = 0; i < kNumTiles * kTuneStride; ++i) times_ms99[i] = -1.0f;  // from the cache: not timed
    return NPS_OK;
  };
  if (cache_path) {
    if (FILE* f = std::fopen(cache_path, "r")) {
      char line[512], k[256];
      int a[7];
      bool found = false;
      while (std::fgets(line, sizeof(line), f))
        if (std::sscanf(line, "%255s %d %d %d %d %d %d %d", k, &a[0], &a[1], &a[2], &a[3], &a[4], &a[5], &a[6]) ==
                8 &&
            std::strcmp(k, key) == 0 && valid_variant((uint32_t)a[0], a[1], a[2], a[3]) &&
            valid_variant((uint32_t)a[0], a[4], a[5], a[6])) {
          found = true;
          o->tile = (uint32_t)a[0];
          o->fwd_form = a[1], o->fwd_ppt = a[2], o->fwd_stage = a[3];
          o->bwd_form = a[4], o->bwd_ppt = a[5], o->bwd_stage = a[6];
        }
      std::fclose(f);
      if (found) {
        o->gkey = 0;
        o->fwd_valid = o->loss_valid = false;
        return report(false);
      }
    }
  }
  if (times_ms99)
    for (int i = 0; i < kNumTiles * kTuneStride; ++i) times_ms99[i] = 0.0f;  // 0: not a variant of that tile
  cudaStream_t s = o->ctx->stream;
  const uint32_t M = o->n * o->nv;
  NPS_TRY(o->g2.ensure(sizeof(float) * gs::kG2 * ((size_t)M + 1)));
  cudaEvent_t e0, e1;
  NPS_CUDA(cudaEventCreate(&e0));
  NPS_CUDA(cudaEventCreate(&e1));
  float best_total = 1e30f;
  uint32_t best_tile = o->tile;
  RasterVariant best_pick[2] = {{o->fwd_form, o->fwd_ppt, o->fwd_stage}, {o->bwd_form, o->bwd_ppt, o->bwd_stage}};
  constexpr int kReps = 3;
  int rc = NPS_OK;
  for (int ti = 0; ti < kNumTiles && rc == NPS_OK; ++ti) {
    const uint32_t tile = kTiles[ti];
    if (o->deterministic && tile != 16) continue;
    o->tile = tile;
    o->fwd_form = 1;  // a variant every tile has, for the binning runs
    o->fwd_ppt = tile == 8 ? 1 : tile == 32 ? 4 : 2;
    o->fwd_stage = 128;
    float bin = 0.0f;
    if ((rc = binning_ms(o, &bin)) != NPS_OK || (rc = binning_ms(o, &bin)) != NPS_OK) break;  // warm-up, timed
    if ((rc = nps_gs_loss(o, nullptr)) != NPS_OK) break;
    float* tt = times_ms99 ? times_ms99 + ti * kTuneStride : nullptr;
    if (tt) tt[0] = bin;
    float best[2] = {1e30f, 1e30f};
    RasterVariant pick[2] = {{1, o->fwd_ppt, 128}, {1, o->fwd_ppt, 128}};
    for (int pass = 0; pass < 2 && rc == NPS_OK; ++pass) {
      for (int vi = 0; vi < kNumVariants && rc == NPS_OK; ++vi) {
        const RasterVariant& va = kVariants[vi];
        if (!valid_variant(tile, va.form, va.ppt, va.stage)) continue;
        float tot = 0.0f;
        for (int r = 0; r <= kReps && rc == NPS_OK; ++r) {  // the first launch warms up
          if (pass == 1) NPS_CUDA(cudaMemsetAsync(o->g2.p, 0, sizeof(float) * gs::kG2 * M, s));
          NPS_CUDA(cudaEventRecord(e0, s));
          rc = pass == 0 ? launch_fwd_raster(o, va.form, va.ppt, va.stage)
                         : launch_bwd_raster(o, va.form, va.ppt, va.stage, o->dimg.as<float4>());
          NPS_CUDA(cudaEventRecord(e1, s));
          NPS_CUDA(cudaEventSynchronize(e1));
          float ms = 0.0f;
          NPS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          if (r > 0) tot += ms;
        }
        const float avg = tot / kReps;
        if (tt) tt[1 + kNumVariants * pass + vi] = avg;
        if (avg < best[pass]) best[pass] = avg, pick[pass] = va;
      }
      // the backward is timed after the chosen forward (the persistent
      // backward's work order comes from the forward's per-tile results)
      if (pass == 0 && rc == NPS_OK) rc = launch_fwd_raster(o, pick[0].form, pick[0].ppt, pick[0].stage);
    }
    const float total = bin + best[0] + best[1];
    if (rc == NPS_OK && total < best_total) {
      best_total = total;
      best_tile = tile;
      best_pick[0] = pick[0];
      best_pick[1] = pick[1];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  o->tile = best_tile;
  o->fwd_form = best_pick[0].form, o->fwd_ppt = best_pick[0].ppt, o->fwd_stage = best_pick[0].stage;
  o->bwd_form = best_pick[1].form, o->bwd_ppt = best_pick[1].ppt, o->bwd_stage = best_pick[1].stage;
  o->fwd_valid = o->loss_valid = false;
  o->gkey = 0;
  NPS_TRY(rc);
  NPS_TRY(report(true));
  if (cache_path) {
    if (FILE* f = std::fopen(cache_path, "a")) {
      std::fprintf(f, "%s %u %d %d %d %d %d %d %.4f\n", key, best_tile, best_pick[0].form, best_pick[0].ppt,
                   best_pick[0].stage, best_pick[1].form, best_pick[1].ppt, best_pick[1].stage, best_total);
      std::fclose(f);
    }
  }
  return NPS_OK;
}

// The earlier interface: the chosen (pixels per thread, records per stage)
// of each pass (choice4) and, per pass, the time of the five 16 x 16
// one-CTA-per-tile variants (times_ms10).
int nps_gs_autotune(nps_gs* o, const char* cache_path, int* choice4, float* times_ms10) {
  int c7[7];
  float t[kNumTiles * kTuneStride];
  NPS_TRY(nps_gs_autotune_raster(o, cache_path, c7, t));
  if (choice4) {
    choice4[0] = c7[2]; choice4[1] = c7[3];
    choice4[2] = c7[5]; choice4[3] = c7[6];
  }
  if (times_ms10)
    for (int pass = 0; pass < 2; ++pass)
      for (int vi = 0; vi < 5; ++vi) times_ms10[5 * pass + vi] = t[1 * kTuneStride + 1 + kNumVariants * pass + vi];
  return NPS_OK;
}

int nps_gs_set_loss(nps_gs* o, int kind, float ssim_weight) {
  NPS_TRY(check_gs(o));
  if (kind < gs::kLossL1Dssim || kind > gs::kLossL2 || !(ssim_weight >= 0.0f && ssim_weight <= 1.0f)) {
    set_error("gs_set_loss: kind %d (0: L1 + D-SSIM, 1: L1, 2: L2), SSIM weight %g (0..1)", kind, ssim_weight);
    return NPS_ERR_INVALID;
  }
  o->loss_kind = kind;
  o->lambda = ssim_weight;
  o->loss_valid = false;
  o->gkey = 0;
  return NPS_OK;
}

int nps_gs_set_sort_guard(nps_gs* o, uint32_t spin_limit, uint32_t stall_tile) {
  NPS_TRY(check_gs(o));
  for (SortWork* w : {&o->sw_depth, &o->sw_tile}) {
    w->spin_limit = spin_limit ? spin_limit : (1u << 20);
    w->stall_tile = stall_tile;
  }
  o->gkey = 0;
  return NPS_OK;
}

int nps_gs_set_deterministic(nps_gs* o, int enable) {
  NPS_TRY(check_gs(o));
  if (enable && o->tile != 16) NPS_TRY(nps_gs_set_tile(o, 16));  // the two-pass backward's tiles
  o->deterministic = enable != 0;
  o->gkey = 0;
  return NPS_OK;
}

int nps_gs_set_accumulate(nps_gs* o, int accumulate, uint32_t loss_views) {
  NPS_TRY(check_gs(o));
  o->accumulate = accumulate != 0;
  o->loss_views = loss_views;
  o->gkey = 0;
  return NPS_OK;
}

int nps_gs_set_timing(nps_gs* o, int enable) {
  NPS_TRY(check_gs(o));
  o->timing = enable != 0;
  return NPS_OK;
}

int nps_gs_stage_times(nps_gs* o, double* ms, uint64_t* calls, uint32_t n, int reset) {
  NPS_TRY(check_gs(o));
  NPS_TRY(collect_graph_timers(o));
  if (!o->ev_used.empty()) NPS_CUDA(cudaStreamSynchronize(o->ctx->stream));
  for (auto& u : o->ev_used) {
    float t = 0.0f;
    NPS_CUDA(cudaEventElapsedTime(&t, u.second.first, u.second.second));
    o->stage_ms[u.first] += t;
    o->stage_calls[u.first] += 1;
    o->ev_pool.push_back(u.second.first);
    o->ev_pool.push_back(u.second.second);
  }
  o->ev_used.clear();
  for (uint32_t k = 0; k < n && k < ST_COUNT; ++k) {
    if (ms) ms[k] = o->stage_ms[k];
    if (calls) calls[k] = o->stage_calls[k];
  }
  if (reset)
    for (int k = 0; k < 16; ++k) { o->stage_ms[k] = 0; o->stage_calls[k] = 0; }
  return NPS_OK;
}

int nps_gs_stats(nps_gs* o, nps_stats* out) {
  NPS_TRY(check_gs(o));
  if (!out) return NPS_ERR_INVALID;
  o->stats.step_count = o->step;
  o->stats.reserved[0] = o->graph_kernels;
  o->stats.reserved[1] = o->skipped;
  {
    // raster staging waits that timed out (a device counter; 0 unless the hardware misbehaved)
    uint32_t st[8];
    NPS_CUDA(cudaMemcpyAsync(st, o->stepst.p, 32, cudaMemcpyDeviceToHost, o->ctx->stream));
    NPS_CUDA(cudaStreamSynchronize(o->ctx->stream));
    o->stats.reserved[2] = st[6];
  }
  if (o->graph_mode && o->gexec && o->h_status) {
    NPS_CUDA(cudaEventSynchronize(o->gdone));
    o->stats.pairs = o->h_status[0];  // pairs of the last replay
    const uint32_t sk = o->h_status[1];
    if (sk != o->skip_seen) {
      o->skipped += sk - o->skip_seen;
      o->skip_seen = sk;
      o->gkey = 0;
    }
    o->stats.reserved[1] = o->skipped;
  }
  *out = o->stats;
  return NPS_OK;
}

}  // extern "C"
