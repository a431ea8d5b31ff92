// binning.cuh — tile binning shared by the reference-semantics paths.
//
// The reference tests every primitive against every 16x16 tile
// (splat_backward.wgsl:148-195, bezier_backward.wgsl:119-156) with the
// predicate !(min.x > tile_max.x || max.x < tile_min.x || min.y > tile_max.y
// || max.y < tile_min.y), where the tile bounds are pixel centres
// (pixel_to_p of the tile's first pixel and of min(first + 16, dims)).  The
// bounds increase with the tile index along x and decrease along y, so the
// tiles a primitive overlaps form a rectangle found by four binary searches
// over per-axis tables of the exact same float bounds.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace nps {
namespace bin {

// splat_backward.wgsl:34-40, one axis at a time
__device__ __forceinline__ float pixel_px(uint32_t px, uint32_t w, float aspect) {
  float u = ((float)px + 0.5f) / (float)w;
  return (u * 2.0f - 1.0f) * aspect;
}
__device__ __forceinline__ float pixel_py(uint32_t py, uint32_t h) {
  float u = ((float)py + 0.5f) / (float)h;
  return -(u * 2.0f - 1.0f);
}

// tabs: [tile_min.x (tiles_x) | tile_max.x (tiles_x) | tile_min.y (tiles_y) | tile_max.y (tiles_y)]
__global__ void k_tile_tables(float* tabs, uint32_t tiles_x, uint32_t tiles_y, uint32_t w, uint32_t h);

// Tile rectangle [x0, x1) x [y0, y1) whose tiles pass the reference predicate
// for the screen box [smin, smax]; returns false if empty.
__device__ __forceinline__ bool tile_rect(const float* tabs, uint32_t tiles_x, uint32_t tiles_y, float smin_x,
                                          float smin_y, float smax_x, float smax_y, uint2* rect) {
  const float* tminx = tabs;
  const float* tmaxx = tabs + tiles_x;
  const float* tminy = tabs + 2 * tiles_x;
  const float* tmaxy = tabs + 2 * tiles_x + tiles_y;
  uint32_t lo = 0, hi = tiles_x;
  while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (!(smin_x > tmaxx[m])) hi = m; else lo = m + 1; }
  const uint32_t x0 = lo;
  lo = 0; hi = tiles_x;
  while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (smax_x < tminx[m]) hi = m; else lo = m + 1; }
  const uint32_t x1 = lo;
  lo = 0; hi = tiles_y;
  while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (!(smax_y < tminy[m])) hi = m; else lo = m + 1; }
  const uint32_t y0 = lo;
  lo = 0; hi = tiles_y;
  while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (smin_y > tmaxy[m]) hi = m; else lo = m + 1; }
  const uint32_t y1 = lo;
  if (x1 > x0 && y1 > y0) {
    *rect = make_uint2(x0 | (x1 << 16), y0 | (y1 << 16));
    return true;
  }
  return false;
}

// One (view * tiles + tile, primitive) pair per overlapped tile, written in
// (view, primitive) order starting at offsets[g].
__global__ void k_emit(const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                       const uint2* __restrict__ rects, uint32_t n, uint32_t nv, uint32_t tiles_x, uint32_t num_tiles,
                       uint32_t cap, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals);

// Tile list bounds in the sorted key array.
__global__ void k_ranges(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ total, uint32_t cap,
                         uint32_t* __restrict__ rstart, uint32_t* __restrict__ rend);

}  // namespace bin
}  // namespace nps
