// binning.cu — kernels declared in binning.cuh (compiled with --fmad=false:
// the tile bounds must equal the reference's float values bit for bit).
#include "binning.cuh"

namespace nps {
namespace bin {

__global__ void k_tile_tables(float* tabs, uint32_t tiles_x, uint32_t tiles_y, uint32_t w, uint32_t h) {
  const float aspect = (float)w / (float)h;
  for (uint32_t t = threadIdx.x; t < tiles_x; t += blockDim.x) {
    tabs[t] = pixel_px(t * 16u, w, aspect);
    tabs[tiles_x + t] = pixel_px(min(t * 16u + 16u, w), w, aspect);
  }
  for (uint32_t t = threadIdx.x; t < tiles_y; t += blockDim.x) {
    tabs[2 * tiles_x + t] = pixel_py(min(t * 16u + 16u, h), h);
    tabs[2 * tiles_x + tiles_y + t] = pixel_py(t * 16u, h);
  }
}

__global__ void k_emit(const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                       const uint2* __restrict__ rects, uint32_t n, uint32_t nv, uint32_t tiles_x, uint32_t num_tiles,
                       uint32_t cap, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nv * n) return;
  const uint32_t c = counts[g];
  if (c == 0) return;
  const uint32_t v = g / n, i = g - v * n;
  uint32_t pos = offsets[g];
  const uint2 r = rects[g];
  const uint32_t x0 = r.x & 0xffffu, x1 = r.x >> 16, y0 = r.y & 0xffffu, y1 = r.y >> 16;
  for (uint32_t ty = y0; ty < y1; ++ty)
    for (uint32_t tx = x0; tx < x1; ++tx) {
      if (pos < cap) {
        keys[pos] = v * num_tiles + ty * tiles_x + tx;
        vals[pos] = i;
      }
      ++pos;
    }
}

__global__ void k_ranges(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ total, uint32_t cap,
                         uint32_t* __restrict__ rstart, uint32_t* __restrict__ rend) {
  const uint32_t K = min(*total, cap);
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < K; p += gridDim.x * blockDim.x) {
    const uint32_t k = keys[p];
    if (p == 0 || keys[p - 1] != k) rstart[k] = p;
    if (p == K - 1 || keys[p + 1] != k) rend[k] = p + 1;
  }
}

}  // namespace bin
}  // namespace nps
