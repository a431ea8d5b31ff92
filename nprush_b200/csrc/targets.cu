// targets.cu — target preprocessing passes on device images: the separable
// Gaussian blur (src/lib/gpu/blur.wgsl:23-48, GpuBlurPipelineManager), the
// depth-aware bilateral blur (depth_aware_blur.wgsl:12-53,
// GpuDepthAwareBlurPipelineManager) and the Sobel depth-edge pass
// (splat_edge.wgsl:13-44), which feed the Bezier layers' targets.
//
// Images are H x W float4 RGBA in device memory (a depth image uses .x).  The
// reference stores into rgba8unorm textures; `quantize` applies that
// conversion (clamp to [0, 1], round to the nearest of 256 levels) so the
// outputs equal what the reference's textures hold, and without it the kernels
// return the stored float values.  One thread per output pixel, 16 x 16
// blocks; inputs are read through the read-only cache (every neighbourhood
// overlaps its neighbours').
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"
#include "context.h"

namespace nps {
namespace tgt {

__device__ __forceinline__ float unorm8(float x) { return rintf(fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f) / 255.0f; }

__device__ __forceinline__ float4 finish(float r, float g, float b, int quantize) {
  if (quantize) return make_float4(unorm8(r), unorm8(g), unorm8(b), 1.0f);
  return make_float4(r, g, b, 1.0f);
}

__device__ __forceinline__ float srgb_to_linear(float c) {
  return c > 0.04045f ? powf((c + 0.055f) / 1.055f, 2.4f) : c / 12.92f;
}
__device__ __forceinline__ float linear_to_srgb(float c) {
  const float s = fmaxf(c, 0.0f);
  return s > 0.0031308f ? 1.055f * powf(s, 1.0f / 2.4f) - 0.055f : s * 12.92f;
}

// blur.wgsl:23-48: taps along `dir`, edge-clamped, weights exp(-i^2 / 2 sigma^2)
__global__ void k_blur(const float4* __restrict__ src, float4* __restrict__ dst, int w, int h, int dx, int dy,
                       int radius, uint32_t flags, float sigma, int quantize) {
  const int x = blockIdx.x * 16 + threadIdx.x, y = blockIdx.y * 16 + threadIdx.y;
  if (x >= w || y >= h) return;
  const bool in_srgb = flags & 1u, out_srgb = flags & 2u;
  float sr = 0.0f, sg = 0.0f, sb = 0.0f, ws = 0.0f;
  for (int i = -radius; i <= radius; ++i) {
    const int cx = min(max(x + dx * i, 0), w - 1), cy = min(max(y + dy * i, 0), h - 1);
    const float4 c = __ldg(src + (size_t)cy * w + cx);
    float r = c.x, g = c.y, b = c.z;
    if (in_srgb) r = srgb_to_linear(r), g = srgb_to_linear(g), b = srgb_to_linear(b);
    const float wt = expf(-(float)(i * i) / (2.0f * sigma * sigma));
    sr += r * wt;
    sg += g * wt;
    sb += b * wt;
    ws += wt;
  }
  float r = sr / ws, g = sg / ws, b = sb / ws;
  if (out_srgb) r = linear_to_srgb(r), g = linear_to_srgb(g), b = linear_to_srgb(b);
  dst[(size_t)y * w + x] = finish(r, g, b, quantize);
}

// depth_aware_blur.wgsl:12-53: (2r+1)^2 window, spatial / colour / depth
// Gaussian weights (sigmas 10, 0.5, 0.5), out-of-image neighbours weigh 0
__global__ void k_depth_blur(const float4* __restrict__ color, const float4* __restrict__ depth,
                             float4* __restrict__ dst, int w, int h, int radius, int quantize) {
  const int x = blockIdx.x * 16 + threadIdx.x, y = blockIdx.y * 16 + threadIdx.y;
  if (x >= w || y >= h) return;
  const float4 cc = __ldg(color + (size_t)y * w + x);
  const float cd = __ldg(depth + (size_t)y * w + x).x;
  const float ss = 10.0f, sc = 0.5f, sd = 0.5f;
  float sr = 0.0f, sg = 0.0f, sb = 0.0f, sw = 0.0f;
  for (int dy = -radius; dy <= radius; ++dy)
    for (int dx = -radius; dx <= radius; ++dx) {
      const int nx = x + dx, ny = y + dy;
      const bool in = nx >= 0 && nx < w && ny >= 0 && ny < h;
      const int sx = min(max(nx, 0), w - 1), sy = min(max(ny, 0), h - 1);
      const float4 nc = __ldg(color + (size_t)sy * w + sx);
      const float nd = __ldg(depth + (size_t)sy * w + sx).x;
      const float d2 = (float)(dx * dx + dy * dy);
      const float er = nc.x - cc.x, eg = nc.y - cc.y, eb = nc.z - cc.z;
      const float dc2 = er * er + eg * eg + eb * eb;
      const float dd2 = (nd - cd) * (nd - cd);
      const float wr = expf(-d2 / (2.0f * ss * ss)) * expf(-dc2 / (2.0f * sc * sc)) * expf(-dd2 / (2.0f * sd * sd));
      const float wt = in ? wr : 0.0f;
      sr += nc.x * wt;
      sg += nc.y * wt;
      sb += nc.z * wt;
      sw += wt;
    }
  const float inv = fmaxf(sw, 1e-5f);
  dst[(size_t)y * w + x] = finish(sr / inv, sg / inv, sb / inv, quantize);
}

// splat_edge.wgsl:13-44: Sobel magnitude of the depth, edge-clamped, through
// smoothstep(thr_min, thr_max, .)
__global__ void k_edge(const float4* __restrict__ depth, float4* __restrict__ dst, int w, int h, float tmin,
                       float tmax, int quantize) {
  const int x = blockIdx.x * 16 + threadIdx.x, y = blockIdx.y * 16 + threadIdx.y;
  if (x >= w || y >= h) return;
  auto at = [&](int ox, int oy) {
    const int cx = min(max(x + ox, 0), w - 1), cy = min(max(y + oy, 0), h - 1);
    return __ldg(depth + (size_t)cy * w + cx).x;
  };
  const float tl = at(-1, -1), tc = at(0, -1), tr = at(1, -1), ml = at(-1, 0), mr = at(1, 0);
  const float bl = at(-1, 1), bc = at(0, 1), br = at(1, 1);
  const float gx = -tl - 2.0f * ml - bl + tr + 2.0f * mr + br;
  const float gy = -tl - 2.0f * tc - tr + bl + 2.0f * bc + br;
  const float e = sqrtf(gx * gx + gy * gy);
  const float t = fminf(fmaxf((e - tmin) / (tmax - tmin), 0.0f), 1.0f);
  const float v = t * t * (3.0f - 2.0f * t);
  dst[(size_t)y * w + x] = finish(v, v, v, quantize);
}

}  // namespace tgt
}  // namespace nps

using namespace nps;

namespace {
int check_image(nps_ctx* ctx, const void* a, const void* b, const void* out, uint32_t w, uint32_t h) {
  if (!ctx || !a || !b || !out || w == 0 || h == 0 || w > 65536 || h > 65536) {
    set_error("target pass: bad arguments");
    return NPS_ERR_INVALID;
  }
  if ((((uintptr_t)a | (uintptr_t)b | (uintptr_t)out) & 15) != 0) {
    set_error("target pass: images must be 16-byte aligned float4 arrays");
    return NPS_ERR_INVALID;
  }
  return bind_device(ctx);
}
}  // namespace

extern "C" {

int nps_blur(nps_ctx* ctx, const float* src_rgba, float* dst_rgba, uint32_t w, uint32_t h, int32_t dir_x,
             int32_t dir_y, int32_t radius, uint32_t flags, float sigma, int quantize) {
  NPS_TRY(check_image(ctx, src_rgba, src_rgba, dst_rgba, w, h));
  if (radius < 0 || radius > 1024 || !(sigma > 0.0f) || src_rgba == dst_rgba) {
    set_error("nps_blur: radius in [0, 1024], sigma > 0, distinct source and destination");
    return NPS_ERR_INVALID;
  }
  const dim3 grid(div_up(w, 16), div_up(h, 16));
  tgt::k_blur<<<grid, dim3(16, 16), 0, ctx->stream>>>((const float4*)src_rgba, (float4*)dst_rgba, (int)w, (int)h,
                                                      dir_x, dir_y, radius, flags, sigma, quantize);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int nps_depth_aware_blur(nps_ctx* ctx, const float* color_rgba, const float* depth_rgba, float* dst_rgba, uint32_t w,
                         uint32_t h, int32_t radius, int quantize) {
  NPS_TRY(check_image(ctx, color_rgba, depth_rgba, dst_rgba, w, h));
  if (radius < 0 || radius > 64 || color_rgba == dst_rgba) {
    set_error("nps_depth_aware_blur: radius in [0, 64], distinct source and destination");
    return NPS_ERR_INVALID;
  }
  const dim3 grid(div_up(w, 16), div_up(h, 16));
  tgt::k_depth_blur<<<grid, dim3(16, 16), 0, ctx->stream>>>((const float4*)color_rgba, (const float4*)depth_rgba,
                                                            (float4*)dst_rgba, (int)w, (int)h, radius, quantize);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int nps_splat_edge(nps_ctx* ctx, const float* depth_rgba, float* dst_rgba, uint32_t w, uint32_t h, float thr_min,
                   float thr_max, int quantize) {
  NPS_TRY(check_image(ctx, depth_rgba, depth_rgba, dst_rgba, w, h));
  if (depth_rgba == dst_rgba) {
    set_error("nps_splat_edge: distinct source and destination");
    return NPS_ERR_INVALID;
  }
  const dim3 grid(div_up(w, 16), div_up(h, 16));
  tgt::k_edge<<<grid, dim3(16, 16), 0, ctx->stream>>>((const float4*)depth_rgba, (float4*)dst_rgba, (int)w, (int)h,
                                                      thr_min, thr_max, quantize);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

}  // extern "C"
