// capi.cpp — context, error and version entry points of libnprush_cuda.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "context.h"

namespace nps {
static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int bind_device(nps_ctx* ctx) {
  if (!ctx) {
    set_error("null context");
    return NPS_ERR_INVALID;
  }
  NPS_CUDA(cudaSetDevice(ctx->device));
  return NPS_OK;
}
}  // namespace nps

extern "C" {

const char* nps_last_error(void) { return nps::g_err; }

const char* nps_version(void) { return "nprush-b200 0.1 (sm_100a)"; }

int nps_create(int device, nps_ctx** out) {
  if (!out) {
    nps::set_error("nps_create: null out");
    return NPS_ERR_INVALID;
  }
  *out = nullptr;
  int n = 0;
  NPS_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) {
    nps::set_error("nps_create: device %d out of range (%d devices)", device, n);
    return NPS_ERR_INVALID;
  }
  NPS_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  NPS_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) {
    nps::set_error("nps_create: device %d is sm_%d%d; this library is built for sm_100a", device, prop.major,
                   prop.minor);
    return NPS_ERR_INVALID;
  }
  nps_ctx* c = new nps_ctx();
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    nps::set_error("cudaStreamCreate: %s", cudaGetErrorString(e));
    return NPS_ERR_CUDA;
  }
  *out = c;
  return NPS_OK;
}

int nps_destroy(nps_ctx* ctx) {
  if (!ctx) return NPS_OK;
  cudaSetDevice(ctx->device);
  if (ctx->own_stream && ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
  return NPS_OK;
}

int nps_sync(nps_ctx* ctx) {
  NPS_TRY(nps::bind_device(ctx));
  NPS_CUDA(cudaStreamSynchronize(ctx->stream));
  return NPS_OK;
}

int nps_set_stream(nps_ctx* ctx, void* cuda_stream) {
  NPS_TRY(nps::bind_device(ctx));
  if (ctx->own_stream && ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  ctx->stream = (cudaStream_t)cuda_stream;
  ctx->own_stream = false;
  return NPS_OK;
}

}  // extern "C"
