// context.h — the nps_ctx object shared by all entry points.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

struct nps_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  int sm_count = 148;
};

namespace nps {
// Makes ctx's device current on the calling thread.
int bind_device(nps_ctx* ctx);
}  // namespace nps
