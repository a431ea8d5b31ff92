// common.cuh — shared helpers of libnprush_cuda (error model, device buffers).
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstddef>
#include <cstdint>
#include <cstdio>

#include "../../include/nprush.h"

namespace nps {

void set_error(const char* fmt, ...);

#define NPS_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      nps::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));     \
      return e_ == cudaErrorMemoryAllocation ? NPS_ERR_NOMEM : NPS_ERR_CUDA;                 \
    }                                                                                        \
  } while (0)

#define NPS_CHECK_LAUNCH() NPS_CUDA(cudaGetLastError())

#define NPS_TRY(expr)              \
  do {                             \
    int rc_ = (expr);              \
    if (rc_ != NPS_OK) return rc_; \
  } while (0)

// Growable device allocation owned by one object.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int ensure(size_t b) {
    if (b <= bytes) return NPS_OK;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t want = b < 256 ? 256 : b;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
      set_error("cudaMalloc(%zu): %s", want, cudaGetErrorString(e));
      return NPS_ERR_NOMEM;
    }
    bytes = want;
    return NPS_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return (T*)p; }
};

constexpr int kNumSMs = 148;

inline unsigned div_up(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// ------------------------------------------------------------- scan / sort
// Work buffers for the device-wide scan and the radix sort.  Sizes depend only
// on the grid, never on the number of keys, so no host sync is needed.
struct SortWork {
  DevBuf hist;      // per-pass digit histograms, tile counters, own timeout counter
  DevBuf partial;   // scan partial sums
  DevBuf lookback;  // per pass and tile: the published per-digit counts
  DevBuf keys_alt, vals_alt;
  // bounded look-back: polls of an unpublished tile status before giving up
  // (counted in *err, or in the work's own counter when err is null); tests
  // may name one tile whose status is treated as never published
  uint32_t* err = nullptr;
  uint32_t spin_limit = 1u << 20;
  uint32_t stall_tile = 0xffffffffu;
};

// Exclusive scan of n u32 (n read on the host); writes out[0..n) and *total.
int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* total, SortWork& w, cudaStream_t s);

// Stable LSD radix sort (onesweep) of (key, value) pairs by the low `bits`
// key bits (at most 32, at most 2^30 - 1 pairs).
// The number of pairs is read from device memory (*count_dev, clamped to cap).
// keys/vals hold the input; on return *keys_out / *vals_out point at the sorted
// arrays (either the inputs or the work buffers).
int radix_sort_u32(uint32_t* keys, uint32_t* vals, const uint32_t* count_dev, uint32_t cap, int bits, SortWork& w,
                   cudaStream_t s, uint32_t** keys_out, uint32_t** vals_out);


}  // namespace nps
