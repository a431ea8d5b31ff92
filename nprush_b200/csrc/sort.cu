// sort.cu — device-wide exclusive scan and stable LSD radix sort.
//
// Used for the (view, tile[, depth]) keys of the binning stage.  The sort is
// a onesweep radix sort: one histogram kernel for all 8-bit digits, then one
// kernel per digit that ranks each tile of keys stably (warp-level ranking in
// original order from per-bit ballots), finds the tile's global offsets by a
// bounded decoupled look-back over the earlier tiles, and scatters.  The grid
// never depends on the key count (read from device memory), so the whole sort
// can be captured in a CUDA graph.  The exclusive scan is reduce-then-scan.
#include <cuda_runtime.h>

#include "common.cuh"
#include "context.h"

namespace nps {
namespace {

#ifndef NPS_SORT_MATCH
#define NPS_SORT_MATCH 0
#endif
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kItems = 12;
constexpr int kTile = kSortThreads * kItems;  // 3072 keys
constexpr int kSortGrid = 4 * kNumSMs;  // four resident blocks per SM (64 registers)

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Exclusive block scan of one value per thread; returns the prefix, *total set.
template <int THREADS>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t* total) {
  __shared__ uint32_t warp_sums[THREADS / 32];
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
    uint32_t s = lane < THREADS / 32 ? warp_sums[lane] : 0u;
    uint32_t si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += y;
    }
    if (lane < THREADS / 32) warp_sums[lane] = si - s;
    if (lane == THREADS / 32 - 1) *total = si;
  }
  __syncthreads();
  uint32_t r = warp_sums[wid] + inc - x;
  __syncthreads();
  return r;
}

__global__ void k_scan_reduce(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ partial) {
  __shared__ uint32_t tot;
  const uint32_t base = blockIdx.x * kScanTile;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    uint32_t i = base + threadIdx.x * kScanItems + k;
    if (i < n) s += in[i];
  }
  block_exclusive_scan<kScanThreads>(s, &tot);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

// In-place exclusive scan of m values with one block (loops over chunks).
__global__ void k_scan_single(uint32_t* __restrict__ data, uint32_t m, uint32_t* __restrict__ total) {
  __shared__ uint32_t chunk_total;
  uint32_t carry = 0;
  for (uint32_t base = 0; base < m; base += kScanTile) {
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      uint32_t i = base + threadIdx.x * kScanItems + k;
      v[k] = i < m ? data[i] : 0u;
      s += v[k];
    }
    uint32_t pre = block_exclusive_scan<kScanThreads>(s, &chunk_total) + carry;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      uint32_t i = base + threadIdx.x * kScanItems + k;
      if (i < m) data[i] = pre;
      pre += v[k];
    }
    carry += chunk_total;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void k_scan_down(const uint32_t* __restrict__ in, uint32_t n, const uint32_t* __restrict__ partial,
                            uint32_t* __restrict__ out) {
  __shared__ uint32_t tot;
  const uint32_t base = blockIdx.x * kScanTile;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    uint32_t i = base + threadIdx.x * kScanItems + k;
    v[k] = i < n ? in[i] : 0u;
    s += v[k];
  }
  uint32_t pre = block_exclusive_scan<kScanThreads>(s, &tot) + partial[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    uint32_t i = base + threadIdx.x * kScanItems + k;
    if (i < n) out[i] = pre;
    pre += v[k];
  }
}

__device__ __forceinline__ void block_range(const uint32_t* count_dev, uint32_t cap, uint32_t* n, uint32_t* t0,
                                            uint32_t* t1) {
  uint32_t nn = min(*count_dev, cap);
  uint32_t tiles = (nn + kTile - 1) / kTile;
  uint32_t per = (tiles + gridDim.x - 1) / gridDim.x;
  *n = nn;
  *t0 = min(blockIdx.x * per, tiles);
  *t1 = min(*t0 + per, tiles);
}

// ---------------------------------------------------------------- onesweep
// One launch per 8-bit digit (Adinets and Merrill's onesweep): a CTA claims
// the next tile of kTile keys from a counter (tiles are claimed in order, so
// every tile a CTA waits for belongs to a CTA that is already running), ranks
// its keys locally and stably, publishes its per-digit counts, and finds the
// number of keys of each digit in all earlier tiles by looking back through
// their published counts (decoupled look-back: an aggregate adds and the
// search goes on, an inclusive prefix adds and ends it), then publishes its
// own inclusive prefix and scatters.  The digit offsets of a pass come from a
// histogram of every pass taken in one read of the keys beforehand.
//
// Status word per (tile, digit): bits 31..30 flag (0 none yet, 1 aggregate,
// 2 inclusive prefix), bits 29..0 the count.  The look-back is bounded: a
// status that stays unpublished for spin_limit polls makes the CTA count a
// timeout in *err and carry on as if the count were 0; it still publishes
// its own prefix (so no later tile waits on it) and scatters only inside the
// output (positions are clamped to the key count), so the results are wrong
// but the kernel ends and never writes outside its buffers.  For tests,
// stall_tile names one tile whose status is treated as never published.
constexpr uint32_t kFlagAgg = 1u << 30, kFlagInc = 2u << 30, kCountMask = (1u << 30) - 1u;

__device__ __forceinline__ uint32_t ld_status(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_status(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Digit histograms of every pass in one read: ghist[pass * 256 + digit].
template <class K>
__global__ void __launch_bounds__(kSortThreads) k_hist_all(const K* __restrict__ keys, const uint32_t* count_dev,
                                                            uint32_t cap, int passes, uint32_t* __restrict__ ghist) {
  __shared__ uint32_t h[4][256];
  for (int i = threadIdx.x; i < 4 * 256; i += kSortThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  const uint32_t n = min(*count_dev, cap);
  for (uint32_t i = blockIdx.x * kSortThreads + threadIdx.x; i < n; i += gridDim.x * kSortThreads) {
    const K k = keys[i];
    for (int p = 0; p < passes; ++p) atomicAdd(&h[p][(uint32_t)(k >> (8 * p)) & 255u], 1u);
  }
  __syncthreads();
  for (int p = 0; p < passes; ++p) {
    const uint32_t c = h[p][threadIdx.x];
    if (c) atomicAdd(ghist + p * 256 + threadIdx.x, c);
  }
}

template <class K>
__global__ void __launch_bounds__(kSortThreads, 4) k_onesweep(const K* __restrict__ kin,
                                                               const uint32_t* __restrict__ vin, K* __restrict__ kout,
                                                               uint32_t* __restrict__ vout, const uint32_t* count_dev,
                                                               uint32_t cap, int shift,
                                                               const uint32_t* __restrict__ ghist,
                                                               uint32_t* __restrict__ status,
                                                               uint32_t* __restrict__ tile_counter,
                                                               uint32_t* __restrict__ err, uint32_t spin_limit,
                                                               uint32_t stall_tile) {
  __shared__ uint32_t pass_off[256];
  __shared__ uint32_t run[256];
  __shared__ uint32_t toff[256];
  __shared__ uint32_t wh[kSortWarps][256];
  __shared__ K sk[kTile];
  __shared__ uint32_t sv[kTile];
  __shared__ uint32_t scan_total, s_tile;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t d_own = threadIdx.x;  // the digit this thread publishes and looks back for
  const uint32_t n = min(*count_dev, cap);
  const uint32_t tiles = (n + kTile - 1) / kTile;
  // this pass's digit offsets: exclusive scan of its histogram
  pass_off[d_own] = block_exclusive_scan<kSortThreads>(ghist[d_own], &scan_total);
  const uint32_t lt = lanemask_lt();
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&wh[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= tiles) break;
    const uint32_t base = tile * kTile + wid * (32 * kItems);
    K k[kItems];
    uint32_t v[kItems], dg[kItems], rk[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const uint32_t idx = base + j * 32 + lane;
      const bool ok = idx < n;
      k[j] = ok ? kin[idx] : (K)0;
      v[j] = ok ? vin[idx] : 0u;
      dg[j] = ok ? ((uint32_t)(k[j] >> shift) & 255u) : 256u;
    }
    // stable local rank: per warp in (item, lane) order, warps in order
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const uint32_t d = dg[j];
#if NPS_SORT_MATCH
      const uint32_t peers = __match_any_sync(0xffffffffu, d);
#else
      uint32_t peers = 0xffffffffu;
#pragma unroll
      for (int b = 0; b < 9; ++b) {
        const bool bit = (d >> b) & 1u;
        const uint32_t bal = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? bal : ~bal;
      }
#endif
      const int leader = __ffs(peers) - 1;
      uint32_t old = 0;
      if (lane == leader && d < 256u) old = wh[wid][d];
      old = __shfl_sync(0xffffffffu, old, leader);
      if (lane == leader && d < 256u) wh[wid][d] = old + __popc(peers);
      rk[j] = old + __popc(peers & lt);
      __syncwarp();
    }
    __syncthreads();
    uint32_t tot;
    {
      uint32_t acc = 0;
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t x = wh[w][d_own];
        wh[w][d_own] = acc;
        acc += x;
      }
      tot = acc;
      toff[d_own] = block_exclusive_scan<kSortThreads>(acc, &scan_total);
    }
    // publish this tile's count of digit d_own (tile 0: already the prefix)
    uint32_t* st = status + (size_t)tile * 256 + d_own;
    st_status(st, (tile == 0 ? kFlagInc : kFlagAgg) | tot);
    __syncthreads();
    // local sort into shared memory while the look-back runs
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const uint32_t d = dg[j];
      if (d < 256u) {
        const uint32_t lp = toff[d] + wh[wid][d] + rk[j];
        sk[lp] = k[j];
        sv[lp] = v[j];
      }
    }
    // decoupled look-back for digit d_own
    uint32_t excl = 0;
    bool gave_up = false;
    if (tile > 0) {
      uint32_t j = tile - 1, polls = 0;
      for (;;) {
        uint32_t w = ld_status(status + (size_t)j * 256 + d_own);
        if (j == stall_tile) w = 0u;
        if ((w & ~kCountMask) == 0u) {
          if (++polls > spin_limit) {
            gave_up = true;
            break;
          }
          continue;
        }
        excl += w & kCountMask;
        if ((w & ~kCountMask) == kFlagInc || j == 0) break;
        --j;
      }
      st_status(st, kFlagInc | ((excl + tot) & kCountMask));
    }
    run[d_own] = pass_off[d_own] + excl;
    if (__syncthreads_or(gave_up) && threadIdx.x == 0) atomicAdd(err, 1u);
    const uint32_t cnt = scan_total;  // valid items of this tile
    for (uint32_t i = threadIdx.x; i < cnt; i += kSortThreads) {
      const K kk = sk[i];
      const uint32_t d = (uint32_t)(kk >> shift) & 255u;
      const uint32_t pos = run[d] + (i - toff[d]);
      if (pos < n) {
        kout[pos] = kk;
        vout[pos] = sv[i];
      }
    }
    __syncthreads();
  }
}

template <class K>
int radix_sort_impl(K* keys, uint32_t* vals, const uint32_t* count_dev, uint32_t cap, int bits, SortWork& w,
                    cudaStream_t s, K** keys_out, uint32_t** vals_out) {
  if (cap >= (1u << 30)) {
    set_error("radix sort: capacity %u beyond the look-back's 30-bit counts", cap);
    return NPS_ERR_INVALID;
  }
  const int passes = (bits + 7) / 8;
  const uint32_t max_tiles = (cap + kTile - 1) / kTile;
  // hist: the per-pass histograms, the per-pass tile counters and the
  // timeout counter of callers without their own; lookback: per pass and tile
  NPS_TRY(w.hist.ensure(sizeof(uint32_t) * (4 * 256 + 4 + 1)));
  NPS_TRY(w.lookback.ensure(sizeof(uint32_t) * 256 * (size_t)max_tiles * 4 + 256));
  NPS_TRY(w.keys_alt.ensure(sizeof(K) * (size_t)cap));
  NPS_TRY(w.vals_alt.ensure(sizeof(uint32_t) * (size_t)cap));
  uint32_t* ghist = w.hist.as<uint32_t>();
  uint32_t* counters = ghist + 4 * 256;
  uint32_t* err = w.err ? w.err : counters + 4;
  NPS_CUDA(cudaMemsetAsync(ghist, 0, sizeof(uint32_t) * (4 * 256 + 4), s));
  NPS_CUDA(cudaMemsetAsync(w.lookback.p, 0, sizeof(uint32_t) * 256 * (size_t)max_tiles * passes, s));
  k_hist_all<K><<<kSortGrid, kSortThreads, 0, s>>>(keys, count_dev, cap, passes, ghist);
  NPS_CHECK_LAUNCH();
  K* ka = keys;
  uint32_t* va = vals;
  K* kb = w.keys_alt.as<K>();
  uint32_t* vb = w.vals_alt.as<uint32_t>();
  for (int p = 0; p < passes; ++p) {
    k_onesweep<K><<<kSortGrid, kSortThreads, 0, s>>>(ka, va, kb, vb, count_dev, cap, 8 * p, ghist + 256 * p,
                                                     w.lookback.as<uint32_t>() + (size_t)256 * max_tiles * p,
                                                     counters + p, err, w.spin_limit, w.stall_tile);
    NPS_CHECK_LAUNCH();
    K* tk = ka; ka = kb; kb = tk;
    uint32_t* tv = va; va = vb; vb = tv;
  }
  *keys_out = ka;
  *vals_out = va;
  return NPS_OK;
}

}  // namespace

int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* total, SortWork& w, cudaStream_t s) {
  if (n == 0) {
    NPS_CUDA(cudaMemsetAsync(total, 0, sizeof(uint32_t), s));
    return NPS_OK;
  }
  const uint32_t blocks = div_up(n, kScanTile);
  NPS_TRY(w.partial.ensure(sizeof(uint32_t) * (blocks + 1)));
  uint32_t* partial = w.partial.as<uint32_t>();
  k_scan_reduce<<<blocks, kScanThreads, 0, s>>>(in, n, partial);
  k_scan_single<<<1, kScanThreads, 0, s>>>(partial, blocks, total);
  k_scan_down<<<blocks, kScanThreads, 0, s>>>(in, n, partial, out);
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int radix_sort_u32(uint32_t* keys, uint32_t* vals, const uint32_t* count_dev, uint32_t cap, int bits, SortWork& w,
                   cudaStream_t s, uint32_t** keys_out, uint32_t** vals_out) {
  return radix_sort_impl<uint32_t>(keys, vals, count_dev, cap, bits, w, s, keys_out, vals_out);
}


}  // namespace nps

// ------------------------------------------------------------- C ABI
extern "C" int nps_sort_pairs(nps_ctx* ctx, uint32_t* keys, uint32_t* vals, uint32_t n, int bits,
                              uint32_t spin_limit, uint32_t stall_tile) {
  using namespace nps;
  NPS_TRY(bind_device(ctx));
  if (!keys || !vals || bits < 1 || bits > 32 || n >= (1u << 30)) {
    set_error("sort_pairs: null buffer, bits %d outside 1..32 or %u pairs beyond 2^30 - 1", bits, n);
    return NPS_ERR_INVALID;
  }
  if ((((uintptr_t)keys | (uintptr_t)vals) & 3u) != 0) {
    set_error("sort_pairs: keys and values must be 4-byte aligned");
    return NPS_ERR_INVALID;
  }
  if (n == 0) return NPS_OK;
  cudaStream_t s = ctx->stream;
  SortWork w;
  DevBuf count;
  int rc = count.ensure(16);
  uint32_t* ko = nullptr;
  uint32_t* vo = nullptr;
  w.spin_limit = spin_limit ? spin_limit : (1u << 20);
  w.stall_tile = stall_tile;
  if (rc == NPS_OK) {
    const uint32_t cnt[4] = {n, 0u, 0u, 0u};
    rc = cudaMemcpyAsync(count.p, cnt, sizeof(cnt), cudaMemcpyHostToDevice, s) == cudaSuccess ? NPS_OK : NPS_ERR_CUDA;
    w.err = count.as<uint32_t>() + 1;  // zero: the look-back's timeouts
  }
  if (rc == NPS_OK) rc = radix_sort_u32(keys, vals, count.as<uint32_t>(), n, bits, w, s, &ko, &vo);
  if (rc == NPS_OK && ko != keys) {
    if (cudaMemcpyAsync(keys, ko, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(vals, vo, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      rc = NPS_ERR_CUDA;
  }
  uint32_t timeouts = 0;
  if (rc == NPS_OK &&
      (cudaMemcpyAsync(&timeouts, count.as<uint32_t>() + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s) !=
           cudaSuccess ||
       cudaStreamSynchronize(s) != cudaSuccess))
    rc = NPS_ERR_CUDA;
  if (rc == NPS_ERR_CUDA) set_error("sort_pairs: %s", cudaGetErrorString(cudaGetLastError()));
  cudaStreamSynchronize(s);
  for (DevBuf* b : {&w.hist, &w.partial, &w.lookback, &w.keys_alt, &w.vals_alt, &count}) b->release();
  if (rc == NPS_OK && timeouts) {
    set_error("sort_pairs: %u look-back waits gave up (the output is not sorted)", timeouts);
    return NPS_ERR_TIMEOUT;
  }
  return rc;
}

