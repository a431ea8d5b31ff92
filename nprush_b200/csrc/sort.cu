// sort.cu — device-wide exclusive scan and stable LSD radix sort.
//
// Used for the (view, tile[, depth]) keys of the binning stage.  The sort is a
// fixed-grid reduce-then-scan radix sort: per 8-bit digit, an upsweep kernel
// histograms each block's contiguous key range, a three-kernel scan turns the
// digit-major histogram into offsets, and a downsweep kernel ranks keys stably
// (warp-level ranking in original order from per-bit ballots) and scatters them.
// The grid never depends on the key count (read from device memory), so the
// whole sort can be captured in a CUDA graph, and there is no inter-block
// waiting anywhere (no decoupled look-back spin), so it cannot hang.
#include <cuda_runtime.h>

#include "common.cuh"

namespace nps {
namespace {

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

template <class K>
__global__ void __launch_bounds__(kSortThreads) k_upsweep(const K* __restrict__ keys, const uint32_t* count_dev,
                                                           uint32_t cap, int shift, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[kSortWarps][256];
  const int wid = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&h[0][0])[i] = 0;
  __syncthreads();
  uint32_t n, t0, t1;
  block_range(count_dev, cap, &n, &t0, &t1);
  const uint32_t end = min(t1 * (uint32_t)kTile, n);
  for (uint32_t i = t0 * kTile + threadIdx.x; i < end; i += kSortThreads)
    atomicAdd(&h[wid][(uint32_t)(keys[i] >> shift) & 255u], 1u);
  __syncthreads();
  uint32_t s = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) s += h[w][threadIdx.x];
  hist[threadIdx.x * gridDim.x + blockIdx.x] = s;  // digit-major
}

template <class K>
__global__ void __launch_bounds__(kSortThreads) k_downsweep(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                             K* __restrict__ kout, uint32_t* __restrict__ vout,
                                                             const uint32_t* count_dev, uint32_t cap, int shift,
                                                             const uint32_t* __restrict__ offsets) {
  __shared__ uint32_t run[256];
  __shared__ uint32_t tot[256];
  __shared__ uint32_t toff[256];
  __shared__ uint32_t wh[kSortWarps][256];
  // the tile in local sorted order, so that the global writes come out as
  // contiguous runs per digit
  __shared__ K sk[kTile];
  __shared__ uint32_t sv[kTile];
  __shared__ uint32_t scan_total;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  run[threadIdx.x] = offsets[threadIdx.x * gridDim.x + blockIdx.x];
  uint32_t n, t0, t1;
  block_range(count_dev, cap, &n, &t0, &t1);
  const uint32_t lt = lanemask_lt();
  for (uint32_t tile = t0; tile < t1; ++tile) {
    for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortThreads) (&wh[0][0])[i] = 0;
    const uint32_t base = tile * kTile + wid * (32 * kItems);
    K k[kItems];
    uint32_t v[kItems], dg[kItems], rk[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      uint32_t idx = base + j * 32 + lane;
      bool ok = idx < n;
      k[j] = ok ? kin[idx] : (K)0;
      v[j] = ok ? vin[idx] : 0u;
      dg[j] = ok ? ((uint32_t)(k[j] >> shift) & 255u) : 256u;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const uint32_t d = dg[j];
      // lanes holding the same digit: intersect the ballots of its nine bits
      // (bit 8 marks an invalid item), cheaper than a match-any
      uint32_t peers = 0xffffffffu;
#pragma unroll
      for (int b = 0; b < 9; ++b) {
        const bool bit = (d >> b) & 1u;
        const uint32_t bal = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? bal : ~bal;
      }
      const int leader = __ffs(peers) - 1;
      uint32_t old = 0;
      if (lane == leader && d < 256u) old = wh[wid][d];
      old = __shfl_sync(0xffffffffu, old, leader);
      if (lane == leader && d < 256u) wh[wid][d] = old + __popc(peers);
      rk[j] = old + __popc(peers & lt);
      __syncwarp();
    }
    __syncthreads();
    {
      uint32_t acc = 0;
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w) {
        uint32_t x = wh[w][threadIdx.x];
        wh[w][threadIdx.x] = acc;
        acc += x;
      }
      tot[threadIdx.x] = acc;
      toff[threadIdx.x] = block_exclusive_scan<kSortThreads>(acc, &scan_total);
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      const uint32_t d = dg[j];
      if (d < 256u) {
        const uint32_t lp = toff[d] + wh[wid][d] + rk[j];
        sk[lp] = k[j];
        sv[lp] = v[j];
      }
    }
    __syncthreads();
    const uint32_t cnt = scan_total;  // valid items of this tile
    for (uint32_t i = threadIdx.x; i < cnt; i += kSortThreads) {
      const K kk = sk[i];
      const uint32_t d = (uint32_t)(kk >> shift) & 255u;
      const uint32_t pos = run[d] + (i - toff[d]);
      kout[pos] = kk;
      vout[pos] = sv[i];
    }
    __syncthreads();
    run[threadIdx.x] += tot[threadIdx.x];
    __syncthreads();
  }
}

template <class K>
int radix_sort_impl(K* keys, uint32_t* vals, const uint32_t* count_dev, uint32_t cap, int bits, SortWork& w,
                    cudaStream_t s, K** keys_out, uint32_t** vals_out) {
  NPS_TRY(w.hist.ensure(sizeof(uint32_t) * (256 * kSortGrid + 1)));
  constexpr uint32_t kHist = 256 * kSortGrid;
  NPS_TRY(w.partial.ensure(sizeof(uint32_t) * (div_up(kHist, kScanTile) + 1)));
  NPS_TRY(w.keys_alt.ensure(sizeof(K) * (size_t)cap));
  NPS_TRY(w.vals_alt.ensure(sizeof(uint32_t) * (size_t)cap));
  K* ka = keys;
  uint32_t* va = vals;
  K* kb = w.keys_alt.as<K>();
  uint32_t* vb = w.vals_alt.as<uint32_t>();
  uint32_t* hist = w.hist.as<uint32_t>();
  for (int shift = 0; shift < bits; shift += 8) {
    k_upsweep<K><<<kSortGrid, kSortThreads, 0, s>>>(ka, count_dev, cap, shift, hist);
    // digit-major histogram -> scatter offsets (multi-block scan, in place)
    k_scan_reduce<<<div_up(kHist, kScanTile), kScanThreads, 0, s>>>(hist, kHist, w.partial.as<uint32_t>());
    k_scan_single<<<1, kScanThreads, 0, s>>>(w.partial.as<uint32_t>(), div_up(kHist, kScanTile), hist + kHist);
    k_scan_down<<<div_up(kHist, kScanTile), kScanThreads, 0, s>>>(hist, kHist, w.partial.as<uint32_t>(), hist);
    k_downsweep<K><<<kSortGrid, kSortThreads, 0, s>>>(ka, va, kb, vb, count_dev, cap, shift, hist);
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
