// gs_raster_ws.cuh — persistent, warp-specialised raster kernels of the
// Gaussian trainer (included by gs.cu inside namespace nps::gs, after the
// record type, the staging helpers and the per-pixel backward state).
//
// One launch covers every (view, tile) work item of a step.  A fixed grid of
// CTAs (as many as fit on the SMs) pulls items from a device queue ordered
// longest first (k_order_items), so long tiles start early and no CTA idles
// behind a short one.  Each CTA has one producer warp and TS * TS / PPT
// consumer threads (PPT vertically adjacent pixels per thread, a TS x TS
// tile, TS = 8, 16 or 32; a warp covers a strip of TS columns by 32 / TS *
// PPT rows):
//
//   producer  takes the next item from the queue, and for each batch of SB
//             records of its tile list waits until a ring slot is free, writes
//             the slot's description (item, offset, count, first / last batch
//             flags), posts the byte count on the slot's "full" mbarrier and
//             issues one cp.async.bulk per record (records are gathered by
//             index, so the bulk form rather than a tensor map);
//   consumers wait on the slot's "full" barrier, composite (forward) or
//             replay and differentiate (backward) their pixels against the
//             staged records, and release the slot.
//
// There is no CTA-wide barrier in the loop: a warp only waits for its own
// data, so warps drift apart by up to the ring's depth instead of meeting at
// every batch.  In the backward the per-record sums of a batch are gathered in
// the slot's shared accumulator; the last warp to finish the batch adds them
// to the (view, Gaussian) records with global atomics and frees the slot.
//
// Every wait is bounded.  A wait that gives up counts in *err (which the host
// reports as NPS_ERR_TIMEOUT and which makes Adam skip the step) and raises
// the CTA's abort flag: the producer stops staging and waits (bounded) for
// the copies it already issued, consumers stop, and the CTA exits without
// writing further results.

constexpr int kWsStages = 3;
constexpr uint32_t kMetaFirst = 1u, kMetaLast = 2u, kMetaEnd = 4u;
constexpr uint32_t kWsWaitLimit = 1u << 22;

struct WsMeta {
  uint32_t item;   // view * num_tiles + tile
  uint32_t off;    // offset of the batch in the tile's list
  uint32_t nb;     // records staged
  uint32_t flags;  // kMetaFirst | kMetaLast | kMetaEnd
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_addr(bar))
               : "memory");
}

// Bounded wait on a phase of an mbarrier that also gives up when the CTA's
// abort flag is raised.  Returns false on a timeout (counted in *err, abort
// raised) or an abort.
__device__ __forceinline__ bool ws_wait(uint64_t* bar, uint32_t parity, volatile uint32_t* abort_flag,
                                        uint32_t* err) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t it = 0; it < kWsWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 63u) == 63u && *abort_flag) return false;
  }
  if (atomicExch(const_cast<uint32_t*>(abort_flag), 1u) == 0u) atomicAdd(err, 1u);
  return false;
}

// Length class of a work item for the queue order: 0 for the longest lists,
// two classes per power of two; items of length 0 get class 63 (forward:
// they still write their background pixels) or are left out (backward).
__device__ __forceinline__ uint32_t ws_length_class(uint32_t len) {
  if (len == 0) return 63u;
  const uint32_t lg = 31u - (uint32_t)__clz(len);
  const uint32_t half = lg > 0 ? (len >> (lg - 1)) & 1u : 0u;
  return 63u - min(63u, 2u * lg + half);
}

// Orders the work items longest first (by length class; within a class in
// no particular order, which does not change any result) into order[] and
// resets the queue: qctl[0] = items queued, qctl[1] = 0 (the head).  One CTA.
// kBwd: the length is the tile's last contributor over its pixels (from the
// forward), and tiles without contributors are left out; otherwise the tile
// list's length.
template <bool kBwd>
__global__ void __launch_bounds__(1024) k_order_items(const uint32_t* __restrict__ rstart,
                                                      const uint32_t* __restrict__ rend,
                                                      const uint32_t* __restrict__ tile_last, uint32_t nitems,
                                                      uint32_t* __restrict__ order, uint32_t* __restrict__ qctl) {
  __shared__ uint32_t hist[64];
  __shared__ uint32_t offs[64];
  const uint32_t tid = threadIdx.x;
  if (tid < 64) hist[tid] = 0;
  __syncthreads();
  for (uint32_t it = tid; it < nitems; it += blockDim.x) {
    const uint32_t len = kBwd ? tile_last[it] : rend[it] - rstart[it];
    if (kBwd && len == 0) continue;
    atomicAdd(&hist[ws_length_class(len)], 1u);
  }
  __syncthreads();
  if (tid < 32) {
    // exclusive scan of 64 counts, two per lane
    const uint32_t a = hist[2 * tid], b = hist[2 * tid + 1];
    uint32_t inc = a + b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if ((int)tid >= o) inc += y;
    }
    const uint32_t ex = inc - a - b;
    offs[2 * tid] = ex;
    offs[2 * tid + 1] = ex + a;
    if (tid == 31) {
      qctl[0] = inc;
      qctl[1] = 0u;
    }
  }
  __syncthreads();
  for (uint32_t it = tid; it < nitems; it += blockDim.x) {
    const uint32_t len = kBwd ? tile_last[it] : rend[it] - rstart[it];
    if (kBwd && len == 0) continue;
    order[atomicAdd(&offs[ws_length_class(len)], 1u)] = it;
  }
}

// Producer side shared by both kernels: claims the next item (lane 0) and
// broadcasts it.  Returns false when the queue is exhausted.
__device__ __forceinline__ bool ws_next_item(uint32_t* qctl, const uint32_t* __restrict__ order, uint32_t nq,
                                             uint32_t lane, uint32_t* item) {
  uint32_t q = 0;
  if (lane == 0) q = atomicAdd(&qctl[1], 1u);
  q = __shfl_sync(0xffffffffu, q, 0);
  if (q >= nq) return false;
  *item = __ldg(order + q);
  return true;
}

// After an abort: wait (bounded) for the bulk copies of the last min(issued,
// S) batches, so that none lands in shared memory after the CTA has exited.
template <int S>
__device__ __forceinline__ void ws_drain(uint64_t* full, uint32_t issued) {
  const uint32_t first = issued > (uint32_t)S ? issued - S : 0u;
  for (uint32_t j = first; j < issued; ++j) (void)mbar_wait(&full[j % S], (j / S) & 1u);
}

// Pixel mapping of a consumer thread in a TS x TS tile: column tid % TS,
// rows PPT (tid / TS) .. + PPT - 1; warp w's strip starts at row PPT RW w.
template <int TS, int PPT>
struct WsTile {
  static constexpr int NC = TS * TS / PPT;           // consumer threads
  static constexpr int NW = NC / 32;                 // consumer warps
  static constexpr int RW = 32 / TS;                 // row groups per warp
  static constexpr float kStripW = (float)(TS - 1);  // strip extent - 1 (pixel centres)
  static constexpr float kStripH = (float)(RW * PPT - 1);
  static_assert(TS == 8 || TS == 16 || TS == 32, "tile size");
  static_assert(NC % 32 == 0 && NC >= 32, "whole warps");
};

// ------------------------------------------------------------ forward
template <int TS, int PPT, int SB>
__global__ void __launch_bounds__(TS * TS / PPT + 32) k_fwd_ws(
    const Rec* __restrict__ recs, const uint32_t* __restrict__ vals, const uint32_t* __restrict__ rstart,
    const uint32_t* __restrict__ rend, const uint32_t* __restrict__ order, uint32_t* __restrict__ qctl, uint32_t W,
    uint32_t H, uint32_t tiles_x, uint32_t num_tiles, float3 bg, float4* __restrict__ img,
    uint32_t* __restrict__ ncontrib, uint32_t* __restrict__ tile_last, uint32_t* __restrict__ err) {
  using TL = WsTile<TS, PPT>;
  constexpr int NW = TL::NW, S = kWsStages;
  static_assert(SB % 32 == 0 && SB <= 256, "batch size");
  __shared__ __align__(16) Rec s_rec[S][SB];
  __shared__ __align__(8) uint64_t s_full[S];
  __shared__ __align__(8) uint64_t s_empty[S];
  __shared__ WsMeta s_meta[S];
  __shared__ volatile uint32_t s_wdone[NW];  // per consumer warp: the CTA-local number of its last finished tile
  __shared__ volatile uint32_t s_abort;
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int k = 0; k < S; ++k) {
      mbar_init(&s_full[k], 1);
      mbar_init(&s_empty[k], NW);
    }
    s_abort = 0u;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < (uint32_t)NW) s_wdone[tid] = 0u;
  __syncthreads();

  if (warp == (uint32_t)NW) {
    // ---------------- producer
    const uint32_t nq = qctl[0];
    uint32_t i = 0, tseq = 0, item = 0;
    bool stop = false;
    while (!stop) {
      const bool fin = !ws_next_item(qctl, order, nq, lane, &item);
      uint32_t start = 0, len = 0;
      if (!fin) {
        start = __ldg(rstart + item);
        len = __ldg(rend + item) - start;
      }
      const uint32_t nbatch = fin ? 1u : max(1u, (len + SB - 1) / SB);
      for (uint32_t b = 0; b < nbatch; ++b) {
        const uint32_t slot = i % S;
        if (i >= (uint32_t)S && !ws_wait(&s_empty[slot], ((i / S) - 1u) & 1u, &s_abort, err)) {
          ws_drain<S>(s_full, i);
          return;
        }
        uint32_t nb = fin ? 0u : min((uint32_t)SB, len - b * SB);
        uint32_t flags = fin ? kMetaEnd : ((b == 0 ? kMetaFirst : 0u) | (b + 1 == nbatch ? kMetaLast : 0u));
        if (!fin && b > 0) {
          // every consumer warp has finished this tile (all its pixels
          // reached T < 1e-4): end the tile with an empty batch
          bool all = true;
#pragma unroll
          for (int w2 = 0; w2 < NW; ++w2) all = all && s_wdone[w2] >= tseq + 1;
          if (all) {
            nb = 0;
            flags |= kMetaLast;
          }
        }
        uint32_t g[SB / 32];
#pragma unroll
        for (int k = 0; k < SB / 32; ++k) {
          const uint32_t r = lane + 32u * k;
          g[k] = r < nb ? __ldg(vals + start + b * SB + r) : 0u;
        }
        if (lane == 0) {
          s_meta[slot] = WsMeta{item, b * SB, nb, flags};
          mbar_expect_tx(&s_full[slot], nb * (uint32_t)sizeof(Rec));
        }
        __syncwarp();
        if (nb > 0) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#pragma unroll
          for (int k = 0; k < SB / 32; ++k) {
            const uint32_t r = lane + 32u * k;
            if (r < nb) bulk_g2s(&s_rec[slot][r], recs + g[k], (uint32_t)sizeof(Rec), &s_full[slot]);
          }
        }
        ++i;
        if (flags & (kMetaLast | kMetaEnd)) break;
      }
      stop = fin;
      ++tseq;
    }
    return;
  }

  // ---------------- consumers
  float T[PPT], C0[PPT], C1[PPT], C2[PPT];
  uint32_t last[PPT];
  bool dn[PPT];
  uint32_t px = 0, py = 0, v = 0;
  float wx0 = 0.0f, wy0 = 0.0f;
  uint32_t tseq = 0;
  bool reported = false;
  for (uint32_t i = 0;; ++i) {
    const uint32_t slot = i % S;
    if (!ws_wait(&s_full[slot], (i / S) & 1u, &s_abort, err)) return;
    const WsMeta m = s_meta[slot];
    if (m.flags & kMetaEnd) return;
    if (m.flags & kMetaFirst) {
      v = m.item / num_tiles;
      const uint32_t tile = m.item - v * num_tiles, ty = tile / tiles_x, tx = tile - ty * tiles_x;
      px = tx * TS + (tid % TS);
      py = ty * TS + PPT * (tid / TS);
      wx0 = (float)(tx * TS);
      wy0 = (float)(ty * TS + PPT * TL::RW * warp);
#pragma unroll
      for (int k = 0; k < PPT; ++k) {
        T[k] = 1.0f; C0[k] = C1[k] = C2[k] = 0.0f; last[k] = 0;
        dn[k] = !(px < W && py + k < H);
      }
      ++tseq;
      reported = false;
    }
    bool mine = true;
#pragma unroll
    for (int k = 0; k < PPT; ++k) mine = mine && dn[k];
    const bool wdone = __all_sync(0xffffffffu, mine);
    if (m.nb > 0 && !wdone) {
      const Rec* sr = s_rec[slot];
      const float fx = (float)px;
      uint32_t hit[SB / 32];
#pragma unroll
      for (int qq = 0; qq < SB / 32; ++qq) {
        const uint32_t jj = qq * 32 + lane;
        bool h = false;
        if (jj < m.nb) h = !rec_misses_box(sr[jj].a, sr[jj].b.x, sr[jj].c, wx0, wy0, TL::kStripW, TL::kStripH);
        hit[qq] = __ballot_sync(0xffffffffu, h);
      }
      bool done = mine;
#pragma unroll
      for (int qq = 0; qq < SB / 32; ++qq)
        for (uint32_t mk = hit[qq]; mk != 0u && !done;) {
          const int bit = __ffs(mk) - 1;
          mk &= mk - 1u;
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
            if (power > 0.0f || power < pmin) continue;  // alpha < 1/255 below pmin
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
            last[k] = m.off + j + 1;
          }
          done = true;
#pragma unroll
          for (int k = 0; k < PPT; ++k) done = done && dn[k];
        }
    }
    if (!reported) {
      bool all = true;
#pragma unroll
      for (int k = 0; k < PPT; ++k) all = all && dn[k];
      if (__all_sync(0xffffffffu, all)) {
        if (lane == 0) s_wdone[warp] = tseq;
        reported = true;
      }
    }
    if (m.flags & kMetaLast) {
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
      wmax = __reduce_max_sync(0xffffffffu, wmax);
      if (lane == 0 && wmax > 0) atomicMax(tile_last + m.item, wmax);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&s_empty[slot]);
  }
}

// ------------------------------------------------------------ backward
template <int TS, int PPT, int SB>
__global__ void __launch_bounds__(TS * TS / PPT + 32) k_bwd_ws(
    const Rec* __restrict__ recs, const uint32_t* __restrict__ vals, const uint32_t* __restrict__ rstart,
    const uint32_t* __restrict__ tile_last, const uint32_t* __restrict__ order, uint32_t* __restrict__ qctl,
    uint32_t W, uint32_t H, uint32_t tiles_x, uint32_t num_tiles, float3 bg, const float4* __restrict__ img,
    const uint32_t* __restrict__ ncontrib, const float4* __restrict__ dimg, float* __restrict__ g2,
    uint32_t* __restrict__ err) {
  using TL = WsTile<TS, PPT>;
  constexpr int NW = TL::NW, S = kWsStages;
  static_assert(SB % 32 == 0 && SB <= 256, "batch size");
  __shared__ __align__(16) Rec s_rec[S][SB];
  __shared__ uint32_t s_g[S][SB];
  __shared__ float s_acc[S][SB][9];
  __shared__ __align__(8) uint64_t s_full[S];
  __shared__ __align__(8) uint64_t s_empty[S];
  __shared__ WsMeta s_meta[S];
  __shared__ uint32_t s_cnt[S];
  __shared__ volatile uint32_t s_abort;
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int k = 0; k < S; ++k) {
      mbar_init(&s_full[k], 1);
      mbar_init(&s_empty[k], 1);
      s_cnt[k] = 0u;
    }
    s_abort = 0u;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (uint32_t r = tid; r < (uint32_t)(S * SB * 9); r += blockDim.x) (&s_acc[0][0][0])[r] = 0.0f;
  __syncthreads();

  if (warp == (uint32_t)NW) {
    // ---------------- producer: each tile's contributors [0, last) in
    // batches from the back
    const uint32_t nq = qctl[0];
    uint32_t i = 0, item = 0;
    for (;;) {
      const bool fin = !ws_next_item(qctl, order, nq, lane, &item);
      uint32_t start = 0, top = 0;
      if (!fin) {
        start = __ldg(rstart + item);
        top = __ldg(tile_last + item);
      }
      const uint32_t nbatch = fin ? 1u : (top + SB - 1) / SB;
      for (uint32_t b = 0; b < nbatch; ++b) {
        const uint32_t slot = i % S;
        if (i >= (uint32_t)S && !ws_wait(&s_empty[slot], ((i / S) - 1u) & 1u, &s_abort, err)) {
          ws_drain<S>(s_full, i);
          return;
        }
        const uint32_t hi = top - b * SB, lo = hi > (uint32_t)SB ? hi - SB : 0u;
        const uint32_t nb = fin ? 0u : hi - lo;
        const uint32_t flags =
            fin ? kMetaEnd : ((b == 0 ? kMetaFirst : 0u) | (b + 1 == nbatch ? kMetaLast : 0u));
        uint32_t g[SB / 32];
#pragma unroll
        for (int k = 0; k < SB / 32; ++k) {
          const uint32_t r = lane + 32u * k;
          g[k] = r < nb ? __ldg(vals + start + lo + r) : 0u;
          if (r < nb) s_g[slot][r] = g[k];
        }
        __syncwarp();
        if (lane == 0) {
          s_meta[slot] = WsMeta{item, lo, nb, flags};
          mbar_expect_tx(&s_full[slot], nb * (uint32_t)sizeof(Rec));
        }
        __syncwarp();
        if (nb > 0) {
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#pragma unroll
          for (int k = 0; k < SB / 32; ++k) {
            const uint32_t r = lane + 32u * k;
            if (r < nb) bulk_g2s(&s_rec[slot][r], recs + g[k], (uint32_t)sizeof(Rec), &s_full[slot]);
          }
        }
        ++i;
      }
      if (fin) return;
    }
  }

  // ---------------- consumers
  PixBwd p[PPT];
  uint32_t wlast = 0;
  float wx0 = 0.0f, wy0 = 0.0f;
  for (uint32_t i = 0;; ++i) {
    const uint32_t slot = i % S;
    if (!ws_wait(&s_full[slot], (i / S) & 1u, &s_abort, err)) return;
    const WsMeta m = s_meta[slot];
    if (m.flags & kMetaEnd) return;
    if (m.flags & kMetaFirst) {
      const uint32_t v = m.item / num_tiles;
      const uint32_t tile = m.item - v * num_tiles, ty = tile / tiles_x, tx = tile - ty * tiles_x;
      const uint32_t px = tx * TS + (tid % TS), py = ty * TS + PPT * (tid / TS);
      wx0 = (float)(tx * TS);
      wy0 = (float)(ty * TS + PPT * TL::RW * warp);
      uint32_t mylast = 0;
#pragma unroll
      for (int k = 0; k < PPT; ++k) {
        pix_bwd_init(p[k], px, py + k, v, W, H, bg, img, ncontrib, dimg);
        mylast = max(mylast, p[k].last);
      }
      wlast = __reduce_max_sync(0xffffffffu, mylast);
    }
    const Rec* sr = s_rec[slot];
    float(*acc)[9] = s_acc[slot];
    if (m.nb > 0 && m.off < wlast) {
      uint32_t hit[SB / 32];
#pragma unroll
      for (int qq = 0; qq < SB / 32; ++qq) {
        const uint32_t jj = qq * 32 + lane;
        bool h = false;
        if (jj < m.nb && m.off + jj < wlast)
          h = !rec_misses_box(sr[jj].a, sr[jj].b.x, sr[jj].c, wx0, wy0, TL::kStripW, TL::kStripH);
        hit[qq] = __ballot_sync(0xffffffffu, h);
      }
#pragma unroll
      for (int qq = SB / 32 - 1; qq >= 0; --qq)
        for (uint32_t mk = hit[qq]; mk != 0u;) {
          const int bit = 31 - __clz(mk);
          mk &= ~(1u << bit);
          const int j = qq * 32 + bit;  // descending within the batch
          const float4 a = sr[j].a;
          const float4 c4 = sr[j].c;
          const float4 b = sr[j].b;
          const uint32_t cur = m.off + (uint32_t)j;
          float gv[9];
#pragma unroll
for (int k = 0; k < 9; ++k) gv[k] = 0.0f;
          bool any = false;
#pragma unroll
          for (int k = 0; k < PPT; ++k) any |= pix_bwd_pair(p[k], a, b, c4, cur, gv);
          if (__any_sync(0xffffffffu, any)) {
            const float tot = warp_sum9(gv, lane);
            const uint32_t k = warp_sum9_index(lane);
            if ((lane & 1) == 0 && k < 9) atomicAdd(&acc[j][k], tot * bwd_term_scale(k));
          }
        }
    }
    // the last warp to finish the batch adds its sums to the records and frees the slot
    __syncwarp();
    __threadfence_block();
    uint32_t c = 0;
    if (lane == 0) {
      c = atomicAdd(&s_cnt[slot], 1u);
      __threadfence_block();
    }
    c = __shfl_sync(0xffffffffu, c, 0);
    __syncwarp();
    if (c == (uint32_t)NW - 1) {
      __threadfence_block();
      for (uint32_t e = lane; e < m.nb * 9u; e += 32) {
        const uint32_t j = e / 9u, k = e - 9u * j;
        const float x = acc[j][k];
        if (x != 0.0f) {
          atomicAdd(g2 + (size_t)s_g[slot][j] * kG2 + k, x);
          acc[j][k] = 0.0f;
        }
      }
      if (lane == 0) s_cnt[slot] = 0u;
      __syncwarp();
      __threadfence_block();
      if (lane == 0) mbar_arrive(&s_empty[slot]);
    }
  }
}
