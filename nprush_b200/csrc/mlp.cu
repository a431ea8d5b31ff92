// mlp.cu — the learned ADC policy network on the 5th-generation tensor cores.
//
// A 16 -> 64 -> 64 -> 3 MLP (ReLU) whose three logits, with a fixed 0 logit
// for "keep", give a softmax over {keep, clone, split, prune}.  Weights are
// kept in fp32 (Adam state too) and rounded to bf16 for the products; every
// product is a tcgen05.mma (kind::f16, bf16 x bf16, fp32 accumulate in TMEM):
//
//   forward   Z1 = X W1^T,  Z2 = H1 W2^T,  Z3 = H2 W3^T          (M = 128 rows)
//   backward  dH2 = dZ3 W3,  dH1 = dZ2 W2                         (M = 128 rows)
//   weights   dW2 = dZ2^T H1, dW1 = dZ1^T X, dW3^T = H2^T dZ3     (K = 128 rows)
//
// The weight-gradient products reduce over the 128 rows of a tile, so the
// rows are the K dimension: the transposed activations are written straight
// into K-major operand tiles, and [dZ2^T ; dZ1^T] and [H2^T ; H1^T] are stacked
// into 128-row A operands so that each product is one M = 128 MMA of which the
// wanted 64-row half is read back.  Those accumulators stay in TMEM across
// all tiles a CTA processes and are added to global memory once per CTA.
//
// Operand tiles use the canonical K-major layout without swizzle: 8-row x
// 16-byte core matrices, consecutive along K (LBO = 128 B), 8-row groups
// SBO = K * 2 * 8 B apart.  One CTA of 128 threads per SM: thread t owns row t
// of the tile and TMEM lane t.  Every wait on the MMA completion barrier is
// bounded; on a timeout the kernel flags an error, stops, and frees its TMEM.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "common.cuh"
#include "context.h"

namespace nps {
namespace mlp {

constexpr int kIn = 16, kH = 64, kOut = 3, kOutPad = 16, kRows = 128, kThreads = 128;
// parameter vector: W1 [64x16], b1 [64], W2 [64x64], b2 [64], W3 [3x64], b3 [3]
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kOut * kH, kNumParams = oB3 + kOut;

// TMEM columns (fp32, 128 lanes)
constexpr uint32_t kTmemCols = 256;
constexpr uint32_t cD1 = 0, cD2 = 64, cD3 = 128, cDA = 144, cDB = 208, cDC = 224;

// shared memory (bytes)
constexpr uint32_t sX = 0;                        // A  [128 x 16]   X
constexpr uint32_t sXT = sX + 128 * 16 * 2;       // B  [16 x 128]   X^T
constexpr uint32_t sH1 = sXT + 16 * 128 * 2;      // A  [128 x 64]   H1
constexpr uint32_t sH2 = sH1 + 128 * 64 * 2;      // A  [128 x 64]   H2
constexpr uint32_t sAh = sH2 + 128 * 64 * 2;      // A  [128 x 128]  [H2^T ; H1^T]
constexpr uint32_t sdZ3 = sAh + 128 * 128 * 2;    // A  [128 x 16]   dZ3 (3 used)
constexpr uint32_t sdZ3T = sdZ3 + 128 * 16 * 2;   // B  [16 x 128]   dZ3^T
constexpr uint32_t sdZ2 = sdZ3T + 16 * 128 * 2;   // A  [128 x 64]   dZ2
constexpr uint32_t sAdz = sdZ2 + 128 * 64 * 2;    // A  [128 x 128]  [dZ2^T ; dZ1^T]
constexpr uint32_t sW1 = sAdz + 128 * 128 * 2;    // B  [64 x 16]    W1
constexpr uint32_t sW2 = sW1 + 64 * 16 * 2;       // B  [64 x 64]    W2
constexpr uint32_t sW3 = sW2 + 64 * 64 * 2;       // B  [16 x 64]    W3 (3 rows used)
constexpr uint32_t sW2T = sW3 + 16 * 64 * 2;      // B  [64 x 64]    W2^T
constexpr uint32_t sW3T = sW2T + 64 * 64 * 2;     // B  [64 x 16]    W3^T (3 columns used)
constexpr uint32_t sBias = sW3T + 64 * 16 * 2;    // fp32 b1[64], b2[64], b3[4]
// per warp: fp32 bias-gradient sums db1[64], db2[64], db3[4], then the loss and the correct count
constexpr uint32_t kRedSlot = 136;
constexpr uint32_t sRed = sBias + 132 * 4;
constexpr uint32_t sBar = (sRed + (kThreads / 32) * kRedSlot * 4 + 15) / 16 * 16;  // mbarrier (8 B) + TMEM address
constexpr uint32_t kSmemBytes = sBar + 16;
static_assert(kSmemBytes <= 227 * 1024, "shared memory budget");

// byte offset of element (r, k) of a K-major operand tile with K columns
__device__ __forceinline__ uint32_t kmaj(uint32_t r, uint32_t k, uint32_t K) {
  return (r >> 3) * (K * 16u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// shared-memory matrix descriptor: canonical K-major, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t K) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)((K * 16u) >> 4) << 32) |
         (1ull << 46);
}

// instruction descriptor, kind::f16: bf16 A and B (K-major), fp32 D
__host__ __device__ constexpr uint32_t idesc(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc));
}

// D[128 x N] (+)= A[128 x K] B[N x K]^T as K/16 MMAs; a, b: tile base addresses
__device__ __forceinline__ void gemm(uint32_t d, uint32_t a, uint32_t b, uint32_t K, uint32_t N, bool acc) {
  for (uint32_t j = 0; j < K / 16; ++j)
    mma(d, sdesc(a + j * 256u, K), sdesc(b + j * 256u, K), idesc(128, N), (acc || j > 0) ? 1u : 0u);
}

__device__ __forceinline__ void commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t phase) {
  for (uint32_t it = 0; it < (1u << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

// 8 consecutive K values of row r as one 16-byte store
__device__ __forceinline__ void st_row8(uint8_t* base, uint32_t r, uint32_t k0, uint32_t K, const float* v) {
  uint4 w;
  w.x = (uint32_t)bf16_bits(v[0]) | ((uint32_t)bf16_bits(v[1]) << 16);
  w.y = (uint32_t)bf16_bits(v[2]) | ((uint32_t)bf16_bits(v[3]) << 16);
  w.z = (uint32_t)bf16_bits(v[4]) | ((uint32_t)bf16_bits(v[5]) << 16);
  w.w = (uint32_t)bf16_bits(v[6]) | ((uint32_t)bf16_bits(v[7]) << 16);
  *reinterpret_cast<uint4*>(base + kmaj(r, k0, K)) = w;
}
__device__ __forceinline__ void st_one(uint8_t* base, uint32_t r, uint32_t k, uint32_t K, float v) {
  *reinterpret_cast<uint16_t*>(base + kmaj(r, k, K)) = bf16_bits(v);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Each block writes its sums to its own row of `partial` (kPartial floats:
// the kNumParams gradient sums, the loss, the correct count); k_mlp_reduce
// then adds the rows in block order, so a batch's gradient is the same bits
// on every run.
constexpr uint32_t kPartial = kNumParams + 2;
struct TrainOut {
  float* partial;    // gridDim.x x kPartial
};

// kTrain: forward + softmax cross-entropy + backward, gradients accumulated;
// otherwise forward only, writing 3 logits per row.
template <bool kTrain>
__global__ void __launch_bounds__(kThreads, 1)
    k_mlp(const float* __restrict__ params, const float* __restrict__ X, const uint32_t* __restrict__ rows,
          const uint8_t* __restrict__ labels, uint32_t n, float4 class_w, float inv_batch, TrainOut out,
          float* __restrict__ logits, uint32_t* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
  const uint32_t bar = sbase + sBar;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + sBar + 8);
  float* bias = reinterpret_cast<float*>(smem + sBias);
  float* red = reinterpret_cast<float*>(smem + sRed);
  float* redw = red + warp * kRedSlot;  // this warp's sums (only its lane 0 writes them)

  // weights to bf16 operand tiles, biases to fp32
  for (uint32_t i = tid; i < kH * kIn; i += kThreads) {
    const uint32_t o = i / kIn, k = i % kIn;
    st_one(smem + sW1, o, k, kIn, params[oW1 + i]);
  }
  for (uint32_t i = tid; i < kH * kH; i += kThreads) {
    const uint32_t o = i / kH, k = i % kH;
    const float w = params[oW2 + i];
    st_one(smem + sW2, o, k, kH, w);
    st_one(smem + sW2T, k, o, kH, w);
  }
  for (uint32_t i = tid; i < kOutPad * kH; i += kThreads) {
    const uint32_t o = i / kH, k = i % kH;
    const float w = o < (uint32_t)kOut ? params[oW3 + o * kH + k] : 0.0f;
    st_one(smem + sW3, o, k, kH, w);
    st_one(smem + sW3T, k, o, kOutPad, w);
  }
  for (uint32_t i = tid; i < 132; i += kThreads)
    bias[i] = i < 64 ? params[oB1 + i] : i < 128 ? params[oB2 + i - 64] : (i - 128 < 3 ? params[oB3 + i - 128] : 0.f);
  for (uint32_t i = tid; i < (kThreads / 32) * kRedSlot; i += kThreads) red[i] = 0.0f;
  // rows 3..15 of dZ3^T stay zero
  for (uint32_t i = tid; i < 16 * 128; i += kThreads) {
    const uint32_t c = i / 128, r = i % 128;
    if (c >= 3) st_one(smem + sdZ3T, c, r, kRows, 0.0f);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(tslot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t tl = tmem + ((warp * 32u) << 16);  // this warp's lanes
  uint32_t phase = 0;
  bool ok = true;
  float loss_acc = 0.0f, correct_acc = 0.0f;
  const uint32_t ntiles = (n + kRows - 1) / kRows;
  bool first = true;

  // one MMA batch: issue (thread 0), commit, everyone waits
  auto sync_mma = [&](auto issue) {
    fence_async_smem();
    fence_before();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      issue();
      commit(bar);
    }
    const bool w = bar_wait(bar, phase);
    phase ^= 1u;
    ok = __syncthreads_and(w ? 1 : 0) != 0;
    fence_after();
  };

  for (uint32_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const uint32_t row = tile * kRows + tid;
    const bool valid = row < n;
    const uint32_t src = valid ? (rows ? rows[row] : row) : 0u;
    float x[kIn];
#pragma unroll
    for (int k = 0; k < kIn; k += 4) {
      const float4 v = valid ? *reinterpret_cast<const float4*>(X + (size_t)src * kIn + k) : make_float4(0, 0, 0, 0);
      x[k] = v.x; x[k + 1] = v.y; x[k + 2] = v.z; x[k + 3] = v.w;
    }
    st_row8(smem + sX, tid, 0, kIn, x);
    st_row8(smem + sX, tid, 8, kIn, x + 8);
    if (kTrain)
#pragma unroll
      for (int k = 0; k < kIn; ++k) st_one(smem + sXT, k, tid, kRows, x[k]);

    // ---- layer 1
    sync_mma([&] { gemm(tmem + cD1, sbase + sX, sbase + sW1, kIn, kH, false); });
    if (!ok) break;
    uint64_t mask1 = 0, mask2 = 0;
    for (int c = 0; c < kH; c += 16) {
      float v[16];
      tmem_ld16(tl + cD1 + c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float z = v[i] + bias[c + i];
        v[i] = z > 0.0f ? z : 0.0f;
        if (z > 0.0f) mask1 |= 1ull << (c + i);
      }
      st_row8(smem + sH1, tid, c, kH, v);
      st_row8(smem + sH1, tid, c + 8, kH, v + 8);
      if (kTrain)
#pragma unroll
        for (int i = 0; i < 16; ++i) st_one(smem + sAh, 64 + c + i, tid, kRows, v[i]);
    }
    // ---- layer 2
    sync_mma([&] { gemm(tmem + cD2, sbase + sH1, sbase + sW2, kH, kH, false); });
    if (!ok) break;
    for (int c = 0; c < kH; c += 16) {
      float v[16];
      tmem_ld16(tl + cD2 + c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float z = v[i] + bias[64 + c + i];
        v[i] = z > 0.0f ? z : 0.0f;
        if (z > 0.0f) mask2 |= 1ull << (c + i);
      }
      st_row8(smem + sH2, tid, c, kH, v);
      st_row8(smem + sH2, tid, c + 8, kH, v + 8);
      if (kTrain)
#pragma unroll
        for (int i = 0; i < 16; ++i) st_one(smem + sAh, c + i, tid, kRows, v[i]);
    }
    // ---- layer 3
    sync_mma([&] { gemm(tmem + cD3, sbase + sH2, sbase + sW3, kH, kOutPad, false); });
    if (!ok) break;
    float l[16];
    tmem_ld16(tl + cD3, l);
    const float z1 = l[0] + bias[128], z2 = l[1] + bias[129], z3 = l[2] + bias[130];
    if constexpr (!kTrain) {
      if (valid) {
        logits[(size_t)row * 3 + 0] = z1;
        logits[(size_t)row * 3 + 1] = z2;
        logits[(size_t)row * 3 + 2] = z3;
      }
      first = false;
      continue;
    } else {
    // ---- softmax cross-entropy over {keep (logit 0), clone, split, prune}
    float d3[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) d3[i] = 0.0f;
    if (valid) {
      const uint32_t y = labels[src] & 3u;
      const float wy = y == 0 ? class_w.x : y == 1 ? class_w.y : y == 2 ? class_w.z : class_w.w;
      const float zz[4] = {0.0f, z1, z2, z3};
      float m = zz[0];
      int am = 0;
      for (int k = 1; k < 4; ++k)
        if (zz[k] > m) m = zz[k], am = k;
      float e[4], se = 0.0f;
      for (int k = 0; k < 4; ++k) se += (e[k] = expf(zz[k] - m));
      loss_acc += wy * (logf(se) - (zz[y] - m)) * inv_batch;
      correct_acc += (uint32_t)am == y ? 1.0f : 0.0f;
      for (int k = 1; k < 4; ++k) d3[k - 1] = wy * (e[k] / se - (k == (int)y ? 1.0f : 0.0f)) * inv_batch;
    }
    for (int k = 0; k < 3; ++k) {
      const float s = warp_sum(d3[k]);
      if (lane == 0) redw[128 + k] += s;
    }
    st_row8(smem + sdZ3, tid, 0, kOutPad, d3);
    st_row8(smem + sdZ3, tid, 8, kOutPad, d3 + 8);
#pragma unroll
    for (int k = 0; k < 3; ++k) st_one(smem + sdZ3T, k, tid, kRows, d3[k]);
    // ---- dH2 = dZ3 W3 and dW3^T += H2^T dZ3
    sync_mma([&] {
      gemm(tmem + cD1, sbase + sdZ3, sbase + sW3T, kOutPad, kH, false);
      gemm(tmem + cDC, sbase + sAh, sbase + sdZ3T, kRows, kOutPad, !first);
    });
    if (!ok) break;
    for (int c = 0; c < kH; c += 16) {
      float v[16];
      tmem_ld16(tl + cD1 + c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        v[i] = ((mask2 >> (c + i)) & 1ull) ? v[i] : 0.0f;
        const float s = warp_sum(v[i]);
        if (lane == 0) redw[64 + c + i] += s;
      }
      st_row8(smem + sdZ2, tid, c, kH, v);
      st_row8(smem + sdZ2, tid, c + 8, kH, v + 8);
#pragma unroll
      for (int i = 0; i < 16; ++i) st_one(smem + sAdz, c + i, tid, kRows, v[i]);
    }
    // ---- dH1 = dZ2 W2
    sync_mma([&] { gemm(tmem + cD2, sbase + sdZ2, sbase + sW2T, kH, kH, false); });
    if (!ok) break;
    for (int c = 0; c < kH; c += 16) {
      float v[16];
      tmem_ld16(tl + cD2 + c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        v[i] = ((mask1 >> (c + i)) & 1ull) ? v[i] : 0.0f;
        const float s = warp_sum(v[i]);
        if (lane == 0) redw[c + i] += s;
      }
#pragma unroll
      for (int i = 0; i < 16; ++i) st_one(smem + sAdz, 64 + c + i, tid, kRows, v[i]);
    }
    // ---- dW2 += dZ2^T H1 (rows 0..63), dW1 += dZ1^T X (rows 64..127)
    sync_mma([&] {
      gemm(tmem + cDA, sbase + sAdz, sbase + sAh + 8u * (kRows * 16u), kRows, kH, !first);
      gemm(tmem + cDB, sbase + sAdz, sbase + sXT, kRows, kIn, !first);
    });
    first = false;
    }
  }

  if (kTrain) {
    float* part = out.partial + (size_t)blockIdx.x * kPartial;
    if (ok && !first) {
      // accumulated weight gradients: TMEM -> this block's row
      if (warp < 2) {
        const uint32_t o = tid;  // output feature of W2, input feature of W3
        for (int c = 0; c < kH; c += 16) {
          float v[16];
          tmem_ld16(tl + cDA + c, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) part[oW2 + o * kH + c + i] = v[i];
        }
        float v[16];
        tmem_ld16(tl + cDC, v);
#pragma unroll
        for (int k = 0; k < kOut; ++k) part[oW3 + k * kH + o] = v[k];
      } else {
        const uint32_t o = tid - 64;  // output feature of W1
        float v[16];
        tmem_ld16(tl + cDB, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) part[oW1 + o * kIn + i] = v[i];
      }
      const float ls = warp_sum(loss_acc), cs = warp_sum(correct_acc);
      if (lane == 0) {
        redw[132] = ls;
        redw[133] = cs;
      }
      __syncthreads();
      // bias gradients, loss and count: the warps' sums in warp order
      for (uint32_t i = tid; i < 133; i += kThreads) {
        const uint32_t src = i < 131 ? i : 132;
        float t = 0.0f;
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w) t += red[w * kRedSlot + src];
        if (i < 131) {
          const int dst = i < 64 ? oB1 + i : i < 128 ? oB2 + (i - 64) : oB3 + (i - 128);
          part[dst] = t;
        } else {
          part[kNumParams] = t;
        }
      }
      if (tid == 0) {
        float c = 0.0f;
        for (int w = 0; w < kThreads / 32; ++w) c += red[w * kRedSlot + 133];
        part[kNumParams + 1] = c;
      }
    } else {
      for (uint32_t i = tid; i < kPartial; i += kThreads) part[i] = 0.0f;
    }
  }
  if (!ok) {
    // a product did not complete in time: give it one more bounded wait, so
    // that TMEM is not released under it, and report the failure
    bar_wait(bar, phase ^ 1u);
    if (tid == 0) atomicExch(err, 1u);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// Adam on the fp32 parameter vector (bias-corrected, no weight decay)
__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, uint32_t n, float lr, float bc1, float bc2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = 0.9f * m[i] + 0.1f * gi, vi = 0.999f * v[i] + 0.001f * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
}

// Adds the blocks' rows of `partial` in block order: gradient sums into
// grads (zeroed by the caller per batch), loss and count into the running
// sums of the epoch.
__global__ void k_mlp_reduce(const float* __restrict__ partial, uint32_t nblocks, float* __restrict__ grads,
                             float* __restrict__ loss, uint32_t* __restrict__ correct) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kPartial) return;
  float t = 0.0f;
  for (uint32_t b = 0; b < nblocks; ++b) t += partial[(size_t)b * kPartial + i];
  if (i < kNumParams) grads[i] += t;
  else if (i == kNumParams) *loss += t;
  else *correct += (uint32_t)(t + 0.5f);
}

}  // namespace mlp
}  // namespace nps

using namespace nps;

struct nps_mlp {
  nps_ctx* ctx = nullptr;
  DevBuf params, grads, m, v, loss, rows, err, partial;
  uint32_t step = 0;
  float last_loss = 0.0f, last_acc = 0.0f;
};

namespace {
int check_mlp(nps_mlp* o) {
  if (!o) {
    set_error("null MLP");
    return NPS_ERR_INVALID;
  }
  return bind_device(o->ctx);
}

int launch_mlp(nps_mlp* o, bool train, const float* X, const uint32_t* rows, const uint8_t* labels, uint32_t n,
               const float* cw4, float inv_batch, float* logits) {
  cudaStream_t s = o->ctx->stream;
  if (train)
    NPS_CUDA(cudaFuncSetAttribute(mlp::k_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::kSmemBytes));
  else
    NPS_CUDA(cudaFuncSetAttribute(mlp::k_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mlp::kSmemBytes));
  const uint32_t ntiles = div_up(n, mlp::kRows);
  const uint32_t grid = ntiles < (uint32_t)o->ctx->sm_count ? ntiles : (uint32_t)o->ctx->sm_count;
  if (train) NPS_TRY(o->partial.ensure(sizeof(float) * (size_t)grid * mlp::kPartial));
  mlp::TrainOut out{train ? o->partial.as<float>() : nullptr};
  const float4 cw = cw4 ? make_float4(cw4[0], cw4[1], cw4[2], cw4[3]) : make_float4(1, 1, 1, 1);
  if (train) {
    mlp::k_mlp<true><<<grid, mlp::kThreads, mlp::kSmemBytes, s>>>(o->params.as<float>(), X, rows, labels, n, cw,
                                                                 inv_batch, out, nullptr, o->err.as<uint32_t>());
    mlp::k_mlp_reduce<<<div_up(mlp::kPartial, 256), 256, 0, s>>>(o->partial.as<float>(), grid, o->grads.as<float>(),
                                                                 o->loss.as<float>(), o->loss.as<uint32_t>() + 1);
  } else {
    mlp::k_mlp<false><<<grid, mlp::kThreads, mlp::kSmemBytes, s>>>(o->params.as<float>(), X, rows, labels, n, cw,
                                                                  inv_batch, out, logits, o->err.as<uint32_t>());
  }
  NPS_CHECK_LAUNCH();
  return NPS_OK;
}

int check_err(nps_mlp* o) {
  uint32_t e = 0;
  NPS_CUDA(cudaMemcpyAsync(&e, o->err.p, 4, cudaMemcpyDeviceToHost, o->ctx->stream));
  NPS_CUDA(cudaStreamSynchronize(o->ctx->stream));
  if (e) {
    NPS_CUDA(cudaMemsetAsync(o->err.p, 0, 4, o->ctx->stream));
    set_error("mlp: a tensor-core wait timed out");
    return NPS_ERR_CUDA;
  }
  return NPS_OK;
}
}  // namespace

extern "C" {

int nps_mlp_create(nps_ctx* ctx, nps_mlp** out) {
  if (!ctx || !out) return NPS_ERR_INVALID;
  NPS_TRY(bind_device(ctx));
  nps_mlp* o = new nps_mlp();
  o->ctx = ctx;
  const size_t pb = sizeof(float) * mlp::kNumParams;
  int rc;
  if ((rc = o->params.ensure(pb)) || (rc = o->grads.ensure(pb)) || (rc = o->m.ensure(pb)) ||
      (rc = o->v.ensure(pb)) || (rc = o->loss.ensure(16)) || (rc = o->err.ensure(16))) {
    delete o;
    return rc;
  }
  cudaStream_t s = ctx->stream;
  cudaMemsetAsync(o->params.p, 0, pb, s);
  cudaMemsetAsync(o->m.p, 0, pb, s);
  cudaMemsetAsync(o->v.p, 0, pb, s);
  cudaMemsetAsync(o->err.p, 0, 16, s);
  *out = o;
  return NPS_OK;
}

int nps_mlp_destroy(nps_mlp* o) {
  if (!o) return NPS_OK;
  bind_device(o->ctx);
  cudaStreamSynchronize(o->ctx->stream);
  for (DevBuf* b : {&o->params, &o->grads, &o->m, &o->v, &o->loss, &o->rows, &o->err, &o->partial}) b->release();
  delete o;
  return NPS_OK;
}

int nps_mlp_num_params(void) { return mlp::kNumParams; }

int nps_mlp_init(nps_mlp* o, uint64_t seed) {
  NPS_TRY(check_mlp(o));
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.0f, 1.0f);
  std::vector<float> p(mlp::kNumParams, 0.0f);
  // He initialisation for the ReLU layers, small output layer, zero biases
  for (int i = 0; i < mlp::kH * mlp::kIn; ++i) p[mlp::oW1 + i] = nd(rng) * std::sqrt(2.0f / mlp::kIn);
  for (int i = 0; i < mlp::kH * mlp::kH; ++i) p[mlp::oW2 + i] = nd(rng) * std::sqrt(2.0f / mlp::kH);
  for (int i = 0; i < mlp::kOut * mlp::kH; ++i) p[mlp::oW3 + i] = nd(rng) * std::sqrt(1.0f / mlp::kH);
  o->step = 0;
  cudaStream_t s = o->ctx->stream;
  NPS_CUDA(cudaMemcpyAsync(o->params.p, p.data(), sizeof(float) * p.size(), cudaMemcpyHostToDevice, s));
  NPS_CUDA(cudaMemsetAsync(o->m.p, 0, sizeof(float) * p.size(), s));
  NPS_CUDA(cudaMemsetAsync(o->v.p, 0, sizeof(float) * p.size(), s));
  NPS_CUDA(cudaStreamSynchronize(s));
  return NPS_OK;
}

int nps_mlp_set_params(nps_mlp* o, const float* params_host) {
  NPS_TRY(check_mlp(o));
  if (!params_host) return NPS_ERR_INVALID;
  NPS_CUDA(cudaMemcpyAsync(o->params.p, params_host, sizeof(float) * mlp::kNumParams, cudaMemcpyHostToDevice,
                           o->ctx->stream));
  NPS_CUDA(cudaStreamSynchronize(o->ctx->stream));
  return NPS_OK;
}

int nps_mlp_get_params(nps_mlp* o, float* params_host) {
  NPS_TRY(check_mlp(o));
  if (!params_host) return NPS_ERR_INVALID;
  NPS_CUDA(cudaMemcpyAsync(params_host, o->params.p, sizeof(float) * mlp::kNumParams, cudaMemcpyDeviceToHost,
                           o->ctx->stream));
  NPS_CUDA(cudaStreamSynchronize(o->ctx->stream));
  return NPS_OK;
}

int nps_mlp_forward(nps_mlp* o, const float* features_dev, uint32_t n, float* logits_dev) {
  NPS_TRY(check_mlp(o));
  if (n == 0) return NPS_OK;
  if (!features_dev || !logits_dev) return NPS_ERR_INVALID;
  NPS_TRY(launch_mlp(o, false, features_dev, nullptr, nullptr, n, nullptr, 0.0f, logits_dev));
  return check_err(o);
}

int nps_mlp_grads(nps_mlp* o, const float* features_dev, const uint8_t* labels_dev, uint32_t n,
                  const float* class_w4, float* grads_host, float* loss_host) {
  NPS_TRY(check_mlp(o));
  if (!features_dev || !labels_dev || n == 0) return NPS_ERR_INVALID;
  cudaStream_t s = o->ctx->stream;
  NPS_CUDA(cudaMemsetAsync(o->grads.p, 0, sizeof(float) * mlp::kNumParams, s));
  NPS_CUDA(cudaMemsetAsync(o->loss.p, 0, 16, s));
  NPS_TRY(launch_mlp(o, true, features_dev, nullptr, labels_dev, n, class_w4, 1.0f / (float)n, nullptr));
  NPS_TRY(check_err(o));
  if (grads_host)
    NPS_CUDA(cudaMemcpyAsync(grads_host, o->grads.p, sizeof(float) * mlp::kNumParams, cudaMemcpyDeviceToHost, s));
  if (loss_host) NPS_CUDA(cudaMemcpyAsync(loss_host, o->loss.p, sizeof(float), cudaMemcpyDeviceToHost, s));
  NPS_CUDA(cudaStreamSynchronize(s));
  return NPS_OK;
}

// Mini-batch Adam over device-resident (features, labels); rows reshuffled
// every epoch (seeded).  loss_curve / acc_curve (host, may be null): mean
// weighted loss and accuracy of each epoch.
int nps_mlp_train(nps_mlp* o, const float* features_dev, const uint8_t* labels_dev, uint32_t n,
                  const float* class_w4, uint32_t epochs, uint32_t batch, float lr, uint64_t seed,
                  float* loss_curve, float* acc_curve) {
  NPS_TRY(check_mlp(o));
  if (!features_dev || !labels_dev || n == 0 || batch == 0) return NPS_ERR_INVALID;
  cudaStream_t s = o->ctx->stream;
  NPS_TRY(o->rows.ensure(sizeof(uint32_t) * n));
  std::vector<uint32_t> perm(n);
  for (uint32_t i = 0; i < n; ++i) perm[i] = i;
  std::mt19937_64 rng(seed);
  const uint32_t nb = (n + batch - 1) / batch;
  for (uint32_t ep = 0; ep < epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    NPS_CUDA(cudaMemcpyAsync(o->rows.p, perm.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s));
    NPS_CUDA(cudaMemsetAsync(o->loss.p, 0, 16, s));
    for (uint32_t b = 0; b < nb; ++b) {
      const uint32_t r0 = b * batch, cnt = std::min(batch, n - r0);
      NPS_CUDA(cudaMemsetAsync(o->grads.p, 0, sizeof(float) * mlp::kNumParams, s));
      NPS_TRY(launch_mlp(o, true, features_dev, o->rows.as<uint32_t>() + r0, labels_dev, cnt, class_w4,
                         1.0f / (float)cnt, nullptr));
      o->step += 1;
      const float bc1 = (float)(1.0 - std::pow(0.9, (double)o->step));
      const float bc2 = (float)(1.0 - std::pow(0.999, (double)o->step));
      mlp::k_mlp_adam<<<div_up(mlp::kNumParams, 256), 256, 0, s>>>(o->params.as<float>(), o->grads.as<float>(),
                                                                    o->m.as<float>(), o->v.as<float>(),
                                                                    mlp::kNumParams, lr, bc1, bc2);
      NPS_CHECK_LAUNCH();
    }
    float lc[2];
    NPS_CUDA(cudaMemcpyAsync(lc, o->loss.p, 8, cudaMemcpyDeviceToHost, s));
    NPS_TRY(check_err(o));
    uint32_t correct;
    std::memcpy(&correct, &lc[1], 4);
    o->last_loss = lc[0] / (float)nb;
    o->last_acc = (float)correct / (float)n;
    if (loss_curve) loss_curve[ep] = o->last_loss;
    if (acc_curve) acc_curve[ep] = o->last_acc;
  }
  return NPS_OK;
}

}  // extern "C"
