// BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05),
// C[M x N] = A[M x K] * B[N x K]^T, both operands K-major (row-major with K
// contiguous), one 128-row tile of C per CTA and an optional split of K
// across gridDim.y. The accumulator lives in TMEM; one elected thread issues
// the MMAs; K chunks are double-buffered in shared memory (cp.async) and a
// chunk's buffer is refilled only after the tcgen05.commit of the MMAs that
// read it has arrived on that buffer's mbarrier.
//
// Epilogues (one thread per row of the tile, 16 TMEM columns per load):
//   kEpiF32    C = acc (+ bias[n])                       fp32, row stride ldc
//   kEpiAtomic C += acc (fp32 atomics; split-K partial sums)
//   kEpiSilu   Z = acc + bias[n] (fp32, optional), H = bf16(silu(Z))
// silu(z) = z * sigmoid(z) with sigmoid(z) = 0.5 + 0.5 tanh(z / 2), tanh from
// the hardware tanh.approx instruction; the same function is used by the
// fused inference kernel, so training and inference see one activation.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "ns_tc.cuh"

namespace ns {
namespace gemm {

constexpr int kEpiF32 = 0;
constexpr int kEpiAtomic = 1;
constexpr int kEpiSilu = 2;

// bounded mbarrier waits: about a second of polling before giving up
constexpr uint32_t kWaitLimit = 1u << 22;
constexpr uint32_t kErrWait = 1u;

struct Args {
  const uint16_t* A;    // [M][lda] bf16
  const uint16_t* B;    // [N][ldb] bf16
  float* C;             // [M][ldc] fp32 (F32 / Atomic), or Z for Silu (may be null)
  uint16_t* H;          // [M][ldh] bf16 (Silu)
  const float* bias;    // [N] or null
  uint32_t M, K;
  uint32_t lda, ldb, ldc, ldh;
  uint32_t k_per_split; // multiple of the chunk
  uint32_t* err;        // device status word (bit 0: a wait gave up)
};

__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sigmoid_t(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }
__device__ __forceinline__ float silu_t(float z) { return z * sigmoid_t(z); }

__device__ __forceinline__ uint16_t f32_to_bf16_rn(float x) {
  const __nv_bfloat16 b = __float2bfloat16_rn(x);
  return *reinterpret_cast<const uint16_t*>(&b);
}

// lo | hi << 16 as BF16, both rounded to nearest even by one packed
// conversion (the same values as two f32_to_bf16_rn)
__device__ __forceinline__ uint32_t pack_bf16x2_rn(float lo, float hi) {
  const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&p);
}

// x = hi + lo with hi = bf16(x): the BF16 pair carries ~16 significant bits
// of x into a tensor-core product whose weight column is duplicated.
__device__ __forceinline__ void split_bf16(float x, uint16_t& hi, uint16_t& lo) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  hi = *reinterpret_cast<const uint16_t*>(&h);
  lo = f32_to_bf16_rn(x - __bfloat162float(h));
}

// Copies rows [0, R) x K-chunk [k0, k0 + KC) of a K-major bf16 matrix into
// the canonical no-swizzle layout of an R x KC tile (16-byte pieces).
template <int R, int KC>
__device__ __forceinline__ void load_tile(uint8_t* dst, const uint16_t* src, uint32_t ld,
                                          uint32_t row0, uint32_t k0) {
  constexpr int kPieces = R * (KC / 8);
#pragma unroll
  for (int q = threadIdx.x; q < kPieces; q += 128) {
    const uint32_t r = (uint32_t)q / (KC / 8), c = (uint32_t)q % (KC / 8);
    const uint16_t* g = src + (uint64_t)(row0 + r) * ld + k0 + c * 8;
    tc::cp_async16(dst + tc::kmajor_offset(r, c * 8, KC), g);
  }
}

template <int N, int KC, int EPI>
__global__ void __launch_bounds__(128) k_gemm(Args g) {
  constexpr uint32_t kABytes = 128u * KC * 2u;
  constexpr uint32_t kBBytes = (uint32_t)N * KC * 2u;
  constexpr uint32_t kStage = kABytes + kBBytes;
  constexpr uint32_t kCols = N < 32 ? 32u : (uint32_t)N;   // TMEM columns (power of two)
  static_assert(N == 16 || N == 32 || N == 64 || N == 128 || N == 256, "N");
  static_assert(KC % 16 == 0, "KC");
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t mbar[2];
  __shared__ uint32_t tmem_base;

  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const uint32_t row0 = blockIdx.x * 128u;
  const uint32_t kb = blockIdx.y * g.k_per_split;
  const uint32_t ke = min(kb + g.k_per_split, g.K);
  const uint32_t nch = ke > kb ? (ke - kb) / KC : 0u;

  if (warp == 0) tc::tmem_alloc(&tmem_base, kCols);
  if (tid == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tacc = tmem_base;
  const uint32_t idesc = tc::idesc_bf16(N);
  bool ok = true;

  if (nch > 0) {
    load_tile<128, KC>(smem, g.A, g.lda, row0, kb);
    load_tile<N, KC>(smem + kABytes, g.B, g.ldb, 0, kb);
    tc::cp_async_commit();
  }
  for (uint32_t c = 0; c < nch; ++c) {
    const uint32_t s = c & 1u;
    tc::cp_async_wait_all();
    tc::fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t a0 = tc::smem_u32(smem + s * kStage);
      const uint32_t b0 = a0 + kABytes;
#pragma unroll
      for (int ks = 0; ks < KC / 16; ++ks) {
        const uint64_t ad = tc::smem_desc(a0 + ks * 256u, 128u, (KC / 8) * 128u);
        const uint64_t bd = tc::smem_desc(b0 + ks * 256u, 128u, (KC / 8) * 128u);
        tc::mma_bf16(tacc, ad, bd, idesc, (c > 0 || ks > 0) ? 1u : 0u);
      }
      tc::commit(&mbar[s]);
    }
    if (c + 1 < nch) {
      const uint32_t s1 = (c + 1) & 1u;
      // the buffer of chunk c + 1 was last read by the MMAs of chunk c - 1
      if (c >= 1 && !tc::mbar_wait(&mbar[s1], ((c - 1) >> 1) & 1u, kWaitLimit)) ok = false;
      load_tile<128, KC>(smem + s1 * kStage, g.A, g.lda, row0, kb + (c + 1) * KC);
      load_tile<N, KC>(smem + s1 * kStage + kABytes, g.B, g.ldb, 0, kb + (c + 1) * KC);
      tc::cp_async_commit();
    }
  }
  // the last commit covers every MMA issued before it
  if (nch > 0 && !tc::mbar_wait(&mbar[(nch - 1) & 1u], ((nch - 1) >> 1) & 1u, kWaitLimit)) ok = false;
  tc::fence_after_sync();

  if (nch > 0) {
    const uint32_t r = row0 + warp * 32u + (tid & 31u);
    const uint32_t tl = tacc + ((warp * 32u) << 16);
#pragma unroll 1
    for (uint32_t j = 0; j < (uint32_t)N; j += 16) {
      float v[16];
      tc::tmem_ld16(tl + j, v);
      if (r < g.M) {
        if (EPI == kEpiF32) {
          float* out = g.C + (uint64_t)r * g.ldc + j;
#pragma unroll
          for (int q = 0; q < 16; ++q) out[q] = v[q] + (g.bias ? g.bias[j + q] : 0.0f);
        } else if (EPI == kEpiAtomic) {
          float* out = g.C + (uint64_t)r * g.ldc + j;
#pragma unroll
          for (int q = 0; q < 16; ++q) atomicAdd(out + q, v[q]);
        } else {
          uint32_t packed[8];
#pragma unroll
          for (int q = 0; q < 16; q += 2) {
            const float z0 = v[q] + (g.bias ? g.bias[j + q] : 0.0f);
            const float z1 = v[q + 1] + (g.bias ? g.bias[j + q + 1] : 0.0f);
            if (g.C) {
              g.C[(uint64_t)r * g.ldc + j + q] = z0;
              g.C[(uint64_t)r * g.ldc + j + q + 1] = z1;
            }
            packed[q / 2] = pack_bf16x2_rn(silu_t(z0), silu_t(z1));
          }
          uint4* hp = reinterpret_cast<uint4*>(g.H + (uint64_t)r * g.ldh + j);
          hp[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
          hp[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
        }
      }
    }
  }
  if (!ok && (tid & 31u) == 0) atomicOr(g.err, kErrWait);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tacc, kCols);
}

template <int N, int KC>
constexpr uint32_t smem_bytes() {
  return 2u * (128u * KC * 2u + (uint32_t)N * KC * 2u);
}

}  // namespace gemm
}  // namespace ns
