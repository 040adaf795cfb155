// Learned Hodgkin-Huxley macro-step: training and standalone inference of the
// 5 -> 128 -> 128 -> 4 SiLU MLP on the tensor cores (tcgen05 BF16 GEMMs of
// ns_gemm.cuh), targets from the network's own Rush-Larsen arithmetic
// (ns_hh.cuh), Adam in FP32. No counterpart in the reference; it replaces
// NS_SUR_SUBSTEPS Rush-Larsen steps of HodgkinHuxleyNeuron::step
// (src/neuron/hodgkin_huxley.rs:46-96) for neurons in the training envelope.
//
// Per training step (batch B rows, all matrices row-major):
//   forward   Z1 = Xp W1p^T + b1, H1 = silu(Z1)        GEMM  B x 128 x 16
//             Z2 = H1 W2^T + b2,  H2 = silu(Z2)         GEMM  B x 128 x 128
//             Y  = H2 W3p^T (+ b3 in the loss kernel)    GEMM  B x 16 x 128
//   loss      L = mean over B x 4 of (Y - T)^2, dY = 2 (Y - T) / (4 B)
//   backward  dH2 = dY W3                               GEMM  B x 128 x 16
//             dZ2 = dH2 * silu'(Z2)
//             dW2 = dZ2^T H1, dW3 = dY^T H2             GEMM  128 x 128 x B (split K)
//             dH1 = dZ2 W2                              GEMM  B x 128 x 128
//             dZ1 = dH1 * silu'(Z1), dW1 = dZ1^T X      GEMM  128 x 16 x B (split K)
//   update    Adam on the FP32 master weights, then their BF16 copies (and
//             the transposed copies the backward GEMMs read).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/neuralsim_surrogate.h"
#include "ns_gemm.cuh"
#include "ns_hh.cuh"
#include "ns_sur_internal.h"

namespace {

constexpr int kH = NS_SUR_HIDDEN;
constexpr int kPW1 = 0, kPB1 = 640, kPW2 = 768, kPB2 = 768 + 16384, kPW3 = kPB2 + 128, kPB3 = kPW3 + 512;
static_assert(kPB3 + 4 == NS_SUR_PARAMS, "parameter count");

struct Norm {
  float in_mean[5], in_scale[5], out_mean[4], out_scale[4];
};
struct HhP {
  float p[7];
};

thread_local std::string g_sur_err;

}  // namespace

struct ns_sur {
  int dev = 0;
  cudaStream_t st = nullptr;
  std::string err;
  HhP hh{};
  float dt = 0.01f;
  uint32_t B = 0;
  uint64_t seed = 0;
  uint64_t sample_seed = 0;             // minibatch sampling stream
  uint64_t t = 0;                       // Adam steps taken
  Norm norm{};
  std::vector<void*> allocs;
  float *P = nullptr, *Am = nullptr, *Av = nullptr;
  uint16_t *W1p = nullptr, *W2b = nullptr, *W2T = nullptr, *W3p = nullptr, *W3T = nullptr;
  float *X = nullptr, *Y = nullptr;     // training set (raw)
  uint64_t n_data = 0;
  float *Xs = nullptr, *Ys = nullptr;   // B rows of caller data (gradient / predict)
  uint16_t *Xp = nullptr, *XT = nullptr, *H1 = nullptr, *H2 = nullptr, *dYb = nullptr, *dYT = nullptr;
  uint16_t *dZ2 = nullptr, *dZ2T = nullptr, *dZ1 = nullptr, *dZ1T = nullptr, *H1T = nullptr, *H2T = nullptr;
  float *Z1 = nullptr, *Z2 = nullptr, *Yo = nullptr, *Tn = nullptr, *dH2 = nullptr, *dH1 = nullptr;
  float *gW1 = nullptr, *gW2 = nullptr, *gW3 = nullptr, *gB = nullptr, *G = nullptr;
  float* lossv = nullptr;
  uint32_t loss_cap = 0;
  uint32_t* errw = nullptr;
};

namespace {

ns_status sfail(ns_sur* s, ns_status st, const std::string& m) {
  if (s) s->err = m; else g_sur_err = m;
  return st;
}

#define SCK(call)                                                                          \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return sfail(s, e_ == cudaErrorMemoryAllocation ? NS_ERR_OOM : NS_ERR_CUDA,          \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                    \
  } while (0)

template <class T> cudaError_t salloc(ns_sur* s, T** p, size_t count) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 16));
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(q, 0, std::max<size_t>(count * sizeof(T), 16), s->st);
  s->allocs.push_back(q);
  *p = (T*)q;
  return e;
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Targets: NS_SUR_SUBSTEPS Rush-Larsen steps with the synaptic current held.
__global__ void k_sur_targets(const float* X, float* Y, uint64_t n, HhP hp, float dt) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    float v = X[i * 5 + 0], m = X[i * 5 + 1], h = X[i * 5 + 2], nn = X[i * 5 + 3];
    const float I = X[i * 5 + 4];
#pragma unroll 1
    for (int q = 0; q < NS_SUR_SUBSTEPS; ++q) ns::hh_rl_step(v, m, h, nn, I, hp.p, dt);
    Y[i * 4 + 0] = v; Y[i * 4 + 1] = m; Y[i * 4 + 2] = h; Y[i * 4 + 3] = nn;
  }
}

// One Rush-Larsen step of the macro-step's length with the current held:
// the base the MLP's output corrects.
__device__ __forceinline__ void sur_base(const float* x, const HhP& hp, float dt_macro, float* b) {
  float v = x[0], m = x[1], h = x[2], n = x[3];
  ns::hh_rl_step(v, m, h, n, x[4], hp.p, dt_macro);
  b[0] = v; b[1] = m; b[2] = h; b[3] = n;
}

// Batch assembly: normalised inputs (Xp [B][16], XT [16][B]; column k < 5
// holds the BF16 value of input k, column 5 + k its BF16 remainder, the
// rest zero) and normalised targets Tn [B][4]: the state 0.1 ms later minus
// the base. Row b takes sample
// hash(seed, step, b) mod n when sampling, else row first + b (zeros past
// n_valid).
__global__ void k_sur_gather(uint32_t B, const float* X, const float* Y, uint64_t n, int sample,
                             uint64_t seed, uint64_t step, uint64_t first, uint64_t n_valid,
                             Norm nm, HhP hp, float dt_macro, uint16_t* Xp, uint16_t* XT, float* Tn) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  uint64_t idx;
  bool valid = true;
  if (sample) {
    idx = mix64(seed ^ mix64(step * 0x100000001B3ull + b)) % n;
  } else {
    idx = first + b;
    valid = idx < n_valid;
  }
  float x[5], y[4];
#pragma unroll
  for (int k = 0; k < 5; ++k) x[k] = valid ? X[idx * 5 + k] : 0.0f;
#pragma unroll
  for (int k = 0; k < 4; ++k) y[k] = (valid && Y) ? Y[idx * 4 + k] : 0.0f;
  uint16_t col[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) col[k] = 0;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const float xn = valid ? (x[k] - nm.in_mean[k]) / nm.in_scale[k] : 0.0f;
    ns::gemm::split_bf16(xn, col[k], col[5 + k]);
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    Xp[(uint64_t)b * 16 + k] = col[k];
    XT[(uint64_t)k * B + b] = col[k];
  }
  if (Tn) {
    float base[4] = {0.f, 0.f, 0.f, 0.f};
    if (valid) sur_base(x, hp, dt_macro, base);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      Tn[(uint64_t)b * 4 + k] = valid ? ((y[k] - base[k]) - nm.out_mean[k]) / nm.out_scale[k] : 0.0f;
  }
}

// Loss and its gradient at the output: Y = Yo + b3; dY = 2 (Y - T) / (4 B)
// into dYb [B][16] (bf16) and dYT [rows 0..3][B]; db3 and the loss summed.
__global__ void k_sur_loss(uint32_t B, const float* Yo, const float* b3, const float* Tn,
                           uint16_t* dYb, uint16_t* dYT, float* gb3, float* loss) {
  __shared__ float red[5][8];
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  const float inv = 2.0f / (4.0f * (float)B);
  float l = 0.0f, g[4] = {0.f, 0.f, 0.f, 0.f};
  if (b < B) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float e = Yo[(uint64_t)b * 16 + j] + b3[j] - Tn[(uint64_t)b * 4 + j];
      l += e * e;
      g[j] = inv * e;
      const uint16_t q = ns::gemm::f32_to_bf16_rn(g[j]);
      dYb[(uint64_t)b * 16 + j] = q;
      dYT[(uint64_t)j * B + b] = q;
    }
  }
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  float v[5] = {l / (4.0f * (float)B), g[0], g[1], g[2], g[3]};
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if (lane == 0) red[q][w] = v[q];
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    float t = 0.0f;
    for (uint32_t q = 0; q < blockDim.x / 32; ++q) t += red[threadIdx.x][q];
    if (threadIdx.x == 0) atomicAdd(loss, t);
    else atomicAdd(gb3 + threadIdx.x - 1, t);
  }
}

// dZ = dH * silu'(Z) (bf16 out) and the bias gradient (column sums). One
// block of 256 threads covers 2 rows x 128 columns per iteration.
__global__ void k_sur_silu_back(uint32_t B, const float* dH, const float* Z, uint16_t* dZ, float* gb) {
  const uint32_t col = threadIdx.x & 127u, half = threadIdx.x >> 7;
  float acc = 0.0f;
  for (uint32_t r = blockIdx.x * 2 + half; r < B; r += gridDim.x * 2) {
    const uint64_t o = (uint64_t)r * kH + col;
    const float z = Z[o];
    const float sg = ns::gemm::sigmoid_t(z);
    const float d = dH[o] * (sg + z * sg * (1.0f - sg));
    dZ[o] = ns::gemm::f32_to_bf16_rn(d);
    acc += d;
  }
  __shared__ float red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  if (half == 0) atomicAdd(gb + col, red[col] + red[col + 128]);
}

// [R][C] -> [C][R], bf16, 32 x 32 tiles.
__global__ void k_transpose16(const uint16_t* in, uint16_t* out, uint32_t R, uint32_t C) {
  __shared__ uint16_t t[32][33];
  const uint32_t c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (uint32_t y = threadIdx.y; y < 32; y += blockDim.y) {
    const uint32_t r = r0 + y, c = c0 + threadIdx.x;
    t[y][threadIdx.x] = (r < R && c < C) ? in[(uint64_t)r * C + c] : (uint16_t)0;
  }
  __syncthreads();
  for (uint32_t y = threadIdx.y; y < 32; y += blockDim.y) {
    const uint32_t c = c0 + y, r = r0 + threadIdx.x;
    if (c < C && r < R) out[(uint64_t)c * R + r] = t[threadIdx.x][y];
  }
}

// Flat gradient from the GEMM accumulators, in parameter order.
__device__ __forceinline__ float grad_of(uint32_t q, const float* gW1, const float* gW2,
                                         const float* gW3, const float* gB) {
  if (q < (uint32_t)kPB1) return gW1[(q / 5) * 16 + (q % 5)] + gW1[(q / 5) * 16 + 5 + (q % 5)];
  if (q < (uint32_t)kPW2) return gB[q - kPB1];
  if (q < (uint32_t)kPB2) return gW2[q - kPW2];
  if (q < (uint32_t)kPW3) return gB[128 + (q - kPB2)];
  if (q < (uint32_t)kPB3) return gW3[q - kPW3];
  return gB[256 + (q - kPB3)];
}

// BF16 operand copies of parameter q (and transposes).
__device__ __forceinline__ void write_bf16(uint32_t q, float w, uint16_t* W1p, uint16_t* W2b,
                                           uint16_t* W2T, uint16_t* W3p, uint16_t* W3T) {
  const uint16_t b = ns::gemm::f32_to_bf16_rn(w);
  if (q < (uint32_t)kPB1) {
    W1p[(q / 5) * 16 + (q % 5)] = b;       // weight of the input's BF16 value
    W1p[(q / 5) * 16 + 5 + (q % 5)] = b;   // and of its remainder
  } else if (q >= (uint32_t)kPW2 && q < (uint32_t)kPB2) {
    const uint32_t o = (q - kPW2) / kH, i = (q - kPW2) % kH;
    W2b[o * kH + i] = b;
    W2T[i * kH + o] = b;
  } else if (q >= (uint32_t)kPW3 && q < (uint32_t)kPB3) {
    const uint32_t o = (q - kPW3) / kH, i = (q - kPW3) % kH;
    W3p[o * kH + i] = b;
    W3T[i * 16 + o] = b;
  }
}

__global__ void k_sur_adam(float* P, float* M, float* V, const float* gW1, const float* gW2,
                           const float* gW3, const float* gB, float lr, float c1, float c2,
                           uint16_t* W1p, uint16_t* W2b, uint16_t* W2T, uint16_t* W3p, uint16_t* W3T,
                           float* G) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= NS_SUR_PARAMS) return;
  const float g = grad_of(q, gW1, gW2, gW3, gB);
  if (G) { G[q] = g; return; }  // gradient only
  const float m = 0.9f * M[q] + 0.1f * g;
  const float v = 0.999f * V[q] + 0.001f * g * g;
  M[q] = m;
  V[q] = v;
  const float w = P[q] - lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
  P[q] = w;
  write_bf16(q, w, W1p, W2b, W2T, W3p, W3T);
}

// Adam from a flat gradient (data-parallel training: the gradient summed
// over ranks by the caller)
__global__ void k_sur_adam_flat(float* P, float* M, float* V, const float* g_in, float scale,
                                float lr, float c1, float c2, uint16_t* W1p, uint16_t* W2b,
                                uint16_t* W2T, uint16_t* W3p, uint16_t* W3T) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= NS_SUR_PARAMS) return;
  const float g = g_in[q] * scale;
  const float m = 0.9f * M[q] + 0.1f * g;
  const float v = 0.999f * V[q] + 0.001f * g * g;
  M[q] = m;
  V[q] = v;
  const float w = P[q] - lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
  P[q] = w;
  write_bf16(q, w, W1p, W2b, W2T, W3p, W3T);
}

__global__ void k_sur_refresh(const float* P, uint16_t* W1p, uint16_t* W2b, uint16_t* W2T,
                              uint16_t* W3p, uint16_t* W3T) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < NS_SUR_PARAMS) write_bf16(q, P[q], W1p, W2b, W2T, W3p, W3T);
}

// raw states 0.1 ms later from the network output
__global__ void k_sur_decode(uint32_t B, uint64_t first, uint64_t n, const float* X, const float* Yo,
                             const float* b3, Norm nm, HhP hp, float dt_macro, float* out) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t i = first + b;
  if (b >= B || i >= n) return;
  float base[4];
  sur_base(X + i * 5, hp, dt_macro, base);
#pragma unroll
  for (int k = 0; k < 4; ++k)
    out[i * 4 + k] = base[k] + (Yo[(uint64_t)b * 16 + k] + b3[k]) * nm.out_scale[k] + nm.out_mean[k];
}

template <int N, int KC, int EPI>
cudaError_t gemm_launch(const ns::gemm::Args& a, uint32_t M, uint32_t splits, cudaStream_t st) {
  const uint32_t sm = ns::gemm::smem_bytes<N, KC>();
  cudaError_t e = cudaFuncSetAttribute(ns::gemm::k_gemm<N, KC, EPI>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  ns::gemm::k_gemm<N, KC, EPI><<<dim3(M / 128, splits), 128, sm, st>>>(a);
  return cudaGetLastError();
}

// Dispatch over N (16 / 128), chunk (64 when the split is a multiple of 64,
// else 16) and epilogue.
cudaError_t gemm(const ns::gemm::Args& a0, uint32_t M, uint32_t N, uint32_t splits, int epi,
                 cudaStream_t st) {
  ns::gemm::Args a = a0;
  a.k_per_split = (a.K + splits - 1) / splits;
  const bool c64 = a.k_per_split % 64 == 0 && a.K % 64 == 0;
  if (!c64) a.k_per_split = (a.k_per_split + 15) / 16 * 16;
#define NS_G(NN, KC)                                                                \
  if (epi == 0) return gemm_launch<NN, KC, ns::gemm::kEpiF32>(a, M, splits, st);    \
  if (epi == 1) return gemm_launch<NN, KC, ns::gemm::kEpiAtomic>(a, M, splits, st); \
  return gemm_launch<NN, KC, ns::gemm::kEpiSilu>(a, M, splits, st);
  if (N == 16) {
    if (c64) { NS_G(16, 64) } else { NS_G(16, 16) }
  } else {
    if (c64) { NS_G(128, 64) } else { NS_G(128, 16) }
  }
#undef NS_G
}

ns::gemm::Args gargs(const uint16_t* A, uint32_t lda, const uint16_t* B, uint32_t ldb, float* C,
                     uint32_t ldc, uint16_t* H, uint32_t ldh, const float* bias, uint32_t M,
                     uint32_t K, uint32_t* err) {
  ns::gemm::Args a{};
  a.A = A; a.B = B; a.C = C; a.H = H; a.bias = bias;
  a.M = M; a.K = K; a.lda = lda; a.ldb = ldb; a.ldc = ldc; a.ldh = ldh;
  a.err = err;
  return a;
}

// Forward of the B rows already assembled in Xp: Z1/H1, Z2/H2, Yo.
cudaError_t forward(ns_sur* s) {
  const uint32_t B = s->B;
  cudaError_t e;
  if ((e = gemm(gargs(s->Xp, 16, s->W1p, 16, s->Z1, kH, s->H1, kH, s->P + kPB1, B, 16, s->errw), B,
                128, 1, 2, s->st)))
    return e;
  if ((e = gemm(gargs(s->H1, kH, s->W2b, kH, s->Z2, kH, s->H2, kH, s->P + kPB2, B, kH, s->errw), B,
                128, 1, 2, s->st)))
    return e;
  return gemm(gargs(s->H2, kH, s->W3p, kH, s->Yo, 16, nullptr, 0, nullptr, B, kH, s->errw), B, 16,
              1, 0, s->st);
}

// Loss, backward and (G == null) the Adam update, or (G != null) the flat
// gradient into G.
cudaError_t backward_update(ns_sur* s, float* loss_slot, float lr, float* G) {
  const uint32_t B = s->B;
  const uint32_t splits = std::max<uint32_t>(1u, B / 512u);
  cudaError_t e;
  if ((e = cudaMemsetAsync(s->gW1, 0, 128 * 16 * 4, s->st))) return e;
  if ((e = cudaMemsetAsync(s->gW2, 0, kH * kH * 4, s->st))) return e;
  if ((e = cudaMemsetAsync(s->gW3, 0, kH * kH * 4, s->st))) return e;
  if ((e = cudaMemsetAsync(s->gB, 0, 260 * 4, s->st))) return e;
  k_sur_loss<<<(B + 255) / 256, 256, 0, s->st>>>(B, s->Yo, s->P + kPB3, s->Tn, s->dYb, s->dYT,
                                                 s->gB + 256, loss_slot);
  // dH2 = dY W3
  if ((e = gemm(gargs(s->dYb, 16, s->W3T, 16, s->dH2, kH, nullptr, 0, nullptr, B, 16, s->errw), B,
                128, 1, 0, s->st)))
    return e;
  k_sur_silu_back<<<256, 256, 0, s->st>>>(B, s->dH2, s->Z2, s->dZ2, s->gB + 128);
  const dim3 tb(32, 8);
  k_transpose16<<<dim3(kH / 32, B / 32), tb, 0, s->st>>>(s->H1, s->H1T, B, kH);
  k_transpose16<<<dim3(kH / 32, B / 32), tb, 0, s->st>>>(s->H2, s->H2T, B, kH);
  k_transpose16<<<dim3(kH / 32, B / 32), tb, 0, s->st>>>(s->dZ2, s->dZ2T, B, kH);
  // dW2 = dZ2^T H1, dW3 = dY^T H2 (rows 4.. of dYT are zero)
  if ((e = gemm(gargs(s->dZ2T, B, s->H1T, B, s->gW2, kH, nullptr, 0, nullptr, kH, B, s->errw), kH,
                128, splits, 1, s->st)))
    return e;
  if ((e = gemm(gargs(s->dYT, B, s->H2T, B, s->gW3, kH, nullptr, 0, nullptr, kH, B, s->errw), kH,
                128, splits, 1, s->st)))
    return e;
  // dH1 = dZ2 W2
  if ((e = gemm(gargs(s->dZ2, kH, s->W2T, kH, s->dH1, kH, nullptr, 0, nullptr, B, kH, s->errw), B,
                128, 1, 0, s->st)))
    return e;
  k_sur_silu_back<<<256, 256, 0, s->st>>>(B, s->dH1, s->Z1, s->dZ1, s->gB);
  k_transpose16<<<dim3(kH / 32, B / 32), tb, 0, s->st>>>(s->dZ1, s->dZ1T, B, kH);
  // dW1 = dZ1^T X
  if ((e = gemm(gargs(s->dZ1T, B, s->XT, B, s->gW1, 16, nullptr, 0, nullptr, kH, B, s->errw), kH,
                16, splits, 1, s->st)))
    return e;
  double c1 = 1.0, c2 = 1.0;
  if (!G) {
    s->t += 1;
    c1 = 1.0 - std::pow(0.9, (double)s->t);
    c2 = 1.0 - std::pow(0.999, (double)s->t);
  }
  k_sur_adam<<<(NS_SUR_PARAMS + 255) / 256, 256, 0, s->st>>>(
      s->P, s->Am, s->Av, s->gW1, s->gW2, s->gW3, s->gB, lr, (float)c1, (float)c2, s->W1p, s->W2b,
      s->W2T, s->W3p, s->W3T, G);
  return cudaGetLastError();
}

ns_status check_err(ns_sur* s) {
  uint32_t e = 0;
  SCK(cudaMemcpyAsync(&e, s->errw, 4, cudaMemcpyDeviceToHost, s->st));
  SCK(cudaStreamSynchronize(s->st));
  if (e) return sfail(s, NS_ERR_DEVICE_TIMEOUT, "a tensor-core wait gave up (mbarrier phase)");
  return NS_OK;
}

ns_status ensure_scratch(ns_sur* s) {
  if (s->Xs) return NS_OK;
  SCK(salloc(s, &s->Xs, (size_t)s->B * 5));
  SCK(salloc(s, &s->Ys, (size_t)s->B * 4));
  return NS_OK;
}

}  // namespace

extern "C" {

const char* ns_sur_last_error(const ns_sur* s) { return s ? s->err.c_str() : g_sur_err.c_str(); }

ns_status ns_sur_create(int device, const float hh_params[7], float dt_fine_ms, uint32_t batch,
                        uint64_t seed, ns_sur** out) {
  ns_sur* s = nullptr;
  if (!out || !hh_params) return sfail(s, NS_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (batch == 0 || batch % 128 != 0 || batch > (1u << 20))
    return sfail(s, NS_ERR_INVALID_ARG, "batch must be a positive multiple of 128 (<= 2^20)");
  if (!(dt_fine_ms > 0.0f)) return sfail(s, NS_ERR_INVALID_ARG, "dt must be positive");
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) {
    cudaGetLastError();
    return sfail(s, NS_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  if (device < 0 || device >= nd) return sfail(s, NS_ERR_INVALID_ARG, "device out of range");
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10)
    return sfail(s, NS_ERR_UNSUPPORTED, "the surrogate kernels need an sm_100 device");
  s = new ns_sur();
  s->dev = device;
  std::memcpy(s->hh.p, hh_params, sizeof(s->hh.p));
  s->dt = dt_fine_ms;
  s->B = batch;
  s->seed = seed;
  s->sample_seed = seed;
  for (int k = 0; k < 5; ++k) { s->norm.in_mean[k] = 0.f; s->norm.in_scale[k] = 1.f; }
  for (int k = 0; k < 4; ++k) { s->norm.out_mean[k] = 0.f; s->norm.out_scale[k] = 1.f; }
  auto bad = [&](cudaError_t e) {
    ns_status r = sfail(nullptr, e == cudaErrorMemoryAllocation ? NS_ERR_OOM : NS_ERR_CUDA,
                        cudaGetErrorString(e));
    ns_sur_destroy(s);
    return r;
  };
  cudaError_t e;
  if ((e = cudaSetDevice(device))) return bad(e);
  if ((e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking))) return bad(e);
  const size_t B = batch;
  if ((e = salloc(s, &s->P, NS_SUR_PARAMS)) || (e = salloc(s, &s->Am, NS_SUR_PARAMS)) ||
      (e = salloc(s, &s->Av, NS_SUR_PARAMS)) || (e = salloc(s, &s->W1p, 128 * 16)) ||
      (e = salloc(s, &s->W2b, kH * kH)) || (e = salloc(s, &s->W2T, kH * kH)) ||
      (e = salloc(s, &s->W3p, 16 * kH)) || (e = salloc(s, &s->W3T, kH * 16)) ||
      (e = salloc(s, &s->Xp, B * 16)) || (e = salloc(s, &s->XT, 16 * B)) ||
      (e = salloc(s, &s->H1, B * kH)) || (e = salloc(s, &s->H2, B * kH)) ||
      (e = salloc(s, &s->dYb, B * 16)) || (e = salloc(s, &s->dYT, (size_t)kH * B)) ||
      (e = salloc(s, &s->dZ2, B * kH)) || (e = salloc(s, &s->dZ2T, B * kH)) ||
      (e = salloc(s, &s->dZ1, B * kH)) || (e = salloc(s, &s->dZ1T, B * kH)) ||
      (e = salloc(s, &s->H1T, B * kH)) || (e = salloc(s, &s->H2T, B * kH)) ||
      (e = salloc(s, &s->Z1, B * kH)) || (e = salloc(s, &s->Z2, B * kH)) ||
      (e = salloc(s, &s->Yo, B * 16)) || (e = salloc(s, &s->Tn, B * 4)) ||
      (e = salloc(s, &s->dH2, B * kH)) || (e = salloc(s, &s->dH1, B * kH)) ||
      (e = salloc(s, &s->gW1, 128 * 16)) || (e = salloc(s, &s->gW2, kH * kH)) ||
      (e = salloc(s, &s->gW3, kH * kH)) || (e = salloc(s, &s->gB, 260)) ||
      (e = salloc(s, &s->G, NS_SUR_PARAMS)) || (e = salloc(s, &s->errw, 1)))
    return bad(e);
  // initialisation U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases
  std::vector<float> p(NS_SUR_PARAMS);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int cnt, int fan_in) {
    std::uniform_real_distribution<float> u(-1.0f / std::sqrt((float)fan_in), 1.0f / std::sqrt((float)fan_in));
    for (int q = 0; q < cnt; ++q) p[off + q] = u(rng);
  };
  fill(kPW1, 640, 5); fill(kPB1, 128, 5);
  fill(kPW2, kH * kH, kH); fill(kPB2, 128, kH);
  fill(kPW3, 4 * kH, kH); fill(kPB3, 4, kH);
  *out = s;
  ns_status r = ns_sur_set_params(s, p.data());
  if (r != NS_OK) { *out = nullptr; ns_sur_destroy(s); return r; }
  return NS_OK;
}

ns_status ns_sur_destroy(ns_sur* s) {
  if (!s) return NS_ERR_NULL_HANDLE;
  cudaSetDevice(s->dev);
  if (s->st) cudaStreamSynchronize(s->st);
  for (void* q : s->allocs) cudaFree(q);
  if (s->st) cudaStreamDestroy(s->st);
  delete s;
  return NS_OK;
}

ns_status ns_sur_set_params(ns_sur* s, const float* params) {
  if (!s) return NS_ERR_NULL_HANDLE;
  if (!params) return sfail(s, NS_ERR_INVALID_ARG, "null params");
  for (int q = 0; q < NS_SUR_PARAMS; ++q)
    if (!std::isfinite(params[q])) return sfail(s, NS_ERR_NONFINITE, "non-finite parameter");
  SCK(cudaSetDevice(s->dev));
  SCK(cudaMemcpyAsync(s->P, params, NS_SUR_PARAMS * 4, cudaMemcpyHostToDevice, s->st));
  SCK(cudaMemsetAsync(s->Am, 0, NS_SUR_PARAMS * 4, s->st));
  SCK(cudaMemsetAsync(s->Av, 0, NS_SUR_PARAMS * 4, s->st));
  k_sur_refresh<<<(NS_SUR_PARAMS + 255) / 256, 256, 0, s->st>>>(s->P, s->W1p, s->W2b, s->W2T, s->W3p, s->W3T);
  SCK(cudaGetLastError());
  SCK(cudaStreamSynchronize(s->st));
  s->t = 0;
  return NS_OK;
}

ns_status ns_sur_get_params(ns_sur* s, float* params) {
  if (!s) return NS_ERR_NULL_HANDLE;
  if (!params) return sfail(s, NS_ERR_INVALID_ARG, "null params");
  SCK(cudaSetDevice(s->dev));
  SCK(cudaMemcpyAsync(params, s->P, NS_SUR_PARAMS * 4, cudaMemcpyDeviceToHost, s->st));
  SCK(cudaStreamSynchronize(s->st));
  return NS_OK;
}

ns_status ns_sur_set_norm(ns_sur* s, const float in_mean[5], const float in_scale[5],
                          const float out_mean[4], const float out_scale[4]) {
  if (!s) return NS_ERR_NULL_HANDLE;
  if (!in_mean || !in_scale || !out_mean || !out_scale) return sfail(s, NS_ERR_INVALID_ARG, "null norm");
  for (int k = 0; k < 5; ++k)
    if (!(in_scale[k] > 0.0f) || !std::isfinite(in_mean[k])) return sfail(s, NS_ERR_INVALID_ARG, "bad input norm");
  for (int k = 0; k < 4; ++k)
    if (!(out_scale[k] > 0.0f) || !std::isfinite(out_mean[k])) return sfail(s, NS_ERR_INVALID_ARG, "bad output norm");
  std::memcpy(s->norm.in_mean, in_mean, 20);
  std::memcpy(s->norm.in_scale, in_scale, 20);
  std::memcpy(s->norm.out_mean, out_mean, 16);
  std::memcpy(s->norm.out_scale, out_scale, 16);
  return NS_OK;
}

ns_status ns_sur_set_data(ns_sur* s, const float* x, uint64_t n, float* y_out) {
  if (!s) return NS_ERR_NULL_HANDLE;
  if (!x || n == 0) return sfail(s, NS_ERR_INVALID_ARG, "empty training set");
  for (uint64_t q = 0; q < n * 5; ++q)
    if (!std::isfinite(x[q])) return sfail(s, NS_ERR_NONFINITE, "non-finite training state");
  SCK(cudaSetDevice(s->dev));
  SCK(cudaStreamSynchronize(s->st));
  if (n != s->n_data) {
    if (s->X) { cudaFree(s->X); cudaFree(s->Y); }
    s->X = s->Y = nullptr;
    s->n_data = 0;
    SCK(cudaMalloc(&s->X, n * 5 * 4));
    cudaError_t e = cudaMalloc(&s->Y, n * 4 * 4);
    if (e != cudaSuccess) { cudaFree(s->X); s->X = nullptr; SCK(e); }
    s->n_data = n;
  }
  SCK(cudaMemcpyAsync(s->X, x, n * 5 * 4, cudaMemcpyHostToDevice, s->st));
  k_sur_targets<<<1184, 128, 0, s->st>>>(s->X, s->Y, n, s->hh, s->dt);
  SCK(cudaGetLastError());
  if (y_out) SCK(cudaMemcpyAsync(y_out, s->Y, n * 4 * 4, cudaMemcpyDeviceToHost, s->st));
  SCK(cudaStreamSynchronize(s->st));
  return NS_OK;
}

ns_status ns_sur_train(ns_sur* s, uint32_t n_steps, float lr, float lr_decay, float* loss_out) {
  if (!s) return NS_ERR_NULL_HANDLE;
  if (!s->X) return sfail(s, NS_ERR_STATE, "no training set");
  if (!(lr > 0.0f) || !(lr_decay > 0.0f)) return sfail(s, NS_ERR_INVALID_ARG, "lr and lr_decay must be positive");
  SCK(cudaSetDevice(s->dev));
  if (n_steps > s->loss_cap) {
    if (s->lossv) cudaFree(s->lossv);
    s->lossv = nullptr;
    s->loss_cap = 0;
    SCK(cudaMalloc(&s->lossv, (size_t)n_steps * 4));
    s->loss_cap = n_steps;
  }
  SCK(cudaMemsetAsync(s->lossv, 0, (size_t)std::max<uint32_t>(n_steps, 1) * 4, s->st));
  SCK(cudaMemsetAsync(s->errw, 0, 4, s->st));
  float l = lr;
  for (uint32_t q = 0; q < n_steps; ++q) {
    k_sur_gather<<<(s->B + 255) / 256, 256, 0, s->st>>>(s->B, s->X, s->Y, s->n_data, 1,
                                                        s->sample_seed, s->t, 0, 0, s->norm, s->hh,
                                                        s->dt * NS_SUR_SUBSTEPS, s->Xp, s->XT, s->Tn);
    SCK(forward(s));
    SCK(backward_update(s, s->lossv + q, l, nullptr));
    l *= lr_decay;
  }
  if (loss_out && n_steps)
    SCK(cudaMemcpyAsync(loss_out, s->lossv, (size_t)n_steps * 4, cudaMemcpyDeviceToHost, s->st));
  SCK(cudaStreamSynchronize(s->st));
  return check_err(s);
}

ns_status ns_sur_set_sample_seed(ns_sur* s, uint64_t seed) {
  if (!s) return NS_ERR_NULL_HANDLE;
  s->sample_seed = seed;
  return NS_OK;
}

ns_status ns_sur_grad_step(ns_sur* s, float* grad_dev, float* loss_out) {
  if (!s) return NS_ERR_NULL_HANDLE;
  if (!s->X) return sfail(s, NS_ERR_STATE, "no training set");
  if (!grad_dev) return sfail(s, NS_ERR_INVALID_ARG, "null gradient buffer");
  SCK(cudaSetDevice(s->dev));
  if (s->loss_cap < 1) {
    SCK(cudaMalloc(&s->lossv, 4));
    s->loss_cap = 1;
  }
  SCK(cudaMemsetAsync(s->lossv, 0, 4, s->st));
  SCK(cudaMemsetAsync(s->errw, 0, 4, s->st));
  k_sur_gather<<<(s->B + 255) / 256, 256, 0, s->st>>>(s->B, s->X, s->Y, s->n_data, 1, s->sample_seed,
                                                      s->t, 0, 0, s->norm, s->hh, s->dt * NS_SUR_SUBSTEPS, s->Xp, s->XT, s->Tn);
  SCK(forward(s));
  SCK(backward_update(s, s->lossv, 0.0f, grad_dev));
  float l = 0.0f;
  SCK(cudaMemcpyAsync(&l, s->lossv, 4, cudaMemcpyDeviceToHost, s->st));
  SCK(cudaStreamSynchronize(s->st));
  if (loss_out) *loss_out = l;
  return check_err(s);
}

ns_status ns_sur_apply_gradient(ns_sur* s, const float* grad_dev, float scale, float lr) {
  if (!s) return NS_ERR_NULL_HANDLE;
  if (!grad_dev) return sfail(s, NS_ERR_INVALID_ARG, "null gradient buffer");
  if (!(lr > 0.0f) || !std::isfinite(scale)) return sfail(s, NS_ERR_INVALID_ARG, "lr > 0 and a finite scale");
  SCK(cudaSetDevice(s->dev));
  s->t += 1;
  const double c1 = 1.0 - std::pow(0.9, (double)s->t), c2 = 1.0 - std::pow(0.999, (double)s->t);
  k_sur_adam_flat<<<(NS_SUR_PARAMS + 255) / 256, 256, 0, s->st>>>(
      s->P, s->Am, s->Av, grad_dev, scale, lr, (float)c1, (float)c2, s->W1p, s->W2b, s->W2T, s->W3p, s->W3T);
  SCK(cudaGetLastError());
  SCK(cudaStreamSynchronize(s->st));
  return NS_OK;
}

ns_status ns_sur_gradient(ns_sur* s, const float* x, const float* y, float* grad_out, float* loss_out) {
  if (!s) return NS_ERR_NULL_HANDLE;
  if (!x || !y || !grad_out) return sfail(s, NS_ERR_INVALID_ARG, "null argument");
  SCK(cudaSetDevice(s->dev));
  ns_status r = ensure_scratch(s);
  if (r) return r;
  SCK(cudaMemcpyAsync(s->Xs, x, (size_t)s->B * 20, cudaMemcpyHostToDevice, s->st));
  SCK(cudaMemcpyAsync(s->Ys, y, (size_t)s->B * 16, cudaMemcpyHostToDevice, s->st));
  SCK(cudaMemsetAsync(s->errw, 0, 4, s->st));
  SCK(cudaMemsetAsync(s->G, 0, NS_SUR_PARAMS * 4, s->st));
  float* lslot = nullptr;
  SCK(cudaMalloc(&lslot, 4));
  cudaMemsetAsync(lslot, 0, 4, s->st);
  k_sur_gather<<<(s->B + 255) / 256, 256, 0, s->st>>>(s->B, s->Xs, s->Ys, s->B, 0, 0, 0, 0, s->B,
                                                      s->norm, s->hh, s->dt * NS_SUR_SUBSTEPS, s->Xp, s->XT, s->Tn);
  cudaError_t e = forward(s);
  if (e == cudaSuccess) e = backward_update(s, lslot, 0.0f, s->G);
  float lh = 0.0f;
  if (e == cudaSuccess) e = cudaMemcpyAsync(grad_out, s->G, NS_SUR_PARAMS * 4, cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&lh, lslot, 4, cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  cudaFree(lslot);
  SCK(e);
  if (loss_out) *loss_out = lh;
  return check_err(s);
}

ns_status ns_sur_predict(ns_sur* s, const float* x, uint64_t n, float* y) {
  if (!s) return NS_ERR_NULL_HANDLE;
  if (!x || !y) return sfail(s, NS_ERR_INVALID_ARG, "null argument");
  if (n == 0) return NS_OK;
  SCK(cudaSetDevice(s->dev));
  SCK(cudaMemsetAsync(s->errw, 0, 4, s->st));
  float *xd = nullptr, *yd = nullptr;
  SCK(cudaMalloc(&xd, n * 20));
  cudaError_t e = cudaMalloc(&yd, n * 16);
  if (e == cudaSuccess) e = cudaMemcpyAsync(xd, x, n * 20, cudaMemcpyHostToDevice, s->st);
  for (uint64_t f = 0; f < n && e == cudaSuccess; f += s->B) {
    k_sur_gather<<<(s->B + 255) / 256, 256, 0, s->st>>>(s->B, xd, nullptr, n, 0, 0, 0, f, n, s->norm,
                                                        s->hh, s->dt * NS_SUR_SUBSTEPS, s->Xp, s->XT, nullptr);
    e = forward(s);
    if (e == cudaSuccess) {
      k_sur_decode<<<(s->B + 255) / 256, 256, 0, s->st>>>(s->B, f, n, xd, s->Yo, s->P + kPB3, s->norm,
                                                           s->hh, s->dt * NS_SUR_SUBSTEPS, yd);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(y, yd, n * 16, cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  cudaFree(xd);
  if (yd) cudaFree(yd);
  SCK(e);
  return check_err(s);
}

ns_status ns_tc_gemm_bf16(const uint16_t* A, const uint16_t* B, float* C, uint16_t* H,
                          const float* bias, uint32_t M, uint32_t N, uint32_t K, uint32_t lda,
                          uint32_t ldb, uint32_t ldc, uint32_t k_splits, int32_t epilogue,
                          void* stream) {
  ns_sur* s = nullptr;
  if (!A || !B) return sfail(s, NS_ERR_INVALID_ARG, "null operand");
  if (M == 0 || M % 128 != 0) return sfail(s, NS_ERR_INVALID_ARG, "M must be a positive multiple of 128");
  if (N != 16 && N != 128) return sfail(s, NS_ERR_INVALID_ARG, "N must be 16 or 128");
  if (K == 0 || K % 16 != 0) return sfail(s, NS_ERR_INVALID_ARG, "K must be a positive multiple of 16");
  if (lda % 8 || ldb % 8 || lda < K || ldb < K) return sfail(s, NS_ERR_INVALID_ARG, "lda/ldb: multiples of 8, >= K");
  if (((uintptr_t)A | (uintptr_t)B) & 15u) return sfail(s, NS_ERR_INVALID_ARG, "operands must be 16-byte aligned");
  if (epilogue < 0 || epilogue > 2) return sfail(s, NS_ERR_INVALID_ARG, "unknown epilogue");
  if (epilogue != 2 && (!C || ldc < N)) return sfail(s, NS_ERR_INVALID_ARG, "C / ldc");
  if (epilogue == 2 && (!H || (C && ldc < N))) return sfail(s, NS_ERR_INVALID_ARG, "H / ldc");
  if (epilogue == 2 && ((uintptr_t)H & 15u)) return sfail(s, NS_ERR_INVALID_ARG, "H must be 16-byte aligned");
  if (k_splits == 0 || (epilogue != 1 && k_splits != 1) || k_splits > K / 16)
    return sfail(s, NS_ERR_INVALID_ARG, "k_splits: 1, or up to K/16 with the atomic epilogue");
  static uint32_t* errw = nullptr;
  if (!errw && cudaMalloc(&errw, 4) != cudaSuccess) return sfail(s, NS_ERR_CUDA, "scratch");
  cudaStream_t st = (cudaStream_t)stream;
  ns::gemm::Args a = gargs(A, lda, B, ldb, C, ldc, H, N, bias, M, K, errw);
  cudaError_t e = gemm(a, M, N, k_splits, epilogue, st);
  if (e != cudaSuccess) return sfail(s, NS_ERR_CUDA, cudaGetErrorString(e));
  return NS_OK;
}

}  // extern "C"

ns_status ns_sur_view_of(const ns_sur* s, ns_sur_view* out) {
  if (!s || !out) return NS_ERR_NULL_HANDLE;
  out->dev = s->dev;
  out->dt = s->dt;
  std::memcpy(out->hh, s->hh.p, sizeof(out->hh));
  out->W1p = s->W1p;
  out->W2b = s->W2b;
  out->W3p = s->W3p;
  out->P = s->P;
  std::memcpy(out->in_mean, s->norm.in_mean, 20);
  std::memcpy(out->in_scale, s->norm.in_scale, 20);
  std::memcpy(out->out_mean, s->norm.out_mean, 16);
  std::memcpy(out->out_scale, s->norm.out_scale, 16);
  return NS_OK;
}
