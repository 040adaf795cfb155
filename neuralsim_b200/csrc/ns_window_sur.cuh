// Windowed Hodgkin-Huxley stepping with the learned macro-step (Rush-Larsen,
// per-target conductances recomputed each step, delay >= window).
//
// One block = one segment of 256 neurons = two 128-row tensor-core tiles.
// Per macro-step of kSub (10) steps:
//  1. every neuron gathers the macro-step's delivered synaptic input (the
//     per-step delay slots, read without clearing) and its drive events, and
//     forms G' = G d + sum of increments and the held synaptic current
//     I = sum_t mean(G_t over the macro-step) (E_t - V);
//  2. the MLP 5 -> 128 -> 128 -> 4 runs on the tensor cores for all 256
//     rows: tcgen05.mma (M 128, BF16 operands in shared memory, FP32 in TMEM)
//     with bias + SiLU epilogues back into shared memory as the next A
//     operand; the output is the normalised increment of (V, m, h, n). In
//     the comparison mode (coarse) one Rush-Larsen step of the macro-step's
//     length with the held current takes the MLP's place;
//  3. a neuron keeps that result when V lay in [v_lo, v_hi], the new V does
//     too, the gates stay in [0, 1] and |V_new - V_trapezoid| <= tol
//     (trapezoidal rule with the held current); its conductances end at
//     G' d^9 and its slot entries are cleared;
//  4. the other neurons are compacted (ascending) onto the first threads of
//     the block, which run the plain Rush-Larsen steps with the per-step
//     inputs (the arithmetic of the step kernels) and report spikes per step
//     into the segment lists the window row walk reads.
// Only the fallback can spike: a neuron whose V leaves the envelope upward
// is integrated by Rush-Larsen, which detects the 0 mV crossing. A window
// tail shorter than a macro-step is stepped by the fallback alone.
#pragma once
#include "ns_gemm.cuh"
#include "ns_tc.cuh"
#include "ns_window.cuh"

namespace ns {

constexpr int kSub = 10;                              // steps per macro-step
constexpr uint32_t kSurW1 = 0;                        // smem: W1 [128][16]
constexpr uint32_t kSurW2 = 128 * 16 * 2;             //       W2 [128][128]
constexpr uint32_t kSurW3 = kSurW2 + 128 * 128 * 2;   //       W3 [16][128]
constexpr uint32_t kSurH = kSurW3 + 16 * 128 * 2;     //       H tiles [2][128][128]
constexpr uint32_t kSurSmem = kSurH + 2 * 128 * 128 * 2;

struct SurDev {
  const uint16_t* W1p;
  const uint16_t* W2b;
  const uint16_t* W3p;
  const float* P;          // flat parameters: b1 at 640, b2 at 17152, b3 at 17792
  float in_mean[5], in_scale[5], out_mean[4], out_scale[4];
  float v_lo, v_hi, tol, dt_macro;
  float gbar[4];           // mean of d^s over s = 0..kSub-1, per synapse type
  float gdec9[4];          // d^(kSub - 1)
  int coarse;              // 1: one Rush-Larsen step of dt_macro instead of the MLP
  unsigned long long* counts;   // [0] macro-steps by the MLP, [1] by the fallback
  uint32_t* err;
};

__device__ __forceinline__ float hh_iion(float v, float m, float h, float n, const float* p) {
  const float n2 = n * n;
  return p[0] * (m * m * m) * h * (v - p[3]) + p[1] * (n2 * n2) * (v - p[4]) + p[2] * (v - p[5]);
}

// waits on the block's MMA barrier; a wait that gives up records the error
__device__ __forceinline__ void sur_wait(uint64_t* mbar, uint32_t& nc, bool& ok) {
  if (!tc::mbar_wait(mbar, nc & 1u, gemm::kWaitLimit)) ok = false;
  ++nc;
  tc::fence_after_sync();
}

// bias + SiLU of one 128-wide TMEM row into the canonical K-major layout of
// the next layer's A operand (row r of a 128 x 128 tile)
__device__ __forceinline__ void sur_hidden_epilogue(uint32_t taddr, const float* bias, uint8_t* H,
                                                    uint32_t r) {
#pragma unroll 1
  for (uint32_t j = 0; j < 128; j += 16) {
    float v[16];
    tc::tmem_ld16(taddr + j, v);
    uint32_t pk[8];
#pragma unroll
    for (int q = 0; q < 16; q += 2) {
      const float a = gemm::silu_t(v[q] + bias[j + q]);
      const float b = gemm::silu_t(v[q + 1] + bias[j + q + 1]);
      pk[q / 2] = (uint32_t)gemm::f32_to_bf16_rn(a) | ((uint32_t)gemm::f32_to_bf16_rn(b) << 16);
    }
    *reinterpret_cast<uint4*>(H + tc::kmajor_offset(r, j, 128)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(H + tc::kmajor_offset(r, j + 8, 128)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  }
}

// The three layers for the block's two tiles; returns this thread's four
// normalised outputs (without b3).
__device__ __forceinline__ void sur_mlp(uint8_t* smem, uint8_t* H, uint32_t tid, uint32_t row,
                                        uint32_t tbase, uint32_t t_row, const float* b1,
                                        const float* b2, uint64_t* mbar, uint32_t& nc, bool& ok,
                                        const float* xn, float* out4) {
  const uint32_t id128 = tc::idesc_bf16(128), id16 = tc::idesc_bf16(16);
  uint32_t pk[8];
#pragma unroll
  for (int q = 0; q < 8; ++q)
    pk[q] = (uint32_t)gemm::f32_to_bf16_rn(xn[2 * q]) | ((uint32_t)gemm::f32_to_bf16_rn(xn[2 * q + 1]) << 16);
  *reinterpret_cast<uint4*>(H + tc::kmajor_offset(row, 0, 16)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
  *reinterpret_cast<uint4*>(H + tc::kmajor_offset(row, 8, 16)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0) {   // layer 1: K = 16
    tc::fence_after_sync();
    const uint32_t w1 = tc::smem_u32(smem + kSurW1);
#pragma unroll
    for (uint32_t t = 0; t < 2; ++t) {
      const uint32_t a = tc::smem_u32(smem + kSurH + t * 32768u);
      tc::mma_bf16(tbase + t * 128u, tc::smem_desc(a, 128u, 256u), tc::smem_desc(w1, 128u, 256u), id128, 0u);
    }
    tc::commit(mbar);
  }
  sur_wait(mbar, nc, ok);
  sur_hidden_epilogue(t_row, b1, H, row);
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0) {   // layer 2: K = 128
    tc::fence_after_sync();
    const uint32_t w2 = tc::smem_u32(smem + kSurW2);
#pragma unroll
    for (uint32_t t = 0; t < 2; ++t) {
      const uint32_t a = tc::smem_u32(smem + kSurH + t * 32768u);
#pragma unroll
      for (uint32_t ks = 0; ks < 8; ++ks)
        tc::mma_bf16(tbase + t * 128u, tc::smem_desc(a + ks * 256u, 128u, 2048u),
                     tc::smem_desc(w2 + ks * 256u, 128u, 2048u), id128, ks > 0 ? 1u : 0u);
    }
    tc::commit(mbar);
  }
  sur_wait(mbar, nc, ok);
  sur_hidden_epilogue(t_row, b2, H, row);
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0) {   // layer 3: N = 16 (4 used)
    tc::fence_after_sync();
    const uint32_t w3 = tc::smem_u32(smem + kSurW3);
#pragma unroll
    for (uint32_t t = 0; t < 2; ++t) {
      const uint32_t a = tc::smem_u32(smem + kSurH + t * 32768u);
#pragma unroll
      for (uint32_t ks = 0; ks < 8; ++ks)
        tc::mma_bf16(tbase + t * 128u, tc::smem_desc(a + ks * 256u, 128u, 2048u),
                     tc::smem_desc(w3 + ks * 256u, 128u, 2048u), id16, ks > 0 ? 1u : 0u);
    }
    tc::commit(mbar);
  }
  sur_wait(mbar, nc, ok);
  float o[16];
  tc::tmem_ld16(t_row, o);
#pragma unroll
  for (int q = 0; q < 4; ++q) out4[q] = o[q];
}

__global__ void __launch_bounds__(256, 2) k_window_sur(NsDev d, SurDev sd, uint32_t j0, uint32_t W) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ float s_b1[128], s_b2[128], s_b3[4];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ uint32_t s_wcnt[8];
  __shared__ uint32_t s_list[256];
  __shared__ unsigned long long s_spk;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t tile = tid >> 7, row = tid & 127u;
  const uint64_t i = (uint64_t)blockIdx.x * kWinThreads + tid;   // < n_pad
  const uint32_t seg = blockIdx.x;
  const uint64_t k0 = d.ctl->step_base + j0;
  const uint64_t words = d.n_pad >> 5;
  uint8_t* const H = smem + kSurH + tile * (128u * 128u * 2u);

  // ---- weights into shared memory (canonical K-major layouts), biases ----
  for (uint32_t q = tid; q < 128u * 2u; q += 256u) {           // W1: 128 rows x 2 pieces
    const uint32_t r = q >> 1, c = q & 1u;
    tc::cp_async16(smem + kSurW1 + tc::kmajor_offset(r, c * 8, 16), sd.W1p + r * 16 + c * 8);
  }
  for (uint32_t q = tid; q < 128u * 16u; q += 256u) {          // W2: 128 rows x 16 pieces
    const uint32_t r = q >> 4, c = q & 15u;
    tc::cp_async16(smem + kSurW2 + tc::kmajor_offset(r, c * 8, 128), sd.W2b + r * 128 + c * 8);
  }
  for (uint32_t q = tid; q < 16u * 16u; q += 256u) {           // W3: 16 rows x 16 pieces
    const uint32_t r = q >> 4, c = q & 15u;
    tc::cp_async16(smem + kSurW3 + tc::kmajor_offset(r, c * 8, 128), sd.W3p + r * 128 + c * 8);
  }
  tc::cp_async_commit();
  if (tid < 128) { s_b1[tid] = sd.P[640 + tid]; s_b2[tid] = sd.P[17152 + tid]; }
  if (tid < 4) s_b3[tid] = sd.P[17792 + tid];
  if (warp == 0) tc::tmem_alloc(&tmem_base, 256);
  if (tid == 0) {
    tc::mbar_init(&mbar, 1);
    tc::fence_mbar_init();
    s_spk = 0ull;
  }
  tc::cp_async_wait_all();
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tmem_base;
  const uint32_t t_row = tbase + (((warp & 3u) * 32u) << 16) + tile * 128u;   // this thread's TMEM row
  uint32_t nc = 0;          // commits waited for
  bool ok = true;

  // ---- neuron state in registers ----
  NState st;
  st.v = d.v[i]; st.m = d.gm[i]; st.h = d.gh[i]; st.n = d.gn[i];
  st.u = 0.f; st.refr = 0; st.I = d.I[i];
  float par[7];
#pragma unroll
  for (int q = 0; q < 7; ++q) par[q] = d.par[q][i];
  float G[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) G[t] = d.G[t][i];
  uint64_t dseed;
  uint32_t dli;
  drive_key(d, i, dseed, dli);
  unsigned long long my_spk = 0, my_out = 0, n_mlp = 0, n_fb = 0;
  const bool real = i < d.n;
  float* const fv = reinterpret_cast<float*>(smem + kSurH);   // [9][256] exchange, inside H

  for (uint32_t ms = 0; ms < W; ms += kSub) {
    const uint64_t kf = k0 + ms;
    const int nsub = (W - ms) < (uint32_t)kSub ? (int)(W - ms) : kSub;
    const bool full = nsub == kSub;   // block-uniform
    bool use = false;
    if (full) {
      // ---- 1. inputs of the macro-step (slots read, not cleared) ----
      float sumS[4] = {0.f, 0.f, 0.f, 0.f};
      float addg = 0.f;
      uint32_t inmask = 0;
#pragma unroll 1
      for (int s = 0; s < kSub; ++s) {
        const uint64_t k = kf + s;
        const uint32_t slot = (uint32_t)(k % d.D);
        uint32_t word = 0;
        if (lane == 0) word = d.inbits[(uint64_t)slot * words + (i >> 5)];
        word = __shfl_sync(0xffffffffu, word, 0);
        if ((word >> lane) & 1u) {
          inmask |= 1u << s;
#pragma unroll
          for (int t = 0; t < 4; ++t)
            sumS[t] += from_fix((long long)d.acc[((uint64_t)t * d.D + slot) * d.n_pad + i]);
        }
        if (d.drive_kind == 4) {
          const U4 y = draw(dseed, dli, k, kStreamDrive);
          if (y.x < d.p_thr) addg += d.drive_amp;
        }
      }
      const float v0 = st.v;
      float Gp[4], isyn = 0.f;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        float inc = sumS[t] * kSyn[t].gmax;
        if (kSyn[t].mg) inc = inc * (1.0f / (1.0f + (1.0f / 3.57f) * expf(-0.062f * v0)));
        float g = G[t] * d.Gdec[t] + inc;
        if (t == 0) g = g + addg;
        Gp[t] = g;
        isyn = isyn + g * sd.gbar[t] * (kSyn[t].erev - v0);
      }
      // ---- 2. MLP on the tensor cores, or one coarse Rush-Larsen step ----
      float nv, nm, nh, nn;
      if (!sd.coarse) {
        const float xin[5] = {st.v, st.m, st.h, st.n, isyn};
        float xn[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) xn[q] = 0.f;
#pragma unroll
        for (int q = 0; q < 5; ++q) xn[q] = (xin[q] - sd.in_mean[q]) / sd.in_scale[q];
        float o[4];
        sur_mlp(smem, H, tid, row, tbase, t_row, s_b1, s_b2, &mbar, nc, ok, xn, o);
        nv = st.v + (o[0] + s_b3[0]) * sd.out_scale[0] + sd.out_mean[0];
        nm = st.m + (o[1] + s_b3[1]) * sd.out_scale[1] + sd.out_mean[1];
        nh = st.h + (o[2] + s_b3[2]) * sd.out_scale[2] + sd.out_mean[2];
        nn = st.n + (o[3] + s_b3[3]) * sd.out_scale[3] + sd.out_mean[3];
      } else {
        nv = st.v; nm = st.m; nh = st.h; nn = st.n;
        hh_rl_step(nv, nm, nh, nn, isyn, par, sd.dt_macro);
      }
      // ---- 3. decision ----
      const float f0 = (isyn - hh_iion(st.v, st.m, st.h, st.n, par)) / par[6];
      const float f1 = (isyn - hh_iion(nv, nm, nh, nn, par)) / par[6];
      const float vtrap = st.v + 0.5f * sd.dt_macro * (f0 + f1);
      use = real && st.v >= sd.v_lo && st.v <= sd.v_hi && nv >= sd.v_lo && nv <= sd.v_hi &&
            nm >= 0.f && nm <= 1.f && nh >= 0.f && nh <= 1.f && nn >= 0.f && nn <= 1.f &&
            fabsf(nv - vtrap) <= sd.tol;
      if (use) {
        st.v = nv; st.m = nm; st.h = nh; st.n = nn; st.I = isyn;
#pragma unroll
        for (int t = 0; t < 4; ++t) G[t] = Gp[t] * sd.gdec9[t];
        // the macro-step's input was consumed: clear this neuron's slot entries
        for (int s = 0; s < kSub; ++s) {
          if (!((inmask >> s) & 1u)) continue;
          const uint32_t slot = (uint32_t)((kf + s) % d.D);
#pragma unroll
          for (int t = 0; t < 4; ++t) d.acc[((uint64_t)t * d.D + slot) * d.n_pad + i] = 0ull;
        }
        ++n_mlp;
      }
    }
    // ---- 4. fallback: compact the other real neurons onto the first threads ----
    const bool fb = real && !use;
    const unsigned bm = __ballot_sync(0xffffffffu, fb);
    if (lane == 0) s_wcnt[warp] = __popc(bm);
    tc::fence_before_sync();
    __syncthreads();          // every TMEM load of this macro-step is done; H is free
    uint32_t off = 0, tot = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint32_t c = s_wcnt[q];
      off += (q < (int)warp) ? c : 0u;
      tot += c;
    }
    const uint32_t p = off + __popc(bm & ((1u << lane) - 1u));
    if (fb) {
      s_list[p] = tid;
      fv[0 * 256 + p] = st.v; fv[1 * 256 + p] = st.m; fv[2 * 256 + p] = st.h; fv[3 * 256 + p] = st.n;
#pragma unroll
      for (int t = 0; t < 4; ++t) fv[(4 + t) * 256 + p] = G[t];
      fv[8 * 256 + p] = st.I;
      if (full) ++n_fb;
    }
    __syncthreads();
    uint32_t fspk = 0;        // spike steps of the worker's neuron
    if (tid < tot) {
      const uint64_t j = (uint64_t)blockIdx.x * kWinThreads + s_list[tid];
      NState ws;
      ws.v = fv[tid]; ws.m = fv[256 + tid]; ws.h = fv[512 + tid]; ws.n = fv[768 + tid];
      ws.u = 0.f; ws.refr = 0; ws.I = fv[2048 + tid];
      float wg[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) wg[t] = fv[(4 + t) * 256 + tid];
      float wp[7];
#pragma unroll
      for (int q = 0; q < 7; ++q) wp[q] = d.par[q][j];
      uint64_t js;
      uint32_t jl;
      drive_key(d, j, js, jl);
#pragma unroll 1
      for (int s = 0; s < nsub; ++s) {
        const uint64_t k = kf + s;
        const uint32_t slot = (uint32_t)(k % d.D);
        float S[4] = {0.f, 0.f, 0.f, 0.f};
        const uint32_t word = d.inbits[(uint64_t)slot * words + (j >> 5)];
        if ((word >> (j & 31u)) & 1u) {
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            unsigned long long* ap = d.acc + ((uint64_t)t * d.D + slot) * d.n_pad + j;
            S[t] = from_fix((long long)*ap);
            *ap = 0ull;
          }
        }
        U4 y{0u, 0u, 0u, 0u};
        if (d.drive_kind != 0) y = draw(js, jl, k, kStreamDrive);
        float addI, kick, addgs;
        drive_of(d, y, 0.f, 0, addI, kick, addgs);
        const bool sp = update_one<2, 4>(d, k, j, ws, wp, 0, S, wg, addI, kick, addgs, nullptr, 0);
        if (sp) {
          fspk |= 1u << s;
          d.last[j] = (long long)k;
          if (d.outp[j]) ++my_out;
        }
      }
      fv[tid] = ws.v; fv[256 + tid] = ws.m; fv[512 + tid] = ws.h; fv[768 + tid] = ws.n;
#pragma unroll
      for (int t = 0; t < 4; ++t) fv[(4 + t) * 256 + tid] = wg[t];
      fv[2048 + tid] = ws.I;
    }
    // per-step compaction of the fallback spikes (workers are in ascending
    // neuron order)
#pragma unroll 1
    for (int s = 0; s < nsub; ++s) {
      const bool sp = (fspk >> s) & 1u;
      const unsigned m = __ballot_sync(0xffffffffu, sp);
      __syncthreads();
      if (lane == 0) s_wcnt[warp] = __popc(m);
      __syncthreads();
      uint32_t o2 = 0, t2 = 0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const uint32_t c = s_wcnt[q];
        o2 += (q < (int)warp) ? c : 0u;
        t2 += c;
      }
      const uint32_t sg = ms + (uint32_t)s;
      if (sp)
        d.seg_lst[(uint64_t)sg * d.n_pad + (uint64_t)seg * kWinThreads + o2 + __popc(m & ((1u << lane) - 1u))] =
            (uint32_t)((uint64_t)blockIdx.x * kWinThreads + s_list[tid]);
      if (tid == 0) d.seg_cnt[(uint64_t)sg * d.nseg + seg] = t2;
      my_spk += sp ? 1ull : 0ull;
    }
    __syncthreads();
    if (fb) {
      st.v = fv[p]; st.m = fv[256 + p]; st.h = fv[512 + p]; st.n = fv[768 + p];
#pragma unroll
      for (int t = 0; t < 4; ++t) G[t] = fv[(4 + t) * 256 + p];
      st.I = fv[2048 + p];
    }
    // the macro-step's slot words of this warp's neurons are consumed
    if (lane < (uint32_t)nsub) {
      const uint32_t slot = (uint32_t)((kf + lane) % d.D);
      d.inbits[(uint64_t)slot * words + (i >> 5)] = 0u;
    }
    __syncthreads();          // the exchange area becomes the next A operand
  }
  d.v[i] = st.v; d.gm[i] = st.m; d.gh[i] = st.h; d.gn[i] = st.n;
#pragma unroll
  for (int t = 0; t < 4; ++t) d.G[t][i] = G[t];
  d.I[i] = st.I;
  // counters (spikes and output spikes are counted by the worker threads)
  for (int o2 = 16; o2 > 0; o2 >>= 1) {
    my_spk += __shfl_down_sync(0xffffffffu, my_spk, o2);
    my_out += __shfl_down_sync(0xffffffffu, my_out, o2);
    n_mlp += __shfl_down_sync(0xffffffffu, n_mlp, o2);
    n_fb += __shfl_down_sync(0xffffffffu, n_fb, o2);
  }
  if (lane == 0 && my_spk) atomicAdd(&s_spk, my_spk);
  if (lane == 0 && my_out) atomicAdd(&d.ctl->out_total, my_out);
  if (lane == 0 && n_mlp) atomicAdd(&sd.counts[0], n_mlp);
  if (lane == 0 && n_fb) atomicAdd(&sd.counts[1], n_fb);
  if (!ok && lane == 0) atomicOr(sd.err, gemm::kErrWait);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (tid == 0 && s_spk) atomicAdd(&d.ctl->spikes_total, s_spk);
  if (warp == 0) tc::tmem_dealloc(tbase, 256);
}

}  // namespace ns
