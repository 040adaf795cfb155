// Windowed Hodgkin-Huxley stepping with the learned macro-step (Rush-Larsen,
// per-target conductances recomputed each step, delay >= window).
//
// One block = one segment of 256 neurons = two 128-row tensor-core tiles.
// Per macro-step of kSub (10) steps:
//  1. every neuron gathers the macro-step's delivered synaptic input (the
//     per-step delay slots, read without clearing) and its drive events; an
//     increment arriving at step r of the macro-step enters the mean
//     conductance and the end conductance with its exact decay from r on, so
//     the held synaptic current I = sum_t mean(G_t over the macro-step)
//     (E_t - V) and the conductances at the end match the per-step updates
//     (the driving force is taken at the macro-step's start V);
//  2. the MLP 5 -> 128 -> 128 -> 4 runs on the tensor cores for all 256
//     rows: tcgen05.mma (M 128, BF16 operands in shared memory, FP32 in TMEM)
//     with bias + SiLU epilogues back into shared memory as the next A
//     operand; the output is the normalised increment of (V, m, h, n). In
//     the comparison mode (coarse) one Rush-Larsen step of the macro-step's
//     length with the held current takes the MLP's place;
//  3. a neuron keeps that result when V lay in [v_lo, v_hi], the new V does
//     too, the gates stay in [0, 1] and |V_new - V_trapezoid| <= tol
//     (trapezoidal rule with the held current); its conductances take their
//     end-of-macro-step values and its slot entries are cleared. Otherwise
//     the neuron is handed over, with its state at the macro-step's start,
//     to the fallback for the rest of the window (k_window_fb): neurons of a
//     window are independent (the delay is at least the window), so the
//     macro-step kernel never waits for a Rush-Larsen chain;
//  4. k_window_fb runs every handed-over neuron (one thread per neuron, in
//     neuron order) with the plain Rush-Larsen steps from its hand-over step, with the
//     per-step inputs and drive (the arithmetic of the step kernels); spikes
//     go into their segment's list by atomic counts, and k_window_sort puts
//     each (step, segment) list in ascending order for the window row walk.
// The MLP predicts the correction to one Rush-Larsen step of the whole
// macro-step (the base), which keeps its outputs small and smooth.
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
  float gdec10[4];         // d^kSub
  float wmean[kSub][4];    // increment arriving at step r: its share of the mean
                           // conductance, (sum_{q=0}^{kSub-1-r} d^q) / kSub
  float wend[kSub][4];     // and of the end conductance, d^(kSub-1-r)
  int coarse;              // 0: the MLP; 1: one Rush-Larsen step of dt_macro;
                           // 2: kSub Rush-Larsen steps with the held current
                           //    (the function the MLP is trained on)
  unsigned long long* counts;   // [0] macro-steps by the MLP, [1] by the fallback
  uint32_t* err;
  uint32_t* hstep;         // [n_pad] step of the window a neuron was handed to the fallback (W: none)
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
      pk[q / 2] = gemm::pack_bf16x2_rn(a, b);
    }
    *reinterpret_cast<uint4*>(H + tc::kmajor_offset(r, j, 128)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(H + tc::kmajor_offset(r, j + 8, 128)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  }
}

// The three layers for the block's two tiles; returns this thread's four
// normalised outputs (without b3). xn: the 5 normalised inputs; layer 1
// reads each as its BF16 value (column k) plus BF16 remainder (column 5 + k)
// against a duplicated weight column.
__device__ __forceinline__ void sur_mlp(uint8_t* smem, uint8_t* H, uint32_t tid, uint32_t row,
                                        uint32_t tbase, uint32_t t_row, const float* b1,
                                        const float* b2, uint64_t* mbar, uint32_t& nc, bool& ok,
                                        const float* xn, float* out4) {
  const uint32_t id128 = tc::idesc_bf16(128), id16 = tc::idesc_bf16(16);
  uint16_t col[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) col[q] = 0;
#pragma unroll
  for (int q = 0; q < 5; ++q) gemm::split_bf16(xn[q], col[q], col[5 + q]);
  uint32_t pk[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) pk[q] = (uint32_t)col[2 * q] | ((uint32_t)col[2 * q + 1] << 16);
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
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t tile = tid >> 7, row = tid & 127u;
  const uint64_t i = (uint64_t)blockIdx.x * kWinThreads + tid;   // < n_pad
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
  // the fallback places this segment's spikes by atomic counts
  for (uint32_t q = tid; q < W; q += 256u) d.seg_cnt[(uint64_t)q * d.nseg + blockIdx.x] = 0u;

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
  PoissonWords pw;
  unsigned long long n_mlp = 0;
  bool active = i < d.n;      // still advanced by the MLP in this window
  uint32_t hand = W;          // step (within the window) handed to the fallback

  const uint32_t slot0 = (uint32_t)(k0 % d.D);
  for (uint32_t ms = 0; ms < W; ms += kSub) {
    const bool full = (W - ms) >= (uint32_t)kSub;
    // block-uniform: leave once no neuron of the block is on the MLP
    if (!__syncthreads_or(active && full)) {
      if (active) { hand = ms; active = false; }
      break;
    }
    const uint64_t kf = k0 + ms;
    const uint32_t slotf = (slot0 + ms) % d.D;   // slot of step kf (ms < W <= D)
    // ---- 1. inputs of the macro-step (slots read, not cleared), each
    //         weighted by its arrival step ----
    float gmean[4] = {0.f, 0.f, 0.f, 0.f}, gend[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t inmask = 0;
    const float v0 = st.v;
    if (active) {
      const float mgf = 1.0f / (1.0f + (1.0f / 3.57f) * expf(-0.062f * v0));
#pragma unroll 1
      for (int s = 0; s < kSub; ++s) {
        const uint64_t k = kf + s;
        const uint32_t slot = (slotf + s) % d.D;
        const uint32_t word = d.inbits[(uint64_t)slot * words + (i >> 5)];
        if ((word >> lane) & 1u) {
          inmask |= 1u << s;
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            if (!((d.type_mask >> t) & 1u)) continue;   // absent type: no input
            float inc = from_fix((long long)d.acc[((uint64_t)t * d.D + slot) * d.n_pad + i]) * kSyn[t].gmax;
            if (kSyn[t].mg) inc = inc * mgf;
            gmean[t] += inc * sd.wmean[s][t];
            gend[t] += inc * sd.wend[s][t];
          }
        }
        if (d.drive_kind == 4 && pw.at(dseed, dli, k) < d.p_thr) {
          gmean[0] += d.drive_amp * sd.wmean[s][0];
          gend[0] += d.drive_amp * sd.wend[s][0];
        }
      }
    }
    float Gp[4], isyn = 0.f;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const float gd = G[t] * d.Gdec[t];
      Gp[t] = G[t] * sd.gdec10[t] + gend[t];           // conductance at the macro-step's end
      isyn = isyn + (gd * sd.gbar[t] + gmean[t]) * (kSyn[t].erev - v0);
    }
    // ---- 2. one coarse Rush-Larsen step of the macro-step's length (the
    //         base), corrected by the MLP on the tensor cores; or the
    //         comparison integrators ----
    float nv = st.v, nm = st.m, nh = st.h, nn = st.n;
    if (active && sd.coarse != 2) hh_rl_step(nv, nm, nh, nn, isyn, par, sd.dt_macro);
    if (!sd.coarse) {
      const float xin[5] = {st.v, st.m, st.h, st.n, isyn};
      float xn[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) xn[q] = active ? (xin[q] - sd.in_mean[q]) / sd.in_scale[q] : 0.f;
      float o[4];
      sur_mlp(smem, H, tid, row, tbase, t_row, s_b1, s_b2, &mbar, nc, ok, xn, o);
      nv += (o[0] + s_b3[0]) * sd.out_scale[0] + sd.out_mean[0];
      nm += (o[1] + s_b3[1]) * sd.out_scale[1] + sd.out_mean[1];
      nh += (o[2] + s_b3[2]) * sd.out_scale[2] + sd.out_mean[2];
      nn += (o[3] + s_b3[3]) * sd.out_scale[3] + sd.out_mean[3];
    } else if (active && sd.coarse == 2) {
#pragma unroll 1
      for (int q = 0; q < kSub; ++q) hh_rl_step(nv, nm, nh, nn, isyn, par, d.dt_f);
    }
    if (!active) continue;
    // ---- 3. decision: keep the macro-step, or hand the neuron over to the
    //         fallback from this step on (state of the macro-step's start) ----
    const float f0 = (isyn - hh_iion(st.v, st.m, st.h, st.n, par)) / par[6];
    const float f1 = (isyn - hh_iion(nv, nm, nh, nn, par)) / par[6];
    const float vtrap = st.v + 0.5f * sd.dt_macro * (f0 + f1);
    const bool use = st.v >= sd.v_lo && st.v <= sd.v_hi && nv >= sd.v_lo && nv <= sd.v_hi &&
                     nm >= 0.f && nm <= 1.f && nh >= 0.f && nh <= 1.f && nn >= 0.f && nn <= 1.f &&
                     fabsf(nv - vtrap) <= sd.tol;
    if (use) {
      st.v = nv; st.m = nm; st.h = nh; st.n = nn; st.I = isyn;
#pragma unroll
      for (int t = 0; t < 4; ++t) G[t] = Gp[t];
      // the macro-step's input was consumed: clear this neuron's slot entries
      for (int s = 0; s < kSub; ++s) {
        if (!((inmask >> s) & 1u)) continue;
        const uint32_t slot = (slotf + s) % d.D;
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if ((d.type_mask >> t) & 1u) d.acc[((uint64_t)t * d.D + slot) * d.n_pad + i] = 0ull;
      }
      ++n_mlp;
    } else {
      hand = ms;
      active = false;
    }
  }
  // state at the window's end, or at the hand-over step for the fallback
  d.v[i] = st.v; d.gm[i] = st.m; d.gh[i] = st.h; d.gn[i] = st.n;
#pragma unroll
  for (int t = 0; t < 4; ++t) d.G[t][i] = G[t];
  d.I[i] = st.I;
  sd.hstep[i] = hand;
  for (int o2 = 16; o2 > 0; o2 >>= 1) n_mlp += __shfl_down_sync(0xffffffffu, n_mlp, o2);
  if (lane == 0 && n_mlp) atomicAdd(&sd.counts[0], n_mlp);
  if (!ok && lane == 0) atomicOr(sd.err, gemm::kErrWait);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tbase, 256);
}

// The fallback of a window: every neuron the macro-step kernel handed over
// continues from its hand-over step to the window's end with the plain
// Rush-Larsen steps (per-step input and drive, the arithmetic of the step
// kernels). One thread per neuron in neuron order: a warp none of whose
// neurons was handed over returns at once; otherwise its lanes step
// together from the warp's earliest hand-over step, each lane from its own,
// so the input words and accumulator rows a step reads are shared or
// coalesced across the warp. Chains are independent: no barrier; a spike
// takes its place in its segment's list of that step by an atomic count, and
// k_window_sort restores the ascending order.
__global__ void __launch_bounds__(256) k_window_fb(NsDev d, SurDev sd, uint32_t j0, uint32_t W) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t hj = j < d.n ? sd.hstep[j] : W;
  const bool mine = hj < W;
  if (__ballot_sync(0xffffffffu, mine) == 0u) return;   // whole warp: nothing handed over
  const uint32_t s0 = __reduce_min_sync(0xffffffffu, mine ? hj : W);
  unsigned long long my_spk = 0, my_out = 0, nfb = 0;
  const uint32_t seg = (uint32_t)(j / kWinThreads);
  const uint64_t k0 = d.ctl->step_base + j0;
  const uint64_t words = d.n_pad >> 5;
  const uint32_t slot0 = (uint32_t)(k0 % d.D);
  NState ws;
  ws.v = 0.f; ws.m = 0.f; ws.h = 0.f; ws.n = 0.f; ws.u = 0.f; ws.refr = 0; ws.I = 0.f;
  float wg[4] = {0.f, 0.f, 0.f, 0.f}, wp[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  uint64_t js = 0;
  uint32_t jl = 0;
  if (mine) {
    ws.v = d.v[j]; ws.m = d.gm[j]; ws.h = d.gh[j]; ws.n = d.gn[j]; ws.I = d.I[j];
#pragma unroll
    for (int t = 0; t < 4; ++t) wg[t] = d.G[t][j];
#pragma unroll
    for (int q = 0; q < 7; ++q) wp[q] = d.par[q][j];
    drive_key(d, j, js, jl);
  }
  PoissonWords wpw;
#pragma unroll 1
  for (uint32_t s = s0; s < W; ++s) {
    const bool on = mine && s >= hj;
    const uint64_t k = k0 + s;
    const uint32_t slot = (slot0 + s) % d.D;
    float S[4] = {0.f, 0.f, 0.f, 0.f};
    const uint32_t word = d.inbits[(uint64_t)slot * words + (j >> 5)];
    if (on && ((word >> (j & 31u)) & 1u)) {
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        if (!((d.type_mask >> t) & 1u)) continue;   // absent type: row stays 0
        unsigned long long* ap = d.acc + ((uint64_t)t * d.D + slot) * d.n_pad + j;
        S[t] = from_fix((long long)*ap);
        *ap = 0ull;
      }
    }
    if (!on) continue;
    U4 y{0u, 0u, 0u, 0u};
    if (d.drive_kind != 0) y.x = wpw.at(js, jl, k);
    float addI, kick, addg;
    drive_of(d, y, 0.f, 0, addI, kick, addg);
    if (update_one<2, 4>(d, k, j, ws, wp, 0, S, wg, addI, kick, addg, nullptr, 0)) {
      d.last[j] = (long long)k;
      const uint32_t p = atomicAdd(&d.seg_cnt[(uint64_t)s * d.nseg + seg], 1u);
      d.seg_lst[(uint64_t)s * d.n_pad + (uint64_t)seg * kWinThreads + p] = (uint32_t)j;
      ++my_spk;
      if (d.outp[j]) ++my_out;
    }
  }
  if (mine) {
    d.v[j] = ws.v; d.gm[j] = ws.m; d.gh[j] = ws.h; d.gn[j] = ws.n;
#pragma unroll
    for (int t = 0; t < 4; ++t) d.G[t][j] = wg[t];
    d.I[j] = ws.I;
    nfb = (W - hj + kSub - 1) / kSub;
  }
  for (int o2 = 16; o2 > 0; o2 >>= 1) {
    my_spk += __shfl_down_sync(0xffffffffu, my_spk, o2);
    my_out += __shfl_down_sync(0xffffffffu, my_out, o2);
    nfb += __shfl_down_sync(0xffffffffu, nfb, o2);
  }
  if (lane == 0 && my_spk) atomicAdd(&d.ctl->spikes_total, my_spk);
  if (lane == 0 && my_out) atomicAdd(&d.ctl->out_total, my_out);
  if (lane == 0 && nfb) atomicAdd(&sd.counts[1], nfb);
}

// One thread per (step, segment) of the window: sorts the segment's spike
// list of that step ascending (lists hold a few entries) and clears the
// segment's input bits of that step's slot.
__global__ void __launch_bounds__(256) k_window_sort(NsDev d, SurDev sd, uint32_t j0, uint32_t W) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (uint64_t)W * d.nseg) return;
  const uint32_t s = (uint32_t)(q / d.nseg), seg = (uint32_t)(q % d.nseg);
  const uint32_t cnt = d.seg_cnt[q];
  uint32_t* lst = d.seg_lst + (uint64_t)s * d.n_pad + (uint64_t)seg * kWinThreads;
  for (uint32_t a = 1; a < cnt; ++a) {
    const uint32_t x = lst[a];
    uint32_t b = a;
    while (b > 0 && lst[b - 1] > x) { lst[b] = lst[b - 1]; --b; }
    lst[b] = x;
  }
  const uint64_t k0 = d.ctl->step_base + j0;
  const uint32_t slot = (uint32_t)((k0 + s) % d.D);
  const uint64_t words = d.n_pad >> 5;
#pragma unroll
  for (uint32_t w = 0; w < kWinThreads / 32u; ++w)
    d.inbits[(uint64_t)slot * words + (uint64_t)seg * (kWinThreads / 32u) + w] = 0u;
}

}  // namespace ns
