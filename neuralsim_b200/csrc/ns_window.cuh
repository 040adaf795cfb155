// Windowed stepping for networks whose synaptic delay is D >= 2 steps and
// that have no plasticity (configs of the LIF and Hodgkin-Huxley families).
// Input generated inside a window of W <= D steps is delivered D steps later,
// so within the window every neuron evolves independently:
//  1. k_window     — one thread per neuron runs W steps with its state in
//                    registers (the same per-neuron arithmetic as k_neuron),
//                    reading a delay slot only when its "has input" bit is
//                    set, and compacts each step's spikes into per-block
//                    segments of 256 neurons (warp ballots, ascending order);
//  2. k_window_rows — one warp per non-empty segment walks the spikers' CSR
//                    rows and delivers into slot (k + D) mod D, setting bits;
//  3. k_window_scan — per-step totals; k_window_finish — the ordered spike
//                    log, then counters and the FP64 clock.
#pragma once
#include "ns_kernels.cuh"

namespace ns {

constexpr int kWinThreads = 256;   // neurons per segment (one block)

// LIF and Izhikevich windows are throughput-bound on large batches: 64
// registers keep 4 blocks resident per SM. The HH window is bound by one
// long dependent chain per neuron; 3 blocks per SM hold a 100k-neuron
// network in one wave.
template <int MODEL>
__host__ __device__ constexpr int window_min_blocks() { return MODEL == 2 ? 3 : 4; }

// STIM: the window starts with the step that takes a pending host stimulus
// (a one-step window; the other windows carry no stimulus code).
template <int MODEL, int MODE, bool STIM>
__global__ void __launch_bounds__(kWinThreads, window_min_blocks<MODEL>()) k_window(NsDev d, uint32_t j0, uint32_t W) {
  __shared__ uint32_t s_wcnt[kWinThreads / 32];
  __shared__ Kick s_kick[32];
  __shared__ int s_nk;
  __shared__ unsigned long long s_spk;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr bool COND = (MODE == 3 || MODE == 4);
  constexpr int NT = COND ? 4 : 1;
  constexpr int NP = MODEL == 0 ? 5 : (MODEL == 1 ? 4 : 7);
  const uint64_t i = (uint64_t)blockIdx.x * kWinThreads + tid;   // < n_pad
  const uint32_t seg = blockIdx.x;
  const uint64_t k0 = d.ctl->step_base + j0;
  if (tid == 0) s_spk = 0ull;
  // state and parameters stay in registers for the whole window
  NState st;
  st.v = d.v[i];
  st.u = MODEL == 1 ? d.u[i] : 0.f;
  st.refr = MODEL == 0 ? d.refr[i] : 0;
  st.I = (MODE == 0 || MODE == 3) ? d.I[i] : 0.f;
  st.m = MODEL == 2 ? d.gm[i] : 0.f;
  st.h = MODEL == 2 ? d.gh[i] : 0.f;
  st.n = MODEL == 2 ? d.gn[i] : 0.f;
  float par[7];
#pragma unroll
  for (int q = 0; q < NP; ++q) par[q] = d.par[q][i];
  const int rs = MODEL == 0 ? d.refr_steps[i] : 0;
  float G[4] = {0.f, 0.f, 0.f, 0.f};
  if (COND) {
#pragma unroll
    for (int t = 0; t < 4; ++t) G[t] = d.G[t][i];
  }
  const uint8_t inh = d.drive_kind == 3 ? d.inh[i] : 0;
  uint64_t dseed;
  uint32_t dli;
  drive_key(d, i, dseed, dli);
  PoissonWords pw;
  float stim0 = 0.f;
  if (STIM && d.ctl->stim_at == k0 + 1) {
    stim0 = d.stim[i];
    if (stim0 != 0.0f) d.stim[i] = 0.f;
  }
  const uint64_t words = d.n_pad >> 5;
  unsigned long long my_spk = 0;
  uint32_t slot = (uint32_t)(k0 % d.D);   // advanced by one (mod D) per step
  uint32_t pref = 0;                       // lane l: input word of step (s & ~31) + l
  for (uint32_t s = 0; s < W; ++s, slot = (slot + 1u == d.D) ? 0u : slot + 1u) {
    const uint64_t k = k0 + s;
    int nk = 0;
    if (d.drive_kind == 1) {
      // reference-shaped global kicks (engine.rs:280-287): lane j computes kick j
      if (warp == 1) {
        U4 x = draw(d.seed, 0, k, kStreamKicks);
        int cnt = 0;
        if (unif(x.x) < d.kick_chance) {
          uint32_t span = d.kick_max - d.kick_min + 1u;
          cnt = (int)(d.kick_min + (uint32_t)(((unsigned long long)x.y * span) >> 32));
        }
        if (lane < cnt) {
          U4 z = draw(d.seed, 1u + (uint32_t)lane, k, kStreamKicks);
          unsigned long long r64 = (unsigned long long)z.x | ((unsigned long long)z.z << 32);
          s_kick[lane].target = (uint32_t)__umul64hi(r64, (unsigned long long)d.n);
          s_kick[lane].amt = unif(z.y) * d.kick_strength;
        }
        if (lane == 0) s_nk = cnt;
      }
      __syncthreads();
      nk = s_nk;
    }
    // delivered input: the warp's "has input" words of the window are final
    // before it starts (delay >= window), so lane l fetches (and clears) the
    // word of step s + l once per 32 steps, off the per-step chain
    if ((s & 31u) == 0) {
      pref = 0u;
      if (s + lane < W) {
        const uint32_t sl = (slot + lane) % d.D;
        uint32_t* wp = d.inbits + (uint64_t)sl * words + (i >> 5);
        pref = *wp;
        if (pref) *wp = 0u;
      }
    }
    const uint32_t word = __shfl_sync(0xffffffffu, pref, s & 31u);
    float S[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) S[t] = 0.f;
    if ((word >> lane) & 1u) {
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        if (COND && !((d.type_mask >> t) & 1u)) continue;   // absent type: row stays 0
        unsigned long long* ap = d.acc + ((uint64_t)t * d.D + slot) * d.n_pad + i;
        S[t] = from_fix((long long)*ap);
        *ap = 0ull;
      }
    }
    // drive
    float z = 0.f;
    U4 y{0u, 0u, 0u, 0u};
    if (d.drive_kind == 3) {
      float z0, z1;
      gauss_pair(draw(dseed, dli >> 1, k, kStreamDrive), z0, z1);
      z = (dli & 1u) ? z1 : z0;
    } else if (d.drive_kind == 1) {
      y = draw(dseed, dli, k, kStreamDrive);
    } else if (d.drive_kind != 0) {
      y.x = pw.at(dseed, dli, k);
    }
    float addI, kick, addg;
    drive_of(d, y, z, inh, addI, kick, addg);
    float stv = 0.f;
    if (STIM) {   // the host stimulus joins the window's first step
      stv = stim0;
      stim0 = 0.f;
    }
    const bool sp = update_one<MODEL, MODE>(d, k, i, st, par, rs, S, G, addI, kick, addg,
                                            s_kick, nk, stv) && (i < d.n);
    if (sp) { d.last[i] = (long long)k; ++my_spk; }
    // compaction of this step's spikes into the segment, ascending
    const unsigned m = __ballot_sync(0xffffffffu, sp);
    if (lane == 0) s_wcnt[warp] = __popc(m);
    __syncthreads();
    uint32_t off = 0, tot = 0;
#pragma unroll
    for (int q = 0; q < kWinThreads / 32; ++q) {
      const uint32_t c = s_wcnt[q];
      off += (q < warp) ? c : 0u;
      tot += c;
    }
    if (sp) d.seg_lst[(uint64_t)s * d.n_pad + (uint64_t)seg * kWinThreads + off +
                      __popc(m & ((1u << lane) - 1u))] = (uint32_t)i;
    if (tid == 0) d.seg_cnt[(uint64_t)s * d.nseg + seg] = tot;
    __syncthreads();
  }
  d.v[i] = st.v;
  if (MODEL == 1) d.u[i] = st.u;
  if (MODEL == 0) d.refr[i] = st.refr;
  if (MODE == 0 || MODE == 3 || MODE == 4) d.I[i] = st.I;
  if (MODEL == 2) { d.gm[i] = st.m; d.gh[i] = st.h; d.gn[i] = st.n; }
  if (COND) {
#pragma unroll
    for (int t = 0; t < 4; ++t) d.G[t][i] = G[t];
  }
  // spike and output-spike counters
  unsigned long long outs = (my_spk && d.outp[i]) ? my_spk : 0ull;
  for (int o = 16; o > 0; o >>= 1) {
    my_spk += __shfl_down_sync(0xffffffffu, my_spk, o);
    outs += __shfl_down_sync(0xffffffffu, outs, o);
  }
  if (lane == 0 && my_spk) atomicAdd(&s_spk, my_spk);
  if (lane == 0 && outs) atomicAdd(&d.ctl->out_total, outs);
  __syncthreads();
  if (tid == 0 && s_spk) atomicAdd(&d.ctl->spikes_total, s_spk);
}

// One warp per non-empty (step, segment): row walks into slot (k + D) mod D.
// LANES lanes walk one row (4 entries per lane per chunk of 4 LANES), so a
// warp has 32 / LANES of the segment's rows in flight: the walk's shape,
// chosen per network-size bucket by the window tuner. Integer atomics make
// the result independent of the shape.
template <bool COND, bool BF16, int LANES = 32>
__global__ void __launch_bounds__(256) k_window_rows(NsDev d, uint32_t j0, uint32_t W) {
  static_assert(LANES == 8 || LANES == 16 || LANES == 32, "8, 16 or 32 lanes per row");
  constexpr uint32_t kGroups = 32u / LANES;
  __shared__ unsigned long long s_ev;
  const int lane = threadIdx.x & 31;
  const uint32_t grp = (uint32_t)lane / LANES, glane = (uint32_t)lane % LANES;
  if (threadIdx.x == 0) s_ev = 0ull;
  __syncthreads();
  const uint64_t k0 = d.ctl->step_base + j0;
  const uint32_t wglob = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  const uint64_t words = d.n_pad >> 5;
  const uint32_t total = W * d.nseg;
  unsigned long long ev = 0ull;
  for (uint32_t g = wglob; g < total; g += nw) {
    const uint32_t c = __ldg(d.seg_cnt + g);
    if (c == 0) continue;
    const uint32_t s = g / d.nseg, seg = g - s * d.nseg;
    const uint64_t k = k0 + s;
    const uint32_t slot = (uint32_t)((k + d.D) % d.D);
    const uint32_t* lst = d.seg_lst + (uint64_t)s * d.n_pad + (uint64_t)seg * kWinThreads;
    for (uint32_t l = grp; l < c; l += kGroups) {
      const uint32_t j = __ldg(lst + l);
      const uint64_t beg = __ldg(d.row_ptr + j), end = __ldg(d.row_ptr + j + 1);
      const uint8_t rt = COND ? __ldg(d.row_type + j) : 0;
      if (glane == 0) ev += end - beg;
      const uint64_t rb = beg & ~3ull;
      for (uint64_t b = rb; b < end; b += 4u * LANES) {
        const uint64_t e0 = b + 4ull * glane;
        if (e0 >= end || e0 + 4 <= beg) continue;
        const uint4 c4 = __ldg(reinterpret_cast<const uint4*>(d.col + e0));
        float w[4];
        load_w4(d, BF16, e0, w);
        const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint64_t e = e0 + q;
          if (e < beg || e >= end) continue;
          int ty = 0;
          if (COND) ty = (rt == 255) ? (int)__ldg(d.type + e) : (int)rt;
          const float val = (COND && (ty == 1 || ty == 2)) ? fabsf(w[q]) : w[q];
          atomicAdd(d.acc + ((uint64_t)ty * d.D + slot) * d.n_pad + cc[q],
                    (unsigned long long)to_fix(val));
          atomicOr(d.inbits + (uint64_t)slot * words + (cc[q] >> 5), 1u << (cc[q] & 31));
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) ev += __shfl_down_sync(0xffffffffu, ev, o);
  if (lane == 0 && ev) atomicAdd(&s_ev, ev);
  __syncthreads();
  if (threadIdx.x == 0 && s_ev) atomicAdd(&d.ctl->events_total, s_ev);
}

// Per-step totals and segment offsets: block s scans the segment counts of
// step s.
__global__ void __launch_bounds__(256) k_window_scan(NsDev d, uint32_t W) {
  const uint32_t s = blockIdx.x;
  if (s >= W) return;
  const uint32_t tot = block_scan_u32(d.seg_cnt + (uint64_t)s * d.nseg,
                                      d.seg_off + (uint64_t)s * (d.nseg + 1), d.nseg);
  if (threadIdx.x == 0) d.step_total[s] = tot;
}

// Ordered spike log and bookkeeping of the window, one launch: block s
// copies step s's segments in order at its place in the log (after the
// window fitted as a whole); the last block to finish then updates the log
// counters, the last-step spike counts and the FP64 clock (dt added once
// per step, as the step path does).
__global__ void __launch_bounds__(256) k_window_finish(NsDev d, uint32_t j0, uint32_t W) {
  __shared__ int s_last;
  __shared__ unsigned int s_sum;
  const uint32_t s = blockIdx.x;
  Ctl* c = d.ctl;
  if (d.log_idx == nullptr && s < W) {
    // no log, so no scan ran: block s totals step s's segment counts
    if (threadIdx.x == 0) s_sum = 0u;
    __syncthreads();
    unsigned int t = 0u;
    const uint32_t* cnt = d.seg_cnt + (uint64_t)s * d.nseg;
#pragma unroll 8
    for (uint32_t seg = threadIdx.x; seg < d.nseg; seg += blockDim.x) t += cnt[seg];
    t = __reduce_add_sync(0xffffffffu, t);
    if ((threadIdx.x & 31) == 0 && t) atomicAdd(&s_sum, t);
    __syncthreads();
    if (threadIdx.x == 0) d.step_total[s] = s_sum;
  }
  if (s < W && d.log_idx != nullptr && !(c->status & kErrLogFull)) {
    unsigned long long all = 0, before = 0;
    for (uint32_t q = 0; q < W; ++q) {
      all += d.step_total[q];
      if (q < s) before += d.step_total[q];
    }
    if (c->log_steps + W <= d.log_steps_cap && c->log_size + all <= d.log_cap) {
      const unsigned long long base = c->log_size + before;
      const uint32_t* off = d.seg_off + (uint64_t)s * (d.nseg + 1);
      for (uint32_t seg = threadIdx.x; seg < d.nseg; seg += blockDim.x) {
        const uint32_t cnt = d.seg_cnt[(uint64_t)s * d.nseg + seg];
        const uint32_t* lst = d.seg_lst + (uint64_t)s * d.n_pad + (uint64_t)seg * kWinThreads;
        for (uint32_t l = 0; l < cnt; ++l) d.log_idx[base + off[seg] + l] = lst[l];
      }
      if (threadIdx.x == 0) d.log_off[c->log_steps + s + 1] = base + d.step_total[s];
    }
  }
  // every block has read the log counters before the last one moves them
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&c->win_done, 1u) == gridDim.x - 1 ? 1 : 0;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  c->win_done = 0u;
  const uint64_t k0 = c->step_base + j0;
  unsigned long long all = 0;
  for (uint32_t q = 0; q < W; ++q) {
    all += d.step_total[q];
    c->step_spikes[(k0 + q) & 3] = d.step_total[q];
    if (d.step_total[q] > c->max_step_spikes) c->max_step_spikes = d.step_total[q];
    c->sim_time += d.dt;
  }
  if (d.log_idx != nullptr && !(c->status & kErrLogFull)) {
    if (c->log_steps + W <= d.log_steps_cap && c->log_size + all <= d.log_cap) {
      if (c->log_steps == 0) c->log_first = k0;
      c->log_steps += W;
      c->log_size += all;
    } else {
      c->status |= kErrLogFull;
    }
  }
}

// After a state upload: rebuild the "has input" bits from the accumulators.
__global__ void k_rebuild_inbits(NsDev d, uint32_t ntypes) {
  const uint64_t words = d.n_pad >> 5;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < (uint64_t)d.D * d.n_pad;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t slot = q / d.n_pad, i = q - slot * d.n_pad;
    bool any = false;
    for (uint32_t t = 0; t < ntypes; ++t)
      any |= d.acc[((uint64_t)t * d.D + slot) * d.n_pad + i] != 0ull;
    const unsigned m = __ballot_sync(0xffffffffu, any);
    if ((threadIdx.x & 31) == 0) d.inbits[slot * words + (i >> 5)] = m;
  }
}

}  // namespace ns
