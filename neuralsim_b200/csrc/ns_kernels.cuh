// Step kernels for one network (sm_100a).
//
// Per simulation step k two kernels run back to back (captured in a CUDA graph):
//  1. k_neuron   — fused drive + neuron update + STDP trace update + ordered
//                  warp-ballot spike compaction (decoupled look-back across
//                  tiles, tiles taken in ticket order), spike bitmap, counters.
//                  Replaces the rayon neuron loop + spike_buffer compaction of
//                  SimulationEngine::step (src/simulation/engine.rs:267-391)
//                  and the deferred phase-2 current/conductance update.
//  2. k_propagate — one warp per spiking row: coalesced 16-byte loads of the
//                  row's column indices and weights, int64 fixed-point
//                  atomicAdd into the target's delay slot, LTP fused into the
//                  same walk (engine.rs:414-473 + :496-537); then one warp per
//                  spiking target for LTD over its plastic incoming synapses.
// Optional third kernel k_homeostasis (engine.rs:569-606, FP64 rate sums).
#pragma once
#include <cstdint>
#include "ns_device.cuh"

namespace ns {

constexpr int kThreads = 256;              // neuron kernel block
constexpr int kTile = 1024;                // neurons per tile (2 pairs per thread)
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kSpinLimit = 1u << 22;  // bounded look-back wait

// device status bits (host maps them to ns_status)
constexpr uint32_t kErrLookback = 1u;
constexpr uint32_t kErrLogFull = 2u;

struct Ctl {
  unsigned long long step_base;   // global step of graph node 0
  unsigned int ticket[2];
  unsigned int status;
  unsigned int pad;
  unsigned long long spikes_total, out_total, events_total;
  unsigned long long step_spikes[4];
  double sim_time;
  unsigned long long log_size;    // indices held
  unsigned long long log_steps;   // steps held
  unsigned long long log_first;   // global step of the first logged step
};

struct Kick { uint32_t target; float amt; };

struct NsDev {
  uint64_t n, n_pad, m;
  uint32_t D, ntiles;
  float dt_f, decay_I;
  double dt;
  int stdp, drive_kind, hh_int, homeo;
  float a_plus, neg_a_minus, w_min, w_max, ep, em;
  uint32_t Kp, Km;
  float drive_p, drive_amp, sig_e, sig_i, kick_chance, kick_strength;
  uint32_t kick_min, kick_max, p_thr;
  uint64_t seed;
  float Gdec[4];
  float cd, one_m_cd;              // contribution EMA
  float h_target_unused;
  double h_target, h_tau;
  float h_tau_f;
  // neuron state (padded to n_pad)
  float *v, *u, *I, *gm, *gh, *gn;
  int32_t* refr;
  float* par[7];
  int32_t* refr_steps;
  uint8_t *inh, *outp;
  float *pre, *post, *qdec;
  long long* last;
  double* rate;
  float* G[4];
  // synapses
  const uint64_t* row_ptr;
  const uint32_t* col;
  float* w32;
  uint16_t* w16;
  const uint8_t* type;
  const uint8_t* plastic;
  const uint8_t* row_plastic;      // 0 none, 1 all, 2 mixed
  const uint8_t* row_type;         // type, or 255 mixed
  const uint64_t* in_ptr;          // plastic incoming (CSC)
  const uint2* in_list;            // (source, CSR position)
  const uint64_t* all_in_ptr;      // all incoming (homeostasis)
  const uint32_t* all_in_pos;
  float* contrib;
  unsigned long long* acc;         // [type][slot][n_pad]
  uint32_t* spk;                   // this step's ordered spike list
  uint32_t* bitmap;                // n_pad / 32 words
  unsigned long long* flags;       // look-back flags per tile
  Ctl* ctl;
  const float *Ep, *Em;
  uint32_t* log_idx;
  unsigned long long* log_off;
  unsigned long long log_cap;
  unsigned long long log_steps_cap;
  unsigned long long* trace_pos;   // traced step only
  const unsigned long long* trace_off;
  unsigned long long trace_cap;
};

__device__ __forceinline__ bool bit_of(const uint32_t* bm, uint32_t i) {
  return (bm[i >> 5] >> (i & 31)) & 1u;
}

__device__ __forceinline__ unsigned long long flag_pack(uint32_t tag, uint32_t st, uint32_t val) {
  return ((unsigned long long)tag << 34) | ((unsigned long long)st << 32) | val;
}

// ---------------------------------------------------------------------------
// One neuron, one step. Arithmetic order is the specification the float
// oracle mirrors: LifNeuron::step (src/neuron/lif.rs:15-61),
// IzhikevichNeuron::step (src/neuron/izhikevich.rs:20-52), HH
// (src/neuron/hodgkin_huxley.rs:20-96 for Euler; Rush-Larsen otherwise).
// ---------------------------------------------------------------------------
struct NState {
  float v, u, I, m, h, n, pre, post;
  int refr;
};

__device__ __forceinline__ void hh_rates(float v, float& am, float& bm, float& ah, float& bh,
                                         float& an, float& bn) {
  float x = (v + 40.0f) / 10.0f;
  am = (x == 0.0f) ? 1.0f : x / (-expm1f(-x));
  bm = 4.0f * expf(-(v + 65.0f) / 18.0f);
  ah = 0.07f * expf(-(v + 65.0f) / 20.0f);
  bh = 1.0f / (1.0f + expf(-(v + 35.0f) / 10.0f));
  float y = (v + 55.0f) / 10.0f;
  an = (y == 0.0f) ? 0.1f : (0.1f * y) / (-expm1f(-y));
  bn = 0.125f * expf(-(v + 65.0f) / 80.0f);
}

__device__ __forceinline__ U4 make_drive_draw(const NsDev& d, uint64_t i0, uint64_t k) {
  if (d.drive_kind == 3) return draw(d.seed, (uint32_t)(i0 >> 1), k, kStreamDrive);
  if (d.drive_kind == 0) return U4{0u, 0u, 0u, 0u};
  return draw(d.seed, (uint32_t)i0, k, kStreamDrive);
}

template <int MODEL>
__device__ __forceinline__ bool model_step(const NsDev& d, NState& s, const float* p, int rsteps,
                                           float Iin, float kick, bool delta) {
  const float dt = d.dt_f;
  if (MODEL == 0) {
    if (s.refr > 0) { s.refr -= 1; return false; }
    float t1 = s.v - p[0];
    float t2 = p[4] * Iin;            // input_resistance
    float t3 = (-t1) + t2;
    float t4 = t3 * dt;
    float dv = t4 / p[3];
    float v = s.v + dv;
    if (delta) v = v + kick;
    if (v >= p[1]) { s.v = p[2]; s.refr = rsteps; return true; }
    s.v = v;
    return false;
  } else if (MODEL == 1) {
    if (s.v >= 30.0f) { s.v = p[2]; s.u = s.u + p[3]; return true; }
    float v = s.v, u = s.u;
    float a1 = 0.04f * v;
    float a2 = a1 * v;
    float a3 = 5.0f * v;
    float sm = a2 + a3;
    sm = sm + 140.0f;
    sm = sm - u;
    sm = sm + Iin;
    float dv = sm * dt;
    float b1 = p[1] * v;
    float b2 = b1 - u;
    float b3 = p[0] * b2;
    float du = b3 * dt;
    v = v + dv;
    u = u + du;
    if (delta) v = v + kick;
    s.v = v; s.u = u;
    return false;
  } else {
    float gna = p[0], gk = p[1], gl = p[2], ena = p[3], ek = p[4], el = p[5], cm = p[6];
    float v = s.v, m = s.m, h = s.h, n = s.n;
    float am, bm, ah, bh, an, bn;
    hh_rates(v, am, bm, ah, bh, an, bn);
    bool spk;
    if (d.hh_int == 0) {
      m = m + (am * (1.0f - m) - bm * m) * dt;
      h = h + (ah * (1.0f - h) - bh * h) * dt;
      n = n + (an * (1.0f - n) - bn * n) * dt;
      float ina = gna * (m * m * m) * h * (ena - v);
      float n2 = n * n;
      float ik = gk * (n2 * n2) * (ek - v);
      float il = gl * (el - v);
      float dv = (Iin - ina - ik - il) / cm * dt;
      v = v + dv;
      spk = v >= -55.0f;
      if (spk) v = -70.0f;
    } else {
      float sm = am + bm, sh = ah + bh, sn = an + bn;
      float minf = am / sm, hinf = ah / sh, ninf = an / sn;
      m = minf + (m - minf) * expf(-dt * sm);
      h = hinf + (h - hinf) * expf(-dt * sh);
      n = ninf + (n - ninf) * expf(-dt * sn);
      float n2 = n * n;
      float iion = gna * (m * m * m) * h * (v - ena) + gk * (n2 * n2) * (v - ek) + gl * (v - el);
      float vn = v + dt * (Iin - iion) / cm;
      spk = (v < 0.0f) && (vn >= 0.0f);
      v = vn;
    }
    if (delta) v = v + kick;
    s.v = v; s.m = m; s.h = h; s.n = n;
    return spk;
  }
}

// ---------------------------------------------------------------------------
// Kernel 1: fused neuron update + trace update + ordered compaction.
// Thread t of tile T owns the neuron pairs (T*1024 + r*512 + 2t, +1), r = 0,1,
// so every state array is read with 8-byte coalesced loads and one Philox
// draw feeds the Gaussian drive of both neurons of a pair.
// ---------------------------------------------------------------------------
template <int MODEL, int MODE>
__global__ void __launch_bounds__(kThreads) k_neuron(NsDev d, uint32_t jstep) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_off[2 * kWarps];
  __shared__ uint32_t s_excl, s_total_tile;
  __shared__ Kick s_kick[32];
  __shared__ int s_nk;
  __shared__ unsigned long long s_events;
  __shared__ uint32_t s_outs;
  __shared__ unsigned long long s_log_base;
  __shared__ int s_logging;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t k = d.ctl->step_base + jstep;
  const uint32_t slot = (uint32_t)(k % d.D);
  constexpr bool COND = (MODE == 3 || MODE == 4);
  constexpr int NT = COND ? 4 : 1;

  if (tid == 0) {
    s_tile = atomicAdd(&d.ctl->ticket[k & 1], 1u);
    // log bookkeeping is advanced by the last tile of this step only after
    // every tile has published its flag, so read it before publishing
    s_log_base = d.ctl->log_size;
    s_logging = (d.log_idx != nullptr && d.ctl->log_steps < d.log_steps_cap &&
                 !(d.ctl->status & kErrLogFull)) ? 1 : 0;
    s_events = 0ull;
    s_outs = 0u;
    s_nk = 0;
  }
  if (d.drive_kind == 1 && warp == 1) {
    // reference-shaped global kicks (engine.rs:280-287): lane j computes kick j
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
  const uint32_t tile = s_tile;
  if (tid == 0 && tile == d.ntiles - 1) d.ctl->ticket[k & 1] = 0u;  // every ticket is taken
  const uint64_t base = (uint64_t)tile * kTile;
  const int nk = s_nk;

  bool spk[2][2];
  uint32_t rank[2][2];
  uint64_t idx0[2];

#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const uint64_t i0 = base + (uint64_t)r * 512 + 2 * (uint64_t)tid;
    idx0[r] = i0;
    NState st[2];
    float2 v2 = *reinterpret_cast<const float2*>(d.v + i0);
    st[0].v = v2.x; st[1].v = v2.y;
    if (MODEL == 1) {
      float2 u2 = *reinterpret_cast<const float2*>(d.u + i0);
      st[0].u = u2.x; st[1].u = u2.y;
    }
    if (MODEL == 0) {
      int2 r2 = *reinterpret_cast<const int2*>(d.refr + i0);
      st[0].refr = r2.x; st[1].refr = r2.y;
    }
    if (MODEL == 2) {
      float2 a = *reinterpret_cast<const float2*>(d.gm + i0);
      float2 b = *reinterpret_cast<const float2*>(d.gh + i0);
      float2 c = *reinterpret_cast<const float2*>(d.gn + i0);
      st[0].m = a.x; st[1].m = a.y; st[0].h = b.x; st[1].h = b.y; st[0].n = c.x; st[1].n = c.y;
    }
    if (MODE == 0 || MODE == 3) {
      float2 c = *reinterpret_cast<const float2*>(d.I + i0);
      st[0].I = c.x; st[1].I = c.y;
    }
    constexpr int NP = MODEL == 0 ? 5 : (MODEL == 1 ? 4 : 7);
    float par[2][7];
#pragma unroll
    for (int q = 0; q < NP; ++q) {
      float2 pv = *reinterpret_cast<const float2*>(d.par[q] + i0);
      par[0][q] = pv.x; par[1][q] = pv.y;
    }
    int rs[2] = {0, 0};
    if (MODEL == 0) {
      int2 r2 = *reinterpret_cast<const int2*>(d.refr_steps + i0);
      rs[0] = r2.x; rs[1] = r2.y;
    }
    // delivered synaptic input for this step (read and clear the slot)
    float S[NT][2];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      unsigned long long* ap = d.acc + ((uint64_t)t * d.D + slot) * d.n_pad + i0;
      longlong2 a2 = *reinterpret_cast<const longlong2*>(ap);
      S[t][0] = from_fix(a2.x);
      S[t][1] = from_fix(a2.y);
      *reinterpret_cast<longlong2*>(ap) = make_longlong2(0, 0);
    }
    float G[4][2];
    if (COND) {
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        float2 g2 = *reinterpret_cast<const float2*>(d.G[t] + i0);
        G[t][0] = g2.x; G[t][1] = g2.y;
      }
    }
    // drive draws: one Philox per pair
    U4 x = make_drive_draw(d, i0, k);
    float z[2] = {0.f, 0.f};
    if (d.drive_kind == 3) {
      float u1 = unif_open(x.x), u2 = unif(x.y);
      float l = ln_f(u1);
      float rr = sqrtf(-2.0f * l);
      float sn, cs;
      sincos_2pi(u2, &sn, &cs);
      z[0] = rr * cs;
      z[1] = rr * sn;
    }
    uint8_t inhv[2] = {0, 0};
    if (d.drive_kind == 3) {
      uchar2 ih = *reinterpret_cast<const uchar2*>(d.inh + i0);
      inhv[0] = ih.x; inhv[1] = ih.y;
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const uint64_t i = i0 + e;
      // drive value of this neuron (per-neuron draws for the non-Gaussian kinds)
      float addI = 0.f, kick = 0.f, addg = 0.f;
      if (d.drive_kind == 1 || d.drive_kind == 2 || d.drive_kind == 4) {
        U4 y = (e == 0) ? x : draw(d.seed, (uint32_t)i, k, kStreamDrive);
        if (d.drive_kind == 1) {
          if (unif(y.x) < d.drive_p) addI = unif(y.y) * d.drive_amp;
        } else if (d.drive_kind == 2) {
          if (y.x < d.p_thr) kick = d.drive_amp;
        } else {
          if (y.x < d.p_thr) addg = d.drive_amp;
        }
      } else if (d.drive_kind == 3) {
        addI = (inhv[e] ? d.sig_i : d.sig_e) * z[e];
      }
      float Iv = 0.f, kk = 0.f;
      const float vi = st[e].v;
      if (MODE == 0) {
        Iv = st[e].I;
        if (k > 0) Iv = (Iv + S[0][e]) * d.decay_I;
      } else if (MODE == 1) {
        kk = S[0][e];
      } else if (MODE == 2) {
        Iv = S[0][e];
      } else {
        float isyn = 0.f;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          float inc = S[t][e] * kSyn[t].gmax;
          if (kSyn[t].mg) inc = inc * (1.0f / (1.0f + (1.0f / 3.57f) * expf(-0.062f * vi)));
          float g = G[t][e] * d.Gdec[t] + inc;
          if (t == 0) g = g + addg;
          G[t][e] = g;
          isyn = isyn + g * (kSyn[t].erev - vi);
        }
        Iv = (MODE == 3) ? st[e].I + isyn : isyn;
      }
      Iv = Iv + addI;
      for (int q = 0; q < nk; ++q)
        if (s_kick[q].target == (uint32_t)i) Iv = Iv + s_kick[q].amt;
      kk = kk + kick;
      bool s = model_step<MODEL>(d, st[e], par[e], rs[e], Iv, kk, MODE == 1);
      st[e].I = Iv;
      s = s && (i < d.n);
      spk[r][e] = s;
    }
    // traces (per-neuron pre/post; double decay on a spike as in StdpTrace,
    // src/synapse/plasticity.rs:144-159)
    if (d.stdp) {
      float2 p2 = *reinterpret_cast<const float2*>(d.pre + i0);
      float2 q2 = *reinterpret_cast<const float2*>(d.post + i0);
      float pv[2] = {p2.x * d.ep, p2.y * d.ep};
      float qv[2] = {q2.x * d.em, q2.y * d.em};
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (spk[r][e]) {
          const uint64_t i = i0 + e;
          long long lst = d.last[i];
          long long dk = lst < 0 ? -1 : (long long)k - lst;
          float fp = (dk >= 0 && (unsigned long long)dk < d.Kp) ? d.Ep[dk] : 0.0f;
          float fm = (dk >= 0 && (unsigned long long)dk < d.Km) ? d.Em[dk] : 0.0f;
          d.qdec[i] = qv[e];
          pv[e] = pv[e] * fp + 1.0f;
          qv[e] = qv[e] * fm + 1.0f;
        }
      }
      *reinterpret_cast<float2*>(d.pre + i0) = make_float2(pv[0], pv[1]);
      *reinterpret_cast<float2*>(d.post + i0) = make_float2(qv[0], qv[1]);
    }
#pragma unroll
    for (int e = 0; e < 2; ++e)
      if (spk[r][e]) d.last[i0 + e] = (long long)k;
    // write back state
    *reinterpret_cast<float2*>(d.v + i0) = make_float2(st[0].v, st[1].v);
    if (MODEL == 1) *reinterpret_cast<float2*>(d.u + i0) = make_float2(st[0].u, st[1].u);
    if (MODEL == 0) *reinterpret_cast<int2*>(d.refr + i0) = make_int2(st[0].refr, st[1].refr);
    if (MODEL == 2) {
      *reinterpret_cast<float2*>(d.gm + i0) = make_float2(st[0].m, st[1].m);
      *reinterpret_cast<float2*>(d.gh + i0) = make_float2(st[0].h, st[1].h);
      *reinterpret_cast<float2*>(d.gn + i0) = make_float2(st[0].n, st[1].n);
    }
    if (MODE == 0 || MODE == 3 || MODE == 4)
      *reinterpret_cast<float2*>(d.I + i0) = make_float2(st[0].I, st[1].I);
    if (COND) {
#pragma unroll
      for (int t = 0; t < 4; ++t)
        *reinterpret_cast<float2*>(d.G[t] + i0) = make_float2(G[t][0], G[t][1]);
    }
    // warp ballots: ascending order inside the warp is (lane, parity)
    const unsigned me = __ballot_sync(0xffffffffu, spk[r][0]);
    const unsigned mo = __ballot_sync(0xffffffffu, spk[r][1]);
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t pre_cnt = __popc(me & lt) + __popc(mo & lt);
    rank[r][0] = pre_cnt;
    rank[r][1] = pre_cnt + (spk[r][0] ? 1u : 0u);
    if (lane == 0) s_off[r * kWarps + warp] = __popc(me) + __popc(mo);
    // spike bitmap: bit 2l / 2l+1 of the half-warp's word
    const uint32_t b2 = (spk[r][0] ? 1u : 0u) | (spk[r][1] ? 2u : 0u);
    const uint32_t lo = __reduce_or_sync(0xffffffffu, lane < 16 ? (b2 << (2 * lane)) : 0u);
    const uint32_t hi = __reduce_or_sync(0xffffffffu, lane >= 16 ? (b2 << (2 * (lane - 16))) : 0u);
    if (lane == 0) {
      const uint64_t wi = (base + (uint64_t)r * 512 + (uint64_t)warp * 64) >> 5;
      *reinterpret_cast<uint2*>(d.bitmap + wi) = make_uint2(lo, hi);
    }
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t run = 0;
#pragma unroll
    for (int q = 0; q < 2 * kWarps; ++q) {
      uint32_t c = s_off[q];
      s_off[q] = run;
      run += c;
    }
    s_total_tile = run;
    __threadfence();
    // decoupled look-back over tiles in ticket order (bounded wait)
    const uint32_t tag = (uint32_t)(k % 0x3FFFFFFFull) + 1u;
    volatile unsigned long long* fl = d.flags;
    uint32_t excl = 0;
    if (tile == 0) {
      fl[0] = flag_pack(tag, 2u, run);
    } else {
      fl[tile] = flag_pack(tag, 1u, run);
      int64_t p = (int64_t)tile - 1;
      uint32_t spins = 0;
      while (p >= 0) {
        unsigned long long f = fl[p];
        uint32_t ft = (uint32_t)(f >> 34), fs = (uint32_t)(f >> 32) & 3u;
        if (ft == tag && fs != 0u) {
          excl += (uint32_t)f;
          if (fs == 2u) break;
          --p;
        } else if (++spins > kSpinLimit) {
          atomicOr(&d.ctl->status, kErrLookback);
          break;
        }
      }
      fl[tile] = flag_pack(tag, 2u, excl + run);
    }
    s_excl = excl;
  }
  __syncthreads();
  const uint32_t excl = s_excl;
  const unsigned long long log_base = s_log_base;
  const bool logging = s_logging != 0;
  unsigned long long ev = 0;
  uint32_t outs = 0;
#pragma unroll
  for (int r = 0; r < 2; ++r) {
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      if (spk[r][e]) {
        const uint32_t i = (uint32_t)(idx0[r] + e);
        const uint32_t pos = excl + s_off[r * kWarps + warp] + rank[r][e];
        d.spk[pos] = i;
        if (logging && log_base + pos < d.log_cap) d.log_idx[log_base + pos] = i;
        ev += d.row_ptr[i + 1] - d.row_ptr[i];
        if (d.outp[i]) ++outs;
      }
    }
  }
  // block sums of events and output spikes
  for (int o = 16; o > 0; o >>= 1) {
    ev += __shfl_down_sync(0xffffffffu, ev, o);
    outs += __shfl_down_sync(0xffffffffu, outs, o);
  }
  if (lane == 0 && (ev | outs)) {
    atomicAdd(&s_events, ev);
    atomicAdd(&s_outs, outs);
  }
  __syncthreads();
  if (tid == 0) {
    if (s_events) atomicAdd(&d.ctl->events_total, s_events);
    if (s_outs) atomicAdd(&d.ctl->out_total, (unsigned long long)s_outs);
    if (tile == d.ntiles - 1) {
      // the last tile in order holds the inclusive total of this step
      const uint32_t total = excl + s_total_tile;
      d.ctl->step_spikes[k & 3] = total;
      d.ctl->spikes_total += total;
      d.ctl->sim_time += d.dt;  // FP64 clock, engine.rs:388-389
      if (logging) {
        if (log_base + total <= d.log_cap) {
          const unsigned long long s = d.ctl->log_steps;
          if (s == 0) d.ctl->log_first = k;
          d.log_off[s + 1] = log_base + total;
          d.ctl->log_size = log_base + total;
          d.ctl->log_steps = s + 1;
        } else {
          atomicOr(&d.ctl->status, kErrLogFull);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Kernel 2: propagation (+LTP) over spiking rows, then LTD over spiking
// targets' plastic incoming synapses. Work items: [0, cnt) rows, [cnt, 2cnt)
// incoming lists; one warp per item, grid-stride. Writes are disjoint: rows
// of spiking sources (LTP, and LTP+LTD when the target spiked too) versus
// incoming synapses whose source did not spike (LTD).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_w4(const NsDev& d, bool bf16, uint64_t e0, float w[4]) {
  if (bf16) {
    uint2 raw = *reinterpret_cast<const uint2*>(d.w16 + e0);
    w[0] = bf16_bits_to_f32((uint16_t)(raw.x & 0xffffu));
    w[1] = bf16_bits_to_f32((uint16_t)(raw.x >> 16));
    w[2] = bf16_bits_to_f32((uint16_t)(raw.y & 0xffffu));
    w[3] = bf16_bits_to_f32((uint16_t)(raw.y >> 16));
  } else {
    float4 f = *reinterpret_cast<const float4*>(d.w32 + e0);
    w[0] = f.x; w[1] = f.y; w[2] = f.z; w[3] = f.w;
  }
}

template <bool COND, bool BF16>
__global__ void __launch_bounds__(256) k_propagate(NsDev d, uint32_t jstep) {
  const int lane = threadIdx.x & 31;
  const uint64_t k = d.ctl->step_base + jstep;
  const uint32_t slot = (uint32_t)(k % d.D);
  const uint32_t cnt = (uint32_t)d.ctl->step_spikes[k & 3];
  const bool STDP = d.stdp != 0;
  const bool HOMEO = d.homeo != 0;
  const uint32_t items = STDP ? 2u * cnt : cnt;
  const uint32_t wglob = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t item = wglob; item < items; item += nw) {
    if (item < cnt) {
      const uint32_t j = __ldg(d.spk + item);
      const uint64_t beg = __ldg(d.row_ptr + j), end = __ldg(d.row_ptr + j + 1);
      const uint8_t rp = STDP ? __ldg(d.row_plastic + j) : 0;
      const uint8_t rt = COND ? __ldg(d.row_type + j) : 0;
      const float pj = (STDP && rp) ? d.pre[j] : 0.0f;
      const unsigned long long tbase = d.trace_pos ? d.trace_off[item] : 0ull;
      for (uint64_t b = beg & ~3ull; b < end; b += 128) {
        const uint64_t e0 = b + 4ull * lane;
        if (e0 >= end || e0 + 4 <= beg) continue;
        const uint4 c4 = __ldg(reinterpret_cast<const uint4*>(d.col + e0));
        const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
        float w[4];
        load_w4(d, BF16, e0, w);
        float wn[4] = {w[0], w[1], w[2], w[3]};
        bool inr[4], chg[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint64_t e = e0 + q;
          inr[q] = (e >= beg) && (e < end);
          chg[q] = false;
          if (!inr[q]) continue;
          const uint32_t i = cc[q];
          int t = 0;
          if (COND) t = (rt == 255) ? (int)__ldg(d.type + e) : (int)rt;
          const float val = (COND && (t == 1 || t == 2)) ? fabsf(w[q]) : w[q];
          atomicAdd(d.acc + ((uint64_t)t * d.D + slot) * d.n_pad + i,
                    (unsigned long long)to_fix(val));
          if (d.trace_pos) {
            const unsigned long long tp = tbase + (e - beg);
            if (tp < d.trace_cap) d.trace_pos[tp] = e;
          }
          if (HOMEO) {
            float mag;
            if (COND) {
              float g = w[q] * kSyn[t].gmax;
              if (kSyn[t].mg) g = g * (1.0f / (1.0f + (1.0f / 3.57f) * expf(-0.062f * d.v[i])));
              mag = fabsf(g);
            } else {
              mag = fabsf(w[q]);
            }
            d.contrib[e] = d.contrib[e] * d.cd + mag * d.one_m_cd;
          }
          if (STDP && rp && (rp == 1 || __ldg(d.plastic + e))) {
            float w1;
            if (!bit_of(d.bitmap, i)) {
              w1 = clampw(w[q] + d.a_plus * d.post[i], d.w_min, d.w_max);
            } else {
              w1 = clampw(w[q] + d.a_plus * d.qdec[i], d.w_min, d.w_max);
              w1 = clampw(w1 + d.neg_a_minus * pj, d.w_min, d.w_max);
            }
            wn[q] = w1;
            chg[q] = true;
          }
        }
        if (STDP && rp) {
          if (BF16) {
            if (chg[0] && chg[1] && chg[2] && chg[3]) {
              uint2 raw;
              raw.x = (uint32_t)f32_to_bf16_bits(wn[0]) | ((uint32_t)f32_to_bf16_bits(wn[1]) << 16);
              raw.y = (uint32_t)f32_to_bf16_bits(wn[2]) | ((uint32_t)f32_to_bf16_bits(wn[3]) << 16);
              *reinterpret_cast<uint2*>(d.w16 + e0) = raw;
            } else {
#pragma unroll
              for (int q = 0; q < 4; ++q)
                if (chg[q]) d.w16[e0 + q] = f32_to_bf16_bits(wn[q]);
            }
          } else {
            if (chg[0] && chg[1] && chg[2] && chg[3]) {
              *reinterpret_cast<float4*>(d.w32 + e0) = make_float4(wn[0], wn[1], wn[2], wn[3]);
            } else {
#pragma unroll
              for (int q = 0; q < 4; ++q)
                if (chg[q]) d.w32[e0 + q] = wn[q];
            }
          }
        }
      }
    } else if (STDP) {
      const uint32_t i = __ldg(d.spk + (item - cnt));
      const uint64_t b = __ldg(d.in_ptr + i), e = __ldg(d.in_ptr + i + 1);
      for (uint64_t q = b + lane; q < e; q += 32) {
        const uint2 sp = __ldg(d.in_list + q);
        if (bit_of(d.bitmap, sp.x)) continue;  // handled by the source's row walk
        const float pre = d.pre[sp.x];
        if (BF16) {
          const float w = bf16_bits_to_f32(d.w16[sp.y]);
          d.w16[sp.y] = f32_to_bf16_bits(clampw(w + d.neg_a_minus * pre, d.w_min, d.w_max));
        } else {
          const float w = d.w32[sp.y];
          d.w32[sp.y] = clampw(w + d.neg_a_minus * pre, d.w_min, d.w_max);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Kernel 3 (optional): homeostatic scaling, engine.rs:569-606, with the
// firing-rate EMA of engine.rs:637-642. FP64 rate and contribution sums;
// per-synapse scale in float. One warp per target.
// ---------------------------------------------------------------------------
template <bool BF16>
__global__ void __launch_bounds__(256) k_homeostasis(NsDev d, uint32_t jstep) {
  const int lane = threadIdx.x & 31;
  const uint32_t wglob = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  (void)jstep;
  for (uint64_t i = wglob; i < d.n; i += nw) {
    const double rate = d.rate[i];
    const double err = rate - d.h_target;
    const uint64_t b = d.all_in_ptr[i], e = d.all_in_ptr[i + 1];
    double sum = 0.0;
    for (uint64_t q = b + lane; q < e; q += 32) sum += (double)d.contrib[d.all_in_pos[q]];
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    const uint64_t cnt = e - b;
    if (cnt > 0 && sum >= 1e-12) {
      const double mean = sum / (double)cnt;
      const float nerr = (float)(-err);
      for (uint64_t q = b + lane; q < e; q += 32) {
        const uint32_t s = d.all_in_pos[q];
        const float rel = (float)((double)d.contrib[s] / mean);
        const float arg = nerr * rel * d.dt_f / d.h_tau_f;
        const float scale = expf(arg);
        if (BF16) {
          const float w = bf16_bits_to_f32(d.w16[s]) * scale;
          d.w16[s] = f32_to_bf16_bits(clampw(w, 0.0f, 10.0f));
        } else {
          d.w32[s] = clampw(d.w32[s] * scale, 0.0f, 10.0f);
        }
      }
    }
    if (lane == 0) {
      const double inst = bit_of(d.bitmap, (uint32_t)i) ? 1000.0 / d.dt : 0.0;
      d.rate[i] = rate + (inst - rate) * d.dt / 100.0;
    }
  }
}

__global__ void k_advance(Ctl* ctl, uint32_t steps) { ctl->step_base += steps; }

// exclusive scan of out-degrees of this step's spikers (traced step only)
__global__ void k_trace_offsets(NsDev d, unsigned long long* off) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const uint64_t k = d.ctl->step_base;
  const uint32_t cnt = (uint32_t)d.ctl->step_spikes[k & 3];
  unsigned long long run = 0;
  for (uint32_t q = 0; q < cnt; ++q) {
    off[q] = run;
    const uint32_t j = d.spk[q];
    run += d.row_ptr[j + 1] - d.row_ptr[j];
  }
  off[cnt] = run;
}

}  // namespace ns
