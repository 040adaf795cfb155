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
#include "ns_hh.cuh"
#include "ns_tc.cuh"

namespace ns {

constexpr int kThreads = 256;              // neuron kernel block
constexpr int kPairs = 4;                  // neuron pairs per thread
constexpr int kTile = kThreads * 2 * kPairs;  // 2048 neurons per tile
constexpr int kWarps = kThreads / 32;
static_assert(kPairs * kWarps <= 32, "one warp scans the per-group counts");
constexpr uint32_t kSmemTiles = 4096;       // tile offsets kept in shared memory up to this

// device status bits (host maps them to ns_status)
constexpr uint32_t kErrLogFull = 2u;
constexpr uint32_t kErrStageWait = 4u;   // a neuron kernel's staged loads did not arrive
constexpr uint32_t kErrDeferWindow = 8u; // a deferred-LTD row went more than 32 steps unflushed

struct Ctl {
  unsigned long long step_base;   // global step of graph node 0
  unsigned int tiles_done;        // neuron-kernel tiles finished this step
  unsigned int status;
  unsigned int log_ok[4];         // step k's spikes went to the log (k & 3)
  unsigned long long spikes_total, out_total, events_total;
  unsigned long long step_spikes[4];
  unsigned long long spk_acc[4];  // per-step spike count accumulators
  double sim_time;
  unsigned long long log_size;    // indices held
  unsigned long long log_steps;   // steps held
  unsigned long long log_first;   // global step of the first logged step
  // reward (R-STDP), R-STDP mode and consolidation frame; step k at [k & 1]
  double rew[2];                  // reward seen by phase 2 of step k
  double consA[2];                // frame scale A_k = a^(k - cons_k0)
  float frame[2][8];              // A_k, B_k, 1/A_k, A_k+1, B_k+1, 1/A_k+1, lr*R_k
  unsigned int mode[2];           // 0 no reward, 1 applied in the STDP walks, 2 full pass
  unsigned long long outs[4];     // output spikes of step k at [k & 3]
  double reward_sum;              // reward after each step since `origin`
  double rew_init;                // reward at step `origin`
  unsigned long long origin;
  unsigned long long cons_k0;     // step whose frame is the identity
  unsigned int ezero_init;        // eligibility all 0 and in range at `origin`
  unsigned int tail_done;         // blocks of k_tail finished (renormalisation)
  unsigned int win_done;          // blocks of k_window_finish finished
  // LFP of the reference conductance mode (engine.rs:492): per-step sums
  // of |g (E_rev - V)| in fixed point (2^-24) at [k & 3], folded into an
  // FP64 total one step later
  long long lfp_step[4];
  double lfp_total;
  // host stimulus (SimulationEngine::stimulate, engine.rs:156-161): the
  // values in NsDev::stim join the input current at step stim_at - 1
  // (0: none pending); the consuming thread zeroes them
  unsigned long long stim_at;
  // largest spike count of one step (SimulationStats::active_neurons,
  // engine.rs:624)
  unsigned long long max_step_spikes;
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
  float *pre, *post;
  float2* rec;                     // per step: {decayed pre, decayed post}, sign bit = spiked
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
  uint32_t* spk;                   // this step's spikes, tile-local ordered lists
  uint32_t* bitmap;                // n_pad / 32 words
  uint32_t* tile_cnt;              // spikes per tile this step
  uint32_t* tile_off;              // exclusive scan of tile_cnt (large networks)
  Ctl* ctl;
  const float *Ep, *Em;
  uint32_t* log_idx;
  unsigned long long* log_off;
  unsigned long long log_cap;
  unsigned long long log_steps_cap;
  unsigned long long* trace_pos;   // traced step only
  const unsigned long long* trace_off;
  unsigned long long trace_cap;
  // batched networks: network of each neuron, and per network its drive
  // seed and first neuron (null for a single network)
  const uint32_t* net_of;
  const unsigned long long* net_seed;
  const unsigned long long* net_base;
  // windowed stepping (delay >= 2, no plasticity): "slot has input" bits
  // [D][n_pad/32], and per-window spike segments of 256 neurons
  uint32_t* inbits;
  uint32_t* seg_cnt;               // [W][nseg]
  uint32_t* seg_lst;               // [W][n_pad]
  uint32_t* seg_off;               // [W][nseg + 1]
  uint32_t* step_total;            // [W]
  uint32_t nseg, wmax;
  // R-STDP (plasticity.rs:166-221), consolidation (:269-290) and
  // short-term plasticity (:85-116)
  int rstdp, cons, fuse, plast_any;
  int elig_all;                    // every plastic synapse carries a trace (no flag reads in the walks)
  float ce, rw_min, rw_max;        // exp(-dt/eligibility_tau), R-STDP clamp
  double reward_decay, rstdp_lr, cons_a, cons_T;
  unsigned long long reward_thr;
  // parameter dictionary: when a network has at most 256 distinct
  // parameter rows, the neuron kernel reads a 1-byte index per neuron and
  // the row from a table in shared memory (8 floats per row: the model's
  // parameter arrays in par[] order, the LIF refractory steps as int bits
  // in column 7)
  const uint8_t* pidx;
  const float* ptab;
  uint32_t ptab_rows;
  // single-network sharding: this rank updates tiles [tile0, tile0 +
  // tiles_own); the other tiles' spikes arrive as bitmap words (0 and all
  // tiles on one GPU)
  uint32_t tile0, tiles_own;
  // synapse types present (bit t): accumulator rows of absent types stay
  // zero and are neither read nor cleared (conductance modes)
  uint32_t type_mask;
  float* elig;                     // eligibility values [m_pad]
  const uint8_t* elig_flag;        // synapse carries an eligibility trace [m_pad]
  const float* stp_f;              // STP factor per synapse, or null
  float* stim;                     // pending host stimulus per neuron [n_pad]
  // deferred LTD (step schedule 5): rec[k][i].x holds the bits of i's
  // spikes over the last 32 steps (bit b: step k - b) instead of its decayed
  // pre trace; per source j, lstart[j] = {pre trace after step astep (float
  // bits), astep}: every LTD of j's synapses at steps <= astep is applied,
  // those after wait for j's next row walk or for the row's flush, which
  // comes every 32 steps (rows in 32 contiguous blocks, block k mod 32 at
  // step k).
  uint2* lstart;
  int defer;
  // drive precomputed by k_drive for the Poisson-kick, Gaussian and
  // Poisson-conductance kinds, parity-buffered by step: drv[k & 1][i] is the
  // amount drive_of gives neuron i at step k (the neuron kernel draws the
  // reference-uniform kind itself)
  float* drv;
  // the neuron kernel stages its sub-tiles' input arrays in shared memory
  // with bulk copies (stage_plan); 0: direct loads
  int stage;
};

// ---------------------------------------------------------------------------
// Staged loads of the neuron kernel. A tile of 2048 neurons is updated in four
// sub-tiles of 512 (one neuron pair per thread); every input array's 512
// entries of a sub-tile are brought into shared memory by one bulk copy
// (cp.async.bulk, completion counted in bytes on an mbarrier), two
// sub-tiles in flight at a time. stage_plan gives each array's byte offset in
// a sub-tile buffer (kNoStage: not read) and the buffer's size; host and
// device compute it from the same fields.
// ---------------------------------------------------------------------------
constexpr uint32_t kStageSub = 512;                 // neurons per sub-tile
constexpr uint32_t kNoStage = 0xffffffffu;
constexpr uint32_t kStageMaxBytes = 32u * 1024u;    // per buffer (two per block)

struct StagePlan {
  uint32_t v, u, refr, gm, gh, gn, I, par[7], rsteps, pidx, acc[4], G[4], pre, post, rec, drv;
  uint32_t bytes;
};

__host__ __device__ __forceinline__ StagePlan stage_plan(int model, int mode, bool pt, int stdp,
                                                         int defer, int drive_kind,
                                                         uint32_t type_mask) {
  StagePlan p;
  uint32_t off = 0;
  auto take = [&](bool on, uint32_t esz) -> uint32_t {
    if (!on) return kNoStage;
    const uint32_t at = off;
    off += kStageSub * esz;
    return at;
  };
  const bool cond = mode == 3 || mode == 4;
  const int np = model == 0 ? 5 : (model == 1 ? 4 : 7);
  p.v = take(true, 4);
  p.u = take(model == 1, 4);
  p.refr = take(model == 0, 4);
  p.gm = take(model == 2, 4);
  p.gh = take(model == 2, 4);
  p.gn = take(model == 2, 4);
  p.I = take(mode == 0 || mode == 3, 4);
  for (int q = 0; q < 7; ++q) p.par[q] = take(!pt && q < np, 4);
  p.rsteps = take(!pt && model == 0, 4);
  p.pidx = take(pt, 1);
  for (int t = 0; t < 4; ++t) p.acc[t] = take(cond ? ((type_mask >> t) & 1u) != 0u : t == 0, 8);
  for (int t = 0; t < 4; ++t) p.G[t] = take(cond, 4);
  p.pre = take(stdp != 0, 4);
  p.post = take(stdp != 0, 4);
  p.rec = take(stdp != 0 && defer != 0, 8);
  p.drv = take(drive_kind >= 2, 4);
  p.bytes = off;
  return p;
}

// Thread 0 enqueues the bulk copies of sub-tile `sub` of the block's tile
// (first neuron `first`) into buffer `buf`, completing on `mbar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          tc::smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(tc::smem_u32(mbar))
      : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(mbar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool bit_of(const uint32_t* bm, uint32_t i) {
  return (bm[i >> 5] >> (i & 31)) & 1u;
}

// exclusive scan of n values by one 256-thread block, result in out[0..n];
// returns the total. Thread t owns a contiguous run of ceil(n / 256) values:
// it sums the run (independent loads, two round trips for the whole scan
// rather than one per 1024 values), the block scans the 256 sums, and the
// thread writes the run's offsets (its second read of the run hits L1).
__device__ uint32_t block_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n) {
  __shared__ uint32_t s_w[8];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t per = (n + 255u) / 256u;
  const uint32_t b = min(n, (uint32_t)tid * per), e = min(n, b + per);
  uint32_t loc = 0;
#pragma unroll 8
  for (uint32_t q = b; q < e; ++q) loc += in[q];
  uint32_t inc = loc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  uint32_t wpre = 0, tot = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const uint32_t x = s_w[q];
    wpre += q < warp ? x : 0u;
    tot += x;
  }
  uint32_t run = wpre + inc - loc;
#pragma unroll 8
  for (uint32_t q = b; q < e; ++q) {
    const uint32_t x = in[q];
    out[q] = run;
    run += x;
  }
  if (tid == 0) out[n] = tot;
  __syncthreads();
  return tot;
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

// Drive stream key of neuron i: the handle's seed and i, or, in a batch of
// networks, the network's own seed and i's index inside its network, so that
// a network draws the same drive in a batch as when it runs alone.
__device__ __forceinline__ void drive_key(const NsDev& d, uint64_t i, uint64_t& seed, uint32_t& li) {
  seed = d.seed;
  li = (uint32_t)i;
  if (d.net_of != nullptr) {
    const uint32_t q = d.net_of[i];
    seed = d.net_seed[q];
    li = (uint32_t)(i - d.net_base[q]);
  }
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
    bool spk;
    if (d.hh_int == 0) {
      float am, bm, ah, bh, an, bn;
      hh_rates(v, am, bm, ah, bh, an, bn);
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
      spk = hh_rl_step(v, m, h, n, Iin, p, dt);
    }
    if (delta) v = v + kick;
    s.v = v; s.m = m; s.h = h; s.n = n;
    return spk;
  }
}

// Drive of neuron i at step k from its Philox draw y (kinds 1, 2, 4) or its
// Gaussian sample z (kind 3): added current, voltage kick, added conductance.
__device__ __forceinline__ void drive_of(const NsDev& d, const U4& y, float z, uint8_t inh,
                                         float& addI, float& kick, float& addg) {
  addI = 0.f; kick = 0.f; addg = 0.f;
  if (d.drive_kind == 1) {
    if (unif(y.x) < d.drive_p) addI = unif(y.y) * d.drive_amp;
  } else if (d.drive_kind == 2) {
    if (y.x < d.p_thr) kick = d.drive_amp;
  } else if (d.drive_kind == 4) {
    if (y.x < d.p_thr) addg = d.drive_amp;
  } else if (d.drive_kind == 3) {
    addI = (inh ? d.sig_i : d.sig_e) * z;
  }
}

// Gaussian pair of the draw x: cos for the even neuron, sin for the odd one
// (Box-Muller on the drive's own log / sincos).
__device__ __forceinline__ void gauss_pair(const U4& x, float& z0, float& z1) {
  const float u1 = unif_open(x.x), u2 = unif(x.y);
  const float l = ln_f(u1);
  const float rr = sqrtf(-2.0f * l);
  float sn, cs;
  sincos_2pi(u2, &sn, &cs);
  z0 = rr * cs;
  z1 = rr * sn;
}

// The drive amount of neuron i at step k from its precomputed value: the
// current (uniform, Gaussian), the kick or the added conductance, by kind.
__device__ __forceinline__ void drive_from(const NsDev& d, float val, float& addI, float& kick,
                                           float& addg) {
  addI = (d.drive_kind == 1 || d.drive_kind == 3) ? val : 0.f;
  kick = d.drive_kind == 2 ? val : 0.f;
  addg = d.drive_kind == 4 ? val : 0.f;
}

// Drive of step k for every neuron, precomputed one step ahead beside the
// walks of the previous step (kinds 2, 3, 4: one Philox draw per neuron, or
// per pair for the Gaussian drive; the same draws and arithmetic as the
// neuron kernel's own). Thread per neuron pair.
__global__ void __launch_bounds__(256) k_drive(NsDev d, uint32_t jstep) {
  const uint64_t k = d.ctl->step_base + jstep;
  float* out = d.drv + (k & 1) * d.n_pad;
  const uint64_t pairs = d.n_pad >> 1;
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < pairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = 2 * p;
    U4 y2[2] = {U4{0u, 0u, 0u, 0u}, U4{0u, 0u, 0u, 0u}};
    float z[2] = {0.f, 0.f};
    uchar2 ih = make_uchar2(0, 0);
    if (d.drive_kind == 3) ih = *reinterpret_cast<const uchar2*>(d.inh + i0);
    if (d.net_of == nullptr) {
      if (d.drive_kind == 3) {
        gauss_pair(draw(d.seed, (uint32_t)(i0 >> 1), k, kStreamDrive), z[0], z[1]);
      } else {
        y2[0] = poisson_draw(d.seed, (uint32_t)i0, k);
        y2[1] = poisson_draw(d.seed, (uint32_t)(i0 + 1), k);
      }
    } else {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        uint64_t sd;
        uint32_t li;
        drive_key(d, i0 + e, sd, li);
        if (d.drive_kind == 3) {
          float g0, g1;
          gauss_pair(draw(sd, li >> 1, k, kStreamDrive), g0, g1);
          z[e] = (li & 1u) ? g1 : g0;
        } else {
          y2[e] = poisson_draw(sd, li, k);
        }
      }
    }
    const uint8_t inhv[2] = {ih.x, ih.y};
    float val[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      float addI, kick, addg;
      drive_of(d, y2[e], z[e], inhv[e], addI, kick, addg);
      val[e] = d.drive_kind == 2 ? kick : (d.drive_kind == 4 ? addg : addI);
    }
    *reinterpret_cast<float2*>(out + i0) = make_float2(val[0], val[1]);
  }
}

// Input assembly and model update of one neuron at step k (the arithmetic
// the float oracle mirrors). S: delivered synaptic input per accumulator
// type; G: the neuron's conductances (conductance modes).
template <int MODEL, int MODE>
__device__ __forceinline__ bool update_one(const NsDev& d, uint64_t k, uint64_t i, NState& st,
                                           const float* par, int rs, const float* S, float* G,
                                           float addI, float kick, float addg, const Kick* kicks,
                                           int nk, float stim = 0.f, float* lfp = nullptr) {
  float Iv = 0.f, kk = 0.f;
  const float vi = st.v;
  if (MODE == 0) {
    Iv = st.I;
    if (k > 0) Iv = (Iv + S[0]) * d.decay_I;
  } else if (MODE == 1) {
    kk = S[0];
  } else if (MODE == 2) {
    Iv = S[0];
  } else {
    float isyn = 0.f;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      float inc = S[t] * kSyn[t].gmax;
      // Mg block only on a delivered increment (0 times a finite factor is 0)
      if (kSyn[t].mg && inc != 0.0f) inc = inc * (1.0f / (1.0f + (1.0f / 3.57f) * expf(-0.062f * vi)));
      float g = G[t] * d.Gdec[t] + inc;
      if (t == 0) g = g + addg;
      G[t] = g;
      const float cur = g * (kSyn[t].erev - vi);
      isyn = isyn + cur;
      if (MODE == 3 && lfp != nullptr) *lfp = *lfp + fabsf(cur);   // lfp += |I_syn|, engine.rs:492
    }
    Iv = (MODE == 3) ? st.I + isyn : isyn;
  }
  if (stim != 0.0f) Iv = Iv + stim;   // host stimulus, engine.rs:156-161
  Iv = Iv + addI;
  for (int q = 0; q < nk; ++q)
    if (kicks[q].target == (uint32_t)i) Iv = Iv + kicks[q].amt;
  kk = kk + kick;
  const bool sp = model_step<MODEL>(d, st, par, rs, Iv, kk, MODE == 1);
  st.I = Iv;
  return sp;
}

// ---------------------------------------------------------------------------
// Per-step bookkeeping of the rest of phase 2, run by one thread (k_setup,
// between the neuron kernel and the walks of the step):
//  - the reward seen by step k: the previous step's reward decayed
//    (engine.rs:563, whenever plasticity is on), raised to min(r + 1, 1) when
//    that step had at least reward_threshold output spikes (:626-631);
//  - the R-STDP mode of step k: 0 when |reward| <= 0.001 (engine.rs:547-548);
//    1 when every eligibility trace was zero before the step (the previous
//    step applied the reward), so the walks apply it to the synapses they
//    touch; 2 otherwise (a full pass after the walks);
//  - the consolidation frame: A_k = a^(k - k0), B_k = target*(1 - A_k), with
//    a = 1 - dt*drift/tau (ConsolidationRule::apply, plasticity.rs:286-289).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void phase2_setup(const NsDev& d, unsigned long long k) {
  // the output spikes of step k-1 were counted by its walks (flush_counters)
  Ctl* c = d.ctl;
  double R;
  unsigned ez;
  if (k == c->origin) {
    R = c->rew_init;
    ez = c->ezero_init;
  } else {
    const double Rp = c->rew[(k - 1) & 1];
    const double Rd = d.plast_any ? Rp * d.reward_decay : Rp;
    R = (c->outs[(k - 1) & 3] >= d.reward_thr) ? fmin(Rd + 1.0, 1.0) : Rd;
    c->reward_sum += R;
    ez = c->mode[(k - 1) & 1] != 0u ? 1u : 0u;
  }
  c->rew[k & 1] = R;
  c->outs[(k + 2) & 3] = 0ull;
  const bool active = d.rstdp && fabs(R) > 0.001;
  c->mode[k & 1] = !active ? 0u : ((ez && d.fuse) ? 1u : 2u);
  float* f = c->frame[k & 1];
  f[6] = (float)(d.rstdp_lr * R);
  if (d.cons) {
    const double A0 = (k == c->cons_k0) ? 1.0 : c->consA[(k - 1) & 1] * d.cons_a;
    const double A1 = A0 * d.cons_a;
    c->consA[k & 1] = A0;
    f[0] = (float)A0; f[1] = (float)(d.cons_T * (1.0 - A0)); f[2] = (float)(1.0 / A0);
    f[3] = (float)A1; f[4] = (float)(d.cons_T * (1.0 - A1)); f[5] = (float)(1.0 / A1);
  }
}

__global__ void k_setup(NsDev d, uint32_t jstep) {
  if (threadIdx.x == 0 && blockIdx.x == 0) phase2_setup(d, d.ctl->step_base + jstep);
}

// ---------------------------------------------------------------------------
// Kernel 1: neuron update + trace decay + ordered compaction, with the
// step's drive (precomputed by k_drive one step ahead, or drawn here for the
// reference-uniform kind). Thread t of tile T owns the neuron pairs
// (T*2048 + r*512 + 2t, +1), r < 4, so every state array is read with 8-byte
// coalesced loads. All loads of a pair are issued before any store. Each tile writes its spikes, ascending, to its
// own slice of the spike buffer (warp ballots + a 32-entry scan), so no tile
// waits for another; the last tile to finish does the step's bookkeeping.
// ---------------------------------------------------------------------------
// STIM: this step takes a pending host stimulus (the variant runs for that
// one step; the others carry no stimulus code).
template <int MODEL, int MODE, bool PT, bool STIM>
__global__ void __launch_bounds__(kThreads) k_neuron(NsDev d, uint32_t jstep) {
  extern __shared__ __align__(128) uint8_t s_stage[];   // two sub-tile buffers when staged
  __shared__ __align__(8) uint64_t s_mbar[2];
  __shared__ float s_tab[PT ? 256 * 8 : 1];
  __shared__ uint32_t s_off[kPairs * kWarps];
  __shared__ uint32_t s_me[kPairs * kWarps], s_mo[kPairs * kWarps];
  __shared__ uint32_t s_total;
  __shared__ Kick s_kick[32];
  __shared__ int s_nk;
  __shared__ int s_last;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t k = d.ctl->step_base + jstep;
  const uint32_t slot = (uint32_t)(k % d.D);
  constexpr bool COND = (MODE == 3 || MODE == 4);
  constexpr int NT = COND ? 4 : 1;
  constexpr int NP = MODEL == 0 ? 5 : (MODEL == 1 ? 4 : 7);
  // spike lists, tile counts and trace records are double-buffered by step
  // parity so that the LTD kernel of step k can run beside this kernel
  const uint32_t par_k = (uint32_t)(k & 1);
  uint32_t* const spk_k = d.spk + par_k * d.n_pad;
  uint32_t* const tcnt_k = d.tile_cnt + par_k * (d.ntiles + 1);
  float2* const rec_k = d.rec + par_k * d.n_pad;

  if (tid == 0) s_nk = 0;
  if (MODE == 3 && blockIdx.x == 0 && tid == 0) {
    // the previous step's LFP sum is complete: fold it; clear the next slot
    Ctl* c = d.ctl;
    c->lfp_total += (double)c->lfp_step[(k + 3) & 3] * 0x1p-24;
    c->lfp_step[(k + 3) & 3] = 0ll;
    c->lfp_step[(k + 1) & 3] = 0ll;
  }
  long long lfp_fix = 0;
  const bool stim_on = STIM && d.ctl->stim_at == k + 1;
  if (PT)
    for (uint32_t q = tid; q < d.ptab_rows * 8u; q += kThreads) s_tab[q] = __ldg(d.ptab + q);
  __syncthreads();
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
  const uint32_t tile = blockIdx.x + d.tile0;
  const uint64_t base = (uint64_t)tile * kTile;
  const int nk = s_nk;

  // ---- staged loads: plan, barriers, the first two sub-tiles in flight ----
  const bool stg = d.stage != 0;
  const StagePlan sp = stage_plan(MODEL, MODE, PT, d.stdp, d.defer, d.drive_kind, d.type_mask);
  const uint32_t prev_k = par_k ^ 1u;
  auto issue = [&](int sub) {
    uint8_t* buf = s_stage + (uint32_t)(sub & 1) * sp.bytes;
    uint64_t* mb = &s_mbar[sub & 1];
    const uint64_t f = base + (uint64_t)sub * kStageSub;
    tc::fence_proxy_async();
    mbar_expect_tx(mb, sp.bytes);
    auto cp = [&](uint32_t off, const void* src, uint32_t esz) {
      if (off != kNoStage)
        bulk_g2s(buf + off, reinterpret_cast<const uint8_t*>(src) + f * esz, kStageSub * esz, mb);
    };
    cp(sp.v, d.v, 4);
    cp(sp.u, d.u, 4);
    cp(sp.refr, d.refr, 4);
    cp(sp.gm, d.gm, 4);
    cp(sp.gh, d.gh, 4);
    cp(sp.gn, d.gn, 4);
    cp(sp.I, d.I, 4);
#pragma unroll
    for (int q = 0; q < 7; ++q) cp(sp.par[q], d.par[q], 4);
    cp(sp.rsteps, d.refr_steps, 4);
    cp(sp.pidx, d.pidx, 1);
#pragma unroll
    for (int t = 0; t < 4; ++t) cp(sp.acc[t], d.acc + ((uint64_t)t * d.D + slot) * d.n_pad, 8);
#pragma unroll
    for (int t = 0; t < 4; ++t) cp(sp.G[t], d.G[t], 4);
    cp(sp.pre, d.pre, 4);
    cp(sp.post, d.post, 4);
    cp(sp.rec, d.rec + prev_k * d.n_pad, 8);
    cp(sp.drv, d.drv + par_k * d.n_pad, 4);
  };
  if (stg) {
    if (tid == 0) {
      tc::mbar_init(&s_mbar[0], 1);
      tc::mbar_init(&s_mbar[1], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
      issue(0);
      issue(1);
    }
  }

#pragma unroll 1
  for (int r = 0; r < kPairs; ++r) {
    const uint64_t i0 = base + (uint64_t)r * 512 + 2 * (uint64_t)tid;
    // ---- the pair's inputs: from the staged sub-tile, or loaded here ----
    const uint8_t* sb = s_stage + (uint32_t)(r & 1) * sp.bytes;
    if (stg) {
      bool ok = tc::mbar_wait(&s_mbar[r & 1], (uint32_t)(r >> 1) & 1u, 1u << 22);
      if (!__syncthreads_and(ok)) {
        // the copies did not arrive: record it, give the ones in flight a
        // bounded time to land, and leave the tile (the step is reported)
        if (tid == 0) {
          atomicOr(&d.ctl->status, kErrStageWait);
          tc::mbar_wait(&s_mbar[0], 1u, 1u << 22);
          tc::mbar_wait(&s_mbar[1], 1u, 1u << 22);
        }
        __syncthreads();
        return;
      }
    }
#define NS_LD(T, off, gptr, esz) \
    (stg ? *reinterpret_cast<const T*>(sb + (off) + (esz) * 2u * (uint32_t)tid) \
         : *reinterpret_cast<const T*>(gptr))
    NState st[2];
    const float2 v2 = NS_LD(float2, sp.v, d.v + i0, 4u);
    st[0].v = v2.x; st[1].v = v2.y;
    if (MODEL == 1) {
      const float2 u2 = NS_LD(float2, sp.u, d.u + i0, 4u);
      st[0].u = u2.x; st[1].u = u2.y;
    }
    if (MODEL == 0) {
      const int2 r2 = NS_LD(int2, sp.refr, d.refr + i0, 4u);
      st[0].refr = r2.x; st[1].refr = r2.y;
    }
    if (MODEL == 2) {
      const float2 a = NS_LD(float2, sp.gm, d.gm + i0, 4u);
      const float2 b = NS_LD(float2, sp.gh, d.gh + i0, 4u);
      const float2 c = NS_LD(float2, sp.gn, d.gn + i0, 4u);
      st[0].m = a.x; st[1].m = a.y; st[0].h = b.x; st[1].h = b.y; st[0].n = c.x; st[1].n = c.y;
    }
    if (MODE == 0 || MODE == 3) {
      const float2 c = NS_LD(float2, sp.I, d.I + i0, 4u);
      st[0].I = c.x; st[1].I = c.y;
    }
    float par[2][7];
    int rs[2] = {0, 0};
    if (PT) {
      const uchar2 ix = NS_LD(uchar2, sp.pidx, d.pidx + i0, 1u);
      const float* t0 = s_tab + 8u * ix.x;
      const float* t1 = s_tab + 8u * ix.y;
#pragma unroll
      for (int q = 0; q < NP; ++q) { par[0][q] = t0[q]; par[1][q] = t1[q]; }
      if (MODEL == 0) { rs[0] = __float_as_int(t0[7]); rs[1] = __float_as_int(t1[7]); }
    } else {
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        const float2 pv = NS_LD(float2, sp.par[q], d.par[q] + i0, 4u);
        par[0][q] = pv.x; par[1][q] = pv.y;
      }
      if (MODEL == 0) {
        const int2 r2 = NS_LD(int2, sp.rsteps, d.refr_steps + i0, 4u);
        rs[0] = r2.x; rs[1] = r2.y;
      }
    }
    longlong2 accv[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t)
      accv[t] = (!COND || ((d.type_mask >> t) & 1u))
                    ? NS_LD(longlong2, sp.acc[t], d.acc + ((uint64_t)t * d.D + slot) * d.n_pad + i0, 8u)
                    : make_longlong2(0, 0);
    float G[4][2];
    if (COND) {
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const float2 g2 = NS_LD(float2, sp.G[t], d.G[t] + i0, 4u);
        G[t][0] = g2.x; G[t][1] = g2.y;
      }
    }
    float2 p2 = make_float2(0.f, 0.f), q2 = make_float2(0.f, 0.f);
    uint2 hist = make_uint2(0u, 0u);
    if (d.stdp) {
      p2 = NS_LD(float2, sp.pre, d.pre + i0, 4u);
      q2 = NS_LD(float2, sp.post, d.post + i0, 4u);
      if (d.defer) {
        // spike bits of the previous step's records (the other parity)
        const float4 pr = NS_LD(float4, sp.rec, d.rec + prev_k * d.n_pad + i0, 8u);
        hist = make_uint2(__float_as_uint(pr.x), __float_as_uint(pr.z));
      }
    }
    float2 pdrv = make_float2(0.f, 0.f);
    if (d.drive_kind >= 2) pdrv = NS_LD(float2, sp.drv, d.drv + par_k * d.n_pad + i0, 4u);
#undef NS_LD
    if (stg) {
      // every thread has its pair's inputs: the buffer takes sub-tile r + 2
      __syncthreads();
      if (tid == 0 && r + 2 < kPairs) issue(r + 2);
    }
    // ---- delivered synaptic input for this step (the slot is cleared) ----
    if (d.inbits && lane == 0) {
      uint32_t* ib = d.inbits + (uint64_t)slot * (d.n_pad >> 5) + ((i0 - 2 * (uint64_t)lane) >> 5);
      *reinterpret_cast<uint2*>(ib) = make_uint2(0u, 0u);
    }
    float S[NT][2];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      S[t][0] = from_fix(accv[t].x);
      S[t][1] = from_fix(accv[t].y);
      if (!COND || ((d.type_mask >> t) & 1u))
        *reinterpret_cast<longlong2*>(d.acc + ((uint64_t)t * d.D + slot) * d.n_pad + i0) =
            make_longlong2(0, 0);
    }
    // ---- drive: the reference-uniform kind draws here (one Philox per
    // neuron; batches refuse this kind); the other kinds were precomputed
    // by k_drive ----
    U4 y2[2] = {U4{0u, 0u, 0u, 0u}, U4{0u, 0u, 0u, 0u}};
    if (d.drive_kind == 1) {
      y2[0] = draw(d.seed, (uint32_t)i0, k, kStreamDrive);
      y2[1] = draw(d.seed, (uint32_t)(i0 + 1), k, kStreamDrive);
    }
    float2 sti = make_float2(0.f, 0.f);
    if (stim_on) {
      sti = *reinterpret_cast<const float2*>(d.stim + i0);
      if (sti.x != 0.0f || sti.y != 0.0f)
        *reinterpret_cast<float2*>(d.stim + i0) = make_float2(0.f, 0.f);
    }
    bool spk[2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const uint64_t i = i0 + e;
      float addI, kick, addg;
      if (d.drive_kind >= 2) drive_from(d, e == 0 ? pdrv.x : pdrv.y, addI, kick, addg);
      else drive_of(d, y2[e], 0.f, 0, addI, kick, addg);
      float Se[NT], Ge[4];
#pragma unroll
      for (int t = 0; t < NT; ++t) Se[t] = S[t][e];
#pragma unroll
      for (int t = 0; t < 4; ++t) Ge[t] = COND ? G[t][e] : 0.f;
      float lf = 0.f;
      const bool sp = update_one<MODEL, MODE>(d, k, i, st[e], par[e], rs[e], Se, Ge, addI, kick,
                                              addg, s_kick, nk, e == 0 ? sti.x : sti.y, MODE == 3 ? &lf : nullptr);
      if (MODE == 3) lfp_fix += __float2ll_rn(lf * 0x1p24f);
#pragma unroll
      for (int t = 0; t < 4; ++t) if (COND) G[t][e] = Ge[t];
      spk[e] = sp && (i < d.n);
    }
    // ---- traces: per-step decay here; the spike-time bump (double decay of
    // StdpTrace, src/synapse/plasticity.rs:144-159) is done by the spiker's
    // own row walk in k_propagate. rec[i] carries this step's decayed,
    // pre-bump traces with the sign bit set when i spiked: the one value a
    // synapse's LTP (target side) or LTD (source side) needs.
    if (d.stdp) {
      const float pv0 = p2.x * d.ep, pv1 = p2.y * d.ep;
      const float qv0 = q2.x * d.em, qv1 = q2.y * d.em;
      *reinterpret_cast<float2*>(d.pre + i0) = make_float2(pv0, pv1);
      *reinterpret_cast<float2*>(d.post + i0) = make_float2(qv0, qv1);
      float4 rr;
      if (d.defer) {
        // deferred LTD: spike bits of the last 32 steps instead of the pre
        // trace (the row walks take the source's pre trace from lstart)
        rr = make_float4(__uint_as_float((hist.x << 1) | (spk[0] ? 1u : 0u)), spk[0] ? -qv0 : qv0,
                         __uint_as_float((hist.y << 1) | (spk[1] ? 1u : 0u)), spk[1] ? -qv1 : qv1);
      } else {
        rr = make_float4(spk[0] ? -pv0 : pv0, spk[0] ? -qv0 : qv0,
                         spk[1] ? -pv1 : pv1, spk[1] ? -qv1 : qv1);
      }
      *reinterpret_cast<float4*>(rec_k + i0) = rr;
    }
    // ---- write back state ----
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
    // ---- warp ballots: ascending order inside the warp is (lane, parity) ----
    const unsigned me = __ballot_sync(0xffffffffu, spk[0]);
    const unsigned mo = __ballot_sync(0xffffffffu, spk[1]);
    if (lane == 0) {
      s_off[r * kWarps + warp] = __popc(me) + __popc(mo);
      s_me[r * kWarps + warp] = me;
      s_mo[r * kWarps + warp] = mo;
    }
    // spike bitmap: bit 2l / 2l+1 of the half-warp's word
    const uint32_t b2 = (spk[0] ? 1u : 0u) | (spk[1] ? 2u : 0u);
    const uint32_t lo = __reduce_or_sync(0xffffffffu, lane < 16 ? (b2 << (2 * lane)) : 0u);
    const uint32_t hi = __reduce_or_sync(0xffffffffu, lane >= 16 ? (b2 << (2 * (lane - 16))) : 0u);
    if (lane == 0) {
      const uint64_t wi = (base + (uint64_t)r * 512 + (uint64_t)warp * 64) >> 5;
      *reinterpret_cast<uint2*>(d.bitmap + wi) = make_uint2(lo, hi);
    }
  }
  __syncthreads();
  if (warp == 0) {
    // tile-local exclusive offsets of the kPairs x kWarps (r, warp) groups
    const uint32_t c = lane < kPairs * kWarps ? s_off[lane] : 0u;
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < kPairs * kWarps; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane < kPairs * kWarps) s_off[lane] = incl - c;
    if (lane == kPairs * kWarps - 1) {
      s_total = incl;
      tcnt_k[tile] = incl;
    }
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < kPairs; ++r) {
    const unsigned me = s_me[r * kWarps + warp], mo = s_mo[r * kWarps + warp];
    const bool s0 = (me >> lane) & 1u, s1 = (mo >> lane) & 1u;
    const uint32_t pre_cnt = __popc(me & lt) + __popc(mo & lt);
    const uint32_t i0 = (uint32_t)(base + (uint64_t)r * 512 + 2 * (uint64_t)tid);
    const uint32_t o = s_off[r * kWarps + warp] + pre_cnt;
    if (s0) spk_k[base + o] = i0;
    if (s1) spk_k[base + o + (s0 ? 1u : 0u)] = i0 + 1;
  }
  if (MODE == 3) {
    for (int o = 16; o > 0; o >>= 1) lfp_fix += __shfl_down_sync(0xffffffffu, lfp_fix, o);
    if (lane == 0 && lfp_fix) atomicAdd((unsigned long long*)&d.ctl->lfp_step[k & 3], (unsigned long long)lfp_fix);
  }
  // last tile of the step: counters, FP64 clock, spike-log bookkeeping
  if (tid == 0) {
    if (s_total) atomicAdd(&d.ctl->spk_acc[k & 3], (unsigned long long)s_total);
    __threadfence();
    const unsigned done = atomicAdd(&d.ctl->tiles_done, 1u);
    s_last = (done == d.ntiles - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (d.ntiles > kSmemTiles) block_scan_u32(tcnt_k, d.tile_off + par_k * (d.ntiles + 1), d.ntiles);
  if (tid == 0) {
    Ctl* c = d.ctl;
    const unsigned long long total = atomicAdd(&c->spk_acc[k & 3], 0ull);
    c->spk_acc[(k + 2) & 3] = 0ull;
    c->tiles_done = 0u;
    c->step_spikes[k & 3] = total;
    if (total > c->max_step_spikes) c->max_step_spikes = total;
    c->spikes_total += total;
    c->sim_time += d.dt;  // FP64 clock, engine.rs:388-389
    unsigned ok = 0u;
    if (d.log_idx != nullptr && c->log_steps < d.log_steps_cap && !(c->status & kErrLogFull)) {
      if (c->log_size + total <= d.log_cap) {
        const unsigned long long s = c->log_steps;
        if (s == 0) c->log_first = k;
        d.log_off[s + 1] = c->log_size + total;
        c->log_size += total;
        c->log_steps = s + 1;
        ok = 1u;
      } else {
        atomicOr(&c->status, kErrLogFull);
      }
    }
    c->log_ok[k & 3] = ok;
  }
}

// ---------------------------------------------------------------------------
// Kernel 2: one warp per spike j (grid-stride over the step's spikes). The
// warp walks j's CSR row — coalesced 16-byte loads of column indices and
// weights, int64 fixed-point atomicAdd into each target's delay slot, LTP
// fused into the walk (engine.rs:414-473, :496-537) — and j's plastic
// incoming list (LTD for synapses whose source did not spike). Both lists are
// walked in 128-entry chunks whose loads are all issued before any use, so a
// spike costs about four dependent memory round trips. Writes are disjoint:
// row synapses of spiking sources (LTP, and LTP then LTD when the target
// spiked too) versus incoming synapses of spiking targets whose source did
// not spike (LTD). The spike's own bookkeeping (ordered log entry, last spike
// step, trace bump) is done by the same warp.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_w4(const NsDev& d, bool bf16, uint64_t e0, float w[4]) {
  if (bf16) {
    const uint2 raw = *reinterpret_cast<const uint2*>(d.w16 + e0);
    w[0] = bf16_bits_to_f32((uint16_t)(raw.x & 0xffffu));
    w[1] = bf16_bits_to_f32((uint16_t)(raw.x >> 16));
    w[2] = bf16_bits_to_f32((uint16_t)(raw.y & 0xffffu));
    w[3] = bf16_bits_to_f32((uint16_t)(raw.y >> 16));
  } else {
    const float4 f = *reinterpret_cast<const float4*>(d.w32 + e0);
    w[0] = f.x; w[1] = f.y; w[2] = f.z; w[3] = f.w;
  }
}

__device__ __forceinline__ bool neg(float x) { return (__float_as_uint(x) >> 31) != 0u; }

// Spike list of step k as seen by the consumers: per-tile offsets in shared
// memory (exclusive scan of the tile counts) or, for networks of more than
// kSmemTiles tiles, the scan the neuron kernel's last tile wrote.
struct SpikeView {
  const uint32_t* spk;
  const uint32_t* toff;
  uint32_t ntiles;
  __device__ __forceinline__ uint32_t at(uint32_t rank) const {
    uint32_t lo = 0, hi = ntiles;   // largest t with toff[t] <= rank
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (toff[mid] <= rank) lo = mid; else hi = mid;
    }
    return __ldg(spk + (uint64_t)lo * kTile + (rank - toff[lo]));
  }
};

__device__ __forceinline__ SpikeView spike_view(const NsDev& d, uint64_t k, uint32_t cnt,
                                                uint32_t* s_toff) {
  const uint32_t par_k = (uint32_t)(k & 1);
  const uint32_t* tcnt = d.tile_cnt + par_k * (d.ntiles + 1);
  const bool small = d.ntiles <= kSmemTiles;
  if (small && cnt) block_scan_u32(tcnt, s_toff, d.ntiles);
  __syncthreads();
  SpikeView v;
  v.spk = d.spk + par_k * d.n_pad;
  v.toff = small ? s_toff : d.tile_off + par_k * (d.ntiles + 1);
  v.ntiles = d.ntiles;
  return v;
}


// Per-step context shared by the consumers of the spike list.
struct StepCtx {
  uint64_t k;
  uint32_t slot, cnt;
  bool stdp, homeo, log_ok;
  unsigned long long log_base;
  const float2* rec_k;
};

__device__ __forceinline__ StepCtx step_ctx(const NsDev& d, uint32_t jstep) {
  StepCtx c;
  c.k = d.ctl->step_base + jstep;
  c.slot = (uint32_t)(c.k % d.D);
  c.cnt = (uint32_t)d.ctl->step_spikes[c.k & 3];
  c.stdp = d.stdp != 0;
  c.homeo = d.homeo != 0;
  c.rec_k = d.rec + (c.k & 1) * d.n_pad;
  c.log_ok = d.ctl->log_ok[c.k & 3] != 0u;
  c.log_base = c.log_ok ? d.ctl->log_size - c.cnt : 0ull;
  return c;
}

// Value to store for a synapse whose weight this step's STDP set to w1 (a
// plain weight): w1 in the consolidation frame of step k; or, when the walks
// apply the reward (mode 1) to a synapse with an eligibility trace, the
// weight after the step's consolidation and reward, in the frame of step k+1
// (engine.rs:539-561). The reward changes a weight only where e != 0 or the
// weight lies outside [rstdp_w_min, rstdp_w_max] (elsewhere clamp(w + 0) is
// w). ev: the synapse's eligibility, zeroed when the reward is applied.
template <bool BF16>
__device__ __forceinline__ float ext_store(const NsDev& d, const float* fr, uint32_t mode, float w1,
                                           bool el, float& ev) {
  if (mode == 1u && el) {
    float u1 = d.cons ? (w1 - fr[1]) * fr[2] : w1;
    if (BF16) u1 = bf16_bits_to_f32(f32_to_bf16_bits(u1));
    float x = d.cons ? u1 * fr[3] + fr[4] : u1;
    if (ev != 0.0f || x < d.rw_min || x > d.rw_max) {
      x = clampw(x + fr[6] * ev, d.rw_min, d.rw_max);
      ev = 0.0f;
      return d.cons ? (x - fr[4]) * fr[5] : x;
    }
    return u1;
  }
  return d.cons ? (w1 - fr[1]) * fr[2] : w1;
}

// Deferred LTD. The source's pre trace at step astep + t is its value ps
// after step astep times exp(-dt/tau+) t times, one float rounding per
// multiply: the chain the neuron kernel runs. chain_fill computes it once per
// row, converged across the warp: lane i keeps x_(i+1) in the warp's table
// in shared memory (t = 1 .. min(T, 32)); returns x_min(T, 32).
__device__ __forceinline__ float* warp_chain_table() {
  __shared__ float s_chain[8][32];   // 256-thread blocks: one row of 32 per warp
  return s_chain[threadIdx.x >> 5];
}

__device__ __forceinline__ float chain_fill(const NsDev& d, float ps, uint32_t T, int lane, float* xs) {
  __syncwarp();
  const uint32_t Tc = T < 32u ? T : 32u;
  float x = ps, mine = 0.0f;
  for (uint32_t i = 0; i < Tc; ++i) {
    x = x * d.ep;
    if ((uint32_t)lane == i) mine = x;
  }
  xs[lane] = mine;
  __syncwarp();
  return x;
}

// The pending LTDs of one lane's four synapses: pb[q] holds, for synapse q,
// the bits (b = steps before the current one) of its target's spikes whose
// LTD has not been applied; T = current step - astep, xs the row's chain
// table. Each LTD is the eager one, w = clamp(w - A- pre), stored (BF16:
// rounded) before the next, in step order (highest bit first).
template <bool BF16>
__device__ __forceinline__ void apply_pending(const NsDev& d, const float* xs, uint32_t T,
                                              const uint32_t pb[4], float w[4]) {
  uint32_t U = pb[0] | pb[1] | pb[2] | pb[3];
  while (U) {
    const uint32_t b = 31u - __clz(U);   // step k - b = astep + (T - b)
    const float dm = d.neg_a_minus * xs[T - b - 1u];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if ((pb[q] >> b) & 1u) {
        float y = clampw(w[q] + dm, d.w_min, d.w_max);
        if (BF16) y = bf16_bits_to_f32(f32_to_bf16_bits(y));
        w[q] = y;
      }
    }
    U &= ~(1u << b);
  }
}

// Bits b in [lo, T-1] of a 32-step spike history whose chain index T - b - 1
// lies in the 32-entry table (b >= T - 32). T never exceeds 32 when every
// row is flushed every 32 steps; should it, the older bits are dropped here
// and the walk records kErrDeferWindow.
__device__ __forceinline__ uint32_t pending_mask(uint32_t T, uint32_t lo) {
  if (T > 32u) {
    if (T >= 64u) return 0u;
    lo = lo > T - 32u ? lo : T - 32u;
  }
  const uint32_t m = T >= 32u ? 0xffffffffu : ((1u << T) - 1u);
  return m & ~((1u << lo) - 1u);
}

// Row walk of spiking source j (the item-th spike of the step): bookkeeping
// (log entry, last spike step, trace bump), then the CSR row in 128-entry
// chunks: accumulation into the delay slot and LTP (LTP then LTD when the
// target spiked in this step too). DEFER: the row's pending LTDs (its
// targets' spikes since the row was last walked or flushed) are applied
// first, so that delivery reads the weight the eager schedule would.
template <bool COND, bool BF16, bool EXT, bool DEFER = false>
__device__ __forceinline__ void row_item(const NsDev& d, const StepCtx& c, uint32_t item, uint32_t j,
                                         int lane, unsigned long long& ev, uint32_t& outs) {
  const bool STDP = c.stdp, HOMEO = c.homeo;
  const uint64_t k = c.k;
  // EXT: consolidation frame / reward of this step, eligibility, STP
  const float* fr = EXT ? d.ctl->frame[k & 1] : nullptr;
  const uint32_t mode = EXT ? d.ctl->mode[k & 1] : 0u;
  const uint64_t beg = __ldg(d.row_ptr + j), end = __ldg(d.row_ptr + j + 1);
  const uint8_t rp = STDP ? __ldg(d.row_plastic + j) : 0;
  const uint8_t rt = COND ? __ldg(d.row_type + j) : 0;
  float pj = 0.0f;
  uint2 ls = make_uint2(0u, 0u);
  if (lane == 0) {
    // every load of the spike's bookkeeping is issued before any of its
    // stores: the compiler cannot move a load past a store through another
    // pointer, and a store-load order here costs a memory round trip each
    const long long lst = d.last[j];
    const uint8_t isout = d.outp[j];
    float2 rj = make_float2(0.f, 0.f);
    float pdec = 0.f;
    if (STDP) {
      rj = c.rec_k[j];
      if (DEFER) {
        pdec = d.pre[j];
        ls = d.lstart[j];
      }
    }
    const long long dk = lst < 0 ? -1 : (long long)k - lst;
    float fp = 0.f, fm = 0.f;
    if (STDP) {
      fp = (dk >= 0 && (unsigned long long)dk < d.Kp) ? d.Ep[dk] : 0.0f;
      fm = (dk >= 0 && (unsigned long long)dk < d.Km) ? d.Em[dk] : 0.0f;
    }
    if (c.log_ok) d.log_idx[c.log_base + item] = j;
    ev += end - beg;
    outs += isout ? 1u : 0u;
    d.last[j] = (long long)k;
    if (STDP) {
      // spike-time trace bump: trace * exp(-(t - t_last)/tau) + 1; the
      // decayed pre trace is the record's |x| (eager) or the trace the
      // neuron kernel wrote this step (deferred: the record holds spike bits)
      pj = (DEFER ? pdec : fabsf(rj.x)) * fp + 1.0f;
      d.pre[j] = pj;
      d.post[j] = fabsf(rj.y) * fm + 1.0f;
      if (DEFER) d.lstart[j] = make_uint2(__float_as_uint(pj), (uint32_t)k);
    }
  }
  // deferred LTD: lane 0 holds the row's trace start; it is broadcast in
  // the chunk loop after the chunk's loads and gathers are issued, so that
  // they do not wait for lane 0's loads
  const unsigned long long tbase = d.trace_pos ? d.trace_off[item] : 0ull;
  const uint64_t rb = beg & ~3ull;
  const uint32_t nrow = end > beg ? (uint32_t)((end - rb + 127) >> 7) : 0u;
  for (uint32_t ch = 0; ch < nrow; ++ch) {
    const uint64_t e0 = rb + 128ull * ch + 4ull * lane;
    const bool rv = e0 < end && e0 + 4 > beg;
    uint4 c4 = make_uint4(0u, 0u, 0u, 0u);
    float w[4] = {0.f, 0.f, 0.f, 0.f};
    if (rv) {
      c4 = __ldg(reinterpret_cast<const uint4*>(d.col + e0));
      load_w4(d, BF16, e0, w);
      if (EXT && d.cons) {
        const float A0 = fr[0], B0 = fr[1];
#pragma unroll
        for (int q = 0; q < 4; ++q) w[q] = w[q] * A0 + B0;
      }
    }
    const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
    bool inr[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) inr[q] = rv && (e0 + q >= beg) && (e0 + q < end);
    // target records for LTP, gathered before the atomics are issued
    bool pl[4] = {false, false, false, false};
    float tq[4];
    uint32_t pb[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      pl[q] = STDP && rp && inr[q] && (rp == 1 || __ldg(d.plastic + e0 + q));
      if (DEFER) {
        const float2 r = pl[q] ? c.rec_k[cc[q]] : make_float2(0.f, 0.f);
        tq[q] = r.y;
        pb[q] = __float_as_uint(r.x);
      } else {
        tq[q] = pl[q] ? c.rec_k[cc[q]].y : 0.f;
      }
    }
    if (DEFER && STDP && rp) {
      // the row's pending-bit mask: steps astep+1 .. k-1 (step k's LTD is
      // the same-step one below, with pj); the chain table once per row
      const uint32_t dT = __shfl_sync(0xffffffffu, (uint32_t)k - ls.y, 0);
      if (dT > 32u && ch == 0 && lane == 0) atomicOr(&d.ctl->status, kErrDeferWindow);
      float* xs = warp_chain_table();
      if (ch == 0) chain_fill(d, __uint_as_float(__shfl_sync(0xffffffffu, ls.x, 0)), dT, lane, xs);
      const uint32_t dmask = pending_mask(dT, 1u);
#pragma unroll
      for (int q = 0; q < 4; ++q) pb[q] &= dmask;
      apply_pending<BF16>(d, xs, dT, pb, w);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (!inr[q]) continue;
      const uint64_t e = e0 + q;
      int ty = 0;
      if (COND) ty = (rt == 255) ? (int)__ldg(d.type + e) : (int)rt;
      float val = (COND && (ty == 1 || ty == 2)) ? fabsf(w[q]) : w[q];
      // short-term plasticity: one step of a copy of the synapse's state
      // scales the delivered current (engine.rs:457-463)
      if (EXT && !COND && d.stp_f) val = val * __ldg(d.stp_f + e);
      atomicAdd(d.acc + ((uint64_t)ty * d.D + c.slot) * d.n_pad + cc[q],
                (unsigned long long)to_fix(val));
      if (d.inbits)
        atomicOr(d.inbits + (uint64_t)c.slot * (d.n_pad >> 5) + (cc[q] >> 5), 1u << (cc[q] & 31));
      if (d.trace_pos) {
        const unsigned long long tp = tbase + (e - beg);
        if (tp < d.trace_cap) d.trace_pos[tp] = e;
      }
      if (HOMEO) {
        float mag;
        if (COND) {
          float g = w[q] * kSyn[ty].gmax;
          if (kSyn[ty].mg) g = g * (1.0f / (1.0f + (1.0f / 3.57f) * expf(-0.062f * d.v[cc[q]])));
          mag = fabsf(g);
        } else {
          mag = fabsf(val);
        }
        d.contrib[e] = d.contrib[e] * d.cd + mag * d.one_m_cd;
      }
    }
    if (STDP && rp) {
      pj = __shfl_sync(0xffffffffu, pj, 0);
      float wn[4];
      bool chg = false, all4 = true;
      // eligibility traces of the plastic synapses that carry one
      bool el[4] = {false, false, false, false};
      float evl[4] = {0.f, 0.f, 0.f, 0.f};
      if (EXT && d.rstdp && (pl[0] | pl[1] | pl[2] | pl[3])) {
        if (d.elig_all) {
          el[0] = pl[0]; el[1] = pl[1]; el[2] = pl[2]; el[3] = pl[3];
        } else {
          const uchar4 f4 = *reinterpret_cast<const uchar4*>(d.elig_flag + e0);
          el[0] = pl[0] && f4.x; el[1] = pl[1] && f4.y; el[2] = pl[2] && f4.z; el[3] = pl[3] && f4.w;
        }
        if (el[0] | el[1] | el[2] | el[3]) {
          const float4 v4 = *reinterpret_cast<const float4*>(d.elig + e0);
          evl[0] = v4.x; evl[1] = v4.y; evl[2] = v4.z; evl[3] = v4.w;
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        wn[q] = w[q];
        if (!pl[q]) { all4 = false; continue; }
        const float dp = d.a_plus * fabsf(tq[q]);
        float w1 = clampw(w[q] + dp, d.w_min, d.w_max);
        if (EXT && el[q]) evl[q] = evl[q] * d.ce + dp;   // EligibilityTrace::update, engine.rs:519-522
        if (neg(tq[q])) {
          const float dm = d.neg_a_minus * pj;
          w1 = clampw(w1 + dm, d.w_min, d.w_max);
          if (EXT && el[q]) evl[q] = evl[q] * d.ce + dm;  // engine.rs:531-533
        }
        wn[q] = EXT ? ext_store<BF16>(d, fr, mode, w1, el[q], evl[q]) : w1;
        chg = true;
      }
      if (EXT && (el[0] | el[1] | el[2] | el[3])) {
        if (el[0] & el[1] & el[2] & el[3]) {
          *reinterpret_cast<float4*>(d.elig + e0) = make_float4(evl[0], evl[1], evl[2], evl[3]);
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (el[q]) d.elig[e0 + q] = evl[q];
        }
      }
      if (chg) {
        if (BF16) {
          if (all4) {
            uint2 raw;
            raw.x = (uint32_t)f32_to_bf16_bits(wn[0]) | ((uint32_t)f32_to_bf16_bits(wn[1]) << 16);
            raw.y = (uint32_t)f32_to_bf16_bits(wn[2]) | ((uint32_t)f32_to_bf16_bits(wn[3]) << 16);
            *reinterpret_cast<uint2*>(d.w16 + e0) = raw;
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (pl[q]) d.w16[e0 + q] = f32_to_bf16_bits(wn[q]);
          }
        } else {
          if (all4) {
            *reinterpret_cast<float4*>(d.w32 + e0) = make_float4(wn[0], wn[1], wn[2], wn[3]);
          } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (pl[q]) d.w32[e0 + q] = wn[q];
          }
        }
      }
    }
  }
}

// LTD over the plastic incoming synapses of spiking target j whose source did
// not spike (those whose source spiked are handled by the source's row walk).
template <bool BF16, bool EXT>
__device__ __forceinline__ void ltd_item(const NsDev& d, const StepCtx& c, uint32_t j, int lane) {
  const float* fr = EXT ? d.ctl->frame[c.k & 1] : nullptr;
  const uint32_t mode = EXT ? d.ctl->mode[c.k & 1] : 0u;
  const uint64_t ib = __ldg(d.in_ptr + j), ie = __ldg(d.in_ptr + j + 1);
  for (uint64_t q0 = ib; q0 < ie; q0 += 128) {
    uint2 sp[4];
    bool act[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint64_t q = q0 + lane + 32u * u;
      act[u] = q < ie;
      sp[u] = act[u] ? __ldg(d.in_list + q) : make_uint2(0u, 0u);
    }
    float pre[4], wv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      pre[u] = act[u] ? c.rec_k[sp[u].x].x : 0.0f;
      if (BF16) wv[u] = act[u] ? bf16_bits_to_f32(d.w16[sp[u].y]) : 0.0f;
      else wv[u] = act[u] ? d.w32[sp[u].y] : 0.0f;
      if (EXT && d.cons) wv[u] = wv[u] * fr[0] + fr[1];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (!act[u] || neg(pre[u])) continue;
      const float dm = d.neg_a_minus * pre[u];
      const float w1 = clampw(wv[u] + dm, d.w_min, d.w_max);
      float st = w1;
      if (EXT) {
        const uint32_t pos = sp[u].y;
        const bool el = d.rstdp && (d.elig_all || d.elig_flag[pos]);
        float evq = el ? d.elig[pos] : 0.0f;
        if (el) evq = evq * d.ce + dm;   // EligibilityTrace::update, engine.rs:531-533
        st = ext_store<BF16>(d, fr, mode, w1, el, evq);
        if (el) d.elig[pos] = evq;
      }
      if (BF16) d.w16[sp[u].y] = f32_to_bf16_bits(st);
      else d.w32[sp[u].y] = st;
    }
  }
}

// Flush of source j's row (deferred LTD): applies the LTDs of its targets'
// spikes at steps astep+1 .. k (a target that spikes at step k while j does
// not included, as the eager LTD walk of step k would) and moves the row's
// trace start to step k. The row of a source that spikes at step k is left
// to that step's row walk. Only the synapses of row j are written (a 4-entry
// group that reaches into a neighbouring row is written entry by entry).
template <bool BF16>
__device__ __forceinline__ void flush_row(const NsDev& d, uint64_t k, const float2* rec_k, uint32_t j,
                                          int lane) {
  // the row's metadata in one round trip (independent loads)
  const uint8_t rp = __ldg(d.row_plastic + j);
  const uint32_t hj = __float_as_uint(rec_k[j].x);
  const uint2 ls = d.lstart[j];
  const uint64_t beg = __ldg(d.row_ptr + j), end = __ldg(d.row_ptr + j + 1);
  if (!rp || (hj & 1u)) return;
  const uint32_t T = (uint32_t)k - ls.y;
  if (T == 0u) return;
  if (T > 32u && lane == 0) atomicOr(&d.ctl->status, kErrDeferWindow);
  const uint32_t mask = pending_mask(T, 0u);
  // the chain table; xT, the pre trace at step k, is the row's new start
  float* xs = warp_chain_table();
  const float xT = chain_fill(d, __uint_as_float(ls.x), T, lane, xs);
  const uint64_t rb = beg & ~3ull;
  const uint32_t nrow = end > beg ? (uint32_t)((end - rb + 127) >> 7) : 0u;
  for (uint32_t ch = 0; ch < nrow; ++ch) {
    const uint64_t e0 = rb + 128ull * ch + 4ull * lane;
    if (!(e0 < end && e0 + 4 > beg)) continue;
    const uint4 c4 = __ldg(reinterpret_cast<const uint4*>(d.col + e0));
    const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
    uint32_t pb[4];
    bool all4 = true;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint64_t e = e0 + q;
      const bool pl = e >= beg && e < end && (rp == 1 || __ldg(d.plastic + e));
      all4 = all4 && pl;
      pb[q] = pl ? (__float_as_uint(rec_k[cc[q]].x) & mask) : 0u;
    }
    if (!(pb[0] | pb[1] | pb[2] | pb[3])) continue;
    float w[4];
    load_w4(d, BF16, e0, w);
    apply_pending<BF16>(d, xs, T, pb, w);
    if (BF16) {
      if (all4) {
        uint2 raw;
        raw.x = (uint32_t)f32_to_bf16_bits(w[0]) | ((uint32_t)f32_to_bf16_bits(w[1]) << 16);
        raw.y = (uint32_t)f32_to_bf16_bits(w[2]) | ((uint32_t)f32_to_bf16_bits(w[3]) << 16);
        *reinterpret_cast<uint2*>(d.w16 + e0) = raw;
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (pb[q]) d.w16[e0 + q] = f32_to_bf16_bits(w[q]);
      }
    } else {
      if (all4) {
        *reinterpret_cast<float4*>(d.w32 + e0) = make_float4(w[0], w[1], w[2], w[3]);
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (pb[q]) d.w32[e0 + q] = w[q];
      }
    }
  }
  if (lane == 0) d.lstart[j] = make_uint2(__float_as_uint(xT), (uint32_t)k);
}

// Deferred LTD, step k: the flush of row block k mod 32 (rows
// [b * ceil(n/32), (b+1) * ceil(n/32))). Runs beside the row walks of step k
// (the rows of step k's spikers are skipped) and the neuron update of step
// k+1; the row walks of step k+1 wait for it.
//
// The grid is one block per task (flush_grid): short-lived blocks let the
// higher-priority neuron update and row walks take SMs as they free up.
// A block takes tasks of kFlushRows consecutive rows. First one thread per
// row reads the row's metadata, computes its pre-trace chain table into
// shared memory and moves its trace start to step k; then the block streams
// the task's contiguous CSR range, four positions per thread (coalesced
// column and weight loads), each position finding its row in the task's row
// pointers, gathering its target's spike bits and applying the pending LTDs
// with its row's table. Only changed weights are written, so a 4-entry group
// at a task's edge or over a spiking row touches nothing it does not own.
constexpr uint32_t kFlushRows = 16;

template <bool BF16>
__global__ void __launch_bounds__(256) k_flush(NsDev d, uint32_t jstep) {
  __shared__ float s_tab[kFlushRows][33];
  __shared__ uint64_t s_beg[kFlushRows + 1];
  __shared__ uint32_t s_T[kFlushRows], s_mask[kFlushRows];
  __shared__ uint8_t s_rp[kFlushRows];
  const uint64_t k = d.ctl->step_base + jstep;
  const float2* rec_k = d.rec + (k & 1) * d.n_pad;
  const uint64_t per = (d.n + 31) / 32;
  const uint64_t r0 = (k & 31u) * per;
  const uint64_t r1 = r0 + per < d.n ? r0 + per : d.n;
  const uint32_t tid = threadIdx.x;
  const uint64_t ntask = r1 > r0 ? (r1 - r0 + kFlushRows - 1) / kFlushRows : 0;
  for (uint64_t task = blockIdx.x; task < ntask; task += gridDim.x) {
    const uint64_t ja = r0 + task * kFlushRows;
    const uint32_t nrows = (uint32_t)(ja + kFlushRows <= r1 ? kFlushRows : r1 - ja);
    // ---- phase 1: one thread per row ----
    uint32_t live = 0u;
    if (tid < nrows) {
      const uint64_t j = ja + tid;
      const uint8_t rp = __ldg(d.row_plastic + j);
      const uint32_t hj = __float_as_uint(rec_k[j].x);
      const uint2 ls = d.lstart[j];
      s_beg[tid] = __ldg(d.row_ptr + j);
      uint32_t T = (rp && !(hj & 1u)) ? (uint32_t)k - ls.y : 0u;
      if (T > 32u) atomicOr(&d.ctl->status, kErrDeferWindow);
      s_T[tid] = T;
      s_mask[tid] = T ? pending_mask(T, 0u) : 0u;
      s_rp[tid] = rp;
      if (T) {
        float x = __uint_as_float(ls.x);
        const uint32_t Tc = T < 32u ? T : 32u;
        for (uint32_t i = 0; i < Tc; ++i) {
          x = x * d.ep;
          s_tab[tid][i] = x;
        }
        d.lstart[j] = make_uint2(__float_as_uint(x), (uint32_t)k);
        live = 1u;
      }
    }
    if (tid == 0) s_beg[nrows] = __ldg(d.row_ptr + ja + nrows);
    if (!__syncthreads_or(live)) continue;
    // ---- phase 2: the task's positions, four per thread ----
    const uint64_t pa = s_beg[0], pb_end = s_beg[nrows];
    for (uint64_t e0 = (pa & ~3ull) + 4ull * tid; e0 < pb_end; e0 += 4ull * blockDim.x) {
      // the row of the first position at or after pa in this group
      const uint64_t ef = e0 < pa ? pa : e0;
      uint32_t lo = 0, hi = nrows;      // largest t with s_beg[t] <= ef
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s_beg[mid] <= ef) lo = mid; else hi = mid;
      }
      const uint4 c4 = __ldg(reinterpret_cast<const uint4*>(d.col + e0));
      const uint32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
      uint32_t pb[4] = {0u, 0u, 0u, 0u};
      uint32_t tq[4] = {0u, 0u, 0u, 0u};
      uint32_t t = lo;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint64_t e = e0 + q;
        if (e < pa || e >= pb_end) continue;
        while (t + 1 < nrows && s_beg[t + 1] <= e) ++t;
        tq[q] = t;
        if (!s_T[t]) continue;
        if (s_rp[t] != 1 && !__ldg(d.plastic + e)) continue;
        pb[q] = __float_as_uint(rec_k[cc[q]].x) & s_mask[t];
      }
      if (!(pb[0] | pb[1] | pb[2] | pb[3])) continue;
      float w[4];
      load_w4(d, BF16, e0, w);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t U = pb[q];
        if (!U) continue;
        const uint32_t T = s_T[tq[q]];
        const float* xs = s_tab[tq[q]];
        float y = w[q];
        while (U) {
          const uint32_t b = 31u - __clz(U);
          y = clampw(y + d.neg_a_minus * xs[T - b - 1u], d.w_min, d.w_max);
          if (BF16) y = bf16_bits_to_f32(f32_to_bf16_bits(y));
          U &= ~(1u << b);
        }
        if (BF16) d.w16[e0 + q] = f32_to_bf16_bits(y);
        else d.w32[e0 + q] = y;
      }
    }
    __syncthreads();
  }
}

// Deferred LTD: every row flushed to the last completed step (before the
// host reads or replaces weights, or an eager step runs).
template <bool BF16>
__global__ void __launch_bounds__(256) k_defer_flush_all(NsDev d) {
  const uint64_t k = d.ctl->step_base - 1;
  const float2* rec_k = d.rec + (k & 1) * d.n_pad;
  const int lane = threadIdx.x & 31;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t j = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); j < d.n; j += nw)
    flush_row<BF16>(d, k, rec_k, (uint32_t)j, lane);
}

// Deferred LTD from a state with none pending (after uploads and eager
// steps): every row's trace start is the pre trace after the last completed
// step.
__global__ void k_defer_sync(NsDev d) {
  const uint32_t k1 = (uint32_t)(d.ctl->step_base - 1);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < d.n;
       i += (uint64_t)gridDim.x * blockDim.x)
    d.lstart[i] = make_uint2(__float_as_uint(d.pre[i]), k1);
}

__device__ __forceinline__ void flush_counters(const NsDev& d, uint64_t k, unsigned long long ev,
                                               uint32_t outs, unsigned long long* s_ev,
                                               uint32_t* s_out) {
  const int lane = threadIdx.x & 31;
  for (int o = 16; o > 0; o >>= 1) {
    ev += __shfl_down_sync(0xffffffffu, ev, o);
    outs += __shfl_down_sync(0xffffffffu, outs, o);
  }
  if (lane == 0 && (ev | outs)) {
    atomicAdd(s_ev, ev);
    atomicAdd(s_out, outs);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (*s_ev) atomicAdd(&d.ctl->events_total, *s_ev);
    if (*s_out) {
      atomicAdd(&d.ctl->out_total, (unsigned long long)*s_out);
      atomicAdd(&d.ctl->outs[k & 3], (unsigned long long)*s_out);
    }
  }
}

// Kernel 2 (fused schedule): row walks [0, cnt) and LTD lists [cnt, 2 cnt)
// as warp work items of one grid-stride kernel.
template <bool COND, bool BF16, int MINB, bool EXT>
__global__ void __launch_bounds__(256, MINB) k_prop_fused(NsDev d, uint32_t jstep) {
  __shared__ uint32_t s_toff[kSmemTiles + 1];
  __shared__ unsigned long long s_ev;
  __shared__ uint32_t s_out;
  const int lane = threadIdx.x & 31;
  const StepCtx c = step_ctx(d, jstep);
  if (threadIdx.x == 0) { s_ev = 0ull; s_out = 0u; }
  const SpikeView sv = spike_view(d, c.k, c.cnt, s_toff);
  const uint32_t items = c.stdp ? 2u * c.cnt : c.cnt;
  const uint32_t wglob = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  unsigned long long ev = 0ull;
  uint32_t outs = 0u;
  for (uint32_t item = wglob; item < items; item += nw) {
    const uint32_t rank = item < c.cnt ? item : item - c.cnt;
    const uint32_t j = sv.at(rank);
    if (item < c.cnt) row_item<COND, BF16, EXT>(d, c, item, j, lane, ev, outs);
    else ltd_item<BF16, EXT>(d, c, j, lane);
  }
  flush_counters(d, c.k, ev, outs, &s_ev, &s_out);
}

// Kernel 2a / 2b (split schedule): the row walks, then the LTD lists on a
// second stream beside the next step's neuron kernel.
template <bool COND, bool BF16, bool EXT, bool DEFER = false>
__global__ void __launch_bounds__(256, 4) k_rows(NsDev d, uint32_t jstep) {
  __shared__ uint32_t s_toff[kSmemTiles + 1];
  __shared__ unsigned long long s_ev;
  __shared__ uint32_t s_out;
  const int lane = threadIdx.x & 31;
  const StepCtx c = step_ctx(d, jstep);
  if (threadIdx.x == 0) { s_ev = 0ull; s_out = 0u; }
  const SpikeView sv = spike_view(d, c.k, c.cnt, s_toff);
  const uint32_t wglob = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  unsigned long long ev = 0ull;
  uint32_t outs = 0u;
  for (uint32_t item = wglob; item < c.cnt; item += nw)
    row_item<COND, BF16, EXT, DEFER>(d, c, item, sv.at(item), lane, ev, outs);
  flush_counters(d, c.k, ev, outs, &s_ev, &s_out);
}

template <bool BF16, bool EXT>
__global__ void __launch_bounds__(256, 5) k_ltd(NsDev d, uint32_t jstep) {
  __shared__ uint32_t s_toff[kSmemTiles + 1];
  const int lane = threadIdx.x & 31;
  const StepCtx c = step_ctx(d, jstep);
  const SpikeView sv = spike_view(d, c.k, c.cnt, s_toff);
  const uint32_t wglob = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t item = wglob; item < c.cnt; item += nw) ltd_item<BF16, EXT>(d, c, sv.at(item), lane);
}

// ---------------------------------------------------------------------------
// Kernel 2c (R-STDP / consolidation): after the step's walks. Mode 2: the
// reward of engine.rs:546-561 over every synapse with an eligibility trace,
// in the frame of step k+1 (changing only weights it moves). Renormalisation:
// when A_k+1 < 2^-16 every stored value becomes its plain weight and the
// frame of step k+1 the identity (the last block records it). Returns at once
// in every other step.
// ---------------------------------------------------------------------------
template <bool BF16>
__global__ void __launch_bounds__(256) k_tail(NsDev d, uint32_t jstep) {
  const unsigned long long k = d.ctl->step_base + jstep;
  const uint32_t mode = d.ctl->mode[k & 1];
  const bool renorm = d.cons && d.ctl->consA[k & 1] * d.cons_a < 0x1p-16;
  if (mode != 2u && !renorm) return;
  const float* fr = d.ctl->frame[k & 1];
  const float A1 = fr[3], B1 = fr[4], iA1 = fr[5], lrr = fr[6];
  const bool cons = d.cons != 0;
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < d.m;
       s += (uint64_t)gridDim.x * blockDim.x) {
    const bool ap = mode == 2u && d.elig_flag[s];
    if (!ap && !renorm) continue;
    float x = BF16 ? bf16_bits_to_f32(d.w16[s]) : d.w32[s];
    if (cons) x = x * A1 + B1;
    bool chg = false;
    if (ap) {
      const float evq = d.elig[s];
      if (evq != 0.0f || x < d.rw_min || x > d.rw_max) {
        x = clampw(x + lrr * evq, d.rw_min, d.rw_max);
        d.elig[s] = 0.0f;
        chg = true;
      }
    }
    if (renorm || chg) {
      const float st = (renorm || !cons) ? x : (x - B1) * iA1;
      if (BF16) d.w16[s] = f32_to_bf16_bits(st);
      else d.w32[s] = st;
    }
  }
  if (renorm) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned done = atomicAdd(&d.ctl->tail_done, 1u);
      if (done == gridDim.x - 1) {
        __threadfence();
        Ctl* c = d.ctl;
        c->cons_k0 = k + 1;
        c->frame[k & 1][3] = 1.0f;
        c->frame[k & 1][4] = 0.0f;
        c->frame[k & 1][5] = 1.0f;
        c->tail_done = 0u;
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
  // weights in the consolidation frame of step k+1 (identity without it)
  const unsigned long long kst = d.ctl->step_base + jstep;
  const bool cons = d.cons != 0;
  const float A1 = cons ? d.ctl->frame[kst & 1][3] : 1.0f;
  const float B1 = cons ? d.ctl->frame[kst & 1][4] : 0.0f;
  const float iA1 = cons ? d.ctl->frame[kst & 1][5] : 1.0f;
  // one thread per target; sums in ascending CSR position, as the reference
  // walks synapses_by_target (engine.rs:86-92)
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < d.n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double rate = d.rate[i];
    const double err = rate - d.h_target;
    const uint64_t b = d.all_in_ptr[i], e = d.all_in_ptr[i + 1];
    double sum = 0.0;
    for (uint64_t q = b; q < e; ++q) sum += (double)d.contrib[d.all_in_pos[q]];
    const uint64_t cnt = e - b;
    if (cnt > 0 && sum >= 1e-12) {
      const double mean = sum / (double)cnt;
      const float nerr = (float)(-err);
      for (uint64_t q = b; q < e; ++q) {
        const uint32_t s = d.all_in_pos[q];
        const float rel = (float)((double)d.contrib[s] / mean);
        const float arg = nerr * rel * d.dt_f / d.h_tau_f;
        const float scale = exp_f(arg);
        float u = BF16 ? bf16_bits_to_f32(d.w16[s]) : d.w32[s];
        if (cons) u = u * A1 + B1;
        float w = clampw(u * scale, 0.0f, 10.0f);
        if (cons) w = (w - B1) * iA1;
        if (BF16) d.w16[s] = f32_to_bf16_bits(w);
        else d.w32[s] = w;
      }
    }
    const double inst = bit_of(d.bitmap, (uint32_t)i) ? 1000.0 / d.dt : 0.0;
    d.rate[i] = rate + (inst - rate) * d.dt / 100.0;
  }
}

// ---------------------------------------------------------------------------
// The firing-rate estimate without homeostasis (engine.rs:637-642, FP64):
// the update k_homeostasis makes after its scaling, from this step's bitmap.
__global__ void __launch_bounds__(256) k_rates(NsDev d) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < d.n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const double rate = d.rate[i];
    const double inst = bit_of(d.bitmap, (uint32_t)i) ? 1000.0 / d.dt : 0.0;
    d.rate[i] = rate + (inst - rate) * d.dt / 100.0;
  }
}

// Single-network sharding (one rank per GPU, neurons split by tiles): after
// the step's spike bitmap words of every rank have been gathered, one block
// per tile of the other ranks ("ghost" tiles) rebuilds what the owner's
// neuron kernel produced for it: the tile's ascending spike list and count,
// and its neurons' decayed traces with the spike sign (the same float
// operations as the owner). The tiles count on with the neuron kernel's
// counter, so the last block to finish does the step's bookkeeping exactly
// as the neuron kernel's last tile does without sharding.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_shard_merge(NsDev d, uint32_t jstep) {
  __shared__ uint32_t s_wsum[kThreads / 32];
  __shared__ uint32_t s_total;
  __shared__ int s_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint64_t k = d.ctl->step_base + jstep;
  const uint32_t par_k = (uint32_t)(k & 1);
  uint32_t* const spk_k = d.spk + par_k * d.n_pad;
  uint32_t* const tcnt_k = d.tile_cnt + par_k * (d.ntiles + 1);
  float2* const rec_k = d.rec + par_k * d.n_pad;
  // ghost tile of this block: the tiles outside [tile0, tile0 + tiles_own)
  const uint32_t tile = blockIdx.x < d.tile0 ? blockIdx.x : blockIdx.x + d.tiles_own;
  const uint64_t base = (uint64_t)tile * kTile;
  constexpr int kWords = kTile / 32;                 // bitmap words of a tile
  static_assert(kWords <= kThreads, "one word per thread");
  const uint32_t wbits = tid < kWords ? d.bitmap[(base >> 5) + tid] : 0u;
  // ascending list: exclusive scan of the words' popcounts
  const uint32_t c = __popc(wbits);
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_wsum[warp] = incl;
  __syncthreads();
  uint32_t woff = 0, tot = 0;
#pragma unroll
  for (int q = 0; q < kThreads / 32; ++q) {
    const uint32_t v = s_wsum[q];
    woff += q < warp ? v : 0u;
    tot += v;
  }
  uint32_t o = woff + incl - c;
  for (uint32_t m = wbits; m; m &= m - 1u) spk_k[base + o++] = (uint32_t)(base + 32u * tid + __ffs(m) - 1);
  if (tid == 0) {
    tcnt_k[tile] = tot;
    s_total = tot;
  }
  // traces of the ghost neurons: per-step decay, sign bit = spiked
  if (d.stdp) {
    for (uint32_t q = tid; q < (uint32_t)kTile; q += kThreads) {
      const uint64_t i = base + q;
      const float pv = d.pre[i] * d.ep, qv = d.post[i] * d.em;
      d.pre[i] = pv;
      d.post[i] = qv;
      const bool sp = (d.bitmap[i >> 5] >> (i & 31)) & 1u;
      rec_k[i] = make_float2(sp ? -pv : pv, sp ? -qv : qv);
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (s_total) atomicAdd(&d.ctl->spk_acc[k & 3], (unsigned long long)s_total);
    __threadfence();
    const unsigned done = atomicAdd(&d.ctl->tiles_done, 1u);
    s_last = (done == d.ntiles - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (d.ntiles > kSmemTiles) block_scan_u32(tcnt_k, d.tile_off + par_k * (d.ntiles + 1), d.ntiles);
  if (tid == 0) {
    Ctl* cc = d.ctl;
    const unsigned long long total = atomicAdd(&cc->spk_acc[k & 3], 0ull);
    cc->spk_acc[(k + 2) & 3] = 0ull;
    cc->tiles_done = 0u;
    cc->step_spikes[k & 3] = total;
    if (total > cc->max_step_spikes) cc->max_step_spikes = total;
    cc->spikes_total += total;
    cc->sim_time += d.dt;
    unsigned ok = 0u;
    if (d.log_idx != nullptr && cc->log_steps < d.log_steps_cap && !(cc->status & kErrLogFull)) {
      if (cc->log_size + total <= d.log_cap) {
        const unsigned long long sl = cc->log_steps;
        if (sl == 0) cc->log_first = k;
        d.log_off[sl + 1] = cc->log_size + total;
        cc->log_size += total;
        cc->log_steps = sl + 1;
        ok = 1u;
      } else {
        atomicOr(&cc->status, kErrLogFull);
      }
    }
    cc->log_ok[k & 3] = ok;
  }
}

// The LFP term of the last completed step (reference conductance mode): the
// conductances and currents that the next step's neuron kernel will compute
// (same float operations), summed without consuming the delivered input.
__global__ void __launch_bounds__(256) k_lfp_pending(NsDev d, unsigned long long* out) {
  const uint64_t k = d.ctl->step_base;
  const uint32_t slot = (uint32_t)(k % d.D);
  long long acc = 0;
  // this rank's neurons (all of them without sharding)
  const uint64_t lo = (uint64_t)d.tile0 * kTile;
  const uint64_t hi = min((uint64_t)(d.tile0 + d.tiles_own) * kTile, d.n);
  for (uint64_t i = lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < hi;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float vi = d.v[i];
    float lf = 0.f;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const float S = ((d.type_mask >> t) & 1u)
                          ? from_fix((long long)d.acc[((uint64_t)t * d.D + slot) * d.n_pad + i]) : 0.f;
      float inc = S * kSyn[t].gmax;
      if (kSyn[t].mg && inc != 0.0f) inc = inc * (1.0f / (1.0f + (1.0f / 3.57f) * expf(-0.062f * vi)));
      const float g = d.G[t][i] * d.Gdec[t] + inc;
      lf = lf + fabsf(g * (kSyn[t].erev - vi));
    }
    acc += __float2ll_rn(lf * 0x1p24f);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, (unsigned long long)acc);
}

// Pending host stimulus: distinct neuron ids, values accumulated on the
// host in call order; they join the input current of the next step.
__global__ void k_stim_apply(NsDev d, const uint32_t* ids, const float* vals, uint32_t cnt) {
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x)
    d.stim[ids[q]] = d.stim[ids[q]] + vals[q];
  if (blockIdx.x == 0 && threadIdx.x == 0) d.ctl->stim_at = d.ctl->step_base + 1;
}

__global__ void k_advance(Ctl* ctl, uint32_t steps) { ctl->step_base += steps; }

// exclusive scan of out-degrees of this step's spikers in ascending order
// (traced step only): walks the tile-local lists in tile order
__global__ void k_trace_offsets(NsDev d, unsigned long long* off) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const uint32_t par_k = (uint32_t)(d.ctl->step_base & 1);
  unsigned long long run = 0;
  uint32_t q = 0;
  for (uint32_t t = 0; t < d.ntiles; ++t) {
    const uint32_t c = d.tile_cnt[par_k * (d.ntiles + 1) + t];
    for (uint32_t l = 0; l < c; ++l) {
      off[q++] = run;
      const uint32_t j = d.spk[par_k * d.n_pad + (uint64_t)t * kTile + l];
      run += d.row_ptr[j + 1] - d.row_ptr[j];
    }
  }
  off[q] = run;
}

}  // namespace ns
