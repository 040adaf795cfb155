// ORACLE — test infrastructure only (see oracle.h). CPU restatement of
// NeuralSim's step hot path. Built with -ffp-contract=off and without
// -ffast-math so every float operation rounds exactly once, as on the device.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11). Multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key bumps
// 0x9E3779B9 / 0xBB67AE85, ten rounds.
// ---------------------------------------------------------------------------
inline void philox(const uint32_t c_in[4], const uint32_t k_in[2], uint32_t out[4]) {
  uint32_t c0 = c_in[0], c1 = c_in[1], c2 = c_in[2], c3 = c_in[3];
  uint32_t k0 = k_in[0], k1 = k_in[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    if (r != 9) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Stream ids of the drive (shared specification with the device code).
constexpr uint32_t STREAM_DRIVE = 1;
constexpr uint32_t STREAM_KICKS = 2;

inline void draw(uint64_t seed, uint32_t idx, uint64_t step, uint32_t stream, uint32_t out[4]) {
  uint32_t c[4] = {idx, (uint32_t)step, (uint32_t)(step >> 32), stream};
  uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  philox(c, k, out);
}

// u in [0,1): 24 random bits, exact in float and double.
inline float unif_f(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }
inline double unif_d(uint32_t x) { return (double)(x >> 8) * 0x1p-24; }
// u in (0,1): odd multiples of 2^-24, exact.
inline float unif_open_f(uint32_t x) { return (float)((x >> 9) * 2u + 1u) * 0x1p-24f; }
inline double unif_open_d(uint32_t x) { return (double)((x >> 9) * 2u + 1u) * 0x1p-24; }

// ---------------------------------------------------------------------------
// Own float logarithm and sin/cos of 2*pi*u (used by the Gaussian drive so
// host and device agree bit for bit). Method: natural log by exponent split and
// the atanh series log(m) = 2(s + s^3/3 + s^5/5 + ...), s = (m-1)/(m+1), with m
// in [sqrt(1/2), sqrt(2)); sin/cos by quarter-turn reduction and Taylor
// polynomials on [-pi/4, pi/4]. Only + - * / on floats.
// ---------------------------------------------------------------------------
inline float own_logf(float x) {
  uint32_t b;
  std::memcpy(&b, &x, 4);
  int e = (int)((b >> 23) & 0xffu) - 127;
  uint32_t mb = (b & 0x7fffffu) | 0x3f800000u;
  float m;
  std::memcpy(&m, &mb, 4);
  if (m > 1.41421356f) { m = m * 0.5f; e = e + 1; }
  float f = m - 1.0f;
  float s = f / (2.0f + f);
  float z = s * s;
  float poly = 0.18181818f;                 // 2/11
  poly = 0.22222222f + z * poly;            // 2/9
  poly = 0.28571429f + z * poly;            // 2/7
  poly = 0.4f + z * poly;                   // 2/5
  poly = 0.66666667f + z * poly;            // 2/3
  float lm = (s + s) + (s * z) * poly;
  float ef = (float)e;
  return ef * 0.693145752f + (lm + ef * 1.42860677e-06f);
}

inline void own_sincos2pi(float u, float* sn, float* cs) {
  float t = u * 4.0f;
  float kf = std::floor(t + 0.5f);
  int k = (int)kf;
  float r = t - kf;
  float ph = r * 1.57079633f;
  float p2 = ph * ph;
  float sp = -2.50521084e-08f;              // -1/11!
  sp = 2.75573192e-06f + p2 * sp;           // 1/9!
  sp = -1.98412698e-04f + p2 * sp;          // -1/7!
  sp = 8.33333333e-03f + p2 * sp;           // 1/5!
  sp = -1.66666667e-01f + p2 * sp;          // -1/3!
  float s = ph + (ph * p2) * sp;
  float cp = 2.08767570e-09f;               // 1/12!
  cp = -2.75573192e-07f + p2 * cp;          // -1/10!
  cp = 2.48015873e-05f + p2 * cp;           // 1/8!
  cp = -1.38888889e-03f + p2 * cp;          // -1/6!
  cp = 4.16666667e-02f + p2 * cp;           // 1/4!
  cp = -0.5f + p2 * cp;                     // -1/2!
  float c = 1.0f + p2 * cp;
  switch (k & 3) {
    case 0: *sn = s; *cs = c; break;
    case 1: *sn = c; *cs = -s; break;
    case 2: *sn = -s; *cs = -c; break;
    default: *sn = -c; *cs = s; break;
  }
}

// e^x in float for the homeostatic scale: Cody-Waite reduction with a
// 16-bit head of ln2, Taylor series of e^r to r^7, scaling by 2^n.
inline float own_expf(float x) {
  if (x > 88.0f) x = 88.0f;
  if (x < -87.0f) x = -87.0f;
  const float nf = std::floor(x * 1.44269504f + 0.5f);
  float r = x - nf * 0.693145752f;
  r = r - nf * 1.42860677e-06f;
  float p = 1.98412698e-04f;
  p = 1.38888889e-03f + r * p;
  p = 8.33333333e-03f + r * p;
  p = 4.16666667e-02f + r * p;
  p = 1.66666667e-01f + r * p;
  p = 0.5f + r * p;
  p = 1.0f + r * p;
  p = 1.0f + r * p;
  const uint32_t eb = (uint32_t)((int)nf + 127) << 23;
  float sc;
  std::memcpy(&sc, &eb, 4);
  return p * sc;
}
template <class R> inline R scale_exp(R x) { return std::exp(x); }
template <> inline float scale_exp<float>(float x) { return own_expf(x); }

inline uint16_t f32_to_bf16_rne(float f) {
  uint32_t b;
  std::memcpy(&b, &f, 4);
  if ((b & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((b >> 16) | 0x40u);
  b += 0x7fffu + ((b >> 16) & 1u);
  return (uint16_t)(b >> 16);
}
inline float bf16_to_f32(uint16_t h) {
  uint32_t b = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &b, 4);
  return f;
}

// Synapse dynamics constants, src/synapse/types.rs:15-54.
struct SynDyn { double decay, erev, gmax; int mg; };
const SynDyn kDyn[4] = {
    {2.0, 0.0, 1.0, 0},      // AMPA
    {10.0, -70.0, 1.0, 0},   // GABA
    {150.0, -90.0, 0.5, 0},  // GABA-B
    {100.0, 0.0, 0.5, 1},    // NMDA
};
const double kRise[4] = {0.5, 1.0, 30.0, 2.0};

template <class R> inline R mg_block(int type, R v) {
  // nmda_mg_block, types.rs:88-94: 1 / (1 + [Mg]/3.57 * exp(-0.062 V)), [Mg] = 1 mM
  if (!kDyn[type].mg) return R(1);
  return R(1) / (R(1) + (R(1) / R(3.57)) * std::exp(R(-0.062) * v));
}

// Fixed point used by the float engine for synaptic sums (2^40 per unit).
inline int64_t to_fix(float w) { return (int64_t)std::llrint(w * 0x1p40f); }
inline float from_fix(int64_t a) { return (float)a * 0x1p-40f; }

template <class R> inline R clampw(R x, R lo, R hi) {
  // f64::clamp semantics for non-NaN input (plasticity.rs:41, engine.rs:515-528)
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}

// HH rate functions (hodgkin_huxley.rs:20-42) written with expm1 so the 0/0
// points at V = -40 (alpha_m) and V = -55 (alpha_n) take their limits.
template <class R> struct HHRates { R am, bm, ah, bh, an, bn; };
template <class R> inline HHRates<R> hh_rates(R v) {
  HHRates<R> r;
  R x = (v + R(40)) / R(10);
  r.am = (x == R(0)) ? R(1) : x / (-std::expm1(-x));
  r.bm = R(4) * std::exp(-(v + R(65)) / R(18));
  r.ah = R(0.07) * std::exp(-(v + R(65)) / R(20));
  r.bh = R(1) / (R(1) + std::exp(-(v + R(35)) / R(10)));
  R y = (v + R(55)) / R(10);
  r.an = (y == R(0)) ? R(0.1) : (R(0.1) * y) / (-std::expm1(-y));
  r.bn = R(0.125) * std::exp(-(v + R(65)) / R(80));
  return r;
}

// One HH step. Euler: the reference's forward-Euler step with its current sign
// convention and -55 mV reset (hodgkin_huxley.rs:46-96). Rush-Larsen: exact
// exponential gate update for frozen V, textbook current signs, spike on an
// upward 0 mV crossing, no reset.
template <class R>
inline bool hh_step(R& v, R& m, R& h, R& n, const R* p, R dt, R I, int integrator) {
  R gna = p[0], gk = p[1], gl = p[2], ena = p[3], ek = p[4], el = p[5], cm = p[6];
  HHRates<R> r = hh_rates<R>(v);
  if (integrator == 0) {
    m = m + (r.am * (R(1) - m) - r.bm * m) * dt;
    h = h + (r.ah * (R(1) - h) - r.bh * h) * dt;
    n = n + (r.an * (R(1) - n) - r.bn * n) * dt;
    R ina = gna * (m * m * m) * h * (ena - v);
    R n2 = n * n;
    R ik = gk * (n2 * n2) * (ek - v);
    R il = gl * (el - v);
    R dv = (I - ina - ik - il) / cm * dt;
    v = v + dv;
    if (v >= R(-55)) { v = R(-70); return true; }
    return false;
  }
  R sm = r.am + r.bm, sh = r.ah + r.bh, sn = r.an + r.bn;
  R minf = r.am / sm, hinf = r.ah / sh, ninf = r.an / sn;
  m = minf + (m - minf) * std::exp(-dt * sm);
  h = hinf + (h - hinf) * std::exp(-dt * sh);
  n = ninf + (n - ninf) * std::exp(-dt * sn);
  R n2 = n * n;
  R iion = gna * (m * m * m) * h * (v - ena) + gk * (n2 * n2) * (v - ek) + gl * (v - el);
  R vn = v + dt * (I - iion) / cm;
  bool spk = (v < R(0)) && (vn >= R(0));
  v = vn;
  return spk;
}

// ---------------------------------------------------------------------------
// Drive values. Same stream layout on host and device:
//   per neuron i, step k: philox(ctr = {i, k_lo, k_hi, 1}, key = seed)
//   Gaussian: pairs of neurons share one draw (cos for even, sin for odd).
//   Reference-shaped global kicks: philox({j, k_lo, k_hi, 2}), j = 0 decides,
//   j = 1.. give (target, amount).
// ---------------------------------------------------------------------------
struct Kick { uint64_t target; float amt_f; double amt_d; };

inline void global_kicks(const or_config& c, uint64_t n, uint64_t k, std::vector<Kick>& out) {
  out.clear();
  if (c.drive_kind != 1 || n == 0) return;
  uint32_t x[4];
  draw(c.seed, 0, k, STREAM_KICKS, x);
  float chance = (float)c.kick_chance;
  if (!(unif_f(x[0]) < chance)) return;
  uint32_t span = (uint32_t)(c.kick_max - c.kick_min + 1);
  uint32_t cnt = (uint32_t)c.kick_min + (uint32_t)(((uint64_t)x[1] * span) >> 32);
  for (uint32_t j = 0; j < cnt; ++j) {
    uint32_t z[4];
    draw(c.seed, 1 + j, k, STREAM_KICKS, z);
    Kick kk;
    kk.target = (uint64_t)(((unsigned __int128)((uint64_t)z[0] | ((uint64_t)z[2] << 32)) * n) >> 64);
    kk.amt_f = unif_f(z[1]) * (float)c.kick_strength;
    kk.amt_d = unif_d(z[1]) * c.kick_strength;
    out.push_back(kk);
  }
}

inline uint32_t prob_threshold(double p) {
  if (p <= 0) return 0;
  double t = p * 4294967296.0;
  if (t >= 4294967295.0) return 0xffffffffu;
  return (uint32_t)t;
}

template <class R> struct DriveOut { R add_I; R kick; R add_g; };

template <class R>
inline DriveOut<R> neuron_drive(const or_config& c, const uint8_t* inh, uint64_t i, uint64_t k);

template <> inline DriveOut<float> neuron_drive<float>(const or_config& c, const uint8_t* inh,
                                                       uint64_t i, uint64_t k) {
  DriveOut<float> d{0.f, 0.f, 0.f};
  uint32_t x[4];
  switch (c.drive_kind) {
    case 1:
      draw(c.seed, (uint32_t)i, k, STREAM_DRIVE, x);
      if (unif_f(x[0]) < (float)c.p) d.add_I = unif_f(x[1]) * (float)c.amp;
      break;
    case 2:  // Poisson kinds: one draw serves steps 4q .. 4q+3, word k mod 4
      draw(c.seed, (uint32_t)i, k >> 2, STREAM_DRIVE, x);
      if (x[k & 3] < prob_threshold(c.p)) d.kick = (float)c.amp;
      break;
    case 3: {
      draw(c.seed, (uint32_t)(i >> 1), k, STREAM_DRIVE, x);
      float u1 = unif_open_f(x[0]);
      float u2 = unif_f(x[1]);
      float l = own_logf(u1);
      float rr = std::sqrt(-2.0f * l);
      float sn, cs;
      own_sincos2pi(u2, &sn, &cs);
      float z = rr * ((i & 1) ? sn : cs);
      float sg = (inh && inh[i]) ? (float)c.sigma_inh : (float)c.sigma_exc;
      d.add_I = sg * z;
      break;
    }
    case 4:
      draw(c.seed, (uint32_t)i, k >> 2, STREAM_DRIVE, x);
      if (x[k & 3] < prob_threshold(c.p)) d.add_g = (float)c.amp;
      break;
    default: break;
  }
  return d;
}

template <> inline DriveOut<double> neuron_drive<double>(const or_config& c, const uint8_t* inh,
                                                         uint64_t i, uint64_t k) {
  DriveOut<double> d{0.0, 0.0, 0.0};
  uint32_t x[4];
  switch (c.drive_kind) {
    case 1:
      draw(c.seed, (uint32_t)i, k, STREAM_DRIVE, x);
      if (unif_d(x[0]) < (double)(float)c.p) d.add_I = unif_d(x[1]) * c.amp;
      break;
    case 2:  // Poisson kinds: one draw serves steps 4q .. 4q+3, word k mod 4
      draw(c.seed, (uint32_t)i, k >> 2, STREAM_DRIVE, x);
      if (x[k & 3] < prob_threshold(c.p)) d.kick = c.amp;
      break;
    case 3: {
      draw(c.seed, (uint32_t)(i >> 1), k, STREAM_DRIVE, x);
      double u1 = unif_open_d(x[0]);
      double u2 = unif_d(x[1]);
      double rr = std::sqrt(-2.0 * std::log(u1));
      double a = 2.0 * M_PI * u2;
      double z = rr * ((i & 1) ? std::sin(a) : std::cos(a));
      double sg = (inh && inh[i]) ? c.sigma_inh : c.sigma_exc;
      d.add_I = sg * z;
      break;
    }
    case 4:
      draw(c.seed, (uint32_t)i, k >> 2, STREAM_DRIVE, x);
      if (x[k & 3] < prob_threshold(c.p)) d.add_g = c.amp;
      break;
    default: break;
  }
  return d;
}

inline int64_t refr_steps_of(double tref, double dt) { return (int64_t)std::round(tref / dt); }

// ---------------------------------------------------------------------------
// Fast engine: per-neuron STDP traces, per-target conductances, float engine
// uses int64 fixed-point synaptic sums exactly like the device.
// ---------------------------------------------------------------------------
template <class R> struct Fast {
  or_config c;
  uint64_t n = 0, m = 0;
  std::vector<uint64_t> rp;
  std::vector<uint32_t> col;
  std::vector<uint8_t> type, plastic, inh, outp;
  std::vector<R> w;            // storage-format-rounded weights
  std::vector<uint16_t> wb;    // bf16 storage (float engine, bf16 format)
  bool bf16 = false;
  std::vector<R> par;          // n * ppn
  int ppn = 0;
  std::vector<int32_t> refr_steps;
  std::vector<R> v, u, I, gm, gh, gn, pre, post, qdec;
  std::vector<int32_t> refr;
  std::vector<int64_t> last;
  std::vector<double> rate;
  std::vector<R> contrib;
  std::vector<R> G[4];
  int ntypes_acc = 1;
  std::vector<int64_t> accf;   // float engine: [type][slot][n]
  std::vector<double> accd;    // double engine
  std::vector<uint64_t> in_ptr;     // plastic incoming (CSC)
  std::vector<uint64_t> in_pos;
  std::vector<uint32_t> in_src;
  std::vector<uint64_t> all_in_ptr; // all incoming, for homeostasis
  std::vector<uint64_t> all_in_pos;
  std::vector<R> Ep, Em;
  R ep = 0, em = 0;
  std::vector<uint8_t> spiked;
  std::vector<uint32_t> spk;
  std::vector<uint32_t> log_idx;
  std::vector<uint64_t> log_off{0};
  uint64_t step = 0, events = 0;
  std::vector<Kick> kicks;
  // R-STDP, consolidation, STP (engine.rs:457-463, :519-563, :626-631)
  std::vector<uint8_t> elig;   // synapse carries an eligibility trace
  std::vector<R> e;            // eligibility values
  std::vector<R> stpf;         // STP factor per synapse (empty: no STP)
  R ce = 0;                    // exp(-dt / elig_tau)
  bool plast_any = false, fuse_ok = false;
  uint64_t origin = 0;         // step at which rew_init / ezero_init hold
  double rew_init = 0;
  int ezero_init = 0;
  double rew_prev = 0, reward_sum = 0, R_k = 0;
  uint64_t outs_prev = 0;
  int mode_prev = 0, mode = 0; // 0 no reward, 1 in the STDP walks, 2 full pass
  R lrr = 0;
  double cons_a = 1.0, consA_prev = 1.0, consA_cur = 1.0;
  uint64_t cons_k0 = 0;
  R fr[6] = {1, 0, 1, 1, 0, 1};  // weight frame of step k and k+1: A, B, 1/A
  // LFP of the reference conductance mode (lfp_signal, engine.rs:478-493):
  // per neuron sum_t |g_t (E_t - V)| at the neuron's update, the float engine
  // rounding each neuron's term to 2^-24 fixed point; one step's sum joins
  // the FP64 total at the start of the next step.
  int64_t lfp_fix_prev = 0, lfp_fix_cur = 0;
  double lfp_d_prev = 0, lfp_d_cur = 0, lfp_total = 0;
  // host stimulus (engine.rs:156-161) as the device applies it: amounts
  // summed per neuron in call order, added to the input current of step
  // stim_at - 1 after the synaptic input, before the drive
  std::vector<R> stim;
  uint64_t stim_at = 0;
  void add_input_current(uint64_t cnt, const uint32_t* ids, const double* amounts) {
    if (stim.size() != n) stim.assign(n, R(0));
    for (uint64_t q = 0; q < cnt; ++q) stim[ids[q]] = stim[ids[q]] + (R)amounts[q];
    stim_at = step + 1;
  }
  bool cond() const { return c.input_mode == 3 || c.input_mode == 4; }

  R wget(uint64_t s) const { return bf16 ? (R)bf16_to_f32(wb[s]) : w[s]; }
  void wset(uint64_t s, R x) {
    if (bf16) wb[s] = f32_to_bf16_rne((float)x); else w[s] = x;
  }
  // Consolidation frame: the stored value u of a synapse stands for the
  // weight u*A + B of the frame (A = a^(k - k0), B = target*(1 - A)), so the
  // per-step drift of every weight toward the target is a change of frame.
  R wplain(uint64_t s, int f) const {
    R u = wget(s);
    return c.cons ? u * fr[3 * f] + fr[3 * f + 1] : u;
  }
  void wstore(uint64_t s, R x, int f) { wset(s, c.cons ? (x - fr[3 * f + 1]) * fr[3 * f + 2] : x); }
  // frame of a step from its A (double), as the device rounds it
  void frame_of(double A, R* out) const {
    out[0] = (R)A;
    out[1] = (R)(c.cons_target * (1.0 - A));
    out[2] = (R)(1.0 / A);
  }
  // mode-1 apply of one synapse touched by this step's STDP: w1 plain in
  // frame k; returns the stored value's plain weight in frame k+1 after the
  // reward (engine.rs:546-561 after the consolidation of :539-545)
  // The reward changes a weight only where e != 0 or the weight lies outside
  // [rstdp_w_min, rstdp_w_max]; elsewhere clamp(w + lr*r*0) == w exactly.
  bool reward_moves(R x, R ev) const {
    return ev != R(0) || x < (R)c.rstdp_wmin || x > (R)c.rstdp_wmax;
  }
  R storage_round(R x) const { return bf16 ? (R)bf16_to_f32(f32_to_bf16_rne((float)x)) : x; }
  void store_touched(uint64_t s, R w1) {
    if (mode == 1 && elig[s]) {
      // the value the STDP walk stores, read in the frame of step k+1: the
      // same numbers the full pass would see
      const R u1 = storage_round(c.cons ? (w1 - fr[1]) * fr[2] : w1);
      R x = c.cons ? u1 * fr[3] + fr[4] : u1;
      if (reward_moves(x, e[s])) {
        x = clampw<R>(x + lrr * e[s], (R)c.rstdp_wmin, (R)c.rstdp_wmax);
        e[s] = R(0);
        wstore(s, x, 1);
      } else {
        wset(s, u1);
      }
    } else {
      wstore(s, w1, 0);
    }
  }

  void init(const or_config& cfg, const or_net& net) {
    c = cfg;
    n = net.n; m = net.m;
    rp.assign(net.row_ptr, net.row_ptr + n + 1);
    col.assign(net.col, net.col + m);
    type.assign(m, 0);
    if (net.syn_type) type.assign(net.syn_type, net.syn_type + m);
    plastic.assign(m, 0);
    if (net.plastic) plastic.assign(net.plastic, net.plastic + m);
    inh.assign(n, 0);
    if (net.inhibitory) inh.assign(net.inhibitory, net.inhibitory + n);
    outp.assign(n, 0);
    if (net.is_output) outp.assign(net.is_output, net.is_output + n);
    bf16 = (sizeof(R) == 4) && c.weight_format == 1;
    if (bf16) {
      wb.resize(m);
      for (uint64_t s = 0; s < m; ++s) wb[s] = f32_to_bf16_rne(net.w[s]);
    } else {
      w.resize(m);
      for (uint64_t s = 0; s < m; ++s) w[s] = (R)net.w[s];
    }
    ppn = net.ppn;
    par.resize(n * (uint64_t)ppn);
    for (uint64_t q = 0; q < n * (uint64_t)ppn; ++q) par[q] = (R)net.params[q];
    refr_steps.assign(n, 0);
    if (c.model == 0)
      for (uint64_t i = 0; i < n; ++i)
        refr_steps[i] = (int32_t)refr_steps_of((double)net.params[i * ppn + 4], c.dt);
    v.resize(n); u.assign(n, R(0)); I.assign(n, R(0));
    gm.assign(n, R(0.05f)); gh.assign(n, R(0.6f)); gn.assign(n, R(0.32f));
    for (uint64_t i = 0; i < n; ++i) {
      R rest = c.model == 0 ? par[i * ppn + 0] : (c.model == 1 ? par[i * ppn + 2] : par[i * ppn + 5]);
      v[i] = net.v0 ? (R)net.v0[i] : rest;
      if (net.u0) u[i] = (R)net.u0[i];
      if (net.m0) gm[i] = (R)net.m0[i];
      if (net.h0) gh[i] = (R)net.h0[i];
      if (net.n0) gn[i] = (R)net.n0[i];
    }
    refr.assign(n, 0);
    pre.assign(n, R(0)); post.assign(n, R(0)); qdec.assign(n, R(0));
    last.assign(n, -1);
    rate.assign(n, 0.0);
    contrib.assign(c.homeo ? m : 0, R(0));
    for (int t = 0; t < 4; ++t) G[t].assign(cond() ? n : 0, R(0));
    ntypes_acc = cond() ? 4 : 1;
    uint64_t acc_n = (uint64_t)ntypes_acc * (uint64_t)c.delay_steps * n;
    if (sizeof(R) == 4) accf.assign(acc_n, 0); else accd.assign(acc_n, 0.0);
    // incoming index lists (CSR positions grouped by target, ascending position)
    all_in_ptr.assign(n + 1, 0);
    for (uint64_t s = 0; s < m; ++s) all_in_ptr[col[s] + 1]++;
    for (uint64_t i = 0; i < n; ++i) all_in_ptr[i + 1] += all_in_ptr[i];
    all_in_pos.resize(m);
    {
      std::vector<uint64_t> cur(all_in_ptr.begin(), all_in_ptr.end() - 1);
      for (uint64_t s = 0; s < m; ++s) all_in_pos[cur[col[s]]++] = s;
    }
    in_ptr.assign(n + 1, 0);
    for (uint64_t s = 0; s < m; ++s) if (plastic[s]) in_ptr[col[s] + 1]++;
    for (uint64_t i = 0; i < n; ++i) in_ptr[i + 1] += in_ptr[i];
    in_pos.resize(in_ptr[n]);
    in_src.resize(in_ptr[n]);
    {
      std::vector<uint64_t> cur(in_ptr.begin(), in_ptr.end() - 1);
      for (uint64_t j = 0; j < n; ++j)
        for (uint64_t s = rp[j]; s < rp[j + 1]; ++s)
          if (plastic[s]) { uint64_t q = cur[col[s]]++; in_pos[q] = s; in_src[q] = (uint32_t)j; }
    }
    // trace decay tables: exp(-k dt / tau) for the spike-to-spike factor
    ep = (R)std::exp(-c.dt / c.tau_plus);
    em = (R)std::exp(-c.dt / c.tau_minus);
    auto table = [&](double tau, std::vector<R>& t) {
      uint64_t K = (uint64_t)std::ceil(104.0 * tau / c.dt) + 2;
      if (K > (1u << 22)) K = 1u << 22;
      t.resize(K);
      for (uint64_t q = 0; q < K; ++q) t[q] = (R)std::exp(-(double)q * c.dt / tau);
    };
    if (c.stdp) { table(c.tau_plus, Ep); table(c.tau_minus, Em); }
    spiked.assign(n, 0);
    // R-STDP state
    elig.assign(m, 0);
    e.assign(m, R(0));
    if (c.rstdp)
      for (uint64_t s = 0; s < m; ++s) elig[s] = net.eligible ? (net.eligible[s] ? 1 : 0) : plastic[s];
    ce = (R)std::exp(-c.dt / c.elig_tau);
    plast_any = c.stdp || c.homeo || c.rstdp || c.cons;
    fuse_ok = (!c.stdp || (c.rstdp_wmin <= c.w_min && c.w_max <= c.rstdp_wmax)) &&
              (!c.homeo || (c.rstdp_wmin <= 0.0 && 10.0 <= c.rstdp_wmax)) &&
              (!c.cons || (c.rstdp_wmin <= c.cons_target && c.cons_target <= c.rstdp_wmax));
    origin = 0; rew_init = c.reward_init; ezero_init = 0;
    if (c.cons) cons_a = 1.0 - (c.dt / c.cons_tau) * c.cons_drift;
    cons_k0 = 0;
    // STP: one step of a copy of the synapse's state (engine.rs:457-463)
    stpf.clear();
    if (net.stp && !cond()) {
      stpf.assign(m, R(1));
      for (uint64_t s = 0; s < m; ++s) {
        if (net.has_stp && !net.has_stp[s]) continue;
        stpf[s] = (R)stp_factor(net.stp + 5 * s, c.dt);
      }
    }
  }

  static double stp_factor(const double* q, double dt) {
    // (u + u_se*(1-u)/tau_facil*dt) * r, ShortTermPlasticity::step(dt, true)
    double u = q[3] + q[0] * (1.0 - q[3]) / q[2] * dt;
    return u * q[4];
  }

  // reward, R-STDP mode and consolidation frame of step k (the device's
  // per-step setup in the neuron kernel's last tile)
  void setup(uint64_t k) {
    double Rr;
    int ez;
    if (k == origin) {
      Rr = rew_init;
      ez = ezero_init;
    } else {
      double Rd = plast_any ? rew_prev * c.reward_decay : rew_prev;
      Rr = (outs_prev >= c.reward_thr) ? std::fmin(Rd + 1.0, 1.0) : Rd;
      reward_sum += Rr;
      ez = mode_prev != 0;
    }
    R_k = Rr;
    bool active = c.rstdp && std::fabs(Rr) > 0.001;
    mode = !active ? 0 : ((ez && fuse_ok) ? 1 : 2);
    lrr = (R)(c.rstdp_lr * Rr);
    if (c.cons) {
      consA_cur = (k == cons_k0) ? 1.0 : consA_prev * cons_a;
      frame_of(consA_cur, fr);
      frame_of(consA_cur * cons_a, fr + 3);
    }
  }

  // mode-2 reward pass over every eligible synapse and the frame
  // renormalisation (the device's tail kernel)
  void tail(uint64_t k) {
    const bool renorm = c.cons && consA_cur * cons_a < 0x1p-16;
    if (mode != 2 && !renorm) return;
    for (uint64_t s = 0; s < m; ++s) {
      const bool ap = mode == 2 && elig[s];
      if (!ap && !renorm) continue;
      R x = wplain(s, 1);
      bool chg = false;
      if (ap && reward_moves(x, e[s])) {
        x = clampw<R>(x + lrr * e[s], (R)c.rstdp_wmin, (R)c.rstdp_wmax);
        e[s] = R(0);
        chg = true;
      }
      if (renorm) wset(s, x);
      else if (chg) wstore(s, x, 1);
    }
    if (renorm) {
      cons_k0 = k + 1;
      fr[3] = R(1); fr[4] = R(0); fr[5] = R(1);
    }
  }

  // reward after the last step (phase 3 of engine.rs:626-631)
  double reward_now() const {
    if (step == origin) return rew_init;
    double Rd = plast_any ? rew_prev * c.reward_decay : rew_prev;
    return (outs_prev >= c.reward_thr) ? std::fmin(Rd + 1.0, 1.0) : Rd;
  }

  // SimulationEngine::apply_reward between steps, in the frame of the next step
  void apply_reward(double reward) {
    if (!c.rstdp) return;
    const double now = reward_now();
    R f[3] = {1, 0, 1};
    if (c.cons) frame_of(step == cons_k0 ? 1.0 : consA_prev * cons_a, f);
    const R l = (R)(c.rstdp_lr * reward);
    for (uint64_t s = 0; s < m; ++s) {
      if (!elig[s]) continue;
      R u = wget(s);
      R x = c.cons ? u * f[0] + f[1] : u;
      if (!reward_moves(x, e[s])) continue;
      x = clampw<R>(x + l * e[s], (R)c.rstdp_wmin, (R)c.rstdp_wmax);
      e[s] = R(0);
      wset(s, c.cons ? (x - f[1]) * f[2] : x);
    }
    if (step > origin) reward_sum += now;
    origin = step;
    rew_init = now;
    ezero_init = 1;
  }

  R table_at(const std::vector<R>& t, int64_t dk) const {
    if (dk < 0 || (uint64_t)dk >= t.size()) return R(0);
    return t[(size_t)dk];
  }

  void phase_a(uint64_t k) {
    const R dt = (R)c.dt;
    const uint64_t D = (uint64_t)c.delay_steps;
    const uint64_t slot = k % D;
    global_kicks(c, n, k, kicks);
    spk.clear();
    if (c.input_mode == 3) {
      if (sizeof(R) == 4) lfp_total += (double)lfp_fix_prev * 0x1p-24;
      else lfp_total += lfp_d_prev;
      lfp_fix_cur = 0;
      lfp_d_cur = 0;
    }
    for (uint64_t i = 0; i < n; ++i) {
      R syn = 0;
      R S[4] = {0, 0, 0, 0};
      for (int t = 0; t < ntypes_acc; ++t) {
        uint64_t a = ((uint64_t)t * D + slot) * n + i;
        R val;
        if (sizeof(R) == 4) { val = (R)from_fix(accf[a]); accf[a] = 0; }
        else { val = (R)accd[a]; accd[a] = 0.0; }
        if (cond()) S[t] = val; else syn = val;
      }
      DriveOut<R> d = neuron_drive<R>(c, inh.data(), i, k);
      R Ii = I[i];
      R kick = 0;
      R vi = v[i];
      switch (c.input_mode) {
        case 0:
          if (k > 0) Ii = (Ii + syn) * (R)c.current_decay;
          break;
        case 1:
          Ii = 0;
          kick = syn;
          break;
        case 2:
          Ii = syn;
          break;
        default: {
          R isyn = 0, lf = 0;
          for (int t = 0; t < 4; ++t) {
            R dec = (R)std::exp(-c.dt / kDyn[t].decay);
            R inc = S[t] * (R)kDyn[t].gmax;
            if (kDyn[t].mg) inc = inc * mg_block<R>(t, vi);
            R g = G[t][i] * dec + inc;
            if (t == 0) g = g + d.add_g;
            G[t][i] = g;
            const R cur = g * ((R)kDyn[t].erev - vi);
            isyn = isyn + cur;
            lf = lf + std::fabs(cur);
          }
          if (c.input_mode == 3) {
            if (sizeof(R) == 4) lfp_fix_cur += (int64_t)std::llrint((float)lf * 0x1p24f);
            else lfp_d_cur += (double)lf;
          }
          Ii = (c.input_mode == 3) ? Ii + isyn : isyn;
          break;
        }
      }
      if (stim_at == k + 1) {
        const R sv = stim[i];
        stim[i] = R(0);
        if (sv != R(0)) Ii = Ii + sv;
      }
      Ii = Ii + d.add_I;
      for (const Kick& kk : kicks)
        if (kk.target == i) Ii = Ii + (sizeof(R) == 4 ? (R)kk.amt_f : (R)kk.amt_d);
      kick = kick + d.kick;
      // model update
      bool s = false;
      const R* p = &par[i * ppn];
      if (c.model == 0) {
        if (refr[i] > 0) {
          refr[i] -= 1;
        } else {
          R t1 = vi - p[0];
          R t2 = p[5] * Ii;
          R t3 = (-t1) + t2;
          R t4 = t3 * dt;
          R dv = t4 / p[3];
          vi = vi + dv;
          if (c.input_mode == 1) vi = vi + kick;
          if (vi >= p[1]) { vi = p[2]; refr[i] = refr_steps[i]; s = true; }
        }
      } else if (c.model == 1) {
        if (vi >= R(30)) {
          vi = p[2];
          u[i] = u[i] + p[3];
          s = true;
        } else {
          R ui = u[i];
          R a1 = (sizeof(R) == 4 ? (R)0.04f : (R)0.04) * vi;
          R a2 = a1 * vi;
          R a3 = R(5) * vi;
          R sm = a2 + a3;
          sm = sm + R(140);
          sm = sm - ui;
          sm = sm + Ii;
          R dv = sm * dt;
          R b1 = p[1] * vi;
          R b2 = b1 - ui;
          R b3 = p[0] * b2;
          R du = b3 * dt;
          vi = vi + dv;
          ui = ui + du;
          if (c.input_mode == 1) vi = vi + kick;
          u[i] = ui;
        }
      } else {
        R mm = gm[i], hh = gh[i], nn = gn[i];
        s = hh_step<R>(vi, mm, hh, nn, p, dt, Ii, c.hh_integrator);
        if (c.input_mode == 1) vi = vi + kick;
        gm[i] = mm; gh[i] = hh; gn[i] = nn;
      }
      v[i] = vi;
      I[i] = Ii;
      spiked[i] = s ? 1 : 0;
      if (c.stdp) {
        R pi = pre[i] * ep;
        R qi = post[i] * em;
        if (s) {
          int64_t dk = last[i] < 0 ? -1 : (int64_t)k - last[i];
          qdec[i] = qi;
          pi = pi * table_at(Ep, dk) + R(1);
          qi = qi * table_at(Em, dk) + R(1);
        }
        pre[i] = pi; post[i] = qi;
      }
      if (s) { last[i] = (int64_t)k; spk.push_back((uint32_t)i); }
    }
    if (c.input_mode == 3) { lfp_fix_prev = lfp_fix_cur; lfp_d_prev = lfp_d_cur; }
  }

  // LFP after the last completed step: the folded steps, the last step's
  // sum, then the last step's own term, which the device's next neuron
  // update would compute (the delivered input read, not consumed; no drive).
  double lfp() const {
    if (c.input_mode != 3) return 0.0;
    const uint64_t D = (uint64_t)c.delay_steps;
    const uint64_t slot = step % D;
    int64_t pf = 0;
    double pd = 0;
    for (uint64_t i = 0; i < n; ++i) {
      const R vi = v[i];
      R lf = 0;
      for (int t = 0; t < 4; ++t) {
        R S = 0;
        if (t < ntypes_acc) {
          const uint64_t a = ((uint64_t)t * D + slot) * n + i;
          S = sizeof(R) == 4 ? (R)from_fix(accf[a]) : (R)accd[a];
        }
        R inc = S * (R)kDyn[t].gmax;
        if (kDyn[t].mg) inc = inc * mg_block<R>(t, vi);
        const R g = G[t][i] * (R)std::exp(-c.dt / kDyn[t].decay) + inc;
        lf = lf + std::fabs(g * ((R)kDyn[t].erev - vi));
      }
      if (sizeof(R) == 4) pf += (int64_t)std::llrint((float)lf * 0x1p24f);
      else pd += (double)lf;
    }
    double t = lfp_total;
    if (sizeof(R) == 4) {
      if (step > 0) t += (double)lfp_fix_prev * 0x1p-24;
      t += (double)pf * 0x1p-24;
    } else {
      if (step > 0) t += lfp_d_prev;
      t += pd;
    }
    return t;
  }

  void accumulate(uint64_t slot_base_type, uint64_t i, R val) {
    uint64_t a = slot_base_type * n + i;
    if (sizeof(R) == 4) accf[a] += to_fix((float)val); else accd[a] += (double)val;
  }

  void phase_b(uint64_t k, uint64_t* trace, uint64_t cap, uint64_t* ntr) {
    const uint64_t D = (uint64_t)c.delay_steps;
    const uint64_t slot = k % D;
    const R ap = (R)c.a_plus, nam = (R)(-c.a_minus), wlo = (R)c.w_min, whi = (R)c.w_max;
    const R cd = (R)std::exp(-c.dt / c.contrib_tau);
    const R one_m_cd = R(1) - cd;
    for (uint32_t j : spk) {
      for (uint64_t s = rp[j]; s < rp[j + 1]; ++s) {
        if (trace) { if (*ntr < cap) trace[*ntr] = s; ++*ntr; }
        uint32_t i = col[s];
        R ws = wplain(s, 0);
        int t = cond() ? type[s] : 0;
        R val = ws;
        if (cond() && (t == 1 || t == 2)) val = std::fabs(ws);
        if (!stpf.empty()) val = val * stpf[s];
        accumulate((uint64_t)t * D + slot, i, val);
        ++events;
        if (c.homeo) {
          R mag;
          if (cond()) mag = std::fabs(ws * (R)kDyn[t].gmax * mg_block<R>(t, v[i]));
          else mag = std::fabs(val);
          contrib[s] = contrib[s] * cd + mag * one_m_cd;
        }
        if (c.stdp && plastic[s]) {
          R w1;
          const R dp = ap * (spiked[i] ? qdec[i] : post[i]);
          w1 = clampw<R>(ws + dp, wlo, whi);
          if (elig[s]) e[s] = e[s] * ce + dp;
          if (spiked[i]) {
            const R dm = nam * pre[j];
            w1 = clampw<R>(w1 + dm, wlo, whi);
            if (elig[s]) e[s] = e[s] * ce + dm;
          }
          store_touched(s, w1);
        }
      }
    }
  }

  void phase_c() {
    if (!c.stdp) return;
    const R nam = (R)(-c.a_minus), wlo = (R)c.w_min, whi = (R)c.w_max;
    for (uint32_t i : spk) {
      for (uint64_t q = in_ptr[i]; q < in_ptr[i + 1]; ++q) {
        uint64_t s = in_pos[q];
        uint32_t j = in_src[q];
        if (spiked[j]) continue;
        R ws = wplain(s, 0);
        const R dm = nam * pre[j];
        R w1 = clampw<R>(ws + dm, wlo, whi);
        if (elig[s]) e[s] = e[s] * ce + dm;
        store_touched(s, w1);
      }
    }
  }

  void phase_d() {
    if (!c.homeo) {
      if (c.track_rates)
        for (uint64_t i = 0; i < n; ++i) {
          double inst = spiked[i] ? 1000.0 / c.dt : 0.0;
          rate[i] += (inst - rate[i]) * c.dt / 100.0;
        }
      return;
    }
    const double target = c.h_target;
    for (uint64_t i = 0; i < n; ++i) {
      double err = rate[i] - target;
      uint64_t b = all_in_ptr[i], e = all_in_ptr[i + 1];
      double sum = 0;
      for (uint64_t q = b; q < e; ++q) sum += (double)contrib[all_in_pos[q]];
      uint64_t cnt = e - b;
      if (cnt > 0 && sum >= 1e-12) {
        double mean = sum / (double)cnt;
        for (uint64_t q = b; q < e; ++q) {
          uint64_t s = all_in_pos[q];
          R rel = (R)((double)contrib[s] / mean);
          R arg = (R)(-err) * rel * (R)c.dt / (R)c.h_tau;
          R scale = scale_exp<R>(arg);
          R ws = wplain(s, 1) * scale;
          wstore(s, clampw<R>(ws, R(0), R(10)), 1);
        }
      }
    }
    for (uint64_t i = 0; i < n; ++i) {
      double inst = spiked[i] ? 1000.0 / c.dt : 0.0;
      rate[i] += (inst - rate[i]) * c.dt / 100.0;
    }
  }

  void one_step(uint64_t* trace, uint64_t cap, uint64_t* ntr) {
    uint64_t k = step;
    phase_a(k);
    log_idx.insert(log_idx.end(), spk.begin(), spk.end());
    log_off.push_back(log_idx.size());
    setup(k);
    phase_b(k, trace, cap, ntr);
    phase_c();
    tail(k);
    phase_d();
    uint64_t outs = 0;
    for (uint32_t j : spk) outs += outp[j] ? 1u : 0u;
    outs_prev = outs;
    rew_prev = R_k;
    mode_prev = mode;
    consA_prev = consA_cur;
    ++step;
  }
};

// ---------------------------------------------------------------------------
// Literal engine: FP64, per-synapse state, the reference's loop structure
// (engine.rs:254-680). Synapse vector in CSR order (the reference indexes its
// synapse vector by CSR position, engine.rs:417-428).
// ---------------------------------------------------------------------------
struct LitSyn {
  uint32_t source, target;
  double weight;
  uint8_t type, plastic;
  double pre_trace, post_trace, last_pre, last_post;
  double contribution_avg;
  uint8_t elig, has_stp;   // eligibility trace (with_rstdp), ShortTermPlasticity
  double e;                // EligibilityTrace.value
  double stp[5];           // u_se, tau_rec, tau_facil, u, r
};

struct Lit {
  or_config c;
  uint64_t n = 0, m = 0;
  std::vector<uint64_t> rp;
  std::vector<uint32_t> col;
  std::vector<LitSyn> syn;
  std::vector<double> cond;     // per-synapse conductance
  std::vector<double> par;
  int ppn = 0;
  std::vector<double> v, u, I, gm, gh, gn, last_spike_time, g_ext;
  std::vector<int32_t> refr;
  std::vector<uint64_t> spike_ct;
  std::vector<uint8_t> inh, outp, spiked;
  std::vector<std::vector<uint64_t>> by_target;
  std::vector<double> firing_rates;
  std::vector<double> ring;     // delayed current / kick sums [slot][n]
  std::vector<std::vector<uint64_t>> pending;  // COND_FRESH pending events per slot
  double time = 0;
  uint64_t step = 0, events = 0;
  std::vector<uint32_t> log_idx;
  std::vector<uint64_t> log_off{0};
  std::vector<Kick> kicks;
  double lfp = 0, weight_mean = 0, weight_std = 0, mean_rate = 0;
  uint64_t total_spikes = 0;
  int threads = 1;
  double reward = 0, reward_sum = 0;   // engine.rs:71-77
  bool plast_any = false;

  void init(const or_config& cfg, const or_net& net, int nthreads) {
    c = cfg; n = net.n; m = net.m; threads = nthreads > 0 ? nthreads : 1;
    rp.assign(net.row_ptr, net.row_ptr + n + 1);
    col.assign(net.col, net.col + m);
    syn.resize(m);
    for (uint64_t j = 0; j < n; ++j)
      for (uint64_t s = rp[j]; s < rp[j + 1]; ++s) {
        LitSyn& y = syn[s];
        y.source = (uint32_t)j; y.target = col[s];
        y.weight = (double)net.w[s];
        y.type = net.syn_type ? net.syn_type[s] : 0;
        y.plastic = net.plastic ? net.plastic[s] : 0;
        y.pre_trace = 0; y.post_trace = 0; y.last_pre = -1e9; y.last_post = -1e9;
        y.contribution_avg = 0;
        y.elig = c.rstdp ? (net.eligible ? (net.eligible[s] ? 1 : 0) : y.plastic) : 0;
        y.e = 0;
        y.has_stp = (net.stp && (!net.has_stp || net.has_stp[s])) ? 1 : 0;
        for (int q = 0; q < 5; ++q) y.stp[q] = y.has_stp ? net.stp[5 * s + q] : 0.0;
      }
    reward = c.reward_init;
    plast_any = c.stdp || c.homeo || c.rstdp || c.cons;
    cond.assign(m, 0.0);
    ppn = net.ppn;
    par.resize(n * (uint64_t)ppn);
    for (uint64_t q = 0; q < n * (uint64_t)ppn; ++q) par[q] = (double)net.params[q];
    v.resize(n); u.assign(n, 0.0); I.assign(n, 0.0);
    gm.assign(n, 0.05); gh.assign(n, 0.6); gn.assign(n, 0.32);
    for (uint64_t i = 0; i < n; ++i) {
      double rest = c.model == 0 ? par[i * ppn + 0] : (c.model == 1 ? par[i * ppn + 2] : par[i * ppn + 5]);
      v[i] = net.v0 ? (double)net.v0[i] : rest;
      if (net.u0) u[i] = net.u0[i];
      gm[i] = net.m0 ? (double)net.m0[i] : (double)0.05f;
      gh[i] = net.h0 ? (double)net.h0[i] : (double)0.6f;
      gn[i] = net.n0 ? (double)net.n0[i] : (double)0.32f;
    }
    refr.assign(n, 0);
    spike_ct.assign(n, 0);
    last_spike_time.assign(n, -1e9);
    g_ext.assign(n, 0.0);
    inh.assign(n, 0);
    if (net.inhibitory) inh.assign(net.inhibitory, net.inhibitory + n);
    outp.assign(n, 0);
    if (net.is_output) outp.assign(net.is_output, net.is_output + n);
    spiked.assign(n, 0);
    by_target.assign(n, {});
    for (uint64_t s = 0; s < m; ++s) by_target[syn[s].target].push_back(s);  // engine.rs:86-92
    firing_rates.assign(n, 0.0);
    ring.assign((uint64_t)c.delay_steps * n, 0.0);
    pending.assign(c.delay_steps, {});
  }

  bool neuron_step(uint64_t i, double Iin, double kick) {
    const double* p = &par[i * ppn];
    const double dt = c.dt;
    if (c.model == 0) {
      // LifNeuron::step, lif.rs:15-61
      if (refr[i] > 0) { refr[i] -= 1; return false; }
      double dv = (-(v[i] - p[0]) + p[5] * Iin) * dt / p[3];
      v[i] += dv;
      if (c.input_mode == 1) v[i] += kick;
      if (v[i] >= p[1]) {
        v[i] = p[2];
        refr[i] = (int32_t)std::round(p[4] / dt);
        spike_ct[i] += 1;
        return true;
      }
      return false;
    }
    if (c.model == 1) {
      // IzhikevichNeuron::step, izhikevich.rs:20-52
      if (v[i] >= 30.0) {
        v[i] = p[2];
        u[i] += p[3];
        spike_ct[i] += 1;
        return true;
      }
      double vv = v[i], uu = u[i];
      double dv = (0.04 * vv * vv + 5.0 * vv + 140.0 - uu + Iin) * dt;
      double du = p[0] * (p[1] * vv - uu) * dt;
      v[i] += dv;
      u[i] += du;
      if (c.input_mode == 1) v[i] += kick;
      return false;
    }
    // HodgkinHuxleyNeuron::step (hodgkin_huxley.rs:46-96) or Rush-Larsen
    bool s = hh_step<double>(v[i], gm[i], gh[i], gn[i], p, dt, Iin, c.hh_integrator);
    if (c.input_mode == 1) v[i] += kick;
    if (s) spike_ct[i] += 1;
    return s;
  }

  void one_step() {
    const double dt = c.dt;
    const uint64_t D = (uint64_t)c.delay_steps;
    const uint64_t k = step;
    const uint64_t slot = k % D;
    std::vector<double> kick(n, 0.0);
    // COND_FRESH: conductances are brought to the start of this step
    if (c.input_mode == 4) {
      for (uint64_t s = 0; s < m; ++s) cond[s] *= std::exp(-dt / kDyn[syn[s].type].decay);
      double ed = std::exp(-dt / kDyn[0].decay);
      for (uint64_t i = 0; i < n; ++i) g_ext[i] *= ed;
      for (uint64_t s : pending[slot]) {
        const LitSyn& y = syn[s];
        double gp = y.weight * kDyn[y.type].gmax * mg_block<double>(y.type, v[y.target]);
        if (y.type == 1 || y.type == 2) cond[s] += std::fabs(gp); else cond[s] += gp;
      }
      pending[slot].clear();
      for (uint64_t i = 0; i < n; ++i) {
        DriveOut<double> d = neuron_drive<double>(c, inh.data(), i, k);
        g_ext[i] += d.add_g;
        I[i] = g_ext[i] * (kDyn[0].erev - v[i]);
      }
      for (uint64_t s = 0; s < m; ++s) {
        const LitSyn& y = syn[s];
        I[y.target] += cond[s] * (kDyn[y.type].erev - v[y.target]);
      }
    }
    // delayed current / kick delivery for this step
    if (c.input_mode == 0 || c.input_mode == 2 || c.input_mode == 1) {
      for (uint64_t i = 0; i < n; ++i) {
        double r = ring[slot * n + i];
        ring[slot * n + i] = 0.0;
        if (c.input_mode == 1) kick[i] += r;
        else if (c.input_mode == 2) I[i] += r;
        else if (D > 1 && k > 0) I[i] = (I[i] + r) * c.current_decay;
      }
    }
    // Phase 1: drive (engine.rs:273-287), then the parallel neuron update
    global_kicks(c, n, k, kicks);
    for (uint64_t i = 0; i < n; ++i) {
      DriveOut<double> d = neuron_drive<double>(c, inh.data(), i, k);
      I[i] += d.add_I;
      kick[i] += d.kick;
    }
    for (const Kick& kk : kicks) I[kk.target] += kk.amt_d;
    const double sim_time_now = time;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
      bool s = neuron_step((uint64_t)i, I[i], kick[i]);
      spiked[i] = s ? 1 : 0;
      if (s) last_spike_time[i] = sim_time_now;
    }
    std::vector<uint32_t> spk;
    for (uint64_t i = 0; i < n; ++i) if (spiked[i]) spk.push_back((uint32_t)i);
    log_idx.insert(log_idx.end(), spk.begin(), spk.end());
    log_off.push_back(log_idx.size());
    total_spikes += spk.size();
    if (c.input_mode == 2) std::fill(I.begin(), I.end(), 0.0);
    time += dt;
    // Phase 2 (engine.rs:397-615)
    if (c.input_mode == 3)
      for (uint64_t s = 0; s < m; ++s) cond[s] *= std::exp(-dt / kDyn[syn[s].type].decay);
    const double cdec = std::exp(-dt / c.contrib_tau);
    const uint64_t dslot = (k + D - 1) % D;  // delivered at step k + D
    for (uint32_t j : spk) {
      for (uint64_t s = rp[j]; s < rp[j + 1]; ++s) {
        LitSyn& y = syn[s];
        ++events;
        if (c.input_mode == 3 || c.input_mode == 4) {
          double gp = y.weight * kDyn[y.type].gmax * mg_block<double>(y.type, v[y.target]);
          if (c.input_mode == 3) {
            if (y.type == 1 || y.type == 2) cond[s] += std::fabs(gp); else cond[s] += gp;
          } else {
            pending[(k + D) % D].push_back(s);
          }
          y.contribution_avg = y.contribution_avg * cdec + std::fabs(gp) * (1.0 - cdec);
        } else {
          double cur = y.weight;
          if (y.has_stp) {
            // a copy of the synapse's STP state takes one step (engine.rs:457-463)
            double su = y.stp[3], sr = y.stp[4];
            cur *= or_stp_step(&su, &sr, y.stp[0], y.stp[1], y.stp[2], dt, 1);
          }
          if (D == 1) {
            if (c.input_mode == 0) I[y.target] += cur;
            else ring[0 * n + y.target] += cur;
          } else {
            ring[((k + D) % D) * n + y.target] += cur;
          }
          y.contribution_avg = y.contribution_avg * cdec + std::fabs(cur) * (1.0 - cdec);
        }
      }
    }
    (void)dslot;
    if (c.input_mode == 3) {
      for (uint64_t s = 0; s < m; ++s) {
        double g = cond[s];
        if (std::fabs(g) < 1e-12) continue;
        const LitSyn& y = syn[s];
        double isyn = g * (kDyn[y.type].erev - v[y.target]);
        I[y.target] += isyn;
        lfp += std::fabs(isyn);
      }
    }
    if (c.stdp) {
      const double current_time = time;
      for (uint64_t s = 0; s < m; ++s) {
        LitSyn& y = syn[s];
        if (!y.plastic) continue;
        y.pre_trace *= std::exp(-dt / c.tau_plus);
        y.post_trace *= std::exp(-dt / c.tau_minus);
        bool pre_fired = spiked[y.source] != 0;
        bool post_fired = spiked[y.target] != 0;
        if (pre_fired) {
          double delta = c.a_plus * y.post_trace;
          y.weight = clampw<double>(y.weight + delta, c.w_min, c.w_max);
          double d = current_time - y.last_pre;
          y.pre_trace = y.pre_trace * std::exp(-d / c.tau_plus) + 1.0;
          y.last_pre = current_time;
          if (y.elig) or_eligibility_update(&y.e, dt, c.elig_tau, delta);
        }
        if (post_fired) {
          double delta = -c.a_minus * y.pre_trace;
          y.weight = clampw<double>(y.weight + delta, c.w_min, c.w_max);
          double d = current_time - y.last_post;
          y.post_trace = y.post_trace * std::exp(-d / c.tau_minus) + 1.0;
          y.last_post = current_time;
          if (y.elig) or_eligibility_update(&y.e, dt, c.elig_tau, delta);
        }
      }
    }
    // consolidation of every synapse (engine.rs:539-545)
    if (c.cons)
      for (LitSyn& y : syn) or_consolidation_apply(&y.weight, c.cons_tau, c.cons_target, c.cons_drift, dt);
    // R-STDP while the reward is on (engine.rs:546-561), then its decay (:563)
    if (c.rstdp && std::fabs(reward) > 0.001)
      for (LitSyn& y : syn)
        if (y.elig) or_eligibility_apply(&y.e, reward, &y.weight, c.rstdp_lr, c.rstdp_wmin, c.rstdp_wmax);
    if (plast_any) reward *= c.reward_decay;
    if (c.homeo) {
      for (uint64_t i = 0; i < n; ++i) {
        double rate = firing_rates[i];
        double err = rate - c.h_target;
        double sum = 0;
        uint64_t cnt = 0;
        for (uint64_t s : by_target[i]) { sum += syn[s].contribution_avg; ++cnt; }
        if (cnt == 0 || sum < 1e-12) continue;
        double mean = sum / (double)cnt;
        for (uint64_t s : by_target[i]) {
          double rel = syn[s].contribution_avg / mean;
          double scale = std::exp(-(err * rel) * dt / c.h_tau);
          syn[s].weight *= scale;
          syn[s].weight = clampw<double>(syn[s].weight, 0.0, 10.0);
        }
      }
    }
    if (c.input_mode == 0 && D == 1) {
      for (uint64_t i = 0; i < n; ++i) I[i] *= c.current_decay;
    }
    // Phase 3 (engine.rs:617-670): reward from this step's output spikes
    uint64_t outs = 0;
    for (uint32_t j : spk) outs += outp[j] ? 1u : 0u;
    if (outs >= c.reward_thr) reward = std::fmin(reward + 1.0, 1.0);
    reward_sum += reward;
    for (uint64_t i = 0; i < n; ++i) {
      double inst = spiked[i] ? 1000.0 / dt : 0.0;
      firing_rates[i] += (inst - firing_rates[i]) * dt / 100.0;
    }
    double sr = 0;
    for (double r : firing_rates) sr += r;
    mean_rate = n ? sr / (double)n : 0.0;
    if (m) {
      double mean = 0;
      for (const LitSyn& y : syn) mean += y.weight;
      mean /= (double)m;
      double var = 0;
      for (const LitSyn& y : syn) var += (y.weight - mean) * (y.weight - mean);
      var /= (double)m;
      weight_mean = mean;
      weight_std = std::sqrt(var);
    }
    ++step;
  }
};

// plain weights in the frame of the next step
template <class R> void fast_weights(const Fast<R>* F, double* w) {
  R f[3] = {R(1), R(0), R(1)};
  if (F->c.cons) F->frame_of(F->step == F->cons_k0 ? 1.0 : F->consA_prev * F->cons_a, f);
  for (uint64_t q = 0; q < F->m; ++q) {
    R u = F->wget(q);
    w[q] = (double)(F->c.cons ? u * f[0] + f[1] : u);
  }
}

}  // namespace

extern "C" {

void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  philox(ctr, key, out);
}
float or_logf(float x) { return own_logf(x); }
float or_expf(float x) { return own_expf(x); }
void or_sincos2pi(float u, float* s, float* c) { own_sincos2pi(u, s, c); }

float or_drive_f32(const or_config* cfg, uint64_t n, const uint8_t* inhibitory, uint64_t i,
                   uint64_t k, float I_in) {
  DriveOut<float> d = neuron_drive<float>(*cfg, inhibitory, i, k);
  float I = I_in + d.add_I;
  std::vector<Kick> kk;
  global_kicks(*cfg, n, k, kk);
  for (const Kick& q : kk) if (q.target == i) I = I + q.amt_f;
  return cfg->drive_kind == 2 ? d.kick : (cfg->drive_kind == 4 ? d.add_g : I);
}

int or_lif_step_f64(double* v, int32_t* refr, const double p[6], double dt, double I) {
  if (*refr > 0) { *refr -= 1; return 0; }
  double dv = (-(*v - p[0]) + p[5] * I) * dt / p[3];
  *v += dv;
  if (*v >= p[1]) { *v = p[2]; *refr = (int32_t)std::round(p[4] / dt); return 1; }
  return 0;
}

int or_izh_step_f64(double* v, double* u, const double p[4], double dt, double I) {
  if (*v >= 30.0) { *v = p[2]; *u += p[3]; return 1; }
  double vv = *v, uu = *u;
  double dv = (0.04 * vv * vv + 5.0 * vv + 140.0 - uu + I) * dt;
  double du = p[0] * (p[1] * vv - uu) * dt;
  *v += dv;
  *u += du;
  return 0;
}

int or_hh_step_f64(double* v, double* m, double* h, double* n, const double p[7], double dt,
                   double I, int integrator) {
  return hh_step<double>(*v, *m, *h, *n, p, dt, I, integrator) ? 1 : 0;
}

double or_mg_block(int syn_type, double v) { return mg_block<double>(syn_type & 3, v); }

double or_dual_exp_conductance(int syn_type, double t) {
  // SynapseDynamics::conductance, types.rs:59-83
  int ty = syn_type & 3;
  if (t < 0.0) return 0.0;
  double tr = kRise[ty], td = kDyn[ty].decay, gmax = kDyn[ty].gmax;
  if (td <= 0.0 || tr <= 0.0) return 0.0;
  if (std::fabs(td - tr) < 1e-12) {
    double norm = tr * std::exp(-1.0);
    return gmax * t * std::exp(-t / tr) / norm;
  }
  double tpk = (tr * td / (td - tr)) * std::log(td / tr);
  double norm = std::exp(-tpk / td) - std::exp(-tpk / tr);
  if (norm <= 0.0) return 0.0;
  double g = (std::exp(-t / td) - std::exp(-t / tr)) / norm;
  return gmax * (g > 0.0 ? g : 0.0);
}

void or_trace_on_spike(double* trace, double* last, double time, double tau) {
  double d = time - *last;
  *trace = *trace * std::exp(-d / tau) + 1.0;
  *last = time;
}
void or_trace_decay(double* pre, double* post, double dt, double tau_plus, double tau_minus) {
  *pre *= std::exp(-dt / tau_plus);
  *post *= std::exp(-dt / tau_minus);
}
void or_eligibility_update(double* value, double dt, double tau_e, double delta) {
  *value = *value * std::exp(-dt / tau_e) + delta;
}
void or_eligibility_apply(double* value, double reward, double* w, double lr, double wmin,
                          double wmax) {
  *w = clampw<double>(*w + lr * reward * *value, wmin, wmax);
  *value = 0.0;
}
double or_stdp_weight_change(double a_plus, double a_minus, double tau_plus, double tau_minus,
                             double dt) {
  if (dt > 0.0) return a_plus * std::exp(-dt / tau_plus);
  return -a_minus * std::exp(dt / tau_minus);
}
void or_consolidation_apply(double* w, double tau_c, double target, double drift, double dt) {
  double d = (target - *w) * dt / tau_c;
  *w += d * drift;
}
double or_stp_step(double* u, double* r, double u_se, double tau_rec, double tau_facil, double dt,
                   int spike) {
  if (spike) {
    *u += u_se * (1.0 - *u) / tau_facil * dt;
    double epsp = *u * *r;
    *r -= epsp;
    return epsp;
  }
  *u += (u_se - *u) / tau_facil * dt;
  *r += (1.0 - *r) / tau_rec * dt;
  return 0.0;
}

void or_finalize_csr(uint64_t n, uint64_t m, const uint32_t* src, const uint32_t* tgt,
                     uint64_t* row_ptr, uint32_t* col) {
  // Network::finalize, src/network/mod.rs:79-106: degree count, prefix sum,
  // per-source write cursor in insertion order.
  std::vector<uint32_t> degree(n, 0);
  for (uint64_t s = 0; s < m; ++s) if (src[s] < n) degree[src[s]]++;
  row_ptr[0] = 0;
  uint64_t sum = 0;
  for (uint64_t i = 0; i < n; ++i) { sum += degree[i]; row_ptr[i + 1] = sum; }
  std::vector<uint64_t> cursor(row_ptr, row_ptr + n);
  for (uint64_t s = 0; s < m; ++s)
    if (src[s] < n) col[cursor[src[s]]++] = tgt[s];
}

void* or_fast_create(const or_config* cfg, const or_net* net, int32_t precision) {
  if (precision == 32) { auto* f = new Fast<float>(); f->init(*cfg, *net); return new std::pair<int, void*>(32, f); }
  auto* f = new Fast<double>(); f->init(*cfg, *net); return new std::pair<int, void*>(64, f);
}

#define FAST_DISPATCH(s, body)                                    \
  do {                                                            \
    auto* pr = (std::pair<int, void*>*)(s);                       \
    if (pr->first == 32) { auto* F = (Fast<float>*)pr->second; body; } \
    else { auto* F = (Fast<double>*)pr->second; body; }           \
  } while (0)

void or_fast_step(void* s, int32_t nsteps) {
  FAST_DISPATCH(s, for (int q = 0; q < nsteps; ++q) F->one_step(nullptr, 0, nullptr));
}
uint64_t or_fast_step_traced(void* s, uint64_t* pos_out, uint64_t cap) {
  uint64_t cnt = 0;
  FAST_DISPATCH(s, F->one_step(pos_out, cap, &cnt));
  return cnt;
}
uint64_t or_fast_log_size(void* s) { uint64_t r = 0; FAST_DISPATCH(s, r = F->log_idx.size()); return r; }
uint64_t or_fast_log_steps(void* s) { uint64_t r = 0; FAST_DISPATCH(s, r = F->log_off.size() - 1); return r; }
void or_fast_log(void* s, uint32_t* idx, uint64_t* offsets) {
  FAST_DISPATCH(s, {
    std::copy(F->log_idx.begin(), F->log_idx.end(), idx);
    std::copy(F->log_off.begin(), F->log_off.end(), offsets);
  });
}
void or_fast_state(void* s, double* v, double* u, double* m, double* h, double* n, double* I,
                   int32_t* refr, double* pre, double* post, int64_t* last) {
  FAST_DISPATCH(s, {
    for (uint64_t i = 0; i < F->n; ++i) {
      if (v) v[i] = (double)F->v[i];
      if (u) u[i] = (double)F->u[i];
      if (m) m[i] = (double)F->gm[i];
      if (h) h[i] = (double)F->gh[i];
      if (n) n[i] = (double)F->gn[i];
      if (I) I[i] = (double)F->I[i];
      if (refr) refr[i] = F->refr[i];
      if (pre) pre[i] = (double)F->pre[i];
      if (post) post[i] = (double)F->post[i];
      if (last) last[i] = F->last[i];
    }
  });
}
void or_fast_weights(void* s, double* w) { FAST_DISPATCH(s, fast_weights(F, w)); }
void or_fast_eligibility(void* s, double* e) {
  FAST_DISPATCH(s, for (uint64_t q = 0; q < F->m; ++q) e[q] = (double)F->e[q]);
}
void or_fast_reward(void* s, double* out2) {
  FAST_DISPATCH(s, {
    const double now = F->reward_now();
    out2[0] = now;
    out2[1] = F->reward_sum + (F->step > F->origin ? now : 0.0);
  });
}
void or_fast_apply_reward(void* s, double reward) { FAST_DISPATCH(s, F->apply_reward(reward)); }
void or_fast_rates(void* s, double* rates) {
  FAST_DISPATCH(s, std::copy(F->rate.begin(), F->rate.end(), rates));
}
uint64_t or_fast_events(void* s) { uint64_t r = 0; FAST_DISPATCH(s, r = F->events); return r; }
double or_fast_lfp(void* s) { double r = 0; FAST_DISPATCH(s, r = F->lfp()); return r; }
void or_fast_add_input_current(void* s, uint64_t count, const uint32_t* ids, const double* amounts) {
  FAST_DISPATCH(s, F->add_input_current(count, ids, amounts));
}
// SimulationEngine::stimulate (engine.rs:156-161): input_current += amount
void or_lit_add_input_current(void* s, uint64_t count, const uint32_t* ids, const double* amounts) {
  Lit* L = (Lit*)s;
  for (uint64_t q = 0; q < count; ++q)
    if (ids[q] < L->n) L->I[ids[q]] += amounts[q];
}
void or_fast_destroy(void* s) {
  auto* pr = (std::pair<int, void*>*)s;
  if (pr->first == 32) delete (Fast<float>*)pr->second; else delete (Fast<double>*)pr->second;
  delete pr;
}

void* or_lit_create(const or_config* cfg, const or_net* net, int32_t threads) {
  auto* L = new Lit();
  L->init(*cfg, *net, threads);
  return L;
}
void or_lit_step(void* s, int32_t nsteps) {
  for (int q = 0; q < nsteps; ++q) ((Lit*)s)->one_step();
}
uint64_t or_lit_log_size(void* s) { return ((Lit*)s)->log_idx.size(); }
uint64_t or_lit_log_steps(void* s) { return ((Lit*)s)->log_off.size() - 1; }
void or_lit_log(void* s, uint32_t* idx, uint64_t* offsets) {
  Lit* L = (Lit*)s;
  std::copy(L->log_idx.begin(), L->log_idx.end(), idx);
  std::copy(L->log_off.begin(), L->log_off.end(), offsets);
}
void or_lit_state(void* s, double* v, double* u, double* m, double* h, double* n, double* I) {
  Lit* L = (Lit*)s;
  for (uint64_t i = 0; i < L->n; ++i) {
    if (v) v[i] = L->v[i];
    if (u) u[i] = L->u[i];
    if (m) m[i] = L->gm[i];
    if (h) h[i] = L->gh[i];
    if (n) n[i] = L->gn[i];
    if (I) I[i] = L->I[i];
  }
}
// Warm start (timing samples only): neuron state, per-neuron STDP traces
// and last spike times (each plastic synapse takes its source's pre-trace
// and its target's post-trace, the per-neuron reformulation), weights, the
// clock and the step count. Pending delayed input starts empty.
void or_lit_set_state(void* s, const double* v, const double* u, const double* pre,
                      const double* post, const double* last_spike_time, const double* w,
                      double time, uint64_t step) {
  Lit* L = (Lit*)s;
  for (uint64_t i = 0; i < L->n; ++i) {
    if (v) L->v[i] = v[i];
    if (u) L->u[i] = u[i];
    if (last_spike_time) L->last_spike_time[i] = last_spike_time[i];
  }
  for (uint64_t q = 0; q < L->m; ++q) {
    LitSyn& y = L->syn[q];
    if (w) y.weight = w[q];
    if (pre) y.pre_trace = pre[y.source];
    if (post) y.post_trace = post[y.target];
    if (last_spike_time) {
      y.last_pre = last_spike_time[y.source];
      y.last_post = last_spike_time[y.target];
    }
  }
  std::fill(L->ring.begin(), L->ring.end(), 0.0);
  L->time = time;
  L->step = step;
}

void or_lit_weights(void* s, double* w) {
  Lit* L = (Lit*)s;
  for (uint64_t q = 0; q < L->m; ++q) w[q] = L->syn[q].weight;
}
void or_lit_rates(void* s, double* rates) {
  Lit* L = (Lit*)s;
  std::copy(L->firing_rates.begin(), L->firing_rates.end(), rates);
}
uint64_t or_lit_events(void* s) { return ((Lit*)s)->events; }
void or_lit_stats(void* s, double* out8) {
  Lit* L = (Lit*)s;
  out8[0] = (double)L->total_spikes; out8[1] = L->time; out8[2] = L->mean_rate;
  out8[3] = L->weight_mean; out8[4] = L->weight_std; out8[5] = L->lfp;
  out8[6] = (double)L->events; out8[7] = (double)L->step;
}
void or_lit_eligibility(void* s, double* e) {
  Lit* L = (Lit*)s;
  for (uint64_t q = 0; q < L->m; ++q) e[q] = L->syn[q].e;
}
void or_lit_reward(void* s, double* out2) {
  Lit* L = (Lit*)s;
  out2[0] = L->reward;
  out2[1] = L->reward_sum;
}
// SimulationEngine::apply_reward, engine.rs:158-175
void or_lit_apply_reward(void* s, double reward) {
  Lit* L = (Lit*)s;
  if (!L->c.rstdp) return;
  for (LitSyn& y : L->syn)
    if (y.elig) or_eligibility_apply(&y.e, reward, &y.weight, L->c.rstdp_lr, L->c.rstdp_wmin, L->c.rstdp_wmax);
}
void or_lit_destroy(void* s) { delete (Lit*)s; }

}  // extern "C"
