/*
 * ORACLE — test infrastructure only. CPU restatement of NeuralSim's
 * SimulationEngine::step hot path (src/simulation/engine.rs:254-697) and the
 * neuron / synapse / plasticity modules it calls. Only tests/, the smoke
 * check and bench.py's CPU-baseline leg may load this library; the product
 * (neuralsim_b200) never links or calls it.
 *
 * Parity pinning: the reference is a Rust crate and this image has no Rust
 * toolchain, so the oracle cannot be checked against reference-generated
 * vectors. It is pinned against every known-answer test the reference's own
 * unit tests hold for this path (lif.rs:68-100, izhikevich.rs:73-91,
 * hodgkin_huxley.rs:117-164, types.rs:114-205, plasticity.rs:320-398,
 * engine.rs:826-895) and against the published Philox4x32-10 test vectors.
 * Spike-raster parity beyond those is "parity pinned by restatement".
 *
 * Two engines:
 *  - or_lit_*  : literal restatement, FP64, per-synapse state, the reference
 *                loop structure (O(M) conductance / STDP / homeostasis /
 *                weight-stat loops); OpenMP over neurons as rayon does.
 *  - or_fast_* : per-neuron-trace / per-target-conductance reformulation,
 *                templated on float (bit-for-bit mirror of the device
 *                arithmetic, int64 fixed-point synaptic sums) or double.
 */
#ifndef NS_ORACLE_H
#define NS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_config {
  int32_t model;          /* 0 LIF, 1 IZH, 2 HH */
  int32_t input_mode;     /* 0 DIRECT_DECAY, 1 DELTA_V, 2 RESET, 3 COND_REF, 4 COND_FRESH */
  int32_t hh_integrator;  /* 0 Euler (reference), 1 Rush-Larsen */
  int32_t weight_format;  /* 0 f32, 1 bf16 storage */
  double dt;
  int32_t delay_steps;
  int32_t pad0;
  uint64_t seed;
  double current_decay;
  int32_t stdp;
  int32_t pad1;
  double tau_plus, tau_minus, a_plus, a_minus, w_min, w_max;
  int32_t homeo;
  int32_t pad2;
  double h_target, h_tau, contrib_tau;
  /* drive */
  int32_t drive_kind;
  int32_t kick_min, kick_max;
  int32_t pad3;
  double p, amp, sigma_exc, sigma_inh, kick_chance, kick_strength;
  /* R-STDP and consolidation (engine.rs:519-563, :626-631) */
  int32_t rstdp, cons;
  double rstdp_lr, rstdp_wmin, rstdp_wmax, elig_tau;
  uint64_t reward_thr;
  double reward_decay, reward_init;
  double cons_tau, cons_target, cons_drift;
  /* firing-rate estimate kept without homeostasis too (engine.rs:637-642;
   * the literal engine always keeps it) */
  int32_t track_rates;
  int32_t pad4;
} or_config;

typedef struct or_net {
  uint64_t n, m;
  const uint64_t* row_ptr;
  const uint32_t* col;
  const float* w;
  const uint8_t* syn_type;   /* may be NULL: AMPA */
  const uint8_t* plastic;    /* may be NULL: none */
  const float* params;       /* n * ppn */
  int32_t ppn;
  int32_t pad;
  const uint8_t* inhibitory; /* may be NULL */
  const uint8_t* is_output;  /* may be NULL */
  const float* v0;           /* may be NULL */
  const float* u0;
  const float* m0;
  const float* h0;
  const float* n0;
  const uint8_t* eligible;   /* may be NULL: every plastic synapse (R-STDP) */
  const double* stp;         /* m rows (u_se, tau_rec, tau_facil, u, r) or NULL */
  const uint8_t* has_stp;    /* may be NULL: every synapse (when stp given) */
} or_net;

/* ---- Philox4x32-10 and drive math (restated) ---- */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float or_logf(float x);
float or_expf(float x);
void or_sincos2pi(float u, float* s, float* c);
/* drive value of neuron i at step k as the float engine computes it
 * (current added; for POISSON_KICK the kick) */
float or_drive_f32(const or_config* cfg, uint64_t n, const uint8_t* inhibitory, uint64_t i,
                   uint64_t k, float I_in);

/* ---- single-model steps (FP64 restatements of the model files) ---- */
int or_lif_step_f64(double* v, int32_t* refr, const double p[6], double dt, double I);
int or_izh_step_f64(double* v, double* u, const double p[4], double dt, double I);
int or_hh_step_f64(double* v, double* m, double* h, double* n, const double p[7], double dt,
                   double I, int integrator);
double or_mg_block(int syn_type, double v);
double or_dual_exp_conductance(int syn_type, double t);
void or_trace_on_spike(double* trace, double* last, double time, double tau);
void or_trace_decay(double* pre, double* post, double dt, double tau_plus, double tau_minus);
void or_eligibility_update(double* value, double dt, double tau_e, double delta);
void or_eligibility_apply(double* value, double reward, double* w, double lr, double wmin,
                          double wmax);
double or_stdp_weight_change(double a_plus, double a_minus, double tau_plus, double tau_minus,
                             double dt);
void or_consolidation_apply(double* w, double tau_c, double target, double drift, double dt);
double or_stp_step(double* u, double* r, double u_se, double tau_rec, double tau_facil, double dt,
                   int spike);

/* ---- CSR construction (Network::finalize, src/network/mod.rs:79-106) ---- */
void or_finalize_csr(uint64_t n, uint64_t m, const uint32_t* src, const uint32_t* tgt,
                     uint64_t* row_ptr, uint32_t* col);

/* ---- engines ---- */
void* or_fast_create(const or_config* cfg, const or_net* net, int32_t precision);
void or_fast_step(void* s, int32_t nsteps);
/* runs one step and records propagation CSR positions in traversal order */
uint64_t or_fast_step_traced(void* s, uint64_t* pos_out, uint64_t cap);
uint64_t or_fast_log_size(void* s);
uint64_t or_fast_log_steps(void* s);
void or_fast_log(void* s, uint32_t* idx, uint64_t* offsets);
void or_fast_state(void* s, double* v, double* u, double* m, double* h, double* n, double* I,
                   int32_t* refr, double* pre, double* post, int64_t* last);
void or_fast_weights(void* s, double* w);
void or_fast_rates(void* s, double* rates);
uint64_t or_fast_events(void* s);
/* lfp_signal (engine.rs:492) in the reference conductance mode, as the
 * device sums it (0 in the other modes) */
double or_fast_lfp(void* s);
/* host stimulus: the device's arithmetic (fast) and SimulationEngine::
 * stimulate, engine.rs:156-161 (literal) */
void or_fast_add_input_current(void* s, uint64_t count, const uint32_t* ids, const double* amounts);
void or_lit_add_input_current(void* s, uint64_t count, const uint32_t* ids, const double* amounts);
/* eligibility values (m), reward now and the sum of the reward after each
 * step (out2), and SimulationEngine::apply_reward as the device does it */
void or_fast_eligibility(void* s, double* e);
void or_fast_reward(void* s, double* out2);
void or_fast_apply_reward(void* s, double reward);
void or_fast_destroy(void* s);

void* or_lit_create(const or_config* cfg, const or_net* net, int32_t threads);
void or_lit_step(void* s, int32_t nsteps);
uint64_t or_lit_log_size(void* s);
uint64_t or_lit_log_steps(void* s);
void or_lit_log(void* s, uint32_t* idx, uint64_t* offsets);
void or_lit_state(void* s, double* v, double* u, double* m, double* h, double* n, double* I);
void or_lit_set_state(void* s, const double* v, const double* u, const double* pre,
                      const double* post, const double* last_spike_time, const double* w,
                      double time, uint64_t step);
void or_lit_weights(void* s, double* w);
void or_lit_rates(void* s, double* rates);
uint64_t or_lit_events(void* s);
void or_lit_stats(void* s, double* out8);
void or_lit_eligibility(void* s, double* e);
void or_lit_reward(void* s, double* out2);
void or_lit_apply_reward(void* s, double reward);
void or_lit_destroy(void* s);

#ifdef __cplusplus
}
#endif
#endif
