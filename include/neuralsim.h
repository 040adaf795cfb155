/*
 * neuralsim.h — C ABI of the B200 step backend for NeuralSim's per-timestep
 * hot path (neuron-state update, CSR spike propagation, trace STDP).
 *
 * This is the drop-in seam for the reference crate's `GpuBackend`
 * (src/simulation/gpu_backend.rs:47-1036), which `SimulationEngine::step`
 * dispatches to at src/simulation/engine.rs:255-258 and which
 * `SimulationEngine::init_gpu` builds at src/simulation/engine.rs:181-252.
 *
 * Conventions
 *  - Every function returns an ns_status (0 = NS_OK) and never throws or
 *    aborts across the ABI. ns_last_error() gives the message of the last
 *    failing call on a handle (the reference's GpuError strings,
 *    gpu_backend.rs:25-39, map onto NS_ERR_NO_DEVICE / NS_ERR_CUDA).
 *  - The host owns every pointer it passes in; data is copied. The handle
 *    owns all device memory and one CUDA stream.
 *  - One handle is not thread-safe (the reference guards its engine with a
 *    Mutex, src/simulation/scheduler.rs:23); distinct handles may be driven
 *    from distinct threads.
 *  - There is no CPU fallback: without a usable CUDA device ns_create fails
 *    with NS_ERR_NO_DEVICE.
 */
#ifndef NEURALSIM_H
#define NEURALSIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t ns_status;
#define NS_OK                  0
#define NS_ERR_INVALID_ARG     1
#define NS_ERR_NULL_HANDLE     2
#define NS_ERR_CSR             3  /* row_ptr not monotone, col >= n, m mismatch */
#define NS_ERR_OOM             4
#define NS_ERR_CUDA            5
#define NS_ERR_DEVICE_TIMEOUT  6  /* a bounded device-side wait gave up */
#define NS_ERR_STATE           7  /* call out of order (e.g. step before upload) */
#define NS_ERR_UNSUPPORTED     8
#define NS_ERR_NONFINITE       9  /* NaN/Inf in uploaded state or parameters */
#define NS_ERR_SPIKE_LOG_FULL 10  /* spike log capacity exceeded; stepping went on */
#define NS_ERR_NO_DEVICE      11

typedef struct ns_handle ns_handle;

/* Neuron models: NeuronModelParams::{Lif, Izhikevich, HodgkinHuxley},
 * src/neuron/mod.rs:71-94. One model per handle. Per-neuron parameter rows:
 *   LIF (6): resting, threshold, reset, tau_m, refractory_period, input_resistance
 *   IZH (4): a, b, c, d
 *   HH  (7): g_na, g_k, g_l, e_na, e_k, e_l, c_m                               */
enum ns_model { NS_MODEL_LIF = 0, NS_MODEL_IZHIKEVICH = 1, NS_MODEL_HH = 2 };

/* How synaptic input reaches the neuron.
 *  DIRECT_DECAY     reference current mode: I += w per event, I *= current_decay
 *                   at the end of every step (engine.rs:456-471, :609-614).
 *  DELTA_V          each delivered weight is a voltage kick added right after
 *                   the model's integration step.
 *  RESET_EACH_STEP  I = drive + sum of delivered weights, fresh every step.
 *  CONDUCTANCE_REF  reference conductance mode: per-type conductances decay by
 *                   exp(-dt/tau), events add w*gmax*mg(V) (|.| for GABA types),
 *                   I += sum g*(E_rev - V), I never cleared (engine.rs:406-494).
 *  CONDUCTANCE_FRESH per-target conductances as above, but the synaptic current
 *                   is recomputed every step: I = sum g*(E_rev - V) + drive.   */
enum ns_input_mode {
  NS_INPUT_DIRECT_DECAY = 0,
  NS_INPUT_DELTA_V = 1,
  NS_INPUT_RESET_EACH_STEP = 2,
  NS_INPUT_CONDUCTANCE_REF = 3,
  NS_INPUT_CONDUCTANCE_FRESH = 4
};

/* HH integrator: EULER_REF is HodgkinHuxleyNeuron::step (forward-Euler gates,
 * spike when V >= -55 then V = -70, src/neuron/hodgkin_huxley.rs:46-96);
 * RUSH_LARSEN integrates the gates exactly for frozen V and reports a spike on
 * an upward 0 mV crossing without reset.                                      */
enum ns_hh_integrator { NS_HH_EULER_REF = 0, NS_HH_RUSH_LARSEN = 1 };

enum ns_weight_format { NS_WEIGHT_F32 = 0, NS_WEIGHT_BF16 = 1 };

/* SynapseType, src/synapse/mod.rs:22-28; constants src/synapse/types.rs:15-54. */
enum ns_syn_type { NS_SYN_AMPA = 0, NS_SYN_GABA = 1, NS_SYN_GABA_B = 2, NS_SYN_NMDA = 3 };

/* Drive (background input), replacing the host-side noise loop of
 * engine.rs:273-287 with counter-based Philox4x32-10 streams keyed by
 * (seed, step, neuron), so device and host produce the same numbers.
 *  REF_UNIFORM   per neuron: with probability p, I += U*amplitude; then with
 *                probability kick_chance, kick_min..kick_max random neurons
 *                get I += U*kick_strength (the reference's drive shape).
 *  POISSON_KICK  with probability p per neuron-step, add amplitude (a voltage
 *                kick in DELTA_V mode, a current otherwise).
 *  GAUSS         I += sigma*N(0,1), sigma_exc / sigma_inh by neuron type.
 *  POISSON_CONDUCTANCE with probability p per neuron-step, add amplitude to
 *                the neuron's AMPA conductance (conductance modes only).    */
enum ns_drive_kind {
  NS_DRIVE_NONE = 0,
  NS_DRIVE_REF_UNIFORM = 1,
  NS_DRIVE_POISSON_KICK = 2,
  NS_DRIVE_GAUSS = 3,
  NS_DRIVE_POISSON_CONDUCTANCE = 4
};

typedef struct ns_drive {
  uint32_t kind;
  float p;
  float amplitude;
  float sigma_exc;
  float sigma_inh;
  float kick_chance;
  float kick_strength;
  uint32_t kick_min;
  uint32_t kick_max;
} ns_drive;

/* Mirrors SimulationConfig (src/config/mod.rs:61-68) + PlasticityConfig /
 * StdpRule (src/synapse/mod.rs:122-157, src/synapse/plasticity.rs:8-28). */
typedef struct ns_config {
  uint32_t model;          /* ns_model */
  uint32_t input_mode;     /* ns_input_mode */
  uint32_t hh_integrator;  /* ns_hh_integrator */
  uint32_t weight_format;  /* ns_weight_format */
  double dt_ms;
  uint32_t delay_steps;    /* >= 1; 1 = the reference (delivery at the next update) */
  int32_t device;          /* CUDA ordinal */
  uint64_t seed;
  double current_decay;    /* DIRECT_DECAY factor, 0.92 in the reference */
  /* pair STDP (StdpRule) */
  int32_t stdp_enabled;
  double tau_plus, tau_minus, a_plus, a_minus, w_min, w_max;
  /* homeostatic scaling (engine.rs:569-606) */
  int32_t homeostasis_enabled;
  double homeostatic_target_rate, homeostatic_tau, contribution_tau;
  /* spike log (the StepResult.spiking_neurons stream, engine.rs:35-41) */
  uint64_t spike_log_capacity; /* indices held; 0 = no log */
  uint32_t spike_log_steps;    /* steps held */
  uint32_t graph_chunk;        /* steps per captured CUDA graph; 0 = 1000 */
  /* kernel schedule of a step: 0 = autotune (time every candidate on live
   * steps, keep the fastest), 1 = fused (row walks and LTD lists in one
   * kernel, 6 resident blocks per SM), 2 = split (LTD of step k on a second
   * stream beside the neuron update of step k+1), 3 = fused with 4 resident
   * blocks per SM, 4 = split with a narrow (2 blocks/SM) LTD grid that leaves
   * room for the neuron kernel, 5 = deferred LTD: the LTD of synapse j->i
   * at a spike of i waits, as a bit in i's 32-step spike history, until j's
   * row is next walked (at j's spike, before delivery) or flushed (every
   * row once per 32 steps, a 32nd of the rows per step, beside the walks),
   * so LTD reads and writes weights in CSR order instead of at random
   * positions. Schedule 5 applies to pair STDP on one GPU (no homeostasis,
   * R-STDP, consolidation or STP; schedule 3 is run otherwise). All give
   * bit-identical results. */
  uint32_t step_schedule;
  /* windowed stepping for delay_steps >= 2 without STDP or homeostasis: W
   * steps per neuron kernel (W <= delay_steps), one row-walk pass per window.
   * 0 = on, W tuned at the first ns_step among delay_steps (capped at 1024)
   * and its successive halves down to 2 (ns_get_window), 1 = off (one pass
   * per step), W > 1 = on with that W. Results are identical either way. */
  uint32_t window_steps;
  /* R-STDP (RStdpRule / EligibilityTrace, src/synapse/plasticity.rs:166-221).
   * A synapse that carries an eligibility trace updates it at each of its
   * STDP updates: e = e*exp(-dt/eligibility_tau) + delta, delta being the
   * unclamped weight change (engine.rs:519-533, where the engine passes 200
   * ms). While |reward| > 0.001 at a step, every such synapse takes
   * w = clamp(w + rstdp_lr*reward*e, rstdp_w_min, rstdp_w_max) and e = 0
   * after the step's STDP and consolidation (engine.rs:546-561). The reward
   * decays by reward_decay per step whenever any plasticity is on
   * (engine.rs:563) and becomes min(reward + 1, 1) after a step with at
   * least reward_threshold output spikes (engine.rs:626-631); reward_signal
   * is its value before the first step (with_reward_signal, :151-154). */
  int32_t rstdp_enabled;
  double rstdp_lr, rstdp_w_min, rstdp_w_max, eligibility_tau;
  uint64_t reward_threshold;
  double reward_decay, reward_signal;
  /* Consolidation (ConsolidationRule, plasticity.rs:269-290), applied to
   * every synapse after STDP each step (engine.rs:539-545):
   * w += (consolidation_target - w) * dt / consolidation_tau * consolidation_drift.
   * The device keeps this O(1) per step: weights are stored in a per-step
   * affine frame (see ns_download_state for the plain values). */
  int32_t consolidation_enabled;
  double consolidation_tau, consolidation_target, consolidation_drift;
  /* Per-neuron firing-rate estimate kept every step without homeostasis too
   * (SimulationEngine::firing_rate / mean_firing_rate, engine.rs:637-645,
   * :809-826; FP64, r += (1000/dt * spiked - r) * dt/100). Homeostasis keeps
   * it in any case. Tracking runs the step path (no windowed stepping). */
  uint32_t track_rates;
} ns_config;

/* Fills cfg with the reference defaults: LIF, DIRECT_DECAY, dt 0.5 ms
 * (engine.rs:96), decay 0.92, StdpRule::default, homeostasis 5 Hz / 5000 ms,
 * contribution_tau 1000 ms, seed 42 (engine.rs:99); R-STDP and consolidation
 * off with RStdpRule::default / ConsolidationRule::default parameters
 * (plasticity.rs:177-189, :276-284), eligibility tau 200 ms, reward
 * threshold 5 and decay 0.95 (engine.rs:113-116). */
void ns_config_default(ns_config* cfg);

/* Neuron SoA (NeuronArray, src/neuron/mod.rs:126-163, in f32 as init_gpu
 * uploads it, engine.rs:190-238). Unused arrays may be NULL on upload
 * (defaults: v = model rest, u = 0, refractory = 0, current = 0, gates
 * 0.05/0.6/0.32, traces 0, last spike never). On download every non-NULL
 * pointer is filled. */
typedef struct ns_neuron_soa {
  uint64_t n;
  float* v;
  float* u;
  int32_t* refractory;
  float* current;
  float* hh_m;
  float* hh_h;
  float* hh_n;
  float* params;              /* n * params_per_neuron */
  uint32_t params_per_neuron; /* 6 LIF, 4 IZH, 7 HH */
  uint8_t* inhibitory;        /* NeuronType::Inhibitory flag (drive sigma) */
  uint8_t* is_output;
  float* pre_trace;           /* per-neuron STDP traces */
  float* post_trace;
  int64_t* last_spike_step;   /* -1 = never */
  /* exact resume: synaptic input already propagated but not yet delivered,
   * fixed point 2^-40, layout [type][delay slot][n] with 1 type in current
   * modes and 4 (AMPA, GABA, GABA-B, NMDA) in conductance modes */
  int64_t* pending_input;
  float* conductance;         /* [4][n] per-target conductances */
  double* firing_rate;        /* per-neuron rate estimate (homeostasis) */
} ns_neuron_soa;

typedef struct ns_step_stats {
  uint64_t steps_done;        /* total steps since creation / state upload */
  uint64_t spikes;            /* spikes during this call */
  uint64_t output_spikes;
  uint64_t events;            /* synaptic events (sum of out-degree of spikers) */
  uint64_t last_step_spikes;
  double sim_time_ms;         /* FP64 device clock (engine.rs:388-389) */
  uint64_t max_step_spikes;   /* largest spike count of one step since creation /
                                 state upload (SimulationStats::active_neurons,
                                 engine.rs:624) */
} ns_step_stats;

/* --- lifecycle: GpuBackend::new, gpu_backend.rs:98-124 ------------------ */
ns_status ns_create(const ns_config* cfg, ns_handle** out);
ns_status ns_destroy(ns_handle* h);
const char* ns_last_error(const ns_handle* h);
const char* ns_status_string(ns_status s);
ns_status ns_device_count(int* count);

/* --- uploads: GpuBackend::upload_initial_state / upload_csr,
 *     gpu_backend.rs:640-688 (called from engine.rs:240-247) --------------- */
ns_status ns_upload_neurons(ns_handle* h, const ns_neuron_soa* soa);
/* CSR by source (Network::finalize, src/network/mod.rs:79-106). Synapse
 * arrays MUST already be in CSR order. syn_type NULL = AMPA for all;
 * plastic NULL = no plastic synapse. Validated: row_ptr[0]==0, monotone,
 * row_ptr[n]==m, col<n, weights finite. */
ns_status ns_upload_csr(ns_handle* h, uint64_t n, uint64_t m, const uint64_t* row_ptr,
                        const uint32_t* col, const float* w, const uint8_t* syn_type,
                        const uint8_t* plastic);
/* Drive: the noise loop of engine.rs:273-287 (host RNG in the reference). */
ns_status ns_set_drive(ns_handle* h, const ns_drive* d);

/* --- batches: many independent networks in one launch ------------------
 * Replaces the per-genome engines of Population::evolve_generation
 * (src/evolution/population.rs:117-124) and one-engine-per-point parameter
 * sweeps. One network of a batch: its neuron SoA (the same fields and
 * defaults as ns_upload_neurons), its CSR in local indices (the same rules as
 * ns_upload_csr) and the seed of its own drive stream. */
typedef struct ns_net_desc {
  const ns_neuron_soa* neurons;
  uint64_t m;
  const uint64_t* row_ptr;   /* n + 1 entries, row_ptr[0] == 0, row_ptr[n] == m */
  const uint32_t* col;       /* m local target indices < n */
  const float* w;            /* m */
  const uint8_t* syn_type;   /* m or NULL; all networks give it or none */
  const uint8_t* plastic;    /* m or NULL; all networks give it or none */
  uint64_t seed;             /* drive stream: the stream a lone handle with
                                ns_config.seed == seed would draw */
} ns_net_desc;
/* Concatenates the networks block-diagonally (network q owns neurons
 * first_neuron_out[q] .. first_neuron_out[q+1]-1 of the handle) and uploads
 * them. Every step kernel then runs over all networks at once; network q
 * draws its drive from its own seed and its local neuron indices, so its
 * raster equals the one it produces alone on a handle with the same config
 * and seed. Spike logs, state and weights use the concatenated indices.
 * first_neuron_out: n_nets + 1 entries or NULL. The reference-uniform drive
 * (global kicks per network) is not available for batches
 * (NS_ERR_UNSUPPORTED at ns_step). A later ns_upload_neurons ends batch
 * mode. A batch of the same networks' sizes reuses the device buffers. */
ns_status ns_upload_batch(ns_handle* h, uint32_t n_nets, const ns_net_desc* nets,
                          uint64_t* first_neuron_out);

/* --- stepping: SimulationEngine::step / simulate_ms, engine.rs:254-680,
 *     :792-797; GpuBackend::step_neurons + step_spmv, gpu_backend.rs:852-981.
 *     Runs n_steps on the device (CUDA-graph chunks) and blocks until done. */
ns_status ns_step(ns_handle* h, uint32_t n_steps, ns_step_stats* out);

/* Spike log: ascending neuron indices per step (StepResult.spiking_neurons).
 * Copies steps [first_step, first_step+n_steps) of the log; offsets_out has
 * n_steps+1 entries relative to the first copied index. */
ns_status ns_read_spikes(ns_handle* h, uint64_t first_step, uint32_t n_steps, uint32_t* idx_out,
                         uint64_t* offsets_out, uint64_t cap, uint64_t* n_written);
ns_status ns_clear_spike_log(ns_handle* h);
/* First step held in the log and number of steps held. */
ns_status ns_spike_log_range(ns_handle* h, uint64_t* first_step, uint64_t* n_steps);

/* --- state: checkpoint / resume (io/checkpoint.rs keeps the Network only;
 *     here the device state round-trips exactly, step counter included) ---
 * ns_download_state copies the fields of `out` that are not NULL; with w_out
 * not NULL it first applies every pending deferred LTD (schedule 5), which
 * the neuron state does not depend on. */
ns_status ns_download_state(ns_handle* h, ns_neuron_soa* out, float* w_out);
ns_status ns_upload_state(ns_handle* h, const ns_neuron_soa* in, const float* w_in,
                          uint64_t step);
/* Current global step index (the Philox counter and STDP clock). */
ns_status ns_get_step(ns_handle* h, uint64_t* step);
/* Per-neuron firing-rate estimate (engine.rs:637-642), FP64 on the device;
 * maintained when homeostasis or track_rates is enabled (zeros otherwise). */
ns_status ns_download_rates(ns_handle* h, double* rates_out);
/* Mean firing rate (Hz) of every network of the handle (n_nets entries; 1
 * for a single network) over the logged steps first_step .. first_step +
 * n_steps - 1, as the reference's per-neuron rate estimate averaged over a
 * network's neurons reports it after those steps from rate 0
 * (engine.rs:637-645: r += (1000/dt * spiked - r) * dt/100 each step). The
 * fitness of Population::evolve_generation's RateHomeostasis evaluator
 * (src/evolution/fitness.rs:59-76) is a function of it. Computed on the
 * device from the spike log. */
ns_status ns_network_rates(ns_handle* h, uint64_t first_step, uint32_t n_steps, double* mean_rate_out);

/* Weight mean / std over all synapses (engine.rs:658-669), on demand. */
ns_status ns_weight_stats(ns_handle* h, double* mean, double* stddev);
/* The engine's LFP signal (lfp_signal, engine.rs:64, :492): the sum over
 * steps and synapses of |g (E_rev - V)| in the reference conductance mode,
 * since creation or the last state upload (0 in the other modes). Each
 * neuron's per-type conductance stands for the sum of its synapses'
 * (conductances are >= 0: GABA types take |w|). */
ns_status ns_get_lfp(ns_handle* h, double* lfp);
/* Host stimulus: adds amounts[q] to the input current of neuron ids[q]
 * (SimulationEngine::stimulate, engine.rs:156-161; the host-side edit that
 * GpuBackend::upload_input_current carries, gpu_backend.rs). Amounts are
 * summed per neuron in call order (as float) and join the input current of
 * the next step after the synaptic input, before that step's drive. In the
 * modes whose input current is state (DIRECT_DECAY, CONDUCTANCE_REF) it then
 * stays and decays as the reference's input_current does; in the others it
 * acts for one step. A sharded rank keeps the ids it owns. Refused while a
 * learned HH macro-step is attached. */
ns_status ns_add_input_current(ns_handle* h, uint64_t count, const uint32_t* ids,
                               const double* amounts);

/* --- the rest of phase 2: R-STDP eligibility and reward, short-term
 *     plasticity (engine.rs:457-463, :519-563, :626-631) ---------------- */
/* Which synapses carry an eligibility trace (SynapseState.eligibility is
 * Some, src/synapse/mod.rs:72, set by with_rstdp, :114-119) and its values,
 * CSR order. eligible NULL = every plastic synapse; values NULL = 0. Needs
 * rstdp_enabled; ns_upload_csr resets to (every plastic synapse, 0). */
ns_status ns_upload_eligibility(ns_handle* h, const uint8_t* eligible, const float* values);
/* Current eligibility values (m floats; 0 for synapses without a trace). */
ns_status ns_download_eligibility(ns_handle* h, float* values_out);
/* Per-synapse contribution averages of homeostatic scaling
 * (SynapseState.contribution_avg, src/synapse/mod.rs:79, kept at delivery,
 * engine.rs:448-452, :465-469), m floats in CSR order: for checkpoints.
 * Download gives zeros without homeostasis; upload needs it enabled. */
ns_status ns_download_contributions(ns_handle* h, float* values_out);
ns_status ns_upload_contributions(ns_handle* h, const float* values);
/* SimulationEngine::apply_reward (engine.rs:158-175): every eligible synapse
 * takes w = clamp(w + rstdp_lr*reward*e, rstdp_w_min, rstdp_w_max), e = 0,
 * now, whatever the size of reward. */
ns_status ns_apply_reward(ns_handle* h, double reward);
/* The engine's reward_signal now (after the last step's phase 3), and the
 * sum over the steps since creation / the last ns_set_reward of the reward
 * after each step (RewardAccumulation's fitness, evolution/fitness.rs:110-118).
 * Maintained by the step-synchronous path when R-STDP or consolidation is
 * on; NS_ERR_UNSUPPORTED otherwise, after windowed steps and for batches. */
ns_status ns_get_reward(ns_handle* h, double* reward, double* reward_sum);
/* Sets reward_signal (with_reward_signal) and clears the sum. */
ns_status ns_set_reward(ns_handle* h, double reward);
/* Short-term plasticity (Tsodyks-Markram ShortTermPlasticity,
 * plasticity.rs:85-116). In the current modes the reference scales each
 * delivered weight by the EPSP of one step of a COPY of the synapse's STP
 * state (engine.rs:457-463); the copy is dropped, so the factor
 * (u + u_se*(1-u)/tau_facil*dt) * r is a per-synapse constant, taken in
 * every non-conductance input mode (conductance mode ignores STP, as the
 * reference does). stp: m rows (u_se, tau_rec, tau_facil, u, r), CSR order;
 * has_stp NULL = every synapse has STP. stp NULL removes STP. */
ns_status ns_upload_stp(ns_handle* h, const uint8_t* has_stp, const double* stp);

/* --- traversal trace: runs ONE step and records the CSR position of every
 *     propagation event in traversal order (spikers ascending, each row in
 *     CSR order). For parity tests of the CSR walk. */
ns_status ns_step_traced(ns_handle* h, uint64_t* pos_out, uint64_t cap, uint64_t* n_events);

/* Schedule in use (0 while the autotuner has not decided) and the measured
 * microseconds per step of schedules 1..5 in us_per_step[5] (0 if untimed). */
ns_status ns_get_schedule(ns_handle* h, uint32_t* schedule, double* us_per_step);

/* Windowed stepping: the window length in use (0 = step-synchronous), and
 * the candidates the window tuner timed with their microseconds per step
 * (0 where untimed). The tuner runs at the first ns_step when
 * ns_config.window_steps is 0. */
ns_status ns_get_window(ns_handle* h, uint32_t* window, uint32_t* candidates, double* us_per_step);

/* Windowed stepping: the shape of the window's row walk, which the window
 * tuner picks per network after the window length. lanes = lanes walking one
 * spiking row (32, 16 or 8: a warp has 32/lanes rows in flight),
 * blocks_per_sm = the walk's grid per SM. The candidates timed (lanes,
 * blocks per SM with 0 = the occupancy limit) and their microseconds per
 * step in cand_*[4] and us_per_step[4] (0 where untimed). Every shape gives
 * the same results (integer accumulation). 0s when stepping is not
 * windowed. No reference counterpart: the reference walks on the host. */
ns_status ns_get_walk_shape(ns_handle* h, uint32_t* lanes, uint32_t* blocks_per_sm, uint32_t* cand_lanes,
                            uint32_t* cand_blocks_per_sm, double* us_per_step);

/* Fixes the windowed plan instead of tuning it: window length (2..1024,
 * clamped to the configuration's window), lanes per row (8, 16, 32) and
 * blocks per SM (0 = occupancy limit; larger values are clamped to it). The
 * plan outlives re-uploads. All three 0 hands the choice back to the tuner,
 * which runs at the next ns_step. For a host-side cache of tuned plans per
 * network-size bucket. NS_ERR_STATE while a learned macro-step is
 * attached. */
ns_status ns_set_window_plan(ns_handle* h, uint32_t window, uint32_t lanes, uint32_t blocks_per_sm);

/* Kernel launches issued by this handle since creation (own kernels only). */
ns_status ns_launch_count(ns_handle* h, uint64_t* launches);

/* Running totals since creation / state upload: out[0] steps, out[1]
 * spikes, out[2] output spikes, out[3] synaptic events. */
ns_status ns_counters(ns_handle* h, uint64_t out[4]);

/* The CUDA stream (cudaStream_t) every kernel of this handle is launched on,
 * so a caller can record its own CUDA events around ns_step. */
ns_status ns_get_stream(ns_handle* h, void** stream);

/* Runs n_steps eagerly and serially with CUDA events around every kernel;
 * adds the device time (ms) and launch count of the neuron, row-walk, LTD
 * (under schedule 5: the row-block flush), homeostasis and drive kernels to
 * kernel_ms[5] / launches[5]. The kernels are the ones the step graphs run
 * (the drive precomputed where graph chunks precompute it). Same numerics
 * as ns_step. */
ns_status ns_profile_steps(ns_handle* h, uint32_t n_steps, double* kernel_ms, uint64_t* launches);

/* --- single-network sharding (one process per GPU; no counterpart in the
 *     reference, which runs one network on one device) ------------------
 * A network's neurons are split over `world` ranks by 2048-neuron tiles:
 * rank r updates neurons [lo, hi) (ns_shard_range) and holds the synapses
 * whose target is one of them. Its CSR keeps every source row (row_ptr over
 * all n neurons) with global target indices, all inside [lo, hi); every
 * rank uploads the full neuron SoA. Each step the ranks all-gather the
 * step's spike bitmap (n/8 bytes in all); each rank then rebuilds the other
 * ranks' spike lists and source traces, walks every spiking row into its
 * own targets and runs LTD and homeostasis for its own targets. The union
 * of the ranks' rasters, owned states and weights equals the one-GPU run
 * bit for bit. Windowed stepping, batches, traced and profiled steps are
 * single-GPU only; the schedule is fixed (fused, 4 blocks/SM, unless
 * step_schedule names one). State outside [lo, hi) is not the rank's. */
ns_status ns_shard_range(uint64_t n, uint32_t rank, uint32_t world, uint64_t* lo, uint64_t* hi);
/* Before the uploads. */
ns_status ns_shard_configure(ns_handle* h, uint32_t rank, uint32_t world);
/* NCCL all-gather inside the step graphs: rank 0 makes the id, every rank
 * receives it (e.g. over the job's process group) and initialises; ns_step
 * then steps all ranks in lockstep. NCCL is loaded at run time. */
ns_status ns_shard_nccl_unique_id(char id_out[128]);
ns_status ns_shard_nccl_init(ns_handle* h, const char id[128]);
/* Without NCCL (ranks on one GPU or driven by one process): per step,
 * ns_shard_step_begin on every rank, ns_shard_copy_bitmap(dst, src) for
 * every ordered pair of ranks, then ns_shard_step_end on every rank. */
ns_status ns_shard_step_begin(ns_handle* h);
ns_status ns_shard_copy_bitmap(ns_handle* dst, ns_handle* src);
ns_status ns_shard_step_end(ns_handle* h);

/* --- allocation-free step (no counterpart in the reference) -------------
 * For callers that cannot allocate device memory where they step neurons:
 * one recorded into their own CUDA stream capture (cudaMalloc cannot be
 * captured), a latency-bound loop that cannot take the synchronisation an
 * allocation may cause, or a plugin confined to another framework's memory
 * pool. One Izhikevich step (izhikevich.rs:20-52, the same float arithmetic
 * as ns_step) of n neurons held in the caller's device arrays v, u (updated
 * in place), a, b, c, d and current (input current of this step, NULL = 0),
 * followed by ordered spike compaction: spikes_out (device, capacity n)
 * receives the ascending indices of the neurons that spiked and
 * *n_spikes_out (device) their number. Work is enqueued on `stream`
 * (a cudaStream_t; NULL = legacy default stream) and not waited for.
 * The compaction's scratch is a fixed device array of NS_NOALLOC_MAX_NEURONS
 * + 1024 words (4 MiB + 4 KiB) that every GPU which loads the library holds
 * until exit; n above NS_NOALLOC_MAX_NEURONS is rejected with
 * NS_ERR_INVALID_ARG. Nothing is allocated or freed. The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress with that
 * device current): make that first call before any stream capture. The
 * address is kept for the life of the process and does not survive
 * cudaDeviceReset: after a reset of the device, reload the library before
 * calling this entry point on that device again. All calls
 * on a device share the one scratch array, so calls whose kernels overlap on
 * the GPU (different streams without ordering between them) race; order
 * them on one stream. */
#define NS_NOALLOC_MAX_NEURONS 1048576u
ns_status ns_izhikevich_step_noalloc(uint64_t n, float* v, float* u, const float* a,
                                     const float* b, const float* c, const float* d,
                                     const float* current, float dt_ms, uint32_t* spikes_out,
                                     uint32_t* n_spikes_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NEURALSIM_H */
