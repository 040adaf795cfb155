"""Python host mirror of the reference crate's simulation API, backed by the
device through the C ABI.

`Network` carries what `neural_sim::network::Network` holds for the hot path
(src/network/mod.rs:36-48): the neuron SoA (src/neuron/mod.rs:126-163) and the
CSR synapse arrays. `SimulationEngine` mirrors `SimulationEngine`
(src/simulation/engine.rs:43-823): `step()` returns the spiking neurons of one
step like `StepResult` (engine.rs:35-41), `simulate_ms` is engine.rs:792-797,
`stats()` is engine.rs:799-801. Every call goes through libneuralsim.so.
"""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A

PARAMS_PER_NEURON = {A.MODEL_LIF: 6, A.MODEL_IZHIKEVICH: 4, A.MODEL_HH: 7}


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


@dataclass
class Network:
    """Neuron SoA + CSR-by-source synapses (synapse arrays in CSR order)."""
    model: int
    params: np.ndarray            # (n, ppn) float32
    row_ptr: np.ndarray           # (n+1,) uint64
    col: np.ndarray               # (m,) uint32
    w: np.ndarray                 # (m,) float32
    syn_type: np.ndarray = None   # (m,) uint8
    plastic: np.ndarray = None    # (m,) uint8
    v0: np.ndarray = None
    u0: np.ndarray = None
    m0: np.ndarray = None
    h0: np.ndarray = None
    n0: np.ndarray = None
    inhibitory: np.ndarray = None
    is_output: np.ndarray = None
    eligible: np.ndarray = None   # (m,) uint8: synapse carries an R-STDP eligibility trace
    stp: np.ndarray = None        # (m, 5) float64: u_se, tau_rec, tau_facil, u, r
    has_stp: np.ndarray = None    # (m,) uint8, None = every synapse (when stp is given)
    name: str = "NeuralSim Network"

    @property
    def n(self):
        return int(self.params.shape[0])

    @property
    def m(self):
        return int(self.col.shape[0])

    def __post_init__(self):
        self.params = np.ascontiguousarray(self.params, dtype=np.float32)
        self.row_ptr = np.ascontiguousarray(self.row_ptr, dtype=np.uint64)
        self.col = np.ascontiguousarray(self.col, dtype=np.uint32)
        self.w = np.ascontiguousarray(self.w, dtype=np.float32)
        if self.stp is not None:
            self.stp = np.ascontiguousarray(self.stp, dtype=np.float64).reshape(-1, 5)
        for name in ("syn_type", "plastic", "inhibitory", "is_output", "eligible", "has_stp"):
            a = getattr(self, name)
            if a is not None:
                setattr(self, name, np.ascontiguousarray(a, dtype=np.uint8))
        for name in ("v0", "u0", "m0", "h0", "n0"):
            a = getattr(self, name)
            if a is not None:
                setattr(self, name, np.ascontiguousarray(a, dtype=np.float32))


@dataclass
class SimConfig:
    """Mirrors SimulationConfig + PlasticityConfig (src/config/mod.rs:61-68,
    src/synapse/mod.rs:122-157) plus the semantics switches of this backend."""
    model: int = A.MODEL_LIF
    input_mode: int = A.INPUT_DIRECT_DECAY
    hh_integrator: int = A.HH_EULER_REF
    weight_format: int = A.WEIGHT_F32
    dt_ms: float = 0.5
    delay_steps: int = 1
    device: int = 0
    seed: int = 42
    current_decay: float = 0.92
    stdp_enabled: bool = True
    tau_plus: float = 20.0
    tau_minus: float = 20.0
    a_plus: float = 0.01
    a_minus: float = 0.012
    w_min: float = 0.0
    w_max: float = 10.0
    homeostasis_enabled: bool = True
    homeostatic_target_rate: float = 5.0
    homeostatic_tau: float = 5000.0
    contribution_tau: float = 1000.0
    spike_log_capacity: int = 0
    spike_log_steps: int = 0
    graph_chunk: int = 1000
    step_schedule: int = 0      # 0 autotune, 1 fused, 2 split, 3 fused (4 blocks/SM)
    window_steps: int = 0       # 0 auto (= delay), 1 off, W > 1 explicit
    # R-STDP (RStdpRule::default, plasticity.rs:177-189; engine.rs:113-116, :521)
    rstdp_enabled: bool = False
    rstdp_lr: float = 0.1
    rstdp_w_min: float = 0.0
    rstdp_w_max: float = 10.0
    eligibility_tau: float = 200.0
    reward_threshold: int = 5
    reward_decay: float = 0.95
    reward_signal: float = 0.0
    # consolidation (ConsolidationRule::default, plasticity.rs:276-284)
    consolidation_enabled: bool = False
    consolidation_tau: float = 10000.0
    consolidation_target: float = 0.5
    consolidation_drift: float = 0.001
    track_rates: int = 0

    def to_c(self):
        c = A.NsConfig()
        for name, _ in A.NsConfig._fields_:
            setattr(c, name, type(getattr(c, name))(getattr(self, name)))
        return c


@dataclass
class Drive:
    kind: int = A.DRIVE_NONE
    p: float = 0.0
    amplitude: float = 0.0
    sigma_exc: float = 0.0
    sigma_inh: float = 0.0
    kick_chance: float = 0.0
    kick_strength: float = 0.0
    kick_min: int = 0
    kick_max: int = 0

    def to_c(self):
        d = A.NsDrive()
        for name, _ in A.NsDrive._fields_:
            setattr(d, name, getattr(self, name))
        return d

    @staticmethod
    def reference_default():
        """The reference engine's drive (engine.rs:100-103, :273-287)."""
        return Drive(A.DRIVE_REF_UNIFORM, p=0.3, amplitude=8.0, kick_chance=0.01,
                     kick_strength=20.0, kick_min=5, kick_max=30)


@dataclass
class StepResult:
    """StepResult (engine.rs:35-41)."""
    spike_count: int
    output_spike_count: int
    spiking_neurons: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))
    output_spiking_neurons: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint32))


class SimulationEngine:
    """Device-backed engine. One instance owns one ns_handle (not thread-safe,
    like the Mutex-guarded reference engine, src/simulation/scheduler.rs:23)."""

    def __init__(self, network: Network, config: SimConfig = None, drive: Drive = None,
                 shard=None, plan_cache=None):
        """shard: (rank, world) for one rank of a sharded network (see
        neuralsim_b200.shard.partition_network); None for a whole network.
        plan_cache: a neuralsim_b200.tune.PlanCache (or its file's path)
        holding windowed plans per network-size bucket (use_plan_cache)."""
        self.lib = A.load()
        self.config = config or SimConfig(model=network.model)
        if self.config.model != network.model:
            raise ValueError("config.model differs from network.model")
        self.network = network
        self._h = C.c_void_p()
        cfg = self.config.to_c()
        st = self.lib.ns_create(C.byref(cfg), C.byref(self._h))
        if st != A.NS_OK:
            raise A.NsError(st, (self.lib.ns_last_error(None) or b"").decode())
        try:
            if shard is not None:
                self._check(self.lib.ns_shard_configure(self._h, int(shard[0]), int(shard[1])))
            self._upload(network)
            self.set_drive(drive or Drive())
        except Exception:
            self.close()
            raise
        self._stats_total = {"spikes": 0, "output_spikes": 0, "events": 0}
        self._plan_cache, self._plan_key, self._plan_done = None, None, True
        if plan_cache is not None:
            self.use_plan_cache(plan_cache)

    # -- uploads (init_gpu, engine.rs:181-252) --
    def _upload(self, net: Network):
        soa = A.NsNeuronSoa()
        soa.n = net.n
        soa.params = _ptr(net.params)
        soa.params_per_neuron = PARAMS_PER_NEURON[net.model]
        soa.v = _ptr(net.v0)
        soa.u = _ptr(net.u0)
        soa.hh_m = _ptr(net.m0)
        soa.hh_h = _ptr(net.h0)
        soa.hh_n = _ptr(net.n0)
        soa.inhibitory = _ptr(net.inhibitory)
        soa.is_output = _ptr(net.is_output)
        self._check(self.lib.ns_upload_neurons(self._h, C.byref(soa)))
        self._check(self.lib.ns_upload_csr(
            self._h, net.n, net.m, _ptr(net.row_ptr), _ptr(net.col), _ptr(net.w),
            _ptr(net.syn_type), _ptr(net.plastic)))
        for name, want in (("eligible", (net.m,)), ("has_stp", (net.m,)), ("stp", (net.m, 5))):
            a = getattr(net, name)
            if a is not None and a.shape != want:
                raise ValueError(f"Network.{name} must have shape {want}")
        if self.config.rstdp_enabled and net.eligible is not None:
            self._check(self.lib.ns_upload_eligibility(self._h, _ptr(net.eligible), None))
        if net.stp is not None:
            self._check(self.lib.ns_upload_stp(self._h, _ptr(net.has_stp), _ptr(net.stp)))

    def _check(self, st):
        A.check(st, self._h)

    def set_drive(self, drive: Drive):
        self.drive = drive
        d = drive.to_c()
        self._check(self.lib.ns_set_drive(self._h, C.byref(d)))

    # -- stepping --
    def run(self, n_steps: int) -> A.NsStepStats:
        out = A.NsStepStats()
        self._check(self.lib.ns_step(self._h, int(n_steps), C.byref(out)))
        if not self._plan_done:
            self._record_plan()
        self._stats_total["spikes"] += out.spikes
        self._stats_total["output_spikes"] += out.output_spikes
        self._stats_total["events"] += out.events
        self._last_out = out
        return out

    def step(self) -> StepResult:
        """One step; returns the ascending spiking neuron list when the spike
        log is enabled (spike_log_capacity > 0), else only the counts."""
        k = self.current_step()
        out = self.run(1)
        spikes = np.zeros(0, np.uint32)
        outs = spikes
        if self.config.spike_log_capacity > 0:
            spikes = self.read_spikes(k, 1)[0]
            if self.network.is_output is not None:
                outs = spikes[np.asarray(self.network.is_output)[spikes] != 0]
        return StepResult(int(out.spikes), int(out.output_spikes), spikes, outs)

    def simulate_ms(self, duration_ms: float):
        steps = int(duration_ms / self.config.dt_ms)
        if steps:
            self.run(steps)

    def current_step(self) -> int:
        s = C.c_uint64()
        self._check(self.lib.ns_get_step(self._h, C.byref(s)))
        return int(s.value)

    def stats(self) -> dict:
        """SimulationStats (engine.rs:22-33, filled at :617-670) from the
        totals of this engine's runs, plus the step and event counts. The
        mean firing rate needs the rate estimate (homeostasis or
        track_rates); the weight moments are computed on demand."""
        out = dict(self._stats_total)
        out["steps"] = self.current_step()
        out["sim_time_ms"] = out["steps"] * self.config.dt_ms
        last = getattr(self, "_last_out", None)
        out["total_spikes"] = out["spikes"]
        out["active_neurons"] = int(last.max_step_spikes) if last is not None else 0
        out["weight_updates"] = int(last.last_step_spikes) if last is not None else 0
        out["synchrony_index"] = out["weight_updates"] / self.network.n
        out["mean_firing_rate"] = self.mean_firing_rate()
        out["weight_mean"], out["weight_std"] = self.weight_stats()
        out["seed"] = self.config.seed
        return out

    def weight_stats(self):
        mu, sd = C.c_double(), C.c_double()
        self._check(self.lib.ns_weight_stats(self._h, C.byref(mu), C.byref(sd)))
        return mu.value, sd.value

    # -- spike log --
    def log_range(self):
        a, b = C.c_uint64(), C.c_uint64()
        self._check(self.lib.ns_spike_log_range(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    def read_spikes(self, first_step: int, n_steps: int):
        """List of ascending uint32 arrays, one per step."""
        idx, off = self.read_raster(first_step, n_steps)
        return [idx[int(off[q]):int(off[q + 1])] for q in range(n_steps)]

    def read_raster(self, first_step: int, n_steps: int, out=None):
        """(idx, offsets) flat form of the spike log. out: an optional uint32
        array (e.g. in pinned host memory) that receives the indices when it
        is large enough; the returned idx is then a view of it."""
        off = np.zeros(n_steps + 1, np.uint64)
        nw = C.c_uint64()
        st = self.lib.ns_read_spikes(self._h, first_step, n_steps, None, _ptr(off), 0, C.byref(nw))
        total = int(nw.value)
        if st != A.NS_OK and total == 0:
            self._check(st)
        if out is not None and out.dtype == np.uint32 and out.flags.c_contiguous and out.size >= max(total, 1):
            idx = out
        else:
            idx = np.empty(max(total, 1), np.uint32)
        self._check(self.lib.ns_read_spikes(self._h, first_step, n_steps, _ptr(idx), _ptr(off),
                                            total, C.byref(nw)))
        return idx[:total], off

    def clear_spike_log(self):
        self._check(self.lib.ns_clear_spike_log(self._h))

    # -- state --
    def download_state(self, with_weights=True, fields=None):
        """The neuron state (and the weights): every field of ns_neuron_soa,
        or only those named in `fields` (e.g. ("v",))."""
        n = self.network.n
        ppn = PARAMS_PER_NEURON[self.config.model]
        cond = self.config.input_mode in (A.INPUT_CONDUCTANCE_REF, A.INPUT_CONDUCTANCE_FRESH)
        ntypes = 4 if cond else 1
        st = {
            "v": np.zeros(n, np.float32), "u": np.zeros(n, np.float32),
            "refractory": np.zeros(n, np.int32), "current": np.zeros(n, np.float32),
            "hh_m": np.zeros(n, np.float32), "hh_h": np.zeros(n, np.float32),
            "hh_n": np.zeros(n, np.float32), "params": np.zeros((n, ppn), np.float32),
            "inhibitory": np.zeros(n, np.uint8), "is_output": np.zeros(n, np.uint8),
            "pre_trace": np.zeros(n, np.float32), "post_trace": np.zeros(n, np.float32),
            "last_spike_step": np.zeros(n, np.int64),
            "pending_input": np.zeros(ntypes * self.config.delay_steps * n, np.int64),
            "conductance": np.zeros(4 * n, np.float32), "firing_rate": np.zeros(n, np.float64),
        }
        if fields is not None:
            unknown = set(fields) - set(st)
            if unknown:
                raise ValueError(f"unknown state fields {sorted(unknown)}")
            st = {k: v for k, v in st.items() if k in fields}
        soa = A.NsNeuronSoa()
        for name, arr in st.items():
            setattr(soa, name, _ptr(arr))
        soa.params_per_neuron = ppn
        w = np.zeros(max(self.network.m, 1), np.float32) if with_weights else None
        self._check(self.lib.ns_download_state(self._h, C.byref(soa), _ptr(w)))
        if with_weights:
            st["w"] = w[:self.network.m]
        return st

    def upload_state(self, st: dict, step: int):
        soa = A.NsNeuronSoa()
        soa.n = self.network.n
        for name in ("v", "u", "refractory", "current", "hh_m", "hh_h", "hh_n", "pre_trace",
                     "post_trace", "last_spike_step", "pending_input", "conductance",
                     "firing_rate"):
            if name in st:
                setattr(soa, name, _ptr(st[name]))
        soa.params_per_neuron = PARAMS_PER_NEURON[self.config.model]
        self._check(self.lib.ns_upload_state(self._h, C.byref(soa), _ptr(st.get("w")), int(step)))

    def stimulate(self, neuron_ids, currents):
        """Adds currents to the input current of neurons before the next
        step (SimulationEngine::stimulate, engine.rs:156-161); scalars or
        equal-length sequences."""
        ids = np.ascontiguousarray(np.atleast_1d(neuron_ids), dtype=np.uint32)
        amt = np.ascontiguousarray(np.broadcast_to(np.atleast_1d(currents), ids.shape), dtype=np.float64)
        self._check(self.lib.ns_add_input_current(self._h, ids.size, _ptr(ids), _ptr(amt)))

    def lfp(self) -> float:
        """lfp_signal (engine.rs:492) of the reference conductance mode."""
        x = C.c_double()
        self._check(self.lib.ns_get_lfp(self._h, C.byref(x)))
        return x.value

    # -- R-STDP reward and eligibility (engine.rs:151-175, :546-563, :626-631) --
    def eligibility(self):
        e = np.zeros(max(self.network.m, 1), np.float32)
        self._check(self.lib.ns_download_eligibility(self._h, _ptr(e)))
        return e[:self.network.m]

    def upload_eligibility(self, eligible=None, values=None):
        el = None if eligible is None else np.ascontiguousarray(eligible, np.uint8)
        va = None if values is None else np.ascontiguousarray(values, np.float32)
        for a in (el, va):
            if a is not None and a.size != self.network.m:
                raise ValueError("eligibility arrays need one entry per synapse (m)")
        self._check(self.lib.ns_upload_eligibility(self._h, _ptr(el), _ptr(va)))

    def contributions(self):
        """Per-synapse contribution averages of homeostatic scaling (CSR
        order; zeros without homeostasis)."""
        c = np.zeros(max(self.network.m, 1), np.float32)
        self._check(self.lib.ns_download_contributions(self._h, _ptr(c)))
        return c[:self.network.m]

    def upload_contributions(self, values):
        va = np.ascontiguousarray(values, np.float32)
        if va.size != self.network.m:
            raise ValueError("contributions need one entry per synapse (m)")
        self._check(self.lib.ns_upload_contributions(self._h, _ptr(va)))

    def checkpoint(self):
        """Everything a bit-exact resume needs: the device state and weights
        (download_state), the step index, eligibility traces (R-STDP), the
        contribution averages (homeostasis) and the reward."""
        st = self.download_state()
        st["step"] = self.current_step()
        if self.config.rstdp_enabled:
            st["eligibility"] = self.eligibility()
            st["reward"] = self.reward_signal
        if self.config.homeostasis_enabled:
            st["contributions"] = self.contributions()
        return st

    def restore(self, st: dict):
        """Loads a checkpoint() (or a state read from a saved network):
        state and weights at its step, then eligibility, contributions and
        reward when present."""
        self.upload_state(st, int(st.get("step", 0)))
        if st.get("eligibility") is not None and self.config.rstdp_enabled:
            self.upload_eligibility(st.get("eligible"), st["eligibility"])
        if st.get("contributions") is not None and self.config.homeostasis_enabled:
            self.upload_contributions(st["contributions"])
        if st.get("reward") is not None and self.config.rstdp_enabled:
            self.set_reward(float(st["reward"]))

    def apply_reward(self, reward: float):
        self._check(self.lib.ns_apply_reward(self._h, float(reward)))

    @property
    def reward_signal(self) -> float:
        return self.reward()[0]

    def reward(self):
        """(reward_signal now, sum of the reward after each step)."""
        r, s = C.c_double(), C.c_double()
        self._check(self.lib.ns_get_reward(self._h, C.byref(r), C.byref(s)))
        return r.value, s.value

    def set_reward(self, reward: float):
        self._check(self.lib.ns_set_reward(self._h, float(reward)))

    def rates(self):
        r = np.zeros(self.network.n, np.float64)
        self._check(self.lib.ns_download_rates(self._h, _ptr(r)))
        return r

    def firing_rate(self, neuron: int) -> float:
        """SimulationEngine::firing_rate (engine.rs:809-815): the neuron's
        rate estimate (kept with homeostasis or track_rates), 0 out of range."""
        return float(self.rates()[neuron]) if 0 <= neuron < self.network.n else 0.0

    def mean_firing_rate(self) -> float:
        """SimulationEngine::mean_firing_rate (engine.rs:818-826)."""
        r = self.rates()
        return float(r.sum() / r.size) if r.size else 0.0

    def step_traced(self, cap: int):
        pos = np.zeros(max(cap, 1), np.uint64)
        ne = C.c_uint64()
        self._check(self.lib.ns_step_traced(self._h, _ptr(pos), cap, C.byref(ne)))
        return pos[:min(cap, int(ne.value))], int(ne.value)

    def counters(self):
        """(steps, spikes, output_spikes, events) running totals on the device."""
        c = (C.c_uint64 * 4)()
        self._check(self.lib.ns_counters(self._h, c))
        return tuple(int(x) for x in c)

    def stream(self):
        """cudaStream_t of this handle (as an int)."""
        p = C.c_void_p()
        self._check(self.lib.ns_get_stream(self._h, C.byref(p)))
        return int(p.value or 0)

    def profile_steps(self, n_steps: int):
        """Per-kernel device time over n_steps eager serial steps:
        {"neuron": (ms_total, launches), "rows": ..., "ltd": ..., "homeostasis": ...,
        "drive": ...} (ltd: the row-block flush under the deferred-LTD schedule)"""
        ms = (C.c_double * 5)()
        ln = (C.c_uint64 * 5)()
        self._check(self.lib.ns_profile_steps(self._h, int(n_steps), ms, ln))
        names = ("neuron", "rows", "ltd", "homeostasis", "drive")
        return {names[q]: (ms[q], int(ln[q])) for q in range(5) if ln[q]}

    def schedule(self):
        """(schedule in use, {schedule: measured us/step}) from the autotuner."""
        sc = C.c_uint32()
        us = (C.c_double * 5)()
        self._check(self.lib.ns_get_schedule(self._h, C.byref(sc), us))
        # schedules 1-4 always; 5 (deferred LTD) where it applies and was timed
        return int(sc.value), {q + 1: us[q] for q in range(5) if q < 4 or us[q] > 0}

    def window(self):
        """(window length in use, {candidate W: us per step} timed by the
        window tuner)."""
        w = C.c_uint32()
        cand = np.zeros(4, np.uint32)
        us = np.zeros(4, np.float64)
        self._check(self.lib.ns_get_window(self._h, C.byref(w), _ptr(cand), _ptr(us)))
        return int(w.value), {int(c): float(t) for c, t in zip(cand, us) if c}

    def walk_shape(self):
        """(lanes per row, blocks per SM) of the window row walk in use, and
        {(lanes, blocks per SM or 0 = occupancy limit): us per step} timed by
        the window tuner."""
        lanes, bps = C.c_uint32(), C.c_uint32()
        cl = np.zeros(4, np.uint32)
        cb = np.zeros(4, np.uint32)
        us = np.zeros(4, np.float64)
        self._check(self.lib.ns_get_walk_shape(self._h, C.byref(lanes), C.byref(bps), _ptr(cl),
                                               _ptr(cb), _ptr(us)))
        return (int(lanes.value), int(bps.value)), {(int(a), int(b)): float(t)
                                                     for a, b, t in zip(cl, cb, us) if a}

    def window_plan(self):
        """The windowed plan in use: {"window", "lanes", "blocks_per_sm"}
        (None when stepping is not windowed)."""
        w, _ = self.window()
        if not w:
            return None
        (lanes, bps), _ = self.walk_shape()
        return {"window": w, "lanes": lanes, "blocks_per_sm": bps}

    def use_plan_cache(self, cache):
        """Windowed plans per network-size bucket (neuralsim_b200.tune): a
        cached plan for this network's bucket is fixed at once (no tuning);
        otherwise the plan the window tuner picks at the next step is stored
        in the cache. Returns the cached plan or None."""
        from . import tune
        if not isinstance(cache, tune.PlanCache):
            cache = tune.PlanCache(cache)
        c = self.config
        self._plan_cache = cache
        self._plan_key = tune.bucket_key(c.model, c.input_mode, c.weight_format, c.delay_steps,
                                         self.network.n, self.network.m)
        plan = cache.get(self._plan_key)
        if plan is not None:
            self.set_window_plan(plan["window"], plan["lanes"], plan["blocks_per_sm"])
        self._plan_done = plan is not None
        return plan

    def _record_plan(self):
        w, tried = self.window()
        if not w:
            self._plan_done = True      # not windowed: nothing to cache
            return
        if not tried:
            return                      # the tuner has not run yet
        shape, shape_us = self.walk_shape()
        plan = self.window_plan()
        us = min(shape_us.values()) if shape_us else min(tried.values())
        self._plan_cache.put(self._plan_key, plan, us)
        self._plan_done = True

    def set_window_plan(self, window, lanes, blocks_per_sm):
        """Fixes the windowed plan (no tuning); (0, 0, 0) hands it back to
        the window tuner."""
        self._check(self.lib.ns_set_window_plan(self._h, int(window), int(lanes), int(blocks_per_sm)))

    def network_rates(self, first_step, n_steps):
        """Mean firing rate (Hz) of every network of the handle after the
        logged steps, as the reference's per-neuron rate estimate averaged
        over a network reports it (src/simulation/engine.rs:637-645)."""
        n = len(getattr(self, "networks", [None]))
        out = np.zeros(n, np.float64)
        self._check(self.lib.ns_network_rates(self._h, int(first_step), int(n_steps), _ptr(out)))
        return out

    # -- learned HH macro-step (include/neuralsim_surrogate.h) --
    def attach_surrogate(self, sur, v_lo=-85.0, v_hi=-58.0, residual_mv=0.5):
        """Advance in-envelope neurons with the trained surrogate `sur`
        (None detaches); the handle keeps its own copy of the weights. The
        default v_hi is surrogate.MACRO_V_HI: the macro-step stops short of
        threshold, where the plain steps keep spike times accurate."""
        self._check(self.lib.ns_set_surrogate(self._h, sur.handle if sur is not None else None,
                                              float(v_lo), float(v_hi), float(residual_mv)))

    def macro_step_mode(self, mode):
        """0: the MLP; 1: one Rush-Larsen step of 0.1 ms (comparison)."""
        self._check(self.lib.ns_set_macro_step_mode(self._h, int(mode)))

    def surrogate_counts(self):
        """(neuron macro-steps by the MLP, by the Rush-Larsen fallback)."""
        a, b = C.c_uint64(), C.c_uint64()
        self._check(self.lib.ns_surrogate_counts(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    def launch_count(self):
        c = C.c_uint64()
        self._check(self.lib.ns_launch_count(self._h, C.byref(c)))
        return int(c.value)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self.lib.ns_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_count():
    lib = A.load()
    c = C.c_int()
    lib.ns_device_count(C.byref(c))
    return c.value
