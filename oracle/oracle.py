"""ORACLE — test infrastructure only.

ctypes wrapper of oracle/_build/liboracle.so, the CPU restatement of the
reference's SimulationEngine::step hot path (src/simulation/engine.rs:254-697
and the neuron / synapse / plasticity modules). Only tests/, the smoke check
and bench.py's CPU-baseline leg use it; the product never does.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


class OrConfig(C.Structure):
    _fields_ = [
        ("model", C.c_int32), ("input_mode", C.c_int32), ("hh_integrator", C.c_int32),
        ("weight_format", C.c_int32), ("dt", C.c_double), ("delay_steps", C.c_int32),
        ("pad0", C.c_int32), ("seed", C.c_uint64), ("current_decay", C.c_double),
        ("stdp", C.c_int32), ("pad1", C.c_int32), ("tau_plus", C.c_double),
        ("tau_minus", C.c_double), ("a_plus", C.c_double), ("a_minus", C.c_double),
        ("w_min", C.c_double), ("w_max", C.c_double), ("homeo", C.c_int32), ("pad2", C.c_int32),
        ("h_target", C.c_double), ("h_tau", C.c_double), ("contrib_tau", C.c_double),
        ("drive_kind", C.c_int32), ("kick_min", C.c_int32), ("kick_max", C.c_int32),
        ("pad3", C.c_int32), ("p", C.c_double), ("amp", C.c_double), ("sigma_exc", C.c_double),
        ("sigma_inh", C.c_double), ("kick_chance", C.c_double), ("kick_strength", C.c_double),
        ("rstdp", C.c_int32), ("cons", C.c_int32), ("rstdp_lr", C.c_double),
        ("rstdp_wmin", C.c_double), ("rstdp_wmax", C.c_double), ("elig_tau", C.c_double),
        ("reward_thr", C.c_uint64), ("reward_decay", C.c_double), ("reward_init", C.c_double),
        ("cons_tau", C.c_double), ("cons_target", C.c_double), ("cons_drift", C.c_double),
        ("track_rates", C.c_int32), ("pad4", C.c_int32),
    ]


class OrNet(C.Structure):
    _fields_ = [
        ("n", C.c_uint64), ("m", C.c_uint64), ("row_ptr", C.c_void_p), ("col", C.c_void_p),
        ("w", C.c_void_p), ("syn_type", C.c_void_p), ("plastic", C.c_void_p),
        ("params", C.c_void_p), ("ppn", C.c_int32), ("pad", C.c_int32),
        ("inhibitory", C.c_void_p), ("is_output", C.c_void_p), ("v0", C.c_void_p),
        ("u0", C.c_void_p), ("m0", C.c_void_p), ("h0", C.c_void_p), ("n0", C.c_void_p),
        ("eligible", C.c_void_p), ("stp", C.c_void_p), ("has_stp", C.c_void_p),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    L = C.CDLL(LIB)
    vp, u64 = C.c_void_p, C.c_uint64
    sig = {
        "or_philox4x32_10": (None, [vp, vp, vp]),
        "or_logf": (C.c_float, [C.c_float]),
        "or_expf": (C.c_float, [C.c_float]),
        "or_sincos2pi": (None, [C.c_float, vp, vp]),
        "or_drive_f32": (C.c_float, [C.POINTER(OrConfig), u64, vp, u64, u64, C.c_float]),
        "or_lif_step_f64": (C.c_int, [vp, vp, vp, C.c_double, C.c_double]),
        "or_izh_step_f64": (C.c_int, [vp, vp, vp, C.c_double, C.c_double]),
        "or_hh_step_f64": (C.c_int, [vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int]),
        "or_mg_block": (C.c_double, [C.c_int, C.c_double]),
        "or_dual_exp_conductance": (C.c_double, [C.c_int, C.c_double]),
        "or_trace_on_spike": (None, [vp, vp, C.c_double, C.c_double]),
        "or_trace_decay": (None, [vp, vp, C.c_double, C.c_double, C.c_double]),
        "or_eligibility_update": (None, [vp, C.c_double, C.c_double, C.c_double]),
        "or_eligibility_apply": (None, [vp, C.c_double, vp, C.c_double, C.c_double, C.c_double]),
        "or_stdp_weight_change": (C.c_double, [C.c_double] * 5),
        "or_consolidation_apply": (None, [vp, C.c_double, C.c_double, C.c_double, C.c_double]),
        "or_stp_step": (C.c_double, [vp, vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]),
        "or_finalize_csr": (None, [u64, u64, vp, vp, vp, vp]),
        "or_fast_create": (vp, [C.POINTER(OrConfig), C.POINTER(OrNet), C.c_int32]),
        "or_fast_step": (None, [vp, C.c_int32]),
        "or_fast_step_traced": (u64, [vp, vp, u64]),
        "or_fast_log_size": (u64, [vp]),
        "or_fast_log_steps": (u64, [vp]),
        "or_fast_log": (None, [vp, vp, vp]),
        "or_fast_state": (None, [vp] * 11),
        "or_fast_weights": (None, [vp, vp]),
        "or_fast_rates": (None, [vp, vp]),
        "or_fast_events": (u64, [vp]),
        "or_fast_lfp": (C.c_double, [vp]),
        "or_fast_add_input_current": (None, [vp, u64, vp, vp]),
        "or_lit_add_input_current": (None, [vp, u64, vp, vp]),
        "or_fast_eligibility": (None, [vp, vp]),
        "or_fast_reward": (None, [vp, vp]),
        "or_fast_apply_reward": (None, [vp, C.c_double]),
        "or_fast_destroy": (None, [vp]),
        "or_lit_create": (vp, [C.POINTER(OrConfig), C.POINTER(OrNet), C.c_int32]),
        "or_lit_step": (None, [vp, C.c_int32]),
        "or_lit_log_size": (u64, [vp]),
        "or_lit_log_steps": (u64, [vp]),
        "or_lit_log": (None, [vp, vp, vp]),
        "or_lit_state": (None, [vp] * 7),
        "or_lit_weights": (None, [vp, vp]),
        "or_lit_set_state": (None, [vp, vp, vp, vp, vp, vp, vp, C.c_double, u64]),
        "or_lit_rates": (None, [vp, vp]),
        "or_lit_events": (u64, [vp]),
        "or_lit_stats": (None, [vp, vp]),
        "or_lit_eligibility": (None, [vp, vp]),
        "or_lit_reward": (None, [vp, vp]),
        "or_lit_apply_reward": (None, [vp, C.c_double]),
        "or_lit_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def make_config(cfg, drive):
    """OrConfig from a neuralsim_b200 SimConfig + Drive (plain attribute access)."""
    c = OrConfig()
    c.model = cfg.model
    c.input_mode = cfg.input_mode
    c.hh_integrator = cfg.hh_integrator
    c.weight_format = cfg.weight_format
    c.dt = cfg.dt_ms
    c.delay_steps = cfg.delay_steps
    c.seed = cfg.seed
    c.current_decay = cfg.current_decay
    c.stdp = 1 if cfg.stdp_enabled else 0
    c.tau_plus, c.tau_minus = cfg.tau_plus, cfg.tau_minus
    c.a_plus, c.a_minus = cfg.a_plus, cfg.a_minus
    c.w_min, c.w_max = cfg.w_min, cfg.w_max
    c.homeo = 1 if cfg.homeostasis_enabled else 0
    c.h_target, c.h_tau = cfg.homeostatic_target_rate, cfg.homeostatic_tau
    c.contrib_tau = cfg.contribution_tau
    c.drive_kind = drive.kind
    c.kick_min, c.kick_max = drive.kick_min, drive.kick_max
    # drive parameters travel as float32 on the device; use the same values
    f = lambda x: float(np.float32(x))
    c.p, c.amp = f(drive.p), f(drive.amplitude)
    c.sigma_exc, c.sigma_inh = f(drive.sigma_exc), f(drive.sigma_inh)
    c.kick_chance, c.kick_strength = f(drive.kick_chance), f(drive.kick_strength)
    g = lambda name, dflt: getattr(cfg, name, dflt)
    c.rstdp = 1 if g("rstdp_enabled", False) else 0
    c.rstdp_lr, c.rstdp_wmin, c.rstdp_wmax = g("rstdp_lr", 0.1), g("rstdp_w_min", 0.0), g("rstdp_w_max", 10.0)
    c.elig_tau = g("eligibility_tau", 200.0)
    c.reward_thr, c.reward_decay = g("reward_threshold", 5), g("reward_decay", 0.95)
    c.reward_init = g("reward_signal", 0.0)
    c.cons = 1 if g("consolidation_enabled", False) else 0
    c.cons_tau, c.cons_target = g("consolidation_tau", 10000.0), g("consolidation_target", 0.5)
    c.cons_drift = g("consolidation_drift", 0.001)
    c.track_rates = 1 if g("track_rates", 0) else 0
    return c


class _Base:
    prefix = ""

    def __init__(self, net, cfg, drive):
        self.L = load()
        self.net = net
        self.cfg = make_config(cfg, drive)
        self.n, self.m = net.n, net.m
        nt = OrNet()
        nt.n, nt.m = net.n, net.m
        nt.row_ptr, nt.col, nt.w = _p(net.row_ptr), _p(net.col), _p(net.w)
        nt.syn_type, nt.plastic = _p(net.syn_type), _p(net.plastic)
        nt.params, nt.ppn = _p(net.params), net.params.shape[1]
        nt.inhibitory, nt.is_output = _p(net.inhibitory), _p(net.is_output)
        nt.v0, nt.u0 = _p(net.v0), _p(net.u0)
        nt.m0, nt.h0, nt.n0 = _p(net.m0), _p(net.h0), _p(net.n0)
        nt.eligible = _p(getattr(net, "eligible", None))
        nt.stp, nt.has_stp = _p(getattr(net, "stp", None)), _p(getattr(net, "has_stp", None))
        self._nt = nt

    def raster(self):
        f = getattr(self.L, self.prefix + "log_size")
        g = getattr(self.L, self.prefix + "log_steps")
        tot, steps = f(self.h), g(self.h)
        idx = np.zeros(max(tot, 1), np.uint32)
        off = np.zeros(steps + 1, np.uint64)
        getattr(self.L, self.prefix + "log")(self.h, _p(idx), _p(off))
        return idx[:tot], off

    def weights(self):
        w = np.zeros(max(self.m, 1), np.float64)
        getattr(self.L, self.prefix + "weights")(self.h, _p(w))
        return w[:self.m]

    def rates(self):
        r = np.zeros(self.n, np.float64)
        getattr(self.L, self.prefix + "rates")(self.h, _p(r))
        return r

    def events(self):
        return int(getattr(self.L, self.prefix + "events")(self.h))

    def stimulate(self, ids, amounts):
        """SimulationEngine::stimulate (engine.rs:156-161) for each pair."""
        i = np.ascontiguousarray(np.atleast_1d(ids), dtype=np.uint32)
        a = np.ascontiguousarray(np.broadcast_to(np.atleast_1d(amounts), i.shape), dtype=np.float64)
        getattr(self.L, self.prefix + "add_input_current")(self.h, i.size, _p(i), _p(a))

    def lfp(self):
        """lfp_signal (engine.rs:492) as the device sums it."""
        return float(self.L.or_fast_lfp(self.h))

    def eligibility(self):
        e = np.zeros(max(self.m, 1), np.float64)
        getattr(self.L, self.prefix + "eligibility")(self.h, _p(e))
        return e[:self.m]

    def reward(self):
        """(reward_signal now, sum of the reward after each step)."""
        o = np.zeros(2)
        getattr(self.L, self.prefix + "reward")(self.h, _p(o))
        return float(o[0]), float(o[1])

    def apply_reward(self, reward):
        getattr(self.L, self.prefix + "apply_reward")(self.h, float(reward))

    def close(self):
        if self.h:
            getattr(self.L, self.prefix + "destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FastOracle(_Base):
    """Per-neuron-trace reformulation; precision 32 mirrors the device bit for
    bit (int64 fixed-point sums), precision 64 is the FP64 reference."""
    prefix = "or_fast_"

    def __init__(self, net, cfg, drive, precision=32):
        super().__init__(net, cfg, drive)
        self.h = self.L.or_fast_create(C.byref(self.cfg), C.byref(self._nt), precision)

    def step(self, k=1):
        self.L.or_fast_step(self.h, k)

    def step_traced(self, cap):
        pos = np.zeros(max(cap, 1), np.uint64)
        ne = self.L.or_fast_step_traced(self.h, _p(pos), cap)
        return pos[:min(cap, ne)], int(ne)

    def state(self):
        n = self.n
        out = {k: np.zeros(n) for k in ("v", "u", "m", "h", "n", "I", "pre", "post")}
        refr = np.zeros(n, np.int32)
        last = np.zeros(n, np.int64)
        self.L.or_fast_state(self.h, _p(out["v"]), _p(out["u"]), _p(out["m"]), _p(out["h"]),
                             _p(out["n"]), _p(out["I"]), _p(refr), _p(out["pre"]),
                             _p(out["post"]), _p(last))
        out["refr"], out["last"] = refr, last
        return out


class LiteralOracle(_Base):
    """FP64, per-synapse state, the reference's loop structure."""
    prefix = "or_lit_"

    def __init__(self, net, cfg, drive, threads=1):
        super().__init__(net, cfg, drive)
        self.h = self.L.or_lit_create(C.byref(self.cfg), C.byref(self._nt), threads)

    def step(self, k=1):
        self.L.or_lit_step(self.h, k)

    def state(self):
        n = self.n
        out = {k: np.zeros(n) for k in ("v", "u", "m", "h", "n", "I")}
        self.L.or_lit_state(self.h, _p(out["v"]), _p(out["u"]), _p(out["m"]), _p(out["h"]),
                            _p(out["n"]), _p(out["I"]))
        return out

    def set_state(self, v, u, pre, post, last_spike_time, w, time, step):
        """Warm start for timing samples: neuron state, per-neuron traces and
        last spike times (ms), weights, clock (ms) and step count."""
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        arrs = [f(x) for x in (v, u, pre, post, last_spike_time, w)]
        self._keep = arrs
        self.L.or_lit_set_state(self.h, *[_p(a) for a in arrs], float(time), int(step))

    def stats(self):
        o = np.zeros(8)
        self.L.or_lit_stats(self.h, _p(o))
        return dict(zip(["total_spikes", "time", "mean_rate", "weight_mean", "weight_std", "lfp",
                         "events", "steps"], o.tolist()))


def split_raster(idx, off):
    return [idx[int(off[q]):int(off[q + 1])] for q in range(len(off) - 1)]
