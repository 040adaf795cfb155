"""The reference's on-disk formats: the serde JSON of `Network`
(src/network/mod.rs:36-48) that save_network_json / load_network_json write
and read (src/io/save.rs:5-17, src/io/load.rs:6-17), and the checkpoint
pair `<name>.json` + `<name>_meta.json` of CheckpointManager
(src/io/checkpoint.rs:11-100).

Reading: network_from_dict gives a `Network` for this library (the neuron SoA
with one parameter row per neuron from its `model_params` variant, and the
synapse records in CSR order); state_from_dict gives the dynamic state of a
network saved mid-run (neuron state, per-neuron STDP traces and last spike
steps from the records' traces, weights, eligibility, STP, contribution
averages and the step from `time`), ready for SimulationEngine.restore.

Writing: network_to_dict writes every field of the format, the dynamic ones
from a checkpoint of a running engine when given, so the Rust application
can load the result. It adds one object, `device_state`, with the values an
exact resume on this library needs and the format cannot hold (the input
propagated but not yet delivered, the device's form of the input current,
the per-target conductances, the firing-rate estimates, the traces of
neurons without plastic synapses, the step index); serde skips fields it
does not know, so the Rust application reads the file unchanged.

CSR order. Network::finalize buckets the synapse records by source into
adjacency_indices (mod.rs:79-106), but the engine's propagation loop reads
`net.synapses[idx]` at CSR position idx (engine.rs:417-428): the record in
insertion order. For records already sorted by source (what finalize
produces for networks built source by source, and what this module writes)
the two agree. For unsorted records the Rust application delivers, in its
current modes, the weight of record idx to the adjacency target at position
idx. csr_order="records" (the default) permutes the records into CSR order,
each synapse keeping its own endpoints and weight (what the STDP loop, the
conductance mode and the rest of the engine use per record);
csr_order="positions" reproduces the Rust application's current-mode
delivery instead (the record at position idx supplies weight, type and STP),
for networks without plastic synapses.
"""
import json
import os
import time as _time

import numpy as np

from . import _abi as A
from .engine import Network

_MODEL_OF = {"Lif": A.MODEL_LIF, "Izhikevich": A.MODEL_IZHIKEVICH, "HodgkinHuxley": A.MODEL_HH}
_FIELDS = {
    A.MODEL_LIF: ("resting", "threshold", "reset", "tau_m", "refractory_period", "input_resistance"),
    A.MODEL_IZHIKEVICH: ("a", "b", "c", "d"),
    A.MODEL_HH: ("g_na", "g_k", "g_l", "e_na", "e_k", "e_l", "c_m"),
}
_SYN_TYPES = {"AMPA": A.SYN_AMPA, "GABA": A.SYN_GABA, "GabaB": A.SYN_GABA_B, "NMDA": A.SYN_NMDA}
_SYN_NAMES = {v: k for k, v in _SYN_TYPES.items()}
_NEVER = -1e9   # last spike time of a neuron or trace that never spiked (mod.rs:143, plasticity.rs:137)


def _csr_permutation(d, csr_order):
    """(order, row_ptr, col): record index at each CSR position, the row
    pointers and targets of Network::finalize's bucketing by source."""
    n = len(d["neurons"]["membrane_potential"])
    syn = d["synapses"]
    src = np.array([s["source"] for s in syn], np.int64)
    tgt = np.array([s["target"] for s in syn], np.int64)
    if len(syn) and (src.max() >= n or tgt.max() >= n or src.min() < 0 or tgt.min() < 0):
        raise ValueError("synapse endpoint out of range")
    by_source = np.argsort(src, kind="stable")
    counts = np.bincount(src, minlength=n)
    row_ptr = np.zeros(n + 1, np.uint64)
    row_ptr[1:] = np.cumsum(counts)
    col = tgt[by_source].astype(np.uint32)
    if "adjacency_ptr" in d and len(d["adjacency_ptr"]) == n + 1:
        # a finalized network's adjacency is exactly this bucketing
        if not (np.array_equal(np.asarray(d["adjacency_ptr"], np.uint64), row_ptr) and
                np.array_equal(np.asarray(d["adjacency_indices"], np.uint32), col)):
            raise ValueError("adjacency does not match the synapse records (not finalized?)")
    if csr_order == "records":
        order = by_source
    elif csr_order == "positions":
        order = np.arange(len(syn))
    else:
        raise ValueError("csr_order is 'records' or 'positions'")
    return order, row_ptr, col


def _plastic(s):
    # STDP acts on records with plasticity enabled and a trace (engine.rs:500-502)
    return bool(s["plasticity_enabled"]) and s.get("stdp_trace") is not None


def network_from_dict(d, csr_order="records"):
    """Network from the parsed JSON of a reference `Network`. One neuron
    model per network (the step kernels run one model per handle)."""
    nr = d["neurons"]
    n = len(nr["membrane_potential"])
    variants = [next(iter(p)) for p in nr["model_params"]]
    kinds = set(variants)
    if len(kinds) != 1:
        raise ValueError(f"one neuron model per network, found {sorted(kinds)}")
    model = _MODEL_OF[variants[0]]
    fields = _FIELDS[model]
    params = np.array([[p[variants[0]][f] for f in fields] for p in nr["model_params"]], np.float32)
    syn = d["synapses"]
    order, row_ptr, col = _csr_permutation(d, csr_order)
    if csr_order == "positions" and any(_plastic(s) for s in syn):
        raise ValueError("csr_order='positions' cannot carry plastic synapses: the Rust "
                         "application's STDP loop updates records, not CSR positions")
    w = np.array([syn[i]["weight"] for i in order], np.float32)
    ty = np.array([_SYN_TYPES[syn[i]["synapse_type"]] for i in order], np.uint8)
    pl = np.array([1 if _plastic(syn[i]) else 0 for i in order], np.uint8)
    f32 = lambda key: np.asarray(nr[key], np.float32)
    net = Network(model, params, row_ptr, col, w, syn_type=ty, plastic=pl,
                  v0=f32("membrane_potential"), u0=f32("recovery_variable"),
                  m0=f32("hh_m"), h0=f32("hh_h"), n0=f32("hh_n"),
                  inhibitory=np.array([t == "Inhibitory" for t in nr["neuron_type"]], np.uint8),
                  is_output=np.asarray(nr.get("is_output", [False] * n), np.uint8),
                  name=d.get("name", "NeuralSim Network"))
    elig = [syn[i].get("eligibility") is not None for i in order]
    if any(elig):
        net.eligible = np.array(elig, np.uint8)
    stp = [syn[i].get("stp") for i in order]
    if any(x is not None for x in stp):
        net.has_stp = np.array([x is not None for x in stp], np.uint8)
        net.stp = np.array([[x["u_se"], x["tau_rec"], x["tau_facil"], x["u"], x["r"]]
                            if x is not None else [0.5, 800.0, 1000.0, 0.5, 1.0] for x in stp])
    net.__post_init__()
    return net


def load_network_json(path, csr_order="records"):
    with open(path) as f:
        return network_from_dict(json.load(f), csr_order)


def _step_of(t, dt):
    return int(round(t / dt))


def state_from_dict(d, net, cfg, csr_order="records"):
    """Dynamic state of a saved network for SimulationEngine.restore: neuron
    state (NeuronArray, src/neuron/mod.rs:127-143), per-neuron STDP traces and
    last spike steps (from the records' StdpTrace, plasticity.rs:121-160, and
    NeuronArray.last_spike_time), weights, eligibility values, contribution
    averages (SynapseState, src/synapse/mod.rs:58-79) and the step of
    Network.time. With this library's `device_state` object the resume is
    exact; without it the input current is converted from the reference's
    form (the DIRECT_DECAY current within one float rounding)."""
    nr = d["neurons"]
    n = len(nr["membrane_potential"])
    dt = cfg.dt_ms
    syn = d["synapses"]
    order, _, _ = _csr_permutation(d, csr_order)
    f32 = lambda x: np.asarray(x, np.float32)
    st = {"v": f32(nr["membrane_potential"]), "u": f32(nr["recovery_variable"]),
          "refractory": np.asarray(nr["refractory_counter"], np.int32),
          "hh_m": f32(nr["hh_m"]), "hh_h": f32(nr["hh_h"]), "hh_n": f32(nr["hh_n"]),
          "w": np.array([syn[i]["weight"] for i in order], np.float32)}
    step = _step_of(float(d.get("time", 0.0)), dt)
    # last spike steps: the engine stamps sim_time before its increment
    # (engine.rs:368, :682-697), so a spike at step k reads k * dt
    lst = np.asarray(nr["last_spike_time"], np.float64)
    st["last_spike_step"] = np.where(lst > _NEVER / 2, np.rint(lst / dt), -1).astype(np.int64)
    # per-neuron traces: every plastic record from j carries j's pre trace,
    # every one onto i carries i's post trace (all start at 0 and take the
    # same updates); records that disagree cannot be represented
    pre = np.zeros(n, np.float64)
    post = np.zeros(n, np.float64)
    seen_pre = np.zeros(n, bool)
    seen_post = np.zeros(n, bool)
    for s in syn:
        tr = s.get("stdp_trace")
        if tr is None or not s["plasticity_enabled"]:
            continue
        for arr, seen, who, key in ((pre, seen_pre, s["source"], "pre_trace"),
                                    (post, seen_post, s["target"], "post_trace")):
            if seen[who] and arr[who] != tr[key]:
                raise ValueError(f"synapse traces of neuron {who} differ ({key}); per-neuron "
                                 "traces cannot represent them")
            arr[who] = tr[key]
            seen[who] = True
    st["pre_trace"] = pre.astype(np.float32)
    st["post_trace"] = post.astype(np.float32)
    el = [syn[i].get("eligibility") for i in order]
    if any(x is not None for x in el):
        st["eligible"] = np.array([x is not None for x in el], np.uint8)
        st["eligibility"] = np.array([x["value"] if x is not None else 0.0 for x in el], np.float32)
    if cfg.homeostasis_enabled:
        st["contributions"] = np.array([syn[i].get("contribution_avg", 0.0) for i in order], np.float32)
    cur = f32(nr["input_current"])
    ds = d.get("device_state")
    if ds is not None:
        step = int(ds["step"])
        st["current"] = f32(ds["current"])
        st["pending_input"] = np.asarray(ds["pending_input"], np.int64)
        st["conductance"] = f32(ds["conductance"])
        st["firing_rate"] = np.asarray(ds["firing_rate"], np.float64)
        # every neuron's traces (the records hold those of neurons with
        # plastic synapses only)
        st["pre_trace"] = f32(ds["pre_trace"])
        st["post_trace"] = f32(ds["post_trace"])
        if "reward" in ds:
            st["reward"] = float(ds["reward"])
    else:
        if cfg.input_mode == A.INPUT_DIRECT_DECAY and step > 0:
            # the device applies the decay at the next update: I_ref / decay
            cur = (cur / np.float32(cfg.current_decay)).astype(np.float32)
        st["current"] = cur
    st["step"] = step
    return st


def _spike_time(k, dt, after):
    # the spike stamp of step k: before the clock's increment (NeuronArray),
    # after it (StdpTrace, engine.rs:498)
    return float((k + 1) * dt) if after else float(k * dt)


def _reference_current(st, cfg, step):
    """The reference's input_current after the last step from the device's
    form: in DIRECT_DECAY the delivered input and the decay the device applies
    at the next update (float, the device's own operations)."""
    cur = np.asarray(st["current"], np.float32)
    if cfg.input_mode != A.INPUT_DIRECT_DECAY or step == 0:
        return cur
    n = len(cur)
    slot = step % cfg.delay_steps   # the slot the next update reads
    pend = np.asarray(st["pending_input"], np.int64)[slot * n:(slot + 1) * n]
    delivered = pend.astype(np.float32) * np.float32(2.0 ** -40)
    return ((cur + delivered).astype(np.float32) * np.float32(cfg.current_decay)).astype(np.float32)


def network_to_dict(net, time=0.0, state=None, cfg=None, spike_counts=None):
    """The reference's serde JSON of `Network` for `net`. Without `state`:
    fresh neuron and synapse state (traces at rest, last spike at -1e9, delay
    1 ms). With `state` (SimulationEngine.checkpoint()) and its `cfg`: every
    dynamic field from it, `time` from its step, and the `device_state`
    object. spike_counts: per-neuron spike counts (NeuronArray.spike_count),
    zeros when not given."""
    n, m = net.n, net.m
    model = net.model
    name = {v: k for k, v in _MODEL_OF.items()}[model]
    fields = _FIELDS[model]
    rp = net.row_ptr.astype(np.int64)
    src = np.repeat(np.arange(n), np.diff(rp))
    ty = net.syn_type if net.syn_type is not None else np.zeros(m, np.uint8)
    pl = net.plastic if net.plastic is not None else np.zeros(m, np.uint8)
    dt = cfg.dt_ms if cfg is not None else 1.0
    if state is not None:
        if cfg is None:
            raise ValueError("a state needs its config")
        step = int(state["step"])
        time = step * dt
        w = np.asarray(state["w"], np.float64)
        last = np.asarray(state["last_spike_step"], np.int64)
        pre = np.asarray(state["pre_trace"], np.float64)
        post = np.asarray(state["post_trace"], np.float64)
        contrib = state.get("contributions")
        elig = state.get("eligibility")
    else:
        step = 0
        w = net.w.astype(np.float64)
        last = np.full(n, -1, np.int64)
        pre = post = np.zeros(n)
        contrib = elig = None
    eligible = (net.eligible if net.eligible is not None else pl) if elig is not None else None
    synapses = []
    for p in range(m):
        plastic = bool(pl[p])
        s, t = int(src[p]), int(net.col[p])
        trace = None
        if plastic:
            trace = {"pre_trace": float(pre[s]), "post_trace": float(post[t]),
                     "last_pre_spike": _spike_time(last[s], dt, True) if last[s] >= 0 else _NEVER,
                     "last_post_spike": _spike_time(last[t], dt, True) if last[t] >= 0 else _NEVER}
        stp = None
        if net.stp is not None and (net.has_stp is None or net.has_stp[p]):
            u_se, tau_rec, tau_facil, u, r = (float(x) for x in net.stp[p])
            stp = {"u_se": u_se, "tau_rec": tau_rec, "tau_facil": tau_facil, "u": u, "r": r}
        synapses.append({
            "source": s, "target": t, "weight": float(w[p]), "delay": 1.0,
            "synapse_type": _SYN_NAMES[int(ty[p])], "conductance": 0.0, "is_active": True,
            "conductance_state": ({"g": 0.0, "t_since_spike": 0.0, "pending_spike": False}
                                  if plastic else None),
            "stdp_trace": trace,
            "eligibility": ({"value": float(elig[p])} if eligible is not None and eligible[p] else None),
            "stp": stp, "plasticity_enabled": plastic,
            "contribution_avg": float(contrib[p]) if contrib is not None else 0.0})
    rest = [float(p[0] if model == A.MODEL_LIF else (p[2] if model == A.MODEL_IZHIKEVICH else p[5]))
            for p in net.params]
    lst = lambda a: [float(x) for x in a]
    inh = net.inhibitory if net.inhibitory is not None else np.zeros(n, np.uint8)
    outp = net.is_output if net.is_output is not None else np.zeros(n, np.uint8)
    if state is not None:
        v, u = lst(state["v"]), lst(state["u"])
        refr = [int(x) for x in state["refractory"]]
        hm, hh, hn = lst(state["hh_m"]), lst(state["hh_h"]), lst(state["hh_n"])
        cur = lst(_reference_current(state, cfg, step))
        last_t = [_spike_time(k, dt, False) if k >= 0 else _NEVER for k in last]
        just = [bool(k == step - 1 and step > 0) for k in last]
    else:
        v = lst(net.v0) if net.v0 is not None else rest
        u = lst(net.u0) if net.u0 is not None else [0.0] * n
        refr, cur, last_t, just = [0] * n, [0.0] * n, [_NEVER] * n, [False] * n
        hm = lst(net.m0) if net.m0 is not None else [0.05] * n
        hh = lst(net.h0) if net.h0 is not None else [0.6] * n
        hn = lst(net.n0) if net.n0 is not None else [0.32] * n
    counts = [int(x) for x in spike_counts] if spike_counts is not None else [0] * n
    neurons = {
        "membrane_potential": v, "recovery_variable": u, "refractory_counter": refr,
        "last_spike_time": last_t, "spike_count": counts,
        "neuron_type": ["Inhibitory" if x else "Excitatory" for x in inh],
        "model_params": [{name: {f: float(x) for f, x in zip(fields, row)}} for row in net.params],
        "input_current": cur, "is_output": [bool(x) for x in outp],
        "hh_m": hm, "hh_h": hh, "hh_n": hn, "just_spiked": just,
    }
    out = {"name": net.name, "neurons": neurons, "adjacency_ptr": [int(x) for x in rp],
           "synapses": synapses, "adjacency_indices": [int(x) for x in net.col], "time": float(time),
           "neuron_region": [0] * n, "region_names": ["Default"]}
    if state is not None:
        ds = {"step": step, "current": lst(state["current"]),
              "pending_input": [int(x) for x in state["pending_input"]],
              "conductance": lst(state["conductance"]), "firing_rate": lst(state["firing_rate"]),
              "pre_trace": lst(state["pre_trace"]), "post_trace": lst(state["post_trace"])}
        if state.get("reward") is not None:
            ds["reward"] = float(state["reward"])
        out["device_state"] = ds
    return out


def save_network_json(net, path, time=0.0, state=None, cfg=None, spike_counts=None):
    with open(path, "w") as f:
        json.dump(network_to_dict(net, time, state, cfg, spike_counts), f, indent=2)


class CheckpointManager:
    """CheckpointManager (src/io/checkpoint.rs:21-160): `<name>.json` (the
    network) and `<name>_meta.json` (CheckpointMetadata: name, sim_time_ms,
    neuron_count, synapse_count, total_spikes, timestamp, seed) in one
    directory, at most max_checkpoints kept (the earliest in simulated time
    pruned), auto-save every auto_save_interval_ms of simulated time."""

    def __init__(self, checkpoint_dir, max_checkpoints=10, auto_save_interval_ms=1000.0):
        self.checkpoint_dir = str(checkpoint_dir)
        os.makedirs(self.checkpoint_dir, exist_ok=True)
        self.max_checkpoints = max_checkpoints
        self.auto_save_interval_ms = auto_save_interval_ms
        self.last_save_time = 0.0

    def _paths(self, name):
        return (os.path.join(self.checkpoint_dir, f"{name}.json"),
                os.path.join(self.checkpoint_dir, f"{name}_meta.json"))

    def save(self, net, state, cfg, name, total_spikes=0, seed=None):
        """Saves a network with its dynamic state (SimulationEngine.checkpoint())
        as `<name>.json` and the metadata as `<name>_meta.json`, then prunes."""
        path, meta_path = self._paths(name)
        meta = {"name": name, "sim_time_ms": int(state["step"]) * cfg.dt_ms,
                "neuron_count": net.n, "synapse_count": net.m, "total_spikes": int(total_spikes),
                "timestamp": f"{_time.time():.9f}s", "seed": int(cfg.seed if seed is None else seed)}
        with open(meta_path, "w") as f:
            json.dump(meta, f, indent=2)
        save_network_json(net, path, state=state, cfg=cfg)
        self.prune()
        return path

    def save_engine(self, engine, name):
        """save() of a running SimulationEngine (save_engine, checkpoint.rs:78-82)."""
        return self.save(engine.network, engine.checkpoint(), engine.config, name,
                         total_spikes=engine.counters()[1])

    def load(self, name, cfg, csr_order="records"):
        """(Network, state for SimulationEngine.restore, metadata)."""
        path, meta_path = self._paths(name)
        with open(path) as f:
            d = json.load(f)
        with open(meta_path) as f:
            meta = json.load(f)
        net = network_from_dict(d, csr_order)
        return net, state_from_dict(d, net, cfg, csr_order), meta

    def should_auto_save(self, current_time):
        return current_time - self.last_save_time >= self.auto_save_interval_ms

    def mark_saved(self, current_time):
        self.last_save_time = current_time

    def list_checkpoints(self):
        """Metadata of every checkpoint in the directory, latest simulated
        time first."""
        out = []
        for fn in os.listdir(self.checkpoint_dir):
            if fn.endswith(".json") and "_meta." not in fn:
                meta_path = os.path.join(self.checkpoint_dir, fn[:-5] + "_meta.json")
                try:
                    with open(meta_path) as f:
                        out.append(json.load(f))
                except (OSError, ValueError):
                    continue
        out.sort(key=lambda m: m["sim_time_ms"], reverse=True)
        return out

    def prune(self):
        cps = self.list_checkpoints()
        if len(cps) <= self.max_checkpoints:
            return
        cps.sort(key=lambda m: m["sim_time_ms"])
        for cp in cps[:len(cps) - self.max_checkpoints]:
            for p in self._paths(cp["name"]):
                try:
                    os.remove(p)
                except OSError:
                    pass
