"""The reference's on-disk network format (serde JSON of `Network`,
src/network/mod.rs:36-48, written by save_network_json / read by
load_network_json, src/io/save.rs:5-17, src/io/load.rs:6-17).

load_network_json turns a saved network into a `Network` for this library:
the neuron SoA (NeuronArray, src/neuron/mod.rs:126-163) with one parameter
row per neuron from its `model_params` variant, and the synapse records
(SynapseState, src/synapse/mod.rs:32-80) permuted into CSR order by a
stable sort by source, the order Network::finalize (mod.rs:79-106) gives
the adjacency. save_network_json writes a `Network` back in that format,
synapses in CSR order, so the Rust application can load it.
"""
import json

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


def network_from_dict(d):
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
    m = len(syn)
    src = np.array([s["source"] for s in syn], np.int64)
    tgt = np.array([s["target"] for s in syn], np.int64)
    if m and (src.max() >= n or tgt.max() >= n or src.min() < 0 or tgt.min() < 0):
        raise ValueError("synapse endpoint out of range")
    order = np.argsort(src, kind="stable")
    counts = np.bincount(src, minlength=n)
    row_ptr = np.zeros(n + 1, np.uint64)
    row_ptr[1:] = np.cumsum(counts)
    col = tgt[order].astype(np.uint32)
    if "adjacency_ptr" in d and len(d["adjacency_ptr"]) == n + 1:
        # a finalized network's adjacency is exactly this ordering
        if not (np.array_equal(np.asarray(d["adjacency_ptr"], np.uint64), row_ptr) and
                np.array_equal(np.asarray(d["adjacency_indices"], np.uint32), col)):
            raise ValueError("adjacency does not match the synapse records (not finalized?)")
    w = np.array([syn[i]["weight"] for i in order], np.float32)
    ty = np.array([_SYN_TYPES[syn[i]["synapse_type"]] for i in order], np.uint8)
    # STDP acts on records with plasticity enabled and a trace (engine.rs:500-502)
    pl = np.array([1 if (syn[i]["plasticity_enabled"] and syn[i].get("stdp_trace") is not None) else 0
                   for i in order], np.uint8)
    f32 = lambda key: np.asarray(nr[key], np.float32)
    net = Network(model, params, row_ptr, col, w, syn_type=ty, plastic=pl,
                  v0=f32("membrane_potential"), u0=f32("recovery_variable"),
                  m0=f32("hh_m"), h0=f32("hh_h"), n0=f32("hh_n"),
                  inhibitory=np.array([t == "Inhibitory" for t in nr["neuron_type"]], np.uint8),
                  is_output=np.asarray(nr.get("is_output", [False] * n), np.uint8),
                  name=d.get("name", "NeuralSim Network"))
    return net


def load_network_json(path):
    with open(path) as f:
        return network_from_dict(json.load(f))


def network_to_dict(net, time=0.0):
    """The reference's serde JSON of `Network` for `net` (fresh neuron and
    synapse state: traces at rest, last spike at -1e9, delay 1 ms)."""
    n, m = net.n, net.m
    model = net.model
    name = {v: k for k, v in _MODEL_OF.items()}[model]
    fields = _FIELDS[model]
    rp = net.row_ptr.astype(np.int64)
    src = np.repeat(np.arange(n), np.diff(rp))
    ty = net.syn_type if net.syn_type is not None else np.zeros(m, np.uint8)
    pl = net.plastic if net.plastic is not None else np.zeros(m, np.uint8)
    trace = {"pre_trace": 0.0, "post_trace": 0.0, "last_pre_spike": -1e9, "last_post_spike": -1e9}
    synapses = []
    for p in range(m):
        plastic = bool(pl[p])
        synapses.append({
            "source": int(src[p]), "target": int(net.col[p]), "weight": float(net.w[p]), "delay": 1.0,
            "synapse_type": _SYN_NAMES[int(ty[p])], "conductance": 0.0, "is_active": True,
            "conductance_state": ({"g": 0.0, "t_since_spike": 0.0, "pending_spike": False}
                                  if plastic else None),
            "stdp_trace": dict(trace) if plastic else None, "eligibility": None, "stp": None,
            "plasticity_enabled": plastic, "contribution_avg": 0.0})
    rest = [float(p[0] if model == A.MODEL_LIF else (p[2] if model == A.MODEL_IZHIKEVICH else p[5]))
            for p in net.params]
    arr = lambda a, default: ([float(x) for x in a] if a is not None else default)
    inh = net.inhibitory if net.inhibitory is not None else np.zeros(n, np.uint8)
    outp = net.is_output if net.is_output is not None else np.zeros(n, np.uint8)
    neurons = {
        "membrane_potential": arr(net.v0, rest),
        "recovery_variable": arr(net.u0, [0.0] * n),
        "refractory_counter": [0] * n, "last_spike_time": [-1e9] * n, "spike_count": [0] * n,
        "neuron_type": ["Inhibitory" if x else "Excitatory" for x in inh],
        "model_params": [{name: {f: float(v) for f, v in zip(fields, row)}} for row in net.params],
        "input_current": [0.0] * n, "is_output": [bool(x) for x in outp],
        "hh_m": arr(net.m0, [0.05] * n), "hh_h": arr(net.h0, [0.6] * n), "hh_n": arr(net.n0, [0.32] * n),
        "just_spiked": [False] * n,
    }
    return {"name": net.name, "neurons": neurons, "adjacency_ptr": [int(x) for x in rp],
            "synapses": synapses, "adjacency_indices": [int(x) for x in net.col], "time": float(time),
            "neuron_region": [0] * n, "region_names": ["Default"]}


def save_network_json(net, path, time=0.0):
    with open(path, "w") as f:
        json.dump(network_to_dict(net, time), f, indent=2)
