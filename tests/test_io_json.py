"""The reference's serde-JSON network format (src/io/save.rs, load.rs):
round trip of a generated network, a hand-built document in the reference's
field layout (records in insertion order, permuted to CSR order by a stable
sort by source, as Network::finalize orders the adjacency), and rejection
of mixed models and inconsistent adjacency."""
import json

import numpy as np
import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200 import io as nio
import nets as tnets


def test_round_trip_generated_network(lib, tmp_path):
    net, _, _ = tnets.izh_stdp(n=300, k=20)
    p = tmp_path / "net.json"
    nio.save_network_json(net, p)
    back = nio.load_network_json(p)
    assert back.model == net.model and back.n == net.n and back.m == net.m
    for a, b in ((back.row_ptr, net.row_ptr), (back.col, net.col), (back.w, net.w),
                 (back.syn_type, net.syn_type), (back.plastic, net.plastic),
                 (back.params, net.params), (back.v0, net.v0), (back.u0, net.u0),
                 (back.inhibitory, net.inhibitory)):
        assert np.array_equal(a, b)


def _doc():
    lif = {"Lif": {"resting": -60.0, "threshold": -50.0, "reset": -65.0, "tau_m": 8.0,
                   "refractory_period": 1.5, "input_resistance": 2.0}}

    def syn(s, t, w, ty="AMPA", plastic=False):
        return {"source": s, "target": t, "weight": w, "delay": 1.0, "synapse_type": ty,
                "conductance": 0.0, "is_active": True, "conductance_state": None,
                "stdp_trace": ({"pre_trace": 0.0, "post_trace": 0.0, "last_pre_spike": -1e9,
                                "last_post_spike": -1e9} if plastic else None),
                "eligibility": None, "stp": None, "plasticity_enabled": plastic,
                "contribution_avg": 0.0}
    # insertion order: 2->0, 0->1, 2->1, 0->2, 1->0
    synapses = [syn(2, 0, 1.5), syn(0, 1, 2.0, plastic=True), syn(2, 1, -1.0, "GABA"),
                syn(0, 2, 0.5, "NMDA"), syn(1, 0, 3.0)]
    n = 3
    return {"name": "tiny", "neurons": {
        "membrane_potential": [-60.0, -55.0, -61.0], "recovery_variable": [0.0] * n,
        "refractory_counter": [0] * n, "last_spike_time": [-1e9] * n, "spike_count": [0] * n,
        "neuron_type": ["Excitatory", "Excitatory", "Inhibitory"], "model_params": [lif] * n,
        "input_current": [0.0] * n, "is_output": [False, True, False], "hh_m": [0.05] * n,
        "hh_h": [0.6] * n, "hh_n": [0.32] * n, "just_spiked": [False] * n},
        "adjacency_ptr": [0, 2, 3, 5], "synapses": synapses,
        "adjacency_indices": [1, 2, 0, 0, 1], "time": 0.0, "neuron_region": [0] * n,
        "region_names": ["Default"]}


def test_reference_document_in_csr_order(lib):
    net = nio.network_from_dict(_doc())
    assert net.model == A.MODEL_LIF and net.n == 3 and net.m == 5
    assert list(net.row_ptr) == [0, 2, 3, 5]
    assert list(net.col) == [1, 2, 0, 0, 1]
    assert np.allclose(net.w, [2.0, 0.5, 3.0, 1.5, -1.0])
    assert list(net.syn_type) == [A.SYN_AMPA, A.SYN_NMDA, A.SYN_AMPA, A.SYN_AMPA, A.SYN_GABA]
    assert list(net.plastic) == [1, 0, 0, 0, 0]
    assert list(net.inhibitory) == [0, 0, 1] and list(net.is_output) == [0, 1, 0]
    assert np.allclose(net.params[0], [-60.0, -50.0, -65.0, 8.0, 1.5, 2.0])
    assert np.allclose(net.v0, [-60.0, -55.0, -61.0])


def test_rejects_mixed_models_and_bad_adjacency(lib):
    d = _doc()
    d["neurons"]["model_params"][1] = {"Izhikevich": {"a": 0.02, "b": 0.2, "c": -65.0, "d": 8.0}}
    with pytest.raises(ValueError):
        nio.network_from_dict(d)
    d = _doc()
    d["adjacency_indices"] = [2, 1, 0, 0, 1]
    with pytest.raises(ValueError):
        nio.network_from_dict(json.loads(json.dumps(d)))


def test_csr_position_quirk_on_unsorted_records(lib):
    # the records of _doc() are not sorted by source. Per record (the
    # default) each synapse keeps its endpoints; per CSR position (the Rust
    # application's current-mode delivery, engine.rs:417-471: target =
    # adjacency_indices[idx], current = synapses[idx].weight) the record in
    # insertion order supplies the weight at position idx
    d = _doc()
    for s in d["synapses"]:
        s["plasticity_enabled"], s["stdp_trace"] = False, None
    rec = nio.network_from_dict(d)
    pos = nio.network_from_dict(d, csr_order="positions")
    assert np.array_equal(rec.col, pos.col) and np.array_equal(rec.row_ptr, pos.row_ptr)
    assert np.allclose(pos.w, [s["weight"] for s in d["synapses"]])
    assert not np.allclose(rec.w, pos.w)
    # input each target receives when every neuron spikes once
    adj = np.asarray(d["adjacency_indices"])
    want_pos = np.bincount(adj, weights=[s["weight"] for s in d["synapses"]], minlength=3)
    want_rec = np.bincount([s["target"] for s in d["synapses"]],
                           weights=[s["weight"] for s in d["synapses"]], minlength=3)
    assert np.allclose(np.bincount(pos.col, weights=pos.w, minlength=3), want_pos)
    assert np.allclose(np.bincount(rec.col, weights=rec.w, minlength=3), want_rec)
    assert not np.allclose(want_pos, want_rec)
    # sorted records: both orders agree
    d2 = nio.network_to_dict(rec)
    a, b = nio.network_from_dict(d2), nio.network_from_dict(d2, csr_order="positions")
    assert np.array_equal(a.w, b.w) and np.array_equal(a.syn_type, b.syn_type)
    # plastic records cannot be placed by position
    with pytest.raises(ValueError):
        nio.network_from_dict(_doc(), csr_order="positions")


def _state(net, cfg, step, rng):
    n, m = net.n, net.m
    last = rng.integers(-1, step, n).astype(np.int64)
    return {"v": rng.uniform(-70, -50, n).astype(np.float32),
            "u": rng.uniform(-15, 0, n).astype(np.float32),
            "refractory": rng.integers(0, 3, n).astype(np.int32),
            "current": rng.normal(0, 2, n).astype(np.float32),
            "hh_m": np.full(n, 0.05, np.float32), "hh_h": np.full(n, 0.6, np.float32),
            "hh_n": np.full(n, 0.32, np.float32),
            "pre_trace": np.where(last >= 0, rng.uniform(0, 2, n), 0).astype(np.float32),
            "post_trace": np.where(last >= 0, rng.uniform(0, 2, n), 0).astype(np.float32),
            "last_spike_step": last,
            "pending_input": rng.integers(-2 ** 41, 2 ** 41, n * cfg.delay_steps).astype(np.int64),
            "conductance": np.zeros(4 * n, np.float32),
            "firing_rate": rng.uniform(0, 20, n),
            "w": rng.uniform(0, 6, m).astype(np.float32), "step": step}


@pytest.mark.parametrize("exact", [True, False])
def test_dynamic_state_round_trip(lib, exact):
    # every dynamic field through the reference's format: with the
    # device_state object exactly, without it as the reference's fields give
    # it (the DIRECT_DECAY current converted, the step from Network.time)
    net, cfg, _ = tnets.lif_reference_default(n=120)
    st = _state(net, cfg, 57, np.random.default_rng(3))
    d = json.loads(json.dumps(nio.network_to_dict(net, state=st, cfg=cfg)))
    assert d["time"] == 57 * cfg.dt_ms
    k = 5
    assert d["neurons"]["last_spike_time"][k] == (st["last_spike_step"][k] * cfg.dt_ms
                                                  if st["last_spike_step"][k] >= 0 else -1e9)
    if not exact:
        del d["device_state"]
    back = nio.state_from_dict(d, nio.network_from_dict(d), cfg)
    assert back["step"] == 57
    for key in ("v", "u", "refractory", "pre_trace", "post_trace", "last_spike_step", "w"):
        assert np.array_equal(back[key], st[key]), key
    if exact:
        for key in ("current", "pending_input", "firing_rate"):
            assert np.array_equal(back[key], st[key]), key
    else:
        # the reference's current after the step: (I + delivered) * 0.92;
        # back on the device's side: that / 0.92, within one rounding
        want = (st["current"] + st["pending_input"].astype(np.float32) * np.float32(2.0 ** -40))
        assert np.allclose(back["current"], want, rtol=2e-7, atol=1e-6)


def test_checkpoint_manager_files_and_pruning(lib, tmp_path):
    # CheckpointManager (src/io/checkpoint.rs): <name>.json + <name>_meta.json,
    # listed latest first, the earliest in simulated time pruned
    net, cfg, _ = tnets.lif_reference_default(n=60)
    mgr = nio.CheckpointManager(tmp_path, max_checkpoints=3)
    rng = np.random.default_rng(1)
    for q, step in enumerate((10, 40, 20, 30)):
        mgr.save(net, _state(net, cfg, step, rng), cfg, f"cp{q}", total_spikes=100 + q)
    metas = mgr.list_checkpoints()
    assert [m["sim_time_ms"] for m in metas] == [s * cfg.dt_ms for s in (40, 30, 20)]
    assert not (tmp_path / "cp0.json").exists() and not (tmp_path / "cp0_meta.json").exists()
    m = json.load(open(tmp_path / "cp1_meta.json"))
    assert set(m) == {"name", "sim_time_ms", "neuron_count", "synapse_count", "total_spikes",
                      "timestamp", "seed"}
    assert m["neuron_count"] == net.n and m["synapse_count"] == net.m and m["total_spikes"] == 101
    back, st, meta = mgr.load("cp1", cfg)
    assert meta["name"] == "cp1" and st["step"] == 40 and back.m == net.m
    assert mgr.should_auto_save(1000.0) and not mgr.should_auto_save(999.0)
    mgr.mark_saved(1000.0)
    assert not mgr.should_auto_save(1500.0) and mgr.should_auto_save(2000.0)
