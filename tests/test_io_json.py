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
