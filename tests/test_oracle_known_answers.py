"""The reference's own unit tests for this path, restated against the oracle.

Each test cites the reference test it re-expresses (same dt, inputs and
assertion). These pin the CPU restatement to the reference's observable
behaviour; the reference itself (Rust) cannot be built in this image.
"""
import ctypes as C
import math

import numpy as np
import pytest


def dp(x):
    return C.byref(x)


LIF_DEFAULT = (C.c_double * 6)(-60.0, -50.0, -65.0, 8.0, 1.5, 2.0)  # neuron/mod.rs:106-117


def test_lif_subthreshold(oracle_lib):
    # src/neuron/lif.rs:68-74: default LIF at rest, dt 0.1, I 0 -> no spike
    v, r = C.c_double(-60.0), C.c_int32(0)
    assert oracle_lib.or_lif_step_f64(dp(v), dp(r), LIF_DEFAULT, 0.1, 0.0) == 0


def test_lif_fires_at_threshold(oracle_lib):
    # src/neuron/lif.rs:76-84: V = -49 spikes in one step, resets below -60
    v, r = C.c_double(-49.0), C.c_int32(0)
    assert oracle_lib.or_lif_step_f64(dp(v), dp(r), LIF_DEFAULT, 0.1, 0.0) == 1
    assert v.value < -60.0


def test_lif_refractory_period(oracle_lib):
    # src/neuron/lif.rs:86-99: refractory blocks a spike even with I = 1000
    v, r = C.c_double(-49.0), C.c_int32(0)
    assert oracle_lib.or_lif_step_f64(dp(v), dp(r), LIF_DEFAULT, 0.1, 0.0) == 1
    assert oracle_lib.or_lif_step_f64(dp(v), dp(r), LIF_DEFAULT, 0.1, 1000.0) == 0
    assert r.value == 14  # round(1.5 / 0.1) - 1


def test_izhikevich_fires(oracle_lib):
    # src/neuron/izhikevich.rs:78-91: RS neuron from -65 with I = 10, dt 0.5,
    # fires within 200 steps
    p = (C.c_double * 4)(0.02, 0.2, -65.0, 8.0)
    v, u = C.c_double(-65.0), C.c_double(0.0)
    fired = any(oracle_lib.or_izh_step_f64(dp(v), dp(u), p, 0.5, 10.0) for _ in range(200))
    assert fired


HH = (C.c_double * 7)(120.0, 36.0, 0.3, 50.0, -77.0, -54.387, 1.0)  # hodgkin_huxley.rs:104-116


def test_hh_resting_potential(oracle_lib):
    # src/neuron/hodgkin_huxley.rs:122-129: one step at I 0, dt 0.01 stays within 1 mV of -65
    v, m, h, n = C.c_double(-65.0), C.c_double(0.05), C.c_double(0.6), C.c_double(0.32)
    assert oracle_lib.or_hh_step_f64(dp(v), dp(m), dp(h), dp(n), HH, 0.01, 0.0, 0) == 0
    assert abs(v.value + 65.0) < 1.0


def test_hh_fires_with_current(oracle_lib):
    # src/neuron/hodgkin_huxley.rs:131-144: fires within 500 steps of 0.01 ms at I 10
    v, m, h, n = C.c_double(-65.0), C.c_double(0.05), C.c_double(0.6), C.c_double(0.32)
    fired = any(oracle_lib.or_hh_step_f64(dp(v), dp(m), dp(h), dp(n), HH, 0.01, 10.0, 0)
                for _ in range(500))
    assert fired


def test_hh_gating_state_persists(oracle_lib):
    # src/neuron/hodgkin_huxley.rs:146-163: gates change on successive steps (dt 0.1)
    v, m, h, n = C.c_double(-65.0), C.c_double(0.05), C.c_double(0.6), C.c_double(0.32)
    g0 = (m.value, h.value, n.value)
    oracle_lib.or_hh_step_f64(dp(v), dp(m), dp(h), dp(n), HH, 0.1, 0.0, 0)
    g1 = (m.value, h.value, n.value)
    assert g1 != g0
    oracle_lib.or_hh_step_f64(dp(v), dp(m), dp(h), dp(n), HH, 0.1, 0.0, 0)
    assert (m.value, h.value, n.value) != g1


def test_hh_rush_larsen_rest_is_steady(oracle_lib):
    # the Rush-Larsen variant keeps the squid axon at rest without input
    v, m, h, n = C.c_double(-65.0), C.c_double(0.0529), C.c_double(0.5961), C.c_double(0.3177)
    p = (C.c_double * 7)(120.0, 36.0, 0.3, 50.0, -77.0, -54.4, 1.0)
    for _ in range(1000):
        assert oracle_lib.or_hh_step_f64(dp(v), dp(m), dp(h), dp(n), p, 0.01, 0.0, 1) == 0
    assert abs(v.value + 65.0) < 0.5


def test_hh_rate_singularities_take_limits(oracle_lib):
    # alpha_m at V=-40 and alpha_n at V=-55 are 0/0 in hodgkin_huxley.rs:20-42
    for v0 in (-40.0, -55.0):
        v, m, h, n = C.c_double(v0), C.c_double(0.05), C.c_double(0.6), C.c_double(0.32)
        oracle_lib.or_hh_step_f64(dp(v), dp(m), dp(h), dp(n), HH, 0.01, 0.0, 1)
        assert all(math.isfinite(x) for x in (v.value, m.value, h.value, n.value))


def test_ampa_conductance(oracle_lib):
    # src/synapse/types.rs:114-126
    g0 = oracle_lib.or_dual_exp_conductance(0, 0.0)
    g1 = oracle_lib.or_dual_exp_conductance(0, 1.0)
    gf = oracle_lib.or_dual_exp_conductance(0, 100.0)
    assert abs(g0) < 1e-10 and g1 > 0 and gf < g1


def test_nmda_mg_block(oracle_lib):
    # src/synapse/types.rs:128-166
    assert oracle_lib.or_mg_block(3, 20.0) > 0.7
    assert oracle_lib.or_mg_block(3, -80.0) < 0.3
    b = oracle_lib.or_mg_block(3, -65.0)
    assert 0.01 < b < 0.5
    assert oracle_lib.or_mg_block(0, -65.0) == 1.0


def test_gaba_b_slow(oracle_lib):
    # src/synapse/types.rs:168-189
    g = lambda t: oracle_lib.or_dual_exp_conductance(2, t)
    assert g(30.0) > g(1.0)
    assert g(60.0) > g(300.0)


def test_conductance_peak_normalization(oracle_lib):
    # src/synapse/types.rs:191-204
    tr, td = 0.5, 2.0
    tpk = (tr * td / (td - tr)) * math.log(td / tr)
    assert abs(oracle_lib.or_dual_exp_conductance(0, tpk) - 1.0) < 0.01


def test_stdp_signs_and_clamp(oracle_lib):
    # src/synapse/plasticity.rs:324-344
    assert oracle_lib.or_stdp_weight_change(0.01, 0.012, 20.0, 20.0, 10.0) > 0
    assert oracle_lib.or_stdp_weight_change(0.01, 0.012, 20.0, 20.0, -10.0) < 0


def test_short_term_plasticity(oracle_lib):
    # src/synapse/plasticity.rs:346-353
    u, r = C.c_double(0.5), C.c_double(1.0)
    e1 = oracle_lib.or_stp_step(dp(u), dp(r), 0.5, 100.0, 1000.0, 1.0, 1)
    e2 = oracle_lib.or_stp_step(dp(u), dp(r), 0.5, 100.0, 1000.0, 1.0, 1)
    assert e1 > 0 and e2 <= e1


def test_stdp_trace_decay_known_answer(oracle_lib):
    # src/synapse/plasticity.rs:355-362: on_pre_spike(0, 20) then decay(20) -> 0.3679 +- 0.01
    pre, last = C.c_double(0.0), C.c_double(-1e9)
    oracle_lib.or_trace_on_spike(dp(pre), dp(last), 0.0, 20.0)
    assert pre.value > 0.9
    post = C.c_double(0.0)
    oracle_lib.or_trace_decay(dp(pre), dp(post), 20.0, 20.0, 20.0)
    assert abs(pre.value - 0.3679) < 0.01


def test_eligibility_known_answer(oracle_lib):
    # src/synapse/plasticity.rs:364-373: w 0.5 -> 0.505, trace cleared
    val, w = C.c_double(0.0), C.c_double(0.5)
    oracle_lib.or_eligibility_update(dp(val), 1.0, 200.0, 0.05)
    assert val.value > 0
    oracle_lib.or_eligibility_apply(dp(val), 1.0, dp(w), 0.1, 0.0, 10.0)
    assert abs(w.value - 0.505) < 0.001
    assert abs(val.value) < 1e-10


def test_consolidation_drift(oracle_lib):
    # src/synapse/plasticity.rs:383-389
    w = C.c_double(5.0)
    oracle_lib.or_consolidation_apply(dp(w), 10000.0, 0.5, 0.001, 1000.0)
    assert abs(w.value - 5.0) < 1.0
