"""Pins of the oracle (and of the CUDA path) by values worked out by hand
from the reference's source lines, never produced by oracle/.

Each scenario is a network of two to four neurons whose spikes are forced
(host stimulus or an initial membrane potential above threshold), so that
the expected values follow from the reference's update rules in closed form
or in a few lines of plain FP64 arithmetic written here:

- STDP with pre and post spiking in the same step: LTP with the decayed post
  trace, then the pre trace bumped by on_pre_spike, then LTD with that
  bumped pre trace (src/simulation/engine.rs:512-534), and the trace bump's
  second decay exp(-(t - t_last)/tau) (src/synapse/plasticity.rs:144-159);
- the direct-current mode's input decay: I += w at delivery, I *= 0.92 at
  the end of every step, never cleared (engine.rs:456-471, :609-614);
- the conductance mode's input: g decays by exp(-dt/tau) every step, grows
  by w gmax at a spike, and I += g (E_rev - V) every step, never cleared
  (engine.rs:406-412, :432-455, :476-494);
- homeostatic scaling: contribution EMA at delivery (engine.rs:448-452,
  :465-469), w *= exp(-(rate - target) rel dt / tau) per synapse
  (engine.rs:569-606), and the firing-rate EMA (engine.rs:637-642).

The CPU tests check the FP64 oracle engines (literal and reformulated)
against these values to 1e-12; the GPU tests check the CUDA path through
the C ABI (FP32 state) to the tolerance each test states.
"""
import math

import numpy as np
import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200.engine import Drive, Network, SimConfig
from oracle.oracle import FastOracle, LiteralOracle


# ---------------------------------------------------------------------------
# A: STDP order and the double decay
# ---------------------------------------------------------------------------
STDP_PLAN = {1: (0, 1), 6: (1,), 15: (0,), 22: (0, 1)}   # step -> neurons forced to spike
STDP_STEPS = 25


def stdp_scenario():
    # Izhikevich a .02, b .2, c -70, d 0, at rest (-70, -14); synapse 0 -> 1,
    # plastic, w 0.5; input mode reset-each-step so that a stimulus of 1000
    # acts for one step (V jumps above 30 and the neuron fires at the next
    # step, izhikevich.rs:33-49)
    params = np.array([[0.02, 0.2, -70.0, 0.0]] * 2, np.float32)
    net = Network(A.MODEL_IZHIKEVICH, params, np.array([0, 1, 1], np.uint64),
                  np.array([1], np.uint32), np.array([0.5], np.float32),
                  plastic=np.array([1], np.uint8), v0=np.full(2, -70.0), u0=np.full(2, -14.0))
    cfg = SimConfig(model=A.MODEL_IZHIKEVICH, input_mode=A.INPUT_RESET_EACH_STEP, dt_ms=1.0,
                    stdp_enabled=True, tau_plus=20.0, tau_minus=20.0, a_plus=0.1, a_minus=0.12,
                    w_min=0.0, w_max=10.0, homeostasis_enabled=False,
                    spike_log_capacity=1000, spike_log_steps=100)
    return net, cfg, Drive()


def stdp_expected():
    # per-synapse StdpTrace of engine.rs:497-537 with the spikes of STDP_PLAN
    E = lambda steps: math.exp(-steps / 20.0)
    w = 0.5
    w = min(max(w + 0.1 * 0.0, 0.0), 10.0)                    # step 1: LTP, post trace 0
    pre1 = 0.0 * math.exp(-(1.0 + 1e9) / 20.0) + 1.0           # on_pre_spike from -1e9
    w = min(max(w - 0.12 * pre1, 0.0), 10.0)                   # LTD with the bumped pre trace
    post1 = 1.0
    # step 6, post alone: LTD with the pre trace decayed 5 steps
    w = min(max(w - 0.12 * pre1 * E(5), 0.0), 10.0)
    post6 = (post1 * E(5)) * E(5) + 1.0                        # decayed, then the bump's decay
    # step 15, pre alone: LTP with the post trace decayed 9 steps
    w = min(max(w + 0.1 * post6 * E(9), 0.0), 10.0)
    pre15 = (pre1 * E(14)) * E(14) + 1.0
    # step 22, both: LTP with the decayed post, then LTD with the bumped pre
    w = min(max(w + 0.1 * post6 * E(16), 0.0), 10.0)
    pre22 = (pre15 * E(7)) * E(7) + 1.0
    w = min(max(w - 0.12 * pre22, 0.0), 10.0)
    post22 = (post6 * E(16)) * E(16) + 1.0
    # traces after the last step (25 steps: indices 0..24): 2 more decays
    return w, pre22 * E(2), post22 * E(2)


def drive_plan(step_fn, stim_fn, plan, steps):
    for k in range(steps):
        ids = plan.get(k + 1)
        if ids:
            stim_fn(list(ids), 1000.0)
        step_fn()


def raster_steps(idx, off):
    off = np.asarray(off, np.int64)
    return {k: tuple(int(x) for x in idx[off[k]:off[k + 1]]) for k in range(len(off) - 1)
            if off[k + 1] > off[k]}


@pytest.mark.parametrize("engine", ["fast", "literal"])
def test_stdp_same_step_order_and_double_decay_oracle(oracle_lib, engine):
    net, cfg, drive = stdp_scenario()
    o = FastOracle(net, cfg, drive, precision=64) if engine == "fast" else LiteralOracle(net, cfg, drive)
    drive_plan(lambda: o.step(1), o.stimulate, STDP_PLAN, STDP_STEPS)
    assert raster_steps(*o.raster()) == STDP_PLAN
    w, pre, post = stdp_expected()
    assert o.weights()[0] == pytest.approx(w, rel=1e-12, abs=1e-14)
    if engine == "fast":
        st = o.state()
        assert st["pre"][0] == pytest.approx(pre, rel=1e-12)
        assert st["post"][1] == pytest.approx(post, rel=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("sched", [3, 5])
def test_stdp_same_step_order_and_double_decay_gpu(lib, sched):
    from neuralsim_b200 import SimulationEngine
    net, cfg, drive = stdp_scenario()
    cfg.step_schedule = sched
    eng = SimulationEngine(net, cfg, drive)
    drive_plan(lambda: eng.run(1), eng.stimulate, STDP_PLAN, STDP_STEPS)
    assert raster_steps(*eng.read_raster(0, STDP_STEPS)) == STDP_PLAN
    w, pre, post = stdp_expected()
    st = eng.download_state()
    # FP32 traces and weights: a few float roundings per update
    assert float(st["w"][0]) == pytest.approx(w, rel=2e-6)
    assert float(st["pre_trace"][0]) == pytest.approx(pre, rel=2e-6)
    assert float(st["post_trace"][1]) == pytest.approx(post, rel=2e-6)
    eng.close()


# ---------------------------------------------------------------------------
# B: the direct-current mode's decay of the input current
# ---------------------------------------------------------------------------
LIF_P = [-60.0, -50.0, -65.0, 8.0, 1.5, 2.0]   # rest, threshold, reset, tau_m, t_ref, R


def lif_pair(input_mode, w, syn_type=A.SYN_AMPA):
    # neuron 0 starts at 0 mV: its first integration leaves it above
    # threshold, so it fires at step 0 (lif.rs:42-58) and never again;
    # neuron 1 rests and receives the synapse 0 -> 1
    params = np.array([LIF_P] * 2, np.float32)
    net = Network(A.MODEL_LIF, params, np.array([0, 1, 1], np.uint64), np.array([1], np.uint32),
                  np.array([w], np.float32), syn_type=np.array([syn_type], np.uint8),
                  plastic=np.zeros(1, np.uint8), v0=np.array([0.0, -60.0]))
    cfg = SimConfig(model=A.MODEL_LIF, input_mode=input_mode, dt_ms=0.5, stdp_enabled=False,
                    homeostasis_enabled=False, spike_log_capacity=1000, spike_log_steps=1000)
    return net, cfg, Drive()


def lif_update(v, I):
    rest, _, _, tau, _, R = LIF_P
    return v + (-(v - rest) + R * I) * 0.5 / tau


def f32(x):
    # weights are stored and uploaded as float32
    return float(np.float32(x))


def current_decay_expected(w, steps):
    # step 0: neuron 1 integrates I = 0; then delivery I += w and the decay
    # I *= 0.92 at the end of the step; step k >= 1 integrates w 0.92^k
    w = f32(w)
    v, I = -60.0, 0.0
    for k in range(steps):
        v = lif_update(v, I)
        if k == 0:
            I += w
        I *= 0.92
    return v, I


@pytest.mark.parametrize("engine", ["fast", "literal"])
def test_direct_current_decay_oracle(oracle_lib, engine):
    net, cfg, drive = lif_pair(A.INPUT_DIRECT_DECAY, 2.0)
    o = FastOracle(net, cfg, drive, precision=64) if engine == "fast" else LiteralOracle(net, cfg, drive)
    o.step(40)
    assert raster_steps(*o.raster()) == {0: (0,)}
    v, I = current_decay_expected(2.0, 40)
    st = o.state()
    assert st["v"][1] == pytest.approx(v, rel=1e-12)
    if engine == "literal":
        # the reference's own representation: input_current after the step
        assert st["I"][1] == pytest.approx(I, rel=1e-12)


@pytest.mark.gpu
def test_direct_current_decay_gpu(lib):
    from neuralsim_b200 import SimulationEngine
    net, cfg, drive = lif_pair(A.INPUT_DIRECT_DECAY, 2.0)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(40)
    assert raster_steps(*eng.read_raster(0, 40)) == {0: (0,)}
    v, _ = current_decay_expected(2.0, 40)
    assert float(eng.download_state()["v"][1]) == pytest.approx(v, rel=1e-6)
    eng.close()


# ---------------------------------------------------------------------------
# C: the conductance mode's never-cleared synaptic current
# ---------------------------------------------------------------------------
def conductance_expected(w, steps, dt=0.5, tau=2.0, erev=0.0):
    # per step: neuron update with I; conductance decay (all synapses), the
    # spike's increment w * gmax (AMPA: gmax 1, no Mg block) at step 0, then
    # I += g (E_rev - V) with V after this step's update; I is never cleared
    w = f32(w)
    v, I, g = -60.0, 0.0, 0.0
    for k in range(steps):
        v = lif_update(v, I)
        g *= math.exp(-dt / tau)
        if k == 0:
            g += w * 1.0
        if abs(g) >= 1e-12:
            I += g * (erev - v)
    return v, I


@pytest.mark.parametrize("engine", ["fast", "literal"])
def test_conductance_current_never_cleared_oracle(oracle_lib, engine):
    net, cfg, drive = lif_pair(A.INPUT_CONDUCTANCE_REF, 0.01)
    o = FastOracle(net, cfg, drive, precision=64) if engine == "fast" else LiteralOracle(net, cfg, drive)
    o.step(60)
    assert raster_steps(*o.raster()) == {0: (0,)}
    v, I = conductance_expected(0.01, 60)
    st = o.state()
    # the reformulated engine sums per-target conductances: reassociation only
    assert st["v"][1] == pytest.approx(v, rel=1e-12)
    if engine == "literal":
        assert st["I"][1] == pytest.approx(I, rel=1e-12)


@pytest.mark.gpu
def test_conductance_current_never_cleared_gpu(lib):
    from neuralsim_b200 import SimulationEngine
    net, cfg, drive = lif_pair(A.INPUT_CONDUCTANCE_REF, 0.01)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(60)
    assert raster_steps(*eng.read_raster(0, 60)) == {0: (0,)}
    v, I = conductance_expected(0.01, 60)
    st = eng.download_state()
    assert float(st["v"][1]) == pytest.approx(v, rel=1e-6)
    assert float(st["current"][1]) == pytest.approx(I, rel=1e-5)
    eng.close()


# ---------------------------------------------------------------------------
# D: homeostatic scaling and the firing-rate estimate
# ---------------------------------------------------------------------------
def homeo_scenario():
    # neurons 0 and 1 fire at step 0 (they start at 0 mV) and never again;
    # synapses 0->2 (1.0), 0->3 (0.7), 1->2 (2.0), 3->2 (1.5), in CSR order
    params = np.array([LIF_P] * 4, np.float32)
    rp = np.array([0, 2, 3, 3, 4], np.uint64)
    col = np.array([2, 3, 2, 2], np.uint32)
    w = np.array([1.0, 0.7, 2.0, 1.5], np.float32)
    net = Network(A.MODEL_LIF, params, rp, col, w, plastic=np.ones(4, np.uint8),
                  v0=np.array([0.0, 0.0, -60.0, -60.0]))
    cfg = SimConfig(model=A.MODEL_LIF, input_mode=A.INPUT_DIRECT_DECAY, dt_ms=0.5,
                    stdp_enabled=False, homeostasis_enabled=True, homeostatic_target_rate=5.0,
                    homeostatic_tau=5000.0, contribution_tau=1000.0,
                    spike_log_capacity=1000, spike_log_steps=100)
    return net, cfg, Drive()


def homeo_expected(steps, dt=0.5):
    # contributions exist only on the delivering synapses (step 0); every
    # step each target's synapses scale by exp(-(rate - 5) rel dt / 5000),
    # rate = 0 for the targets 2 and 3 throughout (they never fire), rel =
    # contribution / mean contribution over the target's incoming synapses
    cd = math.exp(-dt / 1000.0)
    w = np.array([1.0, 0.7, 2.0, 1.5], np.float32).astype(np.float64)   # CSR order
    c = np.array([w[0], w[1], w[2], 0.0]) * (1.0 - cd)
    targets = {2: [0, 2, 3], 3: [1]}
    for _ in range(steps):
        for t, syn in targets.items():
            mean = sum(c[s] for s in syn) / len(syn)
            for s in syn:
                rel = c[s] / mean
                w[s] = min(max(w[s] * math.exp(-(0.0 - 5.0) * rel * dt / 5000.0), 0.0), 10.0)
    # rates of the sources: 10 Hz after step 0, then x (1 - dt/100) per step
    r = (1000.0 / dt) * dt / 100.0
    for _ in range(steps - 1):
        r += (0.0 - r) * dt / 100.0
    return w, r


@pytest.mark.parametrize("steps", [1, 3])
@pytest.mark.parametrize("engine", ["fast", "literal"])
def test_homeostatic_scaling_oracle(oracle_lib, engine, steps):
    net, cfg, drive = homeo_scenario()
    o = FastOracle(net, cfg, drive, precision=64) if engine == "fast" else LiteralOracle(net, cfg, drive)
    o.step(steps)
    assert raster_steps(*o.raster()) == {0: (0, 1)}
    w, r = homeo_expected(steps)
    assert np.allclose(o.weights(), w, rtol=1e-12, atol=0)
    rates = o.rates()
    assert rates[0] == pytest.approx(r, rel=1e-12) and rates[1] == pytest.approx(r, rel=1e-12)
    assert rates[2] == 0.0 and rates[3] == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("steps", [1, 3])
def test_homeostatic_scaling_gpu(lib, steps):
    from neuralsim_b200 import SimulationEngine
    net, cfg, drive = homeo_scenario()
    eng = SimulationEngine(net, cfg, drive)
    eng.run(steps)
    assert raster_steps(*eng.read_raster(0, steps)) == {0: (0, 1)}
    w, r = homeo_expected(steps)
    # per-synapse scale in float with the project's exp: a few ulps
    assert np.allclose(eng.download_state()["w"], w, rtol=2e-6, atol=0)
    rates = eng.rates()
    # the rate estimate is FP64 on the device: the same operations
    assert rates[0] == pytest.approx(r, rel=1e-15) and rates[1] == pytest.approx(r, rel=1e-15)
    eng.close()
