"""GPU parity for the rest of phase 2: R-STDP eligibility and reward
(engine.rs:519-563, :626-631; apply_reward :158-175), consolidation
(plasticity.rs:269-290) in the device's affine weight frame, short-term
plasticity (engine.rs:457-463) and the reference conductance mode with all
four synapse types. Against the float oracle, which mirrors the device
arithmetic: bit-exact unless a test states a tolerance."""
import numpy as np
import pytest

from oracle.oracle import FastOracle
from neuralsim_b200 import _abi as A
from neuralsim_b200 import SimulationEngine, NsError
import nets

pytestmark = pytest.mark.gpu


def same_weights(eng, o):
    return np.array_equal(eng.download_state()["w"].astype(np.float64), o.weights())


@pytest.mark.parametrize("wf", [A.WEIGHT_F32, A.WEIGHT_BF16])
def test_rstdp_bit_exact(lib, wf):
    # rewarded stretches start and stop: both reward paths run (in the walks
    # when the previous step applied the reward, else the full pass)
    net, cfg, drive = nets.izh_rstdp(n=4000, k=60, wf=wf)
    cfg.graph_chunk = 50
    eng = SimulationEngine(net, cfg, drive)
    o = FastOracle(net, cfg, drive, precision=32)
    rewards = []
    for _ in range(12):
        eng.run(50)
        o.step(50)
        r_gpu, r_or = eng.reward(), o.reward()
        assert r_gpu[0] == r_or[0] and r_gpu[1] == pytest.approx(r_or[1], rel=1e-12, abs=1e-12)
        rewards.append(r_or[0])
    ra, rb = eng.read_raster(0, 600), o.raster()
    assert len(rb[0]) > 5000
    assert nets.rasters_equal(ra, rb)
    assert same_weights(eng, o)
    assert np.array_equal(eng.eligibility().astype(np.float64), o.eligibility())
    assert o.reward()[1] > 1.0


@pytest.mark.parametrize("sched", [1, 2, 3, 4])
def test_rstdp_schedules_identical(lib, sched):
    net, cfg, drive = nets.izh_rstdp(n=8000, k=60)
    cfg.step_schedule = sched
    cfg.graph_chunk = 100
    eng = SimulationEngine(net, cfg, drive)
    eng.run(350)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(350)
    assert eng.schedule()[0] == sched
    assert nets.rasters_equal(eng.read_raster(0, 350), o.raster())
    assert same_weights(eng, o)
    assert np.array_equal(eng.eligibility().astype(np.float64), o.eligibility())


def test_rstdp_subset_eligible(lib):
    # half of the plastic synapses carry an eligibility trace (with_rstdp on
    # some synapses only): the walks read the per-synapse flags
    net, cfg, drive = nets.izh_rstdp(n=4000, k=60)
    rng = np.random.default_rng(3)
    net.eligible = (rng.random(net.m) < 0.5).astype(np.uint8)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(300)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(300)
    assert nets.rasters_equal(eng.read_raster(0, 300), o.raster())
    assert same_weights(eng, o)
    e = eng.eligibility()
    assert np.array_equal(e.astype(np.float64), o.eligibility())
    assert not np.any(e[net.eligible == 0])


def test_rstdp_full_pass_config(lib):
    # R-STDP range narrower than STDP's: every rewarded step takes the full pass
    net, cfg, drive = nets.izh_rstdp(n=4000, k=60, rstdp_w_max=4.0)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(300)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(300)
    assert nets.rasters_equal(eng.read_raster(0, 300), o.raster())
    assert same_weights(eng, o)
    assert np.array_equal(eng.eligibility().astype(np.float64), o.eligibility())


@pytest.mark.parametrize("wf", [A.WEIGHT_F32, A.WEIGHT_BF16])
def test_consolidation_frame_with_renormalisation(lib, wf):
    # a = 0.9 per step: the frame renormalises every ~105 steps; STDP and
    # R-STDP write through the frame
    net, cfg, drive = nets.izh_rstdp(n=4000, k=60, wf=wf)
    nets.with_consolidation(cfg, tau=10.0, drift=1.0)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(450)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(450)
    assert nets.rasters_equal(eng.read_raster(0, 450), o.raster())
    assert same_weights(eng, o)
    assert np.array_equal(eng.eligibility().astype(np.float64), o.eligibility())
    mean, std = eng.weight_stats()
    w = o.weights()
    assert mean == pytest.approx(w.mean(), rel=1e-9) and std == pytest.approx(w.std(), rel=1e-6)


def test_consolidation_default_rule_slow_drift(lib):
    # the default rule's drift (1e-7 of target - w per step) is tracked
    net, cfg, drive = nets.izh_rstdp(n=4000, k=60)
    nets.with_consolidation(cfg)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(500)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(500)
    assert nets.rasters_equal(eng.read_raster(0, 500), o.raster())
    assert same_weights(eng, o)


def test_rstdp_consolidation_homeostasis(lib):
    # with homeostasis (FP64 rate sums, per-synapse exp): rasters equal the
    # float oracle, weights within 1e-5 relative
    net, cfg, drive = nets.lif_reference_default(n=2000)
    net.is_output = (np.arange(net.n) < 400).astype(np.uint8)
    cfg.rstdp_enabled = True
    cfg.reward_threshold = 2
    nets.with_consolidation(cfg, tau=200.0, drift=0.05)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(100)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(100)
    assert nets.rasters_equal(eng.read_raster(0, 100), o.raster())
    w = eng.download_state()["w"].astype(np.float64)
    assert np.allclose(w, o.weights(), rtol=1e-5, atol=1e-6)
    assert eng.reward()[0] == o.reward()[0]


@pytest.mark.parametrize("mode", ["direct", "delta_delay"])
def test_stp_bit_exact(lib, mode):
    if mode == "direct":
        net, cfg, drive = nets.lif_reference_default(n=3000, stdp=False, homeo=False)
        steps = 200
    else:
        net, cfg, drive = nets.lif_delta(n=5000, k=80)   # windowed path is replaced by the step path
        steps = 600
    nets.with_stp(net)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(steps)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(steps)
    ra, rb = eng.read_raster(0, steps), o.raster()
    assert len(rb[0]) > 100
    assert nets.rasters_equal(ra, rb)
    assert np.array_equal(eng.download_state()["v"].astype(np.float64), o.state()["v"])
    assert eng.window()[0] == 0


def test_apply_reward_and_eligibility_io(lib):
    net, cfg, drive = nets.izh_rstdp(n=4000, k=60, n_out=0)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(150)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(150)
    e = eng.eligibility()
    assert np.count_nonzero(e) > 1000
    assert np.array_equal(e.astype(np.float64), o.eligibility())
    eng.apply_reward(0.7)
    o.apply_reward(0.7)
    assert same_weights(eng, o)
    assert not np.any(eng.eligibility())
    eng.run(80)
    o.step(80)
    assert nets.rasters_equal(eng.read_raster(0, 230), o.raster())
    assert same_weights(eng, o)
    # uploaded values come back; the reward can be set
    vals = np.linspace(-1, 1, net.m).astype(np.float32)
    eng.upload_eligibility(values=vals)
    assert np.array_equal(eng.eligibility(), vals)
    eng.set_reward(0.25)
    assert eng.reward() == (0.25, 0.0)


def test_rstdp_checkpoint_resume_bit_exact(lib):
    # state + eligibility + reward round-trip: the resumed run equals the
    # uninterrupted one
    net, cfg, drive = nets.izh_rstdp(n=4000, k=60)
    a = SimulationEngine(net, cfg, drive)
    a.run(400)
    full_raster = a.read_raster(200, 200)
    full_state = a.download_state()
    full_e = a.eligibility()
    b = SimulationEngine(net, cfg, drive)
    b.run(200)
    snap, snap_e, snap_r = b.download_state(), b.eligibility(), b.reward()[0]
    b.close()
    c = SimulationEngine(net, cfg, drive)
    c.upload_state(snap, 200)
    c.upload_eligibility(values=snap_e)
    c.set_reward(snap_r)
    c.run(200)
    st = c.download_state()
    for key in ("v", "u", "pre_trace", "post_trace", "w"):
        assert np.array_equal(st[key], full_state[key]), key
    assert np.array_equal(c.eligibility(), full_e)
    assert nets.rasters_equal(c.read_raster(200, 200), full_raster)


def test_reward_needs_rstdp_or_consolidation(lib):
    net, cfg, drive = nets.izh_stdp(n=2000, k=40)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(10)
    with pytest.raises(NsError):
        eng.reward()
    # without R-STDP apply_reward is a no-op (engine.rs:158-175)
    w0 = eng.download_state()["w"]
    eng.apply_reward(1.0)
    assert np.array_equal(eng.download_state()["w"], w0)


def test_conductance_ref_all_types(lib):
    net, cfg, drive = nets.lif_conductance_all_types(n=3000)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(100)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(100)
    ra, rb = eng.read_raster(0, 100), o.raster()
    assert len(rb[0]) > 100
    assert nets.rasters_equal(ra, rb)
    v = eng.download_state()["v"].astype(np.float64)
    assert np.allclose(v, o.state()["v"], rtol=1e-5, atol=1e-4)


def test_stp_ignored_in_conductance_mode(lib):
    # the reference applies STP only to direct current injection
    # (engine.rs:457-463): a conductance network steps as without it
    net, cfg, drive = nets.lif_reference_default(n=2000, stdp=False, homeo=False, conductance=True)
    plain = SimulationEngine(net, cfg, drive)
    plain.run(100)
    nets.with_stp(net)
    eng = SimulationEngine(net, cfg, drive)
    eng.run(100)
    assert nets.rasters_equal(eng.read_raster(0, 100), plain.read_raster(0, 100))


def test_rstdp_entry_points_before_stepping_and_without_rstdp(lib):
    net, cfg, drive = nets.izh_rstdp(n=2000, k=20)
    eng = SimulationEngine(net, cfg, drive)
    eng.apply_reward(1.0)                    # before any step: e = 0 everywhere, no change
    assert np.array_equal(eng.download_state()["w"], net.w)
    assert eng.reward() == (cfg.reward_signal, 0.0)
    with pytest.raises(ValueError):
        eng.upload_eligibility(values=np.zeros(net.m - 1, np.float32))   # one entry short
    eng.close()
    net2, cfg2, drive2 = nets.izh_stdp(n=2000, k=20)
    e2 = SimulationEngine(net2, cfg2, drive2)
    with pytest.raises(NsError):
        e2.upload_eligibility(values=np.zeros(net2.m, np.float32))   # R-STDP is off
    e2.close()

