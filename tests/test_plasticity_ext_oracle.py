"""CPU: the rest of phase 2 in the oracle. R-STDP eligibility and reward
(engine.rs:519-563, :626-631), consolidation (plasticity.rs:269-290),
short-term plasticity (engine.rs:457-463) and the reference conductance mode
with all four synapse types. The fast engine (per-neuron traces, consolidation
frame) against the literal restatement (per-synapse state, O(M) loops)."""
import numpy as np
import pytest

from oracle.oracle import FastOracle, LiteralOracle
from neuralsim_b200 import _abi as A
from neuralsim_b200.engine import Drive
import nets


def run_pair(net, cfg, drive, steps, prec=64, every=None):
    f = FastOracle(net, cfg, drive, precision=prec)
    l = LiteralOracle(net, cfg, drive, threads=2)
    traj = []
    if every:
        for _ in range(steps):
            f.step(1)
            l.step(1)
            traj.append((f.reward()[0], l.reward()[0]))
    else:
        f.step(steps)
        l.step(steps)
    return f, l, np.array(traj)


def test_rstdp_fast_equals_literal(oracle_lib):
    # rewarded stretches start and stop (reward decay 0.5): the walks' reward
    # path (mode 1) and the full pass (mode 2) both run; FP64 results equal
    net, cfg, drive = nets.izh_rstdp(n=1500, k=40)
    f, l, traj = run_pair(net, cfg, drive, 300, every=True)
    assert np.array_equal(traj[:, 0], traj[:, 1])
    active = np.abs(traj[:, 0]) > 0.001
    assert np.sum(active[1:] & ~active[:-1]) >= 2 and np.sum(active) > 50
    ra, rb = f.raster(), l.raster()
    assert len(ra[0]) > 1000
    assert nets.rasters_equal(ra, rb)
    assert np.array_equal(f.weights(), l.weights())
    assert np.array_equal(f.eligibility(), l.eligibility())
    assert f.reward() == l.reward()
    assert np.count_nonzero(f.weights() != net.w.astype(np.float64)) > 1000


def test_rstdp_full_pass_config_fast_equals_literal(oracle_lib):
    # R-STDP range narrower than STDP's: the reward always takes the full pass
    net, cfg, drive = nets.izh_rstdp(n=1500, k=40, rstdp_w_max=4.0)
    f, l, _ = run_pair(net, cfg, drive, 250)
    assert nets.rasters_equal(f.raster(), l.raster())
    assert np.array_equal(f.weights(), l.weights())
    assert np.array_equal(f.eligibility(), l.eligibility())
    assert f.weights().max() <= 10.0


def test_eligibility_accumulates_between_rewards(oracle_lib):
    # no output neurons: the reward never comes, traces only accumulate
    net, cfg, drive = nets.izh_rstdp(n=1500, k=40, n_out=0)
    f, l, _ = run_pair(net, cfg, drive, 200)
    e = f.eligibility()
    assert np.count_nonzero(e) > 1000
    assert np.array_equal(e, l.eligibility())
    assert f.reward() == (0.0, 0.0)


def test_apply_reward_fast_equals_literal(oracle_lib):
    # SimulationEngine::apply_reward between steps (engine.rs:158-175)
    net, cfg, drive = nets.izh_rstdp(n=1500, k=40, n_out=0)
    f, l, _ = run_pair(net, cfg, drive, 120)
    f.apply_reward(0.7)
    l.apply_reward(0.7)
    assert np.array_equal(f.weights(), l.weights())
    assert not np.any(f.eligibility())
    f.step(60)
    l.step(60)
    assert nets.rasters_equal(f.raster(), l.raster())
    assert np.array_equal(f.weights(), l.weights())


def test_rstdp_consolidation_homeostasis_reference_engine(oracle_lib):
    # reference defaults (direct current mode, reference drive, STDP and
    # homeostasis) plus R-STDP and consolidation; outputs drive the reward
    net, cfg, drive = nets.lif_reference_default(n=300)
    net.is_output = (np.arange(net.n) < 60).astype(np.uint8)
    cfg.rstdp_enabled = True
    cfg.reward_threshold = 2
    nets.with_consolidation(cfg, tau=200.0, drift=0.05)
    f, l, traj = run_pair(net, cfg, drive, 200, every=True)
    assert np.array_equal(traj[:, 0], traj[:, 1])
    assert np.any(np.abs(traj[:, 0]) > 0.001)
    assert nets.rasters_equal(f.raster(), l.raster())
    # the consolidation frame reassociates the drift: FP64 rounding only
    assert np.allclose(f.weights(), l.weights(), rtol=1e-9, atol=1e-9)
    assert np.allclose(f.eligibility(), l.eligibility(), rtol=1e-9, atol=1e-12)


def test_consolidation_frame_tracks_fp64(oracle_lib):
    # no activity: only consolidation moves the weights. The float frame
    # (w = u*A + B) keeps every weight within 1e-6 of the FP64 per-step drift
    # after 20,000 steps (default rule: a drift of 1e-7 of (target - w) per step)
    net, cfg, drive = nets.izh_stdp(n=400, k=20, wf=A.WEIGHT_F32)
    cfg.stdp_enabled = False
    nets.with_consolidation(cfg)
    f32 = FastOracle(net, cfg, Drive(), precision=32)
    l = LiteralOracle(net, cfg, Drive(), threads=1)
    f32.step(20_000)
    l.step(20_000)
    w0 = net.w.astype(np.float64)
    wl, wf = l.weights(), f32.weights()
    assert len(l.raster()[0]) == 0
    assert np.mean(np.abs(wl - w0)) > 1e-3
    assert np.max(np.abs(wf - wl)) < 1e-6


def test_consolidation_renormalisation(oracle_lib):
    # a = 0.9 per step: the frame renormalises every ~105 steps
    net, cfg, drive = nets.izh_stdp(n=1200, k=40, wf=A.WEIGHT_F32)
    nets.with_consolidation(cfg, tau=10.0, drift=1.0)
    f32 = FastOracle(net, cfg, drive, precision=32)
    l = LiteralOracle(net, cfg, drive, threads=2)
    f32.step(400)
    l.step(400)
    assert nets.rasters_equal(f32.raster(), l.raster())
    assert np.max(np.abs(f32.weights() - l.weights())) < 1e-6


def test_stp_fast_vs_literal(oracle_lib):
    # direct current mode: each delivered weight times the EPSP of one step of
    # a copy of the synapse's STP state
    net, cfg, drive = nets.lif_reference_default(n=300, stdp=False, homeo=False)
    nets.with_stp(net)
    f, l, _ = run_pair(net, cfg, drive, 200)
    ra, rb = f.raster(), l.raster()
    assert len(ra[0]) > 50
    assert nets.rasters_equal(ra, rb)
    assert np.allclose(f.state()["v"], l.state()["v"], rtol=1e-9, atol=1e-9)
    # STP changes the dynamics
    net2, _, _ = nets.lif_reference_default(n=300, stdp=False, homeo=False)
    g = FastOracle(net2, cfg, drive, precision=64)
    g.step(200)
    assert not nets.rasters_equal(g.raster(), ra)


def test_conductance_ref_all_types_fast_vs_literal(oracle_lib):
    # reference conductance mode with AMPA, GABA, GABA-B and NMDA synapses:
    # per-target accumulating conductances equal the per-synapse ones
    net, cfg, drive = nets.lif_conductance_all_types(n=300)
    assert set(np.unique(net.syn_type)) == {0, 1, 2, 3}
    f, l, _ = run_pair(net, cfg, drive, 150)
    ra, rb = f.raster(), l.raster()
    assert len(ra[0]) > 20
    assert nets.rasters_equal(ra, rb)
    assert np.allclose(f.state()["v"], l.state()["v"], rtol=1e-7, atol=1e-6)


def test_conductance_ref_all_types_stdp_homeostasis_fast_vs_literal(oracle_lib):
    # the same mode with STDP and homeostasis: contributions use w*gmax*mg(V)
    net, cfg, drive = nets.lif_conductance_all_types(n=300)
    cfg.stdp_enabled = True
    cfg.homeostasis_enabled = True
    f, l, _ = run_pair(net, cfg, drive, 120)
    ra, rb = f.raster(), l.raster()
    assert len(ra[0]) > 20
    assert nets.rasters_equal(ra, rb)
    assert np.allclose(f.weights(), l.weights(), rtol=1e-9, atol=1e-9)
    assert np.count_nonzero(f.weights() != net.w.astype(np.float64)) > 50


@pytest.mark.parametrize("which", ["default", "all_types"])
def test_lfp_fast_vs_literal(oracle_lib, which):
    # lfp_signal (engine.rs:492): the reference sums |g (E_rev - V)| per
    # synapse after each step's delivery; the reformulated engine sums per
    # neuron and type at the next update, then adds the last step's term.
    # Per-type sums equal per-synapse sums while each type's conductances
    # share one sign (excitatory weights > 0; GABA types take |w|).
    if which == "default":
        net, cfg, drive = nets.lif_reference_default(n=300, stdp=False, homeo=False, conductance=True)
    else:
        net, cfg, drive = nets.lif_conductance_all_types(n=300)
    f = FastOracle(net, cfg, drive, precision=64)
    l = LiteralOracle(net, cfg, drive, threads=2)
    done = 0
    for k in (1, 9, 40, 100):
        f.step(k - done)
        l.step(k - done)
        done = k
        ref = l.stats()["lfp"]
        assert f.lfp() == pytest.approx(ref, rel=1e-12, abs=1e-9)
    assert ref > 1e6
    # reading it consumes nothing
    assert f.lfp() == f.lfp()


def test_lfp_zero_outside_reference_conductance_mode(oracle_lib):
    net, cfg, drive = nets.lif_reference_default(n=300, stdp=False, homeo=False)
    f = FastOracle(net, cfg, drive, precision=32)
    f.step(50)
    assert f.lfp() == 0.0


def test_reward_sum_is_sum_of_rewards(oracle_lib):
    net, cfg, drive = nets.izh_rstdp(n=1500, k=40)
    f = FastOracle(net, cfg, drive, precision=64)
    acc = 0.0
    for _ in range(80):
        f.step(1)
        acc += f.reward()[0]
    assert f.reward()[1] == pytest.approx(acc, rel=1e-12)
