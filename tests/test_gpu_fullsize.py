"""Parity of the benchmark configurations at their full sizes.

The networks the bench times, stepped on the GPU and by the oracle from the
same seeds (the reference's loop is src/simulation/engine.rs:254-680):

- Izhikevich + pair STDP at 1M neurons / 100M BF16 synapses, 100 steps:
  raster, V, u, traces and every weight bit-exact against the float oracle.
- Hodgkin-Huxley at 100k neurons / 10M synapses, Rush-Larsen at dt 0.01 ms,
  10 ms (1000 steps): spike trains against the FP64 oracle, spike by spike,
  and the state within the tolerance stated in the test.
- The 256-network LIF batch (3.9M neurons, 4.8e8 synapses), 1000 steps:
  eight sampled networks (the smallest, the largest and six drawn at random)
  against their stand-alone float-oracle runs, bit for bit, under the
  configuration's drive and under the active drive variant the bench also
  times.
- The learned HH macro-step (C5) on the C4 network: spike times against the
  plain Rush-Larsen run within the tolerance stated in the test.
"""
import copy

import numpy as np
import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200 import configs, SimulationEngine
from neuralsim_b200.batch import BatchEngine
from neuralsim_b200.engine import Drive
from oracle.oracle import FastOracle
import nets

pytestmark = pytest.mark.gpu


def test_c2_full_size_bit_exact_vs_float_oracle(lib):
    net, cfg, drive, _ = configs.izh_c2()
    assert net.n == 1_000_000 and net.m == 100_000_000
    assert cfg.weight_format == A.WEIGHT_BF16
    steps = 100
    cfg.spike_log_capacity, cfg.spike_log_steps = 60_000_000, steps
    eng = SimulationEngine(net, cfg, drive)
    eng.run(steps)
    ra = eng.read_raster(0, steps)
    st = eng.download_state()
    eng.close()
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(steps)
    rb = o.raster()
    assert len(rb[0]) > 100_000
    assert nets.rasters_equal(ra, rb)
    so = o.state()
    for k, ok in (("v", "v"), ("u", "u"), ("pre_trace", "pre"), ("post_trace", "post")):
        assert np.array_equal(st[k].astype(np.float64), so[ok]), k
    w = st["w"].astype(np.float64)
    assert np.array_equal(w, o.weights())
    # STDP moved a large share of the weights
    assert np.count_nonzero(w != np.asarray(net.w, np.float64)) > 1_000_000


def test_c4_full_size_tracks_fp64_oracle(lib):
    # 100k HH neurons, 10M conductance synapses, Rush-Larsen dt 0.01 ms. The
    # device evaluates the rate functions with the hardware exponential, so
    # the comparison is with the FP64 oracle under a tolerance: every spike
    # within 0.05 ms (5 steps) of an FP64 spike, at most 0.1 % of the spikes
    # on either side without a partner, and the state within 1e-2 of
    # max(|x|, floor) for 99.9 % of the neurons (the rest are on a spike's
    # upstroke, where a 5 us shift moves V by tens of mV).
    net, cfg, drive, _ = configs.hh_c4()
    assert net.n == 100_000 and net.m == 10_000_000
    steps = 1000
    cfg.spike_log_capacity, cfg.spike_log_steps = 20_000_000, steps
    eng = SimulationEngine(net, cfg, drive)
    eng.run(steps)
    ra = eng.read_raster(0, steps)
    st = eng.download_state()
    eng.close()
    o = FastOracle(net, cfg, drive, precision=64)
    o.step(steps)
    rb = o.raster()
    n_spk = len(rb[0])
    assert n_spk > 10_000
    d, ua, ub = nets.match_spikes(rb, ra, 5)
    assert ua <= 0.001 * n_spk and ub <= 0.001 * n_spk, (ua, ub, n_spk)
    assert len(d) >= 0.999 * n_spk
    so = o.state()
    floor = {"v": 10.0, "hh_m": 1.0, "hh_h": 1.0, "hh_n": 1.0}
    okey = {"v": "v", "hh_m": "m", "hh_h": "h", "hh_n": "n"}
    for k in ("v", "hh_m", "hh_h", "hh_n"):
        err = np.abs(st[k] - so[okey[k]]) / np.maximum(np.abs(so[okey[k]]), floor[k])
        assert np.quantile(err, 0.999) < 1e-2, (k, np.quantile(err, 0.999))


def _sample(nets_, rng):
    sizes = np.array([x.n for x in nets_])
    pick = {int(np.argmin(sizes)), int(np.argmax(sizes))}
    rest = [q for q in range(len(nets_)) if q not in pick]
    pick.update(int(q) for q in rng.choice(rest, 6, replace=False))
    return sorted(pick)


@pytest.mark.parametrize("variant", ["config_drive", "active_drive"])
def test_c3_full_batch_sampled_networks_bit_exact(lib, variant):
    nets_, seeds, cfg, drive, steps = configs.lif_batch_c3()
    assert len(nets_) == 256
    if variant == "active_drive":
        drive = Drive(A.DRIVE_POISSON_KICK, p=0.02, amplitude=4.0)
    cfg.spike_log_capacity, cfg.spike_log_steps = 400_000_000, steps
    b = BatchEngine(nets_, seeds, cfg, drive)
    b.run(steps)
    parts = b.read_rasters(0, steps)
    st = b.download_state()
    vs = b.split(st["v"])
    rs = b.split(st["refractory"])
    b.close()
    pick = _sample(nets_, np.random.default_rng(2024))
    assert len(pick) == 8
    spikes = 0
    for q in pick:
        c = copy.copy(cfg)
        c.seed = seeds[q]
        o = FastOracle(nets_[q], c, drive, precision=32)
        o.step(steps)
        assert nets.rasters_equal(parts[q], o.raster()), q
        so = o.state()
        assert np.array_equal(vs[q].astype(np.float64), so["v"]), q
        assert np.array_equal(rs[q], so["refr"]), q
        spikes += len(parts[q][0])
    if variant == "active_drive":
        assert spikes > 10_000


def test_c5_full_size_surrogate_spike_times(lib):
    # The learned HH macro-step on the C4 network itself (100k neurons, 10M
    # synapses, dt 0.01 ms), trained as the bench trains it (states of the
    # plain run, 12k Adam steps of 8192). Over 50 ms from the same start the
    # surrogate's spikes are matched to the plain Rush-Larsen run's within
    # 2 ms. Training is not bit-reproducible (split-K atomic gradient sums);
    # its spike-time error measured 0.09-0.19 ms against the 0.2 ms target,
    # so the test asserts 0.25 ms, at most half the error of one Rush-Larsen
    # step of 0.1 ms in the same macro-step scheme, and at most 3 % of the
    # spikes unmatched.
    from neuralsim_b200 import surrogate as S
    net, cfg, drive, _ = configs.hh_c4()
    assert net.n == 100_000 and net.m == 10_000_000
    cfg.window_steps = 100
    steps = 5000
    # training steps the plain run first (2000 warm-up steps, 100 snapshots
    # 50 steps apart) under the same configuration: the log holds them too
    cfg.spike_log_capacity, cfg.spike_log_steps = 50_000_000, 20_000
    sur, x, y, losses = S.train_for_network(net, cfg, drive, warm_steps=2000, snapshots=100,
                                            every_steps=50, batch=8192, steps=12000)
    res = {}
    for mode in ("plain", "surrogate", "coarse"):
        eng = SimulationEngine(net, cfg, drive)
        if mode != "plain":
            eng.attach_surrogate(sur)
            if mode == "coarse":
                eng.macro_step_mode(1)
        eng.run(steps)
        res[mode] = eng.read_raster(0, steps)
        if mode == "surrogate":
            by_mlp, by_fb = eng.surrogate_counts()
        eng.close()
    sur.close()
    w = int(round(2.0 / cfg.dt_ms))
    ds, ua, ub = nets.match_spikes(res["plain"], res["surrogate"], w)
    dc, _, _ = nets.match_spikes(res["plain"], res["coarse"], w)
    n_plain = len(res["plain"][0])
    assert n_plain > 50_000
    err_s = ds.mean() * cfg.dt_ms
    err_c = dc.mean() * cfg.dt_ms
    assert by_mlp > 0.5 * (by_mlp + by_fb)          # most macro-steps by the MLP
    assert err_s <= 0.25, err_s
    assert err_s <= 0.5 * err_c, (err_s, err_c)
    assert ua <= 0.03 * n_plain and ub <= 0.03 * n_plain, (ua, ub, n_plain)
