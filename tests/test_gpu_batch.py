"""Batches of independent networks (ns_upload_batch): every network's raster,
state and weights in the batch equal those of the same network run alone
with its own seed, bit for bit, on the windowed path and the step path, and
for the Gaussian (pair-drawn) drive with odd network sizes."""
import copy

import numpy as np
import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200 import configs, SimulationEngine, NsError
from neuralsim_b200.batch import BatchEngine
from neuralsim_b200.engine import Drive
from oracle.oracle import FastOracle
import nets as tnets

pytestmark = pytest.mark.gpu


def lif_batch(n_nets=7, window=0):
    nets, seeds, cfg, _, _ = configs.lif_batch_c3(n_nets=n_nets, size_range=(300, 3000),
                                                  k_range=(20, 80))
    drive = Drive(A.DRIVE_POISSON_KICK, p=0.02, amplitude=4.0)
    cfg.spike_log_capacity, cfg.spike_log_steps = 20_000_000, 5000
    cfg.window_steps = window
    return nets, seeds, cfg, drive


def alone(net, seed, cfg, drive, steps):
    c = copy.copy(cfg)
    c.seed = seed
    e = SimulationEngine(net, c, drive)
    e.run(steps)
    r = e.read_raster(0, steps), e.download_state()
    e.close()
    return r


@pytest.mark.parametrize("window", [0, 1])
def test_lif_batch_equals_networks_alone(lib, window):
    nets, seeds, cfg, drive = lif_batch(window=window)
    assert any(x.n % 2 for x in nets)
    steps = 600
    b = BatchEngine(nets, seeds, cfg, drive)
    b.run(steps)
    parts = b.read_rasters(0, steps)
    st = b.download_state()
    vs = b.split(st["v"])
    total = 0
    for q, net in enumerate(nets):
        (ra, sa) = alone(net, seeds[q], cfg, drive, steps)
        assert tnets.rasters_equal(parts[q], ra), q
        assert np.array_equal(vs[q], sa["v"])
        total += len(ra[0])
    assert total > 1000
    # and against the oracle for one network
    c = copy.copy(cfg)
    c.seed = seeds[2]
    o = FastOracle(nets[2], c, drive, precision=32)
    o.step(steps)
    assert tnets.rasters_equal(parts[2], o.raster())
    b.close()


@pytest.mark.parametrize("window", [0, 1])
def test_batch_stimulus_equals_network_alone(lib, window):
    # a stimulus given to one network of the batch (by local index) acts as
    # on that network alone; the others are untouched
    nets, seeds, cfg, drive = lif_batch(n_nets=5, window=window)
    ids, amt = [1, 5, 5, 17], [2000.0, 800.0, 800.0, -500.0]   # ~10 mV for neuron 1
    b = BatchEngine(nets, seeds, cfg, drive)
    b.run(100)
    b.stimulate_network(3, ids, amt)
    b.run(200)
    parts = b.read_rasters(0, 300)
    for q, net in enumerate(nets):
        c = copy.copy(cfg)
        c.seed = seeds[q]
        e = SimulationEngine(net, c, drive)
        e.run(100)
        if q == 3:
            e.stimulate(ids, amt)
        e.run(200)
        assert tnets.rasters_equal(parts[q], e.read_raster(0, 300)), q
        e.close()
    c = copy.copy(cfg)
    c.seed = seeds[3]
    plain = alone(nets[3], seeds[3], cfg, drive, 300)[0]
    assert not tnets.rasters_equal(parts[3], plain)   # the stimulus acted
    with pytest.raises(ValueError):
        b.stimulate_network(0, [nets[0].n], [1.0])
    b.close()


def test_izh_stdp_gauss_batch_equals_networks_alone(lib):
    # Gaussian drive pairs neurons (2i, 2i+1): odd sizes make pairs straddle
    # networks in the concatenation; STDP weights stay inside each block
    nets, seeds = [], []
    for q, n in enumerate((501, 777, 1203)):
        net, cfg, drive = tnets.izh_stdp(n=n, k=40, seed=300 + q)
        nets.append(net)
        seeds.append(9000 + q)
    steps = 400
    b = BatchEngine(nets, seeds, cfg, drive)
    b.run(steps)
    parts = b.read_rasters(0, steps)
    st = b.download_state()
    m0 = 0
    for q, net in enumerate(nets):
        ra, sa = alone(net, seeds[q], cfg, drive, steps)
        assert tnets.rasters_equal(parts[q], ra), q
        assert np.array_equal(st["w"][m0:m0 + net.m], sa["w"])
        m0 += net.m
    b.close()


def test_batch_reupload_and_rejections(lib):
    nets, seeds, cfg, drive = lif_batch(n_nets=4)
    b = BatchEngine(nets, seeds, cfg, drive)
    b.run(100)
    r1 = b.read_rasters(0, 100)
    # the same batch again: same buffers, the run restarts from step 0
    b._upload(None)
    b.run(100)
    r2 = b.read_rasters(0, 100)
    for x, y in zip(r1, r2):
        assert tnets.rasters_equal(x, y)
    # reference-uniform drive: global kicks are per network, not per batch
    b.set_drive(Drive.reference_default())
    with pytest.raises(NsError):
        b.run(1)
    b.close()


def test_c3_full_size_batch_runs(lib):
    nets, seeds, cfg, drive, steps = configs.lif_batch_c3()
    n = sum(x.n for x in nets)
    m = sum(x.m for x in nets)
    assert 2.5e6 < n < 5.5e6 and 3e8 < m < 7e8
    b = BatchEngine(nets, seeds, cfg, drive)
    out = b.run(steps)
    assert out.steps_done == steps
    b.close()


def _rates_from_raster(raster, n, steps, dt):
    # the reference's per-neuron estimate (engine.rs:637-645) from rate 0,
    # averaged over the network
    idx, off = raster
    cnt = np.diff(np.asarray(off, np.int64))
    a = dt / 100.0
    r = 0.0
    for s in range(steps):
        r = r * (1.0 - a) + 10.0 * cnt[s]
    return r / n


def test_network_rates_and_population_fitness(lib):
    from neuralsim_b200.population import RateHomeostasis, evaluate_batch
    nets, seeds, cfg, drive = lif_batch(n_nets=5)
    steps = 400
    b = BatchEngine(nets, seeds, cfg, drive)
    b.run(steps)
    rates = b.network_rates(0, steps)
    parts = b.read_rasters(0, steps)
    for q, net in enumerate(nets):
        want = _rates_from_raster(parts[q], net.n, steps, cfg.dt_ms)
        assert abs(rates[q] - want) <= 1e-12 * max(1.0, abs(want))
    assert rates.max() > 1.0
    b.close()
    # a lifetime of 400 steps of 0.1 ms: the population evaluation's fitness
    ev = RateHomeostasis(target_rate=20.0, lifetime_ms=steps * cfg.dt_ms)
    fit, r2 = evaluate_batch(nets, seeds, cfg, drive, ev)
    assert np.allclose(r2, rates, rtol=1e-12, atol=0)
    assert np.allclose(fit, ev.fitness(rates), rtol=0, atol=0)
