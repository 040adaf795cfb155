"""Host stimulus (SimulationEngine::stimulate, src/simulation/engine.rs:156-161):
amounts added to neurons' input current between steps. CPU: the reformulated
oracle against the literal engine, which applies it as the reference does.
GPU (marked): the device against the float oracle, bit for bit, on the step
path and the windowed path, plus the argument checks."""
import numpy as np
import pytest

from oracle.oracle import FastOracle, LiteralOracle
from neuralsim_b200 import SimulationEngine, NsError
from neuralsim_b200 import _abi as A
import nets

# (steps before, ids, amounts) rounds; then 40 more steps
ROUNDS = [
    (20, [3, 7, 7, 100, 250], [20.0, 15.0, 5.0, 30.0, -12.5]),
    (30, list(range(40, 140, 2)), [25.0]),
    (10, [0, 0, 0], [4.0, 4.0, 4.0]),
]


def make(which):
    if which == "ref_current":
        return nets.lif_reference_default(n=300)
    if which == "ref_conductance":
        return nets.lif_reference_default(n=300, stdp=False, homeo=False, conductance=True)
    if which == "izh_reset":
        net, cfg, drive = nets.izh_stdp(n=1500, k=40, wf=A.WEIGHT_F32)
        return net, cfg, drive
    if which == "lif_delta_windowed":
        return nets.lif_delta(n=3000, k=40)
    raise ValueError(which)


def drive_rounds(engines, n):
    for steps, ids, amt in ROUNDS:
        for e in engines:
            (e.run if hasattr(e, "run") else e.step)(steps)
        ids = [i % n for i in ids]
        for e in engines:
            e.stimulate(ids, amt)
    for e in engines:
        (e.run if hasattr(e, "run") else e.step)(40)


@pytest.mark.parametrize("which", ["ref_current", "ref_conductance", "izh_reset"])
def test_stimulus_fast_vs_literal(oracle_lib, which):
    net, cfg, drive = make(which)
    f = FastOracle(net, cfg, drive, precision=64)
    l = LiteralOracle(net, cfg, drive, threads=2)
    drive_rounds([f, l], net.n)
    ra, rb = f.raster(), l.raster()
    assert nets.rasters_equal(ra, rb)
    assert np.allclose(f.state()["v"], l.state()["v"], rtol=1e-7, atol=1e-6)
    # the stimulus changes the run (the conductance network fires at its
    # refractory limit, so there only the state shows it)
    g = FastOracle(net, cfg, drive, precision=64)
    g.step(sum(r[0] for r in ROUNDS) + 40)
    sg, sf = g.state(), f.state()
    assert not nets.rasters_equal(g.raster(), ra) or any(
        not np.array_equal(sg[k], sf[k]) for k in sf if isinstance(sf[k], np.ndarray))


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["ref_current", "ref_conductance", "izh_reset",
                                   "lif_delta_windowed"])
def test_stimulus_matches_oracle(lib, which):
    net, cfg, drive = make(which)
    eng = SimulationEngine(net, cfg, drive)
    o = FastOracle(net, cfg, drive, precision=32)
    drive_rounds([eng, o], net.n)
    steps = sum(r[0] for r in ROUNDS) + 40
    ra, rb = eng.read_raster(0, steps), o.raster()
    assert len(rb[0]) > 20
    assert nets.rasters_equal(ra, rb)
    st, so = eng.download_state(), o.state()
    assert np.array_equal(st["v"].astype(np.float64), so["v"])
    if which == "lif_delta_windowed":
        assert eng.window()[0] > 1   # the windowed path ran
    eng.close()


@pytest.mark.gpu
def test_stimulus_arguments(lib):
    net, cfg, drive = nets.lif_reference_default(n=300)
    eng = SimulationEngine(net, cfg, drive)
    with pytest.raises(NsError):
        eng.stimulate([300], [1.0])
    with pytest.raises(NsError):
        eng.stimulate([1], [float("nan")])
    with pytest.raises(NsError):
        eng.stimulate([1], [1e300])   # not finite in float
    # a refused call leaves nothing pending: the run equals an unstimulated one
    eng.run(50)
    ref = SimulationEngine(net, cfg, drive)
    ref.run(50)
    assert nets.rasters_equal(eng.read_raster(0, 50), ref.read_raster(0, 50))


# Firing-rate estimate without homeostasis (SimulationEngine::firing_rate /
# mean_firing_rate, engine.rs:637-645, :809-826): kept when track_rates is on.

def rate_net():
    net, cfg, drive = nets.lif_reference_default(n=300, stdp=True, homeo=False)
    cfg.track_rates = 1
    return net, cfg, drive


def test_tracked_rates_fast_vs_literal(oracle_lib):
    net, cfg, drive = rate_net()
    f = FastOracle(net, cfg, drive, precision=64)
    l = LiteralOracle(net, cfg, drive, threads=2)
    f.step(120)
    l.step(120)
    assert nets.rasters_equal(f.raster(), l.raster())
    assert np.allclose(f.rates(), l.rates(), rtol=1e-12, atol=1e-12)
    assert f.rates().max() > 0
    cfg.track_rates = 0
    g = FastOracle(net, cfg, drive, precision=64)
    g.step(10)
    assert not g.rates().any()


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["ref_current", "lif_delta"])
def test_tracked_rates_match_oracle(lib, which):
    if which == "ref_current":
        net, cfg, drive = rate_net()
    else:
        net, cfg, drive = nets.lif_delta(n=3000, k=40)   # windowed unless tracking
        cfg.track_rates = 1
    eng = SimulationEngine(net, cfg, drive)
    eng.run(150)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(150)
    assert nets.rasters_equal(eng.read_raster(0, 150), o.raster())
    r = eng.rates()
    assert np.array_equal(r, o.rates())
    assert r.max() > 0
    assert eng.mean_firing_rate() == pytest.approx(r.mean(), rel=1e-15)
    assert eng.firing_rate(5) == r[5] and eng.firing_rate(net.n) == 0.0
    assert eng.window()[0] <= 1   # tracking runs the step path


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["lif_delta_windowed", "hh_windowed"])
def test_windowed_counters_without_log(lib, which):
    # with the spike log off the window skips its segment scan: the step
    # statistics equal those of the logged run
    if which == "lif_delta_windowed":
        net, cfg, drive = nets.lif_delta(n=3000, k=40)
    else:
        net, cfg, drive = nets.hh_cond(n=2000, k=40)
        cfg.delay_steps, cfg.window_steps = 10, 0
    n1 = 150 if which == "lif_delta_windowed" else 900
    logged = SimulationEngine(net, cfg, drive)
    a = [logged.run(n1), logged.run(77)]
    cfg.spike_log_capacity = 0
    bare = SimulationEngine(net, cfg, drive)
    b = [bare.run(n1), bare.run(77)]
    assert bare.window()[0] > 1 and logged.window()[0] > 1
    for x, y in zip(a, b):
        for f in ("steps_done", "spikes", "output_spikes", "events", "last_step_spikes",
                  "max_step_spikes"):
            assert getattr(x, f) == getattr(y, f), f
    assert a[0].spikes + a[1].spikes > 0
    assert np.array_equal(logged.download_state()["v"], bare.download_state()["v"])
