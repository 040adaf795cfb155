"""Deferred LTD (step schedule 5) against the oracle's eager STDP order.

The LTD of synapse j->i at a spike of i waits, as a bit in i's 32-step spike
history, until j's row is walked again (j's next spike, before delivery) or
flushed (each row once per 32 steps). The weights, rasters and traces must
equal the eager order of engine.rs:497-537 bit for bit at every point the
host can observe them: after runs of any length, after weight reads in the
middle of a run (which flush every row), across state uploads and traced
(eager) steps, with a mix of plastic and non-plastic synapses in one row, in
the reference conductance mode and in batches. The autotuner's switches
between schedule 5 and the eager ones are covered by
test_gpu_parity.py::test_autotuner_picks_a_schedule.
"""
import copy

import numpy as np
import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200 import SimulationEngine
from neuralsim_b200.batch import BatchEngine
from neuralsim_b200 import configs
from oracle.oracle import FastOracle
import nets

pytestmark = pytest.mark.gpu


def _engine(net, cfg, drive, sched=5):
    c = copy.copy(cfg)
    c.step_schedule = sched
    return SimulationEngine(net, c, drive)


@pytest.mark.parametrize("wf", [A.WEIGHT_BF16, A.WEIGHT_F32])
@pytest.mark.parametrize("chunk", [1000, 37])
def test_deferred_ltd_equals_oracle(lib, wf, chunk):
    # whole graph chunks and eager remainders of odd lengths (37 is prime to
    # the 32-step flush period)
    net, cfg, drive = nets.izh_stdp(n=20_000, k=100, wf=wf)
    cfg.graph_chunk = chunk
    eng = _engine(net, cfg, drive)
    eng.run(1000)
    assert eng.schedule()[0] == 5
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(1000)
    ra, rb = eng.read_raster(0, 1000), o.raster()
    assert len(rb[0]) > 50_000
    assert nets.rasters_equal(ra, rb)
    st, so = eng.download_state(), o.state()
    for k, ok in (("v", "v"), ("u", "u"), ("pre_trace", "pre"), ("post_trace", "post")):
        assert np.array_equal(st[k].astype(np.float64), so[ok]), k
    assert np.array_equal(st["w"].astype(np.float64), o.weights())
    assert np.count_nonzero(st["w"] != net.w) > 10_000


def test_deferred_ltd_reads_mid_run(lib):
    # weight reads (download, stats) flush every row; stepping goes on from
    # there with identical results, and a state upload resumes exactly
    net, cfg, drive = nets.izh_stdp(n=12_000, k=80)
    eng = _engine(net, cfg, drive)
    o = FastOracle(net, cfg, drive, precision=32)
    done = 0
    for n_steps in (1, 5, 31, 32, 33, 64, 100):
        eng.run(n_steps)
        o.step(n_steps)
        done += n_steps
        w = eng.download_state()["w"].astype(np.float64)
        assert np.array_equal(w, o.weights()), done
        mu, sd = eng.weight_stats()
        assert mu == pytest.approx(o.weights().mean(), rel=1e-9)
    st = eng.download_state()
    eng2 = _engine(net, cfg, drive)
    eng2.upload_state(st, done)
    eng.run(150)
    eng2.run(150)
    o.step(150)
    for e in (eng, eng2):
        assert np.array_equal(e.download_state()["w"].astype(np.float64), o.weights())
    assert nets.rasters_equal(eng2.read_raster(done, 150),
                              (lambda r: (r[0][r[1][done]:], r[1][done:] - r[1][done]))(o.raster()))


def test_deferred_ltd_with_a_traced_step_between(lib):
    # an eager traced step (every row flushed first, the trace starts taken
    # again after it) between deferred steps in graph chunks of 50
    net, cfg, drive = nets.izh_stdp(n=10_000, k=60)
    cfg.graph_chunk = 50
    eng = _engine(net, cfg, drive)
    o = FastOracle(net, cfg, drive, precision=32)
    eng.run(70)
    o.step(70)
    _, ne = eng.step_traced(0)
    o.step(1)
    eng.run(45)
    o.step(45)
    assert np.array_equal(eng.download_state()["w"].astype(np.float64), o.weights())
    assert nets.rasters_equal(eng.read_raster(0, 116), o.raster())


def test_deferred_ltd_mixed_rows(lib):
    # per-synapse plastic flags inside rows (half of each excitatory row)
    net, cfg, drive = nets.izh_stdp(n=8000, k=50, wf=A.WEIGHT_F32)
    rng = np.random.default_rng(5)
    net.plastic = (net.plastic & (rng.random(net.m) < 0.5)).astype(np.uint8)
    eng = _engine(net, cfg, drive)
    eng.run(600)
    assert eng.schedule()[0] == 5
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(600)
    assert nets.rasters_equal(eng.read_raster(0, 600), o.raster())
    assert np.array_equal(eng.download_state()["w"].astype(np.float64), o.weights())


def test_deferred_ltd_conductance_mode_equals_eager(lib):
    # the reference conductance mode with STDP and no homeostasis: the device
    # evaluates per-synapse conductances with expf, so the comparison that is
    # bit for bit is deferred against eager (schedule 3) on the device
    net, cfg, drive = nets.lif_reference_default(n=1500, homeo=False, conductance=True)
    runs = []
    for sched in (5, 3):
        eng = _engine(net, cfg, drive, sched)
        eng.run(400)
        assert eng.schedule()[0] == sched
        runs.append((eng.read_raster(0, 400), eng.download_state()))
        eng.close()
    (ra, sa), (rb, sb) = runs
    assert len(ra[0]) > 1000
    assert nets.rasters_equal(ra, rb)
    for k in ("w", "v", "pre_trace", "post_trace"):
        assert np.array_equal(sa[k], sb[k]), k


def test_deferred_ltd_batch_equals_oracle(lib):
    # a batch of Izhikevich + STDP networks of odd sizes under schedule 5
    nets_, seeds = [], []
    for q, n in enumerate((2001, 3333, 1500)):
        net, cfg, drive = nets.izh_stdp(n=n, k=40, seed=300 + q)
        nets_.append(net)
        seeds.append(9000 + q)
    cfg = copy.copy(cfg)
    cfg.step_schedule = 5
    b = BatchEngine(nets_, seeds, cfg, drive)
    b.run(300)
    parts = b.read_rasters(0, 300)
    st = b.download_state()
    m0 = 0
    for q, net in enumerate(nets_):
        c = copy.copy(cfg)
        c.seed = seeds[q]
        o = FastOracle(net, c, drive, precision=32)
        o.step(300)
        assert nets.rasters_equal(parts[q], o.raster()), q
        assert np.array_equal(st["w"][m0:m0 + net.m].astype(np.float64), o.weights()), q
        m0 += net.m
    b.close()


def test_deferred_schedule_falls_back_where_it_does_not_apply(lib):
    # homeostasis rescales weights every step: schedule 5 runs the fused
    # eager schedule, with the oracle's results
    net, cfg, drive = nets.lif_reference_default(n=400)
    eng = _engine(net, cfg, drive)
    eng.run(100)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(100)
    assert nets.rasters_equal(eng.read_raster(0, 100), o.raster())
    assert np.allclose(eng.download_state()["w"], o.weights(), rtol=1e-5, atol=1e-6)


def test_state_read_without_weights_leaves_ltds_pending(lib):
    # a read of the neuron state alone does not flush the pending LTDs; the
    # state it returns and everything after it equal the oracle
    net, cfg, drive = nets.izh_stdp(n=12_000, k=80)
    eng = _engine(net, cfg, drive)
    o = FastOracle(net, cfg, drive, precision=32)
    eng.run(45)
    o.step(45)
    st = eng.download_state(with_weights=False, fields=("v", "u", "pre_trace", "post_trace"))
    so = o.state()
    for k, ok in (("v", "v"), ("u", "u"), ("pre_trace", "pre"), ("post_trace", "post")):
        assert np.array_equal(st[k].astype(np.float64), so[ok]), k
    assert set(st) == {"v", "u", "pre_trace", "post_trace"}
    eng.run(45)
    o.step(45)
    assert np.array_equal(eng.download_state()["w"].astype(np.float64), o.weights())
    assert nets.rasters_equal(eng.read_raster(0, 90), o.raster())

