"""CPU: the fast oracle (per-neuron traces, per-target conductances) against
the literal restatement of engine.rs (per-synapse state, O(M) loops), and the
float engine against FP64."""
import numpy as np
import pytest

from oracle.oracle import FastOracle, LiteralOracle
from neuralsim_b200 import _abi as A
import nets


def run_pair(net, cfg, drive, steps, prec=64):
    f = FastOracle(net, cfg, drive, precision=prec)
    l = LiteralOracle(net, cfg, drive, threads=2)
    f.step(steps)
    l.step(steps)
    return f, l


def test_lif_delta_delay_fast_equals_literal(oracle_lib):
    net, cfg, drive = nets.lif_delta(n=1500, k=40)
    f, l = run_pair(net, cfg, drive, 600)
    ra, rb = f.raster(), l.raster()
    assert len(ra[0]) > 100
    assert nets.rasters_equal(ra, rb)
    assert np.array_equal(f.state()["v"], l.state()["v"])
    assert f.events() == l.events()


@pytest.mark.parametrize("wf", [A.WEIGHT_F32])
def test_izh_stdp_fast_equals_literal(oracle_lib, wf):
    net, cfg, drive = nets.izh_stdp(n=1500, k=40, wf=wf)
    f, l = run_pair(net, cfg, drive, 300)
    ra, rb = f.raster(), l.raster()
    assert len(ra[0]) > 200
    assert nets.rasters_equal(ra, rb)
    wf_, wl = f.weights(), l.weights()
    assert np.array_equal(wf_, wl)
    sf, sl = f.state(), l.state()
    assert np.array_equal(sf["v"], sl["v"]) and np.array_equal(sf["u"], sl["u"])
    # STDP moved weights
    assert np.count_nonzero(wf_ != net.w.astype(np.float64)) > 100


def test_reference_default_engine_fast_vs_literal(oracle_lib):
    # direct current mode with 0.92 decay, reference drive, STDP + homeostasis:
    # same spikes over a short horizon, weights within FP reassociation
    net, cfg, drive = nets.lif_reference_default(n=300)
    f, l = run_pair(net, cfg, drive, 200)
    ra, rb = f.raster(), l.raster()
    assert len(ra[0]) > 50
    assert nets.rasters_equal(ra, rb)
    assert np.allclose(f.weights(), l.weights(), rtol=1e-9, atol=1e-9)
    assert np.allclose(f.rates(), l.rates(), rtol=1e-12, atol=1e-12)
    assert np.allclose(f.state()["v"], l.state()["v"], rtol=1e-9, atol=1e-9)


def test_reference_conductance_mode_fast_vs_literal(oracle_lib):
    net, cfg, drive = nets.lif_reference_default(n=300, stdp=False, homeo=False, conductance=True)
    f, l = run_pair(net, cfg, drive, 150)
    ra, rb = f.raster(), l.raster()
    assert len(ra[0]) > 20
    assert nets.rasters_equal(ra, rb)
    assert np.allclose(f.state()["v"], l.state()["v"], rtol=1e-7, atol=1e-6)


def test_hh_conductance_fresh_fast_vs_literal(oracle_lib):
    net, cfg, drive = nets.hh_cond(n=400, k=40)
    f, l = run_pair(net, cfg, drive, 1500)
    ra, rb = f.raster(), l.raster()
    assert nets.rasters_equal(ra, rb)
    sf, sl = f.state(), l.state()
    for key in ("v", "m", "h", "n"):
        assert np.allclose(sf[key], sl[key], rtol=1e-9, atol=1e-9), key


# Per-step tolerance: |float - fp64| <= 1e-5 * max(|fp64|, floor), floor 10 mV
# for membrane voltages (a crossing near 0 mV cancels two ~30 mV operands)
# and 1 for u and the gates.
FLOOR = {"v": 10.0, "u": 1.0, "m": 1.0, "h": 1.0, "n": 1.0}


def one_step_error(net, cfg, drive, keys):
    f32 = FastOracle(net, cfg, drive, precision=32)
    f64 = FastOracle(net, cfg, drive, precision=64)
    f32.step(1)
    f64.step(1)
    a, b = f32.state(), f64.state()
    return {k: (np.abs(a[k] - b[k]) / np.maximum(np.abs(b[k]), FLOOR[k])).max() for k in keys}


def test_float_engine_one_step_within_1e5_of_fp64_izh(oracle_lib):
    # per-step state from identical, widely spread states (v in [-80, 29],
    # u in [-20, 10]) with the Gaussian drive: float within 1e-5 relative
    net, cfg, drive = nets.izh_stdp(n=4000, k=20, wf=A.WEIGHT_F32)
    rng = np.random.default_rng(3)
    net.v0 = rng.uniform(-80, 29, net.n).astype(np.float32)
    net.u0 = rng.uniform(-20, 10, net.n).astype(np.float32)
    err = one_step_error(net, cfg, drive, ("v", "u"))
    assert max(err.values()) < 1e-5, err


def test_float_engine_one_step_within_1e5_of_fp64_hh(oracle_lib):
    net, cfg, drive = nets.hh_cond(n=2000, k=20)
    rng = np.random.default_rng(4)
    net.v0 = rng.uniform(-80, 30, net.n).astype(np.float32)
    net.m0 = rng.uniform(0, 1, net.n).astype(np.float32)
    net.h0 = rng.uniform(0, 1, net.n).astype(np.float32)
    net.n0 = rng.uniform(0, 1, net.n).astype(np.float32)
    err = one_step_error(net, cfg, drive, ("v", "m", "h", "n"))
    assert max(err.values()) < 1e-5, err


def test_float_engine_close_to_fp64_over_lif_horizon(oracle_lib):
    # LIF is contracting: the float engine stays within 1e-5 of FP64 over
    # 500 steps as long as the spike trains agree
    net, cfg, drive = nets.lif_delta(n=1000, k=30)
    f32 = FastOracle(net, cfg, drive, precision=32)
    f64 = FastOracle(net, cfg, drive, precision=64)
    f32.step(500)
    f64.step(500)
    assert nets.rasters_equal(f32.raster(), f64.raster())
    a, b = f32.state()["v"], f64.state()["v"]
    assert (np.abs(a - b) / np.maximum(np.abs(b), FLOOR["v"])).max() < 1e-5
