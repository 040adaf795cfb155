"""Golden fixtures (tests/golden/*.npz, written by make_golden.py).

CPU: the network generator still produces the fixture's network (digest) and
the oracle still produces the fixture's raster and state, bit for bit.
GPU: the CUDA path reproduces the fixtures: bit-exact for LIF and
Izhikevich (rasters, state, weights; eligibility and reward for R-STDP,
weights through the consolidation frame, STP-scaled input); the reference-default engine with
homeostasis has equal rasters and weights within 1e-5; for Hodgkin-Huxley (FP64 fixture,
float device) every spike matched within 0.05 ms and the final V within
1e-2 of max(|V|, 10 mV).
"""
import os

import numpy as np
import pytest

import nets
from golden.make_golden import CASES, advance, net_digest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = sorted(CASES)


def fixture(name):
    return dict(np.load(os.path.join(HERE, name + ".npz")))


@pytest.mark.parametrize("name", NAMES)
def test_generator_matches_fixture_network(lib, name):
    net, _, _ = CASES[name][0]()
    assert net_digest(net) == str(fixture(name)["net_sha256"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(lib, oracle_lib, name):
    from golden.make_golden import run_case
    got, want = run_case(name), fixture(name)
    for k in want:
        assert np.array_equal(np.asarray(got[k]), want[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_reproduces_fixture(lib, name):
    from neuralsim_b200 import SimulationEngine
    build, steps, prec = CASES[name][:3]
    net, cfg, drive = build()
    f = fixture(name)
    eng = SimulationEngine(net, cfg, drive)
    advance(eng, CASES[name])
    raster = eng.read_raster(0, steps)
    st = eng.download_state()
    if name.startswith("lif_reference_default"):
        # homeostatic scaling multiplies every weight by a per-step factor:
        # rasters equal, weights and V within 1e-5 relative
        assert nets.rasters_equal(raster, (f["idx"], f["off"]))
        assert np.allclose(st["w"], f["weights"], rtol=1e-5, atol=1e-6)
        assert np.allclose(st["v"], f["v"], rtol=1e-5, atol=1e-4)
    elif prec == 32:
        assert nets.rasters_equal(raster, (f["idx"], f["off"]))
        assert np.array_equal(st["v"].astype(np.float64), f["v"])
        assert np.array_equal(st["w"].astype(np.float32), f["weights"])
        if "u" in f and name.startswith("izh"):
            assert np.array_equal(st["u"].astype(np.float64), f["u"])
        if "lfp" in f:
            assert eng.lfp() == f["lfp"]
        if "rates" in f:
            assert np.array_equal(eng.rates(), f["rates"])
        if "elig" in f:
            assert np.array_equal(eng.eligibility(), f["elig"])
            r, rs = eng.reward()
            assert r == f["reward"][0] and rs == pytest.approx(f["reward"][1], rel=1e-12)
    else:
        dt_steps = int(round(0.05 / cfg.dt_ms))
        d, ua, ub = nets.match_spikes((f["idx"], f["off"]), raster, dt_steps)
        assert ua == 0 and ub == 0 and len(d) == len(f["idx"])
        err = np.abs(st["v"] - f["v"]) / np.maximum(np.abs(f["v"]), 10.0)
        assert err.max() < 1e-2
    eng.close()
