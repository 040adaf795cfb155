"""Windowed plans on the GPU: every window length and row-walk shape (lanes
per row, blocks per SM) gives the same rasters and state, bit for bit; the
window tuner times the shapes; a plan cached for a network-size bucket is
replayed by the next engine of that bucket without tuning."""
import json

import numpy as np
import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200 import configs, tune
from neuralsim_b200.batch import BatchEngine
from neuralsim_b200.engine import Drive
import nets as tnets

pytestmark = pytest.mark.gpu

STEPS = 400


def _batch():
    nets, seeds, cfg, _, _ = configs.lif_batch_c3(n_nets=9, size_range=(300, 4000), k_range=(20, 150))
    drive = Drive(A.DRIVE_POISSON_KICK, p=0.02, amplitude=4.0)
    cfg.spike_log_capacity, cfg.spike_log_steps = 20_000_000, STEPS
    cfg.window_steps = 0
    return nets, seeds, cfg, drive


def _run(plan=None, cache=None):
    nets, seeds, cfg, drive = _batch()
    b = BatchEngine(nets, seeds, cfg, drive, plan_cache=cache)
    if plan is not None:
        b.set_window_plan(*plan)
    b.run(STEPS)
    out = (b.read_raster(0, STEPS), b.download_state()["v"], b.window_plan(), b.window(), b.walk_shape())
    b.close()
    return out


def test_every_plan_gives_the_same_rasters(lib):
    ra, va, plan, (w, tried), (shape, shape_us) = _run()
    assert len(ra[0]) > 5000
    # the tuner timed the window lengths and then the walk's shapes
    assert set(tried) == {10, 5, 3, 2}
    assert {l for l, _ in shape_us} == {32, 16, 8}
    assert all(t > 0 for t in shape_us.values())
    assert plan["window"] in tried and plan["lanes"] in (8, 16, 32)
    for p in [(10, 32, 0), (10, 16, 0), (10, 8, 0), (5, 8, 2), (3, 16, 1), (2, 32, 3), (7, 8, 0)]:
        rb, vb, pb, (wb, triedb), _ = _run(p)
        assert triedb == {}, p              # a fixed plan is not tuned
        assert pb["window"] == p[0] and pb["lanes"] == p[1], (p, pb)
        if p[2]:
            assert pb["blocks_per_sm"] == p[2]
        assert tnets.rasters_equal(ra, rb), p
        assert np.array_equal(va, vb), p


def test_plan_cache_replays_the_tuned_plan(lib, tmp_path):
    path = tmp_path / "plans.json"
    ra, va, plan_a, (_, tried_a), _ = _run(cache=tune.PlanCache(path))
    assert tried_a
    doc = json.loads(path.read_text())
    assert len(doc["plans"]) == 1
    (key, stored), = doc["plans"].items()
    assert key.startswith(f"model{A.MODEL_LIF}/input{A.INPUT_DELTA_V}/")
    assert {k: stored[k] for k in ("window", "lanes", "blocks_per_sm")} == plan_a
    assert stored["us_per_step"] > 0
    # the next engine of the bucket takes the plan without tuning
    rb, vb, plan_b, (_, tried_b), (_, shape_us_b) = _run(cache=str(path))
    assert tried_b == {} and shape_us_b == {}
    assert plan_b == plan_a
    assert tnets.rasters_equal(ra, rb)
    assert np.array_equal(va, vb)


def test_window_plan_arguments_checked(lib):
    nets, seeds, cfg, drive = _batch()
    b = BatchEngine(nets, seeds, cfg, drive)
    for bad in [(10, 12, 0), (1, 32, 0), (2000, 32, 0)]:
        with pytest.raises(A.NsError):
            b.set_window_plan(*bad)
    # a plan longer than the configuration's window is clamped to it
    b.set_window_plan(50, 16, 0)
    b.run(20)
    assert b.window_plan()["window"] == 10
    # back to the tuner
    b.set_window_plan(0, 0, 0)
    b.run(200)
    assert b.window()[1]
    b.close()
