"""The windowed-plan cache (neuralsim_b200.tune) on the host: bucket keys,
the JSON file's round trip, atomic saves and rejected entries."""
import json
import os

import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200 import tune


def test_bucket_keys_group_similar_sizes():
    k = tune.bucket_key(A.MODEL_LIF, A.INPUT_DELTA_V, A.WEIGHT_BF16, 10, 3_947_039, 476_923_104)
    # the same power-of-two bucket of neurons and of mean out-degree
    assert k == tune.bucket_key(A.MODEL_LIF, A.INPUT_DELTA_V, A.WEIGHT_BF16, 10, 4_100_000, 500_000_000)
    # another neuron bucket, degree bucket, delay, model or weight format
    assert k != tune.bucket_key(A.MODEL_LIF, A.INPUT_DELTA_V, A.WEIGHT_BF16, 10, 1_000_000, 120_000_000)
    assert k != tune.bucket_key(A.MODEL_LIF, A.INPUT_DELTA_V, A.WEIGHT_BF16, 10, 3_947_039, 1_900_000_000)
    assert k != tune.bucket_key(A.MODEL_LIF, A.INPUT_DELTA_V, A.WEIGHT_BF16, 5, 3_947_039, 476_923_104)
    assert k != tune.bucket_key(A.MODEL_HH, A.INPUT_DELTA_V, A.WEIGHT_BF16, 10, 3_947_039, 476_923_104)
    assert k != tune.bucket_key(A.MODEL_LIF, A.INPUT_DELTA_V, A.WEIGHT_F32, 10, 3_947_039, 476_923_104)
    # empty and tiny networks have a key too
    assert tune.bucket_key(A.MODEL_LIF, A.INPUT_DELTA_V, A.WEIGHT_BF16, 10, 0, 0).endswith("/n2^0/deg2^0")


def test_plan_cache_round_trip(tmp_path):
    path = tmp_path / "sub" / "plans.json"
    c = tune.PlanCache(path)
    assert c.get("x") is None
    c.put("x", {"window": 10, "lanes": 16, "blocks_per_sm": 0}, us_per_step=37.5)
    c.put("y", {"window": 5, "lanes": 8, "blocks_per_sm": 3})
    assert os.path.exists(path)
    d = tune.PlanCache(path)
    assert d.get("x") == {"window": 10, "lanes": 16, "blocks_per_sm": 0, "us_per_step": 37.5}
    assert d.get("y") == {"window": 5, "lanes": 8, "blocks_per_sm": 3}
    # no temporary file is left beside it
    assert sorted(os.listdir(path.parent)) == ["plans.json"]


@pytest.mark.parametrize("bad", [
    {"window": 1, "lanes": 32, "blocks_per_sm": 0},
    {"window": 10, "lanes": 12, "blocks_per_sm": 0},
    {"window": 10, "lanes": 32, "blocks_per_sm": -1},
    {"window": 10, "lanes": 32},
    "10/32/0",
])
def test_plan_cache_rejects_bad_plans(tmp_path, bad):
    path = tmp_path / "plans.json"
    path.write_text(json.dumps({"version": 1, "plans": {
        "good": {"window": 10, "lanes": 32, "blocks_per_sm": 0}, "bad": bad}}))
    c = tune.PlanCache(path)
    assert c.get("good") is not None and c.get("bad") is None
    with pytest.raises(ValueError):
        c.put("bad", bad if isinstance(bad, dict) else {})


def test_plan_cache_path_from_environment(tmp_path, monkeypatch):
    monkeypatch.setenv("NEURALSIM_PLAN_CACHE", str(tmp_path / "env.json"))
    c = tune.PlanCache()
    assert c.path == str(tmp_path / "env.json")
    c.put("k", {"window": 2, "lanes": 32, "blocks_per_sm": 1})
    assert json.loads((tmp_path / "env.json").read_text())["plans"]["k"]["window"] == 2
