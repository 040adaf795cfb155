"""Windowed-step plans per network-size bucket, cached as JSON.

The window tuner (inside the handle's first ns_step) times the window
lengths D, D/2, ... and then the shape of the window's row walk (lanes per
spiking row: 32, 16 or 8; blocks per SM: the occupancy limit or half of it)
on the network at hand, from one device snapshot. Networks of the same
bucket want the same plan, so a PlanCache keys tuned plans by bucket and an
engine that finds its bucket in the cache fixes that plan with
ns_set_window_plan instead of tuning again. Every plan gives the same
results; only the time per step depends on it.

Bucket: neuron model, input mode, weight format, delay steps, and the
network's neuron count and mean out-degree rounded to powers of two (for a
batch: the concatenation's totals, which set the kernels' grid).
"""
import json
import math
import os
import tempfile

DEFAULT_PATH = os.path.join(os.path.expanduser("~"), ".cache", "neuralsim_b200", "window_plans.json")
_LANES = (8, 16, 32)


def bucket_key(model, input_mode, weight_format, delay_steps, n, m):
    """The size bucket of a network: equal keys share a plan."""
    ln = int(round(math.log2(max(int(n), 1))))
    ld = int(round(math.log2(max(float(m) / max(int(n), 1), 1.0))))
    return (f"model{int(model)}/input{int(input_mode)}/w{int(weight_format)}/D{int(delay_steps)}"
            f"/n2^{ln}/deg2^{ld}")


def valid_plan(p):
    """A plan: {"window": 2..1024, "lanes": 8|16|32, "blocks_per_sm": >= 0}."""
    try:
        return (2 <= int(p["window"]) <= 1024 and int(p["lanes"]) in _LANES
                and int(p["blocks_per_sm"]) >= 0)
    except (KeyError, TypeError, ValueError):
        return False


class PlanCache:
    """Tuned windowed plans by bucket key, in a JSON file (path, else
    $NEURALSIM_PLAN_CACHE, else ~/.cache/neuralsim_b200/window_plans.json).
    Entries that are not valid plans are ignored on load."""

    def __init__(self, path=None):
        self.path = str(path or os.environ.get("NEURALSIM_PLAN_CACHE") or DEFAULT_PATH)
        self.plans = {}
        if os.path.exists(self.path):
            with open(self.path) as f:
                doc = json.load(f)
            self.plans = {k: _norm(v) for k, v in doc.get("plans", {}).items() if valid_plan(v)}

    def get(self, key):
        return self.plans.get(key)

    def put(self, key, plan, us_per_step=None):
        if not valid_plan(plan):
            raise ValueError(f"not a window plan: {plan}")
        p = _norm(plan)
        if us_per_step is not None:
            p["us_per_step"] = float(us_per_step)
        self.plans[key] = p
        self.save()

    def save(self):
        """Writes the file atomically (a temporary file renamed over it)."""
        d = os.path.dirname(os.path.abspath(self.path))
        os.makedirs(d, exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=d, prefix=".window_plans.", suffix=".json")
        try:
            with os.fdopen(fd, "w") as f:
                json.dump({"version": 1, "plans": self.plans}, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except BaseException:
            if os.path.exists(tmp):
                os.unlink(tmp)
            raise


def _norm(p):
    out = {"window": int(p["window"]), "lanes": int(p["lanes"]), "blocks_per_sm": int(p["blocks_per_sm"])}
    if "us_per_step" in p:
        out["us_per_step"] = float(p["us_per_step"])
    return out
