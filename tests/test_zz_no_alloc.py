"""The allocation-free Izhikevich step, called through the C ABI, against the
library's regular stepping path on the same neurons.

Callers that cannot allocate device memory where they step (a stream capture
of their own, a latency-bound loop, a plugin inside another framework's memory
pool) use ns_izhikevich_step_noalloc, whose compaction scratch is a fixed
device array. This file is collected last so that a failure here leaves every
other test already run; it passes alone in a fresh process as well.

Sizes: 50,000 neurons (49 tiles of 1024, one warp of the gather's scan),
200,000 (196 tiles: the scan's cross-warp prefix and more tiles than gather
blocks), NS_NOALLOC_MAX_NEURONS - 1000 (a partial last tile among 1024) and
NS_NOALLOC_MAX_NEURONS itself (1024 full tiles, the scratch's limit).
"""
import ctypes as C

import numpy as np
import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200 import SimulationEngine
from neuralsim_b200.engine import Drive, Network, SimConfig

pytestmark = pytest.mark.gpu

TOL = 0.0  # the same float arithmetic: identical results expected
MAX_N = 1048576  # NS_NOALLOC_MAX_NEURONS
DT = 0.5


def _neurons(n, seed=11):
    rng = np.random.default_rng(seed)
    r = rng.random(n)
    a = (0.02 + 0.08 * r * (r > 0.8)).astype(np.float32)
    b = (0.2 + 0.05 * (r > 0.8)).astype(np.float32)
    c = (-65.0 + 15.0 * r * r).astype(np.float32)
    d = (8.0 - 6.0 * r * r).astype(np.float32)
    v0 = rng.uniform(-75, 35, n).astype(np.float32)
    u0 = (b * v0).astype(np.float32)
    cur = rng.normal(0, 8, n).astype(np.float32)
    return dict(v=v0, u=u0, a=a, b=b, c=c, d=d, cur=cur)


def _regular_path(x, steps=2):
    # a network without synapses whose input current stays constant
    n = len(x["v"])
    params = np.stack([x["a"], x["b"], x["c"], x["d"]], axis=1)
    net = Network(A.MODEL_IZHIKEVICH, params, np.zeros(n + 1, np.uint64), np.zeros(0, np.uint32),
                  np.zeros(0, np.float32), v0=x["v"], u0=x["u"])
    cfg = SimConfig(model=A.MODEL_IZHIKEVICH, input_mode=A.INPUT_DIRECT_DECAY, current_decay=1.0,
                    dt_ms=DT, stdp_enabled=False, homeostasis_enabled=False,
                    spike_log_capacity=4_000_000, spike_log_steps=10)
    eng = SimulationEngine(net, cfg, Drive())
    st = eng.download_state(with_weights=False)
    st["current"][:] = x["cur"]
    eng.upload_state(st, 0)
    eng.run(steps)
    spikes = eng.read_spikes(0, steps)
    ref = eng.download_state(with_weights=False)
    eng.close()
    return spikes, ref


def _device(x):
    import torch
    dev = torch.device("cuda:0")
    t = {k: torch.from_numpy(v.copy()).to(dev) for k, v in x.items()}
    n = len(x["v"])
    t["out"] = torch.zeros(n, dtype=torch.int32, device=dev)
    t["cnt"] = torch.zeros(1, dtype=torch.int32, device=dev)
    return t


def _call(lib, t, stream):
    P = lambda y: C.c_void_p(y.data_ptr())
    n = t["v"].numel()
    return lib.ns_izhikevich_step_noalloc(n, P(t["v"]), P(t["u"]), P(t["a"]), P(t["b"]),
                                          P(t["c"]), P(t["d"]), P(t["cur"]), DT, P(t["out"]),
                                          P(t["cnt"]), C.c_void_p(stream.cuda_stream))


@pytest.mark.parametrize("n", [50_000, 200_000, MAX_N - 1000, MAX_N])
def test_noalloc_step_matches_regular_path_two_calls(lib, n):
    import torch
    x = _neurons(n)
    ref_spikes, ref = _regular_path(x)
    t = _device(x)
    stream = torch.cuda.current_stream(torch.device("cuda:0"))
    got = []
    for _ in range(2):
        assert _call(lib, t, stream) == A.NS_OK
        torch.cuda.synchronize()
        k = int(t["cnt"].item())
        got.append(t["out"][:k].cpu().numpy().astype(np.uint32))
    for q in range(2):
        assert len(got[q]) > 0
        assert np.array_equal(got[q], ref_spikes[q])
    assert np.abs(t["v"].cpu().numpy() - ref["v"]).max() <= TOL
    assert np.abs(t["u"].cpu().numpy() - ref["u"]).max() <= TOL


def test_noalloc_step_in_a_captured_graph(lib):
    # the first call (which looks up the scratch address) runs eagerly on a
    # side stream; two calls are then captured into a CUDA graph and
    # replayed: the replay equals two eager calls bit for bit
    import torch
    n = 300_000
    x = _neurons(n, seed=12)
    eager = _device(x)
    s0 = torch.cuda.current_stream(torch.device("cuda:0"))
    for _ in range(2):
        assert _call(lib, eager, s0) == A.NS_OK
    torch.cuda.synchronize()
    warm = _device(_neurons(1000, seed=13))
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        assert _call(lib, warm, side) == A.NS_OK
    torch.cuda.synchronize()
    cap = _device(x)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        for _ in range(2):
            assert _call(lib, cap, side) == A.NS_OK
    g.replay()
    torch.cuda.synchronize()
    assert int(cap["cnt"].item()) == int(eager["cnt"].item()) > 0
    k = int(cap["cnt"].item())
    assert torch.equal(cap["out"][:k], eager["out"][:k])
    assert torch.equal(cap["v"], eager["v"]) and torch.equal(cap["u"], eager["u"])


def test_noalloc_rejects_sizes_beyond_the_scratch(lib):
    # n above NS_NOALLOC_MAX_NEURONS (1048576) is refused before any device work
    one = C.c_void_p(1)
    assert lib.ns_izhikevich_step_noalloc(MAX_N + 1, one, one, one, one, one, one, None, 0.5,
                                          one, one, None) == 1
    assert lib.ns_izhikevich_step_noalloc(0, one, one, one, one, one, one, None, 0.5,
                                          one, one, None) == 1
