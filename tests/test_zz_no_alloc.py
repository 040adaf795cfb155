"""The allocation-free Izhikevich step, called through the C ABI, against the
library's regular stepping path on the same neurons.

Callers that cannot allocate device memory where they step (a stream capture
of their own, a latency-bound loop, a plugin inside another framework's memory
pool) use ns_izhikevich_step_noalloc, whose compaction scratch is a fixed
device array. This file is collected last so that a failure here leaves every
other test already run; it passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200 import SimulationEngine
from neuralsim_b200.engine import Drive, Network, SimConfig

pytestmark = pytest.mark.gpu

TOL = 0.0  # the same float arithmetic: identical results expected


def test_noalloc_step_matches_regular_path_two_calls(lib):
    import torch
    n = 50_000
    rng = np.random.default_rng(11)
    r = rng.random(n)
    a = (0.02 + 0.08 * r * (r > 0.8)).astype(np.float32)
    b = (0.2 + 0.05 * (r > 0.8)).astype(np.float32)
    c = (-65.0 + 15.0 * r * r).astype(np.float32)
    d = (8.0 - 6.0 * r * r).astype(np.float32)
    v0 = rng.uniform(-75, 35, n).astype(np.float32)
    u0 = (b * v0).astype(np.float32)
    cur = rng.normal(0, 8, n).astype(np.float32)
    dt = 0.5

    # regular path: a network without synapses whose current stays constant
    params = np.stack([a, b, c, d], axis=1)
    net = Network(A.MODEL_IZHIKEVICH, params, np.zeros(n + 1, np.uint64), np.zeros(0, np.uint32),
                  np.zeros(0, np.float32), v0=v0, u0=u0)
    cfg = SimConfig(model=A.MODEL_IZHIKEVICH, input_mode=A.INPUT_DIRECT_DECAY, current_decay=1.0,
                    dt_ms=dt, stdp_enabled=False, homeostasis_enabled=False,
                    spike_log_capacity=1_000_000, spike_log_steps=10)
    eng = SimulationEngine(net, cfg, Drive())
    st = eng.download_state(with_weights=False)
    st["current"][:] = cur
    eng.upload_state(st, 0)
    eng.run(2)
    ref_spikes = eng.read_spikes(0, 2)
    ref = eng.download_state(with_weights=False)

    dev = torch.device("cuda:0")
    t = {k: torch.from_numpy(x).to(dev) for k, x in
         dict(v=v0, u=u0, a=a, b=b, c=c, d=d, cur=cur).items()}
    out = torch.zeros(n, dtype=torch.int32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    P = lambda x: C.c_void_p(x.data_ptr())
    got = []
    for _ in range(2):
        st_ = lib.ns_izhikevich_step_noalloc(n, P(t["v"]), P(t["u"]), P(t["a"]), P(t["b"]),
                                             P(t["c"]), P(t["d"]), P(t["cur"]), dt, P(out), P(cnt),
                                             C.c_void_p(stream.cuda_stream))
        assert st_ == A.NS_OK
        torch.cuda.synchronize()
        k = int(cnt.item())
        got.append(out[:k].cpu().numpy().astype(np.uint32))
    for q in range(2):
        assert len(got[q]) > 0
        assert np.array_equal(got[q], ref_spikes[q])
    assert np.abs(t["v"].cpu().numpy() - ref["v"]).max() <= TOL
    assert np.abs(t["u"].cpu().numpy() - ref["u"]).max() <= TOL


def test_noalloc_rejects_sizes_beyond_the_scratch(lib):
    # n above NS_NOALLOC_MAX_NEURONS (1048576) is refused before any device work
    one = C.c_void_p(1)
    assert lib.ns_izhikevich_step_noalloc(1048577, one, one, one, one, one, one, None, 0.5,
                                          one, one, None) == 1
    assert lib.ns_izhikevich_step_noalloc(0, one, one, one, one, one, one, None, 0.5,
                                          one, one, None) == 1
