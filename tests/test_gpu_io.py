"""Checkpoints in the reference's on-disk format (src/io/checkpoint.rs,
src/io/save.rs, src/io/load.rs) on the GPU: a network in the reference's
serde-JSON form runs K steps, is saved with its dynamic state and metadata,
loaded into a fresh engine and run K more steps; the result equals one run
of 2K steps bit for bit (raster of the second half, neuron state, traces,
last spike steps, weights, and the rule-specific state of each case)."""
import json

import numpy as np
import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200 import SimulationEngine
from neuralsim_b200 import io as nio
import nets

pytestmark = pytest.mark.gpu

K = 150


def _case(which):
    if which == "izh_stdp_bf16":
        net, cfg, drive = nets.izh_stdp(n=6000, k=60)
    elif which == "reference_default":
        # DIRECT_DECAY current, STDP and homeostasis, the reference's drive
        net, cfg, drive = nets.lif_reference_default(n=1500)
    else:
        net, cfg, drive = nets.izh_rstdp(n=4000, k=40)
    return net, cfg, drive


@pytest.mark.parametrize("which", ["izh_stdp_bf16", "reference_default", "rstdp"])
def test_checkpoint_in_reference_format_resumes_bit_exact(lib, tmp_path, which):
    net0, cfg, drive = _case(which)
    # the network as the reference's document, read back
    doc = json.loads(json.dumps(nio.network_to_dict(net0)))
    net = nio.network_from_dict(doc)
    a = SimulationEngine(net, cfg, drive)
    a.run(K)
    mgr = nio.CheckpointManager(tmp_path)
    mgr.save_engine(a, "half")
    meta = json.load(open(tmp_path / "half_meta.json"))
    assert meta["sim_time_ms"] == K * cfg.dt_ms and meta["neuron_count"] == net.n
    net_b, st_b, _ = mgr.load("half", cfg)
    b = SimulationEngine(net_b, cfg, drive)
    b.restore(st_b)
    assert b.current_step() == K
    b.run(K)
    a.run(K)
    ra, rb = a.read_raster(K, K), b.read_raster(K, K)
    assert len(ra[0]) > 0
    assert nets.rasters_equal(ra, rb)
    sa, sb = a.checkpoint(), b.checkpoint()
    for key in ("v", "u", "refractory", "current", "pre_trace", "post_trace", "last_spike_step",
                "pending_input", "w", "firing_rate"):
        assert np.array_equal(sa[key], sb[key]), key
    if which == "reference_default":
        assert np.array_equal(sa["contributions"], sb["contributions"])
    if which == "rstdp":
        assert np.array_equal(sa["eligibility"], sb["eligibility"])
        assert sa["reward"] == sb["reward"]
    a.close()
    b.close()


def test_reference_saved_state_without_device_fields(lib):
    # a document as the Rust application saves it mid-run (no device_state
    # object): neuron state, traces, last spikes, weights and the clock are
    # taken from the reference's own fields; in the reset-each-step input mode
    # nothing else is carried between steps but the input propagated at the
    # last step, so resuming from the saved step with that input cleared
    # equals a run that drops it too
    net, cfg, drive = nets.izh_stdp(n=4000, k=40, wf=A.WEIGHT_F32)
    a = SimulationEngine(net, cfg, drive)
    a.run(K)
    st = a.checkpoint()
    d = json.loads(json.dumps(nio.network_to_dict(a.network, state=st, cfg=cfg)))
    del d["device_state"]
    back = nio.state_from_dict(d, nio.network_from_dict(d), cfg)
    for key in ("v", "u", "last_spike_step", "w"):
        assert np.array_equal(back[key], st[key]), key
    # the records carry the pre traces of sources with plastic synapses (the
    # excitatory neurons) and the post traces of their targets
    src = np.repeat(np.arange(net.n), np.diff(net.row_ptr.astype(np.int64)))
    pl = net.plastic.astype(bool)
    has_pre = np.zeros(net.n, bool)
    has_pre[src[pl]] = True
    has_post = np.zeros(net.n, bool)
    has_post[net.col[pl]] = True
    assert np.array_equal(back["pre_trace"][has_pre], st["pre_trace"][has_pre])
    assert np.array_equal(back["post_trace"][has_post], st["post_trace"][has_post])
    assert back["step"] == K
    b = SimulationEngine(nio.network_from_dict(d), cfg, drive)
    b.restore(back)
    st["pending_input"] = np.zeros_like(st["pending_input"])
    st["pre_trace"] = np.where(has_pre, st["pre_trace"], 0).astype(np.float32)
    st["post_trace"] = np.where(has_post, st["post_trace"], 0).astype(np.float32)
    a.upload_state(st, K)
    a.run(40)
    b.run(40)
    assert np.array_equal(a.download_state()["v"], b.download_state()["v"])
    assert np.array_equal(a.download_state()["w"], b.download_state()["w"])
