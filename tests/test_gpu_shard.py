"""GPU: one network split over ranks (the ranks driven by one process on one
GPU, their spike bitmaps copied between them every step) equals the one-GPU
run bit for bit: rasters, every rank's own neuron state, weights (scattered
back to CSR positions) and the summed synaptic events."""
import numpy as np
import pytest

from neuralsim_b200 import SimulationEngine, NsError
from neuralsim_b200.shard import VirtualShards, partition_network
import nets

pytestmark = pytest.mark.gpu


def compare(net, cfg, drive, steps, world):
    one = SimulationEngine(net, cfg, drive)
    one.run(steps)
    vs = VirtualShards(net, cfg, drive, world)
    vs.run(steps)
    ra, rb = one.read_raster(0, steps), vs.read_raster(0, steps)
    assert len(ra[0]) > 100
    assert nets.rasters_equal(ra, rb)
    sa, sb = one.download_state(), vs.download_state()
    for key in ("v", "u", "pre_trace", "post_trace", "last_spike_step", "w"):
        assert np.array_equal(sa[key], sb[key]), key
    assert vs.events() == int(one.counters()[3])
    return one, vs


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_izhikevich_stdp_equals_one_gpu(lib, world):
    net, cfg, drive = nets.izh_stdp(n=12_000, k=60)
    compare(net, cfg, drive, 300, world)


def test_sharded_reference_engine_with_phase2_rules(lib):
    # direct current mode, reference drive, STDP, homeostasis, R-STDP and
    # consolidation: each rank's rules act on its own synapses; the reward
    # counts every output spike on every rank
    net, cfg, drive = nets.lif_reference_default(n=5000)
    net.is_output = (np.arange(net.n) < 1000).astype(np.uint8)
    cfg.rstdp_enabled = True
    cfg.reward_threshold = 2
    nets.with_consolidation(cfg, tau=200.0, drift=0.05)
    one, vs = compare(net, cfg, drive, 150, 2)
    assert one.reward() == vs.ranks[0].reward() == vs.ranks[1].reward()
    e = np.zeros(net.m, np.float32)
    for r, pos in zip(vs.ranks, vs.pos):
        e[pos] = r.eligibility()
    assert np.array_equal(e, one.eligibility())


def test_sharded_reference_conductance_mode_and_lfp(lib):
    # the reference conductance mode with all four synapse types: rasters,
    # state and conductance-driven dynamics equal; the LFP is each rank's
    # sum over its own neurons, so only the FP64 summation order differs
    net, cfg, drive = nets.lif_conductance_all_types(n=6000)
    one, vs = compare(net, cfg, drive, 120, 2)
    assert one.lfp() > 1e6
    assert vs.lfp() == pytest.approx(one.lfp(), rel=1e-12)


def test_sharded_stimulus_equals_one_gpu(lib):
    # each rank keeps the stimulus of the neurons it owns
    net, cfg, drive = nets.izh_stdp(n=12_000, k=60)
    one = SimulationEngine(net, cfg, drive)
    vs = VirtualShards(net, cfg, drive, 2)
    ids = list(range(0, 12_000, 37))
    for e in (one, vs):
        e.run(50)
        e.stimulate(ids, [30.0])
        e.run(100)
    assert nets.rasters_equal(one.read_raster(0, 150), vs.read_raster(0, 150))
    assert np.array_equal(one.download_state()["v"], vs.download_state()["v"])


def test_sharded_rank_rejects_foreign_synapses(lib):
    net, cfg, drive = nets.izh_stdp(n=6000, k=20)
    part, _ = partition_network(net, 0, 2)
    with pytest.raises(NsError):
        SimulationEngine(net, cfg, drive, shard=(0, 2))   # the whole CSR: targets it does not own
    eng = SimulationEngine(part, cfg, drive, shard=(0, 2))
    with pytest.raises(NsError):
        eng.run(1)                                        # no NCCL: the caller exchanges
    eng.close()


def test_sharded_ranks_without_neurons(lib):
    # 3 ranks over a network of one tile: ranks 1 and 2 own no neurons and
    # hold no synapses, but take part in every step's exchange
    from neuralsim_b200.shard import shard_range
    net, cfg, drive = nets.izh_stdp(n=1500, k=30)
    assert shard_range(net.n, 1, 3) == (net.n, net.n)
    compare(net, cfg, drive, 200, 3)


def test_shard_configure_after_upload_is_refused(lib):
    net, cfg, drive = nets.izh_stdp(n=2000, k=20)
    eng = SimulationEngine(net, cfg, drive)
    with pytest.raises(NsError):
        eng._check(eng.lib.ns_shard_configure(eng._h, 0, 2))
    eng.close()

