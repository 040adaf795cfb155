"""Multi-rank host logic on CPU (gloo, world size 2): sharding of network
batches across ranks and the final gather; raster splitting of a batch.
The device work per rank is stood in for by the oracle (test side only)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from neuralsim_b200 import shard
from neuralsim_b200.batch import split_raster_by_network


def test_assign_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = np.exp(rng.uniform(np.log(2e3), np.log(5e4), 256)) * rng.integers(50, 201, 256)
    for world in (1, 2, 3, 8):
        r = shard.assign(costs, world)
        assert r.min() >= 0 and r.max() < world
        load = np.bincount(r, weights=costs, minlength=world)
        assert np.isclose(load.sum(), costs.sum())
        # LPT bound: no rank exceeds the mean by more than the largest item
        assert load.max() <= costs.sum() / world + costs.max() + 1e-6
        assert np.array_equal(r, shard.assign(costs, world))  # deterministic


def test_split_raster_by_network():
    first = np.array([0, 3, 7, 10])
    # two steps: step 0 spikes 1, 4, 9; step 1 spikes 0, 6
    idx = np.array([1, 4, 9, 0, 6], np.uint32)
    off = np.array([0, 3, 5], np.uint64)
    parts = split_raster_by_network(idx, off, first)
    assert [list(p[0]) for p in parts] == [[1, 0], [1, 3], [2]]
    assert [list(p[1]) for p in parts] == [[0, 1, 2], [0, 1, 2], [0, 1, 1]]


def _small_nets():
    from neuralsim_b200 import configs
    nets, seeds, cfg, drive, _ = configs.lif_batch_c3(n_nets=5, size_range=(200, 500),
                                                      k_range=(10, 30))
    from neuralsim_b200 import _abi as A
    from neuralsim_b200.engine import Drive
    drive = Drive(A.DRIVE_POISSON_KICK, p=0.02, amplitude=4.0)
    cfg.spike_log_capacity, cfg.spike_log_steps = 1_000_000, 1000
    return nets, seeds, cfg, drive


def _oracle_eval(nets, seeds, cfg, drive, steps=200):
    import copy
    from oracle.oracle import FastOracle
    out = []
    for net, sd in zip(nets, seeds):
        c = copy.copy(cfg)
        c.seed = sd
        o = FastOracle(net, c, drive, precision=32)
        o.step(steps)
        out.append(int(len(o.raster()[0])))
        o.close()
    return out


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        nets, seeds, cfg, drive = _small_nets()
        res = shard.run_sharded(nets, seeds, lambda n, s: _oracle_eval(n, s, cfg, drive),
                                rank, world)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_run_sharded_gloo_world2(lib, oracle_lib):
    nets, seeds, cfg, drive = _small_nets()
    want = _oracle_eval(nets, seeds, cfg, drive)
    assert sum(want) > 0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0] == want and got[1] == want


class _FakeSurrogate:
    """Stands in for a device surrogate: a rank-dependent gradient per step
    and a record of the applied (scaled) gradients."""

    def __init__(self, rank):
        self.rank = rank
        self._p = np.full(17796, float(rank + 1), np.float32)
        self.applied = []

    @property
    def params(self):
        return self._p.copy()

    @params.setter
    def params(self, p):
        self._p = np.asarray(p, np.float32).copy()

    def grad_step(self, grad):
        grad.fill_(float(self.rank + 1))
        return 0.5 * (self.rank + 1)

    def apply_gradient(self, grad, scale, lr):
        self.applied.append((float(grad[0]) * scale, lr))


def _dp_worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    from neuralsim_b200.surrogate import train_data_parallel
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        s = _FakeSurrogate(rank)
        losses = train_data_parallel(s, 3, lr=1e-3, lr_final=1e-4, rank=rank, world=world,
                                     grad=torch.zeros(17796))
        q.put((rank, float(s.params[0]), s.applied, [float(x) for x in losses]))
    finally:
        dist.destroy_process_group()


def test_data_parallel_surrogate_training_gloo_world2():
    # every rank applies the mean of the ranks' gradients, starting from
    # rank 0's weights; the reported loss is the mean over ranks
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dp_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict((r[0], r[1:]) for r in (q.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        p0, applied, losses = got[r]
        assert p0 == 1.0                                   # broadcast from rank 0
        assert [a for a, _ in applied] == [1.5, 1.5, 1.5]  # mean of 1 and 2
        assert np.allclose(losses, 0.75)
    assert got[0][1] == got[1][1]


def test_rate_homeostasis_fitness_matches_reference_formula():
    # src/evolution/fitness.rs:59-76
    from neuralsim_b200.population import RateHomeostasis
    ev = RateHomeostasis(target_rate=5.0)
    r = np.array([0.0, 0.5, 1.0, 5.0, 7.5, 499.0, 501.0])
    want = []
    for x in r:
        f = 1.0 / (1.0 + abs(x - 5.0))
        if x < 1.0:
            f *= 0.1
        if x > 500.0:
            f *= 0.1
        want.append(f)
    assert np.allclose(ev.fitness(r), want, rtol=0, atol=1e-15)
