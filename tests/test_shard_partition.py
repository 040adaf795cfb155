"""CPU: splitting one network over ranks by tile-aligned neuron ranges
(neuralsim_b200.shard.partition_network) and the ranks' agreement on it
(gloo, world size 2). The device step of a sharded network is checked
against the one-GPU run in tests/test_gpu_shard.py."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from neuralsim_b200 import shard
import nets


def test_ranges_are_tiles_and_cover(lib):
    for n in (1, 2047, 2048, 10_000, 1_000_000):
        for world in (1, 2, 3, 4, 8):
            r = [shard.shard_range(n, q, world) for q in range(world)]
            assert r[0][0] == 0 and r[-1][1] == n
            for (a, b), (c, _) in zip(r, r[1:]):
                assert b == c and a <= b
            per = r[0][1] - r[0][0]
            assert per % 2048 == 0 or world == 1 or per == n


def test_partition_union_is_the_network(lib):
    net, _, _ = nets.izh_stdp(n=9000, k=40)
    for world in (2, 3):
        w = np.zeros(net.m, np.float32)
        seen = np.zeros(net.m, np.int64)
        for r in range(world):
            part, pos = shard.partition_network(net, r, world)
            lo, hi = shard.shard_range(net.n, r, world)
            assert part.n == net.n and part.row_ptr[-1] == part.m == len(pos)
            assert np.all((part.col >= lo) & (part.col < hi))
            # rows keep their CSR order: positions ascend inside every row
            src = np.repeat(np.arange(net.n), np.diff(part.row_ptr.astype(np.int64)))
            gsrc = np.repeat(np.arange(net.n), np.diff(net.row_ptr.astype(np.int64)))
            assert np.array_equal(src, gsrc[pos]) and np.all(np.diff(pos) > 0)
            assert np.array_equal(part.col, net.col[pos]) and np.array_equal(part.plastic, net.plastic[pos])
            w[pos] = part.w
            seen[pos] += 1
        assert np.all(seen == 1) and np.array_equal(w, net.w)


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        net, _, _ = nets.izh_stdp(n=7000, k=30)
        part, pos = shard.partition_network(net, rank, world)
        mine = (rank, shard.shard_range(net.n, rank, world), int(part.m), pos.tolist())
        got = [None] * world
        dist.all_gather_object(got, mine)
        # the 128-byte id rank 0 makes reaches every rank (ShardedEngine's path)
        box = [bytes(range(128)) if rank == 0 else None]
        dist.broadcast_object_list(box, src=0)
        q.put((rank, got, box[0]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_ranks_agree_on_the_partition_gloo_world2(lib):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict((r, (g, b)) for r, g, b in (q.get(timeout=240) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    net, _, _ = nets.izh_stdp(n=7000, k=30)
    g0, b0 = res[0]
    assert g0 == res[1][0] and b0 == res[1][1] == bytes(range(128))
    allpos = sorted(p for _, _, _, pos in g0 for p in pos)
    assert allpos == list(range(net.m))
    assert g0[0][1][1] == g0[1][1][0] and g0[1][1][1] == net.n
