"""Sharding batches of independent networks across GPUs (one process per
GPU). Networks are bin-packed by synapse count (longest-processing-time
greedy: largest first onto the least-loaded rank), every rank steps its
share as one batch with no per-step communication, and the per-network
results are gathered once at the end. This is the multi-GPU form of the
reference's population evaluation (src/evolution/population.rs:117-124),
whose genomes are independent.
"""
import numpy as np


def assign(costs, world):
    """Rank of every item: largest cost first onto the least-loaded rank
    (ties to the lower rank). Deterministic, so every rank computes the
    same assignment without communication."""
    costs = np.asarray(costs, np.float64)
    order = np.lexsort((np.arange(len(costs)), -costs))
    load = np.zeros(world)
    rank = np.zeros(len(costs), np.int64)
    for i in order:
        r = int(np.argmin(load))
        rank[i] = r
        load[r] += costs[i]
    return rank


def network_cost(net):
    """Work of one network per step: neuron updates plus synapses."""
    return float(net.n) + float(net.m)


def run_sharded(networks, seeds, evaluate, rank, world, group=None):
    """Evaluates this rank's share of `networks` with
    evaluate(nets, seeds) -> list of per-network results (picklable), then
    gathers every rank's results; returns the results of all networks in
    their original order (on every rank)."""
    owner = assign([network_cost(x) for x in networks], world)
    mine = [i for i in range(len(networks)) if owner[i] == rank]
    res = evaluate([networks[i] for i in mine], [seeds[i] for i in mine]) if mine else []
    if len(res) != len(mine):
        raise RuntimeError("evaluate returned a result count that differs from its networks")
    local = list(zip(mine, res))
    if world == 1:
        gathered = [local]
    else:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, local, group=group)
    out = [None] * len(networks)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out


# ---------------------------------------------------------------------------
# One network split over ranks (no counterpart in the reference, which steps
# one network on one device). Rank r owns a tile-aligned neuron range and
# holds the synapses onto it; every step the ranks all-gather the step's
# spike bitmap (ns_shard_* in include/neuralsim.h). The union of the ranks'
# results equals the one-GPU run bit for bit.
# ---------------------------------------------------------------------------

def shard_range(n, rank, world):
    """Neurons [lo, hi) of `rank`: whole 2048-neuron tiles per rank, as the
    library computes them."""
    import ctypes as C
    from . import _abi as A
    lib = A.load()
    lo, hi = C.c_uint64(), C.c_uint64()
    st = lib.ns_shard_range(int(n), int(rank), int(world), C.byref(lo), C.byref(hi))
    if st != A.NS_OK:
        raise A.NsError(st, "ns_shard_range")
    return int(lo.value), int(hi.value)


def partition_network(net, rank, world):
    """The rank's network: every neuron's SoA and the synapses whose target
    the rank owns, in CSR order (each source row keeps its own order), with
    global target indices. Returns (network, positions): positions[e] is the
    CSR position in `net` of the rank's synapse e."""
    from dataclasses import replace
    lo, hi = shard_range(net.n, rank, world)
    mine = (net.col >= lo) & (net.col < hi)
    pos = np.flatnonzero(mine).astype(np.int64)
    src = np.repeat(np.arange(net.n), np.diff(net.row_ptr.astype(np.int64)))
    rp = np.zeros(net.n + 1, np.uint64)
    rp[1:] = np.cumsum(np.bincount(src[mine], minlength=net.n))
    sub = lambda a: None if a is None else a[pos]
    part = replace(net, row_ptr=rp, col=net.col[pos], w=net.w[pos], syn_type=sub(net.syn_type),
                   plastic=sub(net.plastic), eligible=sub(net.eligible),
                   stp=None if net.stp is None else net.stp[pos],
                   has_stp=None if (net.stp is None or net.has_stp is None) else net.has_stp[pos])
    return part, pos


class VirtualShards:
    """`world` ranks of one network driven by one process (on one GPU or
    several): each step every rank updates its own neurons, the ranks copy
    their spike bitmap words to one another, and every rank finishes the
    step. The multi-process form is ShardedEngine."""

    def __init__(self, net, cfg, drive, world, devices=None):
        from .engine import SimulationEngine
        from dataclasses import replace
        self.net, self.world = net, world
        self.ranks, self.pos, self.range = [], [], []
        for r in range(world):
            part, pos = partition_network(net, r, world)
            c = replace(cfg, device=(devices[r] if devices else cfg.device))
            self.ranks.append(SimulationEngine(part, c, drive, shard=(r, world)))
            self.pos.append(pos)
            self.range.append(shard_range(net.n, r, world))

    def run(self, steps):
        from . import _abi as A
        lib = A.load()
        for _ in range(steps):
            for e in self.ranks:
                e._check(lib.ns_shard_step_begin(e._h))
            for d in self.ranks:
                for s in self.ranks:
                    if s is not d:
                        d._check(lib.ns_shard_copy_bitmap(d._h, s._h))
            for e in self.ranks:
                e._check(lib.ns_shard_step_end(e._h))

    def read_raster(self, first_step, n_steps):
        """Every rank logs the whole network's spikes; rank 0's log."""
        return self.ranks[0].read_raster(first_step, n_steps)

    def download_state(self):
        """Owned neurons' state from each rank and the weights scattered to
        the network's CSR positions."""
        out = None
        w = np.zeros(self.net.m, np.float32)
        for e, pos, (lo, hi) in zip(self.ranks, self.pos, self.range):
            st = e.download_state()
            if out is None:
                out = {k: v.copy() for k, v in st.items() if k != "w"}
            for k, v in st.items():
                if k == "w" or v.ndim != 1 or v.shape[0] != self.net.n:
                    continue
                out[k][lo:hi] = v[lo:hi]
            w[pos] = st["w"]
        out["w"] = w
        return out

    def events(self):
        """Synaptic events of all ranks (each walks its own targets)."""
        return sum(int(e.counters()[3]) for e in self.ranks)

    def lfp(self):
        """lfp_signal of the network: the ranks' sums over their own neurons."""
        return sum(e.lfp() for e in self.ranks)

    def stimulate(self, neuron_ids, currents):
        """Host stimulus: every rank keeps the neurons it owns."""
        for e in self.ranks:
            e.stimulate(neuron_ids, currents)

    def close(self):
        for e in self.ranks:
            e.close()


class ShardedEngine:
    """This process's rank of a network split over the ranks of a
    torch.distributed job (one GPU each): rank 0 makes the NCCL id, the
    process group carries it, and every step's spike-bitmap all-gather runs
    inside the captured step graphs."""

    def __init__(self, net, cfg, drive, rank, world, group=None):
        import ctypes as C
        import torch.distributed as dist
        from dataclasses import replace
        from . import _abi as A
        from .engine import SimulationEngine
        lib = A.load()
        part, self.pos = partition_network(net, rank, world)
        self.range = shard_range(net.n, rank, world)
        self.engine = SimulationEngine(part, cfg, drive, shard=(rank, world))
        buf = (C.c_char * 128)()
        if rank == 0:
            st = lib.ns_shard_nccl_unique_id(buf)
            if st != A.NS_OK:
                raise A.NsError(st, (lib.ns_last_error(None) or b"").decode())
        box = [bytes(buf) if rank == 0 else None]
        dist.broadcast_object_list(box, src=0, group=group)
        C.memmove(buf, box[0], 128)
        self.engine._check(lib.ns_shard_nccl_init(self.engine._h, buf))

    def run(self, steps):
        return self.engine.run(steps)

    def lfp(self):
        """This rank's share of lfp_signal (its own neurons); the network's
        value is the sum over ranks."""
        return self.engine.lfp()

    def stimulate(self, neuron_ids, currents):
        """Host stimulus (every rank may pass the same list: each keeps the
        neurons it owns)."""
        self.engine.stimulate(neuron_ids, currents)

    def close(self):
        self.engine.close()
