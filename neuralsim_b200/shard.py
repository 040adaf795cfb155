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
