"""Batches of independent networks stepped together (one handle, one launch
per kernel for all networks).

The reference evaluates populations and sweeps one engine per network
(Population::evolve_generation, src/evolution/population.rs:117-124, one
SimulationEngine per genome). Here the networks are concatenated block-
diagonally on the device by ns_upload_batch; every network keeps its own
drive stream (its seed and its local neuron indices), so each network's
raster equals the raster it produces alone with the same config and seed.
"""
import ctypes as C

import numpy as np

from . import _abi as A
from .engine import PARAMS_PER_NEURON, Network, SimConfig, Drive, SimulationEngine, _ptr


class _BatchShape:
    """The concatenated network as the engine sees it (sizes only)."""

    def __init__(self, networks):
        self.model = networks[0].model
        self.n = int(sum(x.n for x in networks))
        self.m = int(sum(x.m for x in networks))


class BatchEngine(SimulationEngine):
    """Steps `networks` (all of one neuron model, one SimConfig and one drive
    kind) together; network q draws its drive from seeds[q]."""

    def __init__(self, networks, seeds, config: SimConfig, drive: Drive = None, plan_cache=None):
        self.networks = list(networks)
        self.seeds = [int(s) for s in seeds]
        if not self.networks or len(self.seeds) != len(self.networks):
            raise ValueError("one seed per network")
        if any(x.model != self.networks[0].model for x in self.networks):
            raise ValueError("all networks of a batch use one neuron model")
        self.first_neuron = None
        super().__init__(_BatchShape(self.networks), config, drive, plan_cache=plan_cache)

    def _upload(self, _shape):
        nets = self.networks
        descs = (A.NsNetDesc * len(nets))()
        keep = []
        for q, net in enumerate(nets):
            soa = A.NsNeuronSoa()
            soa.n = net.n
            soa.params = _ptr(net.params)
            soa.params_per_neuron = PARAMS_PER_NEURON[net.model]
            soa.v, soa.u = _ptr(net.v0), _ptr(net.u0)
            soa.hh_m, soa.hh_h, soa.hh_n = _ptr(net.m0), _ptr(net.h0), _ptr(net.n0)
            soa.inhibitory, soa.is_output = _ptr(net.inhibitory), _ptr(net.is_output)
            keep.append(soa)
            d = descs[q]
            d.neurons = C.pointer(soa)
            d.m = net.m
            d.row_ptr, d.col, d.w = _ptr(net.row_ptr), _ptr(net.col), _ptr(net.w)
            d.syn_type, d.plastic = _ptr(net.syn_type), _ptr(net.plastic)
            d.seed = self.seeds[q]
        first = np.zeros(len(nets) + 1, np.uint64)
        self._check(self.lib.ns_upload_batch(self._h, len(nets), descs, _ptr(first)))
        self.first_neuron = first.astype(np.int64)
        del keep

    def stimulate_network(self, q, neuron_ids, currents):
        """Host stimulus for neurons of network q, by their index inside it."""
        ids = np.atleast_1d(np.asarray(neuron_ids, dtype=np.int64))
        if ids.size and (ids.min() < 0 or ids.max() >= self.networks[q].n):
            raise ValueError("neuron index outside network %d" % q)
        self.stimulate(ids + int(self.first_neuron[q]), currents)

    def split(self, per_neuron):
        """Splits a per-neuron array of the concatenation into networks."""
        f = self.first_neuron
        return [per_neuron[f[q]:f[q + 1]] for q in range(len(self.networks))]

    def read_rasters(self, first_step, n_steps):
        """Per network: (ascending local indices, per-step offsets)."""
        idx, off = self.read_raster(first_step, n_steps)
        return split_raster_by_network(idx, off, self.first_neuron)

    def spike_counts(self, first_step, n_steps):
        """Spikes per network over the logged steps."""
        idx, _ = self.read_raster(first_step, n_steps)
        net = np.searchsorted(self.first_neuron, idx.astype(np.int64), side="right") - 1
        return np.bincount(net, minlength=len(self.networks))


def split_raster_by_network(idx, off, first_neuron):
    """Splits a raster of the concatenation (ascending global indices per
    step, per-step offsets) into per-network rasters in local indices."""
    idx = np.asarray(idx, np.int64)
    off = np.asarray(off, np.int64)
    f = np.asarray(first_neuron, np.int64)
    n_steps = len(off) - 1
    net = np.searchsorted(f, idx, side="right") - 1
    steps = np.repeat(np.arange(n_steps), np.diff(off))
    out = []
    for q in range(len(f) - 1):
        sel = net == q
        cnt = np.bincount(steps[sel], minlength=n_steps)
        o = np.zeros(n_steps + 1, np.uint64)
        o[1:] = np.cumsum(cnt)
        out.append(((idx[sel] - f[q]).astype(np.uint32), o))
    return out
