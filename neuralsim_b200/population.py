"""Population evaluation on the batched launch.

Population::evolve_generation (src/evolution/population.rs:117-124) builds
one engine per genome and evaluates them in parallel with a
FitnessEvaluator. Here the genomes' networks run as one batch
(ns_upload_batch) per GPU, and the RateHomeostasis evaluator
(src/evolution/fitness.rs:59-76) is computed from the device-side mean
firing rate of every network (ns_network_rates).
"""
from dataclasses import dataclass

import numpy as np

from .batch import BatchEngine
from . import shard


@dataclass
class RateHomeostasis:
    """fitness = 1 / (1 + |mean rate - target|), x0.1 when the mean rate is
    below 1 Hz (penalize_silence) and x0.1 above 500 Hz
    (src/evolution/fitness.rs:34-76; lifetime 500 ms by default)."""
    target_rate: float
    lifetime_ms: float = 500.0
    penalize_silence: bool = True

    def fitness(self, mean_rate):
        r = np.asarray(mean_rate, np.float64)
        f = 1.0 / (1.0 + np.abs(r - self.target_rate))
        if self.penalize_silence:
            f = np.where(r < 1.0, f * 0.1, f)
        return np.where(r > 500.0, f * 0.1, f)


def evaluate_batch(networks, seeds, config, drive, evaluator):
    """Steps every network for the evaluator's lifetime in one batch on this
    GPU and returns (fitness, mean rate) per network."""
    steps = int(evaluator.lifetime_ms / config.dt_ms)
    eng = BatchEngine(networks, seeds, config, drive)
    try:
        eng.run(steps)
        rates = eng.network_rates(0, steps)
    finally:
        eng.close()
    return evaluator.fitness(rates), rates


def evaluate_population(networks, seeds, config, drive, evaluator, rank=0, world=1, group=None):
    """Fitness of every genome's network (original order, on every rank):
    networks bin-packed across ranks, one batch per GPU, one gather."""
    def ev(nets, sds):
        f, r = evaluate_batch(nets, sds, config, drive, evaluator)
        return [(float(a), float(b)) for a, b in zip(f, r)]
    res = shard.run_sharded(networks, seeds, ev, rank, world, group)
    return np.array([x[0] for x in res]), np.array([x[1] for x in res])
