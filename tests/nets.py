"""Small seeded networks of each configuration family, shared by the tests."""
import numpy as np

from neuralsim_b200 import _abi as A
from neuralsim_b200 import configs
from neuralsim_b200.engine import Drive, Network, SimConfig


def lif_delta(n=2000, k=50, seed=43):
    net, cfg, drive, _ = configs.lif_c1(n=n, k=k, seed=seed)
    # a stronger drive so that small nets are active within a few hundred steps
    drive = Drive(A.DRIVE_POISSON_KICK, p=0.02, amplitude=4.0)
    cfg.spike_log_capacity = 50_000_000
    cfg.spike_log_steps = 200_000
    return net, cfg, drive


def izh_stdp(n=2000, k=50, seed=44, wf=A.WEIGHT_BF16):
    net, cfg, drive, _ = configs.izh_c2(n=n, k=k, seed=seed, weight_format=wf)
    cfg.spike_log_capacity = 50_000_000
    cfg.spike_log_steps = 200_000
    return net, cfg, drive


def lif_reference_default(n=300, seed=42, stdp=True, homeo=True, conductance=False):
    """The reference engine's defaults: default LIF params, direct current
    mode with 0.92 decay (or conductance mode), its uniform drive, STDP and
    homeostatic scaling on (src/simulation/engine.rs:83-120)."""
    rng = np.random.default_rng(seed)
    k = 15
    rp, col = configs.topology(n, k, seed)
    n_exc = int(0.8 * n)
    src = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    exc = src < n_exc
    # connect_random weights: AMPA U[1,4), GABA -U[0,2) (src/network/mod.rs:108-127)
    u = rng.random(len(col))
    w = np.where(exc, u * 3.0 + 1.0, -u * 2.0).astype(np.float32)
    ty = np.where(exc, A.SYN_AMPA, A.SYN_GABA).astype(np.uint8)
    pl = np.ones(len(col), np.uint8)
    params = np.tile(np.array([-60.0, -50.0, -65.0, 8.0, 1.5, 2.0], np.float32), (n, 1))
    net = Network(A.MODEL_LIF, params, rp, col, w, syn_type=ty, plastic=pl,
                  inhibitory=(np.arange(n) >= n_exc).astype(np.uint8))
    cfg = SimConfig(model=A.MODEL_LIF, dt_ms=0.5, seed=seed, stdp_enabled=stdp,
                    homeostasis_enabled=homeo,
                    input_mode=A.INPUT_CONDUCTANCE_REF if conductance else A.INPUT_DIRECT_DECAY,
                    spike_log_capacity=10_000_000, spike_log_steps=100_000)
    drive = Drive.reference_default()
    return net, cfg, drive


def hh_cond(n=1000, k=50, seed=46, dt=0.01, integrator=A.HH_RUSH_LARSEN):
    net, cfg, drive, _ = configs.hh_c4(n=n, k=k, seed=seed, integrator=integrator, dt_ms=dt)
    cfg.spike_log_capacity = 20_000_000
    cfg.spike_log_steps = 400_000
    return net, cfg, drive


def rasters_equal(a, b):
    (ia, oa), (ib, ob) = a, b
    return np.array_equal(oa, ob) and np.array_equal(ia, ib)


from neuralsim_b200.raster import spike_times, match_spikes  # noqa: E402,F401
