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


def izh_rstdp(n=2000, k=50, seed=44, wf=A.WEIGHT_F32, reward_decay=0.5, threshold=3,
              n_out=200, rstdp_w_max=10.0, consolidation=False, homeo=False):
    """Izhikevich + pair STDP with R-STDP: the first n_out neurons are outputs,
    every plastic synapse carries an eligibility trace, and a fast reward
    decay makes rewarded stretches start and stop often (both reward paths)."""
    net, cfg, drive = izh_stdp(n=n, k=k, seed=seed, wf=wf)
    out = np.zeros(n, np.uint8)
    out[:n_out] = 1
    net.is_output = out
    cfg.rstdp_enabled = True
    cfg.rstdp_lr = 0.5
    cfg.rstdp_w_max = rstdp_w_max
    cfg.reward_decay = reward_decay
    cfg.reward_threshold = threshold
    cfg.homeostasis_enabled = homeo
    if consolidation:
        cfg.consolidation_enabled = True
    return net, cfg, drive


def with_consolidation(cfg, tau=10000.0, target=0.5, drift=0.001):
    cfg.consolidation_enabled = True
    cfg.consolidation_tau, cfg.consolidation_target, cfg.consolidation_drift = tau, target, drift
    return cfg


def with_stp(net, frac=0.5, seed=7):
    """Tsodyks-Markram state on a fraction of the synapses (u_se, tau_rec,
    tau_facil, u, r), u and r away from their rest values."""
    rng = np.random.default_rng(seed)
    m = net.m
    stp = np.zeros((m, 5))
    stp[:, 0] = rng.uniform(0.1, 0.6, m)
    stp[:, 1] = rng.uniform(50.0, 800.0, m)
    stp[:, 2] = rng.uniform(20.0, 1000.0, m)
    stp[:, 3] = rng.uniform(0.05, 0.9, m)
    stp[:, 4] = rng.uniform(0.3, 1.0, m)
    net.stp = stp
    net.has_stp = (rng.random(m) < frac).astype(np.uint8)
    return net


def lif_conductance_all_types(n=1500, seed=42):
    """Reference conductance mode with all four synapse types: excitatory
    sources split AMPA / NMDA, inhibitory sources GABA / GABA-B."""
    net, cfg, drive = lif_reference_default(n=n, seed=seed, stdp=False, homeo=False, conductance=True)
    rng = np.random.default_rng(seed + 1)
    ty = net.syn_type.copy()
    flip = rng.random(len(ty)) < 0.4
    ty[(ty == A.SYN_AMPA) & flip] = A.SYN_NMDA
    ty[(ty == A.SYN_GABA) & flip] = A.SYN_GABA_B
    net.syn_type = ty
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
