"""Synthetic workloads of the benchmark configurations (seeded; no dataset).

Seeds follow `42 + config_id` (the reference's default seed is 42,
src/simulation/engine.rs:99). Topology and weights come from the library's
generator (include/neuralsim_gen.h); per-neuron parameters from numpy.
Each builder takes the size as an argument so tests can use small cases of
the same shape.
"""
import ctypes as C

import numpy as np

from . import _abi as A
from .engine import Drive, Network, SimConfig


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def topology(n, k, seed, threads=0, with_insertion_order=False):
    """Fixed in-degree CSR (rows ascending in target)."""
    lib = A.load()
    row_ptr = np.zeros(n + 1, np.uint64)
    col = np.zeros(n * k, np.uint32)
    src = np.zeros(n * k, np.uint32) if with_insertion_order else None
    A.check(lib.ns_gen_topology(n, k, seed, _ptr(row_ptr), _ptr(col), _ptr(src), threads))
    return (row_ptr, col, src) if with_insertion_order else (row_ptr, col)


def weights(kind, n, n_exc, row_ptr, seed, a, b, c=0.0, d=0.0, plastic_exc=False, threads=0):
    lib = A.load()
    m = int(row_ptr[-1])
    w = np.zeros(m, np.float32)
    ty = np.zeros(m, np.uint8)
    pl = np.zeros(m, np.uint8)
    A.check(lib.ns_gen_weights(kind, n, n_exc, _ptr(row_ptr), m, seed, a, b, c, d, _ptr(w),
                               _ptr(ty), _ptr(pl), 1 if plastic_exc else 0, threads))
    return w, ty, pl


# ---------------------------------------------------------------------------
# C1: plain LIF, 10,000 neurons, 80/20, in-degree 100, w = +0.5 / -2.5 mV x
# U[0.8,1.2], tau_m 20 ms, V_th -50, V_reset -65, V_rest -65 (assumed), 2 ms
# refractory, dt 0.1 ms, 1 ms delay (10 steps), Poisson drive 8 Hz with
# 0.8 mV kicks, 1 s.
# ---------------------------------------------------------------------------
def lif_c1(n=10_000, k=100, seed=43, threads=0):
    n_exc = int(round(0.8 * n))
    rp, col = topology(n, k, seed, threads)
    w, ty, _ = weights(A.GEN_W_SCALED, n, n_exc, rp, seed, 0.5, -2.5, 0.8, 1.2, threads=threads)
    params = np.tile(np.array([-65.0, -50.0, -65.0, 20.0, 2.0, 1.0], np.float32), (n, 1))
    inh = (np.arange(n) >= n_exc).astype(np.uint8)
    net = Network(A.MODEL_LIF, params, rp, col, w, syn_type=ty, inhibitory=inh)
    cfg = SimConfig(model=A.MODEL_LIF, input_mode=A.INPUT_DELTA_V, dt_ms=0.1, delay_steps=10,
                    seed=seed, stdp_enabled=False, homeostasis_enabled=False)
    drive = Drive(A.DRIVE_POISSON_KICK, p=8.0 * 0.1 / 1000.0, amplitude=0.8)
    return net, cfg, drive, 10_000


# ---------------------------------------------------------------------------
# C2 (headline): Izhikevich + pair STDP, 1,000,000 neurons, 80% regular
# spiking (a .02, b .2, c -65+15r^2, d 8-6r^2), 20% fast spiking
# (a .02+.08r, b .25-.05r, c -65, d 2), in-degree 100 (100M synapses),
# excitatory w ~ U[0,6], inhibitory -U[0,5], BF16 storage, STDP A+ .1,
# A- .12, tau 20 ms, w in [0,10] on excitatory synapses, thalamic noise
# 5 N(0,1) / 2 N(0,1), dt 1 ms, 10 s.
# ---------------------------------------------------------------------------
def izh_c2(n=1_000_000, k=100, seed=44, threads=0, weight_format=A.WEIGHT_BF16):
    n_exc = int(round(0.8 * n))
    rp, col = topology(n, k, seed, threads)
    w, ty, pl = weights(A.GEN_W_UNIFORM, n, n_exc, rp, seed, 6.0, 5.0, plastic_exc=True,
                        threads=threads)
    rng = np.random.default_rng(seed)
    r = rng.random(n)
    exc = np.arange(n) < n_exc
    a = np.where(exc, 0.02, 0.02 + 0.08 * r)
    b = np.where(exc, 0.2, 0.25 - 0.05 * r)
    c = np.where(exc, -65.0 + 15.0 * r * r, -65.0)
    d = np.where(exc, 8.0 - 6.0 * r * r, 2.0)
    params = np.stack([a, b, c, d], axis=1).astype(np.float32)
    v0 = np.full(n, -65.0, np.float32)
    u0 = (params[:, 1] * v0).astype(np.float32)
    inh = (~exc).astype(np.uint8)
    net = Network(A.MODEL_IZHIKEVICH, params, rp, col, w, syn_type=ty, plastic=pl, v0=v0, u0=u0,
                  inhibitory=inh)
    cfg = SimConfig(model=A.MODEL_IZHIKEVICH, input_mode=A.INPUT_RESET_EACH_STEP, dt_ms=1.0,
                    delay_steps=1, seed=seed, weight_format=weight_format, stdp_enabled=True,
                    tau_plus=20.0, tau_minus=20.0, a_plus=0.1, a_minus=0.12, w_min=0.0,
                    w_max=10.0, homeostasis_enabled=False)
    drive = Drive(A.DRIVE_GAUSS, sigma_exc=5.0, sigma_inh=2.0)
    return net, cfg, drive, 10_000


# ---------------------------------------------------------------------------
# C4: Hodgkin-Huxley, 100,000 neurons, squid parameters, in-degree 100,
# AMPA (2 ms) / GABA-A (10 ms) conductance synapses, 80/20, g_syn ~
# lognormal(mu -3, sigma .5) nS, Rush-Larsen at dt .01 ms, Poisson
# conductance drive at 20 Hz, 1 s. The config leaves the membrane area open:
# HH_AREA_CM2 converts nS to mS/cm^2 (g[mS/cm^2] = g[nS] * 1e-6 / area), and
# the 20 Hz drive is K_EXT independent inputs, each event adding the mean
# synaptic conductance (one Bernoulli per neuron-step, p = K_EXT*20 Hz*dt).
# 5e-6 cm^2 (a 500 um^2 soma) gives an active asynchronous network of about
# 40 Hz; at 1e-5 cm^2 the same network is silent (measured on the oracle,
# 2000 neurons, 100 ms: 0 Hz at 1e-5, 13 Hz decaying at 6e-6, 40 Hz at 5e-6).
# ---------------------------------------------------------------------------
HH_AREA_CM2 = 5.0e-6
HH_K_EXT = 100
HH_DELAY_MS = 1.0


def hh_c4(n=100_000, k=100, seed=46, threads=0, integrator=A.HH_RUSH_LARSEN, dt_ms=0.01):
    n_exc = int(round(0.8 * n))
    rp, col = topology(n, k, seed, threads)
    scale = 1e-6 / HH_AREA_CM2
    w, ty, _ = weights(A.GEN_W_LOGNORMAL, n, n_exc, rp, seed, -3.0, 0.5, scale, threads=threads)
    params = np.tile(np.array([120.0, 36.0, 0.3, 50.0, -77.0, -54.4, 1.0], np.float32), (n, 1))
    inh = (np.arange(n) >= n_exc).astype(np.uint8)
    v0 = np.full(n, -65.0, np.float32)
    # gates at their steady state for -65 mV
    m0 = np.full(n, 0.0529, np.float32)
    h0 = np.full(n, 0.5961, np.float32)
    n0 = np.full(n, 0.3177, np.float32)
    net = Network(A.MODEL_HH, params, rp, col, w, syn_type=ty, v0=v0, m0=m0, h0=h0, n0=n0,
                  inhibitory=inh)
    delay = max(1, int(round(HH_DELAY_MS / dt_ms)))
    cfg = SimConfig(model=A.MODEL_HH, input_mode=A.INPUT_CONDUCTANCE_FRESH, hh_integrator=integrator,
                    dt_ms=dt_ms, delay_steps=delay, seed=seed, stdp_enabled=False,
                    homeostasis_enabled=False)
    g_mean = float(np.exp(-3.0 + 0.5 * 0.5 * 0.5) * scale)
    drive = Drive(A.DRIVE_POISSON_CONDUCTANCE, p=HH_K_EXT * 20.0 * dt_ms / 1000.0, amplitude=g_mean)
    return net, cfg, drive, int(round(1000.0 / dt_ms))


# ---------------------------------------------------------------------------
# C3: batched sweep, 256 independent LIF networks, sizes log-uniform in
# [2,000, 50,000], in-degree uniform in {50..200}, per network tau_m ~
# U[10,30] ms and inhibitory/excitatory weight ratio g ~ U[3,6]
# (w_exc = +0.5 mV, w_inh = -g * 0.5 mV, each x U[0.8,1.2] as in C1), 80/20,
# the C1 drive (Poisson 8 Hz, 0.8 mV kicks), 1 ms delay, V_rest -65 mV,
# dt 0.1 ms, 1000 steps. Network q is generated and driven from its own seed.
# ---------------------------------------------------------------------------
def lif_batch_c3(n_nets=256, seed=45, size_range=(2_000, 50_000), k_range=(50, 200), threads=0,
                 drive=None):
    rng = np.random.default_rng(seed)
    lo, hi = np.log(size_range[0]), np.log(size_range[1])
    sizes = np.exp(rng.uniform(lo, hi, n_nets)).astype(np.int64)
    ks = rng.integers(k_range[0], k_range[1] + 1, n_nets)
    taus = rng.uniform(10.0, 30.0, n_nets)
    gs = rng.uniform(3.0, 6.0, n_nets)
    nets, seeds = [], []
    for q in range(n_nets):
        n, k = int(sizes[q]), int(min(ks[q], sizes[q] - 1))
        sq = seed * 1_000_003 + q
        n_exc = int(round(0.8 * n))
        rp, col = topology(n, k, sq, threads)
        w, ty, _ = weights(A.GEN_W_SCALED, n, n_exc, rp, sq, 0.5, -float(gs[q]) * 0.5, 0.8, 1.2,
                           threads=threads)
        params = np.tile(np.array([-65.0, -50.0, -65.0, float(taus[q]), 2.0, 1.0], np.float32),
                         (n, 1))
        inh = (np.arange(n) >= n_exc).astype(np.uint8)
        nets.append(Network(A.MODEL_LIF, params, rp, col, w, syn_type=ty, inhibitory=inh))
        seeds.append(sq)
    cfg = SimConfig(model=A.MODEL_LIF, input_mode=A.INPUT_DELTA_V, dt_ms=0.1, delay_steps=10,
                    seed=seed, stdp_enabled=False, homeostasis_enabled=False)
    drive = drive or Drive(A.DRIVE_POISSON_KICK, p=8.0 * 0.1 / 1000.0, amplitude=0.8)
    return nets, seeds, cfg, drive, 1000
