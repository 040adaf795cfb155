"""Learned Hodgkin-Huxley macro-step (include/neuralsim_surrogate.h).

An MLP 5 -> 128 -> 128 -> 4 (SiLU, BF16 weights, FP32 accumulation on the
tensor cores) advances (V, m, h, n) of a neuron over a 0.1 ms macro-step
given the synaptic current held for that macro-step; it replaces ten
Rush-Larsen steps of 0.01 ms of HodgkinHuxleyNeuron::step
(src/neuron/hodgkin_huxley.rs:46-96). Training data are states sampled from
plain Rush-Larsen network runs; targets are computed on the device with the
network's own Rush-Larsen arithmetic; training runs on the device with the
library's forward and backward kernels.
"""
import ctypes as C

import numpy as np

from . import _abi as A

SQUID = (120.0, 36.0, 0.3, 50.0, -77.0, -54.4, 1.0)
# synapse constants (decay tau ms, reversal mV) of AMPA, GABA_A, GABA_B, NMDA
SYN_TAU = np.array([2.0, 10.0, 150.0, 100.0])
SYN_EREV = np.array([0.0, -70.0, -90.0, 0.0])
SUBSTEPS = 10
N_PARAMS = 17796
# default training envelope of V (mV) and residual tolerance (mV)
V_LO, V_HI, RESIDUAL_MV = -85.0, -52.0, 0.5
# default upper bound of V for the macro-step: above it, on the approach to
# threshold where a small error moves a spike most, the plain Rush-Larsen
# steps take over (C4 network: mean spike-time error 0.09 ms at -58 mV,
# 0.20 ms at -55 mV, 0.14-0.25 ms at the training bound -52 mV)
MACRO_V_HI = -58.0


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _hh_rates(v):
    x = (v + 40.0) / 10.0
    xs = np.where(x == 0.0, 1.0, x)
    am = np.where(x == 0.0, 1.0, xs / (-np.expm1(-xs)))
    bm = 4.0 * np.exp(-(v + 65.0) / 18.0)
    ah = 0.07 * np.exp(-(v + 65.0) / 20.0)
    bh = 1.0 / (1.0 + np.exp(-(v + 35.0) / 10.0))
    y = (v + 55.0) / 10.0
    ys = np.where(y == 0.0, 1.0, y)
    an = np.where(y == 0.0, 0.1, 0.1 * ys / (-np.expm1(-ys)))
    bn = 0.125 * np.exp(-(v + 65.0) / 80.0)
    return am, bm, ah, bh, an, bn


def coarse_base(x, hh_params, dt_macro):
    """One Rush-Larsen step of the macro-step's length with the current held:
    the base whose correction the MLP predicts. x [n][5] -> [n][4]."""
    x = np.asarray(x, np.float64)
    v, m, h, n, I = (x[:, k] for k in range(5))
    gna, gk, gl, ena, ek, el, cm = hh_params
    am, bm, ah, bh, an, bn = _hh_rates(v)
    sm, sh, sn = am + bm, ah + bh, an + bn
    m = am / sm + (m - am / sm) * np.exp(-dt_macro * sm)
    h = ah / sh + (h - ah / sh) * np.exp(-dt_macro * sh)
    n = an / sn + (n - an / sn) * np.exp(-dt_macro * sn)
    iion = gna * m ** 3 * h * (v - ena) + gk * n ** 4 * (v - ek) + gl * (v - el)
    return np.stack([v + dt_macro * (I - iion) / cm, m, h, n], 1)


def macro_current(G, v, dt_fine):
    """Synaptic current held over a macro-step of SUBSTEPS fine steps: the
    mean of each decaying conductance over the macro-step times its driving
    force at the start. G [4][n] (conductances at the start), v [n]."""
    d = np.exp(-dt_fine / SYN_TAU)
    gd = np.asarray(G, np.float64) * d[:, None]
    mean = gd * ((1.0 - d ** SUBSTEPS) / (SUBSTEPS * (1.0 - d)))[:, None]
    return (mean * (SYN_EREV[:, None] - np.asarray(v, np.float64)[None, :])).sum(0)


class Surrogate:
    """One trained (or training) surrogate on one GPU."""

    def __init__(self, hh_params=SQUID, dt_fine=0.01, batch=8192, seed=46, device=0):
        self.lib = A.load()
        self.dt_fine = float(dt_fine)
        self.batch = int(batch)
        self._h = C.c_void_p()
        hp = np.asarray(hh_params, np.float32)
        self.hh_params = tuple(float(q) for q in hp)
        st = self.lib.ns_sur_create(int(device), _p(hp), float(dt_fine), self.batch, int(seed),
                                    C.byref(self._h))
        if st != A.NS_OK:
            raise A.NsError(st, (self.lib.ns_sur_last_error(None) or b"").decode())
        self.norm = None

    def _check(self, st):
        if st != A.NS_OK:
            raise A.NsError(st, (self.lib.ns_sur_last_error(self._h) or b"").decode())

    def set_data(self, x):
        """Training states x [n][5] = (V, m, h, n, I_syn); returns the device
        targets [n][4] (the states 0.1 ms later)."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((len(x), 4), np.float32)
        self._check(self.lib.ns_sur_set_data(self._h, _p(x), len(x), _p(y)))
        return y

    def set_norm(self, in_mean, in_scale, out_mean, out_scale):
        self.norm = {k: np.ascontiguousarray(v, np.float32) for k, v in
                     (("in_mean", in_mean), ("in_scale", in_scale), ("out_mean", out_mean),
                      ("out_scale", out_scale))}
        n = self.norm
        self._check(self.lib.ns_sur_set_norm(self._h, _p(n["in_mean"]), _p(n["in_scale"]),
                                             _p(n["out_mean"]), _p(n["out_scale"])))

    def fit_norm(self, x, y):
        """Normalisation from a training set: inputs to zero mean / unit
        scale, the corrections to the coarse base step likewise."""
        x = np.asarray(x, np.float64)
        dy = np.asarray(y, np.float64) - coarse_base(x, self.hh_params, SUBSTEPS * self.dt_fine)
        self.set_norm(x.mean(0), np.maximum(x.std(0), 1e-6), dy.mean(0), np.maximum(dy.std(0), 1e-9))

    def train(self, steps, lr=2e-3, lr_decay=None, lr_final=1e-4):
        """Adam steps on device minibatches; returns the per-step losses."""
        if lr_decay is None:
            lr_decay = (lr_final / lr) ** (1.0 / max(steps, 1))
        loss = np.zeros(max(int(steps), 1), np.float32)
        self._check(self.lib.ns_sur_train(self._h, int(steps), float(lr), float(lr_decay), _p(loss)))
        return loss[:steps]

    def gradient(self, x, y):
        """(flat gradient, loss) of one batch of raw states and targets."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        if len(x) != self.batch or len(y) != self.batch:
            raise ValueError("gradient takes exactly one batch")
        g = np.zeros(N_PARAMS, np.float32)
        l = np.zeros(1, np.float32)
        self._check(self.lib.ns_sur_gradient(self._h, _p(x), _p(y), _p(g), _p(l)))
        return g, float(l[0])

    def set_sample_seed(self, seed):
        self._check(self.lib.ns_sur_set_sample_seed(self._h, int(seed)))

    def grad_step(self, grad):
        """Gradient of one sampled minibatch into `grad` (a CUDA float32
        tensor of N_PARAMS values); returns the minibatch loss."""
        l = np.zeros(1, np.float32)
        self._check(self.lib.ns_sur_grad_step(self._h, C.c_void_p(grad.data_ptr()), _p(l)))
        return float(l[0])

    def apply_gradient(self, grad, scale, lr):
        """One Adam step with scale * grad (a CUDA float32 tensor)."""
        self._check(self.lib.ns_sur_apply_gradient(self._h, C.c_void_p(grad.data_ptr()),
                                                   float(scale), float(lr)))

    @property
    def params(self):
        p = np.zeros(N_PARAMS, np.float32)
        self._check(self.lib.ns_sur_get_params(self._h, _p(p)))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._check(self.lib.ns_sur_set_params(self._h, _p(p)))

    def predict(self, x):
        """Raw states 0.1 ms later for x [n][5] (through the training GEMMs)."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((len(x), 4), np.float32)
        self._check(self.lib.ns_sur_predict(self._h, _p(x), len(x), _p(y)))
        return y

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            self.lib.ns_sur_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sample_states(engine, n_snapshots, every_steps, rng=None, per_snapshot=None):
    """States (V, m, h, n, I_syn) of a running plain HH engine: every
    `every_steps` steps, all neurons (or `per_snapshot` of them)."""
    rng = rng or np.random.default_rng(0)
    out = []
    for _ in range(n_snapshots):
        engine.run(every_steps)
        st = engine.download_state(with_weights=False)
        n = len(st["v"])
        G = st["conductance"].reshape(4, n)
        isyn = macro_current(G, st["v"], engine.config.dt_ms)
        x = np.stack([st["v"], st["hh_m"], st["hh_h"], st["hh_n"], isyn], 1).astype(np.float32)
        if per_snapshot is not None and per_snapshot < n:
            x = x[rng.choice(n, per_snapshot, replace=False)]
        out.append(x)
    return np.concatenate(out)


def train_for_network(net, cfg, drive, warm_steps=2000, snapshots=100, every_steps=50,
                      v_lo=V_LO, v_hi=V_HI, margin=3.0, batch=8192, steps=4000, lr=2e-3,
                      seed=46, per_snapshot=None, focus_v=-62.0, focus_repeat=4):
    """Samples states from a plain Rush-Larsen run of the network (after
    warm_steps), keeps those with V within the envelope (plus a margin),
    computes their targets on the device and trains a surrogate. States with
    V above focus_v (the approach to threshold, where an error moves a spike
    time most) enter the training set focus_repeat times. The network's
    neurons share one HH parameter row (the first neuron's). Returns
    (surrogate, states, targets, losses)."""
    from .engine import SimulationEngine
    eng = SimulationEngine(net, cfg, drive)
    try:
        eng.run(warm_steps)
        x = sample_states(eng, snapshots, every_steps, per_snapshot=per_snapshot)
    finally:
        eng.close()
    keep = (x[:, 0] >= v_lo - margin) & (x[:, 0] <= v_hi + margin)
    x = x[keep]
    if focus_repeat > 1:
        near = x[x[:, 0] > focus_v]
        x = np.concatenate([x] + [near] * (focus_repeat - 1))
    sur = Surrogate(hh_params=net.params[0], dt_fine=cfg.dt_ms, batch=batch, seed=seed,
                    device=cfg.device)
    y = sur.set_data(x)
    sur.fit_norm(x, y)
    losses = sur.train(steps, lr)
    return sur, x, y, losses


def train_data_parallel(sur, steps, lr=2e-3, lr_final=1e-4, rank=0, world=1, group=None,
                        grad=None):
    """Data-parallel training, one process per GPU: every rank computes the
    gradient of its own minibatch, one all-reduce (sum) of the 17,796 FP32
    gradients averages them, and every rank takes the same Adam step. The
    ranks must hold the same weights before the first step (broadcast from
    rank 0 here) and sample from distinct streams. Returns the mean loss of
    every step over the ranks. `grad`: the gradient buffer (a CUDA tensor);
    allocated here when None."""
    import torch
    if grad is None:
        grad = torch.zeros(N_PARAMS, dtype=torch.float32, device="cuda")
    dist = None
    if world > 1:
        import torch.distributed as dist
        p = torch.from_numpy(sur.params).to(grad.device)
        dist.broadcast(p, 0, group=group)
        sur.params = p.cpu().numpy()
    decay = (lr_final / lr) ** (1.0 / max(steps, 1))
    losses = np.zeros(steps, np.float64)
    l_t = torch.zeros(1, dtype=torch.float64, device=grad.device)
    for q in range(steps):
        loss = sur.grad_step(grad)
        if dist is not None:
            dist.all_reduce(grad, group=group)
            l_t.fill_(loss)
            dist.all_reduce(l_t, group=group)
            loss = float(l_t.item())
        sur.apply_gradient(grad, 1.0 / world, lr * decay ** q)
        losses[q] = loss / world
    return losses


def tc_gemm(A_, B_, C_=None, H_=None, bias=None, splits=1, epilogue=0, stream=None):
    """Tensor-core GEMM on torch tensors (bf16 A [M][K], B [N][K]; fp32 C;
    bf16 H): C = A B^T by the library's tcgen05 kernel."""
    lib = A.load()
    M, K = A_.shape
    N = B_.shape[0]

    def ptr(t):
        return None if t is None else C.c_void_p(t.data_ptr())
    ldc = C_.shape[1] if C_ is not None else N
    st = lib.ns_tc_gemm_bf16(ptr(A_), ptr(B_), ptr(C_), ptr(H_), ptr(bias), M, N, K, A_.stride(0),
                             B_.stride(0), ldc, splits, epilogue,
                             None if stream is None else C.c_void_p(stream))
    if st != A.NS_OK:
        raise A.NsError(st, (lib.ns_sur_last_error(None) or b"").decode())
