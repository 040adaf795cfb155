"""ORACLE — test infrastructure only. FP64 restatement of the surrogate MLP
(5 -> 128 -> 128 -> 4, SiLU) and of its training loss and gradient, and an
FP64 Rush-Larsen integrator of the Hodgkin-Huxley neuron
(src/neuron/hodgkin_huxley.rs:20-42 rates; Rush-Larsen gates, Euler V), for
checking the device's tensor-core forward / backward kernels and its
training targets. Parameter layout (flat, 17,796): W1 [128][5], b1 [128],
W2 [128][128], b2 [128], W3 [4][128], b3 [4]."""
import numpy as np

H = 128
SIZES = [("W1", (H, 5)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (4, H)), ("b3", (4,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SIZES])


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s + z * s * (1.0 - s)


def normalise(x, y, norm, base):
    """Normalised inputs and (if y is given) normalised targets: the state
    0.1 ms later minus `base` (one Rush-Larsen step of 0.1 ms)."""
    x = np.asarray(x, np.float64)
    xn = (x - norm["in_mean"]) / norm["in_scale"]
    tn = None
    if y is not None:
        tn = ((np.asarray(y, np.float64) - base) - norm["out_mean"]) / norm["out_scale"]
    return xn, tn


def forward(p, xn):
    w = unpack(p)
    z1 = xn @ w["W1"].T + w["b1"]
    h1 = silu(z1)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = silu(z2)
    y = h2 @ w["W3"].T + w["b3"]
    return y, (z1, h1, z2, h2)


def loss_and_grad(p, xn, tn):
    """Mean over rows and the 4 outputs of the squared error, and its
    gradient in the flat parameter order."""
    w = unpack(p)
    y, (z1, h1, z2, h2) = forward(p, xn)
    B = xn.shape[0]
    e = y - tn
    loss = float(np.mean(e * e))
    dy = 2.0 * e / (4.0 * B)
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dz2 = (dy @ w["W3"]) * dsilu(z2)
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = (dz2 @ w["W2"]) * dsilu(z1)
    g["W1"], g["b1"] = dz1.T @ xn, dz1.sum(0)
    return loss, pack(g)


def hh_rates(v):
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


def rush_larsen(x, p, dt, steps):
    """x [n][5] = (V, m, h, n, I) -> [n][4] after `steps` Rush-Larsen steps
    with I held; p = (g_na, g_k, g_l, e_na, e_k, e_l, c_m)."""
    v, m, h, n, I = (np.asarray(x[:, k], np.float64).copy() for k in range(5))
    gna, gk, gl, ena, ek, el, cm = p
    for _ in range(steps):
        am, bm, ah, bh, an, bn = hh_rates(v)
        sm, sh, sn = am + bm, ah + bh, an + bn
        m = am / sm + (m - am / sm) * np.exp(-dt * sm)
        h = ah / sh + (h - ah / sh) * np.exp(-dt * sh)
        n = an / sn + (n - an / sn) * np.exp(-dt * sn)
        iion = gna * m ** 3 * h * (v - ena) + gk * n ** 4 * (v - ek) + gl * (v - el)
        v = v + dt * (I - iion) / cm
    return np.stack([v, m, h, n], 1)
