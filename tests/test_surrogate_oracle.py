"""The FP64 surrogate oracle (oracle/surrogate_oracle.py) pinned on its own:
its backpropagated gradient against central finite differences, its
Rush-Larsen integrator against the known answers of the HH neuron, and the
held synaptic current of a macro-step against its definition."""
import numpy as np

from oracle import surrogate_oracle as so
from neuralsim_b200 import surrogate as S


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0.0, 0.2, so.N_PARAMS)
    xn = rng.normal(size=(16, 5))
    tn = rng.normal(size=(16, 4))
    _, g = so.loss_and_grad(p, xn, tn)
    idx = rng.choice(so.N_PARAMS, 40, replace=False)
    idx = np.concatenate([idx, [0, 639, 640, 767, 17151, 17152, 17279, 17280, 17791, 17795]])
    h = 1e-6
    for q in idx:
        e = np.zeros(so.N_PARAMS)
        e[q] = h
        fd = (so.loss_and_grad(p + e, xn, tn)[0] - so.loss_and_grad(p - e, xn, tn)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g[q])), (q, fd, g[q])


def test_oracle_rush_larsen_rest_and_firing():
    # hodgkin_huxley.rs:122-163: rest within 1 mV without input; fires with I = 10
    x = np.array([[-65.0, 0.0529, 0.5961, 0.3177, 0.0]])
    y = so.rush_larsen(x, S.SQUID, 0.01, 1000)
    assert abs(y[0, 0] - (-65.0)) < 1.0
    v, fired = x.copy(), False
    v[0, 4] = 10.0
    for _ in range(500):
        y = so.rush_larsen(v, S.SQUID, 0.01, 1)
        if v[0, 0] < 0.0 <= y[0, 0]:
            fired = True
        v[0, :4] = y[0]
    assert fired


def test_macro_current_is_mean_of_decaying_conductance():
    rng = np.random.default_rng(5)
    G = rng.random((4, 7))
    v = rng.uniform(-80, -50, 7)
    dt = 0.01
    d = np.exp(-dt / S.SYN_TAU)
    mean = np.mean([G * (d ** (s + 1))[:, None] for s in range(S.SUBSTEPS)], axis=0)
    want = (mean * (S.SYN_EREV[:, None] - v[None, :])).sum(0)
    assert np.allclose(S.macro_current(G, v, dt), want, rtol=1e-12, atol=1e-12)
