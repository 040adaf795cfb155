"""The learned HH macro-step on the GPU.

- tcgen05 BF16 GEMM against torch FP32 matmul of the same BF16 values
  (fp32 accumulation: rtol 1e-4, atol 1e-3; bias + SiLU epilogue: the SiLU
  output is BF16, rtol/atol 1e-2);
- training targets (10 Rush-Larsen steps on the device) against the FP64
  integrator: 2e-3 mV for V, 2e-5 for the gates;
- backward kernels: the device gradient against the FP64 oracle's on the
  same batch and weights, per tensor relative L2 error < 3e-2 and cosine
  similarity > 0.999 (BF16 operands and activations on the device);
- training reduces the loss by 20x;
- the fused macro-step kernel of the network step against the GEMM
  inference path on the same states (same BF16 weights): 1e-3 mV / 1e-5;
- the network: surrogate spike times against the plain run (reported, with
  the coarse Rush-Larsen comparison mode as the method in the same cost
  class).
"""
import numpy as np
import pytest

from neuralsim_b200 import _abi as A
from neuralsim_b200 import surrogate as S
from neuralsim_b200 import SimulationEngine
from neuralsim_b200.engine import Drive
from oracle import surrogate_oracle as so
import nets as tnets

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("M,N,K,splits,epi", [
    (128, 128, 16, 1, 0), (256, 128, 128, 1, 0), (256, 16, 128, 1, 0), (384, 16, 16, 1, 0),
    (128, 128, 1024, 8, 1), (128, 16, 512, 4, 1), (256, 128, 128, 1, 2), (128, 128, 48, 1, 0)])
def test_tc_gemm_matches_fp32(lib, M, N, K, splits, epi):
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N * 3 + K)
    Af = torch.randn(M, K, generator=g)
    Bf = torch.randn(N, K, generator=g)
    Ab, Bb = Af.bfloat16().cuda(), Bf.bfloat16().cuda()
    ref = Ab.float() @ Bb.float().T
    C = torch.zeros(M, N, device="cuda")
    if epi == 2:
        bias = torch.randn(N, generator=g).cuda()
        H = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
        S.tc_gemm(Ab, Bb, C, H, bias, 1, 2)
        torch.cuda.synchronize()
        z = ref + bias
        assert torch.allclose(C, z, rtol=1e-4, atol=1e-3)
        assert torch.allclose(H.float(), torch.nn.functional.silu(z), rtol=1e-2, atol=1e-2)
    else:
        S.tc_gemm(Ab, Bb, C, None, None, splits, epi)
        torch.cuda.synchronize()
        assert torch.allclose(C, ref, rtol=1e-4, atol=1e-3), (C - ref).abs().max()


def random_states(n, rng):
    v = rng.uniform(-85.0, -50.0, n)
    am, bm, ah, bh, an, bn = so.hh_rates(v)
    m = np.clip(am / (am + bm) + rng.normal(0, 0.02, n), 0.02, 0.98)
    h = np.clip(ah / (ah + bh) + rng.normal(0, 0.05, n), 0.02, 0.98)
    nn = np.clip(an / (an + bn) + rng.normal(0, 0.05, n), 0.02, 0.98)
    I = rng.uniform(-10.0, 30.0, n)
    return np.stack([v, m, h, nn, I], 1).astype(np.float32)


def test_targets_match_fp64_rush_larsen(lib):
    rng = np.random.default_rng(1)
    x = random_states(20_000, rng)
    s = S.Surrogate(batch=1024)
    y = s.set_data(x)
    want = so.rush_larsen(x.astype(np.float64), S.SQUID, 0.01, 10)
    assert np.abs(y[:, 0] - want[:, 0]).max() < 2e-3
    assert np.abs(y[:, 1:] - want[:, 1:]).max() < 2e-5
    s.close()


def test_gradient_matches_fp64_oracle(lib):
    rng = np.random.default_rng(2)
    s = S.Surrogate(batch=1024, seed=7)
    x = random_states(1024, rng)
    y = s.set_data(x)
    s.fit_norm(x, y)
    g, loss = s.gradient(x, y)
    nm = {k: v.astype(np.float64) for k, v in s.norm.items()}
    base = so.rush_larsen(x.astype(np.float64), S.SQUID, 0.1, 1)
    xn, tn = so.normalise(x, y, nm, base)
    want_loss, want = so.loss_and_grad(s.params.astype(np.float64), xn, tn)
    assert abs(loss - want_loss) <= 0.02 * want_loss
    o = 0
    for name, shape in so.SIZES:
        k = int(np.prod(shape))
        a, b = g[o:o + k].astype(np.float64), want[o:o + k]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
        assert rel < 3e-2 and cos > 0.999, (name, rel, cos)
        o += k
    s.close()


def test_training_reduces_loss(lib):
    rng = np.random.default_rng(3)
    x = random_states(200_000, rng)
    s = S.Surrogate(batch=4096, seed=11)
    y = s.set_data(x)
    s.fit_norm(x, y)
    losses = s.train(1500, lr=2e-3)
    assert np.all(np.isfinite(losses))
    assert losses[-50:].mean() < losses[:10].mean() / 20
    xt = random_states(8192, np.random.default_rng(4))
    yt = s.set_data(xt)          # targets of held-out states
    pred = s.predict(xt)
    dv = yt[:, 0] - xt[:, 0]
    err = pred[:, 0] - yt[:, 0]
    assert np.sqrt(np.mean(err ** 2)) < 0.2 * dv.std()
    s.close()


def test_fused_macro_step_matches_gemm_inference(lib):
    # states in the envelope, no synaptic input, no drive: one macro-step of
    # the network kernel equals the surrogate's GEMM inference
    rng = np.random.default_rng(5)
    n = 1000
    x = random_states(n, rng)
    x[:, 4] = 0.0
    net, cfg, _ = tnets.hh_cond(n=n, k=20)
    net.v0, net.m0, net.h0, net.n0 = (np.ascontiguousarray(x[:, q]) for q in range(4))
    s = S.Surrogate(batch=1024, seed=13)
    s.set_norm(np.zeros(5), np.full(5, 10.0), np.zeros(4), np.full(4, 1e-3))
    eng = SimulationEngine(net, cfg, Drive())
    eng.attach_surrogate(s, v_lo=-100.0, v_hi=0.0, residual_mv=1e9)
    eng.run(10)
    mlp, fb = eng.surrogate_counts()
    assert mlp == n and fb == 0
    st = eng.download_state(with_weights=False)
    want = s.predict(x)
    assert np.abs(st["v"] - want[:, 0]).max() < 1e-3
    for q, k in ((1, "hh_m"), (2, "hh_h"), (3, "hh_n")):
        assert np.abs(st[k] - want[:, q]).max() < 1e-5
    eng.close()
    s.close()


def test_network_spike_times_against_plain(lib):
    # HH network of the C4 shape (2,000 neurons): surrogate trained on the
    # plain run's states; spikes matched nearest within 2 ms to the plain
    # run over 50 ms. The surrogate's mean |dt| must not exceed that of one
    # Rush-Larsen step of 0.1 ms in the same macro-step scheme.
    net, cfg, drive = tnets.hh_cond(n=2000, k=50)
    cfg.window_steps = 100
    sur, x, y, losses = S.train_for_network(net, cfg, drive, warm_steps=2000, snapshots=60,
                                            every_steps=50, batch=8192, steps=6000)
    steps = 5000
    res = {}
    for mode in ("plain", "surrogate", "coarse", "held"):
        eng = SimulationEngine(net, cfg, drive)
        if mode != "plain":
            eng.attach_surrogate(sur)
            if mode != "surrogate":
                eng.macro_step_mode(1 if mode == "coarse" else 2)
        eng.run(steps)
        res[mode] = eng.read_raster(0, steps)
        if mode != "plain":
            res[mode + "_counts"] = eng.surrogate_counts()
        eng.close()
    w = int(round(2.0 / cfg.dt_ms))
    ds, ua, ub = tnets.match_spikes(res["plain"], res["surrogate"], w)
    dc, uca, ucb = tnets.match_spikes(res["plain"], res["coarse"], w)
    n_plain = len(res["plain"][0])
    assert n_plain > 500
    err_s = ds.mean() * cfg.dt_ms
    err_c = dc.mean() * cfg.dt_ms if len(dc) else np.inf
    dh, uha, uhb = tnets.match_spikes(res["plain"], res["held"], w)
    print("surrogate", err_s, ua, ub, res["surrogate_counts"], "coarse", err_c, uca, ucb,
          "held-current RL", dh.mean() * cfg.dt_ms, uha, uhb)
    assert res["surrogate_counts"][0] > 0
    assert err_s <= 0.2
    assert err_s <= err_c
    sur.close()
