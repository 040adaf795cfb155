"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Bit-exact: spike rasters, CSR traversal order, LIF/Izhikevich state and BF16
weights against the float oracle (int64 fixed-point sums make the result
independent of event order). Tolerance (stated per test): FP64 comparisons,
HH (expf on the device) and homeostasis (per-synapse expf).
"""
import numpy as np
import pytest

from oracle.oracle import FastOracle, LiteralOracle
from neuralsim_b200 import _abi as A
from neuralsim_b200 import SimulationEngine, NsError
from neuralsim_b200.engine import Drive, Network, SimConfig
import nets

pytestmark = pytest.mark.gpu


def gpu_run(net, cfg, drive, steps):
    eng = SimulationEngine(net, cfg, drive)
    eng.run(steps)
    return eng


def test_c1_lif_raster_bit_exact_1s(lib):
    # config C1 at full size: 10k LIF, 1M synapses, dt 0.1 ms, 10 ms..1 s
    from neuralsim_b200 import configs
    net, cfg, drive, steps = configs.lif_c1()
    cfg.spike_log_capacity, cfg.spike_log_steps = 20_000_000, steps
    eng = gpu_run(net, cfg, drive, steps)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(steps)
    assert nets.rasters_equal(eng.read_raster(0, steps), o.raster())
    st = eng.download_state()
    assert np.array_equal(st["v"].astype(np.float64), o.state()["v"])
    assert np.array_equal(st["refractory"], o.state()["refr"])


def test_lif_delta_active_raster_bit_exact(lib):
    net, cfg, drive = nets.lif_delta(n=5000, k=80)
    eng = gpu_run(net, cfg, drive, 3000)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(3000)
    ra, rb = eng.read_raster(0, 3000), o.raster()
    assert len(rb[0]) > 10_000
    assert nets.rasters_equal(ra, rb)
    assert np.array_equal(eng.download_state()["v"].astype(np.float64), o.state()["v"])


@pytest.mark.parametrize("wf", [A.WEIGHT_BF16, A.WEIGHT_F32])
def test_izh_stdp_raster_weights_bit_exact_1s(lib, wf):
    # Izhikevich + pair STDP, C2 shape at 20k neurons / 2M synapses, 1 s
    net, cfg, drive = nets.izh_stdp(n=20_000, k=100, wf=wf)
    eng = gpu_run(net, cfg, drive, 1000)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(1000)
    ra, rb = eng.read_raster(0, 1000), o.raster()
    assert len(rb[0]) > 50_000
    assert nets.rasters_equal(ra, rb)
    st, so = eng.download_state(), o.state()
    assert np.array_equal(st["v"].astype(np.float64), so["v"])
    assert np.array_equal(st["u"].astype(np.float64), so["u"])
    assert np.array_equal(st["pre_trace"].astype(np.float64), so["pre"])
    assert np.array_equal(st["post_trace"].astype(np.float64), so["post"])
    assert np.array_equal(st["w"].astype(np.float64), o.weights())
    assert np.count_nonzero(st["w"] != net.w) > 1000


@pytest.mark.parametrize("distinct_rows", [2, 5000])
def test_parameter_rows_dictionary_and_per_neuron(lib, distinct_rows):
    # up to 256 distinct parameter rows: the neuron kernel reads a 1-byte
    # index and a shared-memory table; more rows: the per-neuron arrays.
    # Both give the oracle's results bit for bit.
    net, cfg, drive = nets.izh_stdp(n=20_000, k=60, wf=A.WEIGHT_F32)
    if distinct_rows > 256:
        rng = np.random.default_rng(11)
        p = net.params.copy()
        p[:, 2] = p[:, 2] + rng.uniform(-2.0, 2.0, net.n).astype(np.float32)   # reset c
        net.params = p
    assert len(np.unique(net.params, axis=0)) >= min(distinct_rows, 2)
    eng = gpu_run(net, cfg, drive, 400)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(400)
    assert nets.rasters_equal(eng.read_raster(0, 400), o.raster())
    st = eng.download_state()
    assert np.array_equal(st["v"].astype(np.float64), o.state()["v"])
    assert np.array_equal(st["params"], net.params)


@pytest.mark.parametrize("sched", [1, 2, 3, 4, 5])
def test_step_schedules_identical(lib, sched):
    # fused, split (LTD beside the next neuron update) and fused-4 schedules
    # compute the same step: rasters and BF16 weights bit-identical to the oracle
    net, cfg, drive = nets.izh_stdp(n=30_000, k=100)
    cfg.step_schedule = sched
    cfg.graph_chunk = 100
    eng = gpu_run(net, cfg, drive, 350)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(350)
    assert eng.schedule()[0] == sched
    assert nets.rasters_equal(eng.read_raster(0, 350), o.raster())
    assert np.array_equal(eng.download_state()["w"].astype(np.float64), o.weights())


def test_autotuner_picks_a_schedule(lib):
    net, cfg, drive = nets.izh_stdp(n=30_000, k=100)
    eng = gpu_run(net, cfg, drive, 700)
    sched, us = eng.schedule()
    assert sched in (1, 2, 3, 4, 5) and all(v > 0 for v in us.values()) and len(us) == 5
    assert us[sched] == min(us.values())
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(700)
    assert nets.rasters_equal(eng.read_raster(0, 700), o.raster())


@pytest.mark.parametrize("family", ["lif", "hh"])
def test_windowed_equals_step_path(lib, family):
    # windows of W = delay steps (with a partial window at the end) give the
    # step-synchronous results bit for bit
    if family == "lif":
        net, cfg, drive = nets.lif_delta(n=5000, k=80)
        steps = 1234
    else:
        net, cfg, drive = nets.hh_cond(n=3000, k=50)
        steps = 777
    cfg.graph_chunk = 500
    out = []
    for wsteps in (0, 1):
        cfg.window_steps = wsteps
        eng = gpu_run(net, cfg, drive, steps)
        st = eng.download_state(with_weights=False)
        out.append((eng.read_raster(0, steps), st, eng.counters()))
        eng.close()
    assert len(out[0][0][0]) > 100
    assert nets.rasters_equal(out[0][0], out[1][0])
    for key in ("v", "u", "refractory", "hh_m", "hh_h", "hh_n", "conductance", "pending_input"):
        assert np.array_equal(out[0][1][key], out[1][1][key]), key
    assert out[0][2] == out[1][2]


def test_windowed_checkpoint_and_traced_steps(lib):
    net, cfg, drive = nets.lif_delta(n=5000, k=80)
    a = gpu_run(net, cfg, drive, 400)
    full = (a.read_raster(200, 200), a.download_state(with_weights=False))
    b = gpu_run(net, cfg, drive, 200)
    snap = b.download_state()
    c = SimulationEngine(net, cfg, drive)
    c.upload_state(snap, 200)
    c.run(200)
    assert nets.rasters_equal(c.read_raster(200, 200), full[0])
    assert np.array_equal(c.download_state(with_weights=False)["v"], full[1]["v"])
    # traced (step-synchronous) steps interleaved with windows
    d = SimulationEngine(net, cfg, drive)
    d.run(95)
    d.step_traced(10_000_000)
    d.step_traced(10_000_000)
    d.run(103)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(200)
    assert nets.rasters_equal(d.read_raster(0, 200), o.raster())


def test_csr_traversal_order_bit_exact(lib):
    net, cfg, drive = nets.izh_stdp(n=8000, k=60)
    eng = SimulationEngine(net, cfg, drive)
    o = FastOracle(net, cfg, drive, precision=32)
    eng.run(20)
    o.step(20)
    for _ in range(3):
        pg, ng = eng.step_traced(2_000_000)
        po, no = o.step_traced(2_000_000)
        assert ng == no and ng > 0
        assert np.array_equal(pg, po)


def test_spike_lists_ascending_and_counts(lib):
    net, cfg, drive = nets.izh_stdp(n=30_000, k=50)
    eng = SimulationEngine(net, cfg, drive)
    out = eng.run(200)
    idx, off = eng.read_raster(0, 200)
    assert out.spikes == len(idx)
    deg = np.diff(net.row_ptr.astype(np.int64))
    assert out.events == int(deg[idx].sum())
    for q in range(200):
        s = idx[int(off[q]):int(off[q + 1])].astype(np.int64)
        assert np.all(np.diff(s) > 0)


FLOOR = {"v": 10.0, "u": 1.0, "hh_m": 1.0, "hh_h": 1.0, "hh_n": 1.0}
OKEY = {"v": "v", "u": "u", "hh_m": "m", "hh_h": "h", "hh_n": "n"}


def test_izh_one_step_within_1e5_of_fp64(lib):
    # per-step state from widely spread states: |gpu - fp64| <= 1e-5 max(|fp64|, floor)
    net, cfg, drive = nets.izh_stdp(n=20_000, k=20, wf=A.WEIGHT_F32)
    rng = np.random.default_rng(3)
    net.v0 = rng.uniform(-80, 29, net.n).astype(np.float32)
    net.u0 = rng.uniform(-20, 10, net.n).astype(np.float32)
    eng = gpu_run(net, cfg, drive, 1)
    o = FastOracle(net, cfg, drive, precision=64)
    o.step(1)
    st, so = eng.download_state(), o.state()
    for k in ("v", "u"):
        err = np.abs(st[k] - so[OKEY[k]]) / np.maximum(np.abs(so[OKEY[k]]), FLOOR[k])
        assert err.max() < 1e-5, (k, err.max())


def test_hh_one_step_within_1e5_of_fp64(lib):
    net, cfg, drive = nets.hh_cond(n=20_000, k=20)
    rng = np.random.default_rng(4)
    net.v0 = rng.uniform(-80, 30, net.n).astype(np.float32)
    for g in ("m0", "h0", "n0"):
        setattr(net, g, rng.uniform(0, 1, net.n).astype(np.float32))
    eng = gpu_run(net, cfg, drive, 1)
    o = FastOracle(net, cfg, drive, precision=64)
    o.step(1)
    st, so = eng.download_state(), o.state()
    for k in ("v", "hh_m", "hh_h", "hh_n"):
        err = np.abs(st[k] - so[OKEY[k]]) / np.maximum(np.abs(so[OKEY[k]]), FLOOR[k])
        assert err.max() < 1e-5, (k, err.max())


def test_hh_rush_larsen_network_tracks_fp64(lib):
    # 5 ms of the C4 network shape: spike trains equal to the FP64 oracle's
    # (upward 0 mV crossings). State within 1e-2 of max(|x|, floor) after 500
    # steps: the fast upstroke of a spike amplifies float rounding along the
    # trajectory (the per-step 1e-5 criterion is the one-step test above).
    net, cfg, drive = nets.hh_cond(n=3000, k=50)
    eng = gpu_run(net, cfg, drive, 500)
    o = FastOracle(net, cfg, drive, precision=64)
    o.step(500)
    ra, rb = eng.read_raster(0, 500), o.raster()
    assert nets.rasters_equal(ra, rb)
    st, so = eng.download_state(), o.state()
    for k in ("v", "hh_m", "hh_h", "hh_n"):
        err = np.abs(st[k] - so[OKEY[k]]) / np.maximum(np.abs(so[OKEY[k]]), FLOOR[k])
        assert err.max() < 1e-2, (k, err.max())


def test_bf16_weight_error_vs_fp64(lib):
    # The stated BF16 error. (1) Storage: every weight is its f32 value
    # rounded to 8 significant bits, |w_bf16 - w| <= 2^-8 |w|. (2) One step
    # of STDP from the same state: the BF16 weights stay within one BF16
    # rounding of the FP64 update. (3) Over 300 steps the chaotic dynamics
    # take another spike path, so the comparison is statistical: mean rate
    # within 5%, weight mean within 1% and std within 2% of the FP64 run.
    net, cfg, drive = nets.izh_stdp(n=10_000, k=100, wf=A.WEIGHT_BF16)
    eng = SimulationEngine(net, cfg, drive)
    w0 = eng.download_state()["w"].astype(np.float64)
    # 8 significant bits: unit roundoff 2^-8
    assert np.all(np.abs(w0 - net.w) <= np.abs(net.w) * 2.0 ** -8)
    eng.run(1)
    o = FastOracle(net, cfg, drive, precision=64)
    o.step(1)
    w1, w64 = eng.download_state()["w"].astype(np.float64), o.weights()
    # initial rounding plus the rounding of the stored result
    assert np.all(np.abs(w1 - w64) <= 2.0 ** -8 * (np.abs(net.w) + np.abs(w64)) * 1.01 + 1e-7)
    eng.run(299)
    o.step(299)
    w_gpu, w64 = eng.download_state()["w"].astype(np.float64), o.weights()
    spk_gpu = eng.counters()[1]
    spk_64 = len(o.raster()[0])
    assert abs(spk_gpu - spk_64) <= 0.05 * spk_64
    assert abs(w_gpu.mean() - w64.mean()) <= 0.01 * abs(w64.mean())
    assert abs(w_gpu.std() - w64.std()) <= 0.02 * w64.std()


def single(model, params, v0, I0, dt, steps, u0=None, decay=1.0, hh_int=A.HH_EULER_REF, m0=None):
    n = 1
    net = Network(model, np.array([params], np.float32), np.array([0, 0], np.uint64),
                  np.zeros(0, np.uint32), np.zeros(0, np.float32), v0=np.array([v0], np.float32),
                  u0=None if u0 is None else np.array([u0], np.float32))
    if m0 is not None:
        net.m0, net.h0, net.n0 = (np.array([x], np.float32) for x in m0)
    cfg = SimConfig(model=model, input_mode=A.INPUT_DIRECT_DECAY, dt_ms=dt, current_decay=decay,
                    hh_integrator=hh_int, stdp_enabled=False, homeostasis_enabled=False,
                    spike_log_capacity=100_000, spike_log_steps=100_000)
    eng = SimulationEngine(net, cfg, Drive())
    if I0:
        st = eng.download_state(with_weights=False)
        st["current"][:] = I0
        eng.upload_state(st, 0)
    spikes = []
    for _ in range(steps):
        spikes.append(eng.step().spike_count)
    return eng, spikes


def test_gpu_lif_known_answers(lib):
    p = [-60.0, -50.0, -65.0, 8.0, 1.5, 2.0]
    _, s = single(A.MODEL_LIF, p, -60.0, 0.0, 0.1, 1)           # lif.rs:68-74
    assert s == [0]
    eng, s = single(A.MODEL_LIF, p, -49.0, 0.0, 0.1, 1)         # lif.rs:76-84
    assert s == [1] and eng.download_state()["v"][0] < -60
    eng, s = single(A.MODEL_LIF, p, -49.0, 1000.0, 0.1, 2)      # lif.rs:86-99
    assert s[1] == 0


def test_gpu_izhikevich_known_answer(lib):
    _, s = single(A.MODEL_IZHIKEVICH, [0.02, 0.2, -65.0, 8.0], -65.0, 10.0, 0.5, 200, u0=0.0)
    assert sum(s) > 0                                             # izhikevich.rs:78-91


def test_gpu_hh_known_answers(lib):
    p = [120.0, 36.0, 0.3, 50.0, -77.0, -54.387, 1.0]
    gates = (0.05, 0.6, 0.32)
    eng, s = single(A.MODEL_HH, p, -65.0, 0.0, 0.01, 1, m0=gates)   # hodgkin_huxley.rs:122-129
    assert s == [0] and abs(eng.download_state()["v"][0] + 65.0) < 1.0
    _, s = single(A.MODEL_HH, p, -65.0, 10.0, 0.01, 500, m0=gates)  # :131-144
    assert sum(s) > 0


def test_reference_default_engine_matches_oracle(lib):
    # default engine semantics: direct current with 0.92 decay, reference
    # drive, STDP + homeostasis (FP64 rate sums). Rasters equal the float
    # oracle over 100 steps; weights within 1e-5 relative (per-synapse expf).
    net, cfg, drive = nets.lif_reference_default(n=2000)
    eng = gpu_run(net, cfg, drive, 100)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(100)
    ra, rb = eng.read_raster(0, 100), o.raster()
    assert len(rb[0]) > 100
    assert nets.rasters_equal(ra, rb)
    w = eng.download_state()["w"].astype(np.float64)
    assert np.allclose(w, o.weights(), rtol=1e-5, atol=1e-6)
    assert np.allclose(eng.rates(), o.rates(), rtol=1e-12, atol=1e-9)


def test_reference_conductance_all_types_stdp_homeostasis(lib):
    # reference conductance mode with AMPA, GABA, GABA-B and NMDA synapses,
    # STDP and homeostasis (contributions carry the NMDA Mg block): rasters
    # equal the float oracle; weights and V within 1e-5 (per-synapse exp)
    net, cfg, drive = nets.lif_conductance_all_types(n=3000)
    cfg.stdp_enabled = True
    cfg.homeostasis_enabled = True
    eng = gpu_run(net, cfg, drive, 100)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(100)
    ra, rb = eng.read_raster(0, 100), o.raster()
    assert len(rb[0]) > 100
    assert nets.rasters_equal(ra, rb)
    st = eng.download_state()
    assert np.allclose(st["w"].astype(np.float64), o.weights(), rtol=1e-5, atol=1e-6)
    assert np.allclose(st["v"].astype(np.float64), o.state()["v"], rtol=1e-5, atol=1e-4)
    assert np.count_nonzero(st["w"] != net.w) > 100


def test_reference_conductance_mode_matches_oracle(lib):
    net, cfg, drive = nets.lif_reference_default(n=2000, stdp=False, homeo=False, conductance=True)
    eng = gpu_run(net, cfg, drive, 100)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(100)
    assert nets.rasters_equal(eng.read_raster(0, 100), o.raster())
    v = eng.download_state()["v"].astype(np.float64)
    assert np.allclose(v, o.state()["v"], rtol=1e-5, atol=1e-4)


@pytest.mark.parametrize("which", ["default", "all_types", "all_types_stdp"])
def test_lfp_matches_oracle(lib, which):
    # lfp_signal (engine.rs:492) in the reference conductance mode: each
    # neuron's term rounded to 2^-24, exact int64 step sums, FP64 total in
    # step order, so the float oracle's value is matched bit for bit. The
    # NMDA Mg block (device expf) and STDP (per-synapse exp) leave V within
    # 1e-5 of the oracle's, so with them the LFP agrees to a tolerance.
    if which == "default":
        net, cfg, drive = nets.lif_reference_default(n=2000, stdp=False, homeo=False, conductance=True)
    else:
        net, cfg, drive = nets.lif_conductance_all_types(n=3000)
        if which == "all_types_stdp":
            cfg.stdp_enabled = True
            cfg.homeostasis_enabled = True
    eng = SimulationEngine(net, cfg, drive)
    o = FastOracle(net, cfg, drive, precision=32)
    assert eng.lfp() == o.lfp() == 0.0
    done = 0
    for k in (1, 37, 100):
        eng.run(k - done)
        o.step(k - done)
        done = k
        if which != "default":
            assert eng.lfp() == pytest.approx(o.lfp(), rel=1e-7)
        else:
            assert eng.lfp() == o.lfp()
    assert nets.rasters_equal(eng.read_raster(0, 100), o.raster())
    assert o.lfp() > 1e6
    a = eng.lfp()
    assert eng.lfp() == a   # reading it consumes nothing
    eng.close()


def test_lfp_zero_in_current_mode(lib):
    net, cfg, drive = nets.lif_reference_default(n=500, stdp=False, homeo=False)
    eng = gpu_run(net, cfg, drive, 20)
    assert eng.lfp() == 0.0


def test_checkpoint_resume_bit_exact(lib):
    net, cfg, drive = nets.izh_stdp(n=10_000, k=50)
    a = gpu_run(net, cfg, drive, 400)
    full_raster = a.read_raster(200, 200)
    full_state = a.download_state()
    b = gpu_run(net, cfg, drive, 200)
    snap = b.download_state()
    b.close()
    c = SimulationEngine(net, cfg, drive)
    c.upload_state(snap, 200)
    c.run(200)
    st = c.download_state()
    for key in ("v", "u", "pre_trace", "post_trace", "last_spike_step", "w"):
        assert np.array_equal(st[key], full_state[key]), key
    assert nets.rasters_equal(c.read_raster(200, 200), full_raster)


def test_reupload_same_and_other_shape(lib):
    # re-uploading a same-shaped network reuses buffers (and captured graphs);
    # a different shape reallocates; both give the fresh engine's results
    net, cfg, drive = nets.izh_stdp(n=20_000, k=50)
    cfg.graph_chunk = 100
    eng = gpu_run(net, cfg, drive, 300)
    ref = (eng.read_raster(0, 300), eng.download_state()["w"])
    eng._upload(net)
    eng.run(300)
    assert nets.rasters_equal(eng.read_raster(0, 300), ref[0])
    assert np.array_equal(eng.download_state()["w"], ref[1])
    net2, _, _ = nets.izh_stdp(n=20_000, k=40, seed=7)
    eng._upload(net2)
    eng.run(200)
    o = FastOracle(net2, cfg, drive, precision=32)
    o.step(200)
    assert nets.rasters_equal(eng.read_raster(0, 200), o.raster())


def test_empty_and_ragged_networks(lib):
    # n not a multiple of the tile, rows of zero out-degree, m = 0
    for n in (1, 7, 1025, 3001):
        rng = np.random.default_rng(n)
        deg = rng.integers(0, 4, n)
        rp = np.concatenate([[0], np.cumsum(deg)]).astype(np.uint64)
        col = rng.integers(0, n, int(rp[-1])).astype(np.uint32)
        for j in range(n):
            col[rp[j]:rp[j + 1]].sort()
        w = rng.uniform(0, 3, len(col)).astype(np.float32)
        params = np.tile(np.array([0.02, 0.2, -65.0, 8.0], np.float32), (n, 1))
        net = Network(A.MODEL_IZHIKEVICH, params, rp, col, w, plastic=np.ones(len(col), np.uint8),
                      inhibitory=np.zeros(n, np.uint8))
        cfg = SimConfig(model=A.MODEL_IZHIKEVICH, input_mode=A.INPUT_RESET_EACH_STEP, dt_ms=1.0,
                        seed=n, spike_log_capacity=1_000_000, spike_log_steps=1000,
                        homeostasis_enabled=False)
        drive = Drive(A.DRIVE_GAUSS, sigma_exc=8.0, sigma_inh=8.0)
        eng = gpu_run(net, cfg, drive, 100)
        o = FastOracle(net, cfg, drive, precision=32)
        o.step(100)
        assert nets.rasters_equal(eng.read_raster(0, 100), o.raster()), n
        assert np.array_equal(eng.download_state()["w"].astype(np.float64), o.weights())


def test_invalid_inputs_rejected(lib):
    net, cfg, drive = nets.izh_stdp(n=2000, k=10)
    bad = Network(net.model, net.params, net.row_ptr.copy(), net.col.copy(), net.w)
    bad.col[5] = net.n + 3
    with pytest.raises(NsError) as e:
        SimulationEngine(bad, cfg, drive)
    assert e.value.status == 3
    bad2 = Network(net.model, net.params, net.row_ptr.copy(), net.col, net.w)
    bad2.row_ptr[10], bad2.row_ptr[11] = bad2.row_ptr[11], bad2.row_ptr[10] + 1
    with pytest.raises(NsError):
        SimulationEngine(bad2, cfg, drive)
    bad3 = Network(net.model, net.params, net.row_ptr, net.col, net.w.copy())
    bad3.w[3] = np.nan
    with pytest.raises(NsError) as e:
        SimulationEngine(bad3, cfg, drive)
    assert e.value.status == 9
    bad4 = Network(net.model, net.params.copy(), net.row_ptr, net.col, net.w)
    bad4.params[0, 0] = np.inf
    with pytest.raises(NsError) as e:
        SimulationEngine(bad4, cfg, drive)
    assert e.value.status == 9


def test_spike_log_overflow_reported(lib):
    net, cfg, drive = nets.izh_stdp(n=20_000, k=20)
    cfg.spike_log_capacity = 1000
    cfg.spike_log_steps = 1000
    eng = SimulationEngine(net, cfg, drive)
    with pytest.raises(NsError) as e:
        eng.run(200)
    assert e.value.status == 10
    eng.clear_spike_log()
    eng.run(1)


def test_c2_full_size_deterministic(lib):
    # config C2 at full size (1M neurons, 100M synapses, BF16): two runs of
    # 50 steps give the same raster and weights; events equal the out-degree
    # sum of the logged spikes; no non-finite state
    from neuralsim_b200 import configs
    net, cfg, drive, _ = configs.izh_c2()
    cfg.spike_log_capacity, cfg.spike_log_steps = 50_000_000, 1000
    runs = []
    for _ in range(2):
        eng = SimulationEngine(net, cfg, drive)
        out = eng.run(50)
        idx, off = eng.read_raster(0, 50)
        st = eng.download_state()
        runs.append((idx, off, st["w"], out.events))
        assert np.all(np.isfinite(st["v"])) and np.all(np.isfinite(st["w"]))
        eng.close()
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
    assert np.array_equal(runs[0][2], runs[1][2])
    deg = np.diff(net.row_ptr.astype(np.int64))
    assert runs[0][3] == int(deg[runs[0][0]].sum()) and runs[0][3] > 0


@pytest.mark.parametrize("which", ["ref_default", "windowed"])
def test_simulation_stats_match_oracle(lib, which):
    # SimulationStats (engine.rs:22-33, :617-670): totals, the largest step
    # (active_neurons), the last step (weight_updates, synchrony), the mean
    # rate estimate and the weight moments
    if which == "ref_default":
        net, cfg, drive = nets.lif_reference_default(n=2000)   # homeostasis keeps the rates
    else:
        net, cfg, drive = nets.lif_delta(n=4000, k=40)
        cfg.spike_log_capacity = 10_000_000
    eng = SimulationEngine(net, cfg, drive)
    eng.run(120)
    eng.run(80)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(200)
    idx, off = o.raster()
    counts = np.diff(off.astype(np.int64))
    st = eng.stats()
    assert st["total_spikes"] == len(idx)
    assert st["active_neurons"] == counts.max() > 0
    assert st["weight_updates"] == counts[-1]
    assert st["synchrony_index"] == counts[-1] / net.n
    if which == "ref_default":
        assert st["mean_firing_rate"] == pytest.approx(o.rates().mean(), rel=1e-12)
        w = o.weights()
        assert st["weight_mean"] == pytest.approx(w.mean(), rel=1e-6)
        assert st["weight_std"] == pytest.approx(w.std(), rel=1e-5)
    else:
        assert eng.window()[0] > 1


def test_step_result_lists(lib):
    # StepResult (engine.rs:35-41): the step's ascending spiking neurons and
    # the output neurons among them, as the oracle's raster has them
    net, cfg, drive = nets.lif_reference_default(n=500)
    net.is_output = (np.arange(net.n) % 5 == 0).astype(np.uint8)
    eng = SimulationEngine(net, cfg, drive)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(30)
    idx, off = o.raster()
    seen_out = 0
    for k in range(30):
        r = eng.step()
        want = idx[off[k]:off[k + 1]]
        assert np.array_equal(r.spiking_neurons, want)
        assert r.spike_count == len(want)
        assert np.array_equal(r.output_spiking_neurons, want[want % 5 == 0])
        assert r.output_spike_count == len(r.output_spiking_neurons)
        seen_out += r.output_spike_count
    assert seen_out > 0


@pytest.mark.parametrize("plastic", ["none", "last_target", "first_target"])
def test_incoming_lists_edge_cases(lib, plastic):
    # the plastic incoming lists (one stable sort by target, pointers from
    # lower bounds): no plastic synapse at all, or all of them onto one end
    net, cfg, drive = nets.izh_stdp(n=3000, k=30, wf=A.WEIGHT_F32)
    if plastic == "none":
        pl = np.zeros(net.m, np.uint8)
    else:
        t = net.n - 1 if plastic == "last_target" else 0
        pl = (net.col == t).astype(np.uint8)
        assert pl.sum() > 10
    net.plastic = pl
    eng = gpu_run(net, cfg, drive, 200)
    o = FastOracle(net, cfg, drive, precision=32)
    o.step(200)
    assert nets.rasters_equal(eng.read_raster(0, 200), o.raster())
    w = eng.download_state()["w"].astype(np.float64)
    assert np.array_equal(w, o.weights())
    changed = w != net.w.astype(np.float64)
    assert not np.any(changed & (pl == 0))
