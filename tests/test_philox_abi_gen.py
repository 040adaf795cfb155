"""CPU tests: Philox known-answer vectors, drive math, the C ABI library
(loads, exports every declared symbol, error behaviour without a device) and
the synthetic-network generator."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Published Philox4x32-10 test vectors (Salmon et al., SC'11; Random123 kat_vectors)
KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
]


@pytest.mark.parametrize("ctr,key,out", KAT)
def test_oracle_philox_kat(oracle_lib, ctr, key, out):
    o = (C.c_uint32 * 4)()
    oracle_lib.or_philox4x32_10((C.c_uint32 * 4)(*ctr), (C.c_uint32 * 2)(*key), o)
    assert list(o) == out


def test_drive_log_and_sincos_accuracy(oracle_lib):
    xs = np.random.default_rng(1).uniform(1e-7, 1.0, 4000).astype(np.float32)
    for x in xs:
        ref = np.log(np.float64(x))
        assert abs(oracle_lib.or_logf(float(x)) - ref) <= 3e-7 * max(abs(ref), 1.0)
    s, c = C.c_float(), C.c_float()
    for u in np.linspace(0, 1, 4001, endpoint=False, dtype=np.float32):
        oracle_lib.or_sincos2pi(float(u), C.byref(s), C.byref(c))
        a = 2 * np.pi * np.float64(u)
        assert abs(s.value - np.sin(a)) < 3e-7 and abs(c.value - np.cos(a)) < 3e-7


def test_homeostasis_exp_accuracy(oracle_lib):
    xs = np.concatenate([np.linspace(-20, 20, 4001), np.random.default_rng(2).normal(0, 1e-3, 2000)])
    for x in xs.astype(np.float32):
        ref = np.exp(np.float64(x))
        assert abs(oracle_lib.or_expf(float(x)) - ref) <= 4e-7 * ref


def test_gauss_drive_statistics(oracle_lib):
    from oracle.oracle import make_config
    from neuralsim_b200 import Drive, SimConfig
    from neuralsim_b200 import _abi as A
    cfg = make_config(SimConfig(seed=7), Drive(A.DRIVE_GAUSS, sigma_exc=1.0, sigma_inh=1.0))
    z = np.array([oracle_lib.or_drive_f32(C.byref(cfg), 20000, None, i, 3, 0.0)
                  for i in range(20000)])
    assert abs(z.mean()) < 0.03 and abs(z.std() - 1.0) < 0.03
    assert abs(np.mean(z ** 4) / np.mean(z ** 2) ** 2 - 3.0) < 0.2


def declared_symbols():
    names = []
    import glob
    for h in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"\b(ns_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(lib):
    from neuralsim_b200 import _abi
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
        assert s in _abi.SIGNATURES, f"{s} not bound in _abi.SIGNATURES"


def test_status_strings_and_null_handles(lib):
    assert lib.ns_status_string(0) == b"ok"
    assert lib.ns_step(None, 1, None) == 2
    assert lib.ns_destroy(None) == 2
    cnt = C.c_int(-1)
    assert lib.ns_device_count(C.byref(cnt)) == 0 and cnt.value >= 0


def test_create_rejects_bad_config(lib):
    from neuralsim_b200 import _abi as A
    c = A.NsConfig()
    lib.ns_config_default(C.byref(c))
    assert c.dt_ms == 0.5 and c.seed == 42 and abs(c.current_decay - 0.92) < 1e-12
    h = C.c_void_p()
    c.dt_ms = -1.0
    assert lib.ns_create(C.byref(c), C.byref(h)) == 1
    c.dt_ms = 0.1
    c.input_mode = A.INPUT_CONDUCTANCE_REF
    c.delay_steps = 2
    assert lib.ns_create(C.byref(c), C.byref(h)) == 8


@pytest.mark.skipif(any(os.path.exists(f"/dev/nvidia{i}") for i in range(8)),
                    reason="a device is present")
def test_create_without_device_fails_loudly(lib):
    from neuralsim_b200 import _abi as A
    c = A.NsConfig()
    lib.ns_config_default(C.byref(c))
    h = C.c_void_p()
    assert lib.ns_create(C.byref(c), C.byref(h)) == 11
    assert h.value is None


def test_topology_properties(lib):
    from neuralsim_b200.configs import topology
    n, k = 3000, 40
    rp, col, src = topology(n, k, 5, with_insertion_order=True)
    assert rp[0] == 0 and rp[-1] == n * k and np.all(np.diff(rp.astype(np.int64)) >= 0)
    s = src.reshape(n, k)
    assert np.all(np.diff(s.astype(np.int64), axis=1) > 0)          # distinct, sorted
    assert not np.any(s == np.arange(n)[:, None])                  # no self connection
    for j in range(0, n, 97):                                       # rows ascending in target
        row = col[rp[j]:rp[j + 1]].astype(np.int64)
        assert np.all(np.diff(row) > 0)
    indeg = np.bincount(col, minlength=n)
    assert np.all(indeg == k)


def test_topology_matches_reference_finalize(lib, oracle_lib):
    # CSR equals Network::finalize (src/network/mod.rs:79-106) applied to the
    # insertion-order edge list (targets 0..n-1, their sources in order)
    from neuralsim_b200.configs import topology
    n, k = 2000, 25
    rp, col, src = topology(n, k, 11, with_insertion_order=True)
    tgt = np.repeat(np.arange(n, dtype=np.uint32), k)
    rp2 = np.zeros(n + 1, np.uint64)
    col2 = np.zeros(n * k, np.uint32)
    oracle_lib.or_finalize_csr(n, n * k, C.c_void_p(src.ctypes.data), C.c_void_p(tgt.ctypes.data),
                               C.c_void_p(rp2.ctypes.data), C.c_void_p(col2.ctypes.data))
    assert np.array_equal(rp, rp2) and np.array_equal(col, col2)


def test_generator_deterministic_across_threads(lib):
    from neuralsim_b200.configs import topology, weights
    from neuralsim_b200 import _abi as A
    a = topology(5000, 30, 3, threads=1)
    b = topology(5000, 30, 3, threads=7)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    w1 = weights(A.GEN_W_UNIFORM, 5000, 4000, a[0], 3, 6.0, 5.0, plastic_exc=True, threads=1)
    w2 = weights(A.GEN_W_UNIFORM, 5000, 4000, a[0], 3, 6.0, 5.0, plastic_exc=True, threads=5)
    for x, y in zip(w1, w2):
        assert np.array_equal(x, y)


def test_izh_config_shapes(lib):
    from neuralsim_b200.configs import izh_c2
    net, cfg, drive, steps = izh_c2(n=4000, k=100)
    n_exc = 3200
    src = np.repeat(np.arange(net.n), np.diff(net.row_ptr.astype(np.int64)))
    exc = src < n_exc
    assert np.all((net.w[exc] >= 0) & (net.w[exc] < 6)) and np.all((net.w[~exc] <= 0) & (net.w[~exc] > -5))
    assert np.array_equal(net.plastic.astype(bool), exc)
    a, b, c, d = net.params.T
    assert np.all(a[:n_exc] == np.float32(0.02)) and np.all(c[n_exc:] == np.float32(-65.0))
    assert np.all((c[:n_exc] >= -65) & (c[:n_exc] <= -50)) and np.all((d[:n_exc] >= 2) & (d[:n_exc] <= 8))
    assert steps == 10_000 and cfg.dt_ms == 1.0
