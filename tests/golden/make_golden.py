"""Writes the golden fixtures under tests/golden/.

Each fixture is a small seeded network of one configuration family, run on
the oracle (FP32-mirroring engine for LIF and Izhikevich, FP64 engine for
Hodgkin-Huxley), saved with a digest of the network it ran on so that a
change of the generator shows up as a fixture mismatch instead of a silent
re-pin. The reference crate cannot be built in this image (no Rust
toolchain), so these vectors are generated by the restatement and pinned by
the known-answer tests in test_oracle_known_answers.py.

Usage: python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from neuralsim_b200 import _abi as A  # noqa: E402
import nets  # noqa: E402


def net_digest(net):
    h = hashlib.sha256()
    for a in (net.row_ptr, net.col, net.w, net.params, net.syn_type, net.plastic):
        if a is not None:
            h.update(np.ascontiguousarray(a).tobytes())
    # arrays of the later rules enter the digest only where a network has them
    for a in (net.is_output, net.eligible, net.stp, net.has_stp):
        if a is not None:
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _consolidating(seed):
    net, cfg, drive = nets.izh_stdp(n=800, k=40, seed=seed, wf=A.WEIGHT_F32)
    nets.with_consolidation(cfg, tau=10.0, drift=1.0)   # the frame renormalises every ~105 steps
    return net, cfg, drive


def _with_stp(seed):
    net, cfg, drive = nets.lif_reference_default(n=300, seed=seed, stdp=False, homeo=False)
    nets.with_stp(net)
    return net, cfg, drive


# name -> (builder, steps, oracle precision)
def _cond_stim_rates(seed):
    # reference conductance mode, firing-rate tracking, host stimulus rounds
    net, cfg, drive = nets.lif_reference_default(n=300, seed=seed, stdp=False, homeo=False,
                                                 conductance=True)
    cfg.track_rates = 1
    return net, cfg, drive


# (steps before the call, neuron ids, amounts) of a case's stimulus rounds
STIM_ROUNDS = [(40, [3, 7, 7, 150], [20.0, 15.0, 5.0, 30.0]), (60, list(range(10, 200, 9)), [12.5])]


def advance(obj, case):
    """Steps an oracle (.step) or an engine (.run) through a case, with its
    stimulus rounds when it has them."""
    go = obj.run if hasattr(obj, "run") else obj.step
    rounds = case[3] if len(case) > 3 else None
    done = 0
    for steps, ids, amt in rounds or ():
        go(steps)
        done += steps
        obj.stimulate(ids, amt)
    go(case[1] - done)


CASES = {
    "lif_delta_n600": (lambda: nets.lif_delta(n=600, k=40, seed=143), 1500, 32),
    "izh_stdp_bf16_n800": (lambda: nets.izh_stdp(n=800, k=40, seed=144), 300, 32),
    "izh_stdp_f32_n800": (lambda: nets.izh_stdp(n=800, k=40, seed=145, wf=A.WEIGHT_F32), 300, 32),
    "lif_reference_default_n200": (lambda: nets.lif_reference_default(n=200, seed=142), 300, 32),
    "hh_rush_larsen_n400": (lambda: nets.hh_cond(n=400, k=40, seed=146), 2000, 64),
    "izh_rstdp_f32_n800": (lambda: nets.izh_rstdp(n=800, k=40, seed=147, wf=A.WEIGHT_F32, n_out=80,
                                                  threshold=4), 300, 32),
    "izh_consolidation_f32_n800": (lambda: _consolidating(148), 300, 32),
    "lif_stp_n300": (lambda: _with_stp(149), 200, 32),
    "lif_cond_stim_rates_n300": (lambda: _cond_stim_rates(150), 160, 32, STIM_ROUNDS),
}


def run_case(name):
    from oracle.oracle import FastOracle
    build, steps, prec = CASES[name][:3]
    net, cfg, drive = build()
    o = FastOracle(net, cfg, drive, precision=prec)
    advance(o, CASES[name])
    idx, off = o.raster()
    st = o.state()
    out = {"idx": np.asarray(idx, np.uint32), "off": np.asarray(off, np.uint64),
           "v": np.asarray(st["v"], np.float64), "weights": np.asarray(o.weights(), np.float64 if prec == 64 else np.float32),
           "steps": np.int64(steps), "precision": np.int64(prec),
           "net_sha256": np.array(net_digest(net))}
    for k in ("u", "m", "h", "n", "pre", "post", "refr"):
        if k in st and st[k] is not None:
            out[k] = np.asarray(st[k])
    if cfg.input_mode == A.INPUT_CONDUCTANCE_REF:
        out["lfp"] = np.float64(o.lfp())
    if getattr(cfg, "track_rates", 0):
        out["rates"] = np.asarray(o.rates(), np.float64)
    if getattr(cfg, "rstdp_enabled", False):
        out["elig"] = np.asarray(o.eligibility(), np.float32 if prec == 32 else np.float64)
        out["reward"] = np.asarray(o.reward(), np.float64)
    o.close()
    return out


def main():
    for name in CASES:
        out = run_case(name)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "spikes", len(out["idx"]))


if __name__ == "__main__":
    main()
