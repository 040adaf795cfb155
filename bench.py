#!/usr/bin/env python
"""Benchmark: synaptic events/s on the 1M-neuron / 100M-synapse Izhikevich +
pair-STDP network (BF16 weights, dt 1 ms), one JSON line on rank 0.

A bench "step" is 1000 simulation steps (1 s of simulated time) of that
network, inputs resident in HBM (state 64 MB + synapses ~1.3 GB, larger than
the 126 MB L2, so no flush is needed between steps). `value` is device-timed
with CUDA events on the library's launching stream. `e2e` times complete jobs
through the C ABI with pinned host buffers: upload of the network and
initial state, 10,000 simulation steps (the configuration's 10 s), and the
read-back of the full spike raster and final membrane state.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N > 1 (torchrun): independent replicas of the network, one per GPU ("replicas
only": a single network does not shard here); value = all ranks' events /
max over ranks of the device time.
`--impl reference` times the CPU restatement of the reference's engine loop
(C++, FP64, per-synapse state, OpenMP over neurons as rayon does) on this
host: rank 0 only, each step one simulation step of the same network.
"""
import argparse
import copy
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "syn events/s @1M/100M"
UNIT = "events/s"
WORKLOAD = ("Izhikevich + pair STDP, 1,000,000 neurons (80% RS / 20% FS), in-degree 100 "
            "(100M synapses, CSR, BF16 weights, FP32 accumulation), thalamic noise 5/2 N(0,1), "
            "dt 1 ms; one step = 1000 simulation steps (1 s simulated)")


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--neurons", type=int, default=1_000_000)
    p.add_argument("--in-degree", type=int, default=100)
    p.add_argument("--sim-steps", type=int, default=1000, help="simulation steps per bench step")
    p.add_argument("--e2e-jobs", type=int, default=2)
    p.add_argument("--cpu-seconds", type=float, default=20.0)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-extra", action="store_true", help="skip the LIF and HH configuration lines")
    p.add_argument("--no-surrogate", action="store_true", help="skip the learned HH macro-step line")
    p.add_argument("--only", choices=["c1c4", "c3", "c5", "phase2"], default=None,
                   help="run one secondary configuration alone and print its result (profiling)")
    p.add_argument("--sur-train-steps", type=int, default=12000)
    p.add_argument("--ref-warm-steps", type=int, default=300,
                   help="reference arm: steps from rest before the timed sample (active network)")
    p.add_argument("--c3-nets", type=int, default=256, help="networks of the batched sweep (profiling: fewer)")
    p.add_argument("--sur-only-1m", action="store_true",
                   help="surrogate line: evaluate only the 1M-neuron network (profiling)")
    p.add_argument("--shard", action="store_true",
                   help="under torchrun: one network split over the GPUs (strong scaling) instead of replicas")
    p.add_argument("--schedule", type=int, default=0, choices=[0, 1, 2, 3, 4, 5],
                   help="step schedule: 0 autotune, 1 fused, 2 split, 3 fused 4 blocks/SM, "
                        "4 split narrow LTD, 5 deferred LTD")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s (no MEASURED_PEAKS.json)"


PROFILE_UNIT_STEPS = 20


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, x in enumerate(r) if x == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows),
                "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons, "samples": len(rows)}


def build_network(n, k, seed):
    from neuralsim_b200 import configs
    return configs.izh_c2(n=n, k=k, seed=seed)


def step_bytes(n, sim_steps, spikes, events, in_plastic):
    """Algorithmic HBM bytes of sim_steps simulation steps:
    64 N per step (v,u r/w; a,b,c,d; int64 accumulator read + zero; pre/post
    traces r/w) + 16 S (row_ptr pair, CSC pointer pair) + 8 E_out (col, bf16 w,
    LTP write) + 8 E_in,plastic (incoming index, bf16 w read + write)."""
    return 64.0 * n * sim_steps + 16.0 * spikes + 8.0 * events + 8.0 * in_plastic


def kernel_bytes(n, spikes, events, in_plastic, m_plastic, deferred):
    """Algorithmic HBM bytes per launch of each step kernel (one step):
    neuron: 64 N (v,u r/w; a,b,c,d; int64 accumulator read + zero; pre/post
            traces r/w) + 4 S (spike index);
    rows:   16 S (row_ptr pair) + 24 S (last r/w, trace bump r/w)
            + 8 E_out (column 4, bf16 weight read 2 and LTP write 2);
            deferred LTD adds 16 S (the row's trace start read + write);
            its pending LTDs change weights the walk reads and writes anyway;
    ltd:    eager: 16 S (incoming pointer pair) + 8 E_in,plastic (incoming
            entry 4 of the 8 B (source, position) pair counted as in the
            plan's formula, bf16 weight read 2 + write 2);
            deferred (the row-block flush, a 32nd of the rows per step):
            (16 + 16) N/32 (row_ptr pair, trace start read + write) +
            8 M_plastic/32 (column 4, bf16 weight read 2 + write 2).
    Accumulator atomics and trace-record gathers hit L2-resident arrays and
    count as 0 HBM bytes. `sector_bytes` counts the 32-byte DRAM sector that a
    random 2-byte weight access moves (read + write) for the eager LTD."""
    # drive (precomputed one step ahead): the float written per neuron and
    # the inhibitory flag read (a compute-bound kernel: Philox and Box-Muller)
    if deferred:
        return {
            "neuron": 64.0 * n + 4.0 * spikes,
            "rows": 56.0 * spikes + 8.0 * events,
            "ltd": 32.0 * n / 32.0 + 8.0 * m_plastic / 32.0,
            "drive": 5.0 * n,
        }
    return {
        "neuron": 64.0 * n + 4.0 * spikes,
        "rows": 40.0 * spikes + 8.0 * events,
        "ltd": 16.0 * spikes + 8.0 * in_plastic,
        "ltd_sector": 16.0 * spikes + (8.0 + 64.0) * in_plastic,
        "drive": 5.0 * n,
    }


def run_ours(a):
    import torch
    from neuralsim_b200 import SimulationEngine
    from neuralsim_b200 import _abi as A

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)

    t0 = time.time()
    net, cfg, drive, _ = build_network(a.neurons, a.in_degree, 44 + rank)
    cfg.device = local
    cfg.step_schedule = a.schedule
    gen_s = time.time() - t0
    in_deg_plastic = np.zeros(net.n, np.int64)
    np.add.at(in_deg_plastic, net.col[net.plastic.astype(bool)], 1)

    eng = SimulationEngine(net, cfg, drive)
    stream = torch.cuda.ExternalStream(eng.stream(), device=local)
    S = a.sim_steps
    for _ in range(a.warmup):
        eng.run(S)
    c0 = eng.counters()
    l0 = eng.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(a.steps):
            eng.run(S)
        ev1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    c1 = eng.counters()
    launches = eng.launch_count() - l0
    sched, sched_us = eng.schedule()
    events = c1[3] - c0[3]
    spikes = c1[1] - c0[1]
    sim_steps = c1[0] - c0[0]
    clocks = clk.summary()

    # per-kernel device time (eager serial steps with events around each kernel)
    # The first PROFILE_UNIT_STEPS are profiled one step at a time with each
    # step's spikes and events recorded: the ncu traffic capture of the same
    # command reads these launches, so its DRAM bytes can be set against the
    # algorithmic bytes of exactly those steps.
    pc0 = eng.counters()
    prof, units = {}, []
    for q in range(PROFILE_UNIT_STEPS + 1):
        ca = eng.counters()
        part = eng.profile_steps(1 if q < PROFILE_UNIT_STEPS else 200 - PROFILE_UNIT_STEPS)
        cb = eng.counters()
        if q < PROFILE_UNIT_STEPS:
            units.append([int(cb[1] - ca[1]), int(cb[3] - ca[3])])
        for name, (kms, kl) in part.items():
            t = prof.get(name, (0.0, 0))
            prof[name] = (t[0] + kms, t[1] + kl)
    pc1 = eng.counters()
    prof_steps = 200.0
    prof_spikes = (pc1[1] - pc0[1]) / prof_steps
    prof_events = (pc1[3] - pc0[3]) / prof_steps

    # whole-step algorithmic bytes: plastic in-degree of the spikers is
    # estimated from the mean (80 of 100 incoming synapses are plastic)
    mean_in_plastic = float(in_deg_plastic.mean())
    bytes_total = step_bytes(net.n, sim_steps, spikes, events, spikes * mean_in_plastic)

    if dist:
        t = torch.tensor([ms, float(events)], dtype=torch.float64, device=f"cuda:{local}")
        tm = t.clone()
        dist.all_reduce(tm[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(tm[1:2], op=dist.ReduceOp.SUM)
        ms_max, events_all = float(tm[0]), float(tm[1])
    else:
        ms_max, events_all = ms, float(events)

    # e2e: complete jobs through the C ABI with pinned host buffers
    e2e = None
    if not a.no_e2e:
        e2e = run_e2e(a, net, cfg, drive, local, dist)

    extra = None
    if not a.no_extra:
        batch = run_batch_config(local, rank, world, dist, cpu=not a.no_cpu)
        if rank == 0 and world > 1:
            # single-GPU configurations are reported by the one-GPU run; the
            # other ranks would only wait for them
            extra = {"lif_batch_c3": batch}
        elif rank == 0:
            extra = run_extra_configs(local, cpu=not a.no_cpu)
            extra["lif_batch_c3"] = batch
            extra["izh_c2_phase2_rules"] = run_phase2_rules(local)
            if not a.no_surrogate:
                extra["hh_surrogate_c5"] = run_surrogate_config(local, a.sur_train_steps)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        warm = eng.download_state()
        warm["step"] = int(eng.counters()[0])
        cpu = run_cpu_baseline(net, cfg, drive, a.cpu_seconds, warm,
                               events / max(sim_steps, 1))
        del warm

    if rank == 0:
        peak, peak_src = peaks()
        kb = kernel_bytes(net.n, prof_spikes, prof_events, prof_spikes * mean_in_plastic,
                          float(np.count_nonzero(net.plastic)), sched == 5)
        total_prof_ms = sum(v[0] for v in prof.values())
        kernels = {}
        for name, (kms, kl) in prof.items():
            avg_s = kms / kl / 1e3
            kernels[name] = {"avg_launch_us": avg_s * 1e6, "share": kms / total_prof_ms,
                             "bytes_per_launch": kb.get(name),
                             "achieved_gbs": kb[name] / avg_s / 1e9 if name in kb else None}
        if sched == 5 and "ltd" in kernels:
            kernels["row_block_flush"] = kernels.pop("ltd")
            kb["row_block_flush"] = kb.pop("ltd")
        if "ltd" in kernels:
            kernels["ltd"]["sector_bytes_per_launch"] = kb["ltd_sector"]
            kernels["ltd"]["sector_gbs"] = kb["ltd_sector"] / (kernels["ltd"]["avg_launch_us"] / 1e6) / 1e9
        dom = max(kernels, key=lambda k: kernels[k]["share"])
        nk_bytes = kb[dom]
        nk_avg_s = kernels[dom]["avg_launch_us"] / 1e6
        achieved = nk_bytes / nk_avg_s / 1e9
        value = events_all / (ms_max / 1e3)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_max / a.steps,
            "ms_per_sim_step": ms_max / a.steps / S,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded generator, configuration shapes)",
            "config": {
                "workload": WORKLOAD, "neurons": net.n, "synapses": net.m,
                "sim_steps_per_step": S, "weights": "bf16", "accumulation": "int64 fixed point",
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "l2": "inputs larger than L2 (no flush needed)",
                "spikes_per_sim_step": spikes / max(sim_steps, 1),
                "events_per_sim_step": events / max(sim_steps, 1),
                "sim_time_per_wall_s": (sim_steps * cfg.dt_ms / 1e3) / (ms / 1e3),
                "network_build_s": round(gen_s, 2),
                "step_schedule": {1: "fused", 2: "split (LTD beside next neuron update)",
                                  3: "fused, 4 blocks/SM",
                                  4: "split, narrow LTD grid",
                                  5: "deferred LTD (row walks + row-block flush)"}.get(sched, "undecided"),
                "autotune_us_per_step": sched_us,
            },
            "roofline": {
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None,
                "traffic_note": "DRAM bytes come from an ncu capture of this command, summarised "
                                "under profiles/; bench.py does not measure them",
                "kernel": dom, "bytes_per_launch": nk_bytes, "avg_launch_us": nk_avg_s * 1e6,
                "peak_source": peak_src, "spikes_per_step_profiled": prof_spikes,
                "profile_first_steps_spikes_events": units,
                "kernels": kernels,
            },
            "step_roofline": {
                "algorithmic_bytes_per_sim_step": bytes_total / max(sim_steps, 1),
                "achieved": bytes_total / (ms / 1e3) / 1e9, "unit": "GB/s",
                "frac": bytes_total / (ms / 1e3) / 1e9 / peak,
                "formula": "64N + 16S + 8E_out + 8E_in,plastic",
            },
            "clocks": clocks,
            "gpu_launches": launches,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "other_configs": extra,
            "surrogate": (None if not extra or "hh_surrogate_c5" not in extra else {
                "speedup_vs_plain": extra["hh_surrogate_c5"]["speedup_vs_plain_windowed"],
                "spike_time_err_ms": extra["hh_surrogate_c5"]["surrogate"]["spike_time_err_ms"],
                "coarse_rl_spike_time_err_ms":
                    extra["hh_surrogate_c5"]["coarse_rl_0.1ms"]["spike_time_err_ms"],
                "fallback_fraction": extra["hh_surrogate_c5"]["surrogate"]["fallback_fraction"],
                "speedup_vs_plain_1m_neurons":
                    extra["hh_surrogate_c5"]["same_network_1m_neurons"]["speedup_vs_plain_windowed"],
                "spike_time_err_ms_1m_neurons":
                    extra["hh_surrogate_c5"]["same_network_1m_neurons"]["surrogate"]["spike_time_err_ms"]}),
        }
        print(json.dumps(out), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_sharded_c2(a):
    """--shard under torchrun: the C2 network split over the ranks (strong
    scaling: the same 1M-neuron network whatever N), a spike-bitmap NCCL
    all-gather per simulation step inside the step graphs. `value` counts
    every rank's synaptic events over the slowest rank's device time."""
    import datetime
    import torch
    import torch.distributed as dist
    from neuralsim_b200.shard import ShardedEngine
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    net, cfg, drive, _ = build_network(a.neurons, a.in_degree, 44)
    cfg.device = local
    cfg.step_schedule = a.schedule or 3
    se = ShardedEngine(net, cfg, drive, rank, world)
    eng = se.engine
    stream = torch.cuda.ExternalStream(eng.stream(), device=local)
    S = a.sim_steps
    for _ in range(a.warmup):
        se.run(S)
    c0 = eng.counters()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(a.steps):
            se.run(S)
        ev1.record(stream)
        torch.cuda.synchronize()
    dist.barrier()
    ms = ev0.elapsed_time(ev1)
    c1 = eng.counters()
    t = torch.tensor([ms, float(c1[3] - c0[3])], dtype=torch.float64, device=f"cuda:{local}")
    tm = t.clone()
    dist.all_reduce(tm[0:1], op=dist.ReduceOp.MAX)
    dist.all_reduce(tm[1:2], op=dist.ReduceOp.SUM)
    ms_max, events_all = float(tm[0]), float(tm[1])
    if rank == 0:
        sim_steps = c1[0] - c0[0]
        print(json.dumps({
            "metric": METRIC, "value": events_all / (ms_max / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_max / a.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator, configuration shapes)",
            "config": {"workload": WORKLOAD, "neurons": net.n, "synapses": net.m,
                       "sim_steps_per_step": S, "parallelism": f"one network sharded over {world} GPUs",
                       "exchange": "NCCL all-gather of the spike bitmap per simulation step",
                       "spikes_per_sim_step": (c1[1] - c0[1]) / max(sim_steps, 1),
                       "events_per_sim_step": events_all / max(sim_steps, 1)},
            "roofline": None, "cpu_baseline": None, "e2e": None, "clocks": clk.summary(),
            "gpu_launches": int(eng.launch_count())}), flush=True)
    se.close()
    dist.barrier()
    dist.destroy_process_group()


def timed_run(eng, steps, stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0 = eng.counters()
    torch.cuda.synchronize()
    e0.record(stream)
    eng.run(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    c1 = eng.counters()
    return e0.elapsed_time(e1), c1[1] - c0[1], c1[3] - c0[3]


def literal_sample(net, cfg, drive, seconds, max_steps=2000):
    """The CPU restatement of engine.rs (FP64, per-synapse state, OpenMP over
    the neuron update as rayon parallelises it) on this host's cores, stepped
    from rest for about `seconds` after one warm-up step."""
    from oracle.oracle import LiteralOracle
    threads = os.cpu_count() or 1
    lit = LiteralOracle(net, cfg, drive, threads=threads)
    lit.step(1)
    e0 = lit.events()
    t0 = time.perf_counter()
    steps = 0
    while steps < 2 or (time.perf_counter() - t0 < seconds and steps < max_steps):
        lit.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    ev = lit.events() - e0
    lit.close()
    return {"value": ev / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "ns_per_step": dt * 1e9 / steps, "steps": steps, "events_in_sample": int(ev),
            "x_realtime": steps * cfg.dt_ms / (dt * 1e3),
            "sample": f"{steps} simulation steps from rest after 1 warm-up step ({dt:.1f} s); C++ "
                      "restatement of engine.rs, FP64, per-synapse state; not the Rust binary"}


def run_extra_configs(local, cpu=True):
    """The other configurations on this GPU: the plain LIF network (10k / 1M,
    dt 0.1 ms, 1 ms delay, 1 s) and the plain Hodgkin-Huxley network (100k /
    10M, Rush-Larsen, dt 0.01 ms, 1 ms delay), each timed with windowed
    stepping (W = delay) and with one pass per step."""
    import torch
    from neuralsim_b200 import SimulationEngine, configs
    out = {}
    for name, builder, steps, warm in (("lif_c1", configs.lif_c1, 10_000, 2_000),
                                       ("hh_c4", configs.hh_c4, 20_000, 2_000)):
        net, cfg, drive, full_steps = builder()
        cfg.device = local
        res = {"neurons": net.n, "synapses": net.m, "dt_ms": cfg.dt_ms,
               "delay_steps": cfg.delay_steps, "timed_steps": steps}
        peak, _ = peaks()
        for label, wsteps in (("windowed", 0), ("per_step", 1)):
            cfg.window_steps = wsteps
            eng = SimulationEngine(net, cfg, drive)
            stream = torch.cuda.ExternalStream(eng.stream(), device=local)
            eng.run(warm)
            ms, spikes, events = timed_run(eng, steps, stream)
            eng.close()
            s_step, e_step = spikes / steps, events / steps
            # algorithmic bytes per step: LIF v + refractory r/w 16 and the
            # int64 accumulator read + zero 16 per neuron; HH V, m, h, n r/w
            # 32, AMPA / GABA conductances r/w 16 and two accumulator rows
            # read + zero 16 (64 per neuron); 8 per spike (row_ptr pair) and
            # per event (column 4, weight 4)
            per_n = 32.0 if name == "lif_c1" else 64.0
            b_step = per_n * net.n + 8.0 * s_step + 8.0 * e_step
            res[label] = {"ns_per_step": ms * 1e6 / steps,
                          "x_realtime": (steps * cfg.dt_ms) / ms,
                          "events_per_s": events / (ms / 1e3),
                          "spikes_per_step": s_step,
                          "bytes_per_step": b_step,
                          "hbm_frac": b_step / (ms * 1e-3 / steps) / 1e9 / peak}
        if cpu:
            res["cpu_baseline"] = literal_sample(net, cfg, drive, 8.0 if name == "lif_c1" else 12.0)
            res["speedup_vs_cpu_per_step"] = (res["cpu_baseline"]["ns_per_step"] /
                                              res["windowed"]["ns_per_step"])
        out[name] = res
    return out


def run_phase2_rules(local, warm=500, steps=500):
    """The rest of phase 2 on the C2 network (1M Izhikevich, 100M BF16
    synapses, pair STDP): per-step cost with R-STDP (10% output neurons;
    reward threshold 5, so every step is rewarded and the reward is applied
    in the STDP walks), with an R-STDP range narrower than STDP's (every
    rewarded step takes the full O(M) pass), with consolidation (the O(1)
    frame) and with both."""
    import torch
    from neuralsim_b200 import SimulationEngine
    net, cfg0, drive, _ = build_network(1_000_000, 100, 44)
    net.is_output = (np.arange(net.n) < net.n // 10).astype(np.uint8)
    variants = {
        "stdp": {},
        "rstdp_rewarded": {"rstdp_enabled": True},
        "rstdp_full_pass_each_step": {"rstdp_enabled": True, "rstdp_w_max": 5.0},
        "consolidation": {"consolidation_enabled": True},
        "rstdp_and_consolidation": {"rstdp_enabled": True, "consolidation_enabled": True},
    }
    out = {"neurons": net.n, "synapses": net.m, "timed_steps": steps, "output_neurons": net.n // 10}
    base = None
    for name, kv in variants.items():
        cfg = copy.deepcopy(cfg0)
        cfg.device = local
        for key, val in kv.items():
            setattr(cfg, key, val)
        eng = SimulationEngine(net, cfg, drive)
        stream = torch.cuda.ExternalStream(eng.stream(), device=local)
        eng.run(warm)
        ms, spikes, events = timed_run(eng, steps, stream)
        res = {"ns_per_step": ms * 1e6 / steps, "events_per_s": events / (ms / 1e3),
               "spikes_per_step": spikes / steps, "schedule": eng.schedule()[0]}
        if cfg.rstdp_enabled:
            res["reward"] = eng.reward()[0]
        eng.close()
        if base is None:
            base = res["ns_per_step"]
        res["cost_vs_stdp"] = res["ns_per_step"] / base
        out[name] = res
    return out


def run_batch_config(local, rank, world, dist, n_nets=256, cpu=True):
    """The batched sweep: 256 LIF networks (log-uniform 2k..50k neurons,
    in-degree 50..200), one batch per GPU (networks bin-packed by size across
    ranks, no per-step communication), 1000 steps of dt 0.1 ms timed after
    1000 warm-up steps; time is the max over ranks. Timed with the
    configuration's drive (Poisson 8 Hz, 0.8 mV kicks: nearly silent) and
    with a stronger drive variant (Poisson 200 Hz, 4 mV kicks) that makes
    the networks active, labelled as such."""
    import torch
    from neuralsim_b200 import _abi as A, configs, shard
    from neuralsim_b200.batch import BatchEngine
    from neuralsim_b200.engine import Drive
    nets, seeds, cfg, drive, steps = configs.lif_batch_c3(n_nets=n_nets)
    cfg.device = local
    owner = shard.assign([shard.network_cost(x) for x in nets], world)
    mine = [i for i in range(len(nets)) if owner[i] == rank]
    my_nets = [nets[i] for i in mine]
    my_seeds = [seeds[i] for i in mine]
    n_all = sum(x.n for x in nets)
    m_all = sum(x.m for x in nets)
    res = {"networks": len(nets), "neurons": n_all, "synapses": m_all, "dt_ms": cfg.dt_ms,
           "delay_steps": cfg.delay_steps, "timed_steps": steps,
           "sharding": f"{world} rank(s), networks bin-packed by neurons + synapses"}
    variants = (("config_drive", drive),
                ("active_drive_variant", Drive(A.DRIVE_POISSON_KICK, p=0.02, amplitude=4.0)))
    for label, drv in variants:
        eng = BatchEngine(my_nets, my_seeds, cfg, drv)
        stream = torch.cuda.ExternalStream(eng.stream(), device=local)
        eng.run(steps)
        ms, spikes, events = timed_run(eng, steps, stream)
        wlen, wtune = eng.window()
        plan, (_, shape_us) = eng.window_plan(), eng.walk_shape()
        eng.close()
        if dist:
            t = torch.tensor([ms, float(spikes), float(events)], dtype=torch.float64,
                             device=f"cuda:{local}")
            tm = t.clone()
            dist.all_reduce(tm[0:1], op=dist.ReduceOp.MAX)
            dist.all_reduce(tm[1:3], op=dist.ReduceOp.SUM)
            ms, spikes, events = float(tm[0]), float(tm[1]), float(tm[2])
        s_step, e_step = spikes / steps, events / steps
        # per-step-path bytes: v, refractory r/w 16 + accumulator read/zero 16
        # per neuron, col + w 8 per event, spike index 8
        bytes_step = 32.0 * n_all + 8.0 * s_step + 8.0 * e_step
        peak, _ = peaks()
        res[label] = {"ms": ms, "ns_per_step": ms * 1e6 / steps,
                      "x_realtime": (steps * cfg.dt_ms) / ms,
                      "events_per_s": events / (ms / 1e3),
                      "neuron_updates_per_s": n_all * steps / (ms / 1e3),
                      "spikes_per_step": s_step,
                      "rate_hz": s_step / n_all / (cfg.dt_ms / 1e3),
                      "step_path_bytes_per_s": bytes_step * steps / (ms / 1e3),
                      "hbm_frac": bytes_step * steps / (ms / 1e3) / 1e9 / peak,
                      "window_steps": wlen,
                      "window_tuner_us_per_step": wtune,
                      "window_plan": plan,
                      "walk_shape_tuner_us_per_step": {f"{l} lanes x {b or 'max'} blocks/SM": t
                                                       for (l, b), t in shape_us.items()}}
    if cpu and rank == 0 and world == 1:
        res["cpu_baseline"] = batch_cpu_sample(nets, seeds, cfg, variants)
        for label, _ in variants:
            res[label]["speedup_vs_cpu_per_step"] = (res["cpu_baseline"][label]["ns_per_step"] /
                                                     res[label]["ns_per_step"])
    return res


def batch_cpu_sample(nets, seeds, cfg, variants, n_sample=8, seconds=1.5):
    """The batch on the CPU restatement: the networks run one after another
    (as independent engines would), sampled. Eight networks (the smallest,
    the largest, six drawn at random) are each stepped from rest for about
    `seconds`; the batch's time per step is their time per step scaled by
    the batch's neurons + synapses over theirs."""
    rng = np.random.default_rng(7)
    sizes = np.array([x.n for x in nets])
    pick = {int(np.argmin(sizes)), int(np.argmax(sizes))}
    rest = [q for q in range(len(nets)) if q not in pick]
    pick.update(int(q) for q in rng.choice(rest, n_sample - 2, replace=False))
    pick = sorted(pick)
    cost_all = float(sum(x.n + x.m for x in nets))
    cost_s = float(sum(nets[q].n + nets[q].m for q in pick))
    out = {"sampled_networks": pick, "scale": cost_all / cost_s}
    for label, drv in variants:
        ns_sum, ev_sum, steps_min, threads = 0.0, 0.0, None, 1
        for q in pick:
            c = copy.copy(cfg)
            c.seed = seeds[q]
            r = literal_sample(nets[q], c, drv, seconds)
            ns_sum += r["ns_per_step"]
            ev_sum += r["events_in_sample"] / r["steps"]
            steps_min = r["steps"] if steps_min is None else min(steps_min, r["steps"])
            threads = r["cores"]
        ns_batch = ns_sum * out["scale"]
        ev_batch = ev_sum * out["scale"]
        out[label] = {"value": ev_batch / (ns_batch * 1e-9), "unit": UNIT, "cores": threads,
                      "kind": "port", "ns_per_step": ns_batch,
                      "x_realtime": cfg.dt_ms / (ns_batch * 1e-6),
                      "sample": f"{len(pick)} of {len(nets)} networks, each stepped from rest for "
                                f"about {seconds} s (at least {steps_min} steps), one after "
                                "another; time per step scaled by neurons + synapses "
                                f"(x{out['scale']:.1f}); C++ restatement of engine.rs, FP64"}
    return out


def _surrogate_eval(net, cfg, drive, sur, local, steps):
    """Plain, surrogate and the two comparison modes from the same start,
    timed; spike times matched to the plain run's (nearest within 2 ms)."""
    import torch
    from neuralsim_b200 import SimulationEngine
    from neuralsim_b200.raster import match_spikes
    rasters, res = {}, {}
    for mode in ("plain", "surrogate", "coarse_rl_0.1ms", "held_current_rl"):
        eng = SimulationEngine(net, cfg, drive)
        if mode != "plain":
            eng.attach_surrogate(sur)
            if mode != "surrogate":
                eng.macro_step_mode(1 if mode == "coarse_rl_0.1ms" else 2)
        stream = torch.cuda.ExternalStream(eng.stream(), device=local)
        ms, spikes, events = timed_run(eng, steps, stream)
        rasters[mode] = eng.read_raster(0, steps)
        r = {"ns_per_step": ms * 1e6 / steps, "ns_per_sim_ms": ms * 1e6 / (steps * cfg.dt_ms),
             "spikes": int(spikes)}
        if mode != "plain":
            mlp, fb = eng.surrogate_counts()
            r["macro_steps_mlp"], r["macro_steps_fallback"] = mlp, fb
            r["fallback_fraction"] = fb / max(mlp + fb, 1)
        eng.close()
        res[mode] = r
    w = int(round(2.0 / cfg.dt_ms))
    for mode in ("surrogate", "coarse_rl_0.1ms", "held_current_rl"):
        d, ua, ub = match_spikes(rasters["plain"], rasters[mode], w)
        res[mode]["spike_time_err_ms"] = float(d.mean() * cfg.dt_ms) if len(d) else None
        res[mode]["matched"], res[mode]["unmatched_plain"], res[mode]["unmatched_other"] = len(d), ua, ub
    res["speedup_vs_plain_windowed"] = res["plain"]["ns_per_sim_ms"] / res["surrogate"]["ns_per_sim_ms"]
    return res


def run_surrogate_config(local, train_steps=12000, only_1m=False):
    """The learned HH macro-step on the plain Hodgkin-Huxley network (100k
    neurons, 10M synapses, dt 0.01 ms, Rush-Larsen): about 10M transitions
    sampled from the plain run (100 snapshots of all neurons, 0.5 ms apart,
    after a 20 ms warm-up; those with V in the envelope +- 3 mV kept, the
    approach to threshold weighted x4), targets and training on the device.
    Then, from the same state, the plain and the surrogate paths each timed
    over 100 ms and the surrogate's spike times matched to the plain run's;
    beside them the same macro-step scheme with one Rush-Larsen step of
    0.1 ms in the MLP's place (the plain method in the surrogate's cost
    class) and with ten Rush-Larsen steps with the held current (the function
    the MLP is trained on: the error of the scheme alone). The same trained
    surrogate is also run on the same network shape at 1M neurons (100M
    synapses), where the plain path is no longer bound by one Rush-Larsen
    chain per neuron."""
    from neuralsim_b200 import configs, surrogate as S
    net, cfg, drive, _ = configs.hh_c4()
    cfg.device = local
    cfg.window_steps = 100
    cfg.spike_log_capacity, cfg.spike_log_steps = 50_000_000, 20_000
    t0 = time.time()
    sur, x, y, losses = S.train_for_network(net, cfg, drive, warm_steps=2000, snapshots=100,
                                            every_steps=50, batch=8192, steps=train_steps)
    train_s = time.time() - t0
    res = {"neurons": net.n, "synapses": net.m, "dt_ms": cfg.dt_ms, "macro_step_ms": 0.1,
           "mlp": "5-128-128-4 SiLU, bf16 weights, fp32 accumulation (tcgen05)",
           "train_samples": int(len(x)), "train_steps": train_steps, "train_batch": 8192,
           "train_wall_s": round(train_s, 2), "final_loss": float(np.mean(losses[-100:])),
           "envelope_mv": [S.V_LO, S.MACRO_V_HI], "training_envelope_mv": [S.V_LO, S.V_HI],
           "residual_mv": S.RESIDUAL_MV}
    if not only_1m:
        res.update(_surrogate_eval(net, cfg, drive, sur, local, 10_000))
    big, bcfg, bdrive, _ = configs.hh_c4(n=1_000_000)
    bcfg.device = local
    bcfg.window_steps = 100
    bcfg.spike_log_capacity, bcfg.spike_log_steps = 200_000_000, 5_000
    r1 = _surrogate_eval(big, bcfg, bdrive, sur, local, 2_000)
    r1.update({"neurons": big.n, "synapses": big.m, "timed_steps": 2_000})
    res["same_network_1m_neurons"] = r1
    sur.close()
    return res


def run_e2e(a, net, cfg, drive, local, dist):
    """Whole jobs: pinned host network + state -> device, 10,000 steps,
    raster + final v back to pinned host memory."""
    import torch
    from neuralsim_b200 import SimulationEngine
    from neuralsim_b200.engine import Network
    pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy()
    pnet = Network(net.model, pin(net.params), pin(net.row_ptr), pin(net.col), pin(net.w),
                   syn_type=pin(net.syn_type), plastic=pin(net.plastic), v0=pin(net.v0),
                   u0=pin(net.u0), inhibitory=pin(net.inhibitory))
    job_steps = 10_000
    cfg.spike_log_capacity = 200_000_000
    cfg.spike_log_steps = job_steps
    h2d = (pnet.params.nbytes + pnet.row_ptr.nbytes + pnet.col.nbytes + pnet.w.nbytes +
           pnet.syn_type.nbytes + pnet.plastic.nbytes + pnet.v0.nbytes + pnet.u0.nbytes +
           pnet.inhibitory.nbytes)
    eng = SimulationEngine(pnet, cfg, drive)   # allocations done once
    stream = torch.cuda.ExternalStream(eng.stream(), device=local)
    times, events, d2h, parts = [], [], [], []
    raster_buf = None   # pinned, sized after the warm-up job
    for job in range(a.e2e_jobs + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        eu, er = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        eng._upload(pnet)
        eu.record(stream)
        c0 = eng.counters()
        eng.run(job_steps)
        er.record(stream)
        c1 = eng.counters()
        idx, off = eng.read_raster(c0[0], job_steps, out=raster_buf)
        st = eng.download_state(with_weights=False, fields=("v",))
        e1.record(stream)
        torch.cuda.synchronize()
        if job == 0:
            # warm-up job: the raster buffer of the timed jobs, pinned once
            raster_buf = pin(np.zeros(2 * max(int(idx.size), 1), np.uint32))
            continue
        times.append(e0.elapsed_time(e1))
        parts.append([e0.elapsed_time(eu), eu.elapsed_time(er), er.elapsed_time(e1)])
        events.append(c1[3] - c0[3])
        d2h.append(idx.nbytes + off.nbytes + st["v"].nbytes)
    eng.close()
    ms = sum(times)
    ev = float(sum(events))
    if dist:
        t = torch.tensor([ms, ev], dtype=torch.float64, device=f"cuda:{local}")
        m_ = t[0:1].clone()
        s_ = t[1:2].clone()
        dist.all_reduce(m_, op=dist.ReduceOp.MAX)
        dist.all_reduce(s_, op=dist.ReduceOp.SUM)
        ms, ev = float(m_), float(s_)
    return {"value": ev / (ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(statistics.mean(d2h)),
            "step": "one job: upload network + initial state, 10,000 simulation steps, "
                    "read back raster + final v", "jobs": len(times),
            "ms_per_job": ms / max(len(times), 1),
            "ms_upload_run_readback_per_job": [[round(x, 2) for x in p] for p in parts]}


def run_cpu_baseline(net, cfg, drive, seconds, warm=None, events_per_step=None):
    """The CPU restatement of engine.rs (FP64, per-synapse state) on this
    host, on the same network, for a bounded number of simulation steps,
    started from `warm` (the GPU run's state after its timed region: neuron
    state, traces, last spike steps, weights, step) so that it times the
    same active network."""
    from oracle.oracle import LiteralOracle
    threads = os.cpu_count() or 1
    lit = LiteralOracle(net, cfg, drive, threads=threads)
    if warm is not None:
        lit.set_state(warm["v"], warm["u"], warm["pre_trace"], warm["post_trace"],
                      warm["last_spike_step"].astype(np.float64) * cfg.dt_ms, warm["w"],
                      warm["step"] * cfg.dt_ms, warm["step"])
    lit.step(1)  # warm-up
    e0 = lit.events()
    t0 = time.perf_counter()
    steps = 0
    while steps < 2 or (time.perf_counter() - t0 < seconds and steps < 100):
        lit.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    ev = lit.events() - e0
    lit.close()
    # value: the events the sample itself processed over its time. The
    # network bursts (50-step stretches of ~1M and of ~1k events per step)
    # while the engine's per-step cost is set by its O(M) loops, so the
    # per-simulation-step time is the stable figure; the rate at the GPU
    # workload's mean activity is given beside it
    return {"value": ev / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "ms_per_sim_step": dt * 1e3 / steps, "events_in_sample": int(ev),
            "events_per_sim_step": ev / steps,
            "value_at_workload_mean_events": (events_per_step * steps / dt) if events_per_step else None,
            "workload_mean_events_per_sim_step": events_per_step,
            "sample": f"{steps} simulation steps of the same 1M/100M network, started from the GPU "
                      f"run's state after its timed region, after 1 warm-up step ({dt:.1f} s); "
                      "value = the sample's own events / its time; C++ restatement of engine.rs, "
                      "FP64, per-synapse state, OpenMP over the neuron update only (as rayon); "
                      "not the Rust binary"}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.oracle import FastOracle, LiteralOracle
    net, cfg, drive, _ = build_network(a.neurons, a.in_degree, 44)
    threads = os.cpu_count() or 1
    # an active network to time: the oracle's FP64 engine runs the first
    # ref_warm_steps from rest (the reference's own loop structure costs
    # ~2 s per step at this size), its state then starts the literal engine
    fo = FastOracle(net, cfg, drive, precision=64)
    fo.step(a.ref_warm_steps // 3)
    e_a = fo.events()
    fo.step(a.ref_warm_steps - a.ref_warm_steps // 3)
    # mean events per step of the workload past the onset (bursty network)
    ev_mean = (fo.events() - e_a) / max(a.ref_warm_steps - a.ref_warm_steps // 3, 1)
    st, w = fo.state(), fo.weights()
    fo.close()
    lit = LiteralOracle(net, cfg, drive, threads=threads)
    lit.set_state(st["v"], st["u"], st["pre"], st["post"], st["last"].astype(np.float64) * cfg.dt_ms,
                  w, a.ref_warm_steps * cfg.dt_ms, a.ref_warm_steps)
    del st, w
    for _ in range(a.warmup):
        lit.step(1)
    e0 = lit.events()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        lit.step(1)
    dt = time.perf_counter() - t0
    ev = lit.events() - e0
    # the sample's own events over its own time (the bursty network makes
    # this vary with where the sample falls; ms_per_sim_step is the stable
    # figure, the engine's cost per step being set by its O(M) loops)
    value = ev / dt
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": dt * 1e3 / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, configuration shapes)",
        "config": {"workload": WORKLOAD.replace("one step = 1000 simulation steps (1 s simulated)",
                                                "one step = 1 simulation step"),
                   "neurons": net.n, "synapses": net.m, "sim_steps_per_step": 1},
        "impl": "reference",
        "ms_per_sim_step": dt * 1e3 / a.steps,
        "events_per_sim_step": ev / a.steps,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "ms_per_sim_step": dt * 1e3 / a.steps, "events_in_sample": int(ev),
                         "value_at_warmup_mean_events": ev_mean * a.steps / dt,
                         "sample": f"{a.steps} simulation steps after {a.warmup} warm-up steps, "
                                   f"from the state {a.ref_warm_steps} steps after rest (the "
                                   f"oracle's FP64 engine); value = the sample's own {ev} events "
                                   "/ its time; C++ restatement of engine.rs (the Rust crate does "
                                   "not build here), FP64, per-synapse state, OpenMP over the "
                                   "neuron update"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    a = args_()
    if a.only:
        import torch
        torch.cuda.set_device(0)
        if a.only == "c1c4":
            print(json.dumps(run_extra_configs(0, cpu=not a.no_cpu)), flush=True)
        elif a.only == "c3":
            print(json.dumps(run_batch_config(0, 0, 1, None, a.c3_nets, cpu=not a.no_cpu)), flush=True)
        elif a.only == "phase2":
            print(json.dumps(run_phase2_rules(0)), flush=True)
        else:
            print(json.dumps(run_surrogate_config(0, a.sur_train_steps, a.sur_only_1m)), flush=True)
        return
    if a.impl == "reference":
        run_reference(a)
    elif a.shard and int(os.environ.get("WORLD_SIZE", "1")) > 1:
        run_sharded_c2(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
