"""Benchmark: COBAHH network, 100,000 Hodgkin-Huxley neurons, float32, exponential Euler,
dt = 0.1 ms, connect(p=0.02) (about 2e8 synapses) with per-synapse delays of 1..50 steps.

One bench step = 100 simulation time steps (10 ms of biological time) of the whole network
(fused neuron kernel + spike delivery), replayed from CUDA graphs.  value = synaptic
events/s (spikes x out-degree delivered per second of wall time on the device); the line
also carries neuron-updates/s.  Inputs (state, 1.6 GB of synapse arrays) are resident in
HBM before timing starts; the synapse arrays alone exceed the 126 MB L2.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b2b|reference]
Under torchrun every rank runs an independent replica (weak scaling; the network does not
shard) and rank 0 reports the max time over ranks.
"""
from __future__ import annotations

import argparse
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

DT = 1e-4
N_NEURONS = 100_000
P_CONNECT = 0.02
DMIN, DMAX = 1, 50
SIM_STEPS = 100              # simulation steps per bench step
BYTES_NEURON_UPDATE = 54     # COBAHH f32: 6 vars x 4 B x (R+W) + flag + lastspike
BYTES_EVENT = 16             # post index 4 + weight 4 + target R/W 8
BYTES_BUNDLE = 8             # bundle offsets read per (spike, delay)
METRIC = "synaptic events/s"
UNIT = "events/s"
WORKLOAD = "COBAHH 1e5 HH neurons f32 exp-Euler, p=0.02 (~2e8 synapses), delays U{1..50} steps"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    def __init__(self, gpu: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:7]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------------------------
def cpu_network(steps_budget_s: float, max_steps: int):
    """The oracle port (C++, OpenMP over all host threads) on the same model: same size,
    parameters and connectivity distribution (numpy-drawn instance), timed per step."""
    from brian2cuda_b200 import models
    from oracle.oracle import OracleNet

    rng = np.random.default_rng(models.SEED_BASE + 101)
    net = OracleNet(DT, f32=True)
    P = net.hh_group(N_NEURONS, models.cobahh_hh())
    models.cobahh_init(net, P, N_NEURONS, rng)
    i, j = models.bernoulli_pairs(rng, N_NEURONS, N_NEURONS, P_CONNECT)
    d = rng.integers(DMIN, DMAX + 1, size=len(i)).astype(np.int32)
    ne = int(0.8 * N_NEURONS)
    exc = i < ne
    net.synapses(P, P, "ge", i[exc], j[exc], w_scalar=6e-9, delay=d[exc])
    net.synapses(P, P, "gi", i[~exc], j[~exc], w_scalar=67e-9, delay=d[~exc])
    outdeg = np.bincount(i, minlength=N_NEURONS)
    n_syn = len(i)
    del i, j, d, exc
    net.run(1)  # builds the bundles and queues
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps and time.perf_counter() - t0 < steps_budget_s:
        net.run(5)
        steps += 5
    el = time.perf_counter() - t0
    idx, st = net.spikes(P)
    sel = st >= 1
    events = float(outdeg[idx[sel]].sum())
    return {"events": events, "steps": steps, "seconds": el, "n_syn": n_syn,
            "neuron_updates": float(N_NEURONS) * steps}


def reference_arm(args):
    threads = os.cpu_count()
    t0 = time.perf_counter()
    r = cpu_network(steps_budget_s=min(60.0, 8.0 * (args.steps + args.warmup)),
                    max_steps=20 * (args.steps + args.warmup))
    value = r["events"] / r["seconds"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * r["seconds"] / max(1, r["steps"]) * SIM_STEPS,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "sim_steps_per_step": SIM_STEPS,
                   "neurons": N_NEURONS, "synapses": r["n_syn"]},
        "neuron_updates_per_s": r["neuron_updates"] / r["seconds"],
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{r['steps']} simulation steps of the full network after "
                                   f"setup ({r['seconds']:.1f} s); C++ oracle, OpenMP"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.perf_counter() - t0,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b2b", choices=["b2b", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup(args.gpus)

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch

    from brian2cuda_b200 import Network, models
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream(device=local)
    total_sim = SIM_STEPS * (args.warmup + 2 * args.steps) + 300
    mon_cap = int(N_NEURONS * total_sim * DT * 400)  # room for a mean rate up to 400 Hz
    net = Network(DT, seed=models.SEED_BASE + 1, device=local, steps_per_graph=50,
                  stream=stream.cuda_stream)
    t_setup = time.perf_counter()
    ids = models.build_cobahh(net, n=N_NEURONS, p=P_CONNECT, dmin=DMIN, dmax=DMAX,
                              monitor_capacity=mon_cap)
    net.finalize()
    P = ids["P"]
    outdeg = np.zeros(N_NEURONS, np.int64)
    n_syn = 0
    for sid in (ids["Ce"], ids["Ci"]):
        i = net.syn_get(sid, "i")
        outdeg += np.bincount(i, minlength=N_NEURONS)
        n_syn += len(i)
        del i
    setup_s = time.perf_counter() - t_setup

    for _ in range(args.warmup):
        net.run(SIM_STEPS)
    net.sync()
    barrier(world)
    cursor = net.spikes_fetch(P, 0, cap=1 << 26)[2]

    # ---- device-timed region: inputs resident, CUDA events on the network's stream
    launches0 = net.kernel_launches
    ts0 = net.timestep
    clocks = Clocks(local)
    torch.cuda.synchronize()
    barrier(world)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        net.run(SIM_STEPS)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_total = max_over_ranks(ev0.elapsed_time(ev1), world)
    launches = net.kernel_launches - launches0
    ts1 = net.timestep
    idx, st, cursor = net.spikes_fetch(P, cursor, cap=1 << 27)
    sel = (st >= ts0) & (st < ts1)
    events = float(outdeg[idx[sel]].sum()) * world
    nspk = int(sel.sum())
    seconds = ms_total / 1e3
    value = events / seconds
    neuron_updates = float(N_NEURONS) * (ts1 - ts0) * world / seconds
    rate_hz = nspk / (N_NEURONS * (ts1 - ts0) * DT)

    # ---- end to end through the public API: run + host readback of the step's results
    v_host = np.empty(N_NEURONS, np.float32)
    d2h = 0
    e2e_events = 0.0
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        net.run(SIM_STEPS)
        v_host[:] = net.get_state(P, "v")
        idx, st, cursor = net.spikes_fetch(P, cursor, cap=1 << 24)
        e2e_events += float(outdeg[idx].sum())
        d2h += v_host.nbytes + 12 * len(idx) + 8
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = e2e_events * world / e2e_s

    # ---- per-kernel device times (profiling run: every launch timed with CUDA events)
    prof = net.profile(200)
    hbm, peak_kind = peaks()
    kinds = {1: "neuron (HH update+threshold+compaction)", 2: "delivery on_pre"}
    dom = max(range(len(prof)), key=lambda k: prof[k][1])
    dom_kind, dom_ms = prof[dom]
    if dom_kind == 1:
        alg = BYTES_NEURON_UPDATE * N_NEURONS
        traffic = _traffic("hh_step_kernel")
    else:
        ev_per_step = events / world / max(1, ts1 - ts0)
        spk_per_step = nspk / max(1, ts1 - ts0)
        alg = BYTES_EVENT * ev_per_step + BYTES_BUNDLE * spk_per_step * (DMAX - DMIN + 1) / 2
        traffic = _traffic("deliver_add_kernel")
    achieved = alg / (dom_ms * 1e-3) / 1e9
    kernel_ms = {f"site{k}:{kinds.get(kd, kd)}": round(ms, 5) for k, (kd, ms) in enumerate(prof)}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sim_steps_per_step": SIM_STEPS, "neurons": N_NEURONS,
                   "synapses": n_syn, "parallelism": f"replicas x{world}",
                   "l2": "working set > L2 (1.6 GB synapse arrays)"},
        "neuron_updates_per_s": neuron_updates,
        "firing_rate_hz": rate_hz,
        "setup_s": setup_s,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "kernel": kinds.get(dom_kind, str(dom_kind)), "kernel_ms": dom_ms,
                     "peak_source": peak_kind},
        "kernel_ms": kernel_ms,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": d2h // max(1, args.steps),
                "note": "run(100 steps) + readback of v and of the new spikes each step; the "
                        "network has no per-step external input"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_network(steps_budget_s=20.0, max_steps=400)
        line["cpu_baseline"] = {
            "value": r["events"] / r["seconds"], "unit": UNIT, "cores": os.cpu_count(),
            "kind": "port",
            "sample": f"{r['steps']} simulation steps of the full 1e5-neuron network "
                      f"({r['seconds']:.1f} s), C++ oracle with OpenMP",
            "neuron_updates_per_s": r["neuron_updates"] / r["seconds"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    net.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary, when one exists."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(kernel)
    except Exception:
        return None


if __name__ == "__main__":
    main()
