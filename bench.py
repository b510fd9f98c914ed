"""Benchmark: COBAHH network, 100,000 Hodgkin-Huxley neurons, float32, exponential Euler,
dt = 0.1 ms, connect(p=0.02) (about 2e8 synapses) with per-synapse delays of 1..50 steps,
1 s simulated.

One bench step = the whole configured run: restore the seeded initial state (a device-side
checkpoint) and simulate 1 s = 10,000 time steps (the neuron update and the spike delivery
of each step as two concurrent launches, replayed from CUDA graphs).  The network fires in population bursts about every 140 ms, so
shorter windows would sample the burst cycle unevenly.  value = synaptic events/s (spikes
x out-degree delivered per second of device time); the line also carries
neuron-updates/s.  Inputs (state, 1.6 GB of synapse arrays) are resident in HBM before
timing starts; the synapse arrays alone exceed the 126 MB L2.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b2b|reference]
Under torchrun every rank runs an independent replica (weak scaling; the network fits one
GPU and is not sharded) and rank 0 reports the max time over ranks.
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
SIM_STEPS = 10_000           # simulation steps per bench step (1 s)
BYTES_NEURON_UPDATE = 54     # COBAHH f32: 6 vars x 4 B x (R+W) + flag + lastspike
BYTES_NEURON_FOLD = 16       # two-launch step: pending ge, gi input read and cleared, 4 B each way
BYTES_EVENT = 12             # post index 4 + target R/W 8 (we, wi: one value per Synapses)
BYTES_BUNDLE = 8             # per (spike, delay) bundle visited
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
    """Samples SM clocks and clock-event (throttle) reasons during the timed region: NVML from
    a thread every 10 ms, live before the constructor returns (an nvidia-smi child takes
    longer to start than a short timed region lasts); nvidia-smi where NVML is missing."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu: int, period_s: float = 0.01):
        import threading
        self.samples = []
        self.p = None
        try:
            import pynvml
            pynvml.nvmlInit()
            h = self._nvml_handle(pynvml, gpu)
            bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
        except Exception:
            self._start_smi(gpu)
            return
        self.stop_ev = threading.Event()
        first = threading.Event()

        def loop():
            while True:
                try:
                    sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((float(sm), float(smax),
                                         {nm for nm, b in bits.items() if r & b}))
                except Exception:
                    pass
                first.set()
                if self.stop_ev.wait(period_s):
                    return

        self.th = threading.Thread(target=loop, daemon=True)
        self.th.start()
        first.wait(2.0)

    @staticmethod
    def _nvml_handle(pynvml, gpu: int):
        # the CUDA device's PCI address: NVML numbers every GPU of the machine, CUDA only the
        # visible ones
        try:
            import torch
            pr = torch.cuda.get_device_properties(gpu)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(gpu)

    def _start_smi(self, gpu):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = False

    def stop(self):
        if self.p is False:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        if self.p is None:
            self.stop_ev.set()
            self.th.join()
            samples = list(self.samples)
            source = "nvml"
        else:
            self.p.terminate()
            self.p.wait()
            self.f.flush()
            self.f.seek(0)
            samples = []
            for line in self.f.read().splitlines():
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 7:
                    continue
                try:
                    sm, smax = float(parts[0]), float(parts[1])
                except ValueError:
                    continue
                samples.append((sm, smax, {nm for nm, val in zip(self.NAMES, parts[3:7])
                                           if val.lower() == "active"}))
            os.unlink(self.f.name)
            source = "nvidia-smi"
        sm = [a for a, _, _ in samples]
        smax = [b for _, b, _ in samples]
        reasons = set().union(*[r for _, _, r in samples]) if samples else set()
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm), "source": source}


def dist_setup(n_gpus, backend: str = "nccl"):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE); the process group is
    NCCL on GPUs (gloo for the CPU tests of the same code) with a short timeout, so ranks
    that wait on each other end with an error."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------------------------
def cpu_info():
    """CPU model and the threads the oracle's OpenMP loops use on this host."""
    model = None
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True).stdout
        for ln in out.splitlines():
            if ln.startswith("Model name:"):
                model = ln.split(":", 1)[1].strip()
    except Exception:
        pass
    threads = int(os.environ.get("OMP_NUM_THREADS", "0") or 0) or os.cpu_count()
    return {"cpu_model": model, "omp_threads": threads, "host_cpus": os.cpu_count()}


def delivery_table(net, sids, n_pre: int) -> np.ndarray:
    """cum[n, k] = synapses of presynaptic neuron n (over the Synapses objects sids) whose
    delay is at most k steps; a spike of n at step s of a run of E steps has
    cum[n, min(E - 1 - s, DMAX)] of its synaptic events delivered inside the run."""
    w = DMAX + 1
    cnt = np.zeros(n_pre * w, np.int64)
    for sid in sids:
        key = net.syn_get(sid, "i").astype(np.int64) * w
        key += net.syn_get(sid, "delay").astype(np.int64)
        cnt += np.bincount(key, minlength=n_pre * w)
        del key
    return np.cumsum(cnt.reshape(n_pre, w), axis=1)


def delivered_events(cum: np.ndarray, idx, st, end: int) -> float:
    """Synaptic events of spikes (idx at steps st, relative to the run start) delivered
    before step `end` (events whose delay carries them past the run are not counted)."""
    if len(idx) == 0:
        return 0.0
    k = np.minimum(end - 1 - np.asarray(st, np.int64), cum.shape[1] - 1)
    return float(cum[np.asarray(idx, np.int64), k].sum())


class CpuCobahh:
    """The oracle port (C++, OpenMP over the host threads) on the configured network: the
    same connect(p) (Philox, the same seeds and synapse order as the GPU run), parameters and
    initial state as the GPU arm, so both arms simulate the identical network."""

    def __init__(self):
        from brian2cuda_b200 import models
        from oracle.oracle import OracleNet
        t0 = time.perf_counter()
        self.net = OracleNet(DT, f32=True)
        self.ids = models.build_cobahh(self.net, n=N_NEURONS, p=P_CONNECT, dmin=DMIN, dmax=DMAX,
                                       generated=True)
        self.net.run(0)             # builds the bundle tables and the delay queues
        self.net.store(0)
        self.n_syn = sum(self.net.syn_count(s) for s in (self.ids["Ce"], self.ids["Ci"]))
        self.cum = delivery_table(self.net, (self.ids["Ce"], self.ids["Ci"]), N_NEURONS)
        self.setup_s = time.perf_counter() - t0

    def run_window(self, chunks: int, chunk_steps: int, budget_s: float | None = None):
        """From the initial state, `chunks` chunks of chunk_steps steps, each timed (stops
        early past budget_s); returns (seconds per chunk, steps run, events, spikes)."""
        net, P = self.net, self.ids["P"]
        net.restore(0)
        net.clear_spikes()
        times = []
        t_all = time.perf_counter()
        for _ in range(chunks):
            t0 = time.perf_counter()
            net.run(chunk_steps)
            times.append(time.perf_counter() - t0)
            if budget_s is not None and time.perf_counter() - t_all > budget_s:
                break
        steps = chunk_steps * len(times)
        idx, st = net.spikes(P)
        return times, steps, delivered_events(self.cum, idx, st, steps), len(idx)


def reference_arm(args):
    """The reference's CPU path on the host cores: the oracle port of the reference's
    algorithm (the reference itself is a code generator that needs Brian2, absent here).
    One step = a sample of S = ceil(10,000 / K) simulation steps; the K timed steps cover
    the configured 1 s run from its initial state (simulation steps [0, K*S)), the W warm-up
    steps repeat its first sample from the initial state."""
    t0 = time.perf_counter()
    cpu = CpuCobahh()
    S = -(-SIM_STEPS // args.steps)
    for _ in range(args.warmup):
        cpu.run_window(1, S)
    times, steps, events, nspk = cpu.run_window(args.steps, S)
    seconds = sum(times)
    value = events / seconds
    info = cpu_info()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * seconds / args.steps,
        "firing_rate_hz": nspk / (N_NEURONS * steps * DT),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "sim_steps_per_step": S, "neurons": N_NEURONS,
                   "synapses": cpu.n_syn,
                   "window": f"simulation steps [0, {steps}) of the configured run"},
        "neuron_updates_per_s": float(N_NEURONS) * steps / seconds,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["omp_threads"],
                         "kind": "port",
                         "sample": f"{args.steps} steps of {S} simulation steps = simulation "
                                   f"steps [0, {steps}) of the configured 1 s run of the "
                                   f"identical 1e5-neuron network ({seconds:.1f} s); C++ "
                                   "oracle, OpenMP", **info},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "setup_s": cpu.setup_s,
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
    ap.add_argument("--no-configs", action="store_true",
                    help="only the COBAHH line, without the other configurations' entries")
    ap.add_argument("--ncu-case", type=int, default=0, metavar="STEPS",
                    help="profiling case: build the workload, simulate STEPS steps, print "
                         "nothing (for ncu captures of the step kernels)")
    ap.add_argument("--two-launch", action="store_true",
                    help="run every step as two concurrent launches (neuron update, delivery "
                         "of earlier spikes) where the net allows it")
    ap.add_argument("--one-launch", action="store_true",
                    help="run both halves of every step (update, delivery of earlier spikes) "
                         "as one launch where the net allows it")
    ap.add_argument("--per-step", action="store_true",
                    help="always the per-step kernels (default: the library's choice, which "
                         "the autotuner settles)")
    ap.add_argument("--tune-from", default=None, metavar="FILE",
                    help="apply the launch shapes of the JSON line in FILE (an earlier bench "
                         "output) instead of autotuning; used by the profiling case")
    ap.add_argument("--workload", default="cobahh",
                    choices=["cobahh", "batched", "cuba", "stdp", "hines", "propagation"],
                    help="cobahh: the 1e5-neuron COBAHH network (default line); batched: 256 "
                         "COBAHH instances, plain vs batched vs batched + gating surrogate")
    ap.add_argument("--kernel-case", default=None,
                    choices=["hh4m", "surrogate1m", "mlp_train", "propagation",
                             "propagation3000", "stdp", "stdp_synorder", "hines", "model",
                             "batched"],
                    help="profiling case of one kernel (see kernel_case); prints nothing")
    args = ap.parse_args()
    if args.kernel_case:
        kernel_case(args.kernel_case)
        return
    world, rank, local = dist_setup(args.gpus)

    if args.workload != "cobahh" and args.impl == "b2b":
        if args.workload == "batched":
            line = bench_batched(args, world, rank, local)
        else:
            line = bench_small(args, world, rank, local)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    line = bench_cobahh(args, world, rank, local)
    if line is None:            # the profiling case prints nothing
        return
    if rank == 0 and world == 1 and not args.no_configs:
        # the other configurations, each a shorter timed window (their own lines'
        # value, unit, roofline and CPU baseline), so the default run stays a few minutes
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup = min(args.steps, 5), 3
        configs = {}
        for wl in ("cuba", "stdp", "hines", "propagation", "batched"):
            sub.workload = wl
            t0 = time.perf_counter()
            try:
                entry = (bench_batched if wl == "batched" else bench_small)(sub, world, rank,
                                                                            local)
            except Exception as exc:     # keep the headline line if one entry fails
                entry = {"error": f"{type(exc).__name__}: {exc}"}
            entry["wall_s"] = time.perf_counter() - t0
            configs[wl] = entry
        line["configs"] = configs
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def bench_cobahh(args, world, rank, local):
    import torch

    from brian2cuda_b200 import Network, models
    from brian2cuda_b200.network import atomic_rate
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream(device=local)
    runs = args.warmup + 2 * args.steps + 2
    mon_cap = int(N_NEURONS * SIM_STEPS * DT * 30 * runs)  # mean rate up to 30 Hz
    net = Network(DT, seed=models.SEED_BASE + 1, device=local, steps_per_graph=50,
                  stream=stream.cuda_stream,
                  two_launch=True if args.two_launch else (False if args.per_step else None),
                  one_launch=args.one_launch)
    t_setup = time.perf_counter()
    ids = models.build_cobahh(net, n=N_NEURONS, p=P_CONNECT, dmin=DMIN, dmax=DMAX,
                              monitor_capacity=mon_cap)
    net.finalize()
    P = ids["P"]
    ne = int(0.8 * N_NEURONS)
    n_syn = sum(net.syn_count(s) for s in (ids["Ce"], ids["Ci"]))
    cum = delivery_table(net, (ids["Ce"], ids["Ci"]), N_NEURONS)
    outdeg = cum[:, -1]
    net.store(0)
    init = {v: net.get_state(P, v) for v in ("v", "m", "h", "n", "ge", "gi", "lastspike")}
    setup_s = time.perf_counter() - t_setup
    # launch shapes tuned on the network's own run: every trial covers the first 2000 steps
    # from the initial state (the first population burst, the quiet phase after it and the
    # next burst, ~1400 steps later).  A shorter window weighs the bursts too much: on 300
    # steps the one-launch form wins by 6 %, on the whole run it loses by 4 %.  The autotuner
    # leaves the state where it found it
    tune = None
    if args.tune_from:
        with open(args.tune_from) as f:
            tune = json.loads([ln for ln in f if ln.startswith("{")][-1])["autotune"]
        net.tune_apply(tune)
    else:
        tune = net.autotune(trial_steps=2000)

    if args.ncu_case:
        net.run(args.ncu_case)
        net.sync()
        net.close()
        return None

    def one_run():
        net.restore(0)
        net.run(SIM_STEPS)

    for _ in range(args.warmup):
        one_run()
    net.sync()
    barrier(world)
    cursor = net.spikes_recorded(P)

    # ---- device-timed region: inputs resident, CUDA events on the network's stream
    launches0 = net.kernel_launches
    clocks = Clocks(local)
    torch.cuda.synchronize()
    barrier(world)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        one_run()
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_total = max_over_ranks(ev0.elapsed_time(ev1), world)
    launches = net.kernel_launches - launches0
    idx, st, cursor = net.spikes_fetch(P, cursor, cap=1 << 24)
    nspk = len(idx)
    # every run starts at step 0 from the checkpoint: st is the step within its run
    exc = idx < ne
    ev_exc = delivered_events(cum, idx[exc], st[exc], SIM_STEPS)
    ev_inh = delivered_events(cum, idx[~exc], st[~exc], SIM_STEPS)
    events = (ev_exc + ev_inh) * world
    seconds = ms_total / 1e3
    value = events / seconds
    neuron_updates = float(N_NEURONS) * SIM_STEPS * args.steps * world / seconds
    rate_hz = nspk / (N_NEURONS * SIM_STEPS * args.steps * DT)

    # ---- end to end through the public API: the seeded initial state goes host -> device
    # from pinned memory, the run executes, and the new spikes and v come back every step
    pinned = {}
    for k, a in init.items():
        t = torch.empty(a.shape, dtype=torch.from_numpy(a).dtype, pin_memory=True)
        t.numpy()[:] = a
        pinned[k] = t.numpy()
    h2d = sum(a.nbytes for a in pinned.values())
    d2h = 0
    fetched = []
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        net.restore(0)
        for k, a in pinned.items():
            net.set_state(P, k, a)
        net.run(SIM_STEPS)
        v_host = net.get_state(P, "v")
        idx_e, st_e, cursor = net.spikes_fetch(P, cursor, cap=1 << 24)
        fetched.append((idx_e, st_e))
        d2h += v_host.nbytes + 12 * len(idx_e) + 8
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    # the metric's bookkeeping (events of the fetched spikes) after the timed region
    e2e_events = sum(delivered_events(cum, i_, s_, SIM_STEPS) for i_, s_ in fetched)
    e2e_value = e2e_events * world / e2e_s

    # ---- roofline.  The update and the delivery of a step run as two concurrent launches
    # (or back to back in the per-step form), so neither takes longer than the step's device
    # time over the timed region; bytes / that time is a lower bound on each launch's
    # bandwidth.
    hbm, peak_kind = peaks()
    step_ms = ms_total / (args.steps * SIM_STEPS)
    nd = DMAX - DMIN + 1
    one_launch = net.run_mode == "one-launch"
    two_launch = net.run_mode == "two-launch" or one_launch
    neuron_bytes = float(BYTES_NEURON_UPDATE * N_NEURONS)
    if two_launch:
        # the update also adds in and clears the pending input of ge and gi
        neuron_bytes += BYTES_NEURON_FOLD * N_NEURONS
    run_events = (ev_exc + ev_inh) / args.steps
    deliver_bytes = (BYTES_EVENT * run_events + BYTES_BUNDLE * nd * nspk / args.steps) / SIM_STEPS
    upd_name = ("neuron (HH update+threshold+compaction"
                + (", folding in the pending input)" if two_launch else ")"))
    upd_kernel = "hh_step_kernel@fold" if two_launch else "hh_step_kernel"
    del_name = ("delivery on_pre into the pending input (Ce and Ci, one launch)" if two_launch
                else "delivery on_pre (Ce and Ci, one launch)")
    roof_bytes = neuron_bytes
    if one_launch:
        # one kernel holds both halves of the step: its bytes are the update's and the
        # delivery's
        upd_name = ("one_launch_step_kernel: " + upd_name + " and " + del_name.split(" (")[0]
                    + " in one grid")
        upd_kernel = "one_launch_step_kernel"
        roof_bytes = neuron_bytes + deliver_bytes
    achieved = roof_bytes / (step_ms * 1e-3) / 1e9
    d_achieved = deliver_bytes / (step_ms * 1e-3) / 1e9
    d_rate = run_events / (step_ms * 1e-3 * SIM_STEPS)
    # the delivery's own ceiling: scattered f32 atomics into the population's ge and gi
    # (2e5 floats), one index load per event from HBM
    loaded, hashed, dsmem = atomic_rate(2 * N_NEURONS, 60_000_000, device=local,
                                        stream=stream.cuda_stream)
    # diagnostic only: one configured run from the checkpoint with an event-record node
    # before and after every launch; the nodes lengthen each launch by microseconds, so at
    # this step size the figures give the order of the launches' shares, not their times
    net.restore(0)
    prof, prof_step_ms = net.profile_graph(SIM_STEPS)
    net.spikes_fetch(P, cursor, cap=1 << 24)
    site_label = {1: "neuron", 5: "delivery (pending)", 6: "delivery", 13: "one launch"}
    in_graph = {site_label.get(kd, f"site kind {kd}"): round(ms, 6) for kd, ms in prof}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sim_steps_per_step": SIM_STEPS, "neurons": N_NEURONS,
                   "synapses": n_syn, "parallelism": f"replicas x{world}",
                   "l2": "working set > L2 (1.6 GB synapse arrays); the 5.4 MB of neuron "
                         "state stays L2-resident between steps"},
        "neuron_updates_per_s": neuron_updates,
        "firing_rate_hz": rate_hz,
        "spikes_per_run": nspk / args.steps,
        "events_per_run": (ev_exc + ev_inh) / args.steps,
        "events_counted": "spikes x their synapses whose delay lands inside the run",
        "setup_s": setup_s,
        "run_mode": net.run_mode,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": _traffic_lookup(upd_kernel),
                     "kernel": upd_name, "kernel_ms": step_ms, "peak_source": peak_kind,
                     "bytes_per_launch": roof_bytes,
                     "bytes_per_unit": (f"{BYTES_NEURON_UPDATE} B per neuron-update"
                                        + (f" + {BYTES_NEURON_FOLD} B pending input read and "
                                           "cleared" if two_launch else "")
                                        + (f"; + {BYTES_EVENT} B per event and {BYTES_BUNDLE} "
                                           "B per (spike, delay) bundle" if one_launch
                                           else "")),
                     "timing": "kernel_ms = device time per simulation step over the timed "
                               "region (CUDA events); the step's launches run inside it, so "
                               "it bounds the kernel's duration from above and achieved/frac "
                               "are lower bounds",
                     "note": "the neuron state (5.4 MB) is L2-resident between steps, so the "
                             "update is latency-bound, not HBM-bound"},
        "delivery": {"kernel": del_name, "kernel_ms": step_ms,
                     "bytes_per_launch": deliver_bytes,
                     "bytes_per_unit": f"{BYTES_EVENT} B per event + {BYTES_BUNDLE} B per "
                                       "(spike, delay) bundle",
                     "achieved_gbs": d_achieved, "frac_hbm": d_achieved / hbm,
                     "traffic": _traffic_lookup("deliver_pending_kernel" if two_launch
                                                else "deliver_add_batch_kernel"),
                     "events_per_s_in_kernel": d_rate,
                     "atomic_ceiling_events_per_s": {"index_loaded": loaded,
                                                     "index_in_registers": hashed,
                                                     "cluster_shared_memory": dsmem},
                     "frac_of_atomic_ceiling": d_rate / loaded,
                     "note": "lower bounds from the step time, as for the roofline; at the "
                             "network's ~3 Hz a step delivers ~6e4 events and the kernel is "
                             "latency-bound; configs.propagation measures it under load"},
        "in_graph_event_nodes": {"ms_per_step": in_graph, "step_ms": prof_step_ms,
                                 "note": "event-record nodes around every launch (diagnostic; "
                                         f"they lengthen the {step_ms * 1e3:.2f} us step)"},
        "autotune": tune,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h // max(1, args.steps),
                "note": "restore + upload of the 7 initial state arrays from pinned memory, "
                        "run of 10,000 steps, readback of v and of the run's spikes"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    net.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = CpuCobahh()
        times, steps, ev, _ = cpu.run_window(SIM_STEPS // 500, 500, budget_s=30.0)
        info = cpu_info()
        line["cpu_baseline"] = {
            "value": ev / sum(times), "unit": UNIT, "cores": info["omp_threads"],
            "kind": "port",
            "sample": f"the first {steps} simulation steps of the configured 1 s run of the "
                      f"identical network ({sum(times):.1f} s), C++ oracle, OpenMP",
            "neuron_updates_per_s": float(N_NEURONS) * steps / sum(times), **info}
        del cpu
    return line


# ---- batched COBAHH instances (plain, batched, batched + gating surrogate) -------------------
BATCH_STEPS = 1000           # simulation steps per bench step of the batched workload (0.1 s)
BATCH_WORKLOAD = ("256 COBAHH instances, sizes round(exp(U[ln 1e3, ln 6.4e4])) (3.93e6 neurons), "
                  "p=0.02 (2.65e9 synapses), we~U[4,8] nS, delays U{1..50} steps, f32")
SURR_TOL = 1e-3


def _spike_hits(a, b):
    """(spikes (neuron, step) of a that b has within one step, spikes of a)."""
    keys = set(zip(b[0].tolist(), b[1].tolist()))
    hit = sum(1 for i, t in zip(a[0].tolist(), a[1].tolist())
              if (i, t) in keys or (i, t - 1) in keys or (i, t + 1) in keys)
    return hit, len(a[0])


def _spike_match(a, b):
    """Fraction of spikes (neuron, step) of a that b has within one step."""
    hit, n = _spike_hits(a, b)
    return hit / n if n else 1.0


def bench_batched(args, world, rank, local):
    import torch

    from brian2cuda_b200 import Network, models
    from brian2cuda_b200.surrogate import (GatingSurrogate, gating_targets, physiological,
                                           sample_states, surrogate_stats)
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream(device=local)
    from brian2cuda_b200.sharding import instance_cost, lpt_partition
    sizes_all, we_all = models.batch_sizes()
    n_all = int(sizes_all.sum())
    # one process per GPU: the instances are independent, so each rank simulates its own
    # share (longest processing time first) and only the timings are reduced
    mine = lpt_partition(instance_cost(sizes_all, 0.02), world)[rank]
    sizes, we = sizes_all[mine], we_all[mine]
    n_total = int(sizes.sum())
    runs = args.warmup + args.steps + 2

    def build(surr=None, judge=True, mon_entries=0):
        net = Network(DT, seed=models.SEED_BASE + 5, device=local, steps_per_graph=50,
                      stream=stream.cuda_stream)
        # one monitor buffer per population: the groups' capacities add up
        cap = -(-mon_entries // len(sizes)) if mon_entries else 0
        ids = models.build_cobahh_batch(net, sizes, we, monitor_capacity=cap)
        if surr is not None:
            surr.attach(net, ids["groups"][0], tol=SURR_TOL, judge=judge)
        net.finalize()
        net.store(0)
        return net, ids

    def timed(net, steps):
        for _ in range(args.warmup):
            net.restore(0)
            net.run(BATCH_STEPS)
        net.sync()
        barrier(world)
        torch.cuda.synchronize()
        launches0 = net.kernel_launches
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            net.restore(0)
            net.run(BATCH_STEPS)
        ev1.record(stream)
        ev1.synchronize()
        return max_over_ranks(ev0.elapsed_time(ev1), world), net.kernel_launches - launches0

    # ---- batched, exact integrator (the headline line)
    t0 = time.perf_counter()
    net, ids = build(mon_entries=int(n_total * BATCH_STEPS * DT * 40.0 * runs + n_total * 0.03 * 40))
    setup_s = time.perf_counter() - t0
    n_syn = sum(net.syn_count(s_) for s_ in ids["syns"])
    offs = [net.group_offset(g) for g in ids["groups"]]
    outdeg = np.zeros(max(o + int(n) for o, n in zip(offs, sizes)), np.int64)
    for g, o, n in zip(ids["groups"], offs, sizes):
        outdeg[o:o + int(n)] = net.out_degree(g)
    net.run(300)
    tune = net.autotune(trial_steps=100)
    start = net.spikes_recorded(ids["groups"][0])
    clocks = Clocks(local)
    ms_total, launches = timed(net, args.steps)
    clk = clocks.stop()
    # synaptic events of the timed runs (the warm-up runs repeat the same run from the same
    # checkpoint): recorded spikes x out-degree, per run
    idx, _, _ = net.spikes_fetch_population(ids["groups"][0], start, cap=1 << 27)
    per_run = 1.0 / max(1, args.warmup + args.steps)
    nspk = len(idx) * per_run * args.steps
    events = float(outdeg[idx].sum()) * per_run * args.steps
    del idx
    seconds = ms_total / 1e3
    value = float(n_all) * BATCH_STEPS * args.steps / seconds
    events_per_s = sum_over_ranks(events, world) / seconds
    nspk = sum_over_ranks(nspk, world)
    n_syn = int(sum_over_ranks(float(n_syn), world))
    net.restore(0)
    prof, _ = net.profile_graph(200)
    hbm, peak_kind = peaks()
    neuron_ms = min([ms for k, ms in prof if k == 1][0], ms_total / (args.steps * BATCH_STEPS))
    neuron_bytes = float(BYTES_NEURON_UPDATE * n_total)
    achieved = neuron_bytes / (neuron_ms * 1e-3) / 1e9
    # raster of the exact form, first 300 steps, for the surrogate comparison
    net.close()
    ref_net, ref_ids = build(mon_entries=int(n_total * 300 * DT * 200.0))
    ref_net.run(300)
    ref_ras = {g: ref_net.spikes(g) for g in ref_ids["groups"][-16:]}
    # ---- gating surrogate: training data from the batched net's own trajectories (the three
    # largest instances every 5 steps of the first 500), 1e7 transitions, exact targets
    ref_net.restore(0)
    big = [ref_ids["groups"][int(k)] for k in np.argsort(sizes)[-3:]]
    xs = []
    for _ in range(100):
        ref_net.run(5)
        xs.extend(sample_states(ref_net, g) for g in big)
    ref_net.close()
    x = physiological(torch.cat(xs))
    x = x[torch.randperm(len(x), device=x.device)[:10_000_000]].contiguous()
    t = gating_targets(models.cobahh_hh(), DT, x)
    surr = GatingSurrogate(device=local, seed=3)
    t0 = time.perf_counter()
    losses = surr.fit(x, t, epochs=400, batch=32768, lr=3e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del x, t
    snet, sids = build(surr, judge=True, mon_entries=int(n_total * 300 * DT * 200.0))
    snet.run(300)
    s_ras = {g: snet.spikes(g) for g in sids["groups"][-16:]}
    # pooled over the instances, in both directions (exact spikes the surrogate run has, and
    # surrogate spikes the exact run has), and the worst single instance
    hits = np.zeros((2, 2))
    worst = 1.0
    for g, g2 in zip(ref_ras, s_ras):
        for d, (a, b) in enumerate(((ref_ras[g], s_ras[g2]), (s_ras[g2], ref_ras[g]))):
            h, n = _spike_hits(a, b)
            hits[d] += (h, n)
            worst = min(worst, h / n if n else 1.0)
    hits = np.array([[sum_over_ranks(float(v), world) for v in row] for row in hits])
    match = float(min(hits[0, 0] / max(1.0, hits[0, 1]), hits[1, 0] / max(1.0, hits[1, 1])))
    worst = 1.0 - max_over_ranks(1.0 - worst, world)
    snet.restore(0)
    u0, f0 = surrogate_stats(snet, sids["groups"][0])
    s_ms, _ = timed(snet, args.steps)
    u1, f1 = surrogate_stats(snet, sids["groups"][0])
    snet.close()
    surr_value = float(n_all) * BATCH_STEPS * args.steps / (s_ms / 1e3)
    u_all = sum_over_ranks(float(u1 - u0), world)
    f_all = sum_over_ranks(float(f1 - f0), world)
    # ---- plain exact form: every instance its own network, one after another
    plain_ms = 0.0
    plain_steps = 200
    for k, (n_k, w_k) in enumerate(zip(sizes.tolist(), we.tolist())):
        pn = Network(DT, seed=models.SEED_BASE + 5, device=local, stream=stream.cuda_stream)
        models.build_cobahh(pn, n=int(n_k), we=float(w_k), seed_offset=100 + k)
        pn.finalize()
        pn.run(50)
        pn.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pn.run(plain_steps)
        e1.record(stream)
        e1.synchronize()
        plain_ms += e0.elapsed_time(e1)
        pn.close()
    plain_value = float(n_all) * plain_steps / (max_over_ranks(plain_ms, world) / 1e3)
    line = {
        "metric": "neuron-updates/s", "value": value, "unit": "neuron-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_total / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "sim_steps_per_step": BATCH_STEPS,
                   "instances": len(sizes_all), "neurons": n_all, "synapses": n_syn,
                   "parallelism": f"instances sharded over {world} rank(s), longest first",
                   "l2": "working set > L2 (21 GB)"},
        "synaptic_events_per_s": events_per_s,
        "spikes_per_run": nspk / max(1, args.steps),
        "setup_s": setup_s,
        "autotune": tune,
        "plain": {"neuron_updates_per_s": plain_value,
                  "how": f"each instance its own network, {plain_steps} steps each, "
                         "one after another (the unbatched exact-integrator form)"},
        "surrogate": {"neuron_updates_per_s": surr_value, "vs_plain": surr_value / plain_value,
                      "vs_batched_exact": surr_value / value, "tol": SURR_TOL, "judge": True,
                      "fallback_frac": f_all / max(1.0, u_all),
                      "raster_match_within_1dt_300_steps_last_16_instances": match,
                      "raster_match_worst_instance": worst,
                      "raster_spikes_exact": hits[0, 1],
                      "train_s": train_s, "train_loss": losses[-1],
                      "dataset": "1e7 exact transitions from the batched net's trajectories",
                      "training": "400 epochs, batch 32768, Adam lr 3e-3 with cosine decay"},
        "batched_vs_plain": value / plain_value,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": _traffic_lookup("hh_stream_kernel"),
                     "kernel": "neuron (HH update+threshold+compaction, hh_stream_kernel)",
                     "kernel_ms": neuron_ms, "peak_source": peak_kind,
                     "bytes_per_launch": neuron_bytes},
        "kernel_ms_mean_per_launch": {("neuron" if k == 1 else "delivery" if k == 6 else
                                       f"site {k}"): ms for k, ms in prof},
        "gpu_launches": launches,
        "clocks": clk,
    }
    return line


# ---- CUBA, STDP and multicompartment workloads ------------------------------------------------
WORKLOADS = {
    "cuba": "CUBA 4000 LIF (3200 exc / 800 inh), f64, exact integration, p=0.02 (~3.2e5 "
            "synapses), no delay, 1 s simulated",
    "stdp": "1e4 Poisson inputs at 15 Hz -> 1e3 LIF all-to-all (1e7 synapses), additive STDP "
            "(on_pre + on_post), f32, 1 s simulated per step (the configured run is 10 s)",
    "hines": "1024 multicompartment HH neurons, random binary trees of 200-1000 compartments, "
             "f64 cable solve, f32 channels, dt=0.025 ms, 200 ms simulated (8000 steps)",
    "propagation": "spike propagation at high load: 1e5 Poisson neurons at 300 Hz -> 1e5 "
                   "COBAHH neurons (first 80 % -> ge += 6 nS, last 20 % -> gi += 67 nS), "
                   "p=0.02 (2e8 synapses), delays U{1..50} steps, f32; ~6e6 synaptic events "
                   "per step, 0.1 s simulated per step",
}
PROP_RATE = 300.0
BYTES = {"cuba_neuron": 58, "cuba_event": 20, "stdp_neuron": 16, "poisson": 4,
         "stdp_pre": 40, "stdp_post": 32, "hines_comp": 136}


def build_propagation(net, monitor_capacity=0, rate=PROP_RATE):
    """The propagation workload: Poisson input population S (rate in Hz) driving a COBAHH
    population P through COBAHH's synapse shapes (no recurrent synapses)."""
    from brian2cuda_b200 import models
    n = N_NEURONS
    S = net.poisson_group(n, rate, "float32")
    P = net.hh_group(n, models.cobahh_hh(), "float32")
    models.cobahh_init(net, P, n, models.rng_for(5))
    ne = int(0.8 * n)
    seed = models.SEED_BASE + 5
    net.synapses_random(S, P, "ge", P_CONNECT, DMIN, DMAX, 6e-9, seed, pre_range=(0, ne))
    net.synapses_random(S, P, "gi", P_CONNECT, DMIN, DMAX, 67e-9, seed + 7, pre_range=(ne, n))
    if monitor_capacity:
        net.spike_monitor(S, monitor_capacity)
    return {"S": S, "P": P}


def _line_base(args, world, metric, value, unit, ms_per_step, workload, config, dtype):
    return {"metric": metric, "value": value, "unit": unit, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic", "config": dict({"workload": workload}, **config)}


def _roofline(bytes_per_launch, ms, kernel, step_ms=None):
    """ms: the launch's mean device time per step inside the step graphs, measured with
    event-record nodes around it; those nodes lengthen a launch by microseconds, so where
    that exceeds the step's own device time over the timed region (step_ms), the step time
    (an upper bound on the launch's duration) is used instead."""
    hbm, kind = peaks()
    timing = "in-graph device time (event-record nodes around the launch)"
    if step_ms is not None and ms > step_ms:
        ms = step_ms
        timing = ("device time per simulation step over the timed region (CUDA events), an "
                  "upper bound on the launch's duration: achieved and frac are lower bounds")
    achieved = bytes_per_launch / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": _traffic_lookup(kernel), "kernel": kernel,
            "kernel_ms": ms, "peak_source": kind, "bytes_per_launch": bytes_per_launch,
            "timing": timing}


def _timed_net_runs(net, stream, args, world, local, steps_per_run):
    import torch
    for _ in range(args.warmup):
        net.restore(0)
        net.run(steps_per_run)
    net.sync()
    barrier(world)
    torch.cuda.synchronize()
    launches0 = net.kernel_launches
    clocks = Clocks(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        net.restore(0)
        net.run(steps_per_run)
    ev1.record(stream)
    ev1.synchronize()
    clk = clocks.stop()
    return max_over_ranks(ev0.elapsed_time(ev1), world), net.kernel_launches - launches0, clk


def bench_small(args, world, rank, local):
    """CUBA, STDP or the multicompartment batch (args.workload), with the oracle port timed
    on the host cores beside it."""
    import torch

    from brian2cuda_b200 import Network, models
    from oracle.oracle import OracleHines, OracleNet
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream(device=local)
    wl = args.workload
    line = None
    if wl == "cuba":
        steps_run = 10_000
        net = Network(DT, seed=models.SEED_BASE, device=local, stream=stream.cuda_stream)
        ids = models.build_cuba(net, n=4000, dtype="float64")
        net.finalize()
        net.store(0)
        P = ids["P"]
        outdeg = net.out_degree(P).astype(np.int64)
        net.run(500)
        # trials of 500 steps: ten chunks each, so the comparison of the step's forms (the
        # per-step kernels, the small-network path's one launch per chunk) is not one replay's
        tune = net.autotune(trial_steps=500)
        start = net.spikes_recorded(P)
        ms, launches, clk = _timed_net_runs(net, stream, args, world, local, steps_run)
        idx, _, _ = net.spikes_fetch(P, start, cap=1 << 26)
        runs = args.warmup + args.steps
        events = float(outdeg[idx].sum()) / runs * args.steps
        nspk = len(idx) / runs
        net_mode = net.run_mode
        net.restore(0)
        prof, _ = net.profile_graph(2000)
        sec = ms / 1e3
        value = events * world / sec
        nb = BYTES["cuba_neuron"] * 4000.0
        db = BYTES["cuba_event"] * events / (args.steps * steps_run)
        dom = max(prof, key=lambda kv: kv[1])
        step_ms = ms / (args.steps * steps_run)
        if net_mode == "small":
            # one launch runs a chunk of steps (update and delivery): its time per step is
            # the step's
            roof = _roofline(nb + db, step_ms, "small_pull_kernel / small_cluster_kernel "
                             "(small-network path: update and delivery)", step_ms)
            roof["timing"] = ("device time per simulation step over the timed region (CUDA "
                              "events): one launch runs 50 steps")
        elif dom[0] == 1:
            roof = _roofline(nb, dom[1], "lif_step_kernel", step_ms)
        else:
            roof = _roofline(db, dom[1], "deliver_add_batch_kernel", step_ms)
        line = _line_base(args, world, "synaptic events/s", value, "events/s",
                          ms / args.steps, WORKLOADS[wl],
                          {"sim_steps_per_step": steps_run, "neurons": 4000,
                           "synapses": ids["n_syn"], "parallelism": f"replicas x{world}",
                           "l2": "working set < L2 (the net is 2.6 MB): no flush"},
                          "f64")
        line.update({"neuron_updates_per_s": 4000.0 * steps_run * args.steps * world / sec,
                     "run_mode": net_mode,
                     "firing_rate_hz": nspk / (4000 * steps_run * DT), "roofline": roof,
                     "kernel_ms_mean_per_launch": {f"site {k}": v for k, v in prof},
                     "autotune": tune, "gpu_launches": launches, "clocks": clk})
        net.close()
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            orc = OracleNet(DT, f32=False)
            oids = models.build_cuba(orc, n=4000, dtype="float64")
            orc.finalize()
            t0 = time.perf_counter()
            orc.run(steps_run)
            el = time.perf_counter() - t0
            oi, _ = orc.spikes(oids["P"])
            line["cpu_baseline"] = {"value": float(outdeg[oi].sum()) / el, "unit": "events/s",
                                    "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"the full 1 s run ({el:.1f} s), C++ oracle"}
    elif wl == "stdp":
        steps_run = 10_000
        net = Network(DT, seed=models.SEED_BASE + 2, device=local, stream=stream.cuda_stream)
        # per population; the output neurons (no refractory period) can fire every step
        cap = int(1000 * steps_run * 1.05 * (args.warmup + args.steps + 1))
        ids = models.build_stdp(net, monitor_capacity=cap)
        net.finalize()
        net.store(0)
        tune = net.autotune(trial_steps=50)
        s_in = net.spikes_recorded(ids["inp"])
        ms, launches, clk = _timed_net_runs(net, stream, args, world, local, steps_run)
        runs = args.warmup + args.steps
        n_in = len(net.spikes_fetch(ids["inp"], s_in, cap=1 << 26)[0]) / runs * args.steps
        n_out = len(net.spikes_fetch(ids["out"], s_in, cap=1 << 26)[0]) / runs * args.steps
        ev_pre, ev_post = n_in * 1000.0, n_out * 10_000.0
        net.restore(0)
        prof, _ = net.profile_graph(2000)
        sec = ms / 1e3
        value = (ev_pre + ev_post) * world / sec
        per_launch = {1: None, 2: BYTES["stdp_pre"] * ev_pre / (args.steps * steps_run),
                      3: BYTES["stdp_post"] * ev_post / (args.steps * steps_run)}
        dom = max(prof, key=lambda kv: kv[1])
        kname = {1: "poisson/lif step", 2: "deliver_stdp_pre_kernel",
                 3: "deliver_stdp_post_kernel"}.get(dom[0], "site")
        b = per_launch.get(dom[0]) or (BYTES["stdp_neuron"] * 1000 + BYTES["poisson"] * 10_000)
        line = _line_base(args, world, "synaptic events/s", value, "events/s",
                          ms / args.steps, WORKLOADS[wl],
                          {"sim_steps_per_step": steps_run, "neurons": 11_000,
                           "synapses": 10_000_000, "parallelism": f"replicas x{world}",
                           "l2": "working set > L2 (1e7 synapses x 4 f32 variables = 160 MB)"},
                          "f32")
        roof = _roofline(b, dom[1], kname, ms / (args.steps * steps_run))
        if kname == "deliver_stdp_post_kernel":
            post_grouped = any(t["site_kind"] == 8 and t["choice_a"] == 1 for t in tune)
            roof["traffic"] = _traffic_lookup(kname + ("" if post_grouped else "@synorder"))
        line.update({"on_pre_events_per_s": ev_pre / sec, "on_post_events_per_s": ev_post / sec,
                     "neuron_updates_per_s": 11_000.0 * steps_run * args.steps * world / sec,
                     "roofline": roof,
                     "kernel_ms_mean_per_launch": {f"site {k}": v for k, v in prof},
                     "autotune": tune, "gpu_launches": launches, "clocks": clk})
        net.close()
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            orc = OracleNet(DT, f32=True)
            oids = models.build_stdp(orc, monitor_capacity=cap)
            orc.finalize()
            # the oracle's Poisson group reads supplied uniforms (the GPU draws them with cuRAND)
            sample = 250
            orc.set_uniforms(oids["inp"], np.random.default_rng(7).random((sample, 10_000),
                                                                          dtype=np.float32))
            t0 = time.perf_counter()
            orc.run(sample)
            el = time.perf_counter() - t0
            oin = len(orc.spikes(oids["inp"])[0])
            oout = len(orc.spikes(oids["out"])[0])
            line["cpu_baseline"] = {"value": (oin * 1000.0 + oout * 10_000.0) / el,
                                    "unit": "events/s", "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"the first {sample} steps of the run "
                                              f"({el:.1f} s), C++ oracle"}
    elif wl == "propagation":
        steps_run = 1000
        runs = args.warmup + args.steps
        cap = int(N_NEURONS * PROP_RATE * DT * steps_run * 1.1 * (runs + 2)) + 100_000
        net = Network(DT, seed=models.SEED_BASE + 5, device=local, stream=stream.cuda_stream)
        ids = build_propagation(net, monitor_capacity=cap)
        net.finalize()
        S = ids["S"]
        outdeg = net.out_degree(S).astype(np.int64)
        net.run(2 * DMAX)   # every delay slot of the ring holds spikes from here on
        net.store(0)
        tune = net.autotune(trial_steps=100)
        start = net.spikes_recorded(S)
        ms, launches, clk = _timed_net_runs(net, stream, args, world, local, steps_run)
        idx, st, _ = net.spikes_fetch(S, start, cap=net.spikes_recorded(S) - start + 16)
        events = float(outdeg[idx].sum()) / runs * args.steps
        nspk = len(idx) / runs * args.steps
        del idx, st
        net.restore(0)
        prof, _ = net.profile_graph(200)
        sec = ms / 1e3
        value = events * world / sec
        per_step_events = events / (args.steps * steps_run)
        per_step_bundles = nspk / (args.steps * steps_run) * (DMAX - DMIN + 1)
        db = BYTES_EVENT * per_step_events + BYTES_BUNDLE * per_step_bundles
        dmsk = [m for k, m in prof if k == 6]
        roof = _roofline(db, dmsk[0], "deliver_add_batch_kernel", ms / (args.steps * steps_run))
        roof["traffic"] = _traffic_lookup("deliver_add_batch_kernel@propagation")
        roof["note"] = ("12 B per event (target index 4 B + target read/write 8 B) + 8 B per "
                        "(spike, delay) bundle; bound: one L2 atomic per event")
        from brian2cuda_b200.network import atomic_rate
        loaded, hashed, dsmem = atomic_rate(2 * N_NEURONS, 60_000_000, device=local,
                                            stream=stream.cuda_stream)
        d_rate = per_step_events / (roof["kernel_ms"] * 1e-3)
        roof["events_per_s_in_kernel"] = d_rate
        roof["atomic_ceiling_events_per_s"] = {"index_loaded": loaded,
                                               "index_in_registers": hashed,
                                               "cluster_shared_memory": dsmem}
        roof["frac_of_atomic_ceiling"] = d_rate / loaded
        line = _line_base(args, world, "synaptic events/s", value, "events/s",
                          ms / args.steps, WORKLOADS[wl],
                          {"sim_steps_per_step": steps_run, "neurons": 2 * N_NEURONS,
                           "synapses": int(outdeg.sum()), "parallelism": f"replicas x{world}",
                           "l2": "working set > L2 (0.8 GB of synapse targets)"},
                          "f32")
        line.update({"events_per_sim_step": per_step_events,
                     "input_spikes_per_sim_step": nspk / (args.steps * steps_run),
                     "roofline": roof, "autotune": tune,
                     "kernel_ms_mean_per_launch": {
                         ("delivery" if k == 6 else f"site {k}"): v for k, v in prof},
                     "gpu_launches": launches, "clocks": clk})
        net.close()
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            sample = 20
            orc = OracleNet(DT, f32=True)
            oids = build_propagation(orc, monitor_capacity=N_NEURONS * sample)
            orc.finalize()
            orc.set_uniforms(oids["S"], np.random.default_rng(9).random(
                (2 * DMAX + sample, N_NEURONS), dtype=np.float32))
            orc.run(2 * DMAX)
            n0 = len(orc.spikes(oids["S"])[0])
            t0 = time.perf_counter()
            orc.run(sample)
            el = time.perf_counter() - t0
            oi = orc.spikes(oids["S"])[0]
            # events delivered in the sample: the due bundles of the last 50 steps' spikes,
            # about the steady per-step count of the GPU run
            line["cpu_baseline"] = {"value": per_step_events * sample / el, "unit": "events/s",
                                    "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"{sample} steps after a {2 * DMAX}-step fill "
                                              f"({el:.1f} s, {len(oi) - n0} input spikes), "
                                              "C++ oracle; events counted at the GPU run's "
                                              "mean per step"}
    elif wl == "hines":
        steps_run = 8000
        net = Network(25e-6, seed=models.SEED_BASE + 3, device=local, stream=stream.cuda_stream)
        hb, morph, params, current = models.build_hines(net, n_neurons=1024)
        for _ in range(args.warmup):
            hb.run(steps_run)
        net.sync()
        torch.cuda.synchronize()
        clocks = Clocks(local)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            hb.run(steps_run)
        ev1.record(stream)
        ev1.synchronize()
        net.sync()
        el = max_over_ranks(ev0.elapsed_time(ev1) / 1e3, world)
        clk = clocks.stop()
        n_comp = hb.n_comp
        value = float(n_comp) * steps_run * args.steps * world / el
        line = _line_base(args, world, "compartment-updates/s", value, "compartment-updates/s",
                          1e3 * el / args.steps, WORKLOADS[wl],
                          {"sim_steps_per_step": steps_run, "neurons": 1024,
                           "compartments": n_comp, "parallelism": f"replicas x{world}",
                           "l2": "state held in shared memory across chunks of up to 1000 "
                                 "steps; per chunk it moves through HBM once"},
                          "f64")
        line.update({"neuron_updates_per_s": 1024.0 * steps_run * args.steps * world / el,
                     "roofline": _roofline(BYTES["hines_comp"] * n_comp * steps_run,
                                           1e3 * el / args.steps, "hines_kernel"),
                     "timing": "CUDA events on the net's stream around the runs (one "
                               "kernel per 1000-step chunk)",
                     "gpu_launches": args.steps * (steps_run // 1000), "clocks": clk})
        line["roofline"]["timing"] = ("CUDA events on the net's stream around the runs, per "
                                      "8000-step run (eight launches of 1000 steps)")
        line["roofline"]["note"] = ("achieved = algorithmic 136 B per compartment-step / time; "
                                    "the kernel keeps the state in shared memory, so HBM is "
                                    "not what bounds it")
        net.close()
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            orc = OracleHines(25e-6, morph["comp_off"], morph["sec_off"], morph["sec_start"],
                              morph["sec_end"], morph["sec_parent"], morph["diameter"],
                              morph["length"], params, f32=True)
            for k_, v_ in models.hines_rest_state().items():
                orc.set_state(k_, v_)
            orc.set_current(current)
            t0 = time.perf_counter()
            orc.run(200)
            el2 = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": float(n_comp) * 200 / el2,
                                    "unit": "compartment-updates/s", "cores": os.cpu_count(),
                                    "kind": "port",
                                    "sample": f"200 of the 8000 steps ({el2:.1f} s), C++ oracle"}
    return line


def kernel_case(name: str):
    """Small cases for ncu captures of single kernels (inputs above the L2 size, a few GB at
    most): hh4m = 4e6 HH neurons (hh_stream_kernel), surrogate1m = 1e6 HH neurons with the
    gating surrogate attached (hh_surrogate_step_kernel), mlp_train = one epoch of surrogate
    training on 2e6 transitions (mlp_grad_kernel, mlp_adam_kernel), propagation /
    propagation3000 = the propagation workload at 300 / 3000 Hz of input, 100 filling steps
    then 20 profiled ones (deliver_add_batch_kernel, 6e6 / 6e7 events per step), stdp /
    stdp_synorder = the STDP workload with its records grouped by postsynaptic neuron / in
    synapse order, 200 steps then 20 profiled ones (deliver_stdp_post_kernel), hines = the
    1024-neuron multicompartment batch for one 1000-step launch (hines_kernel), model = a
    generated model (noisy adaptive LIF, 8e6 neurons, 20 steps: model_step_kernel), batched =
    the 256-instance batched workload for 500 steps (20 GB on the device: a launch list only)."""
    import torch

    from brian2cuda_b200 import Network, models
    from brian2cuda_b200.surrogate import GatingSurrogate, gating_targets
    if name in ("hh4m", "surrogate1m"):
        n = 4_000_000 if name == "hh4m" else 1_000_000
        net = Network(DT, seed=1, graphs=False)
        P = net.hh_group(n, models.cobahh_hh(), "float32")
        models.cobahh_init(net, P, n, np.random.default_rng(0))
        s = None
        if name == "surrogate1m":
            s = GatingSurrogate(seed=3)
            s.attach(net, P, tol=SURR_TOL, judge=True)
        net.finalize()
        net.run(6)
        net.sync()
        net.close()
    elif name == "hines":
        net = Network(25e-6, seed=models.SEED_BASE + 3)
        hb, _, _, _ = models.build_hines(net, n_neurons=1024)
        hb.run(1000)            # one launch of the 1000-step chunk
        net.sync()
        net.close()
    elif name in ("stdp", "stdp_synorder"):
        net = Network(DT, seed=models.SEED_BASE + 2)
        models.build_stdp(net)
        net.finalize()
        net.tune_apply([{"site_kind": 8, "site_index": 0, "choice_b": 0,
                         "choice_a": 1 if name == "stdp" else 0}])
        net.run(200)            # 200 launches of each kernel before the profiled ones
        net.profile(20)
        net.sync()
        net.close()
    elif name in ("propagation", "propagation3000"):
        net = Network(DT, seed=models.SEED_BASE + 5)
        build_propagation(net, rate=PROP_RATE if name == "propagation" else 3000.0)
        net.finalize()
        net.run(2 * DMAX)       # 100 delivery launches before the profiled ones
        net.profile(20)
        net.sync()
        net.close()
    elif name == "model":
        # a generated model (noisy adaptive LIF, Euler-Maruyama with one cuRAND normal per
        # neuron and step), 8e6 neurons, float32 (17 B per neuron and step: above the L2):
        # 20 launches of model_step_kernel
        from brian2cuda_b200.lowering import Script
        s = Script(dt=DT, seed=4, dtype="float32",
                   namespace=dict(tau=10e-3, tauw=100e-3, a=0.5, sigma=2e-3, El=-70e-3,
                                  Vt=-50e-3, Vr=-65e-3, b=1e-3, I0=22e-3))
        G = s.NeuronGroup(8_000_000, """dv/dt = (El - v - w + I0) / tau + sigma * xi * tau**-0.5
                                        : volt
                                        dw/dt = (a * (v - El) - w) / tauw : volt""",
                          threshold="v > Vt", reset="v = Vr; w += b", refractory=2e-3)
        G.v = "El + rand()*20*mV"
        net = Network(DT, seed=4, graphs=False)
        s.lower().build(net)
        net.run(20)
        net.sync()
        net.close()
    elif name == "batched":
        # the 256-instance batched workload with the built-in launch shapes: 300 steps (the
        # initial burst), then 200 more (for a launch list of the quiet phase)
        sizes, we = models.batch_sizes()
        net = Network(DT, seed=models.SEED_BASE + 5, steps_per_graph=50)
        models.build_cobahh_batch(net, sizes, we)
        net.finalize()
        net.run(500)
        net.sync()
        net.close()
    elif name == "mlp_train":
        g = torch.Generator(device="cuda").manual_seed(0)
        x = torch.rand((2_000_000, 4), device="cuda", generator=g)
        x[:, 0] = x[:, 0] * 0.13 - 0.085
        t = gating_targets(models.cobahh_hh(), DT, x)
        s = GatingSurrogate(seed=3)
        s.fit(x, t, epochs=1, batch=32768, lr=1e-2)
        torch.cuda.synchronize()


def _traffic_lookup(kernel: str):
    """DRAM bytes per launch from the committed ncu summary, when one exists."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(kernel)
    except Exception:
        return None


if __name__ == "__main__":
    main()
