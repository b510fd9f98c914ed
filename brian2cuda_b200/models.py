"""Synthetic builders for the benchmark networks (seeded; SI units).

Each builder takes a backend with the `Network` interface (the GPU `Network`, or any object
with the same methods) and returns a dict of group / synapse ids.  Shapes and parameters
follow the reference's own model scripts:

  * CUBA      — examples/cuba.py:118-143
  * COBAHH    — examples/cobahh.py:141-215
  * STDP      — examples/stdp.py:100-186, brian2cuda/tests/features/speed.py:618-663
  * multicompartment HH — examples/compartmental/hh_with_spikes_cuda.py:20-50
"""
from __future__ import annotations

import math

import numpy as np

from .network import HH, LIF, STDP, HinesParams

mV, ms, nS, um = 1e-3, 1e-3, 1e-9, 1e-6
SEED_BASE = 20261203


def rng_for(config_id: int) -> np.random.Generator:
    return np.random.default_rng(SEED_BASE + config_id)


def delay_steps(delay_seconds, dt: float) -> np.ndarray:
    """Brian2's rounding of a delay to whole steps, (int)(delay/dt + 0.5)
    (brian2cuda/templates/synapses_push_spikes.cu:375)."""
    return (np.asarray(delay_seconds, dtype=np.float64) / dt + 0.5).astype(np.int32)


def bernoulli_pairs(rng: np.random.Generator, n_pre: int, n_post: int, p: float):
    """All (i, j) with an independent Bernoulli(p) draw each, in (i, j) order
    (Brian2 `connect(p=...)`); geometric skipping keeps this O(synapses)."""
    total = n_pre * n_post
    if p <= 0 or total == 0:
        return np.zeros(0, np.int32), np.zeros(0, np.int32)
    if p >= 1:
        lin = np.arange(total, dtype=np.int64)
    else:
        est = int(total * p + 10 * math.sqrt(total * p) + 100)
        gaps = rng.geometric(p, size=est).astype(np.int64)
        lin = np.cumsum(gaps) - 1
        while lin[-1] < total:
            more = np.cumsum(rng.geometric(p, size=est).astype(np.int64)) + lin[-1]
            lin = np.concatenate([lin, more])
        lin = lin[lin < total]
    return (lin // n_post).astype(np.int32), (lin % n_post).astype(np.int32)


# ---- CUBA (configuration: 4000 LIF, float64, exact integration) -------------------------------
def cuba_lif() -> LIF:
    return LIF(El=-49 * mV, taum=20 * ms, taue=5 * ms, taui=10 * ms, ke=1.0, ki=1.0,
               Vt=-50 * mV, Vr=-60 * mV, refractory=5 * ms, has_threshold=True, has_reset=True,
               unless_refractory=True)


def build_cuba(net, n: int = 4000, p: float = 0.02, dtype="float64", seed_offset: int = 0,
               monitor: bool = True):
    rng = rng_for(0 + seed_offset)
    P = net.lif_group(n, cuba_lif(), dtype)
    Vt, Vr = -50 * mV, -60 * mV
    net.set_state(P, "v", Vr + rng.random(n) * (Vt - Vr))
    ne = int(0.8 * n)
    i, j = bernoulli_pairs(rng, n, n, p)
    exc = i < ne
    we = 60 * 0.27 / 10 * mV      # examples/cuba.py:135
    wi = -20 * 4.5 / 10 * mV      # examples/cuba.py:136
    Ce = net.synapses(P, P, "ge", i[exc], j[exc], w_scalar=we)
    Ci = net.synapses(P, P, "gi", i[~exc], j[~exc], w_scalar=wi)
    if monitor:
        net.spike_monitor(P, 4_000_000)
    return {"P": P, "Ce": Ce, "Ci": Ci, "n_syn": int(len(i))}


# ---- COBAHH (configuration: 1e5 HH, float32, exponential Euler, delays 1..50 steps) ------------
def cobahh_hh() -> HH:
    area = 20000 * um * um
    return HH(Cm=1e-2 * area, gl=5e-5 * 1e4 * area, El=-60 * mV, EK=-90 * mV, ENa=50 * mV,
              gNa=100e-3 * 1e4 * area, gK=30e-3 * 1e4 * area, VT=-63 * mV, Ee=0.0,
              Ei=-80 * mV, taue=5 * ms, taui=10 * ms, Vthr=-20 * mV, refractory=3 * ms)


def cobahh_init(net, P, n: int, rng: np.random.Generator):
    """v0 = El + 5 mV * N(0, 1); ge, gi as examples/cobahh.py:213-215."""
    El = -60 * mV
    net.set_state(P, "v", El + 5 * mV * rng.standard_normal(n))
    net.set_state(P, "ge", (rng.standard_normal(n) * 1.5 + 4) * 10 * nS)
    net.set_state(P, "gi", (rng.standard_normal(n) * 12 + 20) * 10 * nS)


def build_cobahh(net, n: int = 100_000, p: float = 0.02, dmin: int = 1, dmax: int = 50,
                 we: float = 6 * nS, wi: float = 67 * nS, dtype="float32", seed_offset: int = 0,
                 monitor_capacity: int = 0, generated: bool = True):
    """One HH group P; Ce = Synapses(P[:0.8n], P, on_pre='ge += we'), Ci from P[0.8n:] with
    'gi += wi'; each connect(p) with per-synapse delays uniform on [dmin, dmax] steps.
    generated=True draws the connectivity on the GPU (Philox), else with numpy."""
    rng = rng_for(1 + seed_offset)
    P = net.hh_group(n, cobahh_hh(), dtype)
    cobahh_init(net, P, n, rng)
    ne = int(0.8 * n)
    seed = SEED_BASE + 1 + seed_offset
    if generated:
        Ce = net.synapses_random(P, P, "ge", p, dmin, dmax, we, seed, pre_range=(0, ne))
        Ci = net.synapses_random(P, P, "gi", p, dmin, dmax, wi, seed + 7, pre_range=(ne, n))
    else:
        i, j = bernoulli_pairs(rng, n, n, p)
        d = rng.integers(dmin, dmax + 1, size=len(i)).astype(np.int32)
        exc = i < ne
        Ce = net.synapses(P, P, "ge", i[exc], j[exc], w=np.full(exc.sum(), we), delay=d[exc])
        Ci = net.synapses(P, P, "gi", i[~exc], j[~exc], w=np.full((~exc).sum(), wi),
                          delay=d[~exc])
    if monitor_capacity:
        net.spike_monitor(P, monitor_capacity)
    return {"P": P, "Ce": Ce, "Ci": Ci}


def batch_sizes(n_instances: int = 256, lo: int = 1000, hi: int = 64000,
                seed_offset: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Sizes round(exp(U[ln lo, ln hi])) and excitatory weights U[4, 8] nS of the batched
    COBAHH instances (seeded)."""
    rng = rng_for(5 + seed_offset)
    sizes = np.rint(np.exp(rng.uniform(math.log(lo), math.log(hi), n_instances))).astype(np.int64)
    we = rng.uniform(4 * nS, 8 * nS, n_instances)
    return sizes, we


def build_cobahh_batch(net, sizes, we, p: float = 0.02, dmin: int = 1, dmax: int = 50,
                       wi: float = 67 * nS, dtype="float32", seed_offset: int = 0,
                       monitor_capacity: int = 0, instances=None):
    """Independent COBAHH instances in one network: instance k is build_cobahh's network with
    sizes[k] neurons and excitatory weight we[k].  The instances' groups share one population
    and their 2 x len(sizes) Synapses objects one projection, so every step is one neuron
    launch and one delivery launch whatever the number of instances.  `instances` (indices
    into sizes) builds only those instances, each with the seeds and initial state it has in
    the whole batch."""
    rng = rng_for(5 + seed_offset)
    keep = None if instances is None else set(int(k) for k in instances)
    groups, syns = [], []
    for k, (n, w) in enumerate(zip(np.asarray(sizes).tolist(), np.asarray(we).tolist())):
        if keep is not None and k not in keep:
            # consume this instance's draws of the initial state, as cobahh_init would
            rng.standard_normal(int(n))
            rng.standard_normal(int(n))
            rng.standard_normal(int(n))
            continue
        P = net.hh_group(int(n), cobahh_hh(), dtype)
        cobahh_init(net, P, int(n), rng)
        ne = int(0.8 * n)
        seed = SEED_BASE + 1000 + 2 * k + 1000 * seed_offset
        syns.append(net.synapses_random(P, P, "ge", p, dmin, dmax, float(w), seed,
                                        pre_range=(0, ne)))
        syns.append(net.synapses_random(P, P, "gi", p, dmin, dmax, wi, seed + 1,
                                        pre_range=(ne, int(n))))
        if monitor_capacity:
            net.spike_monitor(P, monitor_capacity)
        groups.append(P)
    return {"groups": groups, "syns": syns}


# ---- STDP (configuration: 1e4 Poisson @ 15 Hz -> 1e3 LIF, all-to-all, float32) ----------------
def stdp_lif() -> LIF:
    # dv/dt = (ge*(Ee - vr) + El - v)/taum, dge/dt = -ge/taue; threshold v > vt, reset v = vr
    Ee, vr, El = 0.0, -60 * mV, -74 * mV
    return LIF(El=El, taum=10 * ms, taue=5 * ms, taui=0.0, ke=Ee - vr, ki=0.0, Vt=-54 * mV,
               Vr=vr, refractory=0.0, has_threshold=True, has_reset=True,
               unless_refractory=False)


def stdp_rule(gmax: float = 0.01) -> STDP:
    taupre = taupost = 20 * ms
    dApre = 0.01 * gmax
    dApost = -dApre * taupre / taupost * 1.05
    return STDP(taupre=taupre, taupost=taupost, dApre=dApre, dApost=dApost, wmin=0.0,
                wmax=gmax, pre_adds_weight=True)


def build_stdp(net, n_in: int = 10_000, n_out: int = 1_000, rate: float = 15.0,
               dtype="float32", seed_offset: int = 0, monitor_capacity: int = 0):
    rng = rng_for(2 + seed_offset)
    gmax = 0.01
    inp = net.poisson_group(n_in, rate, dtype)
    out = net.lif_group(n_out, stdp_lif(), dtype)
    net.set_state(out, "v", -60 * mV)
    i = np.repeat(np.arange(n_in, dtype=np.int32), n_out)
    j = np.tile(np.arange(n_out, dtype=np.int32), n_in)
    w = rng.random(len(i)) * gmax
    S = net.synapses(inp, out, "ge", i, j, w=w, stdp=stdp_rule(gmax))
    if monitor_capacity:
        net.spike_monitor(inp, monitor_capacity)
        net.spike_monitor(out, monitor_capacity)
    return {"inp": inp, "out": out, "S": S}


# ---- multicompartment HH batch --------------------------------------------------------------------
def random_morphologies(n_neurons: int, rng: np.random.Generator, comp_range=(200, 1000),
                        sec_len=(2, 10), diam=(0.5 * um, 2 * um), length=(5 * um, 50 * um)):
    """Seeded random binary trees of cylindrical sections.  Each neuron gets a total
    compartment count drawn from comp_range; sections of sec_len compartments are attached,
    breadth-first, to random existing sections with fewer than two children."""
    comp_off, sec_off = [0], [0]
    starts, ends, parents, diameters, lengths = [], [], [], [], []
    for _ in range(n_neurons):
        total = int(rng.integers(comp_range[0], comp_range[1] + 1))
        nc = 0
        kids: list[int] = []
        sec_p: list[int] = []
        while nc < total:
            k = int(min(rng.integers(sec_len[0], sec_len[1] + 1), total - nc))
            if not sec_p:
                par = -1
            else:
                open_secs = [s for s in range(len(sec_p)) if kids[s] < 2]
                par = int(open_secs[int(rng.integers(len(open_secs)))])
                kids[par] += 1
            sec_p.append(par)
            kids.append(0)
            starts.append(nc)
            ends.append(nc + k)
            nc += k
        parents.extend(sec_p)
        d = rng.uniform(*diam, size=nc)
        L = rng.uniform(*length, size=nc)
        diameters.append(d)
        lengths.append(L)
        comp_off.append(comp_off[-1] + nc)
        sec_off.append(sec_off[-1] + len(sec_p))
    return {
        "comp_off": np.array(comp_off, np.int64), "sec_off": np.array(sec_off, np.int32),
        "sec_start": np.array(starts, np.int32), "sec_end": np.array(ends, np.int32),
        "sec_parent": np.array(parents, np.int32),
        "diameter": np.concatenate(diameters), "length": np.concatenate(lengths),
    }


def hines_rest_state():
    """Resting HH 1952 state (v = 0 from rest)."""
    return {"v": 0.0, "m": 0.0529, "h": 0.5961, "n": 0.3177}


def build_hines(net, n_neurons: int = 1024, channel_dtype="float32", seed_offset: int = 0,
                comp_range=(200, 1000)):
    rng = rng_for(3 + seed_offset)
    morph = random_morphologies(n_neurons, rng, comp_range=comp_range)
    params = HinesParams(channel_dtype=channel_dtype)
    hb = net.hines_batch(morph["comp_off"], morph["sec_off"], morph["sec_start"],
                         morph["sec_end"], morph["sec_parent"], morph["diameter"],
                         morph["length"], params)
    rest = hines_rest_state()
    for k, v in rest.items():
        hb.set_state(k, v)
    current = rng.uniform(0.2e-9, 1e-9, size=n_neurons)
    hb.set_current(current)
    return hb, morph, params, current
