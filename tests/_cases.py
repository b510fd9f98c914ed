"""Known-answer cases restated from the reference's own tests, without Brian2.

Each case takes `make(dt, **kw)` returning a backend with the `Network` interface (the CUDA
library or the CPU oracle), builds the network of the reference test, runs it and checks
the answer that test asserts.  Spike steps are exact integers here; the reference compares
spike times t = step*dt.
"""
from __future__ import annotations

import math

import numpy as np

from brian2cuda_b200.network import LIF, spike_steps

DT = 1e-4  # Brian2's defaultclock.dt


def _spike_steps(net, gid):
    idx, st = net.spikes(gid)
    return idx, st


def neuron_v1():
    """`NeuronGroup(N, 'v:1', threshold='v>1', reset='v=0')`."""
    return LIF(El=0.0, taum=math.inf, Vt=1.0, Vr=0.0)


def example_run(make):
    """brian2cuda/__init__.py:50-72: dv/dt = -v/tau, v0 = i/100, 1 ms later
    v == i/100 * exp(-1 ms / 10 ms)."""
    net = make(DT)
    G = net.lif_group(100, LIF(El=0.0, taum=10e-3, Vt=1.0, Vr=0.0, refractory=5e-3),
                      "float64")
    net.set_state(G, "v", np.arange(100) / 100.0)
    net.finalize()
    net.run(10)
    v = net.get_state(G, "v")
    np.testing.assert_allclose(v, np.arange(100) / 100 * np.exp(-1e-3 / 10e-3), rtol=1e-12)


def push_outer_loop(make):
    """test_synaptic_propagations.py:11-48: one input spike at t=0 to 15*1025 targets with
    delays alternating 0 and dt; even targets spike at dt, odd ones at 2 dt."""
    N = 1025 * 15
    net = make(DT)
    inp = net.spikegen_group(1, [0], [0])
    G = net.lif_group(N, neuron_v1(), "float64")
    j = np.arange(N)
    net.synapses(inp, G, "v", np.zeros(N, np.int32), j, w_scalar=1.1, delay=(j % 2))
    net.spike_monitor(G, 4 * N)
    net.finalize()
    net.run(3)
    idx, st = _spike_steps(net, G)
    assert len(idx) == N
    np.testing.assert_array_equal(np.sort(idx[st == 1]), np.arange(0, N, 2))
    np.testing.assert_array_equal(np.sort(idx[st == 2]), np.arange(1, N, 2))


def push_outer_loop2(make):
    """test_synaptic_propagations.py:51-150 with one post block: input 0 spikes in the first
    2048 steps with zero weight, input 1 once at step 2048 with weight 1.1 and delays
    j (j = 1024 gets 1023); target j then spikes at step 2049 + delay."""
    npb = 2048
    net = make(DT)
    inp = net.spikegen_group(2, [0] * npb + [1], np.arange(npb + 1))
    G = net.lif_group(npb, neuron_v1(), "float64")
    i = np.repeat([0, 1], npb).astype(np.int32)
    j = np.tile(np.arange(npb), 2).astype(np.int32)
    w = np.where(i == 0, 0.0, 1.1)
    d = j.copy()
    d[(i == 1) & (j == 1024)] = 1023
    net.synapses(inp, G, "v", i, j, w=w, delay=d)
    net.spike_monitor(G, 4 * npb)
    net.finalize()
    steps = 2 * npb + 2
    net.run(steps)
    idx, st = _spike_steps(net, G)
    assert len(idx) == npb
    for n in range(steps):
        got = np.sort(idx[st == n])
        if n <= npb or n == steps - 1:
            assert len(got) == 0, n
            continue
        s = n - (npb + 1)
        if s == 1023:
            exp = [1023, 1024]
        elif s == 1024:
            exp = []
        else:
            exp = [s]
        np.testing.assert_array_equal(got, exp, err_msg=f"step {n}")


def _circular(net, inp):
    G = net.lif_group(5, neuron_v1(), "float64")
    net.synapses(inp, G, "v", [0], [0], w_scalar=1.1, delay=0)
    net.synapses(inp, G, "v", [0], [1], w_scalar=1.1, delay=2)
    net.synapses(inp, G, "v", [0], [2], w_scalar=1.1, delay=5)
    net.synapses(inp, G, "v", [0, 0], [3, 4], w_scalar=1.1, delay=np.array([3, 4]))
    net.spike_monitor(G, 1000)
    return G


def circular_eventspaces(make):
    """test_synaptic_propagations.py:153-184 (and :343-374): homogeneous delays 0, 2, 5 and
    heterogeneous delays 3, 4; each target spikes the step after its effect arrives."""
    net = make(DT)
    inp = net.spikegen_group(1, [0], [0])
    G = _circular(net, inp)
    net.finalize()
    net.run(7)
    idx, st = _spike_steps(net, G)
    for neuron, step in [(0, 1), (1, 3), (2, 6), (3, 4), (4, 5)]:
        np.testing.assert_array_equal(st[idx == neuron], [step])


def circular_eventspaces_spikegenerator(make):
    """test_synaptic_propagations.py:187-227: input spikes in each of the first 12 steps,
    schedule with resets before synapses."""
    n = 12
    net = make(DT, reset_before_synapses=True)
    inp = net.spikegen_group(1, [0] * n, np.arange(n))
    G = _circular(net, inp)
    net.finalize()
    net.run(n + 6)
    idx, st = _spike_steps(net, G)
    for neuron, first in [(0, 1), (1, 3), (2, 6), (3, 4), (4, 5)]:
        np.testing.assert_array_equal(np.sort(st[idx == neuron]), np.arange(first, first + n))


def multiple_runs_scalar_delay(make):
    """test_network_multiple_runs.py:10-26: an always-spiking input, `v += 1` with delay dt,
    two runs of two steps; v at the start of each step is [0, 0, 1, 2]."""
    net = make(DT)
    inG = net.lif_group(1, LIF(taum=math.inf, Vt=-math.inf, has_reset=False), "float64")
    G = net.lif_group(1, LIF(taum=math.inf, has_threshold=False, has_reset=False), "float64")
    net.set_state(G, "v", 0.0)
    net.synapses(inG, G, "v", [0], [0], w_scalar=1.0, delay=1)
    net.finalize()
    trace = []
    for _run in range(2):
        for _ in range(2):
            trace.append(float(net.get_state(G, "v")[0]))
            net.run(1)
    assert trace == [0.0, 0.0, 1.0, 2.0]


def spikegenerator_extreme_period(make):
    """test_spikegenerator.py:12-27: SpikeGeneratorGroup(5, [0, 1, 2], [0, 1, 2] ms,
    period=1e6 s) run for 10 ms spikes i = [0, 1, 2] at t = [0, 1, 2] ms."""
    net = make(DT)
    SG = net.spikegen_group(5, [0, 1, 2], spike_steps(np.array([0, 1, 2]) * 1e-3, DT),
                            period=int(spike_steps(1e6, DT)))
    net.spike_monitor(SG, 100)
    net.finalize()
    net.run(100)
    idx, st = net.spikes(SG)
    np.testing.assert_array_equal(idx, [0, 1, 2])
    np.testing.assert_array_equal(st, [0, 10, 20])


def spikegenerator_period_repeat(make):
    """test_spikegenerator.py:30-66: one neuron with ten spikes 0.1 ms apart inside a 1 ms
    period; five runs of 1 ms each record all ten."""
    net = make(DT)
    SG = net.spikegen_group(1, np.zeros(10, np.int32), spike_steps(np.arange(0, 1, 0.1) * 1e-3, DT),
                            period=int(spike_steps(1e-3, DT)))
    net.spike_monitor(SG, 100)
    net.finalize()
    counts, seen = [], 0
    for _ in range(5):
        net.run(10)
        n = len(net.spikes(SG)[0])
        counts.append(n - seen)
        seen = n
    assert counts == [10] * 5
    _, st = net.spikes(SG)
    np.testing.assert_array_equal(st, np.arange(50))


def spikegenerator_rounding(make):
    """test_spikegenerator.py:69-104: 100 spike times spread over [0, dt) all fall into the
    first step; 10000 spikes at times k*dt fall into separate steps, so a target that counts
    its inputs (threshold always true, reset count = 0, resets before synapses) holds 1 at
    the end of every step."""
    net = make(DT)
    times = np.linspace(0, 0.1, 100, endpoint=False) * 1e-3
    SG = net.spikegen_group(100, np.arange(100), spike_steps(times, DT))
    net.spike_monitor(SG, 1000)
    net.finalize()
    net.run(1)
    idx, st = net.spikes(SG)
    np.testing.assert_array_equal(np.sort(idx), np.arange(100))
    assert np.all(st == 0)

    net = make(DT, reset_before_synapses=True)
    SG = net.spikegen_group(1, np.zeros(10000, np.int32), spike_steps(np.arange(10000) * DT, DT))
    T = net.lif_group(1, LIF(taum=math.inf, Vt=-math.inf, Vr=0.0), "float64")
    net.synapses(SG, T, "v", [0], [0], w_scalar=1.0, delay=0)
    mon = net.state_monitor(T, "v", capacity=10001)
    net.finalize()
    net.run(10000)
    steps, vals = net.state_values(mon)
    # recorded at the start of each step, i.e. the count at the end of the step before
    np.testing.assert_array_equal(steps, np.arange(10000))
    np.testing.assert_array_equal(vals[1:, 0], np.ones(9999))
    assert net.get_state(T, "v")[0] == 1.0


def state_monitor_more_threads_than_single_block(make):
    """test_monitor.py:7-20: NeuronGroup(2000, 'v:1') with v = arange(2000), StateMonitor of
    every neuron over three steps: every record equals the initial values."""
    net = make(DT)
    n = 2000
    G = net.lif_group(n, LIF(taum=math.inf, has_threshold=False, has_reset=False), "float64")
    net.set_state(G, "v", np.arange(n, dtype=np.float64))
    mon = net.state_monitor(G, "v", capacity=3)
    net.finalize()
    net.run(3)
    steps, vals = net.state_values(mon)
    np.testing.assert_array_equal(steps, [0, 1, 2])
    for t in range(3):
        np.testing.assert_array_equal(vals[t], np.arange(n))


def spike_monitor_all_attr(make):
    """test_monitor.py:23-45: threshold 'do_spike' with do_spike = [T, F, F, F, T, T]: one
    step records i = [0, 4, 5] at t = 0, counts [1, 0, 0, 0, 1, 1], N = 3; the subgroup
    monitors G[:2], G[2:4], G[4:] hold [0], nothing and [0, 1] (relative indices)."""
    net = make(DT)
    G = net.lif_group(6, LIF(taum=math.inf, Vt=0.5, has_reset=False), "float64")
    net.set_state(G, "v", np.array([1, 0, 0, 0, 1, 1], dtype=np.float64))
    net.spike_monitor(G, 100)
    net.finalize()
    net.run(1)
    idx, st = net.spikes(G)
    np.testing.assert_array_equal(idx, [0, 4, 5])
    np.testing.assert_array_equal(st, [0, 0, 0])
    np.testing.assert_array_equal(np.bincount(idx, minlength=6), [1, 0, 0, 0, 1, 1])
    for (lo, hi), want in (((0, 2), [0]), ((2, 4), []), ((4, 6), [0, 1])):
        i, t = net.spikes(G, sub=(lo, hi))
        np.testing.assert_array_equal(i, want)
        np.testing.assert_array_equal(t, np.zeros(len(want)))
        np.testing.assert_array_equal(np.bincount(i, minlength=hi - lo),
                                      np.bincount(np.array(want, dtype=np.int64),
                                                  minlength=hi - lo))


def binomial_values_seeds(make):
    """test_random_number_generation.py:367-466, for the binomial of a PoissonInput
    (Binomial(100, 0.1) per neuron and step): two draws differ, the same seed reproduces
    the values, another seed changes them."""
    def draws(seed):
        net = make(DT, seed=seed)
        G = net.lif_group(10, LIF(taum=math.inf, has_threshold=False, has_reset=False),
                          "float64")
        net.poisson_input(G, "v", 100, 0.1 / DT, 1.0)
        net.finalize()
        out = []
        for _ in range(2):
            before = net.get_state(G, "v").copy()
            net.run(1)
            out.append(net.get_state(G, "v") - before)
        return np.array(out)
    a, b, c = draws(11400), draws(11400), draws(13579)
    assert not np.array_equal(a[0], a[1])
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)


def threads_per_synapse_bundle(make):
    """test_synaptic_propagations.py:343-374: whatever the threads per synapse bundle, a
    spike at t = 0 with delays j*dt onto neurons 3 and 4 (v += 1.1, threshold v > 1) makes
    them spike at steps 4 and 5.  The launch-shape counterpart here is the delivery's lanes
    per work item (2, 4, 8, 16, 32; the oracle has one form)."""
    shapes = [2, 4, 8, 16, 32]
    for lanes in shapes:
        net = make(DT)
        inp = net.spikegen_group(1, [0], [0])
        G = net.lif_group(5, neuron_v1(), "float64")
        net.synapses(inp, G, "v", [0, 0], [3, 4], w_scalar=1.1, delay=np.array([3, 4], np.int32))
        net.spike_monitor(G, 100)
        net.finalize()
        if not hasattr(net, "tune_apply"):
            shapes = shapes[:1]
        else:
            net.tune_apply([{"site_kind": 6, "site_index": 0, "choice_a": lanes,
                             "choice_b": 148}])
        net.run(6)
        idx, st = net.spikes(G)
        np.testing.assert_array_equal(idx, [3, 4])
        np.testing.assert_array_equal(st, [4, 5])
        if len(shapes) == 1:
            break


def synaptic_effects_onto_one_target(make):
    """test_synaptic_propagations.py:316-340, its on_pre half: 15 x 1024 neurons spiking
    every step, each adding 1 to the v of one neuron with no delay; after two steps v holds
    exactly 2 x 15360 (every one of the same-address additions lands; the on_post half of
    that test needs an additive on_post pathway, which this library does not have)."""
    N = 15 * 1024
    net = make(DT)
    src = net.lif_group(N, LIF(taum=math.inf, Vt=-math.inf, has_reset=False), "float64")
    tgt = net.lif_group(1, LIF(taum=math.inf, has_threshold=False, has_reset=False), "float64")
    net.synapses(src, tgt, "v", np.arange(N, dtype=np.int32), np.zeros(N, np.int32),
                 w_scalar=1.0, delay=0)
    net.finalize()
    net.run(2)
    assert net.get_state(tgt, "v")[0] == 2.0 * N


def poisson_input_schedule(make):
    """PoissonInput acts in the synapses slot (the BinomialFunction of brian2cuda/binomial.py
    runs there): with rate 1/dt every draw is N, so v += N w each step.  A LIF with
    threshold v > 1 and reset v = 0 (N w = 1.5) spikes every second step in the default
    schedule, where the reset follows the synapses and overwrites the input, and every step
    from step 1 when resets come first and the input lands after them."""
    out = {}
    for reset_first in (False, True):
        net = make(DT, reset_before_synapses=reset_first)
        G = net.lif_group(1, LIF(taum=math.inf, Vt=1.0, Vr=0.0), "float64")
        net.poisson_input(G, "v", 3, 1.0 / DT, 0.5)
        net.spike_monitor(G, 100)
        net.finalize()
        net.run(8)
        out[reset_first] = (net.spikes(G)[1], float(net.get_state(G, "v")[0]))
    np.testing.assert_array_equal(out[False][0], [1, 3, 5, 7])
    assert out[False][1] == 0.0          # step 7 spiked: reset after the input
    np.testing.assert_array_equal(out[True][0], np.arange(1, 8))
    assert out[True][1] == 1.5           # reset, then the input


def refractory_without_spikes(make):
    """test_stateupdaters.py:169-194, for the exact integrator: dv/dt = -v/(10 ms) with
    v = (i+1)/11, with and without (unless refractory) and refractory = 1 ms; a group that
    never spikes is never refractory, so both give v = (i+1)/11 exp(-1) after 10 ms."""
    net = make(DT)
    plain = net.lif_group(10, LIF(taum=10e-3, has_threshold=False, has_reset=False), "float64")
    refr = net.lif_group(10, LIF(taum=10e-3, has_threshold=False, has_reset=False,
                                 refractory=1e-3, unless_refractory=True), "float64")
    v0 = (np.arange(10) + 1) / 11.0
    net.set_state(plain, "v", v0)
    net.set_state(refr, "v", v0)
    net.finalize()
    net.run(100)
    np.testing.assert_array_equal(net.get_state(refr, "v"), net.get_state(plain, "v"))
    np.testing.assert_allclose(net.get_state(plain, "v"), v0 * math.exp(-1.0), rtol=1e-12)


def multiple_runs_heterogeneous_delay(make):
    """test_network_multiple_runs.py:89-108: an always-spiking input, `v += 1` with delays
    0 and dt onto two neurons, two runs of two steps; v at the start of each step is
    [0, 1, 2, 3] and [0, 0, 1, 2]."""
    net = make(DT)
    inG = net.lif_group(1, LIF(taum=math.inf, Vt=-math.inf, has_reset=False), "float64")
    G = net.lif_group(2, LIF(taum=math.inf, has_threshold=False, has_reset=False), "float64")
    net.synapses(inG, G, "v", [0, 0], [0, 1], w_scalar=1.0, delay=np.array([0, 1], np.int32))
    mon = net.state_monitor(G, "v", capacity=4)
    net.finalize()
    net.run(2)
    net.run(2)
    steps, vals = net.state_values(mon)
    np.testing.assert_array_equal(steps, [0, 1, 2, 3])
    np.testing.assert_array_equal(vals[:, 0], [0, 1, 2, 3])
    np.testing.assert_array_equal(vals[:, 1], [0, 0, 1, 2])


def _delay_change(make, n_post, before, after):
    """An always-spiking input, `v += 1` onto n_post neurons with delays `before` (steps);
    one step run, delays changed to `after`, five more steps; v at the start of each step."""
    net = make(DT)
    inG = net.lif_group(1, LIF(taum=math.inf, Vt=-math.inf, has_reset=False), "float64")
    G = net.lif_group(n_post, LIF(taum=math.inf, has_threshold=False, has_reset=False),
                      "float64")
    S = net.synapses(inG, G, "v", [0] * n_post, list(range(n_post)), w_scalar=1.0,
                     delay=np.array(before, np.int32))
    mon = net.state_monitor(G, "v", capacity=6)
    net.finalize()
    net.run(1)
    net.syn_set_delays(S, np.array(after, np.int32))
    net.run(5)
    steps, vals = net.state_values(mon)
    np.testing.assert_array_equal(steps, [0, 1, 2, 3, 4, 5])
    return vals


def increasing_delay_scalar(make):
    """test_network_multiple_runs.py:36-57 (expected to fail on the reference's CUDA device,
    issue #302): delay dt, then 2 dt; the spike in flight keeps dt: [0, 0, 1, 1, 2, 3]."""
    np.testing.assert_array_equal(_delay_change(make, 1, [1], [2])[:, 0], [0, 0, 1, 1, 2, 3])


def increasing_delay_heterogeneous(make):
    """test_network_multiple_runs.py:110-131: delays j*dt, then 2*j*dt, onto two neurons:
    [0, 1, 2, 3, 4, 5] and [0, 0, 1, 1, 2, 3]."""
    vals = _delay_change(make, 2, [0, 1], [0, 2])
    np.testing.assert_array_equal(vals[:, 0], [0, 1, 2, 3, 4, 5])
    np.testing.assert_array_equal(vals[:, 1], [0, 0, 1, 1, 2, 3])


def reducing_delay_heterogeneous(make):
    """test_network_multiple_runs.py:134-156: delays 2*j*dt, then j*dt: [0, 1, 2, 3, 4, 5]
    and [0, 0, 0, 2, 3, 4] (the spike in flight and the first new one arrive together)."""
    vals = _delay_change(make, 2, [0, 2], [0, 1])
    np.testing.assert_array_equal(vals[:, 0], [0, 1, 2, 3, 4, 5])
    np.testing.assert_array_equal(vals[:, 1], [0, 0, 0, 2, 3, 4])


def time_after_run(make):
    """test_cuda_standalone.py:139-167: t is 0 before a run, 10 ms after run(10 ms) and
    20 ms after a second one (dt = 0.1 ms)."""
    net = make(DT)
    net.lif_group(10, LIF(taum=10e-3, has_threshold=False, has_reset=False), "float64")
    net.finalize()
    assert net.timestep == 0 and net.t == 0.0
    net.run(100)
    assert net.timestep == 100
    np.testing.assert_allclose(net.t, 10e-3, rtol=1e-12)
    net.run(100)
    assert net.timestep == 200
    np.testing.assert_allclose(net.t, 20e-3, rtol=1e-12)


ALL = [example_run, push_outer_loop, push_outer_loop2, circular_eventspaces,
       circular_eventspaces_spikegenerator, multiple_runs_scalar_delay,
       spikegenerator_extreme_period, spikegenerator_period_repeat, spikegenerator_rounding,
       state_monitor_more_threads_than_single_block, spike_monitor_all_attr,
       binomial_values_seeds, threads_per_synapse_bundle, synaptic_effects_onto_one_target,
       poisson_input_schedule, refractory_without_spikes, multiple_runs_heterogeneous_delay,
       increasing_delay_scalar, increasing_delay_heterogeneous,
       reducing_delay_heterogeneous, time_after_run]
