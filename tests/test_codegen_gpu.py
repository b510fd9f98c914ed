"""Generated neuron models on the GPU against the oracle's own integration of the same
equations (oracle/model_oracle.py), and the generated COBAHH model against the hand-written
COBAHH kernel.

Tolerances: spikes exact (float64); state within 1e-9 relative after a rollout of a few
hundred steps (the exact propagators come from the matrix exponential on the GPU side and
from an order-8 Runge-Kutta integration on the oracle's, which agree to ~1e-13, and the
transcendental functions of the two sides differ in the last bit)."""
import numpy as np
import pytest

from brian2cuda_b200 import examples
from brian2cuda_b200.lowering import Script
from test_codegen import ADAPT_EQS, ADAPT_NS, ALPHA_EQS, ALPHA_NS, HH52_EQS, hh52_namespace

pytestmark = pytest.mark.gpu
DT = 1e-4


def _close(a, b, rtol, atol, what=""):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    bad = np.abs(a - b) > rtol * np.abs(b) + atol
    assert not bad.any(), f"{what}: {bad.sum()} mismatches, worst {np.max(np.abs(a - b))}"


def test_alpha_synapse_network_matches_oracle(gpu_factory, oracle_factory):
    """A second-order (alpha) synapse LIF network, integrated exactly by generated code, with
    recurrent synapses onto the synaptic variable y and delays of 1-8 steps (resting
    potential 1 mV above threshold: every neuron fires repeatedly)."""
    s = Script(dt=DT, seed=11, namespace=dict(ALPHA_NS, El=-49e-3))
    G = s.NeuronGroup(2000, ALPHA_EQS, threshold="v > Vt", reset="v = Vr", refractory=2e-3)
    G.v = "Vr + rand() * 22*mV"
    S = s.Synapses(G, G, on_pre="y += 0.9*mV")
    S.connect(p=0.02)
    from brian2cuda_b200.lowering import UniformDelaySteps
    S.delay = UniformDelaySteps(1, 8)
    s.SpikeMonitor(G, name="spk")
    s.StateMonitor(G, ["v", "x"], record=[0, 17, 1999], name="st")
    s.run(0.04)
    prog = s.lower()
    g = prog.execute(gpu_factory(DT, seed=s.seed))
    o = prog.execute(oracle_factory(DT))
    assert len(g["spk"][0]) > 500
    np.testing.assert_array_equal(g["spk"][1], o["spk"][1])
    np.testing.assert_array_equal(g["spk"][0], o["spk"][0])
    for v in ("v", "x"):
        np.testing.assert_array_equal(g["st"][v][0], o["st"][v][0])
        _close(g["st"][v][1], o["st"][v][1], 1e-9, 1e-15, v)


@pytest.mark.parametrize("n,synapses,chunks", [(1500, True, 6), (700_000, False, 2)])
def test_noisy_adaptive_network_matches_oracle(gpu_factory, oracle_factory, n, synapses,
                                               chunks):
    """Euler-Maruyama with the GPU's cuRAND normal numbers fed to the oracle, a two-statement
    reset, refractoriness, and synapses onto v (a variable the reset writes: the reset is
    deferred until after the delivery, as in Brian2's schedule).  7e5 neurons without
    synapses (the oracle's connect visits every pair): the generated kernel's
    four-neurons-per-thread form."""
    K = 50
    s = Script(dt=DT, seed=5, namespace=ADAPT_NS)
    G = s.NeuronGroup(n, ADAPT_EQS, threshold="v > Vt", reset="v = Vr; w += b",
                      refractory=2e-3)
    G.v = "El + rand()*20*mV"
    if synapses:
        S = s.Synapses(G, G, on_pre="v += 0.3*mV", delay=2e-4)
        S.connect(p=0.02)
    s.SpikeMonitor(G, capacity=max(10**6, n), name="spk")   # the runs are made by hand
    prog = s.lower()
    gnet = gpu_factory(DT, seed=s.seed, steps_per_graph=K)
    onet = oracle_factory(DT)
    gids, oids = prog.build(gnet), prog.build(onet)
    for _ in range(chunks):
        gnet.run(K)
        onet.set_normals(oids[G.name], gnet.rng_normals(gids[G.name], K, 1))
        onet.run(K)
    g, o = prog.collect(gnet, gids), prog.collect(onet, oids)
    assert len(g["spk"][0]) > 300
    np.testing.assert_array_equal(g["spk"][1], o["spk"][1])
    np.testing.assert_array_equal(g["spk"][0], o["spk"][0])
    for v in ("v", "ge"):            # slots of the model's variables v and w
        _close(gnet.get_state(gids[G.name], v), onet.get_state(oids[G.name], v), 1e-9,
               1e-15, v)


def test_hh52_generated_exponential_euler_matches_oracle(gpu_factory, oracle_factory):
    """The Hodgkin-Huxley 1952 model (not the COBAHH kernel's system) integrated by generated
    exponential-Euler code, float64, 400 steps of a constant drive."""
    s = Script(dt=DT, seed=2, namespace=hh52_namespace())
    G = s.NeuronGroup(3000, HH52_EQS.replace("I : amp (constant)\n", ""),
                      threshold="v > -20*mV", refractory=3e-3, method="exponential_euler")
    G.v = "-70*mV + rand()*15*mV"
    G.m = 0.05
    G.h = 0.6
    G.n = 0.32
    s.SpikeMonitor(G, name="spk")
    s.run(0.04)
    prog = s.lower()
    gnet, onet = gpu_factory(DT, seed=2), oracle_factory(DT)
    gids, oids = prog.build(gnet), prog.build(onet)
    gnet.run(400)
    onet.run(400)
    g, o = prog.collect(gnet, gids), prog.collect(onet, oids)
    assert len(g["spk"][0]) > 1000
    np.testing.assert_array_equal(g["spk"][1], o["spk"][1])
    np.testing.assert_array_equal(g["spk"][0], o["spk"][0])
    for slot in ("v", "ge", "gi", "m"):          # v, m, h, n in slot order
        _close(gnet.get_state(gids[G.name], slot), onet.get_state(oids[G.name], slot), 1e-9,
               1e-15, slot)


def test_generated_cobahh_matches_the_handwritten_kernel(gpu_factory):
    """The COBAHH script integrated by generated code and by the hand-written kernel,
    float64, 1e4 neurons with delayed synapses, 200 steps through the initial burst: spikes
    exact, state within 1e-9."""
    out = {}
    for gen in (False, True):
        s, h = examples.cobahh(N=10_000, duration=0.02, dtype="float64")
        s.generated_only = gen
        prog = s.lower()
        kinds = {op.method for op in prog.ops}
        assert ("model_group" in kinds) == gen and ("hh_group" in kinds) != gen
        net = gpu_factory(DT, seed=s.seed)
        res = prog.execute(net)
        # the generated model's state slots follow its own order (synaptic targets first)
        v_slot = prog.groups[h["P"].name]["slots"]["v"]
        out[gen] = (res["spikes"], net.get_state(0, v_slot))
    (gi, gs), gv = out[True]
    (hi, hs), hv = out[False]
    assert len(hi) > 1000
    np.testing.assert_array_equal(gs, hs)
    np.testing.assert_array_equal(gi, hi)
    _close(gv, hv, 1e-9, 1e-15, "v")
