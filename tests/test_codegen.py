"""Generated neuron models (CPU only): models outside the hand-written kernels' systems are
generated with the expected integrator, their CUDA source compiles for sm_100a, and the
oracle's independent derivation of the exact propagator agrees with the generator's."""
import os
import numpy as np
import pytest

from brian2cuda_b200 import codegen
from brian2cuda_b200 import equations as E
from brian2cuda_b200 import examples
from brian2cuda_b200.lowering import ModelUnsupported, Script

DT = 1e-4

ALPHA_EQS = """
dv/dt = (El - v + x) / taum : volt (unless refractory)
dx/dt = (y - x) / taus : volt
dy/dt = -y / taus : volt
"""
ALPHA_NS = dict(El=-65e-3, taum=10e-3, taus=2e-3, Vt=-50e-3, Vr=-70e-3)

ADAPT_EQS = """
dv/dt = (El - v - w + I0) / tau + sigma * xi * tau**-0.5 : volt
dw/dt = (a * (v - El) - w) / tauw : volt
"""
ADAPT_NS = dict(tau=10e-3, tauw=100e-3, a=0.5, sigma=2e-3, El=-70e-3, Vt=-50e-3, Vr=-65e-3,
                b=1e-3, I0=22e-3)

HH52_EQS = """
dv/dt = (gl*(El - v) - gna*m**3*h*(v - ENa) - gk*n**4*(v - EK) + I) / C : volt
dm/dt = alpham*(1 - m) - betam*m : 1
dh/dt = alphah*(1 - h) - betah*h : 1
dn/dt = alphan*(1 - n) - betan*n : 1
alpham = 0.1/mV * 10*mV / exprel((-v + 25*mV - 65*mV) / (10*mV)) / ms : Hz
betam = 4 * exp((-v - 65*mV) / (18*mV)) / ms : Hz
alphah = 0.07 * exp((-v - 65*mV) / (20*mV)) / ms : Hz
betah = 1. / (exp((-v + 30*mV - 65*mV) / (10*mV)) + 1) / ms : Hz
alphan = 0.01/mV * 10*mV / exprel((-v + 10*mV - 65*mV) / (10*mV)) / ms : Hz
betan = 0.125 * exp((-v - 65*mV) / (80*mV)) / ms : Hz
I : amp (constant)
"""


def hh52_namespace():
    area = 20000e-12
    return dict(C=1e-2 * area, gl=3e-4 * 1e4 * area, El=-54.4e-3, EK=-77e-3, ENa=50e-3,
                gna=120e-3 * 1e4 * area, gk=36e-3 * 1e4 * area, I=0.7e-9)


def _model(script):
    ops = [op for op in script.lower().ops if op.method == "model_group"]
    assert len(ops) == 1
    return ops[0].args[1]


def test_alpha_synapse_lif_is_generated_exact():
    s = Script(dt=DT, namespace=ALPHA_NS)
    G = s.NeuronGroup(10, ALPHA_EQS, threshold="v > Vt", reset="v = Vr", refractory=2e-3)
    S = s.Synapses(G, G, on_pre="y += 1*mV")
    S.connect(p=0.5)
    gm = _model(s)
    assert gm.method == "exact" and gm.state[0] == "y"        # the synaptic target first
    assert "refractory" in gm.propagators and gm.reset_mask == 1 << gm.state.index("v")
    assert "if (!not_refractory)" in gm.source


def test_noisy_adaptive_model_is_generated_euler_with_one_normal_draw():
    s = Script(dt=DT, namespace=ADAPT_NS)
    s.NeuronGroup(10, ADAPT_EQS, threshold="v > Vt", reset="v = Vr; w += b", refractory=2e-3)
    gm = _model(s)
    assert gm.method == "euler" and gm.noise == ["xi"] and gm.n_normal == 1
    assert "nrm[0 * stride]" in gm.source
    assert gm.reset_mask == 0b11


def test_hh52_is_generated_exponential_euler():
    s = Script(dt=DT, namespace=hh52_namespace())
    s.NeuronGroup(10, HH52_EQS.replace("I : amp (constant)\n", ""), threshold="v > -20*mV",
                  refractory=3e-3, method="exponential_euler")
    gm = _model(s)
    assert gm.method == "exponential_euler" and gm.state == ["v", "m", "h", "n"]
    assert "b2b::model::exprel<R>" in gm.source


def test_cobahh_with_other_kinetics_is_not_taken_for_the_cobahh_kernel():
    s = Script(dt=DT, namespace=examples.cobahh_namespace())
    s.NeuronGroup(10, examples.COBAHH_EQS.replace("0.128*exp", "0.129*exp"),
                  threshold="v > -20*mV", refractory=3e-3, method="exponential_euler")
    gm = _model(s)
    assert gm.method == "exponential_euler" and len(gm.state) == 6


def test_generated_sources_compile_for_sm100a():
    for eqs, ns, kw in ((ALPHA_EQS, ALPHA_NS, dict(threshold="v > Vt", reset="v = Vr")),
                        (ADAPT_EQS, ADAPT_NS,
                         dict(threshold="v > Vt and w < 5*mV", reset="v = Vr; w += b"))):
        s = Script(dt=DT, namespace=ns)
        s.NeuronGroup(10, eqs, refractory=2e-3, **kw)
        gm = _model(s)
        path = codegen.compile_model(gm.source)
        assert path.endswith(".so")
        # cached by content: the second request compiles nothing
        assert codegen.compile_model(gm.source) == path


def test_oracles_propagator_agrees_with_the_generators():
    """The oracle integrates the linear system with an order-8 Runge-Kutta method; the
    generator takes the matrix exponential: the two propagators agree to 1e-12."""
    from oracle.model_oracle import ModelCallback
    s = Script(dt=DT, namespace=ALPHA_NS)
    s.NeuronGroup(10, ALPHA_EQS, threshold="v > Vt", reset="v = Vr", refractory=2e-3)
    gm = _model(s)
    cb = ModelCallback(gm, DT)
    M, c = gm.propagators["active"]
    np.testing.assert_allclose(cb.M, M, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(cb.c, c, rtol=1e-12, atol=1e-18)
    Mr, cr = gm.propagators["refractory"]
    np.testing.assert_allclose(cb.Mr, Mr, rtol=1e-12, atol=1e-15)


def test_generated_model_runs_on_the_oracle(oracle_factory):
    s = Script(dt=DT, seed=3, namespace=ADAPT_NS)
    G = s.NeuronGroup(200, ADAPT_EQS, threshold="v > Vt", reset="v = Vr; w += b",
                      refractory=2e-3)
    G.v = "El + rand()*20*mV"
    s.SpikeMonitor(G, name="spk")
    prog = s.lower()
    net = oracle_factory(DT)
    ids = prog.build(net)
    net.set_normals(ids[G.name], np.random.default_rng(0).standard_normal((300, 200)))
    net.run(300)
    idx, st = net.spikes(ids[G.name])
    assert len(idx) > 50
    # refractoriness holds: no neuron spikes twice within 2 ms
    for i in np.unique(idx):
        assert np.all(np.diff(st[idx == i]) >= 20)


def test_unsupported_model_forms_fail_clearly():
    s = Script(dt=DT)
    s.NeuronGroup(5, "dv/dt = (rand() - v) / (10*ms) : 1", threshold="v > 1", reset="v = 0")
    with pytest.raises(ModelUnsupported, match="rand"):
        s.lower()
    s = Script(dt=DT)
    s.NeuronGroup(5, "dv/dt = -v/(10*ms) + xi/sqrt(ms) : 1", method="exact")
    with pytest.raises(ModelUnsupported, match="noise"):
        s.lower()
    with pytest.raises(E.EquationError):
        E.parse_equations("dv/dt = -v")


def test_generated_model_reaches_the_c_program(tmp_path):
    """A script with a generated model emits a C program that loads the compiled model
    object through b2b_group_model and compiles against the header."""
    from brian2cuda_b200 import cemit
    s = Script(dt=DT, seed=3, namespace=ALPHA_NS)
    G = s.NeuronGroup(100, ALPHA_EQS, threshold="v > Vt", reset="v = Vr", refractory=2e-3)
    S = s.Synapses(G, G, on_pre="y += 0.9*mV")
    S.connect(p=0.05)
    s.SpikeMonitor(G, name="spk")
    s.run(0.002)
    prog = s.lower()
    text = open(cemit.emit_c(prog, str(tmp_path))).read()
    assert "b2b_group_model(" in text and ".so\"" in text
    exe = cemit.compile_c(str(tmp_path))
    assert os.access(exe, os.X_OK)
