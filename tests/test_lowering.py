"""The Brian2-shaped front end and its lowering (CPU only): model strings parse, the
benchmark models are recognised as the hand-written kernels' systems with the scripts' own
constants, the exact integrator reproduces the reference's analytic example, unsupported
constructs fail with a clear error, and a lowered script runs on the oracle and as a
generated C program that compiles against include/b2b.h."""
import math
import os

import numpy as np
import pytest

from brian2cuda_b200 import equations as E
from brian2cuda_b200 import examples, models
from brian2cuda_b200.lowering import ModelUnsupported, Script, statements

DT = 1e-4


def _ops(script, method):
    return [op for op in script.lower().ops if op.method == method]


def test_parser_reads_multiline_equations_with_units_and_flags():
    m = E.parse_equations(examples.COBAHH_EQS)
    assert m.state == ["v", "m", "n", "h", "ge", "gi"]
    assert [e.name for e in m.eqs if e.kind == "sub"] == ["alpha_m", "beta_m", "alpha_h",
                                                          "beta_h", "alpha_n", "beta_n"]
    m2 = E.parse_equations(examples.CUBA_EQS)
    assert m2.flags("v") == ("unless refractory",)
    assert E.value_of("13.*mV - 4*mV", {}) == pytest.approx(9e-3, rel=1e-15)
    assert E.value_of("Vt + 2*mV", {"Vt": -50e-3}) == pytest.approx(-48e-3, rel=1e-15)


def test_cuba_script_lowers_to_the_lif_kernel_with_the_scripts_constants():
    s, _ = examples.cuba(N=4000)
    (op,) = _ops(s, "lif_group")
    prm = op.args[1]
    ref = models.cuba_lif()
    for f in ("El", "taum", "taue", "taui", "ke", "ki", "Vt", "Vr", "refractory"):
        assert getattr(prm, f) == getattr(ref, f), f
    assert prm.unless_refractory and prm.has_threshold and prm.has_reset
    syn = _ops(s, "synapses_random")
    assert [o.kwargs["pre_range"] for o in syn] == [(0, 3200), (3200, 4000)]
    assert [o.args[2] for o in syn] == ["ge", "gi"]


def test_cobahh_script_lowers_to_the_hh_kernel_with_the_scripts_constants():
    s, _ = examples.cobahh(N=1000)
    (op,) = _ops(s, "hh_group")
    prm, ref = op.args[1], models.cobahh_hh()
    for f in ("Cm", "gl", "El", "EK", "ENa", "gNa", "gK", "VT", "Ee", "Ei", "taue", "taui",
              "Vthr", "refractory"):
        assert getattr(prm, f) == getattr(ref, f), f
    syn = _ops(s, "synapses_random")
    assert [(o.args[4], o.args[5]) for o in syn] == [(1, 50), (1, 50)]
    assert [o.kwargs["pre_range"] for o in syn] == [(0, 800), (800, 1000)]


def test_stdp_script_lowers_to_the_stdp_rule():
    s, _ = examples.stdp(n_in=50, n_out=7)
    (op,) = _ops(s, "synapses")
    rule, ref = op.kwargs["stdp"], models.stdp_rule()
    for f in ("taupre", "taupost", "dApre", "dApost", "wmin", "wmax"):
        assert getattr(rule, f) == pytest.approx(getattr(ref, f), rel=1e-15), f
    assert rule.pre_adds_weight
    assert len(op.args[3]) == 350 and op.kwargs["w"].max() < 0.01
    (lif,) = _ops(s, "lif_group")
    for f in ("El", "taum", "taue", "ke", "Vt", "Vr"):
        assert getattr(lif.args[1], f) == pytest.approx(getattr(models.stdp_lif(), f),
                                                        rel=1e-14), f


def test_exact_integrator_matches_the_references_analytic_example(oracle_factory):
    """brian2cuda/__init__.py:50-72 (example_run): dv/dt = -v/tau, v = i/100 initially;
    after 1 ms, v = i/100 exp(-1 ms / 10 ms)."""
    s = Script(dt=DT, namespace={"tau": 10e-3})
    G = s.NeuronGroup(100, "dv/dt = -v / tau : 1", method="exact")
    G.v = "i / 100."
    mon = s.StateMonitor(G, "v", record=True, name="v")
    s.run(1e-3)
    net = oracle_factory(DT)
    prog = s.lower()
    ids = prog.build(net)
    net.run(10)
    v = net.get_state(ids[G.name], "v")
    np.testing.assert_allclose(v, np.arange(100) / 100 * math.exp(-0.1), rtol=1e-12)
    assert "v" in prog.monitors[mon.name]["vars"]


def test_propagator_of_a_linear_system_is_the_matrix_exponential():
    A = np.array([[-50.0, 50.0], [0.0, -200.0]])
    b = np.array([-2.45, 0.0])
    M, c = E.exact_propagator(A, b, DT)
    # closed form of dv/dt = (El - v + ge)/taum, dge/dt = -ge/taue
    taum, taue, El = 0.02, 0.005, -0.049
    a = math.exp(-DT / taum)
    assert M[0, 0] == pytest.approx(a, rel=1e-14)
    assert c[0] == pytest.approx(El * (1 - a), rel=1e-13)
    # v driven by ge(t) = ge0 exp(-t/taue): v = ge0 taue/(taue - taum) (e^-t/taue - e^-t/taum)
    k = taue / (taue - taum) * (math.exp(-DT / taue) - a)
    assert M[0, 1] == pytest.approx(k, rel=1e-12)
    assert M[1, 1] == pytest.approx(math.exp(-DT / taue), rel=1e-14)


def test_unsupported_constructs_fail_clearly():
    s = Script(dt=DT)
    G = s.NeuronGroup(10, "dv/dt = -v/(10*ms) : 1", threshold="v > 1", reset="v = 0; w = 1")
    with pytest.raises(ModelUnsupported, match="reset"):
        s.lower()
    s = Script(dt=DT)
    G = s.NeuronGroup(10, "dv/dt = -v/(10*ms) : 1", threshold="v > 1", reset="v = 0")
    S = s.Synapses(G, G, on_pre="v_post *= 2")
    S.connect(p=0.5)
    with pytest.raises(ModelUnsupported, match="cannot lower the statement 'v_post \\*= 2'"):
        s.lower()
    with pytest.raises(ModelUnsupported):
        statements("v += ")
    with pytest.raises(E.EquationError, match="undefined"):
        E.resolve(E.parse_equations("dv/dt = -v/tau_undefined : 1"), {})


def test_lowered_cuba_runs_on_the_oracle_like_the_hand_built_network(oracle_factory):
    """The lowered CUBA script and the same network built by hand through the Network
    methods (same Philox connectivity, same initial state) give identical spikes."""
    s, h = examples.cuba(N=600, duration=0.03, p=0.05)
    prog = s.lower()
    out = prog.execute(oracle_factory(DT))
    net = oracle_factory(DT)
    ids = prog.build(net)          # the same calls, made one by one
    net.run(300)
    idx, st = net.spikes(ids[h["P"].name])
    np.testing.assert_array_equal(out["spikes"][0], idx)
    np.testing.assert_array_equal(out["spikes"][1], st)
    assert len(idx) > 50


def test_generated_c_program_compiles_against_the_header(tmp_path):
    from brian2cuda_b200 import cemit
    s, h = examples.stdp(n_in=30, n_out=5, duration=0.002, dtype="float64")
    s.StateMonitor(h["neurons"], ["v", "ge"], record=[0, 3], name="vmon")
    s.PopulationRateMonitor(h["neurons"], name="rate")
    prog = s.lower()
    src = cemit.emit_c(prog, str(tmp_path))
    text = open(src).read()
    for call in ("b2b_create", "b2b_group_poisson", "b2b_group_lif", "b2b_synapses",
                 "b2b_statemon", "b2b_ratemon", "b2b_finalize", "b2b_run", "b2b_destroy"):
        assert call + "(" in text, call
    exe = cemit.compile_c(str(tmp_path))
    assert os.access(exe, os.X_OK)
    assert len(os.listdir(tmp_path / "static_arrays")) >= 4
