"""Brian2-shaped scripts lowered onto the CUDA library, against the same scripts lowered
onto the oracle, and the generated C program (include/b2b.h, linked with -lb2b) against the
Python binding running the same program."""
import os
import subprocess

import numpy as np
import pytest

from brian2cuda_b200 import examples
from brian2cuda_b200.lowering import Script

pytestmark = pytest.mark.gpu
DT = 1e-4


def test_cuba_script_full_second_matches_oracle(gpu_factory, oracle_factory):
    """The CUBA script as configured (4000 neurons, float64, 1 s): spikes exact."""
    s, h = examples.cuba(N=4000, duration=1.0)
    prog = s.lower()
    g = prog.execute(gpu_factory(DT, seed=s.seed))
    o = prog.execute(oracle_factory(DT))
    assert len(g["spikes"][0]) > 10_000
    np.testing.assert_array_equal(g["spikes"][1], o["spikes"][1])
    np.testing.assert_array_equal(g["spikes"][0], o["spikes"][0])


def test_cobahh_script_float64_matches_oracle(gpu_factory, oracle_factory):
    """The COBAHH script (20,000 neurons, delays 1..50 steps, float64) for 200 steps:
    spikes exact."""
    s, h = examples.cobahh(N=20_000, duration=0.02, dtype="float64")
    prog = s.lower()
    g = prog.execute(gpu_factory(DT, seed=s.seed))
    o = prog.execute(oracle_factory(DT))
    assert len(g["spikes"][0]) > 1000
    np.testing.assert_array_equal(g["spikes"][1], o["spikes"][1])
    np.testing.assert_array_equal(g["spikes"][0], o["spikes"][0])


def test_stdp_script_matches_oracle(gpu_factory, oracle_factory):
    """The STDP script (float64, 2000 -> 100) with the GPU's Poisson uniforms fed to the
    oracle: both spike trains exact, weights within 1e-10."""
    K = 50
    s, h = examples.stdp(n_in=2000, n_out=100, rate=40.0, duration=0.02, dtype="float64")
    prog = s.lower()
    gnet = gpu_factory(DT, seed=s.seed, steps_per_graph=K)
    onet = oracle_factory(DT)
    gids, oids = prog.build(gnet), prog.build(onet)
    inp = h["input"].name
    for _ in range(4):
        gnet.run(K)
        onet.set_uniforms(oids[inp], gnet.rng_uniforms(gids[inp], K))
        onet.run(K)
    g, o = prog.collect(gnet, gids), prog.collect(onet, oids)
    for m in ("input_spikes", "output_spikes"):
        np.testing.assert_array_equal(g[m][1], o[m][1])
        np.testing.assert_array_equal(g[m][0], o[m][0])
    assert len(g["output_spikes"][0]) > 20
    S = h["S"].name
    np.testing.assert_allclose(gnet.syn_get(gids[S], "w"), onet.syn_get(oids[S], "w"),
                               rtol=1e-10, atol=1e-18)


def test_generated_c_program_matches_python_binding(gpu_factory, tmp_path):
    """The generated C program, compiled with the host compiler against include/b2b.h and
    linked with libb2b.so, gives the spikes, state-monitor records and rate counts the
    Python binding gives for the same lowered program."""
    from brian2cuda_b200 import cemit
    s, h = examples.cobahh(N=3000, duration=0.03, dtype="float64")
    s.StateMonitor(h["P"], ["v", "ge"], record=[0, 7, 2999], name="vmon")
    s.PopulationRateMonitor(h["P"], name="rate")
    prog = s.lower()
    ref = prog.execute(gpu_factory(DT, seed=s.seed))
    cemit.emit_c(prog, str(tmp_path))
    exe = cemit.compile_c(str(tmp_path))
    os.makedirs(tmp_path / "results", exist_ok=True)
    r = subprocess.run([exe, "results"], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    got = cemit.read_results(prog, str(tmp_path / "results"))
    np.testing.assert_array_equal(got["spikes"][0], ref["spikes"][0])
    np.testing.assert_array_equal(got["spikes"][1], ref["spikes"][1])
    assert len(ref["spikes"][0]) > 100
    for v in ("v", "ge"):
        np.testing.assert_array_equal(got["vmon"][v][0], ref["vmon"][v][0])
        np.testing.assert_array_equal(got["vmon"][v][1], ref["vmon"][v][1])
    np.testing.assert_array_equal(got["rate"][0], ref["rate"][0])
    np.testing.assert_array_equal(got["rate"][1], ref["rate"][1])


def test_generated_c_program_with_a_generated_model(gpu_factory, tmp_path):
    """A C program whose group uses a generated model object (b2b_group_model) gives the
    spikes the Python binding gives."""
    from brian2cuda_b200 import cemit
    from test_codegen import ALPHA_EQS, ALPHA_NS
    s = Script(dt=DT, seed=21, namespace=ALPHA_NS)
    G = s.NeuronGroup(1500, ALPHA_EQS, threshold="v > Vt", reset="v = Vr", refractory=2e-3)
    G.v = "Vr + rand() * 22*mV"
    S = s.Synapses(G, G, on_pre="y += 0.9*mV", delay=3e-4)
    S.connect(p=0.02)
    s.SpikeMonitor(G, name="spk")
    s.run(0.03)
    prog = s.lower()
    ref = prog.execute(gpu_factory(DT, seed=s.seed))
    cemit.emit_c(prog, str(tmp_path))
    exe = cemit.compile_c(str(tmp_path))
    os.makedirs(tmp_path / "results", exist_ok=True)
    r = subprocess.run([exe, "results"], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    got = cemit.read_results(prog, str(tmp_path / "results"))
    assert len(ref["spk"][0]) > 100
    np.testing.assert_array_equal(got["spk"][0], ref["spk"][0])
    np.testing.assert_array_equal(got["spk"][1], ref["spk"][1])
