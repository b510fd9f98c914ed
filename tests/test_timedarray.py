"""TimedArray input (the role of brian2cuda/timedarray.py:10-58): a table of values held
over each interval of the array's dt, the last row after its end, one column for a whole
group or one per neuron.

The reference has no test of its own for it, so the oracle is pinned by closed forms: a
leaky LIF under a drive that is constant over each step is integrated exactly by the
propagator with El + I, and a passive HH (no sodium or potassium conductance) is linear, so
its exponential-Euler step is exact too.  The CUDA library is then compared with the pinned
oracle in every form of the step.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from brian2cuda_b200 import models
from brian2cuda_b200.network import HH, LIF

DT = 1e-4
mV = 1e-3


def _drive_rows(steps, rows, mul, div):
    """Row of the array step ts reads: the interval holding t = ts dt, clamped."""
    return np.minimum(np.arange(steps) * mul // div, rows - 1)


def _lif_closed_form(v0, El, taum, u_of_step):
    A = math.exp(-DT / taum)
    v = np.array(v0, dtype=np.float64)
    out = []
    for u in u_of_step:
        v = (El + u) + (v - El - u) * A
        out.append(v.copy())
    return np.array(out)


def _run_record(net, G, steps, var="v"):
    rec = []
    for _ in range(steps):
        net.run(1)
        rec.append(net.get_state(G, var).copy())
    return np.array(rec)


@pytest.mark.parametrize("coarse", [True, False])
def test_oracle_lif_timedarray_closed_form(oracle_factory, coarse):
    """Per-neuron array sampled every 3 dt (row = ts // 3), or every dt / 2 (row = 2 ts);
    the run passes the array's end, where the last row holds."""
    n, steps = 3, 20
    rng = np.random.default_rng(7)
    vals = rng.uniform(-5 * mV, 15 * mV, size=(4, n))
    mul, div = (1, 3) if coarse else (2, 1)
    dt_array = DT * div / mul
    net = oracle_factory(DT)
    G = net.lif_group(n, LIF(El=-60 * mV, taum=10e-3, has_threshold=False, has_reset=False))
    v0 = np.array([-60 * mV, -55 * mV, -70 * mV])
    net.set_state(G, "v", v0)
    net.timed_array(G, vals, dt_array)
    net.finalize()
    got = _run_record(net, G, steps)
    u = vals[_drive_rows(steps, len(vals), mul, div)]
    want = _lif_closed_form(v0, -60 * mV, 10e-3, u)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-15)


def test_oracle_hh_timedarray_passive_closed_form(oracle_factory):
    """Cm dv/dt = gl (El - v) + I(t) with I from a one-column array: each step relaxes v
    towards El + I/gl with rate gl/Cm."""
    p = models.cobahh_hh()
    p = HH(**{**p.__dict__, "gNa": 0.0, "gK": 0.0, "Vthr": 1.0})
    n, steps = 4, 25
    cur = np.array([0.0, 0.2e-9, 0.5e-9, -0.1e-9, 0.3e-9])   # amperes
    net = oracle_factory(DT)
    G = net.hh_group(n, p)
    v0 = np.array([-60, -65, -58, -62]) * mV
    net.set_state(G, "v", v0)
    net.timed_array(G, cur, 5 * DT)
    net.finalize()
    got = _run_record(net, G, steps)
    I = cur[_drive_rows(steps, len(cur), 1, 5)]
    A = math.exp(-p.gl * DT / p.Cm)
    v = v0.copy()
    want = []
    for i_k in I:
        vinf = p.El + i_k / p.gl
        v = vinf + (v - vinf) * A
        want.append(v.copy())
    np.testing.assert_allclose(got, np.array(want), rtol=1e-12, atol=1e-15)


def _lif_net_with_drive(net, n=600, seed=11):
    """CUBA-like LIF with recurrent delayed synapses and a per-neuron drive that switches
    every 2 ms; 200 steps cover the array's 8 rows and run past its end."""
    rng = np.random.default_rng(seed)
    G = net.lif_group(n, models.cuba_lif(), "float64")
    net.set_state(G, "v", rng.uniform(-60 * mV, -50 * mV, n))
    i, j = models.bernoulli_pairs(rng, n, n, 0.05)
    d = rng.integers(1, 9, size=len(i)).astype(np.int32)
    ne = int(0.8 * n)
    exc = i < ne
    net.synapses(G, G, "ge", i[exc], j[exc], w_scalar=1.62 * mV, delay=d[exc])
    net.synapses(G, G, "gi", i[~exc], j[~exc], w_scalar=-9 * mV, delay=d[~exc])
    net.timed_array(G, rng.uniform(-4 * mV, 6 * mV, size=(8, n)), 20 * DT)
    net.spike_monitor(G, 10**6)
    return G


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["per-step", "two launches", "small"])
def test_lif_timedarray_matches_oracle(gpu_factory, oracle_factory, form):
    out = {}
    for name in ("gpu", "orc"):
        if name == "orc":
            net = oracle_factory(DT)
        else:
            net = gpu_factory(DT, two_launch={"per-step": False, "two launches": True}.get(form),
                              small=form == "small")
        G = _lif_net_with_drive(net)
        net.finalize()
        if name == "gpu":
            assert net.run_mode == {"per-step": "per-step", "two launches": "two-launch",
                                    "small": "small"}[form]
        net.run(120)
        net.run(80)
        idx, st = net.spikes(G)
        out[name] = (idx, st, net.get_state(G, "v"), net.get_state(G, "ge"))
    assert len(out["orc"][0]) > 100
    np.testing.assert_array_equal(out["gpu"][1], out["orc"][1])
    np.testing.assert_array_equal(out["gpu"][0], out["orc"][0])
    np.testing.assert_allclose(out["gpu"][2], out["orc"][2], rtol=1e-10, atol=1e-15)
    np.testing.assert_allclose(out["gpu"][3], out["orc"][3], rtol=1e-10, atol=1e-15)


def _all_within_one_step(a_idx, a_st, b_idx, b_st):
    """Every spike of a has a spike of b at the same neuron within one step."""
    keys = set(zip(b_idx.tolist(), b_st.tolist()))
    return all(any((i, s + o) in keys for o in (-1, 0, 1))
               for i, s in zip(a_idx.tolist(), a_st.tolist()))


@pytest.mark.gpu
def test_hh_timedarray_float32_matches_oracle(gpu_factory, oracle_factory):
    """COBAHH float32 with a one-column current ramp (0 to 0.4 nA over 10 ms): spikes within
    one step of the float32 oracle's, both ways."""
    out = {}
    ramp = np.linspace(0.0, 0.4e-9, 11)
    for name in ("gpu", "orc"):
        net = oracle_factory(DT, f32=True) if name == "orc" else gpu_factory(DT)
        ids = models.build_cobahh(net, n=2000, p=0.02, generated=False, monitor_capacity=10**6)
        net.timed_array(ids["P"], ramp, 10 * DT)
        net.finalize()
        net.run(150)
        out[name] = net.spikes(ids["P"])
    (gi, gs), (oi, os_) = out["gpu"], out["orc"]
    assert len(oi) > 20
    assert _all_within_one_step(gi, gs, oi, os_)
    assert _all_within_one_step(oi, os_, gi, gs)


@pytest.mark.gpu
def test_timedarray_rejects_bad_arguments(gpu_factory):
    net = gpu_factory(DT)
    G = net.lif_group(10, models.cuba_lif(), "float64")
    S = net.spikegen_group(10, [1], [3])
    with pytest.raises(Exception):
        net.timed_array(G, np.zeros((4, 3)), DT)         # neither 1 nor 10 columns
    with pytest.raises(Exception):
        net.timed_array(G, np.zeros(4), 2.5 * DT)         # time grids not aligned
    with pytest.raises(Exception):
        net.timed_array(S, np.zeros(4), DT)               # not a LIF, HH or Poisson group
    net.timed_array(G, np.zeros(4), DT)
    net.finalize()
    with pytest.raises(Exception):
        net.timed_array(G, np.zeros(4), DT)               # after finalize


def test_oracle_poisson_rate_timedarray_known_answer(oracle_factory):
    """PoissonGroup(N, rates='ta(t)'): neuron i spikes at step t when u < rate(t, i) dt; rate
    0 never spikes, rate 1/dt always does."""
    n, steps = 300, 16
    rng = np.random.default_rng(3)
    rates = np.stack([np.zeros(n), rng.uniform(0, 8000, n), np.full(n, 1 / DT),
                      rng.uniform(0, 3000, n)])
    u = rng.uniform(0, 1, size=(steps, n))
    net = oracle_factory(DT)
    P = net.poisson_group(n, 123.0)
    net.timed_array(P, rates, 4 * DT)
    net.spike_monitor(P, 10**6)
    net.finalize()
    net.set_uniforms(P, u)
    net.run(steps)
    idx, st = net.spikes(P)
    want = u < rates[_drive_rows(steps, len(rates), 1, 4)] * DT
    wst, widx = np.nonzero(want)
    np.testing.assert_array_equal(st, wst)
    np.testing.assert_array_equal(idx, widx)
    assert not np.any((st >= 0) & (st < 4))          # rate 0
    assert np.sum((st >= 8) & (st < 12)) == 4 * n     # rate 1/dt


@pytest.mark.gpu
def test_poisson_rate_timedarray_matches_oracle(gpu_factory, oracle_factory):
    """A PoissonGroup whose per-neuron rates follow a TimedArray drives a LIF group; the
    oracle consumes the GPU's uniforms: both spike trains equal, state within 1e-10."""
    K = 50
    rng = np.random.default_rng(8)
    rates = rng.uniform(0, 400, size=(6, 400))
    rates[2] = 0.0
    gpu = gpu_factory(DT, steps_per_graph=K, seed=3)
    orc = oracle_factory(DT)
    ids = {}
    for name, net in (("gpu", gpu), ("orc", orc)):
        P = net.poisson_group(400, 50.0, "float64")
        net.timed_array(P, rates, 30 * DT)
        G = net.lif_group(100, models.cuba_lif(), "float64")
        i, j = models.bernoulli_pairs(np.random.default_rng(1), 400, 100, 0.1)
        net.synapses(P, G, "ge", i, j, w_scalar=0.6 * mV,
                     delay=np.random.default_rng(2).integers(0, 5, len(i)).astype(np.int32))
        net.spike_monitor(P, 10**6)
        net.spike_monitor(G, 10**6)
        net.finalize()
        ids[name] = (P, G)
    for _ in range(5):
        gpu.run(K)
        orc.set_uniforms(ids["orc"][0], gpu.rng_uniforms(ids["gpu"][0], K))
        orc.run(K)
    for k in (0, 1):
        a, b = gpu.spikes(ids["gpu"][k]), orc.spikes(ids["orc"][k])
        np.testing.assert_array_equal(a[1], b[1])
        np.testing.assert_array_equal(a[0], b[0])
    ip, sp = gpu.spikes(ids["gpu"][0])
    assert len(ip) > 500 and not np.any((sp >= 60) & (sp < 90))   # the rate-0 row
    assert len(gpu.spikes(ids["gpu"][1])[0]) > 0
    np.testing.assert_allclose(gpu.get_state(ids["gpu"][1], "v"),
                               orc.get_state(ids["orc"][1], "v"), rtol=1e-10, atol=1e-15)
