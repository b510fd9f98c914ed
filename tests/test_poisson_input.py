"""PoissonInput (Brian2's PoissonInput, drawn by the BinomialFunction of
brian2cuda/binomial.py:12-121): every step each neuron of the target group adds
weight * Binomial(N, rate*dt) to v, ge or gi, in the synapses slot.

The oracle's draw is pinned statistically (the reference has no fixed vectors for it: its
draws come from cuRAND states): after one step of a group without dynamics, v holds the
draws themselves, whose mean and variance must be those of the binomial.  The CUDA library
draws from the same counter-based Philox stream with the same inversion, so it is compared
with the oracle exactly.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from brian2cuda_b200 import models
from brian2cuda_b200.network import LIF

DT = 1e-4
mV = 1e-3


def _draws(make, n_neurons, N, rate, steps=1, seed=5):
    net = make(DT, seed=seed)
    G = net.lif_group(n_neurons, LIF(El=0.0, taum=math.inf, has_threshold=False,
                                     has_reset=False), "float64")
    net.poisson_input(G, "v", N, rate, 1.0)
    net.finalize()
    out = []
    for _ in range(steps):
        before = net.get_state(G, "v").copy()
        net.run(1)
        out.append(net.get_state(G, "v") - before)
    return np.array(out)


@pytest.mark.parametrize("N,rate", [(1000, 10.0), (50, 2000.0), (400, 7000.0), (3, 9000.0)])
def test_oracle_binomial_moments(oracle_factory, N, rate):
    """p = rate*dt from 1e-3 to 0.9 (the upper ones drawn reversed): mean N p and variance
    N p q within 5 standard errors, values integers in [0, N]."""
    x = _draws(oracle_factory, 20000, N, rate, steps=3).ravel()
    p = rate * DT
    assert np.all(x == np.round(x)) and x.min() >= 0 and x.max() <= N
    m, v = N * p, N * p * (1 - p)
    se_mean = math.sqrt(v / len(x))
    assert abs(x.mean() - m) < 5 * se_mean + 1e-12
    # variance of the sample variance ~ (mu4 - v^2)/n, mu4 = v (1 + 3 (N - 2) p q) for the binomial
    mu4 = v * (1 + 3 * (N - 2) * p * (1 - p))
    se_var = math.sqrt(max(mu4 - v * v, 1e-30) / len(x))
    assert abs(x.var() - v) < 5 * se_var + 1e-12


def test_oracle_binomial_streams_differ_by_neuron_and_step(oracle_factory):
    x = _draws(oracle_factory, 5000, 100, 1000.0, steps=2)   # p = 0.1
    assert np.mean(x[0] == x[1]) < 0.3                        # P(equal) ~ 0.13 when independent
    assert len(np.unique(x[0])) > 10
    y = _draws(oracle_factory, 5000, 100, 1000.0, steps=2, seed=6)
    assert not np.array_equal(x, y)


def test_oracle_poisson_input_zero_inputs(oracle_factory):
    assert not np.any(_draws(oracle_factory, 100, 0, 50.0, steps=2))


@pytest.mark.gpu
@pytest.mark.parametrize("N,rate", [(1000, 10.0), (400, 7000.0), (5000, 300.0)])
def test_gpu_binomial_draws_equal_oracle(gpu_factory, oracle_factory, N, rate):
    g = _draws(gpu_factory, 30000, N, rate, steps=3)
    o = _draws(oracle_factory, 30000, N, rate, steps=3)
    np.testing.assert_array_equal(g, o)


def _lif_net_with_inputs(net, n=800, seed=13):
    """CUBA LIF, recurrent synapses with delays, a PoissonInput onto ge and one onto v (the
    reset variable: its order against the reset matters)."""
    rng = np.random.default_rng(seed)
    G = net.lif_group(n, models.cuba_lif(), "float64")
    net.set_state(G, "v", rng.uniform(-60 * mV, -50 * mV, n))
    i, j = models.bernoulli_pairs(rng, n, n, 0.03)
    d = rng.integers(1, 7, size=len(i)).astype(np.int32)
    ne = int(0.8 * n)
    exc = i < ne
    net.synapses(G, G, "ge", i[exc], j[exc], w_scalar=1.62 * mV, delay=d[exc])
    net.synapses(G, G, "gi", i[~exc], j[~exc], w_scalar=-9 * mV, delay=d[~exc])
    net.poisson_input(G, "ge", 200, 20.0, 0.5 * mV)
    net.poisson_input(G, "v", 50, 40.0, 0.8 * mV)
    net.spike_monitor(G, 10**6)
    return G


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["per-step", "two launches", "reset first"])
def test_lif_poisson_input_matches_oracle(gpu_factory, oracle_factory, form):
    out = {}
    rf = form == "reset first"
    for name in ("gpu", "orc"):
        if name == "orc":
            net = oracle_factory(DT, seed=9, reset_before_synapses=rf)
        else:
            net = gpu_factory(DT, seed=9, reset_before_synapses=rf,
                              two_launch=True if form == "two launches" else False)
        G = _lif_net_with_inputs(net)
        net.finalize()
        if name == "gpu":
            assert net.run_mode == ("two-launch" if form == "two launches" else "per-step")
        net.run(150)
        net.run(100)
        idx, st = net.spikes(G)
        out[name] = (idx, st, net.get_state(G, "v"), net.get_state(G, "ge"))
    assert len(out["orc"][0]) > 200
    np.testing.assert_array_equal(out["gpu"][1], out["orc"][1])
    np.testing.assert_array_equal(out["gpu"][0], out["orc"][0])
    np.testing.assert_allclose(out["gpu"][2], out["orc"][2], rtol=1e-10, atol=1e-15)
    np.testing.assert_allclose(out["gpu"][3], out["orc"][3], rtol=1e-10, atol=1e-15)


@pytest.mark.gpu
def test_hh_poisson_input_float32_matches_oracle(gpu_factory, oracle_factory):
    """COBAHH float32 with a PoissonInput onto ge (1000 inputs at 5 Hz, 2 nS): spikes within
    one step of the float32 oracle's, both ways."""
    out = {}
    for name in ("gpu", "orc"):
        net = (oracle_factory(DT, f32=True, seed=4) if name == "orc"
               else gpu_factory(DT, seed=4))
        ids = models.build_cobahh(net, n=2000, p=0.02, generated=False, monitor_capacity=10**6)
        net.poisson_input(ids["P"], "ge", 1000, 5.0, 2e-9)
        net.finalize()
        net.run(150)
        out[name] = net.spikes(ids["P"])
    (gi, gs), (oi, os_) = out["gpu"], out["orc"]
    assert len(oi) > 20
    for a, b in (((gi, gs), (oi, os_)), ((oi, os_), (gi, gs))):
        keys = set(zip(b[0].tolist(), b[1].tolist()))
        assert all(any((i, s + o) in keys for o in (-1, 0, 1))
                   for i, s in zip(a[0].tolist(), a[1].tolist()))


@pytest.mark.gpu
def test_poisson_input_rejects_bad_arguments(gpu_factory):
    net = gpu_factory(DT)
    G = net.lif_group(10, models.cuba_lif(), "float64")
    P = net.poisson_group(10, 5.0)
    with pytest.raises(Exception):
        net.poisson_input(P, "v", 10, 5.0, 1.0)       # not a LIF or HH group
    with pytest.raises(Exception):
        net.poisson_input(G, "m", 10, 5.0, 1.0)       # not v, ge or gi
    with pytest.raises(Exception):
        net.poisson_input(G, "v", 10, 2e4, 1.0)       # rate * dt above 1
    net.poisson_input(G, "v", 10, 5.0, 1.0)
    net.poisson_input(G, "ge", 10, 5.0, 1.0)
    with pytest.raises(Exception):
        net.poisson_input(G, "gi", 10, 5.0, 1.0)      # a third one
