"""Parity of the CUDA library (through the C ABI) with the CPU oracle on seeded inputs.

Tolerances: float64 state within 1e-10 relative of the float64 oracle (the exact-LIF update
is bit-identical: both sides evaluate the same fused multiply-adds); float32 state within
1e-5 relative (plus an absolute floor of 1e-5 of the variable's scale) of the float64
oracle; spike indices, spike counts per step and delay-queue contents exactly.
"""
import math

import numpy as np
import pytest

from brian2cuda_b200 import models
from brian2cuda_b200.network import LIF

pytestmark = pytest.mark.gpu
DT = 1e-4
mV = 1e-3


def _close(a, b, rtol, atol):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    bad = np.abs(a - b) > rtol * np.abs(b) + atol
    assert not bad.any(), f"{bad.sum()} mismatches, worst {np.max(np.abs(a - b))}"


def _random_lif_state(net, G, n, rng, t0_steps):
    net.set_state(G, "v", rng.uniform(-62 * mV, -48 * mV, n))
    net.set_state(G, "ge", rng.uniform(-2 * mV, 5 * mV, n))
    net.set_state(G, "gi", rng.uniform(-9 * mV, 0, n))
    net.set_state(G, "lastspike", (t0_steps - rng.integers(0, 100, n)) * DT)


def test_lif_float64_step_is_bit_exact(gpu_factory, oracle_factory):
    n = 5003
    out = {}
    for name, make in (("gpu", gpu_factory), ("orc", oracle_factory)):
        rng = np.random.default_rng(7)
        net = make(DT)
        G = net.lif_group(n, models.cuba_lif(), "float64")
        _random_lif_state(net, G, n, rng, 0)
        net.spike_monitor(G, 10 * n)
        net.finalize()
        net.run(1)
        out[name] = {v: net.get_state(G, v) for v in ("v", "ge", "gi", "lastspike")}
        out[name]["spk"] = np.sort(net.spikes(G)[0])
    for v in ("v", "ge", "gi", "lastspike"):
        np.testing.assert_array_equal(out["gpu"][v], out["orc"][v], err_msg=v)
    np.testing.assert_array_equal(out["gpu"]["spk"], out["orc"]["spk"])
    assert len(out["gpu"]["spk"]) > 0


def _random_hh_state(net, P, n, rng):
    net.set_state(P, "v", rng.uniform(-80 * mV, 10 * mV, n))
    net.set_state(P, "m", rng.uniform(0, 1, n))
    net.set_state(P, "h", rng.uniform(0, 1, n))
    net.set_state(P, "n", rng.uniform(0, 1, n))
    net.set_state(P, "ge", rng.uniform(0, 80e-9, n))
    net.set_state(P, "gi", rng.uniform(0, 400e-9, n))
    lastspike = -rng.integers(0, 60, n) * DT
    net.set_state(P, "lastspike", lastspike)
    return lastspike


def test_hh_float32_step_within_tolerance(gpu_factory, oracle_factory):
    n = 20000
    res = {}
    for name, make in (("gpu", gpu_factory), ("orc", oracle_factory)):
        rng = np.random.default_rng(11)
        net = make(DT)
        P = net.hh_group(n, models.cobahh_hh(), "float32")
        ls = _random_hh_state(net, P, n, rng)
        net.spike_monitor(P, 10 * n)
        net.finalize()
        net.run(1)
        res[name] = {v: net.get_state(P, v) for v in ("v", "m", "h", "n", "ge", "gi")}
        res[name]["spk"] = np.sort(net.spikes(P)[0])
    scale = {"v": 0.1, "m": 1, "h": 1, "n": 1, "ge": 80e-9, "gi": 400e-9}
    for v in scale:
        _close(res["gpu"][v], res["orc"][v], 1e-5, 1e-5 * scale[v])
    # spikes given the same state: the GPU's own post-update v decides, exactly
    v = res["gpu"]["v"]
    nr = ((0 - ls + 1e-3 * DT) / DT).astype(np.int64) >= 30
    expect = np.nonzero((v > np.float32(-20 * mV)) & nr)[0]
    np.testing.assert_array_equal(res["gpu"]["spk"], expect)


def test_cuba_rollout_float64(gpu_factory, oracle_factory):
    out = {}
    for name, make in (("gpu", gpu_factory), ("orc", oracle_factory)):
        net = make(DT)
        ids = models.build_cuba(net, n=1000, p=0.05, dtype="float64")
        net.finalize()
        net.run(300)
        idx, st = net.spikes(ids["P"])
        out[name] = (idx, st, net.get_state(ids["P"], "v"), net.get_state(ids["P"], "ge"))
    gi, gs, gv, gge = out["gpu"]
    oi, os_, ov, oge = out["orc"]
    assert len(gi) > 100
    np.testing.assert_array_equal(gs, os_)
    np.testing.assert_array_equal(gi, oi)
    _close(gv, ov, 1e-10, 1e-15)
    _close(gge, oge, 1e-10, 1e-15)


def _delay_net(net, n=800, p=0.05, seed=3):
    rng = np.random.default_rng(seed)
    G = net.lif_group(n, models.cuba_lif(), "float64")
    net.set_state(G, "v", rng.uniform(-60 * mV, -50 * mV, n))
    i, j = models.bernoulli_pairs(rng, n, n, p)
    d = rng.integers(1, 17, size=len(i)).astype(np.int32)
    ne = int(0.8 * n)
    exc = i < ne
    Ce = net.synapses(G, G, "ge", i[exc], j[exc], w=np.full(exc.sum(), 1.62 * mV), delay=d[exc])
    Ci = net.synapses(G, G, "gi", i[~exc], j[~exc], w_scalar=-9 * mV, delay=d[~exc])
    net.spike_monitor(G, 10**6)
    return G, Ce, Ci, (i, j, d, exc)


def test_heterogeneous_delays_rollout_and_queue(gpu_factory, oracle_factory):
    out = {}
    for name, make in (("gpu", gpu_factory), ("orc", oracle_factory)):
        net = make(DT)
        G, Ce, Ci, _ = _delay_net(net)
        net.finalize()
        net.run(237)
        idx, st = net.spikes(G)
        out[name] = (idx, st, net.queue(Ce), net.queue(Ci), net.get_state(G, "v"))
    for k in range(4):
        np.testing.assert_array_equal(out["gpu"][k], out["orc"][k], err_msg=str(k))
    assert len(out["gpu"][0]) > 100 and len(out["gpu"][2]) > 0
    _close(out["gpu"][4], out["orc"][4], 1e-10, 1e-15)


def test_merged_synapses_onto_two_variables_of_few_targets(gpu_factory, oracle_factory):
    """Two Synapses objects from disjoint halves of one source onto ge and onto gi of a
    40-neuron target: one projection with two members, delivered with warp-aggregated atomics
    (fewer than 64 targets), so lanes of one warp add to the same index of different
    variables."""
    n_src, n_dst, half = 256, 40, 128
    sg_idx = np.tile(np.arange(n_src), 10)
    sg_step = np.repeat(np.arange(0, 20, 2), n_src)
    i = np.repeat(np.arange(n_src), n_dst).astype(np.int32)
    j = np.tile(np.arange(n_dst), n_src).astype(np.int32)
    e = i < half
    prm = LIF(El=-49 * mV, taum=20e-3, taue=5e-3, taui=10e-3, ke=1.0, ki=1.0,
              has_threshold=False, has_reset=False)
    out = {}
    for name, make in (("gpu", gpu_factory), ("orc", oracle_factory)):
        net = make(DT)
        S = net.spikegen_group(n_src, sg_idx, sg_step)
        G = net.lif_group(n_dst, prm, "float64")
        net.set_state(G, "v", np.full(n_dst, -49 * mV))
        net.synapses(S, G, "ge", i[e], j[e], w_scalar=0.5 * mV,
                     delay=np.ones(int(e.sum()), np.int32))
        net.synapses(S, G, "gi", i[~e], j[~e], w_scalar=-0.25 * mV,
                     delay=np.full(int((~e).sum()), 2, np.int32))
        net.finalize()
        net.run(25)
        out[name] = {v: net.get_state(G, v) for v in ("ge", "gi", "v")}
    assert np.all(out["orc"]["ge"] > 0) and np.all(out["orc"]["gi"] < 0)
    for v in ("ge", "gi", "v"):
        _close(out["gpu"][v], out["orc"][v], 1e-10, 1e-15)


def test_delays_changed_between_runs_match_oracle(gpu_factory, oracle_factory):
    """Delays changed between runs while spikes are in flight (Brian2's `S.delay = ...`):
    first longer than the spike-history ring holds (the ring grows), then with delays of 0
    (the net leaves the two-launch form for the per-step kernels); spikes exact, v within
    1e-10, synapse delays read back in input order."""
    out = {}
    for name, make in (("gpu", gpu_factory), ("orc", oracle_factory)):
        net = make(DT)
        G, Ce, Ci, (i, j, d, exc) = _delay_net(net, n=800)
        net.finalize()
        if name == "gpu":
            assert net.run_mode == "two-launch"
        net.run(100)
        d1 = np.random.default_rng(5).integers(1, 41, size=int(exc.sum())).astype(np.int32)
        net.syn_set_delays(Ce, d1)
        net.run(150)
        d2 = np.random.default_rng(6).integers(0, 6, size=int((~exc).sum())).astype(np.int32)
        net.syn_set_delays(Ci, d2)
        net.run(120)
        if name == "gpu":
            assert net.run_mode == "per-step"
            np.testing.assert_array_equal(net.syn_get(Ce, "delay"), d1)
            np.testing.assert_array_equal(net.syn_get(Ci, "delay"), d2)
        idx, st = net.spikes(G)
        out[name] = (idx, st, net.get_state(G, "v"))
    assert len(out["gpu"][0]) > 150
    np.testing.assert_array_equal(out["gpu"][1], out["orc"][1])
    np.testing.assert_array_equal(out["gpu"][0], out["orc"][0])
    _close(out["gpu"][2], out["orc"][2], 1e-10, 1e-15)


def test_cluster_accumulation_delivers_the_same_input(gpu_factory):
    """Additive delivery accumulated in the distributed shared memory of thread-block
    clusters (autotuner site kind 12) adds the same input as one atomic per event: a
    20,000-neuron Poisson source at 400 Hz onto ge and gi of 50,000 float32 LIF targets that
    do not spike, delays 1-20 steps, per-synapse weights onto ge; ge and gi within 1e-5
    relative after 60 steps (the partial sums are grouped differently)."""
    out = {}
    for cluster in (0, 1):
        net = gpu_factory(DT, seed=3)
        S = net.poisson_group(20_000, 400.0, "float32")
        G = net.lif_group(50_000, LIF(El=0.0, taum=20e-3, taue=5e-3, taui=10e-3, ke=1.0,
                                      ki=1.0, has_threshold=False, has_reset=False), "float32")
        rng = np.random.default_rng(8)
        i, j = models.bernoulli_pairs(rng, 20_000, 50_000, 0.01)
        d = rng.integers(1, 21, size=len(i)).astype(np.int32)
        e = i < 16_000
        net.synapses(S, G, "ge", i[e], j[e], w=rng.uniform(0.5e-3, 1e-3, int(e.sum())),
                     delay=d[e])
        net.synapses(S, G, "gi", i[~e], j[~e], w_scalar=-1e-3, delay=d[~e])
        net.finalize()
        assert net.run_mode == "per-step"
        if cluster:
            net.tune_apply([{"site_kind": 12, "site_index": b, "choice_a": 1, "choice_b": 0}
                            for b in range(2)])
        net.run(60)
        out[cluster] = (net.get_state(G, "ge"), net.get_state(G, "gi"))
    for k in range(2):
        a, b = out[1][k].astype(np.float64), out[0][k].astype(np.float64)
        assert np.abs(b).max() > 0
        _close(a, b, 1e-5, 1e-5 * np.abs(b).max())


def test_synapse_readback_in_input_order(gpu_factory):
    net = gpu_factory(DT)
    G, Ce, Ci, (i, j, d, exc) = _delay_net(net, n=300)
    net.finalize()
    for sid, sel in ((Ce, exc), (Ci, ~exc)):
        np.testing.assert_array_equal(net.syn_get(sid, "i"), i[sel])
        np.testing.assert_array_equal(net.syn_get(sid, "j"), j[sel])
        np.testing.assert_array_equal(net.syn_get(sid, "delay"), d[sel])
    np.testing.assert_array_equal(net.syn_get(Ce, "w"), np.full(exc.sum(), 1.62 * mV))
    np.testing.assert_array_equal(net.syn_get(Ci, "w"), np.full((~exc).sum(), -9 * mV))


def test_generated_connectivity_matches_oracle(gpu_factory, oracle_factory):
    out = {}
    for name, make in (("gpu", gpu_factory), ("orc", oracle_factory)):
        net = make(DT)
        A = net.lif_group(300, models.cuba_lif(), "float64")
        B = net.lif_group(517, models.cuba_lif(), "float64")
        s1 = net.synapses_random(A, B, "ge", 0.05, 1, 20, 1e-3, 12345, pre_range=(0, 240))
        s2 = net.synapses_random(A, B, "gi", 0.1, 3, 3, -1e-3, 999, pre_range=(240, 300))
        net.finalize()
        out[name] = [net.syn_get(s, v) for s in (s1, s2) for v in ("i", "j", "delay")]
    for a, b in zip(out["gpu"], out["orc"]):
        np.testing.assert_array_equal(a, b)
    assert len(out["gpu"][0]) > 1000


# STDP projection 0: records grouped by postsynaptic neuron (autotuner site kind 8)
POST_GROUPED = [{"site_kind": 8, "site_index": 0, "choice_a": 1, "choice_b": 0}]
SYNAPSE_ORDER = [{"site_kind": 8, "site_index": 0, "choice_a": 0, "choice_b": 0}]


@pytest.mark.parametrize("post_grouped", [False, True])
def test_stdp_with_poisson_input(gpu_factory, oracle_factory, post_grouped):
    K = 50
    gpu = gpu_factory(DT, steps_per_graph=K, seed=5)
    orc = oracle_factory(DT)
    ids = {}
    for name, net in (("gpu", gpu), ("orc", orc)):
        ids[name] = models.build_stdp(net, n_in=400, n_out=60, rate=80.0, dtype="float64",
                                      monitor_capacity=10**6)
        net.finalize()
    if post_grouped:
        gpu.tune_apply(POST_GROUPED)
    for _ in range(8):
        gpu.run(K)
        orc.set_uniforms(ids["orc"]["inp"], gpu.rng_uniforms(ids["gpu"]["inp"], K))
        orc.run(K)
    for g in ("inp", "out"):
        a, b = gpu.spikes(ids["gpu"][g]), orc.spikes(ids["orc"][g])
        np.testing.assert_array_equal(a[1], b[1])
        np.testing.assert_array_equal(a[0], b[0])
    assert len(gpu.spikes(ids["gpu"]["out"])[0]) > 0
    for v in ("w", "Apre", "Apost", "lastupdate"):
        _close(gpu.syn_get(ids["gpu"]["S"], v), orc.syn_get(ids["orc"]["S"], v), 1e-10, 1e-18)


def test_stdp_record_order_keeps_snapshots(gpu_factory):
    """Changing the record order permutes the stored snapshot with the live records: runs
    from one snapshot agree whatever order was in use when it was taken or restored."""
    net = gpu_factory(DT, steps_per_graph=25, seed=5)
    ids = models.build_stdp(net, n_in=300, n_out=40, rate=80.0, dtype="float64",
                            monitor_capacity=10**6)
    net.finalize()
    net.run(60)
    w0 = net.syn_get(ids["S"], "w")
    net.store(0)
    res = []
    for order in (SYNAPSE_ORDER, POST_GROUPED, SYNAPSE_ORDER):
        net.tune_apply(order)
        net.restore(0)
        np.testing.assert_array_equal(net.syn_get(ids["S"], "w"), w0)
        start = net.spikes_recorded(ids["out"])
        net.run(90)
        idx, st, _ = net.spikes_fetch(ids["out"], start)
        res.append((idx, st, net.syn_get(ids["S"], "w"), net.syn_get(ids["S"], "Apost")))
    assert len(res[0][0]) > 0
    for r in res[1:]:
        np.testing.assert_array_equal(r[1], res[0][1])
        np.testing.assert_array_equal(np.sort(r[0]), np.sort(res[0][0]))
        _close(r[2], res[0][2], 1e-12, 1e-18)
        _close(r[3], res[0][3], 1e-12, 1e-18)


def test_poisson_spikes_follow_uniforms(gpu_factory):
    K = 20
    net = gpu_factory(DT, steps_per_graph=K, seed=9)
    P = net.poisson_group(1000, 300.0, "float32")
    net.spike_monitor(P, 10**5)
    net.finalize()
    net.run(K)
    u = net.rng_uniforms(P, K)
    idx, st = net.spikes(P)
    exp_st, exp_idx = np.nonzero(u < np.float32(300.0 * DT))
    np.testing.assert_array_equal(st, exp_st)
    np.testing.assert_array_equal(idx, exp_idx)
    assert 0.0 < u.min() and u.max() <= 1.0


def _hines_pair(gpu_factory, channel_dtype, n_neurons=6, steps=300):
    from oracle.oracle import OracleHines
    net = gpu_factory(25e-6)
    hb, morph, params, current = models.build_hines(net, n_neurons=n_neurons,
                                                    channel_dtype=channel_dtype,
                                                    comp_range=(40, 160))
    orc = OracleHines(25e-6, morph["comp_off"], morph["sec_off"], morph["sec_start"],
                      morph["sec_end"], morph["sec_parent"], morph["diameter"], morph["length"],
                      params, f32=(channel_dtype == "float32"))
    for k, v in models.hines_rest_state().items():
        orc.set_state(k, v)
    orc.set_current(current)
    hb.run(steps)
    orc.run(steps)
    return hb, orc


def test_hines_float64_channels(gpu_factory):
    hb, orc = _hines_pair(gpu_factory, "float64")
    for v, atol in (("v", 1e-15), ("m", 1e-15), ("h", 1e-15), ("n", 1e-15), ("Ic", 1e-12)):
        _close(hb.get_state(v), orc.get_state(v), 1e-10, atol)
    np.testing.assert_array_equal(hb.spike_counts(), orc.spike_counts())


def test_hines_float32_channels(gpu_factory):
    hb, orc = _hines_pair(gpu_factory, "float32")
    _close(hb.get_state("v"), orc.get_state("v"), 1e-4, 1e-6)
    for v in ("m", "h", "n"):
        _close(hb.get_state(v), orc.get_state(v), 1e-4, 1e-5)


def test_monitor_overflow_is_reported(gpu_factory):
    from brian2cuda_b200 import B2BError
    net = gpu_factory(DT)
    G = net.lif_group(100, LIF(taum=math.inf, Vt=-math.inf, has_reset=False), "float64")
    net.spike_monitor(G, 150)
    net.finalize()
    net.run(3)
    assert net.sync() == 3  # B2B_ERR_QUEUE_OVERFLOW
    with pytest.raises(B2BError):
        net.spikes(G)


def test_state_and_rate_monitors_match_oracle(gpu_factory, oracle_factory):
    """StateMonitor (start of the step, every k steps) and PopulationRateMonitor (spike count
    at the end of the step) against the oracle, across two runs: CUBA 1000 float64, and two
    groups of one population (the rate monitor of each counts only its own neurons)."""
    out = {}
    for name, make in (("gpu", gpu_factory), ("orc", oracle_factory)):
        net = make(DT)
        ids = models.build_cuba(net, n=1000, p=0.05, dtype="float64")
        P = ids["P"]
        A = net.lif_group(300, models.cuba_lif(), "float64")
        B = net.lif_group(200, models.cuba_lif(), "float64")
        rng = np.random.default_rng(4)
        for G, n in ((A, 300), (B, 200)):
            net.set_state(G, "v", rng.uniform(-60 * mV, -48 * mV, n))
        net.synapses(A, B, "ge", np.arange(300, dtype=np.int32) % 200,
                     np.arange(300, dtype=np.int32) % 200, w_scalar=2 * mV, delay=3)
        mons = [net.state_monitor(P, "v", [0, 17, 999], every=1, capacity=400),
                net.state_monitor(P, "ge", None, every=7, capacity=100),
                net.state_monitor(B, "v", [5, 199], every=3, capacity=100)]
        rates = [net.rate_monitor(G, capacity=400) for G in (P, A, B)]
        net.finalize()
        net.run(120)
        net.run(130)
        out[name] = ([net.state_values(m) for m in mons], [net.rate_counts(r) for r in rates])
    for (gs, gv), (os_, ov) in zip(out["gpu"][0], out["orc"][0]):
        np.testing.assert_array_equal(gs, os_)
        assert gv.shape == ov.shape and len(gs) > 0
        _close(gv, ov, 1e-10, 1e-15)
    assert list(out["gpu"][0][0][0]) == list(range(250))
    assert list(out["gpu"][0][1][0]) == list(range(0, 250, 7))
    for (gs, gc), (os_, oc) in zip(out["gpu"][1], out["orc"][1]):
        np.testing.assert_array_equal(gs, os_)
        np.testing.assert_array_equal(gc, oc)
    assert out["gpu"][1][0][1].sum() > 100 and out["gpu"][1][2][1].sum() > 0


def test_state_monitor_overflow_is_reported(gpu_factory):
    net = gpu_factory(DT)
    G = net.lif_group(100, models.cuba_lif(), "float64")
    m = net.state_monitor(G, "v", None, every=1, capacity=10)
    r = net.rate_monitor(G, capacity=40)
    net.finalize()
    net.run(30)
    assert net.sync() == 3  # B2B_ERR_QUEUE_OVERFLOW
    steps, vals = net.state_values(m)
    assert list(steps) == list(range(10)) and vals.shape == (10, 100)
    assert list(net.rate_counts(r)[0]) == list(range(30))


def test_graph_and_eager_agree(gpu_factory):
    res = []
    for graphs in (True, False):
        net = gpu_factory(DT, graphs=graphs, steps_per_graph=25)
        G, Ce, Ci, _ = _delay_net(net, n=400)
        net.finalize()
        net.run(113)
        res.append(net.spikes(G))
        assert net.kernel_launches > 0
    np.testing.assert_array_equal(res[0][0], res[1][0])
    np.testing.assert_array_equal(res[0][1], res[1][1])


def test_store_restore_replays_identically(gpu_factory):
    net = gpu_factory(DT, steps_per_graph=20)
    G, Ce, Ci, _ = _delay_net(net, n=600)
    net.finalize()
    net.run(37)
    net.store(0)
    q0 = net.queue(Ce)
    n0 = net.spikes_recorded(G)
    net.run(160)
    idx1, st1, _ = net.spikes_fetch(G, n0)
    v1 = net.get_state(G, "v")
    net.restore(0)
    assert net.timestep == 37
    np.testing.assert_array_equal(net.queue(Ce), q0)
    n1 = net.spikes_recorded(G)
    net.run(160)
    idx2, st2, _ = net.spikes_fetch(G, n1)
    order1, order2 = np.lexsort((idx1, st1)), np.lexsort((idx2, st2))
    np.testing.assert_array_equal(st1[order1], st2[order2])
    np.testing.assert_array_equal(idx1[order1], idx2[order2])
    _close(net.get_state(G, "v"), v1, 1e-12, 1e-15)
    assert len(idx1) > 50


# the three forms of a step for nets whose every delay is >= 1 step: Network kwargs
FORMS = {"per-step": dict(two_launch=False), "two-launch": dict(two_launch=True),
         "one-launch": dict(one_launch=True)}


def test_step_forms_agree(gpu_factory):
    """The per-step kernels, the two concurrent launches and the one launch holding both
    halves of a step compute the same network (float64 LIF, delays 1-16 steps; a chunk
    boundary mid-run)."""
    res = {}
    for form, kw in list(FORMS.items()) + [("chained", FORMS["one-launch"])]:
        net = gpu_factory(DT, **kw)
        G, Ce, Ci, _ = _delay_net(net, n=1000)
        net.finalize()
        if form == "chained":
            # each step's launch chained to the previous one (programmatic dependent launch)
            net.tune_apply([{"site_kind": 11, "site_index": 0, "choice_a": 3, "choice_b": 148}])
            assert net.run_mode == "one-launch"
        else:
            assert net.run_mode == form
        net.run(150)
        net.run(89)
        idx, st = net.spikes(G)
        res[form] = (idx, st, net.get_state(G, "v"), net.get_state(G, "ge"), net.queue(Ce))
    assert len(res["per-step"][0]) > 100
    for form in ("two-launch", "one-launch", "chained"):
        for k in (0, 1, 4):
            np.testing.assert_array_equal(res[form][k], res["per-step"][k])
        _close(res[form][2], res["per-step"][2], 1e-10, 1e-15)
        _close(res[form][3], res["per-step"][3], 1e-10, 1e-15)


def test_delivery_lanes_per_item_agree(gpu_factory):
    """Every delivery launch shape computes the same network: lanes per work item 2-32 for the
    per-step delivery (site kind 6) and 2-16 for the pending delivery of the two launches
    (site kind 5), against the built-in shapes (float64 LIF, delays 1-16 steps, bundles of a
    few synapses)."""
    def run(form, tune):
        net = gpu_factory(DT, **FORMS[form])
        G, Ce, Ci, _ = _delay_net(net, n=1000)
        net.finalize()
        if tune:
            net.tune_apply(tune)
        net.run(200)
        idx, st = net.spikes(G)
        return idx, st, net.get_state(G, "v")
    for form, kind, groups in (("per-step", 6, (2, 4, 16, 32)), ("two-launch", 5, (2, 4, 16))):
        ref = run(form, None)
        assert len(ref[0]) > 100
        for g in groups:
            got = run(form, [{"site_kind": kind, "site_index": 0, "choice_a": g,
                              "choice_b": 148}])
            np.testing.assert_array_equal(got[1], ref[1], err_msg=f"{form} {g}")
            np.testing.assert_array_equal(got[0], ref[0], err_msg=f"{form} {g}")
            _close(got[2], ref[2], 1e-10, 1e-15)


def test_profile_advances_like_run(gpu_factory):
    """The profiling run launches every kernel eagerly and times it; in either form of the
    step it reports the form's launch sites and leaves the net where b2b_run would."""
    sites = {"per-step": [1, 6, 6], "two-launch": [5, 1], "one-launch": [13]}
    for form, kw in FORMS.items():
        out = {}
        for how in ("run", "profile"):
            net = gpu_factory(DT, **kw)
            G, Ce, Ci, _ = _delay_net(net, n=1000)
            net.finalize()
            net.run(40)
            if how == "run":
                net.run(130)
            else:
                prof = net.profile(130)
                kinds = [k for k, _ in prof]
                # per-step: Ce (a weight per synapse) and Ci (one scalar weight) are two
                # kernel variants, so two delivery launches
                assert kinds == sites[form], kinds
                assert all(ms > 0 for _, ms in prof)
            assert net.timestep == 170
            net.run(30)
            idx, st = net.spikes(G)
            out[how] = (idx, st, net.get_state(G, "v"), net.get_state(G, "ge"), net.queue(Ce))
        assert len(out["run"][0]) > 50
        for k in (0, 1, 4):
            np.testing.assert_array_equal(out["profile"][k], out["run"][k])
        _close(out["profile"][2], out["run"][2], 1e-12, 1e-15)
        _close(out["profile"][3], out["run"][3], 1e-12, 1e-15)


def test_profile_graph_advances_like_run(gpu_factory):
    """Timing every launch site inside the replayed step graphs (event-record nodes) leaves
    the net where b2b_run would, and the per-site times fit inside the step: in the per-step
    form the sites run one after another, so their sum is at most the step time; in the
    two-launch form each of the two overlapping sites is."""
    sites = {"per-step": [1, 6, 6], "two-launch": [5, 1], "one-launch": [13]}
    for form, kw in FORMS.items():
        out = {}
        for how in ("run", "profile"):
            net = gpu_factory(DT, steps_per_graph=25, **kw)
            G, Ce, Ci, _ = _delay_net(net, n=1000)
            net.finalize()
            net.run(40)
            if how == "run":
                net.run(150)
            else:
                prof, step_ms = net.profile_graph(150)
                kinds = [k for k, _ in prof]
                assert kinds == sites[form], kinds
                assert all(ms > 0 for _, ms in prof) and step_ms > 0
                if form == "two-launch":
                    assert max(ms for _, ms in prof) <= step_ms
                else:
                    assert sum(ms for _, ms in prof) <= step_ms
            assert net.timestep == 190
            net.run(30)
            idx, st = net.spikes(G)
            out[how] = (idx, st, net.get_state(G, "v"), net.queue(Ce))
        assert len(out["run"][0]) > 50
        for k in (0, 1, 3):
            np.testing.assert_array_equal(out["profile"][k], out["run"][k])
        _close(out["profile"][2], out["run"][2], 1e-12, 1e-15)


def _spikes_within_one_step(a_idx, a_stp, b_idx, b_stp):
    """Fraction of spikes of a that b has at the same neuron within one step."""
    keys = set(zip(b_idx.tolist(), b_stp.tolist()))
    hit = sum(1 for i, s in zip(a_idx.tolist(), a_stp.tolist())
              if (i, s) in keys or (i, s - 1) in keys or (i, s + 1) in keys)
    return hit / max(1, len(a_idx))


@pytest.mark.parametrize("form", ["two-launch", "one-launch"])
def test_two_launch_cobahh_float32_matches_oracle(gpu_factory, oracle_factory, form):
    out = {}
    for name, make in (("gpu", gpu_factory), ("orc", oracle_factory)):
        net = make(DT, f32=True) if name == "orc" else make(DT, **FORMS[form])
        ids = models.build_cobahh(net, n=3000, p=0.02, generated=False, monitor_capacity=10**6)
        net.finalize()
        if name == "gpu":
            assert net.run_mode == form
        net.run(60)
        out[name] = (net.spikes(ids["P"]), {v: net.get_state(ids["P"], v)
                                            for v in ("v", "m", "h", "n", "ge", "gi")})
    (gi, gs), gstate = out["gpu"]
    (oi, os_), ostate = out["orc"]
    assert len(gi) > 10
    # a float32 rollout (the GPU's exp and division are the hardware forms, the oracle's the
    # correctly rounded ones): every spike within one step of the other side's, the
    # north star's rollout criterion; exact spike equality from the same state is checked by
    # test_hh_float32_step_within_tolerance
    assert _spikes_within_one_step(gi, gs, oi, os_) == 1.0
    assert _spikes_within_one_step(oi, os_, gi, gs) == 1.0
    assert abs(len(gi) - len(oi)) <= 0.01 * len(oi)
    # neurons caught mid-spike amplify float32 rounding (and the one-ulp-level differences
    # of the hardware exp) over the 60 steps, so bound the fraction; no bound on the largest
    # difference: a spike one step apart moves its targets' ge or gi by a whole weight
    scale = {"v": 0.1, "m": 1, "h": 1, "n": 1, "ge": 80e-9, "gi": 400e-9}
    for v, sc in scale.items():
        a, b = gstate[v].astype(np.float64), ostate[v]
        ok = np.abs(a - b) <= 1e-4 * np.abs(b) + 1e-4 * sc
        assert ok.mean() >= 0.98, (v, ok.mean())


def test_autotune_keeps_state_and_results(gpu_factory):
    """b2b_autotune leaves state, clock and monitors as they were, and the shapes it picks
    compute the same network (CUBA float64: every delivered weight of one target variable
    is equal, so the order of the atomic additions cannot change a sum)."""
    out = {}
    for tuned in (False, True):
        net = gpu_factory(DT)
        ids = models.build_cuba(net, n=1000, p=0.05, dtype="float64")
        net.finalize()
        net.run(100)
        before = (net.timestep, net.get_state(ids["P"], "v").copy(), len(net.spikes(ids["P"])[0]))
        if tuned:
            res = net.autotune(trial_steps=10)
            kinds = {r["site_kind"] for r in res}
            # one population of <= 4096 neurons: the small-network path is tried too (14)
            assert kinds == {1, 6, 14}
            assert all(r["best_ms"] <= r["default_ms"] for r in res)
            small = [r for r in res if r["site_kind"] == 14][0]
            assert net.run_mode == ("small" if small["choice_a"] > 0 else "per-step")
            after = (net.timestep, net.get_state(ids["P"], "v"), len(net.spikes(ids["P"])[0]))
            assert after[0] == before[0] and after[2] == before[2]
            np.testing.assert_array_equal(after[1], before[1])
        net.run(300)
        idx, st = net.spikes(ids["P"])
        out[tuned] = (idx, st, net.get_state(ids["P"], "v"))
    np.testing.assert_array_equal(out[True][0], out[False][0])
    np.testing.assert_array_equal(out[True][1], out[False][1])
    np.testing.assert_array_equal(out[True][2], out[False][2])
    # a small network: the tuner chooses one CTA or one cluster of 8 or 16 (site kind 14)
    net = gpu_factory(DT, small=True)
    models.build_cuba(net, n=1000, p=0.05, dtype="float64")
    net.finalize()
    assert net.run_mode == "small"
    res = net.autotune(trial_steps=5)
    assert [r["site_kind"] for r in res] == [14] and res[0]["choice_a"] in (1, 8, 16)
    assert net.run_mode == "small"


def test_autotune_chooses_step_form(gpu_factory):
    """A net that allows every form of the step (one population, additive synapses onto ge
    and gi, delays >= 1): the tuner tunes the per-step kernels, the two concurrent launches
    and the one launch, keeps the fastest form (site kind 11), leaves the state as it was, and
    every form computes the same network; tune_apply reproduces each form."""
    out = {}
    mode_of = {0: "per-step", 1: "two-launch", 2: "one-launch", 3: "one-launch"}
    for mode in ("untuned", "tuned", "per-step", "two launches", "one launch", "chained"):
        net = gpu_factory(DT)
        G, Ce, Ci, _ = _delay_net(net, n=800)
        net.finalize()
        assert net.run_mode == "two-launch"   # <= 2^18 neurons: the two launches until tuned
        net.run(60)
        v0 = net.get_state(G, "v").copy()
        if mode == "tuned":
            res = net.autotune(trial_steps=20)
            kinds = [r["site_kind"] for r in res]
            assert {1, 6, 5, 11} <= set(kinds), kinds
            form = [r for r in res if r["site_kind"] == 11][0]
            small = [r for r in res if r["site_kind"] == 14]
            if small and small[0]["choice_a"] > 0:   # the small-network path won
                assert net.run_mode == "small"
            else:
                assert net.run_mode == mode_of[form["choice_a"]]
            np.testing.assert_array_equal(net.get_state(G, "v"), v0)
            assert net.timestep == 60
        elif mode != "untuned":
            a = {"per-step": 0, "two launches": 1, "one launch": 2, "chained": 3}[mode]
            net.tune_apply([{"site_kind": 11, "site_index": 0, "choice_a": a,
                             "choice_b": 148 if a >= 2 else 0}])
            assert net.run_mode == mode_of[a]
        net.run(240)
        idx, st = net.spikes(G)
        out[mode] = (idx, st, net.get_state(G, "v"))
    assert len(out["untuned"][0]) > 100
    for mode in ("tuned", "per-step", "two launches", "one launch", "chained"):
        np.testing.assert_array_equal(out[mode][1], out["untuned"][1])
        np.testing.assert_array_equal(out[mode][0], out["untuned"][0])
        _close(out[mode][2], out["untuned"][2], 1e-10, 1e-15)


def test_out_degree_matches_synapses(gpu_factory):
    net = gpu_factory(DT)
    ids = models.build_cobahh(net, n=3000, p=0.03)
    net.finalize()
    want = np.zeros(3000, np.int64)
    for sid in (ids["Ce"], ids["Ci"]):
        want += np.bincount(net.syn_get(sid, "i"), minlength=3000)
    np.testing.assert_array_equal(net.out_degree(ids["P"]), want)


@pytest.mark.parametrize("case", ["cobahh_delays", "lif_onto_v_late_reset", "cuba"])
def test_small_network_path_matches_per_step(gpu_factory, case):
    """The opt-in small-network path runs every step of a chunk in one CTA, or in one
    thread-block cluster of 8 or 16 CTAs (autotuner site kind 14), with the state in shared
    memory, the cluster either pushing the effects or, for synapses without delays or
    weights of their own (CUBA), pulling them at the targets; the result must be the
    per-step kernels' result exactly (every delivered weight of one target variable is
    equal, so the order of the additions cannot change a sum)."""
    from brian2cuda_b200._native import B2BError
    out = {}
    forms = [(1, 0), (8, 0), (16, 0), (8, 1), (16, 1), False]
    for form in forms:
        small = form is not False
        net = gpu_factory(DT, small=small, two_launch=None if small else False)
        if case == "cobahh_delays":
            ids = models.build_cobahh(net, n=3000, p=0.05, monitor_capacity=10**6)
            G, steps = ids["P"], 300
        elif case == "cuba":
            ids = models.build_cuba(net, n=4000, dtype="float64")
            G, steps = ids["P"], 400
        else:
            rng = np.random.default_rng(5)
            n = 700
            G = net.lif_group(n, models.cuba_lif(), "float64")
            net.set_state(G, "v", rng.uniform(-60 * mV, -50 * mV, n))
            i, j = models.bernoulli_pairs(rng, n, n, 0.05)
            d = rng.integers(0, 4, size=len(i)).astype(np.int32)
            net.synapses(G, G, "v", i, j, w_scalar=0.6 * mV, delay=d)
            net.spike_monitor(G, 10**6)
            steps = 200
        net.finalize()
        assert net.run_mode == ("small" if small else "per-step")
        if small and form != (1, 0):
            try:
                net.tune_apply([{"site_kind": 14, "site_index": 0, "choice_a": form[0],
                                 "choice_b": form[1]}])
            except B2BError:
                # the pull form needs synapses without delays; 16-CTA clusters a device
                # that allows them; 8-CTA pushing clusters must always be possible
                assert form != (8, 0)
                continue
        net.run(steps)
        assert net.sync() == 0
        idx, st = net.spikes(G)
        out[form] = (idx, st, {v: net.get_state(G, v) for v in ("v", "ge", "gi", "lastspike")})
    assert len(out[False][0]) > 50
    if case == "cuba":
        assert (8, 1) in out or (16, 1) in out, "the pull form must run CUBA"
    for form in forms[:-1]:
        if form not in out:
            continue
        np.testing.assert_array_equal(out[form][0], out[False][0], err_msg=str(form))
        np.testing.assert_array_equal(out[form][1], out[False][1], err_msg=str(form))
        for v in ("v", "ge", "gi", "lastspike"):
            np.testing.assert_array_equal(out[form][2][v], out[False][2][v],
                                          err_msg=f"{form} {v}")


@pytest.mark.parametrize("inputs", [False, True])
def test_hh_stream_kernel_matches_per_step_kernel(gpu_factory, inputs):
    """A float32 HH population large enough for the streaming kernel (four neurons per
    thread, resident CTAs walking the population, warp-level spike compaction) gives the
    same spikes and state, bit for bit, as the one-neuron-per-thread kernel: the per-neuron
    arithmetic is shared.  With inputs, a PoissonInput onto ge exercises that variant."""
    n = 640_000
    out = {}
    for e in (4, 2, 1):
        net = gpu_factory(DT, seed=2)
        P = net.hh_group(n, models.cobahh_hh(), "float32")
        rng = np.random.default_rng(4)
        net.set_state(P, "v", rng.uniform(-70e-3, -40e-3, n))
        if inputs:
            net.poisson_input(P, "ge", 100, 50.0, 3e-9)
        net.spike_monitor(P, 4 * n)
        net.finalize()
        net.tune_apply([{"site_kind": 1, "site_index": 0, "choice_a": e, "choice_b": 256}])
        net.run(40)
        idx, st = net.spikes(P)
        out[e] = (idx, st, net.get_state(P, "v"), net.get_state(P, "ge"), net.get_state(P, "m"))
    assert len(out[1][0]) > 1000
    for k in range(5):
        np.testing.assert_array_equal(out[4][k], out[1][k], err_msg=str(k))
        np.testing.assert_array_equal(out[2][k], out[1][k], err_msg=f"two per thread, {k}")
