"""The Brian2 device plugin without Brian2 (CPU only): Brian2-shaped stand-in objects (the
attributes the plugin reads: equations, events, event_codes, _refractory, state arrays,
synaptic i/j/delay arrays, pathways, monitor variables) are described, lowered and run on the
oracle, and the results are written back into the stand-ins' arrays as Brian2 would hold
them; the prefs table maps brian2cuda's preference names."""
import types

import numpy as np
import pytest

from brian2cuda_b200 import device, examples
from brian2cuda_b200.lowering import Script

DT = 1e-4


class _Arr:
    """A Brian2 variable as the plugin uses it: get_value / set_value / resize."""

    def __init__(self, a):
        self.a = np.asarray(a)

    def get_value(self):
        return self.a

    def set_value(self, v):
        self.a = np.asarray(v)

    def resize(self, shape):
        self.a = np.zeros(shape, dtype=self.a.dtype)


def _group(name, n, eqs, threshold, reset, refractory, ns, init):
    g = type("NeuronGroup", (), {})()
    g.name, g.N, g.user_equations = name, n, eqs
    g.events, g.event_codes = {"spike": threshold}, {"spike": reset}
    g._refractory = refractory
    g.state_updater = types.SimpleNamespace(method_choice="exact")
    g.namespace = ns
    for k, v in init.items():
        setattr(g, k + "_", np.array(v, dtype=np.float64))
    return g


def _synapses(name, src, dst, on_pre, i, j, delay):
    s = type("Synapses", (), {})()
    s.name, s.source, s.target = name, src, dst
    s._pathways = [types.SimpleNamespace(prepost="pre", code=on_pre)]
    s.equations, s.event_driven = "", None
    s.i, s.j = np.asarray(i), np.asarray(j)
    s.delay_ = np.full(len(i), delay)
    return s


def _monitor(kind, name, source, **kw):
    m = type(kind, (), {})()
    m.name, m.source = name, source
    m.variables = {"i": _Arr(np.zeros(0, np.int32)), "t": _Arr(np.zeros(0)),
                   "count": _Arr(np.zeros(source.N, np.int64)), "N": _Arr(0),
                   "v": _Arr(np.zeros((0, 0))), "rate": _Arr(np.zeros(0))}
    for k, v in kw.items():
        setattr(m, k, v)
    return m


def _cuba_objects(n=500, seed=1):
    rng = np.random.default_rng(seed)
    ns = dict(taum=20e-3, taue=5e-3, taui=10e-3, Vt=-50e-3, Vr=-60e-3, El=-49e-3)
    P = _group("P", n, examples.CUBA_EQS, "v > Vt", "v = Vr", 5e-3, ns,
               {"v": -60e-3 + rng.random(n) * 10e-3, "ge": np.zeros(n), "gi": np.zeros(n)})
    pairs = rng.random((n, n)) < 0.05
    i, j = np.nonzero(pairs)
    ne = int(0.8 * n)
    e = i < ne
    Ce = _synapses("Ce", P, P, "ge += 1.62*mV", i[e], j[e], 0.0)
    Ci = _synapses("Ci", P, P, "gi += -9*mV", i[~e], j[~e], 0.0)
    M = _monitor("SpikeMonitor", "M", P)
    SM = _monitor("StateMonitor", "SM", P, record=np.array([0, 3, 499]),
                  record_variables=("v",), clock=types.SimpleNamespace(dt=DT))
    return [P, Ce, Ci, M, SM], (i, j, e)


def test_prefs_are_mapped():
    s = device.resolve_prefs({
        "devices.cuda_standalone.cuda_backend.gpu_id": 0,
        "devices.cuda_standalone.calc_occupancy": False,
        "devices.cuda_standalone.SM_multiplier": 2,
        "core.default_float_dtype": np.float32})
    assert s.device == 0 and s.autotune is False
    assert any("SM_multiplier" in n for n in s.notes)
    with pytest.raises(KeyError):
        device.resolve_prefs({"devices.cuda_standalone.no_such_pref": 1})
    with pytest.raises(ValueError):
        device.resolve_prefs({"devices.cuda_standalone.cuda_backend.compute_capability": 8.0})
    assert set(device.PREFS) >= {"devices.cuda_standalone.use_atomics",
                                 "devices.cuda_standalone.cuda_backend.extra_compile_args_nvcc"}


def test_register_without_brian2_is_a_no_op():
    try:
        import brian2  # noqa: F401
        pytest.skip("brian2 is installed: registration is exercised for real")
    except ImportError:
        assert device.register() is False


def test_brian2_shaped_objects_run_like_the_direct_script(oracle_factory):
    """The plugin's description of Brian2-shaped objects runs exactly like the same network
    written directly on the front end, and the monitors' records land in the objects'
    arrays."""
    objs, (i, j, e) = _cuba_objects()
    d = device.describe_objects(objs, DT)
    d.script.run(0.03)
    prog = d.script.lower()
    net = oracle_factory(DT)
    ids = prog.build(net)
    net.run(300)
    device.write_back(d, prog, net, ids, DT, objs)
    P, Ce, Ci, M, SM = objs
    # the same network written directly
    s = Script(dt=DT, namespace=dict(taum=20e-3, taue=5e-3, taui=10e-3, Vt=-50e-3,
                                     Vr=-60e-3, El=-49e-3))
    G = s.NeuronGroup(500, examples.CUBA_EQS, threshold="v > Vt", reset="v = Vr",
                      refractory=5e-3, method="exact")
    rng = np.random.default_rng(1)
    G.v = -60e-3 + rng.random(500) * 10e-3
    for sy, sel, code in ((None, e, "ge += 1.62*mV"), (None, ~e, "gi += -9*mV")):
        S = s.Synapses(G, G, on_pre=code)
        S.connect(i=i[sel], j=j[sel])
        S.delay = 0.0
    s.SpikeMonitor(G, name="m")
    s.run(0.03)
    ref = s.lower().execute(oracle_factory(DT))["m"]
    got_i = M.variables["i"].get_value()
    got_t = M.variables["t"].get_value()
    assert len(got_i) > 50
    np.testing.assert_array_equal(got_i, ref[0])
    np.testing.assert_allclose(got_t, ref[1] * DT, rtol=0, atol=1e-15)
    assert M.variables["count"].get_value().sum() == len(got_i)
    v = SM.variables["v"].get_value()
    assert v.shape == (300, 3) and np.all(v < 0)
    # the final state went back into the group's array
    np.testing.assert_array_equal(P.v_, net.get_state(ids["P"], "v"))
