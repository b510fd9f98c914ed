"""The Brian2 device plugin: `set_device('cuda_standalone')` runs a Brian2 network on libb2b.

brian2cuda registers a standalone device under the name 'cuda_standalone'
(`brian2cuda/device.py:71` class, `:2002-2004` registration) that generates, compiles and
runs a CUDA project at `network_run` (`device.py:1508-1765`).  This plugin keeps that name,
the `set_device` / `run` / prefs API and the result arrays Brian2 reads, but runs the network
on the hand-written kernels instead of generated ones:

  * everything before `run()` happens in Brian2's runtime: `connect()` creates the synapses,
    assignments such as `G.v = 'El + rand()*mV'` evaluate, so the network's state is plain
    arrays when the run starts;
  * `network_run` describes the network's objects (`describe_objects`: NeuronGroup with its
    equations, threshold, reset and refractoriness; PoissonGroup; SpikeGeneratorGroup;
    Synapses with their connectivity, delays, weights and on_pre / on_post code; PoissonInput;
    SpikeMonitor, StateMonitor, PopulationRateMonitor) as a `lowering.Script`, lowers it
    onto libb2b (hand-written kernels, or generated code for other models) and runs it;
    later runs of the same network continue on the GPU, with the state re-uploaded from
    Brian2's arrays first (assignments between runs take effect);
  * afterwards the state variables and the monitors' records are written back into Brian2's
    arrays, so `mon.i`, `mon.t`, `statemon.v`, `G.v` read as after any Brian2 run.
Anything outside the lowered forms raises `lowering.ModelUnsupported` with the reason.

Brian2 (2.10.1, the reference's pin) is not installed where this was built, so the class that
subclasses Brian2's RuntimeDevice (`make_device`) is not exercised here; the conversion
(`describe_objects`) works on any objects with Brian2's attributes and is tested with
stand-ins, and the prefs table (`resolve_prefs`) is plain data.
"""
from __future__ import annotations

import warnings
from dataclasses import dataclass, field

import numpy as np

from .lowering import ModelUnsupported, Script, Subgroup

# ---- prefs: devices.cuda_standalone.* (brian2cuda/cuda_prefs.py:39-249) -------------------------
# name -> (default, what it does here)
PREFS = {
    "devices.cuda_standalone.SM_multiplier": (1, "no effect: the autotuner sizes the grids"),
    "devices.cuda_standalone.parallel_blocks": (1, "no effect: one delivery launch per step "
                                                   "covers all targets"),
    "devices.cuda_standalone.launch_bounds": (False, "no effect: kernels carry their own"),
    "devices.cuda_standalone.syn_launch_bounds": (False, "no effect"),
    "devices.cuda_standalone.calc_occupancy": (True, "autotune: True runs b2b_autotune "
                                                     "before the first run"),
    "devices.cuda_standalone.extra_threshold_kernel": (True, "no effect: threshold, reset and "
                                                             "compaction are fused"),
    "devices.cuda_standalone.random_number_generator_type": (
        "CURAND_RNG_PSEUDO_DEFAULT", "CURAND_RNG_PSEUDO_DEFAULT / _PHILOX4_32_10 accepted (the "
                                     "net's generator is Philox-4x32-10); others warn"),
    "devices.cuda_standalone.random_number_generator_ordering": (False, "no effect"),
    "devices.cuda_standalone.push_synapse_bundles": (True, "no effect: no push; the spike-"
                                                           "history ring replaces the queue"),
    "devices.cuda_standalone.threads_per_synapse_bundle": (
        "{max}", "no effect: lanes per work item come from the autotuner"),
    "devices.cuda_standalone.bundle_threads_warp_multiple": (False, "no effect"),
    "devices.cuda_standalone.no_pre_references": (False, "no effect"),
    "devices.cuda_standalone.no_post_references": (False, "no effect"),
    "devices.cuda_standalone.default_functions_integral_convertion": (
        np.float64, "no effect: generated code keeps the group's dtype"),
    "devices.cuda_standalone.use_atomics": (True, "always atomics (the only effect mode)"),
    "devices.cuda_standalone.profile_statemonitor_copy_to_host": (None, "no effect"),
    "devices.cuda_standalone.cuda_backend.gpu_heap_size": (128, "no effect: nothing allocates "
                                                                "on the device heap"),
    "devices.cuda_standalone.cuda_backend.detect_gpus": (True, "no effect"),
    "devices.cuda_standalone.cuda_backend.gpu_id": (None, "device ordinal of the net"),
    "devices.cuda_standalone.cuda_backend.extra_compile_args_nvcc": (
        ["-w", "-use_fast_math"], "no effect: generated models compile with the library's "
                                  "flags (no fast math)"),
    "devices.cuda_standalone.cuda_backend.compute_capability": (None, "must be 10.0 (sm_100a) "
                                                                      "when set"),
    "devices.cuda_standalone.cuda_backend.detect_cuda": (True, "no effect"),
    "devices.cuda_standalone.cuda_backend.cuda_path": (None, "no effect: CUDA_HOME / "
                                                             "/usr/local/cuda"),
    "devices.cuda_standalone.cuda_backend.cuda_runtime_version": (None, "no effect"),
    "devices.cuda_standalone.cuda_backend.device_query_path": (None, "no effect"),
}


@dataclass
class Settings:
    device: int = 0
    autotune: bool = True
    notes: list[str] = field(default_factory=list)


def resolve_prefs(values: dict) -> Settings:
    """Settings from pref values (full names, as in Brian2's prefs).  Unknown names under
    devices.cuda_standalone raise KeyError; accepted names without an effect are noted."""
    s = Settings()
    for name, val in (values or {}).items():
        if not name.startswith("devices.cuda_standalone"):
            continue
        if name not in PREFS:
            raise KeyError(f"unknown preference {name}")
        default, _ = PREFS[name]
        if name.endswith(".gpu_id") and val is not None:
            s.device = int(val)
        elif name.endswith(".calc_occupancy"):
            s.autotune = bool(val)
        elif name.endswith(".random_number_generator_type") and val not in (
                "CURAND_RNG_PSEUDO_DEFAULT", "CURAND_RNG_PSEUDO_PHILOX4_32_10"):
            warnings.warn(f"{name}={val}: the net's cuRAND generator is Philox-4x32-10")
        elif name.endswith(".compute_capability") and val not in (None, 10.0, 10, "10.0"):
            raise ValueError(f"{name}={val}: this backend runs on sm_100a only")
        elif name.endswith(".use_atomics") and not val:
            s.notes.append("use_atomics=False ignored: effects are applied with atomics")
        elif not _equal(val, default):
            s.notes.append(f"{name}={val!r} has no effect ({PREFS[name][1]})")
    return s


def _equal(a, b) -> bool:
    try:
        return bool(a == b)
    except Exception:   # noqa: BLE001
        return False


# ---- Brian2 objects -> plain descriptions ------------------------------------------------------
def _si(q) -> float:
    """A Brian2 Quantity (or a number) in SI base units."""
    return float(np.asarray(q, dtype=np.float64))


def _namespace(obj, run_namespace: dict) -> dict:
    ns = {}
    for src in (run_namespace or {}, getattr(obj, "namespace", None) or {}):
        for k, v in src.items():
            try:
                ns[k] = _si(v)
            except (TypeError, ValueError):
                if isinstance(v, (int, float)):
                    ns[k] = float(v)
    return ns


def _kind(obj) -> str:
    name = type(obj).__name__
    for base in type(obj).__mro__:
        if base.__name__ in ("PoissonGroup", "SpikeGeneratorGroup", "NeuronGroup", "Synapses",
                             "SpikeMonitor", "StateMonitor", "PopulationRateMonitor",
                             "PoissonInput", "Subgroup"):
            return base.__name__
    return name


def _values(obj, var: str) -> np.ndarray:
    """Current values of a variable without units (Brian2's `var_` accessor)."""
    return np.asarray(getattr(obj, var + "_")[:], dtype=np.float64)


@dataclass
class Described:
    script: Script
    groups: dict              # Brian2 object id -> GroupDesc
    synapses: dict            # Brian2 object id -> SynapsesDesc
    monitors: dict            # Brian2 object id -> (monitor description, Brian2 object)


def describe_objects(objects, dt: float, namespace: dict | None = None,
                     dtype: str = "float64", seed: int = 0) -> Described:
    """Plain descriptions of Brian2 objects (in `Network.sorted_objects` order) for the
    lowering, reading the attributes Brian2's objects expose: equations, threshold and reset
    code, refractoriness, state values, synaptic connectivity and code, monitor sources."""
    s = Script(dt=dt, seed=seed, dtype=dtype)
    groups: dict = {}
    syns: dict = {}
    mons: dict = {}

    def source_of(o):
        if _kind(o) == "Subgroup":
            parent = groups[id(o.source)]
            return Subgroup(parent, int(o.start), int(o.stop))
        return groups[id(o)]
    for obj in objects:
        k = _kind(obj)
        if k == "NeuronGroup":
            ns = _namespace(obj, namespace)
            ref = getattr(obj, "_refractory", False)
            refractory = 0.0 if ref is False or ref is None else (
                ref if isinstance(ref, str) else _si(ref))
            thr = getattr(obj, "events", {}).get("spike")
            rst = getattr(obj, "event_codes", {}).get("spike")
            method = getattr(getattr(obj, "state_updater", None), "method_choice", None)
            if isinstance(method, (list, tuple)):
                method = method[0] if len(method) == 1 else None
            g = s.NeuronGroup(int(obj.N), str(obj.user_equations), threshold=thr, reset=rst,
                              refractory=refractory, method=method, namespace=ns,
                              name=obj.name)
            for var in _state_names(obj):
                g.init[var] = _values(obj, var)
            groups[id(obj)] = g
        elif k == "PoissonGroup":
            rates = obj.rates
            if isinstance(rates, str):
                raise ModelUnsupported(f"{obj.name}: rates as an expression")
            r = np.asarray(rates, dtype=np.float64)
            if r.size != 1:
                raise ModelUnsupported(f"{obj.name}: per-neuron rates")
            groups[id(obj)] = s.PoissonGroup(int(obj.N), float(r.reshape(-1)[0]),
                                              name=obj.name)
        elif k == "SpikeGeneratorGroup":
            groups[id(obj)] = s.SpikeGeneratorGroup(
                int(obj.N), np.asarray(obj._neuron_index[:], np.int32),
                np.asarray(obj._spike_time[:], np.float64), period=_si(obj.period),
                name=obj.name)
        elif k == "Synapses":
            ns = _namespace(obj, namespace)
            src, dst = source_of(obj.source), source_of(obj.target)
            on_pre = on_post = ""
            for p in getattr(obj, "_pathways", []):
                if p.prepost == "pre":
                    on_pre = p.code
                elif p.prepost == "post":
                    on_post = p.code
            # Brian2 keeps the event-driven equations apart from the others
            parts = [str(e) for e in (getattr(obj, "equations", None),
                                      getattr(obj, "event_driven", None)) if e]
            model = "\n".join(parts)
            d = s.Synapses(src, dst, model=model, on_pre=on_pre, on_post=on_post,
                           namespace=ns, name=obj.name)
            i = np.asarray(obj.i[:], np.int32)
            j = np.asarray(obj.j[:], np.int32)
            d.connect(i=i, j=j)
            delay = np.asarray(obj.delay_[:], np.float64) if len(i) else np.zeros(0)
            d.delay = (float(delay[0]) if delay.size and np.all(delay == delay[0])
                       else delay)
            if model.strip():
                from .equations import parse_equations
                for var in parse_equations(model).params:
                    if var not in ("lastupdate", "delay"):
                        d.d["init"][var] = _values(obj, var)
            syns[id(obj)] = d
        elif k == "PoissonInput":
            tgt = groups[id(obj.target)]
            s.PoissonInput(tgt, obj.target_var, int(obj.N), _si(obj.rate),
                           obj.weight if isinstance(obj.weight, str) else _si(obj.weight),
                           name=obj.name)
        elif k == "SpikeMonitor":
            m = s.SpikeMonitor(source_of(obj.source), name=obj.name)
            mons[id(obj)] = (m, obj)
        elif k == "StateMonitor":
            rec = obj.record
            every = max(1, int(round(_si(obj.clock.dt) / dt)))
            m = s.StateMonitor(source_of(obj.source), tuple(obj.record_variables),
                               record=np.asarray(rec, np.int64), dt=every * dt, name=obj.name)
            mons[id(obj)] = (m, obj)
        elif k == "PopulationRateMonitor":
            m = s.PopulationRateMonitor(source_of(obj.source), name=obj.name)
            mons[id(obj)] = (m, obj)
        elif k in ("Subgroup",):
            continue
        else:
            raise ModelUnsupported(f"{getattr(obj, 'name', obj)}: {k} is not supported by "
                                   "this backend")
    return Described(s, groups, syns, mons)


def _state_names(obj) -> list[str]:
    eqs = getattr(obj, "user_equations", None)
    names = getattr(eqs, "diff_eq_names", None)
    if names is not None:
        return list(names)
    from .equations import parse_equations
    return parse_equations(str(eqs)).state


# ---- results back into Brian2's arrays ----------------------------------------------------------
def write_back(described: Described, prog, backend, ids, dt: float, objects) -> None:
    """Final state of every NeuronGroup and the monitors' records into the Brian2 objects
    (their arrays, resized as Brian2's dynamic arrays are)."""
    by_id = {id(o): o for o in objects}
    for oid, g in described.groups.items():
        obj = by_id.get(oid)
        info = prog.groups.get(g.name)
        if obj is None or _kind(obj) != "NeuronGroup" or info is None:
            continue
        for var, slot in info["slots"].items():
            getattr(obj, var + "_")[:] = backend.get_state(ids[g.name], slot)
    res = prog.collect(backend, ids)
    for oid, (m, obj) in described.monitors.items():
        r = res[m.name]
        if m.kind == "spike":
            idx, st = r
            _set_dynamic(obj, "i", idx.astype(np.int32))
            _set_dynamic(obj, "t", st.astype(np.float64) * dt)
            n = m.source.N if hasattr(m.source, "N") else len(obj.source)
            obj.variables["count"].get_value()[:] = np.bincount(idx, minlength=n)[:n]
            obj.variables["N"].set_value(len(idx))
        elif m.kind == "rate":
            st, counts = r
            n = m.source.N
            _set_dynamic(obj, "t", st.astype(np.float64) * dt)
            _set_dynamic(obj, "rate", counts.astype(np.float64) / (n * dt))
        else:
            first = True
            for v, (st, vals) in r.items():
                if first:
                    _set_dynamic(obj, "t", st.astype(np.float64) * dt)
                    first = False
                _set_dynamic(obj, v, np.asarray(vals, np.float64))


def _set_dynamic(obj, name, values):
    var = obj.variables[name]
    var.resize(values.shape if values.ndim > 1 else len(values))
    var.get_value()[...] = values


# ---- the device ----------------------------------------------------------------------------------
def make_device():
    """The Brian2 device class (needs brian2): a RuntimeDevice whose network_run runs the
    network on libb2b."""
    from brian2.core.functions import DEFAULT_FUNCTIONS  # noqa: F401 - brian2 is required
    from brian2.core.namespace import get_local_namespace
    from brian2.core.preferences import prefs
    from brian2.devices.device import RuntimeDevice

    from .network import Network

    class CUDAStandaloneDevice(RuntimeDevice):
        """Brian2 device 'cuda_standalone' backed by libb2b (brian2cuda/device.py:71)."""

        def __init__(self):
            super().__init__()
            self.build_options = {}
            self._runs = {}                  # id(Network) -> (described, program, net, ids)

        def activate(self, build_on_run=True, **kwargs):
            super().activate()
            self.build_options.update(kwargs)

        def network_run(self, net, duration, report=None, report_period=None,
                        namespace=None, profile=False, level=0, **kwds):
            if namespace is None:
                namespace = get_local_namespace(level=level + 2)
            objects = net.sorted_objects
            clocks = {o.clock for o in objects}
            if len({round(_si(c.dt), 15) for c in clocks}) > 1:
                raise ModelUnsupported("groups on different clocks")
            dt = _si(next(iter(clocks)).dt)
            settings = resolve_prefs({k: prefs[k] for k in PREFS if k in prefs})
            steps = int(round(_si(duration) / dt))
            key = id(net)
            if key not in self._runs:
                net.before_run(namespace)
                dtype = str(np.dtype(prefs["core.default_float_dtype"]))
                d = describe_objects(objects, dt, namespace, dtype=dtype,
                                     seed=int(self.build_options.get("seed", 0)))
                prog = d.script.lower()
                backend = Network(dt, seed=d.script.seed, device=settings.device)
                ids = prog.build(backend)
                if settings.autotune and steps >= 200:
                    backend.autotune(trial_steps=min(300, steps))
                self._runs[key] = (d, prog, backend, ids)
            else:
                d, prog, backend, ids = self._runs[key]
                # assignments since the last run take effect
                for oid, g in d.groups.items():
                    obj = next((o for o in objects if id(o) == oid), None)
                    info = prog.groups.get(g.name)
                    if obj is None or _kind(obj) != "NeuronGroup":
                        continue
                    for var, slot in info["slots"].items():
                        backend.set_state(ids[g.name], slot, _values(obj, var))
            backend.run(steps)
            status = backend.sync()
            if status != 0:
                raise RuntimeError(f"device status {status} after the run")
            write_back(d, prog, backend, ids, dt, objects)
            net.t_ = _si(net.t) + steps * dt

        def network_store(self, *args, **kwds):
            raise NotImplementedError("store/restore: use brian2cuda_b200.Network.store")

        def network_restore(self, *args, **kwds):
            raise NotImplementedError("store/restore: use brian2cuda_b200.Network.restore")

    return CUDAStandaloneDevice


def register() -> bool:
    """Registers the device as all_devices['cuda_standalone'] when brian2 can be imported;
    returns whether it did."""
    try:
        from brian2.devices.device import all_devices
    except ImportError:
        return False
    all_devices["cuda_standalone"] = make_device()()
    return True
