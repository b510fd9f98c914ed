"""Lowering of Brian2-shaped network descriptions onto the b2b C ABI.

brian2cuda's device turns every Brian2 object into code objects and generated kernels
(`brian2cuda/device.py:234-421` code_object, `cuda_generator.py:281-461` statements); here
the objects are described plainly (a `Script` records NeuronGroup, PoissonGroup,
SpikeGeneratorGroup, Synapses, PoissonInput, SpikeMonitor, StateMonitor and
PopulationRateMonitor with their model strings, namespaces, initial values and runs) and
lowered onto the hand-written kernels:

  * NeuronGroup with method 'exact' whose equations are the linear integrate-and-fire system
    -> b2b_group_lif; method 'exponential_euler' with the conductance-based Hodgkin-Huxley
    system -> b2b_group_hh (recognize.py decides, from the parsed equations); any other model
    -> a generated model (codegen.py) when one can be generated, else ModelUnsupported;
  * Synapses whose on_pre is `x_post += c` (c a constant or a synaptic weight) -> additive
    projections; the event-driven additive STDP rule (traces Apre/Apost decaying
    exponentially, `w = clip(w + A, wmin, wmax)`) -> b2b STDP projections; connect(p=...) with
    constant or uniform-integer delays -> connectivity generated on the GPU (Philox);
  * monitors -> the device monitors; PoissonInput -> b2b_poisson_input.

The same `Program` runs against the GPU `Network` or the CPU oracle (`OracleNet`, which has
the same methods), so a script is checked against the oracle by lowering it twice.
`Program.emit_c` writes the equivalent C program that calls libb2b through include/b2b.h
(the role of the generated main.cu / network.cu, `templates/main.cu:49-104`).
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

import numpy as np

from . import equations as E
from . import recognize as R
from .network import STDP, spike_steps


class ModelUnsupported(ValueError):
    """A Brian2 construct outside what this backend lowers."""


# ---- descriptions ---------------------------------------------------------------------------
@dataclass
class UniformDelaySteps:
    """Per-synapse delays drawn uniformly from the integers [lo, hi] (steps), as the GPU
    connectivity generator draws them."""
    lo: int
    hi: int


class _Described:
    def __init__(self, script, name):
        object.__setattr__(self, "script", script)
        object.__setattr__(self, "name", name)


class GroupDesc(_Described):
    """NeuronGroup / PoissonGroup / SpikeGeneratorGroup; attribute assignment records an
    initial value (a number, an array of N values or a Brian2 expression string)."""

    def __init__(self, script, name, kind, N, **kw):
        super().__init__(script, name)
        object.__setattr__(self, "kind", kind)
        object.__setattr__(self, "N", int(N))
        object.__setattr__(self, "spec", kw)
        object.__setattr__(self, "init", {})

    def __setattr__(self, key, value):
        self.init[key] = value

    def __getitem__(self, sl):
        lo, hi, step = sl.indices(self.N)
        if step != 1:
            raise ModelUnsupported("subgroups must be contiguous")
        return Subgroup(self, lo, hi)

    def __len__(self):
        return self.N


@dataclass
class Subgroup:
    group: GroupDesc
    lo: int
    hi: int

    @property
    def N(self):
        return self.hi - self.lo


class SynapsesDesc(_Described):
    def __init__(self, script, name, source, target, model, on_pre, on_post, delay, namespace):
        super().__init__(script, name)
        d = dict(source=source, target=target, model=model or "", on_pre=on_pre or "",
                 on_post=on_post or "", delay=delay, namespace=dict(namespace or {}),
                 connect=None, init={})
        object.__setattr__(self, "d", d)

    def connect(self, condition: str | None = None, p: float = 1.0, i=None, j=None):
        """Brian2's connect: all pairs (optionally `i<K` / `i>=K`), each with probability p;
        or explicit i, j arrays."""
        self.d["connect"] = {"condition": condition, "p": float(p),
                             "i": None if i is None else np.asarray(i, np.int32),
                             "j": None if j is None else np.asarray(j, np.int32)}

    def __setattr__(self, key, value):
        if key == "delay":
            self.d["delay"] = value
        else:
            self.d["init"][key] = value


@dataclass
class MonitorDesc:
    kind: str                       # "spike", "state", "rate"
    source: object
    variables: tuple = ()
    record: object = True
    every: int = 1
    capacity: int | None = None
    name: str = ""


@dataclass
class PoissonInputDesc:
    target: object
    var: str
    N: int
    rate: float
    weight: object
    name: str = ""


class Script:
    """A network described the way a Brian2 script builds it (units in SI).  Objects are
    recorded in creation order; `run(duration)` appends a run.  `lower()` gives the Program
    that builds and runs it on a backend."""

    def __init__(self, dt: float = 1e-4, seed: int = 0, dtype: str = "float64",
                 namespace: dict | None = None, generated_only: bool = False):
        """generated_only: integrate every NeuronGroup with generated code, also models the
        hand-written kernels would take (to compare the two)."""
        self.dt = float(dt)
        self.seed = int(seed)
        self.dtype = dtype
        self.namespace = dict(namespace or {})
        self.generated_only = bool(generated_only)
        self.objects: list = []
        self.runs: list[int] = []
        self._n = 0

    def _name(self, base):
        self._n += 1
        return f"{base}_{self._n}"

    def NeuronGroup(self, N, model, threshold=None, reset=None, refractory=0.0, method=None,
                    namespace=None, dtype=None, name=None):
        g = GroupDesc(self, name or self._name("neurongroup"), "neuron", N, model=model,
                      threshold=threshold, reset=reset, refractory=refractory, method=method,
                      namespace=dict(namespace or {}), dtype=dtype or self.dtype)
        self.objects.append(g)
        return g

    def PoissonGroup(self, N, rates, dtype=None, name=None):
        g = GroupDesc(self, name or self._name("poissongroup"), "poisson", N, rates=rates,
                      dtype=dtype or self.dtype)
        self.objects.append(g)
        return g

    def SpikeGeneratorGroup(self, N, indices, times, period=0.0, name=None):
        g = GroupDesc(self, name or self._name("spikegeneratorgroup"), "spikegen", N,
                      indices=np.asarray(indices, np.int32),
                      times=np.asarray(times, np.float64), period=float(period))
        self.objects.append(g)
        return g

    def Synapses(self, source, target, model="", on_pre="", on_post="", delay=None,
                 namespace=None, name=None):
        s = SynapsesDesc(self, name or self._name("synapses"), source, target, model, on_pre,
                         on_post, delay, namespace)
        self.objects.append(s)
        return s

    def SpikeMonitor(self, source, capacity=None, name=None):
        m = MonitorDesc("spike", source, capacity=capacity, name=name or self._name("spikemon"))
        self.objects.append(m)
        return m

    def StateMonitor(self, source, variables, record=True, dt=None, capacity=None, name=None):
        every = 1 if dt is None else max(1, int(round(float(dt) / self.dt)))
        vs = (variables,) if isinstance(variables, str) else tuple(variables)
        m = MonitorDesc("state", source, variables=vs, record=record, every=every,
                        capacity=capacity, name=name or self._name("statemon"))
        self.objects.append(m)
        return m

    def PopulationRateMonitor(self, source, capacity=None, name=None):
        m = MonitorDesc("rate", source, capacity=capacity, name=name or self._name("ratemon"))
        self.objects.append(m)
        return m

    def PoissonInput(self, target, target_var, N, rate, weight, name=None):
        p = PoissonInputDesc(target, target_var, int(N), float(rate), weight,
                             name or self._name("poissoninput"))
        self.objects.append(p)
        return p

    def run(self, duration: float):
        self.runs.append(int(round(float(duration) / self.dt)))

    def lower(self) -> "Program":
        return lower(self)


# ---- statements -------------------------------------------------------------------------------
_STMT = re.compile(r"^\s*([A-Za-z_]\w*)\s*(\+=|-=|=)\s*(.+?)\s*$")


def statements(code: str) -> list[tuple[str, str, str]]:
    """(target, operator, expression) of each `x op expr` line or ;-separated statement."""
    out = []
    for part in re.split(r"[;\n]", code or ""):
        part = part.split("#", 1)[0].strip()
        if not part:
            continue
        m = _STMT.match(part)
        if not m:
            raise ModelUnsupported(f"cannot lower the statement {part!r}")
        out.append((m.group(1), m.group(2), m.group(3)))
    return out


def _strip_post(name: str) -> str:
    return name[:-5] if name.endswith("_post") else name


def _ns(script, *extra):
    ns = dict(script.namespace)
    for e in extra:
        ns.update(e or {})
    return ns


_OTHER = "*"    # a threshold or reset the hand-written kernels do not take (generated code)


def _threshold(expr: str | None, ns) -> tuple[str, float | None] | None:
    """(var, value) for `var > value`; (_OTHER, None) for any other condition."""
    if expr is None:
        return None
    m = re.match(r"^\s*([A-Za-z_]\w*)\s*>\s*(.+?)\s*$", expr)
    if m:
        try:
            return m.group(1), E.value_of(m.group(2), ns)
        except E.EquationError:
            pass
    return _OTHER, None


def _reset(expr: str | None, ns) -> tuple[str, float | None] | None:
    """(var, value) for `var = value`; (_OTHER, None) for other statements."""
    if not expr:
        return None
    st = statements(expr)
    if len(st) == 1 and st[0][1] == "=":
        try:
            return st[0][0], E.value_of(st[0][2], ns)
        except E.EquationError:
            pass
    return _OTHER, None


def _seconds(v, ns) -> float:
    if isinstance(v, str):
        return E.value_of(v, ns)
    return float(v or 0.0)


def evaluate_init(value, n: int, ns: dict, rng: np.random.Generator) -> np.ndarray:
    """An initial value: a number, n values, or a Brian2 expression in i, N, rand(), randn()
    and the namespace (each rand()/randn() call draws n fresh values, left to right)."""
    if isinstance(value, str):
        import sympy as sp
        syms: dict = {}
        ex = E.to_sympy(value, syms)
        draws = []

        def draw(fn):
            a = rng.random(n) if fn is E.RAND else rng.standard_normal(n)
            s = sp.Symbol(f"_draw{len(draws)}")
            draws.append((s, a))
            return s
        ex = ex.replace(lambda e: getattr(e, "func", None) in (E.RAND, E.RANDN),
                        lambda e: draw(e.func))
        nsn = E.numeric_namespace(ns)
        rep = {s: sp.Float(nsn[nm], 17) for nm, s in syms.items() if nm in nsn}
        ex = ex.xreplace(rep)
        args = {"i": np.arange(n, dtype=np.float64), "N": float(n)}
        names = [str(s) for s in ex.free_symbols]
        vals = []
        for nm in names:
            if nm in args:
                vals.append(args[nm])
            else:
                hit = [a for s, a in draws if str(s) == nm]
                if not hit:
                    raise ModelUnsupported(f"initial value {value!r}: unknown name {nm}")
                vals.append(hit[0])
        f = sp.lambdify([sp.Symbol(nm) for nm in names], ex, "numpy")
        return np.broadcast_to(np.asarray(f(*vals), dtype=np.float64), (n,)).copy()
    a = np.asarray(value, dtype=np.float64)
    return np.broadcast_to(a, (n,)).copy()


# ---- the program -----------------------------------------------------------------------------
@dataclass
class Op:
    method: str
    args: tuple
    kwargs: dict = field(default_factory=dict)
    key: str | None = None          # the id the call returns is stored under this name


@dataclass
class Program:
    """A sequence of calls on the Network interface (GPU or oracle), then runs."""
    dt: float
    seed: int
    ops: list[Op]
    runs: list[int]
    groups: dict                     # group name -> (kind, N, slot map, dtype)
    monitors: dict                   # monitor name -> description
    notes: list[str] = field(default_factory=list)

    def build(self, backend) -> dict:
        ids: dict = {}

        def res(a):
            if isinstance(a, _Ref):
                return ids[a.key]
            return a
        for op in self.ops:
            r = getattr(backend, op.method)(*[res(a) for a in op.args],
                                            **{k: res(v) for k, v in op.kwargs.items()})
            if op.key:
                ids[op.key] = r
        backend.finalize()
        return ids

    def execute(self, backend) -> dict:
        """Builds the network on `backend`, runs every run() and returns the monitors'
        records: spike monitors (indices, steps), state monitors (steps, values per
        variable), rate monitors (steps, counts)."""
        ids = self.build(backend)
        for steps in self.runs:
            backend.run(steps)
        return self.collect(backend, ids)

    def collect(self, backend, ids) -> dict:
        out = {}
        for name, m in self.monitors.items():
            if m["kind"] == "spike":
                out[name] = backend.spikes(ids[m["group"]], m["sub"])
            elif m["kind"] == "state":
                out[name] = {v: backend.state_values(ids[f"{name}:{v}"]) for v in m["vars"]}
            else:
                out[name] = backend.rate_counts(ids[name])
        return out


@dataclass(frozen=True)
class _Ref:
    key: str


def _group_of(src) -> tuple[GroupDesc, int, int]:
    if isinstance(src, Subgroup):
        return src.group, src.lo, src.hi
    return src, 0, src.N


def lower(script: Script) -> Program:
    ops: list[Op] = []
    groups: dict = {}
    monitors: dict = {}
    notes: list[str] = []
    rng = np.random.default_rng(script.seed)
    total_steps = max(1, sum(script.runs))
    syn_count = 0
    for obj in script.objects:
        if isinstance(obj, GroupDesc):
            _lower_group(script, obj, ops, groups, rng, notes)
        elif isinstance(obj, SynapsesDesc):
            syn_count += 1
            _lower_synapses(script, obj, ops, groups, rng, syn_count)
        elif isinstance(obj, PoissonInputDesc):
            g, lo, hi = _group_of(obj.target)
            if (lo, hi) != (0, g.N):
                raise ModelUnsupported("PoissonInput onto a subgroup")
            slot = groups[g.name]["slots"].get(obj.var)
            if slot not in ("v", "ge", "gi"):
                raise ModelUnsupported(f"PoissonInput onto {obj.var!r}")
            w = _seconds(obj.weight, _ns(script, g.spec.get("namespace")))
            ops.append(Op("poisson_input", (_Ref(g.name), slot, obj.N, obj.rate, w),
                          key=obj.name))
        elif isinstance(obj, MonitorDesc):
            g, lo, hi = _group_of(obj.source)
            info = groups[g.name]
            if obj.kind == "spike":
                if not info.get("spike_monitor"):
                    rate_guess = 200.0
                    cap = obj.capacity or int(g.N * total_steps * script.dt * rate_guess) + 10_000
                    ops.append(Op("spike_monitor", (_Ref(g.name), cap)))
                    info["spike_monitor"] = True
                monitors[obj.name] = {"kind": "spike", "group": g.name,
                                      "sub": None if (lo, hi) == (0, g.N) else (lo, hi)}
            elif obj.kind == "state":
                if obj.record is True:
                    idx = np.arange(lo, hi, dtype=np.int64)
                else:
                    idx = np.asarray(obj.record, dtype=np.int64).reshape(-1) + lo
                cap = obj.capacity or total_steps // obj.every + 1
                for v in obj.variables:
                    slot = info["slots"].get(v, v)
                    ops.append(Op("state_monitor", (_Ref(g.name), slot, idx),
                                  {"every": obj.every, "capacity": cap},
                                  key=f"{obj.name}:{v}"))
                monitors[obj.name] = {"kind": "state", "group": g.name,
                                      "vars": list(obj.variables)}
            else:
                if (lo, hi) != (0, g.N):
                    raise ModelUnsupported("PopulationRateMonitor of a subgroup")
                ops.append(Op("rate_monitor", (_Ref(g.name),),
                              {"capacity": obj.capacity or total_steps + 1}, key=obj.name))
                monitors[obj.name] = {"kind": "rate", "group": g.name}
    return Program(script.dt, script.seed, ops, list(script.runs), groups, monitors, notes)


def _lower_group(script, g: GroupDesc, ops, groups, rng, notes):
    sp_ = g.spec
    if g.kind == "poisson":
        rate = _seconds(sp_["rates"], script.namespace)
        ops.append(Op("poisson_group", (g.N, rate, sp_["dtype"]), key=g.name))
        groups[g.name] = {"kind": "poisson", "N": g.N, "slots": {}, "dtype": sp_["dtype"]}
        return
    if g.kind == "spikegen":
        steps = spike_steps(sp_["times"], script.dt)
        period = int(round(sp_["period"] / script.dt)) if sp_["period"] else 0
        ops.append(Op("spikegen_group", (g.N, sp_["indices"], steps), {"period": period},
                      key=g.name))
        groups[g.name] = {"kind": "spikegen", "N": g.N, "slots": {}}
        return
    ns = _ns(script, sp_["namespace"])
    model = E.parse_equations(sp_["model"])
    res = E.resolve(model, ns)
    thr = _threshold(sp_["threshold"], ns)
    rst = _reset(sp_["reset"], ns)
    refractory = _seconds(sp_["refractory"], ns)
    method = sp_["method"]
    dtype = sp_["dtype"]
    vname = thr[0] if thr else (rst[0] if rst else (res.state[0] if res.state else None))
    if thr and thr[0] == _OTHER or rst and rst[0] == _OTHER or script.generated_only:
        vname = None         # neither hand-written kernel takes this threshold / reset
    lowered = None
    if method in (None, "exact", "linear"):
        m = R.match_lif(res, vname, ns) if vname else None
        if m is not None and (rst is None or rst[0] == vname):
            unl = vname in res.unless_refractory
            others_unl = res.unless_refractory - {vname}
            if not others_unl:
                prm = R.lif_from(m, thr[1] if thr else None, rst[1] if rst else None,
                                 refractory, unl)
                ops.append(Op("lif_group", (g.N, prm, dtype), key=g.name))
                lowered = {"kind": "lif", "N": g.N, "slots": m["slots"]}
    if lowered is None and method in (None, "exponential_euler"):
        m = R.match_cobahh(res, vname or "v", ns) if vname else None
        if m is not None and rst is None and thr is not None and thr[0] == vname and \
                not res.unless_refractory:
            ops.append(Op("hh_group", (g.N, R.hh_from(m, thr[1], refractory), dtype),
                          key=g.name))
            lowered = {"kind": "hh", "N": g.N, "slots": m["slots"]}
    if lowered is None:
        from . import codegen
        lowered = codegen.lower_model(script, g, model, res, thr, rst, refractory, method,
                                      dtype, ops)
    lowered["dtype"] = dtype
    groups[g.name] = lowered
    for var, value in g.init.items():
        slot = lowered["slots"].get(var)
        if slot is None:
            if var in ("lastspike", "not_refractory"):
                slot = var
            else:
                raise ModelUnsupported(f"{g.name}.{var}: not a state variable")
        ops.append(Op("set_state", (_Ref(g.name), slot, evaluate_init(value, g.N, ns, rng))))


def _stdp_rule(model: E.Model, ns, pre, post) -> tuple[STDP, dict]:
    """The event-driven additive STDP rule: returns the rule and the synaptic variables'
    roles (w, Apre, Apost), or raises ModelUnsupported."""
    traces = {e.name: e for e in model.eqs if e.kind == "diff"}
    if any("event-driven" not in e.flags for e in traces.values()) or len(traces) != 2:
        raise ModelUnsupported("plastic Synapses: only two event-driven traces are lowered")
    taus = {}
    for nm, e in traces.items():
        res = E.resolve(E.Model([e]), ns)
        try:
            A, b = E.linear_system(res)
        except E.EquationError:
            raise ModelUnsupported(f"trace {nm}: not an exponential decay") from None
        if b[0] != 0.0 or A[0, 0] >= 0:
            raise ModelUnsupported(f"trace {nm}: not an exponential decay")
        taus[nm] = E.snap(-1.0 / A[0, 0], ns)
    # on_pre: [x_post += w]; Apre += dApre; w = clip(w + Apost, wmin, wmax)
    adds_to = None
    role: dict = {}
    inc = {}
    for tgt, op, ex in pre:
        if op == "+=" and tgt in traces:
            inc[tgt] = E.value_of(ex, ns)
            role.setdefault("pre_trace", tgt)
        elif op == "+=":
            adds_to = _strip_post(tgt)
            role["w"] = ex.strip()
        elif op == "=":
            m = re.match(r"^clip\(\s*(\w+)\s*\+\s*(\w+)\s*,\s*(.+?)\s*,\s*(.+?)\s*\)$", ex.strip())
            if not m or m.group(1) != tgt:
                raise ModelUnsupported(f"on_pre {tgt} = {ex}: not w = clip(w + trace, lo, hi)")
            role["w"] = tgt
            role["post_trace"] = m.group(2)
            wmin, wmax = E.value_of(m.group(3), ns), E.value_of(m.group(4), ns)
    for tgt, op, ex in post:
        if op == "+=" and tgt in traces:
            inc[tgt] = E.value_of(ex, ns)
        elif op == "=":
            m = re.match(r"^clip\(\s*(\w+)\s*\+\s*(\w+)\s*,\s*(.+?)\s*,\s*(.+?)\s*\)$", ex.strip())
            if not m or m.group(1) != role.get("w") or m.group(2) != role.get("pre_trace"):
                raise ModelUnsupported(f"on_post {tgt} = {ex}: not w = clip(w + Apre, lo, hi)")
        else:
            raise ModelUnsupported(f"on_post statement {tgt} {op} {ex}")
    apre, apost = role.get("pre_trace"), role.get("post_trace")
    if apre is None or apost is None or set(inc) != {apre, apost} or "w" not in role:
        raise ModelUnsupported("plastic Synapses: not the additive STDP rule")
    rule = STDP(taupre=taus[apre], taupost=taus[apost], dApre=inc[apre], dApost=inc[apost],
                wmin=wmin, wmax=wmax, pre_adds_weight=adds_to is not None)
    return rule, {"target": adds_to, "w": role["w"], "Apre": apre, "Apost": apost}


def _lower_synapses(script, s: SynapsesDesc, ops, groups, rng, index):
    d = s.d
    src, lo, hi = _group_of(d["source"])
    dst, dlo, dhi = _group_of(d["target"])
    if (dlo, dhi) != (0, dst.N):
        raise ModelUnsupported("Synapses onto a subgroup")
    ns = _ns(script, d["namespace"])
    model = E.parse_equations(d["model"]) if d["model"].strip() else E.Model()
    pre = statements(d["on_pre"])
    post = statements(d["on_post"])
    syn_vars = {e.name for e in model.eqs}
    stdp = None
    roles: dict = {}
    if post or any(e.kind == "diff" for e in model.eqs):
        stdp, roles = _stdp_rule(model, ns, pre, post)
        target = roles["target"]
        w_name = roles["w"]
    else:
        if len(pre) != 1 or pre[0][1] != "+=":
            raise ModelUnsupported(f"on_pre {d['on_pre']!r}: only `x_post += w` is lowered")
        target = _strip_post(pre[0][0])
        w_name = pre[0][2].strip()
    slots = groups[dst.name]["slots"]
    tslot = slots.get(target) if target else "ge"
    if tslot is None:
        raise ModelUnsupported(f"{s.name}: {target!r} is not a state variable of the target")
    per_syn = w_name in syn_vars
    w_scalar = 0.0 if per_syn else E.value_of(w_name, ns)
    conn = d["connect"]
    if conn is None:
        raise ModelUnsupported(f"{s.name}: connect() was never called")
    # presynaptic range: the subgroup and an `i<K` / `i>=K` condition
    plo, phi = lo, hi
    cond = conn["condition"]
    if cond:
        m = re.match(r"^\s*i\s*(<|>=)\s*(.+?)\s*$", cond)
        if not m:
            raise ModelUnsupported(f"connect condition {cond!r}: only i<K / i>=K")
        k = int(round(E.value_of(m.group(2), ns)))
        plo, phi = (lo, min(hi, lo + k)) if m.group(1) == "<" else (max(lo, lo + k), hi)
    delay = d["delay"]
    key = s.name
    explicit = conn["i"] is not None
    if not explicit and not per_syn and stdp is None and (
            delay is None or isinstance(delay, UniformDelaySteps) or np.ndim(delay) == 0):
        if isinstance(delay, UniformDelaySteps):
            dmin, dmax = delay.lo, delay.hi
        else:
            dmin = dmax = int(_seconds(delay, ns) / script.dt + 0.5) if delay is not None else 0
        seed = (script.seed * 1_000_003 + 7919 * index) & ((1 << 63) - 1)
        ops.append(Op("synapses_random", (_Ref(src.name), _Ref(dst.name), tslot, conn["p"],
                                          dmin, dmax, w_scalar, seed),
                      {"pre_range": (plo, phi)}, key=key))
        return
    # explicit connectivity: given pairs, or connect(p) drawn on the host
    if explicit:
        i = conn["i"].astype(np.int32) + lo
        j = conn["j"].astype(np.int32)
    else:
        from .models import bernoulli_pairs
        i, j = bernoulli_pairs(rng, phi - plo, dst.N, conn["p"])
        i = (i + plo).astype(np.int32)
    n = len(i)
    if isinstance(delay, UniformDelaySteps):
        dl = rng.integers(delay.lo, delay.hi + 1, size=n).astype(np.int32)
    elif delay is None:
        dl = 0
    elif np.ndim(delay) == 0:
        dl = int(_seconds(delay, ns) / script.dt + 0.5)
    else:
        dl = (np.asarray(delay, np.float64) / script.dt + 0.5).astype(np.int32)
    w = None
    if per_syn:
        init = d["init"].get(w_name)
        if init is None:
            raise ModelUnsupported(f"{s.name}.{w_name} has no initial value")
        w = evaluate_init(init, n, ns, rng)
    ops.append(Op("synapses", (_Ref(src.name), _Ref(dst.name), tslot, i, j),
                  {"w": w, "w_scalar": w_scalar, "delay": dl, "stdp": stdp}, key=key))


def run_script(script: Script, backend) -> dict:
    """Lowers `script` and runs it on `backend` (a GPU Network or an OracleNet)."""
    return script.lower().execute(backend)


__all__ = ["Script", "Program", "lower", "run_script", "ModelUnsupported", "UniformDelaySteps",
           "evaluate_init", "statements"]
