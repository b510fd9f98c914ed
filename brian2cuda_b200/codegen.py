"""Code generation for neuron models that no hand-written kernel integrates.

The role of brian2cuda's code generator (`brian2cuda/cuda_generator.py:281-461`, statements
from abstract code; `templates/common_group.cu:108-160`, the kernel around them): from the
parsed and resolved equations (equations.py) it writes a C++ struct of device functions —
the integration step, the threshold condition, the reset statements — and compiles it with
nvcc against csrc/model_kernel.cuh into a shared object that the library loads
(b2b_group_model).  Supported:

  * method 'exact' for linear systems with constant coefficients (the affine propagator
    e^{A dt}, with a second propagator for the refractory period when variables are marked
    `(unless refractory)`), 'exponential_euler' for equations linear in their own variable,
    'euler' (with additive noise terms xi, xi_1, ... drawn from the net's cuRAND normal
    buffer, Euler-Maruyama); the default picks exact, then exponential Euler, then Euler;
  * thresholds that are conditions on the state (`and`, `or`, `not`), resets that are
    sequences of assignments, refractoriness;
  * functions exp, log, sqrt, abs, sin, cos, tanh, exprel, clip.
Constants are written into the code as literals (R(...) casts keep float32 models in float32
arithmetic); every distinct model source compiles once into `_build/models/<hash>.so`.
"""
from __future__ import annotations

import hashlib
import os
import re
import subprocess
from dataclasses import dataclass, field

import numpy as np
import sympy as sp
from sympy.printing.c import C99CodePrinter

from . import equations as E
from .lowering import ModelUnsupported, Op, statements

SLOT_NAMES = ["v", "ge", "gi", "m", "h", "n"]
PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
ROOT = os.path.dirname(PKG)
MODEL_DIR = os.path.join(PKG, "_build", "models")


@dataclass
class GeneratedModel:
    """A compiled model: the shared object, the variables' slot order and everything the
    oracle needs to integrate the same model on its own."""
    name: str
    state: list[str]                         # variables in slot order
    method: str
    source: str
    path: str | None = None
    refractory: float = 0.0
    n_normal: int = 0
    noise: list[str] = field(default_factory=list)   # noise symbols, in draw order
    threshold: str | None = None             # condition (Brian2 syntax)
    reset: list = field(default_factory=list)        # [(var, op, expr)]
    resolved: object = None                  # equations.Resolved
    unless_refractory: set = field(default_factory=set)
    namespace: dict = field(default_factory=dict)
    propagators: dict = field(default_factory=dict)  # exact: {"active": (M, c), "refractory": ...}
    reset_mask: int = 0

    def slot(self, var: str) -> str:
        return SLOT_NAMES[self.state.index(var)]


class _Printer(C99CodePrinter):
    """sympy -> CUDA device code in the model's scalar type R."""

    def __init__(self, names: dict[str, str]):
        super().__init__({"math_macros": {}})
        self.names = names

    def _print_Symbol(self, e):
        return self.names.get(e.name, e.name)

    def _print_Float(self, e):
        return f"R({float(e)!r})"

    def _print_Integer(self, e):
        return f"R({int(e)})"

    def _print_Rational(self, e):
        return f"(R({int(e.p)})/R({int(e.q)}))"

    def _print_Pow(self, e):
        b, x = e.args
        bs = self.parenthesize(b, 1000)
        if x.is_Integer and 1 <= int(x) <= 4:
            return "(" + "*".join([bs] * int(x)) + ")"
        if x.is_Integer and -4 <= int(x) <= -1:
            return "(R(1)/(" + "*".join([bs] * -int(x)) + "))"
        if x == sp.Rational(1, 2):
            return f"sqrt({self._print(b)})"
        if x == -sp.Rational(1, 2):
            return f"(R(1)/sqrt({self._print(b)}))"
        return f"pow({self._print(b)}, {self._print(x)})"

    def _print_Function(self, e):
        nm = e.func.__name__
        args = ", ".join(self._print(a) for a in e.args)
        if nm == "exprel":
            return f"b2b::model::exprel<R>({args})"
        if nm == "clip":
            return f"b2b::model::clip<R>({args})"
        if nm in ("rand", "randn"):
            raise ModelUnsupported("rand()/randn() inside equations are not lowered; use xi")
        return super()._print_Function(e)

    def _print_Abs(self, e):
        return f"fabs({self._print(e.args[0])})"

    def _print_BooleanTrue(self, e):
        return "true"

    def _print_BooleanFalse(self, e):
        return "false"


def _substitute_ns(ex, syms: dict, ns: dict, keep: set):
    nsn = E.numeric_namespace(ns)
    return ex.xreplace({s: sp.Float(nsn[n], 17) for n, s in syms.items()
                        if n in nsn and n not in keep})


def _noise_symbols(res: E.Resolved) -> list[sp.Symbol]:
    out = []
    for x in res.state:
        for s in sorted(res.f[x].free_symbols, key=lambda s: s.name):
            if (s.name == "xi" or s.name.startswith("xi_")) and s not in out:
                out.append(s)
    return out


def choose_method(res: E.Resolved, method: str | None) -> str:
    noisy = bool(_noise_symbols(res))
    if method is not None:
        if noisy and method != "euler":
            raise ModelUnsupported(f"noise (xi) needs method 'euler', not {method!r}")
        return method
    if noisy:
        return "euler"
    try:
        E.linear_system(res)
        return "exact"
    except E.EquationError:
        pass
    try:
        E.exponential_euler_split(res)
        return "exponential_euler"
    except E.EquationError:
        return "euler"


def _order_state(script, g, res) -> list[str]:
    """Variables that Synapses add into come first (slots 0-2 are the delivery's targets)."""
    targets = []
    from .lowering import SynapsesDesc, _group_of
    for obj in script.objects:
        if isinstance(obj, SynapsesDesc):
            dst, _, _ = _group_of(obj.d["target"])
            if dst is not g:
                continue
            for tgt, op, _ in statements(obj.d["on_pre"]):
                name = tgt[:-5] if tgt.endswith("_post") else tgt
                if op in ("+=", "-=") and name in res.state and name not in targets:
                    targets.append(name)
    if len(targets) > 3:
        raise ModelUnsupported(f"{g.name}: synapses add into more than three variables")
    return targets + [x for x in res.state if x not in targets]


def generate(model: GeneratedModel, dt: float) -> str:
    """C++ source of the model struct and its exports."""
    res = model.resolved
    state = model.state
    nv = len(state)
    if nv > len(SLOT_NAMES):
        raise ModelUnsupported(f"{model.name}: more than {len(SLOT_NAMES)} state variables")
    names = {x: f"x{k}" for k, x in enumerate(state)}
    noise = _noise_symbols(res)
    for d, s in enumerate(noise):
        names[s.name] = f"nrm[{d} * stride]"
    names["t"] = "R(t)"
    pr = _Printer(names)
    body = [f"    const R x{k} = x[{k}];" for k in range(nv)]
    unl = model.unless_refractory
    method = model.method
    if method == "exact":
        A, b = E.linear_system(res)
        order = [res.state.index(x) for x in state]
        A, b = A[np.ix_(order, order)], b[order]
        M, c = E.exact_propagator(A, b, dt)
        model.propagators["active"] = (M, c)
        variants = [("active", M, c)]
        if unl:
            Ar, br = A.copy(), b.copy()
            for k, x in enumerate(state):
                if x in unl:
                    Ar[k, :] = 0.0
                    br[k] = 0.0
            Mr, cr = E.exact_propagator(Ar, br, dt)
            model.propagators["refractory"] = (Mr, cr)
            variants.append(("refractory", Mr, cr))
        for tag, Mx, cx in variants:
            if tag == "refractory":
                body.append("    if (!not_refractory) {")
            elif unl:
                body.append("    if (not_refractory) {")
            for k in range(nv):
                terms = [f"R({float(Mx[k, j])!r})*x{j}" for j in range(nv)
                         if Mx[k, j] != 0.0]
                terms.append(f"R({float(cx[k])!r})")
                body.append(f"      x[{k}] = " + " + ".join(terms) + ";")
            if unl:
                body.append("    }")
    elif method == "exponential_euler":
        split = E.exponential_euler_split(res)
        for k, x in enumerate(state):
            Ax, Bx = split[x]
            body.append(f"    {{ const R A = {pr.doprint(Ax)};")
            body.append(f"      const R B = {pr.doprint(Bx)};")
            body.append(f"      R xn = A == R(0) ? x{k} + B * R(dt) "
                        f": -B / A + (x{k} + B / A) * exp(A * R(dt));")
            hold = f"not_refractory ? xn : x{k}" if x in unl else "xn"
            body.append(f"      x[{k}] = {hold}; }}")
    elif method == "euler":
        split = E.noise_split(E.Resolved(res.state, {x: res.f[x] for x in res.state},
                                         res.symbols, res.unless_refractory, res.params))
        for k, x in enumerate(state):
            f, gx = split[x]
            # the drift and the noise amplitude (g xi: each noise symbol a separate draw)
            drift = pr.doprint(f)
            line = f"x{k} + ({drift}) * R(dt)"
            for d, s in enumerate(noise):
                gs = sp.diff(res.f[x], s)
                if gs != 0:
                    line += f" + ({pr.doprint(gs.xreplace({s: 0}))}) * R(sqrt_dt) * " \
                            f"nrm[{d} * stride]"
            hold = f"not_refractory ? ({line}) : x{k}" if x in unl else line
            body.append(f"    x[{k}] = {hold};")
    else:
        raise ModelUnsupported(f"method {method!r}")
    # threshold and reset in slot variables
    syms = dict(res.symbols)
    thr = "false"
    if model.threshold:
        ex = _substitute_ns(E.condition_to_sympy(model.threshold, syms), syms,
                            model.namespace, set(state))
        thr = _Printer({x: f"x[{k}]" for k, x in enumerate(state)}).doprint(ex)
    rlines = []
    mask = 0
    rpr = _Printer({x: f"x[{k}]" for k, x in enumerate(state)})
    for var, op, ex in model.reset:
        if var not in state:
            raise ModelUnsupported(f"reset writes {var!r}, not a state variable")
        k = state.index(var)
        mask |= 1 << k
        e = _substitute_ns(E.to_sympy(ex, syms), syms, model.namespace, set(state))
        rhs = rpr.doprint(e)
        cop = {"=": "=", "+=": "+=", "-=": "-=", "*=": "*=", "/=": "/="}[op]
        rlines.append(f"    x[{k}] {cop} {rhs};")
    model.reset_mask = mask
    model.n_normal = len(noise)
    model.noise = [s.name for s in noise]
    return _SOURCE.format(
        name=re.sub(r"\W", "_", model.name), nv=nv, nn=len(noise), mask=mask,
        has_thr="true" if model.threshold else "false", sqrt_dt=repr(float(np.sqrt(dt))),
        body="\n".join(body), thr=thr, reset="\n".join(rlines) or "    (void)x;")


_SOURCE = """// Generated by brian2cuda_b200.codegen: model {name}
#include "model_kernel.cuh"

struct Model_{name} {{
  static constexpr int NV = {nv}, NN = {nn}, NU = 0;
  static constexpr unsigned RESET_MASK = {mask}u;
  static constexpr bool HAS_THRESHOLD = {has_thr};
  template <typename R>
  __device__ static void update(R (&x)[NV], double t, double dt, bool not_refractory,
                                const R* nrm, const R* uni, int64_t stride) {{
    (void)t; (void)dt; (void)not_refractory; (void)nrm; (void)uni; (void)stride;
    constexpr double sqrt_dt = {sqrt_dt};
    (void)sqrt_dt;
{body}
  }}
  template <typename R>
  __device__ static bool threshold(const R (&x)[NV]) {{
    (void)x;
    return {thr};
  }}
  template <typename R>
  __device__ static void reset(R (&x)[NV]) {{
{reset}
  }}
}};

B2B_MODEL_EXPORT(Model_{name})
"""


def _header_digest() -> str:
    h = hashlib.sha256()
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".h", ".cuh")):
            with open(os.path.join(CSRC, f), "rb") as fh:
                h.update(f.encode() + fh.read())
    with open(os.path.join(ROOT, "include", "b2b.h"), "rb") as fh:
        h.update(fh.read())
    return h.hexdigest()


def compile_model(source: str) -> str:
    """Compiles a generated model for sm_100a into _build/models/<hash>.so (once per source
    and header set); returns the shared object's path."""
    from .build import ARCH, NVCC
    key = hashlib.sha256((source + _header_digest()).encode()).hexdigest()[:20]
    os.makedirs(MODEL_DIR, exist_ok=True)
    so = os.path.join(MODEL_DIR, f"model_{key}.so")
    if os.path.exists(so):
        return so
    cu = os.path.join(MODEL_DIR, f"model_{key}.cu")
    with open(cu, "w") as f:
        f.write(source)
    tmp = so + f".{os.getpid()}.tmp"
    cmd = [NVCC] + ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                           "-Xcompiler", "-fvisibility=hidden", "-shared",
                           f"-I{CSRC}", f"-I{os.path.join(ROOT, 'include')}", cu, "-o", tmp]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for the generated model:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, so)
    return so


def lower_model(script, g, model, res, thr, rst, refractory, method, dtype, ops):
    """Lowering hook (lowering._lower_group) for a model no hand-written kernel covers."""
    ns = {}
    ns.update(script.namespace)
    ns.update(g.spec.get("namespace") or {})
    for s in res.state:
        if res.f[s].has(E.RAND) or res.f[s].has(E.RANDN):
            raise ModelUnsupported(f"{g.name}: rand()/randn() inside equations; use xi")
    state = _order_state(script, g, res)
    meth = choose_method(res, method)
    gm = GeneratedModel(name=g.name, state=state, method=meth, source="",
                        refractory=refractory, threshold=g.spec.get("threshold"),
                        reset=statements(g.spec.get("reset") or ""), resolved=res,
                        unless_refractory=set(res.unless_refractory), namespace=ns)
    try:
        gm.source = generate(gm, script.dt)
    except E.EquationError as exc:
        raise ModelUnsupported(f"{g.name}: {exc}") from None
    ops.append(Op("model_group", (g.N, gm, dtype), key=g.name))
    return {"kind": "model", "N": g.N, "slots": {x: gm.slot(x) for x in state}, "model": gm}
