"""Brian2 model strings -> sympy expressions in SI units, and the integrators the device
plugin lowers them with.

Brian2 is not importable here, so this module parses the subset of Brian2's equation syntax
that the supported models use (Brian2 user documentation, "Equations"): lines
``dx/dt = expr : unit [(flags)]`` (differential equations), ``name = expr : unit``
(subexpressions) and ``name : unit [(flags)]`` (parameters), with continuation lines, ``#``
comments, SI unit names and the functions exp, log, sqrt, abs, clip, exprel, rand, randn and
the noise term xi.  Everything is evaluated in SI base units: ``13.*mV`` becomes 0.013.

The integrators follow the mathematics of Brian2's state updaters (brian2cuda passes the
code they generate through `brian2cuda/device.py:203-232`, `make_statements`):

  * ``exact``: a linear system with constant coefficients, dx/dt = A x + b, advanced by the
    exact affine propagator x' = e^{A dt} x + (e^{A dt} - I) A^-1 b (computed from the
    exponential of the augmented matrix [[A, b], [0, 0]], so singular A is allowed);
  * ``exponential_euler``: every variable's equation is linear in that variable,
    dx/dt = A(y) x + B(y) with y the other variables; x' = -B/A + (x + B/A) e^{A dt} with A, B
    from the state at the start of the step (x' = x + B dt where A = 0);
  * ``euler``: x' = x + f(y) dt, plus g(y) sqrt(dt) N(0, 1) for a noise term g(y) xi
    (Euler-Maruyama for additive noise; xi has units second^-1/2).
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

import numpy as np
import sympy as sp
from sympy.parsing.sympy_parser import parse_expr

# SI values of the unit names Brian2 scripts use (Brian2's unit system: prefixed SI units).
_BASE = {"volt": 1.0, "second": 1.0, "siemens": 1.0, "farad": 1.0, "amp": 1.0, "ampere": 1.0,
         "ohm": 1.0, "metre": 1.0, "meter": 1.0, "hertz": 1.0, "Hz": 1.0, "coulomb": 1.0,
         "gram": 1e-3, "kilogram": 1.0, "mole": 1.0, "molar": 1e3, "liter": 1e-3, "litre": 1e-3}
_PREFIX = {"y": 1e-24, "z": 1e-21, "a": 1e-18, "f": 1e-15, "p": 1e-12, "n": 1e-9, "u": 1e-6,
           "m": 1e-3, "c": 1e-2, "d": 1e-1, "k": 1e3, "M": 1e6, "G": 1e9}
_SHORT = {"V": "volt", "s": "second", "S": "siemens", "F": "farad", "A": "amp", "Hz": "Hz",
          "ohm": "ohm", "m": "metre", "M": "molar", "l": "liter", "L": "liter", "g": "gram"}


def _unit_table() -> dict[str, float]:
    t = dict(_BASE)
    for p, f in _PREFIX.items():
        for name, v in _BASE.items():
            t[p + name] = f * v
        for short, long in _SHORT.items():
            t[p + short] = f * _BASE[long]
    for short, long in _SHORT.items():
        if short not in ("m", "s", "g", "l", "L", "M"):   # single letters clash with names
            t[short] = _BASE[long]
    t["ms"] = 1e-3
    t["msecond"] = 1e-3
    t["umetre"] = 1e-6
    t["cm"] = 1e-2
    t["mm"] = 1e-3
    t["um"] = 1e-6
    t["nm"] = 1e-9
    t["mV"] = 1e-3
    t["uV"] = 1e-6
    return t


UNITS = _unit_table()
FUNCTIONS = {"exp": sp.exp, "log": sp.log, "sqrt": sp.sqrt, "abs": sp.Abs, "sin": sp.sin,
             "cos": sp.cos, "tanh": sp.tanh}
_EXPREL = sp.Function("exprel")
_CLIP = sp.Function("clip")
RAND = sp.Function("rand")
RANDN = sp.Function("randn")
XI = sp.Symbol("xi")
T = sp.Symbol("t")
DIMENSIONLESS = {"1", "", "radian", "rad"}
_FLAG_WORDS = {"unless refractory", "constant", "shared", "event-driven", "clock-driven",
               "constant over dt", "linked"}


class EquationError(ValueError):
    """A model string outside the supported subset."""


@dataclass
class Eq:
    kind: str                 # "diff", "sub" or "param"
    name: str
    expr: str | None
    unit: str
    flags: tuple = ()


@dataclass
class Model:
    """A parsed model: differential equations (state variables in order), subexpressions and
    parameters, with their flags."""
    eqs: list[Eq] = field(default_factory=list)

    @property
    def state(self) -> list[str]:
        return [e.name for e in self.eqs if e.kind == "diff"]

    @property
    def params(self) -> list[str]:
        return [e.name for e in self.eqs if e.kind == "param"]

    def get(self, name: str) -> Eq | None:
        for e in self.eqs:
            if e.name == name:
                return e
        return None

    def flags(self, name: str) -> tuple:
        e = self.get(name)
        return e.flags if e else ()


def _split_statements(text: str) -> list[str]:
    """Joins continuation lines: a statement ends on the line where its ':' (unit
    separator, at bracket depth 0) appears."""
    out, cur = [], ""
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].rstrip()
        if not line.strip():
            continue
        cur = (cur + " " + line.strip()) if cur else line.strip()
        depth = 0
        found = False
        for ch in cur:
            if ch in "([":
                depth += 1
            elif ch in ")]":
                depth -= 1
            elif ch == ":" and depth == 0:
                found = True
        if found:
            out.append(cur)
            cur = ""
    if cur:
        raise EquationError(f"statement without a unit: {cur!r}")
    return out


def parse_equations(text: str) -> Model:
    """Parses a Brian2 model string (the supported subset) into a Model."""
    m = Model()
    for st in _split_statements(text):
        depth = 0
        cut = None
        for k, ch in enumerate(st):
            if ch in "([":
                depth += 1
            elif ch in ")]":
                depth -= 1
            elif ch == ":" and depth == 0:
                cut = k
                break
        lhs_rhs, unit_part = st[:cut].strip(), st[cut + 1:].strip()
        flags: tuple = ()
        fm = re.match(r"^(.*?)\s*\(([^()]*)\)\s*$", unit_part)
        if fm and fm.group(2).strip() in _FLAG_WORDS | {
                f.strip() for f in fm.group(2).split(",") if f.strip() in _FLAG_WORDS}:
            unit_part = fm.group(1).strip()
            flags = tuple(f.strip() for f in fm.group(2).split(","))
        if "=" in lhs_rhs:
            lhs, rhs = (x.strip() for x in lhs_rhs.split("=", 1))
            dm = re.match(r"^d\s*([A-Za-z_]\w*)\s*/\s*dt$", lhs)
            if dm:
                m.eqs.append(Eq("diff", dm.group(1), rhs, unit_part, flags))
            elif re.match(r"^[A-Za-z_]\w*$", lhs):
                m.eqs.append(Eq("sub", lhs, rhs, unit_part, flags))
            else:
                raise EquationError(f"cannot parse {st!r}")
        else:
            if not re.match(r"^[A-Za-z_]\w*$", lhs_rhs):
                raise EquationError(f"cannot parse {st!r}")
            m.eqs.append(Eq("param", lhs_rhs, None, unit_part, flags))
    return m


def to_sympy(expr: str, symbols: dict[str, sp.Symbol]) -> sp.Expr:
    """Parses one Brian2 expression; every identifier becomes a Symbol (or a known function),
    so names such as E, I, N or S never mean sympy's constants."""
    names = set(re.findall(r"[A-Za-z_]\w*", expr))
    local: dict = {}
    for nm in names:
        if nm in FUNCTIONS:
            local[nm] = FUNCTIONS[nm]
        elif nm == "exprel":
            local[nm] = _EXPREL
        elif nm == "clip":
            local[nm] = _CLIP
        elif nm == "rand":
            local[nm] = RAND
        elif nm == "randn":
            local[nm] = RANDN
        elif nm == "xi":
            local[nm] = XI
        elif nm == "t":
            local[nm] = T
        else:
            local[nm] = symbols.setdefault(nm, sp.Symbol(nm))
    try:
        return parse_expr(expr, local_dict=local, evaluate=True)
    except Exception as exc:   # noqa: BLE001 - sympy raises many types
        raise EquationError(f"cannot parse expression {expr!r}: {exc}") from None


def condition_to_sympy(cond: str, symbols: dict[str, sp.Symbol]) -> sp.Basic:
    """A Brian2 condition (comparisons joined by and / or, negated by not) as a sympy
    boolean; each operand of and / or is parenthesised, since & and | bind tighter than the
    comparisons in the expression grammar."""
    c = re.sub(r"\bor\b", ") | (", cond)
    c = re.sub(r"\band\b", ") & (", c)
    c = re.sub(r"\bnot\b", "~", c)
    return to_sympy("(" + c + ")", symbols)


def numeric_namespace(namespace: dict) -> dict[str, float]:
    """Unit names and the user's numeric constants (floats in SI)."""
    ns = dict(UNITS)
    for k, v in (namespace or {}).items():
        if isinstance(v, (int, float, np.integer, np.floating)) and not isinstance(v, bool):
            ns[k] = float(v)
    return ns


@dataclass
class Resolved:
    """A model with its subexpressions substituted and every constant replaced by its SI
    value: f[x] is the right-hand side of dx/dt as a sympy expression in the state
    variables (and t, xi, and function-valued names left symbolic)."""
    state: list[str]
    f: dict[str, sp.Expr]
    symbols: dict[str, sp.Symbol]
    unless_refractory: set[str]
    params: list[str]


def resolve(model: Model, namespace: dict, keep: set[str] | None = None) -> Resolved:
    """Substitutes subexpressions and numeric constants into the differential equations.
    Names in `keep` (per-neuron parameters, TimedArray calls) stay symbolic."""
    keep = set(keep or ()) | set(model.params)
    syms: dict[str, sp.Symbol] = {}
    ns = numeric_namespace(namespace)
    subs_exprs = {e.name: to_sympy(e.expr, syms) for e in model.eqs if e.kind == "sub"}
    # subexpressions may refer to each other: substitute until none is left
    for _ in range(len(subs_exprs) + 1):
        changed = False
        for k, ex in subs_exprs.items():
            new = ex.xreplace({syms[n]: subs_exprs[n] for n in subs_exprs
                               if n in syms and syms[n] in ex.free_symbols})
            if new != ex:
                subs_exprs[k] = new
                changed = True
        if not changed:
            break
    state = model.state
    f = {}
    for e in model.eqs:
        if e.kind != "diff":
            continue
        ex = to_sympy(e.expr, syms)
        ex = ex.xreplace({syms[n]: subs_exprs[n] for n in subs_exprs if n in syms})
        rep = {}
        for nm, s in syms.items():
            if nm in state or nm in keep:
                continue
            if nm in ns:
                rep[s] = sp.Float(ns[nm], 17)
        f[e.name] = ex.xreplace(rep)
    for x, ex in f.items():
        unknown = {str(s) for s in ex.free_symbols} - set(state) - keep - {"t", "xi"}
        if unknown:
            raise EquationError(f"d{x}/dt refers to undefined names {sorted(unknown)}")
    unl = {e.name for e in model.eqs if e.kind == "diff" and "unless refractory" in e.flags}
    return Resolved(state, f, syms, unl, list(model.params))


def value_of(expr: str, namespace: dict) -> float:
    """A constant expression (a threshold value, a reset value, a delay) in SI."""
    syms: dict[str, sp.Symbol] = {}
    ex = to_sympy(expr, syms)
    ns = numeric_namespace(namespace)
    ex = ex.xreplace({s: sp.Float(ns[n], 17) for n, s in syms.items() if n in ns})
    if ex.free_symbols:
        raise EquationError(f"{expr!r} is not a constant (free names {ex.free_symbols})")
    return float(ex)


# ---- integrators ------------------------------------------------------------------------------
def linear_system(res: Resolved) -> tuple[np.ndarray, np.ndarray]:
    """(A, b) of dx/dt = A x + b when every right-hand side is affine in the state with
    constant coefficients; raises EquationError otherwise."""
    xs = [res.symbols.get(x, sp.Symbol(x)) for x in res.state]
    n = len(xs)
    A = np.zeros((n, n))
    b = np.zeros(n)
    zero = {y: sp.Integer(0) for y in xs}
    for r, x in enumerate(res.state):
        ex = sp.expand(res.f[x])
        if ex.free_symbols & {XI, T} or any(s.name.startswith("xi_") for s in ex.free_symbols) \
                or ex.has(RAND) or ex.has(RANDN):
            raise EquationError(f"d{x}/dt is not autonomous and deterministic")
        try:
            for c, y in enumerate(xs):
                coef = sp.diff(ex, y)
                if coef.free_symbols:
                    raise TypeError
                A[r, c] = float(coef)
            rest = ex.xreplace(zero)          # affine: the right-hand side at x = 0
            if rest.free_symbols:
                raise TypeError
            b[r] = float(rest)
        except TypeError:
            raise EquationError(f"d{x}/dt is not linear with constant coefficients") from None
    return A, b


def snap(value: float, namespace: dict, rtol: float = 1e-12) -> float:
    """The script's own constant when `value` (derived from the equations by floating-point
    arithmetic) equals one of the namespace's numbers to rtol; else value.  Keeps the
    parameters of a recognised model bit-identical to the constants the script wrote."""
    for v in (namespace or {}).values():
        if isinstance(v, (int, float, np.floating)) and not isinstance(v, bool):
            for cand in (float(v), -float(v)):
                if cand == value or (value != 0.0 and abs(cand - value) <= rtol * abs(value)):
                    return cand
    return value


def exact_propagator(A: np.ndarray, b: np.ndarray, dt: float) -> tuple[np.ndarray, np.ndarray]:
    """(M, c) with x(t + dt) = M x(t) + c for dx/dt = A x + b, from the matrix exponential of
    the augmented system (scaling and squaring with a Pade approximant, scipy.linalg.expm)."""
    from scipy.linalg import expm
    n = len(b)
    aug = np.zeros((n + 1, n + 1))
    aug[:n, :n] = A * dt
    aug[:n, n] = b * dt
    E = expm(aug)
    return E[:n, :n], E[:n, n]


def exponential_euler_split(res: Resolved) -> dict[str, tuple[sp.Expr, sp.Expr]]:
    """Per variable x: (A, B) with dx/dt = A x + B, A and B free of x; raises EquationError
    when a right-hand side is not linear in its own variable."""
    out = {}
    for x in res.state:
        sx = res.symbols.get(x, sp.Symbol(x))
        ex = res.f[x]
        A = sp.diff(ex, sx)
        if sx in A.free_symbols:
            A = sp.simplify(A)
            if sx in A.free_symbols:
                raise EquationError(f"d{x}/dt is not linear in {x} "
                                    "(exponential_euler needs that)")
        # linear in x: B is the right-hand side at x = 0
        B = ex.xreplace({sx: sp.Integer(0)})
        out[x] = (A, B)
    return out


def noise_split(res: Resolved) -> dict[str, tuple[sp.Expr, sp.Expr]]:
    """Per variable: (drift f, noise amplitude g) with dx/dt = f + g xi."""
    out = {}
    for x in res.state:
        ex = sp.expand(res.f[x])
        g = sp.diff(ex, XI)
        if XI in g.free_symbols:
            raise EquationError(f"d{x}/dt: the noise term must be linear in xi")
        out[x] = (sp.expand(ex - g * XI), g)
    return out


def exprel_rewrite(ex: sp.Expr) -> sp.Expr:
    """exprel(z) = (e^z - 1)/z as an explicit expression (its z = 0 limit is handled by the
    code printers)."""
    return ex.replace(_EXPREL, lambda z: (sp.exp(z) - 1) / z)


def is_zero(ex) -> bool:
    try:
        return bool(sp.simplify(ex) == 0)
    except Exception:   # noqa: BLE001
        return False


def sample_points(state: list[str], n: int, rng, ranges: dict[str, tuple[float, float]]):
    return {x: rng.uniform(*ranges.get(x, (-1.0, 1.0)), n) for x in state}


def numeric(ex: sp.Expr, names: list[str]):
    """numpy function of the named symbols."""
    syms = [sp.Symbol(n) for n in names]
    return sp.lambdify(syms, ex, modules=[{"exprel": lambda z: np.expm1(z) / z}, "numpy"])


def finite(x) -> bool:
    return bool(np.all(np.isfinite(np.asarray(x, dtype=np.float64))))


__all__ = ["parse_equations", "resolve", "value_of", "linear_system", "exact_propagator",
           "exponential_euler_split", "noise_split", "EquationError", "Model", "Resolved",
           "UNITS"]
