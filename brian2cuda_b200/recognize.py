"""Recognition of models the hand-written kernels integrate.

A NeuronGroup whose equations, after parsing and constant substitution
(brian2cuda_b200.equations), are the linear integrate-and-fire system of the LIF kernel
(method 'exact') or the conductance-based Hodgkin-Huxley system of the COBAHH kernel (method
'exponential_euler') runs on those kernels; any other model goes to generated code.  The
checks are structural (coefficients of the expanded right-hand sides) plus a numerical
comparison of the rate functions on a grid of membrane potentials, so names, term order and
unit spellings of the script do not matter.
"""
from __future__ import annotations

import math

import numpy as np
import sympy as sp

from . import equations as E
from .network import HH, LIF


def _sym(res: E.Resolved, name: str) -> sp.Symbol:
    return res.symbols.get(name, sp.Symbol(name))


def match_lif(res: E.Resolved, vname: str, namespace: dict | None = None) -> dict | None:
    """The LIF kernel's system: v (the thresholded variable) and up to two synaptic
    variables s1, s2 with ds/dt = -s/tau_s, and dv/dt = (El - v + k1 s1 + k2 s2)/taum.
    Returns the kernel parameters and the slot of every state variable, or None."""
    try:
        A, b = E.linear_system(res)
    except E.EquationError:
        return None
    names = res.state
    if vname not in names or len(names) > 3:
        return None
    iv = names.index(vname)
    others = [k for k in range(len(names)) if k != iv]
    for k in others:
        row = A[k].copy()
        if b[k] != 0.0 or row[k] >= 0.0 or np.any(np.delete(row, k) != 0.0):
            return None
    if A[iv, iv] > 0.0:
        return None
    taum = math.inf if A[iv, iv] == 0.0 else -1.0 / A[iv, iv]
    if math.isinf(taum):
        if b[iv] != 0.0 or any(A[iv, k] != 0.0 for k in others):
            return None
        El, ks = 0.0, [0.0 for _ in others]
    else:
        El = b[iv] * taum
        ks = [A[iv, k] * taum for k in others]
    taus = [-1.0 / A[k, k] for k in others]
    slots = {vname: "v"}
    prm = {"El": El, "taum": taum, "taue": 0.0, "taui": 0.0, "ke": 0.0, "ki": 0.0}
    for (k, kk, tau), slot in zip(zip(others, ks, taus), ("ge", "gi")):
        slots[names[k]] = slot
        prm["ke" if slot == "ge" else "ki"] = kk
        prm["taue" if slot == "ge" else "taui"] = tau
    prm = {k: E.snap(v, namespace) for k, v in prm.items()}
    return {"params": prm, "slots": slots}


# The COBAHH kernel's rate functions (Traub and Miles 1991, as in the reference's
# examples/cobahh.py model), in SI units (V, 1/s), with the threshold offset VT.
def cobahh_rates(v, VT):
    x = np.asarray(v, dtype=np.float64) - VT
    am = 0.32e6 * (13e-3 - x) / np.expm1((13e-3 - x) / 4e-3)
    bm = 0.28e6 * (x - 40e-3) / np.expm1((x - 40e-3) / 5e-3)
    ah = 128.0 * np.exp((17e-3 - x) / 18e-3)
    bh = 4000.0 / (1.0 + np.exp((40e-3 - x) / 5e-3))
    an = 0.032e6 * (15e-3 - x) / np.expm1((15e-3 - x) / 5e-3)
    bn = 500.0 * np.exp((10e-3 - x) / 40e-3)
    return {"m": (am, bm), "h": (ah, bh), "n": (an, bn)}


def _poly_coeffs(ex: sp.Expr, gens: list[sp.Symbol]) -> dict[tuple, float] | None:
    try:
        P = sp.Poly(sp.expand(ex), *gens)
    except sp.PolynomialError:
        return None
    out = {}
    for mon, c in P.terms():
        if getattr(c, "free_symbols", set()):
            return None
        out[mon] = float(c)
    return out


def match_cobahh(res: E.Resolved, vname: str = "v",
                 namespace: dict | None = None) -> dict | None:
    """The COBAHH kernel's system: v, gates m, h, n, conductances ge, gi with
      Cm dv/dt = gl (El - v) + ge (Ee - v) + gi (Ei - v) - gNa m^3 h (v - ENa) - gK n^4 (v - EK)
      dx/dt = alpha_x(v) (1 - x) - beta_x(v) x      (x = m, h, n; Traub-Miles rates, VT)
      dge/dt = -ge/taue, dgi/dt = -gi/taui
    The gating and conductance variables are told apart by their equations (a gate is the
    variable whose cubed / fourth power multiplies the sodium / potassium term).  Returns the
    kernel parameters and each variable's slot, or None."""
    names = res.state
    if len(names) != 6 or vname not in names:
        return None
    v = _sym(res, vname)
    others = [n for n in names if n != vname]
    syms = {n: _sym(res, n) for n in others}
    gens = [v] + [syms[n] for n in others]
    cv = _poly_coeffs(res.f[vname], gens)
    if cv is None:
        return None
    # classify: decaying conductances have ds/dt = -s/tau
    cond = []
    for n in others:
        c = _poly_coeffs(res.f[n], [syms[n]])
        if c is not None and set(c) == {(1,)} and c[(1,)] < 0 and \
                not (res.f[n].free_symbols - {syms[n]}):
            cond.append(n)
    gates = [n for n in others if n not in cond]
    if len(cond) != 2 or len(gates) != 3:
        return None

    def mono(**powers):
        return tuple([powers.get("v", 0)] + [powers.get(n, 0) for n in others])
    # gate roles from the monomials: x^3 * y (sodium), z^4 (potassium)
    role = {}
    for key, c in cv.items():
        pw = dict(zip(["v"] + others, key))
        gp = {g: pw[g] for g in gates if pw[g]}
        if sorted(gp.values()) == [1, 3]:
            role["m"] = [g for g, p in gp.items() if p == 3][0]
            role["h"] = [g for g, p in gp.items() if p == 1][0]
        elif list(gp.values()) == [4]:
            role["n"] = list(gp)[0]
    if set(role) != {"m", "h", "n"}:
        return None
    m, h, n = role["m"], role["h"], role["n"]
    # excitatory / inhibitory conductance: the one with the larger reversal potential is ge
    terms = {}
    for cn in cond:
        a = cv.get(mono(v=1, **{cn: 1}), 0.0)
        c0 = cv.get(mono(**{cn: 1}), 0.0)
        if a >= 0.0:
            return None
        terms[cn] = (-1.0 / a, c0 / -a)     # (Cm, E_rev)
    ge, gi = sorted(cond, key=lambda c: -terms[c][1])
    Cm = terms[ge][0]
    if not math.isclose(terms[gi][0], Cm, rel_tol=1e-9):
        return None
    Ee, Ei = terms[ge][1], terms[gi][1]
    gNa = -cv.get(mono(v=1, **{m: 3, h: 1}), 0.0) * Cm
    ENa = cv.get(mono(**{m: 3, h: 1}), 0.0) * Cm / gNa if gNa else 0.0
    gK = -cv.get(mono(v=1, **{n: 4}), 0.0) * Cm
    EK = cv.get(mono(**{n: 4}), 0.0) * Cm / gK if gK else 0.0
    gl = -cv.get(mono(v=1), 0.0) * Cm
    El = cv.get(mono(), 0.0) * Cm / gl if gl else 0.0
    expected = {mono(v=1, **{ge: 1}), mono(**{ge: 1}), mono(v=1, **{gi: 1}), mono(**{gi: 1}),
                mono(v=1, **{m: 3, h: 1}), mono(**{m: 3, h: 1}), mono(v=1, **{n: 4}),
                mono(**{n: 4}), mono(v=1), mono()}
    if not set(k for k, c in cv.items() if c != 0.0) <= expected or gNa <= 0 or gK <= 0:
        return None
    # gating: A(v) = -(alpha + beta), B(v) = alpha
    try:
        split = E.exponential_euler_split(E.Resolved(list(gates), {x: res.f[x] for x in gates},
                                                     res.symbols, set(), res.params))
    except E.EquationError:
        return None
    fa = {g: E.numeric(split[g][1], [vname]) for g in gates}
    fab = {g: E.numeric(-split[g][0], [vname]) for g in gates}
    # VT from alpha_h at v = 0: alpha_h(0) = 128 exp((17 mV + VT) / 18 mV)
    ah0 = float(np.asarray(fa[h](0.0)))
    if not ah0 > 0:
        return None
    VT = 18e-3 * math.log(ah0 / 128.0) - 17e-3
    grid = np.linspace(-0.1, 0.06, 97) + 1.234e-4   # away from the removable singularities
    ref = cobahh_rates(grid, VT)
    for role_name, g in (("m", m), ("h", h), ("n", n)):
        a_ref, b_ref = ref[role_name]
        a = np.asarray(fa[g](grid), dtype=np.float64) * np.ones_like(grid)
        ab = np.asarray(fab[g](grid), dtype=np.float64) * np.ones_like(grid)
        if not (np.allclose(a, a_ref, rtol=1e-9, atol=0) and
                np.allclose(ab - a, b_ref, rtol=1e-9, atol=1e-9 * np.max(np.abs(b_ref)))):
            return None
    taue = -1.0 / _poly_coeffs(res.f[ge], [syms[ge]])[(1,)]
    taui = -1.0 / _poly_coeffs(res.f[gi], [syms[gi]])[(1,)]
    prm = {"Cm": Cm, "gl": gl, "El": El, "EK": EK, "ENa": ENa, "gNa": gNa, "gK": gK, "VT": VT,
           "Ee": Ee, "Ei": Ei, "taue": taue, "taui": taui}
    prm = {k: E.snap(v, namespace, 1e-9 if k == "VT" else 1e-12) for k, v in prm.items()}
    slots = {vname: "v", m: "m", h: "h", n: "n", ge: "ge", gi: "gi"}
    return {"params": prm, "slots": slots}


def lif_from(match: dict, Vt: float | None, Vr: float | None, refractory: float,
             unless_refractory: bool) -> LIF:
    p = match["params"]
    return LIF(El=p["El"], taum=p["taum"], taue=p["taue"], taui=p["taui"], ke=p["ke"],
               ki=p["ki"], Vt=Vt if Vt is not None else math.inf,
               Vr=Vr if Vr is not None else 0.0, refractory=refractory,
               has_threshold=Vt is not None, has_reset=Vr is not None,
               unless_refractory=unless_refractory)


def hh_from(match: dict, Vthr: float, refractory: float) -> HH:
    p = match["params"]
    return HH(Cm=p["Cm"], gl=p["gl"], El=p["El"], EK=p["EK"], ENa=p["ENa"], gNa=p["gNa"],
              gK=p["gK"], VT=p["VT"], Ee=p["Ee"], Ei=p["Ei"], taue=p["taue"], taui=p["taui"],
              Vthr=Vthr, refractory=refractory)
