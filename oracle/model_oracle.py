"""The oracle's arithmetic for generated neuron models — TEST INFRASTRUCTURE ONLY.

The GPU library integrates a generated model with CUDA code that brian2cuda_b200/codegen.py
prints from the equations; this module integrates the same equations with numpy, through
its own derivation of each integrator, and hands the result to the C++ oracle through its
callback group (oracle.cpp, kind MODEL), which supplies the schedule, refractoriness,
spikes, delays and synapses.  Only the equation parser (brian2cuda_b200/equations.py) is
shared, and it is pinned by the known-answer tests.

  * exact: the propagator of dx/dt = A x + b over one step comes from integrating the
    linear system for the unit vectors and for x = 0 with an explicit Runge-Kutta method of
    order 8 (scipy's DOP853) at relative tolerance 1e-13 — not from the matrix exponential
    the generator uses;
  * exponential_euler: A = d f/d x and B = f - A x evaluated with numpy at the pre-step state,
    x' = -B/A + (x + B/A) exp(A dt);
  * euler: x' = x + f dt + g sqrt(dt) N, with N the GPU's normal numbers of that step.
"""
from __future__ import annotations

import ctypes as C


import numpy as np
import sympy as sp

from brian2cuda_b200 import equations as E

CALLBACK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_double,
                       C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_uint8),
                       C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_double))


def _propagator_rk(A: np.ndarray, b: np.ndarray, dt: float):
    from scipy.integrate import solve_ivp
    n = len(b)

    def rhs(_t, y, bb):
        return A @ y + bb
    M = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        M[:, j] = solve_ivp(rhs, (0, dt), e, method="DOP853", rtol=1e-13, atol=1e-22,
                            args=(np.zeros(n),)).y[:, -1]
    c = solve_ivp(rhs, (0, dt), np.zeros(n), method="DOP853", rtol=1e-13, atol=1e-22,
                  args=(b,)).y[:, -1]
    return M, c


def _numpy_fn(ex, names):
    syms = [sp.Symbol(n) for n in names]
    return sp.lambdify(syms, ex, modules=[{"exprel": lambda z: np.where(
        np.abs(z) < 1e-16, 1.0, np.expm1(z) / np.where(z == 0, 1.0, z)),
        "clip": np.clip}, "numpy"])


class ModelCallback:
    """The callback of one model group; keep a reference while the oracle net lives."""

    def __init__(self, gm, dt: float):
        self.gm = gm
        self.dt = float(dt)
        res = gm.resolved
        self.state = list(gm.state)
        nv = len(self.state)
        self.noise = list(gm.noise)
        unl = set(gm.unless_refractory)
        self.unl = np.array([x in unl for x in self.state])
        if gm.method == "exact":
            A, b = E.linear_system(res)
            order = [res.state.index(x) for x in self.state]
            A, b = A[np.ix_(order, order)], b[order]
            self.M, self.c = _propagator_rk(A, b, self.dt)
            Ar, br = A.copy(), b.copy()
            Ar[self.unl, :] = 0.0
            br[self.unl] = 0.0
            self.Mr, self.cr = _propagator_rk(Ar, br, self.dt)
        elif gm.method == "exponential_euler":
            split = E.exponential_euler_split(res)
            self.AB = [(_numpy_fn(split[x][0], self.state), _numpy_fn(split[x][1], self.state))
                       for x in self.state]
        elif gm.method == "euler":
            xis = [sp.Symbol(n) for n in self.noise]
            self.f = []
            self.g = []
            for x in self.state:
                ex = sp.expand(res.f[x])
                gs = [sp.diff(ex, s) for s in xis]
                drift = ex.xreplace({s: 0 for s in xis})
                self.f.append(_numpy_fn(drift, self.state + ["t"]))
                self.g.append([_numpy_fn(gx, self.state + ["t"]) for gx in gs])
        else:
            raise ValueError(gm.method)
        syms = dict(res.symbols)
        nsn = E.numeric_namespace(gm.namespace)
        self.thr = None
        if gm.threshold:
            ex = E.condition_to_sympy(gm.threshold, syms)
            ex = ex.xreplace({s: sp.Float(nsn[n], 17) for n, s in syms.items()
                              if n in nsn and n not in self.state})
            self.thr = _numpy_fn(ex, self.state)
        self.reset = []
        for var, op, rhs in gm.reset:
            ex = E.to_sympy(rhs, syms)
            ex = ex.xreplace({s: sp.Float(nsn[n], 17) for n, s in syms.items()
                              if n in nsn and n not in self.state})
            self.reset.append((self.state.index(var), op, _numpy_fn(ex, self.state)))
        self.cfunc = CALLBACK(self._call)
        self.n_vars = nv

    def _call(self, _user, phase, ts, t, dt, n, vars_p, mask_p, idx_p, n_idx, nrm_p):
        try:
            nv = self.n_vars
            x = np.ctypeslib.as_array(vars_p, shape=(nv * n,)).reshape(nv, n)
            if phase == 0:
                nr = np.ctypeslib.as_array(mask_p, shape=(n,)).astype(bool)
                if self.gm.method == "exact":
                    new = self.M @ x + self.c[:, None]
                    if self.unl.any():
                        held = self.Mr @ x + self.cr[:, None]
                        new = np.where(nr[None, :], new, held)
                elif self.gm.method == "exponential_euler":
                    cols = [x[k] for k in range(nv)]
                    new = np.empty_like(x)
                    for k, (fa, fb) in enumerate(self.AB):
                        a = np.broadcast_to(np.asarray(fa(*cols), dtype=np.float64), (n,))
                        b = np.broadcast_to(np.asarray(fb(*cols), dtype=np.float64), (n,))
                        with np.errstate(divide="ignore", invalid="ignore"):
                            ee = -b / a + (x[k] + b / a) * np.exp(a * dt)
                        new[k] = np.where(a == 0.0, x[k] + b * dt, ee)
                        if self.unl[k]:
                            new[k] = np.where(nr, new[k], x[k])
                else:
                    cols = [x[k] for k in range(nv)] + [t]
                    nn = len(self.noise)
                    nrm = (np.ctypeslib.as_array(nrm_p, shape=(nn * n,)).reshape(nn, n)
                           if nn else None)
                    new = np.empty_like(x)
                    for k in range(nv):
                        v = x[k] + np.asarray(self.f[k](*cols), dtype=np.float64) * dt
                        for d, gfn in enumerate(self.g[k]):
                            v = v + np.asarray(gfn(*cols), dtype=np.float64) * np.sqrt(dt) * nrm[d]
                        new[k] = np.where(nr, v, x[k]) if self.unl[k] else v
                x[:] = new
            elif phase == 1:
                mask = np.ctypeslib.as_array(mask_p, shape=(n,))
                mask[:] = 0
                if self.thr is not None:
                    mask[:] = np.broadcast_to(np.asarray(self.thr(*[x[k] for k in range(nv)]),
                                                         dtype=bool), (n,))
            else:
                idx = np.ctypeslib.as_array(idx_p, shape=(n_idx,)).astype(np.int64)
                sub = x[:, idx]
                for k, op, fn in self.reset:
                    val = np.broadcast_to(np.asarray(fn(*[sub[j] for j in range(nv)]),
                                                     dtype=np.float64), (len(idx),))
                    if op == "=":
                        sub[k] = val
                    elif op == "+=":
                        sub[k] = sub[k] + val
                    elif op == "-=":
                        sub[k] = sub[k] - val
                    elif op == "*=":
                        sub[k] = sub[k] * val
                    else:
                        sub[k] = sub[k] / val
                x[:, idx] = sub
            return 0
        except Exception:   # noqa: BLE001 - reported through the oracle's error
            import traceback
            traceback.print_exc()
            return 1
