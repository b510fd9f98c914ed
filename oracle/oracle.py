"""ctypes binding of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

`OracleNet` exposes the same methods as `brian2cuda_b200.Network`, so the synthetic model
builders in `brian2cuda_b200.models` can build the same network on either side.  Only the
tests, `__graft_entry__.smoke()` and the CPU-baseline arm of `bench.py` use this module; the
product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
VARS = {"v": 0, "ge": 1, "gi": 2, "m": 3, "h": 4, "n": 5, "lastspike": 6, "not_refractory": 7}
SYN_VARS = {"i": 0, "j": 1, "delay": 2, "w": 3, "Apre": 4, "Apost": 5, "lastupdate": 6}
HINES_VARS = {"v": 0, "m": 1, "h": 2, "n": 3, "Ic": 4}

_lib = None


def build() -> str:
    """Compiles liboracle.so with the Makefile beside this file (g++ -O2 -fopenmp)."""
    r = subprocess.run(["make", "-s", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, I32, I64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        sig = {
            "orc_create": (P, [D, C.c_int]),
            "orc_destroy": (None, [P]),
            "orc_error": (C.c_char_p, [P]),
            "orc_group_lif": (C.c_int, [P, I64, P]),
            "orc_group_hh": (C.c_int, [P, I64, P]),
            "orc_group_poisson": (C.c_int, [P, I64, D]),
            "orc_group_model": (C.c_int, [P, I64, C.c_int, C.c_int, C.c_int, C.c_int, D, P, P]),
            "orc_set_normals": (C.c_int, [P, C.c_int, P, I64, I64]),
            "orc_group_spikegen": (C.c_int, [P, I64, I64, P, P]),
            "orc_timedarray": (C.c_int, [P, C.c_int, P, I64, I64, I64, I64]),
            "orc_poisson_input": (C.c_int, [P, C.c_int, C.c_int, I64, D, D]),
            "orc_set_seed": (None, [P, C.c_uint64]),
            "orc_spikegen_period": (C.c_int, [P, C.c_int, I64]),
            "orc_state_set": (C.c_int, [P, C.c_int, C.c_int, P, I64]),
            "orc_state_get": (C.c_int, [P, C.c_int, C.c_int, P, I64]),
            "orc_synapses": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, I64, P, P, P, D, P,
                                       I32, P]),
            "orc_synapses_random": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, D,
                                              I32, I32, D, C.c_uint64]),
            "orc_syn_count": (I64, [P, C.c_int]),
            "orc_syn_get": (C.c_int, [P, C.c_int, C.c_int, P, I64]),
            "orc_set_uniforms": (C.c_int, [P, C.c_int, P, I64, I64]),
            "orc_run": (C.c_int, [P, I64]),
            "orc_store": (C.c_int, [P]),
            "orc_syn_set_delays": (C.c_int, [P, C.c_int, P, I64]),
            "orc_clear_spikes": (None, [P]),
            "orc_restore": (C.c_int, [P]),
            "orc_timestep": (I64, [P]),
            "orc_spikes": (I64, [P, C.c_int, P, P, I64]),
            "orc_statemon": (C.c_int, [P, C.c_int, C.c_int, P, I64, C.c_int]),
            "orc_statemon_get": (I64, [P, C.c_int, P, P, I64]),
            "orc_ratemon": (C.c_int, [P, C.c_int]),
            "orc_ratemon_get": (I64, [P, C.c_int, P, P, I64]),
            "orc_queue": (I64, [P, C.c_int, P, P, P, I64]),
            "orc_hines_create": (P, [C.c_int, P, P, P, P, P, P, P, P, D, C.c_int]),
            "orc_hines_destroy": (None, [P]),
            "orc_hines_set_current": (C.c_int, [P, P]),
            "orc_hines_state": (C.c_int, [P, C.c_int, P, I64, C.c_int]),
            "orc_hines_run": (C.c_int, [P, I64]),
            "orc_hines_spikes": (C.c_int, [P, P, C.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OracleError(RuntimeError):
    pass


class OracleNet:
    """Sequential CPU simulation with the reference's schedule and spike queues.
    f32=True computes in float32 (the group dtype of the GPU run), else float64."""

    def __init__(self, dt: float, f32: bool = False, reset_before_synapses: bool = False,
                 seed: int = 0, **_ignored):
        self._lib = lib()
        self.dt = float(dt)
        self._h = self._lib.orc_create(self.dt, (1 if f32 else 0) |
                                       (2 if reset_before_synapses else 0))
        self._lib.orc_set_seed(self._h, int(seed))
        self._sizes: list[int] = []
        self._kinds: list[str] = []
        self._smon_n: dict[int, int] = {}

    def close(self):
        if self._h:
            self._lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, r, what):
        if r is None or r < 0:
            raise OracleError(f"{what}: {self._lib.orc_error(self._h).decode()}")
        return r

    # -- groups ---------------------------------------------------------------------------------
    def _add(self, kind, n, gid):
        self._ok(gid, kind)
        self._sizes.append(int(n))
        self._kinds.append(kind)
        return gid

    def lif_group(self, n, params, dtype=None):
        p = np.ascontiguousarray(params.as_array(), dtype=np.float64)
        return self._add("lif", n, self._lib.orc_group_lif(self._h, n, _p(p)))

    def hh_group(self, n, params, dtype=None):
        p = np.ascontiguousarray(params.as_array(), dtype=np.float64)
        return self._add("hh", n, self._lib.orc_group_hh(self._h, n, _p(p)))

    def model_group(self, n, model, dtype=None):
        """A group integrated by the oracle's own numpy evaluation of a generated model
        (model_oracle.ModelCallback) inside the oracle's schedule."""
        from oracle.model_oracle import ModelCallback
        cb = ModelCallback(model, self.dt)
        self._callbacks = getattr(self, "_callbacks", []) + [cb]
        gid = self._lib.orc_group_model(self._h, int(n), cb.n_vars, len(cb.noise),
                                        1 if model.threshold else 0, 1 if model.reset else 0,
                                        float(model.refractory),
                                        C.cast(cb.cfunc, C.c_void_p), None)
        self._model_nn = getattr(self, "_model_nn", {})
        out = self._add("model", n, gid)
        self._model_nn[out] = len(cb.noise)
        return out

    def set_normals(self, gid, u):
        """Queues normal numbers of a model group: rows (steps) of n_normal x size values."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        steps, n = u.shape
        self._ok(self._lib.orc_set_normals(self._h, gid, _p(u), steps, n), "set_normals")

    def poisson_group(self, n, rate, dtype=None):
        return self._add("poisson", n, self._lib.orc_group_poisson(self._h, n, float(rate)))

    def spikegen_group(self, n, indices, steps, period=0):
        idx = np.ascontiguousarray(indices, dtype=np.int32)
        st = np.ascontiguousarray(steps, dtype=np.int64)
        gid = self._add("spikegen", n,
                        self._lib.orc_group_spikegen(self._h, n, len(idx), _p(idx), _p(st)))
        if period:
            self._ok(self._lib.orc_spikegen_period(self._h, gid, int(period)), "period")
        return gid

    def poisson_input(self, gid, var, n, rate, weight):
        """PoissonInput: every step each neuron adds weight * Binomial(n, rate*dt) to var."""
        from brian2cuda_b200._native import VARS
        return self._ok(self._lib.orc_poisson_input(self._h, gid, VARS[var], int(n), float(rate),
                                                    float(weight)), "poisson_input")

    def timed_array(self, gid, values, dt_array):
        """TimedArray input of a LIF (volts), HH (amperes) or Poisson (rate in Hz) group:
        values (rows,) for the whole group or (rows, n) per neuron, each row held for
        dt_array seconds."""
        v = np.asarray(values, dtype=np.float64)
        v = np.ascontiguousarray(v[:, None] if v.ndim == 1 else v)
        r = float(dt_array) / self.dt
        mul, div = (1, int(round(r))) if r >= 1 else (int(round(1 / r)), 1)
        self._ok(self._lib.orc_timedarray(self._h, gid, _p(v), v.shape[0], v.shape[1], mul, div),
                 "timed_array")

    def group_size(self, gid):
        return self._sizes[gid]

    def set_state(self, gid, var, values):
        n = self._sizes[gid]
        a = np.ascontiguousarray(np.broadcast_to(values, (n,)), dtype=np.float64)
        self._ok(self._lib.orc_state_set(self._h, gid, VARS[var], _p(a), n), "set_state")

    def get_state(self, gid, var):
        n = self._sizes[gid]
        a = np.empty(n, dtype=np.float64)
        self._ok(self._lib.orc_state_get(self._h, gid, VARS[var], _p(a), n), "get_state")
        return a

    # -- synapses -------------------------------------------------------------------------------
    def synapses(self, pre, post, target, i, j, w=None, w_scalar=0.0, delay=0, stdp=None):
        i = np.ascontiguousarray(i, dtype=np.int32)
        j = np.ascontiguousarray(j, dtype=np.int32)
        wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
        if np.ndim(delay) == 0:
            da, ds = None, int(delay)
        else:
            da, ds = np.ascontiguousarray(delay, dtype=np.int32), 0
        sp = None if stdp is None else np.ascontiguousarray(stdp.as_array(), dtype=np.float64)
        effect = 1 if stdp is None else 2
        return self._ok(self._lib.orc_synapses(self._h, pre, post, VARS[target], effect, len(i),
                                               _p(i), _p(j), _p(wa), float(w_scalar), _p(da), ds,
                                               _p(sp)), "synapses")

    def synapses_random(self, pre, post, target, p, dmin, dmax, w, seed, pre_range=None):
        lo, hi = pre_range if pre_range is not None else (0, self._sizes[pre])
        return self._ok(self._lib.orc_synapses_random(self._h, pre, int(lo), int(hi), post,
                                                      VARS[target], float(p), int(dmin),
                                                      int(dmax), float(w), int(seed)),
                        "synapses_random")

    def syn_set_delays(self, sid, delay_steps):
        """New delays (steps) of an additive Synapses object between runs; spikes already
        sent keep theirs."""
        d = np.ascontiguousarray(delay_steps, dtype=np.int32)
        self._ok(self._lib.orc_syn_set_delays(self._h, sid, _p(d), len(d)), "syn_set_delays")

    def syn_count(self, sid):
        return self._ok(self._lib.orc_syn_count(self._h, sid), "syn_count")

    def syn_get(self, sid, var):
        n = self.syn_count(sid)
        a = np.empty(n, dtype=np.float64)
        self._ok(self._lib.orc_syn_get(self._h, sid, SYN_VARS[var], _p(a), n), "syn_get")
        if var in ("i", "j", "delay"):
            return a.astype(np.int32)
        return a

    # -- run ------------------------------------------------------------------------------------
    def spike_monitor(self, gid, capacity):
        pass  # the oracle records every spike

    def state_monitor(self, gid, var, indices=None, every=1, capacity=0):
        idx = (np.arange(self._sizes[gid], dtype=np.int64) if indices is None
               else np.ascontiguousarray(indices, dtype=np.int64))
        mid = self._ok(self._lib.orc_statemon(self._h, gid, VARS[var], _p(idx), len(idx),
                                              int(every)), "state_monitor")
        self._smon_n[mid] = len(idx)
        return mid

    def state_values(self, mid):
        """(steps, values[records, indices]) recorded so far."""
        n = self._ok(self._lib.orc_statemon_get(self._h, mid, None, None, 0), "state_values")
        ni = self._smon_n[mid]
        steps = np.empty(n, dtype=np.int64)
        vals = np.empty((n, ni), dtype=np.float64)
        if n:
            self._lib.orc_statemon_get(self._h, mid, _p(steps), _p(vals), n)
        return steps, vals

    def rate_monitor(self, gid, capacity=0):
        return self._ok(self._lib.orc_ratemon(self._h, gid), "rate_monitor")

    def rate_counts(self, mid):
        n = self._ok(self._lib.orc_ratemon_get(self._h, mid, None, None, 0), "rate_counts")
        steps = np.empty(n, dtype=np.int64)
        counts = np.empty(n, dtype=np.int64)
        if n:
            self._lib.orc_ratemon_get(self._h, mid, _p(steps), _p(counts), n)
        return steps, counts

    def finalize(self):
        pass

    def set_uniforms(self, gid, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        steps, n = u.shape
        self._ok(self._lib.orc_set_uniforms(self._h, gid, _p(u), steps, n), "set_uniforms")

    def run(self, steps):
        self._ok(self._lib.orc_run(self._h, int(steps)), "run")

    def sync(self):
        return 0

    def store(self, slot=0):
        """Checkpoint of the dynamic state (one slot): group state and spikespaces, delay
        queues, STDP synapse variables; monitors keep their records across a restore."""
        self._ok(self._lib.orc_store(self._h), "store")

    def restore(self, slot=0):
        self._ok(self._lib.orc_restore(self._h), "restore")

    def clear_spikes(self):
        """Drops every recorded spike (a fresh spike record for the next window)."""
        self._lib.orc_clear_spikes(self._h)

    @property
    def timestep(self):
        return self._lib.orc_timestep(self._h)

    @property
    def t(self):
        return self.timestep * self.dt

    def spikes(self, gid, sub=None):
        n = self._ok(self._lib.orc_spikes(self._h, gid, None, None, 0), "spikes")
        idx = np.empty(n, dtype=np.int32)
        st = np.empty(n, dtype=np.int64)
        self._lib.orc_spikes(self._h, gid, _p(idx), _p(st), n)
        if sub is not None:
            keep = (idx >= sub[0]) & (idx < sub[1])
            idx, st = idx[keep] - sub[0], st[keep]
        return idx, st

    def spikes_last(self, gid):
        idx, st = self.spikes(gid)
        return idx[st == self.timestep - 1]

    def queue(self, sid):
        n = self._ok(self._lib.orc_queue(self._h, sid, None, None, None, 0), "queue")
        a, p, d = (np.empty(n, dtype=np.int32) for _ in range(3))
        self._lib.orc_queue(self._h, sid, _p(a), _p(p), _p(d), n)
        return np.stack([a, p, d], axis=1) if n else np.zeros((0, 3), np.int32)


class OracleHines:
    """The reference's SpatialNeuron update, restated on the CPU, for a batch of neurons."""

    def __init__(self, dt, comp_off, sec_off, sec_start, sec_end, sec_parent, diameter, length,
                 params, f32: bool):
        self._lib = lib()
        self.comp_off = np.ascontiguousarray(comp_off, dtype=np.int64)
        self.n_neurons = len(self.comp_off) - 1
        self.n_comp = int(self.comp_off[-1])
        keep = [np.ascontiguousarray(a, dtype=np.int32)
                for a in (sec_off, sec_start, sec_end, sec_parent)]
        d = np.ascontiguousarray(diameter, dtype=np.float64)
        L = np.ascontiguousarray(length, dtype=np.float64)
        p = np.ascontiguousarray(params.as_array(), dtype=np.float64)
        self._h = self._lib.orc_hines_create(self.n_neurons, _p(self.comp_off),
                                             *[_p(a) for a in keep], _p(d), _p(L), _p(p),
                                             float(dt), 1 if f32 else 0)

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.orc_hines_destroy(self._h)
            self._h = None

    def set_current(self, I):
        a = None if I is None else np.ascontiguousarray(I, dtype=np.float64)
        self._lib.orc_hines_set_current(self._h, _p(a))

    def set_state(self, var, values):
        a = np.ascontiguousarray(np.broadcast_to(values, (self.n_comp,)), dtype=np.float64)
        if self._lib.orc_hines_state(self._h, HINES_VARS[var], _p(a), self.n_comp, 1) != 0:
            raise OracleError("hines set_state")

    def get_state(self, var):
        a = np.empty(self.n_comp, dtype=np.float64)
        if self._lib.orc_hines_state(self._h, HINES_VARS[var], _p(a), self.n_comp, 0) != 0:
            raise OracleError("hines get_state")
        return a

    def run(self, steps):
        self._lib.orc_hines_run(self._h, int(steps))

    def spike_counts(self):
        a = np.empty(self.n_neurons, dtype=np.int32)
        self._lib.orc_hines_spikes(self._h, _p(a), self.n_neurons)
        return a
