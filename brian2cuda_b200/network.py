"""Python view of a libb2b network (the C ABI of include/b2b.h through ctypes).

`Network` mirrors the pieces of a Brian2 network that brian2cuda's generated hot path
handles: neuron groups (exact LIF, exponential-Euler HH, Poisson, spike generators),
Synapses with delays and additive / STDP effects, spike monitors, and a batch of
multicompartment neurons.  Units are SI throughout (volts, seconds, siemens).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _native as N
from ._native import B2BError

_DTYPES = {"float32": N.F32, "float64": N.F64, np.float32: N.F32, np.float64: N.F64}


def _dt_code(dtype) -> int:
    if isinstance(dtype, int):
        return dtype
    key = np.dtype(dtype).type if not isinstance(dtype, str) else dtype
    if key not in _DTYPES:
        raise ValueError(f"unsupported dtype {dtype!r}")
    return _DTYPES[key]


def _np_dtype(code: int):
    return np.float32 if code == N.F32 else np.float64


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class LIF:
    """dv/dt = (El - v + ke*ge + ki*gi)/taum [(unless refractory)], dge/dt = -ge/taue,
    dgi/dt = -gi/taui; threshold v > Vt, reset v = Vr."""
    El: float = 0.0
    taum: float = math.inf
    taue: float = 0.0
    taui: float = 0.0
    ke: float = 0.0
    ki: float = 0.0
    Vt: float = 1.0
    Vr: float = 0.0
    refractory: float = 0.0
    has_threshold: bool = True
    has_reset: bool = True
    unless_refractory: bool = False

    def to_c(self) -> N.LifParams:
        return N.LifParams(self.El, self.taum, self.taue, self.taui, self.ke, self.ki, self.Vt,
                           self.Vr, self.refractory, int(self.has_threshold),
                           int(self.has_reset), int(self.unless_refractory), 0)

    def as_array(self) -> np.ndarray:
        return np.array([self.El, self.taum, self.taue, self.taui, self.ke, self.ki, self.Vt,
                         self.Vr, self.refractory, float(self.has_threshold),
                         float(self.has_reset), float(self.unless_refractory)])


@dataclass
class HH:
    """COBAHH (examples/cobahh.py): conductance-based Hodgkin-Huxley, threshold v > Vthr."""
    Cm: float
    gl: float
    El: float
    EK: float
    ENa: float
    gNa: float
    gK: float
    VT: float
    Ee: float
    Ei: float
    taue: float
    taui: float
    Vthr: float
    refractory: float

    def to_c(self) -> N.HhParams:
        return N.HhParams(*self.as_array())

    def as_array(self) -> np.ndarray:
        return np.array([self.Cm, self.gl, self.El, self.EK, self.ENa, self.gNa, self.gK,
                         self.VT, self.Ee, self.Ei, self.taue, self.taui, self.Vthr,
                         self.refractory])


@dataclass
class STDP:
    """Event-driven additive STDP (examples/stdp.py): traces Apre/Apost, weight clipped to
    [wmin, wmax]; on_pre adds w to the target variable when pre_adds_weight."""
    taupre: float
    taupost: float
    dApre: float
    dApost: float
    wmin: float
    wmax: float
    pre_adds_weight: bool = True

    def to_c(self) -> N.StdpParams:
        return N.StdpParams(self.taupre, self.taupost, self.dApre, self.dApost, self.wmin,
                            self.wmax, int(self.pre_adds_weight), 0)

    def as_array(self) -> np.ndarray:
        return np.array([self.taupre, self.taupost, self.dApre, self.dApost, self.wmin,
                         self.wmax, float(self.pre_adds_weight)])


@dataclass
class HinesParams:
    Cm: float = 0.01          # F/m^2  (1 uF/cm^2)
    Ri: float = 1.0           # ohm*m  (100 ohm*cm)
    El: float = 10.613e-3
    EK: float = -12e-3
    ENa: float = 115e-3
    gl: float = 3.0           # S/m^2  (0.3 mS/cm^2)
    gNa: float = 1200.0       # 120 mS/cm^2
    gK: float = 360.0         # 36 mS/cm^2
    Vthr: float = 50e-3
    channel_dtype: str = "float32"

    def to_c(self) -> N.HinesParams:
        return N.HinesParams(self.Cm, self.Ri, self.El, self.EK, self.ENa, self.gl, self.gNa,
                             self.gK, self.Vthr, _dt_code(self.channel_dtype), 0)

    def as_array(self) -> np.ndarray:
        return np.array([self.Cm, self.Ri, self.El, self.EK, self.ENa, self.gl, self.gNa,
                         self.gK, self.Vthr])


def spike_steps(times, dt: float) -> np.ndarray:
    """Steps of spike times for a SpikeGeneratorGroup: the bin [k dt, (k+1) dt) holding each
    time, by Brian2's timestep(t, dt) = int((t + 1e-3 dt) / dt) (brian2cuda/cuda_generator.py:
    997-1006), so that times computed as k*dt land in bin k despite rounding."""
    t = np.asarray(times, dtype=np.float64)
    return ((t + 1e-3 * dt) / dt).astype(np.int64)


def atomic_rate(n_targets: int, n_events: int, device: int = 0, stream: int | None = None,
                reps: int = 5) -> tuple[float, float, float]:
    """Scattered float32 atomic additions per second that the GPU sustains into an array of
    n_targets floats at uniform indices: (index loaded from device memory per event, index
    computed in registers, into the distributed shared memory of 8-CTA clusters).  The
    ceiling of the additive spike delivery, and of a delivery accumulating in clusters."""
    lib = N.lib()
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    st = lib.b2b_atomic_rate(int(device), stream, int(n_targets), int(n_events), int(reps),
                             C.byref(a), C.byref(b), C.byref(c))
    if st != N.B2B_OK:
        raise B2BError(st, "b2b_atomic_rate")
    return a.value, b.value, c.value


class Network:
    """A network on one GPU.  Build it (groups, synapses, monitors), call `finalize()`,
    then `run(steps)`; state can be read and written between runs."""

    def __init__(self, dt: float, seed: int = 0, device: int = 0, steps_per_graph: int = 50,
                 graphs: bool = True, checked: bool = False, reset_before_synapses: bool = False,
                 stream: int | None = None, two_launch: bool | None = None,
                 small: bool = False, one_launch: bool = False):
        """`stream`: raw cudaStream_t (e.g. torch.cuda.Stream().cuda_stream) to run on; by
        default the network creates its own non-blocking stream.  `two_launch`: True runs every
        step as two concurrent launches (the neuron update, and the delivery of earlier
        steps' spikes into a double-buffered input) where the net allows it, False always
        the per-step kernels, None (default) the two launches for nets that allow them with at
        most 2^18 neurons, until autotune() picks the faster form.  `small`: run
        a small network (one LIF/HH population of <= 4096 neurons, additive synapses onto
        itself) in one CTA per chunk of steps with the state in shared memory; it pays off for
        nets of a few hundred to ~2000 neurons with few delays.  `one_launch`: where the net
        allows the two launches (and every projection has at most 64 delays, no TimedArray or
        PoissonInput drives the population), run both halves of every step as one launch."""
        self._lib = N.lib()
        self.dt = float(dt)
        flags = (0 if graphs else N.NET_NO_GRAPH) | (N.NET_CHECKED if checked else 0)
        if reset_before_synapses:
            flags |= N.NET_RESET_BEFORE_SYNAPSES
        if two_launch is True:
            flags |= N.NET_TWO_LAUNCH
        elif two_launch is False:
            flags |= N.NET_PER_STEP
        if small:
            flags |= N.NET_SMALL
        if one_launch:
            flags |= N.NET_ONE_LAUNCH
        cfg = N.Config(self.dt, device, steps_per_graph, seed, stream, flags, 0)
        h = C.c_void_p()
        st = self._lib.b2b_create(C.byref(cfg), C.byref(h))
        if st != N.B2B_OK:
            raise B2BError(st, "b2b_create")
        self._h = h
        self._groups: list[tuple[str, int, int]] = []   # (kind, n, dtype code)
        self._syns: list[tuple[int, int, int]] = []     # (pre, post, dtype code)
        self._hines: list[HinesBatch] = []
        self._smons: dict[int, tuple[int, type]] = {}   # state monitor: (width, dtype)

    # -- plumbing ---------------------------------------------------------------------------
    def _check(self, st: int, what: str):
        if st != N.B2B_OK:
            buf = C.create_string_buffer(512)
            self._lib.b2b_last_error(self._h, buf, 512)
            raise B2BError(st, f"{what}: {buf.value.decode(errors='replace')}")

    def close(self):
        if getattr(self, "_h", None):
            for hb in self._hines:
                hb._h = None
            self._lib.b2b_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- groups ---------------------------------------------------------------------------------
    def _add(self, kind: str, n: int, dtype: int, gid: C.c_int32) -> int:
        self._groups.append((kind, int(n), dtype))
        return gid.value

    def lif_group(self, n: int, params: LIF, dtype="float64") -> int:
        gid = C.c_int32()
        code = _dt_code(dtype)
        p = params.to_c()
        self._check(self._lib.b2b_group_lif(self._h, n, code, C.byref(p), C.byref(gid)), "lif")
        return self._add("lif", n, code, gid)

    def hh_group(self, n: int, params: HH, dtype="float32") -> int:
        gid = C.c_int32()
        code = _dt_code(dtype)
        p = params.to_c()
        self._check(self._lib.b2b_group_hh(self._h, n, code, C.byref(p), C.byref(gid)), "hh")
        return self._add("hh", n, code, gid)

    def poisson_group(self, n: int, rate: float, dtype="float32") -> int:
        gid = C.c_int32()
        code = _dt_code(dtype)
        self._check(self._lib.b2b_group_poisson(self._h, n, code, float(rate), C.byref(gid)),
                    "poisson")
        return self._add("poisson", n, code, gid)

    def spikegen_group(self, n: int, indices, steps, period: int = 0) -> int:
        """SpikeGeneratorGroup: neuron indices[k] spikes at step steps[k] (spike_steps()
        turns times into steps); period > 0 repeats the pattern every `period` steps."""
        idx = np.ascontiguousarray(indices, dtype=np.int32)
        stp = np.ascontiguousarray(steps, dtype=np.int64)
        gid = C.c_int32()
        self._check(self._lib.b2b_group_spikegen(self._h, n, len(idx), _ptr(idx), _ptr(stp),
                                                 C.byref(gid)), "spikegen")
        if period:
            self._check(self._lib.b2b_spikegen_period(self._h, gid.value, int(period)),
                        "spikegen period")
        return self._add("spikegen", n, N.F32, gid)

    def timed_array(self, gid: int, values, dt_array: float) -> None:
        """TimedArray input of a LIF, HH or Poisson group (the role of brian2cuda/timedarray.py):
        values (rows,) for the whole group or (rows, n) per neuron, each row held for
        dt_array seconds, the last row after the end.  LIF: volts added to El,
        dv/dt = (El + I(t) - v + ...)/taum; HH: amperes, Cm dv/dt = ... + I(t); Poisson: the
        rate in Hz (PoissonGroup(N, rates='ta(t)'))."""
        v = np.asarray(values, dtype=np.float64)
        v = np.ascontiguousarray(v[:, None] if v.ndim == 1 else v)
        if v.ndim != 2:
            raise ValueError("values must be (rows,) or (rows, n)")
        self._check(self._lib.b2b_timedarray(self._h, gid, _ptr(v), v.shape[0], v.shape[1],
                                             float(dt_array)), "timed_array")

    def poisson_input(self, gid: int, var: str, n: int, rate: float, weight: float) -> int:
        """PoissonInput(group, var, N=n, rate=rate, weight=weight): every step each neuron
        adds weight * Binomial(n, rate*dt) to v, ge or gi (synapses slot)."""
        pid = C.c_int32()
        self._check(self._lib.b2b_poisson_input(self._h, gid, N.VARS[var], int(n), float(rate),
                                                float(weight), C.byref(pid)), "poisson_input")
        return pid.value

    def group_size(self, gid: int) -> int:
        return self._groups[gid][1]

    def _var_dtype(self, gid: int, var: str):
        return np.uint8 if var == "not_refractory" else _np_dtype(self._groups[gid][2])

    def set_state(self, gid: int, var: str, values):
        n = self.group_size(gid)
        a = np.ascontiguousarray(np.broadcast_to(values, (n,)), dtype=self._var_dtype(gid, var))
        self._check(self._lib.b2b_state_set(self._h, gid, N.VARS[var], _ptr(a), n),
                    f"set {var}")

    def get_state(self, gid: int, var: str) -> np.ndarray:
        n = self.group_size(gid)
        a = np.empty(n, dtype=self._var_dtype(gid, var))
        self._check(self._lib.b2b_state_get(self._h, gid, N.VARS[var], _ptr(a), n),
                    f"get {var}")
        return a

    def state_ptr(self, gid: int, var: str) -> int:
        p = C.c_void_p()
        n = C.c_int64()
        self._check(self._lib.b2b_state_ptr(self._h, gid, N.VARS[var], C.byref(p), C.byref(n)),
                    "state_ptr")
        return p.value

    # -- synapses -------------------------------------------------------------------------------
    def synapses(self, pre: int, post: int, target: str, i, j, w=None, w_scalar: float = 0.0,
                 delay=0, stdp: STDP | None = None) -> int:
        i = np.ascontiguousarray(i, dtype=np.int32)
        j = np.ascontiguousarray(j, dtype=np.int32)
        code = self._groups[post][2]
        wa = None if w is None else np.ascontiguousarray(w, dtype=_np_dtype(code))
        if np.ndim(delay) == 0:
            da, dscalar = None, int(delay)
        else:
            da, dscalar = np.ascontiguousarray(delay, dtype=np.int32), 0
        sp = stdp.to_c() if stdp is not None else None
        sid = C.c_int32()
        effect = N.EFFECT_STDP if stdp is not None else N.EFFECT_ADD
        self._check(self._lib.b2b_synapses(self._h, pre, post, N.VARS[target], effect, len(i),
                                           _ptr(i), _ptr(j), _ptr(wa), float(w_scalar),
                                           _ptr(da), dscalar,
                                           C.byref(sp) if sp is not None else None,
                                           C.byref(sid)), "synapses")
        self._syns.append((pre, post, code))
        return sid.value

    def synapses_random(self, pre: int, post: int, target: str, p: float, dmin: int, dmax: int,
                        w: float, seed: int, pre_range: tuple[int, int] | None = None) -> int:
        """Brian2 `Synapses(P[lo:hi], Q).connect(p=p)` generated on the GPU; delays uniform
        on the integers [dmin, dmax] (steps)."""
        lo, hi = pre_range if pre_range is not None else (0, self.group_size(pre))
        sid = C.c_int32()
        self._check(self._lib.b2b_synapses_random(self._h, pre, int(lo), int(hi), post,
                                                  N.VARS[target], float(p), int(dmin), int(dmax),
                                                  float(w), int(seed), C.byref(sid)),
                    "synapses_random")
        self._syns.append((pre, post, self._groups[post][2]))
        return sid.value

    def out_degree(self, gid: int) -> np.ndarray:
        """Outgoing synapses of every neuron of the group, over all its Synapses objects."""
        n = self.group_size(gid)
        a = np.empty(n, dtype=np.int32)
        self._check(self._lib.b2b_out_degree(self._h, gid, _ptr(a), n), "out_degree")
        return a

    def syn_set_delays(self, sid: int, delay_steps) -> None:
        """Brian2's `S.delay = ...` between runs: new per-synapse delays (steps, in the order
        the synapses were given); spikes already sent keep the delay they were sent with."""
        d = np.ascontiguousarray(delay_steps, dtype=np.int32)
        self._check(self._lib.b2b_syn_set_delays(self._h, sid, _ptr(d), len(d)),
                    "syn_set_delays")

    def syn_count(self, sid: int) -> int:
        n = C.c_int64()
        self._check(self._lib.b2b_syn_count(self._h, sid, C.byref(n)), "syn_count")
        return n.value

    def syn_get(self, sid: int, var: str) -> np.ndarray:
        n = self.syn_count(sid)
        dt = np.int32 if var in ("i", "j", "delay") else _np_dtype(self._syns[sid][2])
        a = np.empty(n, dtype=dt)
        self._check(self._lib.b2b_syn_get(self._h, sid, N.SYN_VARS[var], _ptr(a), n), "syn_get")
        return a

    # -- monitors and run -----------------------------------------------------------------------
    def spike_monitor(self, gid: int, capacity: int):
        self._check(self._lib.b2b_spikemon(self._h, gid, int(capacity)), "spikemon")

    def state_monitor(self, gid: int, var: str, indices=None, every: int = 1,
                      capacity: int = 0) -> int:
        """Brian2's StateMonitor(G, var, record=indices, dt=every*dt): records `var` of the
        given neurons (all when None) at the start of every step divisible by `every`, into
        a device buffer of `capacity` records.  Returns the monitor index."""
        n = self.group_size(gid)
        idx = (np.arange(n, dtype=np.int64) if indices is None
               else np.ascontiguousarray(indices, dtype=np.int64))
        mid = C.c_int32()
        self._check(self._lib.b2b_statemon(self._h, gid, N.VARS[var],
                                           idx.ctypes.data_as(C.POINTER(C.c_int64)), len(idx),
                                           int(every), int(capacity), C.byref(mid)),
                    "statemon")
        self._smons[mid.value] = (len(idx), self._var_dtype(gid, var))
        return mid.value

    def state_values(self, mid: int) -> tuple[np.ndarray, np.ndarray]:
        """(steps, values[records, indices]) a state monitor has recorded so far."""
        width, dt = self._smons[mid]
        n = C.c_int64()
        self._check(self._lib.b2b_statemon_get(self._h, mid, C.byref(n), None, None, 0),
                    "statemon_get")
        steps = np.empty(n.value, dtype=np.int64)
        vals = np.empty((n.value, width), dtype=dt)
        self._check(self._lib.b2b_statemon_get(
            self._h, mid, C.byref(n), steps.ctypes.data_as(C.POINTER(C.c_int64)),
            _ptr(vals), len(steps)), "statemon_get")
        return steps, vals

    def rate_monitor(self, gid: int, capacity: int) -> int:
        """Brian2's PopulationRateMonitor(G): the group's spike count of every step (rate =
        count / (N dt)), into a device buffer of `capacity` records."""
        mid = C.c_int32()
        self._check(self._lib.b2b_ratemon(self._h, gid, int(capacity), C.byref(mid)), "ratemon")
        return mid.value

    def rate_counts(self, mid: int) -> tuple[np.ndarray, np.ndarray]:
        """(steps, spike counts) a rate monitor has recorded so far."""
        n = C.c_int64()
        self._check(self._lib.b2b_ratemon_get(self._h, mid, C.byref(n), None, None, 0),
                    "ratemon_get")
        steps = np.empty(n.value, dtype=np.int64)
        counts = np.empty(n.value, dtype=np.int32)
        self._check(self._lib.b2b_ratemon_get(
            self._h, mid, C.byref(n), steps.ctypes.data_as(C.POINTER(C.c_int64)),
            counts.ctypes.data_as(C.POINTER(C.c_int32)), len(steps)), "ratemon_get")
        return steps, counts

    def finalize(self):
        self._check(self._lib.b2b_finalize(self._h), "finalize")

    def run(self, steps: int):
        self._check(self._lib.b2b_run(self._h, int(steps)), "run")

    def sync(self) -> int:
        s = C.c_int32()
        self._check(self._lib.b2b_sync(self._h, C.byref(s)), "sync")
        return s.value

    def store(self, slot: int = 0):
        """Device-side checkpoint of the dynamic state (Brian2's Network.store)."""
        self._check(self._lib.b2b_store(self._h, int(slot)), "store")

    def restore(self, slot: int = 0):
        """Restores a checkpoint taken with store() (Brian2's Network.restore)."""
        self._check(self._lib.b2b_restore(self._h, int(slot)), "restore")

    @property
    def timestep(self) -> int:
        ts = C.c_int64()
        self._lib.b2b_time(self._h, C.byref(ts), None)
        return ts.value

    @property
    def t(self) -> float:
        """Time of the next step in seconds (Brian2's net.t / defaultclock.t after a run)."""
        t = C.c_double()
        self._lib.b2b_time(self._h, None, C.byref(t))
        return t.value

    @property
    def run_mode(self) -> str:
        """'two-launch' (two concurrent launches per step), 'one-launch' (both halves of a
        step in one launch), 'small' (one CTA runs every step of a chunk) or 'per-step'
        (graph-replayed kernels)."""
        m = C.c_int32()
        self._check(self._lib.b2b_run_mode(self._h, C.byref(m)), "run_mode")
        return {1: "two-launch", 2: "small", 3: "one-launch"}.get(m.value, "per-step")

    @property
    def kernel_launches(self) -> int:
        n = C.c_int64()
        self._check(self._lib.b2b_kernel_launches(self._h, C.byref(n)), "launches")
        return n.value

    def profile(self, steps: int) -> list[tuple[int, float]]:
        """Advances `steps` steps with every launch timed; returns (site kind, mean ms) per
        launch site (1 population, 6 additive on_pre delivery launch, 2 STDP on_pre delivery,
        3 on_post delivery, 4 late reset, 5 delivery into the pending input of the two-launch
        step, 7 one-CTA step, 9 state monitors, 10 rate monitors)."""
        cap = 256
        ms = (C.c_double * cap)()
        kinds = (C.c_int32 * cap)()
        n = C.c_int32()
        self._check(self._lib.b2b_profile(self._h, int(steps), ms, kinds, cap, C.byref(n)),
                    "profile")
        return [(kinds[k], ms[k]) for k in range(n.value)]

    def profile_graph(self, steps: int) -> tuple[list[tuple[int, float]], float]:
        """Advances `steps` steps (a multiple of steps_per_graph) by replaying step graphs
        that carry an event-record node before and after every launch site; returns
        ((site kind, mean ms per simulated step inside the graphs) per site, mean ms of one
        whole step).  Same sites as profile()."""
        cap = 256
        ms = (C.c_double * cap)()
        kinds = (C.c_int32 * cap)()
        n = C.c_int32()
        step = C.c_double()
        self._check(self._lib.b2b_profile_graph(self._h, int(steps), ms, kinds, cap, C.byref(n),
                                                C.byref(step)), "profile_graph")
        return [(kinds[k], ms[k]) for k in range(n.value)], step.value

    def autotune(self, trial_steps: int = 50) -> list[dict]:
        """Times candidate launch shapes of every launch site on the current state and keeps
        the fastest (state, clock and monitors are left as they were)."""
        cap = 256
        res = (N.TuneResult * cap)()
        n = C.c_int32()
        self._check(self._lib.b2b_autotune(self._h, int(trial_steps), res, cap, C.byref(n)),
                    "autotune")
        return [{"site_kind": r.site_kind, "site_index": r.site_index, "choice_a": r.choice_a,
                 "choice_b": r.choice_b, "best_ms": r.best_ms, "default_ms": r.default_ms}
                for r in res[: n.value]]

    def tune_apply(self, results: list[dict]):
        """Applies the launch shapes of an earlier autotune() of a net built the same way."""
        arr = (N.TuneResult * max(1, len(results)))()
        for k, r in enumerate(results):
            arr[k] = N.TuneResult(r["site_kind"], r["site_index"], r["choice_a"], r["choice_b"],
                                  r.get("best_ms", 0.0), r.get("default_ms", 0.0))
        self._check(self._lib.b2b_tune_apply(self._h, arr, len(results)), "tune_apply")

    def spikes(self, gid: int, sub: tuple[int, int] | None = None
               ) -> tuple[np.ndarray, np.ndarray]:
        """All recorded spikes of a monitored group as (indices, steps), sorted by step; with
        sub = (lo, hi), those of the subgroup G[lo:hi] with indices relative to lo."""
        lo, hi = sub if sub is not None else (0, self.group_size(gid))
        n = C.c_int64()
        self._check(self._lib.b2b_spikemon_get_range(self._h, gid, lo, hi, C.byref(n), None,
                                                     None, 0), "spikemon_get")
        idx = np.empty(n.value, dtype=np.int32)
        stp = np.empty(n.value, dtype=np.int64)
        self._check(self._lib.b2b_spikemon_get_range(self._h, gid, lo, hi, C.byref(n),
                                                     _ptr(idx), _ptr(stp), len(idx)),
                    "spikemon_get")
        return idx, stp

    def spikes_fetch(self, gid: int, start: int, cap: int = 1 << 22):
        """Recorded spikes from monitor entry `start` on, in recording order; returns
        (indices, steps, next_start)."""
        total, n = C.c_int64(), C.c_int64()
        m = max(1, min(int(cap), self.spikes_recorded(gid) - int(start)))
        idx = np.empty(m, dtype=np.int32)
        stp = np.empty(m, dtype=np.int64)
        self._check(self._lib.b2b_spikemon_fetch(self._h, gid, int(start), C.byref(total),
                                                 C.byref(n), _ptr(idx), _ptr(stp), m),
                    "spikemon_fetch")
        nxt = min(total.value, int(start) + cap)
        return idx[: n.value], stp[: n.value], nxt

    def spikes_fetch_population(self, gid: int, start: int, cap: int = 1 << 24):
        """Like spikes_fetch, for every monitored group of gid's population at once, with
        population indices (see group_offset)."""
        total, n = C.c_int64(), C.c_int64()
        m = max(1, min(int(cap), self.spikes_recorded(gid) - int(start)))
        idx = np.empty(m, dtype=np.int32)
        stp = np.empty(m, dtype=np.int64)
        self._check(self._lib.b2b_spikemon_fetch_population(
            self._h, gid, int(start), C.byref(total), C.byref(n), _ptr(idx), _ptr(stp), m),
            "spikemon_fetch_population")
        nxt = min(total.value, int(start) + cap)
        return idx[: n.value], stp[: n.value], nxt

    def group_offset(self, gid: int) -> int:
        """Index of the group's first neuron in its population."""
        o = C.c_int64()
        self._check(self._lib.b2b_group_offset(self._h, gid, C.byref(o)), "group_offset")
        return o.value

    def spikes_recorded(self, gid: int) -> int:
        """Number of entries the monitor of gid's population has recorded so far."""
        total, n = C.c_int64(), C.c_int64()
        self._check(self._lib.b2b_spikemon_fetch(self._h, gid, 0, C.byref(total), C.byref(n),
                                                 None, None, 0), "spikemon_fetch")
        return total.value

    def spikes_last(self, gid: int) -> np.ndarray:
        n = C.c_int64()
        cap = self.group_size(gid)
        idx = np.empty(cap, dtype=np.int32)
        self._check(self._lib.b2b_spikes_last(self._h, gid, C.byref(n), _ptr(idx), cap),
                    "spikes_last")
        return idx[: n.value].copy()

    def queue(self, sid: int) -> np.ndarray:
        """Delay-queue contents as rows (offset, pre, delay), sorted."""
        n = C.c_int64()
        self._check(self._lib.b2b_queue_get(self._h, sid, C.byref(n), None, None, None, 0),
                    "queue")
        a, p, d = (np.empty(n.value, dtype=np.int32) for _ in range(3))
        self._check(self._lib.b2b_queue_get(self._h, sid, C.byref(n), _ptr(a), _ptr(p), _ptr(d),
                                            n.value), "queue")
        return np.stack([a, p, d], axis=1) if n.value else np.zeros((0, 3), np.int32)

    def rng_uniforms(self, gid: int, steps: int) -> np.ndarray:
        n = self.group_size(gid)
        a = np.empty((steps, n), dtype=_np_dtype(self._groups[gid][2]))
        self._check(self._lib.b2b_rng_uniforms_get(self._h, gid, _ptr(a), steps, n), "rng")
        return a

    def rng_normals(self, gid: int, steps: int, n_normal: int) -> np.ndarray:
        """Normal numbers the last run chunk drew for a generated-model group: (steps,
        n_normal * size), draw d of neuron i at [:, d * size + i]."""
        n = n_normal * self.group_size(gid)
        a = np.empty((steps, n), dtype=_np_dtype(self._groups[gid][2]))
        self._check(self._lib.b2b_rng_normals_get(self._h, gid, _ptr(a), steps, n),
                    "rng_normals")
        return a

    def model_group(self, n: int, model, dtype="float64") -> int:
        """A group integrated by a generated model (codegen.GeneratedModel): its source is
        compiled for sm_100a once (cached by content) and the shared object is loaded into
        the net (b2b_group_model)."""
        from .codegen import compile_model
        if model.path is None:
            model.path = compile_model(model.source)
        gid = C.c_int32()
        code = _dt_code(dtype)
        self._check(self._lib.b2b_group_model(self._h, int(n), code, model.path.encode(),
                                              float(model.refractory), C.byref(gid)), "model")
        return self._add("model", n, code, gid)

    # -- multicompartment batch -----------------------------------------------------------------
    def hines_batch(self, comp_off, sec_off, sec_start, sec_end, sec_parent, diameter, length,
                    params: HinesParams) -> "HinesBatch":
        hb = HinesBatch(self, comp_off, sec_off, sec_start, sec_end, sec_parent, diameter,
                        length, params)
        self._hines.append(hb)
        return hb


class HinesBatch:
    """A batch of independent multicompartment HH neurons advanced by one kernel launch."""

    def __init__(self, net: Network, comp_off, sec_off, sec_start, sec_end, sec_parent,
                 diameter, length, params: HinesParams):
        self._net = net
        self._lib = net._lib
        self.comp_off = np.ascontiguousarray(comp_off, dtype=np.int64)
        self.n_neurons = len(self.comp_off) - 1
        self.n_comp = int(self.comp_off[-1])
        arrs = [np.ascontiguousarray(a, dtype=np.int32)
                for a in (sec_off, sec_start, sec_end, sec_parent)]
        d = np.ascontiguousarray(diameter, dtype=np.float64)
        L = np.ascontiguousarray(length, dtype=np.float64)
        self._keep = arrs + [d, L]
        self.channel_dtype = np.float32 if params.channel_dtype in ("float32", np.float32) \
            else np.float64
        p = params.to_c()
        h = C.c_void_p()
        net._check(self._lib.b2b_hines_create(net._h, self.n_neurons, _ptr(self.comp_off),
                                              *[_ptr(a) for a in arrs], _ptr(d), _ptr(L),
                                              C.byref(p), C.byref(h)), "hines_create")
        self._h = h

    def _dtype(self, var: str):
        return np.float64 if var in ("v", "Ic") else self.channel_dtype

    def set_current(self, soma_current):
        a = None if soma_current is None else np.ascontiguousarray(soma_current, np.float64)
        self._net._check(self._lib.b2b_hines_set_current(self._h, _ptr(a)), "hines_current")

    def set_state(self, var: str, values):
        a = np.ascontiguousarray(np.broadcast_to(values, (self.n_comp,)), dtype=self._dtype(var))
        self._net._check(self._lib.b2b_hines_state_set(self._h, N.HINES_VARS[var], _ptr(a),
                                                       self.n_comp), "hines_set")

    def get_state(self, var: str) -> np.ndarray:
        a = np.empty(self.n_comp, dtype=self._dtype(var))
        self._net._check(self._lib.b2b_hines_state_get(self._h, N.HINES_VARS[var], _ptr(a),
                                                       self.n_comp), "hines_get")
        return a

    def run(self, steps: int):
        self._net._check(self._lib.b2b_hines_run(self._h, int(steps)), "hines_run")

    def spike_counts(self) -> np.ndarray:
        a = np.empty(self.n_neurons, dtype=np.int32)
        self._net._check(self._lib.b2b_hines_spike_counts(self._h, _ptr(a), self.n_neurons),
                         "hines_spikes")
        return a
