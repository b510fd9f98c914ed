"""The benchmark networks written the way a Brian2 script writes them (model strings,
namespaces, connect, monitors, run) on the `lowering.Script` front end, so that they run
unchanged on the GPU library and on the CPU oracle.

  * cuba      — the CUBA network of the reference's examples/cuba.py (exact integration)
  * cobahh    — the COBAHH network of examples/cobahh.py (exponential Euler), with the
                per-synapse delays of the benchmark configuration
  * stdp      — 1e4 Poisson inputs onto 1e3 LIF neurons with event-driven additive STDP
                (examples/stdp.py, brian2cuda/tests/features/speed.py:627-663)
  * batched   — independent COBAHH instances of uneven sizes in one script
Units are SI; the unit names inside the strings are resolved by brian2cuda_b200.equations.
"""
from __future__ import annotations

import numpy as np

from .lowering import Script, UniformDelaySteps
from .models import SEED_BASE, batch_sizes

mV, ms, nS, um, Hz = 1e-3, 1e-3, 1e-9, 1e-6, 1.0

CUBA_EQS = """
dv/dt  = (ge + gi - (v - El)) / taum : volt (unless refractory)
dge/dt = -ge / taue : volt
dgi/dt = -gi / taui : volt
"""

COBAHH_EQS = """
dv/dt = (gl*(El - v) + ge*(Ee - v) + gi*(Ei - v)
         - g_na*(m*m*m)*h*(v - ENa) - g_kd*(n*n*n*n)*(v - EK))/Cm : volt
dm/dt = alpha_m*(1 - m) - beta_m*m : 1
dn/dt = alpha_n*(1 - n) - beta_n*n : 1
dh/dt = alpha_h*(1 - h) - beta_h*h : 1
dge/dt = -ge*(1./taue) : siemens
dgi/dt = -gi*(1./taui) : siemens
alpha_m = 0.32*(mV**-1)*(13.*mV - v + VT)/(exp((13.*mV - v + VT)/(4.*mV)) - 1.)/ms : Hz
beta_m = 0.28*(mV**-1)*(v - VT - 40.*mV)/(exp((v - VT - 40.*mV)/(5.*mV)) - 1.)/ms : Hz
alpha_h = 0.128*exp((17.*mV - v + VT)/(18.*mV))/ms : Hz
beta_h = 4./(1. + exp((40.*mV - v + VT)/(5.*mV)))/ms : Hz
alpha_n = 0.032*(mV**-1)*(15.*mV - v + VT)/(exp((15.*mV - v + VT)/(5.*mV)) - 1.)/ms : Hz
beta_n = .5*exp((10.*mV - v + VT)/(40.*mV))/ms : Hz
"""


def cobahh_namespace() -> dict:
    area = 20000 * um * um
    return dict(area=area, Cm=1e-2 * area, gl=5e-5 * 1e4 * area, El=-60 * mV, EK=-90 * mV,
                ENa=50 * mV, g_na=100e-3 * 1e4 * area, g_kd=30e-3 * 1e4 * area, VT=-63 * mV,
                taue=5 * ms, taui=10 * ms, Ee=0 * mV, Ei=-80 * mV)


def cuba(N: int = 4000, duration: float = 1.0, dtype: str = "float64", p: float = 0.02,
         seed: int = SEED_BASE) -> tuple[Script, dict]:
    s = Script(dt=0.1 * ms, seed=seed, dtype=dtype,
               namespace=dict(taum=20 * ms, taue=5 * ms, taui=10 * ms, Vt=-50 * mV,
                              Vr=-60 * mV, El=-49 * mV, Ne=int(0.8 * N)))
    P = s.NeuronGroup(N, CUBA_EQS, threshold="v > Vt", reset="v = Vr", refractory=5 * ms,
                      method="exact")
    P.v = "Vr + rand() * (Vt - Vr)"
    P.ge = 0.0
    P.gi = 0.0
    Ce = s.Synapses(P, P, on_pre="ge += we", namespace={"we": (60 * 0.27 / 10) * mV})
    Ci = s.Synapses(P, P, on_pre="gi += wi", namespace={"wi": (-20 * 4.5 / 10) * mV})
    Ce.connect("i < Ne", p=p)
    Ci.connect("i >= Ne", p=p)
    mon = s.SpikeMonitor(P, name="spikes")
    s.run(duration)
    return s, {"P": P, "Ce": Ce, "Ci": Ci, "spikes": mon}


def cobahh(N: int = 100_000, duration: float = 1.0, dtype: str = "float32", p: float = 0.02,
           dmin: int = 1, dmax: int = 50, seed: int = SEED_BASE + 1) -> tuple[Script, dict]:
    ns = cobahh_namespace()
    ns["Ne"] = int(0.8 * N)
    s = Script(dt=0.1 * ms, seed=seed, dtype=dtype, namespace=ns)
    P = s.NeuronGroup(N, COBAHH_EQS, threshold="v > -20*mV", refractory=3 * ms,
                      method="exponential_euler")
    Ce = s.Synapses(P[:int(0.8 * N)], P, on_pre="ge += we", namespace={"we": 6 * nS})
    Ci = s.Synapses(P[int(0.8 * N):], P, on_pre="gi += wi", namespace={"wi": 67 * nS})
    Ce.connect(p=p)
    Ci.connect(p=p)
    Ce.delay = UniformDelaySteps(dmin, dmax)
    Ci.delay = UniformDelaySteps(dmin, dmax)
    P.v = "El + 5*mV*randn()"
    P.ge = "(randn() * 1.5 + 4) * 10.*nS"
    P.gi = "(randn() * 12 + 20) * 10.*nS"
    mon = s.SpikeMonitor(P, name="spikes")
    s.run(duration)
    return s, {"P": P, "Ce": Ce, "Ci": Ci, "spikes": mon}


def stdp(n_in: int = 10_000, n_out: int = 1_000, rate: float = 15.0, duration: float = 1.0,
         dtype: str = "float32", seed: int = SEED_BASE + 2) -> tuple[Script, dict]:
    gmax = 0.01
    taupre = taupost = 20 * ms
    dApre = 0.01 * gmax
    ns = dict(taum=10 * ms, taue=5 * ms, Ee=0 * mV, vt=-54 * mV, vr=-60 * mV, El=-74 * mV,
              taupre=taupre, taupost=taupost, gmax=gmax, dApre=dApre,
              dApost=-dApre * taupre / taupost * 1.05)
    s = Script(dt=0.1 * ms, seed=seed, dtype=dtype, namespace=ns)
    inp = s.PoissonGroup(n_in, rates=rate * Hz)
    out = s.NeuronGroup(n_out, """dv/dt = (ge * (Ee - vr) + El - v) / taum : volt
                                  dge/dt = -ge / taue : 1""",
                        threshold="v > vt", reset="v = vr", method="exact")
    out.v = "vr"
    S = s.Synapses(inp, out,
                   """w : 1
                      dApre/dt = -Apre / taupre : 1 (event-driven)
                      dApost/dt = -Apost / taupost : 1 (event-driven)""",
                   on_pre="""ge += w
                             Apre += dApre
                             w = clip(w + Apost, 0, gmax)""",
                   on_post="""Apost += dApost
                              w = clip(w + Apre, 0, gmax)""")
    S.connect()
    S.w = "rand() * gmax"
    m_in = s.SpikeMonitor(inp, name="input_spikes")
    m_out = s.SpikeMonitor(out, name="output_spikes")
    s.run(duration)
    return s, {"input": inp, "neurons": out, "S": S, "input_spikes": m_in,
               "output_spikes": m_out}


def batched(n_instances: int = 256, duration: float = 0.1, dtype: str = "float32",
            instances=None, seed: int = SEED_BASE + 5) -> tuple[Script, dict]:
    """Independent COBAHH instances (sizes log-uniform on [1e3, 6.4e4], excitatory weight
    uniform on [4, 8] nS) in one script: the backend merges them into one population and one
    projection.  `instances` restricts the script to some of them."""
    sizes, we = batch_sizes(n_instances)
    keep = range(n_instances) if instances is None else instances
    s = Script(dt=0.1 * ms, seed=seed, dtype=dtype, namespace=cobahh_namespace())
    groups = []
    for k in keep:
        n = int(sizes[k])
        ne = int(0.8 * n)
        P = s.NeuronGroup(n, COBAHH_EQS, threshold="v > -20*mV", refractory=3 * ms,
                          method="exponential_euler", name=f"instance_{k}")
        Ce = s.Synapses(P[:ne], P, on_pre="ge += we", namespace={"we": float(we[k])})
        Ci = s.Synapses(P[ne:], P, on_pre="gi += wi", namespace={"wi": 67 * nS})
        Ce.connect(p=0.02)
        Ci.connect(p=0.02)
        Ce.delay = UniformDelaySteps(1, 50)
        Ci.delay = UniformDelaySteps(1, 50)
        P.v = "El + 5*mV*randn()"
        P.ge = "(randn() * 1.5 + 4) * 10.*nS"
        P.gi = "(randn() * 12 + 20) * 10.*nS"
        s.SpikeMonitor(P, name=f"spikes_{k}")
        groups.append(P)
    s.run(duration)
    return s, {"groups": groups, "sizes": np.asarray([sizes[k] for k in keep])}
