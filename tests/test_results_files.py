"""Brian2 result files (the arrays brian2cuda's _write_arrays writes,
brian2cuda/templates/objects.cu:522-641): written from a network's monitors and read back
with the dtypes and layouts Brian2 loads them with.  Runs on the CPU oracle (the writer only
uses the Network interface, which the CUDA library shares)."""
from __future__ import annotations

import math

import numpy as np

from brian2cuda_b200.network import LIF
from brian2cuda_b200.results import (rate_monitor_arrays, spike_monitor_arrays,
                                     state_monitor_arrays, write_results)

DT = 1e-4


def test_monitor_arrays_round_trip(oracle_factory, tmp_path):
    net = oracle_factory(DT)
    G = net.lif_group(6, LIF(taum=math.inf, Vt=0.5, has_reset=False), "float64")
    net.set_state(G, "v", np.array([1, 0, 0, 0, 1, 1], dtype=np.float64))
    net.spike_monitor(G, 100)
    sm = net.state_monitor(G, "v", indices=[0, 3], capacity=10)
    rm = net.rate_monitor(G, 10)
    net.finalize()
    net.run(3)
    files = {}
    for k, a in spike_monitor_arrays(net, G, DT).items():
        files[f"_dynamic_array_spikemonitor_{k}"] = a
    for k, a in spike_monitor_arrays(net, G, DT, sub=(4, 6)).items():
        files[f"_dynamic_array_spikemonitor_1_{k}"] = a
    for k, a in state_monitor_arrays(net, sm, "v", DT).items():
        files[f"_dynamic_array_statemonitor_{k}"] = a
    for k, a in rate_monitor_arrays(net, rm, 6, DT).items():
        files[f"_dynamic_array_ratemonitor_{k}"] = a
    write_results(str(tmp_path), files, run_time=0.25)

    def load(name, dtype):
        return np.fromfile(tmp_path / name, dtype=dtype)
    # neurons 0, 4, 5 spike in each of the three steps (no reset)
    np.testing.assert_array_equal(load("_dynamic_array_spikemonitor_i", np.int32),
                                  [0, 4, 5] * 3)
    np.testing.assert_allclose(load("_dynamic_array_spikemonitor_t", np.float64),
                               np.repeat([0.0, DT, 2 * DT], 3))
    np.testing.assert_array_equal(load("_dynamic_array_spikemonitor_count", np.int32),
                                  [3, 0, 0, 0, 3, 3])
    np.testing.assert_array_equal(load("_dynamic_array_spikemonitor_N", np.int32), [9])
    np.testing.assert_array_equal(load("_dynamic_array_spikemonitor_1_i", np.int32),
                                  [0, 1] * 3)
    np.testing.assert_array_equal(load("_dynamic_array_spikemonitor_1_count", np.int32), [3, 3])
    # the state monitor's values, record-major: [t][index]
    v = load("_dynamic_array_statemonitor_v", np.float64).reshape(3, 2)
    np.testing.assert_array_equal(v, [[1, 0]] * 3)
    np.testing.assert_allclose(load("_dynamic_array_statemonitor_t", np.float64),
                               [0.0, DT, 2 * DT])
    np.testing.assert_allclose(load("_dynamic_array_ratemonitor_rate", np.float64),
                               [3 / (6 * DT)] * 3)
    run_time, completed = open(tmp_path / "last_run_info.txt").read().split()
    assert float(run_time) == 0.25 and float(completed) == 1.0
