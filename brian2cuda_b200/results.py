"""Brian2 standalone result files from a network's monitors.

brian2cuda's generated `_write_arrays()` (brian2cuda/templates/objects.cu:522-641) writes
every array of the run into the results directory as raw binary, one file per array, named
by Brian2's device (`get_array_filename`), and `last_run_info.txt` with the last run's time
and completed fraction; Brian2 reads them back by name and dtype.  The names are the
caller's (the device that generated the code knows them); this module produces the arrays
of each monitor in Brian2's dtypes and layouts and writes them:

  SpikeMonitor:            i (int32), t (float64 s), count (int32 per neuron), N (int32)
  StateMonitor:            t (float64 s), <var> (float64, record-major [t][index], the
                           order objects.cu:598-604 writes)
  PopulationRateMonitor:   t (float64 s), rate (float64 Hz)

Works with any object of the Network interface (the CUDA library or the CPU oracle).
"""
from __future__ import annotations

import os

import numpy as np


def spike_monitor_arrays(net, gid: int, dt: float, sub: tuple[int, int] | None = None
                         ) -> dict[str, np.ndarray]:
    """Brian2's SpikeMonitor arrays of group gid (or of its subgroup sub = (lo, hi))."""
    idx, steps = net.spikes(gid, sub=sub) if sub is not None else net.spikes(gid)
    n = (sub[1] - sub[0]) if sub is not None else net.group_size(gid)
    return {"i": np.asarray(idx, dtype=np.int32),
            "t": np.asarray(steps, dtype=np.float64) * dt,
            "count": np.bincount(np.asarray(idx, dtype=np.int64), minlength=n).astype(np.int32),
            "N": np.array([len(idx)], dtype=np.int32)}


def state_monitor_arrays(net, mid: int, var: str, dt: float) -> dict[str, np.ndarray]:
    """Brian2's StateMonitor arrays: t and the recorded variable, record-major."""
    steps, vals = net.state_values(mid)
    return {"t": np.asarray(steps, dtype=np.float64) * dt,
            var: np.ascontiguousarray(vals, dtype=np.float64)}


def rate_monitor_arrays(net, mid: int, n_neurons: int, dt: float) -> dict[str, np.ndarray]:
    """Brian2's PopulationRateMonitor arrays: t and rate = count / (N dt) in Hz."""
    steps, counts = net.rate_counts(mid)
    return {"t": np.asarray(steps, dtype=np.float64) * dt,
            "rate": np.asarray(counts, dtype=np.float64) / (n_neurons * dt)}


def write_results(directory: str, files: dict[str, np.ndarray], run_time: float,
                  completed: float = 1.0) -> None:
    """Writes each array as raw binary (native byte order, C order) to directory/<name>,
    and last_run_info.txt as '<run_time> <completed>' (seconds of wall time of the last run
    and the fraction of it that completed)."""
    os.makedirs(directory, exist_ok=True)
    for name, arr in files.items():
        np.ascontiguousarray(arr).tofile(os.path.join(directory, name))
    with open(os.path.join(directory, "last_run_info.txt"), "w") as f:
        f.write(f"{run_time!r} {completed!r}\n")
