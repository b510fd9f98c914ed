"""Sharding of independent network instances over ranks (one process per GPU).

The batched workload (many independent COBAHH instances) partitions with no exchange at all:
every rank builds and simulates its own instances, and only the timing is reduced (max over
ranks).  Instances are assigned longest-processing-time first: by decreasing cost, each to
the rank with the least cost so far, which keeps the largest rank load within 4/3 of the
optimum.  The cost of an instance is its neuron count plus its expected synapse count (the
per-step work is a neuron update per neuron and a delivery per synaptic event, and events
scale with synapses at a given rate).
"""
from __future__ import annotations

import heapq

import numpy as np


def instance_cost(n_neurons, p_connect: float) -> np.ndarray:
    """Relative per-step cost of instances of n neurons connected with probability p."""
    n = np.asarray(n_neurons, dtype=np.float64)
    return n + p_connect * n * n


def lpt_partition(costs, n_parts: int) -> list[list[int]]:
    """Indices of `costs` split into n_parts lists, longest processing time first; each list
    is in increasing index order.  Deterministic (ties go to the lower rank)."""
    if n_parts < 1:
        raise ValueError("n_parts must be positive")
    costs = np.asarray(costs, dtype=np.float64)
    heap = [(0.0, r) for r in range(n_parts)]
    parts: list[list[int]] = [[] for _ in range(n_parts)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]
