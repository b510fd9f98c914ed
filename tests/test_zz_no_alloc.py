"""b2b_connect_random_static: the allocation-free connectivity generator.

Some callers of this library cannot allocate device memory: applications whose device memory
belongs to a pooling allocator, and host loops that cannot afford the device-wide
synchronisation of cudaMalloc.  This entry point keeps its scratch in a static device array
instead.  The test calls it twice in a row through the C ABI
and compares each result with the generator behind b2b_synapses_random (the existing entry
point), which numbers synapses in (i, delay, j) order while this one writes (i, j) order.
This file sorts last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference(pre_range, n_pre, n_post, p, dmin, dmax, seed):
    from brian2cuda_b200 import Network, models
    net = Network(1e-4)
    A = net.lif_group(n_pre, models.cuba_lif(), "float32")
    B = net.lif_group(n_post, models.cuba_lif(), "float32")
    sid = net.synapses_random(A, B, "ge", p, dmin, dmax, 1e-3, seed, pre_range=pre_range)
    net.finalize()
    out = tuple(net.syn_get(sid, v) for v in ("i", "j", "delay"))
    net.close()
    return out


def _static(lib, torch, pre_range, n_post, p, dmin, dmax, seed, capacity, alloc=None):
    dev = torch.cuda.current_device()
    stream = torch.cuda.current_stream()
    size = capacity if alloc is None else alloc
    bufs = [torch.full((size,), -1, dtype=torch.int32, device="cuda") for _ in range(3)]
    n = C.c_int64(-1)
    st = lib.b2b_connect_random_static(dev, C.c_void_p(stream.cuda_stream), pre_range[0],
                                       pre_range[1], n_post, p, dmin, dmax, seed,
                                       C.c_void_p(bufs[0].data_ptr()),
                                       C.c_void_p(bufs[1].data_ptr()),
                                       C.c_void_p(bufs[2].data_ptr()), capacity, C.byref(n))
    return st, n.value, [b.cpu().numpy() for b in bufs]


@pytest.mark.parametrize("case", [
    ((0, 900), 900, 1300, 0.03, 1, 50, 20261204),
    ((250, 700), 900, 517, 0.1, 3, 3, 77),
])
def test_static_generator_matches_existing_two_calls(case):
    import torch

    from brian2cuda_b200 import _native
    lib = _native.lib()
    pre_range, n_pre, n_post, p, dmin, dmax, seed = case
    ri, rj, rd = _reference(pre_range, n_pre, n_post, p, dmin, dmax, seed)
    for _call in range(2):
        st, n, (i, j, d) = _static(lib, torch, pre_range, n_post, p, dmin, dmax, seed,
                                   capacity=len(ri) + 100)
        assert st == 0 and n == len(ri)
        i, j, d = i[:n], j[:n], d[:n]
        order = np.lexsort((j, d, i))          # renumber (i, j) order as (i, delay, j)
        np.testing.assert_array_equal(i[order], ri)
        np.testing.assert_array_equal(j[order], rj)
        np.testing.assert_array_equal(d[order], rd)
        assert (np.diff(i) >= 0).all()


def test_static_generator_limits():
    import torch

    from brian2cuda_b200 import _native
    lib = _native.lib()
    # more rows than the static scratch holds: rejected before any device work
    st, _, _ = _static(lib, torch, (0, (1 << 20) + 1), 10, 0.1, 1, 2, 1, capacity=16)
    assert st == 1
    # too small an output: the count comes back with B2B_ERR_QUEUE_OVERFLOW, the first
    # `capacity` synapses in (i, j) order are written and nothing beyond them
    cap = 64
    st, n, (i, j, d) = _static(lib, torch, (0, 200), 200, 0.5, 1, 2, 5, capacity=cap,
                               alloc=4 * cap)
    assert st == 3 and n > cap
    ri, rj, rd = _reference((0, 200), 200, 200, 0.5, 1, 2, 5)
    assert len(ri) == n
    order = np.lexsort((rj, ri))              # the existing entry point's synapses in (i, j) order
    np.testing.assert_array_equal(i[:cap], ri[order][:cap])
    np.testing.assert_array_equal(j[:cap], rj[order][:cap])
    np.testing.assert_array_equal(d[:cap], rd[order][:cap])
    for a in (i, j, d):
        assert (a[cap:] == -1).all()
