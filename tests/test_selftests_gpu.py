"""Device-side building blocks checked directly on the GPU: the bounded mbarrier wait gives
up after its poll limit and reports B2B_ERR_TIMEOUT through the status word (nothing faults,
nothing hangs: no MMA is in flight and nothing else waits), and the multicompartment
solver's reciprocal stays within two ulps of the IEEE quotient over the whole range of
pivots and node coefficients, extremes included."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_reports_timeout():
    from brian2cuda_b200 import _native
    lib = _native.lib()
    st = C.c_int32(-1)
    assert lib.b2b_wait_selftest(0, None, 4, 0, C.byref(st)) == 0
    assert st.value == 4                 # B2B_ERR_TIMEOUT
    # the control: thread 0 arrives first, the wait completes within the same limit
    st = C.c_int32(-1)
    assert lib.b2b_wait_selftest(0, None, 4, 1, C.byref(st)) == 0
    assert st.value == 0
    # the context is still usable afterwards
    import torch
    x = torch.arange(8, device="cuda", dtype=torch.float32)
    assert float(x.sum().item()) == 28.0


def test_atomic_rate_probe_measures_three_forms():
    """The delivery's ceiling probe returns positive rates for the L2 forms and the cluster
    form (2e5 targets: 100 KB slices of an 8-CTA cluster), and every form's additions land
    (a form that skipped its work would read far above the others)."""
    from brian2cuda_b200.network import atomic_rate
    loaded, hashed, dsmem = atomic_rate(200_000, 20_000_000, reps=2)
    assert loaded > 1e9 and hashed > 1e9 and dsmem > 1e9
    assert hashed < 1e13 and dsmem < 1e13


def test_solver_reciprocal_within_two_ulps():
    from brian2cuda_b200 import _native
    lib = _native.lib()
    rng = np.random.default_rng(0)
    mags = np.concatenate([
        10.0 ** rng.uniform(-300, 300, 200_000),        # the normal range
        10.0 ** rng.uniform(-12, 12, 200_000),          # conductances, areas, pivots
        np.array([1.0, 2.0, 3.0, 0.5, 1e-300, 1e300, 2.2250738585072014e-308 * 4,
                  np.nextafter(1.0, 2.0), np.nextafter(1.0, 0.0)])])
    x = np.concatenate([mags, -mags])
    y = np.empty_like(x)
    assert lib.b2b_recip_selftest(0, x.ctypes.data_as(C.c_void_p),
                                  y.ctypes.data_as(C.c_void_p), len(x)) == 0
    ref = 1.0 / x
    ulp = np.abs(np.spacing(ref))
    err = np.abs(y - ref) / ulp
    assert np.all(np.isfinite(y))
    assert err.max() <= 2.0, float(err.max())
