"""The C ABI: libb2b.so loads and exports every function include/b2b.h declares, the ctypes
table covers them all, and creating a network without a usable GPU fails loudly."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "b2b.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(b2b_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "b2b_create" in names and "b2b_run" in names and "b2b_hines_run" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    from brian2cuda_b200 import _native
    lib = _native.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", _native.lib_path()],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (b2b_[a-z0-9_]+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing
    for n in declared():
        assert getattr(lib, n) is not None


def test_ctypes_table_matches_header():
    from brian2cuda_b200 import _native
    assert sorted(_native.PROTOTYPES) == declared()


def test_abi_version_and_status_strings():
    from brian2cuda_b200 import _native
    lib = _native.lib()
    assert lib.b2b_abi_version() == 1
    assert lib.b2b_status_string(0) == b"ok"
    assert lib.b2b_status_string(3) == b"device buffer overflow"


def test_null_arguments_are_rejected_without_touching_the_gpu():
    from brian2cuda_b200 import _native
    lib = _native.lib()
    assert lib.b2b_create(None, None) == 1
    assert lib.b2b_destroy(None) == 1
    assert lib.b2b_run(None, 1) == 1
    assert lib.b2b_hines_run(None, 1) == 1
    # the group inputs and monitor readers
    assert lib.b2b_timedarray(None, 0, None, 1, 1, 1e-4) == 1
    assert lib.b2b_poisson_input(None, 0, 0, 10, 5.0, 1.0, None) == 1
    assert lib.b2b_spikegen_period(None, 0, 10) == 1
    assert lib.b2b_spikemon_get_range(None, 0, 0, 1, None, None, None, 0) == 1


def test_spike_steps_bins_times_like_brian2_timestep():
    """Times become steps by timestep(t, dt) = int((t + 1e-3 dt) / dt): [k dt, (k+1) dt)
    lands in step k, and k*dt computed in floating point stays in step k."""
    import numpy as np
    from brian2cuda_b200.network import spike_steps
    dt = 1e-4
    k = np.arange(100000)
    np.testing.assert_array_equal(spike_steps(k * dt, dt), k)
    np.testing.assert_array_equal(spike_steps(np.linspace(0, dt, 100, endpoint=False), dt), 0)
    np.testing.assert_array_equal(spike_steps([0.5 * dt, 1.5 * dt, 2.9 * dt], dt), [0, 1, 2])


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_have_gpu(), reason="checks the behaviour on a machine without a GPU")
def test_network_without_gpu_raises():
    from brian2cuda_b200 import B2BError, Network
    with pytest.raises(B2BError):
        Network(1e-4)


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    from brian2cuda_b200 import _native
    monkeypatch.setattr(_native, "_LIB_PATH", str(tmp_path / "libb2b.so"))
    monkeypatch.setattr(_native, "_lib", None)
    with pytest.raises(ImportError):
        _native.lib()


def test_struct_layouts_match_c():
    from brian2cuda_b200 import _native as N
    assert ctypes.sizeof(N.Config) == 40
    assert ctypes.sizeof(N.LifParams) == 9 * 8 + 16
    assert ctypes.sizeof(N.HhParams) == 14 * 8
    assert ctypes.sizeof(N.StdpParams) == 6 * 8 + 8
    assert ctypes.sizeof(N.HinesParams) == 9 * 8 + 8
