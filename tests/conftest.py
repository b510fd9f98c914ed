"""Test configuration: the `gpu` marker, library builds, and backend factories.

CPU runs (`-m "not gpu"`) exercise the oracle, host logic and the C-ABI exports;
`-m gpu` runs compare the CUDA library (through the C ABI) against the oracle.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libb2b.so")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    from oracle import oracle
    oracle.build()


@pytest.fixture
def oracle_factory():
    from oracle.oracle import OracleNet

    def make(dt, f32=False, **kw):
        return OracleNet(dt, f32=f32, **kw)
    return make


@pytest.fixture
def gpu_factory():
    from brian2cuda_b200 import Network

    nets = []

    def make(dt, f32=False, **kw):
        kw.pop("f32", None)
        net = Network(dt, **kw)
        nets.append(net)
        return net
    yield make
    for n in nets:
        n.close()
