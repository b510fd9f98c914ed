"""brian2cuda_b200: a B200 (sm_100a) backend for the hot path of Brian2's cuda_standalone.

The compute lives in libb2b.so (hand-written CUDA kernels behind the C ABI of
include/b2b.h).  This package holds its Python binding (`Network`), the Brian2 device plugin
(`device`: set_device('cuda_standalone') where Brian2 is installed), the Brian2-shaped front
end and its lowering onto the C ABI (`lowering`, `equations`, `recognize`), the code
generator for models the hand-written kernels do not integrate (`codegen`), the generated C
host program (`cemit`), the benchmark networks as scripts (`examples`) and synthetic builders
(`models`).
"""
from ._native import B2BError
from .lowering import ModelUnsupported, Script
from .network import HH, LIF, STDP, HinesBatch, HinesParams, Network

__all__ = ["Network", "HinesBatch", "LIF", "HH", "STDP", "HinesParams", "B2BError", "Script",
           "ModelUnsupported"]
