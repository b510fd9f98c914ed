"""brian2cuda_b200: a B200 (sm_100a) backend for the hot path of Brian2's cuda_standalone.

The compute lives in libb2b.so (hand-written CUDA kernels behind the C ABI of
include/b2b.h); this package holds its Python binding (`Network`), synthetic builders for the
benchmark networks (`models`) and the Brian2 device plugin (`device`).
"""
from ._native import B2BError
from .network import HH, LIF, STDP, HinesBatch, HinesParams, Network

__all__ = ["Network", "HinesBatch", "LIF", "HH", "STDP", "HinesParams", "B2BError"]
