"""Gating surrogate for COBAHH neurons: Python binding of the b2b_mlp_* and b2b_hh_gating_*
entry points of include/b2b.h.

A 4 -> 64 -> 64 -> 3 perceptron with tanh hidden units predicts the exponential-Euler step
of the Hodgkin-Huxley gates (m, h, n) over one dt from (v, m, h, n).  Its forward pass,
backward pass and weight gradients run on the sm_100a tensor cores (tcgen05, BF16 operands,
FP32 accumulation in tensor memory); Adam updates FP32 master weights.  It is trained on
transitions that the exact integrator itself produces (`gating_targets`) from states of
simulated trajectories (`trajectory_states`), and attached to a network with `attach`, where
the exact integrator stays as the fallback and, with `judge=True`, checks every step.

brian2cuda has no counterpart: its COBAHH neurons integrate the gates with the code Brian2
generates for `method='exponential_euler'` (examples/cobahh.py:159-180).

Device buffers are torch CUDA tensors (float32, contiguous; samples as rows (v, m, h, n),
targets and predictions as rows (m', h', n')).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from ._native import B2BError
from .network import HH, Network

NPARAMS = N.MLP_NPARAMS
PARAM_SLICES = {"W1": (0, (64, 4)), "b1": (256, (64,)), "W2": (320, (64, 64)),
                "b2": (4416, (64,)), "W3": (4480, (3, 64)), "b3": (4672, (3,))}


def _check(st: int, what: str):
    if st != N.B2B_OK:
        raise B2BError(st, what)


def _dev_ptr(t, cols: int) -> int:
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and
            t.is_contiguous() and t.dim() == 2 and t.shape[1] == cols):
        raise ValueError(f"expected a contiguous float32 CUDA tensor of shape (n, {cols})")
    return t.data_ptr()


def unpack_params(p: np.ndarray) -> dict[str, np.ndarray]:
    """Splits the flat parameter vector into W1, b1, W2, b2, W3, b3 (views)."""
    return {k: p[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in PARAM_SLICES.items()}


class GatingSurrogate:
    """The network, its scaling and its Adam state on one GPU."""

    def __init__(self, device: int = 0, seed: int = 0, stream: int | None = None):
        self._lib = N.lib()
        self.device = device
        h = C.c_void_p()
        _check(self._lib.b2b_mlp_create(device, stream, int(seed), C.byref(h)), "mlp_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.b2b_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- parameters --------------------------------------------------------------------------
    @property
    def params(self) -> np.ndarray:
        a = np.empty(NPARAMS, dtype=np.float32)
        _check(self._lib.b2b_mlp_params_get(self._h, a.ctypes.data_as(C.c_void_p), NPARAMS),
               "params_get")
        return a

    @params.setter
    def params(self, values):
        a = np.ascontiguousarray(values, dtype=np.float32)
        if a.shape != (NPARAMS,):
            raise ValueError(f"expected {NPARAMS} parameters")
        _check(self._lib.b2b_mlp_params_set(self._h, a.ctypes.data_as(C.c_void_p), NPARAMS),
               "params_set")

    @property
    def scaling(self) -> np.ndarray:
        """in_shift[4], in_scale[4], out_scale[3]."""
        a = np.empty(11, dtype=np.float32)
        _check(self._lib.b2b_mlp_scaling_get(self._h, a.ctypes.data_as(C.c_void_p)),
               "scaling_get")
        return a

    @scaling.setter
    def scaling(self, values):
        a = np.ascontiguousarray(values, dtype=np.float32)
        if a.shape != (11,):
            raise ValueError("expected 11 scaling values")
        _check(self._lib.b2b_mlp_scaling_set(self._h, a.ctypes.data_as(C.c_void_p)),
               "scaling_set")

    def fit_scaling(self, x, t):
        _check(self._lib.b2b_mlp_fit_scaling(self._h, _dev_ptr(x, 4), _dev_ptr(t, 3), len(x)),
               "fit_scaling")

    # -- compute -----------------------------------------------------------------------------
    def forward(self, x, raw: bool = False):
        """Predicted (m', h', n') per row of x, or the network outputs y with raw=True."""
        import torch
        out = torch.empty((len(x), 3), dtype=torch.float32, device=x.device)
        _check(self._lib.b2b_mlp_forward(self._h, _dev_ptr(x, 4), out.data_ptr(), len(x),
                                         1 if raw else 0), "mlp_forward")
        return out

    def grad(self, x, t) -> tuple[np.ndarray, float]:
        """Gradient of the mean loss over all rows, and the loss."""
        g = np.empty(NPARAMS, dtype=np.float32)
        loss = C.c_double()
        _check(self._lib.b2b_mlp_grad(self._h, _dev_ptr(x, 4), _dev_ptr(t, 3), len(x),
                                      g.ctypes.data_as(C.c_void_p), NPARAMS, C.byref(loss)),
               "mlp_grad")
        return g, loss.value

    def train(self, x, t, epochs: int, batch: int = 16384, lr: float = 2e-3) -> list[float]:
        """Adam with a cosine learning-rate decay; returns the mean loss of every epoch."""
        losses = (C.c_double * max(1, epochs))()
        _check(self._lib.b2b_mlp_train(self._h, _dev_ptr(x, 4), _dev_ptr(t, 3), len(x),
                                       int(epochs), int(batch), float(lr), losses), "mlp_train")
        return [losses[i] for i in range(epochs)]

    def fit(self, x, t, epochs: int = 400, batch: int = 32768, lr: float = 3e-3,
            out_scale: float = 0.01) -> list[float]:
        """The training recipe: input scaling from the data, one output scale for all gates
        (it weights the loss towards absolute gate error, which the fallback bound tests),
        then `train`."""
        self.fit_scaling(x, t)
        sc = self.scaling
        sc[8:11] = out_scale
        self.scaling = sc
        return self.train(x, t, epochs=epochs, batch=batch, lr=lr)

    def attach(self, net: Network, gid: int, tol: float = 1e-3, judge: bool = True):
        """Steps every float32 HH group of gid's population with the surrogate gating update
        (call before net.finalize(); keep this object alive as long as the net)."""
        net._check(self._lib.b2b_group_hh_surrogate(net._h, gid, self._h, float(tol),
                                                    1 if judge else 0), "hh_surrogate")
        net._surrogate = self


def gating_targets(params: HH, dt: float, x, device: int = 0, stream: int | None = None):
    """The exact exponential-Euler gating step of every row of x (float32, on the GPU)."""
    import torch
    t = torch.empty((len(x), 3), dtype=torch.float32, device=x.device)
    p = params.to_c()
    _check(N.lib().b2b_hh_gating_exact(C.byref(p), float(dt), _dev_ptr(x, 4), t.data_ptr(),
                                       len(x), device, stream), "hh_gating_exact")
    return t


def sample_states(net: Network, gid: int, n: int | None = None):
    """(v, m, h, n) of the first n neurons of a float32 HH group as a (n, 4) CUDA tensor."""
    import torch
    n = net.group_size(gid) if n is None else int(n)
    x = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    net._check(N.lib().b2b_hh_gating_sample(net._h, gid, x.data_ptr(), n), "hh_gating_sample")
    net.sync()
    return x


def trajectory_states(net: Network, gid: int, n_samples: int, every: int = 10,
                      warmup: int = 0):
    """States of simulated trajectories: runs the (finalized) net and samples the group every
    `every` steps until n_samples rows are collected."""
    import torch
    if warmup:
        net.run(warmup)
    n = net.group_size(gid)
    chunks, have = [], 0
    while have < n_samples:
        net.run(every)
        x = sample_states(net, gid)
        chunks.append(x[: min(n, n_samples - have)])
        have += len(chunks[-1])
    return torch.cat(chunks)


def physiological(x, v_lo: float = -0.15, v_hi: float = 0.1):
    """The rows of x whose values are finite and whose v lies in [v_lo, v_hi] volts.  Training
    data should pass through this: b2b_mlp_fit_scaling maps the data's v range to the
    network's input range, so a few runaway states (a neuron with a negative conductance and
    no input drifts to volts) would leave the physiological range a sliver of it; states
    outside the training range are stepped exactly by the surrogate kernel."""
    import torch
    ok = torch.isfinite(x).all(dim=1) & (x[:, 0] >= v_lo) & (x[:, 0] <= v_hi)
    return x[ok].contiguous()


def surrogate_stats(net: Network, gid: int) -> tuple[int, int]:
    """(neuron-updates made with the surrogate, exact fallbacks among them)."""
    u, f = C.c_int64(), C.c_int64()
    net._check(N.lib().b2b_surrogate_stats(net._h, gid, C.byref(u), C.byref(f)),
               "surrogate_stats")
    return u.value, f.value
