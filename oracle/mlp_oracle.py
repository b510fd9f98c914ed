"""CPU restatement of the gating surrogate's arithmetic — TEST INFRASTRUCTURE ONLY.

Forward pass, loss and gradient of the 4 -> 64 -> 64 -> 3 tanh perceptron that libb2b
trains and runs on the tensor cores (brian2cuda_b200/csrc/surrogate.cu).  The surrogate has
no counterpart in the reference; the exact gating step it approximates is the COBAHH
exponential-Euler update (examples/cobahh.py:159-180), whose oracle is oracle.cpp.

Two modes:
  emulate=True  rounds exactly where the GPU rounds: normalised inputs, pre-activations and
                activations to bf16 (round to nearest even), weights to bf16, output
                gradients and hidden-unit gradients to bf16; sums in float64.  The GPU's
                tanh is the hardware approximation, so GPU and oracle agree to a tolerance,
                not bit for bit.
  emulate=False float64 throughout: the mathematical gradient, checked against finite
                differences by the CPU tests (this pins the backward formulas).
Only the tests and smoke() use this module.
"""
from __future__ import annotations

import numpy as np

SLICES = {"W1": (0, (64, 4)), "b1": (256, (64,)), "W2": (320, (64, 64)), "b2": (4416, (64,)),
          "W3": (4480, (3, 64)), "b3": (4672, (3,))}
NPARAMS = 4675


def bf16(a) -> np.ndarray:
    """Rounds float32 values to bfloat16 (nearest even), returned as float32."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(f.shape)


def unpack(p: np.ndarray) -> dict[str, np.ndarray]:
    return {k: np.asarray(p[o:o + int(np.prod(s))], dtype=np.float64).reshape(s)
            for k, (o, s) in SLICES.items()}


def pack(d: dict[str, np.ndarray]) -> np.ndarray:
    p = np.zeros(NPARAMS, dtype=np.float64)
    for k, (o, s) in SLICES.items():
        p[o:o + int(np.prod(s))] = np.asarray(d[k], dtype=np.float64).ravel()
    return p


def _r(a, emulate):
    return bf16(a).astype(np.float64) if emulate else np.asarray(a, dtype=np.float64)


def forward(p: np.ndarray, scaling: np.ndarray, x: np.ndarray, emulate: bool = True):
    """Network outputs y (n, 3) and the intermediates the backward pass needs."""
    w = unpack(p)
    sh, sc = np.asarray(scaling[:4], np.float32), np.asarray(scaling[4:8], np.float32)
    xh = (np.asarray(x, np.float32) - sh) * sc if emulate else \
        (np.asarray(x, np.float64) - sh.astype(np.float64)) * sc.astype(np.float64)
    xh = _r(xh, emulate)
    W1 = _r(w["W1"], emulate)
    b1 = _r(w["b1"], emulate)
    W2 = _r(w["W2"], emulate)
    W3 = _r(w["W3"], emulate)
    b2 = w["b2"].astype(np.float64)
    b3 = w["b3"].astype(np.float64)
    z1 = xh @ W1.T + b1
    h1 = _r(np.tanh(_r(z1.astype(np.float32) if emulate else z1, emulate)), emulate)
    z2 = h1 @ W2.T + b2
    h2 = _r(np.tanh(_r(z2.astype(np.float32) if emulate else z2, emulate)), emulate)
    y = h2 @ W3.T + b3
    return y, dict(xh=xh, h1=h1, h2=h2, W2=W2, W3=W3)


def targets_hat(scaling: np.ndarray, x: np.ndarray, t: np.ndarray) -> np.ndarray:
    """Regression targets of the outputs: (t - (m, h, n)) / out_scale."""
    os_ = np.asarray(scaling[8:11], np.float64)
    return (np.asarray(t, np.float64) - np.asarray(x, np.float64)[:, 1:4]) / os_


def loss_and_grad(p: np.ndarray, scaling: np.ndarray, x: np.ndarray, t: np.ndarray,
                  emulate: bool = True) -> tuple[float, np.ndarray]:
    """Mean over samples of sum_o (y_o - that_o)^2 and its gradient in parameter order."""
    n = len(x)
    y, c = forward(p, scaling, x, emulate)
    e = y - targets_hat(scaling, x, t)
    loss = float(np.sum(e * e) / n)
    dy = _r((2.0 * e / n).astype(np.float32) if emulate else 2.0 * e / n, emulate)
    dh2 = dy @ c["W3"]
    dz2 = _r((dh2 * (1 - c["h2"] ** 2)).astype(np.float32) if emulate
             else dh2 * (1 - c["h2"] ** 2), emulate)
    dh1 = dz2 @ c["W2"]
    dz1 = _r((dh1 * (1 - c["h1"] ** 2)).astype(np.float32) if emulate
             else dh1 * (1 - c["h1"] ** 2), emulate)
    g = {"W1": dz1.T @ c["xh"], "b1": dz1.sum(0), "W2": dz2.T @ c["h1"], "b2": dz2.sum(0),
         "W3": dy.T @ c["h2"], "b3": dy.sum(0)}
    return loss, pack(g)


def predict(p: np.ndarray, scaling: np.ndarray, x: np.ndarray, emulate: bool = True):
    """Predicted (m', h', n') = clip((m, h, n) + out_scale * y, 0, 1)."""
    y, _ = forward(p, scaling, x, emulate)
    os_ = np.asarray(scaling[8:11], np.float64)
    return np.clip(np.asarray(x, np.float64)[:, 1:4] + os_ * y, 0.0, 1.0)
