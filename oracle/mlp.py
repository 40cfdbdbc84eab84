"""CPU oracle of the per-column microphysics network (TEST INFRASTRUCTURE ONLY).

The reference has no learned part: this module restates, in numpy float64,
the network the CUDA path trains and evaluates (a 4-layer perceptron with
GELU activations, bf16 weights and activations, fp32 accumulation) so that
the tensor-core forward, input-gradient and weight-gradient products and the
fused epilogues can be checked.  GELU is the tanh form
0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), as in the CUDA epilogues.
The bf16 roundings sit where the CUDA path stores bf16 (inputs, weights, pre-activations, activations, output and
hidden gradients); everything else is exact, so the comparison tolerance only
covers accumulation order and the rare value that rounds to the neighbouring
bf16.  Only tests/ import this module.
"""
from __future__ import annotations

import numpy as np


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    x = np.ascontiguousarray(a, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


_C, _A = np.sqrt(2.0 / np.pi), 0.044715


def gelu(x):
    """GELU in its tanh form, 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))."""
    return 0.5 * x * (1.0 + np.tanh(_C * x * (1.0 + _A * x * x)))


def gelu_grad(x):
    th = np.tanh(_C * x * (1.0 + _A * x * x))
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * _C * (1.0 + 3.0 * _A * x * x)


def forward(x, w, b):
    """x [m, d0] and w[l] [d_{l+1}, d_l] (already bf16 values), b[l] fp32.
    Returns the fp32-accumulated output and the stored intermediates."""
    zs, hs = [], [x]
    a = x
    for layer in range(len(w) - 1):
        z = a @ w[layer].T + b[layer]
        zs.append(bf16(z))
        a = bf16(gelu(z))
        hs.append(a)
    y = a @ w[-1].T + b[-1]
    return y, zs, hs


def backward(y, t, zs, hs, w, nvalid):
    """Gradients of mean((y - t)^2) over the first nvalid output columns."""
    m, n = y.shape
    d = np.zeros_like(y)
    d[:, :nvalid] = y[:, :nvalid] - t[:, :nvalid]
    loss = float(np.sum(d * d))
    dz = bf16(d * (2.0 / (m * nvalid)))
    gw = [None] * len(w)
    gb = [None] * len(w)
    for layer in range(len(w) - 1, -1, -1):
        gw[layer] = dz.T @ hs[layer]
        gb[layer] = dz.sum(axis=0)
        if layer > 0:
            dz = bf16((dz @ w[layer]) * gelu_grad(zs[layer - 1]))
    return loss, gw, gb
