"""The network oracle (oracle/mlp.py) against central finite differences in
float64 with the bf16 roundings switched off, and its bf16 rounding against
torch's."""
from __future__ import annotations

import numpy as np
import torch

from oracle import mlp as OM


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(0).standard_normal(10000).astype(np.float32) * 1e3
    want = torch.from_numpy(x).to(torch.bfloat16).double().numpy()
    assert np.array_equal(OM.bf16(x), want)


def test_backward_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(OM, "bf16", lambda a: np.asarray(a, np.float64))
    rng = np.random.default_rng(1)
    dims = [6, 5, 5, 4, 3]
    w = [rng.standard_normal((dims[i + 1], dims[i])) * 0.5 for i in range(4)]
    b = [rng.standard_normal(dims[i + 1]) * 0.1 for i in range(4)]
    x = rng.standard_normal((7, 6))
    t = rng.standard_normal((7, 3))

    def loss_of(ws, bs):
        y, _, _ = OM.forward(x, ws, bs)
        d = y[:, :2] - t[:, :2]
        return float(np.mean(d * d))

    y, zs, hs = OM.forward(x, w, b)
    _, gw, gb = OM.backward(y, t, zs, hs, w, nvalid=2)
    eps = 1e-6
    for layer in range(4):
        for (r, c) in [(0, 0), (dims[layer + 1] - 1, dims[layer] - 1), (1, 2 % dims[layer])]:
            wp = [a.copy() for a in w]
            wm = [a.copy() for a in w]
            wp[layer][r, c] += eps
            wm[layer][r, c] -= eps
            fd = (loss_of(wp, b) - loss_of(wm, b)) / (2 * eps)
            assert abs(fd - gw[layer][r, c]) <= 1e-6 + 1e-5 * abs(fd), (layer, r, c, fd, gw[layer][r, c])
        bp = [a.copy() for a in b]
        bm = [a.copy() for a in b]
        bp[layer][0] += eps
        bm[layer][0] -= eps
        fd = (loss_of(w, bp) - loss_of(w, bm)) / (2 * eps)
        assert abs(fd - gb[layer][0]) <= 1e-6 + 1e-5 * abs(fd)
