"""The golden advect_scalar cotangents (made by the reference's autograd,
tests/golden/make_golden_adjoint.py) against the oracle's forward: the oracle
reproduces the reference's tendency on the fixture's inputs, and central
finite differences of the oracle along random directions equal the golden
gradients' directional derivatives."""
from __future__ import annotations

import numpy as np

from helpers import load_npz
from oracle import dynamics as OD
from pywrf_b200 import synthetic

Z = load_npz("adv_scalar_adj_ref64.npz")


def _grid():
    nz, n = Z["field"].shape[0], Z["field"].shape[1]
    g = synthetic.grid_for(synthetic.CaseSpec(n=n, nz=nz))
    assert g.dx == float(Z["dx"]) and g.dy == float(Z["dy"])
    return g


def _tend(g, field, ru, rv, rom):
    t = np.zeros_like(field)
    OD.advect_scalar(g, field, t, ru, rv, rom, Z["msftx"], Z["fnm"], Z["fnp"], Z["rdnw"])
    return t


def test_oracle_forward_equals_the_reference_on_the_fixture():
    g = _grid()
    t = _tend(g, Z["field"], Z["ru"], Z["rv"], Z["rom"])
    assert np.abs(t - Z["tend"]).max() <= 1e-12 * np.abs(Z["tend"]).max()


def test_golden_gradients_match_oracle_finite_differences():
    g = _grid()
    rng = np.random.default_rng(3)
    base = {k: Z[k] for k in ("field", "ru", "rv", "rom")}
    for name in base:
        d = rng.standard_normal(base[name].shape)
        eps = 1e-6 * float(np.abs(base[name]).max())
        plus = dict(base)
        minus = dict(base)
        plus[name] = base[name] + eps * d
        minus[name] = base[name] - eps * d
        fd = float(((_tend(g, **plus) - _tend(g, **minus)) * Z["cot"]).sum()) / (2 * eps)
        an = float((d * Z["grad_" + name]).sum())
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-9, (name, fd, an)
