"""Golden cotangents of advect_scalar from the reference's own autograd.

Usage:  python tests/golden/make_golden_adjoint.py [--reference /path/to/PyWRF]

Runs the unmodified reference ``pywrf.wrf_dynamics.advect_scalar``
(wrf_dynamics.py:1841-2028) in float64 on CPU with ``requires_grad`` on the
advected field and the three mass fluxes, back-propagates a seeded random
cotangent of the returned tendency with torch autograd, and writes
``adv_scalar_adj_ref64.npz`` next to this script: the inputs, the cotangent,
the forward tendency and the four gradients.  Grid 24x24x12 in the solver's
5-cell frame; fluxes of both signs so that both upwind branches are taken.
This script is the only producer of the fixture and is never run by the tests.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from pywrf_b200 import synthetic  # noqa: E402

N, NZ = 24, 12


def inputs(seed: int = 11) -> dict[str, np.ndarray]:
    rng = np.random.default_rng(seed)
    shape = (NZ, N, N)
    x = np.linspace(0, 2 * np.pi, N)
    smooth = np.sin(x)[None, None, :] * np.cos(0.7 * x)[None, :, None] * np.linspace(1, 2, NZ)[:, None, None]
    return {
        "field": 300.0 + 3.0 * smooth + 0.5 * rng.standard_normal(shape),
        "ru": 20.0 * rng.standard_normal(shape) + 5.0,
        "rv": 20.0 * rng.standard_normal(shape) - 5.0,
        "rom": 2.0 * rng.standard_normal(shape),
        "msftx": 1.0 + 0.05 * rng.random((N, N)),
        "fnm": 0.45 + 0.1 * rng.random(NZ),
        "fnp": 0.45 + 0.1 * rng.random(NZ),
        "rdnw": -(8.0 + 4.0 * rng.random(NZ)),
        "cot": rng.standard_normal(shape),
    }


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=None)
    a = ap.parse_args()
    if a.reference:
        os.environ["PYWRF_REFERENCE_ROOT"] = a.reference
    import torch

    import refharness
    spec = synthetic.CaseSpec(n=N, nz=NZ)
    g = synthetic.grid_for(spec)
    _cp, dyn, _phy, _bdy, _solver = refharness.load_reference(g, dtype="float64")
    d = inputs()
    t = {k: torch.tensor(v, dtype=torch.float64) for k, v in d.items()}
    for k in ("field", "ru", "rv", "rom"):
        t[k].requires_grad_(True)
    tend0 = torch.zeros((NZ, N, N), dtype=torch.float64)
    ones2 = torch.ones((N, N), dtype=torch.float64)
    one1 = torch.ones(NZ, dtype=torch.float64)
    ids, ide, jds, jde = 5, N - 5, 5, N - 5
    out = dyn.advect_scalar(t["field"], t["field"], tend0.clone(), t["ru"], t["rv"], t["rom"], one1, one1 * 0.0,
                            ones2, int(g.dt), ones2, ones2, ones2, ones2, t["msftx"], ones2, t["fnm"], t["fnp"],
                            1.0 / g.dx, 1.0 / g.dy, t["rdnw"],
                            ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)
    (out * t["cot"]).sum().backward()
    save = dict(d)
    save["tend"] = out.detach().numpy()
    for k in ("field", "ru", "rv", "rom"):
        save["grad_" + k] = t[k].grad.numpy()
    save["dx"] = np.array(g.dx)
    save["dy"] = np.array(g.dy)
    np.savez_compressed(os.path.join(HERE, "adv_scalar_adj_ref64.npz"), **save)
    print("wrote adv_scalar_adj_ref64.npz", {k: float(np.abs(v).max()) for k, v in save.items() if k.startswith("grad")})


if __name__ == "__main__":
    main()
