"""Host-side logic on the CPU: the ingest step (WRF arrays -> halo frame)
against the oracle's, the device-state table, the grid record."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import SMALL
from oracle.model import ingest as oracle_ingest
from pywrf_b200 import _native as N
from pywrf_b200 import synthetic
from pywrf_b200.config import Grid
from pywrf_b200.state import field_shape, grid_from_inputs, ingest


@pytest.fixture(scope="module")
def case():
    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    return spec, g, inputs, bdy


def test_grid_from_input_shapes(case):
    spec, g, inputs, _ = case
    g2 = grid_from_inputs(inputs, spec.dx, spec.dx, spec.dt, spec.p_top, spec.soundsteps)
    assert (g2.nx, g2.ny, g2.nz, g2.ids, g2.ide, g2.jds, g2.jde) == (g.nx, g.ny, g.nz, 5, g.nx - 5, 5, g.ny - 5)


def test_ingest_matches_oracle(case):
    _, g, inputs, bdy = case
    host, scal = ingest(g, inputs, bdy)
    ref = oracle_ingest(g, inputs, bdy, np.float32)
    checked = 0
    for k, v in host.items():
        if k in ref and isinstance(ref[k], np.ndarray):
            np.testing.assert_array_equal(v, ref[k], err_msg=k)
            checked += 1
    for fld, d in ref["bdy"].items():
        for key, arr in d.items():
            pre = "bt" if key.startswith("t") else "b"
            np.testing.assert_array_equal(host[f"{fld}_{pre}{key[-2:]}"], arr, err_msg=f"{fld} {key}")
            checked += 1
    for k in ("cf1", "cf2", "cf3", "cfn", "cfn1"):
        assert scal[k] == pytest.approx(float(ref[k]))
    assert checked > 70


def test_ingest_shapes_fit_the_field_table(case):
    _, g, inputs, bdy = case
    host, _ = ingest(g, inputs, bdy)
    table = dict(zip(N.field_names(), N.field_kinds()))
    for k, v in host.items():
        assert k in table, k
        assert v.shape == field_shape(table[k], g), k
        assert v.dtype == np.float32


def test_grid_validation():
    with pytest.raises(ValueError):
        Grid.make(20, 28, 16, 9000.0, 9000.0, 45.0)
    with pytest.raises(ValueError):
        Grid.make(28, 28, 8, 9000.0, 9000.0, 45.0)
