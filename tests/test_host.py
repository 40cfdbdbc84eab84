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


def test_rollout_checkpointing_gives_the_taped_gradient_with_bounded_memory():
    """pywrf_b200.adjoint.rollout: truncated backpropagation through n steps
    of a nonlinear step with a learnable bias (the shape of the config-3
    problem) gives the same gradients with per-step and per-segment
    checkpoints as the fully taped rollout, runs each step's forward once
    more in the backward, and keeps only the segments' input states for the
    backward (the taped rollout keeps every saved operand of every step)."""
    import torch

    from pywrf_b200.adjoint import rollout

    g = torch.Generator().manual_seed(5)
    x0 = torch.randn(6, 8, 8, generator=g, dtype=torch.float64)
    y0 = torch.randn(6, 8, 8, generator=g, dtype=torch.float64)
    target = torch.randn(6, 8, 8, generator=g, dtype=torch.float64)
    calls = {"n": 0}

    def make_step(bias):
        def step(x, y):
            calls["n"] += 1
            lap = torch.roll(x, 1, -1) + torch.roll(x, -1, -1) + torch.roll(x, 1, -2) + torch.roll(x, -1, -2) - 4 * x
            t = torch.tanh(y) * torch.sin(x)
            x1 = x + 0.1 * lap + 0.05 * t * torch.exp(-0.1 * x * x) + bias
            y1 = y - 0.05 * x1 * torch.tanh(y * x1)
            return x1, y1
        return step

    n = 12
    grads, kept = {}, {}
    for every in (0, 1, 4):
        bias = torch.zeros(6, 8, 8, dtype=torch.float64, requires_grad=True)
        xs = x0.clone().requires_grad_(True)
        calls["n"] = 0
        count = {"n": 0}

        def pack(t):
            count["n"] += t.numel()
            return t

        with torch.autograd.graph.saved_tensors_hooks(pack, lambda t: t):
            x, y = rollout(make_step(bias), (xs, y0), n, every=every)
        kept[every] = count["n"]
        assert calls["n"] == n
        loss = ((x[:3] - target[:3]) ** 2).mean() + ((y[:3] - target[:3]) ** 2).mean()
        loss.backward()
        assert calls["n"] == (n if every == 0 else 2 * n)  # one recomputation per step
        grads[every] = (bias.grad.clone(), xs.grad.clone())
    for every in (1, 4):
        for a, b in zip(grads[every], grads[0]):
            assert torch.allclose(a, b, rtol=1e-12, atol=1e-14)
    # elements held for the backward: every saved operand of every step when
    # taped, the two input states per segment when checkpointed
    state = x0.numel()
    assert kept[1] == 2 * state * n and kept[4] == 2 * state * (n // 4)
    assert kept[0] > 4 * kept[1]


def test_adjoint_operators_refuse_cpu_tensors():
    """Every differentiable operator fails loudly on CPU tensors: there is no
    CPU path (the check runs before any library call)."""
    import pytest
    import torch

    from pywrf_b200 import adjoint

    z3 = torch.zeros(12, 24, 24)
    z2 = torch.zeros(24, 24)
    z1 = torch.zeros(12)
    with pytest.raises(TypeError):
        adjoint.advect_scalar(z3, z3, z3, z3, z3, z2, z1, z1, z1, 1e-4, 1e-4)
    with pytest.raises(TypeError):
        adjoint.advect_momentum(0, z3, z3, z3, z3, z3, z2, None, z1, z1, z1, 1e-4, 1e-4)
    with pytest.raises(TypeError):
        adjoint.vsolve_w(z3, z3, z3, z3)
    uv = {k: (z2 if k in ("mu", "muu", "muv", "mudf") else z3) for k in adjoint.UV_INPUTS}
    uvd = {k: (z1 if k in ("fnm", "fnp", "rdnw") else z2) for k in adjoint.UV_DATA}
    with pytest.raises(TypeError):
        adjoint.advance_uv(uv, uvd, 1.0, 0.01, 1.5, -0.6, 0.1, 1e-4, 1e-4)
    pr = {k: (z2 if k in ("mu", "mut") else z3) for k in adjoint.PRHO_INPUTS}
    with pytest.raises(TypeError):
        adjoint.calc_p_rho(pr, z1, 0.1, 1)
    mt = {k: (z2 if k in ("mu", "mut", "muave", "muts", "muu", "muv", "mudf", "mu_tend") else z3)
          for k in adjoint.MUT_INPUTS}
    mtd = {k: (z1 if k in ("dnw", "fnm", "fnp", "rdnw") else z2) for k in adjoint.MUT_DATA}
    with pytest.raises(TypeError):
        adjoint.advance_mu_t(mt, mtd, 1.0, 0.1)
    aw = {k: (z2 if k in ("muave", "muts", "mut", "ht") else z3) for k in adjoint.AW_INPUTS}
    awd = {k: (z1 if k in ("fnm", "fnp", "rdnw", "rdn") else z2) for k in adjoint.AW_DATA}
    with pytest.raises(TypeError):
        adjoint.advance_w(aw, awd, 1.0, 0.1, 1.5, -0.6, 0.1)


def test_boundary_record_schedule_follows_the_reference_loop():
    """bdy_schedule reproduces the reference's reload rule (pywrf/solver.py:
    457-458: before step t with t % bdy_interval == 1, record
    t // bdy_interval), and run_with_boundary_records loads each record into
    the state in place before that step."""
    from pywrf_b200.solver import bdy_schedule, run_with_boundary_records

    for nsteps in (0, 1, 5, 359, 360, 361, 720, 721, 1000):
        for bi in (1, 2, 7, 360):
            # step by step as the reference's loop does it
            want, cur = [], None
            for t in range(1, nsteps + 1):
                if t % bi == 1 and t > 1:
                    cur = t // bi
                    want.append((t, cur))
            segs = bdy_schedule(nsteps, bi)
            assert sum(n for _, n in segs) == nsteps
            got, t = [], 1
            for rec, n in segs:
                if rec is not None:
                    got.append((t, rec))
                t += n
            assert got == want, (nsteps, bi)

    class FakeState:
        def __init__(self):
            self.loaded = []

        def load(self, host):
            self.loaded.append(sorted(host)[0])

    class FakeIt:
        def __init__(self):
            self.state, self.steps, self.log = FakeState(), 0, []

        def run(self, n, graph=True):
            self.log.append((self.steps + 1, len(self.state.loaded)))
            self.steps += n

    import numpy as np

    from pywrf_b200 import synthetic
    from pywrf_b200.state import BDY_FIELDS, _BDY_WRF

    spec = synthetic.CaseSpec(n=24, nz=12)
    g = synthetic.grid_for(spec)
    g = type(g)(**{**g.__dict__, "bdy_interval": 4})
    bdy = {}
    for fld in BDY_FIELDS:
        W = _BDY_WRF[fld]
        nk = g.nz if fld == "ph" else (1 if fld == "mu" else g.nz - 1)
        nj = g.ny - 10 if fld == "v" else g.ny - 11
        ni = g.nx - 10 if fld == "u" else g.nx - 11
        for pre in ("B", "BT"):
            for side, n_ in (("XS", nj), ("XE", nj), ("YS", ni), ("YE", ni)):
                shape = (3, 5, n_) if fld == "mu" else (3, 5, nk, n_)
                bdy[f"{W}_{pre}{side}"] = np.zeros(shape, np.float32)
    it = FakeIt()
    run_with_boundary_records(it, g, bdy, 10)
    # steps 1-4 on record 0, record 1 loaded before step 5, record 2 before step 9
    assert it.log == [(1, 0), (5, 1), (9, 2)] and it.steps == 10


def test_classic_netcdf_files_feed_the_solver_without_xarray(tmp_path, monkeypatch):
    """The synthetic case written as the three WRF files in the classic
    NetCDF format (pywrf_b200.netcdf.write_dataset) is read back by
    WrfSolver._load_datasets when xarray is absent, array for array, and the
    state ingested from the files equals the one ingested from the arrays."""
    import sys

    from pywrf_b200 import netcdf
    from pywrf_b200.solver import WrfSolver

    spec = synthetic.CaseSpec(**SMALL)
    inputs, bdy = synthetic.build(spec)
    run = "test"
    netcdf.write_dataset(str(tmp_path / f"wrf_inout_step3_{run}"), inputs)
    netcdf.write_dataset(str(tmp_path / f"wrfbdy_d01_{run}"), bdy)
    monkeypatch.setenv("PYWRF_DATA_DIR", str(tmp_path))
    monkeypatch.setenv("PYWRF_RUN_NAME", run)
    monkeypatch.setitem(sys.modules, "xarray", None)   # import xarray raises ImportError
    ds_in, ds_bdy, ds_ref = WrfSolver(device="cpu")._load_datasets()
    assert ds_ref is None
    for src, ds in ((inputs, ds_in), (bdy, ds_bdy)):
        assert set(src) == set(ds)
        for k, v in src.items():
            assert ds[k].shape == v.shape and ds[k].dtype == np.float32, k
            assert np.array_equal(ds[k], v), k
    g = synthetic.grid_for(spec)
    a, sa = ingest(g, inputs, bdy)
    b, sb = ingest(g, WrfSolver._arrays(ds_in), WrfSolver._arrays(ds_bdy))
    assert sa == sb and set(a) == set(b)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_netcdf4_files_are_refused_with_a_reason(tmp_path):
    from pywrf_b200 import netcdf

    p = tmp_path / "f.nc"
    p.write_bytes(b"\x89HDF\r\n\x1a\n" + bytes(64))
    with pytest.raises(ValueError, match="NetCDF-4"):
        netcdf.open_dataset(str(p))
