"""Parity of the CUDA step (through the C ABI) with the reference and the oracle.

Every tolerance is stated against the fp64 reference: the CUDA fp32 result
must be within a small multiple of the error the reference itself makes in
fp32 (its fp32 run against its fp64 run, or the fp32 oracle's, which matches
it), field by field.  Bit-level equality with an fp32 run is not expected:
the reference evaluates pow/exp/log through ATen and rounds differently.
"""
from __future__ import annotations

import ctypes
import json

import numpy as np
import pytest
import torch

from helpers import GOLDEN, SMALL, load_npz, load_summary, pick, rel_l2, summary_errors
from oracle import physics as OP
from oracle import dynamics as OD
from oracle.model import OracleModel
from pywrf_b200 import _native as N
from pywrf_b200 import synthetic
from pywrf_b200.solver import Integrator
from pywrf_b200.state import DeviceState

pytestmark = pytest.mark.gpu

# multiple of the reference's own fp32 error allowed for the CUDA fp32 result
K_FLOOR = 3.0
ABS_FLOOR = 1e-9


@pytest.fixture(scope="module", autouse=True)
def _need_cuda():
    if not torch.cuda.is_available():
        pytest.fail("these tests need a CUDA device")


def cuda_run(g, inputs, bdy, nsteps, graph=False):
    st = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    it = Integrator(st)
    it.run(nsteps, graph=graph)
    torch.cuda.synchronize()
    return st, it


def cuda_fields(st):
    return pick(lambda k: st[k].cpu().numpy())


def oracle_fields(g, inputs, bdy, dtype, nsteps):
    m = OracleModel(g, inputs, bdy, dtype)
    m.run(nsteps)
    return pick(lambda k: m.st[k])


@pytest.fixture(scope="module")
def small():
    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    return g, inputs, bdy


@pytest.fixture(scope="module")
def config0():
    spec = synthetic.spec_for_config(0)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    return spec, g, inputs, bdy


def test_small_two_steps_vs_reference_fp64(small):
    g, inputs, bdy = small
    st, it = cuda_run(g, inputs, bdy, SMALL["nsteps"])
    out = cuda_fields(st)
    r64, r32 = load_npz("small_ref64.npz"), load_npz("small_ref32.npz")
    bad = []
    for k, v in out.items():
        err, floor = rel_l2(v, r64[k]), rel_l2(r32[k], r64[k])
        if not err <= K_FLOOR * floor + ABS_FLOOR:
            bad.append((k, err, floor))
    assert not bad, bad
    assert it.status() == {"nan_p": 0, "step": SMALL["nsteps"], "wait_timeouts": 0}


def test_small_one_step_within_1e5_relative_l2(small):
    """After one step, relative L2 against the fp64 reference within 1e-5 for
    every field whose own fp32 reference error is below 1e-5 (the reference
    itself misses 1e-5 on v, w, mu, p, al, ww, qc, qi, h_diabatic)."""
    g, inputs, bdy = small
    st, _ = cuda_run(g, inputs, bdy, 1)
    out = cuda_fields(st)
    o64 = oracle_fields(g, inputs, bdy, np.float64, 1)
    o32 = oracle_fields(g, inputs, bdy, np.float32, 1)
    for k in out:
        floor = rel_l2(o32[k], o64[k])
        err = rel_l2(out[k], o64[k])
        if floor < 3e-6:
            assert err < 1e-5, (k, err, floor)
        assert err <= K_FLOOR * floor + ABS_FLOOR, (k, err, floor)


def test_rows_not_a_multiple_of_16_bytes_vs_oracle_fp64():
    """nx = 30 (rows of 120 bytes, no tensor-map tiles): the tiled advection
    takes its cp.async form; two steps match the fp64 oracle within the fp32
    oracle's own error, field by field, as the tensor-map form does on the
    other grids."""
    spec = synthetic.CaseSpec(**{**SMALL, "n": 30, "seed": 11})
    g = synthetic.grid_for(spec)
    assert g.nx % 4 != 0
    inputs, bdy = synthetic.build(spec)
    st, it = cuda_run(g, inputs, bdy, 2)
    out = cuda_fields(st)
    o64 = oracle_fields(g, inputs, bdy, np.float64, 2)
    o32 = oracle_fields(g, inputs, bdy, np.float32, 2)
    bad = []
    for k in out:
        err, floor = rel_l2(out[k], o64[k]), rel_l2(o32[k], o64[k])
        if not err <= K_FLOOR * floor + ABS_FLOOR:
            bad.append((k, err, floor))
    assert not bad, bad
    assert it.status() == {"nan_p": 0, "step": 2, "wait_timeouts": 0}


def test_config0_ten_steps_vs_oracle_fp64(config0):
    spec, g, inputs, bdy = config0
    st, it = cuda_run(g, inputs, bdy, spec.nsteps, graph=True)
    out = cuda_fields(st)
    o64 = oracle_fields(g, inputs, bdy, np.float64, spec.nsteps)
    o32 = oracle_fields(g, inputs, bdy, np.float32, spec.nsteps)
    bad = []
    for k in out:
        err, floor = rel_l2(out[k], o64[k]), rel_l2(o32[k], o64[k])
        if not err <= K_FLOOR * floor + ABS_FLOOR:
            bad.append((k, err, floor))
    assert not bad, bad
    # column dry-mass drift no worse than the fp32 oracle's
    mu0 = st["mub"].cpu().numpy()
    drift_c = abs(float((out["mu"] + mu0).sum()) - float((o64["mu"] + mu0).sum()))
    drift_o = abs(float((o32["mu"] + mu0).sum()) - float((o64["mu"] + mu0).sum()))
    assert drift_c <= K_FLOOR * drift_o + 1e-3 * out["mu"].size
    assert it.status()["nan_p"] == 0


def test_config0_three_steps_vs_reference_summary(config0):
    _, g, inputs, bdy = config0
    summ = load_summary("c0_ref64_summary.json")
    st, _ = cuda_run(g, inputs, bdy, summ["nsteps"])
    e_c = summary_errors(cuda_fields(st), summ)
    e_o = summary_errors(oracle_fields(g, inputs, bdy, np.float32, summ["nsteps"]), summ)
    for k in e_c:
        assert e_c[k][0] <= 4.0 * e_o[k][0] + 1e-6, (k, e_c[k], e_o[k])
        # norms: the fp32 oracle is unusually close on some norms (qi: 5e-8,
        # where the reference's own fp32 run is off by 2.4e-6 on the small
        # case), so the bound is floored at the 1e-5 relative level
        assert e_c[k][1] <= max(4.0 * e_o[k][1], 1e-5), (k, e_c[k], e_o[k])


# fp32 error of the reference at 240x240x41 after one step, sampled values /
# L2 norm (measured with the fp32 oracle against the fp64 reference summary),
# times four; the qi norm bound is the 1e-5 relative level (the reference's
# own fp32 qi norm error is 2.4e-6 on the small case, 7x the oracle's)
C1_TOL = {
    "u": (1e-5, 1e-6), "v": (5e-5, 1e-6), "w": (2e-4, 2e-5), "t": (4e-6, 1e-6), "ph": (5e-5, 2.5e-5),
    "mu": (1e-4, 1e-5), "p": (3e-4, 1.5e-5), "al": (2e-4, 1e-5), "h_diabatic": (6e-4, 5e-6),
    "rainnc": (1e-6, 1e-6), "muts": (1e-6, 1e-6), "ww": (1.2e-4, 1e-6), "qv": (1e-6, 1e-6),
    "qc": (1e-5, 1e-5), "qr": (1e-5, 3e-6), "qi": (1e-5, 1e-5), "qs": (1e-5, 1e-6), "qg": (1e-6, 1e-6),
}


def test_config1_one_step_vs_reference_summary():
    summ = load_summary("c1_ref64_summary.json")
    spec = synthetic.spec_for_config(1)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    st, it = cuda_run(g, inputs, bdy, summ["nsteps"])
    errs = summary_errors(cuda_fields(st), summ)
    bad = [(k, e, C1_TOL[k]) for k, e in errs.items() if not (e[0] <= C1_TOL[k][0] and e[1] <= C1_TOL[k][1])]
    assert not bad, bad
    assert it.status()["nan_p"] == 0


def test_wrf_solver_drop_in(small):
    """pywrf_b200.WrfSolver as the reference is used: subclass, override
    _load_datasets, solve(); the fields match the fp64 reference fixtures."""
    from pywrf_b200 import WrfSolver

    spec = synthetic.CaseSpec(**SMALL)
    inputs, bdy = synthetic.build(spec)

    class Run(WrfSolver):
        def _load_datasets(self):
            return inputs, bdy, None

    res = Run(nsteps=SMALL["nsteps"], dt=spec.dt, p_top=spec.p_top, dx=spec.dx, dy=spec.dx).solve()
    assert set(res) == {"u", "v", "w", "t", "ph", "mu", "moist"}
    assert all(t.is_cuda for t in res.values())
    r64, r32 = load_npz("small_ref64.npz"), load_npz("small_ref32.npz")
    got = {k: res[k].cpu().numpy() for k in ("u", "v", "w", "t", "ph", "mu")}
    got["qv"] = res["moist"][1].cpu().numpy()
    for k, v in got.items():
        err, floor = rel_l2(v, r64[k]), rel_l2(r32[k], r64[k])
        assert err <= K_FLOOR * floor + ABS_FLOOR, (k, err, floor)


def test_graph_replay_equals_eager_bitwise(small):
    g, inputs, bdy = small
    a, _ = cuda_run(g, inputs, bdy, 2, graph=False)
    b, _ = cuda_run(g, inputs, bdy, 2, graph=True)
    for k in a.names:
        assert torch.equal(a[k], b[k]), k


def test_host_driven_steps_equal_device_steps_bitwise(small):
    """Integrator.run_host (the prognostic fields copied in from pinned
    host memory and back out every step, the two directions of the copies
    overlapped in chunks) leaves in the host buffers exactly the state that
    stepping on the device leaves (3 steps, graph replay both ways)."""
    g, inputs, bdy = small
    a, _ = cuda_run(g, inputs, bdy, 3, graph=True)
    st = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    it = Integrator(st)
    names = ("u", "v", "w", "t", "ph", "mu", "p", "al", "moist")
    host = {k: torch.empty(st[k].shape, dtype=st[k].dtype, pin_memory=True) for k in names}
    for k in names:
        host[k].copy_(st[k])
    it.run_host(host, 3, chunk_bytes=4096)
    torch.cuda.synchronize()
    for k in names:
        assert torch.equal(host[k], a[k].cpu()), k
        assert torch.equal(st[k], a[k]), k
    with pytest.raises(ValueError):
        it.run_host({"u": torch.empty(st["u"].shape)}, 1)


def test_boundary_time_follows_the_device_step_counter(small):
    g, inputs, bdy = small
    st, it = cuda_run(g, inputs, bdy, 3, graph=True)
    assert it.status()["step"] == 3
    dscal = st["dscal"].cpu().numpy()
    assert dscal[0] == pytest.approx(3 * g.dt)
    assert dscal[1] == 3.0


def test_nan_in_the_state_is_reported_not_fatal(small):
    g, inputs, bdy = small
    st = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    st["t"][5, 12, 12] = float("nan")
    it = Integrator(st)
    it.step()
    s = it.status()
    assert s["nan_p"] > 0 and s["step"] == 1


def test_two_split_microphysics_loops_coarse_grid():
    """dt = 240 s makes WSM6 run two time-split loops (the fused physics
    kernel); a 40 km grid keeps the acoustic steps stable."""
    spec = synthetic.CaseSpec(n=28, nz=16, dx=40000.0, dt=240.0, nsteps=1, bdy_tend_amp=1.0e-4, seed=5)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    st, it = cuda_run(g, inputs, bdy, 1)
    out = cuda_fields(st)
    o64 = oracle_fields(g, inputs, bdy, np.float64, 1)
    o32 = oracle_fields(g, inputs, bdy, np.float32, 1)
    for k in out:
        err, floor = rel_l2(out[k], o64[k]), rel_l2(o32[k], o64[k])
        assert err <= K_FLOOR * floor + ABS_FLOOR, (k, err, floor)
    assert it.status()["nan_p"] == 0


def _ptr(t: torch.Tensor):
    assert t.is_cuda and t.is_contiguous() and t.dtype == torch.float32
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("delt", [45.0, 250.0])
def test_wsm6_entry_point_matches_oracle(small, delt):
    """wrf_wsm6 on the physics inputs of a real stepped state against the
    oracle's WSM6 in fp64 (fp32 floor from the oracle's fp32 run); 250 s
    takes two time-split loops."""
    g, inputs, bdy = small
    m = OracleModel(g, inputs, bdy, np.float64)
    m.run(1)
    OP.moist_physics_prep_em(g, m.st)
    s = m.st
    names = ("th_phy", "q1", "q2", "q3", "q4", "q5", "q6", "rho", "pi_phy", "p_phy", "dz8w")
    arrays = {k: (s["moist"][int(k[1])] if k.startswith("q") else s[k]).copy() for k in names}
    pre2 = {k: s[k].copy() for k in ("rainnc", "rainncv", "snownc", "snowncv", "graupelnc", "graupelncv", "sr")}

    def run_oracle(dtype):
        a = {k: v.astype(dtype).copy() for k, v in arrays.items()}
        p2 = {k: v.astype(dtype).copy() for k, v in pre2.items()}
        OP.wsm6(g, a["th_phy"], a["q1"], a["q2"], a["q3"], a["q4"], a["q5"], a["q6"], a["rho"], a["pi_phy"],
                a["p_phy"], a["dz8w"], float(delt), p2["rainnc"], p2["rainncv"], p2["snownc"], p2["snowncv"],
                p2["graupelnc"], p2["graupelncv"], p2["sr"])
        return a, p2

    o64, p64 = run_oracle(np.float64)
    o32, p32 = run_oracle(np.float32)
    dev = {k: torch.tensor(v, dtype=torch.float32, device="cuda") for k, v in arrays.items()}
    d2 = {k: torch.tensor(v, dtype=torch.float32, device="cuda") for k, v in pre2.items()}
    st = DeviceState(g, "cuda")
    L = N.lib()
    rc = L.wrf_wsm6(ctypes.byref(st.cgrid), *[_ptr(dev[k]) for k in names], ctypes.c_float(delt),
                    *[_ptr(d2[k]) for k in ("rainnc", "rainncv", "snownc", "snowncv", "graupelnc", "graupelncv", "sr")],
                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, "wrf_wsm6")
    torch.cuda.synchronize()
    for k in names[:7]:
        c = dev[k].cpu().numpy()
        err, floor = rel_l2(c, o64[k]), rel_l2(o32[k], o64[k])
        assert err <= K_FLOOR * floor + 1e-7, (k, err, floor)
    for k in ("rainnc", "rainncv", "sr"):
        c = d2[k].cpu().numpy()
        err, floor = rel_l2(c, p64[k]), rel_l2(p32[k], p64[k])
        assert err <= K_FLOOR * floor + 1e-7, (k, err, floor)


def test_advect_scalar_entry_point_matches_oracle(small):
    g, inputs, bdy = small
    m = OracleModel(g, inputs, bdy, np.float64)
    m.run(1)
    s = m.st
    field = s["t"]
    ref64 = np.zeros_like(field)
    OD.advect_scalar(g, field, ref64, s["ru"], s["rv"], s["ww"], s["msftx"], s["fnm"], s["fnp"], s["rdnw"])
    s32 = {k: s[k].astype(np.float32) for k in ("t", "ru", "rv", "ww", "msftx", "fnm", "fnp", "rdnw")}
    ref32 = np.zeros_like(s32["t"])
    OD.advect_scalar(g, s32["t"], ref32, s32["ru"], s32["rv"], s32["ww"], s32["msftx"], s32["fnm"], s32["fnp"],
                     s32["rdnw"])
    dev = {k: torch.tensor(v, device="cuda") for k, v in s32.items()}
    tend = torch.zeros_like(dev["t"])
    st = DeviceState(g, "cuda")
    rc = N.lib().wrf_advect_scalar(ctypes.byref(st.cgrid), _ptr(dev["t"]), _ptr(tend), _ptr(dev["ru"]),
                                   _ptr(dev["rv"]), _ptr(dev["ww"]), _ptr(dev["msftx"]), _ptr(dev["fnm"]),
                                   _ptr(dev["fnp"]), _ptr(dev["rdnw"]),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, "wrf_advect_scalar")
    torch.cuda.synchronize()
    err, floor = rel_l2(tend.cpu().numpy(), ref64), rel_l2(ref32, ref64)
    assert err <= K_FLOOR * floor + 1e-9, (err, floor)


@pytest.mark.parametrize("graph", [False, True])
def test_boundary_record_reload_vs_reference_fp64(graph):
    """Boundary interval of 2 steps and three distinct boundary records: the
    reference reloads every boundary array from record 1 before step 3
    (solver.py:457-703).  run_with_boundary_records does the same between
    steps (in place, so the captured graph stays valid); after 4 steps the
    fields are within 3x the reference's own fp32 error of its fp64 run."""
    import dataclasses

    from helpers import bdy_records
    from pywrf_b200.solver import run_with_boundary_records

    spec = synthetic.CaseSpec(**SMALL)
    g = dataclasses.replace(synthetic.grid_for(spec), bdy_interval=2)
    inputs, bdy = synthetic.build(spec)
    recs = bdy_records(bdy)
    st = DeviceState.from_inputs(g, inputs, recs, device="cuda")
    it = Integrator(st)
    run_with_boundary_records(it, g, recs, 4, graph=graph)
    torch.cuda.synchronize()
    r64, r32 = load_npz("small_bdyrec_ref64.npz"), load_npz("small_bdyrec_ref32.npz")
    out = cuda_fields(st)
    bad = []
    for k in ("u", "v", "t", "ph", "mu", "qv"):
        err, floor = rel_l2(out[k], r64[k]), rel_l2(r32[k], r64[k])
        if not err <= K_FLOOR * floor + ABS_FLOOR:
            bad.append((k, err, floor))
    assert not bad, bad
    assert it.status() == {"nan_p": 0, "step": 4, "wait_timeouts": 0}


def test_61_levels_dt30_vs_oracle_fp64():
    """The 512x512x61 workload's vertical grid and time step (nz = 61, dt =
    30 s; WSM6 on 60 levels takes its 32-lane column segments) on a 28x28
    horizontal grid: two steps within 3x the fp32 oracle's own error of the
    fp64 oracle, field by field."""
    spec = synthetic.CaseSpec(n=28, nz=61, dt=30.0, nsteps=2, bdy_tend_amp=1.0e-4, seed=7)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    st, it = cuda_run(g, inputs, bdy, 2, graph=True)
    out = cuda_fields(st)
    o64 = oracle_fields(g, inputs, bdy, np.float64, 2)
    o32 = oracle_fields(g, inputs, bdy, np.float32, 2)
    bad = []
    for k in out:
        err, floor = rel_l2(out[k], o64[k]), rel_l2(o32[k], o64[k])
        if not err <= K_FLOOR * floor + ABS_FLOOR:
            bad.append((k, err, floor))
    assert not bad, bad
    assert it.status() == {"nan_p": 0, "step": 2, "wait_timeouts": 0}


def test_config1_eighty_steps_vs_reference_sample():
    """The 240x240x41 workload for 80 steps (1 h) against the reference's
    float64 run of the same state (tests/golden/c1_80_ref_sample.npz: values
    at 16384 seeded points per field, exact norms, the reference's own
    float32 error over each whole field, dry-mass totals).  Per field, the
    relative L2 over the sampled points must be within 1e-3, or within 3x the
    reference's own float32 error on the same points where that error
    exceeds 1e-3 / 3; the dry-mass drift against the float64 run must be no
    worse than 3x the reference float32 run's."""
    with np.load(f"{GOLDEN}/c1_80_ref_sample.npz") as z:
        ref = {k: z[k] for k in z.files}
    meta = json.loads(str(ref["meta"]))
    spec = synthetic.spec_for_config(meta["config"], seed=meta["seed"])
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    st, it = cuda_run(g, inputs, bdy, meta["nsteps"], graph=True)
    assert it.status() == {"nan_p": 0, "step": meta["nsteps"], "wait_timeouts": 0}
    out = cuda_fields(st)
    report, bad = {}, []
    for k, a in out.items():
        assert list(a.shape) == ref[f"{k}__shape"].tolist(), k
        idx = ref[f"{k}__idx"]
        v64, v32 = ref[f"{k}__v64"], ref[f"{k}__v32"].astype(np.float64)
        err = rel_l2(a.reshape(-1)[idx], v64)
        floor = rel_l2(v32, v64)
        report[k] = (err, floor, float(ref[f"{k}__floor"]))
        if not (err <= 1e-3 or err <= K_FLOOR * floor):
            bad.append((k, err, floor))
    assert not bad, (bad, report)
    R = (slice(g.jds, g.jde - 1), slice(g.ids, g.ide - 1))
    mass = float((out["mu"].astype(np.float64)[R] + st["mub"].cpu().numpy().astype(np.float64)[R]).sum())
    d_cuda = abs(mass - float(ref["mass64"]))
    d_ref32 = abs(float(ref["mass32"]) - float(ref["mass64"]))
    assert d_cuda <= K_FLOOR * d_ref32 + 1e-9 * abs(float(ref["mass64"])), (d_cuda, d_ref32)


def test_wrf_solver_reads_classic_netcdf_files(tmp_path, monkeypatch):
    """WrfSolver.solve() with its default _load_datasets on the small case
    written as WRF files in the classic NetCDF format (no xarray): the fields
    match the fp64 reference fixtures as the in-memory drop-in does."""
    import sys

    from pywrf_b200 import WrfSolver, netcdf

    spec = synthetic.CaseSpec(**SMALL)
    inputs, bdy = synthetic.build(spec)
    netcdf.write_dataset(str(tmp_path / "wrf_inout_step3_nc"), inputs)
    netcdf.write_dataset(str(tmp_path / "wrfbdy_d01_nc"), bdy)
    monkeypatch.setenv("PYWRF_DATA_DIR", str(tmp_path))
    monkeypatch.setenv("PYWRF_RUN_NAME", "nc")
    monkeypatch.setitem(sys.modules, "xarray", None)
    res = WrfSolver(nsteps=SMALL["nsteps"], dt=spec.dt, p_top=spec.p_top, dx=spec.dx, dy=spec.dx).solve()
    r64, r32 = load_npz("small_ref64.npz"), load_npz("small_ref32.npz")
    got = {k: res[k].cpu().numpy() for k in ("u", "v", "w", "t", "ph", "mu")}
    got["qv"] = res["moist"][1].cpu().numpy()
    for k, v in got.items():
        err, floor = rel_l2(v, r64[k]), rel_l2(r32[k], r64[k])
        assert err <= K_FLOOR * floor + ABS_FLOOR, (k, err, floor)
