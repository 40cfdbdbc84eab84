"""The reference-signature shims (pywrf_b200.wrf_physics / wrf_dynamics)
called as the reference solver calls them, checked against the oracle."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import SMALL, rel_l2
from oracle import dynamics as OD
from oracle import physics as OP
from oracle.model import OracleModel
from pywrf_b200 import synthetic, wrf_dynamics, wrf_physics

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stepped():
    if not torch.cuda.is_available():
        pytest.fail("these tests need a CUDA device")
    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    m = OracleModel(g, inputs, bdy, np.float64)
    m.run(1)
    return g, m.st


def test_wsm6_shim_with_the_solver_arguments(stepped):
    g, s = stepped
    s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in s.items()}
    OP.moist_physics_prep_em(g, s)
    names = ("th_phy", "q1", "q2", "q3", "q4", "q5", "q6", "rho", "pi_phy", "p_phy", "dz8w")
    base = {k: (s["moist"][int(k[1])] if k.startswith("q") else s[k]).copy() for k in names}
    pre2 = {k: s[k].copy() for k in ("rainnc", "rainncv", "snownc", "snowncv", "graupelnc", "graupelncv", "sr")}

    def oracle(dtype):
        a = {k: v.astype(dtype) for k, v in base.items()}
        b = {k: v.astype(dtype) for k, v in pre2.items()}
        OP.wsm6(g, a["th_phy"], a["q1"], a["q2"], a["q3"], a["q4"], a["q5"], a["q6"], a["rho"], a["pi_phy"],
                a["p_phy"], a["dz8w"], float(g.dt), b["rainnc"], b["rainncv"], b["snownc"], b["snowncv"],
                b["graupelnc"], b["graupelncv"], b["sr"])
        return a, b

    o64, _ = oracle(np.float64)
    o32, _ = oracle(np.float32)
    d = {k: torch.tensor(v, dtype=torch.float32, device="cuda") for k, v in base.items()}
    d2 = {k: torch.tensor(v, dtype=torch.float32, device="cuda") for k, v in pre2.items()}
    refl = torch.zeros_like(d["th_phy"])
    ids, ide, jds, jde, kds, kde = g.ids + 1, g.ide - 1, g.jds + 1, g.jde - 1, 0, g.nz
    out = wrf_physics.wsm6(d["th_phy"], d["q1"], d["q2"], d["q3"], d["q4"], d["q5"], d["q6"], d["rho"], d["pi_phy"],
                           d["p_phy"], d["dz8w"], float(g.dt), 9.81, 1004.5, 1846.4, 287.0, 461.6,
                           273.149993896484375, 0.608362436294555664, 0.621750414371490479, 1.0e-15, 2850000.0,
                           2500000.0, 350000.0, 1.28, 1000.0, 4190.0, 2106.0, 610.78,
                           d2["rainnc"], d2["rainncv"], d2["snownc"], d2["snowncv"], d2["sr"], refl, 1, 1,
                           d2["graupelnc"], d2["graupelncv"], 0, 0, 0, 0, 0, 0,
                           ids, ide, jds, jde, kds, kde, 0, g.nx, 0, g.ny, 0, g.nz, ids, ide, jds, jde, kds, kde)
    torch.cuda.synchronize()
    assert out[0] is d["th_phy"] and out[7] is d2["rainnc"] and out[11] is d2["graupelnc"]
    for k in names[:7]:
        err, floor = rel_l2(d[k].cpu().numpy(), o64[k]), rel_l2(o32[k], o64[k])
        assert err <= 3.0 * floor + 1e-7, (k, err, floor)


def test_wsm6_shim_rejects_other_tiles_and_constants(stepped):
    g, _ = stepped
    z = torch.zeros((g.nz, g.ny, g.nx), device="cuda")
    z2 = torch.zeros((g.ny, g.nx), device="cuda")
    args = [z] * 11 + [45.0, 9.81, 1004.5, 1846.4, 287.0, 461.6, 273.149993896484375, 0.608362436294555664,
                       0.621750414371490479, 1.0e-15, 2850000.0, 2500000.0, 350000.0, 1.28, 1000.0, 4190.0, 2106.0,
                       610.78] + [z2] * 5 + [z, 1, 1] + [z2] * 2 + [0] * 6
    with pytest.raises(NotImplementedError):
        wrf_physics.wsm6(*args, 5, g.nx - 5, 5, g.ny - 5, 0, g.nz, 0, g.nx, 0, g.ny, 0, g.nz, 5, g.nx - 5, 5,
                         g.ny - 5, 0, g.nz)
    bad = list(args)
    bad[12] = 9.8
    with pytest.raises(ValueError):
        wrf_physics.wsm6(*bad, 6, g.nx - 6, 6, g.ny - 6, 0, g.nz, 0, g.nx, 0, g.ny, 0, g.nz, 6, g.nx - 6, 6,
                         g.ny - 6, 0, g.nz)
    with pytest.raises(TypeError):
        wrf_physics.wsm6(*([z.cpu()] + args[1:]), 6, g.nx - 6, 6, g.ny - 6, 0, g.nz, 0, g.nx, 0, g.ny, 0, g.nz,
                         6, g.nx - 6, 6, g.ny - 6, 0, g.nz)


def test_advect_scalar_shim_with_the_solver_arguments(stepped):
    g, s = stepped
    ref64 = np.zeros_like(s["t"])
    OD.advect_scalar(g, s["t"], ref64, s["ru"], s["rv"], s["ww"], s["msftx"], s["fnm"], s["fnp"], s["rdnw"])
    s32 = {k: s[k].astype(np.float32) for k in ("t", "ru", "rv", "ww", "msftx", "fnm", "fnp", "rdnw")}
    ref32 = np.zeros_like(s32["t"])
    OD.advect_scalar(g, s32["t"], ref32, s32["ru"], s32["rv"], s32["ww"], s32["msftx"], s32["fnm"], s32["fnp"],
                     s32["rdnw"])
    d = {k: torch.tensor(v, device="cuda") for k, v in s32.items()}
    tend = torch.zeros_like(d["t"])
    one = torch.ones((g.ny, g.nx), device="cuda")
    idx = (g.ids, g.ide, g.jds, g.jde, 0, g.nz, 0, g.nx, 0, g.ny, 0, g.nz, g.ids, g.ide, g.jds, g.jde, 0, g.nz)
    out = wrf_dynamics.advect_scalar(d["t"], d["t"], tend, d["ru"], d["rv"], d["ww"], None, None, None, g.dt,
                                     one, one, one, one, d["msftx"], one, d["fnm"], d["fnp"], 1.0 / g.dx,
                                     1.0 / g.dy, d["rdnw"], *idx)
    torch.cuda.synchronize()
    assert out is tend
    err, floor = rel_l2(tend.cpu().numpy(), ref64), rel_l2(ref32, ref64)
    assert err <= 3.0 * floor + 1e-9, (err, floor)


def _cuda(a):
    return torch.tensor(np.asarray(a), dtype=torch.float32, device="cuda").contiguous()


def test_calc_coef_w_shim_against_the_reference():
    """The reference-signature calc_coef_w against the reference's own
    coefficients (tests/golden/coefw_adj_ref64.npz, float64)."""
    from helpers import load_npz
    W = load_npz("coefw_adj_ref64.npz")
    nz, n = W["cqw"].shape[0], W["cqw"].shape[1]
    a, al, ga = (torch.zeros(nz, n, n, device="cuda") for _ in range(3))
    one = torch.ones(nz, device="cuda")
    idx = (5, n - 5, 5, n - 5, 0, nz, 0, n, 0, n, 0, nz, 5, n - 5, 5, n - 5, 0, nz)
    out = wrf_dynamics.calc_coef_w(a, al, ga, _cuda(W["mut"]), one, one, one, one, one, one, one, one, _cuda(W["cqw"]),
                                   _cuda(W["rdn"]), _cuda(W["rdnw"]), _cuda(W["c2a"]), float(W["dts"]), 9.81,
                                   float(W["epssm"]), False, *idx)
    torch.cuda.synchronize()
    assert out[0] is a and out[1] is al and out[2] is ga
    for mine, ref in ((a, W["a"]), (al, W["alpha"]), (ga, W["gamma"])):
        assert rel_l2(mine.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("var", ["t", "u", "v", "h"])
def test_relax_bdytend_shim_against_the_reference(var):
    """The reference-signature relax_bdytend against the reference's own
    tendency (tests/golden/relax_adj_ref64.npz, float64)."""
    from helpers import load_npz
    from pywrf_b200 import wrf_boundary
    Z = load_npz("relax_adj_ref64.npz")
    field = _cuda(Z[f"{var}_field"])
    tend = _cuda(Z[f"{var}_tend0"])
    nz, n = field.shape[0], field.shape[1]
    bdy = [_cuda(Z[f"{var}_{k}"]) for k in ("xs", "xe", "ys", "ye", "txs", "txe", "tys", "tye")]
    idx = (5, n - 5, 5, n - 5, 0, nz, 0, n, 0, n, 0, nz, 0, n, 0, n, 0, nz, 5, n - 5, 5, n - 5, 0, nz)
    out = wrf_boundary.relax_bdytend(field, tend, *bdy, var, 5, 1, 4, float(Z["dtbc"]), wrf_boundary.FCX,
                                     wrf_boundary.GCX, *idx)
    torch.cuda.synchronize()
    assert out is tend
    assert rel_l2(tend.cpu().numpy(), Z[f"{var}_tend"]) < 1e-6
    with pytest.raises(ValueError):
        wrf_boundary.relax_bdytend(field, tend, *bdy, var, 5, 1, 4, 1.0, [0.0, 1.0, 2.0, 3.0, 0.0],
                                   wrf_boundary.GCX, *idx)


def _c(a):
    return torch.tensor(np.asarray(a), dtype=torch.float32, device="cuda").contiguous()


@pytest.mark.parametrize("step", [0, 1])
def test_calc_p_rho_shim_with_the_solver_arguments(step):
    """calc_p_rho called with the reference's argument list against the
    reference's own outputs (tests/golden/prho_adj_ref64.npz); at a later
    step the caller's pm1 is updated in place, as in the reference."""
    from helpers import load_npz

    P = load_npz("prho_adj_ref64.npz")
    nz, n = P["p"].shape[0], P["p"].shape[1]
    one1 = torch.ones(nz, device="cuda")
    t = {k: _c(P[k]) for k in ("al", "p", "ph", "alt", "t_2", "t_1", "c2a", "pm1", "mu", "mut", "rdnw")}
    pm1_in = t["pm1"]
    al, p, pm1 = wrf_dynamics.calc_p_rho(t["al"], t["p"], t["ph"], t["alt"], t["t_2"], t["t_1"], t["c2a"], pm1_in,
                                         t["mu"], t["mut"], one1, one1 * 0, one1, one1 * 0, one1, one1 * 0, one1,
                                         one1 * 0, one1, 300.0, t["rdnw"], one1, float(P["smdiv"]), True, step,
                                         5, n - 5, 5, n - 5, 0, nz, 0, n, 0, n, 0, nz, 5, n - 5, 5, n - 5, 0, nz)
    assert (pm1 is pm1_in) == (step != 0)
    for nm, mine in (("al", al), ("p", p), ("pm1", pm1)):
        assert rel_l2(mine.cpu().numpy(), P[f"s{step}_{nm}_new"]) < 1e-6, nm


def test_advance_mu_t_shim_with_the_solver_arguments():
    """advance_mu_t called with the reference's argument list (as
    solver.py:1380-1393 calls it) against the reference's own outputs
    (tests/golden/mut_adj_ref64.npz)."""
    from helpers import load_npz

    T = load_npz("mut_adj_ref64.npz")
    nz, n = T["ww"].shape[0], T["ww"].shape[1]
    one1 = torch.ones(nz, device="cuda")
    t = {k: _c(T[k]) for k in T if not k.startswith(("cot_", "grad_", "fd_")) and not k.endswith("_new")
         and np.asarray(T[k]).ndim > 0}
    out = wrf_dynamics.advance_mu_t(t["ww"], t["ww_1"], t["u"], t["u_1"], t["v"], t["v_1"], t["mu"], t["mut"],
                                    t["muave"], t["muts"], t["muu"], t["muv"], t["mudf"], one1, one1 * 0, one1,
                                    one1 * 0, one1, one1 * 0, one1, one1 * 0, None, None, None, t["t"], t["t_1"],
                                    t["t_ave"], t["ft"], t["mu_tend"], 1.0 / float(T["dx"]), 1.0 / float(T["dy"]),
                                    float(T["dts"]), float(T["epssm"]), t["dnw"], t["fnm"], t["fnp"], t["rdnw"],
                                    t["msfuy"], t["msfuy"], t["msfvx_inv"], t["msfvx_inv"], t["msfvx_inv"],
                                    t["msftx"], t["msfty"], 1,
                                    5, n - 5, 5, n - 5, 0, nz, 0, n, 0, n, 0, nz, 5, n - 5, 5, n - 5, 0, nz)
    ww, ww_1, tt, t_ave, uam, vam, wwam, muave, muts, mudf, mu = out
    assert ww_1 is t["ww_1"] and uam is None
    for nm, mine in (("ww", ww), ("t", tt), ("t_ave", t_ave), ("muave", muave), ("muts", muts), ("mudf", mudf),
                     ("mu", mu)):
        assert rel_l2(mine.cpu().numpy(), T[f"{nm}_new"]) < 1e-6, nm
    # the inputs are left as they were (the reference clones them)
    assert torch.equal(t["ww"], _c(T["ww"])) and torch.equal(t["mu"], _c(T["mu"]))


def test_advance_w_shim_with_the_solver_arguments():
    """advance_w called with the reference's argument list against the
    reference's own outputs (tests/golden/advw_adj_ref64.npz)."""
    from helpers import load_npz

    A = load_npz("advw_adj_ref64.npz")
    nz, n = A["w"].shape[0], A["w"].shape[1]
    one1 = torch.ones(nz, device="cuda")
    t = {k: _c(A[k]) for k in A if not k.startswith(("cot_", "fd_")) and not k.endswith("_new")
         and np.asarray(A[k]).ndim > 0}
    t2a, w, ph = wrf_dynamics.advance_w(t["w"], t["rw_tend"], t["ww"], t["w_save"], t["u"], t["v"], t["muave"] * 0,
                                        t["mut"], t["muave"], t["muts"], one1, one1 * 0, one1, one1 * 0, one1,
                                        one1 * 0, one1, one1 * 0, t["t_2ave"], t["t_2"], t["t_1"], t["ph"],
                                        t["ph_1"], t["phb"], t["ph_tend"], t["ht"], t["c2a"], t["cqw"], t["alt"],
                                        t["alt"], t["a"], t["alpha"], t["gamma"], 1.0 / float(A["dx"]),
                                        1.0 / float(A["dy"]), float(A["dts"]), 300.0, float(A["epssm"]),
                                        1.0 / t["rdnw"], t["fnm"], t["fnp"], t["rdnw"], t["rdn"], float(A["cf1"]),
                                        float(A["cf2"]), float(A["cf3"]), t["msftx"], t["msfty"], False,
                                        5, n - 5, 5, n - 5, 0, nz, 0, n, 0, n, 0, nz, 5, n - 5, 5, n - 5, 0, nz)
    for nm, mine in (("t_2ave", t2a), ("w", w), ("ph", ph)):
        assert rel_l2(mine.cpu().numpy(), A[f"{nm}_new"]) < 1e-6, nm
