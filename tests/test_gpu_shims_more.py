"""The reference-signature drop-ins of the tendency terms, the flux
averages, the first stage's diffusion, rk_addtend_dry, the halo copies,
calc_p_rho_phi, advance_uv, the boundary updates and microphysics_driver
(pywrf_b200.wrf_dynamics / wrf_boundary / wrf_physics), called with the
arguments the reference solver passes, against the oracle's functions on
the same inputs: the CUDA result within 3x the float32 oracle's own error
against the float64 oracle (plus 1e-6); the copies exactly."""
from __future__ import annotations

import copy

import numpy as np
import pytest
import torch

from helpers import SMALL, rel_l2
from oracle import boundary as OB
from oracle import dynamics as OD
from oracle.model import OracleModel
from pywrf_b200 import synthetic, wrf_boundary, wrf_dynamics, wrf_physics

pytestmark = pytest.mark.gpu

TAGS = ("s1.km", "s1.forces", "s1.diff", "s2.adv", "s2.tend", "s2.acprep", "s2.sub1", "s2.moist", "mp")


@pytest.fixture(scope="module")
def snaps():
    if not torch.cuda.is_available():
        pytest.fail("these tests need a CUDA device")
    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    out = {}

    def probe(name, m):
        if name in TAGS and name not in out:
            out[name] = copy.deepcopy(m.st)

    m = OracleModel(g, inputs, bdy, np.float64)
    m.run(1)
    m.step(2, probe)
    return g, out


def _c(a):
    return torch.tensor(np.asarray(a), dtype=torch.float32, device="cuda").contiguous()


def _cast(s, dtype):
    return {k: (np.array(v, dtype) if isinstance(v, np.ndarray) else v) for k, v in s.items() if k != "bdy"}


def _frame_args(g):
    ids, ide, jds, jde = g.ids, g.ide, g.jds, g.jde
    return dict(ids=ids, ide=ide, jds=jds, jde=jde, kds=0, kde=g.nz, ims=0, ime=g.nx, jms=0, jme=g.ny, kms=0,
                kme=g.nz, its=ids, ite=ide, jts=jds, jte=jde, kts=0, kte=g.nz)


def _close(name, cuda, o64, o32):
    c = cuda.detach().double().cpu().numpy()
    err, floor = rel_l2(c, o64), rel_l2(o32, o64)
    assert err <= 3.0 * floor + 1e-6, (name, err, floor)


def _oracle_forces(g, s, which):
    if which == "rhs_ph":
        OD.rhs_ph(g, s["ph_tend"], s["u"], s["v"], s["ww"], s["ph"], s["phb"], s["w"], s["mut"], s["muu"], s["muv"],
                  s["fnm"], s["fnp"], s["rdnw"], s["cfn"], s["cfn1"], s["msfux"], s["msfvy"], s["msfty"])
    elif which == "hpg":
        OD.horizontal_pressure_gradient(g, s["ru_tend"], s["rv_tend"], s["ph"], s["alt"], s["p"], s["pb"], s["al"],
                                        s["php"], s["cqu"], s["cqv"], s["muu"], s["muv"], s["mu"], s["fnm"],
                                        s["fnp"], s["rdnw"], s["cf1"], s["cf2"], s["cf3"], s["msfux"], s["msfuy"],
                                        s["msfvx"], s["msfvy"])
    elif which == "pg_buoy_w":
        OD.pg_buoy_w(g, s["rw_tend"], s["p"], s["cqw"], s["mu"], s["mub"], s["rdnw"], s["rdn"], s["msfty"])
    elif which == "coriolis":
        OD.coriolis(g, s["ru"], s["rv"], s["rw"], s["ru_tend"], s["rv_tend"], s["rw_tend"], s["msftx"], s["msfty"],
                    s["msfux"], s["msfuy"], s["msfvx"], s["msfvy"], s["f"], s["e"], s["sina"], s["cosa"], s["fnm"],
                    s["fnp"])
    else:
        OD.curvature(g, s["ru"], s["rv"], s["rw"], s["u"], s["v"], s["ru_tend"], s["rv_tend"], s["rw_tend"],
                     s["msfux"], s["msfuy"], s["msfvx"], s["msfvy"], s["msftx"], s["msfty"], s["fnm"], s["fnp"])
    return s


@pytest.mark.parametrize("which", ["rhs_ph", "hpg", "pg_buoy_w", "coriolis", "curvature"])
def test_tendency_term_drop_ins(snaps, which):
    g, sn = snaps
    base = sn["s2.adv"]
    o64 = _oracle_forces(g, _cast(base, np.float64), which)
    o32 = _oracle_forces(g, _cast(base, np.float32), which)
    d = {k: _c(v) for k, v in base.items() if isinstance(v, np.ndarray) and v.dtype != object}
    fa = _frame_args(g)
    sc = {k: float(base[k]) for k in ("cf1", "cf2", "cf3", "cfn", "cfn1")}
    one = torch.ones(g.nz, device="cuda")
    if which == "rhs_ph":
        out = wrf_dynamics.rhs_ph(d["ph_tend"], d["u"], d["v"], d["ww"], d["ph"], d["ph"], d["phb"], d["w"], d["mut"],
                                  d["muu"], d["muv"], one, one, d["fnm"], d["fnp"], d["rdnw"], sc["cfn"], sc["cfn1"],
                                  g.rdx, g.rdy, d["msfux"], d["msfuy"], d["msfvx"], d["msfvx_inv"], d["msfvy"],
                                  d["msftx"], d["msfty"], True, **fa)
        pairs = [("ph_tend", out)]
    elif which == "hpg":
        out = wrf_dynamics.horizontal_pressure_gradient(
            d["ru_tend"], d["rv_tend"], d["ph"], d["alt"], d["p"], d["pb"], d["al"], d["php"], d["cqu"], d["cqv"],
            d["muu"], d["muv"], d["mu"], one, one, d["fnm"], d["fnp"], d["rdnw"], sc["cf1"], sc["cf2"], sc["cf3"],
            sc["cfn"], sc["cfn1"], g.rdx, g.rdy, d["msfux"], d["msfuy"], d["msfvx"], d["msfvy"], d["msftx"],
            d["msfty"], True, False, **fa)
        pairs = [("ru_tend", out[0]), ("rv_tend", out[1])]
    elif which == "pg_buoy_w":
        out = wrf_dynamics.pg_buoy_w(d["rw_tend"], d["p"], d["cqw"], d["mu"], d["mub"], one, one, d["rdnw"], d["rdn"],
                                     9.81, d["msftx"], d["msfty"], **fa)
        pairs = [("rw_tend", out[0]), ("cqw", out[1])]
    elif which == "coriolis":
        out = wrf_dynamics.coriolis(d["ru"], d["rv"], d["rw"], d["ru_tend"], d["rv_tend"], d["rw_tend"], d["msftx"],
                                    d["msfty"], d["msfux"], d["msfuy"], d["msfvx"], d["msfvy"], d["f"], d["e"],
                                    d["sina"], d["cosa"], d["fnm"], d["fnp"], **fa)
        pairs = [("ru_tend", out[0]), ("rv_tend", out[1]), ("rw_tend", out[2])]
    else:
        out = wrf_dynamics.curvature(d["ru"], d["rv"], d["rw"], d["u"], d["v"], d["w"], d["ru_tend"], d["rv_tend"],
                                     d["rw_tend"], d["msfux"], d["msfuy"], d["msfvx"], d["msfvy"], d["msftx"],
                                     d["msfty"], d["clat"], d["fnm"], d["fnp"], g.rdx, g.rdy, **fa)
        pairs = [("ru_tend", out[0]), ("rv_tend", out[1]), ("rw_tend", out[2])]
    torch.cuda.synchronize()
    for k, t in pairs:
        assert t is d[k]  # in place, as the reference
        _close(f"{which}:{k}", t, o64[k], o32[k])


def test_sumflux_drop_in(snaps):
    g, sn = snaps
    base = sn["s2.sub1"]

    def oracle(dtype):
        s = _cast(base, dtype)
        OD.sumflux(g, s, 2, 2)
        return s

    o64, o32 = oracle(np.float64), oracle(np.float32)
    d = {k: _c(base[k]) for k in ("u", "v", "ww", "u_save", "v_save", "ww1", "muu", "muv", "ru_m", "rv_m", "ww_m",
                                  "msfux", "msfuy", "msfvx", "msfvx_inv", "msfvy")}
    one = torch.ones(g.nz, device="cuda")
    out = wrf_dynamics.sumflux(d["u"], d["v"], d["ww"], d["u_save"], d["v_save"], d["ww1"], d["muu"], d["muv"],
                               one, one, one, one, one, one, one, one, d["ru_m"], d["rv_m"], d["ww_m"], 0.1,
                               d["msfux"], d["msfuy"], d["msfvx"], d["msfvx_inv"], d["msfvy"], 2, 2, **_frame_args(g))
    torch.cuda.synchronize()
    for k, t in zip(("ru_m", "rv_m", "ww_m"), out):
        assert t is d[k]
        _close(f"sumflux:{k}", t, o64[k], o32[k])


@pytest.mark.parametrize("name", ["u", "v", "w", "t", "qc"])
def test_horizontal_diffusion_drop_ins(snaps, name):
    g, sn = snaps
    base = sn["s1.km"]
    field_of = lambda s: s["moist"][2] if name == "qc" else s[name]  # noqa: E731
    mut_name = "muts" if name == "qc" else "mut"
    xk_name = "xkmh" if name in ("u", "v", "w") else "xkhh"
    maps = ("msfux", "msfuy", "msfvx", "msfvx_inv", "msfvy", "msftx", "msfty")

    def oracle(dtype):
        s = _cast(base, dtype)
        tend = np.zeros_like(s["t"])
        OD.horizontal_diffusion(g, name if name != "qc" else "m", field_of(s), tend, s[mut_name],
                                *[s[k] for k in maps], s[xk_name], base=s["t_init"] if name == "t" else None)
        return tend

    o64, o32 = oracle(np.float64), oracle(np.float32)
    d = {k: _c(base[k]) for k in maps + (mut_name, xk_name, "t_init")}
    field = _c(field_of(base))
    tend = torch.zeros_like(field)
    fa = _frame_args(g)
    fa.pop("ips", None)
    if name == "t":
        out = wrf_dynamics.horizontal_diffusion_3dmp("t", field, tend, d[mut_name], 1.0, 0.0, d["t_init"],
                                                     *[d[k] for k in maps], 0.0, d[xk_name], g.rdx, g.rdy, **fa)
    else:
        out = wrf_dynamics.horizontal_diffusion(name if name != "qc" else "qc", field, tend, d[mut_name], 1.0, 0.0,
                                                *[d[k] for k in maps], 0.0, d[xk_name], g.rdx, g.rdy, **fa)
    torch.cuda.synchronize()
    assert out is tend
    _close(f"hdiff:{name}", out, o64, o32)


@pytest.mark.parametrize("rk_step", [1, 2])
def test_rk_addtend_dry_drop_in(snaps, rk_step):
    g, sn = snaps
    base = sn["s1.diff"]
    names = ("ru_tend", "rv_tend", "rw_tend", "ph_tend", "t_tend", "ru_tendf", "rv_tendf", "rw_tendf", "ph_tendf",
             "t_tendf", "u_save", "v_save", "w_save", "ph_save", "t_save", "mu_tend", "mu_tendf")

    def oracle(dtype):
        s = _cast(base, dtype)
        OD.rk_addtend_dry(g, *[s[k] for k in names], rk_step, s["h_diabatic"], s["mut"], s["msfty"], s["msfuy"],
                          s["msfvx"], s["msfvx_inv"])
        return s

    o64, o32 = oracle(np.float64), oracle(np.float32)
    d = {k: _c(base[k]) for k in names + ("h_diabatic", "mut", "msftx", "msfty", "msfux", "msfuy", "msfvx",
                                          "msfvx_inv", "msfvy")}
    fa = _frame_args(g)
    out = wrf_dynamics.rk_addtend_dry(*[d[k] for k in names], rk_step, 1.0, 0.0, d["h_diabatic"], d["mut"],
                                      d["msftx"], d["msfty"], d["msfux"], d["msfuy"], d["msfvx"], d["msfvx_inv"],
                                      d["msfvy"], fa["ids"], fa["ide"], fa["jds"], fa["jde"], 0, g.nz, 0, g.nx, 0,
                                      g.ny, 0, g.nz, fa["ids"], fa["ide"], fa["jds"], fa["jde"], 0, g.nz, fa["its"],
                                      fa["ite"], fa["jts"], fa["jte"], 0, g.nz)
    torch.cuda.synchronize()
    for k, t in zip(("ru_tend", "rv_tend", "rw_tend", "ph_tend", "t_tend", "mu_tend"), out):
        assert t is d[k]
        _close(f"addtend:{k}", t, o64[k], o32[k])
    if rk_step == 1:
        for k in ("ru_tendf", "rv_tendf", "rw_tendf", "ph_tendf", "t_tendf"):
            _close(f"addtend:{k}", d[k], o64[k], o32[k])


@pytest.mark.parametrize("var", ["u", "v", "w", "t", "p", "e", "f"])
def test_halo_drop_ins(var):
    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    rng = np.random.default_rng(5)
    a = rng.standard_normal((g.nz, g.ny, g.nx)).astype(np.float32)
    ref = a.copy()
    OD.set_physical_bc3d(g, ref, var)
    t = _c(a)
    fa = _frame_args(g)
    out = wrf_dynamics.set_physical_bc3d(t, var, fa["ids"], fa["ide"], fa["jds"], fa["jde"], 0, g.nz, 0, g.nx, 0,
                                         g.ny, 0, g.nz, fa["ids"], fa["ide"], fa["jds"], fa["jde"], 0, g.nz,
                                         fa["its"], fa["ite"], fa["jts"], fa["jte"], 0, g.nz)
    assert out is t
    assert np.array_equal(t.cpu().numpy(), ref)
    if var in ("u", "v", "t"):
        b = rng.standard_normal((g.ny, g.nx)).astype(np.float32)
        ref2 = b.copy()
        OD.set_physical_bc2d(g, ref2, var)
        t2 = _c(b)
        wrf_dynamics.set_physical_bc2d(t2, var, fa["ids"], fa["ide"], fa["jds"], fa["jde"], 0, g.nx, 0, g.ny,
                                       fa["ids"], fa["ide"], fa["jds"], fa["jde"], fa["its"], fa["ite"], fa["jts"],
                                       fa["jte"])
        assert np.array_equal(t2.cpu().numpy(), ref2)


def test_calc_p_rho_phi_drop_in(snaps):
    g, sn = snaps
    base = sn["s2.moist"]

    def oracle(dtype):
        s = _cast(base, dtype)
        OD.calc_p_rho_phi(g, s["moist"][1], s["al"], s["alb"], s["mu"], s["muts"], s["ph"], s["p"], s["pb"], s["t"],
                          s["rdnw"])
        return s

    o64, o32 = oracle(np.float64), oracle(np.float32)
    d = {k: _c(base[k]) for k in ("moist", "al", "alb", "mu", "muts", "ph", "phb", "p", "pb", "t", "znu", "znw",
                                  "dnw", "rdnw", "rdn")}
    one = torch.ones(g.nz, device="cuda")
    out = wrf_dynamics.calc_p_rho_phi(d["moist"], 7, 0, d["al"], d["alb"], d["mu"], d["muts"], one, one, one, one,
                                      one, one, d["ph"], d["phb"], d["p"], d["pb"], d["t"], 1.0e5, 300.0, 5000.0,
                                      d["znu"], d["znw"], d["dnw"], d["rdnw"], d["rdn"], True, **_frame_args(g))
    torch.cuda.synchronize()
    assert out[0] is d["al"] and out[1] is d["p"] and out[2] is d["ph"]
    _close("eos:al", d["al"], o64["al"], o32["al"])
    _close("eos:p", d["p"], o64["p"], o32["p"])


def test_advance_uv_drop_in(snaps):
    g, sn = snaps
    base = sn["s2.acprep"]
    dts = g.dt / g.soundsteps
    names = ("u", "ru_tend", "v", "rv_tend", "p", "pb", "ph", "php", "alt", "al", "mu", "muu", "cqu", "muv", "cqv",
             "mudf", "msfux", "msfuy", "msfvx", "msfvx_inv", "msfvy")

    def oracle(dtype):
        s = _cast(base, dtype)
        OD.advance_uv(g, *[s[k] for k in names], dts, s["cf1"], s["cf2"], s["cf3"], s["fnm"], s["fnp"], g.emdiv,
                      s["rdnw"])
        return s

    o64, o32 = oracle(np.float64), oracle(np.float32)
    d = {k: _c(base[k]) for k in names + ("fnm", "fnp", "rdnw")}
    u0, v0 = d["u"].clone(), d["v"].clone()
    one = torch.ones(g.nz, device="cuda")
    u, v = wrf_dynamics.advance_uv(d["u"], d["ru_tend"], d["v"], d["rv_tend"], d["p"], d["pb"], d["ph"], d["php"],
                                   d["alt"], d["al"], d["mu"], d["muu"], d["cqu"], d["muv"], d["cqv"], d["mudf"],
                                   one, one, one, one, one, one, one, one, d["msfux"], d["msfuy"], d["msfvx"],
                                   d["msfvx_inv"], d["msfvy"], g.rdx, g.rdy, dts, float(base["cf1"]),
                                   float(base["cf2"]), float(base["cf3"]), d["fnm"], d["fnp"], g.emdiv, d["rdnw"], 1,
                                   True, False, **_frame_args(g))
    torch.cuda.synchronize()
    assert torch.equal(d["u"], u0) and torch.equal(d["v"], v0)  # new tensors, as the reference
    _close("advance_uv:u", u, o64["u"], o32["u"])
    _close("advance_uv:v", v, o64["v"], o32["v"])


def test_boundary_drop_ins(snaps):
    g, sn = snaps
    base = sn["s2.adv"]
    bd = base["bdy"]
    dts = g.dt / g.soundsteps
    fa = dict(_frame_args(g))
    fb = (fa["ids"], fa["ide"], fa["jds"], fa["jde"], 0, g.nz, 0, g.nx, 0, g.ny, 0, g.nz, fa["ids"], fa["ide"],
          fa["jds"], fa["jde"], 0, g.nz, fa["its"], fa["ite"], fa["jts"], fa["jte"], 0, g.nz)
    # spec_bdytend of u and of the 2-D mu
    for var, name, fld in (("u", "ru_tend", "u"), ("m", "mu_tend", "mu")):
        o = {}
        for dtype in (np.float64, np.float32):
            t = np.array(base[name], dtype)
            OB.spec_bdytend(g, t[None] if var == "m" else t, {k: np.array(v, dtype) for k, v in bd[fld].items()}, var)
            o[dtype] = t
        t = _c(base[name])
        b = [_c(bd[fld][k]) for k in ("xs", "xe", "ys", "ye", "txs", "txe", "tys", "tye")]
        out = wrf_boundary.spec_bdytend(t, *b, var, 5, 1, *fb)
        assert out is t
        _close(f"spec_bdytend:{var}", t, o[np.float64], o[np.float32])
    # spec_bdyupdate of t and of the 2-D mu
    for var, name, tname in (("t", "t", "t_tend"), ("m", "mu", "mu_tend")):
        o = {}
        for dtype in (np.float64, np.float32):
            f, tt = np.array(base[name], dtype), np.array(base[tname], dtype)
            OB.spec_bdyupdate(g, f, tt, dts, var)
            o[dtype] = f
        f = _c(base[name])
        out = wrf_boundary.spec_bdyupdate(f, _c(base[tname]), dts, var, 1, *fb)
        assert out is f
        _close(f"spec_bdyupdate:{var}", f, o[np.float64], o[np.float32])
    # spec_bdyupdate_ph and zero_grad_bdy(w)
    o = {}
    for dtype in (np.float64, np.float32):
        s = _cast(base, dtype)
        OB.spec_bdyupdate_ph(g, s["ph_save"], s["ph"], s["ph_tend"], s["mu_tend"], s["muts"], dts)
        OB.zero_grad_bdy(g, s["w"], "w")
        o[dtype] = s
    d = {k: _c(base[k]) for k in ("ph_save", "ph", "ph_tend", "mu_tend", "muts", "w")}
    wrf_boundary.spec_bdyupdate_ph(d["ph_save"], d["ph"], d["ph_tend"], d["mu_tend"], d["muts"], 1.0, 0.0, dts, "h",
                                   1, *fb)
    wrf_boundary.zero_grad_bdy(d["w"], "w", 1, *fb)
    torch.cuda.synchronize()
    _close("spec_bdyupdate_ph", d["ph"], o[np.float64]["ph"], o[np.float32]["ph"])
    assert np.array_equal(d["w"].cpu().numpy(), o[np.float32]["w"])


def test_microphysics_driver_drop_in_equals_wsm6(snaps):
    from oracle import physics as OP

    g, sn = snaps
    s = _cast(sn["s2.moist"], np.float64)
    OP.moist_physics_prep_em(g, s)
    names = ("th_phy", "rho", "pi_phy", "p_phy", "dz8w")
    flat = ("rainnc", "rainncv", "snownc", "snowncv", "sr", "graupelnc", "graupelncv")
    runs = []
    for driver in (True, False):
        d = {k: _c(s[k]) for k in names + flat}
        q = [_c(s["moist"][i]) for i in range(1, 7)]
        refl = torch.zeros_like(d["th_phy"])
        ids, ide, jds, jde = g.ids + 1, g.ide - 1, g.jds + 1, g.jde - 1
        idx = (ids, ide, jds, jde, 0, g.nz, 0, g.nx, 0, g.ny, 0, g.nz, ids, ide, jds, jde, 0, g.nz)
        if driver:
            out = wrf_physics.microphysics_driver(d["th_phy"], d["rho"], d["pi_phy"], d["p_phy"], None, d["dz8w"], None,
                                                  float(g.dt), 9000.0, 9000.0, *q, d["rainnc"], d["rainncv"],
                                                  d["snownc"], d["snowncv"], d["sr"], refl, 1, 1, d["graupelnc"],
                                                  d["graupelncv"], 0, 0, 0, 0, 0, 0, *idx)
        else:
            out = wrf_physics.wsm6(d["th_phy"], *q, d["rho"], d["pi_phy"], d["p_phy"], d["dz8w"], float(g.dt), 9.81,
                                   1004.5, 1846.4, 287.0, 461.6, 273.149993896484375, 0.608362436294555664,
                                   0.621750414371490479, 1.0e-15, 2850000.0, 2500000.0, 350000.0, 1.28, 1000.0,
                                   4190.0, 2106.0, 610.78, d["rainnc"], d["rainncv"], d["snownc"], d["snowncv"],
                                   d["sr"], refl, 1, 1, d["graupelnc"], d["graupelncv"], 0, 0, 0, 0, 0, 0, *idx)
        torch.cuda.synchronize()
        runs.append([t.cpu().numpy() for t in out[:14]])
    for a, b in zip(*runs):
        assert np.array_equal(a, b)
