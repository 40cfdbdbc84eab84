"""The golden advect_scalar cotangents (made by the reference's autograd,
tests/golden/make_golden_adjoint.py) against the oracle's forward: the oracle
reproduces the reference's tendency on the fixture's inputs, and central
finite differences of the oracle along random directions equal the golden
gradients' directional derivatives."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import load_npz
from oracle import boundary as OB
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


R = load_npz("relax_adj_ref64.npz")
FCX = np.array([0., 5.5555557e-3, 3.7037039e-3, 1.8518519e-3, 0.])
GCX = np.array([0., 1.1111111e-3, 7.4074074e-4, 3.7037037e-4, 0.])


def _relax(g, var, field):
    t = R[f"{var}_tend0"].copy()
    bd = {k: R[f"{var}_{k}"] for k in ("xs", "xe", "ys", "ye", "txs", "txe", "tys", "tye")}
    OB.relax_bdytend(g, field, t, bd, var, float(R["dtbc"]), FCX, GCX)
    return t


def test_relax_golden_pinned_by_the_oracle():
    """The oracle's relax_bdytend reproduces the reference's tendency on the
    fixture, and (being linear in the field) its finite differences give the
    golden gradient's directional derivatives."""
    g = _grid()
    rng = np.random.default_rng(4)
    for var in ("t", "u", "v", "h"):
        f = R[f"{var}_field"]
        assert np.abs(_relax(g, var, f) - R[f"{var}_tend"]).max() <= 1e-12 * np.abs(R[f"{var}_tend"]).max()
        d = rng.standard_normal(f.shape)
        fd = float(((_relax(g, var, f + d) - _relax(g, var, f - d)) * R[f"{var}_cot"]).sum()) / 2.0
        an = float((d * R[f"{var}_grad_field"]).sum())
        assert abs(fd - an) <= 1e-9 * abs(an), (var, fd, an)


W = load_npz("coefw_adj_ref64.npz")


def _coefw(g, mut, cqw, c2a):
    a, al, ga = (np.zeros_like(W["cqw"]) for _ in range(3))
    OD.calc_coef_w(g, a, al, ga, mut, cqw, W["rdn"], W["rdnw"], c2a, float(W["dts"]), float(W["epssm"]))
    return a, al, ga


def test_coefw_fixture_pinned_by_the_oracle():
    """The oracle's calc_coef_w reproduces the reference's coefficients on the
    fixture, and its central finite differences reproduce the fixture's
    (made from the reference's forward: its autograd cannot differentiate
    calc_coef_w, which updates gamma in place)."""
    g = _grid()
    a, al, ga = _coefw(g, W["mut"], W["cqw"], W["c2a"])
    for mine, ref in ((a, W["a"]), (al, W["alpha"]), (ga, W["gamma"])):
        assert np.abs(mine - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1.0)
    base = {"mut": W["mut"], "cqw": W["cqw"], "c2a": W["c2a"]}

    def loss(x):
        a, al, ga = _coefw(g, x["mut"], x["cqw"], x["c2a"])
        return float((a * W["cot_a"]).sum() + (al * W["cot_alpha"]).sum() + (ga * W["cot_gamma"]).sum())

    for name in base:
        d = W[f"dir_{name}_0"]
        eps = 1e-6 * float(np.abs(base[name]).max())
        xp, xm = dict(base), dict(base)
        xp[name] = base[name] + eps * d
        xm[name] = base[name] - eps * d
        fd = (loss(xp) - loss(xm)) / (2 * eps)
        ref = float(W[f"fd_{name}_0"])
        assert abs(fd - ref) <= 1e-6 * abs(ref), (name, fd, ref)


M = load_npz("adv_mom_adj_ref64.npz")


def _mom_dir(n, r, shape):
    # the directions of make_golden_adjoint.mom_direction
    return np.random.default_rng(7000 + 10 * n + r).standard_normal(shape)


def _mom(g, comp, field, ru, rv, rom):
    t = np.zeros_like(field, dtype=np.float64)
    f64 = {k: np.asarray(v, np.float64) for k, v in dict(field=field, ru=ru, rv=rv, rom=rom).items()}
    prof = {k: M[k].astype(np.float64) for k in ("fnm", "fnp", "rdnw", "rdn")}
    msf = M[f"{comp}_msf"].astype(np.float64)
    if comp == "u":
        OD.advect_u(g, f64["field"], t, f64["ru"], f64["rv"], f64["rom"], msf, prof["fnm"], prof["fnp"], prof["rdnw"])
    elif comp == "v":
        OD.advect_v(g, f64["field"], t, f64["ru"], f64["rv"], f64["rom"], M["v_msf2"].astype(np.float64), msf,
                    prof["fnm"], prof["fnp"], prof["rdnw"])
    else:
        OD.advect_w(g, f64["field"], t, f64["ru"], f64["rv"], f64["rom"], msf, prof["fnm"], prof["fnp"], prof["rdn"])
    return t


def test_momentum_fixture_pinned_by_the_oracle():
    """advect_u / advect_v / advect_w: the oracle reproduces the reference's
    tendencies on the fixture; for u and v the golden autograd gradients'
    directional derivatives equal the oracle's central differences, and for w
    (whose reference backward raises) the oracle's central differences equal
    the fixture's, made from the reference's float64 forward."""
    g = _grid()
    assert g.dx == float(M["dx"])
    names = ("field", "ru", "rv", "rom")
    for comp in ("u", "v", "w"):
        base = {k: M[f"{comp}_{k}"].astype(np.float64) for k in names}
        ref = M[f"{comp}_tend"]
        assert np.abs(_mom(g, comp, **base) - ref).max() <= 1e-12 * np.abs(ref).max(), comp
        cot = M[f"{comp}_cot"].astype(np.float64)
        for n, name in enumerate(names):
            d = _mom_dir(n, 0, base[name].shape)
            eps = 1e-6 * float(np.abs(base[name]).max())
            xp, xm = dict(base), dict(base)
            xp[name] = base[name] + eps * d
            xm[name] = base[name] - eps * d
            fd = float(((_mom(g, comp, **xp) - _mom(g, comp, **xm)) * cot).sum()) / (2 * eps)
            if comp == "w":
                want = float(M[f"w_fd_{name}_0"])
            else:
                want = float((d * M[f"{comp}_grad_{name}"]).sum())
            assert abs(fd - want) <= 1e-6 * abs(want) + 1e-9, (comp, name, fd, want)


V = load_npz("advuv_adj_ref64.npz")
UV3 = ("u", "ru_tend", "v", "rv_tend", "p", "pb", "ph", "php", "alt", "al", "cqu", "cqv")
UV2 = ("mu", "muu", "muv", "mudf")


def _uv_dir(n, r, shape):
    # the directions of make_golden_adjoint.uv_direction
    return np.random.default_rng(8000 + 100 * n + r).standard_normal(shape)


def _advance_uv(g, x):
    x = {k: np.array(v, np.float64) for k, v in x.items()}
    c = {k: V[k].astype(np.float64) for k in ("msfux", "msfuy", "msfvx", "msfvx_inv", "msfvy", "fnm", "fnp", "rdnw")}
    u, v = OD.advance_uv(g, x["u"], x["ru_tend"], x["v"], x["rv_tend"], x["p"], x["pb"], x["ph"], x["php"], x["alt"],
                         x["al"], x["mu"], x["muu"], x["cqu"], x["muv"], x["cqv"], x["mudf"], c["msfux"], c["msfuy"],
                         c["msfvx"], c["msfvx_inv"], c["msfvy"], float(V["dts"]), float(V["cf1"]), float(V["cf2"]),
                         float(V["cf3"]), c["fnm"], c["fnp"], float(V["emdiv"]), c["rdnw"])
    OB.spec_bdyupdate(g, u, x["ru_tend"], float(V["dts"]), "u")
    OB.spec_bdyupdate(g, v, x["rv_tend"], float(V["dts"]), "v")
    return u, v


def test_advance_uv_fixture_pinned_by_the_oracle():
    """advance_uv + spec_bdyupdate(u), (v): the oracle reproduces the
    reference's u, v on the fixture, and its central differences reproduce
    the fixture's (made from the reference's float64 forward: its autograd
    cannot differentiate advance_uv)."""
    g = _grid()
    base = {k: V[k].astype(np.float64) for k in UV3 + UV2}
    u, v = _advance_uv(g, base)
    for mine, ref in ((u, V["u_new"]), (v, V["v_new"])):
        assert np.abs(mine - ref).max() <= 1e-12 * np.abs(ref).max()
    cu, cv = V["cot_u"].astype(np.float64), V["cot_v"].astype(np.float64)
    for n, name in enumerate(UV3 + UV2):
        d = _uv_dir(n, 0, base[name].shape)
        eps = 1e-6 * float(np.abs(base[name]).max())
        xp, xm = dict(base), dict(base)
        xp[name] = base[name] + eps * d
        xm[name] = base[name] - eps * d
        up, vp = _advance_uv(g, xp)
        um, vm = _advance_uv(g, xm)
        fd = float(((up - um) * cu).sum() + ((vp - vm) * cv).sum()) / (2 * eps)
        ref = float(V[f"fd_{name}_0"])
        assert abs(fd - ref) <= 1e-6 * abs(ref) + 1e-9, (name, fd, ref)


P = load_npz("prho_adj_ref64.npz")
PRHO_IN = ("al", "p", "ph", "alt", "t_2", "t_1", "c2a", "pm1", "mu", "mut")


def _prho(g, x, step):
    x = {k: np.array(v, np.float64) for k, v in x.items()}
    pm1 = OD.calc_p_rho(g, x["al"], x["p"], x["ph"], x["alt"], x["t_2"], x["t_1"], x["c2a"], x["pm1"], x["mu"],
                        x["mut"], P["rdnw"].astype(np.float64), float(P["smdiv"]), step)
    return x["al"], x["p"], pm1


def test_calc_p_rho_fixture_pinned_by_the_oracle():
    """calc_p_rho at step 0 and 1: the oracle reproduces the reference's al,
    p, pm1 on the fixture, and its central differences give the golden
    autograd gradients' directional derivatives."""
    g = _grid()
    rng = np.random.default_rng(5)
    base = {k: P[k].astype(np.float64) for k in PRHO_IN}
    cot = {k: P[f"cot_{k}"].astype(np.float64) for k in ("al", "p", "pm1")}
    for step in (0, 1):
        outs = _prho(g, base, step)
        for nm, mine in zip(("al", "p", "pm1"), outs):
            ref = P[f"s{step}_{nm}_new"]
            assert np.abs(mine - ref).max() <= 1e-12 * np.abs(ref).max(), (step, nm)

        def loss(x):
            return sum(float((o * cot[nm]).sum()) for nm, o in zip(("al", "p", "pm1"), _prho(g, x, step)))

        for name in PRHO_IN:
            d = rng.standard_normal(base[name].shape)
            # a larger step than for the bilinear operators: the loss is
            # ~1e7, and the operator is smooth (rational in t_1 and mut)
            eps = 1e-4 * float(np.abs(base[name]).max())
            xp, xm = dict(base), dict(base)
            xp[name] = base[name] + eps * d
            xm[name] = base[name] - eps * d
            fd = (loss(xp) - loss(xm)) / (2 * eps)
            an = float((d * P[f"s{step}_grad_{name}"].astype(np.float64)).sum())
            assert abs(fd - an) <= 1e-5 * abs(an) + 1e-9, (step, name, fd, an)


T = load_npz("mut_adj_ref64.npz")
MUT3 = ("ww", "ww_1", "u", "u_1", "v", "v_1", "t", "t_1", "t_ave", "ft")
MUT2 = ("mu", "mut", "muave", "muts", "muu", "muv", "mudf", "mu_tend")
MUT_OUT = ("ww", "t", "t_ave", "muave", "muts", "mudf", "mu")
# the oracle's state-dict names of advance_mu_t's arguments
_MUT_ST = {"ww_1": "ww1", "u_1": "u_save", "v_1": "v_save", "t_1": "t_save", "t_ave": "t_2save", "ft": "t_tend"}


def _mut_dir(n, r, shape):
    # the directions of make_golden_adjoint.mut_direction
    return np.random.default_rng(9000 + 100 * n + r).standard_normal(shape)


def _advance_mu_t(g, x):
    st = {_MUT_ST.get(k, k): np.array(v, np.float64) for k, v in x.items()}
    for k in ("msftx", "msfty", "msfuy", "msfvx_inv", "dnw", "fnm", "fnp", "rdnw"):
        st[k] = T[k].astype(np.float64)
    OD.advance_mu_t(g, st, float(T["dts"]), float(T["epssm"]), 1)
    return {o: st[_MUT_ST.get(o, o)] for o in MUT_OUT}


def test_advance_mu_t_fixture_pinned_by_the_oracle():
    """advance_mu_t: the oracle reproduces the reference's seven outputs on
    the fixture, and its central differences equal the fixture's (of the
    reference's float64 forward)."""
    g = _grid()
    base = {k: T[k].astype(np.float64) for k in MUT3 + MUT2}
    outs = _advance_mu_t(g, base)
    for o in MUT_OUT:
        ref = T[f"{o}_new"]
        assert np.abs(outs[o] - ref).max() <= 1e-12 * np.abs(ref).max(), o
    cot = {o: T[f"cot_{o}"].astype(np.float64) for o in MUT_OUT}

    def loss(x):
        out = _advance_mu_t(g, x)
        return sum(float((out[o] * cot[o]).sum()) for o in MUT_OUT)

    for n, name in enumerate(MUT3 + MUT2):
        d = _mut_dir(n, 0, base[name].shape)
        eps = 1e-4 * float(np.abs(base[name]).max())  # the fixture's step
        xp, xm = dict(base), dict(base)
        xp[name] = base[name] + eps * d
        xm[name] = base[name] - eps * d
        fd = (loss(xp) - loss(xm)) / (2 * eps)
        ref = float(T[f"fd_{name}_0"])
        assert abs(fd - ref) <= 1e-6 * abs(ref) + 1e-9, (name, fd, ref)


AWZ = load_npz("advw_adj_ref64.npz")
AW3 = ("w", "rw_tend", "ww", "w_save", "u", "v", "t_2ave", "t_2", "t_1", "ph", "ph_1", "phb", "ph_tend", "c2a",
       "cqw", "alt", "a", "alpha", "gamma")
AW2 = ("muave", "muts", "mut", "ht")
AW_OUT = ("w", "ph", "t_2ave")
_AW_ST = {"t_2ave": "t_2save", "t_2": "t", "t_1": "t_save", "ph_1": "ph_save"}


def _aw_dir(n, r, shape):
    # the directions of make_golden_adjoint.aw_direction
    return np.random.default_rng(10000 + 100 * n + r).standard_normal(shape)


def _advance_w(g, x):
    st = {_AW_ST.get(k, k): np.array(v, np.float64) for k, v in x.items()}
    for k in ("msftx", "msfty", "fnm", "fnp", "rdnw", "rdn"):
        st[k] = AWZ[k].astype(np.float64)
    OD.advance_w(g, st, float(AWZ["dts"]), float(AWZ["epssm"]), float(AWZ["cf1"]), float(AWZ["cf2"]),
                 float(AWZ["cf3"]))
    return {o: st[_AW_ST.get(o, o)] for o in AW_OUT}


def test_advance_w_fixture_pinned_by_the_oracle():
    """advance_w: the oracle reproduces the reference's w, ph, t_2ave on the
    fixture, and its central differences equal the fixture's (of the
    reference's float64 forward)."""
    g = _grid()
    base = {k: AWZ[k].astype(np.float64) for k in AW3 + AW2}
    outs = _advance_w(g, base)
    for o in AW_OUT:
        ref = AWZ[f"{o}_new"]
        assert np.abs(outs[o] - ref).max() <= 1e-12 * np.abs(ref).max(), o
    cot = {"w": AWZ["cot_w"], "ph": AWZ["cot_ph"], "t_2ave": AWZ["cot_t2a"]}

    def loss(x):
        out = _advance_w(g, x)
        return sum(float((out[o] * cot[o].astype(np.float64)).sum()) for o in AW_OUT)

    for n, name in enumerate(AW3 + AW2):
        d = _aw_dir(n, 0, base[name].shape)
        eps = float(AWZ[f"fd_eps_{name}"])  # the fixture's step
        xp, xm = dict(base), dict(base)
        xp[name] = base[name] + eps * d
        xm[name] = base[name] - eps * d
        fd = (loss(xp) - loss(xm)) / (2 * eps)
        ref = float(AWZ[f"fd_{name}_0"])
        # the two float64 forwards round differently (~1e-13 relative), which
        # the finite difference magnifies by |L| / (eps |dL|)
        assert abs(fd - ref) <= 1e-5 * abs(ref) + 1e-9, (name, fd, ref)


FZ = load_npz("forces_adj_ref64.npz")
FORCES = {  # function: (differentiable inputs, outputs), as in make_golden_adjoint.FORCES
    "rhs_ph": (("u", "v", "ww", "ph", "phb", "w", "mut", "muu", "muv"), ("ph_tend",)),
    "hpg": (("ph", "alt", "p", "pb", "al", "php", "cqu", "cqv", "muu", "muv", "mu"), ("ru_tend", "rv_tend")),
    "pg_buoy_w": (("p", "cqw", "mu", "mub"), ("rw_tend", "cqw")),
    "coriolis": (("ru", "rv", "rw"), ("ru_tend", "rv_tend", "rw_tend")),
    "curvature": (("ru", "rv", "rw", "u", "v"), ("ru_tend", "rv_tend", "rw_tend")),
}


def _forces_dir(f, n, r, shape):
    # the directions of make_golden_adjoint.forces_direction
    return np.random.default_rng(20000 + 1000 * f + 10 * n + r).standard_normal(shape)


def _forces_oracle(g, name, x):
    x = {k: np.array(v, np.float64) for k, v in x.items()}
    z = lambda: np.zeros_like(x["u"])  # noqa: E731
    sc = {k: float(FZ[k]) for k in ("cf1", "cf2", "cf3", "cfn", "cfn1")}
    if name == "rhs_ph":
        pt = z()
        OD.rhs_ph(g, pt, x["u"], x["v"], x["ww"], x["ph"], x["phb"], x["w"], x["mut"], x["muu"], x["muv"], x["fnm"],
                  x["fnp"], x["rdnw"], sc["cfn"], sc["cfn1"], x["msfux"], x["msfvy"], x["msfty"])
        return {"ph_tend": pt}
    if name == "hpg":
        ru, rv = z(), z()
        OD.horizontal_pressure_gradient(g, ru, rv, x["ph"], x["alt"], x["p"], x["pb"], x["al"], x["php"], x["cqu"],
                                        x["cqv"], x["muu"], x["muv"], x["mu"], x["fnm"], x["fnp"], x["rdnw"],
                                        sc["cf1"], sc["cf2"], sc["cf3"], x["msfux"], x["msfuy"], x["msfvx"],
                                        x["msfvy"])
        return {"ru_tend": ru, "rv_tend": rv}
    if name == "pg_buoy_w":
        rw, cqw = z(), x["cqw"].copy()
        OD.pg_buoy_w(g, rw, x["p"], cqw, x["mu"], x["mub"], x["rdnw"], x["rdn"], x["msfty"])
        return {"rw_tend": rw, "cqw": cqw}
    ru, rv, rw = z(), z(), z()
    if name == "coriolis":
        OD.coriolis(g, x["ru"], x["rv"], x["rw"], ru, rv, rw, x["msftx"], x["msfty"], x["msfux"], x["msfuy"],
                    x["msfvx"], x["msfvy"], x["f"], x["e"], x["sina"], x["cosa"], x["fnm"], x["fnp"])
    else:
        OD.curvature(g, x["ru"], x["rv"], x["rw"], x["u"], x["v"], ru, rv, rw, x["msfux"], x["msfuy"], x["msfvx"],
                     x["msfvy"], x["msftx"], x["msfty"], x["fnm"], x["fnp"])
    return {"ru_tend": ru, "rv_tend": rv, "rw_tend": rw}


@pytest.mark.parametrize("name", list(FORCES))
def test_tendency_terms_fixture_pinned_by_the_oracle(name):
    """rhs_ph, horizontal_pressure_gradient, pg_buoy_w (with its in-place
    cqw), coriolis, curvature: the oracle's outputs have the reference's
    checksums on the fixture's inputs, and its central differences equal the
    reference's along the fixture's first direction of every input."""
    g = _grid()
    fi = list(FORCES).index(name)
    ins, outs = FORCES[name]
    base = {k: FZ[k] for k in FZ if np.asarray(FZ[k]).ndim > 0 and not k.startswith(name)}
    o0 = _forces_oracle(g, name, base)
    for o in outs:
        l2 = float(np.sqrt((o0[o] ** 2).sum()))
        assert abs(l2 - float(FZ[f"{name}_{o}_l2"])) <= 1e-12 * l2, (o, l2)
        assert abs(float(o0[o].sum()) - float(FZ[f"{name}_{o}_sum"])) <= 1e-12 * l2 * o0[o].size ** 0.5, o

    def loss(x):
        oo = _forces_oracle(g, name, x)
        return sum(float((oo[o] * np.asarray(FZ[f"cot_{o}"], np.float64)).sum()) for o in outs)

    for ni, inp in enumerate(ins):
        d = _forces_dir(fi, ni, 0, np.asarray(base[inp]).shape)
        eps = float(FZ[f"{name}_fd_eps_{inp}"])
        xp, xm = dict(base), dict(base)
        xp[inp] = np.asarray(base[inp], np.float64) + eps * d
        xm[inp] = np.asarray(base[inp], np.float64) - eps * d
        fd = (loss(xp) - loss(xm)) / (2 * eps)
        ref = float(FZ[f"{name}_fd_{inp}_0"])
        assert abs(fd - ref) <= 1e-5 * abs(ref) + 1e-9, (name, inp, fd, ref)


SZ = load_npz("subbdy_adj_ref64.npz")
SUBBDY = {  # case: (differentiable inputs, outputs), as in make_golden_adjoint.SUBBDY
    "sumflux1": (("u", "v", "ww", "u_save", "v_save", "ww1", "muu", "muv"), ("ru_m", "rv_m", "ww_m")),
    "sumflux2": (("u", "v", "ww", "u_save", "v_save", "ww1", "muu", "muv", "ru_m", "rv_m", "ww_m"),
                 ("ru_m", "rv_m", "ww_m")),
    "spec_t": (("t", "t_tend"), ("t",)),
    "spec_m": (("mu", "mu_tend"), ("mu",)),
    "spec_ph": (("ph_save", "ph", "ph_tend", "mu_tend", "muts"), ("ph",)),
}


def _subbdy_dir(f, n, r, shape):
    # the directions of make_golden_adjoint.subbdy_direction
    return np.random.default_rng(30000 + 1000 * f + 10 * n + r).standard_normal(shape)


def _subbdy_oracle(g, name, x):
    x = {k: np.array(v, np.float64) for k, v in x.items()}
    dts = float(SZ["dts"])
    if name.startswith("sumflux"):
        OD.sumflux(g, x, 1 if name == "sumflux1" else 2, 2)
        return {k: x[k] for k in ("ru_m", "rv_m", "ww_m")}
    if name == "spec_t":
        OB.spec_bdyupdate(g, x["t"], x["t_tend"], dts, "t")
        return {"t": x["t"]}
    if name == "spec_m":
        OB.spec_bdyupdate(g, x["mu"], x["mu_tend"], dts, "m")
        return {"mu": x["mu"]}
    OB.spec_bdyupdate_ph(g, x["ph_save"], x["ph"], x["ph_tend"], x["mu_tend"], x["muts"], dts)
    return {"ph": x["ph"]}


@pytest.mark.parametrize("name", list(SUBBDY))
def test_substep_boundary_and_flux_sums_pinned_by_the_oracle(name):
    """sumflux (first and last iteration), spec_bdyupdate ('t', 'm') and
    spec_bdyupdate_ph: the oracle's outputs have the reference's checksums on
    the fixture's inputs, and its central differences equal the reference's
    along the fixture's first direction of every input."""
    g = _grid()
    fi = list(SUBBDY).index(name)
    ins, outs = SUBBDY[name]
    base = {k: SZ[k] for k in SZ if np.asarray(SZ[k]).ndim > 0 and not k.startswith(name)}
    o0 = _subbdy_oracle(g, name, base)
    for o in outs:
        l2 = float(np.sqrt((o0[o] ** 2).sum()))
        assert abs(l2 - float(SZ[f"{name}_{o}_l2"])) <= 1e-12 * l2, (o, l2)
        assert abs(float(o0[o].sum()) - float(SZ[f"{name}_{o}_sum"])) <= 1e-12 * l2 * o0[o].size ** 0.5, o

    def loss(x):
        oo = _subbdy_oracle(g, name, x)
        return sum(float((oo[o] * np.asarray(SZ[f"cot_{o}"], np.float64)).sum()) for o in outs)

    for ni, inp in enumerate(ins):
        d = _subbdy_dir(fi, ni, 0, np.asarray(base[inp]).shape)
        eps = float(SZ[f"{name}_fd_eps_{inp}"])
        xp, xm = dict(base), dict(base)
        xp[inp] = np.asarray(base[inp], np.float64) + eps * d
        xm[inp] = np.asarray(base[inp], np.float64) - eps * d
        fd = (loss(xp) - loss(xm)) / (2 * eps)
        ref = float(SZ[f"{name}_fd_{inp}_0"])
        assert abs(fd - ref) <= 1e-5 * abs(ref) + 1e-9, (name, inp, fd, ref)


PZ = load_npz("prep_adj_ref64.npz")
PREP = {  # function: (differentiable inputs, outputs), as in make_golden_adjoint.PREP
    "calculate_full": (("mub", "mu"), ("mut",)),
    "calc_mu_uv": (("mu", "mub"), ("muu", "muv")),
    "couple_momentum": (("muu", "u", "muv", "v", "mut", "w"), ("ru", "rv", "rw")),
    "calc_ww_cp": (("u", "v", "muu", "muv", "ww"), ("ww",)),
    "calc_cq": (("moist",), ("cqu", "cqv", "cqw")),
    "calc_alt": (("al", "alb"), ("alt",)),
    "calc_php": (("ph", "phb"), ("php",)),
}


def _prep_dir(f, n, r, shape):
    # the directions of make_golden_adjoint.prep_direction
    return np.random.default_rng(40000 + 1000 * f + 10 * n + r).standard_normal(shape)


def _prep_oracle(g, name, x):
    x = {k: np.array(v, np.float64) for k, v in x.items()}
    z3 = lambda: np.zeros_like(x["u"])  # noqa: E731
    z2 = lambda: np.zeros_like(x["mu"])  # noqa: E731
    if name == "calculate_full":
        mut = z2()
        OD.calculate_full(g, mut, x["mub"], x["mu"])
        return {"mut": mut}
    if name == "calc_mu_uv":
        muu, muv = z2(), z2()
        OD.calc_mu_uv(g, x["mu"], x["mub"], muu, muv)
        return {"muu": muu, "muv": muv}
    if name == "couple_momentum":
        ru, rv, rw = z3(), z3(), z3()
        OD.couple_momentum(g, x["muu"], ru, x["u"], x["msfu"], x["muv"], rv, x["v"], x["msfvx_inv"], x["mut"], rw,
                           x["w"], x["msft"])
        return {"ru": ru, "rv": rv, "rw": rw}
    if name == "calc_ww_cp":
        ww = x["ww"].copy()
        OD.calc_ww_cp(g, x["u"], x["v"], x["muu"], x["muv"], np.ones(g.nz), ww, x["msftx"], x["msfuy"],
                      x["msfvx_inv"], x["dnw"])
        return {"ww": ww}
    if name == "calc_cq":
        cqu, cqv, cqw = z3(), z3(), z3()
        OD.calc_cq(g, x["moist"], cqu, cqv, cqw)
        return {"cqu": cqu, "cqv": cqv, "cqw": cqw}
    if name == "calc_alt":
        alt = z3()
        OD.calc_alt(g, alt, x["al"], x["alb"])
        return {"alt": alt}
    php = z3()
    OD.calc_php(g, php, x["ph"], x["phb"])
    return {"php": php}


@pytest.mark.parametrize("name", list(PREP))
def test_rk_step_prep_functions_pinned_by_the_oracle(name):
    """calculate_full, calc_mu_uv, couple_momentum, calc_ww_cp, calc_cq,
    calc_alt, calc_php: the oracle's outputs have the reference's checksums
    on the fixture's inputs, and its central differences equal the
    reference's along the fixture's first direction of every input."""
    g = _grid()
    fi = list(PREP).index(name)
    ins, outs = PREP[name]
    base = {k: PZ[k] for k in PZ if np.asarray(PZ[k]).ndim > 0 and not k.startswith(name)}
    o0 = _prep_oracle(g, name, base)
    for o in outs:
        l2 = float(np.sqrt((o0[o] ** 2).sum()))
        assert abs(l2 - float(PZ[f"{name}_{o}_l2"])) <= 1e-12 * l2, (o, l2)
        assert abs(float(o0[o].sum()) - float(PZ[f"{name}_{o}_sum"])) <= 1e-12 * l2 * o0[o].size ** 0.5, o

    def loss(x):
        oo = _prep_oracle(g, name, x)
        return sum(float((oo[o] * np.asarray(PZ[f"cot_{o}"], np.float64)).sum()) for o in outs)

    for ni, inp in enumerate(ins):
        d = _prep_dir(fi, ni, 0, np.asarray(base[inp]).shape)
        eps = float(PZ[f"{name}_fd_eps_{inp}"])
        xp, xm = dict(base), dict(base)
        xp[inp] = np.asarray(base[inp], np.float64) + eps * d
        xm[inp] = np.asarray(base[inp], np.float64) - eps * d
        fd = (loss(xp) - loss(xm)) / (2 * eps)
        ref = float(PZ[f"{name}_fd_{inp}_0"])
        assert abs(fd - ref) <= 1e-5 * abs(ref) + 1e-9, (name, inp, fd, ref)
