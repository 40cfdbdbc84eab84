"""Golden cotangents of step operators from the reference's own autograd.

Usage:  python tests/golden/make_golden_adjoint.py [--reference /path/to/PyWRF]

Runs unmodified reference functions in float64 on CPU with ``requires_grad``
on their differentiable inputs, back-propagates a seeded random cotangent of
the returned tendency with torch autograd, and writes next to this script:

* ``adv_scalar_adj_ref64.npz`` -- ``pywrf.wrf_dynamics.advect_scalar``
  (wrf_dynamics.py:1841-2028) w.r.t. the advected field and the three mass
  fluxes (fluxes of both signs, so both upwind branches are taken);
* ``relax_adj_ref64.npz`` -- ``pywrf.wrf_boundary.relax_bdytend``
  (wrf_boundary.py:52-147) w.r.t. the field, for the staggers 't', 'u', 'v'
  and 'h', with the solver's fcx / gcx (solver.py:440-441);
* ``adv_mom_adj_ref64.npz`` -- ``pywrf.wrf_dynamics.advect_u`` / ``advect_v``
  / ``advect_w`` (wrf_dynamics.py:1112-1823) w.r.t. the advected component
  and the three coupled velocities ru, rv, rom (both signs everywhere, so the
  upwind choices and the sign-selected boundary values of advect_u / advect_v
  take both branches); advect_w's backward() raises in the reference (its
  vertical part rewrites ``vel`` in place after a product saved it), so for
  w the fixture holds central finite differences of the reference's float64
  forward along 3 seeded directions per input (``mom_direction``);
* ``advuv_adj_ref64.npz`` -- ``pywrf.wrf_dynamics.advance_uv``
  (wrf_dynamics.py:3391-3525) followed by ``spec_bdyupdate`` of u and v
  (wrf_boundary.py:244-290), as the acoustic substep calls them
  (solver.py:1350-1377): the reference's autograd cannot differentiate
  advance_uv (``dpxy`` is rewritten for v after u's update saved a view of
  it), so the fixture holds central differences of the float64 forward of
  L = sum(u' cot_u + v' cot_v) along 3 seeded directions (``uv_direction``)
  in each of the 16 differentiable inputs;
* ``prho_adj_ref64.npz`` -- ``pywrf.wrf_dynamics.calc_p_rho``
  (wrf_dynamics.py:3269-3313) at step 0 and step 1 with autograd w.r.t.
  al, p, ph, alt, t_2, t_1, c2a, pm1, mu and mut;
* ``mut_adj_ref64.npz`` -- ``pywrf.wrf_dynamics.advance_mu_t``
  (wrf_dynamics.py:3528-3638) w.r.t. its 18 array inputs: the reference's
  autograd gradients (``grad_*``; its mu / muts / mudf / muave updates run
  under ``torch.no_grad()``, so those outputs pass their cotangents straight
  to the inputs of the same name and give mut, mu_tend and the divergence
  nothing) and, for the operator itself, central differences of the float64
  forward along 3 seeded directions per input (``mut_direction``);
* ``advw_adj_ref64.npz`` -- ``pywrf.wrf_dynamics.advance_w``
  (wrf_dynamics.py:3641-3796) w.r.t. its 23 array inputs: central
  differences of the float64 forward of L = sum(w' cot_w + ph' cot_ph +
  t_2ave' cot_t2a) along 3 seeded directions per input (``aw_direction``);
  the reference's autograd cannot run backward through its in-place
  tridiagonal sweeps; the upper levels lie in the Rayleigh damping layer;
* ``forces_adj_ref64.npz`` -- the tendency terms rhs_ph, horizontal_pressure_
  gradient, pg_buoy_w, coriolis and curvature (wrf_dynamics.py:2031-2620) on
  one shared input set: per function, checksums of its outputs and central
  differences of the float64 forward of L = sum(output cot) along 3 seeded
  directions (``forces_direction``) in each differentiable input;
* ``subbdy_adj_ref64.npz`` -- the rest of the acoustic substep: sumflux
  (wrf_dynamics.py:3799-3839) at its first and last iteration,
  spec_bdyupdate of a 3-D ('t') and a 2-D ('m') field and spec_bdyupdate_ph
  (wrf_boundary.py:244-355), in the form of ``forces_adj_ref64.npz``
  (``subbdy_direction``);
* ``prep_adj_ref64.npz`` -- rk_step_prep's functions calculate_full,
  calc_mu_uv, couple_momentum, calc_ww_cp, calc_cq, calc_alt, calc_php
  (wrf_dynamics.py:30-163), in the form of ``forces_adj_ref64.npz``
  (``prep_direction``);
* ``coefw_adj_ref64.npz`` -- ``pywrf.wrf_dynamics.calc_coef_w``
  (wrf_dynamics.py:3316-3388): the reference's autograd cannot differentiate
  it (the recurrence updates ``gamma`` in place between its reads, and
  backward() raises), so the fixture holds central finite differences of the
  reference's float64 forward instead: for L = sum(a ca + alpha cal + gamma cg)
  with seeded cotangents, the directional derivatives of L along 3 seeded
  directions in each of mut, cqw and c2a.

Grid 24x24x12 in the solver's 5-cell frame.  This script is the only producer
of the fixtures and is never run by the tests.
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


UV3 = ("u", "ru_tend", "v", "rv_tend", "p", "pb", "ph", "php", "alt", "al", "cqu", "cqv")
UV2 = ("mu", "muu", "muv", "mudf")


def uv_direction(n: int, r: int, shape) -> np.ndarray:
    """Direction r of input n (UV3 + UV2) of the advance_uv finite
    differences (regenerated by the tests, not stored)."""
    return np.random.default_rng(8000 + 100 * n + r).standard_normal(shape)


def advance_uv(dyn, bnd, g) -> None:
    """advance_uv + spec_bdyupdate(u), (v): central differences
    (advuv_adj_ref64.npz)."""
    import torch

    rng = np.random.default_rng(15)
    sh, s2 = (NZ, N, N), (N, N)
    kk = np.arange(NZ, dtype=np.float64)[:, None, None]
    d = {
        "u": 10.0 + 3.0 * rng.standard_normal(sh), "ru_tend": 0.05 * rng.standard_normal(sh),
        "v": 3.0 * rng.standard_normal(sh), "rv_tend": 0.05 * rng.standard_normal(sh),
        "p": 100.0 * rng.standard_normal(sh), "pb": 8.0e4 - 5.0e3 * kk + 100.0 * rng.standard_normal(sh),
        "ph": 50.0 * rng.standard_normal(sh), "php": 1.0e3 * (kk + 1.0) + 10.0 * rng.standard_normal(sh),
        "alt": 1.0 + 0.05 * rng.standard_normal(sh), "al": 0.01 * rng.standard_normal(sh),
        "cqu": 1.0 + 0.01 * rng.standard_normal(sh), "cqv": 1.0 + 0.01 * rng.standard_normal(sh),
        "mu": 100.0 * rng.standard_normal(s2), "muu": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "muv": 8.0e4 + 1.0e3 * rng.standard_normal(s2), "mudf": 10.0 * rng.standard_normal(s2),
        "msfux": 1.0 + 0.02 * rng.random(s2), "msfuy": 1.0 + 0.02 * rng.random(s2),
        "msfvx": 1.0 + 0.02 * rng.random(s2), "msfvy": 1.0 + 0.02 * rng.random(s2),
        "fnm": 0.45 + 0.1 * rng.random(NZ), "rdnw": -(10.0 + rng.random(NZ)),
        "cot_u": rng.standard_normal(sh), "cot_v": rng.standard_normal(sh),
    }
    d["fnp"] = 1.0 - d["fnm"]
    d = {k: v.astype(np.float32) for k, v in d.items()}
    d["msfvx_inv"] = (1.0 / d["msfvx"].astype(np.float64)).astype(np.float32)
    sc = {"dts": 11.25, "emdiv": 0.01, "cf1": 1.5, "cf2": -0.625, "cf3": 0.125}
    t = {k: torch.tensor(v, dtype=torch.float64) for k, v in d.items()}
    one1 = torch.ones(NZ, dtype=torch.float64)
    ids, ide, jds, jde = 5, N - 5, 5, N - 5
    idx = (ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)
    bidx = (ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)

    def run(x):
        u, v = dyn.advance_uv(x["u"], x["ru_tend"], x["v"], x["rv_tend"], x["p"], x["pb"], x["ph"], x["php"],
                              x["alt"], x["al"], x["mu"], x["muu"], x["cqu"], x["muv"], x["cqv"], x["mudf"],
                              one1, one1 * 0, one1, one1 * 0, one1, one1 * 0, one1, one1 * 0,
                              x["msfux"], x["msfuy"], x["msfvx"], x["msfvx_inv"], x["msfvy"], 1.0 / g.dx,
                              1.0 / g.dy, sc["dts"], sc["cf1"], sc["cf2"], sc["cf3"], x["fnm"], x["fnp"],
                              sc["emdiv"], x["rdnw"], 1, True, False, *idx)
        u = bnd.spec_bdyupdate(u, x["ru_tend"], sc["dts"], "u", 1, *bidx)
        v = bnd.spec_bdyupdate(v, x["rv_tend"], sc["dts"], "v", 1, *bidx)
        return u, v

    save = dict(d)
    save.update({k: np.array(v) for k, v in sc.items()})
    save["dx"], save["dy"] = np.array(g.dx), np.array(g.dy)
    with torch.no_grad():
        u, v = run(t)
        save["u_new"], save["v_new"] = u.numpy(), v.numpy()
        cu, cv = t["cot_u"], t["cot_v"]
        for n_, name in enumerate(UV3 + UV2):
            for r in range(3):
                dirn = torch.tensor(uv_direction(n_, r, d[name].shape))
                eps = 1e-6 * float(t[name].abs().max())
                xp, xm = dict(t), dict(t)
                xp[name] = t[name] + eps * dirn
                xm[name] = t[name] - eps * dirn
                up, vp = run(xp)
                um, vm = run(xm)
                save[f"fd_{name}_{r}"] = np.array(float(((up - um) * cu).sum() + ((vp - vm) * cv).sum()) / (2 * eps))
    np.savez_compressed(os.path.join(HERE, "advuv_adj_ref64.npz"), **save)
    print("wrote advuv_adj_ref64.npz")


PRHO_IN = ("al", "p", "ph", "alt", "t_2", "t_1", "c2a", "pm1", "mu", "mut")


def calc_p_rho(dyn, g) -> None:
    """calc_p_rho at step 0 and 1 with autograd (prho_adj_ref64.npz)."""
    import torch

    rng = np.random.default_rng(16)
    sh, s2 = (NZ, N, N), (N, N)
    kk = np.arange(NZ, dtype=np.float64)[:, None, None]
    d = {
        "al": 0.01 * rng.standard_normal(sh), "p": 100.0 * rng.standard_normal(sh),
        "ph": 2.0e3 * kk + 50.0 * rng.standard_normal(sh), "alt": 1.0 + 0.05 * rng.standard_normal(sh),
        "t_2": 100.0 * rng.standard_normal(sh), "t_1": 5.0 * rng.standard_normal(sh),
        "c2a": 1.6e5 + 1.0e4 * rng.standard_normal(sh), "pm1": 100.0 * rng.standard_normal(sh),
        "mu": 100.0 * rng.standard_normal(s2), "mut": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "rdnw": -(10.0 + rng.random(NZ)),
        "cot_al": rng.standard_normal(sh), "cot_p": rng.standard_normal(sh), "cot_pm1": rng.standard_normal(sh),
    }
    d = {k: v.astype(np.float32) for k, v in d.items()}
    save = dict(d)
    save["smdiv"] = np.array(0.1)
    save["dx"], save["dy"] = np.array(g.dx), np.array(g.dy)
    one1 = torch.ones(NZ, dtype=torch.float64)
    ids, ide, jds, jde = 5, N - 5, 5, N - 5
    for step in (0, 1):
        t = {k: torch.tensor(v, dtype=torch.float64) for k, v in d.items()}
        for k in PRHO_IN:
            t[k].requires_grad_(True)
        al, p, pm1 = dyn.calc_p_rho(t["al"].clone(), t["p"].clone(), t["ph"], t["alt"], t["t_2"], t["t_1"], t["c2a"],
                                    t["pm1"].clone(), t["mu"], t["mut"], one1, one1 * 0, one1, one1 * 0, one1,
                                    one1 * 0, one1, one1 * 0, one1, 300.0, t["rdnw"], one1, 0.1, True, step,
                                    ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)
        ((al * t["cot_al"]).sum() + (p * t["cot_p"]).sum() + (pm1 * t["cot_pm1"]).sum()).backward()
        for nm, v in (("al", al), ("p", p), ("pm1", pm1)):
            save[f"s{step}_{nm}_new"] = v.detach().numpy()
        for k in PRHO_IN:
            gk = t[k].grad
            save[f"s{step}_grad_{k}"] = np.zeros(d[k].shape) if gk is None else gk.numpy()
    np.savez_compressed(os.path.join(HERE, "prho_adj_ref64.npz"), **save)
    print("wrote prho_adj_ref64.npz")


MUT3 = ("ww", "ww_1", "u", "u_1", "v", "v_1", "t", "t_1", "t_ave", "ft")
MUT2 = ("mu", "mut", "muave", "muts", "muu", "muv", "mudf", "mu_tend")
MUT_OUT = ("ww", "t", "t_ave", "muave", "muts", "mudf", "mu")


def mut_direction(n: int, r: int, shape) -> np.ndarray:
    """Direction r of input n (MUT3 + MUT2) of the advance_mu_t finite
    differences (regenerated by the tests, not stored)."""
    return np.random.default_rng(9000 + 100 * n + r).standard_normal(shape)


def advance_mu_t(dyn, g) -> None:
    """advance_mu_t: autograd and central differences (mut_adj_ref64.npz)."""
    import torch

    rng = np.random.default_rng(17)
    sh, s2 = (NZ, N, N), (N, N)
    d = {
        "ww": 5.0 * rng.standard_normal(sh), "ww_1": 5.0 * rng.standard_normal(sh),
        "u": 10.0 + 3.0 * rng.standard_normal(sh), "u_1": 10.0 + 3.0 * rng.standard_normal(sh),
        "v": 3.0 * rng.standard_normal(sh), "v_1": 3.0 * rng.standard_normal(sh),
        "t": 100.0 * rng.standard_normal(sh), "t_1": 2.0 + 5.0 * rng.standard_normal(sh),
        "t_ave": 100.0 * rng.standard_normal(sh), "ft": 0.1 * rng.standard_normal(sh),
        "mu": 100.0 * rng.standard_normal(s2), "mut": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "muave": 100.0 * rng.standard_normal(s2), "muts": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "muu": 8.0e4 + 1.0e3 * rng.standard_normal(s2), "muv": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "mudf": 10.0 * rng.standard_normal(s2), "mu_tend": 0.1 * rng.standard_normal(s2),
        "msfuy": 1.0 + 0.02 * rng.random(s2), "msfvx_inv": 1.0 + 0.02 * rng.random(s2),
        "msftx": 1.0 + 0.02 * rng.random(s2), "msfty": 1.0 + 0.02 * rng.random(s2),
        "fnm": 0.45 + 0.1 * rng.random(NZ), "rdnw": -(10.0 + rng.random(NZ)),
    }
    d["fnp"] = 1.0 - d["fnm"]
    d["dnw"] = 1.0 / d["rdnw"]
    for o_ in MUT_OUT:
        d[f"cot_{o_}"] = rng.standard_normal(sh if o_ in MUT3 else s2)
    d = {k: v.astype(np.float32) for k, v in d.items()}
    sc = {"dts": 11.25, "epssm": 0.1}
    save = dict(d)
    save.update({k: np.array(v) for k, v in sc.items()})
    save["dx"], save["dy"] = np.array(g.dx), np.array(g.dy)
    one1 = torch.ones(NZ, dtype=torch.float64)
    ids, ide, jds, jde = 5, N - 5, 5, N - 5

    def run(x):
        o = dyn.advance_mu_t(x["ww"], x["ww_1"], x["u"], x["u_1"], x["v"], x["v_1"], x["mu"], x["mut"], x["muave"],
                             x["muts"], x["muu"], x["muv"], x["mudf"], one1, one1 * 0, one1, one1 * 0, one1,
                             one1 * 0, one1, one1 * 0, None, None, None, x["t"], x["t_1"], x["t_ave"], x["ft"],
                             x["mu_tend"], 1.0 / g.dx, 1.0 / g.dy, sc["dts"], sc["epssm"], x["dnw"], x["fnm"],
                             x["fnp"], x["rdnw"], x["msfuy"], x["msfuy"], x["msfvx_inv"], x["msfvx_inv"],
                             x["msfvx_inv"], x["msftx"], x["msfty"], 1,
                             ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)
        ww, _w1, t, t_ave, _a, _b, _c, muave, muts, mudf, mu = o
        return {"ww": ww, "t": t, "t_ave": t_ave, "muave": muave, "muts": muts, "mudf": mudf, "mu": mu}

    def loss(x):
        outs = run(x)
        return sum((outs[o_] * x[f"cot_{o_}"]).sum() for o_ in MUT_OUT)

    t = {k: torch.tensor(v, dtype=torch.float64) for k, v in d.items()}
    for k in MUT3 + MUT2:
        t[k].requires_grad_(True)
    outs = run(t)
    for o_ in MUT_OUT:
        save[f"{o_}_new"] = outs[o_].detach().numpy()
    sum((outs[o_] * t[f"cot_{o_}"]).sum() for o_ in MUT_OUT).backward()
    for k in MUT3 + MUT2:
        gk = t[k].grad
        save[f"grad_{k}"] = np.zeros(d[k].shape) if gk is None else gk.numpy()
    base = {k: v.detach().clone() for k, v in t.items()}
    with torch.no_grad():
        for n_, name in enumerate(MUT3 + MUT2):
            for r in range(3):
                dirn = torch.tensor(mut_direction(n_, r, d[name].shape))
                # at most cubic in the inputs: a step of 1e-4 keeps the
                # truncation error near 1e-8 and the cancellation small
                eps = 1e-4 * float(base[name].abs().max())
                xp, xm = dict(base), dict(base)
                xp[name] = base[name] + eps * dirn
                xm[name] = base[name] - eps * dirn
                save[f"fd_{name}_{r}"] = np.array(float(loss(xp) - loss(xm)) / (2 * eps))
    np.savez_compressed(os.path.join(HERE, "mut_adj_ref64.npz"), **save)
    print("wrote mut_adj_ref64.npz")


AW3 = ("w", "rw_tend", "ww", "w_save", "u", "v", "t_2ave", "t_2", "t_1", "ph", "ph_1", "phb", "ph_tend", "c2a",
       "cqw", "alt", "a", "alpha", "gamma")
AW2 = ("muave", "muts", "mut", "ht")
AW_OUT = ("w", "ph", "t_2ave")


def aw_direction(n: int, r: int, shape) -> np.ndarray:
    """Direction r of input n (AW3 + AW2) of the advance_w finite
    differences (regenerated by the tests, not stored)."""
    return np.random.default_rng(10000 + 100 * n + r).standard_normal(shape)


def advance_w(dyn, g) -> None:
    """advance_w: central differences (advw_adj_ref64.npz)."""
    import torch

    rng = np.random.default_rng(18)
    sh, s2 = (NZ, N, N), (N, N)
    kk = np.arange(NZ, dtype=np.float64)[:, None, None]
    d = {
        "w": rng.standard_normal(sh), "rw_tend": 0.1 * rng.standard_normal(sh), "ww": 5.0 * rng.standard_normal(sh),
        "w_save": rng.standard_normal(sh), "u": 10.0 + 3.0 * rng.standard_normal(sh),
        "v": 3.0 * rng.standard_normal(sh), "t_2ave": 100.0 * rng.standard_normal(sh),
        "t_2": 100.0 * rng.standard_normal(sh), "t_1": 2.0 + 5.0 * rng.standard_normal(sh),
        "ph": 50.0 * rng.standard_normal(sh), "ph_1": 50.0 * rng.standard_normal(sh),
        "phb": 9.81 * 1800.0 * kk + 100.0 * rng.standard_normal(sh), "ph_tend": 10.0 * rng.standard_normal(sh),
        "c2a": 1.6e5 + 1.0e4 * rng.standard_normal(sh), "cqw": 1.0 + 0.01 * rng.standard_normal(sh),
        "alt": 1.0 + 0.05 * rng.standard_normal(sh), "a": -0.2 * rng.random(sh), "alpha": 0.6 + 0.3 * rng.random(sh),
        "gamma": -0.3 * rng.random(sh),
        "muave": 100.0 * rng.standard_normal(s2), "muts": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "mut": 8.0e4 + 1.0e3 * rng.standard_normal(s2), "ht": 800.0 * rng.random(s2),
        "msftx": 1.0 + 0.02 * rng.random(s2), "msfty": 1.0 + 0.02 * rng.random(s2),
        "fnm": 0.45 + 0.1 * rng.random(NZ), "rdnw": -(10.0 + rng.random(NZ)), "rdn": -(10.0 + rng.random(NZ)),
        "cot_w": rng.standard_normal(sh), "cot_ph": rng.standard_normal(sh), "cot_t2a": rng.standard_normal(sh),
    }
    d["fnp"] = 1.0 - d["fnm"]
    d = {k: v.astype(np.float32) for k, v in d.items()}
    sc = {"dts": 11.25, "epssm": 0.1, "cf1": 1.5, "cf2": -0.625, "cf3": 0.125}
    save = dict(d)
    save.update({k: np.array(v) for k, v in sc.items()})
    save["dx"], save["dy"] = np.array(g.dx), np.array(g.dy)
    one1 = torch.ones(NZ, dtype=torch.float64)
    ids, ide, jds, jde = 5, N - 5, 5, N - 5

    def run(x):
        t2a, w, ph = dyn.advance_w(x["w"], x["rw_tend"], x["ww"], x["w_save"], x["u"], x["v"], x["muave"] * 0,
                                   x["mut"], x["muave"], x["muts"], one1, one1 * 0, one1, one1 * 0, one1, one1 * 0,
                                   one1, one1 * 0, x["t_2ave"], x["t_2"], x["t_1"], x["ph"], x["ph_1"], x["phb"],
                                   x["ph_tend"], x["ht"], x["c2a"], x["cqw"], x["alt"], x["alt"], x["a"], x["alpha"],
                                   x["gamma"], 1.0 / g.dx, 1.0 / g.dy, sc["dts"], 300.0, sc["epssm"], 1.0 / x["rdnw"],
                                   x["fnm"], x["fnp"], x["rdnw"], x["rdn"], sc["cf1"], sc["cf2"], sc["cf3"],
                                   x["msftx"], x["msfty"], False,
                                   ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)
        return {"w": w, "ph": ph, "t_2ave": t2a}

    def loss(x):
        o = run(x)
        return float((o["w"] * x["cot_w"]).sum() + (o["ph"] * x["cot_ph"]).sum() + (o["t_2ave"] * x["cot_t2a"]).sum())

    base = {k: torch.tensor(v, dtype=torch.float64) for k, v in d.items()}
    with torch.no_grad():
        outs = run(base)
        for o_ in AW_OUT:
            save[f"{o_}_new"] = outs[o_].numpy()
        for n_, name in enumerate(AW3 + AW2):
            # L is linear in all but these inputs: there a large step is exact
            # and keeps the cancellation in L (~1e8) out of the difference
            rel = 1e-4 if name in ("t_1", "ph_1", "phb", "muts", "mut", "a", "alpha", "gamma") else 1e-1
            eps = rel * float(base[name].abs().max())
            save[f"fd_eps_{name}"] = np.array(eps)
            for r in range(3):
                dirn = torch.tensor(aw_direction(n_, r, d[name].shape))
                xp, xm = dict(base), dict(base)
                xp[name] = base[name] + eps * dirn
                xm[name] = base[name] - eps * dirn
                save[f"fd_{name}_{r}"] = np.array((loss(xp) - loss(xm)) / (2 * eps))
    np.savez_compressed(os.path.join(HERE, "advw_adj_ref64.npz"), **save)
    print("wrote advw_adj_ref64.npz")


FORCES = {  # function: (differentiable inputs, outputs)
    "rhs_ph": (("u", "v", "ww", "ph", "phb", "w", "mut", "muu", "muv"), ("ph_tend",)),
    "hpg": (("ph", "alt", "p", "pb", "al", "php", "cqu", "cqv", "muu", "muv", "mu"), ("ru_tend", "rv_tend")),
    "pg_buoy_w": (("p", "cqw", "mu", "mub"), ("rw_tend", "cqw")),
    "coriolis": (("ru", "rv", "rw"), ("ru_tend", "rv_tend", "rw_tend")),
    "curvature": (("ru", "rv", "rw", "u", "v"), ("ru_tend", "rv_tend", "rw_tend")),
}


def forces_direction(f: int, n: int, r: int, shape) -> np.ndarray:
    """Direction r of input n of function f (in FORCES order) of the
    tendency-term finite differences (regenerated by the tests)."""
    return np.random.default_rng(20000 + 1000 * f + 10 * n + r).standard_normal(shape)


def forces_inputs(g) -> dict:
    rng = np.random.default_rng(19)
    sh, s2 = (NZ, N, N), (N, N)
    kk = np.arange(NZ, dtype=np.float64)[:, None, None]
    d = {
        "u": 10.0 + 3.0 * rng.standard_normal(sh), "v": 3.0 * rng.standard_normal(sh), "w": rng.standard_normal(sh),
        "ww": 5.0 * rng.standard_normal(sh), "ph": 50.0 * rng.standard_normal(sh),
        "phb": 9.81 * 1800.0 * kk + 100.0 * rng.standard_normal(sh), "alt": 1.0 + 0.05 * rng.standard_normal(sh),
        "p": 100.0 * rng.standard_normal(sh), "pb": 8.0e4 - 5.0e3 * kk + 100.0 * rng.standard_normal(sh),
        "al": 0.01 * rng.standard_normal(sh), "php": 1.0e3 * (kk + 1.0) + 10.0 * rng.standard_normal(sh),
        "cqu": 1.0 + 0.01 * rng.standard_normal(sh), "cqv": 1.0 + 0.01 * rng.standard_normal(sh),
        "cqw": 0.01 * rng.standard_normal(sh), "ru": 8.0e5 + 2.0e5 * rng.standard_normal(sh),
        "rv": 2.0e5 * rng.standard_normal(sh), "rw": 8.0e4 * rng.standard_normal(sh),
        "mut": 8.0e4 + 1.0e3 * rng.standard_normal(s2), "muu": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "muv": 8.0e4 + 1.0e3 * rng.standard_normal(s2), "mu": 100.0 * rng.standard_normal(s2),
        "mub": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "msfux": 1.0 + 0.02 * rng.random(s2), "msfuy": 1.0 + 0.02 * rng.random(s2),
        "msfvx": 1.0 + 0.02 * rng.random(s2), "msfvy": 1.0 + 0.02 * rng.random(s2),
        "msftx": 1.0 + 0.02 * rng.random(s2), "msfty": 1.0 + 0.02 * rng.random(s2),
        "f": 1.0e-4 + 1.0e-5 * rng.standard_normal(s2), "e": 5.0e-5 + 1.0e-5 * rng.standard_normal(s2),
        "sina": 0.01 * rng.standard_normal(s2), "cosa": 1.0 - 0.001 * rng.random(s2),
        "clat": 30.0 + 5.0 * rng.standard_normal(s2),
        "fnm": 0.45 + 0.1 * rng.random(NZ), "rdnw": -(10.0 + rng.random(NZ)), "rdn": -(10.0 + rng.random(NZ)),
        "cot_ph_tend": rng.standard_normal(sh), "cot_ru_tend": rng.standard_normal(sh),
        "cot_rv_tend": rng.standard_normal(sh), "cot_rw_tend": rng.standard_normal(sh),
        "cot_cqw": rng.standard_normal(sh),
    }
    d["fnp"] = 1.0 - d["fnm"]
    d["msfvx_inv"] = 1.0 / d["msfvx"]
    return {k: v.astype(np.float32) for k, v in d.items()}


FORCES_SC = {"cf1": 1.5, "cf2": -0.625, "cf3": 0.125, "cfn": 1.5, "cfn1": -0.5}


def forces_call(dyn, g, name, x):
    """Run one tendency term of the reference with the solver's argument list
    (solver.py rhs_ph .. curvature calls); returns its outputs by name."""
    import torch

    one1 = torch.ones(NZ, dtype=torch.float64)
    z3 = torch.zeros((NZ, N, N), dtype=torch.float64)
    ids, ide, jds, jde = 5, N - 5, 5, N - 5
    idx = (ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)
    sc = FORCES_SC
    if name == "rhs_ph":
        pt = dyn.rhs_ph(z3.clone(), x["u"], x["v"], x["ww"], x["ph"], x["ph"], x["phb"], x["w"], x["mut"], x["muu"],
                        x["muv"], one1, one1 * 0, x["fnm"], x["fnp"], x["rdnw"], sc["cfn"], sc["cfn1"], 1.0 / g.dx,
                        1.0 / g.dy, x["msfux"], x["msfuy"], x["msfvx"], x["msfvx_inv"], x["msfvy"], x["msftx"],
                        x["msfty"], True, *idx)
        return {"ph_tend": pt}
    if name == "hpg":
        ru, rv = dyn.horizontal_pressure_gradient(z3.clone(), z3.clone(), x["ph"], x["alt"], x["p"], x["pb"], x["al"],
                                                  x["php"], x["cqu"], x["cqv"], x["muu"], x["muv"], x["mu"], one1,
                                                  one1 * 0, x["fnm"], x["fnp"], x["rdnw"], sc["cf1"], sc["cf2"],
                                                  sc["cf3"], sc["cfn"], sc["cfn1"], 1.0 / g.dx, 1.0 / g.dy, x["msfux"],
                                                  x["msfuy"], x["msfvx"], x["msfvy"], x["msftx"], x["msfty"], True,
                                                  False, *idx)
        return {"ru_tend": ru, "rv_tend": rv}
    if name == "pg_buoy_w":
        rw, cqw = dyn.pg_buoy_w(z3.clone(), x["p"], x["cqw"].clone(), x["mu"], x["mub"], one1, one1 * 0, x["rdnw"],
                                x["rdn"], 9.81, x["msftx"], x["msfty"], *idx)
        return {"rw_tend": rw, "cqw": cqw}
    if name == "coriolis":
        ru, rv, rw = dyn.coriolis(x["ru"], x["rv"], x["rw"], z3.clone(), z3.clone(), z3.clone(), x["msftx"], x["msfty"],
                                  x["msfux"], x["msfuy"], x["msfvx"], x["msfvy"], x["f"], x["e"], x["sina"], x["cosa"],
                                  x["fnm"], x["fnp"], *idx)
        return {"ru_tend": ru, "rv_tend": rv, "rw_tend": rw}
    ru, rv, rw = dyn.curvature(x["ru"], x["rv"], x["rw"], x["u"], x["v"], x["w"], z3.clone(), z3.clone(), z3.clone(),
                               x["msfux"], x["msfuy"], x["msfvx"], x["msfvy"], x["msftx"], x["msfty"], x["clat"],
                               x["fnm"], x["fnp"], 1.0 / g.dx, 1.0 / g.dy, *idx)
    return {"ru_tend": ru, "rv_tend": rv, "rw_tend": rw}


def forces(dyn, g) -> None:
    """The five tendency terms: checksums and central differences
    (forces_adj_ref64.npz)."""
    import torch

    d = forces_inputs(g)
    save = dict(d)
    save.update({k: np.array(v) for k, v in FORCES_SC.items()})
    save["dx"], save["dy"] = np.array(g.dx), np.array(g.dy)
    base = {k: torch.tensor(v, dtype=torch.float64) for k, v in d.items()}
    with torch.no_grad():
        for fi, (name, (ins, outs)) in enumerate(FORCES.items()):
            o0 = forces_call(dyn, g, name, base)
            for o_ in outs:
                a = o0[o_].numpy()
                save[f"{name}_{o_}_sum"] = np.array(a.sum())
                save[f"{name}_{o_}_l2"] = np.array(np.sqrt((a * a).sum()))

            def loss(x):
                oo = forces_call(dyn, g, name, x)
                return float(sum((oo[o_] * x[f"cot_{o_}"]).sum() for o_ in outs))

            for ni, inp in enumerate(ins):
                eps = 1e-4 * float(base[inp].abs().max())
                for r in range(3):
                    dirn = torch.tensor(forces_direction(fi, ni, r, d[inp].shape))
                    xp, xm = dict(base), dict(base)
                    xp[inp] = base[inp] + eps * dirn
                    xm[inp] = base[inp] - eps * dirn
                    save[f"{name}_fd_{inp}_{r}"] = np.array((loss(xp) - loss(xm)) / (2 * eps))
                save[f"{name}_fd_eps_{inp}"] = np.array(eps)
    np.savez_compressed(os.path.join(HERE, "forces_adj_ref64.npz"), **save)
    print("wrote forces_adj_ref64.npz")


SUBBDY = {  # case: (differentiable inputs, outputs)
    "sumflux1": (("u", "v", "ww", "u_save", "v_save", "ww1", "muu", "muv"), ("ru_m", "rv_m", "ww_m")),
    "sumflux2": (("u", "v", "ww", "u_save", "v_save", "ww1", "muu", "muv", "ru_m", "rv_m", "ww_m"),
                 ("ru_m", "rv_m", "ww_m")),
    "spec_t": (("t", "t_tend"), ("t",)),
    "spec_m": (("mu", "mu_tend"), ("mu",)),
    "spec_ph": (("ph_save", "ph", "ph_tend", "mu_tend", "muts"), ("ph",)),
}


def subbdy_direction(f: int, n: int, r: int, shape) -> np.ndarray:
    """Direction r of input n of case f (in SUBBDY order), regenerated by the tests."""
    return np.random.default_rng(30000 + 1000 * f + 10 * n + r).standard_normal(shape)


def subbdy_inputs() -> dict:
    rng = np.random.default_rng(21)
    sh, s2 = (NZ, N, N), (N, N)
    d = {
        "u": 10.0 + 3.0 * rng.standard_normal(sh), "v": 3.0 * rng.standard_normal(sh),
        "ww": 5.0 * rng.standard_normal(sh), "u_save": 10.0 + 3.0 * rng.standard_normal(sh),
        "v_save": 3.0 * rng.standard_normal(sh), "ww1": 5.0 * rng.standard_normal(sh),
        "ru_m": 8.0e5 * rng.standard_normal(sh), "rv_m": 2.0e5 * rng.standard_normal(sh),
        "ww_m": 5.0 * rng.standard_normal(sh), "t": 100.0 * rng.standard_normal(sh),
        "t_tend": rng.standard_normal(sh), "ph": 50.0 * rng.standard_normal(sh),
        "ph_save": 50.0 * rng.standard_normal(sh), "ph_tend": 10.0 * rng.standard_normal(sh),
        "muu": 8.0e4 + 1.0e3 * rng.standard_normal(s2), "muv": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "mu": 100.0 * rng.standard_normal(s2), "mu_tend": rng.standard_normal(s2),
        "muts": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "msfux": 1.0 + 0.02 * rng.random(s2), "msfuy": 1.0 + 0.02 * rng.random(s2),
        "msfvx": 1.0 + 0.02 * rng.random(s2), "msfvy": 1.0 + 0.02 * rng.random(s2),
        "cot_ru_m": rng.standard_normal(sh), "cot_rv_m": rng.standard_normal(sh), "cot_ww_m": rng.standard_normal(sh),
        "cot_t": rng.standard_normal(sh), "cot_mu": rng.standard_normal(s2), "cot_ph": rng.standard_normal(sh),
    }
    d["msfvx_inv"] = 1.0 / d["msfvx"]
    return {k: v.astype(np.float32) for k, v in d.items()}


SUBBDY_DTS = 11.25


def subbdy_call(dyn, bnd, g, name, x):
    """Run one case with the solver's argument lists (solver.py:1394-1445)."""
    import torch

    one1 = torch.ones(NZ, dtype=torch.float64)
    ids, ide, jds, jde = 5, N - 5, 5, N - 5
    idx = (ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)
    bidx = (ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)
    bidx2 = (ids, ide, jds, jde, 0, 0, 0, N, 0, N, 0, 0, 0, N, 0, N, 0, 0, ids, ide, jds, jde, 0, 0)
    if name.startswith("sumflux"):
        it = 1 if name == "sumflux1" else 2
        ru_m, rv_m, ww_m = dyn.sumflux(x["u"], x["v"], x["ww"], x["u_save"], x["v_save"], x["ww1"], x["muu"], x["muv"],
                                       one1, one1 * 0, one1, one1 * 0, one1, one1 * 0, one1, one1 * 0,
                                       x["ru_m"].clone(), x["rv_m"].clone(), x["ww_m"].clone(), 0.1, x["msfux"],
                                       x["msfuy"], x["msfvx"], x["msfvx_inv"], x["msfvy"], it, 2, *idx)
        return {"ru_m": ru_m, "rv_m": rv_m, "ww_m": ww_m}
    if name == "spec_t":
        return {"t": bnd.spec_bdyupdate(x["t"].clone(), x["t_tend"], SUBBDY_DTS, "t", 1, *bidx)}
    if name == "spec_m":
        return {"mu": bnd.spec_bdyupdate(x["mu"].clone(), x["mu_tend"], SUBBDY_DTS, "m", 1, *bidx2)}
    return {"ph": bnd.spec_bdyupdate_ph(x["ph_save"], x["ph"].clone(), x["ph_tend"], x["mu_tend"], x["muts"], one1,
                                        one1 * 0, SUBBDY_DTS, "h", 1, *bidx)}


def subbdy(dyn, bnd, g) -> None:
    """The rest of the acoustic substep: checksums and central differences
    (subbdy_adj_ref64.npz)."""
    import torch

    d = subbdy_inputs()
    save = dict(d)
    save["dts"] = np.array(SUBBDY_DTS)
    base = {k: torch.tensor(v, dtype=torch.float64) for k, v in d.items()}
    with torch.no_grad():
        for fi, (name, (ins, outs)) in enumerate(SUBBDY.items()):
            o0 = subbdy_call(dyn, bnd, g, name, base)
            for o_ in outs:
                a = o0[o_].numpy()
                save[f"{name}_{o_}_sum"] = np.array(a.sum())
                save[f"{name}_{o_}_l2"] = np.array(np.sqrt((a * a).sum()))

            def loss(x):
                oo = subbdy_call(dyn, bnd, g, name, x)
                return float(sum((oo[o_] * x[f"cot_{o_}"]).sum() for o_ in outs))

            for ni, inp in enumerate(ins):
                eps = 1e-4 * float(base[inp].abs().max())
                save[f"{name}_fd_eps_{inp}"] = np.array(eps)
                for r in range(3):
                    dirn = torch.tensor(subbdy_direction(fi, ni, r, d[inp].shape))
                    xp, xm = dict(base), dict(base)
                    xp[inp] = base[inp] + eps * dirn
                    xm[inp] = base[inp] - eps * dirn
                    save[f"{name}_fd_{inp}_{r}"] = np.array((loss(xp) - loss(xm)) / (2 * eps))
    np.savez_compressed(os.path.join(HERE, "subbdy_adj_ref64.npz"), **save)
    print("wrote subbdy_adj_ref64.npz")


PREP = {  # function: (differentiable inputs, outputs)
    "calculate_full": (("mub", "mu"), ("mut",)),
    "calc_mu_uv": (("mu", "mub"), ("muu", "muv")),
    "couple_momentum": (("muu", "u", "muv", "v", "mut", "w"), ("ru", "rv", "rw")),
    "calc_ww_cp": (("u", "v", "muu", "muv", "ww"), ("ww",)),
    "calc_cq": (("moist",), ("cqu", "cqv", "cqw")),
    "calc_alt": (("al", "alb"), ("alt",)),
    "calc_php": (("ph", "phb"), ("php",)),
}


def prep_direction(f: int, n: int, r: int, shape) -> np.ndarray:
    """Direction r of input n of function f (in PREP order), regenerated by the tests."""
    return np.random.default_rng(40000 + 1000 * f + 10 * n + r).standard_normal(shape)


def prep_inputs() -> dict:
    rng = np.random.default_rng(22)
    sh, s2 = (NZ, N, N), (N, N)
    kk = np.arange(NZ, dtype=np.float64)[:, None, None]
    moist = np.zeros((7,) + sh)
    moist[1] = 0.01 * rng.random(sh)
    moist[2:] = 1.0e-4 * rng.random((5,) + sh)
    d = {
        "u": 10.0 + 3.0 * rng.standard_normal(sh), "v": 3.0 * rng.standard_normal(sh), "w": rng.standard_normal(sh),
        "ww": 5.0 * rng.standard_normal(sh), "ph": 50.0 * rng.standard_normal(sh),
        "phb": 9.81 * 1800.0 * kk + 100.0 * rng.standard_normal(sh), "al": 0.01 * rng.standard_normal(sh),
        "alb": 1.0 + 0.2 * rng.random(sh), "moist": moist,
        "mu": 100.0 * rng.standard_normal(s2), "mub": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "mut": 8.0e4 + 1.0e3 * rng.standard_normal(s2), "muu": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "muv": 8.0e4 + 1.0e3 * rng.standard_normal(s2),
        "msfu": 1.0 + 0.02 * rng.random(s2), "msfv": 1.0 + 0.02 * rng.random(s2), "msft": 1.0 + 0.02 * rng.random(s2),
        "msftx": 1.0 + 0.02 * rng.random(s2), "msfty": 1.0 + 0.02 * rng.random(s2),
        "msfux": 1.0 + 0.02 * rng.random(s2), "msfuy": 1.0 + 0.02 * rng.random(s2),
        "msfvx": 1.0 + 0.02 * rng.random(s2), "msfvy": 1.0 + 0.02 * rng.random(s2),
        "rdnw": -(10.0 + rng.random(NZ)),
    }
    d["msfvx_inv"] = 1.0 / d["msfvx"]
    d["dnw"] = 1.0 / d["rdnw"]
    for o_ in ("mut", "muu", "muv", "ru", "rv", "rw", "ww", "cqu", "cqv", "cqw", "alt", "php"):
        d[f"cot_{o_}"] = rng.standard_normal(s2 if o_ in ("mut", "muu", "muv") else sh)
    return {k: v.astype(np.float32) for k, v in d.items()}


def prep_call(dyn, g, name, x):
    """Run one of rk_step_prep's functions with the solver's argument list
    (solver.py:736-778); returns its outputs by name."""
    import torch

    one1 = torch.ones(NZ, dtype=torch.float64)
    z3 = lambda: torch.zeros((NZ, N, N), dtype=torch.float64)  # noqa: E731
    z2 = lambda: torch.zeros((N, N), dtype=torch.float64)  # noqa: E731
    ids, ide, jds, jde = 5, N - 5, 5, N - 5
    idx = (ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)
    if name == "calculate_full":
        return {"mut": dyn.calculate_full(z2(), x["mub"], x["mu"], *idx)}
    if name == "calc_mu_uv":
        muu, muv = dyn.calc_mu_uv(x["mu"], x["mub"], z2(), z2(), *idx)
        return {"muu": muu, "muv": muv}
    if name == "couple_momentum":
        ru, rv, rw = dyn.couple_momentum(x["muu"], z3(), x["u"], x["msfu"], x["muv"], z3(), x["v"], x["msfv"],
                                         x["msfvx_inv"], x["mut"], z3(), x["w"], x["msft"], one1, one1 * 0, one1,
                                         one1 * 0, *idx)
        return {"ru": ru, "rv": rv, "rw": rw}
    if name == "calc_ww_cp":
        ww = dyn.calc_ww_cp(x["u"], x["v"], x["mu"], x["mub"], x["muu"], x["muv"], one1, one1 * 0, x["ww"].clone(),
                            1.0 / g.dx, 1.0 / g.dy, x["msftx"], x["msfty"], x["msfux"], x["msfuy"], x["msfvx"],
                            x["msfvx_inv"], x["msfvy"], x["dnw"], *idx)
        return {"ww": ww}
    if name == "calc_cq":
        cqu, cqv, cqw = dyn.calc_cq(x["moist"], z3(), z3(), z3(), 7, *idx)
        return {"cqu": cqu, "cqv": cqv, "cqw": cqw}
    if name == "calc_alt":
        return {"alt": dyn.calc_alt(z3(), x["al"], x["alb"], *idx)}
    return {"php": dyn.calc_php(z3(), x["ph"], x["phb"], *idx)}


def prep(dyn, g) -> None:
    """rk_step_prep's functions: checksums and central differences
    (prep_adj_ref64.npz)."""
    import torch

    d = prep_inputs()
    save = dict(d)
    base = {k: torch.tensor(v, dtype=torch.float64) for k, v in d.items()}
    with torch.no_grad():
        for fi, (name, (ins, outs)) in enumerate(PREP.items()):
            o0 = prep_call(dyn, g, name, base)
            for o_ in outs:
                a = o0[o_].numpy()
                save[f"{name}_{o_}_sum"] = np.array(a.sum())
                save[f"{name}_{o_}_l2"] = np.array(np.sqrt((a * a).sum()))

            def loss(x):
                oo = prep_call(dyn, g, name, x)
                return float(sum((oo[o_] * x[f"cot_{o_}"]).sum() for o_ in outs))

            for ni, inp in enumerate(ins):
                eps = 1e-4 * float(base[inp].abs().max())
                save[f"{name}_fd_eps_{inp}"] = np.array(eps)
                for r in range(3):
                    dirn = torch.tensor(prep_direction(fi, ni, r, d[inp].shape))
                    xp, xm = dict(base), dict(base)
                    xp[inp] = base[inp] + eps * dirn
                    xm[inp] = base[inp] - eps * dirn
                    save[f"{name}_fd_{inp}_{r}"] = np.array((loss(xp) - loss(xm)) / (2 * eps))
    np.savez_compressed(os.path.join(HERE, "prep_adj_ref64.npz"), **save)
    print("wrote prep_adj_ref64.npz")


def mom_direction(n: int, r: int, shape) -> np.ndarray:
    """Direction r of input n (field, ru, rv, rom) of the advect_w finite
    differences (regenerated by the tests, not stored)."""
    return np.random.default_rng(7000 + 10 * n + r).standard_normal(shape)


def momentum(dyn, g) -> None:
    """advect_u / advect_v / advect_w with autograd (adv_mom_adj_ref64.npz)."""
    import torch

    rng = np.random.default_rng(14)
    shape = (NZ, N, N)
    ids, ide, jds, jde = 5, N - 5, 5, N - 5
    save = {"dx": np.array(g.dx), "dy": np.array(g.dy)}
    prof = {"fnm": 0.45 + 0.1 * rng.random(NZ), "fnp": 0.45 + 0.1 * rng.random(NZ),
            "rdnw": -(8.0 + 4.0 * rng.random(NZ)), "rdn": -(8.0 + 4.0 * rng.random(NZ))}
    prof = {k: v.astype(np.float32) for k, v in prof.items()}
    save.update(prof)
    ones2 = torch.ones((N, N), dtype=torch.float64)
    one1 = torch.ones(NZ, dtype=torch.float64)
    fn = {"u": dyn.advect_u, "v": dyn.advect_v, "w": dyn.advect_w}
    for comp in ("u", "v", "w"):
        d = {
            "field": 4.0 * rng.standard_normal(shape) + (2.0 if comp == "u" else 0.0),
            "ru": 20.0 * rng.standard_normal(shape) + 5.0,
            "rv": 20.0 * rng.standard_normal(shape) - 5.0,
            "rom": 2.0 * rng.standard_normal(shape),
            "msf": 1.0 + 0.05 * rng.random((N, N)),
            "msf2": 1.0 + 0.05 * rng.random((N, N)),
            "cot": rng.standard_normal(shape),
        }
        # float32-representable inputs, stored as float32 (the float64 forward
        # of the stored values is then exactly what the fixture records)
        d = {k: v.astype(np.float32) for k, v in d.items()}
        t = {k: torch.tensor(v, dtype=torch.float64) for k, v in d.items()}
        for k in ("field", "ru", "rv", "rom"):
            t[k].requires_grad_(True)
        # map factors in the reference's argument order msfux, msfuy, msfvx, msfvy, msftx, msfty:
        # advect_u reads msfux, advect_v msfvx and msfvy, advect_w msftx
        msfs = [ones2] * 6
        if comp == "u":
            msfs[0] = t["msf"]
        elif comp == "v":
            msfs[3], msfs[2] = t["msf"], t["msf2"]
        else:
            msfs[4] = t["msf"]
        rdz = torch.tensor(prof["rdn" if comp == "w" else "rdnw"], dtype=torch.float64)
        fnm, fnp = (torch.tensor(prof[k], dtype=torch.float64) for k in ("fnm", "fnp"))
        def run(x):
            return fn[comp](x["field"], x["field"], torch.zeros(shape, dtype=torch.float64), x["ru"], x["rv"],
                            x["rom"], one1, one1 * 0.0, ones2, int(g.dt), *msfs, fnm, fnp, 1.0 / g.dx, 1.0 / g.dy,
                            rdz, ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)

        for k, v in d.items():
            save[f"{comp}_{k}"] = v
        if comp != "w":
            out = run(t)
            (out * t["cot"]).sum().backward()
            save[f"{comp}_tend"] = out.detach().numpy()
            for k in ("field", "ru", "rv", "rom"):
                save[f"{comp}_grad_{k}"] = t[k].grad.numpy()
            continue
        # advect_w: the reference's vertical part rewrites ``vel`` in place
        # after a product saved it (wrf_dynamics.py:1788), so backward()
        # raises; the fixture holds central differences of its float64
        # forward instead (exact up to rounding: the operator is bilinear in
        # (field, velocities) with piecewise-constant upwind choices)
        base = {k: t[k].detach().clone() for k in ("field", "ru", "rv", "rom")}
        with torch.no_grad():
            save["w_tend"] = run(base).numpy()
            cot = t["cot"]
            for n_, name in enumerate(("field", "ru", "rv", "rom")):
                for r in range(3):
                    dirn = mom_direction(n_, r, shape)
                    eps = 1e-6 * float(base[name].abs().max())
                    xp, xm = dict(base), dict(base)
                    xp[name] = base[name] + eps * torch.tensor(dirn)
                    xm[name] = base[name] - eps * torch.tensor(dirn)
                    save[f"w_fd_{name}_{r}"] = np.array(
                        float(((run(xp) - run(xm)) * cot).sum()) / (2 * eps))
    np.savez_compressed(os.path.join(HERE, "adv_mom_adj_ref64.npz"), **save)
    print("wrote adv_mom_adj_ref64.npz")


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=None)
    ap.add_argument("--only", choices=("scalar", "relax", "coefw", "momentum", "advance_uv", "calc_p_rho", "advance_mu_t", "advance_w",
                             "forces", "subbdy", "prep"), default=None,
                    help="write one fixture only")
    a = ap.parse_args()
    if a.reference:
        os.environ["PYWRF_REFERENCE_ROOT"] = a.reference
    import torch

    import refharness
    spec = synthetic.CaseSpec(n=N, nz=NZ)
    g = synthetic.grid_for(spec)
    _cp, dyn, _phy, _bdy, _solver = refharness.load_reference(g, dtype="float64")
    if a.only == "momentum":
        momentum(dyn, g)
        return
    if a.only == "advance_uv":
        advance_uv(dyn, importlib_bdy(), g)
        return
    if a.only == "calc_p_rho":
        calc_p_rho(dyn, g)
        return
    if a.only == "advance_mu_t":
        advance_mu_t(dyn, g)
        return
    if a.only == "advance_w":
        advance_w(dyn, g)
        return
    if a.only == "forces":
        forces(dyn, g)
        return
    if a.only == "subbdy":
        subbdy(dyn, importlib_bdy(), g)
        return
    if a.only == "prep":
        prep(dyn, g)
        return
    if a.only is not None:
        raise SystemExit("--only: scalar, relax and coefw are written together (no --only)")
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

    # relax_bdytend
    bnd = importlib_bdy()
    rng = np.random.default_rng(12)
    shape = (NZ, N, N)
    gcx = torch.tensor([0., 1.1111111e-3, 7.4074074e-4, 3.7037037e-4, 0.], dtype=torch.float64)
    fcx = torch.tensor([0., 5.5555557e-3, 3.7037039e-3, 1.8518519e-3, 0.], dtype=torch.float64)
    out = {"dtbc": np.array(135.0)}
    for var in ("t", "u", "v", "h"):
        field = torch.tensor(300.0 + rng.standard_normal(shape), dtype=torch.float64, requires_grad=True)
        arrs = [rng.standard_normal((NZ, N, 5)) + 300.0, rng.standard_normal((NZ, N, 5)) + 300.0,
                rng.standard_normal((NZ, 5, N)) + 300.0, rng.standard_normal((NZ, 5, N)) + 300.0,
                1e-3 * rng.standard_normal((NZ, N, 5)), 1e-3 * rng.standard_normal((NZ, N, 5)),
                1e-3 * rng.standard_normal((NZ, 5, N)), 1e-3 * rng.standard_normal((NZ, 5, N))]
        tb = [torch.tensor(a, dtype=torch.float64) for a in arrs]
        tend0 = torch.tensor(rng.standard_normal(shape), dtype=torch.float64)
        cot = rng.standard_normal(shape)
        res = bnd.relax_bdytend(field, tend0.clone(), *tb, var, 5, 1, 4, 135.0, fcx, gcx,
                                ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, 0, N, 0, N, 0, NZ,
                                ids, ide, jds, jde, 0, NZ)
        (res * torch.tensor(cot)).sum().backward()
        out[f"{var}_field"] = field.detach().numpy()
        out[f"{var}_tend0"] = tend0.numpy()
        for nm, a in zip(("xs", "xe", "ys", "ye", "txs", "txe", "tys", "tye"), arrs):
            out[f"{var}_{nm}"] = a
        out[f"{var}_cot"] = cot
        out[f"{var}_tend"] = res.detach().numpy()
        out[f"{var}_grad_field"] = field.grad.numpy()
    np.savez_compressed(os.path.join(HERE, "relax_adj_ref64.npz"), **out)
    print("wrote relax_adj_ref64.npz")

    # calc_coef_w
    rng = np.random.default_rng(13)
    mut = torch.tensor(8.0e4 + 1.0e3 * rng.standard_normal((N, N)), dtype=torch.float64)
    cqw = torch.tensor(0.99 + 0.005 * rng.standard_normal(shape), dtype=torch.float64)
    c2a = torch.tensor(1.6e5 + 1.0e4 * rng.standard_normal(shape), dtype=torch.float64)
    rdn = torch.tensor(-(35.0 + 10.0 * rng.random(NZ)), dtype=torch.float64)
    rdnw = torch.tensor(-(35.0 + 10.0 * rng.random(NZ)), dtype=torch.float64)
    a0, al0, g0 = (torch.zeros(shape, dtype=torch.float64) for _ in range(3))
    one1 = torch.ones(NZ, dtype=torch.float64)
    dts, epssm = 11.25, 0.1
    ca, cal, cg = (rng.standard_normal(shape) for _ in range(3))
    tca, tcal, tcg = torch.tensor(ca), torch.tensor(cal), torch.tensor(cg)
    base = {"mut": mut.detach().clone(), "cqw": cqw.detach().clone(), "c2a": c2a.detach().clone()}

    def loss(x):
        bufs = [torch.zeros(shape, dtype=torch.float64) for _ in range(3)]
        a_, al_, g_ = dyn.calc_coef_w(*bufs, x["mut"], one1, one1 * 0, one1, one1 * 0, one1, one1 * 0, one1,
                                      one1 * 0, x["cqw"], rdn, rdnw, x["c2a"], dts, 9.81, epssm, False,
                                      ids, ide, jds, jde, 0, NZ, 0, N, 0, N, 0, NZ, ids, ide, jds, jde, 0, NZ)
        return float((a_ * tca).sum() + (al_ * tcal).sum() + (g_ * tcg).sum()), (a_, al_, g_)

    _, (a_, al_, g_) = loss(base)
    save = dict(mut=base["mut"].numpy(), cqw=base["cqw"].numpy(), c2a=base["c2a"].numpy(), rdn=rdn.numpy(),
                rdnw=rdnw.numpy(), dts=np.array(dts), epssm=np.array(epssm), a=a_.numpy(), alpha=al_.numpy(),
                gamma=g_.numpy(), cot_a=ca, cot_alpha=cal, cot_gamma=cg)
    for name in ("mut", "cqw", "c2a"):
        for r in range(3):
            d = rng.standard_normal(tuple(base[name].shape))
            eps = 1e-6 * float(base[name].abs().max())
            xp, xm = dict(base), dict(base)
            xp[name] = base[name] + eps * torch.tensor(d)
            xm[name] = base[name] - eps * torch.tensor(d)
            save[f"dir_{name}_{r}"] = d
            save[f"fd_{name}_{r}"] = np.array((loss(xp)[0] - loss(xm)[0]) / (2 * eps))
    np.savez_compressed(os.path.join(HERE, "coefw_adj_ref64.npz"), **save)
    print("wrote coefw_adj_ref64.npz")
    momentum(dyn, g)
    advance_uv(dyn, importlib_bdy(), g)
    calc_p_rho(dyn, g)
    advance_mu_t(dyn, g)
    advance_w(dyn, g)
    forces(dyn, g)
    subbdy(dyn, importlib_bdy(), g)
    prep(dyn, g)


def importlib_bdy():
    import importlib
    return importlib.import_module("pywrf.wrf_boundary")


if __name__ == "__main__":
    main()
