"""Oracle restatement of the dynamics functions (reference pywrf/wrf_dynamics.py).

TEST INFRASTRUCTURE: see oracle/__init__.py.  Conventions: ``g`` is a
``pywrf_b200.config.Grid``; 3-D arrays are ``[nz, ny, nx]``; arrays are
updated in place over exactly the index regions the reference writes; scalars
are Python floats so numpy keeps the arrays' dtype (float32 or float64).
The arithmetic order of each expression follows the reference so that the
fp32 results agree to rounding.
"""
from __future__ import annotations

import numpy as np

G = 9.81
T0 = 300.0
P0 = 1.0e5
CPOVCV = 1.4
R_D = 287.0
RVOVRD = 1.608362
RERADIUS = 1.5698588e-7
C_S = 0.25
PRANDTL = 1.0 / 3.0


def _r(a, k0, k1, j0, j1, i0, i1):
    return a[k0:k1, j0:j1, i0:i1]


# ---------------------------------------------------------------- RK-stage prep

def calculate_full(g, mut, mub, mu):
    """wrf_dynamics.py:30-38"""
    mut[g.jds:g.jde - 1, g.ids:g.ide - 1] = mub[g.jds:g.jde - 1, g.ids:g.ide - 1] + mu[g.jds:g.jde - 1, g.ids:g.ide - 1]
    return mut


def calc_mu_uv(g, mu, mub, muu, muv):
    """wrf_dynamics.py:41-61"""
    js, je = g.jds, g.jde - 1
    i0, ite = g.ids, g.ide
    muu[js:je, i0 + 1:ite - 1] = 0.5 * (mu[js:je, i0 + 1:ite - 1] + mu[js:je, i0:ite - 2]
                                        + mub[js:je, i0 + 1:ite - 1] + mub[js:je, i0:ite - 2])
    muu[js:je, i0] = mu[js:je, i0] + mub[js:je, i0]
    muu[js:je, ite - 1] = mu[js:je, ite - 2] + mub[js:je, ite - 2]
    ie = g.ide - 1
    j0, jte = g.jds, g.jde
    muv[j0 + 1:jte - 1, i0:ie] = 0.5 * (mu[j0 + 1:jte - 1, i0:ie] + mu[j0:jte - 2, i0:ie]
                                         + mub[j0 + 1:jte - 1, i0:ie] + mub[j0:jte - 2, i0:ie])
    muv[j0, i0:ie] = mu[j0, i0:ie] + mub[j0, i0:ie]
    muv[jte - 1, i0:ie] = mu[jte - 2, i0:ie] + mub[jte - 2, i0:ie]
    return muu, muv


def couple_momentum(g, muu, ru, u, msfu, muv, rv, v, msfvx_inv, mut, rw, w, msft):
    """wrf_dynamics.py:64-86"""
    ktf = g.nz - 1
    js, jm = g.jds, g.jde - 1
    ru[0:ktf, js:jm, g.ids:g.ide] = u[0:ktf, js:jm, g.ids:g.ide] * muu[None, js:jm, g.ids:g.ide] / msfu[None, js:jm, g.ids:g.ide]
    rv[0:ktf, js:g.jde, g.ids:g.ide - 1] = (v[0:ktf, js:g.jde, g.ids:g.ide - 1] * muv[None, js:g.jde, g.ids:g.ide - 1]
                                             * msfvx_inv[None, js:g.jde, g.ids:g.ide - 1])
    rw[0:g.nz, js:jm, g.ids:g.ide - 1] = w[0:g.nz, js:jm, g.ids:g.ide - 1] * mut[None, js:jm, g.ids:g.ide - 1] / msft[None, js:jm, g.ids:g.ide - 1]
    return ru, rv, rw


def calc_ww_cp(g, u, v, muu, muv, c1h, ww, msftx, msfuy, msfvx_inv, dnw):
    """wrf_dynamics.py:89-118 (column divergence, its k-sum, upward scan)."""
    ktf = g.nz - 1
    js, je, i0, ie = g.jds, g.jde - 1, g.ids, g.ide - 1
    rdx, rdy = g.rdx, g.rdy
    fu = muu[None, js:je, i0:ie + 1] * u[0:ktf, js:je, i0:ie + 1] / msfuy[None, js:je, i0:ie + 1]
    fv = muv[None, js:je + 1, i0:ie] * v[0:ktf, js:je + 1, i0:ie] * msfvx_inv[None, js:je + 1, i0:ie]
    divv = (msftx[None, js:je, i0:ie] * dnw[0:ktf, None, None]
            * (rdx * (fu[:, :, 1:] - fu[:, :, :-1]) + rdy * (fv[:, 1:, :] - fv[:, :-1, :])))
    dmdt = np.zeros_like(divv[0])
    for k in range(ktf):
        dmdt = dmdt + divv[k]
    for k in range(ktf - 1):
        ww[k + 1, js:je, i0:ie] = ww[k, js:je, i0:ie] - (dnw[k] * c1h[k]) * dmdt - divv[k]
    return ww


def calc_cq(g, moist, cqu, cqv, cqw):
    """wrf_dynamics.py:121-136 (moist[0..6] summed in slot order)."""
    ktf = g.nz - 1
    qs = moist[0].copy()
    for m in range(1, moist.shape[0]):
        qs = qs + moist[m]
    js, jm = g.jds, g.jde - 1
    cqu[0:ktf, js:jm, g.ids:g.ide] = 1.0 / (1.0 + 0.5 * (qs[0:ktf, js:jm, g.ids:g.ide] + qs[0:ktf, js:jm, g.ids - 1:g.ide - 1]))
    cqv[0:ktf, js:g.jde, g.ids:g.ide - 1] = 1.0 / (1.0 + 0.5 * (qs[0:ktf, js:g.jde, g.ids:g.ide - 1] + qs[0:ktf, js - 1:g.jde - 1, g.ids:g.ide - 1]))
    cqw[1:ktf, js:jm, g.ids:g.ide - 1] = 0.5 * (qs[1:ktf, js:jm, g.ids:g.ide - 1] + qs[0:ktf - 1, js:jm, g.ids:g.ide - 1])
    return cqu, cqv, cqw


def calc_alt(g, alt, al, alb):
    """wrf_dynamics.py:139-147"""
    ktf = g.nz - 1
    sl = (slice(0, ktf), slice(g.jds, g.jde - 1), slice(g.ids, g.ide - 1))
    alt[sl] = al[sl] + alb[sl]
    return alt


def calc_php(g, php, ph, phb):
    """wrf_dynamics.py:150-159"""
    ktf = g.nz - 1
    js, jm, i0, im = g.jds, g.jde - 1, g.ids, g.ide - 1
    php[0:ktf, js:jm, i0:im] = 0.5 * (phb[0:ktf, js:jm, i0:im] + phb[1:ktf + 1, js:jm, i0:im]
                                      + ph[0:ktf, js:jm, i0:im] + ph[1:ktf + 1, js:jm, i0:im])
    return php


# -------------------------------------------------------- open lateral halo copies

def set_physical_bc3d(g, dat, var):
    """wrf_dynamics.py:216-278: 3-cell open-boundary halo copy.  x sides first
    (their rows reach into the y halo, which still holds the previous values),
    then y sides."""
    v = {"U": "u", "V": "v", "M": "m", "H": "h"}.get(var, var)
    if v not in ("u", "v", "w", "t", "d", "e", "x", "y", "f", "r", "p"):
        raise ValueError(f"no open-bc copy for stagger {var!r}")
    istag = 0 if v in ("u", "x", "d") else -1
    jstag = 0 if v in ("v", "y", "d") else -1
    if v == "e":
        istag = 0
    if v == "f":
        jstag = 0
    k_end = g.nz if v in ("e", "f", "w") else g.nz - 1
    ids, ide, jds, jde = g.ids, g.ide, g.jds, g.jde
    r0, r1 = g.jds - 4, jde + jstag + 4
    for h in (1, 2, 3):
        dat[0:k_end, r0:r1, ids - h] = dat[0:k_end, r0:r1, ids]
    if v not in ("u", "x"):
        for c in (ide - 1, ide, ide + 1):
            dat[0:k_end, r0:r1, c] = dat[0:k_end, r0:r1, ide - 2]
    else:
        for c in (ide, ide + 1, ide + 2):
            dat[0:k_end, g.jds - 5:r1, c] = dat[0:k_end, g.jds - 5:r1, ide - 1]
    c0, c1 = ids, ide + istag
    for h in (1, 2, 3):
        dat[0:k_end, jds - h, c0:c1] = dat[0:k_end, jds, c0:c1]
    if v not in ("v", "y"):
        for r in (jde - 1, jde, jde + 1):
            dat[0:k_end, r, c0:c1] = dat[0:k_end, jde - 2, c0:c1]
    else:
        for r in (jde, jde + 1, jde + 2):
            dat[0:k_end, r, c0:c1] = dat[0:k_end, jde - 1, c0:c1]
    return dat


def set_physical_bc2d(g, dat, var):
    """wrf_dynamics.py:164-212 (rows of the x copy are not extended)."""
    v = var.lower()
    if v not in ("u", "v", "w", "t", "x", "y", "r", "p"):
        raise ValueError(f"no open-bc copy for stagger {var!r}")
    istag = 0 if v in ("u", "x") else -1
    jstag = 0 if v in ("v", "y") else -1
    ids, ide, jds, jde = g.ids, g.ide, g.jds, g.jde
    r0, r1 = jds, jde + jstag
    for h in (1, 2, 3):
        dat[r0:r1, ids - h] = dat[r0:r1, ids]
    if v not in ("u", "x"):
        for c in (ide - 1, ide, ide + 1):
            dat[r0:r1, c] = dat[r0:r1, ide - 2]
    else:
        for c in (ide, ide + 1, ide + 2):
            dat[r0:r1, c] = dat[r0:r1, ide - 1]
    c0, c1 = max(ids, g.its - 1), min(g.ite + 1, ide + istag)
    for h in (1, 2, 3):
        dat[jds - h, c0:c1] = dat[jds, c0:c1]
    if v not in ("v", "y"):
        for r in (jde - 1, jde, jde + 1):
            dat[r, c0:c1] = dat[jde - 2, c0:c1]
    else:
        for r in (jde, jde + 1, jde + 2):
            dat[r, c0:c1] = dat[jde - 1, c0:c1]
    return dat


# ------------------------------------------------ first-stage diffusion set-up

def compute_diff_metrics(g, ph, phb, z, rdz, rdzw, zx, zy):
    """wrf_dynamics.py:491-536"""
    ktf = g.nz - 1
    js, je = g.jds - 1, g.jde
    i0, ie = g.ids, g.ide - 1
    zaw = np.zeros_like(ph)
    zaw[0:g.nz, js:je, i0:ie] = (ph[0:g.nz, js:je, i0:ie] + phb[0:g.nz, js:je, i0:ie]) / G
    rdzw[0:ktf, js:je, i0:ie] = 1.0 / (zaw[1:ktf + 1, js:je, i0:ie] - zaw[0:ktf, js:je, i0:ie])
    rdz[1:ktf, js:je, i0:ie] = 2.0 / (zaw[2:ktf + 1, js:je, i0:ie] - zaw[0:ktf - 1, js:je, i0:ie])
    rdz[0, js:je, i0:ie] = 2.0 / (zaw[1, js:je, i0:ie] - zaw[0, js:je, i0:ie])
    js, je = g.jds, g.jde - 1
    ids, ide, jds, jde = g.ids, g.ide, g.jds, g.jde
    zx[0:g.nz, js:je, ids + 1:ie] = (g.rdx * (phb[0:g.nz, js:je, ids + 1:ie] - phb[0:g.nz, js:je, ids:ie - 1]) / G
                                     + g.rdx * (ph[0:g.nz, js:je, ids + 1:ie] - ph[0:g.nz, js:je, ids:ie - 1]) / G)
    zy[0:g.nz, jds + 1:je, i0:ie] = (g.rdy * (phb[0:g.nz, jds + 1:je, i0:ie] - phb[0:g.nz, jds:je - 1, i0:ie]) / G
                                     + g.rdy * (ph[0:g.nz, jds + 1:je, i0:ie] - ph[0:g.nz, jds:je - 1, i0:ie]) / G)
    zx[0:ktf, js:je, ide - 1] = 0.0
    zx[0:ktf, js:je, ids - 1] = 0.0
    zy[0:ktf, jde - 1, i0:ie] = 0.0
    zy[0:ktf, jds - 1, i0:ie] = 0.0
    z[0:ktf, js:je, i0:ie] = 0.5 * (ph[0:ktf, js:je, i0:ie] + phb[0:ktf, js:je, i0:ie]
                                    + ph[1:ktf + 1, js:je, i0:ie] + phb[1:ktf + 1, js:je, i0:ie])
    return rdzw, rdz, zx, zy, z


def _hatavg_z(g, hat, hatavg, k_sl_lo, sl_a, sl_b, fnm, fnp, cf1, cf2, cf3, cft1, cft2):
    """Vertical averaging of a horizontally-averaged ``hat`` used by each
    deformation component (wrf_dynamics.py:579-592 and the three repeats):
    ``sl_a``/``sl_b`` select the two horizontal neighbours averaged."""
    ktf = g.nz - 1
    kt1, kt2 = g.nz - 2, g.nz - 3
    ja, ia = sl_a
    jb, ib = sl_b
    jt, it = k_sl_lo
    hatavg[1:ktf, jt, it] = 0.5 * (fnm[1:ktf, None, None] * (hat[1:ktf, ja, ia] + hat[1:ktf, jb, ib])
                                   + fnp[1:ktf, None, None] * (hat[0:ktf - 1, ja, ia] + hat[0:ktf - 1, jb, ib]))
    hatavg[0, jt, it] = 0.5 * (cf1 * hat[0, ja, ia] + cf2 * hat[1, ja, ia] + cf3 * hat[2, ja, ia]
                               + cf1 * hat[0, jb, ib] + cf2 * hat[1, jb, ib] + cf3 * hat[2, jb, ib])
    hatavg[g.nz - 1, jt, it] = 0.5 * (cft1 * (hat[kt1, ja, ia] + hat[kt1, jb, ib])
                                      + cft2 * (hat[kt2, ja, ia] + hat[kt2, jb, ib]))


def cal_deform_and_div(g, u, v, defor11, defor22, defor12, msfux, msfuy, msfvx, msfvy,
                       msftx, msfty, dn, dnw, rdzw, fnm, fnp, cf1, cf2, cf3, zx, zy):
    """wrf_dynamics.py:539-813, restricted to the components the step consumes:
    defor11, defor22 and defor12 feed the Smagorinsky coefficient
    (wrf_dynamics.py:967-986); defor13/23/33 and div only feed the discarded
    Brunt-Vaisala term and are not formed."""
    ktf = g.nz - 1
    kt1 = g.nz - 2
    cft2 = -0.5 * dnw[kt1] / dn[kt1]
    cft1 = 1.0 - cft2
    dt_ = u.dtype
    hat = np.zeros_like(u)
    hatavg = np.zeros_like(u)
    # --- defor11 (A region) ---
    js, je, i0, ie = g.jds, g.jde - 1, g.ids, g.ide - 1
    A = (slice(js, je), slice(i0, ie))
    mm = msftx[A] * msfty[A]
    hat[0:ktf, js:je, i0:ie + 1] = u[0:ktf, js:je, i0:ie + 1] / msfuy[None, js:je, i0:ie + 1]
    _hatavg_z(g, hat, hatavg, A, (slice(js, je), slice(i0, ie)), (slice(js, je), slice(i0 + 1, ie + 1)),
              fnm, fnp, cf1, cf2, cf3, cft1, cft2)
    tmp1 = ((hatavg[1:ktf + 1, js:je, i0:ie] - hatavg[0:ktf, js:je, i0:ie])
            * (0.25 * (zx[0:ktf, js:je, i0:ie] + zx[0:ktf, js:je, i0 + 1:ie + 1]
                       + zx[1:ktf + 1, js:je, i0:ie] + zx[1:ktf + 1, js:je, i0 + 1:ie + 1])
               * rdzw[0:ktf, js:je, i0:ie]))
    tmp1 = mm[None] * (g.rdx * (hat[0:ktf, js:je, i0 + 1:ie + 1] - hat[0:ktf, js:je, i0:ie]) - tmp1)
    defor11[0:ktf, js:je, i0:ie] = 2.0 * tmp1
    # --- defor22 ---
    hat[0:ktf, js:je + 1, i0:ie] = v[0:ktf, js:je + 1, i0:ie] / msfvx[None, js:je + 1, i0:ie]
    _hatavg_z(g, hat, hatavg, A, (slice(js, je), slice(i0, ie)), (slice(js + 1, je + 1), slice(i0, ie)),
              fnm, fnp, cf1, cf2, cf3, cft1, cft2)
    tmp1 = mm[None] * (g.rdy * (hat[0:ktf, js + 1:je + 1, i0:ie] - hat[0:ktf, js:je, i0:ie])
                       - (hatavg[1:ktf + 1, js:je, i0:ie] - hatavg[0:ktf, js:je, i0:ie])
                       * (0.25 * (zy[0:ktf, js:je, i0:ie] + zy[0:ktf, js + 1:je + 1, i0:ie]
                                  + zy[1:ktf + 1, js:je, i0:ie] + zy[1:ktf + 1, js + 1:je + 1, i0:ie])
                          * rdzw[0:ktf, js:je, i0:ie]))
    defor22[0:ktf, js:je, i0:ie] = 2.0 * tmp1
    # --- defor12 (B region: corner points) ---
    i0, ie = g.its + 1, g.ite - 1
    j0, je = g.jts + 1, g.jte - 1
    B = (slice(j0, je), slice(i0, ie))
    mmb = (0.25 * (msfux[j0 - 1:je - 1, i0:ie] + msfux[j0:je, i0:ie])
           * (msfvy[j0:je, i0 - 1:ie - 1] + msfvy[j0:je, i0:ie]))
    hat[0:ktf, j0 - 1:je, i0:ie] = u[0:ktf, j0 - 1:je, i0:ie] / msfux[None, j0 - 1:je, i0:ie]
    _hatavg_z(g, hat, hatavg, B, (slice(j0 - 1, je - 1), slice(i0, ie)), (slice(j0, je), slice(i0, ie)),
              fnm, fnp, cf1, cf2, cf3, cft1, cft2)
    rsum = (rdzw[0:ktf, j0:je, i0:ie] + rdzw[0:ktf, j0:je, i0 - 1:ie - 1]
            + rdzw[0:ktf, j0 - 1:je - 1, i0 - 1:ie - 1] + rdzw[0:ktf, j0 - 1:je - 1, i0:ie])
    tmp1 = ((hatavg[1:ktf + 1, j0:je, i0:ie] - hatavg[0:ktf, j0:je, i0:ie])
            * (0.25 * (zy[0:ktf, j0:je, i0 - 1:ie - 1] + zy[0:ktf, j0:je, i0:ie]
                       + zy[1:ktf + 1, j0:je, i0 - 1:ie - 1] + zy[1:ktf + 1, j0:je, i0:ie]) * 0.25 * rsum))
    d12 = mmb[None] * (g.rdy * (hat[0:ktf, j0:je, i0:ie] - hat[0:ktf, j0 - 1:je - 1, i0:ie]) - tmp1)
    hat[0:ktf, j0:je, i0 - 1:ie] = v[0:ktf, j0:je, i0 - 1:ie] / msfvy[None, j0:je, i0 - 1:ie]
    _hatavg_z(g, hat, hatavg, B, (slice(j0, je), slice(i0 - 1, ie - 1)), (slice(j0, je), slice(i0, ie)),
              fnm, fnp, cf1, cf2, cf3, cft1, cft2)
    rsum = (rdzw[0:ktf, j0:je, i0:ie] + rdzw[0:ktf, j0 - 1:je - 1, i0:ie]
            + rdzw[0:ktf, j0 - 1:je - 1, i0 - 1:ie - 1] + rdzw[0:ktf, j0:je, i0 - 1:ie - 1])
    tmp1 = ((hatavg[1:ktf + 1, j0:je, i0:ie] - hatavg[0:ktf, j0:je, i0:ie])
            * (0.25 * (zx[0:ktf, j0 - 1:je - 1, i0:ie] + zx[0:ktf, j0:je, i0:ie]
                       + zx[1:ktf + 1, j0 - 1:je - 1, i0:ie] + zx[1:ktf + 1, j0:je, i0:ie]) * 0.25 * rsum))
    defor12[0:ktf, j0:je, i0:ie] = d12 + mmb[None] * (g.rdx * (hat[0:ktf, j0:je, i0:ie] - hat[0:ktf, j0:je, i0 - 1:ie - 1]) - tmp1)
    ids, ide, jds, jde = g.ids, g.ide, g.jds, g.jde
    defor12[0:g.nz, g.jts:g.jte, ids] = defor12[0:g.nz, g.jts:g.jte, ids + 1]
    defor12[0:g.nz, g.jts:g.jte, ide - 1] = defor12[0:g.nz, g.jts:g.jte, ide - 2]
    defor12[0:g.nz, jds, g.its:g.ite] = defor12[0:g.nz, jds + 1, g.its:g.ite]
    defor12[0:g.nz, jde - 1, g.its:g.ite] = defor12[0:g.nz, jde - 2, g.its:g.ite]
    del dt_
    return defor11, defor12, defor22


def calculate_km_kh(g, xkmh, xkhh, defor11, defor22, defor12, msftx, msfty):
    """wrf_dynamics.py:958-995 (2-D Smagorinsky).  Outside the computed
    region the reference's clamp ``where(xkmh < 10 l, xkmh, 10 l)`` with
    ``l = 0`` zeroes xkmh; xkhh keeps its previous values there."""
    ktf = g.nz - 1
    i0, ie = g.its + 1, min(g.ite, g.ide - 2)
    j0, je = g.jts + 1, min(g.jte, g.jde - 2)
    d = defor11[0:ktf, j0:je, i0:ie] - defor22[0:ktf, j0:je, i0:ie]
    def2 = 0.25 * (d * d)
    tmp = 0.25 * (defor12[0:ktf, j0:je, i0:ie] + defor12[0:ktf, j0 + 1:je + 1, i0:ie]
                  + defor12[0:ktf, j0:je, i0 + 1:ie + 1] + defor12[0:ktf, j0 + 1:je + 1, i0 + 1:ie + 1])
    def2 = def2 + tmp * tmp
    mlen = np.sqrt(g.dx / msftx[j0:je, i0:ie] * g.dy / msfty[j0:je, i0:ie])
    tmp = np.sqrt(def2)
    val = C_S * C_S * mlen[None] * mlen[None] * tmp
    cap = 10.0 * mlen[None]
    region = np.zeros_like(xkmh)
    region[0:ktf, j0:je, i0:ie] = val
    capfull = np.zeros_like(xkmh)
    capfull[:, j0:je, i0:ie] = cap
    # the clamp runs over the whole array (levels and halos included)
    src = xkmh.copy()
    src[0:ktf, j0:je, i0:ie] = val
    xkmh[...] = np.where(src < capfull, src, capfull)
    xkhh[0:ktf, j0:je, i0:ie] = xkmh[0:ktf, j0:je, i0:ie] / PRANDTL
    return xkmh, xkhh


def _hdiff_core(tend, f, ks, js, is_, mkrdxm, mkrdxp, mrdx, mkrdym, mkrdyp, mrdy, base=None):
    k0, k1 = ks
    j0, j1 = js
    i0, i1 = is_
    c = f[k0:k1, j0:j1, i0:i1]
    fxp, fxm = f[k0:k1, j0:j1, i0 + 1:i1 + 1], f[k0:k1, j0:j1, i0 - 1:i1 - 1]
    fyp, fym = f[k0:k1, j0 + 1:j1 + 1, i0:i1], f[k0:k1, j0 - 1:j1 - 1, i0:i1]
    if base is None:
        dxp, dxm = fxp - c, c - fxm
        dyp, dym = fyp - c, c - fym
    else:
        b = base[k0:k1, j0:j1, i0:i1]
        dxp = fxp - c - base[k0:k1, j0:j1, i0 + 1:i1 + 1] + b
        dxm = c - fxm - b + base[k0:k1, j0:j1, i0 - 1:i1 - 1]
        dyp = fyp - c - base[k0:k1, j0 + 1:j1 + 1, i0:i1] + b
        dym = c - fym - b + base[k0:k1, j0 - 1:j1 - 1, i0:i1]
    tend[k0:k1, j0:j1, i0:i1] = tend[k0:k1, j0:j1, i0:i1] + (
        mrdx * (mkrdxp * dxp - mkrdxm * dxm) + mrdy * (mkrdyp * dyp - mkrdym * dym))


def horizontal_diffusion(g, name, field, tend, mut, msfux, msfuy, msfvx, msfvx_inv, msfvy,
                         msftx, msfty, xkmhd, base=None):
    """wrf_dynamics.py:2623-2838 ('u', 'v', 'w' and scalar 'm'); with ``base``
    it is horizontal_diffusion_3dmp (wrf_dynamics.py:2841-2915)."""
    ktf = g.nz - 1
    rdx, rdy = g.rdx, g.rdy
    X = lambda a, j0, j1, i0, i1: a[None, j0:j1, i0:i1]
    K = lambda k0, k1, j0, j1, i0, i1: xkmhd[k0:k1, j0:j1, i0:i1]
    if name == "u":
        i0, i1 = g.ids + 1, g.ide - 1
        j0, j1 = g.jds + 1, g.jde - 2
        k0, k1 = 0, ktf
        mkrdxm = (X(msftx, j0, j1, i0 - 1, i1 - 1) / X(msfty, j0, j1, i0 - 1, i1 - 1)) * X(mut, j0, j1, i0 - 1, i1 - 1) * K(k0, k1, j0, j1, i0 - 1, i1 - 1) * rdx
        mkrdxp = (X(msftx, j0, j1, i0, i1) / X(msfty, j0, j1, i0, i1)) * X(mut, j0, j1, i0, i1) * K(k0, k1, j0, j1, i0, i1) * rdx
        mrdx = X(msfux, j0, j1, i0, i1) * X(msfuy, j0, j1, i0, i1) * rdx
        mkrdym = (((X(msfuy, j0, j1, i0, i1) + X(msfuy, j0 - 1, j1 - 1, i0, i1))
                   / (X(msfux, j0, j1, i0, i1) + X(msfux, j0 - 1, j1 - 1, i0, i1))) * 0.25
                  * (X(mut, j0, j1, i0, i1) + X(mut, j0 - 1, j1 - 1, i0, i1) + X(mut, j0 - 1, j1 - 1, i0 - 1, i1 - 1) + X(mut, j0, j1, i0 - 1, i1 - 1)) * 0.25
                  * (K(k0, k1, j0, j1, i0, i1) + K(k0, k1, j0 - 1, j1 - 1, i0, i1) + K(k0, k1, j0 - 1, j1 - 1, i0 - 1, i1 - 1) + K(k0, k1, j0, j1, i0 - 1, i1 - 1)) * rdy)
        mkrdyp = (((X(msfuy, j0, j1, i0, i1) + X(msfuy, j0 + 1, j1 + 1, i0, i1))
                   / (X(msfux, j0, j1, i0, i1) + X(msfux, j0 + 1, j1 + 1, i0, i1))) * 0.25
                  * (X(mut, j0, j1, i0, i1) + X(mut, j0 + 1, j1 + 1, i0, i1) + X(mut, j0 + 1, j1 + 1, i0 - 1, i1 - 1) + X(mut, j0, j1, i0 - 1, i1 - 1)) * 0.25
                  * (K(k0, k1, j0, j1, i0, i1) + K(k0, k1, j0 + 1, j1 + 1, i0, i1) + K(k0, k1, j0 + 1, j1 + 1, i0 - 1, i1 - 1) + K(k0, k1, j0, j1, i0 - 1, i1 - 1)) * rdy)
        mrdy = X(msfux, j0, j1, i0, i1) * X(msfuy, j0, j1, i0, i1) * rdy
    elif name == "v":
        i0, i1 = g.ids + 1, g.ide - 2
        j0, j1 = g.jds + 1, g.jde - 1
        k0, k1 = 0, ktf
        mkrdxm = (((X(msfvx, j0, j1, i0, i1) + X(msfvx, j0, j1, i0 - 1, i1 - 1))
                   / (X(msfvy, j0, j1, i0, i1) + X(msfvy, j0, j1, i0 - 1, i1 - 1))) * 0.25
                  * (X(mut, j0, j1, i0, i1) + X(mut, j0 - 1, j1 - 1, i0, i1) + X(mut, j0 - 1, j1 - 1, i0 - 1, i1 - 1) + X(mut, j0, j1, i0 - 1, i1 - 1)) * 0.25
                  * (K(k0, k1, j0, j1, i0, i1) + K(k0, k1, j0 - 1, j1 - 1, i0, i1) + K(k0, k1, j0 - 1, j1 - 1, i0 - 1, i1 - 1) + K(k0, k1, j0, j1, i0 - 1, i1 - 1)) * rdx)
        mkrdxp = (((X(msfvx, j0, j1, i0, i1) + X(msfvx, j0, j1, i0 + 1, i1 + 1))
                   / (X(msfvy, j0, j1, i0, i1) + X(msfvy, j0, j1, i0 + 1, i1 + 1))) * 0.25
                  * (X(mut, j0, j1, i0, i1) + X(mut, j0 - 1, j1 - 1, i0, i1) + X(mut, j0 - 1, j1 - 1, i0 + 1, i1 + 1) + X(mut, j0, j1, i0 + 1, i1 + 1)) * 0.25
                  * (K(k0, k1, j0, j1, i0, i1) + K(k0, k1, j0 - 1, j1 - 1, i0, i1) + K(k0, k1, j0 - 1, j1 - 1, i0 + 1, i1 + 1) + K(k0, k1, j0, j1, i0 + 1, i1 + 1)) * rdx)
        mrdx = X(msfvx, j0, j1, i0, i1) * X(msfvy, j0, j1, i0, i1) * rdx
        mkrdym = (X(msfty, j0 - 1, j1 - 1, i0, i1) / X(msftx, j0 - 1, j1 - 1, i0, i1)) * K(k0, k1, j0 - 1, j1 - 1, i0, i1) * rdy
        mkrdyp = (X(msfty, j0, j1, i0, i1) / X(msftx, j0, j1, i0, i1)) * K(k0, k1, j0, j1, i0, i1) * rdy
        mrdy = X(msfvx, j0, j1, i0, i1) * X(msfvy, j0, j1, i0, i1) * rdy
    elif name == "w":
        i0, i1 = g.ids + 1, g.ide - 2
        j0, j1 = g.jds + 1, g.jde - 2
        k0, k1 = 1, ktf
        m = lambda jj, ii: X(mut, j0 + jj, j1 + jj, i0 + ii, i1 + ii)
        kk = lambda kd, jj, ii: K(k0 + kd, k1 + kd, j0 + jj, j1 + jj, i0 + ii, i1 + ii)
        mkrdxm = ((X(msfux, j0, j1, i0, i1) / X(msfuy, j0, j1, i0, i1)) * 0.25 * (m(0, 0) + m(0, -1) + m(0, 0) + m(0, -1)) * 0.25
                  * (kk(0, 0, 0) + kk(0, 0, -1) + kk(-1, 0, 0) + kk(-1, 0, -1)) * rdx)
        mkrdxp = ((X(msfux, j0, j1, i0 + 1, i1 + 1) / X(msfuy, j0, j1, i0 + 1, i1 + 1)) * 0.25 * (m(0, 1) + m(0, 0) + m(0, 1) + m(0, 0)) * 0.25
                  * (kk(0, 0, 1) + kk(0, 0, 0) + kk(-1, 0, 1) + kk(-1, 0, 0)) * rdx)
        mrdx = X(msftx, j0, j1, i0, i1) * X(msfty, j0, j1, i0, i1) * rdx
        mkrdym = ((X(msfvy, j0, j1, i0, i1) / X(msfvx, j0, j1, i0, i1)) * 0.25 * (m(0, 0) + m(-1, 0) + m(0, 0) + m(-1, 0)) * 0.25
                  * (kk(0, 0, 0) + kk(0, -1, 0) + kk(-1, 0, 0) + kk(-1, -1, 0)) * rdy)
        mkrdyp = ((X(msfvy, j0 + 1, j1 + 1, i0, i1) / X(msfvx, j0 + 1, j1 + 1, i0, i1)) * 0.25 * (m(1, 0) + m(0, 0) + m(1, 0) + m(0, 0)) * 0.25
                  * (kk(0, 1, 0) + kk(0, 0, 0) + kk(-1, 1, 0) + kk(-1, 0, 0)) * rdy)
        mrdy = X(msftx, j0, j1, i0, i1) * X(msfty, j0, j1, i0, i1) * rdy
    else:
        i0, i1 = g.ids + 1, g.ide - 2
        j0, j1 = g.jds + 1, g.jde - 2
        k0, k1 = 0, ktf
        m = lambda jj, ii: X(mut, j0 + jj, j1 + jj, i0 + ii, i1 + ii)
        kk = lambda jj, ii: K(k0, k1, j0 + jj, j1 + jj, i0 + ii, i1 + ii)
        mkrdxm = (X(msfux, j0, j1, i0, i1) / X(msfuy, j0, j1, i0, i1)) * 0.5 * (kk(0, 0) + kk(0, -1)) * 0.5 * (m(0, 0) + m(0, -1)) * rdx
        mkrdxp = (X(msfux, j0, j1, i0 + 1, i1 + 1) / X(msfuy, j0, j1, i0 + 1, i1 + 1)) * 0.5 * (kk(0, 1) + kk(0, 0)) * 0.5 * (m(0, 1) + m(0, 0)) * rdx
        mrdx = X(msftx, j0, j1, i0, i1) * X(msfty, j0, j1, i0, i1) * rdx
        mkrdym = (X(msfvy, j0, j1, i0, i1) * X(msfvx_inv, j0, j1, i0, i1)) * 0.5 * (kk(0, 0) + kk(-1, 0)) * 0.5 * (m(0, 0) + m(-1, 0)) * rdy
        mkrdyp = (X(msfvy, j0 + 1, j1 + 1, i0, i1) * X(msfvx_inv, j0 + 1, j1 + 1, i0, i1)) * 0.5 * (kk(1, 0) + kk(0, 0)) * 0.5 * (m(1, 0) + m(0, 0)) * rdy
        mrdy = X(msftx, j0, j1, i0, i1) * X(msfty, j0, j1, i0, i1) * rdy
    _hdiff_core(tend, field, (k0, k1), (j0, j1), (i0, i1), mkrdxm, mkrdxp, mrdx, mkrdym, mkrdyp, mrdy, base)
    return tend


# ------------------------------------------------------------------- advection

def _sgn(x):
    return np.where(x >= 0, 1.0, -1.0).astype(x.dtype)


def flux3(qm2, qm1, q0, qp1, ua):
    """wrf_dynamics.py:1313-1320 (3rd-order upwind-biased face value)."""
    f4 = (7.0 * (q0 + qm1) - (qp1 + qm2)) / 12.0
    return f4 + _sgn(ua) * ((qp1 - qm2) - 3.0 * (q0 - qm1)) / 12.0


def flux5(qm3, qm2, qm1, q0, qp1, qp2, ua):
    """wrf_dynamics.py:1322-1329 (5th-order upwind-biased face value)."""
    f6 = (37.0 * (q0 + qm1) - 8.0 * (qp1 + qm2) + (qp2 + qm3)) / 60.0
    return f6 - _sgn(ua) * ((qp2 - qm3) - 5.0 * (qp1 - qm2) + 10.0 * (q0 - qm1)) / 60.0


def _yflux5(q, k0, k1, f0, f1, i0, i1, vel, sgn):
    s = lambda d: q[k0:k1, f0 + d:f1 + d, i0:i1]
    return vel * flux5(s(-3), s(-2), s(-1), s(0), s(1), s(2), sgn)


def _xflux5(q, k0, k1, j0, j1, f0, f1, vel, sgn):
    s = lambda d: q[k0:k1, j0:j1, f0 + d:f1 + d]
    return vel * flux5(s(-3), s(-2), s(-1), s(0), s(1), s(2), sgn)


def _zflux5(q, f0, f1, j0, j1, i0, i1, vel, sgn):
    s = lambda d: q[f0 + d:f1 + d, j0:j1, i0:i1]
    return vel * flux5(s(-3), s(-2), s(-1), s(0), s(1), s(2), sgn)


def advect_u(g, u, tend, ru, rv, rom, msfux, fzm, fzp, rdzw):
    """wrf_dynamics.py:1112-1307 (horizontal 5th order, vertical 5th order
    interior, lower orders next to each boundary)."""
    ktf = g.nz - 1
    ids, ide, jds, jde = g.ids, g.ide, g.jds, g.jde
    rdx, rdy = g.rdx, g.rdy
    # y flux at v-faces, for u columns i in [ids+1, ide-1)
    i0, i1 = ids + 1, ide - 1
    fq = np.zeros((ktf, g.ny, g.nx), u.dtype)
    vel = np.zeros((g.nz, g.ny, g.nx), u.dtype)
    f0, f1 = jds + 3, jde - 3
    vel[0:ktf, f0:f1, i0:i1] = 0.5 * (rv[0:ktf, f0:f1, i0:i1] + rv[0:ktf, f0:f1, i0 - 1:i1 - 1])
    fq[:, f0:f1, i0:i1] = _yflux5(u, 0, ktf, f0, f1, i0, i1, vel[0:ktf, f0:f1, i0:i1], vel[0:ktf, f0:f1, i0:i1])
    fq[:, jds + 1, i0:i1] = (0.25 * (rv[0:ktf, jds + 1, i0:i1] + rv[0:ktf, jds + 1, i0 - 1:i1 - 1])
                             * (u[0:ktf, jds + 1, i0:i1] + u[0:ktf, jds, i0:i1]))
    vel[0:ktf, jds + 2, i0:i1] = 0.5 * (rv[0:ktf, jds + 2, i0:i1] + rv[0:ktf, jds + 2, i0 - 1:i1 - 1])
    vv = vel[0:ktf, jds + 2, i0:i1]
    fq[:, jds + 2, i0:i1] = vv * flux3(u[0:ktf, jds, i0:i1], u[0:ktf, jds + 1, i0:i1], u[0:ktf, jds + 2, i0:i1], u[0:ktf, jds + 3, i0:i1], vv)
    fq[:, jde - 2, i0:i1] = (0.25 * (rv[0:ktf, jde - 2, i0:i1] + rv[0:ktf, jde - 2, i0 - 1:i1 - 1])
                             * (u[0:ktf, jde - 2, i0:i1] + u[0:ktf, jde - 3, i0:i1]))
    vel[0:ktf, jde - 3, i0:i1] = 0.5 * (rv[0:ktf, jde - 3, i0:i1] + rv[0:ktf, jde - 3, i0 - 1:i1 - 1])
    # the reference takes the upwind sign from row jde-2, where vel was never set (0 -> +1)
    fq[:, jde - 3, i0:i1] = vel[0:ktf, jde - 3, i0:i1] * flux3(u[0:ktf, jde - 5, i0:i1], u[0:ktf, jde - 4, i0:i1], u[0:ktf, jde - 3, i0:i1],
                                                              u[0:ktf, jde - 2, i0:i1], vel[0:ktf, jde - 2, i0:i1])
    j0, j1 = jds + 1, jde - 2
    tend[0:ktf, j0:j1, i0:i1] = tend[0:ktf, j0:j1, i0:i1] - (msfux[None, j0:j1, i0:i1] * rdy) * (fq[:, j0 + 1:j1 + 1, i0:i1] - fq[:, j0:j1, i0:i1])
    # x flux at mass faces
    j0, j1 = jds, jde - 1
    fq = np.zeros((ktf, g.ny, g.nx), u.dtype)
    f0, f1 = ids + 3, ide - 2
    vel[0:ktf, j0:j1, f0:f1] = 0.5 * (ru[0:ktf, j0:j1, f0:f1] + ru[0:ktf, j0:j1, f0 - 1:f1 - 1])
    vv = vel[0:ktf, j0:j1, f0:f1]
    fq[:, j0:j1, f0:f1] = _xflux5(u, 0, ktf, j0, j1, f0, f1, vv, vv)
    ub = np.where(u[0:ktf, j0:j1, ids + 1] < 0.0, u[0:ktf, j0:j1, ids + 1], u[0:ktf, j0:j1, ids])
    fq[:, j0:j1, ids + 1] = 0.25 * (ru[0:ktf, j0:j1, ids + 1] + ru[0:ktf, j0:j1, ids]) * (u[0:ktf, j0:j1, ids + 1] + ub)
    vel[0:ktf, j0:j1, ids + 2] = 0.5 * (ru[0:ktf, j0:j1, ids + 2] + ru[0:ktf, j0:j1, ids + 1])
    vv = vel[0:ktf, j0:j1, ids + 2]
    fq[:, j0:j1, ids + 2] = vv * flux3(u[0:ktf, j0:j1, ids], u[0:ktf, j0:j1, ids + 1], u[0:ktf, j0:j1, ids + 2], u[0:ktf, j0:j1, ids + 3], vv)
    ub = np.where(u[0:ktf, j0:j1, ide - 2] > 0.0, u[0:ktf, j0:j1, ide - 2], u[0:ktf, j0:j1, ide - 1])
    fq[:, j0:j1, ide - 1] = 0.25 * (ru[0:ktf, j0:j1, ide - 1] + ru[0:ktf, j0:j1, ide - 2]) * (u[0:ktf, j0:j1, ide - 2] + ub)
    vel[0:ktf, j0:j1, ide - 2] = 0.5 * (ru[0:ktf, j0:j1, ide - 2] + ru[0:ktf, j0:j1, ide - 3])
    vv = vel[0:ktf, j0:j1, ide - 2]
    fq[:, j0:j1, ide - 2] = vv * flux3(u[0:ktf, j0:j1, ide - 4], u[0:ktf, j0:j1, ide - 3], u[0:ktf, j0:j1, ide - 2], u[0:ktf, j0:j1, ide - 1], vv)
    i0, i1 = ids + 1, ide - 1
    tend[0:ktf, j0:j1, i0:i1] = tend[0:ktf, j0:j1, i0:i1] - (msfux[None, j0:j1, i0:i1] * rdx) * (fq[:, j0:j1, i0 + 1:i1 + 1] - fq[:, j0:j1, i0:i1])
    # z flux at w levels
    vf = np.zeros((g.nz, g.ny, g.nx), u.dtype)
    avg = lambda k: 0.5 * (rom[k, j0:j1, i0 - 1:i1 - 1] + rom[k, j0:j1, i0:i1]) if isinstance(k, int) else 0.5 * (rom[k, j0:j1, i0 - 1:i1 - 1] + rom[k, j0:j1, i0:i1])
    kf = slice(3, ktf - 2)
    vel[kf, j0:j1, i0:i1] = avg(kf)
    vv = vel[kf, j0:j1, i0:i1]
    vf[kf, j0:j1, i0:i1] = _zflux5(u, 3, ktf - 2, j0, j1, i0, i1, vv, -vv)
    vf[1, j0:j1, i0:i1] = (0.5 * (rom[1, j0:j1, i0:i1] + rom[1, j0:j1, i0 - 1:i1 - 1])
                           * (fzm[1] * u[1, j0:j1, i0:i1] + fzp[1] * u[0, j0:j1, i0:i1]))
    vv = 0.5 * (rom[2, j0:j1, i0:i1] + rom[2, j0:j1, i0 - 1:i1 - 1])
    vf[2, j0:j1, i0:i1] = vv * flux3(u[0, j0:j1, i0:i1], u[1, j0:j1, i0:i1], u[2, j0:j1, i0:i1], u[3, j0:j1, i0:i1], -vv)
    k = ktf - 2
    vv = 0.5 * (rom[k, j0:j1, i0:i1] + rom[k, j0:j1, i0 - 1:i1 - 1])
    vf[k, j0:j1, i0:i1] = vv * flux3(u[k - 2, j0:j1, i0:i1], u[k - 1, j0:j1, i0:i1], u[k, j0:j1, i0:i1], u[k + 1, j0:j1, i0:i1], -vv)
    k = ktf - 1
    vf[k, j0:j1, i0:i1] = (0.5 * (rom[k, j0:j1, i0:i1] + rom[k, j0:j1, i0 - 1:i1 - 1])
                           * (fzm[k] * u[k, j0:j1, i0:i1] + fzp[k] * u[k - 1, j0:j1, i0:i1]))
    tend[0:ktf, j0:j1, i0:i1] = tend[0:ktf, j0:j1, i0:i1] - rdzw[0:ktf, None, None] * (vf[1:ktf + 1, j0:j1, i0:i1] - vf[0:ktf, j0:j1, i0:i1])
    del avg
    return tend


def advect_v(g, v, tend, ru, rv, rom, msfvx, msfvy, fzm, fzp, rdzw):
    """wrf_dynamics.py:1332-1532"""
    ktf = g.nz - 1
    ids, ide, jds, jde = g.ids, g.ide, g.jds, g.jde
    rdx, rdy = g.rdx, g.rdy
    i0, i1 = ids, ide - 1
    fq = np.zeros((ktf, g.ny, g.nx), v.dtype)
    f0, f1 = jds + 3, jde - 2
    vv = 0.5 * (rv[0:ktf, f0:f1, i0:i1] + rv[0:ktf, f0 - 1:f1 - 1, i0:i1])
    fq[:, f0:f1, i0:i1] = _yflux5(v, 0, ktf, f0, f1, i0, i1, vv, vv)
    vb = np.where(v[0:ktf, jds + 1, i0:i1] < 0.0, v[0:ktf, jds + 1, i0:i1], v[0:ktf, jds, i0:i1])
    fq[:, jds + 1, i0:i1] = 0.25 * (rv[0:ktf, jds + 1, i0:i1] + rv[0:ktf, jds, i0:i1]) * (v[0:ktf, jds + 1, i0:i1] + vb)
    vv = 0.5 * (rv[0:ktf, jds + 2, i0:i1] + rv[0:ktf, jds + 1, i0:i1])
    fq[:, jds + 2, i0:i1] = vv * flux3(v[0:ktf, jds, i0:i1], v[0:ktf, jds + 1, i0:i1], v[0:ktf, jds + 2, i0:i1], v[0:ktf, jds + 3, i0:i1], vv)
    vb = np.where(v[0:ktf, jde - 2, i0:i1] > 0.0, v[0:ktf, jde - 2, i0:i1], v[0:ktf, jde - 1, i0:i1])
    fq[:, jde - 1, i0:i1] = 0.25 * (rv[0:ktf, jde - 1, i0:i1] + rv[0:ktf, jde - 2, i0:i1]) * (v[0:ktf, jde - 2, i0:i1] + vb)
    vv = 0.5 * (rv[0:ktf, jde - 2, i0:i1] + rv[0:ktf, jde - 3, i0:i1])
    fq[:, jde - 2, i0:i1] = vv * flux3(v[0:ktf, jde - 4, i0:i1], v[0:ktf, jde - 3, i0:i1], v[0:ktf, jde - 2, i0:i1], v[0:ktf, jde - 1, i0:i1], vv)
    j0, j1 = jds + 1, jde - 1
    tend[0:ktf, j0:j1, i0:i1] = tend[0:ktf, j0:j1, i0:i1] - (msfvy[None, j0:j1, i0:i1] * rdy) * (fq[:, j0 + 1:j1 + 1, i0:i1] - fq[:, j0:j1, i0:i1])
    # x
    j0, j1 = jds + 1, jde - 1
    fq = np.zeros((ktf, g.ny, g.nx), v.dtype)
    f0, f1 = ids + 3, ide - 3
    vv = 0.5 * (ru[0:ktf, j0:j1, f0:f1] + ru[0:ktf, j0 - 1:j1 - 1, f0:f1])
    fq[:, j0:j1, f0:f1] = _xflux5(v, 0, ktf, j0, j1, f0, f1, vv, vv)
    fq[:, j0:j1, ids + 1] = (0.25 * (ru[0:ktf, j0:j1, ids + 1] + ru[0:ktf, j0 - 1:j1 - 1, ids + 1])
                             * (v[0:ktf, j0:j1, ids + 1] + v[0:ktf, j0:j1, ids]))
    vv = 0.5 * (ru[0:ktf, j0:j1, ids + 2] + ru[0:ktf, j0 - 1:j1 - 1, ids + 2])
    fq[:, j0:j1, ids + 2] = vv * flux3(v[0:ktf, j0:j1, ids], v[0:ktf, j0:j1, ids + 1], v[0:ktf, j0:j1, ids + 2], v[0:ktf, j0:j1, ids + 3], vv)
    ie = ide - 2
    fq[:, j0:j1, ide - 2] = (0.25 * (ru[0:ktf, j0:j1, ie] + ru[0:ktf, j0 - 1:j1 - 1, ie])
                             * (v[0:ktf, j0:j1, ie] + v[0:ktf, j0:j1, ie - 1]))
    vv = 0.5 * (ru[0:ktf, j0:j1, ide - 3] + ru[0:ktf, j0 - 1:j1 - 1, ide - 3])
    fq[:, j0:j1, ide - 3] = vv * flux3(v[0:ktf, j0:j1, ide - 5], v[0:ktf, j0:j1, ide - 4], v[0:ktf, j0:j1, ide - 3], v[0:ktf, j0:j1, ide - 2], vv)
    i0, i1 = ids + 1, ide - 2
    tend[0:ktf, j0:j1, i0:i1] = tend[0:ktf, j0:j1, i0:i1] - (msfvy[None, j0:j1, i0:i1] * rdx) * (fq[:, j0:j1, i0 + 1:i1 + 1] - fq[:, j0:j1, i0:i1])
    # z
    i0, i1 = ids, ide - 1
    vf = np.zeros((g.nz, g.ny, g.nx), v.dtype)
    avg = lambda k0, k1: 0.5 * (rom[k0:k1, j0:j1, i0:i1] + rom[k0:k1, j0 - 1:j1 - 1, i0:i1])
    vv = avg(3, ktf - 2)
    vf[3:ktf - 2, j0:j1, i0:i1] = _zflux5(v, 3, ktf - 2, j0, j1, i0, i1, vv, -vv)
    vf[1, j0:j1, i0:i1] = avg(1, 2)[0] * (fzm[1] * v[1, j0:j1, i0:i1] + fzp[1] * v[0, j0:j1, i0:i1])
    vv = avg(2, 3)[0]
    vf[2, j0:j1, i0:i1] = vv * flux3(v[0, j0:j1, i0:i1], v[1, j0:j1, i0:i1], v[2, j0:j1, i0:i1], v[3, j0:j1, i0:i1], -vv)
    k = ktf - 2
    vv = avg(k, k + 1)[0]
    # the reference uses +vel (not -vel) for the sign at ktf-2
    vf[k, j0:j1, i0:i1] = vv * flux3(v[k - 2, j0:j1, i0:i1], v[k - 1, j0:j1, i0:i1], v[k, j0:j1, i0:i1], v[k + 1, j0:j1, i0:i1], vv)
    k = ktf - 1
    vf[k, j0:j1, i0:i1] = avg(k, k + 1)[0] * (fzm[k] * v[k, j0:j1, i0:i1] + fzp[k] * v[k - 1, j0:j1, i0:i1])
    tend[0:ktf, j0:j1, i0:i1] = tend[0:ktf, j0:j1, i0:i1] - ((msfvy[None, j0:j1, i0:i1] / msfvx[None, j0:j1, i0:i1])
                                                             * rdzw[0:ktf, None, None]) * (vf[1:ktf + 1, j0:j1, i0:i1] - vf[0:ktf, j0:j1, i0:i1])
    return tend


def advect_w(g, w, tend, ru, rv, rom, msftx, fzm, fzp, rdzu):
    """wrf_dynamics.py:1535-1822"""
    ktf = g.nz - 1
    ids, ide, jds, jde = g.ids, g.ide, g.jds, g.jde
    rdx, rdy = g.rdx, g.rdy
    fzmc = lambda k0, k1: fzm[k0:k1, None, None]
    fzpc = lambda k0, k1: fzp[k0:k1, None, None]

    def vel_y(j, i0, i1):  # interior levels [1, ktf) then level ktf (top extrapolation)
        lo = fzm[1:ktf, None] * rv[1:ktf, j, i0:i1] + fzp[1:ktf, None] * rv[0:ktf - 1, j, i0:i1]
        top = (2.0 - fzm[ktf - 1]) * rv[ktf - 1, j, i0:i1] - fzp[ktf - 1] * rv[ktf - 2, j, i0:i1]
        return lo, top

    i0, i1 = ids, ide - 1
    fq = np.zeros((g.nz, g.ny, g.nx), w.dtype)
    f0, f1 = jds + 3, jde - 3
    sl = lambda k0, k1, d: w[k0:k1, f0 + d:f1 + d, i0:i1]
    vlo = fzmc(1, ktf) * rv[1:ktf, f0:f1, i0:i1] + fzpc(1, ktf) * rv[0:ktf - 1, f0:f1, i0:i1]
    fq[1:ktf, f0:f1, i0:i1] = vlo * flux5(sl(1, ktf, -3), sl(1, ktf, -2), sl(1, ktf, -1), sl(1, ktf, 0), sl(1, ktf, 1), sl(1, ktf, 2), vlo)
    vt = (2.0 - fzm[ktf - 1]) * rv[ktf - 1, f0:f1, i0:i1] - fzp[ktf - 1] * rv[ktf - 2, f0:f1, i0:i1]
    fq[ktf, f0:f1, i0:i1] = vt * flux5(sl(ktf, ktf + 1, -3)[0], sl(ktf, ktf + 1, -2)[0], sl(ktf, ktf + 1, -1)[0],
                                       sl(ktf, ktf + 1, 0)[0], sl(ktf, ktf + 1, 1)[0], sl(ktf, ktf + 1, 2)[0], vt)
    for jf, jlo in ((jds + 1, jds), (jde - 2, jde - 3)):
        lo, top = vel_y(jf, i0, i1)
        fq[1:ktf, jf, i0:i1] = 0.5 * lo * (w[1:ktf, jf, i0:i1] + w[1:ktf, jlo, i0:i1])
        fq[ktf, jf, i0:i1] = 0.5 * top * (w[ktf, jf, i0:i1] + w[ktf, jlo, i0:i1])
    for jf, (a, b, c, d) in ((jds + 2, (jds, jds + 1, jds + 2, jds + 3)), (jde - 3, (jde - 5, jde - 4, jde - 3, jde - 2))):
        lo, top = vel_y(jf, i0, i1)
        fq[1:ktf, jf, i0:i1] = lo * flux3(w[1:ktf, a, i0:i1], w[1:ktf, b, i0:i1], w[1:ktf, c, i0:i1], w[1:ktf, d, i0:i1], lo)
        fq[ktf, jf, i0:i1] = top * flux3(w[ktf, a, i0:i1], w[ktf, b, i0:i1], w[ktf, c, i0:i1], w[ktf, d, i0:i1], top)
    j0, j1 = jds + 1, jde - 2
    tend[1:ktf + 1, j0:j1, i0:i1] = tend[1:ktf + 1, j0:j1, i0:i1] - (msftx[None, j0:j1, i0:i1] * rdy) * (fq[1:ktf + 1, j0 + 1:j1 + 1, i0:i1] - fq[1:ktf + 1, j0:j1, i0:i1])
    # x
    j0, j1 = jds, jde - 1
    fq = np.zeros((g.nz, g.ny, g.nx), w.dtype)
    f0, f1 = ids + 3, ide - 3

    def vel_x(i):
        lo = fzm[1:ktf, None] * ru[1:ktf, j0:j1, i] + fzp[1:ktf, None] * ru[0:ktf - 1, j0:j1, i]
        top = (2.0 - fzm[ktf - 1]) * ru[ktf - 1, j0:j1, i] - fzp[ktf - 1] * ru[ktf - 2, j0:j1, i]
        return lo, top

    sx = lambda k0, k1, d: w[k0:k1, j0:j1, f0 + d:f1 + d]
    vlo = fzmc(1, ktf) * ru[1:ktf, j0:j1, f0:f1] + fzpc(1, ktf) * ru[0:ktf - 1, j0:j1, f0:f1]
    fq[1:ktf, j0:j1, f0:f1] = vlo * flux5(sx(1, ktf, -3), sx(1, ktf, -2), sx(1, ktf, -1), sx(1, ktf, 0), sx(1, ktf, 1), sx(1, ktf, 2), vlo)
    vt = (2.0 - fzm[ktf - 1]) * ru[ktf - 1, j0:j1, f0:f1] - fzp[ktf - 1] * ru[ktf - 2, j0:j1, f0:f1]
    fq[ktf, j0:j1, f0:f1] = vt * flux5(sx(ktf, ktf + 1, -3)[0], sx(ktf, ktf + 1, -2)[0], sx(ktf, ktf + 1, -1)[0],
                                       sx(ktf, ktf + 1, 0)[0], sx(ktf, ktf + 1, 1)[0], sx(ktf, ktf + 1, 2)[0], vt)
    for iface, ilo in ((ids + 1, ids), (ide - 2, ide - 3)):
        lo, top = vel_x(iface)
        fq[1:ktf, j0:j1, iface] = 0.5 * lo * (w[1:ktf, j0:j1, iface] + w[1:ktf, j0:j1, ilo])
        fq[ktf, j0:j1, iface] = 0.5 * top * (w[ktf, j0:j1, iface] + w[ktf, j0:j1, ilo])
    for iface, (a, b, c, d) in ((ids + 2, (ids, ids + 1, ids + 2, ids + 3)), (ide - 3, (ide - 5, ide - 4, ide - 3, ide - 2))):
        lo, top = vel_x(iface)
        fq[1:ktf, j0:j1, iface] = lo * flux3(w[1:ktf, j0:j1, a], w[1:ktf, j0:j1, b], w[1:ktf, j0:j1, c], w[1:ktf, j0:j1, d], lo)
        fq[ktf, j0:j1, iface] = top * flux3(w[ktf, j0:j1, a], w[ktf, j0:j1, b], w[ktf, j0:j1, c], w[ktf, j0:j1, d], top)
    i0, i1 = ids + 1, ide - 2
    tend[1:ktf + 1, j0:j1, i0:i1] = tend[1:ktf + 1, j0:j1, i0:i1] - (msftx[None, j0:j1, i0:i1] * rdx) * (fq[1:ktf + 1, j0:j1, i0 + 1:i1 + 1] - fq[1:ktf + 1, j0:j1, i0:i1])
    # z
    i0, i1 = ids, ide - 1
    j0, j1 = jds, jde - 1
    vf = np.zeros((g.nz, g.ny, g.nx), w.dtype)
    vv = 0.5 * (rom[3:ktf - 1, j0:j1, i0:i1] + rom[2:ktf - 2, j0:j1, i0:i1])
    vf[3:ktf - 1, j0:j1, i0:i1] = _zflux5(w, 3, ktf - 1, j0, j1, i0, i1, vv, -vv)
    vf[1, j0:j1, i0:i1] = 0.25 * (rom[1, j0:j1, i0:i1] + rom[0, j0:j1, i0:i1]) * (w[1, j0:j1, i0:i1] + w[0, j0:j1, i0:i1])
    vv = 0.5 * (rom[2, j0:j1, i0:i1] + rom[1, j0:j1, i0:i1])
    vf[2, j0:j1, i0:i1] = vv * flux3(w[0, j0:j1, i0:i1], w[1, j0:j1, i0:i1], w[2, j0:j1, i0:i1], w[3, j0:j1, i0:i1], -vv)
    k = ktf - 1
    vv = 0.5 * (rom[k, j0:j1, i0:i1] + rom[k - 1, j0:j1, i0:i1])
    # +vel sign at ktf-1 (reference)
    vf[k, j0:j1, i0:i1] = vv * flux3(w[k - 2, j0:j1, i0:i1], w[k - 1, j0:j1, i0:i1], w[k, j0:j1, i0:i1], w[k + 1, j0:j1, i0:i1], vv)
    vf[ktf, j0:j1, i0:i1] = 0.25 * (rom[ktf, j0:j1, i0:i1] + rom[ktf - 1, j0:j1, i0:i1]) * (w[ktf, j0:j1, i0:i1] + w[ktf - 1, j0:j1, i0:i1])
    tend[1:ktf, j0:j1, i0:i1] = tend[1:ktf, j0:j1, i0:i1] - rdzu[1:ktf, None, None] * (vf[2:ktf + 1, j0:j1, i0:i1] - vf[1:ktf, j0:j1, i0:i1])
    tend[ktf, j0:j1, i0:i1] = tend[ktf, j0:j1, i0:i1] + 2.0 * rdzu[ktf - 1] * vf[ktf, j0:j1, i0:i1]
    return tend


def advect_scalar(g, field, tend, ru, rv, rom, msftx, fzm, fzp, rdzw):
    """wrf_dynamics.py:1841-2028 (mass-point scalar; fluxes are the coupled
    velocities themselves)."""
    ktf = g.nz - 1
    ids, ide, jds, jde = g.ids, g.ide, g.jds, g.jde
    rdx, rdy = g.rdx, g.rdy
    f = field
    i0, i1 = ids, ide - 1
    fq = np.zeros((ktf, g.ny, g.nx), f.dtype)
    f0, f1 = jds + 3, jde - 3
    vv = rv[0:ktf, f0:f1, i0:i1]
    fq[:, f0:f1, i0:i1] = _yflux5(f, 0, ktf, f0, f1, i0, i1, vv, vv)
    fq[:, jds + 1, i0:i1] = 0.5 * rv[0:ktf, jds + 1, i0:i1] * (f[0:ktf, jds + 1, i0:i1] + f[0:ktf, jds, i0:i1])
    vv = rv[0:ktf, jds + 2, i0:i1]
    fq[:, jds + 2, i0:i1] = vv * flux3(f[0:ktf, jds, i0:i1], f[0:ktf, jds + 1, i0:i1], f[0:ktf, jds + 2, i0:i1], f[0:ktf, jds + 3, i0:i1], vv)
    fq[:, jde - 2, i0:i1] = 0.5 * rv[0:ktf, jde - 2, i0:i1] * (f[0:ktf, jde - 2, i0:i1] + f[0:ktf, jde - 3, i0:i1])
    vv = rv[0:ktf, jde - 3, i0:i1]
    fq[:, jde - 3, i0:i1] = vv * flux3(f[0:ktf, jde - 5, i0:i1], f[0:ktf, jde - 4, i0:i1], f[0:ktf, jde - 3, i0:i1], f[0:ktf, jde - 2, i0:i1], vv)
    j0, j1 = jds + 1, jde - 2
    tend[0:ktf, j0:j1, i0:i1] = tend[0:ktf, j0:j1, i0:i1] - (msftx[None, j0:j1, i0:i1] * rdy) * (fq[:, j0 + 1:j1 + 1, i0:i1] - fq[:, j0:j1, i0:i1])
    # x
    j0, j1 = jds, jde - 1
    fq = np.zeros((ktf, g.ny, g.nx), f.dtype)
    f0, f1 = ids + 3, ide - 3
    vv = ru[0:ktf, j0:j1, f0:f1]
    fq[:, j0:j1, f0:f1] = _xflux5(f, 0, ktf, j0, j1, f0, f1, vv, vv)
    fq[:, j0:j1, ids + 1] = 0.5 * ru[0:ktf, j0:j1, ids + 1] * (f[0:ktf, j0:j1, ids + 1] + f[0:ktf, j0:j1, ids])
    vv = ru[0:ktf, j0:j1, ids + 2]
    fq[:, j0:j1, ids + 2] = vv * flux3(f[0:ktf, j0:j1, ids], f[0:ktf, j0:j1, ids + 1], f[0:ktf, j0:j1, ids + 2], f[0:ktf, j0:j1, ids + 3], vv)
    fq[:, j0:j1, ide - 2] = 0.5 * ru[0:ktf, j0:j1, ide - 2] * (f[0:ktf, j0:j1, ide - 2] + f[0:ktf, j0:j1, ide - 3])
    # the reference takes the upwind sign at ide-3 from ru at ide-2
    fq[:, j0:j1, ide - 3] = ru[0:ktf, j0:j1, ide - 3] * flux3(f[0:ktf, j0:j1, ide - 5], f[0:ktf, j0:j1, ide - 4], f[0:ktf, j0:j1, ide - 3],
                                                              f[0:ktf, j0:j1, ide - 2], ru[0:ktf, j0:j1, ide - 2])
    i0, i1 = ids + 1, ide - 2
    tend[0:ktf, j0:j1, i0:i1] = tend[0:ktf, j0:j1, i0:i1] - (msftx[None, j0:j1, i0:i1] * rdx) * (fq[:, j0:j1, i0 + 1:i1 + 1] - fq[:, j0:j1, i0:i1])
    # z
    i0, i1 = ids, ide - 1
    vf = np.zeros((g.nz, g.ny, g.nx), f.dtype)
    vv = rom[3:ktf - 2, j0:j1, i0:i1]
    vf[3:ktf - 2, j0:j1, i0:i1] = _zflux5(f, 3, ktf - 2, j0, j1, i0, i1, vv, -vv)
    vf[1, j0:j1, i0:i1] = rom[1, j0:j1, i0:i1] * (fzm[1] * f[1, j0:j1, i0:i1] + fzp[1] * f[0, j0:j1, i0:i1])
    vv = rom[2, j0:j1, i0:i1]
    vf[2, j0:j1, i0:i1] = vv * flux3(f[0, j0:j1, i0:i1], f[1, j0:j1, i0:i1], f[2, j0:j1, i0:i1], f[3, j0:j1, i0:i1], -vv)
    k = ktf - 2
    vv = rom[k, j0:j1, i0:i1]
    vf[k, j0:j1, i0:i1] = vv * flux3(f[k - 2, j0:j1, i0:i1], f[k - 1, j0:j1, i0:i1], f[k, j0:j1, i0:i1], f[k + 1, j0:j1, i0:i1], -vv)
    k = ktf - 1
    vf[k, j0:j1, i0:i1] = rom[k, j0:j1, i0:i1] * (fzm[k] * f[k, j0:j1, i0:i1] + fzp[k] * f[k - 1, j0:j1, i0:i1])
    tend[0:ktf, j0:j1, i0:i1] = tend[0:ktf, j0:j1, i0:i1] - rdzw[0:ktf, None, None] * (vf[1:ktf + 1, j0:j1, i0:i1] - vf[0:ktf, j0:j1, i0:i1])
    return tend


# ---------------------------------------------- geopotential, PGF, buoyancy, etc.

def rhs_ph(g, ph_tend, u, v, ww, ph, phb, w, mut, muuf, muvf, fnm, fnp, rdnw, cfn, cfn1,
           msfux, msfvy, msfty):
    """wrf_dynamics.py:2031-2297"""
    nz = g.nz
    js, jt, i0, it = g.jds, g.jde - 1, g.ids, g.ide - 1
    rdx, rdy = g.rdx, g.rdy
    wdwn = np.zeros((nz, g.ny, g.nx), ph.dtype)
    wdwn[1:nz, js:jt, i0:it] = (0.5 * (ww[1:nz, js:jt, i0:it] + ww[0:nz - 1, js:jt, i0:it]) * rdnw[0:nz - 1, None, None]
                                * (ph[1:nz, js:jt, i0:it] - ph[0:nz - 1, js:jt, i0:it] + phb[1:nz, js:jt, i0:it] - phb[0:nz - 1, js:jt, i0:it]))
    ph_tend[1:nz - 1, js:jt, i0:it] = ph_tend[1:nz - 1, js:jt, i0:it] - (fnm[1:nz - 1, None, None] * wdwn[2:nz, js:jt, i0:it]
                                                                          + fnp[1:nz - 1, None, None] * wdwn[1:nz - 1, js:jt, i0:it])
    ph_tend[nz - 1, js:jt, i0:it] = 0.0
    ph_tend[1:nz, js:jt, i0:it] = ph_tend[1:nz, js:jt, i0:it] + mut[None, js:jt, i0:it] * G * w[1:nz, js:jt, i0:it] / msfty[None, js:jt, i0:it]

    K = slice(1, nz - 1)
    KT = nz - 1

    def d6(k, j0, j1, i0_, i1_, axis):
        """45/9/1 centred differences of ph then phb, summed in the reference's order."""
        if axis == "y":
            s = lambda a, d: a[k, j0 + d:j1 + d, i0_:i1_]
        else:
            s = lambda a, d: a[k, j0:j1, i0_ + d:i1_ + d]
        return (45.0 * (s(ph, 1) - s(ph, -1)) - 9.0 * (s(ph, 2) - s(ph, -2)) + (s(ph, 3) - s(ph, -3))
                + 45.0 * (s(phb, 1) - s(phb, -1)) - 9.0 * (s(phb, 2) - s(phb, -2)) + (s(phb, 3) - s(phb, -3)))

    def d4(k, j0, j1, i0_, i1_, axis):
        if axis == "y":
            s = lambda a, d: a[k, j0 + d:j1 + d, i0_:i1_]
        else:
            s = lambda a, d: a[k, j0:j1, i0_ + d:i1_ + d]
        return (8.0 * (s(ph, 1) - s(ph, -1)) - (s(ph, 2) - s(ph, -2))
                + 8.0 * (s(phb, 1) - s(phb, -1)) - (s(phb, 2) - s(phb, -2)))

    # y direction
    def yflux(j0, j1, lev):
        if lev == "in":
            return lambda jj: muvf[None, j0 + jj:j1 + jj, i0:it] * (v[1:nz - 1, j0 + jj:j1 + jj, i0:it] + v[0:nz - 2, j0 + jj:j1 + jj, i0:it]) * msfvy[None, j0 + jj:j1 + jj, i0:it]
        return lambda jj: muvf[j0 + jj:j1 + jj, i0:it] * (cfn * v[nz - 2, j0 + jj:j1 + jj, i0:it] + cfn1 * v[nz - 3, j0 + jj:j1 + jj, i0:it]) * msfvy[j0 + jj:j1 + jj, i0:it]

    j0, j1 = g.jds + 3, g.jde - 4
    fl = yflux(j0, j1, "in")
    ph_tend[K, j0:j1, i0:it] = ph_tend[K, j0:j1, i0:it] - (0.25 * rdy / msfty[None, j0:j1, i0:it]) * ((fl(1) + fl(0)) * (1.0 / 60.0)
                                                                                                    * d6(K, j0, j1, i0, it, 'y'))
    fl = yflux(j0, j1, "top")
    ph_tend[KT, j0:j1, i0:it] = ph_tend[KT, j0:j1, i0:it] - (0.5 * rdy / msfty[j0:j1, i0:it]) * ((fl(1) + fl(0)) * (1.0 / 60.0)
                                                                                              * d6(KT, j0, j1, i0, it, 'y'))
    for jj in (g.jds + 2, g.jde - 4):
        fl = yflux(jj, jj + 1, "in")
        ph_tend[K, jj:jj + 1, i0:it] = ph_tend[K, jj:jj + 1, i0:it] - (0.25 * rdy / msfty[None, jj:jj + 1, i0:it]) * ((fl(1) + fl(0)) * (1.0 / 12.0)
                                                                                                                   * d4(K, jj, jj + 1, i0, it, 'y'))
        fl = yflux(jj, jj + 1, "top")
        ph_tend[KT, jj:jj + 1, i0:it] = ph_tend[KT, jj:jj + 1, i0:it] - (0.5 * rdy / msfty[jj:jj + 1, i0:it]) * ((fl(1) + fl(0)) * (1.0 / 12.0)
                                                                                                             * d4(KT, jj, jj + 1, i0, it, 'y'))
    for jj in (g.jds + 1, g.jde - 3):
        fl = yflux(jj, jj + 1, "in")
        dp = lambda d: (phb[K, jj + d:jj + d + 1, i0:it] - phb[K, jj + d - 1:jj + d, i0:it] + ph[K, jj + d:jj + d + 1, i0:it] - ph[K, jj + d - 1:jj + d, i0:it])
        ph_tend[K, jj:jj + 1, i0:it] = ph_tend[K, jj:jj + 1, i0:it] - (0.25 * rdy / msfty[None, jj:jj + 1, i0:it]) * (fl(1) * dp(1) + fl(0) * dp(0))
        fl = yflux(jj, jj + 1, "top")
        dpt = lambda d: (phb[KT, jj + d:jj + d + 1, i0:it] - phb[KT, jj + d - 1:jj + d, i0:it] + ph[KT, jj + d:jj + d + 1, i0:it] - ph[KT, jj + d - 1:jj + d, i0:it])
        ph_tend[KT, jj:jj + 1, i0:it] = ph_tend[KT, jj:jj + 1, i0:it] - (0.5 * rdy / msfty[jj:jj + 1, i0:it]) * (fl(1) * dpt(1) + fl(0) * dpt(0))

    # x direction (no 4th-order columns: only 6th-order interior and 2nd-order at ids+1, ide-3)
    jt0, jt1 = g.jds, g.jde - 1

    def xflux(i0_, i1_, lev):
        if lev == "in":
            return lambda ii: muuf[None, jt0:jt1, i0_ + ii:i1_ + ii] * (u[1:nz - 1, jt0:jt1, i0_ + ii:i1_ + ii] + u[0:nz - 2, jt0:jt1, i0_ + ii:i1_ + ii]) * msfux[None, jt0:jt1, i0_ + ii:i1_ + ii]
        return lambda ii: muuf[jt0:jt1, i0_ + ii:i1_ + ii] * (cfn * u[nz - 2, jt0:jt1, i0_ + ii:i1_ + ii] + cfn1 * u[nz - 3, jt0:jt1, i0_ + ii:i1_ + ii]) * msfux[jt0:jt1, i0_ + ii:i1_ + ii]

    a0, a1 = g.ids + 3, g.ide - 4
    fl = xflux(a0, a1, "in")
    ph_tend[K, jt0:jt1, a0:a1] = ph_tend[K, jt0:jt1, a0:a1] - (0.25 * rdx / msfty[None, jt0:jt1, a0:a1]) * ((fl(1) + fl(0)) * (1.0 / 60.0)
                                                                                                          * d6(K, jt0, jt1, a0, a1, 'x'))
    fl = xflux(a0, a1, "top")
    ph_tend[KT, jt0:jt1, a0:a1] = ph_tend[KT, jt0:jt1, a0:a1] - (0.5 * rdx / msfty[jt0:jt1, a0:a1]) * ((fl(1) + fl(0)) * (1.0 / 60.0)
                                                                                                    * d6(KT, jt0, jt1, a0, a1, 'x'))
    for ii in (g.ids + 1, g.ide - 3):
        fl = xflux(ii, ii + 1, "in")
        dp = lambda d: (phb[K, jt0:jt1, ii + d:ii + d + 1] - phb[K, jt0:jt1, ii + d - 1:ii + d] + ph[K, jt0:jt1, ii + d:ii + d + 1] - ph[K, jt0:jt1, ii + d - 1:ii + d])
        ph_tend[K, jt0:jt1, ii:ii + 1] = ph_tend[K, jt0:jt1, ii:ii + 1] - (0.25 * rdx / msfty[None, jt0:jt1, ii:ii + 1]) * (fl(1) * dp(1) + fl(0) * dp(0))
        fl = xflux(ii, ii + 1, "top")
        dpt = lambda d: (phb[KT, jt0:jt1, ii + d:ii + d + 1] - phb[KT, jt0:jt1, ii + d - 1:ii + d] + ph[KT, jt0:jt1, ii + d:ii + d + 1] - ph[KT, jt0:jt1, ii + d - 1:ii + d])
        ph_tend[KT, jt0:jt1, ii:ii + 1] = ph_tend[KT, jt0:jt1, ii:ii + 1] - (0.5 * rdx / msfty[jt0:jt1, ii:ii + 1]) * (fl(1) * dpt(1) + fl(0) * dpt(0))
    return ph_tend


def _dpn(p, nz, fnm, fnp, cf1, cf2, cf3, a, b):
    """Pressure interpolated to w levels between two horizontal neighbours
    (wrf_dynamics.py:2342-2351, 3470-3477): ``a``/``b`` are (j, i) slices."""
    ja, ia = a
    jb, ib = b
    ktf = nz - 1
    shp = p[0, ja, ia].shape
    dpn = np.zeros((nz,) + shp, p.dtype)
    dpn[0] = 0.5 * (cf1 * (p[0, jb, ib] + p[0, ja, ia]) + cf2 * (p[1, jb, ib] + p[1, ja, ia]) + cf3 * (p[2, jb, ib] + p[2, ja, ia]))
    dpn[nz - 1] = 0.0
    dpn[1:ktf] = 0.5 * (fnm[1:ktf, None, None] * (p[1:ktf, jb, ib] + p[1:ktf, ja, ia])
                        + fnp[1:ktf, None, None] * (p[0:ktf - 1, jb, ib] + p[0:ktf - 1, ja, ia]))
    return dpn


def horizontal_pressure_gradient(g, ru_tend, rv_tend, ph, alt, p, pb, al, php, cqu, cqv, muu, muv, mu,
                                 fnm, fnp, rdnw, cf1, cf2, cf3, msfux, msfuy, msfvx, msfvy):
    """wrf_dynamics.py:2300-2421"""
    nz = g.nz
    ktf = nz - 1
    rdx, rdy = g.rdx, g.rdy
    # y
    i0, i1 = g.ids, g.ide - 1
    j0, j1 = g.jds + 1, g.jde - 1
    A = (slice(j0, j1), slice(i0, i1))
    Bm = (slice(j0 - 1, j1 - 1), slice(i0, i1))
    dpn = _dpn(p, nz, fnm, fnp, cf1, cf2, cf3, A, Bm)
    sl = lambda a, kk, jj: a[kk, j0 + jj:j1 + jj, i0:i1]
    K, K1 = slice(0, ktf), slice(1, ktf + 1)
    dpy = ((msfvy[None, j0:j1, i0:i1] / msfvx[None, j0:j1, i0:i1]) * 0.5 * rdy * muv[None, j0:j1, i0:i1]
           * ((sl(ph, K1, 0) - sl(ph, K1, -1) + sl(ph, K, 0) - sl(ph, K, -1))
              + (sl(alt, K, 0) + sl(alt, K, -1)) * (sl(p, K, 0) - sl(p, K, -1))
              + (sl(al, K, 0) + sl(al, K, -1)) * (sl(pb, K, 0) - sl(pb, K, -1))))
    dpy = dpy + ((msfvy[None, j0:j1, i0:i1] / msfvx[None, j0:j1, i0:i1]) * rdy * (sl(php, K, 0) - sl(php, K, -1))
                 * (rdnw[0:ktf, None, None] * (dpn[1:ktf + 1] - dpn[0:ktf]) - 0.5 * (mu[None, j0 - 1:j1 - 1, i0:i1] + mu[None, j0:j1, i0:i1])))
    rv_tend[K, j0:j1, i0:i1] = rv_tend[K, j0:j1, i0:i1] - cqv[K, j0:j1, i0:i1] * dpy
    # x
    i0, i1 = g.ids + 1, g.ide - 1
    j0, j1 = g.jds, g.jde - 1
    A = (slice(j0, j1), slice(i0, i1))
    Bm = (slice(j0, j1), slice(i0 - 1, i1 - 1))
    dpn = _dpn(p, nz, fnm, fnp, cf1, cf2, cf3, A, Bm)
    sx = lambda a, kk, ii: a[kk, j0:j1, i0 + ii:i1 + ii]
    dpx = ((msfux[None, j0:j1, i0:i1] / msfuy[None, j0:j1, i0:i1]) * 0.5 * rdx * muu[None, j0:j1, i0:i1]
           * ((sx(ph, K1, 0) - sx(ph, K1, -1) + sx(ph, K, 0) - sx(ph, K, -1))
              + (sx(alt, K, 0) + sx(alt, K, -1)) * (sx(p, K, 0) - sx(p, K, -1))
              + (sx(al, K, 0) + sx(al, K, -1)) * (sx(pb, K, 0) - sx(pb, K, -1))))
    dpx = dpx + ((msfux[None, j0:j1, i0:i1] / msfuy[None, j0:j1, i0:i1]) * rdx * (sx(php, K, 0) - sx(php, K, -1))
                 * (rdnw[0:ktf, None, None] * (dpn[1:ktf + 1] - dpn[0:ktf]) - 0.5 * (mu[None, j0:j1, i0 - 1:i1 - 1] + mu[None, j0:j1, i0:i1])))
    ru_tend[K, j0:j1, i0:i1] = ru_tend[K, j0:j1, i0:i1] - cqu[K, j0:j1, i0:i1] * dpx
    return ru_tend, rv_tend


def pg_buoy_w(g, rw_tend, p, cqw, mu, mub, rdnw, rdn, msfty):
    """wrf_dynamics.py:2424-2460 (also replaces cqw by 1/(1+cqw) on levels
    [1, kde-1), which calc_coef_w and advance_w then use)."""
    kde = g.nz
    j0, j1, i0, i1 = g.jds, g.jde - 1, g.ids, g.ide - 1
    R = (slice(j0, j1), slice(i0, i1))
    cq1 = 1.0 / (1.0 + cqw[kde - 2][R])
    cq2 = cqw[kde - 2][R] * cq1
    rw_tend[kde - 1][R] = rw_tend[kde - 1][R] + (1.0 / msfty[R]) * G * (cq1 * 2.0 * rdnw[kde - 2] * (-p[kde - 2][R]) - mu[R] - cq2 * mub[R])
    K = slice(1, kde - 1)
    cq1 = 1.0 / (1.0 + cqw[K, j0:j1, i0:i1])
    cq2 = cqw[K, j0:j1, i0:i1] * cq1
    cqw[K, j0:j1, i0:i1] = cq1
    rw_tend[K, j0:j1, i0:i1] = rw_tend[K, j0:j1, i0:i1] + (1.0 / msfty[None, j0:j1, i0:i1]) * G * (
        cq1 * rdn[K, None, None] * (p[K, j0:j1, i0:i1] - p[0:kde - 2, j0:j1, i0:i1]) - mu[None, j0:j1, i0:i1] - cq2 * mub[None, j0:j1, i0:i1])
    return rw_tend, cqw


def coriolis(g, ru, rv, rw, ru_tend, rv_tend, rw_tend, msftx, msfty, msfux, msfuy, msfvx, msfvy,
             f, e, sina, cosa, fzm, fzp):
    """wrf_dynamics.py:2463-2532"""
    ktf = g.nz - 1
    K, K1 = slice(0, ktf), slice(1, ktf + 1)
    # u
    j0, j1, i0, i1 = g.jts, g.jte - 1, g.ids + 1, g.ide - 1
    X = lambda a, jj, ii: a[None, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    R3 = lambda a, kk, jj, ii: a[kk, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    ru_tend[K, j0:j1, i0:i1] = (ru_tend[K, j0:j1, i0:i1]
                                + (X(msfux, 0, 0) / X(msfuy, 0, 0)) * 0.5 * (X(f, 0, 0) + X(f, 0, -1)) * 0.25
                                * (R3(rv, K, 1, -1) + R3(rv, K, 1, 0) + R3(rv, K, 0, -1) + R3(rv, K, 0, 0))
                                - 0.5 * (X(e, 0, 0) + X(e, 0, -1)) * 0.5 * (X(cosa, 0, 0) + X(cosa, 0, -1)) * 0.25
                                * (R3(rw, K1, 0, -1) + R3(rw, K, 0, -1) + R3(rw, K1, 0, 0) + R3(rw, K, 0, 0)))
    # v
    j0, j1, i0, i1 = g.jds + 1, g.jde - 1, g.its, g.ite - 1
    X = lambda a, jj, ii: a[None, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    R3 = lambda a, kk, jj, ii: a[kk, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    rv_tend[K, j0:j1, i0:i1] = (rv_tend[K, j0:j1, i0:i1]
                                - (X(msfvy, 0, 0) / X(msfvx, 0, 0)) * 0.5 * (X(f, 0, 0) + X(f, -1, 0)) * 0.25
                                * (R3(ru, K, 0, 0) + R3(ru, K, 0, 1) + R3(ru, K, -1, 0) + R3(ru, K, -1, 1))
                                + (X(msfvy, 0, 0) / X(msfvx, 0, 0)) * 0.5 * (X(e, 0, 0) + X(e, -1, 0)) * 0.5 * (X(sina, 0, 0) + X(sina, -1, 0)) * 0.25
                                * (R3(rw, K1, -1, 0) + R3(rw, K, -1, 0) + R3(rw, K1, 0, 0) + R3(rw, K, 0, 0)))
    # w
    j0, j1, i0, i1 = g.jts, g.jte - 1, g.its, g.ite - 1
    KW, KWm = slice(1, ktf), slice(0, ktf - 1)
    X = lambda a, jj, ii: a[None, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    R3 = lambda a, kk, jj, ii: a[kk, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    fm, fp = fzm[KW, None, None], fzp[KW, None, None]
    rw_tend[KW, j0:j1, i0:i1] = rw_tend[KW, j0:j1, i0:i1] + X(e, 0, 0) * (
        X(cosa, 0, 0) * 0.5 * (fm * (R3(ru, KW, 0, 0) + R3(ru, KW, 0, 1)) + fp * (R3(ru, KWm, 0, 0) + R3(ru, KWm, 0, 1)))
        - (X(msftx, 0, 0) / X(msfty, 0, 0)) * X(sina, 0, 0) * 0.5 * (fm * (R3(rv, KW, 0, 0) + R3(rv, KW, 1, 0)) + fp * (R3(rv, KWm, 0, 0) + R3(rv, KWm, 1, 0))))
    return ru_tend, rv_tend, rw_tend


def curvature(g, ru, rv, rw, u, v, ru_tend, rv_tend, rw_tend, msfux, msfuy, msfvx, msfvy, msftx, msfty, fzm, fzp):
    """wrf_dynamics.py:2535-2620"""
    ktf = g.nz - 1
    K, K1 = slice(0, ktf), slice(1, ktf + 1)
    rdx, rdy = g.rdx, g.rdy
    its, ite, jts, jte = g.its, g.ite, g.jts, g.jte
    vxgm = np.zeros((g.nz, g.ny, g.nx), u.dtype)
    j0, j1, i0, i1 = jts, jte - 1, its, ite - 1
    vxgm[K, j0:j1, i0:i1] = (0.5 * (u[K, j0:j1, i0:i1] + u[K, j0:j1, i0 + 1:i1 + 1]) * (msfvx[None, j0 + 1:j1 + 1, i0:i1] - msfvx[None, j0:j1, i0:i1]) * rdy
                             - 0.5 * (v[K, j0:j1, i0:i1] + v[K, j0 + 1:j1 + 1, i0:i1]) * (msfuy[None, j0:j1, i0 + 1:i1 + 1] - msfuy[None, j0:j1, i0:i1]) * rdx)
    vxgm[K, jts:jte - 1, its - 1] = vxgm[K, jts:jte - 1, its]
    vxgm[K, jts:jte - 1, ite - 1] = vxgm[K, jts:jte - 1, ite - 2]
    vxgm[K, jts - 1, its - 1:ite] = vxgm[K, jts, its - 1:ite]
    vxgm[K, jte - 1, its - 1:ite] = vxgm[K, jte - 2, its - 1:ite]
    # u
    j0, j1, i0, i1 = jts, jte - 1, g.ids + 1, g.ide - 1
    R3 = lambda a, kk, jj, ii: a[kk, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    ru_tend[K, j0:j1, i0:i1] = (ru_tend[K, j0:j1, i0:i1]
                                + 0.5 * (R3(vxgm, K, 0, 0) + R3(vxgm, K, 0, -1)) * 0.25
                                * (R3(rv, K, 1, -1) + R3(rv, K, 1, 0) + R3(rv, K, 0, -1) + R3(rv, K, 0, 0))
                                - R3(u, K, 0, 0) * RERADIUS * 0.25 * (R3(rw, K1, 0, -1) + R3(rw, K, 0, -1) + R3(rw, K1, 0, 0) + R3(rw, K, 0, 0)))
    # v
    j0, j1, i0, i1 = g.jds + 1, g.jde - 1, its, ite - 1
    R3 = lambda a, kk, jj, ii: a[kk, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    rv_tend[K, j0:j1, i0:i1] = (rv_tend[K, j0:j1, i0:i1]
                                - 0.5 * (R3(vxgm, K, 0, 0) + R3(vxgm, K, -1, 0)) * 0.25
                                * (R3(ru, K, 0, 0) + R3(ru, K, 0, 1) + R3(ru, K, -1, 0) + R3(ru, K, -1, 1))
                                - (msfvy[None, j0:j1, i0:i1] / msfvx[None, j0:j1, i0:i1]) * R3(v, K, 0, 0) * RERADIUS * 0.25
                                * (R3(rw, K1, -1, 0) + R3(rw, K, -1, 0) + R3(rw, K1, 0, 0) + R3(rw, K, 0, 0)))
    # w
    j0, j1, i0, i1 = jts, jte - 1, its, ite - 1
    KW, KWm = slice(1, ktf), slice(0, ktf - 1)
    R3 = lambda a, kk, jj, ii: a[kk, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    fm, fp = fzm[KW, None, None], fzp[KW, None, None]
    rw_tend[KW, j0:j1, i0:i1] = rw_tend[KW, j0:j1, i0:i1] + RERADIUS * (
        0.5 * (fm * (R3(ru, KW, 0, 0) + R3(ru, KW, 0, 1)) + fp * (R3(ru, KWm, 0, 0) + R3(ru, KWm, 0, 1)))
        * 0.5 * (fm * (R3(u, KW, 0, 0) + R3(u, KW, 0, 1)) + fp * (R3(u, KWm, 0, 0) + R3(u, KWm, 0, 1)))
        + (msftx[None, j0:j1, i0:i1] / msfty[None, j0:j1, i0:i1])
        * 0.5 * (fm * (R3(rv, KW, 0, 0) + R3(rv, KW, 1, 0)) + fp * (R3(rv, KWm, 0, 0) + R3(rv, KWm, 1, 0)))
        * 0.5 * (fm * (R3(v, KW, 0, 0) + R3(v, KW, 1, 0)) + fp * (R3(v, KWm, 0, 0) + R3(v, KWm, 1, 0))))
    return ru_tend, rv_tend, rw_tend


def rk_addtend_dry(g, ru_tend, rv_tend, rw_tend, ph_tend, t_tend, ru_tendf, rv_tendf, rw_tendf,
                   ph_tendf, t_tendf, u_save, v_save, w_save, ph_save, t_save, mu_tend, mu_tendf,
                   rk_step, h_diabatic, mut, msfty, msfuy, msfvx, msfvx_inv):
    """wrf_dynamics.py:3100-3148"""
    nz = g.nz
    j0, jm, i0 = g.jts, g.jde - 1, g.its
    U = (slice(0, nz - 1), slice(j0, jm), slice(i0, g.ite))
    V = (slice(0, nz - 1), slice(j0, g.jte), slice(i0, g.ide - 1))
    W = (slice(0, nz), slice(j0, jm), slice(i0, g.ide - 1))
    T = (slice(0, nz - 1), slice(j0, jm), slice(i0, g.ide - 1))
    m2 = lambda a, s: a[None, s[1], s[2]]
    if rk_step == 1:
        ru_tendf[U] = ru_tendf[U] + u_save[U] * m2(msfuy, U)
    ru_tend[U] = ru_tend[U] + ru_tendf[U] / m2(msfuy, U)
    if rk_step == 1:
        rv_tendf[V] = rv_tendf[V] + v_save[V] * m2(msfvx, V)
    rv_tend[V] = rv_tend[V] + rv_tendf[V] * m2(msfvx_inv, V)
    if rk_step == 1:
        rw_tendf[W] = rw_tendf[W] + w_save[W] * m2(msfty, W)
    rw_tend[W] = rw_tend[W] + rw_tendf[W] / m2(msfty, W)
    if rk_step == 1:
        ph_tendf[W] = ph_tendf[W] + ph_save[W]
    ph_tend[W] = ph_tend[W] + ph_tendf[W] / m2(msfty, W)
    if rk_step == 1:
        t_tendf[T] = t_tendf[T] + t_save[T]
    t_tend[T] = t_tend[T] + t_tendf[T] / m2(msfty, T) + m2(mut, T) * h_diabatic[T] / m2(msfty, T)
    mu_tend[j0:jm, i0:g.ide - 1] = mu_tend[j0:jm, i0:g.ide - 1] + mu_tendf[j0:jm, i0:g.ide - 1]


# ----------------------------------------------------------- acoustic small step

def small_step_prep(g, st, rk_step):
    """wrf_dynamics.py:3152-3266.  ``st`` holds the named state buffers; the
    reference returns clones that the caller rebinds, which is the same as
    updating in place."""
    nz = g.nz
    ktf = nz - 1
    j0, jm, i0, im = g.jts, g.jde - 1, g.its, g.ide - 1
    ieu, jev = g.ite, g.jte
    mub, mu1, mu2 = st["mub"], st["mu_1"], st["mu"]
    muu, muv, mut = st["muu"], st["muv"], st["mut"]
    muus, muvs, muts, mudf = st["muus"], st["muvs"], st["muts"], st["mudf"]
    T2 = (slice(j0, jm), slice(i0, im))
    if rk_step == 1:
        mu1[T2] = mu2[T2]
        st["ww1"][nz - 1][T2] = 0.0
        st["ww1"][0][T2] = 0.0
        mudf[T2] = 0.0
        st["u_1"][0:ktf, j0:jm, i0:ieu] = st["u"][0:ktf, j0:jm, i0:ieu]
        st["v_1"][0:ktf, j0:jev, i0:im] = st["v"][0:ktf, j0:jev, i0:im]
        st["t_1"][0:ktf, j0:jm, i0:im] = st["t"][0:ktf, j0:jm, i0:im]
        st["w_1"][0:nz, j0:jm, i0:im] = st["w"][0:nz, j0:jm, i0:im]
        st["ph_1"][0:nz, j0:jm, i0:im] = st["ph"][0:nz, j0:jm, i0:im]
        muts[T2] = mub[T2] + mu2[T2]
        muus[j0:jm, i0:ieu] = muu[j0:jm, i0:ieu]
        muvs[j0:jev, i0:im] = muv[j0:jev, i0:im]
        st["mu_save"][T2] = mu2[T2]
        mu2[T2] = 0.0
    else:
        muts[T2] = mub[T2] + mu1[T2]
        muus[j0:jm, i0:ieu] = 0.5 * (mub[j0:jm, i0:ieu] + mu1[j0:jm, i0:ieu] + mub[j0:jm, i0 - 1:ieu - 1] + mu1[j0:jm, i0 - 1:ieu - 1])
        muvs[j0:jev, i0:ieu] = 0.5 * (mub[j0:jev, i0:ieu] + mu1[j0:jev, i0:ieu] + mub[j0 - 1:jev - 1, i0:ieu] + mu1[j0 - 1:jev - 1, i0:ieu])
        st["mu_save"][T2] = mu2[T2]
        mu2[T2] = mu1[T2] - mu2[T2]
    st["ww1"][nz - 1][T2] = 0.0
    st["ww1"][0][T2] = 0.0
    st["c2a"][0:ktf, j0:jm, i0:im] = CPOVCV * (st["pb"][0:ktf, j0:jm, i0:im] + st["p"][0:ktf, j0:jm, i0:im]) / st["alt"][0:ktf, j0:jm, i0:im]
    U = (slice(0, ktf), slice(j0, jm), slice(i0, ieu))
    u2 = st["u"][U].copy()
    st["u_save"][U] = u2
    st["u"][U] = (muus[None, j0:jm, i0:ieu] * st["u_1"][U] - muu[None, j0:jm, i0:ieu] * u2) / st["msfuy"][None, j0:jm, i0:ieu]
    V = (slice(0, ktf), slice(j0, jev), slice(i0, im))
    v2 = st["v"][V].copy()
    st["v_save"][V] = v2
    st["v"][V] = (muvs[None, j0:jev, i0:im] * st["v_1"][V] - muv[None, j0:jev, i0:im] * v2) * st["msfvx_inv"][None, j0:jev, i0:im]
    T = (slice(0, ktf), slice(j0, jm), slice(i0, im))
    t2 = st["t"][T].copy()
    st["t_save"][T] = t2
    st["t"][T] = muts[None, j0:jm, i0:im] * st["t_1"][T] - mut[None, j0:jm, i0:im] * t2
    W = (slice(0, nz), slice(j0, jm), slice(i0, im))
    w2 = st["w"][W].copy()
    st["w_save"][W] = w2
    st["w"][W] = (muts[None, j0:jm, i0:im] * st["w_1"][W] - mut[None, j0:jm, i0:im] * w2) / st["msfty"][None, j0:jm, i0:im]
    ph2 = st["ph"][W].copy()
    st["ph_save"][W] = ph2
    st["ph"][W] = st["ph_1"][W] - ph2
    st["ww1"][W] = st["ww"][W]


def calc_p_rho(g, al, p, ph, alt, t_2, t_1, c2a, pm1, mu, mut, rdnw, smdiv, step):
    """wrf_dynamics.py:3269-3313.  Returns the (possibly new) pm1 array: at
    step 0 the reference replaces pm1 by a full copy of p."""
    ktf = g.nz - 1
    R = (slice(0, ktf), slice(g.jts, g.jde - 1), slice(g.its, g.ide - 1))
    m = lambda a: a[None, R[1], R[2]]
    al[R] = -1.0 / m(mut) * (alt[R] * m(mu) + rdnw[0:ktf, None, None] * (ph[1:ktf + 1, R[1], R[2]] - ph[R]))
    p[R] = c2a[R] * (alt[R] * (t_2[R] - m(mu) * t_1[R]) / (m(mut) * (T0 + t_1[R])) - al[R])
    if step == 0:
        return p.copy()
    ptmp = p[R].copy()
    p[R] = p[R] + smdiv * (p[R] - pm1[R])
    pm1[R] = ptmp
    return pm1


def calc_coef_w(g, a, alpha, gamma, mut, cqw, rdn, rdnw, c2a, dts, epssm, top_lid=False):
    """wrf_dynamics.py:3316-3388 (tridiagonal coefficients and forward sweep)."""
    kde = g.nz
    R2 = (slice(g.jts, g.jde - 1), slice(g.its, g.ide - 1))
    lid = 0 if top_lid else 1
    cof = (0.5 * dts * G * (1.0 + epssm)) ** 2
    m = mut[R2]
    mm = m * m
    dt_ = a.dtype
    b = np.zeros((kde,) + m.shape, dt_)
    c = np.zeros((kde,) + m.shape, dt_)
    aa = a[(slice(None),) + R2]
    al_ = alpha[(slice(None),) + R2]
    ga = gamma[(slice(None),) + R2]
    aa[1] = 0.0
    aa[kde - 1] = -2.0 * cof * (rdnw[kde - 2] * rdnw[kde - 2]) * c2a[kde - 2][R2] * lid / mm
    ga[0] = 0.0
    K2 = slice(2, kde - 1)
    aa[K2] = -cqw[K2][(slice(None),) + R2] * cof * rdn[K2, None, None] * rdnw[1:kde - 2, None, None] * c2a[1:kde - 2][(slice(None),) + R2] / mm
    K1 = slice(1, kde - 1)
    cw = cqw[K1][(slice(None),) + R2]
    b[K1] = 1.0 + cw * cof * rdn[K1, None, None] * (rdnw[K1, None, None] * c2a[K1][(slice(None),) + R2] / mm
                                                    + rdnw[0:kde - 2, None, None] * c2a[0:kde - 2][(slice(None),) + R2] / mm)
    c[K1] = -cw * cof * rdn[K1, None, None] * rdnw[K1, None, None] * c2a[K1][(slice(None),) + R2] / mm
    for k in range(1, kde - 1):
        al_[k] = 1.0 / (b[k] - aa[k] * ga[k - 1])
        ga[k] = c[k] * al_[k]
    b[kde - 1] = 1.0 + 2.0 * cof * (rdnw[kde - 2] * rdnw[kde - 2]) * c2a[kde - 2][R2] / mm
    al_[kde - 1] = 1.0 / (b[kde - 1] - aa[kde - 1] * ga[kde - 2])
    ga[kde - 1] = 0.0
    a[(slice(None),) + R2] = aa
    alpha[(slice(None),) + R2] = al_
    gamma[(slice(None),) + R2] = ga
    return a, alpha, gamma


def advance_uv(g, u, ru_tend, v, rv_tend, p, pb, ph, php, alt, al, mu, muu, cqu, muv, cqv, mudf,
               msfux, msfuy, msfvx, msfvx_inv, msfvy, dts, cf1, cf2, cf3, fnm, fnp, emdiv, rdnw):
    """wrf_dynamics.py:3391-3525 (spec_zone = 1)."""
    nz = g.nz
    ktf = nz - 1
    sz = g.spec_zone
    i_s, i_e = g.ids + sz, g.ide - sz - 1
    j_s, j_e = g.jds + sz, g.jde - sz - 1
    i_eu, j_ev = g.ide - sz, g.jde - sz
    dx, dy = 1.0 / g.rdx, 1.0 / g.rdy
    rdx, rdy = g.rdx, g.rdy
    K, K1 = slice(0, ktf), slice(1, ktf + 1)
    # u
    j0, j1, i0, i1 = j_s, j_e, i_s, i_eu
    u[K, j0:j1, i0:i1] = u[K, j0:j1, i0:i1] + dts * ru_tend[K, j0:j1, i0:i1]
    mudf_xy = -emdiv * dx * (mudf[j0:j1, i0:i1] - mudf[j0:j1, i0 - 1:i1 - 1]) / msfuy[j0:j1, i0:i1]
    sx = lambda a, kk, ii: a[kk, j0:j1, i0 + ii:i1 + ii]
    dpxy = ((msfux[None, j0:j1, i0:i1] / msfuy[None, j0:j1, i0:i1]) * 0.5 * rdx * muu[None, j0:j1, i0:i1]
            * (((sx(ph, K1, 0) - sx(ph, K1, -1)) + (sx(ph, K, 0) - sx(ph, K, -1)))
               + (sx(alt, K, 0) + sx(alt, K, -1)) * (sx(p, K, 0) - sx(p, K, -1))
               + (sx(al, K, 0) + sx(al, K, -1)) * (sx(pb, K, 0) - sx(pb, K, -1))))
    dpn = _dpn(p, nz, fnm, fnp, cf1, cf2, cf3, (slice(j0, j1), slice(i0 - 1, i1 - 1)), (slice(j0, j1), slice(i0, i1)))
    dpxy = dpxy + ((msfux[None, j0:j1, i0:i1] / msfuy[None, j0:j1, i0:i1]) * rdx * (sx(php, K, 0) - sx(php, K, -1))
                   * (rdnw[0:ktf, None, None] * (dpn[1:ktf + 1] - dpn[0:ktf]) - 0.5 * (mu[None, j0:j1, i0 - 1:i1 - 1] + mu[None, j0:j1, i0:i1])))
    u[K, j0:j1, i0:i1] = u[K, j0:j1, i0:i1] - dts * cqu[K, j0:j1, i0:i1] * dpxy + mudf_xy[None]
    # v
    j0, j1, i0, i1 = j_s, j_ev, i_s, i_e
    v[K, j0:j1, i0:i1] = v[K, j0:j1, i0:i1] + dts * rv_tend[K, j0:j1, i0:i1]
    mudf_xy = -emdiv * dy * (mudf[j0:j1, i0:i1] - mudf[j0 - 1:j1 - 1, i0:i1]) * msfvx_inv[j0:j1, i0:i1]
    sy = lambda a, kk, jj: a[kk, j0 + jj:j1 + jj, i0:i1]
    dpxy = ((msfvy[None, j0:j1, i0:i1] / msfvx[None, j0:j1, i0:i1]) * 0.5 * rdy * muv[None, j0:j1, i0:i1]
            * (((sy(ph, K1, 0) - sy(ph, K1, -1)) + (sy(ph, K, 0) - sy(ph, K, -1)))
               + (sy(alt, K, 0) + sy(alt, K, -1)) * (sy(p, K, 0) - sy(p, K, -1))
               + (sy(al, K, 0) + sy(al, K, -1)) * (sy(pb, K, 0) - sy(pb, K, -1))))
    dpn = _dpn(p, nz, fnm, fnp, cf1, cf2, cf3, (slice(j0 - 1, j1 - 1), slice(i0, i1)), (slice(j0, j1), slice(i0, i1)))
    dpxy = dpxy + ((msfvy[None, j0:j1, i0:i1] / msfvx[None, j0:j1, i0:i1]) * rdy * (sy(php, K, 0) - sy(php, K, -1))
                   * (rdnw[0:ktf, None, None] * (dpn[1:ktf + 1] - dpn[0:ktf]) - 0.5 * (mu[None, j0 - 1:j1 - 1, i0:i1] + mu[None, j0:j1, i0:i1])))
    v[K, j0:j1, i0:i1] = v[K, j0:j1, i0:i1] - dts * cqv[K, j0:j1, i0:i1] * dpxy + mudf_xy[None]
    return u, v


def advance_mu_t(g, st, dts, epssm, iteration):
    """wrf_dynamics.py:3528-3638.  Uses st: ww, ww1, u, u_save, v, v_save, mu,
    mut, muave, muts, muu, muv, mudf, t, t_save, t_2save, t_tend, mu_tend."""
    nz = g.nz
    k_end = nz - 1
    i0, i1 = g.ids + 1, g.ide - 2
    j0, j1 = g.jds + 1, g.jde - 2
    rdx, rdy = g.rdx, g.rdy
    u, v, u1, v1 = st["u"], st["v"], st["u_save"], st["v_save"]
    muu, muv = st["muu"], st["muv"]
    msftx, msfty, msfuy, msfvx_inv = st["msftx"], st["msfty"], st["msfuy"], st["msfvx_inv"]
    dnw, fnm, fnp, rdnw = st["dnw"], st["fnm"], st["fnp"], st["rdnw"]
    K = slice(0, k_end)
    X = lambda a, jj, ii: a[None, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    R3 = lambda a, kk, jj, ii: a[kk, j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    dvdxi = X(msftx, 0, 0) * X(msfty, 0, 0) * (
        rdy * ((R3(v, K, 1, 0) + X(muv, 1, 0) * R3(v1, K, 1, 0) * X(msfvx_inv, 1, 0)) - (R3(v, K, 0, 0) + X(muv, 0, 0) * R3(v1, K, 0, 0) * X(msfvx_inv, 0, 0)))
        + rdx * ((R3(u, K, 0, 1) + X(muu, 0, 1) * R3(u1, K, 0, 1) / X(msfuy, 0, 1)) - (R3(u, K, 0, 0) + X(muu, 0, 0) * R3(u1, K, 0, 0) / X(msfuy, 0, 0))))
    dmk = dnw[0:k_end, None, None] * dvdxi
    dmdt = np.zeros_like(dmk[0])
    for k in range(k_end):
        dmdt = dmdt + dmk[k]
    mu, muave, muts, mudf, mut, mu_tend = st["mu"], st["muave"], st["muts"], st["mudf"], st["mut"], st["mu_tend"]
    R2 = (slice(j0, j1), slice(i0, i1))
    muave[R2] = mu[R2]
    mu[R2] = mu[R2] + dts * (dmdt + mu_tend[R2])
    mudf[R2] = dmdt + mu_tend[R2]
    muts[R2] = mut[R2] + mu[R2]
    muave[R2] = 0.5 * ((1.0 + epssm) * mu[R2] + (1.0 - epssm) * muave[R2])
    ww = st["ww"]
    for k in range(1, k_end):
        ww[k][R2] = ww[k - 1][R2] - dnw[k - 1] * (dmdt + dvdxi[k - 1] + mu_tend[R2]) / msfty[R2]
    ww[0:k_end, j0:j1, i0:i1] = ww[0:k_end, j0:j1, i0:i1] - st["ww1"][0:k_end, j0:j1, i0:i1]
    t, t1, ft = st["t"], st["t_save"], st["t_tend"]
    st["t_2save"][0:k_end, j0:j1, i0:i1] = t[0:k_end, j0:j1, i0:i1]
    t[0:k_end, j0:j1, i0:i1] = t[0:k_end, j0:j1, i0:i1] + X(msfty, 0, 0) * dts * ft[0:k_end, j0:j1, i0:i1]
    wdtn = np.zeros((nz,) + dmdt.shape, t.dtype)
    wdtn[1:k_end] = ww[1:k_end, j0:j1, i0:i1] * (fnm[1:k_end, None, None] * t1[1:k_end, j0:j1, i0:i1] + fnp[1:k_end, None, None] * t1[0:k_end - 1, j0:j1, i0:i1])
    t[0:k_end, j0:j1, i0:i1] = t[0:k_end, j0:j1, i0:i1] - dts * X(msfty, 0, 0) * (
        X(msftx, 0, 0) * (0.5 * rdy * (R3(v, K, 1, 0) * (R3(t1, K, 1, 0) + R3(t1, K, 0, 0)) - R3(v, K, 0, 0) * (R3(t1, K, 0, 0) + R3(t1, K, -1, 0)))
                          + 0.5 * rdx * (R3(u, K, 0, 1) * (R3(t1, K, 0, 1) + R3(t1, K, 0, 0)) - R3(u, K, 0, 0) * (R3(t1, K, 0, 0) + R3(t1, K, 0, -1))))
        + rdnw[0:k_end, None, None] * (wdtn[1:k_end + 1] - wdtn[0:k_end]))


def advance_w(g, st, dts, epssm, cf1, cf2, cf3):
    """wrf_dynamics.py:3641-3796: w/phi implicit solve with Thomas
    back-substitution and Rayleigh w damping (dampcoef 0.2, zdamp 5000 m,
    pi = 3.14159265359 as hard-coded there)."""
    nz = g.nz
    k_end = nz - 1
    i0, i1 = g.ids + 1, g.ide - 2
    j0, j1 = g.jds + 1, g.jde - 2
    R2 = (slice(j0, j1), slice(i0, i1))
    rdx, rdy = g.rdx, g.rdy
    pi_ = 3.14159265359
    dampmag = dts * 0.2
    hdepth = 5000.0
    w, ph, t_2ave = st["w"], st["ph"], st["t_2save"]
    ww, ph_1, phb, ph_tend = st["ww"], st["ph_save"], st["phb"], st["ph_tend"]
    t_2, t_1 = st["t"], st["t_save"]
    muave, muts, mut = st["muave"], st["muts"], st["mut"]
    msfty, msftx = st["msfty"], st["msftx"]
    fnm, fnp, rdnw, rdn = st["fnm"], st["fnp"], st["rdnw"], st["rdn"]
    c2a, cqw, alt = st["c2a"], st["cqw"], st["alt"]
    a, alpha, gamma = st["a"], st["alpha"], st["gamma"]
    u, v, ht, rw_tend = st["u"], st["v"], st["ht"], st["rw_tend"]
    Z = lambda a_, k0, k1: a_[k0:k1, j0:j1, i0:i1]
    M = lambda a_: a_[None, j0:j1, i0:i1]
    rhs = np.zeros((nz, j1 - j0, i1 - i0), w.dtype)
    msft_inv = 1.0 / M(msfty)
    t_2ave[0:k_end, j0:j1, i0:i1] = 0.5 * ((1.0 + epssm) * Z(t_2, 0, k_end) + (1.0 - epssm) * Z(t_2ave, 0, k_end))
    t_2ave[0:k_end, j0:j1, i0:i1] = (Z(t_2ave, 0, k_end) + M(muave) * T0) / (M(muts) * (T0 + Z(t_1, 0, k_end)))
    wdwn = np.zeros_like(rhs)
    wdwn[1:k_end + 1] = (0.5 * (Z(ww, 1, k_end + 1) + Z(ww, 0, k_end)) * rdnw[0:k_end, None, None]
                         * (Z(ph_1, 1, k_end + 1) - Z(ph_1, 0, k_end) + Z(phb, 1, k_end + 1) - Z(phb, 0, k_end)))
    rhs[1:k_end + 1] = dts * (Z(ph_tend, 1, k_end + 1) + 0.5 * G * (1.0 - epssm) * Z(w, 1, k_end + 1))
    rhs[1:k_end] = rhs[1:k_end] - dts * (fnm[1:k_end, None, None] * wdwn[2:k_end + 1] + fnp[1:k_end, None, None] * wdwn[1:k_end])
    rhs[1:k_end + 1] = Z(ph, 1, k_end + 1) + M(msfty) * rhs[1:k_end + 1] / M(mut)
    cv = lambda kk, jj: cf1 * v[0, j0 + jj:j1 + jj, i0:i1] + cf2 * v[1, j0 + jj:j1 + jj, i0:i1] + cf3 * v[2, j0 + jj:j1 + jj, i0:i1]
    cu = lambda ii: cf1 * u[0, j0:j1, i0 + ii:i1 + ii] + cf2 * u[1, j0:j1, i0 + ii:i1 + ii] + cf3 * u[2, j0:j1, i0 + ii:i1 + ii]
    hh = lambda jj, ii: ht[j0 + jj:j1 + jj, i0 + ii:i1 + ii]
    w[0, j0:j1, i0:i1] = (msfty[R2] * 0.5 * rdy * ((hh(1, 0) - hh(0, 0)) * cv(0, 1) + (hh(0, 0) - hh(-1, 0)) * cv(0, 0))
                          + msftx[R2] * 0.5 * rdx * ((hh(0, 1) - hh(0, 0)) * cu(1) + (hh(0, 0) - hh(0, -1)) * cu(0)))
    K = slice(1, k_end)
    mutk = M(mut)
    X1 = (c2a[1:k_end, j0:j1, i0:i1] * rdnw[1:k_end, None, None] / mutk
          * ((1.0 + epssm) * (rhs[2:k_end + 1] - rhs[1:k_end]) + (1.0 - epssm) * (Z(ph, 2, k_end + 1) - Z(ph, 1, k_end))))
    X2 = (c2a[0:k_end - 1, j0:j1, i0:i1] * rdnw[0:k_end - 1, None, None] / mutk
          * ((1.0 + epssm) * (rhs[1:k_end] - rhs[0:k_end - 1]) + (1.0 - epssm) * (Z(ph, 1, k_end) - Z(ph, 0, k_end - 1))))
    w[K, j0:j1, i0:i1] = (Z(w, 1, k_end) + dts * Z(rw_tend, 1, k_end)
                          + msft_inv * Z(cqw, 1, k_end) * (0.5 * dts * G * rdn[K, None, None] * (X1 - X2))
                          + dts * G * msft_inv * (rdn[K, None, None] * (Z(c2a, 1, k_end) * Z(alt, 1, k_end) * Z(t_2ave, 1, k_end)
                                                                       - Z(c2a, 0, k_end - 1) * Z(alt, 0, k_end - 1) * Z(t_2ave, 0, k_end - 1)) - M(muave)))
    ke = k_end
    w[ke, j0:j1, i0:i1] = (w[ke, j0:j1, i0:i1] + dts * rw_tend[ke, j0:j1, i0:i1]
                           + msft_inv[0] * (-0.5 * dts * G / mut[R2] * (rdnw[ke - 1] * rdnw[ke - 1]) * 2.0 * c2a[ke - 1][R2]
                                            * ((1.0 + epssm) * (rhs[ke] - rhs[ke - 1]) + (1.0 - epssm) * (ph[ke][R2] - ph[ke - 1][R2]))
                                            - dts * G * (2.0 * rdnw[ke - 1] * c2a[ke - 1][R2] * alt[ke - 1][R2] * t_2ave[ke - 1][R2] + muave[R2])))
    for k in range(1, k_end + 1):
        w[k][R2] = (w[k][R2] - a[k][R2] * w[k - 1][R2]) * alpha[k][R2]
    for k in range(k_end - 1, 0, -1):
        w[k][R2] = w[k][R2] - gamma[k][R2] * w[k + 1][R2]
    htop = (ph_1[k_end][R2] + phb[k_end][R2]) / G
    hbot = htop - hdepth
    hk = (Z(ph_1, 1, k_end + 1) + Z(phb, 1, k_end + 1)) / G
    sarg = np.sin(0.5 * pi_ * (hk - hbot[None]) / hdepth)
    dampwt = np.where(hk >= hbot[None], dampmag * (sarg * sarg), 0.0).astype(w.dtype)
    w[1:k_end + 1, j0:j1, i0:i1] = (Z(w, 1, k_end + 1) - dampwt * M(mut) * Z(st["w_save"], 1, k_end + 1)) / (1.0 + dampwt)
    ph[1:k_end + 1, j0:j1, i0:i1] = rhs[1:k_end + 1] + M(msfty) * 0.5 * dts * G * (1.0 + epssm) * Z(w, 1, k_end + 1) / M(muts)


def sumflux(g, st, iteration, nsub):
    """wrf_dynamics.py:3799-3839 (time-averaged mass fluxes)."""
    nz = g.nz
    ru_m, rv_m, ww_m = st["ru_m"], st["rv_m"], st["ww_m"]
    if iteration == 1:
        for a in (ru_m, rv_m, ww_m):
            a[0:nz, g.jts:g.jte, g.its:g.ite] = 0.0
    kk, jj, ii = nz - 1, g.jde - 1, g.ide - 1
    U = (slice(0, kk), slice(g.jts, jj), slice(g.its, g.ite))
    V = (slice(0, kk), slice(g.jts, g.jte), slice(g.its, ii))
    W = (slice(0, nz), slice(g.jts, jj), slice(g.its, ii))
    ru_m[U] = ru_m[U] + st["u"][U]
    rv_m[V] = rv_m[V] + st["v"][V]
    ww_m[W] = ww_m[W] + st["ww"][W]
    if iteration == nsub:
        ru_m[U] = ru_m[U] / nsub + st["muu"][None, U[1], U[2]] * st["u_save"][U] / st["msfuy"][None, U[1], U[2]]
        rv_m[V] = rv_m[V] / nsub + st["muv"][None, V[1], V[2]] * st["v_save"][V] * st["msfvx_inv"][None, V[1], V[2]]
        ww_m[W] = ww_m[W] / nsub + st["ww1"][W]


def calc_mu_uv_1(g, mu, muu, muv):
    """wrf_dynamics.py:3844-3860"""
    js, jm, its, ite = g.jts, g.jde - 1, g.its, g.ite
    muu[js:jm, its + 1:ite - 1] = 0.5 * (mu[js:jm, its + 1:ite - 1] + mu[js:jm, its:ite - 2])
    muu[js:jm, its] = mu[js:jm, its]
    muu[js:jm, ite - 1] = mu[js:jm, ite - 2]
    im, jte = g.ide - 1, g.jte
    muv[js + 1:jte - 1, its:im] = 0.5 * (mu[js + 1:jte - 1, its:im] + mu[js:jte - 2, its:im])
    muv[js, its:im] = mu[js, its:im]
    muv[jte - 1, its:im] = mu[jte - 2, its:im]


def small_step_finish(g, st, nsub, dts, rk_step, rk_order=3):
    """wrf_dynamics.py:3863-3930"""
    nz = g.nz
    j0, jm, i0, im = g.jts, g.jde - 1, g.its, g.ide - 1
    ieu, jev = g.ite, g.jte
    M = lambda a, js_, is_: a[None, js_, is_]
    V = (slice(0, nz - 1), slice(j0, jev), slice(i0, im))
    st["v"][V] = (M(st["msfvx"], V[1], V[2]) * st["v"][V] + st["v_save"][V] * M(st["muv"], V[1], V[2])) / M(st["muvs"], V[1], V[2])
    U = (slice(0, nz - 1), slice(j0, jm), slice(i0, ieu))
    st["u"][U] = (M(st["msfuy"], U[1], U[2]) * st["u"][U] + st["u_save"][U] * M(st["muu"], U[1], U[2])) / M(st["muus"], U[1], U[2])
    W = (slice(0, nz), slice(j0, jm), slice(i0, im))
    st["w"][W] = (M(st["msfty"], W[1], W[2]) * st["w"][W] + st["w_save"][W] * M(st["mut"], W[1], W[2])) / M(st["muts"], W[1], W[2])
    st["ph"][W] = st["ph"][W] + st["ph_save"][W]
    st["ww"][W] = st["ww"][W] + st["ww1"][W]
    T = (slice(0, nz - 1), slice(j0, jm), slice(i0, im))
    mt = M(st["mut"], T[1], T[2])
    if rk_step < rk_order:
        st["t"][T] = (st["t"][T] + st["t_save"][T] * mt) / M(st["muts"], T[1], T[2])
    else:
        st["t"][T] = (st["t"][T] - dts * nsub * mt * st["h_diabatic"][T] + st["t_save"][T] * mt) / M(st["muts"], T[1], T[2])
    R2 = (slice(j0, jm), slice(i0, im))
    st["mu"][R2] = st["mu"][R2] + st["mu_save"][R2]


# ------------------------------------------------------------------ moisture

def rk_update_scalar(g, moist_old, moist, moist_tend, advect_tend, msfty, mu_old, mu_new, mub,
                     rk_step, dt, first=1, last=6):
    """wrf_dynamics.py:4055-4119 (mu-weighted RK update, spec_zone = 1)."""
    nz = g.nz
    full = (slice(0, nz - 1), slice(g.jts, g.jde - 1), slice(g.its, g.ide - 1))
    sz = g.spec_zone
    inner = (slice(0, nz - 1), slice(g.jds + sz, g.jde - sz - 1), slice(g.ids + sz, g.ide - sz - 1))
    muold = mu_old[full[1], full[2]] + mub[full[1], full[2]]
    munew = mu_new[full[1], full[2]] + mub[full[1], full[2]]
    for im in range(first, last + 1):
        tend = np.zeros((nz,) + moist.shape[2:], moist.dtype)
        tend[inner] = advect_tend[im][inner] * msfty[None, inner[1], inner[2]]
        tend[full] = tend[full] + moist_tend[im][full]
        if rk_step == 1:
            moist_old[im] = moist[im]
        moist[im][full] = (muold[None] * moist_old[im][full] + dt * tend[full]) / munew[None]


def calc_p_rho_phi(g, moist_qv, al, alb, mu, muts, ph, p, pb, t, rdnw):
    """wrf_dynamics.py:4124-4164 (full equation of state; the hypsometric
    geopotential update is commented out in the reference)."""
    ktf = g.nz - 1
    R = (slice(0, ktf), slice(g.jts, g.jde - 1), slice(g.its, g.ide - 1))
    m = lambda a: a[None, R[1], R[2]]
    al[R] = -1.0 / m(muts) * (alb[R] * m(mu) + rdnw[0:ktf, None, None] * (ph[1:ktf + 1, R[1], R[2]] - ph[R]))
    qvf = 1.0 + RVOVRD * moist_qv[R]
    temp = (R_D * (T0 + t[R]) * qvf) / (P0 * (al[R] + alb[R]))
    pp = temp ** CPOVCV
    p[R] = pp * P0 - pb[R]


def set_w_surface(g, w, ht, u, v, cf1, cf2, cf3, msftx, msfty):
    """wrf_dynamics.py:4218-4324 (lower boundary w from terrain slope; the
    corner formulas keep the reference's one-sided/zero terms)."""
    its, ite, jts, jte = g.its, g.ite, g.jts, g.jte
    rdx, rdy = g.rdx, g.rdy
    cv = lambda js, is_: cf1 * v[0, js, is_] + cf2 * v[1, js, is_] + cf3 * v[2, js, is_]
    cu = lambda js, is_: cf1 * u[0, js, is_] + cf2 * u[1, js, is_] + cf3 * u[2, js, is_]
    J, I = slice(jts + 1, jte - 2), slice(its + 1, ite - 2)
    Jp, Jm = slice(jts + 2, jte - 1), slice(jts, jte - 3)
    Ip, Im = slice(its + 2, ite - 1), slice(its, ite - 3)
    w[0, J, I] = (msfty[J, I] * 0.5 * rdy * ((ht[Jp, I] - ht[J, I]) * cv(Jp, I) + (ht[J, I] - ht[Jm, I]) * cv(J, I))
                  + msftx[J, I] * 0.5 * rdx * ((ht[J, Ip] - ht[J, I]) * cu(J, Ip) + (ht[J, I] - ht[J, Im]) * cu(J, I)))
    j = jts
    w[0, j, I] = (msfty[j, I] * 0.5 * rdy * ((ht[j + 1, I] - ht[j, I]) * cv(j + 1, I))
                  + msftx[j, I] * 0.5 * rdx * ((ht[j, Ip] - ht[j, I]) * cu(j, Ip) + (ht[j, I] - ht[j, Im]) * cu(j, I)))
    j = jte - 2
    w[0, j, I] = (msfty[j, I] * 0.5 * rdy * ((ht[j, I] - ht[j - 1, I]) * cv(j, I))
                  + msftx[j, I] * 0.5 * rdx * ((ht[j, Ip] - ht[j, I]) * cu(j, Ip) + (ht[j, I] - ht[j, Im]) * cu(j, I)))
    i = its
    w[0, J, i] = (msfty[J, i] * 0.5 * rdy * ((ht[Jp, i] - ht[J, i]) * cv(Jp, i) + (ht[J, i] - ht[Jm, i]) * cv(J, i))
                  + msftx[J, i] * 0.5 * rdx * ((ht[J, i + 1] - ht[J, i]) * cu(J, i + 1)))
    i = ite - 2
    w[0, J, i] = (msfty[J, i] * 0.5 * rdy * ((ht[Jp, i] - ht[J, i]) * cv(Jp, i) + (ht[J, i] - ht[Jm, i]) * cv(J, i))
                  + msftx[J, i] * 0.5 * rdx * ((ht[J, i] - ht[J, i - 1]) * cu(J, i)))
    j, i = jts, its
    w[0, j, i] = msfty[j, i] * 0.5 * rdy * ((ht[j + 1, i] - ht[j, i]) * cv(j + 1, i)) + msftx[j, i] * 0.5 * rdx * ((ht[j, i + 1] - ht[j, i]) * cu(j, i + 1))
    j, i = jte - 2, its
    w[0, j, i] = msfty[j, i] * 0.5 * rdy * ((ht[j, i] - ht[j - 1, i]) * cv(j, i)) + msftx[j, i] * 0.5 * rdx * ((ht[j, i + 1] - ht[j, i]) * cu(j, i + 1))
    j, i = jts, ite - 2
    # reference: the y term differences ht[jts+1] with itself (zero)
    w[0, j, i] = msfty[j, i] * 0.5 * rdy * ((ht[j + 1, i] - ht[j + 1, i]) * cv(j + 1, i)) + msftx[j, i] * 0.5 * rdx * ((ht[j, i] - ht[j, i - 1]) * cu(j, i))
    j, i = jte - 2, ite - 2
    # reference: the x term uses msftx[jts, its]
    w[0, j, i] = msfty[j, i] * 0.5 * rdy * ((ht[j, i] - ht[j - 1, i]) * cv(j, i)) + msftx[jts, its] * 0.5 * rdx * ((ht[j, i] - ht[j, i - 1]) * cu(j, i))
    return w
