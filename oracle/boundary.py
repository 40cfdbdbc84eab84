"""Oracle restatement of the lateral-boundary functions (reference pywrf/wrf_boundary.py).

TEST INFRASTRUCTURE: see oracle/__init__.py.  Boundary arrays use the
reference's in-memory layout after its permutes (pywrf/solver.py:468-482):
x sides ``[nz, ny, 5]`` (b fastest), y sides ``[nz, 5, nx]``; ``b = 0`` is the
outermost (specified) row.  A side dictionary ``bd`` holds
``xs, xe, ys, ye`` (values) and ``txs, txe, tys, tye`` (tendencies).
"""
from __future__ import annotations

import numpy as np


def _extent(g, var):
    """(ibe, jbe, ktf) of the reference's per-stagger bounds."""
    ibe, jbe, ktf = g.ide - 1, g.jde - 1, g.nz - 1
    if var == "u":
        ibe = g.ide
    if var == "v":
        jbe = g.jde
    if var in ("m", "h"):
        ktf = None  # all levels of the field passed
    return ibe, jbe, ktf


def relax_bdytend(g, field, tend, bd, var, dtbc, fcx, gcx):
    """wrf_boundary.py:52-147: relaxation rows b = 1..3 with the 5-point
    fcx/gcx operator on (bdy + dtbc * bdy_tend - field)."""
    ibe, jbe, ktf = _extent(g, var)
    kk = slice(0, field.shape[0] if ktf is None else ktf)
    ibs, jbs = g.ids, g.jds
    ys, tys, ye, tye = bd["ys"], bd["tys"], bd["ye"], bd["tye"]
    xs, txs, xe, txe = bd["xs"], bd["txs"], bd["xe"], bd["txe"]
    for b in (1, 2, 3):
        i0, i1 = ibs + b, ibe - b
        j = jbs + b
        fl = lambda bb, di, jj: ys[kk, bb, i0 + di:i1 + di] + dtbc * tys[kk, bb, i0 + di:i1 + di] - field[kk, jj, i0 + di:i1 + di]
        f0, f1, f2, f3, f4 = fl(b, 0, j), fl(b, -1, j), fl(b, 1, j), fl(b - 1, 0, j - 1), fl(b + 1, 0, j + 1)
        tend[kk, j, i0:i1] = tend[kk, j, i0:i1] + fcx[b] * f0 - gcx[b] * (f1 + f2 + f3 + f4 - 4.0 * f0)
    for b in (1, 2, 3):
        i0, i1 = ibs + b, ibe - b
        j = jbe - 1 - b
        fl = lambda bb, di, jj: ye[kk, bb, i0 + di:i1 + di] + dtbc * tye[kk, bb, i0 + di:i1 + di] - field[kk, jj, i0 + di:i1 + di]
        f0, f1, f2, f3, f4 = fl(b, 0, j), fl(b, -1, j), fl(b, 1, j), fl(b - 1, 0, j + 1), fl(b + 1, 0, j - 1)
        tend[kk, j, i0:i1] = tend[kk, j, i0:i1] + fcx[b] * f0 - gcx[b] * (f1 + f2 + f3 + f4 - 4.0 * f0)
    for b in (1, 2, 3):
        j0, j1 = jbs + b + 1, jbe - b - 1
        i = ibs + b
        fl = lambda bb, dj, ii: xs[kk, j0 + dj:j1 + dj, bb] + dtbc * txs[kk, j0 + dj:j1 + dj, bb] - field[kk, j0 + dj:j1 + dj, ii]
        f0, f1, f2, f3, f4 = fl(b, 0, i), fl(b, -1, i), fl(b, 1, i), fl(b - 1, 0, i - 1), fl(b + 1, 0, i + 1)
        tend[kk, j0:j1, i] = tend[kk, j0:j1, i] + fcx[b] * f0 - gcx[b] * (f1 + f2 + f3 + f4 - 4.0 * f0)
    for b in (1, 2, 3):
        j0, j1 = jbs + b + 1, jbe - b - 1
        i = ibe - 1 - b
        fl = lambda bb, dj, ii: xe[kk, j0 + dj:j1 + dj, bb] + dtbc * txe[kk, j0 + dj:j1 + dj, bb] - field[kk, j0 + dj:j1 + dj, ii]
        f0, f1, f2, f3, f4 = fl(b, 0, i), fl(b, -1, i), fl(b, 1, i), fl(b - 1, 0, i + 1), fl(b + 1, 0, i - 1)
        tend[kk, j0:j1, i] = tend[kk, j0:j1, i] + fcx[b] * f0 - gcx[b] * (f1 + f2 + f3 + f4 - 4.0 * f0)
    return tend


def spec_bdytend(g, tend, bd, var):
    """wrf_boundary.py:189-241: the specified row takes the boundary tendency."""
    ibe, jbe, ktf = _extent(g, var)
    kk = slice(0, tend.shape[0] if ktf is None else ktf)
    ibs, jbs = g.ids, g.jds
    tend[kk, jbs, ibs:ibe] = bd["tys"][kk, 0, ibs:ibe]
    tend[kk, jbe - 1, ibs:ibe] = bd["tye"][kk, 0, ibs:ibe]
    tend[kk, jbs:jbe, ibs] = bd["txs"][kk, jbs:jbe, 0]
    tend[kk, jbs:jbe, ibe - 1] = bd["txe"][kk, jbs:jbe, 0]
    return tend


def spec_bdyupdate(g, field, tend, dt, var):
    """wrf_boundary.py:244-294: field += dt * tend on the specified rows.
    ``var == 'm'`` takes 2-D fields."""
    ibe, jbe, _ = _extent(g, var)
    itf = g.ide if var == "u" else g.ide - 1
    jtf = g.jde if var == "v" else g.jde - 1
    two_d = field.ndim == 2
    f = field[None] if two_d else field
    t = tend[None] if two_d else tend
    kk = slice(0, 1) if two_d else slice(0, g.nz - 1)
    its, jts, jbs = g.its, g.jts, g.jds
    f[kk, jts, its:itf] = f[kk, jts, its:itf] + dt * t[kk, jts, its:itf]
    f[kk, jtf - 1, its:itf] = f[kk, jtf - 1, its:itf] + dt * t[kk, jtf - 1, its:itf]
    f[kk, jbs + 1:jbe - 1, its] = f[kk, jbs + 1:jbe - 1, its] + dt * t[kk, jbs + 1:jbe - 1, its]
    f[kk, jbs + 1:jbe - 1, itf - 1] = f[kk, jbs + 1:jbe - 1, itf - 1] + dt * t[kk, jbs + 1:jbe - 1, itf - 1]
    return field


def spec_bdyupdate_ph(g, ph_save, ph, ph_tend, mu_tend, muts, dt):
    """wrf_boundary.py:297-355: specified-row phi update with the mass
    re-weighting ``mu_old = muts - dt * mu_tend``."""
    ibs, ibe, jbs, jbe = g.ids, g.ide - 1, g.jds, g.jde - 1
    kk = slice(0, g.nz)
    jts = g.jts

    def upd(js, is_):
        mu_old = muts[js, is_] - dt * mu_tend[js, is_]
        mt = muts[js, is_]
        ph[kk, js, is_] = (ph[kk, js, is_] * mu_old[None] / mt[None] + dt * ph_tend[kk, js, is_] / mt[None]
                           + ph_save[kk, js, is_] * (mu_old[None] / mt[None] - 1.0))

    upd(jts, slice(ibs, ibe))
    upd(jbe - 1, slice(ibs, ibe))
    upd(slice(jbs + 1, jbe - 1), ibs)
    upd(slice(jbs + 1, jbe - 1), ibe - 1)
    return ph


def zero_grad_bdy(g, field, var):
    """wrf_boundary.py:358-400 (w: all levels)."""
    ibs, ibe, jbs, jbe = g.ids, g.ide - 1, g.jds, g.jde - 1
    if var == "u":
        ibe = g.ide
    if var == "v":
        jbe = g.jde
    kk = slice(0, g.nz if var == "w" else g.nz - 1)
    field[kk, jbs, ibs] = field[kk, jbs + 1, ibs + 1]
    field[kk, jbs, ibe - 1] = field[kk, jbs + 1, ibe - 2]
    field[kk, jbs, ibs + 1:ibe - 1] = field[kk, jbs + 1, ibs + 1:ibe - 1]
    field[kk, jbe - 1, ibs] = field[kk, jbe - 2, ibs + 1]
    field[kk, jbe - 1, ibe - 1] = field[kk, jbe - 2, ibe - 2]
    field[kk, jbe - 1, ibs + 1:ibe - 1] = field[kk, jbe - 2, ibs + 1:ibe - 1]
    field[kk, jbs + 1:jbe - 1, ibs] = field[kk, jbs + 1:jbe - 1, ibs + 1]
    field[kk, jbs + 1:jbe - 1, ibe - 1] = field[kk, jbs + 1:jbe - 1, ibe - 2]
    return field


def mass_weight(field, mut, rfield, ks, js, is_):
    """wrf_boundary.py:403-410: rfield = field * mut on the given region."""
    rfield[ks, js, is_] = field[ks, js, is_] * mut[None, js, is_]
    return rfield


def flow_dep_bdy(g, field, u, v):
    """wrf_boundary.py:470-508: zero inflow / zero-gradient outflow on the
    outermost row, using the averaged mass fluxes for the flow direction."""
    its, jts = g.its, g.jts
    itf, jtf = g.ide - 1, g.jde - 1
    kk = slice(0, g.nz - 1)
    field[kk, jts, its:itf] = np.where(v[kk, jts, its:itf] < 0.0, field[kk, jts + 1, its:itf], 0.0)
    field[kk, jts, its] = field[kk, jts + 1, its + 1]
    field[kk, jts, itf - 1] = field[kk, jts + 1, itf - 2]
    field[kk, jtf - 1, its:itf] = np.where(v[kk, jtf, its:itf] > 0.0, field[kk, jtf - 2, its:itf], 0.0)
    field[kk, jtf - 1, its] = field[kk, jtf - 2, its + 1]
    field[kk, jtf - 1, itf - 1] = field[kk, jtf - 2, itf - 2]
    field[kk, jts:jtf, its] = np.where(u[kk, jts:jtf, its] < 0.0, field[kk, jts:jtf, its + 1], 0.0)
    field[kk, jts, its] = field[kk, jts + 1, its + 1]
    field[kk, jtf - 1, its] = field[kk, jtf - 2, its + 1]
    field[kk, jts:jtf, itf - 1] = np.where(u[kk, jts:jtf, itf] > 0.0, field[kk, jts:jtf, itf - 2], 0.0)
    field[kk, jts, itf - 1] = field[kk, jts + 1, itf - 2]
    field[kk, jtf - 1, itf - 1] = field[kk, jtf - 2, itf - 2]
    return field


def spec_bdy_final(g, field, mu, msf, bd, var, dtbc):
    """wrf_boundary.py:511-587: specified-row values from the boundary file at
    the end of the step, de-coupled by mu (and msf for u, v, w)."""
    ibe = g.ide if var == "u" else g.ide - 1
    jbe = g.jde if var == "v" else g.jde - 1
    itf = g.ide if var == "u" else g.ide - 1
    jtf = g.jde if var == "v" else g.jde - 1
    ktf = g.nz if var in ("m", "h", "w") else g.nz - 1
    kk = slice(0, ktf)
    its, jts = g.its, g.jts
    msfc = var in ("u", "v", "w")
    muc = var != "m"
    xm = (lambda js, is_: msf[None, js, is_]) if msfc else (lambda js, is_: 1.0)
    xu = (lambda js, is_: mu[None, js, is_]) if muc else (lambda js, is_: 1.0)

    def put(js, is_, val, tnd):
        field[kk, js, is_] = xm(js, is_) * (val + dtbc * tnd) / xu(js, is_)

    put(jts, slice(its, ibe), bd["ys"][kk, 0, its:ibe], bd["tys"][kk, 0, its:ibe])
    put(jtf - 1, slice(its, ibe), bd["ye"][kk, 0, its:ibe], bd["tye"][kk, 0, its:ibe])
    put(slice(jts, jbe), its, bd["xs"][kk, jts:jbe, 0], bd["txs"][kk, jts:jbe, 0])
    put(slice(jts, jbe), itf - 1, bd["xe"][kk, jts:jbe, 0], bd["txe"][kk, jts:jbe, 0])
    return field
