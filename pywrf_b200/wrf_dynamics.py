"""Drop-ins for ``pywrf.wrf_dynamics.advect_scalar``, ``advect_u``,
``advect_v``, ``advect_w``, ``calc_coef_w``, ``calc_p_rho``,
``advance_mu_t`` and ``advance_w`` (reference signatures).

``advect_scalar(...)`` takes the arguments of the reference function
(pywrf/wrf_dynamics.py:1841-1850), adds the flux-form advection of ``field``
to ``tendency`` on the GPU through ``wrf_advect_scalar``
(include/pywrf_b200.h) and returns ``tendency``.  Tensors must be contiguous
float32 CUDA tensors; there is no CPU path.  The index arguments must be the
solver's (the 5-cell frame with tile = patch = domain); ``rdzw`` is the 1-D
``rdnw`` profile the solver passes, ``fzm``/``fzp`` the ``fnm``/``fnp``
profiles.  ``field_old``, ``c1``, ``c2``, ``mut``, ``time_step``, ``msfux``,
``msfuy``, ``msfvx`` and ``msfvy`` are accepted and unused, as in the reference
(its map-factor form uses ``msftx`` only).
"""
from __future__ import annotations

import ctypes

import torch

from . import _native as N
from .config import Grid
from .state import make_cgrid


def _need(name, t):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise TypeError(f"{name}: a contiguous float32 CUDA tensor is required (no CPU path)")
    return ctypes.c_void_p(t.data_ptr())


def advect_scalar(field, field_old, tendency, ru, rv, rom, c1, c2, mut, time_step, msfux, msfuy, msfvx, msfvy,
                  msftx, msfty, fzm, fzp, rdx, rdy, rdzw, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme,
                  kms, kme, its, ite, jts, jte, kts, kte):
    """advect_scalar (pywrf/wrf_dynamics.py:1841-2028) on the GPU."""
    nz, ny, nx = field.shape
    if (ids, jds, ide, jde) != (5, 5, nx - 5, ny - 5) or (its, ite, jts, jte) != (ids, ide, jds, jde) \
            or (kts, kte) != (0, nz):
        raise NotImplementedError("advect_scalar: only the solver's 5-cell frame with tile = domain is supported")
    for nm, t in (("tendency", tendency), ("ru", ru), ("rv", rv), ("rom", rom)):
        if tuple(t.shape) != (nz, ny, nx):
            raise ValueError(f"{nm}: shape {tuple(t.shape)} != {(nz, ny, nx)}")
    g = Grid.make(nx, ny, nz, 1.0 / float(rdx), 1.0 / float(rdy), 1.0)
    cg = make_cgrid(g, {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0, "cfn1": 0.0})
    # the kernels read rdx/rdy as float(1/dx): rebuild dx so that 1/dx == rdx
    cg.dx = 1.0 / float(rdx)
    cg.dy = 1.0 / float(rdy)
    with torch.cuda.device(field.device):
        rc = N.lib().wrf_advect_scalar(ctypes.byref(cg), _need("field", field), _need("tendency", tendency),
                                       _need("ru", ru), _need("rv", rv), _need("rom", rom), _need("msftx", msftx),
                                       _need("fzm", fzm), _need("fzp", fzp), _need("rdzw", rdzw),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, "wrf_advect_scalar")
    return tendency


def _check_frame(name, field, its, ite, jts, jte, kts, kte, ids, ide, jds, jde):
    nz, ny, nx = field.shape
    if (ids, jds, ide, jde) != (5, 5, nx - 5, ny - 5) or (its, ite, jts, jte) != (ids, ide, jds, jde) \
            or (kts, kte) != (0, nz):
        raise NotImplementedError(f"{name}: only the solver's 5-cell frame with tile = domain is supported")
    return nz, ny, nx


def _advect_momentum(component, field, tendency, ru, rv, rom, msf, msf2, fzm, fzp, rdx, rdy, rdz, form=0):
    """tendency += advection of one momentum component (0 u, 1 v, 2 w)
    through ``wrf_advect_momentum``; form 1 forces the one-thread-per-point
    kernel (the same operations as the tiled one)."""
    nz, ny, nx = field.shape
    for nm, t in (("tendency", tendency), ("ru", ru), ("rv", rv), ("rom", rom)):
        if tuple(t.shape) != (nz, ny, nx):
            raise ValueError(f"{nm}: shape {tuple(t.shape)} != {(nz, ny, nx)}")
    g = Grid.make(nx, ny, nz, 1.0 / float(rdx), 1.0 / float(rdy), 1.0)
    cg = make_cgrid(g, {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0, "cfn1": 0.0})
    cg.dx = 1.0 / float(rdx)
    cg.dy = 1.0 / float(rdy)
    with torch.cuda.device(field.device):
        rc = N.lib().wrf_advect_momentum(
            ctypes.byref(cg), int(component), _need("field", field), _need("tendency", tendency), _need("ru", ru),
            _need("rv", rv), _need("rom", rom), _need("msf", msf),
            _need("msf2", msf2) if msf2 is not None else None, _need("fzm", fzm), _need("fzp", fzp),
            _need("rdz", rdz), int(form), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, "wrf_advect_momentum")
    return tendency


def advect_u(u, u_old, tendency, ru, rv, rom, c1, c2, mut, time_step, msfux, msfuy, msfvx, msfvy, msftx, msfty,
             fzm, fzp, rdx, rdy, rdzw, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, its, ite, jts,
             jte, kts, kte):
    """advect_u (pywrf/wrf_dynamics.py:1112-1331) on the GPU: tendency +=
    the advection of u, returned.  u_old, c1, c2, mut, time_step and the map
    factors other than msfux are accepted and unused, as in the reference."""
    _check_frame("advect_u", u, its, ite, jts, jte, kts, kte, ids, ide, jds, jde)
    return _advect_momentum(0, u, tendency, ru, rv, rom, msfux, None, fzm, fzp, rdx, rdy, rdzw)


def advect_v(v, v_old, tendency, ru, rv, rom, c1, c2, mut, time_step, msfux, msfuy, msfvx, msfvy, msftx, msfty,
             fzm, fzp, rdx, rdy, rdzw, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, its, ite, jts,
             jte, kts, kte):
    """advect_v (pywrf/wrf_dynamics.py:1332-1534) on the GPU (map factors
    msfvy and msfvx)."""
    _check_frame("advect_v", v, its, ite, jts, jte, kts, kte, ids, ide, jds, jde)
    return _advect_momentum(1, v, tendency, ru, rv, rom, msfvy, msfvx, fzm, fzp, rdx, rdy, rdzw)


def advect_w(w, w_old, tendency, ru, rv, rom, c1, c2, mut, time_step, msfux, msfuy, msfvx, msfvy, msftx, msfty,
             fzm, fzp, rdx, rdy, rdzu, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, its, ite, jts,
             jte, kts, kte):
    """advect_w (pywrf/wrf_dynamics.py:1535-1823) on the GPU (map factor
    msftx; rdzu is the rdn profile the solver passes)."""
    _check_frame("advect_w", w, its, ite, jts, jte, kts, kte, ids, ide, jds, jde)
    return _advect_momentum(2, w, tendency, ru, rv, rom, msftx, None, fzm, fzp, rdx, rdy, rdzu)


def calc_coef_w(a, alpha, gamma, mut, c1h, c2h, c1f, c2f, c3h, c4h, c3f, c4f, cqw, rdn, rdnw, c2a, dts, g, epssm,
                top_lid, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, its, ite, jts, jte, kts, kte):
    """calc_coef_w (pywrf/wrf_dynamics.py:3316-3388) on the GPU through
    ``wrf_coef_w``: fills a, alpha, gamma on the mass columns and returns
    them.  The c1h..c4f arguments are accepted and unused, as in the
    reference; g must be the solver's 9.81."""
    nz, ny, nx = cqw.shape
    if (ids, jds, ide, jde) != (5, 5, nx - 5, ny - 5) or (its, ite, jts, jte) != (ids, ide, jds, jde) \
            or (kts, kte) != (0, nz):
        raise NotImplementedError("calc_coef_w: only the solver's 5-cell frame with tile = domain is supported")
    if abs(float(g) - 9.81) > 1e-6:
        raise ValueError("calc_coef_w: the kernels use the solver's g = 9.81")
    gr = Grid.make(nx, ny, nz, 9000.0, 9000.0, 1.0)
    cg = make_cgrid(gr, {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0, "cfn1": 0.0})
    cg.epssm = float(epssm)
    cg.top_lid = int(bool(top_lid))
    with torch.cuda.device(cqw.device):
        rc = N.lib().wrf_coef_w(ctypes.byref(cg), _need("mut", mut), _need("cqw", cqw), _need("c2a", c2a),
                                _need("rdn", rdn), _need("rdnw", rdnw), float(dts), _need("a", a),
                                _need("alpha", alpha), _need("gamma", gamma),
                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, "wrf_coef_w")
    return a, alpha, gamma


def _frame(name, shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte):
    nz, ny, nx = shape
    if (ids, jds, ide, jde) != (5, 5, nx - 5, ny - 5) or (its, ite, jts, jte) != (ids, ide, jds, jde) \
            or (kts, kte) != (0, nz):
        raise NotImplementedError(f"{name}: only the solver's 5-cell frame with tile = domain is supported")


def _state_call(fn_name, cg, named, *args):
    from .adjoint import _table  # the state-table builder shared with the adjoints

    dev = next(iter(named.values())).device
    with torch.cuda.device(dev):
        rc = getattr(N.lib(), fn_name)(ctypes.byref(cg), _table(named), *args,
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, fn_name)


def calc_p_rho(al_ori, p_ori, ph, alt, t_2, t_1, c2a, pm1, mu, mut, c1h, c2h, c1f, c2f, c3h, c4h, c3f, c4f, znu, t0,
               rdnw, dnw, smdiv, non_hydrostatic, step, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme,
               its, ite, jts, jte, kts, kte):
    """calc_p_rho (pywrf/wrf_dynamics.py:3269-3313) on the GPU through
    ``wrf_calc_p_rho``: returns new (al, p, pm1) like the reference - at step
    0 pm1 is a new copy of the new p, at a later step the caller's pm1 is
    updated in place and returned.  c1h..c4f, znu and dnw are accepted and
    unused, as in the reference; t0 must be the solver's 300."""
    _frame("calc_p_rho", p_ori.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    if abs(float(t0) - 300.0) > 1e-9:
        raise ValueError("calc_p_rho: the kernels use the solver's t0 = 300")
    nz, ny, nx = p_ori.shape
    cg = make_cgrid(Grid.make(nx, ny, nz, 9000.0, 9000.0, 1.0), {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0,
                                                                 "cfn1": 0.0})
    cg.smdiv = float(smdiv)
    al, p = al_ori.clone(), p_ori.clone()
    pm1_out = torch.empty_like(p) if int(step) == 0 else pm1
    _state_call("wrf_calc_p_rho", cg, {"al": al, "p": p, "ph": ph, "alt": alt, "t": t_2, "t_save": t_1, "c2a": c2a,
                                       "pm1": pm1_out, "mu": mu, "muts": mut, "rdnw": rdnw}, int(step))
    return al, p, pm1_out


def advance_mu_t(ww_ori, ww_1, u, u_1, v, v_1, mu_ori, mut, muave_ori, muts_ori, muu, muv, mudf_ori, c1h, c2h, c1f,
                 c2f, c3h, c4h, c3f, c4f, uam, vam, wwam, t_ori, t_1, t_ave_ori, ft, mu_tend, rdx, rdy, dts, epssm,
                 dnw, fnm, fnp, rdnw, msfux, msfuy, msfvx, msfvx_inv, msfvy, msftx, msfty, step, ids, ide, jds, jde,
                 kds, kde, ims, ime, jms, jme, kms, kme, its, ite, jts, jte, kts, kte):
    """advance_mu_t (pywrf/wrf_dynamics.py:3528-3638) on the GPU through
    ``wrf_advance_mu_t``: returns (ww, ww_1, t, t_ave, uam, vam, wwam, muave,
    muts, mudf, mu) like the reference, the updated ones as new tensors.
    c1h..c4f, msfux, msfvx, msfvy and step are accepted and unused, as in the
    reference."""
    _frame("advance_mu_t", ww_ori.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    nz, ny, nx = ww_ori.shape
    cg = make_cgrid(Grid.make(nx, ny, nz, 1.0 / float(rdx), 1.0 / float(rdy), 1.0),
                    {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0, "cfn1": 0.0})
    cg.dx, cg.dy = 1.0 / float(rdx), 1.0 / float(rdy)
    cg.epssm = float(epssm)
    ww, t, t_ave = ww_ori.clone(), t_ori.clone(), t_ave_ori.clone()
    mu, muave, muts, mudf = mu_ori.clone(), muave_ori.clone(), muts_ori.clone(), mudf_ori.clone()
    _state_call("wrf_advance_mu_t", cg, {
        "ww": ww, "ww1": ww_1, "u": u, "u_save": u_1, "v": v, "v_save": v_1, "mu": mu, "mut": mut, "muave": muave,
        "muts": muts, "muu": muu, "muv": muv, "mudf": mudf, "t": t, "t_save": t_1, "t_2save": t_ave, "t_tend": ft,
        "mu_tend": mu_tend, "dnw": dnw, "fnm": fnm, "fnp": fnp, "rdnw": rdnw, "msfuy": msfuy,
        "msfvx_inv": msfvx_inv, "msftx": msftx, "msfty": msfty}, float(dts))
    return ww, ww_1, t, t_ave, uam, vam, wwam, muave, muts, mudf, mu


def advance_w(w_ori, rw_tend, ww, w_save, u, v, mu1, mut, muave, muts, c1h, c2h, c1f, c2f, c3h, c4h, c3f, c4f,
              t_2ave_ori, t_2, t_1, ph_ori, ph_1, phb, ph_tend, ht, c2a, cqw, alt, alb, a, alpha, gamma, rdx, rdy,
              dts, t0, epssm, dnw, fnm, fnp, rdnw, rdn, cf1, cf2, cf3, msftx, msfty, top_lid, ids, ide, jds, jde,
              kds, kde, ims, ime, jms, jme, kms, kme, its, ite, jts, jte, kts, kte):
    """advance_w (pywrf/wrf_dynamics.py:3641-3796) on the GPU through
    ``wrf_advance_w``: returns new (t_2ave, w, ph) like the reference.  mu1,
    c1h..c4f, alb, dnw and top_lid are accepted and unused, as in the
    reference; t0 must be the solver's 300."""
    _frame("advance_w", w_ori.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    if abs(float(t0) - 300.0) > 1e-9:
        raise ValueError("advance_w: the kernels use the solver's t0 = 300")
    nz, ny, nx = w_ori.shape
    cg = make_cgrid(Grid.make(nx, ny, nz, 1.0 / float(rdx), 1.0 / float(rdy), 1.0),
                    {"cf1": float(cf1), "cf2": float(cf2), "cf3": float(cf3), "cfn": 0.0, "cfn1": 0.0})
    cg.dx, cg.dy = 1.0 / float(rdx), 1.0 / float(rdy)
    cg.epssm = float(epssm)
    cg.cf1, cg.cf2, cg.cf3 = float(cf1), float(cf2), float(cf3)
    w, ph, t_2ave = w_ori.clone(), ph_ori.clone(), t_2ave_ori.clone()
    _state_call("wrf_advance_w", cg, {
        "w": w, "rw_tend": rw_tend, "ww": ww, "w_save": w_save, "u": u, "v": v, "muave": muave, "muts": muts,
        "mut": mut, "t_2save": t_2ave, "t": t_2, "t_save": t_1, "ph": ph, "ph_save": ph_1, "phb": phb,
        "ph_tend": ph_tend, "ht": ht, "c2a": c2a, "cqw": cqw, "alt": alt, "a": a, "alpha": alpha, "gamma": gamma,
        "msftx": msftx, "msfty": msfty, "fnm": fnm, "fnp": fnp, "rdnw": rdnw, "rdn": rdn}, float(dts))
    return t_2ave, w, ph
