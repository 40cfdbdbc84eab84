"""Drop-ins for functions of ``pywrf.wrf_dynamics`` (reference signatures):
``advect_scalar``, ``advect_u``, ``advect_v``, ``advect_w``, ``rhs_ph``,
``horizontal_pressure_gradient``, ``pg_buoy_w``, ``coriolis``,
``curvature``, ``horizontal_diffusion``, ``horizontal_diffusion_3dmp``,
``rk_addtend_dry``, ``advance_uv``, ``calc_coef_w``, ``calc_p_rho``,
``advance_mu_t``, ``advance_w``, ``sumflux``, ``calc_p_rho_phi``,
``set_physical_bc3d`` and ``set_physical_bc2d``.  Each checks that it is
given the solver's 5-cell frame with tile = domain and raises
NotImplementedError otherwise (the library kernels are built for that
frame); arguments the reference accepts without using are accepted and
unused.

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


# ---- the large-step tendency terms, the flux averages, the first stage's
# diffusion, rk_addtend_dry, the halo copies and the equation of state ----

def _grid_like(shape, rdx=1.0 / 9000.0, rdy=1.0 / 9000.0, dt=1.0, **scal):
    nz, ny, nx = shape
    cg = make_cgrid(Grid.make(nx, ny, nz, 1.0 / float(rdx), 1.0 / float(rdy), float(dt)),
                    {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0, "cfn1": 0.0})
    cg.dx, cg.dy = 1.0 / float(rdx), 1.0 / float(rdy)
    for k, v in scal.items():
        setattr(cg, k, float(v))
    return cg


# the state-table operands of wrf_forces by kind (3-D, 2-D, 1-D profile)
_FORCES_3D = ("ph_tend", "ru_tend", "rv_tend", "rw_tend", "cqw", "u", "v", "w", "ww", "ph", "phb", "alt", "p", "pb",
              "al", "php", "cqu", "cqv", "ru", "rv", "rw")
_FORCES_2D = ("mut", "muu", "muv", "mu", "mub", "msfux", "msfuy", "msfvx", "msfvy", "msftx", "msfty", "f", "e",
              "sina", "cosa")
_FORCES_1D = ("fnm", "fnp", "rdnw", "rdn")


def _forces(terms, shape, named, **scal):
    """wrf_forces with the mask ``terms`` on the named operands; the operands
    the selected terms do not touch are filled with zero arrays."""
    nz, ny, nx = shape
    dev = next(iter(named.values())).device
    for k, t in named.items():
        _need(k, t)
    full = dict(named)
    z3 = z2 = z1 = None
    for k in _FORCES_3D + _FORCES_2D + _FORCES_1D:
        if k in full:
            continue
        if k in _FORCES_3D:
            z3 = torch.zeros(nz, ny, nx, device=dev) if z3 is None else z3
            full[k] = z3
        elif k in _FORCES_2D:
            z2 = torch.zeros(ny, nx, device=dev) if z2 is None else z2
            full[k] = z2
        else:
            z1 = torch.zeros(nz, device=dev) if z1 is None else z1
            full[k] = z1
    _state_call("wrf_forces", _grid_like(shape, **scal), full, int(terms))


def rhs_ph(ph_tend, u, v, ww, ph, ph_old, phb, w, mut, muuf, muvf, c1f, c2f, fnm, fnp, rdnw, cfn, cfn1, rdx, rdy,
           msfux, msfuy, msfvx, msfvx_inv, msfvy, msftx, msfty, non_hydrostatic, ids, ide, jds, jde, kds, kde, ims,
           ime, jms, jme, kms, kme, its, ite, jts, jte, kts, kte):
    """rhs_ph (pywrf/wrf_dynamics.py:2031-2297) on the GPU through
    ``wrf_forces``: ph_tend is updated in place and returned, as in the
    reference.  ph_old, c1f, c2f, msfuy, msfvx, msfvx_inv, msftx and
    non_hydrostatic are accepted and unused, as in the reference."""
    _frame("rhs_ph", ph_tend.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    _forces(1, ph_tend.shape, {"ph_tend": ph_tend, "u": u, "v": v, "ww": ww, "ph": ph, "phb": phb, "w": w,
                               "mut": mut, "muu": muuf, "muv": muvf, "fnm": fnm, "fnp": fnp, "rdnw": rdnw,
                               "msfux": msfux, "msfvy": msfvy, "msfty": msfty},
            rdx=rdx, rdy=rdy, cfn=cfn, cfn1=cfn1)
    return ph_tend


def horizontal_pressure_gradient(ru_tend, rv_tend, ph, alt, p, pb, al, php, cqu, cqv, muu, muv, mu, c1h, c2h, fnm,
                                 fnp, rdnw, cf1, cf2, cf3, cfn, cfn1, rdx, rdy, msfux, msfuy, msfvx, msfvy, msftx,
                                 msfty, non_hydrostatic, top_lid, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme,
                                 kms, kme, its, ite, jts, jte, kts, kte):
    """horizontal_pressure_gradient (pywrf/wrf_dynamics.py:2300-2421) on the
    GPU through ``wrf_forces``: ru_tend and rv_tend are updated in place and
    returned.  c1h, c2h, cfn, cfn1, msftx, msfty, non_hydrostatic and
    top_lid are accepted and unused, as in the reference."""
    _frame("horizontal_pressure_gradient", ru_tend.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    _forces(2, ru_tend.shape, {"ru_tend": ru_tend, "rv_tend": rv_tend, "ph": ph, "alt": alt, "p": p, "pb": pb,
                               "al": al, "php": php, "cqu": cqu, "cqv": cqv, "muu": muu, "muv": muv, "mu": mu,
                               "fnm": fnm, "fnp": fnp, "rdnw": rdnw, "msfux": msfux, "msfuy": msfuy,
                               "msfvx": msfvx, "msfvy": msfvy},
            rdx=rdx, rdy=rdy, cf1=cf1, cf2=cf2, cf3=cf3)
    return ru_tend, rv_tend


def pg_buoy_w(rw_tend, p, cqw, muf, mubf, c1f, c2f, rdnw, rdn, g, msftx, msfty, ids, ide, jds, jde, kds, kde, ims,
              ime, jms, jme, kms, kme, its, ite, jts, jte, kts, kte):
    """pg_buoy_w (pywrf/wrf_dynamics.py:2424-2460) on the GPU through
    ``wrf_forces``: rw_tend and cqw (which becomes 1 / (1 + cqw) on levels 1
    .. nz-2) are updated in place and returned.  g must be the built 9.81;
    c1f, c2f and msftx are accepted and unused, as in the reference."""
    _frame("pg_buoy_w", rw_tend.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    if abs(float(g) - 9.81) > 1e-9:
        raise ValueError("pg_buoy_w: the kernels use g = 9.81")
    _forces(4, rw_tend.shape, {"rw_tend": rw_tend, "p": p, "cqw": cqw, "mu": muf, "mub": mubf, "rdnw": rdnw,
                               "rdn": rdn, "msfty": msfty})
    return rw_tend, cqw


def coriolis(ru, rv, rw, ru_tend, rv_tend, rw_tend, msftx, msfty, msfux, msfuy, msfvx, msfvy, f, e, sina, cosa, fzm,
             fzp, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, its, ite, jts, jte, kts, kte):
    """coriolis (pywrf/wrf_dynamics.py:2463-2532) on the GPU through
    ``wrf_forces``: ru_tend, rv_tend and rw_tend are updated in place and
    returned."""
    _frame("coriolis", ru_tend.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    _forces(8, ru_tend.shape, {"ru": ru, "rv": rv, "rw": rw, "ru_tend": ru_tend, "rv_tend": rv_tend,
                               "rw_tend": rw_tend, "msftx": msftx, "msfty": msfty, "msfux": msfux, "msfuy": msfuy,
                               "msfvx": msfvx, "msfvy": msfvy, "f": f, "e": e, "sina": sina, "cosa": cosa,
                               "fnm": fzm, "fnp": fzp})
    return ru_tend, rv_tend, rw_tend


def curvature(ru, rv, rw, u, v, w, ru_tend, rv_tend, rw_tend, msfux, msfuy, msfvx, msfvy, msftx, msfty, xlat, fzm,
              fzp, rdx, rdy, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, its, ite, jts, jte, kts,
              kte):
    """curvature (pywrf/wrf_dynamics.py:2535-2620) on the GPU through
    ``wrf_forces``: ru_tend, rv_tend and rw_tend are updated in place and
    returned.  xlat is accepted and unused, as in the reference."""
    _frame("curvature", ru_tend.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    _forces(16, ru_tend.shape, {"ru": ru, "rv": rv, "rw": rw, "u": u, "v": v, "w": w, "ru_tend": ru_tend,
                                "rv_tend": rv_tend, "rw_tend": rw_tend, "msfux": msfux, "msfuy": msfuy,
                                "msfvx": msfvx, "msfvy": msfvy, "msftx": msftx, "msfty": msfty, "fnm": fzm,
                                "fnp": fzp},
            rdx=rdx, rdy=rdy)
    return ru_tend, rv_tend, rw_tend


def sumflux(ru, rv, ww, u_lin, v_lin, ww_lin, muu, muv, c1h, c2h, c1f, c2f, c3h, c4h, c3f, c4f, ru_m, rv_m, ww_m,
            epssm, msfux, msfuy, msfvx, msfvx_inv, msfvy, iteration, number_of_small_timesteps, ids, ide, jds, jde,
            kds, kde, ims, ime, jms, jme, kms, kme, its, ite, jts, jte, kts, kte):
    """sumflux (pywrf/wrf_dynamics.py:3799-3841) on the GPU through
    ``wrf_sumflux``: ru_m, rv_m and ww_m are updated in place and returned.
    c1h..c4f, epssm, msfux, msfvx and msfvy are accepted and unused, as in
    the reference."""
    _frame("sumflux", ru.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    named = {"u": ru, "v": rv, "ww": ww, "u_save": u_lin, "v_save": v_lin, "ww1": ww_lin, "muu": muu, "muv": muv,
             "ru_m": ru_m, "rv_m": rv_m, "ww_m": ww_m, "msfuy": msfuy, "msfvx_inv": msfvx_inv}
    for k, t in named.items():
        _need(k, t)
    _state_call("wrf_sumflux", _grid_like(ru.shape), named, int(iteration), int(number_of_small_timesteps))
    return ru_m, rv_m, ww_m


def _hdiff(fn, name, field, tendency, mut, base, msfux, msfuy, msfvx, msfvx_inv, msfvy, msftx, msfty, xkmhd, rdx, rdy):
    var = {"u": "u", "v": "v", "w": "w"}.get(str(name).lower(), "m")
    maps = {"msfux": msfux, "msfuy": msfuy, "msfvx": msfvx, "msfvy": msfvy, "msftx": msftx, "msfty": msfty,
            "msfvx_inv": msfvx_inv}
    for k, t in list(maps.items()) + [("field", field), ("tendency", tendency), ("mut", mut), ("xkmhd", xkmhd)]:
        _need(k, t)
    from .adjoint import _table

    cg = _grid_like(field.shape, rdx, rdy)
    with torch.cuda.device(field.device):
        rc = N.lib().wrf_horizontal_diffusion(ctypes.byref(cg), _table(maps), var.encode(), _need("field", field),
                                              None if base is None else _need("base", base), _need("mut", mut),
                                              _need("xkmhd", xkmhd), _need("tendency", tendency),
                                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, fn)
    return tendency


def horizontal_diffusion(name, field, tendency, mut, c1, c2, msfux, msfuy, msfvx, msfvx_inv, msfvy, msftx, msfty,
                         khdif, xkmhd, rdx, rdy, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, its,
                         ite, jts, jte, kts, kte):
    """horizontal_diffusion (pywrf/wrf_dynamics.py:2623-2838) on the GPU
    through ``wrf_horizontal_diffusion``: tendency is updated in place and
    returned; name 'u', 'v', 'w' or any other (a mass-point scalar).  c1, c2
    and khdif are accepted and unused, as in the reference."""
    _frame("horizontal_diffusion", field.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    return _hdiff("wrf_horizontal_diffusion", name, field, tendency, mut, None, msfux, msfuy, msfvx, msfvx_inv,
                  msfvy, msftx, msfty, xkmhd, rdx, rdy)


def horizontal_diffusion_3dmp(name, field, tendency, mut, c1, c2, base_3d, msfux, msfuy, msfvx, msfvx_inv, msfvy,
                              msftx, msfty, khdif, xkmhd, rdx, rdy, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme,
                              kms, kme, its, ite, jts, jte, kts, kte):
    """horizontal_diffusion_3dmp (pywrf/wrf_dynamics.py:2841-2915): the
    diffusion of field - base_3d, a mass-point scalar, on the GPU through
    ``wrf_horizontal_diffusion``; tendency is updated in place and returned.
    name, c1, c2 and khdif are accepted and unused, as in the reference."""
    _frame("horizontal_diffusion_3dmp", field.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    return _hdiff("wrf_horizontal_diffusion", "m", field, tendency, mut, base_3d, msfux, msfuy, msfvx, msfvx_inv,
                  msfvy, msftx, msfty, xkmhd, rdx, rdy)


def rk_addtend_dry(ru_tend, rv_tend, rw_tend, ph_tend, t_tend, ru_tendf, rv_tendf, rw_tendf, ph_tendf, t_tendf,
                   u_save, v_save, w_save, ph_save, t_save, mu_tend, mu_tendf, rk_step, c1, c2, h_diabatic, mut,
                   msftx, msfty, msfux, msfuy, msfvx, msfvx_inv, msfvy, ids, ide, jds, jde, kds, kde, ims, ime, jms,
                   jme, kms, kme, ips, ipe, jps, jpe, kps, kpe, its, ite, jts, jte, kts, kte):
    """rk_addtend_dry (pywrf/wrf_dynamics.py:3100-3148) on the GPU through
    ``wrf_addtend``: the tendencies (and at rk_step 1 the physics tendencies)
    are updated in place; returns (ru_tend, rv_tend, rw_tend, ph_tend,
    t_tend, mu_tend) like the reference.  c1, c2, msftx, msfux and msfvy are
    accepted and unused, as in the reference."""
    _frame("rk_addtend_dry", ru_tend.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    named = {"ru_tend": ru_tend, "rv_tend": rv_tend, "rw_tend": rw_tend, "ph_tend": ph_tend, "t_tend": t_tend,
             "mu_tend": mu_tend, "ru_tendf": ru_tendf, "rv_tendf": rv_tendf, "rw_tendf": rw_tendf,
             "ph_tendf": ph_tendf, "t_tendf": t_tendf, "mu_tendf": mu_tendf, "u_save": u_save, "v_save": v_save,
             "w_save": w_save, "ph_save": ph_save, "t_save": t_save, "h_diabatic": h_diabatic, "mut": mut,
             "msfty": msfty, "msfuy": msfuy, "msfvx": msfvx, "msfvx_inv": msfvx_inv}
    for k, t in named.items():
        _need(k, t)
    _state_call("wrf_addtend", _grid_like(ru_tend.shape), named, int(rk_step))
    return ru_tend, rv_tend, rw_tend, ph_tend, t_tend, mu_tend


def _halo(fn, dat, variable_in, two_d):
    _need("dat", dat)
    shape = (12,) + tuple(dat.shape) if two_d else tuple(dat.shape)
    with torch.cuda.device(dat.device):
        rc = N.lib().wrf_halo(ctypes.byref(_grid_like(shape)), _need("dat", dat), str(variable_in).encode(),
                              1 if two_d else 0, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, fn)
    return dat


def set_physical_bc3d(dat, variable_in, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, ips, ipe, jps,
                      jpe, kps, kpe, its, ite, jts, jte, kts, kte):
    """set_physical_bc3d (pywrf/wrf_dynamics.py:216-278), the open-boundary
    halo copies of one 3-D field for a stagger letter, on the GPU through
    ``wrf_halo``: dat is updated in place and returned."""
    _frame("set_physical_bc3d", dat.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    return _halo("wrf_halo", dat, variable_in, False)


def set_physical_bc2d(dat, variable_in, ids, ide, jds, jde, ims, ime, jms, jme, ips, ipe, jps, jpe, its, ite, jts,
                      jte):
    """set_physical_bc2d (pywrf/wrf_dynamics.py:164-213) of one 2-D field on
    the GPU through ``wrf_halo``: dat is updated in place and returned."""
    ny, nx = dat.shape
    if (ids, jds, ide, jde) != (5, 5, nx - 5, ny - 5) or (its, ite, jts, jte) != (ids, ide, jds, jde):
        raise NotImplementedError("set_physical_bc2d: only the solver's 5-cell frame with tile = domain is supported")
    return _halo("wrf_halo", dat, variable_in, True)


def calc_p_rho_phi(moist, n_moist, hypsometric_opt, al, alb, mu, muts, c1, c2, c3h, c4h, c3f, c4f, ph, phb, p, pb, t,
                   p0, t0, ptop, znu, znw, dnw, rdnw, rdn, non_hydrostatic, ids, ide, jds, jde, kds, kde, ims, ime,
                   jms, jme, kms, kme, its, ite, jts, jte, kts, kte):
    """calc_p_rho_phi (pywrf/wrf_dynamics.py:4124-4164) on the GPU through
    ``wrf_calc_p_rho_phi``: al and p are updated in place; returns (al, p,
    ph) like the reference.  moist is the [n_moist][nz][ny][nx] array (qv in
    slot 1); p0 and t0 must be the solver's 1e5 and 300; the other scalars
    and profiles are accepted and unused, as in the reference."""
    _frame("calc_p_rho_phi", al.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    if abs(float(p0) - 1.0e5) > 1e-6 or abs(float(t0) - 300.0) > 1e-9:
        raise ValueError("calc_p_rho_phi: the kernels use p0 = 1e5 and t0 = 300")
    if moist.dim() != 4 or moist.shape[0] < 2 or tuple(moist.shape[1:]) != tuple(al.shape):
        raise ValueError("calc_p_rho_phi: moist must be [n_moist][nz][ny][nx] with qv in slot 1")
    status = torch.zeros(16, dtype=torch.int32, device=al.device)
    named = {"al": al, "alb": alb, "mu": mu, "muts": muts, "ph": ph, "p": p, "pb": pb, "t": t, "moist": moist,
             "rdnw": rdnw}
    for k, v in named.items():
        _need(k, v)
    from .adjoint import _table

    tab = _table(named)
    tab[N.field_names().index("status")] = status.data_ptr()
    with torch.cuda.device(al.device):
        rc = N.lib().wrf_calc_p_rho_phi(ctypes.byref(_grid_like(al.shape)), tab,
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, "wrf_calc_p_rho_phi")
    return al, p, ph


def advance_uv(u_ori, ru_tend, v_ori, rv_tend, p, pb, ph, php, alt, al, mu, muu, cqu, muv, cqv, mudf, c1h, c2h, c1f,
               c2f, c3h, c4h, c3f, c4f, msfux, msfuy, msfvx, msfvx_inv, msfvy, rdx, rdy, dts, cf1, cf2, cf3, fnm, fnp,
               emdiv, rdnw, spec_zone, non_hydrostatic, top_lid, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme,
               kms, kme, its, ite, jts, jte, kts, kte):
    """advance_uv (pywrf/wrf_dynamics.py:3391-3525) on the GPU through
    ``wrf_advance_uv``: returns new (u, v) like the reference.  The library
    entry also applies the spec_bdyupdate of u and v that follows advance_uv
    in the acoustic substep; the points advance_uv itself leaves alone (the
    specified rows among them) keep u_ori's and v_ori's values.  spec_zone
    must be 1;
    c1h..c4f, non_hydrostatic and top_lid are accepted and unused, as in the
    reference."""
    _frame("advance_uv", u_ori.shape, ids, ide, jds, jde, its, ite, jts, jte, kts, kte)
    if int(spec_zone) != 1:
        raise NotImplementedError("advance_uv: only spec_zone 1 is supported")
    cg = _grid_like(u_ori.shape, rdx, rdy, cf1=cf1, cf2=cf2, cf3=cf3, emdiv=emdiv)
    u, v = u_ori.clone(), v_ori.clone()
    named = {"u": u, "v": v, "ru_tend": ru_tend, "rv_tend": rv_tend, "p": p, "pb": pb, "ph": ph, "php": php,
             "alt": alt, "al": al, "mu": mu, "muu": muu, "muv": muv, "cqu": cqu, "cqv": cqv, "mudf": mudf,
             "msfux": msfux, "msfuy": msfuy, "msfvx": msfvx, "msfvx_inv": msfvx_inv, "msfvy": msfvy, "fnm": fnm,
             "fnp": fnp, "rdnw": rdnw}
    for k, t in named.items():
        _need(k, t)
    _state_call("wrf_advance_uv", cg, named, float(dts))
    # advance_uv itself updates u on [jds+1, jde-2) x [ids+1, ide-1) and v on
    # [jds+1, jde-1) x [ids+1, ide-2), levels below nz-1; every other point
    # keeps the incoming value
    nz = u_ori.shape[0]
    u_out, v_out = u_ori.clone(), v_ori.clone()
    u_out[:nz - 1, jds + 1:jde - 2, ids + 1:ide - 1] = u[:nz - 1, jds + 1:jde - 2, ids + 1:ide - 1]
    v_out[:nz - 1, jds + 1:jde - 1, ids + 1:ide - 2] = v[:nz - 1, jds + 1:jde - 1, ids + 1:ide - 2]
    return u_out, v_out
