"""Drop-ins for ``pywrf.wrf_physics.wsm6`` and ``microphysics_driver``
(reference signatures).

``wsm6(...)`` takes the arguments of the reference function
(pywrf/wrf_physics.py:137-151) and runs the scheme on the GPU through
``wrf_wsm6`` (include/pywrf_b200.h).  Tensors must be contiguous float32 CUDA
tensors of the allocation shape; there is no CPU path.  The physical constants
are those the scheme is built with (config_params.py:114-253); passing
different values raises.  The index arguments must describe the solver's
call, i.e. the tile ``[its, ite) x [jts, jte)`` = ``[ids+1, ide-1)`` (the
scheme then acts on ``[its, ite-1) x [jts, jte-1)``, levels ``[0, kte-1)``).
Returns the updated arrays in the reference's order; they alias the inputs.
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _native as N
from .config import Grid
from .state import make_cgrid

# the constants the microphysics driver passes (pywrf/config_params.py:121-161)
_CONSTANTS = dict(g=9.81, cpd=1004.5, cpv=1846.4, rd=287.0, rv=461.6, t0c=273.149993896484375,
                  ep1=0.608362436294555664, ep2=0.621750414371490479, qmin=1.0e-15, xls=2.85e6, xlv0=2.5e6,
                  xlf0=3.5e5, den0=1.28, denr=1000.0, cliq=4190.0, cice=2106.0, psat=610.78)


def _check_tensor(name, t, shape):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise TypeError(f"{name}: a contiguous float32 CUDA tensor is required (no CPU path)")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name}: shape {tuple(t.shape)} != {tuple(shape)}")


def _grid(nz, ny, nx, dt):
    g = Grid.make(nx, ny, nz, 9000.0, 9000.0, float(dt))
    return make_cgrid(g, {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0, "cfn1": 0.0})


def wsm6(th, q, qc, qr, qi, qs, qg, den, pii, p, delz, delt, g, cpd, cpv, rd, rv, t0c, ep1, ep2, qmin,
         xls, xlv0, xlf0, den0, denr, cliq, cice, psat, rain, rainncv, snow, snowncv, sr,
         refl_10cm, diagflag, do_radar_ref, graupel, graupelncv, has_reqc, has_reqi, has_reqs,
         re_cloud, re_ice, re_snow, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme,
         its, ite, jts, jte, kts, kte):
    """WSM6 (pywrf/wrf_physics.py:137-1214) on the GPU."""
    given = dict(g=g, cpd=cpd, cpv=cpv, rd=rd, rv=rv, t0c=t0c, ep1=ep1, ep2=ep2, qmin=qmin, xls=xls, xlv0=xlv0,
                 xlf0=xlf0, den0=den0, denr=denr, cliq=cliq, cice=cice, psat=psat)
    for k, v in given.items():
        if not math.isclose(float(v), _CONSTANTS[k], rel_tol=1e-5):
            raise ValueError(f"wsm6: constant {k}={v} differs from the built scheme's {_CONSTANTS[k]}")
    nz, ny, nx = th.shape
    # the solver's call: tile [ids+1, ide-1) with ide = nx - 5, ids = 5
    if (ids, jds) != (6, 6) or (ide, jde) != (nx - 6, ny - 6) or (its, ite, jts, jte) != (ids, ide, jds, jde) \
            or (kts, kte) != (0, nz):
        raise NotImplementedError("wsm6: only the solver's tile (ids+1, ide-1 of the 5-cell frame) is supported")
    fields = dict(th=th, q=q, qc=qc, qr=qr, qi=qi, qs=qs, qg=qg, den=den, pii=pii, p=p, delz=delz)
    for k, t in fields.items():
        _check_tensor(k, t, (nz, ny, nx))
    flat = dict(rain=rain, rainncv=rainncv, snow=snow, snowncv=snowncv, graupel=graupel, graupelncv=graupelncv, sr=sr)
    for k, t in flat.items():
        _check_tensor(k, t, (ny, nx))
    cg = _grid(nz, ny, nx, delt)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    with torch.cuda.device(th.device):
        rc = N.lib().wrf_wsm6(ctypes.byref(cg), *[ptr(fields[k]) for k in ("th", "q", "qc", "qr", "qi", "qs", "qg", "den",
                                                                          "pii", "p", "delz")],
                              ctypes.c_float(float(delt)),
                              *[ptr(flat[k]) for k in ("rain", "rainncv", "snow", "snowncv", "graupel", "graupelncv",
                                                       "sr")],
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, "wrf_wsm6")
    return th, q, qc, qr, qi, qs, qg, rain, rainncv, snow, snowncv, graupel, graupelncv, sr, refl_10cm


def microphysics_driver(th, rho, pi_phy, p, ht, dz8w, p8w, dt, dx, dy, qv_curr, qc_curr, qr_curr, qi_curr, qs_curr,
                        qg_curr, rainnc, rainncv, snownc, snowncv, sr, refl_10cm, diagflag, do_radar_ref, graupelnc,
                        graupelncv, has_reqc, has_reqi, has_reqs, re_cloud, re_ice, re_snow, ids, ide, jds, jde, kds,
                        kde, ims, ime, jms, jme, kms, kme, its, ite, jts, jte, kts, kte):
    """microphysics_driver (pywrf/wrf_physics.py:94-135): WSM6 with the
    driver's constants, on the GPU through :func:`wsm6`; returns what the
    reference returns (th, qv .. qg, the precipitation accumulators, sr,
    refl_10cm).  ht, p8w, dx and dy are accepted and unused, as in the
    reference."""
    c = _CONSTANTS
    return wsm6(th, qv_curr, qc_curr, qr_curr, qi_curr, qs_curr, qg_curr, rho, pi_phy, p, dz8w, dt, c["g"], c["cpd"],
                c["cpv"], c["rd"], c["rv"], c["t0c"], c["ep1"], c["ep2"], c["qmin"], c["xls"], c["xlv0"], c["xlf0"],
                c["den0"], c["denr"], c["cliq"], c["cice"], c["psat"], rainnc, rainncv, snownc, snowncv, sr,
                refl_10cm, diagflag, do_radar_ref, graupelnc, graupelncv, has_reqc, has_reqi, has_reqs, re_cloud,
                re_ice, re_snow, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, its, ite, jts, jte, kts,
                kte)
