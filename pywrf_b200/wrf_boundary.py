"""Drop-ins for ``pywrf.wrf_boundary.relax_bdytend``, ``spec_bdytend``,
``spec_bdyupdate``, ``spec_bdyupdate_ph`` and ``zero_grad_bdy`` (reference
signatures; the solver's frame and zone widths only).

``relax_bdytend(...)`` takes the arguments of the reference function
(pywrf/wrf_boundary.py:52-63), adds the lateral-boundary relaxation of
``field`` to ``field_tend`` on the GPU through ``wrf_relax_bdytend``
(include/pywrf_b200.h) and returns ``field_tend``.  Tensors must be
contiguous float32 CUDA tensors (no CPU path); the boundary arrays are in the
solver's permuted layout (x sides [nz, ny, 5], y sides [nz, 5, nx],
pywrf/solver.py:468-482).  The zone widths and the fcx / gcx weights must be
the solver's (spec_bdy_width 5, spec_zone 1, relax_zone 4;
pywrf/solver.py:440-441): the kernels hold those weights.
"""
from __future__ import annotations

import ctypes

import torch

from . import _native as N
from .config import Grid
from .state import make_cgrid

FCX = (0.0, 5.5555557e-3, 3.7037039e-3, 1.8518519e-3, 0.0)
GCX = (0.0, 1.1111111e-3, 7.4074074e-4, 3.7037037e-4, 0.0)


def _ptr(name, t):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise TypeError(f"{name}: a contiguous float32 CUDA tensor is required (no CPU path)")
    return t.data_ptr()


def relax_bdytend(field, field_tend, field_bdy_xs, field_bdy_xe, field_bdy_ys, field_bdy_ye, field_bdy_tend_xs,
                  field_bdy_tend_xe, field_bdy_tend_ys, field_bdy_tend_ye, variable_in, spec_bdy_width, spec_zone,
                  relax_zone, dtbc, fcx, gcx, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, ips, ipe,
                  jps, jpe, kps, kpe, its, ite, jts, jte, kts, kte):
    """relax_bdytend (pywrf/wrf_boundary.py:52-147) on the GPU."""
    nz, ny, nx = field.shape
    if (ids, jds, ide, jde) != (5, 5, nx - 5, ny - 5) or (its, ite, jts, jte) != (ids, ide, jds, jde) \
            or (kts, kte) != (0, nz):
        raise NotImplementedError("relax_bdytend: only the solver's 5-cell frame with tile = domain is supported")
    if (spec_bdy_width, spec_zone, relax_zone) != (5, 1, 4):
        raise NotImplementedError("relax_bdytend: only spec_bdy_width 5, spec_zone 1, relax_zone 4 are supported")
    for name, w, ref in (("fcx", fcx, FCX), ("gcx", gcx, GCX)):
        vals = [float(x) for x in w]
        if len(vals) != 5 or any(abs(a - b) > 1e-9 for a, b in zip(vals, ref)):
            raise ValueError(f"relax_bdytend: {name} must be the solver's weights {ref}")
    if tuple(field_tend.shape) != (nz, ny, nx):
        raise ValueError(f"field_tend: shape {tuple(field_tend.shape)} != {(nz, ny, nx)}")
    bdy = (field_bdy_xs, field_bdy_xe, field_bdy_ys, field_bdy_ye, field_bdy_tend_xs, field_bdy_tend_xe,
           field_bdy_tend_ys, field_bdy_tend_ye)
    arr = (ctypes.c_void_p * 8)(*[_ptr(f"bdy[{i}]", b) for i, b in enumerate(bdy)])
    g = Grid.make(nx, ny, nz, 9000.0, 9000.0, 1.0)
    cg = make_cgrid(g, {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0, "cfn1": 0.0})
    with torch.cuda.device(field.device):
        rc = N.lib().wrf_relax_bdytend(ctypes.byref(cg), _ptr("field", field), _ptr("field_tend", field_tend), arr,
                                       str(variable_in).encode(), float(dtbc),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, "wrf_relax_bdytend")
    return field_tend


def _frame_b(name, shape, ids, ide, jds, jde, its, ite, jts, jte):
    ny, nx = shape[-2], shape[-1]
    if (ids, jds, ide, jde) != (5, 5, nx - 5, ny - 5) or (its, ite, jts, jte) != (ids, ide, jds, jde):
        raise NotImplementedError(f"{name}: only the solver's 5-cell frame with tile = domain is supported")


def _cgrid(shape):
    nz, ny, nx = (12,) + tuple(shape) if len(shape) == 2 else tuple(shape)
    return make_cgrid(Grid.make(nx, ny, nz, 9000.0, 9000.0, 1.0), {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0,
                                                                 "cfn1": 0.0})


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def spec_bdytend(field_tend, field_bdy_xs, field_bdy_xe, field_bdy_ys, field_bdy_ye, field_bdy_tend_xs,
                 field_bdy_tend_xe, field_bdy_tend_ys, field_bdy_tend_ye, variable_in, spec_bdy_width, spec_zone, ids,
                 ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, ips, ipe, jps, jpe, kps, kpe, its, ite, jts, jte,
                 kts, kte):
    """spec_bdytend (pywrf/wrf_boundary.py:188-241) on the GPU through
    ``wrf_spec_bdytend``: the specified rows of field_tend take the boundary
    tendency (the solver's permuted layout); updated in place and returned.
    variable_in 'u', 'v', 't' (or 'q'), 'h', or 'm' with a 2-D field_tend;
    the boundary values are accepted and unused, as in the reference."""
    _frame_b("spec_bdytend", field_tend.shape, ids, ide, jds, jde, its, ite, jts, jte)
    if (spec_bdy_width, spec_zone) != (5, 1):
        raise NotImplementedError("spec_bdytend: only spec_bdy_width 5, spec_zone 1 are supported")
    var = str(variable_in).lower()
    var = "t" if var == "q" else var
    if (var == "m") != (field_tend.dim() == 2):
        raise ValueError("spec_bdytend: 'm' takes a 2-D field_tend, the other letters 3-D")
    bt = [_ptr(n, t) for n, t in (("field_bdy_tend_xs", field_bdy_tend_xs), ("field_bdy_tend_xe", field_bdy_tend_xe),
                                  ("field_bdy_tend_ys", field_bdy_tend_ys), ("field_bdy_tend_ye", field_bdy_tend_ye))]
    with torch.cuda.device(field_tend.device):
        rc = N.lib().wrf_spec_bdytend(ctypes.byref(_cgrid(field_tend.shape)), _ptr("field_tend", field_tend), *bt,
                                      var.encode(), _stream())
    N.check(rc, "wrf_spec_bdytend")
    return field_tend


def spec_bdyupdate(field, field_tend, dt, variable, spec_zone, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms,
                   kme, ips, ipe, jps, jpe, kps, kpe, its, ite, jts, jte, kts, kte):
    """spec_bdyupdate (pywrf/wrf_boundary.py:228-284) on the GPU through
    ``wrf_spec_bdyupdate``: field += dt * field_tend on the specified rows,
    in place, returned; variable 'u', 'v', 't' (3-D) or 'm' (2-D, the
    reference's kds == kde == 0 call)."""
    _frame_b("spec_bdyupdate", field.shape, ids, ide, jds, jde, its, ite, jts, jte)
    if int(spec_zone) != 1:
        raise NotImplementedError("spec_bdyupdate: only spec_zone 1 is supported")
    var = str(variable).lower()
    if (var == "m") != (field.dim() == 2):
        raise ValueError("spec_bdyupdate: 'm' takes 2-D fields, the other letters 3-D")
    with torch.cuda.device(field.device):
        rc = N.lib().wrf_spec_bdyupdate(ctypes.byref(_cgrid(field.shape)), _ptr("field", field),
                                        _ptr("field_tend", field_tend), float(dt), var.encode(), _stream())
    N.check(rc, "wrf_spec_bdyupdate")
    return field


def spec_bdyupdate_ph(ph_save, field, field_tend, mu_tend, muts, c1, c2, dt, variable_in, spec_zone, ids, ide, jds,
                      jde, kds, kde, ims, ime, jms, jme, kms, kme, ips, ipe, jps, jpe, kps, kpe, its, ite, jts, jte,
                      kts, kte):
    """spec_bdyupdate_ph (pywrf/wrf_boundary.py:287-355) on the GPU through
    ``wrf_spec_bdyupdate_ph``: the specified rows of field (ph) are
    re-weighted with mu_old = muts - dt mu_tend, in place; returned.
    variable_in must be 'h'; c1 and c2 are accepted and unused, as in the
    reference."""
    _frame_b("spec_bdyupdate_ph", field.shape, ids, ide, jds, jde, its, ite, jts, jte)
    if int(spec_zone) != 1 or str(variable_in).lower() != "h":
        raise NotImplementedError("spec_bdyupdate_ph: only variable 'h' with spec_zone 1 is supported")
    from .adjoint import _table

    named = {"ph": field, "ph_save": ph_save, "ph_tend": field_tend, "mu_tend": mu_tend, "muts": muts}
    for k, t in named.items():
        _ptr(k, t)
    with torch.cuda.device(field.device):
        rc = N.lib().wrf_spec_bdyupdate_ph(ctypes.byref(_cgrid(field.shape)), _table(named), float(dt), _stream())
    N.check(rc, "wrf_spec_bdyupdate_ph")
    return field


def zero_grad_bdy(field, variable_in, spec_zone, ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme, ips, ipe,
                  jps, jpe, kps, kpe, its, ite, jts, jte, kts, kte):
    """zero_grad_bdy (pywrf/wrf_boundary.py:361-405) of w, the solver's only
    call, on the GPU through ``wrf_zero_grad_w``: the specified rows take
    their inner neighbour's value, in place; returned."""
    _frame_b("zero_grad_bdy", field.shape, ids, ide, jds, jde, its, ite, jts, jte)
    if int(spec_zone) != 1 or str(variable_in).lower() != "w":
        raise NotImplementedError("zero_grad_bdy: only variable 'w' with spec_zone 1 is supported")
    with torch.cuda.device(field.device):
        rc = N.lib().wrf_zero_grad_w(ctypes.byref(_cgrid(field.shape)), _ptr("field", field), _stream())
    N.check(rc, "wrf_zero_grad_w")
    return field
