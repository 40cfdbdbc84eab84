"""Drop-in for ``pywrf.wrf_boundary.relax_bdytend`` (reference signature).

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
