"""Hand-written adjoints of step operators behind ``torch.autograd.Function``.

The reference differentiates its step with PyTorch's taped autograd; here
each operator's reverse product is its own CUDA kernel
(include/pywrf_b200.h, ``wrf_*_adj``), so backpropagation through these
operators keeps no tape of the forward's intermediates.

* :class:`AdvectScalar` -- ``tendency + advect(field; ru, rv, rom)``
  (pywrf/wrf_dynamics.py:1841-2028); gradients with respect to the field, the
  incoming tendency and the three mass fluxes.
"""
from __future__ import annotations

import ctypes

import torch

from . import _native as N
from .config import Grid
from .state import make_cgrid


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise TypeError("a contiguous float32 CUDA tensor is required (no CPU path)")
    return ctypes.c_void_p(t.data_ptr())


def scalar_grid(shape, rdx: float, rdy: float):
    """The C grid record of the solver's 5-cell frame for a field of ``shape``."""
    nz, ny, nx = shape
    g = Grid.make(nx, ny, nz, 1.0 / float(rdx), 1.0 / float(rdy), 1.0)
    cg = make_cgrid(g, {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0, "cfn1": 0.0})
    cg.dx = 1.0 / float(rdx)
    cg.dy = 1.0 / float(rdy)
    return cg


class AdvectScalar(torch.autograd.Function):
    """out = tendency + flux-form advection of ``field`` by (ru, rv, rom)."""

    @staticmethod
    def forward(ctx, field, tendency, ru, rv, rom, msftx, fnm, fnp, rdnw, rdx: float, rdy: float):
        cg = scalar_grid(field.shape, rdx, rdy)
        out = tendency.detach().clone()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_advect_scalar(ctypes.byref(cg), _ptr(field), _ptr(out), _ptr(ru), _ptr(rv), _ptr(rom),
                                           _ptr(msftx), _ptr(fnm), _ptr(fnp), _ptr(rdnw), stream)
        N.check(rc, "wrf_advect_scalar")
        ctx.save_for_backward(field, ru, rv, rom, msftx, fnm, fnp, rdnw)
        ctx.cg = cg
        return out

    @staticmethod
    def backward(ctx, gout):
        field, ru, rv, rom, msftx, fnm, fnp, rdnw = ctx.saved_tensors
        gout = gout.contiguous()
        qb, rub, rvb, romb = (torch.zeros_like(field) for _ in range(4))
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_advect_scalar_adj(ctypes.byref(ctx.cg), _ptr(field), _ptr(ru), _ptr(rv), _ptr(rom),
                                               _ptr(msftx), _ptr(fnm), _ptr(fnp), _ptr(rdnw), _ptr(gout), _ptr(qb),
                                               _ptr(rub), _ptr(rvb), _ptr(romb), stream)
        N.check(rc, "wrf_advect_scalar_adj")
        return qb, gout, rub, rvb, romb, None, None, None, None, None, None


def advect_scalar(field, tendency, ru, rv, rom, msftx, fnm, fnp, rdnw, rdx, rdy):
    """Differentiable ``tendency + advect(field)`` on the GPU."""
    return AdvectScalar.apply(field, tendency, ru, rv, rom, msftx, fnm, fnp, rdnw, rdx, rdy)
