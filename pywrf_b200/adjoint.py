"""Hand-written adjoints of step operators behind ``torch.autograd.Function``.

The reference differentiates its step with PyTorch's taped autograd; here
each operator's reverse product is its own CUDA kernel
(include/pywrf_b200.h, ``wrf_*_adj``), so backpropagation through these
operators keeps no tape of the forward's intermediates.

* :class:`AdvectScalar` -- ``tendency + advect(field; ru, rv, rom)``
  (pywrf/wrf_dynamics.py:1841-2028); gradients with respect to the field, the
  incoming tendency and the three mass fluxes.
* :class:`AdvectMomentum` -- ``tendency + advect_u / advect_v / advect_w``
  (pywrf/wrf_dynamics.py:1112-1823); gradients with respect to the advected
  component, the incoming tendency and ru, rv, rom.
* :class:`AdvanceUV` -- advance_uv followed by spec_bdyupdate of u and v
  (pywrf/wrf_dynamics.py:3391-3525, pywrf/wrf_boundary.py:244-290), the
  horizontal-momentum part of the acoustic substep; gradients with respect to
  u, v, ru_tend, rv_tend, p, pb, ph, php, alt, al, mu, muu, muv, cqu, cqv and
  mudf (map factors and vertical profiles are data).
* :class:`CalcPRho` -- calc_p_rho (pywrf/wrf_dynamics.py:3269-3313): al, p,
  pm1 from ph, alt, t_2, t_1, c2a, pm1, mu, mut at a given acoustic step;
  gradients with respect to all ten.
* :class:`AdvanceMuT` -- advance_mu_t (pywrf/wrf_dynamics.py:3528-3638): the
  column mass, eta-velocity and theta update of the acoustic substep;
  gradients with respect to its 18 array inputs, either of the operator
  (default) or as the reference's autograd gives them (``ref_no_grad``: its
  mu / muts / mudf / muave update runs under ``torch.no_grad()``).
* :class:`AdvanceW` -- advance_w (pywrf/wrf_dynamics.py:3641-3796): the
  vertically implicit w / phi update with its terrain lower boundary and
  Rayleigh damping; gradients with respect to its 23 array inputs.
* :class:`Forces` -- the large-step tendency terms rhs_ph,
  horizontal_pressure_gradient, pg_buoy_w, coriolis and curvature
  (pywrf/wrf_dynamics.py:2031-2620), any subset by a mask; gradients with
  respect to the incoming tendencies, cqw (which pg_buoy_w overwrites) and the
  21 state arrays they read.
* :class:`Sumflux`, :class:`SpecUpdate`, :class:`SpecUpdatePh` -- sumflux
  (pywrf/wrf_dynamics.py:3799-3839), spec_bdyupdate and spec_bdyupdate_ph
  (pywrf/wrf_boundary.py:244-355), the rest of the acoustic substep.
* :class:`Prep` -- rk_step_prep's functions calculate_full, calc_mu_uv,
  couple_momentum, calc_ww_cp, calc_cq, calc_alt, calc_php
  (pywrf/wrf_dynamics.py:30-159), any subset by a mask.
* :class:`RelaxBdytend` -- ``tendency + relax(field)`` toward the lateral
  boundary values (pywrf/wrf_boundary.py:52-147); gradients with respect to
  the field and the incoming tendency (the boundary arrays are data).
* :class:`CoefW` -- calc_coef_w (pywrf/wrf_dynamics.py:3316-3388): the
  implicit solve's coefficients a, alpha, gamma from mut, cqw, c2a;
  gradients with respect to those three.
* :class:`VSolveW` -- the vertically implicit w solve of advance_w
  (pywrf/wrf_dynamics.py:3761-3767); gradients with respect to the
  right-hand side and the coefficients a, alpha, gamma (the transposed solve).
* :class:`HorizontalDiffusion`, :func:`eddy_viscosity`, :class:`MassWeight`
  -- the first RK stage's diffusion (pywrf/wrf_dynamics.py:2623-2915), the
  eddy viscosities (compute_diff_metrics, cal_deform_and_div,
  calculate_km_kh: :491-995) and mass_weight (pywrf/wrf_boundary.py:408).
* :func:`addtend`, :class:`SpecBdytend`, the moisture update
  (rk_update_scalar, flow_dep_bdy, calc_p_rho_phi), :func:`microphysics`
  (moist_physics_prep_em, WSM6, moist_physics_finish_em, calc_p_rho_phi;
  WSM6's reverse in reverse mode over a per-column tape of a restatement) and
  :func:`step_end` (halo copies, spec_bdy_final, set_w_surface).
* Composed in the reference's order: :func:`acoustic_substep`,
  :func:`acoustic_stage`, :func:`dynamics_stage`, :func:`moist_stage`,
  :func:`rk_stage` and :func:`step` (one whole time step,
  pywrf/solver.py:709-1910, with an optional theta-tendency bias).
* :func:`rollout` -- truncated backpropagation through ``n_steps`` of a
  step made of these operators with per-step (or per-segment) checkpointing:
  only each segment's input state is kept, and the backward pass recomputes
  the segment's forward once before back-propagating through it.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Sequence

import torch
from torch.utils.checkpoint import checkpoint

from . import _native as N
from .config import Grid
from .state import make_cgrid


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise TypeError("a contiguous float32 CUDA tensor is required (no CPU path)")
    return ctypes.c_void_p(t.data_ptr())


def _cuda_only(*ts) -> None:
    """Refuse anything but contiguous float32 CUDA tensors before any
    library or stream call (None entries are optional operands)."""
    for t in ts:
        if t is not None:
            _ptr(t)


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
        _cuda_only(field, tendency, ru, rv, rom, msftx, fnm, fnp, rdnw)
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
        qb, rub, rvb, romb = _zeros(field, field, field, field)
        n = ctypes.c_size_t(0)
        N.check(N.lib().wrf_advect_scalar_adj_work(ctypes.byref(ctx.cg), ctypes.byref(n)), "work")
        work = torch.empty(int(n.value), dtype=torch.float32, device=field.device)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_advect_scalar_adj(ctypes.byref(ctx.cg), _ptr(field), _ptr(ru), _ptr(rv), _ptr(rom),
                                               _ptr(msftx), _ptr(fnm), _ptr(fnp), _ptr(rdnw), _ptr(gout), _ptr(qb),
                                               _ptr(rub), _ptr(rvb), _ptr(romb), _ptr(work), n, stream)
        N.check(rc, "wrf_advect_scalar_adj")
        return qb, gout, rub, rvb, romb, None, None, None, None, None, None


def advect_scalar(field, tendency, ru, rv, rom, msftx, fnm, fnp, rdnw, rdx, rdy):
    """Differentiable ``tendency + advect(field)`` on the GPU."""
    return AdvectScalar.apply(field, tendency, ru, rv, rom, msftx, fnm, fnp, rdnw, rdx, rdy)


class AdvectMomentum(torch.autograd.Function):
    """out = tendency + flux-form advection of one momentum component
    (0 u with msf = msfux, 1 v with msf = msfvy and msf2 = msfvx, 2 w with
    msf = msftx; rdz = rdnw for u and v, rdn for w)."""

    @staticmethod
    def forward(ctx, component: int, field, tendency, ru, rv, rom, msf, msf2, fzm, fzp, rdz, rdx: float, rdy: float):
        _cuda_only(field, tendency, ru, rv, rom, msf, msf2, fzm, fzp, rdz)
        if component not in (0, 1, 2):
            raise ValueError("component must be 0 (u), 1 (v) or 2 (w)")
        if component == 1 and msf2 is None:
            raise ValueError("advect_v needs msf2 (msfvx)")
        cg = scalar_grid(field.shape, rdx, rdy)
        out = tendency.detach().clone()
        m2 = _ptr(msf2) if msf2 is not None else None
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_advect_momentum(ctypes.byref(cg), int(component), _ptr(field), _ptr(out), _ptr(ru),
                                             _ptr(rv), _ptr(rom), _ptr(msf), m2, _ptr(fzm), _ptr(fzp), _ptr(rdz),
                                             0, stream)
        N.check(rc, "wrf_advect_momentum")
        ctx.save_for_backward(field, ru, rv, rom, msf, msf if msf2 is None else msf2, fzm, fzp, rdz)
        ctx.cg, ctx.component, ctx.has_msf2 = cg, int(component), msf2 is not None
        return out

    @staticmethod
    def backward(ctx, gout):
        field, ru, rv, rom, msf, msf2, fzm, fzp, rdz = ctx.saved_tensors
        gout = gout.contiguous()
        qb, rub, rvb, romb = _zeros(field, field, field, field)
        m2 = _ptr(msf2) if ctx.has_msf2 else None
        n = ctypes.c_size_t(0)
        N.check(N.lib().wrf_advect_momentum_adj_work(ctypes.byref(ctx.cg), ctypes.byref(n)), "work")
        work = torch.empty(int(n.value), dtype=torch.float32, device=field.device)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_advect_momentum_adj(ctypes.byref(ctx.cg), ctx.component, _ptr(field), _ptr(ru), _ptr(rv),
                                                 _ptr(rom), _ptr(msf), m2, _ptr(fzm), _ptr(fzp), _ptr(rdz), _ptr(gout),
                                                 _ptr(qb), _ptr(rub), _ptr(rvb), _ptr(romb), _ptr(work), n, stream)
        N.check(rc, "wrf_advect_momentum_adj")
        return None, qb, gout, rub, rvb, romb, None, None, None, None, None, None, None


def advect_momentum(component, field, tendency, ru, rv, rom, msf, msf2, fzm, fzp, rdz, rdx, rdy):
    """Differentiable ``tendency + advect_{u,v,w}(field)`` on the GPU
    (component 0, 1, 2)."""
    return AdvectMomentum.apply(component, field, tendency, ru, rv, rom, msf, msf2, fzm, fzp, rdz, rdx, rdy)


UV_INPUTS = ("u", "v", "ru_tend", "rv_tend", "p", "pb", "ph", "php", "alt", "al", "mu", "muu", "muv", "cqu", "cqv",
             "mudf")
UV_DATA = ("msfux", "msfuy", "msfvx", "msfvx_inv", "msfvy", "fnm", "fnp", "rdnw")


def _table(named: dict):
    """A state table (WrfState) holding the given fields by name."""
    names = N.field_names()
    arr = (ctypes.c_void_p * len(names))()
    for k, t in named.items():
        arr[names.index(k)] = _ptr(t).value
    return arr


def _zeros(*likes):
    """Zero float32 tensors shaped like ``likes``, carved (at 256-byte
    aligned offsets) from one buffer that a single fill clears: one launch
    instead of one per cotangent buffer."""
    if not likes:
        return []
    sizes = [(t.numel() + 63) // 64 * 64 for t in likes]
    buf = torch.zeros(sum(sizes), dtype=torch.float32, device=likes[0].device)
    out, o = [], 0
    for t, n in zip(likes, sizes):
        out.append(buf[o:o + t.numel()].view(t.shape))
        o += n
    return out


def _bars(named: dict, fields, grads: dict) -> dict:
    """Cotangent buffers for ``fields``: a clone of the incoming gradient
    where ``grads`` holds one (the adjoint rewrites it in place), zeros from
    one shared buffer for the rest."""
    rest = [k for k in fields if grads.get(k) is None]
    bars = dict(zip(rest, _zeros(*[named[k] for k in rest])))
    for k in fields:
        if k not in bars:
            bars[k] = grads[k].contiguous().clone()
    return bars


class AdvanceUV(torch.autograd.Function):
    """(u', v') = advance_uv + spec_bdyupdate(u), (v); the tensors follow
    UV_INPUTS then UV_DATA, ``scal`` = (dts, emdiv, cf1, cf2, cf3, rdx, rdy)."""

    @staticmethod
    def forward(ctx, scal, *tensors):
        # outputs without a cotangent reach backward as None (its _bars / None
        # checks hand out zeros from one shared buffer) instead of one
        # zero-filled tensor each, which backward would then clone
        ctx.set_materialize_grads(False)
        _cuda_only(*tensors)
        dts, emdiv, cf1, cf2, cf3, rdx, rdy = (float(x) for x in scal)
        named = dict(zip(UV_INPUTS + UV_DATA, tensors))
        cg = scalar_grid(named["u"].shape, rdx, rdy)
        cg.emdiv, cg.cf1, cg.cf2, cg.cf3 = emdiv, cf1, cf2, cf3
        u_new, v_new = named["u"].detach().clone(), named["v"].detach().clone()
        tab = _table({**named, "u": u_new, "v": v_new})
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(u_new.device):
            rc = N.lib().wrf_advance_uv(ctypes.byref(cg), tab, dts, stream)
        N.check(rc, "wrf_advance_uv")
        ctx.save_for_backward(*tensors)
        ctx.cg, ctx.dts = cg, dts
        return u_new, v_new

    @staticmethod
    def backward(ctx, gu, gv):
        tensors = ctx.saved_tensors
        named = dict(zip(UV_INPUTS + UV_DATA, tensors))
        bars = _bars(named, UV_INPUTS[2:] + tuple(k for k, gk in (("u", gu), ("v", gv)) if gk is None), {})
        gu = bars["u"] if gu is None else gu.contiguous()
        gv = bars["v"] if gv is None else gv.contiguous()
        tab = _table(named)
        btab = _table({"u": gu, "v": gv, **bars})
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(gu.device):
            rc = N.lib().wrf_advance_uv_adj(ctypes.byref(ctx.cg), tab, btab, ctx.dts, stream)
        N.check(rc, "wrf_advance_uv_adj")
        return (None, gu, gv) + tuple(bars[k] for k in UV_INPUTS[2:]) + (None,) * len(UV_DATA)


def advance_uv(inputs: dict, data: dict, dts, emdiv, cf1, cf2, cf3, rdx, rdy):
    """Differentiable advance_uv + spec_bdyupdate(u), (v) on the GPU:
    ``inputs`` maps UV_INPUTS, ``data`` UV_DATA to tensors; returns (u', v')."""
    return AdvanceUV.apply((dts, emdiv, cf1, cf2, cf3, rdx, rdy), *[inputs[k] for k in UV_INPUTS],
                           *[data[k] for k in UV_DATA])


FORCES_OUTPUTS = ("ph_tend", "ru_tend", "rv_tend", "rw_tend", "cqw")
FORCES_INPUTS = FORCES_OUTPUTS + ("u", "v", "w", "ww", "ph", "phb", "mut", "muu", "muv", "alt", "p", "pb", "al",
                                  "php", "cqu", "cqv", "mu", "mub", "ru", "rv", "rw")
FORCES_DATA = ("msfux", "msfuy", "msfvx", "msfvy", "msftx", "msfty", "f", "e", "sina", "cosa", "fnm", "fnp", "rdnw",
               "rdn")
FORCES_TERMS = {"rhs_ph": 1, "hpg": 2, "pg_buoy_w": 4, "coriolis": 8, "curvature": 16}


class Forces(torch.autograd.Function):
    """(ph_tend', ru_tend', rv_tend', rw_tend', cqw') = the tendency terms of
    the mask ``terms`` (rhs_ph 1, horizontal_pressure_gradient 2, pg_buoy_w 4,
    coriolis 8, curvature 16) added to the incoming tendencies; the tensors
    follow FORCES_INPUTS then FORCES_DATA, ``scal`` = (terms, rdx, rdy, cf1,
    cf2, cf3, cfn, cfn1)."""

    @staticmethod
    def forward(ctx, scal, *tensors):
        # outputs without a cotangent reach backward as None (its _bars / None
        # checks hand out zeros from one shared buffer) instead of one
        # zero-filled tensor each, which backward would then clone
        ctx.set_materialize_grads(False)
        _cuda_only(*tensors)
        terms = int(scal[0])
        rdx, rdy, cf1, cf2, cf3, cfn, cfn1 = (float(x) for x in scal[1:])
        named = dict(zip(FORCES_INPUTS + FORCES_DATA, tensors))
        cg = scalar_grid(named["u"].shape, rdx, rdy)
        cg.cf1, cg.cf2, cg.cf3, cg.cfn, cg.cfn1 = cf1, cf2, cf3, cfn, cfn1
        outs = {k: named[k].detach().clone() for k in FORCES_OUTPUTS}
        tab = _table({**named, **outs})
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(outs["ph_tend"].device):
            rc = N.lib().wrf_forces(ctypes.byref(cg), tab, terms, stream)
        N.check(rc, "wrf_forces")
        ctx.save_for_backward(*tensors)
        ctx.cg, ctx.terms = cg, terms
        return tuple(outs[k] for k in FORCES_OUTPUTS)

    @staticmethod
    def backward(ctx, *gouts):
        tensors = ctx.saved_tensors
        named = dict(zip(FORCES_INPUTS + FORCES_DATA, tensors))
        bars = _bars(named, FORCES_INPUTS, dict(zip(FORCES_OUTPUTS, gouts)))
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(bars["u"].device):
            rc = N.lib().wrf_forces_adj(ctypes.byref(ctx.cg), _table(named), _table(bars), ctx.terms, stream)
        N.check(rc, "wrf_forces_adj")
        return (None,) + tuple(bars[k] for k in FORCES_INPUTS) + (None,) * len(FORCES_DATA)


def forces(inputs: dict, data: dict, terms, rdx, rdy, cf1, cf2, cf3, cfn, cfn1):
    """Differentiable tendency terms on the GPU: ``inputs`` maps
    FORCES_INPUTS, ``data`` FORCES_DATA to tensors; ``terms`` is a mask or a
    sequence of FORCES_TERMS names; returns (ph_tend', ru_tend', rv_tend',
    rw_tend', cqw')."""
    if not isinstance(terms, int):
        terms = sum(FORCES_TERMS[t] for t in terms)
    return Forces.apply((terms, rdx, rdy, cf1, cf2, cf3, cfn, cfn1), *[inputs[k] for k in FORCES_INPUTS],
                        *[data[k] for k in FORCES_DATA])


SF_INPUTS = ("ru_m", "rv_m", "ww_m", "u", "v", "ww", "u_save", "v_save", "ww1", "muu", "muv")
SF_DATA = ("msfuy", "msfvx_inv")


class Sumflux(torch.autograd.Function):
    """(ru_m', rv_m', ww_m') = sumflux at ``iteration`` of ``nsub``; the
    tensors follow SF_INPUTS then SF_DATA, ``scal`` = (iteration, nsub, rdx,
    rdy)."""

    @staticmethod
    def forward(ctx, scal, *tensors):
        # outputs without a cotangent reach backward as None (its _bars / None
        # checks hand out zeros from one shared buffer) instead of one
        # zero-filled tensor each, which backward would then clone
        ctx.set_materialize_grads(False)
        _cuda_only(*tensors)
        iteration, nsub = int(scal[0]), int(scal[1])
        named = dict(zip(SF_INPUTS + SF_DATA, tensors))
        cg = scalar_grid(named["u"].shape, float(scal[2]), float(scal[3]))
        outs = {k: named[k].detach().clone() for k in SF_INPUTS[:3]}
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(named["u"].device):
            rc = N.lib().wrf_sumflux(ctypes.byref(cg), _table({**named, **outs}), iteration, nsub, stream)
        N.check(rc, "wrf_sumflux")
        ctx.save_for_backward(*tensors)
        ctx.cg, ctx.it = cg, (iteration, nsub)
        return tuple(outs[k] for k in SF_INPUTS[:3])

    @staticmethod
    def backward(ctx, *gouts):
        named = dict(zip(SF_INPUTS + SF_DATA, ctx.saved_tensors))
        bars = _bars(named, SF_INPUTS, dict(zip(SF_INPUTS[:3], gouts)))
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(bars["u"].device):
            rc = N.lib().wrf_sumflux_adj(ctypes.byref(ctx.cg), _table(named), _table(bars), ctx.it[0], ctx.it[1],
                                         stream)
        N.check(rc, "wrf_sumflux_adj")
        return (None,) + tuple(bars[k] for k in SF_INPUTS) + (None,) * len(SF_DATA)


def sumflux(inputs: dict, data: dict, iteration: int, nsub: int, rdx, rdy):
    """Differentiable sumflux on the GPU; returns (ru_m', rv_m', ww_m')."""
    return Sumflux.apply((iteration, nsub, rdx, rdy), *[inputs[k] for k in SF_INPUTS], *[data[k] for k in SF_DATA])


class SpecUpdate(torch.autograd.Function):
    """field' = spec_bdyupdate(field, tend, dt, var) (var 't', 'u', 'v' or
    'm'); ``scal`` = (dt, var, rdx, rdy)."""

    @staticmethod
    def forward(ctx, scal, field, tend):
        _cuda_only(field, tend)
        dt, var = float(scal[0]), str(scal[1])
        shape = field.shape if field.dim() == 3 else (12,) + tuple(field.shape)
        cg = scalar_grid(shape, float(scal[2]), float(scal[3]))
        out = field.detach().clone()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_spec_bdyupdate(ctypes.byref(cg), _ptr(out), _ptr(tend), dt, var.encode(), stream)
        N.check(rc, "wrf_spec_bdyupdate")
        ctx.cg, ctx.dt, ctx.var = cg, dt, var
        return out

    @staticmethod
    def backward(ctx, gout):
        gout = gout.contiguous()
        tb = torch.zeros_like(gout)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(gout.device):
            rc = N.lib().wrf_spec_bdyupdate_adj(ctypes.byref(ctx.cg), _ptr(gout), _ptr(tb), ctx.dt, ctx.var.encode(),
                                                stream)
        N.check(rc, "wrf_spec_bdyupdate_adj")
        return None, gout, tb


def spec_bdyupdate(field, tend, dt, var: str, rdx, rdy):
    """Differentiable spec_bdyupdate on the GPU."""
    return SpecUpdate.apply((dt, var, rdx, rdy), field, tend)


SPH_INPUTS = ("ph", "ph_save", "ph_tend", "mu_tend", "muts")


class SpecUpdatePh(torch.autograd.Function):
    """ph' = spec_bdyupdate_ph(ph_save, ph, ph_tend, mu_tend, muts, dt); the
    tensors follow SPH_INPUTS, ``scal`` = (dt, rdx, rdy)."""

    @staticmethod
    def forward(ctx, scal, *tensors):
        _cuda_only(*tensors)
        named = dict(zip(SPH_INPUTS, tensors))
        cg = scalar_grid(named["ph"].shape, float(scal[1]), float(scal[2]))
        out = named["ph"].detach().clone()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(out.device):
            rc = N.lib().wrf_spec_bdyupdate_ph(ctypes.byref(cg), _table({**named, "ph": out}), float(scal[0]), stream)
        N.check(rc, "wrf_spec_bdyupdate_ph")
        ctx.save_for_backward(*tensors)
        ctx.cg, ctx.dt = cg, float(scal[0])
        return out

    @staticmethod
    def backward(ctx, gout):
        named = dict(zip(SPH_INPUTS, ctx.saved_tensors))
        bars = _bars(named, SPH_INPUTS, {"ph": gout})
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(gout.device):
            rc = N.lib().wrf_spec_bdyupdate_ph_adj(ctypes.byref(ctx.cg), _table(named), _table(bars), ctx.dt, stream)
        N.check(rc, "wrf_spec_bdyupdate_ph_adj")
        return (None,) + tuple(bars[k] for k in SPH_INPUTS)


def spec_bdyupdate_ph(inputs: dict, dt, rdx, rdy):
    """Differentiable spec_bdyupdate_ph on the GPU; ``inputs`` maps SPH_INPUTS."""
    return SpecUpdatePh.apply((dt, rdx, rdy), *[inputs[k] for k in SPH_INPUTS])


PREP_FIELDS = ("mu", "mub", "mut", "muu", "muv", "u", "v", "w", "ru", "rv", "rw", "ww", "moist", "cqu", "cqv",
               "cqw", "al", "alb", "alt", "ph", "phb", "php")
PREP_OUTPUTS = ("mut", "muu", "muv", "ru", "rv", "rw", "ww", "cqu", "cqv", "cqw", "alt", "php")
PREP_DATA = ("msfu", "msfvx_inv", "msft", "msftx", "msfuy", "dnw", "c1h")
PREP_OPS = {"calculate_full": 1, "calc_mu_uv": 2, "couple_momentum": 4, "calc_ww_cp": 8, "calc_cq": 16,
            "calc_alt": 32, "calc_php": 64}


class Prep(torch.autograd.Function):
    """PREP_OUTPUTS' = rk_step_prep's functions of the mask ``ops`` (the
    others pass through); the tensors follow PREP_FIELDS then PREP_DATA,
    ``scal`` = (ops, rdx, rdy)."""

    @staticmethod
    def forward(ctx, scal, *tensors):
        # outputs without a cotangent reach backward as None (its _bars / None
        # checks hand out zeros from one shared buffer) instead of one
        # zero-filled tensor each, which backward would then clone
        ctx.set_materialize_grads(False)
        _cuda_only(*tensors)
        ops = int(scal[0])
        named = dict(zip(PREP_FIELDS + PREP_DATA, tensors))
        cg = scalar_grid(named["u"].shape, float(scal[1]), float(scal[2]))
        outs = {k: named[k].detach().clone() for k in PREP_OUTPUTS}
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(named["u"].device):
            rc = N.lib().wrf_prep(ctypes.byref(cg), _table({**named, **outs}), ops, stream)
        N.check(rc, "wrf_prep")
        ctx.save_for_backward(*tensors)
        ctx.cg, ctx.ops = cg, ops
        return tuple(outs[k] for k in PREP_OUTPUTS)

    @staticmethod
    def backward(ctx, *gouts):
        named = dict(zip(PREP_FIELDS + PREP_DATA, ctx.saved_tensors))
        bars = _bars(named, PREP_FIELDS, dict(zip(PREP_OUTPUTS, gouts)))
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(bars["u"].device):
            rc = N.lib().wrf_prep_adj(ctypes.byref(ctx.cg), _table(named), _table(bars), ctx.ops, stream)
        N.check(rc, "wrf_prep_adj")
        return (None,) + tuple(bars[k] for k in PREP_FIELDS) + (None,) * len(PREP_DATA)


def prep(fields: dict, data: dict, ops, rdx, rdy):
    """Differentiable rk_step_prep functions on the GPU: ``fields`` maps
    PREP_FIELDS, ``data`` PREP_DATA; ``ops`` a mask or PREP_OPS names; returns
    a dict of PREP_OUTPUTS."""
    if not isinstance(ops, int):
        ops = sum(PREP_OPS[o] for o in ops)
    outs = Prep.apply((ops, rdx, rdy), *[fields[k] for k in PREP_FIELDS], *[data[k] for k in PREP_DATA])
    return dict(zip(PREP_OUTPUTS, outs))


class Halo(torch.autograd.Function):
    """field' = set_physical_bc3d / set_physical_bc2d(field, var) (the open
    halo copies); ``scal`` = (var, rdx, rdy)."""

    @staticmethod
    def forward(ctx, scal, field):
        _cuda_only(field)
        var = str(scal[0])
        two_d = field.dim() == 2
        shape = (12,) + tuple(field.shape) if two_d else field.shape
        cg = scalar_grid(shape, float(scal[1]), float(scal[2]))
        out = field.detach().clone()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_halo(ctypes.byref(cg), _ptr(out), var.encode(), int(two_d), stream)
        N.check(rc, "wrf_halo")
        ctx.cg, ctx.var, ctx.two_d = cg, var, two_d
        return out

    @staticmethod
    def backward(ctx, gout):
        gout = gout.contiguous()
        gin = torch.zeros_like(gout)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(gout.device):
            rc = N.lib().wrf_halo_adj(ctypes.byref(ctx.cg), _ptr(gout), _ptr(gin), ctx.var.encode(), int(ctx.two_d),
                                      stream)
        N.check(rc, "wrf_halo_adj")
        return None, gin


def halo(field, var: str, rdx=1.0 / 9000.0, rdy=1.0 / 9000.0):
    """Differentiable open-boundary halo copy of a [nz, ny, nx] or [ny, nx] field."""
    return Halo.apply((var, rdx, rdy), field)


class ZeroGradW(torch.autograd.Function):
    """w' = zero_grad_bdy(w, 'w'); ``scal`` = (rdx, rdy)."""

    @staticmethod
    def forward(ctx, scal, w):
        _cuda_only(w)
        cg = scalar_grid(w.shape, float(scal[0]), float(scal[1]))
        out = w.detach().clone()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(w.device):
            rc = N.lib().wrf_zero_grad_w(ctypes.byref(cg), _ptr(out), stream)
        N.check(rc, "wrf_zero_grad_w")
        ctx.cg = cg
        return out

    @staticmethod
    def backward(ctx, gout):
        gout = gout.contiguous()
        gin = torch.zeros_like(gout)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(gout.device):
            rc = N.lib().wrf_zero_grad_w_adj(ctypes.byref(ctx.cg), _ptr(gout), _ptr(gin), stream)
        N.check(rc, "wrf_zero_grad_w_adj")
        return None, gin


def zero_grad_w(w, rdx=1.0 / 9000.0, rdy=1.0 / 9000.0):
    """Differentiable zero_grad_bdy of w."""
    return ZeroGradW.apply((rdx, rdy), w)


AW_INPUTS = ("w", "rw_tend", "ww", "w_save", "u", "v", "muave", "muts", "mut", "t_2ave", "t_2", "t_1", "ph", "ph_1",
             "phb", "ph_tend", "ht", "c2a", "cqw", "alt", "a", "alpha", "gamma")
AW_DATA = ("msftx", "msfty", "fnm", "fnp", "rdnw", "rdn")
AW_OUTPUTS = ("t_2ave", "w", "ph")
_AW_FIELD = {"t_2ave": "t_2save", "t_2": "t", "t_1": "t_save", "ph_1": "ph_save"}


class AdvanceW(torch.autograd.Function):
    """(t_2ave', w', ph') = advance_w(...); the tensors follow AW_INPUTS then
    AW_DATA, ``scal`` = (dts, epssm, cf1, cf2, cf3, rdx, rdy)."""

    @staticmethod
    def forward(ctx, scal, *tensors):
        # outputs without a cotangent reach backward as None (its _bars / None
        # checks hand out zeros from one shared buffer) instead of one
        # zero-filled tensor each, which backward would then clone
        ctx.set_materialize_grads(False)
        _cuda_only(*tensors)
        dts, epssm, cf1, cf2, cf3, rdx, rdy = (float(x) for x in scal)
        named = dict(zip(AW_INPUTS + AW_DATA, tensors))
        cg = scalar_grid(named["w"].shape, rdx, rdy)
        cg.epssm, cg.cf1, cg.cf2, cg.cf3 = epssm, cf1, cf2, cf3
        outs = {k: named[k].detach().clone() for k in AW_OUTPUTS}
        tab = _table({_AW_FIELD.get(k, k): v for k, v in {**named, **outs}.items()})
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(outs["w"].device):
            rc = N.lib().wrf_advance_w(ctypes.byref(cg), tab, dts, stream)
        N.check(rc, "wrf_advance_w")
        ctx.save_for_backward(*tensors)
        ctx.cg, ctx.dts = cg, dts
        return tuple(outs[k] for k in AW_OUTPUTS)

    @staticmethod
    def backward(ctx, *gouts):
        tensors = ctx.saved_tensors
        named = dict(zip(AW_INPUTS + AW_DATA, tensors))
        bars = _bars(named, tuple(dict.fromkeys(AW_OUTPUTS + AW_INPUTS)), dict(zip(AW_OUTPUTS, gouts)))
        work = torch.empty_like(named["ht"])
        tab = _table({_AW_FIELD.get(k, k): v for k, v in named.items()})
        btab = _table({_AW_FIELD.get(k, k): v for k, v in bars.items()})
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(work.device):
            rc = N.lib().wrf_advance_w_adj(ctypes.byref(ctx.cg), tab, btab, ctx.dts, _ptr(work), stream)
        N.check(rc, "wrf_advance_w_adj")
        return (None,) + tuple(bars[k] for k in AW_INPUTS) + (None,) * len(AW_DATA)


def advance_w(inputs: dict, data: dict, dts, epssm, cf1, cf2, cf3, rdx=1.0 / 9000.0, rdy=1.0 / 9000.0):
    """Differentiable advance_w on the GPU: ``inputs`` maps AW_INPUTS, ``data``
    AW_DATA to tensors; returns a dict of AW_OUTPUTS."""
    outs = AdvanceW.apply((dts, epssm, cf1, cf2, cf3, rdx, rdy), *[inputs[k] for k in AW_INPUTS],
                          *[data[k] for k in AW_DATA])
    return dict(zip(AW_OUTPUTS, outs))


MUT_INPUTS = ("ww", "ww_1", "u", "u_1", "v", "v_1", "t", "t_1", "t_ave", "ft", "mu", "mut", "muave", "muts", "muu",
              "muv", "mudf", "mu_tend")
MUT_DATA = ("dnw", "fnm", "fnp", "rdnw", "msfuy", "msfvx_inv", "msftx", "msfty")
MUT_OUTPUTS = ("ww", "t", "t_ave", "muave", "muts", "mudf", "mu")
# the state-table names of advance_mu_t's arguments in the acoustic substep
_MUT_FIELD = {"ww_1": "ww1", "u_1": "u_save", "v_1": "v_save", "t_1": "t_save", "t_ave": "t_2save", "ft": "t_tend"}


class AdvanceMuT(torch.autograd.Function):
    """The seven outputs MUT_OUTPUTS of advance_mu_t; the tensors follow
    MUT_INPUTS then MUT_DATA, ``scal`` = (dts, epssm, rdx, rdy, ref_no_grad)."""

    @staticmethod
    def forward(ctx, scal, *tensors):
        # outputs without a cotangent reach backward as None (its _bars / None
        # checks hand out zeros from one shared buffer) instead of one
        # zero-filled tensor each, which backward would then clone
        ctx.set_materialize_grads(False)
        _cuda_only(*tensors)
        dts, epssm, rdx, rdy = (float(x) for x in scal[:4])
        named = dict(zip(MUT_INPUTS + MUT_DATA, tensors))
        cg = scalar_grid(named["ww"].shape, rdx, rdy)
        cg.epssm = epssm
        outs = {k: named[k].detach().clone() for k in MUT_OUTPUTS}
        tab = _table({_MUT_FIELD.get(k, k): v for k, v in {**named, **outs}.items()})
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(outs["ww"].device):
            rc = N.lib().wrf_advance_mu_t(ctypes.byref(cg), tab, dts, stream)
        N.check(rc, "wrf_advance_mu_t")
        ctx.save_for_backward(*tensors)
        ctx.cg, ctx.dts, ctx.ref_no_grad = cg, dts, int(bool(scal[4]))
        return tuple(outs[k] for k in MUT_OUTPUTS)

    @staticmethod
    def backward(ctx, *gouts):
        tensors = ctx.saved_tensors
        named = dict(zip(MUT_INPUTS + MUT_DATA, tensors))
        bars = _bars(named, tuple(dict.fromkeys(MUT_OUTPUTS + MUT_INPUTS)), dict(zip(MUT_OUTPUTS, gouts)))
        work = torch.empty_like(named["ww"])
        tab = _table({_MUT_FIELD.get(k, k): v for k, v in named.items()})
        btab = _table({_MUT_FIELD.get(k, k): v for k, v in bars.items()})
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(work.device):
            rc = N.lib().wrf_advance_mu_t_adj(ctypes.byref(ctx.cg), tab, btab, ctx.dts, ctx.ref_no_grad, _ptr(work),
                                              stream)
        N.check(rc, "wrf_advance_mu_t_adj")
        return (None,) + tuple(bars[k] for k in MUT_INPUTS) + (None,) * len(MUT_DATA)


def advance_mu_t(inputs: dict, data: dict, dts, epssm, rdx=1.0 / 9000.0, rdy=1.0 / 9000.0, ref_no_grad=False):
    """Differentiable advance_mu_t on the GPU: ``inputs`` maps MUT_INPUTS,
    ``data`` MUT_DATA to tensors; returns a dict of MUT_OUTPUTS."""
    outs = AdvanceMuT.apply((dts, epssm, rdx, rdy, ref_no_grad), *[inputs[k] for k in MUT_INPUTS],
                            *[data[k] for k in MUT_DATA])
    return dict(zip(MUT_OUTPUTS, outs))


PRHO_INPUTS = ("al", "p", "ph", "alt", "t_2", "t_1", "c2a", "pm1", "mu", "mut")
# the state-table names of calc_p_rho's arguments in the acoustic substep
_PRHO_FIELD = {"t_2": "t", "t_1": "t_save", "mut": "muts"}


class CalcPRho(torch.autograd.Function):
    """(al', p', pm1') = calc_p_rho(...) at acoustic step ``step``; the
    tensors follow PRHO_INPUTS then rdnw, ``scal`` = (smdiv, step, rdx, rdy)."""

    @staticmethod
    def forward(ctx, scal, *tensors):
        # outputs without a cotangent reach backward as None (its _bars / None
        # checks hand out zeros from one shared buffer) instead of one
        # zero-filled tensor each, which backward would then clone
        ctx.set_materialize_grads(False)
        _cuda_only(*tensors)
        smdiv, step, rdx, rdy = float(scal[0]), int(scal[1]), float(scal[2]), float(scal[3])
        named = dict(zip(PRHO_INPUTS + ("rdnw",), tensors))
        cg = scalar_grid(named["p"].shape, rdx, rdy)
        cg.smdiv = smdiv
        outs = {k: named[k].detach().clone() for k in ("al", "p", "pm1")}
        tab = _table({_PRHO_FIELD.get(k, k): v for k, v in {**named, **outs}.items()})
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(outs["p"].device):
            rc = N.lib().wrf_calc_p_rho(ctypes.byref(cg), tab, step, stream)
        N.check(rc, "wrf_calc_p_rho")
        ctx.save_for_backward(*tensors)
        ctx.cg, ctx.step = cg, step
        return outs["al"], outs["p"], outs["pm1"]

    @staticmethod
    def backward(ctx, gal, gp, gpm1):
        tensors = ctx.saved_tensors
        named = dict(zip(PRHO_INPUTS + ("rdnw",), tensors))
        allb = _bars(named, tuple(dict.fromkeys(("al", "p", "pm1") + PRHO_INPUTS)), {"al": gal, "p": gp, "pm1": gpm1})
        out_b = {k: allb[k] for k in ("al", "p", "pm1")}
        bars = {k: v for k, v in allb.items() if k not in out_b}
        tab = _table({_PRHO_FIELD.get(k, k): v for k, v in named.items()})
        btab = _table({_PRHO_FIELD.get(k, k): v for k, v in {**out_b, **bars}.items()})
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(named["p"].device):
            rc = N.lib().wrf_calc_p_rho_adj(ctypes.byref(ctx.cg), tab, btab, ctx.step, stream)
        N.check(rc, "wrf_calc_p_rho_adj")
        allb = {**out_b, **bars}
        return (None,) + tuple(allb[k] for k in PRHO_INPUTS) + (None,)


def calc_p_rho(inputs: dict, rdnw, smdiv, step, rdx=1.0 / 9000.0, rdy=1.0 / 9000.0):
    """Differentiable calc_p_rho on the GPU: ``inputs`` maps PRHO_INPUTS to
    tensors; returns (al', p', pm1')."""
    return CalcPRho.apply((smdiv, step, rdx, rdy), *[inputs[k] for k in PRHO_INPUTS], rdnw)


BDY_NAMES = ("xs", "xe", "ys", "ye", "txs", "txe", "tys", "tye")


class RelaxBdytend(torch.autograd.Function):
    """out = tendency + relax_bdytend(field) for one stagger letter."""

    @staticmethod
    def forward(ctx, field, tendency, variable: str, dtbc: float, *bdy8):
        _cuda_only(field, tendency, *bdy8)
        nz, ny, nx = field.shape
        # 'm' (mu) is 2-D: its [1, ny, nx] field rides on a grid record of
        # the frame's minimum depth, and the library relaxes one level
        cg = scalar_grid((12, ny, nx) if variable == "m" else field.shape, 1.0 / 9000.0, 1.0 / 9000.0)
        out = tendency.detach().clone()
        arr = (ctypes.c_void_p * 8)(*[_ptr(b).value for b in bdy8])
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_relax_bdytend(ctypes.byref(cg), _ptr(field), _ptr(out), arr, variable.encode(),
                                           float(dtbc), stream)
        N.check(rc, "wrf_relax_bdytend")
        ctx.cg, ctx.variable = cg, variable
        ctx.shape = (nz, ny, nx)
        ctx.device = field.device
        return out

    @staticmethod
    def backward(ctx, gout):
        gout = gout.contiguous()
        fb = torch.zeros(ctx.shape, dtype=torch.float32, device=ctx.device)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(ctx.device):
            rc = N.lib().wrf_relax_bdytend_adj(ctypes.byref(ctx.cg), _ptr(gout), _ptr(fb), ctx.variable.encode(),
                                               stream)
        N.check(rc, "wrf_relax_bdytend_adj")
        return (fb, gout, None, None) + (None,) * 8


def relax_bdytend(field, tendency, variable: str, dtbc: float, bdy: dict):
    """Differentiable ``tendency + relax_bdytend(field)``; ``bdy`` maps
    xs xe ys ye txs txe tys tye to the boundary arrays (solver layout)."""
    return RelaxBdytend.apply(field, tendency, variable, dtbc, *[bdy[k] for k in BDY_NAMES])


class VSolveW(torch.autograd.Function):
    """w = implicit solve of (x; a, alpha, gamma) per column; arrays [nz, ...]."""

    @staticmethod
    def forward(ctx, x, a, alpha, gamma):
        _cuda_only(x, a, alpha, gamma)
        nz = x.shape[0]
        ncol = x.numel() // nz
        w = torch.empty_like(x)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(x.device):
            rc = N.lib().wrf_vsolve_w(ncol, nz, _ptr(x), _ptr(a), _ptr(alpha), _ptr(gamma), _ptr(w), stream)
        N.check(rc, "wrf_vsolve_w")
        ctx.save_for_backward(x, a, alpha, gamma)
        return w

    @staticmethod
    def backward(ctx, gw):
        x, a, alpha, gamma = ctx.saved_tensors
        nz = x.shape[0]
        ncol = x.numel() // nz
        gw = gw.contiguous()
        gx, ga, gal, gg = _zeros(x, x, x, x)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(x.device):
            rc = N.lib().wrf_vsolve_w_adj(ncol, nz, _ptr(x), _ptr(a), _ptr(alpha), _ptr(gamma), _ptr(gw), _ptr(gx),
                                          _ptr(ga), _ptr(gal), _ptr(gg), stream)
        N.check(rc, "wrf_vsolve_w_adj")
        return gx, ga, gal, gg


def vsolve_w(x, a, alpha, gamma):
    """Differentiable implicit w solve (all columns of [nz, ...] arrays)."""
    return VSolveW.apply(x, a, alpha, gamma)


class CoefW(torch.autograd.Function):
    """(a, alpha, gamma) = calc_coef_w(mut, cqw, c2a) on the mass columns."""

    @staticmethod
    def forward(ctx, mut, cqw, c2a, rdn, rdnw, dts: float, epssm: float, top_lid: bool, rdx: float, rdy: float):
        # outputs without a cotangent reach backward as None (its _bars / None
        # checks hand out zeros from one shared buffer) instead of one
        # zero-filled tensor each, which backward would then clone
        ctx.set_materialize_grads(False)
        _cuda_only(mut, cqw, c2a, rdn, rdnw)
        cg = scalar_grid(cqw.shape, rdx, rdy)
        cg.epssm = float(epssm)
        cg.top_lid = int(bool(top_lid))
        a, alpha, gamma = (torch.zeros_like(cqw) for _ in range(3))
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(cqw.device):
            rc = N.lib().wrf_coef_w(ctypes.byref(cg), _ptr(mut), _ptr(cqw), _ptr(c2a), _ptr(rdn), _ptr(rdnw),
                                    float(dts), _ptr(a), _ptr(alpha), _ptr(gamma), stream)
        N.check(rc, "wrf_coef_w")
        ctx.save_for_backward(mut, cqw, c2a, rdn, rdnw)
        ctx.cg, ctx.dts = cg, float(dts)
        return a, alpha, gamma

    @staticmethod
    def backward(ctx, ga, galpha, ggamma):
        mut, cqw, c2a, rdn, rdnw = ctx.saved_tensors
        z, mb, cb, c2b = _zeros(cqw, mut, cqw, c2a)
        ga = z if ga is None else ga.contiguous()
        galpha = z if galpha is None else galpha.contiguous()
        ggamma = z if ggamma is None else ggamma.contiguous()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(cqw.device):
            rc = N.lib().wrf_coef_w_adj(ctypes.byref(ctx.cg), _ptr(mut), _ptr(cqw), _ptr(c2a), _ptr(rdn), _ptr(rdnw),
                                        ctx.dts, _ptr(ga), _ptr(galpha), _ptr(ggamma), _ptr(mb), _ptr(cb), _ptr(c2b),
                                        stream)
        N.check(rc, "wrf_coef_w_adj")
        return mb, cb, c2b, None, None, None, None, None, None, None


def coef_w(mut, cqw, c2a, rdn, rdnw, dts, epssm=0.1, top_lid=False, rdx=1.0 / 9000.0, rdy=1.0 / 9000.0):
    """Differentiable calc_coef_w: returns (a, alpha, gamma)."""
    return CoefW.apply(mut, cqw, c2a, rdn, rdnw, dts, epssm, top_lid, rdx, rdy)


def capture(run: Callable[[], object], warmup: int = 2) -> torch.cuda.CUDAGraph:
    """Capture ``run`` -- a forward and its backward through these
    Functions, with fixed input tensors and cotangent seeds -- in a CUDA
    graph, after ``warmup`` eager runs on a side stream; ``graph.replay()``
    then re-runs every kernel of the pass with no host work between them.
    Every Function launches on the current stream, reads its scalars from
    the host arguments (no device-to-host read inside a step) and takes its
    scratch from torch's allocator (the graph's private pool during
    capture), so a whole step forward + reverse is capturable.  The
    gradients that ``run`` leaves (``.grad`` of the leaves) live in the
    graph's pool and are rewritten by each replay."""
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(warmup):
            run()
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        run()
    return graph


def rollout(step: Callable[..., Sequence[torch.Tensor]], state: Sequence[torch.Tensor], n_steps: int,
            every: int = 1) -> tuple[torch.Tensor, ...]:
    """Apply ``state = step(*state)`` ``n_steps`` times, differentiably, with
    checkpoints every ``every`` steps: the forward keeps only the state at
    the start of each segment (plus whatever ``step`` closes over, e.g.
    learnable parameters, which receive their gradients as usual); the
    backward recomputes each segment's forward once, with its operators'
    hand-written adjoints recording what they need, and back-propagates
    through it.  Peak memory is then one segment's intermediates plus
    n_steps / every states, instead of every intermediate of every step.
    ``every=0`` keeps the whole forward (no recomputation)."""
    if n_steps < 0 or every < 0:
        raise ValueError("n_steps and every must be >= 0")
    state = tuple(state)

    def segment(k, *xs):
        for _ in range(k):
            xs = tuple(step(*xs))
        return xs

    done = 0
    while done < n_steps:
        k = n_steps - done if every == 0 else min(every, n_steps - done)
        if every == 0 or not torch.is_grad_enabled():
            state = segment(k, *state)
        else:
            state = tuple(checkpoint(segment, k, *state, use_reentrant=False))
        done += k
    return state


# the fields one acoustic substep reads (state) and the constant arrays it
# takes as data
SUBSTEP_STATE = ("u", "v", "ru_tend", "rv_tend", "p", "pb", "ph", "php", "alt", "al", "mu", "muu", "muv", "cqu", "cqv",
                 "mudf", "ww", "ww1", "u_save", "v_save", "t", "t_save", "t_2save", "t_tend", "mut", "muave", "muts",
                 "mu_tend", "w", "rw_tend", "w_save", "ph_save", "phb", "ph_tend", "ht", "c2a", "cqw", "a", "alpha",
                 "gamma", "ru_m", "rv_m", "ww_m", "pm1")
SUBSTEP_DATA = ("msfux", "msfuy", "msfvx", "msfvx_inv", "msfvy", "msftx", "msfty", "fnm", "fnp", "rdnw", "rdn", "dnw")


def acoustic_substep(st: dict, data: dict, iteration: int, nsub: int, dts: float, *, epssm: float, emdiv: float,
                     smdiv: float, cf1: float, cf2: float, cf3: float, rdx: float, rdy: float) -> dict:
    """One acoustic substep composed from the operators above, in the
    reference's order (pywrf/solver.py:1394-1445): advance_uv with the
    specified-row update of u and v, advance_mu_t, spec_bdyupdate of t, mu
    and muts, advance_w, sumflux, spec_bdyupdate_ph, zero_grad_bdy of w,
    calc_p_rho and the halo copies of ph, al, p, muts, mu and mudf.  ``st``
    maps SUBSTEP_STATE, ``data`` SUBSTEP_DATA to tensors; returns the state
    after the substep (a new dict).  Differentiable end to end: every piece
    is a hand-written reverse kernel, and the chain keeps only the operators'
    inputs."""
    s = dict(st)
    u, v = advance_uv({k: s[k] for k in UV_INPUTS}, {k: data[k] for k in UV_DATA}, dts, emdiv, cf1, cf2, cf3, rdx,
                      rdy)
    s["u"], s["v"] = u, v
    mt_in = {"ww": s["ww"], "ww_1": s["ww1"], "u": u, "u_1": s["u_save"], "v": v, "v_1": s["v_save"], "t": s["t"],
             "t_1": s["t_save"], "t_ave": s["t_2save"], "ft": s["t_tend"], "mu": s["mu"], "mut": s["mut"],
             "muave": s["muave"], "muts": s["muts"], "muu": s["muu"], "muv": s["muv"], "mudf": s["mudf"],
             "mu_tend": s["mu_tend"]}
    mt = advance_mu_t(mt_in, {k: data[k] for k in MUT_DATA}, dts, epssm, rdx, rdy)
    s.update(ww=mt["ww"], t=mt["t"], t_2save=mt["t_ave"], muave=mt["muave"], muts=mt["muts"], mudf=mt["mudf"],
             mu=mt["mu"])
    s["t"] = spec_bdyupdate(s["t"], s["t_tend"], dts, "t", rdx, rdy)
    s["mu"] = spec_bdyupdate(s["mu"], s["mu_tend"], dts, "m", rdx, rdy)
    s["muts"] = spec_bdyupdate(s["muts"], s["mu_tend"], dts, "m", rdx, rdy)
    aw_in = {k: s[k] for k in AW_INPUTS if k not in ("t_2ave", "t_2", "t_1", "ph_1")}
    aw_in.update(t_2ave=s["t_2save"], t_2=s["t"], t_1=s["t_save"], ph_1=s["ph_save"])
    aw = advance_w(aw_in, {k: data[k] for k in AW_DATA}, dts, epssm, cf1, cf2, cf3, rdx, rdy)
    s.update(t_2save=aw["t_2ave"], w=aw["w"], ph=aw["ph"])
    s["ru_m"], s["rv_m"], s["ww_m"] = sumflux({k: s[k] for k in SF_INPUTS}, {k: data[k] for k in SF_DATA},
                                              iteration, nsub, rdx, rdy)
    s["ph"] = spec_bdyupdate_ph({k: s[k] for k in SPH_INPUTS}, dts, rdx, rdy)
    s["w"] = zero_grad_w(s["w"], rdx, rdy)
    pr_in = {"al": s["al"], "p": s["p"], "ph": s["ph"], "alt": s["alt"], "t_2": s["t"], "t_1": s["t_save"],
             "c2a": s["c2a"], "pm1": s["pm1"], "mu": s["mu"], "mut": s["muts"]}
    s["al"], s["p"], s["pm1"] = calc_p_rho(pr_in, data["rdnw"], smdiv, iteration, rdx, rdy)
    s["ph"] = halo(s["ph"], "w", rdx, rdy)
    s["al"] = halo(s["al"], "p", rdx, rdy)
    s["p"] = halo(s["p"], "p", rdx, rdy)
    for k in ("muts", "mu", "mudf"):
        s[k] = halo(s[k], "t", rdx, rdy)
    return s


class _TableOp(torch.autograd.Function):
    """A state-table operator with a hand-written adjoint: ``op`` names the
    fields it reads (``op.fields``, the updated ones ``op.outputs`` among
    them), its constant arrays (``op.data``), and runs the forward
    (``op.fwd(cg, table, stream)``) and the reverse product
    (``op.adj(cg, table, bar_table, stream)``, which rewrites the outputs'
    cotangents to the inputs' and accumulates the rest)."""

    @staticmethod
    def forward(ctx, op, cg, *tensors):
        # outputs without a cotangent reach backward as None (its _bars / None
        # checks hand out zeros from one shared buffer) instead of one
        # zero-filled tensor each, which backward would then clone
        ctx.set_materialize_grads(False)
        _cuda_only(*tensors)
        named = dict(zip(op.fields + op.data, tensors))
        outs = {k: named[k].detach().clone() for k in op.outputs}
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(tensors[0].device):
            N.check(op.fwd(cg, _table({**named, **outs}), stream), op.name)
        ctx.save_for_backward(*tensors)
        ctx.op, ctx.cg = op, cg
        return tuple(outs[k] for k in op.outputs)

    @staticmethod
    def backward(ctx, *gouts):
        op = ctx.op
        saved = ctx.saved_tensors  # read once (checkpoint unpacks each saved tensor once)
        named = dict(zip(op.fields + op.data, saved))
        bars = _bars(named, op.fields, dict(zip(op.outputs, gouts)))
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(saved[0].device):
            N.check(op.adj(ctx.cg, _table(named), _table(bars), stream), op.name + "_adj")
        return (None, None) + tuple(bars[k] for k in op.fields) + (None,) * len(op.data)


class _SmallStepPrep:
    name = "wrf_small_step_prep"
    fields = ("mu", "mu_1", "mub", "mudf", "muts", "mu_save", "muu", "muv", "muus", "muvs", "mut", "u", "u_1",
              "u_save", "v", "v_1", "v_save", "t", "t_1", "t_save", "w", "w_1", "w_save", "ph", "ph_1", "ph_save",
              "ww", "ww1", "c2a", "pb", "p", "alt")
    outputs = ("mu", "mu_1", "mudf", "muts", "mu_save", "muus", "muvs", "u", "u_1", "u_save", "v", "v_1", "v_save",
               "t", "t_1", "t_save", "w", "w_1", "w_save", "ph", "ph_1", "ph_save", "ww1", "c2a")
    data = ("msfuy", "msfvx_inv", "msfty")

    def __init__(self, rk_step, ny, nx, device):
        self.rk_step = rk_step
        self.work = torch.empty(3 * ny * nx, dtype=torch.float32, device=device)

    def fwd(self, cg, tab, stream):
        return N.lib().wrf_small_step_prep(ctypes.byref(cg), tab, self.rk_step, stream)

    def adj(self, cg, tab, btab, stream):
        return N.lib().wrf_small_step_prep_adj(ctypes.byref(cg), tab, btab, self.rk_step,
                                               ctypes.c_void_p(self.work.data_ptr()), stream)


class _SmallStepFinish:
    name = "wrf_small_step_finish"
    fields = ("u", "u_save", "v", "v_save", "w", "w_save", "ph", "ph_save", "ww", "ww1", "t", "t_save", "h_diabatic",
              "mu", "mu_save", "mut", "muts", "muu", "muv", "muus", "muvs")
    outputs = ("u", "v", "w", "ph", "ww", "t", "mu", "muus", "muvs")
    data = ("msfuy", "msfvx", "msfty")

    def __init__(self, dts, nsub, rk_step, ny, nx, device):
        self.dts, self.nsub, self.rk_step = dts, nsub, rk_step
        self.work = torch.empty(2 * ny * nx, dtype=torch.float32, device=device)

    def fwd(self, cg, tab, stream):
        return N.lib().wrf_small_step_finish(ctypes.byref(cg), tab, self.dts, self.nsub, self.rk_step, stream)

    def adj(self, cg, tab, btab, stream):
        return N.lib().wrf_small_step_finish_adj(ctypes.byref(cg), tab, btab, self.dts, self.nsub, self.rk_step,
                                                 ctypes.c_void_p(self.work.data_ptr()), stream)


def small_step_prep(st: dict, data: dict, rk_step: int, rdx, rdy) -> dict:
    """Differentiable small_step_prep (pywrf/wrf_dynamics.py:3152-3266):
    returns ``st`` with the fields it updates replaced."""
    nz, ny, nx = st["u"].shape
    op = _SmallStepPrep(rk_step, ny, nx, st["u"].device)
    cg = scalar_grid(st["u"].shape, rdx, rdy)
    outs = _TableOp.apply(op, cg, *[st[k] for k in op.fields], *[data[k] for k in op.data])
    return {**st, **dict(zip(op.outputs, outs))}


def small_step_finish(st: dict, data: dict, dts: float, nsub: int, rk_step: int, rdx, rdy) -> dict:
    """Differentiable calc_mu_uv_1 + small_step_finish
    (pywrf/wrf_dynamics.py:3844-3930): returns ``st`` with the fields they
    update replaced."""
    nz, ny, nx = st["u"].shape
    op = _SmallStepFinish(dts, nsub, rk_step, ny, nx, st["u"].device)
    cg = scalar_grid(st["u"].shape, rdx, rdy)
    outs = _TableOp.apply(op, cg, *[st[k] for k in op.fields], *[data[k] for k in op.data])
    return {**st, **dict(zip(op.outputs, outs))}


# the fields the acoustic part of an RK stage reads (state) and its constant
# arrays (data)
STAGE_STATE = SUBSTEP_STATE + ("h_diabatic", "mu_1", "mu_save", "mub", "muus", "muvs", "ph_1", "t_1", "u_1", "v_1",
                               "w_1")
STAGE_DATA = SUBSTEP_DATA


def acoustic_stage(st: dict, data: dict, rk_step: int, nsub: int, dts: float, *, epssm: float, emdiv: float,
                   smdiv: float, cf1: float, cf2: float, cf3: float, rdx: float, rdy: float,
                   top_lid: bool = False) -> dict:
    """The acoustic part of one RK stage composed from the operators'
    Functions, in the reference's order (pywrf/solver.py:1258-1492):
    small_step_prep, calc_p_rho at step 0, calc_coef_w, the halo copies that
    follow them, ``nsub`` substeps (:func:`acoustic_substep`), calc_mu_uv_1
    with small_step_finish, and at the last stage the halo copies of the
    averaged fluxes and column masses.  ``st`` maps every field these read;
    returns the state after the stage."""
    s = small_step_prep(st, data, rk_step, rdx, rdy)
    pr = {"al": s["al"], "p": s["p"], "ph": s["ph"], "alt": s["alt"], "t_2": s["t"], "t_1": s["t_save"],
          "c2a": s["c2a"], "pm1": s["pm1"], "mu": s["mu"], "mut": s["muts"]}
    s["al"], s["p"], s["pm1"] = calc_p_rho(pr, data["rdnw"], smdiv, 0, rdx, rdy)
    s["a"], s["alpha"], s["gamma"] = coef_w(s["mut"], s["cqw"], s["c2a"], data["rdn"], data["rdnw"], dts, epssm,
                                            top_lid, rdx, rdy)
    for k, var in (("ru_tend", "u"), ("rv_tend", "v"), ("ph", "w"), ("al", "p"), ("p", "p"), ("t_1", "t"),
                   ("t_save", "t"), ("mu_1", "t"), ("mu", "t"), ("mudf", "t")):
        s[k] = halo(s[k], var, rdx, rdy)
    sc = dict(epssm=epssm, emdiv=emdiv, smdiv=smdiv, cf1=cf1, cf2=cf2, cf3=cf3, rdx=rdx, rdy=rdy)
    for it in range(1, nsub + 1):
        s = acoustic_substep(s, data, it, nsub, dts, **sc)
    s = small_step_finish(s, data, dts, nsub, rk_step, rdx, rdy)
    if rk_step == 3:
        for k, var in (("ru_m", "u"), ("rv_m", "v"), ("ww_m", "w"), ("mut", "t"), ("muts", "t")):
            s[k] = halo(s[k], var, rdx, rdy)
    return s


class _Addtend:
    name = "wrf_addtend"
    fields = ("ru_tend", "rv_tend", "rw_tend", "ph_tend", "t_tend", "mu_tend", "ru_tendf", "rv_tendf", "rw_tendf",
              "ph_tendf", "t_tendf", "mu_tendf", "u_save", "v_save", "w_save", "ph_save", "t_save", "h_diabatic", "mut")
    outputs = ("ru_tend", "rv_tend", "rw_tend", "ph_tend", "t_tend", "mu_tend", "ru_tendf", "rv_tendf", "rw_tendf",
               "ph_tendf", "t_tendf")
    data = ("msfty", "msfuy", "msfvx", "msfvx_inv")

    def __init__(self, rk_step):
        self.rk_step = rk_step

    def fwd(self, cg, tab, stream):
        return N.lib().wrf_addtend(ctypes.byref(cg), tab, self.rk_step, stream)

    def adj(self, cg, tab, btab, stream):
        return N.lib().wrf_addtend_adj(ctypes.byref(cg), tab, btab, self.rk_step, stream)


def addtend(st: dict, data: dict, rk_step: int, rdx, rdy) -> dict:
    """Differentiable rk_addtend_dry (pywrf/wrf_dynamics.py:3100-3148):
    returns ``st`` with the tendencies (and at stage 1 the physics
    tendencies) replaced."""
    op = _Addtend(rk_step)
    cg = scalar_grid(st["ru_tend"].shape, rdx, rdy)
    outs = _TableOp.apply(op, cg, *[st[k] for k in op.fields], *[data[k] for k in op.data])
    return {**st, **dict(zip(op.outputs, outs))}


class SpecBdytend(torch.autograd.Function):
    """tend' = spec_bdytend(tend, boundary tendencies, var): the specified
    rows take the boundary file's tendency (data); ``scal`` = (var, rdx,
    rdy), then the x-start, x-end, y-start, y-end boundary tendencies."""

    @staticmethod
    def forward(ctx, scal, tend, txs, txe, tys, tye):
        _cuda_only(tend, txs, txe, tys, tye)
        var = str(scal[0])
        shape = (12,) + tuple(tend.shape) if tend.dim() == 2 else tend.shape
        cg = scalar_grid(shape, float(scal[1]), float(scal[2]))
        out = tend.detach().clone()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(tend.device):
            rc = N.lib().wrf_spec_bdytend(ctypes.byref(cg), _ptr(out), _ptr(txs), _ptr(txe), _ptr(tys), _ptr(tye),
                                          var.encode(), stream)
        N.check(rc, "wrf_spec_bdytend")
        ctx.cg, ctx.var = cg, var
        return out

    @staticmethod
    def backward(ctx, gout):
        gin = gout.contiguous().clone()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(gin.device):
            rc = N.lib().wrf_spec_bdytend_adj(ctypes.byref(ctx.cg), _ptr(gin), ctx.var.encode(), stream)
        N.check(rc, "wrf_spec_bdytend_adj")
        return None, gin, None, None, None, None


def spec_bdytend(tend, bt: dict, var: str, rdx, rdy):
    """Differentiable spec_bdytend; ``bt`` maps txs txe tys tye to the
    variable's boundary tendencies (solver layout)."""
    return SpecBdytend.apply((var, rdx, rdy), tend, bt["txs"], bt["txe"], bt["tys"], bt["tye"])


HDIFF_DATA = ("msfux", "msfuy", "msfvx", "msfvy", "msftx", "msfty", "msfvx_inv")


class HorizontalDiffusion(torch.autograd.Function):
    """tend' = tend + horizontal_diffusion(field) (pywrf/wrf_dynamics.py:
    2623-2915): ``scal`` = (var, rdx, rdy) with var 'u', 'v', 'w' or 'm' (a
    mass-point scalar; with ``base``, the diffusion of field - base as
    horizontal_diffusion_3dmp forms it), then the field, the incoming
    tendency, the column mass, the eddy viscosity, ``base`` (data, or None)
    and the seven map factors of HDIFF_DATA; gradients with respect to the
    field, the tendency, the mass and the viscosity."""

    @staticmethod
    def forward(ctx, scal, field, tend, mut, xk, base, *maps):
        _cuda_only(field, tend, mut, xk, base, *maps)
        var = str(scal[0])
        cg = scalar_grid(field.shape, float(scal[1]), float(scal[2]))
        out = tend.detach().clone()
        tab = _table(dict(zip(HDIFF_DATA, maps)))
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        bp = None if base is None else _ptr(base)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_horizontal_diffusion(ctypes.byref(cg), tab, var.encode(), _ptr(field), bp, _ptr(mut),
                                                  _ptr(xk), _ptr(out), stream)
        N.check(rc, "wrf_horizontal_diffusion")
        ctx.cg, ctx.var, ctx.has_base = cg, var, base is not None
        ctx.save_for_backward(field, mut, xk, *(() if base is None else (base,)), *maps)
        return out

    @staticmethod
    def backward(ctx, gout):
        saved = ctx.saved_tensors
        field, mut, xk = saved[:3]
        base = saved[3] if ctx.has_base else None
        maps = saved[4:] if ctx.has_base else saved[3:]
        gout = gout.contiguous()
        fb, mb, kb = _zeros(field, mut, xk)
        tab = _table(dict(zip(HDIFF_DATA, maps)))
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        bp = None if base is None else _ptr(base)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_horizontal_diffusion_adj(ctypes.byref(ctx.cg), tab, ctx.var.encode(), _ptr(field), bp,
                                                      _ptr(mut), _ptr(xk), _ptr(gout), _ptr(fb), _ptr(mb), _ptr(kb),
                                                      stream)
        N.check(rc, "wrf_horizontal_diffusion_adj")
        return (None, fb, gout, mb, kb, None) + (None,) * len(HDIFF_DATA)


def horizontal_diffusion(var: str, field, tend, mut, xk, data: dict, rdx, rdy, base=None):
    """Differentiable ``tend + horizontal_diffusion(field)``; ``data`` maps
    the map factors of HDIFF_DATA."""
    return HorizontalDiffusion.apply((var, rdx, rdy), field, tend, mut, xk, base, *[data[k] for k in HDIFF_DATA])


class MassWeight(torch.autograd.Function):
    """out = field * mut on levels below nk of the mass points, zero elsewhere
    (mass_weight, pywrf/wrf_boundary.py:408-414); ``scal`` = (nk, rdx, rdy)."""

    @staticmethod
    def forward(ctx, scal, field, mut):
        _cuda_only(field, mut)
        nk = int(scal[0])
        cg = scalar_grid(field.shape, float(scal[1]), float(scal[2]))
        out = torch.zeros_like(field)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(field.device):
            N.check(N.lib().wrf_mass_weight(ctypes.byref(cg), _ptr(field), _ptr(mut), _ptr(out), nk, stream),
                    "wrf_mass_weight")
        ctx.cg, ctx.nk = cg, nk
        ctx.save_for_backward(field, mut)
        return out

    @staticmethod
    def backward(ctx, gout):
        field, mut = ctx.saved_tensors
        gout = gout.contiguous()
        fb, mb = _zeros(field, mut)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        with torch.cuda.device(field.device):
            rc = N.lib().wrf_mass_weight_adj(ctypes.byref(ctx.cg), _ptr(field), _ptr(mut), _ptr(gout), _ptr(fb),
                                             _ptr(mb), ctx.nk, stream)
        N.check(rc, "wrf_mass_weight_adj")
        return None, fb, mb


def mass_weight(field, mut, nk: int, rdx, rdy):
    """Differentiable mass_weight on levels below ``nk``."""
    return MassWeight.apply((nk, rdx, rdy), field, mut)


class _EddyViscosity:
    name = "wrf_eddy_viscosity"
    fields = ("u", "v", "ph", "xkmh", "xkhh")
    outputs = ("xkmh", "xkhh")
    data = ("phb", "msfux", "msfuy", "msfvx", "msfvy", "msftx", "msfty", "fnm", "fnp", "dn", "dnw")
    scratch = ("rdzw", "zx", "zy", "defor11", "defor22", "defor12")

    def __init__(self, like):
        n3 = like.numel()
        self.buf = torch.empty(len(self.scratch) * n3, dtype=torch.float32, device=like.device)
        self.views = [self.buf[q * n3:(q + 1) * n3] for q in range(len(self.scratch))]
        self.work = torch.empty(6 * n3, dtype=torch.float32, device=like.device)

    def _scratch(self, tab):
        names = N.field_names()
        for k, v in zip(self.scratch, self.views):
            tab[names.index(k)] = v.data_ptr()

    def fwd(self, cg, tab, stream):
        self._scratch(tab)
        return N.lib().wrf_eddy_viscosity(ctypes.byref(cg), tab, stream)

    def adj(self, cg, tab, btab, stream):
        self._scratch(tab)
        return N.lib().wrf_eddy_viscosity_adj(ctypes.byref(cg), tab, btab, ctypes.c_void_p(self.work.data_ptr()),
                                              stream)


def eddy_viscosity(st: dict, data: dict, rdx, rdy, cf1: float, cf2: float, cf3: float):
    """Differentiable first-stage eddy viscosities (compute_diff_metrics,
    cal_deform_and_div, calculate_km_kh: pywrf/wrf_dynamics.py:491-995) from
    u, v and ph; returns (xkmh, xkhh).  ``st`` also maps the incoming xkmh
    and xkhh (which survive outside the formula's region)."""
    op = _EddyViscosity(st["u"])
    cg = scalar_grid(st["u"].shape, rdx, rdy)
    cg.cf1, cg.cf2, cg.cf3 = float(cf1), float(cf2), float(cf3)
    return _TableOp.apply(op, cg, *[st[k] for k in op.fields], *[data[k] for k in op.data])


# the fields the dynamics part of an RK stage reads (state) beyond the
# acoustic stage's, and its constant arrays (data)
DYN_STATE = tuple(dict.fromkeys(STAGE_STATE + PREP_FIELDS + FORCES_INPUTS + _Addtend.fields +
                                ("moist", "xkmh", "xkhh", "moist_tend")))
DYN_DATA = tuple(dict.fromkeys(STAGE_DATA + PREP_DATA + FORCES_DATA + _Addtend.data + _EddyViscosity.data +
                               HDIFF_DATA + ("t_init",)))


def _first_stage_diffusion(s: dict, data: dict, bdy: dict, dtbc: float, rdx, rdy) -> dict:
    """The first stage's horizontal diffusion of u, v, w and theta into the
    physics tendencies and the lateral relaxation into the saved fields
    (pywrf/solver.py:1112-1203)."""
    hd = {k: data[k] for k in HDIFF_DATA}
    for name in ("u", "v", "w"):
        s[f"r{name}_tendf"] = horizontal_diffusion(name, s[name], s[f"r{name}_tendf"], s["mut"], s["xkmh"], hd,
                                                   rdx, rdy)
    s["t_tendf"] = horizontal_diffusion("m", s["t"], s["t_tendf"], s["mut"], s["xkhh"], hd, rdx, rdy,
                                        base=data["t_init"])
    nz = s["u"].shape[0]
    s["u_save"] = relax_bdytend(s["ru"], s["u_save"], "u", dtbc, bdy["u"])
    s["v_save"] = relax_bdytend(s["rv"], s["v_save"], "v", dtbc, bdy["v"])
    s["ph_save"] = relax_bdytend(mass_weight(s["ph"], s["mut"], nz, rdx, rdy), s["ph_save"], "h", dtbc, bdy["h"])
    s["t_save"] = relax_bdytend(mass_weight(s["t"], s["mut"], nz, rdx, rdy), s["t_save"], "t", dtbc, bdy["t"])
    s["mu_tend"] = relax_bdytend(s["mu"][None], s["mu_tend"][None], "m", dtbc, bdy["m"])[0]
    return s


def dynamics_stage(st: dict, data: dict, bt: dict, rk_step: int, nsub: int, dts: float, *, epssm: float,
                   emdiv: float, smdiv: float, cf1: float, cf2: float, cf3: float, cfn: float, cfn1: float,
                   rdx: float, rdy: float, dtbc: float | None = None, theta_bias=None) -> dict:
    """The dynamics of one RK stage composed from the operators' Functions,
    in the reference's order (pywrf/solver.py:736-1492): rk_step_prep and
    its halo copies; at the first stage the physics tendencies from zero, the
    eddy viscosities and their halo copies; the advection of u, v, w and
    theta, the tendency terms; at the first stage the horizontal diffusion
    and the lateral relaxation; rk_addtend_dry (then ``theta_bias``, when
    given, added to t_tend); spec_bdytend of u, v, ph, t, mu; and the
    acoustic part (:func:`acoustic_stage`).  ``bt`` maps 'u', 'v', 'h', 't',
    'm' to dicts of their boundary arrays (txs txe tys tye; at the first
    stage also xs xe ys ye, with ``dtbc`` the boundary time); returns the
    state after the acoustic steps."""
    if rk_step not in (1, 2, 3):
        raise ValueError("rk_step is 1, 2 or 3")
    if rk_step == 1 and dtbc is None:
        raise ValueError("the first stage's relaxation needs dtbc")
    s = dict(st)
    s.update(prep({k: s[k] for k in PREP_FIELDS}, {k: data[k] for k in PREP_DATA}, 127, rdx, rdy))
    for k, var in (("ru", "u"), ("rv", "v"), ("rw", "w"), ("ww", "w"), ("php", "w"), ("alt", "t"), ("p", "p"),
                   ("muu", "u"), ("muv", "v"), ("mut", "t"), ("al", "p"), ("ph", "w")):
        s[k] = halo(s[k], var, rdx, rdy)
    if rk_step == 1:
        for k in ("ru_tendf", "rv_tendf", "rw_tendf", "ph_tendf", "t_tendf", "mu_tendf", "moist_tend"):
            s[k] = torch.zeros_like(st[k])
        s["xkmh"], s["xkhh"] = eddy_viscosity(s, data, rdx, rdy, cf1, cf2, cf3)
        s["xkmh"] = halo(s["xkmh"], "t", rdx, rdy)
        s["xkhh"] = halo(s["xkhh"], "t", rdx, rdy)
    for k in ("ru_tend", "rv_tend", "rw_tend", "t_tend", "ph_tend", "u_save", "v_save", "w_save", "ph_save",
              "t_save", "mu_tend", "mu_save"):
        s[k] = torch.zeros_like(st[k])
    z = lambda k: s[k]  # noqa: E731
    s["ru_tend"] = advect_momentum(0, s["u"], z("ru_tend"), s["ru"], s["rv"], s["ww"], data["msfux"], None,
                                   data["fnm"], data["fnp"], data["rdnw"], rdx, rdy)
    s["rv_tend"] = advect_momentum(1, s["v"], z("rv_tend"), s["ru"], s["rv"], s["ww"], data["msfvy"], data["msfvx"],
                                   data["fnm"], data["fnp"], data["rdnw"], rdx, rdy)
    s["rw_tend"] = advect_momentum(2, s["w"], z("rw_tend"), s["ru"], s["rv"], s["ww"], data["msftx"], None,
                                   data["fnm"], data["fnp"], data["rdn"], rdx, rdy)
    s["t_tend"] = advect_scalar(s["t"], z("t_tend"), s["ru"], s["rv"], s["ww"], data["msftx"], data["fnm"],
                                data["fnp"], data["rdnw"], rdx, rdy)
    outs = forces({k: s[k] for k in FORCES_INPUTS}, {k: data[k] for k in FORCES_DATA}, 31, rdx, rdy, cf1, cf2, cf3,
                  cfn, cfn1)
    s.update(dict(zip(FORCES_OUTPUTS, outs)))
    if rk_step == 1:
        s = _first_stage_diffusion(s, data, bt, dtbc, rdx, rdy)
    s = addtend(s, data, rk_step, rdx, rdy)
    if theta_bias is not None:
        s["t_tend"] = s["t_tend"] + theta_bias
    for k, var in (("ru_tend", "u"), ("rv_tend", "v"), ("ph_tend", "h"), ("t_tend", "t"), ("mu_tend", "m")):
        s[k] = spec_bdytend(s[k], bt[var], var, rdx, rdy)
    return acoustic_stage(s, data, rk_step, nsub, dts, epssm=epssm, emdiv=emdiv, smdiv=smdiv, cf1=cf1, cf2=cf2,
                          cf3=cf3, rdx=rdx, rdy=rdy)


class _MoistUpdate:
    name = "wrf_moist_update"
    fields = ("moist", "moist_old", "moist_tend", "advect_tend", "mu", "mu_1", "mub", "al", "alb", "muts", "ph", "p",
              "pb", "t")
    outputs = ("moist", "moist_old", "al", "p")
    data = ("msfty", "ru_m", "rv_m", "rdnw")

    def __init__(self, rk_step, dt_rk, like):
        self.rk_step, self.dt_rk = rk_step, float(dt_rk)
        self.work = torch.empty(like.numel(), dtype=torch.float32, device=like.device)
        self.status = torch.zeros(16, dtype=torch.int32, device=like.device)

    def fwd(self, cg, tab, stream):
        tab[N.field_names().index("status")] = self.status.data_ptr()
        return N.lib().wrf_moist_update(ctypes.byref(cg), tab, self.rk_step, self.dt_rk, stream)

    def adj(self, cg, tab, btab, stream):
        tab[N.field_names().index("status")] = self.status.data_ptr()
        return N.lib().wrf_moist_update_adj(ctypes.byref(cg), tab, btab, self.rk_step, self.dt_rk,
                                            ctypes.c_void_p(self.work.data_ptr()), stream)


def moist_stage(st: dict, data: dict, rk_step: int, dt_rk: float, rdx, rdy, bt: dict | None = None,
                dtbc: float | None = None) -> dict:
    """The moisture part of an RK stage after its acoustic steps, composed
    from the operators' Functions (pywrf/solver.py:1548-1712): advection of
    qv .. qg by the averaged fluxes; at the first stage the horizontal
    diffusion of each species (mass muts, viscosity xkhh), and the relaxation
    and specified tendency of qv (``bt['q']``: its eight boundary arrays,
    ``dtbc`` the boundary time); rk_update_scalar, flow_dep_bdy of qc .. qg,
    calc_p_rho_phi and, before the last stage, the halo copies."""
    s = dict(st)
    moist = s["moist"]
    adv = [torch.zeros_like(moist[0])]
    for im in range(1, 7):
        adv.append(advect_scalar(moist[im], torch.zeros_like(moist[im]), s["ru_m"], s["rv_m"], s["ww_m"],
                                 data["msftx"], data["fnm"], data["fnp"], data["rdnw"], rdx, rdy))
    s["advect_tend"] = torch.stack(adv)
    if rk_step == 1:
        if bt is None or dtbc is None:
            raise ValueError("the first stage's qv relaxation needs its boundary arrays and dtbc")
        hd = {k: data[k] for k in HDIFF_DATA}
        mt = s["moist_tend"]
        tends = [mt[0]] + [horizontal_diffusion("m", moist[im], mt[im], s["muts"], s["xkhh"], hd, rdx, rdy)
                           for im in range(1, 7)]
        nz = moist.shape[1]
        rq = mass_weight(moist[1], s["mut"], nz - 1, rdx, rdy)
        tends[1] = spec_bdytend(relax_bdytend(rq, tends[1], "t", dtbc, bt["q"]), bt["q"], "t", rdx, rdy)
        s["moist_tend"] = torch.stack(tends)
    op = _MoistUpdate(rk_step, dt_rk, moist[0])
    cg = scalar_grid(s["u"].shape, rdx, rdy)
    dd = {"msfty": data["msfty"], "ru_m": s["ru_m"].detach(), "rv_m": s["rv_m"].detach(), "rdnw": data["rdnw"]}
    outs = _TableOp.apply(op, cg, *[s[k] for k in op.fields], *[dd[k] for k in op.data])
    s.update(dict(zip(op.outputs, outs)))
    if rk_step < 3:
        for k, var in (("u", "U"), ("v", "V"), ("w", "w"), ("t", "p"), ("ph", "w"), ("mu", "t")):
            s[k] = halo(s[k], var, rdx, rdy)
        m = s["moist"]
        s["moist"] = torch.stack([m[0]] + [halo(m[im], "p", rdx, rdy) for im in range(1, 7)])
    return s


RK_STATE = tuple(dict.fromkeys(DYN_STATE + _MoistUpdate.fields + ("ru_m", "rv_m", "ww_m")))
RK_DATA = tuple(dict.fromkeys(DYN_DATA + ("msftx", "fnm", "fnp", "rdnw")))


def rk_stage(st: dict, data: dict, bt: dict, rk_step: int, nsub: int, dts: float, dt_rk: float, **sc) -> dict:
    """One RK stage of the step, composed: :func:`dynamics_stage` then
    :func:`moist_stage`; ``sc`` as for :func:`dynamics_stage` (at the first
    stage ``bt`` also holds 'q', qv's boundary arrays)."""
    s = dynamics_stage(st, data, bt, rk_step, nsub, dts, **sc)
    return moist_stage(s, data, rk_step, dt_rk, sc["rdx"], sc["rdy"], bt, sc.get("dtbc"))


BDY_FINAL_ARRAYS = tuple(f"{v}_{n}" for v in ("u", "v", "t", "ph", "qv")
                         for n in ("bxs", "bxe", "bys", "bye", "btxs", "btxe", "btys", "btye"))


class _BdyFinal:
    name = "wrf_bdy_final"
    fields = ("u", "v", "t", "ph", "moist", "w", "muus", "muvs", "muts")
    outputs = ("u", "v", "t", "ph", "moist", "w")
    data = ("msfuy", "msfvx", "msftx", "msfty", "ht", "dscal") + BDY_FINAL_ARRAYS

    def fwd(self, cg, tab, stream):
        return N.lib().wrf_bdy_final(ctypes.byref(cg), tab, stream)

    def adj(self, cg, tab, btab, stream):
        return N.lib().wrf_bdy_final_adj(ctypes.byref(cg), tab, btab, stream)


def boundary_arrays(bdy: dict) -> dict:
    """The state table's boundary-array fields (u_bxs .. qv_btye) from
    per-variable dicts in the solver layout ('u', 'v', 't', 'ph', 'qv' each
    mapping xs xe ys ye txs txe tys tye)."""
    out = {}
    for v in ("u", "v", "t", "ph", "qv"):
        for n, key in (("bxs", "xs"), ("bxe", "xe"), ("bys", "ys"), ("bye", "ye"), ("btxs", "txs"),
                       ("btxe", "txe"), ("btys", "tys"), ("btye", "tye")):
            out[f"{v}_{n}"] = bdy[v][key]
    return out


def step_end(st: dict, data: dict, bdy: dict, dtbc: float, *, cf1: float, cf2: float, cf3: float, rdx: float,
             rdy: float) -> dict:
    """The end of a step after its microphysics, composed
    (pywrf/solver.py:1776-1910): the halo copies of u_1, u, v_1, v, w_1, w,
    t_1, t, ph_1, ph, mu_1, mu and qv .. qg, spec_bdy_final of u, v, t, ph,
    qv and set_w_surface.  ``bdy`` maps 'u', 'v', 't', 'ph', 'qv' to their
    boundary arrays (xs .. tye)."""
    s = dict(st)
    for k, var in (("u_1", "U"), ("u", "U"), ("v_1", "V"), ("v", "V"), ("w_1", "w"), ("w", "w"), ("t_1", "p"),
                   ("t", "p"), ("ph_1", "w"), ("ph", "w"), ("mu_1", "t"), ("mu", "t")):
        s[k] = halo(s[k], var, rdx, rdy)
    m = s["moist"]
    s["moist"] = torch.stack([m[0]] + [halo(m[im], "p", rdx, rdy) for im in range(1, 7)])
    op = _BdyFinal()
    cg = scalar_grid(s["u"].shape, rdx, rdy)
    cg.cf1, cg.cf2, cg.cf3 = float(cf1), float(cf2), float(cf3)
    dscal = torch.zeros(16, dtype=torch.float32, device=s["u"].device)
    dscal[:1].fill_(float(dtbc))  # a fill launch, not a host copy: the step stays capturable in a CUDA graph
    dd = {**{k: data[k] for k in ("msfuy", "msfvx", "msftx", "msfty", "ht")}, "dscal": dscal,
          **boundary_arrays(bdy)}
    outs = _TableOp.apply(op, cg, *[s[k] for k in op.fields], *[dd[k] for k in op.data])
    s.update(dict(zip(op.outputs, outs)))
    return s


class _Microphysics:
    """The step's microphysics (moist_physics_prep_em, WSM6,
    moist_physics_finish_em, calc_p_rho_phi) as a table operator; the
    precipitation accumulators and the diagnostic tendencies it also writes
    go to scratch (they do not feed back into the state)."""
    name = "wrf_microphysics_op"
    fields = ("t", "moist", "al", "p", "ph", "h_diabatic", "mu", "muts")
    outputs = ("t", "moist", "al", "p", "h_diabatic")
    data = ("alb", "pb", "phb", "rdnw")
    scratch3 = ("qv_diabatic", "qc_diabatic", "wsm_t", "wsm_qr0s")
    scratch2 = ("rainnc", "rainncv", "snownc", "snowncv", "graupelnc", "graupelncv", "sr")

    def __init__(self, like):
        nz, ny, nx = like.shape
        dev = like.device
        self.s3 = {k: torch.zeros(nz, ny, nx, dtype=torch.float32, device=dev) for k in self.scratch3}
        self.s2 = {k: torch.zeros(ny, nx, dtype=torch.float32, device=dev) for k in self.scratch2}
        self.dbar = {k: torch.zeros(nz, ny, nx, dtype=torch.float32, device=dev) for k in ("alb", "pb")}

    def _scratch(self, tab):
        names = N.field_names()
        for k, v in {**self.s3, **self.s2}.items():
            tab[names.index(k)] = v.data_ptr()

    def fwd(self, cg, tab, stream):
        self._scratch(tab)
        return N.lib().wrf_microphysics_op(ctypes.byref(cg), tab, stream)

    def adj(self, cg, tab, btab, stream):
        names = N.field_names()
        # the state after the block, recomputed from clones of the inputs it
        # updates (the other fields are the same tensors)
        ptab = (ctypes.c_void_p * len(names))()
        for q in range(len(names)):
            ptab[q] = tab[q]
        clones = {k: self._saved[k].detach().clone() for k in self.outputs}
        for k, v in clones.items():
            ptab[names.index(k)] = v.data_ptr()
        self._scratch(ptab)
        rc = N.lib().wrf_microphysics_op(ctypes.byref(cg), ptab, stream)
        if rc:
            return rc
        for k, v in self.dbar.items():
            btab[names.index(k)] = v.data_ptr()
        n = ctypes.c_size_t(0)
        rc = N.lib().wrf_microphysics_adj_work(ctypes.byref(cg), ctypes.byref(n))
        if rc:
            return rc
        work = torch.empty(int(n.value), dtype=torch.float32, device=clones["t"].device)
        return N.lib().wrf_microphysics_adj(ctypes.byref(cg), tab, ptab, btab, ctypes.c_void_p(work.data_ptr()), n,
                                            None, stream)


def microphysics(st: dict, data: dict, dt: float, rdx, rdy) -> dict:
    """Differentiable microphysics of the step (pywrf/solver.py:1714-1766):
    returns ``st`` with t, moist, al, p and h_diabatic replaced.  Its reverse
    is the equation of state's exact reverse, then prep + WSM6 + finish in
    reverse mode: each column of a restatement of the scheme runs once on
    taped scalars and one reverse sweep of its tape gives its inputs'
    cotangents (forward-mode tangents for a column whose tape outgrows the
    capacity)."""
    op = _Microphysics(st["t"])
    cg = scalar_grid(st["t"].shape, rdx, rdy)
    cg.dt = float(dt)
    op._saved = {k: st[k] for k in op.outputs}
    outs = _TableOp.apply(op, cg, *[st[k] for k in op.fields], *[data[k] for k in op.data])
    return {**st, **dict(zip(op.outputs, outs))}


STEP_DATA = tuple(dict.fromkeys(RK_DATA + ("msfuy", "msfvx", "msftx", "msfty", "ht")))


def step(st: dict, data: dict, bdy: dict, dtbc: float, *, dt: float, soundsteps: int, microphysics=None,
         theta_bias=None, **sc) -> dict:
    """One time step composed from the operators' Functions
    (pywrf/solver.py:709-1910): the three RK stages (:func:`rk_stage`), then
    ``microphysics`` (a differentiable callable on the state dict, or None
    for none: the step of a model without microphysics), then
    :func:`step_end`.  ``bdy`` maps 'u', 'v', 'ph', 't', 'mu', 'qv' to their
    boundary arrays (xs .. tye); ``sc`` holds epssm, emdiv, smdiv, cf1, cf2,
    cf3, cfn, cfn1, rdx, rdy; ``theta_bias`` is added to t_tend in every
    stage."""
    bt = {"u": bdy["u"], "v": bdy["v"], "h": bdy["ph"], "t": bdy["t"], "m": bdy["mu"], "q": bdy["qv"]}
    s = dict(st)
    for rk in (1, 2, 3):
        nsub = {1: 1, 2: soundsteps // 2, 3: soundsteps}[rk]
        dts = dt / 3.0 if rk == 1 else dt / soundsteps
        dt_rk = {1: dt / 3.0, 2: 0.5 * dt, 3: dt}[rk]
        s = rk_stage(s, data, bt, rk, nsub, dts, dt_rk, dtbc=dtbc, theta_bias=theta_bias, **sc)
    if microphysics is not None:
        s = microphysics(s)
    return step_end(s, data, bdy, dtbc, cf1=sc["cf1"], cf2=sc["cf2"], cf3=sc["cf3"], rdx=sc["rdx"], rdy=sc["rdy"])
