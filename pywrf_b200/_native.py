"""ctypes binding of the C ABI in ``include/pywrf_b200.h``.

The library is ``pywrf_b200/lib/libpywrf_b200.so`` (built in-tree by
:mod:`pywrf_b200.build`).  There is no fallback: if the library is missing or
cannot be loaded, :func:`lib` raises and nothing runs.
"""
from __future__ import annotations

import ctypes
import os

from .build import LIB

WRF_OK = 0
WRF_EINVAL = -1
WRF_ECUDA = -2

WRF_K3, WRF_K2, WRF_K1, WRF_K4 = 3, 2, 1, 4
WRF_KBX, WRF_KBY, WRF_KBX2, WRF_KBY2 = 10, 11, 12, 13
WRF_KSF, WRF_KSI = 20, 21

WRF_ST_NAN_P = 0
WRF_ST_STEP = 1
WRF_ST_WAIT = 2
WRF_FORM_FAST = 0
WRF_FORM_POINT = 1


class WrfGridC(ctypes.Structure):
    """``WrfGrid`` of include/pywrf_b200.h"""
    _fields_ = [(n, ctypes.c_int) for n in ("nx", "ny", "nz", "ids", "ide", "jds", "jde", "soundsteps",
                                             "spec_zone", "bdy_interval", "top_lid")] + \
               [(n, ctypes.c_float) for n in ("dx", "dy", "dt", "smdiv", "emdiv", "epssm", "khdif", "kvdif",
                                               "cf1", "cf2", "cf3", "cfn", "cfn1")]


PROBE_FN = ctypes.CFUNCTYPE(None, ctypes.c_char_p, ctypes.c_void_p)

WRF_MLP_LAYERS = 4
EPI_F32, EPI_BIAS_GELU, EPI_GELU_BWD, EPI_BF16 = 0, 1, 2, 3


class WrfMlpNetC(ctypes.Structure):
    """``WrfMlpNet`` of include/pywrf_b200.h"""
    _fields_ = [("dims", ctypes.c_int * (WRF_MLP_LAYERS + 1)), ("w", ctypes.c_void_p * WRF_MLP_LAYERS),
                ("b", ctypes.c_void_p * WRF_MLP_LAYERS), ("norm", ctypes.c_void_p), ("tol_neg", ctypes.c_float),
                ("tol_sat", ctypes.c_float)]


class WrfMlpWorkC(ctypes.Structure):
    """``WrfMlpWork`` of include/pywrf_b200.h"""
    _fields_ = [("capacity", ctypes.c_int), ("x", ctypes.c_void_p), ("h", ctypes.c_void_p * 2),
                ("y", ctypes.c_void_p), ("list", ctypes.c_void_p), ("err", ctypes.c_void_p),
                ("colstat", ctypes.c_void_p)]


_lib = None
_names: list[str] | None = None
_kinds: list[int] | None = None


class NativeLibraryError(RuntimeError):
    pass


def lib() -> ctypes.CDLL:
    """The loaded kernel library (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        raise NativeLibraryError(f"{LIB} is not built; run `python -m pywrf_b200.build` (needs nvcc)")
    try:
        L = ctypes.CDLL(LIB)
    except OSError as e:  # pragma: no cover - depends on the machine
        raise NativeLibraryError(f"cannot load {LIB}: {e}") from e
    vp, fp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int
    L.wrf_field_count.restype = ip
    L.wrf_field_name.restype = ctypes.c_char_p
    L.wrf_field_name.argtypes = [ip]
    L.wrf_field_kind.restype = ip
    L.wrf_field_kind.argtypes = [ip]
    L.wrf_last_error.restype = ctypes.c_char_p
    L.wrf_rk3_step.restype = ip
    L.wrf_rk3_step.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, PROBE_FN, vp]
    G0 = ctypes.POINTER(WrfGridC)
    for name in ("wrf_step_begin", "wrf_diff_stage1", "wrf_microphysics", "wrf_step_end"):
        getattr(L, name).restype = ip
        getattr(L, name).argtypes = [G0, vp, vp]
    for name in ("wrf_rk_prep", "wrf_tend_stage", "wrf_acoustic_prep", "wrf_acoustic_finish", "wrf_moist_stage"):
        getattr(L, name).restype = ip
        getattr(L, name).argtypes = [G0, vp, ip, vp]
    L.wrf_acoustic_substep.restype = ip
    L.wrf_acoustic_substep.argtypes = [G0, vp, ip, ip, vp]
    L.wrf_advect_scalar.restype = ip
    L.wrf_advect_scalar.argtypes = [ctypes.POINTER(WrfGridC)] + [vp] * 9 + [vp]
    L.wrf_set_kernel_form.restype = ip
    L.wrf_set_kernel_form.argtypes = [ctypes.c_int]
    L.wrf_advect_momentum.restype = ip
    L.wrf_advect_momentum.argtypes = [ctypes.POINTER(WrfGridC), ctypes.c_int] + [vp] * 10 + [ctypes.c_int, vp]
    L.wrf_advance_w.restype = ip
    L.wrf_advance_w.argtypes = [ctypes.POINTER(WrfGridC), vp, ctypes.c_float, vp]
    L.wrf_advance_w_adj.restype = ip
    L.wrf_advance_w_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.c_float, vp, vp]
    L.wrf_advance_mu_t.restype = ip
    L.wrf_advance_mu_t.argtypes = [ctypes.POINTER(WrfGridC), vp, ctypes.c_float, vp]
    L.wrf_advance_mu_t_adj.restype = ip
    L.wrf_advance_mu_t_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.c_float, ctypes.c_int, vp, vp]
    L.wrf_calc_p_rho.restype = ip
    L.wrf_calc_p_rho.argtypes = [ctypes.POINTER(WrfGridC), vp, ctypes.c_int, vp]
    L.wrf_calc_p_rho_adj.restype = ip
    L.wrf_calc_p_rho_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.c_int, vp]
    L.wrf_advance_uv.restype = ip
    L.wrf_advance_uv.argtypes = [ctypes.POINTER(WrfGridC), vp, ctypes.c_float, vp]
    L.wrf_forces.restype = ip
    L.wrf_forces.argtypes = [ctypes.POINTER(WrfGridC), vp, ip, vp]
    L.wrf_forces_adj.restype = ip
    L.wrf_forces_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ip, vp]
    L.wrf_sumflux.restype = ip
    L.wrf_sumflux.argtypes = [ctypes.POINTER(WrfGridC), vp, ip, ip, vp]
    L.wrf_sumflux_adj.restype = ip
    L.wrf_sumflux_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ip, ip, vp]
    L.wrf_spec_bdyupdate.restype = ip
    L.wrf_spec_bdyupdate.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.c_float, ctypes.c_char, vp]
    L.wrf_spec_bdyupdate_adj.restype = ip
    L.wrf_spec_bdyupdate_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.c_float, ctypes.c_char, vp]
    L.wrf_spec_bdyupdate_ph.restype = ip
    L.wrf_spec_bdyupdate_ph.argtypes = [ctypes.POINTER(WrfGridC), vp, ctypes.c_float, vp]
    L.wrf_spec_bdyupdate_ph_adj.restype = ip
    L.wrf_spec_bdyupdate_ph_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.c_float, vp]
    L.wrf_prep.restype = ip
    L.wrf_prep.argtypes = [ctypes.POINTER(WrfGridC), vp, ip, vp]
    L.wrf_prep_adj.restype = ip
    L.wrf_prep_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ip, vp]
    L.wrf_halo.restype = ip
    L.wrf_halo.argtypes = [ctypes.POINTER(WrfGridC), vp, ctypes.c_char, ip, vp]
    L.wrf_halo_adj.restype = ip
    L.wrf_halo_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.c_char, ip, vp]
    L.wrf_zero_grad_w.restype = ip
    L.wrf_zero_grad_w.argtypes = [ctypes.POINTER(WrfGridC), vp, vp]
    L.wrf_zero_grad_w_adj.restype = ip
    L.wrf_zero_grad_w_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, vp]
    L.wrf_small_step_prep.restype = ip
    L.wrf_small_step_prep.argtypes = [ctypes.POINTER(WrfGridC), vp, ip, vp]
    L.wrf_small_step_prep_adj.restype = ip
    L.wrf_small_step_prep_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ip, vp, vp]
    L.wrf_small_step_finish.restype = ip
    L.wrf_small_step_finish.argtypes = [ctypes.POINTER(WrfGridC), vp, ctypes.c_float, ip, ip, vp]
    L.wrf_small_step_finish_adj.restype = ip
    L.wrf_small_step_finish_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.c_float, ip, ip, vp, vp]
    L.wrf_addtend.restype = ip
    L.wrf_addtend.argtypes = [ctypes.POINTER(WrfGridC), vp, ip, vp]
    L.wrf_addtend_adj.restype = ip
    L.wrf_addtend_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ip, vp]
    L.wrf_spec_bdytend.restype = ip
    L.wrf_spec_bdytend.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, vp, vp, vp, ctypes.c_char, vp]
    L.wrf_spec_bdytend_adj.restype = ip
    L.wrf_spec_bdytend_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, ctypes.c_char, vp]
    L.wrf_eddy_viscosity.restype = ip
    L.wrf_eddy_viscosity.argtypes = [ctypes.POINTER(WrfGridC), vp, vp]
    L.wrf_eddy_viscosity_adj.restype = ip
    L.wrf_eddy_viscosity_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, vp, vp]
    L.wrf_horizontal_diffusion.restype = ip
    L.wrf_horizontal_diffusion.argtypes = [ctypes.POINTER(WrfGridC), vp, ctypes.c_char, vp, vp, vp, vp, vp, vp]
    L.wrf_horizontal_diffusion_adj.restype = ip
    L.wrf_horizontal_diffusion_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, ctypes.c_char, vp, vp, vp, vp, vp, vp,
                                               vp, vp, vp]
    L.wrf_mass_weight.restype = ip
    L.wrf_mass_weight.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, vp, ip, vp]
    L.wrf_mass_weight_adj.restype = ip
    L.wrf_mass_weight_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, vp, vp, vp, ip, vp]
    L.wrf_bdy_final.restype = ip
    L.wrf_bdy_final.argtypes = [ctypes.POINTER(WrfGridC), vp, vp]
    L.wrf_bdy_final_adj.restype = ip
    L.wrf_bdy_final_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, vp]
    L.wrf_microphysics_op.restype = ip
    L.wrf_microphysics_op.argtypes = [ctypes.POINTER(WrfGridC), vp, vp]
    L.wrf_microphysics_adj_work.restype = ip
    L.wrf_microphysics_adj_work.argtypes = [ctypes.POINTER(WrfGridC), ctypes.POINTER(ctypes.c_size_t)]
    L.wrf_microphysics_adj.restype = ip
    L.wrf_microphysics_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, vp, vp, ctypes.c_size_t, vp, vp]
    L.wrf_set_microphysics_tape_capacity.restype = ip
    L.wrf_set_microphysics_tape_capacity.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.wrf_calc_p_rho_phi.restype = ip
    L.wrf_calc_p_rho_phi.argtypes = [ctypes.POINTER(WrfGridC), vp, vp]
    L.wrf_moist_update.restype = ip
    L.wrf_moist_update.argtypes = [ctypes.POINTER(WrfGridC), vp, ip, ctypes.c_float, vp]
    L.wrf_moist_update_adj.restype = ip
    L.wrf_moist_update_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ip, ctypes.c_float, vp, vp]
    L.wrf_advance_uv_adj.restype = ip
    L.wrf_advance_uv_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.c_float, vp]
    L.wrf_advect_momentum_adj.restype = ip
    L.wrf_advect_momentum_adj.argtypes = [ctypes.POINTER(WrfGridC), ctypes.c_int] + [vp] * 15 + [ctypes.c_size_t, vp]
    L.wrf_advect_momentum_adj_work.restype = ip
    L.wrf_advect_momentum_adj_work.argtypes = [ctypes.POINTER(WrfGridC), ctypes.POINTER(ctypes.c_size_t)]
    L.wrf_advect_scalar_adj.restype = ip
    L.wrf_advect_scalar_adj.argtypes = [ctypes.POINTER(WrfGridC)] + [vp] * 14 + [ctypes.c_size_t, vp]
    L.wrf_advect_scalar_adj_work.restype = ip
    L.wrf_advect_scalar_adj_work.argtypes = [ctypes.POINTER(WrfGridC), ctypes.POINTER(ctypes.c_size_t)]
    L.wrf_relax_bdytend.restype = ip
    L.wrf_relax_bdytend.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.POINTER(ctypes.c_void_p), ctypes.c_char,
                                    ctypes.c_float, vp]
    L.wrf_relax_bdytend_adj.restype = ip
    L.wrf_relax_bdytend_adj.argtypes = [ctypes.POINTER(WrfGridC), vp, vp, ctypes.c_char, vp]
    L.wrf_vsolve_w.restype = ip
    L.wrf_vsolve_w.argtypes = [ip, ip] + [vp] * 5 + [vp]
    L.wrf_vsolve_w_adj.restype = ip
    L.wrf_vsolve_w_adj.argtypes = [ip, ip] + [vp] * 9 + [vp]
    L.wrf_coef_w.restype = ip
    L.wrf_coef_w.argtypes = [ctypes.POINTER(WrfGridC)] + [vp] * 5 + [ctypes.c_float] + [vp] * 3 + [vp]
    L.wrf_coef_w_adj.restype = ip
    L.wrf_coef_w_adj.argtypes = [ctypes.POINTER(WrfGridC)] + [vp] * 5 + [ctypes.c_float] + [vp] * 6 + [vp]
    L.wrf_wsm6.restype = ip
    L.wrf_wsm6.argtypes = [ctypes.POINTER(WrfGridC)] + [vp] * 11 + [ctypes.c_float] + [vp] * 7 + [vp]
    L.wrf_wsm6_noalloc.restype = ip
    L.wrf_wsm6_noalloc.argtypes = [ctypes.POINTER(WrfGridC)] + [vp] * 11 + [ctypes.c_float] + [vp] * 7 + [vp]
    L.wrf_status_read.restype = ip
    L.wrf_status_read.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_int)]
    L.wrf_last_launch_count.restype = ip
    G = ctypes.POINTER(WrfGridC)
    ll, f32 = ctypes.c_longlong, ctypes.c_float
    L.wrf_mlp_init.restype = ip
    L.wrf_mlp_layout.restype = ip
    L.wrf_mlp_layout.argtypes = [G, ctypes.POINTER(ctypes.c_int)]
    L.wrf_rk3_step_mlp.restype = ip
    L.wrf_rk3_step_mlp.argtypes = [G, vp, ctypes.POINTER(WrfMlpNetC), ctypes.POINTER(WrfMlpWorkC), vp, PROBE_FN, vp]
    L.wrf_mlp_forward.restype = ip
    L.wrf_mlp_forward.argtypes = [ctypes.POINTER(WrfMlpNetC), vp, ip, vp, vp, vp, vp, vp]
    L.wrf_mlp_features.restype = ip
    L.wrf_mlp_features.argtypes = [G, vp, vp, vp, vp, vp]
    L.wrf_mlp_targets.restype = ip
    L.wrf_mlp_targets.argtypes = [G, vp, vp, vp, vp]
    L.wrf_mlp_normalize.restype = ip
    L.wrf_mlp_normalize.argtypes = [G, vp, vp, vp, ll, vp, vp, vp]
    L.wrf_gemm_bf16.restype = ip
    L.wrf_gemm_bf16.argtypes = [vp, vp, ip, ip, ip, ip, ip, vp, vp, vp, ip, ll, vp, vp, ip, vp, vp]
    L.wrf_gemm_splits.restype = ip
    L.wrf_gemm_splits.argtypes = [ip, ip]
    L.wrf_mse_grad.restype = ip
    L.wrf_mse_grad.argtypes = [vp, vp, ip, ip, ip, f32, vp, vp, vp, vp]
    L.wrf_rowsum_bf16.restype = ip
    L.wrf_rowsum_bf16.argtypes = [vp, ip, ip, vp, vp]
    L.wrf_adam.restype = ip
    L.wrf_adam.argtypes = [vp, vp, ip, ll, vp, vp, ip, ip, vp, vp, f32, f32, f32, f32, f32, ip, vp]
    L.wrf_transpose_bf16.restype = ip
    L.wrf_transpose_bf16.argtypes = [vp, ip, ip, vp, vp]
    _lib = L
    return L


def field_names() -> list[str]:
    global _names
    if _names is None:
        L = lib()
        _names = [L.wrf_field_name(i).decode() for i in range(L.wrf_field_count())]
    return _names


def field_kinds() -> list[int]:
    global _kinds
    if _kinds is None:
        L = lib()
        _kinds = [L.wrf_field_kind(i) for i in range(L.wrf_field_count())]
    return _kinds


def check(rc: int, what: str) -> None:
    if rc != WRF_OK:
        msg = lib().wrf_last_error().decode(errors="replace")
        if rc == WRF_EINVAL:
            raise ValueError(f"{what}: {msg}")
        raise RuntimeError(f"{what} failed ({rc}): {msg}")
