"""The C ABI library without a GPU: it loads, exports every entry point that
include/pywrf_b200.h declares, agrees with the header's field table, and
rejects bad arguments before touching the device."""
from __future__ import annotations

import ctypes
import os
import re

import pytest

from pywrf_b200 import _native as N
from pywrf_b200.build import INCLUDE, LIB
from pywrf_b200.config import Grid
from pywrf_b200.state import make_cgrid

HEADER = os.path.join(INCLUDE, "pywrf_b200.h")


def _header_text():
    with open(HEADER) as f:
        return f.read()


def _declared_functions():
    txt = re.sub(r"/\*.*?\*/", "", _header_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(wrf_\w+)\s*\(", txt, flags=re.M)))


def _header_table():
    txt = _header_text()
    body = txt[txt.index("#define WRF_FIELD_TABLE(X)"):txt.index("#define WRF_ENUM_ENTRY")]
    return re.findall(r"X\((\w+),\s*(WRF_K\w+)\)", body)


def test_library_is_built():
    assert os.path.exists(LIB), "run python -m pywrf_b200.build"


def test_every_declared_entry_point_is_exported():
    L = N.lib()
    names = _declared_functions()
    assert {"wrf_rk3_step", "wrf_wsm6", "wrf_advect_scalar", "wrf_status_read"} <= set(names)
    for nm in names:
        assert hasattr(L, nm), nm


def test_field_table_matches_header():
    kinds = {"WRF_K3": 3, "WRF_K2": 2, "WRF_K1": 1, "WRF_K4": 4, "WRF_KBX": 10, "WRF_KBY": 11,
             "WRF_KBX2": 12, "WRF_KBY2": 13, "WRF_KSF": 20, "WRF_KSI": 21}
    table = _header_table()
    assert len(table) == N.lib().wrf_field_count()
    assert N.field_names() == [n.lower() for n, _ in table]
    assert N.field_kinds() == [kinds[k] for _, k in table]
    assert N.lib().wrf_field_name(len(table)) is None


def _cgrid(**kw):
    g = Grid.make(28, 28, 16, 9000.0, 9000.0, 45.0)
    c = make_cgrid(g, {"cf1": 1.0, "cf2": 0.0, "cf3": 0.0, "cfn": 1.0, "cfn1": 0.0})
    for k, v in kw.items():
        setattr(c, k, v)
    return c


@pytest.mark.parametrize("field,value,needle", [
    ("nz", 200, "nz"), ("ids", 4, "frame"), ("spec_zone", 2, "spec_zone"), ("soundsteps", 3, "soundsteps"),
    ("kvdif", 1.0, "kvdif"), ("dt", 0.0, "dt"),
])
def test_bad_grid_is_rejected_before_any_launch(field, value, needle):
    L = N.lib()
    state = (ctypes.c_void_p * L.wrf_field_count())()
    rc = L.wrf_rk3_step(ctypes.byref(_cgrid(**{field: value})), ctypes.cast(state, ctypes.c_void_p), None,
                        N.PROBE_FN(), None)
    assert rc == N.WRF_EINVAL
    assert needle in L.wrf_last_error().decode()


def test_null_state_pointer_is_rejected():
    L = N.lib()
    state = (ctypes.c_void_p * L.wrf_field_count())()
    rc = L.wrf_rk3_step(ctypes.byref(_cgrid()), ctypes.cast(state, ctypes.c_void_p), None, N.PROBE_FN(), None)
    assert rc == N.WRF_EINVAL
    assert "null field u" in L.wrf_last_error().decode()
    with pytest.raises(ValueError, match="null field"):
        N.check(rc, "wrf_rk3_step")


def test_null_arguments_of_function_entry_points_are_rejected():
    L = N.lib()
    nulls = [None] * 11
    rc = L.wrf_wsm6(ctypes.byref(_cgrid()), *nulls, ctypes.c_float(45.0), *([None] * 7), None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_advect_scalar(ctypes.byref(_cgrid()), *([None] * 9), None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_advect_momentum(ctypes.byref(_cgrid()), 0, *([None] * 10), 0, None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_advect_momentum_adj(ctypes.byref(_cgrid()), 1, *([None] * 15), 0, None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_advect_momentum_adj(ctypes.byref(_cgrid()), 3, *([None] * 15), 0, None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_advance_uv(ctypes.byref(_cgrid()), None, ctypes.c_float(1.0), None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_calc_p_rho(ctypes.byref(_cgrid()), None, 1, None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_advance_mu_t(ctypes.byref(_cgrid()), None, ctypes.c_float(1.0), None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_advance_w(ctypes.byref(_cgrid()), None, ctypes.c_float(1.0), None)
    assert rc == N.WRF_EINVAL
    tab = (ctypes.c_void_p * L.wrf_field_count())()
    rc = L.wrf_advance_mu_t_adj(ctypes.byref(_cgrid()), tab, tab, ctypes.c_float(1.0), 0, None, None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_advance_w_adj(ctypes.byref(_cgrid()), tab, tab, ctypes.c_float(1.0), None, None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_calc_p_rho_adj(ctypes.byref(_cgrid()), (ctypes.c_void_p * L.wrf_field_count())(), None, 1, None)
    assert rc == N.WRF_EINVAL
    empty = (ctypes.c_void_p * L.wrf_field_count())()
    rc = L.wrf_advance_uv_adj(ctypes.byref(_cgrid()), empty, empty, ctypes.c_float(1.0), None)
    assert rc == N.WRF_EINVAL
    rc = L.wrf_status_read(None, None, None)
    assert rc == N.WRF_EINVAL


def test_kernel_form_switch():
    L = N.lib()
    assert L.wrf_set_kernel_form(7) == N.WRF_EINVAL
    assert L.wrf_set_kernel_form(N.WRF_FORM_POINT) == N.WRF_FORM_FAST
    assert L.wrf_set_kernel_form(N.WRF_FORM_FAST) == N.WRF_FORM_POINT


def test_header_is_plain_c():
    """include/pywrf_b200.h compiles as C99 and as C++ (plain C types only)."""
    import os
    import shutil
    import subprocess

    import pytest

    hdr = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pywrf_b200.h")
    for cc, lang, std in (("gcc", "c", "-std=c99"), ("g++", "c++", "-std=c++17")):
        if shutil.which(cc) is None:
            pytest.skip(f"{cc} not found")
        r = subprocess.run([cc, "-fsyntax-only", "-Wall", "-Werror", "-x", lang, std, hdr], capture_output=True,
                           text=True)
        assert r.returncode == 0, r.stderr
