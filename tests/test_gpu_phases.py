"""The phase entry points (wrf_step_begin .. wrf_step_end), driven in the
order of the reference's RK3 loop, against the whole-step entry point: the
same kernels on the same state, so every field must agree bit for bit."""
from __future__ import annotations

import ctypes

import pytest
import torch

from helpers import SMALL
from pywrf_b200 import _native as N
from pywrf_b200 import synthetic
from pywrf_b200.solver import Integrator
from pywrf_b200.state import DeviceState

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    return g, inputs, bdy


def test_phases_equal_the_whole_step_bitwise(case):
    g, inputs, bdy = case
    a = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    b = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    ia, ib = Integrator(a), Integrator(b)
    for _ in range(2):
        ia.step()
        ib.step_phases()
    torch.cuda.synchronize()
    for name in N.field_names():
        assert torch.equal(a[name], b[name]), name
    assert ib.status()["step"] == 2


def test_phases_reject_a_stage_or_substep_out_of_range(case):
    g, inputs, bdy = case
    st = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    L = N.lib()
    cg, sp = ctypes.byref(st.cgrid), st.ptr
    h = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.wrf_tend_stage(cg, sp, 4, h) == N.WRF_EINVAL
    assert "rk_step" in L.wrf_last_error().decode()
    assert L.wrf_acoustic_substep(cg, sp, 1, 2, h) == N.WRF_EINVAL   # stage 1 has one substep
    assert L.wrf_acoustic_substep(cg, sp, 3, 0, h) == N.WRF_EINVAL
    assert "iteration" in L.wrf_last_error().decode()
