"""Whole steps with the tiled tensor-map kernels (WRF_FORM_FAST) against the
same steps with the one-thread-per-point and cp.async forms (WRF_FORM_POINT,
which also runs the boundary relaxation over every point instead of the
boundary band): every field of the state must agree to the bit, since both
forms perform the reference's operations in the same order.  Grids: 28x28x16 (partial tiles,
boundary blocks only), 108x108x41 (interior blocks on the branch-free
paths, several level chunks per kernel) and 28x28x61 (four level slots per
thread in the acoustic column kernels).  The fast form's acoustic column
kernel stages its operands by tensor-map copies; the point form's loads them
itself."""
from __future__ import annotations

import pytest
import torch

from pywrf_b200 import _native as N
from pywrf_b200 import synthetic
from pywrf_b200.solver import Integrator
from pywrf_b200.state import DeviceState

pytestmark = pytest.mark.gpu


def _run(spec, form, nsteps):
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    prev = N.lib().wrf_set_kernel_form(form)
    try:
        st = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
        it = Integrator(st)
        it.run(nsteps, graph=False)
        torch.cuda.synchronize()
        assert it.status()["wait_timeouts"] == 0
    finally:
        N.lib().wrf_set_kernel_form(prev)
    return st


@pytest.mark.parametrize("n,nz,nsteps", [(28, 16, 2), (108, 41, 1), (28, 61, 1)],
                         ids=["28x28x16x2", "108x108x41x1", "28x28x61x1"])
def test_tiled_kernels_equal_point_kernels_bitwise(n, nz, nsteps):
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    spec = synthetic.CaseSpec(n=n, nz=nz, nsteps=nsteps, bdy_tend_amp=1.0e-4, seed=23)
    fast = _run(spec, N.WRF_FORM_FAST, nsteps)
    point = _run(spec, N.WRF_FORM_POINT, nsteps)
    bad = [k for k in fast.names if not torch.equal(fast[k], point[k])]
    assert not bad, bad
