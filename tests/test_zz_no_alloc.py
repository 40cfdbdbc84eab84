"""wrf_wsm6_noalloc (WSM6 with its scratch in a fixed device array) against
wrf_wsm6 through the C ABI, on two calls in a row.  The file is collected last
and is independent of the other tests (it also runs alone)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from oracle import physics as OP
from oracle.model import OracleModel
from pywrf_b200 import _native as N
from pywrf_b200 import synthetic
from pywrf_b200.config import Grid
from pywrf_b200.state import make_cgrid

pytestmark = pytest.mark.gpu

NAMES = ("th_phy", "q1", "q2", "q3", "q4", "q5", "q6", "rho", "pi_phy", "p_phy", "dz8w")
FLAT = ("rainnc", "rainncv", "snownc", "snowncv", "graupelnc", "graupelncv", "sr")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture(scope="module")
def physics_inputs():
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    spec = synthetic.spec_for_config(0)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    m = OracleModel(g, inputs, bdy, np.float32)
    m.run(1)
    OP.moist_physics_prep_em(g, m.st)
    s = m.st
    arrays = {k: (s["moist"][int(k[1])] if k.startswith("q") else s[k]).copy() for k in NAMES}
    flat = {k: s[k].copy() for k in FLAT}
    return g, arrays, flat


def _call(fn, g, dev, flat, delt):
    cg = make_cgrid(g, {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0, "cfn1": 0.0})
    return fn(ctypes.byref(cg), *[_ptr(dev[k]) for k in NAMES], ctypes.c_float(delt), *[_ptr(flat[k]) for k in FLAT],
              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_noalloc_equals_wsm6_on_two_calls_in_a_row(physics_inputs):
    g, arrays, flat = physics_inputs
    L = N.lib()
    runs = {}
    for name, fn in (("wsm6", L.wrf_wsm6), ("noalloc", L.wrf_wsm6_noalloc)):
        dev = {k: torch.tensor(v, dtype=torch.float32, device="cuda") for k, v in arrays.items()}
        d2 = {k: torch.tensor(v, dtype=torch.float32, device="cuda") for k, v in flat.items()}
        snaps = []
        for _ in range(2):  # the second call continues from the first call's output
            rc = _call(fn, g, dev, d2, float(g.dt))
            N.check(rc, name)
            torch.cuda.synchronize()
            snaps.append({k: t.clone() for k, t in {**dev, **d2}.items()})
        runs[name] = snaps
    for call in range(2):
        for k in NAMES[:7] + FLAT:
            a, b = runs["wsm6"][call][k], runs["noalloc"][call][k]
            assert torch.equal(a, b), (call, k, float((a - b).abs().max()))
    # the scheme did something (rain or cloud changed between the calls)
    assert not torch.equal(runs["wsm6"][0]["q2"], runs["wsm6"][1]["q2"])


def test_noalloc_rejects_blocks_beyond_its_scratch_and_two_loops(physics_inputs):
    g, arrays, flat = physics_inputs
    L = N.lib()
    dev = {k: torch.zeros(4, dtype=torch.float32, device="cuda") for k in NAMES}
    d2 = {k: torch.zeros(4, dtype=torch.float32, device="cuda") for k in FLAT}
    big = Grid.make(512, 512, 41, 9000.0, 9000.0, 45.0)   # 40 x 499 x 499 block points
    rc = _call(L.wrf_wsm6_noalloc, big, dev, d2, 45.0)
    assert rc == N.WRF_EINVAL
    assert "exceeds the fixed scratch" in L.wrf_last_error().decode()
    rc = _call(L.wrf_wsm6_noalloc, g, dev, d2, 250.0)
    assert rc == N.WRF_EINVAL
    assert "two time-split loops" in L.wrf_last_error().decode()
