"""advect_u / advect_v / advect_w through wrf_advect_momentum: the tiled
tensor-map kernel (form 0) against the one-thread-per-point kernel (form 1)
on the state of a real step.  Both perform the reference's operations in the
reference's order (pywrf/wrf_dynamics.py:1112-1823), so they must agree to
the bit; the point kernel is the one the whole-step parity tests pinned
against the reference before the tiled kernel replaced it in the step.

Grids: n = 28, nz = 16 (one partial tile in x, every block a boundary
block) and n = 108, nz = 41 (interior blocks on the branch-free path, four
level chunks per component)."""
from __future__ import annotations

import pytest
import torch

from pywrf_b200 import synthetic
from pywrf_b200 import wrf_dynamics as WD
from pywrf_b200.solver import Integrator
from pywrf_b200.state import DeviceState

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(28, 16), (108, 41)], ids=["28x28x16", "108x108x41"])
def stepped(request):
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    n, nz = request.param
    spec = synthetic.CaseSpec(n=n, nz=nz, nsteps=1, bdy_tend_amp=1.0e-4, seed=17)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    st = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    Integrator(st).step()
    torch.cuda.synchronize()
    return g, st


@pytest.mark.parametrize("component", [0, 1, 2], ids=["u", "v", "w"])
def test_tiled_momentum_advection_equals_the_point_kernel_bitwise(stepped, component):
    g, st = stepped
    field = st[("u", "v", "w")[component]]
    msf, msf2 = {0: (st["msfux"], None), 1: (st["msfvy"], st["msfvx"]), 2: (st["msftx"], None)}[component]
    rdz = st["rdn"] if component == 2 else st["rdnw"]
    gen = torch.Generator(device="cuda").manual_seed(5 + component)
    tend0 = torch.randn(field.shape, generator=gen, device="cuda", dtype=torch.float32)
    out = []
    for form in (0, 1):
        t = tend0.clone()
        WD._advect_momentum(component, field, t, st["ru"], st["rv"], st["ww"], msf, msf2, st["fnm"], st["fnp"],
                            1.0 / g.dx, 1.0 / g.dy, rdz, form=form)
        out.append(t)
    torch.cuda.synchronize()
    assert not torch.equal(out[0], tend0), "the advection changed nothing"
    diff = (out[0] != out[1]).nonzero()
    assert diff.numel() == 0, f"{diff.shape[0]} points differ, first {diff[:5].tolist()}"


def test_reference_signature_drop_in_runs_the_same_kernel(stepped):
    g, st = stepped
    nz, ny, nx = st["u"].shape
    tend = torch.zeros_like(st["u"])
    args = dict(ru=st["ru"], rv=st["rv"], rom=st["ww"], c1=None, c2=None, mut=None, time_step=0,
                msfux=st["msfux"], msfuy=None, msfvx=st["msfvx"], msfvy=st["msfvy"], msftx=st["msftx"], msfty=None,
                fzm=st["fnm"], fzp=st["fnp"], rdx=1.0 / g.dx, rdy=1.0 / g.dy,
                ids=5, ide=nx - 5, jds=5, jde=ny - 5, kds=0, kde=nz, ims=0, ime=nx, jms=0, jme=ny, kms=0, kme=nz,
                its=5, ite=nx - 5, jts=5, jte=ny - 5, kts=0, kte=nz)
    got = WD.advect_u(st["u"], st["u"], tend, rdzw=st["rdnw"], **args)
    want = torch.zeros_like(st["u"])
    WD._advect_momentum(0, st["u"], want, st["ru"], st["rv"], st["ww"], st["msfux"], None, st["fnm"], st["fnp"],
                        1.0 / g.dx, 1.0 / g.dy, st["rdnw"], form=1)
    assert got is tend and torch.equal(got, want)
    wt = WD.advect_w(st["w"], st["w"], torch.zeros_like(st["w"]), rdzu=st["rdn"], **args)
    ww = torch.zeros_like(st["w"])
    WD._advect_momentum(2, st["w"], ww, st["ru"], st["rv"], st["ww"], st["msftx"], None, st["fnm"], st["fnp"],
                        1.0 / g.dx, 1.0 / g.dy, st["rdn"], form=1)
    assert torch.equal(wt, ww)
