"""The hand-written adjoints (pywrf_b200.adjoint over the library's
``wrf_*_adj`` entries): each operator against the reference's autograd
gradients or float64 central differences of the reference's forward
(tests/golden/*_adj_ref64.npz) or of the oracle; the composed acoustic
substep, acoustic stage, dynamics and RK stages, the microphysics and whole
steps against float64 central differences of the oracle; and the adjoint
configuration's theta-bias gradient against the reference's
(tests/golden/thbias_ref64.npz)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from helpers import load_npz, rel_l2
from pywrf_b200 import adjoint

pytestmark = pytest.mark.gpu


def _cuda(a):
    return torch.tensor(np.asarray(a), dtype=torch.float32, device="cuda").contiguous()


def test_advect_scalar_adjoint_matches_reference_autograd():
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    Z = load_npz("adv_scalar_adj_ref64.npz")
    t = {k: _cuda(Z[k]) for k in ("field", "ru", "rv", "rom", "msftx", "fnm", "fnp", "rdnw", "cot")}
    for k in ("field", "ru", "rv", "rom"):
        t[k].requires_grad_(True)
    tend0 = torch.zeros_like(t["field"], requires_grad=True)
    out = adjoint.advect_scalar(t["field"], tend0, t["ru"], t["rv"], t["rom"], t["msftx"], t["fnm"], t["fnp"],
                                t["rdnw"], 1.0 / float(Z["dx"]), 1.0 / float(Z["dy"]))
    assert rel_l2(out.detach().cpu().numpy(), Z["tend"]) < 1e-6
    (out * t["cot"]).sum().backward()
    # fp32 kernels against the float64 reference: the gradients are sums of
    # a few dozen fp32 products each
    for k in ("field", "ru", "rv", "rom"):
        err = rel_l2(t[k].grad.cpu().numpy(), Z["grad_" + k])
        assert err < 1e-5, (k, err)
    assert torch.equal(tend0.grad, t["cot"])


def test_advect_scalar_adjoint_identity_at_64x64x41():
    g = torch.Generator().manual_seed(21)
    nz, n = 41, 64
    shp = (nz, n, n)

    def rnd(*s, scale=1.0, shift=0.0):
        return (torch.randn(*s, generator=g, dtype=torch.float64) * scale + shift)

    q = rnd(*shp, scale=2.0, shift=300.0)
    ru, rv, rom = rnd(*shp, scale=15.0, shift=3.0), rnd(*shp, scale=15.0), rnd(*shp, scale=1.0)
    msftx = 1.0 + 0.02 * torch.rand(n, n, generator=g, dtype=torch.float64)
    fnm = 0.5 + 0.05 * torch.rand(nz, generator=g, dtype=torch.float64)
    fnp = 1.0 - fnm
    rdnw = -(10.0 + torch.rand(nz, generator=g, dtype=torch.float64))
    c = rnd(*shp)
    dq = rnd(*shp)
    C = {k: v.float().cuda().contiguous() for k, v in dict(q=q, ru=ru, rv=rv, rom=rom, msftx=msftx, fnm=fnm,
                                                             fnp=fnp, rdnw=rdnw, c=c, dq=dq).items()}
    zero = torch.zeros_like(C["q"])

    def fwd(field):
        return adjoint.advect_scalar(field, zero, C["ru"], C["rv"], C["rom"], C["msftx"], C["fnm"], C["fnp"],
                                     C["rdnw"], 1.0 / 9000.0, 1.0 / 9000.0)

    # the operator is linear in the field: A dq = fwd(dq)
    a_dq = fwd(C["dq"]).double()
    qv = C["q"].clone().requires_grad_(True)
    (fwd(qv) * C["c"]).sum().backward()
    lhs = float((a_dq * C["c"].double()).sum())
    rhs = float((C["dq"].double() * qv.grad.double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * (abs(lhs) + abs(rhs)), (lhs, rhs)


@pytest.mark.parametrize("var", ["t", "u", "v", "h"])
def test_relax_bdytend_and_adjoint_match_reference_autograd(var):
    Z = load_npz("relax_adj_ref64.npz")
    field = _cuda(Z[f"{var}_field"]).requires_grad_(True)
    tend0 = _cuda(Z[f"{var}_tend0"]).requires_grad_(True)
    bdy = {k: _cuda(Z[f"{var}_{k}"]) for k in adjoint.BDY_NAMES}
    out = adjoint.relax_bdytend(field, tend0, var, float(Z["dtbc"]), bdy)
    assert rel_l2(out.detach().cpu().numpy(), Z[f"{var}_tend"]) < 1e-6
    (out * _cuda(Z[f"{var}_cot"])).sum().backward()
    err = rel_l2(field.grad.cpu().numpy(), Z[f"{var}_grad_field"])
    assert err < 1e-6, err


def _vsolve_torch(x, a, alpha, gamma):
    """The reference's two loops (wrf_dynamics.py:3761-3767) in torch."""
    w = [x[0]]
    for k in range(1, x.shape[0]):
        w.append((x[k] - a[k] * w[k - 1]) * alpha[k])
    out = list(w)
    for k in range(x.shape[0] - 2, 0, -1):
        out[k] = w[k] - gamma[k] * out[k + 1]
    return torch.stack(out)


def test_vsolve_w_and_its_transposed_solve_match_autograd():
    g = torch.Generator().manual_seed(31)
    nz, ny, nx = 41, 20, 24
    x = torch.randn(nz, ny, nx, generator=g, dtype=torch.float64)
    a = 0.3 * torch.rand(nz, ny, nx, generator=g, dtype=torch.float64)
    alpha = 0.5 + 0.5 * torch.rand(nz, ny, nx, generator=g, dtype=torch.float64)
    gamma = 0.3 * torch.rand(nz, ny, nx, generator=g, dtype=torch.float64)
    cot = torch.randn(nz, ny, nx, generator=g, dtype=torch.float64)
    ref_in = [t.clone().requires_grad_(True) for t in (x, a, alpha, gamma)]
    ref = _vsolve_torch(*ref_in)
    (ref * cot).sum().backward()
    gpu_in = [t.float().cuda().requires_grad_(True) for t in (x, a, alpha, gamma)]
    w = adjoint.vsolve_w(*gpu_in)
    assert rel_l2(w.detach().cpu().numpy(), ref.detach().numpy()) < 1e-6
    (w * cot.float().cuda()).sum().backward()
    for name, r, t in zip(("x", "a", "alpha", "gamma"), ref_in, gpu_in):
        err = rel_l2(t.grad.cpu().numpy(), r.grad.numpy())
        assert err < 1e-5, (name, err)


def test_coef_w_and_its_adjoint_against_the_reference():
    """calc_coef_w's coefficients against the reference's, and the adjoint's
    directional derivatives against central finite differences of the
    reference's float64 forward (tests/golden/coefw_adj_ref64.npz)."""
    W = load_npz("coefw_adj_ref64.npz")
    mut = _cuda(W["mut"]).requires_grad_(True)
    cqw = _cuda(W["cqw"]).requires_grad_(True)
    c2a = _cuda(W["c2a"]).requires_grad_(True)
    a, al, ga = adjoint.coef_w(mut, cqw, c2a, _cuda(W["rdn"]), _cuda(W["rdnw"]), float(W["dts"]),
                               epssm=float(W["epssm"]))
    for mine, ref in ((a, W["a"]), (al, W["alpha"]), (ga, W["gamma"])):
        assert rel_l2(mine.detach().cpu().numpy(), ref) < 1e-5
    L = (a * _cuda(W["cot_a"])).sum() + (al * _cuda(W["cot_alpha"])).sum() + (ga * _cuda(W["cot_gamma"])).sum()
    L.backward()
    for name, t in (("mut", mut), ("cqw", cqw), ("c2a", c2a)):
        gr = t.grad.double().cpu().numpy()
        for r in range(3):
            an = float((gr * W[f"dir_{name}_{r}"]).sum())
            fd = float(W[f"fd_{name}_{r}"])
            assert abs(an - fd) <= 2e-4 * abs(fd), (name, r, an, fd)


def _mom_dir(n, r, shape):
    # the directions of make_golden_adjoint.mom_direction
    return np.random.default_rng(7000 + 10 * n + r).standard_normal(shape)


@pytest.mark.parametrize("comp", ["u", "v", "w"])
def test_advect_momentum_adjoint_matches_the_reference(comp):
    """advect_u / advect_v: the hand-written adjoint against the reference's
    autograd gradients; advect_w (whose reference backward raises): its
    directional derivatives against central differences of the reference's
    float64 forward (tests/golden/adv_mom_adj_ref64.npz)."""
    M = load_npz("adv_mom_adj_ref64.npz")
    c = {"u": 0, "v": 1, "w": 2}[comp]
    t = {k: _cuda(M[f"{comp}_{k}"]) for k in ("field", "ru", "rv", "rom", "msf", "msf2", "cot")}
    for k in ("field", "ru", "rv", "rom"):
        t[k].requires_grad_(True)
    prof = {k: _cuda(M[k]) for k in ("fnm", "fnp", "rdnw", "rdn")}
    tend0 = torch.zeros_like(t["field"], requires_grad=True)
    out = adjoint.advect_momentum(c, t["field"], tend0, t["ru"], t["rv"], t["rom"], t["msf"],
                                  t["msf2"] if comp == "v" else None, prof["fnm"], prof["fnp"],
                                  prof["rdn" if comp == "w" else "rdnw"], 1.0 / float(M["dx"]), 1.0 / float(M["dy"]))
    assert rel_l2(out.detach().cpu().numpy(), M[f"{comp}_tend"]) < 1e-6
    (out * t["cot"]).sum().backward()
    assert torch.equal(tend0.grad, t["cot"])
    for n, k in enumerate(("field", "ru", "rv", "rom")):
        gr = t[k].grad.double().cpu().numpy()
        if comp != "w":
            err = rel_l2(gr, M[f"{comp}_grad_{k}"])
            assert err < 1e-5, (comp, k, err)
        else:
            for r in range(3):
                an = float((gr * _mom_dir(n, r, gr.shape)).sum())
                fd = float(M[f"w_fd_{k}_{r}"])
                assert abs(an - fd) <= 1e-4 * abs(fd), (k, r, an, fd)


@pytest.mark.parametrize("comp", ["u", "v", "w"])
def test_advect_momentum_adjoint_at_64x64x41(comp):
    """At 64x64x41: (1) the identity <A dq, c> = <dq, A^T c> for the field
    (positive fields keep advect_u's / advect_v's sign-selected boundary
    values on one branch, so the operator is linear in the field there);
    (2) the velocity cotangents' directional derivatives against central
    differences of the oracle's float64 forward."""
    from oracle import dynamics as OD
    from pywrf_b200 import synthetic

    c = {"u": 0, "v": 1, "w": 2}[comp]
    nz, n = 41, 64
    shp = (nz, n, n)
    rng = np.random.default_rng(41 + c)
    q = 10.0 + 2.0 * np.abs(rng.standard_normal(shp))
    vel = {"ru": 15.0 * rng.standard_normal(shp) + 3.0, "rv": 15.0 * rng.standard_normal(shp),
           "rom": rng.standard_normal(shp)}
    msf = 1.0 + 0.02 * rng.random((n, n))
    msf2 = 1.0 + 0.02 * rng.random((n, n))
    fnm = 0.5 + 0.05 * rng.random(nz)
    fnp = 1.0 - fnm
    rdz = -(10.0 + rng.random(nz))
    cot = rng.standard_normal(shp)
    dq = np.abs(rng.standard_normal(shp))
    f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    q, msf, msf2, fnm, fnp, rdz, cot, dq = map(f32, (q, msf, msf2, fnm, fnp, rdz, cot, dq))
    vel = {k: f32(v) for k, v in vel.items()}
    C = {k: _cuda(v) for k, v in dict(q=q, msf=msf, msf2=msf2, fnm=fnm, fnp=fnp, rdz=rdz, cot=cot, dq=dq,
                                      **vel).items()}
    zero = torch.zeros_like(C["q"])

    def fwd(field, ru, rv, rom):
        return adjoint.advect_momentum(c, field, zero, ru, rv, rom, C["msf"], C["msf2"] if c == 1 else None,
                                       C["fnm"], C["fnp"], C["rdz"], 1.0 / 9000.0, 1.0 / 9000.0)

    leaves = {k: C[k].clone().requires_grad_(True) for k in ("q", "ru", "rv", "rom")}
    (fwd(leaves["q"], leaves["ru"], leaves["rv"], leaves["rom"]) * C["cot"]).sum().backward()
    a_dq = fwd(C["dq"], C["ru"], C["rv"], C["rom"]).double()
    lhs = float((a_dq * C["cot"].double()).sum())
    rhs = float((C["dq"].double() * leaves["q"].grad.double()).sum())
    assert abs(lhs - rhs) <= 1e-5 * (abs(lhs) + abs(rhs)), (lhs, rhs)

    g = synthetic.grid_for(synthetic.CaseSpec(n=n, nz=nz))

    def oracle(x):
        t = np.zeros(shp)
        if c == 0:
            OD.advect_u(g, q, t, x["ru"], x["rv"], x["rom"], msf, fnm, fnp, rdz)
        elif c == 1:
            OD.advect_v(g, q, t, x["ru"], x["rv"], x["rom"], msf2, msf, fnm, fnp, rdz)
        else:
            OD.advect_w(g, q, t, x["ru"], x["rv"], x["rom"], msf, fnm, fnp, rdz)
        return t

    for k in ("ru", "rv", "rom"):
        d = rng.standard_normal(shp)
        eps = 1e-6 * float(np.abs(vel[k]).max())
        xp, xm = dict(vel), dict(vel)
        xp[k] = vel[k] + eps * d
        xm[k] = vel[k] - eps * d
        fd = float(((oracle(xp) - oracle(xm)) * cot).sum()) / (2 * eps)
        an = float((leaves[k].grad.double().cpu().numpy() * d).sum())
        assert abs(an - fd) <= 1e-4 * abs(fd), (comp, k, an, fd)


def _uv_dir(n, r, shape):
    # the directions of make_golden_adjoint.uv_direction
    return np.random.default_rng(8000 + 100 * n + r).standard_normal(shape)


@pytest.mark.parametrize("form", ["fast", "point"])
def test_advance_uv_and_its_adjoint_against_the_reference(form):
    """advance_uv + spec_bdyupdate(u), (v): u', v' against the reference's
    on the fixture (both kernel forms), and the adjoint's directional
    derivatives against central differences of the reference's float64
    forward (tests/golden/advuv_adj_ref64.npz; its autograd cannot
    differentiate advance_uv)."""
    from pywrf_b200 import _native as N

    V = load_npz("advuv_adj_ref64.npz")
    inputs = {k: _cuda(V[k]).requires_grad_(True) for k in adjoint.UV_INPUTS}
    data = {k: _cuda(V[k]) for k in adjoint.UV_DATA}
    prev = N.lib().wrf_set_kernel_form(N.WRF_FORM_FAST if form == "fast" else N.WRF_FORM_POINT)
    try:
        u, v = adjoint.advance_uv(inputs, data, float(V["dts"]), float(V["emdiv"]), float(V["cf1"]),
                                  float(V["cf2"]), float(V["cf3"]), 1.0 / float(V["dx"]), 1.0 / float(V["dy"]))
    finally:
        N.lib().wrf_set_kernel_form(prev)
    assert rel_l2(u.detach().cpu().numpy(), V["u_new"]) < 1e-6
    assert rel_l2(v.detach().cpu().numpy(), V["v_new"]) < 1e-6
    ((u * _cuda(V["cot_u"])).sum() + (v * _cuda(V["cot_v"])).sum()).backward()
    names = ("u", "ru_tend", "v", "rv_tend", "p", "pb", "ph", "php", "alt", "al", "cqu", "cqv",
             "mu", "muu", "muv", "mudf")
    for n, name in enumerate(names):
        gr = inputs[name].grad.double().cpu().numpy()
        for r in range(3):
            an = float((gr * _uv_dir(n, r, gr.shape)).sum())
            fd = float(V[f"fd_{name}_{r}"])
            assert abs(an - fd) <= 1e-4 * abs(fd), (name, r, an, fd)


@pytest.mark.parametrize("step", [0, 1])
def test_calc_p_rho_and_its_adjoint_match_reference_autograd(step):
    """calc_p_rho at acoustic step 0 (pm1 = p) and 1 (divergence damping):
    al, p, pm1 against the reference's, and the hand-written adjoint against
    its autograd gradients (tests/golden/prho_adj_ref64.npz)."""
    P = load_npz("prho_adj_ref64.npz")
    inputs = {k: _cuda(P[k]).requires_grad_(True) for k in adjoint.PRHO_INPUTS}
    al, p, pm1 = adjoint.calc_p_rho(inputs, _cuda(P["rdnw"]), float(P["smdiv"]), step,
                                    1.0 / float(P["dx"]), 1.0 / float(P["dy"]))
    for nm, mine in (("al", al), ("p", p), ("pm1", pm1)):
        assert rel_l2(mine.detach().cpu().numpy(), P[f"s{step}_{nm}_new"]) < 1e-6, nm
    L = (al * _cuda(P["cot_al"])).sum() + (p * _cuda(P["cot_p"])).sum() + (pm1 * _cuda(P["cot_pm1"])).sum()
    L.backward()
    for k in adjoint.PRHO_INPUTS:
        ref = P[f"s{step}_grad_{k}"]
        mine = inputs[k].grad.cpu().numpy()
        if not np.any(ref):
            assert not np.any(mine), k
            continue
        err = rel_l2(mine, ref)
        assert err < 1e-5, (step, k, err)


def _mut_dir(n, r, shape):
    # the directions of make_golden_adjoint.mut_direction
    return np.random.default_rng(9000 + 100 * n + r).standard_normal(shape)


@pytest.mark.parametrize("ref_no_grad", [True, False], ids=["reference_autograd", "operator"])
def test_advance_mu_t_and_its_adjoint(ref_no_grad):
    """advance_mu_t: the seven outputs against the reference's; with
    ref_no_grad the adjoint against the reference's autograd gradients (its
    mu update runs under torch.no_grad()), without it the adjoint's
    directional derivatives against central differences of the reference's
    float64 forward (tests/golden/mut_adj_ref64.npz)."""
    T = load_npz("mut_adj_ref64.npz")
    inputs = {k: _cuda(T[k]).requires_grad_(True) for k in adjoint.MUT_INPUTS}
    data = {k: _cuda(T[k]) for k in adjoint.MUT_DATA}
    outs = adjoint.advance_mu_t(inputs, data, float(T["dts"]), float(T["epssm"]), 1.0 / float(T["dx"]),
                                1.0 / float(T["dy"]), ref_no_grad=ref_no_grad)
    for k in adjoint.MUT_OUTPUTS:
        assert rel_l2(outs[k].detach().cpu().numpy(), T[f"{k}_new"]) < 1e-6, k
    sum((outs[k] * _cuda(T[f"cot_{k}"])).sum() for k in adjoint.MUT_OUTPUTS).backward()
    names = ("ww", "ww_1", "u", "u_1", "v", "v_1", "t", "t_1", "t_ave", "ft",
             "mu", "mut", "muave", "muts", "muu", "muv", "mudf", "mu_tend")
    for n, k in enumerate(names):
        gr = inputs[k].grad.double().cpu().numpy()
        if ref_no_grad:
            ref = T[f"grad_{k}"]
            if not np.any(ref):
                assert not np.any(gr), k
                continue
            err = rel_l2(gr, ref)
            assert err < 1e-5, (k, err)
        else:
            for r in range(3):
                an = float((gr * _mut_dir(n, r, gr.shape)).sum())
                fd = float(T[f"fd_{k}_{r}"])
                assert abs(an - fd) <= 1e-4 * abs(fd), (k, r, an, fd)


def _aw_dir(n, r, shape):
    # the directions of make_golden_adjoint.aw_direction
    return np.random.default_rng(10000 + 100 * n + r).standard_normal(shape)


def test_advance_w_and_its_adjoint_against_the_reference():
    """advance_w: t_2ave, w, ph against the reference's, and the adjoint's
    directional derivatives against central differences of the reference's
    float64 forward (tests/golden/advw_adj_ref64.npz; the upper levels lie in
    the Rayleigh damping layer)."""
    A = load_npz("advw_adj_ref64.npz")
    inputs = {k: _cuda(A[k]).requires_grad_(True) for k in adjoint.AW_INPUTS}
    data = {k: _cuda(A[k]) for k in adjoint.AW_DATA}
    outs = adjoint.advance_w(inputs, data, float(A["dts"]), float(A["epssm"]), float(A["cf1"]), float(A["cf2"]),
                             float(A["cf3"]), 1.0 / float(A["dx"]), 1.0 / float(A["dy"]))
    for k in adjoint.AW_OUTPUTS:
        assert rel_l2(outs[k].detach().cpu().numpy(), A[f"{k}_new"]) < 1e-6, k
    cot = {"w": "cot_w", "ph": "cot_ph", "t_2ave": "cot_t2a"}
    sum((outs[k] * _cuda(A[cot[k]])).sum() for k in adjoint.AW_OUTPUTS).backward()
    names = ("w", "rw_tend", "ww", "w_save", "u", "v", "t_2ave", "t_2", "t_1", "ph", "ph_1", "phb", "ph_tend",
             "c2a", "cqw", "alt", "a", "alpha", "gamma", "muave", "muts", "mut", "ht")
    for n, k in enumerate(names):
        gr = inputs[k].grad.double().cpu().numpy()
        for r in range(3):
            an = float((gr * _aw_dir(n, r, gr.shape)).sum())
            fd = float(A[f"fd_{k}_{r}"])
            assert abs(an - fd) <= 1e-4 * abs(fd), (k, r, an, fd)


FORCES_FIX = {  # function: (differentiable inputs, outputs), as in tests/golden/make_golden_adjoint.py
    "rhs_ph": (("u", "v", "ww", "ph", "phb", "w", "mut", "muu", "muv"), ("ph_tend",)),
    "hpg": (("ph", "alt", "p", "pb", "al", "php", "cqu", "cqv", "muu", "muv", "mu"), ("ru_tend", "rv_tend")),
    "pg_buoy_w": (("p", "cqw", "mu", "mub"), ("rw_tend", "cqw")),
    "coriolis": (("ru", "rv", "rw"), ("ru_tend", "rv_tend", "rw_tend")),
    "curvature": (("ru", "rv", "rw", "u", "v"), ("ru_tend", "rv_tend", "rw_tend")),
}


@pytest.mark.parametrize("name", list(FORCES_FIX))
def test_tendency_terms_and_their_adjoint_against_the_reference(name):
    """rhs_ph, horizontal_pressure_gradient, pg_buoy_w (with its in-place
    cqw), coriolis and curvature one at a time through
    pywrf_b200.adjoint.forces: the outputs' norms and sums against the
    reference's on the fixture's inputs, and the adjoint's directional
    derivatives in every differentiable input against the reference's
    float64 central differences along three seeded directions
    (tests/golden/forces_adj_ref64.npz)."""
    F = load_npz("forces_adj_ref64.npz")
    fi = list(FORCES_FIX).index(name)
    ins, outs = FORCES_FIX[name]
    z = np.zeros_like(F["u"])
    inputs = {k: _cuda(z if k.endswith("_tend") else F[k]).requires_grad_(True) for k in adjoint.FORCES_INPUTS}
    data = {k: _cuda(F[k]) for k in adjoint.FORCES_DATA}
    sc = {k: float(F[k]) for k in ("cf1", "cf2", "cf3", "cfn", "cfn1")}
    res = dict(zip(adjoint.FORCES_OUTPUTS, adjoint.forces(inputs, data, [name], 1.0 / float(F["dx"]),
                                                          1.0 / float(F["dy"]), sc["cf1"], sc["cf2"], sc["cf3"],
                                                          sc["cfn"], sc["cfn1"])))
    for o in outs:
        a = res[o].detach().double().cpu().numpy()
        l2 = float(np.sqrt((a * a).sum()))
        ref_l2 = float(F[f"{name}_{o}_l2"])
        assert abs(l2 - ref_l2) <= 1e-5 * ref_l2, (o, l2, ref_l2)
        assert abs(float(a.sum()) - float(F[f"{name}_{o}_sum"])) <= 1e-5 * ref_l2 * a.size ** 0.5, o
    loss = sum((res[o] * _cuda(F[f"cot_{o}"])).sum() for o in outs)
    loss.backward()
    for n, inp in enumerate(ins):
        gr = inputs[inp].grad.double().cpu().numpy()
        for r in range(3):
            d = np.random.default_rng(20000 + 1000 * fi + 10 * n + r).standard_normal(gr.shape)
            an = float((gr * d).sum())
            scale = float(np.abs(gr * d).sum())
            fd = float(F[f"{name}_fd_{inp}_{r}"])
            # fp32 partial products against the reference's float64 differences
            assert abs(an - fd) <= 1e-4 * abs(fd) + 1e-6 * scale, (inp, r, an, fd, scale)


SUBBDY_FIX = {  # case: (differentiable inputs, outputs), as in tests/golden/make_golden_adjoint.py
    "sumflux1": (("u", "v", "ww", "u_save", "v_save", "ww1", "muu", "muv"), ("ru_m", "rv_m", "ww_m")),
    "sumflux2": (("u", "v", "ww", "u_save", "v_save", "ww1", "muu", "muv", "ru_m", "rv_m", "ww_m"),
                 ("ru_m", "rv_m", "ww_m")),
    "spec_t": (("t", "t_tend"), ("t",)),
    "spec_m": (("mu", "mu_tend"), ("mu",)),
    "spec_ph": (("ph_save", "ph", "ph_tend", "mu_tend", "muts"), ("ph",)),
}


@pytest.mark.parametrize("name", list(SUBBDY_FIX))
def test_substep_flux_sums_and_specified_rows_against_the_reference(name):
    """sumflux at the first and the last of two iterations, spec_bdyupdate of
    't' and 'm' and spec_bdyupdate_ph: the outputs' norms and sums against the
    reference's, and the adjoints' directional derivatives in every
    differentiable input against the reference's float64 central differences
    (tests/golden/subbdy_adj_ref64.npz)."""
    Z = load_npz("subbdy_adj_ref64.npz")
    fi = list(SUBBDY_FIX).index(name)
    ins, outs = SUBBDY_FIX[name]
    x = {k: _cuda(Z[k]).requires_grad_(True) for k in ("u", "v", "ww", "u_save", "v_save", "ww1", "muu", "muv", "ru_m",
                                                       "rv_m", "ww_m", "t", "t_tend", "mu", "mu_tend", "ph", "ph_save",
                                                       "ph_tend", "muts")}
    dts, rdx = float(Z["dts"]), 1.0 / 9000.0
    if name.startswith("sumflux"):
        res = dict(zip(("ru_m", "rv_m", "ww_m"),
                       adjoint.sumflux(x, {k: _cuda(Z[k]) for k in adjoint.SF_DATA}, 1 if name == "sumflux1" else 2,
                                       2, rdx, rdx)))
    elif name == "spec_t":
        res = {"t": adjoint.spec_bdyupdate(x["t"], x["t_tend"], dts, "t", rdx, rdx)}
    elif name == "spec_m":
        res = {"mu": adjoint.spec_bdyupdate(x["mu"], x["mu_tend"], dts, "m", rdx, rdx)}
    else:
        res = {"ph": adjoint.spec_bdyupdate_ph(x, dts, rdx, rdx)}
    for o in outs:
        a = res[o].detach().double().cpu().numpy()
        l2 = float(np.sqrt((a * a).sum()))
        ref_l2 = float(Z[f"{name}_{o}_l2"])
        assert abs(l2 - ref_l2) <= 1e-6 * ref_l2, (o, l2, ref_l2)
        assert abs(float(a.sum()) - float(Z[f"{name}_{o}_sum"])) <= 1e-6 * ref_l2 * a.size ** 0.5, o
    sum((res[o] * _cuda(Z[f"cot_{o}"])).sum() for o in outs).backward()
    for n, inp in enumerate(ins):
        gr = x[inp].grad.double().cpu().numpy()
        for r in range(3):
            d = np.random.default_rng(30000 + 1000 * fi + 10 * n + r).standard_normal(gr.shape)
            an, scale = float((gr * d).sum()), float(np.abs(gr * d).sum())
            fd = float(Z[f"{name}_fd_{inp}_{r}"])
            assert abs(an - fd) <= 1e-4 * abs(fd) + 1e-6 * scale, (inp, r, an, fd, scale)


PREP_FIX = {  # function: (differentiable inputs, outputs), as in tests/golden/make_golden_adjoint.py
    "calculate_full": (("mub", "mu"), ("mut",)),
    "calc_mu_uv": (("mu", "mub"), ("muu", "muv")),
    "couple_momentum": (("muu", "u", "muv", "v", "mut", "w"), ("ru", "rv", "rw")),
    "calc_ww_cp": (("u", "v", "muu", "muv", "ww"), ("ww",)),
    "calc_cq": (("moist",), ("cqu", "cqv", "cqw")),
    "calc_alt": (("al", "alb"), ("alt",)),
    "calc_php": (("ph", "phb"), ("php",)),
}


@pytest.mark.parametrize("name", list(PREP_FIX))
def test_rk_step_prep_functions_and_their_adjoint_against_the_reference(name):
    """rk_step_prep's functions one at a time through pywrf_b200.adjoint.prep:
    the outputs' norms and sums against the reference's on the fixture's
    inputs (outputs start from zero, as the fixture's calls pass), and the
    adjoints' directional derivatives in every differentiable input against
    the reference's float64 central differences
    (tests/golden/prep_adj_ref64.npz)."""
    Z = load_npz("prep_adj_ref64.npz")
    fi = list(PREP_FIX).index(name)
    ins, outs = PREP_FIX[name]
    fields = {}
    for k in adjoint.PREP_FIELDS:
        src = Z[k] if (k in Z and k not in outs) or k == "ww" else np.zeros_like(Z["ww"] if k not in ("mut", "muu", "muv") else Z["mu"])
        fields[k] = _cuda(src).requires_grad_(True)
    data = {k: _cuda(Z[k]) for k in adjoint.PREP_DATA if k != "c1h"}
    data["c1h"] = _cuda(np.ones(Z["ww"].shape[0], np.float32))
    res = adjoint.prep(fields, data, [name], 1.0 / 9000.0, 1.0 / 9000.0)
    for o in outs:
        a = res[o].detach().double().cpu().numpy()
        l2 = float(np.sqrt((a * a).sum()))
        ref_l2 = float(Z[f"{name}_{o}_l2"])
        assert abs(l2 - ref_l2) <= 2e-6 * ref_l2, (o, l2, ref_l2)
        assert abs(float(a.sum()) - float(Z[f"{name}_{o}_sum"])) <= 2e-6 * ref_l2 * a.size ** 0.5, o
    sum((res[o] * _cuda(Z[f"cot_{o}"])).sum() for o in outs).backward()
    for n, inp in enumerate(ins):
        gr = fields[inp].grad.double().cpu().numpy()
        for r in range(3):
            d = np.random.default_rng(40000 + 1000 * fi + 10 * n + r).standard_normal(gr.shape)
            an, scale = float((gr * d).sum()), float(np.abs(gr * d).sum())
            fd = float(Z[f"{name}_fd_{inp}_{r}"])
            assert abs(an - fd) <= 1e-4 * abs(fd) + 1e-6 * scale, (inp, r, an, fd, scale)


def _oracle_substep(g, s, iteration, nsub, dts):
    """One acoustic substep of the oracle (its model loop, solver.py:1394-1445)
    on the state dict ``s``, in place."""
    from oracle import boundary as OB
    from oracle import dynamics as OD

    OD.advance_uv(g, s["u"], s["ru_tend"], s["v"], s["rv_tend"], s["p"], s["pb"], s["ph"], s["php"], s["alt"],
                  s["al"], s["mu"], s["muu"], s["cqu"], s["muv"], s["cqv"], s["mudf"], s["msfux"], s["msfuy"],
                  s["msfvx"], s["msfvx_inv"], s["msfvy"], dts, s["cf1"], s["cf2"], s["cf3"], s["fnm"], s["fnp"],
                  g.emdiv, s["rdnw"])
    OB.spec_bdyupdate(g, s["u"], s["ru_tend"], dts, "u")
    OB.spec_bdyupdate(g, s["v"], s["rv_tend"], dts, "v")
    OD.advance_mu_t(g, s, dts, g.epssm, iteration)
    OB.spec_bdyupdate(g, s["t"], s["t_tend"], dts, "t")
    OB.spec_bdyupdate(g, s["mu"], s["mu_tend"], dts, "m")
    OB.spec_bdyupdate(g, s["muts"], s["mu_tend"], dts, "m")
    OD.advance_w(g, s, dts, g.epssm, s["cf1"], s["cf2"], s["cf3"])
    OD.sumflux(g, s, iteration, nsub)
    OB.spec_bdyupdate_ph(g, s["ph_save"], s["ph"], s["ph_tend"], s["mu_tend"], s["muts"], dts)
    OB.zero_grad_bdy(g, s["w"], "w")
    s["pm1"] = OD.calc_p_rho(g, s["al"], s["p"], s["ph"], s["alt"], s["t"], s["t_save"], s["c2a"], s["pm1"], s["mu"],
                             s["muts"], s["rdnw"], g.smdiv, iteration)
    OD.set_physical_bc3d(g, s["ph"], "w")
    OD.set_physical_bc3d(g, s["al"], "p")
    OD.set_physical_bc3d(g, s["p"], "p")
    for k in ("muts", "mu", "mudf"):
        OD.set_physical_bc2d(g, s[k], "t")


SUB_OUT = ("u", "v", "w", "ph", "t", "mu", "muts", "p", "al", "ww", "ru_m", "rv_m", "ww_m", "t_2save", "pm1", "mudf",
           "muave")


def test_composed_acoustic_substep_and_its_adjoint_against_the_oracle():
    """pywrf_b200.adjoint.acoustic_substep (the substep composed from the
    operators' Functions) on the small case's state just before stage 2's
    substeps: every output within 3x the float32 oracle's own error of the
    float64 oracle's substep, and the gradient of a seeded linear functional
    of 17 outputs, in 14 inputs, against float64 central differences of the
    oracle's substep along seeded directions (the outputs' error allowance:
    3x the float32 oracle's own error plus 2e-6)."""
    import copy

    from helpers import SMALL
    from oracle.model import OracleModel
    from pywrf_b200 import synthetic

    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    snap = {}

    def probe(name, m):
        if name == "s2.acprep" and not snap:
            snap.update(copy.deepcopy(m.st))

    m = OracleModel(g, inputs, bdy, np.float64)
    m.run(1)
    m.step(2, probe)
    dts = g.dt / g.soundsteps
    it, nsub = 1, g.soundsteps // 2

    def oracle_run(dtype, pert=None):
        s = {k: (np.array(v, dtype) if isinstance(v, np.ndarray) else v) for k, v in snap.items()}
        if pert:
            for k, d in pert.items():
                s[k] = s[k] + d
        _oracle_substep(g, s, it, nsub, dts)
        return s

    o64, o32 = oracle_run(np.float64), oracle_run(np.float32)
    st = {k: _cuda(snap[k]).requires_grad_(True) for k in adjoint.SUBSTEP_STATE}
    data = {k: _cuda(snap[k]) for k in adjoint.SUBSTEP_DATA}
    sc = dict(epssm=g.epssm, emdiv=g.emdiv, smdiv=g.smdiv, cf1=float(snap["cf1"]), cf2=float(snap["cf2"]),
              cf3=float(snap["cf3"]), rdx=g.rdx, rdy=g.rdy)
    out = adjoint.acoustic_substep(st, data, it, nsub, dts, **sc)
    bad = []
    for k in SUB_OUT:
        c = out[k].detach().double().cpu().numpy()
        err, floor = rel_l2(c, o64[k]), rel_l2(o32[k], o64[k])
        # the stand-alone operators round like the fused step's kernels, not
        # like numpy: a 2e-6 allowance on top of 3x the oracle's own error
        if not err <= 3.0 * floor + 2e-6:
            bad.append((k, err, floor))
    assert not bad, bad
    rng = np.random.default_rng(77)
    cot = {k: rng.standard_normal(np.shape(snap[k])) for k in SUB_OUT}
    sum((out[k].double() * torch.tensor(cot[k], device="cuda")).sum() for k in SUB_OUT).backward()

    def loss(pert):
        s = oracle_run(np.float64, pert)
        return sum(float((s[k] * cot[k]).sum()) for k in SUB_OUT)

    for name in ("u", "v", "t", "ph", "w", "mu", "muts", "p", "al", "ww", "ru_tend", "t_tend", "ph_tend", "c2a"):
        gr = st[name].grad.double().cpu().numpy()
        d = rng.standard_normal(gr.shape)
        eps = 1e-6 * float(np.abs(snap[name]).max() or 1.0)
        fd = (loss({name: eps * d}) - loss({name: -eps * d})) / (2 * eps)
        an, scale = float((gr * d).sum()), float(np.abs(gr * d).sum())
        assert abs(an - fd) <= 2e-3 * abs(fd) + 1e-5 * scale, (name, an, fd, scale)


def _oracle_acoustic_stage(g, s, rk_step, nsub, dts):
    """The acoustic part of one RK stage of the oracle (its model loop,
    solver.py:1258-1492) on the state dict ``s``, in place."""
    from oracle import dynamics as OD

    OD.small_step_prep(g, s, rk_step)
    s["pm1"] = OD.calc_p_rho(g, s["al"], s["p"], s["ph"], s["alt"], s["t"], s["t_save"], s["c2a"], s["pm1"], s["mu"],
                             s["muts"], s["rdnw"], g.smdiv, 0)
    OD.calc_coef_w(g, s["a"], s["alpha"], s["gamma"], s["mut"], s["cqw"], s["rdn"], s["rdnw"], s["c2a"], dts, g.epssm,
                   g.top_lid)
    for k, var in (("ru_tend", "u"), ("rv_tend", "v"), ("ph", "w"), ("al", "p"), ("p", "p"), ("t_1", "t"),
                   ("t_save", "t")):
        OD.set_physical_bc3d(g, s[k], var)
    for k in ("mu_1", "mu", "mudf"):
        OD.set_physical_bc2d(g, s[k], "t")
    for it in range(1, nsub + 1):
        _oracle_substep(g, s, it, nsub, dts)
    OD.calc_mu_uv_1(g, s["muts"], s["muus"], s["muvs"])
    OD.small_step_finish(g, s, nsub, dts, rk_step)
    if rk_step == 3:
        for k, var in (("ru_m", "u"), ("rv_m", "v"), ("ww_m", "w")):
            OD.set_physical_bc3d(g, s[k], var)
        OD.set_physical_bc2d(g, s["mut"], "t")
        OD.set_physical_bc2d(g, s["muts"], "t")


STAGE_OUT = ("u", "v", "w", "ph", "t", "mu", "muts", "p", "al", "ww", "ru_m", "rv_m", "ww_m", "t_2save", "pm1")


@pytest.mark.parametrize("rk_step", [2, 3])
def test_composed_acoustic_stage_and_its_adjoint_against_the_oracle(rk_step):
    """pywrf_b200.adjoint.acoustic_stage (small_step_prep, calc_p_rho,
    calc_coef_w, the substeps, calc_mu_uv_1 and small_step_finish composed
    from their Functions) on the small case's state after the tendencies of
    step 2, stage 2 (2 substeps) and stage 3 (4 substeps): the outputs
    against the float64 oracle (3x the float32 oracle's own error plus 2e-6),
    and the gradient of a seeded linear functional of 15 outputs in 12
    inputs against float64 central differences of the oracle's stage."""
    import copy

    from helpers import SMALL
    from oracle.model import OracleModel
    from pywrf_b200 import synthetic

    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    snap = {}
    tag = f"s{rk_step}.tend"

    def probe(name, m):
        if name == tag and not snap:
            snap.update(copy.deepcopy(m.st))

    m = OracleModel(g, inputs, bdy, np.float64)
    m.run(1)
    m.step(2, probe)
    dts = g.dt / g.soundsteps
    nsub = g.soundsteps // 2 if rk_step == 2 else g.soundsteps

    def oracle_run(dtype, pert=None):
        s = {k: (np.array(v, dtype) if isinstance(v, np.ndarray) else v) for k, v in snap.items()}
        if pert:
            for k, d in pert.items():
                s[k] = s[k] + d
        _oracle_acoustic_stage(g, s, rk_step, nsub, dts)
        return s

    o64, o32 = oracle_run(np.float64), oracle_run(np.float32)
    st = {k: _cuda(snap[k]).requires_grad_(True) for k in adjoint.STAGE_STATE}
    data = {k: _cuda(snap[k]) for k in adjoint.STAGE_DATA}
    sc = dict(epssm=g.epssm, emdiv=g.emdiv, smdiv=g.smdiv, cf1=float(snap["cf1"]), cf2=float(snap["cf2"]),
              cf3=float(snap["cf3"]), rdx=g.rdx, rdy=g.rdy)
    out = adjoint.acoustic_stage(st, data, rk_step, nsub, dts, **sc)
    bad = []
    for k in STAGE_OUT:
        c = out[k].detach().double().cpu().numpy()
        err, floor = rel_l2(c, o64[k]), rel_l2(o32[k], o64[k])
        if not err <= 3.0 * floor + 2e-6:
            bad.append((k, err, floor))
    assert not bad, bad
    rng = np.random.default_rng(78)
    cot = {k: rng.standard_normal(np.shape(snap[k])) for k in STAGE_OUT}
    sum((out[k].double() * torch.tensor(cot[k], device="cuda")).sum() for k in STAGE_OUT).backward()

    def loss(pert):
        s = oracle_run(np.float64, pert)
        return sum(float((s[k] * cot[k]).sum()) for k in STAGE_OUT)

    for name in ("u", "v", "t", "ph", "w", "mu", "mu_1", "p", "ww", "ru_tend", "t_tend", "ph_tend"):
        gr = st[name].grad.double().cpu().numpy()
        d = rng.standard_normal(gr.shape)
        eps = 1e-6 * float(np.abs(snap[name]).max() or 1.0)
        fd = (loss({name: eps * d}) - loss({name: -eps * d})) / (2 * eps)
        an, scale = float((gr * d).sum()), float(np.abs(gr * d).sum())
        assert abs(an - fd) <= 2e-3 * abs(fd) + 1e-5 * scale, (name, an, fd, scale)


def _oracle_dynamics_stage(g, s, rk_step, nsub, dts, dtbc=None):
    """The dynamics of one RK stage of the oracle (its model loop,
    solver.py:736-1492) on ``s``; the first stage needs the boundary time
    ``dtbc``."""
    from oracle import boundary as OB
    from oracle import dynamics as OD

    OD.calculate_full(g, s["mut"], s["mub"], s["mu"])
    OD.calc_mu_uv(g, s["mu"], s["mub"], s["muu"], s["muv"])
    OD.couple_momentum(g, s["muu"], s["ru"], s["u"], s["msfu"], s["muv"], s["rv"], s["v"], s["msfvx_inv"], s["mut"],
                       s["rw"], s["w"], s["msft"])
    OD.calc_ww_cp(g, s["u"], s["v"], s["muu"], s["muv"], s["c1h"], s["ww"], s["msftx"], s["msfuy"], s["msfvx_inv"],
                  s["dnw"])
    OD.calc_cq(g, s["moist"], s["cqu"], s["cqv"], s["cqw"])
    OD.calc_alt(g, s["alt"], s["al"], s["alb"])
    OD.calc_php(g, s["php"], s["ph"], s["phb"])
    for nm, var in (("ru", "u"), ("rv", "v"), ("rw", "w"), ("ww", "w"), ("php", "w"), ("alt", "t"), ("p", "p")):
        OD.set_physical_bc3d(g, s[nm], var)
    OD.set_physical_bc2d(g, s["muu"], "u")
    OD.set_physical_bc2d(g, s["muv"], "v")
    OD.set_physical_bc2d(g, s["mut"], "t")
    OD.set_physical_bc3d(g, s["al"], "p")
    OD.set_physical_bc3d(g, s["ph"], "w")
    if rk_step == 1:
        for nm in ("ru_tendf", "rv_tendf", "rw_tendf", "ph_tendf", "t_tendf", "mu_tendf", "moist_tend"):
            s[nm] = np.zeros_like(s[nm])
        for nm in ("z", "rdz", "rdzw", "zx", "zy", "defor11", "defor22", "defor12", "xkmh", "xkhh"):
            s[nm] = s[nm].copy()
        OD.compute_diff_metrics(g, s["ph"], s["phb"], s["z"], s["rdz"], s["rdzw"], s["zx"], s["zy"])
        for nm, var in (("rdzw", "w"), ("rdz", "w"), ("z", "w"), ("zx", "e"), ("zy", "f")):
            OD.set_physical_bc3d(g, s[nm], var)
        OD.cal_deform_and_div(g, s["u"], s["v"], s["defor11"], s["defor22"], s["defor12"], s["msfux"], s["msfuy"],
                              s["msfvx"], s["msfvy"], s["msftx"], s["msfty"], s["dn"], s["dnw"], s["rdzw"], s["fnm"],
                              s["fnp"], s["cf1"], s["cf2"], s["cf3"], s["zx"], s["zy"])
        OD.calculate_km_kh(g, s["xkmh"], s["xkhh"], s["defor11"], s["defor22"], s["defor12"], s["msftx"], s["msfty"])
        OD.set_physical_bc3d(g, s["xkmh"], "t")
        OD.set_physical_bc3d(g, s["xkhh"], "t")
    for nm in ("ru_tend", "rv_tend", "rw_tend", "t_tend", "ph_tend", "u_save", "v_save", "w_save", "ph_save", "t_save"):
        s[nm] = np.zeros_like(s[nm])
    s["mu_tend"] = np.zeros_like(s["mu_tend"])
    s["mu_save"] = np.zeros_like(s["mu_save"])
    OD.advect_u(g, s["u"], s["ru_tend"], s["ru"], s["rv"], s["ww"], s["msfux"], s["fnm"], s["fnp"], s["rdnw"])
    OD.advect_v(g, s["v"], s["rv_tend"], s["ru"], s["rv"], s["ww"], s["msfvx"], s["msfvy"], s["fnm"], s["fnp"], s["rdnw"])
    OD.advect_w(g, s["w"], s["rw_tend"], s["ru"], s["rv"], s["ww"], s["msftx"], s["fnm"], s["fnp"], s["rdn"])
    OD.advect_scalar(g, s["t"], s["t_tend"], s["ru"], s["rv"], s["ww"], s["msftx"], s["fnm"], s["fnp"], s["rdnw"])
    OD.rhs_ph(g, s["ph_tend"], s["u"], s["v"], s["ww"], s["ph"], s["phb"], s["w"], s["mut"], s["muu"], s["muv"],
              s["fnm"], s["fnp"], s["rdnw"], s["cfn"], s["cfn1"], s["msfux"], s["msfvy"], s["msfty"])
    OD.horizontal_pressure_gradient(g, s["ru_tend"], s["rv_tend"], s["ph"], s["alt"], s["p"], s["pb"], s["al"],
                                    s["php"], s["cqu"], s["cqv"], s["muu"], s["muv"], s["mu"], s["fnm"], s["fnp"],
                                    s["rdnw"], s["cf1"], s["cf2"], s["cf3"], s["msfux"], s["msfuy"], s["msfvx"],
                                    s["msfvy"])
    OD.pg_buoy_w(g, s["rw_tend"], s["p"], s["cqw"], s["mu"], s["mub"], s["rdnw"], s["rdn"], s["msfty"])
    OD.coriolis(g, s["ru"], s["rv"], s["rw"], s["ru_tend"], s["rv_tend"], s["rw_tend"], s["msftx"], s["msfty"],
                s["msfux"], s["msfuy"], s["msfvx"], s["msfvy"], s["f"], s["e"], s["sina"], s["cosa"], s["fnm"],
                s["fnp"])
    OD.curvature(g, s["ru"], s["rv"], s["rw"], s["u"], s["v"], s["ru_tend"], s["rv_tend"], s["rw_tend"], s["msfux"],
                 s["msfuy"], s["msfvx"], s["msfvy"], s["msftx"], s["msfty"], s["fnm"], s["fnp"])
    bd = s["bdy"]
    if rk_step == 1:
        mp = (s["msfux"], s["msfuy"], s["msfvx"], s["msfvx_inv"], s["msfvy"], s["msftx"], s["msfty"])
        for name in ("u", "v", "w"):
            OD.horizontal_diffusion(g, name, s[name], s[f"r{name}_tendf"], s["mut"], *mp, s["xkmh"])
        OD.horizontal_diffusion(g, "m", s["t"], s["t_tendf"], s["mut"], *mp, s["xkhh"], base=s["t_init"])
        fcx, gcx = s["fcx"], s["gcx"]
        OB.relax_bdytend(g, s["ru"], s["u_save"], bd["u"], "u", dtbc, fcx, gcx)
        OB.relax_bdytend(g, s["rv"], s["v_save"], bd["v"], "v", dtbc, fcx, gcx)
        mw = (slice(0, g.nz), slice(g.jds, g.jde - 1), slice(g.ids, g.ide - 1))
        s["rfield"] = s["rfield"].copy()
        OB.mass_weight(s["ph"], s["mut"], s["rfield"], *mw)
        OB.relax_bdytend(g, s["rfield"], s["ph_save"], bd["ph"], "h", dtbc, fcx, gcx)
        OB.mass_weight(s["t"], s["mut"], s["rfield"], *mw)
        OB.relax_bdytend(g, s["rfield"], s["t_save"], bd["t"], "t", dtbc, fcx, gcx)
        OB.relax_bdytend(g, s["mu"][None], s["mu_tend"][None], bd["mu"], "m", dtbc, fcx, gcx)
    OD.rk_addtend_dry(g, s["ru_tend"], s["rv_tend"], s["rw_tend"], s["ph_tend"], s["t_tend"], s["ru_tendf"],
                      s["rv_tendf"], s["rw_tendf"], s["ph_tendf"], s["t_tendf"], s["u_save"], s["v_save"],
                      s["w_save"], s["ph_save"], s["t_save"], s["mu_tend"], s["mu_tendf"], rk_step, s["h_diabatic"],
                      s["mut"], s["msfty"], s["msfuy"], s["msfvx"], s["msfvx_inv"])
    OB.spec_bdytend(g, s["ru_tend"], bd["u"], "u")
    OB.spec_bdytend(g, s["rv_tend"], bd["v"], "v")
    OB.spec_bdytend(g, s["ph_tend"], bd["ph"], "h")
    OB.spec_bdytend(g, s["t_tend"], bd["t"], "t")
    OB.spec_bdytend(g, s["mu_tend"][None], bd["mu"], "m")
    _oracle_acoustic_stage(g, s, rk_step, nsub, dts)


@pytest.mark.parametrize("rk_step", [1, 2, 3])
def test_composed_dynamics_stage_and_its_adjoint_against_the_oracle(rk_step):
    """pywrf_b200.adjoint.dynamics_stage (rk_step_prep, at the first stage the
    eddy viscosities, the advection of u, v, w, theta, the tendency terms, at
    the first stage the diffusion and relaxation, rk_addtend_dry,
    spec_bdytend and the acoustic part, composed from their Functions) from
    the small case's state at the start of stage 1 / 2 / 3 of step 2: the
    outputs against the float64 oracle (3x the float32 oracle's own error
    plus 2e-6) and the gradient of a seeded linear functional of 15 outputs
    in 10 inputs against float64 central differences of the oracle's
    stage."""
    g, snap, nsub, dts, dt_rk, dtbc = _stage_start(rk_step)

    def oracle_run(dtype, pert=None):
        s = {k: _cast(v, dtype) for k, v in snap.items()}
        if pert:
            for k, d in pert.items():
                s[k] = s[k] + d
        _oracle_dynamics_stage(g, s, rk_step, nsub, dts, dtbc)
        return s

    o64, o32 = oracle_run(np.float64), oracle_run(np.float32)
    st = {k: _cuda(snap[k]).requires_grad_(True) for k in adjoint.DYN_STATE}
    data = {k: _cuda(snap[k]) for k in adjoint.DYN_DATA}
    bt = _stage_bdy(snap, rk_step == 1)
    sc = dict(epssm=g.epssm, emdiv=g.emdiv, smdiv=g.smdiv, cf1=float(snap["cf1"]), cf2=float(snap["cf2"]),
              cf3=float(snap["cf3"]), cfn=float(snap["cfn"]), cfn1=float(snap["cfn1"]), rdx=g.rdx, rdy=g.rdy,
              dtbc=dtbc)
    out = adjoint.dynamics_stage(st, data, bt, rk_step, nsub, dts, **sc)
    bad = []
    for k in STAGE_OUT:
        c = out[k].detach().double().cpu().numpy()
        err, floor = rel_l2(c, o64[k]), rel_l2(o32[k], o64[k])
        if not err <= 3.0 * floor + 2e-6:
            bad.append((k, err, floor))
    assert not bad, bad
    rng = np.random.default_rng(79)
    cot = {k: rng.standard_normal(np.shape(snap[k])) for k in STAGE_OUT}
    sum((out[k].double() * torch.tensor(cot[k], device="cuda")).sum() for k in STAGE_OUT).backward()

    def loss(pert):
        s = oracle_run(np.float64, pert)
        return sum(float((s[k] * cot[k]).sum()) for k in STAGE_OUT)

    bad = []
    for name in ("u", "v", "t", "ph", "w", "mu", "mu_1", "p", "moist", "ru_tendf"):
        gr = _grad(st[name])
        d = rng.standard_normal(gr.shape)
        eps = 1e-6 * float(np.abs(snap[name]).max() or 1.0)
        fd = (loss({name: eps * d}) - loss({name: -eps * d})) / (2 * eps)
        an, scale = float((gr * d).sum()), float(np.abs(gr * d).sum())
        if not abs(an - fd) <= 2e-3 * abs(fd) + COMPOSED_FLOOR * scale:
            bad.append((name, an, fd, scale))
    assert not bad, bad


# composed operators: the analytic product is a float32 sum over many
# operators' reverse kernels, whose rounding leaves an absolute error of a
# few 1e-6 .. 1e-5 of the sum of the terms' magnitudes (scale) where the
# terms cancel to 1e-3 of it; the floor allows 3e-5 of the scale
COMPOSED_FLOOR = 3e-5


def _grad(t):
    """A leaf's gradient as float64 numpy (zero when the graph never reached
    it: an input the composed operators overwrite before reading)."""
    if t.grad is None:
        return np.zeros(tuple(t.shape))
    return t.grad.double().cpu().numpy()


def _stage_start(rk_step):
    """The small case's float64 oracle state at the start of RK stage
    ``rk_step`` of step 2, with the stage's (nsub, dts, dt_rk) and the
    boundary time dtbc of step 2 (pywrf/solver.py:713-734)."""
    import copy

    from helpers import SMALL
    from oracle.model import OracleModel
    from pywrf_b200 import synthetic

    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    snap = {}
    tag = f"s{rk_step - 1}.moist"

    def probe(name, m):
        if name == tag and not snap:
            snap.update(copy.deepcopy(m.st))

    m = OracleModel(g, inputs, bdy, np.float64)
    m.run(1)
    if rk_step == 1:
        snap.update(copy.deepcopy(m.st))
    else:
        m.step(2, probe)
    dts = g.dt / g.soundsteps
    nsub, dt_rk = {1: (1, g.dt / 3.0), 2: (g.soundsteps // 2, 0.5 * g.dt), 3: (g.soundsteps, g.dt)}[rk_step]
    if rk_step == 1:
        dts = g.dt / 3.0
    assert 2 % g.bdy_interval != 1  # no boundary record is loaded at step 2
    dtbc = g.dt * (2 - m.it_bdy * g.bdy_interval)
    return g, snap, nsub, dts, dt_rk, dtbc


def _cast(v, dtype):
    if isinstance(v, np.ndarray):
        return np.array(v, dtype)
    if isinstance(v, dict):
        return {k: _cast(x, dtype) for k, x in v.items()}
    return v


def _stage_bdy(snap, with_values):
    """The boundary arrays a composed stage takes, by stagger letter."""
    names = ("txs", "txe", "tys", "tye") + (("xs", "xe", "ys", "ye") if with_values else ())
    letters = {"u": "u", "v": "v", "h": "ph", "t": "t", "m": "mu", "q": "qv"}
    return {v: {s_: _cuda(snap["bdy"][f][s_]) for s_ in names} for v, f in letters.items()}


def _oracle_rk_stage(g, s, rk_step, nsub, dts, dt_rk, dtbc=None):
    """One RK stage of the oracle: the dynamics, then the moisture part (its
    model loop, solver.py:1548-1712)."""
    from oracle import boundary as OB
    from oracle import dynamics as OD

    _oracle_dynamics_stage(g, s, rk_step, nsub, dts, dtbc)
    s["advect_tend"] = s["advect_tend"].copy()
    for im in range(1, 7):
        s["advect_tend"][im][0:g.nz, g.jts:g.jte, g.its:g.ite] = 0.0
        OD.advect_scalar(g, s["moist"][im], s["advect_tend"][im], s["ru_m"], s["rv_m"], s["ww_m"], s["msftx"],
                         s["fnm"], s["fnp"], s["rdnw"])
        if rk_step == 1:
            OD.horizontal_diffusion(g, "m", s["moist"][im], s["moist_tend"][im], s["muts"], s["msfux"], s["msfuy"],
                                    s["msfvx"], s["msfvx_inv"], s["msfvy"], s["msftx"], s["msfty"], s["xkhh"])
    if rk_step == 1:
        rq = np.zeros_like(s["t"])
        OB.mass_weight(s["moist"][1], s["mut"], rq, slice(0, g.nz - 1), slice(g.jds, g.jde - 1),
                       slice(g.ids, g.ide - 1))
        OB.relax_bdytend(g, rq, s["moist_tend"][1], s["bdy"]["qv"], "q", dtbc, s["fcx"], s["gcx"])
        OB.spec_bdytend(g, s["moist_tend"][1], s["bdy"]["qv"], "q")
    OD.rk_update_scalar(g, s["moist_old"], s["moist"], s["moist_tend"], s["advect_tend"], s["msfty"], s["mu_1"],
                        s["mu"], s["mub"], rk_step, dt_rk)
    for im in range(2, 7):
        OB.flow_dep_bdy(g, s["moist"][im], s["ru_m"], s["rv_m"])
    OD.calc_p_rho_phi(g, s["moist"][1], s["al"], s["alb"], s["mu"], s["muts"], s["ph"], s["p"], s["pb"], s["t"],
                      s["rdnw"])
    if rk_step < 3:
        for nm, var in (("u", "U"), ("v", "V"), ("w", "w"), ("t", "p"), ("ph", "w")):
            OD.set_physical_bc3d(g, s[nm], var)
        OD.set_physical_bc2d(g, s["mu"], "t")
        for im in range(1, 7):
            OD.set_physical_bc3d(g, s["moist"][im], "p")


RK_OUT = STAGE_OUT + ("moist",)


@pytest.mark.parametrize("rk_step", [1, 2, 3])
def test_composed_rk_stage_and_its_adjoint_against_the_oracle(rk_step):
    """pywrf_b200.adjoint.rk_stage (dynamics_stage -- at the first stage with
    the eddy viscosities, the horizontal diffusion and the relaxation --
    then the moisture advection, at the first stage the moisture diffusion
    and qv's relaxation, rk_update_scalar, flow_dep_bdy and calc_p_rho_phi)
    from the small case's state at the start of stage 1 / 2 / 3 of step 2:
    the outputs (moisture included) against the float64 oracle (3x the
    float32 oracle's own error plus 2e-6), and the gradient of a seeded
    linear functional of 16 outputs in 8 inputs against float64 central
    differences of the oracle's stage."""
    g, snap, nsub, dts, dt_rk, dtbc = _stage_start(rk_step)

    def oracle_run(dtype, pert=None):
        s = {k: _cast(v, dtype) for k, v in snap.items()}
        if pert:
            for k, d in pert.items():
                s[k] = s[k] + d
        _oracle_rk_stage(g, s, rk_step, nsub, dts, dt_rk, dtbc)
        return s

    o64, o32 = oracle_run(np.float64), oracle_run(np.float32)
    st = {k: _cuda(snap[k]).requires_grad_(True) for k in adjoint.RK_STATE}
    data = {k: _cuda(snap[k]) for k in adjoint.RK_DATA}
    bt = _stage_bdy(snap, rk_step == 1)
    sc = dict(epssm=g.epssm, emdiv=g.emdiv, smdiv=g.smdiv, cf1=float(snap["cf1"]), cf2=float(snap["cf2"]),
              cf3=float(snap["cf3"]), cfn=float(snap["cfn"]), cfn1=float(snap["cfn1"]), rdx=g.rdx, rdy=g.rdy,
              dtbc=dtbc)
    out = adjoint.rk_stage(st, data, bt, rk_step, nsub, dts, dt_rk, **sc)
    bad = []
    for k in RK_OUT:
        c = out[k].detach().double().cpu().numpy()
        err, floor = rel_l2(c, o64[k]), rel_l2(o32[k], o64[k])
        if not err <= 3.0 * floor + 2e-6:
            bad.append((k, err, floor))
    assert not bad, bad
    rng = np.random.default_rng(80 + rk_step)
    cot = {k: rng.standard_normal(np.shape(snap[k])) for k in RK_OUT}
    sum((out[k].double() * torch.tensor(cot[k], device="cuda")).sum() for k in RK_OUT).backward()

    def loss(pert):
        s = oracle_run(np.float64, pert)
        return sum(float((s[k] * cot[k]).sum()) for k in RK_OUT)

    bad = []
    for name in ("u", "v", "t", "ph", "w", "mu", "p", "moist") + (("moist_tend",) if rk_step > 1 else ()):
        gr = _grad(st[name])
        d = rng.standard_normal(gr.shape)
        eps = 1e-6 * float(np.abs(snap[name]).max() or 1.0)
        fd = (loss({name: eps * d}) - loss({name: -eps * d})) / (2 * eps)
        an, scale = float((gr * d).sum()), float(np.abs(gr * d).sum())
        if not abs(an - fd) <= 2e-3 * abs(fd) + COMPOSED_FLOOR * scale:
            bad.append((name, an, fd, scale))
    assert not bad, bad


def test_first_stage_viscosity_and_diffusion_operators_against_the_oracle():
    """pywrf_b200.adjoint.eddy_viscosity (compute_diff_metrics,
    cal_deform_and_div, calculate_km_kh), the halo copies of xkmh / xkhh and
    horizontal_diffusion of u, v, w, theta (about t_init) and qc from the
    small case's state at the start of step 2: the outputs against the
    float64 oracle (3x the float32 oracle's own error plus 2e-6), and the
    gradient of a seeded linear functional of the outputs in u, v, w, ph, t,
    mut, muts and qc against float64 central differences of the oracle."""
    from oracle import dynamics as OD

    g, snap, *_ = _stage_start(1)
    outs = ("xkmh", "xkhh", "ru_tendf", "rv_tendf", "rw_tendf", "t_tendf", "qc_tend")
    mp_names = ("msfux", "msfuy", "msfvx", "msfvx_inv", "msfvy", "msftx", "msfty")

    def oracle(dtype, pert=None):
        s = {k: _cast(v, dtype) for k, v in snap.items() if k != "bdy"}
        if pert:
            for k, d in pert.items():
                s[k] = s[k] + d
        OD.compute_diff_metrics(g, s["ph"], s["phb"], s["z"], s["rdz"], s["rdzw"], s["zx"], s["zy"])
        for nm, var in (("rdzw", "w"), ("rdz", "w"), ("z", "w"), ("zx", "e"), ("zy", "f")):
            OD.set_physical_bc3d(g, s[nm], var)
        OD.cal_deform_and_div(g, s["u"], s["v"], s["defor11"], s["defor22"], s["defor12"], s["msfux"], s["msfuy"],
                              s["msfvx"], s["msfvy"], s["msftx"], s["msfty"], s["dn"], s["dnw"], s["rdzw"], s["fnm"],
                              s["fnp"], s["cf1"], s["cf2"], s["cf3"], s["zx"], s["zy"])
        OD.calculate_km_kh(g, s["xkmh"], s["xkhh"], s["defor11"], s["defor22"], s["defor12"], s["msftx"], s["msfty"])
        OD.set_physical_bc3d(g, s["xkmh"], "t")
        OD.set_physical_bc3d(g, s["xkhh"], "t")
        mp = [s[k] for k in mp_names]
        r = {"xkmh": s["xkmh"], "xkhh": s["xkhh"]}
        for name in ("u", "v", "w"):
            r[f"r{name}_tendf"] = np.zeros_like(s[name])
            OD.horizontal_diffusion(g, name, s[name], r[f"r{name}_tendf"], s["mut"], *mp, s["xkmh"])
        r["t_tendf"] = np.zeros_like(s["t"])
        OD.horizontal_diffusion(g, "m", s["t"], r["t_tendf"], s["mut"], *mp, s["xkhh"], base=s["t_init"])
        r["qc_tend"] = np.zeros_like(s["t"])
        OD.horizontal_diffusion(g, "m", s["moist"][2], r["qc_tend"], s["muts"], *mp, s["xkhh"])
        return r

    o64, o32 = oracle(np.float64), oracle(np.float32)
    st = {k: _cuda(snap[k]).requires_grad_(True) for k in ("u", "v", "w", "ph", "t", "mut", "muts", "xkmh", "xkhh")}
    qc = _cuda(snap["moist"][2]).requires_grad_(True)
    data = {k: _cuda(snap[k]) for k in adjoint.DYN_DATA}
    rdx, rdy = g.rdx, g.rdy
    xkmh, xkhh = adjoint.eddy_viscosity(st, data, rdx, rdy, float(snap["cf1"]), float(snap["cf2"]),
                                        float(snap["cf3"]))
    xkmh, xkhh = adjoint.halo(xkmh, "t", rdx, rdy), adjoint.halo(xkhh, "t", rdx, rdy)
    hd = {k: data[k] for k in adjoint.HDIFF_DATA}
    z = lambda: torch.zeros_like(st["u"])  # noqa: E731
    out = {"xkmh": xkmh, "xkhh": xkhh}
    for name in ("u", "v", "w"):
        out[f"r{name}_tendf"] = adjoint.horizontal_diffusion(name, st[name], z(), st["mut"], xkmh, hd, rdx, rdy)
    out["t_tendf"] = adjoint.horizontal_diffusion("m", st["t"], z(), st["mut"], xkhh, hd, rdx, rdy,
                                                  base=data["t_init"])
    out["qc_tend"] = adjoint.horizontal_diffusion("m", qc, z(), st["muts"], xkhh, hd, rdx, rdy)
    bad = []
    for k in outs:
        c = out[k].detach().double().cpu().numpy()
        err, floor = rel_l2(c, o64[k]), rel_l2(o32[k], o64[k])
        if not err <= 3.0 * floor + 2e-6:
            bad.append((k, err, floor))
    assert not bad, bad
    rng = np.random.default_rng(91)
    cot = {k: rng.standard_normal(o64[k].shape) for k in outs}
    sum((out[k].double() * torch.tensor(cot[k], device="cuda")).sum() for k in outs).backward()

    def loss(pert):
        r = oracle(np.float64, pert)
        return sum(float((r[k] * cot[k]).sum()) for k in outs)

    grads = {k: st[k].grad for k in ("u", "v", "w", "ph", "t", "mut", "muts")}
    qpert = lambda d: np.concatenate([np.zeros((2,) + d.shape), d[None], np.zeros((4,) + d.shape)])  # noqa: E731
    for name, gr in list(grads.items()) + [("qc", qc.grad)]:
        gr = gr.double().cpu().numpy()
        d = rng.standard_normal(gr.shape)
        base = snap["moist"][2] if name == "qc" else snap[name]
        eps = 1e-6 * float(np.abs(base).max() or 1.0)
        key, dd = ("moist", qpert(d)) if name == "qc" else (name, d)
        fd = (loss({key: eps * dd}) - loss({key: -eps * dd})) / (2 * eps)
        an, scale = float((gr * d).sum()), float(np.abs(gr * d).sum())
        assert abs(an - fd) <= 2e-3 * abs(fd) + 1e-5 * scale, (name, an, fd, scale)


STEP_OUT = ("u", "v", "w", "ph", "t", "mu", "muts", "p", "al", "ww", "ru_m", "rv_m", "ww_m", "moist", "u_1", "t_1",
            "ph_1", "mu_1")


def _dry_start():
    """The small case after one full oracle step (float64), the model's
    scalars and its boundary arrays (solver layout)."""
    import copy

    from helpers import SMALL
    from oracle.model import OracleModel
    from pywrf_b200 import synthetic

    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    m = OracleModel(g, inputs, bdy, np.float64)
    m.run(1)
    return g, inputs, bdy, copy.deepcopy(m.st)


def test_whole_step_forward_and_reverse_replay_from_a_cuda_graph():
    """adjoint.capture: one whole step with WSM6 (adjoint.step with the
    microphysics), forward and reverse for seeded cotangents, captured once
    in a CUDA graph from the small case's state after its first step; two
    replays give the eager pass's gradients (relative L2 1e-5 per input:
    the scatter kernels' atomics may add in another order), and a replay
    after the inputs are changed in place follows the new inputs."""
    g, inputs, bdy, snap = _dry_start()
    names = tuple(dict.fromkeys(adjoint.RK_STATE + ("u_1", "w_1", "ph_1", "mu_1", "t_1", "v_1")))
    st = {k: _cuda(snap[k]).requires_grad_(True) for k in names}
    data = {k: _cuda(snap[k]) for k in dict.fromkeys(adjoint.STEP_DATA + adjoint._Microphysics.data)}
    bd = {f: {k: _cuda(v) for k, v in snap["bdy"][f].items()} for f in ("u", "v", "ph", "t", "mu", "qv")}
    sc = dict(epssm=g.epssm, emdiv=g.emdiv, smdiv=g.smdiv, cf1=float(snap["cf1"]), cf2=float(snap["cf2"]),
              cf3=float(snap["cf3"]), cfn=float(snap["cfn"]), cfn1=float(snap["cfn1"]), rdx=g.rdx, rdy=g.rdy)
    mp = lambda s: adjoint.microphysics(s, data, g.dt, g.rdx, g.rdy)  # noqa: E731
    gen = torch.Generator(device="cuda").manual_seed(11)
    cot = {k: torch.randn(st[k].shape, generator=gen, device="cuda") for k in STEP_OUT}
    grads = {}

    def run():
        for v in st.values():
            v.grad = None
        o = adjoint.step(st, data, bd, 2.0 * g.dt, dt=g.dt, soundsteps=g.soundsteps, microphysics=mp, **sc)
        sum((o[k] * cot[k]).sum() for k in STEP_OUT).backward()
        grads.clear()
        grads.update({k: v.grad for k, v in st.items() if v.grad is not None})

    def eager():
        run()
        torch.cuda.synchronize()
        return {k: v.detach().clone() for k, v in grads.items()}

    ref = eager()
    graph = adjoint.capture(run)
    captured = dict(grads)
    for _ in range(2):
        graph.replay()
    torch.cuda.synchronize()
    bad = [(k, rel_l2(captured[k].cpu().numpy(), ref[k].cpu().numpy())) for k in ref]
    assert not [b for b in bad if not b[1] <= 1e-5], bad
    # the replay reads the inputs' current values
    with torch.no_grad():
        st["t"].mul_(1.001)
        st["u"].add_(0.01)
    ref2 = eager()
    graph.replay()
    torch.cuda.synchronize()
    bad = [(k, rel_l2(captured[k].cpu().numpy(), ref2[k].cpu().numpy())) for k in ref2]
    assert not [b for b in bad if not b[1] <= 1e-5], bad
    assert any(rel_l2(ref2[k].cpu().numpy(), ref[k].cpu().numpy()) > 1e-4 for k in ref)
    del graph


def _dry_oracle(g, inputs, bdy, snap, dtype, nsteps, pert=None, bias=None):
    from oracle.model import OracleModel

    m = OracleModel(g, inputs, bdy, dtype, theta_bias=bias, microphysics=False)
    m.st = {k: _cast(v, dtype) for k, v in snap.items()}
    if pert:
        for k, d in pert.items():
            m.st[k] = m.st[k] + d
    m.step_count = 1
    m.run(nsteps)
    return m.st


@pytest.mark.parametrize("nsteps", [1, 2])
def test_composed_step_without_microphysics_and_its_adjoint_against_the_oracle(nsteps):
    """pywrf_b200.adjoint.step (the three RK stages and the end-of-step
    boundaries, composed from the operators' Functions) without
    microphysics, run through adjoint.rollout (one step per checkpoint
    segment) from the small case's state after its first step: the state
    after 1 and 2 steps against the float64 oracle's steps without
    microphysics (3x the float32 oracle's own error plus 2e-6), and the
    gradient of a seeded linear functional of 18 outputs with respect to 7
    inputs and a theta-tendency bias against float64 central differences of
    the oracle."""
    g, inputs, bdy, snap = _dry_start()
    o64 = _dry_oracle(g, inputs, bdy, snap, np.float64, nsteps)
    o32 = _dry_oracle(g, inputs, bdy, snap, np.float32, nsteps)
    names = tuple(dict.fromkeys(adjoint.RK_STATE + ("u_1", "w_1", "ph_1", "mu_1", "t_1", "v_1")))
    st = {k: _cuda(snap[k]).requires_grad_(True) for k in names}
    data = {k: _cuda(snap[k]) for k in adjoint.STEP_DATA}
    bd = {f: {k: _cuda(v) for k, v in snap["bdy"][f].items()} for f in ("u", "v", "ph", "t", "mu", "qv")}
    bias = torch.zeros_like(st["t"], requires_grad=True)
    sc = dict(epssm=g.epssm, emdiv=g.emdiv, smdiv=g.smdiv, cf1=float(snap["cf1"]), cf2=float(snap["cf2"]),
              cf3=float(snap["cf3"]), cfn=float(snap["cfn"]), cfn1=float(snap["cfn1"]), rdx=g.rdx, rdy=g.rdy)
    assert 2 % g.bdy_interval != 1 and 3 % g.bdy_interval != 1  # one boundary record throughout

    def one(*xs):
        n = int(round(float(xs[-1].item())))
        dtbc = g.dt * n  # boundary record 0 for every step here
        s = adjoint.step(dict(zip(names, xs[:-1])), data, bd, dtbc, dt=g.dt, soundsteps=g.soundsteps,
                         theta_bias=bias, **sc)
        return tuple(s[k] for k in names) + (xs[-1] + 1,)

    state = tuple(st[k] for k in names) + (torch.tensor(2.0, device="cuda"),)
    outs = adjoint.rollout(one, state, nsteps, every=1)
    out = dict(zip(names, outs))
    bad = []
    for k in STEP_OUT:
        c = out[k].detach().double().cpu().numpy()
        err, floor = rel_l2(c, o64[k]), rel_l2(o32[k], o64[k])
        if not err <= 3.0 * floor + 2e-6:
            bad.append((k, err, floor))
    assert not bad, bad
    rng = np.random.default_rng(97 + nsteps)
    cot = {k: rng.standard_normal(np.shape(snap[k])) for k in STEP_OUT}
    sum((out[k].double() * torch.tensor(cot[k], device="cuda")).sum() for k in STEP_OUT).backward()

    def loss(pert=None, b=None):
        s = _dry_oracle(g, inputs, bdy, snap, np.float64, nsteps, pert, b)
        return sum(float((s[k] * cot[k]).sum()) for k in STEP_OUT)

    for name in ("u", "v", "t", "ph", "w", "mu", "moist", "bias"):
        gr = _grad(bias if name == "bias" else st[name])
        d = rng.standard_normal(gr.shape)
        if name == "bias":
            eps = 1e-6
            fd = (loss(b=eps * d) - loss(b=-eps * d)) / (2 * eps)
        else:
            eps = 1e-6 * float(np.abs(snap[name]).max() or 1.0)
            fd = (loss({name: eps * d}) - loss({name: -eps * d})) / (2 * eps)
        an, scale = float((gr * d).sum()), float(np.abs(gr * d).sum())
        assert abs(an - fd) <= 2e-3 * abs(fd) + COMPOSED_FLOOR * scale, (name, an, fd, scale)


def _oracle_microphysics(g, s):
    """The oracle's microphysics block of the step (solver.py:1714-1766) on
    ``s``: prep, WSM6, finish and the equation of state."""
    from oracle import dynamics as OD
    from oracle import physics as OP

    for k in ("th_phy", "rho", "pi_phy", "p_phy", "dz8w", "h_diabatic", "qv_diabatic", "qc_diabatic", "rainnc",
              "rainncv", "snownc", "snowncv", "graupelnc", "graupelncv", "sr", "t", "al", "p", "moist"):
        s[k] = s[k].copy()
    OP.moist_physics_prep_em(g, s)
    mo = s["moist"]
    OP.wsm6(g, s["th_phy"], mo[1], mo[2], mo[3], mo[4], mo[5], mo[6], s["rho"], s["pi_phy"], s["p_phy"], s["dz8w"],
            float(g.dt), s["rainnc"], s["rainncv"], s["snownc"], s["snowncv"], s["graupelnc"], s["graupelncv"],
            s["sr"])
    OP.moist_physics_finish_em(g, s, g.dt)
    OD.calc_p_rho_phi(g, s["moist"][1], s["al"], s["alb"], s["mu"], s["muts"], s["ph"], s["p"], s["pb"], s["t"],
                      s["rdnw"])
    return s


MP_OUT = ("t", "moist", "al", "p", "h_diabatic")


def test_microphysics_adjoint_against_the_oracle():
    """pywrf_b200.adjoint.microphysics (the step's microphysics forward and
    its reverse: the equation of state's exact reverse, then prep + WSM6 +
    finish by reverse mode over a per-column tape of a restatement of the
    scheme) from the small case's state before the microphysics of step 2:
    the outputs against the float64 oracle (3x the float32 oracle's own
    error plus 2e-6), the restatement's own outputs against the forward's,
    and the gradient of a seeded linear functional of the outputs with
    respect to t, qv .. qg, al, p, ph, mu and muts against float64 central
    differences of the oracle's block."""
    import copy

    from helpers import SMALL
    from oracle.model import OracleModel
    from pywrf_b200 import synthetic

    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    snap = {}

    def probe(name, m):
        if name == "s3.moist" and not snap:
            snap.update(copy.deepcopy(m.st))

    m = OracleModel(g, inputs, bdy, np.float64)
    m.run(1)
    m.step(2, probe)
    assert float(np.abs(snap["moist"][3]).max()) > 0.0  # rain is present: the scheme is active

    def oracle(dtype, pert=None):
        s = {k: _cast(v, dtype) for k, v in snap.items()}
        if pert:
            for k, d in pert.items():
                s[k] = s[k] + d
        return _oracle_microphysics(g, s)

    o64, o32 = oracle(np.float64), oracle(np.float32)
    names = adjoint._Microphysics.fields
    st = {k: _cuda(snap[k]).requires_grad_(True) for k in names}
    data = {k: _cuda(snap[k]) for k in adjoint._Microphysics.data}
    out = adjoint.microphysics(st, data, g.dt, g.rdx, g.rdy)
    bad = []
    for k in MP_OUT:
        c = out[k].detach().double().cpu().numpy()
        err, floor = rel_l2(c, o64[k]), rel_l2(o32[k], o64[k])
        if not err <= 3.0 * floor + 2e-6:
            bad.append((k, err, floor))
    assert not bad, bad
    # the taped code's own outputs (its value path) against the forward's
    from pywrf_b200 import _native as N

    cg = adjoint.scalar_grid(st["t"].shape, g.rdx, g.rdy)
    cg.dt = float(g.dt)
    vals = {k: torch.zeros_like(st[k]) for k in ("t", "moist", "h_diabatic")}
    tab = adjoint._table({**{k: st[k].detach() for k in names}, **data})
    post = adjoint._table({**{k: st[k].detach() for k in names}, **data,
                           **{k: out[k].detach() for k in ("t", "moist", "al", "p")}})
    bars = {k: torch.zeros_like(st[k]) for k in ("t", "moist", "al", "p", "ph", "mu", "muts", "h_diabatic")}
    bars.update({k: torch.zeros_like(st["t"]) for k in ("alb", "pb")})
    n = ctypes.c_size_t(0)
    N.check(N.lib().wrf_microphysics_adj_work(ctypes.byref(cg), ctypes.byref(n)), "work")
    work = torch.empty(int(n.value), dtype=torch.float32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    N.check(N.lib().wrf_microphysics_adj(ctypes.byref(cg), tab, post, adjoint._table(bars),
                                         ctypes.c_void_p(work.data_ptr()), n, adjoint._table(vals), stream), "adj")
    torch.cuda.synchronize()
    R = (slice(0, g.nz - 1), slice(g.jds + 1, g.jde - 1), slice(g.ids + 1, g.ide - 1))
    for k in ("t", "h_diabatic"):
        a, b = vals[k].cpu().numpy()[R], out[k].detach().cpu().numpy()[R]
        assert rel_l2(a, b) <= 1e-5, (k, rel_l2(a, b))
    for im in range(1, 7):
        a, b = vals["moist"][im].cpu().numpy()[R], out["moist"][im].detach().cpu().numpy()[R]
        assert rel_l2(a, b) <= 1e-4, (im, rel_l2(a, b))
    rng = np.random.default_rng(101)
    cot = {k: rng.standard_normal(np.shape(snap[k])) for k in MP_OUT}
    sum((out[k].double() * torch.tensor(cot[k], device="cuda")).sum() for k in MP_OUT).backward()

    def loss(pert):
        s = oracle(np.float64, pert)
        return sum(float((s[k] * cot[k]).sum()) for k in MP_OUT)

    bad = []
    for name in ("t", "moist", "al", "p", "ph", "mu", "muts"):
        gr = st[name].grad.double().cpu().numpy()
        # relative perturbations: zero mixing ratios stay zero and small ones
        # keep their sign, so the differences stay on the scheme's branches
        d = rng.standard_normal(gr.shape) * np.abs(snap[name])
        eps = 1e-6
        fd = (loss({name: eps * d}) - loss({name: -eps * d})) / (2 * eps)
        an, scale = float((gr * d).sum()), float(np.abs(gr * d).sum())
        if not abs(an - fd) <= 2e-3 * abs(fd) + 1e-5 * scale:
            bad.append((name, an, fd, scale))
    assert not bad, bad


def _microphysics_state_before_step2():
    import copy

    from helpers import SMALL
    from oracle.model import OracleModel
    from pywrf_b200 import synthetic

    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    snap = {}

    def probe(name, m):
        if name == "s3.moist" and not snap:
            snap.update(copy.deepcopy(m.st))

    m = OracleModel(g, inputs, bdy, np.float64)
    m.run(1)
    m.step(2, probe)
    return g, snap


@pytest.mark.parametrize("dt, mixed", [(None, (1400, 2000)), (150.0, ()), (250.0, (5000,))])
def test_microphysics_adjoint_tape_and_tangent_columns_agree(dt, mixed):
    """wrf_microphysics_adj with the tape capacity at its default (every
    column taped) against capacity 1 (every column by forward-mode
    tangents) and, where listed, capacities that send only the columns with
    the longest tapes to the tangents (a mix in one call), at the case's dt
    of 45 s (one time-split loop: the tape stops before the point
    processes, which are reversed per level; its columns take 1 400 to
    2 600 entries here), 150 s (one loop of 120 s, the same split) and 250 s
    (two loops: the whole column on the tape twice): the input cotangents
    agree to float32 summation order (relative L2 1e-5 per field), and the
    setting is restored."""
    from pywrf_b200 import _native as N

    g, snap = _microphysics_state_before_step2()
    dt = float(g.dt if dt is None else dt)
    names = adjoint._Microphysics.fields
    st = {k: _cuda(snap[k]) for k in names}
    data = {k: _cuda(snap[k]) for k in adjoint._Microphysics.data}
    out = adjoint.microphysics(st, data, dt, g.rdx, g.rdy)
    cg = adjoint.scalar_grid(st["t"].shape, g.rdx, g.rdy)
    cg.dt = dt
    tab = adjoint._table({**st, **data})
    post = adjoint._table({**st, **data, **{k: out[k].detach() for k in ("t", "moist", "al", "p")}})
    gen = torch.Generator(device="cuda").manual_seed(5)
    seeds = {k: torch.randn(st[k].shape, generator=gen, device="cuda") for k in MP_OUT}
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def reverse(capacity):
        prev = ctypes.c_int(-1)
        N.check(N.lib().wrf_set_microphysics_tape_capacity(capacity, ctypes.byref(prev)), "capacity")
        try:
            bars = {k: torch.zeros_like(st[k]) for k in ("t", "moist", "al", "p", "ph", "mu", "muts", "h_diabatic")}
            bars.update({k: torch.zeros_like(st["t"]) for k in ("alb", "pb")})
            for k in MP_OUT:
                bars[k].copy_(seeds[k])
            n = ctypes.c_size_t(0)
            N.check(N.lib().wrf_microphysics_adj_work(ctypes.byref(cg), ctypes.byref(n)), "work")
            work = torch.empty(int(n.value), dtype=torch.float32, device="cuda")
            N.check(N.lib().wrf_microphysics_adj(ctypes.byref(cg), tab, post, adjoint._table(bars),
                                                 ctypes.c_void_p(work.data_ptr()), n, None, stream), "adj")
            torch.cuda.synchronize()
            return {k: v.double().cpu().numpy() for k, v in bars.items()}
        finally:
            back = ctypes.c_int(-1)
            N.check(N.lib().wrf_set_microphysics_tape_capacity(prev.value, ctypes.byref(back)), "restore")
            assert back.value == capacity

    taped = reverse(0)
    bad = []
    for cap in (1,) + tuple(mixed):
        other = reverse(cap)
        for k in ("t", "moist", "al", "p", "ph", "mu", "muts"):
            e = rel_l2(other[k], taped[k])
            if not e <= 1e-5:
                bad.append((k, cap, e))
    assert not bad, bad
    assert float(np.abs(taped["moist"][3]).max()) > 0.0


def test_theta_bias_gradient_of_two_steps_against_the_reference():
    """The adjoint configuration's check on the 28x28x16 case: two whole
    steps (RK stages, microphysics, end-of-step boundaries) composed from the
    operators' Functions under rollout (one checkpoint per step), from the
    initial state, with a learnable bias added to the theta tendency after
    rk_addtend_dry; loss = MSE of theta and qv on the lowest 10 levels
    against the second seed's state.  The loss at zero bias against the
    reference's (tests/golden/thbias_ref64.npz), and the gradient at the 16
    seeded points against the reference's float64 central differences
    (eps 1e-3): within 1e-2 of each difference plus 1e-3 of their largest."""
    from helpers import SMALL, load_npz
    from oracle.model import OracleModel
    from pywrf_b200 import synthetic

    Z = load_npz("thbias_ref64.npz")
    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    st0 = OracleModel(g, inputs, bdy, np.float32).st
    names = tuple(dict.fromkeys(adjoint.RK_STATE + ("u_1", "w_1", "ph_1", "mu_1", "t_1", "v_1")))
    st = {k: _cuda(st0[k]) for k in names}
    data = {k: _cuda(st0[k]) for k in tuple(dict.fromkeys(adjoint.STEP_DATA + adjoint._Microphysics.data))}
    bd = {f: {k: _cuda(v) for k, v in st0["bdy"][f].items()} for f in ("u", "v", "ph", "t", "mu", "qv")}
    bias = torch.zeros_like(st["t"], requires_grad=True)
    sc = dict(epssm=g.epssm, emdiv=g.emdiv, smdiv=g.smdiv, cf1=float(st0["cf1"]), cf2=float(st0["cf2"]),
              cf3=float(st0["cf3"]), cfn=float(st0["cfn"]), cfn1=float(st0["cfn1"]), rdx=g.rdx, rdy=g.rdy)
    mp = lambda s: adjoint.microphysics(s, data, g.dt, g.rdx, g.rdy)  # noqa: E731

    def one(*xs):
        n = int(round(float(xs[-1].item())))
        s = adjoint.step(dict(zip(names, xs[:-1])), data, bd, g.dt * n, dt=g.dt, soundsteps=g.soundsteps,
                         microphysics=mp, theta_bias=bias, **sc)
        return tuple(s[k] for k in names) + (xs[-1] + 1,)

    outs = adjoint.rollout(one, tuple(st[k] for k in names) + (torch.tensor(1.0, device="cuda"),), 2, every=1)
    out = dict(zip(names, outs))
    R = (slice(0, 10), slice(g.jds, g.jde - 1), slice(g.ids, g.ide - 1))
    tt = torch.tensor(Z["target_t"], device="cuda")
    tq = torch.tensor(Z["target_qv"], device="cuda")
    loss = ((out["t"][R].double() - tt) ** 2).mean() + ((out["moist"][1][R].double() - tq) ** 2).mean()
    l0 = float(loss.detach())
    assert abs(l0 - float(Z["loss0"])) <= 1e-4 * abs(float(Z["loss0"])), (l0, float(Z["loss0"]))
    loss.backward()
    gr = bias.grad.double().cpu().numpy()
    got = np.array([gr[k, j, i] for k, j, i in Z["points"]])
    fd = np.asarray(Z["fd"], np.float64)
    tol = 1e-2 * np.abs(fd) + 1e-3 * np.abs(fd).max()
    print("theta-bias gradient: loss %.9g (reference %.9g); max |adjoint - reference| / max |reference| = %.3g"
          % (l0, float(Z["loss0"]), float(np.abs(got - fd).max() / np.abs(fd).max())))
    assert np.all(np.abs(got - fd) <= tol), list(zip(got, fd))
