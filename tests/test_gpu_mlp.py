"""The tensor-core network kernels: the tcgen05 GEMM and its epilogues
against float64 products of the same bf16 operands, the training gradients
against the numpy oracle (oracle/mlp.py), and the surrogate microphysics step
(gate, WSM6 fallback, and what a trained network gains over no network)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from helpers import SMALL
from oracle import mlp as OM
from pywrf_b200 import _native as N
from pywrf_b200 import surrogate, synthetic
from pywrf_b200.solver import Integrator
from pywrf_b200.state import DeviceState

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def _gemm(a, b, epi, out, ldo, bias=None, aux=None, out_z=None, out_t=None, ldt=0, splits=1, split_stride=0, err=None):
    L = N.lib()
    m, k = a.shape
    n = b.shape[0]
    rc = L.wrf_gemm_bf16(_p(a), _p(b), m, n, k, splits, epi, _p(bias), _p(aux), _p(out), ldo, split_stride,
                         _p(out_z), _p(out_t), ldt, _p(err), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    N.check(rc, "wrf_gemm_bf16")


@pytest.fixture(scope="module")
def operands():
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    g = torch.Generator().manual_seed(7)
    M, N_, K = 300, 144, 192          # partial M and N tiles
    a = (torch.randn(M, K, generator=g)).to(torch.bfloat16).cuda()
    b = (torch.randn(N_, K, generator=g) * 0.1).to(torch.bfloat16).cuda()
    bias = (torch.randn(N_, generator=g) * 0.1).cuda()
    ref = a.double() @ b.double().t()
    return a, b, bias, ref


def _rel(x, ref):
    x, ref = x.double(), ref.double()
    return float((x - ref).norm() / ref.norm())


def test_gemm_f32_bias(operands):
    a, b, bias, ref = operands
    out = torch.full((a.shape[0], b.shape[0]), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _gemm(a, b, N.EPI_F32, out, b.shape[0], bias=bias, err=err)
    torch.cuda.synchronize()
    assert int(err) == 0
    assert _rel(out, ref + bias.double()) < 1e-6


def test_gemm_bias_gelu_with_preactivation_and_transpose(operands):
    a, b, bias, ref = operands
    M, N_ = a.shape[0], b.shape[0]
    h = torch.empty(M, N_, dtype=torch.bfloat16, device="cuda")
    z = torch.empty_like(h)
    ht = torch.empty(N_, M + 20, dtype=torch.bfloat16, device="cuda")   # ldt > M
    _gemm(a, b, N.EPI_BIAS_GELU, h, N_, bias=bias, out_z=z, out_t=ht, ldt=M + 20)
    torch.cuda.synchronize()
    zr = (ref + bias.double()).cpu().numpy()
    assert _rel(z.cpu(), torch.from_numpy(zr)) < 4e-3
    hr = OM.gelu(zr)
    assert _rel(h.cpu(), torch.from_numpy(hr)) < 4e-3
    assert torch.equal(ht[:, :M].t(), h)


def test_gemm_gelu_backward_and_plain_bf16(operands):
    a, b, bias, ref = operands
    M, N_ = a.shape[0], b.shape[0]
    g = torch.Generator().manual_seed(8)
    aux = torch.randn(M, N_, generator=g).to(torch.bfloat16).cuda()
    out = torch.empty(M, N_, dtype=torch.bfloat16, device="cuda")
    _gemm(a, b, N.EPI_GELU_BWD, out, N_, aux=aux)
    plain = torch.empty_like(out)
    _gemm(a, b, N.EPI_BF16, plain, N_)
    torch.cuda.synchronize()
    want = ref.cpu().numpy() * OM.gelu_grad(aux.double().cpu().numpy())
    assert _rel(out.cpu(), torch.from_numpy(want)) < 4e-3
    assert _rel(plain.cpu(), ref.cpu()) < 4e-3


def test_gemm_split_reduction():
    g = torch.Generator().manual_seed(9)
    M, N_, K = 256, 128, 1024
    a = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    b = torch.randn(N_, K, generator=g).to(torch.bfloat16).cuda()
    splits = N.lib().wrf_gemm_splits(K, 5)
    assert splits >= 2
    part = torch.zeros(splits, M, N_, device="cuda")
    _gemm(a, b, N.EPI_F32, part, N_, splits=5, split_stride=M * N_)
    torch.cuda.synchronize()
    assert _rel(part.sum(0), a.double() @ b.double().t()) < 1e-6


def test_gemm_rejects_bad_shapes(operands):
    a, b, bias, _ = operands
    out = torch.empty(a.shape[0], b.shape[0], device="cuda")
    L = N.lib()
    rc = L.wrf_gemm_bf16(_p(a), _p(b), a.shape[0], b.shape[0], 100, 1, N.EPI_F32, None, None, _p(out), b.shape[0],
                         0, None, None, 0, None, None)
    assert rc == N.WRF_EINVAL and "multiple of 64" in L.wrf_last_error().decode()


def _small_net(seed=0):
    lay = dict(km=8, ncx=0, ncy=0, ncols=0, nfeat=120, d0=128, nout=60, d4=64)
    return surrogate.MlpNet(lay, hidden=128, device="cuda", seed=seed)


def test_training_gradients_match_the_oracle():
    net = _small_net()
    g = torch.Generator().manual_seed(11)
    B = 256
    for i in range(4):  # nonzero biases exercise the bias paths
        net.b32[i].copy_(torch.randn(net.dims[i + 1], generator=g) * 0.1)
    tr = surrogate.Trainer(net, batch=B, splits=2)
    x = torch.randn(B, 128, generator=g).to(torch.bfloat16).cuda()
    t = torch.randn(B, 64, generator=g).cuda()
    t[:, 60:] = 0
    tr.loss.zero_()
    tr.forward(x)
    tr.backward(t)
    torch.cuda.synchronize()
    w = [wb.double().cpu().numpy() for wb in net.wb]
    b = [bb.double().cpu().numpy() for bb in net.b32]
    y, zs, hs = OM.forward(x.double().cpu().numpy(), w, b)
    assert _rel(tr.y.cpu(), torch.from_numpy(y)) < 2e-3
    loss, gw, gb = OM.backward(y, t.double().cpu().numpy(), zs, hs, w, 60)
    assert abs(float(tr.loss) - loss) / loss < 1e-3
    for i in range(4):
        got_w = tr.gw[i].sum(0).double().cpu()
        assert _rel(got_w, torch.from_numpy(gw[i])) < 1e-2, i
        assert _rel(tr.gb[i].cpu(), torch.from_numpy(gb[i])) < 1e-2, i


def test_adam_steps_reduce_the_loss():
    net = _small_net(seed=1)
    g = torch.Generator().manual_seed(12)
    B = 512
    tr = surrogate.Trainer(net, batch=B, splits=2, lr=3e-3)
    x = torch.randn(B, 128, generator=g).to(torch.bfloat16).cuda()
    wt = torch.randn(128, 64, generator=g) * 0.1
    t = (x.float().cpu() @ wt).cuda()
    t[:, 60:] = 0
    losses = []
    for _ in range(60):
        tr.loss.zero_()
        tr.step(x, t)
        losses.append(float(tr.loss))
    assert losses[-1] < 0.2 * losses[0], (losses[0], losses[-1])
    # the bf16 copies track the fp32 masters
    assert torch.equal(net.wb[1], net.w32[1].to(torch.bfloat16))
    assert torch.equal(net.wtb[1], net.w32[1].t().to(torch.bfloat16))


@pytest.fixture(scope="module")
def small_case():
    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    return g, inputs, bdy


def _fields(st):
    return {k: st[k].clone() for k in ("u", "v", "w", "t", "ph", "mu", "p", "al", "moist", "rainnc", "h_diabatic")}


def test_surrogate_with_every_column_rejected_equals_the_plain_step(small_case):
    g, inputs, bdy = small_case
    plain = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    it = Integrator(plain)
    it.step()
    sur = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    net = surrogate.MlpNet(surrogate.layout(sur), hidden=128, device="cuda")
    # tol_neg = -1: every new species value is "below -tol_neg" -> all columns rejected
    si = surrogate.SurrogateIntegrator(sur, net, judge_every=0, tol_neg=-1.0)
    si.step_mlp()
    torch.cuda.synchronize()
    assert si.rejected() == surrogate.layout(sur)["ncols"]
    a, b = _fields(plain), _fields(sur)
    for k in a:
        d = float((a[k] - b[k]).abs().max())
        scale = float(a[k].abs().max()) or 1.0
        assert d <= 1e-6 * scale, (k, d)


def test_quiet_columns_take_exactly_what_wsm6_does(small_case):
    """Columns without condensate and below saturation bypass the network;
    WSM6 leaves them unchanged too, so after one step they equal the plain
    step's columns (theta to one rounding of t / pii - th).  The moist
    synthetic state is supersaturated over ice near its cold top in every
    column, so the case is made dry (no vapour, no cloud, dry boundaries)."""
    g, inputs, bdy = small_case
    inputs, bdy = dict(inputs), dict(bdy)
    for key in ("QVAPOR", "QCLOUD"):
        inputs[key] = np.zeros_like(np.asarray(inputs[key]))
    for key in [k for k in bdy if k.startswith("QVAPOR_")]:
        bdy[key] = np.zeros_like(np.asarray(bdy[key]))
    plain = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    Integrator(plain).step()
    sur = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    net = surrogate.MlpNet(surrogate.layout(sur), hidden=128, device="cuda", seed=5)
    si = surrogate.SurrogateIntegrator(sur, net, judge_every=0, tol_neg=1e3, tol_sat=1e3)   # gate open
    si.step_mlp()
    torch.cuda.synchronize()
    lay = surrogate.layout(sur)
    stat = si.colstat.view(lay["ncy"], lay["ncx"])
    quiet = stat == 1
    assert int(quiet.sum()) == lay["ncols"]
    assert si.column_stats()["quiet"] == lay["ncols"] and si.rejected() == 0
    js, is_ = g.jds + 1, g.ids + 1
    sl = (slice(js, js + lay["ncy"]), slice(is_, is_ + lay["ncx"]))
    km = lay["km"]
    for k, base in (("t", None), ("p", "pb"), ("al", "alb")):
        a, b = plain[k][:km][:, sl[0], sl[1]], sur[k][:km][:, sl[0], sl[1]]
        full = a + plain[base][:km][:, sl[0], sl[1]] if base else a + 300.0
        d = float((a - b).abs()[:, quiet].max())
        assert d <= 1e-6 * float(full.abs().max()), (k, d)   # p, al: a few roundings of the full value
    for m in range(1, 7):
        a, b = plain["moist"][m, :km][:, sl[0], sl[1]], sur["moist"][m, :km][:, sl[0], sl[1]]
        assert torch.equal(a[:, quiet], b[:, quiet]), m
    for k in ("rainnc", "rainncv", "sr"):
        assert torch.equal(plain[k][sl][quiet], sur[k][sl][quiet]), k


def test_surrogate_step_runs_in_a_graph_and_keeps_the_state_finite(small_case):
    g, inputs, bdy = small_case
    st = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    net = surrogate.MlpNet(surrogate.layout(st), hidden=128, device="cuda", seed=3)
    for w in net.w32:
        w.mul_(0.0)
    net.load_state_dict(net.state_dict())   # zero network: zero increments
    si = surrogate.SurrogateIntegrator(st, net, judge_every=3)
    si.run(4, graph=True)
    torch.cuda.synchronize()
    assert si.status()["nan_p"] == 0
    for k, v in _fields(st).items():
        assert torch.isfinite(v).all(), k
    assert int(si.err) == 0


def test_trained_network_beats_no_network_on_held_out_columns():
    """Harvest WSM6 increments from 12 steps of a 64x64x41 run, train on a
    random 80 % of the (step, column) rows and compare, on the other 20 %, the
    network's error with the error of leaving the microphysics out (zero
    increments), both in standardised units."""
    spec = synthetic.spec_for_config(0, seed=0)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    st = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    hv = surrogate.Harvester(Integrator(st))
    lay = hv.layout
    rows_in, rows_out = [], []
    for _ in range(12):
        ri, ro = hv.step()
        rows_in.append(ri.clone())
        rows_out.append(ro.clone())
    all_in, all_out = torch.cat(rows_in), torch.cat(rows_out)
    perm = torch.randperm(all_in.shape[0], generator=torch.Generator().manual_seed(5)).cuda()
    ntr = int(0.8 * all_in.shape[0])
    train_in, train_out = all_in[perm[:ntr]], all_out[perm[:ntr]]
    test_in, test_out = all_in[perm[ntr:]], all_out[perm[ntr:]]
    net = surrogate.MlpNet(lay, hidden=256, device="cuda", seed=0)
    net.fit_normalisation(train_in, train_out)
    L = N.lib()

    def prep(ri, ro):
        x = torch.empty(ri.shape[0], lay["d0"], dtype=torch.bfloat16, device="cuda")
        t = torch.empty(ri.shape[0], lay["d4"], device="cuda")
        N.check(L.wrf_mlp_normalize(ctypes.byref(st.cgrid), _p(net.norm), _p(ri), _p(ro), ri.shape[0], _p(x), _p(t),
                                    None), "normalize")
        return x, t

    xtr, ttr = prep(train_in, train_out)
    xte, tte = prep(test_in, test_out)
    tr = surrogate.Trainer(net, batch=1024, splits=2, lr=2e-3)
    losses = tr.fit(xtr, ttr, epochs=40, lr_end=1e-4)
    assert losses[-1] < losses[0]
    # held-out error (standardised units) of the network and of zero increments
    ev = surrogate.Trainer(net, batch=1024, splits=1)
    n = xte.shape[0] - xte.shape[0] % 1024
    se_net, se_zero = 0.0, 0.0
    zero_std = -net.norm[2 * lay["d0"]:2 * lay["d0"] + lay["d4"]] / net.norm[2 * lay["d0"] + lay["d4"]:].clamp_min(1e-30)
    zero_std = torch.where(net.norm[2 * lay["d0"] + lay["d4"]:] > 0, zero_std, torch.zeros_like(zero_std))
    nout = lay["nout"]
    for s0 in range(0, n, 1024):
        y = ev.forward(xte[s0:s0 + 1024])
        t = tte[s0:s0 + 1024]
        se_net += float(((y - t)[:, :nout] ** 2).sum())
        se_zero += float(((zero_std[None, :] - t)[:, :nout] ** 2).sum())
    print(f"held-out standardised squared error: network {se_net:.4g}, no network {se_zero:.4g}")
    assert se_net < 0.5 * se_zero, (se_net, se_zero)
