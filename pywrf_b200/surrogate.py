"""Learned stand-in for WSM6: a per-column network trained and evaluated on
the tensor cores (include/pywrf_b200.h, ``wrf_mlp_*`` / ``wrf_gemm_bf16``).

* :class:`MlpNet` -- the weights (fp32 masters with Adam moments, bf16 copies
  and transposed bf16 copies) and the standardisation table.
* :class:`Harvester` -- runs plain ARW steps and records, at each step's
  microphysics call, the columns' inputs and the increments WSM6 produced.
* :class:`Trainer` -- minibatch training: the forward, loss, input-gradient,
  weight-gradient and Adam steps are all library kernels; PyTorch only owns the
  buffers.
* :class:`SurrogateIntegrator` -- steps with the network in place of WSM6
  (``wrf_rk3_step_mlp``: gate + WSM6 fallback on rejected columns), with a
  plain WSM6 step every ``judge_every`` steps.

The reference (pywrf) has no learned part; the network replaces its call of
``wsm6`` (pywrf/solver.py:1714-1766, pywrf/wrf_physics.py:137-1214).
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _native as N
from .solver import Integrator, _stream_handle
from .state import DeviceState

LAYERS = N.WRF_MLP_LAYERS


def _p(t: torch.Tensor | None) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def init_device(device: torch.device | str) -> None:
    """One-time set-up of the network kernels on a device (before any capture)."""
    with torch.cuda.device(torch.device(device)):
        N.check(N.lib().wrf_mlp_init(), "wrf_mlp_init")


def layout(state: DeviceState) -> dict[str, int]:
    """Column layout of the network rows for the state's grid."""
    out = (ctypes.c_int * 8)()
    N.check(N.lib().wrf_mlp_layout(ctypes.byref(state.cgrid), out), "wrf_mlp_layout")
    return dict(zip(("km", "ncx", "ncy", "ncols", "nfeat", "d0", "nout", "d4"), list(out)))


class MlpNet:
    """Weights of the network d0 -> hidden x 3 -> d4 on one CUDA device."""

    def __init__(self, lay: dict[str, int], hidden: int = 512, device: str | torch.device = "cuda", seed: int = 0):
        if hidden % 64:
            raise ValueError("hidden width must be a multiple of 64")
        self.layout = dict(lay)
        self.device = torch.device(device)
        init_device(self.device)
        self.dims = [lay["d0"], hidden, hidden, hidden, lay["d4"]]
        gen = torch.Generator().manual_seed(seed)
        self.w32, self.b32 = [], []
        for i in range(LAYERS):
            fan_in = self.dims[i]
            scale = math.sqrt(2.0 / fan_in) if i < LAYERS - 1 else math.sqrt(1.0 / fan_in)
            self.w32.append((torch.randn(self.dims[i + 1], fan_in, generator=gen) * scale).to(self.device))
            self.b32.append(torch.zeros(self.dims[i + 1], device=self.device))
        self.wb = [w.to(torch.bfloat16).contiguous() for w in self.w32]
        self.wtb = [w.t().contiguous().to(torch.bfloat16) for w in self.w32]
        self.mw = [torch.zeros_like(w) for w in self.w32]
        self.vw = [torch.zeros_like(w) for w in self.w32]
        self.mb = [torch.zeros_like(b) for b in self.b32]
        self.vb = [torch.zeros_like(b) for b in self.b32]
        d0, d4 = lay["d0"], lay["d4"]
        self.norm = torch.zeros(2 * d0 + 2 * d4, device=self.device)
        self.norm[d0:2 * d0] = 1.0
        self.norm[2 * d0 + d4:] = 1.0
        self.adam_step = 0
        self.precip_weight = 4.0

    def fit_normalisation(self, raw_in: torch.Tensor, raw_out: torch.Tensor) -> None:
        """Standardisation from harvested raw rows (dataset preparation):
        inputs per feature (hydrometeors as log(max(q,0) + 1e-12)), outputs per
        increment; features and outputs that never vary get 1/std = 0 / std = 0
        (the network's output there is pinned to the mean)."""
        L = self.layout
        km, nfeat, nout, d0, d4 = L["km"], L["nfeat"], L["nout"], L["d0"], L["d4"]
        f = raw_in[:, :nfeat].double()
        f[:, 3 * km:] = torch.log(f[:, 3 * km:].clamp_min(0) + 1e-12)
        mean, std = f.mean(0), f.std(0)
        rstd = torch.where(std > 1e-12 * mean.abs().clamp_min(1e-30), 1.0 / std.clamp_min(1e-300), 0.0)
        o = raw_out.double()
        omean, ostd = o.mean(0), o.std(0)
        # per variable, no output's scale below 1 % of the variable's largest
        # (levels that barely changed in the harvest would otherwise dominate
        # the loss); outputs that never changed stay pinned (std 0)
        for v in range(7):
            blk = ostd[v * km:(v + 1) * km]
            blk.copy_(torch.where(blk > 0, blk.clamp_min(0.01 * float(blk.max())), blk))
        ostd = torch.where(ostd > 0, ostd, 0.0)
        # the three precipitation outputs (one value per column against 40
        # per species) weigh precip_weight^2 more in the standardised loss
        ostd[7 * km:] = ostd[7 * km:] / self.precip_weight
        n = torch.zeros(2 * d0 + 2 * d4, dtype=torch.float64, device=self.device)
        n[:nfeat] = mean
        n[d0:d0 + nfeat] = rstd
        n[2 * d0:2 * d0 + nout] = omean
        n[2 * d0 + d4:2 * d0 + d4 + nout] = ostd
        self.norm.copy_(n.float())

    def cstruct(self, tol_neg: float = 1.0e-6, tol_sat: float = 0.05) -> N.WrfMlpNetC:
        c = N.WrfMlpNetC()
        for i in range(LAYERS + 1):
            c.dims[i] = self.dims[i]
        for i in range(LAYERS):
            c.w[i] = self.wb[i].data_ptr()
            c.b[i] = self.b32[i].data_ptr()
        c.norm = self.norm.data_ptr()
        c.tol_neg = tol_neg
        c.tol_sat = tol_sat
        return c

    def state_dict(self) -> dict[str, torch.Tensor]:
        d = {f"w{i}": w for i, w in enumerate(self.w32)}
        d.update({f"b{i}": b for i, b in enumerate(self.b32)})
        d["norm"] = self.norm
        return d

    def load_state_dict(self, d: dict[str, torch.Tensor]) -> None:
        for i in range(LAYERS):
            self.w32[i].copy_(d[f"w{i}"])
            self.b32[i].copy_(d[f"b{i}"])
            self.wb[i].copy_(self.w32[i].to(torch.bfloat16))
            self.wtb[i].copy_(self.w32[i].t().to(torch.bfloat16))
        self.norm.copy_(d["norm"])


class Harvester:
    """Records (columns before, WSM6 increments) pairs from plain steps."""

    def __init__(self, integrator: Integrator):
        self.it = integrator
        self.state = integrator.state
        self.layout = layout(self.state)
        L = self.layout
        dev = self.state.device
        self.raw_in = torch.empty(L["ncols"], 10 * L["km"], device=dev)
        self.raw_out = torch.empty(L["ncols"], L["nout"], device=dev)
        self.lib = N.lib()

    def step(self) -> tuple[torch.Tensor, torch.Tensor]:
        """One plain step; returns the raw rows (inputs, increments) of all columns."""
        st = self.state

        def probe(name: str) -> None:
            if name == "s3.moist":
                N.check(self.lib.wrf_mlp_features(ctypes.byref(st.cgrid), st.ptr, None, None, _p(self.raw_in),
                                                  _stream_handle(None)), "wrf_mlp_features")
            elif name == "mp":
                N.check(self.lib.wrf_mlp_targets(ctypes.byref(st.cgrid), st.ptr, _p(self.raw_in), _p(self.raw_out),
                                                 _stream_handle(None)), "wrf_mlp_targets")
        self.it.step(probe)
        return self.raw_in, self.raw_out


def select_columns(raw_in: torch.Tensor, raw_out: torch.Tensor, km: int, keep_quiet: float,
                   gen: torch.Generator) -> torch.Tensor:
    """Indices of the columns kept for training: every column with
    condensate or a nonzero microphysics increment, and a random fraction
    ``keep_quiet`` of the others (clear, unchanged columns)."""
    cond = raw_in[:, 4 * km:9 * km].abs().amax(1) > 0
    act = raw_out.abs().amax(1) > 0
    busy = cond | act
    r = torch.rand(raw_in.shape[0], generator=gen).to(raw_in.device)
    return torch.nonzero(busy | (r < keep_quiet)).flatten()


class Trainer:
    """Minibatch Adam training of :class:`MlpNet` on the tensor-core kernels."""

    def __init__(self, net: MlpNet, batch: int = 8192, splits: int = 8, lr: float = 1e-3, wd: float = 0.0):
        if batch % 128:
            raise ValueError("batch must be a multiple of 128")
        self.net, self.batch, self.lr, self.wd = net, batch, lr, wd
        self.lib = N.lib()
        d, B, dev = net.dims, batch, net.device
        h = d[1]
        bf = torch.bfloat16
        self.xt = torch.empty(d[0], B, dtype=bf, device=dev)
        self.z = [torch.empty(B, d[i + 1], dtype=bf, device=dev) for i in range(LAYERS - 1)]
        self.h = [torch.empty(B, d[i + 1], dtype=bf, device=dev) for i in range(LAYERS - 1)]
        self.ht = [torch.empty(d[i + 1], B, dtype=bf, device=dev) for i in range(LAYERS - 1)]
        self.y = torch.empty(B, d[4], device=dev)
        self.dy = torch.empty(B, d[4], dtype=bf, device=dev)
        self.dyt = torch.empty(d[4], B, dtype=bf, device=dev)
        self.dz = [torch.empty(B, h, dtype=bf, device=dev) for _ in range(2)]
        self.dzt = [torch.empty(h, B, dtype=bf, device=dev) for _ in range(2)]
        self.splits = [self.lib.wrf_gemm_splits(B, splits) for _ in range(LAYERS)]
        self.gw = [torch.empty(self.splits[i], d[i + 1], d[i], device=dev) for i in range(LAYERS)]
        self.gb = [torch.empty(d[i + 1], device=dev) for i in range(LAYERS)]
        self.loss = torch.zeros(1, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)

    def _gemm(self, a, b, m, n, k, epi, out, ldo, bias=None, aux=None, out_z=None, out_t=None, ldt=0, splits=1,
              split_stride=0):
        rc = self.lib.wrf_gemm_bf16(_p(a), _p(b), m, n, k, splits, epi, _p(bias), _p(aux), _p(out), ldo,
                                    split_stride, _p(out_z), _p(out_t), ldt, _p(self.err), _stream_handle(None))
        N.check(rc, "wrf_gemm_bf16")

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """Training forward of a full batch x [batch, d0] (bf16); keeps the
        pre-activations and transposed activations for the backward pass."""
        net, B, d = self.net, self.batch, self.net.dims
        N.check(self.lib.wrf_transpose_bf16(_p(x), B, d[0], _p(self.xt), _stream_handle(None)), "transpose")
        a = x
        for i in range(LAYERS - 1):
            self._gemm(a, net.wb[i], B, d[i + 1], d[i], N.EPI_BIAS_GELU, self.h[i], d[i + 1], bias=net.b32[i],
                       out_z=self.z[i], out_t=self.ht[i], ldt=B)
            a = self.h[i]
        self._gemm(a, net.wb[3], B, d[4], d[3], N.EPI_F32, self.y, d[4], bias=net.b32[3])
        return self.y

    def backward(self, t: torch.Tensor) -> None:
        """Gradients of the mean squared error against standardised targets
        t [batch, d4] into self.gw (split partial sums) and self.gb."""
        net, B, d = self.net, self.batch, self.net.dims
        nvalid = net.layout["nout"]
        s = _stream_handle(None)
        N.check(self.lib.wrf_mse_grad(_p(self.y), _p(t), B, d[4], nvalid, 2.0 / (B * nvalid), _p(self.dy),
                                      _p(self.dyt), _p(self.loss), s), "mse_grad")
        g_t, g = self.dyt, self.dy
        for i in range(LAYERS - 1, -1, -1):
            inp_t = self.ht[i - 1] if i > 0 else self.xt
            self._gemm(g_t, inp_t, d[i + 1], d[i], B, N.EPI_F32, self.gw[i], d[i], splits=self.splits[i],
                       split_stride=d[i + 1] * d[i])
            N.check(self.lib.wrf_rowsum_bf16(_p(g_t), d[i + 1], B, _p(self.gb[i]), s), "rowsum")
            if i > 0:
                nxt, nxt_t = self.dz[i % 2], self.dzt[i % 2]
                self._gemm(g, net.wtb[i], B, d[i], d[i + 1], N.EPI_GELU_BWD, nxt, d[i], aux=self.z[i - 1],
                           out_t=nxt_t, ldt=B)
                g, g_t = nxt, nxt_t

    def adam(self, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8) -> None:
        net = self.net
        net.adam_step += 1
        s = _stream_handle(None)
        for i in range(LAYERS):
            r, c = net.dims[i + 1], net.dims[i]
            N.check(self.lib.wrf_adam(_p(net.w32[i]), _p(self.gw[i]), self.splits[i], r * c, _p(net.mw[i]),
                                      _p(net.vw[i]), r, c, _p(net.wb[i]), _p(net.wtb[i]), self.lr, b1, b2, eps,
                                      self.wd, net.adam_step, s), "adam")
            N.check(self.lib.wrf_adam(_p(net.b32[i]), _p(self.gb[i]), 1, r, _p(net.mb[i]), _p(net.vb[i]), 1, r,
                                      None, None, self.lr, b1, b2, eps, 0.0, net.adam_step, s), "adam")

    def step(self, x: torch.Tensor, t: torch.Tensor) -> None:
        self.forward(x)
        self.backward(t)
        self.adam()

    def fit(self, x: torch.Tensor, t: torch.Tensor, epochs: int, seed: int = 0, lr_end: float | None = None) -> list[float]:
        """Epochs over the rows of x [n, d0] (bf16) / t [n, d4] (fp32) in
        shuffled full batches; returns the mean loss per epoch."""
        n = x.shape[0] - x.shape[0] % self.batch
        if n == 0:
            raise ValueError("fewer rows than one batch")
        gen = torch.Generator().manual_seed(seed)
        nb = n // self.batch
        lr0 = self.lr
        losses = []
        for ep in range(epochs):
            if lr_end is not None and epochs > 1:
                self.lr = lr0 * (lr_end / lr0) ** (ep / (epochs - 1))
            perm = torch.randperm(x.shape[0], generator=gen)[:n].to(x.device)
            self.loss.zero_()
            for bi in range(nb):
                idx = perm[bi * self.batch:(bi + 1) * self.batch]
                self.step(x.index_select(0, idx), t.index_select(0, idx))
            losses.append(float(self.loss) / (n * self.net.layout["nout"]))
        self.lr = lr0
        if int(self.err):
            raise RuntimeError("a tensor-core kernel's bounded wait ran out during training")
        return losses


class SurrogateIntegrator(Integrator):
    """ARW steps with the network in place of WSM6; every ``judge_every``-th
    step (and every column the gate rejects) runs plain WSM6."""

    def __init__(self, state: DeviceState, net: MlpNet, judge_every: int = 10, tol_neg: float = 1.0e-6,
                 tol_sat: float = 0.05):
        super().__init__(state)
        self.net = net
        self.judge_every = judge_every
        L = layout(state)
        if L["d0"] != net.dims[0] or L["d4"] != net.dims[4]:
            raise ValueError("the network's widths do not match this grid")
        dev = state.device
        cap = L["ncols"]
        self.x = torch.empty(cap, net.dims[0], dtype=torch.bfloat16, device=dev)
        self.hbuf = [torch.empty(cap, max(net.dims[1:4]), dtype=torch.bfloat16, device=dev) for _ in range(2)]
        self.y = torch.empty(cap, net.dims[4], device=dev)
        self.list = torch.zeros(16 + cap, dtype=torch.int32, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.colstat = torch.zeros(cap, dtype=torch.uint8, device=dev)
        self.work = N.WrfMlpWorkC()
        self.work.capacity = cap
        self.work.x = self.x.data_ptr()
        self.work.h[0] = self.hbuf[0].data_ptr()
        self.work.h[1] = self.hbuf[1].data_ptr()
        self.work.y = self.y.data_ptr()
        self.work.list = self.list.data_ptr()
        self.work.err = self.err.data_ptr()
        self.work.colstat = self.colstat.data_ptr()
        self.netc = net.cstruct(tol_neg, tol_sat)
        self._mlp_graph: torch.cuda.CUDAGraph | None = None
        self.nstep = 0
        self.rejected_total = 0

    def step_mlp(self, probe=None, stream: torch.cuda.Stream | None = None) -> None:
        cb = N.PROBE_FN(lambda name, user: probe(name.decode())) if probe else N.PROBE_FN()
        with torch.cuda.device(self.state.device):
            rc = self.lib.wrf_rk3_step_mlp(ctypes.byref(self.state.cgrid), self.state.ptr, ctypes.byref(self.netc),
                                           ctypes.byref(self.work), _stream_handle(stream), cb, None)
        N.check(rc, "wrf_rk3_step_mlp")

    def capture_mlp(self) -> None:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.device(self.state.device):
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    rc = self.lib.wrf_rk3_step_mlp(ctypes.byref(self.state.cgrid), self.state.ptr,
                                                   ctypes.byref(self.netc), ctypes.byref(self.work),
                                                   _stream_handle(s), N.PROBE_FN(), None)
            torch.cuda.current_stream().wait_stream(s)
        N.check(rc, "wrf_rk3_step_mlp (capture)")
        self._mlp_graph = g

    def judged(self, n: int) -> bool:
        return self.judge_every > 0 and n % self.judge_every == self.judge_every - 1

    def run(self, nsteps: int, graph: bool = True, count_rejected: bool = False) -> None:
        for _ in range(nsteps):
            if self.judged(self.nstep):
                if graph:
                    self.replay()
                else:
                    self.step()
            else:
                if graph:
                    if self._mlp_graph is None:
                        self.capture_mlp()
                    self._mlp_graph.replay()
                else:
                    self.step_mlp()
                if count_rejected:
                    self.rejected_total += int(self.list[0])
            self.nstep += 1

    def rejected(self) -> int:
        """Columns the gate rejected in the last surrogate step."""
        return int(self.list[0])

    def column_stats(self) -> dict[str, int]:
        """Counters of the last surrogate step: rejected columns, quiet
        columns (zero increments without the network), and rejections by
        reason (a column can have several)."""
        v = self.list[:5].tolist()
        return {"rejected": v[0], "quiet": v[1], "rejected_positivity": v[2], "rejected_supersaturation": v[3],
                "rejected_nonfinite": v[4], "columns": int(self.colstat.numel())}


def harvest(seeds, nsteps: int, spec_for, per_step: int = 5000, busy_share: float = 0.8, device: str = "cuda",
            gen_seed: int = 0) -> tuple[torch.Tensor, torch.Tensor, dict[str, int]]:
    """Raw (inputs, increments) rows from plain integrations of the synthetic
    workloads ``spec_for(seed)``, ``nsteps`` steps each.  Each step keeps up
    to ``per_step`` columns: up to ``busy_share`` of them among the columns
    with condensate or a microphysics increment, the rest among the others."""
    from . import synthetic
    gen = torch.Generator().manual_seed(gen_seed)
    rows_in, rows_out = [], []
    lay = None
    for seed in seeds:
        spec = spec_for(seed)
        g = synthetic.grid_for(spec)
        inputs, bdy = synthetic.build(spec)
        st = DeviceState.from_inputs(g, inputs, bdy, device=device)
        hv = Harvester(Integrator(st))
        lay = hv.layout
        km = lay["km"]
        for _ in range(nsteps):
            ri, ro = hv.step()
            busy = (ri[:, 4 * km:9 * km].abs().amax(1) > 0) | (ro.abs().amax(1) > 0)
            ib, iq = torch.nonzero(busy).flatten(), torch.nonzero(~busy).flatten()
            nb = min(ib.numel(), int(busy_share * per_step))
            nq = min(iq.numel(), per_step - nb)
            pick = torch.cat([ib[torch.randperm(ib.numel(), generator=gen)[:nb].to(ib.device)],
                              iq[torch.randperm(iq.numel(), generator=gen)[:nq].to(iq.device)]])
            rows_in.append(ri.index_select(0, pick))
            rows_out.append(ro.index_select(0, pick))
        del st, hv
    return torch.cat(rows_in), torch.cat(rows_out), lay


def standardise(net: MlpNet, cgrid, raw_in: torch.Tensor, raw_out: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """bf16 network inputs and fp32 standardised targets of raw rows (kernel k_mlp_normalize)."""
    lay = net.layout
    n = raw_in.shape[0]
    x = torch.empty(n, lay["d0"], dtype=torch.bfloat16, device=net.device)
    t = torch.empty(n, lay["d4"], device=net.device)
    N.check(N.lib().wrf_mlp_normalize(ctypes.byref(cgrid), _p(net.norm), _p(raw_in), _p(raw_out), n, _p(x), _p(t),
                                      _stream_handle(None)), "wrf_mlp_normalize")
    return x, t


def time_forward(cols: int = 51529, hidden: int = 512, km: int = 40, reps: int = 20, device: str = "cuda") -> dict:
    """CUDA-event time of the network's inference chain (``wrf_mlp_forward``:
    four tcgen05 products, bias + GELU fused) on ``cols`` random rows of a
    randomly initialised network of the 240x240x41 layout."""
    nfeat, nout = 9 * km, 7 * km + 3
    lay = dict(km=km, ncx=0, ncy=0, ncols=cols, nfeat=nfeat, d0=(nfeat + 63) // 64 * 64, nout=nout,
               d4=(nout + 63) // 64 * 64)
    net = MlpNet(lay, hidden=hidden, device=device)
    g = torch.Generator().manual_seed(1)
    x = torch.randn(cols, lay["d0"], generator=g).to(torch.bfloat16).to(device)
    h0 = torch.empty(cols, hidden, dtype=torch.bfloat16, device=device)
    h1 = torch.empty_like(h0)
    y = torch.empty(cols, lay["d4"], device=device)
    err = torch.zeros(1, dtype=torch.int32, device=device)
    c = net.cstruct()
    L = N.lib()

    def run(n):
        for _ in range(n):
            N.check(L.wrf_mlp_forward(ctypes.byref(c), _p(x), cols, _p(h0), _p(h1), _p(y), _p(err),
                                      _stream_handle(None)), "wrf_mlp_forward")
    run(3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    run(reps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    flop = 2 * cols * sum(net.dims[i] * net.dims[i + 1] for i in range(LAYERS))
    if int(err):
        raise RuntimeError("a tensor-core kernel's bounded wait ran out")
    return {"cols": cols, "dims": net.dims, "ms": ms, "tflops": flop / (ms / 1e3) / 1e12}


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="time the network's inference chain on the tensor cores")
    ap.add_argument("--cols", type=int, default=51529)
    ap.add_argument("--hidden", type=int, default=512)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args()
    print(json.dumps(time_forward(a.cols, a.hidden, reps=a.reps)))
