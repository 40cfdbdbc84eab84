"""Drop-in ``WrfSolver``: the reference's time loop on the sm_100a kernels.

``WrfSolver.solve`` keeps the reference's contract (pywrf/solver.py:32-1921):
it obtains the input / boundary / reference datasets from
``self._load_datasets()`` (override it to feed other data, exactly as with
the reference), runs ``nsteps`` ARW time steps and returns the final
``{"u", "v", "w", "t", "ph", "mu", "moist"}`` tensors in the reference's
halo-frame layout.  The step itself is :class:`Integrator.step`, one call of
``wrf_rk3_step`` (include/pywrf_b200.h), optionally replayed from a CUDA
graph; nothing of it runs on the CPU.  Every ``bdy_interval`` steps the
boundary arrays are reloaded from the next record of the boundary file, as
the reference's loop does (:func:`bdy_schedule`); the boundary time within
an interval is kept on the device.
"""
from __future__ import annotations

import ctypes
import os
from typing import Callable, Mapping

import numpy as np
import torch

from . import _native as N
from .config import Grid
from .state import DeviceState, grid_from_inputs, ingest_bdy

# run parameters of the reference configuration (pywrf/config_params.py:41-72)
DEFAULTS = dict(dx=9000.0, dy=9000.0, dt=60.0, p_top=1000.0, soundsteps=4, bdy_interval=360, nsteps=720)


def _stream_handle(stream: torch.cuda.Stream | None) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


class Integrator:
    """Advances one :class:`DeviceState` by whole ARW time steps."""

    def __init__(self, state: DeviceState):
        if state.device.type != "cuda":
            raise ValueError("the ARW step runs on a CUDA device only")
        self.state = state
        self.lib = N.lib()
        self._graph: torch.cuda.CUDAGraph | None = None
        self._graph_stream: torch.cuda.Stream | None = None

    def step(self, probe: Callable[[str], None] | None = None, stream: torch.cuda.Stream | None = None) -> None:
        """Enqueue one time step on ``stream`` (default: the current stream).
        ``probe(phase)`` is called after each phase, with the stream not yet
        synchronised."""
        cb = N.PROBE_FN(lambda name, user: probe(name.decode())) if probe else N.PROBE_FN()
        with torch.cuda.device(self.state.device):
            rc = self.lib.wrf_rk3_step(ctypes.byref(self.state.cgrid), self.state.ptr, _stream_handle(stream), cb, None)
        N.check(rc, "wrf_rk3_step")

    def step_phases(self, stream: torch.cuda.Stream | None = None) -> None:
        """One time step through the phase entry points (``wrf_step_begin`` ..
        ``wrf_step_end``), in the order of the reference's RK3 loop
        (pywrf/solver.py:709-1910); enqueues the same kernels as :meth:`step`."""
        L, g, sp = self.lib, ctypes.byref(self.state.cgrid), self.state.ptr
        with torch.cuda.device(self.state.device):
            h = _stream_handle(stream)
            N.check(L.wrf_step_begin(g, sp, h), "wrf_step_begin")
            soundsteps = self.state.cgrid.soundsteps
            for rk in (1, 2, 3):
                N.check(L.wrf_rk_prep(g, sp, rk, h), "wrf_rk_prep")
                if rk == 1:
                    N.check(L.wrf_diff_stage1(g, sp, h), "wrf_diff_stage1")
                N.check(L.wrf_tend_stage(g, sp, rk, h), "wrf_tend_stage")
                N.check(L.wrf_acoustic_prep(g, sp, rk, h), "wrf_acoustic_prep")
                nsub = 1 if rk == 1 else (soundsteps // 2 if rk == 2 else soundsteps)
                for it in range(1, nsub + 1):
                    N.check(L.wrf_acoustic_substep(g, sp, rk, it, h), "wrf_acoustic_substep")
                N.check(L.wrf_acoustic_finish(g, sp, rk, h), "wrf_acoustic_finish")
                N.check(L.wrf_moist_stage(g, sp, rk, h), "wrf_moist_stage")
            N.check(L.wrf_microphysics(g, sp, h), "wrf_microphysics")
            N.check(L.wrf_step_end(g, sp, h), "wrf_step_end")

    def capture(self) -> None:
        """Record one step into a CUDA graph (the step number lives on the
        device, so the same graph serves every step)."""
        g = torch.cuda.CUDAGraph()
        with torch.cuda.device(self.state.device):
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    rc = self.lib.wrf_rk3_step(ctypes.byref(self.state.cgrid), self.state.ptr,
                                               _stream_handle(s), N.PROBE_FN(), None)
            torch.cuda.current_stream().wait_stream(s)
        N.check(rc, "wrf_rk3_step (capture)")
        self._graph, self._graph_stream = g, s

    def replay(self) -> None:
        if self._graph is None:
            self.capture()
        self._graph.replay()

    def run(self, nsteps: int, graph: bool = True) -> None:
        for _ in range(nsteps):
            if graph:
                self.replay()
            else:
                self.step()

    def run_host(self, host: Mapping[str, torch.Tensor], nsteps: int, chunk_bytes: int = 16 << 20) -> None:
        """``nsteps`` steps for a caller that keeps fields of the state in
        pinned host memory (``host``: name -> pinned tensor of the field's
        shape): every step copies them into the device state, runs the
        step (graph replay) and copies them back, so that after the call
        ``host`` holds the state after ``nsteps`` steps.  The copies run on
        two side streams in chunks of about ``chunk_bytes`` (slices along
        the first dimension): a chunk's copy back to the host and the next
        step's copy of it to the device follow each other while the other
        chunks are still in flight, so the two directions of the link
        overlap.  Returns with the current stream ordered after the last
        copy back."""
        st = self.state
        pieces = []
        for k, h in host.items():
            d = st[k]
            if h.shape != d.shape or h.dtype != d.dtype or h.device.type != "cpu" or not h.is_pinned():
                raise ValueError(f"run_host: {k} must be a pinned host tensor shaped like the field")
            row = d[0].numel() * d.element_size() if d.dim() > 1 else d.numel() * d.element_size()
            rows = max(1, chunk_bytes // max(1, row)) if d.dim() > 1 else d.shape[0]
            for a in range(0, d.shape[0], rows):
                pieces.append((d[a:a + rows], h[a:a + rows]))
        with torch.cuda.device(st.device):
            main = torch.cuda.current_stream()
            h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream()
            h2d.wait_stream(main)
            with torch.cuda.stream(h2d):
                for dv, hv in pieces:
                    dv.copy_(hv, non_blocking=True)
            for n in range(nsteps):
                main.wait_stream(h2d)
                self.replay()
                d2h.wait_stream(main)
                back = []
                for dv, hv in pieces:
                    with torch.cuda.stream(d2h):
                        hv.copy_(dv, non_blocking=True)
                    e = torch.cuda.Event()
                    e.record(d2h)
                    back.append(e)
                if n + 1 < nsteps:
                    for (dv, hv), e in zip(pieces, back):
                        h2d.wait_event(e)
                        with torch.cuda.stream(h2d):
                            dv.copy_(hv, non_blocking=True)
            main.wait_stream(d2h)

    def status(self) -> dict[str, int]:
        out = (ctypes.c_int * 16)()
        with torch.cuda.device(self.state.device):
            torch.cuda.current_stream().synchronize()
            rc = self.lib.wrf_status_read(self.state.ptr, _stream_handle(None), out)
        N.check(rc, "wrf_status_read")
        return {"nan_p": out[N.WRF_ST_NAN_P], "step": out[N.WRF_ST_STEP], "wait_timeouts": out[N.WRF_ST_WAIT]}


def bdy_schedule(nsteps: int, bdy_interval: int) -> list[tuple[int | None, int]]:
    """The lateral-boundary records the reference's time loop loads, as
    segments ``(record, steps)``: before step t with ``t % bdy_interval == 1``
    the reference reloads every boundary array from record ``t //
    bdy_interval`` of the boundary file (pywrf/solver.py:457-703); the first
    segment's record (0) is the one the state was built with (None: nothing
    to load)."""
    if nsteps < 0 or bdy_interval < 1:
        raise ValueError("nsteps >= 0 and bdy_interval >= 1 are required")

    def reload_at(t: int) -> bool:
        return t > 1 and bdy_interval > 1 and t % bdy_interval == 1

    segs: list[tuple[int | None, int]] = []
    t = 1
    while t <= nsteps:
        end = t
        while end < nsteps and not reload_at(end + 1):
            end += 1
        segs.append((t // bdy_interval if reload_at(t) else None, end - t + 1))
        t = end + 1
    return segs


def run_with_boundary_records(it, g, bdy, nsteps: int, graph: bool = True) -> None:
    """Advance ``it`` (an :class:`Integrator`) by ``nsteps`` steps, loading
    the boundary record of each segment of :func:`bdy_schedule` into the
    state's boundary arrays in place (same storage, so a captured graph
    stays valid) before the segment's steps."""
    for rec, n in bdy_schedule(nsteps, g.bdy_interval):
        if rec is not None:
            it.state.load(ingest_bdy(g, bdy, rec))
        it.run(n, graph=graph)


class WrfSolver:
    """Orchestrate one WRF run on the GPU (same call pattern as the reference:
    construct, then :meth:`solve`)."""

    def __init__(self, nsteps: int | None = None, device: str | torch.device | None = None, graph: bool = True,
                 **params):
        p = dict(DEFAULTS)
        unknown = set(params) - set(p)
        if unknown:
            raise TypeError(f"unknown parameters {sorted(unknown)}")
        p.update(params)
        if nsteps is not None:
            p["nsteps"] = int(nsteps)
        self.params = p
        self.nsteps = p["nsteps"]
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.graph = graph
        self.integrator: Integrator | None = None

    def _load_datasets(self):
        """Open the input / boundary / reference WRF NetCDF files named by
        PYWRF_DATA_DIR and PYWRF_RUN_NAME (pywrf/solver.py:22-46): through
        xarray when it is installed, else classic-format files through
        :mod:`pywrf_b200.netcdf`."""
        data_dir = os.environ.get("PYWRF_DATA_DIR", "data")
        run = os.environ.get("PYWRF_RUN_NAME", "2024020106")
        paths = [os.path.join(data_dir, f"{stem}_{run}") for stem in ("wrf_inout_step3", "wrfbdy_d01", "wrfout_d01")]
        try:
            import xarray as xr   # I/O only
        except ImportError:
            from .netcdf import open_dataset
            return tuple(open_dataset(p) if os.path.exists(p) or i < 2 else None for i, p in enumerate(paths))
        return tuple(xr.open_dataset(p) for p in paths)

    @staticmethod
    def _arrays(ds) -> Mapping[str, np.ndarray]:
        class _View(dict):
            def __missing__(self, key):
                v = ds[key]
                if not isinstance(v, np.ndarray):   # xarray DataArray (or alike): its .data
                    v = getattr(v, "data", v)
                v = np.asarray(v)
                self[key] = v
                return v
        return _View()

    def prepare(self) -> Integrator:
        wrfinput, wrfbdy, _ = self._load_datasets()
        inputs, bdy = self._arrays(wrfinput), self._arrays(wrfbdy)
        self._bdy = bdy
        p = self.params
        g = grid_from_inputs(inputs, p["dx"], p["dy"], p["dt"], p["p_top"], p["soundsteps"], p["bdy_interval"])
        state = DeviceState.from_inputs(g, inputs, bdy, device=self.device)
        self.integrator = Integrator(state)
        return self.integrator

    def solve(self):
        """Integrate ``nsteps`` steps; returns the final key fields."""
        it = self.prepare()
        run_with_boundary_records(it, it.state.g, self._bdy, self.nsteps, graph=self.graph)
        st = it.status()
        if st["nan_p"]:
            raise FloatingPointError(f"NaN in the diagnosed pressure ({st['nan_p']} stage(s)) by step {st['step']}")
        s = it.state
        return {k: s[k] for k in ("u", "v", "w", "t", "ph", "mu", "moist")}
