"""Host ingest of the WRF input arrays and the device-resident step state.

:func:`ingest` places the WRF-shaped input / boundary arrays into the 5-cell
halo frame exactly as ``WrfSolver.solve`` does before its time loop
(pywrf/solver.py:138-448 for the state, 457-703 for the lateral-boundary
arrays); :class:`DeviceState` owns one CUDA tensor per entry of the C ABI's
field table (include/pywrf_b200.h) and hands the kernels a ``WrfState``
pointer table.  All persistent work buffers of the reference's time loop
(tendencies, saved states, time-averaged fluxes, eddy viscosities ...) are
entries of that table, so the step is a pure function of device memory.
"""
from __future__ import annotations

import ctypes
from typing import Mapping

import numpy as np
import torch

from . import _native as N
from .config import Grid

R_D = 287.0
P1000MB = 1.0e5
CVPM = -0.7142857
T0 = 300.0

SPECIES = ("qv", "qc", "qr", "qi", "qs", "qg")          # moist slots 1..6
_SPECIES_WRF = ("QVAPOR", "QCLOUD", "QRAIN", "QICE", "QSNOW", "QGRAUP")
BDY_FIELDS = ("u", "v", "ph", "t", "mu", "qv")
_BDY_WRF = {"u": "U", "v": "V", "ph": "PH", "t": "T", "mu": "MU", "qv": "QVAPOR"}


def field_shape(kind: int, g: Grid) -> tuple[int, ...]:
    nz, ny, nx = g.nz, g.ny, g.nx
    return {
        N.WRF_K3: (nz, ny, nx), N.WRF_K2: (ny, nx), N.WRF_K1: (nz,), N.WRF_K4: (7, nz, ny, nx),
        N.WRF_KBX: (nz, ny, 5), N.WRF_KBY: (nz, 5, nx), N.WRF_KBX2: (1, ny, 5), N.WRF_KBY2: (1, 5, nx),
        N.WRF_KSF: (16,), N.WRF_KSI: (16,),
    }[kind]


def field_dtype(kind: int):
    return torch.int32 if kind == N.WRF_KSI else torch.float32


def grid_from_inputs(inputs: Mapping[str, np.ndarray], dx: float, dy: float, dt: float,
                     p_top: float, soundsteps: int, bdy_interval: int = 360) -> Grid:
    """Allocated extents from the mass-point input shape ``T`` [1, nz-1, ny-11, nx-11]."""
    t = np.asarray(inputs["T"])
    nz = t.shape[1] + 1
    ny, nx = t.shape[2] + 11, t.shape[3] + 11
    g = Grid.make(nx, ny, nz, dx, dy, dt, p_top=p_top, soundsteps=soundsteps)
    if bdy_interval != g.bdy_interval:
        import dataclasses
        g = dataclasses.replace(g, bdy_interval=int(bdy_interval))
    return g


def ingest(g: Grid, inputs: Mapping[str, np.ndarray], bdy: Mapping[str, np.ndarray], it_bdy: int = 0):
    """Host arrays (float32) for every initialised state field, keyed by the
    field-table names, plus the scalar coefficients ``cf1 .. cfn1``.

    ``inputs`` holds WRF-named arrays with a leading time axis of 1 (the
    shapes ``solve`` slices out of wrfinput); ``bdy`` the wrfbdy arrays with a
    leading boundary-time axis, of which slice ``it_bdy`` is used."""
    f32 = np.float32
    nz, ny, nx = g.nz, g.ny, g.nx
    a = lambda name: np.asarray(inputs[name], f32)[0]
    z3 = lambda: np.zeros((nz, ny, nx), f32)
    z2 = lambda: np.zeros((ny, nx), f32)
    M = (slice(5, ny - 6), slice(5, nx - 6))
    U = (slice(5, ny - 6), slice(5, nx - 5))
    V = (slice(5, ny - 5), slice(5, nx - 6))
    h = slice(0, nz - 1)
    st: dict[str, np.ndarray] = {}
    for k in ("u", "v", "w", "t", "ph", "p", "pb", "phb", "t_init"):
        st[k] = z3()
    st["u"][(h,) + U] = a("U")
    st["v"][(h,) + V] = a("V")
    st["w"][(slice(0, nz),) + M] = a("W")
    for k, name in (("pb", "PB"), ("p", "P"), ("t_init", "T_INIT"), ("t", "T")):
        st[k][(h,) + M] = a(name)
    for k, name in (("phb", "PHB"), ("ph", "PH")):
        st[k][(slice(0, nz),) + M] = a(name)
    for k, name, R in (("mu", "MU", M), ("mub", "MUB", M), ("msfu", "MAPFAC_U", U), ("msfv", "MAPFAC_V", V),
                       ("msfvx_inv", "MF_VX_INV", V), ("msft", "MAPFAC_M", M), ("msftx", "MAPFAC_MX", M),
                       ("msfty", "MAPFAC_MY", M), ("msfux", "MAPFAC_UX", U), ("msfuy", "MAPFAC_UY", U),
                       ("msfvx", "MAPFAC_VX", V), ("msfvy", "MAPFAC_VY", V), ("f", "F", M), ("e", "E", M),
                       ("sina", "SINALPHA", M), ("cosa", "COSALPHA", M), ("ht", "HGT", M)):
        st[k] = z2()
        st[k][R] = a(name)
    moist = np.zeros((7, nz, ny, nx), f32)
    for slot, name in enumerate(_SPECIES_WRF, start=1):
        moist[(slot, h) + M] = a(name)
    st["moist"] = moist
    for k, name in (("rdnw", "RDNW"), ("rdn", "RDN"), ("c1h", "C1H"), ("fnm", "FNM"), ("fnp", "FNP"),
                    ("dn", "DN"), ("dnw", "DNW")):
        st[k] = np.zeros(nz, f32)
        st[k][0:nz - 1] = a(name)
    # base-state inverse density over the whole allocation, perturbation
    # inverse density on the mass interior (solver.py:393-420)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        st["alb"] = (R_D / P1000MB * (st["t_init"] + T0) *
                     np.power(st["pb"] / P1000MB, np.asarray(CVPM, f32))).astype(f32)
        st["al"] = z3()
        R = (h, slice(g.jds, g.jde - 1), slice(g.ids, g.ide - 1))
        mm = (st["mub"] + st["mu"])[None, R[1], R[2]]
        st["al"][R] = -1.0 / mm * (st["alb"][R] * st["mu"][None, R[1], R[2]] +
                                   st["rdnw"][0:nz - 1, None, None] * (st["ph"][1:nz, R[1], R[2]] - st["ph"][R]))
    mub = st["mub"]
    mub[g.jde - 1, :] = mub[g.jde - 2, :]
    mub[:, g.ide - 1] = mub[:, g.ide - 2]
    mub[g.jds - 1, :] = mub[g.jds, :]
    mub[:, g.ids - 1] = mub[:, g.ids]
    st.update(ingest_bdy(g, bdy, it_bdy))
    scal = {k: float(np.asarray(inputs[k.upper()], f32).reshape(-1)[0]) for k in ("cf1", "cf2", "cf3", "cfn", "cfn1")}
    return st, scal


def ingest_bdy(g: Grid, bdy: Mapping[str, np.ndarray], it: int = 0) -> dict[str, np.ndarray]:
    """Lateral-boundary values and tendencies in the permuted layout the
    kernels read: x sides [nzb, ny, 5], y sides [nzb, 5, nx] (solver.py:457-703)."""
    f32 = np.float32
    nz, ny, nx = g.nz, g.ny, g.nx
    out = {}
    for fld in BDY_FIELDS:
        W = _BDY_WRF[fld]
        nk = nz if fld == "ph" else (1 if fld == "mu" else nz - 1)
        tot = 1 if fld == "mu" else nz
        jx = slice(5, ny - 5) if fld == "v" else slice(5, ny - 6)
        iy = slice(5, nx - 5) if fld == "u" else slice(5, nx - 6)
        for side in ("XS", "XE", "YS", "YE"):
            for pre in ("B", "BT"):
                arr = np.asarray(bdy[f"{W}_{pre}{side}"], f32)[it]
                if fld == "mu":
                    arr = arr[:, None, :]
                if side in ("XS", "XE"):
                    buf = np.zeros((5, tot, ny), f32)
                    buf[:, 0:nk, jx] = arr
                    val = buf.transpose(1, 2, 0)
                else:
                    buf = np.zeros((5, tot, nx), f32)
                    buf[:, 0:nk, iy] = arr
                    val = buf.transpose(1, 0, 2)
                out[f"{fld}_{pre.lower()}{side.lower()}"] = np.ascontiguousarray(val)
    return out


class DeviceState:
    """One CUDA tensor per field of the C ABI table, plus its pointer table."""

    def __init__(self, g: Grid, device="cuda", scal: Mapping[str, float] | None = None):
        self.g = g
        self.device = torch.device(device)
        names, kinds = N.field_names(), N.field_kinds()
        self.names = names
        self.t: dict[str, torch.Tensor] = {}
        for nm, kd in zip(names, kinds):
            self.t[nm] = torch.zeros(field_shape(kd, g), dtype=field_dtype(kd), device=self.device)
        self.scal = dict(scal or {"cf1": 0.0, "cf2": 0.0, "cf3": 0.0, "cfn": 0.0, "cfn1": 0.0})
        self._ptrs = (ctypes.c_void_p * len(names))(*[self.t[nm].data_ptr() for nm in names])
        self.cgrid = make_cgrid(g, self.scal)

    @classmethod
    def from_inputs(cls, g: Grid, inputs, bdy, device="cuda", it_bdy: int = 0) -> "DeviceState":
        host, scal = ingest(g, inputs, bdy, it_bdy)
        s = cls(g, device, scal)
        s.load(host)
        return s

    def load(self, host: Mapping[str, np.ndarray]) -> None:
        for k, v in host.items():
            dst = self.t[k]
            src = torch.from_numpy(np.ascontiguousarray(v)).to(dst.dtype)
            if tuple(src.shape) != tuple(dst.shape):
                raise ValueError(f"{k}: shape {tuple(src.shape)} != {tuple(dst.shape)}")
            dst.copy_(src)

    def snapshot(self) -> dict[str, torch.Tensor]:
        """Device copies of every field (status words included)."""
        return {k: v.clone() for k, v in self.t.items()}

    def restore(self, snap: Mapping[str, torch.Tensor]) -> None:
        """Copy a :meth:`snapshot` back in place: the storage, and with it
        every pointer a captured step graph holds, stays the same."""
        for k, v in snap.items():
            self.t[k].copy_(v)

    def __getitem__(self, name: str) -> torch.Tensor:
        return self.t[name]

    @property
    def ptr(self) -> ctypes.c_void_p:
        return ctypes.cast(self._ptrs, ctypes.c_void_p)

    def status(self) -> np.ndarray:
        return self.t["status"].cpu().numpy()

    def numpy(self, name: str) -> np.ndarray:
        return self.t[name].cpu().numpy()


def make_cgrid(g: Grid, scal: Mapping[str, float]) -> N.WrfGridC:
    return N.WrfGridC(nx=g.nx, ny=g.ny, nz=g.nz, ids=g.ids, ide=g.ide, jds=g.jds, jde=g.jde,
                      soundsteps=g.soundsteps, spec_zone=g.spec_zone, bdy_interval=g.bdy_interval,
                      top_lid=int(bool(g.top_lid)), dx=g.dx, dy=g.dy, dt=g.dt, smdiv=g.smdiv,
                      emdiv=g.emdiv, epssm=g.epssm, khdif=g.khdif, kvdif=g.kvdif,
                      cf1=scal["cf1"], cf2=scal["cf2"], cf3=scal["cf3"], cfn=scal["cfn"], cfn1=scal["cfn1"])
