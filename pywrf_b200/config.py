"""Grid / run parameters of one ARW integration.

The reference keeps these as module globals that its kernel modules copy at
import time (pywrf/config_params.py:29-112).  Here they are one immutable
record that is passed explicitly: to the oracle, to the C-ABI library (as
``WrfGrid``, see include/pywrf_b200.h) and to the host step driver.

Index convention (identical to the reference's python-style WRF index sets,
config_params.py:67-99): fields are allocated ``[nz, ny_all, nx_all]``
(k, j, i; x fastest) with a 5-cell frame; ``ids = jds = 5``,
``ide = nx_all - 5``, ``jde = ny_all - 5``; mass points occupy
``[ids, ide-1)``, x-staggered points ``[ids, ide)``; ``kde = kte = nz``.
"""
from __future__ import annotations

import dataclasses


@dataclasses.dataclass(frozen=True)
class Grid:
    nx: int
    ny: int
    nz: int
    ids: int
    ide: int
    jds: int
    jde: int
    kds: int
    kde: int
    dx: float
    dy: float
    dt: float
    p_top: float
    soundsteps: int
    # namelist-style options and diffusion/damping coefficients
    # (config_params.py:29-49, 114-118)
    smdiv: float = 0.1
    emdiv: float = 0.01
    epssm: float = 0.1
    khdif: float = 0.0
    kvdif: float = 0.0
    spec_zone: int = 1
    spec_bdy_width: int = 5
    relax_zone: int = 4
    bdy_interval: int = 360
    top_lid: bool = False

    @staticmethod
    def make(nx_all: int, ny_all: int, nz: int, dx: float, dy: float, dt: float,
             p_top: float = 5000.0, soundsteps: int = 4) -> "Grid":
        if nx_all < 24 or ny_all < 24:
            raise ValueError("grid must be at least 24x24 (5-cell frame + 5th-order stencils)")
        if nz < 12:
            raise ValueError("need at least 12 vertical levels")
        return Grid(nx=nx_all, ny=ny_all, nz=nz, ids=5, ide=nx_all - 5, jds=5, jde=ny_all - 5,
                    kds=0, kde=nz, dx=float(dx), dy=float(dy), dt=float(dt), p_top=float(p_top),
                    soundsteps=int(soundsteps))

    # tile == patch == domain (single patch, as in the reference)
    @property
    def its(self): return self.ids
    @property
    def ite(self): return self.ide
    @property
    def jts(self): return self.jds
    @property
    def jte(self): return self.jde
    @property
    def kts(self): return 0
    @property
    def kte(self): return self.nz
    @property
    def rdx(self): return 1.0 / self.dx
    @property
    def rdy(self): return 1.0 / self.dy
    @property
    def npoints(self): return self.nx * self.ny * self.nz

    def index_tuple(self):
        """(ids, ide, jds, jde, kds, kde, ims, ime, jms, jme, kms, kme,
        its, ite, jts, jte, kts, kte) as the reference passes them."""
        return (self.ids, self.ide, self.jds, self.jde, self.kds, self.kde,
                0, self.nx, 0, self.ny, 0, self.nz,
                self.its, self.ite, self.jts, self.jte, self.kts, self.kte)
