"""Seeded synthetic idealized moist ARW states (the benchmark workloads).

The reference reads three WRF NetCDF files (input, lateral boundaries,
reference output) in ``WrfSolver.solve`` (pywrf/solver.py:40-136, 456-703);
those files are not distributed, so every workload here is built from a
seeded generator instead.  The builder returns arrays with exactly the shapes
that ``solve`` slices out of the NetCDF variables, so the same dictionary can
feed the reference (through a fake dataset) and this package's ingest step
(:func:`pywrf_b200.state.ingest`).

Construction (WRF ARW Tech Note base state, terrain-following eta with
c1=1, c2=0):

* eta full levels ``znw = 1 - (0.3 s + 0.7 s^2)``, ``s = k/(nz-1)``.
* base state: ``p_surf = p00 exp(-T0/A + sqrt((T0/A)^2 - 2 g h/(A R_d)))``,
  ``pb = znu (p_surf - p_top) + p_top``, ``theta_b = (T0 + A ln(pb/p00))
  (p00/pb)^(R_d/cp)``, ``mub = p_surf - p_top``, ``phb`` integrated from
  ``g h`` with ``alb``.
* terrain: Gaussian hill ``h0 exp(-(r/L)^2)`` centred in the domain.
* winds: ``u = u0 + 0.5 N(0,1)``, ``v = 0.5 N(0,1)``, ``w = 0``.
* theta': ``1 K N(0,1)`` plus a warm bubble of ``+3 K`` (radius 20 km,
  centre 1.5 km above ground).
* moisture: qv at 80 % RH below 8 km, tapering to 1e-6 above; qc = 1e-3
  inside the bubble; other hydrometeors zero.
* moist hydrostatic balance: full pressure from the moist column weight,
  inverse density from the equation of state, geopotential integrated with
  the dry-mass coordinate.
* lateral boundaries: boundary values are the coupled initial state in the
  5 outermost rows; tendencies are zero or seeded sinusoids of amplitude
  ``bdy_tend_amp`` (1/s, relative) on u, v, theta and qv.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .config import Grid

# physical constants (the values the reference's configuration module uses)
R_D = 287.0
CP = 1004.5
G = 9.81
P00 = 1.0e5
T0_PERT = 300.0
RVOVRD = 1.608362
CVPM = -0.7142857


@dataclasses.dataclass
class CaseSpec:
    """One synthetic workload: grid size, time step and perturbation knobs."""
    n: int = 64                 # nx_all = ny_all (allocated, 5-cell halo frame)
    nz: int = 41                # full (w) levels
    dx: float = 9000.0
    dt: float = 45.0
    p_top: float = 5000.0
    soundsteps: int = 4
    nsteps: int = 10
    t00: float = 290.0          # base-state sea-level temperature
    lapse_a: float = 50.0       # base-state lapse parameter A
    hill_h: float = 800.0
    hill_l: float = 60000.0
    u0: float = 10.0
    uv_noise: float = 0.5
    th_noise: float = 1.0
    bubble_dth: float = 3.0
    bubble_r: float = 20000.0
    bubble_z: float = 1500.0
    rh: float = 0.8
    moist_top: float = 8000.0
    qc_bubble: float = 1.0e-3
    bdy_tend_amp: float = 0.0   # 1/s, relative amplitude of LBC tendencies
    f_cor: float = 8.4e-5
    e_cor: float = 1.2e-4
    seed: int = 0


def spec_for_config(config: int, seed: int = 0) -> CaseSpec:
    """The BASELINE configurations by index (0: 64x64x41, 1-3: 240x240x41,
    4: 512x512x61)."""
    if config == 0:
        return CaseSpec(n=64, nz=41, dt=45.0, nsteps=10, seed=seed)
    if config in (1, 2, 3):
        return CaseSpec(n=240, nz=41, dt=45.0, nsteps=80, bdy_tend_amp=1.0e-4, seed=seed)
    if config == 4:
        return CaseSpec(n=512, nz=61, dt=30.0, nsteps=36, bdy_tend_amp=1.0e-4, seed=seed)
    raise ValueError(f"unknown config {config}")


def grid_for(spec: CaseSpec) -> Grid:
    return Grid.make(nx_all=spec.n, ny_all=spec.n, nz=spec.nz, dx=spec.dx, dy=spec.dx,
                     dt=spec.dt, p_top=spec.p_top, soundsteps=spec.soundsteps)


def _eta_levels(nz: int):
    s = np.arange(nz, dtype=np.float64) / (nz - 1)
    znw = 1.0 - (0.3 * s + 0.7 * s * s)
    znw[0], znw[-1] = 1.0, 0.0
    znu = 0.5 * (znw[:-1] + znw[1:])
    dnw = znw[1:] - znw[:-1]                       # [nz-1], negative
    dn = np.zeros(nz - 1)
    dn[1:] = znu[1:] - znu[:-1]                    # dn[0] unused (0)
    rdnw = 1.0 / dnw
    rdn = np.zeros(nz - 1)
    rdn[1:] = 1.0 / dn[1:]
    fnm = np.zeros(nz - 1)
    fnp = np.zeros(nz - 1)
    fnm[1:] = 0.5 * dnw[1:] / dn[1:]
    fnp[1:] = 0.5 * dnw[:-1] / dn[1:]
    # surface / top extrapolation weights (WRF Tech Note, module_initialize)
    cof1 = (2.0 * dn[1] + dn[2]) / (dn[1] + dn[2]) * dnw[0] / dn[1]
    cof2 = dn[1] / (dn[1] + dn[2]) * dnw[0] / dn[2]
    cf1 = fnp[1] + cof1
    cf2 = fnm[1] - cof1 - cof2
    cf3 = cof2
    kl = nz - 2
    cfn = (0.5 * dnw[kl] + dn[kl]) / dn[kl]
    cfn1 = -0.5 * dnw[kl] / dn[kl]
    return dict(znw=znw, znu=znu, dnw=dnw, dn=dn, rdnw=rdnw, rdn=rdn, fnm=fnm, fnp=fnp,
                cf1=cf1, cf2=cf2, cf3=cf3, cfn=cfn, cfn1=cfn1)


def _qsat(t_k, p_pa):
    es = 611.2 * np.exp(17.67 * (t_k - 273.15) / (t_k - 29.65))
    es = np.minimum(es, 0.5 * p_pa)
    return 0.622 * es / (p_pa - es)


def build(spec: CaseSpec):
    """Return ``(inputs, bdy)``: WRF-named float32 arrays with the reference's
    NetCDF shapes (``inputs[name]`` has a leading time dimension of 1;
    ``bdy[name]`` has a leading boundary-time dimension of 2)."""
    rng = np.random.default_rng(spec.seed)
    n, nz = spec.n, spec.nz
    nm = n - 11                         # mass points per row in the input files
    nu = n - 10                         # staggered points
    lev = _eta_levels(nz)
    znw, znu, dnw = lev["znw"], lev["znu"], lev["dnw"]

    # horizontal coordinates of mass points (i, j) relative to the domain centre
    xm = (np.arange(nm) - (nm - 1) / 2.0) * spec.dx
    X, Y = np.meshgrid(xm, xm)          # [j, i]
    r2 = X * X + Y * Y
    ht = spec.hill_h * np.exp(-r2 / (spec.hill_l ** 2))

    # base state
    a, t00 = spec.lapse_a, spec.t00
    p_surf = P00 * np.exp(-t00 / a + np.sqrt((t00 / a) ** 2 - 2.0 * G * ht / (a * R_D)))
    mub = p_surf - spec.p_top                                    # [j, i]
    pb = znu[:, None, None] * mub[None] + spec.p_top             # [k, j, i]
    temp_b = t00 + a * np.log(pb / P00)
    theta_b = temp_b * (P00 / pb) ** (R_D / CP)
    t_init = theta_b - T0_PERT
    alb = (R_D / P00) * theta_b * (pb / P00) ** CVPM
    phb = np.zeros((nz, nm, nm))
    phb[0] = G * ht
    for k in range(nz - 1):
        phb[k + 1] = phb[k] - dnw[k] * mub * alb[k]
    z_half = 0.5 * (phb[:-1] + phb[1:]) / G                      # approx height (m)
    zagl = z_half - ht[None]

    # perturbations
    th_pert = spec.th_noise * rng.standard_normal((nz - 1, nm, nm))
    rb = np.sqrt(r2[None] + (zagl - spec.bubble_z) ** 2)
    bubble = rb < spec.bubble_r
    th_pert = th_pert + np.where(bubble, spec.bubble_dth * np.cos(0.5 * np.pi * rb / spec.bubble_r) ** 2, 0.0)
    theta = theta_b + th_pert

    # moisture from relative humidity (uses base pressure for the temperature)
    tk = theta * (pb / P00) ** (R_D / CP)
    qs = _qsat(tk, pb)
    qv = spec.rh * qs
    taper = np.exp(-np.maximum(z_half - spec.moist_top, 0.0) / 1000.0)
    qv = np.maximum(qv * taper, 1.0e-6)
    qv = np.where(z_half > spec.moist_top + 6000.0, 1.0e-6, qv)
    qc = np.where(bubble, spec.qc_bubble, 0.0)

    # moist hydrostatic balance with mu' = 0
    mu = np.zeros((nm, nm))
    pw = np.zeros((nz, nm, nm))
    pw[nz - 1] = spec.p_top
    for k in range(nz - 2, -1, -1):
        pw[k] = pw[k + 1] - dnw[k] * mub * (1.0 + qv[k] + qc[k])
    pfull = 0.5 * (pw[:-1] + pw[1:])
    p = pfull - pb
    al_full = (R_D / P00) * theta * (1.0 + RVOVRD * qv) * (pfull / P00) ** CVPM
    ph_full = np.zeros((nz, nm, nm))
    ph_full[0] = G * ht
    for k in range(nz - 1):
        ph_full[k + 1] = ph_full[k] - dnw[k] * mub * al_full[k]
    ph = ph_full - phb

    # winds on staggered points
    u = spec.u0 + spec.uv_noise * rng.standard_normal((nz - 1, nm, nu))
    v = spec.uv_noise * rng.standard_normal((nz - 1, nu, nm))
    w = np.zeros((nz, nm, nm))

    ones_m = np.ones((nm, nm))
    ones_u = np.ones((nm, nu))
    ones_v = np.ones((nu, nm))
    f32 = lambda x: np.asarray(x, dtype=np.float32)
    e3 = lambda x: f32(x)[None]
    e1 = lambda x: f32(x)[None]

    inputs = {
        "U": e3(u), "V": e3(v), "W": e3(w), "MU": e3(mu), "MUB": e3(mub),
        "MAPFAC_U": e3(ones_u), "MAPFAC_V": e3(ones_v), "MF_VX_INV": e3(ones_v),
        "MAPFAC_M": e3(ones_m), "MAPFAC_MX": e3(ones_m), "MAPFAC_MY": e3(ones_m),
        "MAPFAC_UX": e3(ones_u), "MAPFAC_UY": e3(ones_u), "MAPFAC_VX": e3(ones_v),
        "MAPFAC_VY": e3(ones_v),
        "QVAPOR": e3(qv), "QCLOUD": e3(qc), "QRAIN": e3(np.zeros_like(qv)),
        "QICE": e3(np.zeros_like(qv)), "QSNOW": e3(np.zeros_like(qv)),
        "QGRAUP": e3(np.zeros_like(qv)),
        "PB": e3(pb), "P": e3(p), "T_INIT": e3(t_init), "PHB": e3(phb), "PH": e3(ph),
        "T": e3(theta - T0_PERT),
        "RDNW": e1(lev["rdnw"]), "RDN": e1(lev["rdn"]),
        "C1H": e1(np.ones(nz - 1)), "C2H": e1(np.zeros(nz - 1)),
        "C1F": e1(np.ones(nz)), "C2F": e1(np.zeros(nz)),
        "C3H": e1(znu), "C4H": e1(np.zeros(nz - 1)),
        "C3F": e1(znw), "C4F": e1(np.zeros(nz)),
        "FNM": e1(lev["fnm"]), "FNP": e1(lev["fnp"]),
        "DN": e1(lev["dn"]), "DNW": e1(dnw),
        "CF1": f32([lev["cf1"]]), "CF2": f32([lev["cf2"]]), "CF3": f32([lev["cf3"]]),
        "CFN": f32([lev["cfn"]]), "CFN1": f32([lev["cfn1"]]),
        "F": e3(spec.f_cor * ones_m), "E": e3(spec.e_cor * ones_m),
        "SINALPHA": e3(np.zeros((nm, nm))), "COSALPHA": e3(ones_m),
        "CLAT": e3(35.0 * ones_m),
        "ZNU": e1(znu), "ZNW": e1(znw), "HGT": e3(ht),
        "U_BASE": e1(spec.u0 * np.ones(nz - 1)), "V_BASE": e1(np.zeros(nz - 1)),
        "QV_BASE": e1(qv.mean(axis=(1, 2))),
    }

    # ---- lateral boundary files: coupled values in the 5 outer rows ----
    mut = mub + mu
    muu = np.empty((nm, nu))
    muu[:, 1:-1] = 0.5 * (mut[:, 1:] + mut[:, :-1])
    muu[:, 0] = mut[:, 0]
    muu[:, -1] = mut[:, -1]
    muv = np.empty((nu, nm))
    muv[1:-1] = 0.5 * (mut[1:] + mut[:-1])
    muv[0] = mut[0]
    muv[-1] = mut[-1]
    cu = u * muu[None]
    cv = v * muv[None]
    ct = (theta - T0_PERT) * mut[None]
    cph = ph * mut[None]
    cqv = qv * mut[None]

    def sides(f, stag_x, stag_y):
        """Boundary arrays [5, nz', n_along] for the xs, xe, ys, ye sides."""
        xs = np.stack([f[..., :, b] for b in range(5)])
        xe = np.stack([f[..., :, f.shape[-1] - 1 - b] for b in range(5)])
        ys = np.stack([f[..., b, :] for b in range(5)])
        ye = np.stack([f[..., f.shape[-2] - 1 - b, :] for b in range(5)])
        return xs, xe, ys, ye

    def tend_like(arr, phase):
        if spec.bdy_tend_amp == 0.0:
            return np.zeros_like(arr)
        along = np.arange(arr.shape[-1])
        wave = np.sin(2.0 * np.pi * along / max(arr.shape[-1], 1) + phase)
        return spec.bdy_tend_amp * arr * wave

    bdy = {}
    fields = {"U": (cu, True), "V": (cv, True), "PH": (cph, False), "T": (ct, True),
              "MU": (mu, False), "QVAPOR": (cqv, True)}
    for idx, (name, (arr, seeded)) in enumerate(fields.items()):
        xs, xe, ys, ye = sides(arr, False, False)
        for side, val in (("XS", xs), ("XE", xe), ("YS", ys), ("YE", ye)):
            bdy[f"{name}_B{side}"] = np.stack([val, val]).astype(np.float32)
            if seeded:
                tnd = tend_like(val, phase=0.7 * idx + {"XS": 0.0, "XE": 1.0, "YS": 2.0, "YE": 3.0}[side])
            else:
                tnd = np.zeros_like(val)
            bdy[f"{name}_BT{side}"] = np.stack([tnd, tnd]).astype(np.float32)
    return inputs, bdy
