"""Oracle ARW step driver (TEST INFRASTRUCTURE; see oracle/__init__.py).

``OracleModel`` holds every persistent buffer the reference's
``WrfSolver.solve`` keeps (pywrf/solver.py:138-448) and advances them with
the exact call order of one time step (pywrf/solver.py:709-1910).  Calls
whose results never reach the prognostic state are not made:

* ``phy_prep``/``calculate_phy_tend``/``update_phy_ten``/``phy_prep_part2``
  (the PBL tendencies are identically zero and the physics scratch they fill
  is overwritten by ``moist_physics_prep_em`` before WSM6 reads it);
* the vertical-diffusion calls (``kvdif = 0`` makes every flux exactly 0);
* the Brunt-Vaisala part of ``calculate_km_kh`` and defor13/23/33/div (not
  used by the 2-D Smagorinsky coefficient);
* the 3-slot passive-scalar transport (the scalars are zero and stay zero).

``probe(name, model)`` is called after every phase, with names shared with
the CUDA step driver, so a test can localise the first divergence.
"""
from __future__ import annotations

import numpy as np

from . import boundary as B
from . import dynamics as D
from . import physics as P

R_D = 287.0
P1000MB = 1.0e5
CVPM = -0.7142857
T0 = 300.0
FCX = [0.0, 5.5555557e-3, 3.7037039e-3, 1.8518519e-3, 0.0]
GCX = [0.0, 1.1111111e-3, 7.4074074e-4, 3.7037037e-4, 0.0]

FIELDS_3D = [
    "u", "v", "w", "pb", "p", "t_init", "phb", "ph", "t", "al", "alb", "ru", "rv", "rw", "ww", "ww1",
    "cqu", "cqv", "cqw", "alt", "php", "ru_tendf", "rv_tendf", "rw_tendf", "ph_tendf", "t_tendf",
    "ru_tend", "rv_tend", "rw_tend", "ph_tend", "t_tend", "u_save", "v_save", "w_save", "ph_save",
    "t_save", "rho", "dz8w", "rdz", "rdzw", "zx", "zy", "z", "defor11", "defor22", "defor12", "xkmh",
    "xkhh", "u_1", "v_1", "w_1", "t_1", "ph_1", "c2a", "pm1", "a", "alpha", "gamma", "ru_m", "rv_m",
    "ww_m", "t_2save", "th_phy", "p_phy", "pi_phy", "h_diabatic", "qv_diabatic", "qc_diabatic", "rfield",
]
FIELDS_2D = [
    "mu", "mub", "msfu", "msfv", "msfvx_inv", "msft", "msftx", "msfty", "msfux", "msfuy", "msfvx",
    "msfvy", "f", "e", "sina", "cosa", "clat", "ht", "rainnc", "rainncv", "snownc", "snowncv",
    "graupelnc", "graupelncv", "sr", "mut", "muu", "muv", "mu_tendf", "mu_tend", "mu_save", "mu_1",
    "muus", "muvs", "muts", "mudf", "muave",
]
FIELDS_1D = ["rdnw", "rdn", "c1h", "c2h", "c1f", "c2f", "c3h", "c4h", "c3f", "c4f", "fnm", "fnp", "znu",
             "znw", "dn", "dnw", "u_base", "v_base", "qv_base"]
BDY_FIELDS = ("u", "v", "ph", "t", "mu", "qv")
BDY_NAMES = {"u": "U", "v": "V", "ph": "PH", "t": "T", "mu": "MU", "qv": "QVAPOR"}


def ingest(g, inputs, bdy, dtype=np.float32):
    """Place the WRF-shaped arrays into the halo frame (pywrf/solver.py:138-448)."""
    n, nz = g.nx, g.nz
    st = {}
    for k in FIELDS_3D:
        st[k] = np.zeros((nz, g.ny, g.nx), dtype)
    for k in FIELDS_2D:
        st[k] = np.zeros((g.ny, g.nx), dtype)
    for k in FIELDS_1D:
        st[k] = np.zeros(nz, dtype)
    for k in ("moist", "moist_tend", "advect_tend", "moist_old"):
        st[k] = np.zeros((7, nz, g.ny, g.nx), dtype)
    a = lambda name: np.asarray(inputs[name], dtype)[0]
    M = (slice(5, g.ny - 6), slice(5, g.nx - 6))
    U = (slice(5, g.ny - 6), slice(5, g.nx - 5))
    V = (slice(5, g.ny - 5), slice(5, g.nx - 6))
    st["u"][(slice(0, nz - 1),) + U] = a("U")
    st["v"][(slice(0, nz - 1),) + V] = a("V")
    st["w"][(slice(0, nz),) + M] = a("W")
    st["mu"][M] = a("MU")
    st["mub"][M] = a("MUB")
    st["msfu"][U] = a("MAPFAC_U")
    st["msfv"][V] = a("MAPFAC_V")
    st["msfvx_inv"][V] = a("MF_VX_INV")
    st["msft"][M] = a("MAPFAC_M")
    st["msftx"][M] = a("MAPFAC_MX")
    st["msfty"][M] = a("MAPFAC_MY")
    st["msfux"][U] = a("MAPFAC_UX")
    st["msfuy"][U] = a("MAPFAC_UY")
    st["msfvx"][V] = a("MAPFAC_VX")
    st["msfvy"][V] = a("MAPFAC_VY")
    for slot, name in ((1, "QVAPOR"), (2, "QCLOUD"), (3, "QRAIN"), (4, "QICE"), (5, "QSNOW"), (6, "QGRAUP")):
        st["moist"][(slot, slice(0, nz - 1)) + M] = a(name)
    for k, name in (("pb", "PB"), ("p", "P"), ("t_init", "T_INIT"), ("t", "T")):
        st[k][(slice(0, nz - 1),) + M] = a(name)
    for k, name in (("phb", "PHB"), ("ph", "PH")):
        st[k][(slice(0, nz),) + M] = a(name)
    for k, name in (("rdnw", "RDNW"), ("rdn", "RDN"), ("c1h", "C1H"), ("c2h", "C2H"), ("c3h", "C3H"),
                    ("c4h", "C4H"), ("fnm", "FNM"), ("fnp", "FNP"), ("dn", "DN"), ("dnw", "DNW"),
                    ("u_base", "U_BASE"), ("v_base", "V_BASE"), ("qv_base", "QV_BASE"), ("znu", "ZNU")):
        st[k][0:nz - 1] = a(name)
    for k, name in (("c1f", "C1F"), ("c2f", "C2F"), ("c3f", "C3F"), ("c4f", "C4F"), ("znw", "ZNW")):
        st[k][:] = a(name)
    for k, name in (("cf1", "CF1"), ("cf2", "CF2"), ("cf3", "CF3"), ("cfn", "CFN"), ("cfn1", "CFN1")):
        st[k] = np.asarray(inputs[name], dtype)[0]
    for k, name in (("f", "F"), ("e", "E"), ("sina", "SINALPHA"), ("cosa", "COSALPHA"), ("clat", "CLAT"), ("ht", "HGT")):
        st[k][M] = a(name)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        st["alb"][...] = R_D / P1000MB * (st["t_init"] + T0) * np.power(st["pb"] / P1000MB, np.asarray(CVPM, dtype))
        R = (slice(0, nz - 1), slice(g.jts, g.jde - 1), slice(g.its, g.ide - 1))
        mm = (st["mub"] + st["mu"])[None, R[1], R[2]]
        st["al"][R] = -1.0 / mm * (st["alb"][R] * st["mu"][None, R[1], R[2]]
                                   + st["rdnw"][0:nz - 1, None, None] * (st["ph"][1:nz, R[1], R[2]] - st["ph"][R]))
    mub = st["mub"]
    mub[g.jte - 1, :] = mub[g.jte - 2, :]
    mub[:, g.ite - 1] = mub[:, g.ite - 2]
    mub[g.jts - 1, :] = mub[g.jts, :]
    mub[:, g.its - 1] = mub[:, g.its]
    st["fcx"] = np.asarray(FCX, dtype)
    st["gcx"] = np.asarray(GCX, dtype)
    st["bdy"] = ingest_bdy(g, bdy, 0, dtype)
    return st


def ingest_bdy(g, bdy, it, dtype=np.float32):
    """Boundary arrays in the reference's permuted layout (solver.py:457-703)."""
    n, nz = g.nx, g.nz
    out = {}
    for fld in BDY_FIELDS:
        W = BDY_NAMES[fld]
        nk = nz if fld == "ph" else (1 if fld == "mu" else nz - 1)
        tot = 1 if fld == "mu" else nz
        stag_x = fld == "u"
        stag_y = fld == "v"
        jx = slice(5, n - 5) if stag_y else slice(5, n - 6)   # along-boundary rows of the x sides
        iy = slice(5, n - 5) if stag_x else slice(5, n - 6)   # along-boundary columns of the y sides
        d = {}
        for side, key in (("XS", "xs"), ("XE", "xe"), ("YS", "ys"), ("YE", "ye")):
            for pre, kk in (("B", ""), ("BT", "t")):
                arr = np.asarray(bdy[f"{W}_{pre}{side}"], dtype)[it]
                if fld == "mu":
                    arr = arr[:, None, :]
                if side in ("XS", "XE"):
                    buf = np.zeros((5, tot, g.ny), dtype)
                    buf[:, 0:nk, jx] = arr
                    d[kk + key] = np.ascontiguousarray(buf.transpose(1, 2, 0))
                else:
                    buf = np.zeros((5, tot, g.nx), dtype)
                    buf[:, 0:nk, iy] = arr
                    d[kk + key] = np.ascontiguousarray(buf.transpose(1, 0, 2))
        out[fld] = d
    return out


class OracleModel:
    """Numpy state + one-RK3-step driver following pywrf/solver.py:709-1910."""

    def __init__(self, g, inputs, bdy, dtype=np.float32, theta_bias=None, microphysics=True):
        self.g = g
        self.dtype = dtype
        # False: the step of a model without microphysics (no moist physics
        # prep, WSM6 or finish; the equation of state after them still runs)
        self.microphysics = microphysics
        self.bdy_src = bdy
        # optional [nz, ny, nx] bias added to t_tend after rk_addtend_dry in
        # every RK stage (the learnable parameter of the adjoint configuration)
        self.theta_bias = None if theta_bias is None else np.asarray(theta_bias, dtype)
        self.st = ingest(g, inputs, bdy, dtype)
        self.step_count = 0

    # halo copy shorthands (set_physical_bc3d / set_physical_bc2d)
    def bc3(self, name, var):
        D.set_physical_bc3d(self.g, self.st[name], var)

    def bc2(self, name, var):
        D.set_physical_bc2d(self.g, self.st[name], var)

    def run(self, nsteps, probe=None):
        for _ in range(nsteps):
            self.step(self.step_count + 1, probe)

    def step(self, t_big_step, probe=None):
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            self._step(t_big_step, probe or (lambda name, m: None))
        self.step_count = t_big_step

    def _step(self, t_big_step, probe):
        g, s = self.g, self.st
        bd = s["bdy"]
        if t_big_step % g.bdy_interval == 1:
            self.it_bdy = int(t_big_step / g.bdy_interval)
            # solver.py:457-703: every boundary array from record it_bdy
            # (record 0 at step 1 is the one ingested)
            if t_big_step > 1:
                s["bdy"] = ingest_bdy(g, self.bdy_src, self.it_bdy, self.dtype)
                bd = s["bdy"]
        self.it_bdy = getattr(self, "it_bdy", 0)
        dt = g.dt
        dts = dt / g.soundsteps
        dtbc = dt * (t_big_step - self.it_bdy * g.bdy_interval)
        fcx, gcx = s["fcx"], s["gcx"]
        for rk_step in (1, 2, 3):
            if rk_step == 1:
                dt_rk, dts_rk, nsub = dt / 3.0, dt / 3.0, 1
            elif rk_step == 2:
                dt_rk, dts_rk, nsub = 0.5 * dt, dts, int(g.soundsteps / 2)
            else:
                dt_rk, dts_rk, nsub = dt, dts, g.soundsteps
            tag = f"s{rk_step}"
            # rk_step_prep (solver.py:736-778)
            D.calculate_full(g, s["mut"], s["mub"], s["mu"])
            D.calc_mu_uv(g, s["mu"], s["mub"], s["muu"], s["muv"])
            D.couple_momentum(g, s["muu"], s["ru"], s["u"], s["msfu"], s["muv"], s["rv"], s["v"], s["msfvx_inv"],
                              s["mut"], s["rw"], s["w"], s["msft"])
            D.calc_ww_cp(g, s["u"], s["v"], s["muu"], s["muv"], s["c1h"], s["ww"], s["msftx"], s["msfuy"],
                         s["msfvx_inv"], s["dnw"])
            D.calc_cq(g, s["moist"], s["cqu"], s["cqv"], s["cqw"])
            D.calc_alt(g, s["alt"], s["al"], s["alb"])
            D.calc_php(g, s["php"], s["ph"], s["phb"])
            for nm, var in (("ru", "u"), ("rv", "v"), ("rw", "w"), ("ww", "w"), ("php", "w"), ("alt", "t"), ("p", "p")):
                self.bc3(nm, var)
            self.bc2("muu", "u")
            self.bc2("muv", "v")
            self.bc2("mut", "t")
            self.bc3("al", "p")
            self.bc3("ph", "w")
            probe(tag + ".prep", self)
            if rk_step == 1:
                for nm in ("ru_tendf", "rv_tendf", "rw_tendf", "ph_tendf", "t_tendf"):
                    s[nm][...] = 0.0
                s["mu_tendf"][...] = 0.0
                s["moist_tend"][...] = 0.0
                D.compute_diff_metrics(g, s["ph"], s["phb"], s["z"], s["rdz"], s["rdzw"], s["zx"], s["zy"])
                self.bc3("rdzw", "w")
                self.bc3("rdz", "w")
                self.bc3("z", "w")
                self.bc3("zx", "e")
                self.bc3("zy", "f")
                D.cal_deform_and_div(g, s["u"], s["v"], s["defor11"], s["defor22"], s["defor12"], s["msfux"],
                                     s["msfuy"], s["msfvx"], s["msfvy"], s["msftx"], s["msfty"], s["dn"], s["dnw"],
                                     s["rdzw"], s["fnm"], s["fnp"], s["cf1"], s["cf2"], s["cf3"], s["zx"], s["zy"])
                D.calculate_km_kh(g, s["xkmh"], s["xkhh"], s["defor11"], s["defor22"], s["defor12"], s["msftx"], s["msfty"])
                self.bc3("xkmh", "t")
                self.bc3("xkhh", "t")
                probe(tag + ".km", self)
            for nm in ("ru_tend", "rv_tend", "rw_tend", "t_tend", "ph_tend", "u_save", "v_save", "w_save", "ph_save", "t_save"):
                s[nm][...] = 0.0
            s["mu_tend"][...] = 0.0
            s["mu_save"][...] = 0.0
            D.advect_u(g, s["u"], s["ru_tend"], s["ru"], s["rv"], s["ww"], s["msfux"], s["fnm"], s["fnp"], s["rdnw"])
            D.advect_v(g, s["v"], s["rv_tend"], s["ru"], s["rv"], s["ww"], s["msfvx"], s["msfvy"], s["fnm"], s["fnp"], s["rdnw"])
            D.advect_w(g, s["w"], s["rw_tend"], s["ru"], s["rv"], s["ww"], s["msftx"], s["fnm"], s["fnp"], s["rdn"])
            D.advect_scalar(g, s["t"], s["t_tend"], s["ru"], s["rv"], s["ww"], s["msftx"], s["fnm"], s["fnp"], s["rdnw"])
            probe(tag + ".adv", self)
            D.rhs_ph(g, s["ph_tend"], s["u"], s["v"], s["ww"], s["ph"], s["phb"], s["w"], s["mut"], s["muu"], s["muv"],
                     s["fnm"], s["fnp"], s["rdnw"], s["cfn"], s["cfn1"], s["msfux"], s["msfvy"], s["msfty"])
            D.horizontal_pressure_gradient(g, s["ru_tend"], s["rv_tend"], s["ph"], s["alt"], s["p"], s["pb"], s["al"],
                                           s["php"], s["cqu"], s["cqv"], s["muu"], s["muv"], s["mu"], s["fnm"], s["fnp"],
                                           s["rdnw"], s["cf1"], s["cf2"], s["cf3"], s["msfux"], s["msfuy"], s["msfvx"], s["msfvy"])
            D.pg_buoy_w(g, s["rw_tend"], s["p"], s["cqw"], s["mu"], s["mub"], s["rdnw"], s["rdn"], s["msfty"])
            D.coriolis(g, s["ru"], s["rv"], s["rw"], s["ru_tend"], s["rv_tend"], s["rw_tend"], s["msftx"], s["msfty"],
                       s["msfux"], s["msfuy"], s["msfvx"], s["msfvy"], s["f"], s["e"], s["sina"], s["cosa"], s["fnm"], s["fnp"])
            D.curvature(g, s["ru"], s["rv"], s["rw"], s["u"], s["v"], s["ru_tend"], s["rv_tend"], s["rw_tend"], s["msfux"],
                        s["msfuy"], s["msfvx"], s["msfvy"], s["msftx"], s["msfty"], s["fnm"], s["fnp"])
            probe(tag + ".forces", self)
            if rk_step == 1:
                for name in ("u", "v", "w"):
                    D.horizontal_diffusion(g, name, s[name], s[f"r{name}_tendf"], s["mut"], s["msfux"], s["msfuy"],
                                           s["msfvx"], s["msfvx_inv"], s["msfvy"], s["msftx"], s["msfty"], s["xkmh"])
                D.horizontal_diffusion(g, "m", s["t"], s["t_tendf"], s["mut"], s["msfux"], s["msfuy"], s["msfvx"],
                                       s["msfvx_inv"], s["msfvy"], s["msftx"], s["msfty"], s["xkhh"], base=s["t_init"])
                B.relax_bdytend(g, s["ru"], s["u_save"], bd["u"], "u", dtbc, fcx, gcx)
                B.relax_bdytend(g, s["rv"], s["v_save"], bd["v"], "v", dtbc, fcx, gcx)
                mw = (slice(0, g.nz), slice(g.jds, g.jde - 1), slice(g.ids, g.ide - 1))
                B.mass_weight(s["ph"], s["mut"], s["rfield"], *mw)
                B.relax_bdytend(g, s["rfield"], s["ph_save"], bd["ph"], "h", dtbc, fcx, gcx)
                B.mass_weight(s["t"], s["mut"], s["rfield"], *mw)
                B.relax_bdytend(g, s["rfield"], s["t_save"], bd["t"], "t", dtbc, fcx, gcx)
                B.relax_bdytend(g, s["mu"][None], s["mu_tend"][None], bd["mu"], "m", dtbc, fcx, gcx)
                probe(tag + ".diff", self)
            D.rk_addtend_dry(g, s["ru_tend"], s["rv_tend"], s["rw_tend"], s["ph_tend"], s["t_tend"], s["ru_tendf"],
                             s["rv_tendf"], s["rw_tendf"], s["ph_tendf"], s["t_tendf"], s["u_save"], s["v_save"],
                             s["w_save"], s["ph_save"], s["t_save"], s["mu_tend"], s["mu_tendf"], rk_step,
                             s["h_diabatic"], s["mut"], s["msfty"], s["msfuy"], s["msfvx"], s["msfvx_inv"])
            if self.theta_bias is not None:
                s["t_tend"][...] = s["t_tend"] + self.theta_bias
            B.spec_bdytend(g, s["ru_tend"], bd["u"], "u")
            B.spec_bdytend(g, s["rv_tend"], bd["v"], "v")
            B.spec_bdytend(g, s["ph_tend"], bd["ph"], "h")
            B.spec_bdytend(g, s["t_tend"], bd["t"], "t")
            B.spec_bdytend(g, s["mu_tend"][None], bd["mu"], "m")
            probe(tag + ".tend", self)
            # acoustic set-up (solver.py:1258-1345)
            D.small_step_prep(g, s, rk_step)
            s["pm1"] = D.calc_p_rho(g, s["al"], s["p"], s["ph"], s["alt"], s["t"], s["t_save"], s["c2a"], s["pm1"],
                                    s["mu"], s["muts"], s["rdnw"], g.smdiv, 0)
            D.calc_coef_w(g, s["a"], s["alpha"], s["gamma"], s["mut"], s["cqw"], s["rdn"], s["rdnw"], s["c2a"], dts_rk, g.epssm, g.top_lid)
            self.bc3("ru_tend", "u")
            self.bc3("rv_tend", "v")
            self.bc3("ph", "w")
            self.bc3("al", "p")
            self.bc3("p", "p")
            self.bc3("t_1", "t")
            self.bc3("t_save", "t")
            self.bc2("mu_1", "t")
            self.bc2("mu", "t")
            self.bc2("mudf", "t")
            probe(tag + ".acprep", self)
            for iteration in range(1, nsub + 1):
                D.advance_uv(g, s["u"], s["ru_tend"], s["v"], s["rv_tend"], s["p"], s["pb"], s["ph"], s["php"], s["alt"],
                             s["al"], s["mu"], s["muu"], s["cqu"], s["muv"], s["cqv"], s["mudf"], s["msfux"], s["msfuy"],
                             s["msfvx"], s["msfvx_inv"], s["msfvy"], dts_rk, s["cf1"], s["cf2"], s["cf3"], s["fnm"],
                             s["fnp"], g.emdiv, s["rdnw"])
                B.spec_bdyupdate(g, s["u"], s["ru_tend"], dts_rk, "u")
                B.spec_bdyupdate(g, s["v"], s["rv_tend"], dts_rk, "v")
                D.advance_mu_t(g, s, dts_rk, g.epssm, iteration)
                B.spec_bdyupdate(g, s["t"], s["t_tend"], dts_rk, "t")
                B.spec_bdyupdate(g, s["mu"], s["mu_tend"], dts_rk, "m")
                B.spec_bdyupdate(g, s["muts"], s["mu_tend"], dts_rk, "m")
                D.advance_w(g, s, dts_rk, g.epssm, s["cf1"], s["cf2"], s["cf3"])
                D.sumflux(g, s, iteration, nsub)
                B.spec_bdyupdate_ph(g, s["ph_save"], s["ph"], s["ph_tend"], s["mu_tend"], s["muts"], dts_rk)
                B.zero_grad_bdy(g, s["w"], "w")
                s["pm1"] = D.calc_p_rho(g, s["al"], s["p"], s["ph"], s["alt"], s["t"], s["t_save"], s["c2a"], s["pm1"],
                                        s["mu"], s["muts"], s["rdnw"], g.smdiv, iteration)
                self.bc3("ph", "w")
                self.bc3("al", "p")
                self.bc3("p", "p")
                self.bc2("muts", "t")
                self.bc2("mu", "t")
                self.bc2("mudf", "t")
                probe(f"{tag}.sub{iteration}", self)
            D.calc_mu_uv_1(g, s["muts"], s["muus"], s["muvs"])
            D.small_step_finish(g, s, nsub, dts_rk, rk_step)
            if rk_step == 3:
                self.bc3("ru_m", "u")
                self.bc3("rv_m", "v")
                self.bc3("ww_m", "w")
                self.bc2("mut", "t")
                self.bc2("muts", "t")
            probe(tag + ".acfinish", self)
            # moisture transport (solver.py:1548-1604)
            for im in range(1, 7):
                s["advect_tend"][im][0:g.nz, g.jts:g.jte, g.its:g.ite] = 0.0
                D.advect_scalar(g, s["moist"][im], s["advect_tend"][im], s["ru_m"], s["rv_m"], s["ww_m"], s["msftx"],
                                s["fnm"], s["fnp"], s["rdnw"])
                if rk_step == 1:
                    D.horizontal_diffusion(g, "m", s["moist"][im], s["moist_tend"][im], s["muts"], s["msfux"], s["msfuy"],
                                           s["msfvx"], s["msfvx_inv"], s["msfvy"], s["msftx"], s["msfty"], s["xkhh"])
            if rk_step == 1:
                rq = np.zeros_like(s["t"])
                B.mass_weight(s["moist"][1], s["mut"], rq, slice(0, g.nz - 1), slice(g.jds, g.jde - 1), slice(g.ids, g.ide - 1))
                B.relax_bdytend(g, rq, s["moist_tend"][1], bd["qv"], "q", dtbc, fcx, gcx)
                B.spec_bdytend(g, s["moist_tend"][1], bd["qv"], "q")
            D.rk_update_scalar(g, s["moist_old"], s["moist"], s["moist_tend"], s["advect_tend"], s["msfty"],
                               s["mu_1"], s["mu"], s["mub"], rk_step, dt_rk)
            for im in range(2, 7):
                B.flow_dep_bdy(g, s["moist"][im], s["ru_m"], s["rv_m"])
            D.calc_p_rho_phi(g, s["moist"][1], s["al"], s["alb"], s["mu"], s["muts"], s["ph"], s["p"], s["pb"], s["t"], s["rdnw"])
            self.nan_flag = bool(np.isnan(s["p"]).any())
            if rk_step < 3:
                self.bc3("u", "U")
                self.bc3("v", "V")
                self.bc3("w", "w")
                self.bc3("t", "p")
                self.bc3("ph", "w")
                self.bc2("mu", "t")
                for im in range(1, 7):
                    D.set_physical_bc3d(g, s["moist"][im], "p")
            probe(tag + ".moist", self)
        # microphysics (solver.py:1714-1766)
        if self.microphysics:
            P.moist_physics_prep_em(g, s)
            mo = s["moist"]
            P.wsm6(g, s["th_phy"], mo[1], mo[2], mo[3], mo[4], mo[5], mo[6], s["rho"], s["pi_phy"], s["p_phy"],
                   s["dz8w"], float(dt), s["rainnc"], s["rainncv"], s["snownc"], s["snowncv"], s["graupelnc"],
                   s["graupelncv"], s["sr"])
            P.moist_physics_finish_em(g, s, dt)
        D.calc_p_rho_phi(g, s["moist"][1], s["al"], s["alb"], s["mu"], s["muts"], s["ph"], s["p"], s["pb"], s["t"], s["rdnw"])
        probe("mp", self)
        # end-of-step boundaries (solver.py:1776-1910)
        for nm, var in (("u_1", "U"), ("u", "U"), ("v_1", "V"), ("v", "V"), ("w_1", "w"), ("w", "w"),
                        ("t_1", "p"), ("t", "p"), ("ph_1", "w"), ("ph", "w")):
            self.bc3(nm, var)
        self.bc2("mu_1", "t")
        self.bc2("mu", "t")
        for im in range(1, 7):
            D.set_physical_bc3d(g, s["moist"][im], "p")
        B.spec_bdy_final(g, s["u"], s["muus"], s["msfuy"], bd["u"], "u", dtbc)
        B.spec_bdy_final(g, s["v"], s["muvs"], s["msfvx"], bd["v"], "v", dtbc)
        B.spec_bdy_final(g, s["t"], s["muts"], s["msfty"], bd["t"], "t", dtbc)
        B.spec_bdy_final(g, s["ph"], s["muts"], s["msfty"], bd["ph"], "h", dtbc)
        B.spec_bdy_final(g, s["moist"][1], s["muts"], s["msfty"], bd["qv"], "t", dtbc)
        D.set_w_surface(g, s["w"], s["ht"], s["u"], s["v"], s["cf1"], s["cf2"], s["cf3"], s["msftx"], s["msfty"])
        probe("end", self)
