"""Oracle restatement of WSM6 and the moist-physics wrappers (reference pywrf/wrf_physics.py).

TEST INFRASTRUCTURE: see oracle/__init__.py.  WSM6 is evaluated on the
column block the solver passes it (pywrf/solver.py:1724-1747: i, j in
[ids+1, ide-2), k in [0, nz-1)); every process rate is a pointwise
``where`` chain in the reference's statement order, and sedimentation is a
per-column semi-Lagrangian remap (nislfv_rain_plm / _plm6).
"""
from __future__ import annotations

import numpy as np

G = 9.81
CPD = 1004.5
CPV = 1846.4
RD = 287.0
RV = 461.6
T0C = 273.149993896484375
EP2 = 0.621750414371490479
QMIN = 1.0e-15
XLS = 2850000.0
XLV0 = 2500000.0
XLF0 = 350000.0
DEN0 = 1.28
DENR = 1000.0
CLIQ = 4190.0
CICE = 2106.0
PSAT = 610.78
P0 = 1.0e5
RCP = 0.2857143
T0 = 300.0
# WSM6 parameters (pywrf/config_params.py:163-253)
DTCLDCR = 120.0
N0R = 8.0e6
AVTR = 841.9
QCRMIN = 1.0e-9
N0SMAX = 1.0e11
N0S = 2.0e6
ALPHA = 0.12
PFRZ1 = 100.0
PFRZ2 = 0.66
XNCR = 3.0e8
DICON = 11.9
DIMAX = 500.0e-6
DENS = 100.0
QS0 = 6.0e-4
QC0 = 5.0265482e-04
QCK1 = 6.773895
BVTR = 0.8
G6PBR = 495.4590
PVTR = 2500.064
PACRR = 2.4813369e10
PRECR1 = 3.9207076e07
PRECR2 = 8.2585357e08
ROQIMAX = 8.1250037e-05
BVTS = 0.41
N0G = 4000000.0
BVTG = 0.8
PVTS = 20.05161
PRECS1 = 5200000.0
PRECS2 = 1.8681944e07
PIDN0R = 2.5132743e10
PIDN0S = 6.2831853e08
XLV1 = 2343.6
PACRC = 5.5442112e07
PI = 3.141593
PVTG = 979.9514
PRECG1 = 1.9603538e07
PRECG2 = 2.5852333e08
PIDN0G = 6.2831857e09
RSLOPERMAX = 1.2500000e-05
RSLOPERBMAX = 1.1954404e-04
RSLOPER2MAX = 1.5624999e-10
RSLOPER3MAX = 1.9531248e-15


def _f(dt, x):
    return np.asarray(x, dtype=dt)


def moist_physics_prep_em(g, st):
    """wrf_physics.py:27-91 on i, j in [ids+1, ide-1): the fields WSM6 reads
    (theta, density, Exner, full pressure, layer depths) and the diabatic
    reference copies."""
    nz = g.nz
    ktf = nz - 1
    J, I = slice(g.jds + 1, g.jde - 1), slice(g.ids + 1, g.ide - 1)
    zaw = (st["ph"][0:nz, J, I] + st["phb"][0:nz, J, I]) / G
    st["dz8w"][0:nz - 1, J, I] = zaw[1:nz] - zaw[0:nz - 1]
    st["dz8w"][nz - 1, J, I] = 0.0
    st["th_phy"][0:ktf, J, I] = st["t"][0:ktf, J, I] + T0
    st["h_diabatic"][0:ktf, J, I] = st["th_phy"][0:ktf, J, I]
    st["qv_diabatic"][0:ktf, J, I] = st["moist"][1][0:ktf, J, I]
    st["qc_diabatic"][0:ktf, J, I] = st["moist"][2][0:ktf, J, I]
    st["rho"][0:ktf, J, I] = 1.0 / (st["al"][0:ktf, J, I] + st["alb"][0:ktf, J, I])
    st["pi_phy"][0:ktf, J, I] = ((st["p"][0:ktf, J, I] + st["pb"][0:ktf, J, I]) / P0) ** RCP
    st["p_phy"][0:ktf, J, I] = st["p"][0:ktf, J, I] + st["pb"][0:ktf, J, I]


def moist_physics_finish_em(g, st, dt):
    """wrf_physics.py:2106-2137"""
    ktf = g.nz - 1
    R = (slice(0, ktf), slice(g.jds + 1, g.jde - 1), slice(g.ids + 1, g.ide - 1))
    mpten = st["th_phy"][R] - st["h_diabatic"][R]
    qvten = st["moist"][1][R] - st["qv_diabatic"][R]
    qcten = st["moist"][2][R] - st["qc_diabatic"][R]
    st["t"][R] = st["t"][R] + mpten
    st["h_diabatic"][R] = mpten / dt
    st["qv_diabatic"][R] = qvten / dt
    st["qc_diabatic"][R] = qcten / dt


# ------------------------------------------------------------- slope parameters

def _pw(x, e):
    return np.power(x, np.asarray(e, dtype=x.dtype))


def slope_rain_vt(qr, den, denfac):
    """wrf_physics.py:1988-2003 (terminal velocity only)."""
    lam = _pw(PIDN0R / (qr * den), 0.25)
    rslope = np.where(qr <= QCRMIN, RSLOPERMAX, 1.0 / lam)
    rslopeb = np.where(qr <= QCRMIN, RSLOPERBMAX, _pw(rslope, BVTR))
    vt = PVTR * rslopeb * denfac
    return np.where(qr <= 0.0, 0.0, vt).astype(qr.dtype)


def _n0sfac(t):
    supcol = T0C - t
    return np.maximum(np.minimum(np.exp(ALPHA * supcol), N0SMAX / N0S), 1.0).astype(t.dtype)


def slope_snow_vt(qs, den, denfac, t):
    """wrf_physics.py:2005-2028 (rslopermax / rsloperbmax used for snow)."""
    lam = _pw(PIDN0S * _n0sfac(t) / (qs * den), 0.25)
    rslope = np.where(qs <= QCRMIN, RSLOPERMAX, 1.0 / lam)
    rslopeb = np.where(qs <= QCRMIN, RSLOPERBMAX, _pw(rslope, BVTS))
    vt = PVTS * rslopeb * denfac
    return np.where(qs <= 0.0, 0.0, vt).astype(qs.dtype)


def slope_graup_vt(qg, den, denfac):
    """wrf_physics.py:2030-2046"""
    lam = _pw(PIDN0G / (qg * den), 0.25)
    rslope = np.where(qg <= QCRMIN, RSLOPERMAX, 1.0 / lam)
    rslopeb = np.where(qg <= QCRMIN, RSLOPERBMAX, _pw(rslope, BVTG))
    vt = PVTG * rslopeb * denfac
    return np.where(qg <= 0.0, 0.0, vt).astype(qg.dtype)


def slope_wsm6(qrs, den, denfac, t):
    """wrf_physics.py:2048-2104: (rslope, rslopeb, rslope2, rslope3, vt) for
    rain, snow, graupel; the rain caps are used for all three species."""
    n0sfac = _n0sfac(t)
    lam = [_pw(PIDN0R / (qrs[0] * den), 0.25),
           _pw(PIDN0S * n0sfac / (qrs[1] * den), 0.25),
           _pw(PIDN0G / (qrs[2] * den), 0.25)]
    bexp = [BVTR, BVTS, BVTG]
    pv = [PVTR, PVTS, PVTG]
    rs, rb, r2, r3, vt = [], [], [], [], []
    for m in range(3):
        small = qrs[m] <= QCRMIN
        a = np.where(small, RSLOPERMAX, 1.0 / lam[m]).astype(den.dtype)
        rs.append(a)
        rb.append(np.where(small, RSLOPERBMAX, _pw(a, bexp[m])).astype(den.dtype))
        r2.append(np.where(small, RSLOPER2MAX, a * a).astype(den.dtype))
        r3.append(np.where(small, RSLOPER3MAX, a * a * a).astype(den.dtype))
    for m in range(3):
        v = pv[m] * rb[m] * denfac
        vt.append(np.where(qrs[m] <= 0.0, 0.0, v).astype(den.dtype))
    return rs, rb, r2, r3, vt


# ------------------------------------------------------------ sedimentation

def _fall_velocity_interfaces(ww, dz, dt):
    """Interface fall speeds with the 3rd-order interpolation, the ww==0
    fallback and the downward CFL limiter (wrf_physics.py:1269-1293)."""
    km = ww.shape[0]
    wi = np.zeros((km + 1,) + ww.shape[1:], ww.dtype)
    fa1, fa2 = 9.0 / 16.0, 1.0 / 16.0
    wi[0] = ww[0]
    wi[1] = 0.5 * (ww[1] + ww[0])
    for k in range(2, km - 1):
        wi[k] = fa1 * (ww[k] + ww[k - 1]) - fa2 * (ww[k + 1] + ww[k - 2])
    wi[km - 1] = 0.5 * (ww[km - 1] + ww[km - 2])
    wi[km] = ww[km - 1]
    wi[1:km] = np.where(ww[1:km] == 0.0, ww[0:km - 1], wi[1:km])
    for k in range(km - 1, -1, -1):
        decfl = (wi[k + 1] - wi[k]) * dt / dz[k]
        wi[k] = np.where(decfl > 0.05, wi[k + 1] - 0.05 * dz[k] / dt, wi[k])
    return wi


def _remap(qa, zi, za, dz):
    """Piecewise-constant overlap remap of departure cells onto the grid
    (wrf_physics.py:1339-1357): cell tops of the last layer are 3800 m above
    its base; the top departure cell's mass is dropped (qa[km-1] = 0)."""
    km = dz.shape[0]
    zi_hi = np.concatenate([zi[1:km], zi[km - 1:km] + 3800.0])
    za_hi = np.concatenate([za[1:km], za[km - 1:km] + 3800.0])
    qn = np.zeros_like(dz)
    for ka in range(km):
        ov = np.maximum(0.0, np.minimum(zi_hi, za_hi[ka][None]) - np.maximum(zi[0:km], za[ka][None]))
        qn = qn + qa[ka][None] * ov
    return qn / dz


def _surface_flux(qa, za, dza, km):
    """Mass that left through the ground (wrf_physics.py:1361-1374)."""
    precip = np.zeros_like(qa[0])
    for k in range(km):
        c1 = (za[k] < 0.0) & (za[k + 1] < 0.0)
        precip = np.where(c1, precip + qa[k] * dza[k], precip)
        c3 = (za[k] < 0.0) & (za[k + 1] > 0.0)
        precip = np.where(c3, precip + qa[k] * (0.0 - za[k]), precip)
    return precip


def nislfv_rain_plm(den, denfac, tk, dz, ww, rq, dt, iter_):
    """wrf_physics.py:1216-1381 for one species on a column block
    ``[km, ...]``.  Returns (precip, new rq).  iter_=1: velocity re-estimated
    once from the departure-cell mixing ratio (two passes); iter_=0: one pass
    (the slope update after it is unused)."""
    km = dz.shape[0]
    allold = rq.sum(axis=0)
    zi = np.zeros((km + 1,) + dz.shape[1:], dz.dtype)
    for k in range(km):
        zi[k + 1] = zi[k] + dz[k]
    wd = ww.copy()
    www = ww.copy()
    npass = 2 if iter_ >= 1 else 1
    for n in range(1, npass + 1):
        wi = _fall_velocity_interfaces(www, dz, dt)
        za = zi - wi * dt
        dza = np.zeros_like(za)
        dza[0:km] = za[1:km + 1] - za[0:km]
        dza[km] = zi[km] - za[km]
        qa = np.zeros_like(za)
        qa[0:km] = rq * dz / dza[0:km]
        qr = qa[0:km] / den
        if n <= iter_:
            wa = slope_rain_vt(qr, den, denfac)
            www = 0.5 * (wd + wa)
    qa[km - 1] = 0.0
    qn = _remap(qa, zi, za, dz)
    precip = _surface_flux(qa, za, dza, km)
    ok = allold > 0.0
    return np.where(ok, precip, 0.0).astype(dz.dtype), np.where(ok[None], qn, 0.0).astype(dz.dtype)


def nislfv_rain_plm6(den, denfac, tk, dz, ww, rq, rq2, dt, iter_):
    """wrf_physics.py:1383-1583: snow and graupel share the mass-weighted
    fall speed; each species is then remapped separately."""
    km = dz.shape[0]
    allold = rq.sum(axis=0) + rq2.sum(axis=0)
    zi = np.zeros((km + 1,) + dz.shape[1:], dz.dtype)
    for k in range(km):
        zi[k + 1] = zi[k] + dz[k]
    wd = ww.copy()
    www = ww.copy()
    npass = 2 if iter_ >= 1 else 1
    for n in range(1, npass + 1):
        wi = _fall_velocity_interfaces(www, dz, dt)
        za = zi - wi * dt
        dza = np.zeros_like(za)
        dza[0:km] = za[1:km + 1] - za[0:km]
        dza[km] = zi[km] - za[km]
        qa = np.zeros_like(za)
        qa2 = np.zeros_like(za)
        qa[0:km] = rq * dz / dza[0:km]
        qr = qa[0:km] / den
        qa2[0:km] = rq2 * dz / dza[0:km]
        qr2 = qa2[0:km] / den
        if n <= iter_:
            wa = slope_snow_vt(qr, den, denfac, tk)
            wa2 = slope_graup_vt(qr2, den, denfac)
            tmp = np.maximum(qr + qr2, 1.0e-15)
            wa = np.where(tmp > 1.0e-15, (wa * qr + wa2 * qr2) / tmp, 0.0).astype(dz.dtype)
            www = 0.5 * (wd + wa)
    ok = allold > 0.0
    out = []
    for q in (qa, qa2):
        q = q.copy()
        q[km - 1] = 0.0
        qn = _remap(q, zi, za, dz)
        precip = _surface_flux(q, za, dza, km)
        out.append((np.where(ok, precip, 0.0).astype(dz.dtype), np.where(ok[None], qn, 0.0).astype(dz.dtype)))
    return out[0][0], out[1][0], out[0][1], out[1][1]


# ------------------------------------------------------------------- WSM6

def _fpvs(t, p, dt_):
    """Saturation mixing ratios over water (qs0) and, below the triple point,
    ice (qs1) (wrf_physics.py:246-281, 1142-1170)."""
    hsub, hvap, cvap = XLS, XLV0, CPV
    ttp = T0C + 0.01
    dldt = cvap - CLIQ
    xa = -dldt / RV
    xb = xa + hvap / (RV * ttp)
    dldti = cvap - CICE
    xai = -dldti / RV
    xbi = xai + hsub / (RV * ttp)
    tr = ttp / t
    w1 = PSAT * np.exp(np.log(tr) * xa) * np.exp(xb * (1.0 - tr))
    qs0 = np.minimum(w1, 0.99 * p)
    qs0 = EP2 * qs0 / (p - qs0)
    qs0 = np.maximum(qs0, QMIN)
    w0 = PSAT * np.exp(np.log(tr) * xai) * np.exp(xbi * (1.0 - tr))
    qs1 = np.where(t < ttp, w0, w1)
    qs1 = np.minimum(qs1, 0.99 * p)
    qs1 = EP2 * qs1 / (p - qs1)
    qs1 = np.maximum(qs1, QMIN)
    return qs0.astype(dt_), qs1.astype(dt_)


def _viscos(t, den):
    return 1.496e-6 * (t * np.sqrt(t)) / (t + 120.0) / den


def _diffus(t, p):
    return 8.794e-5 * np.exp(np.log(t) * 1.81) / p


def _xka(t, den):
    return 1.414e3 * _viscos(t, den) * den


def _diffac(a, p, t, den, qs):
    return den * a * a / (_xka(t, den) * RV * t * t) + 1.0 / (qs * _diffus(t, p))


def _venfac(p, t, den):
    return np.exp(np.log(_viscos(t, den) / _diffus(t, p)) * 0.3333333) / np.sqrt(_viscos(t, den)) * np.sqrt(np.sqrt(DEN0 / den))


def wsm6(g, th, q, qc, qr, qi, qs, qg, den, pii, p, delz, delt, rain, rainncv, snow, snowncv,
         graupel, graupelncv, sr):
    """wrf_physics.py:137-1214.  Arrays are full 3-D fields; the scheme runs
    on k in [0, nz-1), j, i in [ids+1, ide-2) and updates them in place."""
    W = lambda a: a[0:g.nz - 1, g.jds + 1:g.jde - 2, g.ids + 1:g.ide - 2]
    W2 = lambda a: a[g.jds + 1:g.jde - 2, g.ids + 1:g.ide - 2]
    dt_ = th.dtype
    with np.errstate(all="ignore"):
        _wsm6_block(W, W2, dt_, th, q, qc, qr, qi, qs, qg, den, pii, p, delz, delt,
                    rain, rainncv, snow, snowncv, graupel, graupelncv, sr)


def _wsm6_block(W, W2, dt_, th, q_, qc, qr, qi, qs, qg, den_, pii_, p_, delz_, delt,
                rain_, rainncv_, snow_, snowncv_, graupel_, graupelncv_, sr_):
    den, pii, p, delz = W(den_).copy(), W(pii_).copy(), W(p_).copy(), W(delz_).copy()
    t = W(th) * pii
    q = W(q_).copy()
    qci = [np.maximum(W(qc), 0.0).astype(dt_), np.maximum(W(qi), 0.0).astype(dt_)]
    qrs = [np.maximum(W(qr), 0.0).astype(dt_), np.maximum(W(qs), 0.0).astype(dt_), np.maximum(W(qg), 0.0).astype(dt_)]
    z = lambda: np.zeros_like(t)
    cpm = np.where(q >= QMIN, CPV * q + (1.0 - q) * CPD, CPD * (1.0 - QMIN) + CPV * QMIN).astype(dt_)
    xl = (XLV0 - XLV1 * (t - T0C)).astype(dt_)
    rainncv = np.zeros_like(W2(rainncv_))
    snowncv = np.zeros_like(rainncv)
    graupelncv = np.zeros_like(rainncv)
    srv = np.zeros_like(rainncv)
    rain = W2(rain_).copy()
    snow = W2(snow_).copy()
    graupel = W2(graupel_).copy()
    loops = max(delt / DTCLDCR, 1)
    dtcld = delt if delt <= DTCLDCR else 1.0 * delt / loops
    nloop = int(loops)
    for _ in range(nloop):
        denfac = np.sqrt(1.0 / den * DEN0)
        qs0, qs1 = _fpvs(t, p, dt_)
        rh0 = np.maximum(q / qs0, QMIN)
        rh1 = np.maximum(q / qs1, QMIN)
        temp = _pw(den * np.maximum(qci[1], QMIN), 0.75)
        xni = np.minimum(np.maximum(5.387e7 * temp, 1.0e3), 1.0e6)
        # sedimentation of rain, snow+graupel, then cloud ice
        rs, rb, r2, r3, vt = slope_wsm6(qrs, den, denfac, t)
        workr = vt[0]
        qsum = np.maximum(qrs[1] + qrs[2], 1.0e-15)
        worka = np.where(qsum > 1.0e-15, (vt[1] * qrs[1] + vt[2] * qrs[2]) / qsum, 0.0).astype(dt_)
        dq1, dq2, dq3 = den * qrs[0], den * qrs[1], den * qrs[2]
        workr = np.where(qrs[0] <= 0.0, 0.0, workr).astype(dt_)
        delq1, dq1 = nislfv_rain_plm(den, denfac, t, delz, workr, dq1, dtcld, 1)
        delq2, delq3, dq2, dq3 = nislfv_rain_plm6(den, denfac, t, delz, worka, dq2, dq3, dtcld, 1)
        qrs = [np.maximum(dq1 / den, 0.0).astype(dt_), np.maximum(dq2 / den, 0.0).astype(dt_), np.maximum(dq3 / den, 0.0).astype(dt_)]
        fall0 = [delq1 / delz[0] / dtcld, delq2 / delz[0] / dtcld, delq3 / delz[0] / dtcld]
        rs, rb, r2, r3, vt = slope_wsm6(qrs, den, denfac, t)
        xlf = XLF0
        supcol = T0C - t
        n0sfac = _n0sfac(t)
        # melting of snow and graupel
        cond = t > T0C
        work2 = np.where(cond, _venfac(p, t, den), 0.0).astype(dt_)
        c2 = (qrs[1] > 0.0) & cond
        coeres = np.where(c2, r2[1] * np.sqrt(rs[1] * rb[1]), 0.0)
        psmlt = np.where(c2, _xka(t, den) / xlf * (T0C - t) * PI / 2.0 * n0sfac * (PRECS1 * r2[1] + PRECS2 * work2 * coeres) / den, 0.0)
        psmlt = np.where(c2, np.minimum(np.maximum(psmlt * dtcld / 1.0, -qrs[1] / 1.0), 0.0), psmlt).astype(dt_)
        qrs[1] = np.where(c2, qrs[1] + psmlt, qrs[1]).astype(dt_)
        qrs[0] = np.where(c2, qrs[0] - psmlt, qrs[0]).astype(dt_)
        t = np.where(c2, t + xlf / cpm * psmlt, t).astype(dt_)
        c2 = (qrs[2] > 0.0) & cond
        coeres = np.where(c2, r2[2] * np.sqrt(rs[2] * rb[2]), 0.0)
        pgmlt = np.where(c2, _xka(t, den) / xlf * (T0C - t) * (PRECG1 * r2[2] + PRECG2 * work2 * coeres) / den, 0.0)
        pgmlt = np.where(c2, np.minimum(np.maximum(pgmlt * dtcld / 1.0, -qrs[2] / 1.0), 0.0), pgmlt).astype(dt_)
        qrs[2] = np.where(c2, qrs[2] + pgmlt, qrs[2]).astype(dt_)
        qrs[0] = np.where(c2, qrs[0] - pgmlt, qrs[0]).astype(dt_)
        t = np.where(c2, t + xlf / cpm * pgmlt, t).astype(dt_)
        # cloud-ice fall
        cond = qci[1] <= 0.0
        wt = np.maximum(np.minimum(DICON * np.sqrt(den * qci[1] / xni), DIMAX), 1.0e-25)
        wt = 1.49e4 * np.exp(np.log(wt) * 1.31)
        work1c = np.where(cond, 0.0, wt).astype(dt_)
        denqci = den * qci[1]
        delqi, denqci = nislfv_rain_plm(den, denfac, t, delz, work1c, denqci, dtcld, 0)
        qci[1] = np.maximum(denqci / den, 0.0).astype(dt_)
        fallc0 = delqi / delz[0] / dtcld
        fallsum = fall0[0] + fall0[1] + fall0[2] + fallc0
        fallsum_qsi = fall0[1] + fallc0
        fallsum_qg = fall0[2]
        acc = lambda fs: fs * delz[0] / DENR * dtcld * 1000.0
        c = fallsum > 0.0
        rainncv = np.where(c, acc(fallsum) + rainncv, rainncv)
        rain = np.where(c, acc(fallsum) + rain, rain)
        c = fallsum_qsi > 0.0
        snowncv = np.where(c, acc(fallsum_qsi) + snowncv, snowncv)
        snow = np.where(c, acc(fallsum_qsi) + snow, snow)
        c = fallsum_qg > 0.0
        graupelncv = np.where(c, acc(fallsum_qg) + graupelncv, graupelncv)
        graupel = np.where(c, acc(fallsum_qg) + graupel, graupel)
        c = fallsum > 0.0
        srv = np.where(c, (snowncv + graupelncv) / (rainncv + 1.0e-12), srv)
        # instantaneous melting / freezing
        supcol = T0C - t
        xlf3 = XLS - xl
        c = (supcol < 0.0) & (qci[1] > 0.0)
        qci[0] = np.where(c, qci[0] + qci[1], qci[0]).astype(dt_)
        t = np.where(c, t - xlf3 / cpm * qci[1], t).astype(dt_)
        qci[1] = np.where(c, 0.0, qci[1]).astype(dt_)
        c = (supcol > 40.0) & (qci[0] > 0.0)
        qci[1] = np.where(c, qci[1] + qci[0], qci[1]).astype(dt_)
        t = np.where(c, t + xlf3 / cpm * qci[0], t).astype(dt_)
        qci[0] = np.where(c, 0.0, qci[0]).astype(dt_)
        c = (supcol > 0.0) & (qci[0] > QMIN)
        pfrzdtc = np.minimum(PFRZ1 * (np.exp(PFRZ2 * np.minimum(supcol, 50.0)) - 1.0) * den / DENR / XNCR * qci[0] * qci[0] * dtcld, qci[0])
        qci[1] = np.where(c, qci[1] + pfrzdtc, qci[1]).astype(dt_)
        t = np.where(c, t + xlf3 / cpm * pfrzdtc, t).astype(dt_)
        qci[0] = np.where(c, qci[0] - pfrzdtc, qci[0]).astype(dt_)
        c = (supcol > 0.0) & (qrs[0] > 0.0)
        pfrzdtr = np.minimum(20.0 * PI * PI * PFRZ1 * N0R * DENR / den * (np.exp(PFRZ2 * np.minimum(supcol, 50.0)) - 1.0)
                             * r3[0] * r3[0] * rs[0] * dtcld, qrs[0])
        qrs[2] = np.where(c, qrs[2] + pfrzdtr, qrs[2]).astype(dt_)
        t = np.where(c, t + xlf3 / cpm * pfrzdtr, t).astype(dt_)
        qrs[0] = np.where(c, qrs[0] - pfrzdtr, qrs[0]).astype(dt_)
        # rates
        rs, rb, r2, r3, vt = slope_wsm6(qrs, den, denfac, t)
        work1_0 = _diffac(xl, p, t, den, qs0)
        work1_1 = _diffac(XLS, p, t, den, qs1)
        work2 = _venfac(p, t, den).astype(dt_)
        supsat = np.maximum(q, QMIN) - qs0
        c = qci[0] > QC0
        praut = QCK1 * _pw(qci[0], 7.0 / 3.0)
        praut = np.where(c, np.minimum(praut, qci[0] / dtcld), 0.0)
        c = (qrs[0] > QCRMIN) & (qci[0] > QMIN)
        pracw = np.where(c, np.minimum(PACRR * r3[0] * rb[0] * qci[0] * denfac, qci[0] / dtcld), 0.0)
        c = qrs[0] > 0.0
        coeres = r2[0] * np.sqrt(rs[0] * rb[0])
        prevp = np.where(c, (rh0 - 1.0) * (PRECR1 * r2[0] + PRECR2 * work2 * coeres) / work1_0, 0.0)
        c2 = (prevp < 0.0) & c
        c3 = (prevp >= 0.0) & c
        prevp = np.where(c2, np.maximum(prevp, -qrs[0] / dtcld), prevp)
        prevp = np.where(c2, np.maximum(prevp, supsat / dtcld / 2.0), prevp)
        prevp = np.where(c3, np.minimum(prevp, supsat / dtcld / 2.0), prevp)
        supcol = T0C - t
        n0sfac = np.maximum(np.minimum(np.exp(ALPHA * supcol), N0SMAX / N0S), 1.0)
        supsat = np.maximum(q, QMIN) - qs1
        satdt = supsat / dtcld
        ifsat = np.zeros(t.shape, dtype=bool)
        wt = _pw(den * np.maximum(qci[1], QMIN), 0.75)
        xni = np.minimum(np.maximum(5.38e7 * wt, 1.0e3), 1.0e6)
        eacrs = np.exp(0.07 * (-supcol))
        xmi = den * qci[1] / xni
        diameter = np.minimum(DICON * np.sqrt(xmi), DIMAX)
        vt2i = 1.49e4 * _pw(diameter, 1.31)
        vt2r = PVTR * rb[0] * denfac
        vt2s = PVTS * rb[1] * denfac
        vt2g = PVTG * rb[2] * denfac
        qsum = np.maximum(qrs[1] + qrs[2], 1.0e-15)
        vt2ave = (vt2s * qrs[1] + vt2g * qrs[2]) / qsum
        vt2ave = np.where(qsum > 1.0e-15, vt2ave, 0.0)
        cnd = (supcol > 0.0) & (qci[1] > QMIN)
        c1 = cnd & (qrs[0] > QCRMIN)
        acrfac = 2.0 * r3[0] + 2.0 * diameter * r2[0] + diameter * diameter * rs[0]
        praci = PI * qci[1] * N0R * np.abs(vt2r - vt2i) * acrfac
        praci = np.where(c1, np.minimum(praci, qci[1] / dtcld), 0.0)
        piacr = PI ** 2 * AVTR * N0R * DENR * xni * denfac * G6PBR * (r3[0] * r3[0]) * rb[0] / 24.0 / den
        piacr = np.where(c1, np.minimum(piacr, qrs[0] / dtcld), 0.0)
        c1 = (qrs[1] > QCRMIN) & cnd
        acrfac = 2.0 * r3[1] + 2.0 * diameter * r2[1] + diameter * diameter * rs[1]
        psaci = PI * qci[1] * eacrs * N0S * n0sfac * np.abs(vt2ave - vt2i) * acrfac / 4.0
        psaci = np.where(c1, np.minimum(psaci, qci[1] / dtcld), 0.0)
        c1 = (qrs[2] > QCRMIN) & cnd
        egi = np.exp(-0.07 * supcol)
        acrfac = 2.0 * r3[2] + 2.0 * diameter * r2[2] + diameter * diameter * rs[2]
        pgaci = PI * egi * qci[1] * N0G * np.abs(vt2ave - vt2i) * acrfac / 4.0
        pgaci = np.where(c1, np.minimum(pgaci, qci[1] / dtcld), 0.0)
        c = (qrs[1] > QCRMIN) & (qci[0] > QMIN)
        psacw = np.where(c, np.minimum(PACRC * n0sfac * r3[1] * rb[1] * qci[0] * denfac, qci[0] / dtcld), 0.0)
        c = (qrs[2] > QCRMIN) & (qci[0] > QMIN)
        pgacw = np.where(c, np.minimum(PACRC * r3[2] * rb[2] * qci[0] * denfac, qci[0] / dtcld), 0.0)
        c = qsum > 1.0e-15
        paacw = np.where(c, (qrs[1] * psacw + qrs[2] * pgacw) / qsum, 0.0)
        c = (qrs[1] > QCRMIN) & (qrs[0] > QCRMIN)
        c1 = (supcol > 0) & c
        acrfac = 5.0 * (r3[1] * r3[1]) * rs[0] + 2.0 * r3[1] * r2[1] * r2[0] + 0.5 * (r2[1] * r2[1]) * r3[0]
        pracs = PI ** 2 * N0R * N0S * n0sfac * np.abs(vt2r - vt2ave) * (DENS / den) * acrfac
        pracs = np.where(c1, np.minimum(pracs, qrs[1] / dtcld), 0.0)
        acrfac = 5.0 * (r3[0] * r3[0]) * rs[1] + 2.0 * r3[0] * r2[0] * r2[1] + 0.5 * (r2[0] * r2[0]) * r3[1]
        psacr = PI ** 2 * N0R * N0S * n0sfac * np.abs(vt2r - vt2ave) * (DENR / den) * acrfac
        psacr = np.where(c, np.minimum(psacr, qrs[0] / dtcld), 0.0)
        c = (qrs[2] > QCRMIN) & (qrs[0] > QCRMIN)
        acrfac = 5.0 * (r3[0] * r3[0]) * rs[2] + 2.0 * r3[0] * r2[0] * r2[2] + 0.5 * (r2[0] * r2[0]) * r3[2]
        pgacr = PI ** 2 * N0R * N0G * np.abs(vt2r - vt2ave) * (DENR / den) * acrfac
        pgacr = np.where(c, np.minimum(pgacr, qrs[0] / dtcld), 0.0)
        pgacs = np.zeros_like(t)     # the reference zeroes it wherever it could act
        cnd = supcol <= 0.0
        c1 = cnd & (qrs[1] > 0.0)
        pseml = np.minimum(np.maximum(CLIQ * supcol * (paacw + psacr) / XLF0, -qrs[1] / dtcld), 0.0)
        pseml = np.where(c1, pseml, 0.0)
        c1 = cnd & (qrs[2] > 0.0)
        pgeml = np.minimum(np.maximum(CLIQ * supcol * (paacw + psacr) / XLF0, -qrs[2] / dtcld), 0.0)
        pgeml = np.where(c1, pgeml, 0.0)
        cnd = supcol > 0.0
        c1 = (qci[1] > 0.0) & (~ifsat) & cnd
        pidep = np.where(c1, 4.0 * diameter * xni * (rh1 - 1.0) / work1_1, 0.0)
        supice = np.where(c1, satdt - prevp, 0.0)
        c2, c3 = (pidep < 0.0) & c1, (pidep >= 0.0) & c1
        pidep = np.where(c2, np.maximum(np.maximum(np.maximum(pidep, satdt / 2), supice), -qci[1] / dtcld), pidep)
        pidep = np.where(c3, np.minimum(np.minimum(pidep, satdt / 2), supice), pidep)
        ifsat = np.where((np.abs(prevp + pidep) >= np.abs(satdt)) & c1, True, ifsat)
        c1 = (qrs[1] > 0.0) & (~ifsat) & cnd
        coeres = r2[1] * np.sqrt(rs[1] * rb[1])
        psdep = (rh1 - 1.0) * n0sfac * (PRECS1 * r2[1] + PRECS2 * work2 * coeres) / work1_1
        psdep = np.where(c1, psdep, 0.0)
        supice = np.where(c1, satdt - prevp - pidep, 0.0)
        c2, c3 = (psdep < 0.0) & c1, (psdep >= 0.0) & c1
        psdep = np.where(c2, np.maximum(np.maximum(np.maximum(psdep, -qrs[1] / dtcld), satdt / 2), supice), psdep)
        psdep = np.where(c3, np.minimum(np.minimum(psdep, satdt / 2), supice), psdep)
        ifsat = np.where((np.abs(prevp + pidep + psdep) >= np.abs(satdt)) & c1, True, ifsat)
        c1 = (qrs[2] > 0.0) & (~ifsat) & cnd
        coeres = r2[2] * np.sqrt(rs[2] * rb[2])
        pgdep = (rh1 - 1.0) * (PRECG1 * r2[2] + PRECG2 * work2 * coeres) / work1_1
        pgdep = np.where(c1, pgdep, 0.0)
        supice = np.where(c1, satdt - prevp - pidep - psdep, 0.0)
        c2, c3 = (pgdep < 0.0) & c1, (pgdep >= 0.0) & c1
        pgdep = np.where(c2, np.maximum(np.maximum(np.maximum(pgdep, -qrs[2] / dtcld), satdt / 2), supice), pgdep)
        pgdep = np.where(c3, np.minimum(np.minimum(pgdep, satdt / 2), supice), pgdep)
        ifsat = np.where((np.abs(prevp + pidep + psdep + pgdep) >= np.abs(satdt)) & c1, True, ifsat)
        c1 = (supsat > 0.0) & (~ifsat) & cnd
        supice = satdt - prevp - pidep - psdep - pgdep
        roqi0 = 4.92e-11 * _pw(1.0e3 * np.exp(0.1 * supcol), 1.33)
        pigen = np.maximum(0.0, (roqi0 / den - np.maximum(qci[1], 0.0)) / dtcld)
        pigen = np.minimum(np.minimum(pigen, satdt), supice)
        pigen = np.where(c1, pigen, 0.0)
        c1 = (qci[1] > 0.0) & cnd
        psaut = np.where(c1, np.maximum(0.0, (qci[1] - ROQIMAX / den) / dtcld), 0.0)
        c1 = (qrs[1] > 0.0) & cnd
        pgaut = np.minimum(np.maximum(0.0, 1.0e-3 * np.exp(-0.09 * supcol) * (qrs[1] - QS0)), qrs[1] / dtcld)
        pgaut = np.where(c1, pgaut, 0.0)
        cnd = supcol < 0.0
        c1 = (qrs[1] > 0.0) & (rh0 < 1.0) & cnd
        coeres = r2[1] * np.sqrt(rs[1] * rb[1])
        psevp = (rh0 - 1.0) * n0sfac * (PRECS1 * r2[1] + PRECS2 * work2 * coeres) / work1_0
        psevp = np.where(c1, np.minimum(np.maximum(psevp, -qrs[1] / dtcld), 0.0), 0.0)
        c1 = (qrs[2] > 0.0) & (rh0 < 1.0) & cnd
        coeres = r2[2] * np.sqrt(rs[2] * rb[2])
        pgevp = (rh0 - 1.0) * (PRECG1 * r2[2] + PRECG2 * work2 * coeres) / work1_0
        pgevp = np.where(c1, np.minimum(np.maximum(pgevp, -qrs[2] / dtcld), 0.0), 0.0)
        # mass-conservation limiters and update, T <= t0c
        delta2 = np.where((qrs[0] < 1.0e-4) & (qrs[1] < 1.0e-4), 1.0, 0.0).astype(dt_)
        delta3 = np.where(qrs[0] < 1.0e-4, 1.0, 0.0).astype(dt_)
        cnd = t <= T0C

        def limit(value, source, cnd_, rates):
            c1_ = (source > value) & cnd_
            factor = value / source
            return [np.where(c1_, r * factor, r) for r in rates]

        praut, pracw, paacw = limit(np.maximum(QMIN, qci[0]), (praut + pracw + paacw + paacw) * dtcld, cnd, [praut, pracw, paacw])
        psaut, pigen, pidep, praci, psaci, pgaci = limit(np.maximum(QMIN, qci[1]), (psaut - pigen - pidep + praci + psaci + pgaci) * dtcld, cnd,
                                                         [psaut, pigen, pidep, praci, psaci, pgaci])
        praut, prevp, pracw, piacr, psacr, pgacr = limit(np.maximum(QMIN, qrs[0]), (-praut - prevp - pracw + piacr + psacr + pgacr) * dtcld, cnd,
                                                         [praut, prevp, pracw, piacr, psacr, pgacr])
        src = -(psdep + psaut - pgaut + paacw + piacr * delta3 + praci * delta3 - pracs * (1.0 - delta2) + psacr * delta2 + psaci - pgacs) * dtcld
        psdep, psaut, pgaut, paacw, piacr, praci, psaci, pracs, psacr, pgacs = limit(
            np.maximum(QMIN, qrs[1]), src, cnd, [psdep, psaut, pgaut, paacw, piacr, praci, psaci, pracs, psacr, pgacs])
        src = -(pgdep + pgaut + piacr * (1.0 - delta3) + praci * (1.0 - delta3) + psacr * (1.0 - delta2) + pracs * (1.0 - delta2)
                + pgaci + paacw + pgacr + pgacs) * dtcld
        pgdep, pgaut, piacr, praci, psacr, pracs, paacw, pgaci, pgacr, pgacs = limit(
            np.maximum(QMIN, qrs[2]), src, cnd, [pgdep, pgaut, piacr, praci, psacr, pracs, paacw, pgaci, pgacr, pgacs])
        work2 = np.where(cnd, -(prevp + psdep + pgdep + pigen + pidep), work2)
        q = np.where(cnd, q + work2 * dtcld, q).astype(dt_)
        qci[0] = np.where(cnd, np.maximum(qci[0] - (praut + pracw + paacw + paacw) * dtcld, 0.0), qci[0]).astype(dt_)
        qrs[0] = np.where(cnd, np.maximum(qrs[0] + (praut + pracw + prevp - piacr - pgacr - psacr) * dtcld, 0.0), qrs[0]).astype(dt_)
        qci[1] = np.where(cnd, np.maximum(qci[1] - (psaut + praci + psaci + pgaci - pigen - pidep) * dtcld, 0.0), qci[1]).astype(dt_)
        qrs[1] = np.where(cnd, np.maximum(qrs[1] + (psdep + psaut + paacw - pgaut + piacr * delta3 + praci * delta3 + psaci - pgacs
                                                    - pracs * (1.0 - delta2) + psacr * delta2) * dtcld, 0.0), qrs[1]).astype(dt_)
        qrs[2] = np.where(cnd, np.maximum(qrs[2] + (pgdep + pgaut + piacr * (1.0 - delta3) + praci * (1.0 - delta3) + psacr * (1.0 - delta2)
                                                    + pracs * (1.0 - delta2) + pgaci + paacw + pgacr + pgacs) * dtcld, 0.0), qrs[2]).astype(dt_)
        xlf3 = XLS - xl
        xlwork2 = -XLS * (psdep + pgdep + pidep + pigen) - xl * prevp - xlf3 * (piacr + paacw + paacw + pgacr + psacr)
        t = np.where(cnd, t - xlwork2 / cpm * dtcld, t).astype(dt_)
        # T > t0c
        cnd = t > T0C
        praut, pracw, paacw = limit(np.maximum(QMIN, qci[0]), (praut + pracw + paacw + paacw) * dtcld, cnd, [praut, pracw, paacw])
        praut, prevp, pracw, paacw, pseml, pgeml = limit(np.maximum(QMIN, qrs[0]), (-paacw - praut + pseml + pgeml - pracw - paacw - prevp) * dtcld,
                                                         cnd, [praut, prevp, pracw, paacw, pseml, pgeml])
        pgacs, psevp, pseml = limit(np.maximum(QCRMIN, qrs[1]), (pgacs - pseml - psevp) * dtcld, cnd, [pgacs, psevp, pseml])
        pgacs, pgevp, pgeml = limit(np.maximum(QCRMIN, qrs[2]), -(pgacs + pgevp + pgeml) * dtcld, cnd, [pgacs, pgevp, pgeml])
        work2 = np.where(cnd, -(prevp + psevp + pgevp), work2)
        q = np.where(cnd, q + work2 * dtcld, q).astype(dt_)
        qci[0] = np.where(cnd, np.maximum(qci[0] - (praut + pracw + paacw + paacw) * dtcld, 0.0), qci[0]).astype(dt_)
        qrs[0] = np.where(cnd, np.maximum(qrs[0] + (praut + pracw + prevp + paacw + paacw - pseml - pgeml) * dtcld, 0.0), qrs[0]).astype(dt_)
        qrs[1] = np.where(cnd, np.maximum(qrs[1] + (psevp - pgacs + pseml) * dtcld, 0.0), qrs[1]).astype(dt_)
        qrs[2] = np.where(cnd, np.maximum(qrs[2] + (pgacs + pgevp + pgeml) * dtcld, 0.0), qrs[2]).astype(dt_)
        xlf3 = XLS - xl
        xlwork2 = -xl * (prevp + psevp + pgevp) - xlf3 * (pseml + pgeml)
        t = np.where(cnd, t - xlwork2 / cpm * dtcld, t).astype(dt_)
        # saturation adjustment
        qs0, qs1 = _fpvs(t, p, dt_)
        w1 = (np.maximum(q, QMIN) - qs0) / (1.0 + xl * xl / (RV * cpm) * qs0 / (t * t))
        pcond = np.minimum(np.maximum(w1 / dtcld, 0.0), np.maximum(q, 0.0) / dtcld)
        c = (qci[0] > 0.0) & (w1 < 0.0)
        pcond = np.where(c, np.maximum(w1, -qci[0]) / dtcld, pcond)
        q = (q - pcond * dtcld).astype(dt_)
        qci[0] = np.maximum(qci[0] + pcond * dtcld, 0.0).astype(dt_)
        t = (t + pcond * xl / cpm * dtcld).astype(dt_)
        qci[0] = np.where(qci[0] <= QMIN, 0.0, qci[0]).astype(dt_)
        qci[1] = np.where(qci[1] <= QMIN, 0.0, qci[1]).astype(dt_)
    W(th)[...] = t / pii
    W(q_)[...] = q
    W(qc)[...] = qci[0]
    W(qi)[...] = qci[1]
    W(qr)[...] = qrs[0]
    W(qs)[...] = qrs[1]
    W(qg)[...] = qrs[2]
    W2(rain_)[...] = rain
    W2(rainncv_)[...] = rainncv
    W2(snow_)[...] = snow
    W2(snowncv_)[...] = snowncv
    W2(graupel_)[...] = graupel
    W2(graupelncv_)[...] = graupelncv
    W2(sr_)[...] = srv
