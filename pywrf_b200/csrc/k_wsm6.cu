// WSM6 single-moment 6-class microphysics and the moist-physics wrappers.
//
// k_physics runs one thread per (j, i) column of [jds, jde-1) x [ids, ide-1)
// and fuses, column by column:
//   moist_physics_prep_em   (wrf_physics.py:27-91, columns [ids+1, ide-1))
//   wsm6                    (wrf_physics.py:137-1214, columns [ids+1, ide-2))
//   moist_physics_finish_em (wrf_physics.py:2106-2137)
//   calc_p_rho_phi          (wrf_dynamics.py:4124-4164, every column)
// so theta, density, Exner function and layer depths never leave the SM.
// Sedimentation follows nislfv_rain_plm / _plm6 (wrf_physics.py:1216-1583):
// 3rd-order interface fall speeds with the CFL limiter, departure cells,
// piecewise-constant overlap remap (the top cell 3800 m deep, the top
// departure cell's mass dropped) and the surface flux.
//
// Arithmetic is IEEE float32 in the reference's operation order; constant
// sub-expressions the reference forms from python floats are formed in double
// and rounded once, as the reference does.
#include "kernels.cuh"

namespace wrf {
namespace mp {
constexpr double CPD = 1004.5, CPV = 1846.4, RV = 461.6, QMIN = 1.0e-15;
constexpr double XLS = 2850000.0, XLV0 = 2500000.0, XLF0 = 350000.0, DEN0 = 1.28, DENR = 1000.0;
constexpr double CLIQ = 4190.0, CICE = 2106.0, PSAT = 610.78, RCP = 0.2857143;
constexpr double T0C = 273.149993896484375, EP2 = 0.621750414371490479;
constexpr double DTCLDCR = 120.0, N0R = 8.0e6, AVTR = 841.9, QCRMIN = 1.0e-9, N0SMAX = 1.0e11, N0S = 2.0e6;
constexpr double ALPHA = 0.12, PFRZ1 = 100.0, PFRZ2 = 0.66, XNCR = 3.0e8, DICON = 11.9, DIMAX = 500.0e-6;
constexpr double DENS = 100.0, QS0 = 6.0e-4, QC0 = 5.0265482e-04, QCK1 = 6.773895, BVTR = 0.8, G6PBR = 495.4590;
constexpr double PVTR = 2500.064, PACRR = 2.4813369e10, PRECR1 = 3.9207076e07, PRECR2 = 8.2585357e08;
constexpr double ROQIMAX = 8.1250037e-05, BVTS = 0.41, N0G = 4000000.0, BVTG = 0.8, PVTS = 20.05161;
constexpr double PRECS1 = 5200000.0, PRECS2 = 1.8681944e07, PIDN0R = 2.5132743e10, PIDN0S = 6.2831853e08;
constexpr double XLV1 = 2343.6, PACRC = 5.5442112e07, PI = 3.141593, PVTG = 979.9514;
constexpr double PRECG1 = 1.9603538e07, PRECG2 = 2.5852333e08, PIDN0G = 6.2831857e09;
constexpr double RSLOPERMAX = 1.2500000e-05, RSLOPERBMAX = 1.1954404e-04, RSLOPER2MAX = 1.5624999e-10;
constexpr double RSLOPER3MAX = 1.9531248e-15;
}  // namespace mp
#define F(x) ((float)(x))

// slope parameters of rain (0), snow (1), graupel (2)
struct Slope { float rs[3], rb[3], r2[3], r3[3], vt[3]; };

__device__ __forceinline__ float n0sfac_of(float t) {
  return fmaxf(fminf(wexp(F(mp::ALPHA) * (F(mp::T0C) - t)), F(mp::N0SMAX / mp::N0S)), 1.0f);
}

// slope_wsm6 (wrf_physics.py:2048-2104); the rain caps serve all species
__device__ __forceinline__ void slope_point(float q0, float q1, float q2, float den, float denfac, float t, Slope& o) {
  const float n0 = n0sfac_of(t);
  const float lam[3] = {wpow(F(mp::PIDN0R) / (q0 * den), 0.25f), wpow(F(mp::PIDN0S) * n0 / (q1 * den), 0.25f),
                        wpow(F(mp::PIDN0G) / (q2 * den), 0.25f)};
  const float be[3] = {F(mp::BVTR), F(mp::BVTS), F(mp::BVTG)};
  const float pv[3] = {F(mp::PVTR), F(mp::PVTS), F(mp::PVTG)};
  const float qq[3] = {q0, q1, q2};
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const bool small = qq[m] <= F(mp::QCRMIN);
    const float a = small ? F(mp::RSLOPERMAX) : 1.0f / lam[m];
    o.rs[m] = a;
    o.rb[m] = small ? F(mp::RSLOPERBMAX) : wpow(a, be[m]);
    o.r2[m] = small ? F(mp::RSLOPER2MAX) : a * a;
    o.r3[m] = small ? F(mp::RSLOPER3MAX) : a * a * a;
    const float v = pv[m] * o.rb[m] * denfac;
    o.vt[m] = qq[m] <= 0.f ? 0.f : v;
  }
}

// terminal velocities alone (wrf_physics.py:1988-2046)
__device__ __forceinline__ float vt_rain(float qr, float den, float denfac) {
  const float lam = wpow(F(mp::PIDN0R) / (qr * den), 0.25f);
  const float rs = qr <= F(mp::QCRMIN) ? F(mp::RSLOPERMAX) : 1.0f / lam;
  const float rb = qr <= F(mp::QCRMIN) ? F(mp::RSLOPERBMAX) : wpow(rs, F(mp::BVTR));
  const float v = F(mp::PVTR) * rb * denfac;
  return qr <= 0.f ? 0.f : v;
}
__device__ __forceinline__ float vt_snow(float qs, float den, float denfac, float t) {
  const float lam = wpow(F(mp::PIDN0S) * n0sfac_of(t) / (qs * den), 0.25f);
  const float rs = qs <= F(mp::QCRMIN) ? F(mp::RSLOPERMAX) : 1.0f / lam;
  const float rb = qs <= F(mp::QCRMIN) ? F(mp::RSLOPERBMAX) : wpow(rs, F(mp::BVTS));
  const float v = F(mp::PVTS) * rb * denfac;
  return qs <= 0.f ? 0.f : v;
}
__device__ __forceinline__ float vt_graup(float qg, float den, float denfac) {
  const float lam = wpow(F(mp::PIDN0G) / (qg * den), 0.25f);
  const float rs = qg <= F(mp::QCRMIN) ? F(mp::RSLOPERMAX) : 1.0f / lam;
  const float rb = qg <= F(mp::QCRMIN) ? F(mp::RSLOPERBMAX) : wpow(rs, F(mp::BVTG));
  const float v = F(mp::PVTG) * rb * denfac;
  return qg <= 0.f ? 0.f : v;
}

// per-column working storage (thread-local; km <= kMaxNz levels)
struct Column {
  float t[kMaxNz], q[kMaxNz], qc0[kMaxNz], qc1[kMaxNz], qr0[kMaxNz], qr1[kMaxNz], qr2[kMaxNz];
  float den[kMaxNz], p[kMaxNz], delz[kMaxNz];
  float denfac[kMaxNz], cpm[kMaxNz], xl[kMaxNz], qs0[kMaxNz], qs1[kMaxNz];
  float rs0[kMaxNz], r30[kMaxNz];          // rain slope after sedimentation (rain freezing)
  float ww[kMaxNz], ww2[kMaxNz], rq[kMaxNz], rq2[kMaxNz], rq3[kMaxNz];
  // sedimentation scratch
  float zi[kMaxNz + 1], wi[kMaxNz + 1], za[kMaxNz + 1], dza[kMaxNz + 1];
  float qa[kMaxNz + 1], qa2[kMaxNz + 1], www[kMaxNz], qn[kMaxNz];
};

// interface fall speeds (wrf_physics.py:1269-1293)
__device__ void fall_interfaces(const float* ww, const float* dz, int km, float dt, float* wi) {
  const float fa1 = 9.0f / 16.0f, fa2 = 1.0f / 16.0f;
  wi[0] = ww[0];
  wi[1] = 0.5f * (ww[1] + ww[0]);
  for (int k = 2; k < km - 1; ++k) wi[k] = fa1 * (ww[k] + ww[k - 1]) - fa2 * (ww[k + 1] + ww[k - 2]);
  wi[km - 1] = 0.5f * (ww[km - 1] + ww[km - 2]);
  wi[km] = ww[km - 1];
  for (int k = 1; k < km; ++k)
    if (ww[k] == 0.0f) wi[k] = ww[k - 1];
  for (int k = km - 1; k >= 0; --k) {
    const float decfl = (wi[k + 1] - wi[k]) * dt / dz[k];
    if (decfl > 0.05f) wi[k] = wi[k + 1] - 0.05f * dz[k] / dt;
  }
}

// overlap remap (wrf_physics.py:1339-1357): qn[k] = sum_ka qa[ka] * overlap / dz[k],
// summed in ka order
__device__ void remap(const float* qa, const float* zi, const float* za, const float* dz, int km, float* qn) {
  for (int k = 0; k < km; ++k) {
    const float lo = zi[k];
    const float hi = (k < km - 1) ? zi[k + 1] : zi[km - 1] + 3800.0f;
    float acc = 0.f;
    for (int ka = 0; ka < km; ++ka) {
      const float alo = za[ka];
      const float ahi = (ka < km - 1) ? za[ka + 1] : za[km - 1] + 3800.0f;
      const float ov = fmaxf(0.0f, fminf(hi, ahi) - fmaxf(lo, alo));
      acc = acc + qa[ka] * ov;
    }
    qn[k] = acc / dz[k];
  }
}

// mass that left through the ground (wrf_physics.py:1361-1374)
__device__ float surface_flux(const float* qa, const float* za, const float* dza, int km) {
  float precip = 0.f;
  for (int k = 0; k < km; ++k) {
    if (za[k] < 0.f && za[k + 1] < 0.f) precip = precip + qa[k] * dza[k];
    if (za[k] < 0.f && za[k + 1] > 0.f) precip = precip + qa[k] * (0.0f - za[k]);
  }
  return precip;
}

__device__ void departure(Column& c, int km, float dt) {
  fall_interfaces(c.www, c.delz, km, dt, c.wi);
  for (int k = 0; k <= km; ++k) c.za[k] = c.zi[k] - c.wi[k] * dt;
  for (int k = 0; k < km; ++k) c.dza[k] = c.za[k + 1] - c.za[k];
  c.dza[km] = c.zi[km] - c.za[km];
}

// nislfv_rain_plm (wrf_physics.py:1216-1381) on rq with fall speed ww;
// iter 1 re-estimates the fall speed once from the departure cells
__device__ float nislfv_plm(Column& c, const float* ww, float* rq, int km, float dt, int iter) {
  float allold = 0.f;
  for (int k = 0; k < km; ++k) allold = allold + rq[k];
  c.zi[0] = 0.f;
  for (int k = 0; k < km; ++k) c.zi[k + 1] = c.zi[k] + c.delz[k];
  for (int k = 0; k < km; ++k) c.www[k] = ww[k];
  const int npass = iter >= 1 ? 2 : 1;
  for (int n = 1; n <= npass; ++n) {
    departure(c, km, dt);
    for (int k = 0; k < km; ++k) c.qa[k] = rq[k] * c.delz[k] / c.dza[k];
    c.qa[km] = 0.f;
    if (n <= iter) {
      for (int k = 0; k < km; ++k) {
        const float qr = c.qa[k] / c.den[k];
        c.www[k] = 0.5f * (ww[k] + vt_rain(qr, c.den[k], c.denfac[k]));
      }
    }
  }
  c.qa[km - 1] = 0.f;
  remap(c.qa, c.zi, c.za, c.delz, km, c.qn);
  const float precip = surface_flux(c.qa, c.za, c.dza, km);
  const bool ok = allold > 0.f;
  for (int k = 0; k < km; ++k) rq[k] = ok ? c.qn[k] : 0.f;
  return ok ? precip : 0.f;
}

// nislfv_rain_plm6 (wrf_physics.py:1383-1583): snow and graupel move with the
// shared mass-weighted fall speed, then each is remapped separately
__device__ void nislfv_plm6(Column& c, const float* ww, float* rq, float* rq2, int km, float dt, int iter,
                            float* p1, float* p2) {
  float allold = 0.f, a2 = 0.f;
  for (int k = 0; k < km; ++k) allold = allold + rq[k];
  for (int k = 0; k < km; ++k) a2 = a2 + rq2[k];
  allold = allold + a2;
  c.zi[0] = 0.f;
  for (int k = 0; k < km; ++k) c.zi[k + 1] = c.zi[k] + c.delz[k];
  for (int k = 0; k < km; ++k) c.www[k] = ww[k];
  const int npass = iter >= 1 ? 2 : 1;
  for (int n = 1; n <= npass; ++n) {
    departure(c, km, dt);
    for (int k = 0; k < km; ++k) {
      c.qa[k] = rq[k] * c.delz[k] / c.dza[k];
      c.qa2[k] = rq2[k] * c.delz[k] / c.dza[k];
    }
    c.qa[km] = 0.f;
    c.qa2[km] = 0.f;
    if (n <= iter) {
      for (int k = 0; k < km; ++k) {
        const float qr = c.qa[k] / c.den[k], qr2 = c.qa2[k] / c.den[k];
        float wa = vt_snow(qr, c.den[k], c.denfac[k], c.t[k]);
        const float wa2 = vt_graup(qr2, c.den[k], c.denfac[k]);
        const float tmp = fmaxf(qr + qr2, 1.0e-15f);
        wa = tmp > 1.0e-15f ? (wa * qr + wa2 * qr2) / tmp : 0.f;
        c.www[k] = 0.5f * (ww[k] + wa);
      }
    }
  }
  const bool ok = allold > 0.f;
  c.qa[km - 1] = 0.f;
  remap(c.qa, c.zi, c.za, c.delz, km, c.qn);
  *p1 = ok ? surface_flux(c.qa, c.za, c.dza, km) : 0.f;
  for (int k = 0; k < km; ++k) rq[k] = ok ? c.qn[k] : 0.f;
  c.qa2[km - 1] = 0.f;
  remap(c.qa2, c.zi, c.za, c.delz, km, c.qn);
  *p2 = ok ? surface_flux(c.qa2, c.za, c.dza, km) : 0.f;
  for (int k = 0; k < km; ++k) rq2[k] = ok ? c.qn[k] : 0.f;
}

// saturation mixing ratios over water and (below the triple point) ice
// (wrf_physics.py:246-281)
__device__ __forceinline__ void fpvs(float t, float p, float& qs0, float& qs1) {
  const double ttp = mp::T0C + 0.01;
  const double dldt = mp::CPV - mp::CLIQ, xa = -dldt / mp::RV, xb = xa + mp::XLV0 / (mp::RV * ttp);
  const double dldti = mp::CPV - mp::CICE, xai = -dldti / mp::RV, xbi = xai + mp::XLS / (mp::RV * ttp);
  const float tr = F(ttp) / t;
  const float w1 = F(mp::PSAT) * wexp(wlog(tr) * F(xa)) * wexp(F(xb) * (1.0f - tr));
  float a = fminf(w1, 0.99f * p);
  a = F(mp::EP2) * a / (p - a);
  qs0 = fmaxf(a, F(mp::QMIN));
  const float w0 = F(mp::PSAT) * wexp(wlog(tr) * F(xai)) * wexp(F(xbi) * (1.0f - tr));
  float b = t < F(ttp) ? w0 : w1;
  b = fminf(b, 0.99f * p);
  b = F(mp::EP2) * b / (p - b);
  qs1 = fmaxf(b, F(mp::QMIN));
}

__device__ __forceinline__ float viscos(float t, float den) { return 1.496e-6f * (t * sqrtf(t)) / (t + 120.0f) / den; }
__device__ __forceinline__ float diffus(float t, float p) { return 8.794e-5f * wexp(wlog(t) * 1.81f) / p; }
__device__ __forceinline__ float xka(float t, float den) { return 1.414e3f * viscos(t, den) * den; }
__device__ __forceinline__ float diffac(float a, float p, float t, float den, float qs) {
  return den * a * a / (xka(t, den) * F(mp::RV) * t * t) + 1.0f / (qs * diffus(t, p));
}
__device__ __forceinline__ float venfac(float p, float t, float den) {
  return wexp(wlog(viscos(t, den) / diffus(t, p)) * 0.3333333f) / sqrtf(viscos(t, den)) *
         sqrtf(sqrtf(F(mp::DEN0) / den));
}

// Point processes after the sedimentation (wrf_physics.py:518-1203):
// instantaneous melting/freezing, the source/sink rates, the mass-conserving
// limiters and update for T <= t0c then T > t0c, saturation adjustment.
__device__ void wsm6_point(float& t, float& q, float& qc0, float& qc1, float& qr0, float& qr1, float& qr2,
                           const float den, const float p, const float denfac, const float cpm, const float xl,
                           const float qs0, const float qs1, const float rs0pre, const float r30pre,
                           const float dtcld) {
  const float t0c = F(mp::T0C);
  const float rh0 = fmaxf(q / qs0, F(mp::QMIN));
  const float rh1 = fmaxf(q / qs1, F(mp::QMIN));
  // instantaneous melting / freezing (one supcol for all four)
  float supcol = t0c - t;
  {
    const float xlf3 = F(mp::XLS) - xl;
    if (supcol < 0.f && qc1 > 0.f) {
      qc0 = qc0 + qc1;
      t = t - xlf3 / cpm * qc1;
      qc1 = 0.f;
    }
    if (supcol > 40.f && qc0 > 0.f) {
      qc1 = qc1 + qc0;
      t = t + xlf3 / cpm * qc0;
      qc0 = 0.f;
    }
    const float pfrzdtc = fminf(F(mp::PFRZ1) * (wexp(F(mp::PFRZ2) * fminf(supcol, 50.0f)) - 1.0f) * den / F(mp::DENR) /
                                    F(mp::XNCR) * qc0 * qc0 * dtcld, qc0);
    if (supcol > 0.f && qc0 > F(mp::QMIN)) {
      qc1 = qc1 + pfrzdtc;
      t = t + xlf3 / cpm * pfrzdtc;
      qc0 = qc0 - pfrzdtc;
    }
    const float pfrzdtr = fminf(F(20.0 * mp::PI * mp::PI * mp::PFRZ1 * mp::N0R * mp::DENR) / den *
                                    (wexp(F(mp::PFRZ2) * fminf(supcol, 50.0f)) - 1.0f) * r30pre * r30pre * rs0pre * dtcld, qr0);
    if (supcol > 0.f && qr0 > 0.f) {
      qr2 = qr2 + pfrzdtr;
      t = t + xlf3 / cpm * pfrzdtr;
      qr0 = qr0 - pfrzdtr;
    }
  }
  Slope sl;
  slope_point(qr0, qr1, qr2, den, denfac, t, sl);
  const float work1_0 = diffac(xl, p, t, den, qs0);
  const float work1_1 = diffac(F(mp::XLS), p, t, den, qs1);
  float work2 = venfac(p, t, den);
  float supsat = fmaxf(q, F(mp::QMIN)) - qs0;
  float praut = F(mp::QCK1) * wpow(qc0, F(7.0 / 3.0));
  praut = qc0 > F(mp::QC0) ? fminf(praut, qc0 / dtcld) : 0.f;
  float pracw = (qr0 > F(mp::QCRMIN) && qc0 > F(mp::QMIN))
                    ? fminf(F(mp::PACRR) * sl.r3[0] * sl.rb[0] * qc0 * denfac, qc0 / dtcld) : 0.f;
  float prevp = 0.f;
  {
    const bool c = qr0 > 0.f;
    const float coeres = sl.r2[0] * sqrtf(sl.rs[0] * sl.rb[0]);
    if (c) prevp = (rh0 - 1.0f) * (F(mp::PRECR1) * sl.r2[0] + F(mp::PRECR2) * work2 * coeres) / work1_0;
    const bool c2 = prevp < 0.f && c, c3 = prevp >= 0.f && c;
    if (c2) {
      prevp = fmaxf(prevp, -qr0 / dtcld);
      prevp = fmaxf(prevp, supsat / dtcld / 2.0f);
    }
    if (c3) prevp = fminf(prevp, supsat / dtcld / 2.0f);
  }
  supcol = t0c - t;
  const float n0sfac = fmaxf(fminf(wexp(F(mp::ALPHA) * supcol), F(mp::N0SMAX / mp::N0S)), 1.0f);
  supsat = fmaxf(q, F(mp::QMIN)) - qs1;
  const float satdt = supsat / dtcld;
  bool ifsat = false;
  const float xni = fminf(fmaxf(5.38e7f * wpow(den * fmaxf(qc1, F(mp::QMIN)), 0.75f), 1.0e3f), 1.0e6f);
  const float eacrs = wexp(0.07f * (-supcol));
  const float xmi = den * qc1 / xni;
  const float diameter = fminf(F(mp::DICON) * sqrtf(xmi), F(mp::DIMAX));
  const float vt2i = 1.49e4f * wpow(diameter, 1.31f);
  const float vt2r = F(mp::PVTR) * sl.rb[0] * denfac;
  const float vt2s = F(mp::PVTS) * sl.rb[1] * denfac;
  const float vt2g = F(mp::PVTG) * sl.rb[2] * denfac;
  const float qsum = fmaxf(qr1 + qr2, 1.0e-15f);
  float vt2ave = (vt2s * qr1 + vt2g * qr2) / qsum;
  if (!(qsum > 1.0e-15f)) vt2ave = 0.f;
  const bool cnd = supcol > 0.f && qc1 > F(mp::QMIN);
  const float pi_ = F(mp::PI);
  float praci = 0.f, piacr = 0.f, psaci = 0.f, pgaci = 0.f;
  if (cnd && qr0 > F(mp::QCRMIN)) {
    const float acrfac = 2.0f * sl.r3[0] + 2.0f * diameter * sl.r2[0] + diameter * diameter * sl.rs[0];
    praci = fminf(pi_ * qc1 * F(mp::N0R) * fabsf(vt2r - vt2i) * acrfac, qc1 / dtcld);
    piacr = fminf(F(mp::PI * mp::PI * mp::AVTR * mp::N0R * mp::DENR) * xni * denfac * F(mp::G6PBR) *
                      (sl.r3[0] * sl.r3[0]) * sl.rb[0] / 24.0f / den, qr0 / dtcld);
  }
  if (qr1 > F(mp::QCRMIN) && cnd) {
    const float acrfac = 2.0f * sl.r3[1] + 2.0f * diameter * sl.r2[1] + diameter * diameter * sl.rs[1];
    psaci = fminf(pi_ * qc1 * eacrs * F(mp::N0S) * n0sfac * fabsf(vt2ave - vt2i) * acrfac / 4.0f, qc1 / dtcld);
  }
  if (qr2 > F(mp::QCRMIN) && cnd) {
    const float egi = wexp(-0.07f * supcol);
    const float acrfac = 2.0f * sl.r3[2] + 2.0f * diameter * sl.r2[2] + diameter * diameter * sl.rs[2];
    pgaci = fminf(pi_ * egi * qc1 * F(mp::N0G) * fabsf(vt2ave - vt2i) * acrfac / 4.0f, qc1 / dtcld);
  }
  const float psacw = (qr1 > F(mp::QCRMIN) && qc0 > F(mp::QMIN))
                          ? fminf(F(mp::PACRC) * n0sfac * sl.r3[1] * sl.rb[1] * qc0 * denfac, qc0 / dtcld) : 0.f;
  const float pgacw = (qr2 > F(mp::QCRMIN) && qc0 > F(mp::QMIN))
                          ? fminf(F(mp::PACRC) * sl.r3[2] * sl.rb[2] * qc0 * denfac, qc0 / dtcld) : 0.f;
  float paacw = qsum > 1.0e-15f ? (qr1 * psacw + qr2 * pgacw) / qsum : 0.f;
  float pracs = 0.f, psacr = 0.f, pgacr = 0.f, pgacs = 0.f;  // pgacs: zero wherever it could act
  {
    const bool c = qr1 > F(mp::QCRMIN) && qr0 > F(mp::QCRMIN);
    if (supcol > 0.f && c) {
      const float acrfac = 5.0f * (sl.r3[1] * sl.r3[1]) * sl.rs[0] + 2.0f * sl.r3[1] * sl.r2[1] * sl.r2[0] +
                           0.5f * (sl.r2[1] * sl.r2[1]) * sl.r3[0];
      pracs = fminf(F(mp::PI * mp::PI * mp::N0R * mp::N0S) * n0sfac * fabsf(vt2r - vt2ave) * (F(mp::DENS) / den) * acrfac,
                    qr1 / dtcld);
    }
    if (c) {
      const float acrfac = 5.0f * (sl.r3[0] * sl.r3[0]) * sl.rs[1] + 2.0f * sl.r3[0] * sl.r2[0] * sl.r2[1] +
                           0.5f * (sl.r2[0] * sl.r2[0]) * sl.r3[1];
      psacr = fminf(F(mp::PI * mp::PI * mp::N0R * mp::N0S) * n0sfac * fabsf(vt2r - vt2ave) * (F(mp::DENR) / den) * acrfac,
                    qr0 / dtcld);
    }
    if (qr2 > F(mp::QCRMIN) && qr0 > F(mp::QCRMIN)) {
      const float acrfac = 5.0f * (sl.r3[0] * sl.r3[0]) * sl.rs[2] + 2.0f * sl.r3[0] * sl.r2[0] * sl.r2[2] +
                           0.5f * (sl.r2[0] * sl.r2[0]) * sl.r3[2];
      pgacr = fminf(F(mp::PI * mp::PI * mp::N0R * mp::N0G) * fabsf(vt2r - vt2ave) * (F(mp::DENR) / den) * acrfac,
                    qr0 / dtcld);
    }
  }
  float pseml = 0.f, pgeml = 0.f;
  if (supcol <= 0.f) {
    if (qr1 > 0.f) pseml = fminf(fmaxf(F(mp::CLIQ) * supcol * (paacw + psacr) / F(mp::XLF0), -qr1 / dtcld), 0.0f);
    if (qr2 > 0.f) pgeml = fminf(fmaxf(F(mp::CLIQ) * supcol * (paacw + psacr) / F(mp::XLF0), -qr2 / dtcld), 0.0f);
  }
  float pidep = 0.f, psdep = 0.f, pgdep = 0.f, pigen = 0.f, psaut = 0.f, pgaut = 0.f;
  const bool cold = supcol > 0.f;
  {
    const bool c1 = qc1 > 0.f && !ifsat && cold;
    float supice = 0.f;
    if (c1) {
      pidep = 4.0f * diameter * xni * (rh1 - 1.0f) / work1_1;
      supice = satdt - prevp;
    }
    if (pidep < 0.f && c1) pidep = fmaxf(fmaxf(fmaxf(pidep, satdt / 2.0f), supice), -qc1 / dtcld);
    else if (pidep >= 0.f && c1) pidep = fminf(fminf(pidep, satdt / 2.0f), supice);
    if (fabsf(prevp + pidep) >= fabsf(satdt) && c1) ifsat = true;
  }
  {
    const bool c1 = qr1 > 0.f && !ifsat && cold;
    float supice = 0.f;
    if (c1) {
      const float coeres = sl.r2[1] * sqrtf(sl.rs[1] * sl.rb[1]);
      psdep = (rh1 - 1.0f) * n0sfac * (F(mp::PRECS1) * sl.r2[1] + F(mp::PRECS2) * work2 * coeres) / work1_1;
      supice = satdt - prevp - pidep;
    }
    if (psdep < 0.f && c1) psdep = fmaxf(fmaxf(fmaxf(psdep, -qr1 / dtcld), satdt / 2.0f), supice);
    else if (psdep >= 0.f && c1) psdep = fminf(fminf(psdep, satdt / 2.0f), supice);
    if (fabsf(prevp + pidep + psdep) >= fabsf(satdt) && c1) ifsat = true;
  }
  {
    const bool c1 = qr2 > 0.f && !ifsat && cold;
    float supice = 0.f;
    if (c1) {
      const float coeres = sl.r2[2] * sqrtf(sl.rs[2] * sl.rb[2]);
      pgdep = (rh1 - 1.0f) * (F(mp::PRECG1) * sl.r2[2] + F(mp::PRECG2) * work2 * coeres) / work1_1;
      supice = satdt - prevp - pidep - psdep;
    }
    if (pgdep < 0.f && c1) pgdep = fmaxf(fmaxf(fmaxf(pgdep, -qr2 / dtcld), satdt / 2.0f), supice);
    else if (pgdep >= 0.f && c1) pgdep = fminf(fminf(pgdep, satdt / 2.0f), supice);
    if (fabsf(prevp + pidep + psdep + pgdep) >= fabsf(satdt) && c1) ifsat = true;
  }
  if (supsat > 0.f && !ifsat && cold) {
    const float supice = satdt - prevp - pidep - psdep - pgdep;
    const float roqi0 = 4.92e-11f * wpow(1.0e3f * wexp(0.1f * supcol), 1.33f);
    pigen = fmaxf(0.0f, (roqi0 / den - fmaxf(qc1, 0.0f)) / dtcld);
    pigen = fminf(fminf(pigen, satdt), supice);
  }
  if (qc1 > 0.f && cold) psaut = fmaxf(0.0f, (qc1 - F(mp::ROQIMAX) / den) / dtcld);
  if (qr1 > 0.f && cold) pgaut = fminf(fmaxf(0.0f, 1.0e-3f * wexp(-0.09f * supcol) * (qr1 - F(mp::QS0))), qr1 / dtcld);
  float psevp = 0.f, pgevp = 0.f;
  if (supcol < 0.f && rh0 < 1.0f) {
    if (qr1 > 0.f) {
      const float coeres = sl.r2[1] * sqrtf(sl.rs[1] * sl.rb[1]);
      const float v = (rh0 - 1.0f) * n0sfac * (F(mp::PRECS1) * sl.r2[1] + F(mp::PRECS2) * work2 * coeres) / work1_0;
      psevp = fminf(fmaxf(v, -qr1 / dtcld), 0.0f);
    }
    if (qr2 > 0.f) {
      const float coeres = sl.r2[2] * sqrtf(sl.rs[2] * sl.rb[2]);
      const float v = (rh0 - 1.0f) * (F(mp::PRECG1) * sl.r2[2] + F(mp::PRECG2) * work2 * coeres) / work1_0;
      pgevp = fminf(fmaxf(v, -qr2 / dtcld), 0.0f);
    }
  }
  // mass-conservation limiters and update, T <= t0c
  const float delta2 = (qr0 < 1.0e-4f && qr1 < 1.0e-4f) ? 1.0f : 0.0f;
  const float delta3 = qr0 < 1.0e-4f ? 1.0f : 0.0f;
  if (t <= t0c) {
    float value = fmaxf(F(mp::QMIN), qc0);
    float source = (praut + pracw + paacw + paacw) * dtcld;
    if (source > value) { const float f = value / source; praut *= f; pracw *= f; paacw *= f; }
    value = fmaxf(F(mp::QMIN), qc1);
    source = (psaut - pigen - pidep + praci + psaci + pgaci) * dtcld;
    if (source > value) {
      const float f = value / source;
      psaut *= f; pigen *= f; pidep *= f; praci *= f; psaci *= f; pgaci *= f;
    }
    value = fmaxf(F(mp::QMIN), qr0);
    source = (-praut - prevp - pracw + piacr + psacr + pgacr) * dtcld;
    if (source > value) {
      const float f = value / source;
      praut *= f; prevp *= f; pracw *= f; piacr *= f; psacr *= f; pgacr *= f;
    }
    value = fmaxf(F(mp::QMIN), qr1);
    source = -(psdep + psaut - pgaut + paacw + piacr * delta3 + praci * delta3 - pracs * (1.0f - delta2) +
               psacr * delta2 + psaci - pgacs) * dtcld;
    if (source > value) {
      const float f = value / source;
      psdep *= f; psaut *= f; pgaut *= f; paacw *= f; piacr *= f;
      praci *= f; psaci *= f; pracs *= f; psacr *= f; pgacs *= f;
    }
    value = fmaxf(F(mp::QMIN), qr2);
    source = -(pgdep + pgaut + piacr * (1.0f - delta3) + praci * (1.0f - delta3) + psacr * (1.0f - delta2) +
               pracs * (1.0f - delta2) + pgaci + paacw + pgacr + pgacs) * dtcld;
    if (source > value) {
      const float f = value / source;
      pgdep *= f; pgaut *= f; piacr *= f; praci *= f; psacr *= f;
      pracs *= f; paacw *= f; pgaci *= f; pgacr *= f; pgacs *= f;
    }
    work2 = -(prevp + psdep + pgdep + pigen + pidep);
    q = q + work2 * dtcld;
    qc0 = fmaxf(qc0 - (praut + pracw + paacw + paacw) * dtcld, 0.0f);
    qr0 = fmaxf(qr0 + (praut + pracw + prevp - piacr - pgacr - psacr) * dtcld, 0.0f);
    qc1 = fmaxf(qc1 - (psaut + praci + psaci + pgaci - pigen - pidep) * dtcld, 0.0f);
    qr1 = fmaxf(qr1 + (psdep + psaut + paacw - pgaut + piacr * delta3 + praci * delta3 + psaci - pgacs -
                       pracs * (1.0f - delta2) + psacr * delta2) * dtcld, 0.0f);
    qr2 = fmaxf(qr2 + (pgdep + pgaut + piacr * (1.0f - delta3) + praci * (1.0f - delta3) + psacr * (1.0f - delta2) +
                       pracs * (1.0f - delta2) + pgaci + paacw + pgacr + pgacs) * dtcld, 0.0f);
    const float xlf3 = F(mp::XLS) - xl;
    const float xlwork2 = -F(mp::XLS) * (psdep + pgdep + pidep + pigen) - xl * prevp -
                          xlf3 * (piacr + paacw + paacw + pgacr + psacr);
    t = t - xlwork2 / cpm * dtcld;
  }
  // T > t0c
  if (t > t0c) {
    float value = fmaxf(F(mp::QMIN), qc0);
    float source = (praut + pracw + paacw + paacw) * dtcld;
    if (source > value) { const float f = value / source; praut *= f; pracw *= f; paacw *= f; }
    value = fmaxf(F(mp::QMIN), qr0);
    source = (-paacw - praut + pseml + pgeml - pracw - paacw - prevp) * dtcld;
    if (source > value) {
      const float f = value / source;
      praut *= f; prevp *= f; pracw *= f; paacw *= f; pseml *= f; pgeml *= f;
    }
    value = fmaxf(F(mp::QCRMIN), qr1);
    source = (pgacs - pseml - psevp) * dtcld;
    if (source > value) { const float f = value / source; pgacs *= f; psevp *= f; pseml *= f; }
    value = fmaxf(F(mp::QCRMIN), qr2);
    source = -(pgacs + pgevp + pgeml) * dtcld;
    if (source > value) { const float f = value / source; pgacs *= f; pgevp *= f; pgeml *= f; }
    work2 = -(prevp + psevp + pgevp);
    q = q + work2 * dtcld;
    qc0 = fmaxf(qc0 - (praut + pracw + paacw + paacw) * dtcld, 0.0f);
    qr0 = fmaxf(qr0 + (praut + pracw + prevp + paacw + paacw - pseml - pgeml) * dtcld, 0.0f);
    qr1 = fmaxf(qr1 + (psevp - pgacs + pseml) * dtcld, 0.0f);
    qr2 = fmaxf(qr2 + (pgacs + pgevp + pgeml) * dtcld, 0.0f);
    const float xlf3 = F(mp::XLS) - xl;
    const float xlwork2 = -xl * (prevp + psevp + pgevp) - xlf3 * (pseml + pgeml);
    t = t - xlwork2 / cpm * dtcld;
  }
  // saturation adjustment
  float s0, s1;
  fpvs(t, p, s0, s1);
  const float w1 = (fmaxf(q, F(mp::QMIN)) - s0) / (1.0f + xl * xl / (F(mp::RV) * cpm) * s0 / (t * t));
  float pcond = fminf(fmaxf(w1 / dtcld, 0.0f), fmaxf(q, 0.0f) / dtcld);
  if (qc0 > 0.f && w1 < 0.f) pcond = fmaxf(w1, -qc0) / dtcld;
  q = q - pcond * dtcld;
  qc0 = fmaxf(qc0 + pcond * dtcld, 0.0f);
  t = t + pcond * xl / cpm * dtcld;
  if (qc0 <= F(mp::QMIN)) qc0 = 0.f;
  if (qc1 <= F(mp::QMIN)) qc1 = 0.f;
}

// precipitation accumulators of one column
struct Precip { float rain, rainncv, snow, snowncv, graupel, graupelncv, sr; };

// WSM6 on a loaded column (c.t temperature, c.q .. c.qr2, c.den, c.p, c.delz)
// (wrf_physics.py:137-1214)
__device__ void wsm6_column(Column& c, int km, float delt, Precip& pr) {
  const float t0c = F(mp::T0C);
  for (int k = 0; k < km; ++k) {
    c.qc0[k] = fmaxf(c.qc0[k], 0.0f);
    c.qc1[k] = fmaxf(c.qc1[k], 0.0f);
    c.qr0[k] = fmaxf(c.qr0[k], 0.0f);
    c.qr1[k] = fmaxf(c.qr1[k], 0.0f);
    c.qr2[k] = fmaxf(c.qr2[k], 0.0f);
    c.cpm[k] = c.q[k] >= F(mp::QMIN) ? F(mp::CPV) * c.q[k] + (1.0f - c.q[k]) * F(mp::CPD)
                                     : F(mp::CPD * (1.0 - mp::QMIN) + mp::CPV * mp::QMIN);
    c.xl[k] = F(mp::XLV0) - F(mp::XLV1) * (c.t[k] - t0c);
  }
  pr.rainncv = 0.f;
  pr.snowncv = 0.f;
  pr.graupelncv = 0.f;
  pr.sr = 0.f;
  const double loops = fmax((double)delt / mp::DTCLDCR, 1.0);
  const float dtcld = ((double)delt <= mp::DTCLDCR) ? delt : F(1.0 * (double)delt / loops);
  const int nloop = (int)loops;
  for (int loop = 0; loop < nloop; ++loop) {
    for (int k = 0; k < km; ++k) {
      c.denfac[k] = sqrtf(1.0f / c.den[k] * F(mp::DEN0));
      fpvs(c.t[k], c.p[k], c.qs0[k], c.qs1[k]);
      Slope sl;
      slope_point(c.qr0[k], c.qr1[k], c.qr2[k], c.den[k], c.denfac[k], c.t[k], sl);
      const float qsum = fmaxf(c.qr1[k] + c.qr2[k], 1.0e-15f);
      c.ww2[k] = qsum > 1.0e-15f ? (sl.vt[1] * c.qr1[k] + sl.vt[2] * c.qr2[k]) / qsum : 0.f;
      c.ww[k] = c.qr0[k] <= 0.f ? 0.f : sl.vt[0];
      c.rq[k] = c.den[k] * c.qr0[k];
      c.rq2[k] = c.den[k] * c.qr1[k];
      c.rq3[k] = c.den[k] * c.qr2[k];
    }
    // sedimentation of rain, then of snow + graupel
    const float delq1 = nislfv_plm(c, c.ww, c.rq, km, dtcld, 1);
    float delq2, delq3;
    nislfv_plm6(c, c.ww2, c.rq2, c.rq3, km, dtcld, 1, &delq2, &delq3);
    const float fall0 = delq1 / c.delz[0] / dtcld, fall1 = delq2 / c.delz[0] / dtcld;
    const float fall2 = delq3 / c.delz[0] / dtcld;
    for (int k = 0; k < km; ++k) {
      const float den = c.den[k];
      c.qr0[k] = fmaxf(c.rq[k] / den, 0.0f);
      c.qr1[k] = fmaxf(c.rq2[k] / den, 0.0f);
      c.qr2[k] = fmaxf(c.rq3[k] / den, 0.0f);
      Slope sl;
      slope_point(c.qr0[k], c.qr1[k], c.qr2[k], den, c.denfac[k], c.t[k], sl);
      c.rs0[k] = sl.rs[0];
      c.r30[k] = sl.r3[0];
      // melting of snow, then graupel
      float t = c.t[k];
      const float n0sfac = n0sfac_of(t);
      const bool cond = t > t0c;
      const float work2 = cond ? venfac(c.p[k], t, den) : 0.f;
      const float xlf = F(mp::XLF0);
      if (c.qr1[k] > 0.f && cond) {
        const float coeres = sl.r2[1] * sqrtf(sl.rs[1] * sl.rb[1]);
        float psmlt = xka(t, den) / xlf * (t0c - t) * F(mp::PI) / 2.0f * n0sfac *
                      (F(mp::PRECS1) * sl.r2[1] + F(mp::PRECS2) * work2 * coeres) / den;
        psmlt = fminf(fmaxf(psmlt * dtcld / 1.0f, -c.qr1[k] / 1.0f), 0.0f);
        c.qr1[k] = c.qr1[k] + psmlt;
        c.qr0[k] = c.qr0[k] - psmlt;
        t = t + xlf / c.cpm[k] * psmlt;
      }
      if (c.qr2[k] > 0.f && cond) {
        const float coeres = sl.r2[2] * sqrtf(sl.rs[2] * sl.rb[2]);
        float pgmlt = xka(t, den) / xlf * (t0c - t) * (F(mp::PRECG1) * sl.r2[2] + F(mp::PRECG2) * work2 * coeres) / den;
        pgmlt = fminf(fmaxf(pgmlt * dtcld / 1.0f, -c.qr2[k] / 1.0f), 0.0f);
        c.qr2[k] = c.qr2[k] + pgmlt;
        c.qr0[k] = c.qr0[k] - pgmlt;
        t = t + xlf / c.cpm[k] * pgmlt;
      }
      c.t[k] = t;
      // cloud-ice fall speed (ice number from the loop-start ice)
      const float qi = c.qc1[k];
      const float xni = fminf(fmaxf(5.387e7f * wpow(den * fmaxf(qi, F(mp::QMIN)), 0.75f), 1.0e3f), 1.0e6f);
      float wt = fmaxf(fminf(F(mp::DICON) * sqrtf(den * qi / xni), F(mp::DIMAX)), 1.0e-25f);
      wt = 1.49e4f * wexp(wlog(wt) * 1.31f);
      c.ww[k] = qi <= 0.f ? 0.f : wt;
      c.rq[k] = den * qi;
    }
    const float delqi = nislfv_plm(c, c.ww, c.rq, km, dtcld, 0);
    for (int k = 0; k < km; ++k) c.qc1[k] = fmaxf(c.rq[k] / c.den[k], 0.0f);
    const float fallc = delqi / c.delz[0] / dtcld;
    const float fallsum = fall0 + fall1 + fall2 + fallc;
    const float fallsum_qsi = fall1 + fallc;
    const float fallsum_qg = fall2;
    const float dz0 = c.delz[0];
    auto acc = [&](float fs) { return fs * dz0 / F(mp::DENR) * dtcld * 1000.0f; };
    if (fallsum > 0.f) {
      pr.rainncv = acc(fallsum) + pr.rainncv;
      pr.rain = acc(fallsum) + pr.rain;
    }
    if (fallsum_qsi > 0.f) {
      pr.snowncv = acc(fallsum_qsi) + pr.snowncv;
      pr.snow = acc(fallsum_qsi) + pr.snow;
    }
    if (fallsum_qg > 0.f) {
      pr.graupelncv = acc(fallsum_qg) + pr.graupelncv;
      pr.graupel = acc(fallsum_qg) + pr.graupel;
    }
    if (fallsum > 0.f) pr.sr = (pr.snowncv + pr.graupelncv) / (pr.rainncv + 1.0e-12f);
    for (int k = 0; k < km; ++k)
      wsm6_point(c.t[k], c.q[k], c.qc0[k], c.qc1[k], c.qr0[k], c.qr1[k], c.qr2[k], c.den[k], c.p[k], c.denfac[k],
                 c.cpm[k], c.xl[k], c.qs0[k], c.qs1[k], c.rs0[k], c.r30[k], dtcld);
  }
}

// calc_p_rho_phi at one mass point (wrf_dynamics.py:4124-4164)
__device__ __forceinline__ void eos_point(const Grid& g, const S& s, int k, size_t p, int c) {
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const float* ph = s[WF_PH];
  const float alb = s[WF_ALB][p];
  const float al = -1.0f / s[WF_MUTS][c] * (alb * s[WF_MU][c] + s[WF_RDNW][k] * (ph[p + lev] - ph[p]));
  s[WF_AL][p] = al;
  const float qvf = 1.0f + (float)RVOVRD * s[WF_MOIST][n3 + p];
  const float temp = ((float)R_D * ((float)T0 + s[WF_T][p]) * qvf) / ((float)P0 * (al + alb));
  s[WF_P][p] = wpow_eos(temp, (float)CPOVCV) * (float)P0 - s[WF_PB][p];
}

// moist_physics_prep_em + wsm6 + moist_physics_finish_em + calc_p_rho_phi
__global__ void __launch_bounds__(128) k_physics(Grid g, S s, float dt) {
  WRF_COLUMN_INDEX(g, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  if (j < jds || j >= jde - 1 || i < ids || i >= ide - 1) return;
  const int km = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const int c2 = g.i2(j, i);
  const bool prep = j >= jds + 1 && j < jde - 1 && i >= ids + 1 && i < ide - 1;
  const bool run = j >= jds + 1 && j < jde - 2 && i >= ids + 1 && i < ide - 2;
  if (run) {
    float* T = s[WF_T];
    float* qv = s[WF_MOIST] + 1 * n3;
    float* qc = s[WF_MOIST] + 2 * n3;
    Column c;
    for (int k = 0; k < km; ++k) {
      const size_t p = k * lev + c2;
      const float th = T[p] + (float)T0;
      const float pfull = s[WF_P][p] + s[WF_PB][p];
      const float pii = wpow(pfull / (float)P0, F(mp::RCP));
      c.t[k] = th * pii;
      c.den[k] = 1.0f / (s[WF_AL][p] + s[WF_ALB][p]);
      c.p[k] = pfull;
      const float zlo = (s[WF_PH][p] + s[WF_PHB][p]) / (float)G;
      const float zhi = (s[WF_PH][p + lev] + s[WF_PHB][p + lev]) / (float)G;
      c.delz[k] = zhi - zlo;
      c.q[k] = qv[p];
      c.qc0[k] = qc[p];
      c.qr0[k] = s[WF_MOIST][3 * n3 + p];
      c.qc1[k] = s[WF_MOIST][4 * n3 + p];
      c.qr1[k] = s[WF_MOIST][5 * n3 + p];
      c.qr2[k] = s[WF_MOIST][6 * n3 + p];
    }
    Precip pr{s[WF_RAINNC][c2], 0.f, s[WF_SNOWNC][c2], 0.f, s[WF_GRAUPELNC][c2], 0.f, 0.f};
    wsm6_column(c, km, dt, pr);
    for (int k = 0; k < km; ++k) {
      const size_t p = k * lev + c2;
      const float thold = T[p] + (float)T0;
      const float pii = wpow((s[WF_P][p] + s[WF_PB][p]) / (float)P0, F(mp::RCP));
      const float mpten = c.t[k] / pii - thold;
      T[p] = T[p] + mpten;
      s[WF_H_DIABATIC][p] = mpten / dt;
      s[WF_QV_DIABATIC][p] = (c.q[k] - qv[p]) / dt;
      s[WF_QC_DIABATIC][p] = (c.qc0[k] - qc[p]) / dt;
      qv[p] = c.q[k];
      qc[p] = c.qc0[k];
      s[WF_MOIST][3 * n3 + p] = c.qr0[k];
      s[WF_MOIST][4 * n3 + p] = c.qc1[k];
      s[WF_MOIST][5 * n3 + p] = c.qr1[k];
      s[WF_MOIST][6 * n3 + p] = c.qr2[k];
    }
    s[WF_RAINNC][c2] = pr.rain;
    s[WF_RAINNCV][c2] = pr.rainncv;
    s[WF_SNOWNC][c2] = pr.snow;
    s[WF_SNOWNCV][c2] = pr.snowncv;
    s[WF_GRAUPELNC][c2] = pr.graupel;
    s[WF_GRAUPELNCV][c2] = pr.graupelncv;
    s[WF_SR][c2] = pr.sr;
  } else if (prep) {
    // prepared but outside the scheme's block: zero tendencies
    for (int k = 0; k < km; ++k) {
      const size_t p = k * lev + c2;
      s[WF_H_DIABATIC][p] = 0.0f;
      s[WF_QV_DIABATIC][p] = 0.0f;
      s[WF_QC_DIABATIC][p] = 0.0f;
    }
  }
  for (int k = 0; k < km; ++k) eos_point(g, s, k, k * lev + c2, c2);
}

// stand-alone WSM6 on caller arrays: columns [ids+1, ide-2) x [jds+1, jde-2),
// levels [0, nz-1); th is potential temperature, pii the Exner function
struct Wsm6Args {
  float *th, *qv, *qc, *qr, *qi, *qs, *qg;
  const float *rho, *pii, *p, *dz8w;
  float *rainnc, *rainncv, *snownc, *snowncv, *graupelnc, *graupelncv, *sr;
};

__global__ void __launch_bounds__(128) k_wsm6(Grid g, Wsm6Args a, float delt) {
  WRF_COLUMN_INDEX(g, j, i);
  if (j < g.jds + 1 || j >= g.jde - 2 || i < g.ids + 1 || i >= g.ide - 2) return;
  const int km = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx;
  const int c2 = g.i2(j, i);
  Column c;
  for (int k = 0; k < km; ++k) {
    const size_t p = k * lev + c2;
    c.t[k] = a.th[p] * a.pii[p];
    c.den[k] = a.rho[p];
    c.p[k] = a.p[p];
    c.delz[k] = a.dz8w[p];
    c.q[k] = a.qv[p];
    c.qc0[k] = a.qc[p];
    c.qr0[k] = a.qr[p];
    c.qc1[k] = a.qi[p];
    c.qr1[k] = a.qs[p];
    c.qr2[k] = a.qg[p];
  }
  Precip pr{a.rainnc[c2], 0.f, a.snownc[c2], 0.f, a.graupelnc[c2], 0.f, 0.f};
  wsm6_column(c, km, delt, pr);
  for (int k = 0; k < km; ++k) {
    const size_t p = k * lev + c2;
    a.th[p] = c.t[k] / a.pii[p];
    a.qv[p] = c.q[k];
    a.qc[p] = c.qc0[k];
    a.qr[p] = c.qr0[k];
    a.qi[p] = c.qc1[k];
    a.qs[p] = c.qr1[k];
    a.qg[p] = c.qr2[k];
  }
  a.rainnc[c2] = pr.rain;
  a.rainncv[c2] = pr.rainncv;
  a.snownc[c2] = pr.snow;
  a.snowncv[c2] = pr.snowncv;
  a.graupelnc[c2] = pr.graupel;
  a.graupelncv[c2] = pr.graupelncv;
  a.sr[c2] = pr.sr;
}

#undef F

int launch_physics(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b(32, 4);
  k_physics<<<col_grid(g, b), b, 0, st>>>(g, s, g.dt);
  return 1;
}

// f: th qv qc qr qi qs qg rho pii p dz8w rainnc rainncv snownc snowncv graupelnc graupelncv sr
int launch_wsm6(const Grid& g, float* const* f, float delt, cudaStream_t st) {
  Wsm6Args a{f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[10],
             f[11], f[12], f[13], f[14], f[15], f[16], f[17]};
  const dim3 b(32, 4);
  k_wsm6<<<col_grid(g, b), b, 0, st>>>(g, a, delt);
  return 1;
}

}  // namespace wrf
