// WSM6 single-moment 6-class microphysics and the moist-physics wrappers.
//
// k_physics gives each (j, i) column of [jds, jde-1) x [ids, ide-1) to a
// segment of lanes (one level per lane and slot) and fuses, column by column:
//   moist_physics_prep_em   (wrf_physics.py:27-91, columns [ids+1, ide-1))
//   wsm6                    (wrf_physics.py:137-1214, columns [ids+1, ide-2))
//   moist_physics_finish_em (wrf_physics.py:2106-2137)
//   calc_p_rho_phi          (wrf_dynamics.py:4124-4164, every column)
// so theta, density, Exner function and layer depths stay in registers.
// Sedimentation follows nislfv_rain_plm / _plm6 (wrf_physics.py:1216-1583):
// 3rd-order interface fall speeds with the CFL limiter, departure cells,
// piecewise-constant overlap remap (the top cell 3800 m deep, the top
// departure cell's mass dropped) and the surface flux.
//
// Arithmetic is IEEE float32 in the reference's operation order; constant
// sub-expressions the reference forms from python floats are formed in double
// and rounded once, as the reference does.
#include <cuda.h>
#include <mutex>
#include "kernels.cuh"
#include "mlp.cuh"
#include "tc_gemm.cuh"
#include "wsm6_const.cuh"

namespace wrf {

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
// ------------------------------------------------------- warp-segment columns
//
// A segment of SEG lanes owns one column; lane l holds levels k = s*SEG + l
// (s < NS) in registers.  Point processes run on all levels at once; the
// column-coupled steps of the sedimentation (interface fall speeds, the CFL
// limiter, the overlap remap, the surface flux) use shuffles inside the
// segment and a small per-segment shared-memory scratch.  Results equal the
// reference's sequential sweeps: sums keep their order (terms that are exactly
// zero are skipped), and the backward CFL recursion is replayed exactly on the
// levels where it can act.
//
// Every function below that shuffles, ballots or syncs (shift, the *_w
// sedimentation steps, surface_flux_w, wsm6_column_w) must be reached by all
// 32 lanes of the warp: segments of one warp belong to different columns, so
// no call may sit under a per-segment condition.

constexpr unsigned kFull = 0xffffffffu;

template <int SEG, int NS>
struct Seg {
  int l;     // lane within the segment
  int base;  // first lane of the segment within the warp
  int km;    // mass levels
  __device__ __forceinline__ int k(int s) const { return s * SEG + l; }
  __device__ __forceinline__ unsigned bits(unsigned ballot) const {
    return SEG == 32 ? ballot : ((ballot >> base) & ((1u << (SEG & 31)) - 1u));
  }
};

template <int SEG, int NS>
struct SegScratch {
  float dz[NS * SEG + 1], zi[NS * SEG + 1], wi[NS * SEG + 1], za[NS * SEG + 1], qa[NS * SEG + 1],
      qa2[NS * SEG + 1];
};

template <int NS>
__device__ __forceinline__ float pick(const float (&v)[NS], int s) {
  float r = v[0];
#pragma unroll
  for (int i = 1; i < NS; ++i)
    if (s == i) r = v[i];
  return r;
}

// out[s] = value at level k(s) + d (unspecified outside [0, NS*SEG))
template <int SEG, int NS>
__device__ __forceinline__ void shift(const float (&v)[NS], int d, int l, float (&out)[NS]) {
  const int src = l + d;
  const int sl = src & (SEG - 1);
  float a[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) a[s] = __shfl_sync(kFull, v[s], sl, SEG);
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    float r = a[s];
    if (src < 0 && s > 0) r = a[s > 0 ? s - 1 : 0];
    if (src >= SEG && s < NS - 1) r = a[s < NS - 1 ? s + 1 : s];
    out[s] = r;
  }
}

// interface fall speeds into sc.wi[0..km] (wrf_physics.py:1269-1293)
template <int SEG, int NS>
__device__ void fall_interfaces_w(const Seg<SEG, NS>& g, const float (&ww)[NS], const float (&dz)[NS], float dt,
                                  SegScratch<SEG, NS>& sc) {
  const int km = g.km;
  const float fa1 = 9.0f / 16.0f, fa2 = 1.0f / 16.0f;
  float wm1[NS], wp1[NS], wm2[NS];
  shift<SEG, NS>(ww, -1, g.l, wm1);
  shift<SEG, NS>(ww, 1, g.l, wp1);
  shift<SEG, NS>(ww, -2, g.l, wm2);
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int k = g.k(s);
    if (k > km) continue;
    float w;
    if (k == 0) w = ww[s];
    else if (k == 1) w = 0.5f * (ww[s] + wm1[s]);
    else if (k == km) w = wm1[s];
    else if (k == km - 1) w = 0.5f * (ww[s] + wm1[s]);
    else w = fa1 * (ww[s] + wm1[s]) - fa2 * (wp1[s] + wm2[s]);
    if (k >= 1 && k < km && ww[s] == 0.0f) w = wm1[s];
    sc.wi[k] = w;
  }
  __syncwarp();
  // backward CFL limiter: flags computed with the unmodified upper neighbour;
  // the sequential replay visits flagged levels and every level below a
  // modified one, which is where the sequential sweep can act
  unsigned long long mask = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int k = g.k(s);
    bool f = false;
    if (k < km) f = (sc.wi[k + 1] - sc.wi[k]) * dt / dz[s] > 0.05f;
    mask |= (unsigned long long)g.bits(__ballot_sync(kFull, f)) << (s * SEG);
  }
  __syncwarp();
  if (g.l == 0 && mask) {
    int k = 63 - __clzll((long long)mask);
    while (true) {
      const float a = sc.wi[k + 1], b = sc.wi[k], dzk = sc.dz[k];
      bool modified = false;
      if ((a - b) * dt / dzk > 0.05f) {
        sc.wi[k] = a - 0.05f * dzk / dt;
        modified = true;
      }
      if (k == 0) break;
      if (modified) {
        --k;
        continue;
      }
      const unsigned long long below = mask & ((1ull << k) - 1ull);
      if (!below) break;
      k = 63 - __clzll((long long)below);
    }
  }
  __syncwarp();
}

// departure points sc.za[0..km] and the departure-cell depths of my levels
template <int SEG, int NS>
__device__ __forceinline__ void departure_w(const Seg<SEG, NS>& g, float dt, SegScratch<SEG, NS>& sc, float (&dza)[NS]) {
  const int km = g.km;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int k = g.k(s);
    if (k <= km) sc.za[k] = sc.zi[k] - sc.wi[k] * dt;
  }
  __syncwarp();
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int k = g.k(s);
    dza[s] = k < km ? sc.za[k + 1] - sc.za[k] : 1.0f;
  }
}

// overlap remap of qa (scratch) onto my levels (wrf_physics.py:1339-1357)
template <int SEG, int NS>
__device__ __forceinline__ void remap_w(const Seg<SEG, NS>& g, const float* qa, const SegScratch<SEG, NS>& sc,
                                        const float (&dz)[NS], float (&qn)[NS]) {
  const int km = g.km;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int k = g.k(s);
    qn[s] = 0.f;
    if (k >= km) continue;
    const float lo = sc.zi[k];
    const float hi = (k < km - 1) ? sc.zi[k + 1] : sc.zi[km - 1] + 3800.0f;
    // first departure cell reaching above lo: mass falls, so it is normally
    // cell k itself; walk down while the cell below still overlaps (the tops
    // za_hi are ordered, so every cell below the start has zero overlap)
    int ka0 = k;
    while (ka0 > 0 && sc.za[ka0] > lo) --ka0;
    float acc = 0.f;
    for (int ka = ka0; ka < km; ++ka) {
      const float alo = sc.za[ka];
      if (alo >= hi) break;  // departure cells are ordered: no later overlap
      const float ahi = (ka < km - 1) ? sc.za[ka + 1] : sc.za[km - 1] + 3800.0f;
      const float ov = fmaxf(0.0f, fminf(hi, ahi) - fmaxf(lo, alo));
      acc = acc + qa[ka] * ov;
    }
    qn[s] = acc / dz[s];
  }
}

// mass through the ground (wrf_physics.py:1361-1374), summed in level order
template <int SEG, int NS>
__device__ __forceinline__ float surface_flux_w(const Seg<SEG, NS>& g, const float* qa, const SegScratch<SEG, NS>& sc) {
  float precip = 0.f;
  if (g.l == 0) {
    for (int k = 0; k < g.km; ++k) {
      const float a = sc.za[k], b = sc.za[k + 1];
      if (!(a < 0.f)) break;  // ordered departure points: no later crossing
      if (b < 0.f) precip = precip + qa[k] * (b - a);
      if (b > 0.f) precip = precip + qa[k] * (0.0f - a);
    }
  }
  return __shfl_sync(kFull, precip, 0, SEG);
}

// nislfv_rain_plm (wrf_physics.py:1216-1381): rq in place, returns precip
template <int SEG, int NS>
__device__ float nislfv_w(const Seg<SEG, NS>& g, const float (&den)[NS], const float (&denfac)[NS],
                          const float (&dz)[NS], const float (&ww0)[NS], float (&rq)[NS], float dt, int iter,
                          SegScratch<SEG, NS>& sc) {
  const int km = g.km;
  bool any = false;
#pragma unroll
  for (int s = 0; s < NS; ++s) any |= (g.k(s) < km && rq[s] > 0.f);
  const unsigned wb = __ballot_sync(kFull, any);
  const bool ok = g.bits(wb) != 0u;
  // no mass in any column of the warp: the result is zero, as the full
  // path would store it
  if (wb == 0u) {
#pragma unroll
    for (int s = 0; s < NS; ++s) rq[s] = 0.f;
    return 0.f;
  }
  float www[NS], dza[NS], qa[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) www[s] = ww0[s];
  const int npass = iter >= 1 ? 2 : 1;
  for (int n = 1; n <= npass; ++n) {
    fall_interfaces_w<SEG, NS>(g, www, dz, dt, sc);
    departure_w<SEG, NS>(g, dt, sc, dza);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      qa[s] = rq[s] * dz[s] / dza[s];
      if (n <= iter && g.k(s) < km) www[s] = 0.5f * (ww0[s] + vt_rain(qa[s] / den[s], den[s], denfac[s]));
    }
    __syncwarp();
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int k = g.k(s);
    if (k < km) sc.qa[k] = (k == km - 1) ? 0.f : qa[s];
  }
  __syncwarp();
  float qn[NS];
  remap_w<SEG, NS>(g, sc.qa, sc, dz, qn);
  const float precip = surface_flux_w<SEG, NS>(g, sc.qa, sc);
#pragma unroll
  for (int s = 0; s < NS; ++s) rq[s] = ok ? qn[s] : 0.f;
  __syncwarp();
  return ok ? precip : 0.f;
}

// nislfv_rain_plm6 (wrf_physics.py:1383-1583): snow (rq) and graupel (rq2)
template <int SEG, int NS>
__device__ void nislfv6_w(const Seg<SEG, NS>& g, const float (&den)[NS], const float (&denfac)[NS],
                          const float (&tk)[NS], const float (&dz)[NS], const float (&ww0)[NS], float (&rq)[NS],
                          float (&rq2)[NS], float dt, int iter, SegScratch<SEG, NS>& sc, float* p1, float* p2) {
  const int km = g.km;
  bool any = false;
#pragma unroll
  for (int s = 0; s < NS; ++s) any |= (g.k(s) < km && (rq[s] > 0.f || rq2[s] > 0.f));
  const unsigned wb = __ballot_sync(kFull, any);
  const bool ok = g.bits(wb) != 0u;
  // no mass in any column of the warp: the results are zero, as the full
  // path would store them
  if (wb == 0u) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      rq[s] = 0.f;
      rq2[s] = 0.f;
    }
    *p1 = 0.f;
    *p2 = 0.f;
    return;
  }
  float www[NS], dza[NS], qa[NS], qa2[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) www[s] = ww0[s];
  const int npass = iter >= 1 ? 2 : 1;
  for (int n = 1; n <= npass; ++n) {
    fall_interfaces_w<SEG, NS>(g, www, dz, dt, sc);
    departure_w<SEG, NS>(g, dt, sc, dza);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      qa[s] = rq[s] * dz[s] / dza[s];
      qa2[s] = rq2[s] * dz[s] / dza[s];
      if (n <= iter && g.k(s) < km) {
        const float qr = qa[s] / den[s], qr2 = qa2[s] / den[s];
        float wa = vt_snow(qr, den[s], denfac[s], tk[s]);
        const float wa2 = vt_graup(qr2, den[s], denfac[s]);
        const float tmp = fmaxf(qr + qr2, 1.0e-15f);
        wa = tmp > 1.0e-15f ? (wa * qr + wa2 * qr2) / tmp : 0.f;
        www[s] = 0.5f * (ww0[s] + wa);
      }
    }
    __syncwarp();
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int k = g.k(s);
    if (k < km) {
      sc.qa[k] = (k == km - 1) ? 0.f : qa[s];
      sc.qa2[k] = (k == km - 1) ? 0.f : qa2[s];
    }
  }
  __syncwarp();
  float qn[NS];
  remap_w<SEG, NS>(g, sc.qa, sc, dz, qn);
  const float f1 = surface_flux_w<SEG, NS>(g, sc.qa, sc);  // all lanes: it shuffles
  *p1 = ok ? f1 : 0.f;
#pragma unroll
  for (int s = 0; s < NS; ++s) rq[s] = ok ? qn[s] : 0.f;
  remap_w<SEG, NS>(g, sc.qa2, sc, dz, qn);
  const float f2 = surface_flux_w<SEG, NS>(g, sc.qa2, sc);  // all lanes: it shuffles
  *p2 = ok ? f2 : 0.f;
#pragma unroll
  for (int s = 0; s < NS; ++s) rq2[s] = ok ? qn[s] : 0.f;
  __syncwarp();
}

// the column state a segment carries through the scheme
template <int NS>
struct WCol {
  float t[NS], q[NS], qc0[NS], qc1[NS], qr0[NS], qr1[NS], qr2[NS], den[NS], p[NS], delz[NS];
};

// WSM6 on one loaded column (wrf_physics.py:137-1214).  With kPoint false
// the column stops after the sedimentation, melting and ice fall of a single
// time-split loop and hands back the rain left by the sedimentation (qr0s),
// from which k_wsm6_finish recomputes the rain slope for the point processes.
template <int SEG, int NS, bool kPoint>
__device__ void wsm6_column_w(const Seg<SEG, NS>& g, WCol<NS>& c, float delt, Precip& pr, SegScratch<SEG, NS>& sc,
                              float (&qr0s)[NS]) {
  const int km = g.km;
  const float t0c = F(mp::T0C);
  float cpm[NS], xl[NS], denfac[NS], qs0[NS], qs1[NS], rs0[NS], r30[NS], ww[NS], ww2[NS], rq[NS], rq2[NS], rq3[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    c.qc0[s] = fmaxf(c.qc0[s], 0.0f);
    c.qc1[s] = fmaxf(c.qc1[s], 0.0f);
    c.qr0[s] = fmaxf(c.qr0[s], 0.0f);
    c.qr1[s] = fmaxf(c.qr1[s], 0.0f);
    c.qr2[s] = fmaxf(c.qr2[s], 0.0f);
    cpm[s] = c.q[s] >= F(mp::QMIN) ? F(mp::CPV) * c.q[s] + (1.0f - c.q[s]) * F(mp::CPD)
                                   : F(mp::CPD * (1.0 - mp::QMIN) + mp::CPV * mp::QMIN);
    xl[s] = F(mp::XLV0) - F(mp::XLV1) * (c.t[s] - t0c);
    const int k = g.k(s);
    if (k < km) sc.dz[k] = c.delz[s];
  }
  __syncwarp();
  if (g.l == 0) {
    float z = 0.f;
    sc.zi[0] = z;
    for (int k = 0; k < km; ++k) {
      z = z + sc.dz[k];
      sc.zi[k + 1] = z;
    }
  }
  __syncwarp();
  const float dz0 = __shfl_sync(kFull, c.delz[0], 0, SEG);
  pr.rainncv = 0.f;
  pr.snowncv = 0.f;
  pr.graupelncv = 0.f;
  pr.sr = 0.f;
  const double loops = fmax((double)delt / mp::DTCLDCR, 1.0);
  const float dtcld = ((double)delt <= mp::DTCLDCR) ? delt : F(1.0 * (double)delt / loops);
  const int nloop = (int)loops;
  for (int loop = 0; loop < nloop; ++loop) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      denfac[s] = sqrtf(1.0f / c.den[s] * F(mp::DEN0));
      fpvs(c.t[s], c.p[s], qs0[s], qs1[s]);
      Slope sl;
      slope_point(c.qr0[s], c.qr1[s], c.qr2[s], c.den[s], denfac[s], c.t[s], sl);
      const float qsum = fmaxf(c.qr1[s] + c.qr2[s], 1.0e-15f);
      ww2[s] = qsum > 1.0e-15f ? (sl.vt[1] * c.qr1[s] + sl.vt[2] * c.qr2[s]) / qsum : 0.f;
      ww[s] = c.qr0[s] <= 0.f ? 0.f : sl.vt[0];
      rq[s] = c.den[s] * c.qr0[s];
      rq2[s] = c.den[s] * c.qr1[s];
      rq3[s] = c.den[s] * c.qr2[s];
    }
    // sedimentation of rain, then of snow + graupel
    const float delq1 = nislfv_w<SEG, NS>(g, c.den, denfac, c.delz, ww, rq, dtcld, 1, sc);
    float delq2, delq3;
    nislfv6_w<SEG, NS>(g, c.den, denfac, c.t, c.delz, ww2, rq2, rq3, dtcld, 1, sc, &delq2, &delq3);
    const float fall0 = delq1 / dz0 / dtcld, fall1 = delq2 / dz0 / dtcld, fall2 = delq3 / dz0 / dtcld;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const float den = c.den[s];
      c.qr0[s] = fmaxf(rq[s] / den, 0.0f);
      c.qr1[s] = fmaxf(rq2[s] / den, 0.0f);
      c.qr2[s] = fmaxf(rq3[s] / den, 0.0f);
      qr0s[s] = c.qr0[s];
      Slope sl;
      slope_point(c.qr0[s], c.qr1[s], c.qr2[s], den, denfac[s], c.t[s], sl);
      rs0[s] = sl.rs[0];
      r30[s] = sl.r3[0];
      // melting of snow, then graupel
      float t = c.t[s];
      const float n0sfac = n0sfac_of(t);
      const bool cond = t > t0c;
      const float work2 = cond ? venfac(c.p[s], t, den) : 0.f;
      const float xlf = F(mp::XLF0);
      if (c.qr1[s] > 0.f && cond) {
        const float coeres = sl.r2[1] * sqrtf(sl.rs[1] * sl.rb[1]);
        float psmlt = xka(t, den) / xlf * (t0c - t) * F(mp::PI) / 2.0f * n0sfac *
                      (F(mp::PRECS1) * sl.r2[1] + F(mp::PRECS2) * work2 * coeres) / den;
        psmlt = fminf(fmaxf(psmlt * dtcld / 1.0f, -c.qr1[s] / 1.0f), 0.0f);
        c.qr1[s] = c.qr1[s] + psmlt;
        c.qr0[s] = c.qr0[s] - psmlt;
        t = t + xlf / cpm[s] * psmlt;
      }
      if (c.qr2[s] > 0.f && cond) {
        const float coeres = sl.r2[2] * sqrtf(sl.rs[2] * sl.rb[2]);
        float pgmlt = xka(t, den) / xlf * (t0c - t) * (F(mp::PRECG1) * sl.r2[2] + F(mp::PRECG2) * work2 * coeres) / den;
        pgmlt = fminf(fmaxf(pgmlt * dtcld / 1.0f, -c.qr2[s] / 1.0f), 0.0f);
        c.qr2[s] = c.qr2[s] + pgmlt;
        c.qr0[s] = c.qr0[s] - pgmlt;
        t = t + xlf / cpm[s] * pgmlt;
      }
      c.t[s] = t;
      // cloud-ice fall speed (ice number from the loop-start ice)
      const float qi = c.qc1[s];
      const float xni = fminf(fmaxf(5.387e7f * wpow(den * fmaxf(qi, F(mp::QMIN)), 0.75f), 1.0e3f), 1.0e6f);
      float wt = fmaxf(fminf(F(mp::DICON) * sqrtf(den * qi / xni), F(mp::DIMAX)), 1.0e-25f);
      wt = 1.49e4f * wexp(wlog(wt) * 1.31f);
      ww[s] = qi <= 0.f ? 0.f : wt;
      rq[s] = den * qi;
    }
    const float delqi = nislfv_w<SEG, NS>(g, c.den, denfac, c.delz, ww, rq, dtcld, 0, sc);
#pragma unroll
    for (int s = 0; s < NS; ++s) c.qc1[s] = fmaxf(rq[s] / c.den[s], 0.0f);
    const float fallc = delqi / dz0 / dtcld;
    const float fallsum = fall0 + fall1 + fall2 + fallc;
    const float fallsum_qsi = fall1 + fallc;
    const float fallsum_qg = fall2;
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
    if constexpr (kPoint) {
#pragma unroll
      for (int s = 0; s < NS; ++s)
        if (g.k(s) < km)
          wsm6_point(c.t[s], c.q[s], c.qc0[s], c.qc1[s], c.qr0[s], c.qr1[s], c.qr2[s], c.den[s], c.p[s], denfac[s],
                     cpm[s], xl[s], qs0[s], qs1[s], rs0[s], r30[s], dtcld);
    } else {
      (void)qs0; (void)qs1; (void)rs0; (void)r30;
      break;  // one time-split loop (the host checks nloop == 1)
    }
  }
}

// calc_p_rho_phi at one mass point (wrf_dynamics.py:4124-4164) given t, qv
__device__ __forceinline__ void eos_point(const Grid& g, const S& s, int k, size_t p, int c, float t, float qv) {
  const size_t lev = (size_t)g.ny * g.nx;
  const float* ph = s[WF_PH];
  const float alb = s[WF_ALB][p];
  const float al = -1.0f / s[WF_MUTS][c] * (alb * s[WF_MU][c] + s[WF_RDNW][k] * (ph[p + lev] - ph[p]));
  s[WF_AL][p] = al;
  const float qvf = 1.0f + (float)RVOVRD * qv;
  const float temp = ((float)R_D * ((float)T0 + t) * qvf) / ((float)P0 * (al + alb));
  s[WF_P][p] = wpow_eos(temp, (float)CPOVCV) * (float)P0 - s[WF_PB][p];
}

constexpr int kWarpsPerBlock = 8;

// dummy column for segments without a column of their own (they take part in
// the segment shuffles; nothing they compute is stored)
template <int NS>
__device__ __forceinline__ void dummy_column(WCol<NS>& c) {
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    c.t[s] = 280.f; c.q[s] = 0.f; c.qc0[s] = 0.f; c.qc1[s] = 0.f; c.qr0[s] = 0.f; c.qr1[s] = 0.f; c.qr2[s] = 0.f;
    c.den[s] = 1.f; c.p[s] = 8.0e4f; c.delz[s] = 100.f;
  }
}

// moist_physics_prep_em + wsm6 + moist_physics_finish_em + calc_p_rho_phi;
// block (x, y): SPB consecutive mass columns of row jds + y.  With kList, the
// columns are those of a list instead (list[0] entries from list[16], each
// j * nx + i of a column of the scheme's block): the fallback of the
// surrogate microphysics for the columns its gate rejected.
template <int SEG, int NS, bool kList = false>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_physics(Grid g, S s, float dt, const int* list = nullptr) {
  constexpr int SPW = 32 / SEG, SPB = kWarpsPerBlock * SPW;
  __shared__ SegScratch<SEG, NS> scratch[SPB];
  if constexpr (kList) {
    if ((int)blockIdx.x * SPB >= __ldg(list)) return;  // whole block past the list (uniform exit)
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int segw = lane / SEG;
  Seg<SEG, NS> sg;
  sg.l = lane % SEG;
  sg.base = segw * SEG;
  sg.km = g.nz - 1;
  const int km = sg.km;
  const int col = warp * SPW + segw;
  int j, i;
  bool mass, run, prep;
  if constexpr (kList) {
    const int idx = blockIdx.x * SPB + col;
    run = idx < __ldg(list);
    const int code = run ? __ldg(list + 16 + idx) : 0;
    j = code / g.nx;
    i = code - j * g.nx;
    mass = prep = run;
  } else {
    j = g.jds + blockIdx.y;
    i = g.ids + blockIdx.x * SPB + col;
    mass = i < g.ide - 1 && j < g.jde - 1;
    run = mass && j >= g.jds + 1 && j < g.jde - 2 && i >= g.ids + 1 && i < g.ide - 2;
    prep = mass && j >= g.jds + 1 && i >= g.ids + 1;
  }
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const int c2 = mass ? g.i2(j, i) : 0;
  float* T = s[WF_T];
  float* qv = s[WF_MOIST] + 1 * n3;
  float* qc = s[WF_MOIST] + 2 * n3;
  WCol<NS> c;
  float th[NS], pii[NS];
  if (run) {
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      const int k = sg.k(q);
      if (k < km) {
        const size_t p = k * lev + c2;
        th[q] = T[p] + (float)T0;
        const float pfull = s[WF_P][p] + s[WF_PB][p];
        pii[q] = wpow(pfull / (float)P0, F(mp::RCP));
        c.t[q] = th[q] * pii[q];
        c.den[q] = 1.0f / (s[WF_AL][p] + s[WF_ALB][p]);
        c.p[q] = pfull;
        const float zlo = (s[WF_PH][p] + s[WF_PHB][p]) / (float)G;
        const float zhi = (s[WF_PH][p + lev] + s[WF_PHB][p + lev]) / (float)G;
        c.delz[q] = zhi - zlo;
        c.q[q] = qv[p];
        c.qc0[q] = qc[p];
        c.qr0[q] = s[WF_MOIST][3 * n3 + p];
        c.qc1[q] = s[WF_MOIST][4 * n3 + p];
        c.qr1[q] = s[WF_MOIST][5 * n3 + p];
        c.qr2[q] = s[WF_MOIST][6 * n3 + p];
      } else {
        th[q] = 300.f; pii[q] = 1.f;
        c.t[q] = 280.f; c.q[q] = 0.f; c.qc0[q] = 0.f; c.qc1[q] = 0.f; c.qr0[q] = 0.f; c.qr1[q] = 0.f; c.qr2[q] = 0.f;
        c.den[q] = 1.f; c.p[q] = 8.0e4f; c.delz[q] = 100.f;
      }
    }
  } else {
    dummy_column<NS>(c);
#pragma unroll
    for (int q = 0; q < NS; ++q) { th[q] = 300.f; pii[q] = 1.f; }
  }
  Precip pr{run ? s[WF_RAINNC][c2] : 0.f, 0.f, run ? s[WF_SNOWNC][c2] : 0.f, 0.f,
            run ? s[WF_GRAUPELNC][c2] : 0.f, 0.f, 0.f};
  // every segment of the warp takes part (shuffles); only run columns store
  float qr0s[NS];
  wsm6_column_w<SEG, NS, true>(sg, c, dt, pr, scratch[col], qr0s);
  if (!mass) return;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    const int k = sg.k(q);
    if (k >= km) continue;
    const size_t p = k * lev + c2;
    float tnew, qvnew;
    if (run) {
      const float mpten = c.t[q] / pii[q] - th[q];
      tnew = T[p] + mpten;
      T[p] = tnew;
      s[WF_H_DIABATIC][p] = mpten / dt;
      s[WF_QV_DIABATIC][p] = (c.q[q] - qv[p]) / dt;
      s[WF_QC_DIABATIC][p] = (c.qc0[q] - qc[p]) / dt;
      qvnew = c.q[q];
      qv[p] = qvnew;
      qc[p] = c.qc0[q];
      s[WF_MOIST][3 * n3 + p] = c.qr0[q];
      s[WF_MOIST][4 * n3 + p] = c.qc1[q];
      s[WF_MOIST][5 * n3 + p] = c.qr1[q];
      s[WF_MOIST][6 * n3 + p] = c.qr2[q];
    } else {
      if (prep) {  // prepared but outside the scheme's block: zero tendencies
        s[WF_H_DIABATIC][p] = 0.0f;
        s[WF_QV_DIABATIC][p] = 0.0f;
        s[WF_QC_DIABATIC][p] = 0.0f;
      }
      tnew = T[p];
      qvnew = qv[p];
    }
    eos_point(g, s, k, p, c2, tnew, qvnew);
  }
  if (run && sg.l == 0) {
    s[WF_RAINNC][c2] = pr.rain;
    s[WF_RAINNCV][c2] = pr.rainncv;
    s[WF_SNOWNC][c2] = pr.snow;
    s[WF_SNOWNCV][c2] = pr.snowncv;
    s[WF_GRAUPELNC][c2] = pr.graupel;
    s[WF_GRAUPELNCV][c2] = pr.graupelncv;
    s[WF_SR][c2] = pr.sr;
  }
}

// stand-alone WSM6 on caller arrays: columns [ids+1, ide-2) x [jds+1, jde-2),
// levels [0, nz-1); th is potential temperature, pii the Exner function
struct Wsm6Args {
  float *th, *qv, *qc, *qr, *qi, *qs, *qg;
  const float *rho, *pii, *p, *dz8w;
  float *rainnc, *rainncv, *snownc, *snowncv, *graupelnc, *graupelncv, *sr;
};

template <int SEG, int NS>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_wsm6(Grid g, Wsm6Args a, float delt) {
  constexpr int SPW = 32 / SEG, SPB = kWarpsPerBlock * SPW;
  __shared__ SegScratch<SEG, NS> scratch[SPB];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int segw = lane / SEG;
  Seg<SEG, NS> sg;
  sg.l = lane % SEG;
  sg.base = segw * SEG;
  sg.km = g.nz - 1;
  const int km = sg.km;
  const int col = warp * SPW + segw;
  const int j = g.jds + 1 + blockIdx.y;
  const int i = g.ids + 1 + blockIdx.x * SPB + col;
  const bool run = i < g.ide - 2 && j < g.jde - 2;
  const size_t lev = (size_t)g.ny * g.nx;
  const int c2 = run ? g.i2(j, i) : 0;
  WCol<NS> c;
  dummy_column<NS>(c);
  if (run) {
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      const int k = sg.k(q);
      if (k >= km) continue;
      const size_t p = k * lev + c2;
      c.t[q] = a.th[p] * a.pii[p];
      c.den[q] = a.rho[p];
      c.p[q] = a.p[p];
      c.delz[q] = a.dz8w[p];
      c.q[q] = a.qv[p];
      c.qc0[q] = a.qc[p];
      c.qr0[q] = a.qr[p];
      c.qc1[q] = a.qi[p];
      c.qr1[q] = a.qs[p];
      c.qr2[q] = a.qg[p];
    }
  }
  Precip pr{run ? a.rainnc[c2] : 0.f, 0.f, run ? a.snownc[c2] : 0.f, 0.f, run ? a.graupelnc[c2] : 0.f, 0.f, 0.f};
  float qr0s[NS];
  wsm6_column_w<SEG, NS, true>(sg, c, delt, pr, scratch[col], qr0s);
  if (!run) return;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    const int k = sg.k(q);
    if (k >= km) continue;
    const size_t p = k * lev + c2;
    a.th[p] = c.t[q] / a.pii[p];
    a.qv[p] = c.q[q];
    a.qc[p] = c.qc0[q];
    a.qr[p] = c.qr0[q];
    a.qi[p] = c.qc1[q];
    a.qs[p] = c.qr1[q];
    a.qg[p] = c.qr2[q];
  }
  if (sg.l == 0) {
    a.rainnc[c2] = pr.rain;
    a.rainncv[c2] = pr.rainncv;
    a.snownc[c2] = pr.snow;
    a.snowncv[c2] = pr.snowncv;
    a.graupelnc[c2] = pr.graupel;
    a.graupelncv[c2] = pr.graupelncv;
    a.sr[c2] = pr.sr;
  }
}

// Split form of the physics step for a single time-split loop (dt < 240 s):
// k_wsm6_sed runs the column-coupled part (sedimentation of rain,
// snow + graupel and ice, melting, precipitation) on warp segments and leaves
// its state in WSM_T (temperature), WSM_QR0S (rain after the sedimentation)
// and the moisture slots; k_wsm6_finish then runs the point processes, the
// finish step and the equation of state one point per thread.  The
// arithmetic is that of k_physics, operation for operation.
// With kList, the columns are those of a list (list[0] entries from
// list[16], each j * nx + i of a column of the scheme's block): the WSM6
// fallback of the surrogate microphysics for the columns its gate rejected.
template <int SEG, int NS, bool kList = false>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_wsm6_sed(Grid g, S s, float dt, const int* list = nullptr) {
  constexpr int SPW = 32 / SEG, SPB = kWarpsPerBlock * SPW;
  __shared__ SegScratch<SEG, NS> scratch[SPB];
  if constexpr (kList) {
    if ((int)blockIdx.x * SPB >= __ldg(list)) return;  // whole block past the list (uniform exit)
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int segw = lane / SEG;
  Seg<SEG, NS> sg;
  sg.l = lane % SEG;
  sg.base = segw * SEG;
  sg.km = g.nz - 1;
  const int km = sg.km;
  const int col = warp * SPW + segw;
  int j, i;
  bool run;
  if constexpr (kList) {
    const int idx = blockIdx.x * SPB + col;
    run = idx < __ldg(list);
    const int code = run ? __ldg(list + 16 + idx) : 0;
    j = code / g.nx;
    i = code - j * g.nx;
  } else {
    j = g.jds + 1 + blockIdx.y;
    i = g.ids + 1 + blockIdx.x * SPB + col;
    run = i < g.ide - 2 && j < g.jde - 2;
  }
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const int c2 = run ? g.i2(j, i) : 0;
  float* M = s[WF_MOIST];
  WCol<NS> c;
  dummy_column<NS>(c);
  if (run) {
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      const int k = sg.k(q);
      if (k >= km) continue;
      const size_t p = k * lev + c2;
      const float th = s[WF_T][p] + (float)T0;
      const float pfull = s[WF_P][p] + s[WF_PB][p];
      c.t[q] = th * wpow(pfull / (float)P0, F(mp::RCP));
      c.den[q] = 1.0f / (s[WF_AL][p] + s[WF_ALB][p]);
      c.p[q] = pfull;
      const float zlo = (s[WF_PH][p] + s[WF_PHB][p]) / (float)G;
      const float zhi = (s[WF_PH][p + lev] + s[WF_PHB][p + lev]) / (float)G;
      c.delz[q] = zhi - zlo;
      c.q[q] = M[n3 + p];
      c.qc0[q] = M[2 * n3 + p];
      c.qr0[q] = M[3 * n3 + p];
      c.qc1[q] = M[4 * n3 + p];
      c.qr1[q] = M[5 * n3 + p];
      c.qr2[q] = M[6 * n3 + p];
    }
  }
  Precip pr{run ? s[WF_RAINNC][c2] : 0.f, 0.f, run ? s[WF_SNOWNC][c2] : 0.f, 0.f,
            run ? s[WF_GRAUPELNC][c2] : 0.f, 0.f, 0.f};
  float qr0s[NS];
  wsm6_column_w<SEG, NS, false>(sg, c, dt, pr, scratch[col], qr0s);
  if (!run) return;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    const int k = sg.k(q);
    if (k >= km) continue;
    const size_t p = k * lev + c2;
    s[WF_WSM_T][p] = c.t[q];
    s[WF_WSM_QR0S][p] = qr0s[q];
    M[3 * n3 + p] = c.qr0[q];
    M[4 * n3 + p] = c.qc1[q];
    M[5 * n3 + p] = c.qr1[q];
    M[6 * n3 + p] = c.qr2[q];
  }
  if (sg.l == 0) {
    s[WF_RAINNC][c2] = pr.rain;
    s[WF_RAINNCV][c2] = pr.rainncv;
    s[WF_SNOWNC][c2] = pr.snow;
    s[WF_SNOWNCV][c2] = pr.snowncv;
    s[WF_GRAUPELNC][c2] = pr.graupel;
    s[WF_GRAUPELNCV][c2] = pr.graupelncv;
    s[WF_SR][c2] = pr.sr;
  }
}

// one mass point of the finish kernel: run = in the scheme's block, prep =
// prepared by moist_physics_prep_em (zero tendencies outside the block)
__device__ __forceinline__ void wsm6_finish_point(const Grid& g, const S& s, int k, int j, int i, float dt,
                                                  float dtcld, bool run, bool prep) {
  const size_t n3 = g.n3();
  const int c2 = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c2;
  float* M = s[WF_MOIST];
  float T = s[WF_T][p];
  float qvnew = M[n3 + p];
  if (run) {
    const float th = T + (float)T0;
    const float pfull = s[WF_P][p] + s[WF_PB][p];
    const float pii = wpow(pfull / (float)P0, F(mp::RCP));
    const float t0 = th * pii;
    const float den = 1.0f / (s[WF_AL][p] + s[WF_ALB][p]);
    const float denfac = sqrtf(1.0f / den * F(mp::DEN0));
    float q = qvnew;
    const float qcold = M[2 * n3 + p];
    float qc0 = fmaxf(qcold, 0.0f);
    const float cpm = q >= F(mp::QMIN) ? F(mp::CPV) * q + (1.0f - q) * F(mp::CPD)
                                       : F(mp::CPD * (1.0 - mp::QMIN) + mp::CPV * mp::QMIN);
    const float xl = F(mp::XLV0) - F(mp::XLV1) * (t0 - F(mp::T0C));
    float qs0, qs1;
    fpvs(t0, pfull, qs0, qs1);
    const float qr0s = s[WF_WSM_QR0S][p];
    const bool small = qr0s <= F(mp::QCRMIN);
    const float rs0 = small ? F(mp::RSLOPERMAX) : 1.0f / wpow(F(mp::PIDN0R) / (qr0s * den), 0.25f);
    const float r30 = small ? F(mp::RSLOPER3MAX) : rs0 * rs0 * rs0;
    float t = s[WF_WSM_T][p];
    float qc1 = M[4 * n3 + p], qr0 = M[3 * n3 + p], qr1 = M[5 * n3 + p], qr2 = M[6 * n3 + p];
    wsm6_point(t, q, qc0, qc1, qr0, qr1, qr2, den, pfull, denfac, cpm, xl, qs0, qs1, rs0, r30, dtcld);
    const float mpten = t / pii - th;
    T = T + mpten;
    s[WF_T][p] = T;
    s[WF_H_DIABATIC][p] = mpten / dt;
    s[WF_QV_DIABATIC][p] = (q - qvnew) / dt;
    s[WF_QC_DIABATIC][p] = (qc0 - qcold) / dt;
    qvnew = q;
    M[n3 + p] = q;
    M[2 * n3 + p] = qc0;
    M[3 * n3 + p] = qr0;
    M[4 * n3 + p] = qc1;
    M[5 * n3 + p] = qr1;
    M[6 * n3 + p] = qr2;
  } else if (prep) {  // prepared but outside the scheme's block: zero tendencies
    s[WF_H_DIABATIC][p] = 0.0f;
    s[WF_QV_DIABATIC][p] = 0.0f;
    s[WF_QC_DIABATIC][p] = 0.0f;
  }
  eos_point(g, s, k, p, c2, T, qvnew);
}

// 8 blocks of 128 per SM (64 registers, a few bytes spilled to L1): the
// point processes are latency-bound, and the extra resident warps measured
// 3 % faster than the unbounded 80-register build
__global__ void __launch_bounds__(128, 8) k_wsm6_finish(Grid g, S s, float dt, float dtcld) {
  WRF_POINT_INDEX(g, k, j, i);
  if (k >= g.nz - 1 || j < g.jds || j >= g.jde - 1 || i < g.ids || i >= g.ide - 1) return;
  const bool run = j >= g.jds + 1 && j < g.jde - 2 && i >= g.ids + 1 && i < g.ide - 2;
  const bool prep = j >= g.jds + 1 && i >= g.ids + 1;
  wsm6_finish_point(g, s, k, j, i, dt, dtcld, run, prep);
}

// the finish kernel on the listed columns (see k_wsm6_sed's list mode):
// thread x = list entry, block y = level
__global__ void __launch_bounds__(128) k_wsm6_finish_list(Grid g, S s, float dt, float dtcld, const int* list) {
  const int n = __ldg(list);
  if ((int)(blockIdx.x * blockDim.x) >= n) return;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (idx >= n) return;
  const int code = __ldg(list + 16 + idx);
  const int j = code / g.nx, i = code - j * g.nx;
  wsm6_finish_point(g, s, k, j, i, dt, dtcld, true, true);
}

// ------------------------------------------------------------- no-alloc WSM6
// wrf_wsm6_noalloc computes wrf_wsm6's result with the split kernels, whose
// intermediate temperature and rain live in a fixed, file-scope device array
// instead of caller memory: for callers that hand over only the scheme's own
// arrays (the reference's wsm6 / microphysics_driver arguments have no room
// for scratch) and must not allocate device memory on their own (an
// allocation synchronises the device and can fail part-way through an
// integration).  Limit: kNoAllocMaxPoints points of the scheme's block
// ((nz-1) x (jde-jds-3) x (ide-ids-3)); 240x240x41 needs 2,061,160.  Nothing
// in the array needs to start at zero: each call writes every element it
// reads.  The array is shared by all calls on a device, so calls whose
// kernels overlap on the GPU (e.g. on two streams) race.
constexpr size_t kNoAllocMaxPoints = size_t(1) << 21;  // per intermediate field
static __device__ __align__(256) float g_wsm6_scratch[2 * kNoAllocMaxPoints];

// column part of WSM6 on caller arrays: writes the scratch (temperature,
// rain after the sedimentation), qr / qi / qs / qg after the sedimentation
// and melting, and the precipitation
template <int SEG, int NS>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_wsm6_sed_args(Grid g, Wsm6Args a, float delt, float* scr_t,
                                                                       float* scr_qr0s) {
  constexpr int SPW = 32 / SEG, SPB = kWarpsPerBlock * SPW;
  __shared__ SegScratch<SEG, NS> scratch[SPB];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int segw = lane / SEG;
  Seg<SEG, NS> sg;
  sg.l = lane % SEG;
  sg.base = segw * SEG;
  sg.km = g.nz - 1;
  const int km = sg.km;
  const int col = warp * SPW + segw;
  const int i0 = g.ids + 1, j0 = g.jds + 1;
  const int ncol = g.ide - 2 - i0, nrow = g.jde - 2 - j0;
  const int j = j0 + blockIdx.y;
  const int i = i0 + blockIdx.x * SPB + col;
  const bool run = i < g.ide - 2 && j < g.jde - 2;
  const size_t lev = (size_t)g.ny * g.nx;
  const int c2 = run ? g.i2(j, i) : 0;
  WCol<NS> c;
  dummy_column<NS>(c);
  if (run) {
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      const int k = sg.k(q);
      if (k >= km) continue;
      const size_t p = k * lev + c2;
      c.t[q] = a.th[p] * a.pii[p];
      c.den[q] = a.rho[p];
      c.p[q] = a.p[p];
      c.delz[q] = a.dz8w[p];
      c.q[q] = a.qv[p];
      c.qc0[q] = a.qc[p];
      c.qr0[q] = a.qr[p];
      c.qc1[q] = a.qi[p];
      c.qr1[q] = a.qs[p];
      c.qr2[q] = a.qg[p];
    }
  }
  Precip pr{run ? a.rainnc[c2] : 0.f, 0.f, run ? a.snownc[c2] : 0.f, 0.f, run ? a.graupelnc[c2] : 0.f, 0.f, 0.f};
  float qr0s[NS];
  wsm6_column_w<SEG, NS, false>(sg, c, delt, pr, scratch[col], qr0s);
  if (!run) return;
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    const int k = sg.k(q);
    if (k >= km) continue;
    const size_t p = k * lev + c2;
    const size_t b = ((size_t)k * nrow + (j - j0)) * ncol + (i - i0);
    scr_t[b] = c.t[q];
    scr_qr0s[b] = qr0s[q];
    a.qr[p] = c.qr0[q];
    a.qi[p] = c.qc1[q];
    a.qs[p] = c.qr1[q];
    a.qg[p] = c.qr2[q];
  }
  if (sg.l == 0) {
    a.rainnc[c2] = pr.rain;
    a.rainncv[c2] = pr.rainncv;
    a.snownc[c2] = pr.snow;
    a.snowncv[c2] = pr.snowncv;
    a.graupelnc[c2] = pr.graupel;
    a.graupelncv[c2] = pr.graupelncv;
    a.sr[c2] = pr.sr;
  }
}

// point processes of WSM6 on caller arrays, one thread per point of the block
__global__ void __launch_bounds__(128) k_wsm6_finish_args(Grid g, Wsm6Args a, float dtcld, const float* scr_t,
                                                          const float* scr_qr0s) {
  WRF_POINT_INDEX(g, k, j, i);
  const int i0 = g.ids + 1, j0 = g.jds + 1;
  if (k >= g.nz - 1 || j < j0 || j >= g.jde - 2 || i < i0 || i >= g.ide - 2) return;
  const int ncol = g.ide - 2 - i0, nrow = g.jde - 2 - j0;
  const size_t p = (size_t)k * g.ny * g.nx + g.i2(j, i);
  const size_t b = ((size_t)k * nrow + (j - j0)) * ncol + (i - i0);
  const float pii = a.pii[p];
  const float t0 = a.th[p] * pii;
  const float den = a.rho[p];
  const float pfull = a.p[p];
  const float denfac = sqrtf(1.0f / den * F(mp::DEN0));
  float q = a.qv[p];
  float qc0 = fmaxf(a.qc[p], 0.0f);
  const float cpm = q >= F(mp::QMIN) ? F(mp::CPV) * q + (1.0f - q) * F(mp::CPD)
                                     : F(mp::CPD * (1.0 - mp::QMIN) + mp::CPV * mp::QMIN);
  const float xl = F(mp::XLV0) - F(mp::XLV1) * (t0 - F(mp::T0C));
  float qs0, qs1;
  fpvs(t0, pfull, qs0, qs1);
  const float qr0s = scr_qr0s[b];
  const bool small = qr0s <= F(mp::QCRMIN);
  const float rs0 = small ? F(mp::RSLOPERMAX) : 1.0f / wpow(F(mp::PIDN0R) / (qr0s * den), 0.25f);
  const float r30 = small ? F(mp::RSLOPER3MAX) : rs0 * rs0 * rs0;
  float t = scr_t[b];
  float qc1 = a.qi[p], qr0 = a.qr[p], qr1 = a.qs[p], qr2 = a.qg[p];
  wsm6_point(t, q, qc0, qc1, qr0, qr1, qr2, den, pfull, denfac, cpm, xl, qs0, qs1, rs0, r30, dtcld);
  a.th[p] = t / pii;
  a.qv[p] = q;
  a.qc[p] = qc0;
  a.qr[p] = qr0;
  a.qi[p] = qc1;
  a.qs[p] = qr1;
  a.qg[p] = qr2;
}

// ------------------------------------------------------ surrogate microphysics
// Apply the network's outputs (increments of theta, qv..qg per level and the
// step's precipitation, standardised) to the mass points of the scheme's
// block.  Per column, in this order:
//   quiet     no condensate at any level and qv below saturation (over ice
//             where T < T0, else over water) at every level: WSM6 has no
//             process to run there, so the column takes zero increments
//             whatever the network says;
//   rejected  (the gate) an output is not finite, a species would go below
//             -tol_neg before clipping, or the new qv exceeds saturation over
//             water by more than the fraction tol_sat: the column is left
//             untouched and appended to list (entries j * nx + i from
//             list[16]); WSM6 then runs on it (k_wsm6_sed and
//             k_wsm6_finish_list in list mode, or k_physics in list mode for
//             two time-split loops);
//   network   otherwise: the increments (species clipped at zero).
// The step's precipitation is clipped to [0, condensate within kMlpMaxFall *
// dt of the ground] (all species for rainncv, snow + ice for snowncv, graupel
// for graupelncv): nothing else can reach the ground in one step.
// Counters: list[0] rejected, list[1] quiet, list[2] rejected for
// positivity, list[3] for supersaturation, list[4] for a non-finite output.
// colstat (optional) receives 0 network / 1 quiet / 2 rejected per column.
// Every other mass point gets the finish step (zero diabatic tendencies) and
// the equation of state, as in k_wsm6_finish.
// Block: 32 consecutive mass columns of one row (lane) x 8 warps over levels.
__global__ void __launch_bounds__(256) k_mlp_apply(Grid g, S s, MlpLayout L, const float* norm, const float* y,
                                                   float tol_neg, float tol_sat, float dt, int* list,
                                                   unsigned char* colstat) {
  __shared__ int sbad[32], squiet[32];
  __shared__ float scap[3][32];   // precipitable condensate near the ground: all, snow + ice, graupel (kg m-2)
  const int tx = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = g.ids + blockIdx.x * 32 + tx, j = g.jds + blockIdx.y;
  const bool mass = i < g.ide - 1;
  const bool run = mass && j >= g.jds + 1 && j < g.jde - 2 && i >= g.ids + 1 && i < g.ide - 2;
  const bool prep = mass && j >= g.jds + 1 && i >= g.ids + 1;
  const int km = L.km;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const int c2 = mass ? g.i2(j, i) : 0;
  const size_t col = run ? (size_t)(j - g.jds - 1) * L.ncx + (i - g.ids - 1) : 0;
  const float* yr = y + col * L.d4;
  const float* omean = norm + norm_out_mean(L);
  const float* ostd = norm + norm_out_std(L);
  float* T = s[WF_T];
  float* M = s[WF_MOIST];
  auto inc = [&](int o) { return yr[o] * ostd[o] + omean[o]; };
  if (w == 0) {
    sbad[tx] = 0;
    squiet[tx] = 1;
    scap[0][tx] = scap[1][tx] = scap[2][tx] = 0.f;
  }
  __syncthreads();
  if (run) {
    int bad = 0, quiet = 1;
    const float* php = s[WF_PH];
    const float* phb = s[WF_PHB];
    const float zs = (php[c2] + phb[c2]) / (float)G;
    const float reach = kMlpMaxFall * dt;
    float cap_all = 0.f, cap_snow = 0.f, cap_graupel = 0.f;
    for (int k = w; k < km; k += 8) {
      const size_t p = k * lev + c2;
      // condensate that can reach the ground within the step (levels whose
      // bottom lies within kMlpMaxFall * dt of it), kg m-2
      const float zb = (php[p] + phb[p]) / (float)G, zt = (php[p + lev] + phb[p + lev]) / (float)G;
      if (zb - zs < reach) {
        const float rdz = (zt - zb) / (s[WF_AL][p] + s[WF_ALB][p]);
        const float qr = fmaxf(M[3 * n3 + p], 0.f), qi = fmaxf(M[4 * n3 + p], 0.f);
        const float qsn = fmaxf(M[5 * n3 + p], 0.f), qg = fmaxf(M[6 * n3 + p], 0.f);
        cap_all += (qr + qi + qsn + qg) * rdz;
        cap_snow += (qi + qsn) * rdz;
        cap_graupel += qg * rdz;
      }
      const float pfull = s[WF_P][p] + s[WF_PB][p];
      const float pii = wpow(pfull / (float)P0, F(mp::RCP));
      float qs0, qs1;
      fpvs((T[p] + (float)T0) * pii, pfull, qs0, qs1);
      float cond = 0.f;
      for (int m = 2; m < 7; ++m) cond = fmaxf(cond, fabsf(M[m * n3 + p]));
      if (cond != 0.f || !(M[n3 + p] < qs1)) quiet = 0;
      const float dth = inc(k);
      const float tnew = T[p] + dth;
      if (!isfinite(dth)) bad |= 4;
      float qvn = 0.f;
      for (int m = 1; m < 7; ++m) {
        const float d = inc(m * km + k);
        const float qn = M[m * n3 + p] + d;
        if (!isfinite(d)) bad |= 4;
        if (qn < -tol_neg) bad |= 1;
        if (m == 1) qvn = fmaxf(qn, 0.f);
      }
      fpvs((tnew + (float)T0) * pii, pfull, qs0, qs1);
      if (!(qvn <= qs0 * (1.0f + tol_sat))) bad |= 2;
    }
    if (w == 0)
      for (int o = 0; o < kOutPrecip; ++o)
        if (!isfinite(inc(kOutVars * km + o))) bad |= 4;
    if (bad) atomicOr(&sbad[tx], bad);
    if (!quiet) atomicAnd(&squiet[tx], 0);
    atomicAdd(&scap[0][tx], cap_all);
    atomicAdd(&scap[1][tx], cap_snow);
    atomicAdd(&scap[2][tx], cap_graupel);
  }
  __syncthreads();
  const bool quiet = run && squiet[tx] != 0;
  const int bad = run && !quiet ? sbad[tx] : 0;
  const bool rejected = bad != 0;
  if (run && w == 0) {
    if (quiet) atomicAdd(list + 1, 1);
    if (rejected) {
      const int slot = atomicAdd(list, 1);
      list[16 + slot] = c2;
      if (bad & 1) atomicAdd(list + 2, 1);
      if (bad & 2) atomicAdd(list + 3, 1);
      if (bad & 4) atomicAdd(list + 4, 1);
    }
    if (colstat) colstat[col] = quiet ? 1 : (rejected ? 2 : 0);
  }
  if (!mass || rejected) return;
  const bool net = run && !quiet;
  for (int k = w; k < km; k += 8) {
    const size_t p = k * lev + c2;
    float tnew, qvnew;
    if (net) {
      const float dth = inc(k);
      tnew = T[p] + dth;
      T[p] = tnew;
      s[WF_H_DIABATIC][p] = dth / dt;
      const float qv0 = M[n3 + p], qc0 = M[2 * n3 + p];
      float qn[7];
      for (int m = 1; m < 7; ++m) qn[m] = fmaxf(M[m * n3 + p] + inc(m * km + k), 0.0f);
      s[WF_QV_DIABATIC][p] = (qn[1] - qv0) / dt;
      s[WF_QC_DIABATIC][p] = (qn[2] - qc0) / dt;
      for (int m = 1; m < 7; ++m) M[m * n3 + p] = qn[m];
      qvnew = qn[1];
    } else {
      if (prep) {
        s[WF_H_DIABATIC][p] = 0.0f;
        s[WF_QV_DIABATIC][p] = 0.0f;
        s[WF_QC_DIABATIC][p] = 0.0f;
      }
      tnew = T[p];
      qvnew = M[n3 + p];
    }
    eos_point(g, s, k, p, c2, tnew, qvnew);
  }
  if (run && w == 0) {
    // precipitation of the step, bounded by what can fall out of the column
    const float rain = net ? fminf(fmaxf(inc(kOutVars * km + 0), 0.0f), scap[0][tx]) : 0.0f;
    const float snow = net ? fminf(fmaxf(inc(kOutVars * km + 1), 0.0f), scap[1][tx]) : 0.0f;
    const float graupel = net ? fminf(fmaxf(inc(kOutVars * km + 2), 0.0f), scap[2][tx]) : 0.0f;
    s[WF_RAINNCV][c2] = rain;
    s[WF_SNOWNCV][c2] = snow;
    s[WF_GRAUPELNCV][c2] = graupel;
    s[WF_RAINNC][c2] = s[WF_RAINNC][c2] + rain;
    s[WF_SNOWNC][c2] = s[WF_SNOWNC][c2] + snow;
    s[WF_GRAUPELNC][c2] = s[WF_GRAUPELNC][c2] + graupel;
    s[WF_SR][c2] = rain > 0.f ? (snow + graupel) / (rain + 1.0e-12f) : 0.0f;
  }
}

#undef F

// 16-lane segments with 3 levels per lane hold up to 47 mass levels; deeper
// columns use whole warps with 2 levels per lane (up to 63)
int launch_physics(const Grid& g, const S& s, cudaStream_t st) {
  const int km = g.nz - 1;
  const dim3 b(32 * kWarpsPerBlock);
  const double loops = fmax(g.dtd / mp::DTCLDCR, 1.0);
  if ((int)loops == 1) {
    const float dtcld = (g.dtd <= mp::DTCLDCR) ? g.dt : (float)(1.0 * g.dtd / loops);
    const int ncol = g.ide - 2 - (g.ids + 1), nrow = g.jde - 2 - (g.jds + 1);
    if (km <= 47) {
      constexpr int SPB = kWarpsPerBlock * 2;
      k_wsm6_sed<16, 3><<<dim3((ncol + SPB - 1) / SPB, nrow), b, 0, st>>>(g, s, g.dt);
    } else {
      constexpr int SPB = kWarpsPerBlock;
      k_wsm6_sed<32, 2><<<dim3((ncol + SPB - 1) / SPB, nrow), b, 0, st>>>(g, s, g.dt);
    }
    const dim3 b3(32, 4);
    k_wsm6_finish<<<point_grid(g, b3), b3, 0, st>>>(g, s, g.dt, dtcld);
    return 2;
  }
  const int ncol = g.ide - 1 - g.ids, nrow = g.jde - 1 - g.jds;
  if (km <= 47) {
    constexpr int SPB = kWarpsPerBlock * 2;
    k_physics<16, 3><<<dim3((ncol + SPB - 1) / SPB, nrow), b, 0, st>>>(g, s, g.dt);
  } else {
    constexpr int SPB = kWarpsPerBlock;
    k_physics<32, 2><<<dim3((ncol + SPB - 1) / SPB, nrow), b, 0, st>>>(g, s, g.dt);
  }
  return 1;
}

// f: th qv qc qr qi qs qg rho pii p dz8w rainnc rainncv snownc snowncv graupelnc graupelncv sr
int launch_wsm6(const Grid& g, float* const* f, float delt, cudaStream_t st) {
  Wsm6Args a{f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[10],
             f[11], f[12], f[13], f[14], f[15], f[16], f[17]};
  const int km = g.nz - 1;
  const int ncol = g.ide - 2 - (g.ids + 1), nrow = g.jde - 2 - (g.jds + 1);
  const dim3 b(32 * kWarpsPerBlock);
  if (km <= 47) {
    constexpr int SPB = kWarpsPerBlock * 2;
    k_wsm6<16, 3><<<dim3((ncol + SPB - 1) / SPB, nrow), b, 0, st>>>(g, a, delt);
  } else {
    constexpr int SPB = kWarpsPerBlock;
    k_wsm6<32, 2><<<dim3((ncol + SPB - 1) / SPB, nrow), b, 0, st>>>(g, a, delt);
  }
  return 1;
}

// The scratch's device address is looked up by the first call in each CUDA
// context (cudaGetSymbolAddress, with the context's device current) and kept
// with that context's handle: after a device reset the new primary context
// differs, and the address is looked up again.  The lookup should come before
// any stream capture on the device.
namespace {
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<CtxGetCurrentFn>(nullptr);
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}
}  // namespace

int launch_wsm6_noalloc(const Grid& g, float* const* f, float delt, cudaStream_t st, const char** err) {
  const int km = g.nz - 1;
  const int ncol = g.ide - 2 - (g.ids + 1), nrow = g.jde - 2 - (g.jds + 1);
  const size_t npts = (size_t)km * (size_t)nrow * (size_t)ncol;
  if (npts > kNoAllocMaxPoints) {
    *err = "wrf_wsm6_noalloc: the scheme's block exceeds the fixed scratch (2097152 points per field)";
    return WRF_EINVAL;
  }
  const double loops = fmax((double)delt / mp::DTCLDCR, 1.0);
  if ((int)loops != 1) {
    *err = "wrf_wsm6_noalloc: delt >= 240 s needs two time-split loops; use wrf_wsm6";
    return WRF_EINVAL;
  }
  constexpr int kMaxDev = 64;
  static CUcontext owner[kMaxDev] = {};
  static float* scratch[kMaxDev] = {};
  static std::mutex setup;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) {
    *err = "wrf_wsm6_noalloc: no current CUDA device (or device index >= 64)";
    return WRF_ECUDA;
  }
  // the calling thread's current context (null before the runtime has bound
  // the device's primary context to the thread: the symbol lookup binds it)
  CUcontext ctx = nullptr;
  const CtxGetCurrentFn get_ctx = ctx_get_current();
  if (!get_ctx || get_ctx(&ctx) != CUDA_SUCCESS) {
    *err = "wrf_wsm6_noalloc: cuCtxGetCurrent is not available from the driver";
    return WRF_ECUDA;
  }
  float* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(setup);
    if (!ctx || !scratch[dev] || owner[dev] != ctx) {
      void* ptr = nullptr;
      const cudaError_t rc = cudaGetSymbolAddress(&ptr, g_wsm6_scratch);
      if (rc != cudaSuccess || !ptr || (!ctx && (get_ctx(&ctx) != CUDA_SUCCESS || !ctx))) {
        *err = "wrf_wsm6_noalloc: cudaGetSymbolAddress of the scratch array failed";
        return WRF_ECUDA;
      }
      scratch[dev] = static_cast<float*>(ptr);
      owner[dev] = ctx;
    }
    base = scratch[dev];
  }
  Wsm6Args a{f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[10],
             f[11], f[12], f[13], f[14], f[15], f[16], f[17]};
  const dim3 b(32 * kWarpsPerBlock);
  if (km <= 47) {
    constexpr int SPB = kWarpsPerBlock * 2;
    k_wsm6_sed_args<16, 3><<<dim3((ncol + SPB - 1) / SPB, nrow), b, 0, st>>>(g, a, delt, base, base + kNoAllocMaxPoints);
  } else {
    constexpr int SPB = kWarpsPerBlock;
    k_wsm6_sed_args<32, 2><<<dim3((ncol + SPB - 1) / SPB, nrow), b, 0, st>>>(g, a, delt, base, base + kNoAllocMaxPoints);
  }
  const float dtcld = ((double)delt <= mp::DTCLDCR) ? delt : (float)(1.0 * (double)delt / loops);
  const dim3 b3(32, 4);
  k_wsm6_finish_args<<<point_grid(g, b3), b3, 0, st>>>(g, a, dtcld, base, base + kNoAllocMaxPoints);
  return 2;
}


int launch_mlp_forward(const MlpNetDev& net, const void* x, int m, void* h0, void* h1, float* y, int* errflag,
                       cudaStream_t st, const char** err) {
  int n = 0;
  const void* in = x;
  void* h[2] = {h0, h1};
  for (int l = 0; l < kMlpLayers; ++l) {
    const bool last = l == kMlpLayers - 1;
    GemmEpi e{};
    e.kind = last ? EPI_F32 : EPI_BIAS_GELU;
    e.bias = net.b[l];
    e.out = last ? static_cast<void*>(y) : h[l & 1];
    e.ldo = net.dims[l + 1];
    e.err = errflag;
    const int r = launch_gemm_tc(in, net.w[l], m, net.dims[l + 1], net.dims[l], 1, e, st, err);
    if (r < 0) return r;
    n += r;
    in = e.out;
  }
  return n;
}

int launch_physics_mlp(const Grid& g, const S& s, const MlpNetDev& net, const MlpWorkDev& work, cudaStream_t st,
                       const char** err) {
  const MlpLayout L = MlpLayout::make(g.nx, g.ny, g.nz, g.ids, g.ide, g.jds, g.jde);
  if (net.dims[0] != L.d0 || net.dims[kMlpLayers] != L.d4) {
    *err = "surrogate: the network's input / output widths do not match this grid's column layout";
    return WRF_EINVAL;
  }
  for (int l = 1; l < kMlpLayers; ++l)
    if (net.dims[l] < 64 || net.dims[l] % 64) {
      *err = "surrogate: hidden widths must be multiples of 64";
      return WRF_EINVAL;
    }
  for (int l = 0; l < kMlpLayers; ++l)
    if (!net.w[l] || !net.b[l]) {
      *err = "surrogate: null weight or bias";
      return WRF_EINVAL;
    }
  if (!net.norm || !work.x || !work.h[0] || !work.h[1] || !work.y || !work.list || work.capacity < L.ncols) {
    *err = "surrogate: null buffer, or work capacity below the block's column count";
    return WRF_EINVAL;
  }
  int n = 0;
  if (cudaMemsetAsync(work.list, 0, 16 * sizeof(int), st) != cudaSuccess) {
    *err = "surrogate: memset of the fallback list failed";
    return WRF_ECUDA;
  }
  int r = launch_mlp_features(g, s, L, net.norm, work.x, nullptr, st);
  if (r < 0) { *err = "surrogate: feature kernel set-up failed"; return r; }
  n += r;
  r = launch_mlp_forward(net, work.x, L.ncols, work.h[0], work.h[1], work.y, work.err, st, err);
  if (r < 0) return r;
  n += r;
  k_mlp_apply<<<dim3((g.ide - 1 - g.ids + 31) / 32, g.jde - 1 - g.jds), 256, 0, st>>>(
      g, s, L, net.norm, work.y, net.tol_neg, net.tol_sat, g.dt, work.list,
      static_cast<unsigned char*>(work.colstat));
  ++n;
  // WSM6 on the rejected columns: the split kernels when one time-split loop
  // suffices (as in launch_physics), else the fused column kernel
  const int km = g.nz - 1;
  const dim3 b(32 * kWarpsPerBlock);
  const double loops = fmax(g.dtd / mp::DTCLDCR, 1.0);
  if ((int)loops == 1) {
    const float dtcld = (g.dtd <= mp::DTCLDCR) ? g.dt : (float)(1.0 * g.dtd / loops);
    if (km <= 47) {
      constexpr int SPB = kWarpsPerBlock * 2;
      k_wsm6_sed<16, 3, true><<<(L.ncols + SPB - 1) / SPB, b, 0, st>>>(g, s, g.dt, work.list);
    } else {
      constexpr int SPB = kWarpsPerBlock;
      k_wsm6_sed<32, 2, true><<<(L.ncols + SPB - 1) / SPB, b, 0, st>>>(g, s, g.dt, work.list);
    }
    k_wsm6_finish_list<<<dim3((L.ncols + 127) / 128, km), 128, 0, st>>>(g, s, g.dt, dtcld, work.list);
    return n + 2;
  }
  if (km <= 47) {
    constexpr int SPB = kWarpsPerBlock * 2;
    k_physics<16, 3, true><<<(L.ncols + SPB - 1) / SPB, b, 0, st>>>(g, s, g.dt, work.list);
  } else {
    constexpr int SPB = kWarpsPerBlock;
    k_physics<32, 2, true><<<(L.ncols + SPB - 1) / SPB, b, 0, st>>>(g, s, g.dt, work.list);
  }
  return n + 1;
}

}  // namespace wrf
