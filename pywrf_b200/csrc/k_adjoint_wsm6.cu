// Adjoint of the step's microphysics (moist_physics_prep_em, WSM6 and
// moist_physics_finish_em: wrf_physics.py:27-91, 137-1214, 2106-2137).
//
// Every output of the block in a column (theta, qv .. qg, h_diabatic) is a
// function of that column's inputs only (t, qv .. qg, al, p below the top
// level and ph on every level; alb, pb and phb are data), so its reverse
// product is formed column by column, one thread per column.  The column is
// restated here as plain per-column code templated on its scalar type
// (column arrays in a global workspace) in the order of the reference's
// statements: the instantaneous processes, the source and sink rates with
// their limiters, the saturation adjustment, and the semi-Lagrangian
// sedimentation (nislfv_rain_plm / _plm6, wrf_physics.py:1216-1583) with its
// interface fall speeds, departure cells and overlap remap.  The derivative
// is that of the branch taken.
//
// The reverse product is taken in reverse mode: the column runs once on
// taped scalars (tape.cuh), the outputs' cotangents seed the adjoints of
// their entries, and one reverse sweep yields every input's cotangent.
// With one time-split loop (split mode) the tape stops before the point
// processes: those read only their own level, so each level's are reversed
// on a thread of its own by forward-mode tangents and added into the
// adjoints of the tape entries its inputs come from, before the sweep.
// Columns are taped in chunks that bound the tape's memory.  A column whose
// tape outgrows the capacity is finished by forward-mode tangents instead:
// the same code on Dual<N> numbers with N inputs seeded per pass, the
// cotangent of each seeded input the dot product of the outputs' cotangents
// with their tangents, ceil(n_inputs / N) passes per column.
#include "dual.cuh"
#include "kernels.cuh"
#include "tape.cuh"
#include "wsm6_const.cuh"

#include <algorithm>

namespace wrf {
namespace mpt {

using namespace mp;

// column arrays of one thread: array a, level k at base[(a * kst + k) * ncol]
template <class T>
struct Col {
  T* base;
  int ncol, kst;
  __device__ __forceinline__ T& operator()(int a, int k) const { return base[((size_t)a * kst + k) * ncol]; }
};

enum {
  A_TIN, A_TH, A_PII, A_T, A_Q, A_QC, A_QI, A_QR, A_QS, A_QG, A_DEN, A_P, A_DELZ, A_CPM, A_XL, A_DENFAC, A_QS0,
  A_QS1, A_RH0, A_RH1, A_XNI, A_R1, A_R2, A_R3, A_W1, A_W2, A_ZI, A_WI, A_ZA, A_DZA, A_QA, A_QA2, A_WD, A_WWW,
  A_SR3, A_SRS, A_COUNT
};

template <class T>
__device__ __forceinline__ T cst(float x) {
  return Lift<T>::c(x);
}

template <class T>
__device__ __forceinline__ T n0sfac(const T& t) {
  return vmax(vmin(vexp(F(ALPHA) * (F(T0C) - t)), F(N0SMAX / N0S)), 1.0f);
}

// terminal velocity of one precipitating species (the slope with the rain
// caps), kind 0 rain, 1 snow, 2 graupel
template <class T>
__device__ T vt_of(int kind, const T& q, const T& den, const T& denfac, const T& t) {
  const float pidn0 = kind == 0 ? F(PIDN0R) : (kind == 1 ? F(PIDN0S) : F(PIDN0G));
  const float bv = kind == 0 ? F(BVTR) : (kind == 1 ? F(BVTS) : F(BVTG));
  const float pv = kind == 0 ? F(PVTR) : (kind == 1 ? F(PVTS) : F(PVTG));
  const bool small = val(q) <= F(QCRMIN);
  T rb;
  if (small) {
    rb = cst<T>(F(RSLOPERBMAX));
  } else {
    const T num = kind == 1 ? pidn0 * n0sfac(t) : cst<T>(pidn0);
    const T lam = vpow(num / (q * den), 0.25f);
    rb = vpow(1.0f / lam, bv);
  }
  return val(q) <= 0.f ? cst<T>(0.f) : pv * rb * denfac;
}

// whether any directional derivative of x is nonzero (always true for a
// plain float, whose value path is the point of running the code)
__device__ __forceinline__ bool live(float) { return true; }
template <int N>
__device__ __forceinline__ bool live(const Dual<N>& x) {
  bool any = false;
#pragma unroll
  for (int n = 0; n < N; ++n) any |= x.d[n] != 0.f;
  return any;
}
__device__ __forceinline__ bool live(const Tv& x) { return x.id >= 0; }

template <class T>
struct Slope3 {
  T rs[3], rb[3], r2[3], r3[3];
};

// slope_wsm6 (wrf_physics.py:2048-2104) at one level
template <class T>
__device__ void slope3(const T& qr, const T& qs, const T& qg, const T& den, const T& t, Slope3<T>& o) {
  const T q[3] = {qr, qs, qg};
  const float bv[3] = {F(BVTR), F(BVTS), F(BVTG)};
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    if (val(q[m]) <= F(QCRMIN)) {
      o.rs[m] = cst<T>(F(RSLOPERMAX));
      o.rb[m] = cst<T>(F(RSLOPERBMAX));
      o.r2[m] = cst<T>(F(RSLOPER2MAX));
      o.r3[m] = cst<T>(F(RSLOPER3MAX));
    } else {
      const T num = m == 0 ? cst<T>(F(PIDN0R)) : (m == 1 ? F(PIDN0S) * n0sfac(t) : cst<T>(F(PIDN0G)));
      const T a = 1.0f / vpow(num / (q[m] * den), 0.25f);
      o.rs[m] = a;
      o.rb[m] = vpow(a, bv[m]);
      o.r2[m] = a * a;
      o.r3[m] = a * a * a;
    }
  }
}

// saturation mixing ratios over water and (below the triple point) ice
template <class T>
__device__ void fpvs(const T& t, const T& p, T& qs0, T& qs1) {
  const double ttp = T0C + 0.01;
  const double dldt = CPV - CLIQ, xa = -dldt / RV, xb = xa + XLV0 / (RV * ttp);
  const double dldti = CPV - CICE, xai = -dldti / RV, xbi = xai + XLS / (RV * ttp);
  const T tr = F(ttp) / t;
  const T w1 = F(PSAT) * vexp(vlog(tr) * F(xa)) * vexp(F(xb) * (1.0f - tr));
  T a = vmin(w1, 0.99f * p);
  a = F(EP2) * a / (p - a);
  qs0 = vmax(a, F(QMIN));
  const T w0 = F(PSAT) * vexp(vlog(tr) * F(xai)) * vexp(F(xbi) * (1.0f - tr));
  T b = val(t) < F(ttp) ? w0 : w1;
  b = vmin(b, 0.99f * p);
  b = F(EP2) * b / (p - b);
  qs1 = vmax(b, F(QMIN));
}

template <class T>
__device__ __forceinline__ T viscos(const T& t, const T& den) {
  return 1.496e-6f * (t * vsqrt(t)) / (t + 120.0f) / den;
}
template <class T>
__device__ __forceinline__ T diffus(const T& t, const T& p) {
  return 8.794e-5f * vexp(vlog(t) * 1.81f) / p;
}
template <class T>
__device__ __forceinline__ T xka(const T& t, const T& den) {
  return 1.414e3f * viscos(t, den) * den;
}
template <class T, class A>
__device__ __forceinline__ T diffac(const A& a, const T& p, const T& t, const T& den, const T& qs) {
  return den * a * a / (xka(t, den) * F(RV) * t * t) + 1.0f / (qs * diffus(t, p));
}
template <class T>
__device__ __forceinline__ T venfac(const T& p, const T& t, const T& den) {
  return vexp(vlog(viscos(t, den) / diffus(t, p)) * 0.3333333f) / vsqrt(viscos(t, den)) * vsqrt(vsqrt(F(DEN0) / den));
}

// interface fall speeds: 3rd-order interpolation of the cell speeds (www),
// the ww == 0 fallback and the downward CFL limiter (wrf_physics.py:1269-1293)
template <class T>
__device__ void fall_interfaces(const Col<T>& C, int km, float dt) {
  const float fa1 = 9.0f / 16.0f, fa2 = 1.0f / 16.0f;
  C(A_WI, 0) = C(A_WWW, 0);
  C(A_WI, 1) = 0.5f * (C(A_WWW, 1) + C(A_WWW, 0));
  for (int k = 2; k < km - 1; ++k)
    C(A_WI, k) = fa1 * (C(A_WWW, k) + C(A_WWW, k - 1)) - fa2 * (C(A_WWW, k + 1) + C(A_WWW, k - 2));
  C(A_WI, km - 1) = 0.5f * (C(A_WWW, km - 1) + C(A_WWW, km - 2));
  C(A_WI, km) = C(A_WWW, km - 1);
  for (int k = 1; k < km; ++k)
    if (val(C(A_WWW, k)) == 0.f) C(A_WI, k) = C(A_WWW, k - 1);
  for (int k = km - 1; k >= 0; --k) {
    const T dz = C(A_DELZ, k);
    const T decfl = (C(A_WI, k + 1) - C(A_WI, k)) * dt / dz;
    if (val(decfl) > 0.05f) C(A_WI, k) = C(A_WI, k + 1) - 0.05f * dz / dt;
  }
}

// the piecewise-constant overlap remap of the departure cells' mass (array
// qa, the top cell's zeroed) onto the grid (wrf_physics.py:1339-1357, the
// last layers 3800 m deep), written into array out.  A pair of cells whose
// overlap is not positive contributes the constant 0 (value and
// derivatives), so the pairs are screened on the values first: only the
// few overlapping departure cells of a level enter the dual arithmetic.
template <class T>
__device__ void remap(const Col<T>& C, int km, int qa, int out) {
  float za[kMaxNz + 1];
  for (int k = 0; k <= km; ++k) za[k] = val(C(A_ZA, k));
  for (int k = 0; k < km; ++k) {
    const T zlo = C(A_ZI, k);
    const T zhi = k < km - 1 ? C(A_ZI, k + 1) : C(A_ZI, km - 1) + 3800.0f;
    const float zlov = val(zlo), zhiv = val(zhi);
    T acc = cst<T>(0.f);
    for (int ka = 0; ka < km; ++ka) {
      const float alov = za[ka], ahiv = ka < km - 1 ? za[ka + 1] : za[km - 1] + 3800.0f;
      if (!(vmin(zhiv, ahiv) - vmax(zlov, alov) > 0.0f)) continue;
      const T alo = C(A_ZA, ka);
      const T ahi = ka < km - 1 ? C(A_ZA, ka + 1) : C(A_ZA, km - 1) + 3800.0f;
      const T ov = vmax(0.0f, vmin(zhi, ahi) - vmax(zlo, alo));
      acc = acc + C(qa, ka) * ov;
    }
    C(out, k) = acc / C(A_DELZ, k);
  }
}

// the mass that left through the ground (wrf_physics.py:1361-1374)
template <class T>
__device__ T surface_flux(const Col<T>& C, int km, int qa) {
  T precip = cst<T>(0.f);
  for (int k = 0; k < km; ++k) {
    const float z0 = val(C(A_ZA, k)), z1 = val(C(A_ZA, k + 1));
    if (z0 < 0.f && z1 < 0.f) precip = precip + C(qa, k) * C(A_DZA, k);
    if (z0 < 0.f && z1 > 0.f) precip = precip + C(qa, k) * (0.0f - C(A_ZA, k));
  }
  return precip;
}

// nislfv_rain_plm (kind 0, rain; kind 2, cloud ice with iter 0) and
// nislfv_rain_plm6 (kind 1: snow in r1 and graupel in r2 with the shared
// mass-weighted speed): the cell speeds are in A_W1, the masses (den q) in
// r1 (and r2), replaced by the sedimented masses; returns the first
// species' surface flux
template <class T>
__device__ T nislfv(const Col<T>& C, int km, int kind, int r1, int r2, float dt, int iter) {
  T allold = cst<T>(0.f);
  for (int k = 0; k < km; ++k) allold = allold + C(r1, k);
  if (kind == 1)
    for (int k = 0; k < km; ++k) allold = allold + C(r2, k);
  if (!(val(allold) > 0.f)) {
    // nothing to fall: the scheme's result is zero (value and derivatives)
    for (int k = 0; k < km; ++k) {
      C(r1, k) = cst<T>(0.f);
      if (kind == 1) C(r2, k) = cst<T>(0.f);
    }
    return cst<T>(0.f);
  }
  C(A_ZI, 0) = cst<T>(0.f);
  for (int k = 0; k < km; ++k) C(A_ZI, k + 1) = C(A_ZI, k) + C(A_DELZ, k);
  for (int k = 0; k < km; ++k) {
    C(A_WD, k) = C(A_W1, k);
    C(A_WWW, k) = C(A_W1, k);
  }
  const int npass = iter >= 1 ? 2 : 1;
  for (int n = 1; n <= npass; ++n) {
    fall_interfaces(C, km, dt);
    for (int k = 0; k <= km; ++k) C(A_ZA, k) = C(A_ZI, k) - C(A_WI, k) * dt;
    for (int k = 0; k < km; ++k) C(A_DZA, k) = C(A_ZA, k + 1) - C(A_ZA, k);
    C(A_DZA, km) = C(A_ZI, km) - C(A_ZA, km);
    for (int k = 0; k < km; ++k) {
      C(A_QA, k) = C(r1, k) * C(A_DELZ, k) / C(A_DZA, k);
      if (kind == 1) C(A_QA2, k) = C(r2, k) * C(A_DELZ, k) / C(A_DZA, k);
    }
    C(A_QA, km) = cst<T>(0.f);
    C(A_QA2, km) = cst<T>(0.f);
    if (n <= iter) {
      for (int k = 0; k < km; ++k) {
        const T den = C(A_DEN, k), denfac = C(A_DENFAC, k);
        const T qr = C(A_QA, k) / den;
        T wa;
        if (kind == 1) {
          const T qr2 = C(A_QA2, k) / den;
          const T wa1 = vt_of(1, qr, den, denfac, C(A_T, k));
          const T wa2 = vt_of(2, qr2, den, denfac, C(A_T, k));
          const T tmp = vmax(qr + qr2, 1.0e-15f);
          wa = val(tmp) > 1.0e-15f ? (wa1 * qr + wa2 * qr2) / tmp : cst<T>(0.f);
        } else {
          wa = vt_of(0, qr, den, denfac, C(A_T, k));
        }
        C(A_WWW, k) = 0.5f * (C(A_WD, k) + wa);
      }
    }
  }
  const bool ok = val(allold) > 0.f;
  T precip = cst<T>(0.f);
  for (int sp = 0; sp < (kind == 1 ? 2 : 1); ++sp) {
    const int qa = sp == 0 ? A_QA : A_QA2, r = sp == 0 ? r1 : r2;
    C(qa, km - 1) = cst<T>(0.f);
    remap(C, km, qa, r);
    const T pr = surface_flux(C, km, qa);
    if (sp == 0) precip = pr;
    if (!ok)
      for (int k = 0; k < km; ++k) C(r, k) = cst<T>(0.f);
  }
  return ok ? precip : cst<T>(0.f);
}

// the rates' limiter: where source > value (and cnd), every listed rate is
// scaled by value / source
template <class T, int M>
__device__ __forceinline__ void limit(const T& value, const T& source, bool cnd, T* const (&r)[M]) {
  if (cnd && val(source) > val(value)) {
    const T f = value / source;
#pragma unroll
    for (int m = 0; m < M; ++m) *r[m] = *r[m] * f;
  }
}

// the processes after the sedimentation at one level (wrf_physics.py:
// 596-1203): instantaneous melting / freezing, the source and sink rates,
// the mass-conserving limiters and updates for T <= t0c and T > t0c, and the
// saturation adjustment.  t, q, qc, qi, qr, qs, qg are updated in place.
template <class T>
__device__ void point_processes(T& t, T& q, T& qc, T& qi, T& qr, T& qs, T& qg, const T& den, const T& p,
                                const T& denfac, const T& cpm, const T& xl, const T& qs0, const T& qs1,
                                const T& rh0, const T& rh1, const Slope3<T>& sl0, float dtcld) {
  const T zero = cst<T>(0.f);
  // instantaneous melting / freezing (supcol from the temperature on entry)
  T supcol = F(T0C) - t;
  T xlf3 = F(XLS) - xl;
  if (val(supcol) < 0.f && val(qi) > 0.f) {
    qc = qc + qi;
    t = t - xlf3 / cpm * qi;
    qi = zero;
  }
  if (val(supcol) > 40.f && val(qc) > 0.f) {
    qi = qi + qc;
    t = t + xlf3 / cpm * qc;
    qc = zero;
  }
  if (val(supcol) > 0.f && val(qc) > F(QMIN)) {
    const T pf = vmin(F(PFRZ1) * (vexp(F(PFRZ2) * vmin(supcol, 50.0f)) - 1.0f) * den / F(DENR) / F(XNCR) * qc * qc *
                          dtcld, qc);
    qi = qi + pf;
    t = t + xlf3 / cpm * pf;
    qc = qc - pf;
  }
  if (val(supcol) > 0.f && val(qr) > 0.f) {
    const T pf = vmin(F(20.0 * PI * PI * PFRZ1 * N0R * DENR) / den * (vexp(F(PFRZ2) * vmin(supcol, 50.0f)) - 1.0f) *
                          sl0.r3[0] * sl0.r3[0] * sl0.rs[0] * dtcld, qr);
    qg = qg + pf;
    t = t + xlf3 / cpm * pf;
    qr = qr - pf;
  }
  // rates
  Slope3<T> sl;
  slope3(qr, qs, qg, den, t, sl);
  const T work1_0 = diffac(xl, p, t, den, qs0);
  const T work1_1 = diffac(F(XLS), p, t, den, qs1);
  T work2 = venfac(p, t, den);
  T supsat = vmax(q, F(QMIN)) - qs0;
  T praut = zero, pracw = zero, prevp = zero;
  if (val(qc) > F(QC0)) praut = vmin(F(QCK1) * vpow(qc, 7.0f / 3.0f), qc / dtcld);
  if (val(qr) > F(QCRMIN) && val(qc) > F(QMIN))
    pracw = vmin(F(PACRR) * sl.r3[0] * sl.rb[0] * qc * denfac, qc / dtcld);
  if (val(qr) > 0.f) {
    const T coeres = sl.r2[0] * vsqrt(sl.rs[0] * sl.rb[0]);
    prevp = (rh0 - 1.0f) * (F(PRECR1) * sl.r2[0] + F(PRECR2) * work2 * coeres) / work1_0;
    if (val(prevp) < 0.f) {
      prevp = vmax(prevp, -qr / dtcld);
      prevp = vmax(prevp, supsat / dtcld / 2.0f);
    } else {
      prevp = vmin(prevp, supsat / dtcld / 2.0f);
    }
  }
  supcol = F(T0C) - t;
  const T n0s = vmax(vmin(vexp(F(ALPHA) * supcol), F(N0SMAX / N0S)), 1.0f);
  supsat = vmax(q, F(QMIN)) - qs1;
  const T satdt = supsat / dtcld;
  bool ifsat = false;
  const T xni = vmin(vmax(5.38e7f * vpow(den * vmax(qi, F(QMIN)), 0.75f), 1.0e3f), 1.0e6f);
  const T eacrs = vexp(0.07f * (-supcol));
  const T xmi = den * qi / xni;
  const T diameter = vmin(F(DICON) * vsqrt(xmi), F(DIMAX));
  const T vt2i = 1.49e4f * vpow(diameter, 1.31f);
  const T vt2r = F(PVTR) * sl.rb[0] * denfac;
  const T vt2s = F(PVTS) * sl.rb[1] * denfac;
  const T vt2g = F(PVTG) * sl.rb[2] * denfac;
  const T qsum = vmax(qs + qg, 1.0e-15f);
  const T vt2ave = val(qsum) > 1.0e-15f ? (vt2s * qs + vt2g * qg) / qsum : zero;
  T praci = zero, piacr = zero, psaci = zero, pgaci = zero, psacw = zero, pgacw = zero, paacw = zero;
  T pracs = zero, psacr = zero, pgacr = zero, pgacs = zero, pseml = zero, pgeml = zero;
  T pidep = zero, psdep = zero, pgdep = zero, pigen = zero, psaut = zero, pgaut = zero, psevp = zero, pgevp = zero;
  const bool cold = val(supcol) > 0.f;
  if (cold && val(qi) > F(QMIN)) {
    if (val(qr) > F(QCRMIN)) {
      const T acrfac = 2.0f * sl.r3[0] + 2.0f * diameter * sl.r2[0] + diameter * diameter * sl.rs[0];
      praci = vmin(F(PI) * qi * F(N0R) * vabs(vt2r - vt2i) * acrfac, qi / dtcld);
      piacr = vmin(F(PI * PI * AVTR * N0R * DENR) * xni * denfac * F(G6PBR) * (sl.r3[0] * sl.r3[0]) * sl.rb[0] /
                       24.0f / den,
                   qr / dtcld);
    }
    if (val(qs) > F(QCRMIN)) {
      const T acrfac = 2.0f * sl.r3[1] + 2.0f * diameter * sl.r2[1] + diameter * diameter * sl.rs[1];
      psaci = vmin(F(PI) * qi * eacrs * F(N0S) * n0s * vabs(vt2ave - vt2i) * acrfac / 4.0f, qi / dtcld);
    }
    if (val(qg) > F(QCRMIN)) {
      const T egi = vexp(-0.07f * supcol);
      const T acrfac = 2.0f * sl.r3[2] + 2.0f * diameter * sl.r2[2] + diameter * diameter * sl.rs[2];
      pgaci = vmin(F(PI) * egi * qi * F(N0G) * vabs(vt2ave - vt2i) * acrfac / 4.0f, qi / dtcld);
    }
  }
  if (val(qs) > F(QCRMIN) && val(qc) > F(QMIN))
    psacw = vmin(F(PACRC) * n0s * sl.r3[1] * sl.rb[1] * qc * denfac, qc / dtcld);
  if (val(qg) > F(QCRMIN) && val(qc) > F(QMIN)) pgacw = vmin(F(PACRC) * sl.r3[2] * sl.rb[2] * qc * denfac, qc / dtcld);
  if (val(qsum) > 1.0e-15f) paacw = (qs * psacw + qg * pgacw) / qsum;
  if (val(qs) > F(QCRMIN) && val(qr) > F(QCRMIN)) {
    if (cold) {
      const T acrfac = 5.0f * (sl.r3[1] * sl.r3[1]) * sl.rs[0] + 2.0f * sl.r3[1] * sl.r2[1] * sl.r2[0] +
                       0.5f * (sl.r2[1] * sl.r2[1]) * sl.r3[0];
      pracs = vmin(F(PI * PI * N0R * N0S) * n0s * vabs(vt2r - vt2ave) * (F(DENS) / den) * acrfac, qs / dtcld);
    }
    const T acrfac = 5.0f * (sl.r3[0] * sl.r3[0]) * sl.rs[1] + 2.0f * sl.r3[0] * sl.r2[0] * sl.r2[1] +
                     0.5f * (sl.r2[0] * sl.r2[0]) * sl.r3[1];
    psacr = vmin(F(PI * PI * N0R * N0S) * n0s * vabs(vt2r - vt2ave) * (F(DENR) / den) * acrfac, qr / dtcld);
  }
  if (val(qg) > F(QCRMIN) && val(qr) > F(QCRMIN)) {
    const T acrfac = 5.0f * (sl.r3[0] * sl.r3[0]) * sl.rs[2] + 2.0f * sl.r3[0] * sl.r2[0] * sl.r2[2] +
                     0.5f * (sl.r2[0] * sl.r2[0]) * sl.r3[2];
    pgacr = vmin(F(PI * PI * N0R * N0G) * vabs(vt2r - vt2ave) * (F(DENR) / den) * acrfac, qr / dtcld);
  }
  if (!cold) {  // supcol <= 0
    const T melt = F(CLIQ) * supcol * (paacw + psacr) / F(XLF0);
    if (val(qs) > 0.f) pseml = vmin(vmax(melt, -qs / dtcld), 0.0f);
    if (val(qg) > 0.f) pgeml = vmin(vmax(melt, -qg / dtcld), 0.0f);
  }
  if (cold) {
    if (val(qi) > 0.f && !ifsat) {
      pidep = 4.0f * diameter * xni * (rh1 - 1.0f) / work1_1;
      const T supice = satdt - prevp;
      if (val(pidep) < 0.f)
        pidep = vmax(vmax(vmax(pidep, satdt / 2.0f), supice), -qi / dtcld);
      else
        pidep = vmin(vmin(pidep, satdt / 2.0f), supice);
      if (fabsf(val(prevp + pidep)) >= fabsf(val(satdt))) ifsat = true;
    }
    if (val(qs) > 0.f && !ifsat) {
      const T coeres = sl.r2[1] * vsqrt(sl.rs[1] * sl.rb[1]);
      psdep = (rh1 - 1.0f) * n0s * (F(PRECS1) * sl.r2[1] + F(PRECS2) * work2 * coeres) / work1_1;
      const T supice = satdt - prevp - pidep;
      if (val(psdep) < 0.f)
        psdep = vmax(vmax(vmax(psdep, -qs / dtcld), satdt / 2.0f), supice);
      else
        psdep = vmin(vmin(psdep, satdt / 2.0f), supice);
      if (fabsf(val(prevp + pidep + psdep)) >= fabsf(val(satdt))) ifsat = true;
    }
    if (val(qg) > 0.f && !ifsat) {
      const T coeres = sl.r2[2] * vsqrt(sl.rs[2] * sl.rb[2]);
      pgdep = (rh1 - 1.0f) * (F(PRECG1) * sl.r2[2] + F(PRECG2) * work2 * coeres) / work1_1;
      const T supice = satdt - prevp - pidep - psdep;
      if (val(pgdep) < 0.f)
        pgdep = vmax(vmax(vmax(pgdep, -qg / dtcld), satdt / 2.0f), supice);
      else
        pgdep = vmin(vmin(pgdep, satdt / 2.0f), supice);
      if (fabsf(val(prevp + pidep + psdep + pgdep)) >= fabsf(val(satdt))) ifsat = true;
    }
    if (val(supsat) > 0.f && !ifsat) {
      const T supice = satdt - prevp - pidep - psdep - pgdep;
      const T roqi0 = 4.92e-11f * vpow(1.0e3f * vexp(0.1f * supcol), 1.33f);
      T pg = vmax(0.0f, (roqi0 / den - vmax(qi, 0.0f)) / dtcld);
      pigen = vmin(vmin(pg, satdt), supice);
    }
    if (val(qi) > 0.f) psaut = vmax(0.0f, (qi - F(ROQIMAX) / den) / dtcld);
    if (val(qs) > 0.f) pgaut = vmin(vmax(0.0f, 1.0e-3f * vexp(-0.09f * supcol) * (qs - F(QS0))), qs / dtcld);
  }
  if (val(supcol) < 0.f && val(rh0) < 1.f) {
    if (val(qs) > 0.f) {
      const T coeres = sl.r2[1] * vsqrt(sl.rs[1] * sl.rb[1]);
      psevp = vmin(vmax((rh0 - 1.0f) * n0s * (F(PRECS1) * sl.r2[1] + F(PRECS2) * work2 * coeres) / work1_0,
                        -qs / dtcld),
                   0.0f);
    }
    if (val(qg) > 0.f) {
      const T coeres = sl.r2[2] * vsqrt(sl.rs[2] * sl.rb[2]);
      pgevp = vmin(vmax((rh0 - 1.0f) * (F(PRECG1) * sl.r2[2] + F(PRECG2) * work2 * coeres) / work1_0, -qg / dtcld),
                   0.0f);
    }
  }
  // limiters and update, T <= t0c
  const float delta2 = (val(qr) < 1.0e-4f && val(qs) < 1.0e-4f) ? 1.f : 0.f;
  const float delta3 = val(qr) < 1.0e-4f ? 1.f : 0.f;
  bool cnd = val(t) <= F(T0C);
  {
    T* const r1[3] = {&praut, &pracw, &paacw};
    limit(vmax(F(QMIN), qc), (praut + pracw + paacw + paacw) * dtcld, cnd, r1);
    T* const r2[6] = {&psaut, &pigen, &pidep, &praci, &psaci, &pgaci};
    limit(vmax(F(QMIN), qi), (psaut - pigen - pidep + praci + psaci + pgaci) * dtcld, cnd, r2);
    T* const r3[6] = {&praut, &prevp, &pracw, &piacr, &psacr, &pgacr};
    limit(vmax(F(QMIN), qr), (-praut - prevp - pracw + piacr + psacr + pgacr) * dtcld, cnd, r3);
    const T src4 = -(psdep + psaut - pgaut + paacw + piacr * delta3 + praci * delta3 - pracs * (1.0f - delta2) +
                     psacr * delta2 + psaci - pgacs) * dtcld;
    T* const r4[10] = {&psdep, &psaut, &pgaut, &paacw, &piacr, &praci, &psaci, &pracs, &psacr, &pgacs};
    limit(vmax(F(QMIN), qs), src4, cnd, r4);
    const T src5 = -(pgdep + pgaut + piacr * (1.0f - delta3) + praci * (1.0f - delta3) + psacr * (1.0f - delta2) +
                     pracs * (1.0f - delta2) + pgaci + paacw + pgacr + pgacs) * dtcld;
    T* const r5[10] = {&pgdep, &pgaut, &piacr, &praci, &psacr, &pracs, &paacw, &pgaci, &pgacr, &pgacs};
    limit(vmax(F(QMIN), qg), src5, cnd, r5);
  }
  if (cnd) {
    work2 = -(prevp + psdep + pgdep + pigen + pidep);
    q = q + work2 * dtcld;
    qc = vmax(qc - (praut + pracw + paacw + paacw) * dtcld, 0.0f);
    qr = vmax(qr + (praut + pracw + prevp - piacr - pgacr - psacr) * dtcld, 0.0f);
    qi = vmax(qi - (psaut + praci + psaci + pgaci - pigen - pidep) * dtcld, 0.0f);
    qs = vmax(qs + (psdep + psaut + paacw - pgaut + piacr * delta3 + praci * delta3 + psaci - pgacs -
                    pracs * (1.0f - delta2) + psacr * delta2) * dtcld,
              0.0f);
    qg = vmax(qg + (pgdep + pgaut + piacr * (1.0f - delta3) + praci * (1.0f - delta3) + psacr * (1.0f - delta2) +
                    pracs * (1.0f - delta2) + pgaci + paacw + pgacr + pgacs) * dtcld,
              0.0f);
    xlf3 = F(XLS) - xl;
    const T xlwork2 = -F(XLS) * (psdep + pgdep + pidep + pigen) - xl * prevp -
                      xlf3 * (piacr + paacw + paacw + pgacr + psacr);
    t = t - xlwork2 / cpm * dtcld;
  }
  // T > t0c
  cnd = val(t) > F(T0C);
  {
    T* const r1[3] = {&praut, &pracw, &paacw};
    limit(vmax(F(QMIN), qc), (praut + pracw + paacw + paacw) * dtcld, cnd, r1);
    T* const r2[6] = {&praut, &prevp, &pracw, &paacw, &pseml, &pgeml};
    limit(vmax(F(QMIN), qr), (-paacw - praut + pseml + pgeml - pracw - paacw - prevp) * dtcld, cnd, r2);
    T* const r3[3] = {&pgacs, &psevp, &pseml};
    limit(vmax(F(QCRMIN), qs), (pgacs - pseml - psevp) * dtcld, cnd, r3);
    T* const r4[3] = {&pgacs, &pgevp, &pgeml};
    limit(vmax(F(QCRMIN), qg), -(pgacs + pgevp + pgeml) * dtcld, cnd, r4);
  }
  if (cnd) {
    work2 = -(prevp + psevp + pgevp);
    q = q + work2 * dtcld;
    qc = vmax(qc - (praut + pracw + paacw + paacw) * dtcld, 0.0f);
    qr = vmax(qr + (praut + pracw + prevp + paacw + paacw - pseml - pgeml) * dtcld, 0.0f);
    qs = vmax(qs + (psevp - pgacs + pseml) * dtcld, 0.0f);
    qg = vmax(qg + (pgacs + pgevp + pgeml) * dtcld, 0.0f);
    xlf3 = F(XLS) - xl;
    const T xlwork2 = -xl * (prevp + psevp + pgevp) - xlf3 * (pseml + pgeml);
    t = t - xlwork2 / cpm * dtcld;
  }
  // saturation adjustment
  T a0, a1;
  fpvs(t, p, a0, a1);
  const T w1 = (vmax(q, F(QMIN)) - a0) / (1.0f + xl * xl / (F(RV) * cpm) * a0 / (t * t));
  T pcond = vmin(vmax(w1 / dtcld, 0.0f), vmax(q, 0.0f) / dtcld);
  if (val(qc) > 0.f && val(w1) < 0.f) pcond = vmax(w1, -qc) / dtcld;
  q = q - pcond * dtcld;
  qc = vmax(qc + pcond * dtcld, 0.0f);
  t = t + pcond * xl / cpm * dtcld;
  if (val(qc) <= F(QMIN)) qc = zero;
  if (val(qi) <= F(QMIN)) qi = zero;
}

// wsm6 (wrf_physics.py:137-1214) on one column of km levels: the arrays
// A_T (temperature), A_Q, A_QC, A_QI, A_QR, A_QS, A_QG, A_DEN, A_P and
// A_DELZ hold the inputs and receive the results
template <class T>
__device__ void wsm6_column(const Col<T>& C, int km, float delt, bool skip_dead = false, bool stop_at_points = false) {
  for (int k = 0; k < km; ++k) {
    const T q = C(A_Q, k), t = C(A_T, k);
    C(A_CPM, k) = val(q) >= F(QMIN) ? F(CPV) * q + (1.0f - q) * F(CPD) : cst<T>(F(CPD * (1.0 - QMIN) + CPV * QMIN));
    C(A_XL, k) = F(XLV0) - F(XLV1) * (t - F(T0C));
    C(A_QC, k) = vmax(C(A_QC, k), 0.0f);
    C(A_QI, k) = vmax(C(A_QI, k), 0.0f);
    C(A_QR, k) = vmax(C(A_QR, k), 0.0f);
    C(A_QS, k) = vmax(C(A_QS, k), 0.0f);
    C(A_QG, k) = vmax(C(A_QG, k), 0.0f);
  }
  const float loops = fmaxf(delt / F(DTCLDCR), 1.0f);
  const float dtcld = delt <= F(DTCLDCR) ? delt : delt / loops;
  const int nloop = (int)loops;
  for (int it = 0; it < nloop; ++it) {
    for (int k = 0; k < km; ++k) {
      const T den = C(A_DEN, k), t = C(A_T, k), q = C(A_Q, k);
      const T denfac = vsqrt(1.0f / den * F(DEN0));
      C(A_DENFAC, k) = denfac;
      T qs0, qs1;
      fpvs(t, C(A_P, k), qs0, qs1);
      C(A_QS0, k) = qs0;
      C(A_QS1, k) = qs1;
      C(A_RH0, k) = vmax(q / qs0, F(QMIN));
      C(A_RH1, k) = vmax(q / qs1, F(QMIN));
      C(A_XNI, k) = vmin(vmax(5.387e7f * vpow(den * vmax(C(A_QI, k), F(QMIN)), 0.75f), 1.0e3f), 1.0e6f);
      const T qr = C(A_QR, k), qs = C(A_QS, k), qg = C(A_QG, k);
      C(A_W1, k) = vt_of(0, qr, den, denfac, t);
      const T qsum = vmax(qs + qg, 1.0e-15f);
      C(A_W2, k) = val(qsum) > 1.0e-15f
                       ? (vt_of(1, qs, den, denfac, t) * qs + vt_of(2, qg, den, denfac, t) * qg) / qsum
                       : cst<T>(0.f);
      C(A_R1, k) = den * qr;
      C(A_R2, k) = den * qs;
      C(A_R3, k) = den * qg;
    }
    nislfv(C, km, 0, A_R1, -1, dtcld, 1);
    for (int k = 0; k < km; ++k) C(A_W1, k) = C(A_W2, k);
    nislfv(C, km, 1, A_R2, A_R3, dtcld, 1);
    const float xlf = F(XLF0);
    for (int k = 0; k < km; ++k) {
      const T den = C(A_DEN, k), p = C(A_P, k), cpm = C(A_CPM, k);
      T qr = vmax(C(A_R1, k) / den, 0.0f), qs = vmax(C(A_R2, k) / den, 0.0f), qg = vmax(C(A_R3, k) / den, 0.0f);
      T t = C(A_T, k);
      Slope3<T> sl;
      slope3(qr, qs, qg, den, t, sl);
      C(A_SR3, k) = sl.r3[0];
      C(A_SRS, k) = sl.rs[0];
      const T n0s = n0sfac(t);
      // melting of snow, then graupel
      const bool warm = val(t) > F(T0C);
      if (warm) {
        const T work2 = venfac(p, t, den);
        if (val(qs) > 0.f) {
          const T coeres = sl.r2[1] * vsqrt(sl.rs[1] * sl.rb[1]);
          T ps = xka(t, den) / xlf * (F(T0C) - t) * F(PI) / 2.0f * n0s *
                 (F(PRECS1) * sl.r2[1] + F(PRECS2) * work2 * coeres) / den;
          ps = vmin(vmax(ps * dtcld / 1.0f, -qs / 1.0f), 0.0f);
          qs = qs + ps;
          qr = qr - ps;
          t = t + xlf / cpm * ps;
        }
        if (val(qg) > 0.f) {
          const T coeres = sl.r2[2] * vsqrt(sl.rs[2] * sl.rb[2]);
          T pg = xka(t, den) / xlf * (F(T0C) - t) * (F(PRECG1) * sl.r2[2] + F(PRECG2) * work2 * coeres) / den;
          pg = vmin(vmax(pg * dtcld / 1.0f, -qg / 1.0f), 0.0f);
          qg = qg + pg;
          qr = qr - pg;
          t = t + xlf / cpm * pg;
        }
      }
      C(A_QR, k) = qr;
      C(A_QS, k) = qs;
      C(A_QG, k) = qg;
      C(A_T, k) = t;
      // cloud-ice fall speed and mass
      const T qi = C(A_QI, k);
      if (val(qi) <= 0.f) {
        C(A_W1, k) = cst<T>(0.f);
      } else {
        T wt = vmax(vmin(F(DICON) * vsqrt(den * qi / C(A_XNI, k)), F(DIMAX)), 1.0e-25f);
        C(A_W1, k) = 1.49e4f * vexp(vlog(wt) * 1.31f);
      }
      C(A_R1, k) = den * qi;
    }
    nislfv(C, km, 2, A_R1, -1, dtcld, 0);
    if (stop_at_points) {
      // (one time-split loop only) the point processes' inputs stay in the
      // column arrays, cloud ice from its sedimented mass in A_QI
      for (int k = 0; k < km; ++k) C(A_QI, k) = vmax(C(A_R1, k) / C(A_DEN, k), 0.0f);
      return;
    }
    for (int k = 0; k < km; ++k) {
      T t = C(A_T, k), q = C(A_Q, k), qc = C(A_QC, k), qr = C(A_QR, k), qs = C(A_QS, k), qg = C(A_QG, k);
      const T den = C(A_DEN, k);
      T qi = vmax(C(A_R1, k) / den, 0.0f);
      // a level whose every operand has zero tangents keeps zero tangents
      // through the processes; its values are not needed when only the
      // derivatives are wanted and no later time-split loop reads them
      if (skip_dead && it == nloop - 1 && !(live(t) || live(q) || live(qc) || live(qr) || live(qs) || live(qg) || live(den) ||
                         live(qi) || live(C(A_P, k)) || live(C(A_DENFAC, k)) || live(C(A_CPM, k)) ||
                         live(C(A_XL, k)) || live(C(A_QS0, k)) || live(C(A_QS1, k)) || live(C(A_RH0, k)) ||
                         live(C(A_RH1, k)) || live(C(A_SR3, k)) || live(C(A_SRS, k))))
        continue;
      Slope3<T> sl0;
      sl0.r3[0] = C(A_SR3, k);
      sl0.rs[0] = C(A_SRS, k);
      point_processes(t, q, qc, qi, qr, qs, qg, den, C(A_P, k), C(A_DENFAC, k), C(A_CPM, k), C(A_XL, k),
                      C(A_QS0, k), C(A_QS1, k), C(A_RH0, k), C(A_RH1, k), sl0, dtcld);
      C(A_T, k) = t;
      C(A_Q, k) = q;
      C(A_QC, k) = qc;
      C(A_QI, k) = qi;
      C(A_QR, k) = qr;
      C(A_QS, k) = qs;
      C(A_QG, k) = qg;
    }
  }
}

// the columns of moist_physics_prep_em's block ([jds+1, jde-1) x [ids+1,
// ide-1)), numbered row by row; WSM6 runs on [jds+1, jde-2) x [ids+1,
// ide-2) of them (run), the others only take the prep and finish
struct ColPos {
  int c2;
  bool run;
};
__device__ __forceinline__ bool col_pos(const Grid& g, int col, ColPos& o) {
  const int wi = g.ide - 1 - (g.ids + 1), wj = g.jde - 1 - (g.jds + 1);
  if (col >= wi * wj) return false;
  const int j = g.jds + 1 + col / wi, i = g.ids + 1 + col % wi;
  o.c2 = g.i2(j, i);
  o.run = j < g.jde - 2 && i < g.ide - 2;
  return true;
}

// the column's inputs are numbered t, qv, qc, qr, qi, qs, qg, al, p at
// levels < km (9 km indices: field f at level k is f km + k), then ph at
// levels < km + 1
__host__ __device__ __forceinline__ int mp_inputs(const Grid& g) { return 9 * (g.nz - 1) + g.nz; }

// moist_physics_prep_em (wrf_physics.py:27-91): theta, Exner function,
// temperature, density, pressure and layer depths of the column and its
// moisture into the column arrays; in(idx, value) makes input idx
template <class T, class In>
__device__ void prep_column(const Grid& g, const S& s, const Col<T>& C, int c2, In in) {
  const int km = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const int slot_of[6] = {A_Q, A_QC, A_QR, A_QI, A_QS, A_QG};
  for (int k = 0; k < km; ++k) {
    const size_t p = k * lev + c2;
    const T tin = in(k, s[WF_T][p]);
    C(A_TIN, k) = tin;
    const T th = tin + (float)T0;
    C(A_TH, k) = th;
    const T pfull = in(8 * km + k, s[WF_P][p]) + s[WF_PB][p];
    const T pii = vpow(pfull / (float)P0, F(RCP));
    C(A_PII, k) = pii;
    C(A_T, k) = th * pii;
    C(A_DEN, k) = 1.0f / (in(7 * km + k, s[WF_AL][p]) + s[WF_ALB][p]);
    C(A_P, k) = pfull;
    const T zlo = (in(9 * km + k, s[WF_PH][p]) + s[WF_PHB][p]) / (float)G;
    const T zhi = (in(9 * km + k + 1, s[WF_PH][p + lev]) + s[WF_PHB][p + lev]) / (float)G;
    C(A_DELZ, k) = zhi - zlo;
    for (int m = 1; m < 7; ++m) C(slot_of[m - 1], k) = in(m * km + k, s[WF_MOIST][m * n3 + p]);
  }
}

// moist_physics_finish_em (wrf_physics.py:2106-2137) at level k: theta's
// new value replaces A_TIN, h_diabatic replaces A_TH
template <class T>
__device__ __forceinline__ void finish_level(const Col<T>& C, int k, float dt) {
  const T mpten = C(A_T, k) / C(A_PII, k) - C(A_TH, k);
  C(A_TIN, k) = C(A_TIN, k) + mpten;
  C(A_TH, k) = mpten / dt;
}

// the array holding moist species m (1 qv .. 6 qg) in the column
__device__ __forceinline__ int moist_slot(int m) {
  const int slot_of[6] = {A_Q, A_QC, A_QR, A_QI, A_QS, A_QG};
  return slot_of[m - 1];
}

// a column that takes no process at all: no cloud, rain, ice, snow or
// graupel at any level, and qv below both saturation mixing ratios
// everywhere.  Every rate is zero, nothing falls, the saturation adjustment
// condenses nothing, and its reverse product is theta's and qv's
// cotangents passed through, zero for the hydrometeors (their results are
// constants: the zero of the empty sedimentation and the final zeroing of
// cloud and ice) and for h_diabatic.
__device__ bool quiet_column(const Grid& g, const S& s, int c2) {
  const int km = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  for (int k = 0; k < km; ++k) {
    const size_t p = k * lev + c2;
    for (int m = 2; m < 7; ++m)
      if (s[WF_MOIST][m * n3 + p] > 0.f) return false;
    const float th = s[WF_T][p] + (float)T0;
    const float pfull = s[WF_P][p] + s[WF_PB][p];
    const float t = th * wpow(pfull / (float)P0, F(RCP));
    float qs0, qs1;
    fpvs(t, pfull, qs0, qs1);
    const float qv = s[WF_MOIST][n3 + p];
    if (!(qv < qs0 && qv < qs1)) return false;
  }
  return true;
}

// the cotangent v of input idx into the cotangent table: assigned for t and
// the moisture (the block overwrites them), added for al, p and ph
__device__ __forceinline__ void put_input_cot(const Grid& g, const S& b, int c2, int idx, float v) {
  const int km = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  if (idx >= 9 * km) {
    b[WF_PH][(size_t)(idx - 9 * km) * lev + c2] += v;
    return;
  }
  const int f = idx / km, k = idx - f * km;
  const size_t p = k * lev + c2;
  if (f == 0) b[WF_T][p] = v;
  else if (f < 7) b[WF_MOIST][f * n3 + p] = v;
  else if (f == 7) b[WF_AL][p] += v;
  else b[WF_P][p] += v;
}

// the taped forward over the columns [c0, c0 + nc) (lane l of the launch
// takes column c0 + l; tape and column arrays interleaved with the
// context's stride): the column runs once on taped scalars and the
// outputs' cotangents yb (theta, qv .. qg, h_diabatic) seed their entries'
// adjoints.  Columns outside WSM6's block pass t and q through and set
// h_diabatic to zero; quiet columns pass theta's and qv's cotangents
// through (unless the values are wanted); both are done here.  vo (when
// its T is not null) receives the outputs' values.  used[col] receives the
// entries the column's tape took (0 when none) and done[col] whether its
// cotangents are (or, after k_mp_tape_rev, will be) written: not when the
// tape outgrew the capacity.
__global__ void __launch_bounds__(kTapeBlock) k_mp_tape(Grid g, S s, S yb, S b, float dt, Tv* ws, TapeCtx tc,
                                                        int c0, int nc, S vo, int* done, int* used, bool split) {
  if (threadIdx.x == 0) g_tape = tc;
  __syncthreads();
  const int lane = tape_lane(), col = c0 + lane;
  ColPos cp;
  if (lane >= nc || !col_pos(g, col, cp)) return;
  const int km = g.nz - 1, c2 = cp.c2;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const bool want = vo[WF_T] != nullptr;
  used[col] = 0;
  done[col] = 1;
  if (!cp.run) {
    for (int k = 0; k < km; ++k) {
      const size_t p = k * lev + c2;
      b[WF_T][p] = yb[WF_T][p];
      for (int m = 1; m < 7; ++m) b[WF_MOIST][m * n3 + p] = yb[WF_MOIST][m * n3 + p];
      b[WF_H_DIABATIC][p] = 0.f;
      if (want) {
        vo[WF_T][p] = s[WF_T][p];
        for (int m = 1; m < 7; ++m) vo[WF_MOIST][m * n3 + p] = s[WF_MOIST][m * n3 + p];
        vo[WF_H_DIABATIC][p] = 0.f;
      }
    }
    return;
  }
  if (!want && quiet_column(g, s, c2)) {
    for (int k = 0; k < km; ++k) {
      const size_t p = k * lev + c2;
      b[WF_T][p] = yb[WF_T][p];
      b[WF_MOIST][n3 + p] = yb[WF_MOIST][n3 + p];
      for (int m = 2; m < 7; ++m) b[WF_MOIST][m * n3 + p] = 0.f;
      b[WF_H_DIABATIC][p] = 0.f;
    }
    return;
  }
  const Col<Tv> C{ws + lane, tc.stride, km + 1};
  tape_reserve(mp_inputs(g));
  prep_column(g, s, C, c2, [](int idx, float v) { return Tv{v, idx, 1.f}; });
  if (split) {
    // the point processes and finish are reversed per level by
    // k_mp_points_adj, which seeds this tape's entries
    wsm6_column(C, km, dt, false, true);
    const int n = g_tape_n[threadIdx.x];
    used[col] = n;
    for (int k = 0; k < km; ++k) b[WF_H_DIABATIC][k * lev + c2] = 0.f;
    if (n > tc.cap) done[col] = 0;
    return;
  }
  wsm6_column(C, km, dt);
  for (int k = 0; k < km; ++k) finish_level(C, k, dt);
  const int n = g_tape_n[threadIdx.x];
  used[col] = n;
  if (want)
    for (int k = 0; k < km; ++k) {
      const size_t p = k * lev + c2;
      vo[WF_T][p] = C(A_TIN, k).v;
      vo[WF_H_DIABATIC][p] = C(A_TH, k).v;
      for (int m = 1; m < 7; ++m) vo[WF_MOIST][m * n3 + p] = C(moist_slot(m), k).v;
    }
  for (int k = 0; k < km; ++k) b[WF_H_DIABATIC][k * lev + c2] = 0.f;
  if (n > tc.cap) {
    done[col] = 0;
    return;
  }
  auto seed = [&](const Tv& y, float w) {
    if (y.id >= 0 && w != 0.f) *tc.adj(y.id, lane) += w * y.s;
  };
  for (int k = 0; k < km; ++k) {
    const size_t p = k * lev + c2;
    seed(C(A_TIN, k), yb[WF_T][p]);
    seed(C(A_TH, k), yb[WF_H_DIABATIC][p]);
    for (int m = 1; m < 7; ++m) seed(C(moist_slot(m), k), yb[WF_MOIST][m * n3 + p]);
  }
}

// The point processes and finish of one level of a column taped in split
// mode, reversed by forward-mode tangents: one thread per (column, level)
// reads the level's inputs from the column arrays k_mp_tape left (their
// values, and the tape entries they are multiples of), evaluates the level
// in Dual<N> arithmetic with N inputs seeded per pass, forms the inputs'
// cotangents from the outputs' (yb: theta, qv .. qg, h_diabatic) and adds
// them into the adjoints of those entries of the column's tape, which
// k_mp_tape_rev then sweeps.  The level's processes read no other level, so
// the chain a thread runs is one level's, not the column's.  vo (when its T
// is not null) receives the level's output values.
constexpr int kPointInputs = 21;
template <int N>
__global__ void __launch_bounds__(128) k_mp_points_adj(Grid g, S yb, Tv* ws, TapeCtx tc, int c0, int nc, S vo,
                                                       const int* done, const int* used, float dt) {
  const int km = g.nz - 1;
  // neighbouring threads take neighbouring columns at one level: their
  // column-array reads coalesce, and their branches mostly agree
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int k = (int)(t / nc), lane = (int)(t - (long long)k * nc);
  if (k >= km) return;
  const int col = c0 + lane;
  const int n = used[col];
  if (!done[col] || n == 0 || n > tc.cap) return;
  ColPos cp;
  col_pos(g, col, cp);
  const Col<Tv> C{ws + lane, tc.stride, km + 1};
  const int arr[kPointInputs] = {A_T,  A_Q,   A_QC,  A_QI,  A_QR,  A_QS,  A_QG,  A_DEN, A_P,  A_DENFAC, A_CPM,
                                 A_XL, A_QS0, A_QS1, A_RH0, A_RH1, A_SR3, A_SRS, A_TIN, A_TH, A_PII};
  Tv in[kPointInputs];
#pragma unroll
  for (int q = 0; q < kPointInputs; ++q) in[q] = C(arr[q], k);
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3(), p = k * lev + cp.c2;
  const float yt = yb[WF_T][p], yh = yb[WF_H_DIABATIC][p];
  float ym[7];
#pragma unroll
  for (int m = 1; m < 7; ++m) ym[m] = yb[WF_MOIST][m * n3 + p];
  float cot[kPointInputs];
#pragma unroll
  for (int q = 0; q < kPointInputs; ++q) cot[q] = 0.f;
  // the time-split loop's step (one loop: dt itself up to the split step)
  const float loops = fmaxf(dt / F(DTCLDCR), 1.0f);
  const float dtcld = dt <= F(DTCLDCR) ? dt : dt / loops;
  using D = Dual<N>;
  for (int j0 = 0; j0 < kPointInputs; j0 += N) {
    D x[kPointInputs];
#pragma unroll
    for (int q = 0; q < kPointInputs; ++q) {
      x[q] = dconst<N>(in[q].v);
#pragma unroll
      for (int d = 0; d < N; ++d)
        if (q == j0 + d) x[q].d[d] = 1.f;
    }
    D tt = x[0], qv = x[1], qc = x[2], qi = x[3], qr = x[4], qs = x[5], qg = x[6];
    Slope3<D> sl0;
    sl0.r3[0] = x[16];
    sl0.rs[0] = x[17];
    point_processes(tt, qv, qc, qi, qr, qs, qg, x[7], x[8], x[9], x[10], x[11], x[12], x[13], x[14], x[15], sl0, dtcld);
    // moist_physics_finish_em at the level
    const D mpten = tt / x[20] - x[19];
    const D tnew = x[18] + mpten;
    const D h = mpten / dt;
#pragma unroll
    for (int d = 0; d < N; ++d) {
      const float v = yt * tnew.d[d] + yh * h.d[d] + ym[1] * qv.d[d] + ym[2] * qc.d[d] + ym[3] * qr.d[d] +
                      ym[4] * qi.d[d] + ym[5] * qs.d[d] + ym[6] * qg.d[d];
#pragma unroll
      for (int q = 0; q < kPointInputs; ++q)
        if (q == j0 + d) cot[q] += v;
    }
    if (j0 == 0 && vo[WF_T]) {
      vo[WF_T][p] = tnew.v;
      vo[WF_H_DIABATIC][p] = h.v;
      const float mv[7] = {0.f, qv.v, qc.v, qr.v, qi.v, qs.v, qg.v};
      for (int m = 1; m < 7; ++m) vo[WF_MOIST][m * n3 + p] = mv[m];
    }
  }
#pragma unroll
  for (int q = 0; q < kPointInputs; ++q)
    if (in[q].id >= 0 && cot[q] != 0.f) atomicAdd(tc.adj(in[q].id, lane), cot[q] * in[q].s);
}

// the reverse sweep of the tapes k_mp_tape left (same chunk and lanes):
// the inputs' cotangents from the adjoints of entries [0, n_inputs)
constexpr int kSweepBlock = 128, kSweepWindow = 16, kSweepRing = 64;
__global__ void __launch_bounds__(kSweepBlock) k_mp_tape_rev(Grid g, S b, TapeCtx tc, int c0, int nc,
                                                             const int* used) {
  __shared__ float acc[kSweepRing * kSweepBlock];
  const int lane = blockIdx.x * blockDim.x + threadIdx.x, col = c0 + lane;
  ColPos cp;
  if (lane >= nc || !col_pos(g, col, cp)) return;
  const int n = used[col];
  if (n == 0 || n > tc.cap) return;
  const int nin = mp_inputs(g);
  tape_sweep<kSweepWindow, kSweepRing, kSweepBlock>(tc, lane, nin, n, acc);
  for (int idx = 0; idx < nin; ++idx) put_input_cot(g, b, cp.c2, idx, __ldcg(tc.adj(idx, lane)));
}

// one pass of forward-mode tangents over the columns that the tape left
// undone: the inputs with indices [pass N, pass N + N) of each column are
// seeded and their cotangents formed from the outputs' cotangents yb
template <int N>
__global__ void __launch_bounds__(64) k_mp_tangent(Grid g, S s, S yb, S b, int pass, float dt, Dual<N>* ws,
                                                   int ncol, const int* done) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  ColPos cp;
  if (col >= ncol || !col_pos(g, col, cp) || done[col] || !cp.run) return;
  const int nin = mp_inputs(g), j0 = pass * N;
  if (j0 >= nin) return;
  const int km = g.nz - 1, c2 = cp.c2;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  using T = Dual<N>;
  const Col<T> C{ws + col, ncol, km + 1};
  prep_column(g, s, C, c2, [&](int idx, float v) {
    T x = dconst<N>(v);
    const int d = idx - j0;
    if (d >= 0 && d < N) x.d[d] = 1.f;
    return x;
  });
  wsm6_column(C, km, dt, true);
  float acc[N];
#pragma unroll
  for (int n = 0; n < N; ++n) acc[n] = 0.f;
  for (int k = 0; k < km; ++k) {
    finish_level(C, k, dt);
    const size_t p = k * lev + c2;
    const T tnew = C(A_TIN, k), h = C(A_TH, k);
    const float yt = yb[WF_T][p], yh = yb[WF_H_DIABATIC][p];
#pragma unroll
    for (int n = 0; n < N; ++n) acc[n] += yt * tnew.d[n] + yh * h.d[n];
    for (int m = 1; m < 7; ++m) {
      const T qo = C(moist_slot(m), k);
      const float y = yb[WF_MOIST][m * n3 + p];
#pragma unroll
      for (int n = 0; n < N; ++n) acc[n] += y * qo.d[n];
    }
  }
#pragma unroll
  for (int n = 0; n < N; ++n)
    if (j0 + n < nin) put_input_cot(g, b, c2, j0 + n, acc[n]);
}

}  // namespace mpt

namespace {

constexpr int kMpDirections = 8;
// entries a column's tape may take per level by default (per time-split
// loop of the whole column; of the column-coupled part in split mode), and
// the memory the tapes of one chunk of columns may take
constexpr int kTapeEntriesPerLevel = 480, kTapeSplitPerLevel = 256;
constexpr size_t kTapeChunkBytes = size_t(24) << 30;
// the capacity set through set_microphysics_tape_capacity (0: default)
int g_tape_capacity = 0;

// the adjoint's workspace, in floats: the outputs' cotangents (9 n3), the
// per-column done flags and tape sizes, then one region shared by the
// chunk's tapes and column arrays and (afterwards) the tangent passes'
// column arrays
struct MpAdjWork {
  size_t done, used, region, tangent, rec, cols, total;
  int ncol, width, cap;
};

MpAdjWork mp_adj_work(const Grid& g) {
  MpAdjWork w;
  const int km = g.nz - 1;
  w.ncol = (g.ide - 1 - (g.ids + 1)) * (g.jde - 1 - (g.jds + 1));
  // the tape holds the column-coupled part in split mode (one time-split
  // loop), the whole column once per loop otherwise
  const int nloop = (int)fmaxf(g.dt / F(mp::DTCLDCR), 1.0f);
  const int per_level = nloop == 1 ? kTapeSplitPerLevel : kTapeEntriesPerLevel * nloop;
  w.cap = g_tape_capacity > 0 ? std::min(kTapeMaxEntries, g_tape_capacity)
                              : std::min(kTapeMaxEntries, per_level * km + mpt::mp_inputs(g));
  const size_t per_col = (size_t)w.cap * 16 + (size_t)mpt::A_COUNT * (km + 1) * sizeof(Tv);
  const size_t fit = std::max<size_t>(64, kTapeChunkBytes / per_col / 64 * 64);
  w.width = (int)std::min<size_t>(fit, ((size_t)w.ncol + 63) / 64 * 64);
  w.done = 9 * g.n3();
  w.used = w.done + w.ncol;
  w.region = (w.used + w.ncol + 3) / 4 * 4;
  w.tangent = (size_t)mpt::A_COUNT * g.nz * w.ncol * (kMpDirections + 1);
  const size_t ent = (size_t)w.cap * w.width;
  w.rec = w.region;
  w.cols = w.rec + 4 * ent;
  const size_t tape = 4 * ent + sizeof(Tv) / sizeof(float) * (size_t)mpt::A_COUNT * (km + 1) * w.width;
  w.total = w.region + std::max(w.tangent, tape);
  return w;
}

}  // namespace

size_t microphysics_adj_work_floats(const Grid& g) { return mp_adj_work(g).total; }

int set_microphysics_tape_capacity(int entries) {
  const int prev = g_tape_capacity;
  g_tape_capacity = entries;
  return prev;
}

int launch_physics_adj(const Grid& g, const S& s, const S& post, const S& b, float* work, float dt, cudaStream_t st,
                       const S* values) {
  const size_t n3 = g.n3();
  const MpAdjWork w = mp_adj_work(g);
  int n = launch_eos_adj(g, post, b, st);
  // the outputs' cotangents, kept while the kernels write the inputs'
  S yb{};
  yb.f[WF_T] = work;
  yb.f[WF_MOIST] = work + n3;
  yb.f[WF_H_DIABATIC] = work + 8 * n3;
  cudaMemcpyAsync(yb.f[WF_T], b[WF_T], n3 * sizeof(float), cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(yb.f[WF_MOIST], b[WF_MOIST], 7 * n3 * sizeof(float), cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(yb.f[WF_H_DIABATIC], b[WF_H_DIABATIC], n3 * sizeof(float), cudaMemcpyDeviceToDevice, st);
  int* done = reinterpret_cast<int*>(work + w.done);
  int* used = reinterpret_cast<int*>(work + w.used);
  S vo{};
  if (values) vo = *values;
  TapeCtx tc;
  tc.rec = reinterpret_cast<TapeRec*>(work + w.rec);
  tc.stride = w.width;
  tc.cap = w.cap;
  auto* cols = reinterpret_cast<Tv*>(work + w.cols);
  // one time-split loop: the point processes are reversed per level
  const bool split = (int)fmaxf(dt / F(mp::DTCLDCR), 1.0f) == 1;
  const int km = g.nz - 1;
  for (int c0 = 0; c0 < w.ncol; c0 += w.width) {
    const int nc = std::min(w.width, w.ncol - c0);
    mpt::k_mp_tape<<<(nc + kTapeBlock - 1) / kTapeBlock, kTapeBlock, 0, st>>>(g, s, yb, b, dt, cols, tc, c0, nc, vo,
                                                                               done, used, split);
    if (split) {
      const long long nt = (long long)nc * km;
      mpt::k_mp_points_adj<4><<<(unsigned)((nt + 127) / 128), 128, 0, st>>>(g, yb, cols, tc, c0, nc, vo, done, used, dt);
      ++n;
    }
    mpt::k_mp_tape_rev<<<(nc + mpt::kSweepBlock - 1) / mpt::kSweepBlock, mpt::kSweepBlock, 0, st>>>(g, b, tc, c0, nc,
                                                                                                    used);
    n += 2;
  }
  // the columns whose tape outgrew the capacity, by tangent passes
  auto* ws = reinterpret_cast<Dual<kMpDirections>*>(work + w.region);
  const int passes = (mpt::mp_inputs(g) + kMpDirections - 1) / kMpDirections;
  for (int pass = 0; pass < passes; ++pass) {
    mpt::k_mp_tangent<kMpDirections><<<(w.ncol + 63) / 64, 64, 0, st>>>(g, s, yb, b, pass, dt, ws, w.ncol, done);
    ++n;
  }
  return n;
}

}  // namespace wrf
