// Adjoints of the large-step tendency terms (wrf_dynamics.py:2031-2620):
// rhs_ph, horizontal_pressure_gradient, pg_buoy_w, coriolis and curvature,
// each selected by a bit of `terms` (1, 2, 4, 8, 16).
//
// Each term adds a local stencil expression to a tendency at its own point.
// The reverse product runs one thread per output point: it forms the
// expression's partial derivatives from the saved inputs (the forward values
// are recomputed, nothing is taped) and adds cotangent x partial into the
// cotangents of the inputs it read, with atomicAdd (a point's cotangent
// gathers contributions from up to a few dozen output points).  The
// incoming tendencies' cotangents are the outgoing ones (tend += f), except
// where a term overwrites its output: rhs_ph sets ph_tend to zero on the top
// level before adding (that cotangent is zeroed), and pg_buoy_w replaces cqw
// by 1/(1+cqw) on levels 1 .. nz-2 of the mass points (that cotangent is
// rewritten to the input's).  Map factors, Coriolis parameters, vertical
// profiles and the grid constants are data.
#include "kernels.cuh"

namespace wrf {

namespace {

__device__ __forceinline__ void acc(float* a, size_t q, float v) {
  if (v != 0.f) atomicAdd(a + q, v);
}

// rhs_ph at the mass point (k >= 1, j, i) with output cotangent T
__device__ void rhs_ph_adj(const Grid& g, const S& s, const S& b, int k, int j, int i, size_t p, float T) {
  const int nz = g.nz, nx = g.nx, ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const size_t lev = (size_t)g.ny * nx;
  const int c = g.i2(j, i);
  const float* ph = s[WF_PH];
  const float* phb = s[WF_PHB];
  const float* ww = s[WF_WW];
  const float* rdnw = s[WF_RDNW];
  const float msfty = s[WF_MSFTY][c];
  const bool top = k == nz - 1;
  if (!top) {
    // t -= fnm(k) wdwn(k+1) + fnp(k) wdwn(k), wdwn(kk) = 0.5 (ww(kk) + ww(kk-1)) rdnw(kk-1) D(kk)
    const float wk[2] = {-s[WF_FNM][k] * T, -s[WF_FNP][k] * T};
    for (int e = 0; e < 2; ++e) {
      const int kk = k + 1 - e;
      const size_t q = kk * lev + c, qm = q - lev;
      const float W = wk[e];
      const float A = 0.5f * (ww[q] + ww[qm]), R = rdnw[kk - 1];
      const float D = ph[q] - ph[qm] + phb[q] - phb[qm];
      acc(b[WF_WW], q, 0.5f * R * D * W);
      acc(b[WF_WW], qm, 0.5f * R * D * W);
      const float h = A * R * W;
      acc(b[WF_PH], q, h);
      acc(b[WF_PH], qm, -h);
      acc(b[WF_PHB], q, h);
      acc(b[WF_PHB], qm, -h);
    }
  }
  // + mut g w / msfty
  const float gf = (float)G;
  acc(b[WF_MUT], c, gf * s[WF_W][p] / msfty * T);
  acc(b[WF_W], p, s[WF_MUT][c] * gf / msfty * T);
  const float cfn = g.cfn, cfn1 = g.cfn1;
  // flux of a face column cc: mu (v(k) + v(k-1)) msf, or its top form
  auto flux_adj = [&](int fmu, int fvel, int fmsf, size_t cc, float F) {
    const float* vel = s[fvel];
    const float mu = s[fmu][cc], msf = s[fmsf][cc];
    if (!top) {
      const size_t q = k * lev + cc, qm = q - lev;
      acc(b[fmu], cc, (vel[q] + vel[qm]) * msf * F);
      acc(b[fvel], q, mu * msf * F);
      acc(b[fvel], qm, mu * msf * F);
    } else {
      const size_t q2 = (size_t)(nz - 2) * lev + cc, q3 = (size_t)(nz - 3) * lev + cc;
      acc(b[fmu], cc, (cfn * vel[q2] + cfn1 * vel[q3]) * msf * F);
      acc(b[fvel], q2, mu * cfn * msf * F);
      acc(b[fvel], q3, mu * cfn1 * msf * F);
    }
  };
  auto flux = [&](int fmu, int fvel, int fmsf, size_t cc) {
    const float* vel = s[fvel];
    if (!top) return s[fmu][cc] * (vel[k * lev + cc] + vel[(k - 1) * lev + cc]) * s[fmsf][cc];
    return s[fmu][cc] * (cfn * vel[(nz - 2) * lev + cc] + cfn1 * vel[(nz - 3) * lev + cc]) * s[fmsf][cc];
  };
  // 6th / 4th / 2nd order differences of ph + phb along a direction of stride st
  auto diff_adj = [&](int order, int st, float Dc) {
    const int n = order == 6 ? 3 : 2;
    for (int m = 1; m <= n; ++m) {
      const float cm = order == 6 ? (m == 1 ? 45.f : (m == 2 ? -9.f : 1.f)) : (m == 1 ? 8.f : -1.f);
      const float w = cm * Dc;
      acc(b[WF_PH], p + (size_t)m * st, w);
      acc(b[WF_PH], p - (size_t)m * st, -w);
      acc(b[WF_PHB], p + (size_t)m * st, w);
      acc(b[WF_PHB], p - (size_t)m * st, -w);
    }
  };
  auto diff = [&](int order, int st) {
    auto d = [&](int m) { return ph[p + (size_t)m * st] - ph[p - (size_t)m * st]; };
    auto db = [&](int m) { return phb[p + (size_t)m * st] - phb[p - (size_t)m * st]; };
    if (order == 6) return 45.f * d(1) - 9.f * d(2) + d(3) + 45.f * db(1) - 9.f * db(2) + db(3);
    return 8.f * d(1) - d(2) + 8.f * db(1) - db(2);
  };
  // y direction
  {
    const float K = (top ? (float)(0.5 * g.rdyd) : (float)(0.25 * g.rdyd)) / msfty;
    const size_t cn = (size_t)(j + 1) * nx + i, c0 = (size_t)j * nx + i;
    int order = 0;
    if (j >= jds + 3 && j < jde - 4) order = 6;
    else if (j == jds + 2 || j == jde - 4) order = 4;
    else if (j == jds + 1 || j == jde - 3) order = 2;
    if (order >= 4) {
      const float E = order == 6 ? (float)(1.0 / 60.0) : (float)(1.0 / 12.0);
      const float F = flux(WF_MUV, WF_V, WF_MSFVY, cn) + flux(WF_MUV, WF_V, WF_MSFVY, c0);
      const float dd = diff(order, nx);
      flux_adj(WF_MUV, WF_V, WF_MSFVY, cn, -K * E * dd * T);
      flux_adj(WF_MUV, WF_V, WF_MSFVY, c0, -K * E * dd * T);
      diff_adj(order, nx, -K * F * E * T);
    } else if (order == 2) {
      auto dp = [&](int d) { const size_t q = p + (size_t)d * nx; return phb[q] - phb[q - nx] + ph[q] - ph[q - nx]; };
      const float f1 = flux(WF_MUV, WF_V, WF_MSFVY, cn), f0 = flux(WF_MUV, WF_V, WF_MSFVY, c0);
      flux_adj(WF_MUV, WF_V, WF_MSFVY, cn, -K * dp(1) * T);
      flux_adj(WF_MUV, WF_V, WF_MSFVY, c0, -K * dp(0) * T);
      const float w1 = -K * f1 * T, w0 = -K * f0 * T;
      acc(b[WF_PH], p + nx, w1);
      acc(b[WF_PHB], p + nx, w1);
      acc(b[WF_PH], p, w0 - w1);
      acc(b[WF_PHB], p, w0 - w1);
      acc(b[WF_PH], p - nx, -w0);
      acc(b[WF_PHB], p - nx, -w0);
    }
  }
  // x direction (6th order interior, 2nd order at ids+1 and ide-3)
  {
    const float K = (top ? (float)(0.5 * g.rdxd) : (float)(0.25 * g.rdxd)) / msfty;
    const size_t ce = (size_t)j * nx + i + 1, c0 = (size_t)j * nx + i;
    if (i >= ids + 3 && i < ide - 4) {
      const float E = (float)(1.0 / 60.0);
      const float F = flux(WF_MUU, WF_U, WF_MSFUX, ce) + flux(WF_MUU, WF_U, WF_MSFUX, c0);
      const float dd = diff(6, 1);
      flux_adj(WF_MUU, WF_U, WF_MSFUX, ce, -K * E * dd * T);
      flux_adj(WF_MUU, WF_U, WF_MSFUX, c0, -K * E * dd * T);
      diff_adj(6, 1, -K * F * E * T);
    } else if (i == ids + 1 || i == ide - 3) {
      auto dp = [&](int d) { const size_t q = p + d; return phb[q] - phb[q - 1] + ph[q] - ph[q - 1]; };
      const float f1 = flux(WF_MUU, WF_U, WF_MSFUX, ce), f0 = flux(WF_MUU, WF_U, WF_MSFUX, c0);
      flux_adj(WF_MUU, WF_U, WF_MSFUX, ce, -K * dp(1) * T);
      flux_adj(WF_MUU, WF_U, WF_MSFUX, c0, -K * dp(0) * T);
      const float w1 = -K * f1 * T, w0 = -K * f0 * T;
      acc(b[WF_PH], p + 1, w1);
      acc(b[WF_PHB], p + 1, w1);
      acc(b[WF_PH], p, w0 - w1);
      acc(b[WF_PHB], p, w0 - w1);
      acc(b[WF_PH], p - 1, -w0);
      acc(b[WF_PHB], p - 1, -w0);
    }
  }
}

// horizontal_pressure_gradient at a u point (dir 0: neighbour c-1) or a v
// point (dir 1: neighbour c-nx), output cotangent X0 of ru_tend / rv_tend
__device__ void hpg_adj(const Grid& g, const S& s, const S& b, int dir, int k, int c, size_t p, float X0) {
  const int nz = g.nz;
  const size_t lev = (size_t)g.ny * g.nx;
  const int off = dir == 0 ? 1 : g.nx;
  const int cm = c - off;
  const size_t q = p, qm = p - off;
  const float* ph = s[WF_PH];
  const float* pp = s[WF_P];
  const float* pb = s[WF_PB];
  const float* al = s[WF_AL];
  const float* alt = s[WF_ALT];
  const float* php = s[WF_PHP];
  const float* mu = s[WF_MU];
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  const float rd = dir == 0 ? g.rdx : g.rdy;
  const float r = dir == 0 ? s[WF_MSFUX][c] / s[WF_MSFUY][c] : s[WF_MSFVY][c] / s[WF_MSFVX][c];
  const int fmu = dir == 0 ? WF_MUU : WF_MUV, fcq = dir == 0 ? WF_CQU : WF_CQV;
  const float muf = s[fmu][c];
  auto dpn = [&](int kk) {  // p at w level kk between the two columns
    if (kk == 0)
      return 0.5f * (g.cf1 * (pp[cm] + pp[c]) + g.cf2 * (pp[lev + cm] + pp[lev + c]) + g.cf3 * (pp[2 * lev + cm] + pp[2 * lev + c]));
    if (kk == nz - 1) return 0.f;
    return 0.5f * (fnm[kk] * (pp[kk * lev + cm] + pp[kk * lev + c]) + fnp[kk] * (pp[(kk - 1) * lev + cm] + pp[(kk - 1) * lev + c]));
  };
  auto dpn_adj = [&](int kk, float D) {
    if (kk == nz - 1) return;
    if (kk == 0) {
      const float w1 = 0.5f * g.cf1 * D, w2 = 0.5f * g.cf2 * D, w3 = 0.5f * g.cf3 * D;
      acc(b[WF_P], cm, w1);
      acc(b[WF_P], c, w1);
      acc(b[WF_P], lev + cm, w2);
      acc(b[WF_P], lev + c, w2);
      acc(b[WF_P], 2 * lev + cm, w3);
      acc(b[WF_P], 2 * lev + c, w3);
      return;
    }
    const float wm = 0.5f * fnm[kk] * D, wp = 0.5f * fnp[kk] * D;
    acc(b[WF_P], kk * lev + cm, wm);
    acc(b[WF_P], kk * lev + c, wm);
    acc(b[WF_P], (kk - 1) * lev + cm, wp);
    acc(b[WF_P], (kk - 1) * lev + c, wp);
  };
  const float Q = (ph[q + lev] - ph[qm + lev] + ph[q] - ph[qm]) + (alt[q] + alt[qm]) * (pp[q] - pp[qm]) +
                  (al[q] + al[qm]) * (pb[q] - pb[qm]);
  const float P = r * 0.5f * rd * muf;
  const float M = s[WF_RDNW][k] * (dpn(k + 1) - dpn(k)) - 0.5f * (mu[cm] + mu[c]);
  const float R2 = r * rd;
  const float dphp = php[q] - php[qm];
  const float dpx = P * Q + R2 * dphp * M;
  // out -= cq dpx
  acc(b[fcq], p, -dpx * X0);
  const float X = -s[fcq][p] * X0;
  acc(b[fmu], c, r * 0.5f * rd * Q * X);
  const float PX = P * X;
  acc(b[WF_PH], q + lev, PX);
  acc(b[WF_PH], qm + lev, -PX);
  acc(b[WF_PH], q, PX);
  acc(b[WF_PH], qm, -PX);
  const float wa = PX * (pp[q] - pp[qm]);
  acc(b[WF_ALT], q, wa);
  acc(b[WF_ALT], qm, wa);
  const float wpp = PX * (alt[q] + alt[qm]);
  acc(b[WF_P], q, wpp);
  acc(b[WF_P], qm, -wpp);
  const float wl = PX * (pb[q] - pb[qm]);
  acc(b[WF_AL], q, wl);
  acc(b[WF_AL], qm, wl);
  const float wb = PX * (al[q] + al[qm]);
  acc(b[WF_PB], q, wb);
  acc(b[WF_PB], qm, -wb);
  const float wphp = R2 * M * X;
  acc(b[WF_PHP], q, wphp);
  acc(b[WF_PHP], qm, -wphp);
  const float Y = R2 * dphp * X;
  acc(b[WF_MU], cm, -0.5f * Y);
  acc(b[WF_MU], c, -0.5f * Y);
  dpn_adj(k + 1, s[WF_RDNW][k] * Y);
  dpn_adj(k, -s[WF_RDNW][k] * Y);
}

// pg_buoy_w at the mass point (k in 1 .. nz-2): rw_tend(k) (and rw_tend(nz-1)
// from level nz-2) and the overwritten cqw(k) = 1 / (1 + cqw(k))
__device__ void pg_buoy_w_adj(const Grid& g, const S& s, const S& b, int k, int c, size_t p) {
  const int nz = g.nz;
  const size_t lev = (size_t)g.ny * g.nx;
  const float* pp = s[WF_P];
  const float x = s[WF_CQW][p];
  const float cq1 = 1.0f / (1.0f + x);
  const float cq2 = x * cq1;
  const float gm = (float)G / s[WF_MSFTY][c];
  const float mub = s[WF_MUB][c];
  float cq1b = b[WF_CQW][p];  // cotangent of the output cqw = cq1
  float cq2b = 0.f;
  float mub_b = 0.f, mu_b = 0.f;
  if (k == nz - 2) {
    const float Z = gm * b[WF_RW_TEND][p + lev];
    const float r2 = 2.0f * s[WF_RDNW][nz - 2];
    acc(b[WF_P], p, -cq1 * r2 * Z);
    mu_b -= Z;
    mub_b -= cq2 * Z;
    cq1b += r2 * (-pp[p]) * Z;
    cq2b -= mub * Z;
  }
  const float Z = gm * b[WF_RW_TEND][p];
  const float rk = s[WF_RDN][k];
  acc(b[WF_P], p, cq1 * rk * Z);
  acc(b[WF_P], p - lev, -cq1 * rk * Z);
  mu_b -= Z;
  mub_b -= cq2 * Z;
  cq1b += rk * (pp[p] - pp[p - lev]) * Z;
  cq2b -= mub * Z;
  acc(b[WF_MU], c, mu_b);
  acc(b[WF_MUB], c, mub_b);
  // d cq1 / dx = -cq1^2, d cq2 / dx = cq1^2
  b[WF_CQW][p] = (cq2b - cq1b) * (cq1 * cq1);
}

// coriolis (cor) and curvature (cur) at a u point (dir 0), v point (dir 1)
// or w point (dir 2), output cotangent T
__device__ void cor_cur_adj(const Grid& g, const S& s, const S& b, bool cor, bool cur, int dir, int k, int c,
                            size_t p, float T) {
  const int nx = g.nx;
  const size_t lev = (size_t)g.ny * nx;
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  const float* f = s[WF_F];
  const float* e = s[WF_E];
  const float* sina = s[WF_SINA];
  const float* cosa = s[WF_COSA];
  const float rr = (float)RERADIUS;
  const float rdx = g.rdx, rdy = g.rdy;
  auto vx = [&](int cc, size_t qq) {
    return 0.5f * (u[qq] + u[qq + 1]) * (s[WF_MSFVX][cc + nx] - s[WF_MSFVX][cc]) * rdy -
           0.5f * (v[qq] + v[qq + nx]) * (s[WF_MSFUY][cc + 1] - s[WF_MSFUY][cc]) * rdx;
  };
  auto vx_adj = [&](int cc, size_t qq, float V) {
    const float wu = 0.5f * (s[WF_MSFVX][cc + nx] - s[WF_MSFVX][cc]) * rdy * V;
    const float wv = -0.5f * (s[WF_MSFUY][cc + 1] - s[WF_MSFUY][cc]) * rdx * V;
    acc(b[WF_U], qq, wu);
    acc(b[WF_U], qq + 1, wu);
    acc(b[WF_V], qq, wv);
    acc(b[WF_V], qq + nx, wv);
  };
  if (dir == 0) {
    const size_t r4[4] = {p + nx - 1, p + nx, p - 1, p};
    const size_t w4[4] = {p + lev - 1, p - 1, p + lev, p};
    float rvb = 0.f, rwb = 0.f;
    if (cor) {
      rvb += (s[WF_MSFUX][c] / s[WF_MSFUY][c]) * 0.5f * (f[c] + f[c - 1]) * 0.25f * T;
      rwb -= 0.5f * (e[c] + e[c - 1]) * 0.5f * (cosa[c] + cosa[c - 1]) * 0.25f * T;
    }
    if (cur) {
      const float* rv = s[WF_RV];
      const float* rw = s[WF_RW];
      const float rvs = rv[r4[0]] + rv[r4[1]] + rv[r4[2]] + rv[r4[3]];
      const float rws = rw[w4[0]] + rw[w4[1]] + rw[w4[2]] + rw[w4[3]];
      rvb += 0.5f * (vx(c, p) + vx(c - 1, p - 1)) * 0.25f * T;
      rwb -= u[p] * rr * 0.25f * T;
      acc(b[WF_U], p, -rr * 0.25f * rws * T);
      const float V = 0.5f * 0.25f * rvs * T;
      vx_adj(c, p, V);
      vx_adj(c - 1, p - 1, V);
    }
    for (int m = 0; m < 4; ++m) {
      acc(b[WF_RV], r4[m], rvb);
      acc(b[WF_RW], w4[m], rwb);
    }
  } else if (dir == 1) {
    const float r = s[WF_MSFVY][c] / s[WF_MSFVX][c];
    const size_t u4[4] = {p, p + 1, p - nx, p - nx + 1};
    const size_t w4[4] = {p + lev - nx, p - nx, p + lev, p};
    float rub = 0.f, rwb = 0.f;
    if (cor) {
      rub -= r * 0.5f * (f[c] + f[c - nx]) * 0.25f * T;
      rwb += r * 0.5f * (e[c] + e[c - nx]) * 0.5f * (sina[c] + sina[c - nx]) * 0.25f * T;
    }
    if (cur) {
      const float* ru = s[WF_RU];
      const float* rw = s[WF_RW];
      const float rus = ru[u4[0]] + ru[u4[1]] + ru[u4[2]] + ru[u4[3]];
      const float rws = rw[w4[0]] + rw[w4[1]] + rw[w4[2]] + rw[w4[3]];
      rub -= 0.5f * (vx(c, p) + vx(c - nx, p - nx)) * 0.25f * T;
      rwb -= r * v[p] * rr * 0.25f * T;
      acc(b[WF_V], p, -r * rr * 0.25f * rws * T);
      const float V = -0.5f * 0.25f * rus * T;
      vx_adj(c, p, V);
      vx_adj(c - nx, p - nx, V);
    }
    for (int m = 0; m < 4; ++m) {
      acc(b[WF_RU], u4[m], rub);
      acc(b[WF_RW], w4[m], rwb);
    }
  } else {
    const float fm = s[WF_FNM][k], fp = s[WF_FNP][k];
    const float rmt = s[WF_MSFTX][c] / s[WF_MSFTY][c];
    float Ab = 0.f, Bb = 0.f;
    if (cor) {
      Ab += e[c] * cosa[c] * 0.5f * T;
      Bb -= e[c] * rmt * sina[c] * 0.5f * T;
    }
    if (cur) {
      const float* ru = s[WF_RU];
      const float* rv = s[WF_RV];
      const float A = fm * (ru[p] + ru[p + 1]) + fp * (ru[p - lev] + ru[p - lev + 1]);
      const float B = fm * (rv[p] + rv[p + nx]) + fp * (rv[p - lev] + rv[p - lev + nx]);
      const float Cu = fm * (u[p] + u[p + 1]) + fp * (u[p - lev] + u[p - lev + 1]);
      const float Cv = fm * (v[p] + v[p + nx]) + fp * (v[p - lev] + v[p - lev + nx]);
      Ab += rr * 0.25f * Cu * T;
      Bb += rr * rmt * 0.25f * Cv * T;
      const float Cub = rr * 0.25f * A * T, Cvb = rr * rmt * 0.25f * B * T;
      acc(b[WF_U], p, fm * Cub);
      acc(b[WF_U], p + 1, fm * Cub);
      acc(b[WF_U], p - lev, fp * Cub);
      acc(b[WF_U], p - lev + 1, fp * Cub);
      acc(b[WF_V], p, fm * Cvb);
      acc(b[WF_V], p + nx, fm * Cvb);
      acc(b[WF_V], p - lev, fp * Cvb);
      acc(b[WF_V], p - lev + nx, fp * Cvb);
    }
    acc(b[WF_RU], p, fm * Ab);
    acc(b[WF_RU], p + 1, fm * Ab);
    acc(b[WF_RU], p - lev, fp * Ab);
    acc(b[WF_RU], p - lev + 1, fp * Ab);
    acc(b[WF_RV], p, fm * Bb);
    acc(b[WF_RV], p + nx, fm * Bb);
    acc(b[WF_RV], p - lev, fp * Bb);
    acc(b[WF_RV], p - lev + nx, fp * Bb);
  }
}

}  // namespace

__global__ void k_forces_adj(Grid g, S s, S b, int terms) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, nz = g.nz, ktf = nz - 1;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const bool mass = j >= jds && j < jde - 1 && i >= ids && i < ide - 1;
  const bool upt = k < ktf && j >= jds && j < jde - 1 && i >= ids + 1 && i < ide - 1;
  const bool vpt = k < ktf && j >= jds + 1 && j < jde - 1 && i >= ids && i < ide - 1;
  const bool cor = terms & 8, cur = terms & 16;
  if ((terms & 1) && mass && k >= 1) {
    const float T = b[WF_PH_TEND][p];
    rhs_ph_adj(g, s, b, k, j, i, p, T);
    if (k == nz - 1) b[WF_PH_TEND][p] = 0.f;  // the top level is set, not incremented
  }
  if ((terms & 2) && upt) hpg_adj(g, s, b, 0, k, c, p, b[WF_RU_TEND][p]);
  if ((terms & 2) && vpt) hpg_adj(g, s, b, 1, k, c, p, b[WF_RV_TEND][p]);
  if ((terms & 4) && mass && k >= 1 && k < nz - 1) pg_buoy_w_adj(g, s, b, k, c, p);
  if ((cor || cur) && upt) cor_cur_adj(g, s, b, cor, cur, 0, k, c, p, b[WF_RU_TEND][p]);
  if ((cor || cur) && vpt) cor_cur_adj(g, s, b, cor, cur, 1, k, c, p, b[WF_RV_TEND][p]);
  if ((cor || cur) && mass && k >= 1 && k < ktf) cor_cur_adj(g, s, b, cor, cur, 2, k, c, p, b[WF_RW_TEND][p]);
}

int launch_forces_adj(const Grid& g, const S& s, const S& b, int terms, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_forces_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, terms);
  return 1;
}

}  // namespace wrf
