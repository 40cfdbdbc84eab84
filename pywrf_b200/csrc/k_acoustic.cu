// Acoustic (small) time step (wrf_dynamics.py:3152-3930, wrf_boundary.py:244-400).
//   k_ssp2d / k_ssp3d   small_step_prep (2-D masses, then 3-D perturbation form)
//   k_p_rho             calc_p_rho (+ zero_grad_bdy(w) after a substep)
//   k_coef_w            calc_coef_w: tridiagonal coefficients + forward sweep
//   k_advance_uv        advance_uv + spec_bdyupdate(u), (v)
//   k_advance_mu_t      advance_mu_t (column) + spec_bdyupdate(t), (mu), (muts)
//   k_advance_w         advance_w (column Thomas solve + damping) + sumflux
//                       + spec_bdyupdate_ph
//   k_mu_uv_1 / k_ssfinish  calc_mu_uv_1, small_step_finish
// Column kernels give one thread a (j, i) column; the vertical recurrences
// (mass divergence sum, ww scan, Thomas sweeps) run in the reference's order.
#include "kernels.cuh"

namespace wrf {

__global__ void k_ssp2d(Grid g, S s, int rk_step) {
  WRF_COLUMN_INDEX(g, j, i);
  const int c = g.i2(j, i);
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  float* mu = s[WF_MU];
  float* mu1 = s[WF_MU_1];
  const float* mub = s[WF_MUB];
  const bool t2 = j >= jts && j < jme && i >= its && i < ime;
  if (rk_step == 1) {
    if (t2) {
      const float m2 = mu[c];
      mu1[c] = m2;
      s[WF_MUDF][c] = 0.f;
      s[WF_MUTS][c] = mub[c] + m2;
      s[WF_MU_SAVE][c] = m2;
      mu[c] = 0.f;
    }
    if (j >= jts && j < jme && i >= its && i < ieu) s[WF_MUUS][c] = s[WF_MUU][c];
    if (j >= jts && j < jev && i >= its && i < ime) s[WF_MUVS][c] = s[WF_MUV][c];
  } else {
    if (t2) {
      s[WF_MUTS][c] = mub[c] + mu1[c];
      const float m2 = mu[c];
      s[WF_MU_SAVE][c] = m2;
      mu[c] = mu1[c] - m2;
    }
    if (j >= jts && j < jme && i >= its && i < ieu)
      s[WF_MUUS][c] = 0.5f * (mub[c] + mu1[c] + mub[c - 1] + mu1[c - 1]);
    if (j >= jts && j < jev && i >= its && i < ieu)
      s[WF_MUVS][c] = 0.5f * (mub[c] + mu1[c] + mub[c - g.nx] + mu1[c - g.nx]);
  }
}

__global__ void k_ssp3d(Grid g, S s, int rk_step) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nz = g.nz, ktf = nz - 1;
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const bool t2 = j >= jts && j < jme && i >= its && i < ime;
  if (k < ktf && j >= jts && j < jme && i >= its && i < ieu) {
    const float u2 = s[WF_U][p];
    if (rk_step == 1) s[WF_U_1][p] = u2;
    s[WF_U_SAVE][p] = u2;
    s[WF_U][p] = (s[WF_MUUS][c] * s[WF_U_1][p] - s[WF_MUU][c] * u2) / s[WF_MSFUY][c];
  }
  if (k < ktf && j >= jts && j < jev && i >= its && i < ime) {
    const float v2 = s[WF_V][p];
    if (rk_step == 1) s[WF_V_1][p] = v2;
    s[WF_V_SAVE][p] = v2;
    s[WF_V][p] = (s[WF_MUVS][c] * s[WF_V_1][p] - s[WF_MUV][c] * v2) * s[WF_MSFVX_INV][c];
  }
  if (t2) {
    const float muts = s[WF_MUTS][c], mut = s[WF_MUT][c];
    if (k < ktf) {
      s[WF_C2A][p] = (float)CPOVCV * (s[WF_PB][p] + s[WF_P][p]) / s[WF_ALT][p];
      const float t2v = s[WF_T][p];
      if (rk_step == 1) s[WF_T_1][p] = t2v;
      s[WF_T_SAVE][p] = t2v;
      s[WF_T][p] = muts * s[WF_T_1][p] - mut * t2v;
    }
    const float w2 = s[WF_W][p];
    if (rk_step == 1) s[WF_W_1][p] = w2;
    s[WF_W_SAVE][p] = w2;
    s[WF_W][p] = (muts * s[WF_W_1][p] - mut * w2) / s[WF_MSFTY][c];
    const float ph2 = s[WF_PH][p];
    if (rk_step == 1) s[WF_PH_1][p] = ph2;
    s[WF_PH_SAVE][p] = ph2;
    s[WF_PH][p] = s[WF_PH_1][p] - ph2;
    s[WF_WW1][p] = s[WF_WW][p];
  }
}

// calc_p_rho (wrf_dynamics.py:3269-3313).  step 0 replaces pm1 by a copy of
// the whole new p; later substeps apply the divergence damping and
// zero_grad_bdy(w) on the specified rows (wrf_boundary.py:358-400).
__global__ void k_p_rho(Grid g, S s, int step) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nz = g.nz, ktf = nz - 1, nx = g.nx;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * nx;
  const size_t p = k * lev + c;
  const bool r = k < ktf && j >= g.jds && j < g.jde - 1 && i >= g.ids && i < g.ide - 1;
  float* pp = s[WF_P];
  float pnew = pp[p];
  if (r) {
    const float muts = s[WF_MUTS][c], mu = s[WF_MU][c];
    const float alt = s[WF_ALT][p], t1 = s[WF_T_SAVE][p];
    const float* ph = s[WF_PH];
    const float al = -1.0f / muts * (alt * mu + s[WF_RDNW][k] * (ph[p + lev] - ph[p]));
    s[WF_AL][p] = al;
    pnew = s[WF_C2A][p] * (alt * (s[WF_T][p] - mu * t1) / (muts * ((float)T0 + t1)) - al);
    if (step == 0) {
      pp[p] = pnew;
    } else {
      const float ptmp = pnew;
      pnew = pnew + g.smdiv * (pnew - s[WF_PM1][p]);
      pp[p] = pnew;
      s[WF_PM1][p] = ptmp;
    }
  }
  if (step == 0) {
    s[WF_PM1][p] = pnew;
    return;
  }
  // zero-gradient w on the specified rows (all levels)
  const int ibs = g.ids, ibe = g.ide - 1, jbs = g.jds, jbe = g.jde - 1;
  float* w = s[WF_W];
  const size_t base = k * lev;
  int sj = -1, si = -1;
  if (j == jbs || j == jbe - 1) {
    if (i >= ibs && i < ibe) {
      const int jn = (j == jbs) ? jbs + 1 : jbe - 2;
      si = (i == ibs) ? ibs + 1 : (i == ibe - 1 ? ibe - 2 : i);
      sj = jn;
    }
  } else if (j > jbs && j < jbe - 1 && (i == ibs || i == ibe - 1)) {
    sj = j;
    si = (i == ibs) ? ibs + 1 : ibe - 2;
  }
  if (sj >= 0) w[base + (size_t)j * nx + i] = w[base + (size_t)sj * nx + si];
}

__global__ void k_coef_w(Grid g, S s, float dts) {
  WRF_COLUMN_INDEX(g, j, i);
  if (j < g.jds || j >= g.jde - 1 || i < g.ids || i >= g.ide - 1) return;
  const int nz = g.nz;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * g.nx;
  const double cofd = (0.5 * (double)dts * G * (1.0 + (double)g.epssm)) * (0.5 * (double)dts * G * (1.0 + (double)g.epssm));
  const float cof = (float)cofd, cofm2 = (float)(-2.0 * cofd), cof2 = (float)(2.0 * cofd);
  const float mut = s[WF_MUT][c];
  const float mm = mut * mut;
  const float* cqw = s[WF_CQW];
  const float* c2a = s[WF_C2A];
  const float* rdn = s[WF_RDN];
  const float* rdnw = s[WF_RDNW];
  float* a = s[WF_A];
  float* alpha = s[WF_ALPHA];
  float* gamma = s[WF_GAMMA];
  const float lid = g.top_lid ? 0.f : 1.f;
  a[lev + c] = 0.f;
  const float atop = cofm2 * (rdnw[nz - 2] * rdnw[nz - 2]) * c2a[(nz - 2) * lev + c] * lid / mm;
  a[(nz - 1) * lev + c] = atop;
  gamma[c] = 0.f;
  float gm = 0.f;
  for (int k = 1; k < nz - 1; ++k) {
    const size_t p = k * lev + c;
    const float cw = cqw[p];
    float ak = 0.f;
    if (k >= 2) {
      ak = -cw * cof * rdn[k] * rdnw[k - 1] * c2a[p - lev] / mm;
      a[p] = ak;
    }
    const float b = 1.0f + cw * cof * rdn[k] * (rdnw[k] * c2a[p] / mm + rdnw[k - 1] * c2a[p - lev] / mm);
    const float cc = -cw * cof * rdn[k] * rdnw[k] * c2a[p] / mm;
    const float al = 1.0f / (b - ak * gm);
    alpha[p] = al;
    gm = cc * al;
    gamma[p] = gm;
  }
  const float btop = 1.0f + cof2 * (rdnw[nz - 2] * rdnw[nz - 2]) * c2a[(nz - 2) * lev + c] / mm;
  alpha[(nz - 1) * lev + c] = 1.0f / (btop - atop * gm);
  gamma[(nz - 1) * lev + c] = 0.f;
}

__global__ void k_advance_uv(Grid g, S s, float dts) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nz = g.nz, ktf = nz - 1, nx = g.nx;
  if (k >= ktf) return;
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * nx;
  const size_t p = k * lev + c;
  const float* pp = s[WF_P];
  const float* pb = s[WF_PB];
  const float* ph = s[WF_PH];
  const float* php = s[WF_PHP];
  const float* alt = s[WF_ALT];
  const float* al = s[WF_AL];
  const float* mu = s[WF_MU];
  const float* mudf = s[WF_MUDF];
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  const float* rdnw = s[WF_RDNW];
  const float rdx = g.rdx, rdy = g.rdy;
  auto dpn = [&](int kk, size_t ca, size_t cb) {
    if (kk == 0)
      return 0.5f * (g.cf1 * (pp[ca] + pp[cb]) + g.cf2 * (pp[lev + ca] + pp[lev + cb]) + g.cf3 * (pp[2 * lev + ca] + pp[2 * lev + cb]));
    if (kk == nz - 1) return 0.f;
    return 0.5f * (fnm[kk] * (pp[kk * lev + ca] + pp[kk * lev + cb]) + fnp[kk] * (pp[(kk - 1) * lev + ca] + pp[(kk - 1) * lev + cb]));
  };
  // u
  if (j >= jds + 1 && j < jde - 2 && i >= ids + 1 && i < ide - 1) {
    float u = s[WF_U][p] + dts * s[WF_RU_TEND][p];
    const float mudf_xy = (float)(-(double)g.emdiv * g.dxd) * (mudf[c] - mudf[c - 1]) / s[WF_MSFUY][c];
    const float r = s[WF_MSFUX][c] / s[WF_MSFUY][c];
    const size_t q = p, qm = p - 1;
    float dp = r * 0.5f * rdx * s[WF_MUU][c] *
               (((ph[q + lev] - ph[qm + lev]) + (ph[q] - ph[qm])) + (alt[q] + alt[qm]) * (pp[q] - pp[qm]) + (al[q] + al[qm]) * (pb[q] - pb[qm]));
    dp = dp + r * rdx * (php[q] - php[qm]) * (rdnw[k] * (dpn(k + 1, c, c - 1) - dpn(k, c, c - 1)) - 0.5f * (mu[c - 1] + mu[c]));
    s[WF_U][p] = u - dts * s[WF_CQU][p] * dp + mudf_xy;
  } else if (((j == jds || j == jde - 2) && i >= ids && i < ide) || (j >= jds + 1 && j < jde - 2 && (i == ids || i == ide - 1))) {
    s[WF_U][p] = s[WF_U][p] + dts * s[WF_RU_TEND][p];   // spec_bdyupdate(u)
  }
  // v
  if (j >= jds + 1 && j < jde - 1 && i >= ids + 1 && i < ide - 2) {
    float v = s[WF_V][p] + dts * s[WF_RV_TEND][p];
    const float mudf_xy = (float)(-(double)g.emdiv * g.dyd) * (mudf[c] - mudf[c - nx]) * s[WF_MSFVX_INV][c];
    const float r = s[WF_MSFVY][c] / s[WF_MSFVX][c];
    const size_t q = p, qm = p - nx;
    float dp = r * 0.5f * rdy * s[WF_MUV][c] *
               (((ph[q + lev] - ph[qm + lev]) + (ph[q] - ph[qm])) + (alt[q] + alt[qm]) * (pp[q] - pp[qm]) + (al[q] + al[qm]) * (pb[q] - pb[qm]));
    dp = dp + r * rdy * (php[q] - php[qm]) * (rdnw[k] * (dpn(k + 1, c, c - nx) - dpn(k, c, c - nx)) - 0.5f * (mu[c - nx] + mu[c]));
    s[WF_V][p] = v - dts * s[WF_CQV][p] * dp + mudf_xy;
  } else if (((j == jds || j == jde - 1) && i >= ids && i < ide - 1) || (j >= jds + 1 && j < jde - 1 && (i == ids || i == ide - 2))) {
    s[WF_V][p] = s[WF_V][p] + dts * s[WF_RV_TEND][p];   // spec_bdyupdate(v)
  }
}

__global__ void k_advance_mu_t(Grid g, S s, float dts) {
  WRF_COLUMN_INDEX(g, j, i);
  const int nz = g.nz, kend = nz - 1, nx = g.nx;
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * nx;
  float* t = s[WF_T];
  const float* ft = s[WF_T_TEND];
  const float* mu_tend = s[WF_MU_TEND];
  const bool inner = j >= jds + 1 && j < jde - 2 && i >= ids + 1 && i < ide - 2;
  if (!inner) {
    // spec_bdyupdate for t, mu and muts on the specified rows
    const bool spec = ((j == jds || j == jde - 2) && i >= ids && i < ide - 1) || (j >= jds + 1 && j < jde - 2 && (i == ids || i == ide - 2));
    if (!spec) return;
    for (int k = 0; k < kend; ++k) t[k * lev + c] = t[k * lev + c] + dts * ft[k * lev + c];
    s[WF_MU][c] = s[WF_MU][c] + dts * mu_tend[c];
    s[WF_MUTS][c] = s[WF_MUTS][c] + dts * mu_tend[c];
    return;
  }
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  const float* u1 = s[WF_U_SAVE];
  const float* v1 = s[WF_V_SAVE];
  const float* muu = s[WF_MUU];
  const float* muv = s[WF_MUV];
  const float* msfuy = s[WF_MSFUY];
  const float* mvi = s[WF_MSFVX_INV];
  const float msftx = s[WF_MSFTX][c], msfty = s[WF_MSFTY][c];
  const float* dnw = s[WF_DNW];
  const float rdx = g.rdx, rdy = g.rdy;
  auto dvdxi = [&](int k) {
    const size_t p = k * lev + c;
    return msftx * msfty *
           (rdy * ((v[p + nx] + muv[c + nx] * v1[p + nx] * mvi[c + nx]) - (v[p] + muv[c] * v1[p] * mvi[c])) +
            rdx * ((u[p + 1] + muu[c + 1] * u1[p + 1] / msfuy[c + 1]) - (u[p] + muu[c] * u1[p] / msfuy[c])));
  };
  float dmdt = 0.f;
  for (int k = 0; k < kend; ++k) dmdt = dmdt + dnw[k] * dvdxi(k);
  const float mt = mu_tend[c];
  float mu = s[WF_MU][c];
  const float muave_old = mu;
  mu = mu + dts * (dmdt + mt);
  s[WF_MU][c] = mu;
  s[WF_MUDF][c] = dmdt + mt;
  s[WF_MUTS][c] = s[WF_MUT][c] + mu;
  s[WF_MUAVE][c] = 0.5f * ((float)(1.0 + (double)g.epssm) * mu + (float)(1.0 - (double)g.epssm) * muave_old);
  float* ww = s[WF_WW];
  const float* ww1 = s[WF_WW1];
  float wprev = ww[c];
  for (int k = 1; k < kend; ++k) {
    const float wk = wprev - dnw[k - 1] * (dmdt + dvdxi(k - 1) + mt) / msfty;
    ww[k * lev + c] = wk;
    wprev = wk;
  }
  for (int k = 0; k < kend; ++k) ww[k * lev + c] = ww[k * lev + c] - ww1[k * lev + c];
  const float* t1 = s[WF_T_SAVE];
  float* t2save = s[WF_T_2SAVE];
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  const float* rdnw = s[WF_RDNW];
  const float cy = (float)(0.5 * g.rdyd), cx = (float)(0.5 * g.rdxd);
  auto wdtn = [&](int kk) {
    if (kk == 0 || kk == nz - 1) return 0.f;
    const size_t q = kk * lev + c;
    return ww[q] * (fnm[kk] * t1[q] + fnp[kk] * t1[q - lev]);
  };
  for (int k = 0; k < kend; ++k) {
    const size_t p = k * lev + c;
    float tt = t[p];
    t2save[p] = tt;
    tt = tt + msfty * dts * ft[p];
    const float hy = cy * (v[p + nx] * (t1[p + nx] + t1[p]) - v[p] * (t1[p] + t1[p - nx]));
    const float hx = cx * (u[p + 1] * (t1[p + 1] + t1[p]) - u[p] * (t1[p] + t1[p - 1]));
    tt = tt - dts * msfty * (msftx * (hy + hx) + rdnw[k] * (wdtn(k + 1) - wdtn(k)));
    t[p] = tt;
  }
}

__global__ void k_advance_w(Grid g, S s, float dts, int iteration, int nsub) {
  WRF_COLUMN_INDEX(g, j, i);
  const int nz = g.nz, kend = nz - 1, nx = g.nx;
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  if (j < jds || j >= jde || i < ids || i >= ide) return;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * nx;
  const bool inner = j >= jds + 1 && j < jde - 2 && i >= ids + 1 && i < ide - 2;
  const float gf = (float)G;
  const float ep = g.epssm;
  const float ep1 = (float)(1.0 + (double)ep), em1 = (float)(1.0 - (double)ep);
  float* w = s[WF_W];
  float* ph = s[WF_PH];
  if (inner) {
    const float* ww = s[WF_WW];
    const float* ph1 = s[WF_PH_SAVE];
    const float* phb = s[WF_PHB];
    const float* ph_tend = s[WF_PH_TEND];
    const float* t2 = s[WF_T];
    const float* t1 = s[WF_T_SAVE];
    float* t2a = s[WF_T_2SAVE];
    const float* fnm = s[WF_FNM];
    const float* fnp = s[WF_FNP];
    const float* rdnw = s[WF_RDNW];
    const float* rdn = s[WF_RDN];
    const float* c2a = s[WF_C2A];
    const float* cqw = s[WF_CQW];
    const float* alt = s[WF_ALT];
    const float* rw_tend = s[WF_RW_TEND];
    const float* a = s[WF_A];
    const float* alpha = s[WF_ALPHA];
    const float* gamma = s[WF_GAMMA];
    const float muave = s[WF_MUAVE][c], muts = s[WF_MUTS][c], mut = s[WF_MUT][c];
    const float msfty = s[WF_MSFTY][c], msftx = s[WF_MSFTX][c];
    const float msft_inv = 1.0f / msfty;
    float rhs[kMaxNz], wl[kMaxNz], t2av[kMaxNz];
    for (int k = 0; k < kend; ++k) {
      const size_t p = k * lev + c;
      float v = 0.5f * (ep1 * t2[p] + em1 * t2a[p]);
      v = (v + muave * (float)T0) / (muts * ((float)T0 + t1[p]));
      t2a[p] = v;
      t2av[k] = v;
    }
    auto wdwn = [&](int kk) {
      const size_t q = kk * lev + c, qm = q - lev;
      return 0.5f * (ww[q] + ww[qm]) * rdnw[kk - 1] * (ph1[q] - ph1[qm] + phb[q] - phb[qm]);
    };
    const float cw = (float)(0.5 * G * (1.0 - (double)ep));
    rhs[0] = 0.f;
    for (int k = 1; k < nz; ++k) {
      const size_t p = k * lev + c;
      float r = dts * (ph_tend[p] + cw * w[p]);
      if (k < kend) r = r - dts * (fnm[k] * wdwn(k + 1) + fnp[k] * wdwn(k));
      rhs[k] = ph[p] + msfty * r / mut;
    }
    // lower boundary: w from the terrain slope and near-surface winds
    {
      const float* u = s[WF_U];
      const float* v = s[WF_V];
      const float* ht = s[WF_HT];
      auto cv = [&](int cc) { return g.cf1 * v[cc] + g.cf2 * v[lev + cc] + g.cf3 * v[2 * lev + cc]; };
      auto cu = [&](int cc) { return g.cf1 * u[cc] + g.cf2 * u[lev + cc] + g.cf3 * u[2 * lev + cc]; };
      wl[0] = msfty * 0.5f * g.rdy * ((ht[c + nx] - ht[c]) * cv(c + nx) + (ht[c] - ht[c - nx]) * cv(c)) +
              msftx * 0.5f * g.rdx * ((ht[c + 1] - ht[c]) * cu(c + 1) + (ht[c] - ht[c - 1]) * cu(c));
    }
    const float cp = (float)(0.5 * (double)dts * G);
    const float cq = (float)((double)dts * G);
    for (int k = 1; k < kend; ++k) {
      const size_t p = k * lev + c;
      const float X1 = c2a[p] * rdnw[k] / mut * (ep1 * (rhs[k + 1] - rhs[k]) + em1 * (ph[p + lev] - ph[p]));
      const float X2 = c2a[p - lev] * rdnw[k - 1] / mut * (ep1 * (rhs[k] - rhs[k - 1]) + em1 * (ph[p] - ph[p - lev]));
      wl[k] = w[p] + dts * rw_tend[p] + msft_inv * cqw[p] * (cp * rdn[k] * (X1 - X2)) +
              cq * msft_inv * (rdn[k] * (c2a[p] * alt[p] * t2av[k] - c2a[p - lev] * alt[p - lev] * t2av[k - 1]) - muave);
    }
    {
      const int ke = kend;
      const size_t p = ke * lev + c, pm = p - lev;
      const float cm = (float)(-0.5 * (double)dts * G);
      wl[ke] = w[p] + dts * rw_tend[p] +
               msft_inv * (cm / mut * (rdnw[ke - 1] * rdnw[ke - 1]) * 2.0f * c2a[pm] *
                               (ep1 * (rhs[ke] - rhs[ke - 1]) + em1 * (ph[p] - ph[pm])) -
                           cq * (2.0f * rdnw[ke - 1] * c2a[pm] * alt[pm] * t2av[ke - 1] + muave));
    }
    for (int k = 1; k <= kend; ++k) {
      const size_t p = k * lev + c;
      wl[k] = (wl[k] - a[p] * wl[k - 1]) * alpha[p];
    }
    for (int k = kend - 1; k >= 1; --k) wl[k] = wl[k] - gamma[k * lev + c] * wl[k + 1];
    // Rayleigh damping of w near the model top (dampcoef 0.2, zdamp 5000 m)
    const float hdepth = 5000.0f;
    const float dampmag = (float)((double)dts * 0.2);
    const float htop = (ph1[kend * lev + c] + phb[kend * lev + c]) / gf;
    const float hbot = htop - hdepth;
    const float hpi = (float)(0.5 * 3.14159265359);
    const float* wsave = s[WF_W_SAVE];
    w[c] = wl[0];
    for (int k = 1; k < nz; ++k) {
      const size_t p = k * lev + c;
      const float hk = (ph1[p] + phb[p]) / gf;
      float dw = 0.f;
      if (hk >= hbot) {
        const float sn = sinf(hpi * (hk - hbot) / hdepth);
        dw = dampmag * (sn * sn);
      }
      const float wk = (wl[k] - dw * mut * wsave[p]) / (1.0f + dw);
      w[p] = wk;
      ph[p] = rhs[k] + msfty * 0.5f * dts * gf * ep1 * wk / muts;
    }
  } else {
    // spec_bdyupdate_ph on the specified rows (wrf_boundary.py:297-355)
    const bool spec = ((j == jds || j == jde - 2) && i >= ids && i < ide - 1) || (j >= jds + 1 && j < jde - 2 && (i == ids || i == ide - 2));
    if (spec) {
      const float muts = s[WF_MUTS][c];
      const float mu_old = muts - dts * s[WF_MU_TEND][c];
      const float* ph_save = s[WF_PH_SAVE];
      const float* ph_tend = s[WF_PH_TEND];
      for (int k = 0; k < nz; ++k) {
        const size_t p = k * lev + c;
        ph[p] = ph[p] * mu_old / muts + dts * ph_tend[p] / muts + ph_save[p] * (mu_old / muts - 1.0f);
      }
    }
  }
  // sumflux (wrf_dynamics.py:3799-3839) on [jts, jte) x [its, ite)
  float* ru_m = s[WF_RU_M];
  float* rv_m = s[WF_RV_M];
  float* ww_m = s[WF_WW_M];
  const bool ur = j < jde - 1;
  const bool vr = i < ide - 1;
  const bool wr = ur && vr;
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  const float* wwv = s[WF_WW];
  const float rn = 1.0f / 1.0f;
  (void)rn;
  for (int k = 0; k < nz; ++k) {
    const size_t p = k * lev + c;
    float a = iteration == 1 ? 0.f : ru_m[p];
    float b = iteration == 1 ? 0.f : rv_m[p];
    float cc = iteration == 1 ? 0.f : ww_m[p];
    if (k < nz - 1 && ur) a = a + u[p];
    if (k < nz - 1 && vr) b = b + v[p];
    if (wr) cc = cc + wwv[p];
    if (iteration == nsub) {
      if (k < nz - 1 && ur) a = a / (float)nsub + s[WF_MUU][c] * s[WF_U_SAVE][p] / s[WF_MSFUY][c];
      if (k < nz - 1 && vr) b = b / (float)nsub + s[WF_MUV][c] * s[WF_V_SAVE][p] * s[WF_MSFVX_INV][c];
      if (wr) cc = cc / (float)nsub + s[WF_WW1][p];
    }
    ru_m[p] = a;
    rv_m[p] = b;
    ww_m[p] = cc;
  }
}

__global__ void k_mu_uv_1(Grid g, S s) {
  WRF_COLUMN_INDEX(g, j, i);
  const int c = g.i2(j, i);
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ite = g.ide, ime = g.ide - 1, jte = g.jde;
  const float* muts = s[WF_MUTS];
  if (j >= jts && j < jme) {
    if (i >= its + 1 && i < ite - 1) s[WF_MUUS][c] = 0.5f * (muts[c] + muts[c - 1]);
    else if (i == its) s[WF_MUUS][c] = muts[c];
    else if (i == ite - 1) s[WF_MUUS][c] = muts[c - 1];
  }
  if (i >= its && i < ime) {
    if (j >= jts + 1 && j < jte - 1) s[WF_MUVS][c] = 0.5f * (muts[c] + muts[c - g.nx]);
    else if (j == jts) s[WF_MUVS][c] = muts[c];
    else if (j == jte - 1) s[WF_MUVS][c] = muts[c - g.nx];
  }
}

__global__ void k_ssfinish(Grid g, S s, float dts, int nsub, int rk_step) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nz = g.nz;
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  if (k < nz - 1 && j >= jts && j < jev && i >= its && i < ime)
    s[WF_V][p] = (s[WF_MSFVX][c] * s[WF_V][p] + s[WF_V_SAVE][p] * s[WF_MUV][c]) / s[WF_MUVS][c];
  if (k < nz - 1 && j >= jts && j < jme && i >= its && i < ieu)
    s[WF_U][p] = (s[WF_MSFUY][c] * s[WF_U][p] + s[WF_U_SAVE][p] * s[WF_MUU][c]) / s[WF_MUUS][c];
  if (j >= jts && j < jme && i >= its && i < ime) {
    const float mut = s[WF_MUT][c], muts = s[WF_MUTS][c];
    s[WF_W][p] = (s[WF_MSFTY][c] * s[WF_W][p] + s[WF_W_SAVE][p] * mut) / muts;
    s[WF_PH][p] = s[WF_PH][p] + s[WF_PH_SAVE][p];
    s[WF_WW][p] = s[WF_WW][p] + s[WF_WW1][p];
    if (k < nz - 1) {
      if (rk_step < 3)
        s[WF_T][p] = (s[WF_T][p] + s[WF_T_SAVE][p] * mut) / muts;
      else
        s[WF_T][p] = (s[WF_T][p] - (float)((double)dts * nsub) * mut * s[WF_H_DIABATIC][p] + s[WF_T_SAVE][p] * mut) / muts;
    }
    if (k == 0) s[WF_MU][c] = s[WF_MU][c] + s[WF_MU_SAVE][c];
  }
}

int launch_small_step_prep(const Grid& g, const S& s, int rk_step, float dts, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  k_ssp2d<<<col_grid(g, b2), b2, 0, st>>>(g, s, rk_step);
  k_ssp3d<<<point_grid(g, b3), b3, 0, st>>>(g, s, rk_step);
  k_p_rho<<<point_grid(g, b3), b3, 0, st>>>(g, s, 0);
  k_coef_w<<<col_grid(g, b2), b2, 0, st>>>(g, s, dts);
  return 4;
}

int launch_substep(const Grid& g, const S& s, float dts, int iteration, int nsub, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  k_advance_uv<<<point_grid(g, b3), b3, 0, st>>>(g, s, dts);
  k_advance_mu_t<<<col_grid(g, b2), b2, 0, st>>>(g, s, dts);
  k_advance_w<<<col_grid(g, b2), b2, 0, st>>>(g, s, dts, iteration, nsub);
  k_p_rho<<<point_grid(g, b3), b3, 0, st>>>(g, s, iteration);
  return 4;
}

int launch_small_step_finish(const Grid& g, const S& s, float dts, int nsub, int rk_step, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  k_mu_uv_1<<<col_grid(g, b2), b2, 0, st>>>(g, s);
  k_ssfinish<<<point_grid(g, b3), b3, 0, st>>>(g, s, dts, nsub, rk_step);
  return 2;
}

}  // namespace wrf
