// Acoustic (small) time step (wrf_dynamics.py:3152-3930, wrf_boundary.py:244-400).
//   k_ssp2d / k_ssp3d   small_step_prep (2-D masses, then 3-D perturbation form)
//   k_p_rho0            calc_p_rho before the first substep
//   k_coef_w            calc_coef_w: tridiagonal coefficients + forward sweep
//   k_advance_uv        advance_uv + spec_bdyupdate(u), (v)
//   k_acoustic_col      advance_mu_t, advance_w, sumflux, spec_bdyupdate of
//                       t / mu / muts / ph and calc_p_rho of one substep
//   k_zero_grad_w       zero_grad_bdy(w)
//   k_mu_uv_1 / k_ssfinish  calc_mu_uv_1, small_step_finish
// The vertical recurrences (mass divergence sum, ww scan, Thomas sweeps) run
// sequentially per column in the reference's order.
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

// calc_p_rho at the start of the acoustic steps (wrf_dynamics.py:3269-3313,
// step 0): al and p from the prepared state; pm1 becomes a copy of the whole
// new p (the later substeps run inside k_acoustic_col)
__global__ void k_p_rho0(Grid g, S s) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ktf = g.nz - 1;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * g.nx;
  const size_t p = k * lev + c;
  float* pp = s[WF_P];
  float pnew = pp[p];
  if (k < ktf && j >= g.jds && j < g.jde - 1 && i >= g.ids && i < g.ide - 1) {
    const float muts = s[WF_MUTS][c], mu = s[WF_MU][c];
    const float alt = s[WF_ALT][p], t1 = s[WF_T_SAVE][p];
    const float* ph = s[WF_PH];
    const float al = -1.0f / muts * (alt * mu + s[WF_RDNW][k] * (ph[p + lev] - ph[p]));
    s[WF_AL][p] = al;
    pnew = s[WF_C2A][p] * (alt * (s[WF_T][p] - mu * t1) / (muts * ((float)T0 + t1)) - al);
    pp[p] = pnew;
  }
  s[WF_PM1][p] = pnew;
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

// Fused acoustic column update of one substep: advance_mu_t, advance_w,
// sumflux, spec_bdyupdate of t / mu / muts / ph, calc_p_rho
// (wrf_dynamics.py:3528-3839, 3269-3313; wrf_boundary.py:244-355).  A block
// owns kColTX adjacent columns of one row and kColKT level groups: the
// explicit parts run in parallel over levels through shared memory, the
// vertical recurrences (column mass divergence sum, ww scan, Thomas sweeps)
// run sequentially per column in the reference's order.  No column reads
// another column's result of this kernel, so no grid-wide ordering is needed;
// zero_grad_bdy(w) follows in k_zero_grad_w.
constexpr int kColTX = 32, kColKT = 8;

struct ColArrays {  // [nz][kColTX] slices of dynamic shared memory
  float *dw, *ww, *t2av, *rhs, *a, *alpha, *gamma, *ph;
  float *muave, *muts, *mu;
};

__device__ __forceinline__ ColArrays col_arrays(float* base, int nz) {
  ColArrays c;
  const int n = nz * kColTX;
  c.dw = base; c.ww = base + n; c.t2av = base + 2 * n; c.rhs = base + 3 * n; c.a = base + 4 * n;
  c.alpha = base + 5 * n; c.gamma = base + 6 * n; c.ph = base + 7 * n;
  c.muave = base + 8 * n; c.muts = c.muave + kColTX; c.mu = c.muts + kColTX;
  return c;
}

size_t acoustic_col_smem(int nz) { return (size_t)(8 * nz * kColTX + 3 * kColTX) * sizeof(float); }

__global__ void __launch_bounds__(kColTX * kColKT) k_acoustic_col(Grid g, S s, float dts, int iteration, int nsub) {
  extern __shared__ float smem_col[];
  const int nz = g.nz, kend = nz - 1, nx = g.nx;
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const int tx = threadIdx.x % kColTX, tk = threadIdx.x / kColTX;
  const int i = ids + blockIdx.x * kColTX + tx;
  const int j = jds + blockIdx.y;
  const bool col = i < ide;                         // j < jde by the grid
  const bool inner = col && j >= jds + 1 && j < jde - 2 && i >= ids + 1 && i < ide - 2;
  const bool spec = col && (((j == jds || j == jde - 2) && i < ide - 1) || (j >= jds + 1 && j < jde - 2 && (i == ids || i == ide - 2)));
  const bool mass = inner || spec;
  const int c = col ? g.i2(j, i) : 0;
  const size_t lev = (size_t)g.ny * nx;
  ColArrays sm = col_arrays(smem_col, nz);
  auto A = [&](float* arr, int k) -> float& { return arr[k * kColTX + tx]; };
  float* t = s[WF_T];
  const float* ft = s[WF_T_TEND];
  const float* t1 = s[WF_T_SAVE];
  float* ww = s[WF_WW];
  const float* ww1 = s[WF_WW1];
  const float* dnw = s[WF_DNW];
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  const float* rdnw = s[WF_RDNW];
  const float* rdn = s[WF_RDN];
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  const float msftx = col ? s[WF_MSFTX][c] : 1.f, msfty = col ? s[WF_MSFTY][c] : 1.f;
  const float mut = col ? s[WF_MUT][c] : 1.f;
  const float mu_tend = col ? s[WF_MU_TEND][c] : 0.f;
  const float ep = g.epssm;
  const float ep1 = (float)(1.0 + (double)ep), em1 = (float)(1.0 - (double)ep);

  // --- A: horizontal mass-flux divergence per level (inner) / spec t, mu, muts
  if (inner) {
    const float* u1 = s[WF_U_SAVE];
    const float* v1 = s[WF_V_SAVE];
    const float* muu = s[WF_MUU];
    const float* muv = s[WF_MUV];
    const float* msfuy = s[WF_MSFUY];
    const float* mvi = s[WF_MSFVX_INV];
    const float rdx = g.rdx, rdy = g.rdy;
    #pragma unroll 4
    for (int k = tk; k < kend; k += kColKT) {
      const size_t p = k * lev + c;
      A(sm.dw, k) = msftx * msfty *
                    (rdy * ((__ldg(&v[p + nx]) + __ldg(&muv[c + nx]) * __ldg(&v1[p + nx]) * __ldg(&mvi[c + nx])) - (__ldg(&v[p]) + __ldg(&muv[c]) * __ldg(&v1[p]) * __ldg(&mvi[c]))) +
                     rdx * ((__ldg(&u[p + 1]) + __ldg(&muu[c + 1]) * __ldg(&u1[p + 1]) / __ldg(&msfuy[c + 1])) - (__ldg(&u[p]) + __ldg(&muu[c]) * __ldg(&u1[p]) / __ldg(&msfuy[c]))));
    }
  } else if (spec) {
    #pragma unroll 4
    for (int k = tk; k < kend; k += kColKT) t[k * lev + c] = t[k * lev + c] + dts * __ldg(&ft[k * lev + c]);
    if (tk == 0) {
      const float mu = s[WF_MU][c] + dts * mu_tend;
      const float muts = s[WF_MUTS][c] + dts * mu_tend;
      s[WF_MU][c] = mu;
      s[WF_MUTS][c] = muts;
      sm.mu[tx] = mu;
      sm.muts[tx] = muts;
    }
  }
  __syncthreads();
  // --- B: column mass tendency and the ww scan (sequential, reference order)
  if (inner && tk == 0) {
    float dmdt = 0.f;
    for (int k = 0; k < kend; ++k) dmdt = dmdt + __ldg(&dnw[k]) * A(sm.dw, k);
    float mu = s[WF_MU][c];
    const float muave_old = mu;
    mu = mu + dts * (dmdt + mu_tend);
    const float muts = mut + mu;
    const float muave = 0.5f * (ep1 * mu + em1 * muave_old);
    s[WF_MU][c] = mu;
    s[WF_MUDF][c] = dmdt + mu_tend;
    s[WF_MUTS][c] = muts;
    s[WF_MUAVE][c] = muave;
    sm.mu[tx] = mu;
    sm.muts[tx] = muts;
    sm.muave[tx] = muave;
    float wprev = ww[c];
    A(sm.ww, 0) = wprev;
    for (int k = 1; k < kend; ++k) {
      const float wk = wprev - __ldg(&dnw[k - 1]) * (dmdt + A(sm.dw, k - 1) + mu_tend) / msfty;
      A(sm.ww, k) = wk;
      wprev = wk;
    }
  }
  __syncthreads();
  // --- C: final ww (inner: scan - ww1), potential temperature (inner)
  if (col) {
    #pragma unroll 4
    for (int k = tk; k < nz; k += kColKT) {
      const size_t p = k * lev + c;
      float w = ww[p];
      if (inner && k < kend) {
        w = A(sm.ww, k) - __ldg(&ww1[p]);
        ww[p] = w;
      }
      A(sm.ww, k) = w;
    }
  }
  __syncthreads();
  const float muave = inner ? sm.muave[tx] : 0.f;
  const float muts = mass ? sm.muts[tx] : 1.f;
  if (inner) {
    const float cy = (float)(0.5 * g.rdyd), cx = (float)(0.5 * g.rdxd);
    auto wdtn = [&](int kk) {
      if (kk == 0 || kk == nz - 1) return 0.f;
      const size_t q = kk * lev + c;
      return A(sm.ww, kk) * (__ldg(&fnm[kk]) * __ldg(&t1[q]) + __ldg(&fnp[kk]) * __ldg(&t1[q - lev]));
    };
    float* t2a = s[WF_T_2SAVE];
    #pragma unroll 4
    for (int k = tk; k < kend; k += kColKT) {
      const size_t p = k * lev + c;
      const float told = t[p];
      float tt = told + msfty * dts * __ldg(&ft[p]);
      const float hy = cy * (__ldg(&v[p + nx]) * (__ldg(&t1[p + nx]) + __ldg(&t1[p])) - __ldg(&v[p]) * (__ldg(&t1[p]) + __ldg(&t1[p - nx])));
      const float hx = cx * (__ldg(&u[p + 1]) * (__ldg(&t1[p + 1]) + __ldg(&t1[p])) - __ldg(&u[p]) * (__ldg(&t1[p]) + __ldg(&t1[p - 1])));
      tt = tt - dts * msfty * (msftx * (hy + hx) + __ldg(&rdnw[k]) * (wdtn(k + 1) - wdtn(k)));
      t[p] = tt;
      // time-averaged theta of advance_w (t_2ave)
      float av = 0.5f * (ep1 * tt + em1 * told);
      av = (av + muave * (float)T0) / (muts * ((float)T0 + __ldg(&t1[p])));
      t2a[p] = av;
      A(sm.t2av, k) = av;
    }
    // --- D: right-hand side of the phi equation, tridiagonal coefficients
    const float* ph1 = s[WF_PH_SAVE];
    const float* phb = s[WF_PHB];
    const float* ph_tend = s[WF_PH_TEND];
    const float* w = s[WF_W];
    const float* ph = s[WF_PH];
    auto wdwn = [&](int kk) {
      const size_t q = kk * lev + c, qm = q - lev;
      return 0.5f * (A(sm.ww, kk) + A(sm.ww, kk - 1)) * __ldg(&rdnw[kk - 1]) * (__ldg(&ph1[q]) - __ldg(&ph1[qm]) + __ldg(&phb[q]) - __ldg(&phb[qm]));
    };
    const float cw = (float)(0.5 * G * (1.0 - (double)ep));
    #pragma unroll 4
    for (int k = tk; k < nz; k += kColKT) {
      const size_t p = k * lev + c;
      A(sm.ph, k) = ph[p];
      A(sm.a, k) = __ldg(&s[WF_A][p]);
      A(sm.alpha, k) = __ldg(&s[WF_ALPHA][p]);
      A(sm.gamma, k) = __ldg(&s[WF_GAMMA][p]);
      if (k == 0) {
        A(sm.rhs, 0) = 0.f;
        continue;
      }
      float r = dts * (__ldg(&ph_tend[p]) + cw * w[p]);
      if (k < kend) r = r - dts * (__ldg(&fnm[k]) * wdwn(k + 1) + __ldg(&fnp[k]) * wdwn(k));
      A(sm.rhs, k) = ph[p] + msfty * r / mut;
    }
  }
  __syncthreads();
  // --- E: explicit part of w (inner)
  if (inner) {
    const float* w = s[WF_W];
    const float* c2a = s[WF_C2A];
    const float* cqw = s[WF_CQW];
    const float* alt = s[WF_ALT];
    const float* rw_tend = s[WF_RW_TEND];
    const float msft_inv = 1.0f / msfty;
    const float cp = (float)(0.5 * (double)dts * G);
    const float cq = (float)((double)dts * G);
    #pragma unroll 4
    for (int k = tk; k <= kend; k += kColKT) {
      const size_t p = k * lev + c;
      float wl;
      if (k == 0) {  // lower boundary: w from the terrain slope and near-surface winds
        const float* ht = s[WF_HT];
        auto cv = [&](int cc) { return g.cf1 * __ldg(&v[cc]) + g.cf2 * __ldg(&v[lev + cc]) + g.cf3 * __ldg(&v[2 * lev + cc]); };
        auto cu = [&](int cc) { return g.cf1 * __ldg(&u[cc]) + g.cf2 * __ldg(&u[lev + cc]) + g.cf3 * __ldg(&u[2 * lev + cc]); };
        wl = msfty * 0.5f * g.rdy * ((__ldg(&ht[c + nx]) - __ldg(&ht[c])) * cv(c + nx) + (__ldg(&ht[c]) - __ldg(&ht[c - nx])) * cv(c)) +
             msftx * 0.5f * g.rdx * ((__ldg(&ht[c + 1]) - __ldg(&ht[c])) * cu(c + 1) + (__ldg(&ht[c]) - __ldg(&ht[c - 1])) * cu(c));
      } else if (k < kend) {
        const float X1 = __ldg(&c2a[p]) * __ldg(&rdnw[k]) / mut *
                         (ep1 * (A(sm.rhs, k + 1) - A(sm.rhs, k)) + em1 * (A(sm.ph, k + 1) - A(sm.ph, k)));
        const float X2 = __ldg(&c2a[p - lev]) * __ldg(&rdnw[k - 1]) / mut *
                         (ep1 * (A(sm.rhs, k) - A(sm.rhs, k - 1)) + em1 * (A(sm.ph, k) - A(sm.ph, k - 1)));
        wl = w[p] + dts * __ldg(&rw_tend[p]) + msft_inv * __ldg(&cqw[p]) * (cp * __ldg(&rdn[k]) * (X1 - X2)) +
             cq * msft_inv *
                 (__ldg(&rdn[k]) * (__ldg(&c2a[p]) * __ldg(&alt[p]) * A(sm.t2av, k) - __ldg(&c2a[p - lev]) * __ldg(&alt[p - lev]) * A(sm.t2av, k - 1)) - muave);
      } else {
        const size_t pm = p - lev;
        const float cm = (float)(-0.5 * (double)dts * G);
        wl = w[p] + dts * __ldg(&rw_tend[p]) +
             msft_inv * (cm / mut * (__ldg(&rdnw[kend - 1]) * __ldg(&rdnw[kend - 1])) * 2.0f * __ldg(&c2a[pm]) *
                             (ep1 * (A(sm.rhs, kend) - A(sm.rhs, kend - 1)) + em1 * (A(sm.ph, kend) - A(sm.ph, kend - 1))) -
                         cq * (2.0f * __ldg(&rdnw[kend - 1]) * __ldg(&c2a[pm]) * __ldg(&alt[pm]) * A(sm.t2av, kend - 1) + muave));
      }
      A(sm.dw, k) = wl;
    }
  }
  __syncthreads();
  // --- F: Thomas sweeps (sequential per column)
  if (inner && tk == 0) {
    float prev = A(sm.dw, 0);
    for (int k = 1; k <= kend; ++k) {
      prev = (A(sm.dw, k) - A(sm.a, k) * prev) * A(sm.alpha, k);
      A(sm.dw, k) = prev;
    }
    for (int k = kend - 1; k >= 1; --k) {
      prev = A(sm.dw, k) - A(sm.gamma, k) * prev;
      A(sm.dw, k) = prev;
    }
  }
  __syncthreads();
  // --- G: Rayleigh damping, w and phi (inner); spec phi; sumflux (all)
  float* ph = s[WF_PH];
  if (inner) {
    float* w = s[WF_W];
    const float* ph1 = s[WF_PH_SAVE];
    const float* phb = s[WF_PHB];
    const float* wsave = s[WF_W_SAVE];
    const float gf = (float)G;
    const float hdepth = 5000.0f;
    const float dampmag = (float)((double)dts * 0.2);
    const float htop = (__ldg(&ph1[kend * lev + c]) + __ldg(&phb[kend * lev + c])) / gf;
    const float hbot = htop - hdepth;
    const float hpi = (float)(0.5 * 3.14159265359);
    #pragma unroll 4
    for (int k = tk; k < nz; k += kColKT) {
      const size_t p = k * lev + c;
      if (k == 0) {
        w[c] = A(sm.dw, 0);
        continue;
      }
      const float hk = (__ldg(&ph1[p]) + __ldg(&phb[p])) / gf;
      float dwd = 0.f;
      if (hk >= hbot) {
        const float sn = sinf(hpi * (hk - hbot) / hdepth);
        dwd = dampmag * (sn * sn);
      }
      const float wk = (A(sm.dw, k) - dwd * mut * __ldg(&wsave[p])) / (1.0f + dwd);
      w[p] = wk;
      const float phk = A(sm.rhs, k) + msfty * 0.5f * dts * gf * ep1 * wk / muts;
      ph[p] = phk;
      A(sm.ph, k) = phk;
    }
  } else if (spec) {
    const float mu_old = muts - dts * mu_tend;
    const float* ph_save = s[WF_PH_SAVE];
    const float* ph_tend = s[WF_PH_TEND];
    #pragma unroll 4
    for (int k = tk; k < nz; k += kColKT) {
      const size_t p = k * lev + c;
      const float phk = ph[p] * mu_old / muts + dts * __ldg(&ph_tend[p]) / muts + ph_save[p] * (mu_old / muts - 1.0f);
      ph[p] = phk;
      A(sm.ph, k) = phk;
    }
  }
  if (col) {
    float* ru_m = s[WF_RU_M];
    float* rv_m = s[WF_RV_M];
    float* ww_m = s[WF_WW_M];
    const bool ur = j < jde - 1, vr = i < ide - 1, wr = ur && vr;
    #pragma unroll 4
    for (int k = tk; k < nz; k += kColKT) {
      const size_t p = k * lev + c;
      float a = iteration == 1 ? 0.f : ru_m[p];
      float b = iteration == 1 ? 0.f : rv_m[p];
      float cc = iteration == 1 ? 0.f : ww_m[p];
      if (k < nz - 1 && ur) a = a + __ldg(&u[p]);
      if (k < nz - 1 && vr) b = b + __ldg(&v[p]);
      if (wr) cc = cc + A(sm.ww, k);
      if (iteration == nsub) {
        if (k < nz - 1 && ur) a = a / (float)nsub + s[WF_MUU][c] * s[WF_U_SAVE][p] / s[WF_MSFUY][c];
        if (k < nz - 1 && vr) b = b / (float)nsub + s[WF_MUV][c] * s[WF_V_SAVE][p] * s[WF_MSFVX_INV][c];
        if (wr) cc = cc / (float)nsub + __ldg(&ww1[p]);
      }
      ru_m[p] = a;
      rv_m[p] = b;
      ww_m[p] = cc;
    }
  }
  __syncthreads();
  // --- H: calc_p_rho with divergence damping (mass columns)
  if (mass) {
    const float mu = sm.mu[tx];
    const float* alt = s[WF_ALT];
    const float* c2a = s[WF_C2A];
    float* al = s[WF_AL];
    float* pp = s[WF_P];
    float* pm1 = s[WF_PM1];
    #pragma unroll 4
    for (int k = tk; k < kend; k += kColKT) {
      const size_t p = k * lev + c;
      const float altk = __ldg(&alt[p]), t1k = __ldg(&t1[p]);
      const float alk = -1.0f / muts * (altk * mu + __ldg(&rdnw[k]) * (A(sm.ph, k + 1) - A(sm.ph, k)));
      al[p] = alk;
      const float pnew = __ldg(&c2a[p]) * (altk * (t[p] - mu * t1k) / (muts * ((float)T0 + t1k)) - alk);
      pp[p] = pnew + g.smdiv * (pnew - pm1[p]);
      pm1[p] = pnew;
    }
  }
}

// zero_grad_bdy(w) on the specified rows, all levels (wrf_boundary.py:358-400)
__global__ void k_zero_grad_w(Grid g, S s) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nx = g.nx;
  const int ibs = g.ids, ibe = g.ide - 1, jbs = g.jds, jbe = g.jde - 1;
  int sj = -1, si = -1;
  if (j == jbs || j == jbe - 1) {
    if (i >= ibs && i < ibe) {
      sj = (j == jbs) ? jbs + 1 : jbe - 2;
      si = (i == ibs) ? ibs + 1 : (i == ibe - 1 ? ibe - 2 : i);
    }
  } else if (j > jbs && j < jbe - 1 && (i == ibs || i == ibe - 1)) {
    sj = j;
    si = (i == ibs) ? ibs + 1 : ibe - 2;
  }
  if (sj < 0) return;
  float* w = s[WF_W];
  const size_t base = (size_t)k * g.ny * nx;
  w[base + (size_t)j * nx + i] = w[base + (size_t)sj * nx + si];
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
  k_p_rho0<<<point_grid(g, b3), b3, 0, st>>>(g, s);
  k_coef_w<<<col_grid(g, b2), b2, 0, st>>>(g, s, dts);
  return 4;
}

int launch_substep(const Grid& g, const S& s, float dts, int iteration, int nsub, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_advance_uv<<<point_grid(g, b3), b3, 0, st>>>(g, s, dts);
  const size_t smem = acoustic_col_smem(g.nz);
  static unsigned attr_set = 0;  // one bit per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (smem > 48 * 1024 && dev < 32 && !(attr_set & (1u << dev))) {
    cudaFuncSetAttribute(k_acoustic_col, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr_set |= 1u << dev;
  }
  const dim3 gc((g.ide - g.ids + kColTX - 1) / kColTX, g.jde - g.jds);
  k_acoustic_col<<<gc, kColTX * kColKT, smem, st>>>(g, s, dts, iteration, nsub);
  k_zero_grad_w<<<point_grid(g, b3), b3, 0, st>>>(g, s);
  return 3;
}

int launch_small_step_finish(const Grid& g, const S& s, float dts, int nsub, int rk_step, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  k_mu_uv_1<<<col_grid(g, b2), b2, 0, st>>>(g, s);
  k_ssfinish<<<point_grid(g, b3), b3, 0, st>>>(g, s, dts, nsub, rk_step);
  return 2;
}

}  // namespace wrf
