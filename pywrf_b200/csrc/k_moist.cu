// Moisture transport, equation of state and end-of-step boundaries.
//   k_hdiff_moist   first-stage horizontal diffusion of qv..qg (rk_scalar_tend,
//                   wrf_dynamics.py:4022-4031; mass = muts, K = xkhh)
//   k_moist_update  rk_update_scalar (wrf_dynamics.py:4055-4119)
//   k_eos_flowdep   flow_dep_bdy for qc..qg (wrf_boundary.py:470-508) and
//                   calc_p_rho_phi (wrf_dynamics.py:4124-4164) + NaN count
//   k_bdy_final     spec_bdy_final u, v, t, ph, qv (wrf_boundary.py:511-587)
//   k_w_surface     set_w_surface (wrf_dynamics.py:4218-4324)
#include "kernels.cuh"

namespace wrf {

__global__ void k_hdiff_moist(Grid g, S s) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  if (k >= g.nz - 1 || j < jds + 1 || j >= jde - 2 || i < ids + 1 || i >= ide - 2) return;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const int c = g.i2(j, i), nx = g.nx;
  const size_t p = k * lev + c;
  const float* mut = s[WF_MUTS];
  const float* K = s[WF_XKHH];
  const float* msfux = s[WF_MSFUX];
  const float* msfuy = s[WF_MSFUY];
  const float* msfvy = s[WF_MSFVY];
  const float* mvi = s[WF_MSFVX_INV];
  const float rdx = g.rdx, rdy = g.rdy;
  const float mkrdxm = (msfux[c] / msfuy[c]) * 0.5f * (K[p] + K[p - 1]) * 0.5f * (mut[c] + mut[c - 1]) * rdx;
  const float mkrdxp = (msfux[c + 1] / msfuy[c + 1]) * 0.5f * (K[p + 1] + K[p]) * 0.5f * (mut[c + 1] + mut[c]) * rdx;
  const float mrdx = s[WF_MSFTX][c] * s[WF_MSFTY][c] * rdx;
  const float mkrdym = (msfvy[c] * mvi[c]) * 0.5f * (K[p] + K[p - nx]) * 0.5f * (mut[c] + mut[c - nx]) * rdy;
  const float mkrdyp = (msfvy[c + nx] * mvi[c + nx]) * 0.5f * (K[p + nx] + K[p]) * 0.5f * (mut[c + nx] + mut[c]) * rdy;
  const float mrdy = s[WF_MSFTX][c] * s[WF_MSFTY][c] * rdy;
  // all six species' updates are formed before any is stored
  float o[6];
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    const float* f = s[WF_MOIST] + (m + 1) * n3;
    const float* tend = s[WF_MOIST_TEND] + (m + 1) * n3;
    const float fc = f[p];
    o[m] = tend[p] + (mrdx * (mkrdxp * (f[p + 1] - fc) - mkrdxm * (fc - f[p - 1])) +
                      mrdy * (mkrdyp * (f[p + nx] - fc) - mkrdym * (fc - f[p - nx])));
  }
#pragma unroll
  for (int m = 0; m < 6; ++m) s[WF_MOIST_TEND][(m + 1) * n3 + p] = o[m];
}

// every species' operands are loaded before any store, so that the loads of
// the six species are in flight together (a store to one species' field would
// otherwise hold back the next species' loads)
__global__ void k_moist_update(Grid g, S s, int rk_step, float dt) {
  WRF_POINT_INDEX(g, k, j, i);
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const int c = g.i2(j, i);
  const size_t p = k * lev + c;
  const bool full = k < g.nz - 1 && j >= g.jds && j < g.jde - 1 && i >= g.ids && i < g.ide - 1;
  const bool inner = full && j >= g.jds + 1 && j < g.jde - 2 && i >= g.ids + 1 && i < g.ide - 2;
  float muold = 0.f, munew = 0.f, msfty = 0.f;
  if (full) {
    muold = s[WF_MU_1][c] + s[WF_MUB][c];
    munew = s[WF_MU][c] + s[WF_MUB][c];
    msfty = s[WF_MSFTY][c];
  }
  float* q = s[WF_MOIST];
  float* qold = s[WF_MOIST_OLD];
  float cur[6], adv[6], mt[6], qo[6];
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    const size_t o = (size_t)(m + 1) * n3 + p;
    cur[m] = q[o];
    adv[m] = inner ? s[WF_ADVECT_TEND][o] : 0.f;
    mt[m] = full ? s[WF_MOIST_TEND][o] : 0.f;
    qo[m] = (full && rk_step != 1) ? qold[o] : cur[m];
  }
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    const size_t o = (size_t)(m + 1) * n3 + p;
    if (rk_step == 1) qold[o] = cur[m];
    if (!full) continue;
    float tend = inner ? adv[m] * msfty : 0.f;
    tend = tend + mt[m];
    q[o] = (muold * qo[m] + dt * tend) / munew;
  }
}

__global__ void k_eos_flowdep(Grid g, S s, int do_flowdep) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nz = g.nz, nx = g.nx;
  const size_t lev = (size_t)g.ny * nx, n3 = g.n3();
  const int c = g.i2(j, i);
  const size_t p = k * lev + c;
  const int its = g.ids, jts = g.jds, itf = g.ide - 1, jtf = g.jde - 1;
  // the equation of state's operands, loaded before the flow-dependent
  // boundary copies store (they write other moisture slots)
  const bool eos = k < nz - 1 && j >= jts && j < g.jde - 1 && i >= its && i < g.ide - 1;
  float phu = 0.f, phk = 0.f, muts = 1.f, mu = 0.f, alb = 0.f, rdk = 0.f, qv = 0.f, tk = 0.f, pbk = 0.f;
  if (eos) {
    const float* ph = s[WF_PH];
    phu = ph[p + lev];
    phk = ph[p];
    muts = s[WF_MUTS][c];
    mu = s[WF_MU][c];
    alb = s[WF_ALB][p];
    rdk = s[WF_RDNW][k];
    qv = s[WF_MOIST][n3 + p];
    tk = s[WF_T][p];
    pbk = s[WF_PB][p];
  }
  if (do_flowdep && k < nz - 1) {
    // zero inflow / zero-gradient outflow for qc..qg on the outer row
    const float* um = s[WF_RU_M];
    const float* vm = s[WF_RV_M];
    int mode = 0, sj = 0, si = 0;  // 1: copy (sj, si); 2: copy if flow condition else 0
    bool cond = false;
    const size_t base = k * lev;
    if (j == jts && i >= its && i < itf) {
      if (i == its) { mode = 1; sj = jts + 1; si = its + 1; }
      else if (i == itf - 1) { mode = 1; sj = jts + 1; si = itf - 2; }
      else { mode = 2; sj = jts + 1; si = i; cond = vm[base + (size_t)jts * nx + i] < 0.f; }
    } else if (j == jtf - 1 && i >= its && i < itf) {
      if (i == its) { mode = 1; sj = jtf - 2; si = its + 1; }
      else if (i == itf - 1) { mode = 1; sj = jtf - 2; si = itf - 2; }
      else { mode = 2; sj = jtf - 2; si = i; cond = vm[base + (size_t)jtf * nx + i] > 0.f; }
    } else if (j > jts && j < jtf - 1 && i == its) {
      mode = 2; sj = j; si = its + 1; cond = um[base + (size_t)j * nx + its] < 0.f;
    } else if (j > jts && j < jtf - 1 && i == itf - 1) {
      mode = 2; sj = j; si = itf - 2; cond = um[base + (size_t)j * nx + itf] > 0.f;
    }
    if (mode) {
      for (int m = 2; m < 7; ++m) {
        float* f = s[WF_MOIST] + m * n3;
        const float src = f[base + (size_t)sj * nx + si];
        f[p] = (mode == 1 || cond) ? src : 0.f;
      }
    }
  }
  if (eos) {
    const float al = -1.0f / muts * (alb * mu + rdk * (phu - phk));
    const float qvf = 1.0f + (float)RVOVRD * qv;
    const float temp = ((float)R_D * ((float)T0 + tk) * qvf) / ((float)P0 * (al + alb));
    const float pv = wpow_eos(temp, (float)CPOVCV) * (float)P0 - pbk;
    s[WF_AL][p] = al;
    s[WF_P][p] = pv;
    if (isnan(pv)) atomicAdd(reinterpret_cast<int*>(s[WF_STATUS]) + WRF_ST_NAN_P, 1);
  }
}

__global__ void k_bdy_final(Grid g, S s, int ring) {
  int k, j, i;
  k = blockIdx.z;
  if (ring) {
    if (!ring_point(g, blockIdx.x * blockDim.x + threadIdx.x, j, i)) return;
  } else {
    i = blockIdx.x * blockDim.x + threadIdx.x;
    j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
  }
  const int nz = g.nz, nx = g.nx, ny = g.ny;
  const size_t lev = (size_t)ny * nx, n3 = g.n3();
  const int c = g.i2(j, i);
  const size_t p = k * lev + c;
  const float dtbc = s[WF_DSCAL][DS_DTBC];
  const int its = g.ids, jts = g.jds;
  // value for one stagger: y rows first, then x columns (which overwrite corners)
  auto put = [&](float* f, int bx, const float* mu, const float* msf, int ibe, int jbe, int itf, int jtf, int ktf) {
    if (k >= ktf) return;
    float val = 0.f;
    bool hit = false;
    auto ybv = [&](int id, int ii) { return s[id][((size_t)k * 5) * nx + ii]; };
    auto xbv = [&](int id, int jj) { return s[id][((size_t)k * ny + jj) * 5]; };
    if (i >= its && i < ibe) {
      if (j == jts) { val = ybv(bx + 2, i) + dtbc * ybv(bx + 6, i); hit = true; }
      if (j == jtf - 1) { val = ybv(bx + 3, i) + dtbc * ybv(bx + 7, i); hit = true; }
    }
    if (j >= jts && j < jbe) {
      if (i == its) { val = xbv(bx + 0, j) + dtbc * xbv(bx + 4, j); hit = true; }
      if (i == itf - 1) { val = xbv(bx + 1, j) + dtbc * xbv(bx + 5, j); hit = true; }
    }
    if (!hit) return;
    f[p] = (msf ? msf[c] : 1.0f) * val / mu[c];
  };
  put(s[WF_U], WF_U_BXS, s[WF_MUUS], s[WF_MSFUY], g.ide, g.jde - 1, g.ide, g.jde - 1, nz - 1);
  put(s[WF_V], WF_V_BXS, s[WF_MUVS], s[WF_MSFVX], g.ide - 1, g.jde, g.ide - 1, g.jde, nz - 1);
  put(s[WF_T], WF_T_BXS, s[WF_MUTS], nullptr, g.ide - 1, g.jde - 1, g.ide - 1, g.jde - 1, nz - 1);
  put(s[WF_PH], WF_PH_BXS, s[WF_MUTS], nullptr, g.ide - 1, g.jde - 1, g.ide - 1, g.jde - 1, nz);
  put(s[WF_MOIST] + n3, WF_QV_BXS, s[WF_MUTS], nullptr, g.ide - 1, g.jde - 1, g.ide - 1, g.jde - 1, nz - 1);
}

__global__ void k_w_surface(Grid g, S s) {
  WRF_COLUMN_INDEX(g, j, i);
  const int its = g.ids, ite = g.ide, jts = g.jds, jte = g.jde, nx = g.nx;
  if (j < jts || j > jte - 2 || i < its || i > ite - 2) return;
  const size_t lev = (size_t)g.ny * nx;
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  const float* ht = s[WF_HT];
  const float* msftx = s[WF_MSFTX];
  const float* msfty = s[WF_MSFTY];
  const int c = g.i2(j, i);
  auto cv = [&](int cc) { return g.cf1 * v[cc] + g.cf2 * v[lev + cc] + g.cf3 * v[2 * lev + cc]; };
  auto cu = [&](int cc) { return g.cf1 * u[cc] + g.cf2 * u[lev + cc] + g.cf3 * u[2 * lev + cc]; };
  const float hy = 0.5f * g.rdy, hx = 0.5f * g.rdx;
  (void)hy; (void)hx;
  const bool jlo = j == jts, jhi = j == jte - 2, ilo = i == its, ihi = i == ite - 2;
  float yterm, xterm;
  // y slope term
  if (jlo && ihi) yterm = (ht[c + nx] - ht[c + nx]) * cv(c + nx);   // reference differences jts+1 with itself
  else if (jlo) yterm = (ht[c + nx] - ht[c]) * cv(c + nx);
  else if (jhi) yterm = (ht[c] - ht[c - nx]) * cv(c);
  else yterm = (ht[c + nx] - ht[c]) * cv(c + nx) + (ht[c] - ht[c - nx]) * cv(c);
  // x slope term
  if (ilo) xterm = (ht[c + 1] - ht[c]) * cu(c + 1);
  else if (ihi) xterm = (ht[c] - ht[c - 1]) * cu(c);
  else xterm = (ht[c + 1] - ht[c]) * cu(c + 1) + (ht[c] - ht[c - 1]) * cu(c);
  const float mx = (jhi && ihi) ? msftx[g.i2(jts, its)] : msftx[c];   // reference corner uses msftx(jts, its)
  s[WF_W][c] = msfty[c] * 0.5f * g.rdy * yterm + mx * 0.5f * g.rdx * xterm;
}

int launch_moist(const Grid& g, const S& s, int rk_step, float dt_rk, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_moist_update<<<point_grid(g, b3), b3, 0, st>>>(g, s, rk_step, dt_rk);
  k_eos_flowdep<<<point_grid(g, b3), b3, 0, st>>>(g, s, 1);
  return 2;
}

// calc_p_rho_phi alone (al and p from ph, t, qv; NaN in p counted)
int launch_eos(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_eos_flowdep<<<point_grid(g, b3), b3, 0, st>>>(g, s, 0);
  return 1;
}

int launch_hdiff_moist(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_hdiff_moist<<<point_grid(g, b3), b3, 0, st>>>(g, s);
  return 1;
}

int launch_bdy_final(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  if (kernel_form() == WRF_FORM_FAST && ring_fits(g))
    k_bdy_final<<<dim3((ring_size(g) + 127) / 128, 1, g.nz), 128, 0, st>>>(g, s, 1);
  else
    k_bdy_final<<<point_grid(g, b3), b3, 0, st>>>(g, s, 0);
  k_w_surface<<<col_grid(g, b2), b2, 0, st>>>(g, s);
  return 2;
}

}  // namespace wrf
