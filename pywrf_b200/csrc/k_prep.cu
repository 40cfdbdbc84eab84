// RK-stage preparation and first-stage Smagorinsky diffusion.
//   k_rk_prep2d   calculate_full + calc_mu_uv        (wrf_dynamics.py:30-61)
//   k_rk_prep3d   couple_momentum, calc_cq, calc_alt, calc_php (:64-159)
//   k_ww_cp       calc_ww_cp: column divergence, k-sum, upward scan (:89-118)
//   k_diff_metrics compute_diff_metrics (rdzw, zx, zy)          (:491-536)
//   k_deform      cal_deform_and_div: defor11, defor22, defor12  (:539-813)
//   k_defor12_bc  the edge copies of defor12                     (:727-730)
//   k_km          calculate_km_kh 2-D Smagorinsky xkmh, xkhh     (:958-995)
//   k_hdiff       horizontal_diffusion u, v, w + _3dmp theta     (:2623-2915)
//   k_relax       relax_bdytend for u, v, ph, t, mu (wrf_boundary.py:52-147)
#include "kernels.cuh"
#include "relax.cuh"

namespace wrf {

__global__ void k_rk_prep2d(Grid g, S s) {
  WRF_COLUMN_INDEX(g, j, i);
  const float* mu = s[WF_MU];
  const float* mub = s[WF_MUB];
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const int c = g.i2(j, i);
  if (j >= jds && j < jde - 1 && i >= ids && i < ide - 1) s[WF_MUT][c] = mub[c] + mu[c];
  if (j >= jds && j < jde - 1) {
    if (i >= ids + 1 && i < ide - 1)
      s[WF_MUU][c] = 0.5f * (mu[c] + mu[c - 1] + mub[c] + mub[c - 1]);
    else if (i == ids)
      s[WF_MUU][c] = mu[c] + mub[c];
    else if (i == ide - 1)
      s[WF_MUU][c] = mu[c - 1] + mub[c - 1];
  }
  if (i >= ids && i < ide - 1) {
    if (j >= jds + 1 && j < jde - 1)
      s[WF_MUV][c] = 0.5f * (mu[c] + mu[c - g.nx] + mub[c] + mub[c - g.nx]);
    else if (j == jds)
      s[WF_MUV][c] = mu[c] + mub[c];
    else if (j == jde - 1)
      s[WF_MUV][c] = mu[c - g.nx] + mub[c - g.nx];
  }
}

__device__ __forceinline__ float qsum7(const float* moist, size_t n3, int p) {
  float q = moist[p];
  for (int m = 1; m < 7; ++m) q = q + moist[(size_t)m * n3 + p];
  return q;
}

// operands first, then the stores: the moisture sums of the point and of its
// west, south and lower neighbours are each formed once (the stores between
// them would otherwise make the compiler reload them)
__global__ void k_rk_prep3d(Grid g, S s) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, nz = g.nz;
  const int p = g.i3(k, j, i);
  const int c = g.i2(j, i);
  const size_t n3 = g.n3();
  const int lev = g.ny * g.nx;
  const float* moist = s[WF_MOIST];
  const bool mrow = j >= jds && j < jde - 1;
  const bool mcol = i >= ids && i < ide - 1;
  const bool du = k < nz - 1 && mrow && i >= ids && i < ide;
  const bool dv = k < nz - 1 && j >= jds && j < jde && mcol;
  const bool dm = k < nz - 1 && mrow && mcol;
  const bool dw = dm && k >= 1;
  const bool dr = mrow && mcol;
  const float qp = (du || dv || dw) ? qsum7(moist, n3, p) : 0.f;
  const float qw = du ? qsum7(moist, n3, p - 1) : 0.f;
  const float qs = dv ? qsum7(moist, n3, p - g.nx) : 0.f;
  const float qb = dw ? qsum7(moist, n3, p - lev) : 0.f;
  float uu = 0.f, muu = 0.f, mfu = 1.f, vv = 0.f, muv = 0.f, mvxi = 0.f;
  if (du) {
    uu = s[WF_U][p];
    muu = s[WF_MUU][c];
    mfu = s[WF_MSFU][c];
  }
  if (dv) {
    vv = s[WF_V][p];
    muv = s[WF_MUV][c];
    mvxi = s[WF_MSFVX_INV][c];
  }
  float alv = 0.f, albv = 0.f, phb0 = 0.f, phb1 = 0.f, ph0 = 0.f, ph1 = 0.f;
  if (dm) {
    alv = s[WF_AL][p];
    albv = s[WF_ALB][p];
    phb0 = s[WF_PHB][p];
    phb1 = s[WF_PHB][p + lev];
    ph0 = s[WF_PH][p];
    ph1 = s[WF_PH][p + lev];
  }
  float wv = 0.f, mutv = 0.f, mft = 1.f;
  if (dr) {
    wv = s[WF_W][p];
    mutv = s[WF_MUT][c];
    mft = s[WF_MSFT][c];
  }
  if (du) {
    s[WF_RU][p] = uu * muu / mfu;
    s[WF_CQU][p] = 1.0f / (1.0f + 0.5f * (qp + qw));
  }
  if (dv) {
    s[WF_RV][p] = vv * muv * mvxi;
    s[WF_CQV][p] = 1.0f / (1.0f + 0.5f * (qp + qs));
  }
  if (dm) {
    s[WF_ALT][p] = alv + albv;
    s[WF_PHP][p] = 0.5f * (phb0 + phb1 + ph0 + ph1);
    if (k >= 1) s[WF_CQW][p] = 0.5f * (qp + qb);
  }
  if (dr) s[WF_RW][p] = wv * mutv / mft;
}

// calc_ww_cp: a block owns 16 adjacent mass columns of one row and 16 level
// groups; the per-level divergences are formed in parallel into shared
// memory, then one thread per column forms the column sum and the upward scan
// in the reference's order, and the levels are stored in parallel again.
constexpr int kWwTX = 16, kWwKT = 16, kWwQ = (kMaxNz + kWwKT - 1) / kWwKT;

__global__ void __launch_bounds__(kWwTX * kWwKT) k_ww_cp(Grid g, S s) {
  __shared__ float sdv[kMaxNz][kWwTX], sww[kMaxNz][kWwTX];
  const int tx = threadIdx.x % kWwTX, tk = threadIdx.x / kWwTX;
  const int i = g.ids + blockIdx.x * kWwTX + tx, j = g.jds + blockIdx.y;
  const bool col = i < g.ide - 1;
  const int ktf = g.nz - 1;
  const int c = col ? g.i2(j, i) : g.i2(j, g.ids), ce = c + 1, cn = c + g.nx;
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  const float* dnw = s[WF_DNW];
  const float* c1h = s[WF_C1H];
  const size_t lev = (size_t)g.ny * g.nx;
  if (col) {
    const float muu0 = s[WF_MUU][c], muu1 = s[WF_MUU][ce], mfu0 = s[WF_MSFUY][c], mfu1 = s[WF_MSFUY][ce];
    const float muv0 = s[WF_MUV][c], muv1 = s[WF_MUV][cn], mfv0 = s[WF_MSFVX_INV][c], mfv1 = s[WF_MSFVX_INV][cn];
    const float msftx = s[WF_MSFTX][c];
    const float rdx = g.rdx, rdy = g.rdy;
    float ue[kWwQ], u0[kWwQ], vn[kWwQ], v0[kWwQ];
#pragma unroll
    for (int q = 0; q < kWwQ; ++q) {
      const int k = tk + q * kWwKT;
      if (k >= ktf) continue;
      const size_t p = k * lev + c;
      ue[q] = __ldg(&u[p + 1]);
      u0[q] = __ldg(&u[p]);
      vn[q] = __ldg(&v[p + g.nx]);
      v0[q] = __ldg(&v[p]);
    }
#pragma unroll
    for (int q = 0; q < kWwQ; ++q) {
      const int k = tk + q * kWwKT;
      if (k >= ktf) continue;
      const float fu1 = muu1 * ue[q] / mfu1, fu0 = muu0 * u0[q] / mfu0;
      const float fv1 = muv1 * vn[q] * mfv1, fv0 = muv0 * v0[q] * mfv0;
      sdv[k][tx] = (msftx * dnw[k]) * (rdx * (fu1 - fu0) + rdy * (fv1 - fv0));
    }
  }
  __syncthreads();
  float* ww = s[WF_WW];
  if (col && tk == 0) {
    float dmdt = 0.f;
    for (int k = 0; k < ktf; ++k) dmdt = dmdt + sdv[k][tx];
    float wk = ww[c];
    for (int k = 0; k < ktf - 1; ++k) {
      wk = wk - (dnw[k] * c1h[k]) * dmdt - sdv[k][tx];
      sww[k + 1][tx] = wk;
    }
  }
  __syncthreads();
  if (col)
    for (int k = 1 + tk; k < ktf; k += kWwKT) ww[k * lev + c] = sww[k][tx];
}

// calc_ww_cp with one thread per mass column (32 x 4 columns per block): the
// column's divergences stay in registers (the level loop is unrolled to the
// 64-level limit and predicated), the column sum and the upward scan run in
// the reference's order; neighbouring threads' columns make every level's
// loads and stores coalesced.  Same operations as k_ww_cp (the divisions by
// the map factors in their correctly rounded reciprocal form).
__global__ void __launch_bounds__(128) k_ww_cp_col(Grid g, S s) {
  const int i = g.ids + blockIdx.x * 32 + threadIdx.x, j = g.jds + blockIdx.y * 4 + threadIdx.y;
  if (i >= g.ide - 1 || j >= g.jde - 1) return;
  const int ktf = g.nz - 1;
  const int c = g.i2(j, i), ce = c + 1, cn = c + g.nx;
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  const float* dnw = s[WF_DNW];
  const float* c1h = s[WF_C1H];
  const size_t lev = (size_t)g.ny * g.nx;
  const float muu0 = s[WF_MUU][c], muu1 = s[WF_MUU][ce], mfu0 = s[WF_MSFUY][c], mfu1 = s[WF_MSFUY][ce];
  const float muv0 = s[WF_MUV][c], muv1 = s[WF_MUV][cn], mfv0 = s[WF_MSFVX_INV][c], mfv1 = s[WF_MSFVX_INV][cn];
  const float r_mfu0 = __frcp_rn(mfu0), r_mfu1 = __frcp_rn(mfu1);
  const float msftx = s[WF_MSFTX][c];
  const float rdx = g.rdx, rdy = g.rdy;
  float sdv[kMaxNz];
  float dmdt = 0.f;
#pragma unroll
  for (int k = 0; k < kMaxNz; ++k) {
    if (k < ktf) {
      const size_t p = k * lev + c;
      const float fu1 = divc(muu1 * __ldg(&u[p + 1]), mfu1, r_mfu1), fu0 = divc(muu0 * __ldg(&u[p]), mfu0, r_mfu0);
      const float fv1 = muv1 * __ldg(&v[p + g.nx]) * mfv1, fv0 = muv0 * __ldg(&v[p]) * mfv0;
      sdv[k] = (msftx * __ldg(&dnw[k])) * (rdx * (fu1 - fu0) + rdy * (fv1 - fv0));
      dmdt = dmdt + sdv[k];
    }
  }
  float* ww = s[WF_WW];
  float wk = ww[c];
#pragma unroll
  for (int k = 0; k < kMaxNz - 1; ++k) {
    if (k < ktf - 1) {
      wk = wk - (__ldg(&dnw[k]) * __ldg(&c1h[k])) * dmdt - sdv[k];
      ww[(k + 1) * lev + c] = wk;
    }
  }
}

__global__ void k_diff_metrics(Grid g, S s) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, nz = g.nz, ktf = nz - 1;
  const int p = g.i3(k, j, i);
  const size_t lev = (size_t)g.ny * g.nx;
  const float* ph = s[WF_PH];
  const float* phb = s[WF_PHB];
  const float gf = (float)G;
  if (k < ktf && j >= jds - 1 && j < jde && i >= ids && i < ide - 1) {
    const float z0 = (ph[p] + phb[p]) / gf, z1 = (ph[p + lev] + phb[p + lev]) / gf;
    s[WF_RDZW][p] = 1.0f / (z1 - z0);
  }
  const float rdx = g.rdx, rdy = g.rdy;
  if (j >= jds && j < jde - 1 && i >= ids + 1 && i < ide - 1)
    s[WF_ZX][p] = rdx * (phb[p] - phb[p - 1]) / gf + rdx * (ph[p] - ph[p - 1]) / gf;
  if (j >= jds + 1 && j < jde - 1 && i >= ids && i < ide - 1)
    s[WF_ZY][p] = rdy * (phb[p] - phb[p - g.nx]) / gf + rdy * (ph[p] - ph[p - g.nx]) / gf;
  if (k < ktf && j >= jds && j < jde - 1 && (i == ide - 1 || i == ids - 1)) s[WF_ZX][p] = 0.f;
  if (k < ktf && (j == jde - 1 || j == jds - 1) && i >= ids && i < ide - 1) s[WF_ZY][p] = 0.f;
}

// vertical average of a horizontally-averaged quantity h(k) = (a(k) + b(k))
// at w level kk (wrf_dynamics.py:579-592): the same form is used by every
// deformation component.
struct HatPair {
  const float* f;    // velocity component
  const float* m0;   // map factor under a
  const float* m1;   // map factor under b
  int pa, pb;        // column offsets of the two neighbours
};

__device__ __forceinline__ float hat(const HatPair& h, int k, size_t lev, bool second) {
  const int pc = second ? h.pb : h.pa;
  const float m = second ? h.m1[pc] : h.m0[pc];
  return h.f[k * lev + pc] / m;
}

__device__ __forceinline__ float hatavg(const Grid& g, const S& s, const HatPair& h, int kk, size_t lev, float cft1, float cft2) {
  const int ktf = g.nz - 1;
  if (kk >= 1 && kk < ktf) {
    const float fnm = s[WF_FNM][kk], fnp = s[WF_FNP][kk];
    return 0.5f * (fnm * (hat(h, kk, lev, false) + hat(h, kk, lev, true)) +
                   fnp * (hat(h, kk - 1, lev, false) + hat(h, kk - 1, lev, true)));
  }
  if (kk == 0) {
    const float cf1 = g.cf1, cf2 = g.cf2, cf3 = g.cf3;
    return 0.5f * (cf1 * hat(h, 0, lev, false) + cf2 * hat(h, 1, lev, false) + cf3 * hat(h, 2, lev, false) +
                   cf1 * hat(h, 0, lev, true) + cf2 * hat(h, 1, lev, true) + cf3 * hat(h, 2, lev, true));
  }
  const int k1 = g.nz - 2, k2 = g.nz - 3;
  return 0.5f * (cft1 * (hat(h, k1, lev, false) + hat(h, k1, lev, true)) +
                 cft2 * (hat(h, k2, lev, false) + hat(h, k2, lev, true)));
}

__global__ void k_deform(Grid g, S s) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, ktf = g.nz - 1;
  if (k >= ktf) return;
  const size_t lev = (size_t)g.ny * g.nx;
  const int c = g.i2(j, i);
  const int p = k * lev + c;
  const float* dnw = s[WF_DNW];
  const float* dn = s[WF_DN];
  const int kt1 = g.nz - 2;
  const float cft2 = -0.5f * dnw[kt1] / dn[kt1];
  const float cft1 = 1.0f - cft2;
  const float* zx = s[WF_ZX];
  const float* zy = s[WF_ZY];
  const float* rdzw = s[WF_RDZW];
  const int nx = g.nx;
  // the three components are formed before any is stored
  float o11 = 0.f, o22 = 0.f, o12 = 0.f;
  const bool d1 = j >= jds && j < jde - 1 && i >= ids && i < ide - 1;
  const bool d2 = j >= jds + 1 && j < jde - 1 && i >= ids + 1 && i < ide - 1;
  if (d1) {
    const float mm = s[WF_MSFTX][c] * s[WF_MSFTY][c];
    HatPair hu{s[WF_U], s[WF_MSFUY], s[WF_MSFUY], c, c + 1};
    const float d = hatavg(g, s, hu, k + 1, lev, cft1, cft2) - hatavg(g, s, hu, k, lev, cft1, cft2);
    const float zsum = zx[p] + zx[p + 1] + zx[p + lev] + zx[p + lev + 1];
    float t1 = d * (0.25f * zsum * rdzw[p]);
    t1 = mm * (g.rdx * (hat(hu, k, lev, true) - hat(hu, k, lev, false)) - t1);
    o11 = 2.0f * t1;
    HatPair hv{s[WF_V], s[WF_MSFVX], s[WF_MSFVX], c, c + nx};
    const float dv = hatavg(g, s, hv, k + 1, lev, cft1, cft2) - hatavg(g, s, hv, k, lev, cft1, cft2);
    const float zys = zy[p] + zy[p + nx] + zy[p + lev] + zy[p + lev + nx];
    t1 = mm * (g.rdy * (hat(hv, k, lev, true) - hat(hv, k, lev, false)) - dv * (0.25f * zys * rdzw[p]));
    o22 = 2.0f * t1;
  }
  if (d2) {
    const float* msfux = s[WF_MSFUX];
    const float* msfvy = s[WF_MSFVY];
    const float mm = 0.25f * (msfux[c - nx] + msfux[c]) * (msfvy[c - 1] + msfvy[c]);
    HatPair hu{s[WF_U], msfux, msfux, c - nx, c};
    float d = hatavg(g, s, hu, k + 1, lev, cft1, cft2) - hatavg(g, s, hu, k, lev, cft1, cft2);
    float rsum = rdzw[p] + rdzw[p - 1] + rdzw[p - nx - 1] + rdzw[p - nx];
    float t1 = d * (0.25f * (zy[p - 1] + zy[p] + zy[p + lev - 1] + zy[p + lev]) * 0.25f * rsum);
    const float d12 = mm * (g.rdy * (hat(hu, k, lev, true) - hat(hu, k, lev, false)) - t1);
    HatPair hv{s[WF_V], msfvy, msfvy, c - 1, c};
    d = hatavg(g, s, hv, k + 1, lev, cft1, cft2) - hatavg(g, s, hv, k, lev, cft1, cft2);
    rsum = rdzw[p] + rdzw[p - nx] + rdzw[p - nx - 1] + rdzw[p - 1];
    t1 = d * (0.25f * (zx[p - nx] + zx[p] + zx[p + lev - nx] + zx[p + lev]) * 0.25f * rsum);
    o12 = d12 + mm * (g.rdx * (hat(hv, k, lev, true) - hat(hv, k, lev, false)) - t1);
  }
  if (d1) {
    s[WF_DEFOR11][p] = o11;
    s[WF_DEFOR22][p] = o22;
  }
  if (d2) s[WF_DEFOR12][p] = o12;
}

__global__ void k_defor12_bc(Grid g, S s) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  float* d = s[WF_DEFOR12];
  const size_t lev = (size_t)g.ny * g.nx;
  const size_t base = k * lev;
  auto at = [&](int jj, int ii) { return d[base + (size_t)jj * g.nx + ii]; };
  // final value after the x copies then the y copies
  auto after_x = [&](int jj, int ii) {
    if (ii == ids) return at(jj, ids + 1);
    if (ii == ide - 1) return at(jj, ide - 2);
    return at(jj, ii);
  };
  float val;
  if ((j == jds || j == jde - 1) && i >= ids && i < ide) {
    val = after_x(j == jds ? jds + 1 : jde - 2, i);
  } else if ((i == ids || i == ide - 1) && j > jds && j < jde - 1) {
    val = at(j, i == ids ? ids + 1 : ide - 2);
  } else {
    return;
  }
  // sources are interior points, which this kernel never writes
  d[base + (size_t)j * g.nx + i] = val;
}

__global__ void k_km(Grid g, S s) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ktf = g.nz - 1;
  const int p = g.i3(k, j, i), c = g.i2(j, i);
  const bool reg = j >= g.jds + 1 && j < g.jde - 2 && i >= g.ids + 1 && i < g.ide - 2;
  float* xkmh = s[WF_XKMH];
  float cap = 0.f;
  if (reg) cap = 10.0f * sqrtf(g.dx / s[WF_MSFTX][c] * g.dy / s[WF_MSFTY][c]);
  if (reg && k < ktf) {
    const float* d11 = s[WF_DEFOR11];
    const float* d22 = s[WF_DEFOR22];
    const float* d12 = s[WF_DEFOR12];
    const int nx = g.nx;
    const float dd = d11[p] - d22[p];
    float def2 = 0.25f * (dd * dd);
    const float t = 0.25f * (d12[p] + d12[p + nx] + d12[p + 1] + d12[p + nx + 1]);
    def2 = def2 + t * t;
    const float mlen = sqrtf(g.dx / s[WF_MSFTX][c] * g.dy / s[WF_MSFTY][c]);
    const float v = (float)(C_S * C_S) * mlen * mlen * sqrtf(def2);
    const float km = v < 10.0f * mlen ? v : 10.0f * mlen;
    xkmh[p] = km;
    s[WF_XKHH][p] = km / (float)PRANDTL;
  } else {
    const float old = xkmh[p];
    xkmh[p] = old < cap ? old : cap;
  }
}

__global__ void k_hdiff(Grid g, S s) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, ktf = g.nz - 1;
  if (k >= ktf) return;
  const size_t lev = (size_t)g.ny * g.nx;
  const int c = g.i2(j, i), p = k * lev + c, nx = g.nx;
  const float* mut = s[WF_MUT];
  const float* msfux = s[WF_MSFUX];
  const float* msfuy = s[WF_MSFUY];
  const float* msfvx = s[WF_MSFVX];
  const float* msfvy = s[WF_MSFVY];
  const float* msftx = s[WF_MSFTX];
  const float* msfty = s[WF_MSFTY];
  const float* msfvx_inv = s[WF_MSFVX_INV];
  const float* K = s[WF_XKMH];
  const float rdx = g.rdx, rdy = g.rdy;
  // the four updated tendencies are stored at the end, so that no store
  // separates the parts' loads (they share mut, K and the map factors)
  float o_u = 0.f, o_v = 0.f, o_w = 0.f, o_t = 0.f;
  auto apply = [&](const float* tend, const float* f, const float* base, float mkrdxm, float mkrdxp, float mrdx,
                   float mkrdym, float mkrdyp, float mrdy) -> float {
    float dxp, dxm, dyp, dym;
    const float fc = f[p];
    if (!base) {
      dxp = f[p + 1] - fc; dxm = fc - f[p - 1]; dyp = f[p + nx] - fc; dym = fc - f[p - nx];
    } else {
      const float b = base[p];
      dxp = f[p + 1] - fc - base[p + 1] + b;
      dxm = fc - f[p - 1] - b + base[p - 1];
      dyp = f[p + nx] - fc - base[p + nx] + b;
      dym = fc - f[p - nx] - b + base[p - nx];
    }
    return tend[p] + (mrdx * (mkrdxp * dxp - mkrdxm * dxm) + mrdy * (mkrdyp * dyp - mkrdym * dym));
  };
  const bool du = j >= jds + 1 && j < jde - 2 && i >= ids + 1 && i < ide - 1;
  const bool dv = j >= jds + 1 && j < jde - 1 && i >= ids + 1 && i < ide - 2;
  const bool dw = k >= 1 && j >= jds + 1 && j < jde - 2 && i >= ids + 1 && i < ide - 2;
  const bool dt = j >= jds + 1 && j < jde - 2 && i >= ids + 1 && i < ide - 2;
  if (du) {  // u
    const float mkrdxm = (msftx[c - 1] / msfty[c - 1]) * mut[c - 1] * K[p - 1] * rdx;
    const float mkrdxp = (msftx[c] / msfty[c]) * mut[c] * K[p] * rdx;
    const float mrdx = msfux[c] * msfuy[c] * rdx;
    const float mkrdym = ((msfuy[c] + msfuy[c - nx]) / (msfux[c] + msfux[c - nx])) * 0.25f *
                         (mut[c] + mut[c - nx] + mut[c - nx - 1] + mut[c - 1]) * 0.25f *
                         (K[p] + K[p - nx] + K[p - nx - 1] + K[p - 1]) * rdy;
    const float mkrdyp = ((msfuy[c] + msfuy[c + nx]) / (msfux[c] + msfux[c + nx])) * 0.25f *
                         (mut[c] + mut[c + nx] + mut[c + nx - 1] + mut[c - 1]) * 0.25f *
                         (K[p] + K[p + nx] + K[p + nx - 1] + K[p - 1]) * rdy;
    const float mrdy = msfux[c] * msfuy[c] * rdy;
    o_u = apply(s[WF_RU_TENDF], s[WF_U], nullptr, mkrdxm, mkrdxp, mrdx, mkrdym, mkrdyp, mrdy);
  }
  if (dv) {  // v
    const float mkrdxm = ((msfvx[c] + msfvx[c - 1]) / (msfvy[c] + msfvy[c - 1])) * 0.25f *
                         (mut[c] + mut[c - nx] + mut[c - nx - 1] + mut[c - 1]) * 0.25f *
                         (K[p] + K[p - nx] + K[p - nx - 1] + K[p - 1]) * rdx;
    const float mkrdxp = ((msfvx[c] + msfvx[c + 1]) / (msfvy[c] + msfvy[c + 1])) * 0.25f *
                         (mut[c] + mut[c - nx] + mut[c - nx + 1] + mut[c + 1]) * 0.25f *
                         (K[p] + K[p - nx] + K[p - nx + 1] + K[p + 1]) * rdx;
    const float mrdx = msfvx[c] * msfvy[c] * rdx;
    const float mkrdym = (msfty[c - nx] / msftx[c - nx]) * K[p - nx] * rdy;
    const float mkrdyp = (msfty[c] / msftx[c]) * K[p] * rdy;
    const float mrdy = msfvx[c] * msfvy[c] * rdy;
    o_v = apply(s[WF_RV_TENDF], s[WF_V], nullptr, mkrdxm, mkrdxp, mrdx, mkrdym, mkrdyp, mrdy);
  }
  if (dw) {  // w
    const float mkrdxm = (msfux[c] / msfuy[c]) * 0.25f * (mut[c] + mut[c - 1] + mut[c] + mut[c - 1]) * 0.25f *
                         (K[p] + K[p - 1] + K[p - lev] + K[p - lev - 1]) * rdx;
    const float mkrdxp = (msfux[c + 1] / msfuy[c + 1]) * 0.25f * (mut[c + 1] + mut[c] + mut[c + 1] + mut[c]) * 0.25f *
                         (K[p + 1] + K[p] + K[p - lev + 1] + K[p - lev]) * rdx;
    const float mrdx = msftx[c] * msfty[c] * rdx;
    const float mkrdym = (msfvy[c] / msfvx[c]) * 0.25f * (mut[c] + mut[c - nx] + mut[c] + mut[c - nx]) * 0.25f *
                         (K[p] + K[p - nx] + K[p - lev] + K[p - lev - nx]) * rdy;
    const float mkrdyp = (msfvy[c + nx] / msfvx[c + nx]) * 0.25f * (mut[c + nx] + mut[c] + mut[c + nx] + mut[c]) *
                         0.25f * (K[p + nx] + K[p] + K[p - lev + nx] + K[p - lev]) * rdy;
    const float mrdy = msftx[c] * msfty[c] * rdy;
    o_w = apply(s[WF_RW_TENDF], s[WF_W], nullptr, mkrdxm, mkrdxp, mrdx, mkrdym, mkrdyp, mrdy);
  }
  if (dt) {  // theta (xkhh, minus t_init)
    const float* Kh = s[WF_XKHH];
    const float mkrdxm = (msfux[c] / msfuy[c]) * 0.5f * (Kh[p] + Kh[p - 1]) * 0.5f * (mut[c] + mut[c - 1]) * rdx;
    const float mkrdxp = (msfux[c + 1] / msfuy[c + 1]) * 0.5f * (Kh[p + 1] + Kh[p]) * 0.5f * (mut[c + 1] + mut[c]) * rdx;
    const float mrdx = msftx[c] * msfty[c] * rdx;
    const float mkrdym = (msfvy[c] * msfvx_inv[c]) * 0.5f * (Kh[p] + Kh[p - nx]) * 0.5f * (mut[c] + mut[c - nx]) * rdy;
    const float mkrdyp = (msfvy[c + nx] * msfvx_inv[c + nx]) * 0.5f * (Kh[p + nx] + Kh[p]) * 0.5f *
                         (mut[c + nx] + mut[c]) * rdy;
    const float mrdy = msftx[c] * msfty[c] * rdy;
    o_t = apply(s[WF_T_TENDF], s[WF_T], s[WF_T_INIT], mkrdxm, mkrdxp, mrdx, mkrdym, mkrdyp, mrdy);
  }
  if (du) s[WF_RU_TENDF][p] = o_u;
  if (dv) s[WF_RV_TENDF][p] = o_v;
  if (dw) s[WF_RW_TENDF][p] = o_w;
  if (dt) s[WF_T_TENDF][p] = o_t;
}

// relaxation of u, v, ph (mass-weighted), theta (mass-weighted) and mu at
// the first RK stage (pywrf/solver.py:1143-1203)
// (k, j, i) of this thread, in ring mode or over every point; false when none
__device__ __forceinline__ bool relax_index(const Grid& g, int ring, int& k, int& j, int& i) {
  k = blockIdx.z;
  if (ring) return ring_point(g, blockIdx.x * blockDim.x + threadIdx.x, j, i);
  i = blockIdx.x * blockDim.x + threadIdx.x;
  j = blockIdx.y * blockDim.y + threadIdx.y;
  return i < g.nx && j < g.ny;
}

__global__ void k_relax(Grid g, S s, int ring) {
  int k, j, i;
  if (!relax_index(g, ring, k, j, i)) return;
  const float dtbc = s[WF_DSCAL][DS_DTBC];
  const int nz = g.nz;
  const size_t lev = (size_t)g.ny * g.nx;
  const int p = g.i3(k, j, i);
  const float* ru = s[WF_RU];
  const float* rv = s[WF_RV];
  const float* ph = s[WF_PH];
  const float* t = s[WF_T];
  const float* mut = s[WF_MUT];
  const int nx = g.nx;
  auto idx = [&](int kk, int jj, int ii) { return (size_t)(kk * g.ny + jj) * nx + ii; };
  if (k < nz - 1) {
    float* o = s[WF_U_SAVE] + p;
    relax_point(g, s, WF_U_BXS, k, j, i, g.ide, g.jde - 1, nz, [&](int kk, int jj, int ii) { return ru[idx(kk, jj, ii)]; }, dtbc, o);
    o = s[WF_V_SAVE] + p;
    relax_point(g, s, WF_V_BXS, k, j, i, g.ide - 1, g.jde, nz, [&](int kk, int jj, int ii) { return rv[idx(kk, jj, ii)]; }, dtbc, o);
    o = s[WF_T_SAVE] + p;
    relax_point(g, s, WF_T_BXS, k, j, i, g.ide - 1, g.jde - 1, nz,
                [&](int kk, int jj, int ii) { return t[idx(kk, jj, ii)] * mut[(size_t)jj * nx + ii]; }, dtbc, o);
  }
  {
    float* o = s[WF_PH_SAVE] + p;
    relax_point(g, s, WF_PH_BXS, k, j, i, g.ide - 1, g.jde - 1, nz,
                [&](int kk, int jj, int ii) { return ph[idx(kk, jj, ii)] * mut[(size_t)jj * nx + ii]; }, dtbc, o);
  }
  if (k == 0) {
    const float* mu = s[WF_MU];
    float* o = s[WF_MU_TEND] + g.i2(j, i);
    relax_point(g, s, WF_MU_BXS, 0, j, i, g.ide - 1, g.jde - 1, 1,
                [&](int kk, int jj, int ii) { (void)kk; return mu[(size_t)jj * nx + ii]; }, dtbc, o);
  }
  (void)lev;
}

// relaxation + specified tendency of qv at the first stage (relax_bdy_scalar,
// spec_bdy_scalar: wrf_boundary.py:413-467, 189-241); rq = qv * mut
__global__ void k_relax_qv(Grid g, S s, int ring) {
  int k, j, i;
  if (!relax_index(g, ring, k, j, i)) return;
  if (k >= g.nz - 1) return;
  const float dtbc = s[WF_DSCAL][DS_DTBC];
  const size_t n3 = g.n3();
  const float* qv = s[WF_MOIST] + n3;
  float* tend = s[WF_MOIST_TEND] + n3;
  const float* mut = s[WF_MUT];
  const int nx = g.nx;
  const int p = g.i3(k, j, i);
  const int ibs = g.ids, jbs = g.jds, ibe = g.ide - 1, jbe = g.jde - 1;
  auto rq = [&](int kk, int jj, int ii) {
    if (jj < g.jds || jj >= g.jde - 1 || ii < g.ids || ii >= g.ide - 1) return 0.f;
    return qv[(size_t)(kk * g.ny + jj) * nx + ii] * mut[(size_t)jj * nx + ii];
  };
  relax_point(g, s, WF_QV_BXS, k, j, i, ibe, jbe, g.nz, rq, dtbc, tend + p);
  // specified row: the boundary tendency replaces the tendency (applied after
  // the relaxation, on disjoint points)
  const float* txs = s[WF_QV_BTXS];
  const float* txe = s[WF_QV_BTXE];
  const float* tys = s[WF_QV_BTYS];
  const float* tye = s[WF_QV_BTYE];
  float val;
  bool hit = false;
  if (i >= ibs && i < ibe && (j == jbs || j == jbe - 1)) {
    // y rows are written first, then the x columns overwrite their corners
    val = (j == jbs) ? tys[((size_t)k * 5 + 0) * nx + i] : tye[((size_t)k * 5 + 0) * nx + i];
    hit = true;
  }
  if (j >= jbs && j < jbe && (i == ibs || i == ibe - 1)) {
    val = (i == ibs) ? txs[((size_t)k * g.ny + j) * 5] : txe[((size_t)k * g.ny + j) * 5];
    hit = true;
  }
  if (hit) tend[p] = val;
}

int launch_prep(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  k_rk_prep2d<<<col_grid(g, b2), b2, 0, st>>>(g, s);
  k_rk_prep3d<<<point_grid(g, b3), b3, 0, st>>>(g, s);
  if (kernel_form() == WRF_FORM_FAST) {
    const dim3 bc(32, 4);
    k_ww_cp_col<<<dim3((g.ide - 1 - g.ids + 31) / 32, (g.jde - 1 - g.jds + 3) / 4), bc, 0, st>>>(g, s);
  } else {
    k_ww_cp<<<dim3((g.ide - 1 - g.ids + kWwTX - 1) / kWwTX, g.jde - 1 - g.jds), kWwTX * kWwKT, 0, st>>>(g, s);
  }
  return 3;
}

int launch_deform(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_deform<<<point_grid(g, b3), b3, 0, st>>>(g, s);
  k_defor12_bc<<<point_grid(g, b3), b3, 0, st>>>(g, s);
  return 2;
}

int launch_km(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b3(32, 4);
  const int n = launch_deform(g, s, st);
  k_km<<<point_grid(g, b3), b3, 0, st>>>(g, s);
  return n + 1;
}

int launch_diff_metrics(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_diff_metrics<<<point_grid(g, b3), b3, 0, st>>>(g, s);
  return 1;
}

int launch_hdiff_relax(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_hdiff<<<point_grid(g, b3), b3, 0, st>>>(g, s);
  if (kernel_form() == WRF_FORM_FAST && ring_fits(g))
    k_relax<<<dim3((ring_size(g) + 127) / 128, 1, g.nz), 128, 0, st>>>(g, s, 1);
  else
    k_relax<<<point_grid(g, b3), b3, 0, st>>>(g, s, 0);
  return 2;
}

int launch_relax_qv(const Grid& g, const S& s, cudaStream_t st) {
  const dim3 b3(32, 4);
  if (kernel_form() == WRF_FORM_FAST && ring_fits(g))
    k_relax_qv<<<dim3((ring_size(g) + 127) / 128, 1, g.nz), 128, 0, st>>>(g, s, 1);
  else
    k_relax_qv<<<point_grid(g, b3), b3, 0, st>>>(g, s, 0);
  return 1;
}

}  // namespace wrf
