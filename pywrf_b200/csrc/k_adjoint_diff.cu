// The first RK stage's operators that the step fuses into its diffusion
// kernels, as stand-alone operators with their adjoints:
//   horizontal_diffusion of u, v, w, of theta about t_init
//     (horizontal_diffusion_3dmp) and of a moisture species
//     (wrf_dynamics.py:2623-2915): tend += mrdx (kxp dxp - kxm dxm)
//     + mrdy (kyp dyp - kym dym), where each k.. = (map-factor ratio) x
//     (average of the column mass over a few points) x (average of the eddy
//     viscosity over a few points) x rd, and d.. are the field's differences
//     to its neighbours.  Bilinear in the field and the viscosity and linear
//     in the column mass; the reverse runs one thread per output point and
//     adds its partial products into the cotangents of the field, the mass
//     and the viscosity (atomically: each is read by several output points).
//   the eddy viscosities: compute_diff_metrics (wrf_dynamics.py:491-536),
//     cal_deform_and_div's defor11/22/12 (:539-813) and the 2-D Smagorinsky
//     calculate_km_kh (:958-995).  The reverse recomputes the metrics and
//     the deformations into caller scratch, then runs km, deformation and
//     metric reverses in turn (scatter form with atomics).
//   mass_weight (wrf_boundary.py:403-410), the product the relaxation of
//     ph, theta and qv reads.
#include "kernels.cuh"

namespace wrf {

namespace {

__device__ __forceinline__ void acc(float* a, size_t q, float v) {
  if (v != 0.f) atomicAdd(a + q, v);
}

// one of the four coefficients: value = ratio * mavg * kavg * rd with the
// averages over nm mut points (dj, di) and nk viscosity points (dk, dj, di),
// each weighted by wm / wk
struct Coef {
  float ratio, rd, wm, wk;
  int nm, nk;
  bool kfirst;  // the viscosity average multiplies before the mass average
  int mj[4], mi[4], kk[4], kj[4], ki[4];
};

enum { DV_U = 0, DV_V = 1, DV_W = 2, DV_M = 3 };

// the four coefficients (x minus, x plus, y minus, y plus) of variable var at
// column c, in the reference's formulas
__device__ void diff_coefs(const Grid& g, const S& s, int var, int c, Coef (&cf)[4]) {
  const int nx = g.nx;
  const float* msftx = s[WF_MSFTX];
  const float* msfty = s[WF_MSFTY];
  const float* msfux = s[WF_MSFUX];
  const float* msfuy = s[WF_MSFUY];
  const float* msfvx = s[WF_MSFVX];
  const float* msfvy = s[WF_MSFVY];
  const float* msfvi = s[WF_MSFVX_INV];
  auto set = [](Coef& a, float ratio, float rd, float wm, float wk, int nm, int nk) {
    a.ratio = ratio; a.rd = rd; a.wm = wm; a.wk = wk; a.nm = nm; a.nk = nk; a.kfirst = false;
  };
  auto mp = [](Coef& a, int e, int dj, int di) { a.mj[e] = dj; a.mi[e] = di; };
  auto kp = [](Coef& a, int e, int dk, int dj, int di) { a.kk[e] = dk; a.kj[e] = dj; a.ki[e] = di; };
  const float rdx = g.rdx, rdy = g.rdy;
  if (var == DV_U) {
    set(cf[0], msftx[c - 1] / msfty[c - 1], rdx, 1.f, 1.f, 1, 1); mp(cf[0], 0, 0, -1); kp(cf[0], 0, 0, 0, -1);
    set(cf[1], msftx[c] / msfty[c], rdx, 1.f, 1.f, 1, 1); mp(cf[1], 0, 0, 0); kp(cf[1], 0, 0, 0, 0);
    for (int e = 0; e < 2; ++e) {
      const int d = e == 0 ? -1 : 1;
      set(cf[2 + e], (msfuy[c] + msfuy[c + d * nx]) / (msfux[c] + msfux[c + d * nx]), rdy, 0.25f, 0.25f, 4, 4);
      mp(cf[2 + e], 0, 0, 0); mp(cf[2 + e], 1, d, 0); mp(cf[2 + e], 2, d, -1); mp(cf[2 + e], 3, 0, -1);
      kp(cf[2 + e], 0, 0, 0, 0); kp(cf[2 + e], 1, 0, d, 0); kp(cf[2 + e], 2, 0, d, -1); kp(cf[2 + e], 3, 0, 0, -1);
    }
  } else if (var == DV_V) {
    for (int e = 0; e < 2; ++e) {
      const int d = e == 0 ? -1 : 1;
      set(cf[e], (msfvx[c] + msfvx[c + d]) / (msfvy[c] + msfvy[c + d]), rdx, 0.25f, 0.25f, 4, 4);
      mp(cf[e], 0, 0, 0); mp(cf[e], 1, -1, 0); mp(cf[e], 2, -1, d); mp(cf[e], 3, 0, d);
      kp(cf[e], 0, 0, 0, 0); kp(cf[e], 1, 0, -1, 0); kp(cf[e], 2, 0, -1, d); kp(cf[e], 3, 0, 0, d);
    }
    set(cf[2], msfty[c - nx] / msftx[c - nx], rdy, 0.f, 1.f, 0, 1); kp(cf[2], 0, 0, -1, 0);
    set(cf[3], msfty[c] / msftx[c], rdy, 0.f, 1.f, 0, 1); kp(cf[3], 0, 0, 0, 0);
  } else if (var == DV_W) {
    // 0.25 (m(a) + m(b) + m(a) + m(b)): the pair is listed twice, as the
    // reference sums it
    set(cf[0], msfux[c] / msfuy[c], rdx, 0.25f, 0.25f, 4, 4);
    mp(cf[0], 0, 0, 0); mp(cf[0], 1, 0, -1); mp(cf[0], 2, 0, 0); mp(cf[0], 3, 0, -1);
    kp(cf[0], 0, 0, 0, 0); kp(cf[0], 1, 0, 0, -1); kp(cf[0], 2, -1, 0, 0); kp(cf[0], 3, -1, 0, -1);
    set(cf[1], msfux[c + 1] / msfuy[c + 1], rdx, 0.25f, 0.25f, 4, 4);
    mp(cf[1], 0, 0, 1); mp(cf[1], 1, 0, 0); mp(cf[1], 2, 0, 1); mp(cf[1], 3, 0, 0);
    kp(cf[1], 0, 0, 0, 1); kp(cf[1], 1, 0, 0, 0); kp(cf[1], 2, -1, 0, 1); kp(cf[1], 3, -1, 0, 0);
    set(cf[2], msfvy[c] / msfvx[c], rdy, 0.25f, 0.25f, 4, 4);
    mp(cf[2], 0, 0, 0); mp(cf[2], 1, -1, 0); mp(cf[2], 2, 0, 0); mp(cf[2], 3, -1, 0);
    kp(cf[2], 0, 0, 0, 0); kp(cf[2], 1, 0, -1, 0); kp(cf[2], 2, -1, 0, 0); kp(cf[2], 3, -1, -1, 0);
    set(cf[3], msfvy[c + nx] / msfvx[c + nx], rdy, 0.25f, 0.25f, 4, 4);
    mp(cf[3], 0, 1, 0); mp(cf[3], 1, 0, 0); mp(cf[3], 2, 1, 0); mp(cf[3], 3, 0, 0);
    kp(cf[3], 0, 0, 1, 0); kp(cf[3], 1, 0, 0, 0); kp(cf[3], 2, -1, 1, 0); kp(cf[3], 3, -1, 0, 0);
  } else {
    set(cf[0], msfux[c] / msfuy[c], rdx, 0.5f, 0.5f, 2, 2);
    mp(cf[0], 0, 0, 0); mp(cf[0], 1, 0, -1); kp(cf[0], 0, 0, 0, 0); kp(cf[0], 1, 0, 0, -1);
    set(cf[1], msfux[c + 1] / msfuy[c + 1], rdx, 0.5f, 0.5f, 2, 2);
    mp(cf[1], 0, 0, 1); mp(cf[1], 1, 0, 0); kp(cf[1], 0, 0, 0, 1); kp(cf[1], 1, 0, 0, 0);
    set(cf[2], msfvy[c] * msfvi[c], rdy, 0.5f, 0.5f, 2, 2);
    mp(cf[2], 0, 0, 0); mp(cf[2], 1, -1, 0); kp(cf[2], 0, 0, 0, 0); kp(cf[2], 1, 0, -1, 0);
    set(cf[3], msfvy[c + nx] * msfvi[c + nx], rdy, 0.5f, 0.5f, 2, 2);
    mp(cf[3], 0, 1, 0); mp(cf[3], 1, 0, 0); kp(cf[3], 0, 0, 1, 0); kp(cf[3], 1, 0, 0, 0);
    for (int e = 0; e < 4; ++e) cf[e].kfirst = true;
  }
}

// the variable's region (k0..k1, j0..j1, i0..i1), half-open
__device__ __forceinline__ bool diff_region(const Grid& g, int var, int k, int j, int i) {
  const int ktf = g.nz - 1;
  int i1 = g.ide - 2, j1 = g.jde - 2, k0 = 0;
  if (var == DV_U) i1 = g.ide - 1;
  if (var == DV_V) j1 = g.jde - 1;
  if (var == DV_W) k0 = 1;
  return k >= k0 && k < ktf && j >= g.jds + 1 && j < j1 && i >= g.ids + 1 && i < i1;
}

struct DiffPoint {
  float kx[4];   // the coefficients
  float mavg[4], kavg[4];
  float d[4];    // dxm, dxp, dym, dyp
  float mr[2];   // mrdx, mrdy
};

__device__ void diff_point(const Grid& g, const S& s, int var, const float* f, const float* base, const float* mut,
                           const float* K, int k, int c, size_t p, const Coef (&cf)[4], DiffPoint& o) {
  const int nx = g.nx;
  const size_t lev = (size_t)g.ny * nx;
  for (int e = 0; e < 4; ++e) {
    float ms = 0.f, ks = 0.f;
    for (int q = 0; q < cf[e].nm; ++q) ms = ms + mut[c + cf[e].mj[q] * nx + cf[e].mi[q]];
    for (int q = 0; q < cf[e].nk; ++q) ks = ks + K[p + (long)cf[e].kk[q] * (long)lev + cf[e].kj[q] * nx + cf[e].ki[q]];
    o.mavg[e] = cf[e].nm ? cf[e].wm * ms : 1.f;
    o.kavg[e] = cf[e].wk * ks;
    o.kx[e] = cf[e].kfirst ? cf[e].ratio * o.kavg[e] * o.mavg[e] * cf[e].rd
                           : cf[e].ratio * o.mavg[e] * o.kavg[e] * cf[e].rd;
  }
  const float cc = f[p];
  const float xm = f[p - 1], xp = f[p + 1], ym = f[p - nx], yp = f[p + nx];
  if (base) {
    const float b = base[p];
    o.d[0] = cc - xm - b + base[p - 1];
    o.d[1] = xp - cc - base[p + 1] + b;
    o.d[2] = cc - ym - b + base[p - nx];
    o.d[3] = yp - cc - base[p + nx] + b;
  } else {
    o.d[0] = cc - xm;
    o.d[1] = xp - cc;
    o.d[2] = cc - ym;
    o.d[3] = yp - cc;
  }
  const float* m1 = var == DV_U ? s[WF_MSFUX] : (var == DV_V ? s[WF_MSFVX] : s[WF_MSFTX]);
  const float* m2 = var == DV_U ? s[WF_MSFUY] : (var == DV_V ? s[WF_MSFVY] : s[WF_MSFTY]);
  o.mr[0] = m1[c] * m2[c] * g.rdx;
  o.mr[1] = m1[c] * m2[c] * g.rdy;
}

// a thread takes one column's levels [z0, z0 + kHdiffLevels) of the
// diffusion region: the column's coefficients once, then its levels
constexpr int kHdiffLevels = 8;
__global__ void k_hdiff_op(Grid g, S s, int var, const float* f, const float* base, const float* mut, const float* K,
                           float* tend) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int z0 = blockIdx.z * kHdiffLevels;
  if (i >= g.nx || j >= g.ny || !diff_region(g, var, g.nz - 2, j, i)) return;
  const int c = g.i2(j, i);
  Coef cf[4];
  diff_coefs(g, s, var, c, cf);
  for (int k = z0; k < z0 + kHdiffLevels && k < g.nz; ++k) {
    if (!diff_region(g, var, k, j, i)) continue;
    const size_t p = (size_t)k * g.ny * g.nx + c;
    DiffPoint o;
    diff_point(g, s, var, f, base, mut, K, k, c, p, cf, o);
    tend[p] = tend[p] + (o.mr[0] * (o.kx[1] * o.d[1] - o.kx[0] * o.d[0]) + o.mr[1] * (o.kx[3] * o.d[3] - o.kx[2] * o.d[2]));
  }
}

// its reverse, over the same level ranges: the field's and the viscosity's
// cotangents scattered with atomics, the column mass's summed over the
// thread's levels first
// (the cotangent outputs are distinct from every operand and from each
// other: __restrict__ lets a level's loads run ahead of the previous
// level's atomic adds)
__global__ void k_hdiff_op_adj(Grid g, S s, int var, const float* __restrict__ f, const float* __restrict__ base,
                               const float* __restrict__ mut, const float* __restrict__ K,
                               const float* __restrict__ tbar, float* __restrict__ fbar, float* __restrict__ mutbar,
                               float* __restrict__ Kbar) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int z0 = blockIdx.z * kHdiffLevels;
  if (i >= g.nx || j >= g.ny || !diff_region(g, var, g.nz - 2, j, i)) return;
  const int nx = g.nx;
  const size_t lev = (size_t)g.ny * nx;
  const int c = g.i2(j, i);
  Coef cf[4];
  diff_coefs(g, s, var, c, cf);
  float wm[4] = {0.f, 0.f, 0.f, 0.f};  // the mass averages' cotangents, per edge
  const float sgn[4] = {-1.f, 1.f, -1.f, 1.f};
#pragma unroll 2
  for (int k = z0; k < z0 + kHdiffLevels && k < g.nz; ++k) {
    if (!diff_region(g, var, k, j, i)) continue;
    const size_t p = (size_t)k * lev + c;
    const float T = tbar[p];
    if (T == 0.f) continue;
    DiffPoint o;
    diff_point(g, s, var, f, base, mut, K, k, c, p, cf, o);
    // d/d(differences): +-mr * k..
    const float gx0 = -o.mr[0] * o.kx[0] * T, gx1 = o.mr[0] * o.kx[1] * T;
    const float gy0 = -o.mr[1] * o.kx[2] * T, gy1 = o.mr[1] * o.kx[3] * T;
    // dxm = c - xm, dxp = xp - c, dym = c - ym, dyp = yp - c (base is data)
    if (fbar) {
      acc(fbar, p, gx0 - gx1 + gy0 - gy1);
      acc(fbar, p - 1, -gx0);
      acc(fbar, p + 1, gx1);
      acc(fbar, p - nx, -gy0);
      acc(fbar, p + nx, gy1);
    }
    // d/d k.. then into the averages
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float mr = e < 2 ? o.mr[0] : o.mr[1];
      const float kb = sgn[e] * mr * o.d[e] * T;  // cotangent of k..
      const float base_c = cf[e].ratio * cf[e].rd * kb;
      if (cf[e].nm) wm[e] += base_c * o.kavg[e] * cf[e].wm;
      if (Kbar) {
        const float wkb = base_c * o.mavg[e] * cf[e].wk;
        for (int q = 0; q < cf[e].nk; ++q)
          acc(Kbar, p + (long)cf[e].kk[q] * (long)lev + cf[e].kj[q] * nx + cf[e].ki[q], wkb);
      }
    }
  }
  if (mutbar)
#pragma unroll
    for (int e = 0; e < 4; ++e)
      for (int q = 0; q < cf[e].nm; ++q) acc(mutbar, c + cf[e].mj[q] * nx + cf[e].mi[q], wm[e]);
}

// ---- the eddy viscosities ----

// calculate_km_kh's reverse: in the region the viscosity's cotangent (xkhh =
// xkmh / Prandtl included) goes to defor11/22 at the point and defor12 at
// its four corners; above the region's levels and outside it the forward
// clamped the incoming xkmh to the cap (zero outside), and xkhh kept its
// incoming value
__global__ void k_km_adj(Grid g, S s, S b, float* d11b, float* d22b, float* d12b) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ktf = g.nz - 1, nx = g.nx;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * nx + c;
  const bool reg = j >= g.jds + 1 && j < g.jde - 2 && i >= g.ids + 1 && i < g.ide - 2;
  float cap = 0.f;
  if (reg) cap = 10.0f * sqrtf(g.dx / s[WF_MSFTX][c] * g.dy / s[WF_MSFTY][c]);
  if (reg && k < ktf) {
    const float X = b[WF_XKMH][p] + b[WF_XKHH][p] / (float)PRANDTL;
    b[WF_XKMH][p] = 0.f;
    b[WF_XKHH][p] = 0.f;
    const float* d11 = s[WF_DEFOR11];
    const float* d22 = s[WF_DEFOR22];
    const float* d12 = s[WF_DEFOR12];
    const float dd = d11[p] - d22[p];
    float def2 = 0.25f * (dd * dd);
    const float t = 0.25f * (d12[p] + d12[p + nx] + d12[p + 1] + d12[p + nx + 1]);
    def2 = def2 + t * t;
    const float mlen = sqrtf(g.dx / s[WF_MSFTX][c] * g.dy / s[WF_MSFTY][c]);
    const float sq = sqrtf(def2);
    const float v = (float)(C_S * C_S) * mlen * mlen * sq;
    if (X == 0.f || !(v < 10.0f * mlen) || !(sq > 0.f)) return;  // clamped, or sqrt's kink at 0
    const float def2b = (float)(C_S * C_S) * mlen * mlen * X * 0.5f / sq;
    d11b[p] = 0.5f * dd * def2b;
    d22b[p] = -0.5f * dd * def2b;
    const float qb = 0.5f * t * def2b;  // d def2 / d d12 = 2 t 0.25
    acc(d12b, p, qb);
    acc(d12b, p + nx, qb);
    acc(d12b, p + 1, qb);
    acc(d12b, p + nx + 1, qb);
  } else {
    const float old = s[WF_XKMH][p];
    if (!(old < cap)) b[WF_XKMH][p] = 0.f;
  }
}

// the reverse of hat(k, column) = f / m at one point
struct HatAdj {
  const float* m0;
  const float* m1;
  int pa, pb;
  float* fb;
};

__device__ __forceinline__ void hat_adj(const HatAdj& h, int k, size_t lev, bool second, float v) {
  const int pc = second ? h.pb : h.pa;
  acc(h.fb, (size_t)k * lev + pc, v / (second ? h.m1[pc] : h.m0[pc]));
}

// the reverse of the vertical average at w level kk (weights as hatavg)
__device__ void hatavg_adj(const Grid& g, const S& s, const HatAdj& h, int kk, size_t lev, float cft1, float cft2,
                           float bar) {
  if (bar == 0.f) return;
  const int ktf = g.nz - 1;
  if (kk >= 1 && kk < ktf) {
    const float a = 0.5f * s[WF_FNM][kk] * bar, b = 0.5f * s[WF_FNP][kk] * bar;
    hat_adj(h, kk, lev, false, a); hat_adj(h, kk, lev, true, a);
    hat_adj(h, kk - 1, lev, false, b); hat_adj(h, kk - 1, lev, true, b);
  } else if (kk == 0) {
    const float w[3] = {0.5f * g.cf1 * bar, 0.5f * g.cf2 * bar, 0.5f * g.cf3 * bar};
    for (int q = 0; q < 3; ++q) {
      hat_adj(h, q, lev, false, w[q]);
      hat_adj(h, q, lev, true, w[q]);
    }
  } else {
    const float a = 0.5f * cft1 * bar, b = 0.5f * cft2 * bar;
    hat_adj(h, g.nz - 2, lev, false, a); hat_adj(h, g.nz - 2, lev, true, a);
    hat_adj(h, g.nz - 3, lev, false, b); hat_adj(h, g.nz - 3, lev, true, b);
  }
}

__device__ __forceinline__ float hat_at(const float* f, const float* m, int k, size_t lev, int pc) {
  return f[(size_t)k * lev + pc] / m[pc];
}

__device__ float hatavg_at(const Grid& g, const S& s, const float* f, const float* m, int pa, int pb, int kk,
                           size_t lev, float cft1, float cft2) {
  const int ktf = g.nz - 1;
  auto h2 = [&](int k) { return hat_at(f, m, k, lev, pa) + hat_at(f, m, k, lev, pb); };
  if (kk >= 1 && kk < ktf) return 0.5f * (s[WF_FNM][kk] * h2(kk) + s[WF_FNP][kk] * h2(kk - 1));
  if (kk == 0) {
    return 0.5f * (g.cf1 * hat_at(f, m, 0, lev, pa) + g.cf2 * hat_at(f, m, 1, lev, pa) +
                   g.cf3 * hat_at(f, m, 2, lev, pa) + g.cf1 * hat_at(f, m, 0, lev, pb) +
                   g.cf2 * hat_at(f, m, 1, lev, pb) + g.cf3 * hat_at(f, m, 2, lev, pb));
  }
  return 0.5f * (cft1 * h2(g.nz - 2) + cft2 * h2(g.nz - 3));
}

// cal_deform_and_div's reverse for defor11, defor22 and defor12 (the
// boundary copies of defor12 are never read by the viscosity)
__global__ void k_deform_adj(Grid g, S s, S b, const float* d11b, const float* d22b, const float* d12b, float* zxb,
                             float* zyb, float* rdzwb) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, ktf = g.nz - 1, nx = g.nx;
  if (k >= ktf) return;
  const size_t lev = (size_t)g.ny * nx;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * lev + c;
  const float cft2 = -0.5f * s[WF_DNW][g.nz - 2] / s[WF_DN][g.nz - 2];
  const float cft1 = 1.0f - cft2;
  const float* zx = s[WF_ZX];
  const float* zy = s[WF_ZY];
  const float* rdzw = s[WF_RDZW];
  const float rdx = g.rdx, rdy = g.rdy;
  const bool d1 = j >= jds && j < jde - 1 && i >= ids && i < ide - 1;
  const bool d2 = j >= jds + 1 && j < jde - 1 && i >= ids + 1 && i < ide - 1;
  if (d1 && (d11b[p] != 0.f || d22b[p] != 0.f)) {
    const float mm = s[WF_MSFTX][c] * s[WF_MSFTY][c];
    const float* msfuy = s[WF_MSFUY];
    const float* msfvx = s[WF_MSFVX];
    {  // defor11 = 2 mm (rdx (hat(c+1) - hat(c)) - D 0.25 zsum rdzw)
      const float G2 = 2.0f * mm * d11b[p];
      HatAdj h{msfuy, msfuy, c, c + 1, b[WF_U]};
      hat_adj(h, k, lev, true, rdx * G2);
      hat_adj(h, k, lev, false, -rdx * G2);
      const float D = hatavg_at(g, s, s[WF_U], msfuy, c, c + 1, k + 1, lev, cft1, cft2) -
                      hatavg_at(g, s, s[WF_U], msfuy, c, c + 1, k, lev, cft1, cft2);
      const float zsum = zx[p] + zx[p + 1] + zx[p + lev] + zx[p + lev + 1];
      const float Db = -G2 * (0.25f * zsum * rdzw[p]);
      hatavg_adj(g, s, h, k + 1, lev, cft1, cft2, Db);
      hatavg_adj(g, s, h, k, lev, cft1, cft2, -Db);
      const float zb = -G2 * D * 0.25f * rdzw[p];
      acc(zxb, p, zb); acc(zxb, p + 1, zb); acc(zxb, p + lev, zb); acc(zxb, p + lev + 1, zb);
      acc(rdzwb, p, -G2 * D * 0.25f * zsum);
    }
    {  // defor22, with v, msfvx, the y neighbour and zy
      const float G2 = 2.0f * mm * d22b[p];
      HatAdj h{msfvx, msfvx, c, c + nx, b[WF_V]};
      hat_adj(h, k, lev, true, rdy * G2);
      hat_adj(h, k, lev, false, -rdy * G2);
      const float D = hatavg_at(g, s, s[WF_V], msfvx, c, c + nx, k + 1, lev, cft1, cft2) -
                      hatavg_at(g, s, s[WF_V], msfvx, c, c + nx, k, lev, cft1, cft2);
      const float zsum = zy[p] + zy[p + nx] + zy[p + lev] + zy[p + lev + nx];
      const float Db = -G2 * (0.25f * zsum * rdzw[p]);
      hatavg_adj(g, s, h, k + 1, lev, cft1, cft2, Db);
      hatavg_adj(g, s, h, k, lev, cft1, cft2, -Db);
      const float zb = -G2 * D * 0.25f * rdzw[p];
      acc(zyb, p, zb); acc(zyb, p + nx, zb); acc(zyb, p + lev, zb); acc(zyb, p + lev + nx, zb);
      acc(rdzwb, p, -G2 * D * 0.25f * zsum);
    }
  }
  if (d2 && d12b[p] != 0.f) {
    const float* msfux = s[WF_MSFUX];
    const float* msfvy = s[WF_MSFVY];
    const float mm = 0.25f * (msfux[c - nx] + msfux[c]) * (msfvy[c - 1] + msfvy[c]);
    const float gm = mm * d12b[p];
    const size_t q[4] = {p, p - 1, p - nx - 1, p - nx};  // the four rdzw points
    float rsum = rdzw[q[0]] + rdzw[q[1]] + rdzw[q[2]] + rdzw[q[3]];
    {  // u part: rdy (hat(c) - hat(c - nx)) - D 0.25 zysum 0.25 rsum
      HatAdj h{msfux, msfux, c - nx, c, b[WF_U]};
      hat_adj(h, k, lev, true, rdy * gm);
      hat_adj(h, k, lev, false, -rdy * gm);
      const float D = hatavg_at(g, s, s[WF_U], msfux, c - nx, c, k + 1, lev, cft1, cft2) -
                      hatavg_at(g, s, s[WF_U], msfux, c - nx, c, k, lev, cft1, cft2);
      const float zsum = zy[p - 1] + zy[p] + zy[p + lev - 1] + zy[p + lev];
      const float Db = -gm * (0.25f * zsum * 0.25f * rsum);
      hatavg_adj(g, s, h, k + 1, lev, cft1, cft2, Db);
      hatavg_adj(g, s, h, k, lev, cft1, cft2, -Db);
      const float zb = -gm * D * 0.0625f * rsum;
      acc(zyb, p - 1, zb); acc(zyb, p, zb); acc(zyb, p + lev - 1, zb); acc(zyb, p + lev, zb);
      const float rb = -gm * D * 0.0625f * zsum;
      for (int e = 0; e < 4; ++e) acc(rdzwb, q[e], rb);
    }
    {  // v part: rdx (hat(c) - hat(c - 1)) - D 0.25 zxsum 0.25 rsum
      HatAdj h{msfvy, msfvy, c - 1, c, b[WF_V]};
      hat_adj(h, k, lev, true, rdx * gm);
      hat_adj(h, k, lev, false, -rdx * gm);
      const float D = hatavg_at(g, s, s[WF_V], msfvy, c - 1, c, k + 1, lev, cft1, cft2) -
                      hatavg_at(g, s, s[WF_V], msfvy, c - 1, c, k, lev, cft1, cft2);
      const float zsum = zx[p - nx] + zx[p] + zx[p + lev - nx] + zx[p + lev];
      const float Db = -gm * (0.25f * zsum * 0.25f * rsum);
      hatavg_adj(g, s, h, k + 1, lev, cft1, cft2, Db);
      hatavg_adj(g, s, h, k, lev, cft1, cft2, -Db);
      const float zb = -gm * D * 0.0625f * rsum;
      acc(zxb, p - nx, zb); acc(zxb, p, zb); acc(zxb, p + lev - nx, zb); acc(zxb, p + lev, zb);
      const float rb = -gm * D * 0.0625f * zsum;
      for (int e = 0; e < 4; ++e) acc(rdzwb, q[e], rb);
    }
  }
}

// compute_diff_metrics' reverse for rdzw, zx and zy (phb is data)
__global__ void k_metrics_adj(Grid g, S s, S b, const float* zxb, const float* zyb, const float* rdzwb) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde, ktf = g.nz - 1;
  const size_t lev = (size_t)g.ny * g.nx;
  const size_t p = (size_t)k * lev + g.i2(j, i);
  const float* ph = s[WF_PH];
  const float* phb = s[WF_PHB];
  float* phbar = b[WF_PH];
  const float gf = (float)G;
  if (k < ktf && j >= jds - 1 && j < jde && i >= ids && i < ide - 1 && rdzwb[p] != 0.f) {
    const float z0 = (ph[p] + phb[p]) / gf, z1 = (ph[p + lev] + phb[p + lev]) / gf;
    const float r = 1.0f / (z1 - z0);
    const float v = r * r / gf * rdzwb[p];
    acc(phbar, p + lev, -v);
    acc(phbar, p, v);
  }
  if (j >= jds && j < jde - 1 && i >= ids + 1 && i < ide - 1 && zxb[p] != 0.f) {
    const float v = g.rdx / gf * zxb[p];
    acc(phbar, p, v);
    acc(phbar, p - 1, -v);
  }
  if (j >= jds + 1 && j < jde - 1 && i >= ids && i < ide - 1 && zyb[p] != 0.f) {
    const float v = g.rdy / gf * zyb[p];
    acc(phbar, p, v);
    acc(phbar, p - g.nx, -v);
  }
}

// ---- mass_weight: out = field * mut on levels < nk of the mass points ----

__device__ __forceinline__ bool mw_region(const Grid& g, int k, int j, int i, int nk) {
  return k < nk && j >= g.jds && j < g.jde - 1 && i >= g.ids && i < g.ide - 1;
}

__global__ void k_mass_weight(Grid g, const float* f, const float* mut, float* out, int nk) {
  WRF_POINT_INDEX(g, k, j, i);
  if (!mw_region(g, k, j, i, nk)) return;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  out[p] = f[p] * mut[c];
}

__global__ void k_mass_weight_adj(Grid g, const float* f, const float* mut, const float* ob, float* fb, float* mb,
                                  int nk) {
  WRF_POINT_INDEX(g, k, j, i);
  if (!mw_region(g, k, j, i, nk)) return;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const float o = ob[p];
  if (o == 0.f) return;
  fb[p] += o * mut[c];
  acc(mb, c, o * f[p]);
}

}  // namespace

// var: 'u', 'v', 'w' or 'm' (a scalar; with base, theta's diffusion about it)
int launch_hdiff_op(const Grid& g, const S& s, char var, const float* f, const float* base, const float* mut,
                    const float* K, float* tend, cudaStream_t st) {
  const int v = var == 'u' ? DV_U : (var == 'v' ? DV_V : (var == 'w' ? DV_W : DV_M));
  const dim3 b3(32, 4), grid((g.nx + 31) / 32, (g.ny + 3) / 4, (g.nz + kHdiffLevels - 1) / kHdiffLevels);
  k_hdiff_op<<<grid, b3, 0, st>>>(g, s, v, f, base, mut, K, tend);
  return 1;
}

int launch_hdiff_op_adj(const Grid& g, const S& s, char var, const float* f, const float* base, const float* mut,
                        const float* K, const float* tbar, float* fbar, float* mutbar, float* Kbar, cudaStream_t st) {
  const int v = var == 'u' ? DV_U : (var == 'v' ? DV_V : (var == 'w' ? DV_W : DV_M));
  const dim3 b3(32, 4), grid((g.nx + 31) / 32, (g.ny + 3) / 4, (g.nz + kHdiffLevels - 1) / kHdiffLevels);
  k_hdiff_op_adj<<<grid, b3, 0, st>>>(g, s, v, f, base, mut, K, tbar, fbar, mutbar, Kbar);
  return 1;
}

// the eddy viscosities as the step forms them at the first stage: metrics,
// their halo copies, deformations and calculate_km_kh (the table's rdzw,
// rdz, z, zx, zy and defor fields are scratch)
int launch_km_op(const Grid& g, const S& s, cudaStream_t st) {
  int n = launch_diff_metrics(g, s, st);
  n += launch_halo(g, s[WF_RDZW], 'w', false, st);
  n += launch_halo(g, s[WF_ZX], 'e', false, st);
  n += launch_halo(g, s[WF_ZY], 'f', false, st);
  return n + launch_km(g, s, st);
}

// work: caller scratch of 6 nz ny nx floats (the deformations' and the
// metrics' cotangents); the table's metric and defor fields are scratch
// that the reverse refills from the forward's inputs
int launch_km_op_adj(const Grid& g, const S& s, const S& b, float* work, cudaStream_t st) {
  const size_t n3 = g.n3();
  float* d11b = work;
  float* d22b = work + n3;
  float* d12b = work + 2 * n3;
  float* zxb = work + 3 * n3;
  float* zyb = work + 4 * n3;
  float* rdzwb = work + 5 * n3;
  cudaMemsetAsync(work, 0, 6 * n3 * sizeof(float), st);
  int n = launch_diff_metrics(g, s, st);
  n += launch_deform(g, s, st);
  const dim3 b3(32, 4);
  k_km_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, d11b, d22b, d12b);
  k_deform_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, d11b, d22b, d12b, zxb, zyb, rdzwb);
  k_metrics_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, zxb, zyb, rdzwb);
  return n + 3;
}

int launch_mass_weight(const Grid& g, const float* f, const float* mut, float* out, int nk, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_mass_weight<<<point_grid(g, b3), b3, 0, st>>>(g, f, mut, out, nk);
  return 1;
}

int launch_mass_weight_adj(const Grid& g, const float* f, const float* mut, const float* ob, float* fb, float* mb,
                           int nk, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_mass_weight_adj<<<point_grid(g, b3), b3, 0, st>>>(g, f, mut, ob, fb, mb, nk);
  return 1;
}

}  // namespace wrf
