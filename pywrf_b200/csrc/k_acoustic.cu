// Acoustic (small) time step (wrf_dynamics.py:3152-3930, wrf_boundary.py:244-400).
//   k_ssp2d / k_ssp3d   small_step_prep (2-D masses, then 3-D perturbation form)
//   k_p_rho0            calc_p_rho before the first substep
//   k_coef_w            calc_coef_w: tridiagonal coefficients + forward sweep
//   k_advance_uv        advance_uv + spec_bdyupdate(u), (v)
//   k_acoustic_col      advance_mu_t, advance_w, sumflux, spec_bdyupdate of
//                       t / mu / muts / ph and calc_p_rho of one substep
//   k_mu_uv_1 / k_ssfinish  calc_mu_uv_1, small_step_finish
// The vertical recurrences (mass divergence sum, ww scan, Thomas sweeps) run
// sequentially per column in the reference's order.
#include "kernels.cuh"
#include "tma.cuh"

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

// all operands are loaded before any store (the stores would otherwise hold
// back the later fields' loads); in stage 1 the *_1 copies are the values
// just read
__global__ void k_ssp3d(Grid g, S s, int rk_step) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nz = g.nz, ktf = nz - 1;
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const bool t2 = j >= jts && j < jme && i >= its && i < ime;
  const bool du = k < ktf && j >= jts && j < jme && i >= its && i < ieu;
  const bool dv = k < ktf && j >= jts && j < jev && i >= its && i < ime;
  const bool r1 = rk_step == 1;
  float u2 = 0.f, u1 = 0.f, muus = 0.f, muu = 0.f, mfuy = 1.f;
  if (du) {
    u2 = s[WF_U][p];
    u1 = r1 ? u2 : s[WF_U_1][p];
    muus = s[WF_MUUS][c];
    muu = s[WF_MUU][c];
    mfuy = s[WF_MSFUY][c];
  }
  float v2 = 0.f, v1 = 0.f, muvs = 0.f, muv = 0.f, mvxi = 0.f;
  if (dv) {
    v2 = s[WF_V][p];
    v1 = r1 ? v2 : s[WF_V_1][p];
    muvs = s[WF_MUVS][c];
    muv = s[WF_MUV][c];
    mvxi = s[WF_MSFVX_INV][c];
  }
  float muts = 0.f, mut = 0.f, pbv = 0.f, ppv = 0.f, altv = 1.f, t2v = 0.f, t1 = 0.f;
  float w2 = 0.f, w1 = 0.f, mfty = 1.f, ph2 = 0.f, ph1 = 0.f, wwv = 0.f;
  if (t2) {
    muts = s[WF_MUTS][c];
    mut = s[WF_MUT][c];
    if (k < ktf) {
      pbv = s[WF_PB][p];
      ppv = s[WF_P][p];
      altv = s[WF_ALT][p];
      t2v = s[WF_T][p];
      t1 = r1 ? t2v : s[WF_T_1][p];
    }
    w2 = s[WF_W][p];
    w1 = r1 ? w2 : s[WF_W_1][p];
    mfty = s[WF_MSFTY][c];
    ph2 = s[WF_PH][p];
    ph1 = r1 ? ph2 : s[WF_PH_1][p];
    wwv = s[WF_WW][p];
  }
  if (du) {
    if (r1) s[WF_U_1][p] = u2;
    s[WF_U_SAVE][p] = u2;
    s[WF_U][p] = (muus * u1 - muu * u2) / mfuy;
  }
  if (dv) {
    if (r1) s[WF_V_1][p] = v2;
    s[WF_V_SAVE][p] = v2;
    s[WF_V][p] = (muvs * v1 - muv * v2) * mvxi;
  }
  if (t2) {
    if (k < ktf) {
      s[WF_C2A][p] = (float)CPOVCV * (pbv + ppv) / altv;
      if (r1) s[WF_T_1][p] = t2v;
      s[WF_T_SAVE][p] = t2v;
      s[WF_T][p] = muts * t1 - mut * t2v;
    }
    if (r1) s[WF_W_1][p] = w2;
    s[WF_W_SAVE][p] = w2;
    s[WF_W][p] = (muts * w1 - mut * w2) / mfty;
    if (r1) s[WF_PH_1][p] = ph2;
    s[WF_PH_SAVE][p] = ph2;
    s[WF_PH][p] = ph1 - ph2;
    s[WF_WW1][p] = wwv;
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
    // operands first, then the stores
    const float muts = s[WF_MUTS][c], mu = s[WF_MU][c];
    const float alt = s[WF_ALT][p], t1 = s[WF_T_SAVE][p];
    const float* ph = s[WF_PH];
    const float phu = ph[p + lev], phk = ph[p], rdnw = s[WF_RDNW][k];
    const float c2 = s[WF_C2A][p], tk = s[WF_T][p];
    const float al = -1.0f / muts * (alt * mu + rdnw * (phu - phk));
    pnew = c2 * (alt * (tk - mu * t1) / (muts * ((float)T0 + t1)) - al);
    s[WF_AL][p] = al;
    pp[p] = pnew;
  }
  s[WF_PM1][p] = pnew;
}

// calc_coef_w: a block owns 16 adjacent mass columns of one row and 16 level
// groups; the per-level coefficients a, b, c are formed in parallel into
// shared memory, one thread per column runs the recurrence alpha = 1 / (b - a
// gamma), gamma = c alpha in the reference's order, and the levels are stored
// in parallel again.
constexpr int kCwTX = 16, kCwKT = 16;

__global__ void __launch_bounds__(kCwTX * kCwKT) k_coef_w(Grid g, S s, float dts) {
  __shared__ float sa[kMaxNz][kCwTX], sb[kMaxNz][kCwTX], sc[kMaxNz][kCwTX];
  __shared__ float stop[2][kCwTX];  // atop, alpha at the top
  const int tx = threadIdx.x % kCwTX, tk = threadIdx.x / kCwTX;
  const int i = g.ids + blockIdx.x * kCwTX + tx, j = g.jds + blockIdx.y;
  const bool col = i < g.ide - 1;
  const int nz = g.nz;
  const int c = col ? g.i2(j, i) : g.i2(j, g.ids);
  const size_t lev = (size_t)g.ny * g.nx;
  const double cofd = (0.5 * (double)dts * G * (1.0 + (double)g.epssm)) * (0.5 * (double)dts * G * (1.0 + (double)g.epssm));
  const float cof = (float)cofd, cofm2 = (float)(-2.0 * cofd), cof2 = (float)(2.0 * cofd);
  const float* cqw = s[WF_CQW];
  const float* c2a = s[WF_C2A];
  const float* rdn = s[WF_RDN];
  const float* rdnw = s[WF_RDNW];
  float* a = s[WF_A];
  float* alpha = s[WF_ALPHA];
  float* gamma = s[WF_GAMMA];
  const float mut = col ? s[WF_MUT][c] : 1.f;
  const float mm = mut * mut;
  if (col) {
    for (int k = 1 + tk; k < nz - 1; k += kCwKT) {
      const size_t p = k * lev + c;
      const float cw = __ldg(&cqw[p]), c2k = __ldg(&c2a[p]), c2m = __ldg(&c2a[p - lev]);
      sa[k][tx] = k >= 2 ? -cw * cof * rdn[k] * rdnw[k - 1] * c2m / mm : 0.f;
      sb[k][tx] = 1.0f + cw * cof * rdn[k] * (rdnw[k] * c2k / mm + rdnw[k - 1] * c2m / mm);
      sc[k][tx] = -cw * cof * rdn[k] * rdnw[k] * c2k / mm;
    }
  }
  __syncthreads();
  if (col && tk == 0) {
    const float lid = g.top_lid ? 0.f : 1.f;
    const float c2t = __ldg(&c2a[(nz - 2) * lev + c]);
    const float atop = cofm2 * (rdnw[nz - 2] * rdnw[nz - 2]) * c2t * lid / mm;
    float gm = 0.f;
    for (int k = 1; k < nz - 1; ++k) {
      const float al = 1.0f / (sb[k][tx] - sa[k][tx] * gm);
      sb[k][tx] = al;  // alpha(k)
      gm = sc[k][tx] * al;
      sc[k][tx] = gm;  // gamma(k)
    }
    const float btop = 1.0f + cof2 * (rdnw[nz - 2] * rdnw[nz - 2]) * c2t / mm;
    stop[0][tx] = atop;
    stop[1][tx] = 1.0f / (btop - atop * gm);
  }
  __syncthreads();
  if (!col) return;
  for (int k = tk; k < nz; k += kCwKT) {
    const size_t p = k * lev + c;
    if (k == 0) {
      gamma[p] = 0.f;
    } else if (k < nz - 1) {
      a[p] = k >= 2 ? sa[k][tx] : 0.f;
      alpha[p] = sb[k][tx];
      gamma[p] = sc[k][tx];
    } else {
      a[p] = stop[0][tx];
      alpha[p] = stop[1][tx];
      gamma[p] = 0.f;
    }
  }
}

// calc_coef_w with one thread per mass column (32 x 4 columns per block): the
// coefficients of level k are formed as the recurrence reaches it, so nothing
// waits on a block barrier and every level's loads and stores are coalesced
// across the warp.  The same operations as k_coef_w, in the same order (the
// divisions by mut^2 and the reciprocals in their correctly rounded forms).
__global__ void __launch_bounds__(128) k_coef_w_col(Grid g, S s, float dts) {
  const int i = g.ids + blockIdx.x * 32 + threadIdx.x, j = g.jds + blockIdx.y * 4 + threadIdx.y;
  if (i >= g.ide - 1 || j >= g.jde - 1) return;
  const int nz = g.nz;
  const int c = g.i2(j, i);
  const size_t lev = (size_t)g.ny * g.nx;
  const double cofd = (0.5 * (double)dts * G * (1.0 + (double)g.epssm)) * (0.5 * (double)dts * G * (1.0 + (double)g.epssm));
  const float cof = (float)cofd, cofm2 = (float)(-2.0 * cofd), cof2 = (float)(2.0 * cofd);
  const float* cqw = s[WF_CQW];
  const float* c2a = s[WF_C2A];
  const float* rdn = s[WF_RDN];
  const float* rdnw = s[WF_RDNW];
  float* a = s[WF_A];
  float* alpha = s[WF_ALPHA];
  float* gamma = s[WF_GAMMA];
  const float mut = s[WF_MUT][c];
  const float mm = mut * mut, r_mm = __frcp_rn(mm);
  gamma[c] = 0.f;
  float gm = 0.f;
  float c2m = __ldg(&c2a[c]);
#pragma unroll 4
  for (int k = 1; k < nz - 1; ++k) {
    const size_t p = k * lev + c;
    const float cw = __ldg(&cqw[p]), c2k = __ldg(&c2a[p]);
    const float rk = __ldg(&rdn[k]), rwk = __ldg(&rdnw[k]), rwm = __ldg(&rdnw[k - 1]);
    const float ak = k >= 2 ? divc(-cw * cof * rk * rwm * c2m, mm, r_mm) : 0.f;
    const float bk = 1.0f + cw * cof * rk * (divc(rwk * c2k, mm, r_mm) + divc(rwm * c2m, mm, r_mm));
    const float ck = divc(-cw * cof * rk * rwk * c2k, mm, r_mm);
    const float al = __frcp_rn(bk - ak * gm);
    gm = ck * al;
    a[p] = ak;
    alpha[p] = al;
    gamma[p] = gm;
    c2m = c2k;
  }
  const float lid = g.top_lid ? 0.f : 1.f;
  const float rwt = __ldg(&rdnw[nz - 2]);
  const float atop = divc(cofm2 * (rwt * rwt) * c2m * lid, mm, r_mm);
  const float btop = 1.0f + divc(cof2 * (rwt * rwt) * c2m, mm, r_mm);
  const size_t pt = (size_t)(nz - 1) * lev + c;
  a[pt] = atop;
  alpha[pt] = __frcp_rn(btop - atop * gm);
  gamma[pt] = 0.f;
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

// advance_uv, tensor-map form (nx a multiple of 4): a block of 32 x 8
// threads owns 32 x 8 columns (u and v points (j, i)) and a chunk of levels.
// Per level one thread loads boxes of alt, al, pb, php at k and ph, p at k+1
// (40 x 9 from x = floor4(i0 - 1), y = j0 - 1: every point's i-1 and j-1
// neighbours) into an mbarrier ring two levels ahead; ph(k), p(k) and the
// vertical pressure averages dpn(k) come from the level below in registers
// (each is the same operation on the same operands as in k_advance_uv), and
// the thread's own u, v, tendencies and cq are loaded a level ahead.  Every
// wait on a box is bounded; a block whose wait runs out stops, drains its
// copies and adds 1 to STATUS[WRF_ST_WAIT].
constexpr int kUvTX = 32, kUvTY = 8, kUvBW = 40, kUvBH = kUvTY + 1;
constexpr int kUvNB = 6;                 // boxes per level: alt al pb php (k), ph p (k+1)
constexpr int kUvSlot = 384;             // floats per box slot (1536 B >= 40 x 9 x 4)
constexpr int kUvOW = 36, kUvOH = kUvTY;  // the thread's own u, ru_tend, v, rv_tend, cqu, cqv at k
constexpr int kUvNO = 6, kUvOSlot = kUvOW * kUvOH;  // 1152 B, a 128-byte multiple
constexpr int kUvRing = 3, kUvKCH = 7;
constexpr uint32_t kUvBytes = kUvNB * kUvBW * kUvBH * 4 + kUvNO * kUvOW * kUvOH * 4;
constexpr long long kUvWaitCycles = 4000000000LL;
static_assert(kUvBW * kUvBH <= kUvSlot && (kUvOSlot * 4) % 128 == 0, "ring slots hold one box, 128-byte aligned");

struct UvTmaArgs {
  CUtensorMap alt, al, pb, php, ph, pp;
  CUtensorMap own[kUvNO];  // u, ru_tend, v, rv_tend, cqu, cqv
  int nchunk;
};

__global__ void __launch_bounds__(kUvTX * kUvTY, 4) k_advance_uv_tma(Grid g, S s, float dts,
                                                                     const __grid_constant__ UvTmaArgs a) {
  __shared__ __align__(128) float box[kUvRing][kUvNB][kUvSlot];
  __shared__ __align__(128) float obox[kUvRing][kUvNO][kUvOSlot];
  __shared__ uint64_t bar[kUvRing];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kUvTX + tx;
  const int nx = g.nx, ny = g.ny, nz = g.nz, ktf = nz - 1;
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const int i0 = ids + blockIdx.x * kUvTX, j0 = jds + blockIdx.y * kUvTY;
  const int i = i0 + tx, j = j0 + ty;
  const int mx = (i0 - 1) & ~3, om = i0 - mx;
  const int ox = i0 & ~3, oo = i0 - ox;
  const int k0 = blockIdx.z * ktf / a.nchunk, k1 = (blockIdx.z + 1) * ktf / a.nchunk;
  const size_t lev = (size_t)ny * nx;
  const bool uin = j >= jds + 1 && j < jde - 2 && i >= ids + 1 && i < ide - 1;
  const bool uspec = ((j == jds || j == jde - 2) && i >= ids && i < ide) ||
                     (j >= jds + 1 && j < jde - 2 && (i == ids || i == ide - 1));
  const bool vin = j >= jds + 1 && j < jde - 1 && i >= ids + 1 && i < ide - 2;
  const bool vspec = ((j == jds || j == jde - 1) && i >= ids && i < ide - 1) ||
                     (j >= jds + 1 && j < jde - 1 && (i == ids || i == ide - 2));
  const bool wu = uin || uspec, wv = vin || vspec;
  const int c = min(j, ny - 1) * nx + min(i, nx - 1);
  const float* pp = s[WF_P];
  const float* ph = s[WF_PH];
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  const float* rdnw = s[WF_RDNW];
  float* U = s[WF_U];
  float* V = s[WF_V];
  const float rdx = g.rdx, rdy = g.rdy;

  if (tid == 0) {
    for (int r = 0; r < kUvRing; ++r) tma::mbar_init(&bar[r], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int k, int r) {
    tma::mbar_expect_tx(&bar[r], kUvBytes);
    tma::load_4d(box[r][0], &a.alt, mx, j0 - 1, k, 0, &bar[r]);
    tma::load_4d(box[r][1], &a.al, mx, j0 - 1, k, 0, &bar[r]);
    tma::load_4d(box[r][2], &a.pb, mx, j0 - 1, k, 0, &bar[r]);
    tma::load_4d(box[r][3], &a.php, mx, j0 - 1, k, 0, &bar[r]);
    tma::load_4d(box[r][4], &a.ph, mx, j0 - 1, k + 1, 0, &bar[r]);
    tma::load_4d(box[r][5], &a.pp, mx, j0 - 1, k + 1, 0, &bar[r]);
    for (int f = 0; f < kUvNO; ++f) tma::load_4d(obox[r][f], &a.own[f], ox, j0, k, 0, &bar[r]);
  };
  int hi = k0 - 1;
  if (tid == 0) {
    for (int k = k0; k < min(k0 + kUvRing - 1, k1); ++k) issue(k, k - k0);
    hi = min(k0 + kUvRing - 1, k1) - 1;
  }
  // per-column constants, in the association order of k_advance_uv
  float mudf_u = 0.f, cu = 0.f, ru = 0.f, muav_u = 0.f, mudf_v = 0.f, cv = 0.f, rv = 0.f, muav_v = 0.f;
  if (uin) {
    const float* mudf = s[WF_MUDF];
    const float* mu = s[WF_MU];
    mudf_u = (float)(-(double)g.emdiv * g.dxd) * (__ldg(&mudf[c]) - __ldg(&mudf[c - 1])) / __ldg(&s[WF_MSFUY][c]);
    const float r = __ldg(&s[WF_MSFUX][c]) / __ldg(&s[WF_MSFUY][c]);
    cu = r * 0.5f * rdx * __ldg(&s[WF_MUU][c]);
    ru = r * rdx;
    muav_u = 0.5f * (__ldg(&mu[c - 1]) + __ldg(&mu[c]));
  }
  if (vin) {
    const float* mudf = s[WF_MUDF];
    const float* mu = s[WF_MU];
    mudf_v = (float)(-(double)g.emdiv * g.dyd) * (__ldg(&mudf[c]) - __ldg(&mudf[c - nx])) * __ldg(&s[WF_MSFVX_INV][c]);
    const float r = __ldg(&s[WF_MSFVY][c]) / __ldg(&s[WF_MSFVX][c]);
    cv = r * 0.5f * rdy * __ldg(&s[WF_MUV][c]);
    rv = r * rdy;
    muav_v = 0.5f * (__ldg(&mu[c - nx]) + __ldg(&mu[c]));
  }
  // ph(k), p(k) at (j, i), (j, i-1), (j-1, i) and dpn(k) of the u and v points
  const int cw = (uin || vin) ? c - 1 : c, cs = (uin || vin) ? c - nx : c;
  float ph_c = 0.f, ph_w = 0.f, ph_s = 0.f, p_c = 0.f, p_w = 0.f, p_s = 0.f, dpn_u = 0.f, dpn_v = 0.f;
  if (uin || vin) {
    const size_t q = (size_t)k0 * lev;
    ph_c = __ldg(&ph[q + c]);
    ph_w = __ldg(&ph[q + cw]);
    ph_s = __ldg(&ph[q + cs]);
    p_c = __ldg(&pp[q + c]);
    p_w = __ldg(&pp[q + cw]);
    p_s = __ldg(&pp[q + cs]);
    if (k0 == 0) {  // dpn(0): cf1..cf3 over the three lowest levels
      const float a1 = __ldg(&pp[lev + c]), a2 = __ldg(&pp[2 * lev + c]);
      const float w1 = __ldg(&pp[lev + cw]), w2 = __ldg(&pp[2 * lev + cw]);
      const float s1 = __ldg(&pp[lev + cs]), s2 = __ldg(&pp[2 * lev + cs]);
      dpn_u = 0.5f * (g.cf1 * (p_c + p_w) + g.cf2 * (a1 + w1) + g.cf3 * (a2 + w2));
      dpn_v = 0.5f * (g.cf1 * (p_c + p_s) + g.cf2 * (a1 + s1) + g.cf3 * (a2 + s2));
    } else if (k0 < nz - 1) {
      const float fm = __ldg(&fnm[k0]), fp = __ldg(&fnp[k0]);
      const size_t qm = q - lev;
      dpn_u = 0.5f * (fm * (p_c + p_w) + fp * (__ldg(&pp[qm + c]) + __ldg(&pp[qm + cw])));
      dpn_v = 0.5f * (fm * (p_c + p_s) + fp * (__ldg(&pp[qm + c]) + __ldg(&pp[qm + cs])));
    }
  }
  const int oA = (ty + 1) * kUvBW + om + tx;
  const int oO = ty * kUvOW + oo + tx;  // (j, i) in an own-value box
  int kstop = k1, slot = 0;
  uint32_t par = 0;
  for (int k = k0; k < k1; ++k) {
    const float rdk = __ldg(&rdnw[k]);
    const float fm1 = k + 1 < nz - 1 ? __ldg(&fnm[k + 1]) : 0.f, fp1 = k + 1 < nz - 1 ? __ldg(&fnp[k + 1]) : 0.f;
    const bool ok = tma::mbar_wait_bounded(&bar[slot], par, kUvWaitCycles);
    if (__syncthreads_or(!ok)) {
      kstop = k;
      break;
    }
    // every thread is past level k-1: its slot takes level k + kUvRing - 1
    if (tid == 0 && k + kUvRing - 1 < k1) {
      issue(k + kUvRing - 1, slot == 0 ? kUvRing - 1 : slot - 1);
      hi = k + kUvRing - 1;
    }
    const float* B = box[slot][0];
    const size_t p = (size_t)k * lev + c;
    const float u0 = obox[slot][0][oO], rt0 = obox[slot][1][oO], v0 = obox[slot][2][oO];
    const float vt0 = obox[slot][3][oO], qu0 = obox[slot][4][oO], qv0 = obox[slot][5][oO];
    float pu_c = 0.f, pu_w = 0.f, pu_s = 0.f, hu_c = 0.f, hu_w = 0.f, hu_s = 0.f;
    if (uin || vin) {
      hu_c = B[4 * kUvSlot + oA];
      pu_c = B[5 * kUvSlot + oA];
      hu_w = B[4 * kUvSlot + oA - 1];
      pu_w = B[5 * kUvSlot + oA - 1];
      hu_s = B[4 * kUvSlot + oA - kUvBW];
      pu_s = B[5 * kUvSlot + oA - kUvBW];
    }
    float unew = 0.f, vnew = 0.f;
    if (uin) {
      const float u = u0 + dts * rt0;
      const float alt_c = B[oA], alt_w = B[oA - 1];
      const float al_c = B[kUvSlot + oA], al_w = B[kUvSlot + oA - 1];
      const float pb_c = B[2 * kUvSlot + oA], pb_w = B[2 * kUvSlot + oA - 1];
      const float php_c = B[3 * kUvSlot + oA], php_w = B[3 * kUvSlot + oA - 1];
      const float dpn_up = k + 1 == nz - 1 ? 0.f : 0.5f * (fm1 * (pu_c + pu_w) + fp1 * (p_c + p_w));
      float dp = cu * (((hu_c - hu_w) + (ph_c - ph_w)) + (alt_c + alt_w) * (p_c - p_w) + (al_c + al_w) * (pb_c - pb_w));
      dp = dp + ru * (php_c - php_w) * (rdk * (dpn_up - dpn_u) - muav_u);
      unew = u - dts * qu0 * dp + mudf_u;
      dpn_u = dpn_up;
    } else if (uspec) {
      unew = u0 + dts * rt0;  // spec_bdyupdate(u)
    }
    if (vin) {
      const float v = v0 + dts * vt0;
      const float alt_c = B[oA], alt_s = B[oA - kUvBW];
      const float al_c = B[kUvSlot + oA], al_s = B[kUvSlot + oA - kUvBW];
      const float pb_c = B[2 * kUvSlot + oA], pb_s = B[2 * kUvSlot + oA - kUvBW];
      const float php_c = B[3 * kUvSlot + oA], php_s = B[3 * kUvSlot + oA - kUvBW];
      const float dpn_up = k + 1 == nz - 1 ? 0.f : 0.5f * (fm1 * (pu_c + pu_s) + fp1 * (p_c + p_s));
      float dp = cv * (((hu_c - hu_s) + (ph_c - ph_s)) + (alt_c + alt_s) * (p_c - p_s) + (al_c + al_s) * (pb_c - pb_s));
      dp = dp + rv * (php_c - php_s) * (rdk * (dpn_up - dpn_v) - muav_v);
      vnew = v - dts * qv0 * dp + mudf_v;
      dpn_v = dpn_up;
    } else if (vspec) {
      vnew = v0 + dts * vt0;  // spec_bdyupdate(v)
    }
    if (wu) U[p] = unew;
    if (wv) V[p] = vnew;
    ph_c = hu_c;
    ph_w = hu_w;
    ph_s = hu_s;
    p_c = pu_c;
    p_w = pu_w;
    p_s = pu_s;
    if (++slot == kUvRing) {
      slot = 0;
      par ^= 1u;
    }
  }
  if (kstop < k1 && tid == 0) {
    for (int k = kstop; k <= hi; ++k)
      tma::mbar_wait_bounded(&bar[(k - k0) % kUvRing], ((k - k0) / kUvRing) & 1, kUvWaitCycles);
    if (s[WF_STATUS]) atomicAdd(reinterpret_cast<int*>(s[WF_STATUS]) + WRF_ST_WAIT, 1);
  }
}

// Fused acoustic column update of one substep: advance_mu_t, advance_w,
// sumflux, spec_bdyupdate of t / mu / muts / ph, calc_p_rho
// (wrf_dynamics.py:3528-3839, 3269-3313; wrf_boundary.py:244-355).  A block
// owns kColTX adjacent columns of one row; thread (tx, tk) handles the levels
// k = tk, tk + kColKT, ... of column tx.  The explicit parts run over levels
// in parallel; the vertical recurrences (column mass divergence sum, ww scan,
// Thomas sweeps) run sequentially per column in the reference's order, from
// separate shared arrays so that their loads pipeline.  Small blocks and few
// registers let several blocks share an SM, which overlaps one block's
// sweeps with the memory phases of the others.  No column reads another
// column's result of this kernel; zero_grad_bdy(w) follows in the substep's
// halo launch (k_bc).
// Divisions by per-column constants use the correctly rounded form divc with
// the column's reciprocals (__frcp_rn).
constexpr int kColTX = 16, kColKT = 16;

// NQ = ceil(nz / kColKT) level slots per thread.  Phases that store to global
// memory first load every slot's operands into registers and only then
// compute and store: the loads of a thread's levels are then all in flight at
// once (the compiler cannot hoist a later level's loads above an earlier
// level's stores through possibly aliasing field pointers).
#ifndef WRF_COL_MINB
#define WRF_COL_MINB 4
#endif
template <int NQ>
__global__ void __launch_bounds__(kColTX * kColKT, WRF_COL_MINB) k_acoustic_col(Grid g, S s, float dts, int iteration, int nsub) {
  __shared__ float sdw[kMaxNz][kColTX], sww[kMaxNz][kColTX], st2av[kMaxNz][kColTX], srhs[kMaxNz][kColTX];
  __shared__ float sa[kMaxNz][kColTX], salpha[kMaxNz][kColTX], sgamma[kMaxNz][kColTX], sph[kMaxNz][kColTX];
  __shared__ float swd[kMaxNz][kColTX];
  __shared__ float pdnw[kMaxNz], prdnw[kMaxNz], prdn[kMaxNz], pfnm[kMaxNz], pfnp[kMaxNz];
  __shared__ float smuave[kColTX], smuts[kColTX], smu[kColTX];
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
  const int lev = g.ny * nx;
  for (int e = threadIdx.x; e < nz; e += kColTX * kColKT) {
    pdnw[e] = __ldg(&s[WF_DNW][e]);
    prdnw[e] = __ldg(&s[WF_RDNW][e]);
    prdn[e] = __ldg(&s[WF_RDN][e]);
    pfnm[e] = __ldg(&s[WF_FNM][e]);
    pfnp[e] = __ldg(&s[WF_FNP][e]);
  }
  float* t = s[WF_T];
  const float* ft = s[WF_T_TEND];
  const float* t1 = s[WF_T_SAVE];
  float* ww = s[WF_WW];
  const float* ww1 = s[WF_WW1];
  const float* u = s[WF_U];
  const float* v = s[WF_V];
  const float msftx = col ? __ldg(&s[WF_MSFTX][c]) : 1.f, msfty = col ? __ldg(&s[WF_MSFTY][c]) : 1.f;
  const float mut = col ? __ldg(&s[WF_MUT][c]) : 1.f;
  const float mu_tend = col ? __ldg(&s[WF_MU_TEND][c]) : 0.f;
  const float r_msfty = __frcp_rn(msfty), r_mut = __frcp_rn(mut);
  const float ep = g.epssm;
  const float ep1 = (float)(1.0 + (double)ep), em1 = (float)(1.0 - (double)ep);
#ifndef WRF_COL_NOPREFETCH
  // Ask L2 for what the later phases of this thread's levels will load: the
  // requests need no registers, and the phases after the column sweeps then
  // find their operands in L2 instead of waiting on DRAM one phase at a time.
  if (col) {
    auto pf = [](const float* a) { asm volatile("prefetch.global.L2 [%0];" ::"l"(a)); };
    const float* fields[] = {ww1, ww, t1, t, ft, s[WF_PH], s[WF_A], s[WF_ALPHA], s[WF_GAMMA], s[WF_PH_SAVE],
                             s[WF_PHB], s[WF_PH_TEND], s[WF_W], s[WF_RW_TEND], s[WF_C2A], s[WF_ALT], s[WF_CQW],
                             s[WF_W_SAVE], s[WF_PM1], s[WF_RU_M], s[WF_RV_M], s[WF_WW_M]};
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= nz) continue;
      const int p = k * lev + c;
#pragma unroll
      for (const float* f : fields) pf(f + p);
      if (inner) {
        pf(t1 + p + nx);
        pf(t1 + p - nx);
        pf(v + p + nx);
      }
    }
  }
#endif

  // --- A: horizontal mass-flux divergence per level (inner) / spec t, mu, muts
  if (inner) {
    const float* u1 = s[WF_U_SAVE];
    const float* v1 = s[WF_V_SAVE];
    const float muvn = __ldg(&s[WF_MUV][c + nx]), mvin = __ldg(&s[WF_MSFVX_INV][c + nx]);
    const float muv0 = __ldg(&s[WF_MUV][c]), mvi0 = __ldg(&s[WF_MSFVX_INV][c]);
    const float muup = __ldg(&s[WF_MUU][c + 1]), mfup = __ldg(&s[WF_MSFUY][c + 1]);
    const float muu0 = __ldg(&s[WF_MUU][c]), mfu0 = __ldg(&s[WF_MSFUY][c]);
    const float r_mfup = __frcp_rn(mfup), r_mfu0 = __frcp_rn(mfu0);
    const float rdx = g.rdx, rdy = g.rdy;
    float vn[NQ], v1n[NQ], v0[NQ], v10[NQ], ue[NQ], u1e[NQ], u0[NQ], u10[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= kend) continue;
      const int p = k * lev + c;
      vn[q] = __ldg(&v[p + nx]);
      v1n[q] = __ldg(&v1[p + nx]);
      v0[q] = __ldg(&v[p]);
      v10[q] = __ldg(&v1[p]);
      ue[q] = __ldg(&u[p + 1]);
      u1e[q] = __ldg(&u1[p + 1]);
      u0[q] = __ldg(&u[p]);
      u10[q] = __ldg(&u1[p]);
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= kend) continue;
      sdw[k][tx] = msftx * msfty *
                   (rdy * ((vn[q] + muvn * v1n[q] * mvin) - (v0[q] + muv0 * v10[q] * mvi0)) +
                    rdx * ((ue[q] + divc(muup * u1e[q], mfup, r_mfup)) - (u0[q] + divc(muu0 * u10[q], mfu0, r_mfu0))));
    }
  } else if (spec) {
    for (int k = tk; k < kend; k += kColKT) {
      const int p = k * lev + c;
      t[p] = t[p] + dts * __ldg(&ft[p]);
    }
    if (tk == 0) {
      const float mu = s[WF_MU][c] + dts * mu_tend;
      const float muts = s[WF_MUTS][c] + dts * mu_tend;
      s[WF_MU][c] = mu;
      s[WF_MUTS][c] = muts;
      smu[tx] = mu;
      smuts[tx] = muts;
    }
  }
  __syncthreads();
  // --- B: column mass tendency (sequential sum, reference order)
  if (inner && tk == 0) {
    float dmdt = 0.f;
#pragma unroll 8
    for (int k = 0; k < kend; ++k) dmdt = dmdt + pdnw[k] * sdw[k][tx];
    float mu = s[WF_MU][c];
    const float muave_old = mu;
    mu = mu + dts * (dmdt + mu_tend);
    const float muts = mut + mu;
    const float muave = 0.5f * (ep1 * mu + em1 * muave_old);
    s[WF_MU][c] = mu;
    s[WF_MUDF][c] = dmdt + mu_tend;
    s[WF_MUTS][c] = muts;
    s[WF_MUAVE][c] = muave;
    smu[tx] = mu;
    smuts[tx] = muts;
    smuave[tx] = muave;
    swd[0][tx] = dmdt;  // broadcast dmdt to the level threads
  }
  __syncthreads();
  // --- B2: increments of the ww scan in parallel, then the scan itself
  if (inner) {
    const float dmdt = swd[0][tx];
    for (int k = tk + 1; k < kend; k += kColKT)
      sww[k][tx] = divc(pdnw[k - 1] * (dmdt + sdw[k - 1][tx] + mu_tend), msfty, r_msfty);
  }
  __syncthreads();
  if (inner && tk == 0) {
    float wprev = ww[c];
    sww[0][tx] = wprev;
#pragma unroll 8
    for (int k = 1; k < kend; ++k) {
      wprev = wprev - sww[k][tx];
      sww[k][tx] = wprev;
    }
  }
  __syncthreads();
  // --- C: final ww (inner: scan - ww1)
  if (col) {
    float wv[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k < nz) wv[q] = (inner && k < kend) ? __ldg(&ww1[k * lev + c]) : ww[k * lev + c];
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= nz) continue;
      float w = wv[q];
      if (inner && k < kend) {
        w = sww[k][tx] - w;
        ww[k * lev + c] = w;
      }
      sww[k][tx] = w;
    }
  }
  __syncthreads();
  const float muave = inner ? smuave[tx] : 0.f;
  const float muts = mass ? smuts[tx] : 1.f;
  const float r_muts = __frcp_rn(muts);
  // --- C2: potential temperature and t_2ave; D1: wdwn, phi, coefficients
  if (inner) {
    const float cy = (float)(0.5 * g.rdyd), cx = (float)(0.5 * g.rdxd);
    float* t2a = s[WF_T_2SAVE];
    float t10[NQ], tup[NQ], tdn[NQ], told[NQ], ftk[NQ], vn[NQ], tn[NQ], v0[NQ], ts[NQ], ue[NQ], te[NQ], u0[NQ],
        tw[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= kend) continue;
      const int p = k * lev + c;
      t10[q] = __ldg(&t1[p]);
      tup[q] = (k + 1 == nz - 1) ? 0.f : __ldg(&t1[p + lev]);
      tdn[q] = (k == 0) ? 0.f : __ldg(&t1[p - lev]);
      told[q] = t[p];
      ftk[q] = __ldg(&ft[p]);
      vn[q] = __ldg(&v[p + nx]);
      tn[q] = __ldg(&t1[p + nx]);
      v0[q] = __ldg(&v[p]);
      ts[q] = __ldg(&t1[p - nx]);
      ue[q] = __ldg(&u[p + 1]);
      te[q] = __ldg(&t1[p + 1]);
      u0[q] = __ldg(&u[p]);
      tw[q] = __ldg(&t1[p - 1]);
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= kend) continue;
      const int p = k * lev + c;
      // wdtn(kk) = ww(kk) (fnm t1(kk) + fnp t1(kk-1)), zero at the bottom and top
      const float wup = (k + 1 == nz - 1) ? 0.f : sww[k + 1][tx] * (pfnm[k + 1] * tup[q] + pfnp[k + 1] * t10[q]);
      const float wdn = (k == 0) ? 0.f : sww[k][tx] * (pfnm[k] * t10[q] + pfnp[k] * tdn[q]);
      float tt = told[q] + msfty * dts * ftk[q];
      const float hy = cy * (vn[q] * (tn[q] + t10[q]) - v0[q] * (t10[q] + ts[q]));
      const float hx = cx * (ue[q] * (te[q] + t10[q]) - u0[q] * (t10[q] + tw[q]));
      tt = tt - dts * msfty * (msftx * (hy + hx) + prdnw[k] * (wup - wdn));
      t[p] = tt;
      float av = 0.5f * (ep1 * tt + em1 * told[q]);
      av = (av + muave * (float)T0) / (muts * ((float)T0 + t10[q]));
      t2a[p] = av;
      st2av[k][tx] = av;
    }
    const float* ph1 = s[WF_PH_SAVE];
    const float* phb = s[WF_PHB];
    float phv[NQ], av[NQ], alv[NQ], gav[NQ], p1[NQ], p1m[NQ], pb[NQ], pbm[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= nz) continue;
      const int p = k * lev + c;
      phv[q] = s[WF_PH][p];
      av[q] = __ldg(&s[WF_A][p]);
      alv[q] = __ldg(&s[WF_ALPHA][p]);
      gav[q] = __ldg(&s[WF_GAMMA][p]);
      if (k >= 1 && k <= kend) {
        p1[q] = __ldg(&ph1[p]);
        p1m[q] = __ldg(&ph1[p - lev]);
        pb[q] = __ldg(&phb[p]);
        pbm[q] = __ldg(&phb[p - lev]);
      }
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= nz) continue;
      sph[k][tx] = phv[q];
      sa[k][tx] = av[q];
      salpha[k][tx] = alv[q];
      sgamma[k][tx] = gav[q];
      // wdwn(k) = 0.5 (ww(k) + ww(k-1)) rdnw(k-1) (ph1(k) - ph1(k-1) + phb(k) - phb(k-1))
      if (k >= 1 && k <= kend)
        swd[k][tx] = 0.5f * (sww[k][tx] + sww[k - 1][tx]) * prdnw[k - 1] * (p1[q] - p1m[q] + pb[q] - pbm[q]);
    }
  }
  __syncthreads();
  // --- D2: right-hand side of the phi equation (inner)
  if (inner) {
    const float cw = (float)(0.5 * G * (1.0 - (double)ep));
    float ptv[NQ], wv[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k < 1 || k >= nz) continue;
      ptv[q] = __ldg(&s[WF_PH_TEND][k * lev + c]);
      wv[q] = s[WF_W][k * lev + c];
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= nz) continue;
      if (k == 0) {
        srhs[0][tx] = 0.f;
        continue;
      }
      float r = dts * (ptv[q] + cw * wv[q]);
      if (k < kend) r = r - dts * (pfnm[k] * swd[k + 1][tx] + pfnp[k] * swd[k][tx]);
      srhs[k][tx] = sph[k][tx] + divc(msfty * r, mut, r_mut);
    }
  }
  __syncthreads();
  // --- E: explicit part of w (inner)
  if (inner) {
    const float* c2a = s[WF_C2A];
    const float* alt = s[WF_ALT];
    const float msft_inv = 1.0f / msfty;
    const float cp = (float)(0.5 * (double)dts * G);
    const float cq = (float)((double)dts * G);
    if (tk == 0) {  // lower boundary: w from the terrain slope and near-surface winds
      const float* ht = s[WF_HT];
      auto cv = [&](int cc) { return g.cf1 * __ldg(&v[cc]) + g.cf2 * __ldg(&v[lev + cc]) + g.cf3 * __ldg(&v[2 * lev + cc]); };
      auto cu = [&](int cc) { return g.cf1 * __ldg(&u[cc]) + g.cf2 * __ldg(&u[lev + cc]) + g.cf3 * __ldg(&u[2 * lev + cc]); };
      const float h0 = __ldg(&ht[c]);
      sdw[0][tx] = msfty * 0.5f * g.rdy * ((__ldg(&ht[c + nx]) - h0) * cv(c + nx) + (h0 - __ldg(&ht[c - nx])) * cv(c)) +
                   msftx * 0.5f * g.rdx * ((__ldg(&ht[c + 1]) - h0) * cu(c + 1) + (h0 - __ldg(&ht[c - 1])) * cu(c));
    }
    float wkv[NQ], rwv[NQ], c2mv[NQ], almv[NQ], c2kv[NQ], alkv[NQ], cqv[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k < 1 || k > kend) continue;
      const int p = k * lev + c;
      wkv[q] = s[WF_W][p];
      rwv[q] = __ldg(&s[WF_RW_TEND][p]);
      c2mv[q] = __ldg(&c2a[p - lev]);
      almv[q] = __ldg(&alt[p - lev]);
      if (k < kend) {
        c2kv[q] = __ldg(&c2a[p]);
        alkv[q] = __ldg(&alt[p]);
        cqv[q] = __ldg(&s[WF_CQW][p]);
      }
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k < 1 || k > kend) continue;
      const float wk = wkv[q], rwk = rwv[q];
      const float c2m = c2mv[q], alm = almv[q];
      const float rdnw_m = prdnw[k - 1];
      float wl;
      if (k < kend) {
        const float c2k = c2kv[q], alk = alkv[q];
        const float X1 = divc(c2k * prdnw[k], mut, r_mut) * (ep1 * (srhs[k + 1][tx] - srhs[k][tx]) + em1 * (sph[k + 1][tx] - sph[k][tx]));
        const float X2 = divc(c2m * rdnw_m, mut, r_mut) * (ep1 * (srhs[k][tx] - srhs[k - 1][tx]) + em1 * (sph[k][tx] - sph[k - 1][tx]));
        wl = wk + dts * rwk + msft_inv * cqv[q] * (cp * prdn[k] * (X1 - X2)) +
             cq * msft_inv * (prdn[k] * (c2k * alk * st2av[k][tx] - c2m * alm * st2av[k - 1][tx]) - muave);
      } else {
        const float cm = (float)(-0.5 * (double)dts * G);
        wl = wk + dts * rwk +
             msft_inv * (divc(cm, mut, r_mut) * (rdnw_m * rdnw_m) * 2.0f * c2m *
                             (ep1 * (srhs[kend][tx] - srhs[kend - 1][tx]) + em1 * (sph[kend][tx] - sph[kend - 1][tx])) -
                         cq * (2.0f * rdnw_m * c2m * alm * st2av[kend - 1][tx] + muave));
      }
      sdw[k][tx] = wl;
    }
  }
  __syncthreads();
  // --- F: Thomas sweeps (sequential per column)
  if (inner && tk == 0) {
    float prev = sdw[0][tx];
#pragma unroll 8
    for (int k = 1; k <= kend; ++k) {
      prev = (sdw[k][tx] - sa[k][tx] * prev) * salpha[k][tx];
      sdw[k][tx] = prev;
    }
#pragma unroll 8
    for (int k = kend - 1; k >= 1; --k) {
      prev = sdw[k][tx] - sgamma[k][tx] * prev;
      sdw[k][tx] = prev;
    }
  }
  __syncthreads();
  // --- G: Rayleigh damping, w and phi (inner); spec phi; sumflux (all)
  float* ph = s[WF_PH];
  if (inner) {
    float* w = s[WF_W];
    const float* ph1 = s[WF_PH_SAVE];
    const float* phb = s[WF_PHB];
    const float gf = (float)G;
    constexpr float r_g = 1.0f / (float)G, r_hd = 1.0f / 5000.0f;
    const float hdepth = 5000.0f;
    const float dampmag = (float)((double)dts * 0.2);
    const float htop = divc(__ldg(&ph1[kend * lev + c]) + __ldg(&phb[kend * lev + c]), gf, r_g);
    const float hbot = htop - hdepth;
    const float hpi = (float)(0.5 * 3.14159265359);
    float p1v[NQ], pbv[NQ], wsv[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k < 1 || k >= nz) continue;
      const int p = k * lev + c;
      p1v[q] = __ldg(&ph1[p]);
      pbv[q] = __ldg(&phb[p]);
      wsv[q] = __ldg(&s[WF_W_SAVE][p]);
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= nz) continue;
      const int p = k * lev + c;
      if (k == 0) {
        w[c] = sdw[0][tx];
        continue;
      }
      const float hk = divc(p1v[q] + pbv[q], gf, r_g);
      float dwd = 0.f;
      if (hk >= hbot) {
        const float sn = sinf(divc(hpi * (hk - hbot), hdepth, r_hd));
        dwd = dampmag * (sn * sn);
      }
      const float num = sdw[k][tx] - dwd * mut * wsv[q];
      const float wk = dwd == 0.f ? num : num / (1.0f + dwd);  // x / 1 == x
      w[p] = wk;
      const float phk = srhs[k][tx] + divc(msfty * 0.5f * dts * gf * ep1 * wk, muts, r_muts);
      ph[p] = phk;
      sph[k][tx] = phk;
    }
  } else if (spec) {
    const float mu_old = muts - dts * mu_tend;
    const float* ph_save = s[WF_PH_SAVE];
    const float* ph_tend = s[WF_PH_TEND];
    float phv[NQ], ptv[NQ], psv[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= nz) continue;
      const int p = k * lev + c;
      phv[q] = ph[p];
      ptv[q] = __ldg(&ph_tend[p]);
      psv[q] = __ldg(&ph_save[p]);
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= nz) continue;
      const int p = k * lev + c;
      const float phk = divc(phv[q] * mu_old, muts, r_muts) + divc(dts * ptv[q], muts, r_muts) +
                        psv[q] * (divc(mu_old, muts, r_muts) - 1.0f);
      ph[p] = phk;
      sph[k][tx] = phk;
    }
  }
  if (col) {
    float* ru_m = s[WF_RU_M];
    float* rv_m = s[WF_RV_M];
    float* ww_m = s[WF_WW_M];
    const bool ur = j < jde - 1, vr = i < ide - 1, wr = ur && vr;
    const bool last = iteration == nsub;
    const float muuc = last && ur ? __ldg(&s[WF_MUU][c]) : 0.f, mfuc = last && ur ? __ldg(&s[WF_MSFUY][c]) : 1.f;
    const float muvc = last && vr ? __ldg(&s[WF_MUV][c]) : 0.f, mvic = last && vr ? __ldg(&s[WF_MSFVX_INV][c]) : 0.f;
    const float r_nsub = __frcp_rn((float)nsub), r_mfuc = __frcp_rn(mfuc);
    float am[NQ], bm[NQ], cm[NQ], uv[NQ], vv[NQ], us[NQ], vs[NQ], w1[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= nz) continue;
      const int p = k * lev + c;
      am[q] = iteration == 1 ? 0.f : ru_m[p];
      bm[q] = iteration == 1 ? 0.f : rv_m[p];
      cm[q] = iteration == 1 ? 0.f : ww_m[p];
      const bool lv = k < nz - 1;
      uv[q] = lv && ur ? __ldg(&u[p]) : 0.f;
      vv[q] = lv && vr ? __ldg(&v[p]) : 0.f;
      us[q] = last && lv && ur ? __ldg(&s[WF_U_SAVE][p]) : 0.f;
      vs[q] = last && lv && vr ? __ldg(&s[WF_V_SAVE][p]) : 0.f;
      w1[q] = last && wr ? __ldg(&ww1[p]) : 0.f;
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= nz) continue;
      const int p = k * lev + c;
      float a = am[q], b = bm[q], cc = cm[q];
      if (k < nz - 1 && ur) a = a + uv[q];
      if (k < nz - 1 && vr) b = b + vv[q];
      if (wr) cc = cc + sww[k][tx];
      if (last) {
        if (k < nz - 1 && ur) a = divc(a, (float)nsub, r_nsub) + divc(muuc * us[q], mfuc, r_mfuc);
        if (k < nz - 1 && vr) b = divc(b, (float)nsub, r_nsub) + muvc * vs[q] * mvic;
        if (wr) cc = divc(cc, (float)nsub, r_nsub) + w1[q];
      }
      ru_m[p] = a;
      rv_m[p] = b;
      ww_m[p] = cc;
    }
  }
  __syncthreads();
  // --- H: calc_p_rho with divergence damping (mass columns)
  if (mass) {
    const float mu = smu[tx];
    float* al = s[WF_AL];
    float* pp = s[WF_P];
    float* pm1 = s[WF_PM1];
    float altv[NQ], t1v[NQ], c2v[NQ], tv[NQ], pmv[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= kend) continue;
      const int p = k * lev + c;
      altv[q] = __ldg(&s[WF_ALT][p]);
      t1v[q] = __ldg(&t1[p]);
      c2v[q] = __ldg(&s[WF_C2A][p]);
      tv[q] = t[p];
      pmv[q] = pm1[p];
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int k = tk + q * kColKT;
      if (k >= kend) continue;
      const int p = k * lev + c;
      const float alk = -r_muts * (altv[q] * mu + prdnw[k] * (sph[k + 1][tx] - sph[k][tx]));
      al[p] = alk;
      const float pnew = c2v[q] * (altv[q] * (tv[q] - mu * t1v[q]) / (muts * ((float)T0 + t1v[q])) - alk);
      pp[p] = pnew + g.smdiv * (pnew - pmv[q]);
      pm1[p] = pnew;
    }
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

// operands first, then the stores (a store would hold back the later
// fields' loads)
__global__ void k_ssfinish(Grid g, S s, float dts, int nsub, int rk_step) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nz = g.nz;
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const bool dv = k < nz - 1 && j >= jts && j < jev && i >= its && i < ime;
  const bool du = k < nz - 1 && j >= jts && j < jme && i >= its && i < ieu;
  const bool m3 = j >= jts && j < jme && i >= its && i < ime;
  float vv = 0.f, vs = 0.f, mfvx = 0.f, muv = 0.f, muvs = 1.f;
  if (dv) {
    vv = s[WF_V][p];
    vs = s[WF_V_SAVE][p];
    mfvx = s[WF_MSFVX][c];
    muv = s[WF_MUV][c];
    muvs = s[WF_MUVS][c];
  }
  float uu = 0.f, us = 0.f, mfuy = 0.f, muu = 0.f, muus = 1.f;
  if (du) {
    uu = s[WF_U][p];
    us = s[WF_U_SAVE][p];
    mfuy = s[WF_MSFUY][c];
    muu = s[WF_MUU][c];
    muus = s[WF_MUUS][c];
  }
  float mut = 0.f, muts = 1.f, mfty = 0.f, ww = 0.f, wsv = 0.f, phv = 0.f, phs = 0.f, wwv = 0.f, ww1 = 0.f;
  float tv = 0.f, ts = 0.f, hd = 0.f, muv0 = 0.f, mus0 = 0.f;
  if (m3) {
    mut = s[WF_MUT][c];
    muts = s[WF_MUTS][c];
    mfty = s[WF_MSFTY][c];
    ww = s[WF_W][p];
    wsv = s[WF_W_SAVE][p];
    phv = s[WF_PH][p];
    phs = s[WF_PH_SAVE][p];
    wwv = s[WF_WW][p];
    ww1 = s[WF_WW1][p];
    if (k < nz - 1) {
      tv = s[WF_T][p];
      ts = s[WF_T_SAVE][p];
      if (rk_step == 3) hd = s[WF_H_DIABATIC][p];
    }
    if (k == 0) {
      muv0 = s[WF_MU][c];
      mus0 = s[WF_MU_SAVE][c];
    }
  }
  if (dv) s[WF_V][p] = (mfvx * vv + vs * muv) / muvs;
  if (du) s[WF_U][p] = (mfuy * uu + us * muu) / muus;
  if (m3) {
    s[WF_W][p] = (mfty * ww + wsv * mut) / muts;
    s[WF_PH][p] = phv + phs;
    s[WF_WW][p] = wwv + ww1;
    if (k < nz - 1) {
      if (rk_step < 3)
        s[WF_T][p] = (tv + ts * mut) / muts;
      else
        s[WF_T][p] = (tv - (float)((double)dts * nsub) * mut * hd + ts * mut) / muts;
    }
    if (k == 0) s[WF_MU][c] = muv0 + mus0;
  }
}

int launch_small_step_prep(const Grid& g, const S& s, int rk_step, float dts, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  k_ssp2d<<<col_grid(g, b2), b2, 0, st>>>(g, s, rk_step);
  k_ssp3d<<<point_grid(g, b3), b3, 0, st>>>(g, s, rk_step);
  k_p_rho0<<<point_grid(g, b3), b3, 0, st>>>(g, s);
  if (kernel_form() == WRF_FORM_FAST) {
    const dim3 bc(32, 4);
    k_coef_w_col<<<dim3((g.ide - 1 - g.ids + 31) / 32, (g.jde - 1 - g.jds + 3) / 4), bc, 0, st>>>(g, s, dts);
  } else {
    k_coef_w<<<dim3((g.ide - 1 - g.ids + kCwTX - 1) / kCwTX, g.jde - 1 - g.jds), kCwTX * kCwKT, 0, st>>>(g, s, dts);
  }
  return 4;
}

// small_step_prep alone (the step's k_ssp2d and k_ssp3d)
int launch_ssp_only(const Grid& g, const S& s, int rk_step, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  k_ssp2d<<<col_grid(g, b2), b2, 0, st>>>(g, s, rk_step);
  k_ssp3d<<<point_grid(g, b3), b3, 0, st>>>(g, s, rk_step);
  return 2;
}

int launch_coef_w(const Grid& g, const float* mut, const float* cqw, const float* c2a, const float* rdn,
                  const float* rdnw, float dts, float* a, float* alpha, float* gamma, cudaStream_t st) {
  S s{};
  s.f[WF_MUT] = const_cast<float*>(mut);
  s.f[WF_CQW] = const_cast<float*>(cqw);
  s.f[WF_C2A] = const_cast<float*>(c2a);
  s.f[WF_RDN] = const_cast<float*>(rdn);
  s.f[WF_RDNW] = const_cast<float*>(rdnw);
  s.f[WF_A] = a;
  s.f[WF_ALPHA] = alpha;
  s.f[WF_GAMMA] = gamma;
  k_coef_w<<<dim3((g.ide - 1 - g.ids + kCwTX - 1) / kCwTX, g.jde - 1 - g.jds), kCwTX * kCwKT, 0, st>>>(g, s, dts);
  return 1;
}

int launch_advance_uv(const Grid& g, const S& s, float dts, cudaStream_t st) {
  if (kernel_form() == WRF_FORM_FAST && g.nx % 4 == 0 && g.nz >= 4) {
    UvTmaArgs a{};
    const char* err = nullptr;
    const int f[6] = {WF_ALT, WF_AL, WF_PB, WF_PHP, WF_PH, WF_P};
    CUtensorMap* m[6] = {&a.alt, &a.al, &a.pb, &a.php, &a.ph, &a.pp};
    bool ok = true;
    for (int e = 0; e < 6 && ok; ++e) ok = tma::encode_f32_4d(m[e], s[f[e]], g.nx, g.ny, g.nz, 1, kUvBW, kUvBH, &err);
    const int fo[kUvNO] = {WF_U, WF_RU_TEND, WF_V, WF_RV_TEND, WF_CQU, WF_CQV};
    for (int e = 0; e < kUvNO && ok; ++e)
      ok = tma::encode_f32_4d(&a.own[e], s[fo[e]], g.nx, g.ny, g.nz, 1, kUvOW, kUvOH, &err);
    if (ok) {
      a.nchunk = min((g.nz - 1 + kUvKCH - 1) / kUvKCH, g.nz - 1);
      const dim3 gr((g.ide + 1 - g.ids + kUvTX - 1) / kUvTX, (g.jde - g.jds + kUvTY - 1) / kUvTY, a.nchunk);
      k_advance_uv_tma<<<gr, dim3(kUvTX, kUvTY), 0, st>>>(g, s, dts, a);
      return 1;
    }
  }
  const dim3 b3(32, 4);
  k_advance_uv<<<point_grid(g, b3), b3, 0, st>>>(g, s, dts);
  return 1;
}

int launch_acoustic_col(const Grid& g, const S& s, float dts, int iteration, int nsub, cudaStream_t st) {
  const dim3 gc((g.ide - g.ids + kColTX - 1) / kColTX, g.jde - g.jds);
  if (g.nz <= 3 * kColKT)
    k_acoustic_col<3><<<gc, kColTX * kColKT, 0, st>>>(g, s, dts, iteration, nsub);
  else
    k_acoustic_col<4><<<gc, kColTX * kColKT, 0, st>>>(g, s, dts, iteration, nsub);
  return 1;
}


int launch_small_step_finish(const Grid& g, const S& s, float dts, int nsub, int rk_step, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  k_mu_uv_1<<<col_grid(g, b2), b2, 0, st>>>(g, s);
  k_ssfinish<<<point_grid(g, b3), b3, 0, st>>>(g, s, dts, nsub, rk_step);
  return 2;
}

}  // namespace wrf
