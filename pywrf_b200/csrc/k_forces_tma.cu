// Large-step forces, tensor-map form: rhs_ph, horizontal_pressure_gradient,
// pg_buoy_w, coriolis and curvature (wrf_dynamics.py:2031-2620), for arrays
// whose rows are a multiple of 16 bytes.  The operations and their order are
// those of k_forces (k_tend.cu), which stays as the point form.
//
// A block of 32 x 8 threads owns 32 x 8 columns and a chunk of levels.  Per
// level one thread loads boxes of ph and phb with a 3-cell halo (44 x 14 from
// x = floor4(i0 - 3), y = j0 - 3: rhs_ph's 6th-order differences) and of u,
// v, ru, rv, rw, alt, al, pb, php and p (40 x 10 from floor4(i0 - 1), j0 - 1:
// every i-1, i+1, j-1, j+1 neighbour) into a ring of three levels: levels k
// and k+1 are read while k+2 loads.  The values of level k-1 that level k
// uses (u, v, ru, rv at the two points each formula takes, the column's p)
// and the vertical averages wdwn(k) and dpn(k) are carried up the column in
// registers; the thread's own tendencies and coefficients are loaded a level
// ahead.  Every wait is bounded; a block whose wait runs out drains its copies
// and adds 1 to STATUS[WRF_ST_WAIT].
#include "kernels.cuh"
#include "tma.cuh"

namespace wrf {
namespace {

constexpr int kFTX = 32, kFTY = 8;
constexpr int kFQW = 44, kFQH = kFTY + 6;  // ph, phb
constexpr int kFMW = 40, kFMH = kFTY + 2;  // the other fields
constexpr int kFQSlot = 640, kFMSlot = 416;
constexpr int kFNM = 10;
enum { FM_U, FM_V, FM_RU, FM_RV, FM_RW, FM_ALT, FM_AL, FM_PB, FM_PHP, FM_PP };
constexpr int kFSlot = 2 * kFQSlot + kFNM * kFMSlot;  // floats per level
constexpr int kFRing = 3, kFKCH = 7;
constexpr uint32_t kFBytes = 2 * kFQW * kFQH * 4 + kFNM * kFMW * kFMH * 4;
constexpr long long kFWaitCycles = 4000000000LL;
static_assert(kFQW * kFQH <= kFQSlot && kFMW * kFMH <= kFMSlot, "a slot holds one box");
static_assert((kFQSlot * 4) % 128 == 0 && (kFMSlot * 4) % 128 == 0, "slots keep boxes 128-byte aligned");

struct ForcesTmaArgs {
  CUtensorMap ph, phb;
  CUtensorMap m[kFNM];
  int nchunk;
};

// 45 (a[1] - a[-1]) - 9 (a[2] - a[-2]) + (a[3] - a[-3]) with stride st
__device__ __forceinline__ float d6s(const float* a, int st) {
  return 45.0f * (a[st] - a[-st]) - 9.0f * (a[2 * st] - a[-2 * st]) + (a[3 * st] - a[-3 * st]);
}

#ifndef WRF_FORCES_MINB
#define WRF_FORCES_MINB 2
#endif
__global__ void __launch_bounds__(kFTX * kFTY, WRF_FORCES_MINB) k_forces_tma(Grid g, S s, const __grid_constant__ ForcesTmaArgs a) {
  extern __shared__ float fsm_raw[];
  float* ring = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(fsm_raw) + 127) & ~uintptr_t(127));
  __shared__ uint64_t bar[kFRing];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kFTX + tx;
  const int nx = g.nx, ny = g.ny, nz = g.nz, ktf = nz - 1;
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const int i0 = ids + blockIdx.x * kFTX, j0 = jds + blockIdx.y * kFTY;
  const int i = i0 + tx, j = j0 + ty;
  const int qx = (i0 - 3) & ~3, mx = (i0 - 1) & ~3;
  const int oq = i0 - 3 - qx, om = i0 - mx;
  const int k0 = blockIdx.z * nz / a.nchunk, k1 = (blockIdx.z + 1) * nz / a.nchunk;
  const int khi = min(k1, nz - 1);  // highest level loaded (k+1 of the chunk's last level)
  const size_t lev = (size_t)ny * nx;
  const bool mass = j >= jds && j < jde - 1 && i >= ids && i < ide - 1;
  const bool uc = j >= jds && j < jde - 1 && i >= ids + 1 && i < ide - 1;
  const bool vc = j >= jds + 1 && j < jde - 1 && i >= ids && i < ide - 1;
  const int c = min(j, ny - 1) * nx + min(i, nx - 1);
  const float gf = (float)G, rdx = g.rdx, rdy = g.rdy, rr = (float)RERADIUS;
  const float* fnm = s[WF_FNM];
  const float* fnp = s[WF_FNP];
  const float* rdnw = s[WF_RDNW];
  const float* rdn = s[WF_RDN];

  if (tid == 0) {
    for (int r = 0; r < kFRing; ++r) tma::mbar_init(&bar[r], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto slot_base = [&](int r) { return ring + r * kFSlot; };
  auto issue = [&](int L, int r) {
    float* d = slot_base(r);
    tma::mbar_expect_tx(&bar[r], kFBytes);
    tma::load_4d(d, &a.ph, qx, j0 - 3, L, 0, &bar[r]);
    tma::load_4d(d + kFQSlot, &a.phb, qx, j0 - 3, L, 0, &bar[r]);
    for (int f = 0; f < kFNM; ++f) tma::load_4d(d + 2 * kFQSlot + f * kFMSlot, &a.m[f], mx, j0 - 1, L, 0, &bar[r]);
  };
  int hi = k0 - 1;
  if (tid == 0) {
    for (int L = k0; L <= min(k0 + 1, khi); ++L) issue(L, L - k0);
    hi = min(k0 + 1, khi);
  }

  // ---- per-column constants, in the association order of k_forces
  float msfty = 1.f, mut = 0.f, mub = 0.f, mu_c = 0.f;
  float muv_c = 0.f, muv_n = 0.f, mvy_c = 0.f, mvy_n = 0.f, muu_c = 0.f, muu_e = 0.f, mux_c = 0.f, mux_e = 0.f;
  float e_c = 0.f, cosa_c = 0.f, sina_c = 0.f, rmt = 0.f, rm = 1.f;
  if (mass) {
    msfty = __ldg(&s[WF_MSFTY][c]);
    mut = __ldg(&s[WF_MUT][c]);
    mub = __ldg(&s[WF_MUB][c]);
    mu_c = __ldg(&s[WF_MU][c]);
    muv_c = __ldg(&s[WF_MUV][c]);
    muv_n = __ldg(&s[WF_MUV][c + nx]);
    mvy_c = __ldg(&s[WF_MSFVY][c]);
    mvy_n = __ldg(&s[WF_MSFVY][c + nx]);
    muu_c = __ldg(&s[WF_MUU][c]);
    muu_e = __ldg(&s[WF_MUU][c + 1]);
    mux_c = __ldg(&s[WF_MSFUX][c]);
    mux_e = __ldg(&s[WF_MSFUX][c + 1]);
    e_c = __ldg(&s[WF_E][c]);
    cosa_c = __ldg(&s[WF_COSA][c]);
    sina_c = __ldg(&s[WF_SINA][c]);
    rmt = __ldg(&s[WF_MSFTX][c]) / msfty;
    rm = 1.0f / msfty;
  }
  // the x / y gradient terms of the metric (vx in k_forces) for the column and
  // its west (u) or south (v) neighbour
  float dmx_c = 0.f, dmy_c = 0.f, dmx_w = 0.f, dmy_w = 0.f, dmx_s = 0.f, dmy_s = 0.f;
  float cpu = 0.f, cpu2 = 0.f, muav_u = 0.f, cu1 = 0.f, cu2 = 0.f;
  float cpv = 0.f, cpv2 = 0.f, muav_v = 0.f, cv1 = 0.f, cv2 = 0.f, r_v = 0.f;
  if (uc || vc) {
    const float* mfvx = s[WF_MSFVX];
    const float* mfuy = s[WF_MSFUY];
    dmx_c = __ldg(&mfvx[c + nx]) - __ldg(&mfvx[c]);
    dmy_c = __ldg(&mfuy[c + 1]) - __ldg(&mfuy[c]);
  }
  if (uc) {
    const float* mfvx = s[WF_MSFVX];
    const float* mfuy = s[WF_MSFUY];
    dmx_w = __ldg(&mfvx[c - 1 + nx]) - __ldg(&mfvx[c - 1]);
    dmy_w = __ldg(&mfuy[c]) - __ldg(&mfuy[c - 1]);
    const float r = __ldg(&s[WF_MSFUX][c]) / __ldg(&mfuy[c]);
    cpu = r * 0.5f * rdx * __ldg(&s[WF_MUU][c]);
    cpu2 = r * rdx;
    muav_u = 0.5f * (__ldg(&s[WF_MU][c - 1]) + __ldg(&s[WF_MU][c]));
    cu1 = r * 0.5f * (__ldg(&s[WF_F][c]) + __ldg(&s[WF_F][c - 1])) * 0.25f;
    cu2 = 0.5f * (__ldg(&s[WF_E][c]) + __ldg(&s[WF_E][c - 1])) * 0.5f *
          (__ldg(&s[WF_COSA][c]) + __ldg(&s[WF_COSA][c - 1])) * 0.25f;
  }
  if (vc) {
    const float* mfvx = s[WF_MSFVX];
    const float* mfuy = s[WF_MSFUY];
    dmx_s = __ldg(&mfvx[c]) - __ldg(&mfvx[c - nx]);
    dmy_s = __ldg(&mfuy[c - nx + 1]) - __ldg(&mfuy[c - nx]);
    r_v = __ldg(&s[WF_MSFVY][c]) / __ldg(&mfvx[c]);
    cpv = r_v * 0.5f * rdy * __ldg(&s[WF_MUV][c]);
    cpv2 = r_v * rdy;
    muav_v = 0.5f * (__ldg(&s[WF_MU][c - nx]) + __ldg(&s[WF_MU][c]));
    cv1 = r_v * 0.5f * (__ldg(&s[WF_F][c]) + __ldg(&s[WF_F][c - nx])) * 0.25f;
    cv2 = r_v * 0.5f * (__ldg(&s[WF_E][c]) + __ldg(&s[WF_E][c - nx])) * 0.5f *
          (__ldg(&s[WF_SINA][c]) + __ldg(&s[WF_SINA][c - nx])) * 0.25f;
  }

  // ---- values of level k0-1 and the vertical averages at k0
  const int cw = uc ? c - 1 : c, cs = vc ? c - nx : c;
  float u_c = 0.f, u_e = 0.f, v_c = 0.f, v_n = 0.f, ru_c = 0.f, ru_e = 0.f, rv_c = 0.f, rv_n = 0.f, p_c = 0.f;
  float dpn_u = 0.f, dpn_v = 0.f, wdwn = 0.f, ww_c = 0.f;
  {
    const float* pp = s[WF_P];
    if (k0 >= 1 && (mass || uc || vc)) {
      const size_t q = (size_t)(k0 - 1) * lev;
      u_c = __ldg(&s[WF_U][q + c]);
      u_e = __ldg(&s[WF_U][q + c + 1]);
      v_c = __ldg(&s[WF_V][q + c]);
      v_n = __ldg(&s[WF_V][q + c + nx]);
      ru_c = __ldg(&s[WF_RU][q + c]);
      ru_e = __ldg(&s[WF_RU][q + c + 1]);
      rv_c = __ldg(&s[WF_RV][q + c]);
      rv_n = __ldg(&s[WF_RV][q + c + nx]);
      p_c = __ldg(&pp[q + c]);
    }
    if (uc || vc) {
      const size_t q = (size_t)k0 * lev;
      if (k0 == 0) {
        dpn_u = 0.5f * (g.cf1 * (__ldg(&pp[cw]) + __ldg(&pp[c])) + g.cf2 * (__ldg(&pp[lev + cw]) + __ldg(&pp[lev + c])) +
                        g.cf3 * (__ldg(&pp[2 * lev + cw]) + __ldg(&pp[2 * lev + c])));
        dpn_v = 0.5f * (g.cf1 * (__ldg(&pp[cs]) + __ldg(&pp[c])) + g.cf2 * (__ldg(&pp[lev + cs]) + __ldg(&pp[lev + c])) +
                        g.cf3 * (__ldg(&pp[2 * lev + cs]) + __ldg(&pp[2 * lev + c])));
      } else if (k0 < nz - 1) {
        const size_t qm = q - lev;
        const float fm = __ldg(&fnm[k0]), fp = __ldg(&fnp[k0]);
        dpn_u = 0.5f * (fm * (__ldg(&pp[q + cw]) + __ldg(&pp[q + c])) + fp * (__ldg(&pp[qm + cw]) + __ldg(&pp[qm + c])));
        dpn_v = 0.5f * (fm * (__ldg(&pp[q + cs]) + __ldg(&pp[q + c])) + fp * (__ldg(&pp[qm + cs]) + __ldg(&pp[qm + c])));
      }
    }
    if (mass) {
      const float* ww = s[WF_WW];
      const size_t q = (size_t)k0 * lev + c;
      ww_c = __ldg(&ww[q]);
      if (k0 >= 1 && k0 < nz - 1) {
        const size_t qm = q - lev;
        const float* ph = s[WF_PH];
        const float* phb = s[WF_PHB];
        wdwn = 0.5f * (ww_c + __ldg(&ww[qm])) * __ldg(&rdnw[k0 - 1]) *
               (__ldg(&ph[q]) - __ldg(&ph[qm]) + __ldg(&phb[q]) - __ldg(&phb[qm]));
      }
    }
  }
  // the thread's own values of a level
  struct Own {
    float pht, w, rut, cqu, rvt, cqv, rwt, cqw, ww1;  // ww1: ww at the level above
  };
  auto own = [&](int k, Own& o) {
    const size_t p = (size_t)k * lev + c;
    o.pht = (mass && k >= 1) ? s[WF_PH_TEND][p] : 0.f;
    o.w = (mass && k >= 1) ? __ldg(&s[WF_W][p]) : 0.f;
    o.rut = (uc && k < ktf) ? s[WF_RU_TEND][p] : 0.f;
    o.cqu = (uc && k < ktf) ? __ldg(&s[WF_CQU][p]) : 0.f;
    o.rvt = (vc && k < ktf) ? s[WF_RV_TEND][p] : 0.f;
    o.cqv = (vc && k < ktf) ? __ldg(&s[WF_CQV][p]) : 0.f;
    o.rwt = (mass && k >= 1) ? s[WF_RW_TEND][p] : 0.f;
    o.cqw = (mass && k >= 1 && k < nz - 1) ? s[WF_CQW][p] : 0.f;
    o.ww1 = (mass && k + 1 < nz) ? __ldg(&s[WF_WW][p + lev]) : 0.f;
  };
  Own cur;
  own(k0, cur);
  const int oA = (ty + 1) * kFMW + om + tx;  // (j, i) in an M box
  const int oQ = (ty + 3) * kFQW + oq + 3 + tx;  // (j, i) in a ph / phb box
  int kstop = k1, r0 = 0, r1 = 1 % kFRing;
  uint32_t p0 = 0, p1 = 1 / kFRing;
  for (int k = k0; k < k1; ++k) {
    Own nxt{};
    if (k + 1 < k1) own(k + 1, nxt);
    bool ok = tma::mbar_wait_bounded(&bar[r0], p0, kFWaitCycles);
    if (k + 1 <= khi) ok = ok && tma::mbar_wait_bounded(&bar[r1], p1, kFWaitCycles);
    if (__syncthreads_or(!ok)) {
      kstop = k;
      break;
    }
    // every thread is past level k-1: its slot takes level k+2
    if (tid == 0 && k + 2 <= khi) {
      issue(k + 2, (r1 + 1) % kFRing);
      hi = k + 2;
    }
    const float* S0 = slot_base(r0);
    const float* S1 = slot_base(r1);
    const float* PH0 = S0;
    const float* PHB0 = S0 + kFQSlot;
    const float* PH1 = S1;
    const float* PHB1 = S1 + kFQSlot;
    auto M0 = [&](int f) { return S0 + 2 * kFQSlot + f * kFMSlot; };
    auto M1 = [&](int f) { return S1 + 2 * kFQSlot + f * kFMSlot; };
    const float uk_c = M0(FM_U)[oA], uk_e = M0(FM_U)[oA + 1];
    const float vk_c = M0(FM_V)[oA], vk_n = M0(FM_V)[oA + kFMW];
    const float ruk_c = M0(FM_RU)[oA], ruk_e = M0(FM_RU)[oA + 1];
    const float rvk_c = M0(FM_RV)[oA], rvk_n = M0(FM_RV)[oA + kFMW];
    const float pk_c = M0(FM_PP)[oA];
    float o_ph = 0.f, o_ru = 0.f, o_rv = 0.f, o_rw = 0.f, o_cqw = 0.f, o_rwt = 0.f;
    float wd_up = wdwn, dpn_up_u = 0.f, dpn_up_v = 0.f;
    // wdwn(k+1) = 0.5 (ww(k+1) + ww(k)) rdnw(k) (ph(k+1) - ph(k) + phb(k+1) - phb(k)),
    // carried up as the next level's wdwn(k)
    if (mass && k < nz - 1) wd_up = 0.5f * (cur.ww1 + ww_c) * __ldg(&rdnw[k]) * (PH1[oQ] - PH0[oQ] + PHB1[oQ] - PHB0[oQ]);
    // ---------------- rhs_ph (wrf_dynamics.py:2031-2297)
    if (mass && k >= 1) {
      float t = cur.pht;
      if (k < nz - 1) {
        t = t - (__ldg(&fnm[k]) * wd_up + __ldg(&fnp[k]) * wdwn);
      } else {
        t = 0.f;
      }
      t = t + mut * gf * cur.w / msfty;
      const bool top = (k == nz - 1);
      float fly_c, fly_n, flx_c, flx_e;
      if (!top) {
        fly_c = muv_c * (vk_c + v_c) * mvy_c;
        fly_n = muv_n * (vk_n + v_n) * mvy_n;
        flx_c = muu_c * (uk_c + u_c) * mux_c;
        flx_e = muu_e * (uk_e + u_e) * mux_e;
      } else {  // v, u at nz-2 (carried) and nz-3
        const float cfn = g.cfn, cfn1 = g.cfn1;
        const size_t q3 = (size_t)(nz - 3) * lev + c;
        fly_c = muv_c * (cfn * v_c + cfn1 * __ldg(&s[WF_V][q3])) * mvy_c;
        fly_n = muv_n * (cfn * v_n + cfn1 * __ldg(&s[WF_V][q3 + nx])) * mvy_n;
        flx_c = muu_c * (cfn * u_c + cfn1 * __ldg(&s[WF_U][q3])) * mux_c;
        flx_e = muu_e * (cfn * u_e + cfn1 * __ldg(&s[WF_U][q3 + 1])) * mux_e;
      }
      const float ky = top ? (float)(0.5 * g.rdyd) : (float)(0.25 * g.rdyd);
      const float* ph = PH0 + oQ;
      const float* phb = PHB0 + oQ;
      if (j >= jds + 3 && j < jde - 4) {
        const float dd = d6s(ph, kFQW) + 45.0f * (phb[kFQW] - phb[-kFQW]) - 9.0f * (phb[2 * kFQW] - phb[-2 * kFQW]) +
                         (phb[3 * kFQW] - phb[-3 * kFQW]);
        t = t - (ky / msfty) * ((fly_n + fly_c) * (float)(1.0 / 60.0) * dd);
      } else if (j == jds + 2 || j == jde - 4) {
        const float dd = 8.0f * (ph[kFQW] - ph[-kFQW]) - (ph[2 * kFQW] - ph[-2 * kFQW]) +
                         8.0f * (phb[kFQW] - phb[-kFQW]) - (phb[2 * kFQW] - phb[-2 * kFQW]);
        t = t - (ky / msfty) * ((fly_n + fly_c) * (float)(1.0 / 12.0) * dd);
      } else if (j == jds + 1 || j == jde - 3) {
        const float dp1 = phb[kFQW] - phb[0] + ph[kFQW] - ph[0];
        const float dp0 = phb[0] - phb[-kFQW] + ph[0] - ph[-kFQW];
        t = t - (ky / msfty) * (fly_n * dp1 + fly_c * dp0);
      }
      const float kx = top ? (float)(0.5 * g.rdxd) : (float)(0.25 * g.rdxd);
      if (i >= ids + 3 && i < ide - 4) {
        const float dd = d6s(ph, 1) + 45.0f * (phb[1] - phb[-1]) - 9.0f * (phb[2] - phb[-2]) + (phb[3] - phb[-3]);
        t = t - (kx / msfty) * ((flx_e + flx_c) * (float)(1.0 / 60.0) * dd);
      } else if (i == ids + 1 || i == ide - 3) {
        const float dp1 = phb[1] - phb[0] + ph[1] - ph[0];
        const float dp0 = phb[0] - phb[-1] + ph[0] - ph[-1];
        t = t - (kx / msfty) * (flx_e * dp1 + flx_c * dp0);
      }
      o_ph = t;
    }
    // ---------------- horizontal pressure gradient (wrf_dynamics.py:2300-2421)
    if (k < ktf && (uc || vc)) {
      const float* AL = M0(FM_AL);
      const float* ALT = M0(FM_ALT);
      const float* PB = M0(FM_PB);
      const float* PHP = M0(FM_PHP);
      const float* PP0 = M0(FM_PP);
      const float* PP1 = M1(FM_PP);
      const float rdk = __ldg(&rdnw[k]);
      const bool last = k + 1 == nz - 1;
      const float fm1 = last ? 0.f : __ldg(&fnm[k + 1]), fp1 = last ? 0.f : __ldg(&fnp[k + 1]);
      if (uc) {
        const int ow = oA - 1;
        const int qw = oQ - 1;
        dpn_up_u = last ? 0.f : 0.5f * (fm1 * (PP1[ow] + PP1[oA]) + fp1 * (PP0[ow] + PP0[oA]));
        float dpx = cpu * ((PH1[oQ] - PH1[qw] + PH0[oQ] - PH0[qw]) + (ALT[oA] + ALT[ow]) * (PP0[oA] - PP0[ow]) +
                           (AL[oA] + AL[ow]) * (PB[oA] - PB[ow]));
        dpx = dpx + cpu2 * (PHP[oA] - PHP[ow]) * (rdk * (dpn_up_u - dpn_u) - muav_u);
        o_ru = cur.rut - cur.cqu * dpx;
      }
      if (vc) {
        const int os = oA - kFMW;
        const int qs = oQ - kFQW;
        dpn_up_v = last ? 0.f : 0.5f * (fm1 * (PP1[os] + PP1[oA]) + fp1 * (PP0[os] + PP0[oA]));
        float dpy = cpv * ((PH1[oQ] - PH1[qs] + PH0[oQ] - PH0[qs]) + (ALT[oA] + ALT[os]) * (PP0[oA] - PP0[os]) +
                           (AL[oA] + AL[os]) * (PB[oA] - PB[os]));
        dpy = dpy + cpv2 * (PHP[oA] - PHP[os]) * (rdk * (dpn_up_v - dpn_v) - muav_v);
        o_rv = cur.rvt - cur.cqv * dpy;
      }
    }
    // ---------------- pg_buoy_w (wrf_dynamics.py:2424-2460); cqw becomes 1/(1+cqw)
    if (mass && k >= 1 && k < nz - 1) {
      if (k == nz - 2) {  // the top level, from the unmodified cqw of level nz-2
        const float cq1 = 1.0f / (1.0f + cur.cqw);
        const float cq2 = cur.cqw * cq1;
        const float rwt_top = (k + 1 < k1) ? nxt.rwt : s[WF_RW_TEND][(size_t)(k + 1) * lev + c];
        o_rwt = rwt_top + rm * gf * (cq1 * 2.0f * __ldg(&rdnw[nz - 2]) * (-pk_c) - mu_c - cq2 * mub);
      }
      const float cq1 = 1.0f / (1.0f + cur.cqw);
      const float cq2 = cur.cqw * cq1;
      o_cqw = cq1;
      o_rw = cur.rwt + rm * gf * (cq1 * __ldg(&rdn[k]) * (pk_c - p_c) - mu_c - cq2 * mub);
    }
    // ---------------- coriolis and curvature (wrf_dynamics.py:2463-2620)
    if (k < ktf && (uc || vc)) {
      const float* U = M0(FM_U);
      const float* V = M0(FM_V);
      const float* RW0 = M0(FM_RW);
      const float* RW1 = M1(FM_RW);
      const float vx_c = 0.5f * (U[oA] + U[oA + 1]) * dmx_c * rdy - 0.5f * (V[oA] + V[oA + kFMW]) * dmy_c * rdx;
      if (uc) {
        const float* RV = M0(FM_RV);
        const float rvs = RV[oA + kFMW - 1] + RV[oA + kFMW] + RV[oA - 1] + RV[oA];
        const float rws = RW1[oA - 1] + RW0[oA - 1] + RW1[oA] + RW0[oA];
        float t = o_ru;
        t = t + cu1 * rvs - cu2 * rws;
        const int ow = oA - 1;
        const float vx_w = 0.5f * (U[ow] + U[ow + 1]) * dmx_w * rdy - 0.5f * (V[ow] + V[ow + kFMW]) * dmy_w * rdx;
        t = t + 0.5f * (vx_c + vx_w) * 0.25f * rvs - U[oA] * rr * 0.25f * rws;
        o_ru = t;
      }
      if (vc) {
        const float* RU = M0(FM_RU);
        const float rus = RU[oA] + RU[oA + 1] + RU[oA - kFMW] + RU[oA - kFMW + 1];
        const float rws = RW1[oA - kFMW] + RW0[oA - kFMW] + RW1[oA] + RW0[oA];
        float t = o_rv;
        t = t - cv1 * rus + cv2 * rws;
        const int os = oA - kFMW;
        const float vx_s = 0.5f * (U[os] + U[os + 1]) * dmx_s * rdy - 0.5f * (V[os] + V[os + kFMW]) * dmy_s * rdx;
        t = t - 0.5f * (vx_c + vx_s) * 0.25f * rus - r_v * V[oA] * rr * 0.25f * rws;
        o_rv = t;
      }
    }
    if (mass && k >= 1 && k < ktf) {  // w
      const float fm = __ldg(&fnm[k]), fp = __ldg(&fnp[k]);
      const float A = fm * (ruk_c + ruk_e) + fp * (ru_c + ru_e);
      const float B = fm * (rvk_c + rvk_n) + fp * (rv_c + rv_n);
      float t = o_rw;
      t = t + e_c * (cosa_c * 0.5f * A - rmt * sina_c * 0.5f * B);
      const float Cu = fm * (uk_c + uk_e) + fp * (u_c + u_e);
      const float Cv = fm * (vk_c + vk_n) + fp * (v_c + v_n);
      t = t + rr * (0.5f * A * 0.5f * Cu + rmt * 0.5f * B * 0.5f * Cv);
      o_rw = t;
    }
    // ---------------- stores
    const size_t p = (size_t)k * lev + c;
    if (mass && k >= 1) s[WF_PH_TEND][p] = o_ph;
    if (uc && k < ktf) s[WF_RU_TEND][p] = o_ru;
    if (vc && k < ktf) s[WF_RV_TEND][p] = o_rv;
    if (mass && k >= 1 && k < nz - 1) {
      s[WF_RW_TEND][p] = o_rw;
      s[WF_CQW][p] = o_cqw;
      if (k == nz - 2) {
        s[WF_RW_TEND][p + lev] = o_rwt;
        nxt.rwt = o_rwt;
      }
    }
    // ---------------- carry level k up
    u_c = uk_c;
    u_e = uk_e;
    v_c = vk_c;
    v_n = vk_n;
    ru_c = ruk_c;
    ru_e = ruk_e;
    rv_c = rvk_c;
    rv_n = rvk_n;
    p_c = pk_c;
    dpn_u = dpn_up_u;
    dpn_v = dpn_up_v;
    wdwn = wd_up;
    ww_c = cur.ww1;
    cur = nxt;
    r0 = r1;
    p0 = p1;
    if (++r1 == kFRing) {
      r1 = 0;
    }
    if (r1 == 0) p1 ^= 1u;
  }
  if (kstop < k1 && tid == 0) {
    for (int L = kstop; L <= hi; ++L)
      tma::mbar_wait_bounded(&bar[(L - k0) % kFRing], ((L - k0) / kFRing) & 1, kFWaitCycles);
    if (s[WF_STATUS]) atomicAdd(reinterpret_cast<int*>(s[WF_STATUS]) + WRF_ST_WAIT, 1);
  }
}

}  // namespace

// k_forces in its tensor-map form; returns 0 (nothing launched) when the
// arrays do not allow tensor maps or the point form is selected
int launch_forces_tma(const Grid& g, const S& s, cudaStream_t st) {
  if (kernel_form() != WRF_FORM_FAST || g.nx % 4 != 0 || g.nz < 4) return 0;
  ForcesTmaArgs a{};
  const char* err = nullptr;
  if (!tma::encode_f32_4d(&a.ph, s[WF_PH], g.nx, g.ny, g.nz, 1, kFQW, kFQH, &err) ||
      !tma::encode_f32_4d(&a.phb, s[WF_PHB], g.nx, g.ny, g.nz, 1, kFQW, kFQH, &err))
    return 0;
  const int f[kFNM] = {WF_U, WF_V, WF_RU, WF_RV, WF_RW, WF_ALT, WF_AL, WF_PB, WF_PHP, WF_P};
  for (int e = 0; e < kFNM; ++e)
    if (!tma::encode_f32_4d(&a.m[e], s[f[e]], g.nx, g.ny, g.nz, 1, kFMW, kFMH, &err)) return 0;
  a.nchunk = min((g.nz + kFKCH - 1) / kFKCH, g.nz);
  const size_t dyn = (size_t)kFRing * kFSlot * sizeof(float) + 128;
  if (cudaFuncSetAttribute(k_forces_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) != cudaSuccess) return 0;
  const dim3 gr((g.ide - g.ids + kFTX - 1) / kFTX, (g.jde - g.jds + kFTY - 1) / kFTY, a.nchunk);
  k_forces_tma<<<gr, dim3(kFTX, kFTY), dyn, st>>>(g, s, a);
  return 1;
}

}  // namespace wrf
