// Adjoints of small_step_prep (wrf_dynamics.py:3152-3266) and of
// calc_mu_uv_1 + small_step_finish (wrf_dynamics.py:3844-3930), the
// conversions into and out of the acoustic steps' perturbation form.
//
// Each forward statement out = f(in) that overwrites `out` is reversed as:
// read out's cotangent, add its partial products into the inputs'
// cotangents, then set out's cotangent to what its incoming value receives
// (zero where it was overwritten, in-place updates keep their own share).
// 2-D operands (the column masses and map factors) serve a column of levels:
// the 3-D passes run a column's levels in one block (k_ssp_cols_adj), sum
// the 2-D cotangents over the levels in a fixed order and add them once;
// 3-D cotangents are each owned by one thread.
#include "kernels.cuh"

namespace wrf {

namespace {

__device__ __forceinline__ void acc(float* a, size_t q, float v) {
  if (v != 0.f) atomicAdd(a + q, v);
}

// the column sums of a column-level kernel: the cotangents of the 2-D
// operands muus, muu, muvs, muv, muts, mut, in that order
constexpr int kColSums = 6;
constexpr int kColGroups = 8;  // level groups of a block (threadIdx.y)

// k_ssp3d's reverse (the 3-D part of small_step_prep) at one point; the
// 2-D cotangents go to a[].  The operand and cotangent arrays may alias as
// far as the compiler knows, so every load is written before the first
// store: the point's loads then issue together instead of one group per
// statement.
__device__ __forceinline__ void ssp3d_adj_point(const Grid& g, const S& s, const S& b, int rk_step, int k, int j,
                                                int i, float* a) {
  const int nz = g.nz, ktf = nz - 1;
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const bool t2 = j >= jts && j < jme && i >= its && i < ime;
  const bool du = k < ktf && j >= jts && j < jme && i >= its && i < ieu;
  const bool dv = k < ktf && j >= jts && j < jev && i >= its && i < ime;
  const bool tk = t2 && k < ktf;
  const bool r1 = rk_step == 1;
  // ---- loads
  float u2 = 0.f, u1 = 0.f, muus = 0.f, muu = 0.f, mu_ = 1.f, U = 0.f, Us = 0.f, U1 = 0.f;
  if (du) {
    u2 = s[WF_U][p];
    u1 = r1 ? u2 : s[WF_U_1][p];
    muus = s[WF_MUUS][c];
    muu = s[WF_MUU][c];
    mu_ = s[WF_MSFUY][c];
    U = b[WF_U][p];
    Us = b[WF_U_SAVE][p];
    U1 = b[WF_U_1][p];
  }
  float v2 = 0.f, v1 = 0.f, muvs = 0.f, muv = 0.f, mv_ = 0.f, V = 0.f, Vs = 0.f, V1 = 0.f;
  if (dv) {
    v2 = s[WF_V][p];
    v1 = r1 ? v2 : s[WF_V_1][p];
    muvs = s[WF_MUVS][c];
    muv = s[WF_MUV][c];
    mv_ = s[WF_MSFVX_INV][c];
    V = b[WF_V][p];
    Vs = b[WF_V_SAVE][p];
    V1 = b[WF_V_1][p];
  }
  float Cb = 0.f, alt = 1.f, pbv = 0.f, pv = 0.f, t2v = 0.f, t1 = 0.f, T = 0.f, Ts = 0.f, T1 = 0.f;
  float PBb = 0.f, Pb = 0.f, ALTb = 0.f;
  if (tk) {
    Cb = b[WF_C2A][p];
    alt = s[WF_ALT][p];
    pbv = s[WF_PB][p];
    pv = s[WF_P][p];
    t2v = s[WF_T][p];
    t1 = r1 ? t2v : s[WF_T_1][p];
    T = b[WF_T][p];
    Ts = b[WF_T_SAVE][p];
    T1 = b[WF_T_1][p];
    PBb = b[WF_PB][p];
    Pb = b[WF_P][p];
    ALTb = b[WF_ALT][p];
  }
  float muts = 0.f, mut = 0.f, w2 = 0.f, w1 = 0.f, mw_ = 1.f, W = 0.f, Ws = 0.f, W1 = 0.f;
  float PH = 0.f, PHs = 0.f, PH1 = 0.f, WW = 0.f, WW1 = 0.f;
  if (t2) {
    muts = s[WF_MUTS][c];
    mut = s[WF_MUT][c];
    w2 = s[WF_W][p];
    w1 = r1 ? w2 : s[WF_W_1][p];
    mw_ = s[WF_MSFTY][c];
    W = b[WF_W][p];
    Ws = b[WF_W_SAVE][p];
    W1 = b[WF_W_1][p];
    PH = b[WF_PH][p];
    PHs = b[WF_PH_SAVE][p];
    PH1 = b[WF_PH_1][p];
    WW = b[WF_WW][p];
    WW1 = b[WF_WW1][p];
  }
  // ---- (field, its _1 copy, its _save copy, the column masses, the factor)
  if (du) {  // u = (muus u_1 - muu u_2) / msfuy
    float u2b = -muu / mu_ * U + Us;
    b[WF_U_SAVE][p] = 0.f;
    if (r1) {
      u2b += U1 + muus / mu_ * U;
      b[WF_U_1][p] = 0.f;
    } else {
      b[WF_U_1][p] = U1 + muus / mu_ * U;
    }
    a[0] += u1 / mu_ * U;
    a[1] += -u2 / mu_ * U;
    b[WF_U][p] = u2b;
  }
  if (dv) {  // v = (muvs v_1 - muv v_2) msfvx_inv
    float v2b = -muv * mv_ * V + Vs;
    b[WF_V_SAVE][p] = 0.f;
    if (r1) {
      v2b += V1 + muvs * mv_ * V;
      b[WF_V_1][p] = 0.f;
    } else {
      b[WF_V_1][p] = V1 + muvs * mv_ * V;
    }
    a[2] += v1 * mv_ * V;
    a[3] += -v2 * mv_ * V;
    b[WF_V][p] = v2b;
  }
  if (!t2) return;
  float mutsb = 0.f, mutb = 0.f;
  if (tk) {
    // c2a = cpovcv (pb + p) / alt
    const float cp = (float)CPOVCV;
    b[WF_PB][p] = PBb + cp / alt * Cb;
    b[WF_P][p] = Pb + cp / alt * Cb;
    b[WF_ALT][p] = ALTb + -cp * (pbv + pv) / (alt * alt) * Cb;
    b[WF_C2A][p] = 0.f;
    // t = muts t_1 - mut t_2
    float t2b = -mut * T + Ts;
    b[WF_T_SAVE][p] = 0.f;
    if (r1) {
      t2b += T1 + muts * T;
      b[WF_T_1][p] = 0.f;
    } else {
      b[WF_T_1][p] = T1 + muts * T;
    }
    mutsb += t1 * T;
    mutb -= t2v * T;
    b[WF_T][p] = t2b;
  }
  {  // w = (muts w_1 - mut w_2) / msfty
    float w2b = -mut / mw_ * W + Ws;
    b[WF_W_SAVE][p] = 0.f;
    if (r1) {
      w2b += W1 + muts / mw_ * W;
      b[WF_W_1][p] = 0.f;
    } else {
      b[WF_W_1][p] = W1 + muts / mw_ * W;
    }
    mutsb += w1 / mw_ * W;
    mutb -= w2 / mw_ * W;
    b[WF_W][p] = w2b;
  }
  {  // ph = ph_1 - ph_2
    float p2b = -PH + PHs;
    b[WF_PH_SAVE][p] = 0.f;
    if (r1) {
      p2b += PH1 + PH;
      b[WF_PH_1][p] = 0.f;
    } else {
      b[WF_PH_1][p] = PH1 + PH;
    }
    b[WF_PH][p] = p2b;
  }
  // ww1 = ww
  b[WF_WW][p] = WW + WW1;
  b[WF_WW1][p] = 0.f;
  a[4] += mutsb;
  a[5] += mutb;
}

// k_ssp2d's reverse (the column masses of small_step_prep)
__global__ void k_ssp2d_adj(Grid g, S s, S b, int rk_step) {
  WRF_COLUMN_INDEX(g, j, i);
  const int c = g.i2(j, i);
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  const bool t2 = j >= jts && j < jme && i >= its && i < ime;
  if (rk_step == 1) {
    if (t2) {
      // mu_1 = mu, mudf = 0, muts = mub + mu, mu_save = mu, mu = 0
      const float mb = b[WF_MU_1][c] + b[WF_MUTS][c] + b[WF_MU_SAVE][c];
      acc(b[WF_MUB], c, b[WF_MUTS][c]);
      b[WF_MU_1][c] = 0.f;
      b[WF_MUDF][c] = 0.f;
      b[WF_MUTS][c] = 0.f;
      b[WF_MU_SAVE][c] = 0.f;
      b[WF_MU][c] = mb;
    }
    if (j >= jts && j < jme && i >= its && i < ieu) {
      acc(b[WF_MUU], c, b[WF_MUUS][c]);
      b[WF_MUUS][c] = 0.f;
    }
    if (j >= jts && j < jev && i >= its && i < ime) {
      acc(b[WF_MUV], c, b[WF_MUVS][c]);
      b[WF_MUVS][c] = 0.f;
    }
  } else {
    if (t2) {
      // muts = mub + mu_1, mu_save = mu, mu = mu_1 - mu
      const float Mt = b[WF_MUTS][c], Mo = b[WF_MU][c];
      acc(b[WF_MUB], c, Mt);
      acc(b[WF_MU_1], c, Mt + Mo);
      b[WF_MU][c] = b[WF_MU_SAVE][c] - Mo;
      b[WF_MUTS][c] = 0.f;
      b[WF_MU_SAVE][c] = 0.f;
    }
    if (j >= jts && j < jme && i >= its && i < ieu) {
      const float h = 0.5f * b[WF_MUUS][c];
      acc(b[WF_MUB], c, h);
      acc(b[WF_MU_1], c, h);
      acc(b[WF_MUB], c - 1, h);
      acc(b[WF_MU_1], c - 1, h);
      b[WF_MUUS][c] = 0.f;
    }
    if (j >= jts && j < jev && i >= its && i < ieu) {
      const float h = 0.5f * b[WF_MUVS][c];
      acc(b[WF_MUB], c, h);
      acc(b[WF_MU_1], c, h);
      acc(b[WF_MUB], c - g.nx, h);
      acc(b[WF_MU_1], c - g.nx, h);
      b[WF_MUVS][c] = 0.f;
    }
  }
}

// k_ssfinish's reverse at one point; the 2-D cotangents go to a[] (loads
// before stores, as in ssp3d_adj_point)
__device__ __forceinline__ void ssfinish_adj_point(const Grid& g, const S& s, const S& b, float dts, int nsub,
                                                   int rk_step, int k, int j, int i, float* a) {
  const int nz = g.nz;
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const bool dv = k < nz - 1 && j >= jts && j < jev && i >= its && i < ime;
  const bool du = k < nz - 1 && j >= jts && j < jme && i >= its && i < ieu;
  const bool m3 = j >= jts && j < jme && i >= its && i < ime;
  const bool tk = m3 && k < nz - 1;
  const bool last = rk_step == 3;
  // ---- loads
  float vv = 0.f, vs = 0.f, mfv = 0.f, mv = 0.f, mvs = 1.f, V = 0.f, Vs = 0.f;
  if (dv) {
    vv = s[WF_V][p];
    vs = s[WF_V_SAVE][p];
    mfv = s[WF_MSFVX][c];
    mv = s[WF_MUV][c];
    mvs = s[WF_MUVS][c];
    V = b[WF_V][p];
    Vs = b[WF_V_SAVE][p];
  }
  float uu = 0.f, us = 0.f, mfu = 0.f, mu = 0.f, mus = 1.f, U = 0.f, Us = 0.f;
  if (du) {
    uu = s[WF_U][p];
    us = s[WF_U_SAVE][p];
    mfu = s[WF_MSFUY][c];
    mu = s[WF_MUU][c];
    mus = s[WF_MUUS][c];
    U = b[WF_U][p];
    Us = b[WF_U_SAVE][p];
  }
  float mut = 0.f, muts = 1.f, ww = 0.f, wsv = 0.f, mfw = 0.f, W = 0.f, Ws = 0.f;
  float PH = 0.f, PHs = 0.f, WW = 0.f, WW1 = 0.f, MU = 0.f, MUs = 0.f;
  if (m3) {
    mut = s[WF_MUT][c];
    muts = s[WF_MUTS][c];
    ww = s[WF_W][p];
    wsv = s[WF_W_SAVE][p];
    mfw = s[WF_MSFTY][c];
    W = b[WF_W][p];
    Ws = b[WF_W_SAVE][p];
    PH = b[WF_PH][p];
    PHs = b[WF_PH_SAVE][p];
    WW = b[WF_WW][p];
    WW1 = b[WF_WW1][p];
    if (k == 0) {
      MU = b[WF_MU][c];
      MUs = b[WF_MU_SAVE][c];
    }
  }
  float tv = 0.f, ts = 0.f, T = 0.f, Ts = 0.f, hd = 0.f, HD = 0.f;
  if (tk) {
    tv = s[WF_T][p];
    ts = s[WF_T_SAVE][p];
    T = b[WF_T][p];
    Ts = b[WF_T_SAVE][p];
    if (last) {
      hd = s[WF_H_DIABATIC][p];
      HD = b[WF_H_DIABATIC][p];
    }
  }
  // ---- cotangents
  if (dv) {  // v = (msfvx v + v_save muv) / muvs
    b[WF_V_SAVE][p] = Vs + mv / mvs * V;
    a[3] += vs / mvs * V;
    a[2] += -(mfv * vv + vs * mv) / (mvs * mvs) * V;
    b[WF_V][p] = mfv / mvs * V;
  }
  if (du) {  // u = (msfuy u + u_save muu) / muus
    b[WF_U_SAVE][p] = Us + mu / mus * U;
    a[1] += us / mus * U;
    a[0] += -(mfu * uu + us * mu) / (mus * mus) * U;
    b[WF_U][p] = mfu / mus * U;
  }
  if (!m3) return;
  float mutb = 0.f, mutsb = 0.f;
  {  // w = (msfty w + w_save mut) / muts
    b[WF_W_SAVE][p] = Ws + mut / muts * W;
    mutb += wsv / muts * W;
    mutsb -= (mfw * ww + wsv * mut) / (muts * muts) * W;
    b[WF_W][p] = mfw / muts * W;
  }
  b[WF_PH_SAVE][p] = PHs + PH;  // ph = ph + ph_save
  b[WF_WW1][p] = WW1 + WW;      // ww = ww + ww1
  if (tk) {  // t = (t [- dts nsub mut h_diabatic] + t_save mut) / muts
    const float a_ = (float)((double)dts * nsub);
    const float num = last ? tv - a_ * mut * hd + ts * mut : tv + ts * mut;
    b[WF_T_SAVE][p] = Ts + mut / muts * T;
    mutb += (ts - (last ? a_ * hd : 0.f)) / muts * T;
    if (last) b[WF_H_DIABATIC][p] = HD + -a_ * mut / muts * T;
    mutsb -= num / (muts * muts) * T;
    b[WF_T][p] = T / muts;
  }
  if (k == 0 && MU != 0.f) b[WF_MU_SAVE][c] = MUs + MU;  // mu = mu + mu_save
  a[5] += mutb;
  a[4] += mutsb;
}

// one column's points by kColGroups level groups (threadIdx.y; levels
// ty, ty + kColGroups, ...), 32 columns of a row a block; the groups' 2-D
// cotangents are summed in a fixed order and added once, so each output
// element has one writer
template <bool kFinish>
__global__ void __launch_bounds__(32 * kColGroups, 3) k_ssp_cols_adj(Grid g, S s, S b, float dts, int nsub, int rk_step) {
  __shared__ float red[kColSums][kColGroups][32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = blockIdx.x * 32 + tx, j = blockIdx.y;
  float a[kColSums];
#pragma unroll
  for (int q = 0; q < kColSums; ++q) a[q] = 0.f;
  if (i < g.nx)
    for (int k = ty; k < g.nz; k += kColGroups) {
      if (kFinish) ssfinish_adj_point(g, s, b, dts, nsub, rk_step, k, j, i, a);
      else ssp3d_adj_point(g, s, b, rk_step, k, j, i, a);
    }
#pragma unroll
  for (int q = 0; q < kColSums; ++q) red[q][ty][tx] = a[q];
  __syncthreads();
  if (ty != 0 || i >= g.nx) return;
  const int c = g.i2(j, i);
  const int f[kColSums] = {WF_MUUS, WF_MUU, WF_MUVS, WF_MUV, WF_MUTS, WF_MUT};
#pragma unroll
  for (int q = 0; q < kColSums; ++q) {
    float t = 0.f;
#pragma unroll
    for (int y = 0; y < kColGroups; ++y) t += red[q][y][tx];
    if (t != 0.f) b[f[q]][c] += t;
  }
}

// calc_mu_uv_1's reverse: muus, muvs from muts
__global__ void k_mu_uv_1_adj(Grid g, S s, S b) {
  WRF_COLUMN_INDEX(g, j, i);
  const int c = g.i2(j, i);
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ite = g.ide, ime = g.ide - 1, jte = g.jde;
  if (j >= jts && j < jme && i >= its && i < ite) {
    const float M = b[WF_MUUS][c];
    if (i >= its + 1 && i < ite - 1) {
      acc(b[WF_MUTS], c, 0.5f * M);
      acc(b[WF_MUTS], c - 1, 0.5f * M);
    } else if (i == its) {
      acc(b[WF_MUTS], c, M);
    } else {
      acc(b[WF_MUTS], c - 1, M);
    }
    b[WF_MUUS][c] = 0.f;
  }
  if (i >= its && i < ime && j >= jts && j < jte) {
    const float M = b[WF_MUVS][c];
    if (j >= jts + 1 && j < jte - 1) {
      acc(b[WF_MUTS], c, 0.5f * M);
      acc(b[WF_MUTS], c - g.nx, 0.5f * M);
    } else if (j == jts) {
      acc(b[WF_MUTS], c, M);
    } else {
      acc(b[WF_MUTS], c - g.nx, M);
    }
    b[WF_MUVS][c] = 0.f;
  }
}

// the column masses muts, muus, muvs as small_step_prep forms them from the
// incoming state (k_ssp2d's arithmetic), into separate arrays: the 3-D part
// of the adjoint needs the values the forward used
__global__ void k_ssp_masses(Grid g, S s, int rk_step, float* muts, float* muus, float* muvs) {
  WRF_COLUMN_INDEX(g, j, i);
  const int c = g.i2(j, i);
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  const float* mu = s[WF_MU];
  const float* mu1 = s[WF_MU_1];
  const float* mub = s[WF_MUB];
  const bool t2 = j >= jts && j < jme && i >= its && i < ime;
  float a = s[WF_MUTS][c], bu = s[WF_MUUS][c], bv = s[WF_MUVS][c];
  if (rk_step == 1) {
    if (t2) a = mub[c] + mu[c];
    if (j >= jts && j < jme && i >= its && i < ieu) bu = s[WF_MUU][c];
    if (j >= jts && j < jev && i >= its && i < ime) bv = s[WF_MUV][c];
  } else {
    if (t2) a = mub[c] + mu1[c];
    if (j >= jts && j < jme && i >= its && i < ieu) bu = 0.5f * (mub[c] + mu1[c] + mub[c - 1] + mu1[c - 1]);
    if (j >= jts && j < jev && i >= its && i < ieu) bv = 0.5f * (mub[c] + mu1[c] + mub[c - g.nx] + mu1[c - g.nx]);
  }
  muts[c] = a;
  muus[c] = bu;
  muvs[c] = bv;
}

// muus, muvs as calc_mu_uv_1 forms them from muts (k_mu_uv_1's arithmetic)
__global__ void k_mu_uv_1_masses(Grid g, S s, float* muus, float* muvs) {
  WRF_COLUMN_INDEX(g, j, i);
  const int c = g.i2(j, i);
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ite = g.ide, ime = g.ide - 1, jte = g.jde;
  const float* muts = s[WF_MUTS];
  float bu = s[WF_MUUS][c], bv = s[WF_MUVS][c];
  if (j >= jts && j < jme) {
    if (i >= its + 1 && i < ite - 1) bu = 0.5f * (muts[c] + muts[c - 1]);
    else if (i == its) bu = muts[c];
    else if (i == ite - 1) bu = muts[c - 1];
  }
  if (i >= its && i < ime) {
    if (j >= jts + 1 && j < jte - 1) bv = 0.5f * (muts[c] + muts[c - g.nx]);
    else if (j == jts) bv = muts[c];
    else if (j == jte - 1) bv = muts[c - g.nx];
  }
  muus[c] = bu;
  muvs[c] = bv;
}

}  // namespace

// work: caller-owned scratch of 3 ny*nx floats
int launch_small_step_prep_adj(const Grid& g, const S& s, const S& b, int rk_step, float* work, cudaStream_t st) {
  const dim3 b2(32, 8);
  const size_t n2 = g.n2();
  k_ssp_masses<<<col_grid(g, b2), b2, 0, st>>>(g, s, rk_step, work, work + n2, work + 2 * n2);
  S sm = s;
  sm.f[WF_MUTS] = work;
  sm.f[WF_MUUS] = work + n2;
  sm.f[WF_MUVS] = work + 2 * n2;
  k_ssp_cols_adj<false><<<dim3((g.nx + 31) / 32, g.ny), dim3(32, kColGroups), 0, st>>>(g, sm, b, 0.f, 0, rk_step);
  k_ssp2d_adj<<<col_grid(g, b2), b2, 0, st>>>(g, s, b, rk_step);
  return 3;
}

// work: caller-owned scratch of 2 ny*nx floats
int launch_small_step_finish_adj(const Grid& g, const S& s, const S& b, float dts, int nsub, int rk_step, float* work,
                                 cudaStream_t st) {
  const dim3 b2(32, 8);
  const size_t n2 = g.n2();
  k_mu_uv_1_masses<<<col_grid(g, b2), b2, 0, st>>>(g, s, work, work + n2);
  S sm = s;
  sm.f[WF_MUUS] = work;
  sm.f[WF_MUVS] = work + n2;
  k_ssp_cols_adj<true><<<dim3((g.nx + 31) / 32, g.ny), dim3(32, kColGroups), 0, st>>>(g, sm, b, dts, nsub, rk_step);
  k_mu_uv_1_adj<<<col_grid(g, b2), b2, 0, st>>>(g, s, b);
  return 3;
}

}  // namespace wrf
