// Adjoints of small_step_prep (wrf_dynamics.py:3152-3266) and of
// calc_mu_uv_1 + small_step_finish (wrf_dynamics.py:3844-3930), the
// conversions into and out of the acoustic steps' perturbation form.
//
// Each forward statement out = f(in) that overwrites `out` is reversed as:
// read out's cotangent, add its partial products into the inputs'
// cotangents, then set out's cotangent to what its incoming value receives
// (zero where it was overwritten, in-place updates keep their own share).
// 2-D operands (the column masses and map factors) serve a column of levels
// and are accumulated atomically; 3-D cotangents are each owned by one
// thread.
#include "kernels.cuh"

namespace wrf {

namespace {

__device__ __forceinline__ void acc(float* a, size_t q, float v) {
  if (v != 0.f) atomicAdd(a + q, v);
}

// k_ssp3d's reverse (the 3-D part of small_step_prep)
__global__ void k_ssp3d_adj(Grid g, S s, S b, int rk_step) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nz = g.nz, ktf = nz - 1;
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const bool t2 = j >= jts && j < jme && i >= its && i < ime;
  const bool du = k < ktf && j >= jts && j < jme && i >= its && i < ieu;
  const bool dv = k < ktf && j >= jts && j < jev && i >= its && i < ime;
  const bool r1 = rk_step == 1;
  // (field, its _1 copy, its _save copy, the column masses, the factor)
  if (du) {
    const float u2 = s[WF_U][p], u1 = r1 ? u2 : s[WF_U_1][p];
    const float muus = s[WF_MUUS][c], muu = s[WF_MUU][c], m = s[WF_MSFUY][c];
    const float U = b[WF_U][p];
    float u2b = -muu / m * U + b[WF_U_SAVE][p];
    b[WF_U_SAVE][p] = 0.f;
    if (r1) {
      u2b += b[WF_U_1][p] + muus / m * U;
      b[WF_U_1][p] = 0.f;
    } else {
      b[WF_U_1][p] += muus / m * U;
    }
    acc(b[WF_MUUS], c, u1 / m * U);
    acc(b[WF_MUU], c, -u2 / m * U);
    b[WF_U][p] = u2b;
  }
  if (dv) {
    const float v2 = s[WF_V][p], v1 = r1 ? v2 : s[WF_V_1][p];
    const float muvs = s[WF_MUVS][c], muv = s[WF_MUV][c], m = s[WF_MSFVX_INV][c];
    const float V = b[WF_V][p];
    float v2b = -muv * m * V + b[WF_V_SAVE][p];
    b[WF_V_SAVE][p] = 0.f;
    if (r1) {
      v2b += b[WF_V_1][p] + muvs * m * V;
      b[WF_V_1][p] = 0.f;
    } else {
      b[WF_V_1][p] += muvs * m * V;
    }
    acc(b[WF_MUVS], c, v1 * m * V);
    acc(b[WF_MUV], c, -v2 * m * V);
    b[WF_V][p] = v2b;
  }
  if (!t2) return;
  const float muts = s[WF_MUTS][c], mut = s[WF_MUT][c];
  float mutsb = 0.f, mutb = 0.f;
  if (k < ktf) {
    // c2a = cpovcv (pb + p) / alt
    const float C = b[WF_C2A][p];
    const float alt = s[WF_ALT][p];
    const float cp = (float)CPOVCV;
    b[WF_PB][p] += cp / alt * C;
    b[WF_P][p] += cp / alt * C;
    b[WF_ALT][p] += -cp * (s[WF_PB][p] + s[WF_P][p]) / (alt * alt) * C;
    b[WF_C2A][p] = 0.f;
    // t = muts t_1 - mut t_2
    const float t2v = s[WF_T][p], t1 = r1 ? t2v : s[WF_T_1][p];
    const float T = b[WF_T][p];
    float t2b = -mut * T + b[WF_T_SAVE][p];
    b[WF_T_SAVE][p] = 0.f;
    if (r1) {
      t2b += b[WF_T_1][p] + muts * T;
      b[WF_T_1][p] = 0.f;
    } else {
      b[WF_T_1][p] += muts * T;
    }
    mutsb += t1 * T;
    mutb -= t2v * T;
    b[WF_T][p] = t2b;
  }
  {  // w = (muts w_1 - mut w_2) / msfty
    const float w2 = s[WF_W][p], w1 = r1 ? w2 : s[WF_W_1][p];
    const float m = s[WF_MSFTY][c];
    const float W = b[WF_W][p];
    float w2b = -mut / m * W + b[WF_W_SAVE][p];
    b[WF_W_SAVE][p] = 0.f;
    if (r1) {
      w2b += b[WF_W_1][p] + muts / m * W;
      b[WF_W_1][p] = 0.f;
    } else {
      b[WF_W_1][p] += muts / m * W;
    }
    mutsb += w1 / m * W;
    mutb -= w2 / m * W;
    b[WF_W][p] = w2b;
  }
  {  // ph = ph_1 - ph_2
    const float P = b[WF_PH][p];
    float p2b = -P + b[WF_PH_SAVE][p];
    b[WF_PH_SAVE][p] = 0.f;
    if (r1) {
      p2b += b[WF_PH_1][p] + P;
      b[WF_PH_1][p] = 0.f;
    } else {
      b[WF_PH_1][p] += P;
    }
    b[WF_PH][p] = p2b;
  }
  // ww1 = ww
  b[WF_WW][p] += b[WF_WW1][p];
  b[WF_WW1][p] = 0.f;
  acc(b[WF_MUTS], c, mutsb);
  acc(b[WF_MUT], c, mutb);
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

// k_ssfinish's reverse
__global__ void k_ssfinish_adj(Grid g, S s, S b, float dts, int nsub, int rk_step) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nz = g.nz;
  const int jts = g.jds, jme = g.jde - 1, its = g.ids, ime = g.ide - 1, ieu = g.ide, jev = g.jde;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const bool dv = k < nz - 1 && j >= jts && j < jev && i >= its && i < ime;
  const bool du = k < nz - 1 && j >= jts && j < jme && i >= its && i < ieu;
  const bool m3 = j >= jts && j < jme && i >= its && i < ime;
  if (dv) {  // v = (msfvx v + v_save muv) / muvs
    const float vv = s[WF_V][p], vs = s[WF_V_SAVE][p], mf = s[WF_MSFVX][c], mv = s[WF_MUV][c], mvs = s[WF_MUVS][c];
    const float V = b[WF_V][p];
    b[WF_V_SAVE][p] += mv / mvs * V;
    acc(b[WF_MUV], c, vs / mvs * V);
    acc(b[WF_MUVS], c, -(mf * vv + vs * mv) / (mvs * mvs) * V);
    b[WF_V][p] = mf / mvs * V;
  }
  if (du) {  // u = (msfuy u + u_save muu) / muus
    const float uu = s[WF_U][p], us = s[WF_U_SAVE][p], mf = s[WF_MSFUY][c], mu = s[WF_MUU][c], mus = s[WF_MUUS][c];
    const float U = b[WF_U][p];
    b[WF_U_SAVE][p] += mu / mus * U;
    acc(b[WF_MUU], c, us / mus * U);
    acc(b[WF_MUUS], c, -(mf * uu + us * mu) / (mus * mus) * U);
    b[WF_U][p] = mf / mus * U;
  }
  if (!m3) return;
  const float mut = s[WF_MUT][c], muts = s[WF_MUTS][c];
  float mutb = 0.f, mutsb = 0.f;
  {  // w = (msfty w + w_save mut) / muts
    const float ww = s[WF_W][p], wsv = s[WF_W_SAVE][p], mf = s[WF_MSFTY][c];
    const float W = b[WF_W][p];
    b[WF_W_SAVE][p] += mut / muts * W;
    mutb += wsv / muts * W;
    mutsb -= (mf * ww + wsv * mut) / (muts * muts) * W;
    b[WF_W][p] = mf / muts * W;
  }
  b[WF_PH_SAVE][p] += b[WF_PH][p];  // ph = ph + ph_save
  b[WF_WW1][p] += b[WF_WW][p];      // ww = ww + ww1
  if (k < nz - 1) {  // t = (t [- dts nsub mut h_diabatic] + t_save mut) / muts
    const float tv = s[WF_T][p], ts = s[WF_T_SAVE][p];
    const float T = b[WF_T][p];
    const bool last = rk_step == 3;
    const float hd = last ? s[WF_H_DIABATIC][p] : 0.f;
    const float a = (float)((double)dts * nsub);
    const float num = last ? tv - a * mut * hd + ts * mut : tv + ts * mut;
    b[WF_T_SAVE][p] += mut / muts * T;
    mutb += (ts - (last ? a * hd : 0.f)) / muts * T;
    if (last) b[WF_H_DIABATIC][p] += -a * mut / muts * T;
    mutsb -= num / (muts * muts) * T;
    b[WF_T][p] = T / muts;
  }
  if (k == 0) acc(b[WF_MU_SAVE], c, b[WF_MU][c]);  // mu = mu + mu_save
  acc(b[WF_MUT], c, mutb);
  acc(b[WF_MUTS], c, mutsb);
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
  const dim3 b2(32, 8), b3(32, 4);
  const size_t n2 = g.n2();
  k_ssp_masses<<<col_grid(g, b2), b2, 0, st>>>(g, s, rk_step, work, work + n2, work + 2 * n2);
  S sm = s;
  sm.f[WF_MUTS] = work;
  sm.f[WF_MUUS] = work + n2;
  sm.f[WF_MUVS] = work + 2 * n2;
  k_ssp3d_adj<<<point_grid(g, b3), b3, 0, st>>>(g, sm, b, rk_step);
  k_ssp2d_adj<<<col_grid(g, b2), b2, 0, st>>>(g, s, b, rk_step);
  return 3;
}

// work: caller-owned scratch of 2 ny*nx floats
int launch_small_step_finish_adj(const Grid& g, const S& s, const S& b, float dts, int nsub, int rk_step, float* work,
                                 cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  const size_t n2 = g.n2();
  k_mu_uv_1_masses<<<col_grid(g, b2), b2, 0, st>>>(g, s, work, work + n2);
  S sm = s;
  sm.f[WF_MUUS] = work;
  sm.f[WF_MUVS] = work + n2;
  k_ssfinish_adj<<<point_grid(g, b3), b3, 0, st>>>(g, sm, b, dts, nsub, rk_step);
  k_mu_uv_1_adj<<<col_grid(g, b2), b2, 0, st>>>(g, s, b);
  return 3;
}

}  // namespace wrf
