// rk_addtend_dry (wrf_dynamics.py:3100-3148) and spec_bdytend
// (wrf_boundary.py:189-241) as stand-alone operators with their adjoints
// (the step runs both inside k_addtend).
//
// rk_addtend_dry: at the first RK stage the physics tendencies first take
// the saved start-of-step fields (ru_tendf += u_save msfuy, ...), then every
// stage adds them to the large-step tendencies with the map-factor division
// and theta takes mut h_diabatic / msfty.  spec_bdytend overwrites the
// specified rows of a tendency with the boundary tendency (data), so its
// adjoint zeroes those rows of the tendency's cotangent.
#include "kernels.cuh"

namespace wrf {

namespace {

__device__ __forceinline__ void acc(float* a, size_t q, float v) {
  if (v != 0.f) atomicAdd(a + q, v);
}

struct AddtendRegions {
  bool U, V, W, T;
};

__device__ __forceinline__ AddtendRegions addtend_regions(const Grid& g, int k, int j, int i) {
  const int nz = g.nz, jts = g.jds, jm = g.jde - 1, its = g.ids, ite = g.ide, jte = g.jde, im = g.ide - 1;
  AddtendRegions r;
  r.U = k < nz - 1 && j >= jts && j < jm && i >= its && i < ite;
  r.V = k < nz - 1 && j >= jts && j < jte && i >= its && i < im;
  r.W = j >= jts && j < jm && i >= its && i < im;
  r.T = k < nz - 1 && r.W;
  return r;
}

__global__ void k_addtend_op(Grid g, S s, int rk_step) {
  WRF_POINT_INDEX(g, k, j, i);
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const AddtendRegions r = addtend_regions(g, k, j, i);
  const bool first = rk_step == 1;
  if (r.U) {
    float f = s[WF_RU_TENDF][p];
    if (first) s[WF_RU_TENDF][p] = f = f + s[WF_U_SAVE][p] * s[WF_MSFUY][c];
    s[WF_RU_TEND][p] = s[WF_RU_TEND][p] + f / s[WF_MSFUY][c];
  }
  if (r.V) {
    float f = s[WF_RV_TENDF][p];
    if (first) s[WF_RV_TENDF][p] = f = f + s[WF_V_SAVE][p] * s[WF_MSFVX][c];
    s[WF_RV_TEND][p] = s[WF_RV_TEND][p] + f * s[WF_MSFVX_INV][c];
  }
  if (r.W) {
    const float m = s[WF_MSFTY][c];
    float f = s[WF_RW_TENDF][p];
    if (first) s[WF_RW_TENDF][p] = f = f + s[WF_W_SAVE][p] * m;
    s[WF_RW_TEND][p] = s[WF_RW_TEND][p] + f / m;
    float h = s[WF_PH_TENDF][p];
    if (first) s[WF_PH_TENDF][p] = h = h + s[WF_PH_SAVE][p];
    s[WF_PH_TEND][p] = s[WF_PH_TEND][p] + h / m;
  }
  if (r.T) {
    const float m = s[WF_MSFTY][c];
    float f = s[WF_T_TENDF][p];
    if (first) s[WF_T_TENDF][p] = f = f + s[WF_T_SAVE][p];
    s[WF_T_TEND][p] = s[WF_T_TEND][p] + f / m + s[WF_MUT][c] * s[WF_H_DIABATIC][p] / m;
  }
  if (k == 0 && r.W) s[WF_MU_TEND][c] = s[WF_MU_TEND][c] + s[WF_MU_TENDF][c];
}

// the tendencies' cotangents pass through; tendf and the saved fields, mut
// and h_diabatic receive theirs
__global__ void k_addtend_op_adj(Grid g, S s, S b, int rk_step) {
  WRF_POINT_INDEX(g, k, j, i);
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const AddtendRegions r = addtend_regions(g, k, j, i);
  const bool first = rk_step == 1;
  // with first: tendf' = tendf + save * msf (its cotangent F' = F + T / msf),
  // and save receives F' msf; else tendf receives T / msf
  if (r.U) {
    const float m = s[WF_MSFUY][c];
    const float F = b[WF_RU_TENDF][p] + b[WF_RU_TEND][p] / m;
    b[WF_RU_TENDF][p] = F;
    if (first) b[WF_U_SAVE][p] += F * m;
  }
  if (r.V) {
    const float F = b[WF_RV_TENDF][p] + b[WF_RV_TEND][p] * s[WF_MSFVX_INV][c];
    b[WF_RV_TENDF][p] = F;
    if (first) b[WF_V_SAVE][p] += F * s[WF_MSFVX][c];
  }
  if (r.W) {
    const float m = s[WF_MSFTY][c];
    const float F = b[WF_RW_TENDF][p] + b[WF_RW_TEND][p] / m;
    b[WF_RW_TENDF][p] = F;
    if (first) b[WF_W_SAVE][p] += F * m;
    const float H = b[WF_PH_TENDF][p] + b[WF_PH_TEND][p] / m;
    b[WF_PH_TENDF][p] = H;
    if (first) b[WF_PH_SAVE][p] += H;
  }
  if (r.T) {
    const float m = s[WF_MSFTY][c];
    const float T = b[WF_T_TEND][p];
    const float F = b[WF_T_TENDF][p] + T / m;
    b[WF_T_TENDF][p] = F;
    if (first) b[WF_T_SAVE][p] += F;
    acc(b[WF_MUT], c, s[WF_H_DIABATIC][p] / m * T);
    b[WF_H_DIABATIC][p] += s[WF_MUT][c] / m * T;
  }
  if (k == 0 && r.W) b[WF_MU_TENDF][c] += b[WF_MU_TEND][c];
}

// the specified rows of spec_bdytend for stagger var (levels < nk)
__device__ __forceinline__ bool spec_tend_row(const Grid& g, char var, int j, int i) {
  const int ibe = var == 'u' ? g.ide : g.ide - 1, jbe = var == 'v' ? g.jde : g.jde - 1;
  const int ibs = g.ids, jbs = g.jds;
  if ((j == jbs || j == jbe - 1) && i >= ibs && i < ibe) return true;
  return j >= jbs && j < jbe && (i == ibs || i == ibe - 1);
}

// the value the specified row takes, from the permuted boundary tendencies
// (x sides [nk][ny][5], y sides [nk][5][nx]); the x sides are applied last
__global__ void k_spec_tend(Grid g, float* tend, const float* txs, const float* txe, const float* tys,
                            const float* tye, char var, int nk) {
  WRF_POINT_INDEX(g, k, j, i);
  if (k >= nk || !spec_tend_row(g, var, j, i)) return;
  const int ibe = var == 'u' ? g.ide : g.ide - 1, jbe = var == 'v' ? g.jde : g.jde - 1;
  const size_t p = (size_t)k * g.ny * g.nx + g.i2(j, i);
  float v;
  if (j >= g.jds && j < jbe && (i == g.ids || i == ibe - 1))
    v = (i == g.ids ? txs : txe)[((size_t)k * g.ny + j) * 5];
  else
    v = (j == g.jds ? tys : tye)[(size_t)k * 5 * g.nx + i];
  tend[p] = v;
}

__global__ void k_spec_tend_adj(Grid g, float* tend_bar, char var, int nk) {
  WRF_POINT_INDEX(g, k, j, i);
  if (k >= nk || !spec_tend_row(g, var, j, i)) return;
  tend_bar[(size_t)k * g.ny * g.nx + g.i2(j, i)] = 0.f;
}

}  // namespace

int launch_addtend_op(const Grid& g, const S& s, int rk_step, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_addtend_op<<<point_grid(g, b3), b3, 0, st>>>(g, s, rk_step);
  return 1;
}

int launch_addtend_op_adj(const Grid& g, const S& s, const S& b, int rk_step, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_addtend_op_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, rk_step);
  return 1;
}

// var 'u', 'v', 't' (levels below nz-1), 'h' (all nz levels), 'm' (2-D)
int launch_spec_tend(const Grid& g, float* tend, const float* const* bt4, char var, cudaStream_t st) {
  const dim3 b3(32, 4);
  Grid g2 = g;
  if (var == 'm') g2.nz = 1;
  const int nk = var == 'm' ? 1 : (var == 'h' ? g.nz : g.nz - 1);
  k_spec_tend<<<point_grid(g2, b3), b3, 0, st>>>(g2, tend, bt4[0], bt4[1], bt4[2], bt4[3], var, nk);
  return 1;
}

int launch_spec_tend_adj(const Grid& g, float* tend_bar, char var, cudaStream_t st) {
  const dim3 b3(32, 4);
  Grid g2 = g;
  if (var == 'm') g2.nz = 1;
  const int nk = var == 'm' ? 1 : (var == 'h' ? g.nz : g.nz - 1);
  k_spec_tend_adj<<<point_grid(g2, b3), b3, 0, st>>>(g2, tend_bar, var, nk);
  return 1;
}

}  // namespace wrf
