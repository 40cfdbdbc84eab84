// The rest of the acoustic substep as stand-alone operators with their
// adjoints (the step runs these inside k_acoustic_col and k_advance_uv):
//   sumflux            wrf_dynamics.py:3799-3839 (time-averaged mass fluxes)
//   spec_bdyupdate     wrf_boundary.py:244-294 (field += dt tend on the
//                      specified rows; 't' 3-D, 'm' 2-D)
//   spec_bdyupdate_ph  wrf_boundary.py:297-355 (specified-row phi with the
//                      mass re-weighting mu_old = muts - dt mu_tend)
// The adjoints read the cotangent of each updated field and rewrite it to
// that of the field's incoming value; the other operands' cotangents are
// accumulated (atomically where a 2-D operand serves a column of levels).
#include "kernels.cuh"

namespace wrf {

namespace {

// sumflux's three regions (u, v and w points of the tile)
__device__ __forceinline__ void sumflux_regions(const Grid& g, int k, int j, int i, bool& U, bool& V, bool& W,
                                                bool& Z) {
  const int nz = g.nz, jts = g.jds, jte = g.jde, its = g.ids, ite = g.ide;
  U = k < nz - 1 && j >= jts && j < g.jde - 1 && i >= its && i < ite;
  V = k < nz - 1 && j >= jts && j < jte && i >= its && i < g.ide - 1;
  W = j >= jts && j < g.jde - 1 && i >= its && i < g.ide - 1;
  Z = j >= jts && j < jte && i >= its && i < ite;  // zeroed at the first iteration
}

__global__ void k_sumflux(Grid g, S s, int iteration, int nsub) {
  WRF_POINT_INDEX(g, k, j, i);
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  bool U, V, W, Z;
  sumflux_regions(g, k, j, i, U, V, W, Z);
  float* ru_m = s[WF_RU_M];
  float* rv_m = s[WF_RV_M];
  float* ww_m = s[WF_WW_M];
  float a = ru_m[p], b = rv_m[p], cc = ww_m[p];
  if (iteration == 1 && Z) a = b = cc = 0.f;
  const bool last = iteration == nsub;
  const float fn = (float)nsub;
  if (U) {
    a = a + s[WF_U][p];
    if (last) a = a / fn + s[WF_MUU][c] * s[WF_U_SAVE][p] / s[WF_MSFUY][c];
  }
  if (V) {
    b = b + s[WF_V][p];
    if (last) b = b / fn + s[WF_MUV][c] * s[WF_V_SAVE][p] * s[WF_MSFVX_INV][c];
  }
  if (W) {
    cc = cc + s[WF_WW][p];
    if (last) cc = cc / fn + s[WF_WW1][p];
  }
  ru_m[p] = a;
  rv_m[p] = b;
  ww_m[p] = cc;
}

__global__ void k_sumflux_adj(Grid g, S s, S bar, int iteration, int nsub) {
  WRF_POINT_INDEX(g, k, j, i);
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  bool U, V, W, Z;
  sumflux_regions(g, k, j, i, U, V, W, Z);
  const bool last = iteration == nsub;
  const float rn = 1.0f / (float)nsub;
  float A = bar[WF_RU_M][p], B = bar[WF_RV_M][p], C = bar[WF_WW_M][p];
  if (U) {
    if (last) {
      atomicAdd(&bar[WF_MUU][c], s[WF_U_SAVE][p] / s[WF_MSFUY][c] * A);
      bar[WF_U_SAVE][p] += s[WF_MUU][c] / s[WF_MSFUY][c] * A;
      A = A * rn;
    }
    bar[WF_U][p] += A;
  }
  if (V) {
    if (last) {
      atomicAdd(&bar[WF_MUV][c], s[WF_V_SAVE][p] * s[WF_MSFVX_INV][c] * B);
      bar[WF_V_SAVE][p] += s[WF_MUV][c] * s[WF_MSFVX_INV][c] * B;
      B = B * rn;
    }
    bar[WF_V][p] += B;
  }
  if (W) {
    if (last) {
      bar[WF_WW1][p] += C;
      C = C * rn;
    }
    bar[WF_WW][p] += C;
  }
  if (iteration == 1 && Z) A = B = C = 0.f;
  bar[WF_RU_M][p] = A;
  bar[WF_RV_M][p] = B;
  bar[WF_WW_M][p] = C;
}

// the specified rows of spec_bdyupdate for stagger var (level k < nk)
__device__ __forceinline__ bool spec_row(const Grid& g, char var, int j, int i) {
  const int itf = var == 'u' ? g.ide : g.ide - 1, jtf = var == 'v' ? g.jde : g.jde - 1;
  const int jbe = var == 'v' ? g.jde : g.jde - 1;
  const int its = g.ids, jts = g.jds, jbs = g.jds;
  if ((j == jts || j == jtf - 1) && i >= its && i < itf) return true;
  return j >= jbs + 1 && j < jbe - 1 && (i == its || i == itf - 1);
}

__global__ void k_spec_update(Grid g, float* field, const float* tend, float dt, char var, int nk) {
  WRF_POINT_INDEX(g, k, j, i);
  if (k >= nk || !spec_row(g, var, j, i)) return;
  const size_t p = (size_t)k * g.ny * g.nx + g.i2(j, i);
  field[p] = field[p] + dt * tend[p];
}

__global__ void k_spec_update_adj(Grid g, const float* field_bar, float* tend_bar, float dt, char var, int nk) {
  WRF_POINT_INDEX(g, k, j, i);
  if (k >= nk || !spec_row(g, var, j, i)) return;
  const size_t p = (size_t)k * g.ny * g.nx + g.i2(j, i);
  tend_bar[p] += dt * field_bar[p];
}

// the specified rows of spec_bdyupdate_ph (all levels)
__device__ __forceinline__ bool spec_row_ph(const Grid& g, int j, int i) {
  const int ibs = g.ids, ibe = g.ide - 1, jbs = g.jds, jbe = g.jde - 1;
  if ((j == jbs || j == jbe - 1) && i >= ibs && i < ibe) return true;
  return j >= jbs + 1 && j < jbe - 1 && (i == ibs || i == ibe - 1);
}

__global__ void k_spec_ph(Grid g, S s, float dt) {
  WRF_POINT_INDEX(g, k, j, i);
  if (!spec_row_ph(g, j, i)) return;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const float mt = s[WF_MUTS][c];
  const float mu_old = mt - dt * s[WF_MU_TEND][c];
  float* ph = s[WF_PH];
  ph[p] = ph[p] * mu_old / mt + dt * s[WF_PH_TEND][p] / mt + s[WF_PH_SAVE][p] * (mu_old / mt - 1.0f);
}

__global__ void k_spec_ph_adj(Grid g, S s, S bar, float dt) {
  WRF_POINT_INDEX(g, k, j, i);
  if (!spec_row_ph(g, j, i)) return;
  const int c = g.i2(j, i);
  const size_t p = (size_t)k * g.ny * g.nx + c;
  const float mt = s[WF_MUTS][c];
  const float mu_old = mt - dt * s[WF_MU_TEND][c];
  const float ph = s[WF_PH][p], pt = s[WF_PH_TEND][p], ps = s[WF_PH_SAVE][p];
  const float P = bar[WF_PH][p];
  bar[WF_PH][p] = P * mu_old / mt;
  bar[WF_PH_TEND][p] += dt / mt * P;
  // d/d ph_save = mu_old / mt - 1 = -dt mu_tend / mt, formed without the
  // cancellation of the difference (which float32 would round to a few
  // significant digits)
  bar[WF_PH_SAVE][p] += -(dt * s[WF_MU_TEND][c]) / mt * P;
  // with mu_old = muts - dt mu_tend the update is
  //   ph - dt ((ph + ph_save) mu_tend - ph_tend) / muts, so
  //   d/d mu_tend = -dt (ph + ph_save) / muts
  //   d/d muts    = dt ((ph + ph_save) mu_tend - ph_tend) / muts^2
  // (the second formed directly: the sum of the partial derivatives through
  // mu_old and through muts cancels to a few digits in float32)
  const float mtn = s[WF_MU_TEND][c];
  atomicAdd(&bar[WF_MUTS][c], dt * ((ph + ps) * mtn - pt) / (mt * mt) * P);
  atomicAdd(&bar[WF_MU_TEND][c], -dt * (ph + ps) / mt * P);
}

}  // namespace

int launch_sumflux(const Grid& g, const S& s, int iteration, int nsub, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_sumflux<<<point_grid(g, b3), b3, 0, st>>>(g, s, iteration, nsub);
  return 1;
}

int launch_sumflux_adj(const Grid& g, const S& s, const S& b, int iteration, int nsub, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_sumflux_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, iteration, nsub);
  return 1;
}

int launch_spec_update(const Grid& g, float* field, const float* tend, float dt, char var, bool two_d, cudaStream_t st) {
  const dim3 b3(32, 4);
  Grid g2 = g;
  if (two_d) g2.nz = 1;
  k_spec_update<<<point_grid(g2, b3), b3, 0, st>>>(g2, field, tend, dt, var, two_d ? 1 : g.nz - 1);
  return 1;
}

int launch_spec_update_adj(const Grid& g, const float* field_bar, float* tend_bar, float dt, char var, bool two_d,
                           cudaStream_t st) {
  const dim3 b3(32, 4);
  Grid g2 = g;
  if (two_d) g2.nz = 1;
  k_spec_update_adj<<<point_grid(g2, b3), b3, 0, st>>>(g2, field_bar, tend_bar, dt, var, two_d ? 1 : g.nz - 1);
  return 1;
}

int launch_spec_ph(const Grid& g, const S& s, float dt, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_spec_ph<<<point_grid(g, b3), b3, 0, st>>>(g, s, dt);
  return 1;
}

int launch_spec_ph_adj(const Grid& g, const S& s, const S& b, float dt, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_spec_ph_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b, dt);
  return 1;
}

}  // namespace wrf
