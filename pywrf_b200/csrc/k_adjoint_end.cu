// The end-of-step lateral boundaries as a stand-alone operator with its
// adjoint: spec_bdy_final of u, v, t, ph and qv (wrf_boundary.py:511-587)
// then set_w_surface (wrf_dynamics.py:4218-4324), as the step's
// launch_bdy_final runs them.
//
// spec_bdy_final overwrites the specified rows with msf (bdy + dtbc
// bdy_tend) / mu, where the boundary arrays are data and mu (muus, muvs or
// muts) is state: the reverse hands the row's cotangent to mu and zeroes it.
// set_w_surface overwrites w at the lowest level with a linear function of
// the lowest three levels of u and v (the terrain slope is data): the
// reverse runs first, since the forward's w reads the u and v that
// spec_bdy_final left.
#include "kernels.cuh"

namespace wrf {

namespace {

__device__ __forceinline__ void acc(float* a, size_t q, float v) {
  if (v != 0.f) atomicAdd(a + q, v);
}

__global__ void k_w_surface_adj(Grid g, S s, S b) {
  WRF_COLUMN_INDEX(g, j, i);
  const int its = g.ids, ite = g.ide, jts = g.jds, jte = g.jde, nx = g.nx;
  if (j < jts || j > jte - 2 || i < its || i > ite - 2) return;
  const size_t lev = (size_t)g.ny * nx;
  const float* ht = s[WF_HT];
  const int c = g.i2(j, i);
  const float W = b[WF_W][c];
  b[WF_W][c] = 0.f;
  if (W == 0.f) return;
  const bool jlo = j == jts, jhi = j == jte - 2, ilo = i == its, ihi = i == ite - 2;
  const float mx = (jhi && ihi) ? s[WF_MSFTX][g.i2(jts, its)] : s[WF_MSFTX][c];
  const float Y = s[WF_MSFTY][c] * 0.5f * g.rdy * W;
  const float X = mx * 0.5f * g.rdx * W;
  const float cf[3] = {g.cf1, g.cf2, g.cf3};
  // w += Y * (slope) * cv(column) and X * (slope) * cu(column)
  auto v_at = [&](int cc, float coef) {
    if (coef == 0.f) return;
    for (int k = 0; k < 3; ++k) acc(b[WF_V], (size_t)k * lev + cc, cf[k] * coef);
  };
  auto u_at = [&](int cc, float coef) {
    if (coef == 0.f) return;
    for (int k = 0; k < 3; ++k) acc(b[WF_U], (size_t)k * lev + cc, cf[k] * coef);
  };
  if (jlo && ihi) {
    // the reference differences row jts+1 with itself: no dependence
  } else if (jlo) {
    v_at(c + nx, Y * (ht[c + nx] - ht[c]));
  } else if (jhi) {
    v_at(c, Y * (ht[c] - ht[c - nx]));
  } else {
    v_at(c + nx, Y * (ht[c + nx] - ht[c]));
    v_at(c, Y * (ht[c] - ht[c - nx]));
  }
  if (ilo) {
    u_at(c + 1, X * (ht[c + 1] - ht[c]));
  } else if (ihi) {
    u_at(c, X * (ht[c] - ht[c - 1]));
  } else {
    u_at(c + 1, X * (ht[c + 1] - ht[c]));
    u_at(c, X * (ht[c] - ht[c - 1]));
  }
}

__global__ void k_bdy_final_adj(Grid g, S s, S b) {
  WRF_POINT_INDEX(g, k, j, i);
  const int nz = g.nz, nx = g.nx, ny = g.ny;
  const size_t lev = (size_t)ny * nx, n3 = g.n3();
  const int c = g.i2(j, i);
  const size_t p = k * lev + c;
  const float dtbc = s[WF_DSCAL][DS_DTBC];
  const int its = g.ids, jts = g.jds;
  auto put = [&](float* fb, int bx, const float* mu, float* mub, const float* msf, int ibe, int jbe, int itf, int jtf,
                 int ktf) {
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
    const float F = fb[p];
    fb[p] = 0.f;
    const float m = mu[c];
    acc(mub, c, -F * ((msf ? msf[c] : 1.0f) * val) / (m * m));
  };
  put(b[WF_U], WF_U_BXS, s[WF_MUUS], b[WF_MUUS], s[WF_MSFUY], g.ide, g.jde - 1, g.ide, g.jde - 1, nz - 1);
  put(b[WF_V], WF_V_BXS, s[WF_MUVS], b[WF_MUVS], s[WF_MSFVX], g.ide - 1, g.jde, g.ide - 1, g.jde, nz - 1);
  put(b[WF_T], WF_T_BXS, s[WF_MUTS], b[WF_MUTS], nullptr, g.ide - 1, g.jde - 1, g.ide - 1, g.jde - 1, nz - 1);
  put(b[WF_PH], WF_PH_BXS, s[WF_MUTS], b[WF_MUTS], nullptr, g.ide - 1, g.jde - 1, g.ide - 1, g.jde - 1, nz);
  put(b[WF_MOIST] + n3, WF_QV_BXS, s[WF_MUTS], b[WF_MUTS], nullptr, g.ide - 1, g.jde - 1, g.ide - 1, g.jde - 1,
      nz - 1);
}

}  // namespace

int launch_bdy_final_op(const Grid& g, const S& s, cudaStream_t st) { return launch_bdy_final(g, s, st); }

int launch_bdy_final_op_adj(const Grid& g, const S& s, const S& b, cudaStream_t st) {
  const dim3 b2(32, 8), b3(32, 4);
  k_w_surface_adj<<<col_grid(g, b2), b2, 0, st>>>(g, s, b);
  k_bdy_final_adj<<<point_grid(g, b3), b3, 0, st>>>(g, s, b);
  return 2;
}

}  // namespace wrf
