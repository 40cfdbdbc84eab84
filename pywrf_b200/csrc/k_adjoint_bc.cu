// Adjoints of the halo copies: set_physical_bc3d / set_physical_bc2d
// (wrf_dynamics.py:164-278) and zero_grad_bdy of w (wrf_boundary.py:358-400).
//
// Both are sequences of copies, so after them every point holds the incoming
// value of one point, its source (itself where nothing was copied).  For the
// open-boundary copies the source of (j, i) is found by undoing the y sides
// (applied last: rows jds-3 .. jds-1 from row jds, and the high rows from
// jde-2, or jde-1 for v-like staggers, on the columns [ids, ide + istag)) and
// then the x sides (applied first, on their rows: columns ids-3 .. ids-1
// from ids, the high columns from ide-2, or ide-1 for u-like staggers).  The
// adjoint adds each point's outgoing cotangent into its source's incoming
// cotangent (atomically: a source feeds up to seven points).
#include "bc.cuh"

namespace wrf {

namespace {

__device__ __forceinline__ void bc_source(const Grid& g, const BcItem& it, int j, int i, int& sj, int& si) {
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  int jj = j, ii = i;
  if (i >= ids && i < ide + it.istag) {  // y sides
    if (j >= jds - 3 && j <= jds - 1) jj = jds;
    else if (!it.vstag && j >= jde - 1 && j <= jde + 1) jj = jde - 2;
    else if (it.vstag && j >= jde && j <= jde + 2) jj = jde - 1;
  }
  const int r0 = it.two_d ? jds : jds - 4;
  const int r1 = it.two_d ? jde + it.jstag : jde + it.jstag + 4;
  const int rhi0 = (it.two_d || !it.ustag) ? r0 : jds - 5;
  if (jj >= r0 && jj < r1 && ii >= ids - 3 && ii <= ids - 1) {
    ii = ids;
  } else if (jj >= rhi0 && jj < r1) {
    if (!it.ustag && ii >= ide - 1 && ii <= ide + 1) ii = ide - 2;
    else if (it.ustag && ii >= ide && ii <= ide + 2) ii = ide - 1;
  }
  sj = jj;
  si = ii;
}

__global__ void k_bc_adj(Grid g, BcItem it, const float* fbar, float* ibar) {
  WRF_POINT_INDEX(g, k, j, i);
  const size_t base = it.two_d ? 0 : (size_t)k * g.ny * g.nx;
  float v = fbar[base + (size_t)j * g.nx + i];
  if (v == 0.f) return;
  int sj = j, si = i;
  if (k < it.k_end) bc_source(g, it, j, i, sj, si);
  atomicAdd(&ibar[base + (size_t)sj * g.nx + si], v);
}

// zero_grad_bdy(w): rows jbs and jbe-1 take row jbs+1 / jbe-2 (corners the
// diagonal neighbour), then columns ibs and ibe-1 of the rows between take
// columns ibs+1 / ibe-2; the sources are never overwritten
__global__ void k_zero_grad_w_adj(Grid g, const float* fbar, float* ibar) {
  WRF_POINT_INDEX(g, k, j, i);
  const int ibs = g.ids, ibe = g.ide - 1, jbs = g.jds, jbe = g.jde - 1;
  const size_t base = (size_t)k * g.ny * g.nx;
  const float v = fbar[base + (size_t)j * g.nx + i];
  if (v == 0.f) return;
  int sj = j, si = i;
  if ((j == jbs || j == jbe - 1) && i >= ibs && i < ibe) {
    sj = j == jbs ? jbs + 1 : jbe - 2;
    si = i == ibs ? ibs + 1 : (i == ibe - 1 ? ibe - 2 : i);
  } else if (j > jbs && j < jbe - 1 && (i == ibs || i == ibe - 1)) {
    si = i == ibs ? ibs + 1 : ibe - 2;
  }
  atomicAdd(&ibar[base + (size_t)sj * g.nx + si], v);
}

}  // namespace

int launch_halo(const Grid& g, float* field, char var, bool two_d, cudaStream_t st) {
  BcBatch b;
  b.add(bc_item(g, field, var, two_d));
  return launch_bc(g, b, st);
}

int launch_halo_adj(const Grid& g, const float* fbar, float* ibar, char var, bool two_d, cudaStream_t st) {
  const BcItem it = bc_item(g, nullptr, var, two_d);
  Grid g2 = g;
  if (two_d) g2.nz = 1;
  const dim3 b3(32, 4);
  k_bc_adj<<<point_grid(g2, b3), b3, 0, st>>>(g2, it, fbar, ibar);
  return 1;
}

int launch_zero_grad_w(const Grid& g, float* w, cudaStream_t st) {
  BcBatch b;
  b.zgw = w;
  return launch_bc(g, b, st);
}

int launch_zero_grad_w_adj(const Grid& g, const float* fbar, float* ibar, cudaStream_t st) {
  const dim3 b3(32, 4);
  k_zero_grad_w_adj<<<point_grid(g, b3), b3, 0, st>>>(g, fbar, ibar);
  return 1;
}

}  // namespace wrf
