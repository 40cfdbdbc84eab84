// Open lateral-boundary halo copies: set_physical_bc3d / set_physical_bc2d
// (pywrf/wrf_dynamics.py:164-278).
//
// The reference copies the x sides first (their rows reach 4 rows into the y
// halo, which at that moment still holds the previous values) and then the y
// sides.  The copies of one level never touch another level, so the block of
// each (level, field) does both sides with a barrier in between; one launch
// handles a batch of fields.
#include "bc.cuh"

namespace wrf {

// one block per (level, field): the x sides first (their rows reach 4 rows
// into the y halo and read the values the y sides will overwrite), then the
// y sides, separated by a block barrier
// zero_grad_bdy(w) on the specified rows of level k (wrf_boundary.py:358-400):
// rows jbs and jbe-1 (columns [ibs, ibe)), then columns ibs and ibe-1 (rows
// (jbs, jbe-1)) take the value of their inner neighbour; the sources are never
// ring points, so the copies are independent
__device__ __forceinline__ void zero_grad_w_level(const Grid& g, float* w, int k) {
  const int ibs = g.ids, ibe = g.ide - 1, jbs = g.jds, jbe = g.jde - 1;
  const int nxr = ibe - ibs, nyr = jbe - jbs - 2;
  const size_t base = (size_t)k * g.ny * g.nx;
  for (int r = threadIdx.x; r < 2 * nxr + 2 * nyr; r += blockDim.x) {
    int j, i, sj, si;
    if (r < 2 * nxr) {
      const bool top = r >= nxr;
      i = ibs + (top ? r - nxr : r);
      j = top ? jbe - 1 : jbs;
      sj = top ? jbe - 2 : jbs + 1;
      si = (i == ibs) ? ibs + 1 : (i == ibe - 1 ? ibe - 2 : i);
    } else {
      const int q = r - 2 * nxr;
      const bool east = q >= nyr;
      j = jbs + 1 + (east ? q - nyr : q);
      i = east ? ibe - 1 : ibs;
      sj = j;
      si = east ? ibe - 2 : ibs + 1;
    }
    w[base + (size_t)j * g.nx + i] = w[base + (size_t)sj * g.nx + si];
  }
}

// one block per (level, field); with b.zgw set, the blocks of the extra row
// f == b.n apply zero_grad_bdy(w) (w is never one of the batch's fields)
__global__ void __launch_bounds__(256) k_bc(Grid g, BcBatch b) {
  const int k = blockIdx.x, f = blockIdx.y;
  if (b.zgw && f == b.n) {
    if (k < g.nz) zero_grad_w_level(g, b.zgw, k);
    return;
  }
  const BcItem it = b.item[f];
  if (k >= it.k_end) return;  // whole block
  float* d = it.ptr + (it.two_d ? 0 : (size_t)k * g.ny * g.nx);
  const int nx = g.nx, ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  // x sides
  const int r0 = it.two_d ? jds : jds - 4;
  const int r1 = it.two_d ? jde + it.jstag : jde + it.jstag + 4;
  const int rhi0 = (it.two_d || !it.ustag) ? r0 : jds - 5;  // u-like high side starts one row lower
  for (int j = threadIdx.x; j < g.ny; j += blockDim.x) {
    float* row = d + (size_t)j * nx;
    if (j >= r0 && j < r1) {
      const float lo = row[ids];
      row[ids - 1] = lo; row[ids - 2] = lo; row[ids - 3] = lo;
    }
    if (j >= rhi0 && j < r1) {
      if (!it.ustag) {
        const float hi = row[ide - 2];
        row[ide - 1] = hi; row[ide] = hi; row[ide + 1] = hi;
      } else {
        const float hi = row[ide - 1];
        row[ide] = hi; row[ide + 1] = hi; row[ide + 2] = hi;
      }
    }
  }
  __syncthreads();
  // y sides
  const int c1 = ide + it.istag;
  for (int i = ids + threadIdx.x; i < c1; i += blockDim.x) {
    const float lo = d[(size_t)jds * nx + i];
    d[(size_t)(jds - 1) * nx + i] = lo; d[(size_t)(jds - 2) * nx + i] = lo; d[(size_t)(jds - 3) * nx + i] = lo;
    if (!it.vstag) {
      const float hi = d[(size_t)(jde - 2) * nx + i];
      d[(size_t)(jde - 1) * nx + i] = hi; d[(size_t)jde * nx + i] = hi; d[(size_t)(jde + 1) * nx + i] = hi;
    } else {
      const float hi = d[(size_t)(jde - 1) * nx + i];
      d[(size_t)jde * nx + i] = hi; d[(size_t)(jde + 1) * nx + i] = hi; d[(size_t)(jde + 2) * nx + i] = hi;
    }
  }
}

// stagger letter -> copy pattern (wrf_dynamics.py:221-254 and 169-186)
BcItem bc_item(const Grid& g, float* ptr, char var, bool two_d) {
  BcItem it{};
  it.ptr = ptr;
  it.two_d = two_d ? 1 : 0;
  char v = var;
  if (v == 'U') v = 'u';
  if (v == 'V') v = 'v';
  const bool u_like = (v == 'u' || v == 'x');
  const bool v_like = (v == 'v' || v == 'y');
  int istag = -1, jstag = -1;
  if (u_like || v == 'd' || v == 'e') istag = 0;
  if (v_like || v == 'd' || v == 'f') jstag = 0;
  it.ustag = u_like ? 1 : 0;
  it.vstag = v_like ? 1 : 0;
  it.istag = istag;
  it.jstag = jstag;
  if (two_d) {
    it.k_end = 1;
  } else {
    it.k_end = (v == 'e' || v == 'f' || v == 'w') ? g.nz : g.nz - 1;
  }
  return it;
}

int launch_bc(const Grid& g, const BcBatch& b, cudaStream_t st) {
  if (b.n == 0 && !b.zgw) return 0;
  int kmax = b.zgw ? g.nz : 1;
  for (int f = 0; f < b.n; ++f) kmax = b.item[f].k_end > kmax ? b.item[f].k_end : kmax;
  k_bc<<<dim3(kmax, b.n + (b.zgw ? 1 : 0)), 256, 0, st>>>(g, b);
  return 1;
}

}  // namespace wrf
