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
__global__ void __launch_bounds__(256) k_bc(Grid g, BcBatch b) {
  const int k = blockIdx.x, f = blockIdx.y;
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
  if (b.n == 0) return 0;
  int kmax = 1;
  for (int f = 0; f < b.n; ++f) kmax = b.item[f].k_end > kmax ? b.item[f].k_end : kmax;
  k_bc<<<dim3(kmax, b.n), 256, 0, st>>>(g, b);
  return 1;
}

}  // namespace wrf
