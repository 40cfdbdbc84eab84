// Open lateral-boundary halo copies: set_physical_bc3d / set_physical_bc2d
// (pywrf/wrf_dynamics.py:164-278).
//
// The reference copies the x sides first (their rows reach 4 rows into the y
// halo, which at that moment still holds the previous values) and then the y
// sides.  Two launches reproduce that order exactly: phase X (one thread per
// (field, k, row)) and phase Y (one thread per (field, k, column)).  Each
// launch handles a batch of fields.
#include "bc.cuh"

namespace wrf {

__global__ void k_bc_x(Grid g, BcBatch b) {
  const int f = blockIdx.z;
  if (f >= b.n) return;
  const BcItem it = b.item[f];
  const int k = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= it.k_end || j >= g.ny) return;
  float* d = it.ptr;
  const int ids = g.ids, ide = g.ide, jds = g.jds, jde = g.jde;
  const size_t row = it.two_d ? (size_t)j * g.nx : ((size_t)k * g.ny + j) * g.nx;
  if (it.two_d) {
    const int r0 = jds, r1 = jde + it.jstag;
    if (j < r0 || j >= r1) return;
    const float lo = d[row + ids];
    d[row + ids - 1] = lo; d[row + ids - 2] = lo; d[row + ids - 3] = lo;
    if (!it.ustag) {
      const float hi = d[row + ide - 2];
      d[row + ide - 1] = hi; d[row + ide] = hi; d[row + ide + 1] = hi;
    } else {
      const float hi = d[row + ide - 1];
      d[row + ide] = hi; d[row + ide + 1] = hi; d[row + ide + 2] = hi;
    }
    return;
  }
  const int r0 = jds - 4, r1 = jde + it.jstag + 4;
  if (j >= r0 && j < r1) {
    const float lo = d[row + ids];
    d[row + ids - 1] = lo; d[row + ids - 2] = lo; d[row + ids - 3] = lo;
  }
  if (!it.ustag) {
    if (j >= r0 && j < r1) {
      const float hi = d[row + ide - 2];
      d[row + ide - 1] = hi; d[row + ide] = hi; d[row + ide + 1] = hi;
    }
  } else if (j >= jds - 5 && j < r1) {
    const float hi = d[row + ide - 1];
    d[row + ide] = hi; d[row + ide + 1] = hi; d[row + ide + 2] = hi;
  }
}

__global__ void k_bc_y(Grid g, BcBatch b) {
  const int f = blockIdx.z;
  if (f >= b.n) return;
  const BcItem it = b.item[f];
  const int k = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= it.k_end) return;
  const int c0 = g.ids, c1 = g.ide + it.istag;
  if (i < c0 || i >= c1) return;
  float* d = it.ptr + (it.two_d ? 0 : (size_t)k * g.ny * g.nx);
  const int nx = g.nx, jds = g.jds, jde = g.jde;
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
  dim3 blk(128, 1, 1);
  k_bc_x<<<dim3((g.ny + 127) / 128, kmax, b.n), blk, 0, st>>>(g, b);
  k_bc_y<<<dim3((g.nx + 127) / 128, kmax, b.n), blk, 0, st>>>(g, b);
  return 2;
}

}  // namespace wrf
