// relax_bdytend at one point (wrf_boundary.py:52-147), shared by the step's
// k_relax / k_relax_qv (k_prep.cu) and the stand-alone operator and its
// adjoint (k_adjoint.cu).
#pragma once
#include "wrf_common.cuh"

namespace wrf {

// one relaxation-zone point of relax_bdytend (wrf_boundary.py:52-147).
// ``fld(k, j, i)`` returns the coupled field value; ibe/jbe per stagger.
template <typename F>
__device__ __forceinline__ bool relax_point(const Grid& g, const S& s, int bx, int k, int j, int i, int ibe, int jbe,
                                            int nzb, F fld, float dtbc, float* out) {
  const int ibs = g.ids, jbs = g.jds, nx = g.nx, ny = g.ny;
  const float* xs = s[bx + 0];
  const float* xe = s[bx + 1];
  const float* ys = s[bx + 2];
  const float* ye = s[bx + 3];
  const float* txs = s[bx + 4];
  const float* txe = s[bx + 5];
  const float* tys = s[bx + 6];
  const float* tye = s[bx + 7];
  (void)nzb;
  auto yv = [&](const float* b, const float* t, int bb, int ii) {
    const size_t q = ((size_t)k * 5 + bb) * nx + ii;
    return b[q] + dtbc * t[q];
  };
  auto xv = [&](const float* b, const float* t, int jj, int bb) {
    const size_t q = ((size_t)k * ny + jj) * 5 + bb;
    return b[q] + dtbc * t[q];
  };
  for (int b = 1; b <= 3; ++b) {
    if (i >= ibs + b && i < ibe - b) {
      if (j == jbs + b) {
        const float f0 = yv(ys, tys, b, i) - fld(k, j, i);
        const float f1 = yv(ys, tys, b, i - 1) - fld(k, j, i - 1);
        const float f2 = yv(ys, tys, b, i + 1) - fld(k, j, i + 1);
        const float f3 = yv(ys, tys, b - 1, i) - fld(k, j - 1, i);
        const float f4 = yv(ys, tys, b + 1, i) - fld(k, j + 1, i);
        *out = *out + kFcx[b] * f0 - kGcx[b] * (f1 + f2 + f3 + f4 - 4.0f * f0);
        return true;
      }
      if (j == jbe - 1 - b) {
        const float f0 = yv(ye, tye, b, i) - fld(k, j, i);
        const float f1 = yv(ye, tye, b, i - 1) - fld(k, j, i - 1);
        const float f2 = yv(ye, tye, b, i + 1) - fld(k, j, i + 1);
        const float f3 = yv(ye, tye, b - 1, i) - fld(k, j + 1, i);
        const float f4 = yv(ye, tye, b + 1, i) - fld(k, j - 1, i);
        *out = *out + kFcx[b] * f0 - kGcx[b] * (f1 + f2 + f3 + f4 - 4.0f * f0);
        return true;
      }
    }
    if (j >= jbs + b + 1 && j < jbe - b - 1) {
      if (i == ibs + b) {
        const float f0 = xv(xs, txs, j, b) - fld(k, j, i);
        const float f1 = xv(xs, txs, j - 1, b) - fld(k, j - 1, i);
        const float f2 = xv(xs, txs, j + 1, b) - fld(k, j + 1, i);
        const float f3 = xv(xs, txs, j, b - 1) - fld(k, j, i - 1);
        const float f4 = xv(xs, txs, j, b + 1) - fld(k, j, i + 1);
        *out = *out + kFcx[b] * f0 - kGcx[b] * (f1 + f2 + f3 + f4 - 4.0f * f0);
        return true;
      }
      if (i == ibe - 1 - b) {
        const float f0 = xv(xe, txe, j, b) - fld(k, j, i);
        const float f1 = xv(xe, txe, j - 1, b) - fld(k, j - 1, i);
        const float f2 = xv(xe, txe, j + 1, b) - fld(k, j + 1, i);
        const float f3 = xv(xe, txe, j, b - 1) - fld(k, j, i + 1);
        const float f4 = xv(xe, txe, j, b + 1) - fld(k, j, i - 1);
        *out = *out + kFcx[b] * f0 - kGcx[b] * (f1 + f2 + f3 + f4 - 4.0f * f0);
        return true;
      }
    }
  }
  return false;
}

// distance b (1..3) of (j, i) from the boundary if relax_point relaxes it,
// else 0 (same zone tests, same order)
__device__ __forceinline__ int relax_zone_b(const Grid& g, int j, int i, int ibe, int jbe) {
  const int ibs = g.ids, jbs = g.jds;
  for (int b = 1; b <= 3; ++b) {
    if (i >= ibs + b && i < ibe - b && (j == jbs + b || j == jbe - 1 - b)) return b;
    if (j >= jbs + b + 1 && j < jbe - b - 1 && (i == ibs + b || i == ibe - 1 - b)) return b;
  }
  return 0;
}

}  // namespace wrf
