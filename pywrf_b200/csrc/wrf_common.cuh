// Shared device-side definitions for the ARW step kernels (sm_100a).
//
// Index conventions follow the reference's python-style WRF index sets
// (pywrf/config_params.py:67-99): 3-D fields are [nz][ny][nx], x fastest;
// mass points occupy [ids, ide-1), x-staggered points [ids, ide); the kernels
// write exactly the index regions the reference writes so that halos and
// persistent work buffers evolve identically across steps.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "pywrf_b200.h"

namespace wrf {

// physical constants (pywrf/config_params.py:114-161); kept as doubles so
// that constant sub-expressions are formed the way the reference forms them
// (in double precision on the host) before the float32 tensor operation.
constexpr double G = 9.81;
constexpr double T0 = 300.0;
constexpr double P0 = 100000.0;
constexpr double R_D = 287.0;
constexpr double CPOVCV = 1.4;
constexpr double RVOVRD = 1.608362;
constexpr double RERADIUS = 1.5698588e-7;
constexpr double C_S = 0.25;
constexpr double PRANDTL = 1.0 / 3.0;

// relaxation-zone weights (pywrf/solver.py:440-441)
static __device__ __constant__ float kFcx[5] = {0.f, 5.5555557e-3f, 3.7037039e-3f, 1.8518519e-3f, 0.f};
static __device__ __constant__ float kGcx[5] = {0.f, 1.1111111e-3f, 7.4074074e-4f, 3.7037037e-4f, 0.f};

// scalar slots of WF_DSCAL
enum { DS_DTBC = 0, DS_STEP = 1 };

struct Grid {
  int nx, ny, nz, ids, ide, jds, jde;
  int soundsteps, spec_zone, top_lid;
  float dx, dy, dt, rdx, rdy;
  double dxd, dyd, dtd, rdxd, rdyd;   // the reference's python-float values
  float smdiv, emdiv, epssm;
  float cf1, cf2, cf3, cfn, cfn1;
  __host__ __device__ __forceinline__ int i3(int k, int j, int i) const { return (k * ny + j) * nx + i; }
  __host__ __device__ __forceinline__ int i2(int j, int i) const { return j * nx + i; }
  __host__ __device__ __forceinline__ size_t n3() const { return (size_t)nz * ny * nx; }
  __host__ __device__ __forceinline__ size_t n2() const { return (size_t)ny * nx; }
};

// device view of the state: typed pointers
struct S {
  float* f[WF_COUNT];
  __host__ __device__ __forceinline__ float* operator[](int id) const { return f[id]; }
};

__device__ __forceinline__ float ldg(const float* p) { return __ldg(p); }

// Transcendentals of the equation of state (wpow_eos) and of the
// microphysics (wpow, wexp, wlog).  With WRF_EOS_DOUBLE / WRF_MP_DOUBLE they
// are evaluated in double precision and rounded once to float.
#ifdef WRF_EOS_DOUBLE
__device__ __forceinline__ float wpow_eos(float a, float b) { return (float)pow((double)a, (double)b); }
#else
__device__ __forceinline__ float wpow_eos(float a, float b) { return powf(a, b); }
#endif
#ifdef WRF_MP_DOUBLE
__device__ __forceinline__ float wpow(float a, float b) { return (float)pow((double)a, (double)b); }
__device__ __forceinline__ float wexp(float a) { return (float)exp((double)a); }
__device__ __forceinline__ float wlog(float a) { return (float)log((double)a); }
#else
__device__ __forceinline__ float wpow(float a, float b) { return powf(a, b); }
__device__ __forceinline__ float wexp(float a) { return expf(a); }
__device__ __forceinline__ float wlog(float a) { return logf(a); }
#endif

// 1.0 if ua >= 0 else -1.0 (fortran_sign(1., ua), wrf_dynamics.py:1309-1311)
__device__ __forceinline__ float sgnf(float ua) { return ua >= 0.f ? 1.f : -1.f; }

// x / d, correctly rounded, for a constant d given r = RN(1/d): the quotient
// estimate x*r is corrected once with the exact residual (Markstein's
// theorem: with r within half an ulp of 1/d the result is the correctly
// rounded quotient for normal results), a multiply and two FMAs in place of
// a full IEEE division
__device__ __forceinline__ float divc(float x, float d, float r) {
  const float q = x * r;
  return fmaf(fmaf(-q, d, x), r, q);
}

// 3rd-order upwind-biased face value (wrf_dynamics.py:1313-1320)
__device__ __forceinline__ float flux3(float qm2, float qm1, float q0, float qp1, float ua) {
  constexpr float r12 = 1.0f / 12.0f;
  const float f4 = divc(7.f * (q0 + qm1) - (qp1 + qm2), 12.f, r12);
  return f4 + divc(sgnf(ua) * ((qp1 - qm2) - 3.f * (q0 - qm1)), 12.f, r12);
}

// 5th-order upwind-biased face value (wrf_dynamics.py:1322-1329)
__device__ __forceinline__ float flux5(float qm3, float qm2, float qm1, float q0, float qp1, float qp2,
                                       float ua) {
  constexpr float r60 = 1.0f / 60.0f;
  const float f6 = divc(37.f * (q0 + qm1) - 8.f * (qp1 + qm2) + (qp2 + qm3), 60.f, r60);
  return f6 - divc(sgnf(ua) * ((qp2 - qm3) - 5.f * (qp1 - qm2) + 10.f * (q0 - qm1)), 60.f, r60);
}

#define WRF_POINT_INDEX(g, k, j, i)                          \
  const int i = blockIdx.x * blockDim.x + threadIdx.x;       \
  const int j = blockIdx.y * blockDim.y + threadIdx.y;       \
  const int k = blockIdx.z;                                  \
  if (i >= (g).nx || j >= (g).ny) return;

#define WRF_COLUMN_INDEX(g, j, i)                            \
  const int i = blockIdx.x * blockDim.x + threadIdx.x;       \
  const int j = blockIdx.y * blockDim.y + threadIdx.y;       \
  if (i >= (g).nx || j >= (g).ny) return;

// The lateral relaxation, the specified rows and the final boundary values
// only act on points within a few cells of the domain edge.  In ring mode a kernel runs one thread per
// point of the band: rows [jds, jds+5) and [jde-5, jde) over columns
// [ids, ide], then columns [ids, ids+5) and [ide-5, ide] of the rows
// between - every point those updates touch, once, when the domain spans at
// least 10 rows and 11 columns (else, and in the WRF_FORM_POINT cross-check
// form, the kernels run over every point).
__device__ __forceinline__ bool ring_point(const Grid& g, int r, int& j, int& i) {
  const int w = g.ide + 1 - g.ids;
  if (r < 10 * w) {
    const int rr = r / w;
    i = g.ids + (r - rr * w);
    j = rr < 5 ? g.jds + rr : g.jde - 10 + rr;
    return true;
  }
  r -= 10 * w;
  if (r >= (g.jde - g.jds - 10) * 11) return false;
  const int cc = r % 11;
  j = g.jds + 5 + r / 11;
  i = cc < 5 ? g.ids + cc : g.ide - 10 + cc;
  return true;
}
inline bool ring_fits(const Grid& g) { return g.jde - g.jds >= 10 && g.ide - g.ids >= 11; }
inline int ring_size(const Grid& g) { return 10 * (g.ide + 1 - g.ids) + (g.jde - g.jds - 10) * 11; }

inline dim3 point_grid(const Grid& g, dim3 b) { return dim3((g.nx + b.x - 1) / b.x, (g.ny + b.y - 1) / b.y, g.nz); }
inline dim3 col_grid(const Grid& g, dim3 b) { return dim3((g.nx + b.x - 1) / b.x, (g.ny + b.y - 1) / b.y, 1); }

}  // namespace wrf
