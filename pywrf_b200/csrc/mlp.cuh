// The per-column microphysics network: data layout shared by the feature,
// target, apply and training kernels (k_mlp.cu, k_wsm6.cu) and the driver.
//
// A column is one mass column of the WSM6 block, i in [ids+1, ide-2),
// j in [jds+1, jde-2), numbered col = (j - jds - 1) * ncx + (i - ids - 1).
// Features of a column (row of the input matrix), variable-major over the km
// mass levels: T, p, rho, qv, qc, qr, qi, qs, qg (hydrometeors as
// log(max(q, 0) + 1e-12)), each standardised with the table's mean and
// 1/std; padded with zeros to d0 (a multiple of 64).  Outputs (row of the
// output matrix), standardised the same way: increments of theta, qv, qc,
// qr, qi, qs, qg per level over the microphysics call, then the step's
// rain, snow and graupel (rainncv, snowncv, graupelncv); padded to d4 (a
// multiple of 64: it is the reduction width of the first input-gradient product).
#pragma once
#include "wrf_common.cuh"

namespace wrf {

constexpr int kMlpLayers = 4;
constexpr int kFeatVars = 9;       // T p rho qv qc qr qi qs qg
constexpr int kRawVars = 10;       // the features + theta perturbation (harvest only)
constexpr int kOutVars = 7;        // theta qv qc qr qi qs qg increments
constexpr int kOutPrecip = 3;      // rainncv snowncv graupelncv
constexpr float kLogFloor = 1.0e-12f;
// upper bound of the scheme's fall speeds (m/s) used to bound one step's precipitation
constexpr float kMlpMaxFall = 15.0f;

struct MlpLayout {
  int km, ncx, ncy, ncols;
  int nfeat, d0;   // 9 km, rounded up to 64
  int nout, d4;    // 7 km + 3, rounded up to 64
  __host__ __device__ static MlpLayout make(int nx, int ny, int nz, int ids, int ide, int jds, int jde) {
    MlpLayout L;
    L.km = nz - 1;
    L.ncx = ide - ids - 3;
    L.ncy = jde - jds - 3;
    L.ncols = L.ncx * L.ncy;
    L.nfeat = kFeatVars * L.km;
    L.d0 = (L.nfeat + 63) / 64 * 64;
    L.nout = kOutVars * L.km + kOutPrecip;
    L.d4 = (L.nout + 63) / 64 * 64;
    (void)nx; (void)ny;
    return L;
  }
};

// normalisation table offsets (fp32): in_mean[d0], in_rstd[d0], out_mean[d4], out_std[d4]
__host__ __device__ inline int norm_in_mean(const MlpLayout&) { return 0; }
__host__ __device__ inline int norm_in_rstd(const MlpLayout& L) { return L.d0; }
__host__ __device__ inline int norm_out_mean(const MlpLayout& L) { return 2 * L.d0; }
__host__ __device__ inline int norm_out_std(const MlpLayout& L) { return 2 * L.d0 + L.d4; }
__host__ __device__ inline int norm_size(const MlpLayout& L) { return 2 * L.d0 + 2 * L.d4; }

struct MlpNetDev {
  int dims[kMlpLayers + 1];
  const void* w[kMlpLayers];
  const float* b[kMlpLayers];
  const float* norm;
  float tol_neg, tol_sat;
};

struct MlpWorkDev {
  int capacity;
  void* x;        // bf16 [capacity][d0]
  void* h[2];     // bf16 [capacity][hidden]
  float* y;       // fp32 [capacity][d4]
  int* list;      // [0] rejected count, [1..4] quiet / rejection-reason counters, [16 + n] j * nx + i
  int* err;       // wait-timeout flag of the GEMMs
  void* colstat;  // optional uint8 [capacity]: 0 network, 1 quiet, 2 rejected
};

// one-time per-device set-up of the network's kernels (shared-memory limits);
// the first call on a device should come before any stream capture
int mlp_prepare_device();
// features of the state's columns into x (bf16, standardised) or raw (fp32
// [ncols][10 km]: the nine variables and theta perturbation, unstandardised)
int launch_mlp_features(const Grid& g, const S& s, const MlpLayout& L, const float* norm, void* x, float* raw,
                        cudaStream_t st);
// harvest targets: raw increments over the call ([ncols][nout]) from the raw features before it
int launch_mlp_targets(const Grid& g, const S& s, const MlpLayout& L, const float* raw_in, float* raw_out,
                       cudaStream_t st);
// training-side kernels (k_mlp.cu); each returns the kernels enqueued
int launch_mlp_normalize(const MlpLayout& L, const float* norm, const float* raw_in, const float* raw_out, long long n,
                         void* x, float* t, cudaStream_t st);
int launch_mse_grad(const float* y, const float* t, int M, int N, int nvalid, float scale, void* dy, void* dyt,
                    float* loss, cudaStream_t st);
int launch_rowsum_bf16(const void* a, int rows, int cols, float* out, cudaStream_t st);
int launch_adam(float* w, const float* gpart, int nsplit, long long split_stride, float* m, float* v, int R, int C,
                void* wb, void* wtb, float lr, float b1, float b2, float eps, float wd, float bc1, float bc2,
                cudaStream_t st);
int launch_transpose_bf16(const void* a, int R, int C, void* out, cudaStream_t st);
// the network's four products on m rows: x -> h0 -> h1 -> h0 -> y (bias + GELU fused)
int launch_mlp_forward(const MlpNetDev& net, const void* x, int m, void* h0, void* h1, float* y, int* errflag,
                       cudaStream_t st, const char** err);
// surrogate microphysics of one step: features, the network, apply + gate, WSM6 on flagged columns
int launch_physics_mlp(const Grid& g, const S& s, const MlpNetDev& net, const MlpWorkDev& work, cudaStream_t st,
                       const char** err);

}  // namespace wrf
