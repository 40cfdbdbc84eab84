// Interface of the tcgen05 BF16 GEMM (k_gemm_tc.cu) and the network kernels
// built on it (k_mlp.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace wrf {

enum GemmEpiKind {
  EPI_F32 = 0,        // out fp32 = acc (+ bias); split reductions write partial sums split_stride apart
  EPI_BIAS_GELU = 1,  // out bf16 = gelu(acc + bias); out_z bf16 = acc + bias (optional)
  EPI_GELU_BWD = 2,   // out bf16 = acc * gelu'(aux)
  EPI_BF16 = 3,       // out bf16 = acc (+ bias)
};

struct GemmEpi {
  int kind;
  const float* bias;          // [N] or null
  const __nv_bfloat16* aux;   // [M][ldo] pre-activation (EPI_GELU_BWD)
  void* out;                  // [M][ldo]
  int ldo;
  long long split_stride;     // elements between the partial sums of two splits (EPI_F32)
  __nv_bfloat16* out_z;       // [M][ldo] pre-activation store (EPI_BIAS_GELU), or null
  __nv_bfloat16* out_t;       // [N][ldt] transposed bf16 copy of the stored values, or null
  int ldt;
  int* err;                   // set to 1 when a bounded wait runs out
};

// C = A B^T on the tensor cores; returns kernels enqueued (1) or WRF_E* with *err
int launch_gemm_tc(const void* A, const void* B, int M, int N, int K, int splits, const GemmEpi& e, cudaStream_t st,
                   const char** err);
// one-time per-device set-up of the GEMM kernel (WRF_OK or WRF_ECUDA)
int gemm_prepare_device();
// number of K splits launch_gemm_tc uses for a requested count
int gemm_splits_used(int K, int splits);

}  // namespace wrf
