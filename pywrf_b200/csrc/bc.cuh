// Batched open-boundary halo copies (see k_bc.cu).
#pragma once
#include "wrf_common.cuh"

namespace wrf {

struct BcItem {
  float* ptr;
  int k_end;     // levels copied
  int istag, jstag;
  int ustag, vstag;
  int two_d;
};

constexpr int kBcMax = 24;
struct BcBatch {
  int n = 0;
  BcItem item[kBcMax];
  float* zgw = nullptr;  // w, when the launch also applies zero_grad_bdy(w)
  void add(const BcItem& it) { item[n++] = it; }
};

BcItem bc_item(const Grid& g, float* ptr, char var, bool two_d);
int launch_bc(const Grid& g, const BcBatch& b, cudaStream_t st);
// one field's halo copy and zero_grad_bdy(w) alone, and their adjoints
// (k_adjoint_bc.cu: the incoming cotangent ibar is accumulated)
int launch_halo(const Grid& g, float* field, char var, bool two_d, cudaStream_t st);
int launch_halo_adj(const Grid& g, const float* fbar, float* ibar, char var, bool two_d, cudaStream_t st);
int launch_zero_grad_w(const Grid& g, float* w, cudaStream_t st);
int launch_zero_grad_w_adj(const Grid& g, const float* fbar, float* ibar, cudaStream_t st);

}  // namespace wrf
