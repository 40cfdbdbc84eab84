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

}  // namespace wrf
