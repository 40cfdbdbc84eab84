// Tensor-memory-accelerator (TMA) tile loads and shared-memory mbarriers,
// shared by the tensor-core GEMM (k_gemm_tc.cu) and the tiled advection
// (k_advect_tiled.cu).  No load here uses cluster multicast.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace wrf {
namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

// one arrival that also announces the bytes the phase's copies will deliver
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

// true once the phase of the given parity has completed
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait: gives up after ~limit_cycles SM cycles or once *abort is set
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b, uint32_t parity, volatile int* abort,
                                                  long long limit_cycles) {
  const long long t0 = clock64();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 255u) == 255u && (*abort || clock64() - t0 > limit_cycles)) return false;
  }
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* b, uint32_t parity, long long limit_cycles) {
  if (mbar_try(b, parity)) return true;  // the common case: no clock read
  const long long t0 = clock64();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 255u) == 255u && clock64() - t0 > limit_cycles) return false;
  }
}

// box of a 4-D tensor map (x fastest) at integer coordinates into shared
// memory; completion is signalled on bar with the box's byte count
__device__ __forceinline__ void load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// host: the driver's cuTensorMapEncodeTiled, fetched once (null with *err set
// when the driver does not provide it)
using EncodeTiled = decltype(&cuTensorMapEncodeTiled);
EncodeTiled encoder(const char** err);

// host: map of nw fp32 arrays [nz][ny][nx] laid end to end (x fastest),
// boxes of bw x bh x 1 x 1 elements; out-of-range elements read as zero.
// Needs a 16-byte aligned base, nx a multiple of 4 and bw a multiple of 4.
bool encode_f32_4d(CUtensorMap* map, const float* base, int nx, int ny, int nz, int nw, int bw, int bh,
                   const char** err);

}  // namespace tma
}  // namespace wrf
