// BF16 GEMM on the 5th-generation tensor cores (tcgen05) with fused epilogues,
// the dense part of the per-column microphysics network:
//
//   C[m, n] = sum_k A[m, k] * B[n, k]      A: M x K, B: N x K, both bf16 row-major
//
// (both operands K-major; a product with a transposed operand is fed the
// transposed copy that the producing epilogue writes).  One CTA computes one
// 128 x 128 tile of C, or its part of the K range when the reduction is split:
//
//   warp 0, one lane   TMA producer: 128 x 64 tiles of A and B into a
//                      2-stage ring of 128-byte-swizzled shared buffers (3 CTAs per SM)
//   warp 1, one lane   MMA issuer: tcgen05.mma.cta_group::1.kind::f16,
//                      M = 128, N = 128, K = 16 per instruction, fp32
//                      accumulator in tensor memory (128 lanes x 128 columns);
//                      tcgen05.commit frees each ring slot and finally
//                      signals the epilogue
//   warps 0-3          epilogue: tcgen05.ld of the warp's 32 accumulator
//                      lanes (= tile rows), bias / GELU / GELU' and the stores
//                      (GELU in its tanh form on the hardware tanh instruction)
//
// Every wait on an mbarrier is bounded (kWaitCycles); a wait that runs out
// sets *err, the CTA skips its stores, frees its tensor memory and returns.
// No load uses cluster multicast.
#include <cuda.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <mutex>
#include "kernels.cuh"
#include "tc_gemm.cuh"
#include "tma.cuh"

namespace wrf {
namespace tc {

#ifndef WRF_GEMM_STAGES
#define WRF_GEMM_STAGES 2
#endif
#ifndef WRF_GEMM_WARPS
#define WRF_GEMM_WARPS 4
#endif
constexpr int BM = 128, BN = 128, BK = 64, STAGES = WRF_GEMM_STAGES, kWarps = WRF_GEMM_WARPS, kThreads = 32 * kWarps;
static_assert(kWarps == 4 || kWarps == 8, "the epilogue maps 4 or 8 warps onto the 4 TMEM lane groups");
constexpr uint32_t kTileBytes = BM * BK * 2;         // 16 KB per operand tile
constexpr uint32_t kStageBytes = 2 * kTileBytes;
constexpr uint32_t kTmemCols = BN;                   // fp32 accumulator: 128 lanes x BN columns
constexpr size_t kSmemBytes = STAGES * kStageBytes + 1024 + 128;
constexpr long long kWaitCycles = 4000000000LL;      // ~2 s at the boost clock

using tma::mbar_expect_tx;
using tma::mbar_init;
using tma::mbar_try;
using tma::smem_u32;

// bounded wait for the phase of the given parity to complete
__device__ __noinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
  const long long t0 = clock64();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 255u) == 255u && clock64() - t0 > kWaitCycles) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor of a K-major tile written by TMA with
// 128-byte swizzle: rows of 128 B (64 bf16), 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t desc_k_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);  // start address, 16-byte units
  d |= (uint64_t)1 << 16;                            // leading byte offset (unused by swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;                  // stride byte offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                            // descriptor version of sm_100
  d |= (uint64_t)2 << 61;                            // 128-byte swizzle
  return d;
}

// instruction descriptor: bf16 x bf16 -> fp32, both K-major, M = 128, N = BN
constexpr uint32_t kIdesc = (1u << 4)                  // accumulator format f32
                            | (1u << 7)                // A bf16
                            | (1u << 10)               // B bf16
                            | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 16 consecutive fp32 accumulator columns of this thread's lane (the wait
// for the load is part of the same asm statement, so no use can precede it)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// GELU in its tanh form, 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), on
// the hardware tanh instruction (a few instructions per element, so that the
// epilogue keeps pace with the tensor cores), and its derivative
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kGeluC = 0.7978845608028654f, kGeluA = 0.044715f;
__device__ __forceinline__ float gelu(float x) {
  const float th = tanh_hw(kGeluC * x * (1.0f + kGeluA * x * x));
  return 0.5f * x * (1.0f + th);
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float x2 = x * x;
  const float th = tanh_hw(kGeluC * x * (1.0f + kGeluA * x2));
  return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * kGeluC * (1.0f + 3.0f * kGeluA * x2);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ void store_row16_bf16(__nv_bfloat16* dst, const float (&v)[16]) {
  uint4 a, b;
  a.x = pack_bf16x2(v[0], v[1]);   a.y = pack_bf16x2(v[2], v[3]);
  a.z = pack_bf16x2(v[4], v[5]);   a.w = pack_bf16x2(v[6], v[7]);
  b.x = pack_bf16x2(v[8], v[9]);   b.y = pack_bf16x2(v[10], v[11]);
  b.z = pack_bf16x2(v[12], v[13]); b.w = pack_bf16x2(v[14], v[15]);
  reinterpret_cast<uint4*>(dst)[0] = a;
  reinterpret_cast<uint4*>(dst)[1] = b;
}

// epilogue of 16 accumulator columns n .. n+15 of output row m (split: the
// partial-sum index of a split reduction, 0 otherwise)
__device__ __forceinline__ void epilogue16(const GemmEpi& e, float (&v)[16], int m, int n, int split) {
  if (e.bias && split == 0) {  // (once over the partial sums of a split reduction)
#pragma unroll
    for (int t = 0; t < 16; ++t) v[t] += __ldg(&e.bias[n + t]);
  }
  switch (e.kind) {
    case EPI_F32: {
      float* o = static_cast<float*>(e.out) + (size_t)split * e.split_stride + (size_t)m * e.ldo + n;
#pragma unroll
      for (int t = 0; t < 16; t += 4) *reinterpret_cast<float4*>(o + t) = make_float4(v[t], v[t + 1], v[t + 2], v[t + 3]);
      break;
    }
    case EPI_BIAS_GELU: {
      if (e.out_z) store_row16_bf16(e.out_z + (size_t)m * e.ldo + n, v);
#pragma unroll
      for (int t = 0; t < 16; ++t) v[t] = gelu(v[t]);
      store_row16_bf16(static_cast<__nv_bfloat16*>(e.out) + (size_t)m * e.ldo + n, v);
      break;
    }
    case EPI_GELU_BWD: {
      const __nv_bfloat16* z = e.aux + (size_t)m * e.ldo + n;
#pragma unroll
      for (int t = 0; t < 16; ++t) v[t] *= gelu_grad(__bfloat162float(z[t]));
      store_row16_bf16(static_cast<__nv_bfloat16*>(e.out) + (size_t)m * e.ldo + n, v);
      break;
    }
    default:  // EPI_BF16
      store_row16_bf16(static_cast<__nv_bfloat16*>(e.out) + (size_t)m * e.ldo + n, v);
      break;
  }
  if (e.out_t) {  // transposed copy [N][ldt] of what was stored (bf16)
#pragma unroll
    for (int t = 0; t < 16; ++t) e.out_t[(size_t)(n + t) * e.ldt + m] = __float2bfloat16_rn(v[t]);
  }
}

__global__ void __launch_bounds__(kThreads, 1)
    k_gemm_tc(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, int M, int N, int K,
              int kb_per_split, GemmEpi e) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = smem;
  uint8_t* sB = smem + STAGES * kTileBytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * kStageBytes);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
  const int kb_total = (K + BK - 1) / BK;
  const int kb0 = blockIdx.z * kb_per_split;
  const int nkb = min(kb_per_split, kb_total - kb0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (nkb > 0 && warp == 0 && lane == 0) {
    // producer
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % STAGES;
      const uint32_t ph = (uint32_t)(kb / STAGES) & 1u;
      if (!mbar_wait(&empty[s], ph ^ 1u)) {
        atomicExch(abort_flag, 1);
        break;
      }
      mbar_expect_tx(&full[s], kStageBytes);
      tma_load_2d(sA + s * kTileBytes, &ta, (kb0 + kb) * BK, m0, &full[s]);
      tma_load_2d(sB + s * kTileBytes, &tb, (kb0 + kb) * BK, n0, &full[s]);
    }
  } else if (nkb > 0 && warp == 1 && lane == 0) {
    // MMA issuer
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % STAGES;
      const uint32_t ph = (uint32_t)(kb / STAGES) & 1u;
      if (!mbar_wait(&full[s], ph)) {
        atomicExch(abort_flag, 1);
        break;
      }
      tc_fence_after();
      const uint32_t a0 = smem_u32(sA + s * kTileBytes), b0 = smem_u32(sB + s * kTileBytes);
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk)
        umma_bf16(tmem, desc_k_sw128(a0 + kk * 32), desc_k_sw128(b0 + kk * 32), (kb | kk) != 0 ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(done);  // arrives once every MMA issued above has completed
  }
  __syncwarp();

  // epilogue
  // (the outcome is made uniform over the CTA: tcgen05.ld is warp-collective)
  if (!(nkb > 0 && mbar_wait(done, 0))) atomicExch(abort_flag, 1);
  tc_fence_after();
  __syncthreads();
  const bool ok = *abort_flag == 0;
  if (!ok && threadIdx.x == 0 && e.err) atomicExch(e.err, 1);
  if (ok) {
    // warp w reads TMEM lane group w % 4 (rows 32 (w % 4) ..); with 8 warps
    // the two warps of a lane group take half of the columns each
    const int lg = warp & 3;
    constexpr int kChunks = BN / 16 / (kWarps / 4);
    const int c0 = (warp >> 2) * kChunks;
    const int r = lg * 32 + lane;
    const int m = m0 + r;
    const bool row = m < M;
    const uint32_t trow = tmem + ((uint32_t)(lg * 32) << 16);
    for (int c = c0; c < c0 + kChunks; ++c) {
      const int n = n0 + c * 16;
      if (n >= N) break;  // N is a multiple of 16
      float v[16];
      tmem_ld16(trow + (uint32_t)(c * 16), v);
      if (!row) continue;
      epilogue16(e, v, m, n, blockIdx.z);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}


// ------------------------------------------------------------ persistent form
// One CTA per SM for products without a split reduction and K <= 512 (every
// layer of the network's forward pass): the CTA keeps its 128-row slice of B
// (the weights, K x 128 bf16 = up to 128 KB) resident in shared memory for the
// whole launch and streams the 128-row tiles of A it owns (m-tiles r, r + R,
// ... of its n-tile) through a ring of kPStages TMA buffers; the accumulator
// is double-buffered in tensor memory (2 x 128 columns), so the epilogue of one
// tile overlaps the MMAs of the next.
//   warp 0 (one lane)  TMA: the B slice once, then A tiles into the ring
//   warp 1 (one lane)  tcgen05.mma into accumulator t % 2; tcgen05.commit
//                      frees ring slots and marks the accumulator full
//   warps 2..          epilogue (kPEpi warps): warp w drains TMEM lane group
//                      w % 4 (a share of its columns), then marks the
//                      accumulator empty
// Every wait is bounded and also gives up once another role has aborted.
#ifndef WRF_GEMM_PEPI
#define WRF_GEMM_PEPI 8
#endif
// kPEpi epilogue warps (a multiple of 4): warp 2 + e drains lane group
// (2 + e) % 4, columns chunks e / 4, e / 4 + kPEpi / 4, ...
constexpr int kPStages = 4, kPEpi = WRF_GEMM_PEPI, kPWarps = 2 + kPEpi, kPThreads = 32 * kPWarps, kPMaxKb = 8;
static_assert(kPEpi % 4 == 0 && kPEpi >= 4, "epilogue warps come in lane-group quadruples");
constexpr uint32_t kPTmemCols = 2 * BN;

__device__ __noinline__ bool mbar_wait_or_abort(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
  const long long t0 = clock64();
  for (uint32_t it = 0;; ++it) {
    if (mbar_try(b, parity)) return true;
    if ((it & 255u) == 255u && (*abort_flag || clock64() - t0 > kWaitCycles)) return false;
  }
}

__global__ void __launch_bounds__(kPThreads, 1)
    k_gemm_tc_persist(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, int M, int N,
                      int K, GemmEpi e) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int kbt = K / BK;
  uint8_t* sB = smem;                                 // kbt boxes of 128 x 64
  uint8_t* sA = smem + (size_t)kbt * kTileBytes;      // kPStages boxes of 128 x 64
  uint64_t* bar = reinterpret_cast<uint64_t*>(sA + (size_t)kPStages * kTileBytes);
  uint64_t* full = bar;                   // [kPStages]
  uint64_t* empty = full + kPStages;      // [kPStages]
  uint64_t* tfull = empty + kPStages;     // [2]
  uint64_t* tempty = tfull + 2;           // [2]
  uint64_t* bready = tempty + 2;          // [1]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bready + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nt = (N + BN - 1) / BN, mt = (M + BM - 1) / BM;
  const int ntile = blockIdx.x % nt, rank = blockIdx.x / nt, nrank = gridDim.x / nt;
  const int n0 = ntile * BN;
  const int my_tiles = rank < mt ? (mt - 1 - rank) / nrank + 1 : 0;

  if (threadIdx.x == 0) {
    for (int q = 0; q < kPStages; ++q) {
      mbar_init(&full[q], 1);
      mbar_init(&empty[q], 1);
    }
    for (int q = 0; q < 2; ++q) {
      mbar_init(&tfull[q], 1);
      mbar_init(&tempty[q], kPEpi);  // one arrive per epilogue warp
    }
    mbar_init(bready, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&ta)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tb)) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kPTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (my_tiles > 0 && warp == 0 && lane == 0) {
    // producer
    mbar_expect_tx(bready, (uint32_t)kbt * kTileBytes);
    for (int kb = 0; kb < kbt; ++kb) tma_load_2d(sB + (size_t)kb * kTileBytes, &tb, kb * BK, n0, bready);
    int it = 0;
    for (int t = 0; t < my_tiles && !*abort_flag; ++t) {
      const int m0 = (rank + t * nrank) * BM;
      for (int kb = 0; kb < kbt; ++kb, ++it) {
        const int q = it % kPStages;
        const uint32_t ph = (uint32_t)(it / kPStages) & 1u;
        if (!mbar_wait_or_abort(&empty[q], ph ^ 1u, abort_flag)) {
          *abort_flag = 1;
          break;
        }
        mbar_expect_tx(&full[q], kTileBytes);
        tma_load_2d(sA + (size_t)q * kTileBytes, &ta, kb * BK, m0, &full[q]);
      }
    }
  } else if (my_tiles > 0 && warp == 1 && lane == 0) {
    // MMA issuer
    bool ok = mbar_wait_or_abort(bready, 0, abort_flag);
    int it = 0;
    for (int t = 0; ok && t < my_tiles; ++t) {
      const int buf = t & 1;
      const uint32_t use = (uint32_t)(t >> 1) & 1u;
      if (!mbar_wait_or_abort(&tempty[buf], use ^ 1u, abort_flag)) { ok = false; break; }
      tc_fence_after();
      const uint32_t acc = tmem + (uint32_t)(buf * BN);
      for (int kb = 0; kb < kbt; ++kb, ++it) {
        const int q = it % kPStages;
        const uint32_t ph = (uint32_t)(it / kPStages) & 1u;
        if (!mbar_wait_or_abort(&full[q], ph, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const uint32_t a0 = smem_u32(sA + (size_t)q * kTileBytes), b0 = smem_u32(sB + (size_t)kb * kTileBytes);
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)
          umma_bf16(acc, desc_k_sw128(a0 + kk * 32), desc_k_sw128(b0 + kk * 32), (kb | kk) != 0 ? 1u : 0u);
        umma_commit(&empty[q]);
      }
      if (!ok) break;
      umma_commit(&tfull[buf]);  // arrives once every MMA of this tile has completed
    }
    if (!ok) *abort_flag = 1;
  } else if (my_tiles > 0 && warp >= 2) {
    // epilogue
    const int lg = warp & 3;
    const uint32_t trow = tmem + ((uint32_t)(lg * 32) << 16);
    for (int t = 0; t < my_tiles; ++t) {
      const int buf = t & 1;
      const uint32_t use = (uint32_t)(t >> 1) & 1u;
      // the lanes' outcome is made uniform: tcgen05.ld is warp-collective
      const bool ready = __all_sync(0xffffffffu, mbar_wait_or_abort(&tfull[buf], use, abort_flag));
      if (!ready) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const int m = (rank + t * nrank) * BM + lg * 32 + lane;
      for (int c = (warp - 2) / 4; c < BN / 16; c += kPEpi / 4) {
        const int n = n0 + c * 16;
        if (n >= N) break;  // N is a multiple of 16
        float v[16];
        tmem_ld16(trow + (uint32_t)(buf * BN + c * 16), v);
        if (m < M) epilogue16(e, v, m, n, 0);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[buf])) : "memory");
    }
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && *abort_flag && e.err) atomicExch(e.err, 1);
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kPTmemCols) : "memory");
  }
}

// ---------------------------------------------------------------- host side
using tma::EncodeTiled;
using tma::encoder;

// 2-D bf16 row-major [rows][cols] operand, 128 x 64 boxes, 128-byte swizzle;
// rows past the end read as zeros
bool make_map(CUtensorMap* map, const void* ptr, int rows, int cols, const char** err) {
  EncodeTiled enc = encoder(err);
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)BM};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    *err = "cuTensorMapEncodeTiled rejected an operand (pointer alignment or shape)";
    return false;
  }
  return true;
}

}  // namespace tc

// the kernel's dynamic shared-memory limit, set once per device (the first
// call should come before any stream capture)
namespace {
constexpr int kMaxDev = 64;
int g_sm_count[kMaxDev] = {};

size_t persist_smem(int kbt) {
  return (size_t)(kbt + tc::kPStages) * tc::kTileBytes + 1024 + 256;
}
}  // namespace

int gemm_prepare_device() {
  static bool done[kMaxDev] = {};
  static std::mutex mu;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return WRF_ECUDA;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return WRF_OK;
  if (cudaFuncSetAttribute(tc::k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::kSmemBytes) !=
          cudaSuccess ||
      cudaFuncSetAttribute(tc::k_gemm_tc_persist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)persist_smem(tc::kPMaxKb)) != cudaSuccess ||
      cudaDeviceGetAttribute(&g_sm_count[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return WRF_ECUDA;
  done[dev] = true;
  return WRF_OK;
}

int launch_gemm_tc(const void* A, const void* B, int M, int N, int K, int splits, const GemmEpi& e, cudaStream_t st,
                   const char** err) {
  using namespace tc;
  if (!A || !B || !e.out) { *err = "gemm: null operand"; return WRF_EINVAL; }
  if (M < 1 || N < 16 || K < 64 || (N % 16) || (K % 64)) {
    *err = "gemm: needs M >= 1, N a multiple of 16, K a multiple of 64";
    return WRF_EINVAL;
  }
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15u) {
    *err = "gemm: operands must be 16-byte aligned";
    return WRF_EINVAL;
  }
  if (e.ldo < N || (e.ldo % 8) || (reinterpret_cast<uintptr_t>(e.out) & 15u)) {
    *err = "gemm: output leading dimension must be >= N and a multiple of 8, output 16-byte aligned";
    return WRF_EINVAL;
  }
  if (e.kind < EPI_F32 || e.kind > EPI_BF16 || (e.kind == EPI_GELU_BWD && !e.aux) ||
      (e.out_t && e.ldt < M) || (e.kind != EPI_F32 && splits != 1)) {
    *err = "gemm: bad epilogue (kind, aux, transposed leading dimension, or a split reduction with a bf16 output)";
    return WRF_EINVAL;
  }
  const int kb_total = K / BK;
  if (splits < 1) splits = 1;
  if (splits > kb_total) splits = kb_total;
  const int kper = (kb_total + splits - 1) / splits;
  splits = (kb_total + kper - 1) / kper;  // every split gets at least one k block
  CUtensorMap ma, mb;
  if (!make_map(&ma, A, M, K, err) || !make_map(&mb, B, N, K, err)) return WRF_EINVAL;
  if (gemm_prepare_device() != WRF_OK) {
    *err = "gemm: cannot reserve the shared memory of the tile ring";
    return WRF_ECUDA;
  }
  if (splits == 1 && kb_total <= kPMaxKb) {
    // persistent form: one CTA per SM, the CTAs of an n-tile share its m-tiles
    int dev = 0;
    cudaGetDevice(&dev);
    const int nt = (N + BN - 1) / BN, mt = (M + BM - 1) / BM;
    const int nsm = g_sm_count[dev] > 0 ? g_sm_count[dev] : 148;
    const int nrank = std::max(1, std::min(mt, nsm / nt));
    k_gemm_tc_persist<<<nt * nrank, kPThreads, persist_smem(kb_total), st>>>(ma, mb, M, N, K, e);
    return 1;
  }
  const dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM, splits);
  k_gemm_tc<<<grid, kThreads, kSmemBytes, st>>>(ma, mb, M, N, K, kper, e);
  return 1;
}

int gemm_splits_used(int K, int splits) {
  const int kb_total = K / tc::BK;
  if (splits < 1) splits = 1;
  if (splits > kb_total) splits = kb_total;
  const int kper = (kb_total + splits - 1) / splits;
  return (kb_total + kper - 1) / kper;
}

}  // namespace wrf
