// Data kernels of the per-column microphysics network (layout in mlp.cuh):
//   k_mlp_features   state columns -> standardised bf16 feature rows (or raw fp32 rows for the harvest)
//   k_mlp_targets    raw increments of one microphysics call (harvest)
//   k_mlp_normalize  raw harvest rows -> bf16 training inputs, fp32 standardised targets
//   k_mse_grad       d(loss)/dy of the mean squared error, row-major and transposed bf16
//   k_rowsum_bf16    bias gradients (row sums of a transposed gradient)
//   k_adam           Adam step on fp32 master weights, refreshing the bf16 copy and its transpose
//   k_transpose_bf16 transposed copy of a bf16 matrix
// The network's products run on the tensor cores (k_gemm_tc.cu).
#include <cuda_bf16.h>
#include <mutex>
#include "kernels.cuh"
#include "mlp.cuh"
#include "tc_gemm.cuh"

namespace wrf {

namespace {
constexpr float kRcp = 0.2857143f;  // R_d / c_p of the microphysics scheme
}

// block: 32 consecutive columns of one row (lane = column) x 8 warps over the
// levels; the rows are staged in shared memory ([feature][33]) and written
// out coalesced, 4 columns per warp
template <bool kRaw>
__global__ void __launch_bounds__(256) k_mlp_features(Grid g, S s, MlpLayout L, const float* norm, __nv_bfloat16* x,
                                                      float* raw) {
  extern __shared__ float fs[];
  const int tx = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ii = blockIdx.x * 32 + tx, jj = blockIdx.y;
  const bool ok = ii < L.ncx;
  const int i = g.ids + 1 + ii, j = g.jds + 1 + jj;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const int c2 = ok ? g.i2(j, i) : 0;
  const int km = L.km;
  constexpr int nv = kRaw ? kRawVars : kFeatVars;
  const float* M = s[WF_MOIST];
  for (int k = w; k < km; k += 8) {
    float f[kRawVars];
    if (ok) {
      const size_t p = k * lev + c2;
      const float tp = s[WF_T][p];
      const float pfull = s[WF_P][p] + s[WF_PB][p];
      f[0] = (tp + (float)T0) * wpow(pfull / (float)P0, kRcp);
      f[1] = pfull;
      f[2] = 1.0f / (s[WF_AL][p] + s[WF_ALB][p]);
#pragma unroll
      for (int m = 1; m < 7; ++m) f[2 + m] = M[m * n3 + p];
      f[9] = tp;
    } else {
#pragma unroll
      for (int v = 0; v < kRawVars; ++v) f[v] = 0.f;
    }
#pragma unroll
    for (int v = 0; v < nv; ++v) {
      float val = f[v];
      if constexpr (!kRaw) {
        if (v >= 3) val = logf(fmaxf(val, 0.0f) + kLogFloor);
        const int idx = v * km + k;
        val = (val - norm[norm_in_mean(L) + idx]) * norm[norm_in_rstd(L) + idx];
      }
      fs[(v * km + k) * 33 + tx] = val;
    }
  }
  __syncthreads();
  const int width = kRaw ? kRawVars * km : L.d0;
  const int nfill = nv * km;
  for (int cc = w * 4; cc < w * 4 + 4; ++cc) {
    const int iic = blockIdx.x * 32 + cc;
    if (iic >= L.ncx) break;
    const size_t col = (size_t)jj * L.ncx + iic;
    for (int f = tx; f < width; f += 32) {
      const float v = f < nfill ? fs[f * 33 + cc] : 0.0f;
      if constexpr (kRaw)
        raw[col * width + f] = v;
      else
        x[col * L.d0 + f] = __float2bfloat16_rn(v);
    }
  }
}

// increments of theta and the six species over the call (the raw features
// before it hold the old values), and the step's precipitation
__global__ void __launch_bounds__(256) k_mlp_targets(Grid g, S s, MlpLayout L, const float* raw_in, float* raw_out) {
  const int tx = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ii = blockIdx.x * 32 + tx, jj = blockIdx.y;
  if (ii >= L.ncx) return;
  const int i = g.ids + 1 + ii, j = g.jds + 1 + jj;
  const size_t lev = (size_t)g.ny * g.nx, n3 = g.n3();
  const int c2 = g.i2(j, i);
  const int km = L.km;
  const size_t col = (size_t)jj * L.ncx + ii;
  const float* in = raw_in + col * (kRawVars * km);
  float* out = raw_out + col * L.nout;
  const float* M = s[WF_MOIST];
  for (int k = w; k < km; k += 8) {
    const size_t p = k * lev + c2;
    out[k] = s[WF_T][p] - in[9 * km + k];
#pragma unroll
    for (int m = 1; m < 7; ++m) out[m * km + k] = M[m * n3 + p] - in[(2 + m) * km + k];
  }
  if (w == 0) {
    out[kOutVars * km + 0] = s[WF_RAINNCV][c2];
    out[kOutVars * km + 1] = s[WF_SNOWNCV][c2];
    out[kOutVars * km + 2] = s[WF_GRAUPELNCV][c2];
  }
}

__global__ void k_mlp_normalize(MlpLayout L, const float* norm, const float* raw_in, const float* raw_out,
                                long long n, __nv_bfloat16* x, float* t) {
  const long long nx = n * L.d0, nt = n * L.d4;
  const int km = L.km;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nx + nt; e += (long long)gridDim.x * blockDim.x) {
    if (e < nx) {
      const long long r = e / L.d0;
      const int f = (int)(e - r * L.d0);
      float v = 0.0f;
      if (f < L.nfeat) {
        v = raw_in[r * (kRawVars * km) + f];
        if (f >= 3 * km) v = logf(fmaxf(v, 0.0f) + kLogFloor);
        v = (v - norm[norm_in_mean(L) + f]) * norm[norm_in_rstd(L) + f];
      }
      x[e] = __float2bfloat16_rn(v);
    } else {
      const long long q = e - nx;
      const long long r = q / L.d4;
      const int o = (int)(q - r * L.d4);
      float v = 0.0f;
      if (o < L.nout) {
        const float sd = norm[norm_out_std(L) + o];
        v = sd > 0.f ? (raw_out[r * L.nout + o] - norm[norm_out_mean(L) + o]) / sd : 0.0f;
      }
      t[q] = v;
    }
  }
}

// dy = scale (y - t) on the first nvalid columns (zero on the padding),
// written row-major and transposed; loss += sum (y - t)^2 over the valid part
__global__ void __launch_bounds__(256) k_mse_grad(const float* y, const float* t, int M, int N, int nvalid, float scale,
                                                 __nv_bfloat16* dy, __nv_bfloat16* dyt, float* loss) {
  __shared__ float tile[32][33];
  __shared__ float red[8];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int n0 = blockIdx.x * 32, m0 = blockIdx.y * 32;
  float acc = 0.f;
  for (int r = ty; r < 32; r += 8) {
    const int m = m0 + r, n = n0 + tx;
    float d = 0.f;
    if (m < M && n < N) {
      if (n < nvalid) d = y[(size_t)m * N + n] - t[(size_t)m * N + n];
      dy[(size_t)m * N + n] = __float2bfloat16_rn(scale * d);
    }
    acc += d * d;
    tile[r][tx] = scale * d;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int n = n0 + r, m = m0 + tx;
    if (n < N && m < M) dyt[(size_t)n * M + m] = __float2bfloat16_rn(tile[tx][r]);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (tx == 0) red[ty] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float sum = 0.f;
    for (int q = 0; q < 8; ++q) sum += red[q];
    atomicAdd(loss, sum);
  }
}

__global__ void __launch_bounds__(256) k_rowsum_bf16(const __nv_bfloat16* a, int cols, float* out) {
  __shared__ float red[8];
  const __nv_bfloat16* row = a + (size_t)blockIdx.x * cols;
  float acc = 0.f;
  for (int c = threadIdx.x; c < cols; c += blockDim.x) acc += __bfloat162float(row[c]);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float sum = 0.f;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) sum += red[q];
    out[blockIdx.x] = sum;
  }
}

// Adam (with decoupled weight decay) on fp32 master parameters; the gradient
// is the sum of nsplit partial sums split_stride apart
__global__ void k_adam(float* w, const float* gpart, int nsplit, long long split_stride, float* m, float* v, int R, int C,
                       __nv_bfloat16* wb, __nv_bfloat16* wtb, float lr, float b1, float b2, float eps, float wd,
                       float bc1, float bc2) {
  const long long n = (long long)R * C;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    float gsum = 0.f;
    for (int s = 0; s < nsplit; ++s) gsum += gpart[s * split_stride + e];
    const float mm = b1 * m[e] + (1.0f - b1) * gsum;
    const float vv = b2 * v[e] + (1.0f - b2) * gsum * gsum;
    m[e] = mm;
    v[e] = vv;
    float ww = w[e];
    ww = ww - lr * ((mm / bc1) / (sqrtf(vv / bc2) + eps) + wd * ww);
    w[e] = ww;
    const __nv_bfloat16 hb = __float2bfloat16_rn(ww);
    if (wb) wb[e] = hb;
    if (wtb) {
      const long long r = e / C, c = e - r * C;
      wtb[c * R + r] = hb;
    }
  }
}

__global__ void __launch_bounds__(256) k_transpose_bf16(const __nv_bfloat16* a, int R, int C, __nv_bfloat16* out) {
  __shared__ __nv_bfloat16 tile[32][34];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int r = ty; r < 32; r += 8)
    if (r0 + r < R && c0 + tx < C) tile[r][tx] = a[(size_t)(r0 + r) * C + c0 + tx];
  __syncthreads();
  for (int c = ty; c < 32; c += 8)
    if (c0 + c < C && r0 + tx < R) out[(size_t)(c0 + c) * R + r0 + tx] = tile[tx][c];
}

// ------------------------------------------------------------------ launchers
namespace {
constexpr size_t kFeatSmemMax = (size_t)kRawVars * (kMaxNz - 1) * 33 * sizeof(float);
}

// dynamic shared-memory limits of the network's kernels, set once per device
// (the first call should come before any stream capture)
int mlp_prepare_device() {
  constexpr int kMaxDev = 64;
  static bool done[kMaxDev] = {};
  static std::mutex mu;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return WRF_ECUDA;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return WRF_OK;
    if (cudaFuncSetAttribute(k_mlp_features<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFeatSmemMax) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_features<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFeatSmemMax) !=
            cudaSuccess)
      return WRF_ECUDA;
    done[dev] = true;
  }
  return gemm_prepare_device();
}

int launch_mlp_features(const Grid& g, const S& s, const MlpLayout& L, const float* norm, void* x, float* raw,
                        cudaStream_t st) {
  const dim3 grid((L.ncx + 31) / 32, L.ncy);
  if (mlp_prepare_device() != WRF_OK) return WRF_ECUDA;
  if (raw) {
    const size_t smem = (size_t)kRawVars * L.km * 33 * sizeof(float);
    k_mlp_features<true><<<grid, 256, smem, st>>>(g, s, L, nullptr, nullptr, raw);
  } else {
    const size_t smem = (size_t)kFeatVars * L.km * 33 * sizeof(float);
    k_mlp_features<false><<<grid, 256, smem, st>>>(g, s, L, norm, static_cast<__nv_bfloat16*>(x), nullptr);
  }
  return 1;
}

int launch_mlp_targets(const Grid& g, const S& s, const MlpLayout& L, const float* raw_in, float* raw_out,
                       cudaStream_t st) {
  const dim3 grid((L.ncx + 31) / 32, L.ncy);
  k_mlp_targets<<<grid, 256, 0, st>>>(g, s, L, raw_in, raw_out);
  return 1;
}

int launch_mlp_normalize(const MlpLayout& L, const float* norm, const float* raw_in, const float* raw_out, long long n,
                         void* x, float* t, cudaStream_t st) {
  k_mlp_normalize<<<148 * 8, 256, 0, st>>>(L, norm, raw_in, raw_out, n, static_cast<__nv_bfloat16*>(x), t);
  return 1;
}

int launch_mse_grad(const float* y, const float* t, int M, int N, int nvalid, float scale, void* dy, void* dyt,
                    float* loss, cudaStream_t st) {
  const dim3 grid((N + 31) / 32, (M + 31) / 32);
  k_mse_grad<<<grid, 256, 0, st>>>(y, t, M, N, nvalid, scale, static_cast<__nv_bfloat16*>(dy),
                                   static_cast<__nv_bfloat16*>(dyt), loss);
  return 1;
}

int launch_rowsum_bf16(const void* a, int rows, int cols, float* out, cudaStream_t st) {
  k_rowsum_bf16<<<rows, 256, 0, st>>>(static_cast<const __nv_bfloat16*>(a), cols, out);
  return 1;
}

int launch_adam(float* w, const float* gpart, int nsplit, long long split_stride, float* m, float* v, int R, int C,
                void* wb, void* wtb, float lr, float b1, float b2, float eps, float wd, float bc1, float bc2,
                cudaStream_t st) {
  const long long n = (long long)R * C;
  const int blocks = (int)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
  k_adam<<<blocks, 256, 0, st>>>(w, gpart, nsplit, split_stride, m, v, R, C, static_cast<__nv_bfloat16*>(wb),
                                 static_cast<__nv_bfloat16*>(wtb), lr, b1, b2, eps, wd, bc1, bc2);
  return 1;
}

int launch_transpose_bf16(const void* a, int R, int C, void* out, cudaStream_t st) {
  const dim3 grid((C + 31) / 32, (R + 31) / 32);
  k_transpose_bf16<<<grid, 256, 0, st>>>(static_cast<const __nv_bfloat16*>(a), R, C, static_cast<__nv_bfloat16*>(out));
  return 1;
}

}  // namespace wrf
