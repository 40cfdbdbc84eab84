// Host side of the TMA helpers: the driver's tensor-map encoder and the fp32
// field maps of the tiled advection, encoded once per (array, box) and
// cached (the step's launchers run every step, often inside graph capture).
#include <mutex>
#include <vector>
#include "tma.cuh"

namespace wrf {
namespace tma {

EncodeTiled encoder(const char** err) {
  static EncodeTiled fn = nullptr;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p) {
      *err = "cuTensorMapEncodeTiled is not available from the driver";
      return nullptr;
    }
    fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

namespace {
struct MapKey {
  const float* base;
  int nx, ny, nz, nw, bw, bh;
  bool operator==(const MapKey& o) const {
    return base == o.base && nx == o.nx && ny == o.ny && nz == o.nz && nw == o.nw && bw == o.bw && bh == o.bh;
  }
};
struct MapEntry {
  MapKey key;
  CUtensorMap map;
};
constexpr size_t kMaxCached = 512;
}  // namespace

bool encode_f32_4d(CUtensorMap* map, const float* base, int nx, int ny, int nz, int nw, int bw, int bh,
                   const char** err) {
  static std::mutex mu;
  static std::vector<MapEntry> cache;
  if (!base || nx < 1 || ny < 1 || nz < 1 || nw < 1 || nx % 4 != 0 || bw % 4 != 0 || bw < 4 || bw > 256 || bh < 1 ||
      bh > 256 || (reinterpret_cast<uintptr_t>(base) & 15u) != 0) {
    *err = "tensor map: needs a 16-byte aligned base, nx and the box width multiples of 4, boxes of at most 256";
    return false;
  }
  const MapKey key{base, nx, ny, nz, nw, bw, bh};
  std::lock_guard<std::mutex> lock(mu);
  for (const MapEntry& e : cache)
    if (e.key == key) {
      *map = e.map;
      return true;
    }
  EncodeTiled enc = encoder(err);
  if (!enc) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)nw};
  const cuuint64_t row = (cuuint64_t)nx * 4;
  const cuuint64_t strides[3] = {row, row * (cuuint64_t)ny, row * (cuuint64_t)ny * (cuuint64_t)nz};
  const cuuint32_t box[4] = {(cuuint32_t)bw, (cuuint32_t)bh, 1, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(base), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    *err = "cuTensorMapEncodeTiled rejected a field map";
    return false;
  }
  if (cache.size() >= kMaxCached) cache.erase(cache.begin());
  cache.push_back(MapEntry{key, *map});
  return true;
}

}  // namespace tma
}  // namespace wrf
