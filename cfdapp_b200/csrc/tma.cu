// Host side of the TMA helpers: tensor-map encoding through the driver entry
// point (no link-time dependency on libcuda).
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "tma.cuh"

namespace cfdb {
namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    cudaGetLastError();
  });
  return fn;
}

}  // namespace

bool encode_tensor_map(CUtensorMap* map, CUtensorMapDataType dtype, int elem_bytes, int rank,
                       const void* base, const uint64_t* dims, const uint32_t* box) {
  EncodeTiledFn fn = encode_fn();
  if (!fn || rank < 1 || rank > 3) return false;
  cuuint64_t gdim[3], gstride[2];
  cuuint32_t bdim[3], estride[3] = {1, 1, 1};
  uint64_t pitch = (uint64_t)elem_bytes;
  for (int d = 0; d < rank; ++d) {
    gdim[d] = dims[d];
    bdim[d] = box[d];
    if (d > 0) gstride[d - 1] = pitch;
    pitch *= dims[d];
  }
  const CUresult r = fn(map, dtype, (cuuint32_t)rank, const_cast<void*>(base), gdim, gstride, bdim,
                        estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace cfdb
