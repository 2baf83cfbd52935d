// Host side of the TMA-fed stages: tensor-map encoding through the driver's
// cuTensorMapEncodeTiled, reached with cudaGetDriverEntryPoint so that the
// library links against the runtime only.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <mutex>

#include "plan.hpp"

namespace dfft {

namespace {
std::once_flag g_encode_once;
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

void load_encode() {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  else
    cudaGetLastError();
}
}  // namespace

bool tma_encode(void* map, const void* base, const TmaSource& t) {
  static_assert(sizeof(CUtensorMap) == 128, "tensor map size");
  if (!t.ok || !base || (reinterpret_cast<std::uintptr_t>(map) & 63) || (reinterpret_cast<std::uintptr_t>(base) & 15))
    return false;
  std::call_once(g_encode_once, load_encode);
  if (!g_encode) return false;
  cuuint64_t dims[5], strides[4];
  cuuint32_t box[5], es[5] = {1, 1, 1, 1, 1};
  for (int d = 0; d < 5; ++d) {
    dims[d] = t.dim[d];
    box[d] = t.box[d];
    if (d > 0) strides[d - 1] = t.stride[d];
  }
  const CUresult r = g_encode(static_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_UINT64, 5,
                              const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace dfft
