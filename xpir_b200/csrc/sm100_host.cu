// Host side of the sm_100a helpers: TMA tensor-map encoding through the driver entry
// point (the library links only the CUDA runtime).
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "sm100.cuh"

namespace xpir {
namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  });
  return fn;
}

}  // namespace

bool encode_tensor_map_u64_4d(CUtensorMap *map, const void *base, const uint64_t dims[4], const uint64_t strides[3],
                              const uint32_t box[4]) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  // TMA rules: 16-byte aligned base, strides multiples of 16 bytes, inner box row a
  // multiple of 16 bytes, box dims <= 256.
  if (((uintptr_t)base & 15) != 0) return false;
  for (int i = 0; i < 3; i++)
    if (strides[i] % 16 != 0) return false;
  if ((box[0] * 8) % 16 != 0) return false;
  cuuint64_t gdim[4] = {dims[0], dims[1], dims[2], dims[3]};
  cuuint64_t gstride[3] = {strides[0], strides[1], strides[2]};
  cuuint32_t b[4] = {box[0], box[1], box[2], box[3]};
  cuuint32_t estride[4] = {1, 1, 1, 1};
  for (int i = 0; i < 4; i++)
    if (gdim[i] == 0 || b[i] == 0 || b[i] > 256) return false;
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, const_cast<void *>(base), gdim, gstride, b, estride,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

cudaError_t allow_max_dynamic_smem(const void *kernel) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  return e;
}

}  // namespace xpir
