// cg_tma_host.cu -- host side of the TMA tile copies: tensor maps of the
// substep input registers, encoded through the driver entry point that the
// CUDA runtime hands out (no link against libcuda).
#include <cudaTypedefs.h>

#include <cstring>

#include "cg_internal.h"

namespace cg {
namespace tma_host {
namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

}  // namespace

bool encode(CUtensorMap* map, void* base, int elem, int nx, int ny, int nz, int nfields, int bz, int by, int bx) {
  std::memset(map, 0, sizeof(*map));
  auto enc = encode_fn();
  if (!enc || !base || (elem != 4 && elem != 8)) return false;
  // the global address and every byte stride must be multiples of 16, and so
  // must the box's innermost extent
  if (reinterpret_cast<uintptr_t>(base) % 16 != 0 || ((size_t)nz * elem) % 16 != 0 || ((size_t)bz * elem) % 16 != 0)
    return false;
  if (bz > 256 || by > 256 || bx > 256) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx, (cuuint64_t)nfields};
  const cuuint64_t strides[3] = {(cuuint64_t)nz * elem, (cuuint64_t)ny * nz * elem, (cuuint64_t)nx * ny * nz * elem};
  const cuuint32_t box[4] = {(cuuint32_t)bz, (cuuint32_t)by, (cuuint32_t)bx, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUtensorMapDataType type = elem == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  return enc(map, type, 4, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace tma_host
}  // namespace cg
