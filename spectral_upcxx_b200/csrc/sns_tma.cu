// Host side of the TMA field tiles (sns_tma.cuh): tensor maps encoded
// through the driver's cuTensorMapEncodeTiled, reached with
// cudaGetDriverEntryPointByVersion so that the library needs no link against
// libcuda.
#include <cudaTypedefs.h>
#include <stdio.h>

#include "sns_common.cuh"
#include "sns_tma.cuh"

namespace sns {
namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

}  // namespace

bool field_box_ok(int nx, int ny, int nz, int esz, int bw, int bg, int bz) {
  if (esz % 8 || bw <= 0 || bg <= 0 || bz <= 0) return false;
  const int64_t units = (int64_t)bw * esz / 8;
  return units <= 256 && bg <= 256 && bz <= 256 && ((int64_t)bw * esz) % 16 == 0 &&
         ((int64_t)nx * esz) % 16 == 0 && nx % bw == 0 && ny % bg == 0 && nz % bz == 0;
}

int field_tensor_map(CUtensorMap* map, const void* base, int nx, int ny, int nz, int esz, int bw,
                     int bg, int bz) {
  if (!field_box_ok(nx, ny, nz, esz, bw, bg, bz) || (reinterpret_cast<uintptr_t>(base) & 15)) {
    set_error("TMA tile: box or field layout not loadable (alignment or size)");
    return ERR_UNSUPPORTED;
  }
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
  if (!fn) {
    set_error("TMA tile: the driver has no cuTensorMapEncodeTiled");
    return ERR_UNSUPPORTED;
  }
  const int u = esz / 8;
  const cuuint64_t dims[3] = {(cuuint64_t)nx * u, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * esz, (cuuint64_t)nx * ny * esz};
  const cuuint32_t box[3] = {(cuuint32_t)(bw * u), (cuuint32_t)bg, (cuuint32_t)bz};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char msg[96];
    snprintf(msg, sizeof(msg), "TMA tile: cuTensorMapEncodeTiled failed (%d)", (int)r);
    set_error(msg);
    return ERR_UNSUPPORTED;
  }
  return OK;
}

}  // namespace sns
