// Host-side construction of TMA tensor maps (cuTensorMapEncodeTiled through the runtime's driver
// entry-point query, so the library does not link libcuda directly).
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include "hf_common.cuh"

namespace hf {

// 2D tensor map over a row-major float32 matrix [rows][cols] with row pitch `pitch_bytes`, read in
// boxes of [box_rows][box_cols].  The base must be 16-byte aligned, the pitch a multiple of 16 and
// box_cols * 4 a multiple of 16.
inline int make_tmap_2d_f32(CUtensorMap *map, const void *base, uint64_t cols, uint64_t rows, uint64_t pitch_bytes,
                            uint32_t box_cols, uint32_t box_rows) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void                           *fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    const cudaError_t e = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      return fail(HF_ERR_CUDA, "tensor map: cuTensorMapEncodeTiled is unavailable");
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  HF_CHECK_ARG((reinterpret_cast<uintptr_t>(base) & 15) == 0 && pitch_bytes % 16 == 0 && (box_cols * 4) % 16 == 0 &&
                   box_cols <= 256 && box_rows <= 256,
               "tensor map: misaligned base, pitch or box");
  const cuuint64_t dims[2]    = {cols, rows};
  const cuuint64_t strides[1] = {pitch_bytes};
  const cuuint32_t box[2]     = {box_cols, box_rows};
  const cuuint32_t estr[2]    = {1, 1};
  const CUresult   r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return fail(HF_ERR_CUDA, "tensor map: cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
  return HF_OK;
}

} // namespace hf
