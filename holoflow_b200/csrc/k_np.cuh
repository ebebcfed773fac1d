// Launch interface of the element kernels behind the thin holonp node kinds (k_np.cu).
#pragma once

#include <type_traits>

#include "hf_common.cuh"

namespace hf {

constexpr int kNpMaxRank = 8;

// Shape and byte strides of a strided copy (rank <= 8).
struct NpLayout {
  int     rank = 0;
  int64_t shape[kNpMaxRank]       = {};
  int64_t src_strides[kNpMaxRank] = {};
  int64_t dst_strides[kNpMaxRank] = {};
};

// Output shape and per-operand element strides (0 along broadcast dimensions).
struct NpBroadcast {
  int     rank = 0;
  int64_t shape[kNpMaxRank]     = {};
  int64_t a_strides[kNpMaxRank] = {};
  int64_t b_strides[kNpMaxRank] = {};
};

int launch_copy_strided(const void *src, void *dst, const NpLayout &l, int elem_size, cudaStream_t s);
// F32 / CF32 operands (x_cplx: 1 = complex64), output CF32 when either is complex.
int launch_multiply(const void *a, int a_cplx, const void *b, int b_cplx, void *out, const NpBroadcast &l,
                    cudaStream_t s);
// |x| of a contiguous tensor: CF32 -> F32 (sqrt(re^2 + im^2)), F32 -> F32, U8 / U16 -> F32.
int launch_abs(const void *in, int in_dtype, float *out, int64_t n, cudaStream_t s);
// out[i] = (float)(start + step * i), in double before the cast (arange.cu:62-75).
int launch_arange(float *out, double start, double step, int64_t n, cudaStream_t s);
// One step of the causal sliding average (causal_sliding_average.cu:35-50): sum += x - hist,
// hist = x, out = sum / divisor, in float32; `hist_slot` is the history slot of this step.
int launch_causal_avg(const float *in, float *out, float *hist_slot, float *sum, int64_t n, float divisor,
                      cudaStream_t s);

} // namespace hf
