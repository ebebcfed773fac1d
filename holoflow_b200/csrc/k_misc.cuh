// Launch interface of the element-wise / reduction kernels (k_misc.cu).
#pragma once

#include <algorithm>
#include <type_traits>

#include "hf_common.cuh"

namespace hf {

constexpr int kMaxMomentBands = 64;

struct MomentWeights {
  float w1[kMaxMomentBands]; // f_k
  float w2[kMaxMomentBands]; // f_k^2 formed in float32
};

struct AsFilter {
  uint32_t r_inner, r_outer, s_inner, s_outer;
};

int launch_unpack12(const uint8_t *in, void *out, int out_dtype, int64_t npix, cudaStream_t s);
int launch_pack12(const uint16_t *in, uint8_t *out, int64_t npix, cudaStream_t s);
int launch_convert(const void *in, int in_dtype, void *out, int out_dtype, int strategy, int64_t n,
                   void *minmax_ws, cudaStream_t s);
int launch_mean_axis(const void *in, int in_dtype, int64_t outer, int64_t n, int64_t inner,
                     void *out, bool abs_values, cudaStream_t s);
int launch_band_moments(const void *planes, int in_dtype, int nz, int64_t P, const MomentWeights &w,
                        int mask, float *out, cudaStream_t s);
int launch_fresnel_lens(float2 *lens, int W, int H, float lambda, float z, float dx, cudaStream_t s);
int launch_as_tf(float2 *tf, int W, int H, float lambda, float z, float dx, int use_filter,
                 const AsFilter &f, cudaStream_t s);

} // namespace hf
