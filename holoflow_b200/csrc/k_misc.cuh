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

// One value of the Fresnel quadratic-phase lens (fresnel_diffraction.cu:326-341): centred
// coordinates x = ((col + (S - W)/2) - S/2) dx and y likewise, S = max(W, H), phase
// pi / (lambda z) (x^2 + y^2), each step rounded in float32 as the reference evaluates it.
// The lens table evaluates it with sincosf; the fused band pass evaluates the same float32 phase
// with cis_reduced below.
__device__ __forceinline__ float fresnel_lens_k(float lambda, float z) {
  return __fdiv_rn(3.14159265358979323846f, __fmul_rn(lambda, z));
}
__device__ __forceinline__ float fresnel_lens_phase(int col, int row, int W, int H, float k, float dx) {
  const int   size = W > H ? W : H;
  const float half = (float)size / 2.0f;
  const float x    = __fmul_rn(__fsub_rn((float)(col + (size - W) / 2), half), dx);
  const float y    = __fmul_rn(__fsub_rn((float)(row + (size - H) / 2), half), dx);
  return __fmul_rn(k, __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)));
}
__device__ __forceinline__ float2 fresnel_lens_value(int col, int row, int W, int H, float k, float dx) {
  float s, c;
  sincosf(fresnel_lens_phase(col, row, W, H, k, dx), &s, &c);
  return make_float2(c, s);
}

// exp(i phase) for |phase| < 256 * 2 pi: Cody-Waite reduction to [-pi, pi] with 2 pi split into
// 6.28125 (8 significant bits, so n * 6.28125 is exact for n < 256 and the first subtraction is
// exact) plus the float32 remainder 2 pi - 6.28125, then the hardware sine / cosine, whose
// absolute error on [-pi, pi] is below 5e-7.  Used where the phase is evaluated per element inside
// a hot kernel (the chosen form's band pass), instead of the lens table's sincosf.
__device__ __forceinline__ float2 cis_reduced(float phase) {
  const float n = rintf(phase * 0.159154943091895336f); // 1 / (2 pi)
  float       r = fmaf(-n, 6.28125f, phase);
  r             = fmaf(-n, 1.93530717958647692e-3f, r);
  float s, c;
  __sincosf(r, &s, &c);
  return make_float2(c, s);
}
int launch_as_tf(float2 *tf, int W, int H, float lambda, float z, float dx, int use_filter,
                 const AsFilter &f, cudaStream_t s);

} // namespace hf
