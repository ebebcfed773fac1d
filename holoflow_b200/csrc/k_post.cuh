// Launch interface of the post-propagation helpers in k_post.cu that the pipeline shares.
#pragma once

#include "hf_common.cuh"

namespace hf {

// out = IFFT2(FFT2(in) x tab) per [H][W] plane, unnormalized (Filter2D); c0 (and c1 for real
// input) are planes * H * W complex scratch buffers distinct from in and out.
int launch_filter2d(const float2 *tab, int64_t planes, int H, int W, int real_in, const void *in, void *out,
                    float2 *c0, float2 *c1, cudaStream_t s);
// The Filter2D annulus mask [H][W] in natural frequency order (filter2d.cu:109-199).
int launch_filter2d_table(float2 *tab, int H, int W, int real_in, uint32_t r_inner, uint32_t r_outer,
                          uint32_t s_inner, uint32_t s_outer, cudaStream_t s);

} // namespace hf
