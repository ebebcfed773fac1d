// Internal entry points of the Shack-Hartmann autofocus (k_shack.cu) for the fused pipeline.
#pragma once

#include <cuda_runtime.h>

#include "holoflow_b200.h"

namespace hf {

// Zeroes the coefficients and phase accumulated over the passes of one spectrum.
int autofocus_begin(hf_autofocus *a, cudaStream_t s);
// One measurement: sub-aperture M0, slopes, Zernike fit and phase map (kept as the pass's phase
// and added to the accumulated ones); `planes` is [nz][H][W] complex64.
int autofocus_measure(hf_autofocus *a, const void *planes, cudaStream_t s);
// out = planes exp(-i phase) with the last measured phase (in place allowed).
int autofocus_correct(hf_autofocus *a, const void *planes, void *out, cudaStream_t s);
// out = lens exp(-i phase): the last measured correction folded into a [H][W] lens.
int autofocus_fold_lens(hf_autofocus *a, const float2 *lens, float2 *out, cudaStream_t s);
// A new propagation distance: rebuilds the short-time Fresnel input lens.
int autofocus_set_z(hf_autofocus *a, float z, cudaStream_t s);
int autofocus_passes(const hf_autofocus *a);
int autofocus_orders(const hf_autofocus *a);
const float *autofocus_cumulative_coeffs(const hf_autofocus *a);

} // namespace hf
