// Launch interface of the spatial 2-D FFT kernels (k_fft2d.cu).
//
// A 2-D transform of a [H][W] complex plane is a row pass (length-W transforms) followed by a
// column pass (length-H transforms).  Each pass reads and writes HBM once; the work that
// surrounds the transform in the reference path is fused into the passes:
//  * row pass load:   zero padding + placement (AngularSpectrum's load callback,
//                     angular_spectrum.cu:189-229), real->complex promotion, a per-element
//                     pre-multiply (the Fresnel lens, fresnel_diffraction.cu:262-303);
//  * column pass:     |.| store (fresnel_diffraction.cu:305-311), post-multiply (output phase,
//                     .cu:359-380), transfer-function multiply followed by the inverse column
//                     transform (angular_spectrum.cu:231-255), or |.| + M0/M1/M2 accumulation
//                     over the band planes with the fftshift applied on the final store
//                     (mean.cu:268-305, multiply.cu:69-94, graph_builder.cc:612-635);
//  * row-moments pass: inverse row transform + |.| + moment accumulation (angular spectrum's
//                     last pass).
#pragma once

#include "hf_common.cuh"

namespace hf {

constexpr int kMaxBands = 64; // moment weights carried by value in the kernel parameters

struct MomentSpec {
  int   nz;           // planes accumulated per window
  int   mask;         // HF_M0 | HF_M1 | HF_M2
  int   fftshift;     // shift the images by (H/2, W/2) on store
  float inv_nz;       // 1 / nz (float32, as the reference's mean divides by (float)n)
  float w1[kMaxBands]; // f_k
  float w2[kMaxBands]; // f_k^2 formed in float32
};

struct RowPass {
  const void   *in;            // complex64 or float32 rows
  int           in_real;       // 1: float32 input
  int64_t       in_win, in_plane, in_row, in_col; // element strides of the input view
  int           IH, IW;        // input plane size
  int           oy, ox;        // placement inside the (H x N) output plane (zero outside)
  float2       *out;           // complex64 output, unit column stride
  int64_t       out_win, out_plane, out_row;
  int           H, N;          // output plane rows / row length (transform length)
  int           nplanes;       // planes per window
  const float2 *pre;           // optional [H][N] pre-multiply (applied to in-plane samples)
  int           inverse;
};

struct ColPass {
  const float2 *in;            // complex64 planes, unit column stride
  int64_t       in_win, in_plane, in_row;
  int           H, W;          // plane size (H = transform length)
  int           nplanes;       // planes per window
  void         *out;           // complex64 / float32 planes, or moment images
  int64_t       out_win, out_plane, out_row;
  int64_t       out_col;       // column stride of complex / magnitude stores (1 = contiguous)
  const float2 *post;          // optional [H][W] post-multiply (complex store only)
  const float2 *tf;            // [H][W] transfer function (TF mode)
  int           inverse;
};

enum ColMode { COL_COMPLEX = 0, COL_MAGNITUDE = 1, COL_MOMENTS = 2, COL_TF_SANDWICH = 3 };

// Whether the fused four-step kernels cover transform length n (n = 32 * N1).
bool fft_fast_length(int n);

int launch_row_pass(const RowPass &a, int nwin, cudaStream_t s);
int launch_col_pass(const ColPass &a, int mode, const MomentSpec *mom, int nwin, cudaStream_t s);
// Inverse/forward row transform + |.| + moments; input/out geometry as ColPass (W = row length).
int launch_row_moments(const ColPass &a, const MomentSpec &mom, int nwin, cudaStream_t s);

} // namespace hf
