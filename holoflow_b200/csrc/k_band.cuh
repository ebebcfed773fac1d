// Launch interface of the temporal band DFT kernels (k_band.cu).
#pragma once

#include "frames.cuh"

namespace hf {

struct BandArgs {
  FrameRing     ring;        // window frames
  int           T;           // frames per window
  int64_t       P;           // pixels per frame (H * W)
  int           H, W;        // frame geometry
  int           nz;          // output bins
  const float2 *wmat;        // [nwin][T][nz] filter+DFT matrices; nullptr = plain DFT bins
  int           z0;          // first bin when wmat == nullptr
  int64_t       wmat_stride; // complex elements between windows (0 = shared matrix)
  const float2 *lens;        // [P] per-pixel multiplier or nullptr
  float2       *out;         // [nwin][nz][OH][OW]
  int           OH, OW;      // output plane geometry (>= H, W when zero-padded)
  int           oy, ox;      // placement of the frame inside the output plane
  int64_t       out_plane;   // OH * OW
  int64_t       out_win;     // nz * OH * OW
  float         scale;       // normalisation
};

int launch_band_dft(const BandArgs &a, int fmt, int nwin, cudaStream_t s);

} // namespace hf
