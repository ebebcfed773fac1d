// Launch interface of the TMA-fed column FFT + moments pass (k_cols_tma.cu).
#pragma once

#include <cuda.h>

#include "k_fft2d.cuh"

namespace hf {

struct ColMomArgs {
  int     H, W;          // plane size; the column transform has length H
  int     nz;            // band planes per window
  int64_t rows_per_win;  // tensor-map rows between consecutive windows (nz * H for packed planes)
  float  *out;           // moment images [nwin][n_moments][out rows][out cols]
  int64_t out_win, out_plane, out_row;
  int    *status;        // receives 21 if a stage wait expires
  int     fast;          // chosen form: hardware square-root approximation, fused moment sums
};

// Columns per CTA strip of the pass.
constexpr int kColMomCols = 4;

// `tmap`: 2D float32 tensor map over the band planes viewed as [rows][2 * W] (complex as two
// floats), box [H or 256 rows][2 * kColMomCols floats], so window w, plane k, row r is tensor row
// w * rows_per_win + k * H + r.
bool col_moments_tma_supported(int H, int W);
int  launch_col_moments_tma(const CUtensorMap &tmap, const ColMomArgs &a, const MomentSpec &m, int nwin,
                            cudaStream_t s);

} // namespace hf
