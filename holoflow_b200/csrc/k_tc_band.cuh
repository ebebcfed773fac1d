// Launch interface of the tensor-core fused band DFT + lens + row FFT pass (k_tc_band.cu).
#pragma once

#include "frames.cuh"

namespace hf {

struct BandRowsArgs {
  FrameRing     ring;        // window frames (packed 12-bit or uint16)
  int           T;           // frames per window (64)
  int           H, W;        // frame geometry (W in {256, 512, 1024})
  int           nz;          // band bins (<= 32)
  const float2 *wmat;        // [nwin][T][nz] filter+DFT matrices (float32)
  int64_t       wmat_stride; // complex elements between windows (0 = shared)
  const float2 *lens;        // non-null: multiply by the Fresnel lens of (lambda, z, dx), computed
                             // in the kernel from the lens table's float32 phase
  float         lambda, z, dx;
  float2       *out;         // row-transformed band planes [nwin][nz][H][W]
  int64_t       out_win, out_plane, out_row;
  int           nwin;
  float         shift;       // sample offset removed before the f16 conversion (2048)
  int          *status;      // device status word (bounded waits)
  int           max_ctas;    // persistent grid size cap (SMs left to concurrent work otherwise)
  int          *row_counter; // device int, zeroed by the launcher: CTAs take rows from it
  int           raw = 0;     // 1: store the band planes as they are (no row FFT; lens normally
                             // null), for steps that act on them before the lens
};

bool band_rows_tc_supported(int fmt, int T, int W, int nz, int64_t frame_bytes);
int  launch_band_rows_tc(const BandRowsArgs &a, int fmt, cudaStream_t s);

// Raw band planes (no lens, no row FFT) in row segments on the tensor cores (k_tc_band_seg.cu):
// T = 32, 64 or 128, W a multiple of 128, Nz <= 64.  Uses ring, T, H, W, nz, wmat, wmat_stride,
// out, out_win / out_plane / out_row, nwin, shift, status, max_ctas and row_counter of `a`.
bool band_seg_tc_supported(int fmt, int T, int W, int nz, int64_t frame_bytes);
int  launch_band_seg_tc(const BandRowsArgs &a, int fmt, cudaStream_t s);

// One persistent segment pass over up to kMaxSegJobs acquisitions of the same T and format: the
// units of all jobs form one work list taken from `counter` (zeroed by the launcher).  seg_cap > 0
// caps the tiles per segment; max_ctas > 0 caps the grid.  Each job uses the fields of `a` listed
// above except status, max_ctas and row_counter.
constexpr int kMaxSegJobs = 16;
int launch_band_seg_tc_multi(const BandRowsArgs *jobs, int njobs, int fmt, int seg_cap, int max_ctas, int *counter,
                             int *status, cudaStream_t s);

} // namespace hf
