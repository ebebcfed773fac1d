// Spatial 2-D FFT passes with fused epilogues (see k_fft2d.cuh for the mapping onto the
// reference's cuFFT plans and callbacks).
#include <algorithm>

#include "fft_core.cuh"
#include "k_fft2d.cuh"

namespace hf {

bool fft_fast_length(int n) {
  switch (n) {
  case 64: case 128: case 256: case 512: case 768: case 1024: case 1536:
    return true;
  default:
    return false;
  }
}

namespace {

// ------------------------------------------------------------------------------------------------
// Row pass: one warp per row, grid-stride over the rows of every plane of a window.
// ------------------------------------------------------------------------------------------------
// Loads row `row` of a window's planes (zero outside the placed input) into lane registers:
// x[n1] = sample (n2 = lane) + 32 * n1, optionally pre-multiplied.
template <int N1>
__device__ __forceinline__ void row_load(const RowPass &a, int w, int64_t row, int lane, float2 *x) {
  const int plane = (int)(row / a.H), r = (int)(row % a.H);
  const int ir    = r - a.oy;
  const bool in_rows = ir >= 0 && ir < a.IH;
  const int64_t ibase = w * a.in_win + plane * a.in_plane + (int64_t)ir * a.in_row;
  if (a.ox == 0 && a.oy == 0 && a.IW == N1 * 32 && a.IH == a.H) {
    // no padding: every sample exists, so all loads (and then all lens loads) issue back to back
    // instead of one bounds-checked load at a time
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const int64_t off = ibase + (int64_t)(lane + 32 * n1) * a.in_col;
      x[n1] = a.in_real ? make_float2(__ldg(reinterpret_cast<const float *>(a.in) + off), 0.f)
                        : __ldg(reinterpret_cast<const float2 *>(a.in) + off);
    }
    if (a.pre != nullptr) {
      const float2 *pr = a.pre + (int64_t)r * (N1 * 32) + lane;
      float2        pv[N1];
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1)
        pv[n1] = __ldg(pr + 32 * n1);
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1)
        x[n1] = cmul(x[n1], pv[n1]);
    }
    return;
  }
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) {
    const int col = lane + 32 * n1;
    const int ic  = col - a.ox;
    float2    v   = make_float2(0.f, 0.f);
    if (in_rows && ic >= 0 && ic < a.IW) {
      const int64_t off = ibase + (int64_t)ic * a.in_col;
      v = a.in_real ? make_float2(__ldg(reinterpret_cast<const float *>(a.in) + off), 0.f)
                    : __ldg(reinterpret_cast<const float2 *>(a.in) + off);
      if (a.pre != nullptr)
        v = cmul(v, __ldg(a.pre + (int64_t)r * (N1 * 32) + col));
    }
    x[n1] = v;
  }
}

// Row pass: one warp per row, grid-stride over the rows of every plane of a window.  Each lane
// loads its 32-stride samples of the row, so a warp load instruction reads 256 contiguous bytes.
template <int N1, bool INV> __global__ void __launch_bounds__(256) row_pass_kernel(RowPass a) {
  constexpr int N = N1 * 32;
  extern __shared__ __align__(16) float smf[];
  TwTable tw{reinterpret_cast<float2 *>(smf), N};
  float2 *xball = reinterpret_cast<float2 *>(smf + 2 * N);
  tw.fill(threadIdx.x, blockDim.x);
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  float2   *xb   = xball + warp * XBuf<N1>::kSize;
  const int w    = blockIdx.y;
  const int64_t nrows  = (int64_t)a.nplanes * a.H;
  const int64_t stride = (int64_t)gridDim.x * nwarps;
  for (int64_t row = (int64_t)blockIdx.x * nwarps + warp; row < nrows; row += stride) {
    float2 x[N1];
    row_load<N1>(a, w, row, lane, x);
    const int plane = (int)(row / a.H), r = (int)(row % a.H);
    float2   *orow  = a.out + w * a.out_win + plane * a.out_plane + r * a.out_row;
    four_step_a<N1, INV>(x, lane, tw, xb);
    __syncwarp();
    for (int k1 = lane; k1 < N1; k1 += 32) {
      float2 y[32];
      four_step_b<N1, INV>(y, k1, xb);
#pragma unroll
      for (int k2 = 0; k2 < 32; ++k2)
        orow[k1 + N1 * k2] = y[k2];
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------------------------------------
// Column pass over strips of C columns; thread (n2, c) = (tid / C, tid % C).
// ------------------------------------------------------------------------------------------------
template <int N1, int C, bool INV, int MODE>
__global__ void __launch_bounds__(32 * C) col_pass_kernel(ColPass a, MomentSpec m) {
  constexpr int N  = N1 * 32;
  constexpr int CS = XBuf<N1>::kSize;
  extern __shared__ __align__(16) float smf[];
  SmemTwiddles tw{smf, smf + N, N};
  float2      *xball = reinterpret_cast<float2 *>(smf + 2 * N);
  float       *acc   = reinterpret_cast<float *>(xball + C * CS); // [3][N][C] (moments)
  tw.fill(threadIdx.x, blockDim.x);

  const int  tid   = threadIdx.x;
  const int  n2    = tid / C, c = tid % C; // load role
  const int  k1    = tid / C;              // store role (same mapping)
  const int  col   = blockIdx.x * C + c;
  const bool valid = col < a.W;
  const int  w     = blockIdx.z;
  float2    *xb    = xball + c * CS;

  if constexpr (MODE == COL_MOMENTS) {
    for (int i = tid; i < 3 * N * C; i += blockDim.x)
      acc[i] = 0.f;
  }
  __syncthreads();

  // work items: (plane) for the moments mode (the CTA owns its strip across planes), otherwise
  // (plane) for a fixed strip with the grid's y dimension striding over planes
  const int p_begin  = MODE == COL_MOMENTS ? 0 : blockIdx.y;
  const int p_end    = a.nplanes;
  const int p_stride = MODE == COL_MOMENTS ? 1 : gridDim.y;
  float2    nxt[N1];
  {
    const float2 *src = a.in + w * a.in_win + (int64_t)p_begin * a.in_plane + col;
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1)
      nxt[n1] = (valid && p_begin < p_end) ? __ldg(src + (int64_t)(n2 + 32 * n1) * a.in_row)
                                           : make_float2(0.f, 0.f);
  }
  for (int plane = p_begin; plane < p_end; plane += p_stride) {
    float2 x[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1)
      x[n1] = nxt[n1];
    if (plane + p_stride < p_end) {
      const float2 *src = a.in + w * a.in_win + (int64_t)(plane + p_stride) * a.in_plane + col;
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1)
        nxt[n1] = valid ? __ldg(src + (int64_t)(n2 + 32 * n1) * a.in_row) : make_float2(0.f, 0.f);
    }
    four_step_a<N1, INV>(x, n2, tw, xb);
    __syncthreads();

    float2 y[32];
    for (int kk = k1; kk < N1; kk += 32) {
      four_step_b<N1, INV>(y, kk, xb);
      if constexpr (MODE == COL_COMPLEX) {
        if (valid) {
          float2 *dst = reinterpret_cast<float2 *>(a.out) + w * a.out_win + plane * a.out_plane + col * a.out_col;
#pragma unroll
          for (int k2 = 0; k2 < 32; ++k2) {
            const int row = kk + N1 * k2;
            float2    v   = y[k2];
            if (a.post != nullptr)
              v = cmul(v, __ldg(a.post + (int64_t)row * a.W + col));
            dst[(int64_t)row * a.out_row] = v;
          }
        }
      } else if constexpr (MODE == COL_MAGNITUDE) {
        if (valid) {
          float *dst = reinterpret_cast<float *>(a.out) + w * a.out_win + plane * a.out_plane + col * a.out_col;
#pragma unroll
          for (int k2 = 0; k2 < 32; ++k2)
            dst[(int64_t)(kk + N1 * k2) * a.out_row] = hypotf(y[k2].x, y[k2].y);
        }
      } else if constexpr (MODE == COL_MOMENTS) {
        const float f1 = m.w1[plane], f2 = m.w2[plane];
#pragma unroll
        for (int k2 = 0; k2 < 32; ++k2) {
          const int   idx = (kk + N1 * k2) * C + c;
          const float mag = hypotf(y[k2].x, y[k2].y);
          acc[idx]             = __fadd_rn(acc[idx], mag);
          acc[N * C + idx]     = __fadd_rn(acc[N * C + idx], __fmul_rn(f1, mag));
          acc[2 * N * C + idx] = __fadd_rn(acc[2 * N * C + idx], __fmul_rn(f2, mag));
        }
      } else { // COL_TF_SANDWICH (N1 <= 32: one kk per thread)
#pragma unroll
        for (int k2 = 0; k2 < 32; ++k2) {
          const int row = kk + N1 * k2;
          y[k2]         = valid ? cmul(y[k2], __ldg(a.tf + (int64_t)row * a.W + col)) : y[k2];
        }
      }
    }
    if constexpr (MODE == COL_TF_SANDWICH) {
      __syncthreads();
      if (k1 < N1)
        four_step_rev_a<N1, !INV>(y, k1, tw, xb);
      __syncthreads();
      four_step_rev_b<N1, !INV>(x, n2, xb);
      if (valid) {
        float2 *dst = reinterpret_cast<float2 *>(a.out) + w * a.out_win + plane * a.out_plane + col * a.out_col;
#pragma unroll
        for (int ka = 0; ka < N1; ++ka)
          dst[(int64_t)(n2 + 32 * ka) * a.out_row] = x[ka];
      }
    }
    __syncthreads();
  }

  if constexpr (MODE == COL_MOMENTS) {
    if (!valid)
      return;
    const float nzf = (float)m.nz;
    float      *out = reinterpret_cast<float *>(a.out) + w * a.out_win;
    const int   cc  = m.fftshift ? (col + a.W / 2) % a.W : col;
    int         mi  = 0;
    for (int mo = 0; mo < 3; ++mo) {
      if (!(m.mask & (1 << mo)))
        continue;
      for (int row = k1; row < N; row += 32) {
        const int rr = m.fftshift ? (row + N / 2) % N : row;
        out[mi * a.out_plane + (int64_t)rr * a.out_row + cc] = __fdiv_rn(acc[mo * N * C + row * C + c], nzf);
      }
      ++mi;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Row transform + |.| + moments: a warp owns one image row across all planes of a window.
// ------------------------------------------------------------------------------------------------
template <int N1, bool INV>
__global__ void __launch_bounds__(128) row_moments_kernel(ColPass a, MomentSpec m) {
  constexpr int N = N1 * 32;
  extern __shared__ __align__(16) float smf[];
  SmemTwiddles tw{smf, smf + N, N};
  const int    warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  float2      *xb   = reinterpret_cast<float2 *>(smf + 2 * N) + warp * XBuf<N1>::kSize;
  float       *acc  = smf + 2 * N + 2 * nwarps * XBuf<N1>::kSize + warp * 3 * N;
  tw.fill(threadIdx.x, blockDim.x);
  __syncthreads();

  const int r = blockIdx.x * nwarps + warp;
  const int w = blockIdx.y;
  if (r >= a.H)
    return;
  for (int i = lane; i < 3 * N; i += 32)
    acc[i] = 0.f;
  __syncwarp();
  for (int k = 0; k < m.nz; ++k) {
    const float2 *src = a.in + w * a.in_win + k * a.in_plane + (int64_t)r * a.in_row;
    float2        x[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1)
      x[n1] = __ldg(src + lane + 32 * n1);
    four_step_a<N1, INV>(x, lane, tw, xb);
    __syncwarp();
    const float f1 = m.w1[k], f2 = m.w2[k];
    for (int k1 = lane; k1 < N1; k1 += 32) {
      float2 y[32];
      four_step_b<N1, INV>(y, k1, xb);
#pragma unroll
      for (int k2 = 0; k2 < 32; ++k2) {
        const int   i   = k1 + N1 * k2;
        const float mag = hypotf(y[k2].x, y[k2].y);
        acc[i]         = __fadd_rn(acc[i], mag);
        acc[N + i]     = __fadd_rn(acc[N + i], __fmul_rn(f1, mag));
        acc[2 * N + i] = __fadd_rn(acc[2 * N + i], __fmul_rn(f2, mag));
      }
    }
    __syncwarp();
  }
  const float nzf = (float)m.nz;
  float      *out = reinterpret_cast<float *>(a.out) + w * a.out_win;
  const int   rr  = m.fftshift ? (r + a.H / 2) % a.H : r;
  int         mi  = 0;
  for (int mo = 0; mo < 3; ++mo) {
    if (!(m.mask & (1 << mo)))
      continue;
    for (int i = lane; i < N; i += 32) {
      const int cc = m.fftshift ? (i + N / 2) % N : i;
      out[mi * a.out_plane + (int64_t)rr * a.out_row + cc] = __fdiv_rn(acc[mo * N + i], nzf);
    }
    ++mi;
  }
}

// ------------------------------------------------------------------------------------------------
// Direct-DFT fallback for lengths the four-step kernels do not cover (O(n^2) per line).
// ------------------------------------------------------------------------------------------------
template <bool INV> __device__ __forceinline__ float2 unit_root(int64_t m, int n) {
  float s, c;
  sincospif((INV ? 2.0f : -2.0f) * (float)m / (float)n, &s, &c);
  return make_float2(c, s);
}

template <bool INV> __global__ void row_dft_generic_kernel(RowPass a) {
  const int     w     = blockIdx.y;
  const int64_t total = (int64_t)a.nplanes * a.H * a.N;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int k     = (int)(e % a.N);
    const int64_t row = e / a.N;
    const int plane = (int)(row / a.H), r = (int)(row % a.H);
    const int ir    = r - a.oy;
    float2    acc   = make_float2(0.f, 0.f);
    if (ir >= 0 && ir < a.IH) {
      const int64_t ibase = w * a.in_win + plane * a.in_plane + (int64_t)ir * a.in_row;
      for (int col = 0; col < a.N; ++col) {
        const int ic = col - a.ox;
        if (ic < 0 || ic >= a.IW)
          continue;
        const int64_t off = ibase + (int64_t)ic * a.in_col;
        float2 v = a.in_real ? make_float2(reinterpret_cast<const float *>(a.in)[off], 0.f)
                             : reinterpret_cast<const float2 *>(a.in)[off];
        if (a.pre)
          v = cmul(v, a.pre[(int64_t)r * a.N + col]);
        acc = cadd(acc, cmul(v, unit_root<INV>(((int64_t)col * k) % a.N, a.N)));
      }
    }
    a.out[w * a.out_win + plane * a.out_plane + (int64_t)r * a.out_row + k] = acc;
  }
}

// Column DFT: complex in -> complex out (optionally x post), or -> |.| (float).
template <bool INV> __global__ void col_dft_generic_kernel(ColPass a, int magnitude) {
  const int     w     = blockIdx.y;
  const int64_t total = (int64_t)a.nplanes * a.H * a.W;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int     col   = (int)(e % a.W);
    const int64_t rest  = e / a.W;
    const int     k     = (int)(rest % a.H);
    const int     plane = (int)(rest / a.H);
    const float2 *src   = a.in + w * a.in_win + plane * a.in_plane + col;
    float2        acc   = make_float2(0.f, 0.f);
    for (int row = 0; row < a.H; ++row)
      acc = cadd(acc, cmul(src[(int64_t)row * a.in_row], unit_root<INV>(((int64_t)row * k) % a.H, a.H)));
    const int64_t o = w * a.out_win + plane * a.out_plane + (int64_t)k * a.out_row + col * a.out_col;
    if (magnitude) {
      reinterpret_cast<float *>(a.out)[o] = hypotf(acc.x, acc.y);
    } else {
      if (a.post)
        acc = cmul(acc, a.post[(int64_t)k * a.W + col]);
      reinterpret_cast<float2 *>(a.out)[o] = acc;
    }
  }
}

int grid_for(int64_t total, int threads) {
  const int64_t blocks = (total + threads - 1) / threads;
  return (int)std::min<int64_t>(blocks, (int64_t)sm_count() * 32);
}

template <int N1, bool INV> int launch_row_fast(const RowPass &a, int nwin, cudaStream_t s) {
  constexpr int N       = N1 * 32;
  const int     threads = 256;
  const size_t  smem    = 2 * N * sizeof(float) + (threads / 32) * XBuf<N1>::kSize * sizeof(float2);
  HF_CUDA(cudaFuncSetAttribute(row_pass_kernel<N1, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  const int64_t rows   = (int64_t)a.nplanes * a.H;
  const int64_t blocks = std::min<int64_t>((rows + 7) / 8, (int64_t)sm_count() * 8);
  row_pass_kernel<N1, INV><<<dim3((unsigned)blocks, nwin), threads, smem, s>>>(a);
  note_launch();
  return launch_status("row_pass_kernel");
}

template <int N1, bool INV>
int launch_col_fast(const ColPass &a, int mode, const MomentSpec &m, int nwin, cudaStream_t s) {
  constexpr int N = N1 * 32;
  constexpr int C = N1 <= 32 ? 8 : 4;
  const size_t  base = 2 * N * sizeof(float) + C * XBuf<N1>::kSize * sizeof(float2);
  const int     strips = (a.W + C - 1) / C;
  // CTAs along planes: enough for ~2 CTAs per SM overall, each striding over the rest
  const int64_t want       = std::max<int64_t>(1, (2LL * sm_count() + (int64_t)strips * nwin - 1) /
                                                    ((int64_t)strips * nwin));
  const int     plane_grid = (int)std::min<int64_t>(a.nplanes, want);
  switch (mode) {
#define HF_COL_CASE(MODE, EXTRA, PLANES)                                                           \
  case MODE: {                                                                                     \
    const size_t smem = base + (EXTRA);                                                            \
    HF_CUDA(cudaFuncSetAttribute(col_pass_kernel<N1, C, INV, MODE>,                                \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));         \
    col_pass_kernel<N1, C, INV, MODE><<<dim3(strips, PLANES, nwin), 32 * C, smem, s>>>(a, m);      \
    note_launch();                                                                                 \
    return launch_status("col_pass_kernel");                                                       \
  }
    HF_COL_CASE(COL_COMPLEX, 0, plane_grid)
    HF_COL_CASE(COL_MAGNITUDE, 0, plane_grid)
    HF_COL_CASE(COL_MOMENTS, (size_t)3 * N * C * sizeof(float), 1)
#undef HF_COL_CASE
  case COL_TF_SANDWICH:
    if constexpr (N1 <= 32) {
      const size_t smem = base;
      HF_CUDA(cudaFuncSetAttribute(col_pass_kernel<N1, C, INV, COL_TF_SANDWICH>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      col_pass_kernel<N1, C, INV, COL_TF_SANDWICH>
          <<<dim3(strips, plane_grid, nwin), 32 * C, smem, s>>>(a, m);
      note_launch();
      return launch_status("col_pass_kernel");
    }
    return fail(HF_ERR_UNSUPPORTED, "transfer-function column pass needs H <= 1024");
  default:
    return fail(HF_ERR_INVALID, "unknown column mode");
  }
}

template <int N1, bool INV>
int launch_rowmom_fast(const ColPass &a, const MomentSpec &m, int nwin, cudaStream_t s) {
  constexpr int N       = N1 * 32;
  const int     threads = 128;
  const int     nwarps  = threads / 32;
  const size_t  smem    = 2 * N * sizeof(float) + nwarps * XBuf<N1>::kSize * sizeof(float2) +
                      (size_t)nwarps * 3 * N * sizeof(float);
  HF_CUDA(cudaFuncSetAttribute(row_moments_kernel<N1, INV>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  row_moments_kernel<N1, INV><<<dim3((a.H + nwarps - 1) / nwarps, nwin), threads, smem, s>>>(a, m);
  note_launch();
  return launch_status("row_moments_kernel");
}

#define HF_DISPATCH_N1(n, CALL)                                                                    \
  switch ((n) / 32) {                                                                              \
  case 2: { constexpr int N1 = 2; CALL; }                                                          \
  case 4: { constexpr int N1 = 4; CALL; }                                                          \
  case 8: { constexpr int N1 = 8; CALL; }                                                          \
  case 16: { constexpr int N1 = 16; CALL; }                                                        \
  case 24: { constexpr int N1 = 24; CALL; }                                                        \
  case 32: { constexpr int N1 = 32; CALL; }                                                        \
  case 48: { constexpr int N1 = 48; CALL; }                                                        \
  default: break;                                                                                  \
  }

} // namespace

int launch_row_pass(const RowPass &a, int nwin, cudaStream_t s) {
  HF_CHECK_ARG(a.N > 0 && a.H > 0 && a.nplanes > 0 && nwin > 0, "row pass: empty problem");
  if (fft_fast_length(a.N)) {
    if (a.inverse) {
      HF_DISPATCH_N1(a.N, return (launch_row_fast<N1, true>(a, nwin, s)))
    } else {
      HF_DISPATCH_N1(a.N, return (launch_row_fast<N1, false>(a, nwin, s)))
    }
  }
  const int64_t total = (int64_t)a.nplanes * a.H * a.N;
  if (a.inverse)
    row_dft_generic_kernel<true><<<dim3(grid_for(total, 256), nwin), 256, 0, s>>>(a);
  else
    row_dft_generic_kernel<false><<<dim3(grid_for(total, 256), nwin), 256, 0, s>>>(a);
  note_launch();
  return launch_status("row_dft_generic_kernel");
}

int launch_col_pass(const ColPass &a, int mode, const MomentSpec *mom, int nwin, cudaStream_t s) {
  HF_CHECK_ARG(a.H > 0 && a.W > 0 && a.nplanes > 0 && nwin > 0, "column pass: empty problem");
  MomentSpec m{};
  if (mom)
    m = *mom;
  if (mode == COL_MOMENTS)
    HF_CHECK_ARG(mom != nullptr && mom->nz == a.nplanes && a.nplanes <= kMaxBands,
                 "column moments: bad moment spec");
  if (fft_fast_length(a.H)) {
    if (a.inverse) {
      HF_DISPATCH_N1(a.H, return (launch_col_fast<N1, true>(a, mode, m, nwin, s)))
    } else {
      HF_DISPATCH_N1(a.H, return (launch_col_fast<N1, false>(a, mode, m, nwin, s)))
    }
  }
  if (mode != COL_COMPLEX && mode != COL_MAGNITUDE)
    return fail(HF_ERR_UNSUPPORTED, "fused column mode needs a four-step length");
  const int64_t total = (int64_t)a.nplanes * a.H * a.W;
  if (a.inverse)
    col_dft_generic_kernel<true><<<dim3(grid_for(total, 256), nwin), 256, 0, s>>>(a, mode == COL_MAGNITUDE);
  else
    col_dft_generic_kernel<false><<<dim3(grid_for(total, 256), nwin), 256, 0, s>>>(a, mode == COL_MAGNITUDE);
  note_launch();
  return launch_status("col_dft_generic_kernel");
}

int launch_row_moments(const ColPass &a, const MomentSpec &m, int nwin, cudaStream_t s) {
  HF_CHECK_ARG(fft_fast_length(a.W), "row moments: unsupported row length");
  HF_CHECK_ARG(m.nz > 0 && m.nz <= kMaxBands, "row moments: bad moment spec");
  if (a.inverse) {
    HF_DISPATCH_N1(a.W, return (launch_rowmom_fast<N1, true>(a, m, nwin, s)))
  } else {
    HF_DISPATCH_N1(a.W, return (launch_rowmom_fast<N1, false>(a, m, nwin, s)))
  }
  return fail(HF_ERR_UNSUPPORTED, "row moments: unsupported row length");
}

} // namespace hf
