// Column FFT + |.| + M0/M1/M2 over the band planes of a window, fed by TMA.
//
// This is the last pass of the Fresnel path: after the band DFT, lens and row FFT, each band plane
// S_k needs its column transform, and the moment images are M_j = mean_k f_k^j |S_k| over the band
// (graph_builder.cc:604-631; Abs = sqrtf(x*x + y*y) as holonp/src/abs.cu:67-70, Mean over the band
// axis as holonp/src/mean.cu:268-305, accumulated in band order in float32 and divided by Nz).
// The plain form keeps exactly that float32 sequence; the chosen form (FAST) takes the hardware
// square-root approximation and fuses the weighted sums, which removes about a seventh of the
// pass's instructions for a relative change far below its 1e-3 error budget.
//
// A CTA owns a strip of C = kColMomCols (4) columns of one window for all Nz planes, and two
// CTAs share an SM (128 threads, under 255 registers, 74 KB of shared memory each), so one CTA's
// barrier or stage wait is covered by the other's work (strips of 8 columns in one CTA per SM took
// 8 % longer):
//  - one thread issues 2D TMA tile loads of a plane's [H][C] strip into one of two shared-memory
//    stages, so the next plane streams in while this one is transformed;
//  - thread (n2, c) loads its column's samples n2 + 32 n1 from the stage, runs the N1-point DFT in
//    registers, twiddles by w_N^(n2 k1) from a [N1][32] table (one shared load, no index math)
//    and writes the exchange back into the same stage at k1 * (32 C + C) + n2 * C + c: a warp
//    reads 32 / C rows k1 of C entries each, and the C-entry pad per row shifts consecutive rows
//    by C bank pairs, so the transposed reads are conflict-free, and every address is the
//    thread's base plus a compile-time offset;
//  - thread (k1, c) reads Y[0..31][k1], runs the 32-point DFT and accumulates |X| f^j for its 32
//    output rows k1 + N1 k2 in registers.
// Waits on the stage barriers are bounded: an expired wait sets the status word and every thread
// leaves the plane loop together.
#include "k_cols_tma.cuh"

#include "fft_core.cuh"
#include "tc_common.cuh"

namespace hf {
namespace {

constexpr int kColC = kColMomCols; // columns per CTA strip

__device__ __forceinline__ bool wait_stage(uint64_t *mbar, uint32_t parity, volatile int *abort, int *status) {
  const uint64_t t0 = tc::globaltimer_ns();
  for (uint32_t i = 0; i < tc::kWaitLimit; ++i) {
    if (tc::mbar_try_wait(mbar, parity))
      return true;
    if ((i & 255u) == 255u && (*abort || tc::globaltimer_ns() - t0 > tc::kWaitNs))
      break;
  }
  if (*abort)
    return false;
  if (status)
    atomicCAS(status, 0, 21);
  *abort = 1;
  return false;
}

template <int N1, int C, bool FAST>
__global__ void __launch_bounds__(32 * C, 1)
    col_moments_tma_kernel(const __grid_constant__ CUtensorMap tmap, ColMomArgs a, MomentSpec m) {
  constexpr int      N        = N1 * 32;
  constexpr int      NT       = 32 * C;
  constexpr int      kBoxRows = N < 256 ? N : 256;
  constexpr int      kBoxes   = N / kBoxRows;
  constexpr uint32_t kStage   = (uint32_t)N * C * sizeof(float2); // bytes one plane's boxes bring
  constexpr int      kXRow    = 32 * C + C;                      // exchange row (one k1) in float2
  constexpr int      kSlot    = (N1 * kXRow + 15) / 16 * 16;    // stage slot (128-byte multiple)
  extern __shared__ __align__(128) uint8_t smem[];
  float2   *stage      = reinterpret_cast<float2 *>(smem);     // [2][kSlot]
  float2   *tw         = stage + 2 * kSlot;                    // [N1][32]: w_N^(k1 * n2)
  uint64_t *mbar       = reinterpret_cast<uint64_t *>(tw + N); // [2]
  int      *abort_flag = reinterpret_cast<int *>(mbar + 2);

  const int tid = threadIdx.x, n2 = tid / C, c = tid % C;
  const int strip = blockIdx.x, w = blockIdx.y;
  const int col   = strip * C + c;
  const int k1    = n2; // store role

  for (int i = tid; i < N; i += NT) {
    float sv, cv;
    sincospif(-2.0f * (float)((i >> 5) * (i & 31)) / (float)N, &sv, &cv);
    tw[i] = make_float2(cv, sv);
  }
  if (tid == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
    *abort_flag = 0;
    tc::mbar_fence_init();
    tc::tma_prefetch_desc(&tmap);
  }
  __syncthreads();

  const int64_t row_base = (int64_t)w * a.rows_per_win;
  auto issue = [&](int plane, int s) {
    tc::mbar_arrive_expect_tx(&mbar[s], kStage);
#pragma unroll
    for (int b = 0; b < kBoxes; ++b)
      tc::tma_load_2d(stage + (size_t)s * kSlot + (size_t)b * kBoxRows * C, &tmap, strip * C * 2,
                      (int)(row_base + (int64_t)plane * N + b * kBoxRows), &mbar[s]);
  };
  if (tid == 0) {
    issue(0, 0);
    if (a.nz > 1)
      issue(1, 1);
  }

  // moment sums of output rows (k2, k2 + 1) as packed pairs: each fp32x2 add / multiply / FMA
  // rounds every lane as its scalar form, so the sums are those of the scalar sequence
  float2 acc0[16], acc1[16], acc2[16];
#pragma unroll
  for (int i = 0; i < 16; ++i)
    acc0[i] = acc1[i] = acc2[i] = make_float2(0.f, 0.f);
  volatile int *abortv = abort_flag;

  for (int plane = 0; plane < a.nz; ++plane) {
    const int s  = plane & 1;
    float2   *st = stage + (size_t)s * kSlot;
    const bool ok = wait_stage(&mbar[s], (uint32_t)((plane >> 1) & 1), abortv, a.status);
    float2     x[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1)
      x[n1] = st[(n2 + 32 * n1) * C + c];
    if (__syncthreads_or(!ok)) // every sample is in registers; the stage becomes the exchange
      break;
    dft_reg<N1, false>(x);
#pragma unroll
    for (int k = 0; k < N1; ++k) {
      float2 v = x[k];
      if (k != 0)
        v = cmul(v, tw[k * 32 + n2]);
      st[k * kXRow + n2 * C + c] = v;
    }
    __syncthreads();
    if (k1 < N1) {
      float2 y[32];
#pragma unroll
      for (int j = 0; j < 32; ++j)
        y[j] = st[k1 * kXRow + j * C + c];
      dft_reg<32, false>(y);
      const float2 f1 = make_float2(m.w1[plane], m.w1[plane]), f2 = make_float2(m.w2[plane], m.w2[plane]);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        float2 mag;
        if constexpr (FAST) { // sqrt.approx (relative error ~2^-22) and fused weighted sums
          asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(mag.x) : "f"(fmaf(y[2 * i].x, y[2 * i].x, y[2 * i].y * y[2 * i].y)));
          asm("sqrt.approx.ftz.f32 %0, %1;"
              : "=f"(mag.y)
              : "f"(fmaf(y[2 * i + 1].x, y[2 * i + 1].x, y[2 * i + 1].y * y[2 * i + 1].y)));
          acc0[i] = cadd(acc0[i], mag);
          acc1[i] = cfma2(f1, mag, acc1[i]);
          acc2[i] = cfma2(f2, mag, acc2[i]);
        } else { // the reference's float32 sequence: sqrtf(x*x + y*y), then sums in band order
          mag.x   = __fsqrt_rn(__fmaf_rn(y[2 * i].x, y[2 * i].x, __fmul_rn(y[2 * i].y, y[2 * i].y)));
          mag.y   = __fsqrt_rn(__fmaf_rn(y[2 * i + 1].x, y[2 * i + 1].x, __fmul_rn(y[2 * i + 1].y, y[2 * i + 1].y)));
          acc0[i] = cadd(acc0[i], mag);
          acc1[i] = cadd(acc1[i], pmul2(f1, mag));
          acc2[i] = cadd(acc2[i], pmul2(f2, mag));
        }
      }
    }
    tc::fence_proxy_async_smem(); // this thread's generic accesses to the stage precede the refill
    __syncthreads();
    if (tid == 0 && plane + 2 < a.nz)
      issue(plane + 2, s);
  }

  if (*abortv || k1 >= N1 || col >= a.W)
    return;
  const float nzf = (float)m.nz;
  float      *out = a.out + (int64_t)w * a.out_win;
  const int   cc  = m.fftshift ? (col + a.W / 2) % a.W : col;
  int         mi  = 0;
#pragma unroll
  for (int mo = 0; mo < 3; ++mo) {
    if (!(m.mask & (1 << mo)))
      continue;
    const float2 *acc = mo == 0 ? acc0 : (mo == 1 ? acc1 : acc2);
#pragma unroll
    for (int k2 = 0; k2 < 32; ++k2) {
      const int row = k1 + N1 * k2;
      const int rr  = m.fftshift ? (row + N / 2) % N : row;
      out[mi * a.out_plane + (int64_t)rr * a.out_row + cc] = __fdiv_rn((k2 & 1) ? acc[k2 >> 1].y : acc[k2 >> 1].x, nzf);
    }
    ++mi;
  }
}

template <int N1> int launch_n1(const CUtensorMap &tmap, const ColMomArgs &a, const MomentSpec &m, int nwin,
                                cudaStream_t s) {
  constexpr int N    = N1 * 32;
  const size_t  slot = (size_t)(N1 * (32 * kColC + kColC) + 15) / 16 * 16;
  const size_t  smem = 2 * slot * sizeof(float2) + (size_t)N * sizeof(float2) + 32;
  auto          kern = a.fast ? col_moments_tma_kernel<N1, kColC, true> : col_moments_tma_kernel<N1, kColC, false>;
  HF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const dim3 grid((unsigned)((a.W + kColC - 1) / kColC), (unsigned)nwin);
  kern<<<grid, 32 * kColC, smem, s>>>(tmap, a, m);
  note_launch();
  return launch_status("col_moments_tma_kernel");
}

} // namespace

bool col_moments_tma_supported(int H, int W) {
  return (H == 64 || H == 128 || H == 256 || H == 512 || H == 768 || H == 1024) && W >= 2 && W % 2 == 0;
}

int launch_col_moments_tma(const CUtensorMap &tmap, const ColMomArgs &a, const MomentSpec &m, int nwin,
                           cudaStream_t s) {
  HF_CHECK_ARG(col_moments_tma_supported(a.H, a.W) && a.nz >= 1 && a.nz <= kMaxBands,
               "column moments: unsupported plane size");
  switch (a.H / 32) {
  case 2: return launch_n1<2>(tmap, a, m, nwin, s);
  case 4: return launch_n1<4>(tmap, a, m, nwin, s);
  case 8: return launch_n1<8>(tmap, a, m, nwin, s);
  case 16: return launch_n1<16>(tmap, a, m, nwin, s);
  case 24: return launch_n1<24>(tmap, a, m, nwin, s);
  default: return launch_n1<32>(tmap, a, m, nwin, s);
  }
}

} // namespace hf
