// Chosen form, raw band planes on the tensor cores, in row segments.
//
// The fused pass (k_tc_band.cu) needs a whole image row in shared memory and TMEM because it runs
// the row FFT; that fixes T = 64, W <= 1024 and Nz <= 32.  Without the row FFT no full row is
// needed, so this pass covers the other shapes of the path: T = 32, 64 or 128 frames, any width
// that is a multiple of 128, up to 64 band bins, and every propagation (the angular spectrum and
// the autofocus need the band planes before any lens).  It stores
//   S[p][k] = sum_t (x_t[p] - 2048) (Wh + Wl)[t][k] + 2048 sum_t (Wh + Wl)[t][k]
// for each pixel p of a segment of `seg` 128-pixel tiles of one row, with Wh = f16(W) and
// Wl = f16(W - Wh) as in the fused pass: A = the segment's samples x - 2048 (exact in f16 for
// 12-bit data), MN-major [T][128] per tile; B = Wh / Wl as real/imaginary rows, K-major in 64-frame
// atoms; tcgen05.mma M = 128, N = 16 ceil(2 Nz / 16), K = 16, f32 accumulators in TMEM (tile j ->
// columns j * ncol .. j * ncol + N - 1, ncol the power of two >= N).  The later passes (row FFT
// with the lens, column FFT and moments, or the angular spectrum) read the planes as the plain
// band DFT leaves them.
//
// Warp roles (384 threads, one CTA per SM, persistent over segments taken from a counter):
//   warps 0-3  : load + unpack the next segment into A, rebuild B per window, and (thread 0)
//                issue the MMAs once the epilogue has released TMEM;
//   warps 4-11 : epilogue; warp 4 + 4h + q reads TMEM lane quarter q of the tiles j = h (mod 2),
//                adds the DC correction and stores each bin's 32 pixels as one coalesced row.
// mbarriers `full` (MMAs of a segment complete: TMEM readable, A/B reusable) and `free` (the 8
// epilogue warps finished reading TMEM), with bounded waits as in the fused pass.
//
// One launch can serve several acquisitions of the same window length and sample format (the
// batched uneven acquisitions): each is a job with its own ring, W, planes and geometry, and the
// units of all jobs form one work list, (job, window, row, segment) in order, taken from the one
// counter.
#include <algorithm>
#include <initializer_list>

#include <cuda_fp16.h>

#include "k_tc_band.cuh"
#include "tc_band_common.cuh"
#include "tc_common.cuh"

namespace hf {

namespace {

using tcb::GroupLoad;
using tcb::mbar_arrive;
using tcb::mbar_arrive_cnt;
using tcb::named_bar;
using tcb::wait_or_abort;

constexpr int kSegLoaders  = 128; // warps 0-3
constexpr int kSegEpilogue = 256; // warps 4-11
constexpr int kSegThr      = kSegLoaders + kSegEpilogue;
constexpr int kSegABytes   = 131072; // A operand: seg tiles x T frames x 128 pixels, f16 (seg T <= 512)
constexpr int kSegMaxN     = 128;    // MMA N (Nz <= 64)

struct SegGeom {
  int N;    // MMA N, 16 ceil(2 Nz / 16)
  int ncol; // TMEM columns per tile: the power of two >= N (>= 32)
  int seg;  // tiles per segment
  int spr;  // segments per row
};

// One acquisition of a launch.
struct SegJob {
  FrameRing     ring;
  const float2 *wmat;
  int64_t       wmat_stride;
  float2       *out;
  int64_t       out_win, out_plane, out_row;
  int64_t       unit0; // first unit of this job in the launch's work list
  int           H, W, nz, nwin;
  float         shift;
  SegGeom       g;
};

struct SegJobs {
  int     njob;
  int     bpart_max; // bytes of one W part at the largest N of the launch
  int64_t nunits;    // units of all jobs
  int    *status;
  int    *counter;
  SegJob  job[kMaxSegJobs];
};

// Job of unit u (the jobs' first units ascend).
__device__ __forceinline__ int job_of(const SegJobs &J, int64_t u) {
  int ji = 0;
  while (ji + 1 < J.njob && u >= J.job[ji + 1].unit0)
    ++ji;
  return ji;
}

template <int FMT, int T>
__global__ void __launch_bounds__(kSegThr, 1) band_seg_tc_kernel(const __grid_constant__ SegJobs J) {
  constexpr int KA   = (T + 63) / 64; // 64-frame K atoms of B
  constexpr int KS   = T / 16;        // k-steps per W part
  constexpr int TILE = T * 256;       // A tile bytes: [T][128] f16
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // aligned by pointer arithmetic on the shared array, so every derived pointer stays a shared-space
  // pointer
  uint8_t  *smem   = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t  *sA     = smem;                                        // g.seg tiles
  uint8_t  *sB     = sA + kSegABytes;                             // hi [KA][N][128 B], then lo
  float    *colsum = reinterpret_cast<float *>(sB + 2 * J.bpart_max); // [2][128], by window parity
  int64_t  *foff   = reinterpret_cast<int64_t *>(colsum + 256);   // [T] frame offsets of the window
  int64_t  *unitbuf = foff + 128;                                 // [2] unit of iteration k, by parity
  uint64_t *mbar   = reinterpret_cast<uint64_t *>(unitbuf + 2);   // [0] full, [1] free
  uint32_t *tslot  = reinterpret_cast<uint32_t *>(mbar + 2);
  int      *abort_flag = reinterpret_cast<int *>(tslot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    tc::mbar_init(&mbar[0], 2); // the MMA commit + the issuing thread's release arrive
    tc::mbar_init(&mbar[1], kSegEpilogue / 32);
    *abort_flag = 0;
    tc::mbar_fence_init();
  }
  if (warp == 0)
    tc::tmem_alloc(tslot, 512);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase  = *tslot;
  volatile int  *abortv = abort_flag;
  const int64_t  nunits = J.nunits;

  if (tid < kSegLoaders) {
    // ------------------------------------------------------------------ loader / MMA warps
    int k = 0, cur_ji = -1, cur_w = -1, wpar = 1;
    for (;; ++k) {
      if (k > 0) // MMAs of the previous segment done: A and B may be overwritten
        wait_or_abort(&mbar[0], (uint32_t)((k - 1) & 1), abortv, J.status, 31);
      if (tid == 0)
        unitbuf[k & 1] = atomicAdd(J.counter, 1);
      named_bar(1, kSegLoaders);
      const int64_t u = unitbuf[k & 1];
      if (u >= nunits) { // no segments left: complete this phase empty so that the epilogue ends too
        if (tid == 0) {
          // only after the epilogue has released the previous segment (see the fused pass)
          if (k > 0)
            wait_or_abort(&mbar[1], (uint32_t)((k - 1) & 1), abortv, J.status, 34);
          mbar_arrive_cnt(&mbar[0], 2);
        }
        break;
      }
      const int     ji  = job_of(J, u);
      const SegJob &a   = J.job[ji];
      const SegGeom g   = a.g;
      const int     bpart = KA * g.N * 128;
      const int64_t uj  = u - a.unit0;
      const int     w   = (int)(uj / ((int64_t)a.H * g.spr));
      const int64_t rem = uj % ((int64_t)a.H * g.spr);
      const int     r = (int)(rem / g.spr), sg = (int)(rem % g.spr);
      const int     j0 = sg * g.seg, nt = min(g.seg, a.W / 128 - j0);
      const bool    new_w = w != cur_w || ji != cur_ji;
      if (new_w) { // per window: frame offsets and B = (Wh, Wl) rows n = 2 bin + {re, im}
        cur_ji = ji;
        cur_w  = w;
        wpar ^= 1;
        for (int t = tid; t < T; t += kSegLoaders)
          foff[t] = a.ring.frame(w, t) - a.ring.base;
        const float2 *wm = a.wmat + (int64_t)w * a.wmat_stride;
        for (int e = tid; e < g.N * (T / 8); e += kSegLoaders) {
          const int n = e / (T / 8), c8 = e % (T / 8); // one 16-byte chunk = 8 frames
          __half    hv[8], lv[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int t = 8 * c8 + i;
            float     v = 0.f;
            if ((n >> 1) < a.nz) {
              const float2 z = __ldg(wm + (int64_t)t * a.nz + (n >> 1));
              v              = (n & 1) ? z.y : z.x;
            }
            hv[i] = __float2half_rn(v);
            lv[i] = __float2half_rn(v - __half2float(hv[i]));
          }
          const int off = (c8 >> 3) * g.N * 128 + n * 128 + (((c8 & 7) ^ (n & 7)) << 4);
          *reinterpret_cast<uint4 *>(sB + off)         = *reinterpret_cast<const uint4 *>(hv);
          *reinterpret_cast<uint4 *>(sB + bpart + off) = *reinterpret_cast<const uint4 *>(lv);
        }
        named_bar(1, kSegLoaders); // frame offsets visible to every loader
      }
      // A: tile j = pixels [128 (j0 + j), +128) of row r; element (m, t) at
      //    (m/64)*(128 T) + (t/8)*1024 + (t%8)*128 + ((m%64/8) ^ (t%8))*16 + (m%8)*2.
      //    Work item `it` = (tile j, frame t, 32-pixel group grp); consecutive threads take the four
      //    groups of one frame row, so each quad reads 128 contiguous pixels.  The packed words of
      //    round rd + 1 are loaded before round rd is unpacked.
      {
        using GL          = GroupLoad<FMT>;
        constexpr int U   = GL::kPerRound;
        constexpr int NR  = (kSegABytes / 256 * 4 / kSegLoaders + U - 1) / U; // rounds at most
        const int  nitems = nt * T * 4;
        uint32_t   raw[2][U][GL::kWords];
        const float magic = 8388608.f + a.shift; // x - shift exactly: (2^23 + x) - (2^23 + shift)
        auto load_round = [&](int rd, uint32_t (&dst)[U][GL::kWords]) {
#pragma unroll
          for (int uu = 0; uu < U; ++uu) {
            const int it = (rd * U + uu) * kSegLoaders + tid;
            if (it < nitems) {
              const int j = it / (T * 4), t = (it >> 2) % T, grp = it & 3;
              GL::raw(a.ring.base + foff[t] + ((int64_t)r * a.W + 128 * (j0 + j) + 32 * grp) * GL::kBytes / 32,
                      dst[uu]);
            }
          }
        };
        load_round(0, raw[0]);
#pragma unroll
        for (int rd = 0; rd < NR; ++rd) {
          if (rd + 1 < NR)
            load_round(rd + 1, raw[(rd + 1) & 1]);
#pragma unroll
          for (int uu = 0; uu < U; ++uu) {
            const int it = (rd * U + uu) * kSegLoaders + tid;
            if (it >= nitems)
              continue;
            const int j = it / (T * 4), t = (it >> 2) % T, grp = it & 3;
            uint32_t  v[32];
            GL::unpack(raw[rd & 1][uu], v);
            uint8_t *tile = sA + j * TILE;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int m0 = 32 * grp + 8 * q;
              __half2   h[4];
#pragma unroll
              for (int i = 0; i < 4; ++i)
                h[i] = __floats2half2_rn(__uint_as_float(0x4B000000u | v[8 * q + 2 * i]) - magic,
                                         __uint_as_float(0x4B000000u | v[8 * q + 2 * i + 1]) - magic);
              const int chunk = (m0 & 63) >> 3;
              uint8_t  *dst   = tile + (m0 >> 6) * (T * 128) + (t >> 3) * 1024 + (t & 7) * 128 + ((chunk ^ (t & 7)) << 4);
              *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(h);
            }
          }
        }
      }
      named_bar(1, kSegLoaders); // A (and B) complete
      if (new_w && tid < g.N) { // DC correction of the shifted samples: shift * sum_t (hi + lo)[t][n]
        float sacc = 0.f;
        for (int t = 0; t < T; ++t) {
          const int c   = (t & 63) >> 3;
          const int off = (t >> 6) * g.N * 128 + tid * 128 + ((c ^ (tid & 7)) << 4) + (t & 7) * 2;
          sacc += __half2float(*reinterpret_cast<const __half *>(sB + off)) +
                  __half2float(*reinterpret_cast<const __half *>(sB + bpart + off));
        }
        colsum[wpar * 128 + tid] = a.shift * sacc;
      }
      tc::fence_proxy_async_smem();
      named_bar(1, kSegLoaders);
      if (tid == 0) {
        if (k > 0) // the epilogue has read the previous segment out of TMEM
          wait_or_abort(&mbar[1], (uint32_t)((k - 1) & 1), abortv, J.status, 32);
        tc::fence_after_sync();
        if (!*abortv) {
          const uint32_t idesc = tc::idesc_f16(128, g.N, true, false);
          for (int j = 0; j < nt; ++j)
#pragma unroll
            for (int s = 0; s < 2 * KS; ++s) { // k-steps 0..KS-1 with W hi, then the same with W lo
              const int      part = s / KS, ks = s % KS;
              const uint64_t ad   = tc::sw128_desc(tc::smem_u32(sA + j * TILE + ks * 2048), T * 128, 1024);
              const uint64_t bd =
                  tc::sw128_desc(tc::smem_u32(sB + part * bpart + (ks >> 2) * g.N * 128 + (ks & 3) * 32), 16, 1024);
              tc::mma_f16(tbase + (uint32_t)(j * g.ncol), ad, bd, idesc, s > 0 ? 1u : 0u);
            }
        }
        tc::mma_commit(&mbar[0]);
        mbar_arrive(&mbar[0]); // release: the unit index, B and the DC correction are in place
      }
    }
  } else {
    // ------------------------------------------------------------------ epilogue warps
    const int e = warp - 4, q = warp & 3, half = e >> 2;
    int       k = 0, cur_ji = -1, cur_w = -1, wpar = 1;
    for (;; ++k) {
      wait_or_abort(&mbar[0], (uint32_t)(k & 1), abortv, J.status, 33);
      tc::fence_after_sync();
      const int64_t u = unitbuf[k & 1];
      if (u >= nunits || *abortv)
        break;
      const int     ji   = job_of(J, u);
      const SegJob &a    = J.job[ji];
      const SegGeom g    = a.g;
      const int     ngrp = (2 * a.nz + 7) / 8; // 8-column groups = 4 bins
      const int64_t uj   = u - a.unit0;
      const int     w    = (int)(uj / ((int64_t)a.H * g.spr));
      const int64_t rem  = uj % ((int64_t)a.H * g.spr);
      const int     r = (int)(rem / g.spr), sg = (int)(rem % g.spr);
      const int     j0 = sg * g.seg, nt = min(g.seg, a.W / 128 - j0);
      if (w != cur_w || ji != cur_ji) {
        cur_ji = ji;
        cur_w  = w;
        wpar ^= 1;
      }
      const float *cs   = colsum + wpar * 128;
      float2      *orow = a.out + (int64_t)w * a.out_win + (int64_t)r * a.out_row + 32 * q + lane;
      for (int j = half; j < nt; j += 2) {
        float2 *op = orow + 128 * (j0 + j);
        for (int g0 = 0; g0 < ngrp; g0 += 4) { // four TMEM loads in flight, one wait
          uint32_t  v[4][8];
          const int ng = min(4, ngrp - g0);
#pragma unroll
          for (int gi = 0; gi < 4; ++gi)
            if (gi < ng)
              tc::tmem_ld8(tbase + ((uint32_t)(32 * q) << 16) + (uint32_t)(j * g.ncol + 8 * (g0 + gi)), v[gi]);
          tc::tmem_wait_ld();
#pragma unroll
          for (int gi = 0; gi < 4; ++gi)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
              const int bin = 4 * (g0 + gi) + b;
              if (gi < ng && bin < a.nz)
                op[(int64_t)bin * a.out_plane] =
                    cadd(make_float2(__uint_as_float(v[gi][2 * b]), __uint_as_float(v[gi][2 * b + 1])),
                         reinterpret_cast<const float2 *>(cs)[bin]);
            }
        }
      }
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0)
        mbar_arrive(&mbar[1]);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, 512);
  }
}

// seg_cap > 0 caps the tiles per segment (the autotuner's tile parameter); 0 takes the most that A
// and TMEM hold.
SegGeom seg_geom(int T, int W, int nz, int seg_cap) {
  SegGeom g{};
  g.N    = 16 * ((2 * nz + 15) / 16);
  g.ncol = g.N <= 32 ? 32 : (g.N <= 64 ? 64 : 128);
  g.seg  = std::min({512 / g.ncol, kSegABytes / (T * 256), W / 128});
  if (seg_cap > 0)
    g.seg = std::min(g.seg, seg_cap);
  g.spr  = (W / 128 + g.seg - 1) / g.seg;
  return g;
}

template <int FMT, int T> int launch_t(SegJobs &J, int max_ctas, cudaStream_t s) {
  const size_t smem = 1024 + (size_t)kSegABytes + 2 * (size_t)J.bpart_max + 256 * 4 + 128 * 8 + 2 * 8 + 2 * 8 + 16;
  HF_CUDA(cudaFuncSetAttribute(band_seg_tc_kernel<FMT, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int cap  = max_ctas > 0 ? std::min(max_ctas, sm_count()) : sm_count();
  const int grid = (int)std::min<int64_t>(J.nunits, cap);
  HF_CUDA(cudaMemsetAsync(J.counter, 0, sizeof(int), s));
  band_seg_tc_kernel<FMT, T><<<grid, kSegThr, smem, s>>>(J);
  note_launch();
  return launch_status("band_seg_tc_kernel");
}

} // namespace

bool band_seg_tc_supported(int fmt, int T, int W, int nz, int64_t frame_bytes) {
  return (fmt == HF_MONO12P || fmt == HF_U16) && (T == 32 || T == 64 || T == 128) && W >= 128 && W % 128 == 0 &&
         nz >= 1 && 2 * nz <= kSegMaxN && frame_bytes % 16 == 0;
}

int launch_band_seg_tc_multi(const BandRowsArgs *jobs, int njobs, int fmt, int seg_cap, int max_ctas, int *counter,
                             int *status, cudaStream_t s) {
  HF_CHECK_ARG(jobs != nullptr && njobs >= 1 && njobs <= kMaxSegJobs, "band segments: 1 to 16 jobs per launch");
  HF_CHECK_ARG(counter != nullptr, "band segments: unit counter missing");
  const int T = jobs[0].T;
  SegJobs   J{};
  J.njob = njobs, J.status = status, J.counter = counter;
  for (int i = 0; i < njobs; ++i) {
    const BandRowsArgs &a = jobs[i];
    HF_CHECK_ARG(a.T == T, "band segments: the jobs of one launch share the window length");
    HF_CHECK_ARG(band_seg_tc_supported(fmt, a.T, a.W, a.nz, a.ring.frame_bytes),
                 "band segments (tensor core): unsupported shape");
    HF_CHECK_ARG(((uintptr_t)a.ring.base & 15) == 0, "band segments (tensor core): ring must be 16-byte aligned");
    HF_CHECK_ARG(a.nwin >= 1 && a.H >= 1, "band segments: empty job");
    SegJob &j = J.job[i];
    j.ring = a.ring, j.wmat = a.wmat, j.wmat_stride = a.wmat_stride, j.out = a.out;
    j.out_win = a.out_win, j.out_plane = a.out_plane, j.out_row = a.out_row;
    j.H = a.H, j.W = a.W, j.nz = a.nz, j.nwin = a.nwin, j.shift = a.shift;
    j.g     = seg_geom(T, a.W, a.nz, seg_cap);
    j.unit0 = J.nunits;
    J.nunits += (int64_t)a.nwin * a.H * j.g.spr;
    J.bpart_max = std::max(J.bpart_max, ((T + 63) / 64) * j.g.N * 128);
  }
  switch (T) {
  case 32: return fmt == HF_MONO12P ? launch_t<HF_MONO12P, 32>(J, max_ctas, s) : launch_t<HF_U16, 32>(J, max_ctas, s);
  case 64: return fmt == HF_MONO12P ? launch_t<HF_MONO12P, 64>(J, max_ctas, s) : launch_t<HF_U16, 64>(J, max_ctas, s);
  default:
    return fmt == HF_MONO12P ? launch_t<HF_MONO12P, 128>(J, max_ctas, s) : launch_t<HF_U16, 128>(J, max_ctas, s);
  }
}

int launch_band_seg_tc(const BandRowsArgs &a, int fmt, cudaStream_t s) {
  return launch_band_seg_tc_multi(&a, 1, fmt, 0, a.max_ctas, a.row_counter, a.status, s);
}

} // namespace hf
