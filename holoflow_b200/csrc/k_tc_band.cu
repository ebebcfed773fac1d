// Chosen form, fused pass 1: temporal band DFT (with the SVD clutter filter folded into W) on the
// tensor cores, lens multiply and the row FFT of every band plane, one image row at a time.
//
// Per image row r of window w (W pixels = W/128 M-tiles):
//   S[p][k] = sum_t (x_t[p] - 2048) (Wh + Wl)[t][k] + 2048 sum_t (Wh + Wl)[t][k]
// with Wh = f16(W) and Wl = f16(W - Wh), is a [W x 64] x [64 x 2nz] product taken twice (Wh, then
// Wl, into the same accumulator): A = the row's samples x - 2048 (exact in f16 for 12-bit data),
// MN-major (pixels contiguous per frame, as they arrive), B = Wh / Wl as real/imaginary columns,
// K-major; tcgen05.mma M = 128, N = 64, K = 16, f32 accumulators in TMEM (tile j -> columns
// 64j .. 64j+63, all 512 columns for W = 1024).
// The epilogue moves 4 bins at a time from TMEM into shared memory (adding the DC correction and
// multiplying by the Fresnel lens), runs each bin's length-W row FFT in place (four-step, padded
// exchange) and stores the row of that band plane.  In raw mode (`raw`, lens null) it stores the
// DC-corrected band rows themselves, for steps that act on the planes before the lens (Filter2D,
// the autofocus).
//
// Warp roles (384 threads, one CTA per SM, persistent over rows):
//   warps 0-3  : load + unpack the next row into the A operand, rebuild B per window, and (thread 0)
//                issue the MMAs once the epilogue has released TMEM;
//   warps 4-11 : epilogue, two teams of four (each warp owns the TMEM lane quarter warp % 4).
// mbarriers: `full` (MMAs of a row complete: TMEM readable, A/B reusable) and `free` (the 8
// epilogue warps finished reading TMEM).  Every wait is bounded; an expired wait sets the status
// word and an abort flag that turns the remaining waits into no-ops, so the kernel always exits.
#include <cuda_fp16.h>

#include "fft_core.cuh"
#include "k_misc.cuh"
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


constexpr int kLoaders   = 128; // warps 0-3
constexpr int kEpilogue  = 256; // warps 4-11
constexpr int kBandTcThr = kLoaders + kEpilogue;
constexpr int kTileBytes = 16384; // [K = 64][M = 128] f16 in two 64-pixel MN atoms of 8 K atoms

template <int FMT, int N1>
__global__ void __launch_bounds__(kBandTcThr, 1) band_rows_tc_kernel(BandRowsArgs a) {
  constexpr int W      = N1 * 32;
  constexpr int NTILE  = W / 128;
  // TMEM is allocated in powers of two columns (>= 32): 6 tiles (W = 768) take 512
  constexpr int NCOL   = NTILE * 64 <= 32 ? 32 : (NTILE * 64 <= 128 ? 128 : (NTILE * 64 <= 256 ? 256 : 512));
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // aligned by pointer arithmetic on the shared array, so every derived pointer stays a shared-space
  // pointer (an integer round trip would turn the accesses into generic ones)
  uint8_t *smem = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t *sA   = smem;                                  // NTILE x 16 KB
  uint8_t *sB   = sA + NTILE * kTileBytes;               // W16 hi, then lo: 2 x 64 rows x 128 B
  constexpr int RS = XBuf<N1>::kSize > W ? XBuf<N1>::kSize : W; // gbuf row stride (room for the exchange)
  float2  *gbuf = reinterpret_cast<float2 *>(sB + 16384); // 8 bins x RS
  float2  *twt  = gbuf + 8 * RS;                         // [N1][32] twiddles w_W^(k1 n2)
  float   *colsum = reinterpret_cast<float *>(twt + W);   // [2][64], indexed by window parity
  int64_t *foff = reinterpret_cast<int64_t *>(colsum + 128); // [64] frame offsets of the window
  int64_t *rowbuf = foff + 64;                               // [2] row of iteration k, by parity
  uint64_t *mbar = reinterpret_cast<uint64_t *>(rowbuf + 2); // [0] full, [1] free
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 2);
  int      *abort_flag = reinterpret_cast<int *>(tslot + 1);
  TwTable   tw{twt, W};

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    tc::mbar_init(&mbar[0], 2); // the MMA commit + the issuing thread's release arrive
    tc::mbar_init(&mbar[1], kEpilogue / 32);
    *abort_flag = 0;
    tc::mbar_fence_init();
  }
  tw.fill(tid, blockDim.x);
  if (warp == 0)
    tc::tmem_alloc(tslot, NCOL);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  volatile int  *abortv = abort_flag;
  constexpr uint32_t idesc = tc::idesc_f16(128, 64, true, false);
  const int64_t nrows = (int64_t)a.nwin * a.H;
  const float   lens_k = a.lens != nullptr ? fresnel_lens_k(a.lambda, a.z) : 0.f;

  if (tid < kLoaders) {
    // ------------------------------------------------------------------ loader / MMA warps
    int k = 0, cur_w = -1, wpar = 1;
    for (;; ++k) {
      if (k > 0) // MMAs of the previous row done: A and B may be overwritten
        wait_or_abort(&mbar[0], (uint32_t)((k - 1) & 1), abortv, a.status, 11);
      if (tid == 0) // rows are taken dynamically, so a CTA that starts late simply does fewer
        rowbuf[k & 1] = atomicAdd(a.row_counter, 1);
      named_bar(1, kLoaders);
      const int64_t row = rowbuf[k & 1];
      if (row >= nrows) { // no rows left: complete this phase empty so that the epilogue ends too
        if (tid == 0) {
          // Only after the epilogue has released the previous row, and so has seen that row's
          // phase: completing this phase earlier could put `full` two phases ahead of the
          // epilogue's parity wait, which could then never succeed.
          if (k > 0)
            wait_or_abort(&mbar[1], (uint32_t)((k - 1) & 1), abortv, a.status, 14);
          mbar_arrive_cnt(&mbar[0], 2);
        }
        break;
      }
      const int w = (int)(row / a.H), r = (int)(row % a.H);
      const bool new_w = w != cur_w;
      if (new_w) { // per window: frame offsets, B = (Wh, Wl) and its DC correction
        cur_w = w;
        wpar ^= 1;
        if (tid < 64)
          foff[tid] = (a.ring.frame(w, tid) - a.ring.base);
      }
      // B (K-major, 128-byte swizzle): row n = 2*bin + {re, im}, K = frame t.  W is split into
      // f16 hi + lo parts (lo = f16(W - hi)); both multiply the same A into one accumulator, so
      // the band carries W to about 22 bits instead of f16's 11 (clutter 100x the signal would
      // otherwise leak through the filter at the f16 rounding of W).
      const float2 *wm = a.wmat + (int64_t)w * a.wmat_stride;
      if (new_w)
      for (int e = tid; e < 64 * 8; e += kLoaders) {
        const int n = e >> 3, c = e & 7; // one 16-byte chunk = 8 frames
        __half hv[8], lv[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int t = 8 * c + i;
          float     v = 0.f;
          if ((n >> 1) < a.nz) {
            const float2 z = __ldg(wm + (int64_t)t * a.nz + (n >> 1));
            v              = (n & 1) ? z.y : z.x;
          }
          hv[i] = __float2half_rn(v);
          lv[i] = __float2half_rn(v - __half2float(hv[i]));
        }
        const int off = n * 128 + ((c ^ (n & 7)) << 4);
        *reinterpret_cast<uint4 *>(sB + off)        = *reinterpret_cast<const uint4 *>(hv);
        *reinterpret_cast<uint4 *>(sB + 8192 + off) = *reinterpret_cast<const uint4 *>(lv);
      }
      if (new_w)
        named_bar(1, kLoaders); // frame offsets visible to every loader
      // A: tile j = pixels [128 j, 128 j + 128) of row r; element (m, t) at
      //    (m/64)*8192 + (t/8)*1024 + (t%8)*128 + ((m%64/8) ^ (t%8))*16 + (m%8)*2.
      //    Work item u of a round is one 32-sample group (frame t, pixels 32 grp ..) of tile j;
      //    the packed words of round rd + 1 are loaded before round rd is unpacked.
      {
        using GL            = GroupLoad<FMT>;
        constexpr int U     = GL::kPerRound;               // groups per thread per round
        constexpr int TPR   = U / 2;                       // tiles per round
        constexpr int NR    = (NTILE + TPR - 1) / TPR;     // rounds per row
        uint32_t      raw[2][U][GL::kWords];
        // x - shift exactly, without an integer conversion: (2^23 + x) - (2^23 + shift)
        const float   magic = 8388608.f + a.shift;
        auto load_round = [&](int rd, uint32_t (&dst)[U][GL::kWords]) {
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int j = rd * TPR + (u >> 1), item = tid + (u & 1) * kLoaders;
            const int t = item >> 2, grp = item & 3;
            if (j < NTILE)
              GL::raw(a.ring.base + foff[t] + ((int64_t)r * W + 128 * j + 32 * grp) * GL::kBytes / 32, dst[u]);
          }
        };
        load_round(0, raw[0]);
#pragma unroll
        for (int rd = 0; rd < NR; ++rd) {
          if (rd + 1 < NR)
            load_round(rd + 1, raw[(rd + 1) & 1]);
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int j = rd * TPR + (u >> 1), item = tid + (u & 1) * kLoaders;
            const int t = item >> 2, grp = item & 3;
            if (j >= NTILE)
              continue;
            uint32_t v[32];
            GL::unpack(raw[rd & 1][u], v);
            uint8_t *tile = sA + j * kTileBytes;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int m0 = 32 * grp + 8 * q;
              __half2 h[4];
#pragma unroll
              for (int i = 0; i < 4; ++i)
                h[i] = __floats2half2_rn(__uint_as_float(0x4B000000u | v[8 * q + 2 * i]) - magic,
                                         __uint_as_float(0x4B000000u | v[8 * q + 2 * i + 1]) - magic);
              const int chunk = (m0 & 63) >> 3;
              uint8_t  *dst   = tile + (m0 >> 6) * 8192 + (t >> 3) * 1024 + (t & 7) * 128 + ((chunk ^ (t & 7)) << 4);
              *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(h);
            }
          }
        }
      }
      named_bar(1, kLoaders); // A (and B) complete
      if (new_w && tid < 64) { // DC correction of the shifted samples: shift * sum_t (hi + lo)[t][n]
        float sacc = 0.f;
        for (int t = 0; t < 64; ++t) {
          const int    c  = t >> 3;
          const int    off = tid * 128 + ((c ^ (tid & 7)) << 4) + (t & 7) * 2;
          sacc += __half2float(*reinterpret_cast<const __half *>(sB + off)) +
                  __half2float(*reinterpret_cast<const __half *>(sB + 8192 + off));
        }
        colsum[wpar * 64 + tid] = a.shift * sacc;
      }
      tc::fence_proxy_async_smem();
      named_bar(1, kLoaders);
      if (tid == 0) {
        if (k > 0) // the epilogue has read the previous row out of TMEM
          wait_or_abort(&mbar[1], (uint32_t)((k - 1) & 1), abortv, a.status, 12);
        tc::fence_after_sync();
        if (!*abortv) {
#pragma unroll
          for (int j = 0; j < NTILE; ++j)
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) { // k-steps 0-3 with W hi, 4-7 with W lo
              const uint64_t ad = tc::sw128_desc(tc::smem_u32(sA + j * kTileBytes + (ks & 3) * 2048), 8192, 1024);
              const uint64_t bd = tc::sw128_desc(tc::smem_u32(sB + (ks >> 2) * 8192 + (ks & 3) * 32), 16, 1024);
              tc::mma_f16(tbase + 64 * j, ad, bd, idesc, ks > 0 ? 1u : 0u);
            }
        }
        tc::mma_commit(&mbar[0]);
        mbar_arrive(&mbar[0]); // release: the row index, B and the DC correction are in place
      }
    }
  } else {
    // ------------------------------------------------------------------ epilogue warps
    // Two teams of four warps; warp q of a team reads TMEM lane quarter q.  A team takes a group
    // of 4 bins (8 TMEM columns per tile), reads it for every tile with one wait, writes the bins'
    // rows (DC-corrected, times the lens) to its half of gbuf and then each of its warps
    // transforms one bin row.  The teams take alternate groups, starting with the other team on
    // every other row, so readout and transforms of the two teams overlap and balance out.
    const int e    = warp - 4;   // 0..7
    const int q    = warp & 3;   // TMEM lane quarter
    const int team = e >> 2;
    float2   *tbuf = gbuf + team * 4 * RS;
    const int bar  = 2 + team;
    const int ngrp = (a.nz + 3) / 4;
    int k = 0, cur_w = -1, wpar = 1;
    for (;; ++k) {
      wait_or_abort(&mbar[0], (uint32_t)(k & 1), abortv, a.status, 13);
      tc::fence_after_sync();
      const int64_t row = rowbuf[k & 1];
      if (row >= nrows || *abortv)
        break;
      const int w = (int)(row / a.H), r = (int)(row % a.H);
      if (w != cur_w) {
        cur_w = w;
        wpar ^= 1;
      }
      const int g0 = (team + k) & 1;
      if (g0 >= ngrp) { // nothing for this team on this row: TMEM is released at once
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0)
          mbar_arrive(&mbar[1]);
        continue;
      }
      // the lens values of this lane's pixels: the lens table's float32 phase, turned into
      // exp(i phase) here (reduced argument, hardware sine/cosine) rather than loaded, so a row
      // starts without a global-load wait
      float2 L[NTILE];
#pragma unroll
      for (int j = 0; j < NTILE; ++j)
        L[j] = a.lens != nullptr ? cis_reduced(fresnel_lens_phase(128 * j + 32 * q + lane, r, W, a.H, lens_k, a.dx))
                                 : make_float2(1.f, 0.f);
      const float *cs = colsum + wpar * 64;
      for (int g = g0; g < ngrp; g += 2) {
        uint32_t v[NTILE][8];
#pragma unroll
        for (int j = 0; j < NTILE; ++j)
          tc::tmem_ld8(tbase + ((uint32_t)(32 * q) << 16) + 64 * j + 8 * g, v[j]);
        tc::tmem_wait_ld();
        if (g + 2 >= ngrp) { // this warp's last TMEM read of the row
          tc::fence_before_sync();
          __syncwarp();
          if (lane == 0)
            mbar_arrive(&mbar[1]);
        }
#pragma unroll
        for (int j = 0; j < NTILE; ++j)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const float2 sv = cadd(make_float2(__uint_as_float(v[j][2 * b]), __uint_as_float(v[j][2 * b + 1])),
                                   reinterpret_cast<const float2 *>(cs)[4 * g + b]);
            tbuf[b * RS + 128 * j + 32 * q + lane] = cmul(sv, L[j]);
          }
        named_bar(bar, 128);
        const int bin = 4 * g + q;
        if (bin < a.nz && a.raw) { // the bin's row as it is, coalesced
          const float2 *buf  = tbuf + q * RS;
          float2       *orow = a.out + (int64_t)w * a.out_win + (int64_t)bin * a.out_plane + (int64_t)r * a.out_row;
#pragma unroll 4
          for (int n1 = 0; n1 < N1; ++n1)
            orow[lane + 32 * n1] = buf[lane + 32 * n1];
        } else if (bin < a.nz) {
          float2 *buf = tbuf + q * RS;
          float2  x[N1];
#pragma unroll
          for (int n1 = 0; n1 < N1; ++n1)
            x[n1] = buf[lane + 32 * n1];
          __syncwarp(); // the row is in registers: its buffer becomes the padded exchange
          four_step_a<N1, false>(x, lane, tw, buf);
          __syncwarp();
          float2 *orow = a.out + (int64_t)w * a.out_win + (int64_t)bin * a.out_plane + (int64_t)r * a.out_row;
          for (int k1 = lane; k1 < N1; k1 += 32) {
            float2 y[32];
            four_step_b<N1, false>(y, k1, buf);
#pragma unroll
            for (int k2 = 0; k2 < 32; ++k2)
              orow[k1 + N1 * k2] = y[k2];
          }
        }
        named_bar(bar, 128);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, NCOL);
  }
}

template <int FMT, int N1> int launch_n1(const BandRowsArgs &a, cudaStream_t s) {
  constexpr int W     = N1 * 32;
  constexpr int NTILE = W / 128;
  constexpr int RS    = XBuf<N1>::kSize > W ? XBuf<N1>::kSize : W;
  const size_t  smem  = 1024 + (size_t)NTILE * kTileBytes + 16384 + (size_t)8 * RS * 8 + (size_t)W * 8 + 128 * 4 +
                      64 * 8 + 2 * 8 + 16 + 8;
  HF_CUDA(cudaFuncSetAttribute(band_rows_tc_kernel<FMT, N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t nrows = (int64_t)a.nwin * a.H;
  const int     cap   = a.max_ctas > 0 ? std::min(a.max_ctas, sm_count()) : sm_count();
  const int     grid  = (int)std::min<int64_t>(nrows, cap);
  HF_CHECK_ARG(a.row_counter != nullptr, "band rows: row counter missing");
  HF_CUDA(cudaMemsetAsync(a.row_counter, 0, sizeof(int), s));
  band_rows_tc_kernel<FMT, N1><<<grid, kBandTcThr, smem, s>>>(a);
  note_launch();
  return launch_status("band_rows_tc_kernel");
}

} // namespace

bool band_rows_tc_supported(int fmt, int T, int W, int nz, int64_t frame_bytes) {
  return (fmt == HF_MONO12P || fmt == HF_U16) && T == 64 && (W == 256 || W == 512 || W == 768 || W == 1024) && nz >= 1 &&
         nz <= 32 && frame_bytes % 16 == 0;
}

int launch_band_rows_tc(const BandRowsArgs &a, int fmt, cudaStream_t s) {
  HF_CHECK_ARG(band_rows_tc_supported(fmt, a.T, a.W, a.nz, a.ring.frame_bytes), "band rows (tensor core): unsupported shape");
  HF_CHECK_ARG(((uintptr_t)a.ring.base & 15) == 0, "band rows (tensor core): ring must be 16-byte aligned");
  switch (a.W) {
  case 256: return fmt == HF_MONO12P ? launch_n1<HF_MONO12P, 8>(a, s) : launch_n1<HF_U16, 8>(a, s);
  case 512: return fmt == HF_MONO12P ? launch_n1<HF_MONO12P, 16>(a, s) : launch_n1<HF_U16, 16>(a, s);
  case 768: return fmt == HF_MONO12P ? launch_n1<HF_MONO12P, 24>(a, s) : launch_n1<HF_U16, 24>(a, s);
  default: return fmt == HF_MONO12P ? launch_n1<HF_MONO12P, 32>(a, s) : launch_n1<HF_U16, 32>(a, s);
  }
}

} // namespace hf
