// Tensor-core (tcgen05) Gram matrix of a window's frames — the chosen form's covariance.
//
// G' = (X - 2048)^T (X - 2048) with X = [T][P] 12-bit samples: (x - 2048) is exact in f16, the
// products are exact in the f32 accumulator, and the shift is undone in float64 by the shared
// finalize kernel (k_pca.cu) from exact integer frame sums.  Per CTA: a ring of 4 shared-memory
// stages of 128 pixels x T frames in the canonical K-major 128-byte-swizzled layout (rows = frames,
// K = pixels).  All threads unpack the next stage while the tensor core consumes the previous ones;
// one thread issues M = N = T, K = 16 MMAs (A and B are the same tile) into a TMEM accumulator and
// commits each stage to its mbarrier, which gates the stage's reuse.
#include <cuda_fp16.h>

#include "k_pca.cuh"
#include "tc_common.cuh"

namespace hf {

namespace {

constexpr int kTcPX     = 128; // pixels per stage (two K-subtiles of 64)
constexpr int kTcStages = 4;

template <int FMT> struct TcBpp;
template <> struct TcBpp<HF_MONO12P> { static constexpr int num = 3, den = 2, words = 3; };
template <> struct TcBpp<HF_U16> { static constexpr int num = 2, den = 1, words = 4; };
template <> struct TcBpp<HF_U8> { static constexpr int num = 1, den = 1, words = 2; };

template <int FMT> __device__ __forceinline__ void unpack_group(const uint32_t *w, uint32_t (&v)[8]) {
  if constexpr (FMT == HF_MONO12P) {
    unpack8(w[0], w[1], w[2], v);
  } else if constexpr (FMT == HF_U16) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      v[2 * i]     = w[i] & 0xFFFFu;
      v[2 * i + 1] = w[i] >> 16;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
        v[4 * i + j] = (w[i] >> (8 * j)) & 0xFFu;
  }
}

template <int FMT, int T>
__global__ void __launch_bounds__(128) cov_tc_kernel(CovArgs a, int *status) {
  constexpr int SUB   = T * 128;       // bytes of one 64-pixel K-subtile (T rows x 128 B)
  constexpr int STAGE = 2 * SUB;       // 128 pixels
  constexpr int NCOL  = T == 64 ? 64 : 128;
  constexpr int TPT   = T * 16 / 128;  // (frame, 8-pixel group) items per thread per stage
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte alignment of the swizzle atoms
  uint8_t  *smem  = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u); // stays a shared-space pointer
  uint64_t *mbar  = reinterpret_cast<uint64_t *>(smem + kTcStages * STAGE);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + kTcStages);
  unsigned long long *ssum = reinterpret_cast<unsigned long long *>(tslot + 2);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int w   = blockIdx.y;
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s)
      tc::mbar_init(&mbar[s], 1);
    tc::mbar_fence_init();
  }
  for (int t = tid; t < T; t += blockDim.x)
    ssum[t] = 0ull;
  if (warp == 0)
    tc::tmem_alloc(tslot, NCOL);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  constexpr uint32_t idesc = tc::idesc_f16(T, T, false, false);

  // this thread's fixed (frame, group) items: t = tid/16 + 8k, g = tid % 16
  const int g = tid & 15;
  uint32_t  isum[TPT];
#pragma unroll
  for (int k = 0; k < TPT; ++k)
    isum[k] = 0u;

  const int64_t ntiles = (a.P + kTcPX - 1) / kTcPX;
  int           nj     = 0;
  bool          ok     = true;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++nj) {
    const int s = nj % kTcStages;
    bool      w_ok = true;
    if (nj >= kTcStages)
      w_ok = tc::mbar_wait_bounded(&mbar[s], (uint32_t)((nj / kTcStages) - 1) & 1u, status, 1);
    ok = __syncthreads_and(w_ok) != 0; // uniform: every thread leaves together on a timeout
    if (!ok)
      break;
    uint8_t      *st = smem + s * STAGE;
    const int64_t p  = tile * kTcPX + g * 8;
    const bool    valid = p < a.P;
#pragma unroll
    for (int k = 0; k < TPT; ++k) {
      const int t = (tid >> 4) + 8 * k;
      uint32_t  v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (valid) {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(a.ring.frame(w, t) +
                                                                 p * TcBpp<FMT>::num / TcBpp<FMT>::den);
        uint32_t wv[TcBpp<FMT>::words];
#pragma unroll
        for (int i = 0; i < TcBpp<FMT>::words; ++i)
          wv[i] = __ldg(src + i);
        unpack_group<FMT>(wv, v);
      }
      __half2 h[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        isum[k] += valid ? v[2 * i] + v[2 * i + 1] : 0u;
        const float x0 = valid ? (float)v[2 * i] - a.shift : 0.f;
        const float x1 = valid ? (float)v[2 * i + 1] - a.shift : 0.f;
        h[i] = __floats2half2_rn(x0, x1);
      }
      const int sub = g >> 3, c = g & 7;
      uint4    *dst = reinterpret_cast<uint4 *>(st + sub * SUB + t * 128 + ((c ^ (t & 7)) << 4));
      *dst = *reinterpret_cast<const uint4 *>(h);
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int sub = 0; sub < 2; ++sub)
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
          const uint64_t d = tc::sw128_desc(tc::smem_u32(st + sub * SUB + ks * 32), 16, 1024);
          tc::mma_f16(tbase, d, d, idesc, (nj > 0 || sub > 0 || ks > 0) ? 1u : 0u);
        }
      tc::mma_commit(&mbar[s]);
    }
  }
  // drain: the last commit covers every MMA issued before it
  if (nj > 0 && ok) {
    const int last = nj - 1;
    ok = tc::mbar_wait_bounded(&mbar[last % kTcStages], (uint32_t)(last / kTcStages) & 1u, status, 2);
  }
  ok = __syncthreads_and(ok) != 0;
  tc::fence_after_sync();
#pragma unroll
  for (int k = 0; k < TPT; ++k)
    atomicAdd(&ssum[(tid >> 4) + 8 * k], (unsigned long long)isum[k]);

  const int64_t pidx = ((int64_t)w * a.nblk + blockIdx.x) * T * T;
  if constexpr (T == 64) {
    // M = 64 accumulator: row m sits in TMEM lane 32*(m/16) + m%16 (the lower half of each
    // 32-lane subpartition), columns 0..63 hold N = 0..63
    uint32_t r0[32], r1[32];
    tc::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16), r0);
    tc::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16) + 32, r1);
    tc::tmem_wait_ld();
    const int i = tid & 31;
    if (i < 16) {
      const int m = 16 * warp + i;
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        a.partial[pidx + m * T + c]      = (nj > 0 && ok) ? __uint_as_float(r0[c]) : 0.f;
        a.partial[pidx + m * T + 32 + c] = (nj > 0 && ok) ? __uint_as_float(r1[c]) : 0.f;
      }
    }
  } else {
    const int m = 32 * warp + (tid & 31);
#pragma unroll
    for (int cb = 0; cb < 4; ++cb) {
      uint32_t r[32];
      tc::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16) + 32 * cb, r);
      tc::tmem_wait_ld();
#pragma unroll
      for (int c = 0; c < 32; ++c)
        a.partial[pidx + m * T + 32 * cb + c] = (nj > 0 && ok) ? __uint_as_float(r[c]) : 0.f;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  for (int t = tid; t < T; t += blockDim.x)
    a.sums[((int64_t)w * gridDim.x + blockIdx.x) * T + t] = (double)ssum[t];
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, NCOL);
  }
}

// ------------------------------------------------------------------------------------------------
// Exact integer variant for samples of at most 12 bits: x - shift = 64 h + l with h in [-32, 31],
// l in [0, 63] (both int8).  The stage holds R = 2T K-major rows [h of every frame; l of every
// frame]; one kind::i8 MMA per 32-pixel K-step and 128-row M-block yields D = [H; L][H; L]^T in
// int32, and G' = 4096 HH + 64 (HL + LH) + LL is folded into a per-window int64 accumulator with
// integer atomics (exact, so the result does not depend on their order).
// ------------------------------------------------------------------------------------------------
template <int FMT, int T>
__global__ void __launch_bounds__(128) cov_tc_i8_kernel(FrameRing ring, int64_t P, float shift,
                                                      unsigned long long *acc, unsigned long long *sums,
                                                      int *status) {
  constexpr int R     = 2 * T;           // operand rows
  constexpr int STAGE = R * 128;         // 128 pixels (int8 K) per row
  constexpr int NMB   = R / 128;         // 128-row M-blocks
  constexpr int NCOL  = NMB * R;         // TMEM columns (int32)
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t  *smem  = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u); // stays a shared-space pointer
  uint64_t *mbar  = reinterpret_cast<uint64_t *>(smem + kTcStages * STAGE);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + kTcStages);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int w   = blockIdx.y;
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s)
      tc::mbar_init(&mbar[s], 1);
    tc::mbar_fence_init();
  }
  if (warp == 0)
    tc::tmem_alloc(tslot, NCOL);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  constexpr uint32_t idesc = tc::idesc_i8(128, R, false, false);

  // items: (frame t, 32-pixel group grp) with t = (tid >> 2) + 32 * k, grp = tid & 3; each item is
  // one 16-byte-aligned run of packed bytes (48 B for 12-bit, 32 B for 8-bit samples)
  constexpr int IPT = T * 4 / 128; // items per thread per stage
  const int grp = tid & 3;
  uint32_t  isum[IPT];
#pragma unroll
  for (int k = 0; k < IPT; ++k)
    isum[k] = 0u;
  const int ishift = (int)shift;
  constexpr int GW = FMT == HF_MONO12P ? 12 : 8; // words per item

  auto load_items = [&](int64_t tile, uint32_t (&raw)[IPT][GW]) {
    const int64_t p = tile * kTcPX + grp * 32;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int t = (tid >> 2) + 32 * k;
      if (tile >= 0 && p < P) {
        const uint4 *src = reinterpret_cast<const uint4 *>(ring.frame(w, t) + p * TcBpp<FMT>::num / TcBpp<FMT>::den);
#pragma unroll
        for (int i = 0; i < GW / 4; ++i) {
          const uint4 v = __ldg(src + i);
          raw[k][4 * i] = v.x, raw[k][4 * i + 1] = v.y, raw[k][4 * i + 2] = v.z, raw[k][4 * i + 3] = v.w;
        }
      }
    }
  };

  const int64_t ntiles = (P + kTcPX - 1) / kTcPX;
  int           nj     = 0;
  bool          ok     = true;
  uint32_t      nxt[IPT][GW];
  load_items(blockIdx.x < ntiles ? (int64_t)blockIdx.x : -1, nxt);
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++nj) {
    const int s = nj % kTcStages;
    uint32_t  cur[IPT][GW];
#pragma unroll
    for (int k = 0; k < IPT; ++k)
#pragma unroll
      for (int i = 0; i < GW; ++i)
        cur[k][i] = nxt[k][i];
    const bool valid = tile * kTcPX + grp * 32 < P;
    if (tile + gridDim.x < ntiles) // prefetch the next tile's samples while this one is staged
      load_items(tile + gridDim.x, nxt);
    bool w_ok = true;
    if (nj >= kTcStages)
      w_ok = tc::mbar_wait_bounded(&mbar[s], (uint32_t)((nj / kTcStages) - 1) & 1u, status, 3);
    ok = __syncthreads_and(w_ok) != 0;
    if (!ok)
      break;
    uint8_t *st = smem + s * STAGE;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int t = (tid >> 2) + 32 * k;
      uint32_t  v[32];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t p8[8];
        if constexpr (FMT == HF_MONO12P) {
          unpack8(cur[k][3 * q], cur[k][3 * q + 1], cur[k][3 * q + 2], p8);
        } else {
#pragma unroll
          for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
              p8[4 * i + j] = (cur[k][2 * q + i] >> (8 * j)) & 0xFFu;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i)
          v[8 * q + i] = valid ? p8[i] : 0u;
      }
      uint32_t hw[8], lw[8];
#pragma unroll
      for (int i = 0; i < 8; ++i)
        hw[i] = lw[i] = 0u;
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        isum[k] += v[i];
        const int d = valid ? (int)v[i] - ishift : 0; // in [-2048, 2047]
        hw[i >> 2] |= (uint32_t)((d >> 6) & 0xFF) << (8 * (i & 3)); // floor(d / 64): [-32, 31]
        lw[i >> 2] |= (uint32_t)(d & 63) << (8 * (i & 3));           // [0, 63]
      }
      // 32 pixels = two 16-byte chunks of a 128-byte row, chunk index 2*grp + {0, 1}
      const int tl = T + t;
#pragma unroll
      for (int hc = 0; hc < 2; ++hc) {
        const int c = 2 * grp + hc;
        *reinterpret_cast<uint4 *>(st + t * 128 + ((c ^ (t & 7)) << 4)) =
            make_uint4(hw[4 * hc], hw[4 * hc + 1], hw[4 * hc + 2], hw[4 * hc + 3]);
        *reinterpret_cast<uint4 *>(st + tl * 128 + ((c ^ (tl & 7)) << 4)) =
            make_uint4(lw[4 * hc], lw[4 * hc + 1], lw[4 * hc + 2], lw[4 * hc + 3]);
      }
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const uint64_t bdesc = tc::sw128_desc(tc::smem_u32(st + ks * 32), 16, 1024);
#pragma unroll
        for (int mb = 0; mb < NMB; ++mb) {
          const uint64_t adesc = tc::sw128_desc(tc::smem_u32(st + mb * 128 * 128 + ks * 32), 16, 1024);
          tc::mma_i8(tbase + mb * R, adesc, bdesc, idesc, (nj > 0 || ks > 0) ? 1u : 0u);
        }
      }
      tc::mma_commit(&mbar[s]);
    }
  }
  if (nj > 0 && ok) {
    const int last = nj - 1;
    ok = tc::mbar_wait_bounded(&mbar[last % kTcStages], (uint32_t)(last / kTcStages) & 1u, status, 4);
  }
  ok = __syncthreads_and(ok) != 0;
  tc::fence_after_sync();
#pragma unroll
  for (int k = 0; k < IPT; ++k)
    atomicAdd(&sums[(int64_t)w * T + (tid >> 2) + 32 * k], (unsigned long long)isum[k]);
  if (nj > 0 && ok) {
    unsigned long long *aw = acc + (int64_t)w * T * T;
#pragma unroll
    for (int mb = 0; mb < NMB; ++mb) {
      const int row = mb * 128 + 32 * warp + (tid & 31); // operand row held by this thread
      const bool is_h = row < T;
      const int  a    = is_h ? row : row - T;
      // this row's contribution to G'[a][b]: h-row -> 4096 HH + 64 HL, l-row -> 64 LH + LL
      const long long wa = is_h ? 4096 : 64, wb = is_h ? 64 : 1;
#pragma unroll
      for (int cb = 0; cb < T / 32; ++cb) {
        uint32_t r0[32], r1[32];
        tc::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16) + mb * R + 32 * cb, r0);
        tc::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16) + mb * R + T + 32 * cb, r1);
        tc::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const long long v = wa * (long long)(int)r0[c] + wb * (long long)(int)r1[c];
          atomicAdd(&aw[a * T + 32 * cb + c], (unsigned long long)v);
        }
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

// ------------------------------------------------------------------------------------------------
// Shared-frame variant for T = 64 and a hop that is a multiple of 8 (8..32): a CTA owns a group of
// up to four consecutive windows, i.e. the frames w0*hop + [0, F) with F = 64 + 3 hop, and stages
// every frame of the group once per 128-pixel tile instead of once per window.
//  - Operand rows come in 8-frame pairs of swizzle atoms, [h of frames 8p..8p+7][l of the same
//    frames], so window wl's 128 operand rows [h;l] are the 16 consecutive atoms from pair
//    wl*hop/8: one descriptor offset selects them, and its M = N = 128 kind::i8 MMAs accumulate
//    D_wl into its own 128 TMEM columns (512 columns for four windows, one CTA per SM).
//  - Packed samples travel global -> shared through a ring of per-thread cp.async copies, D tiles
//    deep; each thread unpacks exactly the bytes it copied, so no barrier guards the raw ring.
//  - The split needs no pixel value: for x in [0, 4096), x - 2048 = 64 ((x >> 6) - 32) + (x & 63),
//    so the 6-bit fields of the packed stream are masked out in 16-bit lanes, packed to bytes with
//    byte permutes and re-centred with one byte-wise subtraction; frame sums are 64 S(x >> 6) +
//    S(x & 63) from byte dot products.  8-bit samples use x - 128 = 64 ((x >> 6) - 2) + (x & 63).
// Operand row r of a window holds frame 8 (r / 16) + r % 8, kind h when (r / 8) is even; the h-row
// and l-row of a frame sit 8 lanes apart in one warp and are folded with a shuffle before the
// integer atomics.
// Warp roles: the producer warps fill the stages and arrive (one arrival per warp) on the stage's
// `full` barrier; the last warp waits on it, issues the stage's MMAs and commits them to the
// stage's `free` barrier, so no producer waits for the others between tiles.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tc::smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// 24 packed bits (two 12-bit pixels p0 | p1 << 12) -> 16-bit lanes of their low and high 6 bits
__device__ __forceinline__ void split_pair12(uint32_t t, uint32_t &lo, uint32_t &hi) {
  lo = (t & 0x3Fu) | ((t << 4) & 0x003F0000u);
  hi = ((t >> 6) & 0x3Fu) | ((t >> 2) & 0x003F0000u);
}

template <int FMT, int HOP8> struct GroupCov {
  static constexpr int F    = 64 + 24 * HOP8;              // frames of a four-window group
  static constexpr int NT   = 4 * F;                       // one (frame, 32-pixel run) per thread
  static constexpr int RB   = FMT == HF_MONO12P ? 48 : 32; // packed bytes of a 32-pixel run
  static constexpr int D    = F <= 112 ? 4 : 3;            // raw ring depth (tiles)
  static constexpr int S    = F <= 136 ? 3 : 2;            // operand stages
  static constexpr int STG  = 256 * F;                     // 2F rows x 128 B
  static constexpr int NTHR = NT + 32;                     // producers + the MMA warp
  static constexpr size_t smem = 1024 + (size_t)S * STG + (size_t)D * NT * RB + 2 * S * 8 + 16;
};

// Bounded mbarrier wait that also gives up once another thread has raised `abort`; the first
// thread to time out records `code` in the status word and raises it.
__device__ __forceinline__ bool wait_or_abort(uint64_t *mbar, uint32_t parity, volatile int *abort, int *status,
                                              int code) {
  const uint64_t t0 = tc::globaltimer_ns();
  for (uint32_t i = 0; i < tc::kWaitLimit; ++i) {
    if (tc::mbar_try_wait(mbar, parity))
      return true;
    if ((i & 255u) == 255u && (*abort || tc::globaltimer_ns() - t0 > tc::kWaitNs))
      break;
  }
  if (!*abort && status)
    atomicCAS(status, 0, code);
  *abort = 1;
  return false;
}

template <int FMT, int HOP8>
__global__ void __launch_bounds__(GroupCov<FMT, HOP8>::NTHR, 1)
    cov_tc_group_kernel(FrameRing ring, int64_t P, int nwin, uint32_t ncols, unsigned long long *acc,
                        unsigned long long *sums, int *status) {
  using G                = GroupCov<FMT, HOP8>;
  constexpr int T        = 64;
  constexpr int HOP      = 8 * HOP8;
  constexpr uint32_t kHS = FMT == HF_MONO12P ? 0x20202020u : 0x02020202u; // shift / 64 per byte
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t  *smem  = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u); // stays a shared-space pointer
  uint8_t  *raw   = smem + G::S * G::STG;
  uint64_t *mbar  = reinterpret_cast<uint64_t *>(raw + (size_t)G::D * G::NT * G::RB); // [S] free
  uint64_t *fullb = mbar + G::S;                                                        // [S] full
  uint32_t *tslot = reinterpret_cast<uint32_t *>(fullb + G::S);
  int      *abort_flag = reinterpret_cast<int *>(tslot + 1);
  volatile int *abortv = abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int w0  = 4 * blockIdx.y;
  const int g   = min(4, nwin - w0);   // windows of this group
  const int Fg  = T + (g - 1) * HOP;   // frames of this group
  const bool producer = tid < G::NT;   // the last warp issues the MMAs
  if (tid == 0) {
    for (int s = 0; s < G::S; ++s) {
      tc::mbar_init(&mbar[s], 1);              // the MMA commit of the stage's tile
      tc::mbar_init(&fullb[s], G::NT / 32);    // one arrival per producer warp
    }
    *abort_flag = 0;
    tc::mbar_fence_init();
  }
  if (warp == 0)
    tc::tmem_alloc(tslot, ncols);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *tslot;
  constexpr uint32_t idesc = tc::idesc_i8(128, 128, false, false);

  const int      f      = tid >> 2, grp = tid & 3;
  const bool     active = f < Fg;
  const uint8_t *fbase  = active ? ring.frame(w0, f) : nullptr;
  uint8_t       *myraw  = raw + (size_t)tid * G::RB;
  // this thread's rows in the stage: frame f -> pair f / 8, row f % 8 of the pair's h and l atoms
  const int rr = f & 7, pr = f >> 3;

  const int64_t ntiles = (P + kTcPX - 1) / kTcPX;
  auto issue = [&](int64_t tile, int slot) {
    const int64_t p = tile * kTcPX + grp * 32;
    if (active && tile < ntiles && p < P) {
      const uint8_t *src = fbase + p * TcBpp<FMT>::num / TcBpp<FMT>::den;
      uint8_t       *dst = myraw + (size_t)slot * G::NT * G::RB;
#pragma unroll
      for (int i = 0; i < G::RB / 16; ++i)
        cp_async16(dst + 16 * i, src + 16 * i);
    }
    cp_async_commit();
  };
  uint32_t sx = 0u, sl = 0u; // sums of the high and low 6-bit fields
  int      nj = 0;
  bool     ok = true;
  if (producer) {
#pragma unroll
  for (int d = 0; d < G::D - 1; ++d)
    issue(blockIdx.x + (int64_t)d * gridDim.x, d);
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++nj) {
    const int s = nj % G::S;
    issue(tile + (int64_t)(G::D - 1) * gridDim.x, (nj + G::D - 1) % G::D);
    bool w_ok = true;
    if (nj >= G::S) // the MMAs that read this stage S tiles ago are done
      w_ok = wait_or_abort(&mbar[s], (uint32_t)((nj / G::S) - 1) & 1u, abortv, status, 5);
    cp_async_wait<G::D - 1>();
    const bool valid = active && tile * kTcPX + grp * 32 < P;
    if (w_ok && active) {
      uint32_t hw[8], lw[8];
      if (valid) {
        const uint4 *src = reinterpret_cast<const uint4 *>(myraw + (size_t)(nj % G::D) * G::NT * G::RB);
        uint32_t     wv[G::RB / 4];
#pragma unroll
        for (int i = 0; i < G::RB / 16; ++i) {
          const uint4 v = src[i];
          wv[4 * i] = v.x, wv[4 * i + 1] = v.y, wv[4 * i + 2] = v.z, wv[4 * i + 3] = v.w;
        }
        if constexpr (FMT == HF_MONO12P) {
#pragma unroll
          for (int q = 0; q < 4; ++q) { // 8 pixels from 3 words
            const uint32_t a0 = wv[3 * q], a1 = wv[3 * q + 1], a2 = wv[3 * q + 2];
            uint32_t       l0, h0, l1, h1, l2, h2, l3, h3;
            split_pair12(a0, l0, h0);
            split_pair12(__funnelshift_r(a0, a1, 24), l1, h1);
            split_pair12(__funnelshift_r(a1, a2, 16), l2, h2);
            split_pair12(a2 >> 8, l3, h3);
            lw[2 * q]     = __byte_perm(l0, l1, 0x6420);
            lw[2 * q + 1] = __byte_perm(l2, l3, 0x6420);
            hw[2 * q]     = __byte_perm(h0, h1, 0x6420);
            hw[2 * q + 1] = __byte_perm(h2, h3, 0x6420);
          }
        } else {
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            lw[i] = wv[i] & 0x3F3F3F3Fu;
            hw[i] = (wv[i] >> 6) & 0x03030303u;
          }
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          sx    = __dp4a(hw[i], 0x01010101u, sx);
          sl    = __dp4a(lw[i], 0x01010101u, sl);
          hw[i] = __vsub4(hw[i], kHS);
        }
      } else {
#pragma unroll
        for (int i = 0; i < 8; ++i)
          hw[i] = lw[i] = 0u;
      }
      uint8_t *hrow = smem + s * G::STG + pr * 2048 + rr * 128;
#pragma unroll
      for (int hc = 0; hc < 2; ++hc) {
        const int c = 2 * grp + hc;
        *reinterpret_cast<uint4 *>(hrow + ((c ^ rr) << 4)) =
            make_uint4(hw[4 * hc], hw[4 * hc + 1], hw[4 * hc + 2], hw[4 * hc + 3]);
        *reinterpret_cast<uint4 *>(hrow + 1024 + ((c ^ rr) << 4)) =
            make_uint4(lw[4 * hc], lw[4 * hc + 1], lw[4 * hc + 2], lw[4 * hc + 3]);
      }
    }
    tc::fence_proxy_async_smem(); // this thread's stage writes before the async proxy reads them
    __syncwarp();
    if (lane == 0)
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(&fullb[s])) : "memory");
    if (!w_ok || *abortv) {
      ok = false;
      break;
    }
  }
  cp_async_wait<0>(); // no copy may land in shared memory after the CTA has left
  } else {
    // MMA warp: issue each stage's MMAs as soon as every producer warp has filled it
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++nj) {
      const int s = nj % G::S;
      if (!wait_or_abort(&fullb[s], (uint32_t)(nj / G::S) & 1u, abortv, status, 7)) {
        ok = false;
        break;
      }
      if (lane == 0) {
        tc::fence_after_sync();
        const uint8_t *st = smem + s * G::STG;
        for (int wl = 0; wl < g; ++wl) {
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            const uint64_t d = tc::sw128_desc(tc::smem_u32(st + wl * HOP8 * 2048 + ks * 32), 16, 1024);
            tc::mma_i8(tbase + 128 * wl, d, d, idesc, (nj > 0 || ks > 0) ? 1u : 0u);
          }
        }
        tc::mma_commit(&mbar[s]);
      }
      __syncwarp();
    }
    if (nj > 0 && ok) { // drain: the last commit covers every MMA issued before it
      const int last = nj - 1;
      ok = wait_or_abort(&mbar[last % G::S], (uint32_t)(last / G::S) & 1u, abortv, status, 6);
    }
  }
  ok = __syncthreads_and(ok && !*abortv) != 0;
  tc::fence_after_sync();

  // frame sums: the four runs of a frame are adjacent lanes; each window holding frame f gets it
  unsigned long long fs = 64ull * sx + sl;
  fs += __shfl_xor_sync(0xFFFFFFFFu, fs, 1);
  fs += __shfl_xor_sync(0xFFFFFFFFu, fs, 2);
  if (producer && active && grp == 0)
    for (int wl = 0; wl < g; ++wl) {
      const int t = f - wl * HOP;
      if (t >= 0 && t < T)
        atomicAdd(&sums[(int64_t)(w0 + wl) * T + t], fs);
    }

  constexpr int NQ = G::NT / 128; // complete warp quads: each reads all 128 TMEM lanes
  if (nj > 0 && ok && warp < 4 * NQ) {
    const int       q      = warp & 3;
    const int       r      = 32 * q + lane;
    const bool      is_h   = ((r >> 3) & 1) == 0;
    const int       a      = 8 * (r >> 4) + (r & 7);
    const long long wh     = is_h ? 4096 : 64, wlw = is_h ? 64 : 1;
    for (int wl = warp >> 2; wl < g; wl += NQ) {
      unsigned long long *aw = acc + (int64_t)(w0 + wl) * T * T + a * T;
#pragma unroll
      for (int cb = 0; cb < 4; ++cb) {
        uint32_t v[32];
        tc::tmem_ld32(tbase + ((uint32_t)(32 * q) << 16) + 128 * wl + 32 * cb, v);
        tc::tmem_wait_ld();
#pragma unroll
        for (int half = 0; half < 2; ++half)
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            // columns 16 half + c (h of frame b) and 16 half + 8 + c (l of frame b)
            long long e = wh * (long long)(int)v[16 * half + c] + wlw * (long long)(int)v[16 * half + 8 + c];
            e += __shfl_xor_sync(0xFFFFFFFFu, e, 8);
            if (is_h)
              atomicAdd(&aw[16 * cb + 8 * half + c], (unsigned long long)e);
          }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, ncols);
  }
}

// int64 accumulator -> float64 Gram with the shift undone exactly.
__global__ void cov_i8_finalize_kernel(const unsigned long long *acc, const unsigned long long *sums, int T,
                                       int64_t P, long long shift, double *gram) {
  const int w = blockIdx.y;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= T * T)
    return;
  const int       i = e / T, j = e % T;
  const long long g = (long long)acc[(int64_t)w * T * T + e] +
                      shift * (long long)(sums[(int64_t)w * T + i] + sums[(int64_t)w * T + j]) -
                      shift * shift * (long long)P;
  gram[(int64_t)w * T * T + e] = (double)g;
}

int launch_i8_finalize(const unsigned long long *acc, const unsigned long long *sums, int T, int64_t P,
                       long long shift, int nwin, double *gram, cudaStream_t s) {
  cov_i8_finalize_kernel<<<dim3((T * T + 255) / 256, nwin), 256, 0, s>>>(acc, sums, T, P, shift, gram);
  note_launch();
  return launch_status("cov_i8_finalize_kernel");
}

template <int FMT, int T>
int launch_tc(const FrameRing &ring, int64_t P, int nwin, void *ws, double *gram, int *status,
              cudaStream_t s) {
  const size_t smem = 1024 + (size_t)kTcStages * 2 * T * 128 + kTcStages * 8 + 8 + T * 8;
  const int64_t ntiles = (P + kTcPX - 1) / kTcPX;
  const int ctas = (int)std::max<int64_t>(1, std::min<int64_t>(3LL * sm_count() / nwin, ntiles));
  CovArgs a;
  a.ring    = ring;
  a.T       = T;
  a.P       = P;
  a.shift   = FMT == HF_U8 ? 128.f : 2048.f;
  a.nblk    = ctas;
  a.partial = reinterpret_cast<float *>(ws);
  a.sums    = reinterpret_cast<double *>(reinterpret_cast<uint8_t *>(ws) +
                                      (size_t)nwin * ctas * T * T * sizeof(float));
  HF_CUDA(cudaFuncSetAttribute(cov_tc_kernel<FMT, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cov_tc_kernel<FMT, T><<<dim3(ctas, nwin), 128, smem, s>>>(a, status);
  note_launch();
  HF_TRY(launch_status("cov_tc_kernel"));
  return launch_cov_finalize(a.partial, a.sums, a.nblk, ctas, T, P, (double)a.shift, gram, nwin, s);
}

template <int FMT, int T>
int launch_tc_i8(const FrameRing &ring, int64_t P, int nwin, void *ws, double *gram, int *status,
                 cudaStream_t s) {
  constexpr int R    = 2 * T;
  const size_t  smem = 1024 + (size_t)kTcStages * R * 128 + kTcStages * 8 + 8;
  const int64_t ntiles = (P + kTcPX - 1) / kTcPX;
  // at most ~256K pixels per CTA keeps every int32 accumulator entry below 63*63*256K < 2^31
  const int64_t min_ctas = (P + (1 << 18) - 1) >> 18;
  const int     per_sm   = T == 64 ? 3 : 1;
  // one wave: the CTAs of all windows fit the SMs at once (a partial second wave doubles the time)
  const int ctas = (int)std::max<int64_t>(
      min_ctas, std::min<int64_t>(std::max<int64_t>(1, (int64_t)per_sm * sm_count() / nwin), ntiles));
  auto *acc  = reinterpret_cast<unsigned long long *>(ws);
  auto *sums = acc + (size_t)nwin * T * T;
  HF_CUDA(cudaMemsetAsync(acc, 0, ((size_t)nwin * T * T + (size_t)nwin * T) * sizeof(unsigned long long), s));
  HF_CUDA(cudaFuncSetAttribute(cov_tc_i8_kernel<FMT, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cov_tc_i8_kernel<FMT, T><<<dim3(ctas, nwin), 128, smem, s>>>(ring, P, FMT == HF_U8 ? 128.f : 2048.f, acc, sums,
                                                               status);
  note_launch();
  HF_TRY(launch_status("cov_tc_i8_kernel"));
  return launch_i8_finalize(acc, sums, T, P, FMT == HF_U8 ? 128 : 2048, nwin, gram, s);
}

template <int FMT, int HOP8>
int launch_tc_group(const FrameRing &ring, int64_t P, int nwin, void *ws, double *gram, int *status,
                    cudaStream_t s) {
  using G               = GroupCov<FMT, HOP8>;
  constexpr int T       = 64;
  const int     ngroups = (nwin + 3) / 4;
  const int64_t ntiles  = (P + kTcPX - 1) / kTcPX;
  const int64_t min_ctas = (P + (1 << 18) - 1) >> 18; // int32 accumulator bound, as above
  // one CTA per SM (it holds the whole TMEM), the SMs split evenly between the window groups
  const int ctas = (int)std::max<int64_t>(
      min_ctas, std::min<int64_t>(std::max<int64_t>(1, (int64_t)sm_count() / ngroups), ntiles));
  const uint32_t ncols = nwin >= 3 ? 512u : 256u;
  auto *acc  = reinterpret_cast<unsigned long long *>(ws);
  auto *sums = acc + (size_t)nwin * T * T;
  HF_CUDA(cudaMemsetAsync(acc, 0, ((size_t)nwin * T * T + (size_t)nwin * T) * sizeof(unsigned long long), s));
  HF_CUDA(cudaFuncSetAttribute(cov_tc_group_kernel<FMT, HOP8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)G::smem));
  cov_tc_group_kernel<FMT, HOP8><<<dim3(ctas, ngroups), G::NTHR, G::smem, s>>>(ring, P, nwin, ncols, acc, sums,
                                                                                status);
  note_launch();
  HF_TRY(launch_status("cov_tc_group_kernel"));
  return launch_i8_finalize(acc, sums, T, P, FMT == HF_U8 ? 128 : 2048, nwin, gram, s);
}

template <int FMT>
int launch_group_hop(const FrameRing &ring, int64_t P, int nwin, void *ws, double *gram, int *status,
                     cudaStream_t s) {
  switch (ring.hop / 8) {
  case 1: return launch_tc_group<FMT, 1>(ring, P, nwin, ws, gram, status, s);
  case 2: return launch_tc_group<FMT, 2>(ring, P, nwin, ws, gram, status, s);
  case 3: return launch_tc_group<FMT, 3>(ring, P, nwin, ws, gram, status, s);
  default: return launch_tc_group<FMT, 4>(ring, P, nwin, ws, gram, status, s);
  }
}

} // namespace

size_t cov_tc_workspace_bytes(int T, int64_t P, int nwin) {
  const int64_t ntiles = (P + kTcPX - 1) / kTcPX;
  const int64_t ctas   = std::max<int64_t>(1, std::min<int64_t>((3LL * sm_count() + nwin - 1) / nwin, ntiles));
  const size_t f16 = (size_t)(nwin * ctas) * T * T * sizeof(float) + (size_t)(nwin * ctas) * T * sizeof(double) + 256;
  const size_t i8  = ((size_t)nwin * T * T + (size_t)nwin * T) * sizeof(unsigned long long) + 256;
  return std::max(f16, i8);
}

bool cov_tc_supported(int fmt, int T, int64_t P, int64_t frame_bytes) {
  if (fmt == HF_MONO12P || fmt == HF_U8) // 16-byte loads of 32-pixel runs
    return (T == 64 || T == 128) && P % 32 == 0 && frame_bytes % 16 == 0;
  return fmt == HF_U16 && (T == 64 || T == 128) && P % 8 == 0 && frame_bytes % 4 == 0;
}

int launch_covariance_tc(const FrameRing &ring, int fmt, int T, int64_t P, int nwin, void *ws,
                         double *gram, int *status, cudaStream_t s) {
  HF_CHECK_ARG(cov_tc_supported(fmt, T, P, ring.frame_bytes), "tensor-core covariance: unsupported shape");
  // overlapping 64-frame windows on an 8-frame grid: stage each frame once per window group
  if ((fmt == HF_MONO12P || fmt == HF_U8) && T == 64 && nwin >= 2 && ring.hop >= 8 && ring.hop <= 32 &&
      ring.hop % 8 == 0)
    return fmt == HF_MONO12P ? launch_group_hop<HF_MONO12P>(ring, P, nwin, ws, gram, status, s)
                             : launch_group_hop<HF_U8>(ring, P, nwin, ws, gram, status, s);
  // samples of at most 12 bits: exact int8 split; 16-bit samples: f16 operands
  if (fmt == HF_MONO12P)
    return T == 64 ? launch_tc_i8<HF_MONO12P, 64>(ring, P, nwin, ws, gram, status, s)
                   : launch_tc_i8<HF_MONO12P, 128>(ring, P, nwin, ws, gram, status, s);
  if (fmt == HF_U8)
    return T == 64 ? launch_tc_i8<HF_U8, 64>(ring, P, nwin, ws, gram, status, s)
                   : launch_tc_i8<HF_U8, 128>(ring, P, nwin, ws, gram, status, s);
  if (T == 64) {
    if (fmt == HF_MONO12P) return launch_tc<HF_MONO12P, 64>(ring, P, nwin, ws, gram, status, s);
    if (fmt == HF_U16) return launch_tc<HF_U16, 64>(ring, P, nwin, ws, gram, status, s);
    return launch_tc<HF_U8, 64>(ring, P, nwin, ws, gram, status, s);
  }
  if (fmt == HF_MONO12P) return launch_tc<HF_MONO12P, 128>(ring, P, nwin, ws, gram, status, s);
  if (fmt == HF_U16) return launch_tc<HF_U16, 128>(ring, P, nwin, ws, gram, status, s);
  return launch_tc<HF_U8, 128>(ring, P, nwin, ws, gram, status, s);
}

} // namespace hf
