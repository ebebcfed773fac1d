// Temporal band DFT: per pixel S_k = scale * sum_t x_t W[t][k] for k < nz, written as complex
// planes [nz][OH][OW] (optionally multiplied by a per-pixel lens and placed at an offset inside
// a larger zero-padded plane).
//
// W is the T x nz complex matrix a window's SVD clutter filter and its band DFT reduce to,
// W = (I - V V^T) D[:, z0:z1]  (D the unnormalised DFT, V the removed eigenvectors), so this one
// kernel stands for RFFT/FFT along T + Slice + Copy (holonp/src/rfft.cu:150-160,
// fft.cu:234-252, graph_builder.cc:264-267) and for the filter, and Fresnel's lens multiply
// (the load callback of fresnel_diffraction.cu:262-303) is fused into its store.
//
// Plain form: FP32 CUDA-core FMAs.  A CTA stages the packed samples of a 1024-pixel tile for all
// T frames in shared memory once, then each thread accumulates 7 bins x 8 pixels in registers.
#include "frames.cuh"
#include "k_band.cuh"

namespace hf {

namespace {

constexpr int kBandNB  = 7;   // bins per thread
constexpr int kBandPX  = 8;   // pixels per thread
constexpr int kBandHalf = 2;  // bin chunks processed side by side by the two halves of a CTA

template <int FMT> struct FmtBytes;
template <> struct FmtBytes<HF_MONO12P> { static constexpr int num = 3, den = 2; };
template <> struct FmtBytes<HF_U16> { static constexpr int num = 2, den = 1; };
template <> struct FmtBytes<HF_U8> { static constexpr int num = 1, den = 1; };
template <> struct FmtBytes<HF_F32> { static constexpr int num = 4, den = 1; };

// 8 consecutive samples of one frame from the staged tile (words, 4-byte aligned)
template <int FMT>
__device__ __forceinline__ void load8(const uint32_t *row, int g, float (&x)[kBandPX]) {
  if constexpr (FMT == HF_MONO12P) {
    uint32_t p[8];
    unpack8(row[3 * g], row[3 * g + 1], row[3 * g + 2], p);
#pragma unroll
    for (int i = 0; i < 8; ++i)
      x[i] = (float)p[i];
  } else if constexpr (FMT == HF_U16) {
    const uint4 v = reinterpret_cast<const uint4 *>(row)[g];
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      x[2 * i]     = (float)(w[i] & 0xFFFFu);
      x[2 * i + 1] = (float)(w[i] >> 16);
    }
  } else if constexpr (FMT == HF_U8) {
    const uint2 v = reinterpret_cast<const uint2 *>(row)[g];
    const uint32_t w[2] = {v.x, v.y};
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
        x[4 * i + j] = (float)((w[i] >> (8 * j)) & 0xFFu);
  } else { // F32
    const float4 a = reinterpret_cast<const float4 *>(row)[2 * g];
    const float4 b = reinterpret_cast<const float4 *>(row)[2 * g + 1];
    x[0] = a.x, x[1] = a.y, x[2] = a.z, x[3] = a.w;
    x[4] = b.x, x[5] = b.y, x[6] = b.z, x[7] = b.w;
  }
}

// Entry (t, k) of window w's matrix: the supplied W, or the DFT bin exp(-2 pi i t (z0+k) / T).
__device__ __forceinline__ float2 wmat_entry(const BandArgs &a, int w, int t, int k) {
  if (a.wmat != nullptr)
    return a.wmat[(int64_t)w * a.wmat_stride + (int64_t)t * a.nz + k];
  const int m = (int)(((int64_t)t * (a.z0 + k)) % a.T);
  float     s, c;
  sincospif(-2.0f * (float)m / (float)a.T, &s, &c);
  return make_float2(c, s);
}

template <int FMT>
__global__ void __launch_bounds__(256) band_dft_tiled_kernel(BandArgs a, int tile_px) {
  extern __shared__ __align__(16) uint8_t smem[];
  constexpr int num = FmtBytes<FMT>::num, den = FmtBytes<FMT>::den;
  const int     w         = blockIdx.y;
  const int64_t tile0     = (int64_t)blockIdx.x * tile_px;
  const int     row_bytes = tile_px * num / den;
  const int     row_words = row_bytes / 4;
  const int     groups    = tile_px / kBandPX; // threads per bin chunk
  const int     nzpad     = ((a.nz + kBandNB * kBandHalf - 1) / (kBandNB * kBandHalf)) * kBandNB * kBandHalf;

  uint32_t *tile  = reinterpret_cast<uint32_t *>(smem);
  float2   *w_sh  = reinterpret_cast<float2 *>(smem + (size_t)a.T * row_bytes);
  float2   *lens  = w_sh + (size_t)a.T * nzpad;

  const int tid = threadIdx.x;
  // stage the packed tile of every frame (4-byte words, coalesced per frame)
  const int64_t tile_byte0 = tile0 * num / den;
  const int64_t valid_px   = min((int64_t)tile_px, a.P - tile0);
  const int     valid_words = (int)(valid_px * num / den + 3) / 4;
  // asynchronous 4-byte copies: every frame's words are in flight at once instead of one
  // load-then-store at a time (the tail beyond the image is zero-filled, src-size 0)
  for (int t = 0; t < a.T; ++t) {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(a.ring.frame(w, t) + tile_byte0);
    for (int i = tid; i < row_words; i += blockDim.x) {
      const bool     ok  = i < valid_words;
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared(tile + t * row_words + i);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(ok ? src + i : src),
                   "r"(ok ? 4 : 0)
                   : "memory");
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  for (int i = tid; i < a.T * nzpad; i += blockDim.x) {
    const int t = i / nzpad, k = i % nzpad;
    w_sh[i]     = k < a.nz ? wmat_entry(a, w, t, k) : make_float2(0.f, 0.f);
  }
  if (a.lens != nullptr)
    for (int i = tid; i < tile_px; i += blockDim.x)
      lens[i] = (tile0 + i < a.P) ? a.lens[tile0 + i] : make_float2(1.f, 0.f);
  __syncthreads();

  const int g    = tid % groups;
  const int half = tid / groups;
  const int64_t p0 = tile0 + (int64_t)g * kBandPX;
  const bool active = half < kBandHalf && p0 < a.P;
  const int r = (int)(p0 / a.W), c = (int)(p0 % a.W);
  float2 *outw = a.out + (int64_t)w * a.out_win + (int64_t)(r + a.oy) * a.OW + (c + a.ox);

  for (int kc = half * kBandNB; kc < a.nz; kc += kBandNB * kBandHalf) {
    float2 acc[kBandNB][kBandPX];
#pragma unroll
    for (int b = 0; b < kBandNB; ++b)
#pragma unroll
      for (int p = 0; p < kBandPX; ++p)
        acc[b][p] = make_float2(0.f, 0.f);
    if (active) {
#pragma unroll 2
      for (int t = 0; t < a.T; ++t) {
        float x[kBandPX];
        load8<FMT>(tile + t * row_words, g, x);
        const float2 *wr = w_sh + t * nzpad + kc;
#pragma unroll
        for (int b = 0; b < kBandNB; ++b) {
          const float2 wv = wr[b];
#pragma unroll
          for (int p = 0; p < kBandPX; ++p) {
            acc[b][p].x = fmaf(x[p], wv.x, acc[b][p].x);
            acc[b][p].y = fmaf(x[p], wv.y, acc[b][p].y);
          }
        }
      }
#pragma unroll
      for (int b = 0; b < kBandNB; ++b) {
        const int k = kc + b;
        if (k < a.nz) {
          float4 *dst = reinterpret_cast<float4 *>(outw + (int64_t)k * a.out_plane);
#pragma unroll
          for (int p = 0; p < kBandPX; p += 2) {
            float2 v0 = cscale(acc[b][p], a.scale), v1 = cscale(acc[b][p + 1], a.scale);
            if (a.lens != nullptr) {
              v0 = cmul(v0, lens[g * kBandPX + p]);
              v1 = cmul(v1, lens[g * kBandPX + p + 1]);
            }
            dst[p / 2] = make_float4(v0.x, v0.y, v1.x, v1.y);
          }
        }
      }
    }
  }
}

// One thread per pixel; any format (complex frames included), any P.
template <int FMT> __global__ void band_dft_simple_kernel(BandArgs a) {
  const int     w = blockIdx.y;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.P)
    return;
  const int r = (int)(p / a.W), c = (int)(p % a.W);
  float2 *outp = a.out + (int64_t)w * a.out_win + (int64_t)(r + a.oy) * a.OW + (c + a.ox);
  const float2 L = a.lens ? a.lens[p] : make_float2(1.f, 0.f);
  for (int k0 = 0; k0 < a.nz; k0 += 8) {
    float2 acc[8];
#pragma unroll
    for (int b = 0; b < 8; ++b)
      acc[b] = make_float2(0.f, 0.f);
    for (int t = 0; t < a.T; ++t) {
      const uint8_t *fr = a.ring.frame(w, t);
      float2 x;
      if constexpr (FMT == HF_CF32)
        x = reinterpret_cast<const float2 *>(fr)[p];
      else
        x = make_float2(sample<FMT>(fr, p), 0.f);
#pragma unroll
      for (int b = 0; b < 8; ++b)
        if (k0 + b < a.nz)
          acc[b] = cadd(acc[b], cmul(x, wmat_entry(a, w, t, k0 + b)));
    }
#pragma unroll
    for (int b = 0; b < 8; ++b)
      if (k0 + b < a.nz) {
        float2 v = cscale(acc[b], a.scale);
        if (a.lens)
          v = cmul(v, L);
        outp[(int64_t)(k0 + b) * a.out_plane] = v;
      }
  }
}

template <int FMT> size_t tiled_smem(const BandArgs &a, int tile_px) {
  const int nzpad = ((a.nz + kBandNB * kBandHalf - 1) / (kBandNB * kBandHalf)) * kBandNB * kBandHalf;
  return (size_t)a.T * (tile_px * FmtBytes<FMT>::num / FmtBytes<FMT>::den) +
         (size_t)a.T * nzpad * sizeof(float2) + (size_t)tile_px * sizeof(float2);
}

template <int FMT> int launch_tiled(const BandArgs &a, int nwin, cudaStream_t s) {
  int tile_px = 1024;
  while (tile_px > 128 && tiled_smem<FMT>(a, tile_px) > 110 * 1024)
    tile_px /= 2;
  const size_t smem = tiled_smem<FMT>(a, tile_px);
  if (smem > 200 * 1024)
    return HF_ERR_UNSUPPORTED;
  HF_CUDA(cudaFuncSetAttribute(band_dft_tiled_kernel<FMT>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((unsigned)((a.P + tile_px - 1) / tile_px), nwin);
  const int threads = (tile_px / kBandPX) * kBandHalf;
  band_dft_tiled_kernel<FMT><<<grid, threads, smem, s>>>(a, tile_px);
  note_launch();
  return launch_status("band_dft_tiled_kernel");
}

template <int FMT> int launch_simple(const BandArgs &a, int nwin, cudaStream_t s) {
  dim3 grid((unsigned)((a.P + 127) / 128), nwin);
  band_dft_simple_kernel<FMT><<<grid, 128, 0, s>>>(a);
  note_launch();
  return launch_status("band_dft_simple_kernel");
}

} // namespace

int launch_band_dft(const BandArgs &a, int fmt, int nwin, cudaStream_t s) {
  HF_CHECK_ARG(a.T > 0 && a.P > 0 && a.nz > 0 && nwin > 0, "band_dft: empty problem");
  const bool tiled_ok = (a.P % kBandPX == 0) && (a.W % kBandPX == 0) && ((a.OW * 8) % 16 == 0) &&
                        (a.ox % 2 == 0) && (a.ring.frame_bytes % 4 == 0) &&
                        (((uintptr_t)a.ring.base & 3) == 0); // 4-byte cp.async copies of frame words
  if (tiled_ok) {
    int rc = HF_ERR_UNSUPPORTED;
    switch (fmt) {
    case HF_MONO12P: rc = launch_tiled<HF_MONO12P>(a, nwin, s); break;
    case HF_U16: rc = launch_tiled<HF_U16>(a, nwin, s); break;
    case HF_U8: rc = launch_tiled<HF_U8>(a, nwin, s); break;
    case HF_F32: rc = launch_tiled<HF_F32>(a, nwin, s); break;
    default: break;
    }
    if (rc != HF_ERR_UNSUPPORTED)
      return rc;
  }
  switch (fmt) {
  case HF_MONO12P: return launch_simple<HF_MONO12P>(a, nwin, s);
  case HF_U16: return launch_simple<HF_U16>(a, nwin, s);
  case HF_U8: return launch_simple<HF_U8>(a, nwin, s);
  case HF_F32: return launch_simple<HF_F32>(a, nwin, s);
  case HF_CF32: return launch_simple<HF_CF32>(a, nwin, s);
  default: return fail(HF_ERR_INVALID, "band_dft: unsupported input dtype");
  }
}

} // namespace hf
