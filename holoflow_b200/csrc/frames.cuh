// Frame-window addressing and per-format sample access shared by the temporal kernels.
#pragma once

#include "hf_common.cuh"

namespace hf {

// A window of T frames taken from a device ring of `ring_frames` frames of `frame_bytes` bytes:
// frame t of window w is ring[(first + w*hop + t) mod ring_frames].
struct FrameRing {
  const uint8_t *base;
  int64_t        ring_frames;
  int64_t        first;
  int64_t        hop;
  int64_t        frame_bytes;
  __device__ __forceinline__ const uint8_t *frame(int w, int t) const {
    int64_t f = (first + (int64_t)w * hop + t) % ring_frames;
    return base + f * frame_bytes;
  }
};

__host__ __device__ inline int64_t frame_bytes_of(int fmt, int64_t P) {
  switch (fmt) {
  case HF_U8:
    return P;
  case HF_U16:
    return 2 * P;
  case HF_F32:
    return 4 * P;
  case HF_CF32:
    return 8 * P;
  case HF_MONO12P:
    return (3 * P) / 2;
  default:
    return -1;
  }
}

// Value of pixel p in a frame of format FMT (real formats only).
template <int FMT> __device__ __forceinline__ float sample(const uint8_t *frame, int64_t p) {
  if constexpr (FMT == HF_U8) {
    return (float)frame[p];
  } else if constexpr (FMT == HF_U16) {
    return (float)reinterpret_cast<const uint16_t *>(frame)[p];
  } else if constexpr (FMT == HF_F32) {
    return reinterpret_cast<const float *>(frame)[p];
  } else { // HF_MONO12P
    const int64_t  q  = (p >> 1) * 3;
    const uint32_t b0 = frame[q], b1 = frame[q + 1], b2 = frame[q + 2];
    return (p & 1) ? (float)((b1 >> 4) | (b2 << 4)) : (float)(b0 | ((b1 & 0xFu) << 8));
  }
}

} // namespace hf
