// Pieces shared by the tensor-core band DFT kernels (k_tc_band.cu: the fused pass over whole
// rows; k_tc_band_seg.cu: raw band planes in row segments): bounded mbarrier waits that turn into
// no-ops once any wait of the CTA has expired, named barriers, plain arrives, and the loads of 32
// consecutive samples of one frame in the ring's packed 12-bit or uint16 format.
#pragma once

#include "hf_common.cuh"
#include "tc_common.cuh"

namespace hf {
namespace tcb {

__device__ __forceinline__ bool wait_or_abort(uint64_t *mbar, uint32_t parity, volatile int *abort, int *status,
                                              int code) {
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
    atomicCAS(status, 0, code);
  *abort = 1;
  return false;
}

__device__ __forceinline__ void named_bar(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(mbar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_cnt(uint64_t *mbar, uint32_t cnt) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(mbar)), "r"(cnt) : "memory");
}

// 32 consecutive samples of one frame: `raw` issues the 16-byte loads of their packed bytes,
// `unpack` turns the packed words into the 32 sample values.  Splitting the two lets the loaders
// keep the next round's loads in flight while they unpack the current one.
template <int FMT> struct GroupLoad;
template <> struct GroupLoad<HF_MONO12P> {
  static constexpr int kBytes = 48, kWords = 12, kPerRound = 4; // groups in flight per thread
  __device__ static void raw(const uint8_t *src, uint32_t (&w)[kWords]) {
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const uint4 a = __ldg(s + i);
      w[4 * i] = a.x, w[4 * i + 1] = a.y, w[4 * i + 2] = a.z, w[4 * i + 3] = a.w;
    }
  }
  __device__ static void unpack(const uint32_t (&w)[kWords], uint32_t (&v)[32]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t p[8];
      unpack8(w[3 * q], w[3 * q + 1], w[3 * q + 2], p);
#pragma unroll
      for (int i = 0; i < 8; ++i)
        v[8 * q + i] = p[i];
    }
  }
};
template <> struct GroupLoad<HF_U16> {
  static constexpr int kBytes = 64, kWords = 16, kPerRound = 2;
  __device__ static void raw(const uint8_t *src, uint32_t (&w)[kWords]) {
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint4 a = __ldg(s + i);
      w[4 * i] = a.x, w[4 * i + 1] = a.y, w[4 * i + 2] = a.z, w[4 * i + 3] = a.w;
    }
  }
  __device__ static void unpack(const uint32_t (&w)[kWords], uint32_t (&v)[32]) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      v[2 * i]     = w[i] & 0xFFFFu;
      v[2 * i + 1] = w[i] >> 16;
    }
  }
};

} // namespace tcb
} // namespace hf
