// Common definitions for the holoflow_b200 CUDA library: status codes, error capture and small
// device helpers shared by every kernel translation unit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "holoflow_b200.h"

namespace hf {

// Thread-local last-error text behind hf_last_error(); set by every failing entry point.
void set_error(const std::string &msg);
void clear_error();

// Records `msg` and returns `code`; used as `return fail(HF_ERR_INVALID, "...")`.
int fail(int code, const std::string &msg);

// Maps a CUDA error (if any) to HF_ERR_CUDA with a message naming the call site.
int cuda_status(cudaError_t e, const char *where);

inline int launch_status(const char *where) { return cuda_status(cudaGetLastError(), where); }

// Counts kernel launches enqueued by this thread (reported by hf_launch_count()).
void note_launch(int n = 1);

#define HF_TRY(expr)                                                                             \
  do {                                                                                           \
    int hf_rc__ = (expr);                                                                        \
    if (hf_rc__ != HF_OK)                                                                        \
      return hf_rc__;                                                                            \
  } while (0)

#define HF_CUDA(expr)                                                                            \
  do {                                                                                           \
    cudaError_t hf_e__ = (expr);                                                                 \
    if (hf_e__ != cudaSuccess)                                                                   \
      return ::hf::cuda_status(hf_e__, #expr);                                                   \
  } while (0)

#define HF_CHECK_ARG(cond, msg)                                                                  \
  do {                                                                                           \
    if (!(cond))                                                                                 \
      return ::hf::fail(HF_ERR_INVALID, msg);                                                    \
  } while (0)

constexpr int kNumSMs = 148; // B200: 2 dies x 74 SMs; grids are sized in multiples of this.

// SM count of the current device, cached per device ordinal (grid splits depend on it, so a thread
// that switches devices must see each device's own count).
inline int sm_count() {
  constexpr int kMaxDev = 64;
  static thread_local int cached[kMaxDev] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev)
    return kNumSMs;
  if (cached[dev] == 0) {
    int n = 0;
    cached[dev] = (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n > 0) ? n
                                                                                                          : kNumSMs;
  }
  return cached[dev];
}

// ------------------------------------------------------------------------------------------------
// Device helpers
// ------------------------------------------------------------------------------------------------

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// complex add / subtract as one packed fp32x2 instruction (each lane rounds as the scalar op)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
// d = a * b + c per lane, one packed fp32x2 instruction
__device__ __forceinline__ float2 cfma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
// d = a * b per lane, one packed fp32x2 instruction
__device__ __forceinline__ float2 pmul2(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  float2 d;
  asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
      "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
      : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float cabs_hypot(float2 a) { return hypotf(a.x, a.y); }

// 12-bit little-endian packed pair (Mono12p): 3 bytes -> 2 pixels.
__device__ __forceinline__ void unpack_pair(uint32_t b0, uint32_t b1, uint32_t b2, uint32_t &p0,
                                            uint32_t &p1) {
  p0 = b0 | ((b1 & 0xFu) << 8);
  p1 = (b1 >> 4) | (b2 << 4);
}

// 12 bytes (three little-endian words) -> 8 pixels.
__device__ __forceinline__ void unpack8(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t (&p)[8]) {
  // bytes: w0 = b0 b1 b2 b3, w1 = b4 b5 b6 b7, w2 = b8 b9 b10 b11
  p[0] = w0 & 0xFFFu;
  p[1] = (w0 >> 12) & 0xFFFu;
  p[2] = (w0 >> 24) | ((w1 & 0xFu) << 8);
  p[3] = (w1 >> 4) & 0xFFFu;
  p[4] = (w1 >> 16) & 0xFFFu;
  p[5] = (w1 >> 28) | ((w2 & 0xFFu) << 4);
  p[6] = (w2 >> 8) & 0xFFFu;
  p[7] = (w2 >> 20) & 0xFFFu;
}

} // namespace hf
