// Host-side helpers shared by the C ABI translation units: device allocation bookkeeping and
// parameter conversions.
#pragma once

#include <cmath>
#include <string>

#include "k_fft2d.cuh"

namespace hf {

// Where plan and camera-stream buffers come from.  By default cudaMalloc / cudaFree; inside an
// AllocScope with a memory pool, stream-ordered cudaMallocFromPoolAsync / cudaFreeAsync on the
// scope's stream, which neither synchronise the device nor wait for other streams -- the
// streaming server opens and closes streams this way while other streams' work runs.
struct AllocCtx {
  cudaMemPool_t pool   = nullptr;
  cudaStream_t  stream = nullptr;
};
inline AllocCtx &alloc_ctx() {
  static thread_local AllocCtx c;
  return c;
}
class AllocScope {
public:
  AllocScope(cudaMemPool_t pool, cudaStream_t stream) : saved_(alloc_ctx()) { alloc_ctx() = AllocCtx{pool, stream}; }
  ~AllocScope() { alloc_ctx() = saved_; }
  AllocScope(const AllocScope &)            = delete;
  AllocScope &operator=(const AllocScope &) = delete;

private:
  AllocCtx saved_;
};

template <typename T> inline int dev_alloc(T **p, size_t count, size_t &total) {
  *p = nullptr;
  if (count == 0)
    return HF_OK;
  const size_t    bytes = count * sizeof(T);
  const AllocCtx &ctx   = alloc_ctx();
  cudaError_t     e     = ctx.pool ? cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, ctx.pool, ctx.stream)
                                   : cudaMalloc(reinterpret_cast<void **>(p), bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    (void)cudaGetLastError();
    return fail(HF_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
  }
  total += bytes;
  return HF_OK;
}

template <typename T> inline void dev_free(T *&p) {
  if (p) {
    const AllocCtx &ctx = alloc_ctx();
    if (ctx.pool)
      cudaFreeAsync(p, ctx.stream);
    else
      cudaFree(p);
  }
  p = nullptr;
}

inline float norm_scale(int norm, int n) {
  if (norm == HF_NORM_FORWARD)
    return (float)(1.0 / (double)n);
  if (norm == HF_NORM_ORTHO)
    return (float)(1.0 / std::sqrt((double)n));
  return 1.0f;
}

inline bool real_fmt(int f) { return f == HF_U8 || f == HF_U16 || f == HF_F32 || f == HF_MONO12P; }

// f_k = start + k*df evaluated in double and cast (arange.cu:62-75); f_k^2 in float32
// (graph_builder.cc:624-627).  The two-sided method's nz planes are the positive band's nz / 2
// and then the negative band's, weighted arange(f0 - fs, f1 - fs, df) (graph_builder.cc:590-594).
inline void fill_weights(MomentSpec &m, int T, int z0, int nz, double fs, bool two_sided = false) {
  const double df  = fs / (double)T;
  const double f0  = z0 * df;
  const int    nzh = two_sided ? nz / 2 : nz;
  for (int k = 0; k < kMaxBands; ++k) {
    float f = 0.f;
    if (k < nzh)
      f = (float)(f0 + df * (double)k);
    else if (k < nz)
      f = (float)((f0 - fs) + df * (double)(k - nzh));
    m.w1[k] = f;
    m.w2[k] = f * f;
  }
}

} // namespace hf
