// Element kernels behind the thin holonp node kinds GraphBuilder wires between the path's stages
// (graph_builder.cc:256-287, 578-631): strided copies (Copy, a copying Reshape, Concatenate),
// broadcast Multiply, Abs, Arange, and the causal sliding average of the autofocus chain.  All
// are single memory-bound passes, one element per thread in a grid-stride loop over a grid sized
// to the SMs.
#include "k_np.cuh"

namespace hf {

namespace {

int np_blocks(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)sm_count() * 16));
}

// dst element i (row-major over `shape`) <- src at sum_d coord_d * src_strides_d bytes, written at
// sum_d coord_d * dst_strides_d bytes.
template <typename E> __global__ void copy_strided_kernel(const uint8_t *src, uint8_t *dst, NpLayout l, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t rem = i, so = 0, doff = 0;
    for (int d = l.rank - 1; d >= 0; --d) {
      const int64_t c = rem % l.shape[d];
      rem /= l.shape[d];
      so += c * l.src_strides[d];
      doff += c * l.dst_strides[d];
    }
    *reinterpret_cast<E *>(dst + doff) = *reinterpret_cast<const E *>(src + so);
  }
}

// out[i] = a[...] * b[...] over broadcast strides (0 along broadcast dimensions), in elements.
template <typename A, typename B, typename O>
__global__ void multiply_kernel(const A *a, const B *b, O *out, NpBroadcast l, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t rem = i, ao = 0, bo = 0;
    for (int d = l.rank - 1; d >= 0; --d) {
      const int64_t c = rem % l.shape[d];
      rem /= l.shape[d];
      ao += c * l.a_strides[d];
      bo += c * l.b_strides[d];
    }
    if constexpr (std::is_same_v<O, float>) {
      out[i] = a[ao] * b[bo];
    } else {
      float2 x, y;
      if constexpr (std::is_same_v<A, float>)
        x = make_float2(a[ao], 0.f);
      else
        x = a[ao];
      if constexpr (std::is_same_v<B, float>)
        y = make_float2(b[bo], 0.f);
      else
        y = b[bo];
      // (x.re y.re - x.im y.im, x.re y.im + x.im y.re), each product rounded before the sum
      out[i] = make_float2(__fsub_rn(__fmul_rn(x.x, y.x), __fmul_rn(x.y, y.y)),
                           __fadd_rn(__fmul_rn(x.x, y.y), __fmul_rn(x.y, y.x)));
    }
  }
}

template <typename I> __global__ void abs_kernel(const I *in, float *out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if constexpr (std::is_same_v<I, float2>) {
      const float2 v = in[i];
      out[i]         = __fsqrt_rn(__fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y))); // abs.cu:67-70
    } else if constexpr (std::is_same_v<I, float>) {
      out[i] = fabsf(in[i]);
    } else {
      out[i] = (float)in[i];
    }
  }
}

__global__ void arange_kernel(float *out, double start, double step, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)(start + step * (double)i);
}

__global__ void causal_avg_kernel(const float *in, float *out, float *hist, float *sum, int64_t n, float divisor) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = in[i], old = hist[i];
    const float s = sum[i] + v - old;
    hist[i]       = v;
    sum[i]        = s;
    out[i]        = s / divisor;
  }
}

} // namespace

int launch_copy_strided(const void *src, void *dst, const NpLayout &l, int elem_size, cudaStream_t s) {
  int64_t n = 1;
  for (int d = 0; d < l.rank; ++d)
    n *= l.shape[d];
  if (n == 0)
    return HF_OK;
  const auto *a = reinterpret_cast<const uint8_t *>(src);
  auto       *b = reinterpret_cast<uint8_t *>(dst);
  switch (elem_size) {
  case 1: copy_strided_kernel<uint8_t><<<np_blocks(n), 256, 0, s>>>(a, b, l, n); break;
  case 2: copy_strided_kernel<uint16_t><<<np_blocks(n), 256, 0, s>>>(a, b, l, n); break;
  case 4: copy_strided_kernel<uint32_t><<<np_blocks(n), 256, 0, s>>>(a, b, l, n); break;
  case 8: copy_strided_kernel<uint2><<<np_blocks(n), 256, 0, s>>>(a, b, l, n); break;
  default: return fail(HF_ERR_INVALID, "strided copy: element size must be 1, 2, 4 or 8");
  }
  note_launch();
  return launch_status("copy_strided_kernel");
}

int launch_multiply(const void *a, int a_cplx, const void *b, int b_cplx, void *out, const NpBroadcast &l,
                    cudaStream_t s) {
  int64_t n = 1;
  for (int d = 0; d < l.rank; ++d)
    n *= l.shape[d];
  if (n == 0)
    return HF_OK;
  const int g = np_blocks(n);
  if (!a_cplx && !b_cplx)
    multiply_kernel<float, float, float><<<g, 256, 0, s>>>((const float *)a, (const float *)b, (float *)out, l, n);
  else if (a_cplx && b_cplx)
    multiply_kernel<float2, float2, float2><<<g, 256, 0, s>>>((const float2 *)a, (const float2 *)b, (float2 *)out, l, n);
  else if (a_cplx)
    multiply_kernel<float2, float, float2><<<g, 256, 0, s>>>((const float2 *)a, (const float *)b, (float2 *)out, l, n);
  else
    multiply_kernel<float, float2, float2><<<g, 256, 0, s>>>((const float *)a, (const float2 *)b, (float2 *)out, l, n);
  note_launch();
  return launch_status("multiply_kernel");
}

int launch_abs(const void *in, int in_dtype, float *out, int64_t n, cudaStream_t s) {
  if (n == 0)
    return HF_OK;
  const int g = np_blocks(n);
  switch (in_dtype) {
  case HF_CF32: abs_kernel<float2><<<g, 256, 0, s>>>((const float2 *)in, out, n); break;
  case HF_F32: abs_kernel<float><<<g, 256, 0, s>>>((const float *)in, out, n); break;
  case HF_U16: abs_kernel<uint16_t><<<g, 256, 0, s>>>((const uint16_t *)in, out, n); break;
  case HF_U8: abs_kernel<uint8_t><<<g, 256, 0, s>>>((const uint8_t *)in, out, n); break;
  default: return fail(HF_ERR_INVALID, "abs: unsupported dtype");
  }
  note_launch();
  return launch_status("abs_kernel");
}

int launch_arange(float *out, double start, double step, int64_t n, cudaStream_t s) {
  if (n == 0)
    return HF_OK;
  arange_kernel<<<np_blocks(n), 256, 0, s>>>(out, start, step, n);
  note_launch();
  return launch_status("arange_kernel");
}

int launch_causal_avg(const float *in, float *out, float *hist_slot, float *sum, int64_t n, float divisor,
                      cudaStream_t s) {
  if (n == 0)
    return HF_OK;
  causal_avg_kernel<<<np_blocks(n), 256, 0, s>>>(in, out, hist_slot, sum, n, divisor);
  note_launch();
  return launch_status("causal_avg_kernel");
}

} // namespace hf
