// Element-wise and reduction kernels of the path: 12-bit unpack/pack, dtype conversion, Mean /
// MeanAbs over one axis, band moments from planes, and the Fresnel lens / angular-spectrum
// transfer-function tables (float32 arguments evaluated operation by operation, no contraction,
// as written in the reference kernels).
#include <math_constants.h>

#include "k_misc.cuh"

namespace hf {

namespace {

int blocks_for(int64_t n, int threads) {
  const int64_t b = (n + threads - 1) / threads;
  return (int)std::min<int64_t>(std::max<int64_t>(b, 1), (int64_t)sm_count() * 64);
}

// ---- 12-bit unpack: one thread per 8 pixels (12 bytes) -----------------------------------------
template <int OUT>
__global__ void unpack12_vec_kernel(const uint32_t *in, void *out, int64_t ngroups) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ngroups;
       g += (int64_t)gridDim.x * blockDim.x) {
    uint32_t p[8];
    unpack8(__ldg(in + 3 * g), __ldg(in + 3 * g + 1), __ldg(in + 3 * g + 2), p);
    if constexpr (OUT == HF_U16) {
      reinterpret_cast<uint4 *>(out)[g] =
          make_uint4(p[0] | (p[1] << 16), p[2] | (p[3] << 16), p[4] | (p[5] << 16), p[6] | (p[7] << 16));
    } else if constexpr (OUT == HF_F32) {
      float4 *o = reinterpret_cast<float4 *>(out) + 2 * g;
      o[0]      = make_float4((float)p[0], (float)p[1], (float)p[2], (float)p[3]);
      o[1]      = make_float4((float)p[4], (float)p[5], (float)p[6], (float)p[7]);
    } else {
      float4 *o = reinterpret_cast<float4 *>(out) + 4 * g;
#pragma unroll
      for (int i = 0; i < 4; ++i)
        o[i] = make_float4((float)p[2 * i], 0.f, (float)p[2 * i + 1], 0.f);
    }
  }
}

template <int OUT>
__global__ void unpack12_scalar_kernel(const uint8_t *in, void *out, int64_t first, int64_t npix) {
  const int64_t i = first + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npix)
    return;
  const int64_t  q  = (i >> 1) * 3;
  const uint32_t b0 = in[q], b1 = in[q + 1], b2 = in[q + 2];
  const uint32_t v  = (i & 1) ? ((b1 >> 4) | (b2 << 4)) : (b0 | ((b1 & 0xFu) << 8));
  if constexpr (OUT == HF_U16)
    reinterpret_cast<uint16_t *>(out)[i] = (uint16_t)v;
  else if constexpr (OUT == HF_F32)
    reinterpret_cast<float *>(out)[i] = (float)v;
  else
    reinterpret_cast<float2 *>(out)[i] = make_float2((float)v, 0.f);
}

__global__ void pack12_kernel(const uint16_t *in, uint8_t *out, int64_t npairs) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npairs)
    return;
  const uint32_t p0 = in[2 * i] & 0xFFFu, p1 = in[2 * i + 1] & 0xFFFu;
  out[3 * i]     = (uint8_t)(p0 & 0xFFu);
  out[3 * i + 1] = (uint8_t)((p0 >> 8) | ((p1 & 0xFu) << 4));
  out[3 * i + 2] = (uint8_t)(p1 >> 4);
}

// ---- Conversion (conversion.cu:156-216) ---------------------------------------------------------
__device__ __forceinline__ unsigned int f2ord(float f) {
  const unsigned int b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned int u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

__global__ void minmax_init_kernel(unsigned int *mm) {
  mm[0] = 0xFFFFFFFFu; // min (ordered encoding)
  mm[1] = 0u;          // max
}

__global__ void minmax_kernel(const float *in, int64_t n, unsigned int *mm) {
  unsigned int lo = 0xFFFFFFFFu, hi = 0u;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned int e = f2ord(in[i]);
    lo                   = min(lo, e);
    hi                   = max(hi, e);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mm, lo);
    atomicMax(mm + 1, hi);
  }
}

template <int TOP>
__global__ void f32_scaled_kernel(const float *in, void *out, int64_t n, const unsigned int *mm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const float mn = ord2f(mm[0]), mx = ord2f(mm[1]);
  const float scale = __fdiv_rn((float)TOP, __fsub_rn(mx, mn));
  const int   val   = (int)__fadd_rn(__fmul_rn(__fsub_rn(in[i], mn), scale), 0.5f);
  const float cl    = fminf(fmaxf((float)val, 0.f), (float)TOP);
  if constexpr (TOP == 255)
    reinterpret_cast<uint8_t *>(out)[i] = (uint8_t)cl;
  else
    reinterpret_cast<uint16_t *>(out)[i] = (uint16_t)cl;
}

template <typename TI, int MODE> // MODE 0: real->F32, 1: real->CF32, 2: modulus, 3: argument
__global__ void convert_kernel(const TI *in, void *out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  if constexpr (MODE == 0) {
    reinterpret_cast<float *>(out)[i] = (float)in[i];
  } else if constexpr (MODE == 1) {
    reinterpret_cast<float2 *>(out)[i] = make_float2((float)in[i], 0.f);
  } else {
    const float2 v = reinterpret_cast<const float2 *>(in)[i];
    reinterpret_cast<float *>(out)[i] = MODE == 2 ? hypotf(v.x, v.y) : atan2f(v.y, v.x);
  }
}

// ---- Mean / MeanAbs over the middle axis of [outer][n][inner] -----------------------------------
template <typename TI, bool ABS>
__global__ void mean_axis_kernel(const TI *in, int64_t outer, int64_t n, int64_t inner, void *out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= outer * inner)
    return;
  const int64_t o = e / inner, i = e % inner;
  const TI     *p = in + o * n * inner + i;
  const float   nf = (float)n;
  if constexpr (std::is_same<TI, float2>::value && !ABS) {
    float2 acc = make_float2(0.f, 0.f);
    for (int64_t j = 0; j < n; ++j)
      acc = make_float2(__fadd_rn(acc.x, p[j * inner].x), __fadd_rn(acc.y, p[j * inner].y));
    reinterpret_cast<float2 *>(out)[e] = make_float2(__fdiv_rn(acc.x, nf), __fdiv_rn(acc.y, nf));
  } else {
    float acc = 0.f;
    for (int64_t j = 0; j < n; ++j) {
      float v;
      if constexpr (std::is_same<TI, float2>::value) {
        const float2 c = p[j * inner];
        v              = __fsqrt_rn(__fadd_rn(__fmul_rn(c.x, c.x), __fmul_rn(c.y, c.y)));
      } else {
        v = ABS ? fabsf((float)p[j * inner]) : (float)p[j * inner];
      }
      acc = __fadd_rn(acc, v);
    }
    reinterpret_cast<float *>(out)[e] = __fdiv_rn(acc, nf);
  }
}

// ---- band moments from planes --------------------------------------------------------------------
template <bool CPLX>
__global__ void band_moments_kernel(const void *planes, int nz, int64_t P, MomentWeights w,
                                    int mask, float *out) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P)
    return;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  for (int k = 0; k < nz; ++k) {
    float m;
    if constexpr (CPLX) {
      const float2 v = reinterpret_cast<const float2 *>(planes)[(int64_t)k * P + p];
      m              = hypotf(v.x, v.y);
    } else {
      m = reinterpret_cast<const float *>(planes)[(int64_t)k * P + p];
    }
    a0 = __fadd_rn(a0, m);
    a1 = __fadd_rn(a1, __fmul_rn(w.w1[k], m));
    a2 = __fadd_rn(a2, __fmul_rn(w.w2[k], m));
  }
  const float nf = (float)nz;
  int         mi = 0;
  if (mask & HF_M0)
    out[(mi++) * P + p] = __fdiv_rn(a0, nf);
  if (mask & HF_M1)
    out[(mi++) * P + p] = __fdiv_rn(a1, nf);
  if (mask & HF_M2)
    out[(mi++) * P + p] = __fdiv_rn(a2, nf);
}

// ---- lens / transfer function tables ------------------------------------------------------------
__global__ void fresnel_lens_kernel(float2 *lens, int W, int H, float lambda, float z, float dx) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= W || row >= H)
    return;
  lens[(int64_t)row * W + col] = fresnel_lens_value(col, row, W, H, fresnel_lens_k(lambda, z), dx);
}

__device__ float as_filter_weight(int x, int y, int W, int H, AsFilter f) {
  const float rx   = __fsub_rn((float)x, __fdiv_rn((float)W, 2.0f));
  const float ry   = __fsub_rn((float)y, __fdiv_rn((float)H, 2.0f));
  const float dist = hypotf(rx, ry);
  const float is = __fsub_rn((float)f.r_inner, (float)f.s_inner);
  const float ie = __fadd_rn((float)f.r_inner, (float)f.s_inner);
  const float os = __fsub_rn((float)f.r_outer, (float)f.s_outer);
  const float oe = __fadd_rn((float)f.r_outer, (float)f.s_outer);
  float       v  = 0.f;
  if (dist < is) {
    v = 0.f;
  } else if (dist < ie) {
    const float a = __fmul_rn(__fdiv_rn(CUDART_PI_F, __fmul_rn(2.0f, (float)f.s_inner)), __fsub_rn(dist, is));
    v             = __fmul_rn(0.5f, __fadd_rn(1.0f, sinf(a)));
  } else if (dist < os) {
    v = 1.f;
  } else if (dist < oe) {
    const float a = __fmul_rn(__fdiv_rn(CUDART_PI_F, __fmul_rn(2.0f, (float)f.s_outer)), __fsub_rn(oe, dist));
    v             = __fmul_rn(0.5f, __fadd_rn(1.0f, sinf(a)));
  }
  return __fmul_rn(v, v);
}

// Writes swap_corners(TF * w^2): destination (row, col) takes the centred value of its source.
__global__ void as_tf_kernel(float2 *tf, int W, int H, float lambda, float z, float dx, int use_filter,
                             AsFilter f) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y * blockDim.y + threadIdx.y;
  if (col >= W || row >= H)
    return;
  const int wh = W / 2, hh = H / 2;
  int       sc = col, sr = row;
  if (col < 2 * wh && row < 2 * hh) {
    sc = col < wh ? col + wh : col - wh;
    sr = row < hh ? row + hh : row - hh;
  }
  const float du   = __fdiv_rn(1.0f, __fmul_rn((float)W, dx));
  const float dv   = __fdiv_rn(1.0f, __fmul_rn((float)H, dx));
  const float u    = __fmul_rn((float)(sc - W / 2), du);
  const float v    = __fmul_rn((float)(sr - H / 2), dv);
  float       tmp  = __fsub_rn(1.0f, __fmul_rn(__fmul_rn(lambda, lambda), __fadd_rn(__fmul_rn(u, u), __fmul_rn(v, v))));
  tmp              = fmaxf(tmp, 0.0f);
  const float k    = __fdiv_rn(__fmul_rn(__fmul_rn(2.0f, CUDART_PI_F), z), lambda);
  const float ph   = __fmul_rn(k, __fsqrt_rn(tmp));
  float       s, c;
  sincosf(ph, &s, &c);
  if (use_filter) {
    const float wgt = as_filter_weight(sc, sr, W, H, f);
    c               = __fmul_rn(c, wgt);
    s               = __fmul_rn(s, wgt);
  }
  tf[(int64_t)row * W + col] = make_float2(c, s);
}

} // namespace

int launch_unpack12(const uint8_t *in, void *out, int out_dtype, int64_t npix, cudaStream_t s) {
  HF_CHECK_ARG(npix >= 0 && npix % 2 == 0, "unpack12: npix must be even");
  HF_CHECK_ARG(out_dtype == HF_U16 || out_dtype == HF_F32 || out_dtype == HF_CF32,
               "unpack12: out_dtype must be U16, F32 or CF32");
  if (npix == 0)
    return HF_OK;
  const bool aligned = ((uintptr_t)in % 4 == 0) && ((uintptr_t)out % 16 == 0);
  const int64_t ngroups = aligned ? npix / 8 : 0;
  if (ngroups > 0) {
    const int b = blocks_for(ngroups, 256);
    const uint32_t *iw = reinterpret_cast<const uint32_t *>(in);
    if (out_dtype == HF_U16)
      unpack12_vec_kernel<HF_U16><<<b, 256, 0, s>>>(iw, out, ngroups);
    else if (out_dtype == HF_F32)
      unpack12_vec_kernel<HF_F32><<<b, 256, 0, s>>>(iw, out, ngroups);
    else
      unpack12_vec_kernel<HF_CF32><<<b, 256, 0, s>>>(iw, out, ngroups);
    note_launch();
    HF_TRY(launch_status("unpack12_vec_kernel"));
  }
  const int64_t first = ngroups * 8, rest = npix - first;
  if (rest > 0) {
    const unsigned b = (unsigned)((rest + 255) / 256);
    if (out_dtype == HF_U16)
      unpack12_scalar_kernel<HF_U16><<<b, 256, 0, s>>>(in, out, first, npix);
    else if (out_dtype == HF_F32)
      unpack12_scalar_kernel<HF_F32><<<b, 256, 0, s>>>(in, out, first, npix);
    else
      unpack12_scalar_kernel<HF_CF32><<<b, 256, 0, s>>>(in, out, first, npix);
    note_launch();
    HF_TRY(launch_status("unpack12_scalar_kernel"));
  }
  return HF_OK;
}

int launch_pack12(const uint16_t *in, uint8_t *out, int64_t npix, cudaStream_t s) {
  HF_CHECK_ARG(npix >= 0 && npix % 2 == 0, "pack12: npix must be even");
  if (npix == 0)
    return HF_OK;
  const int64_t pairs = npix / 2;
  pack12_kernel<<<(unsigned)((pairs + 255) / 256), 256, 0, s>>>(in, out, pairs);
  note_launch();
  return launch_status("pack12_kernel");
}

int launch_convert(const void *in, int in_dtype, void *out, int out_dtype, int strategy, int64_t n,
                   void *minmax_ws, cudaStream_t s) {
  if (n == 0)
    return HF_OK;
  const unsigned b = (unsigned)((n + 255) / 256);
  if (strategy == HF_CONV_REAL) {
    if (in_dtype == HF_U8 && out_dtype == HF_F32)
      convert_kernel<uint8_t, 0><<<b, 256, 0, s>>>((const uint8_t *)in, out, n);
    else if (in_dtype == HF_U8 && out_dtype == HF_CF32)
      convert_kernel<uint8_t, 1><<<b, 256, 0, s>>>((const uint8_t *)in, out, n);
    else if (in_dtype == HF_U16 && out_dtype == HF_CF32)
      convert_kernel<uint16_t, 1><<<b, 256, 0, s>>>((const uint16_t *)in, out, n);
    else if (in_dtype == HF_F32 && out_dtype == HF_CF32)
      convert_kernel<float, 1><<<b, 256, 0, s>>>((const float *)in, out, n);
    else
      return fail(HF_ERR_INVALID, "Conversion: unsupported (input, target, Real) combination");
  } else if (strategy == HF_CONV_MODULUS || strategy == HF_CONV_ARGUMENT) {
    HF_CHECK_ARG(in_dtype == HF_CF32 && out_dtype == HF_F32,
                 "Conversion: Modulus/Argument map CF32 to F32");
    if (strategy == HF_CONV_MODULUS)
      convert_kernel<float, 2><<<b, 256, 0, s>>>((const float *)in, out, n);
    else
      convert_kernel<float, 3><<<b, 256, 0, s>>>((const float *)in, out, n);
  } else if (strategy == HF_CONV_SCALED) {
    HF_CHECK_ARG(in_dtype == HF_F32 && (out_dtype == HF_U8 || out_dtype == HF_U16),
                 "Conversion: Scaled maps F32 to U8 or U16");
    HF_CHECK_ARG(minmax_ws != nullptr, "Conversion: Scaled needs the min/max scratch");
    unsigned int *mm = reinterpret_cast<unsigned int *>(minmax_ws);
    minmax_init_kernel<<<1, 1, 0, s>>>(mm);
    minmax_kernel<<<blocks_for(n, 256), 256, 0, s>>>((const float *)in, n, mm);
    if (out_dtype == HF_U8)
      f32_scaled_kernel<255><<<b, 256, 0, s>>>((const float *)in, out, n, mm);
    else
      f32_scaled_kernel<65535><<<b, 256, 0, s>>>((const float *)in, out, n, mm);
    note_launch(2);
  } else {
    return fail(HF_ERR_INVALID, "Conversion: unknown strategy");
  }
  note_launch();
  return launch_status("convert_kernel");
}

int launch_mean_axis(const void *in, int in_dtype, int64_t outer, int64_t n, int64_t inner,
                     void *out, bool abs_values, cudaStream_t s) {
  HF_CHECK_ARG(outer >= 0 && n > 0 && inner >= 0, "mean: bad extents");
  const int64_t total = outer * inner;
  if (total == 0)
    return HF_OK;
  const unsigned b = (unsigned)((total + 255) / 256);
  switch (in_dtype) {
  case HF_U8:
    HF_CHECK_ARG(!abs_values, "MeanAbs: input must be F32 or CF32");
    mean_axis_kernel<uint8_t, false><<<b, 256, 0, s>>>((const uint8_t *)in, outer, n, inner, out);
    break;
  case HF_U16:
    HF_CHECK_ARG(!abs_values, "MeanAbs: input must be F32 or CF32");
    mean_axis_kernel<uint16_t, false><<<b, 256, 0, s>>>((const uint16_t *)in, outer, n, inner, out);
    break;
  case HF_F32:
    if (abs_values)
      mean_axis_kernel<float, true><<<b, 256, 0, s>>>((const float *)in, outer, n, inner, out);
    else
      mean_axis_kernel<float, false><<<b, 256, 0, s>>>((const float *)in, outer, n, inner, out);
    break;
  case HF_CF32:
    if (abs_values)
      mean_axis_kernel<float2, true><<<b, 256, 0, s>>>((const float2 *)in, outer, n, inner, out);
    else
      mean_axis_kernel<float2, false><<<b, 256, 0, s>>>((const float2 *)in, outer, n, inner, out);
    break;
  default:
    return fail(HF_ERR_INVALID, "mean: unsupported dtype");
  }
  note_launch();
  return launch_status("mean_axis_kernel");
}

int launch_band_moments(const void *planes, int in_dtype, int nz, int64_t P, const MomentWeights &w,
                        int mask, float *out, cudaStream_t s) {
  HF_CHECK_ARG(nz > 0 && nz <= kMaxMomentBands && P > 0, "band moments: bad extents");
  HF_CHECK_ARG((mask & 7) != 0, "band moments: empty moment mask");
  const unsigned b = (unsigned)((P + 255) / 256);
  if (in_dtype == HF_CF32)
    band_moments_kernel<true><<<b, 256, 0, s>>>(planes, nz, P, w, mask, out);
  else if (in_dtype == HF_F32)
    band_moments_kernel<false><<<b, 256, 0, s>>>(planes, nz, P, w, mask, out);
  else
    return fail(HF_ERR_INVALID, "band moments: planes must be F32 or CF32");
  note_launch();
  return launch_status("band_moments_kernel");
}

int launch_fresnel_lens(float2 *lens, int W, int H, float lambda, float z, float dx, cudaStream_t s) {
  dim3 blk(16, 16), grd((W + 15) / 16, (H + 15) / 16);
  fresnel_lens_kernel<<<grd, blk, 0, s>>>(lens, W, H, lambda, z, dx);
  note_launch();
  return launch_status("fresnel_lens_kernel");
}

int launch_as_tf(float2 *tf, int W, int H, float lambda, float z, float dx, int use_filter,
                 const AsFilter &f, cudaStream_t s) {
  dim3 blk(16, 16), grd((W + 15) / 16, (H + 15) / 16);
  as_tf_kernel<<<grd, blk, 0, s>>>(tf, W, H, lambda, z, dx, use_filter, f);
  note_launch();
  return launch_status("as_tf_kernel");
}

} // namespace hf
