// FFT building blocks for the spatial propagation kernels.
//
// A length-N transform (N = N1 * 32) is computed "four-step" style with every butterfly in
// registers and exactly one shared-memory exchange:
//   input index j = n2 + 32*n1  (lane n2 holds the N1 samples n1 = 0..N1-1)
//   1. N1-point DFT over n1 in registers            -> Y[n2][k1]
//   2. twiddle  Y[n2][k1] *= w_N^(n2*k1)             (shared-memory table, conflict-free swizzle)
//   3. exchange through a padded [N1][33] buffer     (lane k1 now holds Y[0..31][k1])
//   4. 32-point DFT over n2 in registers            -> X[k1 + N1*k2]
// so a load of "lane n2, element n1" and a store of "lane k1, element k2" are both coalesced
// along the transform axis.  The inverse direction runs the same steps with conjugate twiddles,
// and `four_step_rev` runs the transposed order (input distributed as k1 + N1*k2) so that a
// forward transform followed by an inverse one returns the data to the load distribution.
#pragma once

#include "hf_common.cuh"
#include "twiddles.inc"

namespace hf {

// ------------------------------------------------------------------------------------------------
// Compile-time helpers
// ------------------------------------------------------------------------------------------------
__host__ __device__ constexpr int ilog2_c(int n) { return n <= 1 ? 0 : 1 + ilog2_c(n >> 1); }
__host__ __device__ constexpr int brev_c(int v, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i)
    r |= ((v >> i) & 1) << (bits - 1 - i);
  return r;
}

// exp(-2 pi i k / N) from the constant tables (k is a compile-time constant after unrolling)
template <int N> __device__ __forceinline__ float2 ctw(int k);
template <> __device__ __forceinline__ float2 ctw<4>(int k) { return c_tw4[k & 3]; }
template <> __device__ __forceinline__ float2 ctw<8>(int k) { return c_tw8[k & 7]; }
template <> __device__ __forceinline__ float2 ctw<16>(int k) { return c_tw16[k & 15]; }
template <> __device__ __forceinline__ float2 ctw<24>(int k) { return c_tw24[k % 24]; }
template <> __device__ __forceinline__ float2 ctw<32>(int k) { return c_tw32[k & 31]; }
template <> __device__ __forceinline__ float2 ctw<48>(int k) { return c_tw48[k % 48]; }
template <> __device__ __forceinline__ float2 ctw<64>(int k) { return c_tw64[k & 63]; }

// Tangent-form twiddles (m, t) of c_twtN (see gen_twiddles.py): w = m (1 + i t) when the angle is
// within 45 degrees of the real axis, w = m (t + i) otherwise.
template <int N> __device__ __forceinline__ float2 ctwt(int k);
template <> __device__ __forceinline__ float2 ctwt<2>(int) { return make_float2(0.f, 0.f); } // all trivial
template <> __device__ __forceinline__ float2 ctwt<4>(int k) { return c_twt4[k & 3]; }        // all trivial
template <> __device__ __forceinline__ float2 ctwt<8>(int k) { return c_twt8[k & 7]; }
template <> __device__ __forceinline__ float2 ctwt<16>(int k) { return c_twt16[k & 15]; }
template <> __device__ __forceinline__ float2 ctwt<24>(int k) { return c_twt24[k % 24]; }
template <> __device__ __forceinline__ float2 ctwt<32>(int k) { return c_twt32[k & 31]; }
template <> __device__ __forceinline__ float2 ctwt<48>(int k) { return c_twt48[k % 48]; }
template <> __device__ __forceinline__ float2 ctwt<64>(int k) { return c_twt64[k & 63]; }
__host__ __device__ constexpr bool tw_near_real(int k, int n) {
  return 8 * (k % (n / 2)) <= n || 8 * (k % (n / 2)) >= 3 * n;
}

// b * exp(-+2 pi i k/N) with the trivial angles handled without a multiply.
template <int N, bool INV> __device__ __forceinline__ float2 twmul_c(float2 b, int k) {
  k %= N;
  if (k == 0)
    return b;
  if (4 * k == N) // -i (forward) / +i (inverse)
    return INV ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
  if (2 * k == N)
    return make_float2(-b.x, -b.y);
  if (4 * k == 3 * N)
    return INV ? make_float2(b.y, -b.x) : make_float2(-b.y, b.x);
  float2 w = ctw<N>(k);
  if (INV)
    w.y = -w.y;
  return cmul(b, w);
}

// Radix-2 butterfly (a, b) <- (a + w b, a - w b), w = exp(-+2 pi i k/N).  w = +-1 and w = -+i cost
// one packed fp32x2 add and one packed subtract (of b or its swapped, negated pair); the other
// angles go through the tangent form of w: two scalar fused multiply-adds for (u, v) = w b / m,
// then two packed ones for a +- m (u, v).  Every lane rounds exactly as the scalar form would.
template <int N, bool INV> __device__ __forceinline__ void bfly(float2 &a, float2 &b, int k) {
  k %= N;
  if (k == 0 || 4 * k == N || 2 * k == N || 4 * k == 3 * N) {
    const float2 wb = twmul_c<N, INV>(b, k);
    b               = csub(a, wb);
    a               = cadd(a, wb);
  } else if (tw_near_real(k, N)) { // w = m (1 + i t); the inverse uses w* = m (1 - i t)
    const float2 mt = ctwt<N>(k);
    const float  m = mt.x, t = INV ? -mt.y : mt.y;
    const float2 uv = make_float2(fmaf(-t, b.y, b.x), fmaf(t, b.x, b.y));
    b               = cfma2(make_float2(-m, -m), uv, a);
    a               = cfma2(make_float2(m, m), uv, a);
  } else { // w = m (t + i); the inverse uses w* = (-m)(-t + i)
    const float2 mt = ctwt<N>(k);
    const float  m = INV ? -mt.x : mt.x, t = INV ? -mt.y : mt.y;
    const float2 uv = make_float2(fmaf(t, b.x, -b.y), fmaf(t, b.y, b.x));
    b               = cfma2(make_float2(-m, -m), uv, a);
    a               = cfma2(make_float2(m, m), uv, a);
  }
}

// ------------------------------------------------------------------------------------------------
// In-register DFTs (natural order in, natural order out)
// ------------------------------------------------------------------------------------------------
template <int N, bool INV> __device__ __forceinline__ void dft_pow2(float2 *x) {
  constexpr int LOG = ilog2_c(N);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const int j = brev_c(i, LOG);
    if (j > i) {
      float2 t = x[i];
      x[i]     = x[j];
      x[j]     = t;
    }
  }
#pragma unroll
  for (int s = 1; s <= LOG; ++s) {
    const int m = 1 << s;
    const int h = m >> 1;
#pragma unroll
    for (int k = 0; k < h; ++k) {
#pragma unroll
      for (int i = 0; i < N; i += m)
        bfly<N, INV>(x[i + k], x[i + k + h], k * (N / m));
    }
  }
}

// N = 3*M: three interleaved M-point DFTs then radix-3 butterflies.
template <int N, bool INV> __device__ __forceinline__ void dft_mixed3(float2 *x) {
  constexpr int M = N / 3;
  float2        y[3][M];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int m = 0; m < M; ++m)
      y[j][m] = x[3 * m + j];
#pragma unroll
  for (int j = 0; j < 3; ++j)
    dft_pow2<M, INV>(y[j]);
  const float s3 = 0.8660254037844386f; // sqrt(3)/2
#pragma unroll
  for (int k = 0; k < M; ++k) {
    const float2 a = y[0][k];
    const float2 b = twmul_c<N, INV>(y[1][k], k);
    const float2 c = twmul_c<N, INV>(y[2][k], 2 * k);
    const float2 t1 = cadd(b, c);
    const float2 t2 = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
    const float2 d  = csub(b, c);
    // t3 = -+ i * s3 * (b - c)
    const float2 t3 = INV ? make_float2(-s3 * d.y, s3 * d.x) : make_float2(s3 * d.y, -s3 * d.x);
    x[k]         = cadd(a, t1);
    x[k + M]     = cadd(t2, t3);
    x[k + 2 * M] = csub(t2, t3);
  }
}

template <int N, bool INV> __device__ __forceinline__ void dft_reg(float2 *x) {
  if constexpr (N == 1) {
    return;
  } else if constexpr (N % 3 == 0) {
    dft_mixed3<N, INV>(x);
  } else {
    dft_pow2<N, INV>(x);
  }
}

// ------------------------------------------------------------------------------------------------
// Shared-memory twiddle table for w_N^m, m < N: separate cos / sin arrays, entry m stored at
// m ^ ((m >> 5) & 31) so that the strided lookups of the four-step spread over all banks.
// ------------------------------------------------------------------------------------------------
struct SmemTwiddles {
  float *c;
  float *s;
  int    n;
  __device__ __forceinline__ static int slot(int m) { return m ^ ((m >> 5) & 31); }
  // Cooperative fill by the whole block (caller synchronises).
  __device__ __forceinline__ void fill(int tid, int nthreads) {
    for (int m = tid; m < n; m += nthreads) {
      float sv, cv;
      sincospif(-2.0f * (float)m / (float)n, &sv, &cv);
      c[slot(m)] = cv;
      s[slot(m)] = sv;
    }
  }
  template <bool INV> __device__ __forceinline__ float2 get(int m) const {
    const int q = slot(m);
    return make_float2(c[q], INV ? -s[q] : s[q]);
  }
};

// Shared-memory table T[k1][n2] = w_N^(k1 n2) (k1 < N1, n2 < 32, so k1 n2 < N): in the forward
// four-step lane n2 reads T[k1][n2] for compile-time k1 -- one 64-bit load at a constant offset
// from the lane's base, conflict-free, with no index arithmetic.
struct TwTable {
  float2 *t;
  int     n; // transform length N = 32 * N1 (the table has N entries)
  __device__ __forceinline__ void fill(int tid, int nthreads) {
    for (int i = tid; i < n; i += nthreads) {
      float sv, cv;
      sincospif(-2.0f * (float)((i >> 5) * (i & 31)) / (float)n, &sv, &cv);
      t[i] = make_float2(cv, sv);
    }
  }
  template <bool INV> __device__ __forceinline__ float2 get(int k1, int n2) const {
    const float2 w = t[k1 * 32 + n2];
    return INV ? make_float2(w.x, -w.y) : w;
  }
};

// exchange-buffer geometry: [N1 rows][33 columns] per transform (33 breaks bank aliasing)
template <int N1> struct XBuf {
  static constexpr int kRow  = 33;
  static constexpr int kSize = N1 * kRow + 4; // +4 complex: decorrelates adjacent transforms
};

// Step 1-2 of the forward (or inverse) four-step for one lane: x[n1] holds sample n2 + 32*n1.
// Leaves Y[n2][k1] (twiddled) in x[k1] and writes it to xb[k1*33 + n2].
template <int N1, bool INV>
__device__ __forceinline__ void four_step_a(float2 *x, int n2, const SmemTwiddles &tw, float2 *xb) {
  dft_reg<N1, INV>(x);
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) {
    float2 v = x[k1];
    if (k1 != 0)
      v = cmul(v, tw.get<INV>((n2 * k1) % (N1 * 32)));
    xb[k1 * XBuf<N1>::kRow + n2] = v;
  }
}

// Step 3-4: lane k1 (< N1) gathers Y[0..31][k1] and leaves X[k1 + N1*k2] in y[k2].
template <int N1, bool INV>
__device__ __forceinline__ void four_step_b(float2 *y, int k1, const float2 *xb) {
#pragma unroll
  for (int n2 = 0; n2 < 32; ++n2)
    y[n2] = xb[k1 * XBuf<N1>::kRow + n2];
  dft_reg<32, INV>(y);
}

// Transposed four-step, first half: lane a (< N1) holds input j = a + N1*b in y[b] (b < 32).
// 32-point DFT over b, twiddle w_N^(a*kb), write to xb[a*33 + kb].
template <int N1, bool INV>
__device__ __forceinline__ void four_step_rev_a(float2 *y, int a, const SmemTwiddles &tw,
                                                float2 *xb) {
  dft_reg<32, INV>(y);
#pragma unroll
  for (int kb = 0; kb < 32; ++kb) {
    float2 v = y[kb];
    if (kb != 0)
      v = cmul(v, tw.get<INV>((a * kb) % (N1 * 32)));
    xb[a * XBuf<N1>::kRow + kb] = v;
  }
}

// Transposed four-step, second half: lane kb (< 32) gathers [0..N1-1][kb], N1-point DFT over a,
// leaving X[kb + 32*ka] in x[ka] — the same distribution as the forward load.
template <int N1, bool INV>
__device__ __forceinline__ void four_step_rev_b(float2 *x, int kb, const float2 *xb) {
#pragma unroll
  for (int a = 0; a < N1; ++a)
    x[a] = xb[a * XBuf<N1>::kRow + kb];
  dft_reg<N1, INV>(x);
}

// In-place variants of the forward four-step for a buffer of exactly N = 32*N1 complex values:
// the exchange uses index k1*32 + (n2 ^ k1) (an XOR swizzle instead of padding), so the same
// buffer that held the natural-order input can hold the exchange without bank conflicts.
template <int N1, bool INV>
__device__ __forceinline__ void four_step_a_sw(float2 *x, int n2, const SmemTwiddles &tw, float2 *xb) {
  dft_reg<N1, INV>(x);
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) {
    float2 v = x[k1];
    if (k1 != 0)
      v = cmul(v, tw.get<INV>((n2 * k1) % (N1 * 32)));
    xb[k1 * 32 + (n2 ^ k1)] = v;
  }
}
// The same with twiddles from a TwTable.
template <int N1, bool INV>
__device__ __forceinline__ void four_step_a_sw(float2 *x, int n2, const TwTable &tw, float2 *xb) {
  dft_reg<N1, INV>(x);
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) {
    float2 v = x[k1];
    if (k1 != 0)
      v = cmul(v, tw.get<INV>(k1, n2));
    xb[k1 * 32 + (n2 ^ k1)] = v;
  }
}
template <int N1, bool INV>
__device__ __forceinline__ void four_step_a(float2 *x, int n2, const TwTable &tw, float2 *xb) {
  dft_reg<N1, INV>(x);
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) {
    float2 v = x[k1];
    if (k1 != 0)
      v = cmul(v, tw.get<INV>(k1, n2));
    xb[k1 * XBuf<N1>::kRow + n2] = v;
  }
}
template <int N1, bool INV>
__device__ __forceinline__ void four_step_b_sw(float2 *y, int k1, const float2 *xb) {
#pragma unroll
  for (int n2 = 0; n2 < 32; ++n2)
    y[n2] = xb[k1 * 32 + (n2 ^ k1)];
  dft_reg<32, INV>(y);
}

} // namespace hf
