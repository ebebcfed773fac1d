// Shack-Hartmann autofocus (graph_builder.cc:307-501): the band planes of one spectrum are cut
// into nb x nb sub-apertures, each propagated with a one-FFT Fresnel transform
// (ShortTimeFresnelDiffraction), their magnitudes averaged over the band, and every sub-aperture
// image is phase-correlated with the centre one.  The peak offsets are wavefront slopes; a
// least-squares fit turns them into Zernike coefficients, whose phase map corrects the planes.
//
// Sub-aperture sides are W / nb with nb odd (102, 170, 204, 73, ...), which the four-step
// power-of-two passes of the Fresnel path do not cover.  This file therefore carries its own
// shared-memory FFT for any length 2 <= n <= 1024: a Stockham auto-sort sequence of stages, one
// per radix p of a factorisation of n planned on the host.
//  - Factors 4, 2, 3, 5 are merged pairwise into the composite radices 6, 8, 9, 10, 12, 15, 16
//    (one shared-memory pass and barrier fewer per pair).
//  - Primes 3..17 take register butterflies in the symmetric form; a composite radix takes a
//    register Cooley-Tukey split; any larger prime takes p-term sums per output.
// A stage of radix p over sub-transforms of span Ns reads x[j + r n/p], twiddles input r by
// w_n^(r m (j mod Ns)) with m = n / (Ns p) (the powers by recurrence from one table load), takes
// the p-point DFT and writes output q to ((j / Ns) Ns p + j mod Ns) + q Ns.  Twiddles come from
// a per-length table w_n^e built in float64 on the host; index divisions are multiply-high
// divisions by invariant integers.
//
// Kernels (the transforms are instruction- and barrier-bound, the rest memory-bound or tiny):
//  - shk_rows_kernel<MODE>: R rows of length n per CTA, gathered with the pre-operation of MODE
//    (window gather x input lens for the short-time Fresnel transform; mean removal and cosine
//    taper inside the correlation ROI; normalised cross power against the reference spectrum),
//    transformed in shared memory and stored contiguously.
//  - shk_cols_kernel<MODE>: a strip of C columns of one image, transposed into shared memory,
//    transformed along the height, with the post-operation of MODE (complex, |.|, or real part x
//    scale).
//  - shk_cols_mean_kernel: the same for the mean of |.| over the band planes, kMeanPlanes planes'
//    strips per transform, the next group's strips arriving by cp.async into a third buffer while
//    the current group is transformed, and the per-sub-aperture fftshift fused into the store.
//  - shk_roi_mean_kernel, shk_peak_kernel (first maximum + parabolic refinement, one CTA per map),
//    shk_slopes_kernel and shk_zfit_kernel (one thread each: the reference's float32 sequences),
//    shk_zernike_phase_kernel, shk_correct_phase_kernel, shk_wrap2pi_kernel.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "hf_common.cuh"
#include "k_shack.cuh"

namespace hf {
namespace {

constexpr int kShkMaxN     = 1024; // longest transform side
constexpr int kShkStages   = 16;
constexpr int kShkThreads  = 256;
constexpr int kRedThreads  = 1024; // one CTA per correlation map for the ROI mean and the peak
constexpr int kShkMaxRows  = 16;   // rows per CTA of the row pass
constexpr int kMeanPlanes  = 4;    // planes per transform in the band-mean column pass
constexpr int kShkMaxModes = 9; // Noll 2..10

// Division by a run-time invariant d as a multiply-high and a shift (Granlund and Montgomery,
// "Division by invariant integers using multiplication", 1994, round-up variant): with
// l = ceil(log2 d), m = ceil(2^(31+l) / d) < 2^32 and x < 2^31, x / d = umulhi(x, m) >> (l - 1).
struct FastDiv {
  uint32_t d, m;
  int      s;
};

FastDiv make_div(uint32_t d) {
  if (d <= 1)
    return {1u, 0u, 0};
  int l = 0;
  while ((1u << l) < d)
    ++l;
  const uint64_t p = 31 + (uint64_t)l;
  return {d, (uint32_t)(((1ull << p) + d - 1) / d), (int)(p - 32)};
}

__device__ __forceinline__ int fdiv(int x, const FastDiv &f) {
  return f.d == 1 ? x : (int)(__umulhi((uint32_t)x, f.m) >> f.s);
}

struct Stage {
  int     p, Ns, m, nb; // radix, span of the sub-transforms before the stage, n / (Ns p), n / p
  FastDiv by_nb, by_Ns, by_p;
};

struct GPlan {
  int     n, nst;
  FastDiv by_n;
  Stage   st[kShkStages];
};

bool make_plan(int n, GPlan &pl) {
  if (n < 2 || n > kShkMaxN)
    return false;
  std::memset(&pl, 0, sizeof(pl));
  pl.n = n, pl.nst = 0, pl.by_n = make_div((uint32_t)n);
  int rem = n, Ns = 1;
  auto push = [&](int p) {
    Stage &st = pl.st[pl.nst++];
    st.p = p, st.Ns = Ns, st.m = n / (Ns * p), st.nb = n / p;
    st.by_nb = make_div((uint32_t)st.nb), st.by_Ns = make_div((uint32_t)Ns), st.by_p = make_div((uint32_t)p);
    Ns *= p;
  };
  // prime-power factors first (4 before 2), then pairs of the small ones merged into one
  // register radix (6, 8, 9, 10, 12, 15, 16): one shared-memory pass and barrier fewer per pair
  std::vector<int> f;
  for (int p : {4, 2, 3, 5, 7, 11, 13, 17})
    while (rem % p == 0)
      f.push_back(p), rem /= p;
  for (int p = 19; rem > 1; p += 2)
    while (rem % p == 0)
      f.push_back(p), rem /= p;
  auto mergeable = [](int a, int b) {
    const int c = a * b;
    return (a <= 5 && b <= 5) && (c == 6 || c == 8 || c == 9 || c == 10 || c == 12 || c == 15 || c == 16);
  };
  std::vector<int> radices;
  for (size_t i = 0; i < f.size(); ++i) {
    size_t best = f.size();
    if (f[i] <= 5)
      for (size_t k = i + 1; k < f.size(); ++k)
        if (f[k] > 0 && mergeable(f[i], f[k]) && (best == f.size() || f[i] * f[k] > f[i] * f[best]))
          best = k;
    if (f[i] == 0)
      continue;
    if (best < f.size()) {
      radices.push_back(f[i] * f[best]);
      f[best] = 0;
    } else {
      radices.push_back(f[i]);
    }
  }
  if ((int)radices.size() > kShkStages)
    return false;
  for (int p : radices)
    push(p);
  return true;
}

std::vector<float2> twiddle_table(int n) {
  std::vector<float2> t((size_t)n);
  for (int e = 0; e < n; ++e) {
    const double a = -2.0 * M_PI * (double)e / (double)n;
    t[(size_t)e]   = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  return t;
}

// A transform length's plan and twiddle table in device memory (the kernels copy both into
// shared memory).
struct DevPlan {
  int     n   = 0;
  GPlan  *pl  = nullptr;
  float2 *tw  = nullptr;
};

void release(DevPlan &d) {
  cudaFree(d.pl), cudaFree(d.tw);
  d.pl = nullptr, d.tw = nullptr;
}

int dev_plan_init(DevPlan &d, int n) {
  GPlan pl;
  if (!make_plan(n, pl))
    return fail(HF_ERR_UNSUPPORTED, "autofocus: transform sides must be in 2..1024");
  d.n                         = n;
  const std::vector<float2> t = twiddle_table(n);
  HF_TRY(cuda_status(cudaMalloc(&d.pl, sizeof(GPlan)), "autofocus: plan"));
  HF_TRY(cuda_status(cudaMalloc(&d.tw, t.size() * sizeof(float2)), "autofocus: twiddles"));
  HF_TRY(cuda_status(cudaMemcpy(d.pl, &pl, sizeof(GPlan), cudaMemcpyHostToDevice), "autofocus: plan"));
  return cuda_status(cudaMemcpy(d.tw, t.data(), t.size() * sizeof(float2), cudaMemcpyHostToDevice),
                     "autofocus: twiddles");
}

__device__ __forceinline__ float2 twid(const float2 *tw, int e, bool inv) {
  const float2 w = tw[e];
  return inv ? make_float2(w.x, -w.y) : w;
}

__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}

// P-point DFT in registers.  2 and 4 take the exact butterflies; an odd P takes the symmetric form
// Y[q] = v0 + sum_r (v_r + v_{P-r}) cos(2 pi q r / P) - i sum_r (v_r - v_{P-r}) sin(2 pi q r / P),
// r = 1 .. (P-1)/2, with Y[P-q] the same with +i: ((P-1)/2)^2 complex-by-real products for both.
// cos and sin of 2 pi m / P come from the length-n table at m n / P.
template <int P> struct Split { // P = A B with A the radix taken first (0: P is 2, 4 or prime)
  static constexpr int A = P % 4 == 0 && P > 4 ? 4 : (P % 2 == 0 && P > 4 ? 2 : (P % 3 == 0 && P > 3 ? 3 : 0));
  static constexpr int B = A ? P / A : 0;
};

template <int P> __device__ __forceinline__ void dft_small(float2 (&v)[P], bool inv, const float2 *tw, int step);

// Composite P = A B in registers (Cooley-Tukey): B DFTs of length A over v[i2 + B i1], the inner
// twiddles w_P^(i2 k1) (table entries (i2 k1) n / P), A DFTs of length B; output k1 + A k2.
template <int P> __device__ __forceinline__ void dft_composite(float2 (&v)[P], bool inv, const float2 *tw, int step) {
  constexpr int A = Split<P>::A, B = Split<P>::B;
  float2        u[P];
#pragma unroll
  for (int i2 = 0; i2 < B; ++i2) {
    float2 t[A];
#pragma unroll
    for (int i1 = 0; i1 < A; ++i1)
      t[i1] = v[i2 + B * i1];
    dft_small<A>(t, inv, tw, step * B);
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1)
      u[i2 * A + k1] = (i2 == 0 || k1 == 0) ? t[k1] : cmul(t[k1], twid(tw, ((i2 * k1) % P) * step, inv));
  }
#pragma unroll
  for (int k1 = 0; k1 < A; ++k1) {
    float2 t[B];
#pragma unroll
    for (int i2 = 0; i2 < B; ++i2)
      t[i2] = u[i2 * A + k1];
    dft_small<B>(t, inv, tw, step * A);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2)
      v[k1 + A * k2] = t[k2];
  }
}

template <int P> __device__ __forceinline__ void dft_small(float2 (&v)[P], bool inv, const float2 *tw, int step) {
  if constexpr (Split<P>::A != 0) {
    dft_composite<P>(v, inv, tw, step);
  } else if constexpr (P == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b), v[1] = csub(a, b);
  } else if constexpr (P == 4) {
    const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const float2 a2 = cadd(v[1], v[3]), a3 = csub(v[1], v[3]);
    const float2 r = inv ? make_float2(-a3.y, a3.x) : make_float2(a3.y, -a3.x); // (+i or -i) a3
    v[0] = cadd(a0, a2), v[2] = csub(a0, a2);
    v[1] = cadd(a1, r), v[3] = csub(a1, r);
  } else {
    constexpr int H = (P - 1) / 2;
    float2        a[H + 1], b[H + 1];
    float         cs[H + 1], sn[H + 1];
    float2        y0 = v[0];
#pragma unroll
    for (int r = 1; r <= H; ++r) {
      a[r] = cadd(v[r], v[P - r]), b[r] = csub(v[r], v[P - r]);
      y0   = cadd(y0, a[r]);
      const float2 w = tw[r * step]; // (cos, -sin) of 2 pi r / P
      cs[r] = w.x, sn[r] = -w.y;
    }
    float2 out[P];
    out[0] = y0;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      float2 sc = v[0], ss = make_float2(0.f, 0.f);
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        const int   mm = (q * r) % P;
        const float c  = mm <= H ? cs[mm] : cs[P - mm];
        const float sv = mm <= H ? sn[mm] : -sn[P - mm];
        sc.x = fmaf(a[r].x, c, sc.x), sc.y = fmaf(a[r].y, c, sc.y);
        ss.x = fmaf(b[r].x, sv, ss.x), ss.y = fmaf(b[r].y, sv, ss.y);
      }
      const float2 yq = make_float2(sc.x + ss.y, sc.y - ss.x); // sc - i ss
      const float2 yp = make_float2(sc.x - ss.y, sc.y + ss.x); // sc + i ss
      out[q]     = inv ? yp : yq;
      out[P - q] = inv ? yq : yp;
    }
#pragma unroll
    for (int q = 0; q < P; ++q)
      v[q] = out[q];
  }
}

// Odd P: the symmetric form of dft_small, with the inputs folded into a_r = v_r + v_(P-r) and
// b_r = v_r - v_(P-r) as they are loaded (the twiddle of input P - r is w^P conj(w^r)) and each
// output pair stored as soon as it is formed, so no P-element array stays live.
template <int P>
__device__ void stage_bfly_odd(const float2 *x, float2 *y, int pitch, int rows, const Stage &st, const float2 *tw,
                               int n, bool inv) {
  constexpr int H  = (P - 1) / 2;
  const int     nb = st.nb, Ns = st.Ns, total = rows * nb, step = n / P;
  float         cs[H + 1], sn[H + 1];
#pragma unroll
  for (int r = 1; r <= H; ++r) {
    const float2 w = tw[r * step]; // (cos, -sin) of 2 pi r / P
    cs[r] = w.x, sn[r] = -w.y;
  }
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int     row = fdiv(t, st.by_nb), j = t - row * nb;
    const int     jb = fdiv(j, st.by_Ns), k = j - jb * Ns;
    const int     e  = st.m * k;
    const float2 *xr = x + row * pitch;
    float2       *yr = y + row * pitch;
    const float2  v0 = xr[j];
    float2        a[H + 1], b[H + 1];
    float2        y0 = v0;
    if (e > 0) {
      const float2 w1 = twid(tw, e, inv);
      float2       wr = w1, wh = w1;
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        if (r > 1)
          wr = cmul(wr, w1);
        if (r == H)
          wh = wr;
        a[r] = cmul(xr[j + r * nb], wr);
      }
      const float2 wp = cmul(cmul(wh, wh), w1); // w^P
      wr              = w1;
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        if (r > 1)
          wr = cmul(wr, w1);
        const float2 u = cmul(xr[j + (P - r) * nb], cmul(wp, make_float2(wr.x, -wr.y)));
        b[r]           = csub(a[r], u);
        a[r]           = cadd(a[r], u);
        y0             = cadd(y0, a[r]);
      }
    } else {
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        const float2 vr = xr[j + r * nb], vp = xr[j + (P - r) * nb];
        a[r] = cadd(vr, vp), b[r] = csub(vr, vp);
        y0   = cadd(y0, a[r]);
      }
    }
    const int base = jb * Ns * P + k;
    yr[base]       = y0;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      float2 sc = v0, ss = make_float2(0.f, 0.f);
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        const int   mm = (q * r) % P;
        const float c  = mm <= H ? cs[mm] : cs[P - mm];
        const float sv = mm <= H ? sn[mm] : -sn[P - mm];
        sc.x = fmaf(a[r].x, c, sc.x), sc.y = fmaf(a[r].y, c, sc.y);
        ss.x = fmaf(b[r].x, sv, ss.x), ss.y = fmaf(b[r].y, sv, ss.y);
      }
      const float2 yq = make_float2(sc.x + ss.y, sc.y - ss.x); // sc - i ss
      const float2 yp = make_float2(sc.x - ss.y, sc.y + ss.x); // sc + i ss
      yr[base + q * Ns]       = inv ? yp : yq;
      yr[base + (P - q) * Ns] = inv ? yq : yp;
    }
  }
}

template <int P>
__device__ void stage_bfly(const float2 *x, float2 *y, int pitch, int rows, const Stage &st, const float2 *tw, int n,
                           bool inv) {
  if constexpr (P % 2 == 1 && Split<P>::A == 0) {
    stage_bfly_odd<P>(x, y, pitch, rows, st, tw, n, inv);
    return;
  }
  const int nb = st.nb, Ns = st.Ns, total = rows * nb, step = n / P;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int     row = fdiv(t, st.by_nb), j = t - row * nb;
    const int     jb = fdiv(j, st.by_Ns), k = j - jb * Ns;
    const int     e  = st.m * k; // twiddle of input r: w_n^(r m k) = (w_n^(m k))^r
    const float2 *xr = x + row * pitch;
    float2       *yr = y + row * pitch;
    float2        v[P];
#pragma unroll
    for (int r = 0; r < P; ++r)
      v[r] = xr[j + r * nb];
    if (e > 0) {
      const float2 w1 = twid(tw, e, inv);
      float2       wr = w1;
#pragma unroll
      for (int r = 1; r < P; ++r) {
        v[r] = cmul(v[r], wr);
        if (r + 1 < P)
          wr = cmul(wr, w1);
      }
    }
    dft_small<P>(v, inv, tw, step);
    const int base = jb * Ns * P + k;
#pragma unroll
    for (int q = 0; q < P; ++q)
      yr[base + q * Ns] = v[q];
  }
}

// Any radix: one p-term sum per output, the exponent stepped by s = m (k + q Ns) modulo n.
__device__ void stage_generic(const float2 *x, float2 *y, int pitch, int rows, const Stage &st, const FastDiv &by_n,
                              const float2 *tw, int n, bool inv) {
  const int p = st.p, nb = st.nb, Ns = st.Ns;
  for (int t = threadIdx.x; t < rows * n; t += blockDim.x) {
    const int     row = fdiv(t, by_n), o = t - row * n;
    const int     on = fdiv(o, st.by_Ns), k = o - on * Ns;
    const int     jb = fdiv(on, st.by_p), q = on - jb * p;
    const int     j  = jb * Ns + k;
    const int     s  = st.m * (k + q * Ns); // < n
    const float2 *xr = x + row * pitch;
    float2        acc = make_float2(0.f, 0.f);
    int           e   = 0;
    for (int r = 0; r < p; ++r) {
      acc = cfma(xr[j + r * nb], twid(tw, e, inv), acc);
      e += s;
      if (e >= n)
        e -= n;
    }
    y[row * pitch + o] = acc;
  }
}

// Transforms `rows` rows of `a` (pitch `pitch`), ping-ponging with `b`; returns the buffer that
// holds the result.  Every thread of the CTA calls it; the rows must be in `a` and visible.
__device__ float2 *fft_rows_smem(float2 *a, float2 *b, int pitch, int rows, const GPlan &pl, const float2 *tw, bool inv) {
  for (int s = 0; s < pl.nst; ++s) {
    const Stage &st = pl.st[s];
    switch (st.p) {
    case 2: stage_bfly<2>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 3: stage_bfly<3>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 4: stage_bfly<4>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 5: stage_bfly<5>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 7: stage_bfly<7>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 11: stage_bfly<11>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 13: stage_bfly<13>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 17: stage_bfly<17>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 6: stage_bfly<6>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 8: stage_bfly<8>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 9: stage_bfly<9>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 10: stage_bfly<10>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 12: stage_bfly<12>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 15: stage_bfly<15>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    case 16: stage_bfly<16>(a, b, pitch, rows, st, tw, pl.n, inv); break;
    default: stage_generic(a, b, pitch, rows, st, pl.by_n, tw, pl.n, inv); break;
    }
    __syncthreads();
    float2 *t = a;
    a = b, b = t;
  }
  return a;
}

// ------------------------------------------------------------------------------------------------
// Row pass
// ------------------------------------------------------------------------------------------------
enum RowMode { ROW_STFD = 0, ROW_XPACK = 1, ROW_CROSS = 2, ROW_PAIR = 3 };

struct Roi {
  float cx, cy, rx, ry, c, s; // c, s: cos and sin of the angle
};

__device__ __forceinline__ float roi_sq_distance(int x, int y, int w, int h, const Roi &r) {
  const float xn = ((float)x + 0.5f) / (float)w, yn = ((float)y + 0.5f) / (float)h;
  const float dx = xn - r.cx, dy = yn - r.cy;
  const float xr = r.c * dx + r.s * dy, yr = -r.s * dx + r.c * dy;
  return (xr * xr) / (r.rx * r.rx) + (yr * yr) / (r.ry * r.ry);
}

struct RowArgs {
  const GPlan  *pl;       // device copy of the transform plan along the row
  int           n;        // row length
  const float2 *tw;       // [n]
  int           R;        // rows per CTA
  int64_t       n_rows;   // rows in all
  bool          inv;
  float2       *out;      // [n_rows][n]
  // ROW_STFD: field [planes][H][W] (real or complex) -> rows (plane, gy, gx, j)
  const void   *field;
  int           real_in, H, W, win_h, nwx, nwy, stride_y, stride_x, global_lens;
  const float2 *lens; // [H][W] (global) or [win_h][n] (local)
  // ROW_XPACK: images [n_img][h][n] float; ROW_CROSS: spectra [n_img][h][n] complex
  const float  *img;
  const float  *means; // [n_img]
  const float  *taper; // [h][n]: the ROI's cosine taper, -1 outside
  int           h;
  const float2 *spec;
  int           ref_img;
  // ROW_PAIR: map m of the batch is pair pair0 + m, moving image pair_src, reference pair_dst
  const int    *pair_src, *pair_dst;
  int64_t       pair0;
};

template <int MODE> __global__ void __launch_bounds__(kShkThreads, 4) shk_rows_kernel(RowArgs a) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ GPlan spl;
  const int        n  = a.n;
  float2          *tw = sm, *b0 = sm + n, *b1 = b0 + (size_t)a.R * n;
  for (int e = threadIdx.x; e < n; e += blockDim.x)
    tw[e] = a.tw[e];
  for (int i = threadIdx.x; i < (int)(sizeof(GPlan) / 4); i += blockDim.x)
    reinterpret_cast<int *>(&spl)[i] = reinterpret_cast<const int *>(a.pl)[i];
  const int64_t row0 = (int64_t)blockIdx.x * a.R;
  const int     rows = (int)min((int64_t)a.R, a.n_rows - row0);
  // per-row decode once (64-bit divisions), then per element only the row / column split
  __shared__ int64_t s_off[kShkMaxRows], s_aux[kShkMaxRows];
  __shared__ int     s_y[kShkMaxRows];
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    const int64_t row = row0 + r;
    if constexpr (MODE == ROW_STFD) {
      int64_t   rem = row;
      const int j   = (int)(rem % a.win_h);
      rem /= a.win_h;
      const int gx = (int)(rem % a.nwx);
      rem /= a.nwx;
      const int     gy = (int)(rem % a.nwy);
      const int64_t pl = rem / a.nwy;
      const int     fy = gy * a.stride_y + j, fx = gx * a.stride_x;
      s_off[r] = (pl * a.H + fy) * (int64_t)a.W + fx;                                  // field row start
      s_aux[r] = a.global_lens ? (int64_t)fy * a.W + fx : (int64_t)j * n;              // lens row start
    } else if constexpr (MODE == ROW_PAIR) {
      const int64_t m = row / a.h, pr = a.pair0 + m;
      s_y[r]   = (int)(row - m * a.h);
      s_off[r] = ((int64_t)a.pair_src[pr] * a.h + s_y[r]) * n; // the moving image's row
      s_aux[r] = ((int64_t)a.pair_dst[pr] * a.h + s_y[r]) * n; // the reference's row
    } else {
      const int64_t im = row / a.h;
      s_y[r]   = (int)(row - im * a.h);
      s_off[r] = im;
      s_aux[r] = ((int64_t)a.ref_img * a.h + s_y[r]) * n; // ROW_CROSS: the reference's row
    }
  }
  __syncthreads();
  // U independent global loads in flight per thread before any is used
  constexpr int U = 8;
  for (int t0 = threadIdx.x; t0 < rows * n; t0 += U * blockDim.x) {
    float2 ld[U], aux[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t >= rows * n)
        break;
      const int     r = fdiv(t, spl.by_n), i = t - r * n;
      const int64_t row = row0 + r;
      if constexpr (MODE == ROW_STFD) {
        const int64_t src = s_off[r] + i;
        ld[u]  = a.real_in ? make_float2(static_cast<const float *>(a.field)[src], 0.f)
                           : static_cast<const float2 *>(a.field)[src];
        aux[u] = a.lens[s_aux[r] + i];
      } else if constexpr (MODE == ROW_XPACK) {
        ld[u] = make_float2(a.img[row * n + i], 0.f);
      } else if constexpr (MODE == ROW_PAIR) {
        ld[u]  = a.spec[s_off[r] + i];
        aux[u] = a.spec[s_aux[r] + i];
      } else {
        ld[u]  = a.spec[row * n + i];
        aux[u] = a.spec[s_aux[r] + i];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t >= rows * n)
        break;
      float2 v;
      if constexpr (MODE == ROW_STFD) {
        v = cmul(ld[u], aux[u]);
      } else if constexpr (MODE == ROW_XPACK) {
        const int   r = fdiv(t, spl.by_n), i = t - r * n;
        const float tp = a.taper[(int64_t)s_y[r] * n + i];
        // (v - mean) * 0.5 (1 + cos(pi sqrt(d))) inside the ellipse, 0 outside
        v = make_float2(tp >= 0.f ? (ld[u].x - a.means[s_off[r]]) * tp : 0.f, 0.f);
      } else { // ROW_CROSS / ROW_PAIR: unit-magnitude cross power moving x conj(reference)
        const float2 mv = ld[u], rf = aux[u];
        const float2 p   = make_float2(mv.x * rf.x + mv.y * rf.y, mv.y * rf.x - mv.x * rf.y);
        const float  mag = sqrtf(p.x * p.x + p.y * p.y);
        v                = mag <= 1e-12f ? make_float2(0.f, 0.f) : make_float2(p.x / mag, p.y / mag);
      }
      b0[t] = v;
    }
  }
  __syncthreads();
  const float2 *res = fft_rows_smem(b0, b1, n, rows, spl, tw, a.inv);
  for (int t = threadIdx.x; t < rows * n; t += blockDim.x)
    a.out[row0 * n + t] = res[t];
}

// ------------------------------------------------------------------------------------------------
// Column pass
// ------------------------------------------------------------------------------------------------
enum ColMode { COL_COMPLEX = 0, COL_MAG = 1, COL_MEAN_MAG = 2, COL_REAL = 3 };

struct ColArgs {
  const GPlan  *pl; // device copy of the transform plan along the column
  int           h;  // column length
  const float2 *tw; // [h]
  int           C, pitch, nstrip, w;
  bool          inv;
  const float2 *in;   // [images][h][w]
  float2       *outc; // COL_COMPLEX (may equal in)
  float        *outf; // COL_MAG, COL_MEAN_MAG, COL_REAL
  const float2 *post; // COL_COMPLEX: optional [h][w] factor (window lens)
  int           planes;  // COL_MEAN_MAG: planes averaged; image = plane * nwin + window
  int64_t       nwin;
  int           shift;   // COL_MEAN_MAG: fftshift of every image on store
  float         scale;   // COL_REAL
  FastDiv       by_hc;   // h C (plane index of a strip element)
};

// One image's strip (COL_COMPLEX, COL_MAG, COL_REAL): loads, transform, post-operation.
template <int MODE> __global__ void __launch_bounds__(kShkThreads, 3) shk_cols_kernel(ColArgs a) {
  static_assert(MODE != COL_MEAN_MAG, "the band mean runs in shk_cols_mean_kernel");
  extern __shared__ __align__(16) float2 sm[];
  __shared__ GPlan spl;
  const int h = a.h, C = a.C, P = a.pitch;
  float2   *tw = sm, *b0 = sm + h, *b1 = b0 + (size_t)C * P;
  for (int e = threadIdx.x; e < h; e += blockDim.x)
    tw[e] = a.tw[e];
  for (int i = threadIdx.x; i < (int)(sizeof(GPlan) / 4); i += blockDim.x)
    reinterpret_cast<int *>(&spl)[i] = reinterpret_cast<const int *>(a.pl)[i];
  const int     strip = (int)(blockIdx.x % a.nstrip);
  const int64_t img   = blockIdx.x / a.nstrip;
  const int     x0 = strip * C, cw = min(C, a.w - x0);
  const int     lc = 31 - __clz(C); // C is a power of two
  constexpr int U  = 8;             // independent loads in flight per thread
  for (int t0 = threadIdx.x; t0 < h * C; t0 += U * blockDim.x) {
    float2 ld[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t >= h * C)
        break;
      const int y = t >> lc, c = t & (C - 1);
      ld[u] = c < cw ? a.in[(img * h + y) * (int64_t)a.w + x0 + c] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t >= h * C)
        break;
      const int y = t >> lc, c = t & (C - 1);
      b0[c * P + y] = ld[u];
    }
  }
  __syncthreads();
  const float2 *res = fft_rows_smem(b0, b1, P, C, spl, tw, a.inv);
  for (int t = threadIdx.x; t < h * C; t += blockDim.x) {
    const int y = t >> lc, c = t & (C - 1);
    if (c >= cw)
      continue;
    const float2  v = res[c * P + y];
    const int64_t o = (img * h + y) * (int64_t)a.w + x0 + c;
    if constexpr (MODE == COL_COMPLEX)
      a.outc[o] = a.post ? cmul(v, a.post[(int64_t)y * a.w + x0 + c]) : v;
    else if constexpr (MODE == COL_MAG)
      a.outf[o] = sqrtf(v.x * v.x + v.y * v.y);
    else
      a.outf[o] = v.x * a.scale;
  }
}

__device__ __forceinline__ void cp_async8(float2 *dst, const float2 *src, bool ok) {
  // src-size 0 fills the 8 bytes with zeros (columns past the image edge)
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(ok ? 8 : 0)
               : "memory");
}

// The band-mean column pass (COL_MEAN_MAG) with its loads overlapped: each group of kMeanPlanes
// planes' strips arrives by cp.async into a third buffer while the previous group is transformed
// and accumulated.  |.| = sqrtf(x^2 + y^2) summed in band order in float32, then divided by the
// plane count.
__global__ void __launch_bounds__(kShkThreads, 2) shk_cols_mean_kernel(ColArgs a) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ GPlan spl;
  constexpr int G  = kMeanPlanes;
  const int     h = a.h, C = a.C, P = a.pitch;
  float2       *tw = sm, *bx = sm + h, *b1 = bx + (size_t)G * C * P, *by = b1 + (size_t)G * C * P;
  float        *acc = reinterpret_cast<float *>(by + (size_t)G * C * P); // [h * C]
  for (int e = threadIdx.x; e < h; e += blockDim.x)
    tw[e] = a.tw[e];
  for (int i = threadIdx.x; i < (int)(sizeof(GPlan) / 4); i += blockDim.x)
    reinterpret_cast<int *>(&spl)[i] = reinterpret_cast<const int *>(a.pl)[i];
  const int     strip = (int)(blockIdx.x % a.nstrip);
  const int64_t img   = blockIdx.x / a.nstrip;
  const int     x0 = strip * C, cw = min(C, a.w - x0);
  const int     lc = 31 - __clz(C); // C is a power of two
  for (int t = threadIdx.x; t < h * C; t += blockDim.x)
    acc[t] = 0.f;
  // the strip of plane g of a group sits at rows [g C, g C + C) of a buffer, transposed
  const auto issue = [&](int pl, float2 *dst) {
    const int ng = min(G, a.planes - pl);
    for (int t = threadIdx.x; t < ng * h * C; t += blockDim.x) {
      const int     g = fdiv(t, a.by_hc), r = t - g * h * C, y = r >> lc, c = r & (C - 1);
      const int64_t src = (int64_t)(pl + g) * a.nwin + img;
      const bool    ok  = c < cw;
      cp_async8(dst + (g * C + c) * P + y, a.in + (src * h + y) * (int64_t)a.w + x0 + (ok ? c : 0), ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  float2 *cur = bx, *spare = by;
  issue(0, cur);
  for (int pl = 0; pl < a.planes; pl += G) {
    const int ng = min(G, a.planes - pl);
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads(); // every thread's copies of this group have landed
    if (pl + G < a.planes)
      issue(pl + G, spare); // the next group streams in during this group's transforms
    const float2 *res = fft_rows_smem(cur, b1, P, ng * C, spl, tw, a.inv);
    for (int t = threadIdx.x; t < h * C; t += blockDim.x) {
      const int y = t >> lc, c = t & (C - 1);
      if (c >= cw)
        continue;
      const float2 v = res[c * P + y];
      float        s = acc[t] + sqrtf(v.x * v.x + v.y * v.y); // band order, float32
#pragma unroll
      for (int g = 1; g < G; ++g)
        if (g < ng) {
          const float2 u = res[(g * C + c) * P + y];
          s += sqrtf(u.x * u.x + u.y * u.y);
        }
      acc[t] = s;
    }
    __syncthreads(); // this group's buffers are read: `cur` takes the copies after next
    float2 *tmp = cur;
    cur         = spare;
    spare       = tmp;
  }
  const float nz = (float)a.planes;
  for (int t = threadIdx.x; t < h * C; t += blockDim.x) {
    const int y = t >> lc, c = t & (C - 1);
    if (c >= cw)
      continue;
    const int yy = a.shift ? (y + h / 2) % h : y;
    const int xx = a.shift ? (x0 + c + a.w / 2) % a.w : x0 + c;
    a.outf[(img * h + yy) * (int64_t)a.w + xx] = acc[t] / nz;
  }
}

size_t rows_smem(int n, int R) { return (size_t)n * sizeof(float2) * (1 + 2 * (size_t)R); }
int    rows_per_cta(int n) { return std::max(1, std::min(kShkMaxRows, 4096 / n)); }
int    col_strip(int h, bool mean) {
  const int c = h <= 256 ? 16 : (h <= 512 ? 8 : 4);
  return mean ? std::max(1, c / kMeanPlanes) : c; // the mean pass holds kMeanPlanes planes' strips
}
size_t cols_smem(int h, int C, bool mean) {
  const int P = h | 1; // odd pitch: the transposed loads spread over the banks
  const int G = mean ? kMeanPlanes : 1;
  // the band-mean pass holds a third buffer for the group in flight
  return (size_t)h * sizeof(float2) + (mean ? 3 : 2) * (size_t)G * C * P * sizeof(float2) +
         (mean ? (size_t)h * C * sizeof(float) : 0);
}

template <int MODE> int launch_rows(RowArgs a, cudaStream_t s) {
  a.R             = rows_per_cta(a.n);
  const size_t sm = rows_smem(a.n, a.R);
  HF_CUDA(cudaFuncSetAttribute(shk_rows_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int64_t grid = (a.n_rows + a.R - 1) / a.R;
  if (grid > INT_MAX)
    return fail(HF_ERR_UNSUPPORTED, "short-time Fresnel: too many rows");
  shk_rows_kernel<MODE><<<(unsigned)grid, kShkThreads, sm, s>>>(a);
  note_launch();
  return launch_status("shk_rows_kernel");
}

template <int MODE> int launch_cols(ColArgs a, int64_t images, cudaStream_t s) {
  a.C             = col_strip(a.h, MODE == COL_MEAN_MAG);
  a.pitch         = a.h | 1;
  a.nstrip        = (a.w + a.C - 1) / a.C;
  a.by_hc         = make_div((uint32_t)(a.h * a.C));
  const size_t sm = cols_smem(a.h, a.C, MODE == COL_MEAN_MAG);
  const int64_t grid = images * a.nstrip;
  if (grid > INT_MAX)
    return fail(HF_ERR_UNSUPPORTED, "short-time Fresnel: too many column strips");
  if constexpr (MODE == COL_MEAN_MAG) {
    HF_CUDA(cudaFuncSetAttribute(shk_cols_mean_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    shk_cols_mean_kernel<<<(unsigned)grid, kShkThreads, sm, s>>>(a);
    note_launch();
    return launch_status("shk_cols_mean_kernel");
  } else {
    HF_CUDA(cudaFuncSetAttribute(shk_cols_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    shk_cols_kernel<MODE><<<(unsigned)grid, kShkThreads, sm, s>>>(a);
    note_launch();
    return launch_status("shk_cols_kernel");
  }
}

// ------------------------------------------------------------------------------------------------
// Lenses
// ------------------------------------------------------------------------------------------------
// stft_input_phase_kernel (short_time_fresnel_diffraction.cu:320-333): float32 phase
// pi / (lambda z) (x^2 + y^2) with x = col dx + x_origin, each operation rounded on its own (no
// contraction), as the lens of the Fresnel path.
__global__ void shk_input_lens_kernel(float2 *lens, int w, int h, float dx, float dy, float x0, float y0, float k) {
  const int64_t n = (int64_t)w * h;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int   col = (int)(i % w), row = (int)(i / w);
    const float x = __fadd_rn(__fmul_rn((float)col, dx), x0), y = __fadd_rn(__fmul_rn((float)row, dy), y0);
    float       sv, cv;
    sincosf(__fmul_rn(k, __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y))), &sv, &cv);
    lens[i] = make_float2(cv, sv);
  }
}

// stft_win_lens_kernel (short_time_fresnel_diffraction.cu:405-420): the output-plane lens of one
// window, pitch dx on both axes.
__global__ void shk_window_lens_kernel(float2 *lens, int w, int h, float lambda, float z, float dx) {
  const int64_t n = (int64_t)w * h;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int   col = (int)(i % w), row = (int)(i / w);
    const int   size = w > h ? w : h, ox = (size - w) / 2, oy = (size - h) / 2;
    const float x  = __fmul_rn((float)(col + ox) - (float)size / 2.0f, dx);
    const float y  = __fmul_rn((float)(row + oy) - (float)size / 2.0f, dx);
    const float ph = __fmul_rn(3.14159265358979f / (lambda * z), __fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)));
    float       sv, cv;
    sincosf(ph, &sv, &cv);
    lens[i] = make_float2(cv, sv);
  }
}

int grid_1d(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

// ------------------------------------------------------------------------------------------------
// Correlation helpers
// ------------------------------------------------------------------------------------------------
// compute_means_kernel (cross_correlation2.cu:352-402): mean of the pixels inside the ROI, 0 when
// none is.
// The correlation ROI of every image, once per operator: the cosine taper
// 0.5 (1 + cos(pi sqrt(d))) where the normalised elliptical distance d <= 1, -1 outside (the taper
// is >= 0 inside, so the sign is the mask).  The same float32 expressions as evaluated per element
// before, so the masked mean and the tapered images are unchanged.
__global__ void shk_roi_taper_kernel(float *taper, int h, int w, Roi roi) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)h * w; i += (int64_t)gridDim.x * blockDim.x) {
    const int   y = (int)(i / w), x = (int)(i - (int64_t)y * w);
    const float d = roi_sq_distance(x, y, w, h, roi);
    taper[i]      = d <= 1.0f ? 0.5f * (1.0f + cospif(sqrtf(d))) : -1.0f;
  }
}

// Mean of each image over the ROI (the taper's mask), one CTA per image.
__global__ void __launch_bounds__(kRedThreads) shk_roi_mean_kernel(const float *img, float *means, int h, int w,
                                                                    const float *taper) {
  const float *im = img + (int64_t)blockIdx.x * h * w;
  const int    N = h * w, B = blockDim.x;
  float        sum = 0.f;
  int          cnt = 0;
  int          i   = threadIdx.x;
  for (; i + 3 * B < N; i += 4 * B) { // four elements' loads in flight, summed in index order
    float tp[4], v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      tp[u] = taper[i + u * B], v[u] = im[i + u * B];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (tp[u] >= 0.f) {
        sum += v[u];
        ++cnt;
      }
  }
  for (; i < N; i += B) {
    if (taper[i] >= 0.f) {
      sum += im[i];
      ++cnt;
    }
  }
  __shared__ float ss[kRedThreads];
  __shared__ int   sc[kRedThreads];
  ss[threadIdx.x] = sum, sc[threadIdx.x] = cnt;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      ss[threadIdx.x] += ss[threadIdx.x + st], sc[threadIdx.x] += sc[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    means[blockIdx.x] = sc[0] > 0 ? ss[0] / (float)sc[0] : 0.f;
}

__device__ __forceinline__ float parabolic(float vm, float v0, float vp) {
  const float den = vm - 2.0f * v0 + vp;
  return fabsf(den) <= 1e-9f ? 0.0f : 0.5f * (vm - vp) / den;
}

__device__ __forceinline__ float signed_coord(int p, int n) { return p < (n + 1) / 2 ? (float)p : (float)p - (float)n; }

// recover_phase_correlation_peaks (shack_hartmann_slopes.cu:124-158): the first maximum in
// row-major order (a strict > scan), found here by a block reduction that keeps the smaller
// index among equal values; then the parabolic refinement on the circular neighbours.
// (value, index) of the larger value, the smaller index among equal values (INT_MAX: none yet)
__device__ __forceinline__ void peak_combine(float &v, int &i, float v2, int i2) {
  if (i2 != INT_MAX && (i == INT_MAX || v2 > v || (v2 == v && i2 < i)))
    v = v2, i = i2;
}

__global__ void __launch_bounds__(kRedThreads) shk_peak_kernel(const float *maps, float2 *shifts, int h, int w) {
  const float *m    = maps + (int64_t)blockIdx.x * h * w;
  const int    N    = h * w, B = blockDim.x;
  float        best = -FLT_MAX;
  int          bi   = INT_MAX;
  int          i    = threadIdx.x;
  for (; i + 3 * B < N; i += 4 * B) { // four loads in flight, compared in index order
    float v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      v[u] = m[i + u * B];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (v[u] > best)
        best = v[u], bi = i + u * B;
  }
  for (; i < N; i += B) {
    const float v = m[i];
    if (v > best)
      best = v, bi = i;
  }
  // the rule picks the same (value, index) in any combining order
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    peak_combine(best, bi, __shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, bi, o));
  __shared__ float sv[kRedThreads / 32];
  __shared__ int   si[kRedThreads / 32];
  if ((threadIdx.x & 31) == 0)
    sv[threadIdx.x >> 5] = best, si[threadIdx.x >> 5] = bi;
  __syncthreads();
  if (threadIdx.x < 32) {
    best = threadIdx.x < B / 32 ? sv[threadIdx.x] : -FLT_MAX;
    bi   = threadIdx.x < B / 32 ? si[threadIdx.x] : INT_MAX;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      peak_combine(best, bi, __shfl_xor_sync(0xffffffffu, best, o), __shfl_xor_sync(0xffffffffu, bi, o));
    if (threadIdx.x == 0)
      si[0] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int p  = si[0] == INT_MAX ? 0 : si[0];
    const int py = p / w, px = p - py * w;
    const int xm = (px + w - 1) % w, xp = (px + 1) % w, ym = (py + h - 1) % h, yp = (py + 1) % h;
    const float dxs = parabolic(m[py * w + xm], m[py * w + px], m[py * w + xp]);
    const float dys = parabolic(m[ym * w + px], m[py * w + px], m[yp * w + px]);
    shifts[blockIdx.x] = make_float2(signed_coord(px, w) + dxs, signed_coord(py, h) + dys);
  }
}

// FullPairwise: the shifts of a batch of pairs, scaled to slopes, added to rhs[src] and
// subtracted from rhs[dst] (accumulate_complete_graph_rhs, shack_hartmann_slopes_full_pairwise.cuh:
// 223-239).  One thread in pair order, so the float32 sums do not depend on scheduling.
__global__ void shk_pair_rhs_kernel(const float2 *shifts, const int *src, const int *dst, int64_t pair0, int npairs,
                                    float2 *rhs, float sppx, float sppy) {
  if (blockIdx.x != 0 || threadIdx.x != 0)
    return;
  for (int m = 0; m < npairs; ++m) {
    const float sx = shifts[m].x * sppx, sy = shifts[m].y * sppy;
    float2     &a = rhs[src[pair0 + m]], &b = rhs[dst[pair0 + m]];
    a.x += sx, a.y += sy;
    b.x -= sx, b.y -= sy;
  }
}

// The complete-graph Laplacian solve in the zero-mean gauge (solve_complete_graph_and_scatter,
// shack_hartmann_slopes_full_pairwise.cuh:241-262): slope_i = rhs_i / N - mean_k (rhs_k / N) over
// the N active samples, in the reference's float32 order; inactive samples are 0.
__global__ void shk_pair_solve_kernel(const float2 *rhs, const int *active_dense, int nact, int count, float *slopes) {
  if (blockIdx.x != 0 || threadIdx.x != 0)
    return;
  const float fn = (float)nact;
  float       mx = 0.f, my = 0.f;
  for (int i = 0; i < nact; ++i) {
    mx += rhs[i].x / fn;
    my += rhs[i].y / fn;
  }
  mx /= fn, my /= fn;
  for (int i = 0; i < 2 * count; ++i)
    slopes[i] = 0.f;
  for (int i = 0; i < nact; ++i) {
    const int d       = active_dense[i];
    slopes[2 * d]     = rhs[i].x / fn - mx;
    slopes[2 * d + 1] = rhs[i].y / fn - my;
  }
}

// recover_zero_mean_slopes (shack_hartmann_slopes.cu:160-192), one thread, same sums in order.
__global__ void shk_slopes_kernel(const float2 *shifts, const uint8_t *active, float *slopes, int count, int center,
                                  float sppx, float sppy) {
  if (blockIdx.x != 0 || threadIdx.x != 0)
    return;
  const float2 b  = shifts[center];
  float        sx = 0.f, sy = 0.f;
  int          na = 0;
  for (int i = 0; i < count; ++i) {
    if (!active[i])
      continue;
    sx += (shifts[i].x - b.x) * sppx;
    sy += (shifts[i].y - b.y) * sppy;
    ++na;
  }
  const float mx = sx / (float)na, my = sy / (float)na;
  for (int i = 0; i < count; ++i) {
    if (active[i]) {
      slopes[2 * i]     = (shifts[i].x - b.x) * sppx - mx;
      slopes[2 * i + 1] = (shifts[i].y - b.y) * sppy - my;
    } else {
      slopes[2 * i] = slopes[2 * i + 1] = 0.f;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Zernike fit, phase and correction
// ------------------------------------------------------------------------------------------------
struct ZFit {
  int   count, nobs, nidx;
  int   pos[kShkMaxModes];                   // output position of observable mode m
  float gtg[kShkMaxModes][kShkMaxModes];     // normal matrix (ridge included), built on the host
  float rad_per_m;
};

// The data-dependent half of ZernikeFromSlopes::execute (zernike_from_slopes.cc:246-277) in one
// thread, with the host's float32 operations made explicit (no contraction) so that the result is
// the reference's bit for bit: gts[i] += gx_i sx + gy_i sy over the active samples in row-major
// order, then Gaussian elimination with partial pivoting and back substitution.
__device__ void zfit_solve(const ZFit &z, const float *g, const float *slopes, float *coeffs) {
  float m[kShkMaxModes][kShkMaxModes], rhs[kShkMaxModes], sol[kShkMaxModes];
  const int n = z.nobs;
  for (int i = 0; i < n; ++i) {
    rhs[i] = 0.f, sol[i] = 0.f;
    for (int j = 0; j < n; ++j)
      m[i][j] = z.gtg[i][j];
  }
  for (int s = 0; s < z.count; ++s) {
    const float *gs = g + (size_t)s * 2 * kShkMaxModes; // [gx[0..8], gy[0..8]] (mean removed); NaN marks inactive
    if (isnan(gs[0]) && n > 0)
      continue;
    const float sx = slopes[2 * s], sy = slopes[2 * s + 1];
    for (int i = 0; i < n; ++i)
      rhs[i] = __fadd_rn(rhs[i], __fadd_rn(__fmul_rn(gs[i], sx), __fmul_rn(gs[kShkMaxModes + i], sy)));
  }
  bool singular = false;
  for (int c = 0; c < n && !singular; ++c) {
    int   piv = c;
    float bv  = fabsf(m[c][c]);
    for (int r = c + 1; r < n; ++r)
      if (fabsf(m[r][c]) > bv)
        bv = fabsf(m[r][c]), piv = r;
    if (bv < 1e-12f) {
      singular = true;
      break;
    }
    if (piv != c) {
      for (int j = 0; j < n; ++j) {
        const float t = m[piv][j];
        m[piv][j] = m[c][j], m[c][j] = t;
      }
      const float t = rhs[piv];
      rhs[piv] = rhs[c], rhs[c] = t;
    }
    const float pv = m[c][c];
    for (int j = c; j < n; ++j)
      m[c][j] = __fdiv_rn(m[c][j], pv);
    rhs[c] = __fdiv_rn(rhs[c], pv);
    for (int r = c + 1; r < n; ++r) {
      const float f = m[r][c];
      for (int j = c; j < n; ++j)
        m[r][j] = __fsub_rn(m[r][j], __fmul_rn(f, m[c][j]));
      rhs[r] = __fsub_rn(rhs[r], __fmul_rn(f, rhs[c]));
    }
  }
  if (!singular)
    for (int r = n - 1; r >= 0; --r) {
      float v = rhs[r];
      for (int c = r + 1; c < n; ++c)
        v = __fsub_rn(v, __fmul_rn(m[r][c], sol[c]));
      sol[r] = v;
    }
  for (int i = 0; i < z.nidx; ++i)
    coeffs[i] = 0.f;
  for (int i = 0; i < n; ++i)
    coeffs[z.pos[i]] = singular ? 0.f : __fmul_rn(sol[i], z.rad_per_m);
}

__global__ void shk_zfit_kernel(ZFit z, const float *g, const float *slopes, float *coeffs, float *cumulative) {
  if (blockIdx.x != 0 || threadIdx.x != 0)
    return;
  zfit_solve(z, g, slopes, coeffs);
  if (cumulative)
    for (int i = 0; i < z.nidx; ++i)
      cumulative[i] += coeffs[i];
}

struct ZModes {
  int n;
  int idx[kShkMaxModes];
};

// eval_zernike_noll_value_device (zernike_phase.cu:118-149)
__device__ __forceinline__ float zernike_value(int noll, float x, float y) {
  constexpr float s3 = 1.7320508075688772f, s6 = 2.4494897427831781f, s8 = 2.8284271247461903f;
  switch (noll) {
  case 2: return 2.0f * x;
  case 3: return 2.0f * y;
  case 4: return s3 * (2.0f * (x * x + y * y) - 1.0f);
  case 5: return 2.0f * s6 * x * y;
  case 6: return s6 * (x * x - y * y);
  case 7: return s8 * y * (3.0f * x * x - y * y);
  case 8: return s8 * y * (3.0f * x * x + 3.0f * y * y - 2.0f);
  case 9: return s8 * x * (3.0f * x * x + 3.0f * y * y - 2.0f);
  case 10: return s8 * x * (x * x - 3.0f * y * y);
  default: return 0.0f;
  }
}

// zernike_phase_kernel (zernike_phase.cu:151-180): every pixel, pupil of radius min(ny, nx) / 2
// centred on the grid.  `accumulate` adds the phase to `phase` (the cumulative map of repeated
// passes) instead of overwriting it.
// Rows over blockIdx.y, columns over the threads: no index division per pixel.
__global__ void shk_zernike_phase_kernel(const float *coeffs, ZModes zm, int ny, int nx, float *phase, float *cumulative) {
  const float cy = ((float)ny - 1.0f) * 0.5f, cx = ((float)nx - 1.0f) * 0.5f;
  const float r  = 0.5f * (float)(ny < nx ? ny : nx);
  float       c[kShkMaxModes];
#pragma unroll
  for (int m = 0; m < kShkMaxModes; ++m)
    c[m] = m < zm.n ? coeffs[m] : 0.f;
  for (int yi = blockIdx.y; yi < ny; yi += gridDim.y) {
    const float y = ((float)yi - cy) / r;
    for (int xi = blockIdx.x * blockDim.x + threadIdx.x; xi < nx; xi += gridDim.x * blockDim.x) {
      const float   x  = ((float)xi - cx) / r;
      float         ph = 0.f;
      for (int m = 0; m < zm.n; ++m)
        ph += c[m] * zernike_value(zm.idx[m], x, y);
      const int64_t i = (int64_t)yi * nx + xi;
      phase[i]        = ph;
      if (cumulative)
        cumulative[i] += ph;
    }
  }
}

// correct_phase_cf32_kernel / correct_phase_f32_to_cf32_kernel (correct_phase.cu:76-106):
// E exp(-i phi) with the phase map broadcast over the planes.
// out = in x exp(-i phase) for every plane: one sine/cosine per pixel, then the planes' elements of
// that pixel in turn (the same values, in place or not, as one sincosf per element)
__global__ void shk_correct_phase_kernel(const void *in, int complex_in, const float *phase, int64_t planes,
                                         int64_t plane, float2 *out) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < plane; p += (int64_t)gridDim.x * blockDim.x) {
    float sv, cv;
    sincosf(phase[p], &sv, &cv);
    int64_t k = 0;
    for (; k + 3 < planes; k += 4) { // four independent loads in flight
      if (complex_in) {
        float2 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          v[u] = static_cast<const float2 *>(in)[(k + u) * plane + p];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          out[(k + u) * plane + p] = make_float2(v[u].x * cv + v[u].y * sv, v[u].y * cv - v[u].x * sv);
      } else {
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          v[u] = static_cast<const float *>(in)[(k + u) * plane + p];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          out[(k + u) * plane + p] = make_float2(v[u] * cv, -v[u] * sv);
      }
    }
    for (; k < planes; ++k) {
      const int64_t i = k * plane + p;
      if (complex_in) {
        const float2 v = static_cast<const float2 *>(in)[i];
        out[i]         = make_float2(v.x * cv + v.y * sv, v.y * cv - v.x * sv);
      } else {
        const float v = static_cast<const float *>(in)[i];
        out[i]        = make_float2(v * cv, -v * sv);
      }
    }
  }
}

// wrap2pi_kernel (wrap2pi.cu:60-70)
__global__ void shk_wrap2pi_kernel(const float *in, float *out, int64_t n) {
  const float two_pi = 2.0f * 3.14159265358979f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float v = fmodf(in[i], two_pi);
    if (v < 0.0f)
      v += two_pi;
    out[i] = v;
  }
}

// ------------------------------------------------------------------------------------------------
// Host-side geometry and fit (shack_hartmann_geometry.cc:20-57, zernike_from_slopes.cc:95-277)
// ------------------------------------------------------------------------------------------------
struct Sample {
  float xn, yn;
  bool  active;
};

float geometry(int sy, int sx, int sub_h, int sub_w, int stride_y, int stride_x, float dy, float dx, bool skip,
               std::vector<Sample> &out) {
  const float pitch_x = (float)stride_x * dx, pitch_y = (float)stride_y * dy;
  const float aw = (float)((size_t)(sx - 1) * stride_x + sub_w) * dx;
  const float ah = (float)((size_t)(sy - 1) * stride_y + sub_h) * dy;
  const float r  = 0.5f * std::min(aw, ah);
  const float cx = ((float)sx - 1.0f) * 0.5f, cy = ((float)sy - 1.0f) * 0.5f;
  out.clear();
  for (int iy = 0; iy < sy; ++iy)
    for (int ix = 0; ix < sx; ++ix) {
      const float xm = ((float)ix - cx) * pitch_x, ym = ((float)iy - cy) * pitch_y;
      const float xn = xm / r, yn = ym / r;
      out.push_back({xn, yn, !skip || xn * xn + yn * yn <= 1.0f});
    }
  return r;
}

void zernike_derivative(int noll, float x, float y, float &dx, float &dy) {
  const float s3 = std::sqrt(3.0f), s6 = std::sqrt(6.0f), s8 = std::sqrt(8.0f);
  switch (noll) {
  case 2: dx = 2.0f, dy = 0.0f; break;
  case 3: dx = 0.0f, dy = 2.0f; break;
  case 4: dx = 4.0f * s3 * x, dy = 4.0f * s3 * y; break;
  case 5: dx = 2.0f * s6 * y, dy = 2.0f * s6 * x; break;
  case 6: dx = 2.0f * s6 * x, dy = -2.0f * s6 * y; break;
  case 7: dx = 6.0f * s8 * x * y, dy = 3.0f * s8 * (x * x - y * y); break;
  case 8: dx = 6.0f * s8 * x * y, dy = s8 * (3.0f * x * x + 9.0f * y * y - 2.0f); break;
  case 9: dx = s8 * (9.0f * x * x + 3.0f * y * y - 2.0f), dy = 6.0f * s8 * x * y; break;
  default: dx = 3.0f * s8 * (x * x - y * y), dy = -6.0f * s8 * x * y; break;
  }
}

int check_indexes(const int *idx, int n, const char *who) {
  if (idx == nullptr || n <= 0)
    return fail(HF_ERR_INVALID, std::string(who) + ": indexes must not be empty");
  if (n > kShkMaxModes)
    return fail(HF_ERR_INVALID, std::string(who) + ": too many requested Zernike modes");
  std::vector<int> u(idx, idx + n);
  for (int v : u)
    if (v < 2 || v > 10)
      return fail(HF_ERR_INVALID, std::string(who) + ": only Noll indexes 2..10 are supported");
  std::sort(u.begin(), u.end());
  if (std::adjacent_find(u.begin(), u.end()) != u.end())
    return fail(HF_ERR_INVALID, std::string(who) + ": indexes must be unique");
  return HF_OK;
}

} // namespace
} // namespace hf

using namespace hf;

// ================================================================================================
// C ABI
// ================================================================================================
struct hf_stfd {
  int64_t planes;
  int     H, W, real_in, win_h, win_w, sy, sx, nwy, nwx, global, output, skip_phase_shift, shift;
  float   lambda, dx, dy, z;
  DevPlan pw, ph;
  float2 *lens = nullptr, *wlens = nullptr, *scratch = nullptr;
};

namespace {
void release(hf_stfd *f) {
  if (!f)
    return;
  release(f->pw), release(f->ph);
  cudaFree(f->lens), cudaFree(f->wlens), cudaFree(f->scratch);
  delete f;
}


int stfd_lenses(hf_stfd *f, cudaStream_t s) {
  // input_lens_geometry (short_time_fresnel_diffraction.cu:342-369): the largest side of the frame
  // (the whole field, or one window) sets the origin.
  const int   w = f->global ? f->W : f->win_w, h = f->global ? f->H : f->win_h;
  const int   size = std::max(w, h), ox = (size - w) / 2, oy = (size - h) / 2;
  const float x0 = ((float)ox - (float)size / 2.0f) * f->dx, y0 = ((float)oy - (float)size / 2.0f) * f->dy;
  const float k  = 3.14159265358979f / (f->lambda * f->z);
  shk_input_lens_kernel<<<grid_1d((int64_t)w * h), 256, 0, s>>>(f->lens, w, h, f->dx, f->dy, x0, y0, k);
  note_launch();
  HF_TRY(launch_status("shk_input_lens_kernel"));
  if (f->wlens) {
    shk_window_lens_kernel<<<grid_1d((int64_t)f->win_w * f->win_h), 256, 0, s>>>(f->wlens, f->win_w, f->win_h,
                                                                                f->lambda, f->z, f->dx);
    note_launch();
    HF_TRY(launch_status("shk_window_lens_kernel"));
  }
  return HF_OK;
}
} // namespace

extern "C" {

int hf_stfd_create(int64_t planes, int height, int width, int real_input, int win_h, int win_w, int stride_y,
                   int stride_x, float lambda, float dx, float dy, float z, int phase_ref, int output,
                   int skip_phase_shift, int fftshift_windows, hf_stream_t s, hf_stfd **out) {
  clear_error();
  HF_CHECK_ARG(out != nullptr, "ShortTimeFresnelDiffractionFactory: null argument");
  *out = nullptr;
  HF_CHECK_ARG(planes >= 1 && height >= 1 && width >= 1, "ShortTimeFresnelDiffractionFactory: input must not be empty");
  HF_CHECK_ARG(lambda > 0.f, "ShortTimeFresnelDiffractionFactory: lambda must be positive");
  HF_CHECK_ARG(dx > 0.f, "ShortTimeFresnelDiffractionFactory: dx must be positive");
  HF_CHECK_ARG(dy > 0.f, "ShortTimeFresnelDiffractionFactory: dy must be positive");
  HF_CHECK_ARG(dx == dy, "ShortTimeFresnelDiffractionFactory: dx must equal dy");
  HF_CHECK_ARG(z != 0.f, "ShortTimeFresnelDiffractionFactory: z must be non-zero");
  HF_CHECK_ARG(win_h >= 1 && win_w >= 1, "ShortTimeFresnelDiffractionFactory: window dimensions must be >= 1");
  HF_CHECK_ARG(stride_y >= 1 && stride_x >= 1, "ShortTimeFresnelDiffractionFactory: strides must be >= 1");
  HF_CHECK_ARG(win_h <= height && win_w <= width, "ShortTimeFresnelDiffractionFactory: window dimensions exceed field size");
  HF_CHECK_ARG(phase_ref == HF_STFD_LOCAL || phase_ref == HF_STFD_GLOBAL, "ShortTimeFresnelDiffractionFactory: unknown phase_ref");
  HF_CHECK_ARG(output >= HF_STFD_COMPLEX && output <= HF_STFD_MEAN_MAGNITUDE,
               "ShortTimeFresnelDiffractionFactory: unknown output");
  auto *f = new (std::nothrow) hf_stfd();
  if (!f)
    return fail(HF_ERR_NOMEM, "ShortTimeFresnelDiffraction: host allocation failed");
  if (win_w > kShkMaxN || win_h > kShkMaxN) {
    delete f;
    return fail(HF_ERR_UNSUPPORTED, "ShortTimeFresnelDiffraction: window sides must be in 2..1024");
  }
  f->planes = planes, f->H = height, f->W = width, f->real_in = real_input ? 1 : 0;
  f->win_h = win_h, f->win_w = win_w, f->sy = stride_y, f->sx = stride_x;
  f->nwy = (height - win_h) / stride_y + 1, f->nwx = (width - win_w) / stride_x + 1;
  f->global = phase_ref == HF_STFD_GLOBAL, f->output = output, f->skip_phase_shift = skip_phase_shift ? 1 : 0;
  f->shift = fftshift_windows ? 1 : 0;
  f->lambda = lambda, f->dx = dx, f->dy = dy, f->z = z;
  const size_t lens_px = f->global ? (size_t)height * width : (size_t)win_h * win_w;
  const size_t out_px  = (size_t)planes * f->nwy * f->nwx * win_h * win_w;
  int          rc      = dev_plan_init(f->pw, win_w);
  if (rc == HF_OK)
    rc = dev_plan_init(f->ph, win_h);
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&f->lens, lens_px * sizeof(float2)), "ShortTimeFresnelDiffraction: lens");
  if (rc == HF_OK && output == HF_STFD_COMPLEX && !f->skip_phase_shift)
    rc = cuda_status(cudaMalloc(&f->wlens, (size_t)win_h * win_w * sizeof(float2)), "ShortTimeFresnelDiffraction: lens");
  if (rc == HF_OK && output != HF_STFD_COMPLEX)
    rc = cuda_status(cudaMalloc(&f->scratch, out_px * sizeof(float2)), "ShortTimeFresnelDiffraction: spectra");
  if (rc == HF_OK)
    rc = stfd_lenses(f, s);
  if (rc != HF_OK) {
    release(f);
    return rc;
  }
  *out = f;
  return HF_OK;
}

int hf_stfd_grid(const hf_stfd *f, int *ny, int *nx) {
  clear_error();
  HF_CHECK_ARG(f != nullptr && ny != nullptr && nx != nullptr, "ShortTimeFresnelDiffraction: null argument");
  *ny = f->nwy, *nx = f->nwx;
  return HF_OK;
}

int hf_stfd_set_z(hf_stfd *f, float z, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(f != nullptr, "ShortTimeFresnelDiffraction: null argument");
  HF_CHECK_ARG(z != 0.f, "ShortTimeFresnelDiffractionFactory: z must be non-zero");
  f->z = z;
  return stfd_lenses(f, s);
}

int hf_stfd_exec(hf_stfd *f, const void *in, void *out, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(f != nullptr && in != nullptr && out != nullptr, "ShortTimeFresnelDiffraction: null argument");
  const int64_t nwin = (int64_t)f->nwy * f->nwx;
  float2       *rows = f->output == HF_STFD_COMPLEX ? static_cast<float2 *>(out) : f->scratch;
  RowArgs       ra{};
  ra.pl = f->pw.pl, ra.n = f->pw.n, ra.tw = f->pw.tw, ra.n_rows = f->planes * nwin * f->win_h, ra.inv = false, ra.out = rows;
  ra.field = in, ra.real_in = f->real_in, ra.H = f->H, ra.W = f->W, ra.win_h = f->win_h, ra.nwx = f->nwx;
  ra.nwy = f->nwy, ra.stride_y = f->sy, ra.stride_x = f->sx, ra.global_lens = f->global, ra.lens = f->lens;
  HF_TRY(launch_rows<ROW_STFD>(ra, s));
  ColArgs ca{};
  ca.pl = f->ph.pl, ca.h = f->ph.n, ca.tw = f->ph.tw, ca.w = f->win_w, ca.inv = false, ca.in = rows;
  switch (f->output) {
  case HF_STFD_COMPLEX:
    ca.outc = static_cast<float2 *>(out), ca.post = f->wlens;
    return launch_cols<COL_COMPLEX>(ca, f->planes * nwin, s);
  case HF_STFD_MAGNITUDE:
    ca.outf = static_cast<float *>(out);
    return launch_cols<COL_MAG>(ca, f->planes * nwin, s);
  default:
    ca.outf = static_cast<float *>(out), ca.planes = (int)f->planes, ca.nwin = nwin, ca.shift = f->shift;
    return launch_cols<COL_MEAN_MAG>(ca, nwin, s);
  }
}

int hf_stfd_destroy(hf_stfd *f) {
  clear_error();
  release(f);
  return HF_OK;
}

} // extern "C"

// ------------------------------------------------------------------------------------------------
// Shack-Hartmann slopes
// ------------------------------------------------------------------------------------------------
struct hf_shslopes {
  int      sy, sx, h, w, center, count;
  float    sppx, sppy;
  Roi      roi;
  DevPlan  pw, ph;
  float2  *spec = nullptr, *cross = nullptr, *shifts = nullptr;
  float   *means = nullptr, *maps = nullptr;
  float   *taper = nullptr; // [h][w]: the ROI's cosine taper inside the ellipse, -1 outside
  uint8_t *active = nullptr;
  std::vector<uint8_t> active_host;
  // FullPairwise mode: pairs (i < j) of active samples in the reference's edge order, processed
  // pair_batch at a time; rhs indexed by active rank, pair_src / pair_dst by dense index into the
  // spectra and rank into rhs (src_rank / dst_rank)
  int      mode = 0, nact = 0, pair_batch = 0;
  int64_t  npairs = 0;
  int     *pair_src = nullptr, *pair_dst = nullptr, *pair_srank = nullptr, *pair_drank = nullptr;
  int     *active_dense = nullptr;
  float2  *pcross = nullptr, *pshift = nullptr, *rhs = nullptr;
  float   *pmaps = nullptr;
};

namespace {
void release(hf_shslopes *p) {
  if (!p)
    return;
  release(p->pw), release(p->ph);
  cudaFree(p->spec), cudaFree(p->cross), cudaFree(p->shifts);
  cudaFree(p->means), cudaFree(p->maps), cudaFree(p->taper), cudaFree(p->active);
  cudaFree(p->pair_src), cudaFree(p->pair_dst), cudaFree(p->pair_srank), cudaFree(p->pair_drank);
  cudaFree(p->active_dense), cudaFree(p->pcross), cudaFree(p->pshift), cudaFree(p->rhs), cudaFree(p->pmaps);
  delete p;
}
int shslopes_set_mode(hf_shslopes *p, int mode, int pair_batch_size);
} // namespace

extern "C" {

int hf_shslopes_create(int sy, int sx, int height, int width, int sub_h, int sub_w, int stride_y, int stride_x,
                       float lambda, float dx, float dy, float z, const hf_ellipse *roi, int skip_outside, hf_stream_t s,
                       hf_shslopes **out) {
  return hf_shslopes_create_mode(sy, sx, height, width, sub_h, sub_w, stride_y, stride_x, lambda, dx, dy, z, roi,
                                 skip_outside, HF_SHSLOPES_SINGLE_REFERENCE, 256, s, out);
}

int hf_shslopes_create_mode(int sy, int sx, int height, int width, int sub_h, int sub_w, int stride_y, int stride_x,
                            float lambda, float dx, float dy, float z, const hf_ellipse *roi, int skip_outside, int mode,
                            int pair_batch_size, hf_stream_t s, hf_shslopes **out) {
  clear_error();
  HF_CHECK_ARG(out != nullptr, "ShackHartmannSlopesFactory inference error: null argument");
  *out = nullptr;
  HF_CHECK_ARG(mode == HF_SHSLOPES_SINGLE_REFERENCE || mode == HF_SHSLOPES_FULL_PAIRWISE,
               "Unknown Shack-Hartmann slope mode");
  HF_CHECK_ARG(sy > 0 && sx > 0, "ShackHartmannSlopesFactory inference error: subaperture grid dimensions must be positive");
  if (mode == HF_SHSLOPES_SINGLE_REFERENCE)
    HF_CHECK_ARG(sy % 2 == 1 && sx % 2 == 1, "ShackHartmannSlopesFactory inference error: subaperture grid dimensions "
                                             "must be odd for an unambiguous center reference");
  HF_CHECK_ARG(height >= 2 && width >= 2, "ShackHartmannSlopesFactory inference error: reconstruction dimensions must be at least 2");
  HF_CHECK_ARG(lambda > 0.f, "ShackHartmannSlopesFactory inference error: wavelength must be > 0");
  HF_CHECK_ARG(dx > 0.f && dy > 0.f, "ShackHartmannSlopesFactory inference error: pixel pitches must be > 0");
  HF_CHECK_ARG(z > 0.f, "ShackHartmannSlopesFactory inference error: propagation distance must be > 0");
  const hf_ellipse e = roi ? *roi : hf_ellipse{0.5f, 0.5f, 0.5f, 0.5f, 0.f};
  HF_CHECK_ARG(e.rx > 0.f && e.ry > 0.f, "ShackHartmannSlopesFactory inference error: correlation ROI radii must be positive");
  if (sub_h <= 0 && sub_w <= 0 && stride_y <= 0 && stride_x <= 0) // 0: the image size, stride = size
    sub_h = stride_y = height, sub_w = stride_x = width;
  HF_CHECK_ARG(sub_h > 0 && sub_w > 0, "ShackHartmannSlopesFactory inference error: subaperture dimensions must be positive");
  HF_CHECK_ARG(stride_y > 0 && stride_x > 0, "ShackHartmannSlopesFactory inference error: strides must be positive");
  std::vector<Sample> geo;
  const float r = geometry(sy, sx, sub_h, sub_w, stride_y, stride_x, dy, dx, skip_outside != 0, geo);
  HF_CHECK_ARG(r > 0.f, "ShackHartmannSlopesFactory inference error: pupil radius must be positive");
  HF_CHECK_ARG(std::any_of(geo.begin(), geo.end(), [](const Sample &g) { return g.active; }),
               "ShackHartmannSlopesFactory inference error: at least one subaperture must be active");
  auto *p = new (std::nothrow) hf_shslopes();
  if (!p)
    return fail(HF_ERR_NOMEM, "ShackHartmannSlopes: host allocation failed");
  if (width > kShkMaxN || height > kShkMaxN) {
    delete p;
    return fail(HF_ERR_UNSUPPORTED, "ShackHartmannSlopes: subaperture sides must be in 2..1024");
  }
  p->sy = sy, p->sx = sx, p->h = height, p->w = width, p->count = sy * sx, p->center = (sy / 2) * sx + sx / 2;
  // delta_out / z with delta_out = lambda z / (n d) (shack_hartmann_slopes.cu:268-275)
  p->sppx = lambda * z / ((float)width * dx) / z;
  p->sppy = lambda * z / ((float)height * dy) / z;
  const float th = e.angle * (3.14159265358979f / 180.0f);
  p->roi         = Roi{e.cx, e.cy, e.rx, e.ry, std::cos(th), std::sin(th)};
  for (const Sample &g : geo)
    p->active_host.push_back(g.active ? 1 : 0);
  const size_t px = (size_t)p->count * height * width;
  int          rc = dev_plan_init(p->pw, width);
  if (rc == HF_OK)
    rc = dev_plan_init(p->ph, height);
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&p->spec, px * sizeof(float2)), "ShackHartmannSlopes: spectra");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&p->cross, px * sizeof(float2)), "ShackHartmannSlopes: cross power");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&p->maps, px * sizeof(float)), "ShackHartmannSlopes: maps");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&p->means, (size_t)p->count * sizeof(float)), "ShackHartmannSlopes: means");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&p->taper, (size_t)height * width * sizeof(float)), "ShackHartmannSlopes: ROI taper");
  if (rc == HF_OK) {
    shk_roi_taper_kernel<<<grid_1d((int64_t)height * width), 256, 0, s>>>(p->taper, height, width, p->roi);
    note_launch();
    rc = launch_status("shk_roi_taper_kernel");
  }
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&p->shifts, (size_t)p->count * sizeof(float2)), "ShackHartmannSlopes: shifts");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&p->active, (size_t)p->count), "ShackHartmannSlopes: active");
  if (rc == HF_OK)
    rc = cuda_status(cudaMemcpy(p->active, p->active_host.data(), (size_t)p->count, cudaMemcpyHostToDevice),
                     "ShackHartmannSlopes: active");
  if (rc == HF_OK && mode == HF_SHSLOPES_FULL_PAIRWISE)
    rc = shslopes_set_mode(p, mode, pair_batch_size);
  if (rc != HF_OK) {
    release(p);
    return rc;
  }
  *out = p;
  return HF_OK;
}

int hf_shslopes_active(const hf_shslopes *p, uint8_t *active) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && active != nullptr, "ShackHartmannSlopes: null argument");
  std::memcpy(active, p->active_host.data(), p->active_host.size());
  return HF_OK;
}

} // extern "C"

namespace {
// Switches a created slopes object to `mode`, allocating the pair lists and batch buffers.
int shslopes_set_mode(hf_shslopes *p, int mode, int pair_batch_size) {
  HF_CHECK_ARG(mode == HF_SHSLOPES_SINGLE_REFERENCE || mode == HF_SHSLOPES_FULL_PAIRWISE,
               "Unknown Shack-Hartmann slope mode");
  HF_CHECK_ARG(pair_batch_size > 0, "ShackHartmannSlopesFactory inference error: pair_batch_size must be positive");
  if (mode == HF_SHSLOPES_SINGLE_REFERENCE) {
    p->mode = 0;
    return HF_OK;
  }
  std::vector<int> dense;
  for (int i = 0; i < p->count; ++i)
    if (p->active_host[i])
      dense.push_back(i);
  const int nact = (int)dense.size();
  HF_CHECK_ARG(nact >= 2, "ShackHartmannSlopesFactory inference error: FullPairwise mode requires at least two "
                          "active subapertures");
  // edges (i, j), i < j over the active ranks, source-major (generate_complete_graph_pairs)
  const int64_t    npairs = (int64_t)nact * (nact - 1) / 2;
  std::vector<int> src, dst, srank, drank;
  for (int i = 0; i < nact; ++i)
    for (int j = i + 1; j < nact; ++j)
      src.push_back(dense[i]), dst.push_back(dense[j]), srank.push_back(i), drank.push_back(j);
  const int    batch = (int)std::min<int64_t>(pair_batch_size, npairs);
  const size_t px    = (size_t)batch * p->h * p->w;
  cudaFree(p->pair_src), cudaFree(p->pair_dst), cudaFree(p->pair_srank), cudaFree(p->pair_drank);
  cudaFree(p->active_dense), cudaFree(p->pcross), cudaFree(p->pshift), cudaFree(p->rhs), cudaFree(p->pmaps);
  p->pair_src = p->pair_dst = p->pair_srank = p->pair_drank = p->active_dense = nullptr;
  p->pcross = p->pshift = p->rhs = nullptr;
  p->pmaps  = nullptr;
  p->mode   = 0;
  const struct {
    int                  **dst;
    const std::vector<int> *src;
  } arrays[5] = {{&p->pair_src, &src}, {&p->pair_dst, &dst}, {&p->pair_srank, &srank}, {&p->pair_drank, &drank},
                 {&p->active_dense, &dense}};
  for (const auto &a : arrays) {
    HF_CUDA(cudaMalloc(a.dst, a.src->size() * sizeof(int)));
    HF_CUDA(cudaMemcpy(*a.dst, a.src->data(), a.src->size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  HF_CUDA(cudaMalloc(&p->pcross, px * sizeof(float2)));
  HF_CUDA(cudaMalloc(&p->pmaps, px * sizeof(float)));
  HF_CUDA(cudaMalloc(&p->pshift, (size_t)batch * sizeof(float2)));
  HF_CUDA(cudaMalloc(&p->rhs, (size_t)nact * sizeof(float2)));
  p->mode = 1, p->nact = nact, p->npairs = npairs, p->pair_batch = batch;
  return HF_OK;
}
} // namespace

extern "C" {

int hf_shslopes_exec(hf_shslopes *p, const float *images, float *slopes, float *maps, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && images != nullptr && slopes != nullptr, "ShackHartmannSlopes: null argument");
  const int64_t rows = (int64_t)p->count * p->h;
  float        *mo   = maps ? maps : p->maps;
  shk_roi_mean_kernel<<<p->count, kRedThreads, 0, s>>>(images, p->means, p->h, p->w, p->taper);
  note_launch();
  HF_TRY(launch_status("shk_roi_mean_kernel"));
  // forward transform of the prepared images: rows (mean removal + taper fused), then columns
  RowArgs ra{};
  ra.pl = p->pw.pl, ra.n = p->pw.n, ra.tw = p->pw.tw, ra.n_rows = rows, ra.inv = false, ra.out = p->spec;
  ra.img = images, ra.means = p->means, ra.taper = p->taper, ra.h = p->h;
  HF_TRY(launch_rows<ROW_XPACK>(ra, s));
  ColArgs ca{};
  ca.pl = p->ph.pl, ca.h = p->ph.n, ca.tw = p->ph.tw, ca.w = p->w, ca.inv = false, ca.in = p->spec, ca.outc = p->spec;
  HF_TRY(launch_cols<COL_COMPLEX>(ca, p->count, s));
  if (p->mode == 1) { // FullPairwise: every pair of active samples, pair_batch maps at a time
    HF_CHECK_ARG(maps == nullptr, "ShackHartmannSlopes: FullPairwise correlation-map output is not supported");
    HF_CUDA(cudaMemsetAsync(p->rhs, 0, (size_t)p->nact * sizeof(float2), s));
    for (int64_t e0 = 0; e0 < p->npairs; e0 += p->pair_batch) {
      const int nb = (int)std::min<int64_t>(p->pair_batch, p->npairs - e0);
      RowArgs   rp{};
      rp.pl = p->pw.pl, rp.n = p->pw.n, rp.tw = p->pw.tw, rp.n_rows = (int64_t)nb * p->h, rp.inv = true;
      rp.out = p->pcross, rp.spec = p->spec, rp.h = p->h, rp.pair_src = p->pair_src, rp.pair_dst = p->pair_dst;
      rp.pair0 = e0;
      HF_TRY(launch_rows<ROW_PAIR>(rp, s));
      ColArgs cp{};
      cp.pl = p->ph.pl, cp.h = p->ph.n, cp.tw = p->ph.tw, cp.w = p->w, cp.inv = true, cp.in = p->pcross, cp.outf = p->pmaps;
      cp.scale = (float)(1.0 / ((double)p->h * p->w)); // inverse_fft_scale
      HF_TRY(launch_cols<COL_REAL>(cp, nb, s));
      shk_peak_kernel<<<nb, kRedThreads, 0, s>>>(p->pmaps, p->pshift, p->h, p->w);
      note_launch();
      HF_TRY(launch_status("shk_peak_kernel"));
      shk_pair_rhs_kernel<<<1, 32, 0, s>>>(p->pshift, p->pair_srank, p->pair_drank, e0, nb, p->rhs, p->sppx, p->sppy);
      note_launch();
      HF_TRY(launch_status("shk_pair_rhs_kernel"));
    }
    shk_pair_solve_kernel<<<1, 32, 0, s>>>(p->rhs, p->active_dense, p->nact, p->count, slopes);
    note_launch();
    return launch_status("shk_pair_solve_kernel");
  }
  // cross power against the centre spectrum (fused into the inverse row pass), inverse columns
  RowArgs rb{};
  rb.pl = p->pw.pl, rb.n = p->pw.n, rb.tw = p->pw.tw, rb.n_rows = rows, rb.inv = true, rb.out = p->cross;
  rb.spec = p->spec, rb.ref_img = p->center, rb.h = p->h;
  HF_TRY(launch_rows<ROW_CROSS>(rb, s));
  ColArgs cb{};
  cb.pl = p->ph.pl, cb.h = p->ph.n, cb.tw = p->ph.tw, cb.w = p->w, cb.inv = true, cb.in = p->cross, cb.outf = mo;
  cb.scale = (float)(1.0 / ((double)p->h * p->w)); // backward norm (cross_correlation2.cu:119-125)
  HF_TRY(launch_cols<COL_REAL>(cb, p->count, s));
  shk_peak_kernel<<<p->count, kRedThreads, 0, s>>>(mo, p->shifts, p->h, p->w);
  note_launch();
  HF_TRY(launch_status("shk_peak_kernel"));
  shk_slopes_kernel<<<1, 32, 0, s>>>(p->shifts, p->active, slopes, p->count, p->center, p->sppx, p->sppy);
  note_launch();
  return launch_status("shk_slopes_kernel");
}

int hf_shslopes_destroy(hf_shslopes *p) {
  clear_error();
  release(p);
  return HF_OK;
}

} // extern "C"

// ------------------------------------------------------------------------------------------------
// Zernike fit
// ------------------------------------------------------------------------------------------------
struct hf_zernike_fit {
  ZFit               z;
  int                idx[kShkMaxModes];
  float              pupil_radius;
  std::vector<float> g;        // [count][2][9]: mean-removed derivatives / radius; NaN row = inactive
  float             *g_dev = nullptr;
};

namespace {
void release(hf_zernike_fit *f) {
  if (!f)
    return;
  cudaFree(f->g_dev);
  delete f;
}

// Host copy of the fit (the reference runs it on the host): same sequence as zfit_solve.
void zfit_host(const hf_zernike_fit *f, const float *slopes, float *coeffs) {
  const ZFit &z = f->z;
  const int   n = z.nobs;
  float       m[kShkMaxModes][kShkMaxModes], rhs[kShkMaxModes] = {}, sol[kShkMaxModes] = {};
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      m[i][j] = z.gtg[i][j];
  for (int s = 0; s < z.count; ++s) {
    const float *gs = f->g.data() + (size_t)s * 2 * kShkMaxModes;
    if (std::isnan(gs[0]) && n > 0)
      continue;
    const volatile float sx = slopes[2 * s], sy = slopes[2 * s + 1];
    for (int i = 0; i < n; ++i) {
      const volatile float a = gs[i] * sx, b = gs[kShkMaxModes + i] * sy;
      rhs[i] += a + b;
    }
  }
  bool singular = false;
  for (int c = 0; c < n && !singular; ++c) {
    int   piv = c;
    float bv  = std::fabs(m[c][c]);
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(m[r][c]) > bv)
        bv = std::fabs(m[r][c]), piv = r;
    if (bv < 1e-12f) {
      singular = true;
      break;
    }
    if (piv != c) {
      for (int j = 0; j < n; ++j)
        std::swap(m[piv][j], m[c][j]);
      std::swap(rhs[piv], rhs[c]);
    }
    const float pv = m[c][c];
    for (int j = c; j < n; ++j)
      m[c][j] /= pv;
    rhs[c] /= pv;
    for (int r = c + 1; r < n; ++r) {
      const float fct = m[r][c];
      for (int j = c; j < n; ++j) {
        const volatile float t = fct * m[c][j];
        m[r][j] -= t;
      }
      const volatile float t = fct * rhs[c];
      rhs[r] -= t;
    }
  }
  if (!singular)
    for (int r = n - 1; r >= 0; --r) {
      float v = rhs[r];
      for (int c = r + 1; c < n; ++c) {
        const volatile float t = m[r][c] * sol[c];
        v -= t;
      }
      sol[r] = v;
    }
  for (int i = 0; i < z.nidx; ++i)
    coeffs[i] = 0.f;
  for (int i = 0; i < n; ++i)
    coeffs[z.pos[i]] = singular ? 0.f : sol[i] * z.rad_per_m;
}
} // namespace

extern "C" {

int hf_zernike_fit_create(int sy, int sx, int sub_h, int sub_w, int stride_y, int stride_x, float lambda, float dx,
                          float dy, int skip_outside, const int *indexes, int n_indexes, hf_zernike_fit **out) {
  clear_error();
  HF_CHECK_ARG(out != nullptr, "ZernikeFromSlopesFactory inference error: null argument");
  *out = nullptr;
  HF_CHECK_ARG(sy > 0 && sx > 0, "ZernikeFromSlopesFactory inference error: subaperture grid dimensions must be positive");
  HF_CHECK_ARG(lambda > 0.f, "ZernikeFromSlopesFactory inference error: wavelength must be > 0");
  HF_CHECK_ARG(dx > 0.f && dy > 0.f, "ZernikeFromSlopesFactory inference error: pixel pitches must be > 0");
  HF_CHECK_ARG(sub_h > 0 && sub_w > 0, "ZernikeFromSlopesFactory inference error: subaperture dimensions must be positive");
  HF_CHECK_ARG(stride_y > 0 && stride_x > 0, "ZernikeFromSlopesFactory inference error: strides must be positive");
  HF_TRY(check_indexes(indexes, n_indexes, "ZernikeFromSlopesFactory inference error"));
  std::vector<Sample> geo;
  const float r = geometry(sy, sx, sub_h, sub_w, stride_y, stride_x, dy, dx, skip_outside != 0, geo);
  HF_CHECK_ARG(r > 0.f, "ZernikeFromSlopesFactory inference error: pupil radius must be positive");
  HF_CHECK_ARG(std::any_of(geo.begin(), geo.end(), [](const Sample &g) { return g.active; }),
               "ZernikeFromSlopesFactory inference error: at least one subaperture must be active");
  auto *f = new (std::nothrow) hf_zernike_fit();
  if (!f)
    return fail(HF_ERR_NOMEM, "ZernikeFromSlopes: host allocation failed");
  ZFit &z = f->z;
  z.count = sy * sx, z.nidx = n_indexes, z.nobs = 0;
  for (int i = 0; i < n_indexes; ++i) {
    f->idx[i] = indexes[i];
    if (indexes[i] != 2 && indexes[i] != 3)
      z.pos[z.nobs++] = i;
  }
  f->pupil_radius = r;
  z.rad_per_m     = 2.0f * std::acos(-1.0f) / lambda;
  // derivatives / radius and their means over the active samples, accumulated in sample order
  // (zernike_from_slopes.cc:221-244), then the normal matrix in row-major sample order (:246-266)
  const int          n = z.nobs;
  std::vector<float> dxv((size_t)z.count * kShkMaxModes, 0.f), dyv((size_t)z.count * kShkMaxModes, 0.f);
  float              mx[kShkMaxModes] = {}, my[kShkMaxModes] = {};
  size_t             na = 0;
  for (int s = 0; s < z.count; ++s) {
    if (!geo[s].active)
      continue;
    ++na;
    for (int m = 0; m < n; ++m) {
      float ddx, ddy;
      zernike_derivative(indexes[z.pos[m]], geo[s].xn, geo[s].yn, ddx, ddy);
      dxv[(size_t)s * kShkMaxModes + m] = ddx / r;
      dyv[(size_t)s * kShkMaxModes + m] = ddy / r;
      mx[m] += dxv[(size_t)s * kShkMaxModes + m];
      my[m] += dyv[(size_t)s * kShkMaxModes + m];
    }
  }
  for (int m = 0; m < n; ++m)
    mx[m] /= (float)na, my[m] /= (float)na;
  std::memset(z.gtg, 0, sizeof(z.gtg));
  f->g.assign((size_t)z.count * 2 * kShkMaxModes, 0.f);
  for (int s = 0; s < z.count; ++s) {
    float *gs = f->g.data() + (size_t)s * 2 * kShkMaxModes;
    if (!geo[s].active) {
      gs[0] = NAN;
      continue;
    }
    for (int i = 0; i < n; ++i) {
      const float gxi = dxv[(size_t)s * kShkMaxModes + i] - mx[i], gyi = dyv[(size_t)s * kShkMaxModes + i] - my[i];
      gs[i] = gxi, gs[kShkMaxModes + i] = gyi;
      for (int j = 0; j < n; ++j) {
        const float gxj = dxv[(size_t)s * kShkMaxModes + j] - mx[j], gyj = dyv[(size_t)s * kShkMaxModes + j] - my[j];
        const volatile float a = gxi * gxj, b = gyi * gyj;
        z.gtg[i][j] += a + b;
      }
    }
  }
  for (int m = 0; m < n; ++m)
    z.gtg[m][m] += 1e-9f;
  int rc = cuda_status(cudaMalloc(&f->g_dev, f->g.size() * sizeof(float)), "ZernikeFromSlopes: derivatives");
  if (rc == HF_OK)
    rc = cuda_status(cudaMemcpy(f->g_dev, f->g.data(), f->g.size() * sizeof(float), cudaMemcpyHostToDevice),
                     "ZernikeFromSlopes: derivatives");
  if (rc != HF_OK) {
    release(f);
    return rc;
  }
  *out = f;
  return HF_OK;
}

int hf_zernike_fit_pupil_radius(const hf_zernike_fit *f, float *r) {
  clear_error();
  HF_CHECK_ARG(f != nullptr && r != nullptr, "ZernikeFromSlopes: null argument");
  *r = f->pupil_radius;
  return HF_OK;
}

int hf_zernike_fit_exec(hf_zernike_fit *f, const float *slopes, float *coeffs, float *cumulative, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(f != nullptr && slopes != nullptr && coeffs != nullptr, "ZernikeFromSlopes: null argument");
  shk_zfit_kernel<<<1, 32, 0, s>>>(f->z, f->g_dev, slopes, coeffs, cumulative);
  note_launch();
  return launch_status("shk_zfit_kernel");
}

int hf_zernike_fit_host(const hf_zernike_fit *f, const float *slopes, float *coeffs) {
  clear_error();
  HF_CHECK_ARG(f != nullptr && slopes != nullptr && coeffs != nullptr, "ZernikeFromSlopes: null argument");
  zfit_host(f, slopes, coeffs);
  return HF_OK;
}

int hf_zernike_fit_destroy(hf_zernike_fit *f) {
  clear_error();
  release(f);
  return HF_OK;
}

int hf_zernike_phase(const float *coeffs, const int *indexes, int n_indexes, int ny, int nx, float *phase,
                     float *cumulative, hf_stream_t s) {
  clear_error();
  HF_TRY(check_indexes(indexes, n_indexes, "ZernikePhaseFactory inference error"));
  HF_CHECK_ARG(ny > 0 && nx > 0, "ZernikePhaseFactory inference error: Resolution ny and nx must be greater than 0");
  HF_CHECK_ARG(coeffs != nullptr && phase != nullptr, "ZernikePhase: null argument");
  ZModes zm{};
  zm.n = n_indexes;
  for (int i = 0; i < n_indexes; ++i)
    zm.idx[i] = indexes[i];
  const dim3 zg((unsigned)std::min(4, (nx + 255) / 256), (unsigned)std::min(ny, 65535));
  shk_zernike_phase_kernel<<<zg, 256, 0, s>>>(coeffs, zm, ny, nx, phase, cumulative);
  note_launch();
  return launch_status("shk_zernike_phase_kernel");
}

int hf_correct_phase(const void *in, int complex_input, const float *phase, int64_t planes, int height, int width,
                     void *out, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(in != nullptr && phase != nullptr && out != nullptr, "CorrectPhase: null argument");
  HF_CHECK_ARG(planes >= 1 && height >= 1 && width >= 1, "CorrectPhaseFactory: input must not be empty");
  const int64_t plane = (int64_t)height * width;
  shk_correct_phase_kernel<<<grid_1d(plane), 256, 0, s>>>(in, complex_input ? 1 : 0, phase, planes, plane,
                                                          static_cast<float2 *>(out));
  note_launch();
  return launch_status("shk_correct_phase_kernel");
}

int hf_wrap2pi(const float *in, float *out, int64_t n, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(in != nullptr && out != nullptr && n >= 0, "Wrap2Pi: null argument");
  if (n == 0)
    return HF_OK;
  shk_wrap2pi_kernel<<<grid_1d(n), 256, 0, s>>>(in, out, n);
  note_launch();
  return launch_status("shk_wrap2pi_kernel");
}

int hf_defocus_z(float a4, float lambda, float z_curr, float pupil_radius, double *delta_inv_z, double *z_new,
                 double *delta_z_mm) {
  clear_error();
  HF_CHECK_ARG(lambda > 0.f, "ZernikeDefocusZPropFactory inference error: lambda must be positive");
  HF_CHECK_ARG(z_curr != 0.f, "ZernikeDefocusZPropFactory inference error: z_curr must be non-zero");
  HF_CHECK_ARG(pupil_radius > 0.f, "ZernikeDefocusZPropFactory inference error: pupil_radius must be positive");
  HF_CHECK_ARG(delta_inv_z != nullptr && z_new != nullptr && delta_z_mm != nullptr, "ZernikeDefocusZProp: null argument");
  // estimate_z_prop_from_a4 (zernike_defocus_z_prop.cc:84-97), float64
  const double r2 = (double)pupil_radius * pupil_radius;
  const double di = (2.0 * std::sqrt(3.0) * lambda * a4) / (M_PI * r2);
  const double zn = 1.0 / (1.0 / z_curr - di);
  if (!std::isfinite(a4) || !std::isfinite(zn) || std::fabs(1.0 / zn) <= 1e-18)
    return fail(HF_ERR_INVALID, "ZernikeDefocusZProp: estimated z_prop is undefined");
  *delta_inv_z = di, *z_new = zn, *delta_z_mm = 1000.0 * (zn - z_curr);
  return HF_OK;
}

} // extern "C"

// ------------------------------------------------------------------------------------------------
// One autofocus pass over a spectrum (build_shack_hartmann, graph_builder.cc:307-501)
// ------------------------------------------------------------------------------------------------
struct hf_autofocus {
  int             nz, H, W, nb, sh, sw, n_iter, nidx;
  int             idx[kShkMaxModes];
  float           pupil_radius;
  hf_stfd        *stfd  = nullptr;
  hf_shslopes    *sl    = nullptr;
  hf_zernike_fit *fit   = nullptr;
  hf_flatfield   *ff    = nullptr; // optional high-pass of the sub-aperture images
  float          *m0    = nullptr, *slopes = nullptr, *coeffs = nullptr, *cum_coeffs = nullptr;
  float          *phase = nullptr, *cum_phase = nullptr;
  // causal sliding average of the sub-aperture images over the last acc_n spectra
  // (pp_accumulation, graph_builder.cc:348): float32 history [acc_n][m0] and running sum
  int             acc_n = 1, pass = 0;
  int64_t         acc_count = 0;
  float          *acc_hist = nullptr, *acc_sum = nullptr;
};

namespace {
void release(hf_autofocus *a) {
  if (!a)
    return;
  release(a->stfd), release(a->sl), release(a->fit);
  hf_flatfield_destroy(a->ff);
  cudaFree(a->m0), cudaFree(a->slopes), cudaFree(a->coeffs), cudaFree(a->cum_coeffs);
  cudaFree(a->phase), cudaFree(a->cum_phase);
  cudaFree(a->acc_hist), cudaFree(a->acc_sum);
  delete a;
}
} // namespace

extern "C" {

int hf_autofocus_create(int nz, int height, int width, int nb_subaps, int n_iter, float lambda, float dx, float z,
                        float roi_radius, int skip_outside, const int *indexes, int n_indexes,
                        float flatfield_period, hf_stream_t s, hf_autofocus **out) {
  clear_error();
  HF_CHECK_ARG(out != nullptr, "Autofocus: null argument");
  *out = nullptr;
  HF_CHECK_ARG(nz >= 1 && height >= 1 && width >= 1, "Autofocus: input must not be empty");
  HF_CHECK_ARG(n_iter > 0, "autofocus_nb_iter must be positive");
  HF_CHECK_ARG(nb_subaps > 0, "autofocus_nb_subaps must be positive");
  HF_CHECK_ARG(nb_subaps % 2 == 1, "autofocus_nb_subaps must be odd");
  HF_CHECK_ARG(width / nb_subaps > 0 && height / nb_subaps > 0, "autofocus_nb_subaps is too large for the current frame size");
  if (n_indexes > 0)
    HF_TRY(check_indexes(indexes, n_indexes, "Autofocus"));
  auto *a = new (std::nothrow) hf_autofocus();
  if (!a)
    return fail(HF_ERR_NOMEM, "Autofocus: host allocation failed");
  a->nz = nz, a->H = height, a->W = width, a->nb = nb_subaps, a->n_iter = n_iter, a->nidx = n_indexes;
  a->sh = height / nb_subaps, a->sw = width / nb_subaps;
  for (int i = 0; i < n_indexes; ++i)
    a->idx[i] = indexes[i];
  a->pupil_radius = 0.5f * std::min((float)(a->sw * nb_subaps) * dx, (float)(a->sh * nb_subaps) * dx);
  const hf_ellipse roi{0.5f, 0.5f, roi_radius, roi_radius, 0.0f};
  const size_t     nsub = (size_t)nb_subaps * nb_subaps;
  int rc = hf_stfd_create(nz, height, width, 0, a->sh, a->sw, a->sh, a->sw, lambda, dx, dx, z, HF_STFD_GLOBAL,
                          HF_STFD_MEAN_MAGNITUDE, 1, 1, s, &a->stfd);
  if (rc == HF_OK)
    rc = hf_shslopes_create(nb_subaps, nb_subaps, a->sh, a->sw, a->sh, a->sw, a->sh, a->sw, lambda, dx, dx, z, &roi,
                            skip_outside, s, &a->sl);
  if (rc == HF_OK && n_indexes > 0)
    rc = hf_zernike_fit_create(nb_subaps, nb_subaps, a->sh, a->sw, a->sh, a->sw, lambda, dx, dx, skip_outside, indexes,
                               n_indexes, &a->fit);
  if (rc == HF_OK && flatfield_period > 0.f) {
    // graph_builder.cc:348-352: sigma = 0.187 period / pitch, with the one-FFT Fresnel output
    // pitch lambda |z| / (n d) of a sub-aperture (fresnel_1fft_output_pitch), in float32
    const float dy_out = lambda * std::fabs(z) / ((float)a->sh * dx);
    const float dx_out = lambda * std::fabs(z) / ((float)a->sw * dx);
    rc = hf_flatfield_create((int64_t)nsub, a->sh, a->sw, 0.187f * flatfield_period / dy_out,
                             0.187f * flatfield_period / dx_out, s, &a->ff);
  }
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&a->m0, nsub * a->sh * a->sw * sizeof(float)), "Autofocus: M0");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&a->slopes, nsub * 2 * sizeof(float)), "Autofocus: slopes");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&a->coeffs, kShkMaxModes * sizeof(float)), "Autofocus: coefficients");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&a->cum_coeffs, kShkMaxModes * sizeof(float)), "Autofocus: coefficients");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&a->phase, (size_t)height * width * sizeof(float)), "Autofocus: phase");
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(&a->cum_phase, (size_t)height * width * sizeof(float)), "Autofocus: phase");
  if (rc != HF_OK) {
    release(a);
    return rc;
  }
  *out = a;
  return HF_OK;
}

int hf_autofocus_set_accumulation(hf_autofocus *a, int pp_accumulation, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(a != nullptr, "Autofocus: null argument");
  HF_CHECK_ARG(pp_accumulation > 0, "pp_accumulation must be positive");
  HF_CHECK_ARG(pp_accumulation == 1 || a->n_iter == 1, "sliding Shack-Hartmann correction only supports one autofocus "
                                                       "iteration");
  cudaFree(a->acc_hist), cudaFree(a->acc_sum);
  a->acc_hist = a->acc_sum = nullptr;
  a->acc_n = 1, a->acc_count = 0;
  if (pp_accumulation > 1) {
    const size_t n = (size_t)a->nb * a->nb * a->sh * a->sw;
    HF_CUDA(cudaMalloc(&a->acc_hist, (size_t)pp_accumulation * n * sizeof(float)));
    HF_CUDA(cudaMalloc(&a->acc_sum, n * sizeof(float)));
    HF_CUDA(cudaMemsetAsync(a->acc_hist, 0, (size_t)pp_accumulation * n * sizeof(float), s));
    HF_CUDA(cudaMemsetAsync(a->acc_sum, 0, n * sizeof(float), s));
    a->acc_n = pp_accumulation;
  }
  return HF_OK;
}

int hf_autofocus_reset(hf_autofocus *a, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(a != nullptr, "Autofocus: null argument");
  a->acc_count = 0;
  if (a->acc_n > 1) {
    const size_t n = (size_t)a->nb * a->nb * a->sh * a->sw;
    HF_CUDA(cudaMemsetAsync(a->acc_hist, 0, (size_t)a->acc_n * n * sizeof(float), s));
    HF_CUDA(cudaMemsetAsync(a->acc_sum, 0, n * sizeof(float), s));
  }
  return HF_OK;
}

int hf_autofocus_set_slope_mode(hf_autofocus *a, int mode, int pair_batch_size, float roi_radius, int skip_outside,
                                float lambda, float dx, float z, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(a != nullptr, "Autofocus: null argument");
  const hf_ellipse roi{0.5f, 0.5f, roi_radius > 0.f ? roi_radius : 0.5f, roi_radius > 0.f ? roi_radius : 0.5f, 0.0f};
  hf_shslopes     *sl = nullptr;
  HF_TRY(hf_shslopes_create_mode(a->nb, a->nb, a->sh, a->sw, a->sh, a->sw, a->sh, a->sw, lambda, dx, dx, z, &roi,
                                 skip_outside, mode, pair_batch_size, s, &sl));
  release(a->sl);
  a->sl = sl;
  return HF_OK;
}

int hf_autofocus_pupil_radius(const hf_autofocus *a, float *r) {
  clear_error();
  HF_CHECK_ARG(a != nullptr && r != nullptr, "Autofocus: null argument");
  *r = a->pupil_radius;
  return HF_OK;
}

int hf_autofocus_exec(hf_autofocus *a, const void *planes, const void *delayed, void *corrected, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(a != nullptr && planes != nullptr && corrected != nullptr, "Autofocus: null argument");
  const int64_t total = (int64_t)a->nz * a->H * a->W;
  HF_TRY(hf::autofocus_begin(a, s));
  for (int pass = 0; pass < a->n_iter; ++pass) {
    // pass 0 measures the current spectrum and corrects the delayed one; later passes measure and
    // correct their predecessor's output (graph_builder.cc:149-153)
    const void *cur = pass == 0 ? planes : corrected;
    const void *del = pass == 0 ? (delayed ? delayed : planes) : corrected;
    HF_TRY(hf::autofocus_measure(a, cur, s));
    if (a->nidx > 0)
      HF_TRY(hf_correct_phase(del, 1, a->phase, a->nz, a->H, a->W, corrected, s));
    else if (del != corrected) // no Zernike orders: a zero phase map, E exp(-i 0) = E
      HF_CUDA(cudaMemcpyAsync(corrected, del, (size_t)total * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  }
  return HF_OK;
}

int hf_autofocus_outputs(const hf_autofocus *a, float *m0, float *slopes, float *coeffs, float *phase, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(a != nullptr, "Autofocus: null argument");
  const size_t nsub = (size_t)a->nb * a->nb;
  const struct {
    float       *dst;
    const float *src;
    size_t       n;
  } cp[4] = {{m0, a->m0, nsub * a->sh * a->sw},
             {slopes, a->slopes, nsub * 2},
             {coeffs, a->cum_coeffs, (size_t)a->nidx},
             {phase, a->cum_phase, (size_t)a->H * a->W}};
  for (const auto &c : cp)
    if (c.dst && c.n)
      HF_CUDA(cudaMemcpyAsync(c.dst, c.src, c.n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  return HF_OK;
}

int hf_autofocus_destroy(hf_autofocus *a) {
  clear_error();
  release(a);
  return HF_OK;
}

} // extern "C"

// ------------------------------------------------------------------------------------------------
// Internal entry points of the fused pipeline (k_shack.cuh)
// ------------------------------------------------------------------------------------------------
namespace hf {
namespace {
// causal_sliding_average_kernel (causal_sliding_average.cu:35-50): in place on the sub-aperture
// images, sum += x - history[slot], history[slot] = x, x = sum / divisor, in float32.
__global__ void shk_causal_avg_kernel(float *x, float *hist, float *sum, int64_t n, float divisor) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float v = x[i], old = hist[i];
    const float s = sum[i] + v - old;
    hist[i] = v;
    sum[i]  = s;
    x[i]    = s / divisor;
  }
}

// lens exp(-i phase): the correction folded into the Fresnel lens that the row pass multiplies by
__global__ void shk_fold_lens_kernel(const float2 *lens, const float *phase, float2 *out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float sv, cv;
    sincosf(phase[i], &sv, &cv);
    const float2 l = lens[i];
    out[i]         = make_float2(l.x * cv + l.y * sv, l.y * cv - l.x * sv);
  }
}
} // namespace

int autofocus_begin(hf_autofocus *a, cudaStream_t s) {
  a->pass = 0;
  HF_CUDA(cudaMemsetAsync(a->cum_coeffs, 0, kShkMaxModes * sizeof(float), s));
  HF_CUDA(cudaMemsetAsync(a->cum_phase, 0, (size_t)a->H * a->W * sizeof(float), s));
  return HF_OK;
}

int autofocus_measure(hf_autofocus *a, const void *planes, cudaStream_t s) {
  HF_TRY(hf_stfd_exec(a->stfd, planes, a->m0, s));
  if (a->acc_n > 1 && a->pass == 0) { // the first pass of a spectrum enters the sliding average
    const int64_t n    = (int64_t)a->nb * a->nb * a->sh * a->sw;
    const int64_t slot = a->acc_count % a->acc_n;
    const float   div  = (float)std::min<int64_t>(a->acc_count + 1, a->acc_n);
    shk_causal_avg_kernel<<<grid_1d(n), 256, 0, s>>>(a->m0, a->acc_hist + slot * n, a->acc_sum, n, div);
    note_launch();
    HF_TRY(launch_status("shk_causal_avg_kernel"));
    ++a->acc_count;
  }
  ++a->pass;
  if (a->ff) // in place: each pass reads its input only where it writes, or before it writes
    HF_TRY(hf_flatfield_exec(a->ff, a->m0, a->m0, s));
  HF_TRY(hf_shslopes_exec(a->sl, a->m0, a->slopes, nullptr, s));
  if (a->nidx > 0) {
    HF_TRY(hf_zernike_fit_exec(a->fit, a->slopes, a->coeffs, a->cum_coeffs, s));
    HF_TRY(hf_zernike_phase(a->coeffs, a->idx, a->nidx, a->H, a->W, a->phase, a->cum_phase, s));
  }
  return HF_OK;
}

int autofocus_correct(hf_autofocus *a, const void *planes, void *out, cudaStream_t s) {
  return hf_correct_phase(planes, 1, a->phase, a->nz, a->H, a->W, out, s);
}

int autofocus_fold_lens(hf_autofocus *a, const float2 *lens, float2 *out, cudaStream_t s) {
  const int64_t n = (int64_t)a->H * a->W;
  shk_fold_lens_kernel<<<grid_1d(n), 256, 0, s>>>(lens, a->phase, out, n);
  note_launch();
  return launch_status("shk_fold_lens_kernel");
}

int autofocus_set_z(hf_autofocus *a, float z, cudaStream_t s) { return hf_stfd_set_z(a->stfd, z, s); }
int autofocus_passes(const hf_autofocus *a) { return a->n_iter; }
int autofocus_orders(const hf_autofocus *a) { return a->nidx; }
const float *autofocus_cumulative_coeffs(const hf_autofocus *a) { return a->cum_coeffs; }

} // namespace hf
