// FP32 C++/OpenMP restatement of the per-window laser Doppler path (plain form) for the host cores.
//
// TEST AND BASELINE INFRASTRUCTURE ONLY: the CPU baseline that bench.py times beside the GPU
// (and the reference arm, `bench.py --impl reference`), checked against the FP64 oracle
// (oracle/oracle.py) by tests/test_cpu_path.py.  The library never links or calls it.
//
// The reference has no host implementation of this path (its arithmetic runs in cuFFT, cuBLAS and
// cuSOLVER on the GPU), so this is a restatement of the same steps, in the reference's order and
// conventions, written for CPUs:
//   1. 12-bit Mono12p (or uint16) frames -> float samples;
//   2. Gram matrix X^T X over the pixels (pca.cc:92-98, no centring, no 1/N): float32 products of
//      the samples shifted by 2048 (exact) summed per 256-pixel block, blocks summed in float64,
//      the shift undone with exact integer frame sums;
//   3. cyclic Jacobi eigendecomposition in float64, ascending (pca_heev.cc order);
//   4. the filter+DFT matrix W = (I - V V^T) D[:, z0:z1] in float64, V the top `clutter_rank`
//      eigenvectors (the one-sided band of rfft.cu + slice, graph_builder.cc:264-267);
//   5. band planes S_k = sum_t x_t W[t][k] in float32, times the Fresnel lens
//      (fresnel_diffraction.cu:326-341: float32 phase, no contraction) when propagating by Fresnel;
//   6. 2D FFT of every plane (radix-2, float32, eight rows per SIMD pass, twiddles from float64
//      sin/cos): Fresnel =
//      forward unnormalised (fresnel_diffraction.cu:427); angular spectrum = forward, times the
//      corner-swapped transfer function (angular_spectrum.cu:261-278, 332-363), inverse
//      unnormalised (408-431);
//   7. |.| and M0/M1/M2 = mean over the band of |S_k|, f_k |S_k|, f_k^2 |S_k| with
//      f_k = arange(z0 df, z1 df, df) in float32, f_k^2 formed in float32 (graph_builder.cc:578-631).
// OpenMP parallelises over pixel blocks (steps 1-2, 5) and over rows of all planes (step 6).
#include <omp.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <vector>

namespace {

using cf = std::complex<float>;
constexpr int kBlock = 256; // pixels per Gram / band block

struct Cfg {
  int32_t H, W, T, z0, z1, clutter_rank, propagation, fmt; // propagation: 0 none, 1 Fresnel, 2 AS
  float   lam, pitch, z, fs;                              // fmt: 16 Mono12p, 1 uint16
};

inline void unpack_block(const uint8_t *frame, int fmt, int64_t p0, int n, float *dst) {
  if (fmt == 16) { // 2 pixels in 3 bytes, p0 even
    const uint8_t *b = frame + (p0 / 2) * 3;
    for (int i = 0; i < n; i += 2, b += 3) {
      dst[i]     = (float)(b[0] | ((b[1] & 0xF) << 8));
      dst[i + 1] = (float)((b[1] >> 4) | (b[2] << 4));
    }
  } else {
    const uint16_t *s = reinterpret_cast<const uint16_t *>(frame) + p0;
    for (int i = 0; i < n; ++i)
      dst[i] = (float)s[i];
  }
}

// Cyclic Jacobi on a symmetric n x n matrix a (row-major, destroyed): eigenvalues ascending in w,
// eigenvector j in column j of v.
void jacobi(std::vector<double> &a, int n, std::vector<double> &w, std::vector<double> &v) {
  v.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    v[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        (i == j ? diag : off) += a[(size_t)i * n + j] * a[(size_t)i * n + j];
    if (off <= 1e-30 * diag || off == 0.0)
      break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[(size_t)p * n + q];
        if (apq == 0.0)
          continue;
        const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) { // columns p, q
          const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
          a[(size_t)k * n + p] = c * akp - s * akq;
          a[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) { // rows p, q
          const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
          a[(size_t)p * n + k] = c * apk - s * aqk;
          a[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
          v[(size_t)k * n + p] = c * vkp - s * vkq;
          v[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i)
    order[i] = i;
  std::sort(order.begin(), order.end(), [&](int x, int y) { return a[(size_t)x * n + x] < a[(size_t)y * n + y]; });
  std::vector<double> vs((size_t)n * n);
  w.resize(n);
  for (int j = 0; j < n; ++j) {
    w[j] = a[(size_t)order[j] * n + order[j]];
    for (int i = 0; i < n; ++i)
      vs[(size_t)i * n + j] = v[(size_t)i * n + order[j]];
  }
  v.swap(vs);
}

// Radix-2 FFTs of 8 rows at once, the rows side by side in SIMD lanes: re/im are [n][8]; the
// gather puts row element j at position bitrev(j), so the butterflies run in natural order.
struct Fft8 {
  int                n, logn;
  std::vector<int>   rev;
  std::vector<float> wr, wi; // exp(-2 pi i k / n), k < n / 2
  explicit Fft8(int n_) : n(n_), logn(0), rev(n_), wr(n_ / 2 > 0 ? n_ / 2 : 1), wi(n_ / 2 > 0 ? n_ / 2 : 1) {
    while ((1 << logn) < n)
      ++logn;
    for (int j = 0; j < n; ++j) {
      int r = 0;
      for (int b = 0; b < logn; ++b)
        r |= ((j >> b) & 1) << (logn - 1 - b);
      rev[j] = r;
    }
    for (int k = 0; k < n / 2; ++k) {
      wr[k] = (float)std::cos(-2.0 * M_PI * k / n);
      wi[k] = (float)std::sin(-2.0 * M_PI * k / n);
    }
  }
  // the 8 rows starting at `data` ([rows][n]) in place; re / im: scratch of n * 8 floats each
  void run8(cf *data, bool inverse, float *re, float *im) const {
    for (int r = 0; r < 8; ++r) {
      const cf *src = data + (int64_t)r * n;
      for (int j = 0; j < n; ++j) {
        re[rev[j] * 8 + r] = src[j].real();
        im[rev[j] * 8 + r] = src[j].imag();
      }
    }
    const float sgn = inverse ? -1.f : 1.f;
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len >> 1, step = n / len;
      for (int i = 0; i < n; i += len)
        for (int k = 0; k < half; ++k) {
          const float w_r = wr[k * step], w_i = sgn * wi[k * step];
          float *ar = re + (i + k) * 8, *ai = im + (i + k) * 8;
          float *br = re + (i + k + half) * 8, *bi = im + (i + k + half) * 8;
#pragma omp simd
          for (int l = 0; l < 8; ++l) {
            const float tr = br[l] * w_r - bi[l] * w_i, ti = br[l] * w_i + bi[l] * w_r;
            br[l] = ar[l] - tr, bi[l] = ai[l] - ti;
            ar[l] = ar[l] + tr, ai[l] = ai[l] + ti;
          }
        }
    }
    for (int r = 0; r < 8; ++r) {
      cf *dst = data + (int64_t)r * n;
      for (int j = 0; j < n; ++j)
        dst[j] = cf(re[j * 8 + r], im[j * 8 + r]);
    }
  }
};

// FFTs of every row of a [rows][n] array (rows a multiple of 8), in parallel.
void fft_rows(cf *data, int64_t rows, const Fft8 &f, bool inverse) {
#pragma omp parallel
  {
    std::vector<float> re((size_t)f.n * 8), im((size_t)f.n * 8);
#pragma omp for schedule(static)
    for (int64_t r = 0; r < rows; r += 8)
      f.run8(data + r * f.n, inverse, re.data(), im.data());
  }
}

// Blocked transpose of nplanes planes [h][w] -> [w][h].
void transpose(const cf *src, cf *dst, int nplanes, int h, int w) {
  constexpr int B = 32;
#pragma omp parallel for collapse(3) schedule(static)
  for (int k = 0; k < nplanes; ++k)
    for (int i0 = 0; i0 < h; i0 += B)
      for (int j0 = 0; j0 < w; j0 += B) {
        const cf *s = src + (int64_t)k * h * w;
        cf       *d = dst + (int64_t)k * h * w;
        for (int i = i0; i < std::min(i0 + B, h); ++i)
          for (int j = j0; j < std::min(j0 + B, w); ++j)
            d[(int64_t)j * h + i] = s[(int64_t)i * w + j];
      }
}

bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Plane buffers kept across calls (as a streaming implementation keeps its working set): no
// allocation, zeroing or first-touch page faults per window once the largest size has been seen.
struct Workspace {
  std::unique_ptr<cf[]> a, b;
  size_t                n = 0;
  cf *get(size_t need, int which) {
    if (need > n) {
      a.reset(reinterpret_cast<cf *>(new float[2 * need]));
      b.reset(reinterpret_cast<cf *>(new float[2 * need]));
      n = need;
    }
    return which ? b.get() : a.get();
  }
};
Workspace g_ws;

} // namespace

extern "C" {

int hfc_version(void) { return 1; }

// OpenMP threads a call with threads <= 0 uses.
int hfc_threads(void) { return omp_get_max_threads(); }

// One window of T frames (consecutive in `frames`, frame_bytes apart) -> out [3][H][W] float32
// (M0, M1, M2).  threads <= 0: all OpenMP threads.  Returns 0, or -1 for an unsupported setting.
static double now_s() { return omp_get_wtime(); }
static void phase(const char *name, double &t) {
  static const bool on = getenv("HFC_TIMING") != nullptr;
  const double n = now_s();
  if (on)
    fprintf(stderr, "%-10s %.4f s\n", name, n - t);
  t = n;
}

int hfc_window(const Cfg *c, const uint8_t *frames, float *out, int threads) {
  double tph = now_s();
  const int     H = c->H, W = c->W, T = c->T, nz = c->z1 - c->z0;
  const int64_t P = (int64_t)H * W;
  if (!pow2(H) || !pow2(W) || H < 8 || W < 8 || T < 2 || T > 256 || nz < 1 || c->z0 < 0 || c->z1 > T || P % kBlock != 0 ||
      (c->fmt != 16 && c->fmt != 1) || c->clutter_rank < 0 || c->clutter_rank >= T)
    return -1;
  if (threads > 0)
    omp_set_num_threads(threads);
  const int64_t fbytes = c->fmt == 16 ? P * 3 / 2 : P * 2;
  const int64_t nblk   = P / kBlock;

  // ---- Gram matrix (only when the clutter filter needs it) ----------------------------------------
  std::vector<double> V;
  if (c->clutter_rank > 0) {
    std::vector<double>  gram((size_t)T * T, 0.0);
    std::vector<int64_t> colsum(T, 0);
#pragma omp parallel
    {
      std::vector<double>  g((size_t)T * T, 0.0);
      std::vector<int64_t> cs(T, 0);
      std::vector<float>   x((size_t)T * kBlock), gb((size_t)T * T);
#pragma omp for schedule(static)
      for (int64_t b = 0; b < nblk; ++b) {
        for (int t = 0; t < T; ++t) {
          float *xt = x.data() + (size_t)t * kBlock;
          unpack_block(frames + t * fbytes, c->fmt, b * kBlock, kBlock, xt);
          int64_t s = 0;
          for (int i = 0; i < kBlock; ++i) {
            s += (int64_t)xt[i];
            xt[i] -= 2048.f; // exact; products of shifted samples sum exactly in float per block
          }
          cs[t] += s;
        }
        for (int t1 = 0; t1 < T; ++t1)
          for (int t2 = t1; t2 < T; ++t2) {
            const float *a = x.data() + (size_t)t1 * kBlock, *bb = x.data() + (size_t)t2 * kBlock;
            float        acc = 0.f;
#pragma omp simd reduction(+ : acc)
            for (int i = 0; i < kBlock; ++i)
              acc += a[i] * bb[i];
            gb[(size_t)t1 * T + t2] = acc;
          }
        for (int t1 = 0; t1 < T; ++t1)
          for (int t2 = t1; t2 < T; ++t2)
            g[(size_t)t1 * T + t2] += gb[(size_t)t1 * T + t2];
      }
#pragma omp critical
      {
        for (size_t i = 0; i < g.size(); ++i)
          gram[i] += g[i];
        for (int t = 0; t < T; ++t)
          colsum[t] += cs[t];
      }
    }
    // (x' + 2048)^T (x' + 2048) = x'^T x' + 2048 (s'_i + s'_j) + 2048^2 P, s' = s - 2048 P
    for (int t1 = 0; t1 < T; ++t1)
      for (int t2 = t1; t2 < T; ++t2) {
        const double s1 = (double)colsum[t1] - 2048.0 * P, s2 = (double)colsum[t2] - 2048.0 * P;
        const double v  = gram[(size_t)t1 * T + t2] + 2048.0 * (s1 + s2) + 2048.0 * 2048.0 * (double)P;
        gram[(size_t)t1 * T + t2] = gram[(size_t)t2 * T + t1] = v;
      }
    std::vector<double> w, vec;
    jacobi(gram, T, w, vec);
    V.assign((size_t)T * c->clutter_rank, 0.0);
    for (int t = 0; t < T; ++t)
      for (int r = 0; r < c->clutter_rank; ++r)
        V[(size_t)t * c->clutter_rank + r] = vec[(size_t)t * T + (T - c->clutter_rank + r)];
  }

  phase("gram+eig", tph);
  // ---- W = (I - V V^T) D[:, z0:z1] ---------------------------------------------------------------
  std::vector<std::complex<double>> Wd((size_t)T * nz);
  for (int t = 0; t < T; ++t)
    for (int k = 0; k < nz; ++k) {
      const int64_t m = ((int64_t)t * (c->z0 + k)) % T;
      Wd[(size_t)t * nz + k] = std::polar(1.0, -2.0 * M_PI * (double)m / T);
    }
  if (c->clutter_rank > 0) {
    const int r = c->clutter_rank;
    std::vector<std::complex<double>> VtD((size_t)r * nz, 0.0);
    for (int j = 0; j < r; ++j)
      for (int k = 0; k < nz; ++k)
        for (int t = 0; t < T; ++t)
          VtD[(size_t)j * nz + k] += V[(size_t)t * r + j] * Wd[(size_t)t * nz + k];
    for (int t = 0; t < T; ++t)
      for (int k = 0; k < nz; ++k) {
        std::complex<double> s = 0.0;
        for (int j = 0; j < r; ++j)
          s += V[(size_t)t * r + j] * VtD[(size_t)j * nz + k];
        Wd[(size_t)t * nz + k] -= s;
      }
  }
  std::vector<float> Wr((size_t)T * nz), Wi((size_t)T * nz);
  for (size_t i = 0; i < Wd.size(); ++i)
    Wr[i] = (float)Wd[i].real(), Wi[i] = (float)Wd[i].imag();

  // ---- Fresnel lens (float32 phase as quadratic_lens_kernel, then cos / sin in float64) ----------
  std::vector<cf> lens;
  if (c->propagation == 1) {
    lens.resize((size_t)P);
    const int   size = std::max(H, W);
    const float half = (float)size / 2.0f, dx = c->pitch;
    const float kk   = (float)M_PI / (c->lam * c->z);
#pragma omp parallel for schedule(static)
    for (int r = 0; r < H; ++r) {
      volatile float y = ((float)(r + (size - H) / 2) - half) * dx;
      for (int col = 0; col < W; ++col) {
        volatile float x  = ((float)(col + (size - W) / 2) - half) * dx;
        volatile float xx = x * x, yy = y * y;
        volatile float r2 = xx + yy;
        volatile float ph = kk * r2;
        lens[(size_t)r * W + col] = cf((float)std::cos((double)ph), (float)std::sin((double)ph));
      }
    }
  }

  // ---- band planes [nz][P]: a [256 x T] x [T x 2 nz] product per pixel block, 8 pixels x 4 bins
  // (8 real accumulators) per register block ------------------------------------------------------
  const int nzp = (nz + 3) / 4 * 4;
  std::vector<float> Wc((size_t)T * 2 * nzp, 0.f); // [t][2 k + {re, im}], bins padded to 4
  for (int t = 0; t < T; ++t)
    for (int k = 0; k < nz; ++k) {
      Wc[(size_t)t * 2 * nzp + 2 * k]     = Wr[(size_t)t * nz + k];
      Wc[(size_t)t * 2 * nzp + 2 * k + 1] = Wi[(size_t)t * nz + k];
    }
  phase("w+lens", tph);
  cf *planes = g_ws.get((size_t)nz * P, 0);
  phase("alloc", tph);
#pragma omp parallel
  {
    std::vector<float> x((size_t)T * kBlock);
#pragma omp for schedule(static)
    for (int64_t b = 0; b < nblk; ++b) {
      for (int t = 0; t < T; ++t)
        unpack_block(frames + t * fbytes, c->fmt, b * kBlock, kBlock, x.data() + (size_t)t * kBlock);
      for (int k0 = 0; k0 < nz; k0 += 4)
        for (int i0 = 0; i0 < kBlock; i0 += 8) {
          float acc[8][8] = {};
          for (int t = 0; t < T; ++t) {
            const float *xt = x.data() + (size_t)t * kBlock + i0;
            const float *wt = Wc.data() + (size_t)t * 2 * nzp + 2 * k0;
            for (int j = 0; j < 8; ++j) {
              const float wj = wt[j];
#pragma omp simd
              for (int i = 0; i < 8; ++i)
                acc[j][i] += xt[i] * wj;
            }
          }
          for (int kk = 0; kk < 4 && k0 + kk < nz; ++kk) {
            cf *dst = planes + (size_t)(k0 + kk) * P + b * kBlock + i0;
            for (int i = 0; i < 8; ++i) {
              const float sr = acc[2 * kk][i], si = acc[2 * kk + 1][i];
              if (c->propagation == 1) {
                const cf L = lens[(size_t)(b * kBlock + i0 + i)];
                dst[i] = cf(sr * L.real() - si * L.imag(), sr * L.imag() + si * L.real());
              } else {
                dst[i] = cf(sr, si);
              }
            }
          }
        }
    }
  }

  phase("band", tph);
  // ---- propagation: 2D FFTs; `tr` says whether the planes are left transposed ([W][H]) -------------
  bool tr = false;
  if (c->propagation == 1 || c->propagation == 2) {
    const Fft8            fW(W), fH(H);
    cf                   *tmp = g_ws.get((size_t)nz * P, 1);
    fft_rows(planes, (int64_t)nz * H, fW, false);
    transpose(planes, tmp, nz, H, W); // [nz][W][H]
    fft_rows(tmp, (int64_t)nz * W, fH, false);
    if (c->propagation == 1) {
      planes = tmp;
      tr     = true;
    } else {
      // transfer function exp(i 2 pi z / lam sqrt(max(0, 1 - lam^2 (u^2 + v^2)))) in float32
      // arithmetic (spectral_lens_kernel), corner-swapped, applied in the transposed layout
      std::vector<cf> tf((size_t)P);
      const float     lam = c->lam, zf = c->z, px = c->pitch;
      const float     du = 1.0f / ((float)W * px), dv = 1.0f / ((float)H * px);
      const float     kk = (2.0f * (float)M_PI * zf) / lam;
      for (int r = 0; r < H; ++r)
        for (int col = 0; col < W; ++col) {
          volatile float u = (float)(col - W / 2) * du, v = (float)(r - H / 2) * dv;
          volatile float s = u * u + v * v;
          volatile float l2 = lam * lam;
          volatile float tmpv = 1.0f - l2 * s;
          const float    tm = tmpv > 0.f ? (float)tmpv : 0.f;
          volatile float ph = kk * std::sqrt(tm);
          const int      rr = (r + H / 2) % H, cc = (col + W / 2) % W; // swap_corners (even sizes)
          tf[(size_t)rr * W + cc] = cf((float)std::cos((double)ph), (float)std::sin((double)ph));
        }
#pragma omp parallel for schedule(static)
      for (int64_t k = 0; k < nz; ++k)
        for (int col = 0; col < W; ++col)
          for (int r = 0; r < H; ++r)
            tmp[(size_t)k * P + (size_t)col * H + r] *= tf[(size_t)r * W + col];
      fft_rows(tmp, (int64_t)nz * W, fH, true);
      transpose(tmp, planes, nz, W, H); // back to [nz][H][W]
      fft_rows(planes, (int64_t)nz * H, fW, true);
    }
  }

  phase("fft", tph);
  // ---- |.| and moments ------------------------------------------------------------------------------
  const double df = (double)c->fs / T;
  std::vector<float> w1(nz), w2(nz);
  for (int k = 0; k < nz; ++k) {
    w1[k] = (float)(c->z0 * df + df * (double)k);
    w2[k] = w1[k] * w1[k];
  }
  const float inv = 1.0f / (float)nz;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < P; ++p) {
    double m0 = 0, m1 = 0, m2 = 0;
    for (int k = 0; k < nz; ++k) {
      const cf    v = planes[(size_t)k * P + p];
      const float a = std::sqrt(v.real() * v.real() + v.imag() * v.imag());
      m0 += a;
      m1 += (double)(w1[k] * a);
      m2 += (double)(w2[k] * a);
    }
    const int64_t q = tr ? (p % H) * W + p / H : p; // transposed layout: p = col * H + row
    out[q]         = (float)m0 * inv;
    out[P + q]     = (float)m1 * inv;
    out[2 * P + q] = (float)m2 * inv;
  }
  phase("moments", tph);
  return 0;
}

} // extern "C"
