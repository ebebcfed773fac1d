// PCA / SVD clutter filter kernels: Gram matrix of a window's frames, FP64 Jacobi
// eigendecomposition, the filter+DFT matrix of the band, and the PCA projection.
//
// Reference: PcaTask::execute (holotask/src/syncs/pca.cc:68-119) computes C = X^T X with
// cublasGemmEx (FP16 tensor-core compute), an ascending eigendecomposition with cuSolverDx heev
// (pca_heev.cc:35-133) and the projection X V[:, begin:end].  Here the Gram matrix is
// accumulated in FP32 over pixel tiles on shifted samples (x - 2048 is exact for 12-bit data)
// and reduced in FP64 with the shift undone exactly; the eigensolver is FP64 throughout.
#include <algorithm>
#include <cfloat>
#include <mutex>
#include <string>

#include "k_pca.cuh"

namespace hf {

namespace {

constexpr int kCovPT = 128; // pixels per tile

template <int T> struct CovGeom {
  static constexpr int NB     = T / 4;                 // 4x4 blocks per side
  static constexpr int U      = NB * (NB + 1) / 2;     // upper-triangle blocks
  static constexpr int G      = T == 32 ? 4 : (T == 64 ? 2 : 1); // pixel groups
  static constexpr int THR    = U * G;
  static constexpr int XS     = T + 4;                 // padded row of the unpacked tile
};

template <int FMT> struct Bpp;  // bytes per pixel (numerator / denominator)
template <> struct Bpp<HF_MONO12P> { static constexpr int num = 3, den = 2; };
template <> struct Bpp<HF_U16> { static constexpr int num = 2, den = 1; };
template <> struct Bpp<HF_U8> { static constexpr int num = 1, den = 1; };
template <> struct Bpp<HF_F32> { static constexpr int num = 4, den = 1; };

template <int FMT, int T>
__global__ void __launch_bounds__(CovGeom<T>::THR) cov_tiled_kernel(CovArgs a) {
  using Gm = CovGeom<T>;
  constexpr int RB  = kCovPT * Bpp<FMT>::num / Bpp<FMT>::den; // packed bytes per frame row
  constexpr int RW  = RB / 4 + 1;                             // padded words per staged row
  extern __shared__ __align__(16) uint8_t smem[];
  uint32_t *stage = reinterpret_cast<uint32_t *>(smem);             // [T][RW]
  float    *xs    = reinterpret_cast<float *>(smem + T * RW * 4);  // [PT][XS]
  unsigned long long *ssum = reinterpret_cast<unsigned long long *>(xs + kCovPT * Gm::XS); // [T]

  const int tid = threadIdx.x;
  const int w   = blockIdx.y;
  const int grp = tid / Gm::U, blk = tid % Gm::U;
  // upper-triangle block index -> (bi, bj), bi <= bj
  int bi = 0, rem = blk;
  while (rem >= Gm::NB - bi) {
    rem -= Gm::NB - bi;
    ++bi;
  }
  const int bj = bi + rem;

  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
      acc[i][j] = 0.f;
  for (int t = tid; t < T; t += blockDim.x)
    ssum[t] = 0;

  const int64_t ntiles = (a.P + kCovPT - 1) / kCovPT;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t p0 = tile * kCovPT;
    const int     np = (int)min((int64_t)kCovPT, a.P - p0);
    const int     nw = (np * Bpp<FMT>::num / Bpp<FMT>::den + 3) / 4;
    __syncthreads();
    for (int i = tid; i < T * (RB / 4); i += blockDim.x) {
      const int t = i / (RB / 4), j = i % (RB / 4);
      const uint32_t *src = reinterpret_cast<const uint32_t *>(
          a.ring.frame(w, t) + p0 * Bpp<FMT>::num / Bpp<FMT>::den);
      stage[t * RW + j] = j < nw ? __ldg(src + j) : 0u;
    }
    __syncthreads();
    // unpack: thread (t, 8-pixel group); lanes run along t (conflict-free xs writes)
    for (int i = tid; i < T * (kCovPT / 8); i += blockDim.x) {
      const int t = i % T, g = i / T;
      float     v[8];
      if constexpr (FMT == HF_MONO12P) {
        uint32_t p[8];
        unpack8(stage[t * RW + 3 * g], stage[t * RW + 3 * g + 1], stage[t * RW + 3 * g + 2], p);
#pragma unroll
        for (int k = 0; k < 8; ++k)
          v[k] = (float)p[k];
      } else if constexpr (FMT == HF_U16) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const uint32_t wv = stage[t * RW + 4 * g + k];
          v[2 * k]     = (float)(wv & 0xFFFFu);
          v[2 * k + 1] = (float)(wv >> 16);
        }
      } else if constexpr (FMT == HF_U8) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const uint32_t wv = stage[t * RW + 2 * g + k];
#pragma unroll
          for (int j = 0; j < 4; ++j)
            v[4 * k + j] = (float)((wv >> (8 * j)) & 0xFFu);
        }
      } else {
#pragma unroll
        for (int k = 0; k < 8; ++k)
          v[k] = __uint_as_float(stage[t * RW + 8 * g + k]);
      }
      unsigned int isum = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int p = 8 * g + k;
        const bool in = p < np;
        if constexpr (FMT != HF_F32)
          isum += in ? (unsigned int)v[k] : 0u;
        xs[p * Gm::XS + t] = in ? v[k] - a.shift : 0.f;
      }
      if constexpr (FMT != HF_F32)
        atomicAdd(&ssum[t], (unsigned long long)isum);
    }
    __syncthreads();
    // accumulate this group's share of the tile
    if (grp < Gm::G) {
      for (int p = grp; p < kCovPT; p += Gm::G) {
        const float4 xa = *reinterpret_cast<const float4 *>(xs + p * Gm::XS + 4 * bi);
        const float4 xb = *reinterpret_cast<const float4 *>(xs + p * Gm::XS + 4 * bj);
        const float  va[4] = {xa.x, xa.y, xa.z, xa.w};
        const float  vb[4] = {xb.x, xb.y, xb.z, xb.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j)
            acc[i][j] = fmaf(va[i], vb[j], acc[i][j]);
      }
    }
  }
  __syncthreads();
  if (grp < Gm::G) {
    const int64_t pidx = ((int64_t)w * a.nblk + (int64_t)blockIdx.x * Gm::G + grp) * T * T;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
        a.partial[pidx + (4 * bi + i) * T + 4 * bj + j] = acc[i][j];
  }
  for (int t = tid; t < T; t += blockDim.x)
    a.sums[((int64_t)w * gridDim.x + blockIdx.x) * T + t] = (double)ssum[t];
}

// Deterministic reduction of the partials; undoes the shift exactly (float64).
__global__ void cov_finalize_kernel(const float *partial, const double *sums, int nblk,
                                    int nsum, int T, int64_t P, double shift, double *gram) {
  const int w = blockIdx.y;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= T * T)
    return;
  const int i = e / T, j = e % T;
  if (i > j)
    return;
  // the tiled kernel writes every entry (i, j) with block(i) <= block(j), so i <= j is present
  double g = 0.0;
  const float *pp = partial + (int64_t)w * nblk * T * T + i * T + j;
  for (int b = 0; b < nblk; ++b)
    g += (double)pp[(int64_t)b * T * T];
  if (shift != 0.0) {
    double si = 0.0, sj = 0.0;
    const double *sp = sums + (int64_t)w * nsum * T;
    for (int b = 0; b < nsum; ++b) {
      si += sp[(int64_t)b * T + i];
      sj += sp[(int64_t)b * T + j];
    }
    g += shift * (si + sj) - shift * shift * (double)P;
  }
  gram[(int64_t)w * T * T + i * T + j] = g;
  gram[(int64_t)w * T * T + j * T + i] = g;
}

// Any T (small problems): one thread per upper entry, float64 accumulation, no shift.
template <int FMT>
__global__ void cov_generic_kernel(FrameRing ring, int T, int64_t P, double *gram) {
  const int w = blockIdx.y;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= T * T)
    return;
  const int i = e / T, j = e % T;
  if (i > j)
    return;
  const uint8_t *fi = ring.frame(w, i), *fj = ring.frame(w, j);
  double g = 0.0;
  for (int64_t p = 0; p < P; ++p)
    g += (double)sample<FMT>(fi, p) * (double)sample<FMT>(fj, p);
  gram[(int64_t)w * T * T + i * T + j] = g;
  gram[(int64_t)w * T * T + j * T + i] = g;
}

int cov_ctas_per_window(int64_t P, int nwin) {
  const int64_t ntiles = (P + kCovPT - 1) / kCovPT;
  int           ctas   = (2 * sm_count() + nwin - 1) / nwin;
  ctas = (int)std::max<int64_t>(1, std::min<int64_t>(ctas, ntiles));
  return ctas;
}

// `max_ctas` > 0 caps the CTAs per window (and so the workspace) below the default split.
template <int FMT, int T>
int launch_cov_tiled(const FrameRing &ring, int64_t P, int nwin, void *ws, double *gram,
                     cudaStream_t s, int max_ctas = 0) {
  using Gm = CovGeom<T>;
  constexpr int RB   = kCovPT * Bpp<FMT>::num / Bpp<FMT>::den;
  constexpr int RW   = RB / 4 + 1;
  const size_t  smem = (size_t)T * RW * 4 + (size_t)kCovPT * Gm::XS * 4 + T * 8;
  const int     ctas = max_ctas > 0 ? std::min(max_ctas, cov_ctas_per_window(P, nwin))
                                    : cov_ctas_per_window(P, nwin);
  CovArgs       a;
  a.ring    = ring;
  a.T       = T;
  a.P       = P;
  a.shift   = FMT == HF_F32 ? 0.f : (FMT == HF_U8 ? 128.f : 2048.f);
  a.nblk    = ctas * Gm::G;
  a.partial = reinterpret_cast<float *>(ws);
  a.sums    = reinterpret_cast<double *>(reinterpret_cast<uint8_t *>(ws) +
                                      (size_t)nwin * a.nblk * T * T * sizeof(float));
  HF_CUDA(cudaFuncSetAttribute(cov_tiled_kernel<FMT, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  cov_tiled_kernel<FMT, T><<<dim3(ctas, nwin), Gm::THR, smem, s>>>(a);
  note_launch();
  HF_TRY(launch_status("cov_tiled_kernel"));
  return launch_cov_finalize(a.partial, a.sums, a.nblk, ctas, T, P, (double)a.shift, gram, nwin, s);
}

template <int FMT>
int launch_cov_fmt(const FrameRing &ring, int T, int64_t P, int nwin, void *ws, double *gram,
                   cudaStream_t s) {
  if constexpr (FMT != HF_CF32) {
    // the tiled kernel reads frames as 4-byte words: the base must be 4-byte aligned too
    const bool tiled = (P % 8 == 0) && (ring.frame_bytes % 4 == 0) && (((uintptr_t)ring.base & 3) == 0);
    if (tiled && T == 32)
      return launch_cov_tiled<FMT, 32>(ring, P, nwin, ws, gram, s);
    if (tiled && T == 64)
      return launch_cov_tiled<FMT, 64>(ring, P, nwin, ws, gram, s);
    if (tiled && T == 128)
      return launch_cov_tiled<FMT, 128>(ring, P, nwin, ws, gram, s);
  }
  cov_generic_kernel<FMT><<<dim3((T * T + 127) / 128, nwin), 128, 0, s>>>(ring, T, P, gram);
  note_launch();
  return launch_status("cov_generic_kernel");
}

// ------------------------------------------------------------------------------------------------
// Jacobi
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void pair_of(int r, int k, int n, int &p, int &q) {
  if (k == 0) {
    p = n - 1;
    q = r;
  } else {
    p = (r + k) % (n - 1);
    q = (r - k + (n - 1)) % (n - 1);
  }
  if (p > q) {
    const int t = p;
    p = q;
    q = t;
  }
}

// Packed upper-triangle index of the symmetric matrix (i <= j).
__device__ __forceinline__ int sym_idx(int i, int j, int np) {
  if (i > j) {
    const int t = i;
    i = j;
    j = t;
  }
  return i * np - (i * (i - 1)) / 2 + (j - i);
}

// Parallel cyclic Jacobi (round-robin pairing, np/2 disjoint rotations per step).  The matrix is
// kept as a packed upper triangle and the rotation accumulator transposed (Vt[p][:] = V[:, p]),
// both in shared memory (194 KB at n = 128).  Every thread owns a fixed set of 2x2 blocks (k, l)
// and accumulator entries for the whole solve, so a step is: rotations of the np/2 pairs,
// barrier, block and accumulator updates, barrier.
constexpr int kJacobiThreads = 1024;
constexpr int kJacobiMaxBlk  = 3;  // 2x2 blocks per thread: ceil(65*64/2 / 1024)
constexpr int kJacobiMaxV    = 8;  // accumulator entries per thread: 64*128 / 1024

__global__ void __launch_bounds__(kJacobiThreads) jacobi_kernel(const double *a_in, double *evecs,
                                                                double *evals, int *info, int n) {
  extern __shared__ __align__(16) double dsm[];
  const int np   = n + (n & 1);
  const int half = np / 2;
  const int npk  = np * (np + 1) / 2;
  double   *A    = dsm;                                    // packed [npk]
  double   *Vt   = A + npk;                                // [np][np]
  double   *cs   = Vt + np * np;                           // [half][2]
  int      *pq   = reinterpret_cast<int *>(cs + 2 * half); // [half][2]
  int      *flag = pq + 2 * half;
  const int tid = threadIdx.x, nt = blockDim.x;
  const double *src = a_in + (int64_t)blockIdx.x * n * n;

  for (int e = tid; e < np * np; e += nt) {
    const int i = e / np, j = e % np;
    Vt[e] = i == j ? 1.0 : 0.0;
    if (i <= j) {
      double v = 0.0;
      if (i < n && j < n)
        v = 0.5 * (src[i * n + j] + src[j * n + i]);
      else if (i == j)
        v = -DBL_MAX; // padding entry of an odd order: sorts first and is dropped
      A[sym_idx(i, j, np)] = v;
    }
  }
  // absolute rotation threshold: entries below 2^-52 of the trace (the matrix is a Gram matrix,
  // so the trace bounds its norm) are at the rounding level of the largest eigenvalues and cannot
  // be reduced further by two-sided rotations
  __syncthreads(); // the cooperative load of A above must be complete
  if (tid == 0) {
    double tr = 0.0;
    for (int i = 0; i < n; ++i)
      tr += fabs(A[sym_idx(i, i, np)]);
    cs[0] = tr * 2.220446049250313e-16;
  }
  __syncthreads();
  const double tol_abs = cs[0];
  __syncthreads();
  // this thread's fixed work items
  const int nblocks = half * (half + 1) / 2;
  int       bk[kJacobiMaxBlk], bl[kJacobiMaxBlk], nb = 0;
  for (int e = tid; e < nblocks && nb < kJacobiMaxBlk; e += nt) {
    int k = 0, rem = e;
    while (rem >= half - k) {
      rem -= half - k;
      ++k;
    }
    bk[nb] = k;
    bl[nb] = k + rem;
    ++nb;
  }
  int vk[kJacobiMaxV], vj[kJacobiMaxV], nv = 0;
  for (int f = tid; f < half * np && nv < kJacobiMaxV; f += nt) {
    vk[nv] = f / np;
    vj[nv] = f % np;
    ++nv;
  }
  __syncthreads();

  const int max_sweeps = 40;
  int       sweep      = 0;
  for (; sweep < max_sweeps; ++sweep) {
    if (tid == 0)
      flag[0] = 0;
    __syncthreads();
    for (int r = 0; r < np - 1; ++r) {
      if (tid < half) {
        int p, q;
        pair_of(r, tid, np, p, q);
        const double app = A[sym_idx(p, p, np)], aqq = A[sym_idx(q, q, np)];
        const double apq = A[sym_idx(p, q, np)];
        double       c = 1.0, s = 0.0;
        const bool   pad = (p >= n) || (q >= n);
        if (!pad && fabs(apq) > tol_abs && fabs(apq) > 1e-15 * sqrt(fabs(app * aqq))) {
          // t = tan(phi) of the annihilating rotation, the smaller root of t^2 + 2 theta t - 1 = 0
          // with theta = d / (2 apq), d = aqq - app, written with one square root and one division
          const double d  = aqq - app;
          const double a2 = 2.0 * apq;
          const double t  = (d >= 0.0 ? a2 : -a2) / (fabs(d) + sqrt(fma(d, d, a2 * a2)));
          c = rsqrt(fma(t, t, 1.0));
          s = t * c;
          flag[0] = 1;
        }
        cs[2 * tid]     = c;
        cs[2 * tid + 1] = s;
        pq[2 * tid]     = p;
        pq[2 * tid + 1] = q;
      }
      __syncthreads();
#pragma unroll
      for (int b = 0; b < kJacobiMaxBlk; ++b) {
        if (b >= nb)
          break;
        const int    k = bk[b], l = bl[b];
        const double ck = cs[2 * k], sk = cs[2 * k + 1], cl = cs[2 * l], sl = cs[2 * l + 1];
        if (sk == 0.0 && sl == 0.0)
          continue;
        const int pk = pq[2 * k], qk = pq[2 * k + 1], pl = pq[2 * l], ql = pq[2 * l + 1];
        const int i00 = sym_idx(pk, pl, np), i01 = sym_idx(pk, ql, np);
        const int i10 = sym_idx(qk, pl, np), i11 = sym_idx(qk, ql, np);
        const double b00 = A[i00], b01 = A[i01], b10 = A[i10], b11 = A[i11];
        // M = B J_l ;  B' = J_k^T M   with J = [[c, s], [-s, c]]
        const double m00 = cl * b00 - sl * b01, m01 = sl * b00 + cl * b01;
        const double m10 = cl * b10 - sl * b11, m11 = sl * b10 + cl * b11;
        const double n00 = ck * m00 - sk * m10, n01 = ck * m01 - sk * m11;
        const double n10 = sk * m00 + ck * m10, n11 = sk * m01 + ck * m11;
        if (k == l) { // diagonal block: i01 == i10 is the annihilated entry
          A[i00] = n00;
          A[i11] = n11;
          A[i01] = 0.0;
        } else {
          A[i00] = n00;
          A[i01] = n01;
          A[i10] = n10;
          A[i11] = n11;
        }
      }
#pragma unroll
      for (int v = 0; v < kJacobiMaxV; ++v) {
        if (v >= nv)
          break;
        const int    k = vk[v], j = vj[v];
        const double c = cs[2 * k], s = cs[2 * k + 1];
        if (s != 0.0) {
          const int    p = pq[2 * k], q = pq[2 * k + 1];
          const double vp = Vt[p * np + j], vq = Vt[q * np + j];
          Vt[p * np + j] = c * vp - s * vq;
          Vt[q * np + j] = s * vp + c * vq;
        }
      }
      __syncthreads();
    }
    const int any = flag[0];
    __syncthreads();
    if (any == 0)
      break;
  }
  // ascending rank sort (ties by index) and write out
  double *ev  = evals + (int64_t)blockIdx.x * n;
  double *vec = evecs + (int64_t)blockIdx.x * n * n;
  for (int i = tid; i < np; i += nt) {
    const double li   = A[sym_idx(i, i, np)];
    int          rank = 0;
    for (int j = 0; j < np; ++j) {
      const double lj = A[sym_idx(j, j, np)];
      rank += (lj < li) || (lj == li && j < i);
    }
    if (np != n)
      rank -= 1;
    if (i < n) {
      ev[rank] = li;
      for (int t = 0; t < n; ++t)
        vec[t * n + rank] = Vt[i * np + t];
    }
  }
  if (tid == 0 && info != nullptr)
    info[blockIdx.x] = (sweep >= max_sweeps) ? sweep : 0;
}

// W = (I - V V^T) D[:, bins]; one CTA per window.  bins = [z0, z1), followed for the two-sided
// method by [T - z1, T - z0) (graph_builder.cc:270-287: the positive then the negative band).
__device__ __forceinline__ int band_bin(int kk, int z0, int z1, int T) {
  const int nzh = z1 - z0;
  return kk < nzh ? z0 + kk : T - z1 + (kk - nzh);
}

__global__ void band_matrix_kernel(const double *evecs, int T, int rank, int z0, int z1, int two_sided,
                                   float2 *wmat) {
  extern __shared__ __align__(16) double bsm[];
  const int     nz = (z1 - z0) * (two_sided ? 2 : 1);
  const double *V  = evecs + (int64_t)blockIdx.x * T * T;
  double       *cr = bsm;            // [rank][nz] re
  double       *ci = bsm + rank * nz; // [rank][nz] im
  for (int e = threadIdx.x; e < rank * nz; e += blockDim.x) {
    const int m = e / nz, kk = e % nz;
    const int col = T - rank + m;
    double    sr = 0.0, si = 0.0;
    for (int t = 0; t < T; ++t) {
      double s, c;
      sincospi(-2.0 * (double)((t * band_bin(kk, z0, z1, T)) % T) / (double)T, &s, &c);
      sr += V[t * T + col] * c;
      si += V[t * T + col] * s;
    }
    cr[e] = sr;
    ci[e] = si;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < T * nz; e += blockDim.x) {
    const int t = e / nz, kk = e % nz;
    double    s, c;
    sincospi(-2.0 * (double)((t * band_bin(kk, z0, z1, T)) % T) / (double)T, &s, &c);
    double wr = c, wi = s;
    for (int m = 0; m < rank; ++m) {
      const double v = V[t * T + (T - rank + m)];
      wr -= v * cr[m * nz + kk];
      wi -= v * ci[m * nz + kk];
    }
    wmat[(int64_t)blockIdx.x * T * nz + e] = make_float2((float)wr, (float)wi);
  }
}

__global__ void pca_project_kernel(const float *in, int T, int64_t P, const double *evecs,
                                   int begin, int ncomp, float *out) {
  extern __shared__ float vsh[]; // [T][ncomp]
  const int64_t b = blockIdx.y;
  const double *V = evecs + b * T * T;
  for (int e = threadIdx.x; e < T * ncomp; e += blockDim.x)
    vsh[e] = (float)V[(e / ncomp) * T + begin + (e % ncomp)];
  __syncthreads();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P)
    return;
  const float *x = in + b * T * P + p;
  for (int c0 = 0; c0 < ncomp; c0 += 8) {
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int t = 0; t < T; ++t) {
      const float xv = x[(int64_t)t * P];
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (c0 + j < ncomp)
          acc[j] = fmaf(xv, vsh[t * ncomp + c0 + j], acc[j]);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (c0 + j < ncomp)
        out[(b * ncomp + c0 + j) * P + p] = acc[j];
  }
}

} // namespace

int launch_cov_finalize(const float *partial, const double *sums, int nblk, int nsum, int T, int64_t P,
                        double shift, double *gram, int nwin, cudaStream_t s) {
  cov_finalize_kernel<<<dim3((T * T + 255) / 256, nwin), 256, 0, s>>>(partial, sums, nblk, nsum, T, P, shift,
                                                                      gram);
  note_launch();
  return launch_status("cov_finalize_kernel");
}

size_t cov_workspace_bytes(int T, int64_t P, int nwin) {
  const int ctas = cov_ctas_per_window(P, nwin);
  const int G    = T == 32 ? 4 : (T == 64 ? 2 : 1);
  return (size_t)nwin * ctas * G * T * T * sizeof(float) + (size_t)nwin * ctas * T * sizeof(double) + 256;
}

int launch_covariance(const FrameRing &ring, int fmt, int T, int64_t P, int nwin, void *ws,
                      double *gram, cudaStream_t s) {
  HF_CHECK_ARG(T > 0 && P > 0 && nwin > 0, "covariance: empty problem");
  switch (fmt) {
  case HF_MONO12P: return launch_cov_fmt<HF_MONO12P>(ring, T, P, nwin, ws, gram, s);
  case HF_U16: return launch_cov_fmt<HF_U16>(ring, T, P, nwin, ws, gram, s);
  case HF_U8: return launch_cov_fmt<HF_U8>(ring, T, P, nwin, ws, gram, s);
  case HF_F32: return launch_cov_fmt<HF_F32>(ring, T, P, nwin, ws, gram, s);
  default: return fail(HF_ERR_INVALID, "covariance: unsupported input dtype");
  }
}

int launch_jacobi(const double *a, double *evecs, double *evals, int *info, int n, int64_t batch,
                  cudaStream_t s) {
  HF_CHECK_ARG(n >= 1 && n <= 128 && batch >= 1, "jacobi: order must be in [1, 128]");
  const int    np   = n + (n & 1);
  const size_t smem = (size_t)(np * (np + 1) / 2) * 8 + (size_t)np * np * 8 + (size_t)np * 8 +
                      (size_t)np * 4 + 16;
  HF_CUDA(cudaFuncSetAttribute(jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  jacobi_kernel<<<(unsigned)batch, kJacobiThreads, smem, s>>>(a, evecs, evals, info, n);
  note_launch();
  return launch_status("jacobi_kernel");
}

int launch_band_matrix(const double *evecs, int64_t batch, int T, int rank, int z0, int z1,
                       float2 *wmat, cudaStream_t s, bool two_sided) {
  HF_CHECK_ARG(T > 0 && z0 >= 0 && z1 > z0 && z1 <= T && rank >= 0 && rank <= T, "band matrix: bad range");
  const size_t smem = (size_t)2 * std::max(rank, 1) * (z1 - z0) * (two_sided ? 2 : 1) * sizeof(double);
  HF_CUDA(cudaFuncSetAttribute(band_matrix_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  band_matrix_kernel<<<(unsigned)batch, 256, smem, s>>>(evecs, T, rank, z0, z1, two_sided ? 1 : 0, wmat);
  note_launch();
  return launch_status("band_matrix_kernel");
}

int launch_pca_project(const float *in, int64_t batch, int T, int64_t P, const double *evecs,
                       int begin, int end, float *out, cudaStream_t s) {
  HF_CHECK_ARG(begin >= 0 && end > begin && end <= T, "pca projection: bad component range");
  const int    ncomp = end - begin;
  const size_t smem  = (size_t)T * ncomp * sizeof(float);
  HF_CUDA(cudaFuncSetAttribute(pca_project_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  pca_project_kernel<<<dim3((unsigned)((P + 255) / 256), (unsigned)batch), 256, smem, s>>>(
      in, T, P, evecs, begin, ncomp, out);
  note_launch();
  return launch_status("pca_project_kernel");
}

// ------------------------------------------------------------------------------------------------
// Gram matrices with a fixed, library-owned workspace (hf_covariance_noalloc).
//
// The workspace is a file-scope device array, so the module loader reserves it once per device
// and the call itself never allocates.  Its device address is looked up once per device (with
// that device current) and cached.  The tiled kernel writes every partial and per-frame sum the
// reduction reads before it is read, so nothing in the array has to start at zero.  Every call
// on a device uses the same array: calls whose work overlaps in time race on it.
// ------------------------------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_cov_scratch[HF_COVARIANCE_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxScratchDevices = 64;
std::mutex    g_scratch_mu;
void         *g_scratch_ptr[kMaxScratchDevices] = {};

int scratch_address(void **ptr) {
  int dev = 0;
  HF_CUDA(cudaGetDevice(&dev));
  HF_CHECK_ARG(dev >= 0 && dev < kMaxScratchDevices, "hf_covariance_noalloc: device ordinal above 63");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void             *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_cov_scratch);
    if (e != cudaSuccess)
      return cuda_status(e, "hf_covariance_noalloc: cudaGetSymbolAddress of the fixed workspace");
    g_scratch_ptr[dev] = p;
  }
  *ptr = g_scratch_ptr[dev];
  return HF_OK;
}

// CTAs per window that fit the fixed workspace (0 when even one does not).
template <int T> int fitting_ctas(int nwin) {
  using Gm                 = CovGeom<T>;
  const size_t per_cta     = (size_t)Gm::G * T * T * sizeof(float) + (size_t)T * sizeof(double);
  const size_t usable      = HF_COVARIANCE_NOALLOC_SCRATCH_BYTES - 256;
  const size_t fit         = usable / ((size_t)nwin * per_cta);
  return (int)std::min<size_t>(fit, (size_t)1 << 20);
}

template <int FMT, int T>
int cov_fixed_tiled(const FrameRing &ring, int64_t P, int nwin, void *ws, double *gram, cudaStream_t s) {
  const int fit = fitting_ctas<T>(nwin);
  if (fit < 1)
    return fail(HF_ERR_INVALID,
                "hf_covariance_noalloc: batch " + std::to_string(nwin) + " at T = " + std::to_string(T) +
                    " needs more than the fixed " +
                    std::to_string(HF_COVARIANCE_NOALLOC_SCRATCH_BYTES >> 20) +
                    " MiB workspace; split the batch or use hf_covariance with a workspace");
  return launch_cov_tiled<FMT, T>(ring, P, nwin, ws, gram, s, fit);
}

template <int FMT>
int cov_fixed_fmt(const FrameRing &ring, int T, int64_t P, int nwin, double *gram, cudaStream_t s) {
  const bool tiled = (P % 8 == 0) && (ring.frame_bytes % 4 == 0) && (((uintptr_t)ring.base & 3) == 0) &&
                     (T == 32 || T == 64 || T == 128);
  if (!tiled) { // the direct kernel needs no workspace (and takes any alignment)
    cov_generic_kernel<FMT><<<dim3((T * T + 127) / 128, nwin), 128, 0, s>>>(ring, T, P, gram);
    note_launch();
    return launch_status("cov_generic_kernel");
  }
  void *ws = nullptr;
  HF_TRY(scratch_address(&ws));
  if (T == 32)
    return cov_fixed_tiled<FMT, 32>(ring, P, nwin, ws, gram, s);
  if (T == 64)
    return cov_fixed_tiled<FMT, 64>(ring, P, nwin, ws, gram, s);
  return cov_fixed_tiled<FMT, 128>(ring, P, nwin, ws, gram, s);
}
} // namespace

int launch_covariance_fixed_scratch(const FrameRing &ring, int fmt, int T, int64_t P, int nwin, double *gram,
                                    cudaStream_t s) {
  HF_CHECK_ARG(T > 0 && P > 0 && nwin > 0, "covariance: empty problem");
  switch (fmt) {
  case HF_MONO12P: return cov_fixed_fmt<HF_MONO12P>(ring, T, P, nwin, gram, s);
  case HF_U16: return cov_fixed_fmt<HF_U16>(ring, T, P, nwin, gram, s);
  case HF_U8: return cov_fixed_fmt<HF_U8>(ring, T, P, nwin, gram, s);
  case HF_F32: return cov_fixed_fmt<HF_F32>(ring, T, P, nwin, gram, s);
  default: return fail(HF_ERR_INVALID, "covariance: unsupported input dtype");
  }
}

} // namespace hf
