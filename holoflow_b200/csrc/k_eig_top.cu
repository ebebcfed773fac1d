// The r largest eigenpairs of a batch of symmetric n x n float64 matrices (n <= 128, r <= 16).
//
// The clutter filter W = (I - V_r V_r^T) D needs only the top clutter_rank eigenvectors of each
// window's Gram matrix, and the full cyclic Jacobi solve (k_pca.cu) spends O(n^3) shared-memory
// traffic per sweep over ~11 sweeps.  Here one CTA of 256 threads per matrix runs:
//  1. Householder reduction to tridiagonal form, A = Q T Q^T (Golub & Van Loan, Matrix
//     Computations, 4th ed., Alg. 8.3.1), with the reflectors v_k kept in column k below the
//     subdiagonal and beta_k in a side array: per step one house vector, one matrix-vector product
//     p = beta A v (a warp per row), w = p - (beta/2)(p^T v) v, and the rank-2 update A -= v w^T + w v^T;
//  2. the r largest eigenvalues of T by Sturm-sequence multisection (Wilkinson): a warp evaluates
//     32 shifts at once, each lane counting the sign changes of the leading-minor sequence
//     p_j = (d_j - x) p_{j-1} - e_{j-1}^2 p_{j-2} (rescaled by powers of two, no division), and the
//     bracket shrinks 33x per round;
//  3. their eigenvectors of T by inverse iteration (Wilkinson): three solves with the tridiagonal
//     LU factorisation of T - lambda I with partial pivoting, pivots floored at eps ||T||, from
//     distinct starting vectors, orthonormalised (modified Gram-Schmidt) within clusters of close
//     eigenvalues after each solve;
//  4. back-transformation V_r = Q Y by the reflectors in reverse order, a warp per column.
// The eigenvalues ascend in evals[n - r .. n - 1] and the vectors go to the matching columns of
// evecs ([n][n], column = eigenvalue index, as the Jacobi solver lays them out); the other entries
// are not written.  info = 0, or 1 when the input is not finite.
#include <cfloat>

#include "k_pca.cuh"

namespace hf {

namespace {

constexpr int kEigThr  = 256;
constexpr int kEigWarps = kEigThr / 32;
constexpr int kEigMaxN = 128;
constexpr int kEigMaxR = 16;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Number of eigenvalues of the tridiagonal (d, e) below x: sign changes of the leading minors of
// T - x I.  A zero minor counts as a change; consecutive minors are rescaled together by 2^-/+600
// when they leave [2^-600, 2^600], which keeps every sign.
__device__ int sturm_count(const double *d, const double *e2, int n, double x) {
  double pm = 1.0, p = d[0] - x;
  int    cnt = p <= 0.0 ? 1 : 0; // p_0 = 1 > 0
  if (p == 0.0)
    p = -DBL_MIN; // counted; continue from a tiny negative minor
  for (int j = 1; j < n; ++j) {
    double q = fma(d[j] - x, p, -e2[j - 1] * pm);
    if (q == 0.0)
      q = p > 0.0 ? -DBL_MIN : DBL_MIN;
    cnt += (q < 0.0) != (p < 0.0);
    pm = p;
    p  = q;
    const double a = fabs(p);
    if (a > 0x1p600) {
      p *= 0x1p-600;
      pm *= 0x1p-600;
    } else if (a < 0x1p-600 && fabs(pm) < 0x1p-600) {
      p *= 0x1p600;
      pm *= 0x1p600;
    }
  }
  return cnt;
}

__global__ void __launch_bounds__(kEigThr) eig_top_kernel(const double *a_in, double *evecs, double *evals,
                                                          int *info, int n, int r) {
  extern __shared__ __align__(16) double esm[];
  const int ld   = n + 1;                 // padded row stride
  double   *A    = esm;                   // [n][ld]
  double   *beta = A + n * ld;            // [n]
  double   *d    = beta + n;              // [n] diagonal of T
  double   *e    = d + n;                 // [n] subdiagonal of T (e[n-1] = 0)
  double   *e2   = e + n;                 // [n] e^2
  double   *vv   = e2 + n;                // [n] current house vector
  double   *pw   = vv + n;                // [n] p, then w
  double   *lam  = pw + n;                // [kEigMaxR] eigenvalues, descending
  double   *Y    = lam + kEigMaxR;        // [kEigMaxR][n] eigenvectors of T, then of A
  double   *lu   = Y + kEigMaxR * n;      // [kEigMaxR][4][n] LU factors of one shift
  double   *red  = lu + kEigMaxR * 4 * n; // [kEigWarps + 4] reductions and scalars
  int      *flag = reinterpret_cast<int *>(red + kEigWarps + 4);

  const int     tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const double *src = a_in + (int64_t)blockIdx.x * n * n;
  if (tid == 0)
    *flag = 0;
  __syncthreads();
  for (int x = tid; x < n * n; x += kEigThr) {
    const int    i = x / n, j = x % n;
    const double v = 0.5 * (src[i * n + j] + src[j * n + i]);
    if (!isfinite(v))
      *flag = 1;
    A[i * ld + j] = v;
  }
  __syncthreads();
  if (*flag) { // not finite: report, leave the outputs alone
    if (tid == 0 && info != nullptr)
      info[blockIdx.x] = 1;
    return;
  }

  // ---- 1. Householder tridiagonalisation ------------------------------------------------------
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1; // trailing block rows / cols k+1 .. n-1
    if (warp == 0) {         // house vector of x = A[k+1.., k]
      double s = 0.0;
      for (int i = 1 + lane; i < m; i += 32) {
        const double x = A[(k + 1 + i) * ld + k];
        s              = fma(x, x, s);
      }
      s               = warp_sum(s);
      const double x0 = A[(k + 1) * ld + k];
      double       v0 = 1.0, b = 0.0, alpha = x0;
      if (s > 0.0) {
        const double mu = sqrt(fma(x0, x0, s));
        v0              = x0 <= 0.0 ? x0 - mu : -s / (x0 + mu); // x0 - mu without cancellation
        b               = 2.0 / fma(v0, v0, s);
        alpha           = mu;
      }
      for (int i = lane; i < m; i += 32)
        vv[i] = i == 0 ? v0 : A[(k + 1 + i) * ld + k];
      if (lane == 0) {
        A[(k + 1) * ld + k] = v0;
        beta[k]             = b;
        d[k]                = A[k * ld + k];
        e[k]                = alpha;
      }
    }
    __syncthreads();
    const double b = beta[k];
    if (b == 0.0)
      continue; // the column is already reduced: H = I
    // p = beta A' v, a warp per row
    for (int i = warp; i < m; i += kEigWarps) {
      const double *row = A + (k + 1 + i) * ld + k + 1;
      double        s   = 0.0;
      for (int j = lane; j < m; j += 32)
        s = fma(row[j], vv[j], s);
      s = warp_sum(s);
      if (lane == 0)
        pw[i] = b * s;
    }
    __syncthreads();
    if (warp == 0) { // w = p - (beta/2)(p^T v) v
      double s = 0.0;
      for (int i = lane; i < m; i += 32)
        s = fma(pw[i], vv[i], s);
      const double kk = 0.5 * b * warp_sum(s);
      for (int i = lane; i < m; i += 32)
        pw[i] = fma(-kk, vv[i], pw[i]);
    }
    __syncthreads();
    for (int x = tid; x < m * m; x += kEigThr) { // A' -= v w^T + w v^T
      const int i = x / m, j = x % m;
      double   &aij = A[(k + 1 + i) * ld + k + 1 + j];
      aij           = fma(-vv[i], pw[j], fma(-pw[i], vv[j], aij));
    }
    __syncthreads();
  }
  if (tid == 0) {
    for (int k = n - 2; k < n; ++k)
      if (k >= 0)
        d[k] = A[k * ld + k];
    if (n >= 2)
      e[n - 2] = A[(n - 1) * ld + n - 2];
    if (n >= 1)
      e[n - 1] = 0.0;
  }
  __syncthreads();
  for (int i = tid; i < n; i += kEigThr)
    e2[i] = e[i] * e[i];
  // Gershgorin bounds and ||T|| (warp 0)
  if (warp == 0) {
    double lo = DBL_MAX, hi = -DBL_MAX, nrm = 0.0;
    for (int i = lane; i < n; i += 32) {
      const double rad = fabs(e[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0);
      lo               = fmin(lo, d[i] - rad);
      hi               = fmax(hi, d[i] + rad);
      nrm              = fmax(nrm, fabs(d[i]) + rad);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo  = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi  = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      nrm = fmax(nrm, __shfl_xor_sync(0xffffffffu, nrm, o));
    }
    if (lane == 0) {
      const double pad = 2.0 * DBL_EPSILON * nrm + DBL_MIN;
      red[0]           = lo - pad;
      red[1]           = hi + pad;
      red[2]           = nrm;
    }
  }
  __syncthreads();

  // ---- 2. eigenvalues n-1, n-2, ..., n-r by multisection, a warp each ---------------------------
  for (int t = warp; t < r; t += kEigWarps) {
    const int idx = n - 1 - t; // ascending index: count(a) <= idx < count(b)
    double    a = red[0], b = red[1];
    for (int round = 0; round < 24; ++round) {
      const double x   = a + (b - a) * (double)(lane + 1) / 33.0;
      const int    c   = sturm_count(d, e2, n, x);
      const unsigned m = __ballot_sync(0xffffffffu, c > idx);
      const int    f   = m ? __ffs(m) - 1 : 32; // first shift with more than idx eigenvalues below
      const double xf  = __shfl_sync(0xffffffffu, x, f & 31);
      const double xp  = __shfl_sync(0xffffffffu, x, (f + 31) & 31);
      const double na  = f == 0 ? a : xp;
      const double nb  = f == 32 ? b : xf;
      a                = na;
      b                = nb;
      if (b - a <= 2.0 * DBL_EPSILON * fmax(fabs(a), fabs(b)) + DBL_MIN)
        break;
    }
    if (lane == 0)
      lam[t] = 0.5 * (a + b);
  }
  __syncthreads();

  // ---- 3. eigenvectors of T by inverse iteration, lane t of warp 0 -------------------------------
  if (warp == 0) {
    const double nrm  = red[2];
    const double tiny = DBL_EPSILON * nrm + DBL_MIN; // pivot floor
    const double clus = 1e-7 * nrm;                  // eigenvalues closer than this share a cluster
    const int    t    = lane;
    double      *y    = Y + t * n;
    double *u0 = lu + (t * 4 + 0) * n, *u1 = lu + (t * 4 + 1) * n, *u2 = lu + (t * 4 + 2) * n,
           *ml = lu + (t * 4 + 3) * n;
    uint32_t swp[kEigMaxN / 32] = {0u, 0u, 0u, 0u}; // row j and j+1 exchanged at step j
    if (t < r) {
      // Gaussian elimination of M = T - lambda I with partial pivoting.  The working row holds the
      // entries (a0, a1) of columns j, j+1 (its column-(j+2) entry is always 0); row j+1 of M is
      // (e_j, d_{j+1} - lambda, e_{j+1}) on columns j, j+1, j+2.  U gets (u0, u1, u2) per row.
      const double lm = lam[t];
      double       a0 = d[0] - lm, a1 = n > 1 ? e[0] : 0.0;
      for (int j = 0; j + 1 < n; ++j) {
        const double b0 = e[j], b1 = d[j + 1] - lm, b2 = j + 2 < n ? e[j + 1] : 0.0;
        if (fabs(a0) >= fabs(b0)) {
          const double piv = fabs(a0) < tiny ? copysign(tiny, a0) : a0;
          const double l   = b0 / piv;
          u0[j] = piv, u1[j] = a1, u2[j] = 0.0, ml[j] = l;
          a0 = b1 - l * a1;
          a1 = b2;
        } else {
          const double l = a0 / b0;
          u0[j] = b0, u1[j] = b1, u2[j] = b2, ml[j] = l;
          swp[j >> 5] |= 1u << (j & 31);
          a0 = a1 - l * b1;
          a1 = -l * b2;
        }
      }
      u0[n - 1] = fabs(a0) < tiny ? copysign(tiny, a0) : a0;
      // a starting vector with every component nonzero, distinct per eigenvalue
      for (int i = 0; i < n; ++i)
        y[i] = 1.0 + 0.01 * (double)(((i * 7 + t * 13) % 17) - 8);
    }
    for (int it = 0; it < 3; ++it) {
      if (t < r) { // solve M y' = y in place, then normalise
        for (int j = 0; j + 1 < n; ++j) {
          if ((swp[j >> 5] >> (j & 31)) & 1u) {
            const double zj = y[j], zk = y[j + 1];
            y[j]     = zk;
            y[j + 1] = zj - ml[j] * zk;
          } else {
            y[j + 1] -= ml[j] * y[j];
          }
        }
        y[n - 1] /= u0[n - 1];
        if (n >= 2)
          y[n - 2] = (y[n - 2] - u1[n - 2] * y[n - 1]) / u0[n - 2];
        for (int j = n - 3; j >= 0; --j)
          y[j] = (y[j] - u1[j] * y[j + 1] - u2[j] * y[j + 2]) / u0[j];
        double mx = 0.0;
        for (int i = 0; i < n; ++i)
          mx = fmax(mx, fabs(y[i]));
        if (mx > 0.0) { // scale first (the solve grows y by up to 1 / (eps ||T||)), then normalise
          const double im = 1.0 / mx;
          double       ss = 0.0;
          for (int i = 0; i < n; ++i) {
            y[i] *= im;
            ss = fma(y[i], y[i], ss);
          }
          const double inv = 1.0 / sqrt(ss);
          for (int i = 0; i < n; ++i)
            y[i] *= inv;
        }
      }
      __syncwarp();
      // modified Gram-Schmidt within clusters, in descending eigenvalue order
      for (int s2 = 1; s2 < r; ++s2) {
        if (t == s2) {
          bool any = false;
          for (int q = 0; q < s2; ++q) {
            if (fabs(lam[q] - lam[s2]) > clus)
              continue;
            const double *yq = Y + q * n;
            double        dt = 0.0;
            for (int i = 0; i < n; ++i)
              dt = fma(yq[i], y[i], dt);
            for (int i = 0; i < n; ++i)
              y[i] = fma(-dt, yq[i], y[i]);
            any = true;
          }
          if (any) {
            double ss = 0.0;
            for (int i = 0; i < n; ++i)
              ss = fma(y[i], y[i], ss);
            if (ss > 0.0) {
              const double inv = 1.0 / sqrt(ss);
              for (int i = 0; i < n; ++i)
                y[i] *= inv;
            }
          }
        }
        __syncwarp();
      }
    }
  }
  __syncthreads();

  // ---- 4. back-transformation V = Q Y, a warp per column -----------------------------------------
  for (int t = warp; t < r; t += kEigWarps) {
    double *y = Y + t * n;
    for (int k = n - 3; k >= 0; --k) {
      const double b = beta[k];
      if (b == 0.0)
        continue;
      const int m = n - k - 1;
      double    s = 0.0;
      for (int i = lane; i < m; i += 32)
        s = fma(A[(k + 1 + i) * ld + k], y[k + 1 + i], s);
      s = b * warp_sum(s);
      for (int i = lane; i < m; i += 32)
        y[k + 1 + i] = fma(-s, A[(k + 1 + i) * ld + k], y[k + 1 + i]);
      __syncwarp();
    }
    const int idx = n - 1 - t;
    double   *vec = evecs + (int64_t)blockIdx.x * n * n;
    for (int i = lane; i < n; i += 32)
      vec[i * n + idx] = y[i];
    if (lane == 0)
      evals[(int64_t)blockIdx.x * n + idx] = lam[t];
  }
  if (tid == 0 && info != nullptr)
    info[blockIdx.x] = 0;
}

} // namespace

size_t eig_top_smem_bytes(int n) {
  return ((size_t)n * (n + 1) + 6 * (size_t)n + kEigMaxR + (size_t)kEigMaxR * n + (size_t)kEigMaxR * 4 * n +
          kEigWarps + 4) * sizeof(double) + 16;
}

bool eig_top_supported(int n, int r) { return n >= 1 && n <= kEigMaxN && r >= 1 && r <= kEigMaxR && r <= n; }

int launch_eig_top(const double *a, double *evecs, double *evals, int *info, int n, int r, int64_t batch,
                   cudaStream_t s) {
  HF_CHECK_ARG(eig_top_supported(n, r) && batch >= 1, "eig_top: order must be in [1, 128] and 1 <= r <= min(16, n)");
  const size_t smem = eig_top_smem_bytes(n);
  HF_CUDA(cudaFuncSetAttribute(eig_top_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  eig_top_kernel<<<(unsigned)batch, kEigThr, smem, s>>>(a, evecs, evals, info, n, r);
  note_launch();
  return launch_status("eig_top_kernel");
}

} // namespace hf
