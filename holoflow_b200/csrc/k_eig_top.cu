// The r largest eigenpairs of a batch of symmetric n x n float64 matrices (n <= 128, r <= 16).
//
// The clutter filter W = (I - V_r V_r^T) D needs only the top clutter_rank eigenvectors of each
// window's Gram matrix, and the full cyclic Jacobi solve (k_pca.cu) spends O(n^3) shared-memory
// traffic per sweep over ~11 sweeps.  Here one CTA of 256 threads per matrix runs:
//  1. Householder reduction to tridiagonal form, A = Q T Q^T (Golub & Van Loan, Matrix
//     Computations, 4th ed., Alg. 8.3.1), with the reflectors v_k kept in column k below the
//     subdiagonal and beta_k in a side array.  Two barriers per step: the matrix-vector product
//     p = beta A v (a thread pair per row, each summing half the row) with per-warp partials of
//     p^T v; then the rank-2 update A -= v w^T + w v^T with w = p - (beta/2)(p^T v) v formed on the
//     fly, where warp 0 updates the trailing block's first column and at once builds the next
//     step's house vector from it (the house vectors alternate between two buffers);
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

// Stride of the per-eigenvalue vectors, = 1 (mod 16) doubles, so the lanes of the inverse iteration
// (one per eigenvalue, r <= 16) address distinct bank pairs.
__host__ __device__ inline int eig_ldy(int n) { return 16 * ((n + 15) / 16) + 1; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Number of eigenvalues of the tridiagonal (d, e) below x: sign changes of the leading minors of
// T - x I.  T is scaled by a power of two to ||T|| <= 1, so a minor grows at most 3x per step; two
// steps at a time, consecutive minors are rescaled together by 2^-/+800 when they leave
// [2^-800, 2^800], which keeps every sign.  A zero minor counts as a change.
__device__ int sturm_count(const double *d, const double *e2, int n, double x) {
  double pm = 1.0, p = d[0] - x;
  int    cnt = p <= 0.0 ? 1 : 0; // p_0 = 1 > 0
  if (p == 0.0)
    p = -DBL_MIN; // counted; continue from a tiny negative minor
  const auto step = [&](int j) {
    double q = fma(d[j] - x, p, -e2[j - 1] * pm);
    if (q == 0.0)
      q = p > 0.0 ? -DBL_MIN : DBL_MIN;
    cnt += (q < 0.0) != (p < 0.0);
    pm = p;
    p  = q;
  };
  int j = 1;
  for (; j + 1 < n; j += 2) {
    step(j);
    step(j + 1);
    const double a = fabs(p);
    const double f = a > 0x1p800 ? 0x1p-800 : (a < 0x1p-800 && fabs(pm) < 0x1p-800 ? 0x1p800 : 1.0);
    p *= f;
    pm *= f;
  }
  if (j < n)
    step(j);
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
  double   *e2   = e + n;                 // [n] e^2, scaled by sc^2
  double   *ds   = e2 + n;                // [n] d, scaled by sc (||T|| sc <= 1)
  double   *vvb  = ds + n;                // [2][n] house vectors of even / odd steps
  double   *pw   = vvb + 2 * n;           // [n] p = beta A v
  double   *lam  = pw + n;                // [kEigMaxR] eigenvalues, descending
  const int ldy  = eig_ldy(n);            // per-vector stride: lane t's entries in bank pair t
  double   *Y    = lam + kEigMaxR;        // [kEigMaxR][ldy] eigenvectors of T, then of A
  double   *lu   = Y + kEigMaxR * ldy;    // [4][kEigMaxR][ldy] LU factors of each shift
  double   *red  = lu + 4 * kEigMaxR * ldy; // [kEigWarps + 4] reductions and scalars
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
  // house vector of step k from column k below the diagonal (warp 0); its reflector replaces the
  // column's entries, beta_k, d_k and e_k go to their arrays
  const auto house = [&](int k) {
    const int m = n - k - 1;
    double   *v = vvb + (k & 1) * n;
    double    s = 0.0;
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
      v[i] = i == 0 ? v0 : A[(k + 1 + i) * ld + k];
    __syncwarp();
    if (lane == 0) {
      A[(k + 1) * ld + k] = v0;
      beta[k]             = b;
      d[k]                = A[k * ld + k];
      e[k]                = alpha;
    }
  };
  if (warp == 0 && n >= 3)
    house(0);
  __syncthreads();
  for (int k = 0; k + 2 < n; ++k) {
    const int     m = n - k - 1; // trailing block rows / cols k+1 .. n-1
    const double  b = beta[k];
    const double *v = vvb + (k & 1) * n;
    if (b == 0.0) { // the column is already reduced: H = I, the trailing block stays
      if (warp == 0 && k + 3 < n)
        house(k + 1);
      __syncthreads();
      continue;
    }
    { // p = beta A' v: threads 2i and 2i+1 sum the two halves of row i (read as column i of the
      // symmetric block, so a warp's loads are contiguous), then the warp's share of p^T v
      const int i = tid >> 1, hm = (m + 1) >> 1;
      double    s0 = 0.0, s1 = 0.0;
      if (i < m) {
        const int     j1  = min(m, (tid & 1) * hm + hm);
        const double *col = A + (k + 1) * ld + k + 1 + i;
        int           j   = (tid & 1) * hm;
        double        s2 = 0.0, s3 = 0.0;
        for (; j + 3 < j1; j += 4) {
          s0 = fma(col[j * ld], v[j], s0);
          s1 = fma(col[(j + 1) * ld], v[j + 1], s1);
          s2 = fma(col[(j + 2) * ld], v[j + 2], s2);
          s3 = fma(col[(j + 3) * ld], v[j + 3], s3);
        }
        for (; j < j1; ++j)
          s0 = fma(col[j * ld], v[j], s0);
        s0 += s2;
        s1 += s3;
      }
      double sp = s0 + s1;
      sp += __shfl_xor_sync(0xffffffffu, sp, 1);
      double pv = 0.0;
      if (i < m && (tid & 1) == 0) {
        const double p = b * sp;
        pw[i]          = p;
        pv             = p * v[i];
      }
      pv = warp_sum(pv);
      if (lane == 0)
        red[warp] = pv;
    }
    __syncthreads();
    double dot = 0.0; // p^T v, summed in warp order
#pragma unroll
    for (int q = 0; q < kEigWarps; ++q)
      dot += red[q];
    const double kk = 0.5 * b * dot; // w = p - kk v
    if (warp == 0) {
      // the trailing block's column 0 (column k+1 of A), then the house vector of step k+1 from it
      const double w0 = fma(-kk, v[0], pw[0]), v0 = v[0];
      for (int i = lane; i < m; i += 32) {
        const double wi = fma(-kk, v[i], pw[i]);
        double      &a  = A[(k + 1 + i) * ld + k + 1];
        a               = fma(-v[i], w0, fma(-wi, v0, a));
      }
      __syncwarp();
      if (k + 3 < n)
        house(k + 1);
    } else { // columns 1 .. m-1, a row at a time per warp; lane owns columns 1 + lane + 32 c
      double vj[kEigMaxN / 32], wj[kEigMaxN / 32];
#pragma unroll
      for (int c = 0; c < kEigMaxN / 32; ++c) {
        const int j = 1 + lane + 32 * c;
        vj[c]       = j < m ? v[j] : 0.0;
        wj[c]       = j < m ? fma(-kk, v[j], pw[j]) : 0.0;
      }
      for (int i = warp - 1; i < m; i += kEigWarps - 1) {
        const double vi = v[i], wi = fma(-kk, v[i], pw[i]);
        double      *row = A + (k + 1 + i) * ld + k + 1;
#pragma unroll
        for (int c = 0; c < kEigMaxN / 32; ++c) {
          const int j = 1 + lane + 32 * c;
          if (j < m)
            row[j] = fma(-vi, wj[c], fma(-wi, vj[c], row[j]));
        }
      }
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
      int          ex  = 0;
      frexp(nrm, &ex);
      red[0] = lo - pad;
      red[1] = hi + pad;
      red[2] = nrm;
      red[3] = nrm > 0.0 ? ldexp(1.0, -ex) : 1.0; // sc: a power of two with ||T|| sc < 1
    }
  }
  __syncthreads();
  const double sc = red[3];
  for (int i = tid; i < n; i += kEigThr) { // the Sturm sequences run on T sc (exactly scaled)
    const double es = e[i] * sc;
    ds[i]           = d[i] * sc;
    e2[i]           = es * es;
  }
  __syncthreads();

  // ---- 2. eigenvalues n-1, n-2, ..., n-r by multisection, a warp each: 32 shifts per round ------
  for (int t = warp; t < r; t += kEigWarps) {
    const int idx = n - 1 - t; // ascending index: count(a) <= idx < count(b)
    double    a = red[0] * sc, b = red[1] * sc;
    for (int round = 0; round < 24; ++round) {
      const double x   = a + (b - a) * (double)(lane + 1) / 33.0;
      const int    c   = sturm_count(ds, e2, n, x);
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
      lam[t] = 0.5 * (a + b) * (1.0 / sc); // 1 / sc is a power of two: exact
  }
  __syncthreads();

  // ---- 3. eigenvectors of T by inverse iteration: eigenvalue t in warp t % 8, whose lane 0 runs
  //         the LU factorisation and the solves while the warp normalises; close eigenvalues are
  //         orthogonalised in descending order between block barriers ----------------------------
  {
    const double  nrm  = red[2];
    const double  tiny = DBL_EPSILON * nrm + DBL_MIN; // pivot floor
    const double  clus = 1e-7 * nrm;                  // eigenvalues closer than this share a cluster
    constexpr int kPer = kEigMaxR / kEigWarps;         // eigenvalues per warp
    uint32_t      swp[kPer][kEigMaxN / 32];            // row j and j+1 exchanged at step j
    for (int u = 0; u < kPer; ++u) {
      const int t = warp + kEigWarps * u;
#pragma unroll
      for (int q = 0; q < kEigMaxN / 32; ++q)
        swp[u][q] = 0u;
      if (t >= r)
        continue;
      double *y = Y + t * ldy;
      double *u0 = lu + (0 * kEigMaxR + t) * ldy, *u1 = lu + (1 * kEigMaxR + t) * ldy,
             *u2 = lu + (2 * kEigMaxR + t) * ldy, *ml = lu + (3 * kEigMaxR + t) * ldy;
      if (lane == 0) {
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
            swp[u][j >> 5] |= 1u << (j & 31);
            a0 = a1 - l * b1;
            a1 = -l * b2;
          }
        }
        u0[n - 1] = fabs(a0) < tiny ? copysign(tiny, a0) : a0;
      }
      __syncwarp();
      for (int j = lane; j < n; j += 32) { // the solves multiply by the pivots' reciprocals
        u0[j] = 1.0 / u0[j];
        y[j]  = 1.0 + 0.01 * (double)(((j * 7 + t * 13) % 17) - 8); // start: nonzero, distinct per t
      }
    }
    bool clustered = false; // any two of the r eigenvalues closer than clus
    for (int q = 1; q < r; ++q)
      clustered |= fabs(lam[q] - lam[q - 1]) <= clus;
    for (int it = 0; it < 3; ++it) {
      for (int u = 0; u < kPer; ++u) {
        const int t = warp + kEigWarps * u;
        if (t >= r)
          continue;
        double       *y  = Y + t * ldy;
        const double *u0 = lu + (0 * kEigMaxR + t) * ldy, *u1 = lu + (1 * kEigMaxR + t) * ldy,
                     *u2 = lu + (2 * kEigMaxR + t) * ldy, *ml = lu + (3 * kEigMaxR + t) * ldy;
        __syncwarp();
        if (lane == 0) { // solve M y' = y in place, the running entry carried in a register
          double c = y[0];
          for (int j = 0; j + 1 < n; ++j) {
            const double nx = y[j + 1];
            if ((swp[u][j >> 5] >> (j & 31)) & 1u) { // rows j, j+1 exchanged
              y[j] = nx;
              c    = c - ml[j] * nx;
            } else {
              y[j] = c;
              c    = nx - ml[j] * c;
            }
          }
          double c1 = c * u0[n - 1], c2 = 0.0; // y[j+1], y[j+2] of the back substitution
          y[n - 1]  = c1;
          for (int j = n - 2; j >= 0; --j) {
            const double c0 = (y[j] - u1[j] * c1 - u2[j] * c2) * u0[j];
            y[j]            = c0;
            c2              = c1;
            c1              = c0;
          }
        }
        __syncwarp();
        // scale by the largest entry first (the solve grows y by up to 1 / (eps ||T||)), then
        // normalise
        double mx = 0.0;
        for (int i = lane; i < n; i += 32)
          mx = fmax(mx, fabs(y[i]));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (mx > 0.0) {
          const double im = 1.0 / mx;
          double       ss = 0.0;
          for (int i = lane; i < n; i += 32) {
            const double yi = y[i] * im;
            y[i]            = yi;
            ss              = fma(yi, yi, ss);
          }
          const double inv = 1.0 / sqrt(warp_sum(ss));
          for (int i = lane; i < n; i += 32)
            y[i] *= inv;
        }
      }
      if (!clustered)
        continue;
      __syncthreads();
      // modified Gram-Schmidt within clusters, in descending eigenvalue order, by the warp of s2
      for (int s2 = 1; s2 < r; ++s2) {
        if (warp == s2 % kEigWarps) {
          double *y   = Y + s2 * ldy;
          bool    any = false;
          for (int q = 0; q < s2; ++q) {
            if (fabs(lam[q] - lam[s2]) > clus)
              continue;
            const double *yq = Y + q * ldy;
            double        dt = 0.0;
            for (int i = lane; i < n; i += 32)
              dt = fma(yq[i], y[i], dt);
            dt = warp_sum(dt);
            for (int i = lane; i < n; i += 32)
              y[i] = fma(-dt, yq[i], y[i]);
            __syncwarp();
            any = true;
          }
          if (any) {
            double ss = 0.0;
            for (int i = lane; i < n; i += 32)
              ss = fma(y[i], y[i], ss);
            ss = warp_sum(ss);
            if (ss > 0.0) {
              const double inv = 1.0 / sqrt(ss);
              for (int i = lane; i < n; i += 32)
                y[i] *= inv;
            }
          }
        }
        __syncthreads();
      }
    }
  }
  __syncthreads();

  // ---- 4. back-transformation V = Q Y, a warp per column, entries i = lane + 32 c in registers ---
  for (int t = warp; t < r; t += kEigWarps) {
    const double *ys = Y + t * ldy;
    double        y[kEigMaxN / 32];
#pragma unroll
    for (int c = 0; c < kEigMaxN / 32; ++c) {
      const int i = lane + 32 * c;
      y[c]        = i < n ? ys[i] : 0.0;
    }
    for (int k = n - 3; k >= 0; --k) {
      const double b = beta[k];
      if (b == 0.0)
        continue;
      double vr[kEigMaxN / 32], s = 0.0; // reflector k: column k of A, rows k+1 .. n-1
#pragma unroll
      for (int c = 0; c < kEigMaxN / 32; ++c) {
        const int i = lane + 32 * c;
        vr[c]       = i > k && i < n ? A[i * ld + k] : 0.0;
        s           = fma(vr[c], y[c], s);
      }
      s = b * warp_sum(s);
#pragma unroll
      for (int c = 0; c < kEigMaxN / 32; ++c)
        y[c] = fma(-s, vr[c], y[c]);
    }
    const int idx = n - 1 - t;
    double   *vec = evecs + (int64_t)blockIdx.x * n * n;
#pragma unroll
    for (int c = 0; c < kEigMaxN / 32; ++c) {
      const int i = lane + 32 * c;
      if (i < n)
        vec[i * n + idx] = y[c];
    }
    if (lane == 0)
      evals[(int64_t)blockIdx.x * n + idx] = lam[t];
  }
  if (tid == 0 && info != nullptr)
    info[blockIdx.x] = 0;
}

} // namespace

size_t eig_top_smem_bytes(int n) {
  return ((size_t)n * (n + 1) + 8 * (size_t)n + kEigMaxR + 5 * (size_t)kEigMaxR * eig_ldy(n) + kEigWarps + 4) *
             sizeof(double) +
         16;
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
