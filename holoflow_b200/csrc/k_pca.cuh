// Launch interface of the PCA / SVD-clutter-filter kernels (k_pca.cu).
#pragma once

#include "frames.cuh"

namespace hf {

// Per-window Gram matrix of the frames, G = X^T X (T x T, float64), X = [T][P].
//  partial: float32 [nwin][nblk][T*T] block partials of the shifted Gram, and
//  sums:    float64 [nwin][nblk][T] exact per-frame sums used to undo the shift.
struct CovArgs {
  FrameRing ring;
  int       T;
  int64_t   P;
  float     shift;   // samples are accumulated as (x - shift); 2048 for 12-bit data
  float    *partial;
  double   *sums;
  int       nblk;    // CTAs per window (partials per window)
};

size_t cov_workspace_bytes(int T, int64_t P, int nwin);
// Deterministic float64 reduction of block partials; undoes the sample shift exactly.
int launch_cov_finalize(const float *partial, const double *sums, int nblk, int nsum, int T, int64_t P,
                        double shift, double *gram, int nwin, cudaStream_t s);

// Tensor-core (tcgen05, f16 operands, f32 accumulation) Gram matrix for 8/12/16-bit samples and
// T in {64, 128}; `status` receives a nonzero code if a bounded mbarrier wait expires.
bool   cov_tc_supported(int fmt, int T, int64_t P, int64_t frame_bytes);
size_t cov_tc_workspace_bytes(int T, int64_t P, int nwin);
int    launch_covariance_tc(const FrameRing &ring, int fmt, int T, int64_t P, int nwin, void *ws,
                            double *gram, int *status, cudaStream_t s);
// Full Gram computation: block partials -> deterministic float64 reduction -> gram[nwin][T][T].
int launch_covariance(const FrameRing &ring, int fmt, int T, int64_t P, int nwin, void *ws,
                      double *gram, cudaStream_t s);
// The same computation on the library's fixed device workspace (no allocation; see
// hf_covariance_noalloc for the limits).
int launch_covariance_fixed_scratch(const FrameRing &ring, int fmt, int T, int64_t P, int nwin, double *gram,
                                    cudaStream_t s);

// FP64 cyclic Jacobi, one CTA per matrix (n <= 128).  Eigenvalues ascending, eigenvector j in
// column j of evecs (row-major).
int launch_jacobi(const double *a, double *evecs, double *evals, int *info, int n, int64_t batch,
                  cudaStream_t s);

// The r largest eigenpairs of symmetric n x n float64 matrices (k_eig_top.cu): Householder
// tridiagonalisation, Sturm multisection, inverse iteration, back-transformation.  Writes
// evals[n - r .. n - 1] (ascending) and the matching columns of evecs ([n][n]); info 0, or 1 for a
// non-finite input.
bool   eig_top_supported(int n, int r);
size_t eig_top_smem_bytes(int n);
int    launch_eig_top(const double *a, double *evecs, double *evals, int *info, int n, int r, int64_t batch,
                      cudaStream_t s);

// W = (I - V V^T) D[:, z0:z1] as complex64 [batch][T][nz]; V = last `rank` columns of evecs.
// two_sided: columns for bins [z0, z1) then [T - z1, T - z0) (2 (z1 - z0) columns)
int launch_band_matrix(const double *evecs, int64_t batch, int T, int rank, int z0, int z1,
                       float2 *wmat, cudaStream_t s, bool two_sided = false);

int launch_pca_project(const float *in, int64_t batch, int T, int64_t P, const double *evecs,
                       int begin, int end, float *out, cudaStream_t s);

} // namespace hf
