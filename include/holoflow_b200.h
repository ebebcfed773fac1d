/*
 * holoflow_b200 — C ABI of the B200 (sm_100a) laser Doppler reconstruction library.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns an int status
 * (HF_OK = 0, negative = error class; the text is in hf_last_error(), thread-local), never
 * throws, and only enqueues work on the stream it is given (no host synchronisation unless the
 * comment says so).  Device pointers must be device-accessible memory of the current device.
 *
 * Each function names the Holoflow interface it replaces (paths relative to the Holoflow source
 * tree).  The C++ node layer (include/holoflow_b200/core.hh, nodes.hh: the task interface with
 * factories registered under the reference's kind strings) is built on these calls and reached
 * from C through the hf_node_* functions at the end of this file.
 */
#ifndef HOLOFLOW_B200_H
#define HOLOFLOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *hf_stream_t; /* identical to cudaStream_t */

/* ---- status codes ------------------------------------------------------------------------- */
enum {
  HF_OK              = 0,
  HF_ERR_INVALID     = -1, /* bad argument / shape / setting (reference: std::invalid_argument) */
  HF_ERR_CUDA        = -2, /* CUDA runtime error (reference: curaii::CudaError)                  */
  HF_ERR_UNSUPPORTED = -3, /* valid request this build does not implement                        */
  HF_ERR_NOMEM       = -4, /* device allocation failed / admission refused                      */
  HF_ERR_TIMEOUT     = -5, /* a bounded device wait expired (status word set by a kernel)       */
  HF_ERR_STATE       = -6, /* object used in the wrong state                                     */
  HF_ERR_CANCELLED   = -7  /* cooperative cancellation observed                                  */
};

/* ---- element types (first four in the order of holoflow::core::DType, tensor.hh:29-34) ----- */
enum {
  HF_U8      = 0,
  HF_U16     = 1,
  HF_F32     = 2,
  HF_CF32    = 3,
  HF_MONO12P = 16 /* 12-bit, 2 pixels in 3 bytes, LSB-first: b0=p0[7:0], b1=p0[11:8]|p1[3:0]<<4,
                     b2=p1[11:4]; a frame of P pixels (P even) is 3P/2 bytes                      */
};

/* Conversion strategies (ConversionSettings::Strategy, holotask/syncs/conversion.hh:27-67) */
enum { HF_CONV_REAL = 0, HF_CONV_SCALED = 1, HF_CONV_MODULUS = 2, HF_CONV_ARGUMENT = 3 };

/* FFT normalisation (holonp FftNorm, holonp/src/fft.cu:100-109) */
enum { HF_NORM_BACKWARD = 0, HF_NORM_FORWARD = 1, HF_NORM_ORTHO = 2 };

/* Spatial propagation methods (holovibes Settings::spacial_method) */
enum { HF_PROP_NONE = 0, HF_PROP_FRESNEL = 1, HF_PROP_ANGULAR_SPECTRUM = 2 };

/* Moment selection bits (holovibes MomentType M0/M1/M2, graph_builder.cc:604-631) */
enum { HF_M0 = 1, HF_M1 = 2, HF_M2 = 4 };

/* Numeric form of the pipeline: all-FP32 ("plain") or tensor-core ("chosen") */
enum { HF_FORM_PLAIN = 0, HF_FORM_CHOSEN = 1 };

/* ---- library ------------------------------------------------------------------------------ */
const char *hf_last_error(void);
int         hf_version(void);
/* Number of kernel launches this thread's calls have enqueued since the last reset. */
int64_t     hf_launch_count(void);
void        hf_reset_launch_count(void);

/* ---- a1: 12-bit unpack (new: the reference has no 12-bit path, holofile.cc:247-250) -------- */
/* packed: 3*npix/2 bytes, npix even.  out_dtype: HF_U16, HF_F32 or HF_CF32 (imag = 0). */
int hf_unpack12(const uint8_t *packed, void *out, int out_dtype, int64_t npix, hf_stream_t s);
/* Inverse of hf_unpack12 for uint16 values < 4096 (acquisition / test support). */
int hf_pack12(const uint16_t *in, uint8_t *packed, int64_t npix, hf_stream_t s);

/* ---- a2: Conversion (ConversionTask::execute, holotask/src/syncs/conversion.cu:237-258) ----- */
/* Supported (in_dtype, out_dtype, strategy) triples are those of conversion.cu:138-150.
 * HF_CONV_SCALED needs `minmax_ws`: device scratch of at least 64 bytes. */
int hf_convert(const void *in, int in_dtype, void *out, int out_dtype, int strategy, int64_t n,
               void *minmax_ws, hf_stream_t s);

/* ---- a5/a6/a7: temporal FFT / RFFT along the frame axis + band slice ------------------------
 * Replaces holonp FFT (fft.cu:234-252) / RFFT (rfft.cu:150-160) on axis 1 of [B, T, H, W]
 * followed by Slice+Copy of bins [z0, z1) (graph_builder.cc:264-267).
 * in: [batch][T][P] of in_dtype (HF_U8, HF_U16, HF_MONO12P, HF_F32 or HF_CF32; MONO12P frames
 * are 3P/2 bytes).  out: [batch][z1-z0][P] complex64, bin k = scale * sum_t x_t e^{-2 pi i t k/T}.
 */
int hf_temporal_dft(const void *in, int in_dtype, int64_t batch, int T, int64_t P, int z0, int z1,
                    int norm, void *out, hf_stream_t s);

/* ---- a8: PCA / SVD clutter filter (PcaTask, holotask/src/syncs/pca.cc:68-119) -------------
 * hf_covariance: gram[b] = X_b^T X_b (T x T, float64, row-major, symmetric), X_b = [T][P] frames
 * of in_dtype (HF_U8, HF_U16, HF_MONO12P, HF_F32).  No centring, no 1/N (pca.cc:92-98).
 * `ws` must hold hf_covariance_workspace_bytes(T, P) bytes per batch item (it may be NULL when
 * `in` is not 4-byte aligned: such input takes the direct kernel, which needs no workspace). */
size_t hf_covariance_workspace_bytes(int T, int64_t P);
int    hf_covariance(const void *in, int in_dtype, int64_t batch, int T, int64_t P, double *gram,
                     void *ws, hf_stream_t s);

/* hf_covariance_noalloc: hf_covariance without a caller workspace and without any allocation.
 * It has no counterpart in the reference (PcaTask gets its buffers from the task's allocator).
 * It is for callers that hold device pointers to frames and the Gram output but cannot allocate
 * device memory when they call: a camera callback or real-time acquisition thread, where
 * cudaMalloc's implicit device synchronisation would stall the stream, or a host program that
 * has no device allocator of its own to make a workspace with.
 * The workspace is a fixed HF_COVARIANCE_NOALLOC_SCRATCH_BYTES array inside the library, one per
 * device, reserved when the library's device code is loaded.  Nothing in it has to start at zero.
 *  - The first call on a device (made with that device current) looks up the array's address
 *    and caches it; make that first call before any stream capture on that device.  The cached
 *    address belongs to the device's primary context: after cudaDeviceReset on that device it is
 *    stale, so a process that resets a device must not call this function on it again.
 *  - `in` may have any alignment: a base that is not 4-byte aligned takes the direct kernel.
 *  - A batch whose partial sums cannot fit (batch x one CTA's partials, T*T*4*G + T*8 bytes with
 *    G = 4, 2, 1 for T = 32, 64, 128) is rejected with HF_ERR_INVALID; larger problems are split
 *    over fewer CTAs so that they fit, which can change the float32 rounding of the partials.
 *  - Calls on one device share the array: calls whose work can overlap in time (different
 *    streams without ordering, or different host threads) race; serialise them on one stream.
 * Arguments, results and errors are otherwise those of hf_covariance. */
#define HF_COVARIANCE_NOALLOC_SCRATCH_BYTES (16u << 20)
int    hf_covariance_noalloc(const void *in, int in_dtype, int64_t batch, int T, int64_t P, double *gram,
                             hf_stream_t s);

/* Symmetric eigendecomposition (PcaHeevSolver::launch, pca_heev.cc:101-121) by FP64 cyclic
 * Jacobi, one CTA per matrix, n <= 128.  a: [batch][n][n] row-major symmetric; on return
 * evecs[b] holds eigenvector j in COLUMN j (row-major [n][n]), evals[b] ascending.  info[b] = 0 on
 * convergence, else the number of sweeps run (non-converged). */
int hf_eigh_jacobi_f64(const double *a, double *evecs, double *evals, int *info, int n,
                       int64_t batch, hf_stream_t s);
/* The r largest eigenpairs only (the clutter filter's need), n <= 128, 1 <= r <= min(16, n):
 * Householder tridiagonalisation, Sturm multisection, inverse iteration, back-transformation, one
 * CTA per matrix.  Same layout as hf_eigh_jacobi_f64, but only evals[b][n - r .. n - 1] (ascending)
 * and the matching columns of evecs[b] are written.  info[b] = 0, or 1 when a[b] is not finite. */
int hf_eigh_top_f64(const double *a, double *evecs, double *evals, int *info, int n, int r, int64_t batch,
                    hf_stream_t s);

/* Projection onto eigenvectors [begin, end) (pca.cc:106-116): out[b][c][p] =
 * sum_t X_b[t][p] * evecs_b[t][begin + c].  in: float32 [batch][T][P]. */
int hf_pca_project(const float *in, int64_t batch, int T, int64_t P, const double *evecs,
                   int begin, int end, float *out, hf_stream_t s);

/* Per-window filter+DFT matrix W = (I - V V^T) D[:, z0:z1] (V = the `rank` eigenvectors with the
 * largest eigenvalues, last columns of `evecs`), D the unnormalised DFT; float32 complex
 * [batch][T][z1-z0].  rank = 0 gives the plain band DFT matrix. */
int hf_band_matrix(const double *evecs, int64_t batch, int T, int rank, int z0, int z1,
                   void *wmat, hf_stream_t s);

/* ---- a9: Fresnel diffraction (FresnelDiffraction, fresnel_diffraction.cu:410-441) ----------
 * out = FFT2_forward(in * L) over (H, W), L[r][c] = exp(i pi/(lambda z) (x^2 + y^2)),
 * x = ((c + (S-W)/2) - S/2) dx, S = max(H, W); unnormalised, no fftshift.  If output_magnitude
 * the output is float32 |.|; otherwise complex, times L again unless skip_phase_shift.
 * Element strides (in elements of the input / output type) describe [batch][H][W] views;
 * the W stride must be 1 for the fast path (other strides use the general kernels). */
typedef struct hf_fresnel_plan hf_fresnel_plan;
int hf_fresnel_plan_create(int64_t batch, int H, int W, int in_dtype, float lambda, float dx,
                           float z, int output_magnitude, int skip_phase_shift,
                           hf_fresnel_plan **plan, hf_stream_t s);
/* z-only update without re-planning (FresnelDiffractionFactory::update, .cu:634-668). */
int hf_fresnel_plan_set_z(hf_fresnel_plan *plan, float z, hf_stream_t s);
int hf_fresnel_exec(hf_fresnel_plan *plan, const void *in, int64_t in_batch_stride,
                    int64_t in_row_stride, int64_t in_col_stride, void *out,
                    int64_t out_batch_stride, int64_t out_row_stride, int64_t out_col_stride,
                    hf_stream_t s);
int hf_fresnel_plan_destroy(hf_fresnel_plan *plan);

/* ---- a10: Angular spectrum (AngularSpectrum, angular_spectrum.cu:408-431) -----------------
 * out = IFFT2(FFT2(pad_center(in)) * TF), TF = swap_corners(exp(i 2 pi z/lambda sqrt(max(0,
 * 1 - lambda^2 (u^2+v^2)))) * w^2), both transforms unnormalised.  in: [batch][H][W] HF_F32 or
 * HF_CF32 (C-contiguous); out: [batch][OH][OW] complex64.  pad_w/pad_h = 0 for no padding;
 * in == out is allowed for CF32 without padding.  use_filter selects the raised-sine annulus
 * (r_inner, r_outer, s_inner, s_outer) of multiply_filter_2d_kernel. */
typedef struct hf_as_plan hf_as_plan;
int hf_as_plan_create(int64_t batch, int H, int W, int in_dtype, float lambda, float dx, float z,
                      int pad_w, int pad_h, int use_filter, uint32_t r_inner, uint32_t r_outer,
                      uint32_t s_inner, uint32_t s_outer, hf_as_plan **plan, hf_stream_t s);
int hf_as_exec(hf_as_plan *plan, const void *in, void *out, hf_stream_t s);
int hf_as_plan_destroy(hf_as_plan *plan);

/* ---- a11/a12/a13: Mean, MeanAbs and weighted band moments ---------------------------------
 * hf_mean_axis: mean over the middle axis of a [outer][n][inner] view (Mean with one reduced
 * axis, holonp/src/mean.cu:268-305): F32 -> F32, CF32 -> CF32, U8/U16 -> F32.
 * hf_mean_abs_axis: the same with |.| (MeanAbs, mean_abs.cu:240-275), F32 or CF32 -> F32.
 * hf_band_moments: from |S| planes [nz][P] (F32) or S planes (CF32), writes the selected
 * moments (M0 = mean |S_k|, M1 = mean f_k |S_k|, M2 = mean f_k^2 |S_k|, with f_k^2 formed in
 * float32; graph_builder.cc:612-631) as consecutive [P] float planes in M0, M1, M2 order. */
int hf_mean_axis(const void *in, int in_dtype, int64_t outer, int64_t n, int64_t inner, void *out,
                 hf_stream_t s);
int hf_mean_abs_axis(const void *in, int in_dtype, int64_t outer, int64_t n, int64_t inner,
                     float *out, hf_stream_t s);
int hf_band_moments(const void *planes, int in_dtype, int nz, int64_t P, const float *freqs,
                    int moment_mask, float *out, hf_stream_t s);

/* ---- a14: the fused per-window path ------------------------------------------------------ */
typedef struct hf_desc {
  int32_t height, width;     /* frame size                                                    */
  int32_t frames;            /* T: frames per window                                           */
  int32_t hop;               /* S: frames between consecutive windows                          */
  int32_t z_begin, z_end;    /* band bins [z0, z1) of the T-point DFT                          */
  int32_t input_dtype;       /* HF_MONO12P, HF_U16, HF_U8 or HF_F32                            */
  int32_t propagation;       /* HF_PROP_*                                                      */
  int32_t clutter_rank;      /* eigenvectors removed by the SVD clutter filter (0 = none)      */
  int32_t moment_mask;       /* HF_M0 | HF_M1 | HF_M2                                          */
  int32_t fftshift;          /* fftshift the moment images (graph_builder.cc:633-635)          */
  int32_t form;              /* HF_FORM_PLAIN or HF_FORM_CHOSEN                                */
  int32_t max_batch;         /* windows per hf_pipeline_exec call (>= 1)                       */
  float   lambda, pitch, z;  /* wavelength, pixel pitch (dx = dy), propagation distance [m]    */
  float   fs;                /* sampling rate of the moment weights [Hz] (reference: 37e3)     */
  int32_t pad_w, pad_h;      /* angular-spectrum padding (0 = none)                           */
  int32_t as_filter;         /* angular-spectrum raised-sine annulus on/off                   */
  uint32_t r_inner, r_outer, s_inner, s_outer;
  int32_t time_method;       /* HF_TIME_RFFT (0): the band [z0, z1); HF_TIME_FFT: the two-sided
                                method, [z0, z1) then [T - z1, T - z0), 2 (z1 - z0) planes
                                (graph_builder.cc:270-287, weights 590-594)                   */
  /* Shack-Hartmann autofocus before the Fresnel propagation (graph_builder.cc:139-153, 307-501):
   * each window's band planes are measured on nb x nb sub-apertures and corrected by the fitted
   * Zernike phase.  0 sub-apertures or 0 orders: off.  Fresnel propagation only.             */
  int32_t autofocus_nb_subaps;   /* odd                                                        */
  int32_t autofocus_n_iter;      /* passes (0 reads as 1)                                      */
  int32_t autofocus_n_orders;    /* entries of autofocus_orders in use                         */
  int32_t autofocus_orders[9];   /* Noll indexes 2..10                                         */
  float   autofocus_roi_radius;  /* correlation ROI radius (pp_pctclip_radius; 0 reads as 0.5) */
  int32_t autofocus_keep_outside; /* 1: keep sub-apertures outside the pupil                   */
  float   autofocus_flatfield_period; /* pp_flatfield cutoff period [m] on the sub-aperture images (0 = off) */
  /* pp_accumulation (0 or 1: off): the sub-aperture images are averaged causally over the last n
   * windows and the fit corrects the window d = (n - 1) / 2 earlier, which the plan keeps
   * (the dual-reader queue's delayed window, dual_reader_batch_queue.cc:214-227; graph_builder.cc:
   * 128-153).  Output window w is then the corrected window w - d, and the first d windows of a
   * sequence are zero images.  One pass only.  hf_plan_autofocus_reset starts a new sequence.   */
  int32_t autofocus_pp_accumulation;
  int32_t autofocus_full_pairwise; /* 1: graph-Laplacian slopes (autofocus_use_graph_laplacian)   */
} hf_desc;
#define HF_TIME_RFFT 0
#define HF_TIME_FFT 1

typedef struct hf_plan hf_plan;
/* Allocates every device buffer the path needs for max_batch windows (reference create()). */
int hf_plan_create(const hf_desc *desc, hf_plan **plan, hf_stream_t s);
int hf_plan_destroy(hf_plan *plan);
/* Rebuilds the lens / transfer function for a new z (reference z-only update()). */
int hf_plan_set_z(hf_plan *plan, float z, hf_stream_t s);
/* Output image size of the plan (AS padding enlarges it) and the number of moment planes. */
int hf_plan_output_shape(const hf_plan *plan, int32_t *out_h, int32_t *out_w, int32_t *n_moments);
/* Bytes of device memory the plan holds. */
int hf_plan_device_bytes(const hf_plan *plan, size_t *bytes);
/* Which band-DFT pass the plan runs (for 16-byte-aligned frame rings; a misaligned ring takes the
 * FP32 pass): HF_BAND_FP32 (the plain form's tiled SIMT DFT), HF_BAND_TC_ROWS (tensor cores fused
 * with the lens and the row FFT), HF_BAND_TC_RAW_ROWS (tensor cores, raw planes of whole rows, before
 * Filter2D or the autofocus) or HF_BAND_TC_SEGMENTS (tensor cores, raw planes in row segments: the
 * other chosen-form shapes). */
#define HF_BAND_FP32 0
#define HF_BAND_TC_ROWS 1
#define HF_BAND_TC_RAW_ROWS 2
#define HF_BAND_TC_SEGMENTS 3
int hf_plan_band_pass(const hf_plan *plan, int *kind);

/* Runs `nwin` (<= max_batch) windows.  Window w consists of frames
 * ring + ((first_frame + w*hop + t) mod ring_frames) * frame_bytes, t = 0..T-1, i.e. windows of
 * a device ring of `ring_frames` frames; out: [nwin][n_moments][OH][OW] float32. */
int hf_pipeline_exec(hf_plan *plan, const void *ring, int64_t ring_frames, int64_t first_frame,
                     int nwin, float *out, hf_stream_t s);

/* Per-stage device timing of hf_pipeline_exec, measured with CUDA events recorded on the exec
 * stream between stages (up to 128 execs after hf_plan_timing(plan, 1), which also resets the
 * record).  hf_plan_stage_times sums, per stage, the elapsed milliseconds over the recorded execs
 * (call after synchronising the stream); names[k] (optional) receives static stage names. */
#define HF_MAX_STAGES 16
int hf_plan_timing(hf_plan *plan, int enable);
int hf_plan_stage_times(hf_plan *plan, float *ms, const char **names, int *nstages, int *nexec);

/* Device status word of the plan (synchronises the device): 0, or the code of the first bounded
 * device-side wait (tensor-core pipeline mbarriers) that expired; `reset` clears it. */
int hf_plan_status(hf_plan *plan, int *status, int reset);

/* With autofocus on: window w's Zernike coefficients (radians, summed over the passes, in
 * autofocus_orders order) of the last hf_pipeline_exec, copied into the device buffer `coeffs`
 * (autofocus_n_orders floats) on stream s. */
int hf_plan_autofocus_coefficients(hf_plan *plan, int w, float *coeffs, hf_stream_t s);
/* Starts a new window sequence for autofocus_pp_accumulation: clears the sliding average and the
 * kept delayed windows (a camera stream does this when it is created). */
int hf_plan_autofocus_reset(hf_plan *plan, hf_stream_t s);

/* Debug/inspection: after hf_pipeline_exec, copy window `w`'s T x T Gram matrix (float64) and
 * its filter+DFT matrix W (complex64 [T][Nz]) to device buffers (either may be NULL). */
int hf_pipeline_inspect(hf_plan *plan, int w, double *gram, void *wmat, hf_stream_t s);

/* ---- a3/a4: per-camera stream (replaces BatchQueue's host ring, batch_queue.cc:92-174, with a
 * device-resident ring; overlapping windows hop < T are allowed) --------------------------------
 * A stream owns a device ring of `ring_frames` frames of the plan's input format and a window
 * cursor.  hf_stream_push appends frames (host or device memory; copies are enqueued on `s`;
 * HF_ERR_INVALID if it would overwrite frames of a window not yet processed).  hf_stream_process
 * reconstructs up to min(max_windows, max_batch) ready windows in one hf_pipeline_exec, and
 * computes the Gram matrices of the next ready batch so that its eigen phase overlaps this
 * batch's propagation on a side stream.
 * Pushes may be issued on a different CUDA stream than processes (to overlap the H2D copy of
 * later frames with the reconstruction of earlier ones): a process waits for the pushes that
 * brought its frames, and a push waits for the processes still reading the slots it overwrites.
 * All pushes of one camera stream must use one CUDA stream, and all processes one CUDA stream.
 * out_is_host: 0 = `out` is device memory; 1 = pinned host memory, copied in order on `s` (the
 * images are on the host when `s` reaches that point); 2 = pinned host memory, copied on the
 * camera stream's own copy stream so that the copy overlaps later work on `s` -- the images are
 * on the host once hf_stream_output_wait has returned with host_block = 1, or once a stream made
 * to wait by hf_stream_output_wait(st, s2, 0) reaches that point.  Two consecutive mode-2 calls
 * use two staging buffers, so the host buffer of a call must stay untouched until its copy is
 * known to be complete. */
typedef struct hf_stream hf_stream;
int     hf_stream_create(hf_plan *plan, int64_t ring_frames, hf_stream **stream);
int     hf_stream_destroy(hf_stream *stream);
int     hf_stream_push(hf_stream *stream, const void *frames, int64_t nframes, hf_stream_t s);
int64_t hf_stream_ready(const hf_stream *stream);
int     hf_stream_process(hf_stream *stream, int max_windows, float *out, int out_is_host, int *nwin,
                          hf_stream_t s);
/* Waits for the most recent asynchronous (out_is_host = 2) output copy: on the host when
 * host_block, else by making `s` wait for it. */
int     hf_stream_output_wait(hf_stream *stream, hf_stream_t s, int host_block);

/* ---- streaming server: many camera streams on one GPU, continuous batching -------------------
 * Each open stream owns a plan, a device frame ring and its own CUDA streams; plans and rings come
 * from a server-owned stream-ordered memory pool, so opening and closing never synchronise the
 * device or stall other streams' batches.  hf_server_open admits a stream only while the device
 * keeps `hbm_reserve_bytes` available (free, or held unused by the pool) after the stream's
 * buffers are created (else HF_ERR_NOMEM: retry after other streams close).  hf_server_step gives every
 * open stream with ready windows one batch on its own CUDA stream, so batches of different streams
 * run concurrently; images of stream i go to out[i] (pinned host, [max_batch][n_moments][OH][OW],
 * NULL to skip the stream) and n_done[i] receives the windows done.  out[i] may be read, and a
 * later step may reuse it, once hf_server_poll counts the step's windows (or hf_server_sync, which
 * waits for the server's own streams, has returned).  A window's frame-to-image latency (from the
 * push that brought its last frame to its images reaching the host) is collected by poll / sync
 * and read by hf_server_latencies. */
typedef struct hf_server hf_server;
int     hf_server_create(size_t hbm_reserve_bytes, int max_streams, hf_server **server);
int     hf_server_destroy(hf_server *server);
int     hf_server_open(hf_server *server, const hf_desc *desc, int64_t ring_frames, int *stream_id);
int     hf_server_close(hf_server *server, int stream_id);
int     hf_server_push(hf_server *server, int stream_id, const void *frames, int64_t nframes);
int64_t hf_server_ready(const hf_server *server, int stream_id);
int     hf_server_step(hf_server *server, float *const *out, int *n_done);
int     hf_server_sync(hf_server *server);
/* Non-blocking completion: collects every batch whose images have reached the host (latencies
 * included) without waiting for the others, and writes each slot's cumulative count of delivered
 * windows into completed[max_streams] (NULL: skip).  A stream's out[i] buffer of a step may be
 * reused once the windows of that step are counted.  hf_server_inflight: batches of stream `id`
 * still on the device.  hf_server_reserve: grows the server's memory pool by `bytes` once (plans
 * and rings of later streams then come from it without new device allocations; synchronous). */
int     hf_server_poll(hf_server *server, int64_t *completed);
int     hf_server_inflight(const hf_server *server, int stream_id);
int     hf_server_reserve(hf_server *server, size_t bytes);
int     hf_server_latencies(hf_server *server, float *ms, int cap, int *n);
int     hf_server_open_count(const hf_server *server);

/* ---- many acquisitions in one graph launch ----------------------------------------------------
 * hf_multi_create makes one plan per acquisition (frame size, window length, band, z, fs and form
 * may all differ).  hf_multi_exec reconstructs nwin[i] (NULL: max_batch) windows of every
 * acquisition i from its device ring (rings[i], ring_frames[i], first window frame first[i]) into
 * outs[i] ([nwin][n_moments][OH][OW] float32) as ONE CUDA graph launch on `s`: the graph forks
 * into branches that each run a share of the acquisitions and joins at the end.  With a fused
 * schedule, the acquisitions whose band pass is the tensor-core segment pass (hf_plan_band_pass
 * HF_BAND_TC_SEGMENTS) and that share a window length and sample format run that pass as ONE
 * persistent launch over all their (window, row, segment) units, between their Gram/eigen/W
 * fronts and their row/column backs; the images are the same as without fusion (an expired
 * bounded wait inside a fused launch sets the status word of the group's first acquisition,
 * hf_plan_status on hf_multi_plan(multi, i)).  hf_multi_tune
 * times candidate schedules on the given buffers and keeps the fastest: the number of branches and
 * the assignment (largest-first or round-robin), then fusion with its tile parameters (tiles per
 * segment, grid cap).  *best_streams receives the branch count (negative for round-robin) and
 * *best_ms the time of one launch.  The graph is captured on the first exec (and again whenever
 * the buffers or the schedule change): make that call outside any other capture. */
typedef struct hf_multi hf_multi;
typedef struct hf_multi_schedule {
  int32_t branches;      /* 1 .. 6 */
  int32_t largest_first; /* 1: acquisitions dealt largest-first to the least-loaded branch; 0: round-robin */
  int32_t fused;         /* 1: one segment-pass launch per (window length, format) */
  int32_t seg_tiles;     /* tiles per segment of the fused launch; 0 = the most A and TMEM hold */
  int32_t band_ctas;     /* grid cap of the fused launch; 0 = every SM */
} hf_multi_schedule;
int hf_multi_create(int n_acquisitions, const hf_desc *descs, hf_multi **multi);
int hf_multi_destroy(hf_multi *multi);
int hf_multi_exec(hf_multi *multi, const void *const *rings, const int64_t *ring_frames, const int64_t *first,
                  const int *nwin, float *const *outs, hf_stream_t s);
int hf_multi_tune(hf_multi *multi, const void *const *rings, const int64_t *ring_frames, const int64_t *first,
                  const int *nwin, float *const *outs, int reps, hf_stream_t s, int *best_streams, float *best_ms);
/* The plan of acquisition i (owned by the multi). */
int hf_multi_plan(hf_multi *multi, int i, hf_plan **plan);
/* Read or set the schedule (hf_multi_tune sets it; a set schedule is checked and used from the next
 * exec). */
int hf_multi_get_schedule(const hf_multi *multi, hf_multi_schedule *schedule);
int hf_multi_set_schedule(hf_multi *multi, const hf_multi_schedule *schedule);

/* ---- node layer: compute nodes by kind string (ISyncTaskFactory / ISyncTask, tasks.hh:182-304;
 * kinds registered by string, registry.hh:24-68, manager.cc:159-237) ---------------------------
 * Kinds: "FresnelDiffraction", "AngularSpectrum", "Pca", "FFT", "RFFT", "Mean", "MeanAbs",
 * "Conversion", "FFTShiftNp", "Flatfield", "Filter2D", "PctClip", "Holofile", the autofocus kinds,
 * the thin holonp kinds "Slice", "Reshape", "Copy", "Concatenate", "Arange", "Multiply", "Abs",
 * "CausalSlidingAverage", the asynchronous "BatchQueue", "DualReaderBatchQueue", "SlidingAverage"
 * (the reference's, with its JSON settings keys) and "DopplerMoments" (the fused per-window path).  A descriptor mirrors holoflow::core::TDesc: dtype in DType order (HF_U8,
 * HF_U16, HF_F32, HF_CF32), strides in BYTES (all zero = C-contiguous), mem_loc 1 = device.
 * infer() failures return HF_ERR_INVALID with "<Factory> inference error: ..." in hf_last_error();
 * work is enqueued on the stream given at create/update. */
#define HF_TDESC_MAX_RANK 8
typedef struct hf_tdesc {
  int32_t rank, dtype, mem_loc, reserved;
  int64_t shape[HF_TDESC_MAX_RANK];
  int64_t strides[HF_TDESC_MAX_RANK];
  int64_t offset;
} hf_tdesc;
typedef struct hf_node hf_node;
/* Comma-separated list of the registered kinds. */
int hf_node_kinds(char *buf, size_t cap);
/* Output descriptors of a node without creating it (ITaskFactory::infer). */
int hf_node_infer(const char *kind, const char *json_settings, int n_inputs, const hf_tdesc *inputs, int *n_outputs,
                  hf_tdesc *outputs, int outputs_cap);
/* infer + create (ISyncTaskFactory::create); the node keeps the descriptors. */
int hf_node_create(const char *kind, const char *json_settings, int n_inputs, const hf_tdesc *inputs, hf_stream_t s,
                   hf_node **node);
/* ISyncTaskFactory::update: reuses the task where the factory can (z-only changes). */
int hf_node_update(hf_node *node, const char *json_settings, int n_inputs, const hf_tdesc *inputs, hf_stream_t s);
/* ISyncTask::execute on tensors given by their origin pointers; *op_result receives the
 * OpResult (0 = Ok).  An output the node owns (InferResult::owned_outputs, e.g. a cached
 * "Holofile" source) takes NULL here: the node publishes its own pointer, which
 * hf_node_output_ptr returns after the call. */
int hf_node_execute(hf_node *node, void *const *inputs, void *const *outputs, int *op_result);
int hf_node_output_desc(const hf_node *node, int index, hf_tdesc *out);
/* Origin pointer of output `index` as of the last hf_node_execute (the caller's pointer for a
 * caller-provided output, the node's own for an owned one); *owned = 1 if the node owns it. */
int hf_node_output_ptr(const hf_node *node, int index, void **ptr, int *owned);
int hf_node_destroy(hf_node *node);
/* In-place outputs (InferResult::in_place, e.g. "Slice" and a viewing "Reshape"): output `index`
 * is a view of input *input_index (-1: not a view); hf_node_execute takes NULL for it and
 * hf_node_output_ptr returns the view's origin inside the input. */
int hf_node_output_alias(const hf_node *node, int index, int *input_index);
/* Asynchronous kinds (IAsyncTask, tasks.hh:208-250: "BatchQueue", "DualReaderBatchQueue",
 * "SlidingAverage"), created by hf_node_create with AsyncCreateCtx{s, s}.  The producer takes the
 * view of owned input `index` to write (*ptr NULL: no room now), then hf_node_try_push publishes it;
 * the consumer's hf_node_try_pop (op_result 1 = NotReady) hands out owned outputs, read through
 * hf_node_output_ptr, and takes caller buffers for the outputs the node does not own (NULL entries
 * for owned ones); hf_node_release_output retires an owned output of the last pop. */
int hf_node_is_async(const hf_node *node);
int hf_node_acquire_input(hf_node *node, int index, void **ptr);
int hf_node_try_push(hf_node *node, int *op_result);
int hf_node_try_pop(hf_node *node, void *const *outputs, int *op_result);
int hf_node_release_output(hf_node *node, int index);

/* ---- post-moment display chain (graph_builder.cc:633-676) -------------------------------------
 * The steps between a moment image and the display: fftshift, flatfield, sliding average,
 * percentile clip, then hf_convert(..., HF_CONV_SCALED) to U8.  Work is enqueued on `s`;
 * create functions allocate their device state on the current device (hf_pctclip_create also
 * synchronizes `s` once to count the region's pixels, as the reference does at create). */

/* holonp FFTShift (holonp/src/fftshift.cu:98-134): out[j] = in[(j + n/2) mod n] along every axis
 * k with bit k of axes_mask set (axis 0 = outermost); in and out must not alias. */
int hf_fftshift(const void *in, void *out, int elem_size, int ndim, const int64_t *shape, uint32_t axes_mask,
                hf_stream_t s);

/* Flatfield (holotask/src/syncs/flatfield.cu): out = in - Gaussian(in) on each [height][width]
 * plane of planes; sigmas in pixels.  Kernels of fewer than 65 taps run spatially with
 * clamp-at-edge borders, longer ones as the analytic Fourier high-pass (image sides in
 * {64..1536}, height <= 1024); hf_flatfield_is_fourier tells which. */
typedef struct hf_flatfield hf_flatfield;
int hf_flatfield_create(int64_t planes, int height, int width, float sigma_y, float sigma_x, hf_stream_t s,
                        hf_flatfield **ff);
int hf_flatfield_is_fourier(const hf_flatfield *ff, int *fourier);
int hf_flatfield_exec(hf_flatfield *ff, const float *in, float *out, hf_stream_t s);
int hf_flatfield_destroy(hf_flatfield *ff);

/* Filter2D (holotask/src/syncs/filter2d.cu): out = IFFT2(FFT2(in) x mask) per [height][width]
 * plane, unnormalized, mask = the band-pass annulus a (1 - b) of radii r_inner / r_outer with
 * raised-cosine edges s_inner / s_outer.  real_input = 0: complex64 in and out (in place allowed),
 * the mask applied as (g, g) like the reference's complex path; real_input = 1: float32 in and
 * out, the mask (g, 0).  Image sides in {64..1536}, height <= 1024. */
typedef struct hf_filter2d hf_filter2d;
int hf_filter2d_create(int64_t planes, int height, int width, int real_input, uint32_t r_inner, uint32_t r_outer,
                       uint32_t s_inner, uint32_t s_outer, hf_stream_t s, hf_filter2d **f);
int hf_filter2d_exec(hf_filter2d *f, const void *in, void *out, hf_stream_t s);
int hf_filter2d_destroy(hf_filter2d *f);

/* PctClip (holotask/src/syncs/pct_clip.cu): clips [depth][height][width] to the values at
 * ranks int(pct / 100 * (count - 1)) of the pixels inside the ellipse (normalized centre, radii
 * and angle in degrees, applied to every slice).  `bounds` (optional, device float[2]) receives
 * the two values. */
typedef struct hf_ellipse {
  float cx, cy, rx, ry, angle;
} hf_ellipse;
typedef struct hf_pctclip hf_pctclip;
int hf_pctclip_create(int depth, int height, int width, float min_pct, float max_pct, const hf_ellipse *roi,
                      hf_stream_t s, hf_pctclip **pc);
int hf_pctclip_roi_count(const hf_pctclip *pc, int *count);
int hf_pctclip_exec(hf_pctclip *pc, const float *in, float *out, float *bounds, hf_stream_t s);
int hf_pctclip_destroy(hf_pctclip *pc);

/* SlidingAverage (holotask/src/asyncs/slide_avg.cu): the mean of the last window_size images,
 * kept as a float32 running average (avg += x / n; avg -= x_old / n).  The first discard_first
 * images are dropped; *ready becomes 1 (and `out`, if given, holds the average) once window_size
 * images have entered. */
typedef struct hf_slideavg hf_slideavg;
int hf_slideavg_create(int64_t npix, int window_size, int discard_first, hf_stream_t s, hf_slideavg **sa);
int hf_slideavg_push(hf_slideavg *sa, const float *in, float *out, int *ready, hf_stream_t s);
int hf_slideavg_destroy(hf_slideavg *sa);

/* ---- .holo acquisition files (holofile/include/holofile/holofile.hh:87-152) -------------------
 * A 64-byte little-endian header (magic "HOLO", version 66, bits_per_pixel, width, height,
 * frame_count, data_size_in_bytes, endianness), the frames, then an optional JSON footer.
 * bits_per_pixel 8 and 16 are the reference's pixel types; 12 holds Mono12p frames (2 pixels in
 * 3 bytes, the HF_MONO12P layout).  Errors: HF_ERR_INVALID for a malformed file (message
 * "Holofile: Incomplete header" / "Invalid magic number" / "Invalid frame size" as the
 * reference's exceptions), HF_ERR_STATE for I/O failures and reading past the last frame
 * ("Holofile: End of file reached"). */
#pragma pack(push, 1)
typedef struct hf_holo_header {
  uint32_t magic_number;
  uint16_t version, bits_per_pixel;
  uint32_t frame_width, frame_height, frame_count;
  uint64_t data_size_in_bytes; /* at byte 20: the struct is packed */
  uint8_t  endianness;
  char     padding[35];
} hf_holo_header; /* byte-for-byte the file's 64-byte header */
#pragma pack(pop)
typedef struct hf_holo_reader hf_holo_reader;
typedef struct hf_holo_writer hf_holo_writer;
int hf_holo_open(const char *path, hf_holo_reader **reader);
int hf_holo_header_get(const hf_holo_reader *reader, hf_holo_header *header);
/* The footer JSON text (NUL-terminated) in buf; *len receives its length, 0 when the file has
 * no valid footer.  buf may be NULL to query the length. */
int hf_holo_footer(const hf_holo_reader *reader, char *buf, size_t cap, size_t *len);
int hf_holo_seek(hf_holo_reader *reader, int64_t frame_index);
int hf_holo_tell(const hf_holo_reader *reader, int64_t *frame_index);
/* Reads `count` frames at the cursor into host memory `dst` (pageable or pinned). */
int hf_holo_read(hf_holo_reader *reader, void *dst, int64_t count);
int hf_holo_close(hf_holo_reader *reader);
/* Creates `path` with a header for frame_count frames of width x height at bits_per_pixel
 * (8, 12 or 16) and the footer JSON text (NULL or empty for an empty object). */
int hf_holo_create(const char *path, uint32_t frame_count, uint32_t width, uint32_t height, uint16_t bits_per_pixel,
                   const char *footer_json, hf_holo_writer **writer);
int hf_holo_write(hf_holo_writer *writer, const void *src, int64_t count);
/* Appends the footer and closes the file. */
int hf_holo_finish(hf_holo_writer *writer);

/* ---- Shack-Hartmann autofocus (graph_builder.cc:307-501) --------------------------------------
 * Sub-aperture and correlation transforms take any side 2..1024 (HF_ERR_UNSUPPORTED beyond).
 * Validation failures return HF_ERR_INVALID with the reference factory's message.
 *
 * ShortTimeFresnelDiffraction (holotask/include/holotask/syncs/short_time_fresnel_diffraction.hh:
 * 40-56): `planes` fields [planes][H][W] (complex64, or float32 when real_input), windows of
 * win_h x win_w every stride_y / stride_x pixels, each times the quadratic input lens (the whole
 * field's frame for HF_STFD_GLOBAL, the window's for HF_STFD_LOCAL), unnormalised 2D forward FFT.
 * Outputs: HF_STFD_COMPLEX [planes][ny][nx][win_h][win_w] complex64 (times the window lens unless
 * skip_phase_shift); HF_STFD_MAGNITUDE the same shape in float32 (output_magnitude); and
 * HF_STFD_MEAN_MAGNITUDE [ny][nx][win_h][win_w] float32, the mean of |.| over the planes (the
 * reference's following Mean over the band axis), each window fftshifted when fftshift_windows.
 * hf_stfd_set_z replaces the distance (the factory's z-only update). */
#define HF_STFD_LOCAL 0
#define HF_STFD_GLOBAL 1
#define HF_STFD_COMPLEX 0
#define HF_STFD_MAGNITUDE 1
#define HF_STFD_MEAN_MAGNITUDE 2
typedef struct hf_stfd hf_stfd;
int hf_stfd_create(int64_t planes, int height, int width, int real_input, int win_h, int win_w, int stride_y,
                   int stride_x, float lambda, float dx, float dy, float z, int phase_ref, int output,
                   int skip_phase_shift, int fftshift_windows, hf_stream_t s, hf_stfd **f);
int hf_stfd_grid(const hf_stfd *f, int *ny, int *nx);
int hf_stfd_set_z(hf_stfd *f, float z, hf_stream_t s);
int hf_stfd_exec(hf_stfd *f, const void *in, void *out, hf_stream_t s);
int hf_stfd_destroy(hf_stfd *f);

/* ShackHartmannSlopes, single-reference mode (holotask/include/holotask/syncs/
 * shack_hartmann_slopes.hh:28-61): images [sy][sx][h][w] float32 (sy, sx odd) -> slopes
 * [sy][sx][2] float32: each image phase-correlated with the centre one inside the ROI ellipse
 * (mean removed, cosine taper), peak offset with parabolic refinement, times lambda / (n d),
 * centre offset and the mean over the active sub-apertures removed (inactive ones 0).  The
 * active set comes from the sub-aperture geometry (sub_h x sub_w every stride_y / stride_x
 * pixels; all four 0: the image size).  `maps`
 * (optional, [sy][sx][h][w]) receives the correlation maps.  hf_shslopes_active writes the
 * active flags (1 byte per sub-aperture). */
typedef struct hf_shslopes hf_shslopes;
int hf_shslopes_create(int sy, int sx, int height, int width, int sub_h, int sub_w, int stride_y, int stride_x,
                       float lambda, float dx, float dy, float z, const hf_ellipse *roi, int skip_outside_pupil,
                       hf_stream_t s, hf_shslopes **p);
int hf_shslopes_active(const hf_shslopes *p, uint8_t *active);
int hf_shslopes_exec(hf_shslopes *p, const float *images, float *slopes, float *maps, hf_stream_t s);
/* hf_shslopes_create with a slope recovery mode (ShackHartmannSlopeMode, shack_hartmann_slopes.hh:
 * 27-31; the graph-Laplacian `autofocus_use_graph_laplacian` switch of graph_builder.cc:359-361).
 * FULL_PAIRWISE phase-correlates every pair (i < j) of active samples, pair_batch_size maps at a time
 * (its memory bound), and solves the complete-graph Laplacian in the zero-mean gauge
 * (shack_hartmann_slopes_full_pairwise.cuh:69-262): it takes any grid with at least two active
 * samples and gives no correlation maps.  Synchronous (uploads the pair lists). */
#define HF_SHSLOPES_SINGLE_REFERENCE 0
#define HF_SHSLOPES_FULL_PAIRWISE 1
int hf_shslopes_create_mode(int sy, int sx, int height, int width, int sub_h, int sub_w, int stride_y, int stride_x,
                            float lambda, float dx, float dy, float z, const hf_ellipse *roi, int skip_outside, int mode,
                            int pair_batch_size, hf_stream_t s, hf_shslopes **p);
int hf_shslopes_destroy(hf_shslopes *p);

/* ZernikeFromSlopes (holotask/include/holotask/syncs/zernike_from_slopes.hh:27-45): Noll indexes
 * 2..10 (unique, at most 9); tip and tilt stay 0; the other coefficients (radians) are the
 * least-squares fit of the zero-mean slopes.  hf_zernike_fit_exec runs on the device (device
 * slopes [sy*sx*2] -> device coefficients; `cumulative`, optional, accumulates them) with the
 * reference's float32 sequence; hf_zernike_fit_host runs the same on host arrays. */
typedef struct hf_zernike_fit hf_zernike_fit;
int hf_zernike_fit_create(int sy, int sx, int sub_h, int sub_w, int stride_y, int stride_x, float lambda, float dx,
                          float dy, int skip_outside_pupil, const int *indexes, int n_indexes, hf_zernike_fit **f);
int hf_zernike_fit_pupil_radius(const hf_zernike_fit *f, float *radius);
int hf_zernike_fit_exec(hf_zernike_fit *f, const float *slopes, float *coeffs, float *cumulative, hf_stream_t s);
int hf_zernike_fit_host(const hf_zernike_fit *f, const float *slopes, float *coeffs);
int hf_zernike_fit_destroy(hf_zernike_fit *f);

/* ZernikePhase (zernike_phase.hh): device coefficients -> device phase [ny][nx] (optional
 * `cumulative` += phase).  CorrectPhase (correct_phase.cu): out = in exp(-i phase), the [H][W]
 * phase broadcast over `planes`, complex64 or float32 input, complex64 output (in place allowed
 * for complex input).  Wrap2Pi (wrap2pi.cu): fmod by 2 pi into [0, 2 pi).  hf_defocus_z is
 * ZernikeDefocusZProp's estimate (zernike_defocus_z_prop.cc:84-97) from the defocus coefficient. */
int hf_zernike_phase(const float *coeffs, const int *indexes, int n_indexes, int ny, int nx, float *phase,
                     float *cumulative, hf_stream_t s);
int hf_correct_phase(const void *in, int complex_input, const float *phase, int64_t planes, int height, int width,
                     void *out, hf_stream_t s);
int hf_wrap2pi(const float *in, float *out, int64_t n, hf_stream_t s);
int hf_defocus_z(float a4, float lambda, float z_curr, float pupil_radius, double *delta_inv_z, double *z_new,
                 double *delta_z_mm);

/* One autofocus pass chain on one spectrum (build_shack_hartmann, graph_builder.cc:307-501, with
 * pp_accumulation 1): sub-apertures of W / nb x H / nb (nb odd), short-time Fresnel with the
 * global phase, mean |.| over the nz planes, fftshift, optionally the flatfield of pp_flatfield
 * (flatfield_period > 0: the cutoff period in metres, sigma = 0.187 period / (lambda |z| / (n dx));
 * 0: off), single-reference slopes
 * in the ROI circle of radius roi_radius, device Zernike fit, phase map over H x W, and
 * corrected = delayed exp(-i phase) (delayed NULL: the planes themselves).  n_iter passes chain
 * as the reference's (each later pass measures and corrects the previous output);
 * hf_autofocus_outputs copies (on stream s, into device buffers; NULL skips one) the last exec's
 * M0 [nb][nb][sh][sw], slopes [nb][nb][2], and the coefficients [n_indexes] and phase [H][W]
 * summed over the passes.  With n_indexes 0 the planes pass through. */
typedef struct hf_autofocus hf_autofocus;
int hf_autofocus_create(int nz, int height, int width, int nb_subaps, int n_iter, float lambda, float dx, float z,
                        float roi_radius, int skip_outside_pupil, const int *indexes, int n_indexes,
                        float flatfield_period, hf_stream_t s, hf_autofocus **a);
/* pp_accumulation > 1 (graph_builder.cc:128-153, 348): the sub-aperture images of each exec's
 * first pass enter a causal sliding average over the last pp_accumulation execs (divisor
 * min(k + 1, n), float32 running sum, causal_sliding_average.cu:35-90) before the slopes; one pass
 * only.  The caller supplies the delayed spectrum to correct (hf_autofocus_exec's `delayed`).
 * hf_autofocus_reset clears the average (a new stream).  Both enqueue on s. */
int hf_autofocus_set_accumulation(hf_autofocus *a, int pp_accumulation, hf_stream_t s);
int hf_autofocus_reset(hf_autofocus *a, hf_stream_t s);
/* Slope recovery of the pass: HF_SHSLOPES_SINGLE_REFERENCE or HF_SHSLOPES_FULL_PAIRWISE (the
 * `autofocus_use_graph_laplacian` switch, graph_builder.cc:359-361) with the same ROI radius,
 * pupil rule and optics as at create. */
int hf_autofocus_set_slope_mode(hf_autofocus *a, int mode, int pair_batch_size, float roi_radius,
                                int skip_outside_pupil, float lambda, float dx, float z, hf_stream_t s);
int hf_autofocus_pupil_radius(const hf_autofocus *a, float *radius);
int hf_autofocus_exec(hf_autofocus *a, const void *planes, const void *delayed, void *corrected, hf_stream_t s);
int hf_autofocus_outputs(const hf_autofocus *a, float *m0, float *slopes, float *coeffs, float *phase, hf_stream_t s);
int hf_autofocus_destroy(hf_autofocus *a);

#ifdef __cplusplus
}
#endif

#endif /* HOLOFLOW_B200_H */
