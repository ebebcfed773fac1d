// C ABI of the library: status/error plumbing, stage entry points and the plans (fused
// per-window pipeline, Fresnel and angular-spectrum nodes).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "k_band.cuh"
#include "k_fft2d.cuh"
#include "k_misc.cuh"
#include "k_pca.cuh"
#include "k_tc_band.cuh"

namespace hf {

namespace {
thread_local std::string g_error;
thread_local int64_t     g_launches = 0;
} // namespace

void set_error(const std::string &msg) { g_error = msg; }
void clear_error() { g_error.clear(); }
int  fail(int code, const std::string &msg) {
  g_error = msg;
  return code;
}
int cuda_status(cudaError_t e, const char *where) {
  if (e == cudaSuccess)
    return HF_OK;
  g_error = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return e == cudaErrorMemoryAllocation ? HF_ERR_NOMEM : HF_ERR_CUDA;
}
void note_launch(int n) { g_launches += n; }

namespace {

template <typename T> int dev_alloc(T **p, size_t count, size_t &total) {
  *p = nullptr;
  if (count == 0)
    return HF_OK;
  const size_t bytes = count * sizeof(T);
  cudaError_t  e     = cudaMalloc(reinterpret_cast<void **>(p), bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    (void)cudaGetLastError();
    return fail(HF_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
  }
  total += bytes;
  return HF_OK;
}

template <typename T> void dev_free(T *&p) {
  if (p)
    cudaFree(p);
  p = nullptr;
}

float norm_scale(int norm, int n) {
  if (norm == HF_NORM_FORWARD)
    return (float)(1.0 / (double)n);
  if (norm == HF_NORM_ORTHO)
    return (float)(1.0 / std::sqrt((double)n));
  return 1.0f;
}

bool real_fmt(int f) { return f == HF_U8 || f == HF_U16 || f == HF_F32 || f == HF_MONO12P; }

// f_k = start + k*df evaluated in double and cast (arange.cu:62-75); f_k^2 in float32
// (graph_builder.cc:624-627).
void fill_weights(MomentSpec &m, int T, int z0, int nz, double fs) {
  const double df = fs / (double)T;
  const double f0 = z0 * df;
  for (int k = 0; k < kMaxBands; ++k) {
    const float f = k < nz ? (float)(f0 + df * (double)k) : 0.f;
    m.w1[k]       = f;
    m.w2[k]       = f * f;
  }
}

} // namespace
} // namespace hf

using namespace hf;

// ================================================================================================
// Fused per-window pipeline plan
// ================================================================================================
struct hf_plan {
  hf_desc    d{};
  int        P = 0, nz = 0, nmom = 0, OH = 0, OW = 0;
  bool       fast = false;
  int64_t    frame_bytes = 0;
  MomentSpec mom{};
  float2    *lens = nullptr, *tf = nullptr, *band = nullptr, *band2 = nullptr;
  float2    *wmat = nullptr, *wmat_plain = nullptr;
  double    *gram = nullptr, *evecs = nullptr, *evals = nullptr;
  int       *info = nullptr;
  int       *status = nullptr; // device status word: nonzero when a bounded device wait expired
  void      *cov_ws = nullptr;
  bool       cov_tc = false;   // tensor-core Gram matrix (chosen form)
  bool       rows_tc = false;  // tensor-core band DFT fused with lens + row FFT (chosen form)
  size_t     bytes = 0;
  // optional per-stage CUDA-event timing (hf_plan_timing / hf_plan_stage_times)
  static constexpr int kSets = 128, kMarks = HF_MAX_STAGES + 1;
  bool        timing = false;
  int         nexec = 0;
  cudaEvent_t ev[kSets][kMarks] = {};
  int         marks[kSets] = {};
  const char *stage_name[HF_MAX_STAGES] = {};
  int         nstages = 0;
};

// Marks a stage boundary when timing is on (event k of the current exec's set).
static void mark(hf_plan *p, cudaStream_t s, int k, const char *name_of_prev) {
  if (!p->timing || p->nexec >= hf_plan::kSets)
    return;
  cudaEventRecord(p->ev[p->nexec][k], s);
  p->marks[p->nexec] = k + 1;
  if (k > 0 && name_of_prev)
    p->stage_name[k - 1] = name_of_prev;
}

static int finish_exec(hf_plan *p) {
  if (p->timing && p->nexec < hf_plan::kSets) {
    p->nstages = p->marks[p->nexec] - 1;
    ++p->nexec;
  }
  return HF_OK;
}

static void plan_free(hf_plan *p) {
  for (int i = 0; i < hf_plan::kSets; ++i)
    for (int k = 0; k < hf_plan::kMarks; ++k)
      if (p->ev[i][k]) {
        cudaEventDestroy(p->ev[i][k]);
        p->ev[i][k] = nullptr;
      }
  dev_free(p->lens);
  dev_free(p->tf);
  dev_free(p->band);
  dev_free(p->band2);
  dev_free(p->wmat);
  dev_free(p->wmat_plain);
  dev_free(p->gram);
  dev_free(p->evecs);
  dev_free(p->evals);
  dev_free(p->info);
  dev_free(p->status);
  if (p->cov_ws)
    cudaFree(p->cov_ws);
  p->cov_ws = nullptr;
}

static int plan_tables(hf_plan *p, cudaStream_t s) {
  const hf_desc &d = p->d;
  if (d.propagation == HF_PROP_FRESNEL)
    HF_TRY(launch_fresnel_lens(p->lens, d.width, d.height, d.lambda, d.z, d.pitch, s));
  if (d.propagation == HF_PROP_ANGULAR_SPECTRUM) {
    AsFilter f{d.r_inner, d.r_outer, d.s_inner, d.s_outer};
    HF_TRY(launch_as_tf(p->tf, p->OW, p->OH, d.lambda, d.z, d.pitch, d.as_filter, f, s));
  }
  return HF_OK;
}

extern "C" {

const char *hf_last_error(void) { return g_error.c_str(); }
int         hf_version(void) { return 10000; }
int64_t     hf_launch_count(void) { return g_launches; }
void        hf_reset_launch_count(void) { g_launches = 0; }

int hf_plan_create(const hf_desc *desc, hf_plan **out, hf_stream_t stream) {
  clear_error();
  HF_CHECK_ARG(desc != nullptr && out != nullptr, "hf_plan_create: null argument");
  *out = nullptr;
  const hf_desc &d = *desc;
  HF_CHECK_ARG(d.height > 0 && d.width > 0, "plan: frame size must be positive");
  HF_CHECK_ARG(d.frames >= 2 && d.frames <= 128, "plan: frames per window must be in [2, 128]");
  HF_CHECK_ARG(d.hop >= 1, "plan: hop must be >= 1");
  HF_CHECK_ARG(d.z_begin >= 0 && d.z_end > d.z_begin && d.z_end <= d.frames,
               "plan: band must satisfy 0 <= z_begin < z_end <= frames");
  HF_CHECK_ARG(d.z_end - d.z_begin <= kMaxBands, "plan: at most 64 band bins");
  HF_CHECK_ARG(d.input_dtype == HF_MONO12P || d.input_dtype == HF_U16 || d.input_dtype == HF_U8 ||
                   d.input_dtype == HF_F32,
               "plan: input dtype must be MONO12P, U16, U8 or F32");
  HF_CHECK_ARG(d.input_dtype != HF_MONO12P || ((int64_t)d.height * d.width) % 2 == 0,
               "plan: 12-bit packed frames need an even pixel count");
  HF_CHECK_ARG(d.propagation >= HF_PROP_NONE && d.propagation <= HF_PROP_ANGULAR_SPECTRUM,
               "plan: unknown propagation");
  HF_CHECK_ARG(d.clutter_rank >= 0 && d.clutter_rank < d.frames, "plan: clutter rank must be < frames");
  HF_CHECK_ARG((d.moment_mask & 7) != 0 && (d.moment_mask & ~7) == 0, "plan: bad moment mask");
  HF_CHECK_ARG(d.max_batch >= 1, "plan: max_batch must be >= 1");
  HF_CHECK_ARG(d.form == HF_FORM_PLAIN || d.form == HF_FORM_CHOSEN, "plan: unknown form");
  if (d.propagation != HF_PROP_NONE) {
    HF_CHECK_ARG(d.lambda > 0.f && d.pitch > 0.f, "plan: wavelength and pitch must be positive");
  }
  const bool padded = d.propagation == HF_PROP_ANGULAR_SPECTRUM && (d.pad_w > 0 || d.pad_h > 0);
  if (padded)
    HF_CHECK_ARG(d.pad_w >= d.width && d.pad_h >= d.height && (d.pad_w - d.width) % 2 == 0 &&
                     (d.pad_h - d.height) % 2 == 0,
                 "plan: padding must be >= the frame and leave even margins");
  hf_plan *p = new (std::nothrow) hf_plan();
  if (!p)
    return fail(HF_ERR_NOMEM, "plan: host allocation failed");
  p->d           = d;
  p->P           = d.height * d.width;
  p->nz          = d.z_end - d.z_begin;
  p->nmom        = __builtin_popcount(d.moment_mask);
  p->OH          = padded ? d.pad_h : d.height;
  p->OW          = padded ? d.pad_w : d.width;
  p->frame_bytes = frame_bytes_of(d.input_dtype, p->P);
  p->fast = fft_fast_length(p->OH) && fft_fast_length(p->OW);
  if (d.propagation == HF_PROP_ANGULAR_SPECTRUM && !(p->fast && p->OH <= 1024)) {
    delete p;
    return fail(HF_ERR_UNSUPPORTED,
                "plan: angular spectrum pipeline needs padded sizes in {64..1536} (rows <= 1024)");
  }
  p->mom.nz       = p->nz;
  p->mom.mask     = d.moment_mask;
  p->mom.fftshift = d.fftshift;
  p->mom.inv_nz   = 1.0f / (float)p->nz;
  fill_weights(p->mom, d.frames, d.z_begin, p->nz, d.fs > 0.f ? d.fs : 37e3);

  const int64_t B = d.max_batch;
  int rc = HF_OK;
  do {
    const int64_t plane = (int64_t)p->P, oplane = (int64_t)p->OH * p->OW;
    if ((rc = dev_alloc(&p->band, (size_t)(B * p->nz * plane), p->bytes)))
      break;
    const bool need_band2 = d.propagation == HF_PROP_ANGULAR_SPECTRUM ||
                            (d.propagation == HF_PROP_FRESNEL && !p->fast);
    if (need_band2 && (rc = dev_alloc(&p->band2, (size_t)(B * p->nz * oplane), p->bytes)))
      break;
    if (d.propagation == HF_PROP_FRESNEL && (rc = dev_alloc(&p->lens, (size_t)plane, p->bytes)))
      break;
    if (d.propagation == HF_PROP_ANGULAR_SPECTRUM && (rc = dev_alloc(&p->tf, (size_t)oplane, p->bytes)))
      break;
    if (d.clutter_rank > 0) {
      const int T = d.frames;
      if ((rc = dev_alloc(&p->gram, (size_t)(B * T * T), p->bytes)) ||
          (rc = dev_alloc(&p->evecs, (size_t)(B * T * T), p->bytes)) ||
          (rc = dev_alloc(&p->evals, (size_t)(B * T), p->bytes)) ||
          (rc = dev_alloc(&p->info, (size_t)B, p->bytes)) ||
          (rc = dev_alloc(&p->wmat, (size_t)(B * T * p->nz), p->bytes)))
        break;
      p->cov_tc = d.form == HF_FORM_CHOSEN && cov_tc_supported(d.input_dtype, T, p->P, p->frame_bytes);
      size_t wsb = cov_workspace_bytes(T, p->P, (int)B) + cov_workspace_bytes(T, p->P, 1);
      if (p->cov_tc)
        wsb = std::max(wsb, cov_tc_workspace_bytes(T, p->P, (int)B) + cov_tc_workspace_bytes(T, p->P, 1));
      uint8_t *ws = nullptr;
      if ((rc = dev_alloc(&ws, wsb, p->bytes)))
        break;
      p->cov_ws = ws;
    } else {
      if ((rc = dev_alloc(&p->wmat_plain, (size_t)d.frames * p->nz, p->bytes)))
        break;
      if ((rc = launch_band_matrix(nullptr, 1, d.frames, 0, d.z_begin, d.z_end, p->wmat_plain, stream)))
        break;
    }
    if ((rc = dev_alloc(&p->status, 1, p->bytes)))
      break;
    if ((rc = cuda_status(cudaMemsetAsync(p->status, 0, sizeof(int), stream), "status reset")))
      break;
    p->rows_tc = d.form == HF_FORM_CHOSEN && d.propagation == HF_PROP_FRESNEL && p->fast &&
                 band_rows_tc_supported(d.input_dtype, d.frames, d.width, p->nz, p->frame_bytes);
    rc = plan_tables(p, stream);
  } while (0);
  if (rc != HF_OK) {
    plan_free(p);
    delete p;
    return rc;
  }
  *out = p;
  return HF_OK;
}

int hf_plan_destroy(hf_plan *p) {
  if (!p)
    return HF_OK;
  cudaDeviceSynchronize();
  plan_free(p);
  delete p;
  return HF_OK;
}

int hf_plan_set_z(hf_plan *p, float z, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(p != nullptr, "hf_plan_set_z: null plan");
  p->d.z = z;
  return plan_tables(p, s);
}

int hf_plan_output_shape(const hf_plan *p, int32_t *oh, int32_t *ow, int32_t *nm) {
  HF_CHECK_ARG(p != nullptr, "hf_plan_output_shape: null plan");
  if (oh)
    *oh = p->OH;
  if (ow)
    *ow = p->OW;
  if (nm)
    *nm = p->nmom;
  return HF_OK;
}

int hf_plan_device_bytes(const hf_plan *p, size_t *bytes) {
  HF_CHECK_ARG(p != nullptr && bytes != nullptr, "hf_plan_device_bytes: null argument");
  *bytes = p->bytes;
  return HF_OK;
}

int hf_pipeline_exec(hf_plan *p, const void *ring, int64_t ring_frames, int64_t first_frame,
                     int nwin, float *out, hf_stream_t stream) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && ring != nullptr && out != nullptr, "hf_pipeline_exec: null argument");
  HF_CHECK_ARG(nwin >= 1 && nwin <= p->d.max_batch, "hf_pipeline_exec: nwin must be in [1, max_batch]");
  HF_CHECK_ARG(ring_frames >= p->d.frames && first_frame >= 0,
               "hf_pipeline_exec: the ring must hold at least one window");
  const hf_desc &d = p->d;
  cudaStream_t   s = stream;
  FrameRing      fr{reinterpret_cast<const uint8_t *>(ring), ring_frames, first_frame % ring_frames,
               (int64_t)d.hop, p->frame_bytes};
  const int T = d.frames;
  int       mk = 0;
  // the tensor-core passes read 16-byte runs of the ring: fall back to the plain kernels otherwise
  const bool aligned16 = (reinterpret_cast<uintptr_t>(ring) & 15) == 0;
  const bool cov_tc    = p->cov_tc && aligned16;
  const bool rows_tc   = p->rows_tc && aligned16;
  mark(p, s, mk++, nullptr);

  // 1. SVD clutter filter: Gram -> FP64 Jacobi -> W = (I - V V^T) D_band
  BandArgs ba{};
  if (d.clutter_rank > 0) {
    if (cov_tc)
      HF_TRY(launch_covariance_tc(fr, d.input_dtype, T, p->P, nwin, p->cov_ws, p->gram, p->status, s));
    else
      HF_TRY(launch_covariance(fr, d.input_dtype, T, p->P, nwin, p->cov_ws, p->gram, s));
    mark(p, s, mk++, "covariance");
    HF_TRY(launch_jacobi(p->gram, p->evecs, p->evals, p->info, T, nwin, s));
    HF_TRY(launch_band_matrix(p->evecs, nwin, T, d.clutter_rank, d.z_begin, d.z_end, p->wmat, s));
    mark(p, s, mk++, "eigen_filter");
    ba.wmat        = p->wmat;
    ba.wmat_stride = (int64_t)T * p->nz;
  } else {
    ba.wmat        = p->wmat_plain;
    ba.wmat_stride = 0;
  }
  if (rows_tc) {
    // chosen form: tensor-core band DFT + lens + row FFT in one pass, then columns + moments
    BandRowsArgs br{};
    br.ring        = fr;
    br.T           = T;
    br.H           = d.height;
    br.W           = d.width;
    br.nz          = p->nz;
    br.wmat        = ba.wmat;
    br.wmat_stride = ba.wmat_stride;
    br.lens        = p->lens;
    br.out         = p->band;
    br.out_win     = (int64_t)p->nz * p->P;
    br.out_plane   = p->P;
    br.out_row     = d.width;
    br.nwin        = nwin;
    br.shift       = 2048.f;
    br.status      = p->status;
    HF_CUDA(cudaPeekAtLastError());
    HF_TRY(launch_band_rows_tc(br, d.input_dtype, s));
    mark(p, s, mk++, "band_dft_rows");
    ColPass cp{};
    cp.in        = p->band;
    cp.in_win    = br.out_win;
    cp.in_plane  = p->P;
    cp.in_row    = d.width;
    cp.H         = d.height;
    cp.W         = d.width;
    cp.nplanes   = p->nz;
    cp.out       = out;
    cp.out_win   = (int64_t)p->nmom * p->OH * p->OW;
    cp.out_plane = (int64_t)p->OH * p->OW;
    cp.out_row   = p->OW;
    cp.out_col   = 1;
    HF_TRY(launch_col_pass(cp, COL_MOMENTS, &p->mom, nwin, s));
    mark(p, s, mk++, "fft_cols_moments");
    return finish_exec(p);
  }
  // 2. band DFT (+ lens for Fresnel) -> band planes [nwin][nz][H][W]
  ba.ring      = fr;
  ba.T         = T;
  ba.P         = p->P;
  ba.H         = d.height;
  ba.W         = d.width;
  ba.nz        = p->nz;
  ba.lens      = d.propagation == HF_PROP_FRESNEL ? p->lens : nullptr;
  ba.out       = p->band;
  ba.OH        = d.height;
  ba.OW        = d.width;
  ba.oy        = 0;
  ba.ox        = 0;
  ba.out_plane = p->P;
  ba.out_win   = (int64_t)p->nz * p->P;
  ba.scale     = 1.0f;
  HF_TRY(launch_band_dft(ba, d.input_dtype, nwin, s));
  mark(p, s, mk++, "band_dft");

  const int64_t oplane = (int64_t)p->OH * p->OW;
  const int64_t owin   = (int64_t)p->nmom * oplane;
  if (d.propagation == HF_PROP_NONE) {
    MomentWeights mw;
    memcpy(mw.w1, p->mom.w1, sizeof(mw.w1));
    memcpy(mw.w2, p->mom.w2, sizeof(mw.w2));
    for (int w = 0; w < nwin; ++w)
      HF_TRY(launch_band_moments(p->band + w * ba.out_win, HF_CF32, p->nz, p->P, mw, d.moment_mask,
                                 out + w * owin, s));
    mark(p, s, mk++, "moments");
    return finish_exec(p);
  }

  if (d.propagation == HF_PROP_FRESNEL) {
    RowPass rp{};
    rp.in = p->band;
    rp.in_real = 0;
    rp.in_win = ba.out_win;
    rp.in_plane = p->P;
    rp.in_row = d.width;
    rp.in_col = 1;
    rp.IH = d.height;
    rp.IW = d.width;
    rp.H = d.height;
    rp.N = d.width;
    rp.nplanes = p->nz;
    rp.pre = nullptr;
    rp.inverse = 0;
    rp.out = p->fast ? p->band : p->band2;
    rp.out_win = ba.out_win;
    rp.out_plane = p->P;
    rp.out_row = d.width;
    HF_TRY(launch_row_pass(rp, nwin, s));
    mark(p, s, mk++, "fft_rows");
    ColPass cp{};
    cp.in = rp.out;
    cp.in_win = ba.out_win;
    cp.in_plane = p->P;
    cp.in_row = d.width;
    cp.H = d.height;
    cp.W = d.width;
    cp.nplanes = p->nz;
    cp.inverse = 0;
    if (p->fast) {
      cp.out = out;
      cp.out_win = owin;
      cp.out_plane = oplane;
      cp.out_row = p->OW;
      cp.out_col = 1;
      HF_TRY(launch_col_pass(cp, COL_MOMENTS, &p->mom, nwin, s));
      mark(p, s, mk++, "fft_cols_moments");
      return finish_exec(p);
    }
    // general sizes: complex column DFT back into `band`, then the moment reduction
    cp.out = p->band;
    cp.out_win = ba.out_win;
    cp.out_plane = p->P;
    cp.out_row = d.width;
    cp.out_col = 1;
    HF_TRY(launch_col_pass(cp, COL_COMPLEX, nullptr, nwin, s));
    MomentWeights mw;
    memcpy(mw.w1, p->mom.w1, sizeof(mw.w1));
    memcpy(mw.w2, p->mom.w2, sizeof(mw.w2));
    for (int w = 0; w < nwin; ++w) {
      if (d.fftshift)
        return fail(HF_ERR_UNSUPPORTED, "fftshift needs four-step frame sizes");
      HF_TRY(launch_band_moments(p->band + w * ba.out_win, HF_CF32, p->nz, p->P, mw,
                                 d.moment_mask, out + w * owin, s));
    }
    mark(p, s, mk++, "fft_cols_moments");
    return finish_exec(p);
  }

  // angular spectrum: rows forward (with placement) -> columns fwd x TF inv -> rows inverse + moments
  RowPass rp{};
  rp.in = p->band;
  rp.in_real = 0;
  rp.in_win = ba.out_win;
  rp.in_plane = p->P;
  rp.in_row = d.width;
  rp.in_col = 1;
  rp.IH = d.height;
  rp.IW = d.width;
  rp.oy = (p->OH - d.height) / 2;
  rp.ox = (p->OW - d.width) / 2;
  rp.H = p->OH;
  rp.N = p->OW;
  rp.nplanes = p->nz;
  rp.inverse = 0;
  rp.out = p->band2;
  rp.out_win = (int64_t)p->nz * oplane;
  rp.out_plane = oplane;
  rp.out_row = p->OW;
  HF_TRY(launch_row_pass(rp, nwin, s));
  mark(p, s, mk++, "fft_rows");
  ColPass cp{};
  cp.in = p->band2;
  cp.in_win = rp.out_win;
  cp.in_plane = oplane;
  cp.in_row = p->OW;
  cp.H = p->OH;
  cp.W = p->OW;
  cp.nplanes = p->nz;
  cp.out = p->band2;
  cp.out_win = rp.out_win;
  cp.out_plane = oplane;
  cp.out_row = p->OW;
  cp.out_col = 1;
  cp.tf = p->tf;
  cp.inverse = 0;
  HF_TRY(launch_col_pass(cp, COL_TF_SANDWICH, nullptr, nwin, s));
  mark(p, s, mk++, "fft_cols_tf");
  ColPass rm = cp;
  rm.out = out;
  rm.out_win = owin;
  rm.out_plane = oplane;
  rm.out_row = p->OW;
  rm.inverse = 1;
  HF_TRY(launch_row_moments(rm, p->mom, nwin, s));
  mark(p, s, mk++, "fft_rows_moments");
  return finish_exec(p);
}

int hf_plan_timing(hf_plan *p, int enable) {
  clear_error();
  HF_CHECK_ARG(p != nullptr, "hf_plan_timing: null plan");
  if (enable) {
    for (int i = 0; i < hf_plan::kSets; ++i)
      for (int k = 0; k < hf_plan::kMarks; ++k)
        if (!p->ev[i][k])
          HF_CUDA(cudaEventCreate(&p->ev[i][k]));
  }
  p->timing = enable != 0;
  p->nexec  = 0;
  return HF_OK;
}

int hf_plan_stage_times(hf_plan *p, float *ms, const char **names, int *nstages, int *nexec) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && ms != nullptr && nstages != nullptr, "hf_plan_stage_times: null argument");
  const int ns = p->nstages;
  for (int k = 0; k < HF_MAX_STAGES; ++k)
    ms[k] = 0.f;
  for (int i = 0; i < p->nexec; ++i) {
    for (int k = 0; k + 1 < p->marks[i] && k < ns; ++k) {
      float t = 0.f;
      cudaError_t e = cudaEventElapsedTime(&t, p->ev[i][k], p->ev[i][k + 1]);
      if (e == cudaErrorNotReady)
        return fail(HF_ERR_STATE, "hf_plan_stage_times: synchronise the stream first");
      HF_CUDA(e);
      ms[k] += t;
    }
  }
  if (names)
    for (int k = 0; k < ns; ++k)
      names[k] = p->stage_name[k];
  *nstages = ns;
  if (nexec)
    *nexec = p->nexec;
  return HF_OK;
}

int hf_plan_status(hf_plan *p, int *status, int reset) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && status != nullptr, "hf_plan_status: null argument");
  HF_CUDA(cudaDeviceSynchronize());
  HF_CUDA(cudaMemcpy(status, p->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (reset)
    HF_CUDA(cudaMemset(p->status, 0, sizeof(int)));
  return HF_OK;
}

int hf_pipeline_inspect(hf_plan *p, int w, double *gram, void *wmat, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && w >= 0 && w < p->d.max_batch, "hf_pipeline_inspect: bad window");
  const int T = p->d.frames;
  if (gram) {
    HF_CHECK_ARG(p->gram != nullptr, "hf_pipeline_inspect: plan has no clutter filter");
    HF_CUDA(cudaMemcpyAsync(gram, p->gram + (int64_t)w * T * T, sizeof(double) * T * T,
                            cudaMemcpyDeviceToDevice, s));
  }
  if (wmat) {
    const float2 *src = p->wmat ? p->wmat + (int64_t)w * T * p->nz : p->wmat_plain;
    HF_CUDA(cudaMemcpyAsync(wmat, src, sizeof(float2) * T * p->nz, cudaMemcpyDeviceToDevice, s));
  }
  return HF_OK;
}

// ================================================================================================
// Stage entry points
// ================================================================================================
int hf_unpack12(const uint8_t *packed, void *out, int out_dtype, int64_t npix, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(npix == 0 || (packed != nullptr && out != nullptr), "hf_unpack12: null pointer");
  return launch_unpack12(packed, out, out_dtype, npix, s);
}

int hf_pack12(const uint16_t *in, uint8_t *packed, int64_t npix, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(npix == 0 || (in != nullptr && packed != nullptr), "hf_pack12: null pointer");
  return launch_pack12(in, packed, npix, s);
}

int hf_convert(const void *in, int in_dtype, void *out, int out_dtype, int strategy, int64_t n,
               void *minmax_ws, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(n >= 0, "hf_convert: negative size");
  HF_CHECK_ARG(n == 0 || (in != nullptr && out != nullptr), "hf_convert: null pointer");
  return launch_convert(in, in_dtype, out, out_dtype, strategy, n, minmax_ws, s);
}

int hf_temporal_dft(const void *in, int in_dtype, int64_t batch, int T, int64_t P, int z0, int z1,
                    int norm, void *out, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(in != nullptr && out != nullptr, "hf_temporal_dft: null pointer");
  HF_CHECK_ARG(batch >= 1 && T >= 1 && P >= 1, "hf_temporal_dft: empty problem");
  HF_CHECK_ARG(z0 >= 0 && z1 > z0 && z1 <= T, "hf_temporal_dft: bins must satisfy 0 <= z0 < z1 <= T");
  HF_CHECK_ARG(real_fmt(in_dtype) || in_dtype == HF_CF32, "hf_temporal_dft: unsupported dtype");
  HF_CHECK_ARG(in_dtype != HF_MONO12P || P % 2 == 0, "hf_temporal_dft: packed frames need even P");
  HF_CHECK_ARG(norm >= HF_NORM_BACKWARD && norm <= HF_NORM_ORTHO, "hf_temporal_dft: bad norm");
  HF_CHECK_ARG(batch <= 65535, "hf_temporal_dft: batch too large");
  BandArgs a{};
  a.ring        = FrameRing{reinterpret_cast<const uint8_t *>(in), batch * T, 0, T,
                     frame_bytes_of(in_dtype, P)};
  a.T           = T;
  a.P           = P;
  a.H           = 1;
  a.W           = (int)P;
  a.nz          = z1 - z0;
  a.wmat        = nullptr;
  a.z0          = z0;
  a.wmat_stride = 0;
  a.lens        = nullptr;
  a.out         = reinterpret_cast<float2 *>(out);
  a.OH          = 1;
  a.OW          = (int)P;
  a.out_plane   = P;
  a.out_win     = (int64_t)(z1 - z0) * P;
  a.scale       = norm_scale(norm, T);
  HF_CHECK_ARG(P <= INT32_MAX, "hf_temporal_dft: frame too large");
  return launch_band_dft(a, in_dtype, (int)batch, s);
}

size_t hf_covariance_workspace_bytes(int T, int64_t P) {
  if (T <= 0 || P <= 0)
    return 0;
  return cov_workspace_bytes(T, P, 1);
}

int hf_covariance(const void *in, int in_dtype, int64_t batch, int T, int64_t P, double *gram,
                  void *ws, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(in != nullptr && gram != nullptr, "hf_covariance: null pointer");
  HF_CHECK_ARG(batch >= 1 && batch <= 65535 && T >= 1 && P >= 1, "hf_covariance: bad extents");
  HF_CHECK_ARG(real_fmt(in_dtype), "hf_covariance: unsupported dtype");
  HF_CHECK_ARG(in_dtype != HF_MONO12P || P % 2 == 0, "hf_covariance: packed frames need even P");
  FrameRing fr{reinterpret_cast<const uint8_t *>(in), batch * T, 0, T, frame_bytes_of(in_dtype, P)};
  const bool tiled = (T == 32 || T == 64 || T == 128) && P % 8 == 0 && fr.frame_bytes % 4 == 0;
  if (tiled)
    HF_CHECK_ARG(ws != nullptr, "hf_covariance: workspace required");
  return launch_covariance(fr, in_dtype, T, P, (int)batch, ws, gram, s);
}

int hf_eigh_jacobi_f64(const double *a, double *evecs, double *evals, int *info, int n,
                       int64_t batch, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(a != nullptr && evecs != nullptr && evals != nullptr, "hf_eigh_jacobi_f64: null pointer");
  return launch_jacobi(a, evecs, evals, info, n, batch, s);
}

int hf_pca_project(const float *in, int64_t batch, int T, int64_t P, const double *evecs,
                   int begin, int end, float *out, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(in != nullptr && evecs != nullptr && out != nullptr, "hf_pca_project: null pointer");
  HF_CHECK_ARG(batch >= 1 && batch <= 65535 && T >= 1 && P >= 1, "hf_pca_project: bad extents");
  return launch_pca_project(in, batch, T, P, evecs, begin, end, out, s);
}

int hf_band_matrix(const double *evecs, int64_t batch, int T, int rank, int z0, int z1, void *wmat,
                   hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(wmat != nullptr && (rank == 0 || evecs != nullptr), "hf_band_matrix: null pointer");
  HF_CHECK_ARG(batch >= 1 && batch <= 65535, "hf_band_matrix: bad batch");
  return launch_band_matrix(evecs, batch, T, rank, z0, z1, reinterpret_cast<float2 *>(wmat), s);
}

int hf_mean_axis(const void *in, int in_dtype, int64_t outer, int64_t n, int64_t inner, void *out,
                 hf_stream_t s) {
  clear_error();
  return launch_mean_axis(in, in_dtype, outer, n, inner, out, false, s);
}

int hf_mean_abs_axis(const void *in, int in_dtype, int64_t outer, int64_t n, int64_t inner,
                     float *out, hf_stream_t s) {
  clear_error();
  return launch_mean_axis(in, in_dtype, outer, n, inner, out, true, s);
}

int hf_band_moments(const void *planes, int in_dtype, int nz, int64_t P, const float *freqs,
                    int moment_mask, float *out, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(planes != nullptr && out != nullptr && freqs != nullptr, "hf_band_moments: null pointer");
  HF_CHECK_ARG(nz >= 1 && nz <= kMaxMomentBands, "hf_band_moments: nz must be in [1, 64]");
  MomentWeights w{};
  for (int k = 0; k < nz; ++k) {
    w.w1[k] = freqs[k];
    w.w2[k] = freqs[k] * freqs[k];
  }
  return launch_band_moments(planes, in_dtype, nz, P, w, moment_mask, out, s);
}

} // extern "C"

// ================================================================================================
// Fresnel node plan
// ================================================================================================
struct hf_fresnel_plan {
  int64_t batch = 0;
  int     H = 0, W = 0, in_dtype = 0;
  float   lambda = 0, dx = 0, z = 0;
  int     magnitude = 0, skip_phase = 1;
  float2 *lens = nullptr, *scratch = nullptr;
  size_t  bytes = 0;
};

extern "C" {

int hf_fresnel_plan_create(int64_t batch, int H, int W, int in_dtype, float lambda, float dx,
                           float z, int output_magnitude, int skip_phase_shift,
                           hf_fresnel_plan **plan, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(plan != nullptr, "hf_fresnel_plan_create: null plan pointer");
  *plan = nullptr;
  HF_CHECK_ARG(batch >= 1 && batch <= 65535 && H >= 1 && W >= 1, "FresnelDiffraction: bad extents");
  HF_CHECK_ARG(in_dtype == HF_F32 || in_dtype == HF_CF32, "FresnelDiffraction: input must be F32 or CF32");
  HF_CHECK_ARG(lambda > 0.f && dx > 0.f, "FresnelDiffraction: lambda and dx must be positive");
  auto *p = new (std::nothrow) hf_fresnel_plan();
  if (!p)
    return fail(HF_ERR_NOMEM, "FresnelDiffraction: host allocation failed");
  p->batch = batch, p->H = H, p->W = W, p->in_dtype = in_dtype;
  p->lambda = lambda, p->dx = dx, p->z = z;
  p->magnitude = output_magnitude, p->skip_phase = skip_phase_shift;
  int rc = dev_alloc(&p->lens, (size_t)H * W, p->bytes);
  if (rc == HF_OK)
    rc = dev_alloc(&p->scratch, (size_t)batch * H * W, p->bytes);
  if (rc == HF_OK)
    rc = launch_fresnel_lens(p->lens, W, H, lambda, z, dx, s);
  if (rc != HF_OK) {
    dev_free(p->lens);
    dev_free(p->scratch);
    delete p;
    return rc;
  }
  *plan = p;
  return HF_OK;
}

int hf_fresnel_plan_set_z(hf_fresnel_plan *p, float z, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(p != nullptr, "hf_fresnel_plan_set_z: null plan");
  p->z = z;
  return launch_fresnel_lens(p->lens, p->W, p->H, p->lambda, z, p->dx, s);
}

int hf_fresnel_exec(hf_fresnel_plan *p, const void *in, int64_t in_batch_stride,
                    int64_t in_row_stride, int64_t in_col_stride, void *out,
                    int64_t out_batch_stride, int64_t out_row_stride, int64_t out_col_stride,
                    hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && in != nullptr && out != nullptr, "hf_fresnel_exec: null argument");
  RowPass rp{};
  rp.in       = in;
  rp.in_real  = p->in_dtype == HF_F32;
  rp.in_win   = 0;
  rp.in_plane = in_batch_stride;
  rp.in_row   = in_row_stride;
  rp.in_col   = in_col_stride;
  rp.IH       = p->H;
  rp.IW       = p->W;
  rp.H        = p->H;
  rp.N        = p->W;
  rp.nplanes  = (int)p->batch;
  rp.pre      = p->lens;
  rp.out      = p->scratch;
  rp.out_plane = (int64_t)p->H * p->W;
  rp.out_row  = p->W;
  HF_TRY(launch_row_pass(rp, 1, s));
  ColPass cp{};
  cp.in       = p->scratch;
  cp.in_plane = (int64_t)p->H * p->W;
  cp.in_row   = p->W;
  cp.H        = p->H;
  cp.W        = p->W;
  cp.nplanes  = (int)p->batch;
  cp.out      = out;
  cp.out_plane = out_batch_stride;
  cp.out_row  = out_row_stride;
  cp.out_col  = out_col_stride;
  cp.post     = (!p->magnitude && !p->skip_phase) ? p->lens : nullptr;
  return launch_col_pass(cp, p->magnitude ? COL_MAGNITUDE : COL_COMPLEX, nullptr, 1, s);
}

int hf_fresnel_plan_destroy(hf_fresnel_plan *p) {
  if (!p)
    return HF_OK;
  cudaDeviceSynchronize();
  dev_free(p->lens);
  dev_free(p->scratch);
  delete p;
  return HF_OK;
}

} // extern "C"

// ================================================================================================
// Angular-spectrum node plan
// ================================================================================================
struct hf_as_plan {
  int64_t batch = 0;
  int     H = 0, W = 0, OH = 0, OW = 0, in_dtype = 0;
  bool    fast = false;
  float2 *tf = nullptr, *scratch = nullptr;
  size_t  bytes = 0;
};

extern "C" {

int hf_as_plan_create(int64_t batch, int H, int W, int in_dtype, float lambda, float dx, float z,
                      int pad_w, int pad_h, int use_filter, uint32_t r_inner, uint32_t r_outer,
                      uint32_t s_inner, uint32_t s_outer, hf_as_plan **plan, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(plan != nullptr, "hf_as_plan_create: null plan pointer");
  *plan = nullptr;
  HF_CHECK_ARG(batch >= 1 && batch <= 65535 && H >= 1 && W >= 1, "AngularSpectrum: bad extents");
  HF_CHECK_ARG(in_dtype == HF_F32 || in_dtype == HF_CF32, "AngularSpectrum: input must be F32 or CF32");
  HF_CHECK_ARG(lambda > 0.f && dx > 0.f, "AngularSpectrum: lambda and dx must be positive");
  int OH = H, OW = W;
  if (pad_w > 0 || pad_h > 0) {
    HF_CHECK_ARG(pad_w >= W && pad_h >= H, "AngularSpectrum: padding must be at least the input size");
    HF_CHECK_ARG((pad_w - W) % 2 == 0 && (pad_h - H) % 2 == 0, "AngularSpectrum: padding must be even");
    OH = pad_h, OW = pad_w;
  }
  auto *p = new (std::nothrow) hf_as_plan();
  if (!p)
    return fail(HF_ERR_NOMEM, "AngularSpectrum: host allocation failed");
  p->batch = batch, p->H = H, p->W = W, p->OH = OH, p->OW = OW, p->in_dtype = in_dtype;
  p->fast  = fft_fast_length(OH) && fft_fast_length(OW) && OH <= 1024;
  int rc = dev_alloc(&p->tf, (size_t)OH * OW, p->bytes);
  if (rc == HF_OK && !p->fast)
    rc = dev_alloc(&p->scratch, (size_t)batch * OH * OW, p->bytes);
  if (rc == HF_OK) {
    AsFilter f{r_inner, r_outer, s_inner, s_outer};
    rc = launch_as_tf(p->tf, OW, OH, lambda, z, dx, use_filter, f, s);
  }
  if (rc != HF_OK) {
    dev_free(p->tf);
    dev_free(p->scratch);
    delete p;
    return rc;
  }
  *plan = p;
  return HF_OK;
}

int hf_as_exec(hf_as_plan *p, const void *in, void *out, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && in != nullptr && out != nullptr, "hf_as_exec: null argument");
  const bool padded = p->OH != p->H || p->OW != p->W;
  HF_CHECK_ARG(in != out || (!padded && p->in_dtype == HF_CF32),
               "hf_as_exec: in-place needs complex input without padding");
  const int64_t oplane = (int64_t)p->OH * p->OW;
  RowPass rp{};
  rp.in       = in;
  rp.in_real  = p->in_dtype == HF_F32;
  rp.in_plane = (int64_t)p->H * p->W;
  rp.in_row   = p->W;
  rp.in_col   = 1;
  rp.IH       = p->H;
  rp.IW       = p->W;
  rp.oy       = (p->OH - p->H) / 2;
  rp.ox       = (p->OW - p->W) / 2;
  rp.H        = p->OH;
  rp.N        = p->OW;
  rp.nplanes  = (int)p->batch;
  rp.out_plane = oplane;
  rp.out_row  = p->OW;
  ColPass cp{};
  cp.in_plane = oplane;
  cp.in_row   = p->OW;
  cp.H        = p->OH;
  cp.W        = p->OW;
  cp.nplanes  = (int)p->batch;
  cp.out_plane = oplane;
  cp.out_row  = p->OW;
  cp.out_col  = 1;
  float2 *o = reinterpret_cast<float2 *>(out);
  if (p->fast) {
    rp.out = o; // a warp reads its whole row before writing it back, so in == out is safe
    HF_TRY(launch_row_pass(rp, 1, s));
    cp.in  = o;
    cp.out = o;
    cp.tf  = p->tf;
    HF_TRY(launch_col_pass(cp, COL_TF_SANDWICH, nullptr, 1, s));
    RowPass ri{};
    ri.in = o, ri.in_real = 0, ri.in_plane = oplane, ri.in_row = p->OW, ri.in_col = 1;
    ri.IH = p->OH, ri.IW = p->OW, ri.H = p->OH, ri.N = p->OW, ri.nplanes = (int)p->batch;
    ri.out = o, ri.out_plane = oplane, ri.out_row = p->OW, ri.inverse = 1;
    return launch_row_pass(ri, 1, s);
  }
  // general sizes: direct DFTs through the scratch plane
  rp.out = p->scratch;
  HF_TRY(launch_row_pass(rp, 1, s));
  cp.in   = p->scratch;
  cp.out  = o;
  cp.post = p->tf;
  HF_TRY(launch_col_pass(cp, COL_COMPLEX, nullptr, 1, s));
  cp.in      = o;
  cp.out     = p->scratch;
  cp.post    = nullptr;
  cp.inverse = 1;
  HF_TRY(launch_col_pass(cp, COL_COMPLEX, nullptr, 1, s));
  RowPass ri{};
  ri.in = p->scratch, ri.in_real = 0, ri.in_plane = oplane, ri.in_row = p->OW, ri.in_col = 1;
  ri.IH = p->OH, ri.IW = p->OW, ri.H = p->OH, ri.N = p->OW, ri.nplanes = (int)p->batch;
  ri.out = o, ri.out_plane = oplane, ri.out_row = p->OW, ri.inverse = 1;
  return launch_row_pass(ri, 1, s);
}

int hf_as_plan_destroy(hf_as_plan *p) {
  if (!p)
    return HF_OK;
  cudaDeviceSynchronize();
  dev_free(p->tf);
  dev_free(p->scratch);
  delete p;
  return HF_OK;
}

} // extern "C"

// ================================================================================================
// Camera stream: device-resident frame ring + window cursor bound to a plan
// ================================================================================================
struct hf_stream {
  hf_plan *plan        = nullptr;
  uint8_t *ring        = nullptr;
  int64_t  ring_frames = 0;
  int64_t  pushed      = 0; // frames appended since creation
  int64_t  next_win    = 0; // index of the next window to reconstruct
  float   *dev_out     = nullptr; // staging for host outputs [max_batch][nmom][OH][OW]
  size_t   bytes       = 0;
};

extern "C" {

int hf_stream_create(hf_plan *plan, int64_t ring_frames, hf_stream **out) {
  clear_error();
  HF_CHECK_ARG(plan != nullptr && out != nullptr, "hf_stream_create: null argument");
  *out = nullptr;
  const int64_t need = plan->d.frames + (int64_t)(plan->d.max_batch - 1) * plan->d.hop;
  HF_CHECK_ARG(ring_frames >= need, "hf_stream_create: ring must hold max_batch overlapping windows");
  auto *st = new (std::nothrow) hf_stream();
  if (!st)
    return fail(HF_ERR_NOMEM, "hf_stream_create: host allocation failed");
  st->plan        = plan;
  st->ring_frames = ring_frames;
  int rc = dev_alloc(&st->ring, (size_t)(ring_frames * plan->frame_bytes), st->bytes);
  if (rc == HF_OK)
    rc = dev_alloc(&st->dev_out, (size_t)plan->d.max_batch * plan->nmom * plan->OH * plan->OW, st->bytes);
  if (rc != HF_OK) {
    dev_free(st->ring);
    dev_free(st->dev_out);
    delete st;
    return rc;
  }
  *out = st;
  return HF_OK;
}

int hf_stream_destroy(hf_stream *st) {
  if (!st)
    return HF_OK;
  cudaDeviceSynchronize();
  dev_free(st->ring);
  dev_free(st->dev_out);
  delete st;
  return HF_OK;
}

int64_t hf_stream_ready(const hf_stream *st) {
  if (!st)
    return 0;
  const hf_desc &d = st->plan->d;
  if (st->pushed < d.frames)
    return 0;
  const int64_t complete = (st->pushed - d.frames) / d.hop + 1;
  return complete - st->next_win;
}

int hf_stream_push(hf_stream *st, const void *frames, int64_t nframes, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(st != nullptr && (frames != nullptr || nframes == 0) && nframes >= 0,
               "hf_stream_push: bad argument");
  const hf_desc &d     = st->plan->d;
  const int64_t  keep0 = st->next_win * d.hop; // first frame still needed
  HF_CHECK_ARG(st->pushed + nframes - keep0 <= st->ring_frames,
               "hf_stream_push: ring overrun (process ready windows first)");
  const int64_t fb  = st->plan->frame_bytes;
  const auto   *src = reinterpret_cast<const uint8_t *>(frames);
  int64_t       done = 0;
  while (done < nframes) {
    const int64_t slot = (st->pushed + done) % st->ring_frames;
    const int64_t n    = std::min(nframes - done, st->ring_frames - slot);
    HF_CUDA(cudaMemcpyAsync(st->ring + slot * fb, src + done * fb, (size_t)(n * fb), cudaMemcpyDefault, s));
    done += n;
  }
  st->pushed += nframes;
  return HF_OK;
}

int hf_stream_process(hf_stream *st, int max_windows, float *out, int out_is_host, int *nwin,
                      hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(st != nullptr && out != nullptr, "hf_stream_process: null argument");
  const int64_t ready = hf_stream_ready(st);
  const int     n     = (int)std::min<int64_t>({ready, (int64_t)max_windows, (int64_t)st->plan->d.max_batch});
  if (nwin)
    *nwin = n;
  if (n <= 0)
    return HF_OK;
  float *dst = out_is_host ? st->dev_out : out;
  HF_TRY(hf_pipeline_exec(st->plan, st->ring, st->ring_frames,
                          (st->next_win * st->plan->d.hop) % st->ring_frames, n, dst, s));
  if (out_is_host) {
    const size_t bytes = (size_t)n * st->plan->nmom * st->plan->OH * st->plan->OW * sizeof(float);
    HF_CUDA(cudaMemcpyAsync(out, st->dev_out, bytes, cudaMemcpyDeviceToHost, s));
  }
  st->next_win += n;
  return HF_OK;
}

} // extern "C"
