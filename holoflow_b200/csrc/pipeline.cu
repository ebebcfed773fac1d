// The fused per-window reconstruction (hf_plan / hf_pipeline_exec) and camera streams
// (hf_stream_*): the composition of the stage kernels that replaces the reference graph
// GraphBuilder wires for one window (graph_builder.cc:245-305 time-frequency analysis, 522-566
// propagation, 604-631 moments), plus the device-resident frame ring that replaces BatchQueue
// (batch_queue.cc:92-174).
//
// A window goes through three phases:
//   covariance  Gram matrix of the window's frames               (bandwidth-bound, whole GPU)
//   eigen       FP64 Jacobi + filter/DFT matrix W                (latency-bound, one CTA/window)
//   propagate   band DFT (+ lens) -> row FFT -> column FFT + |.| + moments
// hf_pipeline_exec runs them in order on the caller's stream.  A camera stream with frames of
// the next batch already in its ring overlaps the next batch's eigen phase (on a side stream)
// with the current batch's propagation; the per-window W matrices are the stream's device state.
#include <algorithm>
#include <cstring>
#include <new>

#include "host_util.cuh"
#include "k_band.cuh"
#include "k_cols_tma.cuh"
#include "k_fft2d.cuh"
#include "k_misc.cuh"
#include "k_pca.cuh"
#include "k_post.cuh"
#include "k_shack.cuh"
#include "k_tc_band.cuh"
#include "tma_host.cuh"

using namespace hf;

namespace {

// ---- per-stage CUDA-event timing ------------------------------------------------------------
enum Stage {
  ST_COV = 0,
  ST_EIGEN,
  ST_BAND,
  ST_ROWS,
  ST_BAND_ROWS,
  ST_COLS_MOM,
  ST_COLS_TF,
  ST_ROWS_MOM,
  ST_AUTOFOCUS,
  ST_COUNT
};
const char *kStageName[ST_COUNT] = {"covariance",       "eigen_filter", "band_dft",         "fft_rows",
                                    "band_dft_rows",    "fft_cols_moments", "fft_cols_tf", "fft_rows_moments",
                                    "autofocus"};
static_assert(ST_COUNT <= HF_MAX_STAGES, "stage table");

struct StageTimer {
  static constexpr int kRec = 2048;
  bool        on = false;
  int         n = 0, nexec = 0;
  cudaEvent_t b[kRec] = {}, e[kRec] = {};
  int         stage[kRec] = {};
  int begin(cudaStream_t s, int st) {
    if (!on || n >= kRec)
      return -1;
    cudaEventRecord(b[n], s);
    stage[n] = st;
    return n++;
  }
  void end(cudaStream_t s, int rec) {
    if (rec >= 0)
      cudaEventRecord(e[rec], s);
  }
  void destroy() {
    for (int i = 0; i < kRec; ++i) {
      if (b[i])
        cudaEventDestroy(b[i]);
      if (e[i])
        cudaEventDestroy(e[i]);
      b[i] = e[i] = nullptr;
    }
  }
};

// Buffers of one batch's filter state (Gram -> eigenvectors -> W).
struct FilterSet {
  double *gram = nullptr, *evecs = nullptr, *evals = nullptr;
  int    *info = nullptr;
  float2 *wmat = nullptr;
};

} // namespace

struct hf_plan {
  hf_desc    d{};
  int        P = 0, nz = 0, nmom = 0, OH = 0, OW = 0;
  bool       fast = false;
  int64_t    frame_bytes = 0;
  MomentSpec mom{};
  float2    *lens = nullptr, *tf = nullptr, *band = nullptr, *band2 = nullptr;
  float2    *wmat_plain = nullptr;
  FilterSet  set[2];          // [0] for hf_pipeline_exec and stream batches, [1] stream lookahead
  int       *status = nullptr; // device status word: nonzero when a bounded device wait expired
  int       *row_counter = nullptr; // row queue of the persistent band pass
  void      *cov_ws = nullptr;
  bool       cov_tc = false;   // tensor-core Gram matrix (chosen form)
  bool       rows_tc = false;  // tensor-core band DFT fused with lens + row FFT (chosen form)
  bool       raw_tc = false;   // tensor-core band DFT storing raw planes (chosen form, Filter2D or autofocus)
  bool       seg_tc = false;   // tensor-core raw band planes in row segments (chosen form, other shapes)
  bool       cols_tma = false; // TMA-fed column FFT + moments over `band` through band_tmap
  CUtensorMap band_tmap{};
  size_t     bytes = 0;
  StageTimer timer;
  // Filter2D on the band planes before the Fresnel lens (graph_builder.cc:124-126, 568-576)
  bool    filter2d = false;
  float2 *f2d      = nullptr; // [H][W] annulus mask in natural frequency order
  // Shack-Hartmann autofocus on every window's band planes before the lens (graph_builder.cc:139-153)
  hf_autofocus *af       = nullptr;
  // without a sliding average across windows (pp_accumulation <= 1) the windows' measurements are
  // independent: odd windows take a second instance on a side stream, so one window's slopes and
  // fit (small, latency-bound kernels) run beside the next window's sub-aperture transforms
  hf_autofocus *af2      = nullptr;
  cudaStream_t  af_side  = nullptr;
  cudaEvent_t   af_fork = nullptr, af_join = nullptr;
  float2       *lens_af  = nullptr; // [H][W] lens with the window's correction folded in
  float        *af_coeff = nullptr; // [max_batch][9] coefficients of the last exec
  // pp_accumulation > 1: the raw band planes of the last af_delay windows of the sequence (the
  // dual reader's delayed windows), double-buffered so a call can read the old set while it
  // writes the new one, and the sequence position
  int           af_delay = 0;
  float2       *af_hist[2] = {nullptr, nullptr};
  int64_t       af_seq     = 0;
  AllocCtx      alloc{}; // where the buffers came from (a pool + stream, or cudaMalloc)
};

static void plan_free(hf_plan *p) {
  AllocScope scope(p->alloc.pool, p->alloc.stream); // free the way the buffers were allocated
  hf_autofocus_destroy(p->af);
  hf_autofocus_destroy(p->af2);
  p->af = p->af2 = nullptr;
  if (p->af_side)
    cudaStreamDestroy(p->af_side);
  if (p->af_fork)
    cudaEventDestroy(p->af_fork);
  if (p->af_join)
    cudaEventDestroy(p->af_join);
  p->af_side = nullptr, p->af_fork = p->af_join = nullptr;
  dev_free(p->lens_af);
  dev_free(p->af_coeff);
  dev_free(p->af_hist[0]);
  dev_free(p->af_hist[1]);
  dev_free(p->f2d);
  dev_free(p->lens);
  dev_free(p->tf);
  dev_free(p->band);
  dev_free(p->band2);
  dev_free(p->wmat_plain);
  for (auto &fs : p->set) {
    dev_free(fs.gram);
    dev_free(fs.evecs);
    dev_free(fs.evals);
    dev_free(fs.info);
    dev_free(fs.wmat);
  }
  dev_free(p->status);
  dev_free(p->row_counter);
  dev_free(p->cov_ws);
  p->timer.destroy();
}

static int plan_tables(hf_plan *p, cudaStream_t s) {
  const hf_desc &d = p->d;
  if (d.propagation == HF_PROP_FRESNEL)
    HF_TRY(launch_fresnel_lens(p->lens, d.width, d.height, d.lambda, d.z, d.pitch, s));
  if (d.propagation == HF_PROP_ANGULAR_SPECTRUM) {
    AsFilter f{d.r_inner, d.r_outer, d.s_inner, d.s_outer};
    HF_TRY(launch_as_tf(p->tf, p->OW, p->OH, d.lambda, d.z, d.pitch, d.as_filter, f, s));
  }
  if (p->filter2d && p->f2d == nullptr) { // z-independent: built once
    HF_TRY(dev_alloc(&p->f2d, (size_t)p->P, p->bytes));
    HF_TRY(launch_filter2d_table(p->f2d, d.height, d.width, 0, d.r_inner, d.r_outer, d.s_inner, d.s_outer, s));
  }
  return HF_OK;
}

static FrameRing ring_of(const hf_plan *p, const void *ring, int64_t ring_frames, int64_t first) {
  return FrameRing{reinterpret_cast<const uint8_t *>(ring), ring_frames, first % ring_frames, (int64_t)p->d.hop,
                   p->frame_bytes};
}

// ---- phases ----------------------------------------------------------------------------------
static int phase_cov(hf_plan *p, const FrameRing &fr, int nwin, double *gram, cudaStream_t s) {
  const hf_desc &d  = p->d;
  const bool     tc = p->cov_tc && (reinterpret_cast<uintptr_t>(fr.base) & 15) == 0;
  const int      rec = p->timer.begin(s, ST_COV);
  if (tc)
    HF_TRY(launch_covariance_tc(fr, d.input_dtype, d.frames, p->P, nwin, p->cov_ws, gram, p->status, s));
  else
    HF_TRY(launch_covariance(fr, d.input_dtype, d.frames, p->P, nwin, p->cov_ws, gram, s));
  p->timer.end(s, rec);
  return HF_OK;
}

static int phase_eigen(hf_plan *p, const FilterSet &fs, int nwin, cudaStream_t s) {
  const hf_desc &d   = p->d;
  const int      rec = p->timer.begin(s, ST_EIGEN);
  // the filter needs the clutter_rank largest eigenvectors only: tridiagonalisation + multisection +
  // inverse iteration; the full Jacobi solve for ranks beyond that solver's limit
  if (eig_top_supported(d.frames, d.clutter_rank))
    HF_TRY(launch_eig_top(fs.gram, fs.evecs, fs.evals, fs.info, d.frames, d.clutter_rank, nwin, s));
  else
    HF_TRY(launch_jacobi(fs.gram, fs.evecs, fs.evals, fs.info, d.frames, nwin, s));
  HF_TRY(launch_band_matrix(fs.evecs, nwin, d.frames, d.clutter_rank, d.z_begin, d.z_end, fs.wmat, s,
                            d.time_method == HF_TIME_FFT));
  p->timer.end(s, rec);
  return HF_OK;
}

// Column FFT + |.| + moments of the band planes in p->band into `out`.
static int cols_moments(hf_plan *p, int nwin, float *out, cudaStream_t s) {
  const hf_desc &d      = p->d;
  const int64_t  win_px = (int64_t)p->nz * p->P;
  const int64_t  oplane = (int64_t)p->OH * p->OW;
  const int      rec    = p->timer.begin(s, ST_COLS_MOM);
  if (p->cols_tma) {
    ColMomArgs ca{};
    ca.H = d.height, ca.W = d.width, ca.nz = p->nz, ca.rows_per_win = (int64_t)p->nz * d.height;
    ca.out = out, ca.out_win = (int64_t)p->nmom * oplane, ca.out_plane = oplane, ca.out_row = p->OW;
    ca.status = p->status;
    ca.fast   = d.form == HF_FORM_CHOSEN;
    HF_TRY(launch_col_moments_tma(p->band_tmap, ca, p->mom, nwin, s));
  } else {
    ColPass cp{};
    cp.in = p->band, cp.in_win = win_px, cp.in_plane = p->P, cp.in_row = d.width;
    cp.H = d.height, cp.W = d.width, cp.nplanes = p->nz, cp.inverse = 0;
    cp.out = out, cp.out_win = (int64_t)p->nmom * oplane, cp.out_plane = oplane, cp.out_row = p->OW, cp.out_col = 1;
    HF_TRY(launch_col_pass(cp, COL_MOMENTS, &p->mom, nwin, s));
  }
  p->timer.end(s, rec);
  return HF_OK;
}

static int phase_band(hf_plan *p, const FrameRing &fr, int nwin, const float2 *wmat, int64_t wstride, cudaStream_t s,
                      int reserve_sms, bool *lens_fused, int *rec);
static int phase_after_band(hf_plan *p, int nwin, float *out, cudaStream_t s, bool lens_fused, int rec);

// Band DFT with W (per window, or shared when wstride == 0), propagation and moments.
// `reserve_sms` SMs are left to concurrently running work by the persistent tensor-core pass.
static int phase_propagate(hf_plan *p, const FrameRing &fr, int nwin, const float2 *wmat, int64_t wstride,
                           float *out, cudaStream_t s, int reserve_sms) {
  const hf_desc &d      = p->d;
  const int64_t  win_px = (int64_t)p->nz * p->P;
  const bool     rows_tc = p->rows_tc && (reinterpret_cast<uintptr_t>(fr.base) & 15) == 0;

  if (rows_tc) { // chosen form: tensor-core band DFT + lens + row FFT, then columns + moments
    BandRowsArgs br{};
    br.ring = fr, br.T = d.frames, br.H = d.height, br.W = d.width, br.nz = p->nz;
    br.wmat = wmat, br.wmat_stride = wstride, br.lens = p->lens, br.out = p->band;
    br.lambda = d.lambda, br.z = d.z, br.dx = d.pitch;
    br.out_win = win_px, br.out_plane = p->P, br.out_row = d.width, br.nwin = nwin, br.shift = 2048.f;
    br.status = p->status, br.max_ctas = std::max(1, sm_count() - reserve_sms);
    br.row_counter = p->row_counter;
    int rec = p->timer.begin(s, ST_BAND_ROWS);
    HF_TRY(launch_band_rows_tc(br, d.input_dtype, s));
    p->timer.end(s, rec);
    return cols_moments(p, nwin, out, s);
  }

  bool lens_fused = false;
  int  rec        = -1;
  HF_TRY(phase_band(p, fr, nwin, wmat, wstride, s, reserve_sms, &lens_fused, &rec));
  return phase_after_band(p, nwin, out, s, lens_fused, rec);
}

// The band DFT of the paths other than the fused row pass, into p->band.  `lens_fused`: the pass
// multiplied the planes by the Fresnel lens.  `rec` is the band stage's open timer record.
static int phase_band(hf_plan *p, const FrameRing &fr, int nwin, const float2 *wmat, int64_t wstride, cudaStream_t s,
                      int reserve_sms, bool *lens_fused, int *rec) {
  const hf_desc &d      = p->d;
  const int64_t  win_px = (int64_t)p->nz * p->P;
  *rec                  = p->timer.begin(s, ST_BAND);
  const bool aligned16  = (reinterpret_cast<uintptr_t>(fr.base) & 15) == 0;
  *lens_fused           = false;
  if ((p->raw_tc || p->seg_tc) && aligned16) {
    // chosen form, raw planes on the tensor cores: whole rows (T = 64, before Filter2D or the
    // autofocus) or row segments (the other shapes)
    BandRowsArgs br{};
    br.ring = fr, br.T = d.frames, br.H = d.height, br.W = d.width, br.nz = p->nz;
    br.wmat = wmat, br.wmat_stride = wstride, br.lens = nullptr, br.out = p->band, br.raw = 1;
    br.lambda = d.lambda, br.z = d.z, br.dx = d.pitch;
    br.out_win = win_px, br.out_plane = p->P, br.out_row = d.width, br.nwin = nwin, br.shift = 2048.f;
    br.status = p->status, br.max_ctas = std::max(1, sm_count() - reserve_sms);
    br.row_counter = p->row_counter;
    HF_TRY(p->raw_tc ? launch_band_rows_tc(br, d.input_dtype, s) : launch_band_seg_tc(br, d.input_dtype, s));
  } else {
    BandArgs ba{};
    ba.ring = fr, ba.T = d.frames, ba.P = p->P, ba.H = d.height, ba.W = d.width, ba.nz = p->nz;
    ba.wmat = wmat, ba.wmat_stride = wstride, ba.z0 = d.z_begin;
    ba.lens = d.propagation == HF_PROP_FRESNEL && !p->filter2d && !p->af ? p->lens : nullptr;
    ba.out = p->band, ba.OH = d.height, ba.OW = d.width, ba.oy = 0, ba.ox = 0;
    ba.out_plane = p->P, ba.out_win = win_px, ba.scale = 1.0f;
    HF_TRY(launch_band_dft(ba, d.input_dtype, nwin, s));
    *lens_fused = ba.lens != nullptr;
  }
  return HF_OK;
}

// Everything after the band DFT: Filter2D, the autofocus, propagation and moments of the band
// planes in p->band.  `rec`: the band stage's timer record, closed after Filter2D.
static int phase_after_band(hf_plan *p, int nwin, float *out, cudaStream_t s, bool lens_fused, int rec) {
  const hf_desc &d      = p->d;
  const int64_t  win_px = (int64_t)p->nz * p->P;
  const int64_t  oplane = (int64_t)p->OH * p->OW;
  const int64_t  owin   = (int64_t)p->nmom * oplane;
  if (p->filter2d) // band planes -> FFT2 x annulus -> IFFT2, in place, before the lens
    HF_TRY(launch_filter2d(p->f2d, (int64_t)nwin * p->nz, d.height, d.width, 0, p->band, p->band, p->band2, nullptr, s));
  p->timer.end(s, rec);

  if (d.propagation == HF_PROP_NONE) {
    MomentWeights mw;
    memcpy(mw.w1, p->mom.w1, sizeof(mw.w1));
    memcpy(mw.w2, p->mom.w2, sizeof(mw.w2));
    rec = p->timer.begin(s, ST_COLS_MOM);
    for (int w = 0; w < nwin; ++w)
      HF_TRY(launch_band_moments(p->band + w * win_px, HF_CF32, p->nz, p->P, mw, d.moment_mask, out + w * owin, s));
    p->timer.end(s, rec);
    return HF_OK;
  }

  if (d.propagation == HF_PROP_FRESNEL) {
    RowPass rp{};
    rp.in = p->band, rp.in_real = 0, rp.in_win = win_px, rp.in_plane = p->P, rp.in_row = d.width, rp.in_col = 1;
    rp.IH = d.height, rp.IW = d.width, rp.H = d.height, rp.N = d.width, rp.nplanes = p->nz, rp.inverse = 0;
    rp.out = p->fast ? p->band : p->band2, rp.out_win = win_px, rp.out_plane = p->P, rp.out_row = d.width;
    rp.pre = lens_fused ? nullptr : p->lens; // the lens, when the band pass did not fuse it
    int64_t zero_first = 0;                   // leading windows without a delayed window
    if (p->af) {
      // per window: passes 1..n-1 correct the planes in place, the last pass's correction is
      // folded into the lens of the window's row pass (no extra read and write of the planes)
      rec = p->timer.begin(s, ST_AUTOFOCUS);
      const bool two = p->af2 != nullptr && nwin > 1; // odd windows on the second instance
      if (two) {
        HF_CUDA(cudaEventRecord(p->af_fork, s));
        HF_CUDA(cudaStreamWaitEvent(p->af_side, p->af_fork, 0));
      }
      for (int w = 0; w < nwin; ++w) {
        float2            *planes = p->band + w * win_px;
        hf_autofocus      *a      = two && (w & 1) ? p->af2 : p->af;
        const cudaStream_t q      = two && (w & 1) ? p->af_side : s;
        HF_TRY(autofocus_begin(a, q));
        for (int pass = 0; pass < autofocus_passes(a); ++pass) {
          HF_TRY(autofocus_measure(a, planes, q));
          if (pass + 1 < autofocus_passes(a))
            HF_TRY(autofocus_correct(a, planes, planes, q));
        }
        HF_TRY(autofocus_fold_lens(a, p->lens, p->lens_af + (int64_t)w * p->P, q));
        HF_CUDA(cudaMemcpyAsync(p->af_coeff + 9 * w, autofocus_cumulative_coeffs(a), 9 * sizeof(float),
                                cudaMemcpyDeviceToDevice, q));
      }
      if (two) {
        HF_CUDA(cudaEventRecord(p->af_join, p->af_side));
        HF_CUDA(cudaStreamWaitEvent(s, p->af_join, 0));
      }
      p->timer.end(s, rec);
      // Window w's correction applies to window w - dl (dl = 0 without pp_accumulation).  The
      // delayed planes are this batch's raw planes or the kept ones of the previous calls; the
      // kept set for the next call (the sequence's last dl raw windows) is copied first, since
      // the row passes below overwrite the raw planes in place.
      const int  dl   = p->af_delay;
      const auto seqw = [&](int w) { return p->af_seq + w - dl; }; // sequence index of w's delayed window
      if (dl > 0)
        for (int i = 0; i < dl; ++i) { // concatenation (old kept ++ batch), last dl entries
          const int     idx = nwin + i;
          const float2 *src = idx < dl ? p->af_hist[0] + (int64_t)idx * win_px : p->band + (int64_t)(idx - dl) * win_px;
          HF_CUDA(cudaMemcpyAsync(p->af_hist[1] + (int64_t)i * win_px, src, (size_t)win_px * sizeof(float2),
                                  cudaMemcpyDeviceToDevice, s));
        }
      rec = p->timer.begin(s, ST_ROWS);
      // one row pass per window, each with its own lens; in decreasing order, so that the raw
      // planes a later pass reads as its delayed window (w - dl < w) are not yet overwritten
      for (int w = nwin - 1; w >= 0; --w) {
        if (seqw(w) < 0)
          continue; // no delayed window yet: the images of w are zero (set below)
        RowPass rw = rp;
        rw.in      = w >= dl ? p->band + (int64_t)(w - dl) * win_px : p->af_hist[0] + (int64_t)w * win_px;
        rw.out     = rp.out + w * win_px;
        rw.pre     = p->lens_af + (int64_t)w * p->P;
        HF_TRY(launch_row_pass(rw, 1, s));
      }
      p->timer.end(s, rec);
      std::swap(p->af_hist[0], p->af_hist[1]);
      zero_first = std::max<int64_t>(0, std::min<int64_t>(nwin, dl - p->af_seq));
      p->af_seq += nwin;
    } else {
      rec = p->timer.begin(s, ST_ROWS);
      HF_TRY(launch_row_pass(rp, nwin, s));
      p->timer.end(s, rec);
    }
    // windows whose delayed window precedes the sequence give zero images (after the moments,
    // which compute every window of the batch)
    const auto zero_leading = [&]() -> int {
      if (zero_first > 0)
        HF_CUDA(cudaMemsetAsync(out, 0, (size_t)zero_first * owin * sizeof(float), s));
      return HF_OK;
    };
    if (p->fast) {
      HF_TRY(cols_moments(p, nwin, out, s));
      return zero_leading();
    }
    ColPass cp{};
    cp.in = rp.out, cp.in_win = win_px, cp.in_plane = p->P, cp.in_row = d.width;
    cp.H = d.height, cp.W = d.width, cp.nplanes = p->nz, cp.inverse = 0;
    rec = p->timer.begin(s, ST_COLS_MOM);
    { // general sizes: complex column DFT back into `band`, then the moment reduction
      HF_CHECK_ARG(!d.fftshift, "fftshift needs four-step frame sizes");
      cp.out = p->band, cp.out_win = win_px, cp.out_plane = p->P, cp.out_row = d.width, cp.out_col = 1;
      HF_TRY(launch_col_pass(cp, COL_COMPLEX, nullptr, nwin, s));
      MomentWeights mw;
      memcpy(mw.w1, p->mom.w1, sizeof(mw.w1));
      memcpy(mw.w2, p->mom.w2, sizeof(mw.w2));
      for (int w = 0; w < nwin; ++w)
        HF_TRY(launch_band_moments(p->band + w * win_px, HF_CF32, p->nz, p->P, mw, d.moment_mask, out + w * owin, s));
    }
    p->timer.end(s, rec);
    return zero_leading();
  }

  // angular spectrum: rows forward (with placement) -> columns fwd x TF inv -> rows inverse + moments
  RowPass rp{};
  rp.in = p->band, rp.in_real = 0, rp.in_win = win_px, rp.in_plane = p->P, rp.in_row = d.width, rp.in_col = 1;
  rp.IH = d.height, rp.IW = d.width, rp.oy = (p->OH - d.height) / 2, rp.ox = (p->OW - d.width) / 2;
  rp.H = p->OH, rp.N = p->OW, rp.nplanes = p->nz, rp.inverse = 0;
  rp.out = p->band2, rp.out_win = (int64_t)p->nz * oplane, rp.out_plane = oplane, rp.out_row = p->OW;
  rec = p->timer.begin(s, ST_ROWS);
  HF_TRY(launch_row_pass(rp, nwin, s));
  p->timer.end(s, rec);
  ColPass cp{};
  cp.in = p->band2, cp.in_win = rp.out_win, cp.in_plane = oplane, cp.in_row = p->OW;
  cp.H = p->OH, cp.W = p->OW, cp.nplanes = p->nz;
  cp.out = p->band2, cp.out_win = rp.out_win, cp.out_plane = oplane, cp.out_row = p->OW, cp.out_col = 1;
  cp.tf = p->tf, cp.inverse = 0;
  rec = p->timer.begin(s, ST_COLS_TF);
  HF_TRY(launch_col_pass(cp, COL_TF_SANDWICH, nullptr, nwin, s));
  p->timer.end(s, rec);
  ColPass rm = cp;
  rm.out = out, rm.out_win = owin, rm.out_plane = oplane, rm.out_row = p->OW, rm.inverse = 1;
  rec = p->timer.begin(s, ST_ROWS_MOM);
  HF_TRY(launch_row_moments(rm, p->mom, nwin, s));
  p->timer.end(s, rec);
  return HF_OK;
}

extern "C" {

int hf_plan_create(const hf_desc *desc, hf_plan **out, hf_stream_t stream) {
  clear_error();
  HF_CHECK_ARG(desc != nullptr && out != nullptr, "hf_plan_create: null argument");
  *out = nullptr;
  HF_CHECK_ARG(alloc_ctx().pool == nullptr || alloc_ctx().stream == stream,
               "hf_plan_create: a pooled plan must be created on its allocation stream");
  const hf_desc &d = *desc;
  HF_CHECK_ARG(d.height > 0 && d.width > 0, "plan: frame size must be positive");
  HF_CHECK_ARG(d.frames >= 2 && d.frames <= 128, "plan: frames per window must be in [2, 128]");
  HF_CHECK_ARG(d.hop >= 1, "plan: hop must be >= 1");
  HF_CHECK_ARG(d.z_begin >= 0 && d.z_end > d.z_begin && d.z_end <= d.frames,
               "plan: band must satisfy 0 <= z_begin < z_end <= frames");
  HF_CHECK_ARG(d.time_method == HF_TIME_RFFT || d.time_method == HF_TIME_FFT, "plan: unknown time method");
  HF_CHECK_ARG((d.z_end - d.z_begin) * (d.time_method == HF_TIME_FFT ? 2 : 1) <= kMaxBands,
               "plan: at most 64 band planes (32 bins for the two-sided method)");
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
  if (d.propagation != HF_PROP_NONE)
    HF_CHECK_ARG(d.lambda > 0.f && d.pitch > 0.f, "plan: wavelength and pitch must be positive");
  const bool padded = d.propagation == HF_PROP_ANGULAR_SPECTRUM && (d.pad_w > 0 || d.pad_h > 0);
  if (padded)
    HF_CHECK_ARG(d.pad_w >= d.width && d.pad_h >= d.height && (d.pad_w - d.width) % 2 == 0 &&
                     (d.pad_h - d.height) % 2 == 0,
                 "plan: padding must be >= the frame and leave even margins");
  const int OH = padded ? d.pad_h : d.height, OW = padded ? d.pad_w : d.width;
  if (d.propagation == HF_PROP_ANGULAR_SPECTRUM && !(fft_fast_length(OH) && fft_fast_length(OW) && OH <= 1024))
    return fail(HF_ERR_UNSUPPORTED, "plan: angular spectrum pipeline needs padded sizes in {64..1536} (rows <= 1024)");

  hf_plan *p = new (std::nothrow) hf_plan();
  if (!p)
    return fail(HF_ERR_NOMEM, "plan: host allocation failed");
  p->alloc       = alloc_ctx();
  p->d           = d;
  p->P           = d.height * d.width;
  p->nz          = (d.z_end - d.z_begin) * (d.time_method == HF_TIME_FFT ? 2 : 1);
  p->nmom        = __builtin_popcount(d.moment_mask);
  p->OH          = OH;
  p->OW          = OW;
  p->frame_bytes = frame_bytes_of(d.input_dtype, p->P);
  p->fast        = fft_fast_length(OH) && fft_fast_length(OW);
  p->filter2d    = d.as_filter != 0 && d.propagation != HF_PROP_ANGULAR_SPECTRUM;
  const bool autofocus = d.autofocus_nb_subaps > 0 && d.autofocus_n_orders > 0;
  p->mom.nz       = p->nz;
  p->mom.mask     = d.moment_mask;
  p->mom.fftshift = d.fftshift;
  p->mom.inv_nz   = 1.0f / (float)p->nz;
  fill_weights(p->mom, d.frames, d.z_begin, p->nz, d.fs > 0.f ? d.fs : 37e3, d.time_method == HF_TIME_FFT);

  const int64_t B  = d.max_batch;
  const int     T  = d.frames;
  int           rc = HF_OK;
  do {
    if (p->filter2d && !(p->fast && d.height <= 1024)) {
      rc = fail(HF_ERR_UNSUPPORTED, "plan: Filter2D needs frame sides in {64..1536} (height <= 1024)");
      break;
    }
    if (autofocus) {
      if (d.propagation == HF_PROP_ANGULAR_SPECTRUM) { // graph_builder.cc:535-537
        rc = fail(HF_ERR_INVALID, "Angular Spectrum is not supported with Shack-Hartmann autofocus");
        break;
      }
      if (d.propagation != HF_PROP_FRESNEL || !p->fast) {
        rc = fail(HF_ERR_UNSUPPORTED, "plan: autofocus needs Fresnel propagation on frame sides in {64..1536}");
        break;
      }
      if (d.autofocus_n_orders > 9) {
        rc = fail(HF_ERR_INVALID, "plan: at most 9 autofocus orders");
        break;
      }
      if (d.autofocus_pp_accumulation < 0) {
        rc = fail(HF_ERR_INVALID, "pp_accumulation must be positive");
        break;
      }
      if (d.autofocus_pp_accumulation > 1 && std::max(1, d.autofocus_n_iter) > 1) { // graph_builder.cc:143-146
        rc = fail(HF_ERR_INVALID, "sliding Shack-Hartmann correction only supports one autofocus iteration");
        break;
      }
      if ((rc = hf_autofocus_create(p->nz, d.height, d.width, d.autofocus_nb_subaps, std::max(1, d.autofocus_n_iter),
                                    d.lambda, d.pitch, d.z,
                                    d.autofocus_roi_radius > 0.f ? d.autofocus_roi_radius : 0.5f,
                                    d.autofocus_keep_outside ? 0 : 1, d.autofocus_orders, d.autofocus_n_orders,
                                    d.autofocus_flatfield_period, stream, &p->af)))
        break;
      if ((rc = dev_alloc(&p->lens_af, (size_t)(B * p->P), p->bytes)) ||
          (rc = dev_alloc(&p->af_coeff, (size_t)(9 * B), p->bytes)))
        break;
      if (d.autofocus_full_pairwise &&
          (rc = hf_autofocus_set_slope_mode(p->af, HF_SHSLOPES_FULL_PAIRWISE, 256,
                                            d.autofocus_roi_radius > 0.f ? d.autofocus_roi_radius : 0.5f,
                                            d.autofocus_keep_outside ? 0 : 1, d.lambda, d.pitch, d.z, stream)))
        break;
      if (d.autofocus_pp_accumulation <= 1 && B > 1) { // the second instance for odd windows
        if ((rc = hf_autofocus_create(p->nz, d.height, d.width, d.autofocus_nb_subaps, std::max(1, d.autofocus_n_iter),
                                      d.lambda, d.pitch, d.z,
                                      d.autofocus_roi_radius > 0.f ? d.autofocus_roi_radius : 0.5f,
                                      d.autofocus_keep_outside ? 0 : 1, d.autofocus_orders, d.autofocus_n_orders,
                                      d.autofocus_flatfield_period, stream, &p->af2)))
          break;
        if (d.autofocus_full_pairwise &&
            (rc = hf_autofocus_set_slope_mode(p->af2, HF_SHSLOPES_FULL_PAIRWISE, 256,
                                              d.autofocus_roi_radius > 0.f ? d.autofocus_roi_radius : 0.5f,
                                              d.autofocus_keep_outside ? 0 : 1, d.lambda, d.pitch, d.z, stream)))
          break;
        if ((rc = cuda_status(cudaStreamCreateWithFlags(&p->af_side, cudaStreamNonBlocking), "autofocus stream")) ||
            (rc = cuda_status(cudaEventCreateWithFlags(&p->af_fork, cudaEventDisableTiming), "autofocus event")) ||
            (rc = cuda_status(cudaEventCreateWithFlags(&p->af_join, cudaEventDisableTiming), "autofocus event")))
          break;
      }
      if (d.autofocus_pp_accumulation > 1) {
        if ((rc = hf_autofocus_set_accumulation(p->af, d.autofocus_pp_accumulation, stream)))
          break;
        p->af_delay = (d.autofocus_pp_accumulation - 1) / 2;
        const size_t hist = (size_t)p->af_delay * p->nz * p->P;
        if (hist && ((rc = dev_alloc(&p->af_hist[0], hist, p->bytes)) || (rc = dev_alloc(&p->af_hist[1], hist, p->bytes))))
          break;
      }
    }
    const int64_t plane = (int64_t)p->P, oplane = (int64_t)OH * OW;
    if ((rc = dev_alloc(&p->band, (size_t)(B * p->nz * plane), p->bytes)))
      break;
    const bool need_band2 = d.propagation == HF_PROP_ANGULAR_SPECTRUM || (d.propagation == HF_PROP_FRESNEL && !p->fast) ||
                            p->filter2d;
    if (need_band2 && (rc = dev_alloc(&p->band2, (size_t)(B * p->nz * oplane), p->bytes)))
      break;
    if (d.propagation == HF_PROP_FRESNEL && (rc = dev_alloc(&p->lens, (size_t)plane, p->bytes)))
      break;
    if (d.propagation == HF_PROP_ANGULAR_SPECTRUM && (rc = dev_alloc(&p->tf, (size_t)oplane, p->bytes)))
      break;
    if (d.clutter_rank > 0) {
      for (auto &fs : p->set)
        if ((rc = dev_alloc(&fs.gram, (size_t)(B * T * T), p->bytes)) ||
            (rc = dev_alloc(&fs.evecs, (size_t)(B * T * T), p->bytes)) ||
            (rc = dev_alloc(&fs.evals, (size_t)(B * T), p->bytes)) || (rc = dev_alloc(&fs.info, (size_t)B, p->bytes)) ||
            (rc = dev_alloc(&fs.wmat, (size_t)(B * T * p->nz), p->bytes)))
          break;
      if (rc)
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
      if ((rc = dev_alloc(&p->wmat_plain, (size_t)T * p->nz, p->bytes)))
        break;
      if ((rc = launch_band_matrix(nullptr, 1, T, 0, d.z_begin, d.z_end, p->wmat_plain, stream,
                                   d.time_method == HF_TIME_FFT)))
        break;
    }
    if ((rc = dev_alloc(&p->status, 1, p->bytes)) || (rc = dev_alloc(&p->row_counter, 1, p->bytes)))
      break;
    if ((rc = cuda_status(cudaMemsetAsync(p->status, 0, sizeof(int), stream), "status reset")))
      break;
    // the tensor-core band pass holds 2 (z1 - z0) real columns per pixel: the one-sided band only
    const bool tc_band = d.form == HF_FORM_CHOSEN && d.propagation == HF_PROP_FRESNEL && p->fast &&
                         d.time_method == HF_TIME_RFFT &&
                         band_rows_tc_supported(d.input_dtype, T, d.width, p->nz, p->frame_bytes);
    p->rows_tc = tc_band && !p->filter2d && !p->af;
    p->raw_tc  = tc_band && (p->filter2d || p->af);
    // every other chosen-form shape the segment pass takes (T = 32 / 128, wide rows, two-sided
    // band, angular spectrum): raw band planes on the tensor cores, the lens in the row pass
    p->seg_tc = d.form == HF_FORM_CHOSEN && !p->rows_tc && !p->raw_tc &&
                band_seg_tc_supported(d.input_dtype, T, d.width, p->nz, p->frame_bytes);
    if (d.propagation == HF_PROP_FRESNEL && p->fast && col_moments_tma_supported(d.height, d.width)) {
      const uint64_t rows = (uint64_t)B * p->nz * d.height;
      if ((rc = make_tmap_2d_f32(&p->band_tmap, p->band, 2 * (uint64_t)d.width, rows, 8 * (uint64_t)d.width,
                                 2 * kColMomCols,
                                 (uint32_t)std::min(d.height, 256))))
        break;
      p->cols_tma = true;
    }
    rc = plan_tables(p, stream);
  } while (0);
  if (rc != HF_OK) {
    const std::string msg = hf_last_error(); // releasing the parts built so far must not erase it
    plan_free(p);
    delete p;
    set_error(msg);
    return rc;
  }
  *out = p;
  return HF_OK;
}

int hf_plan_destroy(hf_plan *p) {
  if (!p)
    return HF_OK;
  // a pooled plan waits for its own stream only (its buffers are freed in that stream's order);
  // otherwise for the device, as cudaFree would
  if (p->alloc.pool)
    cudaStreamSynchronize(p->alloc.stream);
  else
    cudaDeviceSynchronize();
  plan_free(p);
  delete p;
  return HF_OK;
}

int hf_plan_set_z(hf_plan *p, float z, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(p != nullptr, "hf_plan_set_z: null plan");
  p->d.z = z;
  HF_TRY(plan_tables(p, s));
  if (p->af) // the sub-aperture transform's input lens depends on z; the slopes and the fit do not
    HF_TRY(autofocus_set_z(p->af, z, s));
  if (p->af2)
    HF_TRY(autofocus_set_z(p->af2, z, s));
  return HF_OK;
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

int hf_plan_band_pass(const hf_plan *p, int *kind) {
  HF_CHECK_ARG(p != nullptr && kind != nullptr, "hf_plan_band_pass: null argument");
  *kind = p->rows_tc ? HF_BAND_TC_ROWS : p->raw_tc ? HF_BAND_TC_RAW_ROWS : p->seg_tc ? HF_BAND_TC_SEGMENTS : HF_BAND_FP32;
  return HF_OK;
}

int hf_pipeline_exec(hf_plan *p, const void *ring, int64_t ring_frames, int64_t first_frame, int nwin, float *out,
                     hf_stream_t stream) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && ring != nullptr && out != nullptr, "hf_pipeline_exec: null argument");
  HF_CHECK_ARG(nwin >= 1 && nwin <= p->d.max_batch, "hf_pipeline_exec: nwin must be in [1, max_batch]");
  HF_CHECK_ARG(ring_frames >= p->d.frames && first_frame >= 0, "hf_pipeline_exec: the ring must hold at least one window");
  const FrameRing fr = ring_of(p, ring, ring_frames, first_frame);
  if (p->d.clutter_rank > 0) {
    HF_TRY(phase_cov(p, fr, nwin, p->set[0].gram, stream));
    HF_TRY(phase_eigen(p, p->set[0], nwin, stream));
    HF_TRY(phase_propagate(p, fr, nwin, p->set[0].wmat, (int64_t)p->d.frames * p->nz, out, stream, 0));
  } else {
    HF_TRY(phase_propagate(p, fr, nwin, p->wmat_plain, 0, out, stream, 0));
  }
  if (p->timer.on)
    ++p->timer.nexec;
  return HF_OK;
}

int hf_plan_timing(hf_plan *p, int enable) {
  clear_error();
  HF_CHECK_ARG(p != nullptr, "hf_plan_timing: null plan");
  if (enable)
    for (int i = 0; i < StageTimer::kRec; ++i) {
      if (!p->timer.b[i])
        HF_CUDA(cudaEventCreate(&p->timer.b[i]));
      if (!p->timer.e[i])
        HF_CUDA(cudaEventCreate(&p->timer.e[i]));
    }
  p->timer.on    = enable != 0;
  p->timer.n     = 0;
  p->timer.nexec = 0;
  return HF_OK;
}

int hf_plan_autofocus_reset(hf_plan *p, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(p != nullptr, "hf_plan_autofocus_reset: null argument");
  p->af_seq = 0;
  if (p->af)
    HF_TRY(hf_autofocus_reset(p->af, s));
  if (p->af2)
    HF_TRY(hf_autofocus_reset(p->af2, s));
  return HF_OK;
}

int hf_plan_autofocus_coefficients(hf_plan *p, int w, float *coeffs, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && coeffs != nullptr, "hf_plan_autofocus_coefficients: null argument");
  HF_CHECK_ARG(p->af != nullptr, "hf_plan_autofocus_coefficients: the plan has no autofocus");
  HF_CHECK_ARG(w >= 0 && w < p->d.max_batch, "hf_plan_autofocus_coefficients: window out of range");
  HF_CUDA(cudaMemcpyAsync(coeffs, p->af_coeff + 9 * w, (size_t)p->d.autofocus_n_orders * sizeof(float),
                          cudaMemcpyDeviceToDevice, s));
  return HF_OK;
}

int hf_plan_stage_times(hf_plan *p, float *ms, const char **names, int *nstages, int *nexec) {
  clear_error();
  HF_CHECK_ARG(p != nullptr && ms != nullptr && nstages != nullptr, "hf_plan_stage_times: null argument");
  for (int k = 0; k < HF_MAX_STAGES; ++k)
    ms[k] = 0.f;
  for (int i = 0; i < p->timer.n; ++i) {
    float       t = 0.f;
    cudaError_t e = cudaEventElapsedTime(&t, p->timer.b[i], p->timer.e[i]);
    if (e == cudaErrorNotReady)
      return fail(HF_ERR_STATE, "hf_plan_stage_times: synchronise the stream first");
    HF_CUDA(e);
    ms[p->timer.stage[i]] += t;
  }
  if (names)
    for (int k = 0; k < ST_COUNT; ++k)
      names[k] = kStageName[k];
  *nstages = ST_COUNT;
  if (nexec)
    *nexec = p->timer.nexec;
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
    HF_CHECK_ARG(p->set[0].gram != nullptr, "hf_pipeline_inspect: plan has no clutter filter");
    HF_CUDA(cudaMemcpyAsync(gram, p->set[0].gram + (int64_t)w * T * T, sizeof(double) * T * T,
                            cudaMemcpyDeviceToDevice, s));
  }
  if (wmat) {
    const float2 *src = p->set[0].wmat ? p->set[0].wmat + (int64_t)w * T * p->nz : p->wmat_plain;
    HF_CUDA(cudaMemcpyAsync(wmat, src, sizeof(float2) * T * p->nz, cudaMemcpyDeviceToDevice, s));
  }
  return HF_OK;
}

} // extern "C"

// ================================================================================================
// Camera stream: device-resident frame ring + window cursor + lookahead filter state
// ================================================================================================
struct hf_stream {
  hf_plan     *plan        = nullptr;
  uint8_t     *ring        = nullptr;
  int64_t      ring_frames = 0;
  int64_t      pushed      = 0;       // frames appended since creation
  int64_t      next_win    = 0;       // index of the next window to reconstruct
  float       *stage[2]    = {};      // staging for host outputs, 2 x [max_batch][nmom][OH][OW]
  size_t       bytes       = 0;
  cudaStream_t side        = nullptr; // eigen phase of the lookahead batch
  cudaEvent_t  ev_cov      = nullptr; // lookahead Gram matrices written (main stream)
  cudaEvent_t  ev_ready    = nullptr; // lookahead W matrices written (side stream)
  bool         look_valid  = false;   // set[look_set] holds W for windows [look_base, +look_n)
  int64_t      look_base   = 0;
  int          look_n      = 0;
  int          look_set    = 1;

  // Ordering between pushes and processes issued on different CUDA streams: the absolute frame
  // range each recent push wrote and each recent process read, with an event recorded after it.
  static constexpr int kHist = 8;
  struct Rec {
    int64_t     lo = 0, hi = -1;
    cudaEvent_t ev = nullptr;
  };
  Rec     push_rec[kHist];
  Rec     proc_rec[kHist];
  int64_t npush = 0, nproc = 0;

  // Asynchronous host output (out_is_host == 2): the copy of stage[k] runs on `d2h`.
  cudaStream_t d2h            = nullptr;
  cudaEvent_t  ev_out[2]      = {}; // stage[k] written by the compute stream
  cudaEvent_t  ev_d2h[2]      = {}; // stage[k] copied to the host
  bool         d2h_pending[2] = {};
  int          stage_k        = 0;
  int          last_k         = -1;
  AllocCtx     alloc{}; // where ring and staging came from (a pool + stream, or cudaMalloc)
};

namespace {
// Makes `s` wait until every push that wrote frames up to absolute index `need_hi` has landed.
// Pushes of one camera stream are issued in order on one CUDA stream, so the oldest recorded push
// that reaches `need_hi` covers all earlier ones.
int wait_for_pushes(hf_stream *st, int64_t need_hi, cudaStream_t s) {
  const int64_t first = std::max<int64_t>(0, st->npush - hf_stream::kHist);
  for (int64_t i = first; i < st->npush; ++i) {
    const hf_stream::Rec &r = st->push_rec[i % hf_stream::kHist];
    if (r.hi >= need_hi)
      return cuda_status(cudaStreamWaitEvent(s, r.ev, 0), "hf_stream_process: wait for pushed frames");
  }
  return fail(HF_ERR_STATE, "hf_stream_process: frames of the batch were never pushed");
}

// Makes `s` wait until no recorded process still reads a frame in [dlo, dhi] (the frames a push is
// about to overwrite).  Processes are issued in order on one CUDA stream, so waiting for the most
// recent one that started at or below dhi covers all earlier ones; if every recorded process
// starts above dhi but older ones were dropped from the record, the oldest recorded one covers them.
int wait_for_readers(hf_stream *st, int64_t dhi, cudaStream_t s) {
  const int64_t first = std::max<int64_t>(0, st->nproc - hf_stream::kHist);
  for (int64_t i = st->nproc - 1; i >= first; --i) {
    const hf_stream::Rec &r = st->proc_rec[i % hf_stream::kHist];
    if (r.lo <= dhi)
      return cuda_status(cudaStreamWaitEvent(s, r.ev, 0), "hf_stream_push: wait for readers");
  }
  if (first > 0)
    return cuda_status(cudaStreamWaitEvent(s, st->proc_rec[first % hf_stream::kHist].ev, 0),
                       "hf_stream_push: wait for readers");
  return HF_OK;
}
} // namespace

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
  st->alloc       = alloc_ctx();
  const size_t out_elems = (size_t)plan->d.max_batch * plan->nmom * plan->OH * plan->OW;
  int rc = dev_alloc(&st->ring, (size_t)(ring_frames * plan->frame_bytes), st->bytes);
  for (int k = 0; k < 2 && rc == HF_OK; ++k)
    rc = dev_alloc(&st->stage[k], out_elems, st->bytes);
  if (rc == HF_OK)
    rc = cuda_status(cudaStreamCreateWithFlags(&st->side, cudaStreamNonBlocking), "side stream");
  if (rc == HF_OK)
    rc = cuda_status(cudaStreamCreateWithFlags(&st->d2h, cudaStreamNonBlocking), "output copy stream");
  cudaEvent_t *evs[] = {&st->ev_cov, &st->ev_ready, &st->ev_out[0], &st->ev_out[1], &st->ev_d2h[0], &st->ev_d2h[1]};
  for (cudaEvent_t *e : evs)
    if (rc == HF_OK)
      rc = cuda_status(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "stream event");
  for (int i = 0; i < hf_stream::kHist && rc == HF_OK; ++i) {
    rc = cuda_status(cudaEventCreateWithFlags(&st->push_rec[i].ev, cudaEventDisableTiming), "stream event");
    if (rc == HF_OK)
      rc = cuda_status(cudaEventCreateWithFlags(&st->proc_rec[i].ev, cudaEventDisableTiming), "stream event");
  }
  if (rc == HF_OK && plan->af) // a camera stream is a new window sequence
    rc = hf_plan_autofocus_reset(plan, plan->alloc.pool ? plan->alloc.stream : nullptr);
  if (rc != HF_OK) {
    hf_stream_destroy(st);
    return rc;
  }
  *out = st;
  return HF_OK;
}

int hf_stream_destroy(hf_stream *st) {
  if (!st)
    return HF_OK;
  // pooled: wait for this camera stream's own CUDA streams (the caller has synchronised the
  // streams it pushed and processed on) and free in the allocation stream's order
  if (st->alloc.pool) {
    for (cudaStream_t q : {st->side, st->d2h, st->alloc.stream})
      if (q)
        cudaStreamSynchronize(q);
  } else {
    cudaDeviceSynchronize();
  }
  AllocScope scope(st->alloc.pool, st->alloc.stream);
  dev_free(st->ring);
  for (float *&b : st->stage)
    dev_free(b);
  for (cudaStream_t q : {st->side, st->d2h})
    if (q)
      cudaStreamDestroy(q);
  for (cudaEvent_t e : {st->ev_cov, st->ev_ready, st->ev_out[0], st->ev_out[1], st->ev_d2h[0], st->ev_d2h[1]})
    if (e)
      cudaEventDestroy(e);
  for (int i = 0; i < hf_stream::kHist; ++i) {
    if (st->push_rec[i].ev)
      cudaEventDestroy(st->push_rec[i].ev);
    if (st->proc_rec[i].ev)
      cudaEventDestroy(st->proc_rec[i].ev);
  }
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
  HF_CHECK_ARG(st != nullptr && (frames != nullptr || nframes == 0) && nframes >= 0, "hf_stream_push: bad argument");
  const hf_desc &d = st->plan->d;
  // frames still needed: those of the next window to process and of a prepared lookahead batch
  const int64_t keep0 = st->next_win * d.hop;
  HF_CHECK_ARG(st->pushed + nframes - keep0 <= st->ring_frames,
               "hf_stream_push: ring overrun (process ready windows first)");
  if (nframes == 0)
    return HF_OK;
  // the slots about to be written held frames [pushed - R, pushed + n - R): wait for their readers
  const int64_t dhi = st->pushed + nframes - st->ring_frames - 1;
  if (dhi >= 0)
    HF_TRY(wait_for_readers(st, dhi, s));
  const int64_t fb   = st->plan->frame_bytes;
  const auto   *src  = reinterpret_cast<const uint8_t *>(frames);
  int64_t       done = 0;
  while (done < nframes) {
    const int64_t slot = (st->pushed + done) % st->ring_frames;
    const int64_t n    = std::min(nframes - done, st->ring_frames - slot);
    HF_CUDA(cudaMemcpyAsync(st->ring + slot * fb, src + done * fb, (size_t)(n * fb), cudaMemcpyDefault, s));
    done += n;
  }
  hf_stream::Rec &r = st->push_rec[st->npush % hf_stream::kHist];
  r.lo = st->pushed;
  r.hi = st->pushed + nframes - 1;
  HF_CUDA(cudaEventRecord(r.ev, s));
  ++st->npush;
  st->pushed += nframes;
  return HF_OK;
}

int hf_stream_process(hf_stream *st, int max_windows, float *out, int out_is_host, int *nwin, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(st != nullptr && out != nullptr, "hf_stream_process: null argument");
  HF_CHECK_ARG(out_is_host >= 0 && out_is_host <= 2, "hf_stream_process: out_is_host must be 0, 1 or 2");
  hf_plan       *p     = st->plan;
  const hf_desc &d     = p->d;
  const int64_t  ready = hf_stream_ready(st);
  const int n = (int)std::min<int64_t>({ready, (int64_t)max_windows, (int64_t)d.max_batch});
  if (nwin)
    *nwin = n;
  if (n <= 0)
    return HF_OK;
  const int64_t base = st->next_win;
  auto win_ring = [&](int64_t w0) { return ring_of(p, st->ring, st->ring_frames, (w0 * d.hop) % st->ring_frames); };
  const int64_t wstride = (int64_t)d.frames * p->nz;
  // windows of the lookahead batch (their Gram matrices are computed by this call)
  const int n2 = d.clutter_rank == 0 ? 0 : (int)std::min<int64_t>(ready - n, (int64_t)d.max_batch);

  // frames read by this call: windows [base, base + n + n2); wait for the pushes that bring them
  const int64_t read_lo = base * d.hop;
  const int64_t read_hi = (base + n + n2 - 1) * d.hop + d.frames - 1;
  HF_TRY(wait_for_pushes(st, read_hi, s));

  float *dst = out;
  int    k   = -1;
  if (out_is_host) { // stage the images; the staging buffer's previous copy must have finished
    k           = st->stage_k;
    st->stage_k = k ^ 1;
    if (st->d2h_pending[k])
      HF_CUDA(cudaStreamWaitEvent(s, st->ev_d2h[k], 0));
    dst = st->stage[k];
  }

  if (d.clutter_rank == 0) {
    HF_TRY(phase_propagate(p, win_ring(base), n, p->wmat_plain, 0, dst, s, 0));
  } else {
    // 1. W for this batch: prepared by the previous call's lookahead, or computed now
    int cur;
    if (st->look_valid && st->look_base == base && st->look_n == n) {
      cur = st->look_set;
      HF_CUDA(cudaStreamWaitEvent(s, st->ev_ready, 0));
    } else {
      // a stale lookahead (different window range) still owns look_set: let it finish, use the
      // other set, and recompute this batch's filter here
      if (st->look_valid)
        HF_CUDA(cudaStreamWaitEvent(s, st->ev_ready, 0));
      cur = st->look_valid ? st->look_set ^ 1 : 0;
      HF_TRY(phase_cov(p, win_ring(base), n, p->set[cur].gram, s));
      HF_TRY(phase_eigen(p, p->set[cur], n, s));
    }
    st->look_valid = false;
    // 2. lookahead: Gram matrices of the next batch now (whole GPU), its eigen phase on the side
    //    stream concurrently with this batch's propagation
    int reserve = 0;
    if (n2 > 0) {
      const int nxt = cur ^ 1;
      HF_TRY(phase_cov(p, win_ring(base + n), n2, p->set[nxt].gram, s));
      HF_CUDA(cudaEventRecord(st->ev_cov, s));
      HF_CUDA(cudaStreamWaitEvent(st->side, st->ev_cov, 0));
      HF_TRY(phase_eigen(p, p->set[nxt], n2, st->side));
      HF_CUDA(cudaEventRecord(st->ev_ready, st->side));
      st->look_valid = true;
      st->look_base  = base + n;
      st->look_n     = n2;
      st->look_set   = nxt;
      // the full Jacobi solve (ranks beyond the top-r solver) takes ~1 ms per 64 x 64 matrix: keep
      // one SM per lookahead matrix free of the persistent band pass; the top-r solver finishes
      // within the columns pass that follows, so the band pass takes every SM
      reserve = eig_top_supported(d.frames, d.clutter_rank) ? 0 : n2;
    }
    // 3. this batch's propagation
    HF_TRY(phase_propagate(p, win_ring(base), n, p->set[cur].wmat, wstride, dst, s, reserve));
  }
  // every frame read by this call has been consumed once `s` passes this point
  hf_stream::Rec &r = st->proc_rec[st->nproc % hf_stream::kHist];
  r.lo = read_lo;
  r.hi = read_hi;
  HF_CUDA(cudaEventRecord(r.ev, s));
  ++st->nproc;

  const size_t bytes = (size_t)n * p->nmom * p->OH * p->OW * sizeof(float);
  if (out_is_host == 1) { // copy in stream order: the images are on the host once `s` passes here
    HF_CUDA(cudaMemcpyAsync(out, st->stage[k], bytes, cudaMemcpyDeviceToHost, s));
    st->d2h_pending[k] = false;
  } else if (out_is_host == 2) { // copy on the stream's own copy engine queue, overlapping later work
    HF_CUDA(cudaEventRecord(st->ev_out[k], s));
    HF_CUDA(cudaStreamWaitEvent(st->d2h, st->ev_out[k], 0));
    HF_CUDA(cudaMemcpyAsync(out, st->stage[k], bytes, cudaMemcpyDeviceToHost, st->d2h));
    HF_CUDA(cudaEventRecord(st->ev_d2h[k], st->d2h));
    st->d2h_pending[k] = true;
    st->last_k         = k;
  }
  st->next_win += n;
  if (p->timer.on)
    ++p->timer.nexec;
  return HF_OK;
}

int hf_stream_output_wait(hf_stream *st, hf_stream_t s, int host_block) {
  clear_error();
  HF_CHECK_ARG(st != nullptr, "hf_stream_output_wait: null stream");
  if (st->last_k < 0 || !st->d2h_pending[st->last_k])
    return HF_OK;
  if (host_block)
    HF_CUDA(cudaEventSynchronize(st->ev_d2h[st->last_k]));
  else
    HF_CUDA(cudaStreamWaitEvent(s, st->ev_d2h[st->last_k], 0));
  return HF_OK;
}

} // extern "C"

// ---- split form of hf_pipeline_exec for the multi-acquisition executor --------------------------
namespace hf {

int pipeline_front(hf_plan *p, const void *ring, int64_t ring_frames, int64_t first, int nwin, cudaStream_t s) {
  HF_CHECK_ARG(p != nullptr && ring != nullptr, "pipeline front: null argument");
  HF_CHECK_ARG(nwin >= 1 && nwin <= p->d.max_batch, "pipeline front: nwin must be in [1, max_batch]");
  HF_CHECK_ARG(ring_frames >= p->d.frames && first >= 0, "pipeline front: the ring must hold at least one window");
  if (p->d.clutter_rank > 0) {
    const FrameRing fr = ring_of(p, ring, ring_frames, first);
    HF_TRY(phase_cov(p, fr, nwin, p->set[0].gram, s));
    HF_TRY(phase_eigen(p, p->set[0], nwin, s));
  }
  return HF_OK;
}

bool pipeline_seg_eligible(const hf_plan *p, const void *ring) {
  return p != nullptr && p->seg_tc && (reinterpret_cast<uintptr_t>(ring) & 15) == 0;
}

int pipeline_seg_job(hf_plan *p, const void *ring, int64_t ring_frames, int64_t first, int nwin, BandRowsArgs *job) {
  HF_CHECK_ARG(job != nullptr && pipeline_seg_eligible(p, ring), "pipeline segment job: the plan does not take the segment pass");
  HF_CHECK_ARG(nwin >= 1 && nwin <= p->d.max_batch, "pipeline segment job: nwin must be in [1, max_batch]");
  const hf_desc &d = p->d;
  BandRowsArgs   br{};
  br.ring = ring_of(p, ring, ring_frames, first), br.T = d.frames, br.H = d.height, br.W = d.width, br.nz = p->nz;
  br.wmat        = d.clutter_rank > 0 ? p->set[0].wmat : p->wmat_plain;
  br.wmat_stride = d.clutter_rank > 0 ? (int64_t)d.frames * p->nz : 0;
  br.lens = nullptr, br.out = p->band, br.raw = 1;
  br.out_win = (int64_t)p->nz * p->P, br.out_plane = p->P, br.out_row = d.width, br.nwin = nwin, br.shift = 2048.f;
  br.status = p->status, br.row_counter = p->row_counter;
  *job = br;
  return HF_OK;
}

int pipeline_back(hf_plan *p, int nwin, float *out, cudaStream_t s) {
  HF_CHECK_ARG(p != nullptr && out != nullptr, "pipeline back: null argument");
  return phase_after_band(p, nwin, out, s, false, -1);
}

int *plan_status_word(hf_plan *p) { return p ? p->status : nullptr; }

} // namespace hf
