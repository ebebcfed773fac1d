// holoflow_b200 node layer: the Doppler path's compute nodes behind the restated task interface
// (core.hh), registered under the reference's kind strings (manager.cc:159-237).  Each factory
// parses the same JSON settings keys as the reference node, performs the same inference checks
// with the same "<Factory> inference error: " messages, and executes through the C ABI
// (include/holoflow_b200.h) on the stream given at create()/update().
#pragma once

#include <optional>

#include "holoflow_b200/core.hh"

namespace hfb::nodes {

// ---- settings (same keys as the reference) ------------------------------------------------------
struct FresnelDiffractionSettings { // fresnel_diffraction.cu:40-64
  float            lambda = 0.f, dx = 0.f, dy = 0.f, z = 0.f;
  std::vector<int> axes{-2, -1};
  bool             skip_phase_shift = false;
  bool             output_magnitude = false;
};
struct AngularSpectrumFilter { // angular_spectrum.cu:40-55
  uint32_t r_inner = 0, r_outer = 0, s_inner = 0, s_outer = 0;
};
struct AngularSpectrumPadding { // angular_spectrum.cu:57-66
  int width = 0, height = 0;
};
struct AngularSpectrumSettings { // angular_spectrum.cu:68-99
  float                                lambda = 0.f, dx = 0.f, dy = 0.f, z = 0.f;
  std::optional<AngularSpectrumFilter>  filter;
  std::optional<AngularSpectrumPadding> padding;
};
struct PcaSettings { // pca.cc:141-151
  int begin = 0, end = 0;
  int components() const { return end - begin; }
};
enum class FftNorm { Backward, Forward, Ortho }; // fft_common.cc:45-62
struct FFTSettings {                             // fft.cu:33-52
  int     axis = -1;
  FftNorm norm = FftNorm::Backward;
};
struct MeanSettings { // mean.cu:30-70
  std::vector<int> axis;
  bool             keepdims = false;
};
struct ConversionSettings { // conversion.cu:40-103
  enum class Target { U8, U16, F32, CF32 } target = Target::F32;
  enum class Strategy { Real, Scaled, Modulus, Argument } strategy = Strategy::Real;
};
// The fused per-window path (no single reference node: it replaces the chain GraphBuilder wires,
// graph_builder.cc:245-678).  Keys follow the reference's Settings names where one exists.
struct DopplerMomentsSettings {
  int                                   time_z_begin = 0, time_z_end = 0; // settings.hh:111-112
  int                                   clutter_rank = 0;                 // SVD filter rank removed
  std::string                           propagation  = "fresnel";         // fresnel | angular_spectrum | none
  std::string                           input_format = "u16";             // u8 | u16 | f32 | mono12p
  int                                   height = 0, width = 0;            // frame size (mono12p rows)
  float                                 lambda = 0.f, dx = 0.f, z = 0.f, fs = 37e3f;
  std::vector<std::string>              moments{"M0", "M1", "M2"};
  bool                                  fftshift = false;
  std::string                           form     = "plain";               // plain | chosen
  std::string                           time_method = "rfft";            // rfft | fft (settings.hh TimeMethod)
  std::optional<AngularSpectrumFilter>  filter;
  std::optional<AngularSpectrumPadding> padding;
  // Shack-Hartmann autofocus before the Fresnel propagation, under the reference's Settings names
  // (settings.hh autofocus_*, pp_pctclip_radius for the correlation ROI)
  bool             autofocus_enabled = false;
  int              autofocus_nb_subaps = 0, autofocus_nb_iter = 1;
  std::vector<int> autofocus_zernike_orders;
  bool             autofocus_skip_subapertures_outside_pupil = true;
  float            pp_pctclip_radius = 0.5f;
  bool             pp_flatfield = false;            // flatfield of the sub-aperture images
  float            pp_flatfield_cutoff_period_m = 0.f;
  int              pp_accumulation = 1;                    // sliding correction over n windows
  bool             autofocus_use_graph_laplacian = false;  // FullPairwise slopes
};

// Source node reading a .holo file (holotask/include/holotask/sources/holofile.hh:30-50).
struct HolofileSettings {
  enum class LoadKind { Live, CPUCached, GPUCached } load_kind = LoadKind::Live;
  std::string        path;
  int                start_frame = 0, end_frame = 0, batch_size = 0;
  std::optional<int> max_fps;           // playback cap in frames per second
  bool               keep_cursor = true; // keep the read position across update()
};

// Post-moment display chain (holonp/include/holonp/fftshift.hh, holotask/syncs/flatfield.hh,
// holotask/syncs/pct_clip.hh): the same keys.
struct FFTShiftSettings {
  std::vector<int> axes; // empty: every axis
};
struct Filter2DSettings { // filter2d.cu:26-40
  uint32_t r_inner = 0, r_outer = 0, s_inner = 0, s_outer = 0;
  bool     operator==(const Filter2DSettings &) const = default;
};
struct FlatfieldSettings {
  float sigma_y = 0.f, sigma_x = 0.f; // Gaussian sigmas in pixels
};
struct PctClipSettings {
  struct Ellipse {
    float cx = 0.5f, cy = 0.5f, rx = 0.5f, ry = 0.5f, angle = 0.f; // normalized; angle in degrees
    bool  operator==(const Ellipse &) const = default;
  };
  float   min_pct = 0.f, max_pct = 100.f;
  Ellipse roi;
  bool    operator==(const PctClipSettings &) const = default;
};

// Shack-Hartmann autofocus (holotask/include/holotask/syncs/short_time_fresnel_diffraction.hh,
// shack_hartmann_slopes.hh, zernike_from_slopes.hh, zernike_phase.hh, zernike_defocus_z_prop.hh):
// the same keys and defaults.
struct ShortTimeFresnelDiffractionSettings {
  float            lambda = 0.f, dx = 0.f, dy = 0.f, z = 0.f;
  size_t           win_h = 0, win_w = 0, stride_y = 0, stride_x = 0;
  std::string      phase_ref        = "LOCAL"; // LOCAL | GLOBAL
  bool             skip_phase_shift = true, output_magnitude = false;
  std::vector<int> axes             = {-2, -1};
  bool             operator==(const ShortTimeFresnelDiffractionSettings &) const = default;
};
struct ShackHartmannSlopeSettings {
  std::string             mode   = "single_reference"; // single_reference (full_pairwise: not built)
  float                   lambda = 0.f, dx = 0.f, dy = 0.f, z = 0.f;
  size_t                  subaperture_height = 0, subaperture_width = 0, stride_y = 0, stride_x = 0;
  PctClipSettings::Ellipse correlation_roi;
  bool                    skip_subapertures_outside_pupil = true, output_xcorr_maps = false;
  size_t                  pair_batch_size                 = 256;
  bool                    operator==(const ShackHartmannSlopeSettings &) const = default;
};
struct ZernikeFromSlopesSettings {
  std::vector<int> indexes;
  float            lambda = 0.f, dx = 0.f, dy = 0.f;
  size_t           subaperture_height = 0, subaperture_width = 0, stride_y = 0, stride_x = 0, ny = 1, nx = 1;
  bool             skip_subapertures_outside_pupil = true;
  bool             operator==(const ZernikeFromSlopesSettings &) const = default;
};
struct ZernikePhaseSettings {
  std::vector<int> indexes;
  int              ny = 0, nx = 0;
  core::MemLoc     output = core::MemLoc::Host;
  bool             operator==(const ZernikePhaseSettings &) const = default;
};
struct ZernikeDefocusZPropSettings {
  std::vector<int> indexes;
  float            lambda = 0.f, z_curr = 0.f, pupil_radius = 0.f;
  bool             operator==(const ZernikeDefocusZPropSettings &) const = default;
};

void from_json(const nlohmann::json &j, ShortTimeFresnelDiffractionSettings &s);
void from_json(const nlohmann::json &j, ShackHartmannSlopeSettings &s);
void from_json(const nlohmann::json &j, ZernikeFromSlopesSettings &s);
void from_json(const nlohmann::json &j, ZernikePhaseSettings &s);
void from_json(const nlohmann::json &j, ZernikeDefocusZPropSettings &s);
void from_json(const nlohmann::json &j, FresnelDiffractionSettings &s);
void from_json(const nlohmann::json &j, FFTShiftSettings &s);
void from_json(const nlohmann::json &j, FlatfieldSettings &s);
void from_json(const nlohmann::json &j, Filter2DSettings &s);
void from_json(const nlohmann::json &j, PctClipSettings &s);
void from_json(const nlohmann::json &j, HolofileSettings::LoadKind &s);
void from_json(const nlohmann::json &j, HolofileSettings &s);
void from_json(const nlohmann::json &j, AngularSpectrumFilter &s);
void from_json(const nlohmann::json &j, AngularSpectrumPadding &s);
void from_json(const nlohmann::json &j, AngularSpectrumSettings &s);
void from_json(const nlohmann::json &j, PcaSettings &s);
void from_json(const nlohmann::json &j, FftNorm &s);
void from_json(const nlohmann::json &j, FFTSettings &s);
void from_json(const nlohmann::json &j, MeanSettings &s);
void from_json(const nlohmann::json &j, ConversionSettings &s);
void from_json(const nlohmann::json &j, DopplerMomentsSettings &s);

// ---- factories ------------------------------------------------------------------------------------
using core::InferResult;
using core::ISyncTask;
using core::ISyncTaskFactory;
using core::SyncCreateCtx;
using core::TDesc;

#define HFB_SYNC_FACTORY(Name)                                                                            \
  class Name final : public ISyncTaskFactory {                                                            \
  public:                                                                                                 \
    InferResult infer(std::span<const TDesc> input_descs, const nlohmann::json &jsettings) const override; \
    std::unique_ptr<ISyncTask> create(std::span<const TDesc> input_descs, const nlohmann::json &jsettings, \
                                      const SyncCreateCtx &ctx) const override;                           \
    std::unique_ptr<ISyncTask> update(std::unique_ptr<ISyncTask> old_task, std::span<const TDesc> input_descs, \
                                      const nlohmann::json &jsettings, const SyncCreateCtx &ctx) const override; \
  }

HFB_SYNC_FACTORY(FresnelDiffractionFactory);
HFB_SYNC_FACTORY(AngularSpectrumFactory);
HFB_SYNC_FACTORY(PcaFactory);
HFB_SYNC_FACTORY(FFTFactory);
HFB_SYNC_FACTORY(RFFTFactory);
HFB_SYNC_FACTORY(MeanFactory);
HFB_SYNC_FACTORY(MeanAbsFactory);
HFB_SYNC_FACTORY(ConversionFactory);
HFB_SYNC_FACTORY(DopplerMomentsFactory);
HFB_SYNC_FACTORY(FFTShiftFactory);  // kind "FFTShiftNp"
HFB_SYNC_FACTORY(FlatfieldFactory);
HFB_SYNC_FACTORY(Filter2DFactory);
HFB_SYNC_FACTORY(PctClipFactory);
HFB_SYNC_FACTORY(ShortTimeFresnelDiffractionFactory);
HFB_SYNC_FACTORY(ShackHartmannSlopesFactory); // [1, sy, sx, h, w] -> slopes [1, sy, sx, 2] (+ maps)
HFB_SYNC_FACTORY(ZernikeFromSlopesFactory);   // Host input as the reference; Device input runs the device fit
HFB_SYNC_FACTORY(ZernikePhaseFactory);
HFB_SYNC_FACTORY(CorrectPhaseFactory);
HFB_SYNC_FACTORY(Wrap2PiFactory);
HFB_SYNC_FACTORY(ZernikeDefocusZPropFactory); // sink: no outputs; the task keeps the last estimate
HFB_SYNC_FACTORY(HolofileFactory); // frames [batch, H, W] (12-bit: packed rows [batch, H, 3W/2] U8)
// the thin holonp kinds GraphBuilder wires between the path's stages (nodes_np.cc)
HFB_SYNC_FACTORY(SliceFactory);   // a strided view of the input (in place)
HFB_SYNC_FACTORY(ReshapeFactory); // a view when the layout allows, else a contiguous copy
HFB_SYNC_FACTORY(CopyFactory);
HFB_SYNC_FACTORY(ConcatenateFactory);
HFB_SYNC_FACTORY(ArangeFactory);
HFB_SYNC_FACTORY(MultiplyFactory);
HFB_SYNC_FACTORY(AbsFactory);
HFB_SYNC_FACTORY(CausalSlidingAverageFactory);
#undef HFB_SYNC_FACTORY

using core::AsyncCreateCtx;
using core::IAsyncTask;
using core::IAsyncTaskFactory;

#define HFB_ASYNC_FACTORY(Name)                                                                           \
  class Name final : public IAsyncTaskFactory {                                                           \
  public:                                                                                                 \
    InferResult infer(std::span<const TDesc> input_descs, const nlohmann::json &jsettings) const override; \
    std::unique_ptr<IAsyncTask> create(std::span<const TDesc> input_descs, const nlohmann::json &jsettings, \
                                       const AsyncCreateCtx &ctx) const override;                         \
  }

// the queues (holotask/src/asyncs): owned inputs written through acquire_input, zero-copy views out
HFB_ASYNC_FACTORY(BatchQueueFactory);
HFB_ASYNC_FACTORY(DualReaderBatchQueueFactory);
HFB_ASYNC_FACTORY(SlidingAverageFactory);
#undef HFB_ASYNC_FACTORY

// Registers the kinds of nodes_np.cc: "Slice", "Reshape", "Copy", "Concatenate", "Arange",
// "Multiply", "Abs", "CausalSlidingAverage" and the asynchronous "BatchQueue",
// "DualReaderBatchQueue" and "SlidingAverage".
void register_np_kinds(core::Registry &registry);

// Registers every node above under its kind string: "FresnelDiffraction", "AngularSpectrum",
// "Pca", "FFT", "RFFT", "Mean", "MeanAbs", "Conversion", "FFTShiftNp", "Flatfield", "Filter2D",
// "PctClip", "Holofile" (the reference's) and "DopplerMoments".
void register_path_kinds(core::Registry &registry);

// The process-wide registry the C ABI's hf_node_* functions use.
core::Registry &default_registry();

} // namespace hfb::nodes
