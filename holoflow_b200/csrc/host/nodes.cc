// The Doppler path's compute nodes (hfb::nodes) over the C ABI.  Every factory mirrors the
// reference node named in its comment: settings keys, inference checks and messages, output
// descriptors, in-place and ownership declarations; execution goes through the hf_* entry points
// on the task's stream.
#include "holoflow_b200/nodes.hh"

#include <algorithm>
#include <cstring>
#include <numeric>

#include "holoflow_b200.h"

namespace hfb::nodes {

using core::DType;
using core::MemLoc;
using core::OpResult;
using core::SyncCtx;

// ================================================================================================
// settings
// ================================================================================================
void from_json(const nlohmann::json &j, FresnelDiffractionSettings &s) {
  j.at("lambda").get_to(s.lambda);
  j.at("dx").get_to(s.dx);
  j.at("dy").get_to(s.dy);
  j.at("z").get_to(s.z);
  s.axes = {-2, -1};
  if (j.contains("axes"))
    j.at("axes").get_to(s.axes);
  if (j.contains("skip_phase_shift"))
    j.at("skip_phase_shift").get_to(s.skip_phase_shift);
  if (j.contains("output_magnitude"))
    j.at("output_magnitude").get_to(s.output_magnitude);
}
void from_json(const nlohmann::json &j, AngularSpectrumFilter &f) {
  j.at("r_inner").get_to(f.r_inner);
  j.at("r_outer").get_to(f.r_outer);
  j.at("s_inner").get_to(f.s_inner);
  j.at("s_outer").get_to(f.s_outer);
}
void from_json(const nlohmann::json &j, AngularSpectrumPadding &p) {
  j.at("width").get_to(p.width);
  j.at("height").get_to(p.height);
}
void from_json(const nlohmann::json &j, AngularSpectrumSettings &s) {
  j.at("lambda").get_to(s.lambda);
  j.at("dx").get_to(s.dx);
  j.at("dy").get_to(s.dy);
  j.at("z").get_to(s.z);
  if (j.contains("filter"))
    s.filter = j.at("filter").get<AngularSpectrumFilter>();
  if (j.contains("padding"))
    s.padding = j.at("padding").get<AngularSpectrumPadding>();
}
void from_json(const nlohmann::json &j, PcaSettings &s) {
  j.at("begin").get_to(s.begin);
  j.at("end").get_to(s.end);
}
void from_json(const nlohmann::json &j, FftNorm &n) {
  if (j.is_null()) {
    n = FftNorm::Backward;
    return;
  }
  const auto s = j.get<std::string>();
  if (s == "backward" || s == "none")
    n = FftNorm::Backward;
  else if (s == "forward")
    n = FftNorm::Forward;
  else if (s == "ortho")
    n = FftNorm::Ortho;
  else
    throw std::invalid_argument("FftNorm: unsupported norm '" + s + "'");
}
void from_json(const nlohmann::json &j, FFTSettings &s) {
  s.axis = j.contains("axis") ? j.at("axis").get<int>() : -1;
  s.norm = j.contains("norm") ? j.at("norm").get<FftNorm>() : FftNorm::Backward;
}
void from_json(const nlohmann::json &j, MeanSettings &s) {
  s.axis.clear();
  for (const char *key : {"axis", "axes"}) {
    if (!j.contains(key))
      continue;
    const auto &ja = j.at(key);
    if (ja.is_null())
      s.axis.clear();
    else if (ja.is_number_integer())
      s.axis = {ja.get<int>()};
    else if (ja.is_array())
      ja.get_to(s.axis);
    else
      throw std::invalid_argument(std::string("MeanSettings: ") + key + " must be int, array, or null");
    break;
  }
  s.keepdims = j.contains("keepdims") ? j.at("keepdims").get<bool>() : false;
}
void from_json(const nlohmann::json &j, ConversionSettings &s) {
  const auto t = j.at("target").get<std::string>();
  if (t == "U8")
    s.target = ConversionSettings::Target::U8;
  else if (t == "U16")
    s.target = ConversionSettings::Target::U16;
  else if (t == "F32")
    s.target = ConversionSettings::Target::F32;
  else if (t == "CF32")
    s.target = ConversionSettings::Target::CF32;
  else
    throw std::invalid_argument("Unknown target type for conversion: " + t);
  const auto st = j.at("strategy").get<std::string>();
  if (st == "Real")
    s.strategy = ConversionSettings::Strategy::Real;
  else if (st == "Scaled")
    s.strategy = ConversionSettings::Strategy::Scaled;
  else if (st == "Modulus")
    s.strategy = ConversionSettings::Strategy::Modulus;
  else if (st == "Argument")
    s.strategy = ConversionSettings::Strategy::Argument;
  else
    throw std::invalid_argument("Unknown strategy type for conversion: " + st);
}
void from_json(const nlohmann::json &j, DopplerMomentsSettings &s) {
  j.at("time_z_begin").get_to(s.time_z_begin);
  j.at("time_z_end").get_to(s.time_z_end);
  auto opt = [&](const char *k, auto &v) {
    if (j.contains(k))
      j.at(k).get_to(v);
  };
  opt("clutter_rank", s.clutter_rank);
  opt("propagation", s.propagation);
  opt("input_format", s.input_format);
  opt("height", s.height);
  opt("width", s.width);
  opt("lambda", s.lambda);
  opt("dx", s.dx);
  opt("z", s.z);
  opt("fs", s.fs);
  opt("moments", s.moments);
  opt("fftshift", s.fftshift);
  opt("form", s.form);
  opt("time_method", s.time_method);
  if (j.contains("filter"))
    s.filter = j.at("filter").get<AngularSpectrumFilter>();
  if (j.contains("padding"))
    s.padding = j.at("padding").get<AngularSpectrumPadding>();
  opt("autofocus_enabled", s.autofocus_enabled);
  opt("autofocus_nb_subaps", s.autofocus_nb_subaps);
  opt("autofocus_nb_iter", s.autofocus_nb_iter);
  opt("autofocus_zernike_orders", s.autofocus_zernike_orders);
  opt("autofocus_skip_subapertures_outside_pupil", s.autofocus_skip_subapertures_outside_pupil);
  opt("pp_pctclip_radius", s.pp_pctclip_radius);
  opt("pp_flatfield", s.pp_flatfield);
  opt("pp_flatfield_cutoff_period_m", s.pp_flatfield_cutoff_period_m);
  opt("pp_accumulation", s.pp_accumulation);
  opt("autofocus_use_graph_laplacian", s.autofocus_use_graph_laplacian);
}

// ================================================================================================
// helpers
// ================================================================================================
namespace {

struct Check {
  const char *factory;
  void        operator()(bool cond, const std::string &msg) const {
    if (!cond)
      throw std::invalid_argument(std::string(factory) + " inference error: " + msg);
  }
};

// Maps a C-ABI status onto the reference's exception types.
void hf_ok(int rc, const char *who) {
  if (rc == HF_OK)
    return;
  const std::string msg = std::string(who) + ": " + hf_last_error();
  if (rc == HF_ERR_INVALID || rc == HF_ERR_UNSUPPORTED)
    throw std::invalid_argument(msg);
  throw core::CudaError(msg);
}

int hf_dtype(DType d) {
  switch (d) {
  case DType::U8: return HF_U8;
  case DType::U16: return HF_U16;
  case DType::F32: return HF_F32;
  case DType::CF32: return HF_CF32;
  }
  return -1;
}

size_t prod(const std::vector<size_t> &s, size_t b, size_t e) {
  size_t n = 1;
  for (size_t i = b; i < e && i < s.size(); ++i)
    n *= s[i];
  return n;
}

int norm_axis(int axis, size_t rank) { return axis < 0 ? axis + (int)rank : axis; }

// Device buffer owned by a task.
struct DevBuf {
  void *p = nullptr;
  DevBuf() = default;
  explicit DevBuf(size_t bytes) {
    if (bytes && cudaMalloc(&p, bytes) != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      throw core::CudaError("device allocation of " + std::to_string(bytes) + " bytes failed");
    }
  }
  DevBuf(const DevBuf &)            = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p) { o.p = nullptr; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) {
      if (p)
        cudaFree(p);
      p   = o.p;
      o.p = nullptr;
    }
    return *this;
  }
  ~DevBuf() {
    if (p)
      cudaFree(p);
  }
  template <class T> T *as() const { return static_cast<T *>(p); }
};

InferResult sync_result(const TDesc &in, const TDesc &out, std::vector<core::InPlace> in_place = {}) {
  InferResult r;
  r.input_descs   = {in};
  r.output_descs  = {out};
  r.in_place      = std::move(in_place);
  r.owned_inputs  = {false};
  r.owned_outputs = {false};
  r.kind          = core::TaskKind::Sync;
  return r;
}

} // namespace

// ================================================================================================
// FresnelDiffraction (fresnel_diffraction.cu:466-668)
// ================================================================================================
namespace {
// How the planes of a transform over axes (ax0, ax1) are launched: the dimensions other than the
// two axes split into one batch group, a run of them that collapses into a single uniform stride in
// both the input and the output (the largest such run), and the rest, whose index combinations
// become one launch each at a byte offset (the batch-group selection of fresnel_diffraction.cu:
// 130-200, 545-570).
struct PlaneLaunches {
  int                  ax0 = 0, ax1 = 0;
  int64_t              batch = 1;                   // planes per launch
  int64_t              in_bstride = 0, out_bstride = 0; // elements between planes of a launch
  std::vector<int64_t> in_off, out_off;              // byte offset of each launch
};

PlaneLaunches plane_launches(const TDesc &in, const TDesc &out, int ax0, int ax1) {
  PlaneLaunches pl;
  pl.ax0 = ax0, pl.ax1 = ax1;
  const int        rank = (int)in.rank();
  std::vector<int> outer;
  for (int d = 0; d < rank; ++d)
    if (d != ax0 && d != ax1)
      outer.push_back(d);
  const auto collapses = [&](int a, int b) {
    return in.strides[(size_t)a] == in.strides[(size_t)b] * in.shape[(size_t)b] &&
           out.strides[(size_t)a] == out.strides[(size_t)b] * out.shape[(size_t)b];
  };
  size_t best_lo = 0, best_hi = 0; // run outer[best_lo, best_hi)
  int64_t best = outer.empty() ? 1 : 0;
  for (size_t lo = 0; lo < outer.size(); ++lo) {
    int64_t n  = (int64_t)in.shape[(size_t)outer[lo]];
    size_t  hi = lo + 1;
    while (hi < outer.size() && collapses(outer[hi - 1], outer[hi]))
      n *= (int64_t)in.shape[(size_t)outer[hi++]];
    if (n >= best)
      best = n, best_lo = lo, best_hi = hi;
  }
  const size_t ie = core::size_of(in.dtype), oe = core::size_of(out.dtype);
  pl.batch        = best;
  if (best_hi > best_lo) {
    pl.in_bstride  = (int64_t)(in.strides[(size_t)outer[best_hi - 1]] / ie);
    pl.out_bstride = (int64_t)(out.strides[(size_t)outer[best_hi - 1]] / oe);
  }
  std::vector<int> rest;
  for (size_t i = 0; i < outer.size(); ++i)
    if (i < best_lo || i >= best_hi)
      rest.push_back(outer[i]);
  pl.in_off.push_back(0), pl.out_off.push_back(0);
  for (int d : rest) { // every index combination of the remaining dimensions
    std::vector<int64_t> ni, no;
    for (size_t k = 0; k < in.shape[(size_t)d]; ++k)
      for (size_t j = 0; j < pl.in_off.size(); ++j) {
        ni.push_back(pl.in_off[j] + (int64_t)(k * in.strides[(size_t)d]));
        no.push_back(pl.out_off[j] + (int64_t)(k * out.strides[(size_t)d]));
      }
    pl.in_off.swap(ni), pl.out_off.swap(no);
  }
  return pl;
}

class FresnelTask final : public ISyncTask {
public:
  hf_fresnel_plan           *plan = nullptr;
  cudaStream_t               stream{};
  FresnelDiffractionSettings s;
  TDesc                      idesc;
  PlaneLaunches              pl;
  ~FresnelTask() override {
    if (plan)
      hf_fresnel_plan_destroy(plan);
  }
  OpResult execute(SyncCtx &ctx) override {
    auto      &in = ctx.inputs[0];
    auto      &out = ctx.outputs[0];
    const auto ie = core::size_of(in.desc.dtype), oe = core::size_of(out.desc.dtype);
    const auto a0 = (size_t)pl.ax0, a1 = (size_t)pl.ax1;
    for (size_t k = 0; k < pl.in_off.size(); ++k)
      hf_ok(hf_fresnel_exec(plan, in.data() + pl.in_off[k], pl.in_bstride, (int64_t)(in.desc.strides[a0] / ie),
                            (int64_t)(in.desc.strides[a1] / ie), out.data() + pl.out_off[k], pl.out_bstride,
                            (int64_t)(out.desc.strides[a0] / oe), (int64_t)(out.desc.strides[a1] / oe), stream),
            "FresnelDiffraction");
    return OpResult::Ok;
  }
};
} // namespace

InferResult FresnelDiffractionFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"FresnelDiffractionFactory"};
  const auto  s = j.get<FresnelDiffractionSettings>();
  check(input_descs.size() == 1, "expected exactly one input");
  const auto &idesc = input_descs[0];
  check(idesc.rank() >= 2, "input must be a tensor of rank 2 or higher");
  check(idesc.dtype == DType::CF32 || idesc.dtype == DType::F32, "input must be complex float32 or real float32");
  check(idesc.mem_loc == MemLoc::Device, "input must be in device memory");
  check(s.axes.size() == 2, "axes must contain exactly two dimensions");
  const int rank = (int)idesc.rank();
  const int ax0 = norm_axis(s.axes[0], rank), ax1 = norm_axis(s.axes[1], rank);
  check(ax0 >= 0 && ax0 < rank && ax1 >= 0 && ax1 < rank, "axes out of bounds");
  check(ax0 != ax1, "axes must be distinct");
  check(idesc.strides[ax0] % idesc.strides[ax1] == 0, "stride of ax0 (H) must be a multiple of stride of ax1 (W)");
  check(s.lambda > 0.0f, "wavelength must be positive");
  check(s.dx > 0.0f, "dx must be positive");
  check(s.dy > 0.0f, "dy must be positive");
  check(s.dx == s.dy, "dx must equal dy");
  TDesc odesc;
  if (s.output_magnitude)
    odesc = TDesc(idesc.shape, DType::F32, idesc.mem_loc);
  else if (idesc.dtype == DType::CF32)
    odesc = idesc;
  else
    odesc = TDesc(idesc.shape, DType::CF32, idesc.mem_loc);
  return sync_result(idesc, odesc);
}

std::unique_ptr<ISyncTask> FresnelDiffractionFactory::create(std::span<const TDesc> input_descs,
                                                             const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  const auto  inf = infer(input_descs, j);
  auto        t   = std::make_unique<FresnelTask>();
  const auto &d   = input_descs[0];
  t->s            = j.get<FresnelDiffractionSettings>();
  t->idesc        = d;
  t->stream       = ctx.stream;
  const int rank  = (int)d.rank();
  t->pl = plane_launches(d, inf.output_descs[0], norm_axis(t->s.axes[0], rank), norm_axis(t->s.axes[1], rank));
  hf_ok(hf_fresnel_plan_create(t->pl.batch, (int)d.shape[(size_t)t->pl.ax0], (int)d.shape[(size_t)t->pl.ax1],
                               hf_dtype(d.dtype), t->s.lambda, t->s.dx, t->s.z, t->s.output_magnitude ? 1 : 0,
                               t->s.skip_phase_shift ? 1 : 0, &t->plan, ctx.stream),
        "FresnelDiffraction");
  return t;
}

// Same input and settings but z: rebuild the lens only (fresnel_diffraction.cu:634-668).
std::unique_ptr<ISyncTask> FresnelDiffractionFactory::update(std::unique_ptr<ISyncTask> old,
                                                             std::span<const TDesc> input_descs,
                                                             const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  auto *t = dynamic_cast<FresnelTask *>(old.get());
  if (t && input_descs.size() == 1 && input_descs[0] == t->idesc) {
    (void)infer(input_descs, j);
    const auto s = j.get<FresnelDiffractionSettings>();
    if (s.lambda == t->s.lambda && s.dx == t->s.dx && s.dy == t->s.dy && s.axes == t->s.axes &&
        s.skip_phase_shift == t->s.skip_phase_shift && s.output_magnitude == t->s.output_magnitude) {
      if (s.z != t->s.z)
        hf_ok(hf_fresnel_plan_set_z(t->plan, s.z, ctx.stream), "FresnelDiffraction");
      t->s      = s;
      t->stream = ctx.stream;
      return old;
    }
  }
  old.reset();
  return create(input_descs, j, ctx);
}

// ================================================================================================
// AngularSpectrum (angular_spectrum.cu:446-580)
// ================================================================================================
namespace {
class AngularSpectrumTask final : public ISyncTask {
public:
  hf_as_plan  *plan = nullptr;
  cudaStream_t stream{};
  ~AngularSpectrumTask() override {
    if (plan)
      hf_as_plan_destroy(plan);
  }
  OpResult execute(SyncCtx &ctx) override {
    hf_ok(hf_as_exec(plan, ctx.inputs[0].data(), ctx.outputs[0].data(), stream), "AngularSpectrum");
    return OpResult::Ok;
  }
};
} // namespace

InferResult AngularSpectrumFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"AngularSpectrumFactory"};
  const auto  s = j.get<AngularSpectrumSettings>();
  check(input_descs.size() == 1, "expected exactly one input");
  const auto &idesc = input_descs[0];
  check(idesc.rank() >= 2, "input must be a tensor of rank 2 or higher");
  check(idesc.dtype == DType::CF32 || idesc.dtype == DType::F32, "input must be complex float32 or real float32");
  check(idesc.mem_loc == MemLoc::Device, "input must be in device memory");
  check(idesc.is_contiguous(), "input must be C-contiguous");
  check(s.lambda > 0.0f, "wavelength must be positive");
  check(s.dx > 0.0f, "dx must be positive");
  check(s.dy > 0.0f, "dy must be positive");
  check(s.dx == s.dy, "dx must equal dy");
  const size_t r = idesc.rank();
  const int    height = (int)idesc.shape[r - 2], width = (int)idesc.shape[r - 1];
  auto         oshape = idesc.shape;
  if (s.padding) {
    const auto &p = *s.padding;
    check(p.width > 0, "padding width must be positive");
    check(p.height > 0, "padding height must be positive");
    check(p.width >= width, "padding width must be at least the input width");
    check(p.height >= height, "padding height must be at least the input height");
    check((p.width - width) % 2 == 0, "horizontal padding must be even");
    check((p.height - height) % 2 == 0, "vertical padding must be even");
    oshape[r - 2] = (size_t)p.height;
    oshape[r - 1] = (size_t)p.width;
  }
  std::vector<core::InPlace> in_place;
  if (idesc.dtype == DType::CF32 && !s.padding)
    in_place.push_back({0, 0});
  return sync_result(idesc, TDesc(oshape, DType::CF32, idesc.mem_loc), std::move(in_place));
}

std::unique_ptr<ISyncTask> AngularSpectrumFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                          const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  const auto  s = j.get<AngularSpectrumSettings>();
  const auto &d = input_descs[0];
  const auto  r = d.rank();
  auto        t = std::make_unique<AngularSpectrumTask>();
  t->stream     = ctx.stream;
  const AngularSpectrumFilter f = s.filter.value_or(AngularSpectrumFilter{});
  hf_ok(hf_as_plan_create((int64_t)prod(d.shape, 0, r - 2), (int)d.shape[r - 2], (int)d.shape[r - 1], hf_dtype(d.dtype),
                          s.lambda, s.dx, s.z, s.padding ? s.padding->width : 0, s.padding ? s.padding->height : 0,
                          s.filter ? 1 : 0, f.r_inner, f.r_outer, f.s_inner, f.s_outer, &t->plan, ctx.stream),
        "AngularSpectrum");
  return t;
}

std::unique_ptr<ISyncTask> AngularSpectrumFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> in,
                                                          const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  old.reset();
  return create(in, j, ctx);
}

// ================================================================================================
// Pca (pca.cc:68-193): C = X^T X, ascending eigendecomposition, projection on [begin, end)
// ================================================================================================
namespace {
class PcaTask final : public ISyncTask {
public:
  cudaStream_t stream{};
  PcaSettings  s;
  int64_t      batch = 0, P = 0;
  int          F = 0;
  DevBuf       gram, evecs, evals, info, ws;
  OpResult     execute(SyncCtx &ctx) override {
    const void *x = ctx.inputs[0].data();
    hf_ok(hf_covariance(x, HF_F32, batch, F, P, gram.as<double>(), ws.p, stream), "Pca");
    hf_ok(hf_eigh_jacobi_f64(gram.as<double>(), evecs.as<double>(), evals.as<double>(), info.as<int>(), F, batch,
                             stream),
          "Pca");
    hf_ok(hf_pca_project(static_cast<const float *>(x), batch, F, P, evecs.as<double>(), s.begin, s.end,
                         reinterpret_cast<float *>(ctx.outputs[0].data()), stream),
          "Pca");
    return OpResult::Ok;
  }
};
} // namespace

InferResult PcaFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"PcaFactory"};
  const auto  s = j.get<PcaSettings>();
  check(input_descs.size() == 1, "expected exactly one input");
  const auto &idesc = input_descs[0];
  check(idesc.rank() >= 3, "expected input rank >= 3");
  check(idesc.dtype == DType::F32, "PCA supports F32 input only");
  check(idesc.mem_loc == MemLoc::Device, "expected input in device memory");
  check(s.begin < s.end, "expected begin < end");
  check(s.begin >= 0, "expected begin >= 0");
  const size_t feat = idesc.rank() - 3;
  check(s.end <= (int)idesc.shape.at(feat), "expected end <= n_features");
  check(idesc.is_contiguous(), "expected C-contiguous input");
  check(idesc.shape.at(feat) <= 128, "at most 128 features");
  auto oshape  = idesc.shape;
  oshape[feat] = (size_t)s.components();
  return sync_result(idesc, TDesc(oshape, idesc.dtype, idesc.mem_loc));
}

std::unique_ptr<ISyncTask> PcaFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                              const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  const auto &d    = input_descs[0];
  const auto  r    = d.rank();
  auto        t    = std::make_unique<PcaTask>();
  t->stream        = ctx.stream;
  t->s             = j.get<PcaSettings>();
  t->batch         = (int64_t)prod(d.shape, 0, r - 3);
  t->F             = (int)d.shape[r - 3];
  t->P             = (int64_t)prod(d.shape, r - 2, r);
  const size_t FF  = (size_t)t->F * t->F;
  t->gram          = DevBuf(sizeof(double) * FF * t->batch);
  t->evecs         = DevBuf(sizeof(double) * FF * t->batch);
  t->evals         = DevBuf(sizeof(double) * t->F * t->batch);
  t->info          = DevBuf(sizeof(int) * t->batch);
  t->ws            = DevBuf(std::max<size_t>(16, hf_covariance_workspace_bytes(t->F, t->P) * (size_t)t->batch));
  return t;
}

std::unique_ptr<ISyncTask> PcaFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> in,
                                              const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  old.reset();
  return create(in, j, ctx);
}

// ================================================================================================
// FFT / RFFT along one axis (fft.cu:234-252, rfft.cu:142-170)
// ================================================================================================
namespace {
class AxisDftTask final : public ISyncTask {
public:
  cudaStream_t stream{};
  int          dtype = 0, norm = 0, T = 0, bins = 0;
  int64_t      batch = 0, P = 0;
  OpResult     execute(SyncCtx &ctx) override {
    hf_ok(hf_temporal_dft(ctx.inputs[0].data(), dtype, batch, T, P, 0, bins, norm, ctx.outputs[0].data(), stream),
          "FFT");
    return OpResult::Ok;
  }
};

InferResult axis_dft_infer(const char *factory, bool real, std::span<const TDesc> input_descs, const nlohmann::json &j) {
  const Check check{factory};
  const auto  s = j.get<FFTSettings>();
  check(input_descs.size() == 1, "expected exactly one input");
  const auto &idesc = input_descs[0];
  check(idesc.rank() >= 1, "input must have rank >= 1");
  check(idesc.mem_loc == MemLoc::Device, "input must be in device memory");
  check(idesc.is_contiguous(), "input must be C-contiguous");
  if (real)
    check(idesc.dtype != DType::CF32, "input must be real");
  const int ax = norm_axis(s.axis, idesc.rank());
  check(ax >= 0 && ax < (int)idesc.rank(), "axis out of range");
  auto oshape = idesc.shape;
  if (real)
    oshape[ax] = oshape[ax] / 2 + 1;
  return sync_result(idesc, TDesc(oshape, DType::CF32, idesc.mem_loc));
}

std::unique_ptr<ISyncTask> axis_dft_create(bool real, std::span<const TDesc> input_descs, const nlohmann::json &j,
                                           const SyncCreateCtx &ctx) {
  const auto  s  = j.get<FFTSettings>();
  const auto &d  = input_descs[0];
  const int   ax = norm_axis(s.axis, d.rank());
  auto        t  = std::make_unique<AxisDftTask>();
  t->stream      = ctx.stream;
  t->dtype       = hf_dtype(d.dtype);
  t->norm = s.norm == FftNorm::Backward ? HF_NORM_BACKWARD : (s.norm == FftNorm::Forward ? HF_NORM_FORWARD : HF_NORM_ORTHO);
  t->batch = (int64_t)prod(d.shape, 0, (size_t)ax);
  t->T     = (int)d.shape[ax];
  t->P     = (int64_t)prod(d.shape, (size_t)ax + 1, d.rank());
  t->bins  = real ? t->T / 2 + 1 : t->T;
  return t;
}
} // namespace

InferResult FFTFactory::infer(std::span<const TDesc> in, const nlohmann::json &j) const {
  return axis_dft_infer("FFTFactory", false, in, j);
}
std::unique_ptr<ISyncTask> FFTFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                              const SyncCreateCtx &ctx) const {
  (void)infer(in, j);
  return axis_dft_create(false, in, j, ctx);
}
std::unique_ptr<ISyncTask> FFTFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> in,
                                              const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  old.reset();
  return create(in, j, ctx);
}
InferResult RFFTFactory::infer(std::span<const TDesc> in, const nlohmann::json &j) const {
  return axis_dft_infer("RFFTFactory", true, in, j);
}
std::unique_ptr<ISyncTask> RFFTFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                               const SyncCreateCtx &ctx) const {
  (void)infer(in, j);
  return axis_dft_create(true, in, j, ctx);
}
std::unique_ptr<ISyncTask> RFFTFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> in,
                                               const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  old.reset();
  return create(in, j, ctx);
}

// ================================================================================================
// Mean (mean.cu:355-400) and MeanAbs (mean_abs.cu:236-275) over one run of adjacent axes
// ================================================================================================
namespace {
class MeanTask final : public ISyncTask {
public:
  cudaStream_t stream{};
  bool         absolute = false;
  int          dtype    = 0;
  int64_t      outer = 0, n = 0, inner = 0;
  OpResult     execute(SyncCtx &ctx) override {
    if (absolute)
      hf_ok(hf_mean_abs_axis(ctx.inputs[0].data(), dtype, outer, n, inner,
                             reinterpret_cast<float *>(ctx.outputs[0].data()), stream),
            "MeanAbs");
    else
      hf_ok(hf_mean_axis(ctx.inputs[0].data(), dtype, outer, n, inner, ctx.outputs[0].data(), stream), "Mean");
    return OpResult::Ok;
  }
};

// Reduced axes as [lo, hi) (all axes when none are given); throws when they are not adjacent.
std::pair<size_t, size_t> reduced_run(const Check &check, const MeanSettings &s, size_t rank) {
  if (s.axis.empty())
    return {0, rank};
  std::vector<int> ax;
  for (int a : s.axis) {
    const int n = norm_axis(a, rank);
    check(n >= 0 && n < (int)rank, "axis out of range");
    ax.push_back(n);
  }
  std::sort(ax.begin(), ax.end());
  check(std::adjacent_find(ax.begin(), ax.end()) == ax.end(), "duplicate axis");
  check(ax.back() - ax.front() + 1 == (int)ax.size(), "reduced axes must be adjacent in this implementation");
  return {(size_t)ax.front(), (size_t)ax.back() + 1};
}

InferResult mean_infer(const char *factory, bool absolute, std::span<const TDesc> input_descs, const nlohmann::json &j) {
  const Check check{factory};
  const auto  s = j.get<MeanSettings>();
  check(input_descs.size() == 1, "expected exactly one input");
  const auto &idesc = input_descs[0];
  check(idesc.mem_loc == MemLoc::Device, "input must be in device memory");
  check(idesc.is_contiguous(), "input must be C-contiguous");
  if (absolute)
    check(idesc.dtype == DType::F32 || idesc.dtype == DType::CF32, "input must be F32 or CF32");
  const auto [lo, hi] = reduced_run(check, s, idesc.rank());
  std::vector<size_t> oshape;
  for (size_t i = 0; i < idesc.rank(); ++i) {
    if (i >= lo && i < hi) {
      if (s.keepdims)
        oshape.push_back(1);
    } else {
      oshape.push_back(idesc.shape[i]);
    }
  }
  const DType odt = (!absolute && idesc.dtype == DType::CF32) ? DType::CF32 : DType::F32;
  return sync_result(idesc, TDesc(oshape, odt, idesc.mem_loc));
}

std::unique_ptr<ISyncTask> mean_create(bool absolute, std::span<const TDesc> input_descs, const nlohmann::json &j,
                                       const SyncCreateCtx &ctx) {
  const auto  s = j.get<MeanSettings>();
  const auto &d = input_descs[0];
  const auto [lo, hi] = reduced_run(Check{absolute ? "MeanAbsFactory" : "MeanFactory"}, s, d.rank());
  auto t      = std::make_unique<MeanTask>();
  t->stream   = ctx.stream;
  t->absolute = absolute;
  t->dtype    = hf_dtype(d.dtype);
  t->outer    = (int64_t)prod(d.shape, 0, lo);
  t->n        = (int64_t)prod(d.shape, lo, hi);
  t->inner    = (int64_t)prod(d.shape, hi, d.rank());
  return t;
}
} // namespace

InferResult MeanFactory::infer(std::span<const TDesc> in, const nlohmann::json &j) const {
  return mean_infer("MeanFactory", false, in, j);
}
std::unique_ptr<ISyncTask> MeanFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                               const SyncCreateCtx &ctx) const {
  (void)infer(in, j);
  return mean_create(false, in, j, ctx);
}
std::unique_ptr<ISyncTask> MeanFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> in,
                                               const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  old.reset();
  return create(in, j, ctx);
}
InferResult MeanAbsFactory::infer(std::span<const TDesc> in, const nlohmann::json &j) const {
  return mean_infer("MeanAbsFactory", true, in, j);
}
std::unique_ptr<ISyncTask> MeanAbsFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                                  const SyncCreateCtx &ctx) const {
  (void)infer(in, j);
  return mean_create(true, in, j, ctx);
}
std::unique_ptr<ISyncTask> MeanAbsFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> in,
                                                  const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  old.reset();
  return create(in, j, ctx);
}

// ================================================================================================
// Conversion (conversion.cu:138-150 supported configurations, 389-445 infer/create)
// ================================================================================================
namespace {
struct ConvCfg {
  DType                          in;
  ConversionSettings::Target     target;
  ConversionSettings::Strategy   strategy;
  DType                          out;
};
using CT = ConversionSettings::Target;
using CS = ConversionSettings::Strategy;
const ConvCfg kConv[] = {
    {DType::U8, CT::F32, CS::Real, DType::F32},        {DType::U8, CT::CF32, CS::Real, DType::CF32},
    {DType::U16, CT::CF32, CS::Real, DType::CF32},     {DType::F32, CT::U8, CS::Scaled, DType::U8},
    {DType::F32, CT::U16, CS::Scaled, DType::U16},     {DType::F32, CT::CF32, CS::Real, DType::CF32},
    {DType::CF32, CT::F32, CS::Modulus, DType::F32},   {DType::CF32, CT::F32, CS::Argument, DType::F32},
};
const ConvCfg *conv_cfg(DType in, const ConversionSettings &s) {
  for (const auto &c : kConv)
    if (c.in == in && c.target == s.target && c.strategy == s.strategy)
      return &c;
  return nullptr;
}
int hf_strategy(CS s) {
  switch (s) {
  case CS::Real: return HF_CONV_REAL;
  case CS::Scaled: return HF_CONV_SCALED;
  case CS::Modulus: return HF_CONV_MODULUS;
  case CS::Argument: return HF_CONV_ARGUMENT;
  }
  return -1;
}
class ConversionTask final : public ISyncTask {
public:
  cudaStream_t stream{};
  int          in_dt = 0, out_dt = 0, strategy = 0;
  int64_t      n = 0;
  DevBuf       minmax{64};
  OpResult     execute(SyncCtx &ctx) override {
    hf_ok(hf_convert(ctx.inputs[0].data(), in_dt, ctx.outputs[0].data(), out_dt, strategy, n, minmax.p, stream),
          "Conversion");
    return OpResult::Ok;
  }
};
} // namespace

InferResult ConversionFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"ConversionFactory"};
  const auto  s = j.get<ConversionSettings>();
  check(input_descs.size() == 1, "Expected exactly one input tensor");
  const auto &idesc = input_descs[0];
  check(idesc.mem_loc == MemLoc::Device, "Input tensor must be in device memory");
  check(idesc.is_contiguous(), "Input tensor must be C-contiguous");
  const ConvCfg *c = conv_cfg(idesc.dtype, s);
  check(c != nullptr, "Unsupported conversion configuration");
  return sync_result(idesc, TDesc(idesc.shape, c->out, MemLoc::Device));
}

std::unique_ptr<ISyncTask> ConversionFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                     const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  const auto     s = j.get<ConversionSettings>();
  const ConvCfg *c = conv_cfg(input_descs[0].dtype, s);
  auto           t = std::make_unique<ConversionTask>();
  t->stream        = ctx.stream;
  t->in_dt         = hf_dtype(c->in);
  t->out_dt        = hf_dtype(c->out);
  t->strategy      = hf_strategy(s.strategy);
  t->n             = (int64_t)input_descs[0].num_elements();
  return t;
}
std::unique_ptr<ISyncTask> ConversionFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> in,
                                                     const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  old.reset();
  return create(in, j, ctx);
}

// ================================================================================================
// DopplerMoments: windows [n_windows][T][H][W] (or packed [n_windows][T][3 H W / 2] bytes) ->
// moment images [n_windows][n_moments][OH][OW] through hf_pipeline_exec
// ================================================================================================
namespace {
struct DopplerPlan {
  hf_desc d{};
  int     nwin = 0, nmom = 0, OH = 0, OW = 0;
};

DopplerPlan doppler_plan(const Check &check, const TDesc &idesc, const DopplerMomentsSettings &s) {
  DopplerPlan dp;
  hf_desc    &d = dp.d;
  check(idesc.mem_loc == MemLoc::Device, "input must be in device memory");
  check(idesc.is_contiguous(), "input must be C-contiguous");
  const bool packed = s.input_format == "mono12p";
  if (packed) {
    check(idesc.dtype == DType::U8 && idesc.rank() == 3, "mono12p input must be U8 [n_windows][T][3 H W / 2]");
    check(s.height > 0 && s.width > 0 && (size_t)s.height * s.width * 3 / 2 == idesc.shape[2] &&
              ((size_t)s.height * s.width) % 2 == 0,
          "height x width must match the packed frame size");
    d.height = s.height, d.width = s.width, d.input_dtype = HF_MONO12P;
  } else {
    check(idesc.rank() == 4, "input must be [n_windows][T][H][W]");
    const std::string want = idesc.dtype == DType::U8 ? "u8" : (idesc.dtype == DType::U16 ? "u16" : "f32");
    check(idesc.dtype != DType::CF32 && s.input_format == want, "input_format does not match the input dtype");
    d.height = (int)idesc.shape[2], d.width = (int)idesc.shape[3], d.input_dtype = hf_dtype(idesc.dtype);
  }
  dp.nwin  = (int)idesc.shape[0];
  d.frames = (int)idesc.shape[1];
  d.hop    = d.frames; // windows are consecutive, non-overlapping blocks of the input
  check(dp.nwin >= 1, "expected at least one window");
  d.z_begin = s.time_z_begin, d.z_end = s.time_z_end;
  check(s.time_z_begin >= 0 && s.time_z_end > s.time_z_begin && s.time_z_end <= d.frames, "bad band [time_z_begin, time_z_end)");
  check(s.time_method == "rfft" || s.time_method == "fft", "time_method must be rfft or fft");
  d.time_method = s.time_method == "fft" ? HF_TIME_FFT : HF_TIME_RFFT;
  check((s.time_z_end - s.time_z_begin) * (d.time_method == HF_TIME_FFT ? 2 : 1) <= 64, "at most 64 band planes");
  d.clutter_rank = s.clutter_rank;
  if (s.propagation == "fresnel")
    d.propagation = HF_PROP_FRESNEL;
  else if (s.propagation == "angular_spectrum")
    d.propagation = HF_PROP_ANGULAR_SPECTRUM;
  else if (s.propagation == "none")
    d.propagation = HF_PROP_NONE;
  else
    check(false, "propagation must be fresnel, angular_spectrum or none");
  d.moment_mask = 0;
  for (const auto &m : s.moments) {
    check(m == "M0" || m == "M1" || m == "M2", "moments must be among M0, M1, M2");
    d.moment_mask |= m == "M0" ? HF_M0 : (m == "M1" ? HF_M1 : HF_M2);
  }
  check(d.moment_mask != 0, "at least one moment");
  d.fftshift = s.fftshift ? 1 : 0;
  check(s.form == "plain" || s.form == "chosen", "form must be plain or chosen");
  d.form      = s.form == "chosen" ? HF_FORM_CHOSEN : HF_FORM_PLAIN;
  d.max_batch = dp.nwin;
  d.lambda = s.lambda, d.pitch = s.dx, d.z = s.z, d.fs = s.fs;
  if (d.propagation != HF_PROP_NONE)
    check(s.lambda > 0.f && s.dx > 0.f, "wavelength and dx must be positive");
  if (s.padding) {
    check(d.propagation == HF_PROP_ANGULAR_SPECTRUM, "padding applies to angular_spectrum only");
    d.pad_w = s.padding->width, d.pad_h = s.padding->height;
  }
  if (s.filter) {
    d.as_filter = 1;
    d.r_inner = s.filter->r_inner, d.r_outer = s.filter->r_outer;
    d.s_inner = s.filter->s_inner, d.s_outer = s.filter->s_outer;
  }
  if (s.autofocus_enabled) { // graph_builder.cc:139-147, 311-334
    check(d.propagation == HF_PROP_FRESNEL, "Shack-Hartmann autofocus needs fresnel propagation");
    check(s.autofocus_nb_iter > 0, "autofocus_nb_iter must be positive");
    check(s.autofocus_nb_subaps > 0, "autofocus_nb_subaps must be positive");
    check(s.autofocus_nb_subaps % 2 == 1, "autofocus_nb_subaps must be odd");
    check(s.autofocus_zernike_orders.size() <= 9, "at most 9 autofocus_zernike_orders");
    d.autofocus_nb_subaps = s.autofocus_nb_subaps, d.autofocus_n_iter = s.autofocus_nb_iter;
    d.autofocus_n_orders  = (int)s.autofocus_zernike_orders.size();
    for (size_t i = 0; i < s.autofocus_zernike_orders.size(); ++i)
      d.autofocus_orders[i] = s.autofocus_zernike_orders[i];
    d.autofocus_roi_radius   = s.pp_pctclip_radius;
    d.autofocus_keep_outside = s.autofocus_skip_subapertures_outside_pupil ? 0 : 1;
    if (s.pp_flatfield) {
      check(s.pp_flatfield_cutoff_period_m > 0.f, "flatfield cutoff period and image pitches must be positive");
      d.autofocus_flatfield_period = s.pp_flatfield_cutoff_period_m;
    }
    // graph_builder.cc:128-146: the dual reader's delayed window with a sliding correction
    check(s.pp_accumulation > 0, "pp_accumulation must be positive");
    check(!(s.pp_accumulation > 1 && s.autofocus_nb_iter > 1),
          "sliding Shack-Hartmann correction only supports one autofocus iteration");
    d.autofocus_pp_accumulation = s.pp_accumulation;
    d.autofocus_full_pairwise   = s.autofocus_use_graph_laplacian ? 1 : 0;
  }
  dp.nmom = __builtin_popcount((unsigned)d.moment_mask);
  dp.OH   = d.pad_h ? d.pad_h : d.height;
  dp.OW   = d.pad_w ? d.pad_w : d.width;
  return dp;
}

class DopplerTask final : public ISyncTask {
public:
  hf_plan     *plan = nullptr;
  cudaStream_t stream{};
  DopplerPlan  dp;
  ~DopplerTask() override {
    if (plan)
      hf_plan_destroy(plan);
  }
  OpResult execute(SyncCtx &ctx) override {
    hf_ok(hf_pipeline_exec(plan, ctx.inputs[0].data(), (int64_t)dp.nwin * dp.d.frames, 0, dp.nwin,
                           reinterpret_cast<float *>(ctx.outputs[0].data()), stream),
          "DopplerMoments");
    return OpResult::Ok;
  }
};
} // namespace

InferResult DopplerMomentsFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"DopplerMomentsFactory"};
  const auto  s = j.get<DopplerMomentsSettings>();
  check(input_descs.size() == 1, "expected exactly one input");
  const auto dp = doppler_plan(check, input_descs[0], s);
  return sync_result(input_descs[0],
                     TDesc({(size_t)dp.nwin, (size_t)dp.nmom, (size_t)dp.OH, (size_t)dp.OW}, DType::F32, MemLoc::Device));
}

std::unique_ptr<ISyncTask> DopplerMomentsFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                         const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t    = std::make_unique<DopplerTask>();
  t->dp     = doppler_plan(Check{"DopplerMomentsFactory"}, input_descs[0], j.get<DopplerMomentsSettings>());
  t->stream = ctx.stream;
  hf_ok(hf_plan_create(&t->dp.d, &t->plan, ctx.stream), "DopplerMoments");
  return t;
}

// Same input and settings but z: rebuild the lens / transfer function only.
std::unique_ptr<ISyncTask> DopplerMomentsFactory::update(std::unique_ptr<ISyncTask> old,
                                                         std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                         const SyncCreateCtx &ctx) const {
  auto *t = dynamic_cast<DopplerTask *>(old.get());
  if (t && input_descs.size() == 1) {
    const auto dp = doppler_plan(Check{"DopplerMomentsFactory"}, input_descs[0], j.get<DopplerMomentsSettings>());
    hf_desc    a = dp.d, b = t->dp.d;
    a.z = b.z = 0.f;
    if (std::memcmp(&a, &b, sizeof(hf_desc)) == 0 && dp.nwin == t->dp.nwin) {
      if (dp.d.z != t->dp.d.z)
        hf_ok(hf_plan_set_z(t->plan, dp.d.z, ctx.stream), "DopplerMoments");
      t->dp     = dp;
      t->stream = ctx.stream;
      return old;
    }
  }
  old.reset();
  return create(input_descs, j, ctx);
}

// ================================================================================================
// Post-moment display chain: FFTShiftNp (holonp/src/fftshift.cu:185-290), Flatfield
// (holotask/src/syncs/flatfield.cu:296-453), PctClip (holotask/src/syncs/pct_clip.cu:230-333)
// ================================================================================================
void from_json(const nlohmann::json &j, FFTShiftSettings &s) {
  s.axes.clear();
  if (j.contains("axes") && !j.at("axes").is_null())
    j.at("axes").get_to(s.axes);
}
void from_json(const nlohmann::json &j, FlatfieldSettings &s) {
  j.at("sigma_y").get_to(s.sigma_y);
  j.at("sigma_x").get_to(s.sigma_x);
}
void from_json(const nlohmann::json &j, Filter2DSettings &s) {
  j.at("r_inner").get_to(s.r_inner);
  j.at("r_outer").get_to(s.r_outer);
  j.at("s_inner").get_to(s.s_inner);
  j.at("s_outer").get_to(s.s_outer);
}
void from_json(const nlohmann::json &j, PctClipSettings &s) {
  j.at("min_pct").get_to(s.min_pct);
  j.at("max_pct").get_to(s.max_pct);
  const auto &r = j.at("roi");
  r.at("cx").get_to(s.roi.cx);
  r.at("cy").get_to(s.roi.cy);
  r.at("rx").get_to(s.roi.rx);
  r.at("ry").get_to(s.roi.ry);
  r.at("angle").get_to(s.roi.angle);
}

namespace {
// The reference's FFTShift checks throw "FFTShift: <msg>" (fftshift.cu:30-34).
void shift_check(bool cond, const std::string &msg) {
  if (!cond)
    throw std::invalid_argument("FFTShift: " + msg);
}

uint32_t shift_axes_mask(const std::vector<int> &axes, int ndim) {
  if (axes.empty())
    return ndim >= 32 ? 0xFFFFFFFFu : ((1u << ndim) - 1u);
  uint32_t mask = 0;
  for (int a : axes) {
    if (a < 0)
      a += ndim;
    shift_check(a >= 0 && a < ndim, "axis out of range");
    shift_check(!(mask & (1u << a)), "axes must be unique");
    mask |= 1u << a;
  }
  return mask;
}

class FFTShiftTask final : public ISyncTask {
public:
  TDesc        idesc;
  uint32_t     mask = 0;
  cudaStream_t stream{};
  OpResult     execute(SyncCtx &ctx) override {
    std::vector<int64_t> shape(idesc.shape.begin(), idesc.shape.end());
    hf_ok(hf_fftshift(ctx.inputs[0].data(), ctx.outputs[0].data(), (int)core::size_of(idesc.dtype),
                      (int)shape.size(), shape.data(), mask, stream),
          "FFTShift");
    return OpResult::Ok;
  }
};

class FlatfieldTask final : public ISyncTask {
public:
  hf_flatfield     *ff = nullptr;
  FlatfieldSettings settings;
  TDesc             idesc;
  cudaStream_t      stream{};
  ~FlatfieldTask() override { hf_flatfield_destroy(ff); }
  OpResult execute(SyncCtx &ctx) override {
    hf_ok(hf_flatfield_exec(ff, reinterpret_cast<const float *>(ctx.inputs[0].data()),
                            reinterpret_cast<float *>(ctx.outputs[0].data()), stream),
          "Flatfield");
    return OpResult::Ok;
  }
};

class Filter2DTask final : public ISyncTask {
public:
  hf_filter2d     *f = nullptr;
  Filter2DSettings settings;
  TDesc            idesc;
  cudaStream_t     stream{};
  ~Filter2DTask() override { hf_filter2d_destroy(f); }
  OpResult execute(SyncCtx &ctx) override {
    hf_ok(hf_filter2d_exec(f, ctx.inputs[0].data(), ctx.outputs[0].data(), stream), "Filter2D");
    return OpResult::Ok;
  }
};

class PctClipTask final : public ISyncTask {
public:
  hf_pctclip     *pc = nullptr;
  PctClipSettings settings;
  TDesc           idesc;
  cudaStream_t    stream{};
  ~PctClipTask() override { hf_pctclip_destroy(pc); }
  OpResult execute(SyncCtx &ctx) override {
    hf_ok(hf_pctclip_exec(pc, reinterpret_cast<const float *>(ctx.inputs[0].data()),
                          reinterpret_cast<float *>(ctx.outputs[0].data()), nullptr, stream),
          "PctClip");
    return OpResult::Ok;
  }
};

bool same_desc(const TDesc &a, const TDesc &b) {
  return a.shape == b.shape && a.strides == b.strides && a.dtype == b.dtype && a.mem_loc == b.mem_loc &&
         a.offset == b.offset;
}
} // namespace

InferResult FFTShiftFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const auto s = j.get<FFTShiftSettings>();
  shift_check(input_descs.size() == 1, "expected exactly 1 input");
  const auto &idesc = input_descs[0];
  shift_check(idesc.mem_loc == MemLoc::Device, "only Device tensors are supported");
  shift_check(idesc.is_contiguous(), "input must be C-contiguous");
  const int ndim = (int)idesc.rank();
  shift_check(ndim > 0, "input ndim must be > 0");
  shift_check(ndim <= 16, "input ndim too large");
  (void)shift_axes_mask(s.axes, ndim);
  shift_check(idesc.num_elements() > 0, "input tensor has zero elements");
  return sync_result(idesc, idesc);
}

std::unique_ptr<ISyncTask> FFTShiftFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                   const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t    = std::make_unique<FFTShiftTask>();
  t->idesc  = input_descs[0];
  t->mask   = shift_axes_mask(j.get<FFTShiftSettings>().axes, (int)t->idesc.rank());
  t->stream = ctx.stream;
  return t;
}

std::unique_ptr<ISyncTask> FFTShiftFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> input_descs,
                                                   const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  old.reset();
  return create(input_descs, j, ctx);
}

InferResult FlatfieldFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"FlatfieldFactory"};
  const auto  s = j.get<FlatfieldSettings>();
  check(input_descs.size() == 1, "expected exactly one input");
  const auto &idesc = input_descs[0];
  check(idesc.rank() >= 2, "input must be a tensor of rank 2 or higher");
  check(idesc.dtype == DType::F32, "input must be float32");
  check(idesc.mem_loc == MemLoc::Device, "input must be in device memory");
  check(idesc.is_contiguous(), "input must be C-contiguous");
  check(idesc.num_elements() > 0, "input must not be empty");
  check(s.sigma_y > 0.0f, "sigma_y must be positive");
  check(s.sigma_x > 0.0f, "sigma_x must be positive");
  return sync_result(idesc, idesc);
}

std::unique_ptr<ISyncTask> FlatfieldFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                    const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t      = std::make_unique<FlatfieldTask>();
  t->settings = j.get<FlatfieldSettings>();
  t->idesc    = input_descs[0];
  t->stream   = ctx.stream;
  const size_t r = t->idesc.rank();
  int64_t      planes = 1;
  for (size_t i = 0; i + 2 < r; ++i)
    planes *= (int64_t)t->idesc.shape[i];
  const int rc = hf_flatfield_create(planes, (int)t->idesc.shape[r - 2], (int)t->idesc.shape[r - 1],
                                     t->settings.sigma_y, t->settings.sigma_x, ctx.stream, &t->ff);
  if (rc == HF_ERR_INVALID) // sigma too small for a kernel: the reference's inference error
    Check{"FlatfieldFactory"}(false, "sigma is too small to form a Gaussian kernel");
  hf_ok(rc, "Flatfield");
  return t;
}

std::unique_ptr<ISyncTask> FlatfieldFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> input_descs,
                                                    const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto *t = dynamic_cast<FlatfieldTask *>(old.get());
  if (t && t->settings.sigma_y == j.get<FlatfieldSettings>().sigma_y &&
      t->settings.sigma_x == j.get<FlatfieldSettings>().sigma_x && same_desc(t->idesc, input_descs[0])) {
    t->stream = ctx.stream;
    return old;
  }
  old.reset();
  return create(input_descs, j, ctx);
}

// filter2d.cu:262-297: the same checks; complex input is filtered in place
InferResult Filter2DFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"Filter2DFactory"};
  (void)j.get<Filter2DSettings>();
  check(input_descs.size() == 1, "expected exactly one input");
  const auto &idesc = input_descs[0];
  check(idesc.rank() >= 2, "input must be a tensor of rank 2 or higher");
  check(idesc.dtype == DType::CF32 || idesc.dtype == DType::F32, "input must be complex float32 or real float32");
  check(idesc.mem_loc == MemLoc::Device, "input must be in device memory");
  check(idesc.is_contiguous(), "input must be C-contiguous");
  std::vector<core::InPlace> in_place;
  if (idesc.dtype == DType::CF32)
    in_place.push_back({0, 0});
  return sync_result(idesc, idesc, std::move(in_place));
}

std::unique_ptr<ISyncTask> Filter2DFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                   const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t      = std::make_unique<Filter2DTask>();
  t->settings = j.get<Filter2DSettings>();
  t->idesc    = input_descs[0];
  t->stream   = ctx.stream;
  const size_t r = t->idesc.rank();
  int64_t      planes = 1;
  for (size_t i = 0; i + 2 < r; ++i)
    planes *= (int64_t)t->idesc.shape[i];
  const auto &s = t->settings;
  hf_ok(hf_filter2d_create(planes, (int)t->idesc.shape[r - 2], (int)t->idesc.shape[r - 1],
                           t->idesc.dtype == DType::F32 ? 1 : 0, s.r_inner, s.r_outer, s.s_inner, s.s_outer, ctx.stream,
                           &t->f),
        "Filter2D");
  return t;
}

std::unique_ptr<ISyncTask> Filter2DFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> input_descs,
                                                   const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto *t = dynamic_cast<Filter2DTask *>(old.get());
  if (t && t->settings == j.get<Filter2DSettings>() && same_desc(t->idesc, input_descs[0])) {
    t->stream = ctx.stream;
    return old;
  }
  old.reset();
  return create(input_descs, j, ctx);
}

InferResult PctClipFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"PctClipFactory"};
  const auto  s = j.get<PctClipSettings>();
  check(s.min_pct >= 0.0f, "min_pct must be >= 0");
  check(s.min_pct <= 100.0f, "min_pct must be <= 100");
  check(s.max_pct >= 0.0f, "max_pct must be >= 0");
  check(s.max_pct <= 100.0f, "max_pct must be <= 100");
  check(s.min_pct < s.max_pct, "min_pct must be < max_pct");
  check(s.roi.rx > 0.0f, "roi.rx must be > 0");
  check(s.roi.rx <= 1.0f, "roi.rx must be <= 1");
  check(s.roi.ry > 0.0f, "roi.ry must be > 0");
  check(s.roi.ry <= 1.0f, "roi.ry must be <= 1");
  check(s.roi.cx >= 0.0f, "roi.cx must be >= 0");
  check(s.roi.cx <= 1.0f, "roi.cx must be <= 1");
  check(s.roi.cy >= 0.0f, "roi.cy must be >= 0");
  check(s.roi.cy <= 1.0f, "roi.cy must be <= 1");
  check(input_descs.size() == 1, "expected exactly one input");
  const auto &idesc = input_descs[0];
  check(idesc.dtype == DType::F32, "input must be float32");
  check(idesc.rank() == 3, "input must be 3D");
  check(idesc.mem_loc == MemLoc::Device, "input must be in device memory");
  check(idesc.is_contiguous(), "input must be C-contiguous");
  return sync_result(idesc, idesc);
}

std::unique_ptr<ISyncTask> PctClipFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                  const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t      = std::make_unique<PctClipTask>();
  t->settings = j.get<PctClipSettings>();
  t->idesc    = input_descs[0];
  t->stream   = ctx.stream;
  const hf_ellipse roi{t->settings.roi.cx, t->settings.roi.cy, t->settings.roi.rx, t->settings.roi.ry,
                       t->settings.roi.angle};
  hf_ok(hf_pctclip_create((int)t->idesc.shape[0], (int)t->idesc.shape[1], (int)t->idesc.shape[2],
                          t->settings.min_pct, t->settings.max_pct, &roi, ctx.stream, &t->pc),
        "PctClip");
  return t;
}

std::unique_ptr<ISyncTask> PctClipFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> input_descs,
                                                  const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto *t = dynamic_cast<PctClipTask *>(old.get());
  if (t && t->settings == j.get<PctClipSettings>() && same_desc(t->idesc, input_descs[0])) {
    t->stream = ctx.stream;
    return old;
  }
  old.reset();
  return create(input_descs, j, ctx);
}

// ================================================================================================
// Shack-Hartmann autofocus: ShortTimeFresnelDiffraction (short_time_fresnel_diffraction.cu:604-840),
// ShackHartmannSlopes (shack_hartmann_slopes.cu:326-440), ZernikeFromSlopes
// (zernike_from_slopes.cc:283-377), ZernikePhase (zernike_phase.cu:270-363), CorrectPhase
// (correct_phase.cu:160-226), Wrap2Pi (wrap2pi.cu), ZernikeDefocusZProp (zernike_defocus_z_prop.cc)
// ================================================================================================
namespace {
void read_indexes(const nlohmann::json &j, std::vector<int> &v) {
  v.clear();
  if (j.contains("indexes"))
    j.at("indexes").get_to(v);
  else if (j.contains("indices"))
    j.at("indices").get_to(v);
}
void read_ellipse(const nlohmann::json &j, PctClipSettings::Ellipse &e) {
  if (j.contains("cx"))
    j.at("cx").get_to(e.cx);
  if (j.contains("cy"))
    j.at("cy").get_to(e.cy);
  if (j.contains("rx"))
    j.at("rx").get_to(e.rx);
  if (j.contains("ry"))
    j.at("ry").get_to(e.ry);
  if (j.contains("angle"))
    j.at("angle").get_to(e.angle);
}
core::MemLoc read_memloc(const nlohmann::json &j) {
  const std::string v = j.get<std::string>();
  if (v == "Host")
    return core::MemLoc::Host;
  if (v == "Device")
    return core::MemLoc::Device;
  throw std::invalid_argument("invalid MemLoc string");
}
} // namespace

void from_json(const nlohmann::json &j, ShortTimeFresnelDiffractionSettings &s) {
  j.at("lambda").get_to(s.lambda);
  j.at("dx").get_to(s.dx);
  j.at("dy").get_to(s.dy);
  j.at("z").get_to(s.z);
  j.at("win_h").get_to(s.win_h);
  j.at("win_w").get_to(s.win_w);
  j.at("stride_y").get_to(s.stride_y);
  j.at("stride_x").get_to(s.stride_x);
  if (j.contains("phase_ref"))
    j.at("phase_ref").get_to(s.phase_ref);
  if (s.phase_ref != "LOCAL" && s.phase_ref != "GLOBAL")
    throw std::invalid_argument("ShortTimeFresnelDiffraction: unknown phase_ref " + s.phase_ref);
  if (j.contains("skip_phase_shift"))
    j.at("skip_phase_shift").get_to(s.skip_phase_shift);
  if (j.contains("output_magnitude"))
    j.at("output_magnitude").get_to(s.output_magnitude);
  if (j.contains("axes"))
    j.at("axes").get_to(s.axes);
}
void from_json(const nlohmann::json &j, ShackHartmannSlopeSettings &s) {
  s.mode = j.value("mode", std::string("single_reference"));
  if (s.mode != "single_reference" && s.mode != "full_pairwise")
    throw std::invalid_argument("Unknown Shack-Hartmann slope mode: " + s.mode);
  j.at("lambda").get_to(s.lambda);
  j.at("dx").get_to(s.dx);
  j.at("dy").get_to(s.dy);
  j.at("z").get_to(s.z);
  j.at("subaperture_height").get_to(s.subaperture_height);
  j.at("subaperture_width").get_to(s.subaperture_width);
  j.at("stride_y").get_to(s.stride_y);
  j.at("stride_x").get_to(s.stride_x);
  if (j.contains("correlation_roi"))
    read_ellipse(j.at("correlation_roi"), s.correlation_roi);
  s.skip_subapertures_outside_pupil = j.value("skip_subapertures_outside_pupil", true);
  s.output_xcorr_maps               = j.value("output_xcorr_maps", false);
  s.pair_batch_size                 = j.value("pair_batch_size", size_t{256});
}
void from_json(const nlohmann::json &j, ZernikeFromSlopesSettings &s) {
  read_indexes(j, s.indexes);
  j.at("lambda").get_to(s.lambda);
  j.at("dx").get_to(s.dx);
  j.at("dy").get_to(s.dy);
  j.at("subaperture_height").get_to(s.subaperture_height);
  j.at("subaperture_width").get_to(s.subaperture_width);
  j.at("stride_y").get_to(s.stride_y);
  j.at("stride_x").get_to(s.stride_x);
  s.ny                              = j.value("ny", size_t{1});
  s.nx                              = j.value("nx", size_t{1});
  s.skip_subapertures_outside_pupil = j.value("skip_subapertures_outside_pupil", true);
}
void from_json(const nlohmann::json &j, ZernikePhaseSettings &s) {
  read_indexes(j, s.indexes);
  j.at("ny").get_to(s.ny);
  j.at("nx").get_to(s.nx);
  if (j.contains("output"))
    s.output = read_memloc(j.at("output"));
  else if (j.contains("device"))
    s.output = read_memloc(j.at("device"));
  else
    s.output = core::MemLoc::Host;
}
void from_json(const nlohmann::json &j, ZernikeDefocusZPropSettings &s) {
  read_indexes(j, s.indexes);
  j.at("lambda").get_to(s.lambda);
  j.at("z_curr").get_to(s.z_curr);
  j.at("pupil_radius").get_to(s.pupil_radius);
}

namespace {
void check_noll(const Check &check, const std::vector<int> &idx) {
  check(!idx.empty(), "indexes must not be empty");
  check(idx.size() <= 9, "too many requested Zernike modes");
  for (int v : idx)
    check(v >= 2 && v <= 10, "only Noll indexes 2..10 are supported");
  auto u = idx;
  std::sort(u.begin(), u.end());
  check(std::adjacent_find(u.begin(), u.end()) == u.end(), "indexes must be unique");
}

class ShortTimeFresnelTask final : public ISyncTask {
public:
  hf_stfd                            *f = nullptr;
  ShortTimeFresnelDiffractionSettings settings;
  TDesc                               idesc;
  cudaStream_t                        stream{};
  ~ShortTimeFresnelTask() override { hf_stfd_destroy(f); }
  OpResult execute(SyncCtx &ctx) override {
    hf_ok(hf_stfd_exec(f, ctx.inputs[0].data(), ctx.outputs[0].data(), stream), "ShortTimeFresnelDiffraction");
    return OpResult::Ok;
  }
};

class ShackHartmannSlopesTask final : public ISyncTask {
public:
  hf_shslopes               *p = nullptr;
  ShackHartmannSlopeSettings settings;
  TDesc                      idesc;
  cudaStream_t               stream{};
  ~ShackHartmannSlopesTask() override { hf_shslopes_destroy(p); }
  OpResult execute(SyncCtx &ctx) override {
    float *maps = settings.output_xcorr_maps ? reinterpret_cast<float *>(ctx.outputs[1].data()) : nullptr;
    hf_ok(hf_shslopes_exec(p, reinterpret_cast<const float *>(ctx.inputs[0].data()),
                           reinterpret_cast<float *>(ctx.outputs[0].data()), maps, stream),
          "ShackHartmannSlopes");
    return OpResult::Ok;
  }
};

class ZernikeFromSlopesTask final : public ISyncTask {
public:
  hf_zernike_fit           *f = nullptr;
  ZernikeFromSlopesSettings settings;
  TDesc                     idesc;
  cudaStream_t              stream{};
  ~ZernikeFromSlopesTask() override { hf_zernike_fit_destroy(f); }
  OpResult execute(SyncCtx &ctx) override {
    const auto *in  = reinterpret_cast<const float *>(ctx.inputs[0].data());
    auto       *out = reinterpret_cast<float *>(ctx.outputs[0].data());
    if (idesc.mem_loc == MemLoc::Host) { // the reference's host fit, after the producer's stream
      if (cudaStreamSynchronize(stream) != cudaSuccess)
        throw std::runtime_error("ZernikeFromSlopes: stream synchronisation failed");
      hf_ok(hf_zernike_fit_host(f, in, out), "ZernikeFromSlopes");
    } else {
      hf_ok(hf_zernike_fit_exec(f, in, out, nullptr, stream), "ZernikeFromSlopes");
    }
    return OpResult::Ok;
  }
};

float zernike_value_host(int noll, float x, float y) { // eval_zernike_noll_value (zernike_phase.cu:88-113)
  const float s3 = std::sqrt(3.0f), s6 = std::sqrt(6.0f), s8 = std::sqrt(8.0f);
  switch (noll) {
  case 2: return 2.0f * x;
  case 3: return 2.0f * y;
  case 4: return s3 * (2.0f * (x * x + y * y) - 1.0f);
  case 5: return 2.0f * s6 * x * y;
  case 6: return s6 * (x * x - y * y);
  case 7: return s8 * y * (3.0f * x * x - y * y);
  case 8: return s8 * y * (3.0f * x * x + 3.0f * y * y - 2.0f);
  case 9: return s8 * x * (3.0f * x * x + 3.0f * y * y - 2.0f);
  default: return s8 * x * (x * x - 3.0f * y * y);
  }
}

class ZernikePhaseTask final : public ISyncTask {
public:
  ZernikePhaseSettings settings;
  cudaStream_t         stream{};
  OpResult             execute(SyncCtx &ctx) override {
    const auto *c   = reinterpret_cast<const float *>(ctx.inputs[0].data());
    auto       *out = reinterpret_cast<float *>(ctx.outputs[0].data());
    const int   ny = settings.ny, nx = settings.nx;
    if (settings.output == MemLoc::Device) {
      hf_ok(hf_zernike_phase(c, settings.indexes.data(), (int)settings.indexes.size(), ny, nx, out, nullptr, stream),
            "ZernikePhase");
      return OpResult::Ok;
    }
    const float cy = ((float)ny - 1.0f) * 0.5f, cx = ((float)nx - 1.0f) * 0.5f;
    const float r  = 0.5f * (float)std::min(ny, nx);
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const float xn = ((float)x - cx) / r, yn = ((float)y - cy) / r;
        float       ph = 0.f;
        for (size_t i = 0; i < settings.indexes.size(); ++i)
          ph += c[i] * zernike_value_host(settings.indexes[i], xn, yn);
        out[(size_t)y * nx + x] = ph;
      }
    return OpResult::Ok;
  }
};

class CorrectPhaseTask final : public ISyncTask {
public:
  TDesc        idesc;
  cudaStream_t stream{};
  OpResult     execute(SyncCtx &ctx) override {
    const size_t r      = idesc.rank();
    int64_t      planes = 1;
    for (size_t i = 0; i + 2 < r; ++i)
      planes *= (int64_t)idesc.shape[i];
    hf_ok(hf_correct_phase(ctx.inputs[0].data(), idesc.dtype == DType::CF32 ? 1 : 0,
                           reinterpret_cast<const float *>(ctx.inputs[1].data()), planes, (int)idesc.shape[r - 2],
                           (int)idesc.shape[r - 1], ctx.outputs[0].data(), stream),
          "CorrectPhase");
    return OpResult::Ok;
  }
};

class Wrap2PiTask final : public ISyncTask {
public:
  TDesc        idesc;
  cudaStream_t stream{};
  OpResult     execute(SyncCtx &ctx) override {
    hf_ok(hf_wrap2pi(reinterpret_cast<const float *>(ctx.inputs[0].data()), reinterpret_cast<float *>(ctx.outputs[0].data()),
                     (int64_t)idesc.num_elements(), stream),
          "Wrap2Pi");
    return OpResult::Ok;
  }
};

class ZernikeDefocusZPropTask final : public ISyncTask {
public:
  ZernikeDefocusZPropSettings settings;
  TDesc                       idesc;
  cudaStream_t                stream{};
  double                      estimate[3] = {0.0, 0.0, 0.0}; // delta 1/z, new z, delta z (mm)
  bool                        valid       = false;
  OpResult                    execute(SyncCtx &ctx) override {
    const size_t pos = (size_t)(std::find(settings.indexes.begin(), settings.indexes.end(), 4) - settings.indexes.begin());
    const float *src = reinterpret_cast<const float *>(ctx.inputs[0].data()) + pos;
    float        a4  = 0.f;
    if (idesc.mem_loc == MemLoc::Device) {
      if (cudaMemcpyAsync(&a4, src, sizeof(float), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
          cudaStreamSynchronize(stream) != cudaSuccess)
        throw std::runtime_error("ZernikeDefocusZProp: copy of the defocus coefficient failed");
    } else {
      a4 = *src;
    }
    // an undefined estimate leaves the previous one in place (the reference only logs it)
    valid = hf_defocus_z(a4, settings.lambda, settings.z_curr, settings.pupil_radius, &estimate[0], &estimate[1],
                         &estimate[2]) == HF_OK;
    return OpResult::Ok;
  }
};

int64_t leading_planes(const TDesc &d) {
  int64_t p = 1;
  for (size_t i = 0; i + 2 < d.rank(); ++i)
    p *= (int64_t)d.shape[i];
  return p;
}
} // namespace

InferResult ShortTimeFresnelDiffractionFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"ShortTimeFresnelDiffractionFactory"};
  const auto  s = j.get<ShortTimeFresnelDiffractionSettings>();
  check(input_descs.size() == 1, "expected exactly one input");
  const auto &id = input_descs[0];
  check(id.rank() >= 2, "input must be rank >= 2");
  check(id.dtype == DType::CF32 || id.dtype == DType::F32, "input must be CF32 or F32");
  check(id.mem_loc == MemLoc::Device, "input must be on device");
  check(id.is_contiguous(), "input must be C-contiguous");
  check(s.lambda > 0.f, "lambda must be positive");
  check(s.dx > 0.f, "dx must be positive");
  check(s.dy > 0.f, "dy must be positive");
  check(s.dx == s.dy, "dx must equal dy");
  check(s.z != 0.f, "z must be non-zero");
  check(s.win_h >= 1 && s.win_w >= 1, "window dimensions must be >= 1");
  check(s.stride_y >= 1 && s.stride_x >= 1, "strides must be >= 1");
  const int rank = (int)id.rank();
  check(s.axes.size() == 2 || s.axes.empty(), "axes must contain exactly two elements");
  if (s.axes.size() == 2) {
    const int a0 = s.axes[0] < 0 ? s.axes[0] + rank : s.axes[0], a1 = s.axes[1] < 0 ? s.axes[1] + rank : s.axes[1];
    check(a0 >= 0 && a0 < rank && a1 >= 0 && a1 < rank, "axes out of bounds");
    check(a0 != a1, "axes must be distinct");
    check(a0 == rank - 2 && a1 == rank - 1, "only trailing axes (-2, -1) are supported");
  }
  const size_t H = id.shape[rank - 2], W = id.shape[rank - 1];
  check(s.win_h <= H && s.win_w <= W, "window dimensions exceed field size");
  std::vector<size_t> shape(id.shape.begin(), id.shape.end() - 2);
  shape.push_back((H - s.win_h) / s.stride_y + 1);
  shape.push_back((W - s.win_w) / s.stride_x + 1);
  shape.push_back(s.win_h);
  shape.push_back(s.win_w);
  return sync_result(id, TDesc(shape, s.output_magnitude ? DType::F32 : DType::CF32, MemLoc::Device));
}

std::unique_ptr<ISyncTask> ShortTimeFresnelDiffractionFactory::create(std::span<const TDesc> input_descs,
                                                                      const nlohmann::json &j,
                                                                      const SyncCreateCtx  &ctx) const {
  (void)infer(input_descs, j);
  auto t      = std::make_unique<ShortTimeFresnelTask>();
  t->settings = j.get<ShortTimeFresnelDiffractionSettings>();
  t->idesc    = input_descs[0];
  t->stream   = ctx.stream;
  const auto  &s = t->settings;
  const size_t r = t->idesc.rank();
  hf_ok(hf_stfd_create(leading_planes(t->idesc), (int)t->idesc.shape[r - 2], (int)t->idesc.shape[r - 1],
                       t->idesc.dtype == DType::F32 ? 1 : 0, (int)s.win_h, (int)s.win_w, (int)s.stride_y,
                       (int)s.stride_x, s.lambda, s.dx, s.dy, s.z, s.phase_ref == "GLOBAL" ? HF_STFD_GLOBAL : HF_STFD_LOCAL,
                       s.output_magnitude ? HF_STFD_MAGNITUDE : HF_STFD_COMPLEX, s.skip_phase_shift ? 1 : 0, 0,
                       ctx.stream, &t->f),
        "ShortTimeFresnelDiffraction");
  return t;
}

// update: the same task for the same settings, the lenses rebuilt when only z changed (:780-840)
std::unique_ptr<ISyncTask> ShortTimeFresnelDiffractionFactory::update(std::unique_ptr<ISyncTask> old,
                                                                      std::span<const TDesc> input_descs,
                                                                      const nlohmann::json &j,
                                                                      const SyncCreateCtx  &ctx) const {
  (void)infer(input_descs, j);
  auto *t = dynamic_cast<ShortTimeFresnelTask *>(old.get());
  if (t && same_desc(t->idesc, input_descs[0])) {
    auto s = j.get<ShortTimeFresnelDiffractionSettings>();
    if (s == t->settings) {
      t->stream = ctx.stream;
      return old;
    }
    auto z_only = s;
    z_only.z    = t->settings.z;
    if (z_only == t->settings) {
      hf_ok(hf_stfd_set_z(t->f, s.z, ctx.stream), "ShortTimeFresnelDiffraction");
      t->settings = s, t->stream = ctx.stream;
      return old;
    }
  }
  old.reset();
  return create(input_descs, j, ctx);
}

InferResult ShackHartmannSlopesFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"ShackHartmannSlopesFactory"};
  const auto  s = j.get<ShackHartmannSlopeSettings>();
  check(input_descs.size() == 1, "task must have exactly one input");
  const auto &in = input_descs[0];
  check(in.mem_loc == MemLoc::Device, "input memory location must be Device");
  check(in.dtype == DType::F32, "input dtype must be F32");
  check(in.rank() == 5, "input rank must be 5");
  check(in.shape[0] == 1, "only batch size 1 is supported");
  check(in.shape[1] > 0 && in.shape[2] > 0, "subaperture grid dimensions must be positive");
  if (s.mode == "single_reference")
    check(in.shape[1] % 2 == 1 && in.shape[2] % 2 == 1,
          "subaperture grid dimensions must be odd for an unambiguous center reference");
  check(in.shape[3] >= 2 && in.shape[4] >= 2, "reconstruction dimensions must be at least 2");
  check(s.lambda > 0.f, "wavelength must be > 0");
  check(s.dx > 0.f && s.dy > 0.f, "pixel pitches must be > 0");
  check(s.z > 0.f, "propagation distance must be > 0");
  check(s.subaperture_height > 0 && s.subaperture_width > 0, "subaperture dimensions must be positive");
  check(s.stride_y > 0 && s.stride_x > 0, "strides must be positive");
  check(s.correlation_roi.rx > 0.f && s.correlation_roi.ry > 0.f, "correlation ROI radii must be positive");
  check(s.pair_batch_size > 0, "pair_batch_size must be positive");
  check(!(s.mode == "full_pairwise" && s.output_xcorr_maps), "FullPairwise correlation-map output is not supported");
  if (s.mode == "full_pairwise")
    check(in.shape[1] * in.shape[2] >= 2, "FullPairwise mode requires at least two active subapertures");
  std::vector<TDesc> outs{TDesc({1, in.shape[1], in.shape[2], 2}, DType::F32, MemLoc::Device)};
  if (s.output_xcorr_maps)
    outs.emplace_back(in.shape, DType::F32, MemLoc::Device);
  InferResult r = sync_result(in, outs[0]);
  r.output_descs  = outs;
  r.owned_outputs = std::vector<bool>(outs.size(), false);
  return r;
}

std::unique_ptr<ISyncTask> ShackHartmannSlopesFactory::create(std::span<const TDesc> input_descs,
                                                              const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t      = std::make_unique<ShackHartmannSlopesTask>();
  t->settings = j.get<ShackHartmannSlopeSettings>();
  t->idesc    = input_descs[0];
  t->stream   = ctx.stream;
  const auto      &s = t->settings;
  const hf_ellipse roi{s.correlation_roi.cx, s.correlation_roi.cy, s.correlation_roi.rx, s.correlation_roi.ry,
                       s.correlation_roi.angle};
  // FullPairwise: the complete-graph recovery (shack_hartmann_slopes_full_pairwise.cuh); the
  // active-count check ("requires at least two active subapertures") runs at create, where the
  // pupil geometry is built
  hf_ok(hf_shslopes_create_mode((int)t->idesc.shape[1], (int)t->idesc.shape[2], (int)t->idesc.shape[3],
                                (int)t->idesc.shape[4], (int)s.subaperture_height, (int)s.subaperture_width,
                                (int)s.stride_y, (int)s.stride_x, s.lambda, s.dx, s.dy, s.z, &roi,
                                s.skip_subapertures_outside_pupil ? 1 : 0,
                                s.mode == "full_pairwise" ? HF_SHSLOPES_FULL_PAIRWISE : HF_SHSLOPES_SINGLE_REFERENCE,
                                (int)s.pair_batch_size, ctx.stream, &t->p),
        "ShackHartmannSlopes");
  return t;
}

std::unique_ptr<ISyncTask> ShackHartmannSlopesFactory::update(std::unique_ptr<ISyncTask> old,
                                                              std::span<const TDesc> input_descs,
                                                              const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto *t = dynamic_cast<ShackHartmannSlopesTask *>(old.get());
  if (t && t->settings == j.get<ShackHartmannSlopeSettings>() && same_desc(t->idesc, input_descs[0])) {
    t->stream = ctx.stream;
    return old;
  }
  old.reset();
  return create(input_descs, j, ctx);
}

InferResult ZernikeFromSlopesFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"ZernikeFromSlopesFactory"};
  const auto  s = j.get<ZernikeFromSlopesSettings>();
  check(input_descs.size() == 1, "task must have exactly one input");
  const auto &in = input_descs[0];
  check(in.dtype == DType::F32, "input dtype must be F32");
  check(in.rank() == 4, "input rank must be 4");
  check(in.shape[0] == 1, "only batch size 1 is supported");
  check(in.shape[1] > 0 && in.shape[2] > 0, "subaperture grid dimensions must be positive");
  check(in.shape[3] == 2, "last input dimension must contain [dW/dx, dW/dy]");
  check(in.is_contiguous(), "input must be C-contiguous");
  check(s.lambda > 0.f, "wavelength must be > 0");
  check(s.dx > 0.f && s.dy > 0.f, "pixel pitches must be > 0");
  check(s.subaperture_height > 0 && s.subaperture_width > 0, "subaperture dimensions must be positive");
  check(s.stride_y > 0 && s.stride_x > 0, "strides must be positive");
  check(s.ny == 1 && s.nx == 1, "only global fitting with ny = nx = 1 is supported for zero-mean slopes");
  check_noll(check, s.indexes);
  return sync_result(in, TDesc({1, 1, s.indexes.size()}, DType::F32, in.mem_loc));
}

std::unique_ptr<ISyncTask> ZernikeFromSlopesFactory::create(std::span<const TDesc> input_descs,
                                                            const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t      = std::make_unique<ZernikeFromSlopesTask>();
  t->settings = j.get<ZernikeFromSlopesSettings>();
  t->idesc    = input_descs[0];
  t->stream   = ctx.stream;
  const auto &s = t->settings;
  hf_ok(hf_zernike_fit_create((int)t->idesc.shape[1], (int)t->idesc.shape[2], (int)s.subaperture_height,
                              (int)s.subaperture_width, (int)s.stride_y, (int)s.stride_x, s.lambda, s.dx, s.dy,
                              s.skip_subapertures_outside_pupil ? 1 : 0, s.indexes.data(), (int)s.indexes.size(), &t->f),
        "ZernikeFromSlopesFactory");
  return t;
}

std::unique_ptr<ISyncTask> ZernikeFromSlopesFactory::update(std::unique_ptr<ISyncTask> old,
                                                            std::span<const TDesc> input_descs,
                                                            const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto *t = dynamic_cast<ZernikeFromSlopesTask *>(old.get());
  if (t && t->settings == j.get<ZernikeFromSlopesSettings>() && same_desc(t->idesc, input_descs[0])) {
    t->stream = ctx.stream;
    return old;
  }
  old.reset();
  return create(input_descs, j, ctx);
}

InferResult ZernikePhaseFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"ZernikePhaseFactory"};
  const auto  s = j.get<ZernikePhaseSettings>();
  check(input_descs.size() == 1, "ZernikePhase task must have exactly one input");
  const auto &in = input_descs[0];
  check(in.mem_loc == s.output, "Input coefficients must be in the output memory location");
  check(in.dtype == DType::F32, "Input coefficients dtype must be F32");
  check(in.rank() == 1, "Input coefficients rank must be 1");
  check(in.is_contiguous(), "Input coefficients must be C-contiguous");
  check(!s.indexes.empty(), "indexes must not be empty");
  check(s.indexes.size() <= 9, "Too many requested Zernike modes");
  for (int v : s.indexes)
    check(v >= 2 && v <= 10, "Only zernike Noll indexes 2..10 are supported");
  auto u = s.indexes;
  std::sort(u.begin(), u.end());
  check(std::adjacent_find(u.begin(), u.end()) == u.end(), "indexes must be unique");
  check(s.ny > 0 && s.nx > 0, "Resolution ny and nx must be greater than 0");
  check(in.shape[0] == s.indexes.size(), "Input coefficient count must match settings.indexes size");
  return sync_result(in, TDesc({(size_t)s.ny, (size_t)s.nx}, DType::F32, s.output));
}

std::unique_ptr<ISyncTask> ZernikePhaseFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                       const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t      = std::make_unique<ZernikePhaseTask>();
  t->settings = j.get<ZernikePhaseSettings>();
  t->stream   = ctx.stream;
  return t;
}

std::unique_ptr<ISyncTask> ZernikePhaseFactory::update(std::unique_ptr<ISyncTask> old,
                                                       std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                       const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto *t = dynamic_cast<ZernikePhaseTask *>(old.get());
  if (t && t->settings == j.get<ZernikePhaseSettings>()) {
    t->stream = ctx.stream;
    return old;
  }
  old.reset();
  return create(input_descs, j, ctx);
}

InferResult CorrectPhaseFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &) const {
  const Check check{"CorrectPhaseFactory"};
  check(input_descs.size() == 2, "expected exactly two inputs");
  const auto &id = input_descs[0], &md = input_descs[1];
  check(id.mem_loc == MemLoc::Device, "input must be in device memory");
  check(md.mem_loc == MemLoc::Device, "phase mask must be in device memory");
  check(id.dtype == DType::F32 || id.dtype == DType::CF32, "input dtype must be F32 or CF32");
  check(md.dtype == DType::F32, "phase mask dtype must be F32");
  check(id.rank() >= 2, "input rank must be at least 2");
  check(md.rank() >= 2, "phase mask rank must be at least 2");
  check(id.shape[id.rank() - 2] == md.shape[md.rank() - 2], "phase mask height must match the input");
  check(id.shape[id.rank() - 1] == md.shape[md.rank() - 1], "phase mask width must match the input");
  check(id.is_contiguous() && md.is_contiguous(), "inputs must be C-contiguous");
  size_t mask_planes = 1;
  for (size_t i = 0; i + 2 < md.rank(); ++i)
    mask_planes *= md.shape[i];
  check(mask_planes == 1, "the phase mask must be one [H, W] plane");
  InferResult r = sync_result(id, TDesc(id.shape, DType::CF32, MemLoc::Device));
  r.input_descs  = {id, md};
  r.owned_inputs = {false, false};
  return r;
}

std::unique_ptr<ISyncTask> CorrectPhaseFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                       const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t    = std::make_unique<CorrectPhaseTask>();
  t->idesc  = input_descs[0];
  t->stream = ctx.stream;
  return t;
}

std::unique_ptr<ISyncTask> CorrectPhaseFactory::update(std::unique_ptr<ISyncTask> old,
                                                       std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                       const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto *t = dynamic_cast<CorrectPhaseTask *>(old.get());
  if (t && same_desc(t->idesc, input_descs[0])) {
    t->stream = ctx.stream;
    return old;
  }
  old.reset();
  return create(input_descs, j, ctx);
}

InferResult Wrap2PiFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &) const {
  const Check check{"Wrap2PiFactory"};
  check(input_descs.size() == 1, "expected exactly one input");
  const auto &id = input_descs[0];
  check(id.mem_loc == MemLoc::Device, "input must be in device memory");
  check(id.dtype == DType::F32, "input dtype must be F32");
  check(id.is_contiguous(), "input must be C-contiguous");
  return sync_result(id, id, {{0, 0}});
}

std::unique_ptr<ISyncTask> Wrap2PiFactory::create(std::span<const TDesc> input_descs, const nlohmann::json &j,
                                                  const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t    = std::make_unique<Wrap2PiTask>();
  t->idesc  = input_descs[0];
  t->stream = ctx.stream;
  return t;
}

std::unique_ptr<ISyncTask> Wrap2PiFactory::update(std::unique_ptr<ISyncTask> old, std::span<const TDesc> input_descs,
                                                  const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto *t = dynamic_cast<Wrap2PiTask *>(old.get());
  if (t && same_desc(t->idesc, input_descs[0])) {
    t->stream = ctx.stream;
    return old;
  }
  old.reset();
  return create(input_descs, j, ctx);
}

InferResult ZernikeDefocusZPropFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"ZernikeDefocusZPropFactory"};
  const auto  s = j.get<ZernikeDefocusZPropSettings>();
  check(s.lambda > 0.f, "lambda must be positive");
  check(s.z_curr != 0.f, "z_curr must be non-zero");
  check(s.pupil_radius > 0.f, "pupil_radius must be positive");
  check(!s.indexes.empty(), "indexes must not be empty");
  check(std::find(s.indexes.begin(), s.indexes.end(), 4) != s.indexes.end(), "indexes must contain Z4 defocus");
  auto u = s.indexes;
  std::sort(u.begin(), u.end());
  check(std::adjacent_find(u.begin(), u.end()) == u.end(), "indexes must be unique");
  check(input_descs.size() == 1, "ZernikeDefocusZProp task must have exactly one input");
  const auto &id = input_descs[0];
  check(id.dtype == DType::F32, "Input coefficients dtype must be F32");
  check(id.rank() == 1, "Input coefficients rank must be 1");
  check(id.is_contiguous(), "Input coefficients must be C-contiguous");
  check(id.shape[0] == s.indexes.size(), "Input coefficient count must match settings.indexes size");
  InferResult r = sync_result(id, id);
  r.output_descs.clear();
  r.owned_outputs.clear();
  return r;
}

std::unique_ptr<ISyncTask> ZernikeDefocusZPropFactory::create(std::span<const TDesc> input_descs,
                                                              const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto t      = std::make_unique<ZernikeDefocusZPropTask>();
  t->settings = j.get<ZernikeDefocusZPropSettings>();
  t->idesc    = input_descs[0];
  t->stream   = ctx.stream;
  return t;
}

std::unique_ptr<ISyncTask> ZernikeDefocusZPropFactory::update(std::unique_ptr<ISyncTask> old,
                                                              std::span<const TDesc> input_descs,
                                                              const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  (void)infer(input_descs, j);
  auto *t = dynamic_cast<ZernikeDefocusZPropTask *>(old.get());
  if (t && t->settings == j.get<ZernikeDefocusZPropSettings>() && same_desc(t->idesc, input_descs[0])) {
    t->stream = ctx.stream;
    return old;
  }
  old.reset();
  return create(input_descs, j, ctx);
}

// ================================================================================================
// registry
// ================================================================================================
void register_path_kinds(core::Registry &r) {
  r.register_sync("FresnelDiffraction", std::make_unique<FresnelDiffractionFactory>());
  r.register_sync("AngularSpectrum", std::make_unique<AngularSpectrumFactory>());
  r.register_sync("Pca", std::make_unique<PcaFactory>());
  r.register_sync("FFT", std::make_unique<FFTFactory>());
  r.register_sync("RFFT", std::make_unique<RFFTFactory>());
  r.register_sync("Mean", std::make_unique<MeanFactory>());
  r.register_sync("MeanAbs", std::make_unique<MeanAbsFactory>());
  r.register_sync("Conversion", std::make_unique<ConversionFactory>());
  r.register_sync("DopplerMoments", std::make_unique<DopplerMomentsFactory>());
  r.register_sync("Holofile", std::make_unique<HolofileFactory>());
  r.register_sync("FFTShiftNp", std::make_unique<FFTShiftFactory>());
  r.register_sync("Flatfield", std::make_unique<FlatfieldFactory>());
  r.register_sync("Filter2D", std::make_unique<Filter2DFactory>());
  r.register_sync("PctClip", std::make_unique<PctClipFactory>());
  r.register_sync("ShortTimeFresnelDiffraction", std::make_unique<ShortTimeFresnelDiffractionFactory>());
  r.register_sync("ShackHartmannSlopes", std::make_unique<ShackHartmannSlopesFactory>());
  r.register_sync("ZernikeFromSlopes", std::make_unique<ZernikeFromSlopesFactory>());
  r.register_sync("ZernikePhase", std::make_unique<ZernikePhaseFactory>());
  r.register_sync("CorrectPhase", std::make_unique<CorrectPhaseFactory>());
  r.register_sync("Wrap2Pi", std::make_unique<Wrap2PiFactory>());
  r.register_sync("ZernikeDefocusZProp", std::make_unique<ZernikeDefocusZPropFactory>());
}

core::Registry &default_registry() {
  static core::Registry *reg = [] {
    auto *r = new core::Registry();
    register_path_kinds(*r);
    register_np_kinds(*r);
    return r;
  }();
  return *reg;
}

} // namespace hfb::nodes
