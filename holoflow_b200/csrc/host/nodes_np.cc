// The thin node kinds GraphBuilder wires around the path's compute stages, restated so that the
// node graph the reference builds for one window loads against this registry node by node:
//   synchronous  : Slice (a view), Reshape (a view, or a copy), Copy, Concatenate, Arange,
//                  Multiply (broadcasting), Abs, CausalSlidingAverage
//                  (holonp/src/{slice,reshape,copy,concatenate,arange,multiply,abs}.cu;
//                  holotask/src/syncs/causal_sliding_average.cu);
//   asynchronous : BatchQueue, DualReaderBatchQueue, SlidingAverage
//                  (holotask/src/asyncs/{batch_queue,dual_reader_batch_queue}.cc, slide_avg.cu).
// Settings keys, inference checks and messages follow the reference's; the element work runs in
// this library's kernels (k_np.cu) on the stream given at create().  The queues are host-side
// control over device (or host) rings: the producer writes into the view acquire_input returns,
// try_push publishes it, try_pop hands out zero-copy views and release_output retires them.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <variant>

#include "hf_common.cuh"
#include "holoflow_b200.h"
#include "holoflow_b200/nodes.hh"
#include "k_np.cuh"

namespace hfb::nodes {

using core::AsyncCreateCtx;
using core::AsyncPopCtx;
using core::AsyncPushCtx;
using core::DType;
using core::IAsyncTask;
using core::IAsyncTaskFactory;
using core::MemLoc;
using core::OpResult;
using core::Storage;
using core::SyncCtx;
using core::TView;

namespace {

struct Check { // "<Factory> inference error: <message>" (the holotask factories' form)
  const char *factory;
  void        operator()(bool cond, const std::string &msg) const {
    if (!cond)
      throw std::invalid_argument(std::string(factory) + " inference error: " + msg);
  }
};

struct Fail { // "<Prefix>: <message>" (the holonp ops' message form)
  const char *prefix;
  void        operator()(bool cond, const std::string &msg) const {
    if (!cond)
      throw std::invalid_argument(std::string(prefix) + msg);
  }
};

void cuda_ok(int rc, const char *who) {
  if (rc == HF_OK)
    return;
  const std::string msg = std::string(who) + ": " + hf_last_error();
  if (rc == HF_ERR_INVALID || rc == HF_ERR_UNSUPPORTED)
    throw std::invalid_argument(msg);
  throw core::CudaError(msg);
}

void cuda_ok(cudaError_t e, const char *who) {
  if (e != cudaSuccess)
    throw core::CudaError(std::string(who) + ": " + cudaGetErrorString(e));
}

InferResult sync_io(std::vector<TDesc> in, std::vector<TDesc> out) {
  InferResult r;
  r.input_descs   = std::move(in);
  r.output_descs  = std::move(out);
  r.owned_inputs  = std::vector<bool>(r.input_descs.size(), false);
  r.owned_outputs = std::vector<bool>(r.output_descs.size(), false);
  r.kind          = core::TaskKind::Sync;
  return r;
}

hf::NpLayout layout_copy(const TDesc &src, const TDesc &dst) {
  hf::NpLayout l;
  l.rank = (int)src.rank();
  for (int d = 0; d < l.rank; ++d) {
    l.shape[d]       = (int64_t)src.shape[(size_t)d];
    l.src_strides[d] = (int64_t)src.strides[(size_t)d];
    l.dst_strides[d] = (int64_t)dst.strides[(size_t)d];
  }
  return l;
}

// A task with no work of its own (views: the output aliases the input's storage).
class NoOpTask final : public ISyncTask {
public:
  OpResult execute(SyncCtx &) override { return OpResult::Ok; }
};

// A strided copy of input 0 into the contiguous output 0.
class CopyTask final : public ISyncTask {
public:
  TDesc        in, out;
  cudaStream_t stream{};
  OpResult     execute(SyncCtx &ctx) override {
    cuda_ok(hf::launch_copy_strided(ctx.inputs[0].data(), ctx.outputs[0].data(), layout_copy(in, out),
                                        (int)core::size_of(in.dtype), stream),
                "Copy");
    return OpResult::Ok;
  }
};

// ---- Slice ------------------------------------------------------------------------------------
struct SliceRange {
  std::optional<int64_t> start, stop;
  int64_t                step = 1;
};
using SliceItem = std::variant<SliceRange, int64_t>;

std::vector<SliceItem> parse_slices(const nlohmann::json &j) {
  std::vector<SliceItem> v;
  for (const auto &e : j.at("slices")) {
    if (e.is_number_integer()) {
      v.emplace_back(e.get<int64_t>());
    } else {
      SliceRange r;
      if (e.contains("start") && !e.at("start").is_null())
        r.start = e.at("start").get<int64_t>();
      if (e.contains("stop") && !e.at("stop").is_null())
        r.stop = e.at("stop").get<int64_t>();
      r.step = e.value("step", (int64_t)1);
      v.emplace_back(r);
    }
  }
  return v;
}

} // namespace

// Slice (holonp/src/slice.cu:185-250): numpy basic indexing as a strided view of the input
// (in place: input 0 -> output 0, no copy).  An integer item drops its dimension.
InferResult SliceFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Fail check{"Slice: "};
  const auto items = parse_slices(j);
  check(input_descs.size() == 1, "expected exactly 1 input");
  const TDesc &in   = input_descs[0];
  const int    ndim = (int)in.rank();
  check(ndim > 0, "input ndim must be > 0");
  check(ndim <= hf::kNpMaxRank, "input ndim too large");
  check((int)items.size() == ndim, "number of slice items must match input ndim");
  std::vector<size_t> shape, strides;
  size_t              offset = in.offset;
  for (int d = 0; d < ndim; ++d) {
    const int64_t dim = (int64_t)in.shape[(size_t)d];
    const size_t  st  = in.strides[(size_t)d];
    if (std::holds_alternative<int64_t>(items[(size_t)d])) {
      check(dim > 0, "cannot index into 0-sized dimension");
      int64_t idx = std::get<int64_t>(items[(size_t)d]);
      if (idx < 0)
        idx += dim;
      check(idx >= 0 && idx < dim, "index out of range");
      offset += (size_t)idx * st;
      continue;
    }
    const SliceRange &r = std::get<SliceRange>(items[(size_t)d]);
    check(r.step > 0, "only positive step is supported for now");
    auto clamp = [&](std::optional<int64_t> v, int64_t dflt) {
      if (!v)
        return dflt;
      int64_t x = *v < 0 ? *v + dim : *v;
      return std::clamp<int64_t>(x, 0, dim);
    };
    const int64_t a = clamp(r.start, 0), b = clamp(r.stop, dim);
    const int64_t n = b > a ? (b - a + r.step - 1) / r.step : 0;
    offset += (size_t)a * st;
    shape.push_back((size_t)n);
    strides.push_back(st * (size_t)r.step);
  }
  InferResult res = sync_io({in}, {TDesc(shape, in.dtype, in.mem_loc, strides, offset)});
  res.in_place    = {core::InPlace{0, 0}};
  return res;
}
std::unique_ptr<ISyncTask> SliceFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                                const SyncCreateCtx &) const {
  (void)infer(in, j);
  return std::make_unique<NoOpTask>();
}
std::unique_ptr<ISyncTask> SliceFactory::update(std::unique_ptr<ISyncTask>, std::span<const TDesc> in,
                                                const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  return create(in, j, ctx);
}

// ---- Reshape (holonp/src/reshape.cu) ------------------------------------------------------------
namespace {
std::vector<size_t> reshape_target(const TDesc &in, const std::vector<int64_t> &req) {
  const size_t total = in.num_elements();
  int          neg   = -1;
  size_t       known = 1;
  for (size_t i = 0; i < req.size(); ++i) {
    if (req[i] == -1) {
      if (neg >= 0)
        throw std::invalid_argument("Reshape: Only one dimension can be -1");
      neg = (int)i;
    } else if (req[i] < 0) {
      throw std::invalid_argument("Reshape: Dimensions cannot be negative (except -1)");
    } else {
      known *= (size_t)req[i];
    }
  }
  std::vector<size_t> out(req.begin(), req.end());
  if (neg >= 0) {
    if (known == 0 || total % known != 0)
      throw std::invalid_argument("Reshape: Total elements must be divisible by known dimensions");
    out[(size_t)neg] = total / known;
  }
  size_t n = 1;
  for (size_t v : out)
    n *= v;
  if (n != total)
    throw std::invalid_argument("Reshape: Total elements mismatch between input and target shape");
  return out;
}

// Strides of `shape` viewing the same elements as `in` without a copy, if there are any: every run
// of dimensions merged or split must be contiguous in the input.
std::optional<std::vector<size_t>> view_strides(const TDesc &in, const std::vector<size_t> &shape) {
  std::vector<size_t> os, ost; // input without size-1 dimensions
  for (size_t i = 0; i < in.rank(); ++i)
    if (in.shape[i] != 1)
      os.push_back(in.shape[i]), ost.push_back(in.strides[i]);
  std::vector<size_t> st(shape.size(), 0);
  size_t              oi = 0, ni = 0;
  const size_t        es = core::size_of(in.dtype);
  while (ni < shape.size()) {
    if (shape[ni] == 1) { // any stride for a size-1 dimension
      st[ni] = ni + 1 < shape.size() ? 0 : es;
      ++ni;
      continue;
    }
    if (oi >= os.size())
      return std::nullopt;
    // grow an input chunk and a new chunk until their element counts agree
    size_t a = os[oi], b = shape[ni];
    size_t o_end = oi + 1, n_end = ni + 1;
    while (a != b) {
      if (a < b) {
        if (o_end >= os.size())
          return std::nullopt;
        a *= os[o_end++];
      } else {
        while (n_end < shape.size() && shape[n_end] == 1)
          ++n_end;
        if (n_end >= shape.size())
          return std::nullopt;
        b *= shape[n_end++];
      }
    }
    for (size_t k = oi; k + 1 < o_end; ++k) // the input chunk must be contiguous
      if (ost[k] != os[k + 1] * ost[k + 1])
        return std::nullopt;
    size_t cur = ost[o_end - 1];
    for (size_t k = n_end; k-- > ni;) {
      st[k] = cur;
      cur *= shape[k];
    }
    oi = o_end, ni = n_end;
  }
  if (oi != os.size())
    return std::nullopt;
  for (size_t k = 0; k < shape.size(); ++k) // size-1 dimensions: the stride of what follows
    if (shape[k] == 1)
      st[k] = k + 1 < shape.size() ? st[k + 1] * shape[k + 1] : es;
  return st;
}

class ReshapeCopyTask final : public ISyncTask {
public:
  TDesc        in, out; // `out` is the input's shape with contiguous strides (the copy's layout)
  cudaStream_t stream{};
  OpResult     execute(SyncCtx &ctx) override {
    cuda_ok(hf::launch_copy_strided(ctx.inputs[0].data(), ctx.outputs[0].data(), layout_copy(in, out),
                                        (int)core::size_of(in.dtype), stream),
                "Reshape");
    return OpResult::Ok;
  }
};
} // namespace

InferResult ReshapeFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  if (input_descs.size() != 1)
    throw std::invalid_argument("Reshape: expected exactly 1 input");
  const TDesc &in    = input_descs[0];
  const auto   shape = reshape_target(in, j.at("shape").get<std::vector<int64_t>>());
  const bool   force = j.contains("copy") && !j.at("copy").is_null() && j.at("copy").get<bool>();
  const auto   view  = force ? std::nullopt : view_strides(in, shape);
  if (j.contains("copy") && !j.at("copy").is_null() && !j.at("copy").get<bool>() && !view)
    throw std::invalid_argument("Reshape: a view is not possible for this input layout (copy=false)");
  if (view) {
    InferResult r = sync_io({in}, {TDesc(shape, in.dtype, in.mem_loc, *view, in.offset)});
    r.in_place    = {core::InPlace{0, 0}};
    return r;
  }
  if (in.mem_loc != MemLoc::Device)
    throw std::invalid_argument("Reshape: a copying reshape needs a Device tensor");
  return sync_io({in}, {TDesc(shape, in.dtype, in.mem_loc)});
}
std::unique_ptr<ISyncTask> ReshapeFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                                  const SyncCreateCtx &ctx) const {
  const auto r = infer(in, j);
  if (!r.in_place.empty())
    return std::make_unique<NoOpTask>();
  auto t    = std::make_unique<ReshapeCopyTask>();
  t->in     = in[0];
  t->out    = TDesc(in[0].shape, in[0].dtype, in[0].mem_loc);
  t->stream = ctx.stream;
  return t;
}
std::unique_ptr<ISyncTask> ReshapeFactory::update(std::unique_ptr<ISyncTask>, std::span<const TDesc> in,
                                                  const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  return create(in, j, ctx);
}

// ---- Copy (holonp/src/copy.cu): a contiguous copy of a (possibly strided) Device tensor ---------
InferResult CopyFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &) const {
  const Fail check{"Copy: "};
  check(input_descs.size() == 1, "expected exactly 1 input");
  const TDesc &in = input_descs[0];
  check(in.mem_loc == MemLoc::Device, "only Device tensors are supported");
  check(in.rank() <= (size_t)hf::kNpMaxRank, "input ndim too large");
  return sync_io({in}, {TDesc(in.shape, in.dtype, in.mem_loc)});
}
std::unique_ptr<ISyncTask> CopyFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                               const SyncCreateCtx &ctx) const {
  const auto r = infer(in, j);
  auto       t = std::make_unique<CopyTask>();
  t->in = in[0], t->out = r.output_descs[0], t->stream = ctx.stream;
  return t;
}
std::unique_ptr<ISyncTask> CopyFactory::update(std::unique_ptr<ISyncTask>, std::span<const TDesc> in,
                                               const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  return create(in, j, ctx);
}

// ---- Concatenate (holonp/src/concatenate.cu) ---------------------------------------------------
namespace {
class ConcatTask final : public ISyncTask {
public:
  std::vector<TDesc> in;
  TDesc              out;
  int                axis = 0;
  cudaStream_t       stream{};
  OpResult           execute(SyncCtx &ctx) override {
    size_t at = 0;
    for (size_t i = 0; i < in.size(); ++i) { // each input into its slab of the output
      hf::NpLayout l = layout_copy(in[i], out);
      cuda_ok(hf::launch_copy_strided(ctx.inputs[i].data(), ctx.outputs[0].data() + at * out.strides[(size_t)axis], l,
                                      (int)core::size_of(out.dtype), stream),
              "Concatenate");
      at += in[i].shape[(size_t)axis];
    }
    return OpResult::Ok;
  }
};
} // namespace

InferResult ConcatenateFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Fail check{"Concatenate: "};
  check(!input_descs.empty(), "expected at least 1 input");
  const TDesc &a = input_descs[0];
  check(a.mem_loc == MemLoc::Device, "only Device tensors are supported");
  const int ndim = (int)a.rank();
  check(ndim > 0, "input ndim must be > 0");
  check(ndim <= hf::kNpMaxRank, "input ndim too large");
  int axis = 0;
  if (j.contains("axis") && !j.at("axis").is_null()) {
    check(j.at("axis").is_number_integer(), "axis must be int or null");
    axis = j.at("axis").get<int>();
  }
  if (axis < 0)
    axis += ndim;
  check(axis >= 0 && axis < ndim, "axis out of range");
  std::vector<size_t> shape = a.shape;
  shape[(size_t)axis]       = 0;
  for (const TDesc &d : input_descs) {
    check(d.mem_loc == a.mem_loc, "all inputs must share the same mem_loc");
    check(d.dtype == a.dtype, "all inputs must share the same dtype");
    check((int)d.rank() == ndim, "all inputs must share the same rank");
    for (int i = 0; i < ndim; ++i)
      if (i != axis)
        check(d.shape[(size_t)i] == a.shape[(size_t)i], "input shapes must match except along the axis");
    shape[(size_t)axis] += d.shape[(size_t)axis];
  }
  return sync_io(std::vector<TDesc>(input_descs.begin(), input_descs.end()), {TDesc(shape, a.dtype, a.mem_loc)});
}
std::unique_ptr<ISyncTask> ConcatenateFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                                      const SyncCreateCtx &ctx) const {
  const auto r = infer(in, j);
  auto       t = std::make_unique<ConcatTask>();
  t->in.assign(in.begin(), in.end());
  t->out  = r.output_descs[0];
  int ax  = j.contains("axis") && !j.at("axis").is_null() ? j.at("axis").get<int>() : 0;
  t->axis = ax < 0 ? ax + (int)in[0].rank() : ax;
  t->stream = ctx.stream;
  return t;
}
std::unique_ptr<ISyncTask> ConcatenateFactory::update(std::unique_ptr<ISyncTask>, std::span<const TDesc> in,
                                                      const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  return create(in, j, ctx);
}

// ---- Arange (holonp/src/arange.cu): [n] float32 on the device, start + step i in double --------
namespace {
struct ArangeArgs {
  double start = 0.0, stop = 1.0, step = 1.0;
};
ArangeArgs arange_args(const nlohmann::json &j) {
  ArangeArgs a;
  a.start = j.value("start", 0.0), a.stop = j.value("stop", 1.0), a.step = j.value("step", 1.0);
  return a;
}
int64_t arange_len(const ArangeArgs &a) {
  if ((a.step > 0 && a.stop <= a.start) || (a.step < 0 && a.stop >= a.start))
    return 0;
  const double n = std::ceil((a.stop - a.start) / a.step);
  if (!std::isfinite(n) || n <= 0)
    throw std::invalid_argument("Arange: invalid resulting length");
  if (n > 9.0e15)
    throw std::invalid_argument("Arange: resulting length too large");
  return (int64_t)n;
}
class ArangeTask final : public ISyncTask {
public:
  ArangeArgs   a;
  int64_t      n = 0;
  cudaStream_t stream{};
  OpResult     execute(SyncCtx &ctx) override {
    cuda_ok(hf::launch_arange(reinterpret_cast<float *>(ctx.outputs[0].data()), a.start, a.step, n, stream), "Arange");
    return OpResult::Ok;
  }
};
} // namespace

InferResult ArangeFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"ArangeFactory"};
  check(input_descs.empty(), "expected zero inputs");
  if (j.contains("device") && !j.at("device").is_null())
    check(j.at("device").get<std::string>() == "Device", "only Device output is supported (for now)");
  if (j.contains("dtype") && !j.at("dtype").is_null())
    check(j.at("dtype").get<std::string>() == "F32", "only F32 output is supported");
  const ArangeArgs a = arange_args(j);
  check(a.step != 0.0, "step must be non-zero");
  return sync_io({}, {TDesc({(size_t)arange_len(a)}, DType::F32, MemLoc::Device)});
}
std::unique_ptr<ISyncTask> ArangeFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                                 const SyncCreateCtx &ctx) const {
  (void)infer(in, j);
  auto t = std::make_unique<ArangeTask>();
  t->a = arange_args(j), t->n = arange_len(t->a), t->stream = ctx.stream;
  return t;
}
std::unique_ptr<ISyncTask> ArangeFactory::update(std::unique_ptr<ISyncTask>, std::span<const TDesc> in,
                                                 const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  return create(in, j, ctx);
}

// ---- Multiply (holonp/src/multiply.cu): numpy broadcasting, F32 / CF32 ---------------------------
namespace {
class MultiplyTask final : public ISyncTask {
public:
  hf::NpBroadcast l;
  int             a_cplx = 0, b_cplx = 0;
  cudaStream_t    stream{};
  OpResult        execute(SyncCtx &ctx) override {
    cuda_ok(hf::launch_multiply(ctx.inputs[0].data(), a_cplx, ctx.inputs[1].data(), b_cplx, ctx.outputs[0].data(), l,
                                stream),
            "Multiply");
    return OpResult::Ok;
  }
};
std::vector<size_t> broadcast_shape(const TDesc &a, const TDesc &b, const Fail &check) {
  const size_t        r = std::max(a.rank(), b.rank());
  std::vector<size_t> s(r);
  for (size_t i = 0; i < r; ++i) {
    const size_t da = i < r - a.rank() ? 1 : a.shape[i - (r - a.rank())];
    const size_t db = i < r - b.rank() ? 1 : b.shape[i - (r - b.rank())];
    check(da == db || da == 1 || db == 1, "input shapes are not broadcastable");
    s[i] = std::max(da, db);
  }
  return s;
}
} // namespace

InferResult MultiplyFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &) const {
  const Fail check{"Multiply: "};
  check(input_descs.size() == 2, "expected exactly 2 input tensors");
  const TDesc &a = input_descs[0], &b = input_descs[1];
  check(a.mem_loc == MemLoc::Device, "input 0 must be in device memory");
  check(b.mem_loc == MemLoc::Device, "input 1 must be in device memory");
  check((a.dtype == DType::F32 || a.dtype == DType::CF32) && (b.dtype == DType::F32 || b.dtype == DType::CF32),
        "only F32 and CF32 operands are supported");
  const auto shape = broadcast_shape(a, b, check);
  check(shape.size() <= (size_t)hf::kNpMaxRank, "input ndim too large");
  const DType o = (a.dtype == DType::CF32 || b.dtype == DType::CF32) ? DType::CF32 : DType::F32;
  return sync_io({a, b}, {TDesc(shape, o, MemLoc::Device)});
}
std::unique_ptr<ISyncTask> MultiplyFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                                   const SyncCreateCtx &ctx) const {
  const auto r = infer(in, j);
  auto       t = std::make_unique<MultiplyTask>();
  const auto &shape = r.output_descs[0].shape;
  t->l.rank         = (int)shape.size();
  for (int k = 0; k < 2; ++k) {
    const TDesc &d  = in[(size_t)k];
    const size_t es = core::size_of(d.dtype);
    for (size_t i = 0; i < shape.size(); ++i) {
      const size_t off = shape.size() - d.rank();
      const int64_t st = i < off || d.shape[i - off] == 1 ? 0 : (int64_t)(d.strides[i - off] / es);
      (k == 0 ? t->l.a_strides : t->l.b_strides)[i] = st;
    }
  }
  for (size_t i = 0; i < shape.size(); ++i)
    t->l.shape[i] = (int64_t)shape[i];
  t->a_cplx = in[0].dtype == DType::CF32, t->b_cplx = in[1].dtype == DType::CF32, t->stream = ctx.stream;
  return t;
}
std::unique_ptr<ISyncTask> MultiplyFactory::update(std::unique_ptr<ISyncTask>, std::span<const TDesc> in,
                                                   const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  return create(in, j, ctx);
}

// ---- Abs (holonp/src/abs.cu): contiguous Device tensor; CF32 -> F32, real dtypes keep theirs ----
namespace {
class AbsTask final : public ISyncTask {
public:
  TDesc        in;
  cudaStream_t stream{};
  OpResult     execute(SyncCtx &ctx) override {
    const int64_t n = (int64_t)in.num_elements();
    if (in.dtype == DType::CF32 || in.dtype == DType::F32)
      cuda_ok(hf::launch_abs(ctx.inputs[0].data(), in.dtype == DType::CF32 ? HF_CF32 : HF_F32,
                             reinterpret_cast<float *>(ctx.outputs[0].data()), n, stream),
              "Abs");
    else // unsigned values are their own magnitude
      cuda_ok(cudaMemcpyAsync(ctx.outputs[0].data(), ctx.inputs[0].data(), in.num_bytes(), cudaMemcpyDeviceToDevice,
                              stream),
              "Abs");
    return OpResult::Ok;
  }
};
} // namespace

InferResult AbsFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &) const {
  const Fail check{"Abs: "};
  check(input_descs.size() == 1, "expected exactly 1 input");
  const TDesc &in = input_descs[0];
  check(in.mem_loc == MemLoc::Device, "only Device tensors are supported");
  check(in.num_elements() > 0, "input tensor has zero elements");
  check(in.is_contiguous(), "input tensor must be contiguous");
  const DType o = in.dtype == DType::CF32 ? DType::F32 : in.dtype;
  return sync_io({in}, {TDesc(in.shape, o, MemLoc::Device)});
}
std::unique_ptr<ISyncTask> AbsFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                              const SyncCreateCtx &ctx) const {
  (void)infer(in, j);
  auto t = std::make_unique<AbsTask>();
  t->in = in[0], t->stream = ctx.stream;
  return t;
}
std::unique_ptr<ISyncTask> AbsFactory::update(std::unique_ptr<ISyncTask>, std::span<const TDesc> in,
                                              const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  return create(in, j, ctx);
}

// ---- CausalSlidingAverage (causal_sliding_average.cu:35-170) ---------------------------------------
namespace {
class CausalAvgTask final : public ISyncTask {
public:
  size_t       window = 1, count = 0;
  int64_t      n      = 0;
  float       *hist = nullptr, *sum = nullptr;
  cudaStream_t stream{};
  ~CausalAvgTask() override {
    cudaFree(hist);
    cudaFree(sum);
  }
  OpResult execute(SyncCtx &ctx) override {
    const size_t slot = count % window;
    const float  div  = (float)std::min(count + 1, window);
    cuda_ok(hf::launch_causal_avg(reinterpret_cast<const float *>(ctx.inputs[0].data()),
                                  reinterpret_cast<float *>(ctx.outputs[0].data()), hist + (int64_t)slot * n, sum, n, div,
                                  stream),
            "CausalSlidingAverage");
    ++count;
    return OpResult::Ok;
  }
};
} // namespace

InferResult CausalSlidingAverageFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"CausalSlidingAverageFactory"};
  const size_t window = j.at("window_size").get<size_t>();
  check(input_descs.size() == 1, "task must have exactly one input");
  const TDesc &in = input_descs[0];
  check(in.dtype == DType::F32, "input dtype must be F32");
  check(in.mem_loc == MemLoc::Device, "input must be in device memory");
  check(in.rank() > 0, "input rank must be positive");
  check(in.is_contiguous(), "input must be contiguous");
  check(window > 0, "window_size must be positive");
  return sync_io({in}, {in});
}
std::unique_ptr<ISyncTask> CausalSlidingAverageFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                                               const SyncCreateCtx &ctx) const {
  (void)infer(in, j);
  auto t    = std::make_unique<CausalAvgTask>();
  t->window = j.at("window_size").get<size_t>();
  t->n      = (int64_t)in[0].num_elements();
  t->stream = ctx.stream;
  cuda_ok(cudaMalloc(&t->hist, t->window * (size_t)t->n * sizeof(float)), "CausalSlidingAverage");
  cuda_ok(cudaMalloc(&t->sum, (size_t)t->n * sizeof(float)), "CausalSlidingAverage");
  cuda_ok(cudaMemsetAsync(t->hist, 0, t->window * (size_t)t->n * sizeof(float), ctx.stream), "CausalSlidingAverage");
  cuda_ok(cudaMemsetAsync(t->sum, 0, (size_t)t->n * sizeof(float), ctx.stream), "CausalSlidingAverage");
  return t;
}
std::unique_ptr<ISyncTask> CausalSlidingAverageFactory::update(std::unique_ptr<ISyncTask>, std::span<const TDesc> in,
                                                               const nlohmann::json &j, const SyncCreateCtx &ctx) const {
  return create(in, j, ctx);
}

// =================================================================================================
// Asynchronous queues
// =================================================================================================
namespace {

// A ring of `slots` elements of `elem` bytes in device (or pinned host) memory.
struct Ring {
  std::byte *buf    = nullptr;
  bool       device = true;
  size_t     slots = 0, elem = 0;
  ~Ring() {
    if (buf)
      device ? (void)cudaFree(buf) : (void)cudaFreeHost(buf);
  }
  void alloc(MemLoc loc, size_t nslots, size_t elem_bytes) {
    device = loc == MemLoc::Device, slots = nslots, elem = elem_bytes;
    void *p = nullptr;
    cuda_ok(device ? cudaMalloc(&p, slots * elem) : cudaMallocHost(&p, slots * elem), "queue ring");
    buf = static_cast<std::byte *>(p);
  }
  std::byte *at(size_t i) const { return buf + i * elem; }
  size_t     dist(size_t from, size_t to) const { return to >= from ? to - from : to + slots - from; }
};

// BatchQueue (batch_queue.cc:92-239): pushes of `in` elements, pops of windows of output_size
// elements every output_stride elements, each a zero-copy view into the ring (the ring size is a
// multiple of both the push and the stride, so no window wraps).
class BatchQueueTask final : public IAsyncTask {
public:
  size_t in_n = 0, out_size = 0, stride = 0;
  TDesc  idesc, odesc;
  Ring   ring;
  size_t write = 0, read = 0;
  std::optional<TView> acquire_input(int index) override {
    if (index != 0)
      throw std::out_of_range("BatchQueue::acquire_input: invalid index");
    if (ring.slots - ring.dist(read, write) <= in_n)
      return std::nullopt;
    Storage &st = storage_access().owned_input_storage(0);
    st.ptr      = ring.at(write);
    return TView{idesc, &st};
  }
  void release_output(int index) override {
    if (index != 0)
      throw std::out_of_range("BatchQueue::release_output: invalid index");
    read = read + stride == ring.slots ? 0 : read + stride;
    storage_access().owned_output_storage(0).ptr = nullptr;
  }
  OpResult try_push(AsyncPushCtx &) override {
    write = write + in_n >= ring.slots ? 0 : write + in_n;
    storage_access().owned_input_storage(0).ptr = nullptr;
    return OpResult::Ok;
  }
  OpResult try_pop(AsyncPopCtx &ctx) override {
    if (ring.dist(read, write) < stride)
      return OpResult::NotReady;
    Storage &st    = storage_access().owned_output_storage(0);
    st.ptr         = ring.at(read);
    ctx.outputs[0] = TView{odesc, &st};
    return OpResult::Ok;
  }
};

// DualReaderBatchQueue (dual_reader_batch_queue.cc:66-227): pushes of `in` elements, pops of ONE
// element as two views -- the current element and the one `delay` = (window_size - 1) / 2 pops
// earlier (a zero element until the stream has that many) -- and a host U8 flag that is 1 once
// window_size - 1 elements have been popped before this one.
class DualReaderTask final : public IAsyncTask {
public:
  size_t     in_n = 0, delay = 0, window = 1, seq = 0;
  TDesc      idesc, odesc;
  Ring       ring;
  std::byte *zero = nullptr; // one zero element (device or host, as the ring)
  size_t     write = 0, cur = 0, del = 0;
  bool       active = false, del_active = false, cur_rel = false, del_rel = false;
  ~DualReaderTask() override {
    if (zero)
      ring.device ? (void)cudaFree(zero) : (void)cudaFreeHost(zero);
  }
  size_t inc(size_t i) const { return i + 1 == ring.slots ? 0 : i + 1; }
  std::optional<TView> acquire_input(int index) override {
    if (index != 0)
      throw std::out_of_range("DualReaderBatchQueue::acquire_input: invalid index");
    if (ring.slots - ring.dist(del, write) <= in_n) // the delayed reader holds the oldest slot
      return std::nullopt;
    Storage &st = storage_access().owned_input_storage(0);
    st.ptr      = ring.at(write);
    return TView{idesc, &st};
  }
  void release_output(int index) override {
    if (index != 0 && index != 1)
      throw std::out_of_range("DualReaderBatchQueue::release_output: invalid index");
    if (!active)
      throw std::logic_error("DualReaderBatchQueue::release_output: no active output");
    storage_access().owned_output_storage((size_t)index).ptr = nullptr;
    (index == 0 ? cur_rel : del_rel) = true;
    if (!cur_rel || !del_rel)
      return;
    cur = inc(cur);
    if (del_active)
      del = inc(del);
    ++seq;
    active = false;
  }
  OpResult try_push(AsyncPushCtx &) override {
    size_t next = write + in_n;
    write       = next >= ring.slots ? 0 : next;
    storage_access().owned_input_storage(0).ptr = nullptr;
    return OpResult::Ok;
  }
  OpResult try_pop(AsyncPopCtx &ctx) override {
    if (ring.dist(cur, write) < 1)
      return OpResult::NotReady;
    if (active)
      throw std::logic_error("DualReaderBatchQueue::try_pop: prior output was not released");
    Storage &c = storage_access().owned_output_storage(0);
    Storage &d = storage_access().owned_output_storage(1);
    c.ptr      = ring.at(cur);
    del_active = seq >= delay;
    d.ptr      = del_active ? ring.at(del) : zero;
    ctx.outputs[0] = TView{odesc, &c};
    ctx.outputs[1] = TView{odesc, &d};
    *reinterpret_cast<uint8_t *>(ctx.outputs[2].data()) = seq >= window - 1 ? 1 : 0;
    cur_rel = del_rel = false;
    active            = true;
    return OpResult::Ok;
  }
};

// SlidingAverage (holotask/src/asyncs/slide_avg.cu): one image [1, H, W] F32 per push, a float32
// running average over the last window_size images (the first discard_first dropped); a pop hands
// out the average once window_size images have entered, one pop per push after that.
class SlidingAverageTask final : public IAsyncTask {
public:
  TDesc        idesc;
  hf_slideavg *sa    = nullptr;
  float       *slot  = nullptr, *avg = nullptr;
  bool         avail = false, popped = false;
  cudaStream_t stream{};
  ~SlidingAverageTask() override {
    hf_slideavg_destroy(sa);
    cudaFree(slot);
    cudaFree(avg);
  }
  std::optional<TView> acquire_input(int index) override {
    if (index != 0)
      throw std::out_of_range("SlidingAverage::acquire_input: invalid index");
    if (avail) // the last average has not been taken yet
      return std::nullopt;
    Storage &st = storage_access().owned_input_storage(0);
    st.ptr      = reinterpret_cast<std::byte *>(slot);
    return TView{idesc, &st};
  }
  void release_output(int index) override {
    if (index != 0)
      throw std::out_of_range("SlidingAverage::release_output: invalid index");
    storage_access().owned_output_storage(0).ptr = nullptr;
    popped = false;
  }
  OpResult try_push(AsyncPushCtx &) override {
    int ready = 0;
    cuda_ok(hf_slideavg_push(sa, slot, avg, &ready, stream), "SlidingAverage");
    storage_access().owned_input_storage(0).ptr = nullptr;
    avail = ready != 0;
    return OpResult::Ok;
  }
  OpResult try_pop(AsyncPopCtx &ctx) override {
    if (!avail || popped)
      return OpResult::NotReady;
    Storage &st    = storage_access().owned_output_storage(0);
    st.ptr         = reinterpret_cast<std::byte *>(avg);
    ctx.outputs[0] = TView{idesc, &st};
    avail = false, popped = true;
    return OpResult::Ok;
  }
};

size_t lcm_above(size_t x, size_t y, size_t minimum) {
  const size_t base = std::lcm(x, y);
  if (base == 0)
    throw std::overflow_error("queue: capacity alignment overflow");
  return (minimum + base - 1) / base * base;
}

InferResult async_io(std::vector<TDesc> in, std::vector<TDesc> out, std::vector<bool> owned_out) {
  InferResult r;
  r.input_descs   = std::move(in);
  r.output_descs  = std::move(out);
  r.owned_inputs  = std::vector<bool>(r.input_descs.size(), true);
  r.owned_outputs = std::move(owned_out);
  r.kind          = core::TaskKind::Async;
  return r;
}

} // namespace

InferResult BatchQueueFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"BatchQueueFactory"};
  const size_t cap = j.at("target_capacity").get<size_t>(), size = j.at("output_size").get<size_t>(),
               stride = j.at("output_stride").get<size_t>();
  check(input_descs.size() == 1, "BatchQueue task must have exactly one input");
  check(input_descs[0].rank() > 0, "BatchQueue task input must have rank > 0");
  check(input_descs[0].is_contiguous(), "BatchQueue task input must be contiguous");
  check(cap > 0, "BatchQueue task target capacity must be > 0");
  check(size > 0, "BatchQueue task output size must be > 0");
  check(stride > 0, "BatchQueue task output stride must be > 0");
  check(stride % size == 0, "BatchQueue task output stride must be a multiple of output size");
  TDesc o    = input_descs[0];
  o.shape[0] = size;
  return async_io({input_descs[0]}, {TDesc(o.shape, o.dtype, o.mem_loc)}, {true});
}
std::unique_ptr<IAsyncTask> BatchQueueFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                                      const AsyncCreateCtx &) const {
  const auto r = infer(in, j);
  auto       t = std::make_unique<BatchQueueTask>();
  t->in_n      = in[0].shape[0];
  t->out_size  = j.at("output_size").get<size_t>();
  t->stride    = j.at("output_stride").get<size_t>();
  t->idesc = in[0], t->odesc = r.output_descs[0];
  t->ring.alloc(in[0].mem_loc, lcm_above(t->in_n, t->stride, j.at("target_capacity").get<size_t>() + t->in_n),
                in[0].num_bytes() / t->in_n);
  return t;
}

InferResult DualReaderBatchQueueFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"DualReaderBatchQueueFactory"};
  const size_t cap = j.at("target_capacity").get<size_t>(), window = j.at("window_size").get<size_t>();
  check(input_descs.size() == 1, "task must have exactly one input");
  const TDesc &in = input_descs[0];
  check(in.rank() > 0, "input rank must be positive");
  check(in.shape[0] > 0, "input leading dimension must be positive");
  check(in.is_contiguous(), "input must be contiguous");
  check(cap > 0, "target_capacity must be positive");
  check(window > 0, "window_size must be positive");
  std::vector<size_t> s = in.shape;
  s[0]                  = 1;
  const TDesc o(s, in.dtype, in.mem_loc);
  return async_io({in}, {o, o, TDesc({1}, DType::U8, MemLoc::Host)}, {true, true, false});
}
std::unique_ptr<IAsyncTask> DualReaderBatchQueueFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                                                const AsyncCreateCtx &ctx) const {
  const auto r = infer(in, j);
  auto       t = std::make_unique<DualReaderTask>();
  t->in_n      = in[0].shape[0];
  t->window    = j.at("window_size").get<size_t>();
  t->delay     = (t->window - 1) / 2;
  t->idesc = in[0], t->odesc = r.output_descs[0];
  const size_t elem = in[0].num_bytes() / t->in_n;
  t->ring.alloc(in[0].mem_loc, lcm_above(t->in_n, 1, j.at("target_capacity").get<size_t>() + t->in_n + t->delay + 1),
                elem);
  void *z = nullptr;
  if (t->ring.device) {
    cuda_ok(cudaMalloc(&z, elem), "DualReaderBatchQueue");
    cuda_ok(cudaMemsetAsync(z, 0, elem, ctx.consumer_stream), "DualReaderBatchQueue");
    cuda_ok(cudaStreamSynchronize(ctx.consumer_stream), "DualReaderBatchQueue");
  } else {
    cuda_ok(cudaMallocHost(&z, elem), "DualReaderBatchQueue");
    std::fill_n(static_cast<std::byte *>(z), elem, std::byte{0});
  }
  t->zero = static_cast<std::byte *>(z);
  return t;
}

InferResult SlidingAverageFactory::infer(std::span<const TDesc> input_descs, const nlohmann::json &j) const {
  const Check check{"SlidingAverageFactory"};
  const size_t cap = j.at("target_capacity").get<size_t>(), window = j.at("window_size").get<size_t>();
  check(input_descs.size() == 1, "task must have exactly one input");
  const TDesc &in = input_descs[0];
  check(in.dtype == DType::F32, "input must be float32");
  check(in.rank() == 3, "input must be 3D");
  check(in.shape[0] == 1, "input batch size must be 1");
  check(in.mem_loc == MemLoc::Device, "input must be in device memory");
  check(in.is_contiguous(), "input must be contiguous");
  check(cap > 0, "target_capacity must be greater or equal than zero");
  check(window > 0, "window_size must be greater or equal than zero");
  return async_io({in}, {in}, {true});
}
std::unique_ptr<IAsyncTask> SlidingAverageFactory::create(std::span<const TDesc> in, const nlohmann::json &j,
                                                          const AsyncCreateCtx &ctx) const {
  (void)infer(in, j);
  auto t    = std::make_unique<SlidingAverageTask>();
  t->idesc  = in[0];
  t->stream = ctx.consumer_stream;
  const int64_t n = (int64_t)in[0].num_elements();
  cuda_ok(cudaMalloc(&t->slot, (size_t)n * sizeof(float)), "SlidingAverage");
  cuda_ok(cudaMalloc(&t->avg, (size_t)n * sizeof(float)), "SlidingAverage");
  cuda_ok(hf_slideavg_create(n, j.at("window_size").get<int>(), j.value("discard_first", 0), ctx.consumer_stream,
                             &t->sa),
          "SlidingAverage");
  return t;
}

void register_np_kinds(core::Registry &r) {
  r.register_sync("Slice", std::make_unique<SliceFactory>());
  r.register_sync("Reshape", std::make_unique<ReshapeFactory>());
  r.register_sync("Copy", std::make_unique<CopyFactory>());
  r.register_sync("Concatenate", std::make_unique<ConcatenateFactory>());
  r.register_sync("Arange", std::make_unique<ArangeFactory>());
  r.register_sync("Multiply", std::make_unique<MultiplyFactory>());
  r.register_sync("Abs", std::make_unique<AbsFactory>());
  r.register_sync("CausalSlidingAverage", std::make_unique<CausalSlidingAverageFactory>());
  r.register_async("BatchQueue", std::make_unique<BatchQueueFactory>());
  r.register_async("DualReaderBatchQueue", std::make_unique<DualReaderBatchQueueFactory>());
  r.register_async("SlidingAverage", std::make_unique<SlidingAverageFactory>());
}

} // namespace hfb::nodes
