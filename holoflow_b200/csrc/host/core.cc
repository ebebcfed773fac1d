// hfb::core: tensor descriptors, the default update() and the kind registry (the restated
// holoflow::core surface; tensor.hh, tasks.cc, registry.hh:24-68).
#include "holoflow_b200/core.hh"

#include <algorithm>

namespace hfb::core {

size_t size_of(DType dtype) noexcept {
  switch (dtype) {
  case DType::U8: return 1;
  case DType::U16: return 2;
  case DType::F32: return 4;
  case DType::CF32: return 8;
  }
  return 0;
}

std::string_view to_string(DType dtype) noexcept {
  switch (dtype) {
  case DType::U8: return "U8";
  case DType::U16: return "U16";
  case DType::F32: return "F32";
  case DType::CF32: return "CF32";
  }
  return "?";
}

static std::vector<size_t> contiguous_strides(const std::vector<size_t> &shape, DType dtype) {
  std::vector<size_t> st(shape.size());
  size_t              acc = size_of(dtype);
  for (size_t i = shape.size(); i-- > 0;) {
    st[i] = acc;
    acc *= shape[i];
  }
  return st;
}

TDesc::TDesc(std::vector<size_t> s, DType d, MemLoc m)
    : shape(std::move(s)), dtype(d), mem_loc(m), strides(contiguous_strides(shape, d)) {}

TDesc::TDesc(std::vector<size_t> s, DType d, MemLoc m, std::vector<size_t> st, size_t off)
    : shape(std::move(s)), dtype(d), mem_loc(m), strides(std::move(st)), offset(off) {
  if (strides.empty())
    strides = contiguous_strides(shape, dtype);
  if (strides.size() != shape.size())
    throw std::invalid_argument("TDesc: strides must have one entry per dimension");
}

size_t TDesc::num_elements() const {
  size_t n = 1;
  for (size_t d : shape)
    n *= d;
  return n;
}

size_t TDesc::num_bytes() const { return num_elements() * size_of(dtype); }

bool TDesc::is_contiguous() const { return strides == contiguous_strides(shape, dtype); }

bool operator==(const TDesc &a, const TDesc &b) {
  return a.shape == b.shape && a.dtype == b.dtype && a.mem_loc == b.mem_loc && a.strides == b.strides &&
         a.offset == b.offset;
}

std::unique_ptr<ISyncTask> ISyncTaskFactory::update(std::unique_ptr<ISyncTask> old_task,
                                                    std::span<const TDesc> input_descs,
                                                    const nlohmann::json &jsettings, const SyncCreateCtx &ctx) const {
  old_task.reset();
  return create(input_descs, jsettings, ctx);
}

std::unique_ptr<IAsyncTask> IAsyncTaskFactory::update(std::unique_ptr<IAsyncTask> old_task,
                                                      std::span<const TDesc> input_descs,
                                                      const nlohmann::json &jsettings, const AsyncCreateCtx &ctx) const {
  old_task.reset();
  return create(input_descs, jsettings, ctx);
}

std::optional<TView> ITask::acquire_input(int) { throw std::out_of_range("Input index out of range"); }

void ITask::release_output(int) { throw std::out_of_range("Output index out of range"); }

void ITask::bind_storage_access(IOStorageAccess *storage_access) {
  if (storage_access == nullptr)
    throw std::logic_error("Cannot bind null storage access to task");
  storage_access_ = storage_access;
}

IOStorageAccess &ITask::storage_access() {
  if (storage_access_ == nullptr)
    throw std::logic_error("Storage access not bound to task");
  return *storage_access_;
}

void Registry::register_sync(const Key &kind, SyncPtr factory) {
  if (sync_factories_.count(kind) || async_factories_.count(kind))
    throw std::invalid_argument("Registry: kind '" + kind + "' is already registered");
  sync_factories_.emplace(kind, std::move(factory));
}

void Registry::register_async(const Key &kind, AsyncPtr factory) {
  if (sync_factories_.count(kind) || async_factories_.count(kind))
    throw std::invalid_argument("Registry: kind '" + kind + "' is already registered");
  async_factories_.emplace(kind, std::move(factory));
}

const IAsyncTaskFactory &Registry::get_async(const Key &kind) const {
  auto it = async_factories_.find(kind);
  if (it == async_factories_.end())
    throw std::out_of_range("Registry: no asynchronous task of kind '" + kind + "'");
  return *it->second;
}

bool Registry::is_async_registered(const Key &kind) const noexcept { return async_factories_.count(kind) != 0; }

const ISyncTaskFactory &Registry::get_sync(const Key &kind) const {
  auto it = sync_factories_.find(kind);
  if (it == sync_factories_.end())
    throw std::out_of_range("Registry: no synchronous task of kind '" + kind + "'");
  return *it->second;
}

bool Registry::is_sync_registered(const Key &kind) const noexcept { return sync_factories_.count(kind) != 0; }

std::vector<Registry::Key> Registry::kinds() const {
  std::vector<Key> out;
  for (const auto &kv : sync_factories_)
    out.push_back(kv.first);
  for (const auto &kv : async_factories_)
    out.push_back(kv.first);
  std::sort(out.begin(), out.end());
  return out;
}

} // namespace hfb::core
