// holoflow_b200 node layer: the dataflow task interface of Holoflow's core, restated for the
// Doppler path so that this library's compute nodes can be created, updated and executed the way
// Holoflow's compiler and tests drive theirs.
//
// The types mirror holoflow::core (tensor.hh: DType, MemLoc, Storage, TDesc, TView;
// tasks.hh:81-332: SyncCtx, AsyncPushCtx, AsyncPopCtx, OpResult, IOStorageAccess, ITask (with
// acquire_input / release_output for owned tensors), ISyncTask, IAsyncTask, InPlace, TaskKind,
// InferResult, SyncCreateCtx, AsyncCreateCtx, ITaskFactory, ISyncTaskFactory, IAsyncTaskFactory;
// registry.hh:24-68: Registry) with the same member names and
// meanings: TDesc strides are in BYTES, infer() throws std::invalid_argument prefixed
// "<Factory> inference error: ", execute() returns OpResult for control flow only and reports
// failures by exception.  They live in namespace hfb::core so that a program can link this library
// next to Holoflow's own core without symbol clashes.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <map>
#include <memory>
#include <nlohmann/json.hpp>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

namespace hfb::core {

enum class DType : uint8_t { U8, U16, F32, CF32 };
enum class MemLoc : uint8_t { Host, Device };

[[nodiscard]] size_t           size_of(DType dtype) noexcept;
[[nodiscard]] std::string_view to_string(DType dtype) noexcept;

struct Storage {
  MemLoc     mem_loc = MemLoc::Device;
  size_t     bytes   = 0;
  std::byte *ptr     = nullptr;
};

struct TDesc {
  std::vector<size_t> shape;
  DType               dtype   = DType::F32;
  MemLoc              mem_loc = MemLoc::Device;
  std::vector<size_t> strides; // bytes; C-contiguous when constructed without strides
  size_t              offset = 0;

  TDesc() = default;
  TDesc(std::vector<size_t> shape, DType dtype, MemLoc mem_loc);
  TDesc(std::vector<size_t> shape, DType dtype, MemLoc mem_loc, std::vector<size_t> strides, size_t offset = 0);

  size_t rank() const noexcept { return shape.size(); }
  size_t num_elements() const;
  size_t num_bytes() const; // bytes of the dense logical tensor
  bool   is_contiguous() const;
};

bool operator==(const TDesc &a, const TDesc &b);

struct TView {
  TDesc    desc    = {};
  Storage *storage = nullptr;
  std::byte *data() { return storage ? storage->ptr + desc.offset : nullptr; }
  bool       is_nullptr() { return storage == nullptr || storage->ptr == nullptr; }
};

// The reference's event channel types (holoflow_event/router.hh); opaque here: the path's tasks
// neither emit nor read events, but the context carries them for tasks that do.
struct EventWriter;
struct EventReader;

struct SyncCtx {
  std::span<TView>   inputs;
  std::span<TView>   outputs;
  std::atomic<bool> *cancelled    = nullptr;
  EventWriter       *event_writer = nullptr;
  EventReader       *event_reader = nullptr;
};

struct AsyncPushCtx {
  std::span<TView>   inputs;
  std::atomic<bool> *cancelled = nullptr;
};

struct AsyncPopCtx {
  std::span<TView>   outputs;
  std::atomic<bool> *cancelled = nullptr;
};

enum class OpResult : uint8_t { Ok, NotReady, Cancelled, Eof };

// Storage of the tensors a task owns (InferResult::owned_inputs / owned_outputs): the scheduler
// keeps one Storage per owned tensor and the task points it at its own memory.
class IOStorageAccess {
public:
  virtual ~IOStorageAccess()                                      = default;
  [[nodiscard]] virtual Storage &owned_input_storage(size_t index)  = 0;
  [[nodiscard]] virtual Storage &owned_output_storage(size_t index) = 0;
};

struct InPlace {
  int in_idx;
  int out_idx;
};

enum class TaskKind { Sync, Async };

struct InferResult {
  std::vector<TDesc>   input_descs;
  std::vector<TDesc>   output_descs;
  std::vector<InPlace> in_place;
  std::vector<bool>    owned_inputs;
  std::vector<bool>    owned_outputs;
  TaskKind             kind = TaskKind::Sync;
};

struct SyncCreateCtx {
  cudaStream_t stream = static_cast<cudaStream_t>(0);
};

struct AsyncCreateCtx {
  cudaStream_t producer_stream = static_cast<cudaStream_t>(0);
  cudaStream_t consumer_stream = static_cast<cudaStream_t>(0);
};

class ITask {
public:
  virtual ~ITask() = default;
  // An owned input's view to write into before the push (nullopt: no room now).  The defaults
  // throw std::out_of_range: a task without owned tensors has no such index (tasks.cc).
  [[nodiscard]] virtual std::optional<TView> acquire_input(int index);
  // The consumer has finished with owned output `index` of the last pop.
  virtual void release_output(int index);
  void         bind_storage_access(IOStorageAccess *storage_access);

protected:
  // @throw std::logic_error when no storage access is bound
  [[nodiscard]] IOStorageAccess &storage_access();

private:
  IOStorageAccess *storage_access_ = nullptr;
};

class ISyncTask : public ITask {
public:
  [[nodiscard]] virtual OpResult execute(SyncCtx &ctx) = 0;
};

// A queue-like task: the producer pushes (after writing its owned inputs), the consumer pops
// (and later releases the owned outputs); both return NotReady when they cannot proceed now.
class IAsyncTask : public ITask {
public:
  [[nodiscard]] virtual OpResult try_push(AsyncPushCtx &ctx) = 0;
  [[nodiscard]] virtual OpResult try_pop(AsyncPopCtx &ctx)   = 0;
};

class ITaskFactory {
public:
  virtual ~ITaskFactory() = default;
  [[nodiscard]] virtual InferResult infer(std::span<const TDesc> input_descs, const nlohmann::json &jsettings) const = 0;
};

class ISyncTaskFactory : public ITaskFactory {
public:
  virtual std::unique_ptr<ISyncTask> create(std::span<const TDesc> input_descs, const nlohmann::json &jsettings,
                                            const SyncCreateCtx &ctx) const = 0;
  // Default: re-create (tasks.cc).  Factories override it to reuse allocations.
  virtual std::unique_ptr<ISyncTask> update(std::unique_ptr<ISyncTask> old_task, std::span<const TDesc> input_descs,
                                            const nlohmann::json &jsettings, const SyncCreateCtx &ctx) const;
};

class IAsyncTaskFactory : public ITaskFactory {
public:
  virtual std::unique_ptr<IAsyncTask> create(std::span<const TDesc> input_descs, const nlohmann::json &jsettings,
                                             const AsyncCreateCtx &ctx) const = 0;
  // Default: re-create (tasks.cc).
  virtual std::unique_ptr<IAsyncTask> update(std::unique_ptr<IAsyncTask> old_task, std::span<const TDesc> input_descs,
                                             const nlohmann::json &jsettings, const AsyncCreateCtx &ctx) const;
};

class Registry {
public:
  using Key      = std::string;
  using SyncPtr  = std::unique_ptr<ISyncTaskFactory>;
  using AsyncPtr = std::unique_ptr<IAsyncTaskFactory>;
  // @throw std::invalid_argument if `kind` is already registered (as either kind of task)
  void register_sync(const Key &kind, SyncPtr factory);
  void register_async(const Key &kind, AsyncPtr factory);
  // @throw std::out_of_range if `kind` is not registered
  const ISyncTaskFactory  &get_sync(const Key &kind) const;
  const IAsyncTaskFactory &get_async(const Key &kind) const;
  bool                     is_sync_registered(const Key &kind) const noexcept;
  bool                     is_async_registered(const Key &kind) const noexcept;
  std::vector<Key>         kinds() const; // both kinds, sorted

private:
  std::map<Key, SyncPtr>  sync_factories_;
  std::map<Key, AsyncPtr> async_factories_;
};

// A CUDA runtime failure inside a task (the reference's curaii::CudaError role).
class CudaError : public std::runtime_error {
public:
  using std::runtime_error::runtime_error;
};

} // namespace hfb::core
