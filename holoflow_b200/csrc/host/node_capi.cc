// C ABI over the node layer: create / update / execute the path's compute nodes by kind string and
// JSON settings, the way Holoflow's compiler drives ISyncTaskFactory (infer -> create/update ->
// execute, compiler.cc:436-476, 961-1103) and its tests drive run_sync_factory
// (sync_task_runner.cc:84-96).  Exceptions become statuses: std::invalid_argument and JSON errors
// HF_ERR_INVALID, a CUDA failure HF_ERR_CUDA; the message is in hf_last_error().
#include <cstring>

#include "hf_common.cuh"
#include "holoflow_b200.h"
#include "holoflow_b200/nodes.hh"

using namespace hfb;

struct hf_node : core::IOStorageAccess {
  std::string                        kind;
  const core::ISyncTaskFactory      *factory  = nullptr;
  const core::IAsyncTaskFactory     *afactory = nullptr; // set for an asynchronous kind
  std::unique_ptr<core::ISyncTask>   task;
  std::unique_ptr<core::IAsyncTask>  atask;
  std::vector<core::TDesc>           in_descs, out_descs;
  std::vector<bool>                  owned;     // outputs the task publishes itself
  std::vector<bool>                  owned_in;  // inputs the task provides (acquire_input)
  std::vector<int>                   alias;     // per output: the input it views (in place), or -1
  std::vector<void *>                published; // output origins as of the last execute / pop
  std::vector<core::Storage>         in_st, out_st; // storage of the owned tensors
  core::Storage &owned_input_storage(size_t i) override { return in_st.at(i); }
  core::Storage &owned_output_storage(size_t i) override { return out_st.at(i); }
  core::ITask   *any_task() { return afactory ? static_cast<core::ITask *>(atask.get()) : task.get(); }
  void           set_io(const core::InferResult &inf) {
    out_descs = inf.output_descs;
    owned.assign(out_descs.size(), false);
    for (size_t i = 0; i < inf.owned_outputs.size() && i < owned.size(); ++i)
      owned[i] = inf.owned_outputs[i];
    owned_in.assign(in_descs.size(), false);
    for (size_t i = 0; i < inf.owned_inputs.size() && i < owned_in.size(); ++i)
      owned_in[i] = inf.owned_inputs[i];
    alias.assign(out_descs.size(), -1);
    for (const auto &ip : inf.in_place)
      if (ip.out_idx >= 0 && ip.out_idx < (int)alias.size())
        alias[(size_t)ip.out_idx] = ip.in_idx;
    published.assign(out_descs.size(), nullptr);
    in_st.resize(in_descs.size());
    out_st.resize(out_descs.size());
    for (size_t i = 0; i < in_st.size(); ++i)
      in_st[i] = core::Storage{in_descs[i].mem_loc, in_descs[i].num_bytes(), nullptr};
    for (size_t i = 0; i < out_st.size(); ++i)
      out_st[i] = core::Storage{out_descs[i].mem_loc, out_descs[i].num_bytes(), nullptr};
  }
};

namespace {

core::TDesc to_desc(const hf_tdesc &t) {
  if (t.rank < 0 || t.rank > HF_TDESC_MAX_RANK)
    throw std::invalid_argument("hf_tdesc: rank must be in [0, 8]");
  if (t.dtype < 0 || t.dtype > 3)
    throw std::invalid_argument("hf_tdesc: dtype must be HF_U8, HF_U16, HF_F32 or HF_CF32");
  std::vector<size_t> shape(t.shape, t.shape + t.rank), strides;
  bool                given = false;
  for (int i = 0; i < t.rank; ++i)
    given |= t.strides[i] != 0;
  if (given)
    strides.assign(t.strides, t.strides + t.rank);
  return core::TDesc(std::move(shape), static_cast<core::DType>(t.dtype),
                     t.mem_loc ? core::MemLoc::Device : core::MemLoc::Host, std::move(strides), (size_t)t.offset);
}

hf_tdesc from_desc(const core::TDesc &d) {
  hf_tdesc t{};
  t.rank    = (int32_t)d.rank();
  t.dtype   = (int32_t)d.dtype;
  t.mem_loc = d.mem_loc == core::MemLoc::Device ? 1 : 0;
  for (size_t i = 0; i < d.rank() && i < HF_TDESC_MAX_RANK; ++i) {
    t.shape[i]   = (int64_t)d.shape[i];
    t.strides[i] = (int64_t)d.strides[i];
  }
  t.offset = (int64_t)d.offset;
  return t;
}

std::vector<core::TDesc> to_descs(int n, const hf_tdesc *in) {
  if (n < 0 || (n > 0 && in == nullptr))
    throw std::invalid_argument("input descriptors: bad count or null pointer");
  std::vector<core::TDesc> v;
  for (int i = 0; i < n; ++i)
    v.push_back(to_desc(in[i]));
  return v;
}

nlohmann::json parse(const char *json) {
  return json && *json ? nlohmann::json::parse(json) : nlohmann::json::object();
}

template <class F> int guarded(F &&f) {
  hf::clear_error();
  try {
    return f();
  } catch (const core::CudaError &e) {
    return hf::fail(HF_ERR_CUDA, e.what());
  } catch (const std::invalid_argument &e) {
    return hf::fail(HF_ERR_INVALID, e.what());
  } catch (const std::out_of_range &e) {
    return hf::fail(HF_ERR_INVALID, e.what());
  } catch (const nlohmann::json::exception &e) {
    return hf::fail(HF_ERR_INVALID, std::string("settings: ") + e.what());
  } catch (const std::exception &e) {
    return hf::fail(HF_ERR_STATE, e.what());
  }
}

} // namespace

extern "C" {

int hf_node_kinds(char *buf, size_t cap) {
  return guarded([&]() -> int {
    std::string s;
    for (const auto &k : nodes::default_registry().kinds())
      s += (s.empty() ? "" : ",") + k;
    HF_CHECK_ARG(buf != nullptr && cap > s.size(), "hf_node_kinds: buffer too small");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return HF_OK;
  });
}

int hf_node_infer(const char *kind, const char *json, int n_in, const hf_tdesc *in, int *n_out, hf_tdesc *out,
                  int out_cap) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(kind != nullptr && n_out != nullptr, "hf_node_infer: null argument");
    const auto                &reg = nodes::default_registry();
    const core::ITaskFactory &f   = reg.is_async_registered(kind)
                                        ? static_cast<const core::ITaskFactory &>(reg.get_async(kind))
                                        : static_cast<const core::ITaskFactory &>(reg.get_sync(kind));
    const auto  descs = to_descs(n_in, in);
    const auto  r     = f.infer(descs, parse(json));
    *n_out            = (int)r.output_descs.size();
    HF_CHECK_ARG(out != nullptr && out_cap >= *n_out, "hf_node_infer: output descriptor array too small");
    for (int i = 0; i < *n_out; ++i)
      out[i] = from_desc(r.output_descs[i]);
    return HF_OK;
  });
}

int hf_node_create(const char *kind, const char *json, int n_in, const hf_tdesc *in, hf_stream_t s, hf_node **node) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(kind != nullptr && node != nullptr, "hf_node_create: null argument");
    *node        = nullptr;
    auto        n   = std::make_unique<hf_node>();
    const auto &reg = nodes::default_registry();
    n->kind         = kind;
    n->in_descs     = to_descs(n_in, in);
    const auto j    = parse(json);
    auto      *cs   = reinterpret_cast<cudaStream_t>(s);
    if (reg.is_async_registered(kind)) {
      n->afactory = &reg.get_async(kind);
      n->set_io(n->afactory->infer(n->in_descs, j));
      n->atask = n->afactory->create(n->in_descs, j, core::AsyncCreateCtx{cs, cs});
    } else {
      n->factory = &reg.get_sync(kind);
      n->set_io(n->factory->infer(n->in_descs, j));
      n->task = n->factory->create(n->in_descs, j, core::SyncCreateCtx{cs});
    }
    n->any_task()->bind_storage_access(n.get());
    *node = n.release();
    return HF_OK;
  });
}

int hf_node_update(hf_node *node, const char *json, int n_in, const hf_tdesc *in, hf_stream_t s) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(node != nullptr && node->any_task() != nullptr, "hf_node_update: node was not created");
    const auto descs = to_descs(n_in, in);
    const auto j     = parse(json);
    auto      *cs    = reinterpret_cast<cudaStream_t>(s);
    if (node->afactory) {
      auto inf    = node->afactory->infer(descs, j);
      node->atask = node->afactory->update(std::move(node->atask), descs, j, core::AsyncCreateCtx{cs, cs});
      node->in_descs = descs;
      node->set_io(inf);
    } else {
      auto inf   = node->factory->infer(descs, j);
      node->task = node->factory->update(std::move(node->task), descs, j, core::SyncCreateCtx{cs});
      node->in_descs = descs;
      node->set_io(inf);
    }
    node->any_task()->bind_storage_access(node);
    return HF_OK;
  });
}

int hf_node_execute(hf_node *node, void *const *inputs, void *const *outputs, int *op_result) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(node != nullptr && node->task != nullptr, "hf_node_execute: node was not created (or is "
                                                            "asynchronous: use hf_node_try_push / hf_node_try_pop)");
    HF_CHECK_ARG(node->in_descs.empty() || inputs != nullptr, "hf_node_execute: null tensor array");
    std::vector<core::Storage> st(node->in_descs.size() + node->out_descs.size());
    std::vector<core::TView>   iv(node->in_descs.size()), ov(node->out_descs.size());
    for (size_t i = 0; i < iv.size(); ++i) {
      HF_CHECK_ARG(inputs[i] != nullptr, "hf_node_execute: null input pointer");
      st[i] = core::Storage{node->in_descs[i].mem_loc, node->in_descs[i].num_bytes(), static_cast<std::byte *>(inputs[i])};
      iv[i] = core::TView{node->in_descs[i], &st[i]};
      iv[i].desc.offset = 0; // the pointer given is the tensor's origin
    }
    for (size_t i = 0; i < ov.size(); ++i) {
      const int a = node->alias[i];
      if (a >= 0) { // a view of input a: its storage, at the view's offset from the input's origin
        ov[i]             = core::TView{node->out_descs[i], &st[(size_t)a]};
        ov[i].desc.offset = node->out_descs[i].offset - node->in_descs[(size_t)a].offset;
        continue;
      }
      void *p = outputs ? outputs[i] : nullptr;
      HF_CHECK_ARG(node->owned[i] || p != nullptr, "hf_node_execute: null output pointer");
      auto &s = st[iv.size() + i];
      s       = core::Storage{node->out_descs[i].mem_loc, node->out_descs[i].num_bytes(), static_cast<std::byte *>(p)};
      ov[i]   = core::TView{node->out_descs[i], &s};
      ov[i].desc.offset = 0;
    }
    std::atomic<bool> cancelled{false};
    core::SyncCtx     ctx{std::span<core::TView>(iv), std::span<core::TView>(ov), &cancelled};
    const auto        r = node->task->execute(ctx);
    for (size_t i = 0; i < ov.size(); ++i)
      node->published[i] = ov[i].data();
    if (op_result)
      *op_result = (int)r;
    return HF_OK;
  });
}

int hf_node_output_desc(const hf_node *node, int i, hf_tdesc *out) {
  hf::clear_error();
  HF_CHECK_ARG(node != nullptr && out != nullptr && i >= 0 && i < (int)node->out_descs.size(),
               "hf_node_output_desc: bad argument");
  *out = from_desc(node->out_descs[i]);
  return HF_OK;
}

int hf_node_output_ptr(const hf_node *node, int i, void **ptr, int *owned) {
  hf::clear_error();
  HF_CHECK_ARG(node != nullptr && ptr != nullptr && i >= 0 && i < (int)node->out_descs.size(),
               "hf_node_output_ptr: bad argument");
  *ptr = node->published[i];
  if (owned)
    *owned = node->owned[i] ? 1 : 0;
  return HF_OK;
}

int hf_node_is_async(const hf_node *node) { return node != nullptr && node->afactory != nullptr ? 1 : 0; }

int hf_node_output_alias(const hf_node *node, int i, int *input_index) {
  hf::clear_error();
  HF_CHECK_ARG(node != nullptr && input_index != nullptr && i >= 0 && i < (int)node->out_descs.size(),
               "hf_node_output_alias: bad argument");
  *input_index = node->alias[(size_t)i];
  return HF_OK;
}

int hf_node_acquire_input(hf_node *node, int index, void **ptr) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(node != nullptr && ptr != nullptr, "hf_node_acquire_input: null argument");
    *ptr   = nullptr;
    auto v = node->any_task()->acquire_input(index);
    if (v)
      *ptr = v->data();
    return HF_OK;
  });
}

int hf_node_try_push(hf_node *node, int *op_result) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(node != nullptr && node->atask != nullptr, "hf_node_try_push: not an asynchronous node");
    std::vector<core::TView> iv(node->in_descs.size());
    for (size_t i = 0; i < iv.size(); ++i)
      iv[i] = core::TView{node->in_descs[i], &node->in_st[i]};
    std::atomic<bool>  cancelled{false};
    core::AsyncPushCtx ctx{std::span<core::TView>(iv), &cancelled};
    const auto         r = node->atask->try_push(ctx);
    if (op_result)
      *op_result = (int)r;
    return HF_OK;
  });
}

int hf_node_try_pop(hf_node *node, void *const *outputs, int *op_result) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(node != nullptr && node->atask != nullptr, "hf_node_try_pop: not an asynchronous node");
    std::vector<core::TView>   ov(node->out_descs.size());
    std::vector<core::Storage> given(ov.size());
    for (size_t i = 0; i < ov.size(); ++i) {
      if (node->owned[i]) {
        ov[i] = core::TView{node->out_descs[i], &node->out_st[i]};
        continue;
      }
      void *p = outputs ? outputs[i] : nullptr;
      HF_CHECK_ARG(p != nullptr, "hf_node_try_pop: null pointer for an output the node does not own");
      given[i] = core::Storage{node->out_descs[i].mem_loc, node->out_descs[i].num_bytes(), static_cast<std::byte *>(p)};
      ov[i]    = core::TView{node->out_descs[i], &given[i]};
    }
    std::atomic<bool> cancelled{false};
    core::AsyncPopCtx ctx{std::span<core::TView>(ov), &cancelled};
    const auto        r = node->atask->try_pop(ctx);
    if (r == core::OpResult::Ok)
      for (size_t i = 0; i < ov.size(); ++i)
        node->published[i] = ov[i].data();
    if (op_result)
      *op_result = (int)r;
    return HF_OK;
  });
}

int hf_node_release_output(hf_node *node, int index) {
  return guarded([&]() -> int {
    HF_CHECK_ARG(node != nullptr && node->any_task() != nullptr, "hf_node_release_output: null node");
    node->any_task()->release_output(index);
    return HF_OK;
  });
}

int hf_node_destroy(hf_node *node) {
  return guarded([&]() -> int {
    delete node;
    return HF_OK;
  });
}

} // extern "C"
