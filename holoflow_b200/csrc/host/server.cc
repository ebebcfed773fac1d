// Streaming server: many concurrent camera streams on one GPU with continuous batching.
//
// A stream is a slot holding its own plan (hf_plan), device frame ring (hf_stream), a compute CUDA
// stream and an H2D CUDA stream.  Streams are admitted while the device has room: a stream is
// opened only if, after creating its buffers, the free device memory stays above the server's
// reserve (otherwise HF_ERR_NOMEM and the caller retries once others have closed).  Every
// hf_server_step gives each open stream with ready windows one batch (up to its plan's
// max_batch) on its own CUDA stream, so batches of different streams -- of different frame
// sizes, rates and propagation distances -- run concurrently on the device; a stream opened or
// closed between steps joins or leaves the next step.  Each push is timestamped by a CUDA event;
// a window's frame-to-image latency runs from the push that brought its last frame to the end of
// the D2H copy of its images.
//
// Nothing in the serving loop waits for the whole device.  Plans and rings of the streams come
// from a server-owned stream-ordered memory pool (cudaMallocFromPoolAsync / cudaFreeAsync on the
// slot's own stream, the pool keeping freed memory for the next stream), so opening or closing a
// stream neither synchronises the device nor stalls the batches of the others; completions are
// observed per batch by querying its event (hf_server_poll), so a step can be issued while earlier
// batches are still on the device.
#include <algorithm>
#include <deque>
#include <mutex>
#include <new>
#include <vector>

#include "hf_common.cuh"
#include "holoflow_b200.h"
#include "host_util.cuh"

using namespace hf;

namespace {
struct PushMark {
  int64_t     last_frame; // absolute index of the last frame this push brought
  cudaEvent_t ev;         // recorded on the H2D stream before the copy
};
struct DoneMark {
  int64_t     last_frame; // last frame of the batch's last window
  int         nwin;
  cudaEvent_t ev; // recorded after the batch's images reached the host
  std::vector<int64_t> window_last; // last frame of each window of the batch
};
struct Slot {
  bool                 open = false;
  hf_desc              d{};
  hf_plan             *plan = nullptr;
  hf_stream           *cam  = nullptr;
  cudaStream_t         comp = nullptr, h2d = nullptr, mark = nullptr;
  int64_t              pushed = 0, next_win = 0;
  std::deque<PushMark> pushes;
  std::deque<DoneMark> done;
  int64_t              completed = 0; // windows whose images have reached the host
};
} // namespace

struct hf_server {
  size_t              reserve = 0;
  cudaMemPool_t       mem     = nullptr; // plans and rings of every stream
  std::vector<Slot>   slots;
  std::vector<float>  latencies; // completed windows, ms
  std::vector<cudaEvent_t> pool;  // recycled timing events
  cudaEvent_t take_event() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess)
      return nullptr;
    return e;
  }
};

static void slot_release(hf_server *srv, Slot &s) {
  for (cudaStream_t q : {s.comp, s.h2d, s.mark}) // this stream's work only, not the device's
    if (q)
      cudaStreamSynchronize(q);
  if (s.cam)
    hf_stream_destroy(s.cam); // pooled: frees on s.comp, waits for its own streams
  if (s.plan)
    hf_plan_destroy(s.plan);
  for (cudaStream_t q : {s.comp, s.h2d, s.mark})
    if (q)
      cudaStreamDestroy(q);
  for (auto &p : s.pushes)
    srv->pool.push_back(p.ev);
  for (auto &d : s.done)
    srv->pool.push_back(d.ev);
  s = Slot{};
}

extern "C" {

int hf_server_create(size_t hbm_reserve_bytes, int max_streams, hf_server **out) {
  clear_error();
  HF_CHECK_ARG(out != nullptr && max_streams >= 1 && max_streams <= 1024, "hf_server_create: bad argument");
  auto *srv = new (std::nothrow) hf_server();
  if (!srv)
    return fail(HF_ERR_NOMEM, "hf_server_create: host allocation failed");
  srv->reserve = hbm_reserve_bytes;
  srv->slots.resize((size_t)max_streams);
  int dev = 0;
  cudaMemPoolProps props{};
  props.allocType     = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  cudaError_t e       = cudaGetDevice(&dev);
  props.location.id   = dev;
  if (e == cudaSuccess)
    e = cudaMemPoolCreate(&srv->mem, &props);
  uint64_t keep = UINT64_MAX; // freed memory stays in the pool for the next stream
  if (e == cudaSuccess)
    e = cudaMemPoolSetAttribute(srv->mem, cudaMemPoolAttrReleaseThreshold, &keep);
  if (e != cudaSuccess) {
    if (srv->mem)
      cudaMemPoolDestroy(srv->mem);
    delete srv;
    return cuda_status(e, "hf_server_create: memory pool");
  }
  *out = srv;
  return HF_OK;
}

// Device memory a new stream can use: free device memory plus what the pool holds unused.
static int available_bytes(hf_server *srv, size_t *avail) {
  size_t   free_b = 0, total_b = 0;
  uint64_t reserved = 0, used = 0;
  HF_CUDA(cudaMemGetInfo(&free_b, &total_b));
  HF_CUDA(cudaMemPoolGetAttribute(srv->mem, cudaMemPoolAttrReservedMemCurrent, &reserved));
  HF_CUDA(cudaMemPoolGetAttribute(srv->mem, cudaMemPoolAttrUsedMemCurrent, &used));
  *avail = free_b + (size_t)(reserved > used ? reserved - used : 0);
  return HF_OK;
}

int hf_server_reserve(hf_server *srv, size_t bytes) {
  clear_error();
  HF_CHECK_ARG(srv != nullptr, "hf_server_reserve: null server");
  if (bytes == 0)
    return HF_OK;
  cudaStream_t q = nullptr;
  HF_CUDA(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
  void       *p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, srv->mem, q);
  if (e == cudaSuccess)
    e = cudaFreeAsync(p, q);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(q);
  cudaStreamDestroy(q);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return fail(HF_ERR_NOMEM, "hf_server_reserve: the pool could not reserve " + std::to_string(bytes) + " bytes");
  }
  return HF_OK;
}

int hf_server_destroy(hf_server *srv) {
  if (!srv)
    return HF_OK;
  for (auto &s : srv->slots)
    if (s.open)
      slot_release(srv, s);
  for (cudaEvent_t e : srv->pool)
    cudaEventDestroy(e);
  if (srv->mem) {
    cudaDeviceSynchronize(); // pooled frees are stream-ordered: let them land before the pool goes
    cudaMemPoolDestroy(srv->mem);
  }
  delete srv;
  return HF_OK;
}

int hf_server_open(hf_server *srv, const hf_desc *desc, int64_t ring_frames, int *id) {
  clear_error();
  HF_CHECK_ARG(srv != nullptr && desc != nullptr && id != nullptr, "hf_server_open: null argument");
  *id = -1;
  int k = -1;
  for (size_t i = 0; i < srv->slots.size(); ++i)
    if (!srv->slots[i].open) {
      k = (int)i;
      break;
    }
  if (k < 0)
    return fail(HF_ERR_NOMEM, "hf_server_open: every stream slot is in use");
  size_t avail = 0;
  HF_TRY(available_bytes(srv, &avail));
  if (avail < srv->reserve)
    return fail(HF_ERR_NOMEM, "hf_server_open: free device memory is below the reserve");
  Slot &s = srv->slots[(size_t)k];
  s.d     = *desc;
  int rc  = cuda_status(cudaStreamCreateWithFlags(&s.comp, cudaStreamNonBlocking), "server stream");
  if (rc == HF_OK)
    rc = cuda_status(cudaStreamCreateWithFlags(&s.h2d, cudaStreamNonBlocking), "server stream");
  if (rc == HF_OK)
    rc = cuda_status(cudaStreamCreateWithFlags(&s.mark, cudaStreamNonBlocking), "server stream");
  if (rc == HF_OK) { // plan and ring from the pool, in the order of this stream's compute stream
    AllocScope scope(srv->mem, s.comp);
    rc = hf_plan_create(desc, &s.plan, s.comp);
    if (rc == HF_OK)
      rc = hf_stream_create(s.plan, ring_frames, &s.cam);
  }
  if (rc == HF_OK) { // pushes on the H2D stream start after the ring exists in stream order
    cudaEvent_t ev = srv->take_event();
    rc = ev ? cuda_status(cudaEventRecord(ev, s.comp), "server event") : fail(HF_ERR_CUDA, "server event");
    if (rc == HF_OK)
      rc = cuda_status(cudaStreamWaitEvent(s.h2d, ev, 0), "server event");
    if (ev)
      srv->pool.push_back(ev);
  }
  if (rc == HF_OK) {
    rc = available_bytes(srv, &avail);
    if (rc == HF_OK && avail < srv->reserve)
      rc = fail(HF_ERR_NOMEM, "hf_server_open: admitting this stream would leave less free device memory "
                              "than the reserve");
  }
  if (rc != HF_OK) {
    const std::string msg = hf_last_error();
    slot_release(srv, s);
    set_error(msg);
    return rc == HF_ERR_CUDA && msg.find("out of memory") != std::string::npos ? HF_ERR_NOMEM : rc;
  }
  s.open = true;
  *id    = k;
  return HF_OK;
}

int hf_server_close(hf_server *srv, int id) {
  clear_error();
  HF_CHECK_ARG(srv != nullptr && id >= 0 && id < (int)srv->slots.size() && srv->slots[(size_t)id].open,
               "hf_server_close: no such open stream");
  slot_release(srv, srv->slots[(size_t)id]);
  return HF_OK;
}

int hf_server_push(hf_server *srv, int id, const void *frames, int64_t nframes) {
  clear_error();
  HF_CHECK_ARG(srv != nullptr && id >= 0 && id < (int)srv->slots.size() && srv->slots[(size_t)id].open,
               "hf_server_push: no such open stream");
  if (nframes == 0)
    return HF_OK;
  Slot       &s  = srv->slots[(size_t)id];
  cudaEvent_t ev = srv->take_event();
  if (!ev)
    return fail(HF_ERR_CUDA, "hf_server_push: event creation failed");
  HF_CUDA(cudaEventRecord(ev, s.h2d));
  const int rc = hf_stream_push(s.cam, frames, nframes, s.h2d);
  if (rc != HF_OK) {
    srv->pool.push_back(ev);
    return rc;
  }
  s.pushed += nframes;
  s.pushes.push_back(PushMark{s.pushed - 1, ev});
  return HF_OK;
}

int64_t hf_server_ready(const hf_server *srv, int id) {
  if (!srv || id < 0 || id >= (int)srv->slots.size() || !srv->slots[(size_t)id].open)
    return 0;
  return hf_stream_ready(srv->slots[(size_t)id].cam);
}

int hf_server_step(hf_server *srv, float *const *out, int *n_done) {
  clear_error();
  HF_CHECK_ARG(srv != nullptr && out != nullptr && n_done != nullptr, "hf_server_step: null argument");
  for (size_t i = 0; i < srv->slots.size(); ++i) {
    Slot &s   = srv->slots[i];
    n_done[i] = 0;
    if (!s.open || out[i] == nullptr || hf_stream_ready(s.cam) <= 0)
      continue;
    int n = 0;
    HF_TRY(hf_stream_process(s.cam, s.d.max_batch, out[i], 2, &n, s.comp));
    n_done[i] = n;
    if (n <= 0)
      continue;
    // completion mark: after this batch's images are on the host
    HF_TRY(hf_stream_output_wait(s.cam, s.mark, 0));
    DoneMark dm{};
    dm.ev   = srv->take_event();
    dm.nwin = n;
    if (!dm.ev)
      return fail(HF_ERR_CUDA, "hf_server_step: event creation failed");
    HF_CUDA(cudaEventRecord(dm.ev, s.mark));
    for (int w = 0; w < n; ++w)
      dm.window_last.push_back((s.next_win + w) * s.d.hop + s.d.frames - 1);
    dm.last_frame = dm.window_last.back();
    s.next_win += n;
    s.done.push_back(std::move(dm));
  }
  return HF_OK;
}

// Turns the completed batches of slot `s` (their events have fired) into per-window latencies,
// counts their windows and recycles the push marks no pending window needs any more.  Never
// waits: a batch still on the device stays queued.
static int collect(hf_server *srv, Slot &s) {
  while (!s.done.empty()) {
    DoneMark         &dm = s.done.front();
    const cudaError_t q  = cudaEventQuery(dm.ev);
    if (q == cudaErrorNotReady)
      break;
    if (q != cudaSuccess)
      return cuda_status(q, "hf_server_poll: batch event");
    for (int64_t last : dm.window_last) {
      // the push that brought frame `last`
      auto it = std::find_if(s.pushes.begin(), s.pushes.end(), [&](const PushMark &p) { return p.last_frame >= last; });
      if (it == s.pushes.end())
        continue;
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, it->ev, dm.ev) == cudaSuccess)
        srv->latencies.push_back(ms);
    }
    s.completed += dm.nwin;
    srv->pool.push_back(dm.ev);
    s.done.pop_front();
  }
  // pushes whose frames all precede the oldest window still to be delivered are no longer needed
  const int64_t oldest      = s.done.empty() ? s.next_win : s.next_win - [&] {
    int64_t n = 0;
    for (const auto &dm : s.done)
      n += dm.nwin;
    return n;
  }();
  const int64_t first_needed = oldest * s.d.hop + s.d.frames - 1;
  while (s.pushes.size() > 1 && s.pushes.front().last_frame < first_needed) {
    srv->pool.push_back(s.pushes.front().ev);
    s.pushes.pop_front();
  }
  return HF_OK;
}

int hf_server_poll(hf_server *srv, int64_t *completed) {
  clear_error();
  HF_CHECK_ARG(srv != nullptr, "hf_server_poll: null server");
  for (size_t i = 0; i < srv->slots.size(); ++i) {
    Slot &s = srv->slots[i];
    if (s.open)
      HF_TRY(collect(srv, s));
    if (completed)
      completed[i] = s.open ? s.completed : 0;
  }
  return HF_OK;
}

int hf_server_inflight(const hf_server *srv, int id) {
  if (!srv || id < 0 || id >= (int)srv->slots.size() || !srv->slots[(size_t)id].open)
    return 0;
  int n = 0;
  for (const auto &dm : srv->slots[(size_t)id].done)
    n += cudaEventQuery(dm.ev) == cudaErrorNotReady ? 1 : 0;
  return n;
}

// Waits for every open stream's own CUDA streams (not the device), then collects as poll does.
int hf_server_sync(hf_server *srv) {
  clear_error();
  HF_CHECK_ARG(srv != nullptr, "hf_server_sync: null server");
  for (auto &s : srv->slots) {
    if (!s.open)
      continue;
    HF_CUDA(cudaStreamSynchronize(s.h2d));
    HF_CUDA(cudaStreamSynchronize(s.comp));
    HF_CUDA(cudaStreamSynchronize(s.mark));
    HF_TRY(collect(srv, s));
  }
  return HF_OK;
}

int hf_server_latencies(hf_server *srv, float *ms, int cap, int *n) {
  clear_error();
  HF_CHECK_ARG(srv != nullptr && n != nullptr && (cap == 0 || ms != nullptr), "hf_server_latencies: bad argument");
  const int k = (int)std::min<size_t>((size_t)cap, srv->latencies.size());
  std::copy(srv->latencies.begin(), srv->latencies.begin() + k, ms);
  srv->latencies.erase(srv->latencies.begin(), srv->latencies.begin() + k);
  *n = k;
  return HF_OK;
}

int hf_server_open_count(const hf_server *srv) {
  if (!srv)
    return 0;
  int c = 0;
  for (const auto &s : srv->slots)
    c += s.open ? 1 : 0;
  return c;
}

} // extern "C"
