// Many acquisitions of uneven frame size and window length in one graph launch.
//
// hf_multi holds one plan per acquisition.  hf_multi_exec runs every acquisition's windows as a
// single CUDA graph: the graph forks into `nstreams` branches, each branch runs its share of the
// acquisitions back to back (hf_pipeline_exec, captured), and the branches join at the end, so one
// launch covers the whole set and small acquisitions fill the SMs that large ones leave idle.
// The schedule -- how many branches and which acquisition goes to which -- is chosen by
// hf_multi_tune: it captures each candidate (1, 2, 3, 4 or 6 branches; acquisitions dealt
// largest-first to the least-loaded branch, or round-robin in the given order), times a few
// launches of each with CUDA events and keeps the fastest.  The graph is re-captured only when
// the schedule or the buffers change.
#include <algorithm>
#include <new>
#include <numeric>
#include <vector>

#include "hf_common.cuh"
#include "holoflow_b200.h"

using namespace hf;

namespace {
struct Acq {
  hf_desc  d{};
  hf_plan *plan = nullptr;
  double   cost = 0.0; // bytes the acquisition's windows stream per exec (the schedule's weight)
};
struct Buffers {
  std::vector<const void *> rings;
  std::vector<int64_t>      ring_frames, first;
  std::vector<int>          nwin;
  std::vector<float *>      outs;
  bool operator==(const Buffers &o) const {
    return rings == o.rings && ring_frames == o.ring_frames && first == o.first && nwin == o.nwin && outs == o.outs;
  }
};
} // namespace

struct hf_multi {
  std::vector<Acq>          acq;
  std::vector<cudaStream_t> branch;          // capture streams: [0] the capture origin, [k] branch k
  std::vector<cudaEvent_t>  fork_ev, join_ev;
  int                       nstreams = 1;
  bool                      lpt      = true;  // largest-first assignment (else round-robin)
  cudaGraph_t               graph    = nullptr;
  cudaGraphExec_t           exec     = nullptr;
  Buffers                   captured;
  int                       cap_nstreams = 0;
  bool                      cap_lpt      = true;
};

static constexpr int kMaxBranches = 6;

static void drop_graph(hf_multi *m) {
  if (m->exec)
    cudaGraphExecDestroy(m->exec);
  if (m->graph)
    cudaGraphDestroy(m->graph);
  m->exec  = nullptr;
  m->graph = nullptr;
}

// Acquisition order per branch for a schedule.
static std::vector<std::vector<int>> assign(const hf_multi *m, int nstreams, bool lpt) {
  std::vector<std::vector<int>> br((size_t)nstreams);
  std::vector<int>              order(m->acq.size());
  std::iota(order.begin(), order.end(), 0);
  if (lpt) {
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return m->acq[a].cost > m->acq[b].cost; });
    std::vector<double> load((size_t)nstreams, 0.0);
    for (int i : order) {
      const size_t k = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
      br[k].push_back(i);
      load[k] += m->acq[i].cost;
    }
  } else {
    for (size_t i = 0; i < order.size(); ++i)
      br[i % (size_t)nstreams].push_back(order[i]);
  }
  return br;
}

// Captures the schedule on the executor's own origin stream (a graph is then launched on any
// stream; capture cannot start on the legacy default stream a caller may use).
static int capture(hf_multi *m, const Buffers &b, int nstreams, bool lpt) {
  drop_graph(m);
  cudaStream_t s = m->branch[0];
  const auto br = assign(m, nstreams, lpt);
  HF_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = cuda_status(cudaEventRecord(m->fork_ev[0], s), "fork");
  for (int k = 0; k < nstreams && rc == HF_OK; ++k) {
    cudaStream_t q = k == 0 ? s : m->branch[(size_t)k];
    if (k > 0)
      rc = cuda_status(cudaStreamWaitEvent(q, m->fork_ev[0], 0), "fork");
    for (int i : br[(size_t)k]) {
      if (rc != HF_OK || b.nwin[(size_t)i] <= 0)
        continue;
      rc = hf_pipeline_exec(m->acq[(size_t)i].plan, b.rings[(size_t)i], b.ring_frames[(size_t)i], b.first[(size_t)i],
                            b.nwin[(size_t)i], b.outs[(size_t)i], q);
    }
    if (k > 0 && rc == HF_OK) {
      rc = cuda_status(cudaEventRecord(m->join_ev[(size_t)k], q), "join");
      if (rc == HF_OK)
        rc = cuda_status(cudaStreamWaitEvent(s, m->join_ev[(size_t)k], 0), "join");
    }
  }
  const std::string err = rc == HF_OK ? "" : hf_last_error();
  cudaGraph_t       g   = nullptr;
  const cudaError_t e   = cudaStreamEndCapture(s, &g);
  if (rc != HF_OK) {
    if (g)
      cudaGraphDestroy(g);
    set_error(err);
    return rc;
  }
  HF_CUDA(e);
  m->graph = g;
  HF_CUDA(cudaGraphInstantiate(&m->exec, m->graph, 0));
  m->captured     = b;
  m->cap_nstreams = nstreams;
  m->cap_lpt      = lpt;
  return HF_OK;
}

static Buffers buffers_of(const hf_multi *m, const void *const *rings, const int64_t *ring_frames, const int64_t *first,
                          const int *nwin, float *const *outs) {
  Buffers b;
  const size_t n = m->acq.size();
  b.rings.assign(rings, rings + n);
  b.ring_frames.assign(ring_frames, ring_frames + n);
  b.first.assign(first, first + n);
  b.outs.assign(outs, outs + n);
  b.nwin.resize(n);
  for (size_t i = 0; i < n; ++i)
    b.nwin[i] = nwin ? nwin[i] : m->acq[i].d.max_batch;
  return b;
}

extern "C" {

int hf_multi_create(int n, const hf_desc *descs, hf_multi **out) {
  clear_error();
  HF_CHECK_ARG(n >= 1 && n <= 4096 && descs != nullptr && out != nullptr, "hf_multi_create: bad argument");
  *out   = nullptr;
  auto m = new (std::nothrow) hf_multi();
  if (!m)
    return fail(HF_ERR_NOMEM, "hf_multi_create: host allocation failed");
  int rc = HF_OK;
  for (int i = 0; i < n && rc == HF_OK; ++i) {
    Acq a;
    a.d = descs[i];
    rc  = hf_plan_create(&descs[i], &a.plan, nullptr);
    if (rc == HF_OK) {
      const double px = (double)a.d.height * a.d.width, nz = a.d.z_end - a.d.z_begin;
      a.cost          = (double)a.d.max_batch * px * (1.5 * a.d.frames + 16.0 * nz);
      m->acq.push_back(a);
    }
  }
  m->branch.resize(kMaxBranches, nullptr);
  m->fork_ev.resize(1, nullptr);
  m->join_ev.resize(kMaxBranches, nullptr);
  for (int k = 0; k < kMaxBranches && rc == HF_OK; ++k)
    rc = cuda_status(cudaStreamCreateWithFlags(&m->branch[(size_t)k], cudaStreamNonBlocking), "branch stream");
  if (rc == HF_OK)
    rc = cuda_status(cudaEventCreateWithFlags(&m->fork_ev[0], cudaEventDisableTiming), "event");
  for (int k = 0; k < kMaxBranches && rc == HF_OK; ++k)
    rc = cuda_status(cudaEventCreateWithFlags(&m->join_ev[(size_t)k], cudaEventDisableTiming), "event");
  if (rc != HF_OK) {
    const std::string err = hf_last_error();
    hf_multi_destroy(m);
    set_error(err);
    return rc;
  }
  *out = m;
  return HF_OK;
}

int hf_multi_destroy(hf_multi *m) {
  if (!m)
    return HF_OK;
  cudaDeviceSynchronize();
  drop_graph(m);
  for (auto &a : m->acq)
    hf_plan_destroy(a.plan);
  for (cudaStream_t q : m->branch)
    if (q)
      cudaStreamDestroy(q);
  for (cudaEvent_t e : m->fork_ev)
    if (e)
      cudaEventDestroy(e);
  for (cudaEvent_t e : m->join_ev)
    if (e)
      cudaEventDestroy(e);
  delete m;
  return HF_OK;
}

int hf_multi_exec(hf_multi *m, const void *const *rings, const int64_t *ring_frames, const int64_t *first,
                  const int *nwin, float *const *outs, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(m != nullptr && rings != nullptr && ring_frames != nullptr && first != nullptr && outs != nullptr,
               "hf_multi_exec: null argument");
  const Buffers b = buffers_of(m, rings, ring_frames, first, nwin, outs);
  if (!m->exec || !(b == m->captured) || m->cap_nstreams != m->nstreams || m->cap_lpt != m->lpt)
    HF_TRY(capture(m, b, m->nstreams, m->lpt));
  HF_CUDA(cudaGraphLaunch(m->exec, s));
  note_launch();
  return HF_OK;
}

int hf_multi_tune(hf_multi *m, const void *const *rings, const int64_t *ring_frames, const int64_t *first,
                  const int *nwin, float *const *outs, int reps, hf_stream_t s, int *best_streams, float *best_ms) {
  clear_error();
  HF_CHECK_ARG(m != nullptr && reps >= 1, "hf_multi_tune: bad argument");
  const Buffers b   = buffers_of(m, rings, ring_frames, first, nwin, outs);
  cudaEvent_t   e0 = nullptr, e1 = nullptr;
  HF_CUDA(cudaEventCreate(&e0));
  HF_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int   bn = 1;
  bool  bl = true;
  int   rc = HF_OK;
  for (int ns : {1, 2, 3, 4, 6}) {
    if (ns > (int)m->acq.size())
      continue;
    for (bool lpt : {true, false}) {
      if (ns == 1 && !lpt)
        continue;
      if ((rc = capture(m, b, ns, lpt)) != HF_OK)
        break;
      cudaGraphLaunch(m->exec, s); // warm-up
      cudaEventRecord(e0, s);
      for (int r = 0; r < reps; ++r)
        cudaGraphLaunch(m->exec, s);
      cudaEventRecord(e1, s);
      if ((rc = cuda_status(cudaEventSynchronize(e1), "hf_multi_tune")) != HF_OK)
        break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= (float)reps;
      if (ms < best) {
        best = ms, bn = ns, bl = lpt;
      }
    }
    if (rc != HF_OK)
      break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  HF_TRY(rc);
  m->nstreams = bn;
  m->lpt      = bl;
  drop_graph(m); // the next exec captures the chosen schedule
  if (best_streams)
    *best_streams = bl ? bn : -bn;
  if (best_ms)
    *best_ms = best;
  return HF_OK;
}

int hf_multi_plan(hf_multi *m, int i, hf_plan **plan) {
  clear_error();
  HF_CHECK_ARG(m != nullptr && plan != nullptr && i >= 0 && i < (int)m->acq.size(), "hf_multi_plan: bad index");
  *plan = m->acq[(size_t)i].plan;
  return HF_OK;
}

} // extern "C"
