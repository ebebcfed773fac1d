// Many acquisitions of uneven frame size and window length in one graph launch.
//
// hf_multi holds one plan per acquisition.  hf_multi_exec runs every acquisition's windows as a
// single CUDA graph: the graph forks into branches, each branch runs its share of the acquisitions
// back to back (hf_pipeline_exec, captured), and the branches join at the end, so one launch covers
// the whole set and small acquisitions fill the SMs that large ones leave idle.
// With a fused schedule, the acquisitions whose band pass is the tensor-core segment pass are split
// at that pass: their fronts (Gram matrices, eigenpairs, W) run first in their branches, then ONE
// persistent segment launch per group of acquisitions with the same window length and format takes
// every (acquisition, window, row, segment) unit of the group from one counter, and their backs
// (row pass, column pass and moments) follow in their branches.
// The schedule -- branches, assignment, fusion, and the fused launch's tiles per segment and grid
// cap -- is chosen by hf_multi_tune: it captures each candidate, times a few launches of each with
// CUDA events and keeps the fastest.  The graph is re-captured only when the schedule or the
// buffers change.
#include <algorithm>
#include <map>
#include <new>
#include <numeric>
#include <utility>
#include <vector>

#include "hf_common.cuh"
#include "holoflow_b200.h"
#include "pipeline_split.cuh"

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
bool same(const hf_multi_schedule &a, const hf_multi_schedule &b) {
  return a.branches == b.branches && a.largest_first == b.largest_first && a.fused == b.fused &&
         a.seg_tiles == b.seg_tiles && a.band_ctas == b.band_ctas;
}
} // namespace

struct hf_multi {
  std::vector<Acq>          acq;
  std::vector<cudaStream_t> branch;          // capture streams: [0] the capture origin, [k] branch k
  cudaStream_t              band = nullptr;  // capture stream of the fused segment launches
  std::vector<cudaEvent_t>  fork_ev, join_ev;
  std::vector<cudaEvent_t>  front_ev;        // per acquisition: its front is done
  std::vector<cudaEvent_t>  band_ev;         // per fused group: its segment launch is done
  int                      *counter = nullptr; // device unit counter of the fused launches (one stream)
  hf_multi_schedule         sch{1, 1, 0, 0, 0};
  cudaGraph_t               graph = nullptr;
  cudaGraphExec_t           exec  = nullptr;
  Buffers                   captured;
  hf_multi_schedule         cap_sch{0, 0, 0, 0, 0};
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

// Fused groups for these buffers: acquisitions that take the segment pass, by (format, window
// length), in chunks of at most kMaxSegJobs; only chunks of two or more are fused.
static std::vector<std::vector<int>> fused_groups(const hf_multi *m, const Buffers &b) {
  std::map<std::pair<int, int>, std::vector<int>> by;
  for (size_t i = 0; i < m->acq.size(); ++i)
    if (b.nwin[i] > 0 && pipeline_seg_eligible(m->acq[i].plan, b.rings[i]))
      by[{m->acq[i].d.input_dtype, m->acq[i].d.frames}].push_back((int)i);
  std::vector<std::vector<int>> groups;
  for (auto &kv : by)
    for (size_t c = 0; c < kv.second.size(); c += kMaxSegJobs) {
      const size_t e = std::min(kv.second.size(), c + kMaxSegJobs);
      if (e - c >= 2)
        groups.emplace_back(kv.second.begin() + (long)c, kv.second.begin() + (long)e);
    }
  return groups;
}

static int ensure_events(std::vector<cudaEvent_t> &v, size_t n) {
  while (v.size() < n) {
    cudaEvent_t e = nullptr;
    HF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    v.push_back(e);
  }
  return HF_OK;
}

// Captures the schedule on the executor's own origin stream (a graph is then launched on any
// stream; capture cannot start on the legacy default stream a caller may use).
static int capture(hf_multi *m, const Buffers &b, const hf_multi_schedule &sch) {
  drop_graph(m);
  cudaStream_t s  = m->branch[0];
  const auto   br = assign(m, sch.branches, sch.largest_first != 0);
  std::vector<std::vector<int>> groups;
  std::vector<int>              group_of(m->acq.size(), -1);
  if (sch.fused) {
    groups = fused_groups(m, b);
    for (size_t g = 0; g < groups.size(); ++g)
      for (int i : groups[g])
        group_of[(size_t)i] = (int)g;
    HF_TRY(ensure_events(m->band_ev, groups.size()));
  }
  const auto strm = [&](int k) { return k == 0 ? s : m->branch[(size_t)k]; };
  HF_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = cuda_status(cudaEventRecord(m->fork_ev[0], s), "fork");
  // each branch: the fronts of its fused acquisitions first, so the fused launches can start early,
  // then the whole pipeline of its other acquisitions
  for (int k = 0; k < sch.branches && rc == HF_OK; ++k) {
    cudaStream_t q = strm(k);
    if (k > 0)
      rc = cuda_status(cudaStreamWaitEvent(q, m->fork_ev[0], 0), "fork");
    for (int i : br[(size_t)k]) {
      if (rc != HF_OK || b.nwin[(size_t)i] <= 0 || group_of[(size_t)i] < 0)
        continue;
      rc = pipeline_front(m->acq[(size_t)i].plan, b.rings[(size_t)i], b.ring_frames[(size_t)i], b.first[(size_t)i],
                          b.nwin[(size_t)i], q);
      if (rc == HF_OK)
        rc = cuda_status(cudaEventRecord(m->front_ev[(size_t)i], q), "front");
    }
    for (int i : br[(size_t)k]) {
      if (rc != HF_OK || b.nwin[(size_t)i] <= 0 || group_of[(size_t)i] >= 0)
        continue;
      rc = hf_pipeline_exec(m->acq[(size_t)i].plan, b.rings[(size_t)i], b.ring_frames[(size_t)i], b.first[(size_t)i],
                            b.nwin[(size_t)i], b.outs[(size_t)i], q);
    }
  }
  // one persistent segment launch per group, in sequence on the band stream (each takes every SM
  // it is given, and the launches share the unit counter)
  for (size_t g = 0; g < groups.size() && rc == HF_OK; ++g) {
    std::vector<BandRowsArgs> jobs;
    for (int i : groups[g]) {
      if (rc == HF_OK)
        rc = cuda_status(cudaStreamWaitEvent(m->band, m->front_ev[(size_t)i], 0), "band wait");
      BandRowsArgs a{};
      if (rc == HF_OK)
        rc = pipeline_seg_job(m->acq[(size_t)i].plan, b.rings[(size_t)i], b.ring_frames[(size_t)i],
                              b.first[(size_t)i], b.nwin[(size_t)i], &a);
      jobs.push_back(a);
    }
    if (rc == HF_OK)
      rc = launch_band_seg_tc_multi(jobs.data(), (int)jobs.size(), m->acq[(size_t)groups[g][0]].d.input_dtype,
                                    sch.seg_tiles, sch.band_ctas, m->counter,
                                    plan_status_word(m->acq[(size_t)groups[g][0]].plan), m->band);
    if (rc == HF_OK)
      rc = cuda_status(cudaEventRecord(m->band_ev[g], m->band), "band");
  }
  // the backs of the fused acquisitions, each after its group's launch
  for (int k = 0; k < sch.branches && rc == HF_OK; ++k) {
    cudaStream_t q = strm(k);
    for (int i : br[(size_t)k]) {
      if (rc != HF_OK || b.nwin[(size_t)i] <= 0 || group_of[(size_t)i] < 0)
        continue;
      rc = cuda_status(cudaStreamWaitEvent(q, m->band_ev[(size_t)group_of[(size_t)i]], 0), "back wait");
      if (rc == HF_OK)
        rc = pipeline_back(m->acq[(size_t)i].plan, b.nwin[(size_t)i], b.outs[(size_t)i], q);
    }
    if (k > 0 && rc == HF_OK) {
      rc = cuda_status(cudaEventRecord(m->join_ev[(size_t)k], q), "join");
      if (rc == HF_OK)
        rc = cuda_status(cudaStreamWaitEvent(s, m->join_ev[(size_t)k], 0), "join");
    }
  }
  for (size_t g = 0; g < groups.size() && rc == HF_OK; ++g) // the band stream joins too
    rc = cuda_status(cudaStreamWaitEvent(s, m->band_ev[g], 0), "join");
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
  m->captured = b;
  m->cap_sch  = sch;
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
    rc = cuda_status(cudaStreamCreateWithFlags(&m->band, cudaStreamNonBlocking), "band stream");
  if (rc == HF_OK)
    rc = cuda_status(cudaEventCreateWithFlags(&m->fork_ev[0], cudaEventDisableTiming), "event");
  for (int k = 0; k < kMaxBranches && rc == HF_OK; ++k)
    rc = cuda_status(cudaEventCreateWithFlags(&m->join_ev[(size_t)k], cudaEventDisableTiming), "event");
  if (rc == HF_OK)
    rc = ensure_events(m->front_ev, m->acq.size());
  if (rc == HF_OK)
    rc = cuda_status(cudaMalloc(reinterpret_cast<void **>(&m->counter), sizeof(int)), "unit counter");
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
  if (m->band)
    cudaStreamDestroy(m->band);
  for (auto *v : {&m->fork_ev, &m->join_ev, &m->front_ev, &m->band_ev})
    for (cudaEvent_t e : *v)
      if (e)
        cudaEventDestroy(e);
  if (m->counter)
    cudaFree(m->counter);
  delete m;
  return HF_OK;
}

int hf_multi_exec(hf_multi *m, const void *const *rings, const int64_t *ring_frames, const int64_t *first,
                  const int *nwin, float *const *outs, hf_stream_t s) {
  clear_error();
  HF_CHECK_ARG(m != nullptr && rings != nullptr && ring_frames != nullptr && first != nullptr && outs != nullptr,
               "hf_multi_exec: null argument");
  const Buffers b = buffers_of(m, rings, ring_frames, first, nwin, outs);
  if (!m->exec || !(b == m->captured) || !same(m->cap_sch, m->sch))
    HF_TRY(capture(m, b, m->sch));
  HF_CUDA(cudaGraphLaunch(m->exec, s));
  note_launch();
  return HF_OK;
}

// Candidate schedules, in the order they are timed: branches x assignment without fusion; then,
// when the buffers hold a fused group, fusion at each branch count with the best assignment; then
// the fused launch's tile parameters (tiles per segment, grid cap) at the best of those.
int hf_multi_tune(hf_multi *m, const void *const *rings, const int64_t *ring_frames, const int64_t *first,
                  const int *nwin, float *const *outs, int reps, hf_stream_t s, int *best_streams, float *best_ms) {
  clear_error();
  HF_CHECK_ARG(m != nullptr && reps >= 1, "hf_multi_tune: bad argument");
  HF_CHECK_ARG(rings != nullptr && ring_frames != nullptr && first != nullptr && outs != nullptr,
               "hf_multi_tune: null argument");
  const Buffers b  = buffers_of(m, rings, ring_frames, first, nwin, outs);
  cudaEvent_t   e0 = nullptr, e1 = nullptr;
  HF_CUDA(cudaEventCreate(&e0));
  HF_CUDA(cudaEventCreate(&e1));
  float             best = 1e30f;
  hf_multi_schedule bs   = m->sch;
  int               rc   = HF_OK;
  const auto time_one = [&](const hf_multi_schedule &c) {
    if (rc != HF_OK || c.branches > (int)m->acq.size())
      return;
    if ((rc = capture(m, b, c)) != HF_OK)
      return;
    cudaGraphLaunch(m->exec, s); // warm-up
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; ++r)
      cudaGraphLaunch(m->exec, s);
    cudaEventRecord(e1, s);
    if ((rc = cuda_status(cudaEventSynchronize(e1), "hf_multi_tune")) != HF_OK)
      return;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= (float)reps;
    if (ms < best)
      best = ms, bs = c;
  };
  const int branch_counts[] = {1, 2, 3, 4, 6};
  for (int ns : branch_counts)
    for (int lpt : {1, 0})
      if (ns > 1 || lpt)
        time_one(hf_multi_schedule{ns, lpt, 0, 0, 0});
  if (rc == HF_OK && !fused_groups(m, b).empty()) {
    const int lpt = bs.largest_first;
    for (int ns : branch_counts)
      time_one(hf_multi_schedule{ns, lpt, 1, 0, 0});
    if (bs.fused) {
      const hf_multi_schedule f = bs;
      for (int tiles : {0, 4, 2})
        for (int ctas : {0, 3 * sm_count() / 4})
          if (tiles != 0 || ctas != 0)
            time_one(hf_multi_schedule{f.branches, f.largest_first, 1, tiles, ctas});
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  HF_TRY(rc);
  m->sch = bs;
  drop_graph(m); // the next exec captures the chosen schedule
  if (best_streams)
    *best_streams = bs.largest_first ? bs.branches : -bs.branches;
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

int hf_multi_get_schedule(const hf_multi *m, hf_multi_schedule *sch) {
  clear_error();
  HF_CHECK_ARG(m != nullptr && sch != nullptr, "hf_multi_get_schedule: null argument");
  *sch = m->sch;
  return HF_OK;
}

int hf_multi_set_schedule(hf_multi *m, const hf_multi_schedule *sch) {
  clear_error();
  HF_CHECK_ARG(m != nullptr && sch != nullptr, "hf_multi_set_schedule: null argument");
  HF_CHECK_ARG(sch->branches >= 1 && sch->branches <= kMaxBranches, "hf_multi_set_schedule: branches must be in [1, 6]");
  HF_CHECK_ARG((sch->largest_first == 0 || sch->largest_first == 1) && (sch->fused == 0 || sch->fused == 1),
               "hf_multi_set_schedule: largest_first and fused are 0 or 1");
  HF_CHECK_ARG(sch->seg_tiles >= 0 && sch->band_ctas >= 0, "hf_multi_set_schedule: negative tile parameter");
  m->sch = *sch;
  return HF_OK;
}

} // extern "C"
