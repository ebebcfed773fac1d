// Split form of hf_pipeline_exec (pipeline.cu) for the multi-acquisition executor (host/multi.cc).
// For a plan whose band pass is the tensor-core segment pass, hf_pipeline_exec equals
//   pipeline_front -> launch_band_seg_tc_multi over the job of pipeline_seg_job -> pipeline_back
// on one stream order, so the segment passes of several acquisitions can share one persistent
// launch.
#pragma once

#include "holoflow_b200.h"
#include "k_tc_band.cuh"

namespace hf {

// The plan takes the segment pass for frames in `ring` (chosen form, a shape outside the fused row
// pass, a 16-byte aligned ring).
bool pipeline_seg_eligible(const hf_plan *p, const void *ring);
// Gram matrices, eigenpairs and W of nwin windows (nothing without the clutter filter).
int pipeline_front(hf_plan *p, const void *ring, int64_t ring_frames, int64_t first, int nwin, cudaStream_t s);
// The segment pass's arguments for these windows (into the plan's band planes).
int pipeline_seg_job(hf_plan *p, const void *ring, int64_t ring_frames, int64_t first, int nwin, BandRowsArgs *job);
// Filter2D, the autofocus, propagation and moments of the band planes into `out`.
int pipeline_back(hf_plan *p, int nwin, float *out, cudaStream_t s);
// The plan's device status word (bounded waits).
int *plan_status_word(hf_plan *p);

} // namespace hf
