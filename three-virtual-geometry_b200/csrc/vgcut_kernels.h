// Host-callable launchers of the cut engine's kernels (vgcut_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "vgcut_internal.h"

namespace vgc {

// Resident 128-thread blocks per SM of the instance / chunk kernels (their persistent grid size); multi: the
// variants of a multi-scene launch.
cudaError_t configure_select(bool multi, int *instances_per_sm, int *chunks_per_sm);
// ctl: per-batch control words: [0] visible units, [1..2] a view redoes a cut in round 1..2, [3] chunks queued
cudaError_t launch_reset(const ViewConst *views, uint32_t nviews, uint32_t *ctl, cudaStream_t st);
// Scene arguments: a launch over one context passes its Scene and scenes = nullptr; a multi-scene launch passes
// a device table of Scene records that each view's `scene` indexes (S is then unused).
cudaError_t launch_cells(const Scene &S, const Scene *scenes, const ViewConst *views, uint32_t nviews,
                         uint32_t total_units, uint2 *units, uint32_t *unit_count, cudaStream_t st);
// round < 0: the triangleBudget search's histogram pass (k_instances / k_chunks), then launch_budget picks the
// threshold of each budget view.
cudaError_t launch_budget(const ViewConst *views, uint32_t nviews, uint32_t *ctl, cudaStream_t st);
// chunk_shift: windows of 2^chunk_shift meshlets per chunk (kChunkShiftMin..Max; the default 9 = 512 meshlets).
// overflow: a bit per warp-unit (4 per unit of `units`), zero between passes: k_instances marks the units whose
// items did not fit the queue, and launch_instances_redo (after launch_chunks of the same pass) tests their items
// in place and clears the bits.
cudaError_t launch_instances(const Scene &S, const Scene *scenes, const ViewConst *views, const uint2 *units,
                             uint32_t *ctl, uint4 *queue, uint32_t capacity, int round, uint32_t grid,
                             uint32_t *overflow, cudaStream_t st, uint32_t chunk_shift = kChunkShiftDefault);
cudaError_t launch_instances_redo(const Scene &S, const Scene *scenes, const ViewConst *views, const uint2 *units,
                                  uint32_t *ctl, uint4 *queue, uint32_t capacity, int round, uint32_t *overflow,
                                  uint32_t grid, cudaStream_t st, uint32_t chunk_shift = kChunkShiftDefault);
// The meshlet work queue (spans and chunks) lives in `queue`, `capacity` uint4 entries; ctl[4..5] counts it.
cudaError_t launch_chunks(const Scene &S, const Scene *scenes, const ViewConst *views, uint4 *queue,
                          uint32_t *ctl, uint32_t capacity, int round, uint32_t grid, cudaStream_t st);
// 32 words per view: the VGC_COUNTER_HEADER counter words, then the threshold the cut used (float bits).
cudaError_t launch_gather_stats(const ViewConst *views, uint32_t nviews, uint32_t *out, cudaStream_t st);
// computeCell on the device for n cells from c0 of one mesh (bit-identical to the host's computation).
cudaError_t launch_cells_update(const float4 *inst, const double sphere[4], uint32_t instance_base,
                                uint32_t instance_count, uint32_t cell_base, uint32_t slot, uint32_t c0, uint32_t n,
                                CellRec *cells, cudaStream_t st);
cudaError_t launch_finish(const ViewConst *views, uint32_t nviews, uint32_t *ctl, int round, cudaStream_t st);
cudaError_t launch_expand(const Scene &S, const ViewConst *view, uint32_t cut, uint32_t *out, uint64_t capacity,
                          uint32_t grid, cudaStream_t st);
cudaError_t launch_hzb(const float *depth, const HzbDesc &H, float *out, int copy_mip0, cudaStream_t st);
// HZB builds of the views whose constants carry build_hzb (grid covers the largest depth image).
cudaError_t launch_hzb_views(const ViewConst *views, uint32_t nviews, uint32_t max_w,
                             uint32_t max_h, bool tail, cudaStream_t st);
// The same builds as one stream of strips (k_hzb_stream, levels 0..4) from the launch's HZB plan in device memory;
// `grid` blocks (hzb_stream_blocks_per_sm() per SM), then the tail kernel for levels 5+ when `tail`.
cudaError_t launch_hzb_stream(const unsigned char *plan, uint32_t grid, const ViewConst *views, uint32_t nviews,
                              bool tail, cudaStream_t st);
// The bounded mbarrier wait of the strip stream on a barrier nothing completes (out[0]: completed, out[1]: ns waited).
cudaError_t launch_wait_probe(uint64_t limit_ns, unsigned long long *out, cudaStream_t st);
// Blocks of k_hzb_stream resident per SM (sets its shared-memory limit on the first call for the current device).
uint32_t hzb_stream_blocks_per_sm();
cudaError_t launch_select_cut(const Scene &S, uint32_t slot, uint32_t mcount, uint32_t count, const float *vm16,
                              const float *params, float threshold, float blend, uint8_t *lo, uint8_t *hi, uint32_t grid,
                              cudaStream_t st);

}  // namespace vgc
