// Host-callable launchers of the cut engine's kernels (vgcut_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "vgcut_internal.h"

namespace vgc {

size_t select_smem_bytes();
// Sets k_select's shared-memory limit and returns its resident blocks per SM.
cudaError_t configure_select(int *blocks_per_sm);
cudaError_t launch_reset(const ViewConst *views, uint32_t nviews, uint32_t words, uint32_t *unit_count, cudaStream_t st);
cudaError_t launch_cells(const Scene &S, const ViewConst *views, uint32_t nviews, uint32_t total_units, uint2 *units,
                         uint32_t *unit_count, cudaStream_t st);
cudaError_t launch_select(const Scene &S, const ViewConst *views, const HzbDesc *hzbs, const uint2 *units,
                          const uint32_t *unit_count, int round, uint32_t grid, cudaStream_t st);
cudaError_t launch_finish(const ViewConst *views, uint32_t nviews, uint32_t slot_capacity, uint32_t slots_used,
                          int round, cudaStream_t st);
cudaError_t launch_expand(const Scene &S, const ViewConst *view, uint32_t cut, uint32_t *out, uint64_t capacity,
                          uint32_t grid, cudaStream_t st);
cudaError_t launch_hzb(const float *depth, const HzbDesc &H, float *out, int copy_mip0, cudaStream_t st);
cudaError_t launch_select_cut(const Scene &S, uint32_t slot, uint32_t mcount, uint32_t count, const float *vm16,
                              const float *params, float threshold, float blend, uint8_t *lo, uint8_t *hi, uint32_t grid,
                              cudaStream_t st);

}  // namespace vgc
