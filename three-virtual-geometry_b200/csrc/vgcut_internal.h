// Device data layout shared by the kernels and the host context of the cut engine.
//
// HBM layout of a resident scene (one context):
//   meshes      MeshRec[slot_capacity]            mesh table (GeometryPool.ts:449-460: spheres, levers, flags)
//   levels      LevelRec[]                        level tables (GeometryPool.ts:432-445), 32 B per level
//   m_lod       float4[M]  LOD sphere              | meshletBounds (buildVirtualMesh.ts:85-91) split into
//   m_parent    float4[M]  parent LOD sphere       | structure-of-arrays so each pass reads only the 16-byte
//   m_err       float4[M]  (error, parentError,    | columns it needs, coalesced (one float4 per lane), in
//                           triCount bits, id)     | the engine's test order (m_err.w: pool-global meshlet id)
//   m_cull      float4[M]  culling sphere          |
//   m_info      uint4[M]   triangleCount, firstIndex (pool-global), lodLevel, vertexOffset (pool-global)
//   positions   float4[]   vertex positions of the meshes that carry vertex data (occluders), pool-global
//   m_verts     u32[]      meshlet-local -> pool-global vertex id (meshletVertices)
//   m_tris      u32[]      packed local triangles (meshletTriangles), pool-global
//   lsamples    float2[64 * levels]  per level, at positions k * count / 64 of its meshlets in test order: the
//                          parent error there (non-decreasing) and the smallest own error from there to the level's end
//   inst        float4[4 I] instance matrix columns, Morton order per mesh (GeometryPool.ts:484-497)
//   inst_slot   u32[I]     mesh slot of each instance
//   cells       CellRec[C] 128 consecutive instances of one mesh (GeometryPool.ts:519-545)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "vgcut.h"

namespace vgc {

constexpr uint32_t kCellSize = 128;        // GeometryPool.ts:96
constexpr uint32_t kMaxLevels = 48;        // GeometryPool.ts:101
constexpr uint32_t kFastPathMax = 4;       // constants.ts FAST_PATH_MAX_MESHLETS
constexpr uint32_t kFullFadeBits = 255u << 16;
constexpr uint32_t kLocalVertexBits = 7;   // ceil(log2(MAX_MESHLET_VERTICES = 128))
constexpr uint32_t kMaxHzbLevels = 16;
constexpr uint32_t kStateWords = 8;        // S_SCALE 0..1, S_FILL 2..3, S_RETRY 4..5
constexpr uint32_t kBudgetBins = 256;
constexpr uint32_t kChunkShiftMin = 8, kChunkShiftDefault = 9, kChunkShiftMax = 10;  // meshlets per chunk: 256..1024
#ifndef VGC_RETRY_CHUNK_SHIFT
// meshlets per chunk in the retry rounds: 2^shift (0: as in round 0). The few views a retry round usually redoes
// spread over more warps with 256-meshlet chunks (a view's retry: 0.51 -> 0.49 ms per 32-view step; 64-meshlet chunks:
// 0.48 ms, but 7% slower when most views redo)
#define VGC_RETRY_CHUNK_SHIFT 8
#endif
constexpr uint32_t kChunkShiftRetry = VGC_RETRY_CHUNK_SHIFT, kChunkShiftFloor = 6;
constexpr uint32_t kLevelSamples = 64;     // per level: samples of the meshlets in test order (item trimming)

struct MeshRec {  // 96 bytes
  float4 sphere;
  float4 lod;
  float4 cull;
  float max_draw_distance, min_pixel_radius;
  uint32_t level_count, level_base;
  uint32_t enabled, shadow, occlusion, meshlet_base;
  uint32_t range_cut;  // 1: every meshlet's LOD and parent spheres lie in `lod`, so items may be trimmed
  uint32_t occluder;   // 1: drawn by the occluder depth pass (has vertex data)
  uint32_t vertices;   // 1: the mesh carries vertex data (positions, meshletVertices)
  uint32_t pad;
};

struct LevelRec {  // 32 bytes
  uint32_t first, count;
  float min_own, max_parent, max_own, min_parent;
  uint32_t pad0, pad1;
};

struct CellRec {  // 32 bytes
  float4 sphere;
  float max_radius;
  uint32_t slot, first, count;
};

struct Scene {
  const MeshRec *meshes;
  const LevelRec *levels;
  const float4 *m_lod, *m_parent, *m_err, *m_cull;
  const uint4 *m_info;
  const uint32_t *m_tris;
  const float2 *lsamples;  // kLevelSamples per level (global level index)
  const float4 *positions;  // vertex positions (meshes with vertex data)
  const uint32_t *m_verts;  // meshletVertices
  const float4 *inst;
  const uint32_t *inst_slot;
  const CellRec *cells;
  const struct HzbDesc *hzbs;  // the context's HZB slot descriptors (ViewConst::hzb indexes them)
  uint32_t cell_count, instance_count, meshlet_count, slot_capacity, slots_used;
};

struct HzbDesc {
  const float *data;
  uint32_t levels;
  uint32_t off[kMaxHzbLevels], w[kMaxHzbLevels], h[kMaxHzbLevels];
};

// The HZB builds of one launch sequence as one stream of 128 x 32 mip-0 strips (k_hzb_stream): a header, one job per
// view that brings a depth image, then one tensor map per job. Written on the host into pinned memory and copied
// with the view constants.
struct HzbPlanHead {
  uint32_t jobs, tiles;  // jobs; strips of all jobs
  uint32_t maps;         // byte offset of the tensor maps (kTensorMapBytes each, in job order)
  uint32_t pad[13];
};
struct HzbJob {
  const float *depth;    // the view's depth image: mip 0
  const HzbDesc *desc;   // the HZB slot's descriptor (device)
  uint32_t *error;       // the view's VGC_COUNTER_ERROR word
  uint32_t tile0;        // the job's first strip in the stream; strip tile0 + y * tiles_x + x is at (128 x, 32 y)
  uint16_t tiles_x;
  uint8_t tma;           // 1: the job's tensor map describes the depth image (else plain loads)
  uint8_t copy_mip0;     // 1: mip 0 is copied into the slot (0: the cut reads it from the depth image)
};
constexpr uint32_t kTensorMapBytes = 128;  // CUtensorMap, 64-byte aligned
constexpr uint32_t kHzbStripW = 128, kHzbStripH = 32;  // strip of the stream (and box of its tensor maps)
__host__ __device__ constexpr size_t hzb_plan_maps(uint32_t jobs) {  // byte offset of the tensor maps
  return sizeof(HzbPlanHead) + (((size_t)jobs * sizeof(HzbJob) + 63) & ~size_t(63));
}
__host__ __device__ constexpr size_t hzb_plan_bytes(uint32_t jobs) {
  return hzb_plan_maps(jobs) + (size_t)jobs * kTensorMapBytes;
}
static_assert(sizeof(HzbJob) == 32 && sizeof(HzbPlanHead) == 64, "plan layout");

// Per-view constants derived on the host in double precision (VirtualGeometry.ts:414-442) and stored as float.
struct ViewConst {
  float V[12];        // rows 0..2 of world->view, row-major 3x4
  float plane[24];    // 6 view-space frustum planes (xyz normal, w), normalised (a cascade's: its clip volume)
  float sweep[6];     // per-plane max(dot(world normal, shadowSweep), 0)
  float proj_scale, near_, P0, P5, P8, P9, P10, P14;
  float inv_proj_scale;  // 1 / proj_scale, rounded once from double
  float error_threshold, lod_blend_max, shadow_error_scale, lod_scale_limit, min_pixel_radius;
  float budget, budget_lo, budget_hi;  // triangleBudget search (0 = off)
  uint32_t frustum, occl_active;
  uint32_t unit_offset;  // first padded (view, cell) unit of this view in the cell pass
  uint32_t max_drawn;
  uint32_t index_capacity[2];
  int32_t hzb;          // HZB slot or -1
  uint32_t build_hzb;   // 1: build HZB slot `hzb` from `depth` before the cut
  uint32_t fresh_state; // 1: k_reset puts the controller state back to its initial words first
  uint32_t cascade;     // 1: shadow cascade (no camera cut; plane[] are the cascade's planes, sweep[] zero)
  const float *depth;   // occluder depth of this frame (build_hzb)
  const float *hzb_mip0;  // VGC_VIEW_DEPTH_AS_MIP0: the HZB's mip 0 is `depth` (not copied into the slot); else null
  uint32_t *counters;   // VGC_COUNTER_* header, then per (cut, slot, part): count, start
  uint32_t *state;      // kStateWords, carried between frames
  uint4 *draw_list;     // 2 * max_drawn
  uint32_t *draw_args;  // 2 cuts * slot_capacity * 2 parts * 5
  float *dyn;           // [0] error threshold of this frame (errorThreshold or the budget search result),
                        // [1..5] its bands: low (cut 0, 1), high (cut 0, 1), fade scale
  unsigned long long *hist;  // 2 * kBudgetBins: triangles entering / leaving the cut per threshold bin
  unsigned long long budget_tris;  // triangleBudget as an integer (the search compares T(t) <= budget_tris)
  const HzbDesc *hzb_desc;  // the HZB slot's descriptor in the view's context (null without an HZB; HZB builds)
  uint32_t scene;           // multi-scene launch: the view's entry in the launch's scene table (else 0)
  uint32_t slot_capacity;   // the view's context: mesh slots its counters and draw args are laid out for,
  uint32_t slots_used;      //   slots in use,
  uint32_t counter_words;   //   counter words of one output slot
};

#ifdef __CUDACC__
// Work handed out to warps from a counter, B consecutive pieces at a time (a warp that drew cheap pieces takes more,
// so a persistent grid finishes together). Lane 0 requests the warp's next batch a whole batch ahead, so the
// counter's round trip overlaps the work; B > 1 keeps the counter's rate of atomics down when pieces are short.
// All lanes of the warp call start() and next() together; `i` is the current piece.
template <uint32_t B>
struct WarpFeed {
  uint32_t *ctr;
  uint32_t ahead;  // lane 0: the batch after the current one
  uint32_t i, end;
  __device__ __forceinline__ void start(uint32_t *counter) {
    ctr = counter;
    ahead = 0;
    if ((threadIdx.x & 31) == 0) ahead = atomicAdd(ctr, 1u);
    take();
  }
  __device__ __forceinline__ void take() {
    const uint32_t b = __shfl_sync(0xffffffffu, ahead, 0);
    if ((threadIdx.x & 31) == 0) ahead = atomicAdd(ctr, 1u);
    i = b * B;
    end = i + B;
  }
  // moves to the next piece and returns it
  __device__ __forceinline__ uint32_t next() {
    if (++i == end) take();
    return i;
  }
};
#endif

}  // namespace vgc
