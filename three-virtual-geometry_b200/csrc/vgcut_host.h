// Host-side state of the cut engine shared by the translation units of libvgcut: the opaque context and batch
// types of include/vgcut.h, launch scratch, and the helpers the serving loop reuses from the plain path.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "vgcut.h"
#include "vgcut_internal.h"

using namespace vgc;

namespace vgch {

// Records `msg` as this thread's last error (vgc_last_error) and returns `code`.
int fail(int code, const std::string &msg);

#define CUDA_TRY(expr)                                                                              \
  do {                                                                                              \
    cudaError_t _e = (expr);                                                                        \
    if (_e != cudaSuccess) return fail(VGC_DEVICE_ERROR, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
};

struct MeshHost {
  bool used = false;
  uint32_t meshlet_base = 0, meshlet_count = 0;
  uint32_t level_base = 0, level_count = 0;
  uint32_t triangle_base = 0, triangle_count = 0;
  uint32_t instance_base = 0, instance_count = 0;
  uint32_t cell_base = 0, cell_count = 0;
  uint32_t vertex_base = 0, vertex_count = 0;  // vertex data (0 when the mesh has none)
  float sphere[4];
};

struct HzbSlot {
  DevBuf data;
  HzbDesc desc{};
  bool valid = false;
};

inline uint32_t pad32(uint32_t x) { return (x + 31u) & ~31u; }

}  // namespace vgch

using namespace vgch;

// Launch scratch: view constants and the (view, cell) unit list of one launch sequence.
struct LaunchScratch {
  vgc_context *owner = nullptr;   // the context whose byte count holds this scratch's device buffers
  uint32_t hzb_w = 0, hzb_h = 0;  // largest depth image the views of this launch build an HZB from (0: none)
  bool hzb_tail = false;
  bool any_budget = false;        // a view of this launch searches its threshold for a triangleBudget
  ViewConst *h_views = nullptr;  // pinned
  ViewConst *d_views = nullptr;
  uint2 *d_units = nullptr;
  uint32_t *d_overflow = nullptr;   // after d_units' entries: a bit per warp-unit (launch_instances), zero between passes
  uint32_t *d_unit_count = nullptr;  // control words (see launch_reset)
  uint4 *d_chunks = nullptr;      // meshlet work queue (spans and chunks)
  uint32_t chunk_capacity = 0;    // its entries
  uint32_t queue_want = 0;        // entries the last launch sequence asked for (grown to before the next one)
  uint32_t *h_ctl = nullptr;      // pinned copy of the control words at the end of the last launch sequence
  uint32_t grid_instances = 0;    // persistent grids of k_instances / k_chunks (0: the context's occupancy defaults)
  uint32_t grid_chunks = 0;
  uint32_t chunk_shift = kChunkShiftDefault;  // 2^chunk_shift meshlets per k_chunks work unit
  uint32_t view_capacity = 0;
  size_t unit_capacity = 0;
  size_t units_total = 0;         // (view, cell) units of the prepared launch (each view: its scene's cells, padded)
  bool multi = false;             // the prepared views belong to several contexts (a multi-scene launch)
  Scene *h_scenes = nullptr;      // pinned: the multi-scene launch's scene table (ViewConst::scene indexes it)
  Scene *d_scenes = nullptr;
  uint32_t scene_count = 0, scene_capacity = 0;
  unsigned char *h_plan = nullptr;  // pinned: the HZB plan (HzbPlanHead) of the prepared launch, view_capacity jobs
  unsigned char *d_plan = nullptr;
  struct PlanKey {                  // per job: the depth image the tensor map at `maps` + 128 j describes
    const float *depth = nullptr;
    uint32_t w = 0, h = 0, tma = 0;
  };
  std::vector<PlanKey> plan_keys;
  size_t plan_maps = 0;             // byte offset of the tensor maps the keys were made for
  cudaStream_t side = nullptr;      // the cell pass beside the HZB build (forked from and joined to the launch stream)
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaEvent_t done = nullptr;
  bool pending = false;
};

struct vgc_context {
  vgc_options opts{};
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 0;
  uint32_t select_grid = 0;  // persistent grid of k_instances
  uint32_t chunk_grid = 0;   // persistent grid of k_chunks
  uint32_t hzb_grid = 0;     // persistent grid of k_hzb_stream (0: the per-view tile kernel instead)
  uint64_t bytes = 0;
  std::mutex mu;
  // host mirrors of the resident scene
  std::vector<MeshHost> mesh_host;
  std::vector<MeshRec> meshes;
  std::vector<LevelRec> levels;
  std::vector<float4> m_lod, m_parent, m_err, m_cull;
  std::vector<float2> lsamples;  // kLevelSamples per level
  std::vector<float4> positions;
  std::vector<uint32_t> m_verts;
  std::vector<uint4> m_info;
  std::vector<uint32_t> m_tris;
  std::vector<float4> inst;
  std::vector<uint32_t> inst_slot;
  std::vector<CellRec> cells;
  uint32_t slot_capacity = 64;
  uint32_t slots_used = 0;
  bool dirty = true;
  // device copies
  DevBuf d_meshes, d_levels, d_m_lod, d_m_parent, d_m_err, d_m_cull, d_m_info, d_m_tris, d_inst, d_inst_slot, d_cells;
  DevBuf d_lsamples, d_positions, d_m_verts;
  DevBuf d_raster;  // occluder depth pass: the tile pass's work lists
  DevBuf d_resort;  // instance re-sort: centres, keys, permutation scratch (grows only)
  // output slots
  uint32_t out_slots = 0;
  uint32_t out_slot_capacity = 0;  // slot_capacity the output buffers were sized for
  uint32_t counter_words = 0;
  DevBuf d_counters, d_draw, d_args, d_dyn, d_hist;
  // controller state slots
  DevBuf d_state;
  uint32_t state_slots = 0;
  // HZB slots
  std::vector<HzbSlot> hzb;
  DevBuf d_hzb_desc;
  static constexpr uint32_t kHzbSlots = 256;
  LaunchScratch scratch;
  // profiling: events around plain-path launches, resolved lazily
  bool profiling = false;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_pending;
  std::vector<cudaEvent_t> prof_free;
  double prof_ms[VGC_KERNEL_KINDS] = {0};
  uint32_t prof_count[VGC_KERNEL_KINDS] = {0};
};

struct vgc_batch {
  vgc_context *ctx = nullptr;
  uint32_t max_views = 0;
  LaunchScratch scratch;
  cudaStream_t capture_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint32_t graph_views = 0;
  uint32_t graph_cells = 0;
  uint32_t graph_slots = 0;
  uint32_t graph_hzb_w = 0, graph_hzb_h = 0;
  bool graph_hzb_tail = false;
  bool graph_budget = false;
  const uint4 *graph_queue = nullptr;  // work queue the graph was captured with
  uint32_t graph_grids[2] = {0, 0};    // persistent grids the graph was captured with
  uint32_t graph_chunk_shift = 0;      // chunk size it was captured with
};

namespace vgch {

int dev_alloc(vgc_context *ctx, DevBuf &b, size_t bytes);
void dev_free(vgc_context *ctx, DevBuf &b);
int sync_scene(vgc_context *ctx);
Scene scene_of(const vgc_context *ctx);
// Output slots [0, slots) allocated for the current mesh-slot capacity; state slots [0, slot] allocated.
int ensure_outputs(vgc_context *ctx, uint32_t slots);
int ensure_state(vgc_context *ctx, uint32_t slot);
// Device bytes one output slot (with its state slot) takes at the context's current mesh-slot capacity.
size_t output_slot_bytes(const vgc_context *ctx);
// Scratch for `views` views and `units` (view, cell) units; grows only.
int ensure_scratch(vgc_context *ctx, LaunchScratch &s, uint32_t views, size_t units);
void free_scratch(LaunchScratch &s);
// View constants and HZB slots of one launch sequence; view i writes output slot slots[i] (or first_slot + i when
// slots is null).
int prepare(vgc_context *ctx, LaunchScratch &s, const vgc_view *views, uint32_t count, uint32_t first_slot,
            const uint32_t *slots = nullptr);
// Views of several contexts in one launch sequence: view i is a view of ctxs[scene[i]] and writes that context's
// output slot slots[i]. Views carry no depth image (their HZB slots must be built). Launch it with enqueue(ctxs[0]).
int prepare_multi(vgc_context *const *ctxs, uint32_t nctx, LaunchScratch &s, const vgc_view *views,
                  const uint32_t *scene, uint32_t count, const uint32_t *slots);
// The launch sequence of `count` prepared views on `st` (capture: recorded into a CUDA graph).
int enqueue(vgc_context *ctx, LaunchScratch &s, uint32_t count, cudaStream_t st, bool capture);
// vgc_stats of one view from its counter header and dyn[0] (the threshold the cut used).
void decode_stats(const vgc_context *ctx, const uint32_t *counters, float threshold, vgc_stats *s);
// Host mirror: cell `cell` of mesh `slot` from its instances (computeCell, GeometryPool.ts:519-545).
void compute_cell(vgc_context *ctx, uint32_t slot, uint32_t cell);
// Host mirror: mortonOrder (GeometryPool.ts:1263-1284) of n column-major matrices.
void morton_order(const float *m, uint32_t n, const float *sphere, std::vector<uint32_t> &order);

}  // namespace vgch
