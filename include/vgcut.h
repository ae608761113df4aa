/*
 * vgcut.h - C ABI of the sm_100a instance-culling + meshlet-DAG LOD-cut engine.
 *
 * Drop-in for the per-frame compute path of three-virtual-geometry: the passes GeometryPool.build() emits
 * (src/core/runtime/GeometryPool.ts:568-1092, dispatched by VirtualGeometry.update() at
 * src/core/runtime/VirtualGeometry.ts:484) and the HZB occlusion test (src/core/runtime/OcclusionCulling.ts:119-170).
 * Inputs keep the reference's layout (VirtualMeshData, 16-float column-major instance matrices, the same levers);
 * outputs are the same visible-cluster list (uvec4 per drawn meshlet) and drawIndexedIndirect args (5 u32 per
 * cut, mesh slot and part), left in device memory like the reference's storage buffers.
 *
 * Conventions
 *   - Every function returns vgc_status (0 = OK). On error, vgc_last_error() returns a message for this thread.
 *   - Caller memory is copied at the call; nothing is retained. Device output pointers stay valid until the next
 *     cut that writes the same output slot, or until the context is destroyed.
 *   - One context per host thread for the plain API (a context is not thread-safe). `stream` may be 0 (the
 *     context's own stream).
 */
#ifndef VGCUT_H
#define VGCUT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum vgc_status {
  VGC_OK = 0,
  VGC_INVALID_ARG = -1,
  VGC_OOM = -2,
  VGC_OVER_BUDGET = -3,  /* admission refused: the request would exceed the context's HBM budget */
  VGC_TIMEOUT = -4,      /* a bounded wait ran out (host deadline or a device-side iteration limit) */
  VGC_DEVICE_ERROR = -5,
  VGC_NOT_FOUND = -6,
} vgc_status;

typedef struct vgc_context vgc_context;
typedef struct vgc_batch vgc_batch;
typedef void *vgc_stream; /* cudaStream_t */

/* Per-context capacities. Reference: VirtualGeometryOptions (VirtualGeometry.ts:62-75) and PoolCapacity
   (GeometryPool.ts:142-149); the 120 MB WebGPU binding cap does not exist here (one resident buffer set). */
typedef struct vgc_options {
  uint32_t max_triangles;        /* camera-cut index capacity per view, in triangles (reference default 10M) */
  uint32_t max_shadow_triangles; /* shadow-cut index capacity per view (reference default 4M) */
  uint32_t max_meshlets;         /* draw-list capacity per cut per view (reference default 1 << 20) */
  uint32_t output_slots;         /* views whose outputs can be resident at once (batch width), default 1 */
  int32_t device;                /* CUDA device ordinal */
  uint64_t hbm_budget_bytes;     /* admission limit for this context's allocations; 0 = no limit */
} vgc_options;

/* The part of VirtualMeshData (buildVirtualMesh.ts:75-138) that the cut reads. */
typedef struct vgc_mesh_data {
  uint32_t meshlet_count;
  const float *meshlet_bounds;       /* 16 floats per meshlet */
  const uint32_t *meshlet_info;      /* 4 u32 per meshlet: triangleCount, firstIndex, lodLevel, vertexOffset */
  uint32_t meshlet_triangle_count;
  const uint32_t *meshlet_triangles; /* packed local triangles (for vgc_expand); may be NULL */
  uint32_t level_count;
  const uint32_t *level_ranges;      /* 2 per level */
  const float *level_errors;         /* 2 per level */
  const float *level_guard_errors;   /* 2 per level */
  float lod_bounds_sphere[4];
  float cull_bounds_sphere[4];
  float bounding_sphere[4];
  /* Optional vertex data (VirtualMeshData.positions / meshletVertices, buildVirtualMesh.ts:75-98), needed only by
     meshes drawn in the occluder depth pass (vgc_mesh_opts.occluder); NULL / 0 otherwise. */
  const float *positions;           /* xyz per vertex */
  uint32_t vertex_count;
  const uint32_t *meshlet_vertices; /* vertex ids, per meshlet in meshlet-local order (meshlet_info.vertexOffset) */
  uint32_t meshlet_vertex_count;
} vgc_mesh_data;

/* Per-mesh levers: VirtualMeshOptions (VirtualMesh.ts:39-62) and the mesh-table flags (GeometryPool.ts:449-477). */
typedef struct vgc_mesh_opts {
  float max_draw_distance;  /* world units; <= 0 or >= 1e30 = never culled by distance */
  float min_pixel_radius;   /* combined with the view's (the larger wins) */
  uint32_t enabled;         /* mesh.visible */
  uint32_t shadow;          /* the shadow cut includes this mesh */
  uint32_t occlusion;       /* occlusion culling may remove this mesh's instances and meshlets */
  uint32_t occluder;        /* mesh.occluder: drawn by vgc_occluder_depth (needs the mesh's vertex data) */
} vgc_mesh_opts;

/* vgc_view.flags */
enum {
  VGC_VIEW_FRESH_STATE = 1, /* the capacity controller starts this cut from its initial state (threshold scale 1, no
                               fill history) instead of the state slot's contents; the slot then holds this cut's
                               state as usual */
  VGC_VIEW_CASCADE = 2      /* the view is one shadow cascade of its camera (no counterpart in the reference, whose
                               shadow cut keeps the casters inside the camera frustum swept along shadowSweep): no
                               camera cut; the shadow cut keeps its reference semantics (LOD from the camera: view,
                               projection, threshold x shadowErrorScale; no occlusion) but culls against the clip
                               volume of `cascade_clip`; shadowSweep is not used; triangle_budget must be 0 */,
  VGC_VIEW_DEPTH_AS_MIP0 = 4 /* with `depth` and hzb >= 0 (no counterpart in the reference, which copies the depth
                               texture into the HZB's first level every frame): the cut reads the HZB's mip 0 from
                               `depth` itself instead of copying the image into the slot; mips 1 and up are built as
                               usual, and the results are the same. The slot's mip 0 keeps its previous contents, so
                               a later cut that uses the slot without a new `depth` must follow a build without this
                               flag. Saves writing 4 bytes per depth pixel when the HZB is rebuilt every frame. */
};

/* One cut request: the uniforms VirtualGeometry.update() writes (VirtualGeometry.ts:414-442) and the levers
   (:78-183). Matrices are column-major like three.js Matrix4.elements. */
typedef struct vgc_view {
  double view[16];              /* camera.matrixWorldInverse (rigid) */
  double proj[16];              /* camera.projectionMatrix, [0, 1] depth (WebGPU coordinate system) */
  double near_;                 /* camera.near */
  double viewport_height;       /* drawing-buffer height in CSS pixels: projScale = proj[5] * height / 2 */
  double error_threshold;       /* errorThreshold, pixels */
  double lod_blend;             /* lodBlend (<= 1: off) */
  double min_pixel_radius;      /* minPixelRadius */
  double shadow_error_scale;    /* shadowErrorScale */
  double max_error_threshold;   /* maxErrorThreshold (capacity controller limit) */
  double shadow_sweep[3];       /* shadowSweep */
  double triangle_budget;       /* triangleBudget: > 0 selects the threshold by device histogram search */
  double threshold_range[2];    /* thresholdRange searched by the budget (reference default [0.5, 3]) */
  uint32_t frustum_culling;     /* frustumCulling */
  int32_t hzb;                  /* HZB slot for occlusion culling of the camera cut; -1 = off */
  uint32_t state_slot;          /* capacity-controller state carried between frames of one camera */
  uint32_t flags;               /* VGC_VIEW_* bits */
  /* Optional occluder depth of this frame (device memory, NDC depth, row 0 at the top): when set with hzb >= 0,
     the cut first builds HZB slot `hzb` from it in the same launch sequence, as the reference prepends its HZB
     kernels to the frame's compute submission (VirtualGeometry.ts:482-484). NULL: use the slot as built. An image
     whose width is a multiple of 4, at least 128 x 32, with a 16-byte aligned pointer is streamed in with bulk-tensor
     copies; any other is read with plain loads (same result). */
  const float *depth;
  uint32_t depth_width, depth_height;
  /* VGC_VIEW_CASCADE: the cascade's clip matrix (light projection x light view, column-major, [0, 1] depth),
     world -> clip; its six planes bound the shadow cut */
  double cascade_clip[16];
} vgc_view;

/* Device pointers of one output slot. */
typedef struct vgc_output {
  const uint32_t *draw_list[2]; /* per cut: uvec4 (instance, meshlet, firstIndex in region, triCount|lo<<8|hi<<16) */
  const uint32_t *draw_args;    /* ((cut * mesh_slots + slot) * 2 + part) * 5 u32: drawIndexedIndirect args */
  const uint32_t *counters;     /* VGC_COUNTER_* words, then per (cut, slot, part) requested indices and region start */
  uint32_t max_drawn;
  uint32_t mesh_slots;
} vgc_output;

/* Counter words of an output slot (GeometryPool.ts:112-119, plus this engine's round bookkeeping). */
enum {
  VGC_COUNTER_CELLS = 0,
  VGC_COUNTER_OCCLUDED = 1,
  VGC_COUNTER_CUT0 = 2, /* + VGC_CUT_SELECTED.. for the camera cut */
  VGC_COUNTER_CUT1 = 7, /* + VGC_CUT_SELECTED.. for the shadow cut */
  VGC_COUNTER_REDO0 = 12,
  VGC_COUNTER_REDO1 = 13,
  VGC_COUNTER_ROUNDS = 14,
  VGC_COUNTER_ERROR = 15,           /* VGC_FAULT_* bits of this view's launch sequence */
  VGC_COUNTER_INSTANCES_TESTED = 16, /* instances of visible cells (all rounds) */
  VGC_COUNTER_MESHLETS_TESTED = 17,  /* meshlets run through the per-meshlet test (all rounds) */
  VGC_COUNTER_FAST_EMITTED = 18,     /* meshlets emitted by the instance fast path (all rounds) */
  VGC_COUNTER_LEVELS_READ = 19,      /* level-table entries read (sum over visible cells, all rounds) */
  VGC_COUNTER_PREDICTED_LO = 20,     /* triangleBudget search: plain camera-cut triangles predicted at the */
  VGC_COUNTER_PREDICTED_HI = 21,     /*   chosen threshold (64-bit, low and high words) */
  VGC_COUNTER_BUDGET_BIN = 22,       /* the chosen threshold bin k: t = lo + (hi - lo) k / 255 */
  VGC_COUNTER_MESHLETS_QUEUED = 23,  /* meshlets of the items after trimming the ones that fail the LOD band for
                                        certain (tested in the meshlet pass; MESHLETS_TESTED counts the full ranges) */
  VGC_COUNTER_HEADER = 24,
};
/* Device-side failures a kernel reports instead of waiting on: VGC_FAULT_HZB_WAIT = a tile copy of the HZB
 * build did not arrive within about a second (the launch's HZBs are incomplete; its cuts may keep occluded geometry
 * or drop visible geometry). */
enum { VGC_FAULT_HZB_WAIT = 1 };
enum { VGC_CUT_SELECTED = 0, VGC_CUT_DRAWN = 1, VGC_CUT_SURVIVED = 2, VGC_CUT_WORK = 3, VGC_CUT_REQUESTED = 4 };

/* Stats of one output slot: VirtualGeometryStats (VirtualGeometry.ts:24-47) per view. */
typedef struct vgc_stats {
  uint32_t visible_cells;
  uint32_t occluded_instances;
  uint32_t selected[2], drawn[2], survived[2], work[2], requested_indices[2];
  uint32_t rounds;
  uint32_t overflow;            /* a cut exceeded its draw buffers after the last retry round */
  float threshold_scale[2];     /* capacity controller scale per cut */
  float fill[2];
  float effective_threshold;    /* errorThreshold used (after a budget search) */
  uint32_t instances_tested, meshlets_tested, fast_emitted, levels_read; /* work done, all rounds */
  uint64_t predicted_triangles; /* triangleBudget search: predicted plain camera-cut triangles */
  uint32_t meshlets_queued;     /* meshlets the meshlet pass tested after item trimming (all rounds) */
  uint32_t faults;              /* VGC_FAULT_* bits (0: none) */
} vgc_stats;

const char *vgc_last_error(void);
const char *vgc_version(void);

/* ---------------------------------------------------------------- context and scene residency */
void vgc_default_options(vgc_options *opts);
/* new VirtualGeometry(options) (VirtualGeometry.ts:191-198) */
int vgc_context_create(const vgc_options *opts, vgc_context **out);
/* VirtualGeometry.dispose() */
int vgc_context_destroy(vgc_context *ctx);
/* Bytes of device memory this context holds. */
int vgc_context_footprint(const vgc_context *ctx, uint64_t *bytes);

/* vg.createMesh(data, material, {matrices}, options) (VirtualGeometry.ts:231, VirtualMesh.ts:159-233,
   GeometryPool.add :302-355): copies the DAG and the instances (Morton-ordered on the host, GeometryPool.ts:1263)
   into device memory and returns the mesh slot. gpu_to_input (optional, n entries) receives the Morton order. */
int vgc_mesh_add(vgc_context *ctx, const vgc_mesh_data *data, const float *matrices, uint32_t instance_count,
                 const vgc_mesh_opts *opts, uint32_t *slot, uint32_t *gpu_to_input);
/* mesh.maxDrawDistance / minPixelRadius / visible / castShadow / occlusionCulling (GeometryPool.writeFlags :463-477);
   a resident scene gets the one mesh record uploaded (synchronous). */
int vgc_mesh_set_flags(vgc_context *ctx, uint32_t slot, const vgc_mesh_opts *opts);
/* mesh.setMatrixAt + commitInstances (VirtualMesh.ts:305-314, GeometryPool.ts:499-512): `count` matrices for GPU
   (Morton) indices [first, first + count) of the mesh; the cells they touch are recomputed. With the scene resident,
   only the changed matrices are uploaded and the cells are recomputed on the device (synchronous: it waits for the
   device's earlier work and finishes before returning); the Morton order of the instances is kept. */
int vgc_instances_update(vgc_context *ctx, uint32_t slot, uint32_t first, uint32_t count, const float *matrices);
/* Re-sort of a mesh's instances along the Morton curve of their current positions (mortonOrder,
   GeometryPool.ts:1263-1284, which the reference runs only when a mesh is added): after instances have moved,
   consecutive GPU indices are close again and the 128-instance cells compact. With the scene resident the codes,
   the stable radix sort, the permutation and the cells are computed on the device; the host mirror follows.
   Stable with respect to the current GPU order. new_to_old (optional, instance_count entries) receives, for each new
   GPU index, the GPU index the instance had before; draw lists cut before the call keep the previous indices.
   Synchronous; the first call allocates the context's re-sort scratch (about 110 bytes per instance, kept). */
int vgc_instances_resort(vgc_context *ctx, uint32_t slot, uint32_t *new_to_old);
/* mesh.dispose() (GeometryPool.remove :358-363) */
int vgc_mesh_remove(vgc_context *ctx, uint32_t slot);
/* Highest used mesh slot + 1 and the slot capacity (mesh table size). */
int vgc_mesh_slots(const vgc_context *ctx, uint32_t *used, uint32_t *capacity);

/* ---------------------------------------------------------------- HZB (OcclusionCulling.ts:284-350) */
/* Builds the max-reduced mip chain of a depth image (NDC depth, row 0 at the top) into HZB slot `hzb`.
   depth_is_device: the pointer is device memory (else host memory, copied). The view's proj[] is used by the
   test, so the image must come from the same projection. */
int vgc_hzb_build(vgc_context *ctx, int32_t hzb, const float *depth, uint32_t width, uint32_t height,
                  int depth_is_device, vgc_stream stream);

/* ---------------------------------------------------------------- the cut */
/* Plain per-view launch (the drop-in for renderer.compute(pool.computeNodes)): runs the cut for `count` views into
   output slots [first_slot, first_slot + count) as a sequence of kernel launches on `stream`. Asynchronous. */
int vgc_cut(vgc_context *ctx, const vgc_view *views, uint32_t count, uint32_t first_slot, vgc_stream stream);

/* The plain single-view cut with no device allocation on the call. It has no counterpart in the reference. For
   callers that cannot call cudaMalloc while they run - a renderer's real-time frame thread, which must not stall on
   the device-wide synchronisation an allocation can cause, or a host that reserves all of its GPU memory up front
   and hands nothing else out - it keeps its per-call scratch in a fixed 1.5 MiB device array inside the library
   (held by every GPU that loads it until the process exits) rather than in context allocations. Limits: a scene of at most 65,536 cells (8,388,608 instances); the
   output slot, the view's state slot and (for a view with `depth`) its HZB slot at that size must already exist
   (create the context with enough output_slots; build the HZB once with vgc_hzb_build); the scene must have been
   published by an earlier vgc_cut after the last mesh change. Meshlet chunks past the fixed queue are tested in
   place, so the result is the same as vgc_cut's. The first call on a device looks the array's device address up
   (make that call before any stream capture). Every call shares the one array: calls whose GPU work overlaps -
   on two streams, or two contexts on one device - race; order them on one stream. Asynchronous on `stream`. */
int vgc_cut_noalloc(vgc_context *ctx, const vgc_view *view, uint32_t slot, vgc_stream stream);

/* Batched launch: the same kernels for up to `max_views` views captured once into a CUDA graph, replayed with the
   new views' constants. Output slots are [first_slot, first_slot + count). */
int vgc_batch_create(vgc_context *ctx, uint32_t max_views, vgc_batch **out);
int vgc_batch_run(vgc_batch *batch, const vgc_view *views, uint32_t count, uint32_t first_slot, vgc_stream stream);
int vgc_batch_destroy(vgc_batch *batch);

/* Autotuner (no counterpart in the reference): times the batch's launch sequence for `views` (reps replays each,
   median) under every combination of the meshlet kernel's work-unit size (chunks of 256, 512 or 1024 meshlets) and
   the persistent grid sizes of the instance and meshlet kernels (blocks per SM: quarters of each kernel's occupancy
   limit), and keeps the fastest for the batch's later runs. Results are the same under every candidate: these only
   decide how the work is cut up and which warp takes which piece. Runs the views' cut (outputs are left as a normal
   run leaves them). */
typedef struct {
  uint32_t instances_blocks_per_sm, chunks_blocks_per_sm;
  float ms; /* median device time of one run */
  uint32_t chunk_meshlets; /* meshlets per k_chunks work unit */
} vgc_tune_result;
int vgc_batch_autotune(vgc_batch *batch, const vgc_view *views, uint32_t count, uint32_t first_slot, vgc_stream stream,
                       uint32_t reps, vgc_tune_result *best);
/* Applies a tuning (for instance one vgc_batch_autotune returned earlier, kept by the caller) to the batch's later
   runs: blocks per SM of the two kernels (0: the occupancy default) and meshlets per chunk (256, 512 or 1024). */
int vgc_batch_set_tuning(vgc_batch *batch, const vgc_tune_result *tuning);

/* ---------------------------------------------------------------- serving (no counterpart in the reference) */
/* A request loop over several resident scenes (one context each). The reference cuts once per rendered frame of
   one camera; a server takes cut requests (scene, view) from any thread as they arrive. One worker thread admits a
   request while an output slot of its scene is free and the output-slot bytes of the admitted, unreleased requests
   stay within the HBM budget; it batches the oldest admitted requests - of any scenes, each view reading its own
   scene's data in the same kernels (cross_scene), or of the oldest request's scene only - into one launch sequence
   and keeps up to `streams` batches in flight, so requests that arrive while others run start as soon as a stream
   and slots free up (continuous batching). Each request runs as vgc_cut of its view alone would with VGC_VIEW_FRESH_STATE, its
   output slot doubling as its state slot: the result is the same alone and in any mix. While a server runs, its
   contexts take no other cut or scene change; completed requests' outputs are read with vgc_get_output /
   vgc_read_draw_list on (scene context, result.slot) until vgc_server_release. */
typedef struct vgc_server vgc_server;
typedef struct {
  uint32_t streams;          /* batches in flight at once (default 2) */
  uint32_t max_batch;        /* views per launch (default 64) */
  uint32_t slots_per_scene;  /* output slots reserved per scene (default streams * max_batch) */
  uint64_t hbm_budget_bytes; /* admission limit on the output-slot bytes of admitted, unreleased requests (0: none) */
  uint32_t linger_us;        /* while another batch runs, a batch smaller than max_batch waits up to this long (from
                                its oldest request) for more requests; with every stream idle it starts at once
                                (default 0: never waits) */
  uint64_t max_batch_instances; /* views x scene instances per batch at most (default 32M; 0: no limit): large
                                   scenes go in smaller batches, which keeps their latency and work queue bounded */
  uint32_t cross_scene;      /* 1 (default): a batch mixes scenes (all contexts on one device); 0: one scene each */
} vgc_server_options;
typedef struct {
  uint64_t ticket;
  uint32_t scene, slot;       /* scene index and the output slot holding the result */
  int32_t status;             /* VGC_OK, or the error of the launch that carried it */
  uint32_t batch_views;       /* views in that launch */
  double submit_us, start_us, done_us; /* host steady clock, microseconds: submitted, launched, seen complete */
  float batch_gpu_ms;         /* device time of that launch (CUDA events on its stream) */
  vgc_stats stats;            /* its counters, copied back with the launch */
  uint32_t batch_scenes;      /* scenes in that launch */
} vgc_serve_result;
typedef struct {
  uint64_t submitted, completed, batches, views_launched;
  uint64_t bytes_in_use, max_bytes_in_use; /* admitted output-slot bytes now / at most */
  uint32_t max_in_flight;                 /* most batches in flight at once */
  uint64_t multi_scene_batches;           /* batches that mixed scenes */
} vgc_server_stats;
void vgc_server_default_options(vgc_server_options *opts);
int vgc_server_create(vgc_context *const *scenes, uint32_t scene_count, const vgc_server_options *opts,
                      vgc_server **out);
/* Thread-safe. `view` is copied; its state_slot and VGC_VIEW_FRESH_STATE are set by the server. */
int vgc_server_submit(vgc_server *server, uint32_t scene, const vgc_view *view, uint64_t *ticket);
/* Waits up to timeout_ms for the request; VGC_TIMEOUT if it has not completed. */
int vgc_server_wait(vgc_server *server, uint64_t ticket, uint32_t timeout_ms, vgc_serve_result *out);
/* Frees the request's output slot (and its HBM share) for later requests; its outputs are no longer valid. */
int vgc_server_release(vgc_server *server, uint64_t ticket);
/* Waits until every submitted request has completed (VGC_TIMEOUT after timeout_ms). */
int vgc_server_drain(vgc_server *server, uint32_t timeout_ms);
int vgc_server_stats_get(vgc_server *server, vgc_server_stats *out);
int vgc_server_destroy(vgc_server *server);

/* Occluder depth pass (OcclusionCulling.ts:244-273, step 1): draws the camera cut held in output slot `src_slot` -
   the previous frame's - depth-only with this frame's camera `view` into `depth` (device memory, width x height
   floats, row 0 at the top, NDC depth in [0, 1], 1 where nothing is drawn), for the meshes flagged occluder. As in the
   reference, only the meshlets drawn over every pixel (part 0) are drawn, back faces are culled, and a triangle is
   sampled at pixel centres. A triangle crossing the near plane (clip z = 0) is clipped in clip space into one or two
   triangles (crossing points interpolated from the corner in front, at depth 0), as a GPU's clipper does; wholly
   behind it, it is not drawn. Pass `depth` as this frame's vgc_view.depth to build the HZB from it in the cut's own
   launch sequence. The first call allocates the context's triangle queues (about 54 MB, shared with
   vgc_visibility; up to 131,072 near-plane-crossing triangles a call are clipped, more are left out); calls on one
   context whose GPU work overlaps (different streams) race on them: order them on one stream. Asynchronous on
   `stream`. */
int vgc_occluder_depth(vgc_context *ctx, uint32_t src_slot, const vgc_view *view, float *depth, uint32_t width,
                       uint32_t height, vgc_stream stream);
/* vgc_occluder_depth for `count` images of one size in one call, in order on `stream`: image i draws output slot
   src_slots[i] with views[i] into depth[i] (an array of `count` device pointers, in host memory). The same images as
   count single calls; for a renderer with many views (split screen, probes, a serving batch) it saves the per-call
   host work. */
int vgc_occluder_depth_batch(vgc_context *ctx, uint32_t count, const uint32_t *src_slots, const vgc_view *views,
                             float *const *depth, uint32_t width, uint32_t height, vgc_stream stream);

/* Visibility buffer: a headless consumer of a cut's output, after vgc_expand. Draws the index buffer `indices`
   (device, `capacity` indices) that vgc_expand wrote for output slot `slot` and cut `cut`, region by region as the
   cut's draw args give them, with the reference's vertex pulling (GeometryPool.ts:1095-1131: draw-list entry,
   meshletVertices, positions, the instance's model, the draw-distance shrink toward the instance origin measured
   from `fade_view`, NULL = `view`) and LOD blend mask (lodBlend.ts:36-45: interleaved gradient noise at the pixel
   centre, `frame` as lodBlendFrame), rasterized with `view` at pixel centres, back faces culled and triangles
   crossing the near plane clipped as in vgc_occluder_depth, into `vis` (device, width x height u64, row 0 at the top): per pixel the
   minimum of (NDC depth bits << 32 | drawSlot << 7 | triangle in its meshlet), VGC_VIS_EMPTY where nothing is
   drawn. Meshes without vertex data are not drawn. Uses the context's triangle queues (see vgc_occluder_depth):
   calls whose GPU work overlaps race on them. Asynchronous on `stream`. */
#define VGC_VIS_EMPTY 0x3f800000ffffffffull
int vgc_visibility(vgc_context *ctx, uint32_t slot, uint32_t cut, const vgc_view *view, const vgc_view *fade_view,
                   const uint32_t *indices, uint64_t capacity, uint64_t *vis, uint32_t width, uint32_t height,
                   uint32_t frame, vgc_stream stream);

/* Layout of HZB slot `hzb`: levels, per-level offset (floats) / width / height (16 entries each), and the device
   pointer of the mip chain (level i at data + offset[i], row-major). */
int vgc_hzb_info(const vgc_context *ctx, int32_t hzb, uint32_t *levels, uint32_t *offset, uint32_t *width,
                 uint32_t *height, const float **data);

/* Device pointers of an output slot (valid after the cut's stream work completes). */
int vgc_get_output(const vgc_context *ctx, uint32_t slot, vgc_output *out);
/* vg.readStats (VirtualGeometry.ts:591-632) for one output slot; synchronises with `stream`. */
int vgc_read_stats(vgc_context *ctx, uint32_t slot, vgc_stats *stats, vgc_stream stream);
/* Copies an output slot's draw list of `cut` into host memory: up to `capacity` entries (4 u32 each); *count
   receives the number of drawn entries. Synchronises with `stream`. */
int vgc_read_draw_list(vgc_context *ctx, uint32_t slot, uint32_t cut, uint32_t *entries, uint32_t capacity,
                       uint32_t *count, vgc_stream stream);
/* Capacity-controller state words of a state slot (8 u32, fixed point x 10000): read or overwrite. */
int vgc_state_access(vgc_context *ctx, uint32_t state_slot, uint32_t *words, int write, vgc_stream stream);

/* Index expansion (GeometryPool.ts:998-1021): writes 3 indices per drawn triangle, (drawSlot << 7) | localVertex,
   into `index_buffer` (device, capacity of the cut in indices) for output slot `slot` and cut `cut`. */
int vgc_expand(vgc_context *ctx, uint32_t slot, uint32_t cut, uint32_t *index_buffer, uint64_t capacity,
               vgc_stream stream);

/* ---------------------------------------------------------------- CPU-API equivalents on the GPU */
/* selectCut / selectBlendCut (cut.ts:26-77) for mesh `slot` under `count` view-model matrices, in one launch:
   per view i, viewmodel16[i*16..], proj_scale[i], near_[i], scale[i]; lo/hi receive count * meshlet_count bytes
   (hi == 0: not drawn; blend <= 1 gives the plain cut with lo = 0, hi = 255). Synchronous. */
int vgc_select_cut(vgc_context *ctx, uint32_t slot, uint32_t count, const double *viewmodel16, const double *proj_scale,
                   const double *near_, const double *scale, double threshold, double blend, uint8_t *lo, uint8_t *hi);

/* ---------------------------------------------------------------- profiling (no counterpart in the reference) */
enum { VGC_KERNEL_RESET = 0, VGC_KERNEL_CELLS = 1, VGC_KERNEL_SELECT0 = 2, VGC_KERNEL_SELECT_RETRY = 3,
       VGC_KERNEL_FINISH = 4, VGC_KERNEL_HZB = 5, VGC_KERNEL_CHUNKS0 = 6, VGC_KERNEL_BUDGET = 7, VGC_KERNEL_KINDS = 8 };
/* With `enable`, the plain path (vgc_cut, vgc_hzb_build) records CUDA events around each of its kernel launches
   on the launching stream. vgc_kernel_times synchronises and returns, per VGC_KERNEL_* kind, the summed device
   milliseconds and the launch count since the last reset (reset = 1 clears them). */
int vgc_set_profiling(vgc_context *ctx, int enable);
int vgc_kernel_times(vgc_context *ctx, double *ms, uint32_t *launches, int reset);

/* ---------------------------------------------------------------- test support (no counterpart in the reference) */
/* Host copies of the resident cell records (8 floats: centre xyz, radius, max instance radius, slot, first instance,
   count; GeometryPool.ts:544 layout) and of the Morton-ordered instance matrices (16 floats each). */
int vgc_debug_scene(const vgc_context *ctx, float *cells, uint32_t cell_capacity, float *matrices,
                    uint32_t matrix_capacity, uint32_t *cell_count, uint32_t *instance_count);
/* The device's cell records in the same 8-float form (after the pending upload, if any): instance updates recompute
   them on the device, and they must equal the host's. */
int vgc_debug_cells_device(vgc_context *ctx, float *cells, uint32_t capacity, uint32_t *count);
/* Runs the device's bounded mbarrier wait (the one the HZB strip stream waits with) on a barrier that nothing
   completes, with a limit of `limit_us` microseconds: *completed = 0 and *waited_ns = the time it waited before it
   gave up; the context stays usable. */
int vgc_debug_wait_probe(vgc_context *ctx, uint32_t limit_us, uint32_t *completed, uint64_t *waited_ns);

#ifdef __cplusplus
}
#endif
#endif
