/*
 * vg_oracle.h - CPU oracle for the cull + LOD-cut path. TEST INFRASTRUCTURE ONLY.
 *
 * This code is the checker, never the product: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may load it. It restates, in plain C:
 *   Part A - the reference's CPU cut evaluator, in double precision like JavaScript:
 *            src/core/runtime/cut.ts:26-215 (selectCut, selectBlendCut, verifyCutOverlap, verifyCutCoverage,
 *            instanceMeshletRange, instanceGuaranteedRange) and src/core/runtime/lodBlend.ts:52-61 (lodFadeRange).
 *   Part B - the reference's per-frame GPU passes (src/core/runtime/GeometryPool.ts:653-1069: bands, cells,
 *            instance + selectLevels, meshlet, prefix, capacity check/retry, steer) and the HZB build and test
 *            (src/core/runtime/OcclusionCulling.ts:119-170, 302-350), compiled twice:
 *              *_f32 - float arithmetic in the operation order the sm_100a kernels use (no contraction), so a
 *                      correct kernel matches it bit for bit;
 *              *_f64 - the same steps in double, standing for the reference's semantics; decisions whose
 *                      relative slack is within VGO_MARGIN are reported, not failed.
 *
 * Parity pinning: the reference ships no golden vectors and its TypeScript cannot run here (no Node), so the
 * oracle is pinned by the reference's own invariant tests (tests/cut.test.ts, tests/fastpath.test.ts), ported to
 * pytest over meshes built in this repository, plus hand-derived known-answer vectors in tests/golden/.
 */
#ifndef VG_ORACLE_H
#define VG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VGO_ERROR_INFINITY 1e30
#define VGO_FAST_PATH_MAX_MESHLETS 4
#define VGO_FAST_PATH_MARGIN 1e-3
#define VGO_LOD_FADE_STEPS 255
#define VGO_MARGIN 1e-5

/* ---------------------------------------------------------------- Part A (cut.ts, double) */
int vgo_lod_fade_range(double own, double parent, double threshold, double blend, int *lo, int *hi);
void vgo_select_cut(const float *bounds, uint32_t meshlet_count, const double view16[16], double proj_scale,
                    double near_, double scale, double threshold, uint8_t *selected);
void vgo_select_blend_cut(const float *bounds, uint32_t meshlet_count, const double view16[16], double proj_scale,
                          double near_, double scale, double threshold, double blend, uint8_t *lo, uint8_t *hi);
uint32_t vgo_verify_overlap(uint32_t meshlet_count, const int32_t *replacement_group, const uint32_t *replacement_start,
                            const uint32_t *replacement_indices, const uint8_t *selected, uint32_t *out);
uint32_t vgo_verify_coverage(uint32_t meshlet_count, const uint32_t *meshlet_info, const int32_t *replacement_group,
                             const uint32_t *replacement_start, const uint32_t *replacement_indices,
                             const uint8_t *selected, uint32_t *out);
/* Replacement links of one mesh (VirtualMeshData.replacementGroup / replacementStart / replacementIndices). */
typedef struct vgo_dag {
  uint32_t meshlet_count;
  const uint32_t *info; /* meshletInfo, 4 per meshlet (lodLevel at [2]) */
  const int32_t *group;
  const uint32_t *start, *list;
} vgo_dag;
/* verifyCutCoverage + verifyCutOverlap per drawn instance and blend step of one cut's entries (see vg_cut.c). */
uint64_t vgo_cut_invariant(const vgo_dag *dags, const uint32_t *base, uint32_t mesh_count, const uint32_t *inst_slot,
                           uint32_t instance_count, const uint32_t *entries, uint64_t n, const uint32_t *steps,
                           uint32_t nsteps, int threads, uint64_t *checked);
void vgo_instance_meshlet_range(const uint32_t *level_ranges, const float *level_errors, uint32_t level_count,
                                const float lod_bounds[4], const double view16[16], double proj_scale, double near_,
                                double scale, double threshold, double blend, uint32_t *start, uint32_t *end);
int vgo_instance_guaranteed_range(const uint32_t *level_ranges, const float *level_errors,
                                  const float *level_guard_errors, uint32_t level_count, const float lod_bounds[4],
                                  const double view16[16], double proj_scale, double near_, double scale,
                                  double threshold, double blend, uint32_t *start, uint32_t *end);

/* ---------------------------------------------------------------- Part B (GeometryPool.ts passes) */

/* A resident scene: pool-global arrays in the layout GeometryPool.add writes (GeometryPool.ts:386-545). */
typedef struct vgo_scene {
  uint32_t mesh_count;
  const float *mesh_sphere;          /* 4 per mesh: boundingSphere */
  const float *mesh_lod_bounds;      /* 4 per mesh */
  const float *mesh_cull_bounds;     /* 4 per mesh */
  const float *mesh_max_draw_distance;
  const float *mesh_min_pixel_radius;
  const uint32_t *mesh_level_count;
  const uint32_t *mesh_level_base;   /* first level-table entry */
  const uint32_t *mesh_enabled, *mesh_shadow, *mesh_occlusion;
  const uint32_t *level_first;       /* pool-global first meshlet of each level-table entry */
  const uint32_t *level_size;
  const float *level_errors;         /* 2 per entry: min own, max parent */
  const float *level_guard_errors;   /* 2 per entry: max own, min parent */
  uint32_t meshlet_count;
  const float *meshlet_bounds;       /* 16 per meshlet (reference AoS layout), pool-global */
  const uint32_t *meshlet_tri_count;
  uint32_t instance_count;
  const float *instance_matrices;    /* 16 per instance, column-major */
  uint32_t cell_count;
  const float *cell_data;            /* 8 per cell: centre xyz, radius, max instance radius, slot, first, count
                                        (slot/first/count stored as float values) */
} vgo_scene;

/* One camera view (VirtualGeometry.update uniforms, VirtualGeometry.ts:414-442, plus levers :78-183). */
typedef struct vgo_view {
  double view[16];            /* world -> view, column-major (camera.matrixWorldInverse) */
  double proj[16];            /* projection, column-major, [0,1] depth (WebGPU) */
  double near_;               /* camera.near */
  double viewport_height;     /* CSS pixels */
  double error_threshold;
  double lod_blend;           /* lodBlend lever; <= 1 disables blending */
  double min_pixel_radius;
  double shadow_error_scale;
  double max_error_threshold;
  double shadow_sweep[3];
  uint32_t frustum_culling;
  uint32_t occlusion_active;  /* HZB valid this frame */
  const float *hzb;           /* mip chain: level i at hzb + hzb_offset[i], hzb_width[i] x hzb_height[i] */
  uint32_t hzb_levels;
  uint32_t hzb_offset[16], hzb_width[16], hzb_height[16];
  uint32_t max_drawn;         /* draw-list capacity per cut (maxMeshlets) */
  uint32_t index_capacity[2]; /* index-buffer capacity per cut (3 x maxTriangles, 3 x maxShadowTriangles) */
  uint32_t state[8];          /* capacity controller state words (fixed point x 10000), carried between frames */
  double triangle_budget;     /* > 0: pick errorThreshold by the histogram search over threshold_range */
  double threshold_range[2];
  double chosen_threshold;    /* out: errorThreshold the budget search picked */
  uint64_t predicted_triangles; /* out: camera-cut triangles the histogram predicts at that threshold */
  uint32_t cascade;           /* shadow cascade: no camera cut, the shadow cut bounded by cascade_clip's planes */
  double cascade_clip[16];    /* world -> clip of the cascade, column-major, [0,1] depth */
  uint32_t cut_state[2][2];   /* out: per cut, the controller scales (state words 0, 1) its final computation ran
                                 with (a retry round redoes only the cuts that overflowed; the steer after the last
                                 round moves state[0..1] on for the next frame) */
  uint32_t pin_state;         /* 1: one round at `state` as given, no capacity check, retry or steer (to assess the
                                 cut's decisions at the controller state another run ended with) */
} vgo_view;

typedef struct vgo_result {
  uint32_t entry_capacity;    /* entries the caller allocated per cut */
  uint32_t *entries[2];       /* 3 u32 per entry: instance, meshlet, packed (triCount | lo << 8 | hi << 16) */
  uint32_t entry_count[2];
  uint32_t counters[12];      /* [0] visible cells, [1] occluded instances, then per cut: selected, drawn,
                                 survived, work, requested (GeometryPool.ts:112-119) */
  uint32_t *mesh_counts;      /* 2 cuts x mesh_count x 2 parts: requested indices */
  uint32_t *draw_args;        /* 2 cuts x mesh_count x 2 parts x 5 u32 */
  uint32_t rounds;            /* selection rounds run (1 + retries) */
  uint32_t max_selected[2];   /* per cut, the most meshlets any round selected: above max_drawn, that round kept an
                                 atomic-order-dependent subset on a GPU, and the capacity controller's next scale
                                 (from the kept entries' index count) depends on it */
} vgo_result;

/* Occluder depth pass (vg_raster.c): entries n x 4 u32 (instance, pool-global meshlet, firstIndex, packed), instance
   matrices 16 floats (4 columns) in GPU order, per-instance mesh slot, per-slot occluder flag, pool-global meshlet
   info (4 u32), packed triangles, meshlet vertex ids and xyz positions; depth receives width x height floats. */
int vgo_occluder_depth(const uint32_t *entries, uint32_t n, const float *inst, const uint32_t *inst_slot,
                       const uint32_t *slot_occluder, const uint32_t *m_info, const uint32_t *m_tris,
                       const uint32_t *m_verts, const float *positions, const double *view, const double *proj,
                       uint32_t width, uint32_t height, float *depth);
/* visibility buffer of a cut's expanded index buffer (vgc_visibility), and its per-pixel blend keep test */
int vgo_blend_keep(int px, int py, uint32_t frame, uint32_t lo, uint32_t hi);
int vgo_visibility(const uint32_t *indices, uint64_t capacity, const uint32_t *draw_list, uint32_t draw_slots,
                   const uint32_t *args, uint32_t regions, const float *inst, uint32_t instances,
                   const uint32_t *inst_slot, const uint32_t *slot_vertices, const float *slot_max_draw_distance,
                   const uint32_t *m_info, uint32_t meshlets, const uint32_t *m_verts, uint32_t meshlet_vertices,
                   const float *positions, uint32_t vertices, const double *view, const double *proj,
                   const double *fade_view, uint32_t width, uint32_t height, uint32_t frame, uint64_t *vis);

/* Full per-frame pass, float mirror of the kernels / double semantics. threads: 0 = all. */
int vgo_cull_pass_f32(const vgo_scene *scene, vgo_view *view, vgo_result *result, int threads);
int vgo_cull_pass_f64(const vgo_scene *scene, vgo_view *view, vgo_result *result, int threads);

/* Smallest relative slack (double) of the decisions that decide whether (instance, meshlet) is drawn by `cut`,
   including the cell, instance, level-range, fast-path, frustum, occlusion, LOD and blend-step decisions.
   Differences between a float and the double selection must all have slack <= VGO_MARGIN. */
double vgo_explain_f64(const vgo_scene *scene, const vgo_view *view, uint32_t cut, uint32_t instance, uint32_t meshlet);

/* HZB (OcclusionCulling.ts:284-350): mip 0 = depth, mip i = max of 2x2 of mip i-1, ceil halving, edge clamp.
   Writes the layout into view->hzb_* and the mips into `out` (capacity in floats). Returns floats used or -1. */
int64_t vgo_hzb_build(const float *depth, uint32_t width, uint32_t height, float *out, uint64_t out_capacity,
                      uint32_t *levels, uint32_t offset[16], uint32_t w[16], uint32_t h[16]);

/* Portable natural log used by both the kernels and the float mirror: frexp-style split and the atanh series
   ln(m) = 2 (s + s^3/3 + s^5/5 + ...), s = (m - 1) / (m + 1) (Abramowitz & Stegun 4.1.27), in float basic ops. */
float vgo_logf(float x);
/* three.js Frustum.setFromProjectionMatrix(m, WebGPUCoordinateSystem): planes right, left, bottom, top, far, near. */
void vgo_frustum_planes(const double m[16], double out[24]);

#ifdef __cplusplus
}
#endif
#endif
