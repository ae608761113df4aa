/*
 * vgbuild.h - host-side cluster-DAG builder and seeded scene generators.
 *
 * The cut engine (vgcut.h) consumes the per-mesh cluster DAG that three-virtual-geometry's
 * `buildVirtualMesh` produces (src/core/preprocess/buildVirtualMesh.ts:75-138, packed by `pack`
 * at :484-601). That builder depends on meshoptimizer, so this library writes the SAME layout
 * from its own clusterizer, spatial partitioner and quadric simplifier:
 *
 *   meshlet_bounds      16 floats per meshlet: [0..3] LOD sphere, [4..7] parent LOD sphere,
 *                       [8] error, [9] parent error (1e30 for roots), [10..11] 0, [12..15] cull sphere
 *   meshlet_info        4 u32 per meshlet: triangleCount, firstIndex, lodLevel, vertexOffset
 *   meshlet_vertices    global vertex id per meshlet-local vertex
 *   meshlet_triangles   one packed triangle per entry: local ids in bits 0-7, 8-15, 16-23
 *   level_ranges        per LOD level: firstMeshlet, meshletCount (meshlets sorted by level)
 *   level_errors        per level: smallest own error, largest parent error
 *   level_guard_errors  per level: largest own error, smallest parent error
 *   replacement_*       DAG links used by the coverage / overlap verifiers
 *
 * Builder output is host memory owned by the returned vgb_mesh; free with vgb_mesh_free.
 * Every function returns 0 on success and a negative code on error (vgb_last_error() explains).
 */
#ifndef VGBUILD_H
#define VGBUILD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors VirtualMeshData (buildVirtualMesh.ts:75-138) minus normals/colors/uvs (render side). */
typedef struct vgb_mesh {
  uint32_t vertex_count;
  float *positions;              /* 3 per vertex */
  uint32_t index_count;
  uint32_t *indices;             /* concatenated meshlet triangle lists (global vertex ids) */
  uint32_t meshlet_count;
  float *meshlet_bounds;         /* 16 per meshlet */
  uint32_t *meshlet_info;        /* 4 per meshlet */
  uint32_t meshlet_vertex_count;
  uint32_t *meshlet_vertices;
  uint32_t meshlet_triangle_count;
  uint32_t *meshlet_triangles;
  uint32_t level_count;
  uint32_t *level_ranges;        /* 2 per level */
  float *level_errors;           /* 2 per level */
  float *level_guard_errors;     /* 2 per level */
  float lod_bounds_sphere[4];
  float cull_bounds_sphere[4];
  float bounding_sphere[4];
  int32_t *replacement_group;    /* meshlet_count entries, -1 for the coarsest meshlets */
  uint32_t group_count;
  uint32_t *replacement_start;   /* group_count + 1 entries */
  uint32_t replacement_index_count;
  uint32_t *replacement_indices;
  /* stats (buildVirtualMesh.ts:126-137) */
  uint32_t leaf_triangles, leaf_meshlets, root_triangles, root_meshlets, lod_levels;
  double build_ms;
} vgb_mesh;

typedef struct vgb_options {
  uint32_t group_size;           /* meshlets per simplification group (reference default 12) */
  uint32_t max_lod_levels;       /* reference default 24 */
  float simplify_ratio;          /* target triangle fraction per group step (0.5) */
  float max_group_keep_ratio;    /* a group that keeps more than this fraction stays a root (0.9) */
  float min_level_reduction;     /* stop when a level removes less than this fraction (0.03) */
  uint32_t min_root_triangles;   /* tail stops at this many triangles (4) */
  uint32_t threads;              /* 0 = all host threads */
} vgb_options;

void vgb_default_options(vgb_options *opts);

/* Builds the cluster DAG of an indexed triangle mesh. positions: 3 floats per vertex. */
int vgb_build(const float *positions, uint32_t vertex_count, const uint32_t *indices, uint32_t index_count,
              const vgb_options *opts, vgb_mesh **out);
void vgb_mesh_free(vgb_mesh *mesh);

/* ---------------------------------------------------------------- seeded generators */

/* Raw indexed triangle mesh produced by a generator (free with vgb_raw_free). */
typedef struct vgb_raw {
  uint32_t vertex_count;
  float *positions;
  uint32_t index_count;
  uint32_t *indices;
} vgb_raw;
void vgb_raw_free(vgb_raw *raw);

/* Geodesic icosphere: each icosahedron face split into n*n triangles (20*n*n in total), radius r,
   displaced along the normal by amplitude*r*fbm(perlin(seed)) at the given feature frequency. */
int vgb_gen_icosphere(uint32_t n, float radius, float amplitude, float frequency, uint32_t seed, vgb_raw **out);
/* Lattice of boxes (ruins-like walls and pillars): `boxes` boxes, each face a k*k grid, seeded sizes and
   offsets inside a cube of half-extent `extent`, small seeded displacement of the face grids. */
int vgb_gen_box_lattice(uint32_t boxes, uint32_t k, float extent, uint32_t seed, vgb_raw **out);
/* Height-field terrain: a (segments+1)^2 grid of `size` x `size` centred at the origin in the xz plane,
   y = amplitude * sin(fx * x) * cos(fz * z) (the reference's cut-test terrain uses 400, 96, 30, 0.05, 0.04). */
int vgb_gen_terrain(float size, uint32_t segments, float amplitude, float fx, float fz, vgb_raw **out);

/* Seeded PRNG (mulberry32, a published 32-bit generator) so Python and C draw identical streams. */
uint32_t vgb_mulberry32_next(uint32_t *state);
double vgb_mulberry32_float(uint32_t *state);

/* Ken Perlin's improved noise (2002), seeded permutation; returns about [-1, 1]. */
float vgb_perlin3(uint32_t seed, float x, float y, float z);

/* Synthetic occluder depth image: `quads` screen-aligned rectangles at view depths U[dmin, dmax], written as
   the reference's NDC depth P[14]/depth - P[10]; background 1.0. width*height floats, row 0 = top. */
int vgb_gen_depth_image(uint32_t width, uint32_t height, uint32_t quads, float dmin, float dmax, float p10, float p14,
                        uint32_t seed, float *out);

/* 30-bit Morton order of instance sphere centres (GeometryPool.ts:1263-1311 behaviour: stable LSD radix sort).
   matrices: 16 floats column-major per instance; sphere: the mesh's bounding sphere. out: n indices. */
int vgb_morton_order(const float *matrices, uint32_t n, const float sphere[4], uint32_t *out);
/* Checksum of a .vgeo file (serialize.ts:429-437) over the u32 words from byte `start`. */
uint32_t vgb_vgeo_checksum(const uint8_t *bytes, uint64_t length, uint64_t start);

/* meshoptimizer's vertex buffer codec (versions 0 and 1) and index buffer codec (versions 0 and 1), the two codecs of
   the reference's compressed `.vgeo` fields (serialize.ts:244 `meshopt-vertex`, :290 `meshlet-triangles`).
   vgb_vertex_decode: `count` vertices of `stride` bytes (a multiple of 4, <= 256) from `size` bytes; 0 = OK, -1 bad
   header or version, -2 truncated, -3 bytes left over, -4 bad arguments. vgb_vertex_encode writes version 0 or 1 into
   `dst` (at least vgb_vertex_encode_bound bytes) and returns its length (0 on bad arguments). vgb_index_decode:
   `index_count` (a multiple of 3) 32-bit indices, the same codes; vgb_index_encode writes version 0 or 1 (at least
   vgb_index_encode_bound(index_count, largest index + 1) bytes). */
size_t vgb_vertex_encode_bound(size_t count, size_t stride);
size_t vgb_vertex_encode(uint8_t *dst, size_t capacity, const void *vertices, size_t count, size_t stride, int version);
int vgb_vertex_decode(void *vertices, size_t count, size_t stride, const uint8_t *src, size_t size);
size_t vgb_index_encode_bound(size_t index_count, size_t vertex_count);
size_t vgb_index_encode(uint8_t *dst, size_t capacity, const uint32_t *indices, size_t index_count, int version);
int vgb_index_decode(uint32_t *indices, size_t index_count, const uint8_t *src, size_t size);

const char *vgb_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
