// sm_100a kernels of the cull + LOD-cut engine.
//
// Pass structure for a batch of views (all views of one scene in each launch):
//   k_cells    one thread per (view, cell): the cell tests of GeometryPool.ts:728-760; surviving (view, cell)
//              units are compacted with one atomic per warp (__ballot_sync / __popc).
//   k_instances one warp per 32 instances of a visible unit: the instance tests (GeometryPool.ts:846-913) and the
//              LOD level range (selectLevels :771-843). Fast-path instances emit their meshlets with warp-aggregated
//              atomics; the others queue their range as chunks of <= 256 meshlets (one warp-wide reservation).
//   k_chunks   one warp per chunk: the meshlet tests (GeometryPool.ts:916-970), reading the struct-of-arrays
//              bounds coalesced; drawn meshlets are staged per warp and placed with one atomic per cut and part.
//   k_finish   one warp per view: the prefix pass (GeometryPool.ts:973-995) as a warp scan over mesh slots, the
//              capacity check that schedules a retry round (:1032-1054), and after the last round the steer (:1056-1069).
//   k_expand   one warp per drawn meshlet: index expansion (GeometryPool.ts:998-1021).
//   k_hzb_*    HZB mip chain (OcclusionCulling.ts:302-350): 32x32 tiles reduce five levels in shared memory, one
//              block finishes the small top levels.
//
// Arithmetic: this file is compiled with -fmad=false and IEEE division / square root, so every decision
// expression rounds step by step in the order written, which the oracle's float mirror repeats.
#include <cuda_runtime.h>

#include <cstdint>

#include "vgcut_internal.h"
#include "vgcut_kernels.h"

namespace vgc {

#define C_CUT(cut) (VGC_COUNTER_CUT0 + (cut) * 5)

__device__ __forceinline__ float fmn(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmx(float a, float b) { return a > b ? a : b; }

// Natural log from float basic operations and fused multiply-adds (same steps as the oracle's vgo_logf): x = m 2^e,
// m in [sqrt(1/2), sqrt(2)), ln x = e ln2 + 2 atanh((m-1)/(m+1)) by its odd series (Abramowitz & Stegun 4.1.27) in
// Horner form, ln2 split in a high part with trailing zero bits and a low correction.
__device__ __forceinline__ float vg_logf(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -__int_as_float(0x7f800000) : __int_as_float(0x7fc00000);
  if (x == __int_as_float(0x7f800000)) return x;
  uint32_t u = __float_as_uint(x);
  int e = 0;
  if ((u >> 23) == 0) {
    x = x * 8388608.0f;
    u = __float_as_uint(x);
    e = -23;
  }
  e += int((u >> 23) & 0xffu) - 127;
  float m = __uint_as_float((u & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421356f) {
    m = m * 0.5f;
    e += 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float p = __fmaf_rn(s2, 0.0909090936f, 0.111111112f);
  p = __fmaf_rn(s2, p, 0.142857149f);
  p = __fmaf_rn(s2, p, 0.2f);
  p = __fmaf_rn(s2, p, 0.333333343f);
  p = s2 * p;
  float lnm = __fmaf_rn(s, p, s) * 2.0f;
  float fe = float(e);
  return __fmaf_rn(fe, 0.693145752f, __fmaf_rn(fe, 1.42860677e-06f, lnm));
}

struct Bands {
  float low[2], high[2], fade_scale;
};

__device__ __forceinline__ float get_state(const uint32_t *state, int i) { return float(state[i]) / 10000.0f; }
__device__ __forceinline__ uint32_t to_state(float v) { return uint32_t(rintf(v * 10000.0f)); }

// GeometryPool.ts:653-665; `threshold` is the view's errorThreshold (or the budget search's result)
__device__ void load_bands(const ViewConst &V, float threshold, Bands &b) {
  float camera_scale = get_state(V.state, 0);
  float shadow_scale = get_state(V.state, 1);
  float x = threshold * camera_scale;
  float t = (x - 1.25f) / 1.25f;
  t = fmn(fmx(t, 0.0f), 1.0f);
  float smooth = (t * t) * (3.0f - 2.0f * t);
  float width = 1.0f + (V.lod_blend_max - 1.0f) * smooth;
  bool blending = width > float(1.001);
  b.fade_scale = blending ? 255.0f / vg_logf(width) : 0.0f;
  float t0 = threshold * camera_scale;
  float t1 = (threshold * V.shadow_error_scale) * fmx(camera_scale, shadow_scale);
  b.low[0] = t0;
  b.low[1] = t1;
  b.high[0] = blending ? t0 * width : t0;
  b.high[1] = blending ? t1 * width : t1;
}

// Products summed with fused multiply-adds from the constant term up (the oracle's float build uses fmaf in the same
// order): M c = fma(M2, z, fma(M1, y, fma(M0, x, M3))) per row, |v|^2 = fma(v2, v2, fma(v1, v1, v0 v0)).
__device__ __forceinline__ void xform(const float *M, float x, float y, float z, float out[3]) {
#pragma unroll
  for (int r = 0; r < 3; r++)
    out[r] = __fmaf_rn(M[r * 4 + 2], z, __fmaf_rn(M[r * 4 + 1], y, __fmaf_rn(M[r * 4 + 0], x, M[r * 4 + 3])));
}

__device__ __forceinline__ float len3(const float v[3]) {
  return sqrtf(__fmaf_rn(v[2], v[2], __fmaf_rn(v[1], v[1], v[0] * v[0])));
}

// VM = V * M (rows 0..2, row-major 3x4) and the instance scale (GeometryPool.ts:670-675)
__device__ __forceinline__ void model_view(const float *Vr, const float4 *cols, float *VM, float &scale) {
  float4 c[4] = {cols[0], cols[1], cols[2], cols[3]};
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int k = 0; k < 4; k++)
      VM[r * 4 + k] = __fmaf_rn(Vr[r * 4 + 3], c[k].w,
                                __fmaf_rn(Vr[r * 4 + 2], c[k].z, __fmaf_rn(Vr[r * 4 + 1], c[k].y, Vr[r * 4 + 0] * c[k].x)));
  float l0[3] = {c[0].x, c[0].y, c[0].z}, l1[3] = {c[1].x, c[1].y, c[1].z}, l2[3] = {c[2].x, c[2].y, c[2].z};
  scale = fmx(len3(l0), fmx(len3(l1), len3(l2)));
}

// frustumDistance (GeometryPool.ts:690-698) in view space
__device__ __forceinline__ float frustum(const ViewConst &V, const float c[3], bool swept) {
  float m = 1e30f;
#pragma unroll
  for (int p = 0; p < 6; p++) {
    float d = __fmaf_rn(V.plane[p * 4 + 2], c[2], __fmaf_rn(V.plane[p * 4 + 1], c[1], __fmaf_rn(V.plane[p * 4], c[0], V.plane[p * 4 + 3])));
    if (swept) d = d + V.sweep[p];
    m = fmn(m, d);
  }
  return m;
}

__device__ __forceinline__ uint32_t ceil_log2(uint32_t e) { return e <= 1 ? 0u : 32u - __clz(e - 1u); }

// OcclusionCulling.ts:119-170: true only when the sphere is certainly behind the HZB occluders. The footprint
// level is computed in integers; samples go through the read-only (texture / L1) path.
__device__ bool hzb_occluded(const ViewConst &V, const HzbDesc &H, const float c[3], float radius) {
  float depth = -c[2];
  float near_depth = depth - radius;
  if (!(near_depth > V.near_)) return false;
  float far_depth = depth + radius;
  float xlo = c[0] - radius, xhi = c[0] + radius, ylo = c[1] - radius, yhi = c[1] + radius;
  // x / depth as x * (1 / depth): two divisions instead of nine
  const float inv_near = 1.0f / near_depth, inv_far = 1.0f / far_depth;
  float min_x = __fmaf_rn(fmn(xlo * inv_near, xlo * inv_far), V.P0, -V.P8);
  float max_x = __fmaf_rn(fmx(xhi * inv_near, xhi * inv_far), V.P0, -V.P8);
  float min_y = __fmaf_rn(fmn(ylo * inv_near, ylo * inv_far), V.P5, -V.P9);
  float max_y = __fmaf_rn(fmx(yhi * inv_near, yhi * inv_far), V.P5, -V.P9);
  float min_z = __fmaf_rn(V.P14, inv_near, -V.P10);
  if (!(min_z < 1.0f)) return false;
  float W = float(H.w[0]), Hh = float(H.h[0]);
  float fx0 = floorf(__fmaf_rn(min_x, 0.5f, 0.5f) * W);
  float fx1 = floorf(__fmaf_rn(max_x, 0.5f, 0.5f) * W);
  float fy0 = floorf(__fmaf_rn(-max_y, 0.5f, 0.5f) * Hh);
  float fy1 = floorf(__fmaf_rn(-min_y, 0.5f, 0.5f) * Hh);
  uint32_t x0 = uint32_t(fmn(fmx(fx0, 0.0f), W - 1.0f));
  uint32_t x1 = uint32_t(fmn(fmx(fx1, 0.0f), W - 1.0f));
  uint32_t y0 = uint32_t(fmn(fmx(fy0, 0.0f), Hh - 1.0f));
  uint32_t y1 = uint32_t(fmn(fmx(fy1, 0.0f), Hh - 1.0f));
  uint32_t dx = x1 > x0 ? x1 - x0 : 0u, dy = y1 > y0 ? y1 - y0 : 0u;
  uint32_t level = ceil_log2((dx > dy ? dx : dy) + 1u);
  if (level > H.levels - 1) level = H.levels - 1;
  uint32_t lw = H.w[level], lh = H.h[level];
  // mip 0 from the view's depth image when the build left it there (VGC_VIEW_DEPTH_AS_MIP0; same size and values)
  const float *mip = (level == 0 && V.hzb_mip0) ? V.hzb_mip0 : H.data + H.off[level];
  uint32_t tx0 = min(x0 >> level, lw - 1), tx1 = min(x1 >> level, lw - 1);
  uint32_t ty0 = min(y0 >> level, lh - 1), ty1 = min(y1 >> level, lh - 1);
  float s00 = __ldg(mip + ty0 * lw + tx0), s10 = __ldg(mip + ty0 * lw + tx1);
  float s01 = __ldg(mip + ty1 * lw + tx0), s11 = __ldg(mip + ty1 * lw + tx1);
  float hmax = fmx(fmx(s00, s10), fmx(s01, s11));
  return min_z > hmax + float(1e-6);
}

// The scene a view reads. A launch over one context passes its Scene by value (kernel parameter space: no registers
// held) and its HZB descriptors as a read-only parameter; a multi-scene launch (views of several contexts in one
// batch) reads the view's entry of a scene table, and that scene's descriptors.
template <bool MULTI>
struct SceneOf {
  __device__ __forceinline__ static const Scene &get(const Scene &S, const Scene *, const ViewConst &) { return S; }
  __device__ __forceinline__ static const HzbDesc *hzbs(const HzbDesc *hzbs, const Scene &) { return hzbs; }
};
template <>
struct SceneOf<true> {
  __device__ __forceinline__ static Scene get(const Scene &, const Scene *scenes, const ViewConst &V) {
    return scenes[V.scene];
  }
  __device__ __forceinline__ static const HzbDesc *hzbs(const HzbDesc *, const Scene &S) { return S.hzbs; }
};

// occludedSphere (GeometryPool.ts:701-705): the sphere grows by the camera band's top error in pixels
__device__ __forceinline__ bool occluded(const ViewConst &V, const HzbDesc *hzbs, float high0, bool on, const float c[3],
                                         float r) {
  if (!on || !V.occl_active || V.hzb < 0) return false;
  float margin = (fabsf(c[2]) * high0) * V.inv_proj_scale;
  return hzb_occluded(V, hzbs[V.hzb], c, r + margin);
}

// projectedError (GeometryPool.ts:678-683) in two parts: pixels = num / dist, num = (error * scale) * projScale,
// dist = max(|VM c| - r scale, near) > 0. A band edge x is tested as num <= x * dist (no division); the value itself
// is divided out only where the fade steps or the budget bins need it. error >= 1e30 / 2 (no parent) is infinite.
struct ProjErr {
  float num, dist;
};
constexpr float kErrInf = float(1e30 * 0.5);

__device__ __forceinline__ ProjErr proj_parts(const ViewConst &V, const float *VM, float scale, float4 s, float error) {
  float c[3];
  xform(VM, s.x, s.y, s.z, c);
  return {(error * scale) * V.proj_scale, fmx(__fmaf_rn(-s.w, scale, len3(c)), V.near_)};
}
// pixels <= x
__device__ __forceinline__ bool err_le(ProjErr p, float error, float x) { return error < kErrInf && p.num <= x * p.dist; }
// pixels > x
__device__ __forceinline__ bool err_gt(ProjErr p, float error, float x) { return error >= kErrInf || p.num > x * p.dist; }
__device__ __forceinline__ float err_value(float num, float dist, float error) {
  return error >= kErrInf ? 1e30f : num / dist;
}

// lodFadeRange's step of a projected error e against the band's low edge (1 / low passed in): rint(ln(e / low) *
// fadeScale) clamped to [0, 255]
__device__ __forceinline__ uint32_t fade_step(float e, float inv_low, float fade_scale) {
  float x = rintf(vg_logf(fmx(e, float(1e-30)) * inv_low) * fade_scale);
  x = fmn(fmx(x, 0.0f), 255.0f);
  return uint32_t(x);
}

__device__ __forceinline__ uint32_t part_of(uint32_t packed) { return (packed & 0xffff00u) == kFullFadeBits ? 0u : 1u; }

__device__ __forceinline__ uint32_t *mesh_count(const ViewConst &V, uint32_t slot_capacity, uint32_t cut, uint32_t slot,
                                                uint32_t part) {
  return V.counters + VGC_COUNTER_HEADER + (((cut * slot_capacity + slot) * 2 + part) * 2);
}

// ------------------------------------------------------------------------------------------------ k_cells
template <bool MULTI>
__global__ void __launch_bounds__(256) k_cells(Scene S0, const Scene *__restrict__ scenes,
                                               const ViewConst *__restrict__ views, uint32_t nviews,
                                               uint32_t total_units, uint2 *__restrict__ units,
                                               uint32_t *__restrict__ unit_count) {
  const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  if ((u & ~31u) >= total_units) return;  // whole warp out of range
  // view of this unit: each view's range starts at a multiple of 32, so a warp never spans two views
  uint32_t lo = 0, hi = nviews;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (views[mid].unit_offset <= u) lo = mid;
    else hi = mid;
  }
  const uint32_t v = lo;
  const ViewConst &V = views[v];
  const auto &S = SceneOf<MULTI>::get(S0, scenes, V);
  const uint32_t cell = u - V.unit_offset;
  bool vis = false;
  if (cell < S.cell_count) {
    CellRec cr = S.cells[cell];
    const MeshRec &mesh = S.meshes[cr.slot];
    vis = mesh.enabled != 0 && (!V.cascade || mesh.shadow != 0);  // a cascade draws shadow casters only
    float c[3];
    xform(V.V, cr.sphere.x, cr.sphere.y, cr.sphere.z, c);
    float radius = cr.sphere.w;
    if (vis && V.frustum && frustum(V, c, mesh.shadow != 0) < -radius) vis = false;
    if (vis) {
      float min_pixels = fmx(V.min_pixel_radius, mesh.min_pixel_radius);
      float max_r = cr.max_radius;
      float gap = len3(c) - radius;
      if (gap > max_r && (max_r * V.proj_scale) / fmx(gap, float(1e-6)) < min_pixels) vis = false;
      if (gap > mesh.max_draw_distance) vis = false;
    }
  }
  const uint32_t mask = __ballot_sync(0xffffffffu, vis);
  if (!mask) return;
  const uint32_t leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) {
    base = atomicAdd(unit_count, __popc(mask));
    atomicAdd(V.counters + VGC_COUNTER_CELLS, __popc(mask));
  }
  base = __shfl_sync(0xffffffffu, base, leader);
  if (vis) units[base + __popc(mask & ((1u << lane) - 1u))] = make_uint2(v, cell);
}

// ------------------------------------------------------------------------------------------------ k_instances
constexpr int kWarpStage = 96;   // staged draw entries per warp (a step adds <= 32; one cut at a time)
// The meshlet work queue between k_instances and k_chunks, in one buffer of `capacity` uint4: spans (one item's
// meshlets inside one window of 2^chunk_shift meshlets of its warp's items laid end to end; 512 unless the batch's
// autotuner picked 256 or 1024) and chunks (the <= 32 spans of one window: one (view, cell, cut)). ctl[4..5] is the 64-bit reservation counter: spans low, chunks high.
struct WorkQueue {
  uint4 *spans, *chunks;
  uint32_t span_cap, chunk_cap;
};

__device__ __forceinline__ WorkQueue work_queue(uint4 *buf, uint32_t capacity) {
  WorkQueue q;
  q.chunk_cap = capacity / 4;
  q.span_cap = capacity - q.chunk_cap;
  q.spans = buf;
  q.chunks = buf + q.span_cap;
  return q;
}

__device__ __forceinline__ unsigned long long *queue_counter(uint32_t *ctl) {
  return reinterpret_cast<unsigned long long *>(ctl + 4);
}

// Work is handed out to warps from counters (WarpFeed; ctl[8]: chunks, ctl[9]: instance units, ctl[11]: redo words),
// so warps that drew cheap pieces take more and the persistent grid ends together; the counters empty with the
// queue.
constexpr uint32_t kCtlNextChunk = 8, kCtlNextUnit = 9;
constexpr uint32_t kCtlOverflowed = 10, kCtlNextRedo = 11;  // a unit's items did not fit the queue; k_instances_redo's counter
__device__ __forceinline__ uint32_t warp_grab(uint32_t *ctl, uint32_t word) {
  uint32_t i = 0;
  if ((threadIdx.x & 31) == 0) i = atomicAdd(ctl + word, 1u);
  return __shfl_sync(0xffffffffu, i, 0);
}

// End of a pass over the work queue (one thread): ctl[6] / ctl[7] keep the most spans / chunks any pass of the
// launch sequence asked for (the host grows the queue from them for the next launch), and the queue empties.
__device__ __forceinline__ void retire_queue(uint32_t *ctl) {
  const unsigned long long q = *queue_counter(ctl);
  ctl[6] = max(ctl[6], uint32_t(q));
  ctl[7] = max(ctl[7], uint32_t(q >> 32));
  *queue_counter(ctl) = 0;
  ctl[kCtlNextChunk] = 0;
  ctl[kCtlNextUnit] = 0;
  ctl[kCtlOverflowed] = 0;
  ctl[kCtlNextRedo] = 0;
}

// Band values of a view for the current round, written by k_reset and by the capacity check (dyn[1..5]).
struct ViewBands {
  float low0, low1, high0, high1, fade_scale;
};

__device__ __forceinline__ ViewBands bands_of(const ViewConst &V) {
  const float *d = V.dyn;
  return ViewBands{d[1], d[2], d[3], d[4], d[5]};
}

__device__ __forceinline__ void store_bands(const ViewConst &V, float threshold) {
  Bands b;
  load_bands(V, threshold, b);
  V.dyn[0] = threshold;
  V.dyn[1] = b.low[0];
  V.dyn[2] = b.low[1];
  V.dyn[3] = b.high[0];
  V.dyn[4] = b.high[1];
  V.dyn[5] = b.fade_scale;
}

// Drawn entries of one warp waiting for their draw-list positions; the counts are warp-uniform registers.
struct WarpStage {  // a warp stages one cut at a time: every stage is flushed before the warp switches cut
  uint4 e[kWarpStage];
};

struct WarpCount {
  uint32_t n;     // staged entries of this cut
  uint32_t idx0;  // index counts per part, relative to the warp's next region reservation
  uint32_t idx1;
};

__device__ __forceinline__ uint32_t warp_scan_incl(uint32_t v) {
  const uint32_t lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= (uint32_t)o) v += t;
  }
  return v;
}

// Writes one warp's staged entries of `cut` to the view's draw list: one global atomic for the list position and
// one per part for the mesh's index region (GeometryPool.ts:959-965). Entries past max_drawn are dropped and only
// the kept ones are counted in the index region, as the reference does.
__device__ __forceinline__ void warp_flush(WarpStage &ws, WarpCount &wc, const ViewConst &V, uint32_t slot_capacity,
                                           uint32_t slot, uint32_t cut) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = wc.n;
  if (!n) return;
  __syncwarp();
  uint32_t base = 0, kept = 0, b0 = 0, b1 = 0;
  if (lane == 0) {
    base = atomicAdd(V.counters + C_CUT(cut) + VGC_CUT_SELECTED, n);
    kept = base >= V.max_drawn ? 0u : min(n, V.max_drawn - base);
    uint32_t add0 = wc.idx0, add1 = wc.idx1;
    if (kept != n) {  // overflow: re-pack the kept prefix
      add0 = add1 = 0;
      for (uint32_t s = 0; s < kept; s++) {
        uint4 &e = ws.e[s];
        const uint32_t tri3 = (e.w & 255u) * 3u;
        if (part_of(e.w)) {
          e.z = add1;
          add1 += tri3;
        } else {
          e.z = add0;
          add0 += tri3;
        }
      }
    }
    b0 = add0 ? atomicAdd(mesh_count(V, slot_capacity, cut, slot, 0), add0) : 0u;
    b1 = add1 ? atomicAdd(mesh_count(V, slot_capacity, cut, slot, 1), add1) : 0u;
  }
  base = __shfl_sync(0xffffffffu, base, 0);
  kept = __shfl_sync(0xffffffffu, kept, 0);
  b0 = __shfl_sync(0xffffffffu, b0, 0);
  b1 = __shfl_sync(0xffffffffu, b1, 0);
  __syncwarp();
  uint4 *dst = V.draw_list + (size_t)cut * V.max_drawn + base;
  for (uint32_t s = lane; s < kept; s += 32) {
    uint4 e = ws.e[s];
    e.z += part_of(e.w) ? b1 : b0;
    dst[s] = e;
  }
  __syncwarp();
  wc.n = 0;
  wc.idx0 = wc.idx1 = 0;
}

// Stages the drawn entries of one warp-wide step (warp-aggregated: one ballot, one packed 16 + 16-bit scan of the
// two parts' index counts), flushing when the next step might not fit.
__device__ __forceinline__ void warp_stage(WarpStage &ws, WarpCount &wc, const ViewConst &V, uint32_t slot_capacity,
                                           uint32_t slot, uint32_t cut, bool drawn, uint32_t instance, uint32_t meshlet,
                                           uint32_t packed) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t mask = __ballot_sync(0xffffffffu, drawn);
  if (!mask) return;
  const uint32_t tri3 = drawn ? (packed & 255u) * 3u : 0u;
  const uint32_t part = part_of(packed);
  const uint32_t mine = part == 0 ? tri3 : (tri3 << 16);
  const uint32_t incl = warp_scan_incl(mine);
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  if (drawn) {
    const uint32_t excl = incl - mine;
    const uint32_t local = part == 0 ? wc.idx0 + (excl & 0xffffu) : wc.idx1 + (excl >> 16);
    ws.e[wc.n + __popc(mask & ((1u << lane) - 1u))] = make_uint4(instance, meshlet, local, packed);
  }
  wc.n += __popc(mask);
  wc.idx0 += total & 0xffffu;
  wc.idx1 += total >> 16;
  if (wc.n > kWarpStage - 32) warp_flush(ws, wc, V, slot_capacity, slot, cut);
}

// The per-meshlet test of GeometryPool.ts:938-957. The conditions are evaluated LOD band first (it rejects most
// meshlets and needs no HZB samples), then the culling sphere against the frustum and, for the camera cut, the HZB;
// `drawn` is their conjunction either way. `packed` receives triCount | lo << 8 | hi << 16.
__device__ __forceinline__ bool test_meshlet(const Scene &S, const ViewConst &V, const HzbDesc *hzbs, float low,
                                             float high, float fs, float high0, uint32_t cut, bool occl_on,
                                             bool inside, const float *VM, uint32_t meshlet, uint32_t &packed,
                                             uint32_t &id) {
  const float scale = VM[12];
  const float4 ls = __ldg(S.m_lod + meshlet), ps = __ldg(S.m_parent + meshlet), er = __ldg(S.m_err + meshlet);
  const ProjErr own = proj_parts(V, VM, scale, ls, er.x);
  const ProjErr parent = proj_parts(V, VM, scale, ps, er.y);
  if (!(err_le(own, er.x, high) && err_gt(parent, er.y, low))) return false;
  id = __float_as_uint(er.w);  // pool-global meshlet id (the columns are in test order)
  uint32_t lo = 0u, hi = 255u;
  if (fs > 0.0f) {
    const float inv_low = 1.0f / low;
    lo = fade_step(err_value(own.num, own.dist, er.x), inv_low, fs);
    hi = fade_step(err_value(parent.num, parent.dist, er.y), inv_low, fs);
  }
  if (!(hi > lo)) return false;
  packed = __float_as_uint(er.z) | (lo << 8) | (hi << 16);
  const float4 cs = __ldg(S.m_cull + meshlet);
  float c[3];
  xform(VM, cs.x, cs.y, cs.z, c);
  const float r = cs.w * scale;
  // `inside`: the instance's cullBoundsSphere, which encloses every meshlet's culling sphere, is inside the frustum
  if (V.frustum && !inside && !(frustum(V, c, cut == 1) >= -r)) return false;
  if (cut == 0 && occluded(V, hzbs, high0, occl_on, c, r)) return false;
  return true;
}

struct LevelRange {
  uint32_t first, last, possible, guaranteed;
  uint32_t lfirst, llast;  // first and last possible level
};

// selectLevels' level loop (GeometryPool.ts:788-812) over the mesh's level table (read through L1: every lane
// of a warp reads the same entries)
__device__ __forceinline__ LevelRange level_range(const LevelRec *L, uint32_t levels, float low, float high,
                                                  float px_min, float px_max) {
  LevelRange r{0xffffffffu, 0u, 0u, 0u, 0u, 0u};
  for (uint32_t l = 0; l < levels; l++) {
    const LevelRec e = L[l];
    const bool possible = e.min_own * px_max <= high && (e.max_parent >= float(1e30 * 0.5) || e.max_parent * px_min > low);
    const bool sure = e.max_own * px_min <= low * float(1 - 1e-3) &&
                      (e.min_parent >= float(1e30 * 0.5) || e.min_parent * px_max > high * float(1 + 1e-3));
    if (possible) {
      if (r.possible == 0) r.lfirst = l;
      r.llast = l;
      r.first = min(r.first, e.first);
      r.last = max(r.last, e.first + e.count);
      r.possible += e.count;
      if (sure) r.guaranteed += e.count;
    }
  }
  return r;
}

// The meshlets of an item that can pass the LOD band (own <= high && parent > low). With every meshlet's LOD and
// parent spheres inside the mesh's LOD sphere, each meshlet's max(|V M c| - r s, near) lies between the mesh's
// max(d - R s, near) and max(d + R s, near), so its projected parent error is at most parentError * px_min and its
// own at least ownError * px_max. Within a level the meshlets are in parent-error order: the first possible level's
// meshlets with parentError * px_min below `low` form a prefix, and the last possible level's meshlets from the point
// where the smallest remaining ownError * px_max exceeds `high` form a suffix; both fail for certain and are cut.
// The level samples give the cut points to 1/64 of a level; the margin of 1e-4 covers float rounding.
__device__ __forceinline__ void trim_item(const Scene &S, const MeshRec &mesh, const LevelRec *L, const LevelRange &r,
                                          float low, float high, float px_min, float px_max, uint32_t &first,
                                          uint32_t &last) {
  first = r.first;
  last = r.last;
  if (!mesh.range_cut || !(r.last > r.first)) return;
  const float2 *a = S.lsamples + (size_t)(mesh.level_base + r.lfirst) * kLevelSamples;
  int k = -1;  // last sample whose parent error surely fails (samples are non-decreasing)
#pragma unroll
  for (int step = 32; step > 0; step >>= 1) {
    const float e = a[k + step].x;
    if (k + step < int(kLevelSamples) && e < float(1e30 * 0.5) && (e * px_min) * 1.0001f <= low) k += step;
  }
  const LevelRec lf = L[r.lfirst];
  if (k > 0) first = lf.first + uint32_t(((uint64_t)k * lf.count) / kLevelSamples);
  const float2 *b = S.lsamples + (size_t)(mesh.level_base + r.llast) * kLevelSamples;
  int j = int(kLevelSamples);  // first sample from which every own error surely fails (suffix minima non-decreasing)
#pragma unroll
  for (int step = 32; step > 0; step >>= 1) {
    if (j - step >= 0 && (b[j - step].y * px_max) > high * 1.0001f) j -= step;
  }
  const LevelRec ll = L[r.llast];
  if (j < int(kLevelSamples)) last = ll.first + uint32_t(((uint64_t)j * ll.count) / kLevelSamples);
  if (last < first) last = first;
}

// Fast-path entries of one cut for a warp (GeometryPool.ts:827-836): up to 4 meshlets per lane, placed with one
// atomic for the list position and one for the mesh's region (part 0: drawn over every pixel).
__device__ __forceinline__ void emit_fast(const Scene &S, const ViewConst &V, uint32_t slot, uint32_t cut,
                                          uint32_t n, uint32_t first, uint32_t instance) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t incl_n = warp_scan_incl(n);
  const uint32_t total_n = __shfl_sync(0xffffffffu, incl_n, 31);
  if (!total_n) return;
  uint32_t base = 0;
  if (lane == 0) base = atomicAdd(V.counters + C_CUT(cut) + VGC_CUT_SELECTED, total_n);
  base = __shfl_sync(0xffffffffu, base, 0) + (incl_n - n);
  uint32_t tri[kFastPathMax], id[kFastPathMax];
  uint32_t kept_tri3 = 0;
#pragma unroll
  for (uint32_t k = 0; k < kFastPathMax; k++) {
    const float4 er = k < n ? S.m_err[first + k] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    tri[k] = __float_as_uint(er.z);
    id[k] = __float_as_uint(er.w);
    if (k < n && base + k < V.max_drawn) kept_tri3 += tri[k] * 3u;
  }
  const uint32_t incl_t = warp_scan_incl(kept_tri3);
  const uint32_t total_t = __shfl_sync(0xffffffffu, incl_t, 31);
  uint32_t ib = 0;
  if (lane == 0 && total_t) ib = atomicAdd(mesh_count(V, S.slot_capacity, cut, slot, 0), total_t);
  uint32_t acc = __shfl_sync(0xffffffffu, ib, 0) + (incl_t - kept_tri3);
  uint4 *dst = V.draw_list + (size_t)cut * V.max_drawn;
#pragma unroll
  for (uint32_t k = 0; k < kFastPathMax; k++)
    if (k < n && base + k < V.max_drawn) {
      dst[base + k] = make_uint4(instance, id[k], acc, tri[k] | kFullFadeBits);
      acc += tri[k] * 3u;
    }
}

// ---- triangleBudget search. Thresholds t_k = lo + (hi - lo) * (k / 255) over thresholdRange, effective
// e_k = t_k * cameraScale, band high edge high_k (e_k * width while the LOD-blend band is open at t_k, else e_k).
// A meshlet of a visible instance is drawn in the camera cut at t_k (blend band included) iff b_own <= k < b_par,
// with b_own = the first k such that own <= high_k and b_par = the first k such that parent <= e_k. Its triangles
// enter the histogram at b_own and leave at b_par, so T(t_k) counts the triangles the cut at t_k draws.
__device__ __forceinline__ float budget_e(const ViewConst &V, float s, uint32_t k) {
  return (V.budget_lo + (V.budget_hi - V.budget_lo) * (float(k) / 255.0f)) * s;
}

// high_k, with load_bands' arithmetic for the threshold t_k (the final pass at the chosen bin uses the same value)
__device__ __forceinline__ float budget_high(const ViewConst &V, float s, uint32_t k) {
  const float x = budget_e(V, s, k);
  float t = (x - 1.25f) / 1.25f;
  t = fmn(fmx(t, 0.0f), 1.0f);
  const float smooth = (t * t) * (3.0f - 2.0f * t);
  const float width = 1.0f + (V.lod_blend_max - 1.0f) * smooth;
  return width > float(1.001) ? x * width : x;
}

// first k with own <= high_k (kBudgetBins when none); high_k does not decrease with k. The comparisons are the
// cut's own (err_le), so the bins agree with the decisions of the pass at the chosen threshold.
__device__ __forceinline__ uint32_t budget_bin_high(const ViewConst &V, float s, ProjErr p, float error) {
  if (error >= kErrInf) return kBudgetBins;
  uint32_t lo = 0, hi = kBudgetBins;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (err_le(p, error, budget_high(V, s, mid))) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// first k with parent <= e_k (kBudgetBins when none)
__device__ __forceinline__ uint32_t budget_bin(const ViewConst &V, float s, ProjErr p, float error) {
  if (error >= kErrInf) return kBudgetBins;
  // estimate, then exact comparisons with e_k (bounded: the estimate is off by a few bins at most)
  const float x = p.num / p.dist;
  const float guess = ((x / s - V.budget_lo) / (V.budget_hi - V.budget_lo)) * 255.0f;
  int k = guess != guess ? 0 : (guess < 0.0f ? 0 : (guess > 256.0f ? 256 : int(guess)));
  for (int i = 0; i < 600 && k > 0 && err_le(p, error, budget_e(V, s, uint32_t(k - 1))); i++) k--;
  for (int i = 0; i < 600 && k < int(kBudgetBins) && !err_le(p, error, budget_e(V, s, uint32_t(k))); i++) k++;
  return uint32_t(k);
}

// Histogram bins of one meshlet (camera cut): false when it is in no cut of the range or culled.
__device__ __forceinline__ bool hist_meshlet(const Scene &S, const ViewConst &V, const HzbDesc *hzbs, float s,
                                             float high0, bool occl_on, bool inside, const float *VM, uint32_t meshlet,
                                             uint32_t &bo, uint32_t &bp, uint32_t &tris) {
  const float scale = VM[12];
  const float4 ls = __ldg(S.m_lod + meshlet), ps = __ldg(S.m_parent + meshlet), er = __ldg(S.m_err + meshlet);
  bo = budget_bin_high(V, s, proj_parts(V, VM, scale, ls, er.x), er.x);
  bp = budget_bin(V, s, proj_parts(V, VM, scale, ps, er.y), er.y);
  if (!(bo < bp)) return false;
  tris = __float_as_uint(er.z);
  const float4 cs = __ldg(S.m_cull + meshlet);
  float c[3];
  xform(VM, cs.x, cs.y, cs.z, c);
  const float r = cs.w * scale;
  if (V.frustum && !inside && !(frustum(V, c, false) >= -r)) return false;
  if (occluded(V, hzbs, high0, occl_on, c, r)) return false;
  return true;
}

// Adds one warp step's triangles to the view's histogram: one atomic per distinct bin in the warp.
__device__ __forceinline__ void warp_hist_add(unsigned long long *hist, bool add, uint32_t bin, uint32_t tris) {
  uint32_t pending = __ballot_sync(0xffffffffu, add && bin < kBudgetBins);
  while (pending) {
    const uint32_t key = __shfl_sync(0xffffffffu, bin, __ffs(pending) - 1);
    const uint32_t group = __ballot_sync(0xffffffffu, add && bin == key);
    const uint32_t sum = __reduce_add_sync(0xffffffffu, (group >> (threadIdx.x & 31)) & 1u ? tris : 0u);
    if ((threadIdx.x & 31) == __ffs(group) - 1) atomicAdd(hist + key, (unsigned long long)sum);
    pending &= ~group;
  }
}

// Tests a whole item (one instance's meshlets [first, first + count) of one cut) with the warp: the fallback when
// the chunk queue is full. HIST: the budget histogram instead of the draw list.
template <bool HIST>
__device__ void warp_item(const Scene &S, const ViewConst &V, const HzbDesc *hzbs, WarpStage &ws, uint32_t slot,
                          uint32_t cut, bool occl_on, bool inside, const float *VM, uint32_t instance, uint32_t first,
                          uint32_t count) {
  const ViewBands b = bands_of(V);
  if (HIST) {
    const float s = get_state(V.state, 0);
    for (uint32_t base = 0; base < count; base += 32) {
      const uint32_t t = base + (threadIdx.x & 31);
      uint32_t bo = 0, bp = 0, tris = 0;
      const bool add = t < count && hist_meshlet(S, V, hzbs, s, b.high0, occl_on, inside, VM, first + t, bo, bp, tris);
      warp_hist_add(V.hist, add, bo, tris);
      warp_hist_add(V.hist + kBudgetBins, add, bp, tris);
    }
    return;
  }
  const float low = cut ? b.low1 : b.low0, high = cut ? b.high1 : b.high0;
  WarpCount wc{0, 0, 0};
  for (uint32_t base = 0; base < count; base += 32) {
    const uint32_t t = base + (threadIdx.x & 31);
    bool drawn = false;
    uint32_t packed = 0, id = 0;
    if (t < count)
      drawn = test_meshlet(S, V, hzbs, low, high, b.fade_scale, b.high0, cut, occl_on, inside, VM, first + t, packed, id);
    warp_stage(ws, wc, V, S.slot_capacity, slot, cut, drawn, instance, id, packed);
  }
  warp_flush(ws, wc, V, S.slot_capacity, slot, cut);
}

// Meshlets of one chunk that passed the LOD band (HIST: that enter the cut somewhere in the threshold range),
// waiting for the rest of their test with all 32 lanes busy: about a third of the tested meshlets pass, and testing
// them in place would leave most lanes idle.
struct LodQueue {
  uint32_t pos[64], span[64];
  float own[64], parent[64];  // the projected errors' distances (ProjErr::dist); HIST: the bins b_own, b_par as integers
};

// Per warp: the view-model matrix of each span's instance (rows 0..2, scale), its instance and inside flag, and the
// offset from a laid-out position in the chunk to the meshlet it names.
struct SpanFrame {
  float4 vm[32][4];  // [3] = (VM[12] scale, instance as bits, inside as bits, first meshlet - start as bits)
};

__device__ __forceinline__ uint32_t frame_vm(const SpanFrame &F, uint32_t j, float *VM, uint32_t &instance,
                                             bool &inside) {
  const float4 a = F.vm[j][0], b = F.vm[j][1], c = F.vm[j][2], d = F.vm[j][3];
  VM[0] = a.x, VM[1] = a.y, VM[2] = a.z, VM[3] = a.w;
  VM[4] = b.x, VM[5] = b.y, VM[6] = b.z, VM[7] = b.w;
  VM[8] = c.x, VM[9] = c.y, VM[10] = c.z, VM[11] = c.w;
  VM[12] = d.x;
  instance = __float_as_uint(d.y);
  inside = __float_as_uint(d.z) != 0;
  return __float_as_uint(d.w);
}

// The rest of the meshlet test for queue entries [0, n): fade steps (the projected errors divided out here, for the
// meshlets that passed the band), culling sphere against the frustum, HZB; then staging (draw list) or the histogram
// (HIST).
template <bool HIST>
__device__ __forceinline__ void drain_queue(const Scene &S, const ViewConst &V, const HzbDesc *hzbs, const LodQueue &q,
                                            const SpanFrame &F, uint32_t n, WarpStage &ws, WarpCount &wc, float inv_low,
                                            float fs, float high0, uint32_t cut, bool occl_on, uint32_t slot) {
  const uint32_t lane = threadIdx.x & 31;
  bool drawn = false;
  uint32_t packed = 0, id = 0, instance = 0, lo = 0, hi = 255;
  if (lane < n) {
    const uint32_t pos = q.pos[lane];
    float VM[13];
    bool inside;
    frame_vm(F, q.span[lane], VM, instance, inside);
    const float4 er = __ldg(S.m_err + pos);
    const float4 cs = __ldg(S.m_cull + pos);
    float c[3];
    xform(VM, cs.x, cs.y, cs.z, c);
    const float r = cs.w * VM[12];
    // visible: the culling sphere against the frustum and, for the camera cut, the HZB; a meshlet is drawn when it
    // is visible and its fade range [lo, hi) is not empty, so the fade steps (a division and a log each) are taken
    // only for the visible ones
    const bool visible = !(V.frustum && !inside && !(frustum(V, c, cut == 1) >= -r)) &&
                         !(cut == 0 && occluded(V, hzbs, high0, occl_on, c, r));
    if (HIST) {
      lo = __float_as_uint(q.own[lane]);
      hi = __float_as_uint(q.parent[lane]);
      drawn = visible;
    } else if (visible) {
      if (fs > 0.0f) {
        lo = fade_step(err_value((er.x * VM[12]) * V.proj_scale, q.own[lane], er.x), inv_low, fs);
        hi = fade_step(err_value((er.y * VM[12]) * V.proj_scale, q.parent[lane], er.y), inv_low, fs);
      }
      drawn = hi > lo;
    }
    id = __float_as_uint(er.w);
    packed = HIST ? __float_as_uint(er.z) : (__float_as_uint(er.z) | (lo << 8) | (hi << 16));
  }
  if (HIST) {
    warp_hist_add(V.hist, drawn, lo, packed);
    warp_hist_add(V.hist + kBudgetBins, drawn, hi, packed);
  } else {
    warp_stage(ws, wc, V, S.slot_capacity, slot, cut, drawn, instance, id, packed);
  }
}

// Survivors of a half-unit's instance tests, compacted per warp: instance index in the cell (7 bits) and flags, the
// LOD sphere's pixel scales at its near and far distances.
struct Survivor {
  uint32_t bits;  // il | camera << 7 | shadow << 8 | inside0 << 9 | inside1 << 10
  float px_min, px_max;
};
constexpr uint32_t kHalfUnit = 64;  // instances of one (view, cell) unit a warp tests at a time

// One half-unit w (instances 64 (w & 1) .. + 63 of the visible (view, cell) unit w >> 1) of the instance pass. The
// warp first runs the instance tests (frustum, minimum pixel size, draw distance, occlusion) over the half-unit, 32
// instances at a time, and compacts the survivors in order into `list`; the level ranges, item trimming, fast path,
// counters and span / chunk emission then run on full warps of survivors (pass p: survivors 32 p .. 32 p + 31).
// Overflow bit 2 w + p marks a pass whose items did not fit the chunk queue. REDO: pass `redo_pass` of such a
// half-unit; its tests are repeated (the same arithmetic and order, so the same survivors and items) and its items
// tested in place; its counters and fast-path meshlets were already emitted.
template <bool HIST, bool MULTI, bool REDO>
__device__ __forceinline__ void instance_unit(const Scene &S0, const Scene *__restrict__ scenes,
                                              const ViewConst *__restrict__ views, const HzbDesc *__restrict__ hzbs0,
                                              const uint2 *__restrict__ units, uint32_t *__restrict__ ctl,
                                              uint4 *__restrict__ queue, uint32_t capacity, int round,
                                              uint32_t chunk_shift, uint32_t *__restrict__ overflow, WarpStage *ws,
                                              Survivor *__restrict__ list, uint32_t w, uint32_t redo_pass) {
  const uint32_t lane = threadIdx.x & 31;
  const uint2 unit = units[w >> 1];
  const ViewConst &V = views[unit.x];
  if (HIST && !(V.budget > 0.0f)) return;
  bool redo0 = true, redo1 = !HIST;
  if (round > 0) {
    redo0 = V.counters[VGC_COUNTER_REDO0] != 0;
    redo1 = V.counters[VGC_COUNTER_REDO1] != 0;
    if (!redo0 && !redo1) return;
  }
  const auto &S = SceneOf<MULTI>::get(S0, scenes, V);
  const HzbDesc *__restrict__ hzbs = SceneOf<MULTI>::hzbs(hzbs0, S);
  const CellRec cell = S.cells[unit.y];
  const uint32_t base = (w & 1u) * kHalfUnit;
  if (base >= cell.count) return;
  const MeshRec &mesh = S.meshes[cell.slot];
  const ViewBands b = bands_of(V);
  const uint32_t levels = min(mesh.level_count, kMaxLevels);
  const LevelRec *L = S.levels + mesh.level_base;
  const bool occl_on = mesh.occlusion != 0;
  const bool no_frustum = !V.frustum;
  // ---- instance tests, compacted
  uint32_t n_surv = 0, n_occl = 0;  // warp-uniform
  for (uint32_t q = 0; q < kHalfUnit && base + q < cell.count; q += 32) {
    const uint32_t il = base + q + lane;
    bool camera = false, shadow = false, inside0 = true, inside1 = true;
    float px_min = 0.0f, px_max = 0.0f;
    bool occluded_now = false;
    if (il < cell.count) {
      float VM[13];
      model_view(V.V, S.inst + (size_t)(cell.first + il) * 4, VM, VM[12]);
      const float scale = VM[12];
      float c[3];
      xform(VM, mesh.sphere.x, mesh.sphere.y, mesh.sphere.z, c);
      const float radius = mesh.sphere.w * scale;
      bool in_camera = !V.cascade && (no_frustum || frustum(V, c, false) >= -radius);
      bool in_shadow = mesh.shadow != 0 && (no_frustum || frustum(V, c, true) >= -radius);
      in_camera = in_camera && redo0;
      in_shadow = in_shadow && redo1;
      const float min_pixels = fmx(V.min_pixel_radius, mesh.min_pixel_radius);
      const float view_distance = len3(c);
      const bool too_small = view_distance > radius && (radius * V.proj_scale) / view_distance < min_pixels;
      const bool too_far = view_distance - radius > mesh.max_draw_distance;
      if ((in_camera || in_shadow) && !too_small && !too_far) {
        if (in_camera && occluded(V, hzbs, b.high0, occl_on, c, radius)) {
          in_camera = false;
          occluded_now = true;
        }
        if (in_camera || in_shadow) {
          float lc[3];
          xform(VM, mesh.lod.x, mesh.lod.y, mesh.lod.z, lc);
          const float d = len3(lc), r = mesh.lod.w * scale;
          px_min = (scale * V.proj_scale) / fmx(d - r, V.near_);
          px_max = (scale * V.proj_scale) / fmx(d + r, V.near_);
          float cc[3];
          xform(VM, mesh.cull.x, mesh.cull.y, mesh.cull.z, cc);
          const float cr = mesh.cull.w * scale;
          // inside: the cullBoundsSphere lies in the frustum, so every meshlet passes its frustum test
          if (in_camera) inside0 = no_frustum || frustum(V, cc, false) >= cr;
          if (in_shadow) inside1 = no_frustum || frustum(V, cc, true) >= cr;
          camera = in_camera;
          shadow = in_shadow;
        }
      }
    }
    const bool alive = camera || shadow;
    const uint32_t mask = __ballot_sync(0xffffffffu, alive);
    if (alive)
      list[n_surv + __popc(mask & ((1u << lane) - 1u))] =
          Survivor{il | (camera ? 1u << 7 : 0u) | (shadow ? 1u << 8 : 0u) | (inside0 ? 1u << 9 : 0u) |
                       (inside1 ? 1u << 10 : 0u),
                   px_min, px_max};
    n_surv += __popc(mask);
    n_occl += __popc(__ballot_sync(0xffffffffu, occluded_now));
  }
  __syncwarp();
  if (!HIST && !REDO && lane == 0) {
    uint32_t *ctr = V.counters;
    if (n_occl) atomicAdd(ctr + VGC_COUNTER_OCCLUDED, n_occl);
    atomicAdd(ctr + VGC_COUNTER_INSTANCES_TESTED, min(kHalfUnit, cell.count - base));
    if (base == 0) atomicAdd(ctr + VGC_COUNTER_LEVELS_READ, levels);
  }
  // ---- level ranges, items and their spans / chunks, on full warps of survivors
  for (uint32_t pass = 0; pass * 32 < n_surv; pass++) {
    if (REDO && pass != redo_pass) continue;
    const bool valid = pass * 32 + lane < n_surv;
    Survivor sv{0u, 0.0f, 0.0f};
    if (valid) sv = list[pass * 32 + lane];
    const uint32_t il = sv.bits & 127u, instance = cell.first + il;
    const bool in_camera = (sv.bits >> 7) & 1u, in_shadow = (sv.bits >> 8) & 1u;
    const bool inside0 = (sv.bits >> 9) & 1u, inside1 = (sv.bits >> 10) & 1u;
    const float px_min = sv.px_min, px_max = sv.px_max;
    LevelRange r0{0xffffffffu, 0, 0, 0, 0, 0}, r1{0xffffffffu, 0, 0, 0, 0, 0};
    uint32_t t0f = 0, t0l = 0, t1f = 0, t1l = 0;  // the items' trimmed meshlet ranges
    bool fast0 = false, fast1 = false;
    if (HIST && in_camera) {
      const float sc = get_state(V.state, 0);
      const float e0 = budget_e(V, sc, 0), h255 = budget_high(V, sc, 255);
      r0 = level_range(L, levels, e0, h255, px_min, px_max);
      trim_item(S, mesh, L, r0, e0, h255, px_min, px_max, t0f, t0l);
    } else if (in_camera) {
      r0 = level_range(L, levels, b.low0, b.high0, px_min, px_max);
      fast0 = r0.last > r0.first && r0.possible == r0.last - r0.first && r0.guaranteed == r0.possible &&
              r0.possible <= kFastPathMax && inside0;
      trim_item(S, mesh, L, r0, b.low0, b.high0, px_min, px_max, t0f, t0l);
    }
    if (in_shadow) {
      r1 = level_range(L, levels, b.low1, b.high1, px_min, px_max);
      fast1 = r1.last > r1.first && r1.possible == r1.last - r1.first && r1.guaranteed == r1.possible &&
              r1.possible <= kFastPathMax && inside1;
      trim_item(S, mesh, L, r1, b.low1, b.high1, px_min, px_max, t1f, t1l);
    }
    const bool surv0 = r0.last > r0.first, surv1 = r1.last > r1.first;
    const bool item0 = surv0 && !fast0, item1 = surv1 && !fast1;
    if (!HIST && !REDO) {
      // warp totals for the view's counters (one atomic per counter and warp)
      const uint32_t n_s0 = __popc(__ballot_sync(0xffffffffu, surv0)), n_s1 = __popc(__ballot_sync(0xffffffffu, surv1));
      const uint32_t n_i0 = __popc(__ballot_sync(0xffffffffu, item0)), n_i1 = __popc(__ballot_sync(0xffffffffu, item1));
      const uint32_t fast_m = __reduce_add_sync(0xffffffffu, (fast0 ? r0.possible : 0u) + (fast1 ? r1.possible : 0u));
      const uint32_t tested =
          __reduce_add_sync(0xffffffffu, (item0 ? r0.last - r0.first : 0u) + (item1 ? r1.last - r1.first : 0u));
      const uint32_t queued = __reduce_add_sync(0xffffffffu, (item0 ? t0l - t0f : 0u) + (item1 ? t1l - t1f : 0u));
      if (lane == 0) {
        uint32_t *ctr = V.counters;
        if (n_s0) atomicAdd(ctr + C_CUT(0) + VGC_CUT_SURVIVED, n_s0);
        if (n_s1) atomicAdd(ctr + C_CUT(1) + VGC_CUT_SURVIVED, n_s1);
        if (n_i0) atomicAdd(ctr + C_CUT(0) + VGC_CUT_WORK, n_i0);
        if (n_i1) atomicAdd(ctr + C_CUT(1) + VGC_CUT_WORK, n_i1);
        if (fast_m) atomicAdd(ctr + VGC_COUNTER_FAST_EMITTED, fast_m);
        if (tested) atomicAdd(ctr + VGC_COUNTER_MESHLETS_TESTED, tested);
        if (queued) atomicAdd(ctr + VGC_COUNTER_MESHLETS_QUEUED, queued);
      }
      emit_fast(S, V, cell.slot, 0, fast0 ? r0.possible : 0u, r0.first, instance);
      emit_fast(S, V, cell.slot, 1, fast1 ? r1.possible : 0u, r1.first, instance);
    }
    // items -> spans -> chunks: per cut, the warp's items laid end to end in lane order and cut into windows of
    // 2^chunk_shift meshlets; a window's spans (<= 32, one per item) form one chunk of one (view, cell, cut)
    const uint32_t n0 = item0 ? t0l - t0f : 0u, n1 = item1 ? t1l - t1f : 0u;
    const uint32_t s0 = warp_scan_incl(n0) - n0, s1 = warp_scan_incl(n1) - n1;  // starts in the laid-out items
    const uint32_t T0 = __shfl_sync(0xffffffffu, s0 + n0, 31), T1 = __shfl_sync(0xffffffffu, s1 + n1, 31);
    if (T0 + T1 == 0) continue;
    const uint32_t chunk = 1u << chunk_shift;
    const uint32_t p0 = n0 ? ((s0 + n0 - 1) >> chunk_shift) - (s0 >> chunk_shift) + 1 : 0u;  // spans of this lane's item
    const uint32_t p1 = n1 ? ((s1 + n1 - 1) >> chunk_shift) - (s1 >> chunk_shift) + 1 : 0u;
    const uint32_t q0 = warp_scan_incl(p0) - p0, q1 = warp_scan_incl(p1) - p1;
    const uint32_t P0 = __shfl_sync(0xffffffffu, q0 + p0, 31), P1 = __shfl_sync(0xffffffffu, q1 + p1, 31);
    const uint32_t N0 = (T0 + chunk - 1) >> chunk_shift, N1 = (T1 + chunk - 1) >> chunk_shift;
    if (!REDO) {
      unsigned long long got = 0;
      if (lane == 0)
        got = atomicAdd(queue_counter(ctl), ((unsigned long long)(N0 + N1) << 32) | (unsigned long long)(P0 + P1));
      got = __shfl_sync(0xffffffffu, got, 0);
      const uint32_t span_at = uint32_t(got), chunk_at = uint32_t(got >> 32);
      const WorkQueue Q = work_queue(queue, capacity);
      if (span_at + P0 + P1 <= Q.span_cap && chunk_at + N0 + N1 <= Q.chunk_cap) {
#pragma unroll
        for (uint32_t cut = 0; cut < 2; cut++) {
          const uint32_t n = cut ? n1 : n0, st = cut ? s1 : s0, np = cut ? p1 : p0;
          const uint32_t first = cut ? t1f : t0f;
          const uint32_t flags = il | ((cut ? inside1 : inside0) ? 1u << 7 : 0u);
          uint4 *dst = Q.spans + span_at + (cut ? P0 + q1 : q0);
          for (uint32_t k = 0; k < np; k++) {
            const uint32_t win = (st >> chunk_shift) + k;
            const uint32_t lo = max(st, win << chunk_shift), hi = min(st + n, (win + 1) << chunk_shift);
            dst[k] = make_uint4(flags, first + (lo - st), hi - lo, 0u);
          }
          // chunk t (lane t % 32) starts at the span holding laid-out position X = t * chunk: that of the last item
          // starting at or before X, plus the windows that item crossed before t; its spans are the non-empty items
          // meeting [X, X + chunk). The lanes' starts `st` and ends `st + n` do not decrease with the lane, so each is
          // a search over the lanes (by shuffles).
          const uint32_t N = cut ? N1 : N0, q = cut ? q1 : q0, e = st + n;
          const uint32_t nonempty = __ballot_sync(0xffffffffu, n > 0);
          for (uint32_t t0 = 0; t0 < N; t0 += 32) {
            const uint32_t t = t0 + lane, X = t << chunk_shift;
            uint32_t owner = 0, a = 0, b = 0;  // last lane with st <= X; with st < X + chunk; with st + n <= X
#pragma unroll
            for (uint32_t step = 16; step > 0; step >>= 1) {
              if (__shfl_sync(0xffffffffu, st, owner + step) <= X) owner += step;
              if (__shfl_sync(0xffffffffu, st, a + step) < X + chunk) a += step;
              if (__shfl_sync(0xffffffffu, e, b + step) <= X) b += step;
            }
            const uint32_t o_q = __shfl_sync(0xffffffffu, q, owner), o_st = __shfl_sync(0xffffffffu, st, owner);
            const uint32_t e0 = __shfl_sync(0xffffffffu, e, 0);
            const uint32_t before = e0 <= X ? __popc(nonempty & ((2u << b) - 1u)) : 0u;  // items ending by X
            const uint32_t spans = __popc(nonempty & ((2u << a) - 1u)) - before;
            if (t < N)
              Q.chunks[chunk_at + (cut ? N0 : 0u) + t] =
                  make_uint4(unit.x, unit.y, cut | ((cut == 0 && occl_on) ? 2u : 0u) | (spans << 8),
                             span_at + (cut ? P0 : 0u) + o_q + t - (o_st >> chunk_shift));
          }
        }
        continue;
      }
      // the queue is full: chunk slots reserved below its capacity become empty records, and the pass is marked for
      // k_instances_redo, which tests its items in place
      for (uint32_t t = lane; t < N0 + N1; t += 32)
        if (chunk_at + t < Q.chunk_cap) Q.chunks[chunk_at + t] = make_uint4(0u, 0u, 0u, 0u);
      const uint32_t bit = 2u * w + pass;
      if (lane == 0) {
        atomicOr(overflow + (bit >> 5), 1u << (bit & 31));
        ctl[kCtlOverflowed] = 1;
      }
    }
    if (REDO) {
      uint32_t over = __ballot_sync(0xffffffffu, n0 + n1 > 0);
      while (over) {
        const uint32_t j = __ffs(over) - 1;
        over &= over - 1;
        const uint32_t inst = cell.first + __shfl_sync(0xffffffffu, il, j);
        // instance j's view-model matrix, recomputed (the same arithmetic as in the tests) rather than kept live
        float vmj[13];
        model_view(V.V, S.inst + (size_t)inst * 4, vmj, vmj[12]);
        const bool jin0 = __shfl_sync(0xffffffffu, inside0 ? 1 : 0, j) != 0;
        const bool jin1 = __shfl_sync(0xffffffffu, inside1 ? 1 : 0, j) != 0;
        const uint32_t f0 = __shfl_sync(0xffffffffu, t0f, j), c0 = __shfl_sync(0xffffffffu, n0, j);
        const uint32_t f1 = __shfl_sync(0xffffffffu, t1f, j), c1 = __shfl_sync(0xffffffffu, n1, j);
        if (c0) warp_item<HIST>(S, V, hzbs, *ws, cell.slot, 0, occl_on, jin0, vmj, inst, f0, c0);
        if (c1) warp_item<HIST>(S, V, hzbs, *ws, cell.slot, 1, false, jin1, vmj, inst, f1, c1);
      }
    }
  }
}

// The instance pass of GeometryPool.ts:846-913, one warp per 64 instances of a visible (view, cell) unit (a
// half-unit), taken from a counter. Fast-path instances emit their meshlets; the others hand their level range to
// k_chunks as chunks of <= 2^chunk_shift meshlets. HIST: the budget search's pass (views with a triangleBudget only):
// the camera cut's level range over the whole threshold range, no fast path, no counters. Without the in-place test
// of a pass whose items do not fit the queue (k_instances_redo does that), the kernel keeps to 64 registers at 8
// blocks per SM.
template <bool HIST, bool MULTI>
__global__ void __launch_bounds__(128, MULTI ? 6 : 8) k_instances(Scene S0, const Scene *__restrict__ scenes,
                                                   const ViewConst *__restrict__ views,
                                                   const HzbDesc *__restrict__ hzbs0, const uint2 *__restrict__ units,
                                                   uint32_t *__restrict__ ctl, uint4 *__restrict__ queue,
                                                   uint32_t capacity, int round, uint32_t chunk_shift,
                                                   uint32_t *__restrict__ overflow) {
  __shared__ Survivor lists[4][kHalfUnit];
  if (round > 0 && ctl[round] == 0) return;  // no view redoes a cut in this round
  const uint32_t work = ctl[0] * 2;
  WarpFeed<1> feed;
  feed.start(ctl + kCtlNextUnit);
  for (uint32_t w = feed.i; w < work; w = feed.next()) {
    instance_unit<HIST, MULTI, false>(S0, scenes, views, hzbs0, units, ctl, queue, capacity, round, chunk_shift,
                                      overflow, nullptr, lists[threadIdx.x >> 5], w, 0);
    __syncwarp();  // the survivor list is rewritten by the next half-unit
  }
}

// The survivor passes k_instances found the chunk queue full for (bits of `overflow`: bit 2 w + p for pass p of
// half-unit w, cleared here), their items tested in place by the whole warp. Launched after each pass's k_chunks;
// returns at once when nothing overflowed.
template <bool HIST, bool MULTI>
__global__ void __launch_bounds__(128, 4) k_instances_redo(Scene S0, const Scene *__restrict__ scenes,
                                                            const ViewConst *__restrict__ views,
                                                            const HzbDesc *__restrict__ hzbs0,
                                                            const uint2 *__restrict__ units, uint32_t *__restrict__ ctl,
                                                            uint4 *__restrict__ queue, uint32_t capacity, int round,
                                                            uint32_t chunk_shift, uint32_t *__restrict__ overflow) {
  __shared__ WarpStage stage[4];
  __shared__ Survivor lists[4][kHalfUnit];
  if (round > 0 && ctl[round] == 0) return;
  if (ctl[kCtlOverflowed] == 0) return;
  const uint32_t words = (ctl[0] * 4 + 31) / 32;
  for (uint32_t i = warp_grab(ctl, kCtlNextRedo); i < words; i = warp_grab(ctl, kCtlNextRedo)) {
    uint32_t bits = overflow[i];
    __syncwarp();
    if ((threadIdx.x & 31) == 0 && bits) overflow[i] = 0;
    while (bits) {
      const uint32_t b = __ffs(bits) - 1;
      bits &= bits - 1;
      const uint32_t bit = i * 32 + b;
      instance_unit<HIST, MULTI, true>(S0, scenes, views, hzbs0, units, ctl, queue, capacity, round, chunk_shift,
                                       overflow, &stage[threadIdx.x >> 5], lists[threadIdx.x >> 5], bit >> 1, bit & 1u);
      __syncwarp();
    }
  }
}

// ------------------------------------------------------------------------------------------------ k_chunks
// The meshlet pass (GeometryPool.ts:916-970) over the chunks k_instances queued, one chunk per warp: the chunk's
// spans (instances of one cell) get their view-model matrices once, in parallel, into shared memory; then the lanes
// walk the chunk's meshlets end to end, 32 per step whatever span they belong to. The LOD band comes first; the
// meshlets that pass queue up and finish 32 at a time (drain_queue). One draw-list flush per chunk.
// HIST: the budget histogram of the chunks the budget pass queued.
template <bool HIST, bool MULTI>
__global__ void __launch_bounds__(128, MULTI ? 6 : 8) k_chunks(Scene S0, const Scene *__restrict__ scenes,
                                                            const ViewConst *__restrict__ views,
                                                            const HzbDesc *__restrict__ hzbs0,
                                                            uint4 *__restrict__ queue, uint32_t *__restrict__ ctl,
                                                            uint32_t capacity, int round) {
  __shared__ WarpStage stage[4];
  __shared__ LodQueue queues[4];
  __shared__ SpanFrame frames[4];
  WarpStage &ws = stage[threadIdx.x >> 5];
  LodQueue &q = queues[threadIdx.x >> 5];
  SpanFrame &F = frames[threadIdx.x >> 5];
  if (round > 0 && ctl[round] == 0) return;  // no view redoes a cut in this round
  const WorkQueue Q = work_queue(queue, capacity);
  const uint32_t n_chunks = min(uint32_t(*queue_counter(ctl) >> 32), Q.chunk_cap);
  const uint32_t lane = threadIdx.x & 31;
  WarpFeed<1> feed;
  feed.start(ctl + kCtlNextChunk);
  for (uint32_t c = feed.i; c < n_chunks; c = feed.next()) {
    const uint4 ch = Q.chunks[c];
    const uint32_t ns = ch.z >> 8;
    if (ns == 0) continue;
    const ViewConst &V = views[ch.x];
    const auto &S = SceneOf<MULTI>::get(S0, scenes, V);
    const HzbDesc *__restrict__ hzbs = SceneOf<MULTI>::hzbs(hzbs0, S);
    const CellRec cell = S.cells[ch.y];
    const uint32_t cut = ch.z & 1u;
    const bool occl_on = (ch.z & 2u) != 0;
    const ViewBands b = bands_of(V);
    const float low = cut ? b.low1 : b.low0, high = cut ? b.high1 : b.high0;
    const float inv_low = 1.0f / low;
    const float sc = HIST ? get_state(V.state, 0) : 0.0f;
    // spans: one lane each, laid end to end from position 0
    uint4 sp = make_uint4(0u, 0u, 0u, 0u);
    if (lane < ns) sp = Q.spans[ch.w + lane];
    const uint32_t sp_off = warp_scan_incl(sp.z) - sp.z;
    const uint32_t total = __shfl_sync(0xffffffffu, sp_off + sp.z, 31);
    if (lane < ns) {
      const uint32_t instance = cell.first + (sp.x & 127u);
      float VM[13];
      model_view(V.V, S.inst + (size_t)instance * 4, VM, VM[12]);
      F.vm[lane][0] = make_float4(VM[0], VM[1], VM[2], VM[3]);
      F.vm[lane][1] = make_float4(VM[4], VM[5], VM[6], VM[7]);
      F.vm[lane][2] = make_float4(VM[8], VM[9], VM[10], VM[11]);
      F.vm[lane][3] = make_float4(VM[12], __uint_as_float(instance), __uint_as_float((sp.x >> 7) & 1u),
                                  __uint_as_float(sp.y - sp_off));
    }
    __syncwarp();
    WarpCount wc{0, 0, 0};
    uint32_t qn = 0;       // warp-uniform
    uint32_t started = 0;  // warp-uniform: spans starting before this step's first position
    const uint32_t lanes_le = (2u << lane) - 1u;
    for (uint32_t base = 0; base < total; base += 32) {
      const uint32_t p = base + lane;
      // span of position p: the last span starting at or before it (spans are non-empty and in order, so each step
      // holds a bit per span starting in it)
      const uint32_t rel = sp_off - base;
      const uint32_t starts = __reduce_or_sync(0xffffffffu, lane < ns && rel < 32u ? 1u << rel : 0u);
      const uint32_t j = started + __popc(starts & lanes_le) - 1u;
      started += __popc(starts);
      bool pass = false;
      float own = 0.0f, parent = 0.0f;
      uint32_t m = 0;
      if (p < total) {
        float VM[13];
        uint32_t inst;
        bool inside;
        m = p + frame_vm(F, j, VM, inst, inside);
        const float4 ls = __ldg(S.m_lod + m), ps = __ldg(S.m_parent + m);
        const float2 er = __ldg(reinterpret_cast<const float2 *>(S.m_err + m));
        const ProjErr po = proj_parts(V, VM, VM[12], ls, er.x), pp = proj_parts(V, VM, VM[12], ps, er.y);
        if (HIST) {
          const uint32_t bo = budget_bin_high(V, sc, po, er.x), bp = budget_bin(V, sc, pp, er.y);
          pass = bo < bp;
          own = __uint_as_float(bo);
          parent = __uint_as_float(bp);
        } else {
          pass = err_le(po, er.x, high) && err_gt(pp, er.y, low);
          own = po.dist;
          parent = pp.dist;
        }
      }
      const uint32_t mask = __ballot_sync(0xffffffffu, pass);
      if (pass) {
        const uint32_t at = qn + __popc(mask & ((1u << lane) - 1u));
        q.pos[at] = m;
        q.span[at] = j;
        q.own[at] = own;
        q.parent[at] = parent;
      }
      qn += __popc(mask);
      __syncwarp();
      if (qn >= 32) {
        drain_queue<HIST>(S, V, hzbs, q, F, 32, ws, wc, inv_low, b.fade_scale, b.high0, cut, occl_on, cell.slot);
        qn -= 32;
        __syncwarp();
        if (lane < qn) {
          q.pos[lane] = q.pos[32 + lane];
          q.span[lane] = q.span[32 + lane];
          q.own[lane] = q.own[32 + lane];
          q.parent[lane] = q.parent[32 + lane];
        }
        __syncwarp();
      }
    }
    if (qn) drain_queue<HIST>(S, V, hzbs, q, F, qn, ws, wc, inv_low, b.fade_scale, b.high0, cut, occl_on, cell.slot);
    __syncwarp();
    if (!HIST) warp_flush(ws, wc, V, S.slot_capacity, cell.slot, cut);
    __syncwarp();  // the frame and queue are rewritten by the next chunk
  }
}

// ------------------------------------------------------------------------------------------------ k_budget
// One warp per view with a triangleBudget: T(t_k) = prefix sum of (entering - leaving) triangles; the smallest k with
// T(t_k) <= budget (255 when none) sets this frame's errorThreshold and bands. Also empties the chunk queue for the
// frame's first selection round.
__global__ void __launch_bounds__(128) k_budget(const ViewConst *__restrict__ views, uint32_t nviews,
                                                uint32_t *__restrict__ ctl) {
  if (blockIdx.x == 0 && threadIdx.x == 0) retire_queue(ctl);
  const uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (v >= nviews) return;
  const ViewConst &V = views[v];
  if (!(V.budget > 0.0f)) return;
  long long carry = 0;
  uint32_t pick = kBudgetBins - 1;
  long long predicted = 0;
  bool found = false;
  for (uint32_t base = 0; base < kBudgetBins && !found; base += 32) {
    const uint32_t k = base + lane;
    long long d = (long long)V.hist[k] - (long long)V.hist[kBudgetBins + k];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, d, o);
      if (lane >= (uint32_t)o) d += t;
    }
    const long long T = carry + d;
    const uint32_t ok = __ballot_sync(0xffffffffu, T <= (long long)V.budget_tris);
    if (ok) {
      const uint32_t j = __ffs(ok) - 1;
      pick = base + j;
      predicted = __shfl_sync(0xffffffffu, T, j);
      found = true;
    }
    carry += __shfl_sync(0xffffffffu, d, 31);
  }
  if (!found) predicted = carry;
  if (lane == 0) {
    const float t = V.budget_lo + (V.budget_hi - V.budget_lo) * (float(pick) / 255.0f);
    store_bands(V, t);
    V.counters[VGC_COUNTER_PREDICTED_LO] = (uint32_t)((unsigned long long)predicted & 0xffffffffull);
    V.counters[VGC_COUNTER_PREDICTED_HI] = (uint32_t)((unsigned long long)predicted >> 32);
    V.counters[VGC_COUNTER_BUDGET_BIN] = pick;
  }
}

// ------------------------------------------------------------------------------------------------ k_finish
__device__ __forceinline__ float fill_of(const ViewConst &V, uint32_t cut) {
  const float requested = float(V.counters[C_CUT(cut) + VGC_CUT_REQUESTED]);
  const float selected = float(V.counters[C_CUT(cut) + VGC_CUT_SELECTED]);
  return fmx(requested / float(V.index_capacity[cut]), selected / float(V.max_drawn));
}

__global__ void __launch_bounds__(128) k_finish(const ViewConst *__restrict__ views, uint32_t nviews,
                                                uint32_t *__restrict__ ctl, int round) {
  const uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (blockIdx.x == 0 && threadIdx.x == 0) retire_queue(ctl);  // the next round's work queue starts empty
  if (v >= nviews) return;
  const ViewConst &V = views[v];
  const uint32_t slot_capacity = V.slot_capacity, slots_used = V.slots_used;
  uint32_t *ctr = V.counters;
  const bool redo[2] = {round == 0 || ctr[VGC_COUNTER_REDO0] != 0, round == 0 || ctr[VGC_COUNTER_REDO1] != 0};
  // prefix (GeometryPool.ts:973-995)
  for (uint32_t cut = 0; cut < 2; cut++) {
    if (!redo[cut]) continue;
    const uint32_t capacity = V.index_capacity[cut];
    uint32_t carry = 0;
    for (uint32_t b = 0; b < slots_used; b += 32) {
      const uint32_t slot = b + lane;
      uint32_t r0 = 0, r1 = 0;
      if (slot < slots_used) {
        r0 = mesh_count(V, slot_capacity, cut, slot, 0)[0];
        r1 = mesh_count(V, slot_capacity, cut, slot, 1)[0];
      }
      const uint32_t sum = r0 + r1;
      uint32_t incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
      }
      if (slot < slots_used) {
        const uint32_t starts[2] = {carry + (incl - sum), carry + (incl - sum) + r0};
        const uint32_t req[2] = {r0, r1};
        for (uint32_t p = 0; p < 2; p++) {
          mesh_count(V, slot_capacity, cut, slot, p)[1] = starts[p];
          const uint32_t room = starts[p] < capacity ? capacity - starts[p] : 0u;
          uint32_t *a = V.draw_args + ((cut * slot_capacity + slot) * 2 + p) * 5;
          a[0] = min(req[p], room);
          a[1] = 1;
          a[2] = starts[p];
          a[3] = 0;
          a[4] = 0;
        }
      }
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) {
      ctr[C_CUT(cut) + VGC_CUT_REQUESTED] = carry;
      ctr[C_CUT(cut) + VGC_CUT_DRAWN] = min(ctr[C_CUT(cut) + VGC_CUT_SELECTED], V.max_drawn);
    }
  }
  __syncwarp();
  if (round < 2) {
    // capacity check: an overflowing cut is redone at a coarser threshold (GeometryPool.ts:1032-1054)
    uint32_t again = 0;
    if (lane == 0) {
      for (uint32_t cut = 0; cut < 2; cut++) {
        const float fill = fill_of(V, cut);
        const float scale = get_state(V.state, cut);
        V.state[4 + cut] = 0;
        if (fill > 1.0f && scale < V.lod_scale_limit) {
          const float q = fmn(fmx(sqrtf(fill / float(0.82)), float(1.1)), 4.0f);
          V.state[cut] = to_state(fmn(scale * q, V.lod_scale_limit));
          V.state[4 + cut] = 10000u;
          again |= 1u << cut;
          for (int c = 0; c < 5; c++) ctr[C_CUT(cut) + c] = 0;
          if (cut == 0) ctr[VGC_COUNTER_OCCLUDED] = 0;
        }
        ctr[VGC_COUNTER_REDO0 + cut] = (again >> cut) & 1u;
      }
      if (again) store_bands(V, V.dyn[0]);  // the redone round selects with the new scale
      if (again) {
        ctr[VGC_COUNTER_ROUNDS] += 1;
        atomicOr(&ctl[1 + round], 1u);
      }
    }
    again = __shfl_sync(0xffffffffu, again, 0);
    for (uint32_t cut = 0; cut < 2; cut++)
      if ((again >> cut) & 1u)
        for (uint32_t slot = lane; slot < slots_used; slot += 32) {
          mesh_count(V, slot_capacity, cut, slot, 0)[0] = 0;
          mesh_count(V, slot_capacity, cut, slot, 1)[0] = 0;
        }
  } else if (lane == 0) {
    // steer between frames (GeometryPool.ts:1056-1069)
    for (uint32_t cut = 0; cut < 2; cut++) {
      const float fill = fill_of(V, cut);
      float scale = get_state(V.state, cut);
      if (fill > float(0.9)) {
        scale = scale * fmn(sqrtf(fill / float(0.82)), float(1.03));
      } else if (fill < float(0.75)) {
        scale = scale / float(1.01);
      }
      V.state[cut] = to_state(fmx(fmn(scale, V.lod_scale_limit), 1.0f));
      V.state[2 + cut] = to_state(fill);
    }
    ctr[VGC_COUNTER_ROUNDS] += 1;
  }
}

// ------------------------------------------------------------------------------------------------ k_expand
__global__ void __launch_bounds__(256) k_expand(Scene S, const ViewConst *__restrict__ view, uint32_t cut,
                                                uint32_t *__restrict__ out, uint64_t capacity) {
  const ViewConst &V = *view;
  const uint32_t n = min(V.counters[C_CUT(cut) + VGC_CUT_SELECTED], V.max_drawn);
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < n; e += warps) {
    const uint32_t draw_slot = e + cut * V.max_drawn;
    const uint4 d = V.draw_list[draw_slot];
    const uint32_t slot = S.inst_slot[d.x];
    const uint32_t region = mesh_count(V, S.slot_capacity, cut, slot, part_of(d.w))[1];
    const uint32_t first_tri = S.m_info[d.y].y / 3;
    const uint32_t base = draw_slot << kLocalVertexBits;
    const uint32_t tris = d.w & 255u;
    for (uint32_t i = lane; i < tris; i += 32) {
      const uint64_t index = (uint64_t)region + d.z + i * 3;
      if (index + 2 < capacity) {
        const uint32_t p = S.m_tris[first_tri + i];
        out[index] = base | (p & 255u);
        out[index + 1] = base | ((p >> 8) & 255u);
        out[index + 2] = base | ((p >> 16) & 255u);
      }
    }
  }
}

// ------------------------------------------------------------------------------------------------ HZB
// Max-reduced mip chain (OcclusionCulling.ts:320-350): mip i texel (x, y) = max of mip i-1 texels (2x, 2y),
// (min(2x+1, w-1), 2y), (2x, min(2y+1, h-1)), (min(2x+1, w-1), min(2y+1, h-1)), sizes halved rounding up. By
// induction every texel of mip i is the max over its mip-0 footprint [2^i x, 2^i (x+1)) x [2^i y, 2^i (y+1)) inside
// the image, so a reduction whose loads clamp to the image edge gives the same values.
//
// One 64x64 tile of mip 0 per block of 256 threads: each thread reduces a 4x4 patch (float4 rows when the image
// allows) to its 2x2 texels of mip 1 and its texel of mip 2 in registers; mips 3..6 of the tile come from shared
// memory (tiles are aligned to 64, so every clamped neighbour lies inside the tile); mips 7+ by the tail kernel.
constexpr uint32_t kHzbTile = 64, kHzbTileLevels = 7;

__device__ __forceinline__ void hzb_store(const HzbDesc &H, float *__restrict__ out, uint32_t l, uint32_t x, uint32_t y,
                                          float v) {
  if (l < H.levels && x < H.w[l] && y < H.h[l]) out[H.off[l] + (size_t)y * H.w[l] + x] = v;
}

// Levels 3..6 of the tile use no clamped reads: a texel's neighbour past the level's edge holds the max over the
// edge texels of the same rows (or columns), which the in-range texel's footprint already contains, so the max over
// the 2x2 block equals the max over its clamped reads. Level 3 is warp-local (a warp holds two rows of level 2); one
// barrier hands the tile's 8x8 level-3 texels to warp 0 for levels 4..6.
// This thread's 4x4 patch of mip 0 of the tile at (ox, oy) (loads clamped to the image).
__device__ __forceinline__ void hzb_load(const float *__restrict__ depth, const HzbDesc &H, uint32_t ox, uint32_t oy,
                                         float v[4][4]) {
  const uint32_t t = threadIdx.x, tx = t & 15u, ty = t >> 4;
  const uint32_t W = H.w[0], Hh = H.h[0];
  const uint32_t gx = ox + 4 * tx, gy = oy + 4 * ty;
  const bool vec = (W & 3u) == 0 && (reinterpret_cast<uintptr_t>(depth) & 15u) == 0 && gx + 3 < W;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const uint32_t y = min(gy + r, Hh - 1);
    const float *row = depth + (size_t)y * W;
    if (vec) {
      const float4 q = __ldg(reinterpret_cast<const float4 *>(row + gx));
      v[r][0] = q.x, v[r][1] = q.y, v[r][2] = q.z, v[r][3] = q.w;
    } else {
#pragma unroll
      for (int c = 0; c < 4; c++) v[r][c] = __ldg(row + min(gx + c, W - 1));
    }
  }
}

// Mips 0..6 of the tile at (ox, oy) from the patches hzb_load read (every thread of the block calls it).
__device__ __forceinline__ void hzb_tile64(const float *__restrict__ depth, const HzbDesc &H, float *__restrict__ out,
                                           bool copy_mip0, uint32_t ox, uint32_t oy, float (*s3)[9],
                                           const float (&v)[4][4]) {
  const uint32_t t = threadIdx.x, tx = t & 15u, ty = t >> 4, lane = t & 31u, warp = t >> 5;
  const uint32_t W = H.w[0], Hh = H.h[0];
  const uint32_t gx = ox + 4 * tx, gy = oy + 4 * ty;
  const bool vec = (W & 3u) == 0 && (reinterpret_cast<uintptr_t>(depth) & 15u) == 0 && gx + 3 < W;
  if (copy_mip0) {
    float *o0 = out + H.off[0];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      if (gy + r >= Hh) continue;
      float *row = o0 + (size_t)(gy + r) * W;
      if (vec && (reinterpret_cast<uintptr_t>(o0) & 15u) == 0) {
        *reinterpret_cast<float4 *>(row + gx) = make_float4(v[r][0], v[r][1], v[r][2], v[r][3]);
      } else {
#pragma unroll
        for (int c = 0; c < 4; c++)
          if (gx + c < W) row[gx + c] = v[r][c];
      }
    }
  }
  float a[2][2];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++)
      a[i][j] = fmaxf(fmaxf(v[2 * i][2 * j], v[2 * i][2 * j + 1]), fmaxf(v[2 * i + 1][2 * j], v[2 * i + 1][2 * j + 1]));
  if (H.levels > 1) {
    float *o1 = out + H.off[1];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const uint32_t x = gx / 2 + j, y = gy / 2 + i;
        if (x < H.w[1] && y < H.h[1]) o1[(size_t)y * H.w[1] + x] = a[i][j];
      }
  }
  const float b = fmaxf(fmaxf(a[0][0], a[0][1]), fmaxf(a[1][0], a[1][1]));
  hzb_store(H, out, 2, gx / 4, gy / 4, b);
  // level 3: texel (tx / 2, warp) of the tile from lanes tx, tx ^ 1 of rows 2 warp, 2 warp + 1
  float m = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, 1));
  m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 16));
  if ((lane & 17u) == 0) {
    hzb_store(H, out, 3, (ox >> 3) + (tx >> 1), (oy >> 3) + warp, m);
    s3[warp][tx >> 1] = m;
  }
  __syncthreads();
  if (warp != 0 || H.levels <= 4) return;
  // levels 4..6 by warp 0: lane = 4 y + x of level 4 (16 lanes), then xor 1 / 4 and xor 2 / 8 pair up the blocks
  const uint32_t x4 = lane & 3u, y4 = (lane >> 2) & 3u;
  float m4 = fmaxf(fmaxf(s3[2 * y4][2 * x4], s3[2 * y4][2 * x4 + 1]), fmaxf(s3[2 * y4 + 1][2 * x4], s3[2 * y4 + 1][2 * x4 + 1]));
  if (lane < 16) hzb_store(H, out, 4, (ox >> 4) + x4, (oy >> 4) + y4, m4);
  float m5 = fmaxf(m4, __shfl_xor_sync(0xffffffffu, m4, 1));
  m5 = fmaxf(m5, __shfl_xor_sync(0xffffffffu, m5, 4));
  if (lane < 16 && (lane & 5u) == 0) hzb_store(H, out, 5, (ox >> 5) + (x4 >> 1), (oy >> 5) + (y4 >> 1), m5);
  float m6 = fmaxf(m5, __shfl_xor_sync(0xffffffffu, m5, 2));
  m6 = fmaxf(m6, __shfl_xor_sync(0xffffffffu, m6, 8));
  if (lane == 0) hzb_store(H, out, 6, ox >> 6, oy >> 6, m6);
}

// Two vertically adjacent tiles per block: both tiles' loads are in flight before the first tile is reduced.
__device__ __forceinline__ void hzb_tile_pair(const float *__restrict__ depth, const HzbDesc &H, float *__restrict__ out,
                                              bool copy_mip0, uint32_t ox, uint32_t oy, float (*s3)[9]) {
  const bool second = oy + kHzbTile < H.h[0];  // uniform over the block
  float a[4][4], b[4][4];
  hzb_load(depth, H, ox, oy, a);
  if (second) hzb_load(depth, H, ox, oy + kHzbTile, b);
  hzb_tile64(depth, H, out, copy_mip0, ox, oy, s3, a);
  if (second) {
    __syncthreads();  // warp 0 has read the first tile's level 3 from s3
    hzb_tile64(depth, H, out, copy_mip0, ox, oy + kHzbTile, s3, b);
  }
}

__global__ void __launch_bounds__(256) k_hzb_tiles(const float *__restrict__ depth, HzbDesc H, float *__restrict__ out,
                                                   int copy_mip0) {
  __shared__ float s3[8][9];
  hzb_tile_pair(depth, H, out, copy_mip0 != 0, blockIdx.x * kHzbTile, blockIdx.y * 2 * kHzbTile, s3);
}

// The HZB builds of a batch: grid.z = view, views without a depth image skip.
__global__ void __launch_bounds__(256) k_hzb_tiles_views(const ViewConst *__restrict__ views) {
  __shared__ float s3[8][9];
  const ViewConst &V = views[blockIdx.z];
  if (!V.build_hzb) return;
  const HzbDesc &H = *V.hzb_desc;
  const uint32_t ox = blockIdx.x * kHzbTile, oy = blockIdx.y * 2 * kHzbTile;
  if (ox >= H.w[0] || oy >= H.h[0]) return;
  hzb_tile_pair(V.depth, H, const_cast<float *>(H.data), V.hzb_mip0 == nullptr, ox, oy, s3);
}

// Levels `first` and up of each building view's HZB, one block per view (the tile kernels wrote the levels below).
__global__ void __launch_bounds__(1024) k_hzb_tail_views(const ViewConst *__restrict__ views, uint32_t first) {
  const ViewConst &V = views[blockIdx.x];
  if (!V.build_hzb) return;
  const HzbDesc &H = *V.hzb_desc;
  float *out = const_cast<float *>(H.data);
  for (uint32_t l = first; l < H.levels; l++) {
    const float *src = out + H.off[l - 1];
    const uint32_t sw = H.w[l - 1], sh = H.h[l - 1];
    for (uint32_t i = threadIdx.x; i < H.w[l] * H.h[l]; i += blockDim.x) {
      const uint32_t x = i % H.w[l], y = i / H.w[l];
      const uint32_t x0 = 2 * x, y0 = 2 * y, x1 = min(x0 + 1, sw - 1), y1 = min(y0 + 1, sh - 1);
      const float a = fmaxf(src[y0 * sw + x0], src[y0 * sw + x1]);
      const float b = fmaxf(src[y1 * sw + x0], src[y1 * sw + x1]);
      out[H.off[l] + i] = fmaxf(a, b);
    }
    __syncthreads();
  }
}

// Levels 7 and up (at most 15 x 9 texels for a 1080p mip 0) by one block.
__global__ void __launch_bounds__(1024) k_hzb_tail(HzbDesc H, float *__restrict__ out) {
  for (uint32_t l = kHzbTileLevels; l < H.levels; l++) {
    const float *src = out + H.off[l - 1];
    const uint32_t sw = H.w[l - 1], sh = H.h[l - 1];
    for (uint32_t i = threadIdx.x; i < H.w[l] * H.h[l]; i += blockDim.x) {
      const uint32_t x = i % H.w[l], y = i / H.w[l];
      const uint32_t x0 = 2 * x, y0 = 2 * y, x1 = min(x0 + 1, sw - 1), y1 = min(y0 + 1, sh - 1);
      const float a = fmaxf(src[y0 * sw + x0], src[y0 * sw + x1]);
      const float b = fmaxf(src[y1 * sw + x0], src[y1 * sw + x1]);
      out[H.off[l] + i] = fmaxf(a, b);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------ HZB strip stream
// The HZB builds of a launch sequence as one persistent pass over 128 x 32 strips of mip 0 of all its jobs (the
// views that bring a depth image; HzbPlanHead / HzbJob), levels 1..4; levels 5 and up by k_hzb_tail_views. Block b
// takes the contiguous strips [b T / grid, (b + 1) T / grid) of the stream's T strips.
//
// Warp 8 streams the strips in: lane 0 waits until the consumers released a stage (an `empty` mbarrier, one arrival
// per consumer warp), looks up the strip's job and issues a 2D bulk-tensor copy (TMA) of the strip from the depth
// image into the block's own stage, completing on the stage's `full` mbarrier; kHzbStages strips are in flight. The TMA unit fills texels past the image's edge with zeros; the consumers' reads clamp to the image, so the
// values are those of clamped loads. A job whose image no tensor map describes (width not a multiple of 4, pointer not
// 16-byte aligned, or smaller than a strip) has its strips loaded by the consumers themselves, in the same pass.
//
// Warps 0..7 reduce: warp w takes the 32 x 16 pixels at column 32 (w & 3), row 16 (w >> 2) of the strip, lane l the
// 4 x 4 patch at (4 (l & 7), 4 (l >> 3)) of those; levels 1 and 2 of the patch in registers, level 3 (2 x 2 patches:
// lanes l ^ 1, l ^ 8) and level 4 (4 x 4 patches: lanes l ^ 2, l ^ 16) by shuffles, so no warp waits for another.
// Every wait gives up after about a second (or when another warp gave up): the block then sets VGC_FAULT_HZB_WAIT in
// every job's view and leaves, the streaming lane after its copies still in flight have landed.
#ifndef VGC_HZB_STAGES
#define VGC_HZB_STAGES 4  // strips in flight per block
#endif
#ifndef VGC_HZB_BLOCKS_PER_SM
#define VGC_HZB_BLOCKS_PER_SM 3
#endif
constexpr uint32_t kHzbStages = VGC_HZB_STAGES;
constexpr uint32_t kStripW = kHzbStripW, kStripH = kHzbStripH, kStripFloats = kStripW * kStripH;
constexpr uint32_t kStripBytes = kStripFloats * 4;
constexpr uint32_t kHzbStripLevels = 5;  // levels 1..4 per strip; k_hzb_tail_views from level 5
constexpr size_t kHzbStreamSmem = (size_t)kHzbStages * kStripBytes + 128;  // + slack to align the stages to 128
constexpr uint64_t kWaitLimitNs = 1000000000ull;
constexpr uint32_t kHzbConsumerWarps = 8, kHzbStreamThreads = 32 * (kHzbConsumerWarps + 1);
static_assert(kStripW == 128 && kStripH == 32, "the consumer layout covers 128 x 32 strips with 8 warps");

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Phase `parity` of `bar` completed: false once `limit_ns` (or 2^30 polls) passed without it, or once `*abort`
// (when given) is set.
__device__ __noinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile uint32_t *abort,
                                       uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t i = 0; i < (1u << 30); i++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63u) == 0 && (global_ns() - t0 > limit_ns || (abort && *abort))) return false;
  }
  return false;
}

// mbar_wait on a barrier that nothing arrives at: out[0] = 1 if it completed (never), out[1] = nanoseconds waited.
__global__ void k_wait_probe(uint64_t limit_ns, unsigned long long *out) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint64_t t0 = global_ns();
    const bool done = mbar_wait(&bar, 0, nullptr, limit_ns);
    out[1] = global_ns() - t0;
    out[0] = done ? 1ull : 0ull;
  }
}

// The tensor map was written to global memory by a copy before this launch: order that write before its use by
// the tensor-map proxy.
__device__ __forceinline__ void tensormap_acquire(const void *map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

// The strip (128 x 32 floats) at element (x, y) of the map's image into `dst`, completing on `bar`. x is a multiple
// of 128 (512 bytes), so the copy starts on a 16-byte boundary.
__device__ __forceinline__ void tma_strip(float *dst, const void *map, uint32_t x, uint32_t y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// Sizes and offsets of levels 0..4 of a job's HZB slot, held in registers while a warp works on the job.
struct StripDesc {
  float *out;
  uint32_t levels;
  uint32_t off[5], w[5], h[5];
};

__device__ __forceinline__ void strip_desc(const HzbDesc &H, StripDesc &D) {
  D.out = const_cast<float *>(H.data);
  D.levels = H.levels;
#pragma unroll
  for (int l = 0; l < 5; l++) D.off[l] = H.off[l], D.w[l] = H.w[l], D.h[l] = H.h[l];
}

__device__ __forceinline__ void strip_store(const StripDesc &D, uint32_t l, uint32_t x, uint32_t y, float v) {
  if (l < D.levels && x < D.w[l] && y < D.h[l]) D.out[D.off[l] + (size_t)y * D.w[l] + x] = v;
}

__global__ void __launch_bounds__(kHzbStreamThreads, VGC_HZB_BLOCKS_PER_SM) k_hzb_stream(
    const unsigned char *__restrict__ plan) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  // kHzbStages strips from the first 128-byte boundary of the dynamic shared memory (a bulk-tensor destination)
  float *stage = reinterpret_cast<float *>(dyn_smem + ((128u - (smem_addr(dyn_smem) & 127u)) & 127u));
  __shared__ __align__(8) uint64_t full[kHzbStages], empty[kHzbStages];
  __shared__ uint4 meta[kHzbStages];  // job, ox, oy, tma of the strip in each stage
  __shared__ uint32_t abort;
  const HzbPlanHead &P = *reinterpret_cast<const HzbPlanHead *>(plan);
  const HzbJob *jobs = reinterpret_cast<const HzbJob *>(plan + sizeof(HzbPlanHead));
  const uint32_t njobs = P.jobs;
  const uint32_t first = (uint32_t)((uint64_t)P.tiles * blockIdx.x / gridDim.x);
  const uint32_t last = (uint32_t)((uint64_t)P.tiles * (blockIdx.x + 1) / gridDim.x);
  if (first >= last) return;
  const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31u;
  if (t == 0) {
    for (uint32_t s = 0; s < kHzbStages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kHzbConsumerWarps);
    }
    abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  volatile uint32_t *flag = &abort;
  auto give_up = [&] {  // a wait gave up: stop the other warps and report it in every job's view
    *flag = 1;
    for (uint32_t j = 0; j < njobs; j++)
      if (jobs[j].error) atomicOr(jobs[j].error, (uint32_t)VGC_FAULT_HZB_WAIT);
  };
  if (warp == kHzbConsumerWarps) {  // the streaming warp: lane 0 issues every copy of the block
    if (lane != 0) return;
    const unsigned char *maps = plan + P.maps;
    uint32_t acquired = ~0u, k = 0;
    for (;; k++) {
      const uint32_t item = first + k;
      if (item >= last) return;  // the consumers wait for the copies issued so far
      const uint32_t s = k % kHzbStages;
      if (k >= kHzbStages && !mbar_wait(&empty[s], (k / kHzbStages - 1) & 1u, flag)) break;
      uint32_t lo = 0, hi = njobs;  // the last job whose first strip is <= item
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (jobs[mid].tile0 <= item) lo = mid;
        else hi = mid;
      }
      const uint32_t r = item - jobs[lo].tile0, sx = jobs[lo].tiles_x, tma = jobs[lo].tma;
      const uint32_t ox = (r % sx) * kStripW, oy = (r / sx) * kStripH;
      meta[s] = make_uint4(lo, ox, oy, tma);
      if (tma) {
        const void *map = maps + (size_t)lo * kTensorMapBytes;
        if (lo != acquired) {
          tensormap_acquire(map);
          acquired = lo;
        }
        mbar_arrive_tx(&full[s], kStripBytes);
        tma_strip(stage + s * kStripFloats, map, ox, oy, &full[s]);
      } else {
        mbar_arrive(&full[s]);  // the consumers load this strip themselves
      }
    }
    give_up();  // then let the copies in flight land before this lane exits
    for (uint32_t q = k > kHzbStages ? k - kHzbStages : 0; q < k; q++)
      mbar_wait(&full[q % kHzbStages], (q / kHzbStages) & 1u, nullptr);
    return;
  }
  const uint32_t px = 32u * (warp & 3u) + 4u * (lane & 7u), py = 16u * (warp >> 2) + 4u * (lane >> 3);  // in the strip
  StripDesc D;
  uint32_t job = ~0u, W = 0, Hh = 0;
  bool copy_mip0 = false;
  const float *depth = nullptr;
  for (uint32_t k = 0;; k++) {
    if (first + k >= last) return;  // every strip of this block reduced
    const uint32_t s = k % kHzbStages;
    if (!__all_sync(0xffffffffu, mbar_wait(&full[s], (k / kHzbStages) & 1u, flag))) {
      if (lane == 0) give_up();
      return;
    }
    const uint4 m = meta[s];
    if (m.x != job) {
      job = m.x;
      const HzbJob &J = jobs[job];
      strip_desc(*J.desc, D);
      W = D.w[0], Hh = D.h[0], copy_mip0 = J.copy_mip0 != 0, depth = J.depth;
    }
    const uint32_t gx = m.y + px, gy = m.z + py;  // this lane's patch in the image
    float v[4][4];
    const bool inside = m.y + kStripW <= W && m.z + kStripH <= Hh;
    if (m.w) {
      const float *st = stage + s * kStripFloats;
      if (inside) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const float4 q = *reinterpret_cast<const float4 *>(st + (py + r) * kStripW + px);
          v[r][0] = q.x, v[r][1] = q.y, v[r][2] = q.z, v[r][3] = q.w;
        }
      } else {  // clamped to the image (every index stays inside the strip: m.y < W, m.z < Hh)
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const uint32_t y = min(gy + r, Hh - 1) - m.z;
#pragma unroll
          for (int c = 0; c < 4; c++) v[r][c] = st[y * kStripW + (min(gx + c, W - 1) - m.y)];
        }
      }
    } else {
      const bool vec = (W & 3u) == 0 && (reinterpret_cast<uintptr_t>(depth) & 15u) == 0 && gx + 3 < W;
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const float *row = depth + (size_t)min(gy + r, Hh - 1) * W;
        if (vec) {
          const float4 q = __ldg(reinterpret_cast<const float4 *>(row + gx));
          v[r][0] = q.x, v[r][1] = q.y, v[r][2] = q.z, v[r][3] = q.w;
        } else {
#pragma unroll
          for (int c = 0; c < 4; c++) v[r][c] = __ldg(row + min(gx + c, W - 1));
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with stage s
    if (copy_mip0) {
      float *o0 = D.out + D.off[0];
      const bool vec = (W & 3u) == 0 && (reinterpret_cast<uintptr_t>(o0) & 15u) == 0 && gx + 3 < W;
#pragma unroll
      for (int r = 0; r < 4; r++) {
        if (gy + r >= Hh) continue;
        float *row = o0 + (size_t)(gy + r) * W;
        if (vec) {
          *reinterpret_cast<float4 *>(row + gx) = make_float4(v[r][0], v[r][1], v[r][2], v[r][3]);
        } else {
#pragma unroll
          for (int c = 0; c < 4; c++)
            if (gx + c < W) row[gx + c] = v[r][c];
        }
      }
    }
    float a[2][2];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 2; j++) {
        a[i][j] = fmaxf(fmaxf(v[2 * i][2 * j], v[2 * i][2 * j + 1]), fmaxf(v[2 * i + 1][2 * j], v[2 * i + 1][2 * j + 1]));
        strip_store(D, 1, gx / 2 + j, gy / 2 + i, a[i][j]);
      }
    const float b = fmaxf(fmaxf(a[0][0], a[0][1]), fmaxf(a[1][0], a[1][1]));
    strip_store(D, 2, gx / 4, gy / 4, b);
    float m3 = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, 1));
    m3 = fmaxf(m3, __shfl_xor_sync(0xffffffffu, m3, 8));
    if ((lane & 9u) == 0) strip_store(D, 3, gx / 8, gy / 8, m3);
    float m4 = fmaxf(m3, __shfl_xor_sync(0xffffffffu, m3, 2));
    m4 = fmaxf(m4, __shfl_xor_sync(0xffffffffu, m4, 16));
    if ((lane & 27u) == 0) strip_store(D, 4, gx / 16, gy / 16, m4);
    if (*flag) return;  // another warp gave up
  }
}

// ------------------------------------------------------------------------------------------------ selectCut
// cut.ts:26-77 on the GPU: one thread per (view-model matrix, meshlet) of one mesh. Float arithmetic in the
// kernels' order; lodFadeRange rounds halves up like JavaScript's Math.round.
__global__ void __launch_bounds__(256) k_select_cut(Scene S, uint32_t slot, uint32_t mcount, uint32_t count,
                                                    const float *__restrict__ vm16,
                                                    const float *__restrict__ params, float threshold, float blend,
                                                    uint8_t *__restrict__ lo, uint8_t *__restrict__ hi) {
  const uint32_t base = S.meshes[slot].meshlet_base;
  const uint64_t total = (uint64_t)count * mcount;
  const float high = blend > 1.0f ? threshold * blend : threshold;
  const float fscale = blend > 1.0f ? 255.0f / vg_logf(blend) : 0.0f;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = uint32_t(i / mcount), m = uint32_t(i % mcount), g = base + m;
    const float *e = vm16 + (size_t)v * 16;
    float VM[12];
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 4; c++) VM[r * 4 + c] = e[c * 4 + r];
    const float ps = params[v * 3], nr = params[v * 3 + 1], sc = params[v * 3 + 2];
    const float4 ls = S.m_lod[g], pp = S.m_parent[g], er = S.m_err[g];
    auto project = [&](float4 s, float err) {
      float c[3];
      xform(VM, s.x, s.y, s.z, c);
      const float dist = fmx(__fmaf_rn(-s.w, sc, len3(c)), nr);
      return ((err * sc) / dist) * ps;
    };
    const bool own_inf = er.x >= float(1e30 * 0.5), parent_inf = er.y >= float(1e30 * 0.5);
    const float own = own_inf ? 1e30f : project(ls, er.x);
    const float parent = parent_inf ? 1e30f : project(pp, er.y);
    uint8_t l = 0, h = 0;
    if (own <= high && parent > threshold) {
      if (!(blend > 1.0f)) {
        h = 255;
      } else {
        const float fl = floorf(vg_logf(fmx(own, float(1e-30)) / threshold) * fscale + 0.5f);
        const uint32_t sl = uint32_t(fmn(255.0f, fmx(0.0f, fl)));
        uint32_t sh = 255u;
        if (!parent_inf) {
          const float fh = floorf(vg_logf(fmx(parent, float(1e-30)) / threshold) * fscale + 0.5f);
          sh = uint32_t(fmn(255.0f, fmx(0.0f, fh)));
        }
        if (sh > sl) {
          l = uint8_t(sl);
          h = uint8_t(sh);
        }
      }
    }
    const size_t out = (size_t)v * mcount + (__float_as_uint(er.w) - base);  // the caller's meshlet order
    lo[out] = l;
    hi[out] = h;
  }
}

// ------------------------------------------------------------------------------------------------ k_reset
// Zeroes each view's counter block (reset pass, GeometryPool.ts:714-725) and the batch's unit count; reads the
// output pointers from the view constants, so a captured graph serves any output slots.
__global__ void __launch_bounds__(256) k_reset(const ViewConst *__restrict__ views, uint32_t nviews,
                                               uint32_t *__restrict__ ctl) {
  if (blockIdx.x == 0 && threadIdx.x < 16) ctl[threadIdx.x] = 0;
  for (uint32_t v = blockIdx.x; v < nviews; v += gridDim.x) {
    uint32_t *c = views[v].counters;
    const uint32_t words = views[v].counter_words;
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) c[i] = 0;
    if (threadIdx.x == 0) {
      if (views[v].fresh_state) {  // initial controller state: scales 1.0 (fixed point x10000), no fill, no retry
        uint32_t *st = views[v].state;
        for (uint32_t i = 0; i < kStateWords; i++) st[i] = i < 2 ? 10000u : 0u;
      }
      // budget views: the search's pass uses the band at the top of the threshold range
      store_bands(views[v], views[v].budget > 0.0f ? views[v].budget_hi : views[v].error_threshold);
    }
    if (views[v].budget > 0.0f)
      for (uint32_t i = threadIdx.x; i < 2 * kBudgetBins; i += blockDim.x) views[v].hist[i] = 0;
  }
}

// Each view's counter header and the threshold its cut used, 32 words per view, for one device-to-host copy.
__global__ void __launch_bounds__(32) k_gather_stats(const ViewConst *__restrict__ views, uint32_t nviews,
                                                     uint32_t *__restrict__ out) {
  const uint32_t v = blockIdx.x, t = threadIdx.x;
  if (v >= nviews) return;
  uint32_t w = 0;
  if (t < VGC_COUNTER_HEADER) w = views[v].counters[t];
  else if (t == VGC_COUNTER_HEADER) w = __float_as_uint(views[v].dyn[0]);
  out[v * 32 + t] = w;
}

// ------------------------------------------------------------------------------------------------ cell update
// computeCell (GeometryPool.ts:519-545) on the device for cells [c0, c0 + gridDim.x) of one mesh after an instance
// update: the box of the instances' world spheres gives the centre, the radius reaches every instance sphere, both
// inflated (1e-4 / 1e-3). Double precision in the host's operation order (min / max reductions are exact in any
// order), so each record equals the host's computation bit for bit. One block of kCellSize threads per cell.
__global__ void __launch_bounds__(128) k_cells_update(const float4 *__restrict__ inst, double sx, double sy, double sz,
                                                      double sr, uint32_t instance_base, uint32_t instance_count,
                                                      uint32_t cell_base, uint32_t slot, uint32_t c0,
                                                      CellRec *__restrict__ cells) {
  __shared__ double red[7][kCellSize];
  const uint32_t cell = c0 + blockIdx.x, t = threadIdx.x;
  const uint32_t first = cell * kCellSize, end = min(first + kCellSize, instance_count);
  const uint32_t g = first + t;
  const bool on = g < end;
  double s[4] = {0, 0, 0, 0};
  if (on) {
    const float4 *c = inst + (size_t)(instance_base + g) * 4;
    const float4 a = c[0], b = c[1], d = c[2], e = c[3];
    s[0] = (double)a.x * sx + (double)b.x * sy + (double)d.x * sz + (double)e.x;
    s[1] = (double)a.y * sx + (double)b.y * sy + (double)d.y * sz + (double)e.y;
    s[2] = (double)a.z * sx + (double)b.z * sy + (double)d.z * sz + (double)e.z;
    const double n0 = sqrt((double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z);
    const double n1 = sqrt((double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z);
    const double n2 = sqrt((double)d.x * d.x + (double)d.y * d.y + (double)d.z * d.z);
    s[3] = sr * fmax(n0, fmax(n1, n2));
  }
  for (int a = 0; a < 3; a++) {
    red[a][t] = on ? s[a] - s[3] : INFINITY;
    red[3 + a][t] = on ? s[a] + s[3] : -INFINITY;
  }
  red[6][t] = on ? s[3] : 0.0;
  __syncthreads();
  for (uint32_t w = kCellSize / 2; w > 0; w >>= 1) {
    if (t < w) {
      for (int a = 0; a < 3; a++) {
        red[a][t] = fmin(red[a][t], red[a][t + w]);
        red[3 + a][t] = fmax(red[3 + a][t], red[3 + a][t + w]);
      }
      red[6][t] = fmax(red[6][t], red[6][t + w]);
    }
    __syncthreads();
  }
  const double cx = (red[0][0] + red[3][0]) / 2, cy = (red[1][0] + red[4][0]) / 2, cz = (red[2][0] + red[5][0]) / 2;
  const double max_radius = red[6][0];
  __syncthreads();
  red[0][t] = on ? sqrt((s[0] - cx) * (s[0] - cx) + (s[1] - cy) * (s[1] - cy) + (s[2] - cz) * (s[2] - cz)) + s[3] : 0.0;
  __syncthreads();
  for (uint32_t w = kCellSize / 2; w > 0; w >>= 1) {
    if (t < w) red[0][t] = fmax(red[0][t], red[0][t + w]);
    __syncthreads();
  }
  if (t == 0) {
    CellRec r;
    r.sphere = make_float4((float)cx, (float)cy, (float)cz, (float)(red[0][0] * (1 + 1e-4) + 1e-3));
    r.max_radius = (float)(max_radius * (1 + 1e-4) + 1e-4);
    r.slot = slot;
    r.first = instance_base + first;
    r.count = end - first;
    cells[cell_base + cell] = r;
  }
}

// ------------------------------------------------------------------------------------------------ launchers
cudaError_t launch_cells_update(const float4 *inst, const double sphere[4], uint32_t instance_base,
                                uint32_t instance_count, uint32_t cell_base, uint32_t slot, uint32_t c0, uint32_t n,
                                CellRec *cells, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_cells_update<<<n, kCellSize, 0, st>>>(inst, sphere[0], sphere[1], sphere[2], sphere[3], instance_base,
                                          instance_count, cell_base, slot, c0, cells);
  return cudaGetLastError();
}

cudaError_t launch_gather_stats(const ViewConst *views, uint32_t nviews, uint32_t *out, cudaStream_t st) {
  k_gather_stats<<<nviews, 32, 0, st>>>(views, nviews, out);
  return cudaGetLastError();
}

cudaError_t launch_reset(const ViewConst *views, uint32_t nviews, uint32_t *ctl, cudaStream_t st) {
  const uint32_t blocks = nviews < 1024 ? (nviews ? nviews : 1) : 1024;
  k_reset<<<blocks, 256, 0, st>>>(views, nviews, ctl);
  return cudaGetLastError();
}

cudaError_t launch_cells(const Scene &S, const Scene *scenes, const ViewConst *views, uint32_t nviews,
                         uint32_t total_units, uint2 *units, uint32_t *unit_count, cudaStream_t st) {
  if (total_units == 0) return cudaSuccess;
  const uint32_t blocks = (total_units + 255) / 256;
  if (scenes)
    k_cells<true><<<blocks, 256, 0, st>>>(S, scenes, views, nviews, total_units, units, unit_count);
  else
    k_cells<false><<<blocks, 256, 0, st>>>(S, nullptr, views, nviews, total_units, units, unit_count);
  return cudaGetLastError();
}

cudaError_t configure_select(bool multi, int *instances_per_sm, int *chunks_per_sm) {
  cudaError_t e = multi ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(instances_per_sm, k_instances<false, true>, 128, 0)
                        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(instances_per_sm, k_instances<false, false>, 128, 0);
  if (e != cudaSuccess) return e;
  return multi ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(chunks_per_sm, k_chunks<false, true>, 128, 0)
               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(chunks_per_sm, k_chunks<false, false>, 128, 0);
}

template <bool MULTI>
static void instances_kernel(const Scene &S, const Scene *scenes, const ViewConst *views, const uint2 *units,
                             uint32_t *ctl, uint4 *queue, uint32_t capacity, int round, uint32_t grid,
                             uint32_t chunk_shift, uint32_t *overflow, cudaStream_t st) {
  if (round < 0)  // the budget search's pass
    k_instances<true, MULTI><<<grid, 128, 0, st>>>(S, scenes, views, S.hzbs, units, ctl, queue, capacity, 0,
                                                   chunk_shift, overflow);
  else
    k_instances<false, MULTI><<<grid, 128, 0, st>>>(S, scenes, views, S.hzbs, units, ctl, queue, capacity, round,
                                                    chunk_shift, overflow);
}

cudaError_t launch_instances(const Scene &S, const Scene *scenes, const ViewConst *views, const uint2 *units,
                             uint32_t *ctl, uint4 *queue, uint32_t capacity, int round, uint32_t grid,
                             uint32_t *overflow, cudaStream_t st, uint32_t chunk_shift) {
  if (chunk_shift < kChunkShiftFloor || chunk_shift > kChunkShiftMax || !overflow) return cudaErrorInvalidValue;
  if (scenes)
    instances_kernel<true>(S, scenes, views, units, ctl, queue, capacity, round, grid, chunk_shift, overflow, st);
  else
    instances_kernel<false>(S, nullptr, views, units, ctl, queue, capacity, round, grid, chunk_shift, overflow, st);
  return cudaGetLastError();
}

template <bool MULTI>
static void instances_redo_kernel(const Scene &S, const Scene *scenes, const ViewConst *views, const uint2 *units,
                                  uint32_t *ctl, uint4 *queue, uint32_t capacity, int round, uint32_t chunk_shift,
                                  uint32_t *overflow, uint32_t grid, cudaStream_t st) {
  if (round < 0)
    k_instances_redo<true, MULTI><<<grid, 128, 0, st>>>(S, scenes, views, S.hzbs, units, ctl, queue, capacity, 0,
                                                        chunk_shift, overflow);
  else
    k_instances_redo<false, MULTI><<<grid, 128, 0, st>>>(S, scenes, views, S.hzbs, units, ctl, queue, capacity,
                                                         round, chunk_shift, overflow);
}

cudaError_t launch_instances_redo(const Scene &S, const Scene *scenes, const ViewConst *views, const uint2 *units,
                                  uint32_t *ctl, uint4 *queue, uint32_t capacity, int round, uint32_t *overflow,
                                  uint32_t grid, cudaStream_t st, uint32_t chunk_shift) {
  if (chunk_shift < kChunkShiftFloor || chunk_shift > kChunkShiftMax || !overflow || grid == 0)
    return cudaErrorInvalidValue;
  if (scenes)
    instances_redo_kernel<true>(S, scenes, views, units, ctl, queue, capacity, round, chunk_shift, overflow, grid, st);
  else
    instances_redo_kernel<false>(S, nullptr, views, units, ctl, queue, capacity, round, chunk_shift, overflow, grid,
                                 st);
  return cudaGetLastError();
}

template <bool MULTI>
static void chunks_kernel(const Scene &S, const Scene *scenes, const ViewConst *views, uint4 *queue, uint32_t *ctl,
                          uint32_t capacity, int round, uint32_t grid, cudaStream_t st) {
  if (round < 0)
    k_chunks<true, MULTI><<<grid, 128, 0, st>>>(S, scenes, views, S.hzbs, queue, ctl, capacity, 0);
  else
    k_chunks<false, MULTI><<<grid, 128, 0, st>>>(S, scenes, views, S.hzbs, queue, ctl, capacity, round);
}

cudaError_t launch_chunks(const Scene &S, const Scene *scenes, const ViewConst *views, uint4 *queue, uint32_t *ctl,
                          uint32_t capacity, int round, uint32_t grid, cudaStream_t st) {
  if (scenes)
    chunks_kernel<true>(S, scenes, views, queue, ctl, capacity, round, grid, st);
  else
    chunks_kernel<false>(S, nullptr, views, queue, ctl, capacity, round, grid, st);
  return cudaGetLastError();
}

cudaError_t launch_budget(const ViewConst *views, uint32_t nviews, uint32_t *ctl, cudaStream_t st) {
  const uint32_t blocks = (nviews * 32 + 127) / 128;
  k_budget<<<blocks, 128, 0, st>>>(views, nviews, ctl);
  return cudaGetLastError();
}

cudaError_t launch_finish(const ViewConst *views, uint32_t nviews, uint32_t *ctl, int round, cudaStream_t st) {
  const uint32_t blocks = (nviews * 32 + 127) / 128;
  k_finish<<<blocks, 128, 0, st>>>(views, nviews, ctl, round);
  return cudaGetLastError();
}

cudaError_t launch_expand(const Scene &S, const ViewConst *view, uint32_t cut, uint32_t *out, uint64_t capacity,
                          uint32_t grid, cudaStream_t st) {
  k_expand<<<grid, 256, 0, st>>>(S, view, cut, out, capacity);
  return cudaGetLastError();
}

cudaError_t launch_hzb(const float *depth, const HzbDesc &H, float *out, int copy_mip0, cudaStream_t st) {
  dim3 grid((H.w[0] + kHzbTile - 1) / kHzbTile, (H.h[0] + 2 * kHzbTile - 1) / (2 * kHzbTile));
  k_hzb_tiles<<<grid, 256, 0, st>>>(depth, H, out, copy_mip0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || H.levels <= kHzbTileLevels) return e;
  k_hzb_tail<<<1, 1024, 0, st>>>(H, out);
  return cudaGetLastError();
}

cudaError_t launch_hzb_views(const ViewConst *views, uint32_t nviews, uint32_t max_w,
                             uint32_t max_h, bool tail, cudaStream_t st) {
  dim3 grid((max_w + kHzbTile - 1) / kHzbTile, (max_h + 2 * kHzbTile - 1) / (2 * kHzbTile), nviews);
  k_hzb_tiles_views<<<grid, 256, 0, st>>>(views);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !tail) return e;
  k_hzb_tail_views<<<nviews, 1024, 0, st>>>(views, kHzbTileLevels);
  return cudaGetLastError();
}

cudaError_t launch_wait_probe(uint64_t limit_ns, unsigned long long *out, cudaStream_t st) {
  k_wait_probe<<<1, 32, 0, st>>>(limit_ns, out);
  return cudaGetLastError();
}

uint32_t hzb_stream_blocks_per_sm() {
  if (cudaFuncSetAttribute(k_hzb_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHzbStreamSmem) !=
      cudaSuccess)
    return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_hzb_stream, kHzbStreamThreads, kHzbStreamSmem) !=
      cudaSuccess)
    return 0;
  return (uint32_t)n;
}

cudaError_t launch_hzb_stream(const unsigned char *plan, uint32_t grid, const ViewConst *views, uint32_t nviews,
                              bool tail, cudaStream_t st) {
  k_hzb_stream<<<grid, kHzbStreamThreads, kHzbStreamSmem, st>>>(plan);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !tail) return e;
  k_hzb_tail_views<<<nviews, 1024, 0, st>>>(views, kHzbStripLevels);
  return cudaGetLastError();
}

cudaError_t launch_select_cut(const Scene &S, uint32_t slot, uint32_t mcount, uint32_t count, const float *vm16,
                              const float *params, float threshold, float blend, uint8_t *lo, uint8_t *hi, uint32_t grid,
                              cudaStream_t st) {
  k_select_cut<<<grid, 256, 0, st>>>(S, slot, mcount, count, vm16, params, threshold, blend, lo, hi);
  return cudaGetLastError();
}

}  // namespace vgc
