// sm_100a kernels of the cull + LOD-cut engine.
//
// Pass structure for a batch of views (all views of one scene in each launch):
//   k_cells    one thread per (view, cell): the cell tests of GeometryPool.ts:728-760; surviving (view, cell)
//              units are compacted with one atomic per warp (__ballot_sync / __popc).
//   k_select   persistent blocks of 128 threads, one visible unit at a time. Thread i tests instance i of the
//              cell (GeometryPool.ts:846-913) and picks its LOD level range (selectLevels :771-843). Fast-path
//              instances emit their meshlets directly; the others become work items kept in shared memory, whose
//              meshlets the block then tests one per thread over a flattened (item, meshlet) index
//              (GeometryPool.ts:916-970), reading the struct-of-arrays bounds coalesced. Drawn meshlets are staged
//              in shared memory (one shared atomic per warp) and flushed with one global atomic per cut and part.
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

// Natural log from float basic operations (same steps as the oracle's vgo_logf): x = m 2^e, m in
// [sqrt(1/2), sqrt(2)), ln x = e ln2 + 2 atanh((m-1)/(m+1)) by its odd series (Abramowitz & Stegun 4.1.27),
// ln2 split in a high part with trailing zero bits and a low correction.
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
  float p = s2 * (0.333333343f + s2 * (0.2f + s2 * (0.142857149f + s2 * (0.111111112f + s2 * 0.0909090936f))));
  float lnm = (s + s * p) * 2.0f;
  float fe = float(e);
  return fe * 0.693145752f + (fe * 1.42860677e-06f + lnm);
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

__device__ __forceinline__ void xform(const float *M, float x, float y, float z, float out[3]) {
#pragma unroll
  for (int r = 0; r < 3; r++) out[r] = ((M[r * 4 + 0] * x + M[r * 4 + 1] * y) + M[r * 4 + 2] * z) + M[r * 4 + 3];
}

__device__ __forceinline__ float len3(const float v[3]) { return sqrtf((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]); }

// VM = V * M (rows 0..2, row-major 3x4) and the instance scale (GeometryPool.ts:670-675)
__device__ __forceinline__ void model_view(const float *Vr, const float4 *cols, float *VM, float &scale) {
  float4 c[4] = {cols[0], cols[1], cols[2], cols[3]};
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int k = 0; k < 4; k++)
      VM[r * 4 + k] = ((Vr[r * 4 + 0] * c[k].x + Vr[r * 4 + 1] * c[k].y) + Vr[r * 4 + 2] * c[k].z) + Vr[r * 4 + 3] * c[k].w;
  float l0[3] = {c[0].x, c[0].y, c[0].z}, l1[3] = {c[1].x, c[1].y, c[1].z}, l2[3] = {c[2].x, c[2].y, c[2].z};
  scale = fmx(len3(l0), fmx(len3(l1), len3(l2)));
}

// frustumDistance (GeometryPool.ts:690-698) in view space
__device__ __forceinline__ float frustum(const ViewConst &V, const float c[3], bool swept) {
  float m = 1e30f;
#pragma unroll
  for (int p = 0; p < 6; p++) {
    float d = ((V.plane[p * 4] * c[0] + V.plane[p * 4 + 1] * c[1]) + V.plane[p * 4 + 2] * c[2]) + V.plane[p * 4 + 3];
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
  float min_x = fmn(xlo / near_depth, xlo / far_depth) * V.P0 - V.P8;
  float max_x = fmx(xhi / near_depth, xhi / far_depth) * V.P0 - V.P8;
  float min_y = fmn(ylo / near_depth, ylo / far_depth) * V.P5 - V.P9;
  float max_y = fmx(yhi / near_depth, yhi / far_depth) * V.P5 - V.P9;
  float min_z = V.P14 / near_depth - V.P10;
  if (!(min_z < 1.0f)) return false;
  float W = float(H.w[0]), Hh = float(H.h[0]);
  float fx0 = floorf((min_x * 0.5f + 0.5f) * W);
  float fx1 = floorf((max_x * 0.5f + 0.5f) * W);
  float fy0 = floorf((0.5f - max_y * 0.5f) * Hh);
  float fy1 = floorf((0.5f - min_y * 0.5f) * Hh);
  uint32_t x0 = uint32_t(fmn(fmx(fx0, 0.0f), W - 1.0f));
  uint32_t x1 = uint32_t(fmn(fmx(fx1, 0.0f), W - 1.0f));
  uint32_t y0 = uint32_t(fmn(fmx(fy0, 0.0f), Hh - 1.0f));
  uint32_t y1 = uint32_t(fmn(fmx(fy1, 0.0f), Hh - 1.0f));
  uint32_t dx = x1 > x0 ? x1 - x0 : 0u, dy = y1 > y0 ? y1 - y0 : 0u;
  uint32_t level = ceil_log2((dx > dy ? dx : dy) + 1u);
  if (level > H.levels - 1) level = H.levels - 1;
  uint32_t lw = H.w[level], lh = H.h[level];
  const float *mip = H.data + H.off[level];
  uint32_t tx0 = min(x0 >> level, lw - 1), tx1 = min(x1 >> level, lw - 1);
  uint32_t ty0 = min(y0 >> level, lh - 1), ty1 = min(y1 >> level, lh - 1);
  float s00 = __ldg(mip + ty0 * lw + tx0), s10 = __ldg(mip + ty0 * lw + tx1);
  float s01 = __ldg(mip + ty1 * lw + tx0), s11 = __ldg(mip + ty1 * lw + tx1);
  float hmax = fmx(fmx(s00, s10), fmx(s01, s11));
  return min_z > hmax + float(1e-6);
}

// occludedSphere (GeometryPool.ts:701-705): the sphere grows by the camera band's top error in pixels
__device__ __forceinline__ bool occluded(const ViewConst &V, const HzbDesc *hzbs, float high0, bool on, const float c[3],
                                         float r) {
  if (!on || !V.occl_active || V.hzb < 0) return false;
  float margin = (fabsf(c[2]) * high0) / V.proj_scale;
  return hzb_occluded(V, hzbs[V.hzb], c, r + margin);
}

// projectedError (GeometryPool.ts:678-683)
__device__ __forceinline__ float proj_error(const ViewConst &V, const float *VM, float scale, float4 s, float error) {
  float c[3];
  xform(VM, s.x, s.y, s.z, c);
  float dist = fmx(len3(c) - s.w * scale, V.near_);
  float pixels = ((error * scale) / dist) * V.proj_scale;
  return error >= float(1e30 * 0.5) ? 1e30f : pixels;
}

__device__ __forceinline__ uint32_t fade_step(float e, float low, float fade_scale) {
  float x = rintf(vg_logf(fmx(e, float(1e-30)) / low) * fade_scale);
  x = fmn(fmx(x, 0.0f), 255.0f);
  return uint32_t(x);
}

__device__ __forceinline__ uint32_t part_of(uint32_t packed) { return (packed & 0xffff00u) == kFullFadeBits ? 0u : 1u; }

__device__ __forceinline__ uint32_t *mesh_count(const ViewConst &V, uint32_t slot_capacity, uint32_t cut, uint32_t slot,
                                                uint32_t part) {
  return V.counters + VGC_COUNTER_HEADER + (((cut * slot_capacity + slot) * 2 + part) * 2);
}

// ------------------------------------------------------------------------------------------------ k_cells
__global__ void __launch_bounds__(256) k_cells(Scene S, const ViewConst *__restrict__ views, uint32_t nviews,
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
  const uint32_t cell = u - V.unit_offset;
  bool vis = false;
  if (cell < S.cell_count) {
    CellRec cr = S.cells[cell];
    const MeshRec &mesh = S.meshes[cr.slot];
    vis = mesh.enabled != 0;
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

// ------------------------------------------------------------------------------------------------ k_select
constexpr int kSelThreads = 128;
constexpr int kStage = 512;  // staged draw entries per cut (fast path: up to 4 per instance)

struct SelectSmem {
  ViewConst view;
  LevelRec levels[kMaxLevels];
  float vm[kCellSize][13];
  uint4 items[2][kCellSize];       // per cut: (instance local | occl << 31, first, last, 0)
  uint32_t prefix[2][kCellSize + 1];
  uint4 stage[2][kStage];
  uint32_t n_items[2];
  uint32_t stage_n[2];
  uint32_t idx_n[2][2];
  uint32_t base_sel[2], base_idx[2][2], kept[2];
  uint32_t survived[2], work[2], occluded, fast[2];
  Bands bands;
  float threshold;
  uint32_t redo[2];
  int skip;
};

// Appends drawn entries of one warp to the block's staging area: one shared atomic for the slot count and one
// for the two parts' index counts (packed 16 + 16 bits: a warp adds at most 32 * 384 indices per part).
__device__ __forceinline__ void stage_entries(SelectSmem &sm, uint32_t cut, bool drawn, uint32_t instance,
                                              uint32_t meshlet, uint32_t packed) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t mask = __ballot_sync(0xffffffffu, drawn);
  if (!mask) return;
  const uint32_t tri3 = drawn ? (packed & 255u) * 3u : 0u;
  const uint32_t part = part_of(packed);
  const uint32_t mine = part == 0 ? tri3 : (tri3 << 16);
  uint32_t incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t n = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (uint32_t)o) incl += n;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  uint32_t slot_base = 0, idx0 = 0, idx1 = 0;
  if (lane == 0) {
    slot_base = atomicAdd(&sm.stage_n[cut], __popc(mask));
    idx0 = atomicAdd(&sm.idx_n[cut][0], total & 0xffffu);
    idx1 = atomicAdd(&sm.idx_n[cut][1], total >> 16);
  }
  slot_base = __shfl_sync(0xffffffffu, slot_base, 0);
  idx0 = __shfl_sync(0xffffffffu, idx0, 0);
  idx1 = __shfl_sync(0xffffffffu, idx1, 0);
  if (drawn) {
    const uint32_t excl = incl - mine;
    const uint32_t local = part == 0 ? idx0 + (excl & 0xffffu) : idx1 + (excl >> 16);
    sm.stage[cut][slot_base + __popc(mask & ((1u << lane) - 1u))] = make_uint4(instance, meshlet, local, packed);
  }
}

// Writes the staged entries to the view's draw list: one global atomic per cut for the list position and one per
// (cut, part) for the index region, then a coalesced copy. Entries past max_drawn are dropped, and only the kept
// ones are counted in the index region, as the reference does (GeometryPool.ts:959-965).
__device__ void flush_stage(SelectSmem &sm, uint32_t slot_capacity, uint32_t slot) {
  __syncthreads();
  const ViewConst &V = sm.view;
  if (threadIdx.x == 0) {
    for (uint32_t cut = 0; cut < 2; cut++) {
      const uint32_t n = sm.stage_n[cut];
      sm.kept[cut] = 0;
      if (!n) continue;
      const uint32_t base = atomicAdd(V.counters + C_CUT(cut) + VGC_CUT_SELECTED, n);
      sm.base_sel[cut] = base;
      const uint32_t kept = base >= V.max_drawn ? 0u : min(n, V.max_drawn - base);
      sm.kept[cut] = kept;
      uint32_t add[2] = {sm.idx_n[cut][0], sm.idx_n[cut][1]};
      if (kept != n) {  // overflow: re-pack the kept prefix
        add[0] = add[1] = 0;
        for (uint32_t s = 0; s < kept; s++) {
          uint4 &e = sm.stage[cut][s];
          const uint32_t p = part_of(e.w);
          e.z = add[p];
          add[p] += (e.w & 255u) * 3u;
        }
      }
      for (uint32_t p = 0; p < 2; p++)
        sm.base_idx[cut][p] = add[p] ? atomicAdd(mesh_count(V, slot_capacity, cut, slot, p), add[p]) : 0u;
    }
  }
  __syncthreads();
  for (uint32_t cut = 0; cut < 2; cut++) {
    const uint32_t kept = sm.kept[cut];
    uint4 *dst = V.draw_list + (size_t)cut * V.max_drawn + sm.base_sel[cut];
    for (uint32_t s = threadIdx.x; s < kept; s += blockDim.x) {
      uint4 e = sm.stage[cut][s];
      e.z += sm.base_idx[cut][part_of(e.w)];
      dst[s] = e;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    sm.stage_n[0] = sm.stage_n[1] = 0;
    sm.idx_n[0][0] = sm.idx_n[0][1] = sm.idx_n[1][0] = sm.idx_n[1][1] = 0;
  }
  __syncthreads();
}

// selectLevels (GeometryPool.ts:771-843) for one instance and cut; returns true when the instance survives
__device__ __forceinline__ void select_levels(SelectSmem &sm, const Scene &S, const MeshRec &mesh, uint32_t cut,
                                              uint32_t il, uint32_t instance, bool occl_flag, const float *VM,
                                              float scale, float px_min, float px_max, uint32_t levels,
                                              uint32_t &fast_n, uint32_t &fast_first) {
  const float low = sm.bands.low[cut], high = sm.bands.high[cut];
  uint32_t first = 0xffffffffu, last = 0, possible_m = 0, guaranteed = 0;
  for (uint32_t l = 0; l < levels; l++) {
    const LevelRec &L = sm.levels[l];
    bool possible = L.min_own * px_max <= high && (L.max_parent >= float(1e30 * 0.5) || L.max_parent * px_min > low);
    bool sure = L.max_own * px_min <= low * float(1 - 1e-3) &&
                (L.min_parent >= float(1e30 * 0.5) || L.min_parent * px_max > high * float(1 + 1e-3));
    if (possible) {
      first = min(first, L.first);
      last = max(last, L.first + L.count);
      possible_m += L.count;
      if (sure) guaranteed += L.count;
    }
  }
  fast_n = 0;
  if (!(last > first)) return;
  float cc[3];
  xform(VM, mesh.cull.x, mesh.cull.y, mesh.cull.z, cc);
  const float cr = mesh.cull.w * scale;
  const bool fast = possible_m > 0 && possible_m == last - first && guaranteed == possible_m &&
                    possible_m <= kFastPathMax && (!sm.view.frustum || frustum(sm.view, cc, cut == 1) >= cr);
  atomicAdd(&sm.survived[cut], 1u);
  if (fast) {
    fast_n = possible_m;
    fast_first = first;
    atomicAdd(&sm.fast[cut], possible_m);
  } else {
    const uint32_t k = atomicAdd(&sm.n_items[cut], 1u);
    sm.items[cut][k] = make_uint4(il | (occl_flag ? 0x80000000u : 0u), first, last, 0);
  }
}

__global__ void __launch_bounds__(kSelThreads) k_select(Scene S, const ViewConst *__restrict__ views,
                                                        const HzbDesc *__restrict__ hzbs,
                                                        const uint2 *__restrict__ units,
                                                        const uint32_t *__restrict__ unit_count, int round) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SelectSmem &sm = *reinterpret_cast<SelectSmem *>(smem_raw);
  const uint32_t tid = threadIdx.x;
  const uint32_t n_units = *unit_count;
  for (uint32_t u = blockIdx.x; u < n_units; u += gridDim.x) {
    __syncthreads();
    const uint2 unit = units[u];
    {  // view constants into shared memory
      const uint32_t *src = reinterpret_cast<const uint32_t *>(views + unit.x);
      uint32_t *dst = reinterpret_cast<uint32_t *>(&sm.view);
      for (uint32_t i = tid; i < sizeof(ViewConst) / 4; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const ViewConst &V = sm.view;
    if (tid == 0) {
      sm.redo[0] = round == 0 ? 1u : V.counters[VGC_COUNTER_REDO0];
      sm.redo[1] = round == 0 ? 1u : V.counters[VGC_COUNTER_REDO1];
      sm.skip = !(sm.redo[0] || sm.redo[1]);
      sm.threshold = V.budget > 0.0f ? V.dyn[0] : V.error_threshold;
      load_bands(V, sm.threshold, sm.bands);
      sm.n_items[0] = sm.n_items[1] = 0;
      sm.stage_n[0] = sm.stage_n[1] = 0;
      sm.idx_n[0][0] = sm.idx_n[0][1] = sm.idx_n[1][0] = sm.idx_n[1][1] = 0;
      sm.survived[0] = sm.survived[1] = sm.work[0] = sm.work[1] = sm.occluded = 0;
      sm.fast[0] = sm.fast[1] = 0;
    }
    const CellRec cell = S.cells[unit.y];
    const MeshRec &mesh = S.meshes[cell.slot];
    const uint32_t levels = min(mesh.level_count, kMaxLevels);
    {
      const uint32_t *src = reinterpret_cast<const uint32_t *>(S.levels + mesh.level_base);
      uint32_t *dst = reinterpret_cast<uint32_t *>(sm.levels);
      for (uint32_t i = tid; i < levels * (sizeof(LevelRec) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    if (sm.skip) continue;

    // ---- instance phase (GeometryPool.ts:874-912)
    uint32_t fast_n[2] = {0, 0}, fast_first[2] = {0, 0};
    const uint32_t instance = cell.first + tid;
    if (tid < cell.count) {
      float VM[12], scale;
      model_view(V.V, S.inst + (size_t)instance * 4, VM, scale);
#pragma unroll
      for (int i = 0; i < 12; i++) sm.vm[tid][i] = VM[i];
      sm.vm[tid][12] = scale;
      float c[3];
      xform(VM, mesh.sphere.x, mesh.sphere.y, mesh.sphere.z, c);
      const float radius = mesh.sphere.w * scale;
      const bool no_frustum = !V.frustum;
      bool in_camera = no_frustum || frustum(V, c, false) >= -radius;
      bool in_shadow = mesh.shadow != 0 && (no_frustum || frustum(V, c, true) >= -radius);
      if (round > 0) {
        in_camera = in_camera && sm.redo[0];
        in_shadow = in_shadow && sm.redo[1];
      }
      const float min_pixels = fmx(V.min_pixel_radius, mesh.min_pixel_radius);
      const float view_distance = len3(c);
      const bool too_small = view_distance > radius && (radius * V.proj_scale) / view_distance < min_pixels;
      const bool too_far = view_distance - radius > mesh.max_draw_distance;
      if ((in_camera || in_shadow) && !too_small && !too_far) {
        const bool occl_on = mesh.occlusion != 0;
        if (in_camera && occluded(V, hzbs, sm.bands.high[0], occl_on, c, radius)) {
          in_camera = false;
          atomicAdd(&sm.occluded, 1u);
        }
        float lc[3];
        xform(VM, mesh.lod.x, mesh.lod.y, mesh.lod.z, lc);
        const float d = len3(lc), r = mesh.lod.w * scale;
        const float px_min = (scale * V.proj_scale) / fmx(d - r, V.near_);
        const float px_max = (scale * V.proj_scale) / fmx(d + r, V.near_);
        if (in_camera)
          select_levels(sm, S, mesh, 0, tid, instance, occl_on, VM, scale, px_min, px_max, levels, fast_n[0], fast_first[0]);
        if (in_shadow)
          select_levels(sm, S, mesh, 1, tid, instance, false, VM, scale, px_min, px_max, levels, fast_n[1], fast_first[1]);
      }
    }
    // fast path entries (at most 4 per instance and cut), staged warp by warp
#pragma unroll
    for (uint32_t cut = 0; cut < 2; cut++)
      for (uint32_t k = 0; k < kFastPathMax; k++) {
        const bool emit = k < fast_n[cut];
        uint32_t meshlet = fast_first[cut] + k, packed = 0;
        if (emit) packed = __float_as_uint(S.m_err[meshlet].z) | kFullFadeBits;
        stage_entries(sm, cut, emit, instance, meshlet, packed);
      }
    __syncthreads();
    // flattened (item, meshlet) index: prefix over item sizes, per cut
    if (tid < 64) {
      const uint32_t cut = tid >> 5, lane = tid & 31;
      const uint32_t n = sm.n_items[cut];
      uint32_t carry = 0;
      if (lane == 0) sm.prefix[cut][0] = 0;
      for (uint32_t b = 0; b < n; b += 32) {
        const uint32_t k = b + lane;
        const uint32_t sz = k < n ? sm.items[cut][k].z - sm.items[cut][k].y : 0u;
        uint32_t incl = sz;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= (uint32_t)o) incl += t;
        }
        if (k < n) sm.prefix[cut][k + 1] = carry + incl;
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) sm.work[cut] = n;
    }
    __syncthreads();
    if (sm.stage_n[0] + sm.stage_n[1]) flush_stage(sm, S.slot_capacity, cell.slot);

    // ---- meshlet phase (GeometryPool.ts:938-967)
    for (uint32_t cut = 0; cut < 2; cut++) {
      const uint32_t n = sm.n_items[cut];
      const uint32_t total = n ? sm.prefix[cut][n] : 0u;
      const float low = sm.bands.low[cut], high = sm.bands.high[cut], fs = sm.bands.fade_scale;
      for (uint32_t base = 0; base < total; base += kSelThreads) {
        const uint32_t t = base + tid;
        bool drawn = false;
        uint32_t inst = 0, meshlet = 0, packed = 0;
        if (t < total) {
          uint32_t a = 0, b = n;  // largest k with prefix[k] <= t
          while (b - a > 1) {
            const uint32_t mid = (a + b) >> 1;
            if (sm.prefix[cut][mid] <= t) a = mid;
            else b = mid;
          }
          const uint4 item = sm.items[cut][a];
          const uint32_t il = item.x & 0xffffu;
          const bool occl_on = (item.x >> 31) != 0;
          meshlet = item.y + (t - sm.prefix[cut][a]);
          inst = cell.first + il;
          const float *VM = sm.vm[il];
          const float scale = VM[12];
          const float4 cs = __ldg(S.m_cull + meshlet);
          float c[3];
          xform(VM, cs.x, cs.y, cs.z, c);
          const float r = cs.w * scale;
          bool visible = !V.frustum || frustum(V, c, cut == 1) >= -r;
          if (cut == 0 && visible) visible = !occluded(V, hzbs, sm.bands.high[0], occl_on, c, r);
          if (visible) {
            const float4 ls = __ldg(S.m_lod + meshlet), ps = __ldg(S.m_parent + meshlet), er = __ldg(S.m_err + meshlet);
            const float own = proj_error(V, VM, scale, ls, er.x);
            const float parent = proj_error(V, VM, scale, ps, er.y);
            const uint32_t lo = fs > 0.0f ? fade_step(own, low, fs) : 0u;
            const uint32_t hi = fs > 0.0f ? fade_step(parent, low, fs) : 255u;
            drawn = own <= high && parent > low && hi > lo;
            packed = __float_as_uint(er.z) | (lo << 8) | (hi << 16);
          }
        }
        stage_entries(sm, cut, drawn, inst, meshlet, packed);
        __syncthreads();
        if (sm.stage_n[cut] > kStage - kSelThreads) flush_stage(sm, S.slot_capacity, cell.slot);
      }
    }
    flush_stage(sm, S.slot_capacity, cell.slot);
    if (tid == 0) {
      for (uint32_t cut = 0; cut < 2; cut++) {
        if (sm.survived[cut]) atomicAdd(V.counters + C_CUT(cut) + VGC_CUT_SURVIVED, sm.survived[cut]);
        if (sm.work[cut]) atomicAdd(V.counters + C_CUT(cut) + VGC_CUT_WORK, sm.work[cut]);
      }
      if (sm.occluded) atomicAdd(V.counters + VGC_COUNTER_OCCLUDED, sm.occluded);
      const uint32_t tested = (sm.n_items[0] ? sm.prefix[0][sm.n_items[0]] : 0u) + (sm.n_items[1] ? sm.prefix[1][sm.n_items[1]] : 0u);
      atomicAdd(V.counters + VGC_COUNTER_INSTANCES_TESTED, cell.count);
      if (tested) atomicAdd(V.counters + VGC_COUNTER_MESHLETS_TESTED, tested);
      if (sm.fast[0] + sm.fast[1]) atomicAdd(V.counters + VGC_COUNTER_FAST_EMITTED, sm.fast[0] + sm.fast[1]);
      atomicAdd(V.counters + VGC_COUNTER_LEVELS_READ, levels);
    }
  }
}

// ------------------------------------------------------------------------------------------------ k_finish
__device__ __forceinline__ float fill_of(const ViewConst &V, uint32_t cut) {
  const float requested = float(V.counters[C_CUT(cut) + VGC_CUT_REQUESTED]);
  const float selected = float(V.counters[C_CUT(cut) + VGC_CUT_SELECTED]);
  return fmx(requested / float(V.index_capacity[cut]), selected / float(V.max_drawn));
}

__global__ void __launch_bounds__(128) k_finish(const ViewConst *__restrict__ views, uint32_t nviews,
                                                uint32_t slot_capacity, uint32_t slots_used, int round) {
  const uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (v >= nviews) return;
  const ViewConst &V = views[v];
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
      if (again) ctr[VGC_COUNTER_ROUNDS] += 1;
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
// 32x32 tile of mip 0 per block; levels 1..5 of the tile are reduced in shared memory. Mip i texel (x, y) is the
// max of texels (2x, 2y), (min(2x+1, w-1), 2y), ... of mip i-1: tile borders fall on even coordinates at every
// level, so the clamped neighbour is always inside the tile.
__global__ void __launch_bounds__(256) k_hzb_tiles(const float *__restrict__ depth, HzbDesc H, float *__restrict__ out,
                                                   int copy_mip0) {
  __shared__ float buf[2][32][33];
  const uint32_t ox = blockIdx.x * 32, oy = blockIdx.y * 32;
  const uint32_t W = H.w[0], Hh = H.h[0];
  for (uint32_t i = threadIdx.x; i < 1024; i += blockDim.x) {
    const uint32_t lx = i & 31, ly = i >> 5, gx = ox + lx, gy = oy + ly;
    float v = 0.0f;
    if (gx < W && gy < Hh) {
      v = depth[(size_t)gy * W + gx];
      if (copy_mip0) out[H.off[0] + (size_t)gy * W + gx] = v;
    }
    buf[0][ly][lx] = v;
  }
  __syncthreads();
  const uint32_t top = min(H.levels, 6u);
  for (uint32_t l = 1; l < top; l++) {
    const uint32_t s = 32u >> l;
    const uint32_t px = ox >> (l - 1), py = oy >> (l - 1);  // tile origin at level l-1
    const uint32_t qx = ox >> l, qy = oy >> l;              // tile origin at level l
    const float(*src)[33] = buf[(l - 1) & 1];
    float(*dst)[33] = buf[l & 1];
    for (uint32_t i = threadIdx.x; i < s * s; i += blockDim.x) {
      const uint32_t lx = i % s, ly = i / s, gx = qx + lx, gy = qy + ly;
      if (gx < H.w[l] && gy < H.h[l]) {
        const uint32_t x0 = 2 * gx, y0 = 2 * gy;
        const uint32_t x1 = min(x0 + 1, H.w[l - 1] - 1), y1 = min(y0 + 1, H.h[l - 1] - 1);
        const float a = fmaxf(src[y0 - py][x0 - px], src[y0 - py][x1 - px]);
        const float b = fmaxf(src[y1 - py][x0 - px], src[y1 - py][x1 - px]);
        const float v = fmaxf(a, b);
        dst[ly][lx] = v;
        out[H.off[l] + (size_t)gy * H.w[l] + gx] = v;
      }
    }
    __syncthreads();
  }
}

// Levels 6 and up (at most 60 x 34 texels for a 1080p mip 0) by one block.
__global__ void __launch_bounds__(1024) k_hzb_tail(HzbDesc H, float *__restrict__ out) {
  for (uint32_t l = 6; l < H.levels; l++) {
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
      const float dist = fmx(len3(c) - s.w * sc, nr);
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
    lo[i] = l;
    hi[i] = h;
  }
}

// ------------------------------------------------------------------------------------------------ k_reset
// Zeroes each view's counter block (reset pass, GeometryPool.ts:714-725) and the batch's unit count; reads the
// output pointers from the view constants, so a captured graph serves any output slots.
__global__ void __launch_bounds__(256) k_reset(const ViewConst *__restrict__ views, uint32_t nviews, uint32_t words,
                                               uint32_t *__restrict__ unit_count) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *unit_count = 0;
  for (uint32_t v = blockIdx.x; v < nviews; v += gridDim.x) {
    uint32_t *c = views[v].counters;
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) c[i] = 0;
  }
}

// ------------------------------------------------------------------------------------------------ launchers
cudaError_t launch_reset(const ViewConst *views, uint32_t nviews, uint32_t words, uint32_t *unit_count, cudaStream_t st) {
  const uint32_t blocks = nviews < 1024 ? (nviews ? nviews : 1) : 1024;
  k_reset<<<blocks, 256, 0, st>>>(views, nviews, words, unit_count);
  return cudaGetLastError();
}

size_t select_smem_bytes() { return sizeof(SelectSmem); }

cudaError_t launch_cells(const Scene &S, const ViewConst *views, uint32_t nviews, uint32_t total_units, uint2 *units,
                         uint32_t *unit_count, cudaStream_t st) {
  if (total_units == 0) return cudaSuccess;
  const uint32_t blocks = (total_units + 255) / 256;
  k_cells<<<blocks, 256, 0, st>>>(S, views, nviews, total_units, units, unit_count);
  return cudaGetLastError();
}

cudaError_t configure_select(int *blocks_per_sm) {
  cudaError_t e = cudaFuncSetAttribute(k_select, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SelectSmem));
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_select, kSelThreads, sizeof(SelectSmem));
}

cudaError_t launch_select(const Scene &S, const ViewConst *views, const HzbDesc *hzbs, const uint2 *units,
                          const uint32_t *unit_count, int round, uint32_t grid, cudaStream_t st) {
  k_select<<<grid, kSelThreads, sizeof(SelectSmem), st>>>(S, views, hzbs, units, unit_count, round);
  return cudaGetLastError();
}

cudaError_t launch_finish(const ViewConst *views, uint32_t nviews, uint32_t slot_capacity, uint32_t slots_used,
                          int round, cudaStream_t st) {
  const uint32_t blocks = (nviews * 32 + 127) / 128;
  k_finish<<<blocks, 128, 0, st>>>(views, nviews, slot_capacity, slots_used, round);
  return cudaGetLastError();
}

cudaError_t launch_expand(const Scene &S, const ViewConst *view, uint32_t cut, uint32_t *out, uint64_t capacity,
                          uint32_t grid, cudaStream_t st) {
  k_expand<<<grid, 256, 0, st>>>(S, view, cut, out, capacity);
  return cudaGetLastError();
}

cudaError_t launch_hzb(const float *depth, const HzbDesc &H, float *out, int copy_mip0, cudaStream_t st) {
  dim3 grid((H.w[0] + 31) / 32, (H.h[0] + 31) / 32);
  k_hzb_tiles<<<grid, 256, 0, st>>>(depth, H, out, copy_mip0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || H.levels <= 6) return e;
  k_hzb_tail<<<1, 1024, 0, st>>>(H, out);
  return cudaGetLastError();
}

cudaError_t launch_select_cut(const Scene &S, uint32_t slot, uint32_t mcount, uint32_t count, const float *vm16,
                              const float *params, float threshold, float blend, uint8_t *lo, uint8_t *hi, uint32_t grid,
                              cudaStream_t st) {
  k_select_cut<<<grid, 256, 0, st>>>(S, slot, mcount, count, vm16, params, threshold, blend, lo, hi);
  return cudaGetLastError();
}

}  // namespace vgc
