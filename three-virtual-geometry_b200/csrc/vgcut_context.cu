// Host side of the cut engine behind the C ABI of include/vgcut.h: scene residency in HBM, view constants,
// the plain launch sequence, the CUDA-graph batch, HZB slots, stats and the CPU-API equivalents.
//
// The reference keeps a GeometryPool per 120 MB of WebGPU bindings (VirtualGeometry.ts:314-331) and grows its
// buffers by reallocation (GeometryPool.ts:169-208). Here one context holds one resident buffer set per array;
// growth re-uploads the host mirror into a larger allocation. Output slots (one per view of a batch) hold the
// per-view results: counters, draw list, draw args.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "vgcut_host.h"
#include "vgcut_kernels.h"

namespace vgch {
namespace {
thread_local std::string g_error;
}  // namespace

int fail(int code, const std::string &msg) {
  g_error = msg;
  return code;
}

void decode_stats(const vgc_context *ctx, const uint32_t *c, float threshold, vgc_stats *s) {
  std::memset(s, 0, sizeof *s);
  s->visible_cells = c[VGC_COUNTER_CELLS];
  s->occluded_instances = c[VGC_COUNTER_OCCLUDED];
  for (int cut = 0; cut < 2; cut++) {
    const uint32_t *k = c + VGC_COUNTER_CUT0 + cut * 5;
    s->selected[cut] = k[VGC_CUT_SELECTED];
    s->drawn[cut] = k[VGC_CUT_DRAWN];
    s->survived[cut] = k[VGC_CUT_SURVIVED];
    s->work[cut] = k[VGC_CUT_WORK];
    s->requested_indices[cut] = k[VGC_CUT_REQUESTED];
    const uint32_t cap = cut == 0 ? ctx->opts.max_triangles * 3 : ctx->opts.max_shadow_triangles * 3;
    if (k[VGC_CUT_SELECTED] > ctx->opts.max_meshlets || k[VGC_CUT_REQUESTED] > cap) s->overflow = 1;
  }
  s->rounds = c[VGC_COUNTER_ROUNDS];
  s->instances_tested = c[VGC_COUNTER_INSTANCES_TESTED];
  s->meshlets_tested = c[VGC_COUNTER_MESHLETS_TESTED];
  s->fast_emitted = c[VGC_COUNTER_FAST_EMITTED];
  s->levels_read = c[VGC_COUNTER_LEVELS_READ];
  s->predicted_triangles = (uint64_t)c[VGC_COUNTER_PREDICTED_LO] | ((uint64_t)c[VGC_COUNTER_PREDICTED_HI] << 32);
  s->meshlets_queued = c[VGC_COUNTER_MESHLETS_QUEUED];
  s->faults = c[VGC_COUNTER_ERROR];
  s->effective_threshold = threshold;
}

}  // namespace vgch

namespace {
constexpr double kNoDrawDistance = 1e30;  // GeometryPool.ts:111
}  // namespace

namespace vgch {

int dev_alloc(vgc_context *ctx, DevBuf &b, size_t bytes) {
  if (b.bytes >= bytes && b.ptr) return VGC_OK;
  size_t want = std::max<size_t>(bytes, 256);
  if (ctx->opts.hbm_budget_bytes && ctx->bytes - b.bytes + want > ctx->opts.hbm_budget_bytes)
    return fail(VGC_OVER_BUDGET, "allocation of " + std::to_string(want) + " bytes exceeds the context's HBM budget");
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(VGC_OOM, "cudaMalloc(" + std::to_string(want) + "): " + cudaGetErrorString(e));
  }
  if (b.ptr) {
    cudaFree(b.ptr);
    ctx->bytes -= b.bytes;
  }
  b.ptr = p;
  b.bytes = want;
  ctx->bytes += want;
  return VGC_OK;
}

void dev_free(vgc_context *ctx, DevBuf &b) {
  if (b.ptr) {
    cudaFree(b.ptr);
    ctx->bytes -= b.bytes;
  }
  b.ptr = nullptr;
  b.bytes = 0;
}

template <class T>
int upload(vgc_context *ctx, DevBuf &b, const std::vector<T> &v) {
  size_t bytes = v.size() * sizeof(T);
  if (bytes == 0) bytes = sizeof(T);
  int rc = dev_alloc(ctx, b, bytes + bytes / 2);  // grow ahead
  if (rc) return rc;
  if (!v.empty()) CUDA_TRY(cudaMemcpy(b.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return VGC_OK;
}

// Local meshlet ids in test order: each level's meshlets sorted by parent error (ties by id), levels in place. The
// meshlets of one DAG group share their parent error and parent sphere, so a group's meshlets are tested side by side
// (their parent-sphere reads hit the same lines).
void test_order(const vgc_mesh_data *d, std::vector<uint32_t> &order) {
  order.resize(d->meshlet_count);
  std::vector<std::pair<uint32_t, uint32_t>> keyed;
  for (uint32_t l = 0; l < d->level_count; l++) {
    const uint32_t f = d->level_ranges[l * 2], c = d->level_ranges[l * 2 + 1];
    keyed.clear();
    for (uint32_t i = f; i < f + c; i++) {
      const float e = d->meshlet_bounds[(size_t)i * 16 + 9];
      uint32_t key;  // non-negative floats order like their bit patterns; NaN sorts last, negatives first
      std::memcpy(&key, &e, 4);
      key = e != e ? 0xffffffffu : (e <= 0.0f ? 0u : key);
      keyed.emplace_back(key, i);
    }
    std::sort(keyed.begin(), keyed.end());
    for (uint32_t k = 0; k < c; k++) order[f + k] = keyed[k].second;
  }
}

int sync_scene(vgc_context *ctx) {
  if (!ctx->dirty) return VGC_OK;
  // buffers may be reallocated: no launch of any stream may still read the old ones
  CUDA_TRY(cudaDeviceSynchronize());
  int rc;
  if ((rc = upload(ctx, ctx->d_meshes, ctx->meshes))) return rc;
  if ((rc = upload(ctx, ctx->d_levels, ctx->levels))) return rc;
  if ((rc = upload(ctx, ctx->d_m_lod, ctx->m_lod))) return rc;
  if ((rc = upload(ctx, ctx->d_m_parent, ctx->m_parent))) return rc;
  if ((rc = upload(ctx, ctx->d_m_err, ctx->m_err))) return rc;
  if ((rc = upload(ctx, ctx->d_m_cull, ctx->m_cull))) return rc;
  if ((rc = upload(ctx, ctx->d_m_info, ctx->m_info))) return rc;
  if ((rc = upload(ctx, ctx->d_m_tris, ctx->m_tris))) return rc;
  if ((rc = upload(ctx, ctx->d_lsamples, ctx->lsamples))) return rc;
  if ((rc = upload(ctx, ctx->d_positions, ctx->positions))) return rc;
  if ((rc = upload(ctx, ctx->d_m_verts, ctx->m_verts))) return rc;
  if ((rc = upload(ctx, ctx->d_inst, ctx->inst))) return rc;
  if ((rc = upload(ctx, ctx->d_inst_slot, ctx->inst_slot))) return rc;
  if ((rc = upload(ctx, ctx->d_cells, ctx->cells))) return rc;
  ctx->dirty = false;
  return VGC_OK;
}

Scene scene_of(const vgc_context *ctx) {
  Scene S;
  S.meshes = (const MeshRec *)ctx->d_meshes.ptr;
  S.levels = (const LevelRec *)ctx->d_levels.ptr;
  S.m_lod = (const float4 *)ctx->d_m_lod.ptr;
  S.m_parent = (const float4 *)ctx->d_m_parent.ptr;
  S.m_err = (const float4 *)ctx->d_m_err.ptr;
  S.m_cull = (const float4 *)ctx->d_m_cull.ptr;
  S.m_info = (const uint4 *)ctx->d_m_info.ptr;
  S.m_tris = (const uint32_t *)ctx->d_m_tris.ptr;
  S.lsamples = (const float2 *)ctx->d_lsamples.ptr;
  S.positions = (const float4 *)ctx->d_positions.ptr;
  S.m_verts = (const uint32_t *)ctx->d_m_verts.ptr;
  S.inst = (const float4 *)ctx->d_inst.ptr;
  S.inst_slot = (const uint32_t *)ctx->d_inst_slot.ptr;
  S.cells = (const CellRec *)ctx->d_cells.ptr;
  S.hzbs = (const HzbDesc *)ctx->d_hzb_desc.ptr;
  S.cell_count = (uint32_t)ctx->cells.size();
  S.instance_count = (uint32_t)ctx->inst_slot.size();
  S.meshlet_count = (uint32_t)ctx->m_lod.size();
  S.slot_capacity = ctx->slot_capacity;
  S.slots_used = ctx->slots_used;
  return S;
}

// Output buffers for `slots` views, sized for the current mesh-slot capacity.
int ensure_outputs(vgc_context *ctx, uint32_t slots) {
  if (slots <= ctx->out_slots && ctx->out_slot_capacity == ctx->slot_capacity) return VGC_OK;
  CUDA_TRY(cudaDeviceSynchronize());
  uint32_t n = std::max(slots, ctx->out_slots);
  ctx->counter_words = VGC_COUNTER_HEADER + ctx->slot_capacity * 8;
  const size_t md = ctx->opts.max_meshlets;
  int rc;
  if ((rc = dev_alloc(ctx, ctx->d_counters, (size_t)n * ctx->counter_words * 4))) return rc;
  if ((rc = dev_alloc(ctx, ctx->d_draw, (size_t)n * 2 * md * 16))) return rc;
  if ((rc = dev_alloc(ctx, ctx->d_args, (size_t)n * 2 * ctx->slot_capacity * 2 * 5 * 4))) return rc;
  if ((rc = dev_alloc(ctx, ctx->d_dyn, (size_t)n * 8 * 4))) return rc;
  if ((rc = dev_alloc(ctx, ctx->d_hist, (size_t)n * 2 * kBudgetBins * 8))) return rc;
  CUDA_TRY(cudaMemset(ctx->d_counters.ptr, 0, (size_t)n * ctx->counter_words * 4));
  CUDA_TRY(cudaMemset(ctx->d_args.ptr, 0, (size_t)n * 2 * ctx->slot_capacity * 2 * 5 * 4));
  ctx->out_slots = n;
  ctx->out_slot_capacity = ctx->slot_capacity;
  return VGC_OK;
}

size_t output_slot_bytes(const vgc_context *ctx) {
  const size_t words = VGC_COUNTER_HEADER + (size_t)ctx->slot_capacity * 8;
  return words * 4 + 2 * (size_t)ctx->opts.max_meshlets * 16 + 2 * (size_t)ctx->slot_capacity * 2 * 5 * 4 + 8 * 4 +
         2 * kBudgetBins * 8 + kStateWords * 4;
}

int ensure_state(vgc_context *ctx, uint32_t slot) {
  if (slot < ctx->state_slots) return VGC_OK;
  uint32_t n = std::max<uint32_t>(slot + 1, ctx->state_slots * 2);
  n = std::max<uint32_t>(n, 16);
  std::vector<uint32_t> init((size_t)n * kStateWords, 0);
  for (uint32_t i = 0; i < n; i++) init[(size_t)i * kStateWords] = init[(size_t)i * kStateWords + 1] = 10000u;
  if (ctx->state_slots) {
    CUDA_TRY(cudaDeviceSynchronize());
    CUDA_TRY(cudaMemcpy(init.data(), ctx->d_state.ptr, (size_t)ctx->state_slots * kStateWords * 4, cudaMemcpyDeviceToHost));
  }
  DevBuf fresh;
  std::swap(fresh, ctx->d_state);
  ctx->bytes -= fresh.bytes;
  int rc = dev_alloc(ctx, ctx->d_state, init.size() * 4);
  if (fresh.ptr) cudaFree(fresh.ptr);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpy(ctx->d_state.ptr, init.data(), init.size() * 4, cudaMemcpyHostToDevice));
  ctx->state_slots = n;
  return VGC_OK;
}

// the unit list of `n` (view, cell) units and, after it, the overflow bits of its 4 n warp-units
static size_t unit_bytes(size_t n) { return n * sizeof(uint2) + (n * 4 + 31) / 32 * sizeof(uint32_t); }

int ensure_scratch(vgc_context *ctx, LaunchScratch &s, uint32_t views, size_t units) {
  if (!s.owner) s.owner = ctx;  // growth below is counted where the scratch was first counted
  ctx = s.owner;
  if (views > s.view_capacity) {
    if (s.h_views) cudaFreeHost(s.h_views);
    if (s.d_views) {
      cudaFree(s.d_views);
      ctx->bytes -= sizeof(ViewConst) * s.view_capacity;
    }
    if (s.h_plan) cudaFreeHost(s.h_plan);
    if (s.d_plan) {
      cudaFree(s.d_plan);
      ctx->bytes -= hzb_plan_bytes(s.view_capacity);
    }
    s.h_views = nullptr;
    s.d_views = nullptr;
    s.h_plan = s.d_plan = nullptr;
    s.view_capacity = 0;
    CUDA_TRY(cudaMallocHost(&s.h_views, sizeof(ViewConst) * views));
    CUDA_TRY(cudaMalloc(&s.d_views, sizeof(ViewConst) * views));
    CUDA_TRY(cudaMallocHost(&s.h_plan, hzb_plan_bytes(views)));
    CUDA_TRY(cudaMalloc(&s.d_plan, hzb_plan_bytes(views)));
    ctx->bytes += sizeof(ViewConst) * views + hzb_plan_bytes(views);
    s.plan_keys.assign(views, LaunchScratch::PlanKey{});
    s.plan_maps = 0;
    s.view_capacity = views;
  }
  if (units > s.unit_capacity || !s.d_units) {
    if (s.d_units) {
      cudaFree(s.d_units);
      ctx->bytes -= unit_bytes(s.unit_capacity);
    }
    s.d_units = nullptr;
    s.d_overflow = nullptr;
    size_t n = std::max<size_t>(units, 32);
    CUDA_TRY(cudaMalloc(&s.d_units, unit_bytes(n)));
    s.d_overflow = reinterpret_cast<uint32_t *>(s.d_units + n);
    CUDA_TRY(cudaMemset(s.d_overflow, 0, unit_bytes(n) - n * sizeof(uint2)));
    ctx->bytes += unit_bytes(n);
    s.unit_capacity = n;
  }
  if (!s.d_unit_count) CUDA_TRY(cudaMalloc(&s.d_unit_count, 64));
  // meshlet work queue: about one span per instance with a level range and cut, one chunk per 512 meshlets of a
  // warp's items. Sized for 64k entries per view; a warp that cannot reserve tests its items itself, so a full
  // queue costs time, not correctness.
  const uint32_t want_chunks = std::max<uint32_t>(std::max<uint32_t>(65536, views * 65536u), s.queue_want);
  if (want_chunks > s.chunk_capacity) {
    if (s.d_chunks) {
      cudaFree(s.d_chunks);
      ctx->bytes -= (size_t)s.chunk_capacity * sizeof(uint4);
    }
    s.d_chunks = nullptr;
    CUDA_TRY(cudaMalloc(&s.d_chunks, (size_t)want_chunks * sizeof(uint4)));
    ctx->bytes += (size_t)want_chunks * sizeof(uint4);
    s.chunk_capacity = want_chunks;
  }
  if (!s.done) CUDA_TRY(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
  if (!s.side) CUDA_TRY(cudaStreamCreateWithFlags(&s.side, cudaStreamNonBlocking));
  if (!s.fork) CUDA_TRY(cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming));
  if (!s.join) CUDA_TRY(cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming));
  if (!s.h_ctl) {
    CUDA_TRY(cudaMallocHost(&s.h_ctl, 64));
    std::memset(s.h_ctl, 0, 64);
  }
  return VGC_OK;
}

void free_scratch(LaunchScratch &s) {
  if (s.pending && s.done) cudaEventSynchronize(s.done);
  if (s.h_scenes) cudaFreeHost(s.h_scenes);
  if (s.d_scenes) cudaFree(s.d_scenes);
  if (s.h_views) cudaFreeHost(s.h_views);
  if (s.d_views) cudaFree(s.d_views);
  if (s.h_plan) cudaFreeHost(s.h_plan);
  if (s.d_plan) cudaFree(s.d_plan);
  if (s.d_units) cudaFree(s.d_units);
  if (s.d_unit_count) cudaFree(s.d_unit_count);
  if (s.d_chunks) cudaFree(s.d_chunks);
  if (s.h_ctl) cudaFreeHost(s.h_ctl);
  if (s.done) cudaEventDestroy(s.done);
  if (s.fork) cudaEventDestroy(s.fork);
  if (s.join) cudaEventDestroy(s.join);
  if (s.side) cudaStreamDestroy(s.side);
  s = LaunchScratch();
}

// Frustum planes of a column-major clip matrix, [0, 1] depth, normalised (Gribb & Hartmann plane extraction;
// three.js Frustum.setFromProjectionMatrix with WebGPUCoordinateSystem, VirtualGeometry.ts:429-437).
void planes_of(const double *me, double out[6][4]) {
  double p[6][4] = {
      {me[3] - me[0], me[7] - me[4], me[11] - me[8], me[15] - me[12]},
      {me[3] + me[0], me[7] + me[4], me[11] + me[8], me[15] + me[12]},
      {me[3] + me[1], me[7] + me[5], me[11] + me[9], me[15] + me[13]},
      {me[3] - me[1], me[7] - me[5], me[11] - me[9], me[15] - me[13]},
      {me[3] - me[2], me[7] - me[6], me[11] - me[10], me[15] - me[14]},
      {me[2], me[6], me[10], me[14]},
  };
  for (int i = 0; i < 6; i++) {
    double l = std::sqrt(p[i][0] * p[i][0] + p[i][1] * p[i][1] + p[i][2] * p[i][2]);
    double inv = l > 0 ? 1.0 / l : 0;
    for (int k = 0; k < 4; k++) out[i][k] = p[i][k] * inv;
  }
}

// Inverse of a rigid column-major 4x4 (rotation + translation): R^T and -R^T t.
void rigid_inverse(const double *m, double *out) {
  for (int c = 0; c < 3; c++)
    for (int r = 0; r < 3; r++) out[c * 4 + r] = m[r * 4 + c];
  for (int r = 0; r < 3; r++) {
    double s = 0;
    for (int i = 0; i < 3; i++) s += m[r * 4 + i] * m[12 + i];
    out[12 + r] = -s;
  }
  out[3] = out[7] = out[11] = 0;
  out[15] = 1;
}

// a * b, column-major 4x4
void mat4_mul(const double *a, const double *b, double *out) {
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) {
      double s = 0;
      for (int i = 0; i < 4; i++) s += a[i * 4 + r] * b[c * 4 + i];
      out[c * 4 + r] = s;
    }
}

HzbDesc hzb_layout(uint32_t width, uint32_t height, size_t *total_floats) {
  HzbDesc desc{};
  uint32_t lw = width, lh = height, n = 0;
  size_t total = 0;
  for (;;) {
    desc.off[n] = (uint32_t)total;
    desc.w[n] = lw;
    desc.h[n] = lh;
    total += (size_t)lw * lh;
    n++;
    if ((lw == 1 && lh == 1) || n == kMaxHzbLevels) break;
    lw = lw > 1 ? (lw + 1) / 2 : 1;
    lh = lh > 1 ? (lh + 1) / 2 : 1;
  }
  desc.levels = n;
  *total_floats = total;
  return desc;
}

// Allocates / lays out HZB slot `hzb` for a width x height mip 0 and publishes its descriptor; returns whether the
// device descriptor array changed (the caller uploads it).
// cuTensorMapEncodeTiled of the driver, found once through the runtime (the library does not link libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// The tensor map k_hzb_stream reads a float depth image through: 128 x 32 boxes, zeros past the image's edge. False
// (the plain loads then read the image) when the image breaks a bulk-tensor copy rule - base 16-byte aligned, row
// pitch a multiple of 16 bytes - or is smaller than a box.
bool depth_tensor_map(const float *depth, uint32_t w, uint32_t h, void *out) {
  const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode || (w & 3u) || (reinterpret_cast<uintptr_t>(depth) & 15u) || w < kHzbStripW || h < kHzbStripH)
    return false;
  const cuuint64_t dims[2] = {w, h}, pitch[1] = {(cuuint64_t)w * 4};
  const cuuint32_t box[2] = {kHzbStripW, kHzbStripH}, step[2] = {1, 1};
  return encode(static_cast<CUtensorMap *>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(depth), dims,
                pitch, box, step, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The HZB plan of the prepared views in `s.h_plan`: one job per view that brings a depth image, strips in view order.
// A tensor map is encoded again only when its job's image changed since the last launch of this scratch.
void build_hzb_plan(vgc_context *ctx, LaunchScratch &s, const vgc_view *views, uint32_t count) {
  HzbPlanHead &P = *reinterpret_cast<HzbPlanHead *>(s.h_plan);
  HzbJob *jobs = reinterpret_cast<HzbJob *>(s.h_plan + sizeof(HzbPlanHead));
  const size_t maps = hzb_plan_maps(count);
  if (s.plan_maps != maps) {
    s.plan_keys.assign(s.view_capacity, LaunchScratch::PlanKey{});
    s.plan_maps = maps;
  }
  uint32_t n = 0, tiles = 0;
  for (uint32_t i = 0; i < count; i++) {
    const vgc_view &v = views[i];
    if (v.hzb < 0 || !v.depth) continue;
    const uint32_t w = v.depth_width, h = v.depth_height;
    const uint32_t tx = (w + kHzbStripW - 1) / kHzbStripW, ty = (h + kHzbStripH - 1) / kHzbStripH;
    LaunchScratch::PlanKey &key = s.plan_keys[n];
    if (key.depth != v.depth || key.w != w || key.h != h) {
      key.depth = v.depth;
      key.w = w;
      key.h = h;
      key.tma = depth_tensor_map(v.depth, w, h, s.h_plan + maps + (size_t)n * kTensorMapBytes) ? 1u : 0u;
    }
    HzbJob &J = jobs[n++];
    J.depth = v.depth;
    J.desc = (const HzbDesc *)ctx->d_hzb_desc.ptr + v.hzb;
    J.error = s.h_views[i].counters + VGC_COUNTER_ERROR;
    J.tile0 = tiles;
    J.tiles_x = (uint16_t)tx;
    J.tma = (uint8_t)key.tma;
    J.copy_mip0 = s.h_views[i].hzb_mip0 == nullptr ? 1 : 0;
    tiles += tx * ty;
  }
  std::memset(&P, 0, sizeof P);
  P.jobs = n;
  P.tiles = tiles;
  P.maps = (uint32_t)maps;
}

int hzb_prepare(vgc_context *ctx, int32_t hzb, uint32_t width, uint32_t height, bool *changed) {
  if (width == 0 || height == 0 || width > 32768 || height > 32768) return fail(VGC_INVALID_ARG, "HZB size out of range");
  size_t total = 0;
  HzbDesc desc = hzb_layout(width, height, &total);
  auto &h = ctx->hzb[hzb];
  if (h.data.bytes < total * 4) {
    CUDA_TRY(cudaDeviceSynchronize());
    int rc = dev_alloc(ctx, h.data, total * 4);
    if (rc) return rc;
  }
  desc.data = (const float *)h.data.ptr;
  *changed = !h.valid || std::memcmp(&desc, &h.desc, sizeof desc) != 0;
  h.desc = desc;
  h.valid = true;
  return VGC_OK;
}

int view_constants(vgc_context *ctx, const vgc_view &in, uint32_t out_slot, uint32_t unit_offset, ViewConst &k) {
  if (!(in.viewport_height > 0) || !(in.error_threshold > 0) || !(in.near_ > 0))
    return fail(VGC_INVALID_ARG, "view: viewport_height, error_threshold and near must be > 0");
  if (in.hzb >= (int32_t)vgc_context::kHzbSlots) return fail(VGC_INVALID_ARG, "view: hzb slot out of range");
  if (in.hzb >= 0 && !in.depth && !ctx->hzb[in.hzb].valid)
    return fail(VGC_INVALID_ARG, "view: hzb slot " + std::to_string(in.hzb) + " has no HZB and the view brings no depth");
  int rc = ensure_state(ctx, in.state_slot);
  if (rc) return rc;
  std::memset(&k, 0, sizeof k);
  double pvm[16];
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) {
      double s = 0;
      for (int i = 0; i < 4; i++) s += in.proj[i * 4 + r] * in.view[c * 4 + i];
      pvm[c * 4 + r] = s;
    }
  double pv[6][4], pw[6][4];
  planes_of(in.proj, pv);
  planes_of(pvm, pw);
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 4; c++) k.V[r * 4 + c] = (float)in.view[c * 4 + r];
  const bool cascade = (in.flags & VGC_VIEW_CASCADE) != 0;
  if (cascade) {
    if (in.triangle_budget > 0) return fail(VGC_INVALID_ARG, "view: a cascade has no camera cut to budget");
    // the cascade's planes in camera view space: clip = C * V^-1 * x_view
    double vinv[16], cm[16];
    rigid_inverse(in.view, vinv);
    mat4_mul(in.cascade_clip, vinv, cm);
    planes_of(cm, pv);
  }
  for (int p = 0; p < 6; p++) {
    for (int i = 0; i < 4; i++) k.plane[p * 4 + i] = (float)pv[p][i];
    double d = pw[p][0] * in.shadow_sweep[0] + pw[p][1] * in.shadow_sweep[1] + pw[p][2] * in.shadow_sweep[2];
    k.sweep[p] = cascade ? 0.0f : (float)(d > 0 ? d : 0);
  }
  k.cascade = cascade ? 1u : 0u;
  k.proj_scale = (float)(in.proj[5] * in.viewport_height * 0.5);
  k.inv_proj_scale = (float)(1.0 / (in.proj[5] * in.viewport_height * 0.5));
  k.near_ = (float)in.near_;
  k.P0 = (float)in.proj[0];
  k.P5 = (float)in.proj[5];
  k.P8 = (float)in.proj[8];
  k.P9 = (float)in.proj[9];
  k.P10 = (float)in.proj[10];
  k.P14 = (float)in.proj[14];
  k.error_threshold = (float)in.error_threshold;
  k.lod_blend_max = (float)(in.lod_blend > 1 ? in.lod_blend : 1);
  double limit = in.max_error_threshold / in.error_threshold;
  k.lod_scale_limit = (float)(limit > 1 ? limit : 1);
  k.min_pixel_radius = (float)in.min_pixel_radius;
  k.shadow_error_scale = (float)in.shadow_error_scale;
  k.budget = (float)(in.triangle_budget > 0 ? in.triangle_budget : 0);
  k.budget_tris = in.triangle_budget > 0 ? (unsigned long long)in.triangle_budget : 0ull;
  if (in.triangle_budget > 0 && !(in.threshold_range[0] > 0 && in.threshold_range[1] > in.threshold_range[0]))
    return fail(VGC_INVALID_ARG, "view: triangle_budget needs 0 < threshold_range[0] < threshold_range[1]");
  k.budget_lo = (float)in.threshold_range[0];
  k.budget_hi = (float)in.threshold_range[1];
  k.frustum = in.frustum_culling ? 1u : 0u;
  k.occl_active = in.hzb >= 0 ? 1u : 0u;
  k.hzb = in.hzb;
  k.hzb_desc = in.hzb >= 0 ? (const HzbDesc *)ctx->d_hzb_desc.ptr + in.hzb : nullptr;
  k.scene = 0;
  k.slot_capacity = ctx->slot_capacity;
  k.slots_used = ctx->slots_used;
  k.counter_words = VGC_COUNTER_HEADER + ctx->slot_capacity * 8;
  k.build_hzb = (in.hzb >= 0 && in.depth) ? 1u : 0u;
  k.fresh_state = (in.flags & VGC_VIEW_FRESH_STATE) ? 1u : 0u;
  k.depth = in.depth;
  k.hzb_mip0 = (k.build_hzb && (in.flags & VGC_VIEW_DEPTH_AS_MIP0)) ? in.depth : nullptr;
  k.unit_offset = unit_offset;
  k.max_drawn = ctx->opts.max_meshlets;
  k.index_capacity[0] = ctx->opts.max_triangles * 3;
  k.index_capacity[1] = ctx->opts.max_shadow_triangles * 3;
  k.counters = (uint32_t *)ctx->d_counters.ptr + (size_t)out_slot * ctx->counter_words;
  k.state = (uint32_t *)ctx->d_state.ptr + (size_t)in.state_slot * kStateWords;
  k.draw_list = (uint4 *)ctx->d_draw.ptr + (size_t)out_slot * 2 * ctx->opts.max_meshlets;
  k.draw_args = (uint32_t *)ctx->d_args.ptr + (size_t)out_slot * 2 * ctx->slot_capacity * 2 * 5;
  k.dyn = (float *)ctx->d_dyn.ptr + (size_t)out_slot * 8;
  k.hist = (unsigned long long *)ctx->d_hist.ptr + (size_t)out_slot * 2 * kBudgetBins;
  return VGC_OK;
}

// Prepares scene, outputs and the views' constants in `s.h_views` (pinned).
int prepare(vgc_context *ctx, LaunchScratch &s, const vgc_view *views, uint32_t count, uint32_t first_slot,
            const uint32_t *slots) {
  if (!views || count == 0) return fail(VGC_INVALID_ARG, "no views");
  int rc = sync_scene(ctx);
  if (rc) return rc;
  uint32_t slot_end = first_slot + count;
  if (slots) {
    slot_end = 0;
    for (uint32_t i = 0; i < count; i++) slot_end = std::max(slot_end, slots[i] + 1);
  }
  if ((rc = ensure_outputs(ctx, slot_end))) return rc;
  if (s.pending) CUDA_TRY(cudaEventSynchronize(s.done));
  s.pending = false;
  if (s.h_ctl) {  // the last sequence's peak queue demand (spans take 3/4 of the entries, chunks 1/4), plus 25%
    const uint64_t need = std::max<uint64_t>((uint64_t)s.h_ctl[6] * 4 / 3, (uint64_t)s.h_ctl[7] * 4) * 5 / 4;
    if (need > s.chunk_capacity) s.queue_want = (uint32_t)std::min<uint64_t>((need + 65535) & ~65535ull, 1u << 28);
  }
  const uint32_t cells = pad32((uint32_t)ctx->cells.size());
  if ((rc = ensure_scratch(ctx, s, count, (size_t)count * cells))) return rc;
  s.multi = false;
  s.units_total = (size_t)count * cells;
  bool changed = false;
  s.hzb_w = s.hzb_h = 0;
  s.hzb_tail = false;
  s.any_budget = false;
  for (uint32_t i = 0; i < count; i++) s.any_budget = s.any_budget || views[i].triangle_budget > 0;
  for (uint32_t i = 0; i < count; i++) {
    const vgc_view &v = views[i];
    if (v.hzb >= 0 && v.depth) {
      for (uint32_t j = 0; j < i; j++)
        if (views[j].hzb == v.hzb && views[j].depth) return fail(VGC_INVALID_ARG, "two views build the same HZB slot");
      bool c = false;
      if ((rc = hzb_prepare(ctx, v.hzb, v.depth_width, v.depth_height, &c))) return rc;
      changed = changed || c;
      s.hzb_w = std::max(s.hzb_w, v.depth_width);
      s.hzb_h = std::max(s.hzb_h, v.depth_height);
      // the tail kernel builds levels 5+ after the strip stream (7+ after the per-view tile kernel)
      s.hzb_tail = s.hzb_tail || ctx->hzb[v.hzb].desc.levels > (ctx->hzb_grid ? 5u : 7u);
    }
  }
  if (changed) {
    std::vector<HzbDesc> all(vgc_context::kHzbSlots);
    for (uint32_t i = 0; i < vgc_context::kHzbSlots; i++) all[i] = ctx->hzb[i].desc;
    CUDA_TRY(cudaMemcpy(ctx->d_hzb_desc.ptr, all.data(), sizeof(HzbDesc) * all.size(), cudaMemcpyHostToDevice));
  }
  for (uint32_t i = 0; i < count; i++)
    if ((rc = view_constants(ctx, views[i], slots ? slots[i] : first_slot + i, i * cells, s.h_views[i]))) return rc;
  if (s.hzb_w) build_hzb_plan(ctx, s, views, count);
  return VGC_OK;
}

cudaEvent_t prof_event(vgc_context *ctx) {
  if (!ctx->prof_free.empty()) {
    cudaEvent_t e = ctx->prof_free.back();
    ctx->prof_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Runs `launch` between two events on `st` when profiling is on (never inside a graph capture).
template <class F>
cudaError_t timed(vgc_context *ctx, bool capture, int kind, cudaStream_t st, F &&launch) {
  if (!ctx->profiling || capture) return launch();
  cudaEvent_t a = prof_event(ctx), b = prof_event(ctx);
  cudaEventRecord(a, st);
  cudaError_t e = launch();
  cudaEventRecord(b, st);
  ctx->prof_pending.push_back({kind, {a, b}});
  return e;
}

// The launch sequence of one frame: reset, cells, then select + finish for the first round and two retry rounds
// (GeometryPool.ts:1081-1092 without the dispatch-argument kernels, which persistent launches do not need).
int prepare_multi(vgc_context *const *ctxs, uint32_t nctx, LaunchScratch &s, const vgc_view *views,
                  const uint32_t *scene, uint32_t count, const uint32_t *slots) {
  if (!ctxs || nctx == 0 || !views || !scene || !slots || count == 0) return fail(VGC_INVALID_ARG, "no views");
  std::vector<uint32_t> slot_end(nctx, 0);
  for (uint32_t i = 0; i < count; i++) {
    if (scene[i] >= nctx) return fail(VGC_INVALID_ARG, "view scene index out of range");
    if (views[i].depth) return fail(VGC_INVALID_ARG, "a multi-scene launch takes built HZB slots, not depth images");
    slot_end[scene[i]] = std::max(slot_end[scene[i]], slots[i] + 1);
  }
  int rc;
  size_t units = 0;
  for (uint32_t k = 0; k < nctx; k++) {
    if ((rc = sync_scene(ctxs[k]))) return rc;
    if (slot_end[k] && (rc = ensure_outputs(ctxs[k], slot_end[k]))) return rc;
  }
  for (uint32_t i = 0; i < count; i++) units += pad32((uint32_t)ctxs[scene[i]]->cells.size());
  if (s.pending) CUDA_TRY(cudaEventSynchronize(s.done));
  s.pending = false;
  if (s.h_ctl) {  // the last sequence's peak queue demand, as in prepare
    const uint64_t need = std::max<uint64_t>((uint64_t)s.h_ctl[6] * 4 / 3, (uint64_t)s.h_ctl[7] * 4) * 5 / 4;
    if (need > s.chunk_capacity) s.queue_want = (uint32_t)std::min<uint64_t>((need + 65535) & ~65535ull, 1u << 28);
  }
  if ((rc = ensure_scratch(ctxs[0], s, count, units))) return rc;
  if (nctx > s.scene_capacity) {
    vgc_context *owner = s.owner ? s.owner : ctxs[0];
    if (s.h_scenes) cudaFreeHost(s.h_scenes);
    if (s.d_scenes) {
      cudaFree(s.d_scenes);
      owner->bytes -= sizeof(Scene) * s.scene_capacity;
    }
    s.h_scenes = nullptr;
    s.d_scenes = nullptr;
    s.scene_capacity = 0;
    CUDA_TRY(cudaMallocHost(&s.h_scenes, sizeof(Scene) * nctx));
    CUDA_TRY(cudaMalloc(&s.d_scenes, sizeof(Scene) * nctx));
    owner->bytes += sizeof(Scene) * nctx;
    s.scene_capacity = nctx;
  }
  for (uint32_t k = 0; k < nctx; k++) s.h_scenes[k] = scene_of(ctxs[k]);
  s.scene_count = nctx;
  s.multi = true;
  s.units_total = units;
  s.hzb_w = s.hzb_h = 0;
  s.hzb_tail = false;
  s.any_budget = false;
  uint32_t offset = 0;
  for (uint32_t i = 0; i < count; i++) {
    vgc_context *ctx = ctxs[scene[i]];
    s.any_budget = s.any_budget || views[i].triangle_budget > 0;
    if ((rc = view_constants(ctx, views[i], slots[i], offset, s.h_views[i]))) return rc;
    s.h_views[i].scene = scene[i];
    offset += pad32((uint32_t)ctx->cells.size());
  }
  return VGC_OK;
}

int enqueue(vgc_context *ctx, LaunchScratch &s, uint32_t count, cudaStream_t st, bool capture) {
  const Scene S = scene_of(ctx);
  const Scene *scenes = s.multi ? s.d_scenes : nullptr;
  const uint32_t select_grid = s.grid_instances ? s.grid_instances : ctx->select_grid;
  const uint32_t chunk_grid = s.grid_chunks ? s.grid_chunks : ctx->chunk_grid;
  CUDA_TRY(cudaMemcpyAsync(s.d_views, s.h_views, sizeof(ViewConst) * count, cudaMemcpyHostToDevice, st));
  if (s.multi) CUDA_TRY(cudaMemcpyAsync(s.d_scenes, s.h_scenes, sizeof(Scene) * s.scene_count, cudaMemcpyHostToDevice, st));
  if (s.hzb_w && ctx->hzb_grid)
    CUDA_TRY(cudaMemcpyAsync(s.d_plan, s.h_plan, hzb_plan_bytes(count), cudaMemcpyHostToDevice, st));
  CUDA_TRY(timed(ctx, capture, VGC_KERNEL_RESET, st,
                 [&] { return launch_reset(s.d_views, count, s.d_unit_count, st); }));
  // the HZB build (after the reset, which clears the counter word a failed wait of the build reports in) and the
  // cell pass do not depend on each other: the cell pass runs on a second stream beside the build (a parallel branch
  // of the captured graph), submitted after it so that the build's persistent blocks are resident first, and joins
  // before the instance pass
  if (s.hzb_w) {
    CUDA_TRY(cudaEventRecord(s.fork, st));
    CUDA_TRY(cudaStreamWaitEvent(s.side, s.fork, 0));
    CUDA_TRY(timed(ctx, capture, VGC_KERNEL_HZB, st, [&] {
      return ctx->hzb_grid ? launch_hzb_stream(s.d_plan, ctx->hzb_grid, s.d_views, count, s.hzb_tail, st)
                           : launch_hzb_views(s.d_views, count, s.hzb_w, s.hzb_h, s.hzb_tail, st);
    }));
  }
  const cudaStream_t cells_st = s.hzb_w ? s.side : st;
  CUDA_TRY(timed(ctx, capture, VGC_KERNEL_CELLS, cells_st, [&] {
    return launch_cells(S, scenes, s.d_views, count, s.units_total, s.d_units, s.d_unit_count, cells_st);
  }));
  if (s.hzb_w) {
    CUDA_TRY(cudaEventRecord(s.join, s.side));
    CUDA_TRY(cudaStreamWaitEvent(st, s.join, 0));
  }
  const uint32_t redo_grid = (uint32_t)ctx->sm_count * 2;
  if (s.any_budget) {  // the triangleBudget search: histogram pass, then the threshold of each budget view
    CUDA_TRY(timed(ctx, capture, VGC_KERNEL_BUDGET, st, [&] {
      cudaError_t e = launch_instances(S, scenes, s.d_views, s.d_units, s.d_unit_count, s.d_chunks, s.chunk_capacity, -1,
                                       select_grid, s.d_overflow, st, s.chunk_shift);
      if (e == cudaSuccess)
        e = launch_chunks(S, scenes, s.d_views, s.d_chunks, s.d_unit_count, s.chunk_capacity, -1, chunk_grid, st);
      if (e == cudaSuccess)
        e = launch_instances_redo(S, scenes, s.d_views, s.d_units, s.d_unit_count, s.d_chunks, s.chunk_capacity, -1,
                                  s.d_overflow, redo_grid, st, s.chunk_shift);
      if (e == cudaSuccess) e = launch_budget(s.d_views, count, s.d_unit_count, st);
      return e;
    }));
  }
  for (int round = 0; round < 3; round++) {
    const uint32_t shift = round > 0 && kChunkShiftRetry ? kChunkShiftRetry : s.chunk_shift;
    CUDA_TRY(timed(ctx, capture, round == 0 ? VGC_KERNEL_SELECT0 : VGC_KERNEL_SELECT_RETRY, st, [&] {
      return launch_instances(S, scenes, s.d_views, s.d_units, s.d_unit_count, s.d_chunks, s.chunk_capacity, round,
                              select_grid, s.d_overflow, st, shift);
    }));
    CUDA_TRY(timed(ctx, capture, round == 0 ? VGC_KERNEL_CHUNKS0 : VGC_KERNEL_SELECT_RETRY, st, [&] {
      return launch_chunks(S, scenes, s.d_views, s.d_chunks, s.d_unit_count, s.chunk_capacity, round, chunk_grid, st);
    }));
    // units whose items did not fit the queue (returns at once when there are none)
    CUDA_TRY(timed(ctx, capture, VGC_KERNEL_SELECT_RETRY, st, [&] {
      return launch_instances_redo(S, scenes, s.d_views, s.d_units, s.d_unit_count, s.d_chunks, s.chunk_capacity,
                                   round, s.d_overflow, redo_grid, st, shift);
    }));
    CUDA_TRY(timed(ctx, capture, VGC_KERNEL_FINISH, st, [&] {
      return launch_finish(s.d_views, count, s.d_unit_count, round, st);
    }));
  }
  // control words (peak queue demand) for the next prepare
  CUDA_TRY(cudaMemcpyAsync(s.h_ctl, s.d_unit_count, 64, cudaMemcpyDeviceToHost, st));
  return VGC_OK;
}

void compute_cell(vgc_context *ctx, uint32_t slot, uint32_t cell) {
  // Bounding sphere of one cell's instances (GeometryPool.ts:519-545): the box of the instances' world spheres
  // gives the centre, the radius reaches every instance sphere, and both radii are inflated so float rounding on
  // the GPU cannot make the cell test stricter than the per-instance test.
  const MeshHost &m = ctx->mesh_host[slot];
  const uint32_t first = cell * kCellSize, end = std::min(first + kCellSize, m.instance_count);
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  double max_radius = 0;
  std::vector<double> sph((size_t)(end - first) * 4);
  for (uint32_t g = first; g < end; g++) {
    const float4 *c = &ctx->inst[(size_t)(m.instance_base + g) * 4];
    const double sx = m.sphere[0], sy = m.sphere[1], sz = m.sphere[2], sr = m.sphere[3];
    double *s = &sph[(size_t)(g - first) * 4];
    s[0] = c[0].x * sx + c[1].x * sy + c[2].x * sz + c[3].x;
    s[1] = c[0].y * sx + c[1].y * sy + c[2].y * sz + c[3].y;
    s[2] = c[0].z * sx + c[1].z * sy + c[2].z * sz + c[3].z;
    const double c0 = std::sqrt((double)c[0].x * c[0].x + (double)c[0].y * c[0].y + (double)c[0].z * c[0].z);
    const double c1 = std::sqrt((double)c[1].x * c[1].x + (double)c[1].y * c[1].y + (double)c[1].z * c[1].z);
    const double c2 = std::sqrt((double)c[2].x * c[2].x + (double)c[2].y * c[2].y + (double)c[2].z * c[2].z);
    s[3] = sr * std::max(c0, std::max(c1, c2));
    for (int a = 0; a < 3; a++) {
      lo[a] = std::min(lo[a], s[a] - s[3]);
      hi[a] = std::max(hi[a], s[a] + s[3]);
    }
    max_radius = std::max(max_radius, s[3]);
  }
  const double cx = (lo[0] + hi[0]) / 2, cy = (lo[1] + hi[1]) / 2, cz = (lo[2] + hi[2]) / 2;
  double radius = 0;
  for (uint32_t g = first; g < end; g++) {
    const double *s = &sph[(size_t)(g - first) * 4];
    radius = std::max(radius, std::sqrt((s[0] - cx) * (s[0] - cx) + (s[1] - cy) * (s[1] - cy) + (s[2] - cz) * (s[2] - cz)) + s[3]);
  }
  CellRec &r = ctx->cells[m.cell_base + cell];
  r.sphere = make_float4((float)cx, (float)cy, (float)cz, (float)(radius * (1 + 1e-4) + 1e-3));
  r.max_radius = (float)(max_radius * (1 + 1e-4) + 1e-4);
  r.slot = slot;
  r.first = m.instance_base + first;
  r.count = end - first;
}

uint32_t spread10(uint32_t v) {
  v &= 0x3ff;
  uint32_t r = 0;
  for (int b = 0; b < 10; b++) r |= ((v >> b) & 1u) << (3 * b);
  return r;
}

// 30-bit Morton order of the instance sphere centres, stable (GeometryPool.ts:1263-1311).
void morton_order(const float *m, uint32_t n, const float *sphere, std::vector<uint32_t> &order) {
  std::vector<double> c((size_t)n * 3);
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = 0; i < n; i++) {
    const float *e = m + (size_t)i * 16;
    const double sx = sphere[0], sy = sphere[1], sz = sphere[2];
    const double p[3] = {e[0] * sx + e[4] * sy + e[8] * sz + e[12], e[1] * sx + e[5] * sy + e[9] * sz + e[13],
                         e[2] * sx + e[6] * sy + e[10] * sz + e[14]};
    for (int a = 0; a < 3; a++) {
      c[(size_t)i * 3 + a] = p[a];
      lo[a] = std::min(lo[a], p[a]);
      hi[a] = std::max(hi[a], p[a]);
    }
  }
  const double extent = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-9});
  std::vector<std::pair<uint32_t, uint32_t>> keys(n);
  for (uint32_t i = 0; i < n; i++) {
    uint32_t q[3];
    for (int a = 0; a < 3; a++) {
      double f = std::floor((c[(size_t)i * 3 + a] - lo[a]) / extent * 1024.0);
      q[a] = (uint32_t)std::min(1023.0, std::max(0.0, f));
    }
    keys[i] = {spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2), i};
  }
  std::stable_sort(keys.begin(), keys.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
  order.resize(n);
  for (uint32_t i = 0; i < n; i++) order[i] = keys[i].second;
}

// A changed mesh record goes to the device at once when the scene is resident (after every launch that may still
// read it); otherwise the pending full upload carries it.
int publish_mesh_record(vgc_context *ctx, uint32_t slot) {
  if (ctx->dirty || !ctx->d_meshes.ptr) {
    ctx->dirty = true;
    return VGC_OK;
  }
  cudaSetDevice(ctx->device);
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy((MeshRec *)ctx->d_meshes.ptr + slot, &ctx->meshes[slot], sizeof(MeshRec), cudaMemcpyHostToDevice));
  return VGC_OK;
}

void write_flags(vgc_context *ctx, uint32_t slot, const vgc_mesh_opts *o) {
  MeshRec &r = ctx->meshes[slot];
  double dd = o ? o->max_draw_distance : 0;
  r.max_draw_distance = (float)((dd > 0 && dd < kNoDrawDistance) ? dd : kNoDrawDistance);
  r.min_pixel_radius = o ? std::max(0.0f, o->min_pixel_radius) : 0.0f;
  r.enabled = o ? (o->enabled ? 1u : 0u) : 1u;
  r.shadow = o ? (o->shadow ? 1u : 0u) : 0u;
  r.occlusion = o ? (o->occlusion ? 1u : 0u) : 0u;
  r.occluder = (o && o->occluder && ctx->mesh_host[slot].vertex_count) ? 1u : 0u;
  r.vertices = ctx->mesh_host[slot].vertex_count ? 1u : 0u;
}

}  // namespace vgch

extern "C" {

const char *vgc_last_error(void) { return g_error.c_str(); }
const char *vgc_version(void) { return "vgcut 0.1.0 (sm_100a)"; }

void vgc_default_options(vgc_options *o) {
  o->max_triangles = 10000000;
  o->max_shadow_triangles = 4000000;
  o->max_meshlets = 1u << 20;
  o->output_slots = 1;
  o->device = 0;
  o->hbm_budget_bytes = 0;
}

int vgc_context_create(const vgc_options *opts, vgc_context **out) {
  if (!out) return fail(VGC_INVALID_ARG, "out is null");
  *out = nullptr;
  vgc_options o;
  vgc_default_options(&o);
  if (opts) o = *opts;
  if (o.max_meshlets == 0 || o.max_meshlets > (1u << 24)) return fail(VGC_INVALID_ARG, "max_meshlets must be in [1, 2^24]");
  if (o.max_triangles == 0 || o.max_shadow_triangles == 0) return fail(VGC_INVALID_ARG, "triangle capacities must be > 0");
  if (o.max_triangles > 0x55555555u || o.max_shadow_triangles > 0x55555555u)
    return fail(VGC_INVALID_ARG, "triangle capacities must fit 32-bit index counts");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(VGC_DEVICE_ERROR, "no CUDA device: the cut engine has no CPU fallback");
  }
  if (o.device < 0 || o.device >= ndev) return fail(VGC_INVALID_ARG, "device ordinal out of range");
  vgc_context *ctx = new vgc_context();
  ctx->opts = o;
  ctx->device = o.device;
  cudaSetDevice(o.device);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, o.device);
  ctx->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return fail(VGC_DEVICE_ERROR, "cudaStreamCreate failed");
  }
  int per_sm = 0, chunks_per_sm = 0;
  if (configure_select(false, &per_sm, &chunks_per_sm) != cudaSuccess) {
    cudaGetLastError();
    per_sm = chunks_per_sm = 1;
  }
  ctx->select_grid = (uint32_t)std::max(1, per_sm) * ctx->sm_count;
  ctx->chunk_grid = (uint32_t)std::max(1, chunks_per_sm) * ctx->sm_count;
  ctx->hzb_grid = hzb_stream_blocks_per_sm() * ctx->sm_count;
  cudaGetLastError();
  ctx->meshes.resize(ctx->slot_capacity);
  ctx->mesh_host.resize(ctx->slot_capacity);
  ctx->hzb.resize(vgc_context::kHzbSlots);
  int rc = dev_alloc(ctx, ctx->d_hzb_desc, sizeof(HzbDesc) * vgc_context::kHzbSlots);
  if (!rc) rc = ensure_outputs(ctx, std::max<uint32_t>(1, o.output_slots));
  if (!rc) rc = ensure_state(ctx, 0);
  if (rc) {
    vgc_context_destroy(ctx);
    return rc;
  }
  cudaMemset(ctx->d_hzb_desc.ptr, 0, sizeof(HzbDesc) * vgc_context::kHzbSlots);
  *out = ctx;
  return VGC_OK;
}

int vgc_context_destroy(vgc_context *ctx) {
  if (!ctx) return VGC_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_scratch(ctx->scratch);
  for (DevBuf *b : {&ctx->d_meshes, &ctx->d_levels, &ctx->d_m_lod, &ctx->d_m_parent, &ctx->d_m_err, &ctx->d_m_cull,
                    &ctx->d_lsamples, &ctx->d_positions, &ctx->d_m_verts, &ctx->d_raster, &ctx->d_resort,
                    &ctx->d_m_info, &ctx->d_m_tris, &ctx->d_inst, &ctx->d_inst_slot, &ctx->d_cells, &ctx->d_counters,
                    &ctx->d_draw, &ctx->d_args, &ctx->d_dyn, &ctx->d_hist, &ctx->d_state, &ctx->d_hzb_desc})
    dev_free(ctx, *b);
  for (auto &h : ctx->hzb) dev_free(ctx, h.data);
  for (auto &p : ctx->prof_pending) {
    cudaEventDestroy(p.second.first);
    cudaEventDestroy(p.second.second);
  }
  for (cudaEvent_t e : ctx->prof_free) cudaEventDestroy(e);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return VGC_OK;
}

int vgc_context_footprint(const vgc_context *ctx, uint64_t *bytes) {
  if (!ctx || !bytes) return fail(VGC_INVALID_ARG, "null argument");
  *bytes = ctx->bytes;
  return VGC_OK;
}

int vgc_mesh_add(vgc_context *ctx, const vgc_mesh_data *d, const float *matrices, uint32_t n, const vgc_mesh_opts *opts,
                 uint32_t *slot_out, uint32_t *gpu_to_input) {
  if (!ctx || !d || !slot_out) return fail(VGC_INVALID_ARG, "null argument");
  if (n && !matrices) return fail(VGC_INVALID_ARG, "matrices is null");
  if (!d->meshlet_bounds || !d->meshlet_info || !d->level_ranges || !d->level_errors || !d->level_guard_errors)
    return fail(VGC_INVALID_ARG, "mesh data arrays missing");
  if (d->meshlet_count == 0 || d->level_count == 0) return fail(VGC_INVALID_ARG, "mesh has no meshlets or levels");
  if (d->level_count > kMaxLevels) return fail(VGC_INVALID_ARG, "mesh has more than 48 LOD levels");
  // validate the level table against the meshlets (meshlets sorted by level, levels contiguous)
  uint32_t expect = 0;
  for (uint32_t l = 0; l < d->level_count; l++) {
    if (d->level_ranges[l * 2] != expect) return fail(VGC_INVALID_ARG, "level_ranges are not contiguous from 0");
    expect += d->level_ranges[l * 2 + 1];
  }
  if (expect != d->meshlet_count) return fail(VGC_INVALID_ARG, "level_ranges do not cover meshlet_count");
  uint64_t tri_total = 0;
  for (uint32_t i = 0; i < d->meshlet_count; i++) {
    const uint32_t tc = d->meshlet_info[(size_t)i * 4];
    if (tc == 0 || tc > 128) return fail(VGC_INVALID_ARG, "meshlet triangle count outside 1..128");
    tri_total += tc;
  }
  // every index the kernels follow must stay inside the arrays: triangles (expand, occluder pass), vertices
  const bool has_vertices = d->positions || d->meshlet_vertices;
  if (has_vertices && (!d->positions || !d->meshlet_vertices || !d->vertex_count || !d->meshlet_vertex_count ||
                       !d->meshlet_triangles))
    return fail(VGC_INVALID_ARG, "vertex data needs positions, meshlet_vertices and meshlet_triangles");
  if (d->meshlet_triangles)
    for (uint32_t i = 0; i < d->meshlet_count; i++) {
      const uint32_t *info = d->meshlet_info + (size_t)i * 4;
      if (info[1] % 3 || (uint64_t)info[1] / 3 + info[0] > d->meshlet_triangle_count)
        return fail(VGC_INVALID_ARG, "meshlet " + std::to_string(i) + ": triangles outside meshlet_triangles");
      if (!has_vertices) continue;
      uint32_t top = 0;
      for (uint32_t t = 0; t < info[0]; t++) {
        const uint32_t p = d->meshlet_triangles[info[1] / 3 + t];
        top = std::max(top, std::max(p & 255u, std::max((p >> 8) & 255u, (p >> 16) & 255u)));
      }
      if ((uint64_t)info[3] + top >= d->meshlet_vertex_count)
        return fail(VGC_INVALID_ARG, "meshlet " + std::to_string(i) + ": vertices outside meshlet_vertices");
    }
  if (has_vertices)
    for (uint32_t i = 0; i < d->meshlet_vertex_count; i++)
      if (d->meshlet_vertices[i] >= d->vertex_count) return fail(VGC_INVALID_ARG, "meshlet_vertices id out of range");
  std::lock_guard<std::mutex> lock(ctx->mu);
  uint32_t slot = 0;
  while (slot < ctx->slots_used && ctx->mesh_host[slot].used) slot++;
  if (slot >= ctx->slot_capacity) {
    uint32_t cap = ctx->slot_capacity * 2;
    ctx->meshes.resize(cap);
    ctx->mesh_host.resize(cap);
    ctx->slot_capacity = cap;
  }
  MeshHost &m = ctx->mesh_host[slot];
  m = MeshHost();
  m.used = true;
  m.meshlet_base = (uint32_t)ctx->m_lod.size();
  m.meshlet_count = d->meshlet_count;
  m.level_base = (uint32_t)ctx->levels.size();
  m.level_count = d->level_count;
  m.triangle_base = (uint32_t)ctx->m_tris.size();
  // vertex data (occluders): positions and meshletVertices rebased to pool-global ids (GeometryPool.ts:424-429)
  const uint32_t meshlet_vertex_base = (uint32_t)ctx->m_verts.size();
  if (d->positions && d->meshlet_vertices && d->vertex_count && d->meshlet_vertex_count) {
    m.vertex_base = (uint32_t)ctx->positions.size();
    m.vertex_count = d->vertex_count;
    for (uint32_t v = 0; v < d->vertex_count; v++)
      ctx->positions.push_back(make_float4(d->positions[v * 3], d->positions[v * 3 + 1], d->positions[v * 3 + 2], 1.0f));
    for (uint32_t i = 0; i < d->meshlet_vertex_count; i++) ctx->m_verts.push_back(d->meshlet_vertices[i] + m.vertex_base);
  }
  m.triangle_count = d->meshlet_triangles ? d->meshlet_triangle_count : 0;
  m.instance_base = (uint32_t)ctx->inst_slot.size();
  m.instance_count = n;
  m.cell_base = (uint32_t)ctx->cells.size();
  m.cell_count = (n + kCellSize - 1) / kCellSize;
  std::memcpy(m.sphere, d->bounding_sphere, sizeof m.sphere);
  // Test order of the meshlets: within each level (levels stay the same contiguous ranges) by parent error. The test
  // columns
  // (m_lod, m_parent, m_err, m_cull) follow the test order and m_err.w carries the meshlet's pool-global id, which is
  // what every output (draw list, selectCut) reports; m_info and the triangles stay in the caller's order.
  std::vector<uint32_t> order_of_test;
  test_order(d, order_of_test);
  for (uint32_t k = 0; k < d->meshlet_count; k++) {
    const uint32_t i = order_of_test[k];
    const float *b = d->meshlet_bounds + (size_t)i * 16;
    const uint32_t *info = d->meshlet_info + (size_t)i * 4;
    ctx->m_lod.push_back(make_float4(b[0], b[1], b[2], b[3]));
    ctx->m_parent.push_back(make_float4(b[4], b[5], b[6], b[7]));
    float tc, id;
    std::memcpy(&tc, &info[0], 4);
    const uint32_t global = m.meshlet_base + i;
    std::memcpy(&id, &global, 4);
    ctx->m_err.push_back(make_float4(b[8], b[9], tc, id));
    ctx->m_cull.push_back(make_float4(b[12], b[13], b[14], b[15]));
  }
  for (uint32_t i = 0; i < d->meshlet_count; i++) {
    const uint32_t *info = d->meshlet_info + (size_t)i * 4;
    // rebased to pool-global index / vertex ranges (GeometryPool.ts:417-426)
    ctx->m_info.push_back(make_uint4(info[0], info[1] + m.triangle_base * 3, info[2], info[3] + meshlet_vertex_base));
  }
  if (d->meshlet_triangles) ctx->m_tris.insert(ctx->m_tris.end(), d->meshlet_triangles, d->meshlet_triangles + d->meshlet_triangle_count);
  // item trimming data: per level, samples of the parent errors (non-decreasing in test order) and suffix minima of
  // the own errors; valid only when every meshlet's LOD and parent spheres lie inside the mesh's LOD sphere
  // (then max(|V M c| - r s, near) >= max(d - R s, near) for each of them, the bound k_instances relies on)
  for (uint32_t l = 0; l < d->level_count; l++) {
    const uint32_t f = d->level_ranges[l * 2], c = d->level_ranges[l * 2 + 1];
    std::vector<float> sufmin(c);
    float mn = INFINITY;
    for (uint32_t k = c; k-- > 0;) {
      mn = std::min(mn, d->meshlet_bounds[(size_t)order_of_test[f + k] * 16 + 8]);
      sufmin[k] = mn;
    }
    for (uint32_t k = 0; k < kLevelSamples; k++) {
      const uint32_t pos = (uint32_t)(((uint64_t)k * c) / kLevelSamples);
      const float parent = d->meshlet_bounds[(size_t)order_of_test[f + pos] * 16 + 9];
      ctx->lsamples.push_back(make_float2(parent, sufmin[pos]));
    }
  }
  bool contained = true;
  {
    const double C[3] = {d->lod_bounds_sphere[0], d->lod_bounds_sphere[1], d->lod_bounds_sphere[2]};
    const double R = d->lod_bounds_sphere[3];
    for (uint32_t i = 0; i < d->meshlet_count && contained; i++)
      for (int sph = 0; sph < 2; sph++) {
        const float *b = d->meshlet_bounds + (size_t)i * 16 + sph * 4;
        const double dx = b[0] - C[0], dy = b[1] - C[1], dz = b[2] - C[2];
        if (!(std::sqrt(dx * dx + dy * dy + dz * dz) + b[3] <= R)) contained = false;
      }
  }
  for (uint32_t l = 0; l < d->level_count; l++) {
    LevelRec L;
    L.first = d->level_ranges[l * 2] + m.meshlet_base;
    L.count = d->level_ranges[l * 2 + 1];
    L.min_own = d->level_errors[l * 2];
    L.max_parent = d->level_errors[l * 2 + 1];
    L.max_own = d->level_guard_errors[l * 2];
    L.min_parent = d->level_guard_errors[l * 2 + 1];
    L.pad0 = L.pad1 = 0;
    ctx->levels.push_back(L);
  }
  std::vector<uint32_t> order;
  morton_order(matrices, n, d->bounding_sphere, order);
  for (uint32_t g = 0; g < n; g++) {
    const float *e = matrices + (size_t)order[g] * 16;
    for (int c = 0; c < 4; c++) ctx->inst.push_back(make_float4(e[c * 4], e[c * 4 + 1], e[c * 4 + 2], e[c * 4 + 3]));
    ctx->inst_slot.push_back(slot);
    if (gpu_to_input) gpu_to_input[g] = order[g];
  }
  ctx->cells.resize(ctx->cells.size() + m.cell_count);
  for (uint32_t c = 0; c < m.cell_count; c++) compute_cell(ctx, slot, c);
  MeshRec &r = ctx->meshes[slot];
  r.sphere = make_float4(d->bounding_sphere[0], d->bounding_sphere[1], d->bounding_sphere[2], d->bounding_sphere[3]);
  r.lod = make_float4(d->lod_bounds_sphere[0], d->lod_bounds_sphere[1], d->lod_bounds_sphere[2], d->lod_bounds_sphere[3]);
  r.cull = make_float4(d->cull_bounds_sphere[0], d->cull_bounds_sphere[1], d->cull_bounds_sphere[2], d->cull_bounds_sphere[3]);
  r.level_count = d->level_count;
  r.level_base = m.level_base;
  r.meshlet_base = m.meshlet_base;
  r.range_cut = contained ? 1u : 0u;
  vgc_mesh_opts def = {0.0f, 0.0f, 1u, 0u, 0u};
  write_flags(ctx, slot, opts ? opts : &def);
  ctx->slots_used = std::max(ctx->slots_used, slot + 1);
  ctx->dirty = true;
  (void)tri_total;
  *slot_out = slot;
  return VGC_OK;
}

int vgc_mesh_set_flags(vgc_context *ctx, uint32_t slot, const vgc_mesh_opts *opts) {
  if (!ctx || !opts) return fail(VGC_INVALID_ARG, "null argument");
  if (slot >= ctx->slots_used || !ctx->mesh_host[slot].used) return fail(VGC_NOT_FOUND, "no mesh in slot");
  write_flags(ctx, slot, opts);
  return publish_mesh_record(ctx, slot);
}

int vgc_instances_update(vgc_context *ctx, uint32_t slot, uint32_t first, uint32_t count, const float *matrices) {
  if (!ctx || (count && !matrices)) return fail(VGC_INVALID_ARG, "null argument");
  if (slot >= ctx->slots_used || !ctx->mesh_host[slot].used) return fail(VGC_NOT_FOUND, "no mesh in slot");
  MeshHost &m = ctx->mesh_host[slot];
  if ((uint64_t)first + count > m.instance_count) return fail(VGC_INVALID_ARG, "instance range out of bounds");
  if (count == 0) return VGC_OK;
  for (uint32_t g = 0; g < count; g++) {
    const float *e = matrices + (size_t)g * 16;
    for (int c = 0; c < 4; c++) ctx->inst[(size_t)(m.instance_base + first + g) * 4 + c] = make_float4(e[c * 4], e[c * 4 + 1], e[c * 4 + 2], e[c * 4 + 3]);
  }
  const uint32_t c0 = first / kCellSize, c1 = (first + count - 1) / kCellSize;
  for (uint32_t c = c0; c <= c1; c++) compute_cell(ctx, slot, c);  // the host mirror stays current
  if (ctx->dirty) return VGC_OK;  // a full upload is pending anyway
  // resident scene: upload the changed matrices and recompute their cells on the device (GeometryPool.ts:505-512
  // commitInstances), after every launch that may still read them and before any later one
  cudaSetDevice(ctx->device);
  CUDA_TRY(cudaDeviceSynchronize());
  float4 *d_inst = (float4 *)ctx->d_inst.ptr + (size_t)(m.instance_base + first) * 4;
  CUDA_TRY(cudaMemcpyAsync(d_inst, &ctx->inst[(size_t)(m.instance_base + first) * 4], (size_t)count * 64,
                           cudaMemcpyHostToDevice, ctx->stream));
  const double sphere[4] = {m.sphere[0], m.sphere[1], m.sphere[2], m.sphere[3]};
  CUDA_TRY(launch_cells_update((const float4 *)ctx->d_inst.ptr, sphere, m.instance_base, m.instance_count, m.cell_base,
                               slot, c0, c1 - c0 + 1, (CellRec *)ctx->d_cells.ptr, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return VGC_OK;
}

int vgc_mesh_remove(vgc_context *ctx, uint32_t slot) {
  if (!ctx) return fail(VGC_INVALID_ARG, "null argument");
  if (slot >= ctx->slots_used || !ctx->mesh_host[slot].used) return fail(VGC_NOT_FOUND, "no mesh in slot");
  // its cells stay in the cell buffer but point at a disabled slot (GeometryPool.ts:358-363)
  ctx->meshes[slot].enabled = 0;
  ctx->mesh_host[slot].used = false;
  return publish_mesh_record(ctx, slot);
}

int vgc_debug_wait_probe(vgc_context *ctx, uint32_t limit_us, uint32_t *completed, uint64_t *waited_ns) {
  if (!ctx || !completed || !waited_ns || limit_us == 0 || limit_us > 2000000)
    return fail(VGC_INVALID_ARG, "vgc_debug_wait_probe: bad arguments (limit 1 us .. 2 s)");
  cudaSetDevice(ctx->device);
  unsigned long long *d = nullptr, h[2] = {0, 0};
  CUDA_TRY(cudaMalloc(&d, sizeof h));
  cudaError_t e = launch_wait_probe((uint64_t)limit_us * 1000u, d, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(VGC_DEVICE_ERROR, std::string("vgc_debug_wait_probe: ") + cudaGetErrorString(e));
  *completed = (uint32_t)h[0];
  *waited_ns = h[1];
  return VGC_OK;
}

int vgc_debug_cells_device(vgc_context *ctx, float *cells, uint32_t capacity, uint32_t *count) {
  if (!ctx || !count) return fail(VGC_INVALID_ARG, "null argument");
  int rc = sync_scene(ctx);
  if (rc) return rc;
  const uint32_t n = (uint32_t)ctx->cells.size();
  *count = n;
  if (!cells) return VGC_OK;
  std::vector<CellRec> tmp(std::min(capacity, n));
  CUDA_TRY(cudaDeviceSynchronize());
  if (!tmp.empty())
    CUDA_TRY(cudaMemcpy(tmp.data(), ctx->d_cells.ptr, tmp.size() * sizeof(CellRec), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < tmp.size(); i++) {
    const CellRec &c = tmp[i];
    float *o = cells + i * 8;
    o[0] = c.sphere.x; o[1] = c.sphere.y; o[2] = c.sphere.z; o[3] = c.sphere.w;
    o[4] = c.max_radius; o[5] = (float)c.slot; o[6] = (float)c.first; o[7] = (float)c.count;
  }
  return VGC_OK;
}

int vgc_mesh_slots(const vgc_context *ctx, uint32_t *used, uint32_t *capacity) {
  if (!ctx) return fail(VGC_INVALID_ARG, "null argument");
  if (used) *used = ctx->slots_used;
  if (capacity) *capacity = ctx->slot_capacity;
  return VGC_OK;
}

int vgc_hzb_build(vgc_context *ctx, int32_t hzb, const float *depth, uint32_t width, uint32_t height, int on_device,
                  vgc_stream stream) {
  if (!ctx || !depth) return fail(VGC_INVALID_ARG, "null argument");
  if (hzb < 0 || hzb >= (int32_t)vgc_context::kHzbSlots) return fail(VGC_INVALID_ARG, "hzb slot out of range");
  if (width == 0 || height == 0 || width > 32768 || height > 32768) return fail(VGC_INVALID_ARG, "HZB size out of range");
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  bool changed = false;
  int rc = hzb_prepare(ctx, hzb, width, height, &changed);
  if (rc) return rc;
  HzbSlot &h = ctx->hzb[hzb];
  const HzbDesc desc = h.desc;
  float *out = (float *)h.data.ptr;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(st, &cs);
  const bool capture = cs != cudaStreamCaptureStatusNone;
  if (!on_device) {
    CUDA_TRY(cudaMemcpyAsync(out, depth, (size_t)width * height * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(timed(ctx, capture, VGC_KERNEL_HZB, st, [&] { return launch_hzb(out, desc, out, 0, st); }));
  } else {
    CUDA_TRY(timed(ctx, capture, VGC_KERNEL_HZB, st, [&] { return launch_hzb(depth, desc, out, 1, st); }));
  }
  if (changed)
    CUDA_TRY(cudaMemcpyAsync((HzbDesc *)ctx->d_hzb_desc.ptr + hzb, &h.desc, sizeof(HzbDesc), cudaMemcpyHostToDevice, st));
  return VGC_OK;
}

int vgc_hzb_info(const vgc_context *ctx, int32_t hzb, uint32_t *levels, uint32_t *offset, uint32_t *width,
                 uint32_t *height, const float **data) {
  if (!ctx) return fail(VGC_INVALID_ARG, "null context");
  if (hzb < 0 || hzb >= (int32_t)vgc_context::kHzbSlots || !ctx->hzb[hzb].valid) return fail(VGC_NOT_FOUND, "no HZB in slot");
  const HzbDesc &d = ctx->hzb[hzb].desc;
  if (levels) *levels = d.levels;
  for (uint32_t i = 0; i < kMaxHzbLevels; i++) {
    if (offset) offset[i] = d.off[i];
    if (width) width[i] = d.w[i];
    if (height) height[i] = d.h[i];
  }
  if (data) *data = d.data;
  return VGC_OK;
}

int vgc_cut(vgc_context *ctx, const vgc_view *views, uint32_t count, uint32_t first_slot, vgc_stream stream) {
  if (!ctx) return fail(VGC_INVALID_ARG, "null context");
  cudaSetDevice(ctx->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  int rc = prepare(ctx, ctx->scratch, views, count, first_slot);
  if (rc) return rc;
  if ((rc = enqueue(ctx, ctx->scratch, count, st, false))) return rc;
  CUDA_TRY(cudaEventRecord(ctx->scratch.done, st));
  ctx->scratch.pending = true;
  return VGC_OK;
}

int vgc_batch_create(vgc_context *ctx, uint32_t max_views, vgc_batch **out) {
  if (!ctx || !out || max_views == 0) return fail(VGC_INVALID_ARG, "bad arguments");
  vgc_batch *b = new vgc_batch();
  b->ctx = ctx;
  b->max_views = max_views;
  if (cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return fail(VGC_DEVICE_ERROR, "cudaStreamCreate failed");
  }
  *out = b;
  return VGC_OK;
}

int vgc_batch_run(vgc_batch *b, const vgc_view *views, uint32_t count, uint32_t first_slot, vgc_stream stream) {
  if (!b) return fail(VGC_INVALID_ARG, "null batch");
  if (count > b->max_views) return fail(VGC_INVALID_ARG, "more views than the batch was created for");
  vgc_context *ctx = b->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  int rc = prepare(ctx, b->scratch, views, count, first_slot);
  if (rc) return rc;
  const uint32_t cells = (uint32_t)ctx->cells.size();
  if (!b->exec || b->graph_views != count || b->graph_cells != cells || b->graph_slots != ctx->slot_capacity ||
      b->graph_hzb_w != b->scratch.hzb_w || b->graph_hzb_h != b->scratch.hzb_h || b->graph_hzb_tail != b->scratch.hzb_tail ||
      b->graph_budget != b->scratch.any_budget || b->graph_queue != b->scratch.d_chunks ||
      b->graph_grids[0] != b->scratch.grid_instances || b->graph_grids[1] != b->scratch.grid_chunks ||
      b->graph_chunk_shift != b->scratch.chunk_shift) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
    rc = enqueue(ctx, b->scratch, count, b->capture_stream, true);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->capture_stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return fail(VGC_DEVICE_ERROR, std::string("graph capture: ") + cudaGetErrorString(e));
    b->graph = g;
    CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->graph_views = count;
    b->graph_cells = cells;
    b->graph_slots = ctx->slot_capacity;
    b->graph_hzb_w = b->scratch.hzb_w;
    b->graph_hzb_h = b->scratch.hzb_h;
    b->graph_hzb_tail = b->scratch.hzb_tail;
    b->graph_budget = b->scratch.any_budget;
    b->graph_queue = b->scratch.d_chunks;
    b->graph_grids[0] = b->scratch.grid_instances;
    b->graph_grids[1] = b->scratch.grid_chunks;
    b->graph_chunk_shift = b->scratch.chunk_shift;
  }
  CUDA_TRY(cudaGraphLaunch(b->exec, st));
  CUDA_TRY(cudaEventRecord(b->scratch.done, st));
  b->scratch.pending = true;
  return VGC_OK;
}

int vgc_batch_autotune(vgc_batch *b, const vgc_view *views, uint32_t count, uint32_t first_slot, vgc_stream stream,
                       uint32_t reps, vgc_tune_result *best) {
  if (!b || !views || !best || count == 0) return fail(VGC_INVALID_ARG, "bad arguments");
  vgc_context *ctx = b->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  const uint32_t sms = (uint32_t)ctx->sm_count;
  const uint32_t max_i = std::max(1u, ctx->select_grid / sms), max_c = std::max(1u, ctx->chunk_grid / sms);
  // candidate blocks per SM: quarters of the occupancy limit, each at least 1
  auto steps = [](uint32_t mx) {
    std::vector<uint32_t> v;
    for (uint32_t q = 1; q <= 4; q++) {
      const uint32_t x = std::max(1u, (mx * q + 3) / 4);
      if (v.empty() || v.back() != x) v.push_back(x);
    }
    return v;
  };
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  reps = std::max(1u, reps);
  vgc_tune_result top{0, 0, INFINITY, 0};
  int rc = VGC_OK;
  for (uint32_t shift = kChunkShiftMin; shift <= kChunkShiftMax && !rc; shift++)
  for (uint32_t bi : steps(max_i)) {
    for (uint32_t bc : steps(max_c)) {
      b->scratch.grid_instances = bi * sms;
      b->scratch.grid_chunks = bc * sms;
      b->scratch.chunk_shift = shift;
      if ((rc = vgc_batch_run(b, views, count, first_slot, stream))) break;  // capture + warm-up
      std::vector<float> ms;
      for (uint32_t r = 0; r < reps; r++) {  // replays of the captured graph: device time only
        cudaEventRecord(e0, st);
        cudaGraphLaunch(b->exec, st);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
          rc = fail(VGC_DEVICE_ERROR, "autotune replay failed");
          break;
        }
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        ms.push_back(t);
      }
      if (rc) break;
      std::sort(ms.begin(), ms.end());
      const float med = ms[ms.size() / 2];
      if (med < top.ms) top = vgc_tune_result{bi, bc, med, 1u << shift};
    }
    if (rc) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  b->scratch.grid_instances = top.instances_blocks_per_sm * sms;
  b->scratch.grid_chunks = top.chunks_blocks_per_sm * sms;
  b->scratch.chunk_shift = (uint32_t)__builtin_ctz(top.chunk_meshlets);
  *best = top;
  return VGC_OK;
}

int vgc_batch_set_tuning(vgc_batch *b, const vgc_tune_result *t) {
  if (!b || !t) return fail(VGC_INVALID_ARG, "null argument");
  const uint32_t c = t->chunk_meshlets;
  if (c != 256 && c != 512 && c != 1024) return fail(VGC_INVALID_ARG, "chunk_meshlets must be 256, 512 or 1024");
  const uint32_t sms = (uint32_t)b->ctx->sm_count;
  const uint32_t max_i = std::max(1u, b->ctx->select_grid / sms), max_c = std::max(1u, b->ctx->chunk_grid / sms);
  if (t->instances_blocks_per_sm > max_i || t->chunks_blocks_per_sm > max_c)
    return fail(VGC_INVALID_ARG, "blocks per SM above the kernels' occupancy limit");
  b->scratch.grid_instances = t->instances_blocks_per_sm * sms;
  b->scratch.grid_chunks = t->chunks_blocks_per_sm * sms;
  b->scratch.chunk_shift = (uint32_t)__builtin_ctz(c);
  return VGC_OK;
}

int vgc_batch_destroy(vgc_batch *b) {
  if (!b) return VGC_OK;
  cudaSetDevice(b->ctx->device);
  if (b->scratch.pending) cudaEventSynchronize(b->scratch.done);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
  if (b->scratch.d_views)
    b->ctx->bytes -= sizeof(ViewConst) * b->scratch.view_capacity + hzb_plan_bytes(b->scratch.view_capacity);
  if (b->scratch.d_units) b->ctx->bytes -= unit_bytes(b->scratch.unit_capacity);
  free_scratch(b->scratch);
  delete b;
  return VGC_OK;
}

int vgc_get_output(const vgc_context *ctx, uint32_t slot, vgc_output *out) {
  if (!ctx || !out) return fail(VGC_INVALID_ARG, "null argument");
  if (slot >= ctx->out_slots) return fail(VGC_NOT_FOUND, "output slot not allocated");
  const size_t md = ctx->opts.max_meshlets;
  const uint4 *draw = (const uint4 *)ctx->d_draw.ptr + (size_t)slot * 2 * md;
  out->draw_list[0] = (const uint32_t *)draw;
  out->draw_list[1] = (const uint32_t *)(draw + md);
  out->draw_args = (const uint32_t *)ctx->d_args.ptr + (size_t)slot * 2 * ctx->slot_capacity * 2 * 5;
  out->counters = (const uint32_t *)ctx->d_counters.ptr + (size_t)slot * ctx->counter_words;
  out->max_drawn = (uint32_t)md;
  out->mesh_slots = ctx->slot_capacity;
  return VGC_OK;
}

int vgc_read_stats(vgc_context *ctx, uint32_t slot, vgc_stats *s, vgc_stream stream) {
  if (!ctx || !s) return fail(VGC_INVALID_ARG, "null argument");
  if (slot >= ctx->out_slots) return fail(VGC_NOT_FOUND, "output slot not allocated");
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  CUDA_TRY(cudaStreamSynchronize(st));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  uint32_t c[VGC_COUNTER_HEADER];
  CUDA_TRY(cudaMemcpy(c, (const uint32_t *)ctx->d_counters.ptr + (size_t)slot * ctx->counter_words, sizeof c, cudaMemcpyDeviceToHost));
  float dyn = 0;
  CUDA_TRY(cudaMemcpy(&dyn, (const float *)ctx->d_dyn.ptr + (size_t)slot * 8, 4, cudaMemcpyDeviceToHost));
  decode_stats(ctx, c, dyn, s);
  return VGC_OK;
}

int vgc_read_draw_list(vgc_context *ctx, uint32_t slot, uint32_t cut, uint32_t *entries, uint32_t capacity,
                       uint32_t *count, vgc_stream stream) {
  if (!ctx || !count || cut > 1 || (capacity && !entries)) return fail(VGC_INVALID_ARG, "bad arguments");
  if (slot >= ctx->out_slots) return fail(VGC_NOT_FOUND, "output slot not allocated");
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  CUDA_TRY(cudaStreamSynchronize(st));
  uint32_t sel = 0;
  CUDA_TRY(cudaMemcpy(&sel, (const uint32_t *)ctx->d_counters.ptr + (size_t)slot * ctx->counter_words + VGC_COUNTER_CUT0 + cut * 5 + VGC_CUT_SELECTED, 4, cudaMemcpyDeviceToHost));
  const uint32_t n = std::min(sel, ctx->opts.max_meshlets);
  *count = n;
  const uint32_t copy = std::min(n, capacity);
  if (copy) {
    const uint4 *src = (const uint4 *)ctx->d_draw.ptr + ((size_t)slot * 2 + cut) * ctx->opts.max_meshlets;
    CUDA_TRY(cudaMemcpy(entries, src, (size_t)copy * 16, cudaMemcpyDeviceToHost));
  }
  return VGC_OK;
}

int vgc_state_access(vgc_context *ctx, uint32_t state_slot, uint32_t *words, int write, vgc_stream stream) {
  if (!ctx || !words) return fail(VGC_INVALID_ARG, "null argument");
  int rc = ensure_state(ctx, state_slot);
  if (rc) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  CUDA_TRY(cudaStreamSynchronize(st));
  uint32_t *dst = (uint32_t *)ctx->d_state.ptr + (size_t)state_slot * kStateWords;
  if (write) CUDA_TRY(cudaMemcpy(dst, words, kStateWords * 4, cudaMemcpyHostToDevice));
  else CUDA_TRY(cudaMemcpy(words, dst, kStateWords * 4, cudaMemcpyDeviceToHost));
  return VGC_OK;
}

int vgc_expand(vgc_context *ctx, uint32_t slot, uint32_t cut, uint32_t *index_buffer, uint64_t capacity, vgc_stream stream) {
  if (!ctx || !index_buffer || cut > 1) return fail(VGC_INVALID_ARG, "bad arguments");
  if (slot >= ctx->out_slots) return fail(VGC_NOT_FOUND, "output slot not allocated");
  for (uint32_t m = 0; m < ctx->slots_used; m++)
    if (ctx->mesh_host[m].used && ctx->mesh_host[m].triangle_count == 0)
      return fail(VGC_INVALID_ARG, "vgc_expand needs meshlet_triangles for every mesh (slot " + std::to_string(m) + ")");
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  // the view constants of this slot, rebuilt from the output pointers (only the pointers and sizes are read)
  ViewConst k{};
  k.max_drawn = ctx->opts.max_meshlets;
  k.counters = (uint32_t *)ctx->d_counters.ptr + (size_t)slot * ctx->counter_words;
  k.draw_list = (uint4 *)ctx->d_draw.ptr + (size_t)slot * 2 * ctx->opts.max_meshlets;
  int rc = ensure_scratch(ctx, ctx->scratch, 1, 32);
  if (rc) return rc;
  if (ctx->scratch.pending) CUDA_TRY(cudaEventSynchronize(ctx->scratch.done));
  ctx->scratch.h_views[0] = k;
  CUDA_TRY(cudaMemcpyAsync(ctx->scratch.d_views, ctx->scratch.h_views, sizeof(ViewConst), cudaMemcpyHostToDevice, st));
  CUDA_TRY(launch_expand(scene_of(ctx), ctx->scratch.d_views, cut, index_buffer, capacity, ctx->sm_count * 8, st));
  CUDA_TRY(cudaEventRecord(ctx->scratch.done, st));
  ctx->scratch.pending = true;
  return VGC_OK;
}

int vgc_select_cut(vgc_context *ctx, uint32_t slot, uint32_t count, const double *vm16, const double *proj_scale,
                   const double *near_, const double *scale, double threshold, double blend, uint8_t *lo, uint8_t *hi) {
  if (!ctx || !vm16 || !proj_scale || !near_ || !scale || !lo || !hi) return fail(VGC_INVALID_ARG, "null argument");
  if (slot >= ctx->slots_used || !ctx->mesh_host[slot].used) return fail(VGC_NOT_FOUND, "no mesh in slot");
  if (count == 0) return VGC_OK;
  cudaSetDevice(ctx->device);
  int rc = sync_scene(ctx);
  if (rc) return rc;
  const uint32_t mcount = ctx->mesh_host[slot].meshlet_count;
  std::vector<float> m((size_t)count * 16), p((size_t)count * 3);
  for (size_t i = 0; i < m.size(); i++) m[i] = (float)vm16[i];
  for (uint32_t i = 0; i < count; i++) {
    p[i * 3] = (float)proj_scale[i];
    p[i * 3 + 1] = (float)near_[i];
    p[i * 3 + 2] = (float)scale[i];
  }
  const size_t outn = (size_t)count * mcount;
  void *d = nullptr;
  CUDA_TRY(cudaMalloc(&d, m.size() * 4 + p.size() * 4 + outn * 2 + 64));
  float *dm = (float *)d, *dp = dm + m.size();
  uint8_t *dlo = (uint8_t *)(dp + p.size()), *dhi = dlo + outn;
  cudaStream_t st = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(dm, m.data(), m.size() * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, p.data(), p.size() * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = launch_select_cut(scene_of(ctx), slot, mcount, count, dm, dp, (float)threshold, (float)blend, dlo, dhi,
                          ctx->sm_count * 8, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(lo, dlo, outn, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hi, dhi, outn, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d);
  if (e != cudaSuccess) return fail(VGC_DEVICE_ERROR, std::string("select_cut: ") + cudaGetErrorString(e));
  return VGC_OK;
}

int vgc_set_profiling(vgc_context *ctx, int enable) {
  if (!ctx) return fail(VGC_INVALID_ARG, "null context");
  ctx->profiling = enable != 0;
  return VGC_OK;
}

int vgc_kernel_times(vgc_context *ctx, double *ms, uint32_t *launches, int reset) {
  if (!ctx) return fail(VGC_INVALID_ARG, "null context");
  for (auto &p : ctx->prof_pending) {
    CUDA_TRY(cudaEventSynchronize(p.second.second));
    float t = 0;
    CUDA_TRY(cudaEventElapsedTime(&t, p.second.first, p.second.second));
    ctx->prof_ms[p.first] += t;
    ctx->prof_count[p.first] += 1;
    ctx->prof_free.push_back(p.second.first);
    ctx->prof_free.push_back(p.second.second);
  }
  ctx->prof_pending.clear();
  for (int k = 0; k < VGC_KERNEL_KINDS; k++) {
    if (ms) ms[k] = ctx->prof_ms[k];
    if (launches) launches[k] = ctx->prof_count[k];
    if (reset) {
      ctx->prof_ms[k] = 0;
      ctx->prof_count[k] = 0;
    }
  }
  return VGC_OK;
}

// Test support: the scene's cell records (8 floats each: centre, radius, max radius, slot, first, count as float
// values, the reference's cell layout GeometryPool.ts:544) and the Morton-ordered instance matrices.
int vgc_debug_scene(const vgc_context *ctx, float *cells, uint32_t cell_capacity, float *matrices,
                    uint32_t matrix_capacity, uint32_t *cell_count, uint32_t *instance_count) {
  if (!ctx) return fail(VGC_INVALID_ARG, "null context");
  if (cell_count) *cell_count = (uint32_t)ctx->cells.size();
  if (instance_count) *instance_count = (uint32_t)ctx->inst_slot.size();
  if (cells)
    for (uint32_t i = 0; i < std::min<uint32_t>(cell_capacity, (uint32_t)ctx->cells.size()); i++) {
      const CellRec &c = ctx->cells[i];
      float *o = cells + (size_t)i * 8;
      o[0] = c.sphere.x; o[1] = c.sphere.y; o[2] = c.sphere.z; o[3] = c.sphere.w;
      o[4] = c.max_radius; o[5] = (float)c.slot; o[6] = (float)c.first; o[7] = (float)c.count;
    }
  if (matrices)
    for (uint32_t i = 0; i < std::min<uint32_t>(matrix_capacity, (uint32_t)ctx->inst_slot.size()); i++)
      std::memcpy(matrices + (size_t)i * 16, &ctx->inst[(size_t)i * 4], 64);
  return VGC_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------ no-alloc cut
// vgc_cut_noalloc: the single-view cut for callers that must not allocate device memory on the call (a renderer's
// real-time frame thread that must not stall on cudaMalloc, a host that pre-reserves all of its GPU memory). Its
// per-call scratch - the batch control words, the view constants, the (view, cell) unit list and the meshlet chunk
// queue - lives in this fixed file-scope device array instead of the context's launch scratch. Every GPU that loads
// the library holds the array until the process exits.
namespace {
constexpr size_t kNoAllocCtl = 0;                                   // 16 control words
constexpr size_t kNoAllocView = 256;                                // one ViewConst
constexpr uint32_t kNoAllocMaxUnits = 65536;                        // visible (view, cell) units: cells of the scene
constexpr uint32_t kNoAllocMaxChunks = 65536;                       // meshlet work queue entries (beyond: tested in place)
constexpr size_t kNoAllocUnits = 1024;
constexpr size_t kNoAllocChunks = kNoAllocUnits + (size_t)kNoAllocMaxUnits * sizeof(uint2);
constexpr size_t kNoAllocOverflow = kNoAllocChunks + (size_t)kNoAllocMaxChunks * sizeof(uint4);
constexpr size_t kNoAllocBytes = kNoAllocOverflow + (size_t)kNoAllocMaxUnits * 4 / 32 * sizeof(uint32_t);  // 1.53 MiB
static_assert(sizeof(ViewConst) <= kNoAllocUnits - kNoAllocView, "view constants must fit their scratch slot");
static_assert(kNoAllocChunks % 256 == 0, "chunk queue must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_ptr[64] = {nullptr};  // device address of g_noalloc_scratch per device ordinal

// Device address of the scratch array on `device`, looked up once per device with that device current: in host code
// the array's name only stands in for the symbol, so kernels must receive this address instead.
int noalloc_scratch(int device, unsigned char **out) {
  if (device < 0 || device >= 64) return fail(VGC_INVALID_ARG, "device ordinal out of range for the no-alloc scratch");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    int current = -1;
    cudaError_t ce = cudaGetDevice(&current);
    if (ce != cudaSuccess) return fail(VGC_DEVICE_ERROR, std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
    if (current != device)
      return fail(VGC_DEVICE_ERROR, "no-alloc scratch: device " + std::to_string(device) + " is not current");
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(VGC_DEVICE_ERROR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_ptr[device] = (unsigned char *)p;
  }
  *out = g_noalloc_ptr[device];
  return VGC_OK;
}
}  // namespace

// Writes the view constants into the scratch array. They travel as a kernel argument, which the launch copies, so
// no host buffer has to outlive the call and nothing is copied from host memory.
static_assert(sizeof(ViewConst) % 4 == 0, "view constants are copied as 32-bit words");
__global__ void k_noalloc_store_view(const ViewConst k, ViewConst *dst) {
  const uint32_t *src = reinterpret_cast<const uint32_t *>(&k);
  uint32_t *out = reinterpret_cast<uint32_t *>(dst);
  for (uint32_t i = threadIdx.x; i < sizeof(ViewConst) / 4; i += blockDim.x) out[i] = src[i];
}

extern "C" int vgc_cut_noalloc(vgc_context *ctx, const vgc_view *view, uint32_t slot, vgc_stream stream) {
  if (!ctx || !view) return fail(VGC_INVALID_ARG, "null argument");
  cudaError_t se = cudaSetDevice(ctx->device);
  if (se != cudaSuccess) return fail(VGC_DEVICE_ERROR, std::string("cudaSetDevice: ") + cudaGetErrorString(se));
  // everything this call writes must exist already: it allocates nothing
  if (ctx->dirty)
    return fail(VGC_INVALID_ARG, "vgc_cut_noalloc: the scene changed since the last upload; one allocating call "
                                 "(vgc_cut) must publish it first");
  if (slot >= ctx->out_slots || ctx->out_slot_capacity != ctx->slot_capacity)
    return fail(VGC_INVALID_ARG, "vgc_cut_noalloc: output slot " + std::to_string(slot) +
                                     " is not allocated (create the context with enough output_slots)");
  if (view->state_slot >= ctx->state_slots)
    return fail(VGC_INVALID_ARG, "vgc_cut_noalloc: state slot " + std::to_string(view->state_slot) + " is not allocated");
  const uint32_t cells = pad32((uint32_t)ctx->cells.size());
  if (cells > kNoAllocMaxUnits)
    return fail(VGC_INVALID_ARG, "vgc_cut_noalloc: the scene has " + std::to_string(ctx->cells.size()) +
                                     " cells; the fixed scratch holds at most " + std::to_string(kNoAllocMaxUnits));
  bool build_hzb = false;
  if (view->hzb >= 0) {
    if (view->hzb >= (int32_t)vgc_context::kHzbSlots) return fail(VGC_INVALID_ARG, "view: hzb slot out of range");
    const HzbSlot &h = ctx->hzb[view->hzb];
    if (view->depth) {
      size_t total = 0;
      HzbDesc want = hzb_layout(view->depth_width, view->depth_height, &total);
      if (!h.valid || h.data.bytes < total * 4 || h.desc.levels != want.levels || h.desc.w[0] != want.w[0] ||
          h.desc.h[0] != want.h[0])
        return fail(VGC_INVALID_ARG, "vgc_cut_noalloc: HZB slot " + std::to_string(view->hzb) +
                                         " is not laid out for this depth size (build it once with vgc_hzb_build)");
      build_hzb = true;
    } else if (!h.valid) {
      return fail(VGC_INVALID_ARG, "view: hzb slot " + std::to_string(view->hzb) + " has no HZB");
    }
  }
  unsigned char *scratch = nullptr;
  int rc = noalloc_scratch(ctx->device, &scratch);
  if (rc) return rc;
  ViewConst k;
  if ((rc = view_constants(ctx, *view, slot, 0, k))) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  uint32_t *ctl = (uint32_t *)(scratch + kNoAllocCtl);
  ViewConst *d_view = (ViewConst *)(scratch + kNoAllocView);
  uint2 *units = (uint2 *)(scratch + kNoAllocUnits);
  uint4 *chunks = (uint4 *)(scratch + kNoAllocChunks);
  uint32_t *overflow = (uint32_t *)(scratch + kNoAllocOverflow);  // zero at load; every pass leaves it zero
  const uint32_t redo_grid = (uint32_t)ctx->sm_count * 2;
  // the constants go in by value (k_reset clears the control words)
  k_noalloc_store_view<<<1, 128, 0, st>>>(k, d_view);
  CUDA_TRY(cudaGetLastError());
  const Scene S = scene_of(ctx);
  if (build_hzb) {
    const HzbDesc &d = ctx->hzb[view->hzb].desc;
    CUDA_TRY(launch_hzb_views(d_view, 1, d.w[0], d.h[0], d.levels > 7, st));
  }
  CUDA_TRY(launch_reset(d_view, 1, ctl, st));
  CUDA_TRY(launch_cells(S, nullptr, d_view, 1, cells, units, ctl, st));
  if (view->triangle_budget > 0) {
    CUDA_TRY(launch_instances(S, nullptr, d_view, units, ctl, chunks, kNoAllocMaxChunks, -1, ctx->select_grid, overflow,
                              st));
    CUDA_TRY(launch_chunks(S, nullptr, d_view, chunks, ctl, kNoAllocMaxChunks, -1, ctx->chunk_grid, st));
    CUDA_TRY(launch_instances_redo(S, nullptr, d_view, units, ctl, chunks, kNoAllocMaxChunks, -1, overflow, redo_grid,
                                   st));
    CUDA_TRY(launch_budget(d_view, 1, ctl, st));
  }
  for (int round = 0; round < 3; round++) {
    CUDA_TRY(launch_instances(S, nullptr, d_view, units, ctl, chunks, kNoAllocMaxChunks, round, ctx->select_grid,
                              overflow, st));
    CUDA_TRY(launch_chunks(S, nullptr, d_view, chunks, ctl, kNoAllocMaxChunks, round, ctx->chunk_grid, st));
    CUDA_TRY(launch_instances_redo(S, nullptr, d_view, units, ctl, chunks, kNoAllocMaxChunks, round, overflow,
                                   redo_grid, st));
    CUDA_TRY(launch_finish(d_view, 1, ctl, round, st));
  }
  return VGC_OK;
}
