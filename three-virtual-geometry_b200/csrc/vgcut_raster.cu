// Occluder depth pass (vgc_occluder_depth): the reference draws the occluder meshes' previous-frame camera cuts
// depth-only with the current camera into a small depth target before the HZB build (OcclusionCulling.ts:244-273,
// through the pools' vertex pulling, GeometryPool.ts:1095-1131). Here it is a CUDA rasterizer over the draw list of
// an output slot:
//
//  * one warp per draw-list entry of part 0 (drawn over every pixel; the blended ones are left out, as in the
//    reference's proxy) whose mesh is an occluder; clip = (P V M) p with the instance's model matrix;
//  * a triangle is clipped against the near plane (clip.z >= 0, WebGPU depth) as a GPU's clipper would: the part in
//    front is a triangle or a quad (two triangles) with the crossing points at depth 0; a triangle that faces away
//    (the reference's proxy is single-sided) is dropped;
//  * pixel centres (x + 0.5, y + 0.5) inside all three edge functions (edges included) take the depth interpolated
//    from the vertices' NDC depths (affine in screen space) through an atomic minimum on the float's bits (depth is
//    >= 0, so the unsigned order is the float order); the image starts at 1 (far);
//  * each meshlet vertex is transformed once, into the warp's shared-memory vertex buffer (meshlet-local ids < 256);
//    a meshlet's loads are issued together (its triangles, then its vertex ids, then positions, 128 at a time) and
//    the warp's next entry is fetched while it draws this one: every step of this pass waits on memory;
//  * triangles are sorted by the pixels of their bounding box: small ones (at most kLaneRasterMax) are drawn at once
//    by the warp, their pixels laid end to end, a lane per pixel; medium ones (at most kWarpRasterMax) are queued, one atomic per warp and round of 32 triangles
//    on one of kSubQueues counters, and drawn by the second kernel, a warp per triangle; larger ones are queued as
//    32 x 16 pixel tiles of their bounding box, a warp per tile. The second kernel spreads both over the whole
//    grid: a meshlet close to the camera, with a hundred triangles of a few hundred pixels each, would otherwise
//    keep one warp drawing long after the rest have finished. When a queue is full its triangles are drawn by the
//    warp that set them up;
//  * the atomics' results are unused, so they do not wait (a load-then-atomic early depth test measured slower: it
//    puts an L2 round trip on every pixel). The image is the minimum over all drawn pixels, whatever the order.
//
// The visibility pass (vgc_visibility, below) draws a cut's expanded index buffer through the same triangle setup,
// size classes and queues, with 64-bit (depth | triangle id) fragments.
//
// Every expression rounds step by step in the written order (the library is compiled with -fmad=false), so the
// oracle's C restatement reproduces the image bit for bit.
#include "vgcut_host.h"
#include "vgcut_kernels.h"

namespace {

constexpr uint32_t kLaneRasterMax = 16;     // bounding-box pixels up to which a triangle is drawn by its lane
constexpr uint32_t kWarpRasterMax = 1024;   // ... by one warp of the second kernel; beyond, as tiles
constexpr uint32_t kTileW = 32, kTileH = 16;
constexpr uint32_t kQueuedMedium = 1u << 19;  // queue capacities: medium triangles,
constexpr uint32_t kSubQueues = 256;          //   in sub-queues (record i of sub-queue q at i * kSubQueues + q),
constexpr uint32_t kClipCtl = 4 + kSubQueues;   // occluder pass: triangles crossing the near plane, queued
constexpr uint32_t kCtlWords = kClipCtl + 1;
constexpr uint32_t kClipQueue = 1u << 17;       //   (draw-list entry, triangle) records, clipped by a later kernel
constexpr uint32_t kQueuedLarge = 1u << 16;   // large triangles,
constexpr uint32_t kTileUnits = 1u << 20;     // and their tiles
constexpr uint32_t kNoTri = 0xffffffffu;      // an empty tile record
constexpr uint32_t kRecord = 5;               // float4 per queued triangle
constexpr uint32_t kMaxImages = 64;           // occluder images per launch set (vgc_occluder_depth_batch)

// Where the fragments go, and the queues of the second kernel.
struct RasterArgs {
  uint32_t width, height;
  uint32_t *depth[kMaxImages];   // occluder pass: float bits per pixel of image i (a fragment's TriTag::id)
  unsigned long long *vis;       // visibility pass: (depth bits << 32 | id) per pixel
  uint32_t frame;                // visibility pass: lodBlendFrame
  // queues: ctl[1] = large triangles, ctl[2..3] = tiles (64-bit), ctl[4 + q] = medium triangles of sub-queue q;
  // triangle records (kRecord float4: the ScreenTri, its tile columns and its tag); tile records (large triangle,
  // tile index in its bounding box, row-major)
  uint32_t *ctl;
  float4 *medium;
  float4 *large;
  uint2 *tiles;
  uint2 *clip;  // occluder pass: crossing triangles (ctl[kClipCtl] of them)
};

// The occluder pass's inputs: per image, the camera and the cut it draws.
struct OccluderImage {
  float vp[16];  // P * V, row-major 4x4 (float of the double product)
  const uint4 *draw_list;      // cut 0 entries of the source slot
  const uint32_t *counters;    // its counter header
};
struct OccluderArgs {
  OccluderImage img[kMaxImages];
  uint32_t count, max_drawn;
};

struct ScreenTri {
  float ax, ay, az, bx, by, bz, cx, cy, cz, area;
  int x0, x1, y0, y1;  // pixel bounding box, inclusive
};

// What a fragment carries besides its depth: for the visibility pass the entry's blend range and the triangle's id,
// for the occluder pass (lo = hi = 0) the image it belongs to in `id`.
struct TriTag {
  uint32_t lo, hi, id;
};

// Clip coordinates of a position: (P V M) p.
__device__ __forceinline__ float4 clip_vertex(const float mvp[4][4], float4 v) {
  float c[4];
#pragma unroll
  for (int r = 0; r < 4; r++) c[r] = ((mvp[r][0] * v.x + mvp[r][1] * v.y) + mvp[r][2] * v.z) + mvp[r][3];
  return make_float4(c[0], c[1], c[2], c[3]);
}

// A clip-space vertex in screen space: x, y (pixels, y down), NDC depth; w = 1 when usable (in front of the near
// plane), else all 0.
__device__ __forceinline__ float4 screen_of(float4 c, float W, float H) {
  if (!(c.w > 0.0f) || !(c.z >= 0.0f)) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float nx = c.x / c.w, ny = c.y / c.w, nz = c.z / c.w;
  return make_float4((nx * 0.5f + 0.5f) * W, (0.5f - ny * 0.5f) * H, nz, 1.0f);
}

__device__ __forceinline__ float4 screen_vertex(const float mvp[4][4], float4 v, float W, float H) {
  return screen_of(clip_vertex(mvp, v), W, H);
}

// Setup of one triangle from its screen-space corners; false when it is dropped.
__device__ __forceinline__ bool setup_triangle(float4 v0, float4 v1, float4 v2, float W, float H, ScreenTri &t) {
  if (v0.w == 0.0f || v1.w == 0.0f || v2.w == 0.0f) return false;  // a corner behind the near plane
  // screen space is y-down: a triangle facing the camera (counter-clockwise in NDC) has a negative area here
  const float area0 = (v1.x - v0.x) * (v2.y - v0.y) - (v2.x - v0.x) * (v1.y - v0.y);
  if (!(area0 < 0.0f)) return false;  // back-facing, degenerate or not finite
  // order A, B, C = 0, 2, 1: positive area
  t.ax = v0.x, t.ay = v0.y, t.az = v0.z;
  t.bx = v2.x, t.by = v2.y, t.bz = v2.z;
  t.cx = v1.x, t.cy = v1.y, t.cz = v1.z;
  t.area = (t.bx - t.ax) * (t.cy - t.ay) - (t.cx - t.ax) * (t.by - t.ay);
  if (!(t.area > 0.0f)) return false;
  float mnx = fminf(fminf(t.ax, t.bx), t.cx), mxx = fmaxf(fmaxf(t.ax, t.bx), t.cx);
  float mny = fminf(fminf(t.ay, t.by), t.cy), mxy = fmaxf(fmaxf(t.ay, t.by), t.cy);
  // pixel centres px + 0.5 in [mn, mx]; clamped in float before the integer conversion
  mnx = fmaxf(mnx, -1.0f), mxx = fminf(mxx, W + 1.0f);
  mny = fmaxf(mny, -1.0f), mxy = fminf(mxy, H + 1.0f);
  t.x0 = max(0, int(ceilf(mnx - 0.5f)));
  t.x1 = min(int(W) - 1, int(floorf(mxx - 0.5f)));
  t.y0 = max(0, int(ceilf(mny - 0.5f)));
  t.y1 = min(int(H) - 1, int(floorf(mxy - 0.5f)));
  return t.x0 <= t.x1 && t.y0 <= t.y1;
}

// Near-plane clipping (Sutherland-Hodgman against clip.z >= 0) of the triangle with clip-space corners c0, c1, c2;
// the part in front is a triangle or a quad, set up as screen triangles into t0 (and t1); returns how many (0..2),
// t0 holding the first. With A the corner in front (one in front) or the corner after the one behind (two in front)
// in the order c0 -> c1 -> c2, and B, C the next ones: one in front -> (A, AB, CA); two in front (A, B) ->
// (A, B, BC) and (A, BC, CA), where XY = X + s (Y - X), s = X.z / (X.z - Y.z), is the crossing point at depth 0.
// A triangle wholly in front gives exactly setup_triangle of its screen corners.
__device__ __forceinline__ float4 crossing(float4 p, float4 q) {
  const float s = p.z / (p.z - q.z);
  return make_float4(p.x + s * (q.x - p.x), p.y + s * (q.y - p.y), 0.0f, p.w + s * (q.w - p.w));
}

__device__ __forceinline__ float4 pick3(int i, float4 a, float4 b, float4 c) { return i == 0 ? a : (i == 1 ? b : c); }

__device__ __forceinline__ int setup_clipped(float4 c0, float4 c1, float4 c2, float W, float H, ScreenTri &t0,
                                             ScreenTri &t1) {
  const int in = (c0.z >= 0.0f ? 1 : 0) + (c1.z >= 0.0f ? 1 : 0) + (c2.z >= 0.0f ? 1 : 0);
  if (in == 3) return setup_triangle(screen_of(c0, W, H), screen_of(c1, W, H), screen_of(c2, W, H), W, H, t0) ? 1 : 0;
  if (in == 0) return 0;
  // the corner that starts the polygon: the one in front (in == 1) or the one after the corner behind (in == 2)
  const int lone = in == 1 ? (c0.z >= 0.0f ? 0 : (c1.z >= 0.0f ? 1 : 2)) : (c0.z < 0.0f ? 0 : (c1.z < 0.0f ? 1 : 2));
  const int ia = in == 1 ? lone : (lone + 1) % 3;
  const float4 A = pick3(ia, c0, c1, c2), B = pick3((ia + 1) % 3, c0, c1, c2), C = pick3((ia + 2) % 3, c0, c1, c2);
  const float4 sa = screen_of(A, W, H);
  if (in == 1)
    return setup_triangle(sa, screen_of(crossing(A, B), W, H), screen_of(crossing(A, C), W, H), W, H, t0) ? 1 : 0;
  const float4 sbc = screen_of(crossing(B, C), W, H);
  const bool first = setup_triangle(sa, screen_of(B, W, H), sbc, W, H, t0);
  const bool second = setup_triangle(sa, sbc, screen_of(crossing(A, C), W, H), W, H, t1);
  if (!first && second) t0 = t1;
  return int(first) + int(second);
}

// lodBlendMask (lodBlend.ts:36-45) at pixel (px, py): true when the pixel's step lies in [lo, hi).
__device__ __forceinline__ bool blend_keep(int px, int py, uint32_t frame, uint32_t lo, uint32_t hi) {
  const float x = (float(px) + 0.5f) + float(frame) * 5.588238f, y = float(py) + 0.5f;
  const float a = x * 0.06711056f + y * 0.00583715f;
  const float b = (a - floorf(a)) * 52.9829189f;
  const float step = floorf((b - floorf(b)) * 255.0f);
  return step >= float(lo) && step < float(hi);
}

// One pixel of t: covered when its centre is inside the three edge functions (edges included); the depth is the
// screen-space interpolation of the corners' NDC depths, kept as a minimum (depth >= 0, so the unsigned order of
// the bits is the float order; the atomics' results are unused, so they do not wait).
template <bool VIS>
__device__ __forceinline__ void shade_pixel(const RasterArgs &R, const ScreenTri &t, const TriTag &g, int px, int py) {
  const float x = float(px) + 0.5f, y = float(py) + 0.5f;
  const float wa = (t.cx - t.bx) * (y - t.by) - (t.cy - t.by) * (x - t.bx);  // edge B -> C
  const float wb = (t.ax - t.cx) * (y - t.cy) - (t.ay - t.cy) * (x - t.cx);  // edge C -> A
  const float wc = (t.bx - t.ax) * (y - t.ay) - (t.by - t.ay) * (x - t.ax);  // edge A -> B
  if (wa >= 0.0f && wb >= 0.0f && wc >= 0.0f && (!VIS || blend_keep(px, py, R.frame, g.lo, g.hi))) {
    float z = ((wa * t.az + wb * t.bz) + wc * t.cz) / t.area;
    z = z > 0.0f ? z : 0.0f;  // +0 for rounding below zero (and never -0, whose bits would sort last)
    const size_t at = (size_t)py * R.width + px;
    if (VIS)
      atomicMin(R.vis + at, ((unsigned long long)__float_as_uint(z) << 32) | g.id);
    else
      atomicMin(R.depth[g.id] + at, __float_as_uint(z));
  }
}

__device__ __forceinline__ void write_record(float4 *r, const ScreenTri &t, uint32_t tx, const TriTag &g) {
  r[0] = make_float4(t.ax, t.ay, t.az, t.bx);
  r[1] = make_float4(t.by, t.bz, t.cx, t.cy);
  r[2] = make_float4(t.cz, t.area, __int_as_float(t.x0), __int_as_float(t.y0));
  r[3] = make_float4(__int_as_float(t.x1), __int_as_float(t.y1), __uint_as_float(tx), 0.0f);
  r[4] = make_float4(__uint_as_float(g.lo), __uint_as_float(g.hi), __uint_as_float(g.id), 0.0f);
}

__device__ __forceinline__ ScreenTri read_record(const float4 *r, uint32_t &tx, TriTag &g) {
  const float4 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4];
  ScreenTri t;
  t.ax = r0.x, t.ay = r0.y, t.az = r0.z, t.bx = r0.w;
  t.by = r1.x, t.bz = r1.y, t.cx = r1.z, t.cy = r1.w;
  t.cz = r2.x, t.area = r2.y, t.x0 = __float_as_int(r2.z), t.y0 = __float_as_int(r2.w);
  t.x1 = __float_as_int(r3.x), t.y1 = __float_as_int(r3.y);
  tx = __float_as_uint(r3.z);
  g.lo = __float_as_uint(r4.x), g.hi = __float_as_uint(r4.y), g.id = __float_as_uint(r4.z);
  return t;
}

// The whole warp over t's bounding box, 32 consecutive pixels (row-major) per step.
template <bool VIS>
__device__ __forceinline__ void warp_draw(const RasterArgs &R, const ScreenTri &t, const TriTag &g, uint32_t lane) {
  const uint32_t bw = uint32_t(t.x1 - t.x0 + 1), count = bw * uint32_t(t.y1 - t.y0 + 1);
  const uint32_t q = 32 / bw, r = 32 % bw;  // a step of 32 pixels: q rows and r columns
  uint32_t x = lane % bw, y = lane / bw;
  for (uint32_t i = lane; i < count; i += 32) {
    shade_pixel<VIS>(R, t, g, t.x0 + int(x), t.y0 + int(y));
    x += r, y += q;
    if (x >= bw) x -= bw, y++;
  }
}

__device__ __forceinline__ uint32_t warp_scan_incl(uint32_t v) {
  const uint32_t lane = threadIdx.x & 31;
#pragma unroll
  for (uint32_t o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Per warp: the small triangles of one round, staged so that the warp can draw their pixels 32 at a time whatever
// triangle they belong to (structure of arrays: lanes reading different triangles hit different banks).
struct SmallStage {
  float ax[32], ay[32], az[32], bx[32], by[32], bz[32], cx[32], cy[32], cz[32], area[32];
  int x0[32], y0[32];
  uint32_t bw[32], lo[32], hi[32], id[32];
};

// One triangle per lane of the warp (ok: set up; t, g: its setup and tag). Small triangles are drawn here; medium
// and large ones are queued, one reservation of each kind for the whole warp (the atomics are issued before the small
// triangles are drawn, so that their round trips overlap the drawing). Returns true for a lane whose triangle a full
// queue turned away: the caller draws it with the whole warp.
template <bool VIS>
__device__ bool queue_triangles(const RasterArgs &R, SmallStage &sm, uint32_t sub, uint32_t lane, bool ok,
                                const ScreenTri &t, const TriTag &g) {
  const uint32_t px = ok ? uint32_t(t.x1 - t.x0 + 1) * uint32_t(t.y1 - t.y0 + 1) : 0u;
  const bool medium = px > kLaneRasterMax && px <= kWarpRasterMax, large = px > kWarpRasterMax;
  const uint32_t mm = __ballot_sync(0xffffffffu, medium), lm = __ballot_sync(0xffffffffu, large);
  const uint32_t tx = large ? (uint32_t(t.x1 - t.x0) + kTileW) / kTileW : 0u;
  const uint32_t nt = large ? tx * ((uint32_t(t.y1 - t.y0) + kTileH) / kTileH) : 0u;
  uint32_t ts = 0, total = 0;
  if (lm) {
    ts = warp_scan_incl(nt) - nt;
    total = __shfl_sync(0xffffffffu, ts + nt, 31);
  }
  uint32_t at_m = 0, tri = 0;
  unsigned long long at_t = 0;
  if (lane == 0) {
    if (mm) at_m = atomicAdd(R.ctl + 4 + sub, __popc(mm));
    if (lm) {
      tri = atomicAdd(R.ctl + 1, __popc(lm));
      at_t = atomicAdd(reinterpret_cast<unsigned long long *>(R.ctl + 2), (unsigned long long)total);
    }
  }
  // small triangles: their bounding-box pixels laid end to end in lane order, 32 per step (a lane per pixel), so a
  // step's cost does not follow the largest small triangle of the round
  const uint32_t n_small = (px && px <= kLaneRasterMax) ? px : 0u;
  const uint32_t incl = warp_scan_incl(n_small), all = __shfl_sync(0xffffffffu, incl, 31);
  if (all) {
    if (n_small) {
      sm.ax[lane] = t.ax, sm.ay[lane] = t.ay, sm.az[lane] = t.az, sm.bx[lane] = t.bx, sm.by[lane] = t.by;
      sm.bz[lane] = t.bz, sm.cx[lane] = t.cx, sm.cy[lane] = t.cy, sm.cz[lane] = t.cz, sm.area[lane] = t.area;
      sm.x0[lane] = t.x0, sm.y0[lane] = t.y0, sm.bw[lane] = uint32_t(t.x1 - t.x0 + 1);
      sm.lo[lane] = g.lo, sm.hi[lane] = g.hi, sm.id[lane] = g.id;
    }
    __syncwarp();
    for (uint32_t base = 0; base < all; base += 32) {
      const uint32_t p = base + lane;
      // owner: the first lane whose inclusive end exceeds p
      uint32_t j = 0;
#pragma unroll
      for (uint32_t k = 16; k > 0; k >>= 1) {
        const uint32_t e = __shfl_sync(0xffffffffu, incl, j + k - 1);
        if (e <= p) j += k;
      }
      const uint32_t start = __shfl_sync(0xffffffffu, incl - n_small, j);
      if (p < all) {
        ScreenTri u;
        u.ax = sm.ax[j], u.ay = sm.ay[j], u.az = sm.az[j], u.bx = sm.bx[j], u.by = sm.by[j], u.bz = sm.bz[j];
        u.cx = sm.cx[j], u.cy = sm.cy[j], u.cz = sm.cz[j], u.area = sm.area[j];
        const TriTag h{sm.lo[j], sm.hi[j], sm.id[j]};
        const uint32_t q = p - start, w = sm.bw[j];
        shade_pixel<VIS>(R, u, h, sm.x0[j] + int(q % w), sm.y0[j] + int(q / w));
      }
    }
    __syncwarp();  // the stage is rewritten by the next round
  }
  bool left = false;
  if (mm) {
    const uint32_t at = __shfl_sync(0xffffffffu, at_m, 0) + __popc(mm & ((1u << lane) - 1u));
    if (medium && at < kQueuedMedium / kSubQueues)
      write_record(R.medium + ((size_t)at * kSubQueues + sub) * kRecord, t, 0u, g);
    else if (medium)
      left = true;
  }
  if (lm) {
    tri = __shfl_sync(0xffffffffu, tri, 0);
    at_t = __shfl_sync(0xffffffffu, at_t, 0);
    if (tri + __popc(lm) <= kQueuedLarge && at_t + total <= kTileUnits) {
      const uint32_t mine = tri + __popc(lm & ((1u << lane) - 1u));
      if (large) write_record(R.large + (size_t)mine * kRecord, t, tx, g);
      for (uint32_t rest = lm; rest; rest &= rest - 1) {  // the tile records, a triangle at a time
        const uint32_t j = __ffs(rest) - 1;
        const uint32_t nj = __shfl_sync(0xffffffffu, nt, j), sj = __shfl_sync(0xffffffffu, ts, j);
        const uint32_t tj = __shfl_sync(0xffffffffu, mine, j);
        for (uint32_t i = lane; i < nj; i += 32) R.tiles[at_t + sj + i] = make_uint2(tj, i);
      }
    } else {  // a queue is full: reserved tile slots below its capacity become empty records
      for (unsigned long long i = at_t + lane; i < at_t + total && i < kTileUnits; i += 32)
        R.tiles[i] = make_uint2(kNoTri, 0u);
      if (large) left = true;
    }
  }
  return left;
}

// The triangles a full queue turned away, one at a time, by the whole warp (left: this lane's).
template <bool VIS>
__device__ __forceinline__ void draw_left(const RasterArgs &R, uint32_t lane, bool left, const ScreenTri &t,
                                          const TriTag &g) {
  for (uint32_t pending = __ballot_sync(0xffffffffu, left); pending; pending &= pending - 1) {
    const uint32_t o = __ffs(pending) - 1;
    ScreenTri u;
    u.ax = __shfl_sync(0xffffffffu, t.ax, o), u.ay = __shfl_sync(0xffffffffu, t.ay, o);
    u.az = __shfl_sync(0xffffffffu, t.az, o), u.bx = __shfl_sync(0xffffffffu, t.bx, o);
    u.by = __shfl_sync(0xffffffffu, t.by, o), u.bz = __shfl_sync(0xffffffffu, t.bz, o);
    u.cx = __shfl_sync(0xffffffffu, t.cx, o), u.cy = __shfl_sync(0xffffffffu, t.cy, o);
    u.cz = __shfl_sync(0xffffffffu, t.cz, o), u.area = __shfl_sync(0xffffffffu, t.area, o);
    u.x0 = __shfl_sync(0xffffffffu, t.x0, o), u.x1 = __shfl_sync(0xffffffffu, t.x1, o);
    u.y0 = __shfl_sync(0xffffffffu, t.y0, o), u.y1 = __shfl_sync(0xffffffffu, t.y1, o);
    TriTag h;
    h.lo = __shfl_sync(0xffffffffu, g.lo, o), h.hi = __shfl_sync(0xffffffffu, g.hi, o);
    h.id = __shfl_sync(0xffffffffu, g.id, o);
    warp_draw<VIS>(R, u, h, lane);
  }
}

// Clears the occluder images (1.0f) and the queues' control words.
__global__ void __launch_bounds__(256) k_occluder_clear(const __grid_constant__ RasterArgs R, uint32_t count,
                                                        size_t pixels) {
  if (blockIdx.x == 0)
    for (uint32_t i = threadIdx.x; i < kCtlWords; i += blockDim.x) R.ctl[i] = 0;
  const size_t n = pixels * count;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    R.depth[i / pixels][i % pixels] = 0x3f800000u;
}

// Clears the image and the queues' control words.
template <typename T>
__global__ void __launch_bounds__(256) k_target_clear(T *image, size_t n, T value, uint32_t *ctl) {
  if (blockIdx.x == 0)
    for (uint32_t i = threadIdx.x; i < kCtlWords; i += blockDim.x) ctl[i] = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    image[i] = value;
}

// The images' entries laid end to end: first[v] = entries of images before v, first[count] = all (block-shared).
__device__ __forceinline__ void image_starts(const OccluderArgs &O, uint32_t *first) {
  if (threadIdx.x < 32) {
    uint32_t carry = 0;
    for (uint32_t v0 = 0; v0 < O.count; v0 += 32) {
      const uint32_t v = v0 + threadIdx.x;
      const uint32_t c = v < O.count ? min(O.img[v].counters[VGC_COUNTER_CUT0 + VGC_CUT_SELECTED], O.max_drawn) : 0u;
      const uint32_t incl = warp_scan_incl(c);
      if (v < O.count) first[v] = carry + incl - c;
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (threadIdx.x == 0) first[O.count] = carry;
  }
  __syncthreads();
}

// The image of laid-out entry e < first[count]: the last v with first[v] <= e.
__device__ __forceinline__ uint32_t image_of(const uint32_t *first, uint32_t count, uint32_t e) {
  uint32_t v = 0;
  for (uint32_t span = count; span > 1;) {
    const uint32_t half = span >> 1;
    if (first[v + half] <= e) v += half;
    span -= half;
  }
  return v;
}

__global__ void __launch_bounds__(128, 5) k_raster_occluders(Scene S, const __grid_constant__ OccluderArgs O,
                                                              const __grid_constant__ RasterArgs R) {
  __shared__ float4 verts[4][256];     // per warp: the current meshlet's vertices in screen space (local ids < 256)
  __shared__ uint32_t packed[4][128];  // ... and its packed triangles
  __shared__ SmallStage stage[4];
  __shared__ uint32_t first[kMaxImages + 1];
  SmallStage &sm = stage[threadIdx.x >> 5];
  float4 *sv = verts[threadIdx.x >> 5];
  uint32_t *st = packed[threadIdx.x >> 5];
  const uint32_t lane = threadIdx.x & 31;
  image_starts(O, first);
  const uint32_t n = first[O.count];
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  const float W = float(R.width), H = float(R.height);
  const uint32_t sub = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) % kSubQueues;  // this warp's medium sub-queue
  // Each step waits on memory several times (entry, instance and meshlet, vertices, triangles): the loads of a step
  // are issued together, and the next entry is fetched while this one is drawn. Entries of all images are laid end
  // to end; a warp's entry belongs to one image.
  uint32_t e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t v_next = e < n ? image_of(first, O.count, e) : 0u;
  uint4 next = e < n ? O.img[v_next].draw_list[e - first[v_next]] : make_uint4(0u, 0u, 0u, 0u);
  for (; e < n; e += warps) {
    const uint4 d = next;
    const uint32_t v = v_next;
    if (e + warps < n) {
      v_next = image_of(first, O.count, e + warps);
      next = O.img[v_next].draw_list[e + warps - first[v_next]];
    }
    const TriTag none{0u, 0u, v};  // the fragments' image
    if ((d.w & 0xffff00u) != (255u << 16)) continue;  // part 1 (blended): not an occluder
    const uint32_t slot = S.inst_slot[d.x];
    const float4 *col = S.inst + (size_t)d.x * 4;
    const float4 c0 = col[0], c1 = col[1], c2 = col[2], c3 = col[3];
    const uint4 info = S.m_info[d.y];
    if (!S.meshes[slot].occluder) continue;
    const uint32_t tris = d.w & 255u, first_tri = info.y / 3, voff = info.w;
    uint32_t pk[4];  // the meshlet's packed triangles (at most 128), loaded at once
#pragma unroll
    for (uint32_t r = 0; r < 4; r++) pk[r] = r * 32 + lane < tris ? S.m_tris[first_tri + r * 32 + lane] : 0u;
    // M's rows from the instance's columns, then clip = (P V) M p
    const float m[4][4] = {{c0.x, c1.x, c2.x, c3.x}, {c0.y, c1.y, c2.y, c3.y}, {c0.z, c1.z, c2.z, c3.z},
                           {c0.w, c1.w, c2.w, c3.w}};
    const float *vp = O.img[v].vp;
    float mvp[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
      for (int k = 0; k < 4; k++)
        mvp[r][k] = ((vp[r * 4] * m[0][k] + vp[r * 4 + 1] * m[1][k]) + vp[r * 4 + 2] * m[2][k]) + vp[r * 4 + 3] * m[3][k];
    // the meshlet's vertices (local ids 0 .. the largest its triangles use), each transformed once, 128 at a time
    uint32_t top = 0;
#pragma unroll
    for (uint32_t r = 0; r < 4; r++)
      top = max(top, max(pk[r] & 255u, max((pk[r] >> 8) & 255u, (pk[r] >> 16) & 255u)));
    top = __reduce_max_sync(0xffffffffu, top);
    __syncwarp();
#pragma unroll
    for (uint32_t r = 0; r < 4; r++) st[r * 32 + lane] = pk[r];
    for (uint32_t base = 0; base <= top; base += 128) {
      uint32_t id[4];
#pragma unroll
      for (uint32_t k = 0; k < 4; k++) id[k] = base + k * 32 + lane <= top ? S.m_verts[voff + base + k * 32 + lane] : 0u;
      float4 pos[4];
#pragma unroll
      for (uint32_t k = 0; k < 4; k++) pos[k] = base + k * 32 + lane <= top ? S.positions[id[k]] : make_float4(0, 0, 0, 1);
#pragma unroll
      for (uint32_t k = 0; k < 4; k++)
        if (base + k * 32 + lane <= top) sv[base + k * 32 + lane] = screen_vertex(mvp, pos[k], W, H);
    }
    __syncwarp();
    uint32_t left = 0;  // this lane's unclipped triangles turned away by a full queue (bit per round)
    for (uint32_t round = 0; round * 32 < tris; round++) {
      const uint32_t ti = round * 32 + lane, p = st[ti];
      ScreenTri t;
      bool ok = false, crossing = false;
      if (ti < tris) {
        const float4 a = sv[p & 255u], b = sv[(p >> 8) & 255u], c = sv[(p >> 16) & 255u];
        crossing = a.w == 0.0f || b.w == 0.0f || c.w == 0.0f;  // a corner behind the near plane
        if (!crossing) ok = setup_triangle(a, b, c, W, H, t);
      }
      // crossing triangles (rare) are clipped by k_raster_clipped: (entry, triangle) records, one atomic per warp
      const uint32_t cm = __ballot_sync(0xffffffffu, crossing);
      if (cm) {
        uint32_t at = 0;
        if (lane == __ffs(cm) - 1) at = atomicAdd(R.ctl + kClipCtl, __popc(cm));
        at = __shfl_sync(0xffffffffu, at, __ffs(cm) - 1) + __popc(cm & ((1u << lane) - 1u));
        if (crossing && at < kClipQueue) R.clip[at] = make_uint2(e - first[v], ti | (v << 8));
      }
      if (queue_triangles<false>(R, sm, sub, lane, ok, t, none)) left |= 1u << round;
    }
    for (uint32_t round = 0; round * 32 < tris; round++) {
      const uint32_t ti = round * 32 + lane, p = st[ti];
      const bool mine = (left >> round) & 1u;
      ScreenTri t;
      if (mine) setup_triangle(sv[p & 255u], sv[(p >> 8) & 255u], sv[(p >> 16) & 255u], W, H, t);
      draw_left<false>(R, lane, mine, t, none);
    }
    __syncwarp();  // the vertex and triangle buffers are rewritten by the next entry
  }
}

// The occluder pass's triangles that cross the near plane, a lane each: the draw-list entry's (P V M), the triangle's
// corners in clip space, clipped (setup_clipped), and its one or two screen triangles through the same size classes
// and queues (k_raster_queued runs after this kernel).
__global__ void __launch_bounds__(128) k_raster_clipped(Scene S, const __grid_constant__ OccluderArgs O,
                                                          const __grid_constant__ RasterArgs R) {
  __shared__ SmallStage stage[4];
  SmallStage &sm = stage[threadIdx.x >> 5];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = min(R.ctl[kClipCtl], kClipQueue);
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t sub = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) % kSubQueues;
  const float W = float(R.width), H = float(R.height);
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
    const uint32_t i = base + lane;
    ScreenTri t, t2;
    int k = 0;
    TriTag none{0u, 0u, 0u};  // the fragments' image
    if (i < n) {
      const uint2 rec = R.clip[i];
      const uint32_t v = rec.y >> 8;
      none.id = v;
      const float *vp = O.img[v].vp;
      const uint4 d = O.img[v].draw_list[rec.x];
      const float4 *col = S.inst + (size_t)d.x * 4;
      const float4 c0 = col[0], c1 = col[1], c2 = col[2], c3 = col[3];
      const float m[4][4] = {{c0.x, c1.x, c2.x, c3.x}, {c0.y, c1.y, c2.y, c3.y}, {c0.z, c1.z, c2.z, c3.z},
                             {c0.w, c1.w, c2.w, c3.w}};
      float mvp[4][4];
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int kk = 0; kk < 4; kk++)
          mvp[r][kk] = ((vp[r * 4] * m[0][kk] + vp[r * 4 + 1] * m[1][kk]) + vp[r * 4 + 2] * m[2][kk]) +
                       vp[r * 4 + 3] * m[3][kk];
      const uint4 info = S.m_info[d.y];
      const uint32_t p = S.m_tris[info.y / 3 + (rec.y & 255u)], voff = info.w;
      const float4 va = clip_vertex(mvp, S.positions[S.m_verts[voff + (p & 255u)]]);
      const float4 vb = clip_vertex(mvp, S.positions[S.m_verts[voff + ((p >> 8) & 255u)]]);
      const float4 vc = clip_vertex(mvp, S.positions[S.m_verts[voff + ((p >> 16) & 255u)]]);
      k = setup_clipped(va, vb, vc, W, H, t, t2);
    }
    const bool l = queue_triangles<false>(R, sm, sub, lane, k >= 1, t, none);
    draw_left<false>(R, lane, l, t, none);
    if (__any_sync(0xffffffffu, k == 2)) {
      const bool l2 = queue_triangles<false>(R, sm, sub, lane, k == 2, t2, none);
      draw_left<false>(R, lane, l2, t2, none);
    }
  }
}

// The queued triangles, spread over the whole grid: a warp per medium triangle, then a warp per tile of a large one
// (a lane per column of the tile).
template <bool VIS>
__global__ void __launch_bounds__(128) k_raster_queued(const __grid_constant__ RasterArgs R) {
  __shared__ uint32_t counts[kSubQueues];  // medium triangles per sub-queue
  __shared__ uint32_t most;
  if (threadIdx.x == 0) most = 0;
  __syncthreads();
  for (uint32_t q = threadIdx.x; q < kSubQueues; q += blockDim.x) {
    counts[q] = min(R.ctl[4 + q], kQueuedMedium / kSubQueues);
    atomicMax(&most, counts[q]);
  }
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  // medium records are interleaved: slot u holds record u / kSubQueues of sub-queue u % kSubQueues
  const uint32_t n_medium = most * kSubQueues;
  const uint32_t n = n_medium + (uint32_t)min(*reinterpret_cast<const unsigned long long *>(R.ctl + 2),
                                              (unsigned long long)kTileUnits);
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
    uint32_t tx;
    TriTag g;
    if (u < n_medium) {
      if (u / kSubQueues < counts[u % kSubQueues]) {
        const ScreenTri t = read_record(R.medium + (size_t)u * kRecord, tx, g);
        warp_draw<VIS>(R, t, g, lane);
      }
      continue;
    }
    const uint2 tile = R.tiles[u - n_medium];
    if (tile.x == kNoTri) continue;
    const ScreenTri t = read_record(R.large + (size_t)tile.x * kRecord, tx, g);
    const int px = t.x0 + int((tile.y % tx) * kTileW + lane), py0 = t.y0 + int((tile.y / tx) * kTileH);
    if (px > t.x1) continue;
    const int py1 = min(t.y1, py0 + int(kTileH) - 1);
    for (int py = py0; py <= py1; py++) shade_pixel<VIS>(R, t, g, px, py);
  }
}

// ------------------------------------------------------------------------------------------------ visibility
// Headless consumer of a cut (vgc_visibility): the cut's expanded index buffer drawn as the draw args say, with the
// reference's vertex pulling (GeometryPool.ts:1095-1131) and LOD blend mask (lodBlend.ts:36-45), into a visibility
// buffer: per pixel the 64-bit minimum of (depth bits << 32 | drawSlot << 7 | triangle in its meshlet).
//
//  * an index is (drawSlot << 7) | localVertex; drawSlot picks the draw-list entry (instance, meshlet), the local
//    vertex its meshletVertices entry and the position; the instance's model maps it to world space, shrunk toward
//    the instance origin by the draw-distance fade clamp((maxDrawDistance - |V origin|) / (0.15 maxDrawDistance),
//    0, 1), V the camera's view (GeometryPool.ts:1112-1119);
//  * triangles are set up as in the occluder pass (pixel centres, edges included, back faces and triangles reaching
//    in front of the near plane left out), one per lane, and drawn through the same size classes and queues;
//  * a fragment is kept when the step floor(255 n) of its pixel lies in the entry's blend range [lo, hi), n the
//    interleaved gradient noise fract(52.9829189 fract(0.06711056 x + 0.00583715 y)) at the pixel centre (x, y),
//    x shifted by 5.588238 per `frame` (lodBlendFrame);
//  * indices or entries outside the context's arrays (an index buffer not written by vgc_expand) drop their
//    triangle.
constexpr float kDrawDistanceFade = 0.15f;   // GeometryPool.ts:109

struct VisArgs {
  float vp[16];    // P * V, row-major
  float view[16];  // the camera's V (draw-distance fade), row-major
  uint32_t width, height, regions;  // regions: mesh slots * 2 (parts)
  const uint32_t *indices;
  uint64_t capacity;
  const uint4 *draw_list;  // the output slot's entries (draw slots of both cuts)
  const uint32_t *args;    // the cut's draw args, 5 u32 per (mesh slot, part)
  uint32_t draw_slots;     // entries in draw_list
  uint32_t meshlets, instances, meshlet_vertices, vertices;
};

// Screen-space vertex of index `idx` (w = 0: unusable), and its entry's draw slot and blend range.
// The clip-space position of index `idx` of the expanded buffer (ok: the index and its data are in range).
__device__ __forceinline__ float4 pulled_clip(const Scene &S, const VisArgs &A, uint32_t idx, bool &ok) {
  const uint32_t ds = idx >> kLocalVertexBits, lv = idx & ((1u << kLocalVertexBits) - 1u);
  ok = false;
  if (ds >= A.draw_slots) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const uint4 ent = A.draw_list[ds];
  if (ent.x >= A.instances || ent.y >= A.meshlets) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const MeshRec &mesh = S.meshes[S.inst_slot[ent.x]];
  const uint32_t mv = S.m_info[ent.y].w + lv;
  if (!mesh.vertices || mv >= A.meshlet_vertices) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const uint32_t vid = S.m_verts[mv];
  if (vid >= A.vertices) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  ok = true;
  const float4 p = S.positions[vid];
  const float4 *col = S.inst + (size_t)ent.x * 4;
  const float4 c0 = col[0], c1 = col[1], c2 = col[2], c3 = col[3];
  // draw-distance fade, from the camera's distance to the instance origin
  const float *V = A.view;
  const float ox = ((V[0] * c3.x + V[1] * c3.y) + V[2] * c3.z) + V[3];
  const float oy = ((V[4] * c3.x + V[5] * c3.y) + V[6] * c3.z) + V[7];
  const float oz = ((V[8] * c3.x + V[9] * c3.y) + V[10] * c3.z) + V[11];
  const float dist = sqrtf((ox * ox + oy * oy) + oz * oz);
  const float maxd = mesh.max_draw_distance;
  const float fade = fminf(fmaxf((maxd - dist) / (maxd * kDrawDistanceFade), 0.0f), 1.0f);
  const float wx = c3.x + ((c0.x * p.x + c1.x * p.y) + c2.x * p.z) * fade;
  const float wy = c3.y + ((c0.y * p.x + c1.y * p.y) + c2.y * p.z) * fade;
  const float wz = c3.z + ((c0.z * p.x + c1.z * p.y) + c2.z * p.z) * fade;
  float c[4];
#pragma unroll
  for (int r = 0; r < 4; r++) c[r] = ((A.vp[r * 4] * wx + A.vp[r * 4 + 1] * wy) + A.vp[r * 4 + 2] * wz) + A.vp[r * 4 + 3];
  return make_float4(c[0], c[1], c[2], c[3]);
}

// One lane per triangle of the cut, in region order (mesh slot, then part), as the draw args give them.
__global__ void __launch_bounds__(256) k_visibility(Scene S, VisArgs A, const __grid_constant__ RasterArgs R) {
  extern __shared__ uint32_t tri_start[];  // per region: first triangle in the laid-out order; [regions] = total
  __shared__ SmallStage stage[8];
  SmallStage &sm = stage[threadIdx.x >> 5];
  if (threadIdx.x < 32) {  // warp 0 scans the regions' triangle counts
    uint32_t carry = 0;
    for (uint32_t r0 = 0; r0 < A.regions; r0 += 32) {
      const uint32_t r = r0 + threadIdx.x;
      const uint32_t c = r < A.regions ? A.args[r * 5] / 3 : 0u;
      const uint32_t incl = warp_scan_incl(c);
      if (r < A.regions) tri_start[r] = carry + incl - c;
      carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (threadIdx.x == 0) tri_start[A.regions] = carry;
  }
  __syncthreads();
  const uint32_t total = tri_start[A.regions];
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t sub = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) % kSubQueues;  // this warp's medium sub-queue
  const uint32_t stride = gridDim.x * blockDim.x;
  // every lane of a warp runs the same number of steps (the warp draws its lanes' large triangles together)
  for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
    const uint32_t t_id = base + lane;
    ScreenTri t, t2;
    int n = 0;
    uint32_t lo = 0, hi = 0, payload = 0;
    if (t_id < total) {
      uint32_t r = 0, span = A.regions;  // the last region starting at or before t_id
      while (span > 1) {
        const uint32_t half = span >> 1;
        if (tri_start[r + half] <= t_id) r += half;
        span -= half;
      }
      const uint64_t first = (uint64_t)A.args[r * 5 + 2] + 3ull * (t_id - tri_start[r]);
      if (first + 2 < A.capacity) {
        const uint32_t i0 = A.indices[first], i1 = A.indices[first + 1], i2 = A.indices[first + 2];
        bool k0, k1, k2;
        const float4 v0 = pulled_clip(S, A, i0, k0), v1 = pulled_clip(S, A, i1, k1), v2 = pulled_clip(S, A, i2, k2);
        if (k0 && k1 && k2) {
          const uint32_t ds = i0 >> kLocalVertexBits;
          const uint4 ent = A.draw_list[ds];
          lo = (ent.w >> 8) & 255u, hi = (ent.w >> 16) & 255u;
          const uint32_t tri = uint32_t((first - A.args[r * 5 + 2] - ent.z) / 3);
          payload = (ds << kLocalVertexBits) | (tri & ((1u << kLocalVertexBits) - 1u));
          n = setup_clipped(v0, v1, v2, float(A.width), float(A.height), t, t2);
        }
      }
    }
    const TriTag g{lo, hi, payload};
    const bool left = queue_triangles<true>(R, sm, sub, lane, n >= 1, t, g);
    draw_left<true>(R, lane, left, t, g);
    if (__any_sync(0xffffffffu, n == 2)) {  // the second triangle of a clipped quad
      const bool left2 = queue_triangles<true>(R, sm, sub, lane, n == 2, t2, g);
      draw_left<true>(R, lane, left2, t2, g);
    }
  }
}

}  // namespace

// The queues of the second kernel (allocated once per context; the passes of one context share them, so calls on
// different streams must not overlap).
static int raster_queues(vgc_context *ctx, RasterArgs &R) {
  const size_t medium_bytes = (size_t)kQueuedMedium * kRecord * 16, large_bytes = (size_t)kQueuedLarge * kRecord * 16;
  const size_t ctl_bytes = 2048;
  static_assert(kCtlWords * 4 <= ctl_bytes, "control words");
  const size_t tile_bytes = (size_t)kTileUnits * 8;
  const int rc = dev_alloc(ctx, ctx->d_raster, ctl_bytes + medium_bytes + large_bytes + tile_bytes + (size_t)kClipQueue * 8);
  if (rc) return rc;
  char *q = (char *)ctx->d_raster.ptr;
  R.ctl = (uint32_t *)q;
  R.medium = (float4 *)(q + ctl_bytes);
  R.large = (float4 *)(q + ctl_bytes + medium_bytes);
  R.tiles = (uint2 *)(q + ctl_bytes + medium_bytes + large_bytes);
  R.clip = (uint2 *)(q + ctl_bytes + medium_bytes + large_bytes + tile_bytes);
  return VGC_OK;
}

// Up to kMaxImages images of the occluder pass in one launch set (arguments checked): image i draws output slot
// slots[i] with views[i] into depth[i].
static int occluder_depth_images(vgc_context *ctx, uint32_t count, const uint32_t *slots, const vgc_view *views,
                                 float *const *depth, uint32_t width, uint32_t height, cudaStream_t st) {
  int rc;
  OccluderArgs O{};
  RasterArgs R{};
  O.count = count;
  O.max_drawn = ctx->opts.max_meshlets;
  for (uint32_t v = 0; v < count; v++) {
    OccluderImage &I = O.img[v];
    for (int r = 0; r < 4; r++)
      for (int c = 0; c < 4; c++) {
        double s = 0;
        for (int i = 0; i < 4; i++) s += views[v].proj[i * 4 + r] * views[v].view[c * 4 + i];
        I.vp[r * 4 + c] = (float)s;
      }
    I.draw_list = (const uint4 *)ctx->d_draw.ptr + (size_t)slots[v] * 2 * ctx->opts.max_meshlets;
    I.counters = (const uint32_t *)ctx->d_counters.ptr + (size_t)slots[v] * ctx->counter_words;
    R.depth[v] = reinterpret_cast<uint32_t *>(depth[v]);
  }
  R.width = width;
  R.height = height;
  if ((rc = raster_queues(ctx, R))) return rc;
  const size_t pixels = (size_t)width * height;
  k_occluder_clear<<<(unsigned)std::min<size_t>((pixels * count + 255) / 256, (size_t)ctx->sm_count * 16), 256, 0,
                     st>>>(R, count, pixels);
  CUDA_TRY(cudaGetLastError());
  if (ctx->positions.empty()) return VGC_OK;  // no mesh carries vertex data: nothing is an occluder
  // persistent grids of exactly the resident blocks: a grid-stride loop over a grid larger than one wave leaves the
  // blocks of the second wave their full share of the work after the first has finished
  static int per_sm[2] = {0, 0};
  if (!per_sm[0]) {
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0], k_raster_occluders, 128, 0));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1], k_raster_queued<false>, 128, 0));
  }
  k_raster_occluders<<<ctx->sm_count * std::max(1, per_sm[0]), 128, 0, st>>>(scene_of(ctx), O, R);
  CUDA_TRY(cudaGetLastError());
  k_raster_clipped<<<ctx->sm_count * 2, 128, 0, st>>>(scene_of(ctx), O, R);
  CUDA_TRY(cudaGetLastError());
  k_raster_queued<false><<<ctx->sm_count * std::max(1, per_sm[1]), 128, 0, st>>>(R);
  CUDA_TRY(cudaGetLastError());
  return VGC_OK;
}

static int occluder_checks(vgc_context *ctx, uint32_t src_slot, const vgc_view *view, const float *depth,
                           uint32_t width, uint32_t height) {
  if (!ctx || !view || !depth) return fail(VGC_INVALID_ARG, "null argument");
  if (width == 0 || height == 0 || width > 16384 || height > 16384)
    return fail(VGC_INVALID_ARG, "occluder depth size must be 1..16384 per side");
  if (src_slot >= ctx->out_slots) return fail(VGC_NOT_FOUND, "output slot not allocated");
  return VGC_OK;
}

extern "C" int vgc_occluder_depth(vgc_context *ctx, uint32_t src_slot, const vgc_view *view, float *depth,
                                  uint32_t width, uint32_t height, vgc_stream stream) {
  int rc = occluder_checks(ctx, src_slot, view, depth, width, height);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  if ((rc = sync_scene(ctx))) return rc;
  return occluder_depth_images(ctx, 1, &src_slot, view, &depth, width, height,
                               stream ? (cudaStream_t)stream : ctx->stream);
}

extern "C" int vgc_occluder_depth_batch(vgc_context *ctx, uint32_t count, const uint32_t *src_slots,
                                        const vgc_view *views, float *const *depth, uint32_t width, uint32_t height,
                                        vgc_stream stream) {
  if (!ctx || (count && (!src_slots || !views || !depth))) return fail(VGC_INVALID_ARG, "null argument");
  int rc;
  for (uint32_t i = 0; i < count; i++)
    if ((rc = occluder_checks(ctx, src_slots[i], &views[i], depth[i], width, height))) return rc;
  cudaSetDevice(ctx->device);
  if ((rc = sync_scene(ctx))) return rc;
  const cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  for (uint32_t i = 0; i < count; i += kMaxImages)
    if ((rc = occluder_depth_images(ctx, std::min(kMaxImages, count - i), src_slots + i, views + i, depth + i, width,
                                    height, st)))
      return rc;
  return VGC_OK;
}

extern "C" int vgc_visibility(vgc_context *ctx, uint32_t slot, uint32_t cut, const vgc_view *view,
                              const vgc_view *fade_view, const uint32_t *indices, uint64_t capacity, uint64_t *vis,
                              uint32_t width, uint32_t height, uint32_t frame, vgc_stream stream) {
  if (!ctx || !view || !indices || !vis || cut > 1) return fail(VGC_INVALID_ARG, "bad arguments");
  if (width == 0 || height == 0 || width > 16384 || height > 16384)
    return fail(VGC_INVALID_ARG, "visibility buffer size must be 1..16384 per side");
  if (slot >= ctx->out_slots) return fail(VGC_NOT_FOUND, "output slot not allocated");
  if (ctx->out_slot_capacity != ctx->slot_capacity)
    return fail(VGC_INVALID_ARG, "vgc_visibility: meshes were added since the cut; cut and expand again first");
  cudaSetDevice(ctx->device);
  int rc = sync_scene(ctx);
  if (rc) return rc;
  cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
  const vgc_view *fv = fade_view ? fade_view : view;
  VisArgs A{};
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) {
      double s = 0;
      for (int i = 0; i < 4; i++) s += view->proj[i * 4 + r] * view->view[c * 4 + i];
      A.vp[r * 4 + c] = (float)s;
      A.view[r * 4 + c] = (float)fv->view[c * 4 + r];
    }
  A.width = width;
  A.height = height;
  A.regions = ctx->out_slot_capacity * 2;
  A.indices = indices;
  A.capacity = capacity;
  A.draw_list = (const uint4 *)ctx->d_draw.ptr + (size_t)slot * 2 * ctx->opts.max_meshlets;
  A.args = (const uint32_t *)ctx->d_args.ptr + (size_t)slot * 2 * ctx->out_slot_capacity * 2 * 5 +
           (size_t)cut * ctx->out_slot_capacity * 2 * 5;
  A.draw_slots = 2 * ctx->opts.max_meshlets;
  A.meshlets = (uint32_t)ctx->m_info.size();
  A.instances = (uint32_t)ctx->inst_slot.size();
  A.meshlet_vertices = (uint32_t)ctx->m_verts.size();
  A.vertices = (uint32_t)ctx->positions.size();
  RasterArgs R{};
  R.width = width;
  R.height = height;
  R.vis = reinterpret_cast<unsigned long long *>(vis);
  R.frame = frame;
  if ((rc = raster_queues(ctx, R))) return rc;
  const size_t pixels = (size_t)width * height;
  k_target_clear<unsigned long long>
      <<<(unsigned)std::min<size_t>((pixels + 255) / 256, (size_t)ctx->sm_count * 16), 256, 0, st>>>(
          R.vis, pixels, (unsigned long long)VGC_VIS_EMPTY, R.ctl);
  CUDA_TRY(cudaGetLastError());
  if (ctx->positions.empty()) return VGC_OK;  // no mesh carries vertex data
  const size_t smem = (A.regions + 1) * sizeof(uint32_t);
  if (smem > 48 * 1024) return fail(VGC_INVALID_ARG, "too many mesh slots for vgc_visibility");
  int per_sm = 0, per_sm_queued = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_visibility, 256, smem));
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_queued, k_raster_queued<true>, 128, 0));
  k_visibility<<<ctx->sm_count * std::max(1, per_sm), 256, smem, st>>>(scene_of(ctx), A, R);
  CUDA_TRY(cudaGetLastError());
  k_raster_queued<true><<<ctx->sm_count * std::max(1, per_sm_queued), 128, 0, st>>>(R);
  CUDA_TRY(cudaGetLastError());
  return VGC_OK;
}
