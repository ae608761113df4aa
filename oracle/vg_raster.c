/* Oracle (test infrastructure only): C restatement of the occluder depth pass of the cut engine, which stands in for
 * the reference's occluder render (OcclusionCulling.ts:244-273: the occluders' previous-frame camera cuts drawn
 * depth-only with the current camera, vertices pulled as in GeometryPool.ts:1095-1131). Same arithmetic, in the
 * same order, as the CUDA rasterizer, so the depth images agree bit for bit:
 *   clip = (P V M) p; a triangle is clipped against the near plane (clip.z >= 0) into one or two triangles, and
 *   dropped when it faces away;
 *   pixel centres inside the three edge functions (edges included) take the screen-space interpolation of the
 *   vertices' NDC depths, kept as a per-pixel minimum over an image cleared to 1.
 * Built with -ffp-contract=off. */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "vg_oracle.h"

typedef struct {
  float ax, ay, az, bx, by, bz, cx, cy, cz, area;
  int x0, x1, y0, y1;
} raster_tri;

/* a clip-space vertex in screen space (x, y in pixels, y down; NDC depth; 1 when in front of the near plane, else all 0) */
static void raster_screen(const float c[4], float W, float H, float out[4]) {
  if (!(c[3] > 0.0f) || !(c[2] >= 0.0f)) {
    out[0] = out[1] = out[2] = out[3] = 0.0f;
    return;
  }
  const float nx = c[0] / c[3], ny = c[1] / c[3], nz = c[2] / c[3];
  out[0] = (nx * 0.5f + 0.5f) * W;
  out[1] = (0.5f - ny * 0.5f) * H;
  out[2] = nz;
  out[3] = 1.0f;
}

static int raster_tri_setup(const float *v0, const float *v1, const float *v2, float W, float H, raster_tri *t) {
  if (v0[3] == 0.0f || v1[3] == 0.0f || v2[3] == 0.0f) return 0;
  const float area0 = (v1[0] - v0[0]) * (v2[1] - v0[1]) - (v2[0] - v0[0]) * (v1[1] - v0[1]);
  if (!(area0 < 0.0f)) return 0;
  t->ax = v0[0], t->ay = v0[1], t->az = v0[2];
  t->bx = v2[0], t->by = v2[1], t->bz = v2[2];
  t->cx = v1[0], t->cy = v1[1], t->cz = v1[2];
  t->area = (t->bx - t->ax) * (t->cy - t->ay) - (t->cx - t->ax) * (t->by - t->ay);
  if (!(t->area > 0.0f)) return 0;
  float mnx = fminf(fminf(t->ax, t->bx), t->cx), mxx = fmaxf(fmaxf(t->ax, t->bx), t->cx);
  float mny = fminf(fminf(t->ay, t->by), t->cy), mxy = fmaxf(fmaxf(t->ay, t->by), t->cy);
  mnx = fmaxf(mnx, -1.0f), mxx = fminf(mxx, W + 1.0f);
  mny = fmaxf(mny, -1.0f), mxy = fminf(mxy, H + 1.0f);
  int x0 = (int)ceilf(mnx - 0.5f), x1 = (int)floorf(mxx - 0.5f);
  int y0 = (int)ceilf(mny - 0.5f), y1 = (int)floorf(mxy - 0.5f);
  t->x0 = x0 > 0 ? x0 : 0;
  t->x1 = x1 < (int)W - 1 ? x1 : (int)W - 1;
  t->y0 = y0 > 0 ? y0 : 0;
  t->y1 = y1 < (int)H - 1 ? y1 : (int)H - 1;
  return t->x0 <= t->x1 && t->y0 <= t->y1;
}

/* the crossing point of edge P -> Q (P in front) with the near plane: P + s (Q - P), s = P.z / (P.z - Q.z), depth 0 */
static void raster_crossing(const float *p, const float *q, float out[4]) {
  const float s = p[2] / (p[2] - q[2]);
  out[0] = p[0] + s * (q[0] - p[0]);
  out[1] = p[1] + s * (q[1] - p[1]);
  out[2] = 0.0f;
  out[3] = p[3] + s * (q[3] - p[3]);
}

/* Near-plane clipping of a triangle in clip space (clip.z >= 0 kept), then its screen triangles: t[0] (and t[1]);
   returns how many (0..2). With A the corner in front (one in front) or the corner after the one behind (two in
   front) in the order c0 -> c1 -> c2, and B, C the next ones: one in front -> (A, AB, CA); two in front ->
   (A, B, BC) and (A, BC, CA). A triangle wholly in front is set up from its screen corners unchanged. */
static int raster_clipped(const float c[3][4], float W, float H, raster_tri t[2]) {
  const int in = (c[0][2] >= 0.0f) + (c[1][2] >= 0.0f) + (c[2][2] >= 0.0f);
  float s0[4], s1[4], s2[4];
  if (in == 3) {
    raster_screen(c[0], W, H, s0);
    raster_screen(c[1], W, H, s1);
    raster_screen(c[2], W, H, s2);
    return raster_tri_setup(s0, s1, s2, W, H, &t[0]);
  }
  if (in == 0) return 0;
  const int lone = in == 1 ? (c[0][2] >= 0.0f ? 0 : (c[1][2] >= 0.0f ? 1 : 2))
                            : (c[0][2] < 0.0f ? 0 : (c[1][2] < 0.0f ? 1 : 2));
  const int ia = in == 1 ? lone : (lone + 1) % 3;
  const float *A = c[ia], *B = c[(ia + 1) % 3], *C = c[(ia + 2) % 3];
  float x[4], y[4], sa[4];
  raster_screen(A, W, H, sa);
  if (in == 1) {
    raster_crossing(A, B, x);
    raster_crossing(A, C, y);
    raster_screen(x, W, H, s1);
    raster_screen(y, W, H, s2);
    return raster_tri_setup(sa, s1, s2, W, H, &t[0]);
  }
  raster_crossing(B, C, x);
  raster_screen(x, W, H, s2); /* BC */
  raster_screen(B, W, H, s1);
  const int first = raster_tri_setup(sa, s1, s2, W, H, &t[0]);
  raster_crossing(A, C, y);
  float s3[4];
  raster_screen(y, W, H, s3);
  const int second = raster_tri_setup(sa, s2, s3, W, H, &t[1]);
  if (!first && second) t[0] = t[1];
  return first + second;
}

int vgo_occluder_depth(const uint32_t *entries, uint32_t n, const float *inst, const uint32_t *inst_slot,
                       const uint32_t *slot_occluder, const uint32_t *m_info, const uint32_t *m_tris,
                       const uint32_t *m_verts, const float *positions, const double *view, const double *proj,
                       uint32_t width, uint32_t height, float *depth) {
  float vp[16];
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) {
      double s = 0;
      for (int i = 0; i < 4; i++) s += proj[i * 4 + r] * view[c * 4 + i];
      vp[r * 4 + c] = (float)s;
    }
  for (size_t i = 0; i < (size_t)width * height; i++) depth[i] = 1.0f;
  const float W = (float)width, H = (float)height;
  for (uint32_t e = 0; e < n; e++) {
    const uint32_t *d = entries + (size_t)e * 4;
    if ((d[3] & 0xffff00u) != (255u << 16)) continue;
    if (!slot_occluder[inst_slot[d[0]]]) continue;
    const float *col = inst + (size_t)d[0] * 16; /* 4 columns */
    float m[4][4], mvp[4][4];
    for (int r = 0; r < 4; r++)
      for (int c = 0; c < 4; c++) m[r][c] = col[c * 4 + r];
    for (int r = 0; r < 4; r++)
      for (int k = 0; k < 4; k++)
        mvp[r][k] = ((vp[r * 4] * m[0][k] + vp[r * 4 + 1] * m[1][k]) + vp[r * 4 + 2] * m[2][k]) + vp[r * 4 + 3] * m[3][k];
    const uint32_t *info = m_info + (size_t)d[1] * 4;
    const uint32_t tris = d[3] & 255u, first_tri = info[1] / 3, voff = info[3];
    for (uint32_t ti = 0; ti < tris; ti++) {
      const uint32_t p = m_tris[first_tri + ti];
      float c[3][4];
      for (int k = 0; k < 3; k++) {
        const float *v = positions + (size_t)m_verts[voff + ((p >> (8 * k)) & 255u)] * 3;
        for (int r = 0; r < 4; r++) c[k][r] = ((mvp[r][0] * v[0] + mvp[r][1] * v[1]) + mvp[r][2] * v[2]) + mvp[r][3];
      }
      raster_tri tt[2];
      const int nt = raster_clipped(c, W, H, tt);
      for (int j = 0; j < nt; j++) {
        const raster_tri t = tt[j];
        for (int py = t.y0; py <= t.y1; py++)
          for (int px = t.x0; px <= t.x1; px++) {
            const float x = (float)px + 0.5f, y = (float)py + 0.5f;
            const float wa = (t.cx - t.bx) * (y - t.by) - (t.cy - t.by) * (x - t.bx);
            const float wb = (t.ax - t.cx) * (y - t.cy) - (t.ay - t.cy) * (x - t.cx);
            const float wc = (t.bx - t.ax) * (y - t.ay) - (t.by - t.ay) * (x - t.ax);
            if (wa >= 0.0f && wb >= 0.0f && wc >= 0.0f) {
              float z = ((wa * t.az + wb * t.bz) + wc * t.cz) / t.area;
              z = z > 0.0f ? z : 0.0f;
              float *o = depth + (size_t)py * width + px;
              if (z < *o) *o = z;
            }
          }
      }
    }
  }
  return 0;
}

/* ---- visibility buffer: the headless consumer of a cut (vgc_visibility), restated. An index of the expanded
 * buffer is (drawSlot << 7) | localVertex; vertex pulling follows GeometryPool.ts:1095-1131 (entry, meshletVertices,
 * position, model, draw-distance shrink toward the instance origin, DRAW_DISTANCE_FADE = 0.15 at :109) and the
 * fragment keep test lodBlend.ts:36-45 (interleaved gradient noise at the pixel centre, lodBlendFrame = frame).
 * Every pixel keeps the minimum of (depth bits << 32 | drawSlot << 7 | triangle in its meshlet). */
static const float kDrawDistanceFade = 0.15f;

typedef struct {
  const uint32_t *draw_list;
  uint32_t draw_slots;
  const float *inst;
  uint32_t instances;
  const uint32_t *inst_slot, *slot_vertices;
  const float *slot_max_draw_distance;
  const uint32_t *m_info;
  uint32_t meshlets;
  const uint32_t *m_verts;
  uint32_t meshlet_vertices;
  const float *positions;
  uint32_t vertices;
  float vp[16], view[16];
} vis_scene;

/* clip coordinates of index `idx`; 0 when an array index is out of range or the mesh has no vertex data */
static int vis_pull(const vis_scene *s, uint32_t idx, float c[4]) {
  const uint32_t ds = idx >> 7, lv = idx & 127u;
  if (ds >= s->draw_slots) return 0;
  const uint32_t *ent = s->draw_list + (size_t)ds * 4;
  if (ent[0] >= s->instances || ent[1] >= s->meshlets) return 0;
  const uint32_t slot = s->inst_slot[ent[0]];
  const uint32_t mv = s->m_info[(size_t)ent[1] * 4 + 3] + lv;
  if (!s->slot_vertices[slot] || mv >= s->meshlet_vertices) return 0;
  const uint32_t vid = s->m_verts[mv];
  if (vid >= s->vertices) return 0;
  const float *p = s->positions + (size_t)vid * 3;
  const float *col = s->inst + (size_t)ent[0] * 16;
  const float *c0 = col, *c1 = col + 4, *c2 = col + 8, *c3 = col + 12;
  const float *V = s->view;
  const float ox = ((V[0] * c3[0] + V[1] * c3[1]) + V[2] * c3[2]) + V[3];
  const float oy = ((V[4] * c3[0] + V[5] * c3[1]) + V[6] * c3[2]) + V[7];
  const float oz = ((V[8] * c3[0] + V[9] * c3[1]) + V[10] * c3[2]) + V[11];
  const float dist = sqrtf((ox * ox + oy * oy) + oz * oz);
  const float maxd = s->slot_max_draw_distance[slot];
  const float fade = fminf(fmaxf((maxd - dist) / (maxd * kDrawDistanceFade), 0.0f), 1.0f);
  const float wx = c3[0] + ((c0[0] * p[0] + c1[0] * p[1]) + c2[0] * p[2]) * fade;
  const float wy = c3[1] + ((c0[1] * p[0] + c1[1] * p[1]) + c2[1] * p[2]) * fade;
  const float wz = c3[2] + ((c0[2] * p[0] + c1[2] * p[1]) + c2[2] * p[2]) * fade;
  for (int r = 0; r < 4; r++) c[r] = ((s->vp[r * 4] * wx + s->vp[r * 4 + 1] * wy) + s->vp[r * 4 + 2] * wz) + s->vp[r * 4 + 3];
  return 1;
}

int vgo_blend_keep(int px, int py, uint32_t frame, uint32_t lo, uint32_t hi) {
  const float x = ((float)px + 0.5f) + (float)frame * 5.588238f, y = (float)py + 0.5f;
  const float a = x * 0.06711056f + y * 0.00583715f;
  const float b = (a - floorf(a)) * 52.9829189f;
  const float step = floorf((b - floorf(b)) * 255.0f);
  return step >= (float)lo && step < (float)hi;
}

int vgo_visibility(const uint32_t *indices, uint64_t capacity, const uint32_t *draw_list, uint32_t draw_slots,
                   const uint32_t *args, uint32_t regions, const float *inst, uint32_t instances,
                   const uint32_t *inst_slot, const uint32_t *slot_vertices, const float *slot_max_draw_distance,
                   const uint32_t *m_info, uint32_t meshlets, const uint32_t *m_verts, uint32_t meshlet_vertices,
                   const float *positions, uint32_t vertices, const double *view, const double *proj,
                   const double *fade_view, uint32_t width, uint32_t height, uint32_t frame, uint64_t *vis) {
  vis_scene s = {draw_list, draw_slots, inst, instances, inst_slot, slot_vertices, slot_max_draw_distance,
                 m_info, meshlets, m_verts, meshlet_vertices, positions, vertices, {0}, {0}};
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) {
      double acc = 0;
      for (int i = 0; i < 4; i++) acc += proj[i * 4 + r] * view[c * 4 + i];
      s.vp[r * 4 + c] = (float)acc;
      s.view[r * 4 + c] = (float)fade_view[c * 4 + r];
    }
  for (size_t i = 0; i < (size_t)width * height; i++) vis[i] = 0x3f800000ffffffffull;
  const float W = (float)width, H = (float)height;
  for (uint32_t rg = 0; rg < regions; rg++) {
    const uint32_t tris = args[rg * 5] / 3, start = args[rg * 5 + 2];
    for (uint32_t i = 0; i < tris; i++) {
      const uint64_t first = (uint64_t)start + 3ull * i;
      if (first + 2 >= capacity) continue;
      float c[3][4];
      int ok = 1;
      for (int k = 0; k < 3; k++) ok &= vis_pull(&s, indices[first + k], c[k]);
      if (!ok) continue;
      const uint32_t ds = indices[first] >> 7;
      const uint32_t *ent = draw_list + (size_t)ds * 4;
      const uint32_t lo = (ent[3] >> 8) & 255u, hi = (ent[3] >> 16) & 255u;
      const uint32_t payload = (ds << 7) | ((uint32_t)((first - start - ent[2]) / 3) & 127u);
      raster_tri tt[2];
      const int nt = raster_clipped(c, W, H, tt);
      for (int j = 0; j < nt; j++) {
        const raster_tri t = tt[j];
        for (int py = t.y0; py <= t.y1; py++)
          for (int px = t.x0; px <= t.x1; px++) {
            const float x = (float)px + 0.5f, y = (float)py + 0.5f;
            const float wa = (t.cx - t.bx) * (y - t.by) - (t.cy - t.by) * (x - t.bx);
            const float wb = (t.ax - t.cx) * (y - t.cy) - (t.ay - t.cy) * (x - t.cx);
            const float wc = (t.bx - t.ax) * (y - t.ay) - (t.by - t.ay) * (x - t.ax);
            if (wa >= 0.0f && wb >= 0.0f && wc >= 0.0f && vgo_blend_keep(px, py, frame, lo, hi)) {
              float z = ((wa * t.az + wb * t.bz) + wc * t.cz) / t.area;
              z = z > 0.0f ? z : 0.0f;
              uint32_t zb;
              memcpy(&zb, &z, 4);
              const uint64_t v = ((uint64_t)zb << 32) | payload;
              uint64_t *o = vis + (size_t)py * width + px;
              if (v < *o) *o = v;
            }
          }
      }
    }
  }
  return 0;
}
