/*
 * Oracle Part B driver (TEST INFRASTRUCTURE ONLY): compiles vg_pass.inc for float and double, and adds the
 * HZB builder, the portable log, the frustum-plane extraction and the margin explainer.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#include "vg_oracle.h"

/* Natural log from float basic operations and correctly rounded fused multiply-adds only, so the float mirror and
   the kernels agree bit for bit: x = m * 2^e with m in [sqrt(1/2), sqrt(2)), ln x = e ln 2 + 2 atanh(s), s = (m - 1) / (m + 1),
   2 atanh(s) = 2 (s + s^3/3 + s^5/5 + s^7/7 + s^9/9 + s^11/11) (Abramowitz & Stegun 4.1.27). */
float vgo_logf(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  if (isinf(x)) return x;
  union {
    float f;
    uint32_t u;
  } v = {x};
  int e = 0;
  if ((v.u >> 23) == 0) { /* subnormal */
    v.f = v.f * 8388608.0f;
    e = -23;
  }
  e += (int)((v.u >> 23) & 0xffu) - 127;
  v.u = (v.u & 0x7fffffu) | 0x3f800000u;
  float m = v.f;
  if (m > 1.41421356f) {
    m = m * 0.5f;
    e += 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float p = fmaf(s2, 0.0909090936f, 0.111111112f); /* Horner form with fused multiply-adds */
  p = fmaf(s2, p, 0.142857149f);
  p = fmaf(s2, p, 0.2f);
  p = fmaf(s2, p, 0.333333343f);
  p = s2 * p;
  float lnm = fmaf(s, p, s) * 2.0f;
  float fe = (float)e;
  return fmaf(fe, 0.693145752f, fmaf(fe, 1.42860677e-06f, lnm));
}

/* Inverse of a rigid column-major 4x4 (rotation + translation): R^T and -R^T t. */
static void oracle_rigid_inverse(const double *m, double *out) {
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

/* Frustum planes of a column-major matrix, [0,1] depth (WebGPU), each normalised by its normal's length:
   Gribb & Hartmann plane extraction from the rows of the clip matrix. */
static void oracle_planes(const double *me, double out[6][4]) {
  double p[6][4] = {
      {me[3] - me[0], me[7] - me[4], me[11] - me[8], me[15] - me[12]},
      {me[3] + me[0], me[7] + me[4], me[11] + me[8], me[15] + me[12]},
      {me[3] + me[1], me[7] + me[5], me[11] + me[9], me[15] + me[13]},
      {me[3] - me[1], me[7] - me[5], me[11] - me[9], me[15] - me[13]},
      {me[3] - me[2], me[7] - me[6], me[11] - me[10], me[15] - me[14]},
      {me[2], me[6], me[10], me[14]},
  };
  for (int i = 0; i < 6; i++) {
    double l = sqrt(p[i][0] * p[i][0] + p[i][1] * p[i][1] + p[i][2] * p[i][2]);
    double inv = l > 0 ? 1.0 / l : 0;
    for (int k = 0; k < 4; k++) out[i][k] = p[i][k] * inv;
  }
}

/* Frustum.setFromProjectionMatrix(m, WebGPUCoordinateSystem) (three.js, used at VirtualGeometry.ts:429-437) as the
   oracle computes it: six normalised planes (nx, ny, nz, constant) in three's order right, left, bottom, top, far,
   near. */
void vgo_frustum_planes(const double m[16], double out[24]) {
  double p[6][4];
  oracle_planes(m, p);
  memcpy(out, p, sizeof p);
}

#define REAL float
#define SFX(name) name##_f32
#define LOG vgo_logf
#define RINT rintf
#define SQRT sqrtf
#define FLOOR floorf
#define FABS fabsf
#define FMA fmaf
#include "vg_pass.inc"
#undef REAL
#undef SFX
#undef LOG
#undef RINT
#undef SQRT
#undef FLOOR
#undef FABS
#undef FMA

#define REAL double
#define SFX(name) name##_f64
#define LOG log
#define RINT rint
#define SQRT sqrt
#define FLOOR floor
#define FABS fabs
#define FMA fma
#include "vg_pass.inc"

int64_t vgo_hzb_build(const float *depth, uint32_t width, uint32_t height, float *out, uint64_t cap, uint32_t *levels,
                      uint32_t offset[16], uint32_t w[16], uint32_t h[16]) {
  uint32_t lw = width, lh = height, n = 0;
  uint64_t total = 0;
  for (;;) {
    offset[n] = (uint32_t)total;
    w[n] = lw;
    h[n] = lh;
    total += (uint64_t)lw * lh;
    n++;
    if ((lw == 1 && lh == 1) || n == 16) break;
    lw = lw > 1 ? (lw + 1) / 2 : 1;
    lh = lh > 1 ? (lh + 1) / 2 : 1;
  }
  if (total > cap) return -1;
  *levels = n;
  memcpy(out, depth, sizeof(float) * width * height);
  for (uint32_t i = 1; i < n; i++) {
    const float *src = out + offset[i - 1];
    float *dst = out + offset[i];
    uint32_t sw = w[i - 1], sh = h[i - 1];
    for (uint32_t y = 0; y < h[i]; y++)
      for (uint32_t x = 0; x < w[i]; x++) {
        uint32_t x0 = 2 * x, y0 = 2 * y;
        uint32_t x1 = x0 + 1 < sw ? x0 + 1 : sw - 1, y1 = y0 + 1 < sh ? y0 + 1 : sh - 1;
        float a = fmaxf(src[y0 * sw + x0], src[y0 * sw + x1]);
        float b = fmaxf(src[y1 * sw + x0], src[y1 * sw + x1]);
        dst[y * w[i] + x] = fmaxf(a, b);
      }
  }
  return (int64_t)total;
}

int vgo_cull_pass_f32(const vgo_scene *s, vgo_view *v, vgo_result *r, int threads) { return cull_pass_impl_f32(s, v, r, threads); }
int vgo_cull_pass_f64(const vgo_scene *s, vgo_view *v, vgo_result *r, int threads) { return cull_pass_impl_f64(s, v, r, threads); }

/* ---------------------------------------------------------------- margin explainer (double) */
static double slack(double a, double b) {
  double m = fmax(fabs(a), fabs(b));
  if (m < 1e-30) m = 1e-30;
  return fabs(a - b) / m;
}

static double floor_slack(double x) {
  double d = fabs(x - floor(x + 0.5));
  return d / fmax(fabs(x), 1.0);
}

static double hzb_slack(const viewk_f64 *k, const vgo_view *v, const double c[3], double radius) {
  double best = 1e300;
  double depth = -c[2];
  double near_depth = depth - radius;
  best = fmin(best, slack(near_depth, k->near_));
  if (!(near_depth > k->near_)) return best;
  double far_depth = depth + radius;
  double xlo = c[0] - radius, xhi = c[0] + radius, ylo = c[1] - radius, yhi = c[1] + radius;
  double min_x = fmin(xlo / near_depth, xlo / far_depth) * k->P0 - k->P8;
  double max_x = fmax(xhi / near_depth, xhi / far_depth) * k->P0 - k->P8;
  double min_y = fmin(ylo / near_depth, ylo / far_depth) * k->P5 - k->P9;
  double max_y = fmax(yhi / near_depth, yhi / far_depth) * k->P5 - k->P9;
  double min_z = k->P14 / near_depth - k->P10;
  best = fmin(best, slack(min_z, 1.0));
  if (!(min_z < 1)) return best;
  double W = v->hzb_width[0], H = v->hzb_height[0];
  best = fmin(best, floor_slack((min_x * 0.5 + 0.5) * W));
  best = fmin(best, floor_slack((max_x * 0.5 + 0.5) * W));
  best = fmin(best, floor_slack((0.5 - max_y * 0.5) * H));
  best = fmin(best, floor_slack((0.5 - min_y * 0.5) * H));
  /* the sampled maximum itself */
  double cc[3] = {c[0], c[1], c[2]};
  (void)cc;
  return best;
}

static double occl_slack(const viewk_f64 *k, const vgo_view *v, const bands_f64 *b, int on, const double c[3], double r) {
  if (!on || !k->occl_active) return 1e300;
  double margin = (fabs(c[2]) * b->high[0]) / k->proj_scale;
  double best = hzb_slack(k, v, c, r + margin);
  /* compare the nearest depth with the sampled maximum: recompute through the double test at +-margin */
  double grow = (r + margin) * VGO_MARGIN;
  int a = hzb_test_f64(k, v, c, r + margin - grow), bb = hzb_test_f64(k, v, c, r + margin + grow);
  if (a != bb) best = 0;
  /* the depth comparison itself (nearest depth against the sampled maximum + 1e-6, both near 1) */
  double zmin, zmax;
  if (hzb_sample_f64(k, v, c, r + margin, &zmin, &zmax)) best = fmin(best, slack(zmin, zmax + 1e-6));
  return best;
}

double vgo_explain_f64(const vgo_scene *s, const vgo_view *v, uint32_t cut, uint32_t instance, uint32_t meshlet) {
  viewk_f64 K;
  view_setup_f64(v, &K);
  /* the bands the frame's final cut ran with: its threshold (the budget search's pick) and controller scales */
  if (v->triangle_budget > 0) K.error_threshold = v->chosen_threshold;
  uint32_t state[8];
  memcpy(state, v->state, sizeof state);
  if (v->cut_state[cut & 1][0]) {
    state[0] = v->cut_state[cut & 1][0];
    state[1] = v->cut_state[cut & 1][1];
  }
  bands_f64 B;
  load_bands_f64(&K, state, &B);
  double best = 1e300;
  /* the cell holding the instance */
  uint32_t cell = 0;
  for (; cell < s->cell_count; cell++) {
    const float *cd = s->cell_data + (size_t)cell * 8;
    uint32_t first = (uint32_t)cd[6], count = (uint32_t)cd[7];
    if (instance >= first && instance < first + count) break;
  }
  if (cell == s->cell_count) return best;
  const float *cd = s->cell_data + (size_t)cell * 8;
  uint32_t slot = (uint32_t)cd[5];
  {
    double c[3];
    xform_f64(K.V, cd[0], cd[1], cd[2], c);
    double radius = cd[3];
    if (K.frustum) best = fmin(best, slack(frustum_f64(&K, c, s->mesh_shadow[slot] != 0), -radius));
    double min_pixels = fmax(K.min_pixel_radius, s->mesh_min_pixel_radius[slot]);
    double max_r = cd[4];
    double gap = len3_f64(c) - radius;
    best = fmin(best, slack(gap, max_r));
    best = fmin(best, slack((max_r * K.proj_scale) / fmax(gap, 1e-6), min_pixels));
    best = fmin(best, slack(gap, s->mesh_max_draw_distance[slot]));
  }
  double VM[3][4], scale;
  model_view_f64(&K, s->instance_matrices + (size_t)instance * 16, VM, &scale);
  const float *sph = s->mesh_sphere + slot * 4;
  double c[3];
  xform_f64(VM, sph[0], sph[1], sph[2], c);
  double radius = sph[3] * scale;
  if (K.frustum) {
    best = fmin(best, slack(frustum_f64(&K, c, 0), -radius));
    if (cut == 1) best = fmin(best, slack(frustum_f64(&K, c, 1), -radius));
  }
  double vd = len3_f64(c);
  double min_pixels = fmax(K.min_pixel_radius, s->mesh_min_pixel_radius[slot]);
  best = fmin(best, slack(vd, radius));
  best = fmin(best, slack((radius * K.proj_scale) / vd, min_pixels));
  best = fmin(best, slack(vd - radius, s->mesh_max_draw_distance[slot]));
  int occl_on = s->mesh_occlusion[slot] != 0;
  if (cut == 0) best = fmin(best, occl_slack(&K, v, &B, occl_on, c, radius));
  const float *lb = s->mesh_lod_bounds + slot * 4;
  double lc[3];
  xform_f64(VM, lb[0], lb[1], lb[2], lc);
  double d = len3_f64(lc), r = lb[3] * scale;
  double px_min = (scale * K.proj_scale) / fmax(d - r, K.near_);
  double px_max = (scale * K.proj_scale) / fmax(d + r, K.near_);
  double low = B.low[cut], high = B.high[cut];
  uint32_t levels = s->mesh_level_count[slot] < 48 ? s->mesh_level_count[slot] : 48;
  uint32_t base = s->mesh_level_base[slot];
  for (uint32_t l = 0; l < levels; l++) {
    double min_own = s->level_errors[(base + l) * 2], max_parent = s->level_errors[(base + l) * 2 + 1];
    double max_own = s->level_guard_errors[(base + l) * 2], min_parent = s->level_guard_errors[(base + l) * 2 + 1];
    best = fmin(best, slack(min_own * px_max, high));
    if (max_parent < 5e29) best = fmin(best, slack(max_parent * px_min, low));
    best = fmin(best, slack(max_own * px_min, low * (1 - 1e-3)));
    if (min_parent < 5e29) best = fmin(best, slack(min_parent * px_max, high * (1 + 1e-3)));
  }
  {
    const float *cb = s->mesh_cull_bounds + slot * 4;
    double cc[3];
    xform_f64(VM, cb[0], cb[1], cb[2], cc);
    if (K.frustum) best = fmin(best, slack(frustum_f64(&K, cc, cut == 1), cb[3] * scale));
  }
  const float *bd = s->meshlet_bounds + (size_t)meshlet * 16;
  double mc[3];
  xform_f64(VM, bd[12], bd[13], bd[14], mc);
  double mr = bd[15] * scale;
  if (K.frustum) best = fmin(best, slack(frustum_f64(&K, mc, cut == 1), -mr));
  if (cut == 0) best = fmin(best, occl_slack(&K, v, &B, occl_on, mc, mr));
  double own = proj_error_f64(&K, VM, scale, bd, bd[8]);
  double parent = proj_error_f64(&K, VM, scale, bd + 4, bd[9]);
  best = fmin(best, slack(own, high));
  if (parent < 5e29) best = fmin(best, slack(parent, low));
  if (B.fade_scale > 0) {
    double xs[2] = {own, parent};
    for (int i = 0; i < 2; i++) {
      if (xs[i] >= 5e29) continue;
      double x = log(fmax(xs[i], 1e-30) / low) * B.fade_scale;
      double dist = fabs(x - (floor(x) + 0.5));
      best = fmin(best, dist / B.fade_scale);
    }
  }
  return best;
}
