/*
 * Part A of the oracle (TEST INFRASTRUCTURE ONLY): the reference's CPU cut evaluator restated in C, in double
 * precision like JavaScript numbers.
 *   vgo_lod_fade_range           <- src/core/runtime/lodBlend.ts:52-61
 *   vgo_select_cut               <- src/core/runtime/cut.ts:26-48
 *   vgo_select_blend_cut         <- src/core/runtime/cut.ts:56-77
 *   vgo_verify_overlap           <- src/core/runtime/cut.ts:83-97
 *   vgo_verify_coverage          <- src/core/runtime/cut.ts:104-122
 *   vgo_instance_meshlet_range   <- src/core/runtime/cut.ts:124-166
 *   vgo_instance_guaranteed_range<- src/core/runtime/cut.ts:180-215
 * JavaScript's Math.round rounds halves up (toward +infinity): floor(x + 0.5) here.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#include "vg_oracle.h"

static double js_round(double x) { return floor(x + 0.5); }

int vgo_lod_fade_range(double own, double parent, double threshold, double blend, int *lo, int *hi) {
  double high = blend > 1 ? threshold * blend : threshold;
  if (!(own <= high && parent > threshold)) return 0;
  if (!(blend > 1)) {
    *lo = 0;
    *hi = VGO_LOD_FADE_STEPS;
    return 1;
  }
  double scale = VGO_LOD_FADE_STEPS / log(blend);
  double el = log(fmax(own, 1e-30) / threshold) * scale;
  int l = (int)fmin(VGO_LOD_FADE_STEPS, fmax(0, js_round(el)));
  int h = VGO_LOD_FADE_STEPS;
  if (isfinite(parent)) {
    double eh = log(fmax(parent, 1e-30) / threshold) * scale;
    h = (int)fmin(VGO_LOD_FADE_STEPS, fmax(0, js_round(eh)));
  }
  if (!(h > l)) return 0;
  *lo = l;
  *hi = h;
  return 1;
}

/* projectedError of cut.ts:32-39: error in pixels of a sphere seen through viewMatrix (= view * model). */
static double projected_error(const double *v, double proj_scale, double near_, double s, double cx, double cy,
                              double cz, double r, double error) {
  if (error >= VGO_ERROR_INFINITY * 0.5) return INFINITY;
  double x = v[0] * cx + v[4] * cy + v[8] * cz + v[12];
  double y = v[1] * cx + v[5] * cy + v[9] * cz + v[13];
  double z = v[2] * cx + v[6] * cy + v[10] * cz + v[14];
  double distance = fmax(sqrt(x * x + y * y + z * z) - r * s, near_);
  return (error * s * proj_scale) / distance;
}

void vgo_select_cut(const float *B, uint32_t n, const double v[16], double proj_scale, double near_, double s,
                    double threshold, uint8_t *selected) {
  for (uint32_t i = 0; i < n; i++) {
    const float *b = B + (size_t)i * 16;
    double own = projected_error(v, proj_scale, near_, s, b[0], b[1], b[2], b[3], b[8]);
    double parent = projected_error(v, proj_scale, near_, s, b[4], b[5], b[6], b[7], b[9]);
    selected[i] = own <= threshold && parent > threshold ? 1 : 0;
  }
}

void vgo_select_blend_cut(const float *B, uint32_t n, const double v[16], double proj_scale, double near_, double s,
                          double threshold, double blend, uint8_t *lo, uint8_t *hi) {
  for (uint32_t i = 0; i < n; i++) {
    const float *b = B + (size_t)i * 16;
    double own = projected_error(v, proj_scale, near_, s, b[0], b[1], b[2], b[3], b[8]);
    double parent = projected_error(v, proj_scale, near_, s, b[4], b[5], b[6], b[7], b[9]);
    int l = 0, h = 0;
    if (vgo_lod_fade_range(own, parent, threshold, blend, &l, &h)) {
      lo[i] = (uint8_t)l;
      hi[i] = (uint8_t)h;
    } else {
      lo[i] = 0;
      hi[i] = 0;
    }
  }
}

/* Memoised recursion over the replacement links; its depth is bounded by the number of LOD levels. */
typedef struct walk_ctx {
  const int32_t *group;
  const uint32_t *start, *list;
  const uint8_t *selected;
  int8_t *memo; /* -1 unknown, 0 no, 1 yes */
} walk_ctx;

/* cut.ts:86-93: a selected meshlet among the coarser replacements of i, recursively */
static int below(walk_ctx *c, uint32_t i) {
  if (c->memo[i] != -1) return c->memo[i] == 1;
  int result = 0;
  int32_t g = c->group[i];
  if (g >= 0)
    for (uint32_t k = c->start[g]; !result && k < c->start[g + 1]; k++)
      result = c->selected[c->list[k]] == 1 || below(c, c->list[k]);
  c->memo[i] = (int8_t)result;
  return result;
}

/* cut.ts:108-115: i or one of its replacements (recursively) is selected */
static int covered(walk_ctx *c, uint32_t i) {
  if (c->memo[i] != -1) return c->memo[i] == 1;
  int result = c->selected[i] == 1;
  int32_t g = c->group[i];
  if (g >= 0)
    for (uint32_t k = c->start[g]; !result && k < c->start[g + 1]; k++) result = covered(c, c->list[k]);
  c->memo[i] = (int8_t)result;
  return result;
}

uint32_t vgo_verify_overlap(uint32_t n, const int32_t *group, const uint32_t *start, const uint32_t *list,
                            const uint8_t *selected, uint32_t *out) {
  walk_ctx c = {group, start, list, selected, (int8_t *)malloc(n ? n : 1)};
  memset(c.memo, -1, n);
  uint32_t count = 0;
  for (uint32_t i = 0; i < n; i++)
    if (selected[i] && below(&c, i)) out[count++] = i;
  free(c.memo);
  return count;
}

uint32_t vgo_verify_coverage(uint32_t n, const uint32_t *info, const int32_t *group, const uint32_t *start,
                             const uint32_t *list, const uint8_t *selected, uint32_t *out) {
  walk_ctx c = {group, start, list, selected, (int8_t *)malloc(n ? n : 1)};
  memset(c.memo, -1, n);
  uint32_t count = 0;
  for (uint32_t i = 0; i < n; i++)
    if (info[(size_t)i * 4 + 2] == 0 && !covered(&c, i)) out[count++] = i;
  free(c.memo);
  return count;
}

/* lodDistanceBounds of cut.ts:125-134 */
static void lod_distance_bounds(const float L[4], const double *v, double near_, double s, double *dmin, double *dmax) {
  double cx = L[0], cy = L[1], cz = L[2], r = L[3];
  double x = v[0] * cx + v[4] * cy + v[8] * cz + v[12];
  double y = v[1] * cx + v[5] * cy + v[9] * cz + v[13];
  double z = v[2] * cx + v[6] * cy + v[10] * cz + v[14];
  double d = sqrt(x * x + y * y + z * z);
  double R = r * s;
  *dmin = fmax(d - R, near_);
  *dmax = fmax(d + R, near_);
}

void vgo_instance_meshlet_range(const uint32_t *ranges, const float *errors, uint32_t levels, const float L[4],
                                const double v[16], double proj_scale, double near_, double s, double threshold,
                                double blend, uint32_t *start, uint32_t *end) {
  double dmin, dmax;
  lod_distance_bounds(L, v, near_, s, &dmin, &dmax);
  double high = threshold * fmax(1, blend);
  double k = s * proj_scale;
  int lo = -1, hi = -1;
  for (uint32_t l = 0; l < levels; l++) {
    double min_own = errors[l * 2], max_parent = errors[l * 2 + 1];
    int own_possible = (min_own * k) / dmax <= high;
    int parent_possible = max_parent >= VGO_ERROR_INFINITY * 0.5 || (max_parent * k) / dmin > threshold;
    if (own_possible && parent_possible) {
      if (lo < 0) lo = (int)l;
      hi = (int)l;
    }
  }
  if (lo < 0) {
    *start = 0;
    *end = 0;
    return;
  }
  *start = ranges[lo * 2];
  *end = ranges[hi * 2] + ranges[hi * 2 + 1];
}

int vgo_instance_guaranteed_range(const uint32_t *ranges, const float *errors, const float *guard, uint32_t levels,
                                  const float L[4], const double v[16], double proj_scale, double near_, double s,
                                  double threshold, double blend, uint32_t *start, uint32_t *end) {
  double dmin, dmax;
  lod_distance_bounds(L, v, near_, s, &dmin, &dmax);
  double high = threshold * fmax(1, blend);
  double margin = VGO_FAST_PATH_MARGIN;
  double k = s * proj_scale;
  int lo = -1, hi = -1;
  uint64_t possible = 0, guaranteed = 0;
  for (uint32_t l = 0; l < levels; l++) {
    double min_own = errors[l * 2], max_parent = errors[l * 2 + 1];
    int own_possible = (min_own * k) / dmax <= high;
    int parent_possible = max_parent >= VGO_ERROR_INFINITY * 0.5 || (max_parent * k) / dmin > threshold;
    if (!own_possible || !parent_possible) continue;
    if (lo < 0) lo = (int)l;
    hi = (int)l;
    uint32_t size = ranges[l * 2 + 1];
    possible += size;
    double max_own = guard[l * 2], min_parent = guard[l * 2 + 1];
    int own_sure = (max_own * k) / dmin <= threshold * (1 - margin);
    int parent_sure = min_parent >= VGO_ERROR_INFINITY * 0.5 || (min_parent * k) / dmax > high * (1 + margin);
    if (own_sure && parent_sure) guaranteed += size;
  }
  if (lo < 0) return 0;
  uint32_t s0 = ranges[lo * 2], e0 = ranges[hi * 2] + ranges[hi * 2 + 1];
  if (possible != (uint64_t)(e0 - s0) || guaranteed != possible) return 0;
  if (possible > VGO_FAST_PATH_MAX_MESHLETS) return 0;
  *start = s0;
  *end = e0;
  return 1;
}

/* The DAG-cut invariant over the full pass's output: verifyCutCoverage and verifyCutOverlap (cut.ts:83-122) applied
   to each drawn instance at each blend step. `entries` are one cut's (instance, pool-global meshlet, packed) rows;
   mesh k's meshlets are [base[k], base[k] + dags[k].meshlet_count). At step s an instance's selection is its
   meshlets with lo <= s < hi (packed bits 8-15 and 16-23). Returns the number of (instance, step) pairs with a hole
   or an overlap; *checked receives the number of instances with entries. */
uint64_t vgo_cut_invariant(const vgo_dag *dags, const uint32_t *base, uint32_t mesh_count, const uint32_t *inst_slot,
                           uint32_t instance_count, const uint32_t *entries, uint64_t n, const uint32_t *steps,
                           uint32_t nsteps, int threads, uint64_t *checked) {
  uint64_t *first = (uint64_t *)calloc((size_t)instance_count + 1, sizeof(uint64_t));
  uint64_t *order = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
  uint64_t bad = 0, seen = 0, skipped = 0;
  for (uint64_t e = 0; e < n; e++) {
    uint32_t inst = entries[e * 3];
    if (inst < instance_count) first[inst + 1]++;
    else skipped++;
  }
  for (uint32_t i = 0; i < instance_count; i++) first[i + 1] += first[i];
  uint64_t *fill = (uint64_t *)malloc(((size_t)instance_count + 1) * sizeof(uint64_t));
  memcpy(fill, first, ((size_t)instance_count + 1) * sizeof(uint64_t));
  for (uint64_t e = 0; e < n; e++) {
    uint32_t inst = entries[e * 3];
    if (inst < instance_count) order[fill[inst]++] = e;
  }
  free(fill);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel reduction(+ : bad, seen)
  {
    uint8_t *sel = NULL;
    int8_t *memo = NULL;
    uint32_t cap = 0;
#pragma omp for schedule(dynamic, 64)
    for (int64_t ii = 0; ii < (int64_t)instance_count; ii++) {
      uint32_t inst = (uint32_t)ii;
      if (first[inst] == first[inst + 1]) continue;
      uint32_t slot = inst_slot[inst];
      if (slot >= mesh_count) { bad += nsteps; continue; }
      const vgo_dag *d = &dags[slot];
      if (d->meshlet_count > cap) {
        cap = d->meshlet_count;
        sel = (uint8_t *)realloc(sel, cap);
        memo = (int8_t *)realloc(memo, cap);
      }
      seen++;
      for (uint32_t s = 0; s < nsteps; s++) {
        memset(sel, 0, d->meshlet_count);
        int broken = 0;
        for (uint64_t k = first[inst]; k < first[inst + 1]; k++) {
          const uint32_t *row = entries + order[k] * 3;
          uint32_t m = row[1] - base[slot], lo = (row[2] >> 8) & 255, hi = (row[2] >> 16) & 255;
          if (row[1] < base[slot] || m >= d->meshlet_count) { broken = 1; continue; }
          if (lo <= steps[s] && steps[s] < hi) {
            if (sel[m]) broken = 1; /* the same meshlet drawn twice */
            sel[m] = 1;
          }
        }
        walk_ctx c = {d->group, d->start, d->list, sel, memo};
        memset(memo, -1, d->meshlet_count);
        for (uint32_t i = 0; i < d->meshlet_count && !broken; i++)
          if (sel[i] && below(&c, i)) broken = 1;
        memset(memo, -1, d->meshlet_count);
        for (uint32_t i = 0; i < d->meshlet_count && !broken; i++)
          if (d->info[(size_t)i * 4 + 2] == 0 && !covered(&c, i)) broken = 1;
        bad += (uint64_t)broken;
      }
    }
    free(sel);
    free(memo);
  }
  free(first);
  free(order);
  if (checked) *checked = seen;
  return bad + skipped;
}
