// Host-side cluster-DAG builder writing the VirtualMeshData layout of three-virtual-geometry
// (src/core/preprocess/buildVirtualMesh.ts:75-138, pack at :484-601).
//
// The reference builds with meshoptimizer (clusterizer + simplifier with LockBorder). This builder is
// its own design, chosen so that the DAG invariants the cut relies on hold by construction:
//   * leaf meshlets: breadth-first clusters of <= 128 triangles / <= 128 vertices;
//   * groups: recursive median bisection of meshlet centres into groups of <= group_size;
//   * simplification: quadric edge collapse to an endpoint (Garland & Heckbert 1997) with every
//     vertex on the group's topological border locked, so neighbouring groups still share edges;
//   * monotone bounds: group error = max child error + max(shape error, 1e-7), group LOD sphere
//     encloses every child LOD sphere, and the same (sphere, error) pair is written as the children's
//     parent and the outputs' own bound, so a cut evaluated with one arithmetic is hole- and overlap-free.
#include "vgbuild.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace vgb_internal {
thread_local std::string g_error;
}
using vgb_internal::g_error;

namespace {

constexpr double kErrorInfinity = 1e30;
constexpr uint32_t kMaxTris = 128;
constexpr uint32_t kMaxVerts = 128;

int fail(const std::string &msg) {
  g_error = msg;
  return -1;
}

struct Sphere {
  double x = 0, y = 0, z = 0, r = 0;
};

struct Meshlet {
  std::vector<uint32_t> tris;  // 3 global vertex ids per triangle
  std::vector<uint32_t> verts; // global ids in local order
  std::vector<uint8_t> local;  // 3 local ids per triangle
  uint32_t level = 0;
  Sphere lod, parent, cull;
  double error = 0, parent_error = kErrorInfinity;
  int replaced_by = -1;  // index of the output list that replaced this meshlet
  double cx = 0, cy = 0, cz = 0;
};

Sphere bounding_sphere(const std::vector<uint32_t> &tris, const float *pos) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (uint32_t v : tris)
    for (int k = 0; k < 3; k++) {
      double p = pos[v * 3 + k];
      lo[k] = std::min(lo[k], p);
      hi[k] = std::max(hi[k], p);
    }
  Sphere s;
  s.x = (lo[0] + hi[0]) * 0.5;
  s.y = (lo[1] + hi[1]) * 0.5;
  s.z = (lo[2] + hi[2]) * 0.5;
  double r2 = 0;
  for (uint32_t v : tris) {
    double dx = pos[v * 3] - s.x, dy = pos[v * 3 + 1] - s.y, dz = pos[v * 3 + 2] - s.z;
    r2 = std::max(r2, dx * dx + dy * dy + dz * dz);
  }
  s.r = std::sqrt(r2);
  return s;
}

// Sphere around a set of spheres: centre of their joint box, radius reaching every member, padded so the
// float32 copy still encloses each float32 member.
Sphere enclosing(const std::vector<Sphere> &in) {
  if (in.size() == 1) return in[0];
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (const Sphere &s : in) {
    double c[3] = {s.x, s.y, s.z};
    for (int k = 0; k < 3; k++) {
      lo[k] = std::min(lo[k], c[k] - s.r);
      hi[k] = std::max(hi[k], c[k] + s.r);
    }
  }
  Sphere o;
  o.x = (lo[0] + hi[0]) * 0.5;
  o.y = (lo[1] + hi[1]) * 0.5;
  o.z = (lo[2] + hi[2]) * 0.5;
  double r = 0;
  for (const Sphere &s : in) r = std::max(r, std::sqrt((s.x - o.x) * (s.x - o.x) + (s.y - o.y) * (s.y - o.y) + (s.z - o.z) * (s.z - o.z)) + s.r);
  o.r = r * 1.0001 + 1e-7;
  return o;
}

inline uint64_t edge_key(uint32_t a, uint32_t b) { return a < b ? (uint64_t(a) << 32) | b : (uint64_t(b) << 32) | a; }

// ---------------------------------------------------------------- clusterizer
// Splits a triangle set into meshlets by recursive median bisection of triangle centroids along the longest
// axis, in chunks that are whole multiples of 128 triangles, so nearly every meshlet is full; a chunk whose
// unique vertices exceed 128 is halved again. Local vertex ids are assigned in first-use order.
void emit_meshlet(const std::vector<uint32_t> &tris_global, const std::vector<uint32_t> &ids, size_t lo, size_t hi,
                  const float *pos, uint32_t level, std::vector<Meshlet> &out) {
  Meshlet m;
  m.level = level;
  m.tris.reserve((hi - lo) * 3);
  m.local.reserve((hi - lo) * 3);
  for (size_t i = lo; i < hi; i++)
    for (int k = 0; k < 3; k++) {
      uint32_t g = tris_global[size_t(ids[i]) * 3 + k];
      size_t l = 0;
      while (l < m.verts.size() && m.verts[l] != g) l++;
      if (l == m.verts.size()) m.verts.push_back(g);
      m.tris.push_back(g);
      m.local.push_back(uint8_t(l));
    }
  m.cull = bounding_sphere(m.tris, pos);
  m.cx = m.cull.x;
  m.cy = m.cull.y;
  m.cz = m.cull.z;
  out.push_back(std::move(m));
}

size_t unique_vertices(const std::vector<uint32_t> &tris_global, const std::vector<uint32_t> &ids, size_t lo, size_t hi,
                       std::vector<uint32_t> &scratch) {
  scratch.clear();
  for (size_t i = lo; i < hi; i++)
    for (int k = 0; k < 3; k++) scratch.push_back(tris_global[size_t(ids[i]) * 3 + k]);
  std::sort(scratch.begin(), scratch.end());
  return size_t(std::unique(scratch.begin(), scratch.end()) - scratch.begin());
}

void split_triangles(const std::vector<uint32_t> &tris_global, std::vector<uint32_t> &ids, size_t lo, size_t hi,
                     const std::vector<float> &centroid, const float *pos, uint32_t level, std::vector<Meshlet> &out,
                     std::vector<uint32_t> &scratch) {
  size_t n = hi - lo;
  if (n <= kMaxTris && unique_vertices(tris_global, ids, lo, hi, scratch) <= kMaxVerts) {
    emit_meshlet(tris_global, ids, lo, hi, pos, level, out);
    return;
  }
  float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
  for (size_t i = lo; i < hi; i++)
    for (int k = 0; k < 3; k++) {
      float c = centroid[size_t(ids[i]) * 3 + k];
      mn[k] = std::min(mn[k], c);
      mx[k] = std::max(mx[k], c);
    }
  int axis = 0;
  for (int k = 1; k < 3; k++)
    if (mx[k] - mn[k] > mx[axis] - mn[axis]) axis = k;
  size_t chunks = (n + kMaxTris - 1) / kMaxTris;
  size_t left = chunks > 1 ? ((chunks + 1) / 2) * kMaxTris : n / 2;
  if (left >= n) left = n / 2;
  std::nth_element(ids.begin() + lo, ids.begin() + lo + left, ids.begin() + hi, [&](uint32_t a, uint32_t b) {
    float ka = centroid[size_t(a) * 3 + axis], kb = centroid[size_t(b) * 3 + axis];
    return ka < kb || (ka == kb && a < b);
  });
  split_triangles(tris_global, ids, lo, lo + left, centroid, pos, level, out, scratch);
  split_triangles(tris_global, ids, lo + left, hi, centroid, pos, level, out, scratch);
}

void clusterize(const std::vector<uint32_t> &tris_global, const float *pos, uint32_t level, std::vector<Meshlet> &out) {
  const size_t T = tris_global.size() / 3;
  if (T == 0) return;
  std::vector<float> centroid(T * 3);
  for (size_t t = 0; t < T; t++)
    for (int k = 0; k < 3; k++)
      centroid[t * 3 + k] = (pos[tris_global[t * 3] * 3 + k] + pos[tris_global[t * 3 + 1] * 3 + k] + pos[tris_global[t * 3 + 2] * 3 + k]) / 3.0f;
  std::vector<uint32_t> ids(T), scratch;
  for (size_t t = 0; t < T; t++) ids[t] = uint32_t(t);
  split_triangles(tris_global, ids, 0, T, centroid, pos, level, out, scratch);
}

// ---------------------------------------------------------------- partition
void bisect(std::vector<uint32_t> &ids, size_t lo, size_t hi, const std::vector<Meshlet> &ms, uint32_t group_size,
            std::vector<std::vector<uint32_t>> &groups) {
  size_t n = hi - lo;
  if (n <= group_size) {
    groups.emplace_back(ids.begin() + lo, ids.begin() + hi);
    return;
  }
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (size_t i = lo; i < hi; i++) {
    const Meshlet &m = ms[ids[i]];
    double c[3] = {m.cx, m.cy, m.cz};
    for (int k = 0; k < 3; k++) {
      mn[k] = std::min(mn[k], c[k]);
      mx[k] = std::max(mx[k], c[k]);
    }
  }
  int axis = 0;
  for (int k = 1; k < 3; k++)
    if (mx[k] - mn[k] > mx[axis] - mn[axis]) axis = k;
  // left part: a whole number of groups, about half
  size_t groups_total = (n + group_size - 1) / group_size;
  size_t left = ((groups_total + 1) / 2) * group_size;
  if (left >= n) left = n / 2;
  auto key = [&](uint32_t i) { return axis == 0 ? ms[i].cx : axis == 1 ? ms[i].cy : ms[i].cz; };
  std::nth_element(ids.begin() + lo, ids.begin() + lo + left, ids.begin() + hi, [&](uint32_t a, uint32_t b) {
    double ka = key(a), kb = key(b);
    return ka < kb || (ka == kb && a < b);
  });
  bisect(ids, lo, lo + left, ms, group_size, groups);
  bisect(ids, lo + left, hi, ms, group_size, groups);
}

// ---------------------------------------------------------------- simplifier
struct Quadric {
  double a[10] = {0};  // xx xy xz xd yy yz yd zz zd dd
  double w = 0;        // accumulated plane weight (triangle area)
  void add_plane(double nx, double ny, double nz, double d, double w) {
    a[0] += w * nx * nx; a[1] += w * nx * ny; a[2] += w * nx * nz; a[3] += w * nx * d;
    a[4] += w * ny * ny; a[5] += w * ny * nz; a[6] += w * ny * d;
    a[7] += w * nz * nz; a[8] += w * nz * d; a[9] += w * d * d;
    this->w += w;
  }
  void add(const Quadric &o) {
    for (int i = 0; i < 10; i++) a[i] += o.a[i];
    w += o.w;
  }
  double eval(double x, double y, double z) const {
    double r = a[0] * x * x + 2 * a[1] * x * y + 2 * a[2] * x * z + 2 * a[3] * x + a[4] * y * y + 2 * a[5] * y * z +
               2 * a[6] * y + a[7] * z * z + 2 * a[8] * z + a[9];
    r = r > 0 ? r : 0;
    return w > 0 ? r / w : r;  // area-weighted mean squared distance to the merged planes
  }
};

struct HeapItem {
  double cost;
  uint32_t src, dst, vs, vd;
  bool operator<(const HeapItem &o) const { return cost > o.cost; }
};

// Simplifies a triangle set (global ids) toward `target` triangles with `locked` vertices fixed.
// Returns the remaining triangles and the geometric error (sqrt of the largest collapse cost).
double simplify(const std::vector<uint32_t> &tris_global, const float *pos, const std::vector<uint8_t> &locked_local,
                const std::vector<uint32_t> &gids, uint32_t target, std::vector<uint32_t> &result) {
  const uint32_t V = uint32_t(gids.size());
  const uint32_t T = uint32_t(tris_global.size() / 3);
  auto lid = [&](uint32_t g) { return uint32_t(std::lower_bound(gids.begin(), gids.end(), g) - gids.begin()); };
  std::vector<uint32_t> tv(size_t(T) * 3);
  for (size_t i = 0; i < tv.size(); i++) tv[i] = lid(tris_global[i]);
  std::vector<double> P(size_t(V) * 3);
  for (uint32_t v = 0; v < V; v++)
    for (int k = 0; k < 3; k++) P[v * 3 + k] = pos[gids[v] * 3 + k];
  std::vector<Quadric> Q(V);
  std::vector<double> tn(size_t(T) * 3);
  for (uint32_t t = 0; t < T; t++) {
    const double *a = &P[tv[t * 3] * 3], *b = &P[tv[t * 3 + 1] * 3], *c = &P[tv[t * 3 + 2] * 3];
    double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (l > 0) {
      n[0] /= l; n[1] /= l; n[2] /= l;
      double d = -(n[0] * a[0] + n[1] * a[1] + n[2] * a[2]);
      for (int k = 0; k < 3; k++) Q[tv[t * 3 + k]].add_plane(n[0], n[1], n[2], d, 0.5 * l);
    }
    for (int k = 0; k < 3; k++) tn[t * 3 + k] = n[k];
  }
  std::vector<std::vector<uint32_t>> vt(V);
  for (uint32_t t = 0; t < T; t++)
    for (int k = 0; k < 3; k++) vt[tv[t * 3 + k]].push_back(t);
  std::vector<uint8_t> tri_alive(T, 1), v_alive(V, 1);
  std::vector<uint32_t> version(V, 0);
  uint32_t alive = T;
  std::vector<HeapItem> heap;
  auto consider = [&](uint32_t a, uint32_t b) {
    double best = 1e300;
    uint32_t s = 0, d = 0;
    if (!locked_local[a]) {
      Quadric q = Q[a];
      q.add(Q[b]);
      double c = q.eval(P[b * 3], P[b * 3 + 1], P[b * 3 + 2]);
      if (c < best) { best = c; s = a; d = b; }
    }
    if (!locked_local[b]) {
      Quadric q = Q[a];
      q.add(Q[b]);
      double c = q.eval(P[a * 3], P[a * 3 + 1], P[a * 3 + 2]);
      if (c < best) { best = c; s = b; d = a; }
    }
    if (best < 1e300) {
      heap.push_back({best, s, d, version[s], version[d]});
      std::push_heap(heap.begin(), heap.end());
    }
  };
  {
    std::vector<uint64_t> ek;
    ek.reserve(size_t(T) * 3);
    for (uint32_t t = 0; t < T; t++)
      for (int k = 0; k < 3; k++) ek.push_back(edge_key(tv[t * 3 + k], tv[t * 3 + (k + 1) % 3]));
    std::sort(ek.begin(), ek.end());
    ek.erase(std::unique(ek.begin(), ek.end()), ek.end());
    for (uint64_t e : ek) consider(uint32_t(e >> 32), uint32_t(e & 0xffffffffu));
  }
  double max_cost = 0;
  std::vector<uint32_t> nbr_s, nbr_d;
  auto neighbours = [&](uint32_t v, std::vector<uint32_t> &out) {
    out.clear();
    for (uint32_t t : vt[v])
      if (tri_alive[t])
        for (int k = 0; k < 3; k++)
          if (tv[t * 3 + k] != v) out.push_back(tv[t * 3 + k]);
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
  };
  while (alive > target && !heap.empty()) {
    std::pop_heap(heap.begin(), heap.end());
    HeapItem h = heap.back();
    heap.pop_back();
    uint32_t s = h.src, d = h.dst;
    if (!v_alive[s] || !v_alive[d] || version[s] != h.vs || version[d] != h.vd) continue;
    // link condition: the common neighbours of s and d are exactly the far corners of their shared triangles
    neighbours(s, nbr_s);
    neighbours(d, nbr_d);
    if (!std::binary_search(nbr_s.begin(), nbr_s.end(), d)) continue;
    uint32_t shared_tris = 0;
    for (uint32_t t : vt[s])
      if (tri_alive[t] && (tv[t * 3] == d || tv[t * 3 + 1] == d || tv[t * 3 + 2] == d)) shared_tris++;
    uint32_t common = 0;
    for (uint32_t x : nbr_s)
      if (std::binary_search(nbr_d.begin(), nbr_d.end(), x)) common++;
    if (common != shared_tris) continue;
    // no flipped or degenerate triangles
    bool ok = true;
    for (uint32_t t : vt[s]) {
      if (!tri_alive[t]) continue;
      uint32_t a = tv[t * 3], b = tv[t * 3 + 1], c = tv[t * 3 + 2];
      if (a == d || b == d || c == d) continue;
      if (a == s) a = d;
      if (b == s) b = d;
      if (c == s) c = d;
      const double *pa = &P[a * 3], *pb = &P[b * 3], *pc = &P[c * 3];
      double e1[3] = {pb[0] - pa[0], pb[1] - pa[1], pb[2] - pa[2]}, e2[3] = {pc[0] - pa[0], pc[1] - pa[1], pc[2] - pa[2]};
      double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
      double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
      if (!(l > 0)) { ok = false; break; }
      double dot = (n[0] * tn[t * 3] + n[1] * tn[t * 3 + 1] + n[2] * tn[t * 3 + 2]) / l;
      if (dot < 0.2) { ok = false; break; }
    }
    if (!ok) continue;
    // apply s -> d
    for (uint32_t t : vt[s]) {
      if (!tri_alive[t]) continue;
      uint32_t *v = &tv[t * 3];
      if (v[0] == d || v[1] == d || v[2] == d) {
        tri_alive[t] = 0;
        alive--;
        continue;
      }
      for (int k = 0; k < 3; k++)
        if (v[k] == s) v[k] = d;
      vt[d].push_back(t);
    }
    v_alive[s] = 0;
    Q[d].add(Q[s]);
    max_cost = std::max(max_cost, h.cost);
    // Only the quadric of d changed: edges at d get new costs, every other queued edge keeps its cost (its
    // flip and link checks run again when it is popped).
    version[d]++;
    neighbours(d, nbr_d);
    for (uint32_t x : nbr_d) consider(d, x);
  }
  result.clear();
  for (uint32_t t = 0; t < T; t++)
    if (tri_alive[t])
      for (int k = 0; k < 3; k++) result.push_back(gids[tv[t * 3 + k]]);
  return std::sqrt(max_cost);
}

double extent_shrink(const std::vector<uint32_t> &before, const std::vector<uint32_t> &after, const float *pos) {
  auto box = [&](const std::vector<uint32_t> &ix, double *lo, double *hi) {
    for (int k = 0; k < 3; k++) { lo[k] = 1e300; hi[k] = -1e300; }
    for (uint32_t v : ix)
      for (int k = 0; k < 3; k++) {
        lo[k] = std::min(lo[k], double(pos[v * 3 + k]));
        hi[k] = std::max(hi[k], double(pos[v * 3 + k]));
      }
  };
  double alo[3], ahi[3], blo[3], bhi[3];
  box(before, alo, ahi);
  if (after.empty()) return std::max({ahi[0] - alo[0], ahi[1] - alo[1], ahi[2] - alo[2]}) * 0.5;
  box(after, blo, bhi);
  double s = 0;
  for (int k = 0; k < 3; k++) s = std::max({s, blo[k] - alo[k], ahi[k] - bhi[k]});
  return s;
}

// Vertices on the topological border of a triangle set: endpoints of edges used by one triangle only.
// `keep_open` false unlocks edges that are also open edges of the whole surface (`surface_open` sorted).
void border_vertices(const std::vector<uint32_t> &tris, const std::vector<uint32_t> &gids, bool keep_open,
                     const std::vector<uint64_t> &surface_open, std::vector<uint8_t> &locked) {
  std::vector<uint64_t> ek;
  ek.reserve(tris.size());
  for (size_t t = 0; t < tris.size(); t += 3)
    for (int k = 0; k < 3; k++) ek.push_back(edge_key(tris[t + k], tris[t + (k + 1) % 3]));
  std::sort(ek.begin(), ek.end());
  locked.assign(gids.size(), 0);
  auto lid = [&](uint32_t g) { return size_t(std::lower_bound(gids.begin(), gids.end(), g) - gids.begin()); };
  for (size_t i = 0; i < ek.size();) {
    size_t j = i;
    while (j < ek.size() && ek[j] == ek[i]) j++;
    if (j - i == 1) {
      bool open = !keep_open && std::binary_search(surface_open.begin(), surface_open.end(), ek[i]);
      if (!open) {
        locked[lid(uint32_t(ek[i] >> 32))] = 1;
        locked[lid(uint32_t(ek[i] & 0xffffffffu))] = 1;
      }
    }
    i = j;
  }
}

std::vector<uint64_t> open_edges(const std::vector<const Meshlet *> &surface) {
  std::vector<uint64_t> ek;
  for (const Meshlet *m : surface)
    for (size_t t = 0; t < m->tris.size(); t += 3)
      for (int k = 0; k < 3; k++) ek.push_back(edge_key(m->tris[t + k], m->tris[t + (k + 1) % 3]));
  std::sort(ek.begin(), ek.end());
  std::vector<uint64_t> open;
  for (size_t i = 0; i < ek.size();) {
    size_t j = i;
    while (j < ek.size() && ek[j] == ek[i]) j++;
    if (j - i == 1) open.push_back(ek[i]);
    i = j;
  }
  return open;
}

struct GroupResult {
  bool reduced = false;
  Sphere lod;
  double error = 0;
  std::vector<Meshlet> outputs;
};

template <class F>
void parallel_for(int n, int threads, F &&f) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
  for (int i = 0; i < n; i++) f(i);
#else
  (void)threads;
  for (int i = 0; i < n; i++) f(i);
#endif
}

}  // namespace

extern "C" {

const char *vgb_last_error(void) { return g_error.c_str(); }

void vgb_default_options(vgb_options *o) {
  o->group_size = 12;
  o->max_lod_levels = 24;
  o->simplify_ratio = 0.5f;
  o->max_group_keep_ratio = 0.9f;
  o->min_level_reduction = 0.03f;
  o->min_root_triangles = 4;
  o->threads = 0;
}

int vgb_build(const float *positions, uint32_t vertex_count, const uint32_t *indices, uint32_t index_count,
              const vgb_options *opts_in, vgb_mesh **out) {
  if (!out) return fail("vgb_build: out is null");
  *out = nullptr;
  if (!positions || !indices || index_count == 0 || index_count % 3 != 0) return fail("vgb_build: empty or ragged index list");
  for (uint32_t i = 0; i < index_count; i++)
    if (indices[i] >= vertex_count) return fail("vgb_build: index out of range");
  vgb_options opts;
  vgb_default_options(&opts);
  if (opts_in) opts = *opts_in;
  if (opts.group_size < 2) opts.group_size = 2;
  int threads = int(opts.threads);
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#else
  threads = 1;
#endif
  auto t0 = std::chrono::steady_clock::now();
  const float *pos = positions;

  std::vector<Meshlet> all;  // every meshlet ever made; index = creation order
  std::vector<std::vector<uint32_t>> replacement_lists;
  {
    std::vector<uint32_t> tris(indices, indices + index_count);
    std::vector<Meshlet> leafs;
    clusterize(tris, pos, 0, leafs);
    for (auto &m : leafs) {
      m.lod = m.cull;
      m.error = 0;
      all.push_back(std::move(m));
    }
  }
  std::vector<uint32_t> current(all.size());
  for (uint32_t i = 0; i < current.size(); i++) current[i] = i;
  std::vector<uint32_t> stuck_roots;  // meshlets of groups that could not be reduced
  auto count_tris = [&](const std::vector<uint32_t> &ids) {
    size_t s = 0;
    for (uint32_t i : ids) s += all[i].tris.size() / 3;
    return s;
  };
  size_t last_tris = count_tris(current);
  uint32_t lod_levels = 1;
  for (uint32_t level = 1; level <= opts.max_lod_levels + 16; level++) {
    if (current.empty()) break;
    const bool single = current.size() == 1;
    if (single && all[current[0]].tris.size() / 3 <= opts.min_root_triangles) break;
    if (!single && level > opts.max_lod_levels) break;
    std::vector<std::vector<uint32_t>> groups;
    {
      std::vector<uint32_t> ids(current.size());
      for (size_t i = 0; i < ids.size(); i++) ids[i] = uint32_t(i);
      std::vector<Meshlet> view;  // centres only
      view.reserve(current.size());
      for (uint32_t c : current) {
        Meshlet m;
        m.cx = all[c].cx; m.cy = all[c].cy; m.cz = all[c].cz;
        view.push_back(std::move(m));
      }
      std::vector<std::vector<uint32_t>> local_groups;
      bisect(ids, 0, ids.size(), view, opts.group_size, local_groups);
      for (auto &g : local_groups) {
        for (auto &i : g) i = current[i];
        std::sort(g.begin(), g.end());
        groups.push_back(std::move(g));
      }
    }
    const bool tail = groups.size() == 1;
    std::vector<uint64_t> surface_open;
    if (tail) {
      std::vector<const Meshlet *> surf;
      for (uint32_t i : current) surf.push_back(&all[i]);
      for (uint32_t i : stuck_roots) surf.push_back(&all[i]);
      surface_open = open_edges(surf);
    }
    std::vector<GroupResult> results(groups.size());
    parallel_for(int(groups.size()), threads, [&](int g) {
      const auto &grp = groups[g];
      std::vector<uint32_t> merged;
      for (uint32_t i : grp) merged.insert(merged.end(), all[i].tris.begin(), all[i].tris.end());
      std::vector<uint32_t> gids(merged);
      std::sort(gids.begin(), gids.end());
      gids.erase(std::unique(gids.begin(), gids.end()), gids.end());
      std::vector<uint8_t> locked;
      border_vertices(merged, gids, !tail, surface_open, locked);
      uint32_t tcount = uint32_t(merged.size() / 3);
      uint32_t target = std::max<uint32_t>(1, uint32_t(double(tcount) * opts.simplify_ratio));
      std::vector<uint32_t> simplified;
      double err = simplify(merged, pos, locked, gids, target, simplified);
      GroupResult &r = results[g];
      if (double(simplified.size()) > double(merged.size()) * opts.max_group_keep_ratio) return;
      double shape = std::max(err, extent_shrink(merged, simplified, pos));
      double child_error = 0;
      std::vector<Sphere> spheres;
      for (uint32_t i : grp) {
        child_error = std::max(child_error, all[i].error);
        spheres.push_back(all[i].lod);
      }
      r.reduced = true;
      r.lod = enclosing(spheres);
      r.error = child_error + std::max(shape, 1e-7);
      if (!simplified.empty()) clusterize(simplified, pos, level, r.outputs);
      for (auto &m : r.outputs) {
        m.lod = r.lod;
        m.error = r.error;
      }
    });
    std::vector<uint32_t> next;
    for (size_t g = 0; g < groups.size(); g++) {
      GroupResult &r = results[g];
      if (!r.reduced) {
        for (uint32_t i : groups[g]) stuck_roots.push_back(i);
        continue;
      }
      int list = -1;
      if (!r.outputs.empty()) {
        list = int(replacement_lists.size());
        replacement_lists.emplace_back();
      }
      for (uint32_t i : groups[g]) {
        all[i].parent = r.lod;
        all[i].parent_error = r.error;
        all[i].replaced_by = list;
      }
      for (auto &m : r.outputs) {
        uint32_t id = uint32_t(all.size());
        all.push_back(std::move(m));
        replacement_lists[list].push_back(id);
        next.push_back(id);
      }
    }
    if (next.empty()) break;
    lod_levels = level + 1;
    current = next;
    size_t tris = count_tris(current);
    if (!single && double(tris) > double(last_tris) * (1.0 - opts.min_level_reduction)) break;
    last_tris = tris;
  }

  // ------------------------------------------------------------ pack (sorted by level, stable)
  const uint32_t M = uint32_t(all.size());
  std::vector<uint32_t> order(M);
  for (uint32_t i = 0; i < M; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return all[a].level < all[b].level; });
  std::vector<uint32_t> index_of(M);
  for (uint32_t i = 0; i < M; i++) index_of[order[i]] = i;

  vgb_mesh *mesh = (vgb_mesh *)std::calloc(1, sizeof(vgb_mesh));
  mesh->vertex_count = vertex_count;
  mesh->positions = (float *)std::malloc(sizeof(float) * 3 * std::max<uint32_t>(1, vertex_count));
  std::memcpy(mesh->positions, positions, sizeof(float) * 3 * vertex_count);
  size_t idx_total = 0, vert_total = 0;
  for (auto &m : all) {
    idx_total += m.tris.size();
    vert_total += m.verts.size();
  }
  mesh->meshlet_count = M;
  mesh->index_count = uint32_t(idx_total);
  mesh->indices = (uint32_t *)std::malloc(sizeof(uint32_t) * std::max<size_t>(1, idx_total));
  mesh->meshlet_bounds = (float *)std::calloc(size_t(M) * 16, sizeof(float));
  mesh->meshlet_info = (uint32_t *)std::calloc(size_t(M) * 4, sizeof(uint32_t));
  mesh->meshlet_vertex_count = uint32_t(vert_total);
  mesh->meshlet_vertices = (uint32_t *)std::malloc(sizeof(uint32_t) * std::max<size_t>(1, vert_total));
  mesh->meshlet_triangle_count = uint32_t(idx_total / 3);
  mesh->meshlet_triangles = (uint32_t *)std::malloc(sizeof(uint32_t) * std::max<size_t>(1, idx_total / 3));
  uint32_t first_index = 0, vertex_offset = 0;
  for (uint32_t i = 0; i < M; i++) {
    const Meshlet &m = all[order[i]];
    std::memcpy(mesh->indices + first_index, m.tris.data(), m.tris.size() * 4);
    std::memcpy(mesh->meshlet_vertices + vertex_offset, m.verts.data(), m.verts.size() * 4);
    for (size_t t = 0; t < m.local.size() / 3; t++)
      mesh->meshlet_triangles[first_index / 3 + t] = uint32_t(m.local[t * 3]) | (uint32_t(m.local[t * 3 + 1]) << 8) | (uint32_t(m.local[t * 3 + 2]) << 16);
    float *b = mesh->meshlet_bounds + size_t(i) * 16;
    b[0] = float(m.lod.x); b[1] = float(m.lod.y); b[2] = float(m.lod.z); b[3] = float(m.lod.r);
    b[4] = float(m.parent.x); b[5] = float(m.parent.y); b[6] = float(m.parent.z); b[7] = float(m.parent.r);
    b[8] = float(m.error);
    b[9] = float(m.parent_error);
    b[12] = float(m.cull.x); b[13] = float(m.cull.y); b[14] = float(m.cull.z); b[15] = float(m.cull.r);
    uint32_t *info = mesh->meshlet_info + size_t(i) * 4;
    uint32_t tc = uint32_t(m.tris.size() / 3);
    info[0] = tc;
    info[1] = first_index;
    info[2] = m.level;
    info[3] = vertex_offset;
    first_index += uint32_t(m.tris.size());
    vertex_offset += uint32_t(m.verts.size());
    if (m.level == 0) {
      mesh->leaf_triangles += tc;
      mesh->leaf_meshlets++;
    }
    if (m.parent_error >= kErrorInfinity) {
      mesh->root_triangles += tc;
      mesh->root_meshlets++;
    }
  }
  // replacement lists, numbered in order of first use by a sorted meshlet
  mesh->replacement_group = (int32_t *)std::malloc(sizeof(int32_t) * std::max<uint32_t>(1, M));
  std::vector<int> list_id(replacement_lists.size(), -1);
  std::vector<uint32_t> starts{0};
  std::vector<uint32_t> rindices;
  for (uint32_t i = 0; i < M; i++) {
    int l = all[order[i]].replaced_by;
    if (l < 0) {
      mesh->replacement_group[i] = -1;
      continue;
    }
    if (list_id[l] < 0) {
      list_id[l] = int(starts.size() - 1);
      for (uint32_t r : replacement_lists[l]) rindices.push_back(index_of[r]);
      starts.push_back(uint32_t(rindices.size()));
    }
    mesh->replacement_group[i] = list_id[l];
  }
  mesh->group_count = uint32_t(starts.size() - 1);
  mesh->replacement_start = (uint32_t *)std::malloc(sizeof(uint32_t) * starts.size());
  std::memcpy(mesh->replacement_start, starts.data(), starts.size() * 4);
  mesh->replacement_index_count = uint32_t(rindices.size());
  mesh->replacement_indices = (uint32_t *)std::malloc(sizeof(uint32_t) * std::max<size_t>(1, rindices.size()));
  if (!rindices.empty()) std::memcpy(mesh->replacement_indices, rindices.data(), rindices.size() * 4);

  const uint32_t L = M ? all[order[M - 1]].level + 1 : 0;
  mesh->level_count = L;
  mesh->lod_levels = lod_levels;
  mesh->level_ranges = (uint32_t *)std::calloc(size_t(L) * 2 + 2, sizeof(uint32_t));
  mesh->level_errors = (float *)std::calloc(size_t(L) * 2 + 2, sizeof(float));
  mesh->level_guard_errors = (float *)std::calloc(size_t(L) * 2 + 2, sizeof(float));
  for (uint32_t l = 0; l < L; l++) {
    mesh->level_errors[l * 2] = INFINITY;
    mesh->level_errors[l * 2 + 1] = 0;
    mesh->level_guard_errors[l * 2] = 0;
    mesh->level_guard_errors[l * 2 + 1] = INFINITY;
  }
  for (uint32_t i = 0; i < M; i++) {
    uint32_t l = mesh->meshlet_info[i * 4 + 2];
    const float *b = mesh->meshlet_bounds + size_t(i) * 16;
    if (mesh->level_ranges[l * 2 + 1] == 0) mesh->level_ranges[l * 2] = i;
    mesh->level_ranges[l * 2 + 1]++;
    mesh->level_errors[l * 2] = std::min(mesh->level_errors[l * 2], b[8]);
    mesh->level_errors[l * 2 + 1] = std::max(mesh->level_errors[l * 2 + 1], b[9]);
    mesh->level_guard_errors[l * 2] = std::max(mesh->level_guard_errors[l * 2], b[8]);
    mesh->level_guard_errors[l * 2 + 1] = std::min(mesh->level_guard_errors[l * 2 + 1], b[9]);
  }
  std::vector<Sphere> lods, culls, leaves;
  for (auto &m : all) {
    lods.push_back(m.lod);
    if (m.parent_error < kErrorInfinity) lods.push_back(m.parent);
    culls.push_back(m.cull);
    if (m.level == 0) leaves.push_back(m.cull);
  }
  // The bounds spheres are stored in float32: pad so each float member still lies inside.
  auto store = [](float *dst, Sphere s) {
    dst[0] = float(s.x); dst[1] = float(s.y); dst[2] = float(s.z);
    dst[3] = float(s.r * 1.0001 + 1e-6);
  };
  store(mesh->lod_bounds_sphere, enclosing(lods));
  store(mesh->cull_bounds_sphere, enclosing(culls));
  store(mesh->bounding_sphere, enclosing(leaves));
  mesh->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *out = mesh;
  return 0;
}

void vgb_mesh_free(vgb_mesh *m) {
  if (!m) return;
  std::free(m->positions); std::free(m->indices); std::free(m->meshlet_bounds); std::free(m->meshlet_info);
  std::free(m->meshlet_vertices); std::free(m->meshlet_triangles); std::free(m->level_ranges);
  std::free(m->level_errors); std::free(m->level_guard_errors); std::free(m->replacement_group);
  std::free(m->replacement_start); std::free(m->replacement_indices);
  std::free(m);
}

}  // extern "C"
