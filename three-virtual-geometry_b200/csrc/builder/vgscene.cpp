// Seeded generators for the synthetic inputs: geodesic icospheres with Perlin displacement, box lattices,
// height-field terrain, occluder depth images, and the Morton instance order.
//
// The reference generates its demo content in TypeScript (examples/demo/noise.ts:3-97 for the seeded RNG and
// noise, examples/demo/ruinsScene.ts for the scene) and orders instances along a Morton curve at mesh creation
// (GeometryPool.ts:1263-1311, VirtualMesh.ts:171-175). These are independent C++ implementations of the
// published methods: mulberry32 (a public-domain 32-bit PRNG) and Ken Perlin's improved noise (SIGGRAPH 2002).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "vgbuild.h"

namespace vgb_internal {
extern thread_local std::string g_error;
}
#define g_scene_error vgb_internal::g_error

namespace {

struct PerlinTable {
  uint8_t p[512];
  explicit PerlinTable(uint32_t seed) {
    uint32_t s = seed;
    uint8_t perm[256];
    for (int i = 0; i < 256; i++) perm[i] = uint8_t(i);
    for (int i = 255; i > 0; i--) {
      int j = int(std::floor(vgb_mulberry32_float(&s) * (i + 1)));
      std::swap(perm[i], perm[j]);
    }
    for (int i = 0; i < 512; i++) p[i] = perm[i & 255];
  }
};

inline double fade(double t) { return t * t * t * (t * (t * 6 - 15) + 10); }
inline double lerp(double t, double a, double b) { return a + t * (b - a); }
inline double grad(int h, double x, double y, double z) {
  h &= 15;
  double u = h < 8 ? x : y;
  double v = h < 4 ? y : (h == 12 || h == 14) ? x : z;
  return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}

double perlin(const PerlinTable &T, double x, double y, double z) {
  const uint8_t *p = T.p;
  int X = int(std::floor(x)) & 255, Y = int(std::floor(y)) & 255, Z = int(std::floor(z)) & 255;
  x -= std::floor(x);
  y -= std::floor(y);
  z -= std::floor(z);
  double u = fade(x), v = fade(y), w = fade(z);
  int A = p[X] + Y, AA = p[A] + Z, AB = p[A + 1] + Z, B = p[X + 1] + Y, BA = p[B] + Z, BB = p[B + 1] + Z;
  return lerp(w,
              lerp(v, lerp(u, grad(p[AA], x, y, z), grad(p[BA], x - 1, y, z)),
                   lerp(u, grad(p[AB], x, y - 1, z), grad(p[BB], x - 1, y - 1, z))),
              lerp(v, lerp(u, grad(p[AA + 1], x, y, z - 1), grad(p[BA + 1], x - 1, y, z - 1)),
                   lerp(u, grad(p[AB + 1], x, y - 1, z - 1), grad(p[BB + 1], x - 1, y - 1, z - 1))));
}

double fbm(const PerlinTable &T, double x, double y, double z, int octaves) {
  double sum = 0, amp = 1, norm = 0;
  for (int i = 0; i < octaves; i++) {
    sum += amp * perlin(T, x, y, z);
    norm += amp;
    amp *= 0.5;
    x *= 2;
    y *= 2;
    z *= 2;
  }
  return sum / norm;
}

vgb_raw *make_raw(const std::vector<float> &pos, const std::vector<uint32_t> &idx) {
  vgb_raw *r = (vgb_raw *)std::calloc(1, sizeof(vgb_raw));
  r->vertex_count = uint32_t(pos.size() / 3);
  r->positions = (float *)std::malloc(std::max<size_t>(4, pos.size() * 4));
  std::memcpy(r->positions, pos.data(), pos.size() * 4);
  r->index_count = uint32_t(idx.size());
  r->indices = (uint32_t *)std::malloc(std::max<size_t>(4, idx.size() * 4));
  std::memcpy(r->indices, idx.data(), idx.size() * 4);
  return r;
}
}  // namespace

extern "C" {

uint32_t vgb_mulberry32_next(uint32_t *state) {
  uint32_t a = (*state += 0x6d2b79f5u);
  uint32_t t = a;
  t = (t ^ (t >> 15)) * (t | 1u);
  t ^= t + (t ^ (t >> 7)) * (t | 61u);
  return t ^ (t >> 14);
}

double vgb_mulberry32_float(uint32_t *state) { return double(vgb_mulberry32_next(state)) / 4294967296.0; }

float vgb_perlin3(uint32_t seed, float x, float y, float z) {
  PerlinTable T(seed);
  return float(perlin(T, x, y, z));
}

void vgb_raw_free(vgb_raw *r) {
  if (!r) return;
  std::free(r->positions);
  std::free(r->indices);
  std::free(r);
}

int vgb_gen_icosphere(uint32_t n, float radius, float amplitude, float frequency, uint32_t seed, vgb_raw **out) {
  if (!out || n == 0 || n > 4096) {
    g_scene_error = "vgb_gen_icosphere: n must be in [1, 4096]";
    return -1;
  }
  const double t = (1.0 + std::sqrt(5.0)) / 2.0;
  const double cv[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                            {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
  const int faces[20][3] = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                            {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
                            {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
  std::vector<double> dirs;  // unit directions
  auto push = [&](double x, double y, double z) {
    double l = std::sqrt(x * x + y * y + z * z);
    dirs.push_back(x / l);
    dirs.push_back(y / l);
    dirs.push_back(z / l);
    return uint32_t(dirs.size() / 3 - 1);
  };
  for (int i = 0; i < 12; i++) push(cv[i][0], cv[i][1], cv[i][2]);
  // canonical edge points: edge (a < b), k = 1..n-1 measured from a
  std::map<std::pair<int, int>, uint32_t> edge_base;
  for (int f = 0; f < 20; f++)
    for (int e = 0; e < 3; e++) {
      int a = faces[f][e], b = faces[f][(e + 1) % 3];
      auto key = std::make_pair(std::min(a, b), std::max(a, b));
      if (edge_base.count(key)) continue;
      edge_base[key] = uint32_t(dirs.size() / 3);
      const double *A = cv[key.first], *B = cv[key.second];
      for (uint32_t k = 1; k < n; k++) {
        double s = double(k) / n;
        push(A[0] + (B[0] - A[0]) * s, A[1] + (B[1] - A[1]) * s, A[2] + (B[2] - A[2]) * s);
      }
    }
  auto edge_vertex = [&](int a, int b, uint32_t k) -> uint32_t {  // k steps from a toward b
    if (k == 0) return uint32_t(a);
    if (k == n) return uint32_t(b);
    if (a < b) return edge_base[{a, b}] + (k - 1);
    return edge_base[{b, a}] + (n - k - 1);
  };
  std::vector<uint32_t> idx;
  idx.reserve(size_t(20) * n * n * 3);
  std::vector<uint32_t> grid;
  for (int f = 0; f < 20; f++) {
    int a = faces[f][0], b = faces[f][1], c = faces[f][2];
    const double *A = cv[a], *B = cv[b], *C = cv[c];
    // grid (i along AB, j along AC), i + j <= n
    grid.assign(size_t(n + 1) * (n + 1), 0);
    for (uint32_t i = 0; i <= n; i++)
      for (uint32_t j = 0; i + j <= n; j++) {
        uint32_t v;
        if (j == 0) v = edge_vertex(a, b, i);
        else if (i == 0) v = edge_vertex(a, c, j);
        else if (i + j == n) v = edge_vertex(b, c, j);
        else {
          double s = double(i) / n, r = double(j) / n;
          v = push(A[0] + (B[0] - A[0]) * s + (C[0] - A[0]) * r, A[1] + (B[1] - A[1]) * s + (C[1] - A[1]) * r,
                   A[2] + (B[2] - A[2]) * s + (C[2] - A[2]) * r);
        }
        grid[i * (n + 1) + j] = v;
      }
    for (uint32_t i = 0; i < n; i++)
      for (uint32_t j = 0; i + j < n; j++) {
        uint32_t v0 = grid[i * (n + 1) + j], v1 = grid[(i + 1) * (n + 1) + j], v2 = grid[i * (n + 1) + j + 1];
        idx.insert(idx.end(), {v0, v1, v2});
        if (i + j + 1 < n) {
          uint32_t v3 = grid[(i + 1) * (n + 1) + j + 1];
          idx.insert(idx.end(), {v1, v3, v2});
        }
      }
  }
  PerlinTable T(seed);
  std::vector<float> pos(dirs.size());
  for (size_t v = 0; v < dirs.size() / 3; v++) {
    double x = dirs[v * 3], y = dirs[v * 3 + 1], z = dirs[v * 3 + 2];
    double h = amplitude == 0 ? 0 : fbm(T, x * frequency + 11.5, y * frequency + 3.25, z * frequency + 7.75, 4);
    double r = radius * (1.0 + amplitude * h);
    pos[v * 3] = float(x * r);
    pos[v * 3 + 1] = float(y * r);
    pos[v * 3 + 2] = float(z * r);
  }
  *out = make_raw(pos, idx);
  return 0;
}

int vgb_gen_box_lattice(uint32_t boxes, uint32_t k, float extent, uint32_t seed, vgb_raw **out) {
  if (!out || boxes == 0 || k == 0 || k > 2048) {
    g_scene_error = "vgb_gen_box_lattice: bad arguments";
    return -1;
  }
  uint32_t s = seed;
  PerlinTable T(seed ^ 0x9e3779b9u);
  std::vector<float> pos;
  std::vector<uint32_t> idx;
  for (uint32_t bi = 0; bi < boxes; bi++) {
    // ruins-like pieces: pillars (tall), wall slabs (long, thin), blocks
    double kind = vgb_mulberry32_float(&s);
    double sx, sy, sz;
    if (kind < 0.35) {
      sx = sz = extent * (0.08 + 0.1 * vgb_mulberry32_float(&s));
      sy = extent * (0.5 + 0.5 * vgb_mulberry32_float(&s));
    } else if (kind < 0.75) {
      sx = extent * (0.4 + 0.6 * vgb_mulberry32_float(&s));
      sy = extent * (0.2 + 0.4 * vgb_mulberry32_float(&s));
      sz = extent * (0.05 + 0.07 * vgb_mulberry32_float(&s));
      if (vgb_mulberry32_float(&s) < 0.5) std::swap(sx, sz);
    } else {
      sx = extent * (0.15 + 0.25 * vgb_mulberry32_float(&s));
      sy = extent * (0.1 + 0.2 * vgb_mulberry32_float(&s));
      sz = extent * (0.15 + 0.25 * vgb_mulberry32_float(&s));
    }
    double cx = (vgb_mulberry32_float(&s) * 2 - 1) * (extent - sx * 0.5);
    double cz = (vgb_mulberry32_float(&s) * 2 - 1) * (extent - sz * 0.5);
    double cy = sy * 0.5;
    // surface grid of a (k+1)^3 lattice: a point is on the surface when a coordinate is 0 or k
    std::vector<int64_t> id(size_t(k + 1) * (k + 1) * (k + 1), -1);
    auto at = [&](uint32_t i, uint32_t j, uint32_t l) -> uint32_t {
      int64_t &slot = id[(size_t(i) * (k + 1) + j) * (k + 1) + l];
      if (slot < 0) {
        double u = double(i) / k - 0.5, v = double(j) / k - 0.5, w = double(l) / k - 0.5;
        double px = cx + u * sx, py = cy + v * sy, pz = cz + w * sz;
        double dn = 0.015 * std::min({sx, sy, sz}) * perlin(T, px * 0.7, py * 0.7, pz * 0.7);
        double len = std::sqrt(u * u + v * v + w * w);
        if (len > 0) {
          px += dn * u / len;
          py += dn * v / len;
          pz += dn * w / len;
        }
        slot = int64_t(pos.size() / 3);
        pos.push_back(float(px));
        pos.push_back(float(py));
        pos.push_back(float(pz));
      }
      return uint32_t(slot);
    };
    // 6 faces; winding outward
    for (int axis = 0; axis < 3; axis++)
      for (int side = 0; side < 2; side++) {
        uint32_t fixed = side ? k : 0;
        for (uint32_t a = 0; a < k; a++)
          for (uint32_t b = 0; b < k; b++) {
            auto P = [&](uint32_t aa, uint32_t bb) {
              if (axis == 0) return at(fixed, aa, bb);
              if (axis == 1) return at(bb, fixed, aa);
              return at(aa, bb, fixed);
            };
            uint32_t p00 = P(a, b), p10 = P(a + 1, b), p01 = P(a, b + 1), p11 = P(a + 1, b + 1);
            if (side) {
              idx.insert(idx.end(), {p00, p10, p11, p00, p11, p01});
            } else {
              idx.insert(idx.end(), {p00, p11, p10, p00, p01, p11});
            }
          }
      }
  }
  *out = make_raw(pos, idx);
  return 0;
}

int vgb_gen_terrain(float size, uint32_t segments, float amplitude, float fx, float fz, vgb_raw **out) {
  if (!out || segments == 0 || segments > 8192) {
    g_scene_error = "vgb_gen_terrain: bad arguments";
    return -1;
  }
  const uint32_t g = segments + 1;
  std::vector<float> pos(size_t(g) * g * 3);
  for (uint32_t iy = 0; iy < g; iy++)
    for (uint32_t ix = 0; ix < g; ix++) {
      // plane in xy from (-s/2, s/2) to (s/2, -s/2), rotated -90 degrees about x: (x, y, 0) -> (x, 0, -y)
      double x = double(ix) * size / segments - size * 0.5;
      double y = size * 0.5 - double(iy) * size / segments;
      double z = -y;
      size_t o = (size_t(iy) * g + ix) * 3;
      pos[o] = float(x);
      pos[o + 2] = float(z);
      pos[o + 1] = float(amplitude * std::sin(double(float(x)) * fx) * std::cos(double(float(z)) * fz));
    }
  std::vector<uint32_t> idx;
  idx.reserve(size_t(segments) * segments * 6);
  for (uint32_t iy = 0; iy < segments; iy++)
    for (uint32_t ix = 0; ix < segments; ix++) {
      uint32_t a = ix + g * iy, b = ix + g * (iy + 1), c = ix + 1 + g * (iy + 1), d = ix + 1 + g * iy;
      idx.insert(idx.end(), {a, b, d, b, c, d});
    }
  *out = make_raw(pos, idx);
  return 0;
}

int vgb_gen_depth_image(uint32_t width, uint32_t height, uint32_t quads, float dmin, float dmax, float p10, float p14,
                        uint32_t seed, float *out) {
  if (!out || width == 0 || height == 0) {
    g_scene_error = "vgb_gen_depth_image: bad arguments";
    return -1;
  }
  std::fill(out, out + size_t(width) * height, 1.0f);
  uint32_t s = seed;
  for (uint32_t q = 0; q < quads; q++) {
    double w = (0.04 + 0.3 * vgb_mulberry32_float(&s)) * width;
    double h = (0.04 + 0.35 * vgb_mulberry32_float(&s)) * height;
    double x0 = vgb_mulberry32_float(&s) * (width - w);
    double y0 = vgb_mulberry32_float(&s) * (height - h);
    double depth = dmin + (dmax - dmin) * vgb_mulberry32_float(&s);
    float z = float(double(p14) / depth - double(p10));
    uint32_t xa = uint32_t(x0), xb = std::min(width, uint32_t(x0 + w)), ya = uint32_t(y0), yb = std::min(height, uint32_t(y0 + h));
    for (uint32_t y = ya; y < yb; y++)
      for (uint32_t x = xa; x < xb; x++) {
        float &d = out[size_t(y) * width + x];
        d = std::min(d, z);
      }
  }
  return 0;
}

int vgb_morton_order(const float *m, uint32_t n, const float sphere[4], uint32_t *out) {
  if (!out || (!m && n)) {
    g_scene_error = "vgb_morton_order: null argument";
    return -1;
  }
  std::vector<double> c(size_t(n) * 3);
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = 0; i < n; i++) {
    const float *e = m + size_t(i) * 16;
    double sx = sphere[0], sy = sphere[1], sz = sphere[2];
    double p[3] = {e[0] * sx + e[4] * sy + e[8] * sz + e[12], e[1] * sx + e[5] * sy + e[9] * sz + e[13],
                   e[2] * sx + e[6] * sy + e[10] * sz + e[14]};
    for (int a = 0; a < 3; a++) {
      c[i * 3 + a] = p[a];
      lo[a] = std::min(lo[a], p[a]);
      hi[a] = std::max(hi[a], p[a]);
    }
  }
  double extent = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-9});
  auto spread = [](uint32_t v) {
    v &= 0x3ff;
    uint32_t r = 0;
    for (int b = 0; b < 10; b++) r |= ((v >> b) & 1u) << (3 * b);
    return r;
  };
  std::vector<std::pair<uint32_t, uint32_t>> keys(n);
  for (uint32_t i = 0; i < n; i++) {
    uint32_t q[3];
    for (int a = 0; a < 3; a++) {
      double f = std::floor((c[i * 3 + a] - lo[a]) / extent * 1024.0);
      q[a] = uint32_t(std::min(1023.0, std::max(0.0, f)));
    }
    keys[i] = {spread(q[0]) | (spread(q[1]) << 1) | (spread(q[2]) << 2), i};
  }
  std::stable_sort(keys.begin(), keys.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
  for (uint32_t i = 0; i < n; i++) out[i] = keys[i].second;
  return 0;
}

// The .vgeo container checksum (serialize.ts:429-437): a 32-bit multiplicative hash over the little-endian u32 words
// from byte `start` (whole words only): h = 0x811c9dc5 ^ words; per word h = (h ^ w) * 0x01000193, h ^= h >> 15.
uint32_t vgb_vgeo_checksum(const uint8_t *bytes, uint64_t length, uint64_t start) {
  const uint64_t n = length > start ? (length - start) >> 2 : 0;
  uint32_t h = 0x811c9dc5u ^ (uint32_t)n;
  for (uint64_t i = 0; i < n; i++) {
    uint32_t w;
    std::memcpy(&w, bytes + start + i * 4, 4);
    h = (h ^ w) * 0x01000193u;
    h ^= h >> 15;
  }
  return h;
}

}  // extern "C"
