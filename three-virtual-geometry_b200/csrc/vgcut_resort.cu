// Instance re-sort (vgc_instances_resort): mortonOrder (GeometryPool.ts:1263-1284) of a mesh's instances at their
// current positions, on the device, so that a streaming scene whose instances have moved gets compact cells back.
// The reference sorts only when a mesh is added; this applies the same order to the current matrices:
//
//   centre = M (sphere.xyz, 1) in double (instanceSphere, :1171-1180); lo / hi over the mesh; extent = max(hi - lo,
//   1e-9); q = clamp(floor((c - lo) / extent * 1024), 0, 1023) per axis; code = spread(qx) | spread(qy) << 1 |
//   spread(qz) << 2 (30 bits); a stable sort by code (the reference's LSD radix order).
//
// Every double expression rounds step by step in the host's order (the library is compiled with -fmad=false), so
// the codes equal the host's. The sort is CUB's stable LSD radix sort over the 30 key bits; the permutation and the
// cells (k_cells_update, double, in the host's operation order) follow on the device, and the host mirror is
// permuted and its cells recomputed from the same matrices.
#include <cub/device/device_radix_sort.cuh>

#include "vgcut_host.h"
#include "vgcut_kernels.h"

namespace {

constexpr uint32_t kBlock = 256;

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Centres of instances [0, n) of the mesh (inst: its first instance's columns), and per block the min / max.
__global__ void __launch_bounds__(kBlock) k_morton_centres(const float4 *__restrict__ inst, uint32_t n, double sx,
                                                           double sy, double sz, double *__restrict__ centres,
                                                           double *__restrict__ partial) {
  __shared__ double red[6][kBlock / 32];
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (i < n) {
    const float4 c0 = inst[(size_t)i * 4], c1 = inst[(size_t)i * 4 + 1], c2 = inst[(size_t)i * 4 + 2],
                 c3 = inst[(size_t)i * 4 + 3];
    const double p[3] = {double(c0.x) * sx + double(c1.x) * sy + double(c2.x) * sz + double(c3.x),
                         double(c0.y) * sx + double(c1.y) * sy + double(c2.y) * sz + double(c3.y),
                         double(c0.z) * sx + double(c1.z) * sy + double(c2.z) * sz + double(c3.z)};
    for (int a = 0; a < 3; a++) {
      centres[(size_t)i * 3 + a] = p[a];
      lo[a] = p[a];
      hi[a] = p[a];
    }
  }
  for (int a = 0; a < 3; a++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = fmin(lo[a], __shfl_down_sync(0xffffffffu, lo[a], o));
      hi[a] = fmax(hi[a], __shfl_down_sync(0xffffffffu, hi[a], o));
    }
  const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int a = 0; a < 3; a++) red[a][w] = lo[a], red[3 + a][w] = hi[a];
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = red[threadIdx.x][0];
    for (uint32_t k = 1; k < kBlock / 32; k++) v = threadIdx.x < 3 ? fmin(v, red[threadIdx.x][k]) : fmax(v, red[threadIdx.x][k]);
    partial[(size_t)blockIdx.x * 6 + threadIdx.x] = v;
  }
}

// One block: the mesh's lo / hi from the blocks' partials, then extent (bounds[0..2] lo, bounds[3] extent).
__global__ void __launch_bounds__(kBlock) k_morton_bounds(const double *__restrict__ partial, uint32_t blocks,
                                                          double *__restrict__ bounds) {
  __shared__ double red[6][kBlock];
  double v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  for (uint32_t b = threadIdx.x; b < blocks; b += kBlock)
    for (int a = 0; a < 6; a++) v[a] = a < 3 ? fmin(v[a], partial[(size_t)b * 6 + a]) : fmax(v[a], partial[(size_t)b * 6 + a]);
  for (int a = 0; a < 6; a++) red[a][threadIdx.x] = v[a];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t k = 1; k < kBlock; k++)
      for (int a = 0; a < 6; a++) v[a] = a < 3 ? fmin(v[a], red[a][k]) : fmax(v[a], red[a][k]);
    double extent = v[3] - v[0];
    extent = fmax(extent, v[4] - v[1]);
    extent = fmax(extent, v[5] - v[2]);
    extent = fmax(extent, 1e-9);
    bounds[0] = v[0], bounds[1] = v[1], bounds[2] = v[2], bounds[3] = extent;
  }
}

__global__ void __launch_bounds__(kBlock) k_morton_codes(const double *__restrict__ centres, uint32_t n,
                                                         const double *__restrict__ bounds, uint32_t *__restrict__ keys,
                                                         uint32_t *__restrict__ index) {
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  const double extent = bounds[3];
  uint32_t q[3];
  for (int a = 0; a < 3; a++) {
    const double f = floor((centres[(size_t)i * 3 + a] - bounds[a]) / extent * 1024.0);
    q[a] = (uint32_t)fmin(1023.0, fmax(0.0, f));
  }
  keys[i] = spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2);
  index[i] = i;
}

// New instance g takes the columns of old instance order[g].
__global__ void __launch_bounds__(kBlock) k_permute(const float4 *__restrict__ inst, uint32_t n,
                                                    const uint32_t *__restrict__ order, float4 *__restrict__ out) {
  const uint32_t t = blockIdx.x * kBlock + threadIdx.x;
  if (t >= n * 4) return;
  const uint32_t g = t >> 2, c = t & 3u;
  out[t] = inst[(size_t)order[g] * 4 + c];
}

}  // namespace

extern "C" int vgc_instances_resort(vgc_context *ctx, uint32_t slot, uint32_t *new_to_old) {
  if (!ctx) return fail(VGC_INVALID_ARG, "null argument");
  if (slot >= ctx->slots_used || !ctx->mesh_host[slot].used) return fail(VGC_NOT_FOUND, "no mesh in slot");
  MeshHost &m = ctx->mesh_host[slot];
  const uint32_t n = m.instance_count;
  std::vector<uint32_t> order(n);
  if (!ctx->dirty && n > 1) {
    // resident scene: codes, sort, permutation and cells on the device
    cudaSetDevice(ctx->device);
    CUDA_TRY(cudaDeviceSynchronize());  // after every launch that may still read the instances
    const uint32_t blocks = (n + kBlock - 1) / kBlock;
    size_t sort_bytes = 0;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                             (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)n, 0, 30,
                                             ctx->stream));
    const size_t centres_b = (size_t)n * 24, partial_b = (size_t)blocks * 48, keys_b = (size_t)n * 4,
                 inst_b = (size_t)n * 64;
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t total = up(centres_b) + up(partial_b) + 256 + 4 * up(keys_b) + up(inst_b) + up(sort_bytes);
    int rc = dev_alloc(ctx, ctx->d_resort, total);  // kept for later re-sorts (grows only)
    if (rc) return rc;
    char *p = (char *)ctx->d_resort.ptr;
    double *centres = (double *)p;
    p += up(centres_b);
    double *partial = (double *)p;
    p += up(partial_b);
    double *bounds = (double *)p;
    p += 256;
    uint32_t *keys_in = (uint32_t *)p, *keys_out = (uint32_t *)(p + up(keys_b)), *idx_in = (uint32_t *)(p + 2 * up(keys_b)),
             *idx_out = (uint32_t *)(p + 3 * up(keys_b));
    p += 4 * up(keys_b);
    float4 *permuted = (float4 *)p;
    p += up(inst_b);
    void *sort_tmp = p;
    float4 *inst = (float4 *)ctx->d_inst.ptr + (size_t)m.instance_base * 4;
    cudaError_t e = cudaSuccess;
    k_morton_centres<<<blocks, kBlock, 0, ctx->stream>>>(inst, n, m.sphere[0], m.sphere[1], m.sphere[2], centres, partial);
    if ((e = cudaGetLastError()) == cudaSuccess) {
      k_morton_bounds<<<1, kBlock, 0, ctx->stream>>>(partial, blocks, bounds);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      k_morton_codes<<<blocks, kBlock, 0, ctx->stream>>>(centres, n, bounds, keys_in, idx_in);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cub::DeviceRadixSort::SortPairs(sort_tmp, sort_bytes, keys_in, keys_out, idx_in, idx_out, (int)n, 0, 30,
                                          ctx->stream);
    if (e == cudaSuccess) {
      k_permute<<<(n * 4 + kBlock - 1) / kBlock, kBlock, 0, ctx->stream>>>(inst, n, idx_out, permuted);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(inst, permuted, inst_b, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e == cudaSuccess) {
      const double sphere[4] = {m.sphere[0], m.sphere[1], m.sphere[2], m.sphere[3]};
      e = launch_cells_update((const float4 *)ctx->d_inst.ptr, sphere, m.instance_base, n, m.cell_base, slot, 0,
                              m.cell_count, (CellRec *)ctx->d_cells.ptr, ctx->stream);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(order.data(), idx_out, keys_b, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(VGC_DEVICE_ERROR, std::string("vgc_instances_resort: ") + cudaGetErrorString(e));
    }
  } else if (n > 1) {
    // the scene is not resident (a full upload is pending): the host order, which that upload carries
    std::vector<float> mats((size_t)n * 16);
    for (uint32_t g = 0; g < n; g++)
      for (int c = 0; c < 4; c++) {
        const float4 v = ctx->inst[(size_t)(m.instance_base + g) * 4 + c];
        mats[(size_t)g * 16 + c * 4] = v.x, mats[(size_t)g * 16 + c * 4 + 1] = v.y;
        mats[(size_t)g * 16 + c * 4 + 2] = v.z, mats[(size_t)g * 16 + c * 4 + 3] = v.w;
      }
    morton_order(mats.data(), n, m.sphere, order);
  } else {
    for (uint32_t g = 0; g < n; g++) order[g] = g;
  }
  // the host mirror: the same permutation, cells recomputed from the same matrices
  std::vector<float4> old(ctx->inst.begin() + (size_t)m.instance_base * 4,
                          ctx->inst.begin() + (size_t)(m.instance_base + n) * 4);
  for (uint32_t g = 0; g < n; g++)
    for (int c = 0; c < 4; c++) ctx->inst[(size_t)(m.instance_base + g) * 4 + c] = old[(size_t)order[g] * 4 + c];
  for (uint32_t c = 0; c < m.cell_count; c++) compute_cell(ctx, slot, c);
  if (new_to_old)
    for (uint32_t g = 0; g < n; g++) new_to_old[g] = order[g];
  return VGC_OK;
}
