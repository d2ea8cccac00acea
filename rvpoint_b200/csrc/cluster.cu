// Euclidean cluster extraction (segmentation/euclidean_clustering.cpp:113-189).
//
// The reference grows clusters by BFS from the lowest unvisited index over
// the graph "squared distance <= tolerance^2"; its clusters are that graph's
// connected components, listed by their lowest index, each sorted, kept when
// min_size <= size <= max_size. Here the components come from a lock-free
// union-find over the same graph: one warp per point walks the grid cells
// of the tight window of radius tolerance (lanes over candidates) and joins
// the point with every later neighbour, always hooking the larger root under
// the smaller, so that each root ends as its component's lowest index. A
// sort by (root, index) then lays every component out in the reference's
// order, and a scan keeps the components within the size limits.
#include "grid_device.cuh"
#include "internal.cuh"

namespace rvp {
using namespace gd;

namespace {

constexpr int kUfLimit = 1 << 22;  // bound on every union-find loop

// root of v: parents only ever point to lower indices, so the walk ends;
// path halving on the way (benign races: every value written is an ancestor)
__device__ __forceinline__ u32 uf_find(u32 *par, u32 v, int *err) {
  u32 cur = __ldcg(&par[v]);
  if (cur == v) return v;
  u32 prev = v;
  for (int it = 0; it < kUfLimit; ++it) {
    const u32 next = __ldcg(&par[cur]);
    if (next >= cur) return cur;
    par[prev] = next;
    prev = cur;
    cur = next;
  }
  atomicExch(err, 1);
  return cur;
}

__device__ __forceinline__ void uf_unite(u32 *par, u32 a, u32 b, int *err) {
  u32 ra = uf_find(par, a, err), rb = uf_find(par, b, err);
  for (int it = 0; it < kUfLimit && ra != rb; ++it) {
    if (ra < rb) {
      const u32 t = ra;
      ra = rb;
      rb = t;
    }
    // hook the larger root under the smaller
    const u32 old = atomicCAS(&par[ra], ra, rb);
    if (old == ra) return;
    ra = uf_find(par, old, err);
    rb = uf_find(par, rb, err);
  }
  if (ra != rb) atomicExch(err, 1);
}

__global__ void k_uf_init(u32 *par, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    par[i] = (u32)i;
}

// one warp per point (grid order); lanes over the window's candidates
__global__ __launch_bounds__(256) void k_uf_edges(GridView g, float tol, u32 *par, int *err) {
  const u64 n = *g.n_points;
  const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
  const GridFrame F = g.frames[0];
  const float tol_sq = fmul(tol, tol);
  for (size_t pos = warp; pos < n; pos += nwarps) {
    const float4 q = g.pts[pos];
    const u32 i = __float_as_uint(q.w) & 0x7FFFFFFFu;
    const Window w = tight_window(F, q.x, q.y, q.z, (double)tol, 0);
    for_each_candidate(g, F, 0, w, false, [&](float4 p, bool valid) {
      const u32 j = __float_as_uint(p.w) & 0x7FFFFFFFu;
      // euclidean_clustering.cpp:92-96: ((dx*dx + dy*dy) + dz*dz) <= tol^2
      if (valid && j > i && dist2(p.x, p.y, p.z, q.x, q.y, q.z) <= tol_sq)
        uf_unite(par, i, j, err);
    });
  }
}

// key (root << 32 | index), value index
__global__ void k_uf_keys(u32 *par, size_t n, u64 *keys, u32 *vals, int *err) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const u32 r = uf_find(par, (u32)i, err);
    keys[i] = ((u64)r << 32) | (u64)i;
    vals[i] = (u32)i;
  }
}

__global__ void k_seg_heads(const u64 *keys, size_t n, u32 *heads) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    heads[k] = (k == 0 || (keys[k] >> 32) != (keys[k - 1] >> 32)) ? 1u : 0u;
}

// per segment: start and end (sorted positions); seg_pos = exclusive scan of
// heads, so the segment of a head at k is seg_pos[k]
__global__ void k_seg_bounds(const u32 *heads, const u64 *seg_pos, size_t n, u64 *seg_start) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    if (heads[k]) seg_start[seg_pos[k]] = k;
  if (blockIdx.x == 0 && threadIdx.x == 0) seg_start[seg_pos[n]] = n;
}

__global__ void k_seg_keep(const u64 *seg_start, const u64 *n_seg_dev, int min_size,
                           int max_size, u32 *keep, u32 *kept_size) {
  const u64 n_seg = *n_seg_dev;
  for (u64 s = blockIdx.x * (u64)blockDim.x + threadIdx.x; s < n_seg;
       s += (u64)gridDim.x * blockDim.x) {
    const u64 sz = seg_start[s + 1] - seg_start[s];
    const bool k = sz >= (u64)min_size && sz <= (u64)max_size;
    keep[s] = k ? 1u : 0u;
    kept_size[s] = k ? (u32)sz : 0u;
  }
}

// kept segments: their cluster offsets
__global__ void k_seg_offsets(const u64 *n_seg_dev, const u32 *keep, const u64 *cid,
                              const u64 *cpos, int64_t *offsets, u64 *n_clusters) {
  const u64 n_seg = *n_seg_dev;
  for (u64 s = blockIdx.x * (u64)blockDim.x + threadIdx.x; s < n_seg;
       s += (u64)gridDim.x * blockDim.x)
    if (keep[s]) offsets[cid[s]] = (int64_t)cpos[s];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    offsets[cid[n_seg]] = (int64_t)cpos[n_seg];
    *n_clusters = cid[n_seg];
  }
}

// their points, in sorted order (one thread per point)
__global__ void k_seg_points(const u32 *heads, const u64 *seg_pos, const u64 *seg_start,
                             const u32 *keep, const u64 *cpos, const u32 *sorted_idx, size_t n,
                             int32_t *indices) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const u64 s = seg_pos[k] + heads[k] - 1;
    if (keep[s]) indices[cpos[s] + (k - seg_start[s])] = (int32_t)sorted_idx[k];
  }
}

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

size_t euclidean_temp_bytes(size_t n) {
  return al(n * 4) + al(n * 8) + al(n * 4) + sort_temp_bytes(n) + al(n * 4) +
         4 * al((n + 1) * 8) + 3 * al((n + 1) * 4) + scan_temp_bytes(n + 1) + 256;
}

void euclidean_clusters_run(rvp_context *ctx, Grid &grid, const float *x, const float *y,
                            const float *z, size_t n, const int64_t *offs_dev, float tolerance,
                            int min_size, int max_size, int64_t *offsets, int32_t *indices,
                            u64 *n_clusters_dev, void *temp) {
  cudaStream_t st = ctx->stream;
  char *p = static_cast<char *>(temp);
  u32 *par = reinterpret_cast<u32 *>(p); p += al(n * 4);
  u64 *keys = reinterpret_cast<u64 *>(p); p += al(n * 8);
  u32 *vals = reinterpret_cast<u32 *>(p); p += al(n * 4);
  SortTemp stt;
  sort_temp_carve(stt, p, n); p += sort_temp_bytes(n);
  u32 *heads = reinterpret_cast<u32 *>(p); p += al(n * 4);
  u64 *seg_pos = reinterpret_cast<u64 *>(p); p += al((n + 1) * 8);
  u64 *seg_start = reinterpret_cast<u64 *>(p); p += al((n + 1) * 8);
  u64 *cid = reinterpret_cast<u64 *>(p); p += al((n + 1) * 8);
  u64 *cpos = reinterpret_cast<u64 *>(p); p += al((n + 1) * 8);
  u32 *keep = reinterpret_cast<u32 *>(p); p += al((n + 1) * 4);
  u32 *ksize = reinterpret_cast<u32 *>(p); p += al((n + 1) * 4);
  p += al((n + 1) * 4);
  void *scan_tmp = p; p += scan_temp_bytes(n + 1);
  int *err = reinterpret_cast<int *>(p);
  RVP_CUDA_TRY(cudaMemsetAsync(err, 0, 4, st));
  // the grid: cells of one tolerance, so that the window spans 3 cells a side
  grid_build(ctx, grid, x, y, z, offs_dev, 1, n, tolerance, KEY_DENSE, 0, 0, nullptr);
  const GridView gv = grid.view(KEY_DENSE, 0, 0);
  const unsigned gb = grid_for(n, 256, ctx->num_sms * 16);
  k_uf_init<<<gb, 256, 0, st>>>(par, n);
  RVP_LAUNCH_CHECK(ctx);
  k_uf_edges<<<grid_for(n * 32, 256, ctx->num_sms * 32), 256, 0, st>>>(gv, tolerance, par, err);
  RVP_LAUNCH_CHECK(ctx);
  k_uf_keys<<<gb, 256, 0, st>>>(par, n, keys, vals, err);
  RVP_LAUNCH_CHECK(ctx);
  radix_sort_pairs(ctx, keys, vals, n, nullptr, stt);
  k_seg_heads<<<gb, 256, 0, st>>>(keys, n, heads);
  RVP_LAUNCH_CHECK(ctx);
  exclusive_scan_u32_to_u64(ctx, heads, seg_pos, n, nullptr, scan_tmp);
  k_seg_bounds<<<gb, 256, 0, st>>>(heads, seg_pos, n, seg_start);
  RVP_LAUNCH_CHECK(ctx);
  const u64 *n_seg = seg_pos + n;
  k_seg_keep<<<gb, 256, 0, st>>>(seg_start, n_seg, min_size, max_size, keep, ksize);
  RVP_LAUNCH_CHECK(ctx);
  exclusive_scan_u32_to_u64(ctx, keep, cid, n, n_seg, scan_tmp);
  exclusive_scan_u32_to_u64(ctx, ksize, cpos, n, n_seg, scan_tmp);
  k_seg_offsets<<<gb, 256, 0, st>>>(n_seg, keep, cid, cpos, offsets, n_clusters_dev);
  RVP_LAUNCH_CHECK(ctx);
  k_seg_points<<<gb, 256, 0, st>>>(heads, seg_pos, seg_start, keep, cpos, vals, n, indices);
  RVP_LAUNCH_CHECK(ctx);
  int h_err = 0;
  RVP_CUDA_TRY(cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, st));
  RVP_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_err) throw Error{RVP_ERR_CUDA, "union-find did not settle within its iteration bound"};
}

}  // namespace rvp
