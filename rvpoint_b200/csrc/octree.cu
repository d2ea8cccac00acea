// Octree and PointerOctree (search/octree.{h,cpp}, search/pointer_octree.{h,cpp})
// and the calls that take them: sor_octree / sor_pointer_octree
// (filters/statistical_outlier_removal.cpp:220-244, 272-301) and
// normal_estimation_rvv with a tree (features/normal_estimation.cpp:155-187,
// 216-253).
//
// Both trees answer radiusSearch with every point at squared distance
// <= radius * radius: their box tests (octree.cpp:96-109,
// pointer_octree.cpp:118-129) round monotonically and never exclude a point
// inside the sphere, and max_nn is ignored. What a tree decides is the ORDER
// of the list: leaves depth-first with children 0..7, each leaf's points in
// index order. No pointer tree is built here. Instead:
//   build    the root box (bbox reduction, then the tree's epsilon rule);
//            one key per point: its child codes (x >= mid) | (y >= mid) << 1 |
//            (z >= mid) << 2 down to max_depth, with the reference's float
//            midpoints (min + max) * 0.5f; a radix sort of the keys; per
//            point the depth at which its node holds <= cap points (group
//            sizes by binary search in the sorted keys), which is the depth
//            of its leaf; the key cut to that depth; a second sort of
//            (leaf key, index) gives every point its rank in the tree.
//   search   the grid's radius lists, re-sorted by (query, rank).
//   SOR      sor_octree: mean over the sorted distances; sor_pointer_octree:
//            std::nth_element as libstdc++ 13 runs it (introselect), one
//            thread per query on its tree-ordered distances, then the sum
//            over positions 1..valid_k as the reference adds them.
//   normals  the reference's covariance over the tree-ordered lists.
#include <math.h>

#include <algorithm>
#include <new>

#include "internal.cuh"

struct rvp_octree {
  rvp_context *ctx = nullptr;
  int kind = RVP_OCTREE;
  int cap = 64, depth = 8;
  float eps = 1e-4f;
  // the tree itself: its copy of the cloud and every point's rank
  rvp::DevBuf x, y, z, offs, rank, order, root;
  size_t n = 0;
  bool has_cloud = false, built = false;
  float box[6] = {0, 0, 0, 0, 0, 0};  // root box (host copy)
};

namespace rvp {
namespace {

// Working buffers live in the context's one-shot scratch (grow-only, shared
// by the entry points of a context, which run one at a time), and the radius
// grid is the context's shared grid: a tree made per call, as the
// reference's callers do, allocates only its own ranks.
enum {
  W_KEYS = 0, W_VALS, W_SORT, W_CNT, W_LOFFS, W_PAIRS, W_PAIRS2, W_BIG, W_SCAN, W_WORK,
  W_STAGE  // W_STAGE + 0..5: staged inputs and outputs
};
inline DevBuf &wb(rvp_context *ctx, int slot) { return ctx->scratch[slot]; }
inline Grid &ctx_grid(rvp_context *ctx) {
  if (!ctx->grid) ctx->grid = new Grid();
  return *ctx->grid;
}

constexpr int kMaxDepth = 21;  // 3 bits per level in a 64-bit key

__device__ __forceinline__ u32 ord_enc(float f) {
  const u32 u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord_dec(u32 e) {
  return __uint_as_float((e & 0x80000000u) ? (e & 0x7FFFFFFFu) : ~e);
}

// enc[0..2]: min, enc[3..5]: max (order-preserving integer images)
__global__ void k_oct_bbox(const float *x, const float *y, const float *z, size_t n, u32 *enc) {
  u32 lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0u, 0u, 0u};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const u32 v[3] = {ord_enc(x[i]), ord_enc(y[i]), ord_enc(z[i])};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = min(lo[a], v[a]);
      hi[a] = max(hi[a], v[a]);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = __reduce_min_sync(0xFFFFFFFFu, lo[a]);
    hi[a] = __reduce_max_sync(0xFFFFFFFFu, hi[a]);
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      atomicMin(&enc[a], lo[a]);
      atomicMax(&enc[3 + a], hi[a]);
    }
  }
}

// octree.cpp:36-53: [min, max + eps]; pointer_octree.cpp:36-63: [min - eps, max + eps]
__global__ void k_oct_root(const u32 *enc, int kind, float eps, float *root) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int a = 0; a < 3; ++a) {
    const float lo = ord_dec(enc[a]), hi = ord_dec(enc[3 + a]);
    root[a] = kind == RVP_OCTREE ? lo : fsub(lo, eps);
    root[3 + a] = fadd(hi, eps);
  }
}

// buildParams (octree.cpp:59-94): child codes down to depth D
__global__ void k_oct_keys(const float *x, const float *y, const float *z, size_t n,
                           const float *root, int D, u64 *keys, u32 *vals) {
  const float r0 = root[0], r1 = root[1], r2 = root[2], r3 = root[3], r4 = root[4],
              r5 = root[5];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float px = x[i], py = y[i], pz = z[i];
    float lx = r0, ly = r1, lz = r2, hx = r3, hy = r4, hz = r5;
    u64 key = 0;
    for (int d = 0; d < D; ++d) {
      const float mx = fmul(fadd(lx, hx), 0.5f), my = fmul(fadd(ly, hy), 0.5f),
                  mz = fmul(fadd(lz, hz), 0.5f);
      const bool bx = px >= mx, by = py >= my, bz = pz >= mz;
      key = (key << 3) | (u64)((int)bx | ((int)by << 1) | ((int)bz << 2));
      if (bx) lx = mx; else hx = mx;
      if (by) ly = my; else hy = my;
      if (bz) lz = mz; else hz = mz;
    }
    keys[i] = key;
    vals[i] = (u32)i;
  }
}

// first position in [lo, hi) whose key >> shift is >= v (upper: > v)
__device__ __forceinline__ size_t key_bound(const u64 *k, size_t lo, size_t hi, int shift, u64 v,
                                            bool upper) {
  while (lo < hi) {
    const size_t m = lo + ((hi - lo) >> 1);
    const u64 p = k[m] >> shift;
    if (upper ? (p <= v) : (p < v)) lo = m + 1;
    else hi = m;
  }
  return lo;
}

// leaf of each point: the first depth at which its node holds <= cap
// points (or depth D); its key cut to that depth, stored by point index
__global__ void k_oct_leaf(const u64 *skeys, const u32 *svals, size_t n, int D, u64 cap,
                           u64 *leaf_by_idx) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n;
       p += (size_t)gridDim.x * blockDim.x) {
    const u64 key = skeys[p];
    size_t lo = 0, hi = n;
    int d = 0;
    for (; d < D; ++d) {
      if ((u64)(hi - lo) <= cap) break;
      const int shift = 3 * (D - d - 1);
      const u64 pre = key >> shift;
      const size_t a = key_bound(skeys, lo, hi, shift, pre, false);
      hi = key_bound(skeys, a, hi, shift, pre, true);
      lo = a;
    }
    const int cut = 3 * (D - d);
    leaf_by_idx[svals[p]] = cut >= 64 ? 0ull : ((key >> cut) << cut);
  }
}

__global__ void k_iota(u32 *v, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    v[i] = (u32)i;
}

__global__ void k_oct_rank(const u32 *sorted_idx, size_t n, u32 *rank) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n;
       p += (size_t)gridDim.x * blockDim.x)
    rank[sorted_idx[p]] = (u32)p;
}

// key (query << 32 | rank of the neighbour), value: position in the list
__global__ void k_oct_list_keys(const u64 *pairs, const u64 *offs, size_t nq, const u32 *rank,
                                u64 *keys, u32 *vals) {
  const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  for (size_t q = warp; q < nq; q += nw) {
    for (u64 e = offs[q] + lane; e < offs[q + 1]; e += 32) {
      keys[e] = ((u64)q << 32) | (u64)rank[(u32)pairs[e] & 0x7FFFFFFFu];
      vals[e] = (u32)e;
    }
  }
}

__global__ void k_gather_u64(const u64 *src, const u32 *perm, size_t n, u64 *dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    dst[i] = src[perm[i]];
}

__global__ void k_unpack_pairs(const u64 *pairs, size_t n, int32_t *idx, float *d2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const u64 k = pairs[i];
    idx[i] = (int32_t)((u32)k & 0x7FFFFFFFu);
    d2[i] = __uint_as_float((u32)(k >> 32));
  }
}

// ---- std::nth_element (libstdc++ 13: introselect) ------------------------
// While the range holds more than 3 elements: move the median of
// (first + 1, middle, last - 1) to first, Hoare-partition the rest around it
// and keep the side that holds nth; after 2 * floor(log2 n) such rounds,
// select with a binary max-heap of the nth + 1 first elements instead. The
// last range is insertion-sorted. Only operator< is used. The explicit index
// bounds in the partition scans are never what stops them (the median of
// three leaves sentinels on both sides); they keep every access provably in
// the list.
__device__ void heap_up(float *a, long hole, long top, float v) {
  long parent = (hole - 1) / 2;
  while (hole > top && a[parent] < v) {
    a[hole] = a[parent];
    hole = parent;
    parent = (hole - 1) / 2;
  }
  a[hole] = v;
}

// the hole goes down to a leaf along the larger children, then v goes up
__device__ void heap_adjust(float *a, long hole, long len, float v) {
  const long top = hole;
  long child = hole;
  while (child < (len - 1) / 2) {
    child = 2 * (child + 1);
    if (a[child] < a[child - 1]) child--;
    a[hole] = a[child];
    hole = child;
  }
  if ((len & 1) == 0 && child == (len - 2) / 2) {
    child = 2 * (child + 1);
    a[hole] = a[child - 1];
    hole = child - 1;
  }
  heap_up(a, hole, top, v);
}

__device__ void nth_element_f(float *a, long n, long nth) {
  if (n <= 0 || nth >= n) return;
  long first = 0, last = n;
  int depth = 2 * (63 - __clzll((unsigned long long)n));
  while (last - first > 3) {
    if (depth == 0) {
      float *h = a + first;
      const long middle = nth + 1 - first, len = last - first;
      if (middle >= 2) {
        for (long parent = (middle - 2) / 2;; --parent) {
          heap_adjust(h, parent, middle, h[parent]);
          if (parent == 0) break;
        }
      }
      for (long i = middle; i < len; ++i) {
        if (h[i] < h[0]) {
          const float v = h[i];
          h[i] = h[0];
          heap_adjust(h, 0, middle, v);
        }
      }
      const float t = a[first];
      a[first] = a[nth];
      a[nth] = t;
      return;
    }
    --depth;
    const long x = first + 1, y = first + (last - first) / 2, z = last - 1;
    long m;
    if (a[x] < a[y]) m = (a[y] < a[z]) ? y : ((a[x] < a[z]) ? z : x);
    else m = (a[x] < a[z]) ? x : ((a[y] < a[z]) ? z : y);
    {
      const float t = a[first];
      a[first] = a[m];
      a[m] = t;
    }
    const float piv = a[first];
    long lo = first + 1, hi = last;
    for (;;) {
      while (lo < last && a[lo] < piv) ++lo;
      --hi;
      while (hi > first && piv < a[hi]) --hi;
      if (!(lo < hi)) break;
      const float t = a[lo];
      a[lo] = a[hi];
      a[hi] = t;
      ++lo;
    }
    if (lo <= nth) first = lo;
    else last = lo;
  }
  for (long i = first + 1; i < last; ++i) {
    const float v = a[i];
    if (v < a[first]) {
      for (long j = i; j > first; --j) a[j] = a[j - 1];
      a[first] = v;
    } else {
      long j = i;
      while (j > first && v < a[j - 1]) {
        a[j] = a[j - 1];
        --j;
      }
      a[j] = v;
    }
  }
}

// SOR means (statistical_outlier_removal.cpp:228-243 / 287-300). Lists in
// (d2, index) order for sor_octree, in tree order for sor_pointer_octree
// (work: a float copy to run nth_element on).
__global__ void k_oct_sor_mean(const u64 *pairs, const u64 *offs, size_t n, int k, float radius,
                               bool nth_mode, float *work, float *mean) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
       q += (size_t)gridDim.x * blockDim.x) {
    const u64 b = offs[q], c = offs[q + 1] - b;
    if (c <= 1) {
      mean[q] = radius;
      continue;
    }
    const int valid_k = k < (int)(c - 1) ? k : (int)(c - 1);
    float sum = 0.0f;
    if (nth_mode) {
      float *a = work + b;
      for (u64 t = 0; t < c; ++t) a[t] = nbr_d2(pairs[b + t]);
      nth_element_f(a, (long)c, valid_k);
      for (int j = 1; j <= valid_k; ++j) sum = fadd(sum, __fsqrt_rn(a[j]));
    } else {
      for (int j = 1; j <= valid_k; ++j) sum = fadd(sum, __fsqrt_rn(nbr_d2(pairs[b + j])));
    }
    mean[q] = fdiv(sum, (float)valid_k);
  }
}

}  // namespace
}  // namespace rvp

using namespace rvp;

namespace {

template <class F>
rvp_status oct_guard(rvp_context *ctx, F &&f) {
  try {
    f();
    return RVP_OK;
  } catch (const Error &e) {
    if (ctx) ctx->last_error = e.msg;
    cudaGetLastError();
    return e.status;
  } catch (const std::bad_alloc &) {
    if (ctx) ctx->last_error = "host allocation failed";
    return RVP_ERR_OOM;
  } catch (...) {
    if (ctx) ctx->last_error = "unknown error";
    return RVP_ERR_CUDA;
  }
}

void oct_sync(rvp_context *ctx) { RVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream)); }

template <class T>
T oct_read(rvp_context *ctx, const T *dev) {
  T v;
  RVP_CUDA_TRY(cudaMemcpyAsync(&v, dev, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  oct_sync(ctx);
  return v;
}

// device pointer as is, or a staged copy of the host array
template <class T>
const T *oct_in(rvp_octree *o, int slot, const T *p, size_t n, int mem) {
  if (mem == RVP_MEM_DEVICE || n == 0) return p;
  DevBuf &b = wb(o->ctx, W_STAGE + slot);
  b.reserve(n * sizeof(T));
  RVP_CUDA_TRY(cudaMemcpyAsync(b.ptr, p, n * sizeof(T), cudaMemcpyHostToDevice, o->ctx->stream));
  return b.as<T>();
}

template <class T>
T *oct_out(rvp_octree *o, int slot, T *p, size_t n, int mem) {
  if (p == nullptr) return nullptr;
  if (mem == RVP_MEM_DEVICE) return p;
  wb(o->ctx, W_STAGE + slot).reserve((n ? n : 1) * sizeof(T));
  return wb(o->ctx, W_STAGE + slot).as<T>();
}

template <class T>
void oct_copy(rvp_octree *o, T *user, const T *dev, size_t n, int mem) {
  if (user == nullptr || mem == RVP_MEM_DEVICE || n == 0) return;
  RVP_CUDA_TRY(cudaMemcpyAsync(user, dev, n * sizeof(T), cudaMemcpyDeviceToHost, o->ctx->stream));
}

void sort_pairs(rvp_octree *o, u64 *keys, u32 *vals, size_t n) {
  wb(o->ctx, W_SORT).reserve(sort_temp_bytes(n));
  SortTemp st;
  sort_temp_carve(st, wb(o->ctx, W_SORT).ptr, n);
  radix_sort_pairs(o->ctx, keys, vals, n, nullptr, st);
}

// radius lists of nq queries against the tree's cloud: CSR offsets (u64,
// device) and pairs (d2 << 32 | index); by_rank: in the tree's order,
// else in (d2, index) order. Returns the total.
u64 oct_lists(rvp_octree *o, const float *qx, const float *qy, const float *qz, size_t nq,
              float radius, bool by_rank, u64 **offs_out, u64 **pairs_out) {
  rvp_context *ctx = o->ctx;
  cudaStream_t st = ctx->stream;
  // grid of cell = radius, bounded to 2^20 cells along the longest axis
  const float ext = std::max(o->box[3] - o->box[0],
                             std::max(o->box[4] - o->box[1], o->box[5] - o->box[2]));
  float cell = radius;
  const float cmin = ext > 0.0f ? ext / 1048576.0f : 0.0f;
  if (!(cell >= cmin)) cell = cmin;
  if (!(cell > 0.0f)) cell = 1.0f;
  Grid &grid = ctx_grid(ctx);
  grid_build(ctx, grid, o->x.as<float>(), o->y.as<float>(), o->z.as<float>(),
             o->offs.as<int64_t>(), 1, o->n, cell, KEY_DENSE, 0, 0, nullptr);
  const GridView gv = grid.view(KEY_DENSE, 0, 0);
  QuerySet qs{qx, qy, qz, nq, nullptr, nullptr, nullptr};
  DevBuf &bcnt = wb(ctx, W_CNT), &boffs = wb(ctx, W_LOFFS), &bscan = wb(ctx, W_SCAN);
  bcnt.reserve(nq * 4 + 16);
  u32 *cnt = bcnt.as<u32>();
  grid_radius_count(ctx, gv, qs, radius, false, cnt);
  boffs.reserve((nq + 1) * 8);
  u64 *offs = boffs.as<u64>();
  bscan.reserve(scan_temp_bytes(nq + 1));
  exclusive_scan_u32_to_u64(ctx, cnt, offs, nq, nullptr, bscan.ptr);
  const u64 tot = oct_read(ctx, offs + nq);
  if (tot >= 0xFFFFFFFFull)
    throw Error{RVP_ERR_INVALID_ARG, "radius lists exceed 2^32 - 1 entries"};
  DevBuf &bpairs = wb(ctx, W_PAIRS), &bbig = wb(ctx, W_BIG);
  bpairs.reserve((tot ? tot : 1) * 8);
  u64 *pairs = bpairs.as<u64>();
  bbig.reserve(nq * 4 + 16);
  u32 *big = bbig.as<u32>();
  grid_radius_fill(ctx, gv, qs, radius, false, offs, 0, pairs, big, big + nq);
  if (!by_rank) {
    sort_big_segments(ctx, offs, pairs, big, big + nq, (u32)std::min<size_t>(nq, 4096));
    *offs_out = offs;
    *pairs_out = pairs;
    return tot;
  }
  if (tot) {
    DevBuf &bkeys = wb(ctx, W_KEYS), &bvals = wb(ctx, W_VALS), &bp2 = wb(ctx, W_PAIRS2);
    bkeys.reserve(tot * 8);
    bvals.reserve(tot * 4);
    k_oct_list_keys<<<grid_for(nq * 32, 256, ctx->num_sms * 32), 256, 0, st>>>(
        pairs, offs, nq, o->rank.as<u32>(), bkeys.as<u64>(), bvals.as<u32>());
    RVP_LAUNCH_CHECK(ctx);
    sort_pairs(o, bkeys.as<u64>(), bvals.as<u32>(), tot);
    bp2.reserve(tot * 8);
    k_gather_u64<<<grid_for(tot, 256, ctx->num_sms * 16), 256, 0, st>>>(pairs, bvals.as<u32>(),
                                                                        tot, bp2.as<u64>());
    RVP_LAUNCH_CHECK(ctx);
    pairs = bp2.as<u64>();
  }
  *offs_out = offs;
  *pairs_out = pairs;
  return tot;
}

}  // namespace

extern "C" {

rvp_status rvp_octree_create(rvp_context *ctx, int kind, rvp_octree **out) {
  if (!ctx || !out || (kind != RVP_OCTREE && kind != RVP_POINTER_OCTREE))
    return RVP_ERR_INVALID_ARG;
  rvp_octree *o = new (std::nothrow) rvp_octree();
  if (!o) return RVP_ERR_OOM;
  o->ctx = ctx;
  o->kind = kind;
  *out = o;
  return RVP_OK;
}

rvp_status rvp_octree_destroy(rvp_octree *o) {
  if (!o) return RVP_ERR_INVALID_ARG;
  cudaSetDevice(o->ctx->device);
  cudaStreamSynchronize(o->ctx->stream);
  for (DevBuf *b : {&o->x, &o->y, &o->z, &o->offs, &o->rank, &o->order, &o->root}) b->release();
  delete o;
  return RVP_OK;
}

rvp_status rvp_octree_set_params(rvp_octree *o, int max_points_per_leaf, int max_depth,
                                 float build_epsilon) {
  if (!o) return RVP_ERR_INVALID_ARG;
  if (max_depth > kMaxDepth) {
    o->ctx->last_error = "max_depth above 21 is not supported";
    return RVP_ERR_INVALID_ARG;
  }
  o->cap = max_points_per_leaf;
  o->depth = max_depth;
  o->eps = build_epsilon;
  o->built = false;
  return RVP_OK;
}

rvp_status rvp_octree_set_input_cloud(rvp_octree *o, const float *x, const float *y,
                                      const float *z, size_t n, int mem) {
  if (!o) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = o->ctx;
  return oct_guard(ctx, [&] {
    RVP_REQUIRE(n == 0 || (x && y && z), "null cloud pointer");
    RVP_REQUIRE(n < 0x7FFFFFFFull, "clouds are limited to 2^31 - 1 points");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    // no cloud until this call has completed (see rvp_hash_set_input_cloud)
    o->has_cloud = false;
    o->built = false;
    o->n = 0;
    o->x.reserve(n * 4 + 16);
    o->y.reserve(n * 4 + 16);
    o->z.reserve(n * 4 + 16);
    o->offs.reserve(16);
    if (n) {
      const cudaMemcpyKind k =
          mem == RVP_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
      RVP_CUDA_TRY(cudaMemcpyAsync(o->x.ptr, x, n * 4, k, ctx->stream));
      RVP_CUDA_TRY(cudaMemcpyAsync(o->y.ptr, y, n * 4, k, ctx->stream));
      RVP_CUDA_TRY(cudaMemcpyAsync(o->z.ptr, z, n * 4, k, ctx->stream));
    }
    const int64_t h[2] = {0, (int64_t)n};
    RVP_CUDA_TRY(cudaMemcpyAsync(o->offs.ptr, h, 16, cudaMemcpyHostToDevice, ctx->stream));
    oct_sync(ctx);
    o->n = n;
    o->has_cloud = true;
    o->built = false;
  });
}

rvp_status rvp_octree_build(rvp_octree *o) {
  if (!o) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = o->ctx;
  return oct_guard(ctx, [&] {
    RVP_REQUIRE(o->has_cloud, "setInputCloud before build");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t n = o->n;
    o->built = false;  // set again only when this build has completed
    if (n == 0) {      // octree.cpp:35: no root, every search returns 0
      o->built = true;
      return;
    }
    cudaStream_t st = ctx->stream;
    const int D = o->depth > 0 ? o->depth : 0;
    // (size_t)max_points_per_leaf_, as octree.cpp:60 compares it
    const u64 cap = (u64)(long long)o->cap;
    o->root.reserve(64);
    u32 *enc = reinterpret_cast<u32 *>(o->root.as<char>() + 32);
    const u32 init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
    RVP_CUDA_TRY(cudaMemcpyAsync(enc, init, 24, cudaMemcpyHostToDevice, st));
    const unsigned gb = grid_for(n, 256, ctx->num_sms * 8);
    k_oct_bbox<<<gb, 256, 0, st>>>(o->x.as<float>(), o->y.as<float>(), o->z.as<float>(), n, enc);
    RVP_LAUNCH_CHECK(ctx);
    float *root = o->root.as<float>();
    k_oct_root<<<1, 32, 0, st>>>(enc, o->kind, o->eps, root);
    RVP_LAUNCH_CHECK(ctx);
    RVP_CUDA_TRY(cudaMemcpyAsync(o->box, root, 24, cudaMemcpyDeviceToHost, st));
    wb(o->ctx, W_KEYS).reserve(n * 8);
    wb(o->ctx, W_VALS).reserve(n * 4);
    u64 *keys = wb(o->ctx, W_KEYS).as<u64>();
    u32 *vals = wb(o->ctx, W_VALS).as<u32>();
    k_oct_keys<<<gb, 256, 0, st>>>(o->x.as<float>(), o->y.as<float>(), o->z.as<float>(), n, root,
                                   D, keys, vals);
    RVP_LAUNCH_CHECK(ctx);
    sort_pairs(o, keys, vals, n);
    // leaf keys by point index, then the stable sort of (leaf key, index)
    wb(o->ctx, W_PAIRS).reserve(n * 8);
    u64 *leaf = wb(o->ctx, W_PAIRS).as<u64>();
    k_oct_leaf<<<gb, 256, 0, st>>>(keys, vals, n, D, cap, leaf);
    RVP_LAUNCH_CHECK(ctx);
    RVP_CUDA_TRY(cudaMemcpyAsync(keys, leaf, n * 8, cudaMemcpyDeviceToDevice, st));
    k_iota<<<gb, 256, 0, st>>>(vals, n);
    RVP_LAUNCH_CHECK(ctx);
    sort_pairs(o, keys, vals, n);
    o->order.reserve(n * 4);
    o->rank.reserve(n * 4);
    RVP_CUDA_TRY(cudaMemcpyAsync(o->order.ptr, vals, n * 4, cudaMemcpyDeviceToDevice, st));
    k_oct_rank<<<gb, 256, 0, st>>>(vals, n, o->rank.as<u32>());
    RVP_LAUNCH_CHECK(ctx);
    oct_sync(ctx);
    o->built = true;
  });
}

rvp_status rvp_octree_order(rvp_octree *o, int mem, int32_t *order) {
  if (!o) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = o->ctx;
  return oct_guard(ctx, [&] {
    RVP_REQUIRE(o->built, "build before reading the order");
    RVP_REQUIRE(order || o->n == 0, "null output");
    if (o->n == 0) return;
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    RVP_CUDA_TRY(cudaMemcpyAsync(order, o->order.ptr, o->n * 4,
                                 mem == RVP_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                       : cudaMemcpyDeviceToHost,
                                 ctx->stream));
    oct_sync(ctx);
  });
}

rvp_status rvp_octree_radius_search(rvp_octree *o, const float *qx, const float *qy,
                                    const float *qz, size_t nq, float radius, int mem,
                                    int64_t *offsets, int32_t *indices, float *dists,
                                    size_t capacity, size_t *total) {
  if (!o) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = o->ctx;
  bool cap_fail = false;
  rvp_status s = oct_guard(ctx, [&] {
    RVP_REQUIRE(o->built, "build before radiusSearch");
    RVP_REQUIRE(offsets && total, "offsets/total required");
    RVP_REQUIRE(nq == 0 || (qx && qy && qz), "null query pointer");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    *total = 0;
    int64_t *doffs = oct_out(o, 0, offsets, nq + 1, mem);
    if (nq == 0 || o->n == 0 || !(radius >= 0.0f)) {
      RVP_CUDA_TRY(cudaMemsetAsync(doffs, 0, (nq + 1) * 8, ctx->stream));
      oct_copy(o, offsets, doffs, nq + 1, mem);
      oct_sync(ctx);
      return;
    }
    const float *dqx = oct_in(o, 1, qx, nq, mem);
    const float *dqy = oct_in(o, 2, qy, nq, mem);
    const float *dqz = oct_in(o, 3, qz, nq, mem);
    u64 *offs, *pairs;
    const u64 tot = oct_lists(o, dqx, dqy, dqz, nq, radius, true, &offs, &pairs);
    *total = (size_t)tot;
    RVP_CUDA_TRY(cudaMemcpyAsync(doffs, offs, (nq + 1) * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    oct_copy(o, offsets, doffs, nq + 1, mem);
    if (tot > capacity) {
      oct_sync(ctx);
      cap_fail = true;
      return;
    }
    int32_t *di = oct_out(o, 4, indices, tot, mem);
    float *dd = oct_out(o, 5, dists, tot, mem);
    RVP_REQUIRE(tot == 0 || (di && dd), "null output");
    if (tot) {
      k_unpack_pairs<<<grid_for(tot, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(pairs, tot,
                                                                                    di, dd);
      RVP_LAUNCH_CHECK(ctx);
    }
    oct_copy(o, indices, di, tot, mem);
    oct_copy(o, dists, dd, tot, mem);
    oct_sync(ctx);
  });
  if (s == RVP_OK && cap_fail) {
    ctx->last_error = "radius search: output capacity too small";
    return RVP_ERR_CAPACITY;
  }
  return s;
}

rvp_status rvp_sor_octree(rvp_octree *o, int k, float alpha, float search_radius, int mem,
                          float *out_aos, size_t *out_count, float *mean_dists, uint8_t *keep) {
  if (!o) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = o->ctx;
  return oct_guard(ctx, [&] {
    RVP_REQUIRE(out_count, "out_count required");
    RVP_REQUIRE(o->built, "build before sor_octree");
    *out_count = 0;
    const size_t n = o->n;
    if (n == 0) return;  // statistical_outlier_removal.cpp:222
    RVP_REQUIRE(out_aos, "null output");
    RVP_REQUIRE(k >= 1, "k must be >= 1");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const float *x = o->x.as<float>(), *y = o->y.as<float>(), *z = o->z.as<float>();
    const bool nth = o->kind == RVP_POINTER_OCTREE;
    u64 *offs, *pairs;
    const u64 tot = oct_lists(o, x, y, z, n, search_radius, nth, &offs, &pairs);
    float *mean = oct_out(o, 0, mean_dists, n, mem);
    if (!mean) {
      wb(o->ctx, W_STAGE + 0).reserve(n * 4);
      mean = wb(o->ctx, W_STAGE + 0).as<float>();
    }
    DevBuf &work = wb(ctx, W_WORK);
    if (nth) work.reserve((tot ? tot : 1) * 4);
    k_oct_sor_mean<<<grid_for(n, 128, ctx->num_sms * 16), 128, 0, st>>>(
        pairs, offs, n, k, search_radius, nth, nth ? work.as<float>() : nullptr, mean);
    RVP_LAUNCH_CHECK(ctx);
    uint8_t *dkeep = oct_out(o, 1, keep, n, mem);
    float *dout = oct_out(o, 2, out_aos, 3 * n, mem);
    wb(ctx, W_STAGE + 3).reserve(64);
    int64_t *so = wb(ctx, W_STAGE + 3).as<int64_t>();
    DevBuf &tmp = wb(ctx, W_STAGE + 4);
    tmp.reserve(sor_filter_temp_bytes(n, 1));
    sor_filter_frames(ctx, x, y, z, mean, o->offs.as<int64_t>(), 1, n, nullptr, alpha, dkeep,
                      dout, so, nullptr, tmp.ptr, nullptr, nullptr, nullptr, nullptr);
    int64_t hs[2];
    RVP_CUDA_TRY(cudaMemcpyAsync(hs, so, 16, cudaMemcpyDeviceToHost, st));
    oct_sync(ctx);
    const size_t kept = (size_t)hs[1];
    oct_copy(o, out_aos, dout, 3 * kept, mem);
    oct_copy(o, mean_dists, mean, n, mem);
    oct_copy(o, keep, dkeep, n, mem);
    oct_sync(ctx);
    *out_count = kept;
  });
}

rvp_status rvp_normals_octree(rvp_octree *o, float radius, float vp_x, float vp_y, float vp_z,
                              int eigen_iters, int mem, float *nx, float *ny, float *nz) {
  if (!o) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = o->ctx;
  return oct_guard(ctx, [&] {
    RVP_REQUIRE(o->built, "build before normal estimation");
    const size_t n = o->n;
    if (n == 0) return;  // normal_estimation.cpp:159
    RVP_REQUIRE(nx && ny && nz, "null output");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    const float *x = o->x.as<float>(), *y = o->y.as<float>(), *z = o->z.as<float>();
    u64 *offs, *pairs;
    oct_lists(o, x, y, z, n, radius, true, &offs, &pairs);
    float *dnx = oct_out(o, 0, nx, n, mem), *dny = oct_out(o, 1, ny, n, mem),
          *dnz = oct_out(o, 2, nz, n, mem);
    normals_from_lists(ctx, x, y, z, pairs, offs, nullptr, 0, n, nullptr, false, eigen_iters,
                       vp_x, vp_y, vp_z, x, y, z, dnx, dny, dnz);
    oct_copy(o, nx, dnx, n, mem);
    oct_copy(o, ny, dny, n, mem);
    oct_copy(o, nz, dnz, n, mem);
    oct_sync(ctx);
  });
}

}  // extern "C"
