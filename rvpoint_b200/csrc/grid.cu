// Cell grid ("SpatialHash") build and neighbour queries for sm_100a.
//
// Build (spatial_hashing.cpp:21-108): bbox reduction, the reference's cell
// function floor((x - min) / cell), one 64-bit key per point, stable radix
// sort of (key, index), bucket heads, an open-addressing table of occupied
// buckets {key, start | count << 32}, and the points re-laid out in bucket
// order as float4 {x, y, z, index} so a bucket is one contiguous run.
//
// Key modes:
//  * KEY_REF_HASH: the reference's hashCell ix + iy*p1 + iz*p2
//    (spatial_hashing.h:43-45). Buckets are then exactly the reference's
//    grid_ entries, collisions included.
//  * KEY_DENSE: per-frame dense keys for many frames in one sort and one
//    table. Keys are hierarchical (a Morton code of the fine cell inside a
//    group of 64 x 64 x 64), so the cells of every level c, 2c, 4c, ... are
//    contiguous runs of the sorted points; the table holds five levels.
//
// Queries: one warp per query. Lanes look up up to 32 window cells at once,
// a warp scan of bucket sizes flattens the window into one candidate stream,
// and lanes walk it 32 candidates at a time (contiguous float4 loads inside a
// bucket). A radius window is the tight cell range of [q - r, q + r]
// computed with a monotone, conservative bound, which provably contains
// every point with d2 <= r2 (so the result equals the reference's larger
// ceil(r/cell)+1 window whenever the hash has no collisions; with
// collisions the reference's own window is scanned instead).
#include <math.h>

#include "internal.cuh"
#include "grid_device.cuh"

namespace rvp {
using namespace gd;

namespace {

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

__device__ __forceinline__ int frame_of_index(const int64_t *offs, int n_frames, size_t i) {
  int lo = 0, hi = n_frames - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((size_t)offs[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// ---------------------------------------------------------------------------
// bbox per frame
// ---------------------------------------------------------------------------
__global__ void k_bbox_init(float *bb, int n_frames) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n_frames; f += gridDim.x * blockDim.x) {
    bb[6 * f + 0] = bb[6 * f + 1] = bb[6 * f + 2] = INFINITY;
    bb[6 * f + 3] = bb[6 * f + 4] = bb[6 * f + 5] = -INFINITY;
  }
}

// One contiguous run of points per warp; running min / max in registers,
// flushed with atomics only where the run crosses into the next frame.
__global__ void k_bbox(const float *__restrict__ x, const float *__restrict__ y,
                       const float *__restrict__ z, const int64_t *offs, int n_frames,
                       size_t n_max, const u64 *n_dev, float *bb) {
  const size_t n = n_dev ? *n_dev : n_max;
  const int lane = threadIdx.x & 31;
  const size_t warps = ((size_t)gridDim.x * blockDim.x) >> 5;
  const size_t w = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t per = ((n + warps - 1) / warps + 31) & ~(size_t)31;
  const size_t a = w * per, e = a + per < n ? a + per : n;
  if (a >= e) return;
  int f = n_frames > 1 ? frame_of_index(offs, n_frames, a) : 0;
  size_t f_end = n_frames > 1 ? (size_t)offs[f + 1] : n;
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  auto flush = [&](int fr) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      for (int o = 16; o; o >>= 1) {
        mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
        mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
      }
      if (lane == 0 && mn[k] <= mx[k]) {
        atomic_min_f(bb + 6 * fr + k, mn[k]);
        atomic_max_f(bb + 6 * fr + 3 + k, mx[k]);
      }
      mn[k] = INFINITY;
      mx[k] = -INFINITY;
    }
  };
  for (size_t base = a; base < e; base += 32) {
    while (n_frames > 1 && base >= f_end && f + 1 < n_frames) {
      flush(f);
      ++f;
      f_end = (size_t)offs[f + 1];
    }
    const size_t i = base + lane;
    if (i < e) {
      const float v[3] = {x[i], y[i], z[i]};
      if (i >= f_end) {  // already in a later frame
        const int fi = frame_of_index(offs, n_frames, i);
        float *bf = bb + 6 * fi;
        atomic_min_f(bf + 0, v[0]); atomic_min_f(bf + 1, v[1]); atomic_min_f(bf + 2, v[2]);
        atomic_max_f(bf + 3, v[0]); atomic_max_f(bf + 4, v[1]); atomic_max_f(bf + 5, v[2]);
      } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          mn[k] = fminf(mn[k], v[k]);
          mx[k] = fmaxf(mx[k], v[k]);
        }
      }
    }
  }
  flush(f);
}

// setInputCloud's padding and grid dimensions (spatial_hashing.cpp:86-95),
// then (dense mode) each frame's first key.
// One block: a thread per frame computes its grid, then a block-wide
// exclusive scan of the level-3 group counts gives each frame's key_base.
__global__ __launch_bounds__(1024) void k_grid_params(GridFrame *fr, const float *bb,
                                                      int n_frames, float cell) {
  __shared__ u64 warp_sum[32];
  __shared__ u64 carry;
  if (blockIdx.x != 0) return;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int f0 = 0; f0 < n_frames; f0 += blockDim.x) {
    const int f = f0 + tid;
    GridFrame g;
    u64 groups = 0;
    if (f < n_frames) {
      const float *b = bb + 6 * f;
      g.cell = cell;
      if (b[0] > b[3]) {  // empty frame
        g.min_x = g.min_y = g.min_z = 0.0f;
        g.gx = g.gy = g.gz = 1;
      } else {
        const float eps = fmul(cell, 0.01f);
        g.min_x = fsub(b[0], eps); g.min_y = fsub(b[1], eps); g.min_z = fsub(b[2], eps);
        const float max_x = fadd(b[3], eps), max_y = fadd(b[4], eps), max_z = fadd(b[5], eps);
        g.gx = (int)ceilf(fdiv(fsub(max_x, g.min_x), cell)) + 1;
        g.gy = (int)ceilf(fdiv(fsub(max_y, g.min_y), cell)) + 1;
        g.gz = (int)ceilf(fdiv(fsub(max_z, g.min_z), cell)) + 1;
      }
      g.g3x = (g.gx + 63) >> 6;
      g.g3y = (g.gy + 63) >> 6;
      g.g3z = (g.gz + 63) >> 6;
      groups = ((u64)g.g3x * (u64)g.g3y * (u64)g.g3z) << 18;
    }
    // inclusive scan of groups over the block
    u64 v = groups;
    for (int o = 1; o < 32; o <<= 1) {
      const u64 t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    if (lane == 31) warp_sum[wid] = v;
    __syncthreads();
    u64 before = carry;
    for (int k = 0; k < wid; ++k) before += warp_sum[k];
    if (f < n_frames) {
      g.key_base = before + v - groups;
      fr[f] = g;
    }
    __syncthreads();
    if (tid == blockDim.x - 1) carry = before + v;
    __syncthreads();
  }
}

__global__ void k_cell_keys(const float *__restrict__ x, const float *__restrict__ y,
                            const float *__restrict__ z, const int64_t *offs, int n_frames,
                            size_t n_max, const u64 *n_dev, const GridFrame *frames, int mode,
                            long long p1, long long p2, u64 *keys, u32 *vals) {
  const size_t n = n_dev ? *n_dev : n_max;
  GridView gv;
  gv.mode = mode; gv.p1 = p1; gv.p2 = p2;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int f = n_frames > 1 ? frame_of_index(offs, n_frames, i) : 0;
    const GridFrame F = frames[f];
    const int cx = cell_axis(x[i], F.min_x, F.cell);
    const int cy = cell_axis(y[i], F.min_y, F.cell);
    const int cz = cell_axis(z[i], F.min_z, F.cell);
    keys[i] = fine_key(gv, F, cx, cy, cz);
    vals[i] = (u32)i;
  }
}

// heads of the buckets of level base + j: key >> 3 (base + j) changes
// (dense mode: j = 0 .. kHeadLevels - 1; the reference hash: base 0, j = 0)
__global__ void k_heads(const u64 *keys, size_t n_max, const u64 *n_dev, int levels, int base,
                        u32 *heads) {
  const size_t n = n_dev ? *n_dev : n_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const u64 k = keys[i];
    const u64 p = i ? keys[i - 1] : 0;
    for (int j = 0; j < levels; ++j) {
      const int sh = 3 * (base + j);
      heads[(size_t)j * n_max + i] = (i == 0 || (k >> sh) != (p >> sh)) ? 1u : 0u;
    }
  }
}

__global__ void k_reorder(const float *__restrict__ x, const float *__restrict__ y,
                          const float *__restrict__ z, const float *__restrict__ aos,
                          const u32 *vals, const u32 *heads,
                          const u64 *bucket_of, size_t n_max, const u64 *n_dev, int levels,
                          float4 *pts, u32 *lstart, const GridFrame *frames, int mode,
                          int *collision, u32 *pos_of) {
  const size_t n = n_dev ? *n_dev : n_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const u32 v = vals[i];
    float px, py, pz;
    if (aos) {
      px = aos[3 * (size_t)v];
      py = aos[3 * (size_t)v + 1];
      pz = aos[3 * (size_t)v + 2];
    } else {
      px = x[v];
      py = y[v];
      pz = z[v];
    }
    pts[i] = make_float4(px, py, pz, __uint_as_float(v));
    pos_of[v] = (u32)i;
    for (int L = 0; L < levels; ++L)
      if (heads[(size_t)L * n_max + i])
        lstart[(size_t)L * n_max + bucket_of[(size_t)L * (n_max + 1) + i]] = (u32)i;
    if (mode == KEY_REF_HASH && !heads[i]) {
      // same key as the previous point: a different cell means a collision
      const u32 u = vals[i - 1];
      const GridFrame F = frames[0];
      if (cell_axis(px, F.min_x, F.cell) != cell_axis(x[u], F.min_x, F.cell) ||
          cell_axis(py, F.min_y, F.cell) != cell_axis(y[u], F.min_y, F.cell) ||
          cell_axis(pz, F.min_z, F.cell) != cell_axis(z[u], F.min_z, F.cell))
        *collision = 1;
    }
  }
}

// The quarter-cell directory of the level-base cells (base 2) of kSubMin to
// kSubMax points: one warp per cell walks its points (sorted by the 6-bit
// Morton code of their quarter cell, the key's low bits) and writes, for
// every code s, the offset of the first point with code >= s to sub_off[st +
// s] (the cell's own positions: it has at least 64).
__global__ void k_sub_dir(const u64 *keys, const u32 *lstart0, const u64 *nbuckets,
                          const u64 *n_dev, uint16_t *sub_off) {
  const u64 n = *n_dev;
  const u64 nb = nbuckets[0];
  const int lane = threadIdx.x & 31;
  const u64 warps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 b = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += warps) {
    const u32 st = lstart0[b];
    const u32 en = b + 1 < nb ? lstart0[b + 1] : (u32)n;
    const u32 ct = en - st;
    if (ct < kSubMin || ct > kSubMax) continue;
    int prev = -1;  // code of the point before this chunk
    for (u32 i0 = st; i0 < en; i0 += 32) {
      const u32 i = i0 + lane;
      const int code = i < en ? (int)(keys[i] & 63u) : 64;
      int before = __shfl_up_sync(0xffffffffu, code, 1);
      if (lane == 0) before = prev;
      // codes (before, code] start at this point
      if (i < en)
        for (int s = before + 1; s <= code; ++s) sub_off[st + s] = (uint16_t)(i - st);
      prev = __shfl_sync(0xffffffffu, code, 31);
      if (prev == 64) {  // the chunk ran past the cell: the last live code
        const unsigned live = __ballot_sync(0xffffffffu, i < en);
        prev = __shfl_sync(0xffffffffu, code, 31 - __clz(live));
      }
    }
    // codes past the last point: the cell's end
    for (int s = prev + 1 + lane; s < 64; s += 32) sub_off[st + s] = (uint16_t)ct;
  }
}

__device__ __forceinline__ void table_put(ulonglong2 *table, u64 mask, u64 key, u64 ent,
                                          int *overflow) {
  u64 slot = mix64(key) & mask;
  for (u64 probe = 0; probe <= mask; ++probe) {
    const u64 prev = atomicCAS(&table[slot].x, kEmptyKey, key);
    if (prev == kEmptyKey || prev == key) {
      table[slot].y = ent;
      return;
    }
    slot = (slot + 1) & mask;
  }
  *overflow = 1;
}

// one thread per bucket of levels 0 .. table_levels-1: {tagged key,
// start | count << 32} into the open-addressing table (linear probing)
__global__ void k_insert(const u64 *keys, const u32 *lstart, const u64 *bucket_of, size_t n_max,
                         const u64 *n_dev, int levels, int table_levels, int base,
                         ulonglong2 *table, u64 mask, u64 *nbuckets, int *overflow) {
  const size_t n = n_dev ? *n_dev : n_max;
  u64 nb[kHeadLevels] = {};
  u64 tot = 0;
  for (int L = 0; L < levels; ++L) {
    nb[L] = bucket_of[(size_t)L * (n_max + 1) + n];
    if (L < table_levels) tot += nb[L];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0)
    for (int L = 0; L < kHeadLevels; ++L) nbuckets[L] = nb[L];
  for (u64 b = blockIdx.x * (u64)blockDim.x + threadIdx.x; b < tot;
       b += (u64)gridDim.x * blockDim.x) {
    int L = 0;
    u64 c = b;
    while (c >= nb[L]) c -= nb[L++];
    const u32 *st = lstart + (size_t)L * n_max;
    const u32 s = st[c];
    const u32 e = (c + 1 < nb[L]) ? st[c + 1] : (u32)n;
    const int La = base + L;  // the bucket's level
    const u64 key = La == 0 ? keys[s] : (((u64)La << 60) | (keys[s] >> (3 * La)));
    table_put(table, mask, key, (u64)s | ((u64)(e - s) << 32), overflow);
  }
}

__global__ void k_set_count(u64 *dst, const u64 *src, u64 value) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = src ? *src : value;
}

}  // namespace

// ---------------------------------------------------------------------------
// Grid storage
// ---------------------------------------------------------------------------
static u64 next_pow2(u64 v) {
  u64 p = 1;
  while (p < v) p <<= 1;
  return p;
}

void Grid::reserve(size_t n, int nf) {
  if (n < 1) n = 1;
  if (nf < 1) nf = 1;
  // every buffer is asked for its size on every call (a no-op when it is
  // large enough), so an allocation that failed part-way leaves nothing
  // marked as reserved that is not
  n_max = n > n_max ? n : n_max;
  n_frames_max = nf > n_frames_max ? nf : n_frames_max;
  b_keys.reserve(n_max * 8);
  b_vals.reserve(n_max * 4);
  b_pts.reserve(n_max * 16);
  b_frames.reserve(al(n_frames_max * sizeof(GridFrame)) + al(n_frames_max * 6 * 4));
  b_begin.reserve(al((n_frames_max + 1) * 8));
  b_sort.reserve(sort_temp_bytes(n_max) + al(kHeadLevels * n_max * 4) +
                 al(kHeadLevels * (n_max + 1) * 8) +
                 kHeadLevels * scan_temp_bytes(n_max));
  b_lstart.reserve(al(kHeadLevels * n_max * 4));
  b_pos.reserve(n_max * 4);
  b_sub.reserve(al(n_max * 2));
  b_misc.reserve(256);
  d_n = b_misc.as<u64>();
  d_nbuckets = d_n + 1;
  d_collision = reinterpret_cast<int *>(d_n + 1 + kHeadLevels);
  d_overflow = d_collision + 1;
  // the buckets of the table levels never exceed kGridLevels n (each holds a
  // point; in practice ~1.4 n): without a measured count the table holds
  // that many, so no insert can fail; rvp_pipeline_fit_tables and the
  // scorer shrink it to the measured count so that it stays in L2
  const size_t want =
      table_cap_req ? table_cap_req
                    : (size_t)next_pow2((u64)(kGridLevels * n_max + n_max / 4 + 1024));
  if (want != table_cap || !b_table.ptr) {
    table_cap = 0;
    b_table.release();
    b_table.reserve(want * 16);
    table_cap = want;
  }
}

void Grid::fit_table(size_t buckets) {
  table_cap_req = (size_t)next_pow2((u64)(buckets * 5 / 2 + 1024));
  reserve(n_max, n_frames_max);
}

void Grid::release() {
  b_keys.release(); b_vals.release(); b_pts.release(); b_table.release();
  b_frames.release(); b_begin.release(); b_sort.release(); b_misc.release();
  b_lstart.release(); b_pos.release(); b_sub.release();
  n_max = 0; n_frames_max = 0; table_cap = 0;
}

GridView Grid::view(int mode, long long p1, long long p2) const {
  GridView v;
  v.pts = b_pts.as<float4>();
  v.table = b_table.as<ulonglong2>();
  v.table_mask = (u64)table_cap - 1;
  v.frames = b_frames.as<GridFrame>();
  v.frame_pt_begin = b_begin.as<u64>();
  v.mode = mode;
  v.p1 = p1;
  v.p2 = p2;
  for (int L = 0; L < kHeadLevels; ++L) v.lstart[L] = b_lstart.as<u32>() + (size_t)L * n_max;
  v.n_level = d_nbuckets;
  v.n_points = d_n;
  v.pos_of = b_pos.as<u32>();
  v.lbase = lbase;
  v.sub_off = mode == KEY_DENSE && lbase == 2 ? b_sub.as<uint16_t>() : nullptr;
  return v;
}

void grid_build(rvp_context *ctx, Grid &g, const float *x, const float *y, const float *z,
                const int64_t *offs, int n_frames, size_t n_points, float cell, int mode,
                long long p1, long long p2, const u64 *n_dev_opt, int base_level,
                const float *xyz_aos) {
  g.reserve(n_points, n_frames);
  const int base = mode == KEY_DENSE ? base_level : 0;
  g.lbase = base;
  cudaStream_t st = ctx->stream;
  const size_t n_max = n_points;
  const u64 *n_dev = n_dev_opt;
  const int levels = mode == KEY_DENSE ? kHeadLevels : 1;
  const int table_levels = mode == KEY_DENSE ? kGridLevels : 1;
  GridFrame *frames = g.b_frames.as<GridFrame>();
  float *bb = reinterpret_cast<float *>(g.b_frames.as<char>() + al(g.n_frames_max * sizeof(GridFrame)));
  u64 *begin = g.b_begin.as<u64>();
  RVP_CUDA_TRY(cudaMemcpyAsync(begin, offs, (n_frames + 1) * 8, cudaMemcpyDeviceToDevice, st));
  char *sp = g.b_sort.as<char>();
  SortTemp t;
  sort_temp_carve(t, sp, g.n_max);
  sp += sort_temp_bytes(g.n_max);
  // per-level arrays use stride n_max (heads, starts) / n_max + 1 (ids)
  u32 *heads = reinterpret_cast<u32 *>(sp); sp += al(kHeadLevels * g.n_max * 4);
  u64 *bucket_of = reinterpret_cast<u64 *>(sp); sp += al(kHeadLevels * (g.n_max + 1) * 8);
  void *scan_tmp = sp;
  u32 *lstart = g.b_lstart.as<u32>();
  // strides below are g.n_max; the kernels are given g.n_max as their n_max
  const size_t nm = g.n_max;

  const int sms = ctx->num_sms;
  const unsigned gb = grid_for(n_max, 256, sms * 16);
  k_set_count<<<1, 32, 0, st>>>(g.d_n, n_dev, (u64)n_max);
  RVP_LAUNCH_CHECK(ctx);
  k_bbox_init<<<grid_for(n_frames, 256, 64), 256, 0, st>>>(bb, n_frames);
  RVP_LAUNCH_CHECK(ctx);
  k_bbox<<<gb, 256, 0, st>>>(x, y, z, offs, n_frames, n_max, n_dev, bb);
  RVP_LAUNCH_CHECK(ctx);
  // the sort cell: the query cell over 2^base (exact in float)
  k_grid_params<<<1, 1024, 0, st>>>(frames, bb, n_frames, ldexpf(cell, -base));
  RVP_LAUNCH_CHECK(ctx);
  k_cell_keys<<<gb, 256, 0, st>>>(x, y, z, offs, n_frames, n_max, n_dev, frames, mode, p1, p2,
                                  g.b_keys.as<u64>(), g.b_vals.as<u32>());
  RVP_LAUNCH_CHECK(ctx);
  radix_sort_pairs(ctx, g.b_keys.as<u64>(), g.b_vals.as<u32>(), n_max, n_dev, t);
  // n for these kernels: the live count (n_dev) or n_max; strides: nm
  const u64 *n_live = n_dev ? n_dev : g.d_n;
  k_heads<<<gb, 256, 0, st>>>(g.b_keys.as<u64>(), nm, n_live, levels, base, heads);
  RVP_LAUNCH_CHECK(ctx);
  // bucket_of[L][i] = number of level-L heads before i (the bucket id of a head)
  exclusive_scan_u32_to_u64_batch(ctx, heads, nm, bucket_of, nm + 1, levels, nm, n_live,
                                  scan_tmp);
  RVP_CUDA_TRY(cudaMemsetAsync(g.b_table.ptr, 0xFF, g.table_cap * 16, st));
  // buckets per level, collision, overflow
  RVP_CUDA_TRY(cudaMemsetAsync(g.d_nbuckets, 0, 8 * kHeadLevels + 8, st));
  k_reorder<<<gb, 256, 0, st>>>(x, y, z, xyz_aos, g.b_vals.as<u32>(), heads, bucket_of, nm,
                                n_live, levels,
                                g.b_pts.as<float4>(), lstart, frames, mode, g.d_collision,
                                g.b_pos.as<u32>());
  RVP_LAUNCH_CHECK(ctx);
  k_insert<<<gb, 256, 0, st>>>(g.b_keys.as<u64>(), lstart, bucket_of, nm, n_live, levels,
                               table_levels, base, g.b_table.as<ulonglong2>(),
                               (u64)g.table_cap - 1,
                               g.d_nbuckets, g.d_overflow);
  RVP_LAUNCH_CHECK(ctx);
  if (mode == KEY_DENSE && base == 2) {
    k_sub_dir<<<sms * 8, 256, 0, st>>>(g.b_keys.as<u64>(), lstart, g.d_nbuckets, n_live,
                                       g.b_sub.as<uint16_t>());
    RVP_LAUNCH_CHECK(ctx);
  }
}

// ===========================================================================
// Queries
// ===========================================================================
namespace {

// ---------------------------------------------------------------------------
// radius search: count pass
// ---------------------------------------------------------------------------
__global__ void k_radius_count(GridView g, QuerySet q, float radius, bool ref_win, u32 *counts) {
  const size_t nq = q.n_dev ? *q.n_dev : q.n_max;
  const int lane = threadIdx.x & 31;
  const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
  const float r2 = fmul(radius, radius);
  for (size_t wi = warp; wi < nq; wi += nwarps) {
    const u32 qi = query_index(q, wi);
    const int f = q.frame_of ? q.frame_of[qi] : 0;
    const GridFrame F = g.frames[f];
    const float qx = q.x[qi], qy = q.y[qi], qz = q.z[qi];
    const Window w = ref_win ? ref_window(F, qx, qy, qz, radius)
                             : tight_window(F, qx, qy, qz, (double)radius);
    u32 cnt = 0;
    for_each_candidate(g, F, f, w, false, [&](float4 p, bool valid) {
      const bool pass = valid && !(__float_as_uint(p.w) & kRemovedBit) &&
                        dist2(p.x, p.y, p.z, qx, qy, qz) <= r2;
      cnt += __popc(__ballot_sync(0xffffffffu, pass));
    });
    if (lane == 0) counts[qi] = cnt;
  }
}

// ---------------------------------------------------------------------------
// radius search: fill pass with per-warp shared-memory staging and sort
// ---------------------------------------------------------------------------
constexpr int FILL_WARPS = 4;
constexpr int FILL_CAP = 1024;  // pairs staged per warp (8 KB)

__device__ __forceinline__ void warp_bitonic_smem(u64 *s, int P) {
  const int lane = threadIdx.x & 31;
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < P; i += 32) {
        const int l = i ^ j;
        if (l > i) {
          const u64 a = s[i], b = s[l];
          const bool up = (i & k) == 0;
          if ((a > b) == up) { s[i] = b; s[l] = a; }
        }
      }
      __syncwarp();
    }
  }
}

__global__ __launch_bounds__(FILL_WARPS * 32) void k_radius_fill(GridView g, QuerySet q,
                                                                 float radius, bool ref_win,
                                                                 const u64 *offsets, u64 *out,
                                                                 u32 *big_list, u32 *big_count) {
  __shared__ u64 stage[FILL_WARPS][FILL_CAP];
  const size_t nq = q.n_dev ? *q.n_dev : q.n_max;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
  const float r2 = fmul(radius, radius);
  u64 *s = stage[wib];
  for (size_t wi = warp; wi < nq; wi += nwarps) {
    const u32 qi = query_index(q, wi);
    const u64 off = offsets[qi];
    const u32 cnt = (u32)(offsets[qi + 1] - off);
    if (cnt == 0) continue;
    const int f = q.frame_of ? q.frame_of[qi] : 0;
    const GridFrame F = g.frames[f];
    const float qx = q.x[qi], qy = q.y[qi], qz = q.z[qi];
    const Window w = ref_win ? ref_window(F, qx, qy, qz, radius)
                             : tight_window(F, qx, qy, qz, (double)radius);
    const bool staged = cnt <= FILL_CAP;
    u32 pos = 0;
    for_each_candidate(g, F, f, w, false, [&](float4 p, bool valid) {
      const u32 idx = __float_as_uint(p.w);
      float d2 = 0.0f;
      bool pass = false;
      if (valid && !(idx & kRemovedBit)) {
        d2 = dist2(p.x, p.y, p.z, qx, qy, qz);
        pass = d2 <= r2;
      }
      const unsigned b = __ballot_sync(0xffffffffu, pass);
      if (pass) {
        const u32 at = pos + __popc(b & ((1u << lane) - 1));
        if (at < cnt) {
          const u64 key = pack_nbr(d2, (int)idx);
          if (staged) s[at] = key; else out[off + at] = key;
        }
      }
      pos += __popc(b);
    });
    if (staged) {
      int P = 1;
      while (P < (int)cnt) P <<= 1;
      for (int i = (int)cnt + lane; i < P; i += 32) s[i] = ~0ull;
      __syncwarp();
      warp_bitonic_smem(s, P);
      for (u32 i = lane; i < cnt; i += 32) out[off + i] = s[i];
      __syncwarp();
    } else if (lane == 0) {
      const u32 slot = atomicAdd(big_count, 1u);
      big_list[slot] = qi;
    }
  }
}

// one block per oversized segment: bitonic sort, in shared memory when it
// fits (<= 8192 pairs), else in global memory.
constexpr int BIG_SMEM = 8192;
__global__ __launch_bounds__(1024) void k_sort_big(const u64 *offsets, u64 *pairs,
                                                   const u32 *big_list, const u32 *big_count) {
  extern __shared__ u64 sb[];
  const u32 nb = *big_count;
  for (u32 b = blockIdx.x; b < nb; b += gridDim.x) {
    const u32 qi = big_list[b];
    const u64 off = offsets[qi];
    const u64 cnt = offsets[qi + 1] - off;
    u64 P = 1;
    while (P < cnt) P <<= 1;
    u64 *a = pairs + off;
    if (P <= BIG_SMEM) {
      for (u64 i = threadIdx.x; i < P; i += blockDim.x) sb[i] = i < cnt ? a[i] : ~0ull;
      __syncthreads();
      for (u64 k = 2; k <= P; k <<= 1)
        for (u64 j = k >> 1; j > 0; j >>= 1) {
          for (u64 i = threadIdx.x; i < P; i += blockDim.x) {
            const u64 l = i ^ j;
            if (l > i) {
              const u64 x = sb[i], y = sb[l];
              if ((x > y) == ((i & k) == 0)) { sb[i] = y; sb[l] = x; }
            }
          }
          __syncthreads();
        }
      for (u64 i = threadIdx.x; i < cnt; i += blockDim.x) a[i] = sb[i];
      __syncthreads();
    } else {
      // virtual padding: indices >= cnt hold +inf and never move
      for (u64 k = 2; k <= P; k <<= 1)
        for (u64 j = k >> 1; j > 0; j >>= 1) {
          for (u64 i = threadIdx.x; i < P; i += blockDim.x) {
            const u64 l = i ^ j;
            if (l > i) {
              const u64 x = i < cnt ? a[i] : ~0ull;
              const u64 y = l < cnt ? a[l] : ~0ull;
              if ((x > y) == ((i & k) == 0)) {
                if (i < cnt) a[i] = y;
                if (l < cnt) a[l] = x;
              }
            }
          }
          __syncthreads();
        }
    }
  }
}

__device__ __forceinline__ u64 bound_of(float tau) { return pack_nbr(tau, 0x7FFFFFFF) | 0xFFFFFFFFull; }


template <int P>
__global__ __launch_bounds__(256, 4) void k_knn_warp(GridView g, QuerySet q, int K, float radius,
                                                  u64 *out, int32_t *out_counts, u32 *stats,
                                                  int out_mode, float *mean) {
  const size_t nq = q.n_dev ? *q.n_dev : q.n_max;
  const int lane = threadIdx.x & 31;
  const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
  const bool two_level = g.mode == KEY_DENSE;
  for (size_t wi = warp; wi < nq; wi += nwarps) {
    if (q.bound && q.bound[wi] == kTauDone) continue;  // finished by the tau pass
    const u32 qi = query_index(q, wi);
    const int f = q.frame_of ? q.frame_of[qi] : 0;
    const GridFrame F = g.frames[f];
    const float qx = q.x[qi], qy = q.y[qi], qz = q.z[qi];
    WarpList<P> L;
    L.init();
    u32 found = 0;
    int path = 5;
    if (radius > 0.0f) {
      const float r2 = fmul(radius, radius);
      const Window w = tight_window(F, qx, qy, qz, (double)radius);
      knn_scan<P>(g, F, f, w, false, qx, qy, qz, K, bound_of(r2), L, found);
    } else {
      float tb = q.bound ? q.bound[wi] : -1.0f;
      bool est_done = false;
      if (tb == kTauEstimate && two_level) {
        // E) no bound, but a radius estimated from the finest level whose
        //    own cell holds K points (r = cell * sqrt(K / count), under one
        //    cell; lanes look the levels up together): the tight window of r
        //    at the finest level where it spans at most 128 cells, scanned
        //    bounded by r^2 -- exact when K points lie within r; else r grows
        //    (by the shortfall) and the window is scanned again
        tb = -1.0f;  // the rings below, should the estimates run out
        const int top = g.lbase + kGridLevels - 1;
        const int fx = cell_axis(qx, F.min_x, F.cell), fy = cell_axis(qy, F.min_y, F.cell),
                  fz = cell_axis(qz, F.min_z, F.cell);
        const int lv = g.lbase + lane;
        u32 ct = 0;
        if (lv <= top) {
          u32 st;
          if (!lookup(g, level_key(g, F, lv, fx >> lv, fy >> lv, fz >> lv), st, ct)) ct = 0;
        }
        const unsigned ok = __ballot_sync(0xffffffffu, lv <= top && ct >= (u32)K);
        const int src = ok ? __ffs(ok) - 1 : 0;
        const u32 c_src = __shfl_sync(0xffffffffu, ct, src);
        float r = F.cell * (float)(1 << top);
        if (ok) {
          const float cs = F.cell * (float)(1 << (g.lbase + src));
          r = fminf(cs * sqrtf((float)K / (float)c_src), cs);
        }
        for (int attempt = 0; attempt < kEstimateTries && !est_done; ++attempt) {
          const float t2 = r * r;
          int lt = -1;
          Window wt;
          for (int l = g.lbase; l <= top; ++l) {
            wt = tight_window(F, qx, qy, qz, sqrt((double)t2), l);
            if (window_cells(wt) <= 128) {
              lt = l;
              break;
            }
          }
          if (lt < 0) break;
          L.init();
          found = 0;
          knn_scan<P>(g, F, f, wt, false, qx, qy, qz, K, bound_of(t2), L, found);
          if (found >= (u32)K) {
            est_done = true;
            path = 0;
          } else {
            r *= found > 0 ? fmaxf(1.3f, 1.1f * sqrtf((float)K / (float)found)) : 2.0f;
          }
        }
        if (!est_done) {
          L.init();
          found = 0;
        }
      }
      if (!est_done) {
      // 0) a known bound: every point with d2 <= tb lies in the tight window
      //    of sqrt(tb), and there are >= K of them -- scan it directly
      Window wr = ring_window(F, qx, qy, qz, 1, g.lbase);
      int lvl = g.lbase;
      if (tb >= 0.0f) {
        found = 0;
      } else {
        // 1) rings of +- 1 cell, coarser (x4) while they hold fewer than K
        knn_scan<P>(g, F, f, wr, false, qx, qy, qz, K, ~0ull - 1, L, found);
      }
      while (tb < 0.0f && found < (u32)K && two_level && lvl + 1 < g.lbase + kGridLevels) {
        ++lvl;
        wr = ring_window(F, qx, qy, qz, 1, lvl);
        L.init();
        found = 0;
        knn_scan<P>(g, F, f, wr, false, qx, qy, qz, K, ~0ull - 1, L, found);
      }
      path = lvl == g.lbase ? 0 : (lvl == g.lbase + 1 ? 2 : 3);
      bool done = false;
      if (found >= (u32)K || tb >= 0.0f) {
        const float tau = tb >= 0.0f ? tb : nbr_d2(L.get(K - 1));
        if (tb < 0.0f) {
          const double cov = coverage(F, wr, qx, qy, qz);
          if (cov > 0.0 && (double)tau < cov * cov * (1.0 - 1e-5)) done = true;
        }
        if (!done) {
          // 2) every point with d2 <= tau lies in the tight window of
          //    sqrt(tau) and there are >= K of them: exact. Scan it at the
          //    finest level whose window has at most 1024 cells (32 lookup
          //    rounds), skipping cells beyond the K-th distance: small cells
          //    keep the scan close to the ball of sqrt(tau)
          const double rt = sqrt((double)tau);
          const int top = two_level ? g.lbase + kGridLevels - 1 : 0;
          for (int lt = two_level ? g.lbase : 0; lt <= top && !done; ++lt) {
            const Window wt = tight_window(F, qx, qy, qz, rt, lt);
            const long long cells = window_cells(wt);
            if (cells <= (two_level ? (lt == top ? 4096 : 1024) : 4096)) {
              L.init();
              found = 0;
              knn_scan<P>(g, F, f, wt, false, qx, qy, qz, K, bound_of(tau), L, found);
              done = true;
              path = 1;
            }
          }
        }
      }
      if (!done) {  // 3) whole frame
        L.init();
        found = 0;
        knn_scan<P>(g, F, f, wr, true, qx, qy, qz, K, ~0ull - 1, L, found);
        path = 4;
      }
      }  // !est_done
    }
    const u32 cnt = found < (u32)K ? found : (u32)K;
    if (out_mode == KNN_OUT_SOR_MEAN || out_mode == KNN_OUT_SOR_MEAN_LIST) {
      // sor_sc's mean (statistical_outlier_removal.cpp:36-40): ascending
      // sum of sqrtf(d2_j), j = 1..k, divided by k (fewer if the frame is
      // smaller than k+1)
      const int valid_k = (int)cnt - 1 < K - 1 ? (int)cnt - 1 : K - 1;
      float sum = 0.0f;
      for (int j = 1; j < K; ++j) {
        const float d = nbr_d2(L.get(j));
        if (j <= valid_k) sum = fadd(sum, __fsqrt_rn(d));
      }
      if (lane == 0) mean[qi] = valid_k > 0 ? fdiv(sum, (float)valid_k) : 0.0f;
      if (out_mode == KNN_OUT_SOR_MEAN_LIST) {  // by grid position, of grid positions
        u32 *row = reinterpret_cast<u32 *>(out) + (size_t)g.pos_of[qi] * K;
#pragma unroll
        for (int s = 0; s < P; ++s) {
          const int j = s * 32 + lane;
          if (j < K)
            row[j] = j < (int)cnt ? g.pos_of[(u32)nbr_idx(L.e[s]) & 0x7FFFFFFFu] : 0xFFFFFFFFu;
        }
      }
    } else {
      const size_t row = out_mode == KNN_OUT_BY_SLOT ? wi : (size_t)qi;
#pragma unroll
      for (int s = 0; s < P; ++s) {
        const int j = s * 32 + lane;
        if (j < (int)cnt) out[row * K + j] = L.e[s];
      }
      if (lane == 0 && out_counts) out_counts[row] = (int32_t)cnt;
    }
    if (lane == 0 && stats) atomicAdd(&stats[path], 1u);
  }
}

}  // namespace

void grid_radius_count(rvp_context *ctx, const GridView &g, const QuerySet &q, float radius,
                       bool ref_window, u32 *counts) {
  const unsigned blocks = grid_for(q.n_max * 32, 256, ctx->num_sms * 16);
  k_radius_count<<<blocks, 256, 0, ctx->stream>>>(g, q, radius, ref_window, counts);
  RVP_LAUNCH_CHECK(ctx);
}

void grid_radius_fill(rvp_context *ctx, const GridView &g, const QuerySet &q, float radius,
                      bool ref_window, const u64 *offsets, int max_nn, u64 *out_pairs,
                      u32 *big_list, u32 *big_count) {
  (void)max_nn;
  RVP_CUDA_TRY(cudaMemsetAsync(big_count, 0, 4, ctx->stream));
  const unsigned blocks = grid_for(q.n_max * 32, FILL_WARPS * 32, ctx->num_sms * 16);
  k_radius_fill<<<blocks, FILL_WARPS * 32, 0, ctx->stream>>>(g, q, radius, ref_window, offsets,
                                                             out_pairs, big_list, big_count);
  RVP_LAUNCH_CHECK(ctx);
}

void sort_big_segments(rvp_context *ctx, const u64 *offsets, u64 *pairs, const u32 *big_list,
                       const u32 *big_count, u32 max_big) {
  static bool attr[64] = {false};
  if (ctx->device < 64 && !attr[ctx->device]) {
    RVP_CUDA_TRY(cudaFuncSetAttribute(k_sort_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      BIG_SMEM * 8));
    attr[ctx->device] = true;
  }
  const unsigned blocks = max_big < 1 ? 1 : (max_big < 4096 ? max_big : 4096);
  k_sort_big<<<blocks, 1024, BIG_SMEM * 8, ctx->stream>>>(offsets, pairs, big_list, big_count);
  RVP_LAUNCH_CHECK(ctx);
}

void grid_knn(rvp_context *ctx, const GridView &g, const QuerySet &q, int k, float radius,
              u64 *out_pairs, int32_t *out_counts, int qpw, int block_threads, u32 *stats,
              int out_mode, float *mean) {
  (void)qpw;
  const int bt = block_threads > 0 ? block_threads : 256;
  const unsigned blocks = grid_for(q.n_max * 32, bt, ctx->num_sms * 32);
  if (k <= 32)
    k_knn_warp<1><<<blocks, bt, 0, ctx->stream>>>(g, q, k, radius, out_pairs, out_counts, stats,
                                                  out_mode, mean);
  else
    k_knn_warp<2><<<blocks, bt, 0, ctx->stream>>>(g, q, k, radius, out_pairs, out_counts, stats,
                                                  out_mode, mean);
  RVP_LAUNCH_CHECK(ctx);
}

}  // namespace rvp
