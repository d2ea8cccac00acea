// Device-side helpers shared by the grid build and the neighbour-query
// kernels (grid.cu, knn_tile.cu): the reference's cell function, dense
// hierarchical keys, bucket-table lookup, query windows and their exact
// coverage bounds, and the warp-cooperative candidate walk.
//
// Dense keys are hierarchical: a level-L cell is 2 x 2 x 2 level-(L-1) cells
// (edge c * 2^L), and the 64-bit key of a fine cell is
//   key_base(frame) + (group cell, x fastest) << 18 + morton(cx, cy, cz),
// a group being 64 x 64 x 64 fine cells and morton the 18-bit interleave of
// the low 6 bits of the cell indices (bit 3i + a = bit i of axis a).
// Sorting by this key makes every cell of every level one contiguous run of
// points; level-L cells are entered in the bucket table under key >> 3L
// tagged with L in bits 60-63.
#pragma once

#include <math.h>

#include "internal.cuh"

namespace rvp {
namespace gd {

constexpr u32 kRemovedBit = 0x80000000u;

// getCellIndices (spatial_hashing.h:47-52)
__device__ __forceinline__ int cell_axis(float v, float mn, float cell) {
  return (int)floorf(fdiv(fsub(v, mn), cell));
}
// Same, saturated to [lo, hi] before the int conversion (window bounds).
__device__ __forceinline__ int cell_axis_clamped(float v, float mn, float cell, int lo, int hi) {
  float t = floorf(fdiv(fsub(v, mn), cell));
  t = fminf(fmaxf(t, (float)lo), (float)hi);
  return (int)t;
}

__device__ __forceinline__ int level_dim(int g, int level) {
  return (g + (1 << level) - 1) >> level;
}

// the low 6 bits of x, y, z interleaved (x in bits 0, 3, 6, ...)
__device__ __forceinline__ u32 spread3(u32 v) {
  v &= 63u;
  v = (v | (v << 8)) & 0x0300Fu;
  v = (v | (v << 4)) & 0x030C3u;
  v = (v | (v << 2)) & 0x09249u;
  return v;
}
__device__ __forceinline__ u64 morton18(int cx, int cy, int cz) {
  return (u64)(spread3((u32)cx) | (spread3((u32)cy) << 1) | (spread3((u32)cz) << 2));
}

__device__ __forceinline__ u64 dense_key(const GridFrame &F, int cx, int cy, int cz) {
  const u64 c3 = ((u64)(cz >> 6) * (u64)F.g3y + (u64)(cy >> 6)) * (u64)F.g3x + (u64)(cx >> 6);
  return F.key_base + (c3 << 18) + morton18(cx, cy, cz);
}

__device__ __forceinline__ u64 fine_key(const GridView &g, const GridFrame &F, int cx, int cy,
                                        int cz) {
  if (g.mode == KEY_REF_HASH) {
    const long long h = (long long)cx + (long long)cy * g.p1 + (long long)cz * g.p2;
    return (u64)h ^ 0x8000000000000000ull;
  }
  return dense_key(F, cx, cy, cz);
}

// table key of the level-L cell (X, Y, Z) (coordinates in level-L cells)
__device__ __forceinline__ u64 level_key(const GridView &g, const GridFrame &F, int level, int X,
                                         int Y, int Z) {
  if (level == 0) return fine_key(g, F, X, Y, Z);
  return ((u64)level << 60) | (dense_key(F, X << level, Y << level, Z << level) >> (3 * level));
}

struct Window {
  int lo[3], hi[3];  // cells, inclusive, at `level`
  int level;         // 0 fine; 1 .. kGridLevels - 1 coarser (dense mode only)
};

__device__ __forceinline__ bool lookup(const GridView &g, u64 key, u32 &start, u32 &count) {
  u64 slot = mix64(key) & g.table_mask;
  for (u64 probe = 0; probe <= g.table_mask; ++probe) {
    const ulonglong2 e = __ldg(&g.table[slot]);
    if (e.x == key) {
      start = (u32)(e.y & 0xFFFFFFFFull);
      count = (u32)(e.y >> 32);
      return true;
    }
    if (e.x == kEmptyKey) return false;
    slot = (slot + 1) & g.table_mask;
  }
  return false;
}

// Tight window of all cells that can hold a point p with d2(p, q) <= r*r:
// |p - q| <= r (1 + 3 * 2^-24) per axis for any such p; the bound is padded
// to r (1 + 1e-6) and rounded outwards, and the cell function is monotone,
// so the window is exact. Clamped to the frame's grid, then taken at `level`
// (fine index >> level).
__device__ __forceinline__ Window tight_window(const GridFrame &F, float qx, float qy, float qz,
                                               double r, int level = 0) {
  const double rp = r * (1.0 + 1e-6) + 1e-30;
  Window w;
  w.level = level;
  const float q[3] = {qx, qy, qz};
  const float mn[3] = {F.min_x, F.min_y, F.min_z};
  const int G[3] = {F.gx, F.gy, F.gz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float lo = __double2float_rd((double)q[a] - rp);
    const float hi = __double2float_ru((double)q[a] + rp);
    w.lo[a] = max(cell_axis_clamped(lo, mn[a], F.cell, -1, G[a]), 0);
    w.hi[a] = min(cell_axis_clamped(hi, mn[a], F.cell, -1, G[a]), G[a] - 1);
    if (level) {
      w.lo[a] >>= level;
      w.hi[a] = w.hi[a] < 0 ? -1 : (w.hi[a] >> level);
    }
  }
  return w;
}

// The reference's window: query cell +- (ceil(r/cell) + 1), unclamped
// (spatial_hashing.cpp:122-129).
__device__ __forceinline__ Window ref_window(const GridFrame &F, float qx, float qy, float qz,
                                             float radius) {
  const int R = (int)ceilf(fdiv(radius, F.cell)) + 1;
  Window w;
  w.level = 0;
  const int c[3] = {cell_axis(qx, F.min_x, F.cell), cell_axis(qy, F.min_y, F.cell),
                    cell_axis(qz, F.min_z, F.cell)};
#pragma unroll
  for (int a = 0; a < 3; ++a) { w.lo[a] = c[a] - R; w.hi[a] = c[a] + R; }
  return w;
}

// The query's own level-L cell +- ring, clamped.
__device__ __forceinline__ Window ring_window(const GridFrame &F, float qx, float qy, float qz,
                                              int ring, int level = 0) {
  Window w;
  w.level = level;
  const float q[3] = {qx, qy, qz};
  const float mn[3] = {F.min_x, F.min_y, F.min_z};
  const int G[3] = {F.gx, F.gy, F.gz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int c = cell_axis_clamped(q[a], mn[a], F.cell, 0, G[a] - 1) >> level;
    w.lo[a] = max(c - ring, 0);
    w.hi[a] = min(c + ring, level_dim(G[a], level) - 1);
  }
  return w;
}

// Lower bound on the distance from q to any point of the frame outside w;
// +inf when w spans the whole grid.
__device__ __forceinline__ double coverage(const GridFrame &F, const Window &w, float qx, float qy,
                                           float qz) {
  const float q[3] = {qx, qy, qz};
  const float mn[3] = {F.min_x, F.min_y, F.min_z};
  const int G[3] = {F.gx, F.gy, F.gz};
  const double cs = (double)F.cell * (double)(1 << w.level);
  double cov = 1e300;
  const double u = 4.0 * 5.960464477539063e-08;  // 4 * 2^-24
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double slack =
        u * (fabs((double)mn[a]) + (double)(w.hi[a] + 2) * cs + fabs((double)q[a])) + 1e-30;
    if (w.lo[a] > 0) {
      const double face = (double)mn[a] + (double)w.lo[a] * cs;
      cov = fmin(cov, (double)q[a] - face - slack);
    }
    if (w.hi[a] < level_dim(G[a], w.level) - 1) {
      const double face = (double)mn[a] + (double)(w.hi[a] + 1) * cs;
      cov = fmin(cov, face - (double)q[a] - slack);
    }
  }
  return cov;
}

// Lower bound on d2(p, q) for any point p of the level-L cell (ux, uy, uz):
// the gap from q to the cell's box, widened on each side by the rounding
// slack of the cell function and of the face positions, then shrunk by
// 1e-5 (the float arithmetic of the bound itself)
__device__ __forceinline__ float cell_lb2(const GridFrame &F, int level, int ux, int uy, int uz,
                                          float qx, float qy, float qz) {
  const float cs = F.cell * (float)(1 << level);
  const int u[3] = {ux, uy, uz};
  const float q[3] = {qx, qy, qz};
  const float mn[3] = {F.min_x, F.min_y, F.min_z};
  float s = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float lo = mn[a] + (float)u[a] * cs;
    const float sl = 4e-6f * (fabsf(mn[a]) + fabsf(q[a]) + (float)(abs(u[a]) + 2) * cs) + 1e-6f;
    const float gap = fmaxf(fmaxf(lo - sl - q[a], q[a] - (lo + cs + sl)), 0.0f);
    s += gap * gap;
  }
  return s * (1.0f - 1e-5f);
}

__device__ __forceinline__ long long window_cells(const Window &w) {
  long long c = 1;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (w.hi[a] < w.lo[a]) return 0;
    c *= (long long)(w.hi[a] - w.lo[a] + 1);
  }
  return c;
}

// Walk every candidate of window w (or of the whole frame when brute):
// fn(float4 p, bool valid) is called by all 32 lanes for each batch of 32.
// A cell is skipped when skip(cx, cy, cz) (cells of w's level) says so.
struct NoSkip {
  __device__ __forceinline__ bool operator()(int, int, int) const { return false; }
};
template <class Fn, class Skip = NoSkip>
__device__ __forceinline__ void for_each_candidate(const GridView &g, const GridFrame &F, int f,
                                                   const Window &w, bool brute, Fn &&fn,
                                                   Skip skip = Skip()) {
  const int lane = threadIdx.x & 31;
  if (brute) {
    const u64 a = g.frame_pt_begin[f], b = g.frame_pt_begin[f + 1];
    for (u64 p0 = a; p0 < b; p0 += 32) {
      const u64 p = p0 + lane;
      const bool valid = p < b;
      float4 v = valid ? __ldg(&g.pts[p]) : make_float4(0, 0, 0, 0);
      fn(v, valid);
    }
    return;
  }
  const long long total = window_cells(w);
  const int ncx = w.hi[0] - w.lo[0] + 1, ncy = w.hi[1] - w.lo[1] + 1;
  for (long long cb = 0; cb < total; cb += 32) {
    const long long j = cb + lane;
    u32 start = 0, count = 0;
    if (j < total) {
      const int cx = w.lo[0] + (int)(j % ncx);
      const int cy = w.lo[1] + (int)((j / ncx) % ncy);
      const int cz = w.lo[2] + (int)(j / ((long long)ncx * ncy));
      if (skip(cx, cy, cz) || !lookup(g, level_key(g, F, w.level, cx, cy, cz), start, count))
        count = 0;
    }
    // flatten: inclusive scan of bucket sizes
    u32 incl = count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    const u32 ex = incl - count;
    const u32 M = __shfl_sync(0xffffffffu, incl, 31);
    for (u32 p0 = 0; p0 < M; p0 += 32) {
      const u32 p = p0 + lane;
      // owner cell: largest lane c with ex_c <= p
      int c = 0;
#pragma unroll
      for (int s = 16; s; s >>= 1) {
        const u32 t = __shfl_sync(0xffffffffu, ex, c + s);
        if (t <= p) c += s;
      }
      const u32 st = __shfl_sync(0xffffffffu, start, c);
      const u32 ec = __shfl_sync(0xffffffffu, ex, c);
      const bool valid = p < M;
      float4 v = valid ? __ldg(&g.pts[st + (p - ec)]) : make_float4(0, 0, 0, 0);
      fn(v, valid);
    }
  }
}

__device__ __forceinline__ u32 query_index(const QuerySet &q, size_t i) {
  return q.order ? (u32)q.order[i] : (u32)i;
}

// ---------------------------------------------------------------------------
// exact kNN: warp-resident sorted list of 32*P keys (lane i, slot s holds
// element 32*s + i); candidates below the K-th key are inserted one by one.
// ---------------------------------------------------------------------------
template <int P>
struct WarpList {
  u64 e[P];
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int s = 0; s < P; ++s) e[s] = ~0ull;
  }
  __device__ __forceinline__ u64 get(int j) const {  // broadcast element j
    u64 v = e[0];
#pragma unroll
    for (int s = 1; s < P; ++s)
      if ((j >> 5) == s) v = e[s];
    return __shfl_sync(0xffffffffu, v, j & 31);
  }
  __device__ __forceinline__ void insert(u64 c) {
    const int lane = threadIdx.x & 31;
    u64 carry = 0;  // last element of the previous slot, before the insert
#pragma unroll
    for (int s = 0; s < P; ++s) {
      const u64 cur = e[s];
      const u64 last = __shfl_sync(0xffffffffu, cur, 31);
      u64 prev = __shfl_up_sync(0xffffffffu, cur, 1);
      bool prev_lt;
      if (lane == 0) prev_lt = (s == 0) ? true : (carry < c);
      else prev_lt = prev < c;
      if (lane == 0 && s > 0) prev = carry;
      if (!(cur < c)) e[s] = prev_lt ? c : prev;
      carry = last;
    }
  }
  // one key per lane (~0 for none) merged at once (32-slot lists): a
  // bitonic sort of the 32 keys, then the 32 smallest of both lists as a
  // bitonic sequence, sorted again
  __device__ __forceinline__ void merge_lanes(u64 key) {
    static_assert(P == 1, "batch merge is for 32-slot lists");
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        const u64 o = __shfl_xor_sync(0xffffffffu, key, j);
        const bool up = (lane & k) == 0, low = (lane & j) == 0;
        key = (low == up) ? (o < key ? o : key) : (o < key ? key : o);
      }
    }
    const u64 rev = __shfl_sync(0xffffffffu, key, 31 - lane);
    u64 v = e[0] < rev ? e[0] : rev;
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) {
      const u64 o = __shfl_xor_sync(0xffffffffu, v, j);
      v = (lane & j) == 0 ? (o < v ? o : v) : (o < v ? v : o);
    }
    e[0] = v;
  }
};

template <int P>
__device__ __forceinline__ void knn_scan(const GridView &g, const GridFrame &F, int f,
                                         const Window &w, bool brute, float qx, float qy,
                                         float qz, int K, u64 bound, WarpList<P> &L,
                                         u32 &found) {
  u64 thr = L.get(K - 1);
  // cells farther than the current K-th distance (or the bound) are skipped
  const float bd2 = nbr_d2(bound);
  auto skip = [&](int cx, int cy, int cz) {
    const float lim = fminf(nbr_d2(thr), bd2);  // NaN (unfilled list) never skips
    return cell_lb2(F, w.level, cx, cy, cz, qx, qy, qz) > lim;
  };
  for_each_candidate(g, F, f, w, brute, [&](float4 p, bool valid) {
    const u32 idx = __float_as_uint(p.w);
    u64 key = ~0ull;
    if (valid && !(idx & kRemovedBit)) key = pack_nbr(dist2(p.x, p.y, p.z, qx, qy, qz), (int)idx);
    const bool in_bound = key <= bound;
    found += __popc(__ballot_sync(0xffffffffu, in_bound));
    unsigned m = __ballot_sync(0xffffffffu, in_bound && key < thr);
    if constexpr (P == 1) {
      if (__popc(m) > 4) {  // many at once: one merge instead of serial inserts
        L.merge_lanes((m >> (threadIdx.x & 31)) & 1u ? key : ~0ull);
        thr = L.get(K - 1);
        m = 0;
      }
    }
    while (m) {
      const int src = __ffs(m) - 1;
      m &= m - 1;
      const u64 c = __shfl_sync(0xffffffffu, key, src);
      if (c < thr) {
        L.insert(c);
        thr = L.get(K - 1);
      }
    }
  }, skip);
}

}  // namespace gd
}  // namespace rvp
