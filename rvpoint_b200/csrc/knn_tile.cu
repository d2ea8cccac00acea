// Tile kNN for dense (batched) grids on sm_100a.
//
// Level by level (cells of c, 2c, 4c, ...): one thread block per bucket of
// the next level up (a group of 2 x 2 x 2 cells) looks up the 4 x 4 x 4
// cells around it once (one lookup per thread), flattens them with a prefix sum
// and stages their points in shared memory (coalesced float4 runs). Every
// open query of the group is then handled by one thread, which scans its own
// 27-cell ring out of shared memory and keeps a register-resident sorted
// top-K (unrolled insertion network; float keys when only distances matter,
// packed (d2, index) keys when ties must follow the reference's (d2, index)
// order). The ring certifies the result when the K-th distance is below the
// ring's coverage (distance to the nearest outside cell, with rounding
// slack); the others stay open for the next, 2x coarser level, and after the
// last level go to a list that the warp-per-query kernel finishes. Epilogues are fused: SOR mean distance
// (statistical_outlier_removal.cpp:36-40) or the reference normal
// (normal_estimation.cpp:90-110) straight from the registers.
#include <type_traits>

#include "grid_device.cuh"
#include "internal.cuh"
#include "normals_device.cuh"

namespace rvp {
using namespace gd;
using namespace nd;

namespace {
constexpr int TT = 256;                      // threads per tile block
constexpr int SIDE = 4;                      // staged cells per axis: a group and its halo
constexpr int NCELL = SIDE * SIDE * SIDE;    // 64
constexpr int CAP = 2560;                    // staged candidates (40 KB)

// the 27 ring cells, nearest first: own cell, 6 faces, 12 edges, 8 corners
__constant__ signed char kRingOrder[27][3] = {
    {0, 0, 0},   {-1, 0, 0},  {1, 0, 0},   {0, -1, 0},  {0, 1, 0},   {0, 0, -1},  {0, 0, 1},
    {-1, -1, 0}, {1, -1, 0},  {-1, 1, 0},  {1, 1, 0},   {-1, 0, -1}, {1, 0, -1},  {-1, 0, 1},
    {1, 0, 1},   {0, -1, -1}, {0, 1, -1},  {0, -1, 1},  {0, 1, 1},   {-1, -1, -1}, {1, -1, -1},
    {-1, 1, -1}, {1, 1, -1},  {-1, -1, 1}, {1, -1, 1},  {-1, 1, 1},  {1, 1, 1}};

template <class T, int K>
__device__ __forceinline__ void list_insert(T (&L)[K], T key) {
#pragma unroll
  for (int j = K - 1; j > 0; --j) {
    const T a = L[j - 1], b = L[j];
    L[j] = key < a ? a : (key < b ? key : b);
  }
  L[0] = key < L[0] ? key : L[0];
}

// SOR statistics of a certified list of packed keys: the mean distance to the
// k nearest other points (statistical_outlier_removal.cpp:36-40, ascending
// sum), and the k+1 indices for the normal stage
template <int K>
__device__ __forceinline__ void sor_list_out(const GridView &g, const TileArgs &a, u32 qidx,
                                             u64 qpos, const u64 (&L)[K]) {
  float sum = 0.0f;
#pragma unroll
  for (int j = 1; j < K; ++j) sum = fadd(sum, __fsqrt_rn(nbr_d2(L[j])));
  a.mean[qidx] = fdiv(sum, (float)(K - 1));
  u32 *row = a.sor_list + (size_t)qpos * K;
#pragma unroll
  for (int j = 0; j < K; ++j) row[j] = g.pos_of[(u32)nbr_idx(L[j]) & 0x7FFFFFFFu];
}

// the same network over float keys carrying an index beside each: a key
// goes after equal keys already in the list
template <int K>
__device__ __forceinline__ void list_insert_kv(float (&L)[K], u32 (&I)[K], float key, u32 idx) {
#pragma unroll
  for (int j = K - 1; j > 0; --j) {
    const bool a = key < L[j - 1], b = key < L[j];
    L[j] = a ? L[j - 1] : (b ? key : L[j]);
    I[j] = a ? I[j - 1] : (b ? idx : I[j]);
  }
  const bool b0 = key < L[0];
  I[0] = b0 ? idx : I[0];
  L[0] = b0 ? key : L[0];
}

template <int K, int MODE>
__global__ __launch_bounds__(TT, MODE == TILE_SOR_MEAN ? 4 : 3) void k_knn_tile(GridView g, TileArgs a, int level,
                                                 uint8_t *qlevel, float *qtau, u32 *stats) {
  using Key = typename std::conditional<MODE == TILE_SOR_MEAN, float, u64>::type;
  __shared__ u32 c_start[NCELL];
  __shared__ u32 c_count[NCELL];
  __shared__ u32 c_pref[NCELL + 1];
  __shared__ float4 cand[CAP];
  __shared__ int s_base[4];
  __shared__ int s_staged;
  __shared__ GridFrame s_F;
  // groups: the buckets one binary level up
  const u64 ngroups = g.n_level[level - g.lbase + 1];
  const u32 *gstart = g.lstart[level - g.lbase + 1];
  const u64 n = *g.n_points;
  const int tid = threadIdx.x;
  const int sh = level;  // level-L cell = fine index >> sh
  Key kMax;
  if constexpr (MODE == TILE_SOR_MEAN) kMax = INFINITY;
  else kMax = ~0ull;
  for (u64 cb = blockIdx.x; cb < ngroups; cb += gridDim.x) {
    const u32 qs = gstart[cb];
    const u32 qe = (cb + 1 < ngroups) ? gstart[cb + 1] : (u32)n;
    if (level > g.lbase) {  // only the queries the previous level left open
      int any = 0;
      for (u32 base = qs; base < qe; base += TT) {
        const u32 i = base + tid;
        any |= __syncthreads_or(i < qe && qlevel[i] == level);
      }
      if (!any) continue;
    }
    __syncthreads();  // the previous group's shared memory is free
    if (tid == 0) {
      const float4 p0 = g.pts[qs];
      const u32 i0 = __float_as_uint(p0.w) & 0x7FFFFFFFu;
      const int f = a.frame_of ? a.frame_of[i0] : 0;
      const GridFrame F = g.frames[f];
      const int gs = sh + 1;  // group cell = fine index >> gs
      s_base[0] = (cell_axis(p0.x, F.min_x, F.cell) >> gs) * 2 - 1;
      s_base[1] = (cell_axis(p0.y, F.min_y, F.cell) >> gs) * 2 - 1;
      s_base[2] = (cell_axis(p0.z, F.min_z, F.cell) >> gs) * 2 - 1;
      s_base[3] = f;
      s_F = F;
    }
    __syncthreads();
    const int bx = s_base[0], by = s_base[1], bz = s_base[2];
    const GridFrame &F = s_F;
    const int dx_ = level_dim(F.gx, level), dy_ = level_dim(F.gy, level),
              dz_ = level_dim(F.gz, level);
    // 1) the 4 x 4 x 4 level-L cells around the group
    for (int t = tid; t < NCELL; t += TT) {
      const int cx = bx + t % SIDE, cy = by + (t / SIDE) % SIDE, cz = bz + t / (SIDE * SIDE);
      u32 st = 0, ct = 0;
      if (cx >= 0 && cy >= 0 && cz >= 0 && cx < dx_ && cy < dy_ && cz < dz_)
        if (!lookup(g, level_key(g, F, level, cx, cy, cz), st, ct)) ct = 0;
      c_start[t] = st;
      c_count[t] = ct;
    }
    __syncthreads();
    // 2) exclusive prefix of the counts (one warp) and the staging decision
    if (tid < 32) {
      u32 run = 0;
      for (int base = 0; base < NCELL; base += 32) {
        const int t = base + tid;
        const u32 v = t < NCELL ? c_count[t] : 0;
        u32 incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const u32 u = __shfl_up_sync(0xffffffffu, incl, o);
          if (tid >= o) incl += u;
        }
        if (t < NCELL) c_pref[t] = run + incl - v;
        run += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (tid == 0) {
        c_pref[NCELL] = run;
        s_staged = run <= (u32)CAP ? 1 : 0;
      }
    }
    __syncthreads();
    const bool staged = s_staged != 0;
    if (staged) {
      const u32 total = c_pref[NCELL];
      for (u32 i = tid; i < total; i += TT) {
        int lo = 0, hi = NCELL - 1;  // owning cell: largest c with c_pref[c] <= i
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (c_pref[mid] <= i) lo = mid; else hi = mid - 1;
        }
        cand[i] = __ldg(&g.pts[c_start[lo] + (i - c_pref[lo])]);
      }
    }
    __syncthreads();
    // 3) one thread per open query of this group
    for (u32 qi = qs + tid; qi < qe; qi += TT) {
      if (level > g.lbase && qlevel[qi] != level) continue;
      const float4 q = g.pts[qi];
      const u32 qidx = __float_as_uint(q.w);
      if (MODE == TILE_NORMALS && (qidx & kRemovedBit)) continue;
      const int lx = (cell_axis(q.x, F.min_x, F.cell) >> sh) - bx;  // 1..2
      const int ly = (cell_axis(q.y, F.min_y, F.cell) >> sh) - by;
      const int lz = (cell_axis(q.z, F.min_z, F.cell) >> sh) - bz;
      Key L[K];
      Key thr = kMax;
      u32 found = 0;
      // distance from q to the faces of its own cell, shrunk by the rounding
      // slack of the cell function: a point of a neighbour cell lies at least
      // this far away along that axis (used to skip whole cells)
      float glx, ghx, gly, ghy, glz, ghz;
      {
        const float cs = F.cell * (float)(1 << sh);
        const float fx = F.min_x + (float)(lx + bx) * cs, fy = F.min_y + (float)(ly + by) * cs,
                    fz = F.min_z + (float)(lz + bz) * cs;
        const float slx = 4e-6f * (fabsf(F.min_x) + fabsf(q.x) + (float)(lx + bx + 2) * cs) + 1e-6f;
        const float sly = 4e-6f * (fabsf(F.min_y) + fabsf(q.y) + (float)(ly + by + 2) * cs) + 1e-6f;
        const float slz = 4e-6f * (fabsf(F.min_z) + fabsf(q.z) + (float)(lz + bz + 2) * cs) + 1e-6f;
        glx = fmaxf(q.x - fx - slx, 0.0f);
        ghx = fmaxf(fx + cs - q.x - slx, 0.0f);
        gly = fmaxf(q.y - fy - sly, 0.0f);
        ghy = fmaxf(fy + cs - q.y - sly, 0.0f);
        glz = fmaxf(q.z - fz - slz, 0.0f);
        ghz = fmaxf(fz + cs - q.z - slz, 0.0f);
      }
      // Scan the cells own +- [lo, hi] nearest first; with `bounded`, only
      // points with d2 <= tb count.
      auto scan = [&](int lox, int hix, int loy, int hiy, int loz, int hiz, bool bounded,
                      float tb) {
#pragma unroll
        for (int j = 0; j < K; ++j) L[j] = kMax;
        thr = kMax;
        found = 0;
        for (int t = 0; t < 27; ++t) {
          const int dx = kRingOrder[t][0], dy = kRingOrder[t][1], dz = kRingOrder[t][2];
          if (dx < lox || dx > hix || dy < loy || dy > hiy || dz < loz || dz > hiz) continue;
          if (t > 0) {
            // skip a cell that cannot hold anything below the current K-th
            // distance (nothing is skipped until the list is full)
            float thr_d2;
            if constexpr (MODE == TILE_SOR_MEAN) thr_d2 = thr;
            else thr_d2 = nbr_d2(thr);
            if (bounded) thr_d2 = fminf(thr_d2, tb);
            const float gx = dx < 0 ? glx : (dx > 0 ? ghx : 0.0f);
            const float gy = dy < 0 ? gly : (dy > 0 ? ghy : 0.0f);
            const float gz = dz < 0 ? glz : (dz > 0 ? ghz : 0.0f);
            if ((gx * gx + gy * gy + gz * gz) * (1.0f - 1e-5f) > thr_d2) continue;
            // (a bounded pass never needs a point beyond tb; fminf keeps NaN
            // from an unfilled u64 list out of the comparison)
          }
          const int c = ((lz + dz) * SIDE + (ly + dy)) * SIDE + (lx + dx);
          const u32 cnt = c_count[c];
          const u32 st = staged ? c_pref[c] : c_start[c];
          for (u32 j = 0; j < cnt; ++j) {
            const float4 p = staged ? cand[st + j] : __ldg(&g.pts[st + j]);
            const u32 pidx = __float_as_uint(p.w);
            if (MODE == TILE_NORMALS && (pidx & kRemovedBit)) continue;
            const float d2 = dist2(p.x, p.y, p.z, q.x, q.y, q.z);
            if (bounded && !(d2 <= tb)) continue;
            ++found;
            Key key;
            if constexpr (MODE == TILE_SOR_MEAN) key = d2;
            else key = pack_nbr(d2, (int)pidx);
            if (key < thr) {
              list_insert<Key, K>(L, key);
              thr = L[K - 1];
            }
          }
        }
      };
      // First pass, bounded: every point with d2 <= tb lies in the tight
      // window of sqrt(tb); if it holds >= K of them the answer is exact.
      // The bound is the level below's K-th distance (a query left open with
      // K points found), or at level 0 a radius estimated from the own
      // cell's occupancy (surface density), kept under one cell.
      float tb = -1.0f;
      if (level > g.lbase) {
        tb = qtau[qi];
      } else if (a.rfac > 0.0f) {
        const u32 n_own = c_count[(lz * SIDE + ly) * SIDE + lx];
        const float csb = F.cell * (float)(1 << sh);
        const float r = fminf(a.rfac * csb * sqrtf((float)K / (float)max(n_own, 1u)),
                              0.999f * csb);
        tb = r * r;
      }
      bool ok = false;
      if (tb >= 0.0f) {
        const Window wt = tight_window(F, q.x, q.y, q.z, sqrt((double)tb), level);
        const int ox = lx + bx, oy = ly + by, oz = lz + bz;
        const int lox = wt.lo[0] - ox, hix = wt.hi[0] - ox, loy = wt.lo[1] - oy,
                  hiy = wt.hi[1] - oy, loz = wt.lo[2] - oz, hiz = wt.hi[2] - oz;
        if (lox >= -1 && hix <= 1 && loy >= -1 && hiy <= 1 && loz >= -1 && hiz <= 1) {
          scan(lox, hix, loy, hiy, loz, hiz, true, tb);
          ok = found >= (u32)K;
        }
      }
      float tau = -1.0f;
      if (!ok) {
        // the ring: certified when the K-th distance is below its coverage
        scan(-1, 1, -1, 1, -1, 1, false, 0.0f);
        if (found >= (u32)K) {
          if constexpr (MODE == TILE_SOR_MEAN) tau = L[K - 1];
          else tau = nbr_d2(L[K - 1]);
          const Window w1 = ring_window(F, q.x, q.y, q.z, 1, level);
          const double cov = coverage(F, w1, q.x, q.y, q.z);
          ok = cov > 0.0 && (double)tau < cov * cov * (1.0 - 1e-5);
        }
      }
      if (!ok) {
        if (level + kChainStep < g.lbase + kChainStep * kChainLevels) {
          qlevel[qi] = (uint8_t)(level + kChainStep);
          qtau[qi] = tau;
        } else {
          const u32 slot = atomicAdd(a.hard_count, 1u);
          a.hard[slot] = qidx & 0x7FFFFFFFu;
          if (a.hard_tau) a.hard_tau[slot] = tau;
        }
        continue;
      }
      if (stats) atomicAdd(stats, 1u);
      if constexpr (MODE == TILE_SOR_MEAN) {
        float sum = 0.0f;
#pragma unroll
        for (int j = 1; j < K; ++j) sum = fadd(sum, __fsqrt_rn(L[j]));
        a.mean[qidx] = fdiv(sum, (float)(K - 1));
      } else if constexpr (MODE == TILE_SOR_LIST) {
        sor_list_out<K>(g, a, qidx, qi, L);
      } else if constexpr (MODE == TILE_NORMALS) {
        float nx, ny, nz;
        normal_from_keys<K>(a.vx, a.vy, a.vz, L, true, a.iters, q.x, q.y, q.z, a.vpx, a.vpy,
                            a.vpz, nx, ny, nz);
        const u64 o = a.out_pos[qidx];
        a.nx[o] = nx;
        a.ny[o] = ny;
        a.nz[o] = nz;
      } else {
#pragma unroll
        for (int j = 0; j < K; ++j) a.pairs[(size_t)qidx * K + j] = L[j];
        if (a.counts) a.counts[qidx] = K;
      }
    }
  }
}

// Per-warp kNN without block barriers, one level at a time. Each warp takes
// 32 consecutive queries in cell order -- at level 0 every grid point, at
// level L > 0 the compacted list of queries the level below left open --
// looks up the union of their 27-cell rings (level-L cells) once into a
// small per-warp table in shared memory (lanes in parallel), and every lane
// then walks its own ring, reading candidates through L1 (lanes of one cell
// read the same addresses). Warps never wait for each other, so one slow
// query only holds its own warp. A query open with a bound tau from the level
// below scans only the tight window of sqrt(tau) (exact with the bound); at
// level 0 a first pass uses a radius estimated from the own cell's
// occupancy. A ring that cannot certify the K-th distance leaves the query
// open for the next level, with tau when K points were found.
constexpr int WT_CELLS = 64;
constexpr int WT_WARPS = TT / 32;

template <int K, int MODE>
__global__ __launch_bounds__(TT, 3) void k_knn_wt(GridView g, TileArgs a, int level,
                                                  const u32 *list, const u64 *n_list,
                                                  uint8_t *qlevel, float *qtau, u32 *stats) {
  // float keys where only distances order the list (SOR); the list mode
  // carries indices beside them and detects ties (below)
  constexpr bool FKEY = MODE == TILE_SOR_MEAN || MODE == TILE_SOR_LIST || MODE == TILE_PAIRS_F;
  constexpr bool KV = MODE == TILE_SOR_LIST || MODE == TILE_PAIRS_F;  // indices beside
  using Key = typename std::conditional<FKEY, float, u64>::type;
  __shared__ uint2 wtab[WT_WARPS][WT_CELLS];
  const u64 n = list ? *n_list : *g.n_points;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const u64 nwarps = (u64)gridDim.x * WT_WARPS;
  const int sh = level;
  Key kMax;
  if constexpr (FKEY) kMax = INFINITY;
  else kMax = ~0ull;
  for (u64 base = ((u64)blockIdx.x * WT_WARPS + wib) * 32; base < n; base += nwarps * 32) {
    const bool active = base + lane < n;
    const u64 pos = active ? (list ? (u64)list[base + lane] : base + lane) : 0;
    const float4 q = active ? g.pts[pos] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const u32 qidx = __float_as_uint(q.w);
    const bool live = active && !(MODE == TILE_NORMALS && (qidx & kRemovedBit));
    const int f = active ? (a.frame_of ? a.frame_of[qidx & 0x7FFFFFFFu] : 0) : -1;
    const int f0 = __shfl_sync(0xffffffffu, f, 0);  // lane 0 is always active
    const bool one_frame = __all_sync(0xffffffffu, !active || f == f0);
    const GridFrame F = g.frames[active ? f : f0];
    const int GX = level_dim(F.gx, level), GY = level_dim(F.gy, level),
              GZ = level_dim(F.gz, level);
    const int cx = cell_axis(q.x, F.min_x, F.cell) >> sh,
              cy = cell_axis(q.y, F.min_y, F.cell) >> sh,
              cz = cell_axis(q.z, F.min_z, F.cell) >> sh;
    // union of the lanes' rings, clamped to the grid
    int bx0 = __reduce_min_sync(0xffffffffu, active ? cx : 0x7FFFFFFF) - 1;
    int by0 = __reduce_min_sync(0xffffffffu, active ? cy : 0x7FFFFFFF) - 1;
    int bz0 = __reduce_min_sync(0xffffffffu, active ? cz : 0x7FFFFFFF) - 1;
    int bx1 = __reduce_max_sync(0xffffffffu, active ? cx : (int)0x80000000) + 1;
    int by1 = __reduce_max_sync(0xffffffffu, active ? cy : (int)0x80000000) + 1;
    int bz1 = __reduce_max_sync(0xffffffffu, active ? cz : (int)0x80000000) + 1;
    bx0 = max(bx0, 0); by0 = max(by0, 0); bz0 = max(bz0, 0);
    bx1 = min(bx1, GX - 1); by1 = min(by1, GY - 1); bz1 = min(bz1, GZ - 1);
    const int wx = bx1 - bx0 + 1, wy = by1 - by0 + 1, wz = bz1 - bz0 + 1;
    const bool use_tab = one_frame && wx > 0 && wy > 0 && wz > 0 && wx * wy * wz <= WT_CELLS;
    if (use_tab) {
      for (int t = lane; t < wx * wy * wz; t += 32) {
        const int ux = bx0 + t % wx, uy = by0 + (t / wx) % wy, uz = bz0 + t / (wx * wy);
        u32 st = 0, ct = 0;
        if (!lookup(g, level_key(g, F, level, ux, uy, uz), st, ct)) ct = 0;
        wtab[wib][t] = make_uint2(st, ct);
      }
    }
    __syncwarp();
    if (live) {
      auto cell_run = [&](int ux, int uy, int uz, u32 &st, u32 &ct) {
        if (ux < 0 || uy < 0 || uz < 0 || ux >= GX || uy >= GY || uz >= GZ) {
          ct = 0;
          return;
        }
        if (use_tab) {
          const uint2 e = wtab[wib][((uz - bz0) * wy + (uy - by0)) * wx + (ux - bx0)];
          st = e.x;
          ct = e.y;
        } else if (!lookup(g, level_key(g, F, level, ux, uy, uz), st, ct)) {
          ct = 0;
        }
      };
      float glx, ghx, gly, ghy, glz, ghz;
      {
        const float cs = F.cell * (float)(1 << sh);
        const float fx = F.min_x + (float)cx * cs, fy = F.min_y + (float)cy * cs,
                    fz = F.min_z + (float)cz * cs;
        const float slx = 4e-6f * (fabsf(F.min_x) + fabsf(q.x) + (float)(cx + 2) * cs) + 1e-6f;
        const float sly = 4e-6f * (fabsf(F.min_y) + fabsf(q.y) + (float)(cy + 2) * cs) + 1e-6f;
        const float slz = 4e-6f * (fabsf(F.min_z) + fabsf(q.z) + (float)(cz + 2) * cs) + 1e-6f;
        glx = fmaxf(q.x - fx - slx, 0.0f);
        ghx = fmaxf(fx + cs - q.x - slx, 0.0f);
        gly = fmaxf(q.y - fy - sly, 0.0f);
        ghy = fmaxf(fy + cs - q.y - sly, 0.0f);
        glz = fmaxf(q.z - fz - slz, 0.0f);
        ghz = fmaxf(fz + cs - q.z - slz, 0.0f);
      }
      Key L[K];
      Key thr = kMax;
      u32 found = 0;
      // list mode: indices, and the value of the last tie met at the
      // boundary (an equal key rejected or evicted)
      u32 I[KV ? K : 1];
      float tie = -1.0f;
      auto scan = [&](int lox, int hix, int loy, int hiy, int loz, int hiz, bool bounded,
                      float tb) {
#pragma unroll
        for (int j = 0; j < K; ++j) L[j] = kMax;
        thr = kMax;
        found = 0;
        tie = -1.0f;
        for (int t = 0; t < 27; ++t) {
          const int dx = kRingOrder[t][0], dy = kRingOrder[t][1], dz = kRingOrder[t][2];
          if (dx < lox || dx > hix || dy < loy || dy > hiy || dz < loz || dz > hiz) continue;
          if (t > 0) {
            float thr_d2;
            if constexpr (FKEY) thr_d2 = thr;
            else thr_d2 = nbr_d2(thr);
            if (bounded) thr_d2 = fminf(thr_d2, tb);
            const float gx = dx < 0 ? glx : (dx > 0 ? ghx : 0.0f);
            const float gy = dy < 0 ? gly : (dy > 0 ? ghy : 0.0f);
            const float gz = dz < 0 ? glz : (dz > 0 ? ghz : 0.0f);
            if ((gx * gx + gy * gy + gz * gz) * (1.0f - 1e-5f) > thr_d2) continue;
          }
          u32 st, cnt;
          cell_run(cx + dx, cy + dy, cz + dz, st, cnt);
          for (u32 j = 0; j < cnt; ++j) {
            const float4 p = __ldg(&g.pts[st + j]);
            const u32 pidx = __float_as_uint(p.w);
            if (MODE == TILE_NORMALS && (pidx & kRemovedBit)) continue;
            const float d2 = dist2(p.x, p.y, p.z, q.x, q.y, q.z);
            if (bounded && !(d2 <= tb)) continue;
            ++found;
            Key key;
            if constexpr (FKEY) key = d2;
            else key = pack_nbr(d2, (int)pidx);
            if (key < thr) {
              if constexpr (KV) {
                // the SOR list keeps grid positions, the feature pairs indices
                list_insert_kv<K>(L, I, key, MODE == TILE_SOR_LIST ? st + j : pidx);
                if (L[K - 1] == thr) tie = thr;  // evicted a key equal to the boundary
              } else {
                list_insert<Key, K>(L, key);
              }
              thr = L[K - 1];
            } else if constexpr (KV) {
              if (key == thr) tie = key;
            }
          }
        }
      };
      // first pass with a bound: the level below's tau, or at level 0 a
      // radius from the own cell's occupancy (kept under one cell)
      float tb = -1.0f;
      if (level > g.lbase) {
        tb = qtau[pos];
      } else if (a.rfac > 0.0f) {
        u32 st0, n_own;
        cell_run(cx, cy, cz, st0, n_own);
        const float csb = F.cell * (float)(1 << sh);
        const float r = fminf(a.rfac * csb * sqrtf((float)K / (float)max(n_own, 1u)),
                              0.999f * csb);
        tb = r * r;
      }
      bool ok = false;
      if (tb >= 0.0f) {
        const Window wt = tight_window(F, q.x, q.y, q.z, sqrt((double)tb), level);
        const int lox = wt.lo[0] - cx, hix = wt.hi[0] - cx, loy = wt.lo[1] - cy,
                  hiy = wt.hi[1] - cy, loz = wt.lo[2] - cz, hiz = wt.hi[2] - cz;
        if (lox >= -1 && hix <= 1 && loy >= -1 && hiy <= 1 && loz >= -1 && hiz <= 1) {
          scan(lox, hix, loy, hiy, loz, hiz, true, tb);
          ok = found >= (u32)K;
        }
      }
      float tau = -1.0f;
      if (!ok) {
        scan(-1, 1, -1, 1, -1, 1, false, 0.0f);
        if (found >= (u32)K) {
          if constexpr (FKEY) tau = L[K - 1];
          else tau = nbr_d2(L[K - 1]);
          const Window w1 = ring_window(F, q.x, q.y, q.z, 1, level);
          const double cov = coverage(F, w1, q.x, q.y, q.z);
          ok = cov > 0.0 && (double)tau < cov * cov * (1.0 - 1e-5);
        }
      }
      if (!ok) {
        // a bound found at the next-to-top level goes straight to the warp
        // kernel, which scans the tight window of sqrt(tau) at the finest
        // level where it stays small; the top-level ring would hold far more
        // points than that window
        // lane_levels: the levels run by these per-lane kernels; past
        // them the warp kernel (lanes over candidates) takes the query
        const int nlev = a.lane_levels > 0 && a.lane_levels < kChainLevels ? a.lane_levels
                                                                            : kChainLevels;
        const int last = g.lbase + kChainStep * (nlev - 1);
        const bool to_warp = level + kChainStep == last && tau >= 0.0f && a.hard_tau;
        if (level < last && !to_warp) {
          qlevel[pos] = (uint8_t)(level + kChainStep);
          qtau[pos] = tau;
        } else {
          const u32 slot = atomicAdd(a.hard_count, 1u);
          a.hard[slot] = qidx & 0x7FFFFFFFu;
          if (a.hard_tau) a.hard_tau[slot] = tau;
        }
      } else {
        if (stats) atomicAdd(stats, 1u);
        if constexpr (MODE == TILE_SOR_MEAN) {
          float sum = 0.0f;
#pragma unroll
          for (int j = 1; j < K; ++j) sum = fadd(sum, __fsqrt_rn(L[j]));
          a.mean[qidx] = fdiv(sum, (float)(K - 1));
        } else if constexpr (MODE == TILE_SOR_LIST) {
          float sum = 0.0f;
#pragma unroll
          for (int j = 1; j < K; ++j) sum = fadd(sum, __fsqrt_rn(L[j]));
          a.mean[qidx] = fdiv(sum, (float)(K - 1));
          // equal distances leave the order (and at the boundary the set)
          // to the scan order instead of the index: such a list is marked
          // unusable and the normal stage searches that point again
          bool tied = tie == L[K - 1];
#pragma unroll
          for (int j = 1; j < K; ++j) tied = tied || L[j] == L[j - 1];
          u32 *row = a.sor_list + (size_t)pos * K;
#pragma unroll
          for (int j = 0; j < K; ++j) row[j] = tied ? 0xFFFFFFFFu : I[j];
        } else if constexpr (MODE == TILE_NORMALS) {
          float nx, ny, nz;
          normal_from_keys<K>(a.vx, a.vy, a.vz, L, true, a.iters, q.x, q.y, q.z, a.vpx, a.vpy,
                              a.vpz, nx, ny, nz);
          const u64 o = a.out_pos[qidx];
          a.nx[o] = nx;
          a.ny[o] = ny;
          a.nz[o] = nz;
        } else if constexpr (MODE == TILE_PAIRS_F) {
          bool tied = tie == L[K - 1];
#pragma unroll
          for (int j = 1; j < K; ++j) tied = tied || L[j] == L[j - 1];
          if (tied) {  // the exact (d2, index) list from the warp kernel
            const u32 slot = atomicAdd(a.hard_count, 1u);
            a.hard[slot] = qidx & 0x7FFFFFFFu;
            if (a.hard_tau) a.hard_tau[slot] = L[K - 1];
          } else {
#pragma unroll
            for (int j = 0; j < K; ++j) a.pairs[(size_t)qidx * K + j] = pack_nbr(L[j], (int)I[j]);
            if (a.counts) a.counts[qidx] = K;
          }
        } else {
#pragma unroll
          for (int j = 0; j < K; ++j) a.pairs[(size_t)qidx * K + j] = L[j];
          if (a.counts) a.counts[qidx] = K;
        }
      }
    }
    __syncwarp();  // the warp's table is reused by its next 32 queries
  }
}

// Cooperative kNN at the first chain level. Every grid point whose own cell
// holds at least `min_own` points is picked (k_knn_route): in such dense
// cells a radius from the occupancy is likely to hold K points inside the
// cell's 27-cell ring. One warp takes 32 consecutive picked queries (a
// compacted list in grid order, so they lie close together), looks up the
// union of their rings once (per-warp table, as in k_knn_wt), and every lane
// takes the bound tb = r^2 with r = rfac * cell * sqrt(K / own-cell count),
// under one cell. The warp walks only the cells some lane can use (box
// distance below that lane's bound): 32 candidates of such a cell go up
// coalesced into a per-warp staging row and every lane tests all of them
// against its query, four at a time (broadcast shared-memory reads, all
// lanes converged, four independent distance chains). A candidate within
// the lane's bound goes, as (d2, grid position), into the lane's buffer in
// shared memory. Every point with d2 <= tb lies in the lane's tight window
// of sqrt(tb), inside its ring, and every cell that can hold one is walked,
// so a lane that found K such points is exact.
//   Selection (float-key SOR modes): at the end the buffer goes through the
// float insertion network once (sorted K smallest distances: the mean), and
// the list row takes the positions of the buffered candidates within the
// K-th distance, each at its rank among those distances; equal distances
// leave the order (or at the boundary the set) to the scan order, and the
// row is marked unusable. A buffer about to overflow is cut to its K smallest (and their
// equals), which then gate what the buffer takes (anything farther cannot be
// among the K nearest); a lane whose cut cannot free room (many equal
// distances) gives up and stays open. Feature pairs (TILE_PAIRS_F) need the
// (d2, index) order: their buffer is merged into a register list with
// indices beside (insertion network) whenever it fills, and at the end.
// The queries that stay open (and warps whose queries span more than the
// table) go to the per-lane kernels, like the queries that were not picked.
constexpr int CP_WARPS = TT / 32;
constexpr int CP_BUF = 48;  // buffered (d2, position) candidates per lane
constexpr int CP_ILP = 4;   // candidates tested together
constexpr size_t CP_SMEM = (size_t)CP_WARPS * (WT_CELLS * sizeof(uint2) + 32 * sizeof(float4) +
                                               CP_BUF * 32 * sizeof(uint2));

template <int K, int MODE>
__global__ __launch_bounds__(TT, 2) void k_knn_coop(GridView g, TileArgs a, int level,
                                                    const u32 *list, const u64 *n_list,
                                                    uint8_t *qlevel, float *qtau, u32 *stats) {
  static_assert(MODE == TILE_SOR_MEAN || MODE == TILE_SOR_LIST || MODE == TILE_PAIRS_F,
                "float-key modes only");
  static_assert(K + CP_ILP <= CP_BUF, "the buffer must hold K candidates and a test group");
  constexpr bool PAIRS = MODE == TILE_PAIRS_F;
  extern __shared__ __align__(16) unsigned char cp_smem[];
  uint2 (*wtab)[WT_CELLS] = reinterpret_cast<uint2 (*)[WT_CELLS]>(cp_smem);
  float4 (*stage)[32] =
      reinterpret_cast<float4 (*)[32]>(cp_smem + CP_WARPS * WT_CELLS * sizeof(uint2));
  uint2 (*sbuf)[CP_BUF][32] = reinterpret_cast<uint2 (*)[CP_BUF][32]>(
      cp_smem + CP_WARPS * (WT_CELLS * sizeof(uint2) + 32 * sizeof(float4)));
  const u64 n = *n_list;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const u64 nwarps = (u64)gridDim.x * CP_WARPS;
  const int sh = level;
  // quarter-cell directories (the cells are of 4 x 4 x 4 fine cells)
  const bool use_dir = g.sub_off != nullptr && level == 2;
  // sub_mask[a][m]: the quarter cells of a cell (bits by Morton code) whose
  // coordinate along axis a is in the 4-bit value set m
  __shared__ u64 sub_mask[3][16];
  if (threadIdx.x < 48) {
    const int ax = threadIdx.x / 16, m = threadIdx.x % 16;
    u64 bits = 0;
    for (int c = 0; c < 64; ++c) {
      const int v = ((c >> ax) & 1) | (((c >> (ax + 3)) & 1) << 1);
      if ((m >> v) & 1) bits |= 1ull << c;
    }
    sub_mask[ax][m] = bits;
  }
  __syncthreads();
  for (u64 base = ((u64)blockIdx.x * CP_WARPS + wib) * 32; base < n; base += nwarps * 32) {
    const bool active = base + lane < n;
    const u64 pos = active ? (u64)list[base + lane] : 0;
    const float4 q = active ? g.pts[pos] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const u32 qidx = __float_as_uint(q.w);
    const int f = active ? (a.frame_of ? a.frame_of[qidx & 0x7FFFFFFFu] : 0) : -1;
    const int f0 = __shfl_sync(0xffffffffu, f, 0);  // lane 0 is always active
    const bool one_frame = __all_sync(0xffffffffu, !active || f == f0);
    const GridFrame F = g.frames[active ? f : f0];
    const int GX = level_dim(F.gx, level), GY = level_dim(F.gy, level),
              GZ = level_dim(F.gz, level);
    const int cx = cell_axis(q.x, F.min_x, F.cell) >> sh,
              cy = cell_axis(q.y, F.min_y, F.cell) >> sh,
              cz = cell_axis(q.z, F.min_z, F.cell) >> sh;
    int bx0 = __reduce_min_sync(0xffffffffu, active ? cx : 0x7FFFFFFF) - 1;
    int by0 = __reduce_min_sync(0xffffffffu, active ? cy : 0x7FFFFFFF) - 1;
    int bz0 = __reduce_min_sync(0xffffffffu, active ? cz : 0x7FFFFFFF) - 1;
    int bx1 = __reduce_max_sync(0xffffffffu, active ? cx : (int)0x80000000) + 1;
    int by1 = __reduce_max_sync(0xffffffffu, active ? cy : (int)0x80000000) + 1;
    int bz1 = __reduce_max_sync(0xffffffffu, active ? cz : (int)0x80000000) + 1;
    bx0 = max(bx0, 0); by0 = max(by0, 0); bz0 = max(bz0, 0);
    bx1 = min(bx1, GX - 1); by1 = min(by1, GY - 1); bz1 = min(bz1, GZ - 1);
    const int wx = bx1 - bx0 + 1, wy = by1 - by0 + 1, wz = bz1 - bz0 + 1;
    const bool use_tab = one_frame && wx > 0 && wy > 0 && wz > 0 && wx * wy * wz <= WT_CELLS;
    // a query this pass cannot finish: open at this level for the
    // per-lane kernels' ring
    auto leave_open = [&]() { qlevel[pos] = (uint8_t)level; };
    if (!use_tab) {
      if (active) leave_open();
      continue;
    }
    const int ncells = wx * wy * wz;
    for (int t = lane; t < ncells; t += 32) {
      const int ux = bx0 + t % wx, uy = by0 + (t / wx) % wy, uz = bz0 + t / (wx * wy);
      u32 st = 0, ct = 0;
      if (!lookup(g, level_key(g, F, level, ux, uy, uz), st, ct)) ct = 0;
      wtab[wib][t] = make_uint2(st, ct);
    }
    __syncwarp();
    // the lane's bound and the distances from q to its own cell's faces
    // (shrunk by the cell function's rounding slack)
    const float cs = F.cell * (float)(1 << sh);
    float tb = -1.0f;
    float glx = 0.0f, ghx = 0.0f, gly = 0.0f, ghy = 0.0f, glz = 0.0f, ghz = 0.0f;
    Window wq;  // the lane's tight window of sqrt(tb) in fine (quarter) cells
    wq.lo[0] = wq.lo[1] = wq.lo[2] = 1;
    wq.hi[0] = wq.hi[1] = wq.hi[2] = 0;
    if (active) {
      const u32 n_own = wtab[wib][((cz - bz0) * wy + (cy - by0)) * wx + (cx - bx0)].y;
      const float r = fminf(a.rfac * cs * sqrtf((float)K / (float)max(n_own, 1u)), 0.999f * cs);
      const Window wt = tight_window(F, q.x, q.y, q.z, sqrt((double)(r * r)), level);
      if (wt.lo[0] >= cx - 1 && wt.hi[0] <= cx + 1 && wt.lo[1] >= cy - 1 &&
          wt.hi[1] <= cy + 1 && wt.lo[2] >= cz - 1 && wt.hi[2] <= cz + 1) {
        tb = r * r;
        if (use_dir) wq = tight_window(F, q.x, q.y, q.z, sqrt((double)(r * r)), 0);
      }
      const float fx = F.min_x + (float)cx * cs, fy = F.min_y + (float)cy * cs,
                  fz = F.min_z + (float)cz * cs;
      const float slx = 4e-6f * (fabsf(F.min_x) + fabsf(q.x) + (float)(cx + 2) * cs) + 1e-6f;
      const float sly = 4e-6f * (fabsf(F.min_y) + fabsf(q.y) + (float)(cy + 2) * cs) + 1e-6f;
      const float slz = 4e-6f * (fabsf(F.min_z) + fabsf(q.z) + (float)(cz + 2) * cs) + 1e-6f;
      glx = fmaxf(q.x - fx - slx, 0.0f);
      ghx = fmaxf(fx + cs - q.x - slx, 0.0f);
      gly = fmaxf(q.y - fy - sly, 0.0f);
      ghy = fmaxf(fy + cs - q.y - sly, 0.0f);
      glz = fmaxf(q.z - fz - slz, 0.0f);
      ghz = fmaxf(fz + cs - q.z - slz, 0.0f);
    }
    float L[K];
    u32 I[PAIRS ? K : 1];
#pragma unroll
    for (int j = 0; j < K; ++j) L[j] = INFINITY;
    float thr = INFINITY;  // PAIRS: the register list's K-th key
    float tie = -1.0f;
    float gate = tb;       // what the buffer takes: d2 <= gate
    bool seen_k = false;   // K candidates within tb were met (the buffer was cut)
    int cnt = 0;           // buffered candidates of this lane
    // PAIRS: merge the buffer into the register list, in buffer order
    auto merge_pairs = [&]() {
      for (int i = 0; __any_sync(0xffffffffu, i < cnt); ++i) {
        if (i < cnt) {
          const uint2 b = sbuf[wib][i][lane];
          const float key = __uint_as_float(b.x);
          if constexpr (PAIRS) {
            if (key < thr) {
              list_insert_kv<K>(L, I, key, b.y);
              if (L[K - 1] == thr) tie = thr;  // evicted a key equal to the boundary
              thr = L[K - 1];
            } else if (key == thr) {
              tie = key;
            }
          }
        }
      }
      cnt = 0;
    };
    // SOR modes: the K smallest buffered distances, sorted (float network)
    auto select_k = [&]() {
#pragma unroll
      for (int j = 0; j < K; ++j) L[j] = INFINITY;
      for (int i = 0; __any_sync(0xffffffffu, i < cnt); ++i) {
        if (i < cnt) {
          const float key = __uint_as_float(sbuf[wib][i][lane].x);
          if (key < L[K - 1]) list_insert<float, K>(L, key);
        }
      }
    };
    // SOR modes, a full buffer: keep its K smallest and their equals
    auto cut = [&]() {
      const bool full = cnt > CP_BUF - CP_ILP;
      const int keep_cnt = cnt;
      if (!full) cnt = 0;  // only the full lanes select
      select_k();
      cnt = keep_cnt;
      if (full) {
        const float t = L[K - 1];
        int m = 0;
        for (int i = 0; i < cnt; ++i) {
          const uint2 b = sbuf[wib][i][lane];
          if (__uint_as_float(b.x) <= t) sbuf[wib][m++][lane] = b;
        }
        seen_k = true;
        cnt = m;
        if (m > CP_BUF - CP_ILP) {  // no room freed: give up (stays open)
          gate = -1.0f;
          cnt = 0;
        } else {
          gate = t;
        }
      }
    };
    // test the staged row (m candidates: x, y, z and the grid position in
    // w; padded to a multiple of CP_ILP with infinitely far points) against
    // the lane's limit and buffer the hits
    auto test_row = [&](u32 m, bool need) {
      const u32 mp = (m + CP_ILP - 1) & ~(u32)(CP_ILP - 1);
      for (u32 s2 = 0; s2 < mp; s2 += CP_ILP) {
        // the lane's limit now (the cut and, for pairs, the merge lower it)
        const float lim = need ? (PAIRS ? fminf(gate, thr) : gate) : -1.0f;
        float d[CP_ILP];
        u32 ps[CP_ILP];
#pragma unroll
        for (int u = 0; u < CP_ILP; ++u) {
          const float4 p = stage[wib][s2 + u];
          d[u] = dist2(p.x, p.y, p.z, q.x, q.y, q.z);
          ps[u] = __float_as_uint(p.w);
        }
#pragma unroll
        for (int u = 0; u < CP_ILP; ++u)
          if (d[u] <= lim) sbuf[wib][cnt++][lane] = make_uint2(__float_as_uint(d[u]), ps[u]);
        if (__any_sync(0xffffffffu, cnt > CP_BUF - CP_ILP)) {
          if constexpr (PAIRS) merge_pairs();
          else cut();
        }
      }
    };
    const float4 far4 = make_float4(INFINITY, INFINITY, INFINITY, 0.0f);
    for (int t = 0; t < ncells; ++t) {
      const uint2 e = wtab[wib][t];
      if (e.y == 0) continue;
      const int ux = bx0 + t % wx, uy = by0 + (t / wx) % wy, uz = bz0 + t / (wx * wy);
      // lower bound on the distance from q to the cell (whole cells between
      // q's cell and it add their edge)
      const int dx = ux - cx, dy = uy - cy, dz = uz - cz;
      const float gx = dx < 0 ? glx + (float)(-dx - 1) * cs : (dx > 0 ? ghx + (float)(dx - 1) * cs : 0.0f);
      const float gy = dy < 0 ? gly + (float)(-dy - 1) * cs : (dy > 0 ? ghy + (float)(dy - 1) * cs : 0.0f);
      const float gz = dz < 0 ? glz + (float)(-dz - 1) * cs : (dz > 0 ? ghz + (float)(dz - 1) * cs : 0.0f);
      const float lim0 = PAIRS ? fminf(gate, thr) : gate;
      const bool need = lim0 >= 0.0f && (gx * gx + gy * gy + gz * gz) * (1.0f - 1e-5f) <= lim0;
      if (!__any_sync(0xffffffffu, need)) continue;
      if (use_dir && e.y >= kSubMin && e.y <= kSubMax) {
        // only the quarter cells inside some needing lane's window: the
        // union of the lanes' boxes of quarter cells, as a 64-bit mask by
        // Morton code
        u64 mk = 0;
        if (need) {
          const int u0[3] = {ux << 2, uy << 2, uz << 2};
          mk = ~0ull;
#pragma unroll
          for (int ax = 0; ax < 3; ++ax) {
            const int lo = max(wq.lo[ax] - u0[ax], 0), hi = min(wq.hi[ax] - u0[ax], 3);
            const int vm = lo <= hi ? (((2 << hi) - 1) & ~((1 << lo) - 1)) : 0;
            mk &= sub_mask[ax][vm];
          }
        }
        const u64 mask = (u64)__reduce_or_sync(0xffffffffu, (u32)mk) |
                         ((u64)__reduce_or_sync(0xffffffffu, (u32)(mk >> 32)) << 32);
        // lane l: quarter cells 2l and 2l + 1 (offsets d0, d1; the next
        // lane's d0 ends the second)
        const uint16_t *dir = g.sub_off + e.x;
        const u32 d0 = dir[2 * lane], d1 = dir[2 * lane + 1];
        u32 e1 = __shfl_down_sync(0xffffffffu, d0, 1);
        if (lane == 31) e1 = e.y;
        const u32 c0 = (mask >> (2 * lane)) & 1 ? d1 - d0 : 0;
        const u32 c1 = (mask >> (2 * lane + 1)) & 1 ? e1 - d1 : 0;
        u32 incl = c0 + c1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const u32 v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        const u32 ex = incl - c0 - c1;
        const u32 M = __shfl_sync(0xffffffffu, incl, 31);
        for (u32 p0 = 0; p0 < M; p0 += 32) {
          const u32 p = p0 + (u32)lane;
          // the owning lane: the last with ex <= p
          int o = 0;
#pragma unroll
          for (int st2 = 16; st2; st2 >>= 1) {
            const u32 v = __shfl_sync(0xffffffffu, ex, o + st2);
            if (v <= p) o += st2;
          }
          const u32 r = p - __shfl_sync(0xffffffffu, ex, o);
          const u32 c0o = __shfl_sync(0xffffffffu, c0, o);
          const u32 d0o = __shfl_sync(0xffffffffu, d0, o);
          const u32 d1o = __shfl_sync(0xffffffffu, d1, o);
          const u32 m = min(32u, M - p0);
          if ((u32)lane < m) {
            const u32 cp = e.x + (r < c0o ? d0o + r : d1o + (r - c0o));
            const float4 v = __ldg(&g.pts[cp]);
            stage[wib][lane] = make_float4(v.x, v.y, v.z, __uint_as_float(cp));
          } else {
            stage[wib][lane] = far4;
          }
          __syncwarp();
          test_row(m, need);
          __syncwarp();  // the staging row is refilled next
        }
      } else {
        for (u32 j0 = 0; j0 < e.y; j0 += 32) {
          const u32 m = min(32u, e.y - j0);
          if ((u32)lane < m) {
            const u32 cp = e.x + j0 + lane;
            const float4 v = __ldg(&g.pts[cp]);
            stage[wib][lane] = make_float4(v.x, v.y, v.z, __uint_as_float(cp));
          } else {
            stage[wib][lane] = far4;
          }
          __syncwarp();
          test_row(m, need);
          __syncwarp();  // the staging row is refilled next
        }
      }
    }
    // the K nearest from what is buffered
    bool found_k;
    if constexpr (PAIRS) {
      // (every candidate within tb went into the buffer: the merged count
      // plus the rest decides)
      merge_pairs();
      found_k = thr < INFINITY;
    } else {
      select_k();
      found_k = gate >= 0.0f && (seen_k || cnt >= K);
    }
    if (active) {
      if (!found_k) {
        leave_open();
      } else {
        qlevel[pos] = 0xFF;
        if (stats) atomicAdd(stats, 1u);
        float sum = 0.0f;
#pragma unroll
        for (int j = 1; j < K; ++j) sum = fadd(sum, __fsqrt_rn(L[j]));
        if constexpr (!PAIRS) a.mean[qidx] = fdiv(sum, (float)(K - 1));
        if constexpr (MODE == TILE_SOR_LIST) {
          // each buffered position within the K-th distance goes to its
          // rank in the sorted distances (the number below its own). Equal
          // distances (ranks that collide, or more than K within the K-th
          // distance) leave the order, or at the boundary the set, to the
          // scan order instead of the index: the row is marked unusable and
          // the normal stage searches that point again
          const float t = L[K - 1];
          u32 *row = a.sor_list + (size_t)pos * K;
          int m = 0;
          for (int i = 0; i < cnt; ++i) {
            const uint2 b = sbuf[wib][i][lane];
            const float d = __uint_as_float(b.x);
            if (d <= t) {
              int r = 0;
#pragma unroll
              for (int j = 0; j < K; ++j) r += L[j] < d ? 1 : 0;
              if (r < K) row[r] = b.y;
              ++m;
            }
          }
          bool tied = m != K;
#pragma unroll
          for (int j = 1; j < K; ++j) tied = tied || L[j] == L[j - 1];
          if (tied)
            for (int j = 0; j < K; ++j) row[j] = 0xFFFFFFFFu;
        } else if constexpr (PAIRS) {
          // equal distances leave the order (and at the boundary the set) to
          // the scan order instead of the index: marked for the exact search
          bool tied = tie == L[K - 1];
#pragma unroll
          for (int j = 1; j < K; ++j) tied = tied || L[j] == L[j - 1];
          if (tied) {
            const u32 slot = atomicAdd(a.hard_count, 1u);
            a.hard[slot] = qidx & 0x7FFFFFFFu;
            if (a.hard_tau) a.hard_tau[slot] = L[K - 1];
          } else {
#pragma unroll
            for (int j = 0; j < K; ++j)
              a.pairs[(size_t)qidx * K + j] = pack_nbr(L[j], (int)__float_as_uint(g.pts[I[j]].w));
            if (a.counts) a.counts[qidx] = K;
          }
        }
      }
    }
    __syncwarp();  // the warp's table and buffers are reused by its next 32 queries
  }
}

// Queries the per-lane chain handed on with a bound tau (the K-th distance
// found in a ring that could not certify it): every point with d2 <= tau
// lies in the tight window of sqrt(tau), and at least K of them do, so a
// scan of that window bounded by tau is exact. One thread per hard slot
// scans the window at the finest table level where it spans at most
// kTauCells cells (its own lookups: the lanes of a warp sit at different
// levels and places), skipping cells farther than min(tau, K-th key), when
// the cells within tau hold at most kTauPoints points. Done slots get tau =
// kTauDone, which the warp-per-query kernel skips; slots without a bound,
// with more candidates, and feature lists with tied distances stay for it.
//   TILE_SOR_MEAN / TILE_SOR_LIST: the mean (and the row of grid positions)
//   TILE_NORMALS: the (d2, index) list by slot (slot_pairs, slot_counts),
//                 as the warp kernel's KNN_OUT_BY_SLOT writes it
//   TILE_PAIRS / TILE_PAIRS_F: the list by original index (a.pairs, a.counts)
constexpr int kTauCells = 64;     // window cells one thread looks up
constexpr u32 kTauPoints = 512;   // candidates one thread scans

template <int K, int MODE>
__global__ __launch_bounds__(TT, 3) void k_knn_tau(GridView g, TileArgs a, const u64 *n_hard,
                                                   u64 *slot_pairs, int32_t *slot_counts,
                                                   u32 *stats) {
  constexpr bool FKEY = MODE == TILE_SOR_MEAN || MODE == TILE_SOR_LIST || MODE == TILE_PAIRS_F;
  constexpr bool KV = MODE == TILE_SOR_LIST || MODE == TILE_PAIRS_F;
  using Key = typename std::conditional<FKEY, float, u64>::type;
  const u64 n = *n_hard;
  for (u64 s = blockIdx.x * (u64)blockDim.x + threadIdx.x; s < n;
       s += (u64)gridDim.x * blockDim.x) {
    const float tau = a.hard_tau[s];
    if (!(tau >= 0.0f)) continue;
    const u32 qi = a.hard[s];
    const u32 pos = g.pos_of[qi];
    const float4 q = g.pts[pos];
    const GridFrame F = g.frames[a.frame_of ? a.frame_of[qi] : 0];
    const double rt = sqrt((double)tau);
    Window w;
    int level = -1;
    for (int L = g.lbase; L < g.lbase + kGridLevels; ++L) {
      w = tight_window(F, q.x, q.y, q.z, rt, L);
      if (window_cells(w) <= kTauCells) {
        level = L;
        break;
      }
    }
    if (level < 0) continue;
    // the points in cells within tau: past kTauPoints the warp kernel (lanes
    // over candidates) is faster than one thread
    {
      u32 total = 0;
      for (int uz = w.lo[2]; uz <= w.hi[2]; ++uz)
        for (int uy = w.lo[1]; uy <= w.hi[1]; ++uy)
          for (int ux = w.lo[0]; ux <= w.hi[0]; ++ux) {
            u32 st, cnt;
            if (cell_lb2(F, level, ux, uy, uz, q.x, q.y, q.z) <= tau &&
                lookup(g, level_key(g, F, level, ux, uy, uz), st, cnt))
              total += cnt;
          }
      if (total > kTauPoints) continue;
    }
    const int sh = level;
    const float cs = F.cell * (float)(1 << sh);
    const int cx = cell_axis(q.x, F.min_x, F.cell) >> sh, cy = cell_axis(q.y, F.min_y, F.cell) >> sh,
              cz = cell_axis(q.z, F.min_z, F.cell) >> sh;
    // distances from q to its own cell's faces, shrunk by the cell
    // function's rounding slack
    float glx, ghx, gly, ghy, glz, ghz;
    {
      const float fx = F.min_x + (float)cx * cs, fy = F.min_y + (float)cy * cs,
                  fz = F.min_z + (float)cz * cs;
      const float slx = 4e-6f * (fabsf(F.min_x) + fabsf(q.x) + (float)(cx + 2) * cs) + 1e-6f;
      const float sly = 4e-6f * (fabsf(F.min_y) + fabsf(q.y) + (float)(cy + 2) * cs) + 1e-6f;
      const float slz = 4e-6f * (fabsf(F.min_z) + fabsf(q.z) + (float)(cz + 2) * cs) + 1e-6f;
      glx = fmaxf(q.x - fx - slx, 0.0f);
      ghx = fmaxf(fx + cs - q.x - slx, 0.0f);
      gly = fmaxf(q.y - fy - sly, 0.0f);
      ghy = fmaxf(fy + cs - q.y - sly, 0.0f);
      glz = fmaxf(q.z - fz - slz, 0.0f);
      ghz = fmaxf(fz + cs - q.z - slz, 0.0f);
    }
    Key kMax;
    if constexpr (FKEY) kMax = INFINITY;
    else kMax = ~0ull;
    Key L[K];
#pragma unroll
    for (int j = 0; j < K; ++j) L[j] = kMax;
    u32 I[KV ? K : 1];
    Key thr = kMax;
    float tie = -1.0f;
    u32 found = 0;
    for (int uz = w.lo[2]; uz <= w.hi[2]; ++uz)
      for (int uy = w.lo[1]; uy <= w.hi[1]; ++uy)
        for (int ux = w.lo[0]; ux <= w.hi[0]; ++ux) {
          // lower bound on the distance from q to the cell (whole cells
          // between q's cell and it add their edge)
          const int dx = ux - cx, dy = uy - cy, dz = uz - cz;
          const float gx = dx < 0 ? glx + (float)(-dx - 1) * cs : (dx > 0 ? ghx + (float)(dx - 1) * cs : 0.0f);
          const float gy = dy < 0 ? gly + (float)(-dy - 1) * cs : (dy > 0 ? ghy + (float)(dy - 1) * cs : 0.0f);
          const float gz = dz < 0 ? glz + (float)(-dz - 1) * cs : (dz > 0 ? ghz + (float)(dz - 1) * cs : 0.0f);
          float thr_d2;
          if constexpr (FKEY) thr_d2 = thr;
          else thr_d2 = nbr_d2(thr);
          if ((gx * gx + gy * gy + gz * gz) * (1.0f - 1e-5f) > fminf(thr_d2, tau)) continue;
          u32 st, cnt;
          if (!lookup(g, level_key(g, F, level, ux, uy, uz), st, cnt)) continue;
          for (u32 j = 0; j < cnt; ++j) {
            const float4 p = __ldg(&g.pts[st + j]);
            const u32 pidx = __float_as_uint(p.w);
            if (MODE == TILE_NORMALS && (pidx & kRemovedBit)) continue;
            const float d2 = dist2(p.x, p.y, p.z, q.x, q.y, q.z);
            if (!(d2 <= tau)) continue;
            ++found;
            Key key;
            if constexpr (FKEY) key = d2;
            else key = pack_nbr(d2, (int)pidx);
            if (key < thr) {
              if constexpr (KV) {
                list_insert_kv<K>(L, I, key, MODE == TILE_SOR_LIST ? st + j : pidx);
                if (L[K - 1] == thr) tie = thr;  // evicted a key equal to the boundary
              } else {
                list_insert<Key, K>(L, key);
              }
              thr = L[K - 1];
            } else if constexpr (KV) {
              if (key == thr) tie = key;
            }
          }
        }
    if (found < (u32)K) continue;  // not reached with a true bound; the warp kernel decides
    bool tied = false;
    if constexpr (KV) {
      tied = tie == L[K - 1];
#pragma unroll
      for (int j = 1; j < K; ++j) tied = tied || L[j] == L[j - 1];
    }
    if constexpr (MODE == TILE_SOR_MEAN || MODE == TILE_SOR_LIST) {
      float sum = 0.0f;
#pragma unroll
      for (int j = 1; j < K; ++j) sum = fadd(sum, __fsqrt_rn(L[j]));
      a.mean[qi] = fdiv(sum, (float)(K - 1));
      if constexpr (MODE == TILE_SOR_LIST) {
        u32 *row = a.sor_list + (size_t)pos * K;
#pragma unroll
        for (int j = 0; j < K; ++j) row[j] = tied ? 0xFFFFFFFFu : I[j];
      }
    } else if constexpr (MODE == TILE_NORMALS) {
#pragma unroll
      for (int j = 0; j < K; ++j) slot_pairs[(size_t)s * K + j] = L[j];
      slot_counts[s] = K;
    } else if constexpr (MODE == TILE_PAIRS_F) {
      if (tied) continue;  // the exact (d2, index) order from the warp kernel
#pragma unroll
      for (int j = 0; j < K; ++j) a.pairs[(size_t)qi * K + j] = pack_nbr(L[j], (int)I[j]);
      if (a.counts) a.counts[qi] = K;
    } else {
#pragma unroll
      for (int j = 0; j < K; ++j) a.pairs[(size_t)qi * K + j] = L[j];
      if (a.counts) a.counts[qi] = K;
    }
    a.hard_tau[s] = kTauDone;
    if (stats) atomicAdd(stats, 1u);
  }
}

// Adaptive per-thread kNN for the queries the cooperative pass leaves open
// (sparse cells, and the dense ones it could not finish): one thread per
// query, no table shared with other lanes. A radius r is estimated from the
// finest chain level whose own cell holds K points (r = cell * sqrt(K /
// count), under one cell; the top level's cell when none does). Then,
// repeatedly: the tight window of r at the finest table level where it
// spans at most kAdaptCells cells; from the second attempt on, a count pass
// over its cells within r (cell box lower bound) -- fewer than K points: r
// doubles, nothing scanned; more than kTauPoints: the query goes to the warp
// kernel (lanes over candidates); then a scan bounded by r^2 (every point
// with d2 <= r^2 lies in the window; a scan that would pass kTauPoints
// candidates stops and the warp kernel takes the query), exact when it
// found K such points, else r grows by sqrt 2.
// Queries left after kAdaptTries attempts go to the hard list without a
// bound. Outputs as k_knn_wt's (the SOR mean and list row, the fused
// normal, or feature pairs; tied lists as there).
constexpr int kAdaptTries = 8;
constexpr int kAdaptCells = 64;  // window cells one thread looks up

template <int K, int MODE>
__global__ __launch_bounds__(TT, 4) void k_knn_adapt(GridView g, TileArgs a, const u32 *list,
                                                     const u64 *n_list, u32 *stats) {
  constexpr bool FKEY = MODE == TILE_SOR_MEAN || MODE == TILE_SOR_LIST || MODE == TILE_PAIRS_F;
  constexpr bool KV = MODE == TILE_SOR_LIST || MODE == TILE_PAIRS_F;
  using Key = typename std::conditional<FKEY, float, u64>::type;
  const u64 n = *n_list;
  const int top = g.lbase + kGridLevels - 1;
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    const u32 pos = list[i];
    const float4 q = g.pts[pos];
    const u32 qidx = __float_as_uint(q.w);
    if (MODE == TILE_NORMALS && (qidx & kRemovedBit)) continue;
    const u32 qi = qidx & 0x7FFFFFFFu;
    const GridFrame F = g.frames[a.frame_of ? a.frame_of[qi] : 0];
    const int fx = cell_axis(q.x, F.min_x, F.cell), fy = cell_axis(q.y, F.min_y, F.cell),
              fz = cell_axis(q.z, F.min_z, F.cell);
    float r = F.cell * (float)(1 << top);
    for (int L = g.lbase; L <= top; ++L) {
      u32 st, ct;
      if (!lookup(g, level_key(g, F, L, fx >> L, fy >> L, fz >> L), st, ct)) ct = 0;
      if (ct >= (u32)K) {
        const float cs = F.cell * (float)(1 << L);
        r = fminf(cs * sqrtf((float)K / (float)ct), cs);
        break;
      }
    }
    Key kMax;
    if constexpr (FKEY) kMax = INFINITY;
    else kMax = ~0ull;
    Key L[K];
    u32 I[KV ? K : 1];
    float tie = -1.0f;
    bool done = false, punt = false;
    for (int attempt = 0; attempt < kAdaptTries && !done && !punt; ++attempt) {
      const float tb = r * r;
      Window w;
      int level = -1;
      for (int Lv = g.lbase; Lv <= top; ++Lv) {
        w = tight_window(F, q.x, q.y, q.z, sqrt((double)tb), Lv);
        if (window_cells(w) <= kAdaptCells) {
          level = Lv;
          break;
        }
      }
      if (level < 0) {
        punt = true;
        break;
      }
      // from the second attempt on, a count pass first (the first radius
      // is mostly generous enough, so its window is scanned at once)
      if (attempt > 0) {
        u32 total = 0;
        for (int uz = w.lo[2]; uz <= w.hi[2]; ++uz)
          for (int uy = w.lo[1]; uy <= w.hi[1]; ++uy)
            for (int ux = w.lo[0]; ux <= w.hi[0]; ++ux) {
              u32 st, cnt;
              if (cell_lb2(F, level, ux, uy, uz, q.x, q.y, q.z) <= tb &&
                  lookup(g, level_key(g, F, level, ux, uy, uz), st, cnt))
                total += cnt;
            }
        if (total < (u32)K) {  // the window cannot hold K points within r
          r *= 2.0f;
          continue;
        }
        if (total > kTauPoints) {
          punt = true;
          break;
        }
      }
#pragma unroll
      for (int j = 0; j < K; ++j) L[j] = kMax;
      Key thr = kMax;
      tie = -1.0f;
      u32 found = 0, scanned = 0;
      for (int uz = w.lo[2]; uz <= w.hi[2] && !punt; ++uz)
        for (int uy = w.lo[1]; uy <= w.hi[1] && !punt; ++uy)
          for (int ux = w.lo[0]; ux <= w.hi[0] && !punt; ++ux) {
            float thr_d2;
            if constexpr (FKEY) thr_d2 = thr;
            else thr_d2 = nbr_d2(thr);
            if (cell_lb2(F, level, ux, uy, uz, q.x, q.y, q.z) > fminf(thr_d2, tb)) continue;
            u32 st, cnt;
            if (!lookup(g, level_key(g, F, level, ux, uy, uz), st, cnt)) continue;
            // a dense window: the warp kernel (lanes over candidates)
            if (scanned + cnt > kTauPoints) {
              punt = true;
              break;
            }
            scanned += cnt;
            for (u32 j = 0; j < cnt; ++j) {
              const float4 p = __ldg(&g.pts[st + j]);
              const u32 pidx = __float_as_uint(p.w);
              if (MODE == TILE_NORMALS && (pidx & kRemovedBit)) continue;
              const float d2 = dist2(p.x, p.y, p.z, q.x, q.y, q.z);
              if (!(d2 <= tb)) continue;
              ++found;
              Key key;
              if constexpr (FKEY) key = d2;
              else key = pack_nbr(d2, (int)pidx);
              if (key < thr) {
                if constexpr (KV) {
                  list_insert_kv<K>(L, I, key, MODE == TILE_SOR_LIST ? st + j : pidx);
                  if (L[K - 1] == thr) tie = thr;  // evicted a key equal to the boundary
                } else {
                  list_insert<Key, K>(L, key);
                }
                thr = L[K - 1];
              } else if constexpr (KV) {
                if (key == thr) tie = key;
              }
            }
          }
      if (punt) break;
      if (found >= (u32)K) done = true;
      else r *= 1.41421356f;
    }
    if (!done) {
      const u32 slot = atomicAdd(a.hard_count, 1u);
      a.hard[slot] = qi;
      if (a.hard_tau) a.hard_tau[slot] = -1.0f;
      continue;
    }
    if (stats) atomicAdd(stats, 1u);
    bool tied = false;
    if constexpr (KV) {
      tied = tie == L[K - 1];
#pragma unroll
      for (int j = 1; j < K; ++j) tied = tied || L[j] == L[j - 1];
    }
    if constexpr (MODE == TILE_SOR_MEAN || MODE == TILE_SOR_LIST) {
      float sum = 0.0f;
#pragma unroll
      for (int j = 1; j < K; ++j) sum = fadd(sum, __fsqrt_rn(L[j]));
      a.mean[qi] = fdiv(sum, (float)(K - 1));
      if constexpr (MODE == TILE_SOR_LIST) {
        u32 *row = a.sor_list + (size_t)pos * K;
#pragma unroll
        for (int j = 0; j < K; ++j) row[j] = tied ? 0xFFFFFFFFu : I[j];
      }
    } else if constexpr (MODE == TILE_NORMALS) {
      float nx, ny, nz;
      normal_from_keys<K>(a.vx, a.vy, a.vz, L, true, a.iters, q.x, q.y, q.z, a.vpx, a.vpy,
                          a.vpz, nx, ny, nz);
      const u64 o = a.out_pos[qi];
      a.nx[o] = nx;
      a.ny[o] = ny;
      a.nz[o] = nz;
    } else if constexpr (MODE == TILE_PAIRS_F) {
      if (tied) {  // the exact (d2, index) list from the warp kernel
        const u32 slot = atomicAdd(a.hard_count, 1u);
        a.hard[slot] = qi;
        if (a.hard_tau) a.hard_tau[slot] = L[K - 1];
      } else {
#pragma unroll
        for (int j = 0; j < K; ++j) a.pairs[(size_t)qi * K + j] = pack_nbr(L[j], (int)I[j]);
        if (a.counts) a.counts[qi] = K;
      }
    } else {
#pragma unroll
      for (int j = 0; j < K; ++j) a.pairs[(size_t)qi * K + j] = L[j];
      if (a.counts) a.counts[qi] = K;
    }
  }
}

// the cooperative pass takes the grid points whose own cell (chain level
// lbase) holds at least min_own points (qlevel = kCoopMark); the others are
// open for the per-lane kernels at that level
constexpr uint8_t kCoopMark = 0xFE;
__global__ void k_knn_route(GridView g, const int32_t *frame_of, u32 min_own, uint8_t *qlevel) {
  const u64 n = *g.n_points;
  const int lb = g.lbase;
  for (u64 pos = blockIdx.x * (u64)blockDim.x + threadIdx.x; pos < n;
       pos += (u64)gridDim.x * blockDim.x) {
    const float4 q = g.pts[pos];
    const u32 qidx = __float_as_uint(q.w) & 0x7FFFFFFFu;
    const GridFrame F = g.frames[frame_of ? frame_of[qidx] : 0];
    const int cx = cell_axis(q.x, F.min_x, F.cell) >> lb, cy = cell_axis(q.y, F.min_y, F.cell) >> lb,
              cz = cell_axis(q.z, F.min_z, F.cell) >> lb;
    u32 st = 0, ct = 0;
    if (!lookup(g, level_key(g, F, lb, cx, cy, cz), st, ct)) ct = 0;
    qlevel[pos] = ct >= min_own ? kCoopMark : (uint8_t)lb;
  }
}

// open queries of `level`, in grid (cell) order: flags -> scan -> positions
__global__ void k_open_flags(const uint8_t *qlevel, const u64 *n_dev, int level, u32 *flags) {
  const u64 n = *n_dev;
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    flags[i] = qlevel[i] == level ? 1u : 0u;
}
__global__ void k_open_scatter(const u32 *flags, const u64 *pos, const u64 *n_dev, u32 *list,
                               u64 *n_list, u64 *n_copy = nullptr) {
  const u64 n = *n_dev;
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    if (flags[i]) list[pos[i]] = (u32)i;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *n_list = pos[n];
    if (n_copy) *n_copy = pos[n];
  }
}

// the open queries (grid positions) to the hard list without a bound: the
// warp-per-query kernel estimates their radius (kTauEstimate)
__global__ void k_open_to_hard(GridView g, const u32 *list, const u64 *n_list, u32 *hard,
                               u32 *hard_count, float *hard_tau) {
  const u64 n = *n_list;
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    const u32 qi = __float_as_uint(g.pts[list[i]].w) & 0x7FFFFFFFu;
    const u32 slot = atomicAdd(hard_count, 1u);
    hard[slot] = qi;
    if (hard_tau) hard_tau[slot] = kTauEstimate;
  }
}

template <int K>
void launch_k(rvp_context *ctx, const GridView &g, int mode, const TileArgs &a_in, int blocks,
              uint8_t *qlevel, u32 *stats) {
  TileArgs a = a_in;
  // the cooperative pass first (float-key modes over every grid point): the
  // points of dense cells, the warps working on 32 queries together; the
  // per-lane kernels then take what stays open, from their ring pass on (no
  // second bounded pass at the first chain level)
  const bool coop = a.coop && a.level0_warp && !a.preset_open &&
                    (mode == TILE_SOR_MEAN || mode == TILE_SOR_LIST || mode == TILE_PAIRS_F);
  if (coop) {
    static bool attr_set[64] = {false};
    if (ctx->device < 64 && !attr_set[ctx->device]) {
      RVP_CUDA_TRY(cudaFuncSetAttribute(k_knn_coop<K, TILE_SOR_MEAN>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)CP_SMEM));
      RVP_CUDA_TRY(cudaFuncSetAttribute(k_knn_coop<K, TILE_SOR_LIST>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)CP_SMEM));
      RVP_CUDA_TRY(cudaFuncSetAttribute(k_knn_coop<K, TILE_PAIRS_F>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)CP_SMEM));
      attr_set[ctx->device] = true;
    }
    const unsigned gb = grid_for(a.n_max, 256, ctx->num_sms * 16);
    const float rf = a.rfac > 0.0f ? a.rfac : 1.0f;
    const u32 min_own = (u32)ceilf(rf * rf * (float)K / 0.998f);
    k_knn_route<<<gb, 256, 0, ctx->stream>>>(g, a.frame_of, min_own, qlevel);
    RVP_LAUNCH_CHECK(ctx);
    k_open_flags<<<gb, 256, 0, ctx->stream>>>(qlevel, g.n_points, kCoopMark, a.open_flags);
    RVP_LAUNCH_CHECK(ctx);
    exclusive_scan_u32_to_u64(ctx, a.open_flags, a.open_pos, a.n_max, g.n_points, a.scan_tmp);
    k_open_scatter<<<gb, 256, 0, ctx->stream>>>(a.open_flags, a.open_pos, g.n_points,
                                                a.open_list, a.open_n, a.routed);
    RVP_LAUNCH_CHECK(ctx);
    cudaEvent_t *ev = a.level_events ? a.level_events + 2 * kChainLevels : nullptr;
    if (ev) cudaEventRecord(ev[0], ctx->stream);
    const int cblocks = ctx->num_sms * 2;
    if (mode == TILE_SOR_MEAN)
      k_knn_coop<K, TILE_SOR_MEAN><<<cblocks, TT, CP_SMEM, ctx->stream>>>(
          g, a, g.lbase, a.open_list, a.open_n, qlevel, a.qtau, stats);
    else if (mode == TILE_SOR_LIST)
      k_knn_coop<K, TILE_SOR_LIST><<<cblocks, TT, CP_SMEM, ctx->stream>>>(
          g, a, g.lbase, a.open_list, a.open_n, qlevel, a.qtau, stats);
    else
      k_knn_coop<K, TILE_PAIRS_F><<<cblocks, TT, CP_SMEM, ctx->stream>>>(
          g, a, g.lbase, a.open_list, a.open_n, qlevel, a.qtau, stats);
    RVP_LAUNCH_CHECK(ctx);
    if (ev) cudaEventRecord(ev[1], ctx->stream);
    a.preset_open = true;
  } else if (a.level_events) {
    // no cooperative pass: a zero-length pair in its slot
    cudaEventRecord(a.level_events[2 * kChainLevels], ctx->stream);
    cudaEventRecord(a.level_events[2 * kChainLevels + 1], ctx->stream);
  }
  if (a.coop && a.level0_warp && a.preset_open) {
    // cooperative mode: what is open (the cooperative pass's leftovers, or
    // the caller's open queries) goes to the adaptive per-thread kernel
    // (normals: to the warp-per-query kernel with an estimated radius),
    // timed in the first chain slot
    const unsigned gb = grid_for(a.n_max, 256, ctx->num_sms * 16);
    k_open_flags<<<gb, 256, 0, ctx->stream>>>(qlevel, g.n_points, g.lbase, a.open_flags);
    RVP_LAUNCH_CHECK(ctx);
    exclusive_scan_u32_to_u64(ctx, a.open_flags, a.open_pos, a.n_max, g.n_points, a.scan_tmp);
    k_open_scatter<<<gb, 256, 0, ctx->stream>>>(a.open_flags, a.open_pos, g.n_points,
                                                a.open_list, a.open_n,
                                                a.routed ? a.routed + 1 : nullptr);
    RVP_LAUNCH_CHECK(ctx);
    if (a.level_events) cudaEventRecord(a.level_events[0], ctx->stream);
    if (mode == TILE_NORMALS && a.hard_tau) {
      // the normal stage's few open queries sit next to removed points, in
      // every kind of neighbourhood: the warp-per-query kernel (lanes over
      // cells and candidates) takes them, with an estimated radius
      k_open_to_hard<<<gb, 256, 0, ctx->stream>>>(g, a.open_list, a.open_n, a.hard,
                                                  a.hard_count, a.hard_tau);
    } else {
      const int ablocks = ctx->num_sms * 4;
#define RVP_ADAPT(M) \
  k_knn_adapt<K, M><<<ablocks, TT, 0, ctx->stream>>>(g, a, a.open_list, a.open_n, stats)
      if (mode == TILE_SOR_MEAN) RVP_ADAPT(TILE_SOR_MEAN);
      else if (mode == TILE_SOR_LIST) RVP_ADAPT(TILE_SOR_LIST);
      else if (mode == TILE_NORMALS) RVP_ADAPT(TILE_NORMALS);
      else if (mode == TILE_PAIRS_F) RVP_ADAPT(TILE_PAIRS_F);
      else RVP_ADAPT(TILE_PAIRS);
#undef RVP_ADAPT
    }
    RVP_LAUNCH_CHECK(ctx);
    if (a.level_events) {
      cudaEventRecord(a.level_events[1], ctx->stream);
      for (int j = 1; j < kChainLevels; ++j) {  // not run: zero length
        cudaEventRecord(a.level_events[2 * j], ctx->stream);
        cudaEventRecord(a.level_events[2 * j + 1], ctx->stream);
      }
    }
    return;
  }
  if (!a.preset_open)
    RVP_CUDA_TRY(cudaMemsetAsync(qlevel, (uint8_t)g.lbase, a.n_max, ctx->stream));
  const int nlev = a.lane_levels > 0 && a.lane_levels < kChainLevels ? a.lane_levels
                                                                      : kChainLevels;
  if (a.level0_warp) {
    // barrier-free per-warp kernels at every chain level; the levels past
    // the first (and the first when the caller marked the open queries)
    // read the compacted list of open queries
    const int wblocks = ctx->num_sms * 3 * 4;
    for (int j = 0; j < nlev; ++j) {
      const int level = g.lbase + kChainStep * j;
      const u32 *list = nullptr;
      if (j > 0 || a.preset_open) {
        const unsigned gb = grid_for(a.n_max, 256, ctx->num_sms * 16);
        k_open_flags<<<gb, 256, 0, ctx->stream>>>(qlevel, g.n_points, level, a.open_flags);
        RVP_LAUNCH_CHECK(ctx);
        exclusive_scan_u32_to_u64(ctx, a.open_flags, a.open_pos, a.n_max, g.n_points, a.scan_tmp);
        k_open_scatter<<<gb, 256, 0, ctx->stream>>>(a.open_flags, a.open_pos, g.n_points,
                                                    a.open_list, a.open_n);
        RVP_LAUNCH_CHECK(ctx);
        list = a.open_list;
      }
      u32 *st = stats ? stats + j : nullptr;
      if (a.level_events) cudaEventRecord(a.level_events[2 * j], ctx->stream);
      if (mode == TILE_SOR_MEAN)
        k_knn_wt<K, TILE_SOR_MEAN><<<wblocks, TT, 0, ctx->stream>>>(g, a, level, list, a.open_n,
                                                                    qlevel, a.qtau, st);
      else if (mode == TILE_SOR_LIST)
        k_knn_wt<K, TILE_SOR_LIST><<<wblocks, TT, 0, ctx->stream>>>(g, a, level, list, a.open_n,
                                                                    qlevel, a.qtau, st);
      else if (mode == TILE_NORMALS)
        k_knn_wt<K, TILE_NORMALS><<<wblocks, TT, 0, ctx->stream>>>(g, a, level, list, a.open_n,
                                                                   qlevel, a.qtau, st);
      else if (mode == TILE_PAIRS_F)
        k_knn_wt<K, TILE_PAIRS_F><<<wblocks, TT, 0, ctx->stream>>>(g, a, level, list, a.open_n,
                                                                   qlevel, a.qtau, st);
      else
        k_knn_wt<K, TILE_PAIRS><<<wblocks, TT, 0, ctx->stream>>>(g, a, level, list, a.open_n,
                                                                 qlevel, a.qtau, st);
      RVP_LAUNCH_CHECK(ctx);
      if (a.level_events) cudaEventRecord(a.level_events[2 * j + 1], ctx->stream);
    }
    for (int j = nlev; j < kChainLevels && a.level_events; ++j) {
      cudaEventRecord(a.level_events[2 * j], ctx->stream);  // not run: zero length
      cudaEventRecord(a.level_events[2 * j + 1], ctx->stream);
    }
    return;
  }
  for (int j = 0; j < kChainLevels; ++j) {
    const int level = g.lbase + kChainStep * j;
    u32 *st = stats ? stats + j : nullptr;
    if (a.level_events) cudaEventRecord(a.level_events[2 * j], ctx->stream);
    if (mode == TILE_SOR_MEAN)
      k_knn_tile<K, TILE_SOR_MEAN><<<blocks, TT, 0, ctx->stream>>>(g, a, level, qlevel, a.qtau,
                                                                   st);
    else if (mode == TILE_SOR_LIST)
      k_knn_tile<K, TILE_SOR_LIST><<<blocks, TT, 0, ctx->stream>>>(g, a, level, qlevel, a.qtau,
                                                                   st);
    else if (mode == TILE_NORMALS)
      k_knn_tile<K, TILE_NORMALS><<<blocks, TT, 0, ctx->stream>>>(g, a, level, qlevel, a.qtau,
                                                                  st);
    else
      k_knn_tile<K, TILE_PAIRS><<<blocks, TT, 0, ctx->stream>>>(g, a, level, qlevel, a.qtau, st);
    RVP_LAUNCH_CHECK(ctx);
    if (a.level_events) cudaEventRecord(a.level_events[2 * j + 1], ctx->stream);
  }
}
}  // namespace

namespace {
// Normals from the SOR stage's neighbour lists. The k+1 nearest points of a
// kept point are its k+1 nearest kept points whenever none of them was
// removed (removal only takes points away, and the (d2, index) order of the
// rest is unchanged), so the first KN entries of its SOR list, when all kept,
// are exactly the list the normal needs. Those points get their normal here;
// the others are marked open (qlevel 0) for the kNN search. One thread per
// grid point: its row of the list (rows by grid position, so a warp reads
// consecutive rows) and its neighbours' float4 grid records (spatially close,
// so mostly cached), whose index word carries the removed flag.
template <int KN>
__global__ __launch_bounds__(256, 4) void k_normals_sor_lists(GridView g, TileArgs a, int ks) {
  const u64 n = *g.n_points;
  for (u64 pos = blockIdx.x * (u64)blockDim.x + threadIdx.x; pos < n;
       pos += (u64)gridDim.x * blockDim.x) {
    const float4 q = g.pts[pos];
    const u32 qidx = __float_as_uint(q.w);
    if (qidx & kRemovedBit) {
      a.qlevel[pos] = 0xFF;
      continue;
    }
    const u32 *row = a.sor_list + (size_t)pos * ks;
    float px[KN], py[KN], pz[KN];
    bool ok = true;
#pragma unroll
    for (int t = 0; t < KN; ++t) {
      const u32 j = __ldg(&row[t]);
      ok = ok && j != 0xFFFFFFFFu;
      const float4 p = ok ? __ldg(&g.pts[j]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      ok = ok && !(__float_as_uint(p.w) & kRemovedBit);
      px[t] = p.x;
      py[t] = p.y;
      pz[t] = p.z;
    }
    if (!ok) {
      a.qlevel[pos] = (uint8_t)g.lbase;  // open at the first chain level
      continue;
    }
    a.qlevel[pos] = 0xFF;
    float nx, ny, nz;
    normal_from_coords<KN>(px, py, pz, true, a.iters, q.x, q.y, q.z, a.vpx, a.vpy, a.vpz, nx,
                           ny, nz);
    const u64 o = a.out_pos[qidx];
    a.nx[o] = nx;
    a.ny[o] = ny;
    a.nz[o] = nz;
  }
}
}  // namespace

bool normals_from_sor_lists(rvp_context *ctx, const GridView &g, const TileArgs &a, int ks,
                            int kn) {
  if (g.mode != KEY_DENSE || !a.sor_list || !a.qlevel || kn > ks) return false;
  const unsigned blocks = grid_for(a.n_max, 256, ctx->num_sms * 16);
  switch (kn) {
#define RVP_NSL(K)                                                                        \
  case K:                                                                                 \
    k_normals_sor_lists<K><<<blocks, 256, 0, ctx->stream>>>(g, a, ks);                    \
    break;
    RVP_NSL(8) RVP_NSL(11) RVP_NSL(16) RVP_NSL(17) RVP_NSL(21) RVP_NSL(31) RVP_NSL(32)
    RVP_NSL(33)
#undef RVP_NSL
    default: return false;
  }
  RVP_LAUNCH_CHECK(ctx);
  return true;
}

bool grid_knn_tau(rvp_context *ctx, const GridView &g, int k, int mode, const TileArgs &a,
                  const u64 *n_hard, u64 *slot_pairs, int32_t *slot_counts, u32 *stats) {
  if (g.mode != KEY_DENSE || !a.hard || !a.hard_tau) return false;
  const int blocks = ctx->num_sms * 3;
  auto go = [&](auto kc) {
    constexpr int K = decltype(kc)::value;
    switch (mode) {
      case TILE_SOR_MEAN:
        k_knn_tau<K, TILE_SOR_MEAN><<<blocks, TT, 0, ctx->stream>>>(g, a, n_hard, slot_pairs,
                                                                    slot_counts, stats);
        break;
      case TILE_SOR_LIST:
        k_knn_tau<K, TILE_SOR_LIST><<<blocks, TT, 0, ctx->stream>>>(g, a, n_hard, slot_pairs,
                                                                    slot_counts, stats);
        break;
      case TILE_NORMALS:
        k_knn_tau<K, TILE_NORMALS><<<blocks, TT, 0, ctx->stream>>>(g, a, n_hard, slot_pairs,
                                                                   slot_counts, stats);
        break;
      case TILE_PAIRS_F:
        k_knn_tau<K, TILE_PAIRS_F><<<blocks, TT, 0, ctx->stream>>>(g, a, n_hard, slot_pairs,
                                                                   slot_counts, stats);
        break;
      default:
        k_knn_tau<K, TILE_PAIRS><<<blocks, TT, 0, ctx->stream>>>(g, a, n_hard, slot_pairs,
                                                                 slot_counts, stats);
    }
  };
  switch (k) {
    case 8: go(std::integral_constant<int, 8>()); break;
    case 11: go(std::integral_constant<int, 11>()); break;
    case 16: go(std::integral_constant<int, 16>()); break;
    case 17: go(std::integral_constant<int, 17>()); break;
    case 21: go(std::integral_constant<int, 21>()); break;
    case 31: go(std::integral_constant<int, 31>()); break;
    case 32: go(std::integral_constant<int, 32>()); break;
    case 33: go(std::integral_constant<int, 33>()); break;
    default: return false;
  }
  RVP_LAUNCH_CHECK(ctx);
  return true;
}

bool grid_knn_tile(rvp_context *ctx, const GridView &g, int k, int mode, const TileArgs &a,
                   int blocks, u32 *stats) {
  if (g.mode != KEY_DENSE || !a.qlevel || !a.qtau) return false;
  if (a.preset_open && !a.level0_warp) return false;
  if (blocks <= 0) blocks = ctx->num_sms * 8;
  switch (k) {
    case 8: launch_k<8>(ctx, g, mode, a, blocks, a.qlevel, stats); break;
    case 11: launch_k<11>(ctx, g, mode, a, blocks, a.qlevel, stats); break;
    case 16: launch_k<16>(ctx, g, mode, a, blocks, a.qlevel, stats); break;
    case 17: launch_k<17>(ctx, g, mode, a, blocks, a.qlevel, stats); break;
    case 21: launch_k<21>(ctx, g, mode, a, blocks, a.qlevel, stats); break;
    case 31: launch_k<31>(ctx, g, mode, a, blocks, a.qlevel, stats); break;
    case 32: launch_k<32>(ctx, g, mode, a, blocks, a.qlevel, stats); break;
    case 33: launch_k<33>(ctx, g, mode, a, blocks, a.qlevel, stats); break;
    default: return false;
  }
  return true;
}

}  // namespace rvp
