// Tile kNN for dense (batched) grids on sm_100a.
//
// Level by level (cells of c, 4c, 16c): one thread block per bucket of the
// next level up (a group of 4 x 4 x 4 cells) looks up the 6 x 6 x 6 cells
// around it once (one lookup per thread), flattens them with a prefix sum
// and stages their points in shared memory (coalesced float4 runs). Every
// open query of the group is then handled by one thread, which scans its own
// 27-cell ring out of shared memory and keeps a register-resident sorted
// top-K (unrolled insertion network; float keys when only distances matter,
// packed (d2, index) keys when ties must follow the reference's (d2, index)
// order). The ring certifies the result when the K-th distance is below the
// ring's coverage (distance to the nearest outside cell, with rounding
// slack); the others stay open for the next, 4x coarser level, and after the
// last level go to a list that the warp-per-query kernel finishes. Epilogues are fused: SOR mean distance
// (statistical_outlier_removal.cpp:36-40) or the reference normal
// (normal_estimation.cpp:141-161) straight from the registers.
#include <type_traits>

#include "grid_device.cuh"
#include "internal.cuh"
#include "normals_device.cuh"

namespace rvp {
using namespace gd;
using namespace nd;

namespace {
constexpr int TT = 256;                      // threads per tile block
constexpr int SIDE = 6;                      // staged fine cells per axis
constexpr int NCELL = SIDE * SIDE * SIDE;    // 216
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

template <int K, int MODE>
__global__ __launch_bounds__(TT) void k_knn_tile(GridView g, TileArgs a, int level,
                                                 uint8_t *qlevel, float *qtau, u32 *stats) {
  using Key = typename std::conditional<MODE == TILE_SOR_MEAN, float, u64>::type;
  __shared__ u32 c_start[NCELL];
  __shared__ u32 c_count[NCELL];
  __shared__ u32 c_pref[NCELL + 1];
  __shared__ float4 cand[CAP];
  __shared__ int s_base[4];
  __shared__ int s_staged;
  const u64 ngroups = g.n_level[level + 1];
  const u32 *gstart = g.lstart[level + 1];
  const u64 n = *g.n_points;
  const int tid = threadIdx.x;
  const int sh = 2 * level;  // level-L cell = fine index >> sh
  Key kMax;
  if constexpr (MODE == TILE_SOR_MEAN) kMax = INFINITY;
  else kMax = ~0ull;
  for (u64 cb = blockIdx.x; cb < ngroups; cb += gridDim.x) {
    const u32 qs = gstart[cb];
    const u32 qe = (cb + 1 < ngroups) ? gstart[cb + 1] : (u32)n;
    if (level > 0) {  // only the queries the previous level left open
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
      const int gs = sh + 2;  // group cell = fine index >> gs
      s_base[0] = (cell_axis(p0.x, F.min_x, F.cell) >> gs) * 4 - 1;
      s_base[1] = (cell_axis(p0.y, F.min_y, F.cell) >> gs) * 4 - 1;
      s_base[2] = (cell_axis(p0.z, F.min_z, F.cell) >> gs) * 4 - 1;
      s_base[3] = f;
    }
    __syncthreads();
    const int bx = s_base[0], by = s_base[1], bz = s_base[2];
    const GridFrame F = g.frames[s_base[3]];
    const int dx_ = level_dim(F.gx, level), dy_ = level_dim(F.gy, level),
              dz_ = level_dim(F.gz, level);
    // 1) the 6 x 6 x 6 level-L cells around the group
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
      if (level > 0 && qlevel[qi] != level) continue;
      const float4 q = g.pts[qi];
      const u32 qidx = __float_as_uint(q.w);
      if (MODE == TILE_NORMALS && (qidx & kRemovedBit)) continue;
      const int lx = (cell_axis(q.x, F.min_x, F.cell) >> sh) - bx;  // 1..4
      const int ly = (cell_axis(q.y, F.min_y, F.cell) >> sh) - by;
      const int lz = (cell_axis(q.z, F.min_z, F.cell) >> sh) - bz;
      Key L[K];
#pragma unroll
      for (int j = 0; j < K; ++j) L[j] = kMax;
      Key thr = kMax;
      u32 found = 0;
      // A query left open by the level below with K points found there
      // carries tau >= its K-th distance: every point with d2 <= tau lies in
      // the tight window of sqrt(tau) (at most the own cell +- 1 here, since
      // sqrt(tau) < one cell of this level), so scanning that window with
      // the bound tau is exact and needs no further check.
      const float tb = level > 0 ? qtau[qi] : -1.0f;
      bool bounded = tb >= 0.0f;
      int lo[3] = {-1, -1, -1}, hi[3] = {1, 1, 1};
      if (bounded) {
        const Window wt = tight_window(F, q.x, q.y, q.z, sqrt((double)tb), level);
        const int own[3] = {lx + bx, ly + by, lz + bz};
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          lo[ax] = wt.lo[ax] - own[ax];
          hi[ax] = wt.hi[ax] - own[ax];
          if (lo[ax] < -1 || hi[ax] > 1) bounded = false;
        }
        if (!bounded)
#pragma unroll
          for (int ax = 0; ax < 3; ++ax) { lo[ax] = -1; hi[ax] = 1; }
      }
      // distance from q to the faces of its own cell, shrunk by the rounding
      // slack of the cell function: a point of a neighbour cell lies at least
      // this far away along that axis
      float gap_lo[3], gap_hi[3];
      {
        const float qq[3] = {q.x, q.y, q.z};
        const float mn[3] = {F.min_x, F.min_y, F.min_z};
        const int own[3] = {lx + bx, ly + by, lz + bz};
        const double cs = (double)F.cell * (double)(1 << sh);
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          const double face0 = (double)mn[ax] + (double)own[ax] * cs;
          const double slack = 2.4e-7 * (fabs((double)mn[ax]) + fabs((double)qq[ax]) +
                                         (double)(own[ax] + 2) * cs) + 1e-30;
          gap_lo[ax] = (float)fmax((double)qq[ax] - face0 - slack, 0.0);
          gap_hi[ax] = (float)fmax(face0 + cs - (double)qq[ax] - slack, 0.0);
        }
      }
      for (int t = 0; t < 27; ++t) {
        const int dx = kRingOrder[t][0], dy = kRingOrder[t][1], dz = kRingOrder[t][2];
        if (dx < lo[0] || dx > hi[0] || dy < lo[1] || dy > hi[1] || dz < lo[2] || dz > hi[2])
          continue;
        if (t > 0) {
          // skip a cell that cannot hold anything below the current K-th
          // distance (nothing is skipped until the list is full)
          float thr_d2;
          if constexpr (MODE == TILE_SOR_MEAN) thr_d2 = thr;
          else thr_d2 = nbr_d2(thr);
          const float gx = dx < 0 ? gap_lo[0] : (dx > 0 ? gap_hi[0] : 0.0f);
          const float gy = dy < 0 ? gap_lo[1] : (dy > 0 ? gap_hi[1] : 0.0f);
          const float gz = dz < 0 ? gap_lo[2] : (dz > 0 ? gap_hi[2] : 0.0f);
          const float box2 = (gx * gx + gy * gy + gz * gz) * (1.0f - 1e-5f);
          if (box2 > thr_d2) continue;
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
      bool ok = bounded && found >= (u32)K;
      float tau = -1.0f;
      if (!ok && found >= (u32)K) {
        if constexpr (MODE == TILE_SOR_MEAN) tau = L[K - 1];
        else tau = nbr_d2(L[K - 1]);
        const Window w1 = ring_window(F, q.x, q.y, q.z, 1, level);
        const double cov = coverage(F, w1, q.x, q.y, q.z);
        ok = cov > 0.0 && (double)tau < cov * cov * (1.0 - 1e-5);
      }
      if (!ok) {
        if (level + 1 < kGridLevels) {
          qlevel[qi] = (uint8_t)(level + 1);
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

// Level 0: one warp per fine cell of the group. Its lanes take the cell's
// queries (32 at a time) and all walk the same 27-cell candidate stream, so
// loop bounds are uniform and every candidate is one broadcast shared-memory
// read; only the insertion into a lane's own list diverges.
template <int K, int MODE>
__global__ __launch_bounds__(TT, MODE == TILE_SOR_MEAN ? 4 : 3) void k_knn_tile0(GridView g, TileArgs a, uint8_t *qlevel,
                                                     float *qtau, u32 *stats) {
  using Key = typename std::conditional<MODE == TILE_SOR_MEAN, float, u64>::type;
  __shared__ u32 c_start[NCELL];
  __shared__ u32 c_count[NCELL];
  __shared__ u32 c_pref[NCELL + 1];
  __shared__ float4 cand[CAP];
  __shared__ GridFrame s_F;
  __shared__ int s_base[3];
  __shared__ int s_staged;
  const u64 ngroups = g.n_level[1];
  const u32 *gstart = g.lstart[1];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  Key kMax;
  if constexpr (MODE == TILE_SOR_MEAN) kMax = INFINITY;
  else kMax = ~0ull;
  for (u64 cb = blockIdx.x; cb < ngroups; cb += gridDim.x) {
    __syncthreads();  // the previous group's shared memory is free
    if (tid == 0) {
      const float4 p0 = g.pts[gstart[cb]];
      const u32 i0 = __float_as_uint(p0.w) & 0x7FFFFFFFu;
      const GridFrame F = g.frames[a.frame_of ? a.frame_of[i0] : 0];
      s_F = F;
      s_base[0] = (cell_axis(p0.x, F.min_x, F.cell) >> 2) * 4 - 1;
      s_base[1] = (cell_axis(p0.y, F.min_y, F.cell) >> 2) * 4 - 1;
      s_base[2] = (cell_axis(p0.z, F.min_z, F.cell) >> 2) * 4 - 1;
    }
    __syncthreads();
    {
      const int bx = s_base[0], by = s_base[1], bz = s_base[2];
      const int gx = s_F.gx, gy = s_F.gy, gz = s_F.gz;
      for (int t = tid; t < NCELL; t += TT) {
        const int cx = bx + t % SIDE, cy = by + (t / SIDE) % SIDE, cz = bz + t / (SIDE * SIDE);
        u32 st = 0, ct = 0;
        if (cx >= 0 && cy >= 0 && cz >= 0 && cx < gx && cy < gy && cz < gz)
          if (!lookup(g, level_key(g, s_F, 0, cx, cy, cz), st, ct)) ct = 0;
        c_start[t] = st;
        c_count[t] = ct;
      }
    }
    __syncthreads();
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
        int lo = 0, hi = NCELL - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (c_pref[mid] <= i) lo = mid; else hi = mid - 1;
        }
        cand[i] = __ldg(&g.pts[c_start[lo] + (i - c_pref[lo])]);
      }
    }
    __syncthreads();
    // the group's own 4 x 4 x 4 cells, one warp each
    for (int oc = warp; oc < 64; oc += TT / 32) {
      const int c = ((1 + (oc >> 4)) * SIDE + (1 + ((oc >> 2) & 3))) * SIDE + (1 + (oc & 3));
      const u32 qn = c_count[c];
      if (qn == 0) continue;
      for (u32 q0 = 0; q0 < qn; q0 += 32) {
        const u32 qj = q0 + lane;
        const bool active = qj < qn;
        float4 q = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (active) q = staged ? cand[c_pref[c] + qj] : __ldg(&g.pts[c_start[c] + qj]);
        const u32 qidx = __float_as_uint(q.w);
        const bool live = active && !(MODE == TILE_NORMALS && (qidx & kRemovedBit));
        if (!__any_sync(0xffffffffu, live)) continue;
        // distance from q to its own cell's faces, less a generous rounding
        // slack (pruning only: a pruned cell holds nothing below the K-th)
        float glx, ghx, gly, ghy, glz, ghz;
        {
          const float cs = s_F.cell;
          const int ox = s_base[0] + 1 + (oc & 3), oy = s_base[1] + 1 + ((oc >> 2) & 3),
                    oz = s_base[2] + 1 + (oc >> 4);
          const float fx = s_F.min_x + (float)ox * cs, fy = s_F.min_y + (float)oy * cs,
                      fz = s_F.min_z + (float)oz * cs;
          const float slx = 4e-6f * (fabsf(s_F.min_x) + fabsf(q.x) + (float)(ox + 2) * cs) + 1e-6f;
          const float sly = 4e-6f * (fabsf(s_F.min_y) + fabsf(q.y) + (float)(oy + 2) * cs) + 1e-6f;
          const float slz = 4e-6f * (fabsf(s_F.min_z) + fabsf(q.z) + (float)(oz + 2) * cs) + 1e-6f;
          glx = fmaxf(q.x - fx - slx, 0.0f);
          ghx = fmaxf(fx + cs - q.x - slx, 0.0f);
          gly = fmaxf(q.y - fy - sly, 0.0f);
          ghy = fmaxf(fy + cs - q.y - sly, 0.0f);
          glz = fmaxf(q.z - fz - slz, 0.0f);
          ghz = fmaxf(fz + cs - q.z - slz, 0.0f);
        }
        Key L[K];
#pragma unroll
        for (int j = 0; j < K; ++j) L[j] = kMax;
        Key thr = kMax;
        u32 found = 0;
#pragma unroll 1
        for (int t = 0; t < 27; ++t) {
          const int dx = kRingOrder[t][0], dy = kRingOrder[t][1], dz = kRingOrder[t][2];
          bool take = live;
          if (t > 0) {
            float thr_d2;
            if constexpr (MODE == TILE_SOR_MEAN) thr_d2 = thr;
            else thr_d2 = nbr_d2(thr);
            const float gx = dx < 0 ? glx : (dx > 0 ? ghx : 0.0f);
            const float gy = dy < 0 ? gly : (dy > 0 ? ghy : 0.0f);
            const float gz = dz < 0 ? glz : (dz > 0 ? ghz : 0.0f);
            take = take && !((gx * gx + gy * gy + gz * gz) * (1.0f - 1e-5f) > thr_d2);
          }
          if (!__any_sync(0xffffffffu, take)) continue;
          const int nc = c + (dz * SIDE + dy) * SIDE + dx;
          const u32 cnt = c_count[nc];
          const u32 st = staged ? c_pref[nc] : c_start[nc];
          for (u32 j = 0; j < cnt; ++j) {
            const float4 p = staged ? cand[st + j] : __ldg(&g.pts[st + j]);
            const u32 pidx = __float_as_uint(p.w);
            if (MODE == TILE_NORMALS && (pidx & kRemovedBit)) continue;
            const float d2 = dist2(p.x, p.y, p.z, q.x, q.y, q.z);
            if (take) {
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
        }
        if (!live) continue;
        float tau = -1.0f;
        bool ok = false;
        if (found >= (u32)K) {
          if constexpr (MODE == TILE_SOR_MEAN) tau = L[K - 1];
          else tau = nbr_d2(L[K - 1]);
          const GridFrame F = s_F;
          const Window w1 = ring_window(F, q.x, q.y, q.z, 1, 0);
          const double cov = coverage(F, w1, q.x, q.y, q.z);
          ok = cov > 0.0 && (double)tau < cov * cov * (1.0 - 1e-5);
        }
        const u32 pos = c_start[c] + qj;  // sorted position of the query
        if (!ok) {
          qlevel[pos] = 1;
          qtau[pos] = tau;
          continue;
        }
        if (stats) atomicAdd(stats, 1u);
        if constexpr (MODE == TILE_SOR_MEAN) {
          float sum = 0.0f;
#pragma unroll
          for (int j = 1; j < K; ++j) sum = fadd(sum, __fsqrt_rn(L[j]));
          a.mean[qidx] = fdiv(sum, (float)(K - 1));
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
}

template <int K>
void launch_k(rvp_context *ctx, const GridView &g, int mode, const TileArgs &a, int blocks,
              uint8_t *qlevel, u32 *stats) {
  RVP_CUDA_TRY(cudaMemsetAsync(qlevel, 0, a.n_max, ctx->stream));
  if (mode == TILE_SOR_MEAN)
    k_knn_tile0<K, TILE_SOR_MEAN><<<blocks, TT, 0, ctx->stream>>>(g, a, qlevel, a.qtau, stats);
  else if (mode == TILE_NORMALS)
    k_knn_tile0<K, TILE_NORMALS><<<blocks, TT, 0, ctx->stream>>>(g, a, qlevel, a.qtau, stats);
  else
    k_knn_tile0<K, TILE_PAIRS><<<blocks, TT, 0, ctx->stream>>>(g, a, qlevel, a.qtau, stats);
  RVP_LAUNCH_CHECK(ctx);
  for (int level = 1; level < kGridLevels; ++level) {
    u32 *st = stats ? stats + level : nullptr;
    if (mode == TILE_SOR_MEAN)
      k_knn_tile<K, TILE_SOR_MEAN><<<blocks, TT, 0, ctx->stream>>>(g, a, level, qlevel, a.qtau,
                                                                   st);
    else if (mode == TILE_NORMALS)
      k_knn_tile<K, TILE_NORMALS><<<blocks, TT, 0, ctx->stream>>>(g, a, level, qlevel, a.qtau,
                                                                  st);
    else
      k_knn_tile<K, TILE_PAIRS><<<blocks, TT, 0, ctx->stream>>>(g, a, level, qlevel, a.qtau, st);
    RVP_LAUNCH_CHECK(ctx);
  }
}
}  // namespace

bool grid_knn_tile(rvp_context *ctx, const GridView &g, int k, int mode, const TileArgs &a,
                   int blocks, u32 *stats) {
  if (g.mode != KEY_DENSE || !a.qlevel || !a.qtau) return false;
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
