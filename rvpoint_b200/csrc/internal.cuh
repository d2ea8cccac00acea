// Internal declarations of the rvpoint_b200 CUDA library (sm_100a).
//
// Layout in HBM (all frames of a batch back to back):
//   * input clouds: SoA float x[], y[], z[] (what the reference's
//     PointCloudSoA views, core/point_types.h:24-29);
//   * grid: points re-ordered by cell key into float4 {x, y, z, idx-bits}
//     (16 B, one vector load per candidate), bucket table of
//     {key, start | count<<32} entries (one 16 B load per probe);
//   * outputs: AoS PointXYZ (12 B) like the reference's PointXYZ* out.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/rvpoint_b200.h"

namespace rvp {

typedef unsigned long long u64;
typedef unsigned int u32;

constexpr u64 kEmptyKey = 0xFFFFFFFFFFFFFFFFull;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct Error {
  rvp_status status;
  std::string msg;
};

#define RVP_CUDA_TRY(expr)                                                   \
  do {                                                                       \
    cudaError_t e_ = (expr);                                                 \
    if (e_ != cudaSuccess)                                                   \
      throw ::rvp::Error{e_ == cudaErrorMemoryAllocation ? RVP_ERR_OOM        \
                                                          : RVP_ERR_CUDA,    \
                         std::string(#expr) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

#define RVP_REQUIRE(cond, msg)                                  \
  do {                                                          \
    if (!(cond)) throw ::rvp::Error{RVP_ERR_INVALID_ARG, (msg)}; \
  } while (0)

// ---------------------------------------------------------------------------
// device buffers
// ---------------------------------------------------------------------------
struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  void reserve(size_t b);  // grow-only; contents are not preserved
  void release();
  template <class T>
  T *as() const { return static_cast<T *>(ptr); }
};

struct HostBuf {  // pinned
  void *ptr = nullptr;
  size_t bytes = 0;
  void reserve(size_t b);
  void release();
  template <class T>
  T *as() const { return static_cast<T *>(ptr); }
};

struct Grid;
struct VoxelWork;
}  // namespace rvp

struct rvp_context {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  std::string last_error;
  unsigned long long launches = 0;
  // scratch owned by one-shot entry points (grow-only, reused across calls)
  rvp::DevBuf scratch[32];  // 0-23 one-shot entry points, 24-27 batched RANSAC
  rvp::HostBuf pinned[4];
  rvp::Grid *grid = nullptr;        // grid reused by one-shot kNN entry points
  rvp::VoxelWork *vwork = nullptr;  // voxel scratch of rvp_voxel_grid
};

namespace rvp {

inline void count_launch(rvp_context *ctx) {
  ctx->launches++;
}

#define RVP_LAUNCH_CHECK(ctx)                                             \
  do {                                                                    \
    ::rvp::count_launch(ctx);                                             \
    cudaError_t e_ = cudaGetLastError();                                  \
    if (e_ != cudaSuccess)                                                \
      throw ::rvp::Error{RVP_ERR_CUDA,                                    \
                         std::string("kernel launch: ") + cudaGetErrorString(e_)}; \
  } while (0)

inline unsigned grid_for(size_t n, int threads, int cap_blocks) {
  size_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (cap_blocks > 0 && b > (size_t)cap_blocks) b = (size_t)cap_blocks;
  return (unsigned)b;
}

// ---------------------------------------------------------------------------
// exact IEEE single-precision helpers: the reference is compiled without FP
// contraction, so every product and sum is rounded on its own.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// d2 = dx*dx + dy*dy + dz*dz with dx = p - q (rvv_common.cpp:37-41)
__device__ __forceinline__ float dist2(float px, float py, float pz, float qx,
                                       float qy, float qz) {
  const float dx = fsub(px, qx), dy = fsub(py, qy), dz = fsub(pz, qz);
  return fadd(fadd(fmul(dx, dx), fmul(dy, dy)), fmul(dz, dz));
}

// (d2, idx) packed so that unsigned order == std::pair<float,int> order for
// d2 >= 0 and idx >= 0 (spatial_hashing.cpp:149-154).
__device__ __forceinline__ u64 pack_nbr(float d2, int idx) {
  return ((u64)__float_as_uint(d2) << 32) | (u64)(u32)idx;
}
__device__ __forceinline__ float nbr_d2(u64 k) { return __uint_as_float((u32)(k >> 32)); }
__device__ __forceinline__ int nbr_idx(u64 k) { return (int)(u32)(k & 0xFFFFFFFFull); }

__device__ __forceinline__ u64 mix64(u64 k) {  // splitmix64 finaliser
  k ^= k >> 30;
  k *= 0xbf58476d1ce4e5b9ull;
  k ^= k >> 27;
  k *= 0x94d049bb133111ebull;
  k ^= k >> 31;
  return k;
}

// float atomics on ordered int images (valid for non-NaN values)
__device__ __forceinline__ void atomic_min_f(float *a, float v) {
  if (v >= 0.0f) atomicMin((int *)a, __float_as_int(v));
  else atomicMax((unsigned *)a, __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_f(float *a, float v) {
  if (v >= 0.0f) atomicMax((int *)a, __float_as_int(v));
  else atomicMin((unsigned *)a, __float_as_uint(v));
}

// ---------------------------------------------------------------------------
// radix sort (radix_sort.cu): stable LSD sort of (u64 key, u32 value) pairs,
// 8-bit digits. Digits that are constant over all keys are skipped (the
// global digit histogram shows it), so keys only pay for their live bits.
// n may live on the device (n_dev) for graph capture; n_max sizes the grid.
// ---------------------------------------------------------------------------
struct SortTemp {
  u64 *keys_alt = nullptr;
  u32 *vals_alt = nullptr;
  u32 *tile_hist = nullptr;    // 256 x tiles(n_max)
  u32 *global_hist = nullptr;  // 256 digit totals of the current pass
  int *pass_info = nullptr;    // OR and AND of all keys (2 x u64)
};
size_t sort_temp_bytes(size_t n_max);
void sort_temp_carve(SortTemp &t, void *base, size_t n_max);
void radix_sort_pairs(rvp_context *ctx, u64 *keys, u32 *vals, size_t n_max,
                      const u64 *n_dev, const SortTemp &t);

// exclusive scan of u32/u64 flags -> u64 offsets (scan.cu). n may be on the
// device. out[n] receives the total. temp: scan_temp_bytes(n_max).
size_t scan_temp_bytes(size_t n_max);
void exclusive_scan_u32_to_u64(rvp_context *ctx, const u32 *in, u64 *out,
                               size_t n_max, const u64 *n_dev, void *temp);
// `batch` such scans at once (array b at in + b in_stride, out + b
// out_stride, elements); temp: batch * scan_temp_bytes(n_max)
void exclusive_scan_u32_to_u64_batch(rvp_context *ctx, const u32 *in, size_t in_stride, u64 *out,
                                     size_t out_stride, int batch, size_t n_max,
                                     const u64 *n_dev, void *temp);

// ---------------------------------------------------------------------------
// cell grid (grid.cu)
// ---------------------------------------------------------------------------
struct GridFrame {  // per-frame grid parameters (device)
  float min_x, min_y, min_z;
  float cell;
  int gx, gy, gz;    // fine cells per axis
  int g3x, g3y, g3z; // level-3 cells (64 x 64 x 64 fine cells) per axis
  u64 key_base;      // dense mode: frame's first key (a multiple of 2^18)
};

enum KeyMode { KEY_REF_HASH = 0, KEY_DENSE = 1 };
// The dense grid is a binary hierarchy: a level-L cell is 2 x 2 x 2 level-(L-1)
// cells (edge c * 2^L); the bucket table holds levels 0 .. kGridLevels - 1
// (c .. 16c), and the run starts of one level more are kept (kHeadLevels).
constexpr int kGridLevels = RVP_GRID_LEVELS;
constexpr int kHeadLevels = kGridLevels + 1;
// The neighbour searches of a batch run on three levels 4x apart (cells of
// c, 4c, 16c: table levels lbase, lbase + 2, lbase + 4), one query per
// lane on each in turn; a grid may be sorted finer than its query cell
// (lbase > 0) so that consecutive points lie close together inside a cell.
constexpr int kChainLevels = 3;
constexpr int kChainStep = 2;
// timed kernels per search stage: the three chain levels and the cooperative pass
constexpr int kTimedKernels = kChainLevels + 1;

struct GridView {  // what the query kernels read
  const float4 *pts;       // cell-sorted {x,y,z,idx}
  const ulonglong2 *table; // {key, start | count<<32}
  u64 table_mask;
  const GridFrame *frames; // per frame
  const u64 *frame_pt_begin;  // per frame: first sorted position
  int mode;
  long long p1, p2;        // mode 0 primes
  const u32 *lstart[kHeadLevels];  // dense mode: first sorted position of each level-L bucket
  const u64 *n_level;      // dense mode: number of level-L buckets (device, [4])
  const u64 *n_points;     // number of grid points (device; set by grid_build)
  const u32 *pos_of;       // sorted position of each point (by original index)
  int lbase;               // dense mode: the finest table level (query cell = fine cell << lbase)
  // lbase == 2: for every level-lbase cell of kSubMin to kSubMax points
  // (start st), sub_off[st + s] = offset in the cell of the first point of
  // its s-th quarter cell (s: the 6-bit Morton code of the quarter cell in
  // the cell; the cell's points are sorted by it); null otherwise
  const uint16_t *sub_off;
};
constexpr u32 kSubMin = 64, kSubMax = 65535;

struct Grid {
  int n_frames_max = 0;
  size_t n_max = 0;
  size_t table_cap = 0;
  size_t table_cap_req = 0;    // 0: sized from n_max
  int lbase = 0;               // see GridView::lbase
  DevBuf b_keys, b_vals, b_pts, b_table, b_frames, b_begin, b_sort, b_misc, b_lstart, b_pos,
      b_sub;
  u64 *d_n = nullptr;          // number of points (device)
  u64 *d_nbuckets = nullptr;   // buckets per level [kHeadLevels] (device)
  int *d_collision = nullptr;  // mode 0: hash collision detected
  int *d_overflow = nullptr;   // a bucket found no free table slot
  GridView view(int mode, long long p1, long long p2) const;
  void reserve(size_t n_max, int n_frames_max);
  // shrink/grow the bucket table to hold `buckets` entries at load <= 1/2.5
  void fit_table(size_t buckets);
  void release();
};

// Build a grid over frames of SoA points. frame_offsets_dev: n_frames+1
// int64 on the device. cell: cell size (same for all frames). Mode 0 uses the
// reference's bbox/eps/grid formulas and prime hash (single frame).
// base_level (dense mode): the points are sorted by cells of cell / 2^base
// and the table holds levels base .. base + kGridLevels - 1 (cells of cell,
// 2 cell, ...). xyz_aos (optional): the same points interleaved x, y, z
// (one 12-byte gather per point when the grid records are written).
void grid_build(rvp_context *ctx, Grid &g, const float *x, const float *y,
                const float *z, const int64_t *frame_offsets_dev, int n_frames,
                size_t n_points, float cell, int mode, long long p1,
                long long p2, const u64 *n_dev_opt, int base_level = 0,
                const float *xyz_aos = nullptr);

// Query helpers (queries are SoA; query q belongs to frame qframe(q)).
struct QuerySet {
  const float *x, *y, *z;
  size_t n_max;
  const u64 *n_dev;              // optional device count
  const int32_t *frame_of;       // optional: frame of each query (else 0)
  const int32_t *order;          // optional: process queries in this order
  const float *bound = nullptr;  // optional, per slot: known d2 >= the K-th (< 0: none)
};

// radius search, two passes. counts[nq]; then offsets via scan; then fill.
void grid_radius_count(rvp_context *ctx, const GridView &g, const QuerySet &q,
                       float radius, bool ref_window, u32 *counts);
void grid_radius_fill(rvp_context *ctx, const GridView &g, const QuerySet &q,
                      float radius, bool ref_window, const u64 *offsets,
                      int max_nn, u64 *out_pairs, u32 *big_list, u32 *big_count);
void sort_big_segments(rvp_context *ctx, const u64 *offsets, u64 *pairs,
                       const u32 *big_list, const u32 *big_count, u32 max_big);

// exact kNN (k <= 64) with ring expansion / brute force fallback. radius > 0
// bounds the search. skip_flag: candidates whose idx has bit 31 set are
// ignored (points removed by an earlier stage). out: nq * k packed pairs.
// stats (optional, 8 counters): queries certified by the fine ring, by a
// fine tight window, by the coarse ring, by a coarse tight window, by a
// whole-frame scan, and the radius-bounded ones.
// KNN_OUT_SOR_MEAN_LIST: the mean, and out_pairs (as u32 rows of k, one row
// per grid position) receives the grid positions of the k nearest,
// 0xFFFFFFFF past the found
enum KnnOut { KNN_OUT_BY_QUERY = 0, KNN_OUT_BY_SLOT = 1, KNN_OUT_SOR_MEAN = 2,
              KNN_OUT_SOR_MEAN_LIST = 3 };
void grid_knn(rvp_context *ctx, const GridView &g, const QuerySet &q, int k,
              float radius, u64 *out_pairs, int32_t *out_counts, int qpw,
              int block_threads, u32 *stats = nullptr, int out_mode = KNN_OUT_BY_QUERY,
              float *mean = nullptr);

// Tile kNN (dense grids): one block per coarse bucket stages the 6x6x6 fine
// cells around it in shared memory, one thread per query scans its own
// 27-cell ring; queries the ring cannot certify go to `hard` (original
// indices) for grid_knn. Modes: SOR mean, fused reference normals, pairs.
// TILE_SOR_LIST: the SOR mean plus the k nearest in (d2, index) order, kept
// for the normal stage (sor_list: one row of k per grid position, holding
// the neighbours' grid positions)
// TILE_PAIRS_F: the TILE_PAIRS output from float distances with an index
// beside each (per-warp kernels only); a list with equal distances, whose
// order the scan would decide, goes to the hard list for the exact search
enum TileMode { TILE_SOR_MEAN = 0, TILE_NORMALS = 1, TILE_PAIRS = 2, TILE_SOR_LIST = 3,
                TILE_PAIRS_F = 4 };
struct TileArgs {
  const int32_t *frame_of;  // frame of each original index
  float *mean;              // TILE_SOR_MEAN / _LIST: by original index
  u32 *sor_list;            // TILE_SOR_LIST: k indices per original index
  const float *vx, *vy, *vz;  // TILE_NORMALS: coordinates by original index
  const u64 *out_pos;       // TILE_NORMALS: output slot of each original index
  float *nx, *ny, *nz;
  int iters;
  float vpx, vpy, vpz;
  u64 *pairs;               // TILE_PAIRS: by original index, k per row
  int32_t *counts;
  u32 *hard;                // uncertified queries (original indices)
  u32 *hard_count;          // device counter (cleared by the caller)
  float *hard_tau;          // per hard slot: K-th distance bound (< 0: none)
  uint8_t *qlevel;          // per grid point: level at which it is still open
  float *qtau;              // per grid point: K-th distance bound from the level below
  float rfac;               // level-0 first-pass radius = rfac * cell * sqrt(K / own-cell count)
  int level0_warp;          // every level by the barrier-free per-warp kernel
  u32 *open_flags;          // n_max: open-query flags of a level
  u64 *open_pos;            // n_max + 1: their exclusive scan
  u32 *open_list;           // n_max: open queries in grid order
  u64 *open_n;              // device count of open_list
  void *scan_tmp;           // scan_temp_bytes(n_max)
  size_t n_max;             // size of qlevel / qtau
  cudaEvent_t *level_events;  // null, or 2 per timed kernel (chain levels, cooperative pass)
  bool preset_open;         // qlevel already holds 0 (open) / 0xFF (done) per grid point
  int lane_levels;          // chain levels of the per-lane kernels (1..kChainLevels; 0: all)
  int coop;                 // cooperative passes (k_knn_coop) before the per-lane kernels
  u64 *routed;              // optional [2]: queries of the cooperative, adaptive kernels
};
// false if k has no tile instantiation (use grid_knn then)
// Normals of the kept points whose SOR neighbour list (TILE_SOR_LIST, ks per
// point) holds kn kept points; marks the rest open (qlevel 0) and the others
// done (0xFF). False (nothing launched) if kn > ks or kn is not instantiated.
bool normals_from_sor_lists(rvp_context *ctx, const GridView &g, const TileArgs &a, int ks,
                            int kn);
bool grid_knn_tile(rvp_context *ctx, const GridView &g, int k, int mode, const TileArgs &a,
                   int blocks, u32 *stats = nullptr);
// The hard slots that carry a bound tau (TileArgs::hard, hard_tau; n_hard on
// the device): one thread per slot scans the tight window of sqrt(tau) at the
// finest level where it spans at most 27 cells -- exact, since at least K
// points lie within tau. Done slots get hard_tau = kTauDone (grid_knn skips
// them). Outputs as the mode's: SOR mean (+ list row), TILE_NORMALS lists by
// slot (slot_pairs / slot_counts, as KNN_OUT_BY_SLOT), pairs by index.
// False (nothing launched) if k has no instantiation.
constexpr float kTauDone = -2.0f;
// a hard slot with hard_tau = kTauEstimate carries no bound: grid_knn
// estimates a radius from the occupancy of the query's own cells and scans
// the tight window of it (growing it until K points lie within), before
// its rings; at most kEstimateTries windows
constexpr float kTauEstimate = -3.0f;
constexpr int kEstimateTries = 6;
bool grid_knn_tau(rvp_context *ctx, const GridView &g, int k, int mode, const TileArgs &a,
                  const u64 *n_hard, u64 *slot_pairs = nullptr, int32_t *slot_counts = nullptr,
                  u32 *stats = nullptr);

// ---------------------------------------------------------------------------
// voxel grid (voxel.cu)
// ---------------------------------------------------------------------------
struct VoxelWork {
  DevBuf keys, vals, sort, misc, heads;
  void reserve(size_t n_max, int n_frames_max);
  void release();
};
// Writes AoS centroids to out_aos, voxel count per frame prefix to
// out_offsets (n_frames+1, int64), and optionally keys (3 ints per voxel).
void voxel_grid_run(rvp_context *ctx, VoxelWork &w, const float *x,
                    const float *y, const float *z,
                    const int64_t *frame_offsets_dev, int n_frames,
                    size_t n_max, const u64 *n_dev, float inv_leaf,
                    float *out_aos, int64_t *out_offsets, int32_t *out_keys,
                    int *error_flag, float *out_x, float *out_y, float *out_z);

// ---------------------------------------------------------------------------
// SOR (sor.cu)
// ---------------------------------------------------------------------------
// mean distance from sorted kNN lists (k+1 incl. self)
void sor_mean_from_knn(rvp_context *ctx, const u64 *pairs, int kk,
                       const int32_t *counts, size_t n_max, const u64 *n_dev,
                       float *mean, float fallback_radius, bool radius_mode);
// per-frame sequential statistics, keep mask and ordered AoS copy-out
void sor_filter_frames(rvp_context *ctx, const float *x, const float *y,
                       const float *z, const float *mean,
                       const int64_t *frame_offsets_dev, int n_frames,
                       size_t n_max, const u64 *n_dev, float alpha,
                       uint8_t *keep, float *out_aos, int64_t *out_offsets,
                       float *thresh, void *temp, float *out_x, float *out_y,
                       float *out_z, u32 *src_index);
size_t sor_filter_temp_bytes(size_t n_max, int n_frames);
// output slot of every input point (exclusive scan of the keep flags; valid
// for kept points) inside a sor_filter_frames temp buffer
u64 *sor_positions(void *temp, size_t n_max);

// ---------------------------------------------------------------------------
// normals (normals.cu)
// ---------------------------------------------------------------------------
// Normals from neighbour lists (CSR, each sorted by (d2, idx)).
// div_centroid: normal_estimation_sc's "/ (k+1)" instead of "* (1/n)".
void normals_from_lists(rvp_context *ctx, const float *x, const float *y,
                        const float *z, const u64 *pairs, const u64 *offsets,
                        const int32_t *fixed_counts, int fixed_k,
                        size_t n_max, const u64 *n_dev, bool div_centroid,
                        int iters, float vpx, float vpy, float vpz,
                        const float *qx, const float *qy, const float *qz,
                        float *nx, float *ny, float *nz, const u32 *order = nullptr,
                        const u64 *out_pos = nullptr);
void normals_precise(rvp_context *ctx, const float *x, const float *y,
                     const float *z, const u64 *pairs, int kk, size_t n,
                     float vpx, float vpy, float vpz, double cond_fp64,
                     float *nx, float *ny, float *nz, float *cond,
                     uint8_t *used_fp64);

// ---------------------------------------------------------------------------
// RANSAC (ransac.cu)
// ---------------------------------------------------------------------------
struct RansacParams {
  float thresh;
  int max_iters;
  float collinear;
  double log_p;  // log(1 - clamp(p, .5, .9999)), computed on the host
};
// Hypothesis source of ransac_frames. Default (cdf null): the reference's
// rand() stream, i = r % n. Weighted: three candidates of the frame drawn
// with probability proportional to their weight (cdf = per-frame inclusive
// prefix sums over the candidates cand[cand_offs[f] .. cand_offs[f+1]), global
// point indices), from a counter-based generator keyed by seed. targets
// (optional, per frame): stop a frame at the first hypothesis whose count
// reaches its target (the adaptive stop is then off); iters_run = hypotheses
// drawn.
struct RansacSampler {
  const u32 *cand = nullptr;
  const int64_t *cand_offs = nullptr;
  const double *cdf = nullptr;
  u64 seed = 0;
  const int32_t *targets = nullptr;
  // given hypotheses instead of drawn ones: n_models planes per frame (a NaN
  // first coefficient marks an empty slot)
  const float4 *models = nullptr;
  int n_models = 0;
  // start each frame from an earlier best (count and model), not from zero
  const int32_t *best_in = nullptr;
  const float *model_in = nullptr;
};
// One cluster of `cluster` blocks (1-8, fewer if the device cannot hold them)
// per frame over SoA clouds; frame f = [off[f], off[f+1]).
void ransac_frames(rvp_context *ctx, const float *x, const float *y,
                   const float *z, const int64_t *frame_offsets_dev,
                   int n_frames, const int *rand_dev, const RansacParams &p,
                   float *model, int32_t *best, int32_t *iters_run,
                   int32_t *counts_all, bool eval_all,
                   const RansacSampler &smp = RansacSampler{}, int cluster = 1);
// Euclidean clusters of one cloud (cluster.cu): CSR offsets (capacity
// n + 1) and indices (capacity n) on the device, count in n_clusters_dev.
// temp: euclidean_temp_bytes(n). Synchronizes.
size_t euclidean_temp_bytes(size_t n);
void euclidean_clusters_run(rvp_context *ctx, Grid &grid, const float *x, const float *y,
                            const float *z, size_t n, const int64_t *offs_dev, float tolerance,
                            int min_size, int max_size, int64_t *offsets, int32_t *indices,
                            u64 *n_clusters_dev, void *temp);

// Weighted proposal with preemptive rounds: each round draws `draws`
// hypotheses per frame, ranks them by their inliers among the frame's
// candidates and counts the best 32 exactly over all points (strict-greater
// update carried over rounds); a frame stops at its target (smp.targets) or
// after max_rounds. draws_run: hypotheses drawn per frame. scratch:
// preemptive_temp_bytes(n_frames).
void ransac_preemptive(rvp_context *ctx, const float *x, const float *y, const float *z,
                       const int64_t *offs, int n_frames, const RansacSampler &smp, int draws,
                       int max_rounds, const RansacParams &p, float *model, int32_t *best,
                       int32_t *draws_run, void *scratch);
size_t preemptive_temp_bytes(int n_frames);
void extract_plane_run(rvp_context *ctx, const float *x, const float *y,
                       const float *z, size_t n, const float *model_dev,
                       float thresh, float *in_aos, float *out_aos,
                       u64 *counts_dev, void *temp);
size_t extract_temp_bytes(size_t n);

}  // namespace rvp
