/*
 * rvpoint_b200 -- C ABI of the B200 (sm_100a) point-cloud hot path.
 *
 * Every entry point takes plain pointers and sizes; no C++ or torch type
 * crosses this boundary. Pointers are host or device memory as the `mem`
 * argument says (RVP_MEM_HOST: the library stages them through pinned
 * buffers; RVP_MEM_DEVICE: used in place, on the context's stream).
 *
 * Each function names the reference interface it replaces (paths inside
 * Mumu-kun/rvpoint). The C++ drop-in of those interfaces (namespace rvpoint,
 * include/rvpoint/...) is implemented on top of these calls.
 *
 * Errors: every call returns an rvp_status; rvp_last_error() gives the
 * message of the last failure on a context. Degenerate inputs keep the
 * reference's behaviour (empty input -> zero outputs, no error).
 */
#ifndef RVPOINT_B200_H
#define RVPOINT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RVP_API __attribute__((visibility("default")))
#else
#define RVP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  RVP_OK = 0,
  RVP_ERR_INVALID_ARG = 1, /* bad pointer, size or parameter */
  RVP_ERR_OOM = 2,         /* device or pinned allocation failed */
  RVP_ERR_CAPACITY = 3,    /* caller's output buffer too small; *total says how much */
  RVP_ERR_TIMEOUT = 4,     /* reserved for a bounded device-side wait that gives up; no
                              kernel of this version waits on another, so no entry
                              point returns it */
  RVP_ERR_CUDA = 5,        /* CUDA runtime error (message in rvp_last_error) */
  RVP_ERR_NO_DEVICE = 6    /* no CUDA device / kernels not loadable */
} rvp_status;

enum { RVP_MEM_HOST = 0, RVP_MEM_DEVICE = 1 };

typedef struct rvp_context rvp_context;
typedef struct rvp_hash rvp_hash;
typedef struct rvp_pipeline rvp_pipeline;
typedef struct rvp_octree rvp_octree;

/* ---- context ------------------------------------------------------------ */
RVP_API rvp_status rvp_context_create(int device, rvp_context **out);
RVP_API rvp_status rvp_context_destroy(rvp_context *ctx);
/* stream: a cudaStream_t (NULL = legacy default stream). */
RVP_API rvp_status rvp_context_set_stream(rvp_context *ctx, void *stream);
RVP_API rvp_status rvp_context_synchronize(rvp_context *ctx);
RVP_API const char *rvp_last_error(const rvp_context *ctx);
RVP_API const char *rvp_status_string(rvp_status s);
/* Number of kernel launches issued on this context so far. */
RVP_API uint64_t rvp_context_launch_count(const rvp_context *ctx);
/* Library version string. */
RVP_API const char *rvp_version(void);

/* ---- test hooks (no counterpart in the reference) ------------------------- */
/* After `after` more successful device or pinned allocations, every further
 * allocation of the library fails as an out-of-memory would (the entry point
 * returns RVP_ERR_OOM, having freed what it allocated); after < 0 turns the
 * injection off. Process-wide; for tests of the error paths. */
RVP_API rvp_status rvp_debug_fail_allocation(long long after);
/* Bytes of device memory and of pinned host memory the library holds now. */
RVP_API rvp_status rvp_debug_live_bytes(long long *device_bytes, long long *pinned_bytes);

/* ---- SpatialHash: search/spatial_hashing.h:12-53 ------------------------- */
RVP_API rvp_status rvp_hash_create(rvp_context *ctx, rvp_hash **out);
RVP_API rvp_status rvp_hash_destroy(rvp_hash *h);
/* setHashPrimes, spatial_hashing.h:24-27 */
RVP_API rvp_status rvp_hash_set_primes(rvp_hash *h, int64_t p1, int64_t p2);
/* setInputCloud, spatial_hashing.cpp:21-96 (bbox, eps pad, grid dims).
 * The cloud is copied to the device (the reference keeps a pointer). */
RVP_API rvp_status rvp_hash_set_input_cloud(rvp_hash *h, const float *x, const float *y,
                                    const float *z, size_t n, float cell_size,
                                    int mem);
/* build, spatial_hashing.cpp:98-108: radix sort of cell keys, bucket
 * offsets, device hash table of occupied buckets. */
RVP_API rvp_status rvp_hash_build(rvp_hash *h);
/* 1 if two different cells share a hash key under the current primes. */
RVP_API rvp_status rvp_hash_has_collisions(rvp_hash *h, int *out);
/* radiusSearch, spatial_hashing.cpp:110-168, for nq queries at once.
 * CSR result: offsets[nq+1] (int64), indices/dists hold offsets[nq] entries,
 * each query's list sorted by (d2, index) and cut at max_nn when max_nn > 0.
 * dists are squared distances, as in the reference. If the total exceeds
 * capacity, returns RVP_ERR_CAPACITY with *total and offsets filled. */
RVP_API rvp_status rvp_hash_radius_search(rvp_hash *h, const float *qx, const float *qy,
                                  const float *qz, size_t nq, float radius,
                                  int max_nn, int mem, int64_t *offsets,
                                  int32_t *indices, float *dists,
                                  size_t capacity, size_t *total);
/* Exact k nearest neighbours (ties by index) of nq queries, k <= 64.
 * radius > 0 bounds the search (radiusSearch with max_nn = k); radius <= 0
 * searches the whole cloud. indices/dists: nq*k row-major; counts[nq]. */
RVP_API rvp_status rvp_hash_knn(rvp_hash *h, const float *qx, const float *qy,
                        const float *qz, size_t nq, int k, float radius, int mem,
                        int32_t *indices, float *dists, int32_t *counts);

/* ---- voxel grid: filters/voxel_grid.h:14-34 ------------------------------ */
/* voxel_grid_downsamp_{sc,rvv,rvv_v2} (x86 semantics of _sc,
 * voxel_grid_downsamp.cpp:183-213): centroids in (ix, iy, iz) order.
 * out_aos: >= 3*n floats; keys (optional): 3 ints per voxel. */
RVP_API rvp_status rvp_voxel_grid(rvp_context *ctx, const float *x, const float *y,
                          const float *z, size_t n, float leaf_size, int mem,
                          float *out_aos, int32_t *keys, size_t *out_count);

/* ---- SOR: filters/statistical_outlier_removal.h:18-36 -------------------- */
/* sor_sc / sor_rvv (statistical_outlier_removal.cpp:19-63): exact k+1 NN
 * over all points. mean_dists (n floats) and keep (n bytes) optional. */
RVP_API rvp_status rvp_sor(rvp_context *ctx, const float *x, const float *y,
                   const float *z, size_t n, int k, float alpha, int mem,
                   float *out_aos, size_t *out_count, float *mean_dists,
                   uint8_t *keep);
/* sor_spatial_hash (statistical_outlier_removal.cpp:246-270) on the hash's
 * cloud: neighbours = radiusSearch(q, search_radius, k+1). */
RVP_API rvp_status rvp_sor_spatial_hash(rvp_hash *h, int k, float alpha,
                                float search_radius, int mem, float *out_aos,
                                size_t *out_count, float *mean_dists,
                                uint8_t *keep);

/* ---- normals: features/normal_estimation.h:15-34 ------------------------- */
/* normal_estimation_rvv(in, const SpatialHash&, ...) (normal_estimation.cpp
 * :189-214) on the hash's cloud: neighbours = radiusSearch(q, radius). */
RVP_API rvp_status rvp_normals_radius(rvp_hash *h, float radius, float vp_x,
                              float vp_y, float vp_z, int eigen_iters, int mem,
                              float *nx, float *ny, float *nz);
/* normal_estimation_sc (normal_estimation.cpp:72-112): k+1 nearest incl.
 * self (ties by index), centroid divided by k+1. */
RVP_API rvp_status rvp_normals_knn(rvp_context *ctx, const float *x, const float *y,
                           const float *z, size_t n, int k, float vp_x,
                           float vp_y, float vp_z, int eigen_iters, int mem,
                           float *nx, float *ny, float *nz);
/* Precision mode (no reference counterpart; the reference path is
 * rvp_normals_knn): covariance of the k+1 nearest accumulated in FP32 about
 * the query point with compensated sums, eigenvector by converged Jacobi,
 * redone in FP64 when the condition number exceeds cond_fp64. cond (optional)
 * receives the condition estimate; used_fp64 (optional) 1 where FP64 ran. */
RVP_API rvp_status rvp_normals_knn_precise(rvp_context *ctx, const float *x,
                                   const float *y, const float *z, size_t n,
                                   int k, float vp_x, float vp_y, float vp_z,
                                   double cond_fp64, int mem, float *nx,
                                   float *ny, float *nz, float *cond,
                                   uint8_t *used_fp64);

/* ---- RANSAC: segmentation/ransac_plane.h:11-45 --------------------------- */
/* ransac_plane_sc / ransac_plane_rvv (ransac_plane.cpp:55-111).
 * rand_stream: 3*max_iters raw rand() values (the reference's
 * srand(0)/rand() sequence); NULL makes the library draw them from libc and
 * leave libc's generator where the reference would leave it.
 * counts (optional, max_iters ints): per-hypothesis inlier counts, with -1 for
 * repeated indices, -2 for collinear triples; giving it evaluates all
 * hypotheses (no early stop in the evaluation; the result is unchanged). */
RVP_API rvp_status rvp_ransac_plane(rvp_context *ctx, const float *x, const float *y,
                            const float *z, size_t n, float dist_thresh,
                            int max_iters, float collinear_thresh,
                            float probability, const int32_t *rand_stream,
                            int mem, float *model, int *best_count,
                            int *iters_run, int32_t *counts);
/* extract_plane_inliers_outliers_rvv (ransac_plane.cpp:327-383); either
 * output may be NULL (extract_plane_inliers_rvv / _outliers_rvv). */
RVP_API rvp_status rvp_extract_plane(rvp_context *ctx, const float *x, const float *y,
                             const float *z, size_t n, const float *model,
                             float dist_thresh, int mem, float *inliers_aos,
                             float *outliers_aos, size_t *n_inliers,
                             size_t *n_outliers);

/* ---- Euclidean clustering: segmentation/euclidean_clustering.h:17-70 ---- */
/* EuclideanClustering::extract (euclidean_clustering.cpp:113-189, without a
 * neighbour searcher): the connected components of "squared distance <=
 * tolerance^2", listed by their lowest index, each sorted ascending, kept
 * when min_size <= size <= max_size. CSR output: offsets (capacity n + 1,
 * n_clusters + 1 written) and indices (capacity n). */
RVP_API rvp_status rvp_euclidean_clusters(rvp_context *ctx, const float *x, const float *y,
                                          const float *z, size_t n, float tolerance,
                                          int min_size, int max_size, int mem,
                                          int64_t *offsets, int32_t *indices,
                                          size_t *n_clusters);

/* ---- Octree / PointerOctree: search/octree.h:20-48, pointer_octree.h:26-62 */
/* Both trees return every point with squared distance <= radius^2 (max_nn
 * ignored, octree.cpp:111-114), in the tree's depth-first leaf order
 * (children 0..7, each leaf's points by index). The tree is not built as
 * nodes: build gives every point its rank in that order (root box by the
 * tree's epsilon rule, float midpoints, leaves of <= max_points_per_leaf
 * points or at max_depth), and searches sort the grid's radius lists by rank.
 * The cloud is copied to the device (the reference keeps a pointer). */
enum { RVP_OCTREE = 0, RVP_POINTER_OCTREE = 1 };
RVP_API rvp_status rvp_octree_create(rvp_context *ctx, int kind, rvp_octree **out);
RVP_API rvp_status rvp_octree_destroy(rvp_octree *o);
/* setMaxPointsPerLeaf / setMaxDepth / setBuildEpsilon (64, 8, 1e-4 by
 * default; octree.h:33-35). max_depth > 21 is rejected. */
RVP_API rvp_status rvp_octree_set_params(rvp_octree *o, int max_points_per_leaf, int max_depth,
                                         float build_epsilon);
/* setInputCloud (octree.cpp:28-30, pointer_octree.cpp:26-28) */
RVP_API rvp_status rvp_octree_set_input_cloud(rvp_octree *o, const float *x, const float *y,
                                              const float *z, size_t n, int mem);
/* build (octree.cpp:32-57, pointer_octree.cpp:30-69) */
RVP_API rvp_status rvp_octree_build(rvp_octree *o);
/* the points in the tree's leaf order (n ints) */
RVP_API rvp_status rvp_octree_order(rvp_octree *o, int mem, int32_t *order);
/* radiusSearch for nq queries (octree.cpp:111-143, pointer_octree.cpp
 * :201-282 incl. radiusSearchScalar). CSR as rvp_hash_radius_search. */
RVP_API rvp_status rvp_octree_radius_search(rvp_octree *o, const float *qx, const float *qy,
                                            const float *qz, size_t nq, float radius, int mem,
                                            int64_t *offsets, int32_t *indices, float *dists,
                                            size_t capacity, size_t *total);
/* sor_octree (RVP_OCTREE, statistical_outlier_removal.cpp:220-244: sorted
 * distances) / sor_pointer_octree (RVP_POINTER_OCTREE, :272-301: the C++
 * library's nth_element on the tree-ordered distances, as the reference
 * runs it) on the tree's cloud; outputs as rvp_sor_spatial_hash. */
RVP_API rvp_status rvp_sor_octree(rvp_octree *o, int k, float alpha, float search_radius,
                                  int mem, float *out_aos, size_t *out_count, float *mean_dists,
                                  uint8_t *keep);
/* normal_estimation_rvv(in, Octree / PointerOctree, ...) (normal_estimation
 * .cpp:155-187, 216-253) on the tree's cloud: covariance over the tree's
 * radiusSearch list, in its order. */
RVP_API rvp_status rvp_normals_octree(rvp_octree *o, float radius, float vp_x, float vp_y,
                                      float vp_z, int eigen_iters, int mem, float *nx,
                                      float *ny, float *nz);

/* ---- PCD input: io/simple_pcd_loader.h:143-291 ---------------------------- */
/* loadPCD's parsing (ascii, binary, binary_compressed) into SoA x, y, z
 * (device arrays with mem = RVP_MEM_DEVICE: binary records are split on the
 * GPU). *n_points receives the point count; when it exceeds capacity the
 * call returns RVP_ERR_CAPACITY and writes nothing. Synchronizes. */
RVP_API rvp_status rvp_pcd_load(rvp_context *ctx, const char *path, int mem, float *x,
                                float *y, float *z, size_t capacity, size_t *n_points);

/* Largest cloud rvp_extract_plane_noalloc accepts. */
#define RVP_NOALLOC_MAX_POINTS 16777216

/* Inlier / outlier split of rvp_extract_plane for callers that cannot
 * allocate device memory at call time (a control loop that forbids
 * allocation once it runs, a host framework that owns every device
 * allocation). No counterpart in the reference. It allocates nothing: its
 * only scratch, one count per 2048 points (32 KB), is a fixed array inside
 * the library that every GPU loading the library keeps until exit and that
 * all calls on a device share -- calls that run on the GPU at the same time
 * race on it. All pointers are device memory: x, y, z (n floats), model
 * (4 floats), inliers_aos / outliers_aos (3 * n floats each, either may be
 * NULL), counts (2 uint64: inliers, outliers). Asynchronous on the context's
 * stream. The first call on a device looks up the array's device address;
 * make that first call before any stream capture. n above
 * RVP_NOALLOC_MAX_POINTS returns RVP_ERR_INVALID_ARG and launches nothing;
 * errors are reported by the status only (rvp_last_error is not updated). */
RVP_API rvp_status rvp_extract_plane_noalloc(rvp_context *ctx, const float *x,
                                             const float *y, const float *z,
                                             size_t n, const float *model,
                                             float dist_thresh, float *inliers_aos,
                                             float *outliers_aos, uint64_t *counts);

/* ---- batched frames (no single reference counterpart: the chain
 *      voxel_grid_downsamp_rvv_v2 -> sor_rvv -> normal_estimation_sc ->
 *      ransac_plane_rvv of tools/pipeline_export.cpp:351-498, per frame) --- */
typedef struct {
  float leaf_size;       /* voxel leaf (m) */
  int sor_k;             /* SOR neighbours */
  float sor_alpha;       /* SOR std multiplier */
  int normal_k;          /* normals: k+1 nearest incl. self */
  int eigen_iters;       /* Jacobi iterations (reference default 4) */
  float vp_x, vp_y, vp_z;/* viewpoint */
  float ransac_thresh;   /* plane distance threshold */
  int ransac_iters;      /* hypotheses */
  float ransac_collinear;
  float ransac_prob;
  float cell_size;       /* grid cell for the neighbour searches (0 = auto) */
  int block_threads;     /* warp-per-query kNN kernel block size: 32..256, a multiple
                            of 32 (0 = 256) */
  int queries_per_warp;  /* kNN kernel mode: 0 one query per lane at every grid level
                            (default), 1 one warp per query, 2 shared-memory tiles,
                            3 a cooperative level-0 pass (all lanes test the same
                            candidate) before the per-lane kernels */
} rvp_pipeline_config;

RVP_API rvp_status rvp_pipeline_create(rvp_context *ctx, const rvp_pipeline_config *cfg,
                               size_t max_points, int max_frames,
                               rvp_pipeline **out);
RVP_API rvp_status rvp_pipeline_destroy(rvp_pipeline *p);
/* Runs the chain over n_frames frames stored back to back in device memory
 * (frame f = points frame_offsets[f] .. frame_offsets[f+1]). All sizes stay
 * on the device; nothing is copied back. Capturable in a CUDA graph. */
RVP_API rvp_status rvp_pipeline_run_device(rvp_pipeline *p, const float *x,
                                   const float *y, const float *z,
                                   const int64_t *frame_offsets_dev,
                                   int n_frames, size_t n_points);
/* Records one rvp_pipeline_run_device over these device inputs as a CUDA
 * graph (replacing any earlier one) without running it; *kernels (may be
 * NULL) receives the kernel launches one replay makes. The graph keeps the
 * input pointers and n_frames / n_points: new data goes into the same
 * buffers. A tuning change needs a new capture. Run the pipeline once
 * before the first capture, so that every buffer has its final size. */
RVP_API rvp_status rvp_pipeline_capture(rvp_pipeline *p, const float *x,
                                        const float *y, const float *z,
                                        const int64_t *frame_offsets_dev,
                                        int n_frames, size_t n_points,
                                        uint64_t *kernels);
/* Launches the captured run on the context's stream. */
RVP_API rvp_status rvp_pipeline_replay(rvp_pipeline *p);
/* Device pointers to the results of the last run (valid until the next run):
 * voxel_aos/voxel_offsets[n_frames+1], sor_aos/sor_offsets, normals (3 SoA
 * arrays over the SOR points), ransac_model[4*n_frames], ransac_count[n_frames],
 * ransac_iters[n_frames]. */
typedef struct {
  const float *voxel_aos;
  const int64_t *voxel_offsets;
  const float *sor_aos;
  const int64_t *sor_offsets;
  const float *nx, *ny, *nz;
  const float *ransac_model;
  const int32_t *ransac_count;
  const int32_t *ransac_iters;
  const float *sor_mean_dists; /* per voxel point */
} rvp_pipeline_outputs;
RVP_API rvp_status rvp_pipeline_outputs_get(rvp_pipeline *p, rvp_pipeline_outputs *o);
/* Re-size the neighbour grid's bucket table to the bucket count of the last
 * run (with 25% headroom, 2.5 slots per bucket rounded up to a power of two)
 * so it stays resident in L2. Call after a first run, before capturing a
 * graph; a later batch with more buckets than that makes rvp_pipeline_check
 * report RVP_ERR_CAPACITY (refit then). */
RVP_API rvp_status rvp_pipeline_fit_tables(rvp_pipeline *p);
/* RVP_ERR_CAPACITY if the last run's bucket table overflowed (results of
 * that run are then incomplete); synchronizes the stream. */
RVP_API rvp_status rvp_pipeline_check(rvp_pipeline *p);
/* Grid levels of the batched neighbour grid: cells of edge c, 2c, 4c, 8c,
 * 16c (c = the pipeline's cell size). */
#define RVP_GRID_LEVELS 5
/* Queries of the last run's SOR kNN kernels in cooperative mode
 * (queries_per_warp 3; zeros otherwise): out[0] the cooperative pass took
 * (points whose own cell holds at least ceil(rfac^2 k) points), out[1] the
 * adaptive per-thread kernel took (what the cooperative pass left open).
 * out[2]. */
RVP_API rvp_status rvp_pipeline_knn_routed(rvp_pipeline *p, uint64_t *out);
/* Diagnostics: enable != 0 makes the kNN kernels count which search path
 * settled each query: out20[0..7] SOR, [8..15] normals (warp-per-query
 * kernel: first-level ring, tight window of a bound, second-level ring,
 * coarser ring, whole frame; per-lane chain levels 1, 2, 3), [16] SOR and
 * [17] normals settled by the per-thread tight window of a handed-on bound,
 * [18..19] reserved. Reads (if out20) and clears the counters. */
RVP_API rvp_status rvp_pipeline_knn_stats(rvp_pipeline *p, int enable, uint32_t *out20);
/* Host copies of the per-frame voxel and SOR offsets of the last run
 * (n_frames+1 int64 each; either may be NULL). Synchronizes the stream. */
RVP_API rvp_status rvp_pipeline_frame_offsets(rvp_pipeline *p, int64_t *voxel_offsets,
                                              int64_t *sor_offsets);
/* Tunables chosen by the autotuner, applied to the next run without
 * reallocating: grid cell size (m), kNN block size (multiple of 32, 0 =
 * default), queries per warp. A graph captured earlier keeps the values it
 * was captured with. */
RVP_API rvp_status rvp_pipeline_set_tuning(rvp_pipeline *p, float cell_size,
                                           int block_threads, int queries_per_warp);
/* First-pass search radius of the kNN, as a factor of cell * sqrt(k /
 * points in the query's cell); with the cooperative pass (queries_per_warp 3)
 * it takes the queries whose own cell holds at least ceil(rfac^2 k) points
 * (0 disables the first pass of the per-lane kernels; results never depend on
 * it, only the work does). */
RVP_API rvp_status rvp_pipeline_set_search_radius_factor(rvp_pipeline *p, float rfac);
/* Levels of the kNN chain (cells of c, 4c and 16c: 1 to 3; 0 = all 3) that
 * run one query per lane; the queries still open after them go to the
 * warp-per-query kernel, which spreads a query's candidates over the lanes.
 * Results never depend on it. */
RVP_API rvp_status rvp_pipeline_set_lane_levels(rvp_pipeline *p, int levels);
/* Stage timing with CUDA events on the context's stream: the next max_runs
 * runs record 8 events each (stage boundaries: voxel, grid build, SOR kNN,
 * SOR statistics, normals kNN, normals, RANSAC), plus a pair around each
 * timed kNN kernel. rvp_pipeline_stage_times synchronizes and returns the
 * mean ms per stage over the recorded runs (ms[0..6]); with n_stages >= 15
 * also the mean ms of the timed kNN kernels (ms[7..10] SOR: the per-lane
 * kernels on cells of c, 4c and 16c, then the cooperative pass; ms[11..14]
 * the same for the normals). It then resets. max_runs = 0 turns timing off. */
RVP_API rvp_status rvp_pipeline_set_timing(rvp_pipeline *p, int max_runs);
RVP_API rvp_status rvp_pipeline_stage_times(rvp_pipeline *p, float *ms, int n_stages,
                                            int *runs);
/* Host entry: copies host frames in, runs, copies the per-frame results out
 * (any output pointer may be NULL). Output arrays are sized by max_points /
 * n_frames; *_offsets are n_frames+1 entries. The voxel results are copied
 * out while SOR and the normals run, the SOR results while the normals and
 * RANSAC run (asynchronous when the host buffers are pinned). */
RVP_API rvp_status rvp_pipeline_run_host(rvp_pipeline *p, const float *x, const float *y,
                                 const float *z, const int64_t *frame_offsets,
                                 int n_frames, float *voxel_aos,
                                 int64_t *voxel_offsets, float *sor_aos,
                                 int64_t *sor_offsets, float *nx, float *ny,
                                 float *nz, float *ransac_model,
                                 int32_t *ransac_count);
/* rvp_pipeline_run_host over n_batches batches in a row (every argument an
 * array of n_batches entries; output entries may be NULL). Batch i + 1 goes
 * up into a second device input set while batch i runs, and batch i's
 * results come down while batch i + 1 runs, so the copies hide behind the
 * work; outputs are the ones rvp_pipeline_run_host writes, bit for bit.
 * Host arrays should be pinned for the copies to overlap. Synchronizes at
 * the end. */
RVP_API rvp_status rvp_pipeline_run_host_batches(
    rvp_pipeline *p, int n_batches, const float *const *x, const float *const *y,
    const float *const *z, const int64_t *const *frame_offsets, const int *n_frames,
    float *const *voxel_aos, int64_t *const *voxel_offsets, float *const *sor_aos,
    int64_t *const *sor_offsets, float *const *nx, float *const *ny, float *const *nz,
    float *const *ransac_model, int32_t *const *ransac_count);
/* Copies the results of the last run (run_device, replay or run_host) of
 * the last n_frames to host arrays, sized and laid out as for
 * rvp_pipeline_run_host (any pointer may be NULL); synchronizes. */
RVP_API rvp_status rvp_pipeline_copy_outputs(rvp_pipeline *p, float *voxel_aos,
                                             int64_t *voxel_offsets, float *sor_aos,
                                             int64_t *sor_offsets, float *nx, float *ny,
                                             float *nz, float *ransac_model,
                                             int32_t *ransac_count);

/* ---------------------------------------------------------------------------
 * Batched plain RANSAC and the learned hypothesis proposal. None of these
 * has a reference counterpart except rvp_ransac_frames, which is
 * ransac_plane_rvv (segmentation/ransac_plane.cpp:116-199, scalar branch
 * :55-111) applied to every frame of a batch. All pointers are device
 * pointers on the context's stream. rvp_ransac_frames (which restores
 * libc's generator), rvp_mlp_gradients, the parameter calls and a
 * rvp_mlp_train_step asked for its loss synchronize; the others only queue
 * work. Scratch is kept in the context between calls.
 * ------------------------------------------------------------------------- */
#define RVP_MLP_INPUTS 8
#define RVP_MLP_HIDDEN 64
/* W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3: 4801 floats */
#define RVP_MLP_PARAMS 4801

/* ransac_plane_rvv on every frame (one srand(0) stream shared by all, as
 * each reference call restarts it; libc's generator is left as the last
 * frame's call leaves it). targets (optional, per frame): stop a frame at
 * the first hypothesis whose inlier count reaches its target, with the
 * adaptive stop off; iters_run then counts the hypotheses drawn. */
RVP_API rvp_status rvp_ransac_frames(rvp_context *ctx, const float *x, const float *y,
                                     const float *z, const int64_t *frame_offsets_dev,
                                     int n_frames, int max_iters, float dist_thresh,
                                     float collinear_thresh, float probability,
                                     const int32_t *targets, float *models, int32_t *best,
                                     int32_t *iters_run);
/* RANSAC whose three points are drawn from each frame's candidates
 * (cand[cand_offsets[f] .. cand_offsets[f+1]), global point indices inside
 * frame f; n_cand = cand_offsets[n_frames]) with probability proportional to their weight, from a
 * counter-based generator keyed by seed. weights: one per candidate, used
 * as given (negatives as 0) when logit_power is 0, else taken as logits and
 * turned into sigmoid(w) ^ logit_power. Counting, model and the
 * strict-greater update are ransac_plane_rvv's. */
RVP_API rvp_status rvp_ransac_weighted(rvp_context *ctx, const float *x, const float *y,
                                       const float *z, const int64_t *frame_offsets_dev,
                                       int n_frames, const uint32_t *cand,
                                       const int64_t *cand_offsets_dev, size_t n_cand,
                                       const float *weights, float logit_power,
                                       uint64_t seed, int max_iters,
                                       float dist_thresh,
                                       float collinear_thresh, float probability,
                                       const int32_t *targets, float *models, int32_t *best,
                                       int32_t *iters_run);
/* The weighted proposal in preemptive rounds: the first round draws `draws`
 * (<= 512) hypotheses per frame from its candidates (at most 2048 per
 * frame) by weight, ranks them by their inliers among the candidates, and
 * counts the best 32 exactly over all of the frame's points; each later
 * round draws 2 * draws and counts the best 64 (the same share), keeping the
 * best exact count with the strict-greater rule across rounds. A frame stops
 * when its count reaches its target (targets, optional) or after max_rounds;
 * draws_run receives the hypotheses drawn per frame. weights as for
 * rvp_ransac_weighted. */
RVP_API rvp_status rvp_ransac_preemptive(rvp_context *ctx, const float *x, const float *y,
                                         const float *z, const int64_t *frame_offsets_dev,
                                         int n_frames, const uint32_t *cand,
                                         const int64_t *cand_offsets_dev, size_t n_cand,
                                         const float *weights, float logit_power, uint64_t seed,
                                         int draws, int max_rounds, float dist_thresh,
                                         float collinear_thresh, const int32_t *targets,
                                         float *models, int32_t *best, int32_t *draws_run);
/* labels[i] = 1 if point i lies within dist_thresh of its frame's model
 * (models: 4 floats per frame), else 0. */
RVP_API rvp_status rvp_plane_labels(rvp_context *ctx, const float *x, const float *y,
                                    const float *z, const int64_t *frame_offsets_dev,
                                    int n_frames, size_t n_points, const float *models,
                                    float dist_thresh, float *labels);

typedef struct rvp_scorer rvp_scorer;
RVP_API rvp_status rvp_scorer_create(rvp_context *ctx, size_t max_points, int max_frames,
                                     rvp_scorer **out);
RVP_API rvp_status rvp_scorer_destroy(rvp_scorer *s);
/* Eight features per candidate (all points if cand is NULL) from its k = 16
 * nearest neighbours within its frame: |normal| (3), curvature, planarity,
 * log of the 16th-neighbour distance r, distance to the local plane / r,
 * distance to the neighbourhood centroid / r. features: n_cand x 8.
 * neighbours = 0: among all of the frame's points; 1: among the frame's
 * candidates only (cand_offsets_dev: n_frames + 1 offsets into cand; a
 * coarser neighbourhood for far less kNN work). */
RVP_API rvp_status rvp_scorer_features(rvp_scorer *s, const float *x, const float *y,
                                       const float *z, const int64_t *frame_offsets_dev,
                                       int n_frames, size_t n_points, float cell_size,
                                       const uint32_t *cand, const int64_t *cand_offsets_dev,
                                       size_t n_cand, int neighbours, float *features);
/* kNN kernels of the features among the candidates (neighbours = 1):
 * queries_per_warp 0 one query per lane (default), 3 a cooperative first
 * pass over the grid's finest level with the bound rfac * cell *
 * sqrt(17 / own-cell count) (rfac > 0), the per-lane kernels after it. The
 * features do not depend on the choice. */
RVP_API rvp_status rvp_scorer_set_knn(rvp_scorer *s, int queries_per_warp, float rfac);
/* Parameters (host arrays): FP32 master weights, RVP_MLP_PARAMS floats;
 * the network computes with their BF16 rounding. set_params resets the
 * optimiser. set_norm: per-feature mean and standard deviation applied
 * before the first layer. */
RVP_API rvp_status rvp_mlp_set_params(rvp_scorer *s, const float *params);
RVP_API rvp_status rvp_mlp_get_params(rvp_scorer *s, float *params);
RVP_API rvp_status rvp_mlp_set_norm(rvp_scorer *s, const float *mean, const float *stddev);
/* logits[i] of features[i] (n x 8), device arrays. */
RVP_API rvp_status rvp_mlp_forward(rvp_scorer *s, const float *features, size_t n,
                                   float *logits);
/* Mean binary cross-entropy of the logits against labels (0/1 floats) and
 * its gradient w.r.t. the parameters (host, RVP_MLP_PARAMS floats). */
RVP_API rvp_status rvp_mlp_gradients(rvp_scorer *s, const float *features, const float *labels,
                                     size_t n, float *grad, double *loss);
/* One Adam step (beta 0.9 / 0.999) on that loss over all n rows, or, with
 * batch > 0, over a minibatch of `batch` rows drawn uniformly with
 * replacement (a counter-based generator keyed by seed and the step count).
 * loss (host, may be NULL) receives the loss before the step. */
RVP_API rvp_status rvp_mlp_train_step(rvp_scorer *s, const float *features, const float *labels,
                                      size_t n, size_t batch, uint64_t seed, float lr,
                                      double *loss);

#ifdef __cplusplus
}
#endif
#endif /* RVPOINT_B200_H */
