/*
 * CPU restatement of RVPoint's scalar hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is the checker, not the product: only tests/, __graft_entry__.smoke()
 * and bench.py's cpu-baseline leg may load it. It restates, in plain C and in
 * the reference's own operation order (compiled without FP contraction), the
 * scalar code that every *_rvv entry of the reference runs on a non-RISC-V
 * host. Each function names the reference lines it follows. It is pinned
 * against the reference itself (oracle/_ref, built from the reference's own
 * sources) and against the committed fixtures in tests/golden/.
 */
#ifndef RVP_ORACLE_H
#define RVP_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* SpatialHash setInputCloud/build/radiusSearch, one call per query.
 * CSR result: offsets[nq+1]; idx/d2 sorted by (d2, idx) per query.
 * p1/p2 are the hash primes (73856093, 19349663 by default).
 * Returns the total count, or -1 if cap was too small (offsets still valid). */
long long rvo_hash_radius_search(const float *x, const float *y, const float *z,
                                 size_t n, float cell, int64_t p1, int64_t p2,
                                 const float *qx, const float *qy,
                                 const float *qz, size_t nq, float radius,
                                 int max_nn, long long *offsets, int *idx,
                                 float *d2, long long cap);

/* voxel_grid_downsamp_sc order and arithmetic. out: AoS, >= 3*n floats.
 * keys (optional, 3*V ints): voxel (ix, iy, iz) of each output point. */
size_t rvo_voxel_grid(const float *x, const float *y, const float *z, size_t n,
                      float leaf, float *out, int *keys);

/* sor_sc: exact k+1 NN over all points. mean_dists/keep optional (n each). */
size_t rvo_sor_exact(const float *x, const float *y, const float *z, size_t n,
                     int k, float alpha, float *out, float *mean_dists,
                     unsigned char *keep);

/* sor_spatial_hash over a SpatialHash of cell size `cell`. */
size_t rvo_sor_radius(const float *x, const float *y, const float *z, size_t n,
                      float cell, int k, float alpha, float search_radius,
                      float *out, float *mean_dists, unsigned char *keep);

/* normal_estimation_rvv(in, SpatialHash, ...). use_f64: same neighbour sets,
 * but centroid/covariance/Jacobi/flip evaluated in double. */
void rvo_normals_radius(const float *x, const float *y, const float *z,
                        size_t n, float cell, float radius, float vpx,
                        float vpy, float vpz, int iters, int use_f64,
                        float *nx, float *ny, float *nz);

/* normal_estimation_sc: k+1 nearest including self, ties broken by index. */
void rvo_normals_knn(const float *x, const float *y, const float *z, size_t n,
                     int k, float vpx, float vpy, float vpz, int iters,
                     int use_f64, float *nx, float *ny, float *nz);

/* ransac_plane_sc driven by a raw rand() stream (3*max_iters values).
 * counts (optional, max_iters): inlier count per hypothesis, -1 for a
 * duplicate index triple, -2 for a collinear triple. models (optional,
 * 4*max_iters). iters_run (optional): iterations the reference executes. */
int rvo_ransac_plane(const float *x, const float *y, const float *z, size_t n,
                     float thresh, int max_iters, float collinear, float prob,
                     const int *rand_stream, float *model, int *counts,
                     float *models, int *iters_run);

/* extract_plane_inliers_outliers_rvv (scalar branch). */
void rvo_extract_plane(const float *x, const float *y, const float *z,
                       size_t n, const float *model, float thresh,
                       float *inliers, float *outliers, size_t *n_in,
                       size_t *n_out);

/* FP64 oracle for the precision study: covariance of the k+1 nearest
 * (incl. self) about their centroid in double, eigenvector of the smallest
 * eigenvalue by cyclic Jacobi iterated to convergence, flipped towards vp.
 * cond (optional): lambda_max / lambda_min of that covariance. */
void rvo_normals_knn_exact_f64(const float *x, const float *y, const float *z,
                               size_t n, const int *nbr_idx, int kk, float vpx,
                               float vpy, float vpz, double *nx, double *ny,
                               double *nz, double *cond);

/* EuclideanClustering::extract without a searcher
 * (segmentation/euclidean_clustering.cpp:113-189): BFS from the lowest
 * unvisited index over points with squared distance <= tolerance^2,
 * clusters kept when min_size <= size <= max_size, each sorted. CSR output
 * (offsets n + 1, indices n); returns the number of clusters. */
long rvo_euclidean_clusters(const float *x, const float *y, const float *z, size_t n,
                            float tolerance, int min_size, int max_size, long long *offsets,
                            int *indices);

/* Octree (search/octree.cpp:32-94) and PointerOctree
 * (search/pointer_octree.cpp:30-116), kind 0 and 1: the points in the
 * trees' depth-first leaf order (children 0..7, each leaf's points in index
 * order), which is the order of their radiusSearch output. cap, max_depth,
 * eps: setMaxPointsPerLeaf / setMaxDepth / setBuildEpsilon (64, 8, 1e-4). */
void rvo_octree_order(int kind, const float *x, const float *y, const float *z, size_t n,
                      int cap, int max_depth, float eps, int *order);

/* Octree::radiusSearch (octree.cpp:111-143) / PointerOctree::radiusSearch
 * (pointer_octree.cpp:201-240): every point with d2 <= radius^2 in the tree's
 * leaf order, max_nn ignored. CSR as rvo_hash_radius_search; returns the
 * total, or -1 if cap was too small. */
long long rvo_octree_radius_search(int kind, const float *x, const float *y, const float *z,
                                   size_t n, int cap_leaf, int max_depth, float eps,
                                   const float *qx, const float *qy, const float *qz,
                                   size_t nq, float radius, long long *offsets, int *idx,
                                   float *d2, long long cap);

/* std::nth_element on floats as libstdc++ (GCC 13) does it: introselect
 * with median-of-three pivots, heap selection when the depth limit
 * 2 * floor(log2 n) runs out, insertion sort of the last range of <= 3.
 * Returns 1 if the heap selection ran. */
int rvo_nth_element(float *a, size_t n, size_t nth);

/* sor_octree (kind 0, statistical_outlier_removal.cpp:220-244: all
 * neighbours in the radius, sorted) and sor_pointer_octree (kind 1,
 * :272-301: nth_element on the tree-ordered distances), then
 * filter_by_mean_dists. mean_dists/keep optional. */
size_t rvo_sor_octree(int kind, const float *x, const float *y, const float *z, size_t n,
                      int cap_leaf, int max_depth, float eps, int k, float alpha,
                      float search_radius, float *out, float *mean_dists, unsigned char *keep);

/* normal_estimation_rvv(in, Octree / PointerOctree, ...) (normal_estimation
 * .cpp:155-187, 216-244): neighbours = the tree's radiusSearch, in its order. */
void rvo_normals_octree(int kind, const float *x, const float *y, const float *z, size_t n,
                        int cap_leaf, int max_depth, float eps, float radius, float vpx,
                        float vpy, float vpz, int iters, float *nx, float *ny, float *nz);

/* The k+1 (= kk) nearest of every point, self included, by brute force,
 * ordered by (d2, idx): idx and d2 hold n * kk entries each. */
void rvo_knn_lists(const float *x, const float *y, const float *z, size_t n, int kk,
                   int *idx, float *d2);

#ifdef __cplusplus
}
#endif
#endif
