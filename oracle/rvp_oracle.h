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

#ifdef __cplusplus
}
#endif
#endif
