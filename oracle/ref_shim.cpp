// Test infrastructure only (the checker). This file is compiled together with
// the UNMODIFIED reference sources (src/**/*.cpp of Mumu-kun/rvpoint) into
// oracle/_ref/librvpoint_ref.so by oracle/Makefile. It adds nothing but a
// plain extern "C" surface so Python tests and bench.py's CPU-baseline leg can
// call the reference's own scalar path through ctypes. Every function below is
// a thin forwarder: all arithmetic happens inside the reference's code.
//
// Built with -O3 -std=c++17 -ffp-contract=off and WITHOUT -march=native:
// FMA contraction would change the bits of d^2 and of the plane distance.

#include "core/point_types.h"
#include "search/spatial_hashing.h"
#include "filters/voxel_grid.h"
#include "filters/statistical_outlier_removal.h"
#include "features/normal_estimation.h"
#include "segmentation/ransac_plane.h"
#include "segmentation/euclidean_clustering.h"
#include "io/simple_pcd_loader.h"
#include "search/octree.h"
#include "search/pointer_octree.h"

#include <algorithm>

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

using namespace rvpoint;

namespace {
PointCloudSoA soa(const float *x, const float *y, const float *z, size_t n) {
  PointCloudSoA c;
  c.x = const_cast<float *>(x);
  c.y = const_cast<float *>(y);
  c.z = const_cast<float *>(z);
  c.n = n;
  return c;
}
}  // namespace

extern "C" {

// SpatialHash::setInputCloud + build + radiusSearch for every query
// (spatial_hashing.cpp:21-168). CSR output: offsets[nq+1]; idx/d2 hold
// offsets[nq] entries. Returns -1 when cap is too small (offsets still valid).
long long ref_hash_radius_search(const float *x, const float *y, const float *z,
                                 size_t n, float cell, const float *qx,
                                 const float *qy, const float *qz, size_t nq,
                                 float radius, int max_nn, long long *offsets,
                                 int *idx, float *d2, long long cap) {
  SpatialHash h;
  h.setInputCloud(soa(x, y, z, n), cell);
  h.build();
  std::vector<int> ind;
  std::vector<float> dd;
  long long tot = 0;
  bool overflow = false;
  offsets[0] = 0;
  for (size_t q = 0; q < nq; ++q) {
    PointXYZ p{qx[q], qy[q], qz[q]};
    size_t c = h.radiusSearch(p, radius, ind, dd, max_nn);
    if (!overflow && tot + (long long)c <= cap) {
      std::memcpy(idx + tot, ind.data(), c * sizeof(int));
      std::memcpy(d2 + tot, dd.data(), c * sizeof(float));
    } else {
      overflow = true;
    }
    tot += (long long)c;
    offsets[q + 1] = tot;
  }
  return overflow ? -1 : tot;
}

// voxel_grid_downsamp_rvv_v2 (voxel_grid_downsamp.cpp:284-335; on x86 it
// falls through to voxel_grid_downsamp_sc :183-213). out: AoS [3*n].
size_t ref_voxel_grid(const float *x, const float *y, const float *z, size_t n,
                      float leaf, float *out) {
#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wdeprecated-declarations"
  return voxel_grid_downsamp_rvv_v2(soa(x, y, z, n),
                                    reinterpret_cast<PointXYZ *>(out), leaf);
#pragma GCC diagnostic pop
}

// sor_rvv (statistical_outlier_removal.cpp:68-190 -> sor_sc :19-63 on x86).
size_t ref_sor_rvv(const float *x, const float *y, const float *z, size_t n,
                   int k, float alpha, float *out) {
  return sor_rvv(soa(x, y, z, n), reinterpret_cast<PointXYZ *>(out), k, alpha);
}

// sor_spatial_hash (statistical_outlier_removal.cpp:246-270) over a
// SpatialHash built with cell size `cell`.
size_t ref_sor_spatial_hash(const float *x, const float *y, const float *z,
                            size_t n, float cell, int k, float alpha,
                            float search_radius, float *out) {
  PointCloudSoA c = soa(x, y, z, n);
  SpatialHash h;
  h.setInputCloud(c, cell);
  h.build();
  return sor_spatial_hash(c, h, reinterpret_cast<PointXYZ *>(out), k, alpha,
                          search_radius);
}

// normal_estimation_rvv(in, SpatialHash, ...) (normal_estimation.cpp:189-214).
void ref_normals_hash(const float *x, const float *y, const float *z, size_t n,
                      float cell, int k, float radius, float vpx, float vpy,
                      float vpz, int iters, float *nx, float *ny, float *nz) {
  PointCloudSoA c = soa(x, y, z, n);
  SpatialHash h;
  h.setInputCloud(c, cell);
  h.build();
  normal_estimation_rvv(c, h, nx, ny, nz, k, radius, vpx, vpy, vpz, iters);
}

// normal_estimation_sc (normal_estimation.cpp:72-112): brute-force k+1 NN.
void ref_normals_sc(const float *aos, size_t n, int k, float radius, float vpx,
                    float vpy, float vpz, int iters, float *nx, float *ny,
                    float *nz) {
  normal_estimation_sc(reinterpret_cast<const PointXYZ *>(aos), n, nx, ny, nz,
                       k, radius, vpx, vpy, vpz, iters);
}

// ransac_plane_rvv (ransac_plane.cpp:116-199 -> ransac_plane_sc :55-111).
int ref_ransac_plane(const float *x, const float *y, const float *z, size_t n,
                     float thresh, int max_iters, float collinear, float prob,
                     float *model) {
  return ransac_plane_rvv(soa(x, y, z, n), thresh, max_iters, model, collinear,
                          prob);
}

// extract_plane_inliers_outliers_rvv (ransac_plane.cpp:327-383).
void ref_extract_plane(const float *x, const float *y, const float *z, size_t n,
                       const float *model, float thresh, float *inliers,
                       float *outliers, size_t *n_in, size_t *n_out) {
  size_t a = 0, b = 0;
  extract_plane_inliers_outliers_rvv(
      soa(x, y, z, n), model, thresh, reinterpret_cast<PointXYZ *>(inliers),
      reinterpret_cast<PointXYZ *>(outliers), a, b);
  *n_in = a;
  *n_out = b;
}

// extract_plane_inliers_rvv (ransac_plane.cpp:234-278): inlier count of one
// plane model, used to pin per-hypothesis inlier counts.
size_t ref_count_plane_inliers(const float *x, const float *y, const float *z,
                               size_t n, const float *model, float thresh,
                               float *scratch_aos) {
  return extract_plane_inliers_rvv(soa(x, y, z, n), model, thresh,
                                   reinterpret_cast<PointXYZ *>(scratch_aos));
}

// EuclideanClustering::extract (euclidean_clustering.cpp:113-189) without a
// neighbour searcher. CSR output: offsets[n_clusters+1] and indices; returns
// the number of clusters (offsets / indices sized by the caller: n + 1, n).
long ref_euclidean_clusters(const float *x, const float *y, const float *z, size_t n,
                            float tolerance, int min_size, int max_size, long long *offsets,
                            int *indices) {
  const PointCloudSoA c = soa(x, y, z, n);
  EuclideanClustering ec;
  ec.setInputCloud(c);
  ec.setClusterTolerance(tolerance);
  ec.setMinClusterSize(min_size);
  ec.setMaxClusterSize(max_size);
  const std::vector<ClusterIndices> cl = ec.extract();
  long long o = 0;
  offsets[0] = 0;
  for (size_t k = 0; k < cl.size(); ++k) {
    for (int i : cl[k].indices) indices[o++] = i;
    offsets[k + 1] = o;
  }
  return (long)cl.size();
}

// loadPCD (io/simple_pcd_loader.h:143-291): AoS points into out (capacity
// cap); returns the reference's count (-1 on failure).
long ref_load_pcd(const char *path, float *out, size_t cap) {
  std::vector<PointXYZ> pts;
  const int k = loadPCD(path, pts);
  if (k < 0) return k;
  for (size_t i = 0; i < pts.size() && i < cap; ++i) {
    out[3 * i + 0] = pts[i].x;
    out[3 * i + 1] = pts[i].y;
    out[3 * i + 2] = pts[i].z;
  }
  return (long)pts.size();
}

// savePCD / savePCDRGB (io/simple_pcd_loader.h:295-386)
void ref_save_pcd(const char *path, const float *aos, size_t n, int binary) {
  std::vector<PointXYZ> pts(n);
  for (size_t i = 0; i < n; ++i) pts[i] = {aos[3 * i], aos[3 * i + 1], aos[3 * i + 2]};
  savePCD(path, pts, binary != 0);
}

void ref_save_pcd_rgb(const char *path, const float *aos, const unsigned char *rgb, size_t n,
                      int binary) {
  std::vector<PointXYZRGB> pts(n);
  for (size_t i = 0; i < n; ++i)
    pts[i] = {aos[3 * i], aos[3 * i + 1], aos[3 * i + 2], rgb[3 * i], rgb[3 * i + 1],
              rgb[3 * i + 2]};
  savePCDRGB(path, pts, binary != 0);
}

// Octree (kind 0), PointerOctree::radiusSearch (kind 1) and
// PointerOctree::radiusSearchScalar (kind 2) for every query; the trees'
// parameters through their setters. Returns the total (entries past
// capacity are dropped).
long ref_octree_radius(int kind, const float *x, const float *y, const float *z, size_t n,
                       int cap, int depth, float eps, const float *qx, const float *qy,
                       const float *qz, size_t nq, float radius, int64_t *offsets,
                       int32_t *idx, float *d2, size_t capacity) {
  const PointCloudSoA c = soa(x, y, z, n);
  Octree ot;
  PointerOctree pt;
  if (kind == 0) {
    ot.setMaxPointsPerLeaf(cap);
    ot.setMaxDepth(depth);
    ot.setBuildEpsilon(eps);
    ot.setInputCloud(c);
    ot.build();
  } else {
    pt.setMaxPointsPerLeaf(cap);
    pt.setMaxDepth(depth);
    pt.setBuildEpsilon(eps);
    pt.setInputCloud(c);
    pt.build();
  }
  std::vector<int> ind;
  std::vector<float> dst;
  size_t tot = 0;
  offsets[0] = 0;
  for (size_t q = 0; q < nq; ++q) {
    PointXYZ p{qx[q], qy[q], qz[q]};
    if (kind == 0) ot.radiusSearch(p, radius, ind, dst);
    else if (kind == 1) pt.radiusSearch(p, radius, ind, dst);
    else pt.radiusSearchScalar(p, radius, ind, dst);
    for (size_t t = 0; t < ind.size(); ++t, ++tot) {
      if (tot < capacity) {
        idx[tot] = ind[t];
        d2[tot] = dst[t];
      }
    }
    offsets[q + 1] = (int64_t)tot;
  }
  return (long)tot;
}

// sor_octree (kind 0) / sor_pointer_octree (kind 1) on a tree of the cloud
size_t ref_sor_octree(int kind, const float *x, const float *y, const float *z, size_t n,
                      int cap, int depth, float eps, int k, float alpha, float radius,
                      float *out) {
  const PointCloudSoA c = soa(x, y, z, n);
  if (kind == 0) {
    Octree t;
    t.setMaxPointsPerLeaf(cap);
    t.setMaxDepth(depth);
    t.setBuildEpsilon(eps);
    t.setInputCloud(c);
    t.build();
    return sor_octree(c, t, reinterpret_cast<PointXYZ *>(out), k, alpha, radius);
  }
  PointerOctree t;
  t.setMaxPointsPerLeaf(cap);
  t.setMaxDepth(depth);
  t.setBuildEpsilon(eps);
  t.setInputCloud(c);
  t.build();
  return sor_pointer_octree(c, t, reinterpret_cast<PointXYZ *>(out), k, alpha, radius);
}

// normal_estimation_rvv with an Octree (kind 0), a PointerOctree (kind 1),
// or the self-building overload (kind 2, default tree parameters)
void ref_normals_octree(int kind, const float *x, const float *y, const float *z, size_t n,
                        int cap, int depth, float eps, float radius, float vx, float vy,
                        float vz, int iters, float *nx, float *ny, float *nz) {
  const PointCloudSoA c = soa(x, y, z, n);
  if (kind == 0) {
    Octree t;
    t.setMaxPointsPerLeaf(cap);
    t.setMaxDepth(depth);
    t.setBuildEpsilon(eps);
    t.setInputCloud(c);
    t.build();
    normal_estimation_rvv(c, t, nx, ny, nz, 10, radius, vx, vy, vz, iters);
  } else if (kind == 1) {
    PointerOctree t;
    t.setMaxPointsPerLeaf(cap);
    t.setMaxDepth(depth);
    t.setBuildEpsilon(eps);
    t.setInputCloud(c);
    t.build();
    normal_estimation_rvv(c, t, nx, ny, nz, 10, radius, vx, vy, vz, iters);
  } else {
    normal_estimation_rvv(c, nx, ny, nz, 10, radius, vx, vy, vz, iters);
  }
}

// PointerOctree::getRoot: the leaves in depth-first order (children 0..7)
// with their points; returns the number of leaves
long ref_pointer_octree_leaves(const float *x, const float *y, const float *z, size_t n,
                               int cap, int depth, float eps, int32_t *order,
                               int64_t *leaf_offsets) {
  PointerOctree t;
  t.setMaxPointsPerLeaf(cap);
  t.setMaxDepth(depth);
  t.setBuildEpsilon(eps);
  t.setInputCloud(soa(x, y, z, n));
  t.build();
  long leaves = 0;
  size_t pos = 0;
  leaf_offsets[0] = 0;
  std::vector<const PointerOctreeNode *> stack;
  if (t.getRoot()) stack.push_back(t.getRoot());
  while (!stack.empty()) {
    const PointerOctreeNode *nd = stack.back();
    stack.pop_back();
    if (nd->is_leaf) {
      for (int i : nd->indices) order[pos++] = i;
      leaf_offsets[++leaves] = (int64_t)pos;
    } else {
      for (int c = 7; c >= 0; --c)
        if (nd->children[c]) stack.push_back(nd->children[c]);
    }
  }
  return leaves;
}

// std::nth_element of the reference's C++ library (the step of
// sor_pointer_octree, statistical_outlier_removal.cpp:290)
void ref_nth_element(float *a, size_t n, size_t nth) { std::nth_element(a, a + nth, a + n); }

// Raw glibc rand() stream after srand(seed): the hypothesis source of
// ransac_plane_sc (ransac_plane.cpp:60,69-71).
void ref_rand_stream(unsigned seed, int count, int *out) {
  std::srand(seed);
  for (int i = 0; i < count; ++i) out[i] = std::rand();
}

}  // extern "C"
