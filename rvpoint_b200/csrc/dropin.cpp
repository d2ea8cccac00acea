// The reference's C++ interface (namespace rvpoint, headers under
// include/rvpoint/) on top of the C ABI. Every function keeps the
// reference's name, arguments, return value and output layout; the work runs
// on the GPU of a process-wide context (device RVPOINT_DEVICE, default 0).
//
// Errors: the reference has no error channel. Degenerate input (empty
// clouds, n < 3 for RANSAC, k + 1 > n for SOR) returns 0 and leaves the
// outputs untouched, as the reference does or where it has undefined
// behaviour; an allocation failure throws std::bad_alloc; a failure of the
// GPU itself throws std::runtime_error with the library's message (the
// reference cannot fail that way, and a silent 0 would hide it).
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "rvpoint_b200.h"

#pragma GCC visibility push(default)
#include "rvpoint/core/point_types.h"
#include "rvpoint/features/normal_estimation.h"
#include "rvpoint/filters/statistical_outlier_removal.h"
#include "rvpoint/filters/voxel_grid.h"
#include "rvpoint/io/simple_pcd_loader.h"
#include "rvpoint/search/octree.h"
#include "rvpoint/search/pointer_octree.h"
#include "rvpoint/search/spatial_hashing.h"
#include "rvpoint/segmentation/ransac_plane.h"
#include "rvpoint/segmentation/euclidean_clustering.h"

namespace {

std::once_flag g_once;
rvp_context *g_ctx = nullptr;
rvp_status g_ctx_status = RVP_OK;
std::mutex g_mu;  // the reference is single-threaded; calls here are serialised

rvp_context *ctx() {
  std::call_once(g_once, [] {
    const char *d = std::getenv("RVPOINT_DEVICE");
    g_ctx_status = rvp_context_create(d ? std::atoi(d) : 0, &g_ctx);
  });
  if (g_ctx_status != RVP_OK || !g_ctx)
    throw std::runtime_error("rvpoint: no usable CUDA device for librvpoint_b200");
  return g_ctx;
}

// true: go on; false: degenerate input, return the reference's 0
bool ok(rvp_status s) {
  if (s == RVP_OK) return true;
  if (s == RVP_ERR_INVALID_ARG) return false;
  if (s == RVP_ERR_OOM) throw std::bad_alloc();
  const char *m = g_ctx ? rvp_last_error(g_ctx) : nullptr;
  throw std::runtime_error(std::string("rvpoint: ") + (m ? m : "CUDA error"));
}

struct Soa {
  std::vector<float> x, y, z;
  explicit Soa(const rvpoint::PointXYZ *in, std::size_t n) : x(n), y(n), z(n) {
    for (std::size_t i = 0; i < n; ++i) {
      x[i] = in[i].x;
      y[i] = in[i].y;
      z[i] = in[i].z;
    }
  }
};

std::size_t voxel(const float *x, const float *y, const float *z, std::size_t n,
                  rvpoint::PointXYZ *out, float leaf) {
  if (n == 0) return 0;
  std::lock_guard<std::mutex> lock(g_mu);
  size_t cnt = 0;
  if (!ok(rvp_voxel_grid(ctx(), x, y, z, n, leaf, RVP_MEM_HOST, reinterpret_cast<float *>(out),
                         nullptr, &cnt)))
    return 0;
  return cnt;
}

std::size_t sor(const float *x, const float *y, const float *z, std::size_t n,
                rvpoint::PointXYZ *out, int k, float alpha) {
  if (n == 0) return 0;
  std::lock_guard<std::mutex> lock(g_mu);
  size_t cnt = 0;
  if (!ok(rvp_sor(ctx(), x, y, z, n, k, alpha, RVP_MEM_HOST, reinterpret_cast<float *>(out),
                  &cnt, nullptr, nullptr)))
    return 0;
  return cnt;
}

int ransac(const float *x, const float *y, const float *z, std::size_t n, float t, int iters,
           float *model, float col, float prob) {
  if (n < 3) return 0;  // ransac_plane.cpp:59: no srand, no rand()
  std::lock_guard<std::mutex> lock(g_mu);
  int best = 0;
  if (!ok(rvp_ransac_plane(ctx(), x, y, z, n, t, iters, col, prob, nullptr, RVP_MEM_HOST, model,
                           &best, nullptr, nullptr)))
    return 0;
  return best;
}

void extract(const rvpoint::PointCloudSoA &c, const float *model, float t,
             rvpoint::PointXYZ *in, rvpoint::PointXYZ *out, std::size_t &ni, std::size_t &no) {
  ni = no = 0;
  if (c.n == 0) return;
  std::lock_guard<std::mutex> lock(g_mu);
  size_t a = 0, b = 0;
  if (!ok(rvp_extract_plane(ctx(), c.x, c.y, c.z, c.n, model, t, RVP_MEM_HOST,
                            reinterpret_cast<float *>(in), reinterpret_cast<float *>(out), &a,
                            &b)))
    return;
  ni = a;
  no = b;
}

}  // namespace

namespace rvpoint {

// ---- SpatialHash (spatial_hashing.cpp:21-168) -----------------------------
SpatialHash::SpatialHash() = default;

SpatialHash::~SpatialHash() {
  if (h_) rvp_hash_destroy(h_);
}

void SpatialHash::setHashPrimes(int64_t p1, int64_t p2) {
  p1_ = p1;
  p2_ = p2;
  if (h_) {
    std::lock_guard<std::mutex> lock(g_mu);
    ok(rvp_hash_set_primes(h_, p1, p2));
  }
}

void SpatialHash::setInputCloud(const PointCloudSoA &cloud, float cell_size) {
  std::lock_guard<std::mutex> lock(g_mu);
  cloud_ = cloud;
  cell_size_ = cell_size;
  if (!h_) {
    if (!ok(rvp_hash_create(ctx(), &h_))) return;
    ok(rvp_hash_set_primes(h_, p1_, p2_));
  }
  ok(rvp_hash_set_input_cloud(h_, cloud.x, cloud.y, cloud.z, cloud.n, cell_size, RVP_MEM_HOST));
}

void SpatialHash::build() {
  if (!h_) return;
  std::lock_guard<std::mutex> lock(g_mu);
  ok(rvp_hash_build(h_));
}

std::size_t SpatialHash::radiusSearch(const PointXYZ &query, float radius,
                                      std::vector<int> &indices, std::vector<float> &dists,
                                      int max_nn) const {
  indices.clear();
  dists.clear();
  if (!h_ || cloud_.n == 0) return 0;
  std::lock_guard<std::mutex> lock(g_mu);
  int64_t offs[2] = {0, 0};
  size_t cap = max_nn > 0 ? (size_t)max_nn : 256, total = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    indices.resize(cap);
    dists.resize(cap);
    const rvp_status s =
        rvp_hash_radius_search(h_, &query.x, &query.y, &query.z, 1, radius, max_nn, RVP_MEM_HOST,
                               offs, indices.data(), dists.data(), cap, &total);
    if (s == RVP_ERR_CAPACITY && attempt == 0) {
      cap = total;
      continue;
    }
    if (!ok(s)) total = 0;
    break;
  }
  indices.resize(total);
  dists.resize(total);
  return total;
}

// ---- Octree / PointerOctree (octree.cpp, pointer_octree.cpp) --------------
namespace {

void tree_build(rvp_octree *&t, int kind, const PointCloudSoA &c, int cap, int depth, float eps) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!t && !ok(rvp_octree_create(ctx(), kind, &t))) return;
  if (rvp_octree_set_params(t, cap, depth, eps) != RVP_OK)
    throw std::runtime_error(std::string("rvpoint: ") + rvp_last_error(ctx()));
  if (!ok(rvp_octree_set_input_cloud(t, c.x, c.y, c.z, c.n, RVP_MEM_HOST))) return;
  ok(rvp_octree_build(t));
}

std::size_t tree_search(rvp_octree *t, std::size_t n, const PointXYZ &query, float radius,
                        std::vector<int> &indices, std::vector<float> &dists) {
  indices.clear();
  dists.clear();
  if (!t || n == 0) return 0;
  std::lock_guard<std::mutex> lock(g_mu);
  int64_t offs[2] = {0, 0};
  size_t cap = 256, total = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    indices.resize(cap);
    dists.resize(cap);
    const rvp_status s = rvp_octree_radius_search(t, &query.x, &query.y, &query.z, 1, radius,
                                                  RVP_MEM_HOST, offs, indices.data(),
                                                  dists.data(), cap, &total);
    if (s == RVP_ERR_CAPACITY && attempt == 0) {
      cap = total;
      continue;
    }
    if (!ok(s)) total = 0;
    break;
  }
  indices.resize(total);
  dists.resize(total);
  return total;
}

void tree_destroy(rvp_octree *t) {
  if (t) rvp_octree_destroy(t);
}

}  // namespace

Octree::Octree() = default;
Octree::~Octree() { tree_destroy(t_); }
// octree.cpp:28-30: the view is kept; build() reads the points
void Octree::setInputCloud(const PointCloudSoA &cloud) { cloud_ = cloud; }
void Octree::build() {
  tree_build(t_, RVP_OCTREE, cloud_, max_points_per_leaf_, max_depth_, build_epsilon_);
}
std::size_t Octree::radiusSearch(const PointXYZ &query, float radius, std::vector<int> &indices,
                                 std::vector<float> &dists, int max_nn) const {
  (void)max_nn;  // octree.cpp:114
  return tree_search(t_, cloud_.n, query, radius, indices, dists);
}

PointerOctree::PointerOctree() = default;
PointerOctree::~PointerOctree() { tree_destroy(t_); }
void PointerOctree::setInputCloud(const PointCloudSoA &cloud) { cloud_ = cloud; }
void PointerOctree::build() {
  tree_build(t_, RVP_POINTER_OCTREE, cloud_, max_points_per_leaf_, max_depth_, build_epsilon_);
}
std::size_t PointerOctree::radiusSearch(const PointXYZ &query, float radius,
                                        std::vector<int> &indices,
                                        std::vector<float> &dists) const {
  return tree_search(t_, cloud_.n, query, radius, indices, dists);
}
std::size_t PointerOctree::radiusSearchScalar(const PointXYZ &query, float radius,
                                              std::vector<int> &indices,
                                              std::vector<float> &dists) const {
  return tree_search(t_, cloud_.n, query, radius, indices, dists);
}

// ---- voxel grid (voxel_grid_downsamp.cpp) ----------------------------------
std::size_t voxel_grid_downsamp_sc(const PointXYZ *in, std::size_t n, PointXYZ *out,
                                   float leaf_size) {
  if (n == 0) return 0;
  Soa s(in, n);
  return voxel(s.x.data(), s.y.data(), s.z.data(), n, out, leaf_size);
}

std::size_t voxel_grid_downsamp_rvv(const PointCloudSoA &in, PointXYZ *out, float leaf_size) {
  return voxel(in.x, in.y, in.z, in.n, out, leaf_size);
}

std::size_t voxel_grid_downsamp_rvv_v2(const PointCloudSoA &in, PointXYZ *out,
                                       float leaf_size) {
  return voxel(in.x, in.y, in.z, in.n, out, leaf_size);
}

// ---- SOR (statistical_outlier_removal.cpp) ---------------------------------
std::size_t sor_sc(const PointXYZ *in, std::size_t n, PointXYZ *out, int k, float alpha) {
  if (n == 0) return 0;
  Soa s(in, n);
  return sor(s.x.data(), s.y.data(), s.z.data(), n, out, k, alpha);
}

std::size_t sor_rvv(const PointCloudSoA &in, PointXYZ *out, int k, float alpha) {
  return sor(in.x, in.y, in.z, in.n, out, k, alpha);
}

// `in` is the cloud `hash` was built on, as in the reference's callers
std::size_t sor_spatial_hash(const PointCloudSoA &in, const SpatialHash &hash, PointXYZ *out,
                             int k, float alpha, float search_radius) {
  if (in.n == 0 || !hash.device_hash()) return 0;
  std::lock_guard<std::mutex> lock(g_mu);
  size_t cnt = 0;
  if (!ok(rvp_sor_spatial_hash(hash.device_hash(), k, alpha, search_radius, RVP_MEM_HOST,
                               reinterpret_cast<float *>(out), &cnt, nullptr, nullptr)))
    return 0;
  return cnt;
}

namespace {
std::size_t sor_tree(const PointCloudSoA &in, rvp_octree *t, PointXYZ *out, int k, float alpha,
                     float search_radius) {
  if (in.n == 0 || !t) return 0;
  std::lock_guard<std::mutex> lock(g_mu);
  size_t cnt = 0;
  if (!ok(rvp_sor_octree(t, k, alpha, search_radius, RVP_MEM_HOST, reinterpret_cast<float *>(out),
                         &cnt, nullptr, nullptr)))
    return 0;
  return cnt;
}
}  // namespace

// `in` is the cloud `tree` was built on, as in the reference's callers
std::size_t sor_octree(const PointCloudSoA &in, const Octree &tree, PointXYZ *out, int k,
                       float alpha, float search_radius) {
  return sor_tree(in, tree.device_tree(), out, k, alpha, search_radius);
}

std::size_t sor_pointer_octree(const PointCloudSoA &in, const PointerOctree &tree, PointXYZ *out,
                               int k, float alpha, float search_radius) {
  return sor_tree(in, tree.device_tree(), out, k, alpha, search_radius);
}

// ---- normals (normal_estimation.cpp) ---------------------------------------
void normal_estimation_sc(const PointXYZ *in, std::size_t n, float *nx, float *ny, float *nz,
                          int k, float radius, float vp_x, float vp_y, float vp_z,
                          int eigen_iters) {
  (void)radius;  // unused by the reference's scalar path too
  if (n == 0) return;
  Soa s(in, n);
  std::lock_guard<std::mutex> lock(g_mu);
  ok(rvp_normals_knn(ctx(), s.x.data(), s.y.data(), s.z.data(), n, k, vp_x, vp_y, vp_z,
                     eigen_iters, RVP_MEM_HOST, nx, ny, nz));
}

void normal_estimation_rvv(const PointCloudSoA &in, const SpatialHash &hash, float *nx,
                           float *ny, float *nz, int k, float radius, float vp_x, float vp_y,
                           float vp_z, int eigen_iters) {
  (void)k;  // the radius search decides the neighbours, as in the reference
  if (in.n == 0 || !hash.device_hash()) return;
  std::lock_guard<std::mutex> lock(g_mu);
  ok(rvp_normals_radius(hash.device_hash(), radius, vp_x, vp_y, vp_z, eigen_iters, RVP_MEM_HOST,
                        nx, ny, nz));
}

namespace {
void normals_tree(const PointCloudSoA &in, rvp_octree *t, float *nx, float *ny, float *nz,
                  float radius, float vp_x, float vp_y, float vp_z, int eigen_iters) {
  if (in.n == 0 || !t) return;
  std::lock_guard<std::mutex> lock(g_mu);
  ok(rvp_normals_octree(t, radius, vp_x, vp_y, vp_z, eigen_iters, RVP_MEM_HOST, nx, ny, nz));
}
}  // namespace

void normal_estimation_rvv(const PointCloudSoA &in, const Octree &octree, float *nx, float *ny,
                           float *nz, int k, float radius, float vp_x, float vp_y, float vp_z,
                           int eigen_iters) {
  (void)k;  // the radius search decides the neighbours, as in the reference
  normals_tree(in, octree.device_tree(), nx, ny, nz, radius, vp_x, vp_y, vp_z, eigen_iters);
}

void normal_estimation_rvv(const PointCloudSoA &in, const PointerOctree &octree, float *nx,
                           float *ny, float *nz, int k, float radius, float vp_x, float vp_y,
                           float vp_z, int eigen_iters) {
  (void)k;
  normals_tree(in, octree.device_tree(), nx, ny, nz, radius, vp_x, vp_y, vp_z, eigen_iters);
}

void normal_estimation_rvv(const PointCloudSoA &in, float *nx, float *ny, float *nz, int k,
                           float radius, float vp_x, float vp_y, float vp_z, int eigen_iters) {
  PointerOctree octree;
  octree.setInputCloud(in);
  octree.build();
  normal_estimation_rvv(in, octree, nx, ny, nz, k, radius, vp_x, vp_y, vp_z, eigen_iters);
}

// ---- RANSAC (ransac_plane.cpp) ---------------------------------------------
int ransac_plane_sc(const PointXYZ *cloud, std::size_t n, float dist_thresh, int max_iters,
                    float *model, float collinear_thresh, float probability) {
  if (n < 3) return 0;
  Soa s(cloud, n);
  return ransac(s.x.data(), s.y.data(), s.z.data(), n, dist_thresh, max_iters, model,
                collinear_thresh, probability);
}

int ransac_plane_rvv(const PointCloudSoA &cloud, float dist_thresh, int max_iters, float *model,
                     float collinear_thresh, float probability) {
  return ransac(cloud.x, cloud.y, cloud.z, cloud.n, dist_thresh, max_iters, model,
                collinear_thresh, probability);
}

std::size_t extract_plane_inliers_rvv(const PointCloudSoA &cloud, const float *model,
                                      float dist_thresh, PointXYZ *inliers) {
  std::size_t ni = 0, no = 0;
  extract(cloud, model, dist_thresh, inliers, nullptr, ni, no);
  return ni;
}

std::size_t extract_plane_outliers_rvv(const PointCloudSoA &cloud, const float *model,
                                       float dist_thresh, PointXYZ *outliers) {
  std::size_t ni = 0, no = 0;
  extract(cloud, model, dist_thresh, nullptr, outliers, ni, no);
  return no;
}

void extract_plane_inliers_outliers_rvv(const PointCloudSoA &cloud, const float *model,
                                        float dist_thresh, PointXYZ *inliers,
                                        PointXYZ *outliers, std::size_t &n_inliers,
                                        std::size_t &n_outliers) {
  extract(cloud, model, dist_thresh, inliers, outliers, n_inliers, n_outliers);
}

// ---- Euclidean clustering (euclidean_clustering.cpp) -----------------------
void EuclideanClustering::setInputCloud(const PointCloudSoA &cloud) { cloud_ = &cloud; }
void EuclideanClustering::setClusterTolerance(float tolerance) { clusterTolerance_ = tolerance; }
void EuclideanClustering::setMinClusterSize(int min_size) { minClusterSize_ = min_size; }
void EuclideanClustering::setMaxClusterSize(int max_size) { maxClusterSize_ = max_size; }
// euclidean_clustering.cpp:35-43: a searcher built on the same cloud lists
// the same neighbours, so the clusters do not depend on it
void EuclideanClustering::setNeighborSearch(const Octree *search) {
  searcher_ = search;
  ptr_searcher_ = nullptr;
}
void EuclideanClustering::setNeighborSearch(const PointerOctree *search) {
  ptr_searcher_ = search;
  searcher_ = nullptr;
}

std::vector<ClusterIndices> EuclideanClustering::extract() const {
  std::vector<ClusterIndices> result;
  if (!cloud_ || cloud_->n == 0) return result;
  const std::size_t n = cloud_->n;
  std::vector<int64_t> offs(n + 1);
  std::vector<int32_t> idx(n);
  size_t k = 0;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!ok(rvp_euclidean_clusters(ctx(), cloud_->x, cloud_->y, cloud_->z, n, clusterTolerance_,
                                   minClusterSize_, maxClusterSize_, RVP_MEM_HOST, offs.data(),
                                   idx.data(), &k)))
      return result;
  }
  result.resize(k);
  for (size_t c = 0; c < k; ++c)
    result[c].indices.assign(idx.begin() + offs[c], idx.begin() + offs[c + 1]);
  return result;
}

// ---- PCD files (io/simple_pcd_loader.h) -----------------------------------
int loadPCD(const std::string &file_path, std::vector<PointXYZ> &points) {
  std::lock_guard<std::mutex> lock(g_mu);
  rvp_context *c = ctx();
  size_t n = 0;
  // first the count (binary files: from the header alone), then the points
  rvp_status s = rvp_pcd_load(c, file_path.c_str(), RVP_MEM_HOST, nullptr, nullptr, nullptr,
                              0, &n);
  if (s == RVP_ERR_CAPACITY) {
    std::vector<float> x(n), y(n), z(n);
    s = rvp_pcd_load(c, file_path.c_str(), RVP_MEM_HOST, x.data(), y.data(), z.data(), n, &n);
    if (s == RVP_OK) {
      points.resize(n);
      for (size_t i = 0; i < n; ++i) points[i] = {x[i], y[i], z[i]};
    }
  } else if (s == RVP_OK) {
    points.clear();  // an ascii file without a readable point line
  }
  if (s == RVP_OK) return static_cast<int>(points.size());
  if (s == RVP_ERR_OOM) throw std::bad_alloc();
  std::cerr << "Error: " << rvp_last_error(c) << std::endl;
  return -1;
}

namespace {

bool pcd_head(std::ofstream &f, const std::string &name, size_t n, bool rgb, bool binary) {
  if (!f.is_open()) {
    std::cerr << "Error: Could not open file " << name << " for writing." << std::endl;
    return false;
  }
  f << "# .PCD v.7 - Point Cloud Data file format\nVERSION .7\n"
    << (rgb ? "FIELDS x y z rgb\nSIZE 4 4 4 4\nTYPE F F F F\nCOUNT 1 1 1 1\n"
            : "FIELDS x y z\nSIZE 4 4 4\nTYPE F F F\nCOUNT 1 1 1\n")
    << "WIDTH " << n << "\nHEIGHT 1\nVIEWPOINT 0 0 0 1 0 0 0\nPOINTS " << n << "\nDATA "
    << (binary ? "binary" : "ascii") << "\n";
  return true;
}

}  // namespace

void savePCD(const std::string &filename, const std::vector<PointXYZ> &points, bool binary) {
  std::ofstream f(filename, binary ? (std::ios::binary | std::ios::out) : std::ios::out);
  if (!pcd_head(f, filename, points.size(), false, binary)) return;
  if (binary) {
    if (!points.empty())
      f.write(reinterpret_cast<const char *>(points.data()),
              static_cast<std::streamsize>(points.size() * sizeof(PointXYZ)));
  } else {
    for (const PointXYZ &p : points) f << p.x << " " << p.y << " " << p.z << "\n";
  }
  f.close();
  std::cout << "Saved " << points.size() << " points to " << filename << std::endl;
}

void savePCDRGB(const std::string &filename, const std::vector<PointXYZRGB> &points,
                bool binary) {
  std::ofstream f(filename, binary ? (std::ios::binary | std::ios::out) : std::ios::out);
  if (!pcd_head(f, filename, points.size(), true, binary)) return;
  for (const PointXYZRGB &p : points) {
    // packed 0x00RRGGBB, stored as the bits of a float
    const std::uint32_t bits = (std::uint32_t(p.r) << 16) | (std::uint32_t(p.g) << 8) | p.b;
    float rgb;
    std::memcpy(&rgb, &bits, 4);
    if (binary) {
      const float rec[4] = {p.x, p.y, p.z, rgb};
      f.write(reinterpret_cast<const char *>(rec), sizeof rec);
    } else {
      f << p.x << " " << p.y << " " << p.z << " " << rgb << "\n";
    }
  }
  f.close();
  std::cout << "Saved " << points.size() << " colored points to " << filename << std::endl;
}

}  // namespace rvpoint
#pragma GCC visibility pop
