// rvpoint drop-in: Octree (src/search/octree.h:20-48 of the reference), served
// by the GPU tree ranks of librvpoint_b200 (rvp_octree_*).
//
// Same public interface and results: radiusSearch returns every point with
// squared distance <= radius^2 in the reference tree's depth-first leaf
// order (children 0..7, each leaf's points by index), max_nn ignored, in the
// reference's output vectors. Differences a caller can see: no node
// structure (OctreeNode) is built or exposed, build() copies the cloud to the
// GPU (later changes to the caller's arrays need another build()), and
// setMaxDepth above 21 is refused (build() then throws std::runtime_error).
#pragma once
#include <cstddef>
#include <vector>

#include "core/point_types.h"

struct rvp_octree;

namespace rvpoint {

class Octree {
 public:
  Octree();
  ~Octree();
  Octree(const Octree &) = delete;
  Octree &operator=(const Octree &) = delete;

  void setInputCloud(const PointCloudSoA &cloud);
  void build();

  std::size_t radiusSearch(const PointXYZ &query, float radius, std::vector<int> &indices,
                           std::vector<float> &dists, int max_nn = 0) const;

  void setMaxPointsPerLeaf(int n) { max_points_per_leaf_ = n; }
  void setMaxDepth(int d) { max_depth_ = d; }
  void setBuildEpsilon(float eps) { build_epsilon_ = eps; }

  // the device tree behind this object (for the library's batched calls)
  rvp_octree *device_tree() const { return t_; }
  const PointCloudSoA &cloud() const { return cloud_; }

 private:
  rvp_octree *t_ = nullptr;
  PointCloudSoA cloud_;
  int max_points_per_leaf_ = 64;
  int max_depth_ = 8;
  float build_epsilon_ = 1e-4f;
};

}  // namespace rvpoint
