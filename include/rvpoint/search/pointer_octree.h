// rvpoint drop-in: PointerOctree (src/search/pointer_octree.h:26-62 of the
// reference), served by the GPU tree ranks of librvpoint_b200 (rvp_octree_*
// with RVP_POINTER_OCTREE: root box [min - eps, max + eps]).
//
// radiusSearch and radiusSearchScalar return the reference's list: every
// point with squared distance <= radius^2 in the tree's depth-first leaf
// order. Differences a caller can see: no node structure is built, so
// getRoot() is not provided; build() copies the cloud to the GPU; setMaxDepth
// above 21 is refused (build() then throws std::runtime_error).
#pragma once
#include <cstddef>
#include <vector>

#include "core/point_types.h"

struct rvp_octree;

namespace rvpoint {

class PointerOctree {
 public:
  PointerOctree();
  ~PointerOctree();
  PointerOctree(const PointerOctree &) = delete;
  PointerOctree &operator=(const PointerOctree &) = delete;

  void setInputCloud(const PointCloudSoA &cloud);
  void build();

  std::size_t radiusSearch(const PointXYZ &query, float radius, std::vector<int> &indices,
                           std::vector<float> &dists) const;
  std::size_t radiusSearchScalar(const PointXYZ &query, float radius, std::vector<int> &indices,
                                 std::vector<float> &dists) const;

  void setMaxPointsPerLeaf(int n) { max_points_per_leaf_ = n; }
  void setMaxDepth(int d) { max_depth_ = d; }
  void setBuildEpsilon(float eps) { build_epsilon_ = eps; }

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
