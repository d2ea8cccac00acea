// rvpoint drop-in: Euclidean cluster extraction
// (src/segmentation/euclidean_clustering.h:17-70 of the reference). Same
// clusters, order and sorted indices as the reference's extract(). A
// neighbour searcher (setNeighborSearch) built on the same cloud gives the
// reference the same clusters as none (its radius lists hold the same
// points); it is accepted and the GPU search is used either way.
#pragma once
#include <cstddef>
#include <cstdint>
#include <limits>
#include <vector>

#include "core/point_types.h"

namespace rvpoint {

struct ClusterIndices {
  std::vector<int> indices;
};

class Octree;
class PointerOctree;

class EuclideanClustering {
 public:
  EuclideanClustering() = default;
  void setInputCloud(const PointCloudSoA &cloud);
  void setClusterTolerance(float tolerance);
  void setMinClusterSize(int min_size);
  void setMaxClusterSize(int max_size);
  void setNeighborSearch(const Octree *search);
  void setNeighborSearch(const PointerOctree *search);
  float clusterTolerance() const { return clusterTolerance_; }
  int minClusterSize() const { return minClusterSize_; }
  int maxClusterSize() const { return maxClusterSize_; }
  std::vector<ClusterIndices> extract() const;

 private:
  const PointCloudSoA *cloud_ = nullptr;
  const Octree *searcher_ = nullptr;
  const PointerOctree *ptr_searcher_ = nullptr;
  float clusterTolerance_ = 0.05f;
  int minClusterSize_ = 1;
  int maxClusterSize_ = std::numeric_limits<int>::max();
};

}  // namespace rvpoint
