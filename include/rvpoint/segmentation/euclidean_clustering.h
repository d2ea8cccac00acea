// rvpoint drop-in: Euclidean cluster extraction
// (src/segmentation/euclidean_clustering.h:17-70 of the reference). Same
// clusters, order and sorted indices as the reference's extract() without a
// neighbour searcher; the octree searcher overloads are not provided.
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

class EuclideanClustering {
 public:
  EuclideanClustering() = default;
  void setInputCloud(const PointCloudSoA &cloud);
  void setClusterTolerance(float tolerance);
  void setMinClusterSize(int min_size);
  void setMaxClusterSize(int max_size);
  float clusterTolerance() const { return clusterTolerance_; }
  int minClusterSize() const { return minClusterSize_; }
  int maxClusterSize() const { return maxClusterSize_; }
  std::vector<ClusterIndices> extract() const;

 private:
  const PointCloudSoA *cloud_ = nullptr;
  float clusterTolerance_ = 0.05f;
  int minClusterSize_ = 1;
  int maxClusterSize_ = std::numeric_limits<int>::max();
};

}  // namespace rvpoint
