// rvpoint drop-in: SpatialHash (src/search/spatial_hashing.h:12-53 of the
// reference), served by the GPU hash of librvpoint_b200 (rvp_hash_*).
//
// Same public interface and results: radiusSearch returns every point with
// squared distance <= radius^2, sorted by (squared distance, index), cut at
// max_nn when max_nn > 0, in the reference's output vectors. Differences a
// caller can see: the class layout (it holds a device hash, not an
// unordered_map), and setInputCloud copies the cloud to the GPU at once, so
// later changes to the caller's arrays are not seen by build().
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "core/point_types.h"

struct rvp_hash;

namespace rvpoint {

class SpatialHash {
 public:
  SpatialHash();
  ~SpatialHash();
  SpatialHash(const SpatialHash &) = delete;
  SpatialHash &operator=(const SpatialHash &) = delete;

  void setInputCloud(const PointCloudSoA &cloud, float cell_size);
  void build();
  std::size_t radiusSearch(const PointXYZ &query, float radius, std::vector<int> &indices,
                           std::vector<float> &dists, int max_nn = 0) const;
  void setHashPrimes(int64_t p1, int64_t p2);

  // the device hash behind this object (for the library's batched calls)
  rvp_hash *device_hash() const { return h_; }
  const PointCloudSoA &cloud() const { return cloud_; }

 private:
  rvp_hash *h_ = nullptr;
  PointCloudSoA cloud_;
  float cell_size_ = 0.0f;
  int64_t p1_ = 73856093LL;
  int64_t p2_ = 19349663LL;
};

}  // namespace rvpoint
