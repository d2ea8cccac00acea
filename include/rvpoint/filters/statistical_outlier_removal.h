// rvpoint drop-in: statistical outlier removal
// (src/filters/statistical_outlier_removal.h:18-42 of the reference). The
// index-accelerated variants run on the cloud the index was built on (`in`
// must be that cloud, as in the reference's callers).
#pragma once
#include <cstddef>

#include "core/point_types.h"

namespace rvpoint {

class SpatialHash;
class Octree;
class PointerOctree;

std::size_t sor_sc(const PointXYZ *in, std::size_t n, PointXYZ *out, int k, float alpha);
std::size_t sor_rvv(const PointCloudSoA &in, PointXYZ *out, int k, float alpha);
std::size_t sor_spatial_hash(const PointCloudSoA &in, const SpatialHash &hash, PointXYZ *out,
                             int k, float alpha, float search_radius = 0.5f);
std::size_t sor_octree(const PointCloudSoA &in, const Octree &tree, PointXYZ *out, int k,
                       float alpha, float search_radius = 0.5f);
std::size_t sor_pointer_octree(const PointCloudSoA &in, const PointerOctree &tree, PointXYZ *out,
                               int k, float alpha, float search_radius = 0.5f);

}  // namespace rvpoint
