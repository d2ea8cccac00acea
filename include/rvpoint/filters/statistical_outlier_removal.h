// rvpoint drop-in: statistical outlier removal
// (src/filters/statistical_outlier_removal.h:18-36 of the reference). The
// octree overloads are not provided.
#pragma once
#include <cstddef>

#include "core/point_types.h"

namespace rvpoint {

class SpatialHash;

std::size_t sor_sc(const PointXYZ *in, std::size_t n, PointXYZ *out, int k, float alpha);
std::size_t sor_rvv(const PointCloudSoA &in, PointXYZ *out, int k, float alpha);
std::size_t sor_spatial_hash(const PointCloudSoA &in, const SpatialHash &hash, PointXYZ *out,
                             int k, float alpha, float search_radius = 0.5f);

}  // namespace rvpoint
