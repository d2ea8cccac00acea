// rvpoint drop-in: voxel-grid downsampling (src/filters/voxel_grid.h:14-34 of
// the reference). All three variants return the x86 reference's output: one
// centroid per occupied voxel, sums in input order, voxels ordered by
// (ix, iy, iz).
#pragma once
#include <cstddef>

#include "core/point_types.h"

namespace rvpoint {

std::size_t voxel_grid_downsamp_sc(const PointXYZ *in, std::size_t n, PointXYZ *out,
                                   float leaf_size);
[[deprecated("Use voxel_grid_downsamp_rvv_v2")]]
std::size_t voxel_grid_downsamp_rvv(const PointCloudSoA &in, PointXYZ *out, float leaf_size);
std::size_t voxel_grid_downsamp_rvv_v2(const PointCloudSoA &in, PointXYZ *out,
                                       float leaf_size);

}  // namespace rvpoint
