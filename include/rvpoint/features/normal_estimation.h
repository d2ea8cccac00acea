// rvpoint drop-in: normal estimation (src/features/normal_estimation.h:15-34
// of the reference). The octree overloads are not provided.
#pragma once
#include <cstddef>

#include "core/point_types.h"

namespace rvpoint {

class SpatialHash;

void normal_estimation_sc(const PointXYZ *in, std::size_t n, float *nx, float *ny, float *nz,
                          int k, float radius, float vp_x = 0, float vp_y = 0, float vp_z = 0,
                          int eigen_iters = 4);
void normal_estimation_rvv(const PointCloudSoA &in, const SpatialHash &hash, float *nx,
                           float *ny, float *nz, int k, float radius, float vp_x = 0,
                           float vp_y = 0, float vp_z = 0, int eigen_iters = 4);

}  // namespace rvpoint
