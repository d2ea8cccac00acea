// rvpoint drop-in: normal estimation (src/features/normal_estimation.h:15-49
// of the reference). The index overloads run on the cloud the index was built
// on (`in` must be that cloud, as in the reference's callers).
#pragma once
#include <cstddef>

#include "core/point_types.h"

namespace rvpoint {

class SpatialHash;
class Octree;
class PointerOctree;

void normal_estimation_sc(const PointXYZ *in, std::size_t n, float *nx, float *ny, float *nz,
                          int k, float radius, float vp_x = 0, float vp_y = 0, float vp_z = 0,
                          int eigen_iters = 4);
void normal_estimation_rvv(const PointCloudSoA &in, const SpatialHash &hash, float *nx,
                           float *ny, float *nz, int k, float radius, float vp_x = 0,
                           float vp_y = 0, float vp_z = 0, int eigen_iters = 4);
void normal_estimation_rvv(const PointCloudSoA &in, const Octree &octree, float *nx, float *ny,
                           float *nz, int k, float radius, float vp_x = 0, float vp_y = 0,
                           float vp_z = 0, int eigen_iters = 4);
void normal_estimation_rvv(const PointCloudSoA &in, const PointerOctree &octree, float *nx,
                           float *ny, float *nz, int k, float radius, float vp_x = 0,
                           float vp_y = 0, float vp_z = 0, int eigen_iters = 4);
// builds a PointerOctree of `in` itself (normal_estimation.cpp:246-253)
void normal_estimation_rvv(const PointCloudSoA &in, float *nx, float *ny, float *nz, int k,
                           float radius, float vp_x = 0, float vp_y = 0, float vp_z = 0,
                           int eigen_iters = 4);

}  // namespace rvpoint
