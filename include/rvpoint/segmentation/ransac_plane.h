// rvpoint drop-in: RANSAC plane segmentation
// (src/segmentation/ransac_plane.h:11-45 of the reference). Like the
// reference, ransac_plane_* call srand(0) and leave libc's generator as
// after 3 rand() calls per executed iteration.
#pragma once
#include <cstddef>

#include "core/point_types.h"

namespace rvpoint {

int ransac_plane_sc(const PointXYZ *cloud, std::size_t n, float dist_thresh, int max_iters,
                    float *model, float collinear_thresh = 1e-6f, float probability = 0.99f);
int ransac_plane_rvv(const PointCloudSoA &cloud, float dist_thresh, int max_iters,
                     float *model, float collinear_thresh = 1e-6f,
                     float probability = 0.99f);
std::size_t extract_plane_inliers_rvv(const PointCloudSoA &cloud, const float *model,
                                      float dist_thresh, PointXYZ *inliers);
std::size_t extract_plane_outliers_rvv(const PointCloudSoA &cloud, const float *model,
                                       float dist_thresh, PointXYZ *outliers);
void extract_plane_inliers_outliers_rvv(const PointCloudSoA &cloud, const float *model,
                                        float dist_thresh, PointXYZ *inliers,
                                        PointXYZ *outliers, std::size_t &n_inliers,
                                        std::size_t &n_outliers);

}  // namespace rvpoint
