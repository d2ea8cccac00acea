// rvpoint drop-in: point types (src/core/point_types.h:12-29 of the
// reference). Same names, members and layout: PointXYZ is 12 bytes of x, y, z;
// PointCloudSoA is a non-owning view of three coordinate arrays.
#pragma once
#include <cstddef>

namespace rvpoint {

struct PointXYZ {
  float x, y, z;
};

struct PointCloudSoA {
  float *x = nullptr;
  float *y = nullptr;
  float *z = nullptr;
  std::size_t n = 0;
};

}  // namespace rvpoint
