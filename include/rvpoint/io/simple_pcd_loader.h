// rvpoint drop-in: PCD file input and output (src/io/simple_pcd_loader.h:143-386
// of the reference). loadPCD reads DATA ascii, binary and binary_compressed
// files with any fields around 4-byte x, y, z and returns the point count or
// -1; savePCD / savePCDRGB write the reference's x y z (rgb) files byte for
// byte. The C ABI's rvp_pcd_load reads the same files straight into device
// arrays.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "core/point_types.h"

namespace rvpoint {

int loadPCD(const std::string &file_path, std::vector<PointXYZ> &points);

void savePCD(const std::string &filename, const std::vector<PointXYZ> &points,
             bool binary = false);

struct PointXYZRGB {
  float x;
  float y;
  float z;
  std::uint8_t r;
  std::uint8_t g;
  std::uint8_t b;
};

void savePCDRGB(const std::string &filename, const std::vector<PointXYZRGB> &points,
                bool binary = false);

}  // namespace rvpoint
