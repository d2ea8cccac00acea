// Test driver of the drop-in PCD functions (io/simple_pcd_loader.h):
//   dropin_pcd load <file.pcd> <out.bin>   count (int64) then x y z records
//   dropin_pcd save <in.bin> <prefix>      in.bin: n (uint64), n x y z, n r g b
//                                          -> prefix{_a,_b,_rgb_a,_rgb_b}.pcd
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "io/simple_pcd_loader.h"

using namespace rvpoint;

int main(int argc, char **argv) {
  if (argc != 4) return 2;
  if (!std::strcmp(argv[1], "load")) {
    std::vector<PointXYZ> pts;
    const int64_t k = loadPCD(argv[2], pts);
    FILE *f = std::fopen(argv[3], "wb");
    if (!f) return 3;
    std::fwrite(&k, 8, 1, f);
    if (k > 0) std::fwrite(pts.data(), sizeof(PointXYZ), pts.size(), f);
    std::fclose(f);
    return 0;
  }
  FILE *f = std::fopen(argv[2], "rb");
  if (!f) return 3;
  uint64_t n = 0;
  if (std::fread(&n, 8, 1, f) != 1) return 4;
  std::vector<PointXYZ> pts(n);
  std::vector<uint8_t> rgb(3 * n);
  if (std::fread(pts.data(), sizeof(PointXYZ), n, f) != n) return 4;
  if (std::fread(rgb.data(), 1, 3 * n, f) != 3 * n) return 4;
  std::fclose(f);
  std::vector<PointXYZRGB> col(n);
  for (uint64_t i = 0; i < n; ++i)
    col[i] = {pts[i].x, pts[i].y, pts[i].z, rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]};
  const std::string p = argv[3];
  savePCD(p + "_a.pcd", pts, false);
  savePCD(p + "_b.pcd", pts, true);
  savePCDRGB(p + "_rgb_a.pcd", col, false);
  savePCDRGB(p + "_rgb_b.pcd", col, true);
  return 0;
}
