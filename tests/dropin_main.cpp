// Drives the rvpoint C++ drop-in (include/rvpoint/) the way the reference's
// pipeline driver does, on a cloud read from a file, and writes every
// result for tests/test_dropin.py to compare with the CPU oracle.
//
//   dropin_main in.bin out.bin
// in.bin:  u64 n, float x[n], y[n], z[n]
// out.bin: a sequence of arrays, each u64 count then the values
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "features/normal_estimation.h"
#include "filters/statistical_outlier_removal.h"
#include "filters/voxel_grid.h"
#include "search/spatial_hashing.h"
#include "segmentation/euclidean_clustering.h"
#include "segmentation/ransac_plane.h"

using namespace rvpoint;

static FILE *g_out;
template <class T>
static void put(const T *p, uint64_t count) {
  std::fwrite(&count, 8, 1, g_out);
  if (count) std::fwrite(p, sizeof(T), count, g_out);
}

int main(int argc, char **argv) {
  if (argc != 3) return 2;
  FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  uint64_t n = 0;
  if (std::fread(&n, 8, 1, f) != 1) return 4;
  std::vector<float> x(n), y(n), z(n);
  if (std::fread(x.data(), 4, n, f) != n || std::fread(y.data(), 4, n, f) != n ||
      std::fread(z.data(), 4, n, f) != n)
    return 5;
  std::fclose(f);
  g_out = std::fopen(argv[2], "wb");
  if (!g_out) return 6;

  PointCloudSoA in{x.data(), y.data(), z.data(), n};
  // voxel 0.05 -> SOR k=10 -> hash -> normals r=0.15 -> RANSAC -> split
  std::vector<PointXYZ> vox(n);
  const std::size_t nv = voxel_grid_downsamp_rvv_v2(in, vox.data(), 0.05f);
  put(reinterpret_cast<float *>(vox.data()), 3 * nv);
  std::vector<PointXYZ> vox_sc(n);
  std::vector<PointXYZ> aos(n);
  for (std::size_t i = 0; i < n; ++i) aos[i] = {x[i], y[i], z[i]};
  const std::size_t nv2 = voxel_grid_downsamp_sc(aos.data(), n, vox_sc.data(), 0.05f);
  put(reinterpret_cast<float *>(vox_sc.data()), 3 * nv2);

  std::vector<float> vx(nv), vy(nv), vz(nv);
  for (std::size_t i = 0; i < nv; ++i) { vx[i] = vox[i].x; vy[i] = vox[i].y; vz[i] = vox[i].z; }
  PointCloudSoA vc{vx.data(), vy.data(), vz.data(), nv};
  std::vector<PointXYZ> sor_out(nv);
  const std::size_t ns = sor_rvv(vc, sor_out.data(), 10, 1.0f);
  put(reinterpret_cast<float *>(sor_out.data()), 3 * ns);
  std::vector<PointXYZ> sor_out2(nv);
  const std::size_t ns2 = sor_sc(vox.data(), nv, sor_out2.data(), 10, 1.0f);
  put(reinterpret_cast<float *>(sor_out2.data()), 3 * ns2);

  std::vector<float> sx(ns), sy(ns), sz(ns);
  for (std::size_t i = 0; i < ns; ++i) { sx[i] = sor_out[i].x; sy[i] = sor_out[i].y; sz[i] = sor_out[i].z; }
  PointCloudSoA sc{sx.data(), sy.data(), sz.data(), ns};
  SpatialHash hash;
  hash.setInputCloud(sc, 0.15f);
  hash.build();
  std::vector<int> idx;
  std::vector<float> d2;
  std::vector<int> all_idx;
  std::vector<float> all_d2;
  std::vector<int64_t> counts;
  for (std::size_t q = 0; q < ns; q += 97) {
    const std::size_t c = hash.radiusSearch(sor_out[q], 0.15f, idx, d2, q % 2 ? 8 : 0);
    counts.push_back((int64_t)c);
    all_idx.insert(all_idx.end(), idx.begin(), idx.end());
    all_d2.insert(all_d2.end(), d2.begin(), d2.end());
  }
  put(counts.data(), counts.size());
  put(all_idx.data(), all_idx.size());
  put(all_d2.data(), all_d2.size());

  std::vector<float> nx(ns), ny(ns), nz(ns);
  normal_estimation_rvv(sc, hash, nx.data(), ny.data(), nz.data(), 16, 0.15f);
  put(nx.data(), ns);
  put(ny.data(), ns);
  put(nz.data(), ns);
  std::vector<PointXYZ> sub(sor_out.begin(), sor_out.begin() + (ns < 3000 ? ns : 3000));
  std::vector<float> kx(sub.size()), ky(sub.size()), kz(sub.size());
  normal_estimation_sc(sub.data(), sub.size(), kx.data(), ky.data(), kz.data(), 16, 0.0f);
  put(kx.data(), kx.size());
  put(ky.data(), ky.size());
  put(kz.data(), kz.size());

  std::vector<PointXYZ> filt(ns);
  const std::size_t nf = sor_spatial_hash(sc, hash, filt.data(), 10, 1.0f, 0.15f);
  put(reinterpret_cast<float *>(filt.data()), 3 * nf);

  float model[4] = {0, 0, 0, 0};
  const int best = ransac_plane_rvv(sc, 0.01f, 1000, model);
  const int after = std::rand();  // libc's generator as the reference leaves it
  int32_t r2[2] = {best, after};
  put(r2, 2);
  put(model, 4);
  float model_sc[4] = {0, 0, 0, 0};
  const int best_sc = ransac_plane_sc(sor_out.data(), ns, 0.01f, 1000, model_sc);
  put(&best_sc, 1);
  put(model_sc, 4);

  std::vector<PointXYZ> pin(ns), pout(ns);
  std::size_t ni = 0, no = 0;
  extract_plane_inliers_outliers_rvv(sc, model, 0.01f, pin.data(), pout.data(), ni, no);
  put(reinterpret_cast<float *>(pin.data()), 3 * ni);
  put(reinterpret_cast<float *>(pout.data()), 3 * no);
  // Euclidean clusters of the SOR output
  EuclideanClustering ec;
  ec.setInputCloud(sc);
  ec.setClusterTolerance(0.08f);
  ec.setMinClusterSize(2);
  const std::vector<ClusterIndices> cl = ec.extract();
  std::vector<int64_t> coffs{0};
  std::vector<int> cidx;
  for (const auto &c : cl) {
    cidx.insert(cidx.end(), c.indices.begin(), c.indices.end());
    coffs.push_back((int64_t)cidx.size());
  }
  put(coffs.data(), coffs.size());
  put(cidx.data(), cidx.size());
  // degenerate inputs return 0 as in the reference
  PointCloudSoA empty{};
  float m0[4] = {9, 9, 9, 9};
  int64_t degenerate[3] = {(int64_t)voxel_grid_downsamp_rvv_v2(empty, vox.data(), 0.05f),
                           (int64_t)ransac_plane_rvv(empty, 0.01f, 100, m0),
                           (int64_t)(m0[0] == 9.0f)};
  put(degenerate, 3);
  std::fclose(g_out);
  return 0;
}
