// Drives the drop-in Octree / PointerOctree calls (include/rvpoint/) the way
// the reference's pipeline driver does (pipeline_export.cpp: PointerOctree ->
// sor_pointer_octree -> rebuild -> normals), plus the Octree variants, on a
// cloud read from a file; writes every result for tests/test_dropin.py.
//
//   dropin_octree in.bin out.bin
// in.bin:  u64 n, float x[n], y[n], z[n]
// out.bin: a sequence of arrays, each u64 count then the values
#include <cstdint>
#include <cstdio>
#include <vector>

#include "features/normal_estimation.h"
#include "filters/statistical_outlier_removal.h"
#include "search/octree.h"
#include "search/pointer_octree.h"
#include "segmentation/euclidean_clustering.h"

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

  // radius lists of the first 50 points, both trees (max_nn is ignored)
  Octree ot;
  ot.setMaxPointsPerLeaf(16);
  ot.setInputCloud(in);
  ot.build();
  PointerOctree pt;
  pt.setInputCloud(in);
  pt.build();
  std::vector<int> ind, all_i;
  std::vector<float> dst, all_d;
  std::vector<int64_t> cnt;
  for (int t = 0; t < 3; ++t) {
    for (uint64_t q = 0; q < 50 && q < n; ++q) {
      const PointXYZ p{x[q], y[q], z[q]};
      const std::size_t m = t == 0   ? ot.radiusSearch(p, 0.1f, ind, dst, 5)
                            : t == 1 ? pt.radiusSearch(p, 0.1f, ind, dst)
                                     : pt.radiusSearchScalar(p, 0.1f, ind, dst);
      cnt.push_back((int64_t)m);
      all_i.insert(all_i.end(), ind.begin(), ind.end());
      all_d.insert(all_d.end(), dst.begin(), dst.end());
    }
  }
  put(cnt.data(), cnt.size());
  put(all_i.data(), all_i.size());
  put(all_d.data(), all_d.size());

  // SOR over both trees (pipeline_export.cpp: radius 0.25, k = 20)
  std::vector<PointXYZ> out(n);
  std::size_t k0 = sor_octree(in, ot, out.data(), 20, 1.0f, 0.25f);
  put(reinterpret_cast<float *>(out.data()), 3 * k0);
  std::size_t k1 = sor_pointer_octree(in, pt, out.data(), 20, 1.0f, 0.25f);
  put(reinterpret_cast<float *>(out.data()), 3 * k1);

  // normals: Octree, PointerOctree and the self-building overload
  std::vector<float> nx(n), ny(n), nz(n);
  normal_estimation_rvv(in, ot, nx.data(), ny.data(), nz.data(), 10, 0.1f);
  put(nx.data(), n); put(ny.data(), n); put(nz.data(), n);
  normal_estimation_rvv(in, pt, nx.data(), ny.data(), nz.data(), 10, 0.1f);
  put(nx.data(), n); put(ny.data(), n); put(nz.data(), n);
  normal_estimation_rvv(in, nx.data(), ny.data(), nz.data(), 10, 0.1f);
  put(nx.data(), n); put(ny.data(), n); put(nz.data(), n);

  // clustering with a PointerOctree searcher
  EuclideanClustering ec;
  ec.setInputCloud(in);
  ec.setClusterTolerance(0.05f);
  ec.setMinClusterSize(3);
  ec.setNeighborSearch(&pt);
  const std::vector<ClusterIndices> cl = ec.extract();
  std::vector<int64_t> offs{0};
  std::vector<int> idx;
  for (const ClusterIndices &c : cl) {
    idx.insert(idx.end(), c.indices.begin(), c.indices.end());
    offs.push_back((int64_t)idx.size());
  }
  put(offs.data(), offs.size());
  put(idx.data(), idx.size());

  // a depth the drop-in refuses: build() throws
  Octree deep;
  deep.setMaxDepth(22);
  deep.setInputCloud(in);
  int64_t threw = 0;
  try {
    deep.build();
  } catch (const std::exception &) {
    threw = 1;
  }
  put(&threw, 1);
  std::fclose(g_out);
  return 0;
}
