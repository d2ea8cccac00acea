// Reference normal arithmetic shared by the normal kernels (normals.cu) and
// the fused kNN + normal tile kernel (knn_tile.cu):
// simple_eigen3x3_smallest (normal_estimation.cpp:67-103) and
// flipNormalTowardsViewpoint (:106-118), every product and sum rounded on its
// own in the reference's order.
#pragma once

#include <math.h>

#include "internal.cuh"

namespace rvp {
namespace nd {

__device__ __forceinline__ void eigen_smallest_ref(float A[3][3], int iters, float &nx, float &ny, float &nz) {
  float V[3][3] = {{1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f}};
  for (int it = 0; it < iters; ++it) {
    int p = 0, q = 1;
    float max_off = fabsf(A[0][1]);
    if (fabsf(A[0][2]) > max_off) { p = 0; q = 2; max_off = fabsf(A[0][2]); }
    if (fabsf(A[1][2]) > max_off) { p = 1; q = 2; }
    const float app = A[p][p], aqq = A[q][q], apq = A[p][q];
    const float phi = fmul(0.5f, atan2f(fmul(2.0f, apq), fsub(app, aqq)));
    const float c = cosf(phi), s = sinf(phi);
    const float cc = fmul(c, c), ss = fmul(s, s), s2c = fmul(fmul(2.0f, s), c);
    // c*c*app - 2*s*c*apq + s*s*aqq ; s*s*app + 2*s*c*apq + c*c*aqq
    A[p][p] = fadd(fsub(fmul(cc, app), fmul(s2c, apq)), fmul(ss, aqq));
    A[q][q] = fadd(fadd(fmul(ss, app), fmul(s2c, apq)), fmul(cc, aqq));
    A[p][q] = 0.0f;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const float vip = V[r][p], viq = V[r][q];
      V[r][p] = fsub(fmul(c, vip), fmul(s, viq));
      V[r][q] = fadd(fmul(s, vip), fmul(c, viq));
    }
  }
  int m = 0;
  if (A[1][1] < A[m][m]) m = 1;
  if (A[2][2] < A[m][m]) m = 2;
  nx = V[0][m];
  ny = V[1][m];
  nz = V[2][m];
}

__device__ __forceinline__ void flip_ref(float px, float py, float pz, float vpx, float vpy,
                                         float vpz, float &nx, float &ny, float &nz) {
  const float vx = fsub(vpx, px), vy = fsub(vpy, py), vz = fsub(vpz, pz);
  const float dot = fadd(fadd(fmul(vx, nx), fmul(vy, ny)), fmul(vz, nz));
  if (dot < 0.0f) {
    nx = -nx;
    ny = -ny;
    nz = -nz;
  }
}


// Centroid, six covariance sums, eigen-solve and flip over the neighbour
// list nb(0..m-1) (indices into x, y, z), in list order. div_centroid:
// normal_estimation_sc's "/ (k+1)"; else compute_covariance_rvv's
// "* (1.0f / n)" (normal_estimation.cpp:141-146 / :168-193).
template <class Idx>
__device__ __forceinline__ void normal_from_list(const float *__restrict__ x,
                                                 const float *__restrict__ y,
                                                 const float *__restrict__ z, Idx nb, int m,
                                                 bool div_centroid, int iters, float qx,
                                                 float qy, float qz, float vpx, float vpy,
                                                 float vpz, float &nx, float &ny, float &nz) {
  float cx = 0.0f, cy = 0.0f, cz = 0.0f;
  for (int t = 0; t < m; ++t) {
    const int j = nb(t);
    cx = fadd(cx, x[j]);
    cy = fadd(cy, y[j]);
    cz = fadd(cz, z[j]);
  }
  if (div_centroid) {
    const float fm = (float)m;
    cx = fdiv(cx, fm);
    cy = fdiv(cy, fm);
    cz = fdiv(cz, fm);
  } else {
    const float inv_n = fdiv(1.0f, (float)m);
    cx = fmul(cx, inv_n);
    cy = fmul(cy, inv_n);
    cz = fmul(cz, inv_n);
  }
  float c00 = 0, c01 = 0, c02 = 0, c11 = 0, c12 = 0, c22 = 0;
  for (int t = 0; t < m; ++t) {
    const int j = nb(t);
    const float dx = fsub(x[j], cx), dy = fsub(y[j], cy), dz = fsub(z[j], cz);
    c00 = fadd(c00, fmul(dx, dx));
    c01 = fadd(c01, fmul(dx, dy));
    c02 = fadd(c02, fmul(dx, dz));
    c11 = fadd(c11, fmul(dy, dy));
    c12 = fadd(c12, fmul(dy, dz));
    c22 = fadd(c22, fmul(dz, dz));
  }
  float A[3][3] = {{c00, c01, c02}, {c01, c11, c12}, {c02, c12, c22}};
  eigen_smallest_ref(A, iters, nx, ny, nz);
  flip_ref(qx, qy, qz, vpx, vpy, vpz, nx, ny, nz);
}

}  // namespace nd
}  // namespace rvp

namespace rvp {
namespace nd {
// normal_from_list over a register-resident list of M packed (d2, index)
// keys (compile-time length: every index below is static).
template <int M>
__device__ __forceinline__ void normal_from_keys(const float *__restrict__ x,
                                                 const float *__restrict__ y,
                                                 const float *__restrict__ z, const u64 (&L)[M],
                                                 bool div_centroid, int iters, float qx, float qy,
                                                 float qz, float vpx, float vpy, float vpz,
                                                 float &nx, float &ny, float &nz) {
  float px[M], py[M], pz[M];
#pragma unroll
  for (int t = 0; t < M; ++t) {
    const int j = nbr_idx(L[t]) & 0x7FFFFFFF;
    px[t] = __ldg(&x[j]);
    py[t] = __ldg(&y[j]);
    pz[t] = __ldg(&z[j]);
  }
  float cx = 0.0f, cy = 0.0f, cz = 0.0f;
#pragma unroll
  for (int t = 0; t < M; ++t) {
    cx = fadd(cx, px[t]);
    cy = fadd(cy, py[t]);
    cz = fadd(cz, pz[t]);
  }
  if (div_centroid) {
    const float fm = (float)M;
    cx = fdiv(cx, fm);
    cy = fdiv(cy, fm);
    cz = fdiv(cz, fm);
  } else {
    const float inv_n = fdiv(1.0f, (float)M);
    cx = fmul(cx, inv_n);
    cy = fmul(cy, inv_n);
    cz = fmul(cz, inv_n);
  }
  float c00 = 0, c01 = 0, c02 = 0, c11 = 0, c12 = 0, c22 = 0;
#pragma unroll
  for (int t = 0; t < M; ++t) {
    const float dx = fsub(px[t], cx), dy = fsub(py[t], cy), dz = fsub(pz[t], cz);
    c00 = fadd(c00, fmul(dx, dx));
    c01 = fadd(c01, fmul(dx, dy));
    c02 = fadd(c02, fmul(dx, dz));
    c11 = fadd(c11, fmul(dy, dy));
    c12 = fadd(c12, fmul(dy, dz));
    c22 = fadd(c22, fmul(dz, dz));
  }
  float A[3][3] = {{c00, c01, c02}, {c01, c11, c12}, {c02, c12, c22}};
  eigen_smallest_ref(A, iters, nx, ny, nz);
  flip_ref(qx, qy, qz, vpx, vpy, vpz, nx, ny, nz);
}
}  // namespace nd
}  // namespace rvp
