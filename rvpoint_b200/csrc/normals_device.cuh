// Reference normal arithmetic shared by the normal kernels (normals.cu) and
// the fused kNN + normal tile kernel (knn_tile.cu):
// simple_eigen3x3_smallest (normal_estimation.cpp:16-52) and
// flipNormalTowardsViewpoint (:55-67), every product and sum rounded on its
// own in the reference's order.
#pragma once

#include <math.h>

#include "internal.cuh"

namespace rvp {
namespace nd {

// The reference's Jacobi loop: each iteration rotates the pair with the
// largest upper off-diagonal |A[p][q]| (first of equals), which it reads from
// the upper triangle only; the lower triangle is never read. The pair is
// picked by selects, not branches (lanes of a warp pick different pairs), so
// each iteration evaluates one angle and one rotation per lane; the
// arithmetic on the picked values is the reference's.
__device__ __forceinline__ void eigen_smallest_ref(float A[3][3], int iters, float &nx, float &ny, float &nz) {
  float m00 = A[0][0], m11 = A[1][1], m22 = A[2][2];
  float m01 = A[0][1], m02 = A[0][2], m12 = A[1][2];
  float V[3][3] = {{1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f}};
  for (int it = 0; it < iters; ++it) {
    // 0: (0,1), 1: (0,2), 2: (1,2)
    int pq = 0;
    float max_off = fabsf(m01);
    if (fabsf(m02) > max_off) { pq = 1; max_off = fabsf(m02); }
    if (fabsf(m12) > max_off) pq = 2;
    const float app = pq == 2 ? m11 : m00;
    const float aqq = pq == 0 ? m11 : m22;
    const float apq = pq == 0 ? m01 : (pq == 1 ? m02 : m12);
    const float phi = fmul(0.5f, atan2f(fmul(2.0f, apq), fsub(app, aqq)));
    float s, c;
    sincosf(phi, &s, &c);
    const float cc = fmul(c, c), ss = fmul(s, s), s2c = fmul(fmul(2.0f, s), c);
    // c*c*app - 2*s*c*apq + s*s*aqq ; s*s*app + 2*s*c*apq + c*c*aqq
    const float npp = fadd(fsub(fmul(cc, app), fmul(s2c, apq)), fmul(ss, aqq));
    const float nqq = fadd(fadd(fmul(ss, app), fmul(s2c, apq)), fmul(cc, aqq));
    m00 = pq != 2 ? npp : m00;
    m11 = pq == 2 ? npp : (pq == 0 ? nqq : m11);
    m22 = pq != 0 ? nqq : m22;
    m01 = pq == 0 ? 0.0f : m01;
    m02 = pq == 1 ? 0.0f : m02;
    m12 = pq == 2 ? 0.0f : m12;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const float vip = pq == 2 ? V[r][1] : V[r][0];
      const float viq = pq == 0 ? V[r][1] : V[r][2];
      const float np = fsub(fmul(c, vip), fmul(s, viq));
      const float nq = fadd(fmul(s, vip), fmul(c, viq));
      V[r][0] = pq != 2 ? np : V[r][0];
      V[r][1] = pq == 2 ? np : (pq == 0 ? nq : V[r][1]);
      V[r][2] = pq != 0 ? nq : V[r][2];
    }
  }
  int m = 0;
  float dm = m00;
  if (m11 < dm) { m = 1; dm = m11; }
  if (m22 < dm) m = 2;
  nx = m == 0 ? V[0][0] : (m == 1 ? V[0][1] : V[0][2]);
  ny = m == 0 ? V[1][0] : (m == 1 ? V[1][1] : V[1][2]);
  nz = m == 0 ? V[2][0] : (m == 1 ? V[2][1] : V[2][2]);
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
// "* (1.0f / n)" (normal_estimation.cpp:90-95 / :117-142).
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
// normal_from_list over a register-resident list of M neighbours'
// coordinates (compile-time length: every index below is static).
template <int M>
__device__ __forceinline__ void normal_from_coords(const float (&px)[M], const float (&py)[M],
                                                   const float (&pz)[M], bool div_centroid,
                                                   int iters, float qx, float qy, float qz,
                                                   float vpx, float vpy, float vpz, float &nx,
                                                   float &ny, float &nz) {
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

// The same over M indices (compile-time length) given by idx(t) into x, y, z.
template <int M, class IdxF>
__device__ __forceinline__ void normal_from_regs(const float *__restrict__ x,
                                                 const float *__restrict__ y,
                                                 const float *__restrict__ z, IdxF idx,
                                                 bool div_centroid, int iters, float qx, float qy,
                                                 float qz, float vpx, float vpy, float vpz,
                                                 float &nx, float &ny, float &nz) {
  float px[M], py[M], pz[M];
#pragma unroll
  for (int t = 0; t < M; ++t) {
    const int j = idx(t);
    px[t] = __ldg(&x[j]);
    py[t] = __ldg(&y[j]);
    pz[t] = __ldg(&z[j]);
  }
  normal_from_coords<M>(px, py, pz, div_centroid, iters, qx, qy, qz, vpx, vpy, vpz, nx, ny, nz);
}

template <int M>
__device__ __forceinline__ void normal_from_keys(const float *__restrict__ x,
                                                 const float *__restrict__ y,
                                                 const float *__restrict__ z, const u64 (&L)[M],
                                                 bool div_centroid, int iters, float qx, float qy,
                                                 float qz, float vpx, float vpy, float vpz,
                                                 float &nx, float &ny, float &nz) {
  normal_from_regs<M>(x, y, z, [&](int t) { return nbr_idx(L[t]) & 0x7FFFFFFF; }, div_centroid,
                      iters, qx, qy, qz, vpx, vpy, vpz, nx, ny, nz);
}
}  // namespace nd
}  // namespace rvp
