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

// One Jacobi rotation of the reference's loop body on the pair (P, Q), with
// every index static so that A and V stay in registers.
template <int P, int Q>
__device__ __forceinline__ void jacobi_rotate_ref(float (&A)[3][3], float (&V)[3][3]) {
  const float app = A[P][P], aqq = A[Q][Q], apq = A[P][Q];
  const float phi = fmul(0.5f, atan2f(fmul(2.0f, apq), fsub(app, aqq)));
  const float c = cosf(phi), s = sinf(phi);
  const float cc = fmul(c, c), ss = fmul(s, s), s2c = fmul(fmul(2.0f, s), c);
  // c*c*app - 2*s*c*apq + s*s*aqq ; s*s*app + 2*s*c*apq + c*c*aqq
  A[P][P] = fadd(fsub(fmul(cc, app), fmul(s2c, apq)), fmul(ss, aqq));
  A[Q][Q] = fadd(fadd(fmul(ss, app), fmul(s2c, apq)), fmul(cc, aqq));
  A[P][Q] = 0.0f;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const float vip = V[r][P], viq = V[r][Q];
    V[r][P] = fsub(fmul(c, vip), fmul(s, viq));
    V[r][Q] = fadd(fmul(s, vip), fmul(c, viq));
  }
}

// The reference's Jacobi loop: each iteration rotates the pair with the
// largest upper off-diagonal |A[p][q]| (first of equals), which it reads from
// the upper triangle only; the lower triangle is never read.
__device__ __forceinline__ void eigen_smallest_ref(float A[3][3], int iters, float &nx, float &ny, float &nz) {
  float (&M)[3][3] = *reinterpret_cast<float (*)[3][3]>(A);
  float V[3][3] = {{1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f}};
  for (int it = 0; it < iters; ++it) {
    int pq = 0;  // 0: (0,1), 1: (0,2), 2: (1,2)
    float max_off = fabsf(M[0][1]);
    if (fabsf(M[0][2]) > max_off) { pq = 1; max_off = fabsf(M[0][2]); }
    if (fabsf(M[1][2]) > max_off) pq = 2;
    if (pq == 0) jacobi_rotate_ref<0, 1>(M, V);
    else if (pq == 1) jacobi_rotate_ref<0, 2>(M, V);
    else jacobi_rotate_ref<1, 2>(M, V);
  }
  float d0 = M[0][0], d1 = M[1][1], d2 = M[2][2];
  int m = 0;
  float dm = d0;
  if (d1 < dm) { m = 1; dm = d1; }
  if (d2 < dm) m = 2;
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
