// PCA normals (features/normal_estimation.cpp).
//
// Reference path: per point, the neighbour list in (d2, index) order,
// centroid (sum then "* (1.0f / n)" in compute_covariance_rvv :117-142, or
// "/ (k+1)" in normal_estimation_sc :90-95), six covariance sums, then
// simple_eigen3x3_smallest (:16-52: `iters` rotations on the largest
// off-diagonal entry, updating only A[p][p], A[q][q], A[p][q] and V) and the
// viewpoint flip (:55-67). Every step keeps the reference's operation order
// with separately rounded products and sums; atan2f/cosf/sinf are CUDA's,
// which is why normals are compared within a tolerance.
//
// Precision path (normals_precise): covariance accumulated in FP32 about the
// query point (differences of nearby points are exact) with compensated
// (Kahan) sums, converged cyclic Jacobi in FP32, and the eigen-solve redone
// in FP64 only when lambda_max / lambda_min exceeds a threshold.
#include <math.h>

#include "internal.cuh"
#include "normals_device.cuh"

namespace rvp {
using namespace nd;

namespace {

// One thread per list slot i: query qi = order ? order[i] : i, neighbours
// pairs[offsets[i] ..) or pairs[i*fixed_k ..), result at out_pos[qi] (or qi).
__global__ void k_normals_lists(const float *__restrict__ x, const float *__restrict__ y,
                                const float *__restrict__ z, const u64 *__restrict__ pairs,
                                const u64 *__restrict__ offsets,
                                const int32_t *__restrict__ fixed_counts, int fixed_k,
                                size_t n_max, const u64 *n_dev, bool div_centroid, int iters,
                                float vpx, float vpy, float vpz, const float *qx,
                                const float *qy, const float *qz, float *nx, float *ny,
                                float *nz, const u32 *order, const u64 *out_pos) {
  const size_t n = n_dev ? *n_dev : n_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const u64 *l;
    int m;
    if (offsets) {
      l = pairs + offsets[i];
      m = (int)(offsets[i + 1] - offsets[i]);
    } else {
      l = pairs + i * (size_t)fixed_k;
      m = fixed_counts ? fixed_counts[i] : fixed_k;
    }
    const size_t qi = order ? (size_t)order[i] : i;
    const size_t oi = out_pos ? (size_t)out_pos[qi] : qi;
    if (m < 3) {  // normal_estimation.cpp:203
      nx[oi] = ny[oi] = nz[oi] = 0.0f;
      continue;
    }
    float a, b, c;
    normal_from_list(x, y, z, [&](int t) { return nbr_idx(l[t]) & 0x7FFFFFFF; }, m, div_centroid,
                     iters, qx[qi], qy[qi], qz[qi], vpx, vpy, vpz, a, b, c);
    nx[oi] = a;
    ny[oi] = b;
    nz[oi] = c;
  }
}

// ---------------------------------------------------------------------------
// precision path
// ---------------------------------------------------------------------------
__device__ __forceinline__ void kahan_add(float &s, float &c, float v) {
  const float y = fsub(v, c);
  const float t = fadd(s, y);
  c = fsub(fsub(t, s), y);
  s = t;
}

template <class T>
__device__ void jacobi_sym3(T A[3][3], T V[3][3], int sweeps) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? T(1) : T(0);
  for (int sw = 0; sw < sweeps; ++sw) {
    const T off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const T dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (!(off > (sizeof(T) == 4 ? T(1e-14) : T(1e-30)) * dia)) break;
#pragma unroll
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0;
      const int q = pq == 0 ? 1 : 2;
      if (A[p][q] == T(0)) continue;
      const T theta = (A[q][q] - A[p][p]) / (T(2) * A[p][q]);
      const T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
      const T c = T(1) / sqrt(t * t + T(1)), s = t * c;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const T arp = A[r][p], arq = A[r][q];
        A[r][p] = c * arp - s * arq;
        A[r][q] = s * arp + c * arq;
      }
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const T apr = A[p][r], aqr = A[q][r];
        A[p][r] = c * apr - s * aqr;
        A[q][r] = s * apr + c * aqr;
      }
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const T vrp = V[r][p], vrq = V[r][q];
        V[r][p] = c * vrp - s * vrq;
        V[r][q] = s * vrp + c * vrq;
      }
    }
  }
}

__global__ void k_normals_precise(const float *__restrict__ x, const float *__restrict__ y,
                                  const float *__restrict__ z, const u64 *__restrict__ pairs,
                                  int kk, size_t n, float vpx, float vpy, float vpz,
                                  double cond_fp64, float *nx, float *ny, float *nz,
                                  float *cond_out, uint8_t *used64) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const u64 *l = pairs + i * (size_t)kk;
    const float qx = x[i], qy = y[i], qz = z[i];
    // shifted, compensated centroid of (p - q)
    float sx = 0, sy = 0, sz = 0, ex = 0, ey = 0, ez = 0;
    for (int t = 0; t < kk; ++t) {
      const int j = nbr_idx(l[t]) & 0x7FFFFFFF;
      kahan_add(sx, ex, fsub(x[j], qx));
      kahan_add(sy, ey, fsub(y[j], qy));
      kahan_add(sz, ez, fsub(z[j], qz));
    }
    const float inv = fdiv(1.0f, (float)kk);
    const float cx = fmul(sx, inv), cy = fmul(sy, inv), cz = fmul(sz, inv);
    float s[6] = {0, 0, 0, 0, 0, 0}, e[6] = {0, 0, 0, 0, 0, 0};
    for (int t = 0; t < kk; ++t) {
      const int j = nbr_idx(l[t]) & 0x7FFFFFFF;
      const float dx = fsub(fsub(x[j], qx), cx);
      const float dy = fsub(fsub(y[j], qy), cy);
      const float dz = fsub(fsub(z[j], qz), cz);
      kahan_add(s[0], e[0], fmul(dx, dx));
      kahan_add(s[1], e[1], fmul(dx, dy));
      kahan_add(s[2], e[2], fmul(dx, dz));
      kahan_add(s[3], e[3], fmul(dy, dy));
      kahan_add(s[4], e[4], fmul(dy, dz));
      kahan_add(s[5], e[5], fmul(dz, dz));
    }
    float A[3][3] = {{s[0], s[1], s[2]}, {s[1], s[3], s[4]}, {s[2], s[4], s[5]}};
    float V[3][3];
    jacobi_sym3<float>(A, V, 8);
    int mi = 0, ma = 0;
    for (int a = 1; a < 3; ++a) {
      if (A[a][a] < A[mi][mi]) mi = a;
      if (A[a][a] > A[ma][ma]) ma = a;
    }
    const float lo = fabsf(A[mi][mi]), hi = fabsf(A[ma][ma]);
    const double cnd = lo > 0.0f ? (double)hi / (double)lo : 1e300;
    double ax, ay, az;
    bool u64path = false;
    if (cnd > cond_fp64) {
      double D[3][3] = {{s[0], s[1], s[2]}, {s[1], s[3], s[4]}, {s[2], s[4], s[5]}};
      // fold the compensation terms back in
      D[0][0] -= e[0]; D[0][1] -= e[1]; D[0][2] -= e[2];
      D[1][1] -= e[3]; D[1][2] -= e[4]; D[2][2] -= e[5];
      D[1][0] = D[0][1]; D[2][0] = D[0][2]; D[2][1] = D[1][2];
      double W[3][3];
      jacobi_sym3<double>(D, W, 32);
      int m2 = 0;
      for (int a = 1; a < 3; ++a)
        if (D[a][a] < D[m2][m2]) m2 = a;
      ax = W[0][m2]; ay = W[1][m2]; az = W[2][m2];
      u64path = true;
    } else {
      ax = V[0][mi]; ay = V[1][mi]; az = V[2][mi];
    }
    const double nr = sqrt(ax * ax + ay * ay + az * az);
    ax /= nr; ay /= nr; az /= nr;
    const double dot = ((double)vpx - qx) * ax + ((double)vpy - qy) * ay + ((double)vpz - qz) * az;
    if (dot < 0) { ax = -ax; ay = -ay; az = -az; }
    nx[i] = (float)ax;
    ny[i] = (float)ay;
    nz[i] = (float)az;
    if (cond_out) cond_out[i] = (float)cnd;
    if (used64) used64[i] = u64path ? 1 : 0;
  }
}

}  // namespace

void normals_from_lists(rvp_context *ctx, const float *x, const float *y, const float *z,
                        const u64 *pairs, const u64 *offsets, const int32_t *fixed_counts,
                        int fixed_k, size_t n_max, const u64 *n_dev, bool div_centroid, int iters,
                        float vpx, float vpy, float vpz, const float *qx, const float *qy,
                        const float *qz, float *nx, float *ny, float *nz, const u32 *order,
                        const u64 *out_pos) {
  k_normals_lists<<<grid_for(n_max, 128, ctx->num_sms * 32), 128, 0, ctx->stream>>>(
      x, y, z, pairs, offsets, fixed_counts, fixed_k, n_max, n_dev, div_centroid, iters, vpx, vpy,
      vpz, qx, qy, qz, nx, ny, nz, order, out_pos);
  RVP_LAUNCH_CHECK(ctx);
}

void normals_precise(rvp_context *ctx, const float *x, const float *y, const float *z,
                     const u64 *pairs, int kk, size_t n, float vpx, float vpy, float vpz,
                     double cond_fp64, float *nx, float *ny, float *nz, float *cond,
                     uint8_t *used_fp64) {
  k_normals_precise<<<grid_for(n, 128, ctx->num_sms * 32), 128, 0, ctx->stream>>>(
      x, y, z, pairs, kk, n, vpx, vpy, vpz, cond_fp64, nx, ny, nz, cond, used_fp64);
  RVP_LAUNCH_CHECK(ctx);
}

}  // namespace rvp
