// Learned hypothesis proposal for batched RANSAC plane fitting.
//
// Per-point features come from the k = 16 nearest neighbours (17 with the
// point itself) found by the batched grid kNN: the shifted covariance of
// the neighbourhood, its eigen-decomposition (cyclic Jacobi, FP32), the
// K-th neighbour distance and the point's offset from the neighbourhood
// centroid. A per-point MLP 8 -> 64 -> 64 -> 1 (ReLU) scores how likely
// the point lies on the plane plain RANSAC would pick; RANSAC then draws
// its three points with probability proportional to the score
// (ransac.cu, RansacSampler), and the exact inlier count over every
// point still decides between hypotheses.
//
// The network's weights are BF16 (rounded from FP32 master weights after
// every optimiser step); activations, sums and gradients are FP32. Training
// runs on the GPU: one fused kernel does the forward and backward pass of
// 128 points per block and reduces the weight gradients of its points in
// shared memory before one atomic add per weight, then Adam updates the
// master weights.
#include <cuda_bf16.h>
#include <math.h>

#include <algorithm>
#include <new>
#include <vector>

#include "internal.cuh"

using rvp::u32;
using rvp::u64;

namespace rvp {
namespace {

constexpr int MI = RVP_MLP_INPUTS;   // 8
constexpr int MH = RVP_MLP_HIDDEN;   // 64
constexpr int NP = RVP_MLP_PARAMS;   // 4801
constexpr int OW1 = 0, OB1 = OW1 + MH * MI, OW2 = OB1 + MH, OB2 = OW2 + MH * MH,
              OW3 = OB2 + MH, OB3 = OW3 + MH;
static_assert(OB3 + 1 == NP, "parameter layout");
constexpr int KF = 17;  // neighbours per feature point (k = 16 and the point)

// ---------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------
template <int P, int Q>
__device__ __forceinline__ void jacobi_pair(float (&A)[3][3], float (&V)[3][3]) {
  const float apq = A[P][Q];
  if (fabsf(apq) < 1e-30f) return;
  const float theta = (A[Q][Q] - A[P][P]) / (2.0f * apq);
  const float t = copysignf(1.0f, theta) / (fabsf(theta) + sqrtf(theta * theta + 1.0f));
  const float c = rsqrtf(t * t + 1.0f), s = t * c;
  const float app = A[P][P], aqq = A[Q][Q];
  A[P][P] = app - t * apq;
  A[Q][Q] = aqq + t * apq;
  A[P][Q] = A[Q][P] = 0.0f;
  constexpr int R = 3 - P - Q;  // the third index
  const float arp = A[R][P], arq = A[R][Q];
  A[R][P] = A[P][R] = c * arp - s * arq;
  A[R][Q] = A[Q][R] = s * arp + c * arq;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const float vp = V[r][P], vq = V[r][Q];
    V[r][P] = c * vp - s * vq;
    V[r][Q] = s * vp + c * vq;
  }
}

// f0..2 |normal|, f3 curvature, f4 planarity, f5 log K-th distance,
// f6 |offset from the local plane| / r, f7 |offset from the centroid| / r,
// from the offsets (neighbour - point) of the m nearest, in distance order,
// and the squared distance r2 of the last of them
__device__ __forceinline__ void plane_features(const float (&dx)[KF], const float (&dy)[KF],
                                               const float (&dz)[KF], int m, float r2,
                                               float (&f)[MI]) {
  float cx = 0, cy = 0, cz = 0;
#pragma unroll
  for (int j = 0; j < KF; ++j)
    if (j < m) {
      cx += dx[j];
      cy += dy[j];
      cz += dz[j];
    }
  const float inv = 1.0f / (float)m;
  cx *= inv; cy *= inv; cz *= inv;
  float A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int j = 0; j < KF; ++j) {
    if (j < m) {
      const float ex = dx[j] - cx, ey = dy[j] - cy, ez = dz[j] - cz;
      A[0][0] += ex * ex; A[0][1] += ex * ey; A[0][2] += ex * ez;
      A[1][1] += ey * ey; A[1][2] += ey * ez; A[2][2] += ez * ez;
    }
  }
  A[1][0] = A[0][1]; A[2][0] = A[0][2]; A[2][1] = A[1][2];
  float V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll 1
  for (int sweep = 0; sweep < 6; ++sweep) {
    jacobi_pair<0, 1>(A, V);
    jacobi_pair<0, 2>(A, V);
    jacobi_pair<1, 2>(A, V);
  }
  float l0 = A[0][0], l1 = A[1][1], l2 = A[2][2];
  float nx = V[0][0], ny = V[1][0], nz = V[2][0];
  // smallest eigenvalue and its vector; then order the other two
  if (l1 < l0) { const float tl = l0; l0 = l1; l1 = tl; nx = V[0][1]; ny = V[1][1]; nz = V[2][1]; }
  if (l2 < l0) { const float tl = l0; l0 = l2; l2 = tl; nx = V[0][2]; ny = V[1][2]; nz = V[2][2]; }
  if (l2 < l1) { const float tl = l1; l1 = l2; l2 = tl; }
  l0 = fmaxf(l0, 0.0f);
  const float sum = l0 + l1 + l2;
  const float r = sqrtf(r2) + 1e-6f;
  f[0] = fabsf(nx);
  f[1] = fabsf(ny);
  f[2] = fabsf(nz);
  f[3] = sum > 0.0f ? l0 / sum : 1.0f;
  f[4] = l2 > 0.0f ? (l1 - l0) / l2 : 0.0f;
  f[5] = logf(r);
  f[6] = fabsf(nx * cx + ny * cy + nz * cz) / r;
  f[7] = sqrtf(cx * cx + cy * cy + cz * cz) / r;
}

__global__ __launch_bounds__(256) void k_features(const float *__restrict__ x,
                                                  const float *__restrict__ y,
                                                  const float *__restrict__ z,
                                                  const u64 *__restrict__ pairs,
                                                  const int32_t *__restrict__ counts,
                                                  const u32 *__restrict__ cand, size_t n_cand,
                                                  size_t n, float *__restrict__ feat) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n_cand;
       t += (size_t)gridDim.x * blockDim.x) {
    const u32 i = cand ? cand[t] : (u32)t;
    const int m = i < n ? min((int)counts[i], KF) : 0;
    float f[MI] = {0, 0, 0, 1, 0, 0, 0, 0};
    if (m >= 3) {
      const float px = x[i], py = y[i], pz = z[i];
      float dx[KF], dy[KF], dz[KF];
      float r2 = 0.0f;
#pragma unroll
      for (int j = 0; j < KF; ++j) {
        if (j < m) {
          const u64 key = pairs[(size_t)i * KF + j];
          const u32 q = min((u32)(nbr_idx(key) & 0x7FFFFFFF), (u32)(n - 1));
          dx[j] = x[q] - px;
          dy[j] = y[q] - py;
          dz[j] = z[q] - pz;
          r2 = nbr_d2(key);
        } else {
          dx[j] = dy[j] = dz[j] = 0.0f;
        }
      }
      plane_features(dx, dy, dz, m, r2, f);
    }
#pragma unroll
    for (int k = 0; k < MI; ++k) feat[t * MI + k] = f[k];
  }
}

__global__ void k_frame_of(const int64_t *offs, int n_frames, size_t n, int32_t *frame) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = n_frames - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if ((u64)offs[mid] <= i) lo = mid; else hi = mid - 1;
    }
    frame[i] = lo;
  }
}

// Feature neighbourhoods among one scene's candidates (a few thousand
// points at most): each of CK_SLICES blocks per scene keeps the scene's
// candidates in shared memory, sorted into a small grid of its own
// (counting sort over at most CK_CELLS cells of at least the given cell
// size), and answers the queries of a run of whole cells (about one
// CK_SLICES-th of them, in cell order); every query, one per
// thread, takes the exact KF nearest by rings of cells around its own cell
// (the own cell, then shells at Chebyshev distance 1, 2, ...) until the KF-th
// distance lies inside the covered box (its distance to every face that has
// cells beyond it, less a rounding slack) or the box covers the grid,
// skipping cells whose box lies beyond the KF-th distance so far; the
// queries go in cell order, so a warp's lanes walk the same cells. Keys
// are packed (d2, index), so the list is the exact (d2, index) order the
// grid kNN gives; d2 is computed as there. A scene of more than CK_MAX
// candidates is searched by brute force over global memory (exact, slow;
// not reached with the proposal's candidate counts).
constexpr int CK_MAX = 2048, CK_CELLS = 2048, CK_TH = 256;
constexpr int CK_SLICES = 2;  // blocks per scene (each builds the scene's grid)
// the 26 cells around a cell, nearest first: 6 faces, 12 edges, 8 corners
__constant__ signed char kNbr26[26][3] = {
    {-1, 0, 0},  {1, 0, 0},   {0, -1, 0},  {0, 1, 0},   {0, 0, -1},  {0, 0, 1},
    {-1, -1, 0}, {1, -1, 0},  {-1, 1, 0},  {1, 1, 0},   {-1, 0, -1}, {1, 0, -1},
    {-1, 0, 1},  {1, 0, 1},   {0, -1, -1}, {0, 1, -1},  {0, -1, 1},  {0, 1, 1},
    {-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1}, {-1, -1, 1}, {1, -1, 1},
    {-1, 1, 1},  {1, 1, 1}};
constexpr size_t CK_SMEM = (size_t)CK_MAX * 16 + (size_t)(2 * CK_CELLS + 1) * 4 + CK_MAX * 2;

__device__ __forceinline__ void insert_u64(u64 (&L)[KF], u64 key) {
#pragma unroll
  for (int j = KF - 1; j > 0; --j) {
    const u64 a = L[j - 1], b = L[j];
    L[j] = key < a ? a : (key < b ? key : b);
  }
  L[0] = key < L[0] ? key : L[0];
}

__global__ __launch_bounds__(CK_TH) void k_cand_knn(const float *__restrict__ x,
                                                    const float *__restrict__ y,
                                                    const float *__restrict__ z,
                                                    const int64_t *offs, int n_frames,
                                                    float cell, u64 *pairs, int32_t *counts) {
  extern __shared__ __align__(16) unsigned char ck_smem[];
  float4 *sp = reinterpret_cast<float4 *>(ck_smem);                // sorted points
  u32 *cstart = reinterpret_cast<u32 *>(sp + CK_MAX);             // CK_CELLS + 1
  u32 *cursor = cstart + CK_CELLS + 1;                            // CK_CELLS
  uint16_t *cellof = reinterpret_cast<uint16_t *>(cursor + CK_CELLS);  // CK_MAX
  __shared__ float s_bb[3];
  __shared__ float s_wmn[CK_TH / 32][3], s_wmx[CK_TH / 32][3];
  __shared__ int s_dim[3];
  __shared__ float s_cell;
  const int tid = threadIdx.x;
  // work items: (scene, slice); each of a scene's CK_SLICES blocks builds
  // the scene's grid and answers its slice's run of cells
  for (int item = blockIdx.x; item < n_frames * CK_SLICES; item += gridDim.x) {
    const int f = item / CK_SLICES, slice = item % CK_SLICES;
    const int64_t a = offs[f], b = offs[f + 1];
    const int m = (int)(b - a);
    if (m <= 0) continue;
    if (m > CK_MAX) {  // brute force over global memory
      for (int i = tid + slice * CK_TH; i < m; i += CK_SLICES * CK_TH) {
        const float qx = x[a + i], qy = y[a + i], qz = z[a + i];
        u64 L[KF];
#pragma unroll
        for (int j = 0; j < KF; ++j) L[j] = ~0ull;
        for (int t = 0; t < m; ++t) {
          const u64 key = pack_nbr(dist2(x[a + t], y[a + t], z[a + t], qx, qy, qz), (int)(a + t));
          if (key < L[KF - 1]) insert_u64(L, key);
        }
#pragma unroll
        for (int j = 0; j < KF; ++j) pairs[(size_t)(a + i) * KF + j] = L[j];
        counts[a + i] = min(m, KF);
      }
      continue;
    }
    // bounding box
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = tid; i < m; i += CK_TH) {
      const float v[3] = {x[a + i], y[a + i], z[a + i]};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        mn[k] = fminf(mn[k], v[k]);
        mx[k] = fmaxf(mx[k], v[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k)
      for (int o = 16; o; o >>= 1) {
        mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
        mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
      }
    // the block's min / max through a per-warp table
    if ((tid & 31) == 0)
      for (int k = 0; k < 3; ++k) {
        s_wmn[tid >> 5][k] = mn[k];
        s_wmx[tid >> 5][k] = mx[k];
      }
    __syncthreads();
    if (tid == 0) {
      float bmn[3] = {INFINITY, INFINITY, INFINITY}, bmx[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int w = 0; w < CK_TH / 32; ++w)
        for (int k = 0; k < 3; ++k) {
          bmn[k] = fminf(bmn[k], s_wmn[w][k]);
          bmx[k] = fmaxf(bmx[k], s_wmx[w][k]);
        }
      // the grid: cells of at least `cell`, at most CK_CELLS of them
      float c = cell;
      int d[3];
      for (int it = 0; it < 64; ++it) {
        long long tot = 1;
        for (int k = 0; k < 3; ++k) {
          d[k] = (int)floorf((bmx[k] - bmn[k]) / c) + 1;
          d[k] = max(d[k], 1);
          tot *= d[k];
        }
        if (tot <= CK_CELLS) break;
        c *= 1.26f;
      }
      for (int k = 0; k < 3; ++k) {
        s_bb[k] = bmn[k];
        s_dim[k] = d[k];
      }
      s_cell = c;
    }
    __syncthreads();
    const float c = s_cell, ic = 1.0f / c;
    const int GX = s_dim[0], GY = s_dim[1], GZ = s_dim[2];
    const float mnx = s_bb[0], mny = s_bb[1], mnz = s_bb[2];
    auto cax = [&](float v, float m0, int G) { return min(max((int)((v - m0) * ic), 0), G - 1); };
    // counting sort into the cells
    for (int j = tid; j < CK_CELLS; j += CK_TH) cursor[j] = 0;
    __syncthreads();
    for (int i = tid; i < m; i += CK_TH) {
      const int cid = (cax(z[a + i], mnz, GZ) * GY + cax(y[a + i], mny, GY)) * GX +
                      cax(x[a + i], mnx, GX);
      cellof[i] = (uint16_t)cid;
      atomicAdd(&cursor[cid], 1u);
    }
    __syncthreads();
    if (tid < 32) {  // exclusive scan of the cell counts (one warp)
      u32 run = 0;
      for (int base = 0; base < CK_CELLS; base += 32) {
        const u32 v = cursor[base + tid];
        u32 incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const u32 t = __shfl_up_sync(0xffffffffu, incl, o);
          if (tid >= o) incl += t;
        }
        cstart[base + tid] = run + incl - v;
        run += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (tid == 0) cstart[CK_CELLS] = run;
    }
    __syncthreads();
    for (int j = tid; j < CK_CELLS; j += CK_TH) cursor[j] = cstart[j];
    __syncthreads();
    for (int i = tid; i < m; i += CK_TH) {
      const u32 p = atomicAdd(&cursor[cellof[i]], 1u);
      sp[p] = make_float4(x[a + i], y[a + i], z[a + i], __int_as_float((int)(a + i)));
    }
    __syncthreads();
    // this block's queries: a run of whole cells in cell order, from the
    // start of the cell holding sorted position slice * m / CK_SLICES to
    // that of the next slice (the cell starts are the same in every block
    // of the scene, while the order inside a cell is not: whole cells keep
    // the split exact); a warp's lanes work on neighbouring points, the same
    // cells, the same ring counts
    auto slice_start = [&](int k) -> int {
      if (k <= 0) return 0;
      if (k >= CK_SLICES) return m;
      const u32 pos = (u32)((long long)k * m / CK_SLICES);
      int lo = 0, hi = CK_CELLS - 1;  // the last cell starting at or before pos
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cstart[mid] <= pos) lo = mid; else hi = mid - 1;
      }
      return (int)cstart[lo];
    };
    const int q0 = slice_start(slice), q1 = slice_start(slice + 1);
    for (int j = q0 + tid; j < q1; j += CK_TH) {
      const float4 qp = sp[j];
      const float qx = qp.x, qy = qp.y, qz = qp.z;
      const int64_t qo = __float_as_int(qp.w);  // its index in the candidate cloud
      const int cx = cax(qx, mnx, GX), cy = cax(qy, mny, GY), cz = cax(qz, mnz, GZ);
      u64 L[KF];
#pragma unroll
      for (int j = 0; j < KF; ++j) L[j] = ~0ull;
      int found = 0;
      // rounding slack of the cell function and the face positions
      const float sl = 4e-6f * (fabsf(mnx) + fabsf(mny) + fabsf(mnz) + fabsf(qx) + fabsf(qy) +
                                fabsf(qz) + (float)(GX + GY + GZ + 3) * c) + 1e-6f;
      // one cell: skipped when its box lies beyond the current KF-th
      // distance (once the list is full), else its points tested
      auto visit = [&](int ux, int uy, int uz, bool test_box) {
        if (ux < 0 || ux >= GX || uy < 0 || uy >= GY || uz < 0 || uz >= GZ) return;
        if (test_box) {
          const float lx = mnx + (float)ux * c, ly = mny + (float)uy * c,
                      lz = mnz + (float)uz * c;
          const float gx = fmaxf(fmaxf(lx - sl - qx, qx - (lx + c + sl)), 0.0f);
          const float gy = fmaxf(fmaxf(ly - sl - qy, qy - (ly + c + sl)), 0.0f);
          const float gz = fmaxf(fmaxf(lz - sl - qz, qz - (lz + c + sl)), 0.0f);
          if ((gx * gx + gy * gy + gz * gz) * (1.0f - 1e-5f) > nbr_d2(L[KF - 1])) return;
        }
        const int cid = (uz * GY + uy) * GX + ux;
        for (u32 t = cstart[cid]; t < cstart[cid + 1]; ++t) {
          const float4 p = sp[t];
          const u64 key = pack_nbr(dist2(p.x, p.y, p.z, qx, qy, qz), __float_as_int(p.w));
          ++found;
          if (key < L[KF - 1]) insert_u64(L, key);
        }
      };
      for (int r = 0;; ++r) {
        if (r == 0) {
          visit(cx, cy, cz, false);
        } else if (r == 1) {  // nearest first: faces, edges, corners
          for (int t = 0; t < 26; ++t)
            visit(cx + kNbr26[t][0], cy + kNbr26[t][1], cz + kNbr26[t][2], true);
        } else {
          for (int dz = -r; dz <= r; ++dz)
            for (int dy = -r; dy <= r; ++dy) {
              const bool edge = dz == -r || dz == r || dy == -r || dy == r;
              for (int dx = -r; dx <= r; dx += (edge ? 1 : 2 * r))
                visit(cx + dx, cy + dy, cz + dz, true);
            }
        }
        // the box of rings 0..r: all points found, or the KF-th inside it
        const bool all = cx - r <= 0 && cy - r <= 0 && cz - r <= 0 && cx + r >= GX - 1 &&
                         cy + r >= GY - 1 && cz + r >= GZ - 1;
        if (all) break;
        if (found >= KF) {
          float cov = INFINITY;
          if (cx - r > 0) cov = fminf(cov, qx - (mnx + (float)(cx - r) * c));
          if (cx + r < GX - 1) cov = fminf(cov, (mnx + (float)(cx + r + 1) * c) - qx);
          if (cy - r > 0) cov = fminf(cov, qy - (mny + (float)(cy - r) * c));
          if (cy + r < GY - 1) cov = fminf(cov, (mny + (float)(cy + r + 1) * c) - qy);
          if (cz - r > 0) cov = fminf(cov, qz - (mnz + (float)(cz - r) * c));
          if (cz + r < GZ - 1) cov = fminf(cov, (mnz + (float)(cz + r + 1) * c) - qz);
          cov -= sl;
          if (cov > 0.0f && nbr_d2(L[KF - 1]) < cov * cov * (1.0f - 1e-5f)) break;
        }
      }
#pragma unroll
      for (int j = 0; j < KF; ++j) pairs[(size_t)qo * KF + j] = L[j];
      counts[qo] = min(m, KF);
    }
    __syncthreads();  // the shared arrays are reused by the next scene
  }
}

__global__ void k_mark_cand(const u32 *cand, size_t n_cand, size_t n, uint8_t *is_cand) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n_cand;
       t += (size_t)gridDim.x * blockDim.x)
    if (cand[t] < n) is_cand[cand[t]] = 1;
}

// grid positions of the candidates open at level 0, the rest done
__global__ void k_open_cand(const float4 *pts, const u64 *n_dev, const uint8_t *is_cand,
                            uint8_t *qlevel) {
  const u64 n = *n_dev;
  for (u64 pos = blockIdx.x * (u64)blockDim.x + threadIdx.x; pos < n;
       pos += (u64)gridDim.x * blockDim.x) {
    const u32 idx = __float_as_uint(pts[pos].w) & 0x7FFFFFFFu;
    qlevel[pos] = (!is_cand || is_cand[idx]) ? 0 : 0xFF;
  }
}

__global__ void k_gather_xyz(const float *x, const float *y, const float *z, const u32 *idx,
                             size_t n, size_t n_src, float *ox, float *oy, float *oz) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const u32 i = idx[t] < n_src ? idx[t] : 0;
    ox[t] = x[i];
    oy[t] = y[i];
    oz[t] = z[i];
  }
}

__global__ void k_widen32(const u32 *a, u64 *b) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *b = *a;
}

// ---------------------------------------------------------------------------
// MLP
// ---------------------------------------------------------------------------
__global__ void k_quantize(const float *w, __nv_bfloat16 *wq, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    wq[i] = __float2bfloat16_rn(w[i]);
}

__device__ __forceinline__ void load_weights(const __nv_bfloat16 *wq, const float *norm,
                                             float *sw, float *snorm) {
  for (int i = threadIdx.x; i < NP; i += blockDim.x) sw[i] = __bfloat162float(wq[i]);
  for (int i = threadIdx.x; i < 2 * MI; i += blockDim.x) snorm[i] = norm[i];
  __syncthreads();
}

__device__ __forceinline__ void normalise(const float *__restrict__ feat, size_t i,
                                          const float *snorm, float (&xn)[MI]) {
#pragma unroll
  for (int k = 0; k < MI; ++k) xn[k] = (feat[i * MI + k] - snorm[k]) * snorm[MI + k];
}

// ---------------------------------------------------------------------------
// Tensor-core forward pass (mma.sync, FP32 accumulation): one warp per tile
// of 16 points. Layer 1 (8 -> 64) is one m16n8k8 TF32 MMA per 8 hidden
// units (inputs rounded to TF32, the BF16 weights exactly representable);
// layer 2 (64 -> 64) four m16n8k16 BF16 MMAs per 8 units, its A fragments
// being layer 1's accumulators (bias, ReLU, rounded to BF16) in place --
// the C layout of two n8 tiles is the A layout of one k16 step; layer 3
// (64 -> 1) is a dot product of the accumulators with w3, reduced over the
// four lanes that share a row. Both weight matrices stay in registers as
// MMA fragments for the warp's whole run.
// ---------------------------------------------------------------------------
__device__ __forceinline__ u32 to_tf32(float f) {
  u32 r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
  return r;
}
__device__ __forceinline__ u32 pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // lo in the low half
  return *reinterpret_cast<const u32 *>(&v);
}
__device__ __forceinline__ void mma_tf32_16x8x8(float (&c)[4], const u32 (&a)[4], u32 b0, u32 b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ void mma_bf16_16x8x16(float (&c)[4], const u32 (&a)[4], u32 b0,
                                                 u32 b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

constexpr int FWD_THREADS = 128;

__global__ __launch_bounds__(FWD_THREADS) void k_mlp_forward(const float *__restrict__ feat,
                                                             size_t n,
                                                             const __nv_bfloat16 *__restrict__ wq,
                                                             const float *__restrict__ norm,
                                                             float *__restrict__ logits) {
  __shared__ float sv[3 * MH + 1];  // b1 | b2 | w3 | b3
  __shared__ float snorm[2 * MI];
  // b1 sits before W2, b2 | w3 | b3 after it
  for (int i = threadIdx.x; i < 3 * MH + 1; i += blockDim.x)
    sv[i] = __bfloat162float(wq[i < MH ? OB1 + i : OB2 + (i - MH)]);
  for (int i = threadIdx.x; i < 2 * MI; i += blockDim.x) snorm[i] = norm[i];
  __syncthreads();
  const float *b1 = sv, *b2 = sv + MH, *w3 = sv + 2 * MH;
  const float b3 = sv[3 * MH];
  const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  // B fragments: W1 (TF32, k = input, n = hidden unit), W2 (BF16 pairs)
  u32 w1f[8][2];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int h = nt * 8 + g;
    w1f[nt][0] = to_tf32(__bfloat162float(wq[OW1 + h * MI + tig]));
    w1f[nt][1] = to_tf32(__bfloat162float(wq[OW1 + h * MI + tig + 4]));
  }
  u32 w2f[8][4][2];
  const u32 *wq32 = reinterpret_cast<const u32 *>(wq);
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const int e = OW2 + (nt * 8 + g) * MH + ks * 16 + 2 * tig;  // even: a BF16 pair
      w2f[nt][ks][0] = __ldg(&wq32[e >> 1]);
      w2f[nt][ks][1] = __ldg(&wq32[(e + 8) >> 1]);
    }
  const float m0 = snorm[tig], m1 = snorm[tig + 4];
  const float s0 = snorm[MI + tig], s1 = snorm[MI + tig + 4];
  const size_t tiles = (n + 15) / 16;
  const size_t warps = (size_t)gridDim.x * (FWD_THREADS / 32);
  for (size_t tile = (size_t)blockIdx.x * (FWD_THREADS / 32) + (threadIdx.x >> 5); tile < tiles;
       tile += warps) {
    const size_t r0 = tile * 16 + g, r1 = r0 + 8;
    const bool v0 = r0 < n, v1 = r1 < n;
    u32 a1[4];
    a1[0] = to_tf32(v0 ? (feat[r0 * MI + tig] - m0) * s0 : 0.0f);
    a1[1] = to_tf32(v1 ? (feat[r1 * MI + tig] - m0) * s0 : 0.0f);
    a1[2] = to_tf32(v0 ? (feat[r0 * MI + tig + 4] - m1) * s1 : 0.0f);
    a1[3] = to_tf32(v1 ? (feat[r1 * MI + tig + 4] - m1) * s1 : 0.0f);
    u32 a2[4][4];
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      float c0[4] = {0.0f, 0.0f, 0.0f, 0.0f}, c1[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      mma_tf32_16x8x8(c0, a1, w1f[2 * ks][0], w1f[2 * ks][1]);
      mma_tf32_16x8x8(c1, a1, w1f[2 * ks + 1][0], w1f[2 * ks + 1][1]);
      const int j0 = 16 * ks + 2 * tig, j1 = j0 + 8;
      a2[ks][0] = pack_bf16x2(fmaxf(c0[0] + b1[j0], 0.0f), fmaxf(c0[1] + b1[j0 + 1], 0.0f));
      a2[ks][1] = pack_bf16x2(fmaxf(c0[2] + b1[j0], 0.0f), fmaxf(c0[3] + b1[j0 + 1], 0.0f));
      a2[ks][2] = pack_bf16x2(fmaxf(c1[0] + b1[j1], 0.0f), fmaxf(c1[1] + b1[j1 + 1], 0.0f));
      a2[ks][3] = pack_bf16x2(fmaxf(c1[2] + b1[j1], 0.0f), fmaxf(c1[3] + b1[j1 + 1], 0.0f));
    }
    float o0 = 0.0f, o1 = 0.0f;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) mma_bf16_16x8x16(c, a2[ks], w2f[nt][ks][0], w2f[nt][ks][1]);
      const int j = nt * 8 + 2 * tig;
      o0 = fmaf(w3[j], fmaxf(c[0] + b2[j], 0.0f), o0);
      o0 = fmaf(w3[j + 1], fmaxf(c[1] + b2[j + 1], 0.0f), o0);
      o1 = fmaf(w3[j], fmaxf(c[2] + b2[j], 0.0f), o1);
      o1 = fmaf(w3[j + 1], fmaxf(c[3] + b2[j + 1], 0.0f), o1);
    }
    o0 += __shfl_xor_sync(0xffffffffu, o0, 1);
    o0 += __shfl_xor_sync(0xffffffffu, o0, 2);
    o1 += __shfl_xor_sync(0xffffffffu, o1, 1);
    o1 += __shfl_xor_sync(0xffffffffu, o1, 2);
    if (tig == 0) {
      if (v0) logits[r0] = o0 + b3;
      if (v1) logits[r1] = o1 + b3;
    }
  }
}

// ---------------------------------------------------------------------------
// Training step on tensor cores: forward and backward of the mean binary
// cross-entropy with logits, 64 points per block iteration (4 warps x 16).
// Phase A (each warp, its 16 points): the forward pass as in k_mlp_forward,
// the output gradient g = (sigmoid(out) - y) / n, delta2 = g * w3 * [h2 > 0]
// and delta1 = (delta2 W2) * [h1 > 0], the latter as m16n8k16 BF16 MMAs
// with delta2's accumulators as A fragments and W2 transposed in shared
// memory as B; delta2, h1, delta1 and the normalised inputs go to shared
// memory transposed (BF16), the bias and w3 sums of the 16 points (FP32) too.
// Phase B (warp w owns rows 16w..16w+15 of dW2 and dW1): dW2 = delta2^T H1
// and dW1 = delta1^T X as MMAs over the iteration's 64 points, accumulated in
// registers across iterations; the vector entries are added in warp order.
// Every gradient entry of a block is written by one thread, and the blocks'
// shares are added in block order afterwards (k_grad_reduce): the same batch
// always gives the same gradient.
// ---------------------------------------------------------------------------
constexpr int TB = 128;                 // threads per training block
constexpr int TP = 64;                  // points per block iteration
constexpr int TS = 72;                  // row stride (BF16) of the shared tiles: no bank conflicts
constexpr int NV = 3 * MH + 1;          // b1 | b2 | w3 | b3
struct TrainSmem {
  __nv_bfloat16 w2[MH * TS];   // W2[j][h]
  __nv_bfloat16 w2t[MH * TS];  // W2[j][h] at [h][j]
  __nv_bfloat16 d2t[MH * TS];  // delta2[m][j] at [j][m]
  __nv_bfloat16 h1t[MH * TS];  // h1[m][h] at [h][m]
  __nv_bfloat16 d1t[MH * TS];  // delta1[m][h] at [h][m]
  __nv_bfloat16 xt[MI * TS];   // x[m][k] at [k][m]
  float vec[NV + 3];
  float norm[2 * MI];
  float vpart[TB / 32][NV + 3];  // per warp: sums of the vector gradients over its points
  double warp_loss[TB / 32];
};
constexpr size_t TRAIN_SMEM = sizeof(TrainSmem);

__device__ __forceinline__ u32 lds32(const __nv_bfloat16 *p) {
  return *reinterpret_cast<const u32 *>(p);
}

__global__ __launch_bounds__(TB) void k_mlp_train(const float *__restrict__ feat,
                                                  const float *__restrict__ labels, size_t n,
                                                  size_t n_src, u64 sample_seed,
                                                  const __nv_bfloat16 *__restrict__ wq,
                                                  const float *__restrict__ norm, float *part,
                                                  double *part_loss) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TrainSmem &S = *reinterpret_cast<TrainSmem *>(smraw);
  float *grad = part + (size_t)blockIdx.x * NP;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane >> 2, tig = lane & 3;
  for (int i = tid; i < MH * MH; i += TB) {
    const int j = i / MH, h = i % MH;
    const __nv_bfloat16 v = wq[OW2 + i];
    S.w2[j * TS + h] = v;
    S.w2t[h * TS + j] = v;
  }
  for (int i = tid; i < NV; i += TB) S.vec[i] = __bfloat162float(wq[i < MH ? OB1 + i : OB2 + (i - MH)]);
  for (int i = tid; i < 2 * MI; i += TB) S.norm[i] = norm[i];
  __syncthreads();
  const float *b1 = S.vec, *b2 = S.vec + MH, *w3 = S.vec + 2 * MH;
  const float b3 = S.vec[3 * MH];
  u32 w1f[8][2];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int h = nt * 8 + g;
    w1f[nt][0] = to_tf32(__bfloat162float(wq[OW1 + h * MI + tig]));
    w1f[nt][1] = to_tf32(__bfloat162float(wq[OW1 + h * MI + tig + 4]));
  }
  const float m0 = S.norm[tig], m1 = S.norm[tig + 4];
  const float s0 = S.norm[MI + tig], s1 = S.norm[MI + tig + 4];
  const float inv_n = 1.0f / (float)n;
  float gw2[8][4], gw1[4] = {0.0f, 0.0f, 0.0f, 0.0f}, gv[2] = {0.0f, 0.0f};
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int r = 0; r < 4; ++r) gw2[nt][r] = 0.0f;
  float loss = 0.0f;
  const int mr0 = 16 * w + g, mr1 = mr0 + 8;  // this thread's rows within the iteration
  for (size_t base = (size_t)blockIdx.x * TP; base < n; base += (size_t)gridDim.x * TP) {
    // ---- phase A: forward and backward of this warp's 16 points
    const size_t slot0 = base + mr0, slot1 = base + mr1;
    const bool v0 = slot0 < n, v1 = slot1 < n;
    const size_t i0 = sample_seed ? (size_t)(mix64(sample_seed ^ mix64(slot0)) % n_src) : slot0;
    const size_t i1 = sample_seed ? (size_t)(mix64(sample_seed ^ mix64(slot1)) % n_src) : slot1;
    const float x00 = v0 ? (feat[i0 * MI + tig] - m0) * s0 : 0.0f;
    const float x10 = v1 ? (feat[i1 * MI + tig] - m0) * s0 : 0.0f;
    const float x01 = v0 ? (feat[i0 * MI + tig + 4] - m1) * s1 : 0.0f;
    const float x11 = v1 ? (feat[i1 * MI + tig + 4] - m1) * s1 : 0.0f;
    S.xt[tig * TS + mr0] = __float2bfloat16_rn(x00);
    S.xt[tig * TS + mr1] = __float2bfloat16_rn(x10);
    S.xt[(tig + 4) * TS + mr0] = __float2bfloat16_rn(x01);
    S.xt[(tig + 4) * TS + mr1] = __float2bfloat16_rn(x11);
    const u32 a1[4] = {to_tf32(x00), to_tf32(x10), to_tf32(x01), to_tf32(x11)};
    u32 a2[4][4];  // h1 as layer-2 A fragments (BF16)
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      float c0[4] = {0.0f, 0.0f, 0.0f, 0.0f}, c1[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      mma_tf32_16x8x8(c0, a1, w1f[2 * ks][0], w1f[2 * ks][1]);
      mma_tf32_16x8x8(c1, a1, w1f[2 * ks + 1][0], w1f[2 * ks + 1][1]);
      const int j0 = 16 * ks + 2 * tig, j1 = j0 + 8;
      a2[ks][0] = pack_bf16x2(fmaxf(c0[0] + b1[j0], 0.0f), fmaxf(c0[1] + b1[j0 + 1], 0.0f));
      a2[ks][1] = pack_bf16x2(fmaxf(c0[2] + b1[j0], 0.0f), fmaxf(c0[3] + b1[j0 + 1], 0.0f));
      a2[ks][2] = pack_bf16x2(fmaxf(c1[0] + b1[j1], 0.0f), fmaxf(c1[1] + b1[j1 + 1], 0.0f));
      a2[ks][3] = pack_bf16x2(fmaxf(c1[2] + b1[j1], 0.0f), fmaxf(c1[3] + b1[j1 + 1], 0.0f));
      // h1 transposed for dW2: (h, m) pairs of this thread
      const __nv_bfloat162 *q = reinterpret_cast<const __nv_bfloat162 *>(a2[ks]);
      S.h1t[j0 * TS + mr0] = q[0].x; S.h1t[(j0 + 1) * TS + mr0] = q[0].y;
      S.h1t[j0 * TS + mr1] = q[1].x; S.h1t[(j0 + 1) * TS + mr1] = q[1].y;
      S.h1t[j1 * TS + mr0] = q[2].x; S.h1t[(j1 + 1) * TS + mr0] = q[2].y;
      S.h1t[j1 * TS + mr1] = q[3].x; S.h1t[(j1 + 1) * TS + mr1] = q[3].y;
    }
    float h2[8][4];
    float o0 = 0.0f, o1 = 0.0f;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
      for (int r = 0; r < 4; ++r) h2[nt][r] = 0.0f;
      const __nv_bfloat16 *wr = S.w2 + (nt * 8 + g) * TS + 2 * tig;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        mma_bf16_16x8x16(h2[nt], a2[ks], lds32(wr + 16 * ks), lds32(wr + 16 * ks + 8));
      const int j = nt * 8 + 2 * tig;
      h2[nt][0] = fmaxf(h2[nt][0] + b2[j], 0.0f);
      h2[nt][1] = fmaxf(h2[nt][1] + b2[j + 1], 0.0f);
      h2[nt][2] = fmaxf(h2[nt][2] + b2[j], 0.0f);
      h2[nt][3] = fmaxf(h2[nt][3] + b2[j + 1], 0.0f);
      o0 = fmaf(w3[j], h2[nt][0], fmaf(w3[j + 1], h2[nt][1], o0));
      o1 = fmaf(w3[j], h2[nt][2], fmaf(w3[j + 1], h2[nt][3], o1));
    }
    o0 += __shfl_xor_sync(0xffffffffu, o0, 1);
    o0 += __shfl_xor_sync(0xffffffffu, o0, 2);
    o1 += __shfl_xor_sync(0xffffffffu, o1, 1);
    o1 += __shfl_xor_sync(0xffffffffu, o1, 2);
    o0 += b3;
    o1 += b3;
    float g0 = 0.0f, g1 = 0.0f;
    if (v0) {
      const float yl = labels[i0];
      if (tig == 0) loss += fmaxf(o0, 0.0f) - yl * o0 + log1pf(expf(-fabsf(o0)));
      g0 = (1.0f / (1.0f + expf(-o0)) - yl) * inv_n;
    }
    if (v1) {
      const float yl = labels[i1];
      if (tig == 0) loss += fmaxf(o1, 0.0f) - yl * o1 + log1pf(expf(-fabsf(o1)));
      g1 = (1.0f / (1.0f + expf(-o1)) - yl) * inv_n;
    }
    // delta2 (in h2's place), its sums and w3's gradient sums over the rows
    float sb2[16], sw3[16];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int j = nt * 8 + 2 * tig;
      const float d00 = h2[nt][0] > 0.0f ? g0 * w3[j] : 0.0f;
      const float d01 = h2[nt][1] > 0.0f ? g0 * w3[j + 1] : 0.0f;
      const float d10 = h2[nt][2] > 0.0f ? g1 * w3[j] : 0.0f;
      const float d11 = h2[nt][3] > 0.0f ? g1 * w3[j + 1] : 0.0f;
      sw3[2 * nt] = g0 * h2[nt][0] + g1 * h2[nt][2];
      sw3[2 * nt + 1] = g0 * h2[nt][1] + g1 * h2[nt][3];
      sb2[2 * nt] = d00 + d10;
      sb2[2 * nt + 1] = d01 + d11;
      h2[nt][0] = d00; h2[nt][1] = d01; h2[nt][2] = d10; h2[nt][3] = d11;
    }
    u32 ad[4][4];  // delta2 as A fragments (BF16), and transposed for dW2
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      ad[ks][0] = pack_bf16x2(h2[2 * ks][0], h2[2 * ks][1]);
      ad[ks][1] = pack_bf16x2(h2[2 * ks][2], h2[2 * ks][3]);
      ad[ks][2] = pack_bf16x2(h2[2 * ks + 1][0], h2[2 * ks + 1][1]);
      ad[ks][3] = pack_bf16x2(h2[2 * ks + 1][2], h2[2 * ks + 1][3]);
      const int j0 = 16 * ks + 2 * tig, j1 = j0 + 8;
      const __nv_bfloat162 *q = reinterpret_cast<const __nv_bfloat162 *>(ad[ks]);
      S.d2t[j0 * TS + mr0] = q[0].x; S.d2t[(j0 + 1) * TS + mr0] = q[0].y;
      S.d2t[j0 * TS + mr1] = q[1].x; S.d2t[(j0 + 1) * TS + mr1] = q[1].y;
      S.d2t[j1 * TS + mr0] = q[2].x; S.d2t[(j1 + 1) * TS + mr0] = q[2].y;
      S.d2t[j1 * TS + mr1] = q[3].x; S.d2t[(j1 + 1) * TS + mr1] = q[3].y;
    }
    // delta1 = (delta2 W2) * [h1 > 0]; its sums
    float sb1[16];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      const __nv_bfloat16 *wr = S.w2t + (nt * 8 + g) * TS + 2 * tig;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        mma_bf16_16x8x16(c, ad[ks], lds32(wr + 16 * ks), lds32(wr + 16 * ks + 8));
      // h1 > 0 at (rows, cols nt*8 + 2 tig + {0, 1}): from the A fragments
      const __nv_bfloat162 *q = reinterpret_cast<const __nv_bfloat162 *>(a2[nt >> 1]);
      const int o = (nt & 1) * 2;
      const float d00 = __bfloat162float(q[o].x) > 0.0f ? c[0] : 0.0f;
      const float d01 = __bfloat162float(q[o].y) > 0.0f ? c[1] : 0.0f;
      const float d10 = __bfloat162float(q[o + 1].x) > 0.0f ? c[2] : 0.0f;
      const float d11 = __bfloat162float(q[o + 1].y) > 0.0f ? c[3] : 0.0f;
      sb1[2 * nt] = d00 + d10;
      sb1[2 * nt + 1] = d01 + d11;
      const int h = nt * 8 + 2 * tig;
      S.d1t[h * TS + mr0] = __float2bfloat16_rn(d00);
      S.d1t[(h + 1) * TS + mr0] = __float2bfloat16_rn(d01);
      S.d1t[h * TS + mr1] = __float2bfloat16_rn(d10);
      S.d1t[(h + 1) * TS + mr1] = __float2bfloat16_rn(d11);
    }
    // the warp's vector sums: rows of the lanes with the same tig, then one
    // lane per column writes
#pragma unroll
    for (int e = 0; e < 16; ++e) {
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        sb1[e] += __shfl_xor_sync(0xffffffffu, sb1[e], o);
        sb2[e] += __shfl_xor_sync(0xffffffffu, sb2[e], o);
        sw3[e] += __shfl_xor_sync(0xffffffffu, sw3[e], o);
      }
    }
    float gs = g0 + g1;  // b3: the 16 rows' g
#pragma unroll
    for (int o = 4; o < 32; o <<= 1) gs += __shfl_xor_sync(0xffffffffu, gs, o);
    if (g == 0) {
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const int c = nt * 8 + 2 * tig;
        S.vpart[w][c] = sb1[2 * nt];
        S.vpart[w][c + 1] = sb1[2 * nt + 1];
        S.vpart[w][MH + c] = sb2[2 * nt];
        S.vpart[w][MH + c + 1] = sb2[2 * nt + 1];
        S.vpart[w][2 * MH + c] = sw3[2 * nt];
        S.vpart[w][2 * MH + c + 1] = sw3[2 * nt + 1];
      }
      if (tig == 0) S.vpart[w][3 * MH] = gs;
    }
    __syncthreads();
    // ---- phase B: this warp's rows of dW2 and dW1 over the 64 points
#pragma unroll
    for (int ks = 0; ks < TP / 16; ++ks) {
      const __nv_bfloat16 *ar = S.d2t + (16 * w + g) * TS + 16 * ks + 2 * tig;
      const u32 a[4] = {lds32(ar), lds32(ar + 8 * TS), lds32(ar + 8), lds32(ar + 8 * TS + 8)};
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const __nv_bfloat16 *br = S.h1t + (nt * 8 + g) * TS + 16 * ks + 2 * tig;
        mma_bf16_16x8x16(gw2[nt], a, lds32(br), lds32(br + 8));
      }
      const __nv_bfloat16 *dr = S.d1t + (16 * w + g) * TS + 16 * ks + 2 * tig;
      const u32 ad1[4] = {lds32(dr), lds32(dr + 8 * TS), lds32(dr + 8), lds32(dr + 8 * TS + 8)};
      const __nv_bfloat16 *xr = S.xt + g * TS + 16 * ks + 2 * tig;
      mma_bf16_16x8x16(gw1, ad1, lds32(xr), lds32(xr + 8));
    }
    // vector entries tid and tid + TB, the warps' sums in warp order
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int v = tid + e * TB;
      if (v < NV) {
        float t = 0.0f;
#pragma unroll
        for (int q = 0; q < TB / 32; ++q) t += S.vpart[q][v];
        gv[e] += t;
      }
    }
    __syncthreads();  // the tiles are rewritten next iteration
  }
  // this block's share of the gradient: each entry written by one thread
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const int j = 16 * w + g, h = nt * 8 + 2 * tig;
    grad[OW2 + j * MH + h] = gw2[nt][0];
    grad[OW2 + j * MH + h + 1] = gw2[nt][1];
    grad[OW2 + (j + 8) * MH + h] = gw2[nt][2];
    grad[OW2 + (j + 8) * MH + h + 1] = gw2[nt][3];
  }
  {
    const int h = 16 * w + g, k = 2 * tig;
    grad[OW1 + h * MI + k] = gw1[0];
    grad[OW1 + h * MI + k + 1] = gw1[1];
    grad[OW1 + (h + 8) * MI + k] = gw1[2];
    grad[OW1 + (h + 8) * MI + k + 1] = gw1[3];
  }
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int v = tid + e * TB;
    if (v < NV) grad[v < MH ? OB1 + v : OB2 + (v - MH)] = gv[e];
  }
  // loss: warp sums, then the warps in order
  for (int o = 16; o; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  if (lane == 0) S.warp_loss[w] = (double)loss;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int q = 0; q < TB / 32; ++q) t += S.warp_loss[q];
    part_loss[blockIdx.x] = t;
  }
}

// the blocks' gradient shares and losses, added in block order
__global__ void k_grad_reduce(const float *part, const double *part_loss, int blocks, float *grad,
                              double *loss_sum) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < NP; p += gridDim.x * blockDim.x) {
    float t = 0.0f;
    for (int b = 0; b < blocks; ++b) t += part[(size_t)b * NP + p];
    grad[p] = t;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double t = 0.0;
    for (int b = 0; b < blocks; ++b) t += part_loss[b];
    *loss_sum = t;
  }
}

__global__ void k_adam(float *w, const float *g, float *m, float *v, int n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

// per-frame inclusive prefix sums (double) of candidate weights; one block
// per frame
__device__ __forceinline__ double cand_weight(float w, float logit_power) {
  if (logit_power > 0.0f) {  // w is a logit: sigmoid(w) ^ power
    const double p = 1.0 / (1.0 + exp(-(double)w));
    return pow(p, (double)logit_power);
  }
  return (double)fmaxf(w, 0.0f);
}

__global__ __launch_bounds__(256) void k_cdf(const float *w, float logit_power,
                                             const int64_t *coffs, double *cdf) {
  const int f = blockIdx.x;
  const int64_t a = coffs[f], b = coffs[f + 1];
  __shared__ double warp_tot[8];
  __shared__ double carry;
  if (threadIdx.x == 0) carry = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int64_t c0 = a; c0 < b; c0 += 256) {
    const int64_t i = c0 + threadIdx.x;
    double v = i < b ? cand_weight(w[i], logit_power) : 0.0;
    for (int o = 1; o < 32; o <<= 1) {
      const double t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    if (lane == 31) warp_tot[wid] = v;
    __syncthreads();
    double before = carry;
    for (int k = 0; k < wid; ++k) before += warp_tot[k];
    if (i < b) cdf[i] = before + v;
    __syncthreads();
    if (threadIdx.x == 255) carry = before + v;
    __syncthreads();
  }
}

// labels: 1 for points within thresh of their frame's model, else 0
__global__ void k_plane_labels(const float *x, const float *y, const float *z, const int32_t *frame,
                               size_t n, const float *models, float t, float *labels) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float *m = models + 4 * frame[i];
    const float d = fadd(fadd(fadd(fmul(m[0], x[i]), fmul(m[1], y[i])), fmul(m[2], z[i])), m[3]);
    labels[i] = fabsf(d) <= t ? 1.0f : 0.0f;
  }
}

}  // namespace
}  // namespace rvp

struct rvp_scorer {
  rvp_context *ctx = nullptr;
  size_t max_points = 0;
  int max_frames = 0;
  rvp::Grid grid;
  rvp::DevBuf frame_of, is_cand, pairs, counts, hard, qlevel, qtau, open;
  rvp::DevBuf w, wq, m, v, grad, norm, loss;
  rvp::DevBuf cand_xyz;  // candidates' own coordinates (neighbours among candidates)
  rvp::DevBuf gpart;     // per-block gradient shares of a training step
  int adam_step = 0;
  size_t fitted_points = 0;  // batch size and cell the bucket table was fitted to
  float fitted_cell = 0.0f;
  int knn_coop = 0;          // features among candidates: cooperative first pass
  float knn_rfac = 1.0f;     // its bound factor
};

namespace {
template <class F>
rvp_status sguard(rvp_context *ctx, F &&f) {
  try {
    f();
    return RVP_OK;
  } catch (const rvp::Error &e) {
    if (ctx) ctx->last_error = e.msg;
    return e.status;
  } catch (const std::bad_alloc &) {
    if (ctx) ctx->last_error = "host allocation failed";
    return RVP_ERR_OOM;
  } catch (...) {
    if (ctx) ctx->last_error = "unknown error";
    return RVP_ERR_CUDA;
  }
}
size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

double clamp_prob(float p) {
  double pc = (double)p;
  return pc < 0.5 ? 0.5 : (pc > 0.9999 ? 0.9999 : pc);
}
}  // namespace

extern "C" {

rvp_status rvp_scorer_create(rvp_context *ctx, size_t max_points, int max_frames,
                             rvp_scorer **out) {
  if (!ctx || !out || max_frames < 1) return RVP_ERR_INVALID_ARG;
  *out = nullptr;
  rvp_scorer *s = new (std::nothrow) rvp_scorer;
  if (!s) return RVP_ERR_OOM;
  s->ctx = ctx;
  s->max_points = max_points > 0 ? max_points : 1;
  s->max_frames = max_frames;
  rvp_status st = sguard(ctx, [&] {
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t N = s->max_points;
    s->grid.reserve(N, max_frames);
    s->frame_of.reserve(N * 4);
    s->is_cand.reserve(N);
    s->pairs.reserve(N * rvp::KF * 8);
    s->counts.reserve(N * 4);
    s->hard.reserve(N * 8 + 256);
    s->qlevel.reserve(N);
    s->qtau.reserve(N * 4);
    s->open.reserve(al256(N * 4) + al256(N * 8 + 8) + al256(N * 4) + 256 + rvp::scan_temp_bytes(N));
    s->w.reserve(rvp::NP * 4);
    s->wq.reserve(rvp::NP * 2);
    s->m.reserve(rvp::NP * 4);
    s->v.reserve(rvp::NP * 4);
    s->grad.reserve(rvp::NP * 4);
    s->norm.reserve(2 * rvp::MI * 4);
    s->loss.reserve(16);
    // He-style uniform initial weights from a fixed seed, zero biases;
    // identity normalisation until rvp_mlp_set_norm
    std::vector<float> w0(rvp::NP, 0.0f);
    unsigned long long st64 = 0x243F6A8885A308D3ull;
    auto uni = [&] {
      st64 = st64 * 6364136223846793005ull + 1442695040888963407ull;
      return ((st64 >> 11) * 0x1.0p-53) * 2.0 - 1.0;
    };
    for (int i = 0; i < rvp::MH * rvp::MI; ++i) w0[rvp::OW1 + i] = (float)(uni() * sqrt(6.0 / rvp::MI));
    for (int i = 0; i < rvp::MH * rvp::MH; ++i) w0[rvp::OW2 + i] = (float)(uni() * sqrt(6.0 / rvp::MH));
    for (int i = 0; i < rvp::MH; ++i) w0[rvp::OW3 + i] = (float)(uni() * sqrt(3.0 / rvp::MH));
    std::vector<float> nm(2 * rvp::MI);
    for (int k = 0; k < rvp::MI; ++k) { nm[k] = 0.0f; nm[rvp::MI + k] = 1.0f; }
    RVP_CUDA_TRY(cudaMemcpy(s->w.ptr, w0.data(), rvp::NP * 4, cudaMemcpyHostToDevice));
    RVP_CUDA_TRY(cudaMemcpy(s->norm.ptr, nm.data(), nm.size() * 4, cudaMemcpyHostToDevice));
    RVP_CUDA_TRY(cudaMemset(s->m.ptr, 0, rvp::NP * 4));
    RVP_CUDA_TRY(cudaMemset(s->v.ptr, 0, rvp::NP * 4));
    rvp::k_quantize<<<8, 256, 0, ctx->stream>>>(s->w.as<float>(), s->wq.as<__nv_bfloat16>(), rvp::NP);
    RVP_LAUNCH_CHECK(ctx);
    RVP_CUDA_TRY(cudaFuncSetAttribute(rvp::k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)rvp::TRAIN_SMEM));
    RVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  });
  if (st != RVP_OK) {
    rvp_scorer_destroy(s);
    return st;
  }
  *out = s;
  return RVP_OK;
}

rvp_status rvp_scorer_destroy(rvp_scorer *s) {
  if (!s) return RVP_ERR_INVALID_ARG;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  rvp::DevBuf *bufs[] = {&s->frame_of, &s->is_cand, &s->pairs, &s->counts, &s->hard, &s->qlevel,
                         &s->qtau, &s->open, &s->w, &s->wq, &s->m, &s->v, &s->grad, &s->norm,
                         &s->loss, &s->cand_xyz, &s->gpart};
  for (auto *b : bufs) b->release();
  s->grid.release();
  delete s;
  return RVP_OK;
}

namespace {
rvp_status features_impl(rvp_scorer *s, const float *x, const float *y, const float *z,
                         const int64_t *frame_offsets_dev, int n_frames, size_t n_points,
                         float cell_size, const uint32_t *cand, size_t n_cand, float *features,
                         int lane_levels = 0, float rfac = 1.0f, bool coop = false) {
  rvp_context *ctx = s->ctx;
  return sguard(ctx, [&] {
    RVP_REQUIRE(x && y && z && frame_offsets_dev && features, "null pointer");
    RVP_REQUIRE(n_frames >= 1 && n_frames <= s->max_frames, "n_frames out of range");
    RVP_REQUIRE(n_points >= 1 && n_points <= s->max_points, "n_points out of range");
    RVP_REQUIRE(cell_size > 0.0f, "cell_size must be > 0");
    if (!cand) n_cand = n_points;
    RVP_REQUIRE(n_cand <= n_points, "more candidates than points");
    if (n_cand == 0) return;
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t N = n_points;
    const int sms = ctx->num_sms;
    const unsigned gb = rvp::grid_for(N, 256, sms * 16);
    rvp::grid_build(ctx, s->grid, x, y, z, frame_offsets_dev, n_frames, N, cell_size,
                    rvp::KEY_DENSE, 0, 0, nullptr);
    if (s->fitted_points != N || s->fitted_cell != cell_size) {
      // size the bucket table to the cells this batch occupies (it stays in
      // L2 instead of spanning 2.5 slots per point), then build again
      u64 nb[rvp::kHeadLevels] = {};
      RVP_CUDA_TRY(cudaMemcpyAsync(nb, s->grid.d_nbuckets, 8 * rvp::kHeadLevels, cudaMemcpyDeviceToHost, st));
      RVP_CUDA_TRY(cudaStreamSynchronize(st));
      size_t tot = 0;
      for (int l = 0; l < rvp::kGridLevels; ++l) tot += (size_t)nb[l];
      s->grid.fit_table(tot + tot / 4);
      s->fitted_points = N;
      s->fitted_cell = cell_size;
      rvp::grid_build(ctx, s->grid, x, y, z, frame_offsets_dev, n_frames, N, cell_size,
                      rvp::KEY_DENSE, 0, 0, nullptr);
    }
    rvp::k_frame_of<<<gb, 256, 0, st>>>(frame_offsets_dev, n_frames, N, s->frame_of.as<int32_t>());
    RVP_LAUNCH_CHECK(ctx);
    const rvp::GridView gv = s->grid.view(rvp::KEY_DENSE, 0, 0);
    uint8_t *is_cand = nullptr;
    if (cand) {
      is_cand = s->is_cand.as<uint8_t>();
      RVP_CUDA_TRY(cudaMemsetAsync(is_cand, 0, N, st));
      rvp::k_mark_cand<<<rvp::grid_for(n_cand, 256, sms * 16), 256, 0, st>>>(cand, n_cand, N,
                                                                            is_cand);
      RVP_LAUNCH_CHECK(ctx);
    }
    // every grid point a query: the cooperative pass marks them itself
    const bool coop_pass = coop && !cand;
    if (!coop_pass) {
      rvp::k_open_cand<<<gb, 256, 0, st>>>(gv.pts, gv.n_points, is_cand,
                                           s->qlevel.as<uint8_t>());
      RVP_LAUNCH_CHECK(ctx);
    }
    u64 *hard_n64 = s->hard.as<u64>();
    u32 *hard_n = reinterpret_cast<u32 *>(hard_n64 + 1);
    u32 *hard = reinterpret_cast<u32 *>(hard_n64 + 2);
    float *hard_tau = reinterpret_cast<float *>(hard + N);
    RVP_CUDA_TRY(cudaMemsetAsync(hard_n64, 0, 16, st));
    RVP_CUDA_TRY(cudaMemsetAsync(s->counts.ptr, 0, N * 4, st));
    rvp::TileArgs ta{};
    ta.frame_of = s->frame_of.as<int32_t>();
    ta.pairs = s->pairs.as<u64>();
    ta.counts = s->counts.as<int32_t>();
    ta.hard = hard;
    ta.hard_count = hard_n;
    ta.hard_tau = hard_tau;
    ta.qlevel = s->qlevel.as<uint8_t>();
    ta.qtau = s->qtau.as<float>();
    ta.rfac = rfac;
    ta.level0_warp = true;
    ta.preset_open = !coop_pass;
    ta.coop = coop_pass ? 1 : 0;
    ta.lane_levels = lane_levels;
    char *op = s->open.as<char>();
    ta.open_flags = reinterpret_cast<u32 *>(op); op += al256(N * 4);
    ta.open_pos = reinterpret_cast<u64 *>(op); op += al256(N * 8 + 8);
    ta.open_list = reinterpret_cast<u32 *>(op); op += al256(N * 4);
    ta.open_n = reinterpret_cast<u64 *>(op); op += 256;
    ta.scan_tmp = op;
    ta.n_max = N;
    RVP_REQUIRE(rvp::grid_knn_tile(ctx, gv, rvp::KF, rvp::TILE_PAIRS_F, ta, 0, nullptr),
                "kNN tile path unavailable");
    rvp::k_widen32<<<1, 32, 0, st>>>(hard_n, hard_n64);
    RVP_LAUNCH_CHECK(ctx);
    rvp::grid_knn_tau(ctx, gv, rvp::KF, rvp::TILE_PAIRS_F, ta, hard_n64);
    rvp::QuerySet qh{x, y, z, N, hard_n64, s->frame_of.as<int32_t>(),
                     reinterpret_cast<int32_t *>(hard)};
    qh.bound = hard_tau;
    rvp::grid_knn(ctx, gv, qh, rvp::KF, 0.0f, s->pairs.as<u64>(), s->counts.as<int32_t>(), 1, 256,
                  nullptr, rvp::KNN_OUT_BY_QUERY, nullptr);
    rvp::k_features<<<rvp::grid_for(n_cand, 256, sms * 16), 256, 0, st>>>(
        x, y, z, s->pairs.as<u64>(), s->counts.as<int32_t>(), cand, n_cand, N, features);
    RVP_LAUNCH_CHECK(ctx);
  });
}
}  // namespace

rvp_status rvp_scorer_features(rvp_scorer *s, const float *x, const float *y, const float *z,
                               const int64_t *frame_offsets_dev, int n_frames, size_t n_points,
                               float cell_size, const uint32_t *cand,
                               const int64_t *cand_offsets_dev, size_t n_cand, int neighbours,
                               float *features) {
  if (!s) return RVP_ERR_INVALID_ARG;
  if (neighbours == 0)  // the batched grid kNN, in the mode rvp_scorer_set_knn chose
    return features_impl(s, x, y, z, frame_offsets_dev, n_frames, n_points, cell_size, cand,
                         n_cand, features, 0, s->knn_coop ? s->knn_rfac : 1.0f,
                         s->knn_coop != 0);
  if (neighbours != 1 || !cand || !cand_offsets_dev) return RVP_ERR_INVALID_ARG;
  // neighbourhoods among the candidates only: their coordinates, frame by
  // frame, become the cloud of the grid search
  rvp_context *ctx = s->ctx;
  const rvp_status st = sguard(ctx, [&] {
    RVP_REQUIRE(x && y && z, "null pointer");
    RVP_REQUIRE(n_cand >= 1 && n_cand <= s->max_points, "n_cand out of range");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    s->cand_xyz.reserve(n_cand * 12);
    float *gx = s->cand_xyz.as<float>();
    rvp::k_gather_xyz<<<rvp::grid_for(n_cand, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(
        x, y, z, cand, n_cand, n_points, gx, gx + n_cand, gx + 2 * n_cand);
    RVP_LAUNCH_CHECK(ctx);
  });
  if (st != RVP_OK) return st;
  // CK_SLICES blocks per scene, each with the scene's candidates in shared
  // memory (no global grid, sort or table)
  return sguard(ctx, [&] {
    RVP_REQUIRE(cell_size > 0.0f, "cell_size must be > 0");
    RVP_REQUIRE(n_frames >= 1 && n_frames <= s->max_frames, "n_frames out of range");
    const float *gx = s->cand_xyz.as<float>();
    static bool attr[64] = {false};
    if (ctx->device < 64 && !attr[ctx->device]) {
      RVP_CUDA_TRY(cudaFuncSetAttribute(rvp::k_cand_knn,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)rvp::CK_SMEM));
      attr[ctx->device] = true;
    }
    const unsigned blocks = (unsigned)std::min(n_frames * rvp::CK_SLICES, ctx->num_sms * 8);
    rvp::k_cand_knn<<<blocks, rvp::CK_TH, rvp::CK_SMEM, ctx->stream>>>(
        gx, gx + n_cand, gx + 2 * n_cand, cand_offsets_dev, n_frames, cell_size,
        s->pairs.as<u64>(), s->counts.as<int32_t>());
    RVP_LAUNCH_CHECK(ctx);
    rvp::k_features<<<rvp::grid_for(n_cand, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(
        gx, gx + n_cand, gx + 2 * n_cand, s->pairs.as<u64>(), s->counts.as<int32_t>(), nullptr,
        n_cand, n_cand, features);
    RVP_LAUNCH_CHECK(ctx);
  });
}

rvp_status rvp_scorer_set_knn(rvp_scorer *s, int queries_per_warp, float rfac) {
  if (!s || (queries_per_warp != 0 && queries_per_warp != 3)) return RVP_ERR_INVALID_ARG;
  if (queries_per_warp == 3 && !(rfac > 0.0f)) return RVP_ERR_INVALID_ARG;
  s->knn_coop = queries_per_warp == 3;
  s->knn_rfac = rfac;
  return RVP_OK;
}


rvp_status rvp_mlp_set_params(rvp_scorer *s, const float *params) {
  if (!s || !params) return RVP_ERR_INVALID_ARG;
  return sguard(s->ctx, [&] {
    RVP_CUDA_TRY(cudaSetDevice(s->ctx->device));
    RVP_CUDA_TRY(cudaMemcpyAsync(s->w.ptr, params, rvp::NP * 4, cudaMemcpyHostToDevice,
                                 s->ctx->stream));
    RVP_CUDA_TRY(cudaMemsetAsync(s->m.ptr, 0, rvp::NP * 4, s->ctx->stream));
    RVP_CUDA_TRY(cudaMemsetAsync(s->v.ptr, 0, rvp::NP * 4, s->ctx->stream));
    s->adam_step = 0;
    rvp::k_quantize<<<8, 256, 0, s->ctx->stream>>>(s->w.as<float>(), s->wq.as<__nv_bfloat16>(),
                                                   rvp::NP);
    RVP_LAUNCH_CHECK(s->ctx);
    RVP_CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  });
}

rvp_status rvp_mlp_get_params(rvp_scorer *s, float *params) {
  if (!s || !params) return RVP_ERR_INVALID_ARG;
  return sguard(s->ctx, [&] {
    RVP_CUDA_TRY(cudaSetDevice(s->ctx->device));
    RVP_CUDA_TRY(cudaMemcpyAsync(params, s->w.ptr, rvp::NP * 4, cudaMemcpyDeviceToHost,
                                 s->ctx->stream));
    RVP_CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  });
}

rvp_status rvp_mlp_set_norm(rvp_scorer *s, const float *mean, const float *stddev) {
  if (!s || !mean || !stddev) return RVP_ERR_INVALID_ARG;
  return sguard(s->ctx, [&] {
    float nm[2 * rvp::MI];
    for (int k = 0; k < rvp::MI; ++k) {
      RVP_REQUIRE(stddev[k] > 0.0f, "stddev must be > 0");
      nm[k] = mean[k];
      nm[rvp::MI + k] = 1.0f / stddev[k];
    }
    RVP_CUDA_TRY(cudaSetDevice(s->ctx->device));
    RVP_CUDA_TRY(cudaMemcpyAsync(s->norm.ptr, nm, sizeof(nm), cudaMemcpyHostToDevice,
                                 s->ctx->stream));
    RVP_CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
  });
}

rvp_status rvp_mlp_forward(rvp_scorer *s, const float *features, size_t n, float *logits) {
  if (!s) return RVP_ERR_INVALID_ARG;
  return sguard(s->ctx, [&] {
    if (n == 0) return;
    RVP_REQUIRE(features && logits, "null pointer");
    RVP_CUDA_TRY(cudaSetDevice(s->ctx->device));
    const unsigned blocks = rvp::grid_for((n + 15) / 16, rvp::FWD_THREADS / 32,
                                          s->ctx->num_sms * 8);
    rvp::k_mlp_forward<<<blocks, rvp::FWD_THREADS, 0, s->ctx->stream>>>(
        features, n, s->wq.as<__nv_bfloat16>(), s->norm.as<float>(), logits);
    RVP_LAUNCH_CHECK(s->ctx);
  });
}

namespace {
void mlp_grad(rvp_scorer *s, const float *features, const float *labels, size_t n,
              size_t n_src = 0, u64 sample_seed = 0) {
  rvp_context *ctx = s->ctx;
  const unsigned blocks =
      (unsigned)std::min<size_t>((n + rvp::TP - 1) / rvp::TP, (size_t)ctx->num_sms);
  s->gpart.reserve((size_t)blocks * rvp::NP * 4 + (size_t)blocks * 8 + 256);
  float *part = s->gpart.as<float>();
  double *part_loss = reinterpret_cast<double *>(
      s->gpart.as<char>() + (((size_t)blocks * rvp::NP * 4 + 255) & ~(size_t)255));
  rvp::k_mlp_train<<<blocks, rvp::TB, rvp::TRAIN_SMEM, ctx->stream>>>(
      features, labels, n, n_src ? n_src : n, sample_seed, s->wq.as<__nv_bfloat16>(),
      s->norm.as<float>(), part, part_loss);
  RVP_LAUNCH_CHECK(ctx);
  rvp::k_grad_reduce<<<(rvp::NP + 255) / 256, 256, 0, ctx->stream>>>(
      part, part_loss, (int)blocks, s->grad.as<float>(), s->loss.as<double>());
  RVP_LAUNCH_CHECK(ctx);
}
}  // namespace

rvp_status rvp_mlp_gradients(rvp_scorer *s, const float *features, const float *labels,
                             size_t n, float *grad, double *loss) {
  if (!s || !grad || !loss) return RVP_ERR_INVALID_ARG;
  return sguard(s->ctx, [&] {
    RVP_REQUIRE(n > 0 && features && labels, "empty batch");
    RVP_CUDA_TRY(cudaSetDevice(s->ctx->device));
    mlp_grad(s, features, labels, n);
    double l = 0.0;
    RVP_CUDA_TRY(cudaMemcpyAsync(grad, s->grad.ptr, rvp::NP * 4, cudaMemcpyDeviceToHost,
                                 s->ctx->stream));
    RVP_CUDA_TRY(cudaMemcpyAsync(&l, s->loss.ptr, 8, cudaMemcpyDeviceToHost, s->ctx->stream));
    RVP_CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
    *loss = l / (double)n;
  });
}

rvp_status rvp_mlp_train_step(rvp_scorer *s, const float *features, const float *labels,
                              size_t n, size_t batch, uint64_t seed, float lr, double *loss) {
  if (!s || !(lr > 0.0f)) return RVP_ERR_INVALID_ARG;
  return sguard(s->ctx, [&] {
    RVP_REQUIRE(n > 0 && features && labels, "empty batch");
    RVP_CUDA_TRY(cudaSetDevice(s->ctx->device));
    if (batch > 0)  // a fresh minibatch every step: the key mixes seed and step
      mlp_grad(s, features, labels, batch, n,
               (seed ^ (0x9E3779B97F4A7C15ull * (u64)(s->adam_step + 1))) | 1ull);
    else
      mlp_grad(s, features, labels, n);
    s->adam_step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f / (1.0f - powf(b1, (float)s->adam_step));
    const float c2 = 1.0f / (1.0f - powf(b2, (float)s->adam_step));
    rvp::k_adam<<<8, 256, 0, s->ctx->stream>>>(s->w.as<float>(), s->grad.as<float>(),
                                               s->m.as<float>(), s->v.as<float>(), rvp::NP, lr,
                                               b1, b2, 1e-8f, c1, c2);
    RVP_LAUNCH_CHECK(s->ctx);
    rvp::k_quantize<<<8, 256, 0, s->ctx->stream>>>(s->w.as<float>(), s->wq.as<__nv_bfloat16>(),
                                                   rvp::NP);
    RVP_LAUNCH_CHECK(s->ctx);
    if (loss) {
      double l = 0.0;
      RVP_CUDA_TRY(cudaMemcpyAsync(&l, s->loss.ptr, 8, cudaMemcpyDeviceToHost, s->ctx->stream));
      RVP_CUDA_TRY(cudaStreamSynchronize(s->ctx->stream));
      *loss = l / (double)n;
    }
  });
}

rvp_status rvp_ransac_frames(rvp_context *ctx, const float *x, const float *y, const float *z,
                             const int64_t *frame_offsets_dev, int n_frames, int max_iters,
                             float dist_thresh, float collinear_thresh, float probability,
                             const int32_t *targets, float *models, int32_t *best,
                             int32_t *iters_run) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return sguard(ctx, [&] {
    RVP_REQUIRE(x && y && z && frame_offsets_dev && models && best, "null pointer");
    RVP_REQUIRE(n_frames >= 1 && max_iters >= 1, "n_frames / max_iters must be >= 1");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    // the reference's srand(0) + rand() stream, drawn from libc, with the
    // generator left where the reference's last call leaves it
    const size_t R = 3 * (size_t)max_iters;
    std::vector<int32_t> rs(R);
    srand(0);
    for (size_t i = 0; i < R; ++i) rs[i] = rand();
    rvp::DevBuf &drand = ctx->scratch[24];
    drand.reserve(R * 4);
    RVP_CUDA_TRY(cudaMemcpyAsync(drand.ptr, rs.data(), R * 4, cudaMemcpyHostToDevice, ctx->stream));
    rvp::RansacParams prm{dist_thresh, max_iters, collinear_thresh,
                          log(1.0 - clamp_prob(probability))};
    rvp::RansacSampler smp;
    smp.targets = targets;
    std::vector<int32_t> it(n_frames, 0);
    int32_t *di = iters_run;
    if (!di) {
      ctx->scratch[25].reserve((size_t)n_frames * 4);
      di = ctx->scratch[25].as<int32_t>();
    }
    rvp::ransac_frames(ctx, x, y, z, frame_offsets_dev, n_frames, drand.as<int>(), prm, models,
                       best, di, nullptr, false, smp, 8);
    RVP_CUDA_TRY(cudaMemcpyAsync(it.data(), di, (size_t)n_frames * 4, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    RVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    srand(0);
    for (long i = 0; i < 3L * it[n_frames - 1]; ++i) (void)rand();
  });
}

rvp_status rvp_ransac_weighted(rvp_context *ctx, const float *x, const float *y, const float *z,
                               const int64_t *frame_offsets_dev, int n_frames,
                               const uint32_t *cand, const int64_t *cand_offsets_dev,
                               size_t n_cand, const float *weights, float logit_power,
                               uint64_t seed,
                               int max_iters, float dist_thresh, float collinear_thresh,
                               float probability, const int32_t *targets, float *models,
                               int32_t *best, int32_t *iters_run) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return sguard(ctx, [&] {
    RVP_REQUIRE(x && y && z && frame_offsets_dev && cand && cand_offsets_dev && weights &&
                    models && best,
                "null pointer");
    RVP_REQUIRE(n_frames >= 1 && max_iters >= 1, "n_frames / max_iters must be >= 1");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    rvp::DevBuf &cdf = ctx->scratch[26];
    cdf.reserve(std::max<size_t>(n_cand, 1) * 8);
    RVP_REQUIRE(logit_power >= 0.0f, "logit_power must be >= 0");
    rvp::k_cdf<<<n_frames, 256, 0, ctx->stream>>>(weights, logit_power, cand_offsets_dev,
                                                  cdf.as<double>());
    RVP_LAUNCH_CHECK(ctx);
    rvp::RansacParams prm{dist_thresh, max_iters, collinear_thresh,
                          log(1.0 - clamp_prob(probability))};
    rvp::RansacSampler smp;
    smp.cand = cand;
    smp.cand_offs = cand_offsets_dev;
    smp.cdf = cdf.as<double>();
    smp.seed = seed;
    smp.targets = targets;
    rvp::ransac_frames(ctx, x, y, z, frame_offsets_dev, n_frames, nullptr, prm, models, best,
                       iters_run, nullptr, false, smp, 8);
  });
}

rvp_status rvp_ransac_preemptive(rvp_context *ctx, const float *x, const float *y,
                                 const float *z, const int64_t *frame_offsets_dev, int n_frames,
                                 const uint32_t *cand, const int64_t *cand_offsets_dev,
                                 size_t n_cand, const float *weights, float logit_power,
                                 uint64_t seed, int draws, int max_rounds, float dist_thresh,
                                 float collinear_thresh, const int32_t *targets, float *models,
                                 int32_t *best, int32_t *draws_run) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return sguard(ctx, [&] {
    RVP_REQUIRE(x && y && z && frame_offsets_dev && cand && cand_offsets_dev && weights &&
                    models && best && draws_run,
                "null pointer");
    RVP_REQUIRE(n_frames >= 1 && max_rounds >= 1, "n_frames / max_rounds must be >= 1");
    RVP_REQUIRE(draws >= 1 && draws <= 512, "draws must be in [1, 512]");
    RVP_REQUIRE(logit_power >= 0.0f, "logit_power must be >= 0");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    rvp::DevBuf &cdf = ctx->scratch[26];
    cdf.reserve(std::max<size_t>(n_cand, 1) * 8);
    rvp::k_cdf<<<n_frames, 256, 0, ctx->stream>>>(weights, logit_power, cand_offsets_dev,
                                                  cdf.as<double>());
    RVP_LAUNCH_CHECK(ctx);
    rvp::DevBuf &tmp = ctx->scratch[28];
    tmp.reserve(rvp::preemptive_temp_bytes(n_frames));
    rvp::RansacParams prm{dist_thresh, 32, collinear_thresh, log(1.0 - 0.9999)};
    rvp::RansacSampler smp;
    smp.cand = cand;
    smp.cand_offs = cand_offsets_dev;
    smp.cdf = cdf.as<double>();
    smp.seed = seed;
    smp.targets = targets;
    rvp::ransac_preemptive(ctx, x, y, z, frame_offsets_dev, n_frames, smp, draws, max_rounds,
                           prm, models, best, draws_run, tmp.ptr);
  });
}

rvp_status rvp_plane_labels(rvp_context *ctx, const float *x, const float *y, const float *z,
                            const int64_t *frame_offsets_dev, int n_frames, size_t n_points,
                            const float *models, float dist_thresh, float *labels) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return sguard(ctx, [&] {
    RVP_REQUIRE(x && y && z && frame_offsets_dev && models && labels, "null pointer");
    RVP_REQUIRE(n_frames >= 1, "n_frames must be >= 1");
    if (n_points == 0) return;
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    rvp::DevBuf &fr = ctx->scratch[27];
    fr.reserve(n_points * 4);
    const unsigned gb = rvp::grid_for(n_points, 256, ctx->num_sms * 16);
    rvp::k_frame_of<<<gb, 256, 0, ctx->stream>>>(frame_offsets_dev, n_frames, n_points,
                                                 fr.as<int32_t>());
    RVP_LAUNCH_CHECK(ctx);
    rvp::k_plane_labels<<<gb, 256, 0, ctx->stream>>>(x, y, z, fr.as<int32_t>(), n_points, models,
                                                     dist_thresh, labels);
    RVP_LAUNCH_CHECK(ctx);
  });
}

}  // extern "C"
