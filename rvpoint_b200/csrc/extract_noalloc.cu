// Plane inlier / outlier extraction that allocates nothing.
//
// Some callers cannot allocate device memory when they call into this
// library: a control loop that forbids allocation once it has started (an
// allocation can block for milliseconds or fail under memory pressure), or a
// host framework that owns every device allocation and hands plug-ins only
// the buffers it made. rvp_extract_plane allocates its scratch on first use;
// this variant keeps its only scratch -- one inlier count per 2048-point
// tile -- in a fixed array compiled into the library, so the caller provides
// just the inputs and outputs.
//
// The array is 8192 counts (32 KB). Every GPU that loads the library holds it
// until the process exits, and every call on a device uses the same array:
// calls whose kernels overlap on the GPU (different streams, no ordering)
// race on it. Each call writes every count it reads before reading it, so
// nothing has to be cleared between calls.
#include <atomic>
#include <mutex>

#include "internal.cuh"

namespace rvp {
namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_ITEMS = 8;
constexpr int NA_TILE = NA_THREADS * NA_ITEMS;  // 2048 points per tile
constexpr int NA_MAX_TILES = 8192;
static_assert((size_t)NA_MAX_TILES * NA_TILE == RVP_NOALLOC_MAX_POINTS,
              "header limit and scratch size disagree");

// the scratch: inliers per tile of the last call on this device
static __device__ __align__(256) u32 g_noalloc_tile_inliers[NA_MAX_TILES];

constexpr int kMaxDevices = 64;
std::atomic<u32 *> g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mutex;

// Device address of the scratch on `device` (which must be current): looked
// up once per device, with cudaGetSymbolAddress, and cached.
cudaError_t scratch_address(int device, u32 **out) {
  u32 *p = g_scratch_addr[device].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    p = g_scratch_addr[device].load(std::memory_order_relaxed);
    if (!p) {
      void *addr = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_tile_inliers);
      if (e != cudaSuccess) return e;
      p = static_cast<u32 *>(addr);
      g_scratch_addr[device].store(p, std::memory_order_release);
    }
  }
  *out = p;
  return cudaSuccess;
}

// -t <= a*x + b*y + c*z + d <= t, the scalar branch of
// extract_plane_inliers_outliers_rvv (ransac_plane.cpp:373-381)
__device__ __forceinline__ bool plane_inlier(const float4 &m, float x, float y, float z,
                                             float t) {
  const float d = fadd(fadd(fadd(fmul(m.x, x), fmul(m.y, y)), fmul(m.z, z)), m.w);
  return d >= -t && d <= t;
}

__device__ __forceinline__ u32 block_sum(u32 v, u32 *red) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  u32 s = 0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < NA_THREADS / 32 ? red[threadIdx.x] : 0;
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  __syncthreads();
  return s;  // valid in thread 0
}

// pass 1: inliers of each tile into the scratch
__global__ __launch_bounds__(NA_THREADS) void k_na_count(const float *__restrict__ x,
                                                         const float *__restrict__ y,
                                                         const float *__restrict__ z, size_t n,
                                                         const float *__restrict__ model,
                                                         float t, u32 *tile_inliers) {
  __shared__ u32 red[NA_THREADS / 32];
  const float4 m = make_float4(model[0], model[1], model[2], model[3]);
  const size_t base = (size_t)blockIdx.x * NA_TILE;
  u32 c = 0;
#pragma unroll
  for (int j = 0; j < NA_ITEMS; ++j) {
    const size_t i = base + (size_t)j * NA_THREADS + threadIdx.x;
    if (i < n && plane_inlier(m, x[i], y[i], z[i], t)) ++c;
  }
  const u32 s = block_sum(c, red);
  if (threadIdx.x == 0) tile_inliers[blockIdx.x] = s;
}

// pass 2: each tile adds up the tiles before it, ranks its points in input
// order and writes inliers and outliers (AoS) to their final positions
__global__ __launch_bounds__(NA_THREADS) void k_na_scatter(
    const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
    size_t n, const float *__restrict__ model, float t, const u32 *tile_inliers,
    float *in_aos, float *out_aos, unsigned long long *counts) {
  __shared__ u32 red[NA_THREADS / 32];
  __shared__ u32 scan[NA_THREADS];
  __shared__ u32 s_before;
  const float4 m = make_float4(model[0], model[1], model[2], model[3]);
  const u32 tile = blockIdx.x;
  u32 part = 0;
  for (u32 k = threadIdx.x; k < tile; k += NA_THREADS) part += tile_inliers[k];
  const u32 before = block_sum(part, red);
  if (threadIdx.x == 0) s_before = before;
  // thread t owns NA_ITEMS consecutive points, so a scan over threads keeps
  // input order
  const size_t base = (size_t)tile * NA_TILE;
  const size_t first = base + (size_t)threadIdx.x * NA_ITEMS;
  bool f[NA_ITEMS];
  u32 c = 0;
#pragma unroll
  for (int j = 0; j < NA_ITEMS; ++j) {
    const size_t i = first + j;
    f[j] = i < n && plane_inlier(m, x[i], y[i], z[i], t);
    c += f[j] ? 1u : 0u;
  }
  scan[threadIdx.x] = c;
  __syncthreads();
  for (int o = 1; o < NA_THREADS; o <<= 1) {
    const u32 v = threadIdx.x >= (u32)o ? scan[threadIdx.x - o] : 0;
    __syncthreads();
    scan[threadIdx.x] += v;
    __syncthreads();
  }
  const u32 in_before_tile = s_before;
  u32 rin = in_before_tile + scan[threadIdx.x] - c;           // inliers before my first point
  u64 rout = (first - rin);                                   // outliers before my first point
#pragma unroll
  for (int j = 0; j < NA_ITEMS; ++j) {
    const size_t i = first + j;
    if (i >= n) break;
    if (f[j]) {
      if (in_aos) {
        in_aos[3 * (size_t)rin + 0] = x[i];
        in_aos[3 * (size_t)rin + 1] = y[i];
        in_aos[3 * (size_t)rin + 2] = z[i];
      }
      ++rin;
    } else {
      if (out_aos) {
        out_aos[3 * rout + 0] = x[i];
        out_aos[3 * rout + 1] = y[i];
        out_aos[3 * rout + 2] = z[i];
      }
      ++rout;
    }
  }
  if (tile == gridDim.x - 1 && threadIdx.x == NA_THREADS - 1) {
    const u64 total_in = (u64)in_before_tile + scan[NA_THREADS - 1];
    counts[0] = total_in;
    counts[1] = (u64)n - total_in;
  }
}

}  // namespace
}  // namespace rvp

extern "C" rvp_status rvp_extract_plane_noalloc(rvp_context *ctx, const float *x, const float *y,
                                                const float *z, size_t n, const float *model,
                                                float dist_thresh, float *inliers_aos,
                                                float *outliers_aos, uint64_t *counts) {
  using namespace rvp;
  if (!ctx || !model || !counts) return RVP_ERR_INVALID_ARG;
  if (n > (size_t)RVP_NOALLOC_MAX_POINTS) return RVP_ERR_INVALID_ARG;
  if (n > 0 && (!x || !y || !z)) return RVP_ERR_INVALID_ARG;
  if (ctx->device < 0 || ctx->device >= kMaxDevices) return RVP_ERR_INVALID_ARG;
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    cudaGetLastError();
    return RVP_ERR_CUDA;
  }
  u32 *scratch = nullptr;
  if (scratch_address(ctx->device, &scratch) != cudaSuccess) {
    cudaGetLastError();
    return RVP_ERR_CUDA;
  }
  cudaStream_t st = ctx->stream;
  if (n == 0) {
    if (cudaMemsetAsync(counts, 0, 2 * sizeof(uint64_t), st) != cudaSuccess) {
      cudaGetLastError();
      return RVP_ERR_CUDA;
    }
    return RVP_OK;
  }
  const unsigned tiles = (unsigned)((n + NA_TILE - 1) / NA_TILE);
  k_na_count<<<tiles, NA_THREADS, 0, st>>>(x, y, z, n, model, dist_thresh, scratch);
  ctx->launches++;
  k_na_scatter<<<tiles, NA_THREADS, 0, st>>>(x, y, z, n, model, dist_thresh, scratch,
                                             inliers_aos, outliers_aos,
                                             reinterpret_cast<unsigned long long *>(counts));
  ctx->launches++;
  if (cudaGetLastError() != cudaSuccess) return RVP_ERR_CUDA;
  return RVP_OK;
}
