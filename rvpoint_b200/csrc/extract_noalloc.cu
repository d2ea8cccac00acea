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
// nothing has to be cleared between calls. The array's device address is
// looked up on the first call on each device (cudaGetSymbolAddress, which
// allocates nothing) and kept: make that first call before any stream
// capture, and do not reset the device (cudaDeviceReset) while the library is
// loaded, since the kept address would then be stale.
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

// Points of a tile are read strided (item j of thread t is point
// base + j * NA_THREADS + t), so every load is coalesced; input order inside
// the tile is then (j, warp, lane).

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

// pass 2: exclusive scan of the tile counts, in place (one block of 1024
// threads, 8 consecutive counts each)
constexpr int NA_SCAN_THREADS = 1024;
static_assert(NA_MAX_TILES == NA_SCAN_THREADS * 8, "scan covers the scratch");
__global__ __launch_bounds__(NA_SCAN_THREADS) void k_na_scan(u32 *tile_inliers, u32 tiles) {
  __shared__ u32 warp_sums[NA_SCAN_THREADS / 32];
  const u32 tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  u32 v[8];
  u32 s = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const u32 k = tid * 8 + j;
    v[j] = k < tiles ? tile_inliers[k] : 0;
    s += v[j];
  }
  u32 incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u32 u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (u32)o) incl += u;
  }
  if (lane == 31) warp_sums[w] = incl;
  __syncthreads();
  if (w == 0) {
    u32 ws = warp_sums[lane];
    u32 wi = ws;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 u = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= (u32)o) wi += u;
    }
    warp_sums[lane] = wi - ws;  // exclusive prefix of the warps
  }
  __syncthreads();
  u32 run = warp_sums[w] + incl - s;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const u32 k = tid * 8 + j;
    if (k < tiles) tile_inliers[k] = run;
    run += v[j];
  }
}

// pass 3: every point's rank among the inliers (or outliers) of the cloud,
// in input order, and its AoS copy at that position
__global__ __launch_bounds__(NA_THREADS) void k_na_scatter(
    const float *__restrict__ x, const float *__restrict__ y, const float *__restrict__ z,
    size_t n, const float *__restrict__ model, float t, const u32 *tile_before,
    float *in_aos, float *out_aos, unsigned long long *counts) {
  constexpr int W = NA_THREADS / 32;
  __shared__ u32 pre[NA_ITEMS * W + 1];  // inliers before (item j, warp w), j-major
  const float4 m = make_float4(model[0], model[1], model[2], model[3]);
  const u32 tile = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const size_t base = (size_t)tile * NA_TILE;
  const unsigned lt = (1u << lane) - 1u;
  unsigned bal[NA_ITEMS];
#pragma unroll
  for (int j = 0; j < NA_ITEMS; ++j) {
    const size_t i = base + (size_t)j * NA_THREADS + threadIdx.x;
    const bool f = i < n && plane_inlier(m, x[i], y[i], z[i], t);
    bal[j] = __ballot_sync(0xffffffffu, f);
    if (lane == 0) pre[j * W + w] = __popc(bal[j]);
  }
  __syncthreads();
  if (w == 0) {  // exclusive scan of the NA_ITEMS * W warp counts (2 per lane)
    const u32 a0 = pre[2 * lane], a1 = pre[2 * lane + 1];
    u32 incl = a0 + a1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u32 u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (u32)o) incl += u;
    }
    const u32 ex = incl - a0 - a1;
    __syncwarp();
    pre[2 * lane] = ex;
    pre[2 * lane + 1] = ex + a0;
    if (lane == 31) pre[NA_ITEMS * W] = incl;
  }
  __syncthreads();
  const u32 before = tile_before[tile];
#pragma unroll
  for (int j = 0; j < NA_ITEMS; ++j) {
    const size_t i = base + (size_t)j * NA_THREADS + threadIdx.x;
    if (i >= n) break;
    const u64 rin = (u64)before + pre[j * W + w] + __popc(bal[j] & lt);  // inliers before i
    if ((bal[j] >> lane) & 1u) {
      if (in_aos) {
        in_aos[3 * rin + 0] = x[i];
        in_aos[3 * rin + 1] = y[i];
        in_aos[3 * rin + 2] = z[i];
      }
    } else if (out_aos) {
      const u64 rout = (u64)i - rin;  // outliers before i
      out_aos[3 * rout + 0] = x[i];
      out_aos[3 * rout + 1] = y[i];
      out_aos[3 * rout + 2] = z[i];
    }
  }
  if (tile == gridDim.x - 1 && threadIdx.x == 0) {
    const u64 total_in = (u64)before + pre[NA_ITEMS * W];
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
  // the caller's current device is put back before returning
  int caller_device = -1;
  if (cudaGetDevice(&caller_device) != cudaSuccess) {
    cudaGetLastError();
    return RVP_ERR_CUDA;
  }
  const bool switch_device = caller_device != ctx->device;
  if (switch_device && cudaSetDevice(ctx->device) != cudaSuccess) {
    cudaGetLastError();
    return RVP_ERR_CUDA;
  }
  rvp_status status = RVP_OK;
  u32 *scratch = nullptr;
  cudaStream_t st = ctx->stream;
  if (scratch_address(ctx->device, &scratch) != cudaSuccess) {
    cudaGetLastError();
    status = RVP_ERR_CUDA;
  } else if (n == 0) {
    if (cudaMemsetAsync(counts, 0, 2 * sizeof(uint64_t), st) != cudaSuccess) {
      cudaGetLastError();
      status = RVP_ERR_CUDA;
    }
  } else {
    const unsigned tiles = (unsigned)((n + NA_TILE - 1) / NA_TILE);
    k_na_count<<<tiles, NA_THREADS, 0, st>>>(x, y, z, n, model, dist_thresh, scratch);
    k_na_scan<<<1, NA_SCAN_THREADS, 0, st>>>(scratch, tiles);
    k_na_scatter<<<tiles, NA_THREADS, 0, st>>>(x, y, z, n, model, dist_thresh, scratch,
                                               inliers_aos, outliers_aos,
                                               reinterpret_cast<unsigned long long *>(counts));
    ctx->launches += 3;
    if (cudaGetLastError() != cudaSuccess) status = RVP_ERR_CUDA;
  }
  if (switch_device) cudaSetDevice(caller_device);
  return status;
}
