// C ABI of rvpoint_b200 (include/rvpoint_b200.h): host/device staging,
// status codes and the orchestration of the kernels for each reference
// entry point.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <new>

#include "internal.cuh"

using rvp::u32;
using rvp::u64;

// ---------------------------------------------------------------------------
// buffers
// ---------------------------------------------------------------------------
namespace rvp {
// Every device and pinned allocation of the library goes through DevBuf /
// HostBuf: the live byte counts are kept here, and a test hook
// (rvp_debug_fail_allocation) can make the allocations after the next n
// fail as an out-of-memory would.
namespace {
std::atomic<long long> g_live_device{0}, g_live_pinned{0};
std::atomic<long long> g_fail_after{-1};  // < 0: off

void check_injected_failure() {
  long long left = g_fail_after.load();
  while (left >= 0) {
    if (left == 0) throw Error{RVP_ERR_OOM, "allocation failed (injected by rvp_debug_fail_allocation)"};
    if (g_fail_after.compare_exchange_weak(left, left - 1)) return;
  }
}
}  // namespace

void DevBuf::reserve(size_t b) {
  if (b <= bytes && ptr) return;
  release();
  if (b == 0) b = 256;
  check_injected_failure();
  RVP_CUDA_TRY(cudaMalloc(&ptr, b));
  bytes = b;
  g_live_device += (long long)b;
}
void DevBuf::release() {
  if (ptr) {
    cudaFree(ptr);
    g_live_device -= (long long)bytes;
  }
  ptr = nullptr;
  bytes = 0;
}
void HostBuf::reserve(size_t b) {
  if (b <= bytes && ptr) return;
  release();
  if (b == 0) b = 256;
  check_injected_failure();
  RVP_CUDA_TRY(cudaMallocHost(&ptr, b));
  bytes = b;
  g_live_pinned += (long long)b;
}
void HostBuf::release() {
  if (ptr) {
    cudaFreeHost(ptr);
    g_live_pinned -= (long long)bytes;
  }
  ptr = nullptr;
  bytes = 0;
}
}  // namespace rvp

extern "C" {
rvp_status rvp_debug_fail_allocation(long long after) {
  rvp::g_fail_after = after < 0 ? -1 : after;
  return RVP_OK;
}

rvp_status rvp_debug_live_bytes(long long *device_bytes, long long *pinned_bytes) {
  if (device_bytes) *device_bytes = rvp::g_live_device.load();
  if (pinned_bytes) *pinned_bytes = rvp::g_live_pinned.load();
  return RVP_OK;
}
}

struct rvp_hash {
  rvp_context *ctx = nullptr;
  rvp::DevBuf x, y, z, offs;
  size_t n = 0;
  float cell = 0.0f;
  long long p1 = 73856093LL, p2 = 19349663LL;
  rvp::Grid grid;
  bool has_cloud = false, built = false;
  int collision = 0;
};

namespace {

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

template <class F>
rvp_status guard(rvp_context *ctx, F &&f) {
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

void set_device(rvp_context *ctx) { RVP_CUDA_TRY(cudaSetDevice(ctx->device)); }

void *scratch(rvp_context *ctx, int slot, size_t bytes) {
  ctx->scratch[slot].reserve(bytes);
  return ctx->scratch[slot].ptr;
}

// input: device pointer as is, or a staged copy of the host array
template <class T>
const T *in_dev(rvp_context *ctx, int slot, const T *p, size_t n, int mem) {
  if (mem == RVP_MEM_DEVICE || n == 0) return p;
  T *d = static_cast<T *>(scratch(ctx, slot, n * sizeof(T)));
  RVP_CUDA_TRY(cudaMemcpyAsync(d, p, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  return d;
}

template <class T>
T *out_dev(rvp_context *ctx, int slot, T *p, size_t n, int mem) {
  if (p == nullptr) return nullptr;
  if (mem == RVP_MEM_DEVICE) return p;
  return static_cast<T *>(scratch(ctx, slot, (n ? n : 1) * sizeof(T)));
}

template <class T>
void out_copy(rvp_context *ctx, T *user, const T *dev, size_t n, int mem) {
  if (user == nullptr || mem == RVP_MEM_DEVICE || n == 0) return;
  RVP_CUDA_TRY(cudaMemcpyAsync(user, dev, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
}

void sync(rvp_context *ctx) { RVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream)); }

template <class T>
T read_back(rvp_context *ctx, const T *dev) {
  T v;
  RVP_CUDA_TRY(cudaMemcpyAsync(&v, dev, sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  sync(ctx);
  return v;
}

// [0, n] on the device: a single frame
int64_t *single_frame_offsets(rvp_context *ctx, int slot, size_t n) {
  int64_t h[2] = {0, (int64_t)n};
  int64_t *d = static_cast<int64_t *>(scratch(ctx, slot, 16));
  RVP_CUDA_TRY(cudaMemcpyAsync(d, h, 16, cudaMemcpyHostToDevice, ctx->stream));
  sync(ctx);  // h lives on this stack frame
  return d;
}

__global__ void k_unpack(const u64 *pairs, size_t total, int32_t *idx, float *d2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const u64 k = pairs[i];
    if (idx) idx[i] = (int32_t)(u32)(k & 0x7FFFFFFFull);
    if (d2) d2[i] = __uint_as_float((u32)(k >> 32));
  }
}

// fixed-stride rows (nq x K, counts[q] valid) -> CSR rows
__global__ void k_rows_to_csr(const u64 *pairs, int K, const int32_t *counts, const u64 *offs,
                              size_t nq, int cut, int32_t *idx, float *d2) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nq * (size_t)K;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t q = t / K;
    const int j = (int)(t % K);
    const int c = min(counts[q], cut);
    if (j >= c) continue;
    const u64 k = pairs[t];
    const u64 o = offs[q] + j;
    idx[o] = (int32_t)(u32)(k & 0x7FFFFFFFull);
    d2[o] = __uint_as_float((u32)(k >> 32));
  }
}

// CSR rows cut to at most `cut` entries
__global__ void k_csr_cut(const u64 *pairs, const u64 *offs_in, const u64 *offs_out, size_t nq,
                          int32_t *idx, float *d2) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nq;
       q += (size_t)gridDim.x * blockDim.x) {
    const u64 a = offs_in[q], o = offs_out[q], c = offs_out[q + 1] - o;
    for (u64 j = 0; j < c; ++j) {
      const u64 k = pairs[a + j];
      idx[o + j] = (int32_t)(u32)(k & 0x7FFFFFFFull);
      d2[o + j] = __uint_as_float((u32)(k >> 32));
    }
  }
}

__global__ void k_min_counts(const u32 *in, size_t n, u32 cut, u32 *out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = in[i] < cut ? in[i] : cut;
}

__global__ void k_i32_to_u32(const int32_t *in, size_t n, u32 *out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = (u32)max(in[i], 0);
}

__global__ void k_fill_rows(const u64 *pairs, int K, const int32_t *counts, size_t nq,
                            int32_t *idx, float *d2) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nq * (size_t)K;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t q = t / K;
    const int j = (int)(t % K);
    if (j < counts[q]) {
      const u64 k = pairs[t];
      if (idx) idx[t] = (int32_t)(u32)(k & 0x7FFFFFFFull);
      if (d2) d2[t] = __uint_as_float((u32)(k >> 32));
    } else {
      if (idx) idx[t] = -1;
      if (d2) d2[t] = INFINITY;
    }
  }
}

__global__ void k_bbox_simple(const float *x, const float *y, const float *z, size_t n,
                              float *bb) {
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float v[3] = {x[i], y[i], z[i]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = fminf(mn[a], v[a]);
      mx[a] = fmaxf(mx[a], v[a]);
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o; o >>= 1) {
      mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
      mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
    }
    if ((threadIdx.x & 31) == 0) {
      rvp::atomic_min_f(&bb[a], mn[a]);
      rvp::atomic_max_f(&bb[3 + a], mx[a]);
    }
  }
}

// ---------------------------------------------------------------------------
// kNN over a device cloud with an automatically chosen cell: build on a
// volume-based guess, measure the k-th neighbour distance of a sample of
// queries, rebuild with cell = median k-th distance (the 27-cell ring then
// usually certifies the answer).
// ---------------------------------------------------------------------------
float auto_cell(rvp_context *ctx, rvp::Grid &g, const float *x, const float *y, const float *z,
                size_t n, const int64_t *offs_dev, int K) {
  float *bb = static_cast<float *>(scratch(ctx, 20, 64));
  float init[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  RVP_CUDA_TRY(cudaMemcpyAsync(bb, init, 24, cudaMemcpyHostToDevice, ctx->stream));
  k_bbox_simple<<<rvp::grid_for(n, 256, ctx->num_sms * 4), 256, 0, ctx->stream>>>(x, y, z, n, bb);
  RVP_LAUNCH_CHECK(ctx);
  float h[6];
  RVP_CUDA_TRY(cudaMemcpyAsync(h, bb, 24, cudaMemcpyDeviceToHost, ctx->stream));
  sync(ctx);
  double ext[3];
  for (int a = 0; a < 3; ++a) ext[a] = std::max(1e-6, (double)h[3 + a] - (double)h[a]);
  const double V = ext[0] * ext[1] * ext[2];
  double c0 = cbrt(V * (double)K / (double)std::max<size_t>(n, 1));
  const double emax = std::max(ext[0], std::max(ext[1], ext[2]));
  c0 = std::min(c0, emax);
  if (!(c0 > 0)) c0 = 1.0;
  const size_t S = std::min<size_t>(n, 1024);
  if (S < 8) return (float)c0;
  rvp::grid_build(ctx, g, x, y, z, offs_dev, 1, n, (float)c0, rvp::KEY_DENSE, 0, 0, nullptr);
  // sample queries: every (n/S)-th point
  float *sq = static_cast<float *>(scratch(ctx, 21, 3 * S * 4));
  {  // every (n/S)-th point as a query, by strided device copies
    const size_t stride = n / S;
    RVP_CUDA_TRY(cudaMemcpy2DAsync(sq, 4, x, stride * 4, 4, S, cudaMemcpyDeviceToDevice, ctx->stream));
    RVP_CUDA_TRY(cudaMemcpy2DAsync(sq + S, 4, y, stride * 4, 4, S, cudaMemcpyDeviceToDevice, ctx->stream));
    RVP_CUDA_TRY(cudaMemcpy2DAsync(sq + 2 * S, 4, z, stride * 4, 4, S, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  u64 *pairs = static_cast<u64 *>(scratch(ctx, 22, S * K * 8));
  int32_t *cnt = static_cast<int32_t *>(scratch(ctx, 23, S * 4));
  rvp::QuerySet qs{sq, sq + S, sq + 2 * S, S, nullptr, nullptr, nullptr};
  rvp::grid_knn(ctx, g.view(rvp::KEY_DENSE, 0, 0), qs, K, 0.0f, pairs, cnt, 1, 256);
  std::vector<u64> hp(S * K);
  std::vector<int32_t> hc(S);
  RVP_CUDA_TRY(cudaMemcpyAsync(hp.data(), pairs, S * K * 8, cudaMemcpyDeviceToHost, ctx->stream));
  RVP_CUDA_TRY(cudaMemcpyAsync(hc.data(), cnt, S * 4, cudaMemcpyDeviceToHost, ctx->stream));
  sync(ctx);
  std::vector<float> kd;
  for (size_t s = 0; s < S; ++s)
    if (hc[s] == K) {
      u32 b = (u32)(hp[s * K + K - 1] >> 32);
      float d2;
      memcpy(&d2, &b, 4);
      kd.push_back(sqrtf(d2));
    }
  if (kd.empty()) return (float)c0;
  std::nth_element(kd.begin(), kd.begin() + kd.size() / 2, kd.end());
  double c = kd[kd.size() / 2];
  c = std::max(c, c0 / 64.0);
  c = std::min(c, c0);
  if (!(c > 0)) c = c0;
  return (float)c;
}

void knn_cloud(rvp_context *ctx, rvp::Grid &g, const float *x, const float *y, const float *z,
               size_t n, int K, u64 *pairs, int32_t *counts) {
  int64_t *offs = single_frame_offsets(ctx, 19, n);
  const float cell = auto_cell(ctx, g, x, y, z, n, offs, K);
  rvp::grid_build(ctx, g, x, y, z, offs, 1, n, cell, rvp::KEY_DENSE, 0, 0, nullptr);
  rvp::QuerySet qs{x, y, z, n, nullptr, nullptr, nullptr};
  rvp::grid_knn(ctx, g.view(rvp::KEY_DENSE, 0, 0), qs, K, 0.0f, pairs, counts, 1, 256);
}

// one scratch grid per context, kept across calls so its buffers are reused
rvp::Grid &ctx_grid(rvp_context *ctx) {
  if (!ctx->grid) ctx->grid = new rvp::Grid();
  return *ctx->grid;
}

}  // namespace

// ===========================================================================
// context
// ===========================================================================
extern "C" {

const char *rvp_version(void) { return "rvpoint_b200 0.1 (sm_100a)"; }

const char *rvp_status_string(rvp_status s) {
  switch (s) {
    case RVP_OK: return "ok";
    case RVP_ERR_INVALID_ARG: return "invalid argument";
    case RVP_ERR_OOM: return "out of memory";
    case RVP_ERR_CAPACITY: return "output capacity too small";
    case RVP_ERR_TIMEOUT: return "device wait timed out";
    case RVP_ERR_CUDA: return "CUDA error";
    case RVP_ERR_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

rvp_status rvp_context_create(int device, rvp_context **out) {
  if (!out) return RVP_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return RVP_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = new (std::nothrow) rvp_context();
  if (!ctx) return RVP_ERR_OOM;
  ctx->device = device;
  rvp_status s = guard(ctx, [&] {
    set_device(ctx);
    RVP_CUDA_TRY(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
  });
  if (s != RVP_OK) {
    delete ctx;
    return s;
  }
  *out = ctx;
  return RVP_OK;
}

rvp_status rvp_context_destroy(rvp_context *ctx) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto &b : ctx->scratch) b.release();
  for (auto &b : ctx->pinned) b.release();
  if (ctx->grid) {
    ctx->grid->release();
    delete ctx->grid;
  }
  if (ctx->vwork) {
    ctx->vwork->release();
    delete ctx->vwork;
  }
  delete ctx;
  return RVP_OK;
}

rvp_status rvp_context_set_stream(rvp_context *ctx, void *stream) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  ctx->stream = static_cast<cudaStream_t>(stream);
  return RVP_OK;
}

rvp_status rvp_context_synchronize(rvp_context *ctx) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return guard(ctx, [&] { set_device(ctx); sync(ctx); });
}

const char *rvp_last_error(const rvp_context *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

uint64_t rvp_context_launch_count(const rvp_context *ctx) { return ctx ? ctx->launches : 0; }

// ===========================================================================
// SpatialHash
// ===========================================================================
rvp_status rvp_hash_create(rvp_context *ctx, rvp_hash **out) {
  if (!ctx || !out) return RVP_ERR_INVALID_ARG;
  rvp_hash *h = new (std::nothrow) rvp_hash();
  if (!h) return RVP_ERR_OOM;
  h->ctx = ctx;
  *out = h;
  return RVP_OK;
}

rvp_status rvp_hash_destroy(rvp_hash *h) {
  if (!h) return RVP_ERR_INVALID_ARG;
  cudaSetDevice(h->ctx->device);
  cudaStreamSynchronize(h->ctx->stream);
  h->x.release(); h->y.release(); h->z.release(); h->offs.release();
  h->grid.release();
  delete h;
  return RVP_OK;
}

rvp_status rvp_hash_set_primes(rvp_hash *h, int64_t p1, int64_t p2) {
  if (!h) return RVP_ERR_INVALID_ARG;
  h->p1 = p1;
  h->p2 = p2;
  h->built = false;
  return RVP_OK;
}

rvp_status rvp_hash_set_input_cloud(rvp_hash *h, const float *x, const float *y, const float *z,
                                    size_t n, float cell_size, int mem) {
  if (!h) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = h->ctx;
  return guard(ctx, [&] {
    RVP_REQUIRE(n == 0 || (x && y && z), "null cloud pointer");
    RVP_REQUIRE(n < 0x7FFFFFFFull, "clouds are limited to 2^31 - 1 points");
    RVP_REQUIRE(cell_size > 0.0f && isfinite(cell_size), "cell_size must be > 0");
    set_device(ctx);
    // no cloud until this call has completed (a failed allocation below
    // leaves the hash without one, not with the previous cloud's size)
    h->has_cloud = false;
    h->built = false;
    h->n = 0;
    h->x.reserve(n * 4 + 16); h->y.reserve(n * 4 + 16); h->z.reserve(n * 4 + 16);
    h->offs.reserve(16);
    if (n) {
      const cudaMemcpyKind k = mem == RVP_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
      RVP_CUDA_TRY(cudaMemcpyAsync(h->x.ptr, x, n * 4, k, ctx->stream));
      RVP_CUDA_TRY(cudaMemcpyAsync(h->y.ptr, y, n * 4, k, ctx->stream));
      RVP_CUDA_TRY(cudaMemcpyAsync(h->z.ptr, z, n * 4, k, ctx->stream));
    }
    int64_t o[2] = {0, (int64_t)n};
    RVP_CUDA_TRY(cudaMemcpyAsync(h->offs.ptr, o, 16, cudaMemcpyHostToDevice, ctx->stream));
    sync(ctx);
    h->n = n;
    h->cell = cell_size;
    h->has_cloud = true;
    h->built = false;
  });
}

rvp_status rvp_hash_build(rvp_hash *h) {
  if (!h) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = h->ctx;
  return guard(ctx, [&] {
    RVP_REQUIRE(h->has_cloud, "setInputCloud before build");
    set_device(ctx);
    h->built = false;  // set again only when this build has completed
    h->collision = 0;
    if (h->n > 0) {
      rvp::grid_build(ctx, h->grid, h->x.as<float>(), h->y.as<float>(), h->z.as<float>(),
                      h->offs.as<int64_t>(), 1, h->n, h->cell, rvp::KEY_REF_HASH, h->p1, h->p2,
                      nullptr);
      h->collision = read_back(ctx, h->grid.d_collision);
    }
    h->built = true;
  });
}

rvp_status rvp_hash_has_collisions(rvp_hash *h, int *out) {
  if (!h || !out) return RVP_ERR_INVALID_ARG;
  *out = h->collision;
  return RVP_OK;
}

rvp_status rvp_hash_radius_search(rvp_hash *h, const float *qx, const float *qy, const float *qz,
                                  size_t nq, float radius, int max_nn, int mem, int64_t *offsets,
                                  int32_t *indices, float *dists, size_t capacity, size_t *total) {
  if (!h) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = h->ctx;
  bool cap_fail = false;
  rvp_status s = guard(ctx, [&] {
    RVP_REQUIRE(h->built, "build before radiusSearch");
    RVP_REQUIRE(offsets && total, "offsets/total required");
    RVP_REQUIRE(nq == 0 || (qx && qy && qz), "null query pointer");
    set_device(ctx);
    *total = 0;
    RVP_REQUIRE(radius >= 0.0f, "radius must be >= 0");
    u64 *offs_d = reinterpret_cast<u64 *>(out_dev(ctx, 0, offsets, nq + 1, mem));
    if (nq == 0 || h->n == 0) {
      RVP_CUDA_TRY(cudaMemsetAsync(offs_d, 0, (nq + 1) * 8, ctx->stream));
      out_copy(ctx, offsets, reinterpret_cast<int64_t *>(offs_d), nq + 1, mem);
      sync(ctx);
      return;
    }
    const float *dqx = in_dev(ctx, 1, qx, nq, mem);
    const float *dqy = in_dev(ctx, 2, qy, nq, mem);
    const float *dqz = in_dev(ctx, 3, qz, nq, mem);
    rvp::QuerySet qs{dqx, dqy, dqz, nq, nullptr, nullptr, nullptr};
    const rvp::GridView gv = h->grid.view(rvp::KEY_REF_HASH, h->p1, h->p2);
    const bool refwin = h->collision != 0;
    void *scan_tmp = scratch(ctx, 4, rvp::scan_temp_bytes(nq + 1));
    if (max_nn > 0 && max_nn <= 64 && !refwin) {
      const int K = max_nn;
      u64 *pairs = static_cast<u64 *>(scratch(ctx, 5, nq * (size_t)K * 8));
      int32_t *cnt = static_cast<int32_t *>(scratch(ctx, 6, nq * 4));
      rvp::grid_knn(ctx, gv, qs, K, radius, pairs, cnt, 1, 256);
      u32 *ucnt = static_cast<u32 *>(scratch(ctx, 7, nq * 4));
      k_i32_to_u32<<<rvp::grid_for(nq, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(cnt, nq, ucnt);
      RVP_LAUNCH_CHECK(ctx);
      rvp::exclusive_scan_u32_to_u64(ctx, ucnt, offs_d, nq, nullptr, scan_tmp);
      const u64 tot = read_back(ctx, offs_d + nq);
      *total = (size_t)tot;
      if (tot > capacity) {
        out_copy(ctx, offsets, reinterpret_cast<int64_t *>(offs_d), nq + 1, mem);
        sync(ctx);
        cap_fail = true;
        return;
      }
      int32_t *di = out_dev(ctx, 8, indices, tot, mem);
      float *dd = out_dev(ctx, 9, dists, tot, mem);
      k_rows_to_csr<<<rvp::grid_for(nq * K, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(
          pairs, K, cnt, offs_d, nq, K, di, dd);
      RVP_LAUNCH_CHECK(ctx);
      out_copy(ctx, offsets, reinterpret_cast<int64_t *>(offs_d), nq + 1, mem);
      out_copy(ctx, indices, di, tot, mem);
      out_copy(ctx, dists, dd, tot, mem);
      sync(ctx);
      return;
    }
    u32 *cnt = static_cast<u32 *>(scratch(ctx, 6, nq * 4));
    rvp::grid_radius_count(ctx, gv, qs, radius, refwin, cnt);
    u64 *full = static_cast<u64 *>(scratch(ctx, 10, (nq + 1) * 8));
    rvp::exclusive_scan_u32_to_u64(ctx, cnt, full, nq, nullptr, scan_tmp);
    const u64 tot_full = read_back(ctx, full + nq);
    u64 tot = tot_full;
    if (max_nn > 0) {
      u32 *ccut = static_cast<u32 *>(scratch(ctx, 7, nq * 4));
      k_min_counts<<<rvp::grid_for(nq, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(
          cnt, nq, (u32)max_nn, ccut);
      RVP_LAUNCH_CHECK(ctx);
      rvp::exclusive_scan_u32_to_u64(ctx, ccut, offs_d, nq, nullptr, scan_tmp);
      tot = read_back(ctx, offs_d + nq);
    } else {
      RVP_CUDA_TRY(cudaMemcpyAsync(offs_d, full, (nq + 1) * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    *total = (size_t)tot;
    if (tot > capacity) {
      out_copy(ctx, offsets, reinterpret_cast<int64_t *>(offs_d), nq + 1, mem);
      sync(ctx);
      cap_fail = true;
      return;
    }
    u64 *pairs = static_cast<u64 *>(scratch(ctx, 5, (tot_full ? tot_full : 1) * 8));
    u32 *big = static_cast<u32 *>(scratch(ctx, 11, nq * 4 + 16));
    u32 *big_count = big + nq;
    rvp::grid_radius_fill(ctx, gv, qs, radius, refwin, full, 0, pairs, big, big_count);
    rvp::sort_big_segments(ctx, full, pairs, big, big_count, (u32)std::min<size_t>(nq, 4096));
    int32_t *di = out_dev(ctx, 8, indices, tot, mem);
    float *dd = out_dev(ctx, 9, dists, tot, mem);
    if (max_nn > 0) {
      k_csr_cut<<<rvp::grid_for(nq, 128, ctx->num_sms * 16), 128, 0, ctx->stream>>>(
          pairs, full, offs_d, nq, di, dd);
    } else {
      k_unpack<<<rvp::grid_for(tot, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(pairs, tot, di, dd);
    }
    RVP_LAUNCH_CHECK(ctx);
    out_copy(ctx, offsets, reinterpret_cast<int64_t *>(offs_d), nq + 1, mem);
    out_copy(ctx, indices, di, tot, mem);
    out_copy(ctx, dists, dd, tot, mem);
    sync(ctx);
  });
  if (s == RVP_OK && cap_fail) {
    ctx->last_error = "radius search: output capacity too small";
    return RVP_ERR_CAPACITY;
  }
  return s;
}

rvp_status rvp_hash_knn(rvp_hash *h, const float *qx, const float *qy, const float *qz, size_t nq,
                        int k, float radius, int mem, int32_t *indices, float *dists,
                        int32_t *counts) {
  if (!h) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = h->ctx;
  return guard(ctx, [&] {
    RVP_REQUIRE(h->built, "build before knn");
    RVP_REQUIRE(k >= 1 && k <= 64, "k must be in [1, 64]");
    RVP_REQUIRE(nq == 0 || (qx && qy && qz), "null query pointer");
    RVP_REQUIRE(h->collision == 0, "knn needs a collision-free hash (change the primes)");
    set_device(ctx);
    if (nq == 0) return;
    int32_t *dc = out_dev(ctx, 6, counts, nq, mem);
    int32_t *di = out_dev(ctx, 8, indices, nq * (size_t)k, mem);
    float *dd = out_dev(ctx, 9, dists, nq * (size_t)k, mem);
    if (h->n == 0) {
      if (dc) RVP_CUDA_TRY(cudaMemsetAsync(dc, 0, nq * 4, ctx->stream));
      if (di) RVP_CUDA_TRY(cudaMemsetAsync(di, 0xFF, nq * (size_t)k * 4, ctx->stream));
      out_copy(ctx, counts, dc, nq, mem);
      out_copy(ctx, indices, di, nq * (size_t)k, mem);
      sync(ctx);
      return;
    }
    const float *dqx = in_dev(ctx, 1, qx, nq, mem);
    const float *dqy = in_dev(ctx, 2, qy, nq, mem);
    const float *dqz = in_dev(ctx, 3, qz, nq, mem);
    rvp::QuerySet qs{dqx, dqy, dqz, nq, nullptr, nullptr, nullptr};
    u64 *pairs = static_cast<u64 *>(scratch(ctx, 5, nq * (size_t)k * 8));
    int32_t *cnt = dc ? dc : static_cast<int32_t *>(scratch(ctx, 7, nq * 4));
    rvp::grid_knn(ctx, h->grid.view(rvp::KEY_REF_HASH, h->p1, h->p2), qs, k, radius, pairs, cnt,
                  1, 256);
    k_fill_rows<<<rvp::grid_for(nq * k, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(
        pairs, k, cnt, nq, di, dd);
    RVP_LAUNCH_CHECK(ctx);
    out_copy(ctx, counts, dc, nq, mem);
    out_copy(ctx, indices, di, nq * (size_t)k, mem);
    out_copy(ctx, dists, dd, nq * (size_t)k, mem);
    sync(ctx);
  });
}

// ===========================================================================
// voxel grid
// ===========================================================================
rvp_status rvp_voxel_grid(rvp_context *ctx, const float *x, const float *y, const float *z,
                          size_t n, float leaf_size, int mem, float *out_aos, int32_t *keys,
                          size_t *out_count) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    RVP_REQUIRE(out_count, "out_count required");
    RVP_REQUIRE(n == 0 || (x && y && z && out_aos), "null pointer");
    RVP_REQUIRE(leaf_size > 0.0f && isfinite(leaf_size), "leaf_size must be > 0");
    RVP_REQUIRE(n < 0x7FFFFFFFull, "clouds are limited to 2^31 - 1 points");
    *out_count = 0;
    if (n == 0) return;  // voxel_grid_downsamp.cpp:185
    set_device(ctx);
    const float *dx = in_dev(ctx, 1, x, n, mem);
    const float *dy = in_dev(ctx, 2, y, n, mem);
    const float *dz = in_dev(ctx, 3, z, n, mem);
    int64_t *offs = single_frame_offsets(ctx, 4, n);
    float *dout = out_dev(ctx, 5, out_aos, 3 * n, mem);
    int32_t *dkeys = out_dev(ctx, 6, keys, 3 * n, mem);
    int64_t *vo = static_cast<int64_t *>(scratch(ctx, 7, 64));
    int *err = reinterpret_cast<int *>(vo + 4);
    if (!ctx->vwork) ctx->vwork = new rvp::VoxelWork();
    const float inv_leaf = 1.0f / leaf_size;  // voxel_grid_downsamp.cpp:189
    rvp::voxel_grid_run(ctx, *ctx->vwork, dx, dy, dz, offs, 1, n, nullptr, inv_leaf, dout, vo, dkeys, err,
                        nullptr, nullptr, nullptr);
    int64_t hv[2];
    int herr = 0;
    RVP_CUDA_TRY(cudaMemcpyAsync(hv, vo, 16, cudaMemcpyDeviceToHost, ctx->stream));
    RVP_CUDA_TRY(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    RVP_REQUIRE(!herr, "voxel index range does not fit one 64-bit key");
    const size_t v = (size_t)hv[1];
    out_copy(ctx, out_aos, dout, 3 * v, mem);
    out_copy(ctx, keys, dkeys, 3 * v, mem);
    sync(ctx);
    *out_count = v;
  });
}

// ===========================================================================
// SOR
// ===========================================================================
static void sor_common(rvp_context *ctx, const float *dx, const float *dy, const float *dz,
                       size_t n, const u64 *pairs, int kk, const int32_t *cnt, bool radius_mode,
                       float fallback, float alpha, int mem, float *out_aos, size_t *out_count,
                       float *mean_dists, uint8_t *keep) {
  float *mean = out_dev(ctx, 12, mean_dists, n, mem);
  if (!mean) mean = static_cast<float *>(scratch(ctx, 12, n * 4));
  uint8_t *dkeep = out_dev(ctx, 13, keep, n, mem);
  rvp::sor_mean_from_knn(ctx, pairs, kk, cnt, n, nullptr, mean, fallback, radius_mode);
  int64_t *offs = single_frame_offsets(ctx, 14, n);
  float *dout = out_dev(ctx, 15, out_aos, 3 * n, mem);
  int64_t *so = static_cast<int64_t *>(scratch(ctx, 16, 64));
  void *tmp = scratch(ctx, 17, rvp::sor_filter_temp_bytes(n, 1));
  rvp::sor_filter_frames(ctx, dx, dy, dz, mean, offs, 1, n, nullptr, alpha, dkeep, dout, so,
                         nullptr, tmp, nullptr, nullptr, nullptr, nullptr);
  int64_t hs[2];
  RVP_CUDA_TRY(cudaMemcpyAsync(hs, so, 16, cudaMemcpyDeviceToHost, ctx->stream));
  sync(ctx);
  const size_t kept = (size_t)hs[1];
  out_copy(ctx, out_aos, dout, 3 * kept, mem);
  out_copy(ctx, mean_dists, mean, n, mem);
  out_copy(ctx, keep, dkeep, n, mem);
  sync(ctx);
  *out_count = kept;
}

rvp_status rvp_sor(rvp_context *ctx, const float *x, const float *y, const float *z, size_t n,
                   int k, float alpha, int mem, float *out_aos, size_t *out_count,
                   float *mean_dists, uint8_t *keep) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    RVP_REQUIRE(out_count, "out_count required");
    *out_count = 0;
    if (n == 0) return;  // statistical_outlier_removal.cpp:70
    RVP_REQUIRE(x && y && z && out_aos, "null pointer");
    RVP_REQUIRE(k >= 1 && k + 1 <= 64, "k must be in [1, 63]");
    RVP_REQUIRE((size_t)k + 1 <= n, "k+1 must not exceed the number of points (the reference reads past its buffer)");
    RVP_REQUIRE(n < 0x7FFFFFFFull, "clouds are limited to 2^31 - 1 points");
    set_device(ctx);
    const float *dx = in_dev(ctx, 1, x, n, mem);
    const float *dy = in_dev(ctx, 2, y, n, mem);
    const float *dz = in_dev(ctx, 3, z, n, mem);
    const int kk = k + 1;
    u64 *pairs = static_cast<u64 *>(scratch(ctx, 9, n * (size_t)kk * 8));
    int32_t *cnt = static_cast<int32_t *>(scratch(ctx, 10, n * 4));
    knn_cloud(ctx, ctx_grid(ctx), dx, dy, dz, n, kk, pairs, cnt);
    sor_common(ctx, dx, dy, dz, n, pairs, kk, cnt, false, 0.0f, alpha, mem, out_aos, out_count,
               mean_dists, keep);
  });
}

rvp_status rvp_sor_spatial_hash(rvp_hash *h, int k, float alpha, float search_radius, int mem,
                                float *out_aos, size_t *out_count, float *mean_dists,
                                uint8_t *keep) {
  if (!h) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = h->ctx;
  return guard(ctx, [&] {
    RVP_REQUIRE(out_count, "out_count required");
    RVP_REQUIRE(h->built, "build before sor_spatial_hash");
    *out_count = 0;
    const size_t n = h->n;
    if (n == 0) return;
    RVP_REQUIRE(out_aos, "null output");
    RVP_REQUIRE(k >= 1 && k + 1 <= 64, "k must be in [1, 63]");
    RVP_REQUIRE(h->collision == 0, "sor_spatial_hash needs a collision-free hash");
    set_device(ctx);
    const int kk = k + 1;
    u64 *pairs = static_cast<u64 *>(scratch(ctx, 9, n * (size_t)kk * 8));
    int32_t *cnt = static_cast<int32_t *>(scratch(ctx, 10, n * 4));
    const float *dx = h->x.as<float>(), *dy = h->y.as<float>(), *dz = h->z.as<float>();
    rvp::QuerySet qs{dx, dy, dz, n, nullptr, nullptr, nullptr};
    rvp::grid_knn(ctx, h->grid.view(rvp::KEY_REF_HASH, h->p1, h->p2), qs, kk, search_radius,
                  pairs, cnt, 1, 256);
    sor_common(ctx, dx, dy, dz, n, pairs, kk, cnt, true, search_radius, alpha, mem, out_aos,
               out_count, mean_dists, keep);
  });
}

// ===========================================================================
// normals
// ===========================================================================
rvp_status rvp_normals_radius(rvp_hash *h, float radius, float vp_x, float vp_y, float vp_z,
                              int eigen_iters, int mem, float *nx, float *ny, float *nz) {
  if (!h) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = h->ctx;
  return guard(ctx, [&] {
    RVP_REQUIRE(h->built, "build before normal estimation");
    const size_t n = h->n;
    if (n == 0) return;  // normal_estimation.cpp:193
    RVP_REQUIRE(nx && ny && nz, "null output");
    set_device(ctx);
    const float *dx = h->x.as<float>(), *dy = h->y.as<float>(), *dz = h->z.as<float>();
    rvp::QuerySet qs{dx, dy, dz, n, nullptr, nullptr, nullptr};
    const rvp::GridView gv = h->grid.view(rvp::KEY_REF_HASH, h->p1, h->p2);
    const bool refwin = h->collision != 0;
    u32 *cnt = static_cast<u32 *>(scratch(ctx, 6, n * 4));
    rvp::grid_radius_count(ctx, gv, qs, radius, refwin, cnt);
    u64 *offs = static_cast<u64 *>(scratch(ctx, 10, (n + 1) * 8));
    rvp::exclusive_scan_u32_to_u64(ctx, cnt, offs, n, nullptr, scratch(ctx, 4, rvp::scan_temp_bytes(n + 1)));
    const u64 tot = read_back(ctx, offs + n);
    u64 *pairs = static_cast<u64 *>(scratch(ctx, 5, (tot ? tot : 1) * 8));
    u32 *big = static_cast<u32 *>(scratch(ctx, 11, n * 4 + 16));
    rvp::grid_radius_fill(ctx, gv, qs, radius, refwin, offs, 0, pairs, big, big + n);
    rvp::sort_big_segments(ctx, offs, pairs, big, big + n, (u32)std::min<size_t>(n, 4096));
    float *dnx = out_dev(ctx, 12, nx, n, mem), *dny = out_dev(ctx, 13, ny, n, mem),
          *dnz = out_dev(ctx, 14, nz, n, mem);
    rvp::normals_from_lists(ctx, dx, dy, dz, pairs, offs, nullptr, 0, n, nullptr, false,
                            eigen_iters, vp_x, vp_y, vp_z, dx, dy, dz, dnx, dny, dnz);
    out_copy(ctx, nx, dnx, n, mem);
    out_copy(ctx, ny, dny, n, mem);
    out_copy(ctx, nz, dnz, n, mem);
    sync(ctx);
  });
}

rvp_status rvp_normals_knn(rvp_context *ctx, const float *x, const float *y, const float *z,
                           size_t n, int k, float vp_x, float vp_y, float vp_z, int eigen_iters,
                           int mem, float *nx, float *ny, float *nz) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    if (n == 0) return;  // normal_estimation.cpp:75
    RVP_REQUIRE(x && y && z && nx && ny && nz, "null pointer");
    RVP_REQUIRE(k >= 1 && k + 1 <= 64, "k must be in [1, 63]");
    RVP_REQUIRE((size_t)k + 1 <= n, "k+1 must not exceed the number of points");
    set_device(ctx);
    const float *dx = in_dev(ctx, 1, x, n, mem);
    const float *dy = in_dev(ctx, 2, y, n, mem);
    const float *dz = in_dev(ctx, 3, z, n, mem);
    const int kk = k + 1;
    u64 *pairs = static_cast<u64 *>(scratch(ctx, 9, n * (size_t)kk * 8));
    int32_t *cnt = static_cast<int32_t *>(scratch(ctx, 10, n * 4));
    knn_cloud(ctx, ctx_grid(ctx), dx, dy, dz, n, kk, pairs, cnt);
    float *dnx = out_dev(ctx, 12, nx, n, mem), *dny = out_dev(ctx, 13, ny, n, mem),
          *dnz = out_dev(ctx, 14, nz, n, mem);
    rvp::normals_from_lists(ctx, dx, dy, dz, pairs, nullptr, cnt, kk, n, nullptr, true,
                            eigen_iters, vp_x, vp_y, vp_z, dx, dy, dz, dnx, dny, dnz);
    out_copy(ctx, nx, dnx, n, mem);
    out_copy(ctx, ny, dny, n, mem);
    out_copy(ctx, nz, dnz, n, mem);
    sync(ctx);
  });
}

rvp_status rvp_normals_knn_precise(rvp_context *ctx, const float *x, const float *y,
                                   const float *z, size_t n, int k, float vp_x, float vp_y,
                                   float vp_z, double cond_fp64, int mem, float *nx, float *ny,
                                   float *nz, float *cond, uint8_t *used_fp64) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    if (n == 0) return;
    RVP_REQUIRE(x && y && z && nx && ny && nz, "null pointer");
    RVP_REQUIRE(k >= 1 && k + 1 <= 64, "k must be in [1, 63]");
    RVP_REQUIRE((size_t)k + 1 <= n, "k+1 must not exceed the number of points");
    set_device(ctx);
    const float *dx = in_dev(ctx, 1, x, n, mem);
    const float *dy = in_dev(ctx, 2, y, n, mem);
    const float *dz = in_dev(ctx, 3, z, n, mem);
    const int kk = k + 1;
    u64 *pairs = static_cast<u64 *>(scratch(ctx, 9, n * (size_t)kk * 8));
    int32_t *cnt = static_cast<int32_t *>(scratch(ctx, 10, n * 4));
    knn_cloud(ctx, ctx_grid(ctx), dx, dy, dz, n, kk, pairs, cnt);
    float *dnx = out_dev(ctx, 12, nx, n, mem), *dny = out_dev(ctx, 13, ny, n, mem),
          *dnz = out_dev(ctx, 14, nz, n, mem);
    float *dc = out_dev(ctx, 15, cond, n, mem);
    uint8_t *du = out_dev(ctx, 16, used_fp64, n, mem);
    rvp::normals_precise(ctx, dx, dy, dz, pairs, kk, n, vp_x, vp_y, vp_z, cond_fp64, dnx, dny,
                         dnz, dc, du);
    out_copy(ctx, nx, dnx, n, mem);
    out_copy(ctx, ny, dny, n, mem);
    out_copy(ctx, nz, dnz, n, mem);
    out_copy(ctx, cond, dc, n, mem);
    out_copy(ctx, used_fp64, du, n, mem);
    sync(ctx);
  });
}

// ===========================================================================
// RANSAC
// ===========================================================================
rvp_status rvp_ransac_plane(rvp_context *ctx, const float *x, const float *y, const float *z,
                            size_t n, float dist_thresh, int max_iters, float collinear_thresh,
                            float probability, const int32_t *rand_stream, int mem, float *model,
                            int *best_count, int *iters_run, int32_t *counts) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    RVP_REQUIRE(model && best_count, "model/best_count required");
    RVP_REQUIRE(max_iters >= 0, "max_iters must be >= 0");
    if (iters_run) *iters_run = 0;
    *best_count = 0;
    if (n < 3) {  // ransac_plane.cpp:59 (no srand, no rand calls)
      return;
    }
    RVP_REQUIRE(x && y && z, "null cloud pointer");
    RVP_REQUIRE(n < 0x7FFFFFFFull, "clouds are limited to 2^31 - 1 points");
    set_device(ctx);
    const float *dx = in_dev(ctx, 1, x, n, mem);
    const float *dy = in_dev(ctx, 2, y, n, mem);
    const float *dz = in_dev(ctx, 3, z, n, mem);
    const size_t R = 3 * (size_t)max_iters;
    const bool own_stream = rand_stream == nullptr;
    std::vector<int32_t> rs;
    if (own_stream) {
      // the reference's srand(0) + rand() sequence, drawn from libc itself
      srand(0);
      rs.resize(R);
      for (size_t i = 0; i < R; ++i) rs[i] = rand();
    }
    int *drand = static_cast<int *>(scratch(ctx, 4, R * 4 + 16));
    if (R) {
      if (own_stream)
        RVP_CUDA_TRY(cudaMemcpyAsync(drand, rs.data(), R * 4, cudaMemcpyHostToDevice, ctx->stream));
      else
        RVP_CUDA_TRY(cudaMemcpyAsync(drand, rand_stream, R * 4,
                                     mem == RVP_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                           : cudaMemcpyHostToDevice,
                                     ctx->stream));
    }
    int64_t *offs = single_frame_offsets(ctx, 5, n);
    float *dm = static_cast<float *>(scratch(ctx, 6, 64));
    int32_t *db = reinterpret_cast<int32_t *>(dm + 8);
    int32_t *di = db + 2;
    int32_t *dcounts = counts ? static_cast<int32_t *>(scratch(ctx, 7, (size_t)max_iters * 4 + 4))
                              : nullptr;
    double pc = (double)probability;
    pc = pc < 0.5 ? 0.5 : (pc > 0.9999 ? 0.9999 : pc);
    rvp::RansacParams prm{dist_thresh, max_iters, collinear_thresh, log(1.0 - pc)};
    if (max_iters > 0)
      rvp::ransac_frames(ctx, dx, dy, dz, offs, 1, drand, prm, dm, db, di, dcounts,
                         counts != nullptr, rvp::RansacSampler{}, 8);
    float hm[4] = {0, 0, 0, 0};
    int32_t hb = 0, hi = 0;
    if (max_iters > 0) {
      RVP_CUDA_TRY(cudaMemcpyAsync(hm, dm, 16, cudaMemcpyDeviceToHost, ctx->stream));
      RVP_CUDA_TRY(cudaMemcpyAsync(&hb, db, 4, cudaMemcpyDeviceToHost, ctx->stream));
      RVP_CUDA_TRY(cudaMemcpyAsync(&hi, di, 4, cudaMemcpyDeviceToHost, ctx->stream));
      if (counts)
        RVP_CUDA_TRY(cudaMemcpyAsync(counts, dcounts, (size_t)max_iters * 4,
                                     mem == RVP_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                           : cudaMemcpyDeviceToHost,
                                     ctx->stream));
    }
    sync(ctx);
    if (own_stream) {
      // leave libc's generator where the reference leaves it: srand(0) and
      // three rand() calls per executed iteration
      srand(0);
      for (long i = 0; i < 3L * hi; ++i) (void)rand();
    }
    memcpy(model, hm, 16);
    *best_count = hb;
    if (iters_run) *iters_run = hi;
  });
}

// ===========================================================================
// Euclidean clustering
// ===========================================================================
rvp_status rvp_euclidean_clusters(rvp_context *ctx, const float *x, const float *y,
                                  const float *z, size_t n, float tolerance, int min_size,
                                  int max_size, int mem, int64_t *offsets, int32_t *indices,
                                  size_t *n_clusters) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    RVP_REQUIRE(offsets && n_clusters, "offsets / n_clusters required");
    *n_clusters = 0;
    if (n == 0) {  // euclidean_clustering.cpp:116-118
      if (mem == RVP_MEM_DEVICE) {
        set_device(ctx);
        RVP_CUDA_TRY(cudaMemsetAsync(offsets, 0, 8, ctx->stream));
        sync(ctx);
      } else {
        offsets[0] = 0;
      }
      return;
    }
    RVP_REQUIRE(x && y && z && indices, "null pointer");
    RVP_REQUIRE(tolerance > 0.0f, "tolerance must be > 0");
    RVP_REQUIRE(n < 0x7FFFFFFFull, "clouds are limited to 2^31 - 1 points");
    set_device(ctx);
    const float *dx = in_dev(ctx, 1, x, n, mem);
    const float *dy = in_dev(ctx, 2, y, n, mem);
    const float *dz = in_dev(ctx, 3, z, n, mem);
    int64_t *doffs = out_dev(ctx, 4, offsets, n + 1, mem);
    int32_t *didx = out_dev(ctx, 5, indices, n, mem);
    int64_t *fo = single_frame_offsets(ctx, 6, n);
    u64 *dcount = static_cast<u64 *>(scratch(ctx, 7, 64));
    rvp::euclidean_clusters_run(ctx, ctx_grid(ctx), dx, dy, dz, n, fo, tolerance, min_size,
                                max_size, doffs, didx, dcount,
                                scratch(ctx, 8, rvp::euclidean_temp_bytes(n)));
    u64 k = 0;
    RVP_CUDA_TRY(cudaMemcpyAsync(&k, dcount, 8, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    *n_clusters = (size_t)k;
    if (mem != RVP_MEM_DEVICE) {
      out_copy(ctx, offsets, doffs, (size_t)k + 1, mem);
      int64_t total = 0;
      RVP_CUDA_TRY(cudaMemcpyAsync(&total, doffs + k, 8, cudaMemcpyDeviceToHost, ctx->stream));
      sync(ctx);
      out_copy(ctx, indices, didx, (size_t)total, mem);
      sync(ctx);
    }
  });
}

rvp_status rvp_extract_plane(rvp_context *ctx, const float *x, const float *y, const float *z,
                             size_t n, const float *model, float dist_thresh, int mem,
                             float *inliers_aos, float *outliers_aos, size_t *n_inliers,
                             size_t *n_outliers) {
  if (!ctx) return RVP_ERR_INVALID_ARG;
  return guard(ctx, [&] {
    RVP_REQUIRE(model, "model required");
    if (n_inliers) *n_inliers = 0;
    if (n_outliers) *n_outliers = 0;
    if (n == 0) return;
    RVP_REQUIRE(x && y && z, "null cloud pointer");
    set_device(ctx);
    const float *dx = in_dev(ctx, 1, x, n, mem);
    const float *dy = in_dev(ctx, 2, y, n, mem);
    const float *dz = in_dev(ctx, 3, z, n, mem);
    const float *dmod = in_dev(ctx, 4, model, 4, mem);
    float *din = out_dev(ctx, 5, inliers_aos, 3 * n, mem);
    float *dout = out_dev(ctx, 6, outliers_aos, 3 * n, mem);
    u64 *dcnt = static_cast<u64 *>(scratch(ctx, 7, 32));
    rvp::extract_plane_run(ctx, dx, dy, dz, n, dmod, dist_thresh, din, dout, dcnt,
                           scratch(ctx, 8, rvp::extract_temp_bytes(n)));
    u64 hc[2];
    RVP_CUDA_TRY(cudaMemcpyAsync(hc, dcnt, 16, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    out_copy(ctx, inliers_aos, din, 3 * hc[0], mem);
    out_copy(ctx, outliers_aos, dout, 3 * hc[1], mem);
    sync(ctx);
    if (n_inliers) *n_inliers = (size_t)hc[0];
    if (n_outliers) *n_outliers = (size_t)hc[1];
  });
}

}  // extern "C"
