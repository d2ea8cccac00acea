// Statistical outlier removal (statistical_outlier_removal.cpp).
//
//  * mean distance per point from its sorted k+1 nearest (self first):
//    sum of sqrtf(d2_j), j = 1..k, in ascending order, divided by k
//    (sor_sc :36-40); the radius-bounded variant (sor_spatial_hash
//    :246-270) divides by min(k, count - 1) and falls back to the search
//    radius for isolated points;
//  * global mean / std (:43-55): the reference sums sequentially in float,
//    so one lane per frame adds the values in input order (a parallel tree
//    sum would round differently and move the threshold), fed through
//    shared memory by its warp;
//  * keep mean <= mu + alpha * sigma and copy kept points out in input order
//    (flag scan + scatter).
#include "internal.cuh"

namespace rvp {

namespace {
inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

__device__ __forceinline__ int frame_of_index(const int64_t *offs, int n_frames, size_t i) {
  int lo = 0, hi = n_frames - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((size_t)offs[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void k_sor_mean(const u64 *pairs, int kk, const int32_t *counts, size_t n_max,
                           const u64 *n_dev, float *mean, float fallback, bool radius_mode) {
  const size_t n = n_dev ? *n_dev : n_max;
  const int k = kk - 1;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int cnt = counts ? counts[i] : kk;
    const u64 *l = pairs + i * (size_t)kk;
    if (radius_mode && cnt <= 1) {
      mean[i] = fallback;
      continue;
    }
    const int valid_k = cnt - 1 < k ? cnt - 1 : k;
    float sum = 0.0f;
    for (int j = 1; j <= valid_k; ++j) sum = fadd(sum, __fsqrt_rn(nbr_d2(l[j])));
    mean[i] = valid_k > 0 ? fdiv(sum, (float)valid_k) : 0.0f;
  }
}

// One warp per frame: lanes stage 1024 consecutive values in shared memory
// (coalesced), then lane 0 adds them in input order -- the same sequence of
// roundings as the reference's loop, without one global load per add.
constexpr int ST_CHUNK = 1024;
__global__ __launch_bounds__(32) void k_sor_stats_warp(const float *__restrict__ mean,
                                                       const int64_t *offs, int n_frames,
                                                       float alpha, float *thresh) {
  __shared__ float buf[ST_CHUNK];
  const int f = blockIdx.x;
  if (f >= n_frames) return;
  const int lane = threadIdx.x;
  const int64_t a = offs[f], b = offs[f + 1];
  const int64_t n = b - a;
  if (n <= 0) {
    if (lane == 0) thresh[f] = 0.0f;
    return;
  }
  float s = 0.0f;
  for (int64_t base = a; base < b; base += ST_CHUNK) {
    const int m = (int)((b - base) < ST_CHUNK ? (b - base) : ST_CHUNK);
    for (int j = lane; j < m; j += 32) buf[j] = __ldg(&mean[base + j]);
    __syncwarp();
    if (lane == 0)
      for (int t = 0; t < m; ++t) s = fadd(s, buf[t]);
    __syncwarp();
  }
  const float mu = __shfl_sync(0xffffffffu, fdiv(s, (float)n), 0);
  float var = 0.0f;
  for (int64_t base = a; base < b; base += ST_CHUNK) {
    const int m = (int)((b - base) < ST_CHUNK ? (b - base) : ST_CHUNK);
    for (int j = lane; j < m; j += 32) buf[j] = __ldg(&mean[base + j]);
    __syncwarp();
    if (lane == 0)
      for (int t = 0; t < m; ++t) {
        const float d = fsub(buf[t], mu);
        var = fadd(var, fmul(d, d));
      }
    __syncwarp();
  }
  if (lane == 0) {
    const float sd = __fsqrt_rn(fdiv(var, (float)n));
    thresh[f] = fadd(mu, fmul(alpha, sd));
  }
}

__global__ void k_sor_keep(const float *mean, const int64_t *offs, int n_frames, size_t n_max,
                           const u64 *n_dev, const float *thresh, uint8_t *keep, u32 *flags) {
  const size_t n = n_dev ? *n_dev : n_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int f = n_frames > 1 ? frame_of_index(offs, n_frames, i) : 0;
    const bool k = mean[i] <= thresh[f];
    if (keep) keep[i] = k ? 1 : 0;
    flags[i] = k ? 1u : 0u;
  }
}

__global__ void k_sor_scatter(const float *x, const float *y, const float *z, const u32 *flags,
                              const u64 *pos, size_t n_max, const u64 *n_dev, float *out_aos,
                              float *out_x, float *out_y, float *out_z, u32 *src_index) {
  const size_t n = n_dev ? *n_dev : n_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    if (!flags[i]) continue;
    const u64 p = pos[i];
    const float a = x[i], b = y[i], c = z[i];
    if (out_aos) {
      out_aos[3 * p + 0] = a;
      out_aos[3 * p + 1] = b;
      out_aos[3 * p + 2] = c;
    }
    if (out_x) {
      out_x[p] = a;
      out_y[p] = b;
      out_z[p] = c;
    }
    if (src_index) src_index[p] = (u32)i;
  }
}

__global__ void k_sor_frame_offsets(const int64_t *offs, int n_frames, const u64 *pos,
                                    int64_t *out) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f <= n_frames; f += gridDim.x * blockDim.x)
    out[f] = (int64_t)pos[offs[f]];
}
}  // namespace

void sor_mean_from_knn(rvp_context *ctx, const u64 *pairs, int kk, const int32_t *counts,
                       size_t n_max, const u64 *n_dev, float *mean, float fallback_radius,
                       bool radius_mode) {
  k_sor_mean<<<grid_for(n_max, 256, ctx->num_sms * 16), 256, 0, ctx->stream>>>(
      pairs, kk, counts, n_max, n_dev, mean, fallback_radius, radius_mode);
  RVP_LAUNCH_CHECK(ctx);
}

u64 *sor_positions(void *temp, size_t n_max) {
  return reinterpret_cast<u64 *>(static_cast<char *>(temp) + al(n_max * 4));
}

size_t sor_filter_temp_bytes(size_t n_max, int n_frames) {
  return al(n_max * 4) + al((n_max + 1) * 8) + al((size_t)(n_frames + 1) * 4) +
         scan_temp_bytes(n_max);
}

void sor_filter_frames(rvp_context *ctx, const float *x, const float *y, const float *z,
                       const float *mean, const int64_t *offs, int n_frames, size_t n_max,
                       const u64 *n_dev, float alpha, uint8_t *keep, float *out_aos,
                       int64_t *out_offsets, float *thresh_out, void *temp, float *out_x,
                       float *out_y, float *out_z, u32 *src_index) {
  char *p = static_cast<char *>(temp);
  u32 *flags = reinterpret_cast<u32 *>(p); p += al(n_max * 4);
  u64 *pos = reinterpret_cast<u64 *>(p); p += al((n_max + 1) * 8);
  float *thresh = thresh_out ? thresh_out : reinterpret_cast<float *>(p);
  p += al((size_t)(n_frames + 1) * 4);
  void *scan_tmp = p;
  cudaStream_t st = ctx->stream;
  k_sor_stats_warp<<<(unsigned)(n_frames > 0 ? n_frames : 1), 32, 0, st>>>(mean, offs, n_frames,
                                                                         alpha, thresh);
  RVP_LAUNCH_CHECK(ctx);
  k_sor_keep<<<grid_for(n_max, 256, ctx->num_sms * 16), 256, 0, st>>>(mean, offs, n_frames, n_max,
                                                                     n_dev, thresh, keep, flags);
  RVP_LAUNCH_CHECK(ctx);
  exclusive_scan_u32_to_u64(ctx, flags, pos, n_max, n_dev, scan_tmp);
  k_sor_scatter<<<grid_for(n_max, 256, ctx->num_sms * 16), 256, 0, st>>>(
      x, y, z, flags, pos, n_max, n_dev, out_aos, out_x, out_y, out_z, src_index);
  RVP_LAUNCH_CHECK(ctx);
  if (out_offsets) {
    k_sor_frame_offsets<<<grid_for(n_frames + 1, 256, 64), 256, 0, st>>>(offs, n_frames, pos,
                                                                        out_offsets);
    RVP_LAUNCH_CHECK(ctx);
  }
}

}  // namespace rvp
