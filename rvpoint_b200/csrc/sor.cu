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
// One block of two warps per frame: warp 1 stages the next chunk of means
// in shared memory while lane 0 of warp 0 adds up the current one in input
// order (the reference's sequential float sums), four values per load.
__global__ __launch_bounds__(64) void k_sor_stats_warp(const float *__restrict__ mean,
                                                       const int64_t *offs, int n_frames,
                                                       float alpha, float *thresh) {
  __shared__ __align__(16) float buf[2][ST_CHUNK];
  __shared__ float s_mu;
  const int f = blockIdx.x;
  if (f >= n_frames) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t a = offs[f], b = offs[f + 1];
  const int64_t n = b - a;
  if (n <= 0) {
    if (tid == 0) thresh[f] = 0.0f;
    return;
  }
  const int nch = (int)((n + ST_CHUNK - 1) / ST_CHUNK);
  auto stage = [&](int c) {
    const int64_t base = a + (int64_t)c * ST_CHUNK;
    const int m = (int)((b - base) < ST_CHUNK ? (b - base) : ST_CHUNK);
    float *dst = buf[c & 1];
    for (int j = lane; j < m; j += 32) dst[j] = __ldg(&mean[base + j]);
  };
  float acc = 0.0f;
  for (int pass = 0; pass < 2; ++pass) {
    const float mu = pass ? s_mu : 0.0f;
    if (warp == 1) stage(0);
    __syncthreads();
    for (int c = 0; c < nch; ++c) {
      if (warp == 1 && c + 1 < nch) stage(c + 1);
      if (tid == 0) {
        const int m = (int)((n - (int64_t)c * ST_CHUNK) < ST_CHUNK ? (n - (int64_t)c * ST_CHUNK)
                                                                   : ST_CHUNK);
        const float *src = buf[c & 1];
        const float4 *src4 = reinterpret_cast<const float4 *>(src);
        int t = 0;
        for (; t + 4 <= m; t += 4) {
          const float4 v = src4[t >> 2];
          if (pass == 0) {
            acc = fadd(acc, v.x); acc = fadd(acc, v.y); acc = fadd(acc, v.z); acc = fadd(acc, v.w);
          } else {
            float d = fsub(v.x, mu); acc = fadd(acc, fmul(d, d));
            d = fsub(v.y, mu); acc = fadd(acc, fmul(d, d));
            d = fsub(v.z, mu); acc = fadd(acc, fmul(d, d));
            d = fsub(v.w, mu); acc = fadd(acc, fmul(d, d));
          }
        }
        for (; t < m; ++t) {
          if (pass == 0) {
            acc = fadd(acc, src[t]);
          } else {
            const float d = fsub(src[t], mu);
            acc = fadd(acc, fmul(d, d));
          }
        }
      }
      __syncthreads();
    }
    if (tid == 0) {
      if (pass == 0) {
        s_mu = fdiv(acc, (float)n);
        acc = 0.0f;
      } else {
        const float sd = __fsqrt_rn(fdiv(acc, (float)n));
        thresh[f] = fadd(s_mu, fmul(alpha, sd));
      }
    }
    __syncthreads();
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
  k_sor_stats_warp<<<(unsigned)(n_frames > 0 ? n_frames : 1), 64, 0, st>>>(mean, offs, n_frames,
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
