// Voxel-grid downsampling (voxel_grid_downsamp_sc, voxel_grid_downsamp.cpp
// :183-213, which is what voxel_grid_downsamp_rvv_v2 runs on a non-RISC-V
// host) for many frames at once.
//
//   key     (frame, ix - min_ix, iy - min_iy, iz - min_iz) packed in 64 bits,
//           ix = (int)floor(x * inv_leaf): unsigned order == the reference's
//           std::map<std::tuple<int,int,int>> order within a frame
//   sort    stable radix sort of (key, point index): each voxel becomes a run
//           whose points keep input order
//   reduce  one thread per voxel sums its run sequentially from 0.0f, in
//           input order (bit-identical to the map's running sums), then
//           centroid = sum * (1.0f / count)
#include "internal.cuh"

namespace rvp {

namespace {
inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

struct VoxelMeta {  // device scratch
  int shift_x, shift_y, shift_f;
  int error;
};

__device__ __forceinline__ int frame_of_index(const int64_t *offs, int n_frames, size_t i) {
  int lo = 0, hi = n_frames - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((size_t)offs[mid] <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void voxel_of(float x, float y, float z, float inv, int &vx, int &vy,
                                         int &vz) {
  vx = (int)floorf(fmul(x, inv));
  vy = (int)floorf(fmul(y, inv));
  vz = (int)floorf(fmul(z, inv));
}

__global__ void k_vox_init(int *mm, int n_frames) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n_frames; f += gridDim.x * blockDim.x) {
    mm[6 * f + 0] = mm[6 * f + 1] = mm[6 * f + 2] = 0x7FFFFFFF;
    mm[6 * f + 3] = mm[6 * f + 4] = mm[6 * f + 5] = (int)0x80000000;
  }
}

// Per-frame voxel-index bounds. Each warp owns one contiguous run of points
// and keeps its running min / max in registers, flushing them with atomics
// only when its run crosses into the next frame (a few atomics per warp
// instead of six per 32 points on the same frame's six words).
__global__ void k_vox_minmax(const float *x, const float *y, const float *z, const int64_t *offs,
                             int n_frames, size_t n_max, const u64 *n_dev, float inv, int *mm) {
  const size_t n = n_dev ? *n_dev : n_max;
  const int lane = threadIdx.x & 31;
  const size_t warps = ((size_t)gridDim.x * blockDim.x) >> 5;
  const size_t w = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t per = ((n + warps - 1) / warps + 31) & ~(size_t)31;
  const size_t a = w * per, e = a + per < n ? a + per : n;
  if (a >= e) return;
  int f = n_frames > 1 ? frame_of_index(offs, n_frames, a) : 0;
  size_t f_end = n_frames > 1 ? (size_t)offs[f + 1] : n;
  int lo[3] = {0x7FFFFFFF, 0x7FFFFFFF, 0x7FFFFFFF};
  int hi[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  auto flush = [&](int fr) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int l = __reduce_min_sync(0xffffffffu, lo[k]);
      const int h = __reduce_max_sync(0xffffffffu, hi[k]);
      if (lane == 0 && l <= h) {
        atomicMin(&mm[6 * fr + k], l);
        atomicMax(&mm[6 * fr + 3 + k], h);
      }
      lo[k] = 0x7FFFFFFF;
      hi[k] = (int)0x80000000;
    }
  };
  for (size_t base = a; base < e; base += 32) {
    // the frame changes at most a few times in a run: flush, then move on
    while (n_frames > 1 && base >= f_end && f + 1 < n_frames) {
      flush(f);
      ++f;
      f_end = (size_t)offs[f + 1];
    }
    const size_t i = base + lane;
    if (i < e) {
      if (i >= f_end) {  // this lane's point already belongs to a later frame
        int v[3];
        voxel_of(x[i], y[i], z[i], inv, v[0], v[1], v[2]);
        const int fi = frame_of_index(offs, n_frames, i);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          atomicMin(&mm[6 * fi + k], v[k]);
          atomicMax(&mm[6 * fi + 3 + k], v[k]);
        }
      } else {
        int v[3];
        voxel_of(x[i], y[i], z[i], inv, v[0], v[1], v[2]);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          lo[k] = min(lo[k], v[k]);
          hi[k] = max(hi[k], v[k]);
        }
      }
    }
  }
  flush(f);
}

__device__ __forceinline__ int bits_for(unsigned long long r) {
  return r == 0 ? 0 : 64 - __clzll((long long)r);
}

__global__ void k_vox_layout(const int *mm, int n_frames, VoxelMeta *meta) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long rx = 0, ry = 0, rz = 0;
  for (int f = 0; f < n_frames; ++f) {
    if (mm[6 * f + 0] > mm[6 * f + 3]) continue;  // empty frame
    rx = max(rx, (unsigned long long)((long long)mm[6 * f + 3] - mm[6 * f + 0]));
    ry = max(ry, (unsigned long long)((long long)mm[6 * f + 4] - mm[6 * f + 1]));
    rz = max(rz, (unsigned long long)((long long)mm[6 * f + 5] - mm[6 * f + 2]));
  }
  const int bx = bits_for(rx), by = bits_for(ry), bz = bits_for(rz);
  const int bf = bits_for((unsigned long long)(n_frames > 0 ? n_frames - 1 : 0));
  meta->shift_y = bz;
  meta->shift_x = bz + by;
  meta->shift_f = bz + by + bx;
  meta->error = (bf + bx + by + bz > 64) ? 1 : 0;
}

__global__ void k_vox_keys(const float *x, const float *y, const float *z, const int64_t *offs,
                           int n_frames, size_t n_max, const u64 *n_dev, float inv, const int *mm,
                           const VoxelMeta *meta, u64 *keys, u32 *vals) {
  const size_t n = n_dev ? *n_dev : n_max;
  const int sx = meta->shift_x, sy = meta->shift_y, sf = meta->shift_f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int f = n_frames > 1 ? frame_of_index(offs, n_frames, i) : 0;
    int vx, vy, vz;
    voxel_of(x[i], y[i], z[i], inv, vx, vy, vz);
    const u64 kx = (u64)(unsigned)(vx - mm[6 * f + 0]);
    const u64 ky = (u64)(unsigned)(vy - mm[6 * f + 1]);
    const u64 kz = (u64)(unsigned)(vz - mm[6 * f + 2]);
    const u64 kf = sf >= 64 ? 0 : ((u64)f << sf);
    keys[i] = kf | (sx >= 64 ? 0 : (kx << sx)) | (ky << sy) | kz;
    vals[i] = (u32)i;
  }
}

__global__ void k_vox_heads(const u64 *keys, size_t n_max, const u64 *n_dev, u32 *heads) {
  const size_t n = n_dev ? *n_dev : n_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    heads[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void k_vox_starts(const u32 *heads, const u64 *vid, size_t n_max, const u64 *n_dev,
                             u32 *vstart) {
  const size_t n = n_dev ? *n_dev : n_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    if (heads[i]) vstart[vid[i]] = (u32)i;
}

// one thread per voxel: sequential sums in input order, as the map did
__global__ void k_vox_centroids(const float *__restrict__ x, const float *__restrict__ y,
                                const float *__restrict__ z, const u32 *__restrict__ perm,
                                const u32 *__restrict__ vstart, const u64 *vid, size_t n_max,
                                const u64 *n_dev, float inv, float *out_aos, float *out_x,
                                float *out_y, float *out_z, int32_t *out_keys,
                                const VoxelMeta *meta) {
  if (meta->error) return;
  const size_t n = n_dev ? *n_dev : n_max;
  const u64 nv = vid[n];
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < nv;
       v += (u64)gridDim.x * blockDim.x) {
    const u32 s = vstart[v];
    const u32 e = (v + 1 < nv) ? vstart[v + 1] : (u32)n;
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (u32 j = s; j < e; ++j) {
      const u32 p = perm[j];
      sx = fadd(sx, x[p]);
      sy = fadd(sy, y[p]);
      sz = fadd(sz, z[p]);
    }
    const float f = fdiv(1.0f, (float)(int)(e - s));
    const float cx = fmul(sx, f), cy = fmul(sy, f), cz = fmul(sz, f);
    if (out_aos) {
      out_aos[3 * v + 0] = cx;
      out_aos[3 * v + 1] = cy;
      out_aos[3 * v + 2] = cz;
    }
    if (out_x) {
      out_x[v] = cx;
      out_y[v] = cy;
      out_z[v] = cz;
    }
    if (out_keys) {
      const u32 p = perm[s];
      int vx, vy, vz;
      voxel_of(x[p], y[p], z[p], inv, vx, vy, vz);
      out_keys[3 * v + 0] = vx;
      out_keys[3 * v + 1] = vy;
      out_keys[3 * v + 2] = vz;
    }
  }
}

// frames stay contiguous after the sort, so frame f's first voxel is the
// voxel id at its first sorted position
__global__ void k_vox_frame_offsets(const int64_t *offs, int n_frames, const u64 *vid,
                                    int64_t *out_offsets, const VoxelMeta *meta) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f <= n_frames; f += gridDim.x * blockDim.x)
    out_offsets[f] = meta->error ? 0 : (int64_t)vid[offs[f]];
}

__global__ void k_vox_error(const VoxelMeta *meta, int *flag) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && flag) *flag = meta->error;
}
}  // namespace

void VoxelWork::reserve(size_t n_max, int nf) {
  if (n_max < 1) n_max = 1;
  if (nf < 1) nf = 1;
  keys.reserve(n_max * 8);
  vals.reserve(n_max * 4);
  sort.reserve(sort_temp_bytes(n_max));
  heads.reserve(al(n_max * 4) + al((n_max + 1) * 8) + al(n_max * 4) + scan_temp_bytes(n_max));
  misc.reserve(al(6 * 4 * (size_t)nf) + al(sizeof(VoxelMeta)));
}

void VoxelWork::release() {
  keys.release(); vals.release(); sort.release(); heads.release(); misc.release();
}

void voxel_grid_run(rvp_context *ctx, VoxelWork &w, const float *x, const float *y,
                    const float *z, const int64_t *offs, int n_frames, size_t n_max,
                    const u64 *n_dev, float inv_leaf, float *out_aos, int64_t *out_offsets,
                    int32_t *out_keys, int *error_flag, float *out_x, float *out_y,
                    float *out_z) {
  w.reserve(n_max, n_frames);
  cudaStream_t st = ctx->stream;
  const int sms = ctx->num_sms;
  int *mm = w.misc.as<int>();
  VoxelMeta *meta = reinterpret_cast<VoxelMeta *>(w.misc.as<char>() + al(6 * 4 * (size_t)n_frames));
  char *hp = w.heads.as<char>();
  u32 *heads = reinterpret_cast<u32 *>(hp); hp += al(n_max * 4);
  u64 *vid = reinterpret_cast<u64 *>(hp); hp += al((n_max + 1) * 8);
  u32 *vstart = reinterpret_cast<u32 *>(hp); hp += al(n_max * 4);
  void *scan_tmp = hp;
  SortTemp t;
  sort_temp_carve(t, w.sort.ptr, n_max);

  k_vox_init<<<grid_for(n_frames, 256, 64), 256, 0, st>>>(mm, n_frames);
  RVP_LAUNCH_CHECK(ctx);
  k_vox_minmax<<<grid_for(n_max, 256, sms * 16), 256, 0, st>>>(x, y, z, offs, n_frames, n_max,
                                                              n_dev, inv_leaf, mm);
  RVP_LAUNCH_CHECK(ctx);
  k_vox_layout<<<1, 32, 0, st>>>(mm, n_frames, meta);
  RVP_LAUNCH_CHECK(ctx);
  k_vox_keys<<<grid_for(n_max, 256, sms * 16), 256, 0, st>>>(x, y, z, offs, n_frames, n_max,
                                                            n_dev, inv_leaf, mm, meta,
                                                            w.keys.as<u64>(), w.vals.as<u32>());
  RVP_LAUNCH_CHECK(ctx);
  radix_sort_pairs(ctx, w.keys.as<u64>(), w.vals.as<u32>(), n_max, n_dev, t);
  k_vox_heads<<<grid_for(n_max, 256, sms * 16), 256, 0, st>>>(w.keys.as<u64>(), n_max, n_dev,
                                                             heads);
  RVP_LAUNCH_CHECK(ctx);
  exclusive_scan_u32_to_u64(ctx, heads, vid, n_max, n_dev, scan_tmp);
  k_vox_starts<<<grid_for(n_max, 256, sms * 16), 256, 0, st>>>(heads, vid, n_max, n_dev, vstart);
  RVP_LAUNCH_CHECK(ctx);
  k_vox_centroids<<<grid_for(n_max, 256, sms * 16), 256, 0, st>>>(
      x, y, z, w.vals.as<u32>(), vstart, vid, n_max, n_dev, inv_leaf, out_aos, out_x, out_y,
      out_z, out_keys, meta);
  RVP_LAUNCH_CHECK(ctx);
  if (out_offsets) {
    k_vox_frame_offsets<<<grid_for(n_frames + 1, 256, 64), 256, 0, st>>>(offs, n_frames, vid,
                                                                        out_offsets, meta);
    RVP_LAUNCH_CHECK(ctx);
  }
  if (error_flag) {
    k_vox_error<<<1, 32, 0, st>>>(meta, error_flag);
    RVP_LAUNCH_CHECK(ctx);
  }
}

}  // namespace rvp
