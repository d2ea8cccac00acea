// Stable LSD radix sort of (u64 key, u32 value) pairs for sm_100a.
//
// Per live 8-bit digit: (1) tile histogram, (2) per-digit scan over tiles,
// (3) tile-local stable ranking with __match_any_sync, reorder in shared
// memory, coalesced scatter of each digit run. A digit is live when the keys
// differ in it (global OR ^ AND of all keys), so a 64-bit key with 30 live
// bits costs 4 passes. Pass kernels read the key count and the live mask from
// device memory; nothing returns to the host, so a sort can sit in a graph.
#include "internal.cuh"

namespace rvp {

namespace {
constexpr int TH = 256;
constexpr int ITEMS = 16;
constexpr int TILE = TH * ITEMS;  // 4096 keys per tile
constexpr int WARPS = TH / 32;
constexpr int CHUNK = TILE / WARPS;  // 512 keys per warp, in order

__host__ __device__ inline size_t tiles_for(size_t n) { return (n + TILE - 1) / TILE; }

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

__device__ __forceinline__ u64 live_mask(const u64 *orand) {
  return orand[0] ^ orand[1];
}
__device__ __forceinline__ bool pass_live(u64 live, int pass) {
  return ((live >> (8 * pass)) & 0xFFull) != 0;
}
// buffer holding the input of `pass`: parity of live passes below it
__device__ __forceinline__ int pass_src(u64 live, int pass) {
  int c = 0;
  for (int q = 0; q < pass; ++q) c += pass_live(live, q) ? 1 : 0;
  return c & 1;
}

__global__ void k_orand(const u64 *__restrict__ keys, size_t n_max,
                        const u64 *__restrict__ n_dev, u64 *orand) {
  const size_t n = n_dev ? *n_dev : n_max;
  u64 o = 0, a = ~0ull;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const u64 k = keys[i];
    o |= k;
    a &= k;
  }
  unsigned olo = __reduce_or_sync(0xffffffffu, (unsigned)o);
  unsigned ohi = __reduce_or_sync(0xffffffffu, (unsigned)(o >> 32));
  unsigned alo = __reduce_and_sync(0xffffffffu, (unsigned)a);
  unsigned ahi = __reduce_and_sync(0xffffffffu, (unsigned)(a >> 32));
  if ((threadIdx.x & 31) == 0) {
    atomicOr(&orand[0], ((u64)ohi << 32) | olo);
    atomicAnd(&orand[1], ((u64)ahi << 32) | alo);
  }
}

__global__ __launch_bounds__(TH) void k_hist(const u64 *k0, const u64 *k1,
                                            size_t n_max, const u64 *n_dev,
                                            const u64 *orand, int pass,
                                            u32 *tile_hist, size_t t_max) {
  const u64 live = live_mask(orand);
  if (!pass_live(live, pass)) return;
  const u64 *kin = pass_src(live, pass) ? k1 : k0;
  const size_t n = n_dev ? *n_dev : n_max;
  const size_t base = (size_t)blockIdx.x * TILE;
  if (base >= n) return;
  __shared__ u32 h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int shift = 8 * pass;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = 0; r < ITEMS; ++r) {
    const size_t i = base + (size_t)w * CHUNK + (size_t)r * 32 + lane;
    const bool valid = i < n;
    const unsigned vm = __ballot_sync(0xffffffffu, valid);
    if (valid) {
      const unsigned d = (unsigned)((kin[i] >> shift) & 0xFF);
      const unsigned m = __match_any_sync(vm, d);
      if ((m & ((1u << lane) - 1)) == 0) atomicAdd(&h[d], __popc(m));
    }
  }
  __syncthreads();
  tile_hist[(size_t)threadIdx.x * t_max + blockIdx.x] = h[threadIdx.x];
}

// block d: exclusive scan over the live tiles of digit d, in place; totals[d].
__global__ __launch_bounds__(TH) void k_scan_digit(u32 *tile_hist, size_t t_max,
                                                  size_t n_max, const u64 *n_dev,
                                                  const u64 *orand, int pass,
                                                  u32 *totals) {
  if (!pass_live(live_mask(orand), pass)) return;
  const size_t n = n_dev ? *n_dev : n_max;
  const size_t T = tiles_for(n);
  u32 *row = tile_hist + (size_t)blockIdx.x * t_max;
  const size_t per = (T + TH - 1) / TH;
  const size_t a = threadIdx.x * per;
  const size_t b = a + per < T ? a + per : T;
  u32 s = 0;
  for (size_t t = a; t < b; ++t) s += row[t];
  __shared__ u32 sh[TH];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < TH; off <<= 1) {
    u32 v = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  u32 run = sh[threadIdx.x] - s;
  for (size_t t = a; t < b; ++t) {
    const u32 c = row[t];
    row[t] = run;
    run += c;
  }
  if (threadIdx.x == TH - 1) totals[blockIdx.x] = sh[TH - 1];
}

__global__ __launch_bounds__(TH) void k_scatter(u64 *k0, u32 *v0, u64 *k1, u32 *v1,
                                               size_t n_max, const u64 *n_dev,
                                               const u64 *orand, int pass,
                                               const u32 *tile_scan, size_t t_max,
                                               const u32 *totals) {
  const u64 live = live_mask(orand);
  if (!pass_live(live, pass)) return;
  const int src = pass_src(live, pass);
  const u64 *kin = src ? k1 : k0;
  const u32 *vin = src ? v1 : v0;
  u64 *kout = src ? k0 : k1;
  u32 *vout = src ? v0 : v1;
  const size_t n = n_dev ? *n_dev : n_max;
  const size_t base = (size_t)blockIdx.x * TILE;
  if (base >= n) return;

  extern __shared__ __align__(16) unsigned char smem[];
  u64 *skeys = reinterpret_cast<u64 *>(smem);                 // TILE
  u32 *svals = reinterpret_cast<u32 *>(skeys + TILE);         // TILE
  u32 *wh = svals + TILE;                                     // WARPS*256
  u32 *dstart = wh + WARPS * 256;                             // 256
  u32 *gbase = dstart + 256;                                  // 256

  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  for (int j = tid; j < WARPS * 256; j += TH) wh[j] = 0;
  // digit bases over the whole key set: exclusive scan of totals
  {
    u32 t = totals[tid];
    dstart[tid] = t;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
      u32 v = tid >= off ? dstart[tid - off] : 0;
      __syncthreads();
      dstart[tid] += v;
      __syncthreads();
    }
    gbase[tid] = dstart[tid] - t + tile_scan[(size_t)tid * t_max + blockIdx.x];
  }
  __syncthreads();

  const int shift = 8 * pass;
  const unsigned lt = (1u << lane) - 1;
  u64 key[ITEMS];
  u32 val[ITEMS];
  unsigned short pos[ITEMS];
#pragma unroll
  for (int r = 0; r < ITEMS; ++r) {
    const size_t i = base + (size_t)w * CHUNK + (size_t)r * 32 + lane;
    const bool valid = i < n;
    key[r] = valid ? kin[i] : 0;
    val[r] = valid ? vin[i] : 0;
  }
#pragma unroll
  for (int r = 0; r < ITEMS; ++r) {
    const size_t i = base + (size_t)w * CHUNK + (size_t)r * 32 + lane;
    const bool valid = i < n;
    const unsigned vm = __ballot_sync(0xffffffffu, valid);
    unsigned m = 0, d = 0, c = 0;
    if (valid) {
      d = (unsigned)((key[r] >> shift) & 0xFF);
      m = __match_any_sync(vm, d);
      c = wh[w * 256 + d];
      pos[r] = (unsigned short)(c + __popc(m & lt));
    }
    __syncwarp();
    if (valid && (m & lt) == 0) wh[w * 256 + d] = c + __popc(m);
    __syncwarp();
  }
  __syncthreads();
  {  // per digit: exclusive over warps, then tile-local digit starts
    u32 run = 0;
    for (int q = 0; q < WARPS; ++q) {
      const u32 c = wh[q * 256 + tid];
      wh[q * 256 + tid] = run;
      run += c;
    }
    __syncthreads();
    dstart[tid] = run;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
      u32 v = tid >= off ? dstart[tid - off] : 0;
      __syncthreads();
      dstart[tid] += v;
      __syncthreads();
    }
    dstart[tid] -= run;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < ITEMS; ++r) {
    const size_t i = base + (size_t)w * CHUNK + (size_t)r * 32 + lane;
    if (i < n) {
      const unsigned d = (unsigned)((key[r] >> shift) & 0xFF);
      const u32 p = dstart[d] + wh[w * 256 + d] + pos[r];
      skeys[p] = key[r];
      svals[p] = val[r];
    }
  }
  __syncthreads();
  const size_t cnt = (n - base) < (size_t)TILE ? (n - base) : (size_t)TILE;
  for (int j = tid; j < (int)cnt; j += TH) {
    const u64 k = skeys[j];
    const unsigned d = (unsigned)((k >> shift) & 0xFF);
    const size_t dst = (size_t)gbase[d] + (size_t)(j - (int)dstart[d]);
    kout[dst] = k;
    vout[dst] = svals[j];
  }
}

__global__ void k_copy_back(u64 *k0, u32 *v0, const u64 *k1, const u32 *v1,
                            size_t n_max, const u64 *n_dev, const u64 *orand) {
  const u64 live = live_mask(orand);
  int c = 0;
  for (int q = 0; q < 8; ++q) c += pass_live(live, q) ? 1 : 0;
  if ((c & 1) == 0) return;
  const size_t n = n_dev ? *n_dev : n_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    k0[i] = k1[i];
    v0[i] = v1[i];
  }
}

constexpr size_t kScatterSmem =
    (size_t)TILE * 8 + (size_t)TILE * 4 + (size_t)WARPS * 256 * 4 + 256 * 4 * 2;
}  // namespace

size_t sort_temp_bytes(size_t n_max) {
  const size_t T = tiles_for(n_max) > 0 ? tiles_for(n_max) : 1;
  return al(n_max * 8) + al(n_max * 4) + al(256 * T * 4) + al(256 * 4) + al(64);
}

void sort_temp_carve(SortTemp &t, void *base, size_t n_max) {
  const size_t T = tiles_for(n_max) > 0 ? tiles_for(n_max) : 1;
  char *p = static_cast<char *>(base);
  t.keys_alt = reinterpret_cast<u64 *>(p); p += al(n_max * 8);
  t.vals_alt = reinterpret_cast<u32 *>(p); p += al(n_max * 4);
  t.tile_hist = reinterpret_cast<u32 *>(p); p += al(256 * T * 4);
  t.global_hist = reinterpret_cast<u32 *>(p); p += al(256 * 4);  // digit totals
  t.pass_info = reinterpret_cast<int *>(p);                      // or/and words
}

void radix_sort_pairs(rvp_context *ctx, u64 *keys, u32 *vals, size_t n_max,
                      const u64 *n_dev, const SortTemp &t) {
  if (n_max == 0) return;
  static bool attr_set[64] = {false};
  int dev = ctx->device;
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    RVP_CUDA_TRY(cudaFuncSetAttribute(k_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kScatterSmem));
    attr_set[dev] = true;
  }
  const size_t T = tiles_for(n_max);
  u64 *orand = reinterpret_cast<u64 *>(t.pass_info);
  RVP_CUDA_TRY(cudaMemsetAsync(orand, 0x00, 8, ctx->stream));
  RVP_CUDA_TRY(cudaMemsetAsync(orand + 1, 0xFF, 8, ctx->stream));
  k_orand<<<grid_for(n_max, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(keys, n_max, n_dev,
                                                                           orand);
  RVP_LAUNCH_CHECK(ctx);
  for (int pass = 0; pass < 8; ++pass) {
    k_hist<<<(unsigned)T, TH, 0, ctx->stream>>>(keys, t.keys_alt, n_max, n_dev, orand, pass,
                                                t.tile_hist, T);
    RVP_LAUNCH_CHECK(ctx);
    k_scan_digit<<<256, TH, 0, ctx->stream>>>(t.tile_hist, T, n_max, n_dev, orand, pass,
                                             t.global_hist);
    RVP_LAUNCH_CHECK(ctx);
    k_scatter<<<(unsigned)T, TH, kScatterSmem, ctx->stream>>>(keys, vals, t.keys_alt,
                                                             t.vals_alt, n_max, n_dev, orand,
                                                             pass, t.tile_hist, T,
                                                             t.global_hist);
    RVP_LAUNCH_CHECK(ctx);
  }
  k_copy_back<<<grid_for(n_max, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(
      keys, vals, t.keys_alt, t.vals_alt, n_max, n_dev, orand);
  RVP_LAUNCH_CHECK(ctx);
}

// ---------------------------------------------------------------------------
// exclusive scan u32 -> u64 (3 kernels: tile sums, scan of tile sums, apply)
// ---------------------------------------------------------------------------
namespace {
// a tile: 256 threads x 16 consecutive items (four 16-byte loads each)
constexpr int SC_TH = 256, SC_IT = 16, SC_TILE = SC_TH * SC_IT;

// the thread's 16 items (zero past n): vector loads where the whole run is
// live and 16-byte aligned
__device__ __forceinline__ void scan_load(const u32 *in, size_t i0, size_t n, u32 (&v)[SC_IT]) {
  if (i0 + SC_IT <= n && (reinterpret_cast<uintptr_t>(in + i0) & 15) == 0) {
    const uint4 *p = reinterpret_cast<const uint4 *>(in + i0);
#pragma unroll
    for (int j = 0; j < SC_IT / 4; ++j) {
      const uint4 t = __ldg(p + j);
      v[4 * j] = t.x; v[4 * j + 1] = t.y; v[4 * j + 2] = t.z; v[4 * j + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < SC_IT; ++j) v[j] = (i0 + j < n) ? in[i0 + j] : 0u;
  }
}

// block-wide exclusive scan of one u64 per thread (warp shuffles, then the
// warps' totals); returns the exclusive prefix, *total the block's sum
__device__ __forceinline__ u64 block_exclusive(u64 s, u64 *warp_tot, u64 &total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  u64 incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u64 t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[w] = incl;
  __syncthreads();
  u64 before = 0;
  total = 0;
#pragma unroll
  for (int k = 0; k < SC_TH / 32; ++k) {
    const u64 t = warp_tot[k];
    if (k < w) before += t;
    total += t;
  }
  return before + incl - s;
}

// (batched scans: blockIdx.y picks the array; strides in elements)
__global__ __launch_bounds__(SC_TH) void k_scan_tiles(const u32 *in, size_t n_max,
                                                      const u64 *n_dev, u64 *tsum,
                                                      size_t in_stride, size_t ts_stride) {
  in += blockIdx.y * in_stride;
  tsum += blockIdx.y * ts_stride;
  const size_t n = n_dev ? *n_dev : n_max;
  const size_t base = (size_t)blockIdx.x * SC_TILE;
  if (base >= n) return;
  u32 v[SC_IT];
  scan_load(in, base + (size_t)threadIdx.x * SC_IT, n, v);
  u64 s64 = 0;
#pragma unroll
  for (int j = 0; j < SC_IT; ++j) s64 += v[j];
  __shared__ u64 sh[SC_TH / 32];
  u64 r = s64;
#pragma unroll
  for (int o = 16; o; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    u64 t = 0;
#pragma unroll
    for (int q = 0; q < SC_TH / 32; ++q) t += sh[q];
    tsum[blockIdx.x] = t;
  }
}

__global__ void k_scan_sums(u64 *tsum, size_t nt_max, size_t n_max, const u64 *n_dev,
                            u64 *out, size_t out_stride, size_t ts_stride) {
  tsum += blockIdx.x * ts_stride;
  out += blockIdx.x * out_stride;
  const size_t n = n_dev ? *n_dev : n_max;
  const size_t nt = (n + SC_TILE - 1) / SC_TILE;
  __shared__ u64 sh[1024];
  const size_t per = (nt + 1023) / 1024;
  const size_t a = threadIdx.x * per, b = a + per < nt ? a + per : nt;
  u64 s = 0;
  for (size_t t = a; t < b; ++t) s += tsum[t];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    u64 v = threadIdx.x >= (unsigned)off ? sh[threadIdx.x - off] : 0;
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  u64 run = sh[threadIdx.x] - s;
  for (size_t t = a; t < b; ++t) {
    const u64 c = tsum[t];
    tsum[t] = run;
    run += c;
  }
  if (threadIdx.x == 1023) out[n] = sh[1023];
  (void)nt_max;
}

__global__ __launch_bounds__(SC_TH) void k_scan_apply(const u32 *in, size_t n_max,
                                                      const u64 *n_dev, const u64 *tsum,
                                                      u64 *out, size_t in_stride,
                                                      size_t out_stride, size_t ts_stride) {
  in += blockIdx.y * in_stride;
  out += blockIdx.y * out_stride;
  tsum += blockIdx.y * ts_stride;
  const size_t n = n_dev ? *n_dev : n_max;
  const size_t base = (size_t)blockIdx.x * SC_TILE;
  if (base >= n) return;
  // thread t owns SC_IT consecutive items
  const size_t i0 = base + (size_t)threadIdx.x * SC_IT;
  u32 v[SC_IT];
  scan_load(in, i0, n, v);
  u64 s = 0;
#pragma unroll
  for (int j = 0; j < SC_IT; ++j) s += v[j];
  __shared__ u64 warp_tot[SC_TH / 32];
  u64 total;
  u64 run = tsum[blockIdx.x] + block_exclusive(s, warp_tot, total);
  if (i0 + SC_IT <= n && (reinterpret_cast<uintptr_t>(out + i0) & 15) == 0) {
    ulonglong2 *o = reinterpret_cast<ulonglong2 *>(out + i0);
#pragma unroll
    for (int j = 0; j < SC_IT; j += 2) {
      const u64 a0 = run;
      run += v[j];
      const u64 a1 = run;
      run += v[j + 1];
      o[j / 2] = make_ulonglong2(a0, a1);
    }
  } else {
#pragma unroll
    for (int j = 0; j < SC_IT; ++j) {
      if (i0 + j < n) out[i0 + j] = run;
      run += v[j];
    }
  }
}
}  // namespace

size_t scan_temp_bytes(size_t n_max) {
  return al(((n_max + SC_TILE - 1) / SC_TILE + 1) * 8);
}

void exclusive_scan_u32_to_u64(rvp_context *ctx, const u32 *in, u64 *out, size_t n_max,
                               const u64 *n_dev, void *temp) {
  exclusive_scan_u32_to_u64_batch(ctx, in, 0, out, 0, 1, n_max, n_dev, temp);
}

void exclusive_scan_u32_to_u64_batch(rvp_context *ctx, const u32 *in, size_t in_stride, u64 *out,
                                     size_t out_stride, int batch, size_t n_max,
                                     const u64 *n_dev, void *temp) {
  const size_t nt = (n_max + SC_TILE - 1) / SC_TILE;
  const size_t ts_stride = scan_temp_bytes(n_max) / 8;
  u64 *tsum = static_cast<u64 *>(temp);
  const dim3 g((unsigned)(nt > 0 ? nt : 1), (unsigned)batch);
  k_scan_tiles<<<g, SC_TH, 0, ctx->stream>>>(in, n_max, n_dev, tsum, in_stride, ts_stride);
  RVP_LAUNCH_CHECK(ctx);
  k_scan_sums<<<(unsigned)batch, 1024, 0, ctx->stream>>>(tsum, nt, n_max, n_dev, out, out_stride,
                                                        ts_stride);
  RVP_LAUNCH_CHECK(ctx);
  k_scan_apply<<<g, SC_TH, 0, ctx->stream>>>(in, n_max, n_dev, tsum, out, in_stride, out_stride,
                                             ts_stride);
  RVP_LAUNCH_CHECK(ctx);
}

}  // namespace rvp
