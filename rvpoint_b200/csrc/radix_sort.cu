// Stable LSD radix sort of (u64 key, u32 value) pairs for sm_100a, one
// kernel per 8-bit digit (single-pass "onesweep" style).
//
// First one kernel counts all eight digits of every key (8 x 256 global
// counters, warp-aggregated with __match_any_sync). A digit is live unless
// one value holds all n keys; dead digits cost nothing, so a 64-bit key with
// 30 live bits costs 4 passes. Each pass then takes tiles of 4096 keys in
// the order its blocks start (a tile id from an atomic counter, so every
// tile a block waits for has started), ranks the tile's keys stably in
// registers and shared memory (per-warp __match_any_sync counts), publishes
// its per-digit counts, and finds the keys before it in earlier tiles by
// looking back over their published counts and prefixes (decoupled
// look-back; every wait is bounded, and a wait that runs out sets an error
// flag instead of hanging). The tile is reordered in shared memory and
// written out one digit run at a time (coalesced). The key count lives in
// device memory and nothing returns to the host, so a sort can sit in a
// graph.
#include "internal.cuh"

namespace rvp {

namespace {
constexpr int TH = 256;
constexpr int ITEMS = 16;
constexpr int TILE = TH * ITEMS;  // 4096 keys per tile
constexpr int WARPS = TH / 32;
constexpr int CHUNK = TILE / WARPS;  // 512 keys per warp, in order
// tile status word: flag in the top two bits, a count below
constexpr u32 ST_AGG = 1u << 30, ST_PRE = 2u << 30, ST_VAL = (1u << 30) - 1;
constexpr int SPIN_LIMIT = 1 << 21;  // look-back polls of one status word
__device__ int g_sort_timeout;       // a look-back wait ran out (results wrong)

__host__ __device__ inline size_t tiles_for(size_t n) { return (n + TILE - 1) / TILE; }

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

// the eight digit histograms of all keys (ghist[pass * 256 + digit])
__global__ __launch_bounds__(TH) void k_digit_hist(const u64 *__restrict__ keys, size_t n_max,
                                                   const u64 *__restrict__ n_dev, u32 *ghist) {
  __shared__ u32 h[8][256];
  for (int j = threadIdx.x; j < 8 * 256; j += TH) (&h[0][0])[j] = 0;
  __syncthreads();
  const size_t n = n_dev ? *n_dev : n_max;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1;
  const size_t stride = (size_t)gridDim.x * TH;
  for (size_t i0 = (size_t)blockIdx.x * TH + (threadIdx.x & ~31); i0 < n; i0 += stride) {
    const size_t i = i0 + lane;
    const bool valid = i < n;
    const unsigned vm = __ballot_sync(0xffffffffu, valid);
    if (valid) {
      const u64 k = keys[i];
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const unsigned d = (unsigned)((k >> (8 * p)) & 0xFF);
        const unsigned m = __match_any_sync(vm, d);
        if ((m & lt) == 0) atomicAdd(&h[p][d], __popc(m));
      }
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < 8 * 256; j += TH) {
    const u32 c = (&h[0][0])[j];
    if (c) atomicAdd(&ghist[j], c);
  }
}

// pass p is live unless one digit value holds all n keys (all 256 threads
// of the block call it)
__device__ __forceinline__ bool pass_live_dev(const u32 *ghist, int pass, u32 n) {
  return !__syncthreads_or(ghist[pass * 256 + threadIdx.x] == n);
}

__global__ __launch_bounds__(TH) void k_onesweep(u64 *k0, u32 *v0, u64 *k1, u32 *v1,
                                                size_t n_max, const u64 *n_dev,
                                                const u32 *ghist, int pass, u32 *status,
                                                u32 *tile_counter) {
  const size_t n = n_dev ? *n_dev : n_max;
  if (n == 0) return;
  // live passes below this one decide which buffer holds its input
  int src = 0;
  for (int q = 0; q < pass; ++q) src ^= pass_live_dev(ghist, q, (u32)n) ? 1 : 0;
  if (!pass_live_dev(ghist, pass, (u32)n)) return;
  const u64 *kin = src ? k1 : k0;
  const u32 *vin = src ? v1 : v0;
  u64 *kout = src ? k0 : k1;
  u32 *vout = src ? v0 : v1;

  extern __shared__ __align__(16) unsigned char smem[];
  u64 *skeys = reinterpret_cast<u64 *>(smem);          // TILE
  u32 *svals = reinterpret_cast<u32 *>(skeys + TILE);  // TILE
  u32 *wh = svals + TILE;                              // WARPS * 256
  u32 *dstart = wh + WARPS * 256;                      // 256: tile-local digit starts
  u32 *gbase = dstart + 256;                           // 256: global start of the tile's run
  __shared__ u32 s_tile;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
  for (int j = tid; j < WARPS * 256; j += TH) wh[j] = 0;
  __syncthreads();
  const u32 tile = s_tile;
  const size_t base = (size_t)tile * TILE;
  if (base >= n) return;  // (block-uniform)
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
  // stable ranks inside each warp's chunk, counts per warp and digit
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
  // thread tid = digit: exclusive over warps; the tile's count of the digit
  u32 cnt = 0;
  for (int q = 0; q < WARPS; ++q) {
    const u32 c = wh[q * 256 + tid];
    wh[q * 256 + tid] = cnt;
    cnt += c;
  }
  // publish this tile's count, then look back for the keys of this digit in
  // earlier tiles
  volatile u32 *st = status;
  st[(size_t)tile * 256 + tid] = (tile == 0 ? ST_PRE : ST_AGG) | cnt;
  u32 before = 0;
  if (tile > 0) {
    long long t = (long long)tile - 1;
    int spins = 0;
    while (t >= 0) {
      const u32 v = st[(size_t)t * 256 + tid];
      if (v & ST_PRE) {
        before += v & ST_VAL;
        break;
      }
      if (v & ST_AGG) {
        before += v & ST_VAL;
        --t;
        continue;
      }
      if (++spins > SPIN_LIMIT) {  // never published: give up, flag it
        g_sort_timeout = 1;
        break;
      }
      __nanosleep(64);
    }
    st[(size_t)tile * 256 + tid] = ST_PRE | (before + cnt);
  }
  // global start of this tile's run of the digit: keys of smaller digits
  // (exclusive prefix of the digit counts) plus this digit's earlier keys
  {
    const u32 t_all = ghist[pass * 256 + tid];
    dstart[tid] = t_all;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
      const u32 v = tid >= off ? dstart[tid - off] : 0;
      __syncthreads();
      dstart[tid] += v;
      __syncthreads();
    }
    gbase[tid] = dstart[tid] - t_all + before;
    __syncthreads();
    // tile-local digit starts: exclusive prefix of the tile's counts
    dstart[tid] = cnt;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
      const u32 v = tid >= off ? dstart[tid - off] : 0;
      __syncthreads();
      dstart[tid] += v;
      __syncthreads();
    }
    dstart[tid] -= cnt;
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
  const size_t c_all = (n - base) < (size_t)TILE ? (n - base) : (size_t)TILE;
  for (int j = tid; j < (int)c_all; j += TH) {
    const u64 k = skeys[j];
    const unsigned d = (unsigned)((k >> shift) & 0xFF);
    const size_t dst = (size_t)gbase[d] + (size_t)(j - (int)dstart[d]);
    kout[dst] = k;
    vout[dst] = svals[j];
  }
}

__global__ void k_copy_back(u64 *k0, u32 *v0, const u64 *k1, const u32 *v1, size_t n_max,
                            const u64 *n_dev, const u32 *ghist) {
  const size_t n = n_dev ? *n_dev : n_max;
  if (n == 0) return;
  int c = 0;
  for (int q = 0; q < 8; ++q) c ^= pass_live_dev(ghist, q, (u32)n) ? 1 : 0;
  if (c == 0) return;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    k0[i] = k1[i];
    v0[i] = v1[i];
  }
}

constexpr size_t kSweepSmem =
    (size_t)TILE * 8 + (size_t)TILE * 4 + (size_t)WARPS * 256 * 4 + 256 * 4 * 2;
}  // namespace

size_t sort_temp_bytes(size_t n_max) {
  const size_t T = tiles_for(n_max) > 0 ? tiles_for(n_max) : 1;
  return al(n_max * 8) + al(n_max * 4) + al(256 * T * 4) + al(8 * 256 * 4) + al(64);
}

void sort_temp_carve(SortTemp &t, void *base, size_t n_max) {
  const size_t T = tiles_for(n_max) > 0 ? tiles_for(n_max) : 1;
  char *p = static_cast<char *>(base);
  t.keys_alt = reinterpret_cast<u64 *>(p); p += al(n_max * 8);
  t.vals_alt = reinterpret_cast<u32 *>(p); p += al(n_max * 4);
  t.tile_hist = reinterpret_cast<u32 *>(p); p += al(256 * T * 4);   // tile status words
  t.global_hist = reinterpret_cast<u32 *>(p); p += al(8 * 256 * 4);  // digit counts
  t.pass_info = reinterpret_cast<int *>(p);                          // 8 tile counters
}

void radix_sort_pairs(rvp_context *ctx, u64 *keys, u32 *vals, size_t n_max,
                      const u64 *n_dev, const SortTemp &t) {
  if (n_max == 0) return;
  RVP_REQUIRE(n_max < ST_VAL, "radix sort: more than 2^30 - 1 keys");
  static bool attr_set[64] = {false};
  int dev = ctx->device;
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    RVP_CUDA_TRY(cudaFuncSetAttribute(k_onesweep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kSweepSmem));
    attr_set[dev] = true;
  }
  const size_t T = tiles_for(n_max);
  u32 *counters = reinterpret_cast<u32 *>(t.pass_info);
  RVP_CUDA_TRY(cudaMemsetAsync(t.global_hist, 0, 8 * 256 * 4, ctx->stream));
  RVP_CUDA_TRY(cudaMemsetAsync(counters, 0, 8 * 4, ctx->stream));
  k_digit_hist<<<grid_for(n_max, TH, ctx->num_sms * 4), TH, 0, ctx->stream>>>(keys, n_max, n_dev,
                                                                              t.global_hist);
  RVP_LAUNCH_CHECK(ctx);
  for (int pass = 0; pass < 8; ++pass) {
    RVP_CUDA_TRY(cudaMemsetAsync(t.tile_hist, 0, T * 256 * 4, ctx->stream));
    k_onesweep<<<(unsigned)T, TH, kSweepSmem, ctx->stream>>>(keys, vals, t.keys_alt, t.vals_alt,
                                                             n_max, n_dev, t.global_hist, pass,
                                                             t.tile_hist, counters + pass);
    RVP_LAUNCH_CHECK(ctx);
  }
  k_copy_back<<<grid_for(n_max, 256, ctx->num_sms * 8), 256, 0, ctx->stream>>>(
      keys, vals, t.keys_alt, t.vals_alt, n_max, n_dev, t.global_hist);
  RVP_LAUNCH_CHECK(ctx);
}

bool sort_timed_out(rvp_context *ctx) {
  int v = 0;
  RVP_CUDA_TRY(cudaMemcpyFromSymbolAsync(&v, g_sort_timeout, sizeof(int), 0,
                                         cudaMemcpyDeviceToHost, ctx->stream));
  RVP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return v != 0;
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

__global__ __launch_bounds__(SC_TH) void k_scan_tiles(const u32 *in, size_t n_max,
                                                      const u64 *n_dev, u64 *tsum) {
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
                            u64 *out) {
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
                                                      u64 *out) {
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
  const size_t nt = (n_max + SC_TILE - 1) / SC_TILE;
  u64 *tsum = static_cast<u64 *>(temp);
  const unsigned g = (unsigned)(nt > 0 ? nt : 1);
  k_scan_tiles<<<g, SC_TH, 0, ctx->stream>>>(in, n_max, n_dev, tsum);
  RVP_LAUNCH_CHECK(ctx);
  k_scan_sums<<<1, 1024, 0, ctx->stream>>>(tsum, nt, n_max, n_dev, out);
  RVP_LAUNCH_CHECK(ctx);
  k_scan_apply<<<g, SC_TH, 0, ctx->stream>>>(in, n_max, n_dev, tsum, out);
  RVP_LAUNCH_CHECK(ctx);
}

}  // namespace rvp
