// RANSAC plane fitting (segmentation/ransac_plane.cpp:18-111) for many
// frames, one thread block per frame; optionally with hypotheses drawn by
// per-point weight (the learned proposal) instead of the rand() stream.
//
// The reference draws three rand() % n indices per iteration after
// srand(0); the raw rand() stream is the same for every call, so it is an
// input table here (rand_dev, 3 * max_iters values) and i = r % n is taken
// on the device. Hypotheses are evaluated 32 at a time: each warp walks the
// frame's points, every lane tests its point against hypothesis h and
// __ballot_sync/__popc turns the 32 tests into one count that lane h
// accumulates. Thread 0 then replays the reference's sequential logic
// (strictly greater count wins, adaptive k_iters with p = 0.99 in double),
// so best count, model and the number of executed iterations are the
// reference's, and the loop stops as early as the reference's does.
#include <cooperative_groups.h>
#include <float.h>

#include <atomic>
#include <math.h>

#include "internal.cuh"

namespace rvp {
namespace cg = cooperative_groups;

namespace {
constexpr int HB = 32;        // hypotheses per batch
constexpr int R_THREADS = 512;
constexpr int R_PTS = 4;      // points per lane per pass (amortises the hypothesis loads)
constexpr int PE_KEEP = HB;   // preemptive rounds: hypotheses counted exactly per round

// compute_plane_coefficients (ransac_plane.cpp:18-50), exact op order.
__device__ __forceinline__ bool plane_coeffs(float x1, float y1, float z1, float x2, float y2,
                                             float z2, float x3, float y3, float z3, float col,
                                             float4 &m) {
  const float v1x = fsub(x2, x1), v1y = fsub(y2, y1), v1z = fsub(z2, z1);
  const float v2x = fsub(x3, x1), v2y = fsub(y3, y1), v2z = fsub(z3, z1);
  float a = fsub(fmul(v1y, v2z), fmul(v1z, v2y));
  float b = fsub(fmul(v1z, v2x), fmul(v1x, v2z));
  float c = fsub(fmul(v1x, v2y), fmul(v1y, v2x));
  const float norm = __fsqrt_rn(fadd(fadd(fmul(a, a), fmul(b, b)), fmul(c, c)));
  if (norm < col) return false;
  a = fdiv(a, norm);
  b = fdiv(b, norm);
  c = fdiv(c, norm);
  const float d = -fadd(fadd(fmul(a, x1), fmul(b, y1)), fmul(c, z1));
  m = make_float4(a, b, c, d);
  return true;
}

// |a*x + b*y + c*z + d| <= t  (ransac_plane.cpp:80-87)
__device__ __forceinline__ bool is_inlier(const float4 &m, float x, float y, float z, float t) {
  return fabsf(fadd(fadd(fadd(fmul(m.x, x), fmul(m.y, y)), fmul(m.z, z)), m.w)) <= t;
}

// The same test with fused multiply-adds, for the preemptive ranking on the
// candidates only: an estimate that orders hypotheses for the exact count,
// which alone decides the result
__device__ __forceinline__ bool is_inlier_fast(const float4 &m, float x, float y, float z,
                                               float t) {
  return fabsf(fmaf(m.x, x, fmaf(m.y, y, fmaf(m.z, z, m.w)))) <= t;
}

// One weighted draw: the candidate whose prefix-sum interval holds u * total,
// returned relative to the frame's first point (a0).
__device__ __forceinline__ u32 weighted_draw(const RansacSampler &smp, int f, int it, int k,
                                             int64_t a0, u32 n) {
  const int64_t c0 = smp.cand_offs[f], c1 = smp.cand_offs[f + 1];
  const double total = smp.cdf[c1 - 1];
  const u64 r = mix64(smp.seed ^ mix64(((u64)f << 34) ^ ((u64)it << 2) ^ (u64)k));
  const double u = (double)(r >> 11) * 0x1.0p-53 * total;
  int64_t lo = c0, hi = c1 - 1;  // first slot with cdf > u
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (smp.cdf[mid] > u) hi = mid; else lo = mid + 1;
  }
  const int64_t rel = (int64_t)smp.cand[lo] - a0;
  return rel >= 0 && rel < (int64_t)n ? (u32)rel : 0xFFFFFFFFu;  // outside the frame: no hypothesis
}

__global__ __launch_bounds__(R_THREADS) void k_ransac(
    const float *__restrict__ X, const float *__restrict__ Y, const float *__restrict__ Z,
    const int64_t *offs, const int *__restrict__ rnd, RansacParams prm, float *model_out,
    int32_t *best_out, int32_t *iters_out, int32_t *counts_all, bool eval_all,
    RansacSampler smp) {
  // a frame is a cluster of G blocks (G = 1 without a cluster launch): every
  // block builds the same hypotheses, counts its share of the points, and
  // reads the others' counts through distributed shared memory; every block
  // then replays the same decisions, so they stop together
  cg::cluster_group cl = cg::this_cluster();
  const u32 G = cl.num_blocks(), cr = cl.block_rank();
  const int f = blockIdx.x / G;
  const bool lead = cr == 0;  // writes the frame's outputs
  const int64_t a0 = offs[f];
  const u32 n = (u32)(offs[f + 1] - a0);
  const float *x = X + a0, *y = Y + a0, *z = Z + a0;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int NW = R_THREADS / 32;

  __shared__ float4 hyp[HB];
  __shared__ int hcode[HB];  // 0 valid, -1 repeated index, -2 collinear
  __shared__ u32 hcnt[HB];   // this block's partial counts
  __shared__ u32 htot[HB];   // the frame's counts
  __shared__ int s_best, s_kiters, s_stop, s_iters;
  __shared__ float4 s_model;

  const bool no_cand = smp.cdf && (smp.cand_offs[f + 1] - smp.cand_offs[f] < 3 ||
                                   !(smp.cdf[smp.cand_offs[f + 1] - 1] > 0.0));
  if (n < 3 || no_cand) {  // ransac_plane.cpp:59
    if (!lead) return;
    if (tid == 0) {
      model_out[4 * f + 0] = model_out[4 * f + 1] = model_out[4 * f + 2] = model_out[4 * f + 3] = 0;
      best_out[f] = 0;
      if (iters_out) iters_out[f] = 0;
    }
    if (counts_all)
      for (int it = tid; it < prm.max_iters; it += R_THREADS)
        counts_all[(size_t)f * prm.max_iters + it] = -3;
    return;
  }
  if (tid == 0) {
    s_best = 0;
    s_kiters = prm.max_iters;
    s_stop = 0;
    s_iters = prm.max_iters;
    s_model = make_float4(0, 0, 0, 0);
    if (smp.best_in) {
      s_best = smp.best_in[f];
      s_model = make_float4(smp.model_in[4 * f + 0], smp.model_in[4 * f + 1],
                            smp.model_in[4 * f + 2], smp.model_in[4 * f + 3]);
      if (smp.targets && s_best >= smp.targets[f]) {  // reached in an earlier round
        s_stop = 1;
        s_iters = 0;
      }
    }
  }
  __syncthreads();

  for (int base = 0; base < prm.max_iters; base += HB) {
    if (s_stop && !eval_all) break;
    if (tid < HB) {
      const int it = base + tid;
      float4 m = make_float4(__int_as_float(0x7fc00000), 0, 0, 0);  // NaN: never an inlier
      int code = -3;
      if (it < prm.max_iters && smp.models) {
        m = smp.models[(size_t)f * smp.n_models + it];
        code = isnan(m.x) ? -2 : 0;
      } else if (it < prm.max_iters) {
        u32 i1, i2, i3;
        if (smp.cdf) {
          i1 = weighted_draw(smp, f, it, 0, a0, n);
          i2 = weighted_draw(smp, f, it, 1, a0, n);
          i3 = weighted_draw(smp, f, it, 2, a0, n);
        } else {
          i1 = (u32)rnd[3 * it + 0] % n;
          i2 = (u32)rnd[3 * it + 1] % n;
          i3 = (u32)rnd[3 * it + 2] % n;
        }
        if (i1 == i2 || i1 == i3 || i2 == i3 || i1 >= n || i2 >= n || i3 >= n) {
          code = -1;
        } else if (!plane_coeffs(x[i1], y[i1], z[i1], x[i2], y[i2], z[i2], x[i3], y[i3], z[i3],
                                 prm.collinear, m)) {
          code = -2;
          m = make_float4(__int_as_float(0x7fc00000), 0, 0, 0);
        } else {
          code = 0;
        }
      }
      hyp[tid] = m;
      hcode[tid] = code;
      hcnt[tid] = 0;
    }
    __syncthreads();

    // hypotheses to count: all of a full batch, else only the valid ones
    // (given models past their end, or frames short of hypotheses, leave
    // empty slots whose counts nothing reads)
    const u32 vmask = __ballot_sync(0xffffffffu, hcode[lane] == 0);
    u32 acc = 0;  // lane h accumulates hypothesis h
    for (u32 p0 = (cr * NW + (u32)wid) * 32 * R_PTS; p0 < n; p0 += G * NW * 32 * R_PTS) {
      float px[R_PTS], py[R_PTS], pz[R_PTS];
      bool pv[R_PTS];
#pragma unroll
      for (int r = 0; r < R_PTS; ++r) {
        const u32 i = p0 + r * 32 + lane;
        pv[r] = i < n;
        px[r] = pv[r] ? __ldg(&x[i]) : 0.0f;
        py[r] = pv[r] ? __ldg(&y[i]) : 0.0f;
        pz[r] = pv[r] ? __ldg(&z[i]) : 0.0f;
      }
      auto count = [&](int h) {
        const float4 m = hyp[h];
        u32 c = 0;
#pragma unroll
        for (int r = 0; r < R_PTS; ++r)
          c += __popc(__ballot_sync(0xffffffffu, pv[r] && is_inlier(m, px[r], py[r], pz[r], prm.thresh)));
        if (lane == h) acc += c;
      };
      if (vmask == 0xffffffffu) {
#pragma unroll 4
        for (int h = 0; h < HB; ++h) count(h);
      } else {
        for (u32 b = vmask; b; b &= b - 1) count(__ffs(b) - 1);
      }
    }
    atomicAdd(&hcnt[lane], acc);
    cl.sync();  // every block's partial counts of this batch are complete
    if (tid < HB) {
      u32 t = 0;
      for (u32 r = 0; r < G; ++r) t += cl.map_shared_rank(hcnt, r)[tid];
      htot[tid] = t;
    }
    cl.sync();  // no block resets its counts while another still reads them

    if (tid == 0) {
      // replay ransac_plane.cpp:67-107 for this batch, in order
      for (int h = 0; h < HB && !s_stop; ++h) {
        const int it = base + h;
        if (it >= s_kiters || it >= prm.max_iters) {
          s_stop = 1;
          s_iters = it;
          break;
        }
        if (hcode[h] != 0) continue;
        const int cur = (int)htot[h];
        if (cur > s_best && smp.targets) {
          s_best = cur;
          s_model = hyp[h];
          if (cur >= smp.targets[f]) {
            s_stop = 1;
            s_iters = it + 1;
          }
        } else if (cur > s_best) {
          s_best = cur;
          s_model = hyp[h];
          const double w = (double)cur / (double)n;
          double p_no = 1.0 - pow(w, 3.0);
          p_no = fmax(DBL_EPSILON, p_no);
          p_no = fmin(1.0 - DBL_EPSILON, p_no);
          const double log_no = log(p_no);
          if (fabs(log_no) > 1e-7) {
            const int dyn = (int)ceil(prm.log_p / log_no);
            if (dyn > 0 && dyn < s_kiters) s_kiters = dyn;
          }
        }
      }
      if (!s_stop && base + HB >= prm.max_iters) {
        s_stop = 1;
        s_iters = prm.max_iters;
      }
    }
    if (lead && counts_all && tid < HB && base + tid < prm.max_iters)
      counts_all[(size_t)f * prm.max_iters + base + tid] =
          hcode[tid] == 0 ? (int32_t)htot[tid] : hcode[tid];
    __syncthreads();
  }
  if (!lead) return;
  if (counts_all && !eval_all) {
    // hypotheses past the early stop were not evaluated
    const int done = ((s_iters + HB - 1) / HB) * HB;
    for (int it = done + tid; it < prm.max_iters; it += R_THREADS)
      counts_all[(size_t)f * prm.max_iters + it] = -3;
  }
  if (tid == 0) {
    model_out[4 * f + 0] = s_model.x;
    model_out[4 * f + 1] = s_model.y;
    model_out[4 * f + 2] = s_model.z;
    model_out[4 * f + 3] = s_model.w;
    best_out[f] = s_best;
    if (iters_out) iters_out[f] = s_iters;
  }
}

// Preemptive round of the weighted proposal, in two kernels. k_preempt_count:
// block (frame, slice) draws the slice's share of the round's `draws`
// hypotheses from the frame's candidates by weight and counts each one's
// inliers among the candidates only (they sit in shared memory); a round
// with few open frames splits each frame over several slices (blocks).
// k_preempt_rank: per frame, the PE_KEEP best (count, then draw order) for
// the exact count over all points. The candidate counts are an estimate that
// orders hypotheses (fused multiply-adds); the exact count alone decides the
// result. Frames that already reached their target write empty slots.
constexpr int PE_THREADS = 1024;
constexpr int PE_MAXC = 2048;
constexpr int PE_MAXH = 512;
constexpr int PE_FIRST = 4;   // with targets: exact counts of the best-ranked few first
constexpr int PE_SLICES = 8;  // blocks per frame in the rounds after the first
constexpr int PE_GROWTH = 2;  // later rounds: this many times the draws and the exact counts
constexpr int PE_HALL = PE_MAXH * PE_GROWTH;  // hypotheses of a round, per frame (stride)
constexpr int PE_KALL = PE_KEEP * PE_GROWTH;  // exactly counted hypotheses of a round (stride)

__device__ __forceinline__ bool pe_skip(const RansacSampler &smp, const int64_t *offs,
                                        const int32_t *best_now, int f) {
  const u32 n = (u32)(offs[f + 1] - offs[f]);
  const int64_t c0 = smp.cand_offs[f], c1 = smp.cand_offs[f + 1];
  const int m = (int)(c1 - c0);
  const bool done = smp.targets && best_now && best_now[f] >= smp.targets[f];
  return done || n < 3 || m < 3 || m > PE_MAXC || !(smp.cdf[c1 - 1] > 0.0);
}

__global__ __launch_bounds__(PE_THREADS) void k_preempt_count(
    const float *__restrict__ X, const float *__restrict__ Y, const float *__restrict__ Z,
    const int64_t *offs, RansacSampler smp, int draws, int slices, int it_base, RansacParams prm,
    const int32_t *best_now, float4 *hyp_out, int *cnt_out) {
  __shared__ float4 P[PE_MAXC];
  __shared__ float4 hyp[PE_MAXH];
  __shared__ int hcnt[PE_MAXH];
  const int f = blockIdx.x / slices, sl = blockIdx.x % slices;
  const int dg = (draws + slices - 1) / slices, h0 = sl * dg;
  const int nh = min(draws, h0 + dg) - h0;
  if (nh <= 0 || pe_skip(smp, offs, best_now, f)) return;
  const int64_t a0 = offs[f];
  const u32 n = (u32)(offs[f + 1] - a0);
  const int64_t c0 = smp.cand_offs[f];
  const int m = (int)(smp.cand_offs[f + 1] - c0);
  const float4 none = make_float4(__int_as_float(0x7fc00000), 0, 0, 0);
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    const u32 g = smp.cand[c0 + j];
    P[j] = make_float4(X[g], Y[g], Z[g], 0.0f);
  }
  const float *x = X + a0, *y = Y + a0, *z = Z + a0;
  for (int h = threadIdx.x; h < nh; h += blockDim.x) {
    const int it = it_base + h0 + h;
    const u32 i1 = weighted_draw(smp, f, it, 0, a0, n);
    const u32 i2 = weighted_draw(smp, f, it, 1, a0, n);
    const u32 i3 = weighted_draw(smp, f, it, 2, a0, n);
    float4 mdl = none;
    if (!(i1 == i2 || i1 == i3 || i2 == i3 || i1 >= n || i2 >= n || i3 >= n) &&
        !plane_coeffs(x[i1], y[i1], z[i1], x[i2], y[i2], z[i2], x[i3], y[i3], z[i3],
                      prm.collinear, mdl))
      mdl = none;
    hyp[h] = mdl;
    hcnt[h] = isnan(mdl.x) ? -1 : 0;
  }
  __syncthreads();
  // S threads per hypothesis, each over every S-th candidate (a warp shares
  // the slice of candidates, so its lanes read the same candidate: a
  // shared-memory broadcast); integer counts add up the same in any order
  const int S = max(1, (int)blockDim.x / nh);
  const int slots = nh * S;
  for (int u = threadIdx.x; u < slots; u += blockDim.x) {
    const int h = u % nh, cs = u / nh;
    const float4 mdl = hyp[h];
    if (isnan(mdl.x)) continue;
    int c = 0;
    for (int j = cs; j < m; j += S)
      c += is_inlier_fast(mdl, P[j].x, P[j].y, P[j].z, prm.thresh) ? 1 : 0;
    if (c) atomicAdd(&hcnt[h], c);
  }
  __syncthreads();
  for (int h = threadIdx.x; h < nh; h += blockDim.x) {
    hyp_out[(size_t)f * PE_HALL + h0 + h] = hyp[h];
    cnt_out[(size_t)f * PE_HALL + h0 + h] = hcnt[h];
  }
}

// rank = #(greater count) + #(equal count, earlier draw). Only the
// hypotheses at or above the keep-th largest count can rank below keep: a
// histogram of the counts finds that count first.
constexpr int PR_THREADS = 512;
__global__ __launch_bounds__(PR_THREADS) void k_preempt_rank(
    const int64_t *offs, RansacSampler smp, int draws, int keep, const int32_t *best_now,
    const float4 *hyp_in, const int *cnt_in, float4 *out) {
  __shared__ int hcnt[PE_HALL];
  __shared__ int hist[PE_MAXC / 2 + 2];  // counts in pairs: (count + 1) >> 1
  __shared__ int s_thr;
  const int f = blockIdx.x;
  float4 *o = out + (size_t)f * PE_KALL;
  const float4 none = make_float4(__int_as_float(0x7fc00000), 0, 0, 0);
  for (int t = threadIdx.x; t < PE_KALL; t += blockDim.x) o[t] = none;
  if (pe_skip(smp, offs, best_now, f)) return;
  const int m = (int)(smp.cand_offs[f + 1] - smp.cand_offs[f]);
  const int nbins = ((m + 1) >> 1) + 1;
  for (int h = threadIdx.x; h < draws; h += blockDim.x) hcnt[h] = cnt_in[(size_t)f * PE_HALL + h];
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  for (int h = threadIdx.x; h < draws; h += blockDim.x) atomicAdd(&hist[(hcnt[h] + 1) >> 1], 1);
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    int above = 0, thr = 0;  // thr: histogram bin; 0 keeps every hypothesis
    for (int top = nbins - 1; top >= 0; top -= 32) {
      const int bb = top - lane;
      int sfx = bb >= 0 ? hist[bb] : 0;  // becomes the sum of bins top .. bb
#pragma unroll
      for (int sh = 1; sh < 32; sh <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, sfx, sh);
        if (lane >= sh) sfx += t;
      }
      const unsigned hit = __ballot_sync(0xffffffffu, bb >= 0 && above + sfx >= keep);
      if (hit) {
        thr = top - (__ffs(hit) - 1);
        break;
      }
      above += __shfl_sync(0xffffffffu, sfx, 31);
    }
    if (lane == 0) s_thr = thr;
  }
  __syncthreads();
  const int cthr = 2 * s_thr - 1;  // the lowest count of bin s_thr
  for (int h = threadIdx.x; h < draws; h += blockDim.x) {
    const int c = hcnt[h];
    if (c < cthr) continue;
    int rank = 0;
    for (int g = 0; g < draws; ++g) {
      const int cg = hcnt[g];
      rank += (cg > c || (cg == c && g < h)) ? 1 : 0;
    }
    if (rank < keep) o[rank] = c >= 0 ? hyp_in[(size_t)f * PE_HALL + h] : none;
  }
}

// draws_run of the frames that stop after this round (reached their
// target, or the last round); open counts the others
__global__ void k_preempt_done(const int32_t *best, const int32_t *targets, int n_frames,
                               int drawn, bool last, int32_t *draws_run, int *open) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n_frames; f += gridDim.x * blockDim.x) {
    if (draws_run[f] >= 0) continue;
    if (last || (targets && best[f] >= targets[f])) draws_run[f] = drawn;
    else atomicAdd(open, 1);
  }
}

__global__ void k_fill_i32(int32_t *p, int n, int v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// extract_plane_inliers_outliers_rvv, scalar branch (ransac_plane.cpp:373-381):
// inlier iff -t <= a*x + b*y + c*z + d <= t.
__global__ void k_plane_flags(const float *x, const float *y, const float *z, size_t n,
                              const float *model, float t, u32 *flags) {
  const float4 m = make_float4(model[0], model[1], model[2], model[3]);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const float d = fadd(fadd(fadd(fmul(m.x, x[i]), fmul(m.y, y[i])), fmul(m.z, z[i])), m.w);
    flags[i] = (d >= -t && d <= t) ? 1u : 0u;
  }
}

__global__ void k_plane_scatter(const float *x, const float *y, const float *z, size_t n,
                                const u32 *flags, const u64 *pos, float *in_aos, float *out_aos,
                                u64 *counts) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const u64 pi = pos[i];
    float *dst = nullptr;
    if (flags[i]) {
      if (in_aos) dst = in_aos + 3 * pi;
    } else {
      if (out_aos) dst = out_aos + 3 * (i - pi);
    }
    if (dst) {
      dst[0] = x[i];
      dst[1] = y[i];
      dst[2] = z[i];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counts[0] = pos[n];
    counts[1] = n - pos[n];
  }
}

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }
}  // namespace

void ransac_frames(rvp_context *ctx, const float *x, const float *y, const float *z,
                   const int64_t *offs, int n_frames, const int *rand_dev, const RansacParams &p,
                   float *model, int32_t *best, int32_t *iters_run, int32_t *counts_all,
                   bool eval_all, const RansacSampler &smp, int cluster) {
  if (n_frames <= 0) return;
  const int want = cluster < 1 ? 1 : (cluster > 8 ? 8 : cluster);
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  cfg.blockDim = dim3(R_THREADS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = ctx->stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  // the largest cluster (<= want) the device holds, found once per device
  // and request, before any stream capture that launches this kernel
  static std::atomic<int> fitted[64][9];
  const int dev = ctx->device >= 0 && ctx->device < 64 ? ctx->device : 0;
  int G = fitted[dev][want].load(std::memory_order_relaxed);
  for (G = G ? G : want; G > 1 && !fitted[dev][want].load(std::memory_order_relaxed); G >>= 1) {
    cfg.gridDim = dim3((unsigned)n_frames * G);
    attr[0].val.clusterDim.x = G;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int active = 0;
    if (cudaOccupancyMaxActiveClusters(&active, k_ransac, &cfg) == cudaSuccess && active > 0) break;
    cudaGetLastError();
  }
  if (G < 1) G = 1;
  fitted[dev][want].store(G, std::memory_order_relaxed);
  cfg.gridDim = dim3((unsigned)n_frames * G);
  attr[0].val.clusterDim.x = G;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = G > 1 ? 1 : 0;
  RVP_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_ransac, x, y, z, offs, rand_dev, p, model, best,
                                  iters_run, counts_all, eval_all, smp));
  ::rvp::count_launch(ctx);
}

void ransac_preemptive(rvp_context *ctx, const float *x, const float *y, const float *z,
                       const int64_t *offs, int n_frames, const RansacSampler &smp0, int draws,
                       int max_rounds, const RansacParams &p, float *model, int32_t *best,
                       int32_t *draws_run, void *scratch) {
  if (n_frames <= 0) return;
  RVP_REQUIRE(draws >= 1 && draws <= PE_MAXH, "draws per round must be in [1, 512]");
  char *sp = static_cast<char *>(scratch);
  float4 *models = reinterpret_cast<float4 *>(sp);  // a round's best, PE_KALL per frame
  sp += al((size_t)n_frames * PE_KALL * 16);
  int *open = reinterpret_cast<int *>(sp);
  int32_t *dummy_iters = reinterpret_cast<int32_t *>(sp + 256);
  sp += 256 + al((size_t)n_frames * 4);
  float4 *hyp_all = reinterpret_cast<float4 *>(sp);  // a round's hypotheses, PE_HALL per frame
  int *cnt_all = reinterpret_cast<int *>(sp + al((size_t)n_frames * PE_HALL * 16));
  cudaStream_t st = ctx->stream;
  k_fill_i32<<<grid_for(n_frames, 256, 64), 256, 0, st>>>(draws_run, n_frames, -1);
  RVP_LAUNCH_CHECK(ctx);
  int it_base = 0;
  for (int r = 0; r < max_rounds; ++r) {
    // the first round holds every frame; later ones only the frames still
    // short of their target: they draw PE_GROWTH times as many hypotheses
    // and count PE_GROWTH times as many exactly (the same share), each frame
    // spread over PE_SLICES blocks
    const int grow = r == 0 ? 1 : PE_GROWTH;
    const int draws_r = draws * grow, keep_r = PE_KEEP * grow;
    const int slices = r == 0 ? 1 : PE_SLICES;
    k_preempt_count<<<(unsigned)n_frames * slices, PE_THREADS, 0, st>>>(
        x, y, z, offs, smp0, draws_r, slices, it_base, p, r > 0 ? best : nullptr, hyp_all,
        cnt_all);
    RVP_LAUNCH_CHECK(ctx);
    k_preempt_rank<<<n_frames, PR_THREADS, 0, st>>>(offs, smp0, draws_r, keep_r,
                                                    r > 0 ? best : nullptr, hyp_all, cnt_all,
                                                    models);
    RVP_LAUNCH_CHECK(ctx);
    it_base += draws_r;
    RansacSampler sm = smp0;
    sm.models = models;
    sm.n_models = PE_KALL;
    sm.best_in = r > 0 ? best : nullptr;
    sm.model_in = r > 0 ? model : nullptr;
    RansacParams pe = p;
    if (smp0.targets && r == 0) {
      // the best-ranked PE_FIRST first: most frames reach their target
      // there; the others go on with the rest, in the same rank order (so
      // the result is the single pass's). Later rounds hold the frames the
      // first could not finish, which rarely stop within the first few.
      pe.max_iters = PE_FIRST;  // a light pass over every frame: one block per frame
      ransac_frames(ctx, x, y, z, offs, n_frames, nullptr, pe, model, best, dummy_iters, nullptr,
                    false, sm, 1);
      sm.models = models + PE_FIRST;
      sm.best_in = best;
      sm.model_in = model;
      pe.max_iters = keep_r - PE_FIRST;
      ransac_frames(ctx, x, y, z, offs, n_frames, nullptr, pe, model, best, dummy_iters, nullptr,
                    false, sm, 8);
    } else {
      pe.max_iters = keep_r;
      ransac_frames(ctx, x, y, z, offs, n_frames, nullptr, pe, model, best, dummy_iters, nullptr,
                    false, sm, 8);
    }
    RVP_CUDA_TRY(cudaMemsetAsync(open, 0, 4, st));
    k_preempt_done<<<grid_for(n_frames, 256, 64), 256, 0, st>>>(
        best, smp0.targets, n_frames, it_base, r + 1 == max_rounds, draws_run, open);
    RVP_LAUNCH_CHECK(ctx);
    if (smp0.targets) {
      int h_open = 0;
      RVP_CUDA_TRY(cudaMemcpyAsync(&h_open, open, 4, cudaMemcpyDeviceToHost, st));
      RVP_CUDA_TRY(cudaStreamSynchronize(st));
      if (h_open == 0) return;
    }
  }
}

size_t preemptive_temp_bytes(int n_frames) {
  return al((size_t)n_frames * PE_KALL * 16) + 256 + al((size_t)n_frames * 4) +
         al((size_t)n_frames * PE_HALL * 16) + al((size_t)n_frames * PE_HALL * 4);
}

size_t extract_temp_bytes(size_t n) {
  return al(n * 4) + al((n + 1) * 8) + scan_temp_bytes(n);
}

void extract_plane_run(rvp_context *ctx, const float *x, const float *y, const float *z, size_t n,
                       const float *model_dev, float thresh, float *in_aos, float *out_aos,
                       u64 *counts_dev, void *temp) {
  char *p = static_cast<char *>(temp);
  u32 *flags = reinterpret_cast<u32 *>(p); p += al(n * 4);
  u64 *pos = reinterpret_cast<u64 *>(p); p += al((n + 1) * 8);
  const unsigned g = grid_for(n, 256, ctx->num_sms * 16);
  k_plane_flags<<<g, 256, 0, ctx->stream>>>(x, y, z, n, model_dev, thresh, flags);
  RVP_LAUNCH_CHECK(ctx);
  exclusive_scan_u32_to_u64(ctx, flags, pos, n, nullptr, p);
  k_plane_scatter<<<g, 256, 0, ctx->stream>>>(x, y, z, n, flags, pos, in_aos, out_aos, counts_dev);
  RVP_LAUNCH_CHECK(ctx);
}

}  // namespace rvp
