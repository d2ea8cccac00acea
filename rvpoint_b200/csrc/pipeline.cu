// Batched frames: the chain tools/pipeline_export.cpp:351-498 runs per frame
// (voxel_grid_downsamp_rvv_v2 -> sor_rvv -> normal_estimation_sc ->
// ransac_plane_rvv), here for many frames of uneven size in one sequence of
// kernels. Frame boundaries and every intermediate size stay in device memory
// (offset arrays), kernels are sized by the batch's point capacity and read
// the live counts on the device, so the whole run can be captured once in a
// CUDA graph and replayed.
//
//   voxel      one sort over (frame, voxel) keys for the whole batch
//   grid       one sort + table over (frame, cell) keys of the voxel points
//   SOR kNN    exact k+1 nearest per voxel point (ring / tight window /
//              brute force fallback), mean distance, per-frame sequential
//              statistics, ordered compaction
//   normals    the removed points are flagged in the same grid, the k+1
//              nearest kept points of every kept point give the covariance
//   RANSAC     one block per frame over the kept points
#include <math.h>

#include <algorithm>
#include <new>

#include "internal.cuh"

using rvp::u32;
using rvp::u64;

struct rvp_pipeline {
  rvp_context *ctx = nullptr;
  rvp_pipeline_config cfg{};
  size_t max_points = 0;
  int max_frames = 0;
  float cell = 0.0f;
  float rfac = 0.9f;
  int lane_levels = 0;  // chain levels of the per-lane kNN kernels (0: all)
  int grid_base = 2;    // the grid is sorted by cells of cell / 2^grid_base
  rvp::VoxelWork vw;
  rvp::Grid grid;
  rvp::DevBuf in_x, in_y, in_z, in_offs;
  rvp::DevBuf vox_aos, vox_x, vox_y, vox_z, vox_offs, vox_frame;
  rvp::DevBuf sor_list, knn_counts, mean, keep, sor_tmp;
  rvp::DevBuf sor_aos, sor_x, sor_y, sor_z, sor_offs, sor_frame, sor_src;
  rvp::DevBuf nrm_pairs, nrm_counts, nx, ny, nz;
  rvp::DevBuf r_model, r_best, r_iters, r_rand;
  rvp::DevBuf stats;  // 20 kNN path counters (diagnostics)
  rvp::DevBuf routed; // SOR queries of the cooperative and the adaptive kNN kernels
  rvp::DevBuf hard;   // queries the tile kernel could not certify (+ counter)
  rvp::DevBuf qlevel; // per grid point: level at which its kNN is still open
  rvp::DevBuf qtau;   // per grid point: K-th distance bound handed to the next level
  rvp::DevBuf open;   // open-query compaction between levels (flags, scan, list)
  bool stats_on = false;
  int n_frames_last = 0;
  // run_host: events after the voxel and SOR stages, so that their results
  // go down (s_out) while the later stages run; sizes read on s_meta
  bool record_stages = false;
  cudaEvent_t ev_stage[2] = {nullptr, nullptr};
  cudaStream_t s_out = nullptr, s_meta = nullptr;
  // run_host_batches: a second input set (batch i + 1 goes up while batch i
  // runs), the copy-in stream, and events for the copies; wait_before holds
  // the events run_device waits for at the voxel, SOR-filter, normal and
  // RANSAC stages (the previous batch's results of that stage are down)
  rvp::DevBuf in2_x, in2_y, in2_z, in2_offs;
  cudaStream_t s_in = nullptr;
  cudaEvent_t ev_h2d[2] = {nullptr, nullptr};
  cudaEvent_t ev_end = nullptr, ev_dv = nullptr, ev_ds = nullptr, ev_dn = nullptr;
  cudaEvent_t wait_before[4] = {nullptr, nullptr, nullptr, nullptr};
  // stage timing: a ring of event sets, one set per run
  // (stage boundaries, then a pair around each grid level's kNN kernel: SOR
  // levels 0-2, normals levels 0-2)
  static constexpr int kStages = 7;
  static constexpr int kLevelKernels = 2 * rvp::kTimedKernels;
  static constexpr int kEventsPerRun = kStages + 1 + 2 * kLevelKernels;
  std::vector<cudaEvent_t> events;  // runs_cap * kEventsPerRun
  int runs_cap = 0, runs_recorded = 0;
  // one run captured as a CUDA graph (rvp_pipeline_capture / _replay)
  cudaGraphExec_t graph = nullptr;
  uint64_t graph_kernels = 0;
  bool capturing = false;
  void mark(int stage) {
    if (capturing || runs_cap == 0 || runs_recorded >= runs_cap) return;
    cudaEventRecord(events[(size_t)runs_recorded * kEventsPerRun + stage], ctx->stream);
  }
  // events around the kNN kernels of the current run (first = 0 SOR, 1 normals)
  cudaEvent_t *level_events(int first) {
    if (capturing || runs_cap == 0 || runs_recorded >= runs_cap) return nullptr;
    return &events[(size_t)runs_recorded * kEventsPerRun + kStages + 1 +
                   first * 2 * rvp::kTimedKernels];
  }
  // a run whose kNN skipped the per-level kernels records zero-length pairs
  void empty_level_events(cudaEvent_t *ev) {
    if (ev)
      for (int j = 0; j < 2 * rvp::kTimedKernels; ++j) cudaEventRecord(ev[j], ctx->stream);
  }
};

namespace {
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

__global__ void k_frame_ids(const int64_t *offs, int n_frames, size_t n_max, int32_t *frame) {
  const u64 n = (u64)offs[n_frames];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n && i < n_max;
       i += (size_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = n_frames - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if ((u64)offs[mid] <= i) lo = mid; else hi = mid - 1;
    }
    frame[i] = lo;
  }
}

__global__ void k_widen(const u32 *a, u64 *b) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *b = *a;
}

__global__ void k_queue_kept(const uint8_t *keep, const u64 *n_dev, size_t n_max, u32 *list,
                             u32 *count) {
  const size_t n = n_dev ? *n_dev : n_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    if (keep[i]) list[atomicAdd(count, 1u)] = (u32)i;
}

// flag grid points whose source point was removed by SOR
__global__ void k_mark_removed(float4 *pts, const uint8_t *keep, const u64 *n_dev, size_t n_max) {
  const size_t n = n_dev ? *n_dev : n_max;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const u32 idx = __float_as_uint(pts[i].w);
    if (!keep[idx & 0x7FFFFFFFu]) pts[i].w = __uint_as_float(idx | 0x80000000u);
  }
}
}  // namespace

namespace {
// frees everything a pipeline holds (also a partly created one) and the
// pipeline itself
void release_pipeline(rvp_pipeline *p) {
  rvp::DevBuf *bufs[] = {&p->in_x, &p->in_y, &p->in_z, &p->in_offs, &p->vox_aos, &p->vox_x,
                         &p->vox_y, &p->vox_z, &p->vox_offs, &p->vox_frame, &p->sor_list,
                         &p->knn_counts, &p->mean, &p->keep, &p->sor_tmp, &p->sor_aos, &p->sor_x,
                         &p->sor_y, &p->sor_z, &p->sor_offs, &p->sor_frame, &p->sor_src,
                         &p->nrm_pairs, &p->nrm_counts, &p->nx, &p->ny, &p->nz, &p->r_model,
                         &p->r_best, &p->r_iters, &p->r_rand, &p->stats, &p->hard, &p->qlevel,
                         &p->qtau, &p->open, &p->routed};
  for (auto *b : bufs) b->release();
  p->vw.release();
  p->grid.release();
  for (auto e : p->events) cudaEventDestroy(e);
  if (p->graph) cudaGraphExecDestroy(p->graph);
  for (auto e : p->ev_stage)
    if (e) cudaEventDestroy(e);
  if (p->s_out) cudaStreamDestroy(p->s_out);
  if (p->s_meta) cudaStreamDestroy(p->s_meta);
  if (p->s_in) cudaStreamDestroy(p->s_in);
  for (cudaEvent_t e : {p->ev_h2d[0], p->ev_h2d[1], p->ev_end, p->ev_dv, p->ev_ds, p->ev_dn})
    if (e) cudaEventDestroy(e);
  for (auto *b : {&p->in2_x, &p->in2_y, &p->in2_z, &p->in2_offs}) b->release();
  delete p;
}
}  // namespace

extern "C" {

rvp_status rvp_pipeline_create(rvp_context *ctx, const rvp_pipeline_config *cfg,
                               size_t max_points, int max_frames, rvp_pipeline **out) {
  if (!ctx || !cfg || !out) return RVP_ERR_INVALID_ARG;
  *out = nullptr;
  rvp_pipeline *p = new (std::nothrow) rvp_pipeline();
  if (!p) return RVP_ERR_OOM;
  rvp_status s = guard(ctx, [&] {
    RVP_REQUIRE(max_points >= 1 && max_points < 0x7FFFFFFFull, "max_points out of range");
    RVP_REQUIRE(max_frames >= 1, "max_frames must be >= 1");
    RVP_REQUIRE(cfg->leaf_size > 0.0f, "leaf_size must be > 0");
    RVP_REQUIRE(cfg->sor_k >= 1 && cfg->sor_k + 1 <= 64, "sor_k must be in [1, 63]");
    RVP_REQUIRE(cfg->normal_k >= 1 && cfg->normal_k + 1 <= 64, "normal_k must be in [1, 63]");
    RVP_REQUIRE(cfg->ransac_iters >= 0, "ransac_iters must be >= 0");
    RVP_REQUIRE(cfg->block_threads >= 0 && cfg->block_threads <= 256 &&
                    cfg->block_threads % 32 == 0,
                "block_threads must be 0 or a multiple of 32 up to 256");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    p->ctx = ctx;
    p->cfg = *cfg;
    p->max_points = max_points;
    p->max_frames = max_frames;
    p->cell = cfg->cell_size > 0.0f ? cfg->cell_size : 2.5f * cfg->leaf_size;
    const size_t N = max_points;
    const size_t F1 = (size_t)max_frames + 1;
    p->in_x.reserve(N * 4); p->in_y.reserve(N * 4); p->in_z.reserve(N * 4);
    p->in_offs.reserve(F1 * 8);
    p->vw.reserve(N, max_frames);
    p->grid.reserve(N, max_frames);
    p->vox_aos.reserve(N * 12);
    p->vox_x.reserve(N * 4); p->vox_y.reserve(N * 4); p->vox_z.reserve(N * 4);
    p->vox_offs.reserve(F1 * 8);
    p->vox_frame.reserve(N * 4);
    const int ks = cfg->sor_k + 1, kn = cfg->normal_k + 1;
    p->sor_list.reserve(N * (size_t)ks * 4);
    p->knn_counts.reserve(N * 4);
    p->mean.reserve(N * 4);
    p->keep.reserve(N);
    p->sor_tmp.reserve(rvp::sor_filter_temp_bytes(N, max_frames));
    p->sor_aos.reserve(N * 12);
    p->sor_x.reserve(N * 4); p->sor_y.reserve(N * 4); p->sor_z.reserve(N * 4);
    p->sor_offs.reserve(F1 * 8);
    p->sor_frame.reserve(N * 4);
    p->sor_src.reserve(N * 4);
    p->nrm_pairs.reserve(N * (size_t)kn * 8);
    p->hard.reserve(N * 8 + 256);
    p->qlevel.reserve(N);
    p->qtau.reserve(N * 4);
    p->routed.reserve(256);
    p->open.reserve(((N * 4 + 255) & ~(size_t)255) + ((N * 8 + 8 + 255) & ~(size_t)255) +
                    ((N * 4 + 255) & ~(size_t)255) + 256 + rvp::scan_temp_bytes(N));
    p->nrm_counts.reserve(N * 4);
    p->nx.reserve(N * 4); p->ny.reserve(N * 4); p->nz.reserve(N * 4);
    p->r_model.reserve((size_t)max_frames * 16);
    p->r_best.reserve((size_t)max_frames * 4);
    p->r_iters.reserve((size_t)max_frames * 4);
    // the reference's srand(0) + rand() stream, shared by every frame
    const size_t R = 3 * (size_t)std::max(cfg->ransac_iters, 1);
    std::vector<int> rs(R);
    srand(0);
    for (size_t i = 0; i < R; ++i) rs[i] = rand();
    srand(0);
    p->r_rand.reserve(R * 4);
    RVP_CUDA_TRY(cudaMemcpy(p->r_rand.ptr, rs.data(), R * 4, cudaMemcpyHostToDevice));
  });
  if (s != RVP_OK) {
    release_pipeline(p);
    return s;
  }
  *out = p;
  return RVP_OK;
}

rvp_status rvp_pipeline_destroy(rvp_pipeline *p) {
  if (!p) return RVP_ERR_INVALID_ARG;
  cudaSetDevice(p->ctx->device);
  cudaStreamSynchronize(p->ctx->stream);
  release_pipeline(p);
  return RVP_OK;
}

rvp_status rvp_pipeline_run_device(rvp_pipeline *p, const float *x, const float *y,
                                   const float *z, const int64_t *offs, int n_frames,
                                   size_t n_points) {
  if (!p) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = p->ctx;
  return guard(ctx, [&] {
    RVP_REQUIRE(n_frames >= 1 && n_frames <= p->max_frames, "n_frames out of range");
    RVP_REQUIRE(n_points <= p->max_points, "n_points exceeds the pipeline capacity");
    RVP_REQUIRE(x && y && z && offs, "null pointer");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    const rvp_pipeline_config &c = p->cfg;
    const size_t N = n_points > 0 ? n_points : 1;
    cudaStream_t st = ctx->stream;
    const int sms = ctx->num_sms;
    p->n_frames_last = n_frames;
    int64_t *vox_offs = p->vox_offs.as<int64_t>();
    const u64 *n_vox = reinterpret_cast<const u64 *>(vox_offs + n_frames);
    int64_t *sor_offs = p->sor_offs.as<int64_t>();
    const u64 *n_sor = reinterpret_cast<const u64 *>(sor_offs + n_frames);

    p->mark(0);
    if (p->wait_before[0]) RVP_CUDA_TRY(cudaStreamWaitEvent(st, p->wait_before[0], 0));
    // 1) voxel grid
    const float inv_leaf = 1.0f / c.leaf_size;
    rvp::voxel_grid_run(ctx, p->vw, x, y, z, offs, n_frames, N, nullptr, inv_leaf,
                        p->vox_aos.as<float>(), vox_offs, nullptr, nullptr, p->vox_x.as<float>(),
                        p->vox_y.as<float>(), p->vox_z.as<float>());
    p->mark(1);
    if (p->record_stages) RVP_CUDA_TRY(cudaEventRecord(p->ev_stage[0], st));
    // 2) grid over the voxel points of every frame: cells of `cell` for the
    //    searches, the points sorted by cells of cell / 4 inside them (so
    //    that consecutive points, a warp's queries, lie close together)
    rvp::grid_build(ctx, p->grid, p->vox_x.as<float>(), p->vox_y.as<float>(),
                    p->vox_z.as<float>(), vox_offs, n_frames, N, p->cell, rvp::KEY_DENSE, 0, 0,
                    n_vox, p->grid_base, p->vox_aos.as<float>());
    k_frame_ids<<<rvp::grid_for(N, 256, sms * 16), 256, 0, st>>>(vox_offs, n_frames, N,
                                                                 p->vox_frame.as<int32_t>());
    RVP_LAUNCH_CHECK(ctx);
    const rvp::GridView gv = p->grid.view(rvp::KEY_DENSE, 0, 0);
    p->mark(2);
    // 3) SOR: exact k+1 nearest and the mean distance, fused in the tile
    //    kernel; the queries its 27-cell ring cannot certify are finished by
    //    the warp kernel (tight windows, coarse level, whole frame)
    const int ks = c.sor_k + 1;
    u64 *hard_n64 = p->hard.as<u64>();                   // widened count (grid_knn)
    u32 *hard_n = reinterpret_cast<u32 *>(hard_n64 + 1);  // atomic counter
    u32 *hard = reinterpret_cast<u32 *>(hard_n64 + 2);    // original indices
    float *hard_tau = reinterpret_cast<float *>(hard + N); // their K-th distance bounds
    u32 *st0 = p->stats_on ? p->stats.as<u32>() : nullptr;
    rvp::TileArgs ta{};
    ta.frame_of = p->vox_frame.as<int32_t>();
    ta.hard = hard;
    ta.hard_count = hard_n;
    ta.hard_tau = hard_tau;
    ta.qlevel = p->qlevel.as<uint8_t>();
    ta.qtau = p->qtau.as<float>();
    ta.rfac = p->rfac;
    ta.lane_levels = p->lane_levels;
    ta.level0_warp = c.queries_per_warp != 2;  // 2: shared-memory tiles instead
    ta.coop = c.queries_per_warp == 3;         // 3: cooperative passes first
    ta.routed = p->routed.as<u64>();
    if (ta.coop) RVP_CUDA_TRY(cudaMemsetAsync(ta.routed, 0, 16, st));
    {
      char *op = p->open.as<char>();
      auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
      ta.open_flags = reinterpret_cast<u32 *>(op); op += al(N * 4);
      ta.open_pos = reinterpret_cast<u64 *>(op); op += al(N * 8 + 8);
      ta.open_list = reinterpret_cast<u32 *>(op); op += al(N * 4);
      ta.open_n = reinterpret_cast<u64 *>(op); op += 256;
      ta.scan_tmp = op;
    }
    ta.n_max = N;
    ta.level_events = p->level_events(0);
    const bool tiled = c.queries_per_warp != 1;
    rvp::QuerySet qh{p->vox_x.as<float>(), p->vox_y.as<float>(), p->vox_z.as<float>(), N,
                     hard_n64, p->vox_frame.as<int32_t>(), reinterpret_cast<int32_t *>(hard)};
    qh.bound = tiled ? hard_tau : nullptr;
    rvp::QuerySet qv{p->vox_x.as<float>(), p->vox_y.as<float>(), p->vox_z.as<float>(), N, n_vox,
                     p->vox_frame.as<int32_t>(), nullptr};
    ta.mean = p->mean.as<float>();
    // with the per-warp kernels the SOR stage also keeps each point's k+1
    // nearest indices, from which the normal stage takes the lists of the
    // points whose neighbours all survive
    const int kn = c.normal_k + 1;
    const bool lists = (c.queries_per_warp == 0 || c.queries_per_warp == 3) && kn <= ks;
    ta.sor_list = lists ? p->sor_list.as<u32>() : nullptr;
    RVP_CUDA_TRY(cudaMemsetAsync(hard_n64, 0, 16, st));
    bool sor_lists = false;
    if (tiled && rvp::grid_knn_tile(ctx, gv, ks, lists ? rvp::TILE_SOR_LIST : rvp::TILE_SOR_MEAN,
                                    ta, 0, st0 ? st0 + 5 : nullptr)) {
      sor_lists = lists;
      k_widen<<<1, 32, 0, st>>>(hard_n, hard_n64);
      RVP_LAUNCH_CHECK(ctx);
      // the hard queries with a bound: their tight windows, one per thread
      rvp::grid_knn_tau(ctx, gv, ks, lists ? rvp::TILE_SOR_LIST : rvp::TILE_SOR_MEAN, ta, hard_n64,
                        nullptr, nullptr, st0 ? st0 + 16 : nullptr);
      rvp::grid_knn(ctx, gv, qh, ks, 0.0f,
                    sor_lists ? reinterpret_cast<u64 *>(p->sor_list.ptr) : nullptr, nullptr, 1,
                    c.block_threads, st0,
                    sor_lists ? rvp::KNN_OUT_SOR_MEAN_LIST : rvp::KNN_OUT_SOR_MEAN,
                    p->mean.as<float>());
    } else {
      p->empty_level_events(ta.level_events);
      rvp::grid_knn(ctx, gv, qv, ks, 0.0f, nullptr, nullptr, 1, c.block_threads, st0,
                    rvp::KNN_OUT_SOR_MEAN, p->mean.as<float>());
    }
    p->mark(3);
    if (p->wait_before[1]) RVP_CUDA_TRY(cudaStreamWaitEvent(st, p->wait_before[1], 0));
    rvp::sor_filter_frames(ctx, p->vox_x.as<float>(), p->vox_y.as<float>(), p->vox_z.as<float>(),
                           p->mean.as<float>(), vox_offs, n_frames, N, n_vox, c.sor_alpha,
                           p->keep.as<uint8_t>(), p->sor_aos.as<float>(), sor_offs, nullptr,
                           p->sor_tmp.ptr, p->sor_x.as<float>(), p->sor_y.as<float>(),
                           p->sor_z.as<float>(), p->sor_src.as<u32>());
    const u64 *sor_pos = rvp::sor_positions(p->sor_tmp.ptr, N);
    p->mark(4);
    if (p->record_stages) RVP_CUDA_TRY(cudaEventRecord(p->ev_stage[1], st));
    if (p->wait_before[2]) RVP_CUDA_TRY(cudaStreamWaitEvent(st, p->wait_before[2], 0));
    // 4) normals: the k+1 nearest kept points of every kept point, with the
    //    reference normal computed in the same tile kernel
    k_mark_removed<<<rvp::grid_for(N, 256, sms * 16), 256, 0, st>>>(
        p->grid.b_pts.as<float4>(), p->keep.as<uint8_t>(), n_vox, N);
    RVP_LAUNCH_CHECK(ctx);
    rvp::TileArgs tn = ta;
    tn.routed = nullptr;
    tn.mean = nullptr;
    tn.vx = p->vox_x.as<float>();
    tn.vy = p->vox_y.as<float>();
    tn.vz = p->vox_z.as<float>();
    tn.out_pos = sor_pos;
    tn.nx = p->nx.as<float>();
    tn.ny = p->ny.as<float>();
    tn.nz = p->nz.as<float>();
    tn.iters = c.eigen_iters;
    tn.vpx = c.vp_x;
    tn.vpy = c.vp_y;
    tn.vpz = c.vp_z;
    tn.level_events = p->level_events(1);
    // the normals' open queries sit next to removed points, where rings are
    // sparse: after one per-lane level the warp kernel is cheaper
    tn.lane_levels = 1;
    RVP_CUDA_TRY(cudaMemsetAsync(hard_n64, 0, 16, st));
    // points whose SOR list holds kn kept points: normal straight from it;
    // the rest open for the kNN search
    tn.preset_open = sor_lists && rvp::normals_from_sor_lists(ctx, gv, tn, ks, kn);
    bool tn_ok = tiled && rvp::grid_knn_tile(ctx, gv, kn, rvp::TILE_NORMALS, tn, 0,
                                             st0 ? st0 + 13 : nullptr);
    if (!tn_ok) {
      p->empty_level_events(tn.level_events);
      // every kept point through the warp kernel: queue them all
      k_queue_kept<<<rvp::grid_for(N, 256, sms * 16), 256, 0, st>>>(p->keep.as<uint8_t>(), n_vox,
                                                                    N, hard, hard_n);
      RVP_LAUNCH_CHECK(ctx);
    }
    k_widen<<<1, 32, 0, st>>>(hard_n, hard_n64);
    RVP_LAUNCH_CHECK(ctx);
    if (tn_ok)
      rvp::grid_knn_tau(ctx, gv, kn, rvp::TILE_NORMALS, tn, hard_n64, p->nrm_pairs.as<u64>(),
                        p->nrm_counts.as<int32_t>(), st0 ? st0 + 17 : nullptr);
    rvp::QuerySet qhn = qh;
    qhn.bound = tn_ok ? hard_tau : nullptr;
    rvp::grid_knn(ctx, gv, qhn, kn, 0.0f, p->nrm_pairs.as<u64>(), p->nrm_counts.as<int32_t>(),
                  1, c.block_threads, st0 ? st0 + 8 : nullptr, rvp::KNN_OUT_BY_SLOT, nullptr);
    p->mark(5);
    rvp::normals_from_lists(ctx, p->vox_x.as<float>(), p->vox_y.as<float>(), p->vox_z.as<float>(),
                            p->nrm_pairs.as<u64>(), nullptr, p->nrm_counts.as<int32_t>(), kn, N,
                            hard_n64, true, c.eigen_iters, c.vp_x, c.vp_y, c.vp_z,
                            p->vox_x.as<float>(), p->vox_y.as<float>(), p->vox_z.as<float>(),
                            p->nx.as<float>(), p->ny.as<float>(), p->nz.as<float>(), hard,
                            sor_pos);
    p->mark(6);
    if (p->wait_before[3]) RVP_CUDA_TRY(cudaStreamWaitEvent(st, p->wait_before[3], 0));
    // 5) RANSAC per frame on the kept points
    double pc = (double)c.ransac_prob;
    pc = pc < 0.5 ? 0.5 : (pc > 0.9999 ? 0.9999 : pc);
    rvp::RansacParams prm{c.ransac_thresh, c.ransac_iters, c.ransac_collinear, log(1.0 - pc)};
    rvp::ransac_frames(ctx, p->sor_x.as<float>(), p->sor_y.as<float>(), p->sor_z.as<float>(),
                       sor_offs, n_frames, p->r_rand.as<int>(), prm, p->r_model.as<float>(),
                       p->r_best.as<int32_t>(), p->r_iters.as<int32_t>(), nullptr, false,
                       rvp::RansacSampler{}, 4);
    p->mark(7);
    if (!p->capturing && p->runs_cap > 0 && p->runs_recorded < p->runs_cap) p->runs_recorded++;
  });
}

rvp_status rvp_pipeline_capture(rvp_pipeline *p, const float *x, const float *y, const float *z,
                                const int64_t *offs, int n_frames, size_t n_points,
                                uint64_t *kernels) {
  if (!p) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = p->ctx;
  cudaStream_t user_stream = ctx->stream;
  cudaStream_t cap = nullptr;
  cudaGraph_t g = nullptr;
  rvp_status run = RVP_OK;
  rvp_status s = guard(ctx, [&] {
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    // the legacy default stream cannot be captured: capture on a private
    // stream ordered after the caller's work; the replay goes to the
    // context's stream
    RVP_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    RVP_CUDA_TRY(cudaStreamSynchronize(user_stream));
    if (p->graph) {
      RVP_CUDA_TRY(cudaGraphExecDestroy(p->graph));
      p->graph = nullptr;
    }
    RVP_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    ctx->stream = cap;
    p->capturing = true;
    const uint64_t l0 = ctx->launches;
    run = rvp_pipeline_run_device(p, x, y, z, offs, n_frames, n_points);
    p->graph_kernels = ctx->launches - l0;
    p->capturing = false;
    ctx->stream = user_stream;
    const cudaError_t e = cudaStreamEndCapture(cap, &g);
    if (run != RVP_OK) return;
    RVP_CUDA_TRY(e);
    RVP_CUDA_TRY(cudaGraphInstantiate(&p->graph, g, 0));
    RVP_CUDA_TRY(cudaGraphUpload(p->graph, user_stream));
  });
  p->capturing = false;
  ctx->stream = user_stream;
  if (g) cudaGraphDestroy(g);
  if (cap) cudaStreamDestroy(cap);
  if (run != RVP_OK) return run;  // its message is already in last_error
  if (s == RVP_OK && kernels) *kernels = p->graph_kernels;
  return s;
}

rvp_status rvp_pipeline_replay(rvp_pipeline *p) {
  if (!p) return RVP_ERR_INVALID_ARG;
  return guard(p->ctx, [&] {
    RVP_REQUIRE(p->graph, "no captured run: call rvp_pipeline_capture first");
    RVP_CUDA_TRY(cudaSetDevice(p->ctx->device));
    RVP_CUDA_TRY(cudaGraphLaunch(p->graph, p->ctx->stream));
    p->ctx->launches += p->graph_kernels;
  });
}

rvp_status rvp_pipeline_fit_tables(rvp_pipeline *p) {
  if (!p) return RVP_ERR_INVALID_ARG;
  return guard(p->ctx, [&] {
    RVP_CUDA_TRY(cudaSetDevice(p->ctx->device));
    u64 nb[rvp::kHeadLevels] = {};
    RVP_CUDA_TRY(cudaMemcpyAsync(nb, p->grid.d_nbuckets, 8 * rvp::kHeadLevels, cudaMemcpyDeviceToHost,
                                 p->ctx->stream));
    RVP_CUDA_TRY(cudaStreamSynchronize(p->ctx->stream));
    // a quarter of headroom for batches whose scenes occupy more cells than
    // this one; the table (2.5 slots per bucket, rounded up to a power of
    // two) then stays inside L2, where every probe of the kNN kernels lands
    size_t tot = 0;
    for (int l = 0; l < rvp::kGridLevels; ++l) tot += (size_t)nb[l];
    p->grid.fit_table(tot + tot / 4);
  });
}

rvp_status rvp_pipeline_check(rvp_pipeline *p) {
  if (!p) return RVP_ERR_INVALID_ARG;
  int flags[2] = {0, 0};
  rvp_status s = guard(p->ctx, [&] {
    RVP_CUDA_TRY(cudaSetDevice(p->ctx->device));
    RVP_CUDA_TRY(cudaMemcpyAsync(flags, p->grid.d_collision, 8, cudaMemcpyDeviceToHost,
                                 p->ctx->stream));
    RVP_CUDA_TRY(cudaStreamSynchronize(p->ctx->stream));
  });
  if (s != RVP_OK) return s;
  if (flags[1]) {
    p->ctx->last_error = "neighbour grid table overflow: refit the tables (rvp_pipeline_fit_tables)";
    return RVP_ERR_CAPACITY;
  }
  return RVP_OK;
}

rvp_status rvp_pipeline_knn_stats(rvp_pipeline *p, int enable, uint32_t *out20) {
  if (!p) return RVP_ERR_INVALID_ARG;
  return guard(p->ctx, [&] {
    RVP_CUDA_TRY(cudaSetDevice(p->ctx->device));
    p->stats.reserve(80);
    if (out20) {
      RVP_CUDA_TRY(cudaMemcpyAsync(out20, p->stats.ptr, 80, cudaMemcpyDeviceToHost,
                                   p->ctx->stream));
      RVP_CUDA_TRY(cudaStreamSynchronize(p->ctx->stream));
    }
    RVP_CUDA_TRY(cudaMemsetAsync(p->stats.ptr, 0, 80, p->ctx->stream));
    p->stats_on = enable != 0;
  });
}

rvp_status rvp_pipeline_knn_routed(rvp_pipeline *p, uint64_t *out) {
  if (!p || !out) return RVP_ERR_INVALID_ARG;
  return guard(p->ctx, [&] {
    RVP_CUDA_TRY(cudaSetDevice(p->ctx->device));
    if (!p->routed.ptr) {
      out[0] = out[1] = 0;
      return;
    }
    RVP_CUDA_TRY(cudaMemcpyAsync(out, p->routed.ptr, 16, cudaMemcpyDeviceToHost,
                                 p->ctx->stream));
    RVP_CUDA_TRY(cudaStreamSynchronize(p->ctx->stream));
  });
}

rvp_status rvp_pipeline_frame_offsets(rvp_pipeline *p, int64_t *voxel_offsets,
                                      int64_t *sor_offsets) {
  if (!p) return RVP_ERR_INVALID_ARG;
  return guard(p->ctx, [&] {
    const size_t b = ((size_t)p->n_frames_last + 1) * 8;
    if (voxel_offsets)
      RVP_CUDA_TRY(cudaMemcpyAsync(voxel_offsets, p->vox_offs.ptr, b, cudaMemcpyDeviceToHost,
                                   p->ctx->stream));
    if (sor_offsets)
      RVP_CUDA_TRY(cudaMemcpyAsync(sor_offsets, p->sor_offs.ptr, b, cudaMemcpyDeviceToHost,
                                   p->ctx->stream));
    RVP_CUDA_TRY(cudaStreamSynchronize(p->ctx->stream));
  });
}

rvp_status rvp_pipeline_set_tuning(rvp_pipeline *p, float cell_size, int block_threads,
                                   int queries_per_warp) {
  if (!p) return RVP_ERR_INVALID_ARG;
  if (!(cell_size > 0.0f)) return RVP_ERR_INVALID_ARG;
  // the warp-per-query kernel is compiled for blocks of at most 256 threads
  if (block_threads < 0 || block_threads > 256 || (block_threads % 32) != 0)
    return RVP_ERR_INVALID_ARG;
  p->cell = cell_size;
  p->cfg.cell_size = cell_size;
  p->cfg.block_threads = block_threads;
  p->cfg.queries_per_warp = queries_per_warp;
  return RVP_OK;
}

rvp_status rvp_pipeline_set_search_radius_factor(rvp_pipeline *p, float rfac) {
  if (!p || !(rfac >= 0.0f)) return RVP_ERR_INVALID_ARG;
  p->rfac = rfac;
  return RVP_OK;
}

rvp_status rvp_pipeline_set_lane_levels(rvp_pipeline *p, int levels) {
  if (!p || levels < 0 || levels > rvp::kChainLevels) return RVP_ERR_INVALID_ARG;
  p->lane_levels = levels;
  return RVP_OK;
}

rvp_status rvp_pipeline_set_timing(rvp_pipeline *p, int max_runs) {
  if (!p || max_runs < 0) return RVP_ERR_INVALID_ARG;
  return guard(p->ctx, [&] {
    RVP_CUDA_TRY(cudaSetDevice(p->ctx->device));
    for (auto e : p->events) cudaEventDestroy(e);
    p->events.clear();
    p->runs_cap = 0;
    p->runs_recorded = 0;
    p->events.resize((size_t)max_runs * rvp_pipeline::kEventsPerRun);
    for (auto &e : p->events) RVP_CUDA_TRY(cudaEventCreate(&e));
    p->runs_cap = max_runs;
  });
}

rvp_status rvp_pipeline_stage_times(rvp_pipeline *p, float *ms, int n_stages, int *runs) {
  using P = rvp_pipeline;
  if (!p || !ms || n_stages < P::kStages) return RVP_ERR_INVALID_ARG;
  return guard(p->ctx, [&] {
    RVP_CUDA_TRY(cudaStreamSynchronize(p->ctx->stream));
    const int n_out = n_stages < P::kStages + P::kLevelKernels ? P::kStages
                                                                : P::kStages + P::kLevelKernels;
    for (int s = 0; s < n_out; ++s) ms[s] = 0.0f;
    const int R = p->runs_recorded;
    // the per-level events exist only on runs whose kNN went through the
    // per-level kernels; a run without them reports 0 there
    int level_runs = 0;
    for (int r = 0; r < R; ++r) {
      cudaEvent_t *ev = &p->events[(size_t)r * P::kEventsPerRun];
      for (int s = 0; s < P::kStages; ++s) {
        float t = 0.0f;
        RVP_CUDA_TRY(cudaEventElapsedTime(&t, ev[s], ev[s + 1]));
        ms[s] += t;
      }
      if (n_out > P::kStages) {
        float lt[P::kLevelKernels];
        bool ok = true;
        for (int j = 0; j < P::kLevelKernels && ok; ++j) {
          const cudaEvent_t *e = ev + P::kStages + 1 + 2 * j;
          ok = cudaEventElapsedTime(&lt[j], e[0], e[1]) == cudaSuccess;
        }
        if (ok) {
          for (int j = 0; j < P::kLevelKernels; ++j) ms[P::kStages + j] += lt[j];
          ++level_runs;
        } else {
          cudaGetLastError();
        }
      }
    }
    if (R > 0)
      for (int s = 0; s < P::kStages; ++s) ms[s] /= (float)R;
    if (level_runs > 0)
      for (int s = P::kStages; s < n_out; ++s) ms[s] /= (float)level_runs;
    if (runs) *runs = R;
    p->runs_recorded = 0;
  });
}

rvp_status rvp_pipeline_outputs_get(rvp_pipeline *p, rvp_pipeline_outputs *o) {
  if (!p || !o) return RVP_ERR_INVALID_ARG;
  o->voxel_aos = p->vox_aos.as<float>();
  o->voxel_offsets = p->vox_offs.as<int64_t>();
  o->sor_aos = p->sor_aos.as<float>();
  o->sor_offsets = p->sor_offs.as<int64_t>();
  o->nx = p->nx.as<float>();
  o->ny = p->ny.as<float>();
  o->nz = p->nz.as<float>();
  o->ransac_model = p->r_model.as<float>();
  o->ransac_count = p->r_best.as<int32_t>();
  o->ransac_iters = p->r_iters.as<int32_t>();
  o->sor_mean_dists = p->mean.as<float>();
  return RVP_OK;
}

rvp_status rvp_pipeline_run_host(rvp_pipeline *p, const float *x, const float *y, const float *z,
                                 const int64_t *frame_offsets, int n_frames, float *voxel_aos,
                                 int64_t *voxel_offsets, float *sor_aos, int64_t *sor_offsets,
                                 float *nx, float *ny, float *nz, float *ransac_model,
                                 int32_t *ransac_count) {
  if (!p) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = p->ctx;
  rvp_status s = guard(ctx, [&] {
    RVP_REQUIRE(frame_offsets && n_frames >= 1 && n_frames <= p->max_frames, "bad frames");
    const size_t n = (size_t)frame_offsets[n_frames];
    RVP_REQUIRE(n <= p->max_points, "batch exceeds the pipeline capacity");
    RVP_REQUIRE(n == 0 || (x && y && z), "null pointer");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (n) {
      RVP_CUDA_TRY(cudaMemcpyAsync(p->in_x.ptr, x, n * 4, cudaMemcpyHostToDevice, st));
      RVP_CUDA_TRY(cudaMemcpyAsync(p->in_y.ptr, y, n * 4, cudaMemcpyHostToDevice, st));
      RVP_CUDA_TRY(cudaMemcpyAsync(p->in_z.ptr, z, n * 4, cudaMemcpyHostToDevice, st));
    }
    RVP_CUDA_TRY(cudaMemcpyAsync(p->in_offs.ptr, frame_offsets, (n_frames + 1) * 8,
                                 cudaMemcpyHostToDevice, st));
  });
  if (s != RVP_OK) return s;
  const size_t n = (size_t)frame_offsets[n_frames];
  s = guard(ctx, [&] {
    if (!p->s_out) {
      RVP_CUDA_TRY(cudaStreamCreateWithFlags(&p->s_out, cudaStreamNonBlocking));
      RVP_CUDA_TRY(cudaStreamCreateWithFlags(&p->s_meta, cudaStreamNonBlocking));
      for (auto &e : p->ev_stage) RVP_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
  });
  if (s != RVP_OK) return s;
  // queue the whole run, then bring each stage's results down as soon as
  // that stage is done: the voxel output under SOR and normals, the SOR
  // output under normals and RANSAC
  p->record_stages = true;
  s = rvp_pipeline_run_device(p, p->in_x.as<float>(), p->in_y.as<float>(), p->in_z.as<float>(),
                              p->in_offs.as<int64_t>(), n_frames, n);
  p->record_stages = false;
  if (s != RVP_OK) return s;
  s = guard(ctx, [&] {
    cudaStream_t st = ctx->stream;
    std::vector<int64_t> vo(n_frames + 1), so(n_frames + 1);
    auto d2h = [&](void *dst, const void *src, size_t b, cudaStream_t on) {
      if (dst && b) RVP_CUDA_TRY(cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToHost, on));
    };
    RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_meta, p->ev_stage[0], 0));
    RVP_CUDA_TRY(cudaMemcpyAsync(vo.data(), p->vox_offs.ptr, (n_frames + 1) * 8,
                                 cudaMemcpyDeviceToHost, p->s_meta));
    RVP_CUDA_TRY(cudaStreamSynchronize(p->s_meta));
    const size_t nv = (size_t)vo[n_frames];
    if (voxel_offsets) memcpy(voxel_offsets, vo.data(), (n_frames + 1) * 8);
    RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_out, p->ev_stage[0], 0));
    d2h(voxel_aos, p->vox_aos.ptr, nv * 12, p->s_out);
    RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_meta, p->ev_stage[1], 0));
    RVP_CUDA_TRY(cudaMemcpyAsync(so.data(), p->sor_offs.ptr, (n_frames + 1) * 8,
                                 cudaMemcpyDeviceToHost, p->s_meta));
    RVP_CUDA_TRY(cudaStreamSynchronize(p->s_meta));
    const size_t ns = (size_t)so[n_frames];
    if (sor_offsets) memcpy(sor_offsets, so.data(), (n_frames + 1) * 8);
    RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_out, p->ev_stage[1], 0));
    d2h(sor_aos, p->sor_aos.ptr, ns * 12, p->s_out);
    d2h(nx, p->nx.ptr, ns * 4, st);
    d2h(ny, p->ny.ptr, ns * 4, st);
    d2h(nz, p->nz.ptr, ns * 4, st);
    d2h(ransac_model, p->r_model.ptr, (size_t)n_frames * 16, st);
    d2h(ransac_count, p->r_best.ptr, (size_t)n_frames * 4, st);
    RVP_CUDA_TRY(cudaStreamSynchronize(p->s_out));
    RVP_CUDA_TRY(cudaStreamSynchronize(st));
  });
  if (s != RVP_OK) {
    cudaStreamSynchronize(p->s_out);
    cudaStreamSynchronize(ctx->stream);
  }
  return s;
}

rvp_status rvp_pipeline_run_host_batches(
    rvp_pipeline *p, int n_batches, const float *const *x, const float *const *y,
    const float *const *z, const int64_t *const *frame_offsets, const int *n_frames,
    float *const *voxel_aos, int64_t *const *voxel_offsets, float *const *sor_aos,
    int64_t *const *sor_offsets, float *const *nx, float *const *ny, float *const *nz,
    float *const *ransac_model, int32_t *const *ransac_count) {
  if (!p || n_batches < 0) return RVP_ERR_INVALID_ARG;
  if (n_batches == 0) return RVP_OK;
  rvp_context *ctx = p->ctx;
  cudaStream_t st = ctx->stream;
  rvp_status s = guard(ctx, [&] {
    RVP_REQUIRE(x && y && z && frame_offsets && n_frames, "null batch arrays");
    for (int i = 0; i < n_batches; ++i) {
      RVP_REQUIRE(frame_offsets[i] && n_frames[i] >= 1 && n_frames[i] <= p->max_frames,
                  "bad frames");
      const size_t n = (size_t)frame_offsets[i][n_frames[i]];
      RVP_REQUIRE(n <= p->max_points, "batch exceeds the pipeline capacity");
      RVP_REQUIRE(n == 0 || (x[i] && y[i] && z[i]), "null pointer");
    }
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    if (!p->s_out) {
      RVP_CUDA_TRY(cudaStreamCreateWithFlags(&p->s_out, cudaStreamNonBlocking));
      RVP_CUDA_TRY(cudaStreamCreateWithFlags(&p->s_meta, cudaStreamNonBlocking));
      for (auto &e : p->ev_stage) RVP_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (!p->s_in) {
      RVP_CUDA_TRY(cudaStreamCreateWithFlags(&p->s_in, cudaStreamNonBlocking));
      for (cudaEvent_t *e : {&p->ev_h2d[0], &p->ev_h2d[1], &p->ev_end, &p->ev_dv, &p->ev_ds,
                             &p->ev_dn})
        RVP_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    const size_t N = p->max_points, F1 = (size_t)p->max_frames + 1;
    p->in2_x.reserve(N * 4); p->in2_y.reserve(N * 4); p->in2_z.reserve(N * 4);
    p->in2_offs.reserve(F1 * 8);
  });
  if (s != RVP_OK) return s;
  rvp::DevBuf *in[2][4] = {{&p->in_x, &p->in_y, &p->in_z, &p->in_offs},
                           {&p->in2_x, &p->in2_y, &p->in2_z, &p->in2_offs}};
  auto h2d = [&](int i) {  // batch i into input set i % 2, on the copy-in stream
    rvp::DevBuf **b = in[i & 1];
    const size_t n = (size_t)frame_offsets[i][n_frames[i]];
    if (n) {
      RVP_CUDA_TRY(cudaMemcpyAsync(b[0]->ptr, x[i], n * 4, cudaMemcpyHostToDevice, p->s_in));
      RVP_CUDA_TRY(cudaMemcpyAsync(b[1]->ptr, y[i], n * 4, cudaMemcpyHostToDevice, p->s_in));
      RVP_CUDA_TRY(cudaMemcpyAsync(b[2]->ptr, z[i], n * 4, cudaMemcpyHostToDevice, p->s_in));
    }
    RVP_CUDA_TRY(cudaMemcpyAsync(b[3]->ptr, frame_offsets[i], (n_frames[i] + 1) * 8,
                                 cudaMemcpyHostToDevice, p->s_in));
    RVP_CUDA_TRY(cudaEventRecord(p->ev_h2d[i & 1], p->s_in));
  };
  auto pick = [&](auto *const *arr, int i) { return arr ? arr[i] : nullptr; };
  for (int i = 0; i < n_batches && s == RVP_OK; ++i) {
    s = guard(ctx, [&] {
      if (i == 0) {
        RVP_CUDA_TRY(cudaEventRecord(p->ev_end, st));  // earlier work on the stream
        RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_in, p->ev_end, 0));
        h2d(0);
      }
      if (i + 1 < n_batches) {
        // input set (i + 1) % 2 is free once batch i - 1's voxel stage is done
        if (i >= 1) RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_in, p->ev_stage[0], 0));
        h2d(i + 1);
      }
      RVP_CUDA_TRY(cudaStreamWaitEvent(st, p->ev_h2d[i & 1], 0));
      cudaEvent_t w[4] = {p->ev_dv, p->ev_ds, p->ev_dn, p->ev_dn};
      for (int k = 0; k < 4; ++k) p->wait_before[k] = i > 0 ? w[k] : nullptr;
    });
    if (s != RVP_OK) break;
    rvp::DevBuf **b = in[i & 1];
    const size_t n = (size_t)frame_offsets[i][n_frames[i]];
    p->record_stages = true;
    s = rvp_pipeline_run_device(p, b[0]->as<float>(), b[1]->as<float>(), b[2]->as<float>(),
                                b[3]->as<int64_t>(), n_frames[i], n);
    p->record_stages = false;
    for (auto &e : p->wait_before) e = nullptr;
    if (s != RVP_OK) break;
    s = guard(ctx, [&] {
      const int nf = n_frames[i];
      RVP_CUDA_TRY(cudaEventRecord(p->ev_end, st));
      std::vector<int64_t> vo(nf + 1), so(nf + 1);
      auto d2h = [&](void *dst, const void *src, size_t bytes) {
        if (dst && bytes)
          RVP_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, p->s_out));
      };
      RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_meta, p->ev_stage[0], 0));
      RVP_CUDA_TRY(cudaMemcpyAsync(vo.data(), p->vox_offs.ptr, (nf + 1) * 8,
                                   cudaMemcpyDeviceToHost, p->s_meta));
      RVP_CUDA_TRY(cudaStreamSynchronize(p->s_meta));
      if (pick(voxel_offsets, i)) memcpy(voxel_offsets[i], vo.data(), (nf + 1) * 8);
      RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_out, p->ev_stage[0], 0));
      d2h(pick(voxel_aos, i), p->vox_aos.ptr, (size_t)vo[nf] * 12);
      RVP_CUDA_TRY(cudaEventRecord(p->ev_dv, p->s_out));
      RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_meta, p->ev_stage[1], 0));
      RVP_CUDA_TRY(cudaMemcpyAsync(so.data(), p->sor_offs.ptr, (nf + 1) * 8,
                                   cudaMemcpyDeviceToHost, p->s_meta));
      RVP_CUDA_TRY(cudaStreamSynchronize(p->s_meta));
      const size_t ns = (size_t)so[nf];
      if (pick(sor_offsets, i)) memcpy(sor_offsets[i], so.data(), (nf + 1) * 8);
      RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_out, p->ev_stage[1], 0));
      d2h(pick(sor_aos, i), p->sor_aos.ptr, ns * 12);
      RVP_CUDA_TRY(cudaEventRecord(p->ev_ds, p->s_out));
      RVP_CUDA_TRY(cudaStreamWaitEvent(p->s_out, p->ev_end, 0));
      d2h(pick(nx, i), p->nx.ptr, ns * 4);
      d2h(pick(ny, i), p->ny.ptr, ns * 4);
      d2h(pick(nz, i), p->nz.ptr, ns * 4);
      d2h(pick(ransac_model, i), p->r_model.ptr, (size_t)nf * 16);
      d2h(pick(ransac_count, i), p->r_best.ptr, (size_t)nf * 4);
      RVP_CUDA_TRY(cudaEventRecord(p->ev_dn, p->s_out));
    });
  }
  const cudaError_t e1 = cudaStreamSynchronize(p->s_out);
  const cudaError_t e2 = cudaStreamSynchronize(st);
  const cudaError_t e3 = p->s_in ? cudaStreamSynchronize(p->s_in) : cudaSuccess;
  if (s == RVP_OK && (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)) {
    ctx->last_error = "batched host run: CUDA error";
    return RVP_ERR_CUDA;
  }
  return s;
}

rvp_status rvp_pipeline_copy_outputs(rvp_pipeline *p, float *voxel_aos, int64_t *voxel_offsets,
                                     float *sor_aos, int64_t *sor_offsets, float *nx, float *ny,
                                     float *nz, float *ransac_model, int32_t *ransac_count) {
  if (!p) return RVP_ERR_INVALID_ARG;
  rvp_context *ctx = p->ctx;
  return guard(ctx, [&] {
    const int n_frames = p->n_frames_last;
    RVP_REQUIRE(n_frames >= 1, "no run to copy");
    RVP_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    std::vector<int64_t> vo(n_frames + 1), so(n_frames + 1);
    RVP_CUDA_TRY(cudaMemcpyAsync(vo.data(), p->vox_offs.ptr, (n_frames + 1) * 8,
                                 cudaMemcpyDeviceToHost, st));
    RVP_CUDA_TRY(cudaMemcpyAsync(so.data(), p->sor_offs.ptr, (n_frames + 1) * 8,
                                 cudaMemcpyDeviceToHost, st));
    RVP_CUDA_TRY(cudaStreamSynchronize(st));
    const size_t nv = (size_t)vo[n_frames], ns = (size_t)so[n_frames];
    if (voxel_offsets) memcpy(voxel_offsets, vo.data(), (n_frames + 1) * 8);
    if (sor_offsets) memcpy(sor_offsets, so.data(), (n_frames + 1) * 8);
    auto d2h = [&](void *dst, const void *src, size_t b) {
      if (dst && b) RVP_CUDA_TRY(cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToHost, st));
    };
    d2h(voxel_aos, p->vox_aos.ptr, nv * 12);
    d2h(sor_aos, p->sor_aos.ptr, ns * 12);
    d2h(nx, p->nx.ptr, ns * 4);
    d2h(ny, p->ny.ptr, ns * 4);
    d2h(nz, p->nz.ptr, ns * 4);
    d2h(ransac_model, p->r_model.ptr, (size_t)n_frames * 16);
    d2h(ransac_count, p->r_best.ptr, (size_t)n_frames * 4);
    RVP_CUDA_TRY(cudaStreamSynchronize(st));
  });
}

}  // extern "C"
