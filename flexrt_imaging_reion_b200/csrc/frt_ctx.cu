// RT context: device memory, the step sequences (fused CUDA-graph step and the reference's
// individual step functions) and the C-ABI entry points declared in include/flexrt.h.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "frt_hostmath.h"
#include "frt_internal.cuh"
#include "frt_tune.h"

using namespace frt;

struct frt_ctx {
  frt_config cfg;
  std::vector<frt_box_desc> boxes;
  Dev d;
  std::vector<BoxP> hbox;
  std::vector<void*> allocs;
  cudaStream_t s_main = nullptr, s_dark = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_t0 = nullptr, ev_t1 = nullptr, ev_d0 = nullptr, ev_d1 = nullptr;
  cudaEvent_t ev_a0 = nullptr, ev_a1 = nullptr;   // around the walk (k_advance)
  static constexpr int kMaxTimedIter = 16;
  cudaEvent_t ev_r[2 * kMaxTimedIter] = {};   // around each ray pass of the step
  float last_raypass_ms = 0.f, last_walk_ms = 0.f;
  // I-front tracking: rounds of the last step (summed over its iterations), a budget that did not
  // settle, and the pinned word the round flag is read into
  static constexpr int kMaxFrontRounds = 4096;
  int if_rounds_last = 0;
  bool if_unsettled = false;
  int* h_flag = nullptr;
  // sources per box (host copy)
  std::vector<std::vector<int>> src_cell;
  std::vector<std::vector<double>> src_lum;
  std::vector<char> gas_ready;
  std::vector<char> restarted;           // gas read from a restart file (init_rt's restart branch)
  std::vector<float> restart_t;          // its time
  std::vector<std::vector<float>> rho;  // host copy of the proper density (set-up output)
  std::vector<std::vector<float>> rho_prev_h;   // the last hydro switch's density (host copy)
  std::vector<char> frac_kept;   // an expansion just kept the ionised fractions (d.frac_h2, frac_he2)
  std::vector<float> step_dt;    // the time step the last step ran with, per box
  std::vector<float> rot;
  // pinned staging
  uint16_t* h_ith_box = nullptr;
  uint16_t* h_ith_src = nullptr;
  Ctl* h_ctl = nullptr;
  cudaGraphExec_t graph = nullptr;
  bool graph_valid = false;
  long long phase_nlit = 0;   // lit cells of the current phased step (frt_step_phase)
  bool phase_async = false;   // phases only enqueue (frt_set_phase_async)
  uint8_t* src_own_buf = nullptr;
  int* chunk_buf = nullptr;   // per-chunk lit counts of the phased step
  frt_step_stats stats_scratch{};
  bool strict = false;
  int grid_rays = 0, grid_cells = 0, grid_lit = 0;
  int nsm = 148;
  std::string dev_name;
  Tune tune;               // launch shapes of the tunable kernels (frt_autotune / frt_set_tuning)
  bool tune_auto = false;  // frt_step follows the remembered shapes of the ray-count bucket
  frt_tuning tune_measured{};
  int grid_dark = 0;       // one block per 256 cells: short blocks that yield SM slots to the lit chain
  float last_step_ms = 0.f, last_dark_ms = 0.f;
  bool rays_moved = false;   // an advance, merge or split ran
  bool merged_any = false;   // a merge combined rays (a merged ray may mix the photons of several sources)
  bool cast_per_source = false;   // unbatched cast in the direct-launch step (comparison baseline)
  AdjDev adj{};
  bool adj_ready = false;
  bool adj_src_stale = true;   // the source-cell map of the adjoint follows the source list
  float* adj_out = nullptr;   // gather buffer of the adjoint's per-cell output (largest box)
  float last_adjoint_ms = 0.f;
  frt_step_stats last{};
  std::string err;
  // glibc rand() streams, one per box (srand(seed) semantics via initstate_r / random_r)
  std::vector<std::vector<char>> rng_state;
  std::vector<struct random_data> rng;
  std::vector<uint16_t> draw_box, draw_src;
};

namespace {

#define CK(x)                                                                          \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) {                                                           \
      ctx->err = std::string(#x) + ": " + cudaGetErrorString(e_);                      \
      return FRT_ERR_CUDA;                                                             \
    }                                                                                  \
  } while (0)

// Copies and fills on the step stream. The library's streams are non-blocking, so they do not
// wait for the legacy default stream: a plain cudaMemcpy from pageable memory or a cudaMemset
// may still be in flight when a kernel on s_main reads the buffer. Each helper returns once the
// operation has completed, in order with the work already queued on s_main.
cudaError_t copy_sync(frt_ctx* ctx, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, ctx->s_main);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(ctx->s_main);
}
cudaError_t fill_sync(frt_ctx* ctx, void* dst, int value, size_t bytes) {
  cudaError_t e = cudaMemsetAsync(dst, value, bytes, ctx->s_main);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(ctx->s_main);
}

template <typename T>
frt_status dalloc(frt_ctx* ctx, T** p, size_t n) {
  *p = nullptr;
  if (n == 0) return FRT_OK;
  void* q = nullptr;
  CK(cudaMalloc(&q, n * sizeof(T)));
  CK(fill_sync(ctx, q, 0, n * sizeof(T)));
  ctx->allocs.push_back(q);
  *p = (T*)q;
  return FRT_OK;
}

#define AL(ptr, n)                                   \
  do {                                               \
    frt_status st_ = dalloc(ctx, &(ptr), (size_t)(n)); \
    if (st_ != FRT_OK) return st_;                   \
  } while (0)

frt_status upload_boxes(frt_ctx* ctx) {
  CK(copy_sync(ctx, ctx->d.box, ctx->hbox.data(), sizeof(BoxP) * ctx->hbox.size(), cudaMemcpyHostToDevice));
  return FRT_OK;
}
frt_status download_boxes(frt_ctx* ctx) {
  CK(copy_sync(ctx, ctx->hbox.data(), ctx->d.box, sizeof(BoxP) * ctx->hbox.size(), cudaMemcpyDeviceToHost));
  return FRT_OK;
}

frt_status check_box(frt_ctx* ctx, int box) {
  if (!ctx || box < 0 || box >= (int)ctx->boxes.size()) {
    if (ctx) ctx->err = "box index out of range";
    return FRT_ERR_INVALID;
  }
  return FRT_OK;
}

frt_status sync_and_check(frt_ctx* ctx) {
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(cudaStreamSynchronize(ctx->s_dark));
  CK(cudaGetLastError());
  Ctl c;
  CK(copy_sync(ctx, &c, ctx->d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
  if (c.err) {
    ctx->err = "device error flags " + std::to_string(c.err) +
               " (1 ray pool full, 2 path_length exceeded, 4 lit-cell list full)";
    return FRT_ERR_CAPACITY;
  }
  return FRT_OK;
}

// Rebuild the concatenated source arrays of all boxes (box order, then (i,j,k) order).
frt_status upload_sources(frt_ctx* ctx) {
  std::vector<int> cell;
  std::vector<uint16_t> box;
  std::vector<double> lum;
  std::vector<float> rdt;
  for (size_t b = 0; b < ctx->boxes.size(); b++)
    for (size_t s = 0; s < ctx->src_cell[b].size(); s++) {
      cell.push_back(ctx->src_cell[b][s]);
      box.push_back((uint16_t)b);
      lum.push_back(ctx->src_lum[b][s]);
      rdt.push_back(0.f);
    }
  const int n = (int)cell.size();
  if (n > ctx->d.src_cap) {
    ctx->err = "more sources than src_capacity";
    return FRT_ERR_CAPACITY;
  }
  ctx->d.nsrc = n;
  // an owner mask (frt_set_source_owner) describes the previous source list: drop it, so that no
  // kernel reads owner bytes that were never written for the new sources (all sources are cast
  // until the caller sets a mask for the new list)
  ctx->d.src_own = nullptr;
  ctx->adj_src_stale = true;
  if (n) {
    CK(copy_sync(ctx, ctx->d.src_cell, cell.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    CK(copy_sync(ctx, ctx->d.src_box, box.data(), sizeof(uint16_t) * n, cudaMemcpyHostToDevice));
    CK(copy_sync(ctx, ctx->d.src_lum, lum.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    CK(copy_sync(ctx, ctx->d.src_ray_dt, rdt.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  }
  ctx->graph_valid = false;
  return FRT_OK;
}

// ---- step sequences ---------------------------------------------------------------------------
// Host bookkeeping of a step about to run: its time step per box (get_nphot_min_max at a hydro
// switch after it uses it), and the fractions an expansion kept are stale once cells update.
void note_step(frt_ctx* ctx) {
  for (size_t b = 0; b < ctx->hbox.size(); b++) ctx->step_dt[b] = ctx->hbox[b].dt;
  std::fill(ctx->frac_kept.begin(), ctx->frac_kept.end(), 0);
}

// The sub-grid model's cell passes take the tuned cell-pass grid, or 8 blocks per SM where that
// grid is the resident count (which only the plain cell passes resolve)
int sg_cell_grid(const frt_ctx* ctx) { return ctx->nsm * (ctx->tune.lit_grid > 0 ? ctx->tune.lit_grid : 8); }

void record(cudaEvent_t e, cudaStream_t s, bool in_graph) {
  if (in_graph) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
  else cudaEventRecord(e, s);
}

void enqueue_begin_advance(frt_ctx* ctx, bool in_graph = false) {
  ctx->rays_moved = true;
  const Dev& d = ctx->d;
  launch_clear_lit(d, ctx->grid_lit, ctx->s_main);
  launch_step_begin(d, ctx->s_main);
  if (d.subgrid) launch_sg_step(d, ctx->s_main);
  record(ctx->ev_a0, ctx->s_main, in_graph);
  launch_walk(d, ctx->nsm * ctx->tune.adv_grid, ctx->s_main, ctx->tune.adv_block, 0, INT_MAX);
  record(ctx->ev_a1, ctx->s_main, in_graph);
  launch_lit_number(d, ctx->grid_rays, ctx->s_main);   // lit cells numbered, moved rays packed
}

// The C2Ray iterations with I-front tracking: per iteration, rounds of (ray pass, budget pass)
// until no front cell's sums change (the host reads the flag after each round), then for the
// last iteration the pass that updates the rays, and the cell pass. Launched directly (the number
// of rounds is known only on the host), never inside a graph.
void enqueue_iterations_ifront(frt_ctx* ctx, bool fused_thermal) {
  Dev& d = ctx->d;
  cudaStream_t s = ctx->s_main;
  const int grid = ctx->grid_lit;
  launch_sg_lit_init(d, grid, s);
  launch_if_lists(d, grid, s);
  ctx->if_rounds_last = 0;
  for (int it = 0; it < d.itercount; it++) {
    bool settled = false;
    for (int round = 0; round < frt_ctx::kMaxFrontRounds; round++) {
      cudaMemsetAsync(&d.ctl->if_changed, 0, sizeof(int), s);
      launch_if_round(d, it, grid, s);
      cudaMemcpyAsync(ctx->h_flag, &d.ctl->if_changed, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (cudaStreamSynchronize(s) != cudaSuccess) return;   // (the step's status check reports it)
      ctx->if_rounds_last += 1;
      if (*ctx->h_flag == 0) {
        settled = true;
        break;
      }
    }
    if (!settled) ctx->if_unsettled = true;
    if (it == d.itercount - 1) launch_if_final(d, it, grid, s);
    launch_sg_litpass(d, it, fused_thermal, sg_cell_grid(ctx), s);
  }
}

void enqueue_iterations(frt_ctx* ctx, bool fused_thermal, bool in_graph = false) {
  const Dev& d = ctx->d;
  if (d.subgrid && d.ifront) {   // I-front tracking: the budget rounds of every C2Ray iteration
    enqueue_iterations_ifront(ctx, fused_thermal);
    return;
  }
  if (d.subgrid) {   // the sub-grid model's passes (frt_subgrid.cu)
    launch_sg_lit_init(d, ctx->grid_lit, ctx->s_main);
    for (int it = 0; it < d.itercount; it++) {
      const bool timed = it < frt_ctx::kMaxTimedIter;
      if (timed) record(ctx->ev_r[2 * it], ctx->s_main, in_graph);
      launch_sg_raypass(d, it, ctx->grid_rays, ctx->s_main);
      if (timed) record(ctx->ev_r[2 * it + 1], ctx->s_main, in_graph);
      launch_sg_litpass(d, it, fused_thermal, sg_cell_grid(ctx), ctx->s_main);
    }
    return;
  }
  launch_lit_init(d, ctx->strict, ctx->grid_lit, ctx->s_main);
  for (int it = 0; it < d.itercount; it++) {
    const bool timed = it < frt_ctx::kMaxTimedIter;
    if (timed) record(ctx->ev_r[2 * it], ctx->s_main, in_graph);
    launch_raypass(d, it, ctx->strict, ctx->nsm * ctx->tune.rp_grid, ctx->s_main, ctx->tune.rp_block,
                   ctx->tune.rp_chunk);
    if (timed) record(ctx->ev_r[2 * it + 1], ctx->s_main, in_graph);
    launch_litpass(d, it, ctx->strict, fused_thermal, ctx->nsm * ctx->tune.lit_grid, ctx->s_main);
  }
}

// The whole step of main.cc:108-264 (fixed redshift): the dark-cell pass runs on a second
// stream concurrently with the lit-cell iteration and the ray life-cycle kernels.
void enqueue_step(frt_ctx* ctx, bool in_graph) {
  const Dev& d = ctx->d;
  cudaStream_t s = ctx->s_main;
  cudaMemcpyAsync(d.itheta_merge, ctx->h_ith_box, sizeof(uint16_t) * d.nbox, cudaMemcpyHostToDevice, s);
  if (d.nsrc) cudaMemcpyAsync(d.src_itheta, ctx->h_ith_src, sizeof(uint16_t) * d.nsrc, cudaMemcpyHostToDevice, s);
  enqueue_begin_advance(ctx, in_graph);
  cudaEventRecord(ctx->ev_fork, s);
  cudaStreamWaitEvent(ctx->s_dark, ctx->ev_fork, 0);
  if (in_graph) cudaEventRecordWithFlags(ctx->ev_d0, ctx->s_dark, cudaEventRecordExternal);
  else cudaEventRecord(ctx->ev_d0, ctx->s_dark);
  if (d.subgrid) launch_sg_dark(d, true, ctx->grid_dark, ctx->s_dark);
  else launch_dark(d, ctx->strict, true, ctx->grid_dark, ctx->s_dark);
  if (in_graph) cudaEventRecordWithFlags(ctx->ev_d1, ctx->s_dark, cudaEventRecordExternal);
  else cudaEventRecord(ctx->ev_d1, ctx->s_dark);
  cudaEventRecord(ctx->ev_join, ctx->s_dark);
  enqueue_iterations(ctx, true, in_graph);
  launch_count_merge(d, ctx->grid_rays, s);
  launch_split_compact(d, ctx->nsm * ctx->tune.split_grid, s);
  cudaStreamWaitEvent(s, ctx->ev_join, 0);
  if (!in_graph && ctx->cast_per_source) launch_cast_per_source(d, s);
  else launch_cast(d, s);
  cudaMemcpyAsync(ctx->h_ctl, d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
}

void fill_stats(frt_ctx* ctx, const Ctl& c, frt_step_stats* st) {
  frt_step_stats o{};
  o.rays_alive = c.nray[c.cur];
  o.rays_moved = c.rays_moved;
  o.crossings = c.crossings;
  o.lit_cells = c.n_lit;
  o.rays_split = c.split;
  o.rays_merged = c.merged;
  o.rays_killed = c.killed;
  o.rays_cast = c.cast;
  o.photons_emitted = c.emitted;
  o.photons_deposited = c.deposited;
  o.photons_killed = c.killed_ph;
  o.photons_overlap = c.overlap;
  o.photons_in_flight = c.in_flight;
  o.t = ctx->hbox.empty() ? 0.0 : 0.0;
  o.dt = ctx->hbox.empty() ? 0.0 : (double)ctx->hbox[0].dt;
  o.error_flags = c.err;
  ctx->last = o;
  if (st) *st = o;
}

frt_status stage_itheta(frt_ctx* ctx, const uint16_t* ith_box, const uint16_t* ith_src) {
  for (int b = 0; b < ctx->d.nbox; b++) {
    const uint16_t v = ith_box ? ith_box[b] : 0;
    if (v >= kNtheta) {
      ctx->err = "itheta out of range";
      return FRT_ERR_INVALID;
    }
    ctx->h_ith_box[b] = v;
  }
  for (int s = 0; s < ctx->d.nsrc; s++) {
    const uint16_t v = ith_src ? ith_src[s] : 0;
    if (v >= kNtheta) {
      ctx->err = "itheta out of range";
      return FRT_ERR_INVALID;
    }
    ctx->h_ith_src[s] = v;
  }
  return FRT_OK;
}

int si_rand(frt_ctx* ctx, int b) {
  int32_t v = 0;
  random_r(&ctx->rng[b], &v);
  return v % kNtheta;
}

frt_status draw(frt_ctx* ctx, uint16_t* ith_box, uint16_t* ith_src) {
  if (ctx->rng.size() != ctx->boxes.size()) {
    ctx->err = "frt_seed_boxes not called";
    return FRT_ERR_STATE;
  }
  // per box: the merge draw first, then one per source of that box (the sources of all boxes
  // are concatenated in box order)
  std::vector<size_t> off(ctx->boxes.size() + 1, 0);
  for (size_t b = 0; b < ctx->boxes.size(); b++) off[b + 1] = off[b] + ctx->src_cell[b].size();
  for (size_t b = 0; b < ctx->boxes.size(); b++) {
    if (ith_box) ith_box[b] = (uint16_t)si_rand(ctx, (int)b);
    if (ith_src)
      for (size_t s = off[b]; s < off[b + 1]; s++) ith_src[s] = (uint16_t)si_rand(ctx, (int)b);
  }
  return FRT_OK;
}

frt_status finish_step(frt_ctx* ctx, frt_step_stats* stats) {
  CK(cudaEventSynchronize(ctx->ev_t1));
  CK(cudaStreamSynchronize(ctx->s_dark));
  CK(cudaGetLastError());
  float ms = 0.f, dms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev_t0, ctx->ev_t1));
  if (cudaEventElapsedTime(&dms, ctx->ev_d0, ctx->ev_d1) != cudaSuccess) {
    cudaGetLastError();
    dms = -1.f;
  }
  ctx->last_step_ms = ms;
  ctx->last_dark_ms = dms;
  float rms = 0.f;
  for (int it = 0; it < std::min(ctx->d.itercount, (int)frt_ctx::kMaxTimedIter); it++) {
    float x = 0.f;
    if (cudaEventElapsedTime(&x, ctx->ev_r[2 * it], ctx->ev_r[2 * it + 1]) != cudaSuccess) {
      cudaGetLastError();
      rms = -1.f;
      break;
    }
    rms += x;
  }
  ctx->last_raypass_ms = rms;
  float ams = 0.f;
  if (cudaEventElapsedTime(&ams, ctx->ev_a0, ctx->ev_a1) != cudaSuccess) {
    cudaGetLastError();
    ams = -1.f;
  }
  ctx->last_walk_ms = ams;
  if (ctx->h_ctl->merged > 0) ctx->merged_any = true;
  fill_stats(ctx, *ctx->h_ctl, stats);
  if (ctx->if_unsettled) {
    ctx->if_unsettled = false;
    ctx->err = "I-front photon budgets did not settle within " + std::to_string(frt_ctx::kMaxFrontRounds) +
               " rounds in a C2Ray iteration";
    return FRT_ERR_STATE;
  }
  if (ctx->h_ctl->err) {
    ctx->err = "device error flags " + std::to_string(ctx->h_ctl->err) +
               " (1 ray pool full, 2 path_length exceeded, 4 lit-cell list full)";
    return FRT_ERR_CAPACITY;
  }
  return FRT_OK;
}

}  // namespace

extern "C" {

const char* frt_last_error(const frt_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

frt_status frt_create(const frt_config* cfg, frt_ctx** out) {
  if (!cfg || !out || cfg->nbox < 1 || !cfg->boxes || cfg->nfreq < 1 || cfg->nfreq > FRT_MAX_FREQ ||
      cfg->path_length < 2 || cfg->path_length > FRT_MAX_PATH || cfg->itercount < 1 || cfg->ray_capacity < 1 ||
      cfg->hpx_lvl < 0 || cfg->hpx_lvl > 6 || cfg->nbox > 65535)
    return FRT_ERR_INVALID;
  frt_ctx* ctx = new frt_ctx();
  *out = ctx;
  ctx->cfg = *cfg;
  ctx->boxes.assign(cfg->boxes, cfg->boxes + cfg->nbox);
  ctx->cfg.boxes = ctx->boxes.data();
  ctx->strict = cfg->precision == FRT_PREC_STRICT;
  CK(cudaSetDevice(cfg->device));
  int nsm = 148;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, cfg->device));
  ctx->nsm = nsm;
  {
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, cfg->device));
    ctx->dev_name = prop.name;
  }
  ctx->grid_rays = nsm * 8;
  ctx->grid_cells = nsm * 8;
  ctx->grid_lit = nsm * 8;
  // The lit-cell chain is the step's critical path; the dark-cell pass on its own stream only
  // has to end before the join. With the chain's stream at the highest priority the block
  // scheduler hands freed SM slots to the chain first and the dark pass fills the rest.
  int prio_least = 0, prio_greatest = 0;
  CK(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
  CK(cudaStreamCreateWithPriority(&ctx->s_main, cudaStreamNonBlocking, prio_greatest));
  CK(cudaStreamCreateWithPriority(&ctx->s_dark, cudaStreamNonBlocking, prio_least));
  CK(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  CK(cudaEventCreate(&ctx->ev_t0));
  CK(cudaEventCreate(&ctx->ev_t1));
  CK(cudaEventCreate(&ctx->ev_d0));
  CK(cudaEventCreate(&ctx->ev_d1));
  CK(cudaEventCreate(&ctx->ev_a0));
  CK(cudaEventCreate(&ctx->ev_a1));
  for (cudaEvent_t& e : ctx->ev_r) CK(cudaEventCreate(&e));

  Dev& d = ctx->d;
  memset(&d, 0, sizeof(d));
  d.nbox = cfg->nbox;
  d.F = cfg->nfreq;
  d.PL = cfg->path_length;
  d.itercount = cfg->itercount;
  d.hpx_lvl = cfg->hpx_lvl;
  d.outputs = cfg->outputs;
  d.nhe_to_nh = (0.246 / 4.) / (1. - 0.246);
  d.const_clump = cfg->const_clump;
  // boxes: tile-aligned concatenation
  ctx->hbox.resize(cfg->nbox);
  long long off = 0;
  for (int b = 0; b < cfg->nbox; b++) {
    const frt_box_desc& bd = cfg->boxes[b];
    if (bd.n < 2 || bd.n > 1024 || !(bd.cl_factor > 0.f)) {
      ctx->err = "bad box description";
      return FRT_ERR_INVALID;
    }
    host::box_params(&ctx->hbox[b], &ctx->cfg, &bd, off);
    off += ((ctx->hbox[b].ncell + kTile - 1) / kTile) * kTile;
  }
  d.ncell_total = off;
  ctx->grid_dark = (int)std::min<long long>((off + 255) / 256, 1LL << 30);
  d.ntile = off / kTile;
  if (off >= (1LL << 31)) {
    ctx->err = "too many cells for 32-bit cell indices";
    return FRT_ERR_INVALID;
  }
  // packed segment offsets are 32-bit: ray_cap * path_length stays below 2^31
  d.ray_cap = (int)std::min<long long>(cfg->ray_capacity, ((1LL << 31) - 64) / d.PL);
  long long lc = cfg->lit_capacity > 0 ? cfg->lit_capacity : off;
  lc = std::min<long long>(lc, std::min<long long>(off, (long long)d.ray_cap * d.PL));
  d.lit_cap = (int)std::max<long long>(lc, 1024);
  d.src_cap = (int)std::max<long long>(cfg->src_capacity, 1);
  // spectrum / cross sections
  for (int nu = 0; nu < FRT_MAX_FREQ; nu++) d.spectrum[nu] = nu < d.F ? cfg->spectrum[nu] : 0.f;
  host::derived_constants(&ctx->cfg, d.sigH1_d, d.sigHe1_d, &d.sigH1_0, &d.sigH1_912, &d.pi_sf_3, &d.log4);
  for (int nu = 0; nu < d.F; nu++) {
    d.sigH1_f[nu] = (float)d.sigH1_d[nu];
    d.sigHe1_f[nu] = (float)d.sigHe1_d[nu];
    d.sigH1_l2[nu] = (float)(d.sigH1_d[nu] * 1.4426950408889634);
    d.sigHe1_l2[nu] = (float)(d.sigHe1_d[nu] * 1.4426950408889634);
  }
  d.nho = 0;
  while (d.nho < d.F && d.sigHe1_f[d.nho] == 0.f) d.nho++;
  // device memory
  AL(d.box, cfg->nbox);
  AL(d.count, cfg->nbox);
  AL(d.need_hist, cfg->nbox);
  AL(d.hist, (size_t)cfg->nbox * kPdfBins);
  AL(d.itheta_merge, cfg->nbox);
  AL(d.lg, 2 * cfg->nbox);
  {
    ctx->rot.resize((size_t)kNtheta * 18);
    host::rotation_table(ctx->rot.data());
    float* r = nullptr;
    AL(r, ctx->rot.size());
    CK(copy_sync(ctx, r, ctx->rot.data(), sizeof(float) * ctx->rot.size(), cudaMemcpyHostToDevice));
    d.rot = r;
    float4* pt = nullptr;
    AL(pt, (size_t)pix_tab_offset(kPixTabMax + 1));
    launch_pix_table(pt, ctx->s_main);
    d.pix_tab = pt;
  }
  {
    std::vector<int16_t> tb(d.ntile, (int16_t)-1);
    for (int b = 0; b < cfg->nbox; b++) {
      const long long t0 = ctx->hbox[b].cell0 >> kTileShift;
      const long long nt = (ctx->hbox[b].ncell + kTile - 1) / kTile;
      for (long long t = t0; t < t0 + nt; t++) tb[t] = (int16_t)b;
    }
    AL(d.tile_box, d.ntile);
    CK(copy_sync(ctx, d.tile_box, tb.data(), sizeof(int16_t) * d.ntile, cudaMemcpyHostToDevice));
  }
  const size_t NC = (size_t)off;
  AL(d.nH, NC); AL(d.nHe, NC); AL(d.nH1, NC); AL(d.nHe1, NC); AL(d.f_H1, NC); AL(d.f_He1, NC);
  AL(d.temp, NC); AL(d.ne, NC); AL(d.heat, NC); AL(d.cool, NC); AL(d.avg_nh1, NC); AL(d.avg_nhe1, NC);
  AL(d.treion, NC); AL(d.treion_flag, NC); AL(d.lit_flag, NC); AL(d.lit_slot, NC);
  AL(d.nH1_prev, NC); AL(d.n_tot, NC); AL(d.dne_dt, NC);
  d.clump = nullptr;
  if (cfg->outputs == FRT_OUT_DIAG) {
    AL(d.rec_h2, NC); AL(d.rec_he2, NC); AL(d.recrate_h2, NC); AL(d.recrate_he2, NC);
    AL(d.mfp, NC); AL(d.mfp912, NC); AL(d.if_speed, NC); AL(d.inc_flux, NC);
  }
  launch_fill_i32(d.lit_slot, -1, (long long)NC, ctx->s_main);
  const size_t L = (size_t)d.lit_cap;
  AL(d.l_cell, L); AL(d.l_box, L); AL(d.l_nh, L); AL(d.l_nhe, L); AL(d.l_y0h, L); AL(d.l_y0he, L); AL(d.l_crec_h, L);
  AL(d.l_crec_he, L); AL(d.l_rec_h2, L); AL(d.l_rec_he2, L); AL(d.l_avg, L);
  AL(d.l_nh1_old, L); AL(d.l_acc, L);
  d.per_bin = (ctx->strict || cfg->outputs == FRT_OUT_DIAG) ? 1 : 0;
  AL(d.l_heat, L);
  if (d.per_bin) {
    AL(d.l_ngam, L * d.F);
    AL(d.l_acc_nu_h, L * d.F);
    AL(d.l_acc_nu_he, L * d.F);
  }
  for (int nu = 0; nu < FRT_MAX_FREQ; nu++) {
    d.cH1_f[nu] = ctx->hbox[0].th.cH1[nu];
    d.cHe1_f[nu] = ctx->hbox[0].th.cHe1[nu];
  }
  const size_t R = (size_t)d.ray_cap;
  for (int p = 0; p < 2; p++) {
    RayPool& P = d.pool[p];
    AL(P.cell, R); AL(P.box, R); AL(P.order, R); AL(P.pixel, R); AL(P.itheta, R);
    AL(P.xh, R); AL(P.yh, R); AL(P.zh, R); AL(P.nphot, R * d.F);
    AL(P.r, R); AL(P.dr, R); AL(P.x, R); AL(P.y, R); AL(P.z, R); AL(P.time, R);
  }
  AL(d.dead, R);
  AL(d.pk, R * d.PL); AL(d.mv_hdr, R);
  // merge bins only when some box can reach its merge threshold with this pool size
  bool merge_reachable = false;
  for (int b = 0; b < cfg->nbox; b++) merge_reachable |= ctx->hbox[b].num_thresh < (long long)d.ray_cap;
  if (merge_reachable) {
    const long long npix = 12LL << (2 * cfg->hpx_lvl);
    if ((long long)NC * npix >= (1LL << 31)) {
      ctx->err = "merge bin table exceeds 32-bit indices";
      return FRT_ERR_INVALID;
    }
    AL(d.bin_base, NC * npix);
    launch_fill_i32(d.bin_base, 0x7fffffff, (long long)NC * npix, ctx->s_main);
    AL(d.ray_bin, R);
    launch_fill_i32(d.ray_bin, -1, (long long)R, ctx->s_main);
    AL(d.merged_flag, R);
  }
  AL(d.src_cell, d.src_cap); AL(d.src_box, d.src_cap); AL(d.src_lum, d.src_cap); AL(d.src_ray_dt, d.src_cap); AL(d.src_pos, d.src_cap);
  AL(d.src_itheta, d.src_cap);
  AL(d.ctl, 1);
  AL(d.rp_queue, kMaxIterQueue);
  CK(cudaMallocHost(&ctx->h_ith_box, sizeof(uint16_t) * cfg->nbox));
  CK(cudaMallocHost(&ctx->h_ith_src, sizeof(uint16_t) * d.src_cap));
  CK(cudaMallocHost(&ctx->h_ctl, sizeof(Ctl)));
  memset(ctx->h_ctl, 0, sizeof(Ctl));
  ctx->src_cell.resize(cfg->nbox);
  ctx->src_lum.resize(cfg->nbox);
  ctx->gas_ready.assign(cfg->nbox, 0);
  ctx->rho_prev_h.resize(cfg->nbox);
  ctx->frac_kept.assign(cfg->nbox, 0);
  ctx->step_dt.assign(cfg->nbox, 0.f);
  ctx->restarted.assign(cfg->nbox, 0);
  ctx->restart_t.assign(cfg->nbox, 0.f);
  ctx->rho.resize(cfg->nbox);
  {
    frt_status st = upload_boxes(ctx);
    if (st) return st;
  }
  CK(cudaStreamSynchronize(ctx->s_main));
  return FRT_OK;
}

frt_status frt_destroy(frt_ctx* ctx) {
  if (!ctx) return FRT_OK;
  if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
  for (void* p : ctx->allocs) cudaFree(p);
  if (ctx->h_ith_box) cudaFreeHost(ctx->h_ith_box);
  if (ctx->h_ith_src) cudaFreeHost(ctx->h_ith_src);
  if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
  if (ctx->h_flag) cudaFreeHost(ctx->h_flag);
  for (cudaEvent_t e : ctx->ev_r)
    if (e) cudaEventDestroy(e);
  cudaEvent_t evs[] = {ctx->ev_fork, ctx->ev_join, ctx->ev_t0, ctx->ev_t1, ctx->ev_d0, ctx->ev_d1, ctx->ev_a0, ctx->ev_a1};
  for (cudaEvent_t e : evs)
    if (e) cudaEventDestroy(e);
  if (ctx->s_main) cudaStreamDestroy(ctx->s_main);
  if (ctx->s_dark) cudaStreamDestroy(ctx->s_dark);
  delete ctx;
  return FRT_OK;
}

frt_status frt_build_rotation_table(float* out) {
  if (!out) return FRT_ERR_INVALID;
  host::rotation_table(out);
  return FRT_OK;
}

frt_status frt_rotation_table(const frt_ctx* ctx, float* out) {
  if (!ctx || !out) return FRT_ERR_INVALID;
  memcpy(out, ctx->rot.data(), sizeof(float) * ctx->rot.size());
  return FRT_OK;
}

frt_status frt_init_gas(frt_ctx* ctx, int box, const float* delta1) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  if (!delta1) return FRT_ERR_INVALID;
  const BoxP& B = ctx->hbox[box];
  const size_t n = (size_t)B.ncell;
  std::vector<float> rho(n), nH(n), nHe(n), nH1(n), nHe1(n), fH1(n), fHe1(n), temp(n), ne(n), ntot(n), rh(n), rhe(n),
      dne(n);
  host::GasInit g{rho.data(), nH.data(), nHe.data(), nH1.data(), nHe1.data(), fH1.data(), fHe1.data(), temp.data(),
                  ne.data(), ntot.data(), rh.data(), rhe.data(), dne.data()};
  host::init_gas(&ctx->cfg, &ctx->boxes[box], delta1, &g);
  Dev& d = ctx->d;
  const size_t o = (size_t)B.cell0;
  auto up = [&](float* dst, const std::vector<float>& src) {
    return copy_sync(ctx, dst + o, src.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
  };
  CK(up(d.nH, nH)); CK(up(d.nHe, nHe)); CK(up(d.nH1, nH1)); CK(up(d.nHe1, nHe1)); CK(up(d.f_H1, fH1));
  CK(up(d.f_He1, fHe1)); CK(up(d.temp, temp)); CK(up(d.ne, ne)); CK(up(d.avg_nh1, nH1)); CK(up(d.avg_nhe1, nHe1));
  CK(up(d.n_tot, ntot)); CK(up(d.dne_dt, dne)); CK(up(d.nH1_prev, nH1));
  CK(fill_sync(ctx, d.heat + o, 0, sizeof(float) * n));
  CK(fill_sync(ctx, d.cool + o, 0, sizeof(float) * n));
  CK(fill_sync(ctx, d.treion + o, 0, sizeof(float) * n));
  CK(fill_sync(ctx, d.treion_flag + o, 0, n));
  if (d.rec_h2) {
    CK(up(d.rec_h2, rh));
    CK(up(d.rec_he2, rhe));
  }
  if (d.rho) CK(up(d.rho, rho));
  ctx->rho[box] = rho;
  ctx->gas_ready[box] = 1;
  ctx->restarted[box] = 0;
  {
    // <rho> of the snapshot (get_ugas, io_funcs.cc:61, then a^-3, gas_funcs.cc:613)
    std::vector<float> tmp(n);
    host::snapshot_rho(B.n, delta1, (float)(1. / (1. + ctx->boxes[box].zz)), tmp.data(), &ctx->hbox[box].avg_rho);
  }
  ctx->rho_prev_h[box].clear();
  return upload_boxes(ctx);
}

frt_status frt_set_sources(frt_ctx* ctx, int box, int nsrc, const int32_t* ijk, const double* lum) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  if (nsrc < 0 || (nsrc > 0 && (!ijk || !lum))) return FRT_ERR_INVALID;
  const int n = ctx->hbox[box].n;
  ctx->src_cell[box].clear();
  ctx->src_lum[box].clear();
  for (int s = 0; s < nsrc; s++) {
    const int i = ijk[3 * s], j = ijk[3 * s + 1], k = ijk[3 * s + 2];
    if (i < 0 || j < 0 || k < 0 || i >= n || j >= n || k >= n) {
      ctx->err = "source cell out of range";
      return FRT_ERR_INVALID;
    }
    ctx->src_cell[box].push_back((i * n + j) * n + k);
    ctx->src_lum[box].push_back(lum[s]);
  }
  return upload_sources(ctx);
}

frt_status frt_set_clump_field(frt_ctx* ctx, int box, const float* clump) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  Dev& d = ctx->d;
  if (!d.clump) {
    if (!clump) return FRT_OK;
    AL(d.clump, (size_t)d.ncell_total);
    // cells of other boxes keep the constant
    std::vector<float> c(d.ncell_total, ctx->cfg.const_clump);
    CK(copy_sync(ctx, d.clump, c.data(), sizeof(float) * c.size(), cudaMemcpyHostToDevice));
    ctx->graph_valid = false;
  }
  const BoxP& B = ctx->hbox[box];
  if (clump) {
    CK(copy_sync(ctx, d.clump + B.cell0, clump, sizeof(float) * B.ncell, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> c(B.ncell, ctx->cfg.const_clump);
    CK(copy_sync(ctx, d.clump + B.cell0, c.data(), sizeof(float) * B.ncell, cudaMemcpyHostToDevice));
  }
  return FRT_OK;
}

static float* field_ptr(frt_ctx* ctx, frt_field f) {
  Dev& d = ctx->d;
  switch (f) {
    case FRT_F_NH: return d.nH;
    case FRT_F_NHE: return d.nHe;
    case FRT_F_NH1: return d.nH1;
    case FRT_F_NHE1: return d.nHe1;
    case FRT_F_NE: return d.ne;
    case FRT_F_F_H1: return d.f_H1;
    case FRT_F_F_HE1: return d.f_He1;
    case FRT_F_TEMP: return d.temp;
    case FRT_F_CLUMP: return d.clump;
    case FRT_F_AVG_NH1: return d.avg_nh1;
    case FRT_F_AVG_NHE1: return d.avg_nhe1;
    case FRT_F_HEAT_RATE: return d.heat;
    case FRT_F_COOL_RATE: return d.cool;
    case FRT_F_TREION: return d.treion;
    case FRT_F_DNE_DT: return d.dne_dt;
    case FRT_F_N_TOT: return d.n_tot;
    case FRT_F_RECOMB_H2: return d.rec_h2;
    case FRT_F_RECOMB_HE2: return d.rec_he2;
    case FRT_F_RECRATE_H2: return d.recrate_h2;
    case FRT_F_RECRATE_HE2: return d.recrate_he2;
    case FRT_F_MFP: return d.mfp;
    case FRT_F_MFP_912: return d.mfp912;
    case FRT_F_IF_SPEED: return d.if_speed;
    case FRT_F_INC_FLUX: return d.inc_flux;
    default: return nullptr;
  }
}

frt_status frt_set_field(frt_ctx* ctx, int box, frt_field f, const float* host) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  if (!host) return FRT_ERR_INVALID;
  if (f == FRT_F_CLUMP) return frt_set_clump_field(ctx, box, host);
  float* p = field_ptr(ctx, f);
  if (!p) {
    ctx->err = "field is not settable";
    return FRT_ERR_INVALID;
  }
  const BoxP& B = ctx->hbox[box];
  CK(copy_sync(ctx, p + B.cell0, host, sizeof(float) * B.ncell, cudaMemcpyHostToDevice));
  return FRT_OK;
}

frt_status frt_get_field(frt_ctx* ctx, int box, frt_field f, float* host) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  if (!host) return FRT_ERR_INVALID;
  Dev& d = ctx->d;
  const BoxP& B = ctx->hbox[box];
  const size_t n = (size_t)B.ncell;
  const int F = d.F;
  auto get = [&](const float* src, float* dst) {
    return copy_sync(ctx, dst, src + B.cell0, sizeof(float) * n, cudaMemcpyDeviceToHost);
  };
  auto sparse = [&](int which, float* dst) -> frt_status {
    float* tmp = nullptr;
    CK(cudaMalloc(&tmp, sizeof(float) * n));
    launch_gather_sparse(d, B.cell0, (long long)n, which, tmp, ctx->s_main);
    CK(cudaStreamSynchronize(ctx->s_main));
    CK(copy_sync(ctx, dst, tmp, sizeof(float) * n, cudaMemcpyDeviceToHost));
    CK(cudaFree(tmp));
    return FRT_OK;
  };
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(cudaStreamSynchronize(ctx->s_dark));
  switch (f) {
    case FRT_F_RHO:
      if (d.rho) {   // moved to the device by a cosmological expansion
        CK(get(d.rho, host));
        return FRT_OK;
      }
      if (ctx->rho[box].size() != n) return FRT_ERR_STATE;
      memcpy(host, ctx->rho[box].data(), sizeof(float) * n);
      return FRT_OK;
    case FRT_F_CLUMP:
      if (!d.clump) {
        for (size_t i = 0; i < n; i++) host[i] = ctx->cfg.const_clump;
        return FRT_OK;
      }
      CK(get(d.clump, host));
      return FRT_OK;
    case FRT_F_NH2:
    case FRT_F_NHE2:
    case FRT_F_F_H2:
    case FRT_F_F_HE2: {
      const bool h = (f == FRT_F_NH2 || f == FRT_F_F_H2);
      std::vector<float> a(n), b(n);
      CK(get(h ? d.nH : d.nHe, a.data()));
      CK(get(h ? d.nH1 : d.nHe1, b.data()));
      const bool frac = (f == FRT_F_F_H2 || f == FRT_F_F_HE2);
      for (size_t i = 0; i < n; i++) {
        const float x2 = a[i] - b[i];          // nH2 = (float) nH - nH1 (ray_tracing.cc:1119)
        host[i] = frac ? x2 / a[i] : x2;       // f_H2 = nH2/nH (ray_tracing.cc:1192)
      }
      return FRT_OK;
    }
    case FRT_F_TREION_FLAG: {
      std::vector<uint8_t> a(n);
      CK(copy_sync(ctx, a.data(), d.treion_flag + B.cell0, n, cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < n; i++) host[i] = a[i] ? 1.f : 0.f;
      return FRT_OK;
    }
    case FRT_F_FION:
    case FRT_F_FION_MAX:
    case FRT_F_TCROSS:
    case FRT_F_DELTA_FION:
    case FRT_F_TREION_OUT:
    case FRT_F_TCROSS_FLAG:
    case FRT_F_NEUTRAL_FLAG:
    case FRT_F_TCROSS_NEW: {
      if (!d.ifront) {
        ctx->err = "the I-front fields exist with I-front tracking only (frt_set_subgrid)";
        return FRT_ERR_STATE;
      }
      if (f == FRT_F_TCROSS_FLAG || f == FRT_F_NEUTRAL_FLAG) {
        std::vector<uint8_t> a(n);
        CK(copy_sync(ctx, a.data(), d.if_flags + B.cell0, n, cudaMemcpyDeviceToHost));
        const uint8_t bit = (f == FRT_F_TCROSS_FLAG) ? 1 : 2;
        for (size_t i = 0; i < n; i++) host[i] = (a[i] & bit) ? 1.f : 0.f;
        return FRT_OK;
      }
      if (f == FRT_F_TCROSS_NEW) {
        CK(copy_sync(ctx, host, d.tcross_new + (size_t)B.cell0 * 10, sizeof(float) * n * 10, cudaMemcpyDeviceToHost));
        return FRT_OK;
      }
      const float* src = f == FRT_F_FION ? d.fion : f == FRT_F_FION_MAX ? d.fion_max : f == FRT_F_TCROSS ? d.tcross
                         : f == FRT_F_DELTA_FION ? d.delta_fion : d.treion_out;
      CK(get(src, host));
      return FRT_OK;
    }
    case FRT_F_GAMMA_H1_TOT: return sparse(0, host);
    case FRT_F_GAMMA_HE1_TOT: return sparse(1, host);
    case FRT_F_GAMMA_H1_NU:
    case FRT_F_GAMMA_HE1_NU:
    case FRT_F_NGAM_NU: {
      const int base = (f == FRT_F_GAMMA_H1_NU) ? 2 : (f == FRT_F_GAMMA_HE1_NU ? 2 + F : 2 + 2 * F);
      if (!d.per_bin) {
        ctx->err = "per-bin rates and photon counts are kept only with diag outputs or strict precision";
        return FRT_ERR_STATE;
      }
      std::vector<float> tmp(n);
      for (int nu = 0; nu < F; nu++) {
        st = sparse(base + nu, tmp.data());
        if (st) return st;
        for (size_t i = 0; i < n; i++) host[i * F + nu] = tmp[i];
      }
      return FRT_OK;
    }
    case FRT_F_U_NU: {
      // u_nu = (float)(spectrum*Gamma/sigma) * h * nu / clight (ray_tracing.cc:1142-1144)
      std::vector<float> g(n);
      st = sparse(0, g.data());
      if (st) return st;
      for (size_t i = 0; i < n; i++)
        for (int nu = 0; nu < F; nu++)
          host[i * F + nu] = (float)(d.spectrum[nu] * g[i] / d.sigH1_d[nu]) * 6.626068e-27 * ctx->cfg.nu_phot[nu] /
                             B.clight;
      return FRT_OK;
    }
    default: {
      const float* p = field_ptr(ctx, f);
      if (!p) {
        ctx->err = "field not kept in this output mode";
        return FRT_ERR_STATE;
      }
      CK(get(p, host));
      return FRT_OK;
    }
  }
}

frt_status frt_init_rt(frt_ctx* ctx) {
  if (!ctx) return FRT_ERR_INVALID;
  Dev& d = ctx->d;
  for (size_t b = 0; b < ctx->boxes.size(); b++)
    if (!ctx->gas_ready[b]) {
      ctx->err = "frt_init_gas not called for every box";
      return FRT_ERR_STATE;
    }
  // ray_dt of the source cells = dt (rt_funcs.cc:85-101, input_grid = FALSE); 0 for a box
  // restarted from files (input_grid = TRUE)
  std::vector<float> rdt;
  for (size_t b = 0; b < ctx->boxes.size(); b++)
    for (size_t s = 0; s < ctx->src_cell[b].size(); s++)
      rdt.push_back(ctx->src_lum[b][s] != 0 && !ctx->restarted[b] ? ctx->hbox[b].dt : 0.f);
  if (!rdt.empty()) CK(copy_sync(ctx, d.src_ray_dt, rdt.data(), sizeof(float) * rdt.size(), cudaMemcpyHostToDevice));
  Ctl c;
  memset(&c, 0, sizeof(c));
  CK(copy_sync(ctx, d.ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice));
  CK(fill_sync(ctx, d.lit_flag, 0, (size_t)d.ncell_total));
  launch_fill_i32(d.lit_slot, -1, d.ncell_total, ctx->s_main);
  CK(cudaStreamSynchronize(ctx->s_main));
  for (size_t b = 0; b < ctx->hbox.size(); b++) {
    ctx->hbox[b].t = ctx->restarted[b] ? ctx->restart_t[b] : 0.f;
    ctx->hbox[b].nphot_merge = 0.f;
  }
  ctx->rays_moved = false;
  ctx->merged_any = false;
  return upload_boxes(ctx);
}

frt_status frt_update_cosmo_expansion(frt_ctx* ctx, const float* a_current, const float* a_prev) {
  if (!ctx || !a_current || !a_prev) return FRT_ERR_INVALID;
  Dev& d = ctx->d;
  for (size_t b = 0; b < ctx->hbox.size(); b++)
    if (!(a_current[b] > 0.f) || !(a_prev[b] > 0.f) || !ctx->gas_ready[b]) {
      ctx->err = "frt_update_cosmo_expansion: scale factors must be positive and the gas set up";
      return FRT_ERR_INVALID;
    }
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(cudaStreamSynchronize(ctx->s_dark));
  if (!d.rho) {
    frt_status st = dalloc(ctx, &d.rho, (size_t)d.ncell_total);
    if (st) return st;
    for (size_t b = 0; b < ctx->hbox.size(); b++)
      CK(copy_sync(ctx, d.rho + ctx->hbox[b].cell0, ctx->rho[b].data(), sizeof(float) * ctx->rho[b].size(),
                    cudaMemcpyHostToDevice));
    if ((st = dalloc(ctx, &d.frac_h2, (size_t)d.ncell_total))) return st;
    if ((st = dalloc(ctx, &d.frac_he2, (size_t)d.ncell_total))) return st;
    ctx->graph_valid = false;   // the graph keeps a copy of the device pointers
  }
  frt_status st = download_boxes(ctx);
  if (st) return st;
  std::vector<float> ratio(ctx->hbox.size());
  std::vector<double> rf(ctx->hbox.size());
  for (size_t b = 0; b < ctx->hbox.size(); b++) {
    // gas_funcs.cc:472-485: dx[i] *= a_current/a_prev; rho *= pow(a_prev/a_current, 3.)
    ratio[b] = a_current[b] / a_prev[b];
    rf[b] = pow(a_prev[b] / a_current[b], 3.);
    ctx->hbox[b].avg_rho *= pow(a_prev[b] / a_current[b], 3.);   // gas_funcs.cc:520
    ctx->frac_kept[b] = 1;
    float dx = ctx->hbox[b].dx;
    dx *= ratio[b];
    host::set_cell_size(&ctx->hbox[b], &ctx->cfg, &ctx->boxes[b], dx);
  }
  if ((st = upload_boxes(ctx))) return st;
  for (size_t b = 0; b < ctx->hbox.size(); b++)
    launch_cosmo_expansion(d, (int)b, ratio[b], rf[b], ctx->grid_cells, ctx->s_main);
  return sync_and_check(ctx);
}

frt_status frt_update_hydro_step(frt_ctx* ctx, int box, const float* delta1, float a_rt, float dt_snap, float zz,
                                 int nsrc, const int32_t* ijk, const double* lum) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  if (!delta1 || !(a_rt > 0.f) || !(dt_snap > 0.f) || !ctx->gas_ready[box] || nsrc < 0 ||
      (nsrc > 0 && (!ijk || !lum))) {
    ctx->err = "frt_update_hydro_step: density, a positive scale factor and snapshot interval, gas set up";
    return FRT_ERR_INVALID;
  }
  Dev& d = ctx->d;
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(cudaStreamSynchronize(ctx->s_dark));
  BoxP& B = ctx->hbox[box];
  const size_t n = (size_t)B.ncell;
  // the new proper density and <rho> (get_ugas, then a_rt^-3)
  std::vector<float> rho(n);
  float avg = 0.f;
  host::snapshot_rho(B.n, delta1, a_rt, rho.data(), &avg);
  // <rho_prev> over the previous snapshot's density (0 before any switch: no d(delta)/dt yet)
  const float avg_prev = ctx->rho_prev_h[box].empty() ? 0.f : host::vol_avg(ctx->rho_prev_h[box].data(), B.n);
  if (!d.rho) {
    if ((st = dalloc(ctx, &d.rho, (size_t)d.ncell_total))) return st;
    for (size_t b = 0; b < ctx->hbox.size(); b++)
      if (ctx->rho[b].size() == (size_t)ctx->hbox[b].ncell)
        CK(copy_sync(ctx, d.rho + ctx->hbox[b].cell0, ctx->rho[b].data(), sizeof(float) * ctx->rho[b].size(),
                      cudaMemcpyHostToDevice));
    ctx->graph_valid = false;
  }
  if (!d.rho_prev) {
    if ((st = dalloc(ctx, &d.rho_prev, (size_t)d.ncell_total))) return st;
    ctx->graph_valid = false;
  }
  if (avg_prev > 0.f && !d.ddelta) {
    if ((st = dalloc(ctx, &d.ddelta, (size_t)d.ncell_total))) return st;   // 0 in the other boxes
    ctx->graph_valid = false;
  }
  CK(copy_sync(ctx, d.rho + B.cell0, rho.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  // the box at the new snapshot: redshift, cell size Lx0 a_rt / N (gas_funcs.cc:590-592, 689-691)
  host::set_cell_size(&B, &ctx->cfg, &ctx->boxes[box], host::snapshot_dx(&ctx->boxes[box], a_rt));
  host::set_redshift(&B, zz);
  B.avg_rho = avg;
  if ((st = upload_boxes(ctx))) return st;
  const bool cached = ctx->frac_kept[box] && d.frac_h2;
  launch_hydro_switch(d, box, cached, avg_prev, dt_snap, ctx->grid_cells, ctx->s_main);
  ctx->frac_kept[box] = 0;
  if ((st = sync_and_check(ctx))) return st;
  ctx->rho[box] = rho;
  ctx->rho_prev_h[box] = rho;
  ctx->boxes[box].zz = zz;
  // read_source_catalog (io_funcs.cc:157-233): the new sources, every ray_dt back to 0
  ctx->src_cell[box].clear();
  ctx->src_lum[box].clear();
  for (int s = 0; s < nsrc; s++) {
    const int i = ijk[3 * s], j = ijk[3 * s + 1], k = ijk[3 * s + 2];
    if (i < 0 || j < 0 || k < 0 || i >= B.n || j >= B.n || k >= B.n) {
      ctx->err = "source cell out of range";
      return FRT_ERR_INVALID;
    }
    ctx->src_cell[box].push_back((i * B.n + j) * B.n + k);
    ctx->src_lum[box].push_back(lum[s]);
  }
  if ((st = upload_sources(ctx))) return st;   // ray_dt of every source 0
  // get_nphot_min_max (main.cc:222) with the new sources and the step's time step
  double mn = 0., mx = 0.;
  if (!ctx->src_lum[box].empty()) {
    BoxP tmp = B;
    tmp.dt = ctx->step_dt[box] > 0.f ? ctx->step_dt[box] : B.dt;
    host::nphot_min_max(&ctx->cfg, &tmp, (int)ctx->src_lum[box].size(), ctx->src_lum[box].data(), &mn, &mx);
  }
  B.nphot_min = mn;
  B.nphot_max = mx;
  {
    std::vector<double> lg(2);   // as frt_get_nphot_min_max: log10 nphot_min and the PDF bin width
    lg[0] = log10(mn);
    lg[1] = (log10(mx) - log10(mn)) / (10000 - 1);
    CK(copy_sync(ctx, d.lg + 2 * box, lg.data(), sizeof(double) * 2, cudaMemcpyHostToDevice));
  }
  const float a4 = (float)(4. * (double)B.nphot_merge), c4 = (float)(4. * B.nphot_min);
  B.split_thr = (c4 >= a4) ? c4 : a4;
  return upload_boxes(ctx);
}

frt_status frt_set_subgrid(frt_ctx* ctx, const frt_subgrid_tables* t) {
  if (!ctx || !t || !t->time_RH || !t->fh1_RH || !t->t_deltaNL || !t->delta_over_sigma || !t->deltaNL)
    return FRT_ERR_INVALID;
  for (size_t b = 0; b < ctx->boxes.size(); b++)
    if (!ctx->gas_ready[b]) {
      ctx->err = "frt_set_subgrid: set up the gas of every box first (the model reads the densities)";
      return FRT_ERR_STATE;
    }
  Dev& d = ctx->d;
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(cudaStreamSynchronize(ctx->s_dark));
  const size_t nrh = (size_t)FRT_SUBGRID_NT * 27 + 1, nd = FRT_SUBGRID_NDLIN;
  auto copy = [&](const float* src, size_t n, const float** dst) -> frt_status {
    float* p = nullptr;
    frt_status st = dalloc(ctx, &p, n);
    if (st) return st;
    CK(copy_sync(ctx, p, src, sizeof(float) * n, cudaMemcpyHostToDevice));
    *dst = p;
    return FRT_OK;
  };
  frt_status st;
  if ((st = copy(t->time_RH, nrh, &d.sg_time)) || (st = copy(t->fh1_RH, nrh, &d.sg_fh1)) ||
      (st = copy(t->t_deltaNL, nd, &d.sg_tdnl)) || (st = copy(t->delta_over_sigma, nd, &d.sg_ds)) ||
      (st = copy(t->deltaNL, nd * nd, &d.sg_dnl)))
    return st;
  d.sg_tinit = t->tinit;
  d.sg_t12 = t->t_z12;
  d.sg_t8 = t->t_z8;
  d.sg_tcap = t->t_z55;
  for (int k = 0; k < 3; k++) d.sg_tre_dom[k] = t->tre_dom[k];
  d.sg_fH1_0 = ctx->cfg.fH1_0;
  d.sg_fHe1_0 = ctx->cfg.fHe1_0;
  d.sg_temp0 = ctx->cfg.temp_0;
  if (t->ifront && !d.ifront) {
    // init_rt with ifront = TRUE (rt_funcs.cc:49-69): no cell passed by a front, neutral_flag set
    const size_t NC = (size_t)d.ncell_total, L = (size_t)d.lit_cap;
    const long long XC = (long long)d.ray_cap * d.PL;
    if ((st = dalloc(ctx, &d.fion, NC)) || (st = dalloc(ctx, &d.fion_max, NC)) || (st = dalloc(ctx, &d.tcross, NC)) ||
        (st = dalloc(ctx, &d.tcross_new, NC * 10)) || (st = dalloc(ctx, &d.delta_fion, NC)) ||
        (st = dalloc(ctx, &d.treion_out, NC)) || (st = dalloc(ctx, &d.tcross_bits, NC)) ||
        (st = dalloc(ctx, &d.if_flags, NC)) || (st = dalloc(ctx, &d.l_fion, L)) || (st = dalloc(ctx, &d.l_free, L)) ||
        (st = dalloc(ctx, &d.l_ng3, 3 * L)) || (st = dalloc(ctx, &d.if_cnt, L)) || (st = dalloc(ctx, &d.if_off, L)) ||
        (st = dalloc(ctx, &d.if_fill, L)) || (st = dalloc(ctx, &d.if_list, (size_t)XC)) ||
        (st = dalloc(ctx, &d.xs_q, (size_t)XC)) || (st = dalloc(ctx, &d.xs_S, (size_t)XC)) ||
        (st = dalloc(ctx, &d.xs_E, (size_t)XC * d.F)) || (st = dalloc(ctx, &d.xs_reach, (size_t)XC)) ||
        (st = dalloc(ctx, &d.ord_cnt, (size_t)d.ray_cap / 256 + 1)) ||
        (st = dalloc(ctx, &d.ord_off, (size_t)d.ray_cap / 256 + 1)))
      return st;
    CK(fill_sync(ctx, d.fion, 0, sizeof(float) * NC));
    CK(fill_sync(ctx, d.fion_max, 0, sizeof(float) * NC));
    CK(fill_sync(ctx, d.tcross, 0, sizeof(float) * NC));
    CK(fill_sync(ctx, d.tcross_new, 0, sizeof(float) * NC * 10));
    CK(fill_sync(ctx, d.delta_fion, 0, sizeof(float) * NC));
    CK(fill_sync(ctx, d.treion_out, 0, sizeof(float) * NC));
    CK(fill_sync(ctx, d.tcross_bits, 0, sizeof(uint16_t) * NC));
    CK(fill_sync(ctx, d.if_flags, 2, NC));   // neutral_flag
    if (!ctx->h_flag) CK(cudaMallocHost(&ctx->h_flag, sizeof(int)));
    d.xs_cap = XC;
    d.ifront = 1;
    d.ordered = 1;
  }
  if (!d.mfp && (st = dalloc(ctx, &d.mfp, (size_t)d.ncell_total))) return st;
  if (!d.l_mfp && (st = dalloc(ctx, &d.l_mfp, (size_t)d.lit_cap))) return st;
  if (!d.rho) {   // the model reads rho / <rho> of every ionised cell
    if ((st = dalloc(ctx, &d.rho, (size_t)d.ncell_total))) return st;
    for (size_t b = 0; b < ctx->hbox.size(); b++)
      if (ctx->rho[b].size() == (size_t)ctx->hbox[b].ncell)
        CK(copy_sync(ctx, d.rho + ctx->hbox[b].cell0, ctx->rho[b].data(), sizeof(float) * ctx->rho[b].size(),
                      cudaMemcpyHostToDevice));
  }
  d.subgrid = 1;
  launch_sg_mfp_init(d, ctx->s_main);
  ctx->graph_valid = false;
  return sync_and_check(ctx);
}

frt_status frt_update_dt(frt_ctx* ctx, float* dt_out) {
  if (!ctx) return FRT_ERR_INVALID;
  if (dt_out)
    for (size_t b = 0; b < ctx->hbox.size(); b++) dt_out[b] = ctx->hbox[b].dt;
  return FRT_OK;
}

frt_status frt_get_nphot_min_max(frt_ctx* ctx, double* nmin_out, double* nmax_out) {
  if (!ctx) return FRT_ERR_INVALID;
  frt_status st = download_boxes(ctx);
  if (st) return st;
  std::vector<double> lg(2 * ctx->hbox.size());
  for (size_t b = 0; b < ctx->hbox.size(); b++) {
    BoxP& B = ctx->hbox[b];
    double mn = 0, mx = 0;
    if (!ctx->src_lum[b].empty())
      host::nphot_min_max(&ctx->cfg, &B, (int)ctx->src_lum[b].size(), ctx->src_lum[b].data(), &mn, &mx);
    B.nphot_min = mn;
    B.nphot_max = mx;
    const double lg_max = log10(mx), lg_min = log10(mn);
    lg[2 * b] = lg_min;
    lg[2 * b + 1] = (lg_max - lg_min) / (10000 - 1);
    const float a = (float)(4. * (double)B.nphot_merge), c = (float)(4. * B.nphot_min);
    B.split_thr = (c >= a) ? c : a;
    if (nmin_out) nmin_out[b] = mn;
    if (nmax_out) nmax_out[b] = mx;
  }
  CK(copy_sync(ctx, ctx->d.lg, lg.data(), sizeof(double) * lg.size(), cudaMemcpyHostToDevice));
  return upload_boxes(ctx);
}

frt_status frt_set_clump(frt_ctx* ctx) { return ctx ? FRT_OK : FRT_ERR_INVALID; }
frt_status frt_set_clight(frt_ctx* ctx) { return ctx ? FRT_OK : FRT_ERR_INVALID; }

frt_status frt_update_rays(frt_ctx* ctx) {
  if (!ctx) return FRT_ERR_INVALID;
  note_step(ctx);
  enqueue_begin_advance(ctx);
  return sync_and_check(ctx);
}

frt_status frt_find_avg_unu(frt_ctx* ctx) {
  if (!ctx) return FRT_ERR_INVALID;
  enqueue_iterations(ctx, false);
  if (ctx->d.subgrid) launch_sg_dark(ctx->d, false, ctx->grid_cells, ctx->s_main);
  else launch_dark(ctx->d, ctx->strict, false, ctx->grid_cells, ctx->s_main);
  return sync_and_check(ctx);
}

frt_status frt_count_rays(frt_ctx* ctx, long long* count_per_box) {
  if (!ctx) return FRT_ERR_INVALID;
  launch_count(ctx->d, ctx->grid_rays, ctx->s_main);
  frt_status st = sync_and_check(ctx);
  if (st) return st;
  if (count_per_box) CK(copy_sync(ctx, count_per_box, ctx->d.count, sizeof(long long) * ctx->d.nbox, cudaMemcpyDeviceToHost));
  return FRT_OK;
}

frt_status frt_merge(frt_ctx* ctx, const uint16_t* itheta_per_box) {
  if (!ctx) return FRT_ERR_INVALID;
  ctx->rays_moved = true;
  frt_status st = stage_itheta(ctx, itheta_per_box, nullptr);
  if (st) return st;
  CK(cudaMemcpyAsync(ctx->d.itheta_merge, ctx->h_ith_box, sizeof(uint16_t) * ctx->d.nbox, cudaMemcpyHostToDevice,
                     ctx->s_main));
  launch_count(ctx->d, ctx->grid_rays, ctx->s_main);
  launch_merge(ctx->d, ctx->grid_rays, ctx->s_main);
  frt_status st2 = sync_and_check(ctx);
  if (st2) return st2;
  long long merged = 0;
  CK(copy_sync(ctx, &merged, &ctx->d.ctl->merged, sizeof merged, cudaMemcpyDeviceToHost));
  if (merged > 0) ctx->merged_any = true;
  return FRT_OK;
}

frt_status frt_split_rays(frt_ctx* ctx) {
  if (!ctx) return FRT_ERR_INVALID;
  ctx->rays_moved = true;
  launch_split_compact(ctx->d, ctx->nsm * ctx->tune.split_grid, ctx->s_main);
  return sync_and_check(ctx);
}

frt_status frt_update_thermal(frt_ctx* ctx) {
  if (!ctx) return FRT_ERR_INVALID;
  if (ctx->d.subgrid) launch_sg_thermal_all(ctx->d, ctx->grid_cells, ctx->s_main);
  else launch_thermal_all(ctx->d, ctx->strict, ctx->grid_cells, ctx->s_main);
  return sync_and_check(ctx);
}

frt_status frt_new_rays(frt_ctx* ctx, const uint16_t* itheta_per_source) {
  if (!ctx) return FRT_ERR_INVALID;
  frt_status st = stage_itheta(ctx, nullptr, itheta_per_source);
  if (st) return st;
  if (ctx->d.nsrc)
    CK(cudaMemcpyAsync(ctx->d.src_itheta, ctx->h_ith_src, sizeof(uint16_t) * ctx->d.nsrc, cudaMemcpyHostToDevice,
                       ctx->s_main));
  launch_cast(ctx->d, ctx->s_main);
  return sync_and_check(ctx);
}

frt_status frt_seed_boxes(frt_ctx* ctx, const unsigned int* seeds) {
  if (!ctx || !seeds) return FRT_ERR_INVALID;
  const size_t nb = ctx->boxes.size();
  ctx->rng_state.assign(nb, std::vector<char>(128, 0));
  ctx->rng.assign(nb, random_data{});
  for (size_t b = 0; b < nb; b++) {
    memset(&ctx->rng[b], 0, sizeof(random_data));
    if (initstate_r(seeds[b], ctx->rng_state[b].data(), 128, &ctx->rng[b]) != 0) {
      ctx->err = "initstate_r failed";
      return FRT_ERR_INVALID;
    }
  }
  return FRT_OK;
}

frt_status frt_draw_cast(frt_ctx* ctx, uint16_t* itheta_per_source) {
  if (!ctx || !itheta_per_source) return FRT_ERR_INVALID;
  return draw(ctx, nullptr, itheta_per_source);
}

frt_status frt_draw_step(frt_ctx* ctx, uint16_t* itheta_per_box, uint16_t* itheta_per_source) {
  if (!ctx || !itheta_per_box) return FRT_ERR_INVALID;
  return draw(ctx, itheta_per_box, itheta_per_source);
}

// ---- remembered launch shapes (frt_autotune) ------------------------------------------------
// One shape set per (device, SM count, cells, precision, power-of-two bucket of the live rays).
static std::mutex g_tune_mu;
static std::map<std::string, Tune> g_tune_cache;

static std::string tune_key(const frt_ctx* ctx, long long rays) {
  int bucket = 0;
  while (bucket < 62 && (2LL << bucket) <= rays) bucket++;
  return ctx->dev_name + "|" + std::to_string(ctx->nsm) + "|" + std::to_string(ctx->d.ncell_total) + "|" +
         (ctx->strict ? "strict" : "mixed") + "|" + std::to_string(bucket);
}

// frt_step: switch to the remembered shapes of the current ray-count bucket, if any
static void follow_tune_cache(frt_ctx* ctx) {
  Tune t;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(tune_key(ctx, ctx->last.rays_alive));
    if (it == g_tune_cache.end()) return;
    t = it->second;
  }
  if (!(t == ctx->tune)) {
    ctx->tune = t;
    ctx->graph_valid = false;
  }
}

// Resolve the step's angle indices: caller-provided, or drawn from the context's streams.
static frt_status step_inputs(frt_ctx* ctx, const uint16_t* ib, const uint16_t* is) {
  if (!ib && !is) {
    ctx->draw_box.resize(ctx->boxes.size());
    ctx->draw_src.resize(std::max(1, ctx->d.nsrc));
    frt_status st = draw(ctx, ctx->draw_box.data(), ctx->draw_src.data());
    if (st) return st;
    return stage_itheta(ctx, ctx->draw_box.data(), ctx->draw_src.data());
  }
  return stage_itheta(ctx, ib, is);
}

frt_status frt_step_plain(frt_ctx* ctx, const uint16_t* itheta_per_box, const uint16_t* itheta_per_source,
                          frt_step_stats* stats) {
  if (!ctx) return FRT_ERR_INVALID;
  frt_status st = step_inputs(ctx, itheta_per_box, itheta_per_source);
  if (st) return st;
  note_step(ctx);
  CK(cudaEventRecord(ctx->ev_t0, ctx->s_main));
  enqueue_step(ctx, false);
  CK(cudaEventRecord(ctx->ev_t1, ctx->s_main));
  return finish_step(ctx, stats);
}

frt_status frt_step(frt_ctx* ctx, const uint16_t* itheta_per_box, const uint16_t* itheta_per_source,
                    frt_step_stats* stats) {
  if (!ctx) return FRT_ERR_INVALID;
  if (ctx->d.ifront) return frt_step_plain(ctx, itheta_per_box, itheta_per_source, stats);   // host-driven rounds
  frt_status st = step_inputs(ctx, itheta_per_box, itheta_per_source);
  if (st) return st;
  if (ctx->tune_auto) follow_tune_cache(ctx);
  if (!ctx->graph_valid) {
    if (ctx->graph) {
      cudaGraphExecDestroy(ctx->graph);
      ctx->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamSynchronize(ctx->s_main));
    CK(cudaStreamBeginCapture(ctx->s_main, cudaStreamCaptureModeThreadLocal));
    enqueue_step(ctx, true);
    CK(cudaStreamEndCapture(ctx->s_main, &g));
    CK(cudaGraphInstantiate(&ctx->graph, g, cudaGraphInstantiateFlagUseNodePriority));   // the streams' priorities
    CK(cudaGraphDestroy(g));
    ctx->graph_valid = true;
  }
  note_step(ctx);
  CK(cudaEventRecord(ctx->ev_t0, ctx->s_main));
  CK(cudaGraphLaunch(ctx->graph, ctx->s_main));
  CK(cudaEventRecord(ctx->ev_t1, ctx->s_main));
  return finish_step(ctx, stats);
}

frt_status frt_last_stats(frt_ctx* ctx, frt_step_stats* stats) {
  if (!ctx || !stats) return FRT_ERR_INVALID;
  Ctl c;
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(copy_sync(ctx, &c, ctx->d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
  fill_stats(ctx, c, stats);
  return FRT_OK;
}

frt_status frt_num_rays(frt_ctx* ctx, int box, long long* n) {
  if (!ctx || !n) return FRT_ERR_INVALID;
  Ctl c;
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(copy_sync(ctx, &c, ctx->d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
  const int nr = std::min(c.nray[c.cur], ctx->d.ray_cap);
  if (box < 0) {
    *n = nr;
    return FRT_OK;
  }
  std::vector<uint16_t> bx(nr);
  std::vector<uint8_t> dead(nr);
  if (nr) {
    CK(copy_sync(ctx, bx.data(), ctx->d.pool[c.cur].box, sizeof(uint16_t) * nr, cudaMemcpyDeviceToHost));
  }
  long long k = 0;
  for (int i = 0; i < nr; i++) k += (bx[i] == box);
  *n = k;
  return FRT_OK;
}

frt_status frt_download_rays(frt_ctx* ctx, int box, int16_t* order, int32_t* pixel, uint16_t* itheta, int32_t* cell,
                             float* geom9, float* nphot) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  Ctl c;
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(copy_sync(ctx, &c, ctx->d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
  const int nr = std::min(c.nray[c.cur], ctx->d.ray_cap);
  const RayPool& P = ctx->d.pool[c.cur];
  const int F = ctx->d.F;
  const size_t cap = (size_t)ctx->d.ray_cap;
  std::vector<uint16_t> bx(nr), ith(nr);
  std::vector<int16_t> ord(nr);
  std::vector<int32_t> pix(nr), cl(nr);
  std::vector<float> g[9], np((size_t)F * nr);
  float* gp[9] = {P.xh, P.yh, P.zh, P.r, P.dr, P.x, P.y, P.z, P.time};
  if (nr) {
    CK(copy_sync(ctx, bx.data(), P.box, sizeof(uint16_t) * nr, cudaMemcpyDeviceToHost));
    CK(copy_sync(ctx, ith.data(), P.itheta, sizeof(uint16_t) * nr, cudaMemcpyDeviceToHost));
    CK(copy_sync(ctx, ord.data(), P.order, sizeof(int16_t) * nr, cudaMemcpyDeviceToHost));
    CK(copy_sync(ctx, pix.data(), P.pixel, sizeof(int32_t) * nr, cudaMemcpyDeviceToHost));
    CK(copy_sync(ctx, cl.data(), P.cell, sizeof(int32_t) * nr, cudaMemcpyDeviceToHost));
    for (int k = 0; k < 9; k++) {
      g[k].resize(nr);
      CK(copy_sync(ctx, g[k].data(), gp[k], sizeof(float) * nr, cudaMemcpyDeviceToHost));
    }
    for (int nu = 0; nu < F; nu++)
      CK(copy_sync(ctx, np.data() + (size_t)nu * nr, P.nphot + nu * cap, sizeof(float) * nr, cudaMemcpyDeviceToHost));
  }
  size_t w = 0;
  for (int i = 0; i < nr; i++) {
    if (bx[i] != box) continue;
    if (order) order[w] = ord[i];
    if (pixel) pixel[w] = pix[i];
    if (itheta) itheta[w] = ith[i];
    if (cell) cell[w] = cl[i];
    if (geom9)
      for (int k = 0; k < 9; k++) geom9[w * 9 + k] = g[k][i];
    if (nphot)
      for (int nu = 0; nu < F; nu++) nphot[w * F + nu] = np[(size_t)nu * nr + i];
    w++;
  }
  return FRT_OK;
}

frt_status frt_set_tau_limit(frt_ctx* ctx, double tau_max) {
  if (!ctx) return FRT_ERR_INVALID;
  if (!(tau_max >= 0.0) || tau_max > 1e30) {
    ctx->err = "frt_set_tau_limit: tau_max must be >= 0 (0 turns the limit off)";
    return FRT_ERR_INVALID;
  }
  Dev& d = ctx->d;
  if (tau_max > 0.0 && d.subgrid) {
    ctx->err = "frt_set_tau_limit: not available with the sub-grid model";
    return FRT_ERR_INVALID;
  }
  if (tau_max > 0.0 && !d.pool[0].col) {
    CK(cudaStreamSynchronize(ctx->s_main));
    for (int p = 0; p < 2; p++) AL(d.pool[p].col, 2 * (size_t)d.ray_cap);   // zero-filled
  }
  d.tau_max = tau_max;
  ctx->graph_valid = false;
  return FRT_OK;
}

frt_status frt_download_ray_columns(frt_ctx* ctx, int box, double* col2) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  if (!col2) return FRT_ERR_INVALID;
  Ctl c;
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(copy_sync(ctx, &c, ctx->d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
  const int nr = std::min(c.nray[c.cur], ctx->d.ray_cap);
  const RayPool& P = ctx->d.pool[c.cur];
  std::vector<uint16_t> bx(nr);
  std::vector<double> ch(nr, 0.0), che(nr, 0.0);
  if (nr) {
    CK(copy_sync(ctx, bx.data(), P.box, sizeof(uint16_t) * nr, cudaMemcpyDeviceToHost));
    if (P.col) {
      CK(copy_sync(ctx, ch.data(), P.col, sizeof(double) * nr, cudaMemcpyDeviceToHost));
      CK(copy_sync(ctx, che.data(), P.col + ctx->d.ray_cap, sizeof(double) * nr, cudaMemcpyDeviceToHost));
    }
  }
  size_t w = 0;
  for (int i = 0; i < nr; i++) {
    if (bx[i] != box) continue;
    col2[2 * w] = ch[i];
    col2[2 * w + 1] = che[i];
    w++;
  }
  return FRT_OK;
}

frt_status frt_set_nphot_merge(frt_ctx* ctx, int box, double nphot_merge) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  if (!(nphot_merge >= 0.0)) return FRT_ERR_INVALID;
  CK(cudaStreamSynchronize(ctx->s_main));
  if ((st = download_boxes(ctx))) return st;
  ctx->hbox[box].nphot_merge = (float)nphot_merge;
  CK(copy_sync(ctx, &ctx->d.box[box].nphot_merge, &ctx->hbox[box].nphot_merge, sizeof(float), cudaMemcpyHostToDevice));
  return FRT_OK;
}

frt_status frt_box_scalars(frt_ctx* ctx, int box, double* out8) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  if (!out8) return FRT_ERR_INVALID;
  CK(cudaStreamSynchronize(ctx->s_main));
  st = download_boxes(ctx);
  if (st) return st;
  const BoxP& B = ctx->hbox[box];
  const double v[8] = {(double)B.t, (double)B.dt, B.nphot_min, B.nphot_max, (double)B.nphot_merge,
                       (double)B.num_thresh, (double)B.dx, (double)B.dx0};
  memcpy(out8, v, sizeof v);
  return FRT_OK;
}

frt_status frt_set_cast_per_source(frt_ctx* ctx, int per_source) {
  if (!ctx) return FRT_ERR_INVALID;
  ctx->cast_per_source = per_source != 0;
  return FRT_OK;
}

// ---- one box shared by several contexts: the step in phases ------------------------------------
// Every context holds the whole box and casts only the sources it owns; the caller combines the
// contexts between phases (OR of the lit flags after the walk, sum of the lit cells' absorbed
// photons after each ray pass) so that all of them run the same cell passes.
frt_status frt_set_source_owner(frt_ctx* ctx, const uint8_t* own) {
  if (!ctx) return FRT_ERR_INVALID;
  Dev& d = ctx->d;
  if (!own) {
    d.src_own = nullptr;
  } else {
    if (d.nsrc < 1) return FRT_ERR_INVALID;
    if (!ctx->src_own_buf) {
      void* q = nullptr;
      CK(cudaMalloc(&q, (size_t)d.src_cap));
      ctx->allocs.push_back(q);
      ctx->src_own_buf = (uint8_t*)q;
    }
    CK(copy_sync(ctx, ctx->src_own_buf, own, (size_t)d.nsrc, cudaMemcpyHostToDevice));
    d.src_own = ctx->src_own_buf;
  }
  ctx->graph_valid = false;   // the step graph holds the Dev block by value
  return FRT_OK;
}

frt_status frt_phase_buffers(frt_ctx* ctx, void** lit_flag, long long* ncell, void** lit_acc, void** lit_heat,
                             long long* nlit) {
  if (!ctx) return FRT_ERR_INVALID;
  if (lit_flag) *lit_flag = ctx->d.lit_flag;
  if (ncell) *ncell = ctx->d.ncell_total;
  if (lit_acc) *lit_acc = ctx->d.l_acc;
  if (lit_heat) *lit_heat = ctx->d.l_heat;
  if (nlit) *nlit = ctx->phase_nlit;
  return FRT_OK;
}

frt_status frt_step_phase(frt_ctx* ctx, int phase, int iter, const uint16_t* itheta_per_box,
                          const uint16_t* itheta_per_source, frt_step_stats* stats) {
  if (!ctx) return FRT_ERR_INVALID;
  Dev& d = ctx->d;
  if (d.per_bin || d.subgrid) {
    ctx->err = "frt_step_phase: needs core outputs, mixed precision and the plain model (the per-bin rates are "
               "not combined across contexts)";
    return FRT_ERR_INVALID;
  }
  cudaStream_t s = ctx->s_main;
  switch (phase) {
    case FRT_PHASE_WALK: {
      frt_status st = step_inputs(ctx, itheta_per_box, itheta_per_source);
      if (st) return st;
      CK(cudaMemcpyAsync(d.itheta_merge, ctx->h_ith_box, sizeof(uint16_t) * d.nbox, cudaMemcpyHostToDevice, s));
      if (d.nsrc)
        CK(cudaMemcpyAsync(d.src_itheta, ctx->h_ith_src, sizeof(uint16_t) * d.nsrc, cudaMemcpyHostToDevice, s));
      note_step(ctx);
      CK(cudaEventRecord(ctx->ev_t0, s));
      ctx->rays_moved = true;
      launch_clear_lit(d, ctx->grid_lit, s);
      launch_step_begin(d, s);
      launch_walk(d, ctx->nsm * ctx->tune.adv_grid, s, ctx->tune.adv_block);
      break;
    }
    case FRT_PHASE_CELLS: {
      // strict cell order, so that every context sharing the box numbers its lit cells alike
      const long long nchunk = (d.ncell_total / 16 + 255) / 256;
      if (!ctx->chunk_buf) {
        void* q = nullptr;
        CK(cudaMalloc(&q, sizeof(int) * (size_t)nchunk));
        ctx->allocs.push_back(q);
        ctx->chunk_buf = (int*)q;
      }
      launch_lit_number_ordered(d, ctx->chunk_buf, nchunk, ctx->grid_rays, s);
      CK(cudaEventRecord(ctx->ev_fork, s));
      CK(cudaStreamWaitEvent(ctx->s_dark, ctx->ev_fork, 0));
      CK(cudaEventRecord(ctx->ev_d0, ctx->s_dark));
      launch_dark(d, ctx->strict, true, ctx->grid_dark, ctx->s_dark);
      CK(cudaEventRecord(ctx->ev_d1, ctx->s_dark));
      CK(cudaEventRecord(ctx->ev_join, ctx->s_dark));
      launch_lit_init(d, ctx->strict, ctx->grid_lit, s);
      int nl = 0;
      CK(cudaMemcpyAsync(&nl, &d.ctl->n_lit, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      ctx->phase_nlit = std::min(nl, d.lit_cap);
      break;
    }
    case FRT_PHASE_RAYPASS:
      if (iter < 0 || iter >= d.itercount) return FRT_ERR_INVALID;
      if (iter < frt_ctx::kMaxTimedIter) CK(cudaEventRecord(ctx->ev_r[2 * iter], s));
      launch_raypass(d, iter, ctx->strict, ctx->nsm * ctx->tune.rp_grid, s, ctx->tune.rp_block, ctx->tune.rp_chunk);
      if (iter < frt_ctx::kMaxTimedIter) CK(cudaEventRecord(ctx->ev_r[2 * iter + 1], s));
      break;
    case FRT_PHASE_CELLPASS:
      if (iter < 0 || iter >= d.itercount) return FRT_ERR_INVALID;
      launch_litpass(d, iter, ctx->strict, true, ctx->nsm * ctx->tune.lit_grid, s);
      break;
    case FRT_PHASE_END:
      launch_count_merge(d, ctx->grid_rays, s);
      launch_split_compact(d, ctx->nsm * ctx->tune.split_grid, s);
      CK(cudaStreamWaitEvent(s, ctx->ev_join, 0));
      launch_cast(d, s);
      CK(cudaMemcpyAsync(ctx->h_ctl, d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
      CK(cudaEventRecord(ctx->ev_t1, s));
      return finish_step(ctx, stats ? stats : &ctx->stats_scratch);
    default:
      return FRT_ERR_INVALID;
  }
  // the caller reads or combines device arrays next: unless it orders its combines on the
  // context's stream (frt_set_phase_async), the phase's work is complete on return
  if (!ctx->phase_async) CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return FRT_OK;
}

frt_status frt_set_phase_async(frt_ctx* ctx, int async) {
  if (!ctx) return FRT_ERR_INVALID;
  ctx->phase_async = async != 0;
  return FRT_OK;
}

frt_status frt_phase_stream(frt_ctx* ctx, void** stream) {
  if (!ctx || !stream) return FRT_ERR_INVALID;
  *stream = (void*)ctx->s_main;
  return FRT_OK;
}

frt_status frt_last_adjoint_timing(frt_ctx* ctx, float* ms) {
  if (!ctx || !ms) return FRT_ERR_INVALID;
  *ms = ctx->last_adjoint_ms;
  return FRT_OK;
}

frt_status frt_last_kernel_timing(frt_ctx* ctx, int which, float* ms) {
  if (!ctx || !ms || which < 0 || which > 2) return FRT_ERR_INVALID;
  *ms = which == 0 ? ctx->last_dark_ms : (which == 1 ? ctx->last_raypass_ms : ctx->last_walk_ms);
  return FRT_OK;
}

frt_status frt_last_timing(frt_ctx* ctx, float* step_ms, float* cell_kernel_ms) {
  if (!ctx) return FRT_ERR_INVALID;
  if (step_ms) *step_ms = ctx->last_step_ms;
  if (cell_kernel_ms) *cell_kernel_ms = ctx->last_dark_ms;
  return FRT_OK;
}

}  // extern "C"

// ---- restart files in the reference's formats ------------------------------------------------
// write_gas_binary (io_funcs.cc:358-393): float t, then per cell 18 floats + nfreq floats;
// write_rays_binary (274-303): packed records {int64 slot, bool active, int16 order, int32 pixel,
// uint16 itheta, 3 floats direction, nfreq floats photons, r, dr, x, y, z, time, int32 cell}
// ended by slot -1; write_treion (338-355): per cell float + 3 bools. In plain mode fion = 1,
// tcross = 0, f_He3 = 0 and neutral_flag stays TRUE; every ray is active at a step boundary.
namespace {

struct Bytes {
  unsigned char* p;
  size_t n, cap;
  template <typename T> void put(const T& v) {
    if (p && n + sizeof(T) <= cap) memcpy(p + n, &v, sizeof(T));
    n += sizeof(T);
  }
};

size_t ray_record_size(int F) { return 8 + 1 + 2 + 4 + 2 + 12 + 4 * (size_t)F + 24 + 4; }

}  // namespace

extern "C" {

frt_status frt_write_gas(frt_ctx* ctx, int box, void* buf, size_t cap, size_t* len) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  const size_t n = (size_t)ctx->hbox[box].ncell;
  const int F = ctx->d.F;
  const size_t need = 4 + n * (18 + (size_t)F) * 4;
  if (len) *len = need;
  if (!buf) return FRT_OK;
  if (cap < need) {
    ctx->err = "frt_write_gas: buffer too small";
    return FRT_ERR_INVALID;
  }
  const frt_field ids[] = {FRT_F_RHO, FRT_F_TEMP, FRT_F_NH1, FRT_F_F_H1, FRT_F_F_HE1, FRT_F_F_H2, FRT_F_F_HE2,
                           FRT_F_GAMMA_H1_TOT, FRT_F_GAMMA_HE1_TOT, FRT_F_HEAT_RATE, FRT_F_COOL_RATE, FRT_F_AVG_NH1,
                           FRT_F_TREION};
  std::vector<std::vector<float>> f(13, std::vector<float>(n));
  for (int k = 0; k < 13; k++) {
    st = frt_get_field(ctx, box, ids[k], f[k].data());
    if (st) return st;
  }
  std::vector<float> mfp(n), mfp912(n), ngam((size_t)n * F, 0.f);
  if (ctx->d.mfp) {
    if ((st = frt_get_field(ctx, box, FRT_F_MFP, mfp.data()))) return st;
    if ((st = frt_get_field(ctx, box, FRT_F_MFP_912, mfp912.data()))) return st;
  } else {
    // core outputs keep no mean free paths: from the final <n_HI> (the reference takes the
    // iterate before the last C2Ray update, ray_tracing.cc:945)
    for (size_t q = 0; q < n; q++) {
      mfp[q] = (float)(1. / ctx->d.sigH1_0 / (double)f[11][q]);
      mfp912[q] = (float)(1. / ctx->d.sigH1_912 / (double)f[11][q]);
    }
  }
  if (ctx->d.per_bin && (st = frt_get_field(ctx, box, FRT_F_NGAM_NU, ngam.data()))) return st;
  if ((st = download_boxes(ctx))) return st;
  Bytes o{(unsigned char*)buf, 0, cap};
  o.put<float>(ctx->hbox[box].t);
  for (size_t q = 0; q < n; q++) {
    for (int k = 0; k < 7; k++) o.put<float>(f[k][q]);      // rho temp nH1 f_H1 f_He1 f_H2 f_He2
    o.put<float>(0.f);                                        // f_He3
    o.put<float>(f[7][q]);
    o.put<float>(f[8][q]);
    o.put<float>(mfp[q]);
    o.put<float>(mfp912[q]);
    o.put<float>(f[9][q]);
    o.put<float>(f[10][q]);
    o.put<float>(f[11][q]);
    o.put<float>(1.f);                                        // fion
    o.put<float>(0.f);                                        // tcross
    o.put<float>(f[12][q]);                                   // treion_out
    for (int nu = 0; nu < F; nu++) o.put<float>(ngam[q * F + nu]);
  }
  return FRT_OK;
}

frt_status frt_write_treion(frt_ctx* ctx, int box, void* buf, size_t cap, size_t* len) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  const size_t n = (size_t)ctx->hbox[box].ncell;
  const size_t need = n * 7;
  if (len) *len = need;
  if (!buf) return FRT_OK;
  if (cap < need) {
    ctx->err = "frt_write_treion: buffer too small";
    return FRT_ERR_INVALID;
  }
  std::vector<float> tre(n), fl(n);
  if ((st = frt_get_field(ctx, box, FRT_F_TREION, tre.data()))) return st;
  if ((st = frt_get_field(ctx, box, FRT_F_TREION_FLAG, fl.data()))) return st;
  Bytes o{(unsigned char*)buf, 0, cap};
  for (size_t q = 0; q < n; q++) {
    o.put<float>(tre[q]);
    o.put<bool>(fl[q] != 0.f);
    o.put<bool>(false);   // tcross_flag
    o.put<bool>(true);    // neutral_flag
  }
  return FRT_OK;
}

frt_status frt_write_rays(frt_ctx* ctx, int box, void* buf, size_t cap, size_t* len) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  long long nr = 0;
  if ((st = frt_num_rays(ctx, box, &nr))) return st;
  const int F = ctx->d.F;
  const size_t need = (size_t)nr * ray_record_size(F) + 8;
  if (len) *len = need;
  if (!buf) return FRT_OK;
  if (cap < need) {
    ctx->err = "frt_write_rays: buffer too small";
    return FRT_ERR_INVALID;
  }
  std::vector<int16_t> ord(nr);
  std::vector<int32_t> pix(nr), cell(nr);
  std::vector<uint16_t> ith(nr);
  std::vector<float> g((size_t)nr * 9), np((size_t)nr * F);
  if ((st = frt_download_rays(ctx, box, ord.data(), pix.data(), ith.data(), cell.data(), g.data(), np.data())))
    return st;
  Bytes o{(unsigned char*)buf, 0, cap};
  for (long long x = 0; x < nr; x++) {
    const float* v = &g[(size_t)x * 9];
    o.put<int64_t>(x);
    o.put<bool>(true);
    o.put<int16_t>(ord[x]);
    o.put<int32_t>(pix[x]);
    o.put<uint16_t>(ith[x]);
    o.put<float>(v[0]); o.put<float>(v[1]); o.put<float>(v[2]);
    for (int nu = 0; nu < F; nu++) o.put<float>(np[(size_t)x * F + nu]);
    for (int k = 3; k < 9; k++) o.put<float>(v[k]);   // r dr x y z time
    o.put<int32_t>(cell[x]);
  }
  o.put<int64_t>(-1);
  return FRT_OK;
}

frt_status frt_read_gas(frt_ctx* ctx, int box, const void* buf, size_t len) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  const BoxP& B = ctx->hbox[box];
  const size_t n = (size_t)B.ncell;
  const int F = ctx->d.F;
  if (!buf || len != 4 + n * (18 + (size_t)F) * 4) {
    ctx->err = "frt_read_gas: record size does not match the box";
    return FRT_ERR_INVALID;
  }
  float t0;
  memcpy(&t0, buf, 4);
  std::vector<float> rec(n * (18 + F));
  memcpy(rec.data(), (const char*)buf + 4, rec.size() * 4);
  std::vector<float> rho(n), nH(n), nHe(n), nH1(n), nHe1(n), fH1(n), fHe1(n), temp(n), ne(n), ntot(n), rh(n), rhe(n),
      dne(n), heat(n), cool(n);
  host::GasInit g{rho.data(), nH.data(), nHe.data(), nH1.data(), nHe1.data(), fH1.data(), fHe1.data(), temp.data(),
                  ne.data(), ntot.data(), rh.data(), rhe.data(), dne.data()};
  host::init_gas_restart(&ctx->cfg, &ctx->boxes[box], host::GasRestart{rec.data(), 18 + F}, &g, heat.data(),
                         cool.data());
  Dev& d = ctx->d;
  const size_t o = (size_t)B.cell0;
  auto up = [&](float* dst, const std::vector<float>& src) {
    return copy_sync(ctx, dst + o, src.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
  };
  CK(up(d.nH, nH)); CK(up(d.nHe, nHe)); CK(up(d.nH1, nH1)); CK(up(d.nHe1, nHe1)); CK(up(d.f_H1, fH1));
  CK(up(d.f_He1, fHe1)); CK(up(d.temp, temp)); CK(up(d.ne, ne)); CK(up(d.avg_nh1, nH1)); CK(up(d.avg_nhe1, nHe1));
  CK(up(d.n_tot, ntot)); CK(up(d.dne_dt, dne)); CK(up(d.nH1_prev, nH1)); CK(up(d.heat, heat)); CK(up(d.cool, cool));
  if (d.rec_h2) {
    CK(up(d.rec_h2, rh));
    CK(up(d.rec_he2, rhe));
  }
  if (d.rho) CK(up(d.rho, rho));
  ctx->rho[box] = rho;
  ctx->gas_ready[box] = 1;
  ctx->restarted[box] = 1;
  ctx->restart_t[box] = t0;
  return FRT_OK;
}

frt_status frt_read_treion(frt_ctx* ctx, int box, const void* buf, size_t len) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  const BoxP& B = ctx->hbox[box];
  const size_t n = (size_t)B.ncell;
  if (!buf || len != n * 7) {
    ctx->err = "frt_read_treion: record size does not match the box";
    return FRT_ERR_INVALID;
  }
  std::vector<float> tre(n);
  std::vector<uint8_t> fl(n);
  const unsigned char* p = (const unsigned char*)buf;
  for (size_t q = 0; q < n; q++) {
    memcpy(&tre[q], p + q * 7, 4);
    fl[q] = p[q * 7 + 4] ? 1 : 0;
  }
  Dev& d = ctx->d;
  CK(copy_sync(ctx, d.treion + B.cell0, tre.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  CK(copy_sync(ctx, d.treion_flag + B.cell0, fl.data(), n, cudaMemcpyHostToDevice));
  return FRT_OK;
}

}  // extern "C"

namespace {
// Appends ray records of the reference's ray-file format (write_rays_binary) to the current pool
// of a box. restart: the restart path of init_rt (the free-slot probe drops a record at slot 0 with
// no first-bin photons, and the loaded photons enter the ledger's in-flight count); otherwise the
// records are rays moved between contexts during or between steps (every record kept, the ledger
// untouched, the new slots' removal flags cleared).
static frt_status append_ray_records(frt_ctx* ctx, int box, const void* buf, size_t len, bool restart,
                                     const char* what) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  if (!buf) return FRT_ERR_INVALID;
  Dev& d = ctx->d;
  const int F = d.F;
  const size_t rs = ray_record_size(F);
  const unsigned char* p = (const unsigned char*)buf;
  std::vector<int32_t> cell, pix;
  std::vector<int16_t> ord;
  std::vector<uint16_t> ith, bx;
  std::vector<float> g[9], np[FRT_MAX_FREQ];
  size_t pos = 0;
  while (true) {
    if (pos + 8 > len) {
      ctx->err = std::string(what) + ": record set not ended by slot -1";
      return FRT_ERR_INVALID;
    }
    int64_t slot;
    memcpy(&slot, p + pos, 8);
    if (slot == -1) break;
    if (pos + rs > len) {
      ctx->err = std::string(what) + ": truncated record";
      return FRT_ERR_INVALID;
    }
    const unsigned char* r = p + pos + 8;
    int16_t o;
    int32_t px, c;
    uint16_t it;
    float v[3 + FRT_MAX_FREQ + 6];
    memcpy(&o, r + 1, 2);
    memcpy(&px, r + 3, 4);
    memcpy(&it, r + 7, 2);
    memcpy(v, r + 9, sizeof(float) * (3 + F + 6));
    memcpy(&c, r + 9 + 4 * (3 + F + 6), 4);
    pos += rs;
    // init_rt's free-slot probe (rt_funcs.cc:117-124): select_index(0) hands out slot 0, and a ray
    // there whose first-bin photon count is 0 is removed
    if (restart && slot == 0 && v[3] == 0.f) continue;
    if (c < 0 || c >= ctx->hbox[box].ncell || px < 0 || o < 0 || o > kLmax || it >= kNtheta) {
      ctx->err = std::string(what) + ": ray outside the box or with an invalid order / pixel / angle index";
      return FRT_ERR_INVALID;
    }
    cell.push_back(c); pix.push_back(px); ord.push_back(o); ith.push_back(it); bx.push_back((uint16_t)box);
    for (int k = 0; k < 3; k++) g[k].push_back(v[k]);
    for (int nu = 0; nu < F; nu++) np[nu].push_back(v[3 + nu]);
    for (int k = 0; k < 6; k++) g[3 + k].push_back(v[3 + F + k]);
  }
  Ctl c;
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(copy_sync(ctx, &c, d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
  const size_t base = (size_t)c.nray[c.cur], m = cell.size();
  if (base + m > (size_t)d.ray_cap) {
    ctx->err = std::string(what) + ": ray pool capacity exceeded";
    return FRT_ERR_CAPACITY;
  }
  double inflight = 0.0;
  if (m) {
    const RayPool& P = d.pool[c.cur];
    CK(copy_sync(ctx, P.cell + base, cell.data(), 4 * m, cudaMemcpyHostToDevice));
    CK(copy_sync(ctx, P.pixel + base, pix.data(), 4 * m, cudaMemcpyHostToDevice));
    CK(copy_sync(ctx, P.order + base, ord.data(), 2 * m, cudaMemcpyHostToDevice));
    CK(copy_sync(ctx, P.itheta + base, ith.data(), 2 * m, cudaMemcpyHostToDevice));
    CK(copy_sync(ctx, P.box + base, bx.data(), 2 * m, cudaMemcpyHostToDevice));
    float* gp[9] = {P.xh, P.yh, P.zh, P.r, P.dr, P.x, P.y, P.z, P.time};
    for (int k = 0; k < 9; k++) CK(copy_sync(ctx, gp[k] + base, g[k].data(), 4 * m, cudaMemcpyHostToDevice));
    for (int nu = 0; nu < F; nu++) {
      CK(copy_sync(ctx, P.nphot + (size_t)nu * d.ray_cap + base, np[nu].data(), 4 * m, cudaMemcpyHostToDevice));
      for (float x : np[nu]) inflight += (double)x;
    }
  }
  if (m && d.pool[c.cur].col) {   // the restart records carry no columns: loaded rays start at 0
    double* col = d.pool[c.cur].col;
    CK(fill_sync(ctx, col + base, 0, sizeof(double) * m));
    CK(fill_sync(ctx, col + d.ray_cap + base, 0, sizeof(double) * m));
  }
  if (m && !restart) CK(fill_sync(ctx, d.dead + base, 0, m));
  c.nray[c.cur] = (int)(base + m);
  if (restart) c.in_flight += inflight * 1e60;   // photon ledger: physical photons of the loaded rays
  CK(copy_sync(ctx, d.ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice));
  return FRT_OK;
}

}  // namespace

extern "C" {

frt_status frt_read_rays(frt_ctx* ctx, int box, const void* buf, size_t len) {
  return append_ray_records(ctx, box, buf, len, true, "frt_read_rays");
}

frt_status frt_put_rays(frt_ctx* ctx, int box, const void* buf, size_t len) {
  return append_ray_records(ctx, box, buf, len, false, "frt_put_rays");
}

frt_status frt_take_rays(frt_ctx* ctx, int box, int in_step, void* buf, size_t cap, size_t* len) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  if (ctx->d.nbox != 1) {
    ctx->err = "frt_take_rays: a context of one box";
    return FRT_ERR_INVALID;
  }
  Dev& d = ctx->d;
  Ctl c;
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(cudaStreamSynchronize(ctx->s_dark));
  CK(copy_sync(ctx, &c, d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost));
  const int nr = std::min(c.nray[c.cur], d.ray_cap);
  // within a step (after its last C2Ray pass) the removal flags of the pool are the step's; between
  // steps they belong to the previous pool and every ray of the current one is live
  std::vector<uint8_t> dead(nr, 0);
  if (nr && in_step) CK(copy_sync(ctx, dead.data(), d.dead, (size_t)nr, cudaMemcpyDeviceToHost));
  long long live = 0;
  for (int i = 0; i < nr; i++) live += dead[i] ? 0 : 1;
  const int F = d.F;
  const size_t need = (size_t)live * ray_record_size(F) + 8;
  if (len) *len = need;
  if (!buf) return FRT_OK;
  if (cap < need) {
    ctx->err = "frt_take_rays: buffer too small";
    return FRT_ERR_INVALID;
  }
  std::vector<int16_t> ord(nr);
  std::vector<int32_t> pix(nr), cell(nr);
  std::vector<uint16_t> ith(nr);
  std::vector<float> g((size_t)nr * 9), np((size_t)nr * F);
  if ((st = frt_download_rays(ctx, box, ord.data(), pix.data(), ith.data(), cell.data(), g.data(), np.data())))
    return st;
  Bytes o{(unsigned char*)buf, 0, cap};
  long long x = 0;
  for (int i = 0; i < nr; i++) {
    if (dead[i]) continue;
    const float* v = &g[(size_t)i * 9];
    o.put<int64_t>(x++);
    o.put<bool>(true);
    o.put<int16_t>(ord[i]);
    o.put<int32_t>(pix[i]);
    o.put<uint16_t>(ith[i]);
    o.put<float>(v[0]); o.put<float>(v[1]); o.put<float>(v[2]);
    for (int nu = 0; nu < F; nu++) o.put<float>(np[(size_t)i * F + nu]);
    for (int k = 3; k < 9; k++) o.put<float>(v[k]);   // r dr x y z time
    o.put<int32_t>(cell[i]);
  }
  o.put<int64_t>(-1);
  // the context keeps none of its rays
  c.nray[c.cur] = 0;
  CK(copy_sync(ctx, &d.ctl->nray[c.cur], &c.nray[c.cur], sizeof(int), cudaMemcpyHostToDevice));
  return FRT_OK;
}

}  // extern "C"

// ---- adjoint of the next step's Gamma field ----------------------------------------------------
namespace {

frt_status adj_alloc(frt_ctx* ctx) {
  if (ctx->adj_ready) return FRT_OK;
  Dev& d = ctx->d;
  AdjDev& a = ctx->adj;
  a.cap = d.lit_cap;
  a.I = d.itercount;
  const size_t NC = (size_t)d.ncell_total, L = (size_t)a.cap, LI = L * (size_t)a.I;
  AL(a.flag, NC); AL(a.slot, NC); AL(a.src_of_cell, NC); AL(a.cell, L); AL(a.in_obj, L);
  AL(a.nH, L); AL(a.nHe, L); AL(a.y0h, L); AL(a.y0he, L); AL(a.crh, L); AL(a.crhe, L);
  AL(a.a, LI); AL(a.b, LI); AL(a.gh, LI); AL(a.ghe, LI);
  AL(a.abar, L); AL(a.bbar, L); AL(a.gbh, L); AL(a.gbhe, L); AL(a.nhbar, L);
  AL(a.dlbar, std::max<size_t>(1, (size_t)d.src_cap)); AL(a.count, 1); AL(a.err, 1); AL(a.J, 1);
  long long maxcell = 1;
  for (const BoxP& B : ctx->hbox) maxcell = std::max(maxcell, B.ncell);
  AL(ctx->adj_out, (size_t)maxcell);
  ctx->adj_ready = true;
  return FRT_OK;
}

// source cell -> context-wide source index, rebuilt after the source list changed
frt_status adj_source_map(frt_ctx* ctx) {
  if (!ctx->adj_src_stale) return FRT_OK;
  const size_t NC = (size_t)ctx->d.ncell_total;
  std::vector<int> soc(NC, -1);
  int s = 0;
  for (size_t b = 0; b < ctx->src_cell.size(); b++)
    for (size_t q = 0; q < ctx->src_cell[b].size(); q++, s++) soc[(size_t)ctx->hbox[b].cell0 + ctx->src_cell[b][q]] = s;
  CK(copy_sync(ctx, ctx->adj.src_of_cell, soc.data(), sizeof(int) * NC, cudaMemcpyHostToDevice));
  ctx->adj_src_stale = false;
  return FRT_OK;
}

}  // namespace

extern "C" {

frt_status frt_adjoint(frt_ctx* ctx, const frt_adj_objective* obj, double* J, double* dL, float* dnH) {
  if (!ctx || !obj) return FRT_ERR_INVALID;
  frt_status st = check_box(ctx, obj->box);
  if (st) return st;
  const BoxP& B = ctx->hbox[obj->box];
  for (int k = 0; k < 3; k++)
    if (obj->lo[k] < 0 || obj->hi[k] > B.n || obj->lo[k] > obj->hi[k]) {
      ctx->err = "frt_adjoint: objective sub-box outside the box";
      return FRT_ERR_INVALID;
    }
  if (ctx->d.subgrid) {
    ctx->err = "frt_adjoint differentiates the plain C2Ray model, not the sub-grid model";
    return FRT_ERR_STATE;
  }
  if (ctx->merged_any || ctx->restarted[obj->box]) {
    ctx->err = "frt_adjoint needs every ray to come from one source's cast: a merge has combined rays of "
               "several sources, or the rays were read from a restart file";
    return FRT_ERR_STATE;
  }
  st = adj_alloc(ctx);
  if (st) return st;
  st = adj_source_map(ctx);
  if (st) return st;
  Dev& d = ctx->d;
  AdjDev& a = ctx->adj;
  a.box = obj->box;
  for (int k = 0; k < 3; k++) {
    a.lo[k] = obj->lo[k];
    a.hi[k] = obj->hi[k];
  }
  cudaStream_t s = ctx->s_main;
  CK(cudaStreamSynchronize(ctx->s_dark));
  CK(cudaMemsetAsync(a.flag, 0, (size_t)d.ncell_total, s));
  launch_fill_i32(a.slot, -1, d.ncell_total, s);
  CK(cudaMemsetAsync(a.count, 0, sizeof(int), s));
  CK(cudaMemsetAsync(a.err, 0, sizeof(unsigned), s));
  CK(cudaMemsetAsync(a.J, 0, sizeof(double), s));
  CK(cudaMemsetAsync(a.dlbar, 0, sizeof(double) * std::max(1, d.src_cap), s));
  CK(cudaEventRecord(ctx->ev_t0, s));
  launch_adjoint(d, a, ctx->grid_rays, s);
  CK(cudaEventRecord(ctx->ev_t1, s));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  CK(cudaEventElapsedTime(&ctx->last_adjoint_ms, ctx->ev_t0, ctx->ev_t1));
  unsigned err = 0;
  double Jv = 0.0;
  CK(copy_sync(ctx, &err, a.err, sizeof err, cudaMemcpyDeviceToHost));
  CK(copy_sync(ctx, &Jv, a.J, sizeof Jv, cudaMemcpyDeviceToHost));
  if (err) {
    ctx->err = "frt_adjoint: " + std::string((err & 1u) ? "path_length exceeded " : "") +
               std::string((err & 2u) ? "path cells above the lit-cell capacity" : "");
    return FRT_ERR_CAPACITY;
  }
  if (J) *J = Jv;
  if (dL) {
    int s0 = 0;
    for (int b = 0; b < obj->box; b++) s0 += (int)ctx->src_cell[b].size();
    const size_t ns = ctx->src_cell[obj->box].size();
    std::vector<double> v(ns);
    if (ns) CK(copy_sync(ctx, v.data(), a.dlbar + s0, sizeof(double) * ns, cudaMemcpyDeviceToHost));
    for (size_t q = 0; q < ns; q++) {
      const double lum = ctx->src_lum[obj->box][q];
      dL[q] = lum != 0.0 ? v[q] / lum : 0.0;
    }
  }
  if (dnH) {
    launch_adjoint_gather(d, a, B.cell0, B.ncell, ctx->adj_out, s);
    CK(copy_sync(ctx, dnH, ctx->adj_out, sizeof(float) * (size_t)B.ncell, cudaMemcpyDeviceToHost));
  }
  return FRT_OK;
}

}  // extern "C"

// ---- field read-back without device allocation ---------------------------------------------
// frt_get_field gathers a lit-cell field (Gamma, photon counts) through a temporary device
// buffer of one box's size, taken with cudaMalloc and released with cudaFree. Some callers must
// not allocate there: an output hook that runs between steps while the ray pool was sized to
// fill the GPU (the allocation fails exactly when the run is largest), and drivers that keep
// the dark-cell stream running across the read (cudaFree waits for the whole device). The entry
// point below gathers into a fixed scratch array in the module's global memory instead and hands
// out at most FRT_NOALLOC_MAX_CELLS cells per call; a caller reads a larger box in windows.
#include <mutex>

namespace {

constexpr long long kNoAllocMaxCells = FRT_NOALLOC_MAX_CELLS;
// The scratch array: 4 MiB of static device memory, one per device the module is loaded on.
// The gather writes every element it later copies out, so nothing in it has to start at zero.
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocMaxCells];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
float* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Address of the scratch array on `device`, looked up once per device with that device current.
cudaError_t noalloc_scratch(int device, float** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
  if (!g_noalloc_ptr[device]) {
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return e;
    if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess) return e;
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (prev != device) {
      const cudaError_t e2 = cudaSetDevice(prev);
      if (e == cudaSuccess) e = e2;
    }
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = static_cast<float*>(p);
  }
  *out = g_noalloc_ptr[device];
  return cudaSuccess;
}

}  // namespace

extern "C" {

frt_status frt_get_sparse_field_noalloc(frt_ctx* ctx, int box, frt_field f, int bin, long long first_cell,
                                        long long count, float* host) {
  frt_status st = check_box(ctx, box);
  if (st) return st;
  Dev& d = ctx->d;
  const BoxP& B = ctx->hbox[box];
  const int F = d.F;
  int which = -1;
  switch (f) {
    case FRT_F_GAMMA_H1_TOT: which = 0; break;
    case FRT_F_GAMMA_HE1_TOT: which = 1; break;
    case FRT_F_GAMMA_H1_NU: which = 2 + bin; break;
    case FRT_F_GAMMA_HE1_NU: which = 2 + F + bin; break;
    case FRT_F_NGAM_NU: which = 2 + 2 * F + bin; break;
    default:
      ctx->err = "frt_get_sparse_field_noalloc: not a lit-cell field (GAMMA_*_TOT, GAMMA_*_NU, NGAM_NU)";
      return FRT_ERR_INVALID;
  }
  const bool per_bin = (f == FRT_F_GAMMA_H1_NU || f == FRT_F_GAMMA_HE1_NU || f == FRT_F_NGAM_NU);
  if (per_bin && (bin < 0 || bin >= F)) {
    ctx->err = "frt_get_sparse_field_noalloc: bin out of range";
    return FRT_ERR_INVALID;
  }
  if (per_bin && !d.per_bin) {
    ctx->err = "per-bin rates and photon counts are kept only with diag outputs or strict precision";
    return FRT_ERR_STATE;
  }
  if (count < 0 || first_cell < 0 || first_cell > B.ncell || count > B.ncell - first_cell) {
    ctx->err = "frt_get_sparse_field_noalloc: cell window outside the box";
    return FRT_ERR_INVALID;
  }
  if (count > kNoAllocMaxCells) {
    ctx->err = "frt_get_sparse_field_noalloc: count " + std::to_string(count) +
               " exceeds FRT_NOALLOC_MAX_CELLS (" + std::to_string(kNoAllocMaxCells) +
               "); read the box in windows";
    return FRT_ERR_INVALID;
  }
  if (count == 0) return FRT_OK;
  if (!host) return FRT_ERR_INVALID;
  float* scratch = nullptr;
  CK(noalloc_scratch(ctx->cfg.device, &scratch));
  CK(cudaStreamSynchronize(ctx->s_main));
  CK(cudaStreamSynchronize(ctx->s_dark));
  launch_gather_sparse(d, B.cell0 + first_cell, count, which, scratch, ctx->s_main);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, scratch, sizeof(float) * (size_t)count, cudaMemcpyDeviceToHost, ctx->s_main));
  CK(cudaStreamSynchronize(ctx->s_main));
  return FRT_OK;
}

}  // extern "C"

// ---- launch shapes and the autotuner ----------------------------------------------------------
namespace {

void tuning_out(const frt_ctx* ctx, frt_tuning* o) {
  const Tune& t = ctx->tune;
  *o = ctx->tune_measured;
  o->raypass_block = t.rp_block;
  o->raypass_blocks_per_sm = t.rp_grid;
  o->raypass_chunk = t.rp_chunk;
  o->walk_block = t.adv_block;
  o->walk_blocks_per_sm = t.adv_grid;
  o->cellpass_blocks_per_sm = t.lit_grid;
  o->split_blocks_per_sm = t.split_grid;
}

bool block_ok(int b) { return b >= 32 && b <= 256 && b % 32 == 0; }
bool grid_ok(int g) { return g >= 1 && g <= 32; }

// Equal shares [lo, hi) of n work items for k candidates.
void share(long long n, int k, int q, int* lo, int* hi) {
  *lo = (int)(n * q / k);
  *hi = (int)(n * (q + 1) / k);
}

}  // namespace

extern "C" {

frt_status frt_get_tuning(frt_ctx* ctx, frt_tuning* out) {
  if (!ctx || !out) return FRT_ERR_INVALID;
  tuning_out(ctx, out);
  return FRT_OK;
}

frt_status frt_set_tuning(frt_ctx* ctx, const frt_tuning* in) {
  if (!ctx || !in) return FRT_ERR_INVALID;
  if (!block_ok(in->raypass_block) || !(in->raypass_blocks_per_sm == 0 || grid_ok(in->raypass_blocks_per_sm)) ||
      in->raypass_chunk < 0 ||
      in->raypass_chunk > 65536 || !block_ok(in->walk_block) || !grid_ok(in->walk_blocks_per_sm) ||
      !(in->cellpass_blocks_per_sm == 0 || grid_ok(in->cellpass_blocks_per_sm)) || !grid_ok(in->split_blocks_per_sm)) {
    ctx->err = "frt_set_tuning: blocks 32..256 in multiples of 32, 1..32 blocks per SM, chunk 0..65536";
    return FRT_ERR_INVALID;
  }
  Tune t;
  t.rp_block = in->raypass_block;
  t.rp_grid = in->raypass_blocks_per_sm;
  t.rp_chunk = in->raypass_chunk;
  t.adv_block = in->walk_block;
  t.adv_grid = in->walk_blocks_per_sm;
  t.lit_grid = in->cellpass_blocks_per_sm;
  t.split_grid = in->split_blocks_per_sm;
  ctx->tune = t;
  ctx->tune_auto = false;
  ctx->tune_measured = frt_tuning{};
  ctx->graph_valid = false;
  return FRT_OK;
}

frt_status frt_autotune(frt_ctx* ctx, int steps, frt_tuning* out) {
  if (!ctx || steps < 1 || steps > 16) return FRT_ERR_INVALID;
  Dev& d = ctx->d;
  if (d.subgrid) {
    ctx->err = "frt_autotune times the plain model's kernels";
    return FRT_ERR_INVALID;
  }
  const int I = d.itercount;
  cudaStream_t s = ctx->s_main;
  const Tune t0 = ctx->tune;
  // candidate values per family; the ray pass and the cell pass get one candidate per C2Ray
  // iteration but the last (a different kernel), the walk and the compaction split their rays
  // into four equal ranges
  const int per_iter = std::max(1, I - 1);
  const bool tune_rp = !ctx->strict && I > 1;
  // (ray-pass grid 0: exactly the blocks resident on the SMs, one wave of the persistent kernel)
  ShapeSearch rp("raypass", Shape{t0.rp_block, t0.rp_grid, t0.rp_chunk}, {128, 256}, {0, 4, 8, 12, 16},
                 {0, 32, 128, 512}, per_iter);
  ShapeSearch adv("walk", Shape{t0.adv_block, t0.adv_grid, 0}, {128, 256}, {4, 8, 16}, {0}, 4);
  ShapeSearch lit("cellpass", Shape{256, t0.lit_grid, 0}, {256}, {0, 2, 4, 8, 16}, {0}, per_iter);
  ShapeSearch spl("split", Shape{256, t0.split_grid, 0}, {256}, {2, 4, 8, 16}, {0}, 4);
  // with three steps or more, the last two validate the search on whole graph steps (below)
  const int search_steps = steps >= 3 ? steps - 2 : steps;
  for (ShapeSearch* f : {&rp, &adv, &lit, &spl}) f->set_max_rounds(search_steps);
  constexpr int kEv = 2 * (4 + 16 + 16 + 4);
  std::vector<cudaEvent_t> ev(kEv, nullptr);
  auto destroy = [&]() {
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  };
  for (cudaEvent_t& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) {
      destroy();
      ctx->err = "frt_autotune: cudaEventCreate failed";
      return FRT_ERR_CUDA;
    }
  frt_status st = FRT_OK;
  double c_rp = 0, c_adv = 0, c_lit = 0, c_spl = 0;
  for (int round = 0; round < search_steps && st == FRT_OK; round++) {
    if ((st = step_inputs(ctx, nullptr, nullptr))) break;
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaStreamSynchronize(ctx->s_dark) != cudaSuccess) {
      st = FRT_ERR_CUDA;
      break;
    }
    Ctl c0;
    if (copy_sync(ctx, &c0, d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost) != cudaSuccess) {
      st = FRT_ERR_CUDA;
      break;
    }
    const long long nray = std::min(c0.nray[c0.cur], d.ray_cap);
    const std::vector<Shape> ca = adv.next_round(), cs = spl.next_round();
    const std::vector<Shape> cr = tune_rp ? rp.next_round() : std::vector<Shape>{rp.best()};
    const std::vector<Shape> cl = lit.next_round();
    int e = 0;
    std::vector<int> e_adv, e_spl, e_rp, e_lit;
    std::vector<long long> n_adv, n_spl;
    cudaMemcpyAsync(d.itheta_merge, ctx->h_ith_box, sizeof(uint16_t) * d.nbox, cudaMemcpyHostToDevice, s);
    if (d.nsrc) cudaMemcpyAsync(d.src_itheta, ctx->h_ith_src, sizeof(uint16_t) * d.nsrc, cudaMemcpyHostToDevice, s);
    note_step(ctx);
    cudaEventRecord(ctx->ev_t0, s);
    ctx->rays_moved = true;
    launch_clear_lit(d, ctx->grid_lit, s);
    launch_step_begin(d, s);
    for (int q = 0; q < (int)ca.size(); q++) {
      int lo, hi;
      share(nray, (int)ca.size(), q, &lo, &hi);
      e_adv.push_back(e);
      n_adv.push_back(hi - lo);
      cudaEventRecord(ev[e++], s);
      launch_walk(d, ctx->nsm * ca[q].grid, s, ca[q].block, lo, hi);
      cudaEventRecord(ev[e++], s);
    }
    launch_lit_number(d, ctx->grid_rays, s);
    launch_lit_init(d, ctx->strict, ctx->grid_lit, s);
    for (int it = 0; it < I; it++) {
      const bool last = it == I - 1;
      const Shape a = (!last && it < (int)cr.size()) ? cr[it] : rp.best();
      const Shape b = (!last && it < (int)cl.size()) ? cl[it] : lit.best();
      const bool ta = !last && it < (int)cr.size() && tune_rp, tb = !last && it < (int)cl.size();
      if (ta) {
        e_rp.push_back(e);
        cudaEventRecord(ev[e++], s);
      }
      launch_raypass(d, it, ctx->strict, ctx->nsm * a.grid, s, a.block, a.chunk);
      if (ta) cudaEventRecord(ev[e++], s);
      if (tb) {
        e_lit.push_back(e);
        cudaEventRecord(ev[e++], s);
      }
      launch_litpass(d, it, ctx->strict, true, ctx->nsm * b.grid, s);
      if (tb) cudaEventRecord(ev[e++], s);
    }
    launch_count_merge(d, ctx->grid_rays, s);
    for (int q = 0; q < (int)cs.size(); q++) {
      int lo, hi;
      share(nray, (int)cs.size(), q, &lo, &hi);
      e_spl.push_back(e);
      n_spl.push_back(hi - lo);
      cudaEventRecord(ev[e++], s);
      launch_split_range(d, ctx->nsm * cs[q].grid, lo, hi, s);
      cudaEventRecord(ev[e++], s);
    }
    launch_swap(d, s);
    // the dark-cell pass after the timed kernels, on the same stream: no concurrent kernel
    // perturbs the candidates' times
    launch_dark(d, ctx->strict, true, ctx->grid_dark, s);
    launch_cast(d, s);
    cudaMemcpyAsync(ctx->h_ctl, d.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(ctx->ev_t1, s);
    if ((st = finish_step(ctx, nullptr))) break;
    const Ctl& c1 = *ctx->h_ctl;
    auto ms = [&](int k) {
      float x = 0.f;
      return cudaEventElapsedTime(&x, ev[k], ev[k + 1]) == cudaSuccess ? (double)x : -1.0;
    };
    for (size_t q = 0; q < e_adv.size(); q++)
      if (n_adv[q] > 0 && ms(e_adv[q]) > 0) adv.record((int)q, 1e6 * ms(e_adv[q]) / (double)n_adv[q]);
    for (size_t q = 0; q < e_spl.size(); q++)
      if (n_spl[q] > 0 && ms(e_spl[q]) > 0) spl.record((int)q, 1e6 * ms(e_spl[q]) / (double)n_spl[q]);
    for (size_t q = 0; q < e_rp.size(); q++)
      if (c1.crossings > 0 && ms(e_rp[q]) > 0) rp.record((int)q, 1e6 * ms(e_rp[q]) / (double)c1.crossings);
    for (size_t q = 0; q < e_lit.size(); q++)
      if (c1.n_lit > 0 && ms(e_lit[q]) > 0) lit.record((int)q, 1e6 * ms(e_lit[q]) / (double)c1.n_lit);
    adv.end_round();
    spl.end_round();
    if (tune_rp) rp.end_round();
    lit.end_round();
    c_rp = rp.best_cost();
    c_adv = adv.best_cost();
    c_lit = lit.best_cost();
    c_spl = spl.best_cost();
  }
  destroy();
  if (st) return st;
  Tune t = t0;
  if (tune_rp) {
    t.rp_block = rp.best().block;
    t.rp_grid = rp.best().grid;
    t.rp_chunk = rp.best().chunk;
  }
  t.adv_block = adv.best().block;
  t.adv_grid = adv.best().grid;
  t.lit_grid = lit.best().grid;
  t.split_grid = spl.best().grid;
  if (steps >= 3) {
    // The search times each kernel family alone, with no dark pass beside it; in the step graph
    // the dark pass shares the SMs with the lit-cell chain. So the search's shapes and the
    // starting ones each run one whole graph step, and the faster per crossing is kept.
    double per_cross[2] = {0.0, 0.0};
    const Tune cand[2] = {t, t0};
    ctx->tune_auto = false;
    for (int k = 0; k < 2 && st == FRT_OK; k++) {
      ctx->tune = cand[k];
      ctx->graph_valid = false;
      frt_step_stats ss{};
      st = frt_step(ctx, nullptr, nullptr, &ss);
      if (st == FRT_OK && ss.crossings > 0) per_cross[k] = (double)ctx->last_step_ms / (double)ss.crossings;
    }
    if (st) return st;
    if (per_cross[1] > 0.0 && per_cross[0] > per_cross[1]) t = t0;
  }
  ctx->tune = t;
  ctx->tune_auto = true;
  ctx->graph_valid = false;
  frt_tuning m{};
  m.steps = steps;
  m.raypass_ns_per_crossing = tune_rp && c_rp < 1e299 ? c_rp : 0.0;
  m.walk_ns_per_ray = c_adv < 1e299 ? c_adv : 0.0;
  m.cellpass_ns_per_cell = c_lit < 1e299 ? c_lit : 0.0;
  m.split_ns_per_ray = c_spl < 1e299 ? c_spl : 0.0;
  ctx->tune_measured = m;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[tune_key(ctx, ctx->last.rays_alive)] = t;
  }
  if (out) tuning_out(ctx, out);
  return FRT_OK;
}

}  // extern "C"
