// Device-side data layout of an RT context and the kernel launchers shared by the .cu files.
//
// HBM layout (all structure-of-arrays, 4-byte fields unless noted):
//  * dense cell state, one entry per cell of every box; boxes are concatenated, each starting
//    on a 1024-cell tile boundary (tile -> box table), cells in C order (i, j, k) with k fastest
//    like the reference's [Nx][Ny][Nz] arrays;
//  * a compact list of the cells touched by a ray segment in the current step ("lit" cells)
//    with the per-iteration C2Ray state of just those cells, so that the 5 C2Ray iterations
//    only revisit lit cells while all other cells do their whole step in one streaming pass;
//  * two ray pools (the current one and the one the next step compacts into) indexed by ray,
//    plus the step's path segments of the moved rays, packed in moved-list order;
//  * a control block with the pool counts, lit count, error word and per-step totals.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/flexrt.h"
#include "frt_physics.cuh"

namespace frt {


enum : unsigned { ERR_RAY_CAP = 1u, ERR_PATH = 2u, ERR_LIT_CAP = 4u, ERR_BIN = 8u };

struct RayPool {
  int* cell;          // local cell index (path[0].ind)
  uint16_t* box;
  int16_t* order;
  int* pixel;
  uint16_t* itheta;
  float *xh, *yh, *zh;
  float* nphot;       // [F][cap]
  float *r, *dr, *x, *y, *z, *time;
  // opt-in optical-depth limit (frt_set_tau_limit; null when off): the HI and HeI column
  // densities ([2][cap], cm^-2 proper, FP64) each ray crossed since its cast
  double* col;
};

struct Ctl {
  int nray[2];             // live rays in pool 0 / 1
  int cur;                 // current pool
  int n_lit;               // lit cells this step
  int n_lit_prev;
  unsigned err;
  int any_merge;           // some box has nphot_merge > 0
  // moved rays this step (high 32 bits) and their segments (low 32 bits), counted together so
  // that one atomicAdd gives a tile of the walk both bases (k_advance)
  unsigned long long mv_seg;
  int ord_surv;            // live rays kept by the ordered compaction (k_order_scan)
  int if_changed;          // I-front budget: some crossing's entry sum changed in the last round
  long long rays_moved, crossings, split, merged, killed, cast;
  double emitted, deposited, killed_ph, overlap, in_flight;
};

struct Dev {
  // sizes
  int nbox, F, PL, itercount, hpx_lvl;
  int ray_cap, lit_cap, src_cap, nsrc;
  long long ncell_total, ntile;
  int outputs;             // FRT_OUT_*
  float nhe_to_nh;
  float const_clump;
  double tau_max;          // opt-in: remove rays whose optical depth exceeds it in every bin (0: off)
  // per-box
  BoxP* box;
  long long* count;        // live rays per box (count_rays)
  int* need_hist;          // per box
  int* hist;               // [nbox][kPdfBins]
  uint16_t* itheta_merge;  // per box
  double* lg;              // per box (log10 nphot_min, PDF bin width) for calc_nphot_merge
  double pi_sf_3, log4;    // pi*safety_factor/3. and log(4.) (l_from_r, ray_tracing.cc:89)
  // spectrum constants
  float spectrum[FRT_MAX_FREQ];
  double sigH1_d[FRT_MAX_FREQ], sigHe1_d[FRT_MAX_FREQ];
  float sigH1_f[FRT_MAX_FREQ], sigHe1_f[FRT_MAX_FREQ];
  float sigH1_l2[FRT_MAX_FREQ], sigHe1_l2[FRT_MAX_FREQ];   // the same times log2(e)
  int nho;                 // leading bins with sigma_HeI = 0 (HI alone absorbs)
  double sigH1_0, sigH1_912;
  // tables
  const float* rot;        // [kNtheta][2][9] forward, inverse
  const float4* pix_tab;   // HEALPix NEST pixel centres of orders 0..kPixTabMax, (float) of pix2vec
  // dense cells
  int16_t* tile_box;
  float *nH, *nHe, *nH1, *nHe1, *f_H1, *f_He1, *temp, *clump, *ne, *heat, *cool, *avg_nh1, *avg_nhe1, *treion;
  uint8_t *treion_flag, *lit_flag;
  int* lit_slot;
  float *nH1_prev, *n_tot, *dne_dt;                              // unfused path
  float* rho;              // proper density, on the device once a cosmological expansion ran
  // hydro snapshots (update_hydro_step): the previous snapshot's density and d(delta)/dt of the
  // temperature equation (both from the second switch on), and the ionised fractions an
  // expansion kept (read by a switch right after it)
  float *rho_prev, *ddelta, *frac_h2, *frac_he2;
  float *rec_h2, *rec_he2, *recrate_h2, *recrate_he2, *mfp, *mfp912, *if_speed, *inc_flux;  // diag
  // lit cells
  int* l_cell;
  uint16_t* l_box;          // box of the lit cell (k_lit_init), so the cell passes reach BoxP in one load
  float *l_nh, *l_nhe, *l_y0h, *l_y0he, *l_crec_h, *l_crec_he, *l_rec_h2, *l_rec_he2;
  float* l_nh1_old;
  // pairs (H, He) side by side: a crossing gathers both averages in one 8-byte load and adds both
  // rates in one vector reduction
  float2* l_avg;           // iteration-averaged (n_HI, n_HeI)
  float2* l_acc;           // (Gamma_HI, Gamma_HeI) summed over the crossings of this iteration
  float2* l_heat;          // bin-weighted photo-heating sums (HI, HeI) (mixed, core outputs)
  float *l_acc_nu_h, *l_acc_nu_he, *l_ngam;   // [F][lit_cap]
  int per_bin;                               // keep per-bin rates (diag outputs or strict)
  float cH1_f[FRT_MAX_FREQ], cHe1_f[FRT_MAX_FREQ];  // h (h_eV nu - Eth)/h_eV
  // rays
  RayPool pool[2];
  int4* mv_hdr;            // [ray_cap] moved ray q: {pool index, first packed segment, segments, box}
  int2* pk;                // [ray_cap * PL] packed segments {cell, then lit slot; dist bits | head bit}, moved-list order
  uint8_t* dead;
  int* ray_bin;            // merge bin of a candidate or -1
  uint8_t* merged_flag;
  int* bin_base;           // [ncell_total * 12*4^lm] or NULL when merging is unreachable
  // sources
  int* src_cell;           // local cell
  uint16_t* src_box;
  double* src_lum;
  float* src_ray_dt;
  uint16_t* src_itheta;
  uint8_t* src_own;          // null, or 1 for the sources this context casts (a share of a box's sources)
  int* src_pos;              // pool position of a source's first new ray this step (k_cast_offsets)
  // control
  Ctl* ctl;
  int* rp_queue;           // [kMaxIterQueue] ray-pass work counters, one per C2Ray iteration (chunked queue)
  // sub-grid model (frt_set_subgrid; frt_subgrid.cu): the RadHydro time and HI-fraction tables in
  // the reference's layout, the linear -> non-linear overdensity table, the cosmic times the model
  // uses, and the cells' mean free paths (per cell, and per lit cell during the iteration)
  int subgrid;
  const float *sg_time, *sg_fh1, *sg_tdnl, *sg_ds, *sg_dnl;
  float sg_tinit, sg_t12, sg_t8, sg_tcap, sg_tre_dom[3];
  float sg_fH1_0, sg_fHe1_0, sg_temp0;   // initial neutral fractions (interp_nh1's cap) and the neutral gas temperature
  float* l_mfp;
  // pool order: with `ordered` the compaction keeps the reference's slot order (live rays in
  // order, then the children in the order of their parents; k_compact_split<1,2>)
  int ordered;
  int2 *ord_cnt, *ord_off;   // per block of 256 pool rays: (live, split) counts and offsets
  // I-front tracking (ifront = TRUE; frt_ifront.cu): the fraction of each cell the fronts have
  // passed and its maximum, the crossing times (total, per tenth of the cell, with the tenths
  // passed as bits), the tcross / neutral flags (bits 0 / 1), the last step's change of fion,
  // the time the cell passed half-ionised; per lit cell fion at the step's start, the atoms of
  // its neutral part and the photon counts of the iteration ([3][lit_cap]: absorbed by the
  // neutral part, the same times sigma_eff_rh times path, entering the neutral part); the
  // budget cells' crossings in ray order (CSR over lit slots); per packed segment its moved ray,
  // the absorbed sum it found on entry, the photons entering the neutral part per bin
  // ([F][ray_cap * PL]) and whether the ray reached it
  int ifront;
  float *fion, *fion_max, *tcross, *tcross_new, *delta_fion, *treion_out;
  uint16_t* tcross_bits;
  uint8_t* if_flags;
  float* l_fion;
  double *l_free, *l_ng3;
  int *if_cnt, *if_off, *if_fill, *if_list;
  int* xs_q;
  double *xs_S, *xs_E;
  uint8_t* xs_reach;
  long long xs_cap;
};

constexpr int kMaxIterQueue = 16;

// The blocks of `kernel` at `block` threads that fit on all SMs at once (its occupancy times the SM
// count), remembered per kernel and block size (a host-side query: no work is enqueued, so it may
// run while a stream is being captured).
template <typename K>
inline int resident_grid(K kernel, int block) {
  struct Entry {
    const void* k;
    int block, grid;
  };
  static Entry cache[64];
  static int n = 0;
  static std::mutex mu;
  std::lock_guard<std::mutex> lock(mu);
  for (int i = 0; i < n; i++)
    if (cache[i].k == (const void*)kernel && cache[i].block == block) return cache[i].grid;
  int dev = 0, nsm = 148, nb = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, block, 0) != cudaSuccess || nb < 1) nb = 1;
  const int g = nb * nsm;
  if (n < 64) cache[n++] = Entry{(const void*)kernel, block, g};
  return g;
}


// Launch shapes of the tunable kernels (frt_tune.h picks them; the defaults are the untuned
// shapes). Grids are in blocks per SM; rp_grid = 0 launches the persistent ray pass with exactly
// the blocks resident at once (one wave), the default: with 8 blocks per SM requested and 5
// resident, the second wave of blocks left 40 % of the slots idle while it ran. rp_chunk = 0 gives
// each warp of the ray pass a static slice of the moved-ray list, rp_chunk > 0 lets warps take
// chunks of that many rays from a device-side queue (one atomicAdd per chunk).
struct Tune {
  int rp_block = 256, rp_grid = 0, rp_chunk = 0;
  int adv_block = 256, adv_grid = 8;
  int lit_grid = 0;
  int split_grid = 8;
  bool operator==(const Tune& o) const {
    return rp_block == o.rp_block && rp_grid == o.rp_grid && rp_chunk == o.rp_chunk && adv_block == o.adv_block &&
           adv_grid == o.adv_grid && lit_grid == o.lit_grid && split_grid == o.split_grid;
  }
};

// Buffers of the adjoint of one step's Gamma field (frt_adjoint.cu). Cells on the paths of the
// step's rays get a slot (in cell order); per slot the constants of the cell, the C2Ray iterates
// a^k, b^k and the ray-pass rates of every iteration k, and the adjoint accumulators.
struct AdjDev {
  int cap, I, box;
  int lo[3], hi[3];
  uint8_t* flag;           // [ncell_total] cell on a path
  int* slot;               // [ncell_total] slot or -1
  int* cell;               // [cap]
  uint8_t* in_obj;         // [cap] inside the objective sub-box
  double *nH, *nHe, *y0h, *y0he, *crh, *crhe;   // [cap]
  double *a, *b, *gh, *ghe;                    // [I][cap]
  double *abar, *bbar, *gbh, *gbhe, *nhbar;    // [cap]
  int* src_of_cell;        // [ncell_total] source index (context-wide) of a source cell, else -1
  double* dlbar;           // [nsrc] sum over the source's rays of n0 * dJ/dn0
  int* count;              // slots in use
  unsigned* err;           // path overflow / slot capacity
  double* J;               // objective
};

inline __host__ __device__ int grid_for(long long n, int block, int maxblocks) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > maxblocks) g = maxblocks;
  return (int)g;
}

// ---- launchers (frt_geom.cu) ----------------------------------------------------------
void launch_step_begin(const Dev& d, cudaStream_t s);
void launch_advance(const Dev& d, int grid, cudaStream_t s, int block = 256, int pack_grid = 0);
// k_advance alone, over pool rays [r_begin, r_end)
void launch_walk(const Dev& d, int grid, cudaStream_t s, int block = 256, int r_begin = 0, int r_end = 0x7fffffff);
void launch_lit_number(const Dev& d, int grid, cudaStream_t s);   // k_lit_compact + k_pk_slots
// the same with the lit cells numbered in strict cell order (chunk: ncell/4096 ints of scratch)
void launch_lit_number_ordered(const Dev& d, int* chunk, long long nchunk, int grid, cudaStream_t s);
void launch_count(const Dev& d, int grid, cudaStream_t s);
void launch_merge(const Dev& d, int grid, cudaStream_t s);
void launch_count_merge(const Dev& d, int grid, cudaStream_t s);   // the step's count + merge
void launch_split_compact(const Dev& d, int grid, cudaStream_t s);
// k_compact_split over pool rays [r_begin, r_end) without the pool swap; then launch_swap
void launch_split_range(const Dev& d, int grid, int r_begin, int r_end, cudaStream_t s);
void launch_swap(const Dev& d, cudaStream_t s);
void launch_cast(const Dev& d, cudaStream_t s);
void launch_cast_per_source(const Dev& d, cudaStream_t s);   // one launch per source
void launch_fill_i32(int* p, int v, long long n, cudaStream_t s);
constexpr int kPixTabMax = 9;
inline long long pix_tab_offset(int order) { return 4ll * ((1ll << (2 * order)) - 1); }   // sum of 12*4^k, k < order
void launch_pix_table(float4* tab, cudaStream_t s);
void launch_cosmo_expansion(const Dev& d, int box, float ratio, double rho_factor, int grid, cudaStream_t s);
// the cells of update_hydro_step for box `box` (d.rho holds the new snapshot's proper density)
void launch_hydro_switch(const Dev& d, int box, bool cached_fractions, float avg_rho_prev, float dt_snap, int grid,
                         cudaStream_t s);
// ---- launchers (frt_phys.cu) ----------------------------------------------------------
void launch_lit_init(const Dev& d, bool strict, int grid, cudaStream_t s);
void launch_raypass(const Dev& d, int iter, bool strict, int grid, cudaStream_t s, int block = 256, int chunk = 0);
void launch_litpass(const Dev& d, int iter, bool strict, bool fused_thermal, int grid, cudaStream_t s,
                    int s_begin = 0, int s_end = 0x7fffffff);
void launch_dark(const Dev& d, bool strict, bool fused_thermal, int grid, cudaStream_t s);
void launch_thermal_all(const Dev& d, bool strict, int grid, cudaStream_t s);
void launch_clear_lit(const Dev& d, int grid, cudaStream_t s);
void launch_gather_sparse(const Dev& d, long long cell0, long long ncell, int which, float* out, cudaStream_t s);
// ---- sub-grid model (frt_subgrid.cu) ---------------------------------------------------
void launch_sg_step(const Dev& d, cudaStream_t s);                         // the step's overdensity domain
void launch_sg_mfp_init(const Dev& d, cudaStream_t s);                     // init()'s mean free paths
void launch_sg_lit_init(const Dev& d, int grid, cudaStream_t s);
void launch_sg_raypass(const Dev& d, int iter, int grid, cudaStream_t s);
void launch_sg_litpass(const Dev& d, int iter, bool fused_thermal, int grid, cudaStream_t s);
void launch_sg_dark(const Dev& d, bool fused_thermal, int grid, cudaStream_t s);
void launch_sg_thermal_all(const Dev& d, int grid, cudaStream_t s);
void launch_if_lists(const Dev& d, int grid, cudaStream_t s);              // front cells' crossings in ray order
void launch_if_round(const Dev& d, int iter, int grid, cudaStream_t s);    // ray pass + budget pass
void launch_if_final(const Dev& d, int iter, int grid, cudaStream_t s);    // the last iteration's ray updates
// ---- adjoint (frt_adjoint.cu) --------------------------------------------------------
void launch_adjoint(const Dev& d, const AdjDev& a, int grid, cudaStream_t s);
void launch_adjoint_gather(const Dev& d, const AdjDev& a, long long cell0, long long ncell, float* out,
                           cudaStream_t s);

}  // namespace frt
