/* flexrt.h -- C ABI of the B200 (sm_100a) radiative-transfer step.
 *
 * Drop-in boundary for the per-timestep RT path of FlexRT. The reference is one C++/OpenMP
 * program whose driver (main.cc:108-264) calls void(void) step functions on process-global
 * arrays. Each entry point below replaces one of those functions (cited per declaration); the
 * state they share lives on the GPU inside an frt_ctx instead of in globals. Host arrays are
 * borrowed only for the duration of a call. Every entry point returns an frt_status; none
 * aborts, and device-side failures (ray-pool or path overflow) come back as FRT_ERR_CAPACITY.
 *
 * Plain C2Ray mode of the reference: c2ray_iter = TRUE, subgrid = FALSE, ifront = FALSE,
 * multi_freq = TRUE, case-B recombination, temperature evolution on (user_inputs.h:6-25).
 * A context may hold several independent periodic boxes (batched ensemble); single-box use
 * is nbox = 1.
 */
#ifndef FLEXRT_H
#define FLEXRT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FRT_MAX_FREQ 8
#define FRT_MAX_PATH 16
#define FRT_NTHETA 42875 /* 35^3 random Euler-angle triples (healpix_funcs.cc:8-9) */

typedef int frt_status;
enum {
  FRT_OK = 0,
  FRT_ERR_INVALID = 1,  /* bad argument / configuration */
  FRT_ERR_CAPACITY = 2, /* ray pool, lit-cell list or per-ray path capacity exceeded */
  FRT_ERR_TIMEOUT = 3,  /* a bounded device wait ran out */
  FRT_ERR_CUDA = 4,     /* CUDA runtime error (message via frt_last_error) */
  FRT_ERR_STATE = 5     /* call out of order (e.g. step before sources/gas are set) */
};

enum { FRT_PREC_MIXED = 0, FRT_PREC_STRICT = 1 };
enum { FRT_OUT_CORE = 0, FRT_OUT_DIAG = 1 };

typedef struct frt_ctx frt_ctx;

/* One periodic box. All boxes of a context share the spectrum and the solver constants. */
typedef struct {
  int n;                /* cells per side: Nx = Ny = Nz (user_inputs.h:75-77) */
  double box_hmpc;      /* comoving side in h^-1 Mpc; Lx0 = box*1e3/hh kpc (user_inputs.h:92) */
  float zz;             /* snapshot redshift; a = 1/(1+zz) (gas_funcs.cc:563-595) */
  float cl_factor;      /* simulated / true speed of light (user_inputs.h:84) */
  int ray_per_cell_max; /* merge threshold parameter (global_variables.cc:40), 22 */
  double rkill_cm;      /* rays with comoving r above this are removed after the advance; 0 = never */
} frt_box_desc;

typedef struct {
  int nfreq;                        /* Nfreq (user_inputs.h:78) */
  double nu_phot[FRT_MAX_FREQ];     /* bin frequencies in Hz (user_inputs.h:95) */
  float spectrum[FRT_MAX_FREQ];     /* photon fraction per bin (set_spectrum, gas_funcs.cc:44-70) */
  int itercount;                    /* C2Ray iterations (user_inputs.h:85), 5 */
  int path_length;                  /* segments stored per ray per step (user_inputs.h:107) */
  int hpx_lvl;                      /* casting / merging HEALPix order (user_inputs.h:81) */
  float safety_factor;              /* split when beam area > dx^2/safety_factor (user_inputs.h:86) */
  float tstep_factor;               /* user_inputs.h:82 */
  float nl_const;                   /* user_inputs.h:83 */
  float const_clump;                /* user_inputs.h:87 */
  float fH1_0, fHe1_0, fHe2_0;      /* initial ionisation state (user_inputs.h:98-100) */
  float temp_0;                     /* initial temperature (user_inputs.h:96) */
  int nbox;
  const frt_box_desc* boxes;
  long long ray_capacity;           /* device ray-pool slots (all boxes) */
  long long lit_capacity;           /* cells touched by rays in one step (all boxes); 0 = all cells */
  long long src_capacity;           /* sources (all boxes) */
  int precision;                    /* FRT_PREC_MIXED (FP32 + FP64 where x_HI < 1e-3) or FRT_PREC_STRICT */
  int outputs;                      /* FRT_OUT_CORE: the state, Gamma totals and heating rates;
                                       FRT_OUT_DIAG also keeps the output-only fields: per-bin Gamma and
                                       photon counts (ngam_nu, io_funcs.cc:387), mfp, recrate, u_nu, vIF.
                                       Strict precision keeps the per-bin fields in either mode. */
  int device;                       /* CUDA device ordinal */
} frt_config;

/* Per-cell fields addressable by frt_get_field / frt_set_field, C order [i][j][k] with k
 * fastest; the *_NU fields carry nfreq values per cell, [cell][nu]. Names follow the reference's
 * globals (global_variables.cc:78-260). */
typedef enum {
  FRT_F_RHO = 0, FRT_F_NH, FRT_F_NHE, FRT_F_NH1, FRT_F_NHE1, FRT_F_NH2, FRT_F_NHE2, FRT_F_NE, FRT_F_N_TOT,
  FRT_F_F_H1, FRT_F_F_HE1, FRT_F_F_H2, FRT_F_F_HE2, FRT_F_TEMP, FRT_F_CLUMP, FRT_F_AVG_NH1, FRT_F_AVG_NHE1,
  FRT_F_GAMMA_H1_TOT, FRT_F_GAMMA_HE1_TOT, FRT_F_HEAT_RATE, FRT_F_COOL_RATE, FRT_F_TREION,
  FRT_F_TREION_FLAG /* as float 0/1 */, FRT_F_DNE_DT, FRT_F_RECOMB_H2, FRT_F_RECOMB_HE2, FRT_F_RECRATE_H2,
  FRT_F_RECRATE_HE2, FRT_F_MFP, FRT_F_MFP_912, FRT_F_IF_SPEED, FRT_F_INC_FLUX,
  FRT_F_GAMMA_H1_NU, FRT_F_GAMMA_HE1_NU, FRT_F_NGAM_NU, FRT_F_U_NU,
  /* I-front tracking (frt_set_subgrid with ifront): the fraction of the cell the fronts passed, its
   * maximum, the crossing time, the last step's change of fion, the time the cell passed
   * half-ionised, tcross_flag and neutral_flag (as float 0/1), and the crossing times of the
   * tenths of the cell ([ncell][10]) */
  FRT_F_FION, FRT_F_FION_MAX, FRT_F_TCROSS, FRT_F_DELTA_FION, FRT_F_TREION_OUT, FRT_F_TCROSS_FLAG,
  FRT_F_NEUTRAL_FLAG, FRT_F_TCROSS_NEW,
  FRT_F_COUNT
} frt_field;

/* Per-step totals (device-computed). Photon counts are physical photons (not 1e60-normalised). */
typedef struct {
  long long rays_alive;      /* after the step (after cast) */
  long long rays_moved;      /* rays advanced this step */
  long long crossings;       /* ray-cell crossings = stored path segments (sum of ray_end) */
  long long lit_cells;       /* cells touched by at least one segment */
  long long rays_split;      /* parents split */
  long long rays_merged;     /* rays merged away */
  long long rays_killed;     /* removed below nphot_min */
  long long rays_cast;       /* new rays */
  double photons_emitted;    /* sum of nphot of the new rays */
  double photons_deposited;  /* photons entering Gamma_HI + Gamma_HeI on the last C2Ray iteration */
  double photons_killed;     /* photons left in rays removed below nphot_min */
  double photons_overlap;    /* photons both dumped into a cell and left in the killed ray */
  double photons_in_flight;  /* sum of nphot over live rays after the step */
  double t;                  /* simulation time after the step [s] */
  double dt;                 /* time step [s] */
  unsigned int error_flags;  /* device error word (0 = ok) */
  unsigned int pad;
} frt_step_stats;

/* ---- life cycle ----------------------------------------------------------------------- */
frt_status frt_create(const frt_config* cfg, frt_ctx** out);
frt_status frt_destroy(frt_ctx* ctx);
const char* frt_last_error(const frt_ctx* ctx);
/* Copy of the rotation coefficient table (FRT_NTHETA x 2 x 9 floats: forward, inverse) that the
 * context built from the reference's float expressions (healpix_funcs.cc:21-39, 102-143). */
frt_status frt_rotation_table(const frt_ctx* ctx, float* out);
/* The same table without a context (host only; no GPU needed). */
frt_status frt_build_rotation_table(float* out);

/* ---- set-up (one call per box) ------------------------------------------------------------ */
/* Gas set-up of the first snapshot: rho from the density cube (1+delta, as read by get_ugas,
 * io_funcs.cc:33-62, times a^-3, gas_funcs.cc:601-610), then init() (init_funcs.cc:10-142). */
frt_status frt_init_gas(frt_ctx* ctx, int box, const float* delta1);
/* Sources gridded per cell in (i,j,k) order as read_source_catalog produces them
 * (io_funcs.cc:157-233): ijk[3*s..3*s+2], lum[s] in photons/s. */
frt_status frt_set_sources(frt_ctx* ctx, int box, int nsrc, const int32_t* ijk, const double* lum);
/* Per-cell clumping factor written over set_clump()'s constant every step (NULL = constant). */
frt_status frt_set_clump_field(frt_ctx* ctx, int box, const float* clump);
frt_status frt_set_field(frt_ctx* ctx, int box, frt_field f, const float* host);
frt_status frt_get_field(frt_ctx* ctx, int box, frt_field f, float* host);

/* ---- the reference's step functions ------------------------------------------------------- */
/* init_rt (rt_funcs.cc:36-126, input_grid = FALSE) */
frt_status frt_init_rt(frt_ctx* ctx);
/* update_dt (rt_funcs.cc:9-12); dt_out[box] may be NULL */
frt_status frt_update_dt(frt_ctx* ctx, float* dt_out);
/* update_cosmo_expansion (gas_funcs.cc:460-548) followed by update_dt, as main.cc:219-237 calls
 * them after new_rays: per box, the scale factors of this step's end and start (a_current[box],
 * a_prev[box], as the caller's cosmic-time table gives them, gas_funcs.cc:461-465). The cell size
 * and ray positions scale by a_current/a_prev, the proper density by (a_prev/a_current)^3, and the
 * number densities follow from it with the ionised fractions kept. */
frt_status frt_update_cosmo_expansion(frt_ctx* ctx, const float* a_current, const float* a_prev);
/* update_hydro_step to a later hydro snapshot of one box (gas_funcs.cc:554-752), with the
 * get_nphot_min_max that follows it (main.cc:221-222); call it where main.cc does, after new_rays
 * and frt_update_cosmo_expansion. delta1: the new snapshot's 1+delta cube as get_ugas reads it
 * (io_funcs.cc:33-62); a_rt: the scale factor at the current time (gas_funcs.cc:566); dt_snap: the
 * cosmic time from this snapshot to the next (gas_funcs.cc:711); zz: this snapshot's redshift; the
 * new sources gridded per cell as read_source_catalog leaves them (io_funcs.cc:157-233). The
 * proper density becomes the new cube's times a_rt^-3, the cell size Lx0 a_rt / N, n_H and n_He
 * follow from it, the ionised densities keep the box's ionised fractions, and n_HI = n_H - n_HII;
 * the rays in flight keep their records. From the second switch on, d(delta)/dt between the
 * last two snapshots enters the temperature equation (gas_funcs.cc:399, 711). The new source
 * list replaces the old one (an owner mask, frt_set_source_owner, is cleared). */
frt_status frt_update_hydro_step(frt_ctx* ctx, int box, const float* delta1, float a_rt, float dt_snap, float zz,
                                 int nsrc, const int32_t* ijk, const double* lum);
/* The sub-grid RadHydro model of the reference (subgrid = TRUE with equilibrium = TRUE,
 * user_inputs.h:11-15), with or without I-front tracking: photo-ionisation equilibrium mean free paths in ionised
 * cells, HI fractions interpolated in the RadHydro tables (get_gamma_interp / interp_nh1,
 * subgrid.cc:257-647), the sub-grid ray deposition (ray_tracing.cc:764-856) and heating / cooling
 * (gas_funcs.cc:134-242, 362-418). Call after the gas set-up and the set-up cast, as main.cc:86-90
 * imports the tables; every later step runs the sub-grid model. The tables are the reference's
 * arrays after import_subgrid_file / import_delta_over_sigma_table (subgrid.cc:20-95): time_RH and
 * fh1_RH in its [Nt][3][3][3] layout, filled at the gamma index q + 1 (Nt * 27 + 1 floats with the
 * last row's spill), times in s; the cosmic times are the reference's cosmic_time() at zinit,
 * z = 12, 8, 5.5 and at the three RadHydro reionisation redshifts. With ifront != 0 (the
 * reference's default, user_inputs.h:11) every cell starts with no front passed (fion = 0,
 * rt_funcs.cc:49-69) and the neutral part of a cell absorbs the photons of the rays that reach it
 * in the order of the reference's ray slots, up to its atoms (ray_tracing.cc:863-919); the fronts
 * then advance by update_fion (subgrid.cc:694-751). The context then keeps its rays in that order
 * and resolves the order-dependent absorption by rounds that run to a fixed point; frt_step runs
 * its kernels without a graph. A step whose budgets do not settle returns FRT_ERR_STATE. The
 * phased step, the autotuner and the adjoint stay with the plain model (FRT_ERR_INVALID /
 * FRT_ERR_STATE). */
#define FRT_SUBGRID_NT 5000
#define FRT_SUBGRID_NDLIN 500
typedef struct {
  const float* time_RH;            /* FRT_SUBGRID_NT * 27 + 1 */
  const float* fh1_RH;             /* FRT_SUBGRID_NT * 27 + 1 */
  const float* t_deltaNL;          /* FRT_SUBGRID_NDLIN cosmic times, s */
  const float* delta_over_sigma;   /* FRT_SUBGRID_NDLIN */
  const float* deltaNL;            /* FRT_SUBGRID_NDLIN x FRT_SUBGRID_NDLIN, one row per time */
  float tinit, t_z12, t_z8, t_z55; /* cosmic_time at zinit, z = 12, 8, 5.5 */
  float tre_dom[3];                /* cosmic_time at z = 12, 8, 6 (init_radhydro_data, subgrid.cc:176-178) */
  int ifront;                      /* I-front tracking (ifront = TRUE) */
} frt_subgrid_tables;
frt_status frt_set_subgrid(frt_ctx* ctx, const frt_subgrid_tables* tables);
/* get_nphot_min_max (ray_tracing.cc:129-154) */
frt_status frt_get_nphot_min_max(frt_ctx* ctx, double* nmin_out, double* nmax_out);
/* set_clump + set_clight (subgrid.cc:799-811, rt_funcs.cc:129-143) */
frt_status frt_set_clump(frt_ctx* ctx);
frt_status frt_set_clight(frt_ctx* ctx);
/* t += dt, then update_rays (rt_funcs.cc:159-208 -> advance_ray, ray_tracing.cc:1222-1512) */
frt_status frt_update_rays(frt_ctx* ctx);
/* find_avg_unu (ray_tracing.cc:623-1216): C2Ray iteration, Gamma deposition, cell update */
frt_status frt_find_avg_unu(frt_ctx* ctx);
/* count_rays (ray_tracing.cc:35-47) per box */
frt_status frt_count_rays(frt_ctx* ctx, long long* count_per_box);
/* set_lmerge/set_merge_domain/get_num_thresh/count_rays/calc_nphot_merge, then merge
 * (main.cc:153-165; ray_tracing.cc:157-227, 324-477). itheta_per_box: one random-angle index per
 * box, drawn by the caller (siRand(Ntheta), ray_tracing.cc:327). */
frt_status frt_merge(frt_ctx* ctx, const uint16_t* itheta_per_box);
/* split_rays (rt_funcs.cc:211-237 -> split_ray, ray_tracing.cc:482-619) */
frt_status frt_split_rays(frt_ctx* ctx);
/* update_thermal (gas_funcs.cc:362-457) */
frt_status frt_update_thermal(frt_ctx* ctx);
/* new_rays (rt_funcs.cc:240-261 -> init_rays, ray_tracing.cc:230-321). itheta_per_source: one
 * index per source of all boxes in order, drawn by the caller (ray_tracing.cc:233). */
frt_status frt_new_rays(frt_ctx* ctx, const uint16_t* itheta_per_source);

/* Random-angle draws of the reference, siRand(Ntheta) = rand() % 42875 (general_funcs.cc:170-173):
 * one glibc rand() stream per box, seeded as srand(seed), held by the context. The reference draws
 * once per step in merge() (ray_tracing.cc:327) and then once per source in init_rays
 * (ray_tracing.cc:233); frt_draw_step fills both arrays in that order, frt_draw_cast only the
 * per-source ones (the set-up cast, main.cc:99). */
frt_status frt_seed_boxes(frt_ctx* ctx, const unsigned int* seeds);
frt_status frt_draw_cast(frt_ctx* ctx, uint16_t* itheta_per_source);
frt_status frt_draw_step(frt_ctx* ctx, uint16_t* itheta_per_box, uint16_t* itheta_per_source);

/* One whole RT step in the order of main.cc:108-264 (fixed redshift), captured once as a CUDA
 * graph and replayed: the fused form of the calls above. Host inputs are the random-angle
 * indices (both NULL: drawn from the context's streams, frt_draw_step); stats (may be NULL)
 * receives the per-step totals of all boxes. */
frt_status frt_step(frt_ctx* ctx, const uint16_t* itheta_per_box, const uint16_t* itheta_per_source,
                    frt_step_stats* stats);
/* The unbatched cast for comparisons: with per_source != 0, frt_step_plain casts the new rays
 * with one kernel launch per source (the way a per-source loop would), not one for all sources.
 * Results are the same; frt_step (the graph) is not affected. */
frt_status frt_set_cast_per_source(frt_ctx* ctx, int per_source);

/* ---- one box over several contexts (one per GPU): the step in phases ------------------------
 * Replaces the reference's whole-box OpenMP loops over rays (update_rays, the ray part of
 * find_avg_unu, split_rays, new_rays; main.cc:127-246) by a share of the sources per context:
 * every context holds the whole box, frt_set_source_owner marks the sources it casts (own[s] = 1;
 * NULL = all), and the caller runs the step as frt_step_phase(WALK), combine A, (CELLS), then per
 * C2Ray iteration it: (RAYPASS, it), combine B, (CELLPASS, it), then (END). A new source list
 * (frt_set_sources) clears the mask: set it again after the sources. Combine A ORs the
 * lit-flag bytes (frt_phase_buffers: ncell of them) over the contexts; combine B sums the float2
 * lit-cell pairs lit_acc[nlit] and, after the last iteration's ray pass, lit_heat[nlit]. Every
 * context then runs the same cell passes, and END returns this context's totals (rays, crossings,
 * photons: sum them over the contexts). Each phase has finished on the device when it returns.
 * Needs core outputs, mixed precision and a box whose ray count cannot reach the merge threshold
 * (FRT_ERR_INVALID otherwise). The draws are the box's own reference-order draws when the
 * itheta pointers are NULL, so contexts seeded alike cast with the same angles. */
#define FRT_PHASE_WALK 0
#define FRT_PHASE_CELLS 1
#define FRT_PHASE_RAYPASS 2
#define FRT_PHASE_CELLPASS 3
#define FRT_PHASE_END 4
frt_status frt_set_source_owner(frt_ctx* ctx, const uint8_t* own);
frt_status frt_step_phase(frt_ctx* ctx, int phase, int iter, const uint16_t* itheta_per_box,
                          const uint16_t* itheta_per_source, frt_step_stats* stats);
/* Device addresses of the arrays the caller combines between phases: lit_flag (ncell bytes, one
 * per cell of all boxes), lit_acc and lit_heat (nlit float2 each; nlit is set by the CELLS phase
 * of the current step). */
frt_status frt_phase_buffers(frt_ctx* ctx, void** lit_flag, long long* ncell, void** lit_acc, void** lit_heat,
                             long long* nlit);
/* Phases that only enqueue (async != 0): each phase returns once its kernels are queued on the
 * context's stream (frt_phase_stream returns it as a cudaStream_t), except CELLS, which waits for
 * the lit-cell count (the length of the combined arrays), and END, which waits for the step's
 * totals. The caller then orders its combines on that stream (e.g. NCCL collectives enqueued on
 * it). Default (async = 0): every phase has finished on the device when it returns. */
frt_status frt_set_phase_async(frt_ctx* ctx, int async);
frt_status frt_phase_stream(frt_ctx* ctx, void** stream);
/* Same as frt_step but launching every kernel directly (no graph) */
frt_status frt_step_plain(frt_ctx* ctx, const uint16_t* itheta_per_box, const uint16_t* itheta_per_source,
                          frt_step_stats* stats);
frt_status frt_last_stats(frt_ctx* ctx, frt_step_stats* stats);

/* ---- launch shapes and the autotuner ----------------------------------------------------------
 * The reference divides its ray loops statically over OpenMP threads (size_cpu,
 * global_variables.cc:44) and rebalances the per-thread ray buffers between steps (balance_cpus,
 * free_cpu; mem_funcs.cc:186-299). Here the matching choices are the launch shapes of the ray and
 * cell kernels: block size and blocks per SM of the ray pass, the walk, the cell pass and the
 * compaction + split, and how the ray pass hands out its moved rays (static per-warp slices, or
 * chunks of a device-side queue). Shapes change only the work distribution, not the arithmetic of
 * a ray or a cell. */
typedef struct {
  int raypass_block, raypass_blocks_per_sm; /* ray pass of a C2Ray iteration (mixed precision);
                                               blocks_per_sm 0: the blocks resident at once */
  int raypass_chunk;                        /* 0: static per-warp slices; > 0: rays per queue chunk */
  int walk_block, walk_blocks_per_sm;       /* cell-boundary walk (update_rays) */
  int cellpass_blocks_per_sm;               /* lit-cell pass of a C2Ray iteration (0: resident) */
  int split_blocks_per_sm;                  /* compaction + split (split_rays) */
  int steps;                                /* frt_autotune: RT steps it took */
  /* frt_autotune: measured cost of the chosen shapes, ns per unit of work (crossing, ray, lit cell) */
  double raypass_ns_per_crossing, walk_ns_per_ray, cellpass_ns_per_cell, split_ns_per_ray;
} frt_tuning;
/* Runs `steps` (>= 1; 4 recommended) whole RT steps of the context (they advance the simulation
 * like frt_step_plain; the draws come from the context's streams) and times candidate shapes on
 * them: every candidate of a round runs on a comparable share of one step's work (one C2Ray
 * iteration's ray or cell pass, or one of k equal ray ranges of the walk and the compaction),
 * costs are time per unit of work, and each round varies one parameter around the best so far.
 * With steps >= 3 the last two steps validate the result on whole graph steps (where the dark
 * pass shares the SMs): one runs the search's shapes, one the starting shapes, and the faster
 * per crossing is kept.
 * The chosen shapes are set on the context, reported in *out, and remembered for contexts of the
 * same device, cell count and live-ray count (power-of-two bucket): frt_step switches to a
 * remembered shape set when its ray count enters that bucket. */
frt_status frt_autotune(frt_ctx* ctx, int steps, frt_tuning* out);
frt_status frt_get_tuning(frt_ctx* ctx, frt_tuning* out);
/* Sets the shapes (blocks 32..256, multiples of 32; blocks per SM 1..32; chunk 0..65536);
 * FRT_ERR_INVALID otherwise. Turns off the remembered-shape switching of frt_step. */
frt_status frt_set_tuning(frt_ctx* ctx, const frt_tuning* in);

/* ---- rays ----------------------------------------------------------------------------------- */
frt_status frt_num_rays(frt_ctx* ctx, int box, long long* n);
/* Live rays of a box in pool order, unpacked like write_rays_binary (io_funcs.cc:274-303):
 * order, pixel, itheta, cell (= path[0].ind, local to the box), geom[9] = xhat, yhat, zhat, r, dr,
 * x, y, z, time; nphot[nfreq]. Arrays must hold frt_num_rays() entries. */
frt_status frt_download_rays(frt_ctx* ctx, int box, int16_t* order, int32_t* pixel, uint16_t* itheta,
                             int32_t* cell, float* geom9, float* nphot);

/* Opt-in optical-depth limit; no counterpart in the reference, whose rays end only below
 * nphot_min (ray_tracing.cc:782, 927-933). With tau_max > 0 every ray carries the HI and HeI
 * column densities it crossed since its cast, summed in FP64 over the segments of each step's
 * last C2Ray iteration (split children inherit them, a merged ray keeps its base ray's, rays read
 * by frt_read_rays start at 0), and after the step's last ray pass a ray whose optical depth
 * sigma_HI(nu) N_HI + sigma_HeI(nu) N_HeI exceeds tau_max in every frequency bin is removed like
 * a ray below nphot_min (its photons counted as killed). 0 turns the limit off (the default);
 * refused with the sub-grid model. Takes effect from the next step. */
frt_status frt_set_tau_limit(frt_ctx* ctx, double tau_max);
/* The HI and HeI column densities (cm^-2, 2 doubles per ray) of a box's live rays in the order of
 * frt_download_rays; zeros while the optical-depth limit was never set. */
frt_status frt_download_ray_columns(frt_ctx* ctx, int box, double* col2);

/* Scalars of one box: t, dt, nphot_min, nphot_max, nphot_merge, num_thresh, dx, dx0 */
frt_status frt_box_scalars(frt_ctx* ctx, int box, double* out8);
/* Kernel time of the last frt_step / frt_step_plain in ms (device events on the step stream),
 * and the time of its dominant cell kernel. */
frt_status frt_last_timing(frt_ctx* ctx, float* step_ms, float* cell_kernel_ms);
/* Device time in ms of one kernel family in the last frt_step / frt_step_plain (CUDA events on its
 * stream): which = 0 the dark-cell kernel, 1 the ray passes of the C2Ray iteration (summed),
 * 2 the walk (update_rays' advance of every ray). */
frt_status frt_last_kernel_timing(frt_ctx* ctx, int which, float* ms);

/* ---- restart files (the reference's own formats) ------------------------------------------------
 * Writers: the records of write_gas_binary (io_funcs.cc:358-393: float t, then per cell rho, temp,
 * nH1, f_H1, f_He1, f_H2, f_He2, f_He3, gamma_H1_tot, gamma_He1_tot, mfp, mfp_912, heat_rate,
 * cool_rate, avg_nh1, fion, tcross, treion_out, ngam_nu[nfreq]), write_rays_binary (274-303:
 * packed {int64 slot, bool active, int16 order, int32 pixel, uint16 itheta, float xhat, yhat,
 * zhat, nphot[nfreq], r, dr, x, y, z, time, int32 cell} ended by slot -1) and write_treion
 * (338-355: per cell float treion, bool treion_flag, tcross_flag, neutral_flag). With buf NULL
 * only *len (the byte count) is returned. With core outputs mfp comes from the final <n_HI> and
 * ngam_nu is 0 (both are output fields; diag outputs write the reference's values).
 * Readers (a restart, input_grid = TRUE): frt_read_gas replaces frt_init_gas (init_funcs.cc:10-19,
 * 62-138), frt_read_treion sets treion and its flag, and after frt_init_rt (which then keeps the
 * file's time and sets ray_dt = 0 at the sources, rt_funcs.cc:95-101) frt_read_rays appends the
 * file's rays (read_rays_binary, io_funcs.cc:119-146, with init_rt's removal of an empty ray in
 * slot 0, rt_funcs.cc:117-124). No set-up cast follows a restart. */
frt_status frt_write_gas(frt_ctx* ctx, int box, void* buf, size_t cap, size_t* len);
frt_status frt_write_rays(frt_ctx* ctx, int box, void* buf, size_t cap, size_t* len);
frt_status frt_write_treion(frt_ctx* ctx, int box, void* buf, size_t cap, size_t* len);
frt_status frt_read_gas(frt_ctx* ctx, int box, const void* buf, size_t len);
frt_status frt_read_treion(frt_ctx* ctx, int box, const void* buf, size_t len);
frt_status frt_read_rays(frt_ctx* ctx, int box, const void* buf, size_t len);

/* Rays moved between the contexts that share one box (the source-shared form over several GPUs,
 * no counterpart in the reference). frt_take_rays writes the live rays of a one-box context in
 * the ray-record format of frt_write_rays and leaves the context without rays: with in_step = 1
 * between the step's last C2Ray pass (FRT_PHASE_CELLPASS of the last iteration) and
 * FRT_PHASE_END, skipping the rays that pass removed; with in_step = 0 between steps. buf = NULL
 * returns the size in *len. frt_put_rays appends such records to a context's rays at the same
 * points (no free-slot probe, no change to the photon ledger). Used to merge the rays of all
 * contexts on one of them when the box's ray count reaches the merge threshold, and to deal them
 * out again after the step. */
frt_status frt_take_rays(frt_ctx* ctx, int box, int in_step, void* buf, size_t cap, size_t* len);
frt_status frt_put_rays(frt_ctx* ctx, int box, const void* buf, size_t len);
/* Sets a box's merge threshold nphot_merge (calc_nphot_merge, ray_tracing.cc:176-227; it persists
 * between the steps that merge and sets the split threshold max(4 nphot_merge, 4 nphot_min)):
 * after the contexts of a shared box merged their rays on one of them, the others take that
 * context's value (frt_box_scalars, index 4) so that every context splits alike. */
frt_status frt_set_nphot_merge(frt_ctx* ctx, int box, double nphot_merge);

/* ---- adjoint of the next step's Gamma field --------------------------------------------------
 * Objective: J = sum of Gamma_HI (gamma_H1_tot, ray_tracing.cc:1152) over the cells
 * [lo, hi) (i, j, k) of one box after the C2Ray iteration of the next step. frt_adjoint returns J
 * and its gradient with respect to every source luminosity of that box (photons/s, in
 * frt_set_sources order) and every cell's hydrogen density n_H (cm^-3; the cell's n_He, n_HI and
 * n_HeI scale with it as one density; ionised fractions, temperature, clumping and nphot_min are
 * held fixed). The segments of the step's rays are recomputed from the ray state, nothing is
 * stored between passes, and the context's state is not modified. Any state of the run will do
 * (after set-up or after any number of steps): a ray's photons are proportional to the luminosity
 * of the source that cast it, found from the ray itself (an unmerged ray lies on the straight
 * line from its source's cell centre along its direction). A merge combines rays of different
 * sources, and rays read from a restart file have no known source: after either, FRT_ERR_STATE.
 * dL (nsrc of the box) and dnH (N^3) may be NULL. No counterpart in the reference. */
typedef struct {
  int box;
  int lo[3], hi[3];
} frt_adj_objective;
frt_status frt_adjoint(frt_ctx* ctx, const frt_adj_objective* obj, double* J, double* dL, float* dnH);
/* Device time of the last frt_adjoint's kernels in ms (CUDA events on the context's stream). */
frt_status frt_last_adjoint_timing(frt_ctx* ctx, float* ms);

/* ---- field read-back without device allocation ---------------------------------------------
 * No counterpart in the reference (its fields live in host arrays). Gathers cells
 * [first_cell, first_cell + count) of one lit-cell field -- GAMMA_H1_TOT, GAMMA_HE1_TOT, or bin
 * `bin` of GAMMA_H1_NU, GAMMA_HE1_NU, NGAM_NU -- into `host`, the same values frt_get_field
 * returns, without allocating device memory: the gather goes through a fixed 4 MiB scratch array
 * in the library's static device memory, so count is limited to FRT_NOALLOC_MAX_CELLS (larger
 * requests return FRT_ERR_INVALID; read a box in windows). The first call on a device looks up
 * the scratch address (cudaGetSymbolAddress, with the context's device made current); make that
 * first call before any stream capture. The scratch array is shared by every context on the
 * device: calls that overlap in time (two host threads, two contexts) race on it and must be
 * serialised by the caller. Blocks until the values are in `host`. */
#define FRT_NOALLOC_MAX_CELLS (1 << 20)
frt_status frt_get_sparse_field_noalloc(frt_ctx* ctx, int box, frt_field f, int bin, long long first_cell,
                                        long long count, float* host);

#ifdef __cplusplus
}
#endif
#endif /* FLEXRT_H */
