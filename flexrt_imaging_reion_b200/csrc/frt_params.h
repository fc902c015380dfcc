// Plain-C++ parameter blocks shared by the host set-up code (g++) and the kernels (nvcc).
#pragma once
#include <stdint.h>

namespace frt {

constexpr int kTileShift = 10;  // 1024 cells per tile
constexpr int kTile = 1 << kTileShift;
constexpr int kNtheta = 42875;
constexpr int kLtab = 16;       // orders 0..15 in the radius tables
constexpr int kLmax = 12;       // l_max (global_variables.cc:55)
constexpr int kPdfBins = 10000; // calc_nphot_merge (ray_tracing.cc:176-227)

// Per-box constants of the thermal update.
struct ThermConst {
  float dt;
  float dx;
  float hub2f;      // 2 H(a) as float (H is a float function, cosmo_funcs.cc:13-15)
  double hub_d;     // H(a) as double for the strict form
  float zz;
  double compton_d; // compton_rate(zz) (rates.cc:234-238)
  float compton_f;
  float nfreq;
  float cH1[8];     // h (h_eV nu - Eth_H1) / h_eV per bin
  float cHe1[8];
  double nu[8];
};

struct BoxP {
  int n, nn;                 // cells per side, n*n
  double inv_n, inv_nn;      // 1/n, 1/(n*n) (cell_ijk)
  long long cell0, ncell;    // first global cell, n^3
  float dx, dx0, scale;      // proper cell, comoving cell, dx/dx0 (float, ray_tracing.cc:1262)
  float dx_half;             // dx/2. (ray_tracing.cc:308)
  float lo_edge;             // min_dist*dx (float)
  float hi_edge;             // dx*(1.-min_dist) rounded to float
  double hi_thr;             // dx*(1.-min_dist/2.) (compared in double)
  float hi_thr_f;            // the smallest float >= hi_thr: (double)x >= hi_thr <=> x >= hi_thr_f
  float mv_hi;               // nc*dx (float)
  double mv_lo;              // (1.-nc)*dx (double)
  float mv_lo_f;             // the smallest float >= mv_lo: (double)x < mv_lo <=> x < mv_lo_f
  float clight, nc;          // cl_factor*cl (float), nl_const
  float dt, t;
  double vol;                // dx*dy*dz in double
  double kdep;               // phot_norm / dt / vol
  float kdep_f;              // the same in float (mixed-precision deposits)
  double rkill;              // comoving cm; 0 = off
  double nphot_min, nphot_max;
  float nmin_ru, nmin_rd;    // nphot_min rounded up / down to float (set at the start of each step)
  float nphot_merge, split_thr;
  long long num_thresh;
  int lm;                    // merging HEALPix order (hpx_lvl)
  int lsource;               // casting order for cells below 10% neutral
  ThermConst th;
  float rmax[kLtab], rmin[kLtab];
  float avg_rho;             // volume-averaged proper density (calc_vol_avg, data_funcs.cc:75-92)
  float sg_dnl_dom[3];       // sub-grid model: the non-linear overdensities of the RadHydro domain this step
};

}  // namespace frt
