// Host-side set-up arithmetic (frt_hostmath.cc, compiled by g++ with -ffp-contract=off).
#pragma once
#include "../../include/flexrt.h"
#include "frt_params.h"

namespace frt {
namespace host {

struct GasInit {  // caller-owned arrays of n^3 floats
  float *rho, *nH, *nHe, *nH1, *nHe1, *f_H1, *f_He1, *temp, *ne, *n_tot, *rec_h2, *rec_he2, *dne_dt;
};

void rotation_table(float* out);  // kNtheta x 18 floats (forward, inverse)
void box_params(BoxP* B, const frt_config* cfg, const frt_box_desc* bd, long long cell0);
// The cell-size dependent members of a box (dx, the cell-edge thresholds, dt of update_dt, the
// deposit normalisation): set up by box_params, and again after a cosmological expansion.
void set_cell_size(BoxP* B, const frt_config* cfg, const frt_box_desc* bd, float dx);
void init_gas(const frt_config* cfg, const frt_box_desc* bd, const float* delta1, GasInit* g);
// The state init() derives on a restart (input_grid = TRUE) from a gas file's per-cell records of
// 18 + nfreq floats (write_gas_binary order); heat and cool rates are taken from the records.
struct GasRestart {
  const float* rec;   // n^3 records
  int stride;         // 18 + nfreq
};
void init_gas_restart(const frt_config* cfg, const frt_box_desc* bd, const GasRestart& r, GasInit* g, float* heat,
                      float* cool);
void nphot_min_max(const frt_config* cfg, const BoxP* B, int nsrc, const double* lum, double* nmin, double* nmax);
// calc_vol_avg (data_funcs.cc:75-92): double sum in cell order, float result
float vol_avg(const float* f, int n);
// A snapshot's proper density as get_ugas reads it (io_funcs.cc:33-62) scaled by a^-3, and its
// volume average (taken before the scaling and scaled the same way, gas_funcs.cc:606-613, 669-684)
void snapshot_rho(int n, const float* delta1, float a, float* rho, float* avg_rho);
// The proper cell size Lx0 a / N kpc_to_cm of a box at scale factor a (init_funcs.cc:23, gas_funcs.cc:689)
float snapshot_dx(const frt_box_desc* bd, float a);
// The redshift-dependent constants of the thermal update (Hubble rate, Compton rate)
void set_redshift(BoxP* B, float zz);
void derived_constants(const frt_config* cfg, double* sigH1, double* sigHe1, double* sig0, double* sig912,
                       double* pi_sf_3, double* log4);

}  // namespace host
}  // namespace frt
