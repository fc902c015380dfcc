// ORACLE TEST INFRASTRUCTURE -- not part of the product. Only the tests, smoke() and the
// CPU-baseline leg of bench.py load this library, and only as the checker.
//
// Single-threaded CPU restatement of the reference's per-timestep RT path (plain C2Ray mode:
// subgrid = FALSE, ifront = FALSE, c2ray_iter = TRUE, multi_freq = TRUE, case-B recombination),
// configured at run time instead of through user_inputs.h. Every routine follows the reference
// expression by expression -- including which sub-expressions are float and which double,
// and which float overloads of the <cmath> functions get picked -- so that with the reference
// compiled for one thread (oracle/build_ref.py) the two agree bit for bit. The ray buffer is a
// list kept in creation order, which is the reference's slot order for one thread while the
// allocation ring has not wrapped (mem_funcs.cc:79-97).
//
// Reference map: rates rates.cc:41-238; spectrum gas_funcs.cc:11-70; init init_funcs.cc:10-142;
// cast ray_tracing.cc:230-321 + rt_funcs.cc:240-261; advance ray_tracing.cc:1222-1512 +
// rt_funcs.cc:159-208; C2Ray iteration ray_tracing.cc:623-1216; merge machinery
// ray_tracing.cc:35-227, 324-477; split ray_tracing.cc:482-619 + rt_funcs.cc:211-237; thermal
// gas_funcs.cc:104-242, 353-457; rotations healpix_funcs.cc:21-39, 102-143; dt rt_funcs.cc:9-12.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>
#include <unordered_map>
#include <vector>

#include "frtd.h"
#include "../flexrt_imaging_reion_b200/csrc/hp_nest.h"

using namespace std;

namespace orc {

// ---- constants (global_constants.h, global_variables.cc) --------------------------------
#define O_PI 3.14159
#define O_H 6.626068e-27
#define O_H_EV 4.135667e-15
#define O_KB 1.38065e-16
#define O_KPC_TO_CM 3.086e21
#define O_CL 2.998e10
#define O_MH 1.672622e-24
#define O_Y 0.246
#define O_HH 0.68
#define O_OMEGA_M 0.305147
#define O_OMEGA_L 0.6948
#define O_MPC_TO_KM 3.086e19
#define O_EV_CGS 1.60218e-12
static const double kPhotNorm = 1e60;
static const float kNheToNh = (O_Y / 4.) / (1. - O_Y);
static const float kTempMin = 1e2;
static const float kMinDist = 1e-4;
static const int kNalpha = 35;
static const int kNtheta = 42875;
static const int kMaxF = 8;
static const int kMaxPL = 16;

static inline float mind(float a, float b) { return (a >= b) ? b : a; }
static inline float maxd(float a, float b) { return (b >= a) ? b : a; }
static inline double mindd(double a, double b) { return (a >= b) ? b : a; }
static inline float absd(float x) { return (x >= 0.) ? x : -1. * x; }
static inline int mins(short a, short b) { return (a >= b) ? b : a; }
static inline int maxs(short a, short b) { return (b >= a) ? b : a; }
static inline int imin(int a, int b) { return (a >= b) ? b : a; }
static inline int imax(int a, int b) { return (a >= b) ? a : b; }
static inline int imod(int a, int b) {
  while (a < 0) a += b;
  return a % b;
}

// ---- atomic data: Verner et al. 1996 cross sections, Hui & Gnedin 1997 rates -------------
static double lambda_x(double T, double Eth) {
  double K2eV = O_KB / O_EV_CGS;
  double eV2K = 1.0 / K2eV;
  return 2 * Eth * eV2K / T;
}
static double verner(double nu, double Eth, double Emax, double E0, double y0, double y1, double yw, double ya,
                     double P) {
  double E = O_H_EV * nu;
  double x = E / E0 - y0;
  double y = pow(pow(x, 2) + pow(y1, 2), 0.5);
  double F = (pow(x - 1, 2) + pow(yw, 2)) * pow(y, 0.5 * P - 5.5) * pow(1 + pow(y / ya, 0.5), -P);
  if (O_H_EV * nu >= Eth && O_H_EV * nu <= Emax) return F;
  return 0;
}
static double sig_H1(double nu) { return 5.475e-14 * verner(nu, 13.6, 5e4, 4.298e-1, 0, 0, 0, 3.288e+1, 2.963); }
static double sig_He1(double nu) {
  return 9.492e-16 * verner(nu, 2.459e+1, 5e4, 1.361e+1, 4.434e-1, 2.136, 2.039, 1.469, 3.188);
}
static double alphaB_H2(double T) {
  double x = lambda_x(T, 13.6);
  return 2.753e-14 * pow(x, 1.500) / pow((1.0 + pow((x / 2.740), 0.407)), 2.2420);
}
static double alphaB_He2(double T) {
  double x = lambda_x(T, 2.459e+1);
  return 1.26e-14 * pow(x, 0.750);
}
static double alphaB_He3(double T) {
  double x = lambda_x(T, 5.442e+1);
  return 2 * 2.753e-14 * pow(x, 1.500) / pow((1.0 + pow((x / 2.740), 0.407)), 2.2420);
}
static double Dalpha_He2(double T) {
  double x = lambda_x(T, 5.442e+1);
  return 1.90e-3 * pow(T, -1.5) * exp(-0.75 * x / 2) * (1 + 0.3 * exp(-0.15 * x / 2));
}
static double rcrB_H2(double T) {
  double x = lambda_x(T, 13.6);
  return 3.435e-30 * T * pow(x, 1.970) / (pow(1. + pow(x / 2.250, 0.376), 3.720));
}
static double rcrB_He2(double T) { return O_KB * T * alphaB_He2(T); }
static double free_free_rate(double T) { return 1.42e-27 * pow(T, 0.5) * 1.30; }
static double compton_rate(double z) { return 5.6072e-36 * pow(1 + z, 4.); }
static float hubble(float a) { return O_HH * 100. / O_MPC_TO_KM * pow(O_OMEGA_M / pow(a, 3.) + O_OMEGA_L, 0.5); }

// sub-grid model rates (rates.cc:128-145, 240-254) and constants (global_variables.cc:241-304)
static double alphaA_H2(double T) {
  double x = lambda_x(T, 13.6);
  return 1.269e-13 * pow(x, 1.503) / pow((1.0 + pow((x / 0.522), 0.470)), 1.923);
}
static double alphaA_He2(double T) {
  double x = lambda_x(T, 2.459e+1);
  return 3.0e-14 * pow(x, 0.654);
}
static double phothtHI(double alpha, double T, double ne) {
  return 1.360e+1 / O_H_EV * O_H *
         ((alpha + 2.8) / (1.8 + alpha) * (1. - pow(4., -1.8 - alpha)) / (1. - pow(4., -2.8 - alpha)) - 1.) *
         alphaA_H2(T) * ne;
}
static double phothtHeI(double alpha, double T, double ne) {
  return 2.459e+1 / O_H_EV * O_H *
         ((alpha + 1.7) / (0.7 + alpha) * (1. - pow(2.2, -0.7 - alpha)) / (1. - pow(2.2, -1.7 - alpha)) - 1.) *
         alphaA_He2(T) * ne;
}
static double photoheat_HIHeI(double alpha, double T, double ne, double nH, double nHe) {
  return phothtHI(alpha, T, ne) * nH + phothtHeI(alpha, T, ne) * nHe;
}
static const float kSigmaEffRH = 2.517139346618065e-18;
static const float kGammaMin = 1e-16;
static const float kMaxSubgridFrac = 0.49;
static const int kNt = 5000;
static const int kNdlin = 500;
// the parameter domain of the RadHydro runs (init_radhydro_data, subgrid.cc:114-128)
static const float kGammaDom[5] = {3e-15f, 3e-14f, 3e-13f, 3e-12f, 3e-11f};

// ---- state -----------------------------------------------------------------------------
struct Ray {
  bool alive, active;
  short order;
  int pixel;
  unsigned short itheta;
  float xhat, yhat, zhat;
  float nphot[kMaxF];
  float r, dr, x, y, z, time;
  int pind[kMaxPL];
  float pdist[kMaxPL];
  short ray_end;
  int src;   // casting source (index into Ctx::src); a merge of rays of several sources gives -1
  // opt-in optical-depth limit (not in the reference): the HI and HeI column densities the ray
  // crossed since its cast (cm^-2 proper, FP64; split children inherit them, a merged ray keeps
  // its base ray's)
  double colH, colHe;
};

struct Src {
  int i, j, k;
  double lum;
};

struct Ctx {
  // configuration
  int N, F, PL, itercount, ray_per_cell_max, hpx_lvl, l_max;
  double nu[kMaxF];
  float cl_factor, tstep_factor, nl_const, safety_factor, const_clump, zz, fH1_0, fHe1_0, fHe2_0, temp_0, Lx0;
  double rkill;
  // scalars
  float dx0, Lx, dxc, dt, t, clight, nc;
  float spectrum[kMaxF];
  double nphot_min, nphot_max, nphot_base_avg;
  double tau_max;   // opt-in: remove a ray once its optical depth exceeds this in every bin (0: off)
  float nphot_merge;
  long num_thresh, total_rays;
  float random_angles[kNtheta][3];
  double sigH1[kMaxF], sigHe1[kMaxF];
  // fields
  std::vector<float> rho, nH, nHe, nH1, nHe1, nH2, nHe2, nHe3, ne, n_tot, f_H1, f_He1, f_H2, f_He2, f_He3, temp,
      clump, clump_in, avg_nh1, avg_nhe1, avg_gamma, avg_gamma_he1, recomb_H2, recomb_He2, recomb_He3, recrate_H2,
      recrate_He2, dne_dt, mfp, mfp_912, treion, treion_out, heat_rate, cool_rate, gamma_H1_tot, gamma_He1_tot,
      nH1_prev, IF_speed, Inc_Flux, ray_dt;
  std::vector<float> gamma_H1_nu, gamma_He1_nu, ngam_nu, u_nu, avg_gamma_nu, avg_gamma_nu_he1;
  std::vector<unsigned char> treion_flag;
  bool have_clump;
  std::vector<Src> src;
  std::vector<Ray> rays;
  long last_crossings, last_moved;
  int step;
  unsigned seed;
  // photon ledger of the last step (physical photons, double): the cast, the photons absorbed on
  // the last C2Ray iteration (dumps included), the photons left in removed rays, and the photons
  // that a dumping ray both deposited and kept until its removal. Bookkeeping only: no field or
  // ray of the restatement depends on it.
  double led_emitted, led_deposited, led_killed, led_overlap;
  // hydro snapshots (update_hydro_step, gas_funcs.cc:554-752): the volume-averaged density, the
  // previous snapshot's density and d(delta)/dt of the temperature equation (gas_funcs.cc:399)
  float avg_rho;
  std::vector<float> rho_prev, ddelta_dt;
  float step_dt;   // the time step the last step ran with (get_nphot_min_max at a switch uses it)
  // sub-grid model (subgrid = TRUE, equilibrium = TRUE, ifront = FALSE): the RadHydro time and
  // HI-fraction tables in the reference's memory layout (see orc_set_subgrid), the linear ->
  // non-linear overdensity table, the cosmic times the model uses, the overdensity domain of the
  // current step and the per-cell HI-fraction interpolants of the current step
  bool subgrid = false;
  std::vector<float> sg_time, sg_fh1, sg_t_dnl, sg_ds, sg_dnl;
  float sg_tinit, sg_t12, sg_t8, sg_tcap, sg_tre_dom[3];
  float sg_dnl_dom[3];
  std::vector<float> sg_fh1_interp;
  // I-front tracking (ifront = TRUE, subgrid.cc:660-751, ray_tracing.cc:863-919, 1003-1053): the
  // fraction of each cell the fronts have passed and its maximum, the crossing time in total and
  // per tenth of the cell (with the tenths already passed), the flags, and the photon counts of
  // one C2Ray iteration per cell: [0] absorbed by the neutral part, [1] the same weighted by
  // sigma_eff_rh times path length, [2] entering the neutral part
  bool ifront = false;
  std::vector<float> fion, fion_max, tcross, tcross_new, Delta_fion;
  std::vector<unsigned char> tcross_check, tcross_flag, neutral_flag;
  std::vector<double> ngam3;
};

static const int kNtcross = 10;   // global_variables.cc:224

// the ionised fraction the sub-grid branch uses for a cell: 1 without I-front tracking
// (rt_funcs.cc:55)
static inline float fion_of(const Ctx& c, long q) { return c.ifront ? c.fion[q] : 1.f; }

static inline long cidx(const Ctx& c, int i, int j, int k) { return ((long)i * c.N + j) * c.N + k; }
static inline void split_ind(const Ctx& c, int ind, int* i, int* j, int* k) {
  const int nyz = c.N * c.N;
  *i = (ind - imod(ind, nyz)) / nyz;
  int jj = ind - *i * nyz;
  *j = (jj - imod(jj, c.N)) / c.N;
  *k = ind - *i * nyz - *j * c.N;
}

static float sum_nphot(const Ctx& c, const Ray& R) {
  float s = 0.;
  for (int nu = 0; nu < c.F; nu++) s += R.nphot[nu];
  return s;
}

// ---- sub-grid model (subgrid.cc), equilibrium = TRUE, ifront = FALSE ----------------------
// interpolate (general_funcs.cc:275-315): linear interpolation with linear extrapolation
static float sg_interpolate(const float* x, const float* y, float x0, int n) {
  float y0 = 0.;
  bool itp = false;
  for (int i = 0; i < n - 1; i++) {
    if (((x[i] <= x0) && (x[i + 1] >= x0)) || ((x[i] >= x0) && (x[i + 1] <= x0))) {
      y0 = y[i] + (y[i + 1] - y[i]) / (x[i + 1] - x[i]) * (x0 - x[i]);
      itp = true;
      break;
    }
  }
  if (!itp) {
    if (x[0] < x[n - 1]) {
      if (x0 > x[n - 1]) {
        float slope = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
        y0 = y[n - 1] + slope * (x0 - x[n - 1]);
      } else {
        float slope = (y[1] - y[0]) / (x[1] - x[0]);
        y0 = y[0] + slope * (x0 - x[0]);
      }
    } else {
      if (x0 < x[n - 1]) {
        float slope = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
        y0 = y[n - 1] + slope * (x0 - x[n - 1]);
      } else {
        float slope = (y[1] - y[0]) / (x[1] - x[0]);
        y0 = y[0] + slope * (x0 - x[0]);
      }
    }
  }
  return y0;
}

// delta_dom_to_deltaNL_dom (subgrid.cc:97-132): the non-linear overdensities of the RadHydro
// domain's linear ones (-sqrt(3), 0, sqrt(3)) at cosmic time `time`, the upper one capped at its
// value at z = 5.5
static void sg_delta_dom(Ctx& c, float time) {
  const float delta_dom[3] = {(float)-pow(3., 0.5), 0.f, (float)pow(3., 0.5)};
  c.sg_dnl_dom[1] = 0.;
  const float tcap = c.sg_tcap;
  int ti_m = 0, ti_p = 1, tcap_m = 0, tcap_p = 1;
  const float* t = c.sg_t_dnl.data();
  for (int i = 0; i < kNdlin - 1; i++) {
    if ((t[i] <= time) && (t[i + 1] >= time)) {
      ti_m = i;
      ti_p = i + 1;
    }
    if ((t[i] <= tcap) && (t[i + 1] >= tcap)) {
      tcap_m = i;
      tcap_p = i + 1;
    }
  }
  const float* ds = c.sg_ds.data();
  auto row = [&](int i) { return c.sg_dnl.data() + (size_t)i * kNdlin; };
  float d0m = sg_interpolate(ds, row(ti_m), delta_dom[0], kNdlin);
  float d0p = sg_interpolate(ds, row(ti_p), delta_dom[0], kNdlin);
  float d2m = sg_interpolate(ds, row(ti_m), delta_dom[2], kNdlin);
  float d2p = sg_interpolate(ds, row(ti_p), delta_dom[2], kNdlin);
  float capm = sg_interpolate(ds, row(tcap_m), delta_dom[2], kNdlin);
  float capp = sg_interpolate(ds, row(tcap_p), delta_dom[2], kNdlin);
  float cap = capm + (capp - capm) / (t[tcap_p] - t[tcap_m]) * (tcap - t[tcap_m]);
  c.sg_dnl_dom[0] = d0m + (d0p - d0m) / (t[ti_p] - t[ti_m]) * (time - t[ti_m]);
  c.sg_dnl_dom[2] = d2m + (d2p - d2m) / (t[ti_p] - t[ti_m]) * (time - t[ti_m]);
  c.sg_dnl_dom[2] = mind(c.sg_dnl_dom[2], cap);
}

// deltaNL_to_deltasig (subgrid.cc:196-205): Mo & White (1996) linear overdensity over sigma
static float sg_deltasig(float deltaNL, float redshift) {
  float dcmode = 5.10655;
  float sigma0 = dcmode / pow(3., 0.5);
  float d_of_z = 1. / (1 + redshift) / 0.78205;
  float delta = -1.35 * pow(1. + deltaNL, -2. / 3.) + 0.78785 * pow(1. + deltaNL, -0.58661) -
                1.12431 * pow(1. + deltaNL, -0.5) + 1.68647;
  return delta / d_of_z / sigma0;
}

// The reference's RadHydro arrays are [Nt][Nzre][Ndelta][Ngamma] with Ngamma = 3, filled and read
// at the gamma index q + 1 (gam_offset, subgrid.cc:24-36; ind_gamma, subgrid.cc:329-331), so every
// access runs one slot past its row into the next: the flat offset below is the reference's own
// address arithmetic, and the arrays here carry one slot more for the last row's spill.
static inline size_t sg_at(int t, int m, int p, int iq) { return (((size_t)t * 3 + m) * 3 + p) * 3 + iq; }

// get_tradhydro_index (subgrid.cc:189-193)
static int sg_tindex(const Ctx& c, float tsince) {
  int i = (int)floor(tsince / c.sg_time[sg_at(kNt - 1, 0, 0, 0)] * (kNt - 1));
  return imax(0, imin(i, kNt - 2));
}

// get_interpolate_gamma_f (subgrid.cc:211-250) with fractype = TRUE, and the extension to the
// outer rates of get_gamma_interp (subgrid.cc:451-452): out[5] over kGammaDom from the time-
// interpolated HI fractions f[tre][delta][gamma]
static void sg_gamma_f(const Ctx& c, float tsince, float tre, float deltaNL, const int ind_tre[2],
                       const int ind_delta[2], float f[2][2][3], float out[5]) {
  const float* tre_dom = c.sg_tre_dom;
  for (int g = 0; g < 3; g++) {
    float f_d0 = log10(f[0][0][g]) + (log10(f[1][0][g]) - log10(f[0][0][g])) *
                                         (log10(tre + tsince) - log10(tre_dom[ind_tre[0]] + tsince)) /
                                         (log10(tre_dom[ind_tre[1]] + tsince) - log10(tre_dom[ind_tre[0]] + tsince));
    float f_d1 = log10(f[0][1][g]) + (log10(f[1][1][g]) - log10(f[0][1][g])) *
                                         (log10(tre + tsince) - log10(tre_dom[ind_tre[0]] + tsince)) /
                                         (log10(tre_dom[ind_tre[1]] + tsince) - log10(tre_dom[ind_tre[0]] + tsince));
    float f_dg = f_d0 + (f_d1 - f_d0) * (log10(1. + deltaNL) - log10(1. + c.sg_dnl_dom[ind_delta[0]])) /
                            (log10(1. + c.sg_dnl_dom[ind_delta[1]]) - log10(1. + c.sg_dnl_dom[ind_delta[0]]));
    out[g + 1] = pow(10., f_dg);
    out[g + 1] = mind(out[g + 1], kMaxSubgridFrac);
  }
  out[0] = pow(kGammaDom[0] / kGammaDom[1], 0.) * out[1];
  out[4] = pow(kGammaDom[4] / kGammaDom[3], -1.) * out[3];
}

// the HI fractions of the RadHydro runs at time x since ionisation, linear in time between the
// table rows itf and itf + 1, for the tre indices ind_tre and the density indices ind_delta
static void sg_fh1_at(const Ctx& c, int itf, float x, const int ind_tre[2], const int ind_delta[2], float f[2][2][3]) {
  const int ind_gamma[3] = {1, 2, 3};
  const float* T = c.sg_time.data();
  const float* H = c.sg_fh1.data();
  for (int m = 0; m < 2; m++)
    for (int p = 0; p < 2; p++)
      for (int g = 0; g < 3; g++) {
        const int im = ind_tre[m], ip = ind_delta[p], iq = ind_gamma[g];
        float v = H[sg_at(itf, im, ip, iq)] + (H[sg_at(itf + 1, im, ip, iq)] - H[sg_at(itf, im, ip, iq)]) /
                                                  (T[sg_at(itf + 1, im, ip, iq)] - T[sg_at(itf, im, ip, iq)]) *
                                                  (x - T[sg_at(itf, im, ip, iq)]);
        f[m][p][g] = mind(maxd(v, 0.), 1.);
      }
}

// get_gamma_interp (subgrid.cc:257-545) for the HI fraction, the one interpolant the equilibrium
// model reads (interp_nh1). Once an I-front has started to cross the cell (tcross_flag), the
// interpolant is the average over the tenths of the cell the fronts have passed, each tenth
// evaluated at its own crossing time, weighted up to fion_max.
static void sg_gamma_interp(Ctx& c, long q, float tre, float deltaNL, float tsince) {
  int ind_tre[2], ind_delta[2];
  tre = maxd(c.sg_t12, tre);
  if (tre > c.sg_t8) { ind_tre[1] = 2; ind_tre[0] = 1; }
  else { ind_tre[1] = 1; ind_tre[0] = 0; }
  if (sg_deltasig(deltaNL, c.zz) < 0.) { ind_delta[1] = 1; ind_delta[0] = 0; }
  else { ind_delta[1] = 2; ind_delta[0] = 1; }
  float out[5];
  {
    float f[2][2][3];
    sg_fh1_at(c, sg_tindex(c, tsince), tsince, ind_tre, ind_delta, f);
    sg_gamma_f(c, tsince, tre, deltaNL, ind_tre, ind_delta, f, out);
  }
  if (c.ifront && c.tcross_flag[q]) {
    const float* tcn = &c.tcross_new[(size_t)q * kNtcross];
    float ftt[kNtcross][5];
    for (int tt = 0; tt < kNtcross; tt++) {
      int ind_tre_tc[2];
      if (tre + tcn[tt] > c.sg_t8) { ind_tre_tc[1] = 2; ind_tre_tc[0] = 1; }
      else { ind_tre_tc[1] = 1; ind_tre_tc[0] = 0; }
      float tc = 0.;
      if (tt == 0) tc = tcn[0] / 2.;
      else tc = tcn[tt - 1] + (tcn[tt] - tcn[tt - 1]) / 2.;
      float f[2][2][3];
      sg_fh1_at(c, sg_tindex(c, tsince - tc), tsince - tc, ind_tre_tc, ind_delta, f);
      sg_gamma_f(c, tsince - tc, tre + tc, deltaNL, ind_tre_tc, ind_delta, f, ftt[tt]);
    }
    const float fmax = c.fion_max[q];
    for (int g = 0; g < 5; g++) {
      float acc = 0.;
      if (fmax == 1.) {
        for (int tt = 0; tt < kNtcross; tt++) {
          float tc_frac = 1. / ((float)kNtcross);
          acc += tc_frac * ftt[tt][g];
        }
      } else {
        for (int tt = 0; tt < kNtcross; tt++) {
          float tc_frac = 1. / ((float)kNtcross);
          if ((fmax >= tt * tc_frac) && (fmax < (tt + 1.) * tc_frac)) {
            for (int ttt = 0; ttt < tt; ttt++) acc += tc_frac * ftt[ttt][g];
            acc += (maxd(0.01, fmax) - tt * tc_frac) * ftt[tt][g];
          }
        }
      }
      acc = acc / maxd(0.01, fmax);
      out[g] = mind(acc, kMaxSubgridFrac);
    }
  }
  for (int g = 0; g < 5; g++) c.sg_fh1_interp[(size_t)q * 5 + g] = out[g];
}

// interp_nh1 (subgrid.cc:629-641), interp_nhe1 (644-647)
static void sg_interp_nh1(Ctx& c, long q, float gammaH1) {
  float gamma = maxd(gammaH1, kGammaMin);
  int g = (int)floor(((float)3 + 2 - 1.) * (log10(gamma) - log10(kGammaDom[0])) /
                     (log10(kGammaDom[3 + 2 - 1]) - log10(kGammaDom[0])));
  g = imax(0, imin(g, 3 + 2 - 2));
  const float* fh = &c.sg_fh1_interp[(size_t)q * 5];
  c.nH1[q] = log10(fh[g]) + (log10(fh[g + 1]) - log10(fh[g])) / (log10(kGammaDom[g + 1]) - log10(kGammaDom[g])) *
                                (log10(gamma) - log10(kGammaDom[g]));
  c.nH1[q] = maxd(mind(pow(10., c.nH1[q]), c.fH1_0), 0.);
  c.nH1[q] *= c.nH[q];
  c.nHe1[q] = c.nH1[q] * c.nHe[q] / c.nH[q];
  c.avg_nhe1[q] = c.nHe1[q];
}

static float rmin_from_l(const Ctx& c, short l) {
  float r = c.dx0 * pow(2, l - 1) * pow(3. / O_PI / c.safety_factor, 0.5);
  if (l == 0) r = 0.;
  return r;
}
static float rmax_from_l(const Ctx& c, short l) { return c.dx0 * pow(2, l) * pow(3. / O_PI / c.safety_factor, 0.5); }
static short l_from_r(const Ctx& c, float r) {
  short l = (short)imin((int)ceil(log(O_PI * c.safety_factor / 3. * pow(r / c.dx0, 2.)) / log(4.)), (int)c.l_max);
  l = mins(c.l_max, maxs(c.hpx_lvl, l));
  if (r / c.dx0 < 1.) l = c.hpx_lvl;
  return l;
}

// forward (direction 0) and inverse (direction 6) ZYX rotation, healpix_funcs.cc:102-143
static void rotate(float a0, float b0, float g0, int direction, double vx, double vy, double vz, double* ox,
                   double* oy, double* oz) {
  float xhat = (float)vx, yhat = (float)vy, zhat = (float)vz, xp, yp, zp;
  if (direction == 0) {
    xp = (cos(b0) * cos(g0)) * xhat + (-cos(b0) * sin(g0)) * yhat + (sin(b0)) * zhat;
    yp = (sin(a0) * sin(b0) * cos(g0) + cos(a0) * sin(g0)) * xhat +
         (-sin(a0) * sin(b0) * sin(g0) + cos(a0) * cos(g0)) * yhat + (-sin(a0) * cos(b0)) * zhat;
    zp = (-cos(a0) * sin(b0) * cos(g0) + sin(a0) * sin(g0)) * xhat +
         (cos(a0) * sin(b0) * sin(g0) + sin(a0) * cos(g0)) * yhat + (cos(a0) * cos(b0)) * zhat;
  } else {
    xp = (cos(g0) * cos(b0)) * xhat + (sin(g0) * cos(a0) + cos(g0) * sin(b0) * sin(a0)) * yhat +
         (sin(g0) * sin(a0) - cos(g0) * sin(b0) * cos(a0)) * zhat;
    yp = (-sin(g0) * cos(b0)) * xhat + (cos(g0) * cos(a0) - sin(g0) * sin(b0) * sin(a0)) * yhat +
         (cos(g0) * sin(a0) + sin(g0) * sin(b0) * cos(a0)) * zhat;
    zp = (sin(b0)) * xhat + (-cos(b0) * sin(a0)) * yhat + (cos(b0) * cos(a0)) * zhat;
  }
  *ox = xp;
  *oy = yp;
  *oz = zp;
}

// ---- set-up -----------------------------------------------------------------------------
struct Params {
  int N, F, path_length, itercount, ray_per_cell_max, hpx_lvl;
  double nu_eV[kMaxF];
  double spectrum_alpha[15];
  double spectrum_table[15][kMaxF];
  float cl_factor, box_hmpc, z, const_clump;
  double rkill_cm;
  unsigned int seed;
};

static void set_spectrum(Ctx& c, const Params& p) {
  // read_spectrum_table + set_spectrum (gas_funcs.cc:11-70) with the table passed in
  const int Nalph = 15;
  double alpha_spec = 1.5;
  int m = floor((alpha_spec - p.spectrum_alpha[0]) / (p.spectrum_alpha[Nalph - 1] - p.spectrum_alpha[0]) * (Nalph - 1));
  m = imin(m, Nalph - 2);
  int q = m + 1;
  float spec_sum = 0.;
  for (int nu = 0; nu < c.F; nu++) {
    c.spectrum[nu] = (float)(p.spectrum_table[m][nu] + (p.spectrum_table[q][nu] - p.spectrum_table[m][nu]) /
                                                           (p.spectrum_alpha[q] - p.spectrum_alpha[m]) *
                                                           (alpha_spec - p.spectrum_alpha[m]));
    spec_sum += c.spectrum[nu];
  }
  for (int nu = 0; nu < c.F; nu++) c.spectrum[nu] /= spec_sum;
}

static void alloc(Ctx& c) {
  const size_t n3 = (size_t)c.N * c.N * c.N;
  std::vector<float>* f[] = {&c.rho, &c.nH, &c.nHe, &c.nH1, &c.nHe1, &c.nH2, &c.nHe2, &c.nHe3, &c.ne, &c.n_tot,
                             &c.f_H1, &c.f_He1, &c.f_H2, &c.f_He2, &c.f_He3, &c.temp, &c.clump, &c.avg_nh1,
                             &c.avg_nhe1, &c.avg_gamma, &c.avg_gamma_he1, &c.recomb_H2, &c.recomb_He2,
                             &c.recomb_He3, &c.recrate_H2, &c.recrate_He2, &c.dne_dt, &c.mfp, &c.mfp_912, &c.treion,
                             &c.treion_out, &c.heat_rate, &c.cool_rate, &c.gamma_H1_tot, &c.gamma_He1_tot,
                             &c.nH1_prev, &c.IF_speed, &c.Inc_Flux, &c.ray_dt, &c.rho_prev, &c.ddelta_dt};
  for (auto* v : f) v->assign(n3, 0.f);
  std::vector<float>* g[] = {&c.gamma_H1_nu, &c.gamma_He1_nu, &c.ngam_nu, &c.u_nu, &c.avg_gamma_nu,
                             &c.avg_gamma_nu_he1};
  for (auto* v : g) v->assign(n3 * c.F, 0.f);
  c.treion_flag.assign(n3, 0);
}

static void init_rays(Ctx& c, int i, int j, int k, double lum, int src);

static void new_rays(Ctx& c) {
  long created = 0;
  for (size_t s = 0; s < c.src.size(); ++s) {
    const Src& S = c.src[s];
    init_rays(c, S.i, S.j, S.k, S.lum, (int)s);
    created += 12 * pow(2, 2 * c.hpx_lvl);
    c.ray_dt[cidx(c, S.i, S.j, S.k)] = 0.;
  }
  c.total_rays += created;
}

static void init_rays(Ctx& c, int i, int j, int k, double lum, int src) {
  const long ci = cidx(c, i, j, k);
  unsigned short itheta = (unsigned short)(rand() % kNtheta);
  float a0 = c.random_angles[itheta][0], b0 = c.random_angles[itheta][1], g0 = c.random_angles[itheta][2];
  int Nside;
  short lpix;
  if (c.nH1[ci] / c.nH[ci] > 0.1) {
    Nside = 1;
    lpix = 0;
  } else {
    Nside = (int)pow(2, c.hpx_lvl);
    lpix = c.hpx_lvl;
  }
  for (int f = 0; f < 12; f++) {
    for (int pnp = 0; pnp < pow(Nside, 2); pnp++) {
      int pix = f * pow(Nside, 2) + pnp;
      double vx, vy, vz;
      hpn::pix2vec(lpix, pix, &vx, &vy, &vz);
      rotate(a0, b0, g0, 0, vx, vy, vz, &vx, &vy, &vz);
      Ray R;
      memset(&R, 0, sizeof R);
      R.alive = true;
      R.active = true;
      R.order = lpix;
      R.pixel = pix;
      R.itheta = itheta;
      R.xhat = vx;
      R.yhat = vy;
      R.zhat = vz;
      for (int nu = 0; nu < c.F; nu++)
        R.nphot[nu] = (float)(c.spectrum[nu] * lum * c.ray_dt[ci] / 12. / pow(Nside, 2.) / kPhotNorm);
      R.r = 0.;
      R.dr = rmax_from_l(c, lpix) - R.r;
      R.x = c.dxc / 2.;
      R.y = c.dxc / 2.;
      R.z = c.dxc / 2.;
      R.time = 0.;
      R.pind[0] = i * c.N * c.N + j * c.N + k;
      R.src = src;
      for (int nu = 0; nu < c.F; nu++) c.led_emitted += (double)R.nphot[nu] * kPhotNorm;
      c.rays.push_back(R);
    }
  }
}

// ---- advance (ray_tracing.cc:1222-1512) ------------------------------------------------------
static void advance_ray(Ctx& c, Ray& R) {
  float tx, ty, tz, tmin = 0;
  int tag;
  const float dxc = c.dxc;
  int i, j, k;
  split_ind(c, R.pind[0], &i, &j, &k);
  float xhat = R.xhat, yhat = R.yhat, zhat = R.zhat;
  float x0 = R.x, y0 = R.y, z0 = R.z;
  R.time += c.dt;
  float deltat = R.time;
  float dist = c.clight * deltat;
  const float nc = c.nc;
  if ((x0 + dist * xhat > nc * dxc) || (y0 + dist * yhat > nc * dxc) || (z0 + dist * zhat > nc * dxc) ||
      (x0 + dist * xhat < (1. - nc) * dxc) || (y0 + dist * yhat < (1. - nc) * dxc) ||
      (z0 + dist * zhat < (1. - nc) * dxc)) {
    float r0 = R.r, dr = R.dr;
    int p = 0;
    R.time = 0.;
    float scale_factor = dxc / c.dx0;
    r0 += dist / scale_factor;
    dr -= dist / scale_factor;
    int in = i, jn = j, kn = k;
    float tlast = 0.;
    while (tlast < deltat) {
      float clgt = c.clight;
      if (xhat > 0.) tx = (dxc - x0) / xhat / clgt;
      else if (xhat < 0.) tx = -1. * x0 / xhat / clgt;
      else tx = 9e99;
      if (yhat > 0.) ty = (dxc - y0) / yhat / clgt;
      else if (yhat < 0.) ty = -1. * y0 / yhat / clgt;
      else ty = 9e99;
      if (zhat > 0.) tz = (dxc - z0) / zhat / clgt;
      else if (zhat < 0.) tz = -1. * z0 / zhat / clgt;
      else tz = 9e99;
      if ((tx <= ty) && (tx <= tz)) { tmin = tx; tag = 0; }
      else if ((ty <= tx) && (ty <= tz)) { tmin = ty; tag = 1; }
      else { tmin = tz; tag = 2; }
      if ((tlast + tmin) < deltat) {
        dist = tmin * clgt;
        if (p >= c.PL) { fprintf(stderr, "oracle: path overflow\n"); abort(); }
        R.pind[p] = in * c.N * c.N + jn * c.N + kn;
        R.pdist[p] = dist;
        p += 1;
        x0 += dist * xhat;
        y0 += dist * yhat;
        z0 += dist * zhat;
        if (tag == 0) {
          if (xhat > 0.) { in = imod(in + 1, c.N); x0 = kMinDist * dxc; }
          else { in = imod(in - 1, c.N); x0 = dxc * (1. - kMinDist); }
        } else if (tag == 1) {
          if (yhat > 0.) { jn = imod(jn + 1, c.N); y0 = kMinDist * dxc; }
          else { jn = imod(jn - 1, c.N); y0 = dxc * (1. - kMinDist); }
        } else {
          if (zhat > 0.) { kn = imod(kn + 1, c.N); z0 = kMinDist * dxc; }
          else { kn = imod(kn - 1, c.N); z0 = dxc * (1. - kMinDist); }
        }
        if (x0 <= 0.) x0 = kMinDist * dxc;
        if (x0 >= dxc * (1. - kMinDist / 2.)) x0 = dxc * (1. - kMinDist);
        if (y0 <= 0.) y0 = kMinDist * dxc;
        if (y0 >= dxc * (1. - kMinDist / 2.)) y0 = dxc * (1. - kMinDist);
        if (z0 <= 0.) z0 = kMinDist * dxc;
        if (z0 >= dxc * (1. - kMinDist / 2.)) z0 = dxc * (1. - kMinDist);
      }
      tlast += tmin;
    }
    // in a cell a front has not fully passed, the last segment is the whole crossing of the cell
    // (ray_tracing.cc:1425-1437)
    if (fion_of(c, in * c.N * c.N + jn * c.N + kn) < 1.) dist = tmin * c.clight;
    else dist = (deltat - tlast + tmin) * c.clight;
    dist = maxd(dist, kMinDist * dxc);
    if (p >= c.PL) { fprintf(stderr, "oracle: path overflow\n"); abort(); }
    R.pind[p] = in * c.N * c.N + jn * c.N + kn;
    R.pdist[p] = dist;
    R.ray_end = p + 1;
    x0 += dist * xhat;
    y0 += dist * yhat;
    z0 += dist * zhat;
    if (x0 <= 0.) x0 = kMinDist * dxc;
    if (x0 >= dxc * (1. - kMinDist / 2.)) x0 = dxc * (1. - kMinDist);
    if (y0 <= 0.) y0 = kMinDist * dxc;
    if (y0 >= dxc * (1. - kMinDist / 2.)) y0 = dxc * (1. - kMinDist);
    if (z0 <= 0.) z0 = kMinDist * dxc;
    if (z0 >= dxc * (1. - kMinDist / 2.)) z0 = dxc * (1. - kMinDist);
    R.active = false;
    R.r = r0;
    R.dr = dr;
    R.x = x0;
    R.y = y0;
    R.z = z0;
  }
}

static void update_rays(Ctx& c) {
  for (const Src& S : c.src) c.ray_dt[cidx(c, S.i, S.j, S.k)] += c.dt;
  for (Ray& R : c.rays)
    if (R.alive) advance_ray(c, R);
}

// the equilibrium mean free paths of an ionised cell (ray_tracing.cc:989-994, 1031-1036)
static void sg_eq_mfp(Ctx& c, long q) {
  c.mfp[q] = maxd(kGammaMin, c.avg_gamma[q]) / c.clump[q] / kSigmaEffRH / alphaB_H2(maxd(kTempMin, c.temp[q])) /
             pow(c.nH[q], 2.) / 1.082;
  c.mfp_912[q] = maxd(kGammaMin, c.avg_gamma[q]) / c.clump[q] / sig_H1(13.6 / O_H_EV) /
                 alphaB_H2(maxd(kTempMin, c.temp[q])) / pow(c.nH[q], 2.) / 1.082;
  c.mfp[q] = maxd(0.f, c.mfp[q]);   // mfp_min = 1e-2*dx[0] taken while dx is still 0 (global_variables.cc:301)
  c.mfp_912[q] = maxd(0.f, c.mfp_912[q]);
}

// set_Treion (subgrid.cc:660-670): the temperature of the newly ionised part of a cell from the
// I-front speed (D'Aloisio et al. 2019 fit), averaged into the cell's temperature
static void set_Treion(Ctx& c, long q, float vIF, float fi_old, float fi_new) {
  float Cn[5] = {9.5432, -1.6441e-2, -9.8010e-3, 4.1664e-3, -2.2710e-4};
  float lnTreion = 0.;
  for (int t = 0; t < 5; t++) lnTreion += Cn[t] * pow(log(vIF / 1e5), t);
  if (fi_new > 0.) c.temp[q] = (fi_old * c.temp[q] + (fi_new - fi_old) * exp(lnTreion)) / fi_new;
}

// update_fion (subgrid.cc:694-751): the front advances by vIF dt / dx with vIF from the photons
// entering the neutral part, and the crossing times are booked per tenth of the cell
static void update_fion(Ctx& c, long q) {
  float tdiff;
  float vIF_min = 5e1 * 1e5;
  double Fl = c.ngam3[(size_t)q * 3 + 2] / pow(c.dxc, 2.) / c.dt;
  float vIF = (float)(Fl / c.nH[q] / (1. + kNheToNh));
  float fion_old = c.fion[q];
  float fion_max_old = c.fion_max[q];
  c.fion[q] = mind(c.fion[q] + vIF * c.dt / c.dxc, 1.);
  if (c.fion[q] > c.fion_max[q]) c.fion_max[q] = c.fion[q];
  if ((vIF > vIF_min) || (fion_old == 0.)) set_Treion(c, q, maxd(vIF, vIF_min), fion_old, c.fion[q]);
  if ((fion_old < 0.5) && (c.fion[q] >= 0.5)) c.treion_out[q] = c.t - c.dt;
  if (c.fion[q] >= 1.) tdiff = 0.5 * c.dt;
  else tdiff = 0.;
  c.IF_speed[q] = vIF;
  c.Inc_Flux[q] = Fl;
  c.Delta_fion[q] = c.fion[q] - fion_old;
  c.tcross[q] += c.dt - tdiff;
  for (int tt = 0; tt < kNtcross; tt++) {
    float tc_frac = 1. / ((float)kNtcross);
    float& tn = c.tcross_new[(size_t)q * kNtcross + tt];
    unsigned char& ck = c.tcross_check[(size_t)q * kNtcross + tt];
    if ((c.fion_max[q] < tc_frac * (tt + 1.)) && !ck) {
      tn += c.dt;
    } else if ((c.fion_max[q] >= tc_frac * (tt + 1.)) && (fion_max_old < tc_frac * (tt + 1.)) && !ck) {
      tn += c.dt * (tc_frac * (tt + 1.) - fion_max_old) / (c.fion_max[q] - fion_max_old);
      ck = 1;
    }
  }
  if (!c.tcross_flag[q]) c.tcross_flag[q] = 1;
}

// ---- C2Ray iteration (ray_tracing.cc:623-1216), plain mode -------------------------------
static void find_avg_unu(Ctx& c) {
  const long n3 = (long)c.N * c.N * c.N;
  const int F = c.F;
  const double vol = ((double)c.dxc) * ((double)c.dxc) * ((double)c.dxc);
  for (int iter = 0; iter < c.itercount; iter++) {
    for (long q = 0; q < n3; q++) {
      c.avg_gamma[q] = 0.;
      c.avg_gamma_he1[q] = 0.;
      c.IF_speed[q] = 0.;
      c.Inc_Flux[q] = 0.;
      if (c.ifront) {
        c.ngam3[(size_t)q * 3] = c.ngam3[(size_t)q * 3 + 1] = c.ngam3[(size_t)q * 3 + 2] = 0.;
        c.Delta_fion[q] = 0.;
      }
      for (int nu = 0; nu < F; nu++) {
        c.ngam_nu[q * F + nu] = 0.;
        c.avg_gamma_nu[q * F + nu] = 0.;
        c.avg_gamma_nu_he1[q * F + nu] = 0.;
        c.u_nu[q * F + nu] = 0.;
      }
      if (iter == 0) {
        c.avg_nh1[q] = c.nH1[q];
        c.avg_nhe1[q] = c.nHe1[q];
        c.recomb_H2[q] = (float)alphaB_H2(maxd(kTempMin, c.temp[q]));
        c.recomb_He2[q] = (float)alphaB_He2(maxd(kTempMin, c.temp[q]));
        c.recomb_He3[q] = (float)alphaB_He3(maxd(kTempMin, c.temp[q]));
        if ((c.temp[q] >= 3e4) && (c.temp[q] <= 1e6)) c.recomb_He2[q] += (float)Dalpha_He2(maxd(kTempMin, c.temp[q]));
        if (!c.subgrid) {
          c.dne_dt[q] = -c.ne[q];
          c.mfp[q] = 1. / c.nH1[q] / c.sigH1[0];
        } else {
          // the gas is taken as fully ionised (ray_tracing.cc:679-682); ionised cells get their
          // HI-fraction interpolants, the others the mfp of their neutral gas (687-693)
          c.dne_dt[q] = -(c.nH[q] + c.nHe[q]);
          if (c.treion_flag[q])
            sg_gamma_interp(c, q, c.treion[q] + c.sg_tinit, c.rho[q] / c.avg_rho - 1., c.t - c.treion[q]);
          else
            c.mfp[q] = 1. / c.nH1[q] / c.sigH1[0];
        }
      }
    }
    // ray pass
    for (Ray& R : c.rays) {
      if (!(R.alive && !R.active)) continue;
      double nphot[kMaxF], tau_h1[kMaxF], dtau_h1[kMaxF], tau_he1[kMaxF], dtau_he1[kMaxF];
      for (int nu = 0; nu < F; nu++) {
        nphot[nu] = R.nphot[nu] * kPhotNorm;
        tau_h1[nu] = 0.;
        dtau_h1[nu] = 0.;
        tau_he1[nu] = 0.;
        dtau_he1[nu] = 0.;
      }
      short p = 0;
      unsigned dump_mask = 0;   // ledger: bins that a dump deposited
      if (c.subgrid) {
        // sub-grid ray pass (ray_tracing.cc:701-938 with subgrid = TRUE): fixed H/He split, Gamma
        // from the sub-grid effective cross section over the effective path in the part of the
        // cell the fronts have passed, the segment's optical depth from the cell's mean free path
        // there (a cell no front has reached keeps the previous segment's dtau); with I-front
        // tracking, the neutral part of a cell absorbs the photons of the rays in ray order up to
        // its hydrogen and helium atoms (ray_tracing.cc:863-919)
        const double frac_h1 = 1. - (O_Y / 4.) / (1. - O_Y + O_Y / 4.);
        const double frac_he1 = (O_Y / 4.) / (1. - O_Y + O_Y / 4.);
        short p_prev = 0;
        while (p < R.ray_end) {
          const long q = R.pind[p];
          const float fion = fion_of(c, q);
          double nphot_in[kMaxF];
          double nphot_in_total = 0.;
          for (int nu = 0; nu < F; nu++) {
            nphot_in[nu] = nphot[nu] * exp(-tau_h1[nu] - tau_he1[nu]);
            nphot_in_total += nphot_in[nu] / kPhotNorm;
          }
          const bool dump = nphot_in_total < c.nphot_min;
          for (int nu = 0; nu < F; nu++) {
            c.ngam_nu[q * F + nu] += (float)(nphot_in[nu] / kPhotNorm);
            if (fion > 0.) {
              float delta_s_eff;
              if (iter == 0) delta_s_eff = fion * R.pdist[p] / frac_h1;
              else delta_s_eff = c.mfp[q] * (1. - exp(-fion * R.pdist[p] / c.mfp[q] / frac_h1));
              c.avg_gamma_nu[q * F + nu] += (float)(frac_h1 * nphot_in[nu] * kSigmaEffRH * delta_s_eff / c.dt / vol / fion);
              c.avg_gamma[q] += (float)(frac_h1 * nphot_in[nu] * kSigmaEffRH * delta_s_eff / c.dt / vol / fion);
              c.avg_gamma_nu_he1[q * F + nu] += (float)(frac_he1 * nphot_in[nu] * kSigmaEffRH * delta_s_eff / c.dt / vol / fion);
              c.avg_gamma_he1[q] += (float)(frac_he1 * nphot_in[nu] * kSigmaEffRH * delta_s_eff / c.dt / vol / fion);
            }
          }
          p = dump ? 99 : p + 1;
          if (fion > 0.)
            for (int nu = 0; nu < F; nu++) {
              dtau_h1[nu] = fion * R.pdist[p_prev] / c.mfp[q];
              dtau_he1[nu] = kNheToNh * dtau_h1[nu];
            }
          double before = 0.;   // ledger: the photons entering the segment
          for (int nu = 0; nu < F; nu++) {
            before += nphot_in[nu];
            tau_h1[nu] += dtau_h1[nu];
            tau_he1[nu] += dtau_he1[nu];
          }
          if (fion < 1.) {
            double* ng = &c.ngam3[(size_t)q * 3];
            const double sum_ngam = ng[0];
            const double chi = kNheToNh;
            const double free_ngam = vol * c.nH[q] * (1. + chi) * (1. - fion);
            double nphot_left = 0.;
            for (int nu = 0; nu < F; nu++) ng[2] += nphot_in[nu] * exp(-(dtau_h1[nu] + dtau_he1[nu]));
            if (sum_ngam < free_ngam) {
              for (int nu = 0; nu < F; nu++) {
                const double ngam_abs = mindd(nphot_in[nu] * exp(-(dtau_h1[nu] + dtau_he1[nu])), free_ngam - sum_ngam);
                ng[0] += ngam_abs;
                ng[1] += ngam_abs * kSigmaEffRH * R.pdist[p_prev];
                nphot_in[nu] = nphot_in[nu] * exp(-(dtau_h1[nu] + dtau_he1[nu])) - ngam_abs;
                nphot_left += nphot_in[nu];
              }
              if (nphot_left == 0.) {
                p = 99;
                for (int nu = 0; nu < F; nu++) tau_h1[nu] = 999.;
              } else {
                for (int nu = 0; nu < F; nu++)
                  tau_h1[nu] += -log(nphot_in[nu] / nphot[nu] / exp(-(tau_h1[nu] + tau_he1[nu])));
              }
            }
          }
          if (iter == c.itercount - 1) {
            // ledger: what the segment took out of the ray
            double after = 0.;
            for (int nu = 0; nu < F; nu++) after += nphot[nu] * exp(-tau_h1[nu] - tau_he1[nu]);
            c.led_deposited += before - after;
          }
          p_prev = p;
        }
      }
      double colH = 0., colHe = 0.;   // the columns of this pass's segments (tau limit)
      while (!c.subgrid && p < R.ray_end) {
        const int ind = R.pind[p];
        const long q = ind;
        colH += (double)c.avg_nh1[q] * (double)R.pdist[p];
        colHe += (double)c.avg_nhe1[q] * (double)R.pdist[p];
        for (int nu = 0; nu < F; nu++) {
          dtau_h1[nu] = c.avg_nh1[q] * c.sigH1[nu] * R.pdist[p];
          dtau_he1[nu] = c.avg_nhe1[q] * c.sigHe1[nu] * R.pdist[p];
        }
        double nphot_in[kMaxF];
        double nphot_in_total = 0.;
        for (int nu = 0; nu < F; nu++) {
          nphot_in[nu] = nphot[nu] * exp(-tau_h1[nu] - tau_he1[nu]);
          nphot_in_total += nphot_in[nu] / kPhotNorm;
        }
        double frac_h1[kMaxF], frac_he1[kMaxF];
        for (int nu = 0; nu < F; nu++) {
          if ((dtau_h1[nu] > 0.) || (dtau_he1[nu] > 0.)) {
            frac_h1[nu] = (1. - exp(-dtau_h1[nu])) * exp(-dtau_he1[nu]) /
                          ((1. - exp(-dtau_h1[nu])) * exp(-dtau_he1[nu]) + (1. - exp(-dtau_he1[nu])) * exp(-dtau_h1[nu]));
            frac_he1[nu] = (1. - exp(-dtau_he1[nu])) * exp(-dtau_h1[nu]) /
                           ((1. - exp(-dtau_h1[nu])) * exp(-dtau_he1[nu]) + (1. - exp(-dtau_he1[nu])) * exp(-dtau_h1[nu]));
          } else {
            frac_h1[nu] = 0.;
            frac_he1[nu] = 0.;
          }
        }
        const bool last_iter = (iter == c.itercount - 1);
        if (nphot_in_total < c.nphot_min) {
          for (int nu = 0; nu < F; nu++) {
            if (last_iter) {
              c.led_deposited += (frac_h1[nu] + frac_he1[nu]) * nphot_in[nu];
              if (frac_h1[nu] + frac_he1[nu] > 0.) dump_mask |= 1u << nu;
            }
            c.ngam_nu[q * F + nu] += (float)(nphot_in[nu] / kPhotNorm);
            c.avg_gamma_nu[q * F + nu] += (float)(frac_h1[nu] * nphot_in[nu] / c.dt / vol / c.avg_nh1[q]);
            c.avg_gamma[q] += (float)(frac_h1[nu] * nphot_in[nu] / c.dt / vol / c.avg_nh1[q]);
            c.avg_gamma_nu_he1[q * F + nu] += (float)(frac_he1[nu] * nphot_in[nu] / c.dt / vol / c.avg_nhe1[q]);
            c.avg_gamma_he1[q] += (float)(frac_he1[nu] * nphot_in[nu] / c.dt / vol / c.avg_nhe1[q]);
          }
          p = 99;
        } else {
          for (int nu = 0; nu < F; nu++) {
            if (last_iter)
              c.led_deposited += (frac_h1[nu] + frac_he1[nu]) * nphot_in[nu] * (1. - exp(-dtau_h1[nu] - dtau_he1[nu]));
            c.ngam_nu[q * F + nu] += (float)(nphot_in[nu] / kPhotNorm);
            c.avg_gamma_nu[q * F + nu] +=
                (float)(frac_h1[nu] * nphot_in[nu] * (1. - exp(-dtau_h1[nu] - dtau_he1[nu])) / c.dt / vol / c.avg_nh1[q]);
            c.avg_gamma[q] +=
                (float)(frac_h1[nu] * nphot_in[nu] * (1. - exp(-dtau_h1[nu] - dtau_he1[nu])) / c.dt / vol / c.avg_nh1[q]);
            c.avg_gamma_nu_he1[q * F + nu] += (float)(frac_he1[nu] * nphot_in[nu] *
                                                      (1. - exp(-dtau_h1[nu] - dtau_he1[nu])) / c.dt / vol / c.avg_nhe1[q]);
            c.avg_gamma_he1[q] += (float)(frac_he1[nu] * nphot_in[nu] * (1. - exp(-dtau_h1[nu] - dtau_he1[nu])) /
                                          c.dt / vol / c.avg_nhe1[q]);
          }
          p += 1;
        }
        for (int nu = 0; nu < F; nu++) {
          tau_h1[nu] += dtau_h1[nu];
          tau_he1[nu] += dtau_he1[nu];
        }
      }
      if (iter == c.itercount - 1) {
        for (int nu = 0; nu < F; nu++) R.nphot[nu] = (float)(nphot[nu] * exp(-tau_h1[nu] - tau_he1[nu]) / kPhotNorm);
        bool tau_over = false;
        if (c.tau_max > 0. && !c.subgrid) {
          // opt-in limit: the ray's optical depth since its cast in its most transparent bin
          R.colH += colH;
          R.colHe += colHe;
          double tau_min = 1e300;
          for (int nu = 0; nu < F; nu++) tau_min = mindd(tau_min, c.sigH1[nu] * R.colH + c.sigHe1[nu] * R.colHe);
          tau_over = tau_min > c.tau_max;
        }
        if (sum_nphot(c, R) > c.nphot_min && !tau_over) {
          R.active = true;
          R.pind[0] = R.pind[R.ray_end - 1];
        } else {
          c.led_killed += (double)sum_nphot(c, R) * kPhotNorm;
          for (int nu = 0; nu < F; nu++)
            if (dump_mask & (1u << nu)) c.led_overlap += (double)R.nphot[nu] * kPhotNorm;
          R.alive = false;
          R.active = false;
        }
      }
    }
    // cell pass B
    for (long q = 0; q < n3 && c.subgrid; q++) {
      // the sub-grid branch (ray_tracing.cc:956-1071, equilibrium = TRUE) and the last-iteration
      // bookkeeping (1138-1209)
      double nelec = (double)(c.nH[q] - c.avg_nh1[q] + c.nHe[q] - c.avg_nhe1[q]);
      const bool last = iter == c.itercount - 1;
      const double* ng = c.ifront ? &c.ngam3[(size_t)q * 3] : nullptr;
      bool first = false;
      if (last && !c.treion_flag[q] && ((c.ifront && ng[1] > 0.) || (c.avg_gamma[q] > 0.))) {
        c.treion[q] = c.t - c.dt;
        c.treion_flag[q] = 1;
        sg_gamma_interp(c, q, c.treion[q] + c.sg_tinit, c.rho[q] / c.avg_rho - 1., c.t - c.treion[q]);
        first = true;
      }
      if (c.treion_flag[q] && fion_of(c, q) > 0.) sg_eq_mfp(c, q);
      if (c.ifront && c.treion_flag[q] && last && (c.fion[q] < 1.)) {
        // I-front correction (ray_tracing.cc:1003-1047)
        const double gamma_fion = ng[1] / c.dt / vol;
        update_fion(c, q);
        if (c.fion[q] >= 1.) c.neutral_flag[q] = 0;
        float clump_fion = c.clump[q];   // equilibrium: C_HII
        if ((c.fion[q] < 1.) && (c.avg_gamma[q] == 0.) && !first)
          c.fion[q] = maxd(0., c.fion[q] - clump_fion * alphaB_H2(maxd(kTempMin, c.temp[q])) * (1. + kNheToNh) *
                                               c.nH[q] * c.fion[q] * c.dt);
        if (first) {   // a newly ionised cell: its rate and mean free path from the front's photons
          c.avg_gamma[q] = gamma_fion;
          sg_eq_mfp(c, q);
        }
      }
      if (c.ifront && (c.fion[q] == 1.) && (c.avg_gamma[q] == 0.) && last) {   // ray_tracing.cc:1051-1054
        float clump_fion_2 = c.clump[q];
        c.fion[q] = maxd(0., c.fion[q] - clump_fion_2 * alphaB_H2(maxd(kTempMin, c.temp[q])) * (1. + kNheToNh) *
                                             c.nH[q] * c.fion[q] * c.dt);
      }
      if (!last) continue;
      if (c.treion_flag[q]) {
        const float fion = fion_of(c, q);
        sg_interp_nh1(c, q, c.avg_gamma[q]);
        c.nH2[q] = c.nH[q] * fion;
        c.nHe2[q] = c.nHe[q] * fion;
        c.nHe3[q] = 0.;
      }
      for (int nu = 0; nu < F; nu++)
        c.u_nu[q * F + nu] = (float)(c.spectrum[nu] * c.avg_gamma[q] / c.sigH1[nu]) * O_H * (c.nu[nu]) / c.clight;
      for (int nu = 0; nu < F; nu++) {
        c.gamma_H1_nu[q * F + nu] = c.avg_gamma_nu[q * F + nu];
        c.gamma_He1_nu[q * F + nu] = c.avg_gamma_nu_he1[q * F + nu];
      }
      c.gamma_H1_tot[q] = c.avg_gamma[q];
      c.gamma_He1_tot[q] = c.avg_gamma_he1[q];
      c.recrate_H2[q] = c.clump[q] * c.recomb_H2[q] * nelec * c.nH2[q];
      c.recrate_He2[q] = c.clump[q] * c.recomb_He2[q] * nelec * c.nHe2[q];
      c.ne[q] = c.nH2[q] + c.nHe2[q] + 2. * c.nHe3[q];
      c.dne_dt[q] += c.nH[q] + c.nHe[q];
      c.n_tot[q] = 2. * (c.nH[q] + c.nHe[q]);
      c.dne_dt[q] /= c.dt;
      c.nH1_prev[q] = c.nH1[q];
      c.f_H2[q] = c.nH2[q] / c.nH[q];
      c.f_He2[q] = c.nHe2[q] / c.nHe[q];
      c.f_He3[q] = c.nHe3[q] / c.nHe[q];
      if (!c.ifront) {
        c.f_H1[q] = c.nH1[q] / c.nH[q];
        c.f_He1[q] = c.nHe1[q] / c.nHe[q];
      } else {
        if (c.fion[q] > 0.) {
          c.f_H2[q] *= c.fion[q];
          c.f_He2[q] *= c.fion[q];
          c.f_He3[q] *= c.fion[q];
        }
        c.f_H1[q] = (float)((double)1. - c.f_H2[q]);
        c.f_He1[q] = (float)((double)1. - c.f_He2[q] - c.f_He3[q]);
      }
    }
    for (long q = 0; q < n3 && !c.subgrid; q++) {
      double nelec = (double)(c.nH[q] - c.avg_nh1[q] + c.nHe[q] - c.avg_nhe1[q]);
      c.mfp[q] = 1. / c.sigH1[0] / c.avg_nh1[q];
      c.mfp_912[q] = 1. / sig_H1(13.6 / O_H_EV) / c.avg_nh1[q];
      double col = 0.;
      double x0 = (double)(1. - c.f_H1[q]);
      double pr = (double)c.avg_gamma[q] + col + c.clump[q] * c.recomb_H2[q] * nelec;
      double xeq = (c.avg_gamma[q] + col) / pr;
      double ti = 1. / pr;
      c.avg_nh1[q] = (float)(c.nH[q] * (1. - (xeq + ti / c.dt * (x0 - xeq) * (1. - exp(-c.dt / ti)))));
      double x0_he = (double)(1. - c.f_He1[q]);
      double pr_he = (double)c.avg_gamma_he1[q] + c.clump[q] * c.recomb_He2[q] * nelec;
      double xeq_he = c.avg_gamma_he1[q] / pr_he;
      double ti_he = 1. / pr_he;
      c.avg_nhe1[q] = (float)(c.nHe[q] * (1. - (xeq_he + ti_he / c.dt * (x0_he - xeq_he) * (1. - exp(-c.dt / ti_he)))));
      if (iter == c.itercount - 1) {
        c.nH1[q] = (float)c.nH[q] * (1. - (xeq + (x0 - xeq) * exp(-c.dt / ti)));
        c.nH2[q] = (float)c.nH[q] - c.nH1[q];
        c.nHe1[q] = (float)c.nHe[q] * (1. - (xeq_he + (x0_he - xeq_he) * exp(-c.dt / ti_he)));
        c.nHe2[q] = (float)c.nHe[q] - c.nHe1[q];
        c.nHe3[q] = 0.;
        if ((c.avg_nh1[q] / c.nH[q] < 0.5) && (c.treion_flag[q] == 0)) {
          c.treion[q] = c.t;
          c.treion_out[q] = c.t;
          c.treion_flag[q] = 1;
        }
        for (int nu = 0; nu < F; nu++)
          c.u_nu[q * F + nu] = (float)(c.spectrum[nu] * c.avg_gamma[q] / c.sigH1[nu]) * O_H * (c.nu[nu]) / c.clight;
        for (int nu = 0; nu < F; nu++) {
          c.gamma_H1_nu[q * F + nu] = c.avg_gamma_nu[q * F + nu];
          c.gamma_He1_nu[q * F + nu] = c.avg_gamma_nu_he1[q * F + nu];
        }
        c.gamma_H1_tot[q] = c.avg_gamma[q];
        c.gamma_He1_tot[q] = c.avg_gamma_he1[q];
        c.recrate_H2[q] = c.clump[q] * c.recomb_H2[q] * nelec * c.nH2[q];
        c.recrate_He2[q] = c.clump[q] * c.recomb_He2[q] * nelec * c.nHe2[q];
        c.ne[q] = c.nH2[q] + c.nHe2[q] + 2. * c.nHe3[q];
        c.dne_dt[q] += c.ne[q];
        c.n_tot[q] = c.nH[q] + c.nHe[q] + c.ne[q];
        c.dne_dt[q] /= c.dt;
        c.f_H2[q] = c.nH2[q] / c.nH[q];
        c.f_He2[q] = c.nHe2[q] / c.nHe[q];
        c.f_He3[q] = c.nHe3[q] / c.nHe[q];
        c.f_H1[q] = c.nH1[q] / c.nH[q];
        c.f_He1[q] = c.nHe1[q] / c.nHe[q];
      }
    }
  }
}

// ---- merge machinery (ray_tracing.cc:35-227, 324-477) -------------------------------------
static long count_rays(const Ctx& c) {
  long n = 0;
  for (const Ray& R : c.rays) n += R.alive ? 1 : 0;
  return n;
}

static void calc_nphot_merge(Ctx& c) {
  double lg_max = log10(c.nphot_max);
  double lg_min = log10(c.nphot_min);
  double del = (lg_max - lg_min) / (10000 - 1);
  static int pdf[10000];
  memset(pdf, 0, sizeof pdf);
  long ray_cum = 0;
  c.nphot_merge = 0.;
  for (const Ray& R : c.rays) {
    if (!R.alive) continue;
    int pdf_ind = (int)maxd((log10(sum_nphot(c, R)) - lg_min) / del, 0.);
    pdf_ind = imin(pdf_ind, 9999);
    pdf[pdf_ind] += 1;
  }
  int pi_ = 9999;
  while (pi_ >= 0) {
    ray_cum += pdf[pi_];
    if (ray_cum >= c.num_thresh) {
      c.nphot_merge = pow(10., pi_ * del + lg_min);
      pi_ = -1;
    } else {
      pi_ -= 1;
    }
  }
}

static void merge(Ctx& c) {
  unsigned short itheta = (unsigned short)(rand() % kNtheta);
  float a0 = c.random_angles[itheta][0], b0 = c.random_angles[itheta][1], g0 = c.random_angles[itheta][2];
  const int lm = c.hpx_lvl;
  const int npix = 12 * (1 << (2 * lm));
  const long n3 = (long)c.N * c.N * c.N;
  std::vector<long> base((size_t)n3 * npix, -1);
  std::vector<unsigned char> flag((size_t)n3 * npix, 0);
  for (size_t xi = 0; xi < c.rays.size(); ++xi) {
    Ray& R = c.rays[xi];
    if (!(R.alive && R.active)) continue;
    if (!(sum_nphot(c, R) < c.nphot_merge)) continue;
    const long q = R.pind[0];
    double vx = R.xhat, vy = R.yhat, vz = R.zhat;
    rotate(a0, b0, g0, 6, vx, vy, vz, &vx, &vy, &vz);
    const int pixel = hpn::vec2pix(lm, vx, vy, vz);
    const size_t b = (size_t)q * npix + pixel;
    if (base[b] == -1) {
      base[b] = (long)xi;
      flag[b] = 0;
      float nt = sum_nphot(c, R);
      R.r /= c.dx0;
      R.r = pow(R.r, 2.) * nt;
      R.dr *= nt;
      R.x *= nt;
      R.y *= nt;
      R.z *= nt;
      R.time *= nt;
    } else {
      Ray& M = c.rays[base[b]];
      float nt = sum_nphot(c, R);
      if (M.src != R.src) M.src = -1;
      for (int nu = 0; nu < c.F; nu++) M.nphot[nu] += R.nphot[nu];
      R.r /= c.dx0;
      M.r += pow(R.r, 2.) * nt;
      M.dr += R.dr * nt;
      M.x += R.x * nt;
      M.y += R.y * nt;
      M.z += R.z * nt;
      M.time += R.time * nt;
      flag[b] = 1;
      R.alive = false;
      R.active = false;
    }
  }
  for (long q = 0; q < n3; q++) {
    for (int pix = 0; pix < npix; pix++) {
      const size_t b = (size_t)q * npix + pix;
      if (base[b] == -1) continue;
      Ray& R = c.rays[base[b]];
      float nt = sum_nphot(c, R);
      R.r /= nt;
      R.r = pow(R.r, 0.5);
      R.r *= c.dx0;
      R.dr /= nt;
      R.x /= nt;
      R.y /= nt;
      R.z /= nt;
      R.time /= nt;
      if (flag[b]) {
        double vx, vy, vz;
        hpn::pix2vec(lm, pix, &vx, &vy, &vz);
        R.itheta = itheta;
        R.order = mins(c.l_max, l_from_r(c, R.r));
        float rmin = rmin_from_l(c, R.order);
        float rmax = rmax_from_l(c, R.order);
        R.r = maxd(rmax - R.dr, rmin);
        R.dr = rmax - R.r;
        R.pixel = hpn::vec2pix(R.order, vx, vy, vz);
        hpn::pix2vec(R.order, R.pixel, &vx, &vy, &vz);
        rotate(a0, b0, g0, 0, vx, vy, vz, &vx, &vy, &vz);
        R.xhat = vx;
        R.yhat = vy;
        R.zhat = vz;
      }
    }
  }
}

// ---- split (rt_funcs.cc:211-237, ray_tracing.cc:482-619) -----------------------------------
static void split_rays(Ctx& c) {
  const size_t n0 = c.rays.size();
  for (size_t xi = 0; xi < n0; ++xi) {
    if (!(c.rays[xi].alive && c.rays[xi].active)) continue;
    const Ray P = c.rays[xi];
    short l = P.order;
    float r = P.r;
    if (!((r > rmax_from_l(c, l)) && (l < c.l_max) && (sum_nphot(c, P) > maxd(4. * c.nphot_merge, 4. * c.nphot_min))))
      continue;
    int ic, jc, kc;
    split_ind(c, P.pind[0], &ic, &jc, &kc);
    float r0 = P.r, x0_old = P.x, y0_old = P.y, z0_old = P.z, time = P.time;
    unsigned short itheta = P.itheta;
    float a0 = c.random_angles[itheta][0], b0 = c.random_angles[itheta][1], g0 = c.random_angles[itheta][2];
    float nph[kMaxF];
    for (int nu = 0; nu < c.F; nu++) nph[nu] = P.nphot[nu] / 4.;
    const double vox = P.xhat, voy = P.yhat, voz = P.zhat;
    c.rays[xi].alive = false;
    c.rays[xi].active = false;
    for (int n = 0; n < 4; n++) {
      int icn = ic, jcn = jc, kcn = kc;
      int pix = 4 * P.pixel + n;
      double vx, vy, vz;
      hpn::pix2vec(l + 1, pix, &vx, &vy, &vz);
      rotate(a0, b0, g0, 0, vx, vy, vz, &vx, &vy, &vz);
      double dxv = vx - vox, dyv = vy - voy, dzv = vz - voz;
      float scale_factor = c.dxc / c.dx0;
      float x0 = x0_old + dxv * (r0 * scale_factor);
      float y0 = y0_old + dyv * (r0 * scale_factor);
      float z0 = z0_old + dzv * (r0 * scale_factor);
      while (x0 > c.dxc) { x0 -= c.dxc; icn = imod(icn + 1, c.N); }
      while (x0 < 0.) { x0 += c.dxc; icn = imod(icn - 1, c.N); }
      while (y0 > c.dxc) { y0 -= c.dxc; jcn = imod(jcn + 1, c.N); }
      while (y0 < 0.) { y0 += c.dxc; jcn = imod(jcn - 1, c.N); }
      while (z0 > c.dxc) { z0 -= c.dxc; kcn = imod(kcn + 1, c.N); }
      while (z0 < 0.) { z0 += c.dxc; kcn = imod(kcn - 1, c.N); }
      Ray Ch;
      memset(&Ch, 0, sizeof Ch);
      Ch.alive = true;
      Ch.active = false;
      float rmax = rmax_from_l(c, l + 1);
      Ch.order = l + 1;
      Ch.pixel = pix;
      Ch.itheta = itheta;
      Ch.xhat = vx;
      Ch.yhat = vy;
      Ch.zhat = vz;
      for (int nu = 0; nu < c.F; nu++) Ch.nphot[nu] = nph[nu];
      Ch.r = r0;
      Ch.dr = rmax - r0;
      Ch.x = x0;
      Ch.y = y0;
      Ch.z = z0;
      Ch.time = time;
      Ch.pind[0] = icn * c.N * c.N + jcn * c.N + kcn;
      Ch.src = P.src;
      Ch.colH = P.colH;
      Ch.colHe = P.colHe;
      c.rays.push_back(Ch);
    }
  }
  for (Ray& R : c.rays)
    if (R.alive && !R.active) R.active = true;
}

// ---- thermal (gas_funcs.cc:104-242, 353-457), plain mode ------------------------------------
static void set_Treion_default(Ctx& c, long q) {
  float fion_new = (c.nH[q] - c.nH1[q]) / c.nH[q];
  float fion_old = (c.nH[q] - c.nH1_prev[q]) / c.nH[q];
  float deltax = c.dxc * (fion_new - fion_old);
  float vIF = deltax / c.dt;
  float Cn[5] = {9.5432, -1.6441e-2, -9.8010e-3, 4.1664e-3, -2.2710e-4};
  float lnTreion = 0.;
  for (int t = 0; t < 5; t++) lnTreion += Cn[t] * pow(log(vIF / 1e5), t);
  if ((fion_new > fion_old) && (fion_new < 0.98)) {
    c.temp[q] = (fion_old * c.temp[q] + (fion_new - fion_old) * exp(lnTreion)) / fion_new;
  }
  c.IF_speed[q] = maxd(0., vIF);
  c.Inc_Flux[q] = (1. + kNheToNh) * c.nH[q] * maxd(0., vIF);
}

static void update_heat_cool(Ctx& c, long q) {
  const int F = c.F;
  c.heat_rate[q] = 0;
  c.cool_rate[q] = 0;
  if (c.subgrid) {
    // the sub-grid model's terms (gas_funcs.cc:165-172, 192-200, 221-227, 236-238): analytic
    // photo-heating above Gamma = 3e-14, the gas taken as fully ionised
    const float tm = maxd(kTempMin, c.temp[q]);
    if (c.gamma_H1_tot[q] > 3e-14)
      c.heat_rate[q] = (float)photoheat_HIHeI(1.5, (double)tm, (double)(c.nH[q] + c.nHe[q]), (double)c.nH[q],
                                              (double)c.nHe[q]);
    else
      c.heat_rate[q] = 0.;
    c.cool_rate[q] += rcrB_H2(maxd(kTempMin, c.temp[q])) * (c.nH[q] + c.nHe[q]) * c.nH[q];
    c.cool_rate[q] += rcrB_He2(maxd(kTempMin, c.temp[q])) * (c.nH[q] + c.nHe[q]) * c.nHe[q];
    float nff = fion_of(c, q) * (c.nH[q] + c.nHe[q]);
    c.cool_rate[q] += free_free_rate(maxd(kTempMin, c.temp[q])) * pow(nff, 2.);
    c.cool_rate[q] -= compton_rate(c.zz) * (c.nH[q] + c.nHe[q]) * (2.726 * (1 + c.zz) - maxd(kTempMin, c.temp[q]));
    return;
  }
  if (c.f_H2[q] > 0.98) {
    for (int nu = 0; nu < F; nu++) {
      c.heat_rate[q] += c.avg_nh1[q] * c.gamma_H1_nu[q * F + nu] * O_H * (O_H_EV * c.nu[nu] - 13.6) / O_H_EV;
      c.heat_rate[q] += c.avg_nhe1[q] * c.gamma_He1_nu[q * F + nu] * O_H * (O_H_EV * c.nu[nu] - 2.459e+1) / O_H_EV;
    }
  } else {
    c.heat_rate[q] = 0.;
  }
  c.cool_rate[q] += rcrB_H2(maxd(kTempMin, c.temp[q])) * c.ne[q] * c.nH2[q];
  c.cool_rate[q] += rcrB_He2(maxd(kTempMin, c.temp[q])) * c.ne[q] * c.nHe2[q];
  float nff = c.nH2[q] + c.nHe2[q] + 4. * c.nHe3[q];
  c.cool_rate[q] += free_free_rate(maxd(kTempMin, c.temp[q])) * c.ne[q] * nff;
  c.cool_rate[q] -= compton_rate(c.zz) * c.ne[q] * (2.726 * (1 + c.zz) - maxd(kTempMin, c.temp[q]));
}

static float get_thermal_tstep(Ctx& c, long q) {
  float dT_dt = 2. / 3. / O_KB / c.n_tot[q] * (c.heat_rate[q] - c.cool_rate[q]) -
                (2. * hubble(1. / (1. + c.zz)) + c.dne_dt[q] / c.n_tot[q]) * c.temp[q];
  float min_dt = 0.1 * c.dt;
  return maxd(min_dt, mind(0.1 * c.temp[q] / absd(dT_dt), c.dt));
}

static void update_thermal(Ctx& c) {
  const long n3 = (long)c.N * c.N * c.N;
  for (long q = 0; q < n3; q++) {
    float t_temp = 0.;
    if (c.subgrid && !c.treion_flag[q]) {   // neutral until ionised (gas_funcs.cc:380-382)
      c.temp[q] = c.temp_0;
      continue;
    }
    if (!c.subgrid) set_Treion_default(c, q);
    while (t_temp < c.dt) {
      float dt_temp = mind(get_thermal_tstep(c, q), c.dt - t_temp);
      update_heat_cool(c, q);
      c.temp[q] = (c.temp[q] + 2. / 3. / O_KB / c.n_tot[q] * (c.heat_rate[q] - c.cool_rate[q]) * dt_temp) /
                  (1. + 2. * hubble(1. / (1. + c.zz)) * dt_temp + 1. / c.n_tot[q] * c.dne_dt[q] * dt_temp -
                   2. * c.ddelta_dt[q] / 3. / (c.rho[q] / c.avg_rho) * dt_temp);
      t_temp += dt_temp;
    }
    c.temp[q] = maxd(c.temp[q], kTempMin);
    if (!c.subgrid) c.nH1_prev[q] = c.nH1[q];
  }
}

// calc_vol_avg (data_funcs.cc:75-92): double sum in (i, j, k) order, float result
static float vol_avg(const Ctx& c, const std::vector<float>& f) {
  double tot = 0.;
  const long n3 = (long)c.N * c.N * c.N;
  for (long q = 0; q < n3; q++) tot += (double)f[q];
  return (float)tot / pow((double)c.N, 3.);
}

static void compact(Ctx& c) {
  size_t w = 0;
  for (size_t r = 0; r < c.rays.size(); ++r)
    if (c.rays[r].alive) c.rays[w++] = c.rays[r];
  c.rays.resize(w);
}

}  // namespace orc

using namespace orc;

extern "C" {

// Create a box from proper-density-free inputs: delta1 is 1+delta on N^3 (float32, C order),
// sources are pre-gridded (i,j,k,lum) in (i,j,k) order, clump may be NULL (C = const_clump).
void* orc_create(const Params* p, const float* delta1, int nsrc, const int32_t* src_ijk, const double* src_lum,
                 const float* clump) {
  Ctx* c = new Ctx();
  c->N = p->N;
  c->F = p->F;
  c->PL = p->path_length;
  c->itercount = p->itercount;
  c->ray_per_cell_max = p->ray_per_cell_max;
  c->hpx_lvl = p->hpx_lvl;
  c->l_max = 12;
  for (int nu = 0; nu < c->F; nu++) c->nu[nu] = p->nu_eV[nu] / O_H_EV;
  c->cl_factor = p->cl_factor;
  c->tstep_factor = 1.0f;
  c->nl_const = 0.5f;
  c->safety_factor = 3.f;
  c->const_clump = p->const_clump;
  c->zz = p->z;
  c->fH1_0 = 1. - 1.2e-3;
  c->fHe1_0 = 1. - 1.2e-3;
  c->fHe2_0 = 1.2e-3;
  c->temp_0 = 1e4;
  c->rkill = p->rkill_cm;
  c->Lx0 = p->box_hmpc * 1e3 / O_HH;
  c->dx0 = c->Lx0 / c->N * O_KPC_TO_CM;
  for (int nu = 0; nu < c->F; nu++) {
    c->sigH1[nu] = sig_H1(c->nu[nu]);
    c->sigHe1[nu] = sig_He1(c->nu[nu]);
  }
  srand(p->seed);
  c->seed = p->seed;
  alloc(*c);
  const long n3 = (long)c->N * c->N * c->N;
  // first-snapshot set-up at a = 1/(1+z) (gas_funcs.cc:595-613, io_funcs.cc:33-62)
  const float a_snap = (float)(1. / (1. + c->zz));
  c->Lx = c->Lx0 * a_snap;
  {
    float rho_c_cgs = 1.87890e-29, ob = 0.0482266, h0 = 0.68;
    double rho_unit = rho_c_cgs * ob * pow(h0, 2.);
    for (long q = 0; q < n3; q++) {
      c->rho[q] = delta1[q];
      c->rho[q] *= (float)rho_unit;
    }
    c->avg_rho = vol_avg(*c, c->rho);
    for (long q = 0; q < n3; q++) c->rho[q] *= pow(a_snap, -3.);
    c->avg_rho *= pow(a_snap, -3.);
  }
  for (int s = 0; s < nsrc; s++) c->src.push_back({src_ijk[3 * s], src_ijk[3 * s + 1], src_ijk[3 * s + 2], src_lum[s]});
  for (int i = 0; i < kNalpha; i++)
    for (int j = 0; j < kNalpha; j++)
      for (int k = 0; k < kNalpha; k++) {
        int ind = i * pow(kNalpha, 2) + j * kNalpha + k;
        c->random_angles[ind][0] = 2. * O_PI / kNalpha * i;
        c->random_angles[ind][1] = 2. * O_PI / kNalpha * j;
        c->random_angles[ind][2] = 2. * O_PI / kNalpha * k;
      }
  // init() (init_funcs.cc:10-142), input_grid = FALSE; fion is still 0 here
  c->dxc = c->Lx / c->N * O_KPC_TO_CM;
  for (long q = 0; q < n3; q++) {
    c->f_H1[q] = c->fH1_0;
    c->f_H2[q] = 1. - c->f_H1[q];
    c->f_He1[q] = c->fHe1_0;
    c->f_He2[q] = c->fHe2_0;
    c->f_He3[q] = 1. - c->f_He1[q] - c->f_He2[q];
    c->temp[q] = c->temp_0;
    c->nH[q] = (1. - O_Y) * c->rho[q] / O_MH;
    c->nHe[q] = O_Y * c->rho[q] / (4. * O_MH);
    c->nH2[q] = c->nH[q] * (1. - c->fH1_0);
    c->nHe2[q] = c->nHe[q] * (1. - c->fHe1_0);
    c->nHe3[q] = 0.;
    c->nH1[q] = c->nH[q] - c->nH2[q];
    c->avg_nh1[q] = c->nH1[q];
    c->nHe1[q] = c->nHe[q] - c->nHe2[q] - c->nHe3[q];
    c->avg_nhe1[q] = c->nHe1[q];
    c->ne[q] = c->nH2[q] + c->nHe2[q] + 2. * c->nHe3[q];
    c->n_tot[q] = c->nH[q] + c->nHe[q] + c->ne[q];
    c->nH1_prev[q] = c->nH1[q];
    c->recomb_H2[q] = alphaB_H2(c->temp[q]);
    c->recomb_He2[q] = alphaB_He2(c->temp[q]);
    c->recomb_He3[q] = alphaB_He3(c->temp[q]);
    c->treion[q] = 0.;
    c->treion_out[q] = 0.;
    c->mfp[q] = 1. / c->sigH1[0] / c->avg_nh1[q];
    c->mfp_912[q] = 1. / sig_H1(13.6 / O_H_EV) / c->avg_nh1[q];
    float dnH2_dt = c->gamma_H1_tot[q] * c->nH1[q] - c->recomb_H2[q] * c->ne[q] * c->nH2[q];
    float dnHe2_dt = c->nHe1[q] * c->gamma_He1_tot[q] - c->recomb_He2[q] * c->ne[q] * c->nHe2[q] +
                     c->recomb_He3[q] * c->ne[q] * c->nHe3[q] - c->nHe2[q] * 0.f;
    float dnHe3_dt = c->nHe2[q] * 0.f - c->recomb_He3[q] * c->ne[q] * c->nHe3[q];
    c->dne_dt[q] = dnH2_dt + dnHe2_dt + 2 * dnHe3_dt;
  }
  // update_dt (rt_funcs.cc:9-12)
  c->dt = c->tstep_factor * c->dxc / c->cl_factor / O_CL;
  set_spectrum(*c, *p);
  // init_rt (rt_funcs.cc:36-126): fion = 1 (ifront FALSE); ray_dt of source cells = dt
  for (const Src& S : c->src)
    if (S.lum != 0) c->ray_dt[cidx(*c, S.i, S.j, S.k)] = c->dt;
  c->have_clump = clump != nullptr;
  if (clump) {
    c->clump_in.assign(clump, clump + n3);
    c->clump = c->clump_in;  // the driver's set-up hook writes the field once before the loop
  }
  c->total_rays = 0;
  c->t = 0.;
  c->nphot_merge = 0.;
  c->step = 0;
  c->led_emitted = c->led_deposited = c->led_killed = c->led_overlap = 0.;
  new_rays(*c);
  // get_nphot_min_max (ray_tracing.cc:129-154)
  {
    int counter = 0;
    c->nphot_base_avg = 0.;
    for (const Src& S : c->src) {
      if (S.lum > 0.) {
        double tmp = 0.;
        for (int nu = 0; nu < c->F; nu++)
          tmp += c->spectrum[nu] * S.lum * c->dt / 12. / pow(2., 2. * c->hpx_lvl) / kPhotNorm;
        c->nphot_base_avg += (double)log10(tmp);
        counter += 1;
      }
    }
    c->nphot_base_avg /= counter;
    c->nphot_base_avg = pow(10., c->nphot_base_avg);
    c->nphot_max = 1e3 * c->nphot_base_avg;
    c->nphot_min = 1e-10 * c->nphot_base_avg;
  }
  c->last_crossings = 0;
  c->last_moved = 0;
  return c;
}

// One RT step in the order of main.cc:108-264 (plain mode, fixed redshift).
void orc_step(void* h) {
  Ctx& c = *(Ctx*)h;
  c.step += 1;
  c.led_emitted = c.led_deposited = c.led_killed = c.led_overlap = 0.;
  c.step_dt = c.dt;
  const long n3 = (long)c.N * c.N * c.N;
  for (long q = 0; q < n3; q++) c.clump[q] = c.const_clump;
  if (c.have_clump) c.clump = c.clump_in;
  c.clight = c.cl_factor * O_CL;
  c.nc = c.nl_const;
  c.t += c.dt;
  if (c.subgrid) sg_delta_dom(c, maxd(c.sg_t12, c.t + c.sg_tinit));   // main.cc:126-128
  update_rays(c);
  c.last_crossings = 0;
  c.last_moved = 0;
  for (const Ray& R : c.rays)
    if (R.alive && !R.active) {
      c.last_crossings += R.ray_end;
      c.last_moved += 1;
    }
  if (c.rkill > 0.0)
    for (Ray& R : c.rays)
      if (R.alive && (double)R.r > c.rkill) {
        c.led_killed += (double)sum_nphot(c, R) * kPhotNorm;
        R.alive = false;
        R.active = false;
      }
  find_avg_unu(c);
  c.num_thresh = 0;
  for (long q = 0; q < n3; q++) c.num_thresh += (long)(c.ray_per_cell_max - 12 * pow(2, 2 * c.hpx_lvl));
  long count = count_rays(c);
  if (count > c.num_thresh) calc_nphot_merge(c);
  merge(c);
  compact(c);
  split_rays(c);
  compact(c);
  update_thermal(c);
  new_rays(c);
  c.dt = c.tstep_factor * c.dxc / c.cl_factor / O_CL;
}

long orc_num_rays(void* h) { return count_rays(*(Ctx*)h); }
long orc_last_crossings(void* h) { return ((Ctx*)h)->last_crossings; }

void orc_scalars(void* h, double* out16) {
  Ctx& c = *(Ctx*)h;
  double sc[16] = {(double)c.t, (double)c.dt, c.nphot_min, c.nphot_max, (double)c.nphot_merge, (double)c.num_thresh,
                   (double)c.total_rays, (double)c.dx0, (double)c.dxc, (double)c.step, (double)c.last_crossings,
                   (double)c.last_moved, c.nphot_base_avg, 0.0, (double)c.src.size(), 1.0};
  memcpy(out16, sc, sizeof sc);
}

int orc_dump(void* h, const char* path) {
  Ctx& c = *(Ctx*)h;
  struct frtd_writer w;
  if (frtd_open(&w, path) != 0) return -1;
  const int64_t n3 = (int64_t)c.N * c.N * c.N;
  const int64_t nf[2] = {n3, c.F};
#define DF(name) frtd_add1(&w, #name, FRTD_F32, n3, c.name.data())
#define DFN(name) frtd_add(&w, #name, FRTD_F32, 2, nf, c.name.data())
  DF(rho); DF(nH); DF(nHe); DF(nH1); DF(nHe1); DF(nH2); DF(nHe2); DF(nHe3); DF(ne); DF(n_tot);
  DF(f_H1); DF(f_He1); DF(f_H2); DF(f_He2); DF(f_He3); DF(temp); DF(clump); DF(avg_nh1); DF(avg_nhe1);
  DF(gamma_H1_tot); DF(gamma_He1_tot); DF(heat_rate); DF(cool_rate); DF(recomb_H2); DF(recomb_He2);
  DF(recomb_He3); DF(recrate_H2); DF(recrate_He2); DF(dne_dt); DF(mfp); DF(mfp_912); DF(treion);
  DF(treion_out); DF(IF_speed); DF(Inc_Flux); DF(avg_gamma); DF(avg_gamma_he1); DF(nH1_prev);
  DFN(gamma_H1_nu); DFN(gamma_He1_nu); DFN(ngam_nu); DFN(u_nu); DFN(avg_gamma_nu); DFN(avg_gamma_nu_he1);
#undef DF
#undef DFN
  frtd_add1(&w, "treion_flag", FRTD_U8, n3, c.treion_flag.data());
  if (c.ifront) {
    frtd_add1(&w, "fion", FRTD_F32, n3, c.fion.data());
    frtd_add1(&w, "fion_max", FRTD_F32, n3, c.fion_max.data());
    frtd_add1(&w, "tcross", FRTD_F32, n3, c.tcross.data());
    frtd_add1(&w, "Delta_fion", FRTD_F32, n3, c.Delta_fion.data());
    const int64_t nt[2] = {n3, kNtcross};
    frtd_add(&w, "tcross_new", FRTD_F32, 2, nt, c.tcross_new.data());
    frtd_add1(&w, "tcross_flag", FRTD_U8, n3, c.tcross_flag.data());
    frtd_add1(&w, "neutral_flag", FRTD_U8, n3, c.neutral_flag.data());
  }
  double sc[16];
  orc_scalars(h, sc);
  frtd_add1(&w, "scalars", FRTD_F64, 16, sc);
  {
    // photon ledger of the last step: emitted, deposited, killed, overlap, in flight
    double in_flight = 0.;
    for (const Ray& R : c.rays)
      if (R.alive)
        for (int nu = 0; nu < c.F; nu++) in_flight += (double)R.nphot[nu] * kPhotNorm;
    const double led[5] = {c.led_emitted, c.led_deposited, c.led_killed, c.led_overlap, in_flight};
    frtd_add1(&w, "ledger", FRTD_F64, 5, led);
  }
  frtd_add1(&w, "spectrum", FRTD_F32, c.F, c.spectrum);
  std::vector<const Ray*> live;
  for (const Ray& R : c.rays)
    if (R.alive) live.push_back(&R);
  const int64_t nr = (int64_t)live.size();
  std::vector<int64_t> slot(nr);
  std::vector<uint8_t> act(nr);
  std::vector<int16_t> ord(nr), rend(nr);
  std::vector<int32_t> pix(nr), cell(nr);
  std::vector<uint16_t> ith(nr);
  std::vector<float> g9(nr * 9), np(nr * c.F);
  for (int64_t q = 0; q < nr; ++q) {
    const Ray& R = *live[q];
    slot[q] = q;
    act[q] = R.active;
    ord[q] = R.order;
    pix[q] = R.pixel;
    ith[q] = R.itheta;
    cell[q] = R.pind[0];
    rend[q] = R.ray_end;
    const float v[9] = {R.xhat, R.yhat, R.zhat, R.r, R.dr, R.x, R.y, R.z, R.time};
    for (int k = 0; k < 9; ++k) g9[q * 9 + k] = v[k];
    for (int nu = 0; nu < c.F; ++nu) np[q * c.F + nu] = R.nphot[nu];
  }
  frtd_add1(&w, "ray_slot", FRTD_I64, nr, slot.data());
  frtd_add1(&w, "ray_active", FRTD_U8, nr, act.data());
  frtd_add1(&w, "ray_order", FRTD_I16, nr, ord.data());
  frtd_add1(&w, "ray_pixel", FRTD_I32, nr, pix.data());
  frtd_add1(&w, "ray_itheta", FRTD_U16, nr, ith.data());
  frtd_add1(&w, "ray_cell", FRTD_I32, nr, cell.data());
  frtd_add1(&w, "ray_end", FRTD_I16, nr, rend.data());
  const int64_t d9[2] = {nr, 9};
  frtd_add(&w, "ray_geom", FRTD_F32, 2, d9, g9.data());
  const int64_t dnf[2] = {nr, c.F};
  frtd_add(&w, "ray_nphot", FRTD_F32, 2, dnf, np.data());
  if (c.tau_max > 0.) {
    std::vector<double> col(nr * 2);
    for (int64_t q = 0; q < nr; ++q) {
      col[q * 2] = live[q]->colH;
      col[q * 2 + 1] = live[q]->colHe;
    }
    const int64_t d2[2] = {nr, 2};
    frtd_add(&w, "ray_col", FRTD_F64, 2, d2, col.data());
    std::vector<double> sig(2 * c.F);
    for (int nu = 0; nu < c.F; nu++) {
      sig[nu] = c.sigH1[nu];
      sig[c.F + nu] = c.sigHe1[nu];
    }
    const int64_t ds[2] = {2, c.F};
    frtd_add(&w, "tau_sigma", FRTD_F64, 2, ds, sig.data());
    frtd_add1(&w, "tau_max", FRTD_F64, 1, &c.tau_max);
  }
  frtd_close(&w);
  return 0;
}

void orc_destroy(void* h) { delete (Ctx*)h; }

// The opt-in optical-depth limit (no counterpart in the reference): from the next step on, a ray
// whose optical depth since its cast exceeds tau_max in every frequency bin is removed like a ray
// below nphot_min; 0 turns it off.
void orc_set_tau_limit(void* h, double tau_max) { ((Ctx*)h)->tau_max = tau_max; }

}  // extern "C"

// ---- cosmological expansion between steps (gas_funcs.cc:460-548) ------------------------------
extern "C" void orc_cosmo_expansion(void* h, float a_current, float a_prev) {
  Ctx& c = *(Ctx*)h;
  const long n3 = (long)c.N * c.N * c.N;
  c.Lx *= a_current / a_prev;
  c.dxc *= a_current / a_prev;
  const float fion = 1.f;   // plain mode (rt_funcs.cc:55)
  for (long q = 0; q < n3; q++) {
    c.rho[q] *= pow(a_prev / a_current, 3.);
    c.nH[q] = (1. - O_Y) * c.rho[q] / O_MH;
    c.nHe[q] = O_Y * c.rho[q] / (4. * O_MH);
    c.nH2[q] = c.f_H2[q] * c.nH[q] / fion;
    c.nHe2[q] = c.f_He2[q] * c.nHe[q] / fion;
    c.nHe3[q] = c.f_He3[q] * c.nHe[q] / fion;
    c.nH1[q] = c.nH[q] - c.nH2[q];
    c.avg_nh1[q] = c.nH1[q];
    c.nHe1[q] = c.nHe[q] - c.nHe2[q] - c.nHe3[q];
    c.avg_nhe1[q] = c.nHe1[q];
    c.ne[q] = c.nH2[q] + c.nHe2[q] + 2. * c.nHe3[q];
    c.n_tot[q] = c.nH[q] + c.nHe[q] + c.ne[q];
    c.nH1_prev[q] = c.nH1[q];
  }
  c.avg_rho *= pow(a_prev / a_current, 3.);
  const float dxc = c.dxc;
  for (Ray& R : c.rays) {
    if (!R.alive) continue;
    R.x *= a_current / a_prev;
    R.y *= a_current / a_prev;
    R.z *= a_current / a_prev;
    if (R.x <= 0.) R.x = kMinDist * dxc;
    if (R.x >= dxc * (1. - kMinDist / 2.)) R.x = dxc * (1. - kMinDist);
    if (R.y <= 0.) R.y = kMinDist * dxc;
    if (R.y >= dxc * (1. - kMinDist / 2.)) R.y = dxc * (1. - kMinDist);
    if (R.z <= 0.) R.z = kMinDist * dxc;
    if (R.z >= dxc * (1. - kMinDist / 2.)) R.z = dxc * (1. - kMinDist);
  }
  c.dt = c.tstep_factor * c.dxc / c.cl_factor / O_CL;   // update_dt (main.cc:237)
}

// update_hydro_step for a later snapshot (gas_funcs.cc:554-752; the branch zz != zinit with a
// next snapshot to come), then get_nphot_min_max and update_dt (main.cc:221-237): delta1 is the
// new 1+delta cube as get_ugas reads it, the sources are gridded (i, j, k, lum) as
// read_source_catalog leaves them (io_funcs.cc:157-233), a_rt the scale factor at the current
// time, dt_snap = cosmic_time(a_next) - cosmic_time(a) of the snapshots, zz the new redshift.
extern "C" void orc_hydro_step(void* h, const float* delta1, int nsrc, const int32_t* src_ijk, const double* src_lum,
                               float a_rt, float dt_snap, float zz_new) {
  Ctx& c = *(Ctx*)h;
  const long n3 = (long)c.N * c.N * c.N;
  c.zz = zz_new;
  c.Lx = c.Lx0 * a_rt;
  // get_ugas (io_funcs.cc:33-62) and the a^-3 of update_hydro_step (gas_funcs.cc:669-684)
  {
    float rho_c_cgs = 1.87890e-29, ob = 0.0482266, h0 = 0.68;
    double rho_unit = rho_c_cgs * ob * pow(h0, 2.);
    for (long q = 0; q < n3; q++) {
      c.rho[q] = delta1[q];
      c.rho[q] *= (float)rho_unit;
    }
    c.avg_rho = vol_avg(c, c.rho);
    for (long q = 0; q < n3; q++) c.rho[q] *= pow(a_rt, -3.);
    c.avg_rho *= pow(a_rt, -3.);
  }
  // read_source_catalog: the new sources; every ray_dt back to 0
  c.src.clear();
  for (int s = 0; s < nsrc; s++) c.src.push_back({src_ijk[3 * s], src_ijk[3 * s + 1], src_ijk[3 * s + 2], src_lum[s]});
  for (long q = 0; q < n3; q++) c.ray_dt[q] = 0.;
  const float avg_rho_prev = vol_avg(c, c.rho_prev);
  c.dxc = c.Lx / c.N * O_KPC_TO_CM;
  const float fion = 1.f;   // plain mode (rt_funcs.cc:55)
  for (long q = 0; q < n3; q++) {
    c.nH[q] = (1. - O_Y) * c.rho[q] / O_MH;
    c.nHe[q] = O_Y * c.rho[q] / (4. * O_MH);
    c.nH2[q] = c.f_H2[q] * c.nH[q] / fion;
    c.nHe2[q] = c.f_He2[q] * c.nHe[q] / fion;
    c.nHe3[q] = c.f_He3[q] * c.nHe[q] / fion;
    c.nH1[q] = c.nH[q] - c.nH2[q];
    c.avg_nh1[q] = c.nH1[q];
    c.nHe1[q] = c.nHe[q] - c.nHe2[q] - c.nHe3[q];
    c.avg_nhe1[q] = c.nHe1[q];
    c.ne[q] = c.nH2[q] + c.nHe2[q] + 2. * c.nHe3[q];
    c.n_tot[q] = c.nH[q] + c.nHe[q] + c.ne[q];
    if (avg_rho_prev > 0.) c.ddelta_dt[q] = (c.rho[q] / c.avg_rho - c.rho_prev[q] / avg_rho_prev) / dt_snap;
    c.rho_prev[q] = c.rho[q];
    c.nH1_prev[q] = c.nH1[q];
  }
  // get_nphot_min_max (ray_tracing.cc:129-154) with the new sources and the time step of the
  // step just taken (update_dt follows it, main.cc:237)
  {
    int counter = 0;
    c.nphot_base_avg = 0.;
    for (const Src& S : c.src) {
      if (S.lum > 0.) {
        double tmp = 0.;
        for (int nu = 0; nu < c.F; nu++)
          tmp += c.spectrum[nu] * S.lum * c.step_dt / 12. / pow(2., 2. * c.hpx_lvl) / kPhotNorm;
        c.nphot_base_avg += (double)log10(tmp);
        counter += 1;
      }
    }
    c.nphot_base_avg /= counter;
    c.nphot_base_avg = pow(10., c.nphot_base_avg);
    c.nphot_max = 1e3 * c.nphot_base_avg;
    c.nphot_min = 1e-10 * c.nphot_base_avg;
  }
  c.dt = c.tstep_factor * c.dxc / c.cl_factor / O_CL;   // update_dt (main.cc:237)
}

// The sub-grid model (subgrid = TRUE, equilibrium = TRUE, ifront = FALSE), set up after the cast
// as main.cc:86-90 does: time_tab and fh1_tab are the reference's time_RH and fh1_RH arrays
// ([Nt][3][3][3] floats, filled at the gamma index q + 1, Nt*27 + 1 floats with the last row's
// spill; times in s), t_dnl / ds / dnl the linear -> non-linear overdensity table (500, 500,
// 500 x 500 floats), consts = {tinit, cosmic_time(z=12), cosmic_time(z=8), cosmic_time(z=5.5),
// tre_dom[0..2]} as the reference's cosmic_time gives them.
extern "C" void orc_set_subgrid(void* h, const float* time_tab, const float* fh1_tab, const float* t_dnl, const float* ds,
                                const float* dnl, const float* consts, int ifront) {
  Ctx& c = *(Ctx*)h;
  const size_t n3 = (size_t)c.N * c.N * c.N;
  c.ifront = ifront != 0;
  if (c.ifront) {   // init_rt with ifront = TRUE (rt_funcs.cc:49-69)
    c.fion.assign(n3, 0.f);
    c.fion_max.assign(n3, 0.f);
    c.tcross.assign(n3, 0.f);
    c.Delta_fion.assign(n3, 0.f);
    c.tcross_new.assign(n3 * kNtcross, 0.f);
    c.tcross_check.assign(n3 * kNtcross, 0);
    c.tcross_flag.assign(n3, 0);
    c.neutral_flag.assign(n3, 1);
    c.ngam3.assign(n3 * 3, 0.);
  }
  const size_t nrh = (size_t)kNt * 27 + 1;
  c.subgrid = true;
  c.sg_time.assign(time_tab, time_tab + nrh);
  c.sg_fh1.assign(fh1_tab, fh1_tab + nrh);
  c.sg_t_dnl.assign(t_dnl, t_dnl + kNdlin);
  c.sg_ds.assign(ds, ds + kNdlin);
  c.sg_dnl.assign(dnl, dnl + (size_t)kNdlin * kNdlin);
  c.sg_tinit = consts[0];
  c.sg_t12 = consts[1];
  c.sg_t8 = consts[2];
  c.sg_tcap = consts[3];
  for (int i = 0; i < 3; i++) c.sg_tre_dom[i] = consts[4 + i];
  c.sg_fh1_interp.assign((size_t)c.N * c.N * c.N * 5, 0.f);
}

// ---- restart files in the reference's formats -------------------------------------------------
// write_gas_binary (io_funcs.cc:358-393), write_rays_binary (274-303), write_treion (338-355):
// fields written one after another with ofstream::write, so the records are packed. In plain mode
// fion = 1 and tcross = 0 everywhere (rt_funcs.cc:49-58) and neutral_flag keeps its initial TRUE
// (it only changes in the sub-grid branch, ray_tracing.cc:1010).
namespace {

struct ByteOut {
  unsigned char* p;
  size_t n, cap;
  template <typename T> void put(const T& v) {
    if (p && n + sizeof(T) <= cap) memcpy(p + n, &v, sizeof(T));
    n += sizeof(T);
  }
};

struct ByteIn {
  const unsigned char* p;
  size_t n, size;
  bool ok = true;
  template <typename T> T get() {
    T v{};
    if (n + sizeof(T) <= size) memcpy(&v, p + n, sizeof(T));
    else ok = false;
    n += sizeof(T);
    return v;
  }
};

}  // namespace

extern "C" {

size_t orc_write_gas(void* h, void* buf, size_t cap) {
  Ctx& c = *(Ctx*)h;
  ByteOut o{(unsigned char*)buf, 0, cap};
  const long n3 = (long)c.N * c.N * c.N;
  o.put<float>(c.t);
  for (long q = 0; q < n3; q++) {
    o.put<float>(c.rho[q]); o.put<float>(c.temp[q]); o.put<float>(c.nH1[q]); o.put<float>(c.f_H1[q]);
    o.put<float>(c.f_He1[q]); o.put<float>(c.f_H2[q]); o.put<float>(c.f_He2[q]); o.put<float>(c.f_He3[q]);
    o.put<float>(c.gamma_H1_tot[q]); o.put<float>(c.gamma_He1_tot[q]); o.put<float>(c.mfp[q]);
    o.put<float>(c.mfp_912[q]); o.put<float>(c.heat_rate[q]); o.put<float>(c.cool_rate[q]); o.put<float>(c.avg_nh1[q]);
    o.put<float>(1.f);              // fion
    o.put<float>(0.f);              // tcross
    o.put<float>(c.treion_out[q]);
    for (int nu = 0; nu < c.F; nu++) o.put<float>(c.ngam_nu[q * c.F + nu]);
  }
  return o.n;
}

size_t orc_write_rays(void* h, void* buf, size_t cap) {
  Ctx& c = *(Ctx*)h;
  ByteOut o{(unsigned char*)buf, 0, cap};
  long x = 0;
  for (const Ray& R : c.rays) {
    if (!R.alive) continue;
    o.put<long>(x++);
    o.put<bool>(R.active);
    o.put<short>(R.order);
    o.put<int>(R.pixel);
    o.put<unsigned short>(R.itheta);
    o.put<float>(R.xhat); o.put<float>(R.yhat); o.put<float>(R.zhat);
    for (int nu = 0; nu < c.F; nu++) o.put<float>(R.nphot[nu]);
    o.put<float>(R.r); o.put<float>(R.dr); o.put<float>(R.x); o.put<float>(R.y); o.put<float>(R.z); o.put<float>(R.time);
    o.put<int>(R.pind[0]);
  }
  o.put<long>(-1);
  return o.n;
}

size_t orc_write_treion(void* h, void* buf, size_t cap) {
  Ctx& c = *(Ctx*)h;
  ByteOut o{(unsigned char*)buf, 0, cap};
  const long n3 = (long)c.N * c.N * c.N;
  for (long q = 0; q < n3; q++) {
    o.put<float>(c.treion[q]);
    o.put<bool>(c.treion_flag[q] != 0);
    o.put<bool>(false);   // tcross_flag
    o.put<bool>(true);    // neutral_flag
  }
  return o.n;
}

// Restart from the three files: read_grid_binary + read_treion (io_funcs.cc:65-116) and init()
// with input_grid = TRUE (init_funcs.cc:10-19, 62-138), then init_rt's restart branch: ray_dt = 0
// at the sources, read_rays_binary (rt_funcs.cc:95-107, io_funcs.cc:119-146), and the free-slot
// probe of rt_funcs.cc:117-124: select_index(0) hands out slot 0 and a ray there whose first-bin
// photon count is 0 is removed (for one processor: the record with slot number 0). The restarted
// run draws from a fresh srand(seed) (no set-up cast precedes it). Replaces the set-up state of a
// box made by orc_create (same grid, sources and seed). Returns 0 on success.
int orc_read_restart(void* h, const void* gas, size_t gas_size, const void* tre, size_t tre_size, const void* rays,
                     size_t ray_size) {
  Ctx& c = *(Ctx*)h;
  const long n3 = (long)c.N * c.N * c.N;
  std::vector<float> fion(n3);
  {
    ByteIn in{(const unsigned char*)gas, 0, gas_size};
    c.t = in.get<float>();
    for (long q = 0; q < n3; q++) {
      c.rho[q] = in.get<float>(); c.temp[q] = in.get<float>(); c.nH1[q] = in.get<float>(); c.f_H1[q] = in.get<float>();
      c.f_He1[q] = in.get<float>(); c.f_H2[q] = in.get<float>(); c.f_He2[q] = in.get<float>();
      c.f_He3[q] = in.get<float>(); c.gamma_H1_tot[q] = in.get<float>(); c.gamma_He1_tot[q] = in.get<float>();
      c.mfp[q] = in.get<float>(); c.mfp_912[q] = in.get<float>(); c.heat_rate[q] = in.get<float>();
      c.cool_rate[q] = in.get<float>(); c.avg_nh1[q] = in.get<float>(); fion[q] = in.get<float>();
      (void)in.get<float>();   // tcross
      c.treion_out[q] = in.get<float>();
      for (int nu = 0; nu < c.F; nu++) c.ngam_nu[q * c.F + nu] = in.get<float>();
    }
    if (!in.ok || in.n != gas_size) return 1;
  }
  {
    ByteIn in{(const unsigned char*)tre, 0, tre_size};
    for (long q = 0; q < n3; q++) {
      c.treion[q] = in.get<float>();
      c.treion_flag[q] = in.get<bool>() ? 1 : 0;
      (void)in.get<bool>();
      (void)in.get<bool>();
    }
    if (!in.ok || in.n != tre_size) return 2;
  }
  for (long q = 0; q < n3; q++) {
    c.nH[q] = (1. - O_Y) * c.rho[q] / O_MH;
    c.nHe[q] = O_Y * c.rho[q] / (4. * O_MH);
    if (fion[q] > 0.) {
      c.nH2[q] = c.f_H2[q] * c.nH[q] / fion[q];
      c.nHe2[q] = c.f_He2[q] * c.nHe[q] / fion[q];
      c.nHe3[q] = c.f_He3[q] * c.nHe[q] / fion[q];
    } else {
      c.nH2[q] = c.nH[q] * (1. - c.fH1_0);
      c.nHe2[q] = c.nHe[q] * (1. - c.fHe1_0);
      c.nHe3[q] = 0.;
    }
    c.nH1[q] = c.nH[q] - c.nH2[q];
    c.avg_nh1[q] = c.nH1[q];
    c.nHe1[q] = c.nHe[q] - c.nHe2[q] - c.nHe3[q];
    c.avg_nhe1[q] = c.nHe1[q];
    c.ne[q] = c.nH2[q] + c.nHe2[q] + 2. * c.nHe3[q];
    c.n_tot[q] = c.nH[q] + c.nHe[q] + c.ne[q];
    c.IF_speed[q] = 0.;
    c.Inc_Flux[q] = 0.;
    c.nH1_prev[q] = c.nH1[q];
    c.recomb_H2[q] = alphaB_H2(c.temp[q]);
    c.recomb_He2[q] = alphaB_He2(c.temp[q]);
    c.recomb_He3[q] = alphaB_He3(c.temp[q]);
    c.avg_gamma[q] = c.gamma_H1_tot[q];
    c.avg_gamma_he1[q] = c.gamma_He1_tot[q];
    float dnH2_dt = c.gamma_H1_tot[q] * c.nH1[q] - c.recomb_H2[q] * c.ne[q] * c.nH2[q];
    float dnHe2_dt = c.nHe1[q] * c.gamma_He1_tot[q] - c.recomb_He2[q] * c.ne[q] * c.nHe2[q] +
                     c.recomb_He3[q] * c.ne[q] * c.nHe3[q] - c.nHe2[q] * 0.f;
    float dnHe3_dt = c.nHe2[q] * 0.f - c.recomb_He3[q] * c.ne[q] * c.nHe3[q];
    c.dne_dt[q] = dnH2_dt + dnHe2_dt + 2 * dnHe3_dt;
  }
  for (const Src& S : c.src) c.ray_dt[cidx(c, S.i, S.j, S.k)] = 0.f;
  srand(c.seed);
  c.rays.clear();
  {
    ByteIn in{(const unsigned char*)rays, 0, ray_size};
    long x = in.get<long>();
    while (in.ok && x != -1) {
      Ray R;
      memset(&R, 0, sizeof R);
      R.alive = true;
      R.active = in.get<bool>();
      R.order = in.get<short>();
      R.pixel = in.get<int>();
      R.itheta = in.get<unsigned short>();
      R.xhat = in.get<float>(); R.yhat = in.get<float>(); R.zhat = in.get<float>();
      for (int nu = 0; nu < c.F; nu++) R.nphot[nu] = in.get<float>();
      R.r = in.get<float>(); R.dr = in.get<float>(); R.x = in.get<float>(); R.y = in.get<float>();
      R.z = in.get<float>(); R.time = in.get<float>();
      R.pind[0] = in.get<int>();
      R.src = -1;   // the restart records do not say which source cast a ray
      if (in.ok && !(x == 0 && R.nphot[0] == 0.)) c.rays.push_back(R);
      x = in.get<long>();
    }
    if (!in.ok) return 3;
  }
  return 0;
}

}  // extern "C"

// ---- FP64 objective of one step and its tangent-linear form (checks of the adjoint) -------------
// The objective J = sum of Gamma_HI over a sub-box after the C2Ray iteration of the next step
// (ray pass ray_tracing.cc:701-938, cell update 1077-1113, Gamma total 1152), as a function of
// per-source luminosity factors lam_s and per-cell density factors s_c. A factor s_c scales the
// cell's n_H together with everything init() derives from the same density (n_He, n_HI, n_HeI;
// init_funcs.cc:34-62); ionised fractions, temperatures and recombination coefficients stay
// fixed. Rays take the photon counts of their set-up cast scaled by lam of their source, and the
// segments of the next advance (advance_ray above). The kill threshold nphot_min stays at its
// set-up value. Evaluated in double throughout (no float storage of the iterates), generic over
// the scalar type so that the same code gives the value (double) and the directional derivative
// (Dual: value and tangent, forward-mode differentiation).
namespace {

struct Dual {
  double v, d;
};
inline Dual mk(double v, double d = 0.) { return Dual{v, d}; }
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dual exp(Dual a) {
  const double e = std::exp(a.v);
  return {e, e * a.d};
}
inline double val(Dual a) { return a.v; }
inline double val(double a) { return a; }
template <typename S> S cst(double v) { return S(v); }
template <> Dual cst<Dual>(double v) { return mk(v); }
inline double expx(double a) { return std::exp(a); }
inline Dual expx(Dual a) { return exp(a); }

struct AdjRay {
  int src;
  int nseg;
  long cell[kMaxPL];
  double dist[kMaxPL];
  double n0[kMaxF];
};

struct AdjProblem {
  std::vector<AdjRay> rays;
  std::vector<long> lit;                         // lit cells (global index)
  std::unordered_map<long, int> slot;            // cell -> lit slot
  std::vector<char> in_obj;                      // per lit slot: inside the objective sub-box
};

AdjProblem adj_setup(Ctx& c, const int* lo, const int* hi) {
  AdjProblem P;
  c.clight = c.cl_factor * O_CL;
  c.nc = c.nl_const;
  for (const Ray& R0 : c.rays) {
    if (!R0.alive) continue;
    Ray R = R0;
    const long cell0 = R.pind[0];
    advance_ray(c, R);
    if (R.active) continue;   // did not leave its cell: no segments this step
    if (c.rkill > 0.0 && (double)R.r > c.rkill) continue;
    AdjRay A;
    A.src = R0.src;   // the source that cast the ray (a ray merged from several sources: -1)
    (void)cell0;
    A.nseg = R.ray_end;
    for (int p = 0; p < R.ray_end; ++p) {
      A.cell[p] = R.pind[p];
      A.dist[p] = R.pdist[p];
      if (!P.slot.count(R.pind[p])) {
        P.slot[R.pind[p]] = (int)P.lit.size();
        P.lit.push_back(R.pind[p]);
      }
    }
    for (int nu = 0; nu < c.F; ++nu) A.n0[nu] = (double)R0.nphot[nu] * kPhotNorm;
    P.rays.push_back(A);
  }
  P.in_obj.resize(P.lit.size());
  for (size_t j = 0; j < P.lit.size(); ++j) {
    int i, jj, k;
    split_ind(c, (int)P.lit[j], &i, &jj, &k);
    P.in_obj[j] = i >= lo[0] && i < hi[0] && jj >= lo[1] && jj < hi[1] && k >= lo[2] && k < hi[2];
  }
  return P;
}

template <typename S>
S adj_objective(const Ctx& c, const AdjProblem& P, const std::vector<S>& lam, const std::vector<S>& sc) {
  const int F = c.F, I = c.itercount;
  const size_t L = P.lit.size();
  const double dt = c.dt, vol = (double)c.dxc * (double)c.dxc * (double)c.dxc;
  std::vector<S> nH(L), nHe(L), a(L), b(L), gh(L), ghe(L);
  std::vector<double> y0h(L), y0he(L), crh(L), crhe(L);
  for (size_t j = 0; j < L; ++j) {
    const long q = P.lit[j];
    nH[j] = cst<S>((double)c.nH[q]) * sc[j];
    nHe[j] = cst<S>((double)c.nHe[q]) * sc[j];
    a[j] = cst<S>((double)c.nH1[q]) * sc[j];
    b[j] = cst<S>((double)c.nHe1[q]) * sc[j];
    y0h[j] = c.f_H1[q];
    y0he[j] = c.f_He1[q];
    const float cl = c.have_clump ? c.clump_in[q] : c.const_clump;
    crh[j] = (double)(cl * (float)alphaB_H2(maxd(kTempMin, c.temp[q])));
    float rhe = (float)alphaB_He2(maxd(kTempMin, c.temp[q]));
    if ((c.temp[q] >= 3e4) && (c.temp[q] <= 1e6)) rhe += (float)Dalpha_He2(maxd(kTempMin, c.temp[q]));
    crhe[j] = (double)(cl * rhe);
  }
  S J = cst<S>(0.);
  for (int it = 0; it < I; ++it) {
    for (size_t j = 0; j < L; ++j) { gh[j] = cst<S>(0.); ghe[j] = cst<S>(0.); }
    for (const AdjRay& R : P.rays) {
      S nin[kMaxF];
      for (int nu = 0; nu < F; ++nu) nin[nu] = cst<S>(R.n0[nu]) * (R.src >= 0 ? lam[R.src] : cst<S>(1.));
      for (int p = 0; p < R.nseg; ++p) {
        const int j = P.slot.at(R.cell[p]);
        double tot = 0.;
        for (int nu = 0; nu < F; ++nu) tot += val(nin[nu]) / kPhotNorm;
        const bool dump = tot < c.nphot_min;
        S tr[kMaxF];
        for (int nu = 0; nu < F; ++nu) {
          const S x = a[j] * cst<S>(c.sigH1[nu] * R.dist[p]);
          const S y = b[j] * cst<S>(c.sigHe1[nu] * R.dist[p]);
          const S ex = expx(-x), ey = expx(-y);
          S fh = cst<S>(0.), fhe = cst<S>(0.);
          if (val(x) > 0. || val(y) > 0.) {
            const S x1 = (cst<S>(1.) - ex) * ey, x2 = (cst<S>(1.) - ey) * ex;
            fh = x1 / (x1 + x2);
            fhe = x2 / (x1 + x2);
          }
          const S absb = dump ? cst<S>(1.) : cst<S>(1.) - ex * ey;
          gh[j] = gh[j] + fh * nin[nu] * absb / cst<S>(dt * vol) / a[j];
          ghe[j] = ghe[j] + fhe * nin[nu] * absb / cst<S>(dt * vol) / b[j];
          tr[nu] = ex * ey;
        }
        if (dump) break;
        for (int nu = 0; nu < F; ++nu) nin[nu] = nin[nu] * tr[nu];
      }
    }
    if (it == I - 1) {
      for (size_t j = 0; j < L; ++j)
        if (P.in_obj[j]) J = J + gh[j];
      break;
    }
    for (size_t j = 0; j < L; ++j) {   // C2Ray update of the lit cells (dark cells never enter J)
      const S ne = nH[j] - a[j] + nHe[j] - b[j];
      const S prh = gh[j] + cst<S>(crh[j]) * ne;
      const S xeq = gh[j] / prh;
      const S a_new = nH[j] * (cst<S>(1.) - (xeq + (cst<S>(1. - y0h[j]) - xeq) * (cst<S>(1.) - expx(-cst<S>(dt) * prh)) /
                                                     (cst<S>(dt) * prh)));
      const S prhe = ghe[j] + cst<S>(crhe[j]) * ne;
      const S xeqhe = ghe[j] / prhe;
      const S b_new = nHe[j] * (cst<S>(1.) - (xeqhe + (cst<S>(1. - y0he[j]) - xeqhe) *
                                                           (cst<S>(1.) - expx(-cst<S>(dt) * prhe)) / (cst<S>(dt) * prhe)));
      a[j] = a_new;
      b[j] = b_new;
    }
  }
  return J;
}

}  // namespace

extern "C" {

// J and, with tangent directions (dlam per source, dsc per cell; NULL = 0), its directional
// derivative. lam / sc are the factors (NULL = all 1); sc and dsc are dense per cell (N^3).
double orc_adj_objective(void* h, const int* lo, const int* hi, const double* lam, const double* sc,
                         const double* dlam, const double* dsc, double* jvp, long* nlit) {
  Ctx& c = *(Ctx*)h;
  AdjProblem P = adj_setup(c, lo, hi);
  if (nlit) *nlit = (long)P.lit.size();
  const size_t ns = c.src.size(), L = P.lit.size();
  if (!dlam && !dsc) {
    std::vector<double> l(ns, 1.), s(L, 1.);
    if (lam) for (size_t i = 0; i < ns; ++i) l[i] = lam[i];
    if (sc) for (size_t j = 0; j < L; ++j) s[j] = sc[P.lit[j]];
    if (jvp) *jvp = 0.;
    return adj_objective<double>(c, P, l, s);
  }
  std::vector<Dual> l(ns), s(L);
  for (size_t i = 0; i < ns; ++i) l[i] = mk(lam ? lam[i] : 1., dlam ? dlam[i] : 0.);
  for (size_t j = 0; j < L; ++j) s[j] = mk(sc ? sc[P.lit[j]] : 1., dsc ? dsc[P.lit[j]] : 0.);
  const Dual J = adj_objective<Dual>(c, P, l, s);
  if (jvp) *jvp = J.d;
  return J.v;
}


// rotation of healpix_funcs.cc:102-143 with the angles of get_random_angles (healpix_funcs.cc:21-39)
void orc_rotate(int itheta, int direction, const double* v, double* out) {
  const int i = itheta / (kNalpha * kNalpha), j = (itheta / kNalpha) % kNalpha, k = itheta % kNalpha;
  float a0 = 2. * O_PI / kNalpha * i, b0 = 2. * O_PI / kNalpha * j, g0 = 2. * O_PI / kNalpha * k;
  rotate(a0, b0, g0, direction, v[0], v[1], v[2], &out[0], &out[1], &out[2]);
}
void orc_pix2vec(int order, int pix, double* v) { hpn::pix2vec(order, pix, &v[0], &v[1], &v[2]); }
int orc_vec2pix(int order, const double* v) { return hpn::vec2pix(order, v[0], v[1], v[2]); }

}  // extern "C"
