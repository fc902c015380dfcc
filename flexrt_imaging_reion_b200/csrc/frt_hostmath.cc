// Host-side set-up arithmetic of an RT context, compiled by g++ with -ffp-contract=off so that
// every float/double expression rounds exactly as in the reference's own g++ build:
//  * the rotation-coefficient table (get_random_angles + get_unit_vector, healpix_funcs.cc:21-39,
//    102-143): the reference multiplies float cosf/sinf values inline for every ray; here each
//    coefficient is formed once per angle triple with the same float expression;
//  * per-box geometry and time-step constants (global_variables.cc:69, init_funcs.cc:22-30,
//    rt_funcs.cc:9-12, 129-143, ray_tracing.cc:66-95, 1362-1417);
//  * the first-snapshot gas set-up (io_funcs.cc:33-62, gas_funcs.cc:601-610, init_funcs.cc:10-142);
//  * the photon thresholds (get_nphot_min_max, ray_tracing.cc:129-154).
#include "frt_hostmath.h"

#include <math.h>

#include <cmath>

using namespace std;

namespace frt {
namespace host {

namespace {
constexpr double kPiRef = 3.14159;        // global_constants.h: #define pi 3.14159
constexpr double kKpcToCm = 3.086e21;
constexpr double kCl = 2.998e10;
constexpr double kHh = 0.68;
constexpr double kMpcToKm = 3.086e19;
constexpr double kOmegaM = 0.305147;
constexpr double kOmegaL = 0.6948;
constexpr double kY = 0.246;
constexpr double kMH = 1.672622e-24;
constexpr double kHPlanck = 6.626068e-27;
constexpr double kHeV = 4.135667e-15;
constexpr float kMinDist = 1e-4f;
constexpr int kNalpha = 35;

double lam(double T, double Eth) {
  double K2eV = 1.38065e-16 / 1.60218e-12;
  double eV2K = 1.0 / K2eV;
  return 2 * Eth * eV2K / T;
}
double alphaB_H2(double T) {
  double x = lam(T, 13.6);
  return 2.753e-14 * pow(x, 1.500) / pow((1.0 + pow((x / 2.740), 0.407)), 2.2420);
}
double alphaB_He2(double T) {
  double x = lam(T, 2.459e+1);
  return 1.26e-14 * pow(x, 0.750);
}
double alphaB_He3(double T) {   // rates.cc:161-165
  double x = lam(T, 5.442e+1);
  return 2 * 2.753e-14 * pow(x, 1.500) / pow((1.0 + pow((x / 2.740), 0.407)), 2.2420);
}
float hubble(float a) { return kHh * 100. / kMpcToKm * pow(kOmegaM / pow(a, 3.) + kOmegaL, 0.5); }
}  // namespace

void rotation_table(float* out) {
  for (int i = 0; i < kNalpha; i++)
    for (int j = 0; j < kNalpha; j++)
      for (int k = 0; k < kNalpha; k++) {
        const int ind = i * pow(kNalpha, 2) + j * kNalpha + k;
        const float a0 = 2. * kPiRef / kNalpha * i;
        const float b0 = 2. * kPiRef / kNalpha * j;
        const float g0 = 2. * kPiRef / kNalpha * k;
        float* m = out + (size_t)ind * 18;
        // direction 0 (forward)
        m[0] = (cos(b0) * cos(g0));
        m[1] = (-cos(b0) * sin(g0));
        m[2] = (sin(b0));
        m[3] = (sin(a0) * sin(b0) * cos(g0) + cos(a0) * sin(g0));
        m[4] = (-sin(a0) * sin(b0) * sin(g0) + cos(a0) * cos(g0));
        m[5] = (-sin(a0) * cos(b0));
        m[6] = (-cos(a0) * sin(b0) * cos(g0) + sin(a0) * sin(g0));
        m[7] = (cos(a0) * sin(b0) * sin(g0) + sin(a0) * cos(g0));
        m[8] = (cos(a0) * cos(b0));
        // direction 6 (inverse)
        m[9] = (cos(g0) * cos(b0));
        m[10] = (sin(g0) * cos(a0) + cos(g0) * sin(b0) * sin(a0));
        m[11] = (sin(g0) * sin(a0) - cos(g0) * sin(b0) * cos(a0));
        m[12] = (-sin(g0) * cos(b0));
        m[13] = (cos(g0) * cos(a0) - sin(g0) * sin(b0) * sin(a0));
        m[14] = (cos(g0) * sin(a0) + sin(g0) * sin(b0) * cos(a0));
        m[15] = (sin(b0));
        m[16] = (-cos(b0) * sin(a0));
        m[17] = (cos(b0) * cos(a0));
      }
}

// The smallest float >= v. For a float x, (double)x >= v <=> x >= float_at_or_above(v) and
// (double)x < v <=> x < float_at_or_above(v), so the device compares in float.
static float float_at_or_above(double v) {
  float f = (float)v;
  if ((double)f < v) f = std::nextafter(f, INFINITY);
  return f;
}

void set_cell_size(BoxP* B, const frt_config* cfg, const frt_box_desc* bd, float dx) {
  B->dx = dx;
  B->scale = dx / B->dx0;                                            // ray_tracing.cc:1262
  B->dx_half = dx / 2.;                                              // ray_tracing.cc:308
  B->lo_edge = kMinDist * dx;                                        // ray_tracing.cc:1366
  B->hi_edge = dx * (1. - kMinDist);                                 // ray_tracing.cc:1370
  B->hi_thr = dx * (1. - kMinDist / 2.);                             // ray_tracing.cc:1403
  B->hi_thr_f = float_at_or_above(B->hi_thr);
  const float nc = B->nc;
  B->mv_hi = nc * dx;                                                // ray_tracing.cc:1252
  B->mv_lo = (1. - nc) * dx;                                         // ray_tracing.cc:1253
  B->mv_lo_f = float_at_or_above(B->mv_lo);
  B->dt = cfg->tstep_factor * dx / bd->cl_factor / kCl;              // rt_funcs.cc:11
  B->vol = ((double)dx) * ((double)dx) * ((double)dx);               // ray_tracing.cc:747
  B->kdep = 1e60 / (double)B->dt / B->vol;
  B->kdep_f = (float)B->kdep;
  B->th.dt = B->dt;
  B->th.dx = dx;
}

void box_params(BoxP* B, const frt_config* cfg, const frt_box_desc* bd, long long cell0) {
  const int n = bd->n;
  B->n = n;
  B->nn = n * n;
  B->inv_n = 1.0 / n;
  B->inv_nn = 1.0 / ((double)n * n);
  B->cell0 = cell0;
  B->ncell = (long long)n * n * n;
  const float Lx0 = bd->box_hmpc * 1e3 / kHh;                        // user_inputs.h:92
  const float dx0 = Lx0 / n * kKpcToCm;                              // global_variables.cc:69
  const float a_snap = (float)(1. / (1. + bd->zz));
  const float Lx = Lx0 * a_snap;                                     // gas_funcs.cc:595
  const float dx = Lx / n * kKpcToCm;                                // init_funcs.cc:23
  B->dx0 = dx0;
  B->nc = cfg->nl_const;                                             // rt_funcs.cc:138
  B->clight = bd->cl_factor * kCl;                                   // rt_funcs.cc:137
  set_cell_size(B, cfg, bd, dx);
  B->t = 0.f;
  B->rkill = bd->rkill_cm;
  B->nphot_min = 0.;
  B->nphot_max = 0.;
  B->nphot_merge = 0.f;
  B->split_thr = 0.f;
  B->lm = cfg->hpx_lvl;
  B->lsource = cfg->hpx_lvl;
  // num_thresh = sum over cells of (ray_per_cell - 12*4^l_merge) (ray_tracing.cc:157-170)
  B->num_thresh = (long long)(bd->ray_per_cell_max - 12 * pow(2, 2 * cfg->hpx_lvl)) * B->ncell;
  for (int l = 0; l < kLtab; l++) {
    float rmax = dx0 * pow(2, l) * pow(3. / kPiRef / cfg->safety_factor, 0.5);        // ray_tracing.cc:76-79
    float rmin = dx0 * pow(2, l - 1) * pow(3. / kPiRef / cfg->safety_factor, 0.5);    // ray_tracing.cc:66-73
    if (l == 0) rmin = 0.;
    B->rmax[l] = rmax;
    B->rmin[l] = rmin;
  }
  ThermConst& th = B->th;
  th.dt = B->dt;
  th.dx = dx;
  set_redshift(B, bd->zz);
  th.nfreq = (float)cfg->nfreq;
  for (int nu = 0; nu < 8; nu++) {
    const double f = nu < cfg->nfreq ? cfg->nu_phot[nu] : 0.0;
    th.nu[nu] = f;
    th.cH1[nu] = (float)(kHPlanck * (kHeV * f - 13.6) / kHeV);      // gas_funcs.cc:155-156
    th.cHe1[nu] = (float)(kHPlanck * (kHeV * f - 2.459e+1) / kHeV);
  }
}

float snapshot_dx(const frt_box_desc* bd, float a) {
  const float Lx0 = bd->box_hmpc * 1e3 / kHh;                        // user_inputs.h:92
  const float Lx = Lx0 * a;                                          // gas_funcs.cc:590
  return Lx / bd->n * kKpcToCm;                                      // gas_funcs.cc:689
}

void set_redshift(BoxP* B, float zz) {
  ThermConst& th = B->th;
  const float Hf = hubble(1. / (1. + zz));                           // gas_funcs.cc:356, 405
  th.hub2f = 2.0f * Hf;
  th.hub_d = Hf;
  th.zz = zz;
  th.compton_d = 5.6072e-36 * pow(1 + (double)zz, 4.);               // rates.cc:234-238
  th.compton_f = (float)th.compton_d;
}

float vol_avg(const float* f, int n) {
  double tot = 0.;
  const long long n3 = (long long)n * n * n;
  for (long long q = 0; q < n3; q++) tot += (double)f[q];
  return (float)tot / pow((double)n, 3.);
}

void snapshot_rho(int n, const float* delta1, float a, float* rho, float* avg_rho) {
  const long long n3 = (long long)n * n * n;
  const float rho_c_cgs = 1.87890e-29, ob = 0.0482266, h0 = 0.68;
  const double rho_unit = rho_c_cgs * ob * pow(h0, 2.);
  for (long long q = 0; q < n3; q++) {
    rho[q] = delta1[q];
    rho[q] *= (float)rho_unit;
  }
  float avg = vol_avg(rho, n);
  for (long long q = 0; q < n3; q++) rho[q] *= pow(a, -3.);
  avg *= pow(a, -3.);
  *avg_rho = avg;
}

void init_gas(const frt_config* cfg, const frt_box_desc* bd, const float* delta1, GasInit* g) {
  const long long n3 = (long long)bd->n * bd->n * bd->n;
  const float a_snap = (float)(1. / (1. + bd->zz));
  // get_ugas (io_funcs.cc:33-62): rho = file * (float) rho_unit; then rho *= a^-3 (gas_funcs.cc:606)
  const float rho_c_cgs = 1.87890e-29, ob = 0.0482266, h0 = 0.68;
  const double rho_unit = rho_c_cgs * ob * pow(h0, 2.);
  const float fH1_0 = cfg->fH1_0, fHe1_0 = cfg->fHe1_0, fHe2_0 = cfg->fHe2_0, temp_0 = cfg->temp_0;
  for (long long q = 0; q < n3; q++) {
    float rho = delta1[q];
    rho *= (float)rho_unit;
    rho *= pow(a_snap, -3.);
    g->rho[q] = rho;
    // init() (init_funcs.cc:34-137), input_grid = FALSE, fion = 0 at this point
    const float f_H1 = fH1_0;
    const float f_He1 = fHe1_0;
    const float nH = (1. - kY) * rho / kMH;
    const float nHe = kY * rho / (4. * kMH);
    const float nH2 = nH * (1. - fH1_0);
    const float nHe2 = nHe * (1. - fHe1_0);
    const float nHe3 = 0.;
    const float nH1 = nH - nH2;
    const float nHe1 = nHe - nHe2 - nHe3;
    const float ne = nH2 + nHe2 + 2. * nHe3;
    g->nH[q] = nH;
    g->nHe[q] = nHe;
    g->nH1[q] = nH1;
    g->nHe1[q] = nHe1;
    g->f_H1[q] = f_H1;
    g->f_He1[q] = f_He1;
    g->temp[q] = temp_0;
    g->ne[q] = ne;
    g->n_tot[q] = nH + nHe + ne;
    const float rec_h2 = alphaB_H2(temp_0);
    const float rec_he2 = alphaB_He2(temp_0);
    g->rec_h2[q] = rec_h2;
    g->rec_he2[q] = rec_he2;
    // initial electron-density derivative with zero photo-ionisation rates (init_funcs.cc:132-136)
    const float dnH2_dt = 0.f * nH1 - rec_h2 * ne * nH2;
    const float dnHe2_dt = nHe1 * 0.f - rec_he2 * ne * nHe2 + 0.f * ne * nHe3 - nHe2 * 0.f;
    const float dnHe3_dt = nHe2 * 0.f - 0.f * ne * nHe3;
    (void)fHe2_0;
    g->dne_dt[q] = dnH2_dt + dnHe2_dt + 2 * dnHe3_dt;
  }
}

void init_gas_restart(const frt_config* cfg, const frt_box_desc* bd, const GasRestart& r, GasInit* g, float* heat,
                      float* cool) {
  const long long n3 = (long long)bd->n * bd->n * bd->n;
  const float fH1_0 = cfg->fH1_0, fHe1_0 = cfg->fHe1_0;
  for (long long q = 0; q < n3; q++) {
    // read_grid_binary order (io_funcs.cc:87-108): rho temp nH1 f_H1 f_He1 f_H2 f_He2 f_He3
    // gamma_H1_tot gamma_He1_tot mfp mfp_912 heat cool avg_nh1 fion tcross treion_out ngam_nu[]
    const float* v = r.rec + (size_t)q * r.stride;
    const float rho = v[0], temp = v[1], f_H1 = v[3], f_He1 = v[4], f_H2 = v[5], f_He2 = v[6], f_He3 = v[7];
    const float g_h1 = v[8], g_he1 = v[9], fion = v[15];
    g->rho[q] = rho;
    // init() with input_grid = TRUE (init_funcs.cc:62-137)
    const float nH = (1. - kY) * rho / kMH;
    const float nHe = kY * rho / (4. * kMH);
    float nH2, nHe2, nHe3;
    if (fion > 0.) {
      nH2 = f_H2 * nH / fion;
      nHe2 = f_He2 * nHe / fion;
      nHe3 = f_He3 * nHe / fion;
    } else {
      nH2 = nH * (1. - fH1_0);
      nHe2 = nHe * (1. - fHe1_0);
      nHe3 = 0.;
    }
    const float nH1 = nH - nH2;
    const float nHe1 = nHe - nHe2 - nHe3;
    const float ne = nH2 + nHe2 + 2. * nHe3;
    g->nH[q] = nH;
    g->nHe[q] = nHe;
    g->nH1[q] = nH1;
    g->nHe1[q] = nHe1;
    g->f_H1[q] = f_H1;
    g->f_He1[q] = f_He1;
    g->temp[q] = temp;
    g->ne[q] = ne;
    g->n_tot[q] = nH + nHe + ne;
    const float rec_h2 = alphaB_H2(temp);
    const float rec_he2 = alphaB_He2(temp);
    const float rec_he3 = alphaB_He3(temp);
    g->rec_h2[q] = rec_h2;
    g->rec_he2[q] = rec_he2;
    const float dnH2_dt = g_h1 * nH1 - rec_h2 * ne * nH2;
    const float dnHe2_dt = nHe1 * g_he1 - rec_he2 * ne * nHe2 + rec_he3 * ne * nHe3 - nHe2 * 0.f;
    const float dnHe3_dt = nHe2 * 0.f - rec_he3 * ne * nHe3;
    g->dne_dt[q] = dnH2_dt + dnHe2_dt + 2 * dnHe3_dt;
    heat[q] = v[12];
    cool[q] = v[13];
  }
}

void nphot_min_max(const frt_config* cfg, const BoxP* B, int nsrc, const double* lum, double* nmin, double* nmax) {
  int counter = 0;
  double avg = 0.;
  for (int s = 0; s < nsrc; s++) {
    if (lum[s] > 0.) {
      double tmp = 0.;
      for (int nu = 0; nu < cfg->nfreq; nu++)
        tmp += cfg->spectrum[nu] * lum[s] * B->dt / 12. / pow(2., 2. * cfg->hpx_lvl) / 1e60;
      avg += (double)log10(tmp);
      counter += 1;
    }
  }
  avg /= counter;
  avg = pow(10., avg);
  *nmax = 1e3 * avg;
  *nmin = 1e-10 * avg;
}

void derived_constants(const frt_config* cfg, double* sigH1, double* sigHe1, double* sig0, double* sig912,
                       double* pi_sf_3, double* log4) {
  auto verner = [](double nu, double Eth, double Emax, double E0, double y0, double y1, double yw, double ya,
                   double P) -> double {
    double E = kHeV * nu;
    double x = E / E0 - y0;
    double y = pow(pow(x, 2) + pow(y1, 2), 0.5);
    double F = (pow(x - 1, 2) + pow(yw, 2)) * pow(y, 0.5 * P - 5.5) * pow(1 + pow(y / ya, 0.5), -P);
    if (kHeV * nu >= Eth && kHeV * nu <= Emax) return F;
    return 0;
  };
  auto sH1 = [&](double nu) { return 5.475e-14 * verner(nu, 13.6, 5e4, 4.298e-1, 0, 0, 0, 3.288e+1, 2.963); };
  auto sHe1 = [&](double nu) {
    return 9.492e-16 * verner(nu, 2.459e+1, 5e4, 1.361e+1, 4.434e-1, 2.136, 2.039, 1.469, 3.188);
  };
  for (int nu = 0; nu < cfg->nfreq; nu++) {
    sigH1[nu] = sH1(cfg->nu_phot[nu]);
    sigHe1[nu] = sHe1(cfg->nu_phot[nu]);
  }
  *sig0 = sH1(cfg->nu_phot[0]);
  *sig912 = sH1(13.6 / kHeV);
  *pi_sf_3 = kPiRef * cfg->safety_factor / 3.;
  *log4 = log(4.);
}

}  // namespace host
}  // namespace frt
