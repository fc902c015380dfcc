// Per-cell physics of the RT step for sm_100a: the C2Ray time-averaged ionisation update
// (ray_tracing.cc:1077-1209), case-B recombination / cooling rates (rates.cc:125-238) and the
// sub-cycled implicit temperature update (gas_funcs.cc:104-242, 353-457).
//
// Two precision policies, selected at compile time:
//  * STRICT = true : the reference's own expressions, with the same float/double split
//    (float storage, double locals), evaluated in double on the device. Differences to the
//    reference come only from CUDA vs glibc transcendental rounding and accumulation order.
//  * STRICT = false (mixed, the default): FP32 arithmetic, with the C2Ray solve in FP64 for
//    cells whose neutral fraction is below 1e-3. The C2Ray average is evaluated in the
//    neutral-fraction form y_avg = y_eq + (y0 - y_eq)(1 - e^-r)/r, r = dt (Gamma + C alpha n_e),
//    which is algebraically the reference's 1 - (x_eq + t_i/dt (x0 - x_eq)(1 - e^-dt/t_i)) but
//    free of the 1 - x cancellation, so FP32 keeps relative accuracy in ionised cells too.
#pragma once
#include <math.h>
#include <stdint.h>

#include "frt_params.h"

namespace frt {

// constants as the reference defines them (global_constants.h, rates.cc:5-39,
// global_variables.cc:85, 302-305)
constexpr double kH = 6.626068e-27;
constexpr double kHeV = 4.135667e-15;
constexpr double kKB = 1.38065e-16;
constexpr double kCL = 2.998e10;
constexpr double kEvCgs = 1.60218e-12;
constexpr double kY = 0.246;
constexpr double kMH = 1.672622e-24;
constexpr double kPhotNorm = 1e60;
constexpr double kEthH1 = 13.6;
constexpr double kEthHe1 = 2.459e+1;
constexpr double kEthHe2 = 5.442e+1;
constexpr float kTempMin = 1e2f;
constexpr float kMinDist = 1e-4f;

// x = lambda(T, Eth) = 2 Eth eV2K / T (rates.cc:41-48)
__host__ __device__ inline double lam_d(double T, double Eth) {
  const double K2eV = kKB / kEvCgs;
  const double eV2K = 1.0 / K2eV;
  return 2 * Eth * eV2K / T;
}
// 2 Eth eV2K for the float path
constexpr float kLamH1 = (float)(2 * kEthH1 * (1.0 / (kKB / kEvCgs)));
constexpr float kLamHe1 = (float)(2 * kEthHe1 * (1.0 / (kKB / kEvCgs)));
constexpr float kLamHe2 = (float)(2 * kEthHe2 * (1.0 / (kKB / kEvCgs)));

// ---- Hui & Gnedin 1997 rates, double (reference form) ----------------------------------
__device__ inline double alphaB_H2_d(double T) {
  double x = lam_d(T, kEthH1);
  return 2.753e-14 * pow(x, 1.500) / pow((1.0 + pow((x / 2.740), 0.407)), 2.2420);
}
__device__ inline double alphaB_He2_d(double T) {
  double x = lam_d(T, kEthHe1);
  return 1.26e-14 * pow(x, 0.750);
}
__device__ inline double Dalpha_He2_d(double T) {
  double x = lam_d(T, kEthHe2);
  return 1.90e-3 * pow(T, -1.5) * exp(-0.75 * x / 2) * (1 + 0.3 * exp(-0.15 * x / 2));
}
__device__ inline double rcrB_H2_d(double T) {
  double x = lam_d(T, kEthH1);
  return 3.435e-30 * T * pow(x, 1.970) / (pow(1. + pow(x / 2.250, 0.376), 3.720));
}
__device__ inline double rcrB_He2_d(double T) { return kKB * T * alphaB_He2_d(T); }
__device__ inline double free_free_d(double T) { return 1.42e-27 * pow(T, 0.5) * 1.30; }

// ---- the same rates in FP32 -------------------------------------------------------------
// x = lambda(T) = 2 Eth eV2K / T enters every rate as a power law, so each rate is evaluated
// from lT = log2(T) as exp2 of a linear combination of log2 x = log2(2 Eth eV2K) - lT.
// log2(2 Eth eV2K) for Eth = 13.6 / 24.59 / 54.42 eV, and log2 of the break points 2.74, 2.25:
constexpr float kLog2LamH1 = 18.26793572782709f;
constexpr float kLog2LamHe1 = 19.122400811285473f;
constexpr float kLog2_274 = 1.4541758931858022f;
constexpr float kLog2_225 = 1.1699250014423124f;

__device__ __forceinline__ float alphaB_H2_lt(float lT) {     // rates.cc:135-138
  const float L = kLog2LamH1 - lT;
  const float q = exp2f(0.407f * (L - kLog2_274));
  return 2.753e-14f * exp2f(1.5f * L - 2.2420f * log2f(1.0f + q));
}
__device__ __forceinline__ float alphaB_He2_lt(float lT) {    // rates.cc:147-151
  return 1.26e-14f * exp2f(0.750f * (kLog2LamHe1 - lT));
}
__device__ __forceinline__ float rcrB_H2_lt(float T, float lT) {   // rates.cc:183-187
  const float L = kLog2LamH1 - lT;
  const float q = exp2f(0.376f * (L - kLog2_225));
  return 3.435e-30f * T * exp2f(1.970f * L - 3.720f * log2f(1.0f + q));
}
__device__ inline float Dalpha_He2_f(float T) {               // rates.cc:168-171
  const float x = kLamHe2 / T;
  return 1.90e-3f * __fdividef(1.0f, T * sqrtf(T)) * expf(-0.375f * x) * (1.0f + 0.3f * expf(-0.075f * x));
}
__device__ __forceinline__ float free_free_f(float T) { return (float)(1.42e-27 * 1.30) * sqrtf(T); }

// Recombination coefficients of one cell at the start of a step (ray_tracing.cc:655-674).
template <bool STRICT>
__device__ inline void recomb_coeffs(float temp, float* rec_h2, float* rec_he2) {
  const float tm = (temp >= kTempMin) ? temp : kTempMin;   // maxd(temp_min, temp)
  if (STRICT) {
    *rec_h2 = (float)alphaB_H2_d(tm);
    float he2 = (float)alphaB_He2_d(tm);
    if ((temp >= 3e4) && (temp <= 1e6)) he2 += (float)Dalpha_He2_d(tm);
    *rec_he2 = he2;
  } else {
    const float lT = log2f(tm);
    *rec_h2 = alphaB_H2_lt(lT);
    float he2 = alphaB_He2_lt(lT);
    if ((temp >= 3e4f) && (temp <= 1e6f)) he2 += Dalpha_He2_f(tm);
    *rec_he2 = he2;
  }
}

// Constants of one C2Ray species update in a cell.
struct C2Species {
  float n;       // nH or nHe
  float y0;      // neutral fraction at the start of the step (f_H1 / f_He1)
  float crec;    // clump * recomb (float product, as the reference forms it)
};

// One C2Ray update of one species (ray_tracing.cc:1084-1113 and, on the last iteration,
// 1116-1127). Returns the time-averaged neutral density; *n_end receives the end-of-step
// neutral density when last is true.
// ZERO_GAMMA: the caller knows gamma = 0 (a cell no ray touched); x_eq = 0 and y_eq = rec/rec = 1
// exactly, which the general form also yields, so both paths give the same bits.
template <bool STRICT, bool ZERO_GAMMA = false>
__device__ inline float c2ray_species(const C2Species& s, float gamma, double nelec_d, float nelec_f, float avg_prev,
                                      float dt, bool last, float* n_end) {
  if (STRICT) {
    const double x0 = (double)(1. - s.y0);
    const double pr = (double)gamma + 0.0 + s.crec * nelec_d;
    const double xeq = ((double)gamma + 0.0) / pr;
    const double ti = 1. / pr;
    const float avg = (float)(s.n * (1. - (xeq + ti / dt * (x0 - xeq) * (1. - exp(-dt / ti)))));
    if (last) *n_end = (float)s.n * (1. - (xeq + (x0 - xeq) * exp(-dt / ti)));
    return avg;
  }
  const float rec = s.crec * nelec_f;
  const float pr = gamma + rec;
  if (!(pr > 0.0f)) {  // no electrons and no photo-ionisation: the state is frozen
    if (last) *n_end = s.n * s.y0;
    return s.n * s.y0;
  }
  const bool fp64 = (s.y0 < 1e-3f) || (avg_prev < 1e-3f * s.n);
  if (fp64) {
    const double prd = (double)gamma + (double)s.crec * nelec_d;
    const double yeq = ZERO_GAMMA ? 1.0 : ((double)s.crec * nelec_d) / prd;
    const double r = (double)dt * prd;
    const double em = -expm1(-r);  // 1 - e^-r
    const double yavg = yeq + ((double)s.y0 - yeq) * (em / r);
    if (last) *n_end = (float)((double)s.n * (yeq + ((double)s.y0 - yeq) * (1.0 - em)));
    return (float)((double)s.n * yavg);
  }
  const float yeq = ZERO_GAMMA ? 1.0f : rec / pr;   // exact division: 1 when gamma = 0
  const float r = dt * pr;
  float em_r, ex;   // (1 - e^-r)/r and e^-r
  if (r < 1e-2f) {
    // Taylor series, truncation error below r^4/120 < 1e-10: the usual case of a cell that is
    // only recombining (r = dt C alpha n_e is ~1e-6 .. 1e-3)
    em_r = 1.0f - r * (0.5f - r * ((1.0f / 6.0f) - r * (1.0f / 24.0f)));
    ex = 1.0f - r * (1.0f - r * (0.5f - r * ((1.0f / 6.0f) - r * (1.0f / 24.0f))));
  } else {
    const float em = -expm1f(-r);
    em_r = __fdividef(em, r);
    ex = 1.0f - em;
  }
  const float yavg = yeq + (s.y0 - yeq) * em_r;
  if (last) *n_end = s.n * (yeq + (s.y0 - yeq) * ex);
  return s.n * yavg;
}

// State of one cell for the thermal update (after the last C2Ray iteration).
struct ThermCell {
  float temp, heat, cool;
  float nH, nH1, nH1_prev, nH2, nHe2, ne, n_tot, dne_dt, f_H2, avg_nh1, avg_nhe1;
  float if_speed, inc_flux;
  // d(delta)/dt and rho / <rho> of the temperature equation (gas_funcs.cc:399); 0 and 1 until a
  // second hydro snapshot gives the density a rate of change
  float ddelta = 0.f, rho_rel = 1.f;
};

// Photo-ionisation input of the heating term. The reference sums over bins
// avg_nh1 gamma_H1_nu h (h_eV nu - Eth)/h_eV (gas_funcs.cc:155-158); that needs either the
// per-bin rates of the cell (mode 1) or, equivalently, their bin-weighted sums
// sum_nu gamma_nu c_nu accumulated by the last ray pass (mode 2). Mode 0: no deposit.
struct HeatSrc {
  const float* g_h1;
  const float* g_he1;
  int stride;
  float hh, hhe;
  int mode;
};

// update_heat_cool (gas_funcs.cc:134-242) for subgrid = FALSE, case B, recombination /
// free-free / Compton cooling on, collisional terms off.
template <bool STRICT>
__device__ inline void heat_cool(ThermCell& c, const ThermConst& k, const HeatSrc& hs, int nfreq) {
  const float* g_h1 = hs.mode == 1 ? hs.g_h1 : nullptr;
  const float* g_he1 = hs.g_he1;
  const int gstride = hs.stride;
  const float tm = (c.temp >= kTempMin) ? c.temp : kTempMin;   // maxd(temp_min, temp)
  if (STRICT) {
    float heat = 0;
    float cool = 0;
    if (c.f_H2 > 0.98) {
      if (g_h1) {
        for (int nu = 0; nu < nfreq; nu++) {
          heat += c.avg_nh1 * g_h1[nu * gstride] * kH * (kHeV * k.nu[nu] - kEthH1) / kHeV;
          heat += c.avg_nhe1 * g_he1[nu * gstride] * kH * (kHeV * k.nu[nu] - kEthHe1) / kHeV;
        }
      } else {
        for (int nu = 0; nu < nfreq; nu++) {
          heat += c.avg_nh1 * 0.0f * kH * (kHeV * k.nu[nu] - kEthH1) / kHeV;
          heat += c.avg_nhe1 * 0.0f * kH * (kHeV * k.nu[nu] - kEthHe1) / kHeV;
        }
      }
    } else {
      heat = 0.;
    }
    cool += rcrB_H2_d(tm) * c.ne * c.nH2;
    cool += rcrB_He2_d(tm) * c.ne * c.nHe2;
    const float nff = c.nH2 + c.nHe2 + 4. * 0.0f;
    cool += free_free_d(tm) * c.ne * nff;
    cool -= k.compton_d * c.ne * (2.726 * (1 + k.zz) - tm);
    c.heat = heat;
    c.cool = cool;
    return;
  }
  float heat = 0.0f;
  if (c.f_H2 > 0.98) {   // double comparison, as the reference (gas_funcs.cc:148)
    if (g_h1) {
      for (int nu = 0; nu < nfreq; nu++) {
        heat += (c.avg_nh1 * g_h1[nu * gstride]) * k.cH1[nu];
        heat += (c.avg_nhe1 * g_he1[nu * gstride]) * k.cHe1[nu];
      }
    } else if (hs.mode == 2) {
      heat = c.avg_nh1 * hs.hh + c.avg_nhe1 * hs.hhe;
    }
  }
  const float lT = log2f(tm);
  const float nenh2 = c.ne * c.nH2;
  const float nenhe2 = c.ne * c.nHe2;
  float cool = rcrB_H2_lt(tm, lT) * nenh2;
  cool += ((float)kKB * tm * alphaB_He2_lt(lT)) * nenhe2;
  cool += free_free_f(tm) * (c.ne * (c.nH2 + c.nHe2));
  cool -= (k.compton_f * (2.726f * (1.0f + k.zz) - tm)) * c.ne;
  c.heat = heat;
  c.cool = cool;
}

template <bool STRICT>
__device__ inline float thermal_tstep(const ThermCell& c, const ThermConst& k) {
  if (STRICT) {
    const float dT_dt = 2. / 3. / kKB / c.n_tot * (c.heat - c.cool) - (2. * (double)(k.hub2f * 0.5f) + c.dne_dt / c.n_tot) * c.temp;
    const float min_dt = 0.1 * k.dt;
    const float adt = (dT_dt >= 0.) ? dT_dt : (float)(-1. * dT_dt);
    const float cand = (float)(0.1 * c.temp / adt);
    const float m1 = (cand >= k.dt) ? k.dt : cand;
    return (m1 >= min_dt) ? m1 : min_dt;
  }
  const float c23 = (float)(2. / 3. / kKB);
  const float inv_n = __fdividef(1.0f, c.n_tot);
  const float dT_dt = (c23 * inv_n) * (c.heat - c.cool) - (k.hub2f + c.dne_dt * inv_n) * c.temp;
  const float min_dt = 0.1f * k.dt;
  const float cand = __fdividef(0.1f * c.temp, fabsf(dT_dt));
  const float m1 = (cand >= k.dt) ? k.dt : cand;
  return (m1 >= min_dt) ? m1 : min_dt;
}

// set_Treion_default (gas_funcs.cc:104-129): post-I-front temperature, I-front speed and flux.
template <bool STRICT>
__device__ inline void treion_default(ThermCell& c, const ThermConst& k, float nhe_to_nh) {
  float fion_new, fion_old, vIF;
  if (STRICT) {
    fion_new = (c.nH - c.nH1) / c.nH;
    fion_old = (c.nH - c.nH1_prev) / c.nH;
    vIF = k.dx * (fion_new - fion_old) / k.dt;
  } else {
    const float inv_nh = __fdividef(1.0f, c.nH);
    fion_new = (c.nH - c.nH1) * inv_nh;
    fion_old = (c.nH - c.nH1_prev) * inv_nh;
    vIF = __fdividef(k.dx * (fion_new - fion_old), k.dt);
  }
  if ((fion_new > fion_old) && (fion_new < 0.98)) {
    const float Cn[5] = {9.5432f, -1.6441e-2f, -9.8010e-3f, 4.1664e-3f, -2.2710e-4f};
    float lnT = 0.f;
    if (STRICT) {
      const double L = log(vIF / 1e5);
      for (int t = 0; t < 5; t++) lnT += Cn[t] * pow(L, (double)t);
    } else {
      const float L = logf(vIF * 1e-5f);
      float Lp = 1.0f;
      for (int t = 0; t < 5; t++) {
        lnT += Cn[t] * Lp;
        Lp *= L;
      }
    }
    c.temp = (fion_old * c.temp + (fion_new - fion_old) * expf(lnT)) / fion_new;
  }
  const float v0 = (vIF >= 0.f) ? vIF : 0.f;   // maxd(0., vIF)
  c.if_speed = v0;
  c.inc_flux = (float)((1. + nhe_to_nh) * c.nH * v0);
}

// update_thermal for one cell (gas_funcs.cc:362-411, temp_ev = TRUE, subgrid = FALSE).
template <bool STRICT>
__device__ inline void thermal_update(ThermCell& c, const ThermConst& k, const HeatSrc& hs, int nfreq,
                                      float nhe_to_nh) {
  float t_temp = 0.f;
  treion_default<STRICT>(c, k, nhe_to_nh);
  int guard = 0;
  while (t_temp < k.dt && guard < 1000) {
    const float ts = thermal_tstep<STRICT>(c, k);
    const float rem = k.dt - t_temp;
    const float dt_temp = (ts >= rem) ? rem : ts;
    heat_cool<STRICT>(c, k, hs, nfreq);
    if (STRICT) {
      c.temp = (c.temp + 2. / 3. / kKB / c.n_tot * (c.heat - c.cool) * dt_temp) /
               (1. + 2. * (double)(k.hub2f * 0.5f) * dt_temp + 1. / c.n_tot * c.dne_dt * dt_temp -
                2. * (double)c.ddelta / 3. / (double)c.rho_rel * dt_temp);
    } else {
      const float c23 = (float)(2. / 3. / kKB);
      const float inv_n = __fdividef(1.0f, c.n_tot);
      c.temp = __fdividef(c.temp + (c23 * inv_n) * (c.heat - c.cool) * dt_temp,
                          1.0f + k.hub2f * dt_temp + (c.dne_dt * inv_n) * dt_temp -
                              __fdividef((2.0f / 3.0f) * c.ddelta, c.rho_rel) * dt_temp);
    }
    t_temp += dt_temp;
    ++guard;
  }
  c.temp = (c.temp >= kTempMin) ? c.temp : kTempMin;
}

}  // namespace frt
