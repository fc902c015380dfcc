// The sub-grid RadHydro model of the reference (subgrid = TRUE with equilibrium = TRUE and
// ifront = FALSE): mean free paths in ionised cells from photo-ionisation equilibrium, HI
// fractions interpolated in the RadHydro tables, the sub-grid ray deposition and the sub-grid
// heating and cooling (ray_tracing.cc:630-1214 and subgrid.cc, gas_funcs.cc:134-457).
//
// Without I-front tracking every cell counts as passed by the front (fion = 1, rt_funcs.cc:55),
// so no crossing draws on a per-cell photon budget and the result of a ray pass does not depend
// on the order of the rays: the step keeps the lit / dark split of the plain model. The walk, the
// lit-cell numbering, the merge, the split and the cast are the plain model's; this file holds the
// cell passes, the ray pass and the thermal update of the sub-grid model, each evaluating the
// reference's float and double expressions (compiled with -fmad=false like the geometry). The
// reference's float overloads of log10 are taken as the double logarithm rounded to float.
#include <limits.h>
#include <math.h>

#include "frt_internal.cuh"

namespace frt {

namespace {

constexpr float kSigmaEffRH = 2.517139346618065e-18f;   // global_variables.cc:241
constexpr float kGammaMin = 1e-16f;                      // global_variables.cc:303
constexpr float kMaxSubgridFrac = 0.49f;                 // global_variables.cc:245
constexpr int kNt = 5000;                                // global_variables.cc:262
constexpr int kNdlin = 500;                              // global_variables.cc:291
constexpr int kNtcross = 10;                             // global_variables.cc:224
// frac_h1 / frac_he1 of the sub-grid ray pass (ray_tracing.cc:765-767)
constexpr double kFracH1 = 1. - (kY / 4.) / (1. - kY + kY / 4.);
constexpr double kFracHe1 = (kY / 4.) / (1. - kY + kY / 4.);
// A cell counts as ionised once any photon deposited a rate there (avg_gamma > 0), however small,
// and float atomics (red / atom .add.f32) flush subnormal operands to zero. The ray passes
// therefore add each crossing's float rate times 2^64, an exact scaling that keeps every nonzero
// rate normal, and the cell pass scales the sums back.
constexpr float kAccScale = 18446744073709551616.f;           // 2^64
constexpr float kAccUnscale = 5.42101086242752217e-20f;       // 2^-64

__device__ __forceinline__ float mind_f(float a, float b) { return (a >= b) ? b : a; }
__device__ __forceinline__ float maxd_f(float a, float b) { return (b >= a) ? b : a; }
__device__ __forceinline__ float flog10(float x) { return (float)log10((double)x); }

// the photo-ionisation rates of the RadHydro runs (init_radhydro_data, subgrid.cc:124-128)
__device__ __forceinline__ float gamma_dom(int g) {
  return g == 0 ? 3e-15f : (g == 1 ? 3e-14f : (g == 2 ? 3e-13f : (g == 3 ? 3e-12f : 3e-11f)));
}

template <typename T>
__device__ __forceinline__ T block_sum(T v) {
  __shared__ T red[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  T r = 0;
  if (w == 0) {
    r = (lane < (int)(blockDim.x >> 5)) ? red[lane] : (T)0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  return r;
}

__device__ __forceinline__ int box_of(const Dev& d, long long gc) { return d.tile_box[gc >> kTileShift]; }

// interpolate (general_funcs.cc:275-315) over n points of global memory
__device__ float interp_lin(const float* x, const float* y, float x0, int n) {
  for (int i = 0; i < n - 1; i++)
    if (((x[i] <= x0) && (x[i + 1] >= x0)) || ((x[i] >= x0) && (x[i + 1] <= x0)))
      return y[i] + (y[i + 1] - y[i]) / (x[i + 1] - x[i]) * (x0 - x[i]);
  const bool up = x[0] < x[n - 1];
  if ((up && x0 > x[n - 1]) || (!up && x0 < x[n - 1])) {
    const float slope = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
    return y[n - 1] + slope * (x0 - x[n - 1]);
  }
  const float slope = (y[1] - y[0]) / (x[1] - x[0]);
  return y[0] + slope * (x0 - x[0]);
}

// The RadHydro arrays are [Nt][3][3][3] floats filled and read at the gamma index q + 1
// (subgrid.cc:24-36, 329-331): the flat offset is the reference's own address arithmetic.
__device__ __forceinline__ size_t rh_at(int t, int m, int p, int iq) {
  return (((size_t)t * 3 + m) * 3 + p) * 3 + iq;
}

// deltaNL_to_deltasig (subgrid.cc:196-205), Mo & White (1996)
__device__ float deltasig(float deltaNL, float redshift) {
  const float dcmode = 5.10655f;
  const float sigma0 = (float)(dcmode / sqrt(3.));
  const float d_of_z = (float)(1. / (1 + redshift) / 0.78205);
  const float delta = (float)(-1.35 * pow(1. + deltaNL, -2. / 3.) + 0.78785 * pow(1. + deltaNL, -0.58661) -
                              1.12431 * pow(1. + deltaNL, -0.5) + 1.68647);
  return delta / d_of_z / sigma0;
}

// the HI fractions of the RadHydro runs at time x since ionisation, linear in time between the
// table rows itf and itf + 1 (subgrid.cc:340-343), for the tre indices it[2] and density
// indices id[2], at the three rates of the runs, clamped to [0, 1]
__device__ void fh1_at(const Dev& d, int itf, float x, const int it[2], const int id[2], float f[2][2][3]) {
  const float* T = d.sg_time;
  const float* H = d.sg_fh1;
  for (int g = 0; g < 3; g++)
    for (int m = 0; m < 2; m++)
      for (int p = 0; p < 2; p++) {
        const size_t a = rh_at(itf, it[m], id[p], g + 1), b = rh_at(itf + 1, it[m], id[p], g + 1);
        const float v = H[a] + (H[b] - H[a]) / (T[b] - T[a]) * (x - T[a]);
        f[m][p][g] = mind_f(maxd_f(v, 0.f), 1.f);
      }
}

// get_tradhydro_index (subgrid.cc:189-193)
__device__ __forceinline__ int rh_tindex(const Dev& d, float tsince) {
  const int i = (int)floorf(tsince / d.sg_time[rh_at(kNt - 1, 0, 0, 0)] * (kNt - 1));
  return max(0, min(i, kNt - 2));
}

// get_interpolate_gamma_f (subgrid.cc:211-250), fractype = TRUE, with the extension to the outer
// rates of get_gamma_interp (subgrid.cc:451-452): log-log in tre + tsince, then in 1 + delta
__device__ void gamma_f(const Dev& d, const BoxP& B, float tsince, float tre, float deltaNL, const int it[2],
                        const int id[2], float f[2][2][3], float out[5]) {
  const float lt = flog10(tre + tsince);
  const float lt0 = flog10(d.sg_tre_dom[it[0]] + tsince), lt1 = flog10(d.sg_tre_dom[it[1]] + tsince);
  const double ld = log10(1. + (double)deltaNL);
  const double ld0 = log10(1. + (double)B.sg_dnl_dom[id[0]]), ld1 = log10(1. + (double)B.sg_dnl_dom[id[1]]);
  for (int g = 0; g < 3; g++) {
    const float fd0 = flog10(f[0][0][g]) + (flog10(f[1][0][g]) - flog10(f[0][0][g])) * (lt - lt0) / (lt1 - lt0);
    const float fd1 = flog10(f[0][1][g]) + (flog10(f[1][1][g]) - flog10(f[0][1][g])) * (lt - lt0) / (lt1 - lt0);
    const float fg = (float)((double)fd0 + (double)(fd1 - fd0) * (ld - ld0) / (ld1 - ld0));
    out[g + 1] = mind_f((float)pow(10., (double)fg), kMaxSubgridFrac);
  }
  out[0] = out[1];                                                              // (g0/g1)^0
  out[4] = (float)(1.0 / (double)(gamma_dom(4) / gamma_dom(3)) * (double)out[3]);   // (g4/g3)^-1
}

// get_gamma_interp (subgrid.cc:257-545) for the HI fraction, the one interpolant the equilibrium
// model reads (interp_nh1): out[5] over the rates gamma_dom. Once I-fronts have started to cross
// the cell (tcross_flag, with I-front tracking) the interpolant is the average over the tenths of
// the cell the fronts passed, each tenth at its own crossing time, weighted up to fion_max.
__device__ void fh1_interp(const Dev& d, const BoxP& B, long long gc, bool tcross_flag, float tre, float deltaNL,
                           float tsince, float out[5]) {
  int it[2], id[2];
  tre = maxd_f(d.sg_t12, tre);
  if (tre > d.sg_t8) { it[1] = 2; it[0] = 1; }
  else { it[1] = 1; it[0] = 0; }
  if (deltasig(deltaNL, B.th.zz) < 0.f) { id[1] = 1; id[0] = 0; }
  else { id[1] = 2; id[0] = 1; }
  {
    float f[2][2][3];
    fh1_at(d, rh_tindex(d, tsince), tsince, it, id, f);
    gamma_f(d, B, tsince, tre, deltaNL, it, id, f, out);
  }
  if (!tcross_flag) return;
  const float* tcn = d.tcross_new + (size_t)gc * kNtcross;
  float ftt[kNtcross][5];
  for (int tt = 0; tt < kNtcross; tt++) {
    int itc[2];
    if (tre + tcn[tt] > d.sg_t8) { itc[1] = 2; itc[0] = 1; }
    else { itc[1] = 1; itc[0] = 0; }
    const float tc = (tt == 0) ? (float)((double)tcn[0] / 2.)
                               : (float)((double)tcn[tt - 1] + (double)(tcn[tt] - tcn[tt - 1]) / 2.);
    float f[2][2][3];
    fh1_at(d, rh_tindex(d, tsince - tc), tsince - tc, itc, id, f);
    gamma_f(d, B, tsince - tc, tre + tc, deltaNL, itc, id, f, ftt[tt]);
  }
  const float fmax = d.fion_max[gc];
  const float tc_frac = (float)(1. / (double)(float)kNtcross);
  for (int g = 0; g < 5; g++) {
    float acc = 0.f;
    if ((double)fmax == 1.) {
      for (int tt = 0; tt < kNtcross; tt++) acc += tc_frac * ftt[tt][g];
    } else {
      for (int tt = 0; tt < kNtcross; tt++)
        if ((fmax >= (float)tt * tc_frac) && ((double)fmax < ((double)tt + 1.) * (double)tc_frac)) {
          for (int ttt = 0; ttt < tt; ttt++) acc += tc_frac * ftt[ttt][g];
          acc += (maxd_f(0.01f, fmax) - (float)tt * tc_frac) * ftt[tt][g];
        }
    }
    acc = acc / maxd_f(0.01f, fmax);
    out[g] = mind_f(acc, kMaxSubgridFrac);
  }
}

// interp_nh1 (subgrid.cc:629-641): the cell's n_HI at its photo-ionisation rate
__device__ float interp_nh1(const float fh[5], float gammaH1, float nH, float fH1_0) {
  const float gamma = maxd_f(gammaH1, kGammaMin);
  const float lg = flog10(gamma), lg0 = flog10(gamma_dom(0));
  int g = (int)floor(4.0 * (double)(lg - lg0) / (double)(flog10(gamma_dom(4)) - lg0));
  g = max(0, min(g, 3));
  float v = flog10(fh[g]) + (flog10(fh[g + 1]) - flog10(fh[g])) / (flog10(gamma_dom(g + 1)) - flog10(gamma_dom(g))) *
                                (lg - flog10(gamma_dom(g)));
  v = maxd_f(mind_f((float)pow(10., (double)v), fH1_0), 0.f);
  return v * nH;
}

// the equilibrium mean free paths of an ionised cell (ray_tracing.cc:989-994)
__device__ void eq_mfp(const Dev& d, float gam, float clump, float temp, float nH, float* mfp, float* mfp912) {
  const float g = maxd_f(kGammaMin, gam) / clump;
  const double ab = alphaB_H2_d((double)maxd_f(kTempMin, temp)), n2 = (double)nH * (double)nH;   // pow(nH, 2.)
  const float m = (float)((double)(g / kSigmaEffRH) / ab / n2 / 1.082);
  const float m912 = (float)((double)g / d.sigH1_912 / ab / n2 / 1.082);
  *mfp = maxd_f(0.f, m);   // mfp_min = 1e-2 dx[0] is taken before dx is set (global_variables.cc:301): 0
  *mfp912 = maxd_f(0.f, m912);
}

// sub-grid photo-heating and cooling (gas_funcs.cc:134-242 with subgrid = TRUE)
__device__ double alphaA_H2_d(double T) {
  const double x = lam_d(T, kEthH1);
  return 1.269e-13 * pow(x, 1.503) / pow((1.0 + pow((x / 0.522), 0.470)), 1.923);
}
__device__ double alphaA_He2_d(double T) { return 3.0e-14 * pow(lam_d(T, kEthHe1), 0.654); }
__device__ double photoheat(double T, double ne, double nH, double nHe) {   // rates.cc:240-254, alpha = 1.5
  const double alpha = 1.5;
  const double hi = kEthH1 / kHeV * kH *
                    ((alpha + 2.8) / (1.8 + alpha) * (1. - pow(4., -1.8 - alpha)) / (1. - pow(4., -2.8 - alpha)) - 1.) *
                    alphaA_H2_d(T) * ne;
  const double hei = kEthHe1 / kHeV * kH *
                     ((alpha + 1.7) / (0.7 + alpha) * (1. - pow(2.2, -0.7 - alpha)) / (1. - pow(2.2, -1.7 - alpha)) - 1.) *
                     alphaA_He2_d(T) * ne;
  return hi * nH + hei * nHe;
}

__device__ void heat_cool_sg(ThermCell& c, const ThermConst& k, float nHe, float gamma_tot, float fion) {
  const float tm = maxd_f(kTempMin, c.temp);
  const float nt = c.nH + nHe;
  c.heat = (gamma_tot > 3e-14) ? (float)photoheat((double)tm, (double)nt, (double)c.nH, (double)nHe) : 0.f;
  float cool = 0.f;
  cool += rcrB_H2_d(tm) * nt * c.nH;
  cool += rcrB_He2_d(tm) * nt * nHe;
  const float nff = fion * nt;   // fion (nH + nHe)
  cool += free_free_d(tm) * ((double)nff * (double)nff);
  cool -= k.compton_d * nt * (2.726 * (1 + k.zz) - tm);
  c.cool = cool;
}

// update_thermal for one cell in the sub-grid model (gas_funcs.cc:362-418): neutral until
// ionised; an ionised cell's temperature is sub-cycled without the post-front heating of the
// plain model (set_Treion_default runs only without the sub-grid model)
__device__ void thermal_sg(ThermCell& c, const ThermConst& k, bool ionised, float nHe, float gamma_tot, float temp_0,
                           float fion) {
  if (!ionised) {
    c.temp = temp_0;
    return;
  }
  float t_temp = 0.f;
  int guard = 0;
  while (t_temp < k.dt && guard < 1000) {
    const float ts = thermal_tstep<true>(c, k);
    const float rem = k.dt - t_temp;
    const float dt_temp = (ts >= rem) ? rem : ts;
    heat_cool_sg(c, k, nHe, gamma_tot, fion);
    c.temp = (c.temp + 2. / 3. / kKB / c.n_tot * (c.heat - c.cool) * dt_temp) /
             (1. + 2. * (double)(k.hub2f * 0.5f) * dt_temp + 1. / c.n_tot * c.dne_dt * dt_temp -
              2. * (double)c.ddelta / 3. / (double)c.rho_rel * dt_temp);
    t_temp += dt_temp;
    ++guard;
  }
  c.temp = maxd_f(c.temp, kTempMin);
}

// set_Treion (subgrid.cc:660-670): the temperature of the newly ionised part of a cell from the
// I-front speed (D'Aloisio et al. 2019 fit), averaged into the cell's temperature
__device__ void set_treion_front(float vIF, float fi_old, float fi_new, float& temp) {
  const float Cn[5] = {9.5432f, -1.6441e-2f, -9.8010e-3f, 4.1664e-3f, -2.2710e-4f};
  float ln_treion = 0.f;
  const double lv = log((double)vIF / 1e5);
  for (int t = 0; t < 5; t++) ln_treion = (float)((double)ln_treion + (double)Cn[t] * pow(lv, (double)t));
  if (fi_new > 0.f) temp = (fi_old * temp + (fi_new - fi_old) * expf(ln_treion)) / fi_new;
}

// update_fion (subgrid.cc:694-751): the front advances by vIF dt / dx with vIF from the photons
// that entered the cell's neutral part (ng2), and the crossing times are booked per tenth of the
// cell; fion and temp are updated in place, the rest of the cell's front state in memory
__device__ void update_front(const Dev& d, const BoxP& B, long long gc, double ng2, float nH, float& fion, float& temp) {
  const float dt = B.dt, dx = B.dx;
  const float vIF_min = (float)(5e1 * 1e5);
  const double Fl = ng2 / pow((double)dx, 2.) / (double)dt;
  const float vIF = (float)(Fl / (double)nH / (1. + (double)d.nhe_to_nh));
  const float fion_old = fion;
  const float fmax_old = d.fion_max[gc];
  float fmax = fmax_old;
  fion = mind_f(fion + vIF * dt / dx, 1.f);
  if (fion > fmax) fmax = fion;
  d.fion_max[gc] = fmax;
  if ((vIF > vIF_min) || (fion_old == 0.f)) set_treion_front(maxd_f(vIF, vIF_min), fion_old, fion, temp);
  if ((fion_old < 0.5f) && (fion >= 0.5f)) d.treion_out[gc] = B.t - dt;
  const float tdiff = (fion >= 1.f) ? (float)(0.5 * (double)dt) : 0.f;
  if (d.outputs == FRT_OUT_DIAG) {
    d.if_speed[gc] = vIF;
    d.inc_flux[gc] = (float)Fl;
  }
  d.delta_fion[gc] = fion - fion_old;
  d.tcross[gc] += dt - tdiff;
  const float tc_frac = (float)(1. / (double)(float)kNtcross);
  unsigned bits = d.tcross_bits[gc];
  float* tcn = d.tcross_new + (size_t)gc * kNtcross;
  for (int tt = 0; tt < kNtcross; tt++) {
    const double edge = (double)tc_frac * ((double)tt + 1.);
    const bool checked = (bits >> tt) & 1u;
    if (((double)fmax < edge) && !checked) {
      tcn[tt] += dt;
    } else if (((double)fmax >= edge) && ((double)fmax_old < edge) && !checked) {
      tcn[tt] = (float)((double)tcn[tt] + (double)dt * (edge - (double)fmax_old) / (double)(fmax - fmax_old));
      bits |= 1u << tt;
    }
  }
  d.tcross_bits[gc] = (uint16_t)bits;
  d.if_flags[gc] |= 1;   // tcross_flag
}

// the ionised fraction of a cell the fronts left, lowered by the recombinations of a dt without
// photons (ray_tracing.cc:1023-1027, 1051-1054)
__device__ __forceinline__ float front_recombine(const Dev& d, float fion, float clump, float temp, float nH, float dt) {
  const double r = (double)fion - (double)clump * alphaB_H2_d((double)maxd_f(kTempMin, temp)) *
                                      (1. + (double)d.nhe_to_nh) * (double)nH * (double)fion * (double)dt;
  return maxd_f(0.f, (float)r);
}

// One cell's last C2Ray iteration and thermal update in the sub-grid model (the sub-grid branch
// ray_tracing.cc:956-1071, the bookkeeping 1116-1209, gas_funcs.cc:362-418). Inputs: the cell's
// step-start state and its rate of this iteration; writes the dense state.
struct SgCell {
  long long gc;
  int box, slot;                     // slot: lit slot, or -1 for a cell no ray touched
  float nH, nHe, nh1, nhe1;          // step start (the iteration-0 averages are these)
  float clump, temp, heat, cool, rec_h2, rec_he2, treion;
  bool flag;
  float gam, gam_he;                 // Gamma_HI, Gamma_HeI of the last iteration
  float fion;                        // the fronts' ionised fraction at the step's start (1 without them)
  double ng1, ng2;                   // I-front photon counts of the last iteration (absorbed x sigma x path, entering)
};

template <bool THERMAL>
__device__ void finish_cell(const Dev& d, const SgCell& s) {
  const BoxP& B = d.box[s.box];
  const float dt = B.dt;
  const bool iff = d.ifront != 0;
  bool flag = s.flag, first = false;
  float treion = s.treion;
  // first photons: the cell is ionised (ray_tracing.cc:964-970)
  if (!flag && ((iff && s.ng1 > 0.) || s.gam > 0.f)) {
    treion = B.t - dt;
    flag = true;
    first = true;
  }
  float fion = s.fion, gam = s.gam, temp = s.temp;
  // the HI-fraction interpolant with the front state of the step's start (get_gamma_interp runs
  // at iteration 0 for ionised cells and before update_fion for new ones)
  float fh[5];
  if (flag) {
    const float rho = d.rho[s.gc];
    const bool tcf = iff && !first && (d.if_flags[s.gc] & 1);
    fh1_interp(d, B, s.gc, tcf, treion + d.sg_tinit, (float)((double)(rho / B.avg_rho) - 1.), B.t - treion, fh);
  }
  float mfp = 0.f, mfp912 = 0.f;
  bool have_mfp = false;
  if (flag && fion > 0.f) {
    eq_mfp(d, gam, s.clump, temp, s.nH, &mfp, &mfp912);
    have_mfp = true;
  }
  if (iff && flag && fion < 1.f) {   // the I-front correction (ray_tracing.cc:1003-1047)
    const double gamma_fion = s.ng1 / (double)dt / B.vol;
    update_front(d, B, s.gc, s.ng2, s.nH, fion, temp);
    if (fion >= 1.f) d.if_flags[s.gc] &= (uint8_t)~2u;   // neutral_flag = FALSE
    if ((fion < 1.f) && (gam == 0.f) && !first) fion = front_recombine(d, fion, s.clump, temp, s.nH, dt);
    if (first) {   // a newly ionised cell: its rate and mean free path from the front's photons
      gam = (float)gamma_fion;
      eq_mfp(d, gam, s.clump, temp, s.nH, &mfp, &mfp912);
      have_mfp = true;
    }
  }
  if (iff && (fion == 1.f) && (gam == 0.f)) fion = front_recombine(d, fion, s.clump, temp, s.nH, dt);
  // n_e of the iteration (ray_tracing.cc:949): the averages stay at their iteration-0 values
  const float nelec_f = s.nH - s.nh1 + s.nHe - s.nhe1;
  float nH1 = s.nh1, nHe1 = s.nhe1, avg_he = s.nhe1;
  // the ionised densities of a cell never ionised keep their set-up values (init_funcs.cc)
  float nH2 = (float)((double)s.nH * (1. - (double)d.sg_fH1_0));
  float nHe2 = (float)((double)s.nHe * (1. - (double)d.sg_fHe1_0));
  if (flag) {
    nH1 = interp_nh1(fh, gam, s.nH, d.sg_fH1_0);
    nHe1 = nH1 * s.nHe / s.nH;
    avg_he = nHe1;
    nH2 = s.nH * fion;
    nHe2 = s.nHe * fion;
  }
  const float ne = nH2 + nHe2;
  const float n_tot = (float)(2. * (double)(s.nH + s.nHe));
  const float dne_dt = (-(s.nH + s.nHe) + (s.nH + s.nHe)) / dt;   // 0: the gas counts as ionised
  const long long gc = s.gc;
  float fH1, fHe1;
  if (iff) {
    float fH2 = nH2 / s.nH, fHe2 = nHe2 / s.nHe;
    if (fion > 0.f) {
      fH2 *= fion;
      fHe2 *= fion;
    }
    fH1 = (float)(1. - (double)fH2);
    fHe1 = (float)(1. - (double)fHe2 - 0.);
    d.fion[gc] = fion;
  } else {
    fH1 = nH1 / s.nH;
    fHe1 = nHe1 / s.nHe;
  }
  d.nH1[gc] = nH1;
  d.nHe1[gc] = nHe1;
  d.avg_nh1[gc] = s.nh1;
  d.avg_nhe1[gc] = avg_he;
  d.f_H1[gc] = fH1;
  d.f_He1[gc] = fHe1;
  d.ne[gc] = ne;
  if (flag) {
    if (have_mfp) d.mfp[gc] = mfp;
    if (!s.flag) {
      d.treion[gc] = treion;
      d.treion_flag[gc] = 1;
    }
  } else {
    d.mfp[gc] = (float)(1. / (double)s.nh1 / d.sigH1_d[0]);   // the step-start gas (ray_tracing.cc:691)
  }
  if (first && iff && s.slot >= 0) d.l_acc[s.slot].x = gam;   // gamma_H1_tot = avg_gamma
  if (d.outputs == FRT_OUT_DIAG) {
    const double nelec_d = (double)nelec_f;
    if (have_mfp) d.mfp912[gc] = mfp912;
    d.rec_h2[gc] = s.rec_h2;
    d.rec_he2[gc] = s.rec_he2;
    d.recrate_h2[gc] = (float)((double)(s.clump * s.rec_h2) * nelec_d * (double)nH2);
    d.recrate_he2[gc] = (float)((double)(s.clump * s.rec_he2) * nelec_d * (double)nHe2);
    d.n_tot[gc] = n_tot;
    d.dne_dt[gc] = dne_dt;
    if (!(iff && flag && s.fion < 1.f)) {   // (update_front wrote them)
      d.if_speed[gc] = 0.f;
      d.inc_flux[gc] = 0.f;
    }
  }
  if (iff && !(flag && s.fion < 1.f)) d.delta_fion[gc] = 0.f;
  if (THERMAL) {
    ThermCell c;
    c.temp = temp;
    c.heat = s.heat;
    c.cool = s.cool;
    c.nH = s.nH;
    c.n_tot = n_tot;
    c.dne_dt = dne_dt;
    if (d.ddelta) {
      c.ddelta = d.ddelta[gc];
      c.rho_rel = d.rho[gc] / B.avg_rho;
    }
    thermal_sg(c, B.th, flag, s.nHe, gam, d.sg_temp0, iff ? fion : 1.f);
    d.temp[gc] = c.temp;
    if (flag) {
      d.heat[gc] = c.heat;
      d.cool[gc] = c.cool;
    }
  } else {
    d.temp[gc] = temp;   // set_Treion's change; update_thermal runs later
  }
}

// ---- kernels ---------------------------------------------------------------------------------
// delta_dom_to_deltaNL_dom (subgrid.cc:97-132) per box at max(t(z=12), t + tinit) (main.cc:127)
__global__ void k_sg_step(Dev d) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < d.nbox; b += gridDim.x * blockDim.x) {
    BoxP& B = d.box[b];
    const float time = maxd_f(d.sg_t12, B.t + d.sg_tinit);
    const float tcap = d.sg_tcap;
    const float dd0 = (float)-1.7320508075688772, dd2 = (float)1.7320508075688772;   // -/+ 3^0.5
    const float* t = d.sg_tdnl;
    int ti_m = 0, ti_p = 1, tc_m = 0, tc_p = 1;
    for (int i = 0; i < kNdlin - 1; i++) {
      if ((t[i] <= time) && (t[i + 1] >= time)) { ti_m = i; ti_p = i + 1; }
      if ((t[i] <= tcap) && (t[i + 1] >= tcap)) { tc_m = i; tc_p = i + 1; }
    }
    const float* ds = d.sg_ds;
    auto row = [&](int i) { return d.sg_dnl + (size_t)i * kNdlin; };
    const float d0m = interp_lin(ds, row(ti_m), dd0, kNdlin), d0p = interp_lin(ds, row(ti_p), dd0, kNdlin);
    const float d2m = interp_lin(ds, row(ti_m), dd2, kNdlin), d2p = interp_lin(ds, row(ti_p), dd2, kNdlin);
    const float cm = interp_lin(ds, row(tc_m), dd2, kNdlin), cp = interp_lin(ds, row(tc_p), dd2, kNdlin);
    const float cap = cm + (cp - cm) / (t[tc_p] - t[tc_m]) * (tcap - t[tc_m]);
    B.sg_dnl_dom[1] = 0.f;
    B.sg_dnl_dom[0] = d0m + (d0p - d0m) / (t[ti_p] - t[ti_m]) * (time - t[ti_m]);
    const float v2 = d2m + (d2p - d2m) / (t[ti_p] - t[ti_m]) * (time - t[ti_m]);
    B.sg_dnl_dom[2] = mind_f(v2, cap);
  }
}

// init()'s mean free paths (init_funcs.cc: 1/sigma(nu_0)/<n_HI>)
__global__ void k_sg_mfp_init(Dev d) {
  for (long long gc = blockIdx.x * (long long)blockDim.x + threadIdx.x; gc < d.ncell_total;
       gc += (long long)gridDim.x * blockDim.x)
    d.mfp[gc] = (float)(1. / d.sigH1_d[0] / (double)d.avg_nh1[gc]);
}

// iteration 0 of the lit cells (ray_tracing.cc:655-693 with subgrid = TRUE)
__global__ void k_sg_lit_init(Dev d) {
  const int n = min(d.ctl->n_lit, d.lit_cap);
  const int F = d.F, L = d.lit_cap;
  if (blockIdx.x == 0 && threadIdx.x < kMaxIterQueue) d.rp_queue[threadIdx.x] = 0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int gc = d.l_cell[s];
    const int bx = box_of(d, gc);
    const float temp = d.temp[gc];
    const float cl = d.clump ? d.clump[gc] : d.const_clump;
    const float nh1 = d.nH1[gc], nhe1 = d.nHe1[gc];
    float rh, rhe;
    recomb_coeffs<true>(temp, &rh, &rhe);
    d.l_box[s] = (uint16_t)bx;
    d.l_nh[s] = d.nH[gc];
    d.l_nhe[s] = d.nHe[gc];
    d.l_rec_h2[s] = rh;
    d.l_rec_he2[s] = rhe;
    d.l_crec_h[s] = cl * rh;
    d.l_crec_he[s] = cl * rhe;
    d.l_avg[s] = make_float2(nh1, nhe1);
    d.l_acc[s] = make_float2(0.f, 0.f);
    d.l_mfp[s] = d.treion_flag[gc] ? d.mfp[gc] : (float)(1. / (double)nh1 / d.sigH1_d[0]);
    if (d.ifront) {
      // the fronts' ionised fraction for the step's ray passes and the atoms of the cell's
      // neutral part, vol nH (1 + chi) (1 - fion) (ray_tracing.cc:873)
      const float fion = d.fion[gc];
      d.l_fion[s] = fion;
      d.l_free[s] = d.box[bx].vol * (double)d.nH[gc] * (1. + (double)d.nhe_to_nh) * (1. - (double)fion);
      d.if_cnt[s] = 0;
      d.if_fill[s] = 0;
    }
    if (d.per_bin)
      for (int nu = 0; nu < F; nu++) {
        d.l_ngam[(size_t)nu * L + s] = 0.f;
        d.l_acc_nu_h[(size_t)nu * L + s] = 0.f;
        d.l_acc_nu_he[(size_t)nu * L + s] = 0.f;
      }
  }
}

// the sub-grid ray pass of one C2Ray iteration (ray_tracing.cc:701-938 with subgrid = TRUE,
// fion = 1): per crossing the rate from the sub-grid cross section over the effective path
// delta_s_eff, then the segment's optical depth from the cell's mean free path; one thread per
// moved ray, double arithmetic as the reference's locals
template <bool LAST>
__global__ void __launch_bounds__(256) k_sg_raypass(Dev d, int iter) {
  const int nmv = min((int)(d.ctl->mv_seg >> 32), d.ray_cap);
  const RayPool A = d.pool[d.ctl->cur];
  const int cap = d.ray_cap, F = d.F, L = d.lit_cap;
  double dep = 0.0, kil = 0.0;
  long long nkill = 0;
  const float fion = 1.f;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nmv; q += gridDim.x * blockDim.x) {
    const int4 hd = d.mv_hdr[q];
    const int i = hd.x, ns = hd.z;
    const int2* sp = d.pk + hd.y;
    const BoxP& B = d.box[hd.w];
    const double nmin = B.nphot_min;
    const double dt = (double)B.dt, vol = B.vol;
    float nph[FRT_MAX_FREQ];
    double tau_h1[FRT_MAX_FREQ], tau_he1[FRT_MAX_FREQ];
    for (int nu = 0; nu < F; nu++) {
      nph[nu] = A.nphot[(size_t)nu * cap + i];
      tau_h1[nu] = 0.;
      tau_he1[nu] = 0.;
    }
    for (int p = 0; p < ns; p++) {
      const int2 sg = sp[p];
      const int slot = sg.x;
      if (slot < 0 || slot >= L) break;
      const float dist = __int_as_float(sg.y & 0x7fffffff);
      const float mfp = d.l_mfp[slot];
      double nin[FRT_MAX_FREQ], total = 0.;
      for (int nu = 0; nu < F; nu++) {
        nin[nu] = ((double)nph[nu] * kPhotNorm) * exp(-tau_h1[nu] - tau_he1[nu]);
        total += nin[nu] / kPhotNorm;
      }
      const bool dump = total < nmin;
      const float delta_s_eff = (iter == 0) ? (float)((double)(fion * dist) / kFracH1)
                                            : (float)((double)mfp * (1. - exp(-(double)(fion * dist / mfp) / kFracH1)));
      float gh_sum = 0.f, ghe_sum = 0.f;
      const float dtau_f = fion * dist / mfp;
      for (int nu = 0; nu < F; nu++) {
        const float gh = (float)(kFracH1 * nin[nu] * (double)kSigmaEffRH * (double)delta_s_eff / dt / vol / (double)fion);
        const float ghe = (float)(kFracHe1 * nin[nu] * (double)kSigmaEffRH * (double)delta_s_eff / dt / vol / (double)fion);
        gh_sum += gh * kAccScale;
        ghe_sum += ghe * kAccScale;
        if (LAST && d.per_bin) {
          atomicAdd(&d.l_ngam[(size_t)nu * L + slot], (float)(nin[nu] / kPhotNorm));
          atomicAdd(&d.l_acc_nu_h[(size_t)nu * L + slot], gh);
          atomicAdd(&d.l_acc_nu_he[(size_t)nu * L + slot], ghe);
        }
        const double dth = (double)dtau_f, dthe = (double)d.nhe_to_nh * dth;
        if (LAST) dep += nin[nu] * (1. - exp(-(dth + dthe))) / kPhotNorm;
        tau_h1[nu] += dth;
        tau_he1[nu] += dthe;
      }
      atomicAdd(&d.l_acc[slot], make_float2(gh_sum, ghe_sum));
      if (dump) break;
    }
    if (LAST) {
      float s = 0.f;
      for (int nu = 0; nu < F; nu++) {
        nph[nu] = (float)(((double)nph[nu] * kPhotNorm) * exp(-tau_h1[nu] - tau_he1[nu]) / kPhotNorm);
        A.nphot[(size_t)nu * cap + i] = nph[nu];
        s += nph[nu];
      }
      if (!(s > nmin)) {
        d.dead[i] = 1;
        nkill += 1;
        kil += (double)s;
      }
    }
  }
  if (LAST) {
    dep = block_sum(dep);
    kil = block_sum(kil);
    nkill = block_sum(nkill);
    if (threadIdx.x == 0) {
      if (dep != 0.0) atomicAdd(&d.ctl->deposited, dep * kPhotNorm);
      if (kil != 0.0) atomicAdd(&d.ctl->killed_ph, kil * kPhotNorm);
      if (nkill) atomicAdd((unsigned long long*)&d.ctl->killed, (unsigned long long)nkill);
    }
  }
}

// the lit cells' sub-grid cell pass of one iteration: the equilibrium mean free path of ionised
// cells for the next ray pass; the last iteration finishes the cells (finish_cell)
template <bool LAST, bool THERMAL>
__global__ void __launch_bounds__(256) k_sg_litpass(Dev d) {
  const int n = min(d.ctl->n_lit, d.lit_cap);
  const int L = d.lit_cap;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int gc = d.l_cell[s];
    const float2 acc = make_float2(d.l_acc[s].x * kAccUnscale, d.l_acc[s].y * kAccUnscale);
    if (!LAST) {
      if (d.treion_flag[gc] && (!d.ifront || d.l_fion[s] > 0.f)) {
        float mfp, m912;
        eq_mfp(d, acc.x, d.clump ? d.clump[gc] : d.const_clump, d.temp[gc], d.l_nh[s], &mfp, &m912);
        d.l_mfp[s] = mfp;
      }
      d.l_acc[s] = make_float2(0.f, 0.f);
      continue;
    }
    d.l_acc[s] = acc;   // the rates as output fields (and for the separate thermal update)
    SgCell c;
    c.gc = gc;
    c.box = d.l_box[s];
    c.nH = d.l_nh[s];
    c.nHe = d.l_nhe[s];
    const float2 av = d.l_avg[s];
    c.nh1 = av.x;
    c.nhe1 = av.y;
    c.clump = d.clump ? d.clump[gc] : d.const_clump;
    c.temp = d.temp[gc];
    c.heat = d.heat[gc];
    c.cool = d.cool[gc];
    c.rec_h2 = d.l_rec_h2[s];
    c.rec_he2 = d.l_rec_he2[s];
    c.treion = d.treion[gc];
    c.flag = d.treion_flag[gc] != 0;
    c.gam = acc.x;
    c.gam_he = acc.y;
    c.slot = s;
    c.fion = d.ifront ? d.l_fion[s] : 1.f;
    c.ng1 = d.ifront ? d.l_ng3[(size_t)L + s] : 0.;
    c.ng2 = d.ifront ? d.l_ng3[2 * (size_t)L + s] : 0.;
    finish_cell<THERMAL>(d, c);
  }
}

// the whole step of a cell no ray touched: Gamma = 0 in every iteration
template <bool THERMAL>
__global__ void __launch_bounds__(256) k_sg_dark(Dev d) {
  for (long long gc = blockIdx.x * (long long)blockDim.x + threadIdx.x; gc < d.ncell_total;
       gc += (long long)gridDim.x * blockDim.x) {
    const int b = box_of(d, gc);
    if (b < 0) continue;
    if (d.lit_flag[gc]) continue;
    const BoxP& B = d.box[b];
    if (gc - B.cell0 >= B.ncell) continue;
    SgCell c;
    c.gc = gc;
    c.box = b;
    c.nH = d.nH[gc];
    c.nHe = d.nHe[gc];
    c.nh1 = d.nH1[gc];
    c.nhe1 = d.nHe1[gc];
    c.clump = d.clump ? d.clump[gc] : d.const_clump;
    c.temp = d.temp[gc];
    c.heat = d.heat[gc];
    c.cool = d.cool[gc];
    recomb_coeffs<true>(c.temp, &c.rec_h2, &c.rec_he2);
    c.treion = d.treion[gc];
    c.flag = d.treion_flag[gc] != 0;
    c.gam = 0.f;
    c.gam_he = 0.f;
    c.slot = -1;
    c.fion = d.ifront ? d.fion[gc] : 1.f;
    c.ng1 = 0.;
    c.ng2 = 0.;
    finish_cell<THERMAL>(d, c);
  }
}

// update_thermal on its own (the call surface: frt_update_thermal after frt_find_avg_unu)
__global__ void k_sg_thermal_all(Dev d) {
  for (long long gc = blockIdx.x * (long long)blockDim.x + threadIdx.x; gc < d.ncell_total;
       gc += (long long)gridDim.x * blockDim.x) {
    const int b = box_of(d, gc);
    if (b < 0) continue;
    const BoxP& B = d.box[b];
    if (gc - B.cell0 >= B.ncell) continue;
    const int slot = d.lit_slot[gc];
    const float gam = (slot >= 0 && slot < d.lit_cap) ? d.l_acc[slot].x : 0.f;
    ThermCell c;
    c.temp = d.temp[gc];
    c.heat = d.heat[gc];
    c.cool = d.cool[gc];
    c.nH = d.nH[gc];
    const float nHe = d.nHe[gc];
    c.n_tot = (float)(2. * (double)(c.nH + nHe));
    c.dne_dt = 0.f;
    if (d.ddelta) {
      c.ddelta = d.ddelta[gc];
      c.rho_rel = d.rho[gc] / B.avg_rho;
    }
    const bool flag = d.treion_flag[gc] != 0;
    thermal_sg(c, B.th, flag, nHe, gam, d.sg_temp0, d.ifront ? d.fion[gc] : 1.f);
    d.temp[gc] = c.temp;
    if (flag) {
      d.heat[gc] = c.heat;
      d.cool[gc] = c.cool;
    }
  }
}

// ---- I-front tracking: the neutral-part photon budget in ray order ---------------------------
// A cell the fronts have not fully passed (fion < 1) absorbs the photons that reach its neutral
// part up to its atoms, ray after ray in the order of the reference's slots (ray_tracing.cc:
// 863-919): a ray that finds the budget spent passes, one that finds it open gives up to the
// remaining atoms and may be absorbed whole (which ends its walk). A ray's entry into a cell thus
// depends on the rays before it in that cell and, through its earlier cells, on rays before it
// there. The step resolves this as a fixed point: each round the ray pass walks every moved ray
// with the budget sums found by the previous round (xs_S, the sum absorbed before the ray at each
// of its front cells), records the photons each crossing brings to the neutral part (xs_E), and
// the budget pass then redoes every front cell's sums over its crossings in ray order. A
// crossing's sum depends only on rays earlier in the order, so the sums settle from the first
// ray on; when a round changes none, the walk is the reference's sequential one.

// crossings of the front cells: count per lit slot, and the moved ray of every packed segment
__global__ void k_if_count(Dev d) {
  const int nmv = min((int)(d.ctl->mv_seg >> 32), d.ray_cap);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nmv; q += gridDim.x * blockDim.x) {
    const int4 hd = d.mv_hdr[q];
    for (int p = 0; p < hd.z; p++) {
      const long long x = (long long)hd.y + p;
      if (x >= d.xs_cap) break;
      d.xs_q[x] = q;
      d.xs_S[x] = 0.;
      d.xs_reach[x] = 0;
      const int slot = d.pk[x].x;
      if (slot >= 0 && slot < d.lit_cap && d.l_fion[slot] < 1.f) atomicAdd(&d.if_cnt[slot], 1);
    }
  }
}

// exclusive offsets of the per-slot counts (one block)
__global__ void __launch_bounds__(1024) k_if_scan(Dev d) {
  __shared__ int wsum[32];
  __shared__ int base_s;
  const int n = min(d.ctl->n_lit, d.lit_cap);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) base_s = 0;
  __syncthreads();
  for (int s0 = 0; s0 < n; s0 += blockDim.x) {
    const int s = s0 + threadIdx.x;
    const int v = (s < n) ? d.if_cnt[s] : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      int u = wsum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, u, o);
        if (lane >= o) u += y;
      }
      wsum[lane] = u;
    }
    __syncthreads();
    if (s < n) d.if_off[s] = base_s + (w > 0 ? wsum[w - 1] : 0) + incl - v;
    __syncthreads();
    if (threadIdx.x == 0) base_s += wsum[31];
    __syncthreads();
  }
}

__global__ void k_if_fill(Dev d) {
  const int nmv = min((int)(d.ctl->mv_seg >> 32), d.ray_cap);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nmv; q += gridDim.x * blockDim.x) {
    const int4 hd = d.mv_hdr[q];
    for (int p = 0; p < hd.z; p++) {
      const long long x = (long long)hd.y + p;
      if (x >= d.xs_cap) break;
      const int slot = d.pk[x].x;
      if (slot >= 0 && slot < d.lit_cap && d.l_fion[slot] < 1.f)
        d.if_list[d.if_off[slot] + atomicAdd(&d.if_fill[slot], 1)] = (int)x;
    }
  }
}

// the crossing order of a front cell: the rays' pool positions (the slot order), then the segment
__device__ __forceinline__ unsigned long long xs_key(const Dev& d, int x) {
  const int4 hd = d.mv_hdr[d.xs_q[x]];
  return ((unsigned long long)(unsigned)hd.x << 8) | (unsigned long long)(unsigned)(x - hd.y);
}

__global__ void k_if_sort(Dev d) {
  const int n = min(d.ctl->n_lit, d.lit_cap);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int cnt = d.if_cnt[s];
    int* lst = d.if_list + d.if_off[s];
    for (int a = 1; a < cnt; a++) {   // insertion sort: the lists are short and nearly ordered
      const int x = lst[a];
      const unsigned long long kx = xs_key(d, x);
      int b = a - 1;
      while (b >= 0 && xs_key(d, lst[b]) > kx) {
        lst[b + 1] = lst[b];
        b--;
      }
      lst[b + 1] = x;
    }
  }
}

__global__ void k_if_zero_acc(Dev d, bool per_bin) {
  const int n = min(d.ctl->n_lit, d.lit_cap);
  const int L = d.lit_cap;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    d.l_acc[s] = make_float2(0.f, 0.f);
    if (per_bin)
      for (int nu = 0; nu < d.F; nu++) {
        d.l_ngam[(size_t)nu * L + s] = 0.f;
        d.l_acc_nu_h[(size_t)nu * L + s] = 0.f;
        d.l_acc_nu_he[(size_t)nu * L + s] = 0.f;
      }
  }
}

// one round of the sub-grid ray pass with I-front tracking (ray_tracing.cc:701-938 with
// subgrid = ifront = TRUE): one thread per moved ray, the reference's double arithmetic. LAST is
// the last C2Ray iteration's pass run once the sums have settled: it also writes the per-bin
// outputs, the rays' photon counts and removals and the ledger.
template <bool LAST>
__global__ void __launch_bounds__(256) k_if_raypass(Dev d, int iter) {
  const int nmv = min((int)(d.ctl->mv_seg >> 32), d.ray_cap);
  const RayPool A = d.pool[d.ctl->cur];
  const int cap = d.ray_cap, F = d.F, L = d.lit_cap;
  const long long XC = d.xs_cap;
  double dep = 0.0, kil = 0.0;
  long long nkill = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nmv; q += gridDim.x * blockDim.x) {
    const int4 hd = d.mv_hdr[q];
    const int i = hd.x, ns = hd.z;
    const BoxP& B = d.box[hd.w];
    const double nmin = B.nphot_min;
    const double dt = (double)B.dt, vol = B.vol;
    double nphot[FRT_MAX_FREQ], tau_h1[FRT_MAX_FREQ], tau_he1[FRT_MAX_FREQ], dtau_h1[FRT_MAX_FREQ],
        dtau_he1[FRT_MAX_FREQ];
    for (int nu = 0; nu < F; nu++) {
      nphot[nu] = (double)A.nphot[(size_t)nu * cap + i] * kPhotNorm;
      tau_h1[nu] = tau_he1[nu] = dtau_h1[nu] = dtau_he1[nu] = 0.;
    }
    bool stopped = false;
    for (int p = 0; p < ns; p++) {
      const long long x = (long long)hd.y + p;
      if (x >= XC) break;
      if (stopped) {
        d.xs_reach[x] = 0;
        continue;
      }
      const int2 sg = d.pk[x];
      const int slot = sg.x;
      if (slot < 0 || slot >= L) {
        stopped = true;
        continue;
      }
      const float dist = __int_as_float(sg.y & 0x7fffffff);
      const float fion = d.l_fion[slot];
      const float mfp = d.l_mfp[slot];
      double nin[FRT_MAX_FREQ], total = 0.;
      for (int nu = 0; nu < F; nu++) {
        nin[nu] = nphot[nu] * exp(-tau_h1[nu] - tau_he1[nu]);
        total += nin[nu] / kPhotNorm;
      }
      const bool dump = total < nmin;
      float gh_sum = 0.f, ghe_sum = 0.f;
      for (int nu = 0; nu < F; nu++) {
        if (LAST && d.per_bin) atomicAdd(&d.l_ngam[(size_t)nu * L + slot], (float)(nin[nu] / kPhotNorm));
        if (fion > 0.f) {
          const float delta_s_eff = (iter == 0)
                                        ? (float)((double)(fion * dist) / kFracH1)
                                        : (float)((double)mfp * (1. - exp(-(double)(fion * dist / mfp) / kFracH1)));
          const float gh = (float)(kFracH1 * nin[nu] * (double)kSigmaEffRH * (double)delta_s_eff / dt / vol / (double)fion);
          const float ghe = (float)(kFracHe1 * nin[nu] * (double)kSigmaEffRH * (double)delta_s_eff / dt / vol / (double)fion);
          gh_sum += gh * kAccScale;
          ghe_sum += ghe * kAccScale;
          if (LAST && d.per_bin) {
            atomicAdd(&d.l_acc_nu_h[(size_t)nu * L + slot], gh);
            atomicAdd(&d.l_acc_nu_he[(size_t)nu * L + slot], ghe);
          }
        }
      }
      if (gh_sum != 0.f || ghe_sum != 0.f) atomicAdd(&d.l_acc[slot], make_float2(gh_sum, ghe_sum));
      if (fion > 0.f)
        for (int nu = 0; nu < F; nu++) {
          dtau_h1[nu] = (double)(fion * dist / mfp);
          dtau_he1[nu] = (double)d.nhe_to_nh * dtau_h1[nu];
        }
      double before = 0.;
      for (int nu = 0; nu < F; nu++) {
        before += nin[nu];
        tau_h1[nu] += dtau_h1[nu];
        tau_he1[nu] += dtau_he1[nu];
      }
      bool absorbed = false;
      if (fion < 1.f) {
        const double S = d.xs_S[x];
        const double free_ngam = d.l_free[slot];
        d.xs_reach[x] = 1;
        double E[FRT_MAX_FREQ];
        for (int nu = 0; nu < F; nu++) {
          E[nu] = nin[nu] * exp(-(dtau_h1[nu] + dtau_he1[nu]));
          d.xs_E[(size_t)nu * XC + x] = E[nu];
        }
        if (S < free_ngam) {
          double left = 0.;
          for (int nu = 0; nu < F; nu++) {
            const double ab = (E[nu] >= free_ngam - S) ? free_ngam - S : E[nu];   // mindd
            nin[nu] = E[nu] - ab;
            left += nin[nu];
          }
          if (left == 0.) {
            absorbed = true;
            for (int nu = 0; nu < F; nu++) tau_h1[nu] = 999.;
          } else {
            for (int nu = 0; nu < F; nu++) tau_h1[nu] += -log(nin[nu] / nphot[nu] / exp(-(tau_h1[nu] + tau_he1[nu])));
          }
        }
      }
      if (LAST) {
        double after = 0.;
        for (int nu = 0; nu < F; nu++) after += nphot[nu] * exp(-tau_h1[nu] - tau_he1[nu]);
        dep += before - after;
      }
      if (dump || absorbed) stopped = true;
    }
    if (LAST) {
      float s = 0.f;
      for (int nu = 0; nu < F; nu++) {
        const float v = (float)(nphot[nu] * exp(-tau_h1[nu] - tau_he1[nu]) / kPhotNorm);
        A.nphot[(size_t)nu * cap + i] = v;
        s += v;
      }
      if (!(s > nmin)) {
        d.dead[i] = 1;
        nkill += 1;
        kil += (double)s;
      }
    }
  }
  if (LAST) {
    dep = block_sum(dep);
    kil = block_sum(kil);
    nkill = block_sum(nkill);
    if (threadIdx.x == 0) {
      if (dep != 0.0) atomicAdd(&d.ctl->deposited, dep);
      if (kil != 0.0) atomicAdd(&d.ctl->killed_ph, kil * kPhotNorm);
      if (nkill) atomicAdd((unsigned long long*)&d.ctl->killed, (unsigned long long)nkill);
    }
  }
}

// the budget pass: every front cell's crossings in ray order, the sums each crossing finds
// (compared with the last round's), and the cell's photon counts of the iteration
__global__ void k_if_budget(Dev d) {
  const int n = min(d.ctl->n_lit, d.lit_cap);
  const int F = d.F, L = d.lit_cap;
  const long long XC = d.xs_cap;
  bool changed = false;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int cnt = d.if_cnt[s];
    double ng0 = 0., ng1 = 0., ng2 = 0.;
    if (cnt > 0) {
      const double free_ngam = d.l_free[s];
      const int* lst = d.if_list + d.if_off[s];
      for (int k = 0; k < cnt; k++) {
        const int x = lst[k];
        double S = 0.;
        if (d.xs_reach[x]) {
          S = ng0;
          const float dist = __int_as_float(d.pk[x].y & 0x7fffffff);
          for (int nu = 0; nu < F; nu++) ng2 += d.xs_E[(size_t)nu * XC + x];
          if (S < free_ngam)
            for (int nu = 0; nu < F; nu++) {
              const double E = d.xs_E[(size_t)nu * XC + x];
              const double ab = (E >= free_ngam - S) ? free_ngam - S : E;
              ng0 += ab;
              ng1 += ab * (double)kSigmaEffRH * (double)dist;
            }
        }
        if (d.xs_S[x] != S) {
          d.xs_S[x] = S;
          changed = true;
        }
      }
    }
    d.l_ng3[s] = ng0;
    d.l_ng3[(size_t)L + s] = ng1;
    d.l_ng3[2 * (size_t)L + s] = ng2;
  }
  if (__syncthreads_or(changed) && threadIdx.x == 0) atomicOr(&d.ctl->if_changed, 1);
}

}  // namespace

void launch_sg_step(const Dev& d, cudaStream_t s) { k_sg_step<<<1, 64, 0, s>>>(d); }
void launch_sg_mfp_init(const Dev& d, cudaStream_t s) { k_sg_mfp_init<<<grid_for(d.ncell_total, 256, 4096), 256, 0, s>>>(d); }
void launch_sg_lit_init(const Dev& d, int grid, cudaStream_t s) { k_sg_lit_init<<<grid, 256, 0, s>>>(d); }
void launch_sg_raypass(const Dev& d, int iter, int grid, cudaStream_t s) {
  if (iter == d.itercount - 1) k_sg_raypass<true><<<grid, 256, 0, s>>>(d, iter);
  else k_sg_raypass<false><<<grid, 256, 0, s>>>(d, iter);
}
void launch_sg_litpass(const Dev& d, int iter, bool fused_thermal, int grid, cudaStream_t s) {
  if (iter != d.itercount - 1) k_sg_litpass<false, false><<<grid, 256, 0, s>>>(d);
  else if (fused_thermal) k_sg_litpass<true, true><<<grid, 256, 0, s>>>(d);
  else k_sg_litpass<true, false><<<grid, 256, 0, s>>>(d);
}
void launch_sg_dark(const Dev& d, bool fused_thermal, int grid, cudaStream_t s) {
  if (fused_thermal) k_sg_dark<true><<<grid, 256, 0, s>>>(d);
  else k_sg_dark<false><<<grid, 256, 0, s>>>(d);
}
void launch_sg_thermal_all(const Dev& d, int grid, cudaStream_t s) { k_sg_thermal_all<<<grid, 256, 0, s>>>(d); }

void launch_if_lists(const Dev& d, int grid, cudaStream_t s) {
  k_if_count<<<grid, 256, 0, s>>>(d);
  k_if_scan<<<1, 1024, 0, s>>>(d);
  k_if_fill<<<grid, 256, 0, s>>>(d);
  k_if_sort<<<grid, 256, 0, s>>>(d);
}

void launch_if_round(const Dev& d, int iter, int grid, cudaStream_t s) {
  k_if_zero_acc<<<grid, 256, 0, s>>>(d, false);
  k_if_raypass<false><<<grid, 256, 0, s>>>(d, iter);
  k_if_budget<<<grid, 256, 0, s>>>(d);
}

void launch_if_final(const Dev& d, int iter, int grid, cudaStream_t s) {
  k_if_zero_acc<<<grid, 256, 0, s>>>(d, d.per_bin != 0);
  k_if_raypass<true><<<grid, 256, 0, s>>>(d, iter);
}

}  // namespace frt
