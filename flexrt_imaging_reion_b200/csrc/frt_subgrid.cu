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
// frac_h1 / frac_he1 of the sub-grid ray pass (ray_tracing.cc:765-767)
constexpr double kFracH1 = 1. - (kY / 4.) / (1. - kY + kY / 4.);
constexpr double kFracHe1 = (kY / 4.) / (1. - kY + kY / 4.);

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

// get_gamma_interp (subgrid.cc:257-486) for the HI fraction, the one interpolant the equilibrium
// model reads (interp_nh1): out[5] over the rates gamma_dom
__device__ void fh1_interp(const Dev& d, const BoxP& B, float tre, float deltaNL, float tsince, float out[5]) {
  int it0, it1, id0, id1;
  tre = maxd_f(d.sg_t12, tre);
  if (tre > d.sg_t8) { it1 = 2; it0 = 1; }
  else { it1 = 1; it0 = 0; }
  if (deltasig(deltaNL, B.th.zz) < 0.f) { id1 = 1; id0 = 0; }
  else { id1 = 2; id0 = 1; }
  const float* T = d.sg_time;
  const float* H = d.sg_fh1;
  // get_tradhydro_index (subgrid.cc:189-193)
  int itf = (int)floorf(tsince / T[rh_at(kNt - 1, 0, 0, 0)] * (kNt - 1));
  itf = max(0, min(itf, kNt - 2));
  const int ind_tre[2] = {it0, it1}, ind_delta[2] = {id0, id1};
  const float lt = flog10(tre + tsince);
  const float lt0 = flog10(d.sg_tre_dom[it0] + tsince), lt1 = flog10(d.sg_tre_dom[it1] + tsince);
  const double ld = log10(1. + (double)deltaNL);
  const double ld0 = log10(1. + (double)B.sg_dnl_dom[id0]), ld1 = log10(1. + (double)B.sg_dnl_dom[id1]);
  for (int g = 0; g < 3; g++) {
    float f[2][2];
    for (int m = 0; m < 2; m++)
      for (int p = 0; p < 2; p++) {
        const size_t a = rh_at(itf, ind_tre[m], ind_delta[p], g + 1), b = rh_at(itf + 1, ind_tre[m], ind_delta[p], g + 1);
        const float v = H[a] + (H[b] - H[a]) / (T[b] - T[a]) * (tsince - T[a]);
        f[m][p] = mind_f(maxd_f(v, 0.f), 1.f);
      }
    // get_interpolate_gamma_f (subgrid.cc:211-250): log-log in tre + tsince, then in 1 + delta
    const float fd0 = flog10(f[0][0]) + (flog10(f[1][0]) - flog10(f[0][0])) * (lt - lt0) / (lt1 - lt0);
    const float fd1 = flog10(f[0][1]) + (flog10(f[1][1]) - flog10(f[0][1])) * (lt - lt0) / (lt1 - lt0);
    const float fg = (float)((double)fd0 + (double)(fd1 - fd0) * (ld - ld0) / (ld1 - ld0));
    out[g + 1] = mind_f((float)pow(10., (double)fg), kMaxSubgridFrac);
  }
  out[0] = out[1];                                                              // (g0/g1)^0
  out[4] = (float)(1.0 / (double)(gamma_dom(4) / gamma_dom(3)) * (double)out[3]);   // (g4/g3)^-1
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

__device__ void heat_cool_sg(ThermCell& c, const ThermConst& k, float nHe, float gamma_tot) {
  const float tm = maxd_f(kTempMin, c.temp);
  const float nt = c.nH + nHe;
  c.heat = (gamma_tot > 3e-14) ? (float)photoheat((double)tm, (double)nt, (double)c.nH, (double)nHe) : 0.f;
  float cool = 0.f;
  cool += rcrB_H2_d(tm) * nt * c.nH;
  cool += rcrB_He2_d(tm) * nt * nHe;
  const float nff = 1.f * nt;   // fion (nH + nHe)
  cool += free_free_d(tm) * ((double)nff * (double)nff);
  cool -= k.compton_d * nt * (2.726 * (1 + k.zz) - tm);
  c.cool = cool;
}

// update_thermal for one cell in the sub-grid model (gas_funcs.cc:362-418): neutral until
// ionised; an ionised cell's temperature is sub-cycled without the post-front heating of the
// plain model (set_Treion_default runs only without the sub-grid model)
__device__ void thermal_sg(ThermCell& c, const ThermConst& k, bool ionised, float nHe, float gamma_tot, float temp_0) {
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
    heat_cool_sg(c, k, nHe, gamma_tot);
    c.temp = (c.temp + 2. / 3. / kKB / c.n_tot * (c.heat - c.cool) * dt_temp) /
             (1. + 2. * (double)(k.hub2f * 0.5f) * dt_temp + 1. / c.n_tot * c.dne_dt * dt_temp -
              2. * (double)c.ddelta / 3. / (double)c.rho_rel * dt_temp);
    t_temp += dt_temp;
    ++guard;
  }
  c.temp = maxd_f(c.temp, kTempMin);
}

// One cell's last C2Ray iteration and thermal update in the sub-grid model (the sub-grid branch
// ray_tracing.cc:956-1071 with ifront = FALSE, the bookkeeping 1116-1209, gas_funcs.cc:362-418).
// Inputs: the cell's step-start state and its rate of this iteration; writes the dense state.
struct SgCell {
  long long gc;
  int box;
  float nH, nHe, nh1, nhe1;          // step start (the iteration-0 averages are these)
  float clump, temp, heat, cool, rec_h2, rec_he2, treion;
  bool flag;
  float gam, gam_he;                 // Gamma_HI, Gamma_HeI of the last iteration
};

template <bool THERMAL>
__device__ void finish_cell(const Dev& d, const SgCell& s) {
  const BoxP& B = d.box[s.box];
  const float dt = B.dt;
  bool flag = s.flag;
  float treion = s.treion;
  if (!flag && s.gam > 0.f) {   // first photons: the cell is ionised (ray_tracing.cc:964-970)
    treion = B.t - dt;
    flag = true;
  }
  float mfp = 0.f, mfp912 = 0.f;
  if (flag) eq_mfp(d, s.gam, s.clump, s.temp, s.nH, &mfp, &mfp912);
  // n_e of the iteration (ray_tracing.cc:949): the averages stay at their iteration-0 values
  const float nelec_f = s.nH - s.nh1 + s.nHe - s.nhe1;
  float nH1 = s.nh1, nHe1 = s.nhe1, nH2 = s.nH - s.nh1, nHe2 = s.nHe - s.nhe1, avg_he = s.nhe1;
  if (flag) {
    float fh[5];
    const float rho = d.rho[s.gc];
    fh1_interp(d, B, treion + d.sg_tinit, (float)((double)(rho / B.avg_rho) - 1.), B.t - treion, fh);
    nH1 = interp_nh1(fh, s.gam, s.nH, d.sg_fH1_0);
    nHe1 = nH1 * s.nHe / s.nH;
    avg_he = nHe1;
    nH2 = s.nH * 1.f;
    nHe2 = s.nHe * 1.f;
  }
  const float ne = nH2 + nHe2;
  const float n_tot = (float)(2. * (double)(s.nH + s.nHe));
  const float dne_dt = (-(s.nH + s.nHe) + (s.nH + s.nHe)) / dt;   // 0: the gas counts as ionised
  const long long gc = s.gc;
  d.nH1[gc] = nH1;
  d.nHe1[gc] = nHe1;
  d.avg_nh1[gc] = s.nh1;
  d.avg_nhe1[gc] = avg_he;
  d.f_H1[gc] = nH1 / s.nH;
  d.f_He1[gc] = nHe1 / s.nHe;
  d.ne[gc] = ne;
  // a neutral cell keeps the mean free path of its step-start gas (ray_tracing.cc:691)
  d.mfp[gc] = flag ? mfp : (float)(1. / (double)s.nh1 / d.sigH1_d[0]);
  if (flag) {
    if (!s.flag) {
      d.treion[gc] = treion;
      d.treion_flag[gc] = 1;
    }
  }
  if (d.outputs == FRT_OUT_DIAG) {
    const double nelec_d = (double)nelec_f;
    if (flag) d.mfp912[gc] = mfp912;
    d.rec_h2[gc] = s.rec_h2;
    d.rec_he2[gc] = s.rec_he2;
    d.recrate_h2[gc] = (float)((double)(s.clump * s.rec_h2) * nelec_d * (double)nH2);
    d.recrate_he2[gc] = (float)((double)(s.clump * s.rec_he2) * nelec_d * (double)nHe2);
    d.n_tot[gc] = n_tot;
    d.dne_dt[gc] = dne_dt;
    d.if_speed[gc] = 0.f;
    d.inc_flux[gc] = 0.f;
  }
  if (THERMAL) {
    ThermCell c;
    c.temp = s.temp;
    c.heat = s.heat;
    c.cool = s.cool;
    c.nH = s.nH;
    c.n_tot = n_tot;
    c.dne_dt = dne_dt;
    if (d.ddelta) {
      c.ddelta = d.ddelta[gc];
      c.rho_rel = d.rho[gc] / B.avg_rho;
    }
    thermal_sg(c, B.th, flag, s.nHe, s.gam, d.sg_temp0);
    d.temp[gc] = c.temp;
    if (flag) {
      d.heat[gc] = c.heat;
      d.cool[gc] = c.cool;
    }
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
        gh_sum += gh;
        ghe_sum += ghe;
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
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int gc = d.l_cell[s];
    const float2 acc = d.l_acc[s];
    if (!LAST) {
      if (d.treion_flag[gc]) {
        float mfp, m912;
        eq_mfp(d, acc.x, d.clump ? d.clump[gc] : d.const_clump, d.temp[gc], d.l_nh[s], &mfp, &m912);
        d.l_mfp[s] = mfp;
      }
      d.l_acc[s] = make_float2(0.f, 0.f);
      continue;
    }
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
    thermal_sg(c, B.th, flag, nHe, gam, d.sg_temp0);
    d.temp[gc] = c.temp;
    if (flag) {
      d.heat[gc] = c.heat;
      d.cool[gc] = c.cool;
    }
  }
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

}  // namespace frt
