// Physics kernels of the RT step: the C2Ray iteration (ray pass with Gamma deposition and the
// cell update, ray_tracing.cc:623-1216) and the thermal update (gas_funcs.cc:362-457).
//
// Work split. A cell that no ray segment touches in a step receives Gamma = 0 in all C2Ray
// iterations, so its whole step -- 5 C2Ray updates, the last-iteration bookkeeping and the
// sub-cycled thermal update -- depends only on its own state. k_dark does that whole step for
// every such cell in one streaming pass over HBM (read the state once, write it once). Cells
// touched by at least one segment ("lit") are gathered into a compact list; only they go
// through the iteration with the ray passes in between (k_lit_init, k_raypass, k_litpass).
// Both paths call the same per-cell device functions (frt_physics.cuh), so a cell gets the same
// arithmetic whichever path handles it.
#include <limits.h>
#include <math.h>

#include "frt_internal.cuh"

namespace frt {

namespace {

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

__device__ __forceinline__ int box_of_cell(const Dev& d, long long gc) { return d.tile_box[gc >> kTileShift]; }

// The density-change term of the temperature equation: d(delta)/dt and rho / <rho> of a cell
// (gas_funcs.cc:399), present once a second hydro snapshot has been read.
__device__ __forceinline__ void density_change(const Dev& d, const BoxP& B, long long gc, ThermCell* c) {
  if (d.ddelta) {
    c->ddelta = d.ddelta[gc];
    c->rho_rel = d.rho[gc] / B.avg_rho;
  }
}

// 1 - e^-x and e^-x of one optical depth x >= 0 (xl = x log2(e)). Below x = 1/4 the absorbed
// part is the Taylor series of 1 - e^-x = x - x^2/2! + x^3/3! - ... to the x^6 term (alternating
// with decreasing terms: truncation below 0.25^6/7! ~ 5e-8 relative) and the transmission is
// 1 - a (>= 0.77); above, the transmission is 2^-xl and the absorbed part 1 - e (e <= 0.78,
// so the subtraction costs under 3 bits). Both forms are evaluated and one is selected, so the
// lanes of a warp never split on the optical depth.
__device__ __forceinline__ float ex2_approx(float x) {   // 2^x, hardware approximation (~2 ulp), flushes tiny results to 0
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ void absorb_transmit(float x, float xl, float* a, float* e) {
  const float ex = ex2_approx(-xl);
  float p = fmaf(x, -1.0f / 720.0f, 1.0f / 120.0f);
  p = fmaf(p, x, -1.0f / 24.0f);
  p = fmaf(p, x, 1.0f / 6.0f);
  p = fmaf(p, x, -0.5f);
  p = fmaf(p, x, 1.0f);
  const float at = x * p;
  const bool small = x <= 0.25f;
  *a = small ? at : 1.0f - ex;
  *e = small ? 1.0f - at : ex;
}

// ---- clear the previous step's lit marks ------------------------------------------------
__global__ void k_clear_lit(Dev d) {
  const int n = min(d.ctl->n_lit, d.lit_cap);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int gc = d.l_cell[s];
    d.lit_flag[gc] = 0;
    d.lit_slot[gc] = -1;
  }
}

// ---- iteration-0 set-up of the lit cells (ray_tracing.cc:630-697, iter == 0) --------------
template <bool STRICT>
__global__ void k_lit_init(Dev d) {
  const int n = min(d.ctl->n_lit, d.lit_cap);
  const int F = d.F, L = d.lit_cap;
  // the ray passes of this step start with empty work queues
  if (blockIdx.x == 0 && threadIdx.x < kMaxIterQueue) d.rp_queue[threadIdx.x] = 0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int gc = d.l_cell[s];
    // every load of the cell first, then the stores (the loads overlap)
    const int bx = box_of_cell(d, gc);
    const float temp = d.temp[gc];
    const float cl = d.clump ? d.clump[gc] : d.const_clump;
    const float nh = d.nH[gc], nhe = d.nHe[gc], y0h = d.f_H1[gc], y0he = d.f_He1[gc];
    const float nh1 = d.nH1[gc], nhe1 = d.nHe1[gc];
    float rh, rhe;
    recomb_coeffs<STRICT>(temp, &rh, &rhe);
    d.l_box[s] = (uint16_t)bx;
    d.l_nh[s] = nh;
    d.l_nhe[s] = nhe;
    d.l_y0h[s] = y0h;
    d.l_y0he[s] = y0he;
    d.l_rec_h2[s] = rh;
    d.l_rec_he2[s] = rhe;
    d.l_crec_h[s] = cl * rh;
    d.l_crec_he[s] = cl * rhe;
    d.l_avg[s] = make_float2(nh1, nhe1);
    d.l_nh1_old[s] = nh1;
    d.l_acc[s] = make_float2(0.f, 0.f);
    d.l_heat[s] = make_float2(0.f, 0.f);
    if (STRICT || d.per_bin)
      for (int nu = 0; nu < F; nu++) {
        d.l_ngam[(size_t)nu * L + s] = 0.f;
        d.l_acc_nu_h[(size_t)nu * L + s] = 0.f;
        d.l_acc_nu_he[(size_t)nu * L + s] = 0.f;
      }
  }
}

// ---- ray pass of one C2Ray iteration (ray_tracing.cc:701-938), plain mode ------------------
// The moved rays walk their packed segments (k_advance and k_pk_slots: lit slot + path length,
// in moved-list order), attenuate the photon count per bin with the current time-averaged neutral densities of
// the lit cells, and deposit Gamma_HI / HeI; LAST also writes the per-bin output fields (diag),
// the new photon counts, and removes rays below nphot_min.

// Strict precision: the reference's double expressions, one thread per moved ray.
template <bool LAST>
__global__ void __launch_bounds__(256) k_raypass_strict(Dev d) {
  const int nmv = min((int)(d.ctl->mv_seg >> 32), d.ray_cap);
  const RayPool A = d.pool[d.ctl->cur];
  const int cap = d.ray_cap, F = d.F, L = d.lit_cap;
  double dep = 0.0, kil = 0.0, ovl = 0.0;
  long long nkill = 0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nmv; q += gridDim.x * blockDim.x) {
    const int4 hd = d.mv_hdr[q];
    const int i = hd.x, ns = hd.z;
    const int2* sp = d.pk + hd.y;
    const BoxP& B = d.box[hd.w];
    const double nmin = B.nphot_min;
    float nph[FRT_MAX_FREQ];
    for (int nu = 0; nu < F; nu++) nph[nu] = A.nphot[(size_t)nu * cap + i];
    bool dumped = false;
    unsigned dump_mask = 0;
    double tau_h1[FRT_MAX_FREQ], tau_he1[FRT_MAX_FREQ];
    for (int nu = 0; nu < F; nu++) { tau_h1[nu] = 0.; tau_he1[nu] = 0.; }
    const double dt = B.dt, vol = B.vol;
    double colh = 0.0, colhe = 0.0;   // optical-depth limit: this pass's columns
    for (int p = 0; p < ns; p++) {
      const int2 sg = sp[p];
      const int slot = sg.x;
      if (slot < 0) continue;
      const float dist = __int_as_float(sg.y & 0x7fffffff);
      const float2 av = d.l_avg[slot];
      const float a = av.x, b = av.y;
      colh += (double)a * (double)dist;
      colhe += (double)b * (double)dist;
      double dth[FRT_MAX_FREQ], dthe[FRT_MAX_FREQ], nin[FRT_MAX_FREQ];
      double total = 0.;
      for (int nu = 0; nu < F; nu++) {
        dth[nu] = a * d.sigH1_d[nu] * dist;
        dthe[nu] = b * d.sigHe1_d[nu] * dist;
        nin[nu] = (nph[nu] * kPhotNorm) * exp(-tau_h1[nu] - tau_he1[nu]);
        total += nin[nu] / kPhotNorm;
      }
      const bool dump = total < nmin;
      for (int nu = 0; nu < F; nu++) {
        double fh = 0., fhe = 0.;
        if ((dth[nu] > 0.) || (dthe[nu] > 0.)) {
          const double den = (1. - exp(-dth[nu])) * exp(-dthe[nu]) + (1. - exp(-dthe[nu])) * exp(-dth[nu]);
          fh = (1. - exp(-dth[nu])) * exp(-dthe[nu]) / den;
          fhe = (1. - exp(-dthe[nu])) * exp(-dth[nu]) / den;
        }
        const double absb = dump ? 1.0 : (1. - exp(-dth[nu] - dthe[nu]));
        const float gh = (float)(fh * nin[nu] * absb / dt / vol / a);
        const float ghe = (float)(fhe * nin[nu] * absb / dt / vol / b);
        atomicAdd(&d.l_acc[slot], make_float2(gh, ghe));
        if (LAST) {
          atomicAdd(&d.l_ngam[(size_t)nu * L + slot], (float)(nin[nu] / kPhotNorm));
          atomicAdd(&d.l_acc_nu_h[(size_t)nu * L + slot], gh);
          atomicAdd(&d.l_acc_nu_he[(size_t)nu * L + slot], ghe);
          dep += (fh + fhe) * nin[nu] * absb / kPhotNorm;
          if (dump && (fh + fhe) > 0.) dump_mask |= 1u << nu;
        }
        tau_h1[nu] += dth[nu];
        tau_he1[nu] += dthe[nu];
      }
      if (dump) { dumped = true; break; }
    }
    if (LAST) {
      float s = 0.f;
      for (int nu = 0; nu < F; nu++) {
        nph[nu] = (float)((nph[nu] * kPhotNorm) * exp(-tau_h1[nu] - tau_he1[nu]) / kPhotNorm);
        A.nphot[(size_t)nu * cap + i] = nph[nu];
        s += nph[nu];
      }
      bool tau_over = false;
      if (A.col) {   // the optical-depth limit (opt-in)
        const double nh = A.col[i] + colh, nhe = A.col[(size_t)cap + i] + colhe;
        A.col[i] = nh;
        A.col[(size_t)cap + i] = nhe;
        double tmin = 1e300;
        for (int nu = 0; nu < F; nu++) tmin = fmin(tmin, d.sigH1_d[nu] * nh + d.sigHe1_d[nu] * nhe);
        tau_over = d.tau_max > 0.0 && tmin > d.tau_max;
      }
      if (!(s > nmin) || tau_over) {
        d.dead[i] = 1;
        nkill += 1;
        kil += (double)s;
        if (dumped)
          for (int nu = 0; nu < F; nu++)
            if (dump_mask & (1u << nu)) ovl += (double)nph[nu];
      }
    }
  }
  if (LAST) {
    dep = block_sum(dep);
    kil = block_sum(kil);
    ovl = block_sum(ovl);
    nkill = block_sum(nkill);
    if (threadIdx.x == 0) {
      if (dep != 0.0) atomicAdd(&d.ctl->deposited, dep * kPhotNorm);
      if (kil != 0.0) atomicAdd(&d.ctl->killed_ph, kil * kPhotNorm);
      if (ovl != 0.0) atomicAdd(&d.ctl->overlap, ovl * kPhotNorm);
      if (nkill) atomicAdd((unsigned long long*)&d.ctl->killed, (unsigned long long)nkill);
    }
  }
}

// Mixed precision, persistent lanes. Rays have 1..path_length segments, so one ray per thread
// leaves most lanes of a warp idle behind its longest ray. Here a lane takes the next ray of its
// warp's share of the moved list as soon as its own ray ends (a ballot and a warp-uniform
// cursor), so every lane walks a segment in every loop trip. The warp's share is either a static
// contiguous slice of the moved list (chunk = 0: no atomics) or a sequence of chunks of `chunk`
// rays taken from a device-side queue (queue[iter], one atomicAdd per chunk by lane 0), which
// evens out warps whose rays happen to be long; the autotuner picks between them. A
// ray's header (pool index, packed segments, count, box) is one 16-byte load and its segments are
// contiguous; the loads run two segments ahead of the arithmetic (the next segment's cell state,
// the segment after it), so a lane's gathers are in flight while it works the current segment.
// Per bin the photon count is carried from segment to segment by its transmission e^-dtau, and
// each bin costs one exp2 when HeI does not absorb there (sigma_HeI = 0 below 24.59 eV) and two
// when it does.
// NF > 0 fixes the number of frequency bins at compile time (the 5-bin spectrum of every
// configuration here), so the per-bin loops unroll exactly; NF = 0 takes d.F at run time.
// CHUNKED compiles the queue form; the static-slice form carries none of its bookkeeping. The
// minimum resident blocks keep the last pass (which also writes the rays' photon counts and
// the heating pairs) at 64 registers, four 256-thread blocks per SM, and the middle passes at
// 40 registers, six blocks per SM (48 warps to cover the lit-cell gathers; 0.246 against 0.255 ms
// per pass at L with five).
// NHO > 0 declares the first NHO bins below the HeI edge (sigma_HeI = 0 there, as in the 5-bin
// spectrum, whose lowest three bins lie below 24.59 eV): those bins skip the HeI optical depth and
// the H/He split, which give frac_h1 = 1 (or 0 where dtau_HI = 0) and frac_he1 = 0 for them.
// TAU (last pass, optical-depth limit on) sums each ray's HI and HeI columns over its segments in
// FP64 (exact products of the float density and path), adds them to the ray's columns and removes
// the ray once its optical depth exceeds d.tau_max in every bin.
template <bool LAST, int NF, bool CHUNKED, int NHO = 0, bool TAU = false>
__global__ void __launch_bounds__(256, LAST ? 4 : 6) k_raypass_mixed(Dev d, int iter, int chunk) {
  constexpr int MAXF = NF > 0 ? NF : FRT_MAX_FREQ;
  constexpr unsigned FULL = 0xffffffffu;
  const int Fr = NF > 0 ? NF : d.F;
  const int nmv = min((int)(d.ctl->mv_seg >> 32), d.ray_cap);
  const RayPool A = d.pool[d.ctl->cur];
  const int cap = d.ray_cap, L = d.lit_cap;
  const int lane = threadIdx.x & 31;
  const unsigned lanes_below = (1u << lane) - 1u;
  // this warp's current share [cursor, slice_end) of the moved list: its static slice, or (chunked
  // queue) empty until the first chunk is taken
  long long cursor = 0, slice_end = 0;
  bool queue_done = false;
  int* queue = d.rp_queue + (iter < kMaxIterQueue ? iter : kMaxIterQueue - 1);
  if (!CHUNKED) {
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    const long long wid = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const long long per = (nmv + nwarps - 1) / nwarps;
    cursor = wid * per;
    slice_end = min((long long)nmv, cursor + per);
    queue_done = true;
  }
  double dep = 0.0, kil = 0.0, ovl = 0.0;
  long long nkill = 0;
  int i = -1, p = 0, ns = 0;
  bool exhausted = false, dumped = false;
  unsigned dump_mask = 0;
  float nin[MAXF];
#pragma unroll
  for (int nu = 0; nu < MAXF; nu++) nin[nu] = 0.f;
  float kdep = 0.f, nmin_ru = 0.f, nmin_rd = 0.f;
  double colh = 0.0, colhe = 0.0;   // TAU: this pass's columns of the current ray
  const int2* sp = nullptr;
  int2 sg0 = make_int2(-1, 0), sg1 = make_int2(-1, 0);   // segments p and p + 1
  float2 av0 = make_float2(0.f, 0.f);                     // cell state of segment p
  while (true) {
    // refill the lanes whose ray ended
    const bool need = (i < 0) && !exhausted;
    const unsigned m = __ballot_sync(FULL, need);
    if (CHUNKED && m && cursor >= slice_end && !queue_done) {
      // the warp's chunk is used up: take the next one from the queue
      int base = 0;
      if (lane == 0) base = atomicAdd(queue, chunk);
      base = __shfl_sync(FULL, base, 0);
      if (base >= nmv) {
        queue_done = true;
      } else {
        cursor = base;
        slice_end = min((long long)nmv, (long long)base + chunk);
      }
    }
    if (m) {
      const long long q = cursor + __popc(m & lanes_below);
      cursor = CHUNKED ? min(cursor + __popc(m), max(cursor, slice_end)) : cursor + __popc(m);
      if (need) {
        if (q < slice_end) {
          const int4 hd = d.mv_hdr[q];
          i = hd.x;
          sp = d.pk + hd.y;
          ns = hd.z;
          p = 0;
          dumped = false;
          colh = colhe = 0.0;
          dump_mask = 0;
          const BoxP& B = d.box[hd.w];
          kdep = B.kdep_f;
          nmin_ru = B.nmin_ru;   // the photon threshold as float bounds (k_step_begin)
          nmin_rd = B.nmin_rd;
          sg0 = sp[0];
          sg1 = (ns > 1) ? sp[1] : make_int2(-1, 0);
#pragma unroll
          for (int nu = 0; nu < MAXF; nu++) nin[nu] = (nu < Fr) ? A.nphot[(size_t)nu * cap + i] : 0.f;
          av0 = (sg0.x >= 0 && sg0.x < L) ? d.l_avg[sg0.x] : make_float2(0.f, 0.f);
        } else if (!CHUNKED || queue_done) {
          exhausted = true;   // (a lane short of a chunk's remainder asks again next trip)
        }
      }
    }
    if (__all_sync(FULL, i < 0)) break;
    if (i < 0) continue;
    // one segment of ray i; the loads of the next two are issued first
    const int2 sg = sg0;
    const float2 av = av0;
    bool done = (p + 1 >= ns);
    {
      float2 av_n = make_float2(0.f, 0.f);
      if (!done && sg1.x >= 0 && sg1.x < L) av_n = d.l_avg[sg1.x];
      int2 sg_n = make_int2(-1, 0);
      if (p + 2 < ns) sg_n = sp[p + 2];
      sg0 = sg1;
      av0 = av_n;
      sg1 = sg_n;
    }
    const int slot = sg.x;
    if (slot >= 0 && slot < L) {
      const float dist = __int_as_float(sg.y & 0x7fffffff);
      const float a = av.x, b = av.y;
      if (TAU) {
        colh += (double)a * (double)dist;
        colhe += (double)b * (double)dist;
      }
      float total = 0.f;
#pragma unroll
      for (int nu = 0; nu < MAXF; nu++) total += (nu < Fr) ? nin[nu] : 0.f;
      const bool dump = total < nmin_ru;
      const float ad = a * dist, bd = b * dist;   // column densities of the segment
      float gsum_h = 0.f, gsum_he = 0.f, hh = 0.f, hhe = 0.f;
#pragma unroll
      for (int nu = 0; nu < MAXF; nu++) {
        if (nu >= Fr) continue;
        const float dth = ad * d.sigH1_f[nu];
        float ah, eh;
        absorb_transmit(dth, ad * d.sigH1_l2[nu], &ah, &eh);
        if (nu < NHO) {   // HI alone absorbs in this bin
          const float gh = (dth > 0.f) ? nin[nu] * (dump ? 1.0f : ah) : 0.f;
          gsum_h += gh;
          if (LAST) {
            hh += gh * d.cH1_f[nu];
            if (d.per_bin) {
              atomicAdd(&d.l_ngam[(size_t)nu * L + slot], nin[nu]);
              if (gh != 0.f) atomicAdd(&d.l_acc_nu_h[(size_t)nu * L + slot], gh * __fdividef(kdep, a));
            }
            if (dump && dth > 0.f) dump_mask |= 1u << nu;
          }
          nin[nu] *= eh;
          continue;
        }
        const float dthe = bd * d.sigHe1_f[nu];
        float fh, fhe, absb, e;
        if (dthe > 0.f) {
          float ahe, ehe;
          absorb_transmit(dthe, bd * d.sigHe1_l2[nu], &ahe, &ehe);
          e = eh * ehe;
          absb = ah + eh * ahe;                   // 1 - e^-(dth+dthe) without cancellation
          // frac_h1 = A e^-b / (A e^-b + B e^-a) (ray_tracing.cc:770-771)
          const float x1 = ah * ehe, x2 = ahe * eh;
          if (x1 + x2 > 1e-30f) {
            const float inv = __fdividef(1.0f, x1 + x2);
            fh = x1 * inv;
            fhe = x2 * inv;
          } else if (dth >= dthe) {                // both optical depths huge: ratio form
            const float r = __fdividef(ahe, ah) * expf(dthe - dth);
            fh = __fdividef(1.0f, 1.0f + r);
            fhe = r * fh;
          } else {
            const float r = __fdividef(ah, ahe) * expf(dth - dthe);
            fhe = __fdividef(1.0f, 1.0f + r);
            fh = r * fhe;
          }
        } else {
          e = eh;
          absb = ah;
          fh = (dth > 0.f) ? 1.0f : 0.0f;           // frac_h1 = 1, frac_he1 = 0 when dtau_he1 = 0
          fhe = 0.f;
        }
        const float qv = nin[nu] * (dump ? 1.0f : absb);
        const float gh = fh * qv, ghe = fhe * qv;
        gsum_h += gh;
        gsum_he += ghe;
        if (LAST) {
          hh += gh * d.cH1_f[nu];
          hhe += ghe * d.cHe1_f[nu];
          if (d.per_bin) {   // per-bin rates and photon counts: output fields (diag outputs)
            const float wh_ = __fdividef(kdep, a), whe_ = __fdividef(kdep, b);
            atomicAdd(&d.l_ngam[(size_t)nu * L + slot], nin[nu]);
            if (gh != 0.f) atomicAdd(&d.l_acc_nu_h[(size_t)nu * L + slot], gh * wh_);
            if (ghe != 0.f) atomicAdd(&d.l_acc_nu_he[(size_t)nu * L + slot], ghe * whe_);
          }
          if (dump && (fh + fhe) > 0.f) dump_mask |= 1u << nu;
        }
        nin[nu] *= e;
      }
      // absorbed photons of the crossing; k_litpass applies the rate weight kdep / <n> per cell
      if (gsum_h != 0.f || gsum_he != 0.f) atomicAdd(&d.l_acc[slot], make_float2(gsum_h, gsum_he));
      if (LAST) {
        // photo-heating weights sum_nu Gamma_nu h (h_eV nu - Eth)/h_eV (gas_funcs.cc:155-158)
        if (hh != 0.f || hhe != 0.f) atomicAdd(&d.l_heat[slot], make_float2(hh, hhe));
        dep += (double)gsum_h + (double)gsum_he;
      }
      if (dump) {
        dumped = true;
        done = true;
      }
    }
    ++p;
    if (done) {
      if (LAST) {
        // the photons leaving the last walked segment become the ray's count
        // (ray_tracing.cc:923-935); below nphot_min the ray is removed
        float s = 0.f;
#pragma unroll
        for (int nu = 0; nu < MAXF; nu++) {
          if (nu >= Fr) continue;
          A.nphot[(size_t)nu * cap + i] = nin[nu];
          s += nin[nu];
        }
        bool tau_over = false;
        if (TAU) {
          const double nh = A.col[i] + colh, nhe = A.col[(size_t)cap + i] + colhe;
          A.col[i] = nh;
          A.col[(size_t)cap + i] = nhe;
          double tmin = 1e300;
          for (int nu = 0; nu < Fr; nu++) tmin = fmin(tmin, d.sigH1_d[nu] * nh + d.sigHe1_d[nu] * nhe);
          tau_over = tmin > d.tau_max;
        }
        if (!(s > nmin_rd) || tau_over) {
          d.dead[i] = 1;
          nkill += 1;
          kil += (double)s;
          if (dumped)
#pragma unroll
            for (int nu = 0; nu < MAXF; nu++)
              if (nu < Fr && (dump_mask & (1u << nu))) ovl += (double)nin[nu];
        }
      }
      i = -1;
    }
  }
  if (LAST) {
    dep = block_sum(dep);
    kil = block_sum(kil);
    ovl = block_sum(ovl);
    nkill = block_sum(nkill);
    if (threadIdx.x == 0) {
      if (dep != 0.0) atomicAdd(&d.ctl->deposited, dep * kPhotNorm);
      if (kil != 0.0) atomicAdd(&d.ctl->killed_ph, kil * kPhotNorm);
      if (ovl != 0.0) atomicAdd(&d.ctl->overlap, ovl * kPhotNorm);
      if (nkill) atomicAdd((unsigned long long*)&d.ctl->killed, (unsigned long long)nkill);
    }
  }
}

// ---- the last-iteration bookkeeping of one cell (ray_tracing.cc:1116-1209) -----------------
struct Final {
  float nH1, nHe1, nH2, nHe2, ne, n_tot, dne_dt, f_H1, f_He1, f_H2;
  bool set_treion;
};

// Mixed precision takes the fractions and dn_e/dt with the fast division (2 ulp); the ratio
// that decides the reionisation flag keeps the correctly rounded one.
template <bool STRICT>
__device__ __forceinline__ Final finalize(float nH, float nHe, float nh1_end, float nhe1_end, float avg_h, float ne_old,
                                          float dt, bool flag) {
  Final f;
  f.nH1 = nh1_end;
  f.nH2 = nH - f.nH1;
  f.nHe1 = nhe1_end;
  f.nHe2 = nHe - f.nHe1;
  f.set_treion = (avg_h / nH < 0.5) && !flag;
  f.ne = (float)((double)(f.nH2 + f.nHe2) + 2. * 0.0);
  f.n_tot = nH + nHe + f.ne;
  if (STRICT) {
    f.dne_dt = (-ne_old + f.ne) / dt;
    f.f_H2 = f.nH2 / nH;
    f.f_H1 = f.nH1 / nH;
    f.f_He1 = f.nHe1 / nHe;
  } else {
    f.dne_dt = __fdividef(-ne_old + f.ne, dt);
    const float inv_nh = __fdividef(1.0f, nH);
    f.f_H2 = f.nH2 * inv_nh;
    f.f_H1 = f.nH1 * inv_nh;
    f.f_He1 = __fdividef(f.nHe1, nHe);
  }
  return f;
}

// ---- cell pass of one C2Ray iteration over the lit cells ----------------------------------
// Lit cells [s_begin, min(s_end, n_lit)) (the autotuner times launch shapes on shares of one
// pass's cells; the step launches them all).
template <bool STRICT, bool LAST, bool THERMAL>
__global__ void __launch_bounds__(256) k_litpass(Dev d, int s_begin, int s_end) {
  const int n = min(min(d.ctl->n_lit, d.lit_cap), s_end);
  const int L = d.lit_cap;
  const bool diag = d.outputs == FRT_OUT_DIAG;
  for (int s = s_begin + blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const BoxP& B = d.box[d.l_box[s]];
    const int gc = LAST ? d.l_cell[s] : 0;   // the middle passes touch only the lit arrays
    const float dt = B.dt;
    const float2 acc = d.l_acc[s], av = d.l_avg[s];
    const float a_prev = av.x, b_prev = av.y;
    // the last pass's dense-cell inputs, loaded before any store so that all loads overlap
    bool flag = false;
    float ne_old = 0.f, nh1_old = 0.f, t_old = 0.f, heat_old = 0.f, cool_old = 0.f;
    float2 ht = make_float2(0.f, 0.f);
    if (LAST) {
      flag = d.treion_flag[gc] != 0;
      ne_old = d.ne[gc];
      nh1_old = d.l_nh1_old[s];
      if (!STRICT) ht = d.l_heat[s];
      if (THERMAL) {
        t_old = d.temp[gc];
        heat_old = d.heat[gc];
        cool_old = d.cool[gc];
      }
    }
    // mixed precision: the ray pass sums the absorbed photons of a cell's crossings and the rate
    // weight kdep / <n> (ray_tracing.cc:787-790), the same for every crossing of the cell in this
    // iteration, is applied here once (strict: the ray pass deposits the reference's rates)
    float g = acc.x, ghe = acc.y;
    float wh = 0.f, whe = 0.f;
    if (!STRICT) {
      wh = __fdividef(B.kdep_f, a_prev);
      whe = __fdividef(B.kdep_f, b_prev);
      g = (acc.x != 0.f) ? acc.x * wh : 0.f;
      ghe = (acc.y != 0.f) ? acc.y * whe : 0.f;
    }
    const float nH = d.l_nh[s], nHe = d.l_nhe[s];
    const float nelec_f = nH - a_prev + nHe - b_prev;
    const double nelec_d = (double)nelec_f;
    const C2Species H{nH, d.l_y0h[s], d.l_crec_h[s]};
    const C2Species He{nHe, d.l_y0he[s], d.l_crec_he[s]};
    float nh1_end = 0.f, nhe1_end = 0.f;
    const float a_new = c2ray_species<STRICT>(H, g, nelec_d, nelec_f, a_prev, dt, LAST, &nh1_end);
    const float b_new = c2ray_species<STRICT>(He, ghe, nelec_d, nelec_f, b_prev, dt, LAST, &nhe1_end);
    if (!LAST) {
      d.l_avg[s] = make_float2(a_new, b_new);
      d.l_acc[s] = make_float2(0.f, 0.f);
      continue;
    }
    if (!STRICT) {
      // the step's outputs keep the rates: Gamma and the bin-weighted heating sums, weighted
      ht = make_float2((ht.x != 0.f) ? ht.x * wh : 0.f, (ht.y != 0.f) ? ht.y * whe : 0.f);
      d.l_acc[s] = make_float2(g, ghe);
      d.l_heat[s] = ht;
    }
    const Final f = finalize<STRICT>(nH, nHe, nh1_end, nhe1_end, a_new, ne_old, dt, flag);
    if (f.set_treion) {
      d.treion[gc] = B.t;
      d.treion_flag[gc] = 1;
    }
    d.nH1[gc] = f.nH1;
    d.nHe1[gc] = f.nHe1;
    d.f_H1[gc] = f.f_H1;
    d.f_He1[gc] = f.f_He1;
    d.ne[gc] = f.ne;
    d.avg_nh1[gc] = a_new;
    d.avg_nhe1[gc] = b_new;
    if (diag) {
      d.mfp[gc] = (float)(1. / d.sigH1_0 / (double)a_prev);
      d.mfp912[gc] = (float)(1. / d.sigH1_912 / (double)a_prev);
      d.rec_h2[gc] = d.l_rec_h2[s];
      d.rec_he2[gc] = d.l_rec_he2[s];
      d.recrate_h2[gc] = (float)((double)d.l_crec_h[s] * nelec_d * (double)f.nH2);
      d.recrate_he2[gc] = (float)((double)d.l_crec_he[s] * nelec_d * (double)f.nHe2);
      d.n_tot[gc] = f.n_tot;
      d.dne_dt[gc] = f.dne_dt;
    }
    if (THERMAL) {
      ThermCell c;
      c.temp = t_old;
      c.heat = heat_old;
      c.cool = cool_old;
      c.nH = nH;
      c.nH1 = f.nH1;
      c.nH1_prev = nh1_old;
      c.nH2 = f.nH2;
      c.nHe2 = f.nHe2;
      c.ne = f.ne;
      c.n_tot = f.n_tot;
      c.dne_dt = f.dne_dt;
      c.f_H2 = f.f_H2;
      c.avg_nh1 = a_new;
      c.avg_nhe1 = b_new;
      HeatSrc hs{d.l_acc_nu_h + s, d.l_acc_nu_he + s, L, 0.f, 0.f, 1};
      if (!STRICT && !d.per_bin) {
        hs.mode = 2;
        hs.hh = ht.x;
        hs.hhe = ht.y;
      }
      density_change(d, B, gc, &c);
      thermal_update<STRICT>(c, B.th, hs, d.F, d.nhe_to_nh);
      d.temp[gc] = c.temp;
      d.heat[gc] = c.heat;
      d.cool[gc] = c.cool;
      if (diag) {
        d.if_speed[gc] = c.if_speed;
        d.inc_flux[gc] = c.inc_flux;
      }
    } else {
      d.nH1_prev[gc] = nh1_old;
      d.n_tot[gc] = f.n_tot;
      d.dne_dt[gc] = f.dne_dt;
    }
  }
}

// ---- whole step of the cells no ray touched -----------------------------------------------
// 5 C2Ray updates with Gamma = 0 (ray_tracing.cc:941-1136), the last-iteration bookkeeping
// (1138-1209) and, when THERMAL, update_thermal (gas_funcs.cc:362-411), all in registers.
template <bool STRICT, bool THERMAL>
__global__ void __launch_bounds__(256, 4) k_dark(Dev d) {
  const long long ncell = d.ncell_total;
  const bool diag = d.outputs == FRT_OUT_DIAG;
  const int I = d.itercount;
  for (long long gc = blockIdx.x * (long long)blockDim.x + threadIdx.x; gc < ncell;
       gc += (long long)gridDim.x * blockDim.x) {
    const int b = box_of_cell(d, gc);
    if (b < 0) continue;   // padding between boxes
    // every input of the cell is requested together with its lit flag (one round trip to memory
    // instead of two; a lit cell's sectors are read for the dark cells beside it anyway), and
    // all before any store
    const uint8_t lit = d.lit_flag[gc];
    const float nH = d.nH[gc], nHe = d.nHe[gc];
    const float nh1 = d.nH1[gc], nhe1 = d.nHe1[gc];
    const float temp0 = d.temp[gc];
    const float cl = d.clump ? d.clump[gc] : d.const_clump;
    const bool flag = d.treion_flag[gc] != 0;
    const float ne_old = d.ne[gc];
    const float heat_old = THERMAL ? d.heat[gc] : 0.f, cool_old = THERMAL ? d.cool[gc] : 0.f;
    const float y0h = d.f_H1[gc], y0he = d.f_He1[gc];
    if (lit) continue;
    const BoxP& B = d.box[b];
    if (gc - B.cell0 >= B.ncell) continue;
    const float dt = B.dt;
    float rh, rhe;
    recomb_coeffs<STRICT>(temp0, &rh, &rhe);
    const C2Species H{nH, y0h, cl * rh};
    const C2Species He{nHe, y0he, cl * rhe};
    float a = nh1, bb = nhe1, a_prev = nh1;
    float nh1_end = 0.f, nhe1_end = 0.f;
    double nelec_last = 0.0;
    for (int it = 0; it < I; it++) {
      const bool last = (it == I - 1);
      const float nelec_f = nH - a + nHe - bb;
      const double nelec_d = (double)nelec_f;
      a_prev = a;
      const float an = c2ray_species<STRICT, true>(H, 0.f, nelec_d, nelec_f, a, dt, last, &nh1_end);
      const float bn = c2ray_species<STRICT, true>(He, 0.f, nelec_d, nelec_f, bb, dt, last, &nhe1_end);
      // An update is a function of (a, bb) alone (Gamma = 0). When it returns its own input, every
      // later iteration repeats it bit for bit, so go straight to the last one (which also forms
      // the end-of-step densities) -- the usual case of a neutral cell after one or two updates.
      if (!last && an == a && bn == bb) it = I - 2;
      a = an;
      bb = bn;
      nelec_last = nelec_d;
    }
    const Final f = finalize<STRICT>(nH, nHe, nh1_end, nhe1_end, a, ne_old, dt, flag);
    if (f.set_treion) {
      d.treion[gc] = B.t;
      d.treion_flag[gc] = 1;
    }
    d.nH1[gc] = f.nH1;
    d.nHe1[gc] = f.nHe1;
    d.f_H1[gc] = f.f_H1;
    d.f_He1[gc] = f.f_He1;
    d.ne[gc] = f.ne;
    d.avg_nh1[gc] = a;
    d.avg_nhe1[gc] = bb;
    if (diag) {
      d.mfp[gc] = (float)(1. / d.sigH1_0 / (double)a_prev);
      d.mfp912[gc] = (float)(1. / d.sigH1_912 / (double)a_prev);
      d.rec_h2[gc] = rh;
      d.rec_he2[gc] = rhe;
      d.recrate_h2[gc] = (float)((double)(cl * rh) * nelec_last * (double)f.nH2);
      d.recrate_he2[gc] = (float)((double)(cl * rhe) * nelec_last * (double)f.nHe2);
      d.n_tot[gc] = f.n_tot;
      d.dne_dt[gc] = f.dne_dt;
    }
    if (THERMAL) {
      ThermCell c;
      c.temp = temp0;
      c.heat = heat_old;
      c.cool = cool_old;
      c.nH = nH;
      c.nH1 = f.nH1;
      c.nH1_prev = nh1;
      c.nH2 = f.nH2;
      c.nHe2 = f.nHe2;
      c.ne = f.ne;
      c.n_tot = f.n_tot;
      c.dne_dt = f.dne_dt;
      c.f_H2 = f.f_H2;
      c.avg_nh1 = a;
      c.avg_nhe1 = bb;
      const HeatSrc hs{nullptr, nullptr, 0, 0.f, 0.f, 0};
      density_change(d, B, gc, &c);
      thermal_update<STRICT>(c, B.th, hs, d.F, d.nhe_to_nh);
      d.temp[gc] = c.temp;
      d.heat[gc] = c.heat;
      d.cool[gc] = c.cool;
      if (diag) {
        d.if_speed[gc] = c.if_speed;
        d.inc_flux[gc] = c.inc_flux;
      }
    } else {
      d.nH1_prev[gc] = nh1;
      d.n_tot[gc] = f.n_tot;
      d.dne_dt[gc] = f.dne_dt;
    }
  }
}

// ---- update_thermal over all cells (the unfused call sequence) ----------------------------
template <bool STRICT>
__global__ void __launch_bounds__(256) k_thermal_all(Dev d) {
  const long long ncell = d.ncell_total;
  const bool diag = d.outputs == FRT_OUT_DIAG;
  const int L = d.lit_cap;
  for (long long gc = blockIdx.x * (long long)blockDim.x + threadIdx.x; gc < ncell;
       gc += (long long)gridDim.x * blockDim.x) {
    const int b = box_of_cell(d, gc);
    if (b < 0) continue;
    const BoxP& B = d.box[b];
    if (gc - B.cell0 >= B.ncell) continue;
    ThermCell c;
    c.temp = d.temp[gc];
    c.heat = d.heat[gc];
    c.cool = d.cool[gc];
    c.nH = d.nH[gc];
    c.nH1 = d.nH1[gc];
    c.nH1_prev = d.nH1_prev[gc];
    c.nH2 = c.nH - c.nH1;
    c.nHe2 = d.nHe[gc] - d.nHe1[gc];
    c.ne = d.ne[gc];
    c.n_tot = d.n_tot[gc];
    c.dne_dt = d.dne_dt[gc];
    c.f_H2 = c.nH2 / c.nH;
    c.avg_nh1 = d.avg_nh1[gc];
    c.avg_nhe1 = d.avg_nhe1[gc];
    const int slot = d.lit_slot[gc];
    HeatSrc hs{nullptr, nullptr, 0, 0.f, 0.f, 0};
    if (slot >= 0) {
      if (!STRICT && !d.per_bin) hs = HeatSrc{nullptr, nullptr, 0, d.l_heat[slot].x, d.l_heat[slot].y, 2};
      else hs = HeatSrc{d.l_acc_nu_h + slot, d.l_acc_nu_he + slot, L, 0.f, 0.f, 1};
    }
    density_change(d, B, gc, &c);
      thermal_update<STRICT>(c, B.th, hs, d.F, d.nhe_to_nh);
    d.temp[gc] = c.temp;
    d.heat[gc] = c.heat;
    d.cool[gc] = c.cool;
    if (diag) {
      d.if_speed[gc] = c.if_speed;
      d.inc_flux[gc] = c.inc_flux;
    }
  }
}

// ---- dense view of a per-step sparse output (zero where no ray deposited) ------------------
// field: 0 gamma_H1_tot, 1 gamma_He1_tot, 2+nu gamma_H1_nu, 2+F+nu gamma_He1_nu, 2+2F+nu ngam_nu
__global__ void k_gather_sparse(Dev d, long long cell0, long long ncell, int which, float* out) {
  const int L = d.lit_cap, F = d.F;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell; c += (long long)gridDim.x * blockDim.x) {
    const int slot = d.lit_slot[cell0 + c];
    float v = 0.f;
    if (slot >= 0) {
      if (which == 0) v = d.l_acc[slot].x;
      else if (which == 1) v = d.l_acc[slot].y;
      else if (which < 2 + F) v = d.l_acc_nu_h[(size_t)(which - 2) * L + slot];
      else if (which < 2 + 2 * F) v = d.l_acc_nu_he[(size_t)(which - 2 - F) * L + slot];
      else v = d.l_ngam[(size_t)(which - 2 - 2 * F) * L + slot];
    }
    out[c] = v;
  }
}

}  // namespace

// ---- launchers -------------------------------------------------------------------------------
void launch_clear_lit(const Dev& d, int grid, cudaStream_t s) { k_clear_lit<<<grid, 256, 0, s>>>(d); }

void launch_lit_init(const Dev& d, bool strict, int grid, cudaStream_t s) {
  if (strict) k_lit_init<true><<<grid, 256, 0, s>>>(d);
  else k_lit_init<false><<<grid, 256, 0, s>>>(d);
}

// grid <= 0: the persistent ray pass with exactly its resident blocks (one wave: every warp's
// static slice starts at once, none waits for a second wave)
void launch_raypass(const Dev& d, int iter, bool strict, int grid, cudaStream_t s, int block, int chunk) {
  const bool last = iter == d.itercount - 1;
  if (strict) {
    if (last) k_raypass_strict<true><<<grid > 0 ? grid : 148 * 8, 256, 0, s>>>(d);
    else k_raypass_strict<false><<<grid > 0 ? grid : 148 * 8, 256, 0, s>>>(d);
    return;
  }
  const bool q = chunk > 0;
  void (*k)(Dev, int, int);
  if (last && d.tau_max > 0.0) {   // the optical-depth limit (opt-in): the generic last pass with the columns
    k = q ? k_raypass_mixed<true, 0, true, 0, true> : k_raypass_mixed<true, 0, false, 0, true>;
  } else if (d.F == 5 && d.nho >= 3) {
    if (last) k = q ? k_raypass_mixed<true, 5, true, 3> : k_raypass_mixed<true, 5, false, 3>;
    else k = q ? k_raypass_mixed<false, 5, true, 3> : k_raypass_mixed<false, 5, false, 3>;
  } else if (d.F == 5) {
    if (last) k = q ? k_raypass_mixed<true, 5, true> : k_raypass_mixed<true, 5, false>;
    else k = q ? k_raypass_mixed<false, 5, true> : k_raypass_mixed<false, 5, false>;
  } else {
    if (last) k = q ? k_raypass_mixed<true, 0, true> : k_raypass_mixed<true, 0, false>;
    else k = q ? k_raypass_mixed<false, 0, true> : k_raypass_mixed<false, 0, false>;
  }
  const int g = grid > 0 ? grid : resident_grid(k, block);
  k<<<g, block, 0, s>>>(d, iter, chunk);
}

// grid <= 0: exactly the resident blocks of the chosen pass (its grid-stride loop then runs in one
// wave; 8 blocks per SM against 5 resident for the middle passes ran 1.6 waves)
void launch_litpass(const Dev& d, int iter, bool strict, bool fused_thermal, int grid, cudaStream_t s, int s_begin,
                    int s_end) {
  const bool last = iter == d.itercount - 1;
  void (*k)(Dev, int, int);
  if (strict) {
    if (!last) k = k_litpass<true, false, false>;
    else if (fused_thermal) k = k_litpass<true, true, true>;
    else k = k_litpass<true, true, false>;
  } else {
    if (!last) k = k_litpass<false, false, false>;
    else if (fused_thermal) k = k_litpass<false, true, true>;
    else k = k_litpass<false, true, false>;
  }
  const int g = grid > 0 ? grid : resident_grid(k, 256);
  k<<<g, 256, 0, s>>>(d, s_begin, s_end);
}

void launch_dark(const Dev& d, bool strict, bool fused_thermal, int grid, cudaStream_t s) {
  if (strict) {
    if (fused_thermal) k_dark<true, true><<<grid, 256, 0, s>>>(d);
    else k_dark<true, false><<<grid, 256, 0, s>>>(d);
  } else {
    if (fused_thermal) k_dark<false, true><<<grid, 256, 0, s>>>(d);
    else k_dark<false, false><<<grid, 256, 0, s>>>(d);
  }
}

void launch_thermal_all(const Dev& d, bool strict, int grid, cudaStream_t s) {
  if (strict) k_thermal_all<true><<<grid, 256, 0, s>>>(d);
  else k_thermal_all<false><<<grid, 256, 0, s>>>(d);
}

void launch_gather_sparse(const Dev& d, long long cell0, long long ncell, int which, float* out, cudaStream_t s) {
  k_gather_sparse<<<grid_for(ncell, 256, 4096), 256, 0, s>>>(d, cell0, ncell, which, out);
}

}  // namespace frt
