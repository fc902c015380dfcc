// Adjoint of one step's Gamma field: J = sum of Gamma_HI over a sub-box after the C2Ray
// iteration of the next step (ray pass ray_tracing.cc:701-938, cell update 1077-1113, the
// Gamma total of 1152), back-propagated to the luminosity of every source and to the hydrogen
// density of every cell.
//
// The ray segments are recomputed from the ray state (the advance's cell walk, frt_dda.cuh) in
// every pass instead of being stored. Everything is FP64. The forward sweep keeps, for the cells
// on the paths, the C2Ray iterates a^k = <n_HI>, b^k = <n_HeI> and the rates Gamma^k of every
// iteration; the reverse sweep walks the iterations backwards:
//   * ray pass k: J_ray = sum_p sum_nu nin_p g_p with nin_p = n0 prod_{q<p} T_q and
//     g_p = absb_p (f_H wH + f_He wHe), wH = Gbar_H K / a_p (the adjoint weight of the cell's
//     rate); dJ/da_p = nin_p dg_p/da_p - sigma_H dist_p R_p with R_p = sum_{q>p} nin_q g_q, and
//     dJ/dn0 = sum_p prod T g_p. Two forward walks per ray (total, then the suffix sums as
//     total - prefix) avoid storing per-segment values.
//   * cell update k-1: a^k = n_H y'(Gamma, n_e) with y' = y_eq + (y0 - y_eq) E(r),
//     E(r) = (1 - e^-r)/r, r = dt (Gamma + C alpha n_e), n_e = n_H - a + n_He - b.
// A cell's n_H scales n_He and the initial n_HI, n_HeI with it (one density, init_funcs.cc:34-62);
// ionised fractions, temperature and recombination coefficients stay fixed; nphot_min stays at
// its set-up value; the dump rule's branch is taken as fixed (a point of non-differentiability).
//
// Compiled with -fmad=false like frt_geom.cu, so the recomputed segments are those of the step.
#include <math.h>

#include "frt_dda.cuh"
#include "frt_internal.cuh"
#include "frt_physics.cuh"

namespace frt {

namespace {

template <typename T>
__device__ __forceinline__ T block_sum_d(T v) {
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

struct RaySegs {
  int n;            // segments (0: the ray does not move this step)
  int slot[16];
  float dist[16];
};

// The ray's segments of the next advance (k_advance's walk, without writing the ray), as slots.
__device__ __forceinline__ void ray_segments(const Dev& d, const AdjDev& a, const RayPool& A, int i, bool mark,
                                             RaySegs* S) {
  S->n = 0;
  const BoxP& B = d.box[A.box[i]];
  const int N = B.n;
  const int ind = A.cell[i];
  const int ii = ind / B.nn, jj = (ind - ii * B.nn) / N, kk = ind - ii * B.nn - jj * N;
  const float xhat = A.xh[i], yhat = A.yh[i], zhat = A.zh[i];
  float x0 = A.x[i], y0 = A.y[i], z0 = A.z[i];
  const float deltat = A.time[i] + B.dt;
  const float dist = B.clight * deltat;
  if (!ray_moves(B, x0, y0, z0, xhat, yhat, zhat, dist)) return;
  float r0 = A.r[i];
  r0 += dist / B.scale;
  if (B.rkill > 0.0 && (double)r0 > B.rkill) return;   // removed right after the advance
  int in = ii, jn = jj, kn = kk;
  const int PL = d.PL < 16 ? d.PL : 16;
  const int ns = dda_walk(B, PL, xhat, yhat, zhat, deltat, x0, y0, z0, in, jn, kn, [&](int p, long long gc, float ds) {
    S->slot[p] = mark ? (int)gc : a.slot[gc];
    S->dist[p] = ds;
  });
  if (ns < 0) {
    atomicOr(a.err, 1u);
    return;
  }
  if (mark)
    for (int p = 0; p < ns; p++) a.flag[S->slot[p]] = 1;
  S->n = ns;
}

__global__ void k_adj_mark(Dev d, AdjDev a) {
  const int cur = d.ctl->cur;
  const int n = d.ctl->nray[cur];
  const RayPool A = d.pool[cur];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    RaySegs S;
    ray_segments(d, a, A, i, true, &S);
  }
}

__global__ void __launch_bounds__(256) k_adj_compact(Dev d, AdjDev a) {
  compact_marked(a.flag, d.ncell_total, a.slot, a.cell, a.count, a.cap, a.err, 2u);
}

// constants and the iteration-0 iterates of the path cells
__global__ void k_adj_init(Dev d, AdjDev a) {
  const int n = min(*a.count, a.cap);
  const BoxP& Bo = d.box[a.box];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int gc = a.cell[j];
    a.nH[j] = d.nH[gc];
    a.nHe[j] = d.nHe[gc];
    a.y0h[j] = d.f_H1[gc];
    a.y0he[j] = d.f_He1[gc];
    float rh, rhe;
    recomb_coeffs<true>(d.temp[gc], &rh, &rhe);
    const float cl = d.clump ? d.clump[gc] : d.const_clump;
    a.crh[j] = (double)(cl * rh);
    a.crhe[j] = (double)(cl * rhe);
    a.a[j] = d.nH1[gc];
    a.b[j] = d.nHe1[gc];
    bool in = false;
    const long long lc = gc - Bo.cell0;
    if (lc >= 0 && lc < Bo.ncell) {
      const int i = (int)(lc / Bo.nn), jj = (int)((lc / Bo.n) % Bo.n), k = (int)(lc % Bo.n);
      in = i >= a.lo[0] && i < a.hi[0] && jj >= a.lo[1] && jj < a.hi[1] && k >= a.lo[2] && k < a.hi[2];
    }
    a.in_obj[j] = in ? 1 : 0;
    a.abar[j] = 0.0;
    a.bbar[j] = 0.0;
    a.nhbar[j] = 0.0;
    a.gbh[j] = in ? 1.0 : 0.0;
    a.gbhe[j] = 0.0;
  }
}

__global__ void k_adj_zero_rates(AdjDev a, int k) {
  const int n = min(*a.count, a.cap);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    a.gh[(size_t)k * a.cap + j] = 0.0;
    a.ghe[(size_t)k * a.cap + j] = 0.0;
  }
}

// Per-bin quantities of one segment: absorbed fraction, H/He split and their derivatives with
// respect to x = dtau_HI and y = dtau_HeI (ray_tracing.cc:763-779, 814-846).
struct SegBin {
  double T;                 // transmission e^-(x+y)
  double absb, fh, fhe;     // absorbed fraction (1 on the dump segment) and the H/He split
  double dabsb_dx, dabsb_dy, dfh_dx, dfh_dy;
};

__device__ __forceinline__ SegBin seg_bin(double x, double y, bool dump) {
  SegBin s;
  const double ex = exp(-x), ey = exp(-y);
  const double ah = -expm1(-x), ahe = -expm1(-y);
  s.T = ex * ey;
  s.absb = dump ? 1.0 : -expm1(-(x + y));
  s.dabsb_dx = dump ? 0.0 : s.T;
  s.dabsb_dy = s.dabsb_dx;
  const double x1 = ah * ey, x2 = ahe * ex, S = x1 + x2;
  if (S > 0.0) {
    s.fh = x1 / S;
    s.fhe = x2 / S;
    const double S2 = S * S;
    s.dfh_dx = (s.T * S - x1 * (s.T - x2)) / S2;
    s.dfh_dy = (-x1 * S - x1 * (s.T - x1)) / S2;
  } else {
    s.fh = s.fhe = s.dfh_dx = s.dfh_dy = 0.0;
  }
  return s;
}

// forward ray pass k: the rates Gamma^k of the path cells
__global__ void k_adj_fwd_ray(Dev d, AdjDev a, int k) {
  const int cur = d.ctl->cur;
  const int n = d.ctl->nray[cur];
  const RayPool A = d.pool[cur];
  const int F = d.F, cap = d.ray_cap;
  const double* ak = a.a + (size_t)k * a.cap;
  const double* bk = a.b + (size_t)k * a.cap;
  double* gh = a.gh + (size_t)k * a.cap;
  double* ghe = a.ghe + (size_t)k * a.cap;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    RaySegs S;
    ray_segments(d, a, A, i, false, &S);
    if (!S.n) continue;
    const BoxP& B = d.box[A.box[i]];
    const double K = 1.0 / ((double)B.dt * B.vol);
    double nin[FRT_MAX_FREQ];
    for (int nu = 0; nu < F; nu++) nin[nu] = (double)A.nphot[(size_t)nu * cap + i] * kPhotNorm;
    for (int p = 0; p < S.n; p++) {
      const int j = S.slot[p];
      if (j < 0 || j >= a.cap) break;
      double tot = 0.0;
      for (int nu = 0; nu < F; nu++) tot += nin[nu] / kPhotNorm;
      const bool dump = tot < B.nphot_min;
      const double av = ak[j], bv = bk[j], ds = S.dist[p];
      double sh = 0.0, she = 0.0;
      for (int nu = 0; nu < F; nu++) {
        const SegBin s = seg_bin(av * d.sigH1_d[nu] * ds, bv * d.sigHe1_d[nu] * ds, dump);
        sh += s.fh * nin[nu] * s.absb;
        she += s.fhe * nin[nu] * s.absb;
        nin[nu] *= s.T;
      }
      atomicAdd(&gh[j], sh * K / av);
      atomicAdd(&ghe[j], she * K / bv);
      if (dump) break;
    }
  }
}

// C2Ray neutral fraction y' = y_eq + (y0 - y_eq) E(r) and its derivatives in Gamma and n_e.
struct C2D {
  double y, dy_dg, dy_dne;
};

__device__ __forceinline__ C2D c2ray_d(double gamma, double crec, double ne, double y0, double dt) {
  C2D o;
  const double rec = crec * ne;
  const double pr = gamma + rec;
  if (!(pr > 0.0)) {
    o.y = y0;
    o.dy_dg = o.dy_dne = 0.0;
    return o;
  }
  const double yeq = rec / pr;
  const double r = dt * pr;
  double E, Ep;   // E(r) = (1 - e^-r)/r and dE/dr
  if (r < 0.1) {
    // series of E = sum (-r)^k / (k+1)! and of its derivative, to r^9 (relative error < 1e-13)
    E = 0.0;
    Ep = 0.0;
    double c = 1.0, rk = 1.0;
    for (int kk = 0; kk <= 9; kk++) {
      c /= (double)(kk + 1);            // 1/(k+1)!
      const double term = ((kk & 1) ? -1.0 : 1.0) * c;
      E += term * rk;
      if (kk + 1 <= 9) Ep += ((kk & 1) ? 1.0 : -1.0) * (double)(kk + 1) * (c / (double)(kk + 2)) * rk;
      rk *= r;
    }
  } else {
    const double em = -expm1(-r);
    E = em / r;
    Ep = (exp(-r) * (1.0 + r) - 1.0) / (r * r);
  }
  o.y = yeq + (y0 - yeq) * E;
  const double dyeq_dg = -yeq / pr;
  const double dyeq_dne = crec / pr * (1.0 - yeq);
  o.dy_dg = dyeq_dg * (1.0 - E) + (y0 - yeq) * Ep * dt;
  o.dy_dne = dyeq_dne * (1.0 - E) + (y0 - yeq) * Ep * dt * crec;
  return o;
}

// forward cell update k -> k+1 of the path cells
__global__ void k_adj_fwd_cell(Dev d, AdjDev a, int k) {
  const int n = min(*a.count, a.cap);
  const size_t o0 = (size_t)k * a.cap, o1 = (size_t)(k + 1) * a.cap;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double ne = a.nH[j] - a.a[o0 + j] + a.nHe[j] - a.b[o0 + j];
    const double dtj = (double)d.box[d.tile_box[a.cell[j] >> kTileShift]].dt;
    const C2D h = c2ray_d(a.gh[o0 + j], a.crh[j], ne, a.y0h[j], dtj);
    const C2D he = c2ray_d(a.ghe[o0 + j], a.crhe[j], ne, a.y0he[j], dtj);
    a.a[o1 + j] = a.nH[j] * h.y;
    a.b[o1 + j] = a.nHe[j] * he.y;
  }
}

__global__ void k_adj_objective(AdjDev a) {
  const int n = min(*a.count, a.cap);
  const double* g = a.gh + (size_t)(a.I - 1) * a.cap;
  double s = 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    if (a.in_obj[j]) s += g[j];
  s = block_sum_d(s);
  if (threadIdx.x == 0 && s != 0.0) atomicAdd(a.J, s);
}

// The source that cast a ray, from the ray alone. The cast puts a ray at the centre of its
// source's cell with r = 0 (ray_tracing.cc:300-312); the advance moves it along its direction
// while r grows by the comoving distance (ray_tracing.cc:1259-1263); a split places each child at
// the parent's position plus (child direction - parent direction) r dx/dx0 (ray_tracing.cc:540-548).
// So every ray that no merge has touched sits at source + r (dx/dx0) direction, up to the corner
// nudges of 1e-4 cells, and in cell units the source cell is floor(i + x/dx - r xhat/dx0)
// (periodic), the same for y and z. Returns the context-wide source index, or -1.
__device__ __forceinline__ int ray_source(const Dev& d, const AdjDev& a, const RayPool& A, int i) {
  const BoxP& B = d.box[A.box[i]];
  const int N = B.n;
  const int ind = A.cell[i];
  const int ii = ind / B.nn, jj = (ind - ii * B.nn) / N, kk = ind - ii * B.nn - jj * N;
  const double r = (double)A.r[i] / (double)B.dx0;
  const double gx = ii + (double)A.x[i] / (double)B.dx - r * (double)A.xh[i];
  const double gy = jj + (double)A.y[i] / (double)B.dx - r * (double)A.yh[i];
  const double gz = kk + (double)A.z[i] / (double)B.dx - r * (double)A.zh[i];
  auto wrap = [N](double g) {
    long long c = (long long)floor(g) % N;
    return (int)(c < 0 ? c + N : c);
  };
  const long long cell = ((long long)wrap(gx) * N + wrap(gy)) * N + wrap(gz);
  return a.src_of_cell[B.cell0 + cell];
}

// reverse ray pass k: from the rate weights Gbar^k of the path cells to abar^k, bbar^k and to
// the sources' photon counts
__global__ void k_adj_rev_ray(Dev d, AdjDev a, int k) {
  const int cur = d.ctl->cur;
  const int n = d.ctl->nray[cur];
  const RayPool A = d.pool[cur];
  const int F = d.F, cap = d.ray_cap;
  const double* ak = a.a + (size_t)k * a.cap;
  const double* bk = a.b + (size_t)k * a.cap;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    RaySegs S;
    ray_segments(d, a, A, i, false, &S);
    if (!S.n) continue;
    const BoxP& B = d.box[A.box[i]];
    const double K = 1.0 / ((double)B.dt * B.vol);
    double n0[FRT_MAX_FREQ], nin[FRT_MAX_FREQ], tot[FRT_MAX_FREQ];
    for (int nu = 0; nu < F; nu++) {
      n0[nu] = (double)A.nphot[(size_t)nu * cap + i] * kPhotNorm;
      nin[nu] = n0[nu];
      tot[nu] = 0.0;
    }
    // walk 1: J_ray per bin
    for (int p = 0; p < S.n; p++) {
      const int j = S.slot[p];
      if (j < 0 || j >= a.cap) break;
      double t = 0.0;
      for (int nu = 0; nu < F; nu++) t += nin[nu] / kPhotNorm;
      const bool dump = t < B.nphot_min;
      const double av = ak[j], bv = bk[j], ds = S.dist[p];
      const double wh = a.gbh[j] * K / av, whe = a.gbhe[j] * K / bv;
      for (int nu = 0; nu < F; nu++) {
        const SegBin s = seg_bin(av * d.sigH1_d[nu] * ds, bv * d.sigHe1_d[nu] * ds, dump);
        tot[nu] += nin[nu] * s.absb * (s.fh * wh + s.fhe * whe);
        nin[nu] *= s.T;
      }
      if (dump) break;
    }
    double dl = 0.0;
    for (int nu = 0; nu < F; nu++) {
      dl += tot[nu];   // n0 dJ/dn0 (J_ray is linear in n0)
      nin[nu] = n0[nu];
    }
    const int src = ray_source(d, a, A, i);
    if (src >= 0 && dl != 0.0) atomicAdd(&a.dlbar[src], dl);
    // walk 2: derivatives of every segment's g and transmission
    double pre[FRT_MAX_FREQ];
    for (int nu = 0; nu < F; nu++) pre[nu] = 0.0;
    for (int p = 0; p < S.n; p++) {
      const int j = S.slot[p];
      if (j < 0 || j >= a.cap) break;
      double t = 0.0;
      for (int nu = 0; nu < F; nu++) t += nin[nu] / kPhotNorm;
      const bool dump = t < B.nphot_min;
      const double av = ak[j], bv = bk[j], ds = S.dist[p];
      const double wh = a.gbh[j] * K / av, whe = a.gbhe[j] * K / bv;
      double da = 0.0, db = 0.0;
      for (int nu = 0; nu < F; nu++) {
        const double sx = d.sigH1_d[nu] * ds, sy = d.sigHe1_d[nu] * ds;
        const SegBin s = seg_bin(av * sx, bv * sy, dump);
        const double gsum = s.fh * wh + s.fhe * whe;
        const double g = s.absb * gsum;
        const double dg_dx = s.dabsb_dx * gsum + s.absb * s.dfh_dx * (wh - whe);
        const double dg_dy = s.dabsb_dy * gsum + s.absb * s.dfh_dy * (wh - whe);
        pre[nu] += nin[nu] * g;
        const double R = dump ? 0.0 : tot[nu] - pre[nu];   // sum of nin g over the later segments
        da += nin[nu] * (dg_dx * sx - s.absb * s.fh * wh / av) - sx * R;
        db += nin[nu] * (dg_dy * sy - s.absb * s.fhe * whe / bv) - sy * R;
        nin[nu] *= s.T;
      }
      if (da != 0.0) atomicAdd(&a.abar[j], da);
      if (db != 0.0) atomicAdd(&a.bbar[j], db);
      if (dump) break;
    }
  }
}

// reverse cell update k-1 -> k: from abar^k, bbar^k to Gbar^{k-1}, abar^{k-1}, bbar^{k-1} and n_H
__global__ void k_adj_rev_cell(Dev d, AdjDev a, int k) {
  const int n = min(*a.count, a.cap);
  const size_t o = (size_t)(k - 1) * a.cap;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double dtj = (double)d.box[d.tile_box[a.cell[j] >> kTileShift]].dt;
    const double nH = a.nH[j], nHe = a.nHe[j];
    const double ne = nH - a.a[o + j] + nHe - a.b[o + j];
    const C2D h = c2ray_d(a.gh[o + j], a.crh[j], ne, a.y0h[j], dtj);
    const C2D he = c2ray_d(a.ghe[o + j], a.crhe[j], ne, a.y0he[j], dtj);
    const double ab = a.abar[j], bb = a.bbar[j];
    const double ne_bar = ab * nH * h.dy_dne + bb * nHe * he.dy_dne;
    const double rhe = nHe / nH;   // n_He moves with n_H
    a.gbh[j] = ab * nH * h.dy_dg;
    a.gbhe[j] = bb * nHe * he.dy_dg;
    a.nhbar[j] += ab * h.y + bb * rhe * he.y + ne_bar * (1.0 + rhe);
    a.abar[j] = -ne_bar;
    a.bbar[j] = -ne_bar;
  }
}

// the iteration-0 iterates are the cell's n_HI, n_HeI, both proportional to n_H
__global__ void k_adj_rev_init(AdjDev a) {
  const int n = min(*a.count, a.cap);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    a.nhbar[j] += (a.abar[j] * a.a[j] + a.bbar[j] * a.b[j]) / a.nH[j];
}

__global__ void k_adj_gather(Dev d, AdjDev a, long long cell0, long long ncell, float* out) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncell;
       c += (long long)gridDim.x * blockDim.x) {
    const int j = a.slot[cell0 + c];
    out[c] = (j >= 0 && j < a.cap) ? (float)a.nhbar[j] : 0.f;
  }
}

}  // namespace

void launch_adjoint(const Dev& d, const AdjDev& a, int grid, cudaStream_t s) {
  k_adj_mark<<<grid, 128, 0, s>>>(d, a);
  k_adj_compact<<<grid_for(d.ncell_total >> 4, 256, 148 * 8), 256, 0, s>>>(d, a);
  k_adj_init<<<grid, 256, 0, s>>>(d, a);
  for (int k = 0; k < a.I; k++) {
    k_adj_zero_rates<<<grid, 256, 0, s>>>(a, k);
    k_adj_fwd_ray<<<grid, 128, 0, s>>>(d, a, k);
    if (k + 1 < a.I) k_adj_fwd_cell<<<grid, 256, 0, s>>>(d, a, k);
  }
  k_adj_objective<<<grid, 256, 0, s>>>(a);
  for (int k = a.I - 1; k >= 0; k--) {
    k_adj_rev_ray<<<grid, 128, 0, s>>>(d, a, k);
    if (k > 0) k_adj_rev_cell<<<grid, 256, 0, s>>>(d, a, k);
  }
  k_adj_rev_init<<<grid, 256, 0, s>>>(a);
}

void launch_adjoint_gather(const Dev& d, const AdjDev& a, long long cell0, long long ncell, float* out,
                           cudaStream_t s) {
  k_adj_gather<<<grid_for(ncell, 256, 4096), 256, 0, s>>>(d, a, cell0, ncell, out);
}

}  // namespace frt
