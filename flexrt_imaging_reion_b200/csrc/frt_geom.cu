// Ray geometry kernels: advance through the grid, split, merge, cast, compaction.
//
// This translation unit is compiled with -fmad=false: the reference's geometry is float
// arithmetic (with a few double sub-expressions) whose results decide cell indices, split and
// merge trees and HEALPix pixels, so every product and sum here is rounded exactly as the
// reference's g++ build rounds it (no a*b+c contraction). Each kernel cites the reference code
// whose arithmetic it reproduces.
#include <limits.h>
#include <math.h>

#include "frt_internal.cuh"
#include "frt_dda.cuh"
#include "hp_nest.h"

namespace frt {

namespace {

// Rotation of a unit vector by the precomputed coefficient table: the reference evaluates
// (c00)*xhat + (c01)*yhat + (c02)*zhat with each coefficient a float product of cosf/sinf
// values (healpix_funcs.cc:102-143); the host builds those coefficients with the same
// expressions, the device does the remaining products and sums.
__device__ __forceinline__ void rot_apply(const float* m, float x, float y, float z, float* ox, float* oy, float* oz) {
  *ox = (m[0] * x + m[1] * y) + m[2] * z;
  *oy = (m[3] * x + m[4] * y) + m[5] * z;
  *oz = (m[6] * x + m[7] * y) + m[8] * z;
}

// Direction of NEST pixel `pix` at HEALPix `order` as the float triple the rotation takes: from
// the table for orders up to kPixTabMax (built by the same pix2vec), else computed (out of line,
// so that the common table path keeps few registers).
__device__ __noinline__ void pix_dir_computed(int order, int pix, float* fx, float* fy, float* fz) {
  double vx, vy, vz;
  hpn::pix2vec(order, pix, &vx, &vy, &vz);
  *fx = (float)vx;
  *fy = (float)vy;
  *fz = (float)vz;
}

__device__ __forceinline__ void pix_dir(const Dev& d, int order, int pix, float* fx, float* fy, float* fz) {
  if (order <= kPixTabMax) {
    const float4 v = d.pix_tab[4ll * ((1ll << (2 * order)) - 1) + pix];
    *fx = v.x;
    *fy = v.y;
    *fz = v.z;
  } else {
    pix_dir_computed(order, pix, fx, fy, fz);
  }
}

__global__ void k_pix_table(float4* tab) {
  const long long n = 4ll * ((1ll << (2 * (kPixTabMax + 1))) - 1);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    int order = 0;
    while (e >= 4ll * ((1ll << (2 * (order + 1))) - 1)) order++;
    const int pix = (int)(e - 4ll * ((1ll << (2 * order)) - 1));
    double vx, vy, vz;
    hpn::pix2vec(order, pix, &vx, &vy, &vz);
    tab[e] = make_float4((float)vx, (float)vy, (float)vz, 0.f);
  }
}

__device__ __forceinline__ float sum_nphot(const RayPool& P, int i, int F, int cap) {
  float s = 0.f;
  for (int nu = 0; nu < F; nu++) s += P.nphot[(size_t)nu * cap + i];
  return s;
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
  return r;  // valid in thread 0
}

// ---------------------------------------------------------------------------------------
// Start of a step: t += dt (main.cc:127), ray_dt of the sources += dt (rt_funcs.cc:163-172),
// per-step counters to zero, the next pool emptied.
__global__ void k_step_begin(Dev d) {
  Ctl* c = d.ctl;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c->n_lit_prev = c->n_lit;
    c->n_lit = 0;
    c->nray[c->cur ^ 1] = 0;
    // after a capacity error the pools may hold unwritten slots: drop every ray so that no
    // kernel ever reads an uninitialised record (the error stays latched for the host)
    if (c->err) c->nray[c->cur] = 0;
    c->rays_moved = c->crossings = c->split = c->merged = c->killed = c->cast = 0;
    c->mv_seg = 0ull;
    c->emitted = c->deposited = c->killed_ph = c->overlap = c->in_flight = 0.0;
  }
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < d.nbox; b += gridDim.x * blockDim.x) {
    BoxP& B = d.box[b];
    B.t += B.dt;
    // for a float x: (double)x < nphot_min <=> x < nmin_ru, (double)x > nphot_min <=> x > nmin_rd
    B.nmin_ru = __double2float_ru(B.nphot_min);
    B.nmin_rd = __double2float_rd(B.nphot_min);
  }
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < d.nsrc; s += gridDim.x * blockDim.x)
    d.src_ray_dt[s] += d.box[d.src_box[s]].dt;
}

// Mark a cell touched by a segment. The lit list is numbered afterwards in cell order
// (k_lit_compact), so that the lit-cell kernels read the dense fields in address order.
__device__ __forceinline__ void mark_lit(const Dev& d, long long gc) {
  d.lit_flag[gc] = 1;   // a plain byte store: no load, so the walk never waits on the flag
}

// Number the marked cells in cell order (compact_marked, frt_dda.cuh).
__global__ void __launch_bounds__(256) k_lit_compact(Dev d) {
  compact_marked(d.lit_flag, d.ncell_total, d.lit_slot, d.l_cell, &d.ctl->n_lit, d.lit_cap, &d.ctl->err, ERR_LIT_CAP);
}

// The lit numbering in strict cell order, for a box shared by several contexts (the phased step):
// every context must give a cell the same slot, so the chunks' bases come from a scan over the
// chunks (k_lit_chunk_scan) instead of one atomicAdd per block. A chunk is 4096 cells: 256
// threads x 16 flag bytes (one 16-byte load; a flag byte is 0 or 1).
__device__ __forceinline__ int flags16(const uint8_t* flag, long long nvec, long long v) {
  if (v >= nvec) return 0;
  const uint4 f = reinterpret_cast<const uint4*>(flag)[v];
  return __popc(f.x) + __popc(f.y) + __popc(f.z) + __popc(f.w);
}

__global__ void __launch_bounds__(256) k_lit_chunk_count(Dev d, int* chunk_cnt, long long nchunk) {
  __shared__ int red[8];
  const long long nvec = d.ncell_total >> 4;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (long long c = blockIdx.x; c < nchunk; c += gridDim.x) {
    int x = flags16(d.lit_flag, nvec, c * 256 + threadIdx.x);
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[w] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int k = 0; k < 8; k++) t += red[k];
      chunk_cnt[c] = t;
    }
    __syncthreads();
  }
}

// one block of 1024 threads: exclusive scan of the chunk counts in place; the total is n_lit
__global__ void __launch_bounds__(1024) k_lit_chunk_scan(Dev d, int* chunk, long long nchunk) {
  __shared__ int wt[32];
  __shared__ long long carry_s;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (long long t0 = 0; t0 < nchunk; t0 += 1024) {
    const long long i = t0 + threadIdx.x;
    const int v = (i < nchunk) ? chunk[i] : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wt[w] = incl;
    __syncthreads();
    if (w == 0) {
      int x = wt[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      wt[lane] = x;   // inclusive prefix over the warps
    }
    __syncthreads();
    const long long carry = carry_s;
    if (i < nchunk) chunk[i] = (int)(carry + (w > 0 ? wt[w - 1] : 0) + incl - v);
    __syncthreads();
    if (threadIdx.x == 0) carry_s = carry + wt[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) d.ctl->n_lit = (int)carry_s;
}

__global__ void __launch_bounds__(256) k_lit_chunk_write(Dev d, const int* chunk_off, long long nchunk) {
  __shared__ int warp_tot[8];
  const long long nvec = d.ncell_total >> 4;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (long long c = blockIdx.x; c < nchunk; c += gridDim.x) {
    const long long v = c * 256 + threadIdx.x;
    uint4 f = make_uint4(0u, 0u, 0u, 0u);
    if (v < nvec) f = reinterpret_cast<const uint4*>(d.lit_flag)[v];
    const int cnt = __popc(f.x) + __popc(f.y) + __popc(f.z) + __popc(f.w);
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
      int x = (lane < 8) ? warp_tot[lane] : 0;
      for (int o = 1; o < 8; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane < 8) warp_tot[lane] = x;
    }
    __syncthreads();
    int s = chunk_off[c] + (w > 0 ? warp_tot[w - 1] : 0) + incl - cnt;
    if (cnt) {
      const unsigned words[4] = {f.x, f.y, f.z, f.w};
      for (int q = 0; q < 4; q++) {
        unsigned m = words[q];
        while (m) {
          const int bit = __ffs(m) - 1;   // flag bytes hold 0 or 1: bit 8k is byte k
          m &= m - 1;
          const long long gc = v * 16 + q * 4 + (bit >> 3);
          if (s < d.lit_cap) {
            d.l_cell[s] = (int)gc;
            d.lit_slot[gc] = s;
          } else {
            atomicOr(&d.ctl->err, ERR_LIT_CAP);
          }
          s++;
        }
      }
    }
    __syncthreads();
  }
}

// advance_ray (ray_tracing.cc:1222-1512) with c2ray_iter = TRUE and fion = 1 (plain mode):
// cell-boundary walk over c_sim * time, path segments {cell, dist}, periodic wrap, corner nudge.
//
// One thread per pool ray: the thread loads its ray (consecutive threads, consecutive rays:
// coalesced), walks it (dda_walk: the exact face time of the reference only for the axes that can
// be the next face) and stores the updated record. The walk also builds the ray passes' input:
// the segments go to the thread's column of a shared-memory tile ([PL][T], dynamic), then the
// block scans its moved rays (moved and not removed) and their segment counts in pool order,
// takes the bases of both with one 64-bit atomicAdd per tile of T rays, and every thread with a
// moved ray writes its 16-byte header {pool index, first packed segment, segment count, box} and
// copies its segments to the packed array (the first segment of a ray carries the head bit in
// the sign of its positive distance). A tile costs two block barriers; the scan's per-warp
// totals are double-buffered by tile parity, so a warp that runs ahead into the next tile never
// overwrites totals another warp still reads. The packed segments hold cells; k_pk_slots turns
// them into lit slots once the lit cells are numbered. Rays [r_begin, min(r_end, pool size)) of
// the pool (the autotuner times launch shapes on shares of one step's rays; the step launches
// the whole pool).
template <int T>
__global__ void __launch_bounds__(T, 1024 / T) k_advance(Dev d, int r_begin, int r_end) {
  constexpr int W = T / 32;
  extern __shared__ int2 s_seg[];      // [PL][T]: segment p of thread t's ray at s_seg[p * T + t]
  __shared__ int s_wq[2][W], s_ws[2][W];   // per-warp inclusive prefixes (moved rays, segments), by tile parity
  __shared__ unsigned long long s_tile[2];
  const int cur = d.ctl->cur;
  const int n = min(d.ctl->nray[cur], r_end);
  const RayPool A = d.pool[cur];
  const int cap = d.ray_cap, PL = d.PL;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  int cross = 0, moved = 0, killed = 0;   // this thread's walks (a few thousand at most)
  double killed_ph = 0.0;
  int par = 0;
  for (int i0 = r_begin + blockIdx.x * T; i0 < n; i0 += gridDim.x * T, par ^= 1) {
    const int i = i0 + t;
    int ns_t = 0;   // segments this thread's ray contributes to the packed list
    uint16_t bx = 0;
    if (i < n) {
      bx = A.box[i];
      const BoxP& B = d.box[bx];
      const float xhat = A.xh[i], yhat = A.yh[i], zhat = A.zh[i];
      float x0 = A.x[i], y0 = A.y[i], z0 = A.z[i];
      const float deltat = A.time[i] + B.dt;
      const float dist = B.clight * deltat;
      if (!ray_moves(B, x0, y0, z0, xhat, yhat, zhat, dist)) {
        A.time[i] = deltat;
        d.dead[i] = 0;
      } else {
        const int N = B.n, NN = B.nn;
        const int ind = A.cell[i];
        float r0 = A.r[i], dr = A.dr[i];
        int in, jn, kn;
        cell_ijk(ind, N, NN, B.inv_n, B.inv_nn, &in, &jn, &kn);
        r0 += dist / B.scale;
        dr -= dist / B.scale;
        int2* sp = s_seg + t;
        const int ns = dda_walk(B, PL, xhat, yhat, zhat, deltat, x0, y0, z0, in, jn, kn,
                                [&](int p, long long gc, float ds) {
                                  sp[p * T] = make_int2((int)gc, __float_as_int(ds));
                                  mark_lit(d, gc);
                                },
                                d.ifront ? d.fion : nullptr);
        if (ns < 0) {
          // path overflow: the record is left as it was and the ray flagged
          atomicOr(&d.ctl->err, ERR_PATH);
          d.dead[i] = 1;
        } else {
          cross += ns;
          moved += 1;
          // optional removal beyond rkill (comoving), applied after update_rays
          bool dead = false;
          if (B.rkill > 0.0 && (double)r0 > B.rkill) {
            dead = true;
            killed += 1;
            killed_ph += (double)sum_nphot(A, i, d.F, cap) * kPhotNorm;
          }
          d.dead[i] = dead ? 1 : 0;
          A.time[i] = 0.f;
          A.r[i] = r0;
          A.dr[i] = dr;
          A.x[i] = x0;
          A.y[i] = y0;
          A.z[i] = z0;
          A.cell[i] = in * NN + jn * N + kn;
          if (!dead) ns_t = ns;
        }
      }
    }
    // the tile's moved rays and their segments, in pool order: warp scans, then the warps'
    // prefixes and one atomicAdd per tile for the bases of both
    const unsigned mq = __ballot_sync(0xffffffffu, ns_t > 0);
    int xs = ns_t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, xs, o);
      if (lane >= o) xs += y;
    }
    if (lane == 31) {
      s_wq[par][w] = __popc(mq);
      s_ws[par][w] = xs;
    }
    __syncthreads();
    if (w == 0) {
      int qa = (lane < W) ? s_wq[par][lane] : 0, sa = (lane < W) ? s_ws[par][lane] : 0;
#pragma unroll
      for (int o = 1; o < W; o <<= 1) {
        const int yq = __shfl_up_sync(0xffffffffu, qa, o), ys = __shfl_up_sync(0xffffffffu, sa, o);
        if (lane >= o) {
          qa += yq;
          sa += ys;
        }
      }
      if (lane < W) {
        s_wq[par][lane] = qa;
        s_ws[par][lane] = sa;
      }
      if (lane == W - 1)
        s_tile[par] = (qa > 0) ? atomicAdd(&d.ctl->mv_seg, ((unsigned long long)qa << 32) | (unsigned long long)sa)
                               : 0ull;
    }
    __syncthreads();
    if (ns_t > 0) {
      // the header and the segments of this thread's ray (consecutive threads' rays are
      // consecutive in the packed list, so a warp's stores cover a few contiguous sectors)
      const unsigned long long tb = s_tile[par];
      const int off = (int)(tb & 0xffffffffull) + (w > 0 ? s_ws[par][w - 1] : 0) + xs - ns_t;
      const int q = (int)(tb >> 32) + (w > 0 ? s_wq[par][w - 1] : 0) + __popc(mq & ((1u << lane) - 1u));
      d.mv_hdr[q] = make_int4(i, off, ns_t, (int)bx);
      int2* dp = d.pk + off;
      for (int p = 0; p < ns_t; p++) {
        const int2 sg = s_seg[p * T + t];
        // dist > 0: its sign bit is free for the head mark
        dp[p] = make_int2(sg.x, (int)(((unsigned)sg.y & 0x7fffffffu) | (p == 0 ? 0x80000000u : 0u)));
      }
    }
  }
  const long long cross_b = block_sum((long long)cross);
  const long long moved_b = block_sum((long long)moved);
  const long long killed_b = block_sum((long long)killed);
  killed_ph = block_sum(killed_ph);
  if (threadIdx.x == 0) {
    if (cross_b) atomicAdd((unsigned long long*)&d.ctl->crossings, (unsigned long long)cross_b);
    if (moved_b) atomicAdd((unsigned long long*)&d.ctl->rays_moved, (unsigned long long)moved_b);
    if (killed_b) atomicAdd((unsigned long long*)&d.ctl->killed, (unsigned long long)killed_b);
    if (killed_ph != 0.0) atomicAdd(&d.ctl->killed_ph, killed_ph);
  }
}

// The packed segments' cells become lit slots once the lit cells are numbered (k_lit_compact or
// the strict-order numbering): a coalesced pass over the packed list with one lit-slot gather per
// segment, four segments per thread in flight.
__global__ void __launch_bounds__(256) k_pk_slots(Dev d) {
  const long long nseg = (long long)(d.ctl->mv_seg & 0xffffffffull);
  int* pkx = reinterpret_cast<int*>(d.pk);
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long x0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; x0 < nseg; x0 += 4 * stride) {
    int c[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const long long x = x0 + u * stride;
      c[u] = (x < nseg) ? pkx[2 * x] : -1;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) c[u] = (c[u] >= 0) ? d.lit_slot[c[u]] : -1;
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const long long x = x0 + u * stride;
      if (x < nseg) pkx[2 * x] = c[u];
    }
  }
}

// count_rays per box (ray_tracing.cc:35-47) after the C2Ray pass removed rays; then the merge
// set-up: num_thresh test and histogram reset (main.cc:153-163).
__global__ void k_count(Dev d) {
  // per-block counts in shared memory (one global atomic per box and block at the end); a warp
  // whose live rays all belong to one box adds its ballot count in one step
  constexpr int kSh = 256;
  __shared__ unsigned long long sh[kSh];
  const int nb = d.nbox;
  const bool use_sh = nb <= kSh;
  for (int k = threadIdx.x; k < kSh; k += blockDim.x) sh[k] = 0ull;
  __syncthreads();
  const int cur = d.ctl->cur;
  const int n = d.ctl->nray[cur];
  const RayPool A = d.pool[cur];
  const int lane = threadIdx.x & 31;
  for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
    const int i = i0 + threadIdx.x;
    const bool alive = (i < n) && !d.dead[i];
    const int b = alive ? (int)A.box[i] : -1;
    const unsigned live = __ballot_sync(0xffffffffu, alive);
    if (!live) continue;
    const int b0 = __shfl_sync(0xffffffffu, b, __ffs(live) - 1);
    const bool same = __all_sync(0xffffffffu, !alive || b == b0);
    int add_box = -1;
    unsigned long long add_n = 0;
    if (same) {
      if (lane == __ffs(live) - 1) { add_box = b0; add_n = __popc(live); }
    } else if (alive) {
      const unsigned m = __match_any_sync(live, b);
      if (lane == __ffs(m) - 1) { add_box = b; add_n = __popc(m); }
    }
    if (add_box >= 0) {
      if (use_sh) atomicAdd(&sh[add_box], add_n);
      else atomicAdd((unsigned long long*)&d.count[add_box], add_n);
    }
  }
  __syncthreads();
  if (use_sh)
    for (int k = threadIdx.x; k < nb; k += blockDim.x)
      if (sh[k]) atomicAdd((unsigned long long*)&d.count[k], sh[k]);
}

__global__ void k_merge_setup(Dev d) {
  const int b = blockIdx.x;
  const bool need = d.count[b] > d.box[b].num_thresh;
  if (threadIdx.x == 0) d.need_hist[b] = need ? 1 : 0;
  if (need)
    for (int k = threadIdx.x; k < kPdfBins; k += blockDim.x) d.hist[(size_t)b * kPdfBins + k] = 0;
}

// calc_nphot_merge histogram (ray_tracing.cc:193-209)
__global__ void k_hist(Dev d, const double* lg) {
  const int cur = d.ctl->cur;
  const int n = d.ctl->nray[cur];
  const RayPool A = d.pool[cur];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (d.dead[i]) continue;
    const int b = A.box[i];
    if (!d.need_hist[b]) continue;
    const double lg_min = lg[2 * b], del = lg[2 * b + 1];
    const float v = (float)((log10f(sum_nphot(A, i, d.F, d.ray_cap)) - lg_min) / del);
    int pdf_ind = (int)((v >= 0.f) ? v : 0.f);   // maxd(..., 0.)
    pdf_ind = (pdf_ind >= 9999) ? 9999 : pdf_ind;
    atomicAdd(&d.hist[(size_t)b * kPdfBins + pdf_ind], 1);
  }
}

// threshold scan from the top of the PDF (ray_tracing.cc:211-224), one thread per box
__global__ void k_merge_thresh(Dev d, const double* lg) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nbox) return;
  BoxP& B = d.box[b];
  if (d.need_hist[b]) {
    const double lg_min = lg[2 * b], del = lg[2 * b + 1];
    long long cum = 0;
    float nm = 0.f;
    for (int k = kPdfBins - 1; k >= 0; --k) {
      cum += d.hist[(size_t)b * kPdfBins + k];
      if (cum >= B.num_thresh) {
        nm = (float)pow(10., k * del + lg_min);
        break;
      }
    }
    B.nphot_merge = nm;
  }
  const float a = (float)(4. * (double)B.nphot_merge), c = (float)(4. * B.nphot_min);
  B.split_thr = (c >= a) ? c : a;   // maxd(4.*nphot_merge, 4.*nphot_min)
  if (B.nphot_merge > 0.f) atomicOr(&d.ctl->any_merge, 1);
}

// l_from_r (ray_tracing.cc:87-95)
__device__ __forceinline__ int l_from_r(const BoxP& B, float r, double pi_sf_3, double log4) {
  const double q = (double)(r / B.dx0);
  int l = (int)ceil(log(pi_sf_3 * (q * q)) / log4);
  l = (l >= kLmax) ? kLmax : l;
  const int lmin = B.lm;
  l = (l >= lmin) ? l : lmin;
  l = (kLmax >= l) ? l : kLmax;
  if (r / B.dx0 < 1.) l = lmin;
  return l;
}

// merge pass 1 (ray_tracing.cc:336-357): bin candidates by (cell, pixel at l_merge in the frame
// of this step's random rotation); the smallest pool index in a bin becomes its base ray.
__global__ void k_merge_bin(Dev d) {
  if (!d.ctl->any_merge) return;
  const int cur = d.ctl->cur;
  const int n = d.ctl->nray[cur];
  const RayPool A = d.pool[cur];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    d.ray_bin[i] = -1;
    if (d.dead[i]) continue;
    const BoxP& B = d.box[A.box[i]];
    if (!(B.nphot_merge > 0.f)) continue;
    if (!(sum_nphot(A, i, d.F, d.ray_cap) < B.nphot_merge)) continue;
    const float* m = d.rot + (size_t)d.itheta_merge[A.box[i]] * 18 + 9;   // inverse rotation
    float vx, vy, vz;
    rot_apply(m, A.xh[i], A.yh[i], A.zh[i], &vx, &vy, &vz);
    const int pix = hpn::vec2pix(B.lm, (double)vx, (double)vy, (double)vz);
    const int npix = 12 << (2 * B.lm);
    const long long bin = (B.cell0 + A.cell[i]) * npix + pix;
    d.ray_bin[i] = (int)bin;
    atomicMin(&d.bin_base[bin], i);
  }
}

// base rays start their photon-weighted sums (ray_tracing.cc:362-377)
__global__ void k_merge_base(Dev d) {
  if (!d.ctl->any_merge) return;
  const int cur = d.ctl->cur;
  const int n = d.ctl->nray[cur];
  const RayPool A = d.pool[cur];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int bin = d.ray_bin[i];
    if (bin < 0 || d.bin_base[bin] != i) continue;
    const BoxP& B = d.box[A.box[i]];
    const float nt = sum_nphot(A, i, d.F, d.ray_cap);
    const float rr = A.r[i] / B.dx0;
    A.r[i] = (float)((double)rr * (double)rr * (double)nt);
    A.dr[i] *= nt;
    A.x[i] *= nt;
    A.y[i] *= nt;
    A.z[i] *= nt;
    A.time[i] *= nt;
    d.merged_flag[i] = 0;
  }
}

// other rays of a bin add their photon-weighted quantities to the base and are removed
// (ray_tracing.cc:379-402)
__global__ void k_merge_accum(Dev d) {
  if (!d.ctl->any_merge) return;
  const int cur = d.ctl->cur;
  const int n = d.ctl->nray[cur];
  const RayPool A = d.pool[cur];
  const int cap = d.ray_cap;
  long long merged = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int bin = d.ray_bin[i];
    if (bin < 0) continue;
    const int base = d.bin_base[bin];
    if (base == i) continue;
    const BoxP& B = d.box[A.box[i]];
    const float nt = sum_nphot(A, i, d.F, cap);
    for (int nu = 0; nu < d.F; nu++) atomicAdd(&A.nphot[(size_t)nu * cap + base], A.nphot[(size_t)nu * cap + i]);
    const float rr = A.r[i] / B.dx0;
    atomicAdd(&A.r[base], (float)((double)rr * (double)rr * (double)nt));
    atomicAdd(&A.dr[base], A.dr[i] * nt);
    atomicAdd(&A.x[base], A.x[i] * nt);
    atomicAdd(&A.y[base], A.y[i] * nt);
    atomicAdd(&A.z[base], A.z[i] * nt);
    atomicAdd(&A.time[base], A.time[i] * nt);
    d.merged_flag[base] = 1;
    d.dead[i] = 1;
    d.ray_bin[i] = -1;
    merged += 1;
  }
  merged = block_sum(merged);
  if (threadIdx.x == 0 && merged) atomicAdd((unsigned long long*)&d.ctl->merged, (unsigned long long)merged);
}

// merge pass 2 (ray_tracing.cc:409-476): normalise; bins that merged > 1 ray get the bin's
// direction, an order from the merged radius, and a pixel at that order.
__global__ void k_merge_final(Dev d, double pi_sf_3, double log4) {
  if (!d.ctl->any_merge) return;
  const int cur = d.ctl->cur;
  const int n = d.ctl->nray[cur];
  const RayPool A = d.pool[cur];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int bin = d.ray_bin[i];
    if (bin < 0) continue;
    d.ray_bin[i] = -1;
    const int b = A.box[i];
    const BoxP& B = d.box[b];
    const float nt = sum_nphot(A, i, d.F, d.ray_cap);
    float r = A.r[i] / nt;
    r = (float)sqrt((double)r);
    r *= B.dx0;
    float dr = A.dr[i] / nt;
    A.x[i] /= nt;
    A.y[i] /= nt;
    A.z[i] /= nt;
    A.time[i] /= nt;
    if (d.merged_flag[i]) {
      const int npix = 12 << (2 * B.lm);
      const int pix = bin % npix;
      double vx, vy, vz;
      hpn::pix2vec(B.lm, pix, &vx, &vy, &vz);
      const uint16_t ith = d.itheta_merge[b];
      A.itheta[i] = ith;
      const int order = l_from_r(B, r, pi_sf_3, log4);
      const float rmin = B.rmin[order], rmax = B.rmax[order];
      const float cand = rmax - dr;
      r = (rmin >= cand) ? rmin : cand;    // maxd(rmax - dr, rmin)
      dr = rmax - r;
      A.order[i] = (int16_t)order;
      const int pixel = hpn::vec2pix(order, vx, vy, vz);
      A.pixel[i] = pixel;
      float fx, fy, fz;
      pix_dir(d, order, pixel, &fx, &fy, &fz);
      float ox, oy, oz;
      rot_apply(d.rot + (size_t)ith * 18, fx, fy, fz, &ox, &oy, &oz);
      A.xh[i] = ox;
      A.yh[i] = oy;
      A.zh[i] = oz;
      d.merged_flag[i] = 0;
    }
    A.r[i] = r;
    A.dr[i] = dr;
    d.bin_base[bin] = 0x7fffffff;
  }
}

// split_rays (rt_funcs.cc:211-237) fused with the compaction into the next pool, one kernel.
// A block takes 256 rays of the pool at a time; every thread loads its ray's record (all loads
// issued back to back) and decides how many slots of the next pool it needs: a dead ray none, a
// live ray one, a ray past rmax(l) with enough photons four (its children, split_ray,
// ray_tracing.cc:482-619: pixels 4*pn + c of order l+1, displaced by (v_child - v_parent)
// r0 dx/dx0). One block-wide scan gives each ray its offset and each split ray its rank among
// the block's split rays, and one atomicAdd per block places the block's outputs contiguously. A
// live ray is written by its own thread from registers; a split ray parks its record in shared
// memory and the block's threads then build the children, four per split ray, spread over all
// threads so that the child arithmetic (pixel table, rotation, wrap) runs at full width.
// MODE 0: each block of 256 rays places its outputs at a base taken with one atomicAdd (live rays
// and the children of split rays interleaved in ray order inside the block). MODE 1 only counts
// each block's live and split rays (ord_cnt); k_order_scan turns the counts into offsets; MODE 2
// then writes the live rays in pool order followed by the children in the order of their parents
// (the order the reference's slots take them in: split_rays appends children after the rays it
// keeps, rt_funcs.cc:211-237), which the I-front photon budget needs.
template <int MODE>
__global__ void __launch_bounds__(256, 4) k_compact_split(Dev d, int r_begin, int r_end) {
  // a split ray's record for its children: position, direction and r * scale as the doubles the
  // children's positions are formed in (ray_tracing.cc:586-588), its cell as (i, j, k)
  __shared__ int s_pixel[256], s_dst[256];
  __shared__ int3 s_ijk[256];
  __shared__ double s_pd[3][256], s_hd[3][256], s_rsd[256];
  __shared__ double s_col[2][256];   // the split ray's columns (optical-depth limit on)
  __shared__ float s_r[256], s_time[256];
  __shared__ float s_nph[FRT_MAX_FREQ][256];
  __shared__ uint16_t s_box[256], s_ith[256];
  __shared__ int16_t s_order[256];
  __shared__ int s_wt[8];
  __shared__ int s_tot, s_base;
  const int cur = d.ctl->cur;
  const int nxt = cur ^ 1;
  const int n = min(d.ctl->nray[cur], r_end);   // rays [r_begin, n): see k_advance
  const RayPool A = d.pool[cur];
  const RayPool Bp = d.pool[nxt];
  const int cap = d.ray_cap, F = d.F;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  long long nsplit = 0;
  double inflight = 0.0;
  for (int i0 = r_begin + blockIdx.x * 256; i0 < n; i0 += gridDim.x * 256) {
    const int i = i0 + t;
    int cell = 0, pixel = 0;
    uint16_t bx = 0, ith = 0;
    int16_t order = 0;
    float xh = 0.f, yh = 0.f, zh = 0.f, r = 0.f, dr = 0.f, x = 0.f, y = 0.f, z = 0.f, tm = 0.f, sum = 0.f;
    float nph[FRT_MAX_FREQ];
    bool split = false, live = false;
    if (i < n) {
      // the record is loaded with the dead flag, not after it (every slot below n holds a written
      // record), so that the tile waits for one round trip to memory instead of two
      live = !d.dead[i];
      cell = A.cell[i];
      bx = A.box[i];
      order = A.order[i];
      pixel = A.pixel[i];
      ith = A.itheta[i];
      xh = A.xh[i];
      yh = A.yh[i];
      zh = A.zh[i];
      r = A.r[i];
      dr = A.dr[i];
      x = A.x[i];
      y = A.y[i];
      z = A.z[i];
      tm = A.time[i];
#pragma unroll
      for (int nu = 0; nu < FRT_MAX_FREQ; nu++) {
        nph[nu] = (nu < F) ? A.nphot[(size_t)nu * cap + i] : 0.f;
        sum += (nu < F) ? nph[nu] : 0.f;
      }
      const BoxP& B = d.box[bx];
      split = live && (r > B.rmax[order]) && (order < kLmax) && (sum > B.split_thr);
    }
    // one block-wide exclusive scan: slots (low 16 bits, at most 1024) and split rank (high bits);
    // in the ordered modes the low bits count the live rays that are not split
    const int want = live ? (split ? 4 : 1) : 0;
    const int key = (MODE == 0 ? want : ((live && !split) ? 1 : 0)) | ((split ? 1 : 0) << 16);
    int incl = key;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) s_wt[w] = incl;
    __syncthreads();
    if (w == 0) {
      int v = (lane < 8) ? s_wt[lane] : 0;
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
      }
      if (lane < 8) s_wt[lane] = v;   // inclusive prefix over the warps
      if (lane == 7) {
        s_tot = v;
        if (MODE == 0) {
          const int slots = v & 0xffff;
          s_base = (slots > 0) ? atomicAdd(&d.ctl->nray[nxt], slots) : 0;
        } else if (MODE == 1) {
          d.ord_cnt[(i0 - r_begin) >> 8] = make_int2(v & 0xffff, v >> 16);
        }
      }
    }
    __syncthreads();
    if (MODE == 1) continue;   // (uniform over the block)
    const int excl = (w > 0 ? s_wt[w - 1] : 0) + incl - key;
    const int nsp = s_tot >> 16;
    int j;
    if (MODE == 0) {
      const int base = s_base;
      if (t == 0 && (long long)base + (s_tot & 0xffff) > (long long)cap) atomicOr(&d.ctl->err, ERR_RAY_CAP);
      j = base + (excl & 0xffff);
    } else {
      const int2 off = d.ord_off[(i0 - r_begin) >> 8];
      j = split ? d.ctl->ord_surv + 4 * (off.y + (excl >> 16)) : off.x + (excl & 0xffff);
    }
    if (live && !split) {
      // a live ray: copied by its own thread
      if (j < cap) {
        Bp.cell[j] = cell;
        Bp.box[j] = bx;
        Bp.order[j] = order;
        Bp.pixel[j] = pixel;
        Bp.itheta[j] = ith;
        Bp.xh[j] = xh;
        Bp.yh[j] = yh;
        Bp.zh[j] = zh;
#pragma unroll
        for (int nu = 0; nu < FRT_MAX_FREQ; nu++)
          if (nu < F) Bp.nphot[(size_t)nu * cap + j] = nph[nu];
        Bp.r[j] = r;
        Bp.dr[j] = dr;
        Bp.x[j] = x;
        Bp.y[j] = y;
        Bp.z[j] = z;
        Bp.time[j] = tm;
        if (A.col) {
          Bp.col[j] = A.col[i];
          Bp.col[(size_t)cap + j] = A.col[(size_t)cap + i];
        }
        inflight += (double)sum;
      }
    } else if (split) {
      const int k = excl >> 16;
      nsplit += 1;
      s_dst[k] = j;
      s_pixel[k] = pixel;
      s_box[k] = bx;
      s_ith[k] = ith;
      s_order[k] = order;
      s_hd[0][k] = (double)xh;
      s_hd[1][k] = (double)yh;
      s_hd[2][k] = (double)zh;
      s_r[k] = r;
      const BoxP& B = d.box[bx];
      s_rsd[k] = (double)(r * B.scale);
      s_pd[0][k] = (double)x;
      s_pd[1][k] = (double)y;
      s_pd[2][k] = (double)z;
      int ic, jcl, kc;
      cell_ijk(cell, B.n, B.nn, B.inv_n, B.inv_nn, &ic, &jcl, &kc);
      s_ijk[k] = make_int3(ic, jcl, kc);
      s_time[k] = tm;
      if (A.col) {
        s_col[0][k] = A.col[i];
        s_col[1][k] = A.col[(size_t)cap + i];
      }
#pragma unroll
      for (int nu = 0; nu < FRT_MAX_FREQ; nu++)
        if (nu < F) s_nph[nu][k] = nph[nu];
    }
    __syncthreads();
    // the children, four per split ray of the block, over all threads
    for (int u = t; u < 4 * nsp; u += 256) {
      const int k = u >> 2, c = u & 3;
      const int jc = s_dst[k] + c;
      if (jc >= cap) continue;
      const uint16_t cbx = s_box[k];
      const BoxP& B = d.box[cbx];
      const int N = B.n;
      const int l = s_order[k];
      const int pix = 4 * s_pixel[k] + c;
      const uint16_t cith = s_ith[k];
      const float r0 = s_r[k];
      const double rsd = s_rsd[k];   // (double)(r0 * scale)
      float fx, fy, fz;
      pix_dir(d, l + 1, pix, &fx, &fy, &fz);
      float nx, ny, nz;
      rot_apply(d.rot + (size_t)cith * 18, fx, fy, fz, &nx, &ny, &nz);
      float x0 = (float)(s_pd[0][k] + ((double)nx - s_hd[0][k]) * rsd);
      float y0 = (float)(s_pd[1][k] + ((double)ny - s_hd[1][k]) * rsd);
      float z0 = (float)(s_pd[2][k] + ((double)nz - s_hd[2][k]) * rsd);
      const int3 ijk = s_ijk[k];
      int icn = ijk.x, jcn = ijk.y, kcn = ijk.z;
      // the reference's mod(i +- 1, N) (imod) of an index in [0, N)
      const float dxb = B.dx;
      for (int g = 0; g < 64 && x0 > dxb; g++) { x0 -= dxb; icn = dda_up(icn, N); }
      for (int g = 0; g < 64 && x0 < 0.f; g++) { x0 += dxb; icn = dda_down(icn, N); }
      for (int g = 0; g < 64 && y0 > dxb; g++) { y0 -= dxb; jcn = dda_up(jcn, N); }
      for (int g = 0; g < 64 && y0 < 0.f; g++) { y0 += dxb; jcn = dda_down(jcn, N); }
      for (int g = 0; g < 64 && z0 > dxb; g++) { z0 -= dxb; kcn = dda_up(kcn, N); }
      for (int g = 0; g < 64 && z0 < 0.f; g++) { z0 += dxb; kcn = dda_down(kcn, N); }
      Bp.cell[jc] = icn * B.nn + jcn * N + kcn;
      Bp.box[jc] = cbx;
      Bp.order[jc] = (int16_t)(l + 1);
      Bp.pixel[jc] = pix;
      Bp.itheta[jc] = cith;
      Bp.xh[jc] = nx;
      Bp.yh[jc] = ny;
      Bp.zh[jc] = nz;
      float cs = 0.f;
      for (int nu = 0; nu < F; nu++) {
        // (float)((double)n / 4.) of split_ray: a division by 4 is exact in double, and the float
        // product n * 0.25f rounds the same exact value (also in the subnormal range)
        const float q = s_nph[nu][k] * 0.25f;
        Bp.nphot[(size_t)nu * cap + jc] = q;
        cs += q;
      }
      inflight += (double)cs;
      Bp.r[jc] = r0;
      Bp.dr[jc] = B.rmax[l + 1] - r0;
      Bp.x[jc] = x0;
      Bp.y[jc] = y0;
      Bp.z[jc] = z0;
      Bp.time[jc] = s_time[k];
      if (A.col) {   // children inherit the columns their parent crossed
        Bp.col[jc] = s_col[0][k];
        Bp.col[(size_t)cap + jc] = s_col[1][k];
      }
    }
    __syncthreads();   // the shared records take the next 256 rays
  }
  nsplit = block_sum(nsplit);
  inflight = block_sum(inflight);
  if (threadIdx.x == 0) {
    if (nsplit) atomicAdd((unsigned long long*)&d.ctl->split, (unsigned long long)nsplit);
    if (inflight != 0.0) atomicAdd(&d.ctl->in_flight, inflight * kPhotNorm);
  }
}

// Offsets of the ordered compaction (k_compact_split<1> counts per block of 256 rays): exclusive
// prefixes of the live and of the split rays over the blocks in pool order; the live rays fill
// the front of the next pool and the children follow them.
__global__ void __launch_bounds__(1024) k_order_scan(Dev d) {
  __shared__ int2 wsum[32];
  __shared__ int2 base_s;
  const int cur = d.ctl->cur, nxt = cur ^ 1;
  const long long nchunk = ((long long)d.ctl->nray[cur] + 255) >> 8;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) base_s = make_int2(0, 0);
  __syncthreads();
  for (long long c0 = 0; c0 < nchunk; c0 += blockDim.x) {
    const long long c = c0 + threadIdx.x;
    const int2 v = (c < nchunk) ? d.ord_cnt[c] : make_int2(0, 0);
    int2 incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int ax = __shfl_up_sync(0xffffffffu, incl.x, o), ay = __shfl_up_sync(0xffffffffu, incl.y, o);
      if (lane >= o) {
        incl.x += ax;
        incl.y += ay;
      }
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      int2 u = wsum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int ax = __shfl_up_sync(0xffffffffu, u.x, o), ay = __shfl_up_sync(0xffffffffu, u.y, o);
        if (lane >= o) {
          u.x += ax;
          u.y += ay;
        }
      }
      wsum[lane] = u;   // inclusive prefix over the warps
    }
    __syncthreads();
    if (c < nchunk) {
      const int2 pre = (w > 0) ? wsum[w - 1] : make_int2(0, 0);
      d.ord_off[c] = make_int2(base_s.x + pre.x + incl.x - v.x, base_s.y + pre.y + incl.y - v.y);
    }
    __syncthreads();
    if (threadIdx.x == 0) base_s = make_int2(base_s.x + wsum[31].x, base_s.y + wsum[31].y);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const long long tot = (long long)base_s.x + 4ll * base_s.y;
    if (tot > d.ray_cap) atomicOr(&d.ctl->err, ERR_RAY_CAP);
    d.ctl->ord_surv = base_s.x;
    d.ctl->nray[nxt] = (int)min(tot, (long long)d.ray_cap);
  }
}

__global__ void k_swap(Dev d) {
  Ctl* c = d.ctl;
  const int nxt = c->cur ^ 1;
  const int n = c->nray[nxt];
  c->nray[nxt] = c->err ? 0 : ((n > d.ray_cap) ? d.ray_cap : n);
  c->nray[c->cur] = 0;
  c->cur = nxt;
}

// new_rays -> init_rays (rt_funcs.cc:240-261, ray_tracing.cc:230-321): 12 Nside^2 rays per source
// at the cell centre, directions of the NEST pixels rotated by the source's random angles.
// The ray count of a source's cast (init_rays, ray_tracing.cc:230-245): 12 rays at the base order,
// or 12 nside^2 at the source level lsource when the source cell is no longer neutral.
__device__ __forceinline__ int cast_count(const Dev& d, int s, int* nside_out, int* lpix_out) {
  if (d.src_own && !d.src_own[s]) return 0;   // another context casts this source
  const BoxP& B = d.box[d.src_box[s]];
  const long long gc = B.cell0 + d.src_cell[s];
  int nside = 1, lpix = 0;
  if (!(d.nH1[gc] / d.nH[gc] > 0.1)) {
    nside = 1 << B.lsource;
    lpix = B.lsource;
  }
  *nside_out = nside;
  *lpix_out = lpix;
  return 12 * nside * nside;
}

// The pool positions of the step's new rays: sources in order, each source's rays together in
// pixel order after the live rays (the order new_rays appends them in, rt_funcs.cc:240-261).
// k_cast_count writes each source's ray count into src_pos (many blocks: the counts read the
// source cells' neutral fractions); k_cast_scan then turns the counts into positions in place
// (one block over the sources, coalesced) and moves the pool count past the new rays.
__global__ void k_cast_count(Dev d) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < d.nsrc; s += gridDim.x * blockDim.x) {
    int nside = 1, lpix = 0;
    d.src_pos[s] = cast_count(d, s, &nside, &lpix);
  }
}

__global__ void __launch_bounds__(1024) k_cast_scan(Dev d) {
  __shared__ int wsum[32];
  __shared__ int base_s;
  const int cur = d.ctl->cur;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (threadIdx.x == 0) base_s = d.ctl->nray[cur];
  __syncthreads();
  // each thread takes K consecutive sources per round (one round for up to 16 384 sources): its
  // own sum, one block-wide scan of the sums, then the K positions in order
  constexpr int K = 16;
  for (int s0 = 0; s0 < d.nsrc; s0 += (int)blockDim.x * K) {
    const int sb = s0 + (int)threadIdx.x * K;
    int cnt[K];
    int tot = 0;
#pragma unroll
    for (int k = 0; k < K; k++) {
      cnt[k] = (sb + k < d.nsrc) ? d.src_pos[sb + k] : 0;
      tot += cnt[k];
    }
    int incl = tot;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
      int v = (lane < (int)(blockDim.x >> 5)) ? wsum[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
      }
      wsum[lane] = v;   // inclusive prefix over the warps
    }
    __syncthreads();
    int off = base_s + (w > 0 ? wsum[w - 1] : 0) + incl - tot;
#pragma unroll
    for (int k = 0; k < K; k++)
      if (sb + k < d.nsrc) {
        d.src_pos[sb + k] = off;
        off += cnt[k];
      }
    __syncthreads();
    if (threadIdx.x == 0) base_s += wsum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (base_s > d.ray_cap) atomicOr(&d.ctl->err, ERR_RAY_CAP);
    d.ctl->nray[cur] = min(base_s, d.ray_cap);
  }
}

__global__ void k_cast(Dev d, int s_begin, int s_end) {
  const int cur = d.ctl->cur;
  const RayPool A = d.pool[cur];
  const int cap = d.ray_cap, F = d.F;
  long long ncast = 0;
  double emitted = 0.0;
  for (int s = s_begin + blockIdx.x * blockDim.x + threadIdx.x; s < s_end; s += gridDim.x * blockDim.x) {
    int nside = 1, lpix = 0;
    const int count = cast_count(d, s, &nside, &lpix);
    if (count == 0) continue;
    const int b = d.src_box[s];
    const BoxP& B = d.box[b];
    const int c = d.src_cell[s];
    const int pos = d.src_pos[s];   // k_cast_scan
    if (pos + count > cap) continue;   // (k_cast_scan flagged the overflow)
    const uint16_t ith = d.src_itheta[s];
    const float* m = d.rot + (size_t)ith * 18;
    const double lum = d.src_lum[s];
    const float rdt = d.src_ray_dt[s];
    float np[FRT_MAX_FREQ];
    double tot = 0.0;
    for (int nu = 0; nu < F; nu++) {
      np[nu] = (float)((double)d.spectrum[nu] * lum * (double)rdt / 12. / (double)(nside * nside) / kPhotNorm);
      tot += (double)np[nu];
    }
    for (int p = 0; p < count; p++) {
      const int j = pos + p;
      float fx, fy, fz;
      pix_dir(d, lpix, p, &fx, &fy, &fz);
      float ox, oy, oz;
      rot_apply(m, fx, fy, fz, &ox, &oy, &oz);
      A.cell[j] = c;
      A.box[j] = (uint16_t)b;
      A.order[j] = (int16_t)lpix;
      A.pixel[j] = p;
      A.itheta[j] = ith;
      A.xh[j] = ox;
      A.yh[j] = oy;
      A.zh[j] = oz;
      for (int nu = 0; nu < F; nu++) A.nphot[(size_t)nu * cap + j] = np[nu];
      A.r[j] = 0.f;
      A.dr[j] = B.rmax[lpix] - 0.f;
      A.x[j] = B.dx_half;
      A.y[j] = B.dx_half;
      A.z[j] = B.dx_half;
      A.time[j] = 0.f;
      if (A.col) {   // optical-depth limit on: no column crossed yet
        A.col[j] = 0.0;
        A.col[(size_t)cap + j] = 0.0;
      }
    }
    d.src_ray_dt[s] = 0.f;
    ncast += count;
    emitted += tot * count;
  }
  ncast = block_sum(ncast);
  emitted = block_sum(emitted);
  if (threadIdx.x == 0) {
    if (ncast) atomicAdd((unsigned long long*)&d.ctl->cast, (unsigned long long)ncast);
    if (emitted != 0.0) {
      atomicAdd(&d.ctl->emitted, emitted * kPhotNorm);
      atomicAdd(&d.ctl->in_flight, emitted * kPhotNorm);
    }
  }
}

// update_cosmo_expansion (gas_funcs.cc:460-548) for one box, plain mode (fion = 1): the proper
// density scales by (a_prev/a)^3 (rho_factor, computed on the host in double as the reference
// does), the number densities follow from it and the stored ionised fractions (f_H2 = nH2/nH and
// f_He2 = nHe2/nHe as the last C2Ray update left them, f_He3 = 0), and the rays' positions in their
// cells scale by a/a_prev (ratio) with the corner nudges of the new cell size (already in the box).
__global__ void k_cosmo_cells(Dev d, int box, double rho_factor) {
  const BoxP& B = d.box[box];
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < B.ncell;
       c += (long long)gridDim.x * blockDim.x) {
    const long long q = B.cell0 + c;
    const float nH0 = d.nH[q], nHe0 = d.nHe[q];
    // the ionised fractions of the last cell pass (f_H2 = nH2 / nH with nH2 = nH - nH1,
    // ray_tracing.cc:1119, 1192); kept for a snapshot switch that follows this expansion
    const float f_H2 = (nH0 - d.nH1[q]) / nH0;
    const float f_He2 = (nHe0 - d.nHe1[q]) / nHe0;
    if (d.frac_h2) {
      d.frac_h2[q] = f_H2;
      d.frac_he2[q] = f_He2;
    }
    float rho = d.rho[q];
    rho *= rho_factor;
    d.rho[q] = rho;
    const float nH = (1. - kY) * rho / kMH;
    const float nHe = kY * rho / (4. * kMH);
    const float nH2 = f_H2 * nH / 1.0f;
    const float nHe2 = f_He2 * nHe / 1.0f;
    const float nH1 = nH - nH2;
    const float nHe1 = nHe - nHe2;
    const float ne = nH2 + nHe2;
    d.nH[q] = nH;
    d.nHe[q] = nHe;
    d.nH1[q] = nH1;
    d.nHe1[q] = nHe1;
    d.avg_nh1[q] = nH1;
    d.avg_nhe1[q] = nHe1;
    d.ne[q] = ne;
    d.n_tot[q] = nH + nHe + ne;
    d.nH1_prev[q] = nH1;
  }
}

// update_hydro_step's cell update for a later snapshot (gas_funcs.cc:686-745, fion = 1 in plain
// mode): n_H, n_He from the new proper density (already in d.rho), the ionised densities keep the
// fractions f_HII, f_HeII (of the last cell pass, or the ones an expansion just before this
// switch kept), n_HI = n_H - n_HII, <n_HI> = n_HI, n_e, n_tot; with a previous snapshot
// (avg_rho_prev > 0) d(delta)/dt = (rho/<rho> - rho_prev/<rho_prev>) / dt_snap; rho_prev = rho.
__global__ void k_hydro_cells(Dev d, int box, bool cached, float avg_rho_prev, float dt_snap) {
  const BoxP& B = d.box[box];
  const float avg_rho = B.avg_rho;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < B.ncell;
       c += (long long)gridDim.x * blockDim.x) {
    const long long q = B.cell0 + c;
    float f_H2, f_He2;
    if (cached) {
      f_H2 = d.frac_h2[q];
      f_He2 = d.frac_he2[q];
    } else {
      const float nH0 = d.nH[q], nHe0 = d.nHe[q];
      f_H2 = (nH0 - d.nH1[q]) / nH0;
      f_He2 = (nHe0 - d.nHe1[q]) / nHe0;
    }
    const float rho = d.rho[q];
    const float nH = (1. - kY) * rho / kMH;
    const float nHe = kY * rho / (4. * kMH);
    const float nH2 = f_H2 * nH / 1.0f;
    const float nHe2 = f_He2 * nHe / 1.0f;
    const float nH1 = nH - nH2;
    const float nHe1 = nHe - nHe2;
    const float ne = nH2 + nHe2;
    d.nH[q] = nH;
    d.nHe[q] = nHe;
    d.nH1[q] = nH1;
    d.nHe1[q] = nHe1;
    d.avg_nh1[q] = nH1;
    d.avg_nhe1[q] = nHe1;
    d.ne[q] = ne;
    d.n_tot[q] = nH + nHe + ne;
    d.nH1_prev[q] = nH1;
    if (avg_rho_prev > 0.f) d.ddelta[q] = (rho / avg_rho - d.rho_prev[q] / avg_rho_prev) / dt_snap;
    d.rho_prev[q] = rho;
  }
}

__global__ void k_cosmo_rays(Dev d, int box, float ratio) {
  const int cur = d.ctl->cur;
  const int n = d.ctl->nray[cur];
  const RayPool A = d.pool[cur];
  const BoxP& B = d.box[box];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (A.box[i] != box) continue;
    float x = A.x[i], y = A.y[i], z = A.z[i];
    x *= ratio;
    y *= ratio;
    z *= ratio;
    if (x <= 0.f) x = B.lo_edge;
    if (x >= B.hi_thr_f) x = B.hi_edge;
    if (y <= 0.f) y = B.lo_edge;
    if (y >= B.hi_thr_f) y = B.hi_edge;
    if (z <= 0.f) z = B.lo_edge;
    if (z >= B.hi_thr_f) z = B.hi_edge;
    A.x[i] = x;
    A.y[i] = y;
    A.z[i] = z;
  }
}

__global__ void k_fill_i32(int* p, int v, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

}  // namespace

// ---- launchers ------------------------------------------------------------------------------
void launch_step_begin(const Dev& d, cudaStream_t s) { k_step_begin<<<grid_for(d.nsrc + 1, 256, 1184), 256, 0, s>>>(d); }

// k_advance's dynamic shared memory holds a tile's segments: block * path_length * 8 bytes
// (32 KB at most: 256 threads, FRT_MAX_PATH = 16)
static void launch_k_advance(const Dev& d, int grid, int block, int r_begin, int r_end, cudaStream_t s) {
  if (block <= 128) k_advance<128><<<grid, 128, sizeof(int2) * 128 * d.PL, s>>>(d, r_begin, r_end);
  else k_advance<256><<<grid, 256, sizeof(int2) * 256 * d.PL, s>>>(d, r_begin, r_end);
}

void launch_advance(const Dev& d, int grid, cudaStream_t s, int block, int pack_grid) {
  launch_k_advance(d, grid, block, 0, INT_MAX, s);
  k_lit_compact<<<grid_for(d.ncell_total >> 4, 256, 148 * 8), 256, 0, s>>>(d);
  k_pk_slots<<<pack_grid > 0 ? pack_grid : resident_grid(k_pk_slots, 256), 256, 0, s>>>(d);
}

void launch_walk(const Dev& d, int grid, cudaStream_t s, int block, int r_begin, int r_end) {
  launch_k_advance(d, grid, block, r_begin, r_end, s);
}

void launch_lit_number(const Dev& d, int grid, cudaStream_t s) {
  k_lit_compact<<<grid_for(d.ncell_total >> 4, 256, 148 * 8), 256, 0, s>>>(d);
  k_pk_slots<<<resident_grid(k_pk_slots, 256), 256, 0, s>>>(d);
}

void launch_lit_number_ordered(const Dev& d, int* chunk, long long nchunk, int grid, cudaStream_t s) {
  k_lit_chunk_count<<<grid, 256, 0, s>>>(d, chunk, nchunk);
  k_lit_chunk_scan<<<1, 1024, 0, s>>>(d, chunk, nchunk);
  k_lit_chunk_write<<<grid, 256, 0, s>>>(d, chunk, nchunk);
  k_pk_slots<<<resident_grid(k_pk_slots, 256), 256, 0, s>>>(d);
}

void launch_count(const Dev& d, int grid, cudaStream_t s) {
  cudaMemsetAsync(d.count, 0, sizeof(long long) * d.nbox, s);
  k_count<<<grid, 256, 0, s>>>(d);
}

// The step's count_rays + merge: when no box can reach its merge threshold with this pool size
// (no merge bins), the per-box counts cannot exceed a threshold, so only the split thresholds are
// refreshed (k_merge_thresh, with every need_hist at its initial 0).
void launch_count_merge(const Dev& d, int grid, cudaStream_t s) {
  if (d.bin_base) {
    launch_count(d, grid, s);
    launch_merge(d, grid, s);
  } else {
    k_merge_thresh<<<grid_for(d.nbox, 128, 1024), 128, 0, s>>>(d, d.lg);
  }
}

void launch_merge(const Dev& d, int grid, cudaStream_t s) {
  k_merge_setup<<<d.nbox, 256, 0, s>>>(d);
  k_hist<<<grid, 256, 0, s>>>(d, d.lg);
  k_merge_thresh<<<grid_for(d.nbox, 128, 1024), 128, 0, s>>>(d, d.lg);
  if (d.bin_base) {
    k_merge_bin<<<grid, 256, 0, s>>>(d);
    k_merge_base<<<grid, 256, 0, s>>>(d);
    k_merge_accum<<<grid, 256, 0, s>>>(d);
    k_merge_final<<<grid, 256, 0, s>>>(d, d.pi_sf_3, d.log4);
  }
}

void launch_split_compact(const Dev& d, int grid, cudaStream_t s) {
  if (d.ordered) {
    k_compact_split<1><<<grid, 256, 0, s>>>(d, 0, INT_MAX);
    k_order_scan<<<1, 1024, 0, s>>>(d);
    k_compact_split<2><<<grid, 256, 0, s>>>(d, 0, INT_MAX);
  } else {
    k_compact_split<0><<<grid, 256, 0, s>>>(d, 0, INT_MAX);
  }
  k_swap<<<1, 1, 0, s>>>(d);
}

void launch_split_range(const Dev& d, int grid, int r_begin, int r_end, cudaStream_t s) {
  k_compact_split<0><<<grid, 256, 0, s>>>(d, r_begin, r_end);
}

void launch_swap(const Dev& d, cudaStream_t s) { k_swap<<<1, 1, 0, s>>>(d); }

void launch_cast_positions(const Dev& d, cudaStream_t s) {
  k_cast_count<<<grid_for(d.nsrc, 256, 4096), 256, 0, s>>>(d);
  k_cast_scan<<<1, 1024, 0, s>>>(d);
}

void launch_cast(const Dev& d, cudaStream_t s) {
  if (d.nsrc > 0) {
    launch_cast_positions(d, s);
    k_cast<<<grid_for(d.nsrc, 128, 4096), 128, 0, s>>>(d, 0, d.nsrc);
  }
}

void launch_cast_per_source(const Dev& d, cudaStream_t s) {
  if (d.nsrc > 0) launch_cast_positions(d, s);
  for (int src = 0; src < d.nsrc; src++) k_cast<<<1, 32, 0, s>>>(d, src, src + 1);
}

void launch_cosmo_expansion(const Dev& d, int box, float ratio, double rho_factor, int grid, cudaStream_t s) {
  k_cosmo_cells<<<grid, 256, 0, s>>>(d, box, rho_factor);
  k_cosmo_rays<<<grid, 256, 0, s>>>(d, box, ratio);
}

void launch_hydro_switch(const Dev& d, int box, bool cached_fractions, float avg_rho_prev, float dt_snap, int grid,
                         cudaStream_t s) {
  k_hydro_cells<<<grid, 256, 0, s>>>(d, box, cached_fractions, avg_rho_prev, dt_snap);
}

void launch_pix_table(float4* tab, cudaStream_t s) { k_pix_table<<<148 * 8, 256, 0, s>>>(tab); }

void launch_fill_i32(int* p, int v, long long n, cudaStream_t s) {
  k_fill_i32<<<grid_for(n, 256, 4096), 256, 0, s>>>(p, v, n);
}

}  // namespace frt
