// The cell-boundary walk of advance_ray (ray_tracing.cc:1222-1512, plain mode), shared by the
// step's advance (frt_geom.cu) and the adjoint's segment recomputation (frt_adjoint.cu). Both
// translation units are compiled with -fmad=false: the walk reproduces the reference's float
// expressions (and its double sub-expressions for rays moving in -x, -y, -z), so the cells and
// distances of the segments are those of the reference to the last bit.
#pragma once
#include <math.h>

#include "frt_internal.cuh"

namespace frt {

// The periodic neighbours of a cell index i in [0, N): the reference's mod(i +- 1, N) without an
// integer division.
__device__ __forceinline__ int dda_up(int i, int N) { return (i + 1 == N) ? 0 : i + 1; }
__device__ __forceinline__ int dda_down(int i, int N) { return (i == 0) ? N - 1 : i - 1; }

// Does the ray, moved by dist, leave its cell this step (ray_tracing.cc:1243-1250)?
__device__ __forceinline__ bool ray_moves(const BoxP& B, float x0, float y0, float z0, float xhat, float yhat,
                                          float zhat, float dist) {
  const float px = x0 + dist * xhat, py = y0 + dist * yhat, pz = z0 + dist * zhat;
  return (px > B.mv_hi) || (py > B.mv_hi) || (pz > B.mv_hi) || (px < B.mv_lo_f) || (py < B.mv_lo_f) ||
         (pz < B.mv_lo_f);   // (double)p < mv_lo, compared in float
}

// Walk c_sim * deltat from (x0, y0, z0) in cell (in, jn, kn): calls seg(p, global cell, dist)
// for each path segment in order and returns their number, or -1 when more than PL segments
// would be needed. On return x0..z0 and in..kn hold the end position and cell, with the
// reference's corner nudges applied. With I-front tracking (fion not null) the last segment in a
// cell the fronts have not fully passed is the whole crossing of the cell (ray_tracing.cc:1425-1437).
template <typename SegFn>
__device__ __forceinline__ int dda_walk(const BoxP& B, int PL, float xhat, float yhat, float zhat, float deltat,
                                        float& x0, float& y0, float& z0, int& in, int& jn, int& kn, SegFn seg,
                                        const float* fion = nullptr) {
  const int N = B.n;
  const float clgt = B.clight;
  const float dxc = B.dx;
  // the double operands of the -x, -y, -z face times that do not change along the walk
  const double xhd = (double)xhat, yhd = (double)yhat, zhd = (double)zhat, cld = (double)clgt;
  float tlast = 0.f, tmin = 0.f, dist;
  int p = 0;
  while (tlast < deltat) {
    float tx, ty, tz;
    if (xhat > 0.f) tx = (dxc - x0) / xhat / clgt;
    else if (xhat < 0.f) tx = (float)(-1. * (double)x0 / xhd / cld);
    else tx = INFINITY;
    if (yhat > 0.f) ty = (dxc - y0) / yhat / clgt;
    else if (yhat < 0.f) ty = (float)(-1. * (double)y0 / yhd / cld);
    else ty = INFINITY;
    if (zhat > 0.f) tz = (dxc - z0) / zhat / clgt;
    else if (zhat < 0.f) tz = (float)(-1. * (double)z0 / zhd / cld);
    else tz = INFINITY;
    int tag;
    if ((tx <= ty) && (tx <= tz)) { tmin = tx; tag = 0; }
    else if ((ty <= tx) && (ty <= tz)) { tmin = ty; tag = 1; }
    else { tmin = tz; tag = 2; }
    if ((tlast + tmin) < deltat) {
      dist = tmin * clgt;
      if (p >= PL - 1) return -1;
      seg(p, B.cell0 + (long long)in * B.nn + jn * N + kn, dist);
      p += 1;
      x0 += dist * xhat;
      y0 += dist * yhat;
      z0 += dist * zhat;
      if (tag == 0) {
        if (xhat > 0.f) { in = dda_up(in, N); x0 = B.lo_edge; }
        else { in = dda_down(in, N); x0 = B.hi_edge; }
      } else if (tag == 1) {
        if (yhat > 0.f) { jn = dda_up(jn, N); y0 = B.lo_edge; }
        else { jn = dda_down(jn, N); y0 = B.hi_edge; }
      } else {
        if (zhat > 0.f) { kn = dda_up(kn, N); z0 = B.lo_edge; }
        else { kn = dda_down(kn, N); z0 = B.hi_edge; }
      }
      if (x0 <= 0.f) x0 = B.lo_edge;
      if (x0 >= B.hi_thr_f) x0 = B.hi_edge;
      if (y0 <= 0.f) y0 = B.lo_edge;
      if (y0 >= B.hi_thr_f) y0 = B.hi_edge;
      if (z0 <= 0.f) z0 = B.lo_edge;
      if (z0 >= B.hi_thr_f) z0 = B.hi_edge;
    }
    tlast += tmin;
  }
  const long long gc_last = B.cell0 + (long long)in * B.nn + jn * N + kn;
  if (fion && fion[gc_last] < 1.f) dist = tmin * clgt;
  else dist = (deltat - tlast + tmin) * clgt;
  dist = (B.lo_edge >= dist) ? B.lo_edge : dist;   // maxd(dist, min_dist*dx)
  seg(p, gc_last, dist);
  x0 += dist * xhat;
  y0 += dist * yhat;
  z0 += dist * zhat;
  if (x0 <= 0.f) x0 = B.lo_edge;
  if (x0 >= B.hi_thr_f) x0 = B.hi_edge;
  if (y0 <= 0.f) y0 = B.lo_edge;
  if (y0 >= B.hi_thr_f) y0 = B.hi_edge;
  if (z0 <= 0.f) z0 = B.lo_edge;
  if (z0 >= B.hi_thr_f) z0 = B.hi_edge;
  return p + 1;
}

// Number the cells whose flag byte is 1 in cell order: each thread takes 16 consecutive flags
// (one 16-byte load; a flag byte is 0 or 1, so the popcount of a word is its number of marked
// cells), a block-wide scan gives every thread its offset and one atomicAdd per block its base.
// Slots are in ascending cell order inside each block's 4096 cells. ncell is a multiple of 16 and
// flags is 16-byte aligned. Slots beyond cap set errbit in *err.
__device__ __forceinline__ void compact_marked(const uint8_t* flag, long long ncell, int* slot, int* cell, int* count,
                                               int cap, unsigned* err, unsigned errbit) {
  __shared__ int warp_tot[8];
  __shared__ int base_s;
  const long long nvec = ncell >> 4;
  const uint4* flags = reinterpret_cast<const uint4*>(flag);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (long long v0 = (long long)blockIdx.x * blockDim.x; v0 < nvec; v0 += (long long)gridDim.x * blockDim.x) {
    const long long v = v0 + threadIdx.x;
    uint4 f = make_uint4(0u, 0u, 0u, 0u);
    if (v < nvec) f = flags[v];
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
      if (lane < 8) warp_tot[lane] = x;   // inclusive prefix over the warps
      if (lane == 7) base_s = (x > 0) ? atomicAdd(count, x) : 0;
    }
    __syncthreads();
    int s = base_s + (w > 0 ? warp_tot[w - 1] : 0) + incl - cnt;
    if (cnt) {
      const unsigned words[4] = {f.x, f.y, f.z, f.w};
      for (int q = 0; q < 4; q++) {
        unsigned m = words[q];
        while (m) {
          const int bit = __ffs(m) - 1;   // flag bytes hold 0 or 1: bit 8k is byte k
          m &= m - 1;
          const long long gc = v * 16 + q * 4 + (bit >> 3);
          if (s < cap) {
            cell[s] = (int)gc;
            slot[gc] = s;
          } else {
            atomicOr(err, errbit);
          }
          s++;
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace frt
