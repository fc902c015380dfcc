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
__host__ __device__ __forceinline__ int dda_up(int i, int N) { return (i + 1 == N) ? 0 : i + 1; }
__host__ __device__ __forceinline__ int dda_down(int i, int N) { return (i == 0) ? N - 1 : i - 1; }

// A float reciprocal for the approximate face times: the hardware approximation on the device
// (PTX rcp.approx.ftz.f32, at most 1 ulp from 1/v for normal v), the IEEE division on the host,
// where the walk is compiled for the CPU test of its face-time ranking.
__host__ __device__ __forceinline__ float rcp_face(float v) {
#ifdef __CUDA_ARCH__
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(v));
  return y;
#else
  return 1.0f / v;
#endif
}

// The (i, j, k) of a box-local cell index ind = i NN + j N + k (NN = N^2) by double-precision
// products with the box's reciprocals instead of integer divisions: (ind + 1/2) / NN lies at
// least 1/(2 NN) from an integer, the computed product differs from it by less than
// (ind + 1/2) / NN * 2^-52 (the reciprocal's rounding and the product's), which is below
// 1/(2 NN) for every ind < 2^31, so truncation gives the exact quotient; likewise for N.
__host__ __device__ __forceinline__ void cell_ijk(int ind, int N, int NN, double inv_n, double inv_nn, int* i, int* j,
                                                  int* k) {
  const int ii = (int)(((double)ind + 0.5) * inv_nn);
  const int r = ind - ii * NN;
  const int jj = (int)(((double)r + 0.5) * inv_n);
  *i = ii;
  *j = jj;
  *k = r - jj * N;
}

// Does the ray, moved by dist, leave its cell this step (ray_tracing.cc:1243-1250)?
__device__ __forceinline__ bool ray_moves(const BoxP& B, float x0, float y0, float z0, float xhat, float yhat,
                                          float zhat, float dist) {
  const float px = x0 + dist * xhat, py = y0 + dist * yhat, pz = z0 + dist * zhat;
  return (px > B.mv_hi) || (py > B.mv_hi) || (pz > B.mv_hi) || (px < B.mv_lo_f) || (py < B.mv_lo_f) ||
         (pz < B.mv_lo_f);   // (double)p < mv_lo, compared in float
}

// The reference's time to the next cell face along one axis (ray_tracing.cc:1273-1296): a float
// quotient for a positive direction component, ((dx - x0) / xhat) / clight in float, a double one
// rounded to float for a negative component, (float)((-x0 / xhat) / clight) in double, infinity
// for a zero component.
__host__ __device__ __forceinline__ float face_time(float pos, float hat, float dxc, float clgt, double cld) {
  if (hat > 0.f) return (dxc - pos) / hat / clgt;
  if (hat < 0.f) return (float)(-1. * (double)pos / (double)hat / cld);
  return INFINITY;
}

// The same time for a nonzero component as one instruction sequence for both signs, so that the
// lanes of a warp never split between a float and a double path. The float quotients of the
// positive case are formed as double quotients rounded to float: for binary32 operands a binary64
// quotient rounded to binary32 is the correctly rounded binary32 quotient, because 53 >= 2*24 + 2
// (double rounding is innocuous for the basic operations under that condition; Figueroa, "When is
// double rounding innocuous?", SIGNUM Newsletter 30(3), 1995), so each of the two roundings
// equals the float division's.
__host__ __device__ __forceinline__ float face_time_nz(float pos, float hat, float dxc, double cld) {
  const bool pos_dir = hat > 0.f;
  const double num = pos_dir ? (double)(dxc - pos) : -1. * (double)pos;
  double q = num / (double)hat;
  if (pos_dir) q = (double)(float)q;   // the float quotient (dx - x0) / xhat
  return (float)(q / cld);
}

// Approximate face times rank the axes; the exact expression is evaluated only for the axes that
// can be the smallest. For a nonzero component the approximation is the face distance times a
// reciprocal of |hat| * clight within 1 ulp: with the product's two roundings it is within
// 4 * 2^-24 relative of the true quotient, and the exact value (two float roundings, or a
// double-to-float one) within 2 * 2^-24, so the two differ by less than 6 * 2^-24 (~2^-21.4).
// An axis whose approximation exceeds the smallest approximation by more than 2^-18 relative is
// therefore strictly slower than the exact minimum under every rounding, can neither be the
// minimum nor tie with it, and its exact time is never needed; the walk selects the same axis and
// the same float tmin as the reference's three exact quotients.
constexpr float kFaceBand = 1.0f + 1.0f / 262144.0f;   // 1 + 2^-18

// Walk c_sim * deltat from (x0, y0, z0) in cell (in, jn, kn): calls seg(p, global cell, dist)
// for each path segment in order and returns their number, or -1 when more than PL segments
// would be needed. On return x0..z0 and in..kn hold the end position and cell, with the
// reference's corner nudges applied. With I-front tracking (fion not null) the last segment in a
// cell the fronts have not fully passed is the whole crossing of the cell (ray_tracing.cc:1425-1437).
template <typename SegFn>
__host__ __device__ __forceinline__ int dda_walk(const BoxP& B, int PL, float xhat, float yhat, float zhat, float deltat,
                                        float& x0, float& y0, float& z0, int& in, int& jn, int& kn, SegFn seg,
                                        const float* fion = nullptr) {
  // the box constants in registers: the segment callback stores to global memory, after which
  // the compiler would otherwise reload every BoxP field the loop reads
  const int N = B.n, NN = B.nn;
  const long long cell0 = B.cell0;
  const float clgt = B.clight;
  const float dxc = B.dx;
  const float lo_edge = B.lo_edge, hi_edge = B.hi_edge, hi_thr = B.hi_thr_f;
  const double cld = (double)clgt;
  // reciprocals of |hat| * clight for the approximate face times; a ray whose reciprocals are not
  // normal floats (a component so small or so large that the product leaves the normal range)
  // takes the exact times of all three axes at every face, and so does a face whose smallest
  // approximate time is below 1e-30 (where a product could leave the normal range)
  const float ivx = rcp_face(fabsf(xhat) * clgt), ivy = rcp_face(fabsf(yhat) * clgt),
              ivz = rcp_face(fabsf(zhat) * clgt);
  const float kLo = 1.2e-38f, kHi = 3.0e38f;
  const bool approx_ok = (xhat == 0.f || (ivx > kLo && ivx < kHi)) && (yhat == 0.f || (ivy > kLo && ivy < kHi)) &&
                         (zhat == 0.f || (ivz > kLo && ivz < kHi));
  float tlast = 0.f, tmin = 0.f, dist;
  int p = 0;
  while (tlast < deltat) {
    const float ax = (xhat > 0.f) ? (dxc - x0) * ivx : ((xhat < 0.f) ? x0 * ivx : INFINITY);
    const float ay = (yhat > 0.f) ? (dxc - y0) * ivy : ((yhat < 0.f) ? y0 * ivy : INFINITY);
    const float az = (zhat > 0.f) ? (dxc - z0) * ivz : ((zhat < 0.f) ? z0 * ivz : INFINITY);
    const float band = fminf(ax, fminf(ay, az)) * kFaceBand;
    const unsigned cand = (ax <= band ? 1u : 0u) | (ay <= band ? 2u : 0u) | (az <= band ? 4u : 0u);
    const bool ranked = approx_ok && band >= 1e-30f;
    int tag;
    if (ranked && (cand == 1u || cand == 2u || cand == 4u)) {
      // one axis can be the smallest: its exact time only
      tag = (cand == 1u) ? 0 : ((cand == 2u) ? 1 : 2);
      const float pos = (tag == 0) ? x0 : ((tag == 1) ? y0 : z0);
      const float hat = (tag == 0) ? xhat : ((tag == 1) ? yhat : zhat);
      tmin = face_time_nz(pos, hat, dxc, cld);   // (an axis with a finite approximation: hat != 0)
    } else {
      // near-ties (or no usable approximation): the exact times of the candidate axes, the
      // others slower than the minimum, and the reference's tie rule
      const unsigned m = (ranked && cand) ? cand : 7u;
      const float tx = (m & 1u) ? face_time(x0, xhat, dxc, clgt, cld) : INFINITY;
      const float ty = (m & 2u) ? face_time(y0, yhat, dxc, clgt, cld) : INFINITY;
      const float tz = (m & 4u) ? face_time(z0, zhat, dxc, clgt, cld) : INFINITY;
      if ((tx <= ty) && (tx <= tz)) { tmin = tx; tag = 0; }
      else if ((ty <= tx) && (ty <= tz)) { tmin = ty; tag = 1; }
      else { tmin = tz; tag = 2; }
    }
    if ((tlast + tmin) < deltat) {
      dist = tmin * clgt;
      if (p >= PL - 1) return -1;
      seg(p, cell0 + (long long)in * NN + jn * N + kn, dist);
      p += 1;
      x0 += dist * xhat;
      y0 += dist * yhat;
      z0 += dist * zhat;
      if (tag == 0) {
        if (xhat > 0.f) { in = dda_up(in, N); x0 = lo_edge; }
        else { in = dda_down(in, N); x0 = hi_edge; }
      } else if (tag == 1) {
        if (yhat > 0.f) { jn = dda_up(jn, N); y0 = lo_edge; }
        else { jn = dda_down(jn, N); y0 = hi_edge; }
      } else {
        if (zhat > 0.f) { kn = dda_up(kn, N); z0 = lo_edge; }
        else { kn = dda_down(kn, N); z0 = hi_edge; }
      }
      if (x0 <= 0.f) x0 = lo_edge;
      if (x0 >= hi_thr) x0 = hi_edge;
      if (y0 <= 0.f) y0 = lo_edge;
      if (y0 >= hi_thr) y0 = hi_edge;
      if (z0 <= 0.f) z0 = lo_edge;
      if (z0 >= hi_thr) z0 = hi_edge;
    }
    tlast += tmin;
  }
  const long long gc_last = cell0 + (long long)in * NN + jn * N + kn;
  if (fion && fion[gc_last] < 1.f) dist = tmin * clgt;
  else dist = (deltat - tlast + tmin) * clgt;
  dist = (lo_edge >= dist) ? lo_edge : dist;   // maxd(dist, min_dist*dx)
  seg(p, gc_last, dist);
  x0 += dist * xhat;
  y0 += dist * yhat;
  z0 += dist * zhat;
  if (x0 <= 0.f) x0 = lo_edge;
  if (x0 >= hi_thr) x0 = hi_edge;
  if (y0 <= 0.f) y0 = lo_edge;
  if (y0 >= hi_thr) y0 = hi_edge;
  if (z0 <= 0.f) z0 = lo_edge;
  if (z0 >= hi_thr) z0 = hi_edge;
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
