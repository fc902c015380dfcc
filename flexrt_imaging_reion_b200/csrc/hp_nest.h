// HEALPix NEST pixelisation (pix2vec / vec2pix) for host and device.
//
// Written from the published scheme of Gorski et al. 2005, ApJ 622:759 (sections 4-5:
// the 12 base faces, ring index j_r, azimuthal index j_phi, the polar-cap and equatorial
// z(j_r) formulas, and the bit-interleaved NEST numbering inside a face). The reference
// links the external HEALPix 3.40 C++ library (T_Healpix_Base<int>(order, NEST).pix2vec /
// .vec2pix, call sites ray_tracing.cc:255,290,348,357,421,444,458-461,515-516,520,533);
// that library is not available here, so results are NOT pinned against it.
//
// What IS guaranteed: the host build of this header (used by the CPU oracle's HEALPix shim)
// and the device build (used by the CUDA kernels) return bit-identical results, because
// every transcendental used here (sin, cos, atan2) is evaluated by the own-code series
// below with plain IEEE double +,-,*,/ and sqrt (correctly rounded on both sides). The
// translation units that include this header must not contract a*b+c into FMA
// (host: -ffp-contract=off, device: -fmad=false).
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define HPN_FN __host__ __device__ inline
#else
#define HPN_FN static inline
#endif

namespace hpn {

// pi/2 as a rounded head and the remainder (pi/2 - head), both exact mathematical values.
#define HPN_PIO2_HI 1.5707963267948966
#define HPN_PIO2_LO 6.123233995736766e-17
#define HPN_PI 3.141592653589793
#define HPN_PI_6 0.5235987755982989
#define HPN_SQRT3 1.7320508075688772
#define HPN_TWO_OVER_PI 0.6366197723675814

// sin and cos of |r| <= pi/4 from their Taylor series (terms through r^21 / r^20; the
// truncation error is below 1e-21 there), evaluated in Horner form in r^2.
HPN_FN double sin_series(double r) {
  const double r2 = r * r;
  double p = 1.0 / 51090942171709440000.0;        // +1/21!
  p = p * r2 - 1.0 / 121645100408832000.0;        // -1/19!
  p = p * r2 + 1.0 / 355687428096000.0;           // +1/17!
  p = p * r2 - 1.0 / 1307674368000.0;             // -1/15!
  p = p * r2 + 1.0 / 6227020800.0;                // +1/13!
  p = p * r2 - 1.0 / 39916800.0;                  // -1/11!
  p = p * r2 + 1.0 / 362880.0;                    // +1/9!
  p = p * r2 - 1.0 / 5040.0;                      // -1/7!
  p = p * r2 + 1.0 / 120.0;                       // +1/5!
  p = p * r2 - 1.0 / 6.0;                         // -1/3!
  return r + r * (r2 * p);
}

HPN_FN double cos_series(double r) {
  const double r2 = r * r;
  double p = 1.0 / 2432902008176640000.0;         // 1/20!
  p = p * r2 - 1.0 / 6402373705728000.0;          // 1/18!
  p = p * r2 + 1.0 / 20922789888000.0;            // 1/16!
  p = p * r2 - 1.0 / 87178291200.0;               // 1/14!
  p = p * r2 + 1.0 / 479001600.0;                 // 1/12!
  p = p * r2 - 1.0 / 3628800.0;                   // 1/10!
  p = p * r2 + 1.0 / 40320.0;                     // 1/8!
  p = p * r2 - 1.0 / 720.0;                       // 1/6!
  p = p * r2 + 1.0 / 24.0;                        // 1/4!
  p = p * r2 - 0.5;                               // 1/2!
  return 1.0 + r2 * p;
}

// sin(x), cos(x) for 0 <= x <= 2*pi (the range of HEALPix longitudes): Cody-Waite style
// reduction by the nearest multiple of pi/2 with a two-part pi/2, then the series above.
HPN_FN void sincos_0_2pi(double x, double* s, double* c) {
  const int k = (int)floor(x * HPN_TWO_OVER_PI + 0.5);
  const double kd = (double)k;
  const double r = (x - kd * HPN_PIO2_HI) - kd * HPN_PIO2_LO;
  const double sr = sin_series(r), cr = cos_series(r);
  switch (k & 3) {
    case 0: *s = sr;  *c = cr;  break;
    case 1: *s = cr;  *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
  }
}

// atan(u) for |u| <= 2 - sqrt(3) (~0.268) from its Maclaurin series through u^33.
HPN_FN double atan_small(double u) {
  const double u2 = u * u;
  double p = -1.0 / 33.0;
  p = p * u2 + 1.0 / 31.0;
  p = p * u2 - 1.0 / 29.0;
  p = p * u2 + 1.0 / 27.0;
  p = p * u2 - 1.0 / 25.0;
  p = p * u2 + 1.0 / 23.0;
  p = p * u2 - 1.0 / 21.0;
  p = p * u2 + 1.0 / 19.0;
  p = p * u2 - 1.0 / 17.0;
  p = p * u2 + 1.0 / 15.0;
  p = p * u2 - 1.0 / 13.0;
  p = p * u2 + 1.0 / 11.0;
  p = p * u2 - 1.0 / 9.0;
  p = p * u2 + 1.0 / 7.0;
  p = p * u2 - 1.0 / 5.0;
  p = p * u2 + 1.0 / 3.0;
  return u - u * (u2 * p);
}

// atan2(y, x) in (-pi, pi]; (0, 0) maps to 0. Octant folding to t = min/max in [0, 1],
// then atan(t) = pi/6 + atan((t*sqrt3 - 1)/(sqrt3 + t)) when t > 2 - sqrt3.
HPN_FN double atan2_own(double y, double x) {
  const double ax = fabs(x), ay = fabs(y);
  if (ax == 0.0 && ay == 0.0) return 0.0;
  const bool swap = ay > ax;
  const double t = swap ? ax / ay : ay / ax;
  double a;
  if (t > 0.2679491924311227) {
    a = HPN_PI_6 + atan_small((t * HPN_SQRT3 - 1.0) / (HPN_SQRT3 + t));
  } else {
    a = atan_small(t);
  }
  if (swap) a = (HPN_PIO2_HI - a) + HPN_PIO2_LO;
  if (x < 0.0) a = (HPN_PI - a);
  if (y < 0.0) a = -a;
  return a;
}

// Base-face tables: ring of the face's southernmost corner in units of nside (j_rll) and the
// longitude index of the face centre in units of pi/4 (j_pll) -- Gorski et al. 2005, Fig. 4.
HPN_FN int face_jrll(int f) { return (f < 4) ? 2 : ((f < 8) ? 3 : 4); }
HPN_FN int face_jpll(int f) {
  const int t[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};
  return t[f];
}

// Gather the even bits (x) of a NEST in-face index into a contiguous integer.
HPN_FN uint32_t compress_even_bits(uint32_t v) {
  v &= 0x55555555u;
  v = (v | (v >> 1)) & 0x33333333u;
  v = (v | (v >> 2)) & 0x0f0f0f0fu;
  v = (v | (v >> 4)) & 0x00ff00ffu;
  v = (v | (v >> 8)) & 0x0000ffffu;
  return v;
}
HPN_FN uint32_t spread_bits(uint32_t v) {
  v &= 0x0000ffffu;
  v = (v | (v << 8)) & 0x00ff00ffu;
  v = (v | (v << 4)) & 0x0f0f0f0fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}

// NEST pixel -> unit vector at HEALPix order `order` (nside = 2^order, order <= 13).
HPN_FN void pix2vec(int order, int pix, double* vx, double* vy, double* vz) {
  const int nside = 1 << order;
  const int npface = nside << order;
  const int face = pix >> (2 * order);
  const uint32_t ipf = (uint32_t)(pix & (npface - 1));
  const int ix = (int)compress_even_bits(ipf);
  const int iy = (int)compress_even_bits(ipf >> 1);
  const int jr = face_jrll(face) * nside - ix - iy - 1;  // ring index, 1 .. 4 nside - 1
  const double fact2 = 4.0 / (12.0 * (double)nside * (double)nside);
  int nr, kshift;
  double z, sth;
  if (jr < nside) {                      // north polar cap
    nr = jr;
    const double tmp = (double)(nr * nr) * fact2;
    z = 1.0 - tmp;
    sth = sqrt(tmp * (2.0 - tmp));
    kshift = 0;
  } else if (jr > 3 * nside) {           // south polar cap
    nr = 4 * nside - jr;
    const double tmp = (double)(nr * nr) * fact2;
    z = tmp - 1.0;
    sth = sqrt(tmp * (2.0 - tmp));
    kshift = 0;
  } else {                               // equatorial belt
    nr = nside;
    const double fact1 = (double)(2 * nside) * fact2;
    z = (double)(2 * nside - jr) * fact1;
    sth = sqrt((1.0 - z) * (1.0 + z));
    kshift = (jr - nside) & 1;
  }
  int jp = (face_jpll(face) * nr + ix - iy + 1 + kshift) / 2;
  if (jp > 4 * nside) jp -= 4 * nside;
  if (jp < 1) jp += 4 * nside;
  const double phi = ((double)jp - (double)(kshift + 1) * 0.5) * (HPN_PIO2_HI / (double)nr);
  double s, c;
  sincos_0_2pi(phi, &s, &c);
  *vx = sth * c;
  *vy = sth * s;
  *vz = z;
}

// Unit (or any non-zero) vector -> NEST pixel at order `order`.
HPN_FN int vec2pix(int order, double vx, double vy, double vz) {
  const int nside = 1 << order;
  const double len = sqrt(vx * vx + vy * vy + vz * vz);
  const double z = vz / len;
  const double za = fabs(z);
  double tt = atan2_own(vy, vx) * HPN_TWO_OVER_PI;   // longitude in units of pi/2
  if (tt < 0.0) tt += 4.0;
  if (tt >= 4.0) tt -= 4.0;
  int face, ix, iy;
  if (za <= 2.0 / 3.0) {                  // equatorial belt
    const double t1 = (double)nside * (0.5 + tt);
    const double t2 = (double)nside * (z * 0.75);
    const int jp = (int)(t1 - t2);        // ascending edge line
    const int jm = (int)(t1 + t2);        // descending edge line
    const int ifp = jp >> order;
    const int ifm = jm >> order;
    face = (ifp == ifm) ? (ifp | 4) : ((ifp < ifm) ? ifp : (ifm + 8));
    ix = jm & (nside - 1);
    iy = nside - (jp & (nside - 1)) - 1;
  } else {                                // polar caps
    int ntt = (int)tt;
    if (ntt > 3) ntt = 3;
    const double tp = tt - (double)ntt;
    double tmp;
    if (za > 0.99) {
      const double sth = sqrt(vx * vx + vy * vy) / len;
      tmp = (double)nside * sth / sqrt((1.0 + za) / 3.0);
    } else {
      tmp = (double)nside * sqrt(3.0 * (1.0 - za));
    }
    int jp = (int)(tp * tmp);
    int jm = (int)((1.0 - tp) * tmp);
    if (jp > nside - 1) jp = nside - 1;
    if (jm > nside - 1) jm = nside - 1;
    if (z >= 0.0) {
      face = ntt;
      ix = nside - jm - 1;
      iy = nside - jp - 1;
    } else {
      face = ntt + 8;
      ix = jp;
      iy = jm;
    }
  }
  return (face << (2 * order)) + (int)(spread_bits((uint32_t)ix) | (spread_bits((uint32_t)iy) << 1));
}

}  // namespace hpn
