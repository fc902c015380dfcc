// ORACLE TEST INFRASTRUCTURE -- not part of the product.
//
// Stand-in for the HEALPix 3.40 C++ header that the reference #includes by absolute path
// (ray_tracing.cc:11, mem_funcs.cc:12). HEALPix is not vendored with the reference and is not
// installed here, so the staged reference copy is pointed at this file instead. It exposes
// exactly the names the reference uses -- T_Healpix_Base<int>(order, NEST), pix2vec(pix),
// vec2pix(vec3), vec3 with operator- and operator/(double) -- and forwards the arithmetic to
// the project's own NEST implementation (flexrt_imaging_reion_b200/csrc/hp_nest.h, written
// from Gorski et al. 2005). Results are therefore pinned between the oracle and the CUDA
// kernels (same code on both sides), not against the real HEALPix library.
#pragma once
#include "../../flexrt_imaging_reion_b200/csrc/hp_nest.h"

enum Healpix_Ordering_Scheme { RING, NEST };

template <typename T> struct vec3_t {
  T x, y, z;
  vec3_t() : x(0), y(0), z(0) {}
  vec3_t(T x_, T y_, T z_) : x(x_), y(y_), z(z_) {}
  vec3_t operator-(const vec3_t& o) const { return vec3_t(x - o.x, y - o.y, z - o.z); }
  vec3_t operator+(const vec3_t& o) const { return vec3_t(x + o.x, y + o.y, z + o.z); }
  vec3_t operator/(double f) const { return vec3_t(x / f, y / f, z / f); }
  vec3_t operator*(double f) const { return vec3_t(x * f, y * f, z * f); }
};
typedef vec3_t<double> vec3;

template <typename I> class T_Healpix_Base {
 public:
  T_Healpix_Base(int order, Healpix_Ordering_Scheme /*scheme: NEST only*/) : order_(order) {}
  vec3 pix2vec(I pix) const {
    vec3 v;
    hpn::pix2vec(order_, (int)pix, &v.x, &v.y, &v.z);
    return v;
  }
  I vec2pix(const vec3& v) const { return (I)hpn::vec2pix(order_, v.x, v.y, v.z); }

 private:
  int order_;
};
