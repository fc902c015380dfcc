// CPU check of the cell walk's face-time ranking (flexrt_imaging_reion_b200/csrc/frt_dda.cuh).
//
// The walk ranks the three axes by approximate face times and evaluates the reference's exact
// quotients only for the axes that can be the smallest. This program compiles that walk for the
// host and compares it, ray by ray, with a walk that evaluates all three exact quotients at every
// face (the expression structure of advance_ray, ray_tracing.cc:1254-1400): the number of
// segments, every segment's cell and distance, and the end position and cell must agree to the
// last bit. Rays: random directions and positions in boxes of the S, M and L sizes, and edge
// cases (positions on the cell faces and at the nudged edges, axis-aligned and diagonal
// directions whose face times tie exactly, components down to the subnormal range, signed zeros,
// walks of zero length and of many cells). It also checks the walk's (i, j, k) of a cell index
// (cell_ijk, double-precision reciprocals) against integer division. Built by nvcc as host code;
// no GPU is used.
//
//   dda_rank_test [rays per box]   prints "ok <rays> <segments> <ties>" or the first mismatch
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "../flexrt_imaging_reion_b200/csrc/frt_dda.cuh"

using frt::BoxP;

namespace {

constexpr int kPL = 16;

struct Walk {
  int ns;
  int cell[kPL];
  uint32_t dist[kPL];
  uint32_t x, y, z;
  int in, jn, kn;
};

long long g_rays = 0, g_segs = 0, g_ties = 0;

uint32_t bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

// All three exact face times at every face and the tie rule of advance_ray.
int walk_three(const BoxP& B, int PL, float xhat, float yhat, float zhat, float deltat, float& x0, float& y0,
               float& z0, int& in, int& jn, int& kn, Walk& w) {
  const int N = B.n;
  const float clgt = B.clight, dxc = B.dx;
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
    {   // faces where a second axis comes within 2^-17 of the smallest time (or ties with it)
      const float o1 = (tag == 0) ? ty : tx, o2 = (tag == 2) ? ty : tz;
      const float second = o1 < o2 ? o1 : o2;
      if (second <= tmin * (1.0f + 1.0f / 131072.0f)) g_ties++;
    }
    if ((tlast + tmin) < deltat) {
      dist = tmin * clgt;
      if (p >= PL - 1) return -1;
      w.cell[p] = (int)(B.cell0 + (long long)in * B.nn + jn * N + kn);
      w.dist[p] = bits(dist);
      p += 1;
      x0 += dist * xhat;
      y0 += dist * yhat;
      z0 += dist * zhat;
      if (tag == 0) {
        if (xhat > 0.f) { in = frt::dda_up(in, N); x0 = B.lo_edge; }
        else { in = frt::dda_down(in, N); x0 = B.hi_edge; }
      } else if (tag == 1) {
        if (yhat > 0.f) { jn = frt::dda_up(jn, N); y0 = B.lo_edge; }
        else { jn = frt::dda_down(jn, N); y0 = B.hi_edge; }
      } else {
        if (zhat > 0.f) { kn = frt::dda_up(kn, N); z0 = B.lo_edge; }
        else { kn = frt::dda_down(kn, N); z0 = B.hi_edge; }
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
  dist = (deltat - tlast + tmin) * clgt;
  dist = (B.lo_edge >= dist) ? B.lo_edge : dist;
  w.cell[p] = (int)(B.cell0 + (long long)in * B.nn + jn * N + kn);
  w.dist[p] = bits(dist);
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

float float_at_or_above(double v) {
  float f = (float)v;
  if ((double)f < v) f = std::nextafter(f, INFINITY);
  return f;
}

// The walk's box constants as the host set-up derives them (box_params, set_cell_size).
BoxP make_box(int n, double box_hmpc, double zz) {
  BoxP B;
  std::memset(&B, 0, sizeof(B));
  B.n = n;
  B.nn = n * n;
  B.cell0 = 0;
  const float Lx0 = box_hmpc * 1e3 / 0.68;
  const float a_snap = (float)(1. / (1. + zz));
  const float Lx = Lx0 * a_snap;
  const float dx = Lx / n * 3.086e21;
  B.dx = dx;
  B.lo_edge = 1e-4f * dx;
  B.hi_edge = dx * (1. - 1e-4f);
  B.hi_thr = dx * (1. - 1e-4f / 2.);
  B.hi_thr_f = float_at_or_above(B.hi_thr);
  B.clight = 2.998e10;
  B.dt = 1.0f * dx / 1.0f / 2.998e10;
  return B;
}

bool same(const Walk& a, const Walk& b) {
  if (a.ns != b.ns) return false;
  if (a.ns < 0) return true;
  for (int p = 0; p < a.ns; p++)
    if (a.cell[p] != b.cell[p] || a.dist[p] != b.dist[p]) return false;
  return a.x == b.x && a.y == b.y && a.z == b.z && a.in == b.in && a.jn == b.jn && a.kn == b.kn;
}

struct Ray {
  float xh, yh, zh, x, y, z, deltat;
  int i, j, k;
};

bool check(const BoxP& B, const Ray& r) {
  Walk a{}, b{};
  {
    float x = r.x, y = r.y, z = r.z;
    int i = r.i, j = r.j, k = r.k;
    a.ns = walk_three(B, kPL, r.xh, r.yh, r.zh, r.deltat, x, y, z, i, j, k, a);
    a.x = bits(x), a.y = bits(y), a.z = bits(z), a.in = i, a.jn = j, a.kn = k;
  }
  {
    float x = r.x, y = r.y, z = r.z;
    int i = r.i, j = r.j, k = r.k;
    b.ns = frt::dda_walk(B, kPL, r.xh, r.yh, r.zh, r.deltat, x, y, z, i, j, k, [&](int p, long long gc, float ds) {
      b.cell[p] = (int)gc;
      b.dist[p] = bits(ds);
    });
    b.x = bits(x), b.y = bits(y), b.z = bits(z), b.in = i, b.jn = j, b.kn = k;
  }
  g_rays++;
  if (a.ns > 0) g_segs += a.ns;
  if (!same(a, b)) {
    std::printf("MISMATCH n=%d dir=(%a %a %a) pos=(%a %a %a) deltat=%a cell=(%d %d %d): ns %d vs %d\n", B.n, r.xh,
                r.yh, r.zh, r.x, r.y, r.z, r.deltat, r.i, r.j, r.k, a.ns, b.ns);
    for (int p = 0; p < (a.ns > b.ns ? a.ns : b.ns) && p < kPL; p++)
      std::printf("  seg %d: %d %08x | %d %08x\n", p, a.cell[p], a.dist[p], b.cell[p], b.dist[p]);
    return false;
  }
  return true;
}

}  // namespace

// cell_ijk against integer division: every index of boxes up to 256^3 (and 96^3), random
// indices of larger boxes up to 2^31 cells
bool check_cell_ijk(std::mt19937_64& rng) {
  const int sizes[] = {32, 64, 96, 128, 256, 300, 512, 1024, 1290};
  for (int N : sizes) {
    const int NN = N * N;
    const long long ncell = (long long)N * NN;
    const double inv_n = 1.0 / N, inv_nn = 1.0 / ((double)N * N);
    const long long count = ncell <= (1ll << 24) ? ncell : 20000000ll;
    for (long long q = 0; q < count; q++) {
      const int ind = (int)(ncell <= (1ll << 24) ? q : (long long)(rng() % (unsigned long long)ncell));
      int i, j, k;
      frt::cell_ijk(ind, N, NN, inv_n, inv_nn, &i, &j, &k);
      if (i != ind / NN || j != (ind % NN) / N || k != ind % N) {
        std::printf("MISMATCH cell_ijk N=%d ind=%d: %d %d %d\n", N, ind, i, j, k);
        return false;
      }
    }
  }
  return true;
}

int main(int argc, char** argv) {
  const long long per_box = argc > 1 ? std::atoll(argv[1]) : 1000000;
  std::mt19937_64 rng(20261204);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  if (!check_cell_ijk(rng)) return 1;
  const BoxP boxes[3] = {make_box(64, 25.0, 8.0), make_box(128, 50.0, 7.0), make_box(256, 100.0, 6.5)};
  for (const BoxP& B : boxes) {
    const float dx = B.dx;
    const float special_pos[] = {B.lo_edge, B.hi_edge, 0.5f * dx, dx, 0.0f, std::nextafter(B.hi_edge, 0.f),
                                 std::nextafter(B.lo_edge, INFINITY), 0.25f * dx};
    const float s3 = (float)(1.0 / std::sqrt(3.0)), s2 = (float)(1.0 / std::sqrt(2.0));
    const float tiny[] = {1e-7f, 1e-20f, 1e-30f, 1e-38f, 1e-44f, 0.0f, -0.0f};
    for (long long q = 0; q < per_box; q++) {
      Ray r;
      // a random direction (float-rounded unit vector)
      const double u = 2 * U(rng) - 1, ph = 2 * M_PI * U(rng), sn = std::sqrt(1 - u * u);
      r.xh = (float)(sn * std::cos(ph));
      r.yh = (float)(sn * std::sin(ph));
      r.zh = (float)u;
      r.x = (float)(B.lo_edge + (B.hi_edge - B.lo_edge) * U(rng));
      r.y = (float)(B.lo_edge + (B.hi_edge - B.lo_edge) * U(rng));
      r.z = (float)(B.lo_edge + (B.hi_edge - B.lo_edge) * U(rng));
      r.deltat = (float)(B.dt * 4.0 * U(rng));
      r.i = (int)(U(rng) * B.n), r.j = (int)(U(rng) * B.n), r.k = (int)(U(rng) * B.n);
      const int mode = (int)(U(rng) * 16);
      if (mode == 1) {   // positions on faces and edges
        r.x = special_pos[(int)(U(rng) * 8)];
        r.y = special_pos[(int)(U(rng) * 8)];
        r.z = special_pos[(int)(U(rng) * 8)];
      } else if (mode == 2) {   // diagonal and axis directions: exact ties between face times
        const float sx = U(rng) < 0.5 ? -1.f : 1.f, sy = U(rng) < 0.5 ? -1.f : 1.f, sz = U(rng) < 0.5 ? -1.f : 1.f;
        const int c = (int)(U(rng) * 4);
        if (c == 0) { r.xh = sx * s3; r.yh = sy * s3; r.zh = sz * s3; }
        else if (c == 1) { r.xh = sx * s2; r.yh = sy * s2; r.zh = 0.f; }
        else if (c == 2) { r.xh = sx; r.yh = 0.f; r.zh = 0.f; }
        else { r.xh = 0.f; r.yh = sy * s2; r.zh = sz * s2; }
        if (U(rng) < 0.5) { r.x = r.y = r.z = special_pos[(int)(U(rng) * 8)]; }
        if (U(rng) < 0.5) { r.y = (r.xh * r.yh > 0.f) ? r.x : dx - r.x; }
      } else if (mode == 3) {   // tiny, zero and subnormal components
        const float t1 = tiny[(int)(U(rng) * 7)];
        const int ax = (int)(U(rng) * 3);
        if (ax == 0) r.xh = (U(rng) < 0.5 ? -1 : 1) * t1;
        else if (ax == 1) r.yh = (U(rng) < 0.5 ? -1 : 1) * t1;
        else r.zh = (U(rng) < 0.5 ? -1 : 1) * t1;
      } else if (mode == 4) {   // walks of zero length and of up to 12 cells
        r.deltat = (U(rng) < 0.5) ? 0.0f : (float)(B.dt * 12.0 * U(rng));
      } else if (mode == 5) {   // positions one ulp either side of the faces the walk aims at
        r.x = U(rng) < 0.5 ? std::nextafter(dx, 0.f) : std::nextafter(0.f, 1.f) * 1e30f;
        r.y = U(rng) < 0.5 ? B.hi_edge : B.lo_edge;
      }
      if (!check(B, r)) return 1;
    }
  }
  std::printf("ok %lld %lld %lld\n", g_rays, g_segs, g_ties);
  return 0;
}
