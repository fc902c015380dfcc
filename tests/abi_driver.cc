// A compiled C++ caller of the C ABI (include/flexrt.h), written the way the reference's own driver
// (main.cc) would call the library once its step functions are replaced: the set-up of
// main.cc:10-106 (init, update_dt, init_rt, the set-up cast, get_nphot_min_max), then per step the
// calls of main.cc:108-264 in their order (set_clump, set_clight, update_rays, find_avg_unu, the
// merge block, split_rays, update_thermal, new_rays, update_dt). Built by tests/test_abi_driver.py
// with g++ against the header and linked to libflexrt_b200.so, so a change of a declaration, an
// argument list or a struct layout in the header breaks this build or its run.
//
//   abi_driver layout
//       prints the size and field offsets of the ABI structs (no GPU needed)
//   abi_driver run <dir> <steps> <fused>
//       reads one box from <dir> (box.txt: n box_hmpc z cl_factor rkill_cm seed nsrc;
//       spectrum.txt: nfreq, then per bin nu_Hz fraction; density.bin: float32 N^3 1+delta;
//       src_ijk.bin: int32 [nsrc][3]; src_lum.bin: float64 [nsrc]) and runs <steps> steps,
//       through the individual step functions (fused = 0) or frt_step (fused = 1); prints one
//       line per step: STEP s status crossings rays_alive rays_cast photons_in_flight
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "flexrt.h"

namespace {

template <typename T>
bool read_all(const std::string& path, std::vector<T>* out, size_t n) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  out->resize(n);
  const size_t got = fread(out->data(), sizeof(T), n, f);
  fclose(f);
  return got == n;
}

int fail(frt_ctx* ctx, const char* what, frt_status st) {
  printf("FAIL %s status %d: %s\n", what, st, ctx ? frt_last_error(ctx) : "");
  return 1;
}

#define CALL(x)                                  \
  do {                                           \
    const frt_status st_ = (x);                  \
    if (st_ != FRT_OK) return fail(ctx, #x, st_); \
  } while (0)

int layout() {
  printf("frt_box_desc %zu n %zu box_hmpc %zu zz %zu cl_factor %zu ray_per_cell_max %zu rkill_cm %zu\n",
         sizeof(frt_box_desc), offsetof(frt_box_desc, n), offsetof(frt_box_desc, box_hmpc),
         offsetof(frt_box_desc, zz), offsetof(frt_box_desc, cl_factor), offsetof(frt_box_desc, ray_per_cell_max),
         offsetof(frt_box_desc, rkill_cm));
  printf("frt_config %zu nfreq %zu nu_phot %zu spectrum %zu itercount %zu path_length %zu hpx_lvl %zu "
         "safety_factor %zu tstep_factor %zu nl_const %zu const_clump %zu fH1_0 %zu fHe1_0 %zu fHe2_0 %zu "
         "temp_0 %zu nbox %zu boxes %zu ray_capacity %zu lit_capacity %zu src_capacity %zu precision %zu "
         "outputs %zu device %zu\n",
         sizeof(frt_config), offsetof(frt_config, nfreq), offsetof(frt_config, nu_phot),
         offsetof(frt_config, spectrum), offsetof(frt_config, itercount), offsetof(frt_config, path_length),
         offsetof(frt_config, hpx_lvl), offsetof(frt_config, safety_factor), offsetof(frt_config, tstep_factor),
         offsetof(frt_config, nl_const), offsetof(frt_config, const_clump), offsetof(frt_config, fH1_0),
         offsetof(frt_config, fHe1_0), offsetof(frt_config, fHe2_0), offsetof(frt_config, temp_0),
         offsetof(frt_config, nbox), offsetof(frt_config, boxes), offsetof(frt_config, ray_capacity),
         offsetof(frt_config, lit_capacity), offsetof(frt_config, src_capacity), offsetof(frt_config, precision),
         offsetof(frt_config, outputs), offsetof(frt_config, device));
  printf("frt_step_stats %zu rays_alive %zu rays_moved %zu crossings %zu lit_cells %zu rays_split %zu "
         "rays_merged %zu rays_killed %zu rays_cast %zu photons_emitted %zu photons_deposited %zu "
         "photons_killed %zu photons_overlap %zu photons_in_flight %zu t %zu dt %zu error_flags %zu pad %zu\n",
         sizeof(frt_step_stats), offsetof(frt_step_stats, rays_alive), offsetof(frt_step_stats, rays_moved),
         offsetof(frt_step_stats, crossings), offsetof(frt_step_stats, lit_cells),
         offsetof(frt_step_stats, rays_split), offsetof(frt_step_stats, rays_merged),
         offsetof(frt_step_stats, rays_killed), offsetof(frt_step_stats, rays_cast),
         offsetof(frt_step_stats, photons_emitted), offsetof(frt_step_stats, photons_deposited),
         offsetof(frt_step_stats, photons_killed), offsetof(frt_step_stats, photons_overlap),
         offsetof(frt_step_stats, photons_in_flight), offsetof(frt_step_stats, t), offsetof(frt_step_stats, dt),
         offsetof(frt_step_stats, error_flags), offsetof(frt_step_stats, pad));
  printf("frt_adj_objective %zu box %zu lo %zu hi %zu\n", sizeof(frt_adj_objective),
         offsetof(frt_adj_objective, box), offsetof(frt_adj_objective, lo), offsetof(frt_adj_objective, hi));
  return 0;
}

int run(const std::string& dir, int steps, bool fused) {
  frt_ctx* ctx = nullptr;
  frt_box_desc bd{};
  unsigned seed = 0;
  int nsrc = 0;
  {
    FILE* f = fopen((dir + "/box.txt").c_str(), "r");
    if (!f) return fail(ctx, "open box.txt", -1);
    const int got = fscanf(f, "%d %lf %f %f %lf %u %d", &bd.n, &bd.box_hmpc, &bd.zz, &bd.cl_factor, &bd.rkill_cm,
                           &seed, &nsrc);
    fclose(f);
    if (got != 7) return fail(ctx, "parse box.txt", -1);
  }
  bd.ray_per_cell_max = 22;   // global_variables.cc:40
  frt_config cfg{};
  {
    FILE* f = fopen((dir + "/spectrum.txt").c_str(), "r");
    if (!f || fscanf(f, "%d", &cfg.nfreq) != 1 || cfg.nfreq < 1 || cfg.nfreq > FRT_MAX_FREQ)
      return fail(ctx, "parse spectrum.txt", -1);
    for (int nu = 0; nu < cfg.nfreq; nu++)
      if (fscanf(f, "%lf %f", &cfg.nu_phot[nu], &cfg.spectrum[nu]) != 2) return fail(ctx, "parse spectrum.txt", -1);
    fclose(f);
  }
  // the reference's plain-mode constants (user_inputs.h:81-100)
  cfg.itercount = 5;
  cfg.path_length = 8;
  cfg.hpx_lvl = 0;
  cfg.safety_factor = 3.f;
  cfg.tstep_factor = 1.f;
  cfg.nl_const = 0.5f;
  cfg.const_clump = 1.f;
  cfg.fH1_0 = 1.f - 1.2e-3f;
  cfg.fHe1_0 = 1.f - 1.2e-3f;
  cfg.fHe2_0 = 1.2e-3f;
  cfg.temp_0 = 1e4f;
  cfg.nbox = 1;
  cfg.boxes = &bd;
  cfg.ray_capacity = 1 << 20;
  cfg.lit_capacity = 0;
  cfg.src_capacity = nsrc > 0 ? nsrc : 1;
  cfg.precision = FRT_PREC_MIXED;
  cfg.outputs = FRT_OUT_CORE;
  cfg.device = 0;
  const size_t ncell = (size_t)bd.n * bd.n * bd.n;
  std::vector<float> delta1;
  std::vector<int32_t> ijk;
  std::vector<double> lum;
  if (!read_all(dir + "/density.bin", &delta1, ncell) || !read_all(dir + "/src_ijk.bin", &ijk, 3 * (size_t)nsrc) ||
      !read_all(dir + "/src_lum.bin", &lum, (size_t)nsrc))
    return fail(ctx, "read inputs", -1);

  // ---- set-up, main.cc:10-106 ----
  CALL(frt_create(&cfg, &ctx));
  CALL(frt_seed_boxes(ctx, &seed));   // srand(seed) of the reference (general_funcs.cc:163-167)
  CALL(frt_init_gas(ctx, 0, delta1.data()));
  CALL(frt_set_sources(ctx, 0, nsrc, ijk.data(), lum.data()));
  float dt = 0.f;
  CALL(frt_update_dt(ctx, &dt));
  CALL(frt_init_rt(ctx));
  std::vector<uint16_t> ith_src(nsrc > 0 ? nsrc : 1);
  uint16_t ith_box = 0;
  CALL(frt_draw_cast(ctx, ith_src.data()));
  CALL(frt_new_rays(ctx, ith_src.data()));
  double nmin = 0., nmax = 0.;
  CALL(frt_get_nphot_min_max(ctx, &nmin, &nmax));
  printf("SETUP dt %.9e nphot_min %.9e nphot_max %.9e\n", (double)dt, nmin, nmax);

  // ---- the step loop, main.cc:108-264 ----
  frt_step_stats st{};
  for (int s = 1; s <= steps; s++) {
    frt_status status = FRT_OK;
    if (fused) {
      status = frt_step(ctx, nullptr, nullptr, &st);
    } else {
      CALL(frt_set_clump(ctx));
      CALL(frt_set_clight(ctx));
      CALL(frt_update_rays(ctx));
      CALL(frt_find_avg_unu(ctx));
      CALL(frt_draw_step(ctx, &ith_box, ith_src.data()));   // merge's draw, then one per source
      CALL(frt_merge(ctx, &ith_box));
      CALL(frt_split_rays(ctx));
      CALL(frt_update_thermal(ctx));
      CALL(frt_new_rays(ctx, ith_src.data()));
      CALL(frt_update_dt(ctx, &dt));
      status = frt_last_stats(ctx, &st);
    }
    printf("STEP %d %d %lld %lld %lld %.9e\n", s, status, st.crossings, st.rays_alive, st.rays_cast,
           st.photons_in_flight);
    if (status != FRT_OK) return fail(ctx, "step", status);
  }
  long long nr = 0;
  CALL(frt_num_rays(ctx, 0, &nr));
  printf("RAYS %lld\n", nr);
  CALL(frt_destroy(ctx));
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc >= 2 && !strcmp(argv[1], "layout")) return layout();
  if (argc >= 5 && !strcmp(argv[1], "run")) return run(argv[2], atoi(argv[3]), atoi(argv[4]) != 0);
  fprintf(stderr, "usage: abi_driver layout | run <dir> <steps> <fused>\n");
  return 2;
}
