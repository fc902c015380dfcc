// ORACLE TEST INFRASTRUCTURE -- not part of the product.
//
// Driver for the reference's own C++/OpenMP RT code, compiled from a staged copy of the
// reference sources (see oracle/build_ref.py). It replaces main.cc and replays the reference
// loop main.cc:108-264 in the order main.cc gives, with these hooks:
//   * srand(seed) instead of the time-based init_rand (general_funcs.cc:163-167);
//   * the snapshot scale factor is a = 1/(1+zinit) instead of the cosmic-time-table round trip
//     in update_hydro_step (gas_funcs.cc:563), and the first-snapshot set-up of
//     update_hydro_step (gas_funcs.cc:595-613) is done here directly from the input files;
//   * optional per-cell clumping field written over clump[] after set_clump() each step;
//   * optional removal of rays with comoving r > rkill after update_rays;
//   * update_cosmo_expansion / update_hydro_step / write_otf are not called (fixed redshift);
//   * state dumps (FRTD files) and per-step timings;
//   * with FRT_RESTART_OUT=<dir> in the environment, the reference's own restart writers
//     (write_gas_binary, write_rays_binary, write_treion) run after the last step;
//   * with FRT_COSMO in the environment, update_cosmo_expansion (gas_funcs.cc:460-548) runs after
//     new_rays as in main.cc:219-220, and the two scale factors it uses are logged (hex floats);
//   * with FRT_HYDRO=<k1>[,<k2>] and FRT_HYDRO_Z=<z1>,<z2>,<z3> in the environment, the
//     reference's own update_hydro_step (gas_funcs.cc:554-752) and get_nphot_min_max run after
//     steps k1 (and k2), after new_rays and the optional expansion (main.cc:219-224): the
//     snapshot list is {zinit, z1, z2, z3}, the n-th switch reads hydro/density.01<n>.<N>,
//     hydro/ndot_catalog_01<n> and hydro/numhalos.01<n> under the stage directory (snapinit =
//     10) and writes its outputs under hydro_out/; the scale factor, the snapshot interval and the
//     redshift it uses are logged as 'HYDRO step a_rt dt_snap zz' (hex floats);
//   * in a stage built with subgrid = TRUE the set-up imports the sub-grid tables after the cast
//     (main.cc:86-90) and every step updates the non-linear overdensity domain after t += dt
//     (main.cc:126-128); the cosmic times the model uses are logged once as 'SUBGRID tinit t12 t8
//     tcap tre0 tre1 tre2' (hex floats);
//   * in a stage built with input_grid = TRUE the set-up is the reference's restart path: the
//     grid is sized as init() would (init_funcs.cc:22-30), the catalogue is read, init() reads the
//     gas and treion restart files, init_rt() reads the ray file, and no rays are cast.
// Usage: ref_driver <input_dir> <nsteps> <seed> <dump_every> <rkill_cm> [clump.bin]
//   input_dir holds density.bin (float32 N^3, 1+delta), catalog.bin (5 doubles per source),
//   numhalos.bin (int64) and receives dump_XXXX.frtd files. cwd must contain input_files/.
#include "rt_funcs.cc"
#include "frtd.h"
#include <string>

static void drv_dump_state(const std::string& path, long step_no, long crossings, long moved) {
  struct frtd_writer w;
  if (frtd_open(&w, path.c_str()) != 0) {
    printf("cannot write %s\n", path.c_str());
    return;
  }
  const int64_t n3 = (int64_t)Nx * Ny * Nz;
  const int64_t nf[2] = {n3, Nfreq};
#define DF(name) frtd_add1(&w, #name, FRTD_F32, n3, &name[0][0][0])
#define DFN(name) frtd_add(&w, #name, FRTD_F32, 2, nf, &name[0][0][0][0])
  DF(rho); DF(nH); DF(nHe); DF(nH1); DF(nHe1); DF(nH2); DF(nHe2); DF(nHe3); DF(ne); DF(n_tot);
  DF(f_H1); DF(f_He1); DF(f_H2); DF(f_He2); DF(f_He3); DF(temp); DF(clump); DF(avg_nh1); DF(avg_nhe1);
  DF(gamma_H1_tot); DF(gamma_He1_tot); DF(heat_rate); DF(cool_rate); DF(recomb_H2); DF(recomb_He2);
  DF(recomb_He3); DF(recrate_H2); DF(recrate_He2); DF(dne_dt); DF(mfp); DF(mfp_912); DF(treion);
  DF(treion_out); DF(IF_speed); DF(Inc_Flux); DF(avg_gamma); DF(avg_gamma_he1); DF(nH1_prev); DF(fion);
  DFN(gamma_H1_nu); DFN(gamma_He1_nu); DFN(ngam_nu); DFN(u_nu); DFN(avg_gamma_nu); DFN(avg_gamma_nu_he1);
#undef DF
#undef DFN
  {
    std::vector<uint8_t> fl(n3);
    for (int64_t c = 0; c < n3; ++c) fl[c] = (&treion_flag[0][0][0])[c] ? 1 : 0;
    frtd_add1(&w, "treion_flag", FRTD_U8, n3, fl.data());
  }
  if (ifront == TRUE) {
    frtd_add1(&w, "fion_max", FRTD_F32, n3, &fion_max[0][0][0]);
    frtd_add1(&w, "tcross", FRTD_F32, n3, &tcross[0][0][0]);
    frtd_add1(&w, "Delta_fion", FRTD_F32, n3, &Delta_fion[0][0][0]);
    const int64_t nt[2] = {n3, Ntcross};
    frtd_add(&w, "tcross_new", FRTD_F32, 2, nt, &tcross_new[0][0][0][0]);
    std::vector<uint8_t> tf(n3), nf3(n3);
    for (int64_t c = 0; c < n3; ++c) {
      tf[c] = (&tcross_flag[0][0][0])[c] ? 1 : 0;
      nf3[c] = (&neutral_flag[0][0][0])[c] ? 1 : 0;
    }
    frtd_add1(&w, "tcross_flag", FRTD_U8, n3, tf.data());
    frtd_add1(&w, "neutral_flag", FRTD_U8, n3, nf3.data());
  }
  // scalars
  double sc[16] = {(double)t, (double)dt, nphot_min, nphot_max, (double)nphot_merge, (double)num_thresh,
                   (double)total_rays, (double)dx0, (double)dx[0], (double)step_no, (double)crossings,
                   (double)moved, nphot_base_avg, (double)avg_rho, (double)num_src, (double)Ncpu};
  frtd_add1(&w, "scalars", FRTD_F64, 16, sc);
  frtd_add1(&w, "spectrum", FRTD_F32, Nfreq, spectrum);
  // rays in slot order
  std::vector<int64_t> slot;
  for (long x = 0; x < size_buffer; ++x)
    if (ray_tags[x]) slot.push_back(x);
  const int64_t nr = (int64_t)slot.size();
  std::vector<uint8_t> act(nr);
  std::vector<int16_t> ord(nr), rend(nr);
  std::vector<int32_t> pix(nr), cell(nr);
  std::vector<uint16_t> ith(nr);
  std::vector<float> f6(nr * 9), np(nr * Nfreq);
  for (int64_t q = 0; q < nr; ++q) {
    const ray_type& R = ray[slot[q]];
    act[q] = R.active ? 1 : 0;
    ord[q] = R.order;
    pix[q] = R.pixel;
    ith[q] = R.itheta;
    cell[q] = R.path[0].ind;
    rend[q] = ray_end[slot[q]];
    const float v[9] = {R.xhat, R.yhat, R.zhat, R.r, R.dr, R.x, R.y, R.z, R.time};
    for (int k = 0; k < 9; ++k) f6[q * 9 + k] = v[k];
    for (int nu = 0; nu < Nfreq; ++nu) np[q * Nfreq + nu] = R.nphot[nu];
  }
  frtd_add1(&w, "ray_slot", FRTD_I64, nr, slot.data());
  frtd_add1(&w, "ray_active", FRTD_U8, nr, act.data());
  frtd_add1(&w, "ray_order", FRTD_I16, nr, ord.data());
  frtd_add1(&w, "ray_pixel", FRTD_I32, nr, pix.data());
  frtd_add1(&w, "ray_itheta", FRTD_U16, nr, ith.data());
  frtd_add1(&w, "ray_cell", FRTD_I32, nr, cell.data());
  frtd_add1(&w, "ray_end", FRTD_I16, nr, rend.data());
  const int64_t d9[2] = {nr, 9};
  frtd_add(&w, "ray_geom", FRTD_F32, 2, d9, f6.data());
  const int64_t dnf[2] = {nr, Nfreq};
  frtd_add(&w, "ray_nphot", FRTD_F32, 2, dnf, np.data());
  frtd_close(&w);
}

int main(int argc, char** argv) {
  if (argc < 6) {
    printf("usage: %s input_dir nsteps seed dump_every rkill_cm [clump.bin]\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1];
  const int nsteps = atoi(argv[2]);
  const unsigned seed = (unsigned)strtoul(argv[3], 0, 10);
  const int dump_every = atoi(argv[4]);
  const double rkill = atof(argv[5]);
  static float clump_in[Nx][Ny][Nz];
  bool have_clump = false;
  if (argc > 6) {
    FILE* f = fopen(argv[6], "rb");
    if (!f) { printf("cannot open clump file\n"); return 2; }
    have_clump = fread(&clump_in[0][0][0], sizeof(float), (size_t)Nx * Ny * Nz, f) == (size_t)Nx * Ny * Nz;
    fclose(f);
    if (!have_clump) { printf("short clump file\n"); return 2; }
  }

  srand(seed);
  double t_setup0 = omp_get_wtime();
  init_lock();
  import_cosmic_time();
  const bool cosmo = getenv("FRT_COSMO") != nullptr;
  int hydro_at[2] = {-1, -1}, n_hydro = 0;
  float hydro_z[3] = {0.f, 0.f, 0.f};
  if (const char* hy = getenv("FRT_HYDRO")) {
    n_hydro = sscanf(hy, "%d,%d", &hydro_at[0], &hydro_at[1]);
    const char* hz = getenv("FRT_HYDRO_Z");
    if (n_hydro < 1 || !hz || sscanf(hz, "%f,%f,%f", &hydro_z[0], &hydro_z[1], &hydro_z[2]) != 3) {
      printf("FRT_HYDRO needs FRT_HYDRO_Z=z1,z2,z3\n");
      return 2;
    }
  }
  if (cosmo || n_hydro > 0) make_scale_factor_table();

  // first-snapshot set-up (gas_funcs.cc:595-613) at a = 1/(1+zinit)
  zz = zinit;
  const float a_snap = (float)(1. / (1. + zinit));
  Lx = Lx0 * a_snap;
  Ly = Ly0 * a_snap;
  Lz = Lz0 * a_snap;
  if (input_grid == TRUE) {
    for (int i = 0; i < Nx; i++) dx[i] = Lx / Nx * kpc_to_cm;
    for (int j = 0; j < Ny; j++) dy[j] = Ly / Ny * kpc_to_cm;
    for (int k = 0; k < Nz; k++) dz[k] = Lz / Nz * kpc_to_cm;
  } else {
    get_ugas((dir + "/density.bin").c_str());
    for (int i = 0; i < Nx; i++)
      for (int j = 0; j < Ny; j++)
        for (int k = 0; k < Nz; k++) rho[i][j][k] *= pow(a_snap, -3.);
    avg_rho *= pow(a_snap, -3.);
  }
  read_source_catalog((dir + "/catalog.bin").c_str(), (dir + "/numhalos.bin").c_str());
  get_random_angles();
  init();
  update_dt();
  if (multi_freq == TRUE) read_spectrum_table();
  set_spectrum();
  init_rt();
  set_ray_per_cell();
  set_lsource();
  if (input_grid == FALSE) new_rays();
  if (subgrid == TRUE) {
    calc_mfp_boost();
    import_delta_over_sigma_table();
    init_radhydro_data();
    printf("SUBGRID %a %a %a %a %a %a %a\n", tinit, cosmic_time(1. / (1. + 12)), cosmic_time(1. / (1. + 8.)),
           cosmic_time(1. / (1. + 5.5)), tre_dom[0], tre_dom[1], tre_dom[2]);
  }
  if (have_clump) memcpy(&clump[0][0][0], &clump_in[0][0][0], sizeof(clump));
  get_nphot_min_max();
  // FRT_RESTART_BALANCE: after the restart set-up, spread the rays read from the file over the
  // threads' buffer regions with the reference's own balance_cpus (mem_funcs.cc:186-236), which
  // its step loop runs at the end of every step (main.cc:258) but the restart set-up does not:
  // without it the first restarted step runs with every ray in the first threads' regions
  if (input_grid == TRUE && getenv("FRT_RESTART_BALANCE")) balance_cpus();
  const double t_setup = omp_get_wtime() - t_setup0;
  printf("SETUP %.6f s num_src=%d dt=%.9e dx=%.9e nphot_min=%.9e\n", t_setup, num_src, (double)dt, (double)dx[0],
         nphot_min);
  if (dump_every > 0) drv_dump_state(dir + "/dump_0000.frtd", 0, 0, 0);

  double tot = 0.0;
  for (int s = 1; s <= nsteps; ++s) {
    step += 1;
    const double w0 = omp_get_wtime();
    set_clump();
    if (have_clump) memcpy(&clump[0][0][0], &clump_in[0][0][0], sizeof(clump));
    set_clight();
    t += dt;
    if (subgrid == TRUE) delta_dom_to_deltaNL_dom(maxd(cosmic_time(1. / (1. + 12)), t + tinit));
    update_rays();
    long crossings = 0, moved = 0;
#pragma omp parallel for reduction(+ : crossings, moved)
    for (long x = 0; x < size_buffer; ++x)
      if (ray_tags[x] == TRUE && ray[x].active == FALSE) {
        crossings += ray_end[x];
        moved += 1;
      }
    if (rkill > 0.0) {
#pragma omp parallel for
      for (long x = 0; x < size_buffer; ++x)
        if (ray_tags[x] == TRUE && (double)ray[x].r > rkill) remove_ray(x);
    }
    const double w1 = omp_get_wtime();
    find_avg_unu();
    const double w2 = omp_get_wtime();
    set_lmerge();
    set_merge_domain();
    get_num_thresh();
    long count = count_rays();
    if (count > num_thresh) calc_nphot_merge();
    merge();
    const double w3 = omp_get_wtime();
    split_rays();
    set_ray_per_cell();
    set_lsource();
    srcstep = mod(srcstep + num_src / Ncpu, num_src);
    const double w4 = omp_get_wtime();
    update_thermal();
    const double w5 = omp_get_wtime();
    new_rays();
    if (cosmo) {
      // the scale factors update_cosmo_expansion takes (gas_funcs.cc:461-465), for the record
      float cosmic_time_current = t + cosmic_time(1. / (1. + zinit));
      float cosmic_time_previous = t + cosmic_time(1. / (1. + zinit)) - dt;
      float a_current = scale_factor(cosmic_time_current);
      float a_prev = scale_factor(cosmic_time_previous);
      printf("COSMO %d %a %a\n", s, a_current, a_prev);
      update_cosmo_expansion();
    }
    for (int hsw = 0; hsw < n_hydro; hsw++)
      if (s == hydro_at[hsw]) {
        hydro_steps.assign({zinit, hydro_z[0], hydro_z[1], hydro_z[2]});
        num_hydro_steps = 4;
        ihydro = hsw + 1;
        const float a_rt = scale_factor(t + cosmic_time(1. / (1. + zinit)));
        const float aa = 1. / (1. + hydro_steps[ihydro]), aa_next = 1. / (1. + hydro_steps[ihydro + 1]);
        const float dt_snap = cosmic_time(aa_next) - cosmic_time(aa);
        printf("HYDRO %d %a %a %a\n", s, a_rt, dt_snap, hydro_steps[ihydro]);
        update_hydro_step();
        get_nphot_min_max();
      }
    update_dt();
    balance_cpus();
    const double w6 = omp_get_wtime();
    tot += w6 - w0;
    printf("STEP %d rays_before=%ld crossings=%ld moved=%ld wall=%.6f adv=%.6f iter=%.6f merge=%.6f split=%.6f "
           "thermal=%.6f cast=%.6f\n",
           s, count, crossings, moved, w6 - w0, w1 - w0, w2 - w1, w3 - w2, w4 - w3, w5 - w4, w6 - w5);
    fflush(stdout);
    if (dump_every > 0 && (s % dump_every == 0 || s == nsteps)) {
      char nm[64];
      snprintf(nm, sizeof nm, "/dump_%04d.frtd", s);
      drv_dump_state(dir + nm, s, crossings, moved);
    }
  }
  printf("TOTAL %.6f s for %d steps\n", tot, nsteps);
  if (const char* rdir = getenv("FRT_RESTART_OUT")) {
    const std::string r = rdir;
    write_gas_binary((r + "/gas.bin").c_str());
    write_rays_binary((r + "/rays.bin").c_str());
    write_treion((r + "/tre.bin").c_str());
  }
  return 0;
}
