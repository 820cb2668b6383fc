/* d3q19_main.c -- the simulation program: the reference's sim_main.c flow
 * (sim_main.c:1-527) on the B200 library.  Reads input_file.txt (or argv[1])
 * from the working directory, writes xyz_ovito_output.txt,
 * velocity_profile_z.txt, velocity_field_final.txt and
 * matlab_postproc/velocity_field_centerline.txt in the reference's formats.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "d3q19_host.h"

#define CHECK(call)                                                                      \
  do {                                                                                   \
    int rc_ = (call);                                                                    \
    if (rc_ != 0) {                                                                      \
      fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, d3q19_last_error(ctx));      \
      return 1;                                                                          \
    }                                                                                    \
  } while (0)

int main(int argc, char** argv) {
  const char* input = argc > 1 ? argv[1] : "input_file.txt";
  d3q19_ctx* ctx = NULL;
  d3q19h_config cfg;
  printf("Int struct size: %lu\n", (unsigned long)sizeof(int_param_struct));
  printf("Flp struct size: %lu\n", (unsigned long)sizeof(flp_param_struct));

  d3q19_device_info di;
  CHECK(d3q19_get_device_info(0, &di));
  printf("Device %s, %d SMs, %.1f GB\n", di.name, di.sm_count, di.global_mem_bytes / 1e9);

  if (d3q19h_parse_file(input, &cfg) != 0) {
    fprintf(stderr, "cannot read %s\n", input);
    return 1;
  }
  printf("%s %d \n", "ViscosityModel = ", cfg.ip.ViscosityModel);
  if (d3q19h_check(&cfg)) return 1;

  float* spherePoints = NULL;
  if (d3q19h_sphere_discretization(&cfg, ".", &spherePoints) != 0) {
    fprintf(stderr, "Error: malformed coordinates read in sphere discretization\n");
    return 1;
  }
  printf("Number of surface points per particle = %d.\n", cfg.ip.PointsPerParticle);
  d3q19h_work_groups(&cfg, di.kernel_work_group_size);

  const long NC = (long)cfg.ip.LatticeSize[0] * cfg.ip.LatticeSize[1] * cfg.ip.LatticeSize[2];
  const int np = cfg.ip.NumParticles;
  const int nfa = cfg.ip.WorkGroupsPerParticle > 0 ? cfg.ip.WorkGroupsPerParticle : 1;
  float* f = (float*)malloc(sizeof(float) * 19 * NC);
  float* u = (float*)malloc(sizeof(float) * 3 * NC);
  float* tau = (float*)malloc(sizeof(float) * NC);
  if (d3q19h_init_lattice(&cfg, f, u, tau) != 0) return 1;
  float* parKin = (float*)calloc(16 * (size_t)(np > 1 ? np : 2), sizeof(float));
  float* parForce = (float*)calloc(8 * (size_t)(np > 0 ? np : 1), sizeof(float));
  float* parFluidForce = (float*)calloc(8 * (size_t)(np > 0 ? np : 1) * nfa, sizeof(float));
  if (d3q19h_init_particles(&cfg, parKin, parForce, parFluidForce) != 0) {
    fprintf(stderr, "Error: initial particle placement failed\n");
    return 1;
  }
  d3q19h_zone_grid(&cfg);
  const int Z = d3q19h_zone_count(&cfg);
  const int nth = cfg.hp.DomainDecomp[0] * cfg.hp.DomainDecomp[1] * cfg.hp.DomainDecomp[2];
  int* parsZone = (int*)calloc(np > 0 ? np : 1, sizeof(int));
  int* zoneMembers = (int*)calloc((size_t)Z * (np > 0 ? np : 1), sizeof(int));
  int* numParInZone = (int*)calloc(Z, sizeof(int));
  int* threadMembers = (int*)calloc((size_t)(nth > 0 ? nth : 1) * (np > 0 ? np : 1), sizeof(int));
  int* numParInThread = (int*)calloc(nth > 0 ? nth : 1, sizeof(int));
  int* znd = (int*)calloc(28 * (size_t)Z, sizeof(int));
  if (np > 0 && d3q19h_init_zones(&cfg, parKin, parsZone, zoneMembers, numParInZone, threadMembers, numParInThread,
                                  znd) != 0) {
    fprintf(stderr, "Error: Particle out of bounds at zone initialization\n");
    return 1;
  }
  const int nper = d3q19_periodic_map(&cfg.ip, NULL, 0);
  int* strMap = (int*)malloc(sizeof(int) * 2 * (nper > 0 ? nper : 1));
  d3q19_periodic_map(&cfg.ip, strMap, 2 * nper);
  printf("Periodic boundary nodes %d\n", nper);

  d3q19_options opt;
  d3q19h_options(&cfg, &opt);
  CHECK(d3q19_create(&cfg.ip, &cfg.fp, &opt, &ctx));
  CHECK(d3q19_write_lattice(ctx, f, u, tau));
  CHECK(d3q19_write_periodic_map(ctx, strMap, nper));
  if (np > 0) {
    CHECK(d3q19_write_particles(ctx, parKin, parForce, parFluidForce, spherePoints));
    CHECK(d3q19_write_zones(ctx, znd, parsZone, zoneMembers, numParInZone, threadMembers, numParInThread));
  }

  FILE* vid = fopen("xyz_ovito_output.txt", "w");
  d3q19h_output_state out = {0, 0.0f, 0.0f};
  const int T = cfg.ip.MaxIterations;
  printf("%s %d\n", "Starting iteration 1, maximum iterations", T);
  int t = 1;
  while (t <= T) {
    /* Advance to the next step that prints or writes output. */
    int stop = t;
    while (stop < T) {
      if (stop % cfg.hp.ConsolePrintFreq == 1 || stop % cfg.hp.VideoFreq == 0 ||
          (stop > 3 * T / 4 && stop % cfg.hp.ShearStressFreq == 0))
        break;
      stop++;
    }
    if (t % cfg.hp.ConsolePrintFreq == 1) printf("%s %d\n", "Starting iteration", t);
    CHECK(d3q19_run(ctx, t, stop - t + 1));
    t = stop;
    if (t % cfg.hp.VideoFreq == 0) {
      CHECK(d3q19_read_u(ctx, u));
      if (np > 0) CHECK(d3q19_read_parkin(ctx, parKin));
      if (vid) d3q19h_continuous_output(&cfg, u, parKin, vid, t);
    }
    if (t > 3 * T / 4 && t % cfg.hp.ShearStressFreq == 0) {
      CHECK(d3q19_read_u(ctx, u));
      d3q19h_compute_shear_stress(&out, &cfg, u, "velocity_profile_z.txt");
    }
    t++;
  }
  CHECK(d3q19_synchronize(ctx));
  printf("Checkpoint: end of simulation loop\n");
  CHECK(d3q19_read_u(ctx, u));
  d3q19h_write_lattice_field(&cfg, u, "velocity_field_final.txt", "matlab_postproc/velocity_field_centerline.txt");
  if (np > 0) {
    CHECK(d3q19_read_parfluidforce(ctx, parFluidForce));
    float ff[3] = {0, 0, 0};
    for (int fa = 0; fa < cfg.ip.WorkGroupsPerParticle; fa++) {
      for (int d = 0; d < 3; d++) ff[d] += parFluidForce[4 * fa + d];
      printf("Final force += %f %f %f\n", parFluidForce[4 * fa], parFluidForce[4 * fa + 1],
             parFluidForce[4 * fa + 2]);
    }
    printf("Final force on particle 1 = %f %f %f\n", ff[0], ff[1], ff[2]);
  }
  long long clamps = d3q19_tau_clamp_count(ctx);
  if (clamps > 0) printf("Warning: tau clamped to 0.505 at %lld node updates\n", clamps);
  printf("Checkpoint: end of output\n");
  if (vid) fclose(vid);
  d3q19_destroy(ctx);
  free(f); free(u); free(tau); free(parKin); free(parForce); free(parFluidForce); free(spherePoints);
  free(parsZone); free(zoneMembers); free(numParInZone); free(threadMembers); free(numParInThread); free(znd);
  free(strMap);
  return 0;
}
