/* d3q19_host.c -- host side of the simulation (see d3q19_host.h).
 *
 * Each routine restates the corresponding host routine of the reference's
 * D3Q19-OpenCL.c (file:line in the comments) with the same float/double
 * evaluation, so that the initial state and the output files are the
 * reference's, byte for byte.  Differences are called out where the
 * reference reads uninitialised memory or loops forever.
 */
#include "d3q19_host.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

enum { T_INT, T_FLOAT, T_INT3, T_FLOAT3, T_FLOAT4, T_STRING, T_UINT };

typedef struct {
  const char* key;
  int type;
  size_t off;  /* byte offset into d3q19h_config */
  const char* def;
} keyword_t;

#define IPO(f) offsetof(d3q19h_config, ip.f)
#define FPO(f) offsetof(d3q19h_config, fp.f)
#define HPO(f) offsetof(d3q19h_config, hp.f)

/* The reference's keyword table with its defaults (D3Q19-OpenCL.c:31-64),
 * in the same order, followed by the new keywords.  maintain_shear_rate is
 * a 3-int keyword stored at MaintainShear, so it also writes ViscosityModel
 * and NumParticles (D3Q19-OpenCL.c:45, 636-641); where the reference copies
 * uninitialised stack values for the missing numbers, 0 is written. */
static const keyword_t KEYWORDS[] = {
    {"iterations", T_INT, IPO(MaxIterations), "1000"},
    {"console_print_freq", T_INT, HPO(ConsolePrintFreq), "10"},
    {"constant_body_force", T_FLOAT3, FPO(ConstBodyForce), "0.0 0.0 0.0"},
    {"newtonian_tau", T_FLOAT, FPO(NewtonianTau), "1.0"},
    {"viscosity_model", T_INT, IPO(ViscosityModel), "0"},
    {"viscosity_params", T_FLOAT4, FPO(ViscosityParams), "0.0 0.0 0.0 0.0"},
    {"total_lattice_size", T_INT3, IPO(LatticeSize), "32 32 32"},
    {"domain_decomposition", T_INT3, HPO(DomainDecomp), "2 2 2"},
    {"lattice_buffer_size", T_INT3, IPO(BufferSize), "1 1 1"},
    {"initial_f", T_STRING, HPO(InitialDist), "zero"},
    {"initial_vel", T_FLOAT3, HPO(InitialVel), "0.0 0.0 0.0"},
    {"boundary_conditions_xyz", T_INT3, IPO(BoundaryConds), "0 0 0"},
    {"tangential_vel_bcs", T_INT3, HPO(TangentialVelBC), "0 0 0"},
    {"maintain_shear_rate", T_INT3, IPO(MaintainShear), "0"},
    {"velocity_bc_upper", T_FLOAT3, FPO(VelUpper), "0.0 0.0 0.0"},
    {"velocity_bc_lower", T_FLOAT3, FPO(VelLower), "0.0 0.0 0.0"},
    {"num_particles", T_INT, IPO(NumParticles), "0"},
    {"initial_particle_distribution", T_INT, HPO(InitialParticleDistribution), "1"},
    {"random_particle_shift", T_FLOAT, HPO(RandParticleShift), "0.0"},
    {"initial_particle_buffer", T_FLOAT, HPO(ParticleBuffer), "4.0"},
    {"z_wall_particle_buffer", T_FLOAT, FPO(ParticleZBuffer), "10.0"},
    {"particle_diameter", T_FLOAT, FPO(ParticleDiam), "8.0"},
    {"particle_density", T_FLOAT, HPO(ParticleDensity), "1.0"},
    {"particle_collision_model", T_INT, IPO(ParForceModel), "1"},
    {"particle_collision_params", T_FLOAT, FPO(ParForceParams), "1.0, 0.0"},
    {"surf_point_write_atomic", T_INT, IPO(MaxSurfPointsPerNode), "8"},
    {"ibm_interpolation_mode", T_INT, HPO(InterpOrderIBM), "1"},
    {"direct_forcing_coeff", T_FLOAT, FPO(DirectForcingCoeff), "1.0"},
    {"rebuild_neigh_list_freq", T_INT, HPO(RebuildFreq), "10"},
    {"video_freq", T_INT, HPO(VideoFreq), "1000"},
    {"shear_stress_freq", T_INT, HPO(ShearStressFreq), "1000"},
    {"fluid_ouput_spacing", T_INT, HPO(FluidOutputSpacing), "1"},
    /* new keywords (no counterpart in the reference) */
    {"use_constant_viscosity", T_INT, HPO(UseConstantViscosity), "1"},
    {"ibm_points_per_particle", T_INT, HPO(PointsOverride), "0"},
    {"fixed_particles", T_INT, HPO(FixedParticles), "0"},
    {"particle_seed", T_UINT, HPO(ParticleSeed), "1"},
    {"min_particle_gap", T_FLOAT, HPO(MinParticleGap), "0.0"},
    {"tau_max", T_FLOAT, HPO(TauMax), "0.0"},
    {"tau_min", T_FLOAT, HPO(TauMin), "0.0"},
    {"casson_regularisation", T_FLOAT, HPO(CassonReg), "0.0"},
    {"lbm_collision", T_INT, HPO(Collision), "0"},
    {"storage_precision", T_INT, HPO(Storage), "0"},
    {"particle_precision", T_INT, HPO(ParticlePrecision), "0"},
    {"reference_arithmetic", T_INT, HPO(Arithmetic), "0"},
    {"fp64_build", T_INT, HPO(Fp64Build), "0"},
    {"inplace_streaming", T_INT, HPO(Inplace), "0"},
    {"periodic_force_smoothing", T_INT, HPO(PeriodicSmoothing), "0"},
};
#define NKEYWORDS ((int)(sizeof(KEYWORDS) / sizeof(KEYWORDS[0])))

void d3q19h_process_line(const char* line, d3q19h_config* cfg) {
  for (int k = 0; k < NKEYWORDS; k++) {
    const keyword_t* kw = &KEYWORDS[k];
    if (!strstr(line, kw->key)) continue;
    char* dst = (char*)cfg + kw->off;
    switch (kw->type) {
      case T_INT: {
        int v = 0;
        sscanf(line, "%*s %d", &v);
        memcpy(dst, &v, sizeof(v));
        break;
      }
      case T_UINT: {
        unsigned v = 0;
        sscanf(line, "%*s %u", &v);
        memcpy(dst, &v, sizeof(v));
        break;
      }
      case T_FLOAT: {
        float v = 0.0f;
        sscanf(line, "%*s %f", &v);
        memcpy(dst, &v, sizeof(v));
        break;
      }
      case T_INT3: {
        int v[3] = {0, 0, 0};
        sscanf(line, "%*s %d %d %d", v, v + 1, v + 2);
        memcpy(dst, v, sizeof(v));
        break;
      }
      case T_FLOAT3: {
        float v[3] = {0, 0, 0};
        sscanf(line, "%*s %f %f %f", v, v + 1, v + 2);
        memcpy(dst, v, sizeof(v));
        break;
      }
      case T_FLOAT4: {
        float v[4] = {0, 0, 0, 0};
        sscanf(line, "%*s %f %f %f %f", v, v + 1, v + 2, v + 3);
        memcpy(dst, v, sizeof(v));
        break;
      }
      case T_STRING: {
        char v[D3Q19H_WORD];
        memset(v, 0, sizeof(v));
        sscanf(line, "%*s %127s", v);
        memcpy(dst, v, sizeof(v));
        break;
      }
    }
  }
}

static void set_defaults(d3q19h_config* cfg) {
  /* D3Q19 velocities and weights (D3Q19-OpenCL.c:9-25). */
  static const int C[19][3] = {{0, 0, 0},  {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
                               {1, 1, 0},  {1, -1, 0},  {1, 0, 1},  {1, 0, -1}, {-1, 1, 0}, {-1, -1, 0}, {-1, 0, 1},
                               {-1, 0, -1}, {0, 1, 1},  {0, 1, -1}, {0, -1, 1}, {0, -1, -1}};
  memset(cfg, 0, sizeof(*cfg));
  for (int q = 0; q < 19; q++) {
    cfg->fp.EqWeights[q] = q == 0 ? 1.0f / 3.0f : (q < 7 ? 1.0f / 18.0f : 1.0f / 36.0f);
    for (int d = 0; d < 3; d++) cfg->ip.BasisVel[q][d] = C[q][d];
  }
  for (int k = 0; k < NKEYWORDS; k++) {
    char line[2 * D3Q19H_WORD + 2];
    snprintf(line, sizeof(line), "%s %s", KEYWORDS[k].key, KEYWORDS[k].def);
    d3q19h_process_line(line, cfg);
  }
}

int d3q19h_parse_text(const char* text, d3q19h_config* cfg) {
  set_defaults(cfg);
  /* Lines as fgets(fLine, 128, ...) delivers them (D3Q19-OpenCL.c:78-84). */
  const char* p = text;
  while (p && *p) {
    char line[128];
    int n = 0;
    while (*p && n < 127) {
      char ch = *p++;
      line[n++] = ch;
      if (ch == '\n') break;
    }
    line[n] = 0;
    d3q19h_process_line(line, cfg);
  }
  return 0;
}

int d3q19h_parse_file(const char* path, d3q19h_config* cfg) {
  FILE* fh = fopen(path, "rb");
  if (!fh) return -1;
  fseek(fh, 0, SEEK_END);
  long n = ftell(fh);
  rewind(fh);
  char* buf = (char*)malloc((size_t)n + 1);
  size_t got = fread(buf, 1, (size_t)n, fh);
  buf[got] = 0;
  fclose(fh);
  int rc = d3q19h_parse_text(buf, cfg);
  free(buf);
  return rc;
}

int d3q19h_check(const d3q19h_config* cfg) {
  const int* bc = cfg->ip.BoundaryConds;
  if (bc[0] + bc[1] + bc[2] > 1) {
    printf("Error: More than 1 pair of faces with velocity boundaries not yet supported.\n");
    return 1;
  }
  return 0;
}

/* --- unit-sphere partitions ---------------------------------------------- */

static double round_half_away(double x) { return x >= 0 ? floor(x + 0.5) : -floor(-x + 0.5); }
static double cap_area(double s) { return 4.0 * M_PI * sin(s / 2) * sin(s / 2); }
static double cap_radius(double area) { return 2.0 * asin(sqrt(area / M_PI) / 2.0); }
static int gcd_i(int a, int b) { return b ? gcd_i(b, a % b) : a; }

void d3q19h_eqsp_points(int N, double* xyz) {
  /* Collars: polar caps of one region each, then collars whose region
   * counts are the ideal (area-proportional) counts rounded with carried
   * discrepancy; region centres at the mid colatitude of each collar, at
   * equally spaced longitudes rotated collar to collar. */
  const double A = 4.0 * M_PI / N;
  double c = N > 2 ? cap_radius(A) : M_PI / 2;
  int nc = N > 2 ? (int)fmax(1.0, round_half_away((M_PI - 2 * c) / sqrt(A))) : 0;
  int* n = (int*)calloc((size_t)nc + 2, sizeof(int));
  double* s = (double*)calloc((size_t)nc + 2, sizeof(double));
  double disc = 0.0;
  for (int k = 0; k < nc + 2; k++) {
    double r = 1.0;
    if (k >= 1 && k <= nc) {
      double af = (M_PI - 2 * c) / nc;
      r = (cap_area(c + k * af) - cap_area(c + (k - 1) * af)) / A;
    }
    n[k] = (int)round_half_away(r + disc);
    disc += r - n[k];
  }
  s[0] = c;
  int sub = 1;
  for (int k = 1; k <= nc; k++) {
    sub += n[k];
    s[k] = cap_radius(sub * A);
  }
  s[nc + 1] = M_PI;
  int pt = 0;
  double phi0[2] = {0.0, 0.0}, th0[2] = {0.0, M_PI};
  xyz[0] = sin(th0[0]) * cos(phi0[0]);
  xyz[1] = sin(th0[0]) * sin(phi0[0]);
  xyz[2] = cos(th0[0]);
  pt = 1;
  double off = 0.0;
  for (int k = 1; k <= nc; k++) {
    const double th = (s[k - 1] + s[k]) / 2;
    const int m = n[k];
    for (int j = 0; j < m; j++) {
      double phi = fmod((j + 0.5) * 2 * M_PI / m + 2 * M_PI * off, 2 * M_PI);
      xyz[3 * pt] = sin(th) * cos(phi);
      xyz[3 * pt + 1] = sin(th) * sin(phi);
      xyz[3 * pt + 2] = cos(th);
      pt++;
    }
    const int nb = n[k + 1];
    off += (1.0 / nb - 1.0 / m) / 2 + (double)gcd_i(m, nb) / (2.0 * m * nb);
    off -= floor(off);
  }
  xyz[3 * pt] = sin(th0[1]) * cos(phi0[1]);
  xyz[3 * pt + 1] = sin(th0[1]) * sin(phi0[1]);
  xyz[3 * pt + 2] = cos(th0[1]);
  free(n);
  free(s);
}

int d3q19h_sphere_discretization(d3q19h_config* cfg, const char* data_dir, float** points) {
  /* D3Q19-OpenCL.c:558-610. */
  float d = cfg->fp.ParticleDiam;
  float area = M_PI * d * d;
  int numPoints = 1;
  int power2 = (int)ceil(log2(area));
  for (int i = 0; i < power2; i++) numPoints *= 2;
  numPoints = numPoints < 128 ? 128 : numPoints;
  numPoints = numPoints > 1024 ? 1024 : numPoints;
  if (cfg->hp.PointsOverride > 0) numPoints = cfg->hp.PointsOverride;
  cfg->ip.PointsPerParticle = numPoints;
  cfg->ip.TotalSurfPoints = numPoints * cfg->ip.NumParticles;
  cfg->fp.PointArea = area / (float)numPoints;
  float* pts = (float*)calloc((size_t)numPoints * 4, sizeof(float));
  char path[4096];
  snprintf(path, sizeof(path), "%s%sunit_sphere_partitions/unit_sphere_partition_%d.txt", data_dir ? data_dir : "",
           (data_dir && *data_dir) ? "/" : "", numPoints);
  FILE* fs = fopen(path, "r");
  double* gen = NULL;
  if (!fs) {
    gen = (double*)malloc(sizeof(double) * 3 * numPoints);
    d3q19h_eqsp_points(numPoints, gen);
  }
  for (int n = 0; n < numPoints; n++) {
    float px, py, pz;
    if (fs) {
      if (fscanf(fs, "%f,%f,%f\n", &px, &py, &pz) != 3) {
        fclose(fs);
        free(pts);
        return -1;
      }
    } else {
      /* The shipped files hold the points to 5 significant digits; the
       * generated points pass through the same text form. */
      char buf[128];
      snprintf(buf, sizeof(buf), "%.5g,%.5g,%.5g", gen[3 * n], gen[3 * n + 1], gen[3 * n + 2]);
      sscanf(buf, "%f,%f,%f", &px, &py, &pz);
    }
    float lenSq = px * px + py * py + pz * pz;
    if (!(lenSq < 1.01 && lenSq > 0.99)) {
      if (fs) fclose(fs);
      free(pts);
      free(gen);
      return -1;
    }
    pts[4 * n] = px * (0.5f * d);
    pts[4 * n + 1] = py * (0.5f * d);
    pts[4 * n + 2] = pz * (0.5f * d);
    pts[4 * n + 3] = 0.0f;
  }
  if (fs) fclose(fs);
  free(gen);
  *points = pts;
  return 0;
}

void d3q19h_work_groups(d3q19h_config* cfg, int wg) {
  /* D3Q19-OpenCL.c:540-550. */
  int power2 = (int)ceil(log2(wg) - 1E-6);
  int workSize = 1;
  for (int i = 0; i < power2; i++) workSize *= 2;
  cfg->ip.PointsPerWorkGroup = workSize > cfg->ip.PointsPerParticle ? cfg->ip.PointsPerParticle : workSize;
  /* New: a marker count the work-group size does not divide (384, 320, 448
   * of the shipped partitions with a 256 work group) gets the largest power
   * of two below it that does, where the reference's NDRange would be
   * invalid; every count the reference runs keeps its work-group size. */
  while (cfg->ip.PointsPerWorkGroup > 1 && cfg->ip.PointsPerParticle % cfg->ip.PointsPerWorkGroup != 0)
    cfg->ip.PointsPerWorkGroup /= 2;
  cfg->ip.WorkGroupsPerParticle = cfg->ip.PointsPerWorkGroup > 0
                                      ? cfg->ip.PointsPerParticle / cfg->ip.PointsPerWorkGroup
                                      : 0;
}

/* Host equilibrium (D3Q19-OpenCL.c:1114-1149). */
static void host_feq(float rho, const float* v, float* f) {
  float vx = v[0], vy = v[1], vz = v[2];
  float vsq = vx * vx + vy * vy + vz * vz;
  f[0] = (rho / 3.0f) * (1.0f - 1.5f * vsq);
  f[1] = (rho / 18.0f) * (1.0f + 3.0f * vx + 4.5f * vx * vx - 1.5f * vsq);
  f[2] = (rho / 18.0f) * (1.0f - 3.0f * vx + 4.5f * vx * vx - 1.5f * vsq);
  f[3] = (rho / 18.0f) * (1.0f + 3.0f * vy + 4.5f * vy * vy - 1.5f * vsq);
  f[4] = (rho / 18.0f) * (1.0f - 3.0f * vy + 4.5f * vy * vy - 1.5f * vsq);
  f[5] = (rho / 18.0f) * (1.0f + 3.0f * vz + 4.5f * vz * vz - 1.5f * vsq);
  f[6] = (rho / 18.0f) * (1.0f - 3.0f * vz + 4.5f * vz * vz - 1.5f * vsq);
  const float pr[12][2] = {{vx, vy},  {vx, -vy},  {vx, vz},  {vx, -vz},  {-vx, vy}, {-vx, -vy},
                           {-vx, vz}, {-vx, -vz}, {vy, vz},  {vy, -vz},  {-vy, vz}, {-vy, -vz}};
  for (int k = 0; k < 12; k++) {
    float cu = pr[k][0] + pr[k][1];
    f[7 + k] = (rho / 36.0f) * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * vsq);
  }
}

int d3q19h_init_lattice(d3q19h_config* cfg, float* f, float* u, float* tau) {
  int_param_struct* ip = &cfg->ip;
  const long NC = (long)ip->LatticeSize[0] * ip->LatticeSize[1] * ip->LatticeSize[2];
  /* SystemSize (D3Q19-OpenCL.c:119-128). */
  for (int d = 0; d < 3; d++)
    ip->SystemSize[d] = ip->LatticeSize[d] - 2 * ip->BufferSize[d] - (ip->BoundaryConds[d] == 0 ? 0 : 1);
  if (strstr(cfg->hp.InitialDist, "poiseuille")) {
    fprintf(stderr, "poiseuille starting profile not supported yet\n");
    return -1;
  }
  float vel[3] = {0.0f, 0.0f, 0.0f}, feq[19];
  const int constant = strstr(cfg->hp.InitialDist, "constant") != NULL;
  if (constant) memcpy(vel, cfg->hp.InitialVel, sizeof(vel));
  host_feq(1.0f, vel, feq);
  for (long i = 0; i < NC; i++) {
    for (int q = 0; q < 19; q++) f[i + q * NC] = feq[q];
    u[i] = vel[0];
    u[i + NC] = vel[1];
    u[i + 2 * NC] = vel[2];
    if (tau) tau[i] = cfg->fp.NewtonianTau;
  }
  return 0;
}

/* splitmix64 (Steele, Lea, Flood 2014): the seeded generator of the new
 * random-sequential-addition placement. */
static uint64_t splitmix64(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static double uniform01(uint64_t* s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

int d3q19h_init_particles(d3q19h_config* cfg, float* parKin, float* parForce, float* parFluidForce) {
  int_param_struct* ip = &cfg->ip;
  flp_param_struct* fp = &cfg->fp;
  const d3q19h_host_params* hp = &cfg->hp;
  const int np = ip->NumParticles;
  /* D3Q19-OpenCL.c:196-198. */
  fp->ParticleMass = (4.0f / 3.0f) * M_PI * hp->ParticleDensity * pow(fp->ParticleDiam, 3);
  fp->ParticleMomInertia = 0.1f * fp->ParticleMass * fp->ParticleDiam * fp->ParticleDiam;
  float* K = parKin;
#define KIN(p, c) K[4 * (p) + (c)]
  if (np == 0) return 0;
  if (hp->InitialParticleDistribution == 1) {
    /* Cubic grid (D3Q19-OpenCL.c:207-241). */
    float pb = hp->ParticleBuffer;
    int gridSize = (int)ceil(pow(np, 1.0 / 3.0));
    float sp[3];
    for (int i = 0; i < 3; i++) {
      if (gridSize > 1) {
        sp[i] = ip->SystemSize[i] - 2 * pb;
        sp[i] /= (gridSize - 1);
      } else {
        sp[i] = 0.0f;
      }
    }
    for (int p = 0; p < np; p++) {
      float px = pb + sp[0] * (p / (gridSize * gridSize));
      float py = pb + sp[1] * ((p / gridSize) % gridSize);
      float pz = pb + sp[2] * (p % gridSize);
      KIN(p, 0) = px; KIN(p, 1) = py; KIN(p, 2) = pz; KIN(p, 3) = 0.0f;
      for (int c = 0; c < 4; c++) KIN(p + np, c) = 0.0f;
    }
  } else if (hp->InitialParticleDistribution == 2) {
    /* Jittered n x n x m grid with overlap rejection, glibc rand() from its
     * default seed (D3Q19-OpenCL.c:242-305).  2*rand() wraps as a 32-bit int
     * there; the same wrap is made explicit here. */
    float pb = hp->ParticleBuffer;
    float wN = ip->SystemSize[0] - 2 * pb;
    float wM = ip->SystemSize[2] - 2 * (pb + fp->ParticleZBuffer);
    int mdn = (int)ceil(wM / wN);
    int npl = 0, n = 0;
    while (npl < np) {
      n++;
      npl = n * n * n * mdn;
    }
    int m = n * mdn;
    float sp[3];
    if (np > 1) {
      sp[0] = (ip->SystemSize[0] - 2.0f * pb) / (n - 1.0f);
      sp[1] = (ip->SystemSize[1] - 2.0f * pb) / (n - 1.0f);
      sp[2] = (ip->SystemSize[2] - 2.0f * (pb + fp->ParticleZBuffer)) / (n * mdn - 1.0f);
    } else {
      sp[0] = sp[1] = sp[2] = 0.0f;
    }
    srand(1);
    const float shift = hp->RandParticleShift;
#define JIT() (shift * ((int)(2u * (unsigned)rand()) / (float)RAND_MAX - 1))
    for (int p = 0; p < np; p++) {
      int placed = 0;
      for (long attempt = 0; !placed; attempt++) {
        if (attempt > 10000000L) return -1;  /* the reference loops forever here */
        float px = pb + sp[0] * (p / (n * m)) + JIT();
        float py = pb + sp[1] * ((p / m) % n) + JIT();
        float pz = pb + fp->ParticleZBuffer + sp[2] * (p % m) + JIT();
        int safe = 1;
        for (int p2 = 0; p2 < p; p2++) {
          float rx = KIN(p2, 0) - px, ry = KIN(p2, 1) - py, rz = KIN(p2, 2) - pz;
          float sepSq = rx * rx + ry * ry + rz * rz;
          if (sepSq < fp->ParticleDiam * fp->ParticleDiam) safe = 0;
        }
        if (safe) {
          KIN(p, 0) = px; KIN(p, 1) = py; KIN(p, 2) = pz; KIN(p, 3) = 0.0f;
          for (int c = 0; c < 4; c++) KIN(p + np, c) = 0.0f;
          placed = 1;
        }
      }
    }
#undef JIT
  } else if (hp->InitialParticleDistribution == 3) {
    /* One sphere at x = initial_particle_buffer, centred in y and z
     * (D3Q19-OpenCL.c:306-321).  The reference writes index 1 as the
     * velocity, which is only right for one sphere; more are rejected. */
    if (np > 1) return -1;
    KIN(0, 0) = hp->ParticleBuffer;
    KIN(0, 1) = ((float)ip->SystemSize[1]) / 2.0f;
    KIN(0, 2) = ((float)ip->SystemSize[2]) / 2.0f;
    KIN(0, 3) = 0.0f;
    for (int c = 0; c < 4; c++) KIN(1, c) = 0.0f;
  } else if (hp->InitialParticleDistribution == 4) {
    /* New: random sequential addition with a seed.  Centres uniform in
     * x,y in [buffer, S - buffer), z in [buffer + z_wall_particle_buffer,
     * S_z - buffer - z_wall_particle_buffer); a candidate is kept when its
     * centre is at least diameter + min_particle_gap from every kept centre
     * (x and y periodic). */
    uint64_t st = (uint64_t)hp->ParticleSeed * 0x2545F4914F6CDD1Dull + 0x1234567ull;
    const double pb = hp->ParticleBuffer, zb = fp->ParticleZBuffer;
    const double dmin = fp->ParticleDiam + hp->MinParticleGap;
    const double S[3] = {(double)ip->SystemSize[0], (double)ip->SystemSize[1], (double)ip->SystemSize[2]};
    const double lo[3] = {pb, pb, pb + zb}, hi[3] = {S[0] - pb, S[1] - pb, S[2] - pb - zb};
    if (!(hi[0] > lo[0] && hi[1] > lo[1] && hi[2] >= lo[2])) return -1;
    for (int p = 0; p < np; p++) {
      int placed = 0;
      for (long attempt = 0; attempt < 2000000L && !placed; attempt++) {
        double c[3];
        for (int d = 0; d < 3; d++) c[d] = lo[d] + (hi[d] - lo[d]) * uniform01(&st);
        int ok = 1;
        for (int q = 0; q < p && ok; q++) {
          double r2 = 0.0;
          for (int d = 0; d < 3; d++) {
            double dd = fabs(KIN(q, d) - c[d]);
            if (d < 2 && ip->BoundaryConds[d] == 0 && dd > S[d] / 2) dd = S[d] - dd;
            r2 += dd * dd;
          }
          if (r2 < dmin * dmin) ok = 0;
        }
        if (ok) {
          KIN(p, 0) = (float)c[0]; KIN(p, 1) = (float)c[1]; KIN(p, 2) = (float)c[2]; KIN(p, 3) = 0.0f;
          for (int k = 0; k < 4; k++) KIN(p + np, k) = 0.0f;
          placed = 1;
        }
      }
      if (!placed) return -1;
    }
  } else {
    return -1;
  }
  for (int p = 0; p < np; p++) {
    KIN(p + 2 * np, 0) = 0.0f; KIN(p + 2 * np, 1) = 0.0f; KIN(p + 2 * np, 2) = 0.0f; KIN(p + 2 * np, 3) = 1.0f;
    for (int c = 0; c < 4; c++) KIN(p + 3 * np, c) = 0.0f;
  }
#undef KIN
  memset(parForce, 0, sizeof(float) * 8 * np);
  memset(parFluidForce, 0, sizeof(float) * 8 * (size_t)np * (ip->WorkGroupsPerParticle > 0 ? ip->WorkGroupsPerParticle : 1));
  return 0;
}

void d3q19h_zone_grid(d3q19h_config* cfg) {
  /* D3Q19-OpenCL.c:348-375. */
  int_param_struct* ip = &cfg->ip;
  flp_param_struct* fp = &cfg->fp;
  float vMax = 0.05f;
  for (int i = 0; i < 3; i++) {
    vMax = vMax < fabsf(fp->VelUpper[i]) ? fabsf(fp->VelUpper[i]) : vMax;
    vMax = vMax < fabsf(fp->VelLower[i]) ? fabsf(fp->VelLower[i]) : vMax;
    float nu = (fp->NewtonianTau - 0.5f) / 3.0f;
    float vMaxNewt = fp->ConstBodyForce[i] * (ip->SystemSize[i]) * (ip->SystemSize[i]) / (12.0f * nu);
    vMax = vMax < vMaxNewt ? vMaxNewt : vMax;
  }
  float minZoneWidth = 2 * (vMax * cfg->hp.RebuildFreq) + fp->ParticleDiam;
  for (int i = 0; i < 3; i++) {
    float w = (float)(ip->SystemSize[i]);
    ip->NumZones[i] = floor(w / minZoneWidth) > 0 ? (int)floor(w / minZoneWidth) : 1;
    fp->ZoneWidth[i] = w / (float)ip->NumZones[i];
  }
}

int d3q19h_zone_count(const d3q19h_config* cfg) {
  return cfg->ip.NumZones[0] * cfg->ip.NumZones[1] * cfg->ip.NumZones[2];
}

int d3q19h_init_zones(const d3q19h_config* cfg, const float* parKin, int* parsZone, int* zoneMembers,
                      int* numParInZone, int* threadMembers, int* numParInThread, int* znd) {
  /* D3Q19-OpenCL.c:377-462. */
  const int_param_struct* ip = &cfg->ip;
  const flp_param_struct* fp = &cfg->fp;
  const int np = ip->NumParticles;
  const int nthreads = cfg->hp.DomainDecomp[0] * cfg->hp.DomainDecomp[1] * cfg->hp.DomainDecomp[2];
  const int Z = d3q19h_zone_count(cfg);
  memset(numParInZone, 0, sizeof(int) * Z);
  memset(numParInThread, 0, sizeof(int) * (nthreads > 0 ? nthreads : 1));
  memset(znd, 0, sizeof(int) * 28 * Z);
  for (int p = 0; p < np; p++) {
    int th = (int)(nthreads * p) / np;
    int k = numParInThread[th]++;
    threadMembers[th * np + k] = p;
    int zx = (int)(parKin[4 * p] / fp->ZoneWidth[0]);
    int zy = (int)(parKin[4 * p + 1] / fp->ZoneWidth[1]);
    int zz = (int)(parKin[4 * p + 2] / fp->ZoneWidth[2]);
    int zid = zx + ip->NumZones[0] * (zy + ip->NumZones[1] * zz);
    if (zid < 0 || zid >= Z) return -1;
    parsZone[p] = zid;
    zoneMembers[zid * np + numParInZone[zid]++] = p;
  }
  const int* NZ = ip->NumZones;
  const int* bc = ip->BoundaryConds;
  for (int k = 0; k < NZ[2]; k++)
    for (int j = 0; j < NZ[1]; j++)
      for (int i = 0; i < NZ[0]; i++) {
        int zid = i + NZ[0] * (j + NZ[1] * k);
        znd[28 * zid] = 0;
        int lm = -1, lp = 1, mm = -1, mp = 1, nm = -1, npl = 1;
        if (bc[0] == 1 && i == 0) lm = 0;
        if (bc[1] == 1 && j == 0) mm = 0;
        if (bc[2] == 1 && k == 0) nm = 0;
        if (bc[0] == 1 && i == NZ[0] - 1) lp = 0;
        if (bc[1] == 1 && j == NZ[1] - 1) mp = 0;
        if (bc[2] == 1 && k == NZ[2] - 1) npl = 0;
        for (int n = nm; n <= npl; n++)
          for (int m = mm; m <= mp; m++)
            for (int l = lm; l <= lp; l++) {
              int ls = i + l, ms = j + m, ns = k + n;
              int lw = ls < 0 ? NZ[0] - 1 : ls % NZ[0];
              int mw = ms < 0 ? NZ[1] - 1 : ms % NZ[1];
              int nw = ns < 0 ? NZ[2] - 1 : ns % NZ[2];
              /* y stride NumZones[2], as D3Q19-OpenCL.c:450 has it. */
              int nid = lw + NZ[0] * (mw + NZ[2] * nw);
              int cnt = ++znd[28 * zid];
              znd[28 * zid + cnt] = nid;
            }
      }
  return 0;
}

int d3q19h_compute_shear_stress(d3q19h_output_state* st, const d3q19h_config* cfg, const float* u_h,
                                const char* profile_path) {
  /* D3Q19-OpenCL.c:670-750. */
  const int_param_struct* ip = &cfg->ip;
  const int n_x = ip->LatticeSize[0], n_y = ip->LatticeSize[1], n_z = ip->LatticeSize[2];
  const int n_L = n_x * n_y * n_z;
  FILE* fPtr = fopen(profile_path, "w");
  if (!fPtr) return -1;
  const int gradBuffer = 1;
  const float n_xy = (float)(n_x - 2) * (n_y - 2);
  float* uMeanX = (float*)calloc(n_z, sizeof(float));
  float dudzMean = 0.0f;
  const float dz = 4.0f;
  for (int i_z = 1; i_z < n_z - 1; i_z++) {
    float uMean[3] = {0.0f, 0.0f, 0.0f};
    for (int i_x = 1; i_x < n_x - 1; i_x++)
      for (int i_y = 1; i_y < n_y - 1; i_y++) {
        int i_1D = i_x + ip->LatticeSize[0] * (i_y + ip->LatticeSize[1] * i_z);
        uMean[0] += u_h[i_1D];
        uMean[1] += u_h[i_1D + n_L];
        uMean[2] += u_h[i_1D + 2 * n_L];
        if (i_z == (1 + dz + gradBuffer) || i_z == (n_z - 2 - gradBuffer)) {
          int i_1D_fd = i_x + ip->LatticeSize[0] * (i_y + ip->LatticeSize[1] * (i_z - dz));
          dudzMean += (u_h[i_1D] - u_h[i_1D_fd]) / dz;
        }
      }
    uMean[0] /= n_xy;
    uMeanX[i_z] = uMean[0];
    uMean[1] /= n_xy;
    uMean[2] /= n_xy;
    fprintf(fPtr, "%8.6f %8.6f %8.6f\n", uMean[0], uMean[1], uMean[2]);
  }
  dudzMean /= (2.0 * n_xy);
  int count = ++(st->ShearStressCount);
  st->ShearStressAvg = (st->ShearStressAvg * (count - 1) + dudzMean) / count;
  printf("Shear rate at wall = %e\n", st->ShearStressAvg);
  int intBuffer = (int)(cfg->fp.ParticleZBuffer + 1E-8) + (int)(cfg->fp.ParticleDiam / 2);
  int zbL = 1 + intBuffer;
  int zbU = (int)(n_z - 2 - intBuffer);
  float actual = 0.0f;
  /* The reference indexes uMeanX without a range check; outside it the
   * particle-region rate is left at 0. */
  if (zbL >= 0 && zbL < n_z && zbU >= 0 && zbU < n_z && zbU != zbL)
    actual = (uMeanX[zbU] - uMeanX[zbL]) / (zbU - zbL);
  st->ActualShearRate = (st->ActualShearRate * (count - 1) + actual) / count;
  printf("Shear rate in particle region = %e\n", st->ActualShearRate);
  fclose(fPtr);
  free(uMeanX);
  return 0;
}

void d3q19h_continuous_output(const d3q19h_config* cfg, const float* u_h, const float* parKin, FILE* vid,
                              int frame) {
  /* D3Q19-OpenCL.c:752-792. */
  const int_param_struct* ip = &cfg->ip;
  const int n_x = ip->LatticeSize[0], n_y = ip->LatticeSize[1], n_z = ip->LatticeSize[2];
  const int n_s = cfg->hp.FluidOutputSpacing;
  const int n_L = n_x * n_y * n_z;
  const int n_fluid = (int)(1 + (n_x - 3) / n_s) * (1 + (n_y - 3) / n_s) * (1 + (n_z - 3) / n_s);
  const int n_par = ip->NumParticles;
  fprintf(vid, "%d\n", n_fluid + n_par);
  fprintf(vid, "D3Q19_output, frame %d\n", frame);
  for (int i_x = 1; i_x < n_x - 1; i_x += n_s)
    for (int i_y = 1; i_y < n_y - 1; i_y += n_s)
      for (int i_z = 1; i_z < n_z - 1; i_z += n_s) {
        int i_1D = i_x + n_x * (i_y + n_y * i_z);
        fprintf(vid, "1 ");
        fprintf(vid, "%d %d %d ", i_x - 1, i_y - 1, i_z - 1);
        fprintf(vid, "%8.6f %8.6f %8.6f\n", u_h[i_1D], u_h[i_1D + n_L], u_h[i_1D + 2 * n_L]);
      }
  for (int p = 0; p < n_par; p++) {
    fprintf(vid, "2 ");
    fprintf(vid, "%.2f %.2f %.2f ", parKin[4 * p], parKin[4 * p + 1], parKin[4 * p + 2]);
    fprintf(vid, "%8.6f %8.6f %8.6f\n", parKin[4 * (p + n_par)], parKin[4 * (p + n_par) + 1],
            parKin[4 * (p + n_par) + 2]);
  }
}

int d3q19h_write_lattice_field(const d3q19h_config* cfg, const float* field, const char* field_path,
                               const char* centerline_path) {
  /* D3Q19-OpenCL.c:794-835. */
  const int_param_struct* ip = &cfg->ip;
  const int n_C = ip->LatticeSize[0] * ip->LatticeSize[1] * ip->LatticeSize[2];
  FILE* f1 = fopen(field_path, "w");
  if (!f1) return -1;
  for (int i_x = 1; i_x < ip->LatticeSize[0] - 1; i_x++)
    for (int i_y = 1; i_y < ip->LatticeSize[1] - 1; i_y++)
      for (int i_z = 1; i_z < ip->LatticeSize[2] - 1; i_z++) {
        int i_1D = i_x + ip->LatticeSize[0] * (i_y + ip->LatticeSize[1] * i_z);
        fprintf(f1, "%d %d %d ", i_x, i_y, i_z);
        fprintf(f1, "%9.7f %9.7f %9.7f\n", field[i_1D], field[i_1D + n_C], field[i_1D + 2 * n_C]);
      }
  fclose(f1);
  FILE* f2 = fopen(centerline_path, "w");
  if (!f2) return -2;
  int i_y = (int)floor((float)ip->LatticeSize[1] / 2.0f);
  for (int i_x = 1; i_x < ip->LatticeSize[0] - 1; i_x++)
    for (int i_z = 1; i_z < ip->LatticeSize[2] - 1; i_z++) {
      int i_1D = i_x + ip->LatticeSize[0] * (i_y + ip->LatticeSize[1] * i_z);
      fprintf(f2, "%d %d %d ", i_x, i_y, i_z);
      fprintf(f2, "%9.7f %9.7f %9.7f\n", field[i_1D], field[i_1D + n_C], field[i_1D + 2 * n_C]);
    }
  fclose(f2);
  return 0;
}

void d3q19h_options(const d3q19h_config* cfg, d3q19_options* o) {
  memset(o, 0, sizeof(*o));
  o->variable_viscosity = cfg->hp.UseConstantViscosity ? 0 : 1;
  o->collision = cfg->hp.Collision;
  o->storage = cfg->hp.Storage;
  o->particle_precision = cfg->hp.ParticlePrecision;
  o->fixed_particles = cfg->hp.FixedParticles;
  o->num_par_threads = cfg->hp.DomainDecomp[0] * cfg->hp.DomainDecomp[1] * cfg->hp.DomainDecomp[2];
  o->rebuild_freq = cfg->hp.RebuildFreq;
  for (int d = 0; d < 3; d++) o->tangential_vel_bc[d] = cfg->hp.TangentialVelBC[d];
  o->tau_max = cfg->hp.TauMax;
  o->tau_min = cfg->hp.TauMin;
  o->arithmetic = cfg->hp.Fp64Build ? 2 : cfg->hp.Arithmetic;
  o->inplace = cfg->hp.Inplace;
  o->periodic_smoothing = cfg->hp.PeriodicSmoothing;
  o->casson_reg = cfg->hp.CassonReg;
}
