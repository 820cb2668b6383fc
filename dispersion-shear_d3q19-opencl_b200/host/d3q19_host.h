/* d3q19_host.h -- host side of the D3Q19 LBM + IBM simulation: input
 * parsing, initial state, particle zones, sphere discretisation and the
 * output writers of SB8/Dispersion-Shear_D3Q19-OpenCL (D3Q19-OpenCL.c), in C,
 * driving the GPU through the C ABI of include/d3q19_b200.h.
 *
 * Keywords, defaults, initialisation order, random-number use and output
 * formats follow the reference so that its input files and post-processing
 * work unchanged.  Keywords the reference does not have are marked "new".
 */
#ifndef D3Q19_HOST_H
#define D3Q19_HOST_H

#include <stdio.h>

#include "../../include/d3q19_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define D3Q19H_WORD 128

/* host_param_struct of D3Q19-OpenCL_header.h:74-93 plus the new keywords. */
typedef struct {
  int ConsolePrintFreq;
  char InitialDist[D3Q19H_WORD];
  float InitialVel[3];
  int InitialParticleDistribution;
  float ParticleBuffer;
  int InterpOrderIBM;
  int DomainDecomp[3];
  float ParticleDensity;
  int RebuildFreq;
  int VideoFreq;
  int FluidOutputSpacing;
  int TangentialVelBC[3];
  int ShearStressFreq;
  float RandParticleShift;
  /* new keywords */
  int UseConstantViscosity;   /* use_constant_viscosity (1 = GPU_program.cl as shipped) */
  int PointsOverride;         /* ibm_points_per_particle (0 = the reference's rule) */
  int FixedParticles;         /* fixed_particles */
  unsigned ParticleSeed;      /* particle_seed, for initial_particle_distribution 4 */
  float MinParticleGap;       /* min_particle_gap, for initial_particle_distribution 4 */
  float TauMax;               /* tau_max (0 = no upper clamp) */
  float TauMin;               /* tau_min (0 = the reference's 0.505) */
  float CassonReg;            /* casson_regularisation (0 = none) */
  int Collision;              /* lbm_collision: 0 MRT (reference), 1 BGK */
  int Storage;                /* storage_precision: 0 fp32, 1 fp16 shifted, 2 bf16 shifted */
  int ParticlePrecision;      /* particle_precision: 0 fp32 (reference), 1 fp64 */
  int Arithmetic;             /* reference_arithmetic: 1 = the reference's evaluation order */
  int Fp64Build;              /* fp64_build: 1 = the FP64 build of the fast kernels (arithmetic 2) */
  int Inplace;                /* inplace_streaming: 1 = one distribution buffer (AA pattern) */
  int PeriodicSmoothing;      /* periodic_force_smoothing: 1 = the force smoothing wraps across periodic axes */
} d3q19h_host_params;

typedef struct {
  int_param_struct ip;
  flp_param_struct fp;
  d3q19h_host_params hp;
} d3q19h_config;

/* initialize_data (D3Q19-OpenCL.c:6-91): defaults, then each line of the
 * text in order; a line sets every keyword it contains as a substring. */
int d3q19h_parse_text(const char* text, d3q19h_config* cfg);
int d3q19h_parse_file(const char* path, d3q19h_config* cfg);
/* One keyword line, as process_input_line (D3Q19-OpenCL.c:612-668). */
void d3q19h_process_line(const char* line, d3q19h_config* cfg);

/* parameter_checking (D3Q19-OpenCL.c:94-109): 0 when usable. */
int d3q19h_check(const d3q19h_config* cfg);

/* sphere_discretization (D3Q19-OpenCL.c:558-610): marker count, point area
 * and the radius-scaled unit-sphere points (float4[P], caller frees).  Reads
 * <data_dir>/unit_sphere_partitions/unit_sphere_partition_<P>.txt when it
 * exists, otherwise generates the same recursive zonal equal-area points.
 * Returns 0, or -1 on a malformed file. */
int d3q19h_sphere_discretization(d3q19h_config* cfg, const char* data_dir, float** points);

/* Recursive zonal equal-area partition of the unit sphere (Leopardi 2006,
 * "A partition of the unit sphere into regions of equal area and small
 * diameter"): region centre points, xyz[3*N]. */
void d3q19h_eqsp_points(int N, double* xyz);

/* create_LB_kernels (D3Q19-OpenCL.c:536-550): work-group split of the IBM
 * markers from the kernel's work-group size. */
void d3q19h_work_groups(d3q19h_config* cfg, int kernel_work_group_size);

/* initialize_lattice_fields (D3Q19-OpenCL.c:111-189); also sets SystemSize.
 * f float[19*N_C], u float[3*N_C], tau float[N_C]. */
int d3q19h_init_lattice(d3q19h_config* cfg, float* f, float* u, float* tau);

/* initialize_particle_fields (D3Q19-OpenCL.c:191-342): parKin float4[4np],
 * parForce float4[2np], parFluidForce float4[2*np*nfa].  Returns 0 or -1. */
int d3q19h_init_particles(d3q19h_config* cfg, float* parKin, float* parForce, float* parFluidForce);

/* initialize_particle_zones (D3Q19-OpenCL.c:344-463).  Sets NumZones and
 * ZoneWidth, then fills the caller's arrays, sized with d3q19h_zone_count()
 * afterwards: parsZone[np], zoneMembers[Z*np], numParInZone[Z],
 * threadMembers[T*np], numParInThread[T], zoneNeighDat[28*Z]. */
void d3q19h_zone_grid(d3q19h_config* cfg);
int d3q19h_zone_count(const d3q19h_config* cfg);
int d3q19h_init_zones(const d3q19h_config* cfg, const float* parKin, int* parsZone, int* zoneMembers,
                      int* numParInZone, int* threadMembers, int* numParInThread, int* zoneNeighDat);

/* Output writers (D3Q19-OpenCL.c:670-835), identical formats. */
typedef struct {
  int ShearStressCount;
  float ShearStressAvg;
  float ActualShearRate;
} d3q19h_output_state;
int d3q19h_compute_shear_stress(d3q19h_output_state* st, const d3q19h_config* cfg, const float* u,
                                const char* profile_path);
void d3q19h_continuous_output(const d3q19h_config* cfg, const float* u, const float* parKin, FILE* vid, int frame);
int d3q19h_write_lattice_field(const d3q19h_config* cfg, const float* u, const char* field_path,
                               const char* centerline_path);

/* Options of the C ABI implied by the configuration. */
void d3q19h_options(const d3q19h_config* cfg, d3q19_options* opt);

#ifdef __cplusplus
}
#endif
#endif
