/* d3q19_oracle.h -- CPU restatement of the reference's D3Q19 LBM + IBM time
 * step (SB8/Dispersion-Shear_D3Q19-OpenCL), used ONLY as the checker.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load this library.  The product path never links it.
 *
 * Each function restates one reference kernel or host routine and cites the
 * reference file:line it follows.  Arrays use the reference's layouts:
 *   f      float[19][N_C]   q-major SoA, x fastest (GPU_program.cl:347-350)
 *   u      float[3][N_C]
 *   gpf    float[3*MaxSurfPointsPerNode][N_C]
 *   parKin float4[4*np]     position, velocity, quaternion, angular velocity
 *
 * Pinning: tests/test_oracle_pin.py compares this oracle with the reference
 * itself, built from its own sources by oracle/refbuild/build_ref.sh and run
 * on the host through a mock OpenCL runtime (golden vectors committed under
 * tests/golden/).
 */
#ifndef D3Q19_ORACLE_H
#define D3Q19_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as struct_header_device.h:4-57 (332 and 176 bytes). */
typedef struct {
  int MaxIterations;
  int BasisVel[19][3];
  int LatticeSize[3];
  int SystemSize[3];
  int BufferSize[3];
  int BoundaryConds[3];
  int NumZones[3];
  int MaintainShear;
  int ViscosityModel;
  int NumParticles;
  int ParForceModel;
  int MaxSurfPointsPerNode;
  int InterpOrderIBM;
  int PointsPerParticle;
  int PointsPerWorkGroup;
  int TotalSurfPoints;
  int WorkGroupsPerParticle;
} orc_int_params;

typedef struct {
  float ConstBodyForce[3];
  float EqWeights[19];
  float VelUpper[3];
  float VelLower[3];
  float NewtonianTau;
  float ViscosityParams[4];
  float ZoneWidth[3];
  float ParticleDiam;
  float ParticleMass;
  float PointArea;
  float ParticleMomInertia;
  float ParForceParams[2];
  float ParticleZBuffer;
  float DirectForcingCoeff;
} orc_flp_params;

typedef struct {
  float x, y, z, w;
} orc_float4;

int orc_sizeof_int_params(void);
int orc_sizeof_flp_params(void);

/* GPU_program.cl:316-624.  variable_viscosity = 0 is the kernel as shipped
 * (USE_CONSTANT_VISCOSITY defined), 1 is the build without that define. */
void orc_collide_stream(const float* f_c, float* f_s, const float* gpf, float* u, float* tau_lb, int* countPoint,
                        const orc_int_params* ip, const orc_flp_params* fp, int variable_viscosity);

/* GPU_program.cl:626-735 over numPeriodicNodes entries of strMap. */
void orc_boundary_periodic(float* f_s, const orc_int_params* ip, const int* strMap, int numPeriodicNodes);

/* GPU_program.cl:737-865 over (L-2)x(L-2)x2 nodes with offset 1. */
void orc_boundary_velocity(float* f_s, const orc_int_params* ip, const orc_flp_params* fp, int wallAxis,
                           int calcRho);

/* GPU_program.cl:292-313 and 258-289 over the interior. */
void orc_reset_particle_fluid_forces(const orc_int_params* ip, float* gpf);
void orc_sum_particle_fluid_forces(const orc_int_params* ip, float* gpf);

/* GPU_program.cl:81-256, work-groups and work-items executed serially in
 * order (race-free slot semantics).  Also returns, for each marker, the
 * corner cell (x_i0,y_i0,z_i0) in marker_cell[3*m] when non-NULL. */
void orc_particle_fluid_forces(const orc_int_params* ip, const orc_flp_params* fp, float* gpf, const float* u,
                               const orc_float4* parKin, orc_float4* parFluidForce, const orc_float4* spherePoints,
                               int* countPoint, int* marker_cell);

/* CPU_program.cl:187-277. */
void orc_particle_dynamics(const orc_int_params* ip, const orc_flp_params* fp, orc_float4* parKin,
                           orc_float4* parForce, const orc_float4* parFluidForce, const int* threadMembers,
                           const int* numParInThread, int numParThreads);

/* CPU_program.cl:76-184 (+ squeeze force 319-343). */
void orc_particle_particle_forces(const orc_int_params* ip, const orc_flp_params* fp, const orc_float4* parKin,
                                  orc_float4* parForce, const int* zoneNeighDat, const int* parsZone,
                                  const int* threadMembers, const int* numParInThread, int numParThreads,
                                  const int* zoneMembers, const int* numParInZone);

/* CPU_program.cl:280-315 (numParInZone must be zeroed by the caller first,
 * as the host does at sim_main.c:431-441). */
void orc_update_particle_zones(const orc_int_params* ip, const orc_flp_params* fp, const orc_float4* parKin,
                               const int* threadMembers, const int* numParInThread, int numParThreads,
                               int* parsZone, int* zoneMembers, int* numParInZone);

/* D3Q19-OpenCL.c:973-1112.  Writes up to N_C*2 ints; returns the count. */
int orc_create_periodic_stream_mapping(const orc_int_params* ip, int* strMap);

/* D3Q19-OpenCL.c:417-462 (27-entry neighbour table per zone, first entry is
 * the count; reproduces the y-stride quirk of D3Q19-OpenCL.c:450). */
void orc_zone_neighbours(const orc_int_params* ip, int* zoneNeighDat);

/* One full time step t in the order of sim_main.c:324-447.  fA/fB are the
 * two distribution buffers; the step reads f_c = (t even ? fA : fB). */
typedef struct {
  float *fA, *fB, *u, *gpf, *tau_lb;
  int* countPoint;
  orc_float4 *parKin, *parForce, *parFluidForce, *spherePoints;
  int *strMap, numPeriodicNodes;
  int *zoneNeighDat, *parsZone, *zoneMembers, *numParInZone, *threadMembers, *numParInThread;
  int numParThreads, rebuildFreq, variable_viscosity;
  int tangentialVelBC[3];
} orc_state;

void orc_step(orc_state* s, const orc_int_params* ip, const orc_flp_params* fp, int t);

#ifdef __cplusplus
}
#endif
#endif
