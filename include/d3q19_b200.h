/* d3q19_b200.h -- C ABI of the B200 (sm_100a) implementation of the D3Q19
 * lattice-Boltzmann + immersed-boundary sphere-suspension time step of
 * SB8/Dispersion-Shear_D3Q19-OpenCL.
 *
 * The library replaces the reference's OpenCL host API calls and kernel
 * contract (sim_main.c:15-527, D3Q19-OpenCL.c:465-556, 847-971): plain
 * pointers and sizes, host buffers owned by the caller, device memory and one
 * CUDA stream owned by the context.  Every entry point returns 0 on success
 * or a negative d3q19_status; no entry point exits the process (the
 * reference's error_check() calls exit(0), D3Q19-OpenCL.c:1169-1246).
 *
 * Array layouts are the reference's (GPU_program.cl:316-350, 81-90):
 *   f       float[19][N_C]        q-major, x fastest, N_C = Lx*Ly*Lz incl. buffer
 *   u       float[3][N_C]
 *   tau_lb  float[N_C]
 *   parKin  float4[4*np]          position, velocity, quaternion, angular velocity
 *   parForce float4[2*np]         force, torque
 *   parFluidForce float4[2*np*nfa]  per work-group force partials, then torques
 *   spherePoints float4[P]        unit-sphere points scaled by the radius
 */
#ifndef D3Q19_B200_H
#define D3Q19_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Parameter blocks, byte-for-byte the layout of struct_header_device.h:4-57
 * (332 and 176 bytes); the reference uploads them raw (sim_main.c:204-205). */
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
} int_param_struct;

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
} flp_param_struct;

enum d3q19_status {
  D3Q19_OK = 0,
  D3Q19_EINVAL = -1,    /* bad argument or unsupported parameter combination */
  D3Q19_ENOMEM = -2,    /* device allocation failed */
  D3Q19_ECUDA = -3,     /* CUDA runtime error (see d3q19_last_error) */
  D3Q19_ENODEV = -4,    /* no usable sm_100 device */
  D3Q19_EOVERFLOW = -5, /* a lattice tile received more IBM markers than its list holds */
  D3Q19_ENUMERIC = -6,  /* non-finite density or velocity detected on the device */
  D3Q19_ESTATE = -7,    /* call out of order (e.g. step before the lattice is written) */
  D3Q19_EBUSY = -8,     /* the pool has no free slot or HBM budget for the request right now */
  D3Q19_EBOUNDS = -9,   /* library built with D3Q19_BOUNDS_CHECK: a device index fell outside its array (the
                           access was skipped); no counterpart in the reference */
  D3Q19_ETIMEDOUT = -10 /* a bounded device wait ran out (a TMA load of the collide-stream pass did not complete
                           within its limit); no counterpart in the reference */
};

/* Options with no counterpart in the reference's parameter structs.  A
 * zero-initialised struct reproduces the reference as shipped. */
typedef struct {
  /* 0: GPU_program.cl as shipped (USE_CONSTANT_VISCOSITY defined, tau =
   * NewtonianTau).  1: the reference's other build, without that define
   * (GPU_program.cl:457-564): local tau from the strain rate (power-law,
   * Casson, Herschel-Bulkley via ViscosityModel). */
  int variable_viscosity;
  /* 0: the reference's MRT rates (GPU_program.cl:453, 567-568).
   * 1: BGK, every rate 1/tau (GPU_program.cl:867-947 generalised). */
  int collision;
  /* 0: FP32 distributions (reference).  1: FP16, 2: BF16 storage of
   * f_i - w_i with FP32 arithmetic. */
  int storage;
  /* 0: FP32 particle state and sums in the reference's order.
   * 1: FP64 sphere state, marker positions, interpolation and forces, the
   * per-sphere force/torque sums and the Newton-Euler integration (the
   * float read-backs hold rounded copies; d3q19_read_parkin64 the state). */
  int particle_precision;
  /* 1: spheres keep their initial position and velocity (forces are still
   * computed and reported). */
  int fixed_particles;
  /* Particle work split of the reference's CPU device (numParThreads =
   * product of domain_decomposition, sim_main.c:65); used to interpret
   * threadMembers/numParInThread. */
  int num_par_threads;
  /* Zone lists are rebuilt after steps with t % rebuild_freq == 0
   * (rebuild_neigh_list_freq, sim_main.c:429). */
  int rebuild_freq;
  /* Experimental tangential velocity boundaries (tangential_vel_bcs,
   * sim_main.c:388-402). */
  int tangential_vel_bc[3];
  /* Upper clamp of the local tau (0 = none, as the reference). */
  float tau_max;
  /* Lower clamp of the local tau (0 = the reference's MIN_TAU 0.505,
   * GPU_program.cl:6). */
  float tau_min;
  /* Casson regularisation: shear rate floor added in quadrature (0 = none). */
  float casson_reg;
  /* CUDA device ordinal. */
  int device;
  /* Markers per lattice tile list (0 = automatic). */
  int ibm_tile_capacity;
  /* 0: fast arithmetic (one forward and one inverse moment transform,
   * contraction allowed, integer fixed-point spreading).  1: the reference's
   * floating-point evaluation order (both transforms as written, no
   * contraction, slot-ordered spreading, contact forces summed in the
   * reference's order): the reference's results bit for bit from the same
   * state, except where a pow() of the viscosity law rounds differently.
   * 2: the FP64 build of the fast kernels (FP64 distributions, arithmetic,
   * local tau, spread smoothing, and particle_precision 1): the oracle the
   * FP32 and 16-bit forms are measured against; the reference's MRT only. */
  int arithmetic;
  /* 0: two distribution buffers, as the reference's fA/fB.  1: one buffer
   * updated in place (AA pattern): even steps read a node's own cells and
   * write them back with the directions reversed, odd steps pull from and
   * push to the neighbours.  Half the distribution memory, the same results
   * bit for bit.  Not with arithmetic 1.  The members of a lattice pool share
   * one layout.  No counterpart in the reference. */
  int inplace;
  /* Collide-stream kernel.  0: the per-tile kernel (fluid_step_kernel).
   * 1: the TMA-pipelined persistent kernel (fluid_tma_kernel) where the
   * context allows it (periodic x and y with walls on z, the reference's MRT,
   * arithmetic 0, FP32 or 16-bit storage, x extent a multiple of 4 (FP32) or
   * 8 (16-bit) nodes), else the per-tile kernel.  The results are the same
   * bit for bit.  On B200 the TMA kernel is the slower of the two for this
   * step (0.0995 against 0.0743 ms per 128^3 fluid step): the step is bound
   * by instruction issue, which staging the loads does not reduce.  No
   * counterpart in the reference. */
  int fluid_kernel;
  /* 0: the reference's 27-point smoothing of the spread force, which reads
   * the buffer layer as zero and does not wrap across periodic axes
   * (GPU_program.cl:356-377): a sphere on a periodic seam loses the part of
   * its reaction force that the smoothing would carry across the seam, and
   * the fluid there gains momentum without a counterpart.  1: the smoothing
   * wraps across periodic x and y, so the spread force on the fluid is the
   * whole marker force.  Not with arithmetic 1.  No counterpart in the
   * reference. */
  int periodic_smoothing;
} d3q19_options;

typedef struct {
  char name[256];
  int sm_count;
  int cc_major, cc_minor;
  size_t global_mem_bytes;
  /* Work-group size the IBM kernel reports; the host derives
   * PointsPerWorkGroup = min(pow2 >= this, PointsPerParticle) from it as the
   * reference does with CL_KERNEL_WORK_GROUP_SIZE (D3Q19-OpenCL.c:536-550). */
  int kernel_work_group_size;
} d3q19_device_info;

typedef struct d3q19_ctx d3q19_ctx;

/* Replaces analyse_platform (D3Q19-OpenCL.c:847-971) and the
 * clGetKernelWorkGroupInfo query (D3Q19-OpenCL.c:536-538). */
int d3q19_get_device_info(int device, d3q19_device_info* out);

/* Replaces clCreateContext / clCreateCommandQueue / program build /
 * clCreateKernel / clCreateBuffer (sim_main.c:15-42, 115-190;
 * D3Q19-OpenCL.c:465-556).  Copies both parameter blocks. */
int d3q19_create(const int_param_struct* ip, const flp_param_struct* fp, const d3q19_options* opt,
                 d3q19_ctx** out);

/* Which collide-stream kernel the context runs: 0 the per-tile kernel
 * (fluid_step_kernel), 1 the TMA-pipelined kernel (fluid_tma_kernel), 2 the
 * reference-order kernel (arithmetic 1); negative on a null context.  No
 * counterpart in the reference. */
int d3q19_fluid_kernel(const d3q19_ctx* ctx);

/* Replaces clEnqueueWriteBuffer of fA/fB/u/tau_lb (sim_main.c:193-198).
 * f is the state the next step reads (both reference buffers start equal);
 * tau_lb may be NULL (filled with NewtonianTau, D3Q19-OpenCL.c:179). */
int d3q19_write_lattice(d3q19_ctx* ctx, const float* f, const float* u, const float* tau_lb);

/* Replaces the particle buffer uploads (sim_main.c:140-150, 189, 202). */
int d3q19_write_particles(d3q19_ctx* ctx, const float* parKin, const float* parForce, const float* parFluidForce,
                          const float* spherePoints);

/* Replaces the zone buffer uploads (sim_main.c:152-177).  zoneNeighDat is
 * int[28*zones], zoneMembers int[zones*np], threadMembers
 * int[num_par_threads*np]. */
int d3q19_write_zones(d3q19_ctx* ctx, const int* zoneNeighDat, const int* parsZone, const int* zoneMembers,
                      const int* numParInZone, const int* threadMembers, const int* numParInThread);

/* Builds the periodic boundary node list of create_periodic_stream_mapping
 * (D3Q19-OpenCL.c:973-1112) into strMap = [indices..., types...] (capacity
 * ints); returns the node count (strMap may be NULL to query it).  Host
 * only, needs no GPU. */
int d3q19_periodic_map(const int_param_struct* ip, int* strMap, int capacity);

/* Replaces the strMap upload (sim_main.c:186, 203).  The periodic copy is
 * fused into the streaming gather, so the map is checked against the one the
 * boundary conditions imply (D3Q19-OpenCL.c:973-1112); a mismatch is
 * D3Q19_EINVAL. */
int d3q19_write_periodic_map(d3q19_ctx* ctx, const int* strMap, int numPeriodicNodes);

/* One time step t (t >= 1) with the order and data dependencies of
 * sim_main.c:324-447: collide-stream with the force spread at step t-1, the
 * periodic and velocity boundaries, the rigid-body update from the forces of
 * step t-1, IBM interpolation of u(t) at the moved markers and spreading,
 * particle-particle forces, and the zone rebuild when t % rebuild_freq == 0.
 * Asynchronous on the context's stream. */
int d3q19_step(d3q19_ctx* ctx, int t);

/* The step in its passes, for kernel-level use; calling them in this order
 * for step t is d3q19_step(ctx, t) (bit for bit), all on the context's
 * stream.  Out-of-order calls return D3Q19_ESTATE.
 *   d3q19_k_collide_stream: collideMRT_stream_D3Q19 + boundary_periodic +
 *     boundary_velocity + the reset and slot sum of the spread force of step
 *     t-1 (GPU_program.cl:258-865), fused;
 *   d3q19_k_particles: particle_dynamics + particle_fluid_forces_linear_stencil
 *     (CPU_program.cl:187-277, GPU_program.cl:81-256);
 *   d3q19_k_contacts: particle_particle_forces (CPU_program.cl:76-184);
 *   d3q19_k_zones: update_particle_zones (CPU_program.cl:280-315), after the
 *     contacts of steps with t % rebuild_neigh_list_freq == 0.
 * The particle passes do nothing without spheres. */
int d3q19_k_collide_stream(d3q19_ctx* ctx, int t);
int d3q19_k_particles(d3q19_ctx* ctx, int t);
int d3q19_k_contacts(d3q19_ctx* ctx, int t);
int d3q19_k_zones(d3q19_ctx* ctx);

/* Steps t0 .. t0+nsteps-1, replayed from captured CUDA graphs: chunks of
 * about 64 steps (a multiple of the step schedule's period, lcm(2,
 * rebuild_neigh_list_freq)) are captured on first use; a shorter rest of at
 * least one period replays a graph captured before by d3q19_prepare_run, and
 * steps one by one otherwise. */
int d3q19_run(d3q19_ctx* ctx, int t0, int nsteps);

/* Captures, without running them, the CUDA graphs a later
 * d3q19_run(ctx, t0, nsteps) replays (with the context's state unchanged),
 * so that the run itself launches no capture: a short run then replays
 * graphs instead of stepping one by one.  Does nothing before the first step
 * after an upload.  No counterpart in the reference. */
int d3q19_prepare_run(d3q19_ctx* ctx, int t0, int nsteps);

/* clFinish (sim_main.c:407, 447): waits for the stream and reports device
 * errors (tile overflow, non-finite values). */
int d3q19_synchronize(d3q19_ctx* ctx);

/* Read-backs (sim_main.c:452-462, 478, 486).  Synchronous. */
int d3q19_read_u(d3q19_ctx* ctx, float* u);
int d3q19_read_tau(d3q19_ctx* ctx, float* tau_lb);
int d3q19_read_parkin(d3q19_ctx* ctx, float* parKin);
int d3q19_read_parforce(d3q19_ctx* ctx, float* parForce);
/* The FP64 sphere state (particle_precision = 1): double[16*np] in the
 * parKin layout.  No counterpart in the reference (its state is float). */
int d3q19_read_parkin64(d3q19_ctx* ctx, double* parKin);
int d3q19_read_parfluidforce(d3q19_ctx* ctx, float* parFluidForce);
/* The distribution buffer the last step wrote, as the reference holds it
 * after the boundary kernels (interior nodes; buffer-layer nodes are 0). */
int d3q19_read_f(d3q19_ctx* ctx, float* f);
/* The spread IBM force field of the last step, as the reference's gpf slot 0
 * after sum_particle_fluid_forces (GPU_program.cl:258-289): float[3][N_C]. */
int d3q19_read_spread_force(d3q19_ctx* ctx, float* gpf0);
/* d3q19_read_spread_force without any device allocation (no counterpart in
 * the reference): the field is built in a fixed array of the library's device
 * image, for callers that may not allocate or free device memory while a run
 * is under way.  Lattices of at most D3Q19_STATIC_SPREAD_MAX_CELLS nodes
 * (N_C, buffer layers included); larger ones return D3Q19_EINVAL.  One array
 * per device and process: calls that overlap in time on the same device race.
 * The first call on each device does a one-time set-up (looks the array up);
 * make it before any stream capture. */
#define D3Q19_STATIC_SPREAD_MAX_CELLS 262144
int d3q19_read_spread_force_static(d3q19_ctx* ctx, float* gpf0);
/* Corner cell (x_i0, y_i0, z_i0) of every marker of the last step
 * (GPU_program.cl:150-156): int[3*TotalSurfPoints]. */
int d3q19_read_marker_cells(d3q19_ctx* ctx, int* cells);
/* Zone lists after the last rebuild (update_particle_zones). */
int d3q19_read_zones(d3q19_ctx* ctx, int* parsZone, int* zoneMembers, int* numParInZone);

/* Sums over every z-plane of the interior nodes, in FP64 on the device (no
 * read-back of the field): out[5*z + 0..2] = sums of u_x, u_y, u_z,
 * out[5*z + 3] = sum of the shear rate du_x/dz + du_z/dx, out[5*z + 4] = sum
 * of the viscous shear stress nu*(du_x/dz + du_z/dx), nu = (tau - 1/2)/3.
 * Central differences, wrapped on periodic axes, one-sided on the wall
 * layers.  out holds 5*LatticeSize[2] doubles (planes 0 and Nz-1 are 0).
 * Device-side form of the averages compute_shear_stress takes on the host
 * (D3Q19-OpenCL.c:670-747). */
int d3q19_plane_stats(d3q19_ctx* ctx, double* out);
/* compute_shear_stress (D3Q19-OpenCL.c:670-747) from the device sums:
 * u_mean[3*z + d] the x-y mean of u_d on plane z (3*Nz doubles, may be
 * NULL), the wall shear rate (forward differences over 4 planes at both
 * walls) and the shear rate across the particle region.  FP64 where the
 * reference accumulates in float. */
int d3q19_shear_profile(d3q19_ctx* ctx, double* u_mean, double* wall_rate, double* region_rate);
/* Domain means over the interior nodes, FP64: the viscous shear stress
 * <nu (du_x/dz + du_z/dx)>, the shear rate <du_x/dz + du_z/dx> and the
 * effective viscosity (their ratio).  No counterpart in the reference. */
int d3q19_mean_stress(d3q19_ctx* ctx, double* stress_xz, double* shear_rate, double* eff_viscosity);

/* Number of lattice nodes whose local tau was clamped to 0.505 since the
 * context was created (the reference prints a device warning instead,
 * GPU_program.cl:1071-1074). */
long long d3q19_tau_clamp_count(d3q19_ctx* ctx);

/* Kernel timing: with enable = 1 the following steps launch eagerly (no graph
 * replay) with CUDA events around every collide-stream and particle launch;
 * enable = 0 stops.  d3q19_profile_read synchronises and returns the summed
 * device time in ms and the launch counts since profiling was enabled.
 * No counterpart in the reference (it has no timers). */
int d3q19_profile(d3q19_ctx* ctx, int enable);
int d3q19_profile_read(d3q19_ctx* ctx, double* fluid_ms, int* fluid_launches, double* particle_ms,
                       int* particle_launches);

/* The context's CUDA stream (cudaStream_t) for callers that order their own
 * work after the step. */
void* d3q19_stream(d3q19_ctx* ctx);

/* Text of the last error on this context (or of the last failed create when
 * ctx is NULL). */
const char* d3q19_last_error(d3q19_ctx* ctx);

/* Checkpoints (no counterpart in the reference, which writes text output
 * only): the whole device state of a context -- the distributions the next
 * step reads, u, the local tau, the sphere state and partial sums, the marker
 * records and tile lists of the last particle pass, the zone lists, the step
 * number and the clamp counter -- in one host buffer of
 * d3q19_checkpoint_bytes bytes.  d3q19_restore loads it into a context
 * created with the same parameter blocks and options; the steps after it are
 * bit-identical to those of the context it came from.  A context with a
 * device error, or left between passes by d3q19_k_*, is not checkpointed
 * (D3Q19_ENUMERIC / D3Q19_EOVERFLOW / D3Q19_ESTATE); a buffer of another
 * lattice, sphere count or option set is refused with D3Q19_EINVAL. */
int d3q19_checkpoint_bytes(d3q19_ctx* ctx, size_t* bytes);
int d3q19_checkpoint(d3q19_ctx* ctx, void* buf, size_t bytes);
int d3q19_restore(d3q19_ctx* ctx, const void* buf, size_t bytes);

/* Replaces clRelease* (sim_main.c:503-525). */
int d3q19_destroy(d3q19_ctx* ctx);

/* ---------------------------------------------------------------------------
 * The lattice pool: many independent shear cells resident on one GPU and
 * advanced together.  No counterpart in the reference (it runs one lattice
 * per process); the members are ordinary contexts (same layouts, same
 * read-backs through d3q19_pool_context) whose steps run in batched
 * persistent kernels over packed work lists -- one launch per kernel of the
 * step for all members, captured as CUDA graphs per chunk length.
 *
 * Members: periodic x and y with velocity walls on z, the fast arithmetic
 * with the reference's MRT, the pool's storage format and zone rebuild
 * period; each keeps its own viscosity law and parameters, lattice size,
 * spheres and markers.  A member's results do not depend on the other
 * members.
 * ------------------------------------------------------------------------- */
typedef struct d3q19_pool d3q19_pool;
/* Threads: every d3q19_pool_* call holds the pool's lock, so several host
 * threads may admit, release, read and advance the same pool (for example one
 * thread admitting arrivals while another drives the chunks).  A member's
 * context (d3q19_pool_context) is for read-backs between calls; it is not
 * stepped on its own.  d3q19_pool_last_error is per pool, not per thread. */

/* Device memory d3q19_create allocates for these parameters (read-back
 * scratch, allocated on first use, not included). */
int d3q19_context_bytes(const int_param_struct* ip, const d3q19_options* opt, size_t* bytes);
/* A pool on `device` for members with distribution storage `storage`
 * (d3q19_options.storage) and zone rebuild period rebuild_freq; at most
 * max_slots members whose d3q19_context_bytes sum to at most hbm_budget. */
int d3q19_pool_create(int device, int storage, int rebuild_freq, int max_slots, size_t hbm_budget,
                      d3q19_pool** out);
/* Admits one solve: creates its context from the parameter blocks and the
 * host arrays of d3q19_write_lattice / _particles / _zones (particle and zone
 * arrays may be NULL without spheres), runs its first period =
 * lcm(2, rebuild_freq) steps alone, and makes it a member (its slot in
 * *slot).  D3Q19_EBUSY when no slot is free or its memory would exceed the
 * budget now; D3Q19_EINVAL for a solve the pool cannot run. */
int d3q19_pool_admit(d3q19_pool* pool, const int_param_struct* ip, const flp_param_struct* fp,
                     const d3q19_options* opt, const float* f, const float* u, const float* tau_lb,
                     const float* parKin, const float* parForce, const float* parFluidForce,
                     const float* spherePoints, const int* zoneNeighDat, const int* parsZone,
                     const int* zoneMembers, const int* numParInZone, int* slot);
/* Advances every member by nsteps (a positive multiple of the period),
 * asynchronously on the pool's stream. */
int d3q19_pool_advance(d3q19_pool* pool, int nsteps);
/* The member's context, for its read-backs and diagnostics (ordered after the
 * pool's work); NULL for a free slot.  Do not step it directly. */
d3q19_ctx* d3q19_pool_context(d3q19_pool* pool, int slot);
/* Steps the member has taken, or -1 for a free slot. */
long long d3q19_pool_slot_steps(d3q19_pool* pool, int slot);
/* d3q19_mean_stress of every member in one pass on the pool's stream (one
 * read-back for all): arrays of max_slots entries; status[s] is 0, the
 * member's D3Q19_ENUMERIC / D3Q19_EOVERFLOW device error, or D3Q19_EINVAL
 * for a free slot (values NaN). */
int d3q19_pool_mean_stress(d3q19_pool* pool, double* stress_xz, double* shear_rate, double* eff_viscosity,
                           int* status);
/* Frees the member's slot and device memory.  Returns without waiting for
 * the pool's chunks already queued: the memory is freed in the pool stream's
 * order after them, and kept reserved for the next members. */
int d3q19_pool_release(d3q19_pool* pool, int slot);
/* Pre-emption: d3q19_pool_evict writes the member's checkpoint to buf
 * (d3q19_checkpoint_bytes of d3q19_pool_context(slot)) and releases the
 * slot; d3q19_pool_readmit creates a member from the same parameter blocks
 * and options and the checkpoint, and continues it from its step (no warm-up
 * steps) in the next advance.  Results equal those of a member that was
 * never evicted.  EBUSY as for d3q19_pool_admit. */
int d3q19_pool_evict(d3q19_pool* pool, int slot, void* buf, size_t bytes);
int d3q19_pool_readmit(d3q19_pool* pool, const int_param_struct* ip, const flp_param_struct* fp,
                       const d3q19_options* opt, const void* buf, size_t bytes, int* slot_out);
/* Budget in use, the budget, and the member count. */
int d3q19_pool_usage(d3q19_pool* pool, size_t* used, size_t* budget, int* members);
/* Grid sizes (CTAs) of the batched passes.  The fluid pass launches one CTA
 * per tile of the members (the tile count rounded up to m * 2^k, m in
 * [8, 15]); d3q19_pool_get_grid reports that grid, and d3q19_pool_set_grid
 * accepts and ignores a fluid_blocks >= 0.  The particle and contact passes
 * are persistent grids of the given sizes.  Results do not depend on them.
 * d3q19_pool_set_grid turns the autotuner off. */
int d3q19_pool_set_grid(d3q19_pool* pool, int fluid_blocks, int particle_blocks, int contact_blocks);
int d3q19_pool_get_grid(d3q19_pool* pool, int* fluid_blocks, int* particle_blocks, int* contact_blocks);
/* Grid autotuner (enable 1 on, 0 off; off when the pool is created).  With
 * it on, d3q19_pool_advance takes the particle and contact grids from a
 * process-wide table keyed by the device (name and SM count), the pool's
 * storage and layout, and the size class of its work (the bit length of its
 * fluid tile count).  While the class has untried candidates -- 1, 2 or 4
 * CTAs per SM for the particle and contact passes -- an
 * advance runs them in segments of 100 steps (rounded up to the period; an
 * advance shorter than two segments is one segment, timed when it has at
 * least 100 steps), one candidate per segment, each timed with events on the
 * pool's stream; the rest of the advance runs at the fastest grid timed so
 * far.  The next pool call collects the times, in ns per fluid tile step,
 * and once every candidate has been timed the fastest becomes the class's
 * choice, used by every later advance of that class on any pool of the
 * process.  Results do not depend on the grid, so the timed segments are
 * ordinary steps of the members. */
int d3q19_pool_autotune(d3q19_pool* pool, int enable);
/* The grid in use (CTAs per SM; fluid 0: one CTA per tile) and the tuner's
 * state for the pool's current work class: settled (0/1), candidates timed,
 * candidates in all.  Waits for a timed advance in flight. */
int d3q19_pool_tune_state(d3q19_pool* pool, int* fluid_per_sm, int* particle_per_sm, int* settled, int* tried,
                          int* total);
/* The candidates of the current class with their times (ns per fluid tile
 * step, negative when not yet timed): *n receives the candidate count; at
 * most cap entries are written to each non-null array. */
int d3q19_pool_tune_trials(d3q19_pool* pool, int* fluid_per_sm, int* particle_per_sm, double* ns_per_tile_step,
                           int cap, int* n);
/* The settled classes of the table as text, one line each, tab-separated:
 * device name, SMs, storage, inplace, class, fluid CTAs per SM (0: one CTA per
 * tile), particle CTAs per SM, ns per fluid tile step.  *len receives the text's length; the text
 * and its NUL are written when cap exceeds it (else ENOMEM, or 0 for cap 0). */
int d3q19_tune_export(char* buf, size_t cap, size_t* len);
/* Adds settled classes in d3q19_tune_export's format (a later line of the
 * same class replaces the earlier entry).  EINVAL, with nothing added, when
 * a line does not parse. */
int d3q19_tune_import(const char* text);
/* Empties the table. */
int d3q19_tune_clear(void);
/* Without waiting: 1 when the work of the last d3q19_pool_advance has
 * finished on the device (or none was queued), 0 while it runs, negative on
 * a CUDA error.  For callers that run their own event loop. */
int d3q19_pool_poll(d3q19_pool* pool);
/* Waits for the pool's work and reports the members' device errors. */
int d3q19_pool_synchronize(d3q19_pool* pool);
/* The pool's CUDA stream (cudaStream_t). */
void* d3q19_pool_stream(d3q19_pool* pool);
const char* d3q19_pool_last_error(d3q19_pool* pool);
int d3q19_pool_destroy(d3q19_pool* pool);

#ifdef __cplusplus
}
#endif
#endif
