// d3q19_internal.h -- types shared by the kernels (d3q19_kernels.cu) and the
// C-ABI layer (d3q19_api.cu).  Not part of the public interface.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace d3q19 {

// Fluid tile handled by one thread block of the collide-stream kernel: a run
// of 32 x-nodes (one warp) by TILE_Y rows by TILE_Z planes; the 256 threads
// (32 x 4 x 2) take TILE_Z/2 planes each.  The IBM force of a tile is
// accumulated over the tile plus a one-node halo.
// D3Q19_TILE_Y: a build knob for measuring other tile heights (2, 4, 8).
// Measured on B200 (collide-stream kernel ms; MLUPS of the batched pool):
// 128^3 suspension 0.1100 (4) / 0.1165 (2) / 0.1145 (8); the same fluid
// without spheres 0.0792 / 0.0777 / 0.0832; 64 batched boxes 16,704 /
// 14,575 / 16,390 MLUPS.  4 is kept: 2 wins only the sphere-free lattice,
// by 2 %.
#ifndef D3Q19_TILE_Y
#define D3Q19_TILE_Y 4
#endif
constexpr int TILE_X = 32;
constexpr int TILE_Y = D3Q19_TILE_Y;
constexpr int TILE_Z = 4;
constexpr int FLUID_THREADS = TILE_X * TILE_Y * 2;
constexpr int HALO_X = TILE_X + 2;
constexpr int HALO_Y = TILE_Y + 2;
constexpr int HALO_Z = TILE_Z + 2;
constexpr int HALO_N = HALO_X * HALO_Y * HALO_Z;
constexpr int TILE_N = TILE_X * TILE_Y * TILE_Z;

// The spread force is accumulated in fixed point (deterministic: integer sums
// do not depend on the order markers are visited in).  A contribution v,
// |v| < 2^FIX_BITS units of 2^-FIX_BITS times the largest marker force of the
// step, is split as v = hi * 2^16 + lo (0 <= lo < 2^16) and the two parts are
// summed with 32-bit atomics: exact for up to 2^(31 + 16 - FIX_BITS) = 256
// contributions of the largest size per node.
constexpr int FIX_BITS = 39;

// Device error word bits.
constexpr unsigned ERR_TILE_OVERFLOW = 1u;
constexpr unsigned ERR_NONFINITE = 2u;
constexpr unsigned ERR_ZONE_RANGE = 4u;
constexpr unsigned ERR_FIXED_RANGE = 8u;
constexpr unsigned ERR_BOUNDS = 16u;  // an index check of the bounds-checked build failed (access skipped)
constexpr unsigned ERR_TIMEOUT = 32u;  // a bounded device wait (a TMA load of the collide-stream pass) ran out

struct Geom {
  int Nx, Ny, Nz;
  long long NC;    // Nx*Ny*Nz
  int periodic[3]; // BoundaryConds == 0
  int wallAxis;    // axis with BoundaryConds == 1, or -1
  int tanBC[3];    // tangential velocity boundaries (only with a wall axis)
  int buffer[3];   // BufferSize
  int ntx, nty, ntz;  // fluid tiles per axis
};

struct FluidParams {
  float g[3];           // ConstBodyForce
  float tauN;           // NewtonianTau
  float velLower[3], velUpper[3];
  int viscModel;
  float visc[4];
  float tauMax;         // 0 = no upper clamp
  float tauMin;         // lower clamp (the reference's MIN_TAU = 0.505)
  float cassonReg;      // 0 = none
  int variable;         // local tau (read only by kernels that choose the law at run time)
  int periodicSmooth;   // the spread-force smoothing wraps across periodic x and y
};

// One IBM marker of the last particle pass, two float4 per marker:
//   a = {wx, wy, wz, bits(x0 | y0 << 16)}, b = {Fx, Fy, Fz, bits(z0)}
// (x0, y0, z0) is the corner cell of the marker's 2x2x2 stencil including
// the buffer offset, w* the reference's linear weights, F the marker force.
struct TileLists {
  int cap;
  int* count;          // [ntiles]
  int* list;           // [ntiles * cap] marker ids
  const float4* mrec;  // [2 * markers]
  unsigned* fmax;      // [2] float bits of the largest |marker force| per step parity
  long long markers;   // marker records in mrec (checked by the bounds-checked build)
};

struct FluidArgs {
  Geom g;
  FluidParams p;
  int t;  // time step (selects the marker-force maximum slot)
  // Distributions, 19 rows of N_C values (q-major): float, or with 16-bit
  // storage the shifted value f_q - w_q as IEEE half or bfloat16 bits.
  const void* fin;
  void* fout;
  float* u;
  float* tau;
  double* tau64;  // local tau of the FP64 build (tau holds its float copy)
  TileLists tiles;
  int has_ibm;
  unsigned* err;
  unsigned long long* clamps;
  // 0: two buffers.  In place (fin == fout): 1 = the next step is an even
  // step (cells read and written at the node), 2 = an odd step.
  int inplace;
};

struct ParticleParams {
  int np, P, L, nfa;        // spheres, markers per sphere, work-group size, groups per sphere
  float S[3];               // SystemSize as float
  int Sint[3];
  int buffer[3];
  float mass, inertia, pointArea, diam, zbuf;
  float g[3];
  float kcol;               // ParForceParams[0]
  int forceModel;           // ParForceModel
  int viscModel;
  float tauN;
  int numZones[3];
  float zoneWidth[3];
  int fixed;
  int exact;  // contact forces summed in the reference's order
  int periodicSmooth;  // list seam markers also in the tiles of their buffer-layer images
};

struct ParticleArgs {
  Geom g;
  ParticleParams p;
  // state at t-1 (read) and t (written)
  const float4* kin_old;
  float4* kin_new;
  const float4* pff_old;   // parFluidForce partials of step t-1
  float4* pff_new;
  const float4* pf_old;    // parForce of step t-1
  float4* pf_new;
  const float4* sphere;    // spherePoints [P]
  const float* u;
  float4* mrec;
  TileLists tiles;
  const int* znd;          // zoneNeighDat [28*Z]
  const int* parsZone;
  const int* zoneMembers;
  const int* numParInZone;
  const int* revStart;     // reverse zone-neighbour table (CSR)
  const int* revList;
  unsigned* err;
  int t;
  // particle_precision = 1: the sphere state and the force/torque partials in
  // double (layouts of kin and pff with double components).
  int p64;
  const double* kin64_old;
  double* kin64_new;
  const double* pff64_old;
  double* pff64_new;
};

struct ZoneArgs {
  ParticleParams p;
  const float4* kin;
  int* parsZone;
  int* zoneMembers;
  int* numParInZone;
  int* zoneOf;
  unsigned* err;
};

// Launchers (d3q19_kernels.cu).
// Storage of the distributions: 0 float, 1 half (f - w), 2 bfloat16 (f - w).
// STORE_F64 is internal: the FP64 build (d3q19_options.arithmetic = 2).
constexpr int STORE_F32 = 0, STORE_F16 = 1, STORE_BF16 = 2, STORE_F64 = 3;
inline int storage_bytes(int storage) { return storage == STORE_F32 ? 4 : (storage == STORE_F64 ? 8 : 2); }

cudaError_t launch_fluid(const FluidArgs& a, bool first, bool variable, int collision, int storage, cudaStream_t s);
// The TMA-pipelined collide-stream pass (d3q19_tma.cu): tensor maps of the
// distribution buffers (boxes of the tile width, and x-widened boxes for the
// pulls), made once per context.  tma_supported: the context's geometry and
// storage allow it (periodic x/y with z walls, FP32 / 16-bit storage,
// 16-byte aligned x rows).  buf: the buffer the step reads.
struct TmaMaps {
  alignas(64) unsigned char f[2][2][128];
  int ready = 0;
};
bool tma_supported(const Geom& g, int storage);
bool tma_make_maps(TmaMaps* m, void* const f[2], const Geom& g, int storage);
cudaError_t launch_fluid_tma(const TmaMaps& m, int buf, const FluidArgs& a, bool first, int storage, cudaStream_t s);
// Copies every population of the periodic x/y buffer-layer nodes of a.fin
// from their periodic images (the copies the TMA kernel's pulls read), for a
// buffer the TMA kernel did not write itself (a restored checkpoint).
cudaError_t launch_fill_ghosts(const FluidArgs& a, int storage, cudaStream_t s);
cudaError_t launch_materialize_f(const FluidArgs& a, int storage, float* out, cudaStream_t s);
// Conversions between float distributions and the stored form (n values,
// row q of each N_C-long row block shifted by w_q).
cudaError_t launch_store_f(const float* in, void* out, long long NC, int storage, cudaStream_t s);
cudaError_t launch_load_f(const void* in, float* out, long long NC, int storage, cudaStream_t s);
// out[k] = in[k] for n values (float to double).
cudaError_t launch_widen(const float* in, double* out, long long n, cudaStream_t s);
// The particle pass (rigid bodies, IBM interpolation and marker lists) and
// the particle-particle forces from the positions it wrote.
cudaError_t launch_particles(const ParticleArgs& a, cudaStream_t s);
cudaError_t launch_contacts(const ParticleArgs& a, cudaStream_t s);
cudaError_t launch_zones(const ZoneArgs& a, cudaStream_t s);
// Batched passes over many lattices (the lattice pool): persistent grids of
// `blocks` CTAs over packed work lists {slot, tile | group | sphere} whose
// lengths are read on the device; per-lattice arguments slots[2*s + parity].
// inplace: 0 two buffers, 1 / 2 the even / odd in-place step of every member.
cudaError_t launch_fluid_batch(const FluidArgs* slots, const int2* work, const int* nwork, int parity, int storage,
                               int inplace, int blocks, cudaStream_t s);
cudaError_t launch_particle_batch(const ParticleArgs* slots, const int2* work, const int* nwork, int parity,
                                  int threads, int blocks, cudaStream_t s);
cudaError_t launch_contact_batch(const ParticleArgs* slots, const int2* work, const int* nwork, int parity,
                                 int blocks, cudaStream_t s);
cudaError_t launch_zone_batch(const ZoneArgs* args, const int* slots, const int* nslots, int parity, int max_slots,
                              cudaStream_t s);
cudaError_t launch_spread_field(const Geom& g, const TileLists& t, int last_step, float* out, unsigned* err,
                                cudaStream_t s);
cudaError_t launch_marker_cells(const float4* mrec, int M, int* cells, cudaStream_t s);
// Per-plane FP64 sums of u, the shear rate du_x/dz + du_z/dx and the viscous
// shear stress: out[5 * Nz].
cudaError_t launch_plane_stats(const Geom& g, const float* u, const float* tau, float tauN, int variable,
                               double* out, cudaStream_t s);
// *out = the device error word (as a double), for batched status reads.
cudaError_t launch_copy_err(const unsigned* err, double* out, cudaStream_t s);
// Reference-exact variants (d3q19_exact.cu, compiled without contraction).
cudaError_t launch_fluid_exact(const FluidArgs& a, bool first, bool variable, int slots, cudaStream_t s);
cudaError_t launch_spread_field_exact(const Geom& g, const TileLists& t, int slots, float* out, unsigned* err,
                                      cudaStream_t s);

}  // namespace d3q19
