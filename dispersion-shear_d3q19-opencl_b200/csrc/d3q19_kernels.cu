// d3q19_kernels.cu -- sm_100a kernels of the D3Q19 LBM + IBM time step.
//
// Kernel map (reference kernel -> kernel here):
//   collideMRT_stream_D3Q19 (GPU_program.cl:316-624)
//   + boundary_periodic     (GPU_program.cl:626-735)
//   + boundary_velocity     (GPU_program.cl:737-865)
//   + reset/sum_particle_fluid_forces and the 27-point force smoothing
//                           (GPU_program.cl:258-313, 356-377)
//       -> fluid_step_kernel: one pass per node.  The reference pushes
//          post-collision populations to the neighbours and then repairs the
//          boundary layer with two more kernels.  Here each node pulls its
//          populations from the neighbours' post-collision values, wrapping
//          periodic axes and rebuilding the wall unknowns in registers, which
//          yields exactly the reference's post-boundary state, then collides
//          and stores its own post-collision values (aligned stores).  The
//          IBM force of the previous step is accumulated per tile in shared
//          memory from the markers listed for that tile (integer fixed-point
//          sums: deterministic) and smoothed with the reference's 27-point
//          stencil, so no dense force field ever touches HBM.
//   particle_dynamics (CPU_program.cl:187-277)
//   + particle_fluid_forces_linear_stencil (GPU_program.cl:81-256)
//   + particle_particle_forces (CPU_program.cl:76-184)
//       -> particle_step_kernel: one block per reference work-group of
//          markers; each block advances its sphere (rigid-body update from
//          the forces of step t-1), interpolates u(t) at its markers,
//          reduces force and torque over the work-group in the reference's
//          tree order, writes the marker records and lists each marker in
//          the fluid tiles its stencil touches (bucket sort by tile).  Extra
//          blocks compute the particle-particle forces, one thread per
//          sphere, from the same updated positions.
//   update_particle_zones (CPU_program.cl:280-315) -> zone_rebuild_kernel.
#include "d3q19_device.cuh"

namespace d3q19 {


// Resident blocks per SM the register allocation is sized for (256 threads
// each).  FP32 storage: 5 (48 registers), 16-bit storage: 4 (64 registers),
// the faster choices measured on the 128^3 suspension.
#ifndef FLUID_MIN_BLOCKS_F32
#define FLUID_MIN_BLOCKS_F32 5
#endif
#ifndef FLUID_MIN_BLOCKS
#define FLUID_MIN_BLOCKS 4
#endif

// One collide-stream pass over a 32x4x4 tile; each thread takes two
// consecutive z-planes.  first != 0: the stored state is the reference's
// post-stream buffer (after an upload), read in place without streaming.
// AA: 0 = two buffers (pull from fin, write fout); 1 and 2 = the even and
// odd steps of the in-place layout (fin == fout).  Even: read the node's own
// cells, write them back with the directions reversed.  Odd: pull the
// reversed cells of the upwind neighbours, push to the downwind ones.
// Every cell is read and then written by one thread only.
template <int COLL, int VISC, int BC, typename ST, int AA = 0>
__device__ __forceinline__ void fluid_tile(const FluidArgs& a, const int first, const int bx, const int by,
                                           const int bz, SpreadSmem& sm) {
  const ST* __restrict__ fin = static_cast<const ST*>(a.fin);
  ST* __restrict__ fout = static_cast<ST*>(a.fout);
  const Geom& g = a.g;
  const int tid = threadIdx.x + TILE_X * (threadIdx.y + TILE_Y * threadIdx.z);
  const int X0 = bx * TILE_X, Y0 = by * TILE_Y, Z0 = bz * TILE_Z;
  const int T = bx + g.ntx * (by + g.nty * bz);
  constexpr bool kRuntimeVisc = VISC < 0;
  const bool var = VISC > 0 || (kRuntimeVisc && a.p.variable);
  const int x = X0 + threadIdx.x;
  const int y = Y0 + threadIdx.y;
  const long long NC = g.NC;
  const bool inxy = x >= 1 && x <= g.Nx - 2 && y >= 1 && y <= g.Ny - 2;
  using R = typename RealOf<ST>::type;
  constexpr bool k64 = sizeof(R) == 8;

  // IBM force of the tile: the markers listed by the particle pass of step
  // t-1, accumulated over the tile's halo and smoothed with the reference's
  // 27-point stencil (GPU_program.cl:356-377), in shared memory only.
  R sg[2][3] = {{R(0), R(0), R(0)}, {R(0), R(0), R(0)}};
  if (a.has_ibm) {
    const int cnt = a.tiles.count[T];
    const int first_id = tid < a.tiles.cap ? a.tiles.list[(long long)T * a.tiles.cap + tid] : 0;  // speculative
    const unsigned fbits = a.tiles.fmax[(a.t + 1) & 1];
    __syncthreads();  // every thread has read the count
    // Consumed: the particle pass of this step refills the list and records
    // its force maximum in the other slot, cleared here.
    if (tid == 0) {
      a.tiles.count[T] = 0;
      if (T == 0) a.tiles.fmax[a.t & 1] = 0u;
    }
    if (cnt > 0) {
      accumulate_tile<R>(sm, g, a.tiles, T, min(cnt, a.tiles.cap), X0, Y0, Z0, tid, fixed_exponent(fbits), first_id,
                         a.err, a.p.periodicSmooth != 0);
      smooth_pair(sm, threadIdx.x, threadIdx.y, threadIdx.z, sg);
    }
  }

  int nclamp = 0;
#ifndef FLUID_ZZ_UNROLL
#define FLUID_ZZ_UNROLL 1
#endif
  constexpr int kZZUnroll = FLUID_ZZ_UNROLL;
#pragma unroll kZZUnroll
  for (int zz = 0; zz < 2; zz++) {
    const int z = Z0 + 2 * threadIdx.z + zz;
    if (!inxy || z < 1 || z > g.Nz - 2) continue;
    const int i = x + g.Nx * (y + g.Ny * z);
    if (out_of_bounds(i, NC, a.err)) continue;
    R f[19];
    if (AA == 0) {
      if (first) {
#pragma unroll
        for (int q = 0; q < 19; q++) f[q] = Stored<ST>::load(fin + q * NC + i, wq<R>(q));
      } else if (BC == BC_ZWALL) {
        const int Nxy = g.Nx * g.Ny;
        const int dxm0 = x == 1 ? g.Nx - 3 : -1;
        const int dxp0 = x == g.Nx - 2 ? -(g.Nx - 3) : 1;
        const int dym0 = (y == 1 ? g.Ny - 3 : -1) * g.Nx;
        const int dyp0 = (y == g.Ny - 2 ? -(g.Ny - 3) : 1) * g.Nx;
        gather(f, fin, NC, i, dxm0, dxp0, dym0, dyp0, -Nxy, Nxy, a.err);
        if (z == 1) velocity_bc<2, 0>(f, a.p.velLower);
        else if (z == g.Nz - 2) velocity_bc<2, 1>(f, a.p.velUpper);
      } else {
        int dxm0, dxp0, dym0, dyp0, dzm0, dzp0;
        neighbour_deltas(g, x, y, z, dxm0, dxp0, dym0, dyp0, dzm0, dzp0);
        gather(f, fin, NC, i, dxm0, dxp0, dym0, dyp0, dzm0, dzp0, a.err);
        boundaries(f, g, a.p, x, y, z);
      }
    } else {
      if (first || AA == 1) {
#pragma unroll
        for (int q = 0; q < 19; q++) f[q] = Stored<ST>::load(fin + q * NC + i, wq<R>(q));
      } else {
        int dxm, dxp, dym, dyp, dzm, dzp;
        layout_deltas<BC>(g, x, y, z, dxm, dxp, dym, dyp, dzm, dzp);
        gather_reversed(f, fin, NC, i, dxm, dxp, dym, dyp, dzm, dzp, a.err);
      }
      // The uploaded state is the reference's buffer after its boundary
      // kernels; every later step rebuilds the wall unknowns.
      if (!first) {
        if (BC == BC_ZWALL) {
          if (z == 1) velocity_bc<2, 0>(f, a.p.velLower);
          else if (z == g.Nz - 2) velocity_bc<2, 1>(f, a.p.velUpper);
        } else {
          boundaries(f, g, a.p, x, y, z);
        }
      }
    }
    const R gx = R(a.p.g[0]) + (zz ? sg[1][0] : sg[0][0]);
    const R gy = R(a.p.g[1]) + (zz ? sg[1][1] : sg[0][1]);
    const R gz = R(a.p.g[2]) + (zz ? sg[1][2] : sg[0][2]);
    R rho = R(0);
#pragma unroll
    for (int q = 0; q < 19; q++) rho += f[q];
    const R jx = f[1] - f[2] + f[7] + f[8] + f[9] + f[10] - f[11] - f[12] - f[13] - f[14];
    const R jy = f[3] - f[4] + f[7] - f[8] + f[11] - f[12] + f[15] + f[16] - f[17] - f[18];
    const R jz = f[5] - f[6] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16] + f[17] - f[18];
    const R ir = RMath<R>::rcp(rho);
    const R ux = (jx + R(0.5f) * gx) * ir, uy = (jy + R(0.5f) * gy) * ir, uz = (jz + R(0.5f) * gz) * ir;
    // Plain stores (also in place): the particle pass reads u right after,
    // from L2.
    a.u[i] = (float)ux;
    a.u[i + NC] = (float)uy;
    a.u[i + 2 * NC] = (float)uz;
    // A non-finite population makes rho non-finite; a vanishing or negative
    // density is flagged too.
    if (!(rho > R(0) && rho < R(1e30f))) atomicOr(a.err, ERR_NONFINITE);
    // The FP64 build keeps tau in double (tau64) and a float copy for
    // read-back.
    R tau = var ? (k64 ? R(a.tau64[i]) : R(a.tau[i])) : R(a.p.tauN);
    bool clamped = false;
    collide<COLL, VISC, R>(f, rho, ir, ux, uy, uz, gx, gy, gz, tau, a.p, clamped);
    if (var) {
      if (k64) a.tau64[i] = (double)tau;
      a.tau[i] = (float)tau;
      nclamp += clamped ? 1 : 0;
    }
    if (AA == 1) {
#pragma unroll
      for (int q = 0; q < 19; q++) Stored<ST>::store_stream(fout + OPPQ(q) * NC + i, f[q], wq<R>(q));
    } else if (AA == 2) {
      // Recomputed here rather than kept live across the collision.
      int dxm, dxp, dym, dyp, dzm, dzp;
      layout_deltas<BC>(g, x, y, z, dxm, dxp, dym, dyp, dzm, dzp);
#pragma unroll
      for (int q = 0; q < 19; q++) {
        const int cx = CXQ(q), cy = CYQ(q), cz = CZQ(q);
        const int dst = i + (cx == 1 ? dxp : (cx == -1 ? dxm : 0)) + (cy == 1 ? dyp : (cy == -1 ? dym : 0)) +
                        (cz == 1 ? dzp : (cz == -1 ? dzm : 0));
        if (out_of_bounds(dst, NC, a.err)) continue;
        Stored<ST>::store_stream(fout + q * NC + dst, f[q], wq<R>(q));
      }
    } else {
#pragma unroll
      for (int q = 0; q < 19; q++) Stored<ST>::store(fout + q * NC + i, f[q], wq<R>(q));
    }
  }
  if (var && nclamp) atomicAdd(a.clamps, (unsigned long long)nclamp);
}

// The in-place variants with FP32 storage: 4 blocks/SM (64 registers, no
// spills) measured faster than 5 with and without spheres.
#ifndef FLUID_MIN_BLOCKS_AA_F32
#define FLUID_MIN_BLOCKS_AA_F32 4
#endif
template <int COLL, int VISC, int BC, typename ST, int AA>
__global__ void __launch_bounds__(FLUID_THREADS, sizeof(ST) == 4   ? (AA ? FLUID_MIN_BLOCKS_AA_F32 : FLUID_MIN_BLOCKS_F32)
                                                 : sizeof(ST) == 8 ? 2
                                                                   : FLUID_MIN_BLOCKS)
    fluid_step_kernel(const FluidArgs a, const int first) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // Everything here reads or writes data of the passes before it: the tile
  // lists, the distributions, and u, which the previous particle pass reads.
  pdl_wait();
  pdl_trigger();
  fluid_tile<COLL, VISC, BC, ST, AA>(a, first, blockIdx.x, blockIdx.y, blockIdx.z,
                                     *reinterpret_cast<SpreadSmem*>(smem_raw));
}

// The collide-stream pass of many independent lattices in one launch: CTA b
// takes work item b of the packed list work[k] = {slot, tile} (*nwork items;
// the grid is at least that long, the CTAs past it return at once).  One CTA
// per tile lets the hardware schedule the tiles: measured on B200, a served
// mix of 48 members ran 9,320 MLUPS against 8,296 with a persistent grid of 4
// CTAs per SM looping over the items, one 150^3 member 6,720 against 6,465.  slots[2*s + parity] holds lattice
// s's arguments for steps of that buffer parity.  The reference's MRT rates,
// periodic x/y with z walls, and each lattice's own viscosity law.
// AA: the pool's layout for this step (every member of a pool shares it and
// sits at the same phase).
// The item's arguments are copied into shared memory first: read from there,
// they need no registers across the tile (read from global memory, the
// compiler held many of them in registers and spilled).  Measured on B200:
// 64 batched boxes 17,500 against 16,710 MLUPS; one 150^3 member 6,440
// against 5,920 MLUPS.
template <typename ST, int AA>
__global__ void __launch_bounds__(FLUID_THREADS, sizeof(ST) == 4 ? (AA ? FLUID_MIN_BLOCKS_AA_F32 : FLUID_MIN_BLOCKS_F32)
                                                                 : FLUID_MIN_BLOCKS)
    fluid_batch_kernel(const FluidArgs* __restrict__ slots, const int2* __restrict__ work,
                       const int* __restrict__ nwork, const int parity) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SpreadSmem& sm = *reinterpret_cast<SpreadSmem*>(smem_raw);
  const int n = *nwork;
  {
    const int w = blockIdx.x;
    if (w >= n) return;
    const int2 it = work[w];
    __shared__ FluidArgs sa;
    {
      static_assert(sizeof(FluidArgs) % 4 == 0, "FluidArgs is copied in 32-bit words");
      const int* src = reinterpret_cast<const int*>(&slots[2 * it.x + parity]);
      int* dst = reinterpret_cast<int*>(&sa);
      const int tid = threadIdx.x + TILE_X * (threadIdx.y + TILE_Y * threadIdx.z);
      for (int k = tid; k < (int)(sizeof(FluidArgs) / 4); k += FLUID_THREADS) dst[k] = src[k];
      __syncthreads();
    }
    const FluidArgs& a = sa;
    const int ntx = a.g.ntx, nty = a.g.nty;
    const int bx = it.y % ntx, by = (it.y / ntx) % nty, bz = it.y / (ntx * nty);
    fluid_tile<0, -1, BC_ZWALL, ST, AA>(a, 0, bx, by, bz, sm);
  }
}

// Post-streaming, post-boundary populations of the last step (what the
// reference's f_s holds after its boundary kernels), for read-back.
template <typename ST>
__global__ void materialize_f_kernel(const FluidArgs a, float* __restrict__ out) {
  const Geom& g = a.g;
  const long long NC = g.NC;
  const long long n = (long long)(g.Nx - 2) * (g.Ny - 2) * (g.Nz - 2);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int x = 1 + (int)(k % (g.Nx - 2));
    const int y = 1 + (int)((k / (g.Nx - 2)) % (g.Ny - 2));
    const int z = 1 + (int)(k / ((long long)(g.Nx - 2) * (g.Ny - 2)));
    const int i = x + g.Nx * (y + g.Ny * z);
    int dxm, dxp, dym, dyp, dzm, dzp;
    neighbour_deltas(g, x, y, z, dxm, dxp, dym, dyp, dzm, dzp);
    typename RealOf<ST>::type f[19];
    const ST* fin = static_cast<const ST*>(a.fin);
    // The next step's inputs: in place after an odd in-place step (the
    // neighbours pushed them), reversed in the upwind cells after an even
    // one, pulled from the other buffer otherwise.
    if (a.inplace == 1) {
#pragma unroll
      for (int q = 0; q < 19; q++) f[q] = Stored<ST>::load(fin + q * NC + i, wq<typename RealOf<ST>::type>(q));
    } else if (a.inplace == 2) {
      gather_reversed(f, fin, NC, i, dxm, dxp, dym, dyp, dzm, dzp, a.err);
    } else {
      gather(f, fin, NC, i, dxm, dxp, dym, dyp, dzm, dzp, a.err);
    }
    boundaries(f, g, a.p, x, y, z);
#pragma unroll
    for (int q = 0; q < 19; q++) out[q * NC + i] = (float)f[q];
  }
}

// Dense spread-force field (the reference's gpf slot 0) from the tile lists,
// for parity read-back.  One block per tile; does not consume the lists.
__global__ void __launch_bounds__(FLUID_THREADS) spread_field_kernel(const Geom g, const TileLists tl, int last_step,
                                                           float* __restrict__ out, unsigned* err) {
  __shared__ SpreadSmem sm;
  const int tid = threadIdx.x;
  const long long T = blockIdx.x + (long long)g.ntx * (blockIdx.y + (long long)g.nty * blockIdx.z);
  const int X0 = blockIdx.x * TILE_X, Y0 = blockIdx.y * TILE_Y, Z0 = blockIdx.z * TILE_Z;
  const int cnt = tl.count[T];
  if (cnt <= 0) return;
  const int first_id = tid < min(cnt, tl.cap) ? tl.list[T * tl.cap + tid] : 0;
  accumulate_tile(sm, g, tl, T, min(cnt, tl.cap), X0, Y0, Z0, tid, fixed_exponent(tl.fmax[last_step & 1]), first_id,
                  err);
  for (int k = tid; k < TILE_X * TILE_Y * TILE_Z; k += blockDim.x) {
    const int x = X0 + k % TILE_X, y = Y0 + (k / TILE_X) % TILE_Y, z = Z0 + k / (TILE_X * TILE_Y);
    if (x < 1 || x > g.Nx - 2 || y < 1 || y > g.Ny - 2 || z < 1 || z > g.Nz - 2) continue;
    const long long i = x + (long long)g.Nx * (y + (long long)g.Ny * z);
    const int h = (x - X0 + 1) + HALO_X * ((y - Y0 + 1) + HALO_Y * (z - Z0 + 1));
    out[i] = sm.g[0][h];
    out[i + g.NC] = sm.g[1][h];
    out[i + 2 * g.NC] = sm.g[2][h];
  }
}

// ---------------------------------------------------------------------------
// Particles.  Float arithmetic of the rigid-body update and the marker
// placement uses explicitly rounded operations (no contraction) so that the
// same update evaluated in different blocks is bit-identical and follows the
// reference's IEEE evaluation order.
__device__ __forceinline__ float4 f4add(float4 a, float4 b) {
  return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z), __fadd_rn(a.w, b.w));
}
__device__ __forceinline__ float4 f4sub(float4 a, float4 b) {
  return make_float4(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z), __fsub_rn(a.w, b.w));
}
__device__ __forceinline__ float4 f4mul(float4 a, float s) {
  return make_float4(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s), __fmul_rn(a.w, s));
}
__device__ __forceinline__ float4 f4div(float4 a, float s) {
  return make_float4(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s), __fdiv_rn(a.w, s));
}
__device__ __forceinline__ float4 f4cross(float4 a, float4 b) {
  return make_float4(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
                     __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
                     __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)), 0.0f);
}

struct Kin {
  float4 x, v, q, w;
};

__device__ __forceinline__ Kin load_kin(const float4* __restrict__ kin, int p, int np) {
  Kin k;
  k.x = kin[p];
  k.v = kin[p + np];
  k.q = kin[p + 2 * np];
  k.w = kin[p + 3 * np];
  return k;
}

// fmodf(a, w) for w > 0: a itself for 0 <= a < w, a - w (exact: Sterbenz)
// for w <= a < 2w, the library function otherwise.  Bit-identical to fmodf.
__device__ __forceinline__ float wrap_mod(float a, float w) {
  if (a >= 0.0f && a < w) return a;
  if (a >= w && a < 2.0f * w) return __fsub_rn(a, w);
  return fmodf(a, w);
}

// particle_dynamics for one sphere (CPU_program.cl:209-276).
__device__ Kin rigid_update(const ParticleArgs& a, int p) {
  const ParticleParams& P = a.p;
  const int np = P.np, nfa = P.nfa;
  Kin k;
  k.x = a.kin_old[p];
  k.v = a.kin_old[p + np];
  k.q = a.kin_old[p + 2 * np];
  k.w = a.kin_old[p + 3 * np];
  if (P.fixed) return k;
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f), aacc = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int fa = 0; fa < nfa; fa++) {
    acc = f4add(acc, a.pff_old[p * nfa + fa]);
    aacc = f4add(aacc, a.pff_old[(p + np) * nfa + fa]);
  }
  acc = f4add(acc, a.pf_old[p]);
  aacc = f4add(aacc, a.pf_old[p + np]);
  acc = f4div(acc, P.mass);
  aacc = f4div(aacc, P.inertia);
  acc.x = __fadd_rn(acc.x, P.g[0]);
  acc.y = __fadd_rn(acc.y, P.g[1]);
  acc.z = __fadd_rn(acc.z, P.g[2]);
  const float4 W = make_float4(P.S[0], P.S[1], P.S[2], 1.0f);
  const float4 rt = f4add(f4add(k.x, k.v), f4mul(acc, 0.5f));
  const float4 rw = f4add(rt, W);
  Kin o;
  o.x = make_float4(wrap_mod(rw.x, W.x), wrap_mod(rw.y, W.y), wrap_mod(rw.z, W.z), wrap_mod(rw.w, W.w));
  o.v = f4add(k.v, acc);
  const float dqw = -__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(k.w.x, k.q.x), __fmul_rn(k.w.y, k.q.y)),
                                         __fmul_rn(k.w.z, k.q.z)),
                               __fmul_rn(k.w.w, k.q.w));
  const float4 dq = f4add(f4mul(k.w, k.q.w), f4cross(k.w, k.q));
  o.q = f4mul(dq, 0.5f);
  o.q.w = __fadd_rn(o.q.w, __fmul_rn(0.5f, dqw));
  o.w = f4add(k.w, aacc);
  return o;
}

// Tile indices along one axis whose halo contains node coordinate c.
__device__ __forceinline__ void tile_range(int c, int T, int nt, int& lo, int& hi) {
  lo = (c + T - 1) / T - 1;
  if (lo < 0) lo = 0;
  hi = (c + 1) / T;
  if (hi > nt - 1) hi = nt - 1;
}

// Distinct tile indices covering two node coordinates (at most 4).  With
// wrap (periodic smoothing of the spread force on a periodic axis of N
// nodes), also the tiles holding the buffer-layer images of stencil nodes on
// the seam, which those tiles' smoothing reads.
__device__ __forceinline__ void tile_add(int c, int T, int nt, int (&out)[4], int& n) {
  int lo, hi;
  tile_range(c, T, nt, lo, hi);
  for (int t = lo; t <= hi && n < 4; t++) {
    bool dup = false;
    for (int j = 0; j < n; j++) dup |= out[j] == t;
    if (!dup) out[n++] = t;
  }
}
__device__ __forceinline__ int tile_set(int c0, int c1, int T, int nt, int (&out)[4], int N = 0, bool wrap = false) {
  int l0, h0, l1, h1, n = 0;
  tile_range(c0, T, nt, l0, h0);
  tile_range(c1, T, nt, l1, h1);
  for (int t = l0; t <= h0 && n < 4; t++) out[n++] = t;
  for (int t = l1; t <= h1 && n < 4; t++) {
    bool dup = false;
    for (int j = 0; j < n; j++) dup |= out[j] == t;
    if (!dup) out[n++] = t;
  }
  if (wrap) {
    const int i0 = seam_image(c0, N, true), i1 = seam_image(c1, N, true);
    if (i0 >= 0) tile_add(i0, T, nt, out, n);
    if (i1 >= 0) tile_add(i1, T, nt, out, n);
  }
  return n;
}

// Pair force of the reference's contact loop (CPU_program.cl:118-169) for
// the pair (A, B), A the higher sphere index: unit vector e (A to B, nearest
// periodic image in x, y and z) and the total magnitude along e (harmonic
// overlap + Newtonian squeeze film; the two exclude each other).
__device__ bool pair_force(const ParticleParams& P, const Kin& A, const Kin& B, float4& e, float& fmag) {
  const float rp = P.diam / 2.0f;
  float4 rij = f4sub(B.x, A.x);
  float* r = &rij.x;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const int sg = (r[d] < 0.0f) ? -1 : (r[d] > 0.0f);
    r[d] = (fabsf(r[d]) < P.S[d] / 2.0f) ? r[d] : __fsub_rn(r[d], __fmul_rn((float)sg, P.S[d]));
  }
  const float rSep = sqrtf(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(rij.x, rij.x), __fmul_rn(rij.y, rij.y)),
                                               __fmul_rn(rij.z, rij.z)),
                                     __fmul_rn(rij.w, rij.w)));
  const float4 vij = f4sub(B.v, A.v);
  const float minSep = __fsub_rn(rSep, 2.0f * rp);
  e = f4div(rij, rSep);
  const float vRel = -__fadd_rn(__fadd_rn(__fmul_rn(e.x, vij.x), __fmul_rn(e.y, vij.y)), __fmul_rn(e.z, vij.z));
  fmag = 0.0f;
  bool any = false;
  const float overlap = -minSep;
  if (overlap > 0 && P.forceModel == 1) {
    fmag = __fmul_rn(P.kcol, overlap);
    any = true;
  }
  if (minSep > 0 && (double)minSep < 0.1 * (double)rp) {
    float sq = 0.0f;
    if (P.viscModel == 1) {  // compute_squeeze_force, CPU_program.cl:319-343
      const float rStar = rp / 2.0f;
      const float ms = minSep < 0.1f ? 0.1f : minSep;
      const double eta0 = (double)((P.tauN - 0.5f) / 3.0f);
      sq = (float)(6.0 * 3.14159265358979323846 * eta0 * rStar * rStar * vRel / ms);
    }
    fmag = any ? __fadd_rn(fmag, sq) : sq;
    any = true;
  }
  return any;
}

// Lists marker gid in every fluid tile whose halo holds one of its stencil
// nodes (up to 2 tiles per axis, 3 where the stencil wraps a periodic edge
// of a lattice whose N-2 is a multiple of the tile size); lanes inserting
// into the same tile share one atomic.  Up to 8 atomics of the warp are
// issued before any result is used, so their round trips overlap.  All 32
// lanes of the warp call it (n = 0 for lanes without a marker).
__device__ __forceinline__ void insert_marker(const ParticleArgs& a, long long gid, int lane, const int (&tx)[4],
                                              const int (&ty)[4], const int (&tz)[4], int nx, int ny, int nz) {
  const Geom& g = a.g;
  const int n = nx * ny * nz;
  int nmax = n;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
  // Entry j of the marker's tile product, j = ia + nx*(ib + ny*ic), advanced
  // incrementally (no divisions).
  int ia = 0, ib = 0, ic = 0;
  for (int j0 = 0; j0 < nmax; j0 += 8) {
    int tileOf[8], baseOf[8];
    unsigned peersOf[8];
#pragma unroll
    for (int jj = 0; jj < 8; jj++) {
      const int j = j0 + jj;
      tileOf[jj] = -1;
      baseOf[jj] = 0;
      peersOf[jj] = 0u;
      if (j >= nmax) continue;
      const bool act = j < n;
      const unsigned amask = __ballot_sync(0xffffffffu, act);
      if (act) {
        const int T = tx[ia] + g.ntx * (ty[ib] + g.nty * tz[ic]);
        const unsigned peers = __match_any_sync(amask, T);
        tileOf[jj] = T;
        peersOf[jj] = peers;
        if (lane == __ffs(peers) - 1) baseOf[jj] = atomicAdd(&a.tiles.count[T], __popc(peers));
        if (++ia == nx) {
          ia = 0;
          if (++ib == ny) {
            ib = 0;
            ++ic;
          }
        }
      }
    }
#pragma unroll
    for (int jj = 0; jj < 8; jj++) {
      if (j0 + jj >= nmax) continue;
      const int base = __shfl_sync(0xffffffffu, baseOf[jj], peersOf[jj] ? __ffs(peersOf[jj]) - 1 : lane);
      if (tileOf[jj] >= 0) {
        const int slot = base + __popc(peersOf[jj] & ((1u << lane) - 1u));
        if (slot < a.tiles.cap) a.tiles.list[(long long)tileOf[jj] * a.tiles.cap + slot] = (int)gid;
        else atomicOr(a.err, ERR_TILE_OVERFLOW);
      }
    }
  }
}

// Largest force component of the step (the fixed-point unit of the spread):
// warp maximum, then one atomic per warp.  All 32 lanes call it.
__device__ __forceinline__ void record_fmax(const ParticleArgs& a, float fx, float fy, float fz, int lane) {
  float fm = fmaxf(fabsf(fx), fmaxf(fabsf(fy), fabsf(fz)));
  if (!(fm == fm)) fm = 3.0e38f;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) fm = fmaxf(fm, __shfl_xor_sync(0xffffffffu, fm, o));
  if (lane == 0 && fm > 0.0f) atomicMax(&a.tiles.fmax[a.t & 1], __float_as_uint(fm));
}

// One reference work-group of markers (group grp of np*nfa) per block:
// red holds 2*blockDim.x float4 (forces, then torques), s_kin the sphere's
// updated state.
__device__ __forceinline__ void particle_group(const ParticleArgs& a, const int grp, float4* red, Kin& s_kin) {
  const ParticleParams& P = a.p;
  const Geom& g = a.g;
  const int np = P.np, nfa = P.nfa, L = P.L;
  const int ngroups = np * nfa;
  const int l = threadIdx.x;
  const int lane = l & 31;
  {
    const int p = grp / nfa;
    const int wg = grp - p * nfa;  // work-group of the sphere
    // The rigid-body update of the sphere, once per block and shared.
    const float4 r0 = l < L ? a.sphere[wg * L + l] : make_float4(0.f, 0.f, 0.f, 0.f);
    // The marker template above is constant.  Everything after the wait reads
    // the previous collide-stream pass's u and lists.  The contact forces of
    // the side stream's pass, which the rigid-body update reads, are ordered
    // by the host's stream wait on that pass's event before this launch, not
    // by this wait (which orders only the preceding kernel of this stream).
    pdl_wait();
    pdl_trigger();
    if (l == 0) {
      const Kin kn = rigid_update(a, p);
      s_kin = kn;
      if (wg == 0) {
        a.kin_new[p] = kn.x;
        a.kin_new[p + np] = kn.v;
        a.kin_new[p + 2 * np] = kn.q;
        a.kin_new[p + 3 * np] = kn.w;
      }
    }
    __syncthreads();
    const Kin k = s_kin;
    float4 force = make_float4(0.f, 0.f, 0.f, 0.f), torque = force;
    int tx[4], ty[4], tz[4], nx = 0, ny = 0, nz = 0;
    const long long gid = (long long)grp * L + l;
    if (l < L) {
      const float4 W = make_float4(P.S[0], P.S[1], P.S[2], 1.0f);
      const float4 rw = f4add(f4add(k.x, r0), W);
      const float4 rpp = make_float4(wrap_mod(rw.x, W.x), wrap_mod(rw.y, W.y), wrap_mod(rw.z, W.z), wrap_mod(rw.w, W.w));
      const float fx = floorf(rpp.x), fy = floorf(rpp.y), fz = floorf(rpp.z);
      const int x0 = (int)fx + P.buffer[0], y0 = (int)fy + P.buffer[1], z0 = (int)fz + P.buffer[2];
      const bool ok = fx == fx && fy == fy && fz == fz && x0 >= 1 && x0 <= g.Nx - 2 && y0 >= 1 &&
                      y0 <= g.Ny - 2 && z0 >= 1 && z0 <= g.Nz - 2;
      if (!ok) {
        atomicOr(a.err, ERR_NONFINITE);
      } else {
        const int xs = (x0 == g.Nx - 2) ? -(g.Nx - 3) : 1;
        const int ys = (y0 == g.Ny - 2) ? -(g.Ny - 3) : 1;
        const int zs = (z0 == g.Nz - 2) ? -(g.Nz - 3) : 1;
        const float wx = __fsub_rn(1.0f, __fsub_rn(rpp.x, fx));
        const float wy = __fsub_rn(1.0f, __fsub_rn(rpp.y, fy));
        const float wz = __fsub_rn(1.0f, __fsub_rn(rpp.z, fz));
        float w[8];
        marker_weights(wx, wy, wz, w);
        const int sh[8][3] = {{0, 0, 0}, {xs, 0, 0}, {0, ys, 0}, {0, 0, zs}, {xs, ys, 0}, {xs, 0, zs},
                              {0, ys, zs}, {xs, ys, zs}};
        float ux = 0.f, uy = 0.f, uz = 0.f;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const long long i =
              (x0 + sh[j][0]) + (long long)g.Nx * ((y0 + sh[j][1]) + (long long)g.Ny * (z0 + sh[j][2]));
          if (out_of_bounds(i, g.NC, a.err)) continue;
          // GPU_program.cl:193-195, without contraction.
          ux = __fadd_rn(ux, __fmul_rn(w[j], a.u[i]));
          uy = __fadd_rn(uy, __fmul_rn(w[j], a.u[i + g.NC]));
          uz = __fadd_rn(uz, __fmul_rn(w[j], a.u[i + 2 * g.NC]));
        }
        const float4 upp = make_float4(ux, uy, uz, 0.0f);
        const float4 vpp = f4add(k.v, f4cross(k.w, r0));
        force = f4mul(f4sub(upp, vpp), P.pointArea);
        torque = f4cross(r0, force);
        a.mrec[2 * gid] = make_float4(wx, wy, wz, __uint_as_float((unsigned)x0 | ((unsigned)y0 << 16)));
        a.mrec[2 * gid + 1] = make_float4(force.x, force.y, force.z, __uint_as_float((unsigned)z0));
        nx = tile_set(x0, x0 + xs, TILE_X, g.ntx, tx, g.Nx, P.periodicSmooth && g.periodic[0]);
        ny = tile_set(y0, y0 + ys, TILE_Y, g.nty, ty, g.Ny, P.periodicSmooth && g.periodic[1]);
        nz = tile_set(z0, z0 + zs, TILE_Z, g.ntz, tz);
      }
    }
    // List the marker in every fluid tile whose halo holds one of its
    // stencil nodes; record the step's largest force component.
    insert_marker(a, gid, lane, tx, ty, tz, nx, ny, nz);
    record_fmax(a, force.x, force.y, force.z, lane);
    // Work-group reduction in the reference's tree order
    // (GPU_program.cl:232-255).
    const int B = blockDim.x;
    red[l] = force;
    red[l + B] = torque;
    __syncthreads();
    for (int s = L / 2; s > 0; s >>= 1) {
      if (l < s) {
        red[l] = f4add(red[l], red[l + s]);
        red[l + B] = f4add(red[l + B], red[l + s + B]);
      }
      __syncthreads();
    }
    if (l == 0) {
      a.pff_new[grp] = red[0];
      a.pff_new[grp + ngroups] = red[B];
    }
  }
}

// ---------------------------------------------------------------------------
// The FP64 particle pass (particle_precision = 1): the same steps as
// particle_group, with the sphere state, the per-sphere force and torque sums
// and the Newton-Euler integration in double.  The fluid-side records (marker
// weights and forces, read-back copies of the state and partials) are float.
struct Kin64 {
  double4 x, v, q, w;
};

__device__ __forceinline__ double4 d4(const double* p) { return make_double4(p[0], p[1], p[2], p[3]); }
__device__ __forceinline__ void d4st(double* p, double4 v) {
  p[0] = v.x;
  p[1] = v.y;
  p[2] = v.z;
  p[3] = v.w;
}
__device__ __forceinline__ double4 d4add(double4 a, double4 b) {
  return make_double4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ double4 d4mul(double4 a, double s) { return make_double4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ double4 d4cross(double4 a, double4 b) {
  return make_double4(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, 0.0);
}
__device__ __forceinline__ double4 f2d(float4 a) { return make_double4(a.x, a.y, a.z, a.w); }
__device__ __forceinline__ float4 d2f(double4 a) {
  return make_float4((float)a.x, (float)a.y, (float)a.z, (float)a.w);
}
__device__ __forceinline__ double wrap_mod64(double a, double w) {
  if (a >= 0.0 && a < w) return a;
  if (a >= w && a < 2.0 * w) return a - w;
  return fmod(a, w);
}

// particle_dynamics (CPU_program.cl:209-276) in double.
__device__ Kin64 rigid_update_f64(const ParticleArgs& a, int p) {
  const ParticleParams& P = a.p;
  const int np = P.np, nfa = P.nfa;
  Kin64 k;
  k.x = d4(a.kin64_old + 4 * (size_t)p);
  k.v = d4(a.kin64_old + 4 * (size_t)(p + np));
  k.q = d4(a.kin64_old + 4 * (size_t)(p + 2 * np));
  k.w = d4(a.kin64_old + 4 * (size_t)(p + 3 * np));
  if (P.fixed) return k;
  double4 acc = make_double4(0, 0, 0, 0), aacc = acc;
  for (int fa = 0; fa < nfa; fa++) {
    acc = d4add(acc, d4(a.pff64_old + 4 * (size_t)(p * nfa + fa)));
    aacc = d4add(aacc, d4(a.pff64_old + 4 * (size_t)((p + np) * nfa + fa)));
  }
  acc = d4add(acc, f2d(a.pf_old[p]));
  aacc = d4add(aacc, f2d(a.pf_old[p + np]));
  acc = d4mul(acc, 1.0 / (double)P.mass);
  aacc = d4mul(aacc, 1.0 / (double)P.inertia);
  acc.x += P.g[0];
  acc.y += P.g[1];
  acc.z += P.g[2];
  const double4 W = make_double4(P.S[0], P.S[1], P.S[2], 1.0);
  const double4 rw = d4add(d4add(d4add(k.x, k.v), d4mul(acc, 0.5)), W);
  Kin64 o;
  o.x = make_double4(wrap_mod64(rw.x, W.x), wrap_mod64(rw.y, W.y), wrap_mod64(rw.z, W.z), wrap_mod64(rw.w, W.w));
  o.v = d4add(k.v, acc);
  const double dqw = -(k.w.x * k.q.x + k.w.y * k.q.y + k.w.z * k.q.z + k.w.w * k.q.w);
  const double4 dq = d4add(d4mul(k.w, k.q.w), d4cross(k.w, k.q));
  o.q = d4mul(dq, 0.5);
  o.q.w += 0.5 * dqw;
  o.w = d4add(k.w, aacc);
  return o;
}

// One work-group of markers, FP64 state and sums; red holds 2*blockDim.x
// double4 (forces, then torques), summed in the reference's tree order.
__device__ __forceinline__ void particle_group_f64(const ParticleArgs& a, const int grp, double4* red, Kin64& s_kin) {
  const ParticleParams& P = a.p;
  const Geom& g = a.g;
  const int np = P.np, nfa = P.nfa, L = P.L;
  const int ngroups = np * nfa;
  const int l = threadIdx.x;
  const int lane = l & 31;
  const int p = grp / nfa;
  const int wg = grp - p * nfa;
  const float4 r0f = l < L ? a.sphere[wg * L + l] : make_float4(0.f, 0.f, 0.f, 0.f);
  if (l == 0) {
    const Kin64 kn = rigid_update_f64(a, p);
    s_kin = kn;
    if (wg == 0) {
      d4st(a.kin64_new + 4 * (size_t)p, kn.x);
      d4st(a.kin64_new + 4 * (size_t)(p + np), kn.v);
      d4st(a.kin64_new + 4 * (size_t)(p + 2 * np), kn.q);
      d4st(a.kin64_new + 4 * (size_t)(p + 3 * np), kn.w);
      a.kin_new[p] = d2f(kn.x);
      a.kin_new[p + np] = d2f(kn.v);
      a.kin_new[p + 2 * np] = d2f(kn.q);
      a.kin_new[p + 3 * np] = d2f(kn.w);
    }
  }
  __syncthreads();
  const Kin64 k = s_kin;
  double4 force = make_double4(0, 0, 0, 0), torque = force;
  int tx[4], ty[4], tz[4], nx = 0, ny = 0, nz = 0;
  const long long gid = (long long)grp * L + l;
  if (l < L) {
    const double4 r0 = f2d(r0f);
    const double4 W = make_double4(P.S[0], P.S[1], P.S[2], 1.0);
    const double4 rw = d4add(d4add(k.x, r0), W);
    const double4 rpp =
        make_double4(wrap_mod64(rw.x, W.x), wrap_mod64(rw.y, W.y), wrap_mod64(rw.z, W.z), wrap_mod64(rw.w, W.w));
    const double fx = floor(rpp.x), fy = floor(rpp.y), fz = floor(rpp.z);
    const int x0 = (int)fx + P.buffer[0], y0 = (int)fy + P.buffer[1], z0 = (int)fz + P.buffer[2];
    const bool ok = fx == fx && fy == fy && fz == fz && x0 >= 1 && x0 <= g.Nx - 2 && y0 >= 1 && y0 <= g.Ny - 2 &&
                    z0 >= 1 && z0 <= g.Nz - 2;
    if (!ok) {
      atomicOr(a.err, ERR_NONFINITE);
    } else {
      const int xs = (x0 == g.Nx - 2) ? -(g.Nx - 3) : 1;
      const int ys = (y0 == g.Ny - 2) ? -(g.Ny - 3) : 1;
      const int zs = (z0 == g.Nz - 2) ? -(g.Nz - 3) : 1;
      const double wx = 1.0 - (rpp.x - fx), wy = 1.0 - (rpp.y - fy), wz = 1.0 - (rpp.z - fz);
      const double w[8] = {wx * wy * wz,
                           (1.0 - wx) * wy * wz,
                           wx * (1.0 - wy) * wz,
                           wx * wy * (1.0 - wz),
                           (1.0 - wx) * (1.0 - wy) * wz,
                           (1.0 - wx) * wy * (1.0 - wz),
                           wx * (1.0 - wy) * (1.0 - wz),
                           (1.0 - wx) * (1.0 - wy) * (1.0 - wz)};
      const int sh[8][3] = {{0, 0, 0}, {xs, 0, 0}, {0, ys, 0}, {0, 0, zs}, {xs, ys, 0}, {xs, 0, zs},
                            {0, ys, zs}, {xs, ys, zs}};
      double ux = 0.0, uy = 0.0, uz = 0.0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const long long i =
            (x0 + sh[j][0]) + (long long)g.Nx * ((y0 + sh[j][1]) + (long long)g.Ny * (z0 + sh[j][2]));
        if (out_of_bounds(i, g.NC, a.err)) continue;
        ux += w[j] * a.u[i];
        uy += w[j] * a.u[i + g.NC];
        uz += w[j] * a.u[i + 2 * g.NC];
      }
      const double4 vpp = d4add(k.v, d4cross(k.w, r0));
      force = d4mul(make_double4(ux - vpp.x, uy - vpp.y, uz - vpp.z, -vpp.w), (double)P.pointArea);
      torque = d4cross(r0, force);
      a.mrec[2 * gid] = make_float4((float)wx, (float)wy, (float)wz, __uint_as_float((unsigned)x0 | ((unsigned)y0 << 16)));
      a.mrec[2 * gid + 1] = make_float4((float)force.x, (float)force.y, (float)force.z, __uint_as_float((unsigned)z0));
      nx = tile_set(x0, x0 + xs, TILE_X, g.ntx, tx, g.Nx, P.periodicSmooth && g.periodic[0]);
      ny = tile_set(y0, y0 + ys, TILE_Y, g.nty, ty, g.Ny, P.periodicSmooth && g.periodic[1]);
      nz = tile_set(z0, z0 + zs, TILE_Z, g.ntz, tz);
    }
  }
  insert_marker(a, gid, lane, tx, ty, tz, nx, ny, nz);
  record_fmax(a, (float)force.x, (float)force.y, (float)force.z, lane);
  const int B = blockDim.x;
  red[l] = force;
  red[l + B] = torque;
  __syncthreads();
  for (int s = L / 2; s > 0; s >>= 1) {
    if (l < s) {
      red[l] = d4add(red[l], red[l + s]);
      red[l + B] = d4add(red[l + B], red[l + s + B]);
    }
    __syncthreads();
  }
  if (l == 0) {
    d4st(a.pff64_new + 4 * (size_t)grp, red[0]);
    d4st(a.pff64_new + 4 * (size_t)(grp + ngroups), red[B]);
    a.pff_new[grp] = d2f(red[0]);
    a.pff_new[grp + ngroups] = d2f(red[B]);
  }
}

__global__ void particle_step_f64_kernel(const ParticleArgs a) {
  extern __shared__ double4 red64[];
  __shared__ Kin64 s_kin;
  particle_group_f64(a, blockIdx.x, red64, s_kin);
}

__global__ void particle_step_kernel(const ParticleArgs a) {
  extern __shared__ float4 red[];
  __shared__ Kin s_kin;
  particle_group(a, blockIdx.x, red, s_kin);
}

// The particle pass of many lattices in one persistent launch: work items
// {slot, group} of the packed list, arguments slots[2*s + parity].
__global__ void particle_batch_kernel(const ParticleArgs* __restrict__ slots, const int2* __restrict__ work,
                                      const int* __restrict__ nwork, const int parity) {
  extern __shared__ float4 red[];
  __shared__ Kin s_kin;
  const int n = *nwork;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const int2 it = work[w];
    particle_group(slots[2 * it.x + parity], it.y, red, s_kin);
    __syncthreads();  // red and s_kin are reused by the next item
  }
}

// Particle-particle forces (CPU_program.cl:76-184) from the positions the
// particle pass of this step wrote, after it (the reference's order:
// particle_dynamics, IBM, particle_particle_forces).  One warp per sphere pi.
__device__ __forceinline__ void contact_sphere(const ParticleArgs& a, const int pi, const int lane) {
  const ParticleParams& P = a.p;
  const int np = P.np;
  // Every pair occurrence the reference's zone loops produce for pi: as the
  // higher index (neighbour zones of pi's zone, members pj < pi; lane t takes
  // neighbour entry t) and as the lower one (zones whose neighbour list names
  // pi's zone, members pk > pi; lanes over the reverse table), then a fixed
  // shuffle reduction: deterministic.
  const int nzones = P.numZones[0] * P.numZones[1] * P.numZones[2];
  const Kin ki = load_kin(a.kin_new, pi, np);
  float4 F = make_float4(0.f, 0.f, 0.f, 0.f);
  const int pz = a.parsZone[pi];
  if (P.exact) {
    // The reference's accumulation order (serial work-items, spheres in
    // increasing index): pi's own pairs in zone/member order, its wall
    // terms, then the pairs of every higher sphere that names pi.
    if (lane != 0) return;
    if (pz >= 0 && pz < nzones) {
      for (int t = 1; t <= a.znd[28 * pz]; t++) {
        const int zid = a.znd[28 * pz + t];
        if (zid < 0 || zid >= nzones) continue;
        for (int j = 0; j < a.numParInZone[zid]; j++) {
          if (out_of_bounds(j, np, a.err)) break;
          const int pj = a.zoneMembers[zid * np + j];
          if (out_of_bounds(pj, np, a.err) || !(pi > pj)) continue;
          const Kin kj = load_kin(a.kin_new, pj, np);
          float4 e;
          float fm;
          if (pair_force(P, ki, kj, e, fm)) F = f4sub(F, f4mul(e, fm));
        }
      }
    }
    const float lo = __fsub_rn(P.zbuf, ki.x.z);
    if (lo > 0) F.z = __fadd_rn(F.z, __fmul_rn(P.kcol, lo));
    const float up = __fsub_rn(ki.x.z, __fsub_rn((float)P.Sint[2], P.zbuf));
    if (up > 0) F.z = __fsub_rn(F.z, __fmul_rn(P.kcol, up));
    if (pz >= 0 && pz < nzones) {
      for (int pk = pi + 1; pk < np; pk++) {
        const int Y = a.parsZone[pk];
        if (Y < 0 || Y >= nzones) continue;
        bool have = false;
        Kin kk;
        for (int t = 1; t <= a.znd[28 * Y]; t++) {
          if (a.znd[28 * Y + t] != pz) continue;
          if (!have) {
            kk = load_kin(a.kin_new, pk, np);
            have = true;
          }
          float4 e;
          float fm;
          if (pair_force(P, kk, ki, e, fm)) F = f4add(F, f4mul(e, fm));
        }
      }
    }
    a.pf_new[pi] = F;
    a.pf_new[pi + np] = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  if (pz >= 0 && pz < nzones) {
    const int nn = a.znd[28 * pz];
    for (int t = lane; t < nn; t += 32) {
      const int zid = a.znd[28 * pz + 1 + t];
      if (zid < 0 || zid >= nzones) continue;  // zone ids past the grid name no zone
      const int cnt = a.numParInZone[zid];
      for (int j = 0; j < cnt; j++) {
        if (out_of_bounds(j, np, a.err)) break;
        const int pj = a.zoneMembers[zid * np + j];
        if (out_of_bounds(pj, np, a.err) || !(pi > pj)) continue;
        const Kin kj = load_kin(a.kin_new, pj, np);
        float4 e;
        float fm;
        if (pair_force(P, ki, kj, e, fm)) F = f4sub(F, f4mul(e, fm));
      }
    }
    for (int r = a.revStart[pz] + lane; r < a.revStart[pz + 1]; r += 32) {
      const int Y = a.revList[r];
      if (out_of_bounds(Y, nzones, a.err)) continue;
      const int cnt = a.numParInZone[Y];
      for (int j = 0; j < cnt; j++) {
        if (out_of_bounds(j, np, a.err)) break;
        const int pk = a.zoneMembers[Y * np + j];
        if (out_of_bounds(pk, np, a.err) || !(pk > pi)) continue;
        const Kin kk = load_kin(a.kin_new, pk, np);
        float4 e;
        float fm;
        if (pair_force(P, kk, ki, e, fm)) F = f4add(F, f4mul(e, fm));
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    F.x = __fadd_rn(F.x, __shfl_xor_sync(0xffffffffu, F.x, o));
    F.y = __fadd_rn(F.y, __shfl_xor_sync(0xffffffffu, F.y, o));
    F.z = __fadd_rn(F.z, __shfl_xor_sync(0xffffffffu, F.z, o));
    F.w = __fadd_rn(F.w, __shfl_xor_sync(0xffffffffu, F.w, o));
  }
  if (lane != 0) return;
  // z-wall repulsion (CPU_program.cl:174-182).
  const float lo = __fsub_rn(P.zbuf, ki.x.z);
  if (lo > 0) F.z = __fadd_rn(F.z, __fmul_rn(P.kcol, lo));
  const float up = __fsub_rn(ki.x.z, __fsub_rn((float)P.Sint[2], P.zbuf));
  if (up > 0) F.z = __fsub_rn(F.z, __fmul_rn(P.kcol, up));
  a.pf_new[pi] = F;
  a.pf_new[pi + np] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// One warp per sphere.
__global__ void contact_kernel(const ParticleArgs a) {
  const int pi = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (pi >= a.p.np) return;  // whole warps
  contact_sphere(a, pi, threadIdx.x & 31);
}

// Contacts of many lattices: one warp per work item {slot, sphere}.
__global__ void contact_batch_kernel(const ParticleArgs* __restrict__ slots, const int2* __restrict__ work,
                                     const int* __restrict__ nwork, const int parity) {
  const int n = *nwork;
  const int warps = gridDim.x * (blockDim.x / 32);
  for (int w = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); w < n; w += warps) {
    const int2 it = work[w];
    contact_sphere(slots[2 * it.x + parity], it.y, threadIdx.x & 31);
  }
}


// update_particle_zones (CPU_program.cl:280-315) for all spheres: members of
// each zone listed in increasing sphere index, the order the reference's
// serial work-item loop produces.
__device__ __forceinline__ void zone_rebuild(const ZoneArgs& a) {
  const ParticleParams& P = a.p;
  const int np = P.np;
  const int nz = P.numZones[0] * P.numZones[1] * P.numZones[2];
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    const float4 x = a.kin[p];
    int zx = (int)(x.x / P.zoneWidth[0]), zy = (int)(x.y / P.zoneWidth[1]), zz = (int)(x.z / P.zoneWidth[2]);
    int zid = zx + P.numZones[0] * (zy + P.numZones[1] * zz);
    if (zid < 0 || zid >= nz) {
      atomicOr(a.err, ERR_ZONE_RANGE);
      zid = zid < 0 ? 0 : nz - 1;
    }
    a.zoneOf[p] = zid;
    a.parsZone[p] = zid;
  }
  __syncthreads();
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    int c = 0;
    for (int p = 0; p < np; p++)
      if (a.zoneOf[p] == z) a.zoneMembers[z * np + c++] = p;
    a.numParInZone[z] = c;
  }
}

__global__ void zone_rebuild_kernel(const ZoneArgs a) { zone_rebuild(a); }

// Zone rebuilds of many lattices: block b rebuilds lattice slots[b].
__global__ void zone_batch_kernel(const ZoneArgs* __restrict__ args, const int* __restrict__ slots,
                                  const int* __restrict__ nslots, const int parity) {
  if ((int)blockIdx.x >= *nslots) return;
  zone_rebuild(args[2 * slots[blockIdx.x] + parity]);
}

// Per-plane FP64 sums over the interior nodes of z-plane blockIdx.x:
// out[5*z + 0..2] = sums of u_x, u_y, u_z, out[5*z + 3] = sum of the shear
// rate g_xz = du_x/dz + du_z/dx, out[5*z + 4] = sum of the viscous shear
// stress nu * g_xz with nu = (tau - 1/2)/3 (lattice units, rho = 1).
// Derivatives are central, wrapped on periodic axes and one-sided on the
// wall layers (the wet nodes at 1 and N-2).  The reduction order is fixed,
// so the sums are deterministic.
__device__ __forceinline__ int axis_step(int c, int d, int N, bool periodic) {
  // Neighbour c+d along an axis of interior nodes 1..N-2: wrapped when
  // periodic, clamped (one-sided difference) otherwise.
  int n = c + d;
  if (n < 1) n = periodic ? N - 2 : 1;
  if (n > N - 2) n = periodic ? 1 : N - 2;
  return n;
}

__global__ void __launch_bounds__(256) plane_stats_kernel(const Geom g, const float* __restrict__ u,
                                                          const float* __restrict__ tau, float tauN, int variable,
                                                          double* __restrict__ out) {
  __shared__ double red[5][256];
  const int z = blockIdx.x;
  const int tid = threadIdx.x;
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (z >= 1 && z <= g.Nz - 2) {
    const long long NC = g.NC;
    const int nx = g.Nx - 2, ny = g.Ny - 2;
    const int zm = axis_step(z, -1, g.Nz, g.periodic[2]), zp = axis_step(z, 1, g.Nz, g.periodic[2]);
    for (int k = tid; k < nx * ny; k += 256) {
      const int x = 1 + k % nx, y = 1 + k / nx;
      const long long i = x + (long long)g.Nx * (y + (long long)g.Ny * z);
      const int xm = axis_step(x, -1, g.Nx, g.periodic[0]), xp = axis_step(x, 1, g.Nx, g.periodic[0]);
      const long long row = (long long)g.Nx * (y + (long long)g.Ny * z);
      const long long izm = x + (long long)g.Nx * (y + (long long)g.Ny * zm);
      const long long izp = x + (long long)g.Nx * (y + (long long)g.Ny * zp);
      const double ux = u[i], uy = u[i + NC], uz = u[i + 2 * NC];
      // Spacing of the difference: 2 for a central one, 1 for a one-sided
      // one, 0 for a single-node axis (no gradient).
      const int hz = (zp != z) + (zm != z), hx = (xp != x) + (xm != x);
      const double dudz = hz ? ((double)u[izp] - (double)u[izm]) / hz : 0.0;
      const double dwdx = hx ? ((double)u[row + xp + 2 * NC] - (double)u[row + xm + 2 * NC]) / hx : 0.0;
      const double gxz = dudz + dwdx;
      const double nu = ((variable ? (double)tau[i] : (double)tauN) - 0.5) / 3.0;
      s[0] += ux;
      s[1] += uy;
      s[2] += uz;
      s[3] += gxz;
      s[4] += nu * gxz;
    }
  }
#pragma unroll
  for (int c = 0; c < 5; c++) red[c][tid] = s[c];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w) {
#pragma unroll
      for (int c = 0; c < 5; c++) red[c][tid] += red[c][tid + w];
    }
    __syncthreads();
  }
  if (tid < 5) out[5 * z + tid] = red[tid][0];
}

__global__ void marker_cells_kernel(const float4* mrec, int M, int* cells) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  int x0, y0, z0;
  decode_marker(mrec[2 * m], mrec[2 * m + 1], x0, y0, z0);
  cells[3 * m] = x0;
  cells[3 * m + 1] = y0;
  cells[3 * m + 2] = z0;
}

// Float distributions <-> stored form, element by element (row q of the
// 19 x N_C array carries the shift w_q).
template <typename ST>
__global__ void store_f_kernel(const float* __restrict__ in, ST* __restrict__ out, long long NC) {
  const long long n = 19 * NC;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(k / NC);
    Stored<ST>::store(out + k, in[k], q == 0 ? WQ(0) : (q <= 6 ? WQ(1) : WQ(7)));
  }
}

template <typename ST>
__global__ void load_f_kernel(const ST* __restrict__ in, float* __restrict__ out, long long NC) {
  const long long n = 19 * NC;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(k / NC);
    out[k] = Stored<ST>::load(in + k, q == 0 ? WQ(0) : (q <= 6 ? WQ(1) : WQ(7)));
  }
}

// ---------------------------------------------------------------------------
// Launchers.

// A launch whose blocks may be scheduled before the previous kernel in the
// stream has completed (programmatic dependent launch); the kernel orders its
// accesses with pdl_wait().
template <typename... KArgs, typename... Args>
static cudaError_t launch_overlapped(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                     Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <int COLL, int VISC, int BC, typename ST>
static cudaError_t launch_fluid_t(const FluidArgs& a, bool first, cudaStream_t s) {
  dim3 block(TILE_X, TILE_Y, 2);
  dim3 grid(a.g.ntx, a.g.nty, a.g.ntz);
  const size_t smem = fluid_smem_bytes(a.has_ibm != 0);
  const int fi = first ? 1 : 0;
  if (a.inplace == 1) return launch_overlapped(fluid_step_kernel<COLL, VISC, BC, ST, 1>, grid, block, smem, s, a, fi);
  if (a.inplace == 2) return launch_overlapped(fluid_step_kernel<COLL, VISC, BC, ST, 2>, grid, block, smem, s, a, fi);
  return launch_overlapped(fluid_step_kernel<COLL, VISC, BC, ST, 0>, grid, block, smem, s, a, fi);
}

template <int COLL, int BC, typename ST>
static cudaError_t launch_fluid_v(const FluidArgs& a, bool first, bool variable, cudaStream_t s) {
  if (!variable) return launch_fluid_t<COLL, 0, BC, ST>(a, first, s);
  switch (a.p.viscModel) {
    case 2: return launch_fluid_t<COLL, 2, BC, ST>(a, first, s);
    case 3: return launch_fluid_t<COLL, 3, BC, ST>(a, first, s);
    case 4: return launch_fluid_t<COLL, 4, BC, ST>(a, first, s);
    default: return launch_fluid_t<COLL, 1, BC, ST>(a, first, s);  // tau = NewtonianTau, stored
  }
}

template <typename ST>
static cudaError_t launch_fluid_st(const FluidArgs& a, bool first, bool variable, int collision, cudaStream_t s) {
  const Geom& g = a.g;
  const bool zwall = g.periodic[0] && g.periodic[1] && g.wallAxis == 2 && !g.tanBC[0] && !g.tanBC[1] && !g.tanBC[2];
  if (collision == 0)
    return zwall ? launch_fluid_v<0, BC_ZWALL, ST>(a, first, variable, s)
                 : launch_fluid_v<0, BC_GENERIC, ST>(a, first, variable, s);
  return zwall ? launch_fluid_v<1, BC_ZWALL, ST>(a, first, variable, s)
               : launch_fluid_v<1, BC_GENERIC, ST>(a, first, variable, s);
}

cudaError_t launch_fluid(const FluidArgs& a, bool first, bool variable, int collision, int storage, cudaStream_t s) {
  if (storage == STORE_F64) {
    // The FP64 build: the reference's MRT only.
    if (collision != 0) return cudaErrorInvalidValue;
    const Geom& g = a.g;
    const bool zwall = g.periodic[0] && g.periodic[1] && g.wallAxis == 2 && !g.tanBC[0] && !g.tanBC[1] && !g.tanBC[2];
    return zwall ? launch_fluid_v<0, BC_ZWALL, double>(a, first, variable, s)
                 : launch_fluid_v<0, BC_GENERIC, double>(a, first, variable, s);
  }
  if (storage == STORE_F16) return launch_fluid_st<__half>(a, first, variable, collision, s);
  if (storage == STORE_BF16) return launch_fluid_st<__nv_bfloat16>(a, first, variable, collision, s);
  return launch_fluid_st<float>(a, first, variable, collision, s);
}

cudaError_t launch_materialize_f(const FluidArgs& a, int storage, float* out, cudaStream_t s) {
  if (storage == STORE_F64) materialize_f_kernel<double><<<1184, 256, 0, s>>>(a, out);
  else if (storage == STORE_F16) materialize_f_kernel<__half><<<1184, 256, 0, s>>>(a, out);
  else if (storage == STORE_BF16) materialize_f_kernel<__nv_bfloat16><<<1184, 256, 0, s>>>(a, out);
  else materialize_f_kernel<float><<<1184, 256, 0, s>>>(a, out);
  return cudaGetLastError();
}

cudaError_t launch_store_f(const float* in, void* out, long long NC, int storage, cudaStream_t s) {
  if (storage == STORE_F64) store_f_kernel<double><<<1184, 256, 0, s>>>(in, static_cast<double*>(out), NC);
  else if (storage == STORE_F16) store_f_kernel<__half><<<1184, 256, 0, s>>>(in, static_cast<__half*>(out), NC);
  else if (storage == STORE_BF16)
    store_f_kernel<__nv_bfloat16><<<1184, 256, 0, s>>>(in, static_cast<__nv_bfloat16*>(out), NC);
  else store_f_kernel<float><<<1184, 256, 0, s>>>(in, static_cast<float*>(out), NC);
  return cudaGetLastError();
}

cudaError_t launch_load_f(const void* in, float* out, long long NC, int storage, cudaStream_t s) {
  if (storage == STORE_F64) load_f_kernel<double><<<1184, 256, 0, s>>>(static_cast<const double*>(in), out, NC);
  else if (storage == STORE_F16) load_f_kernel<__half><<<1184, 256, 0, s>>>(static_cast<const __half*>(in), out, NC);
  else if (storage == STORE_BF16)
    load_f_kernel<__nv_bfloat16><<<1184, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(in), out, NC);
  else load_f_kernel<float><<<1184, 256, 0, s>>>(static_cast<const float*>(in), out, NC);
  return cudaGetLastError();
}

cudaError_t launch_particles(const ParticleArgs& a, cudaStream_t s) {
  const int ngroups = a.p.np * a.p.nfa;
  const int threads = a.p.L < 128 ? 128 : a.p.L;
  if (a.p64) {
    particle_step_f64_kernel<<<ngroups, threads, sizeof(double4) * 2 * threads, s>>>(a);
    return cudaGetLastError();
  }
  const size_t smem = sizeof(float4) * 2 * threads;
  return launch_overlapped(particle_step_kernel, dim3(ngroups), dim3(threads), smem, s, a);
}

cudaError_t launch_contacts(const ParticleArgs& a, cudaStream_t s) {
  contact_kernel<<<(a.p.np + 3) / 4, 128, 0, s>>>(a);
  return cudaGetLastError();
}

// Batched passes (the lattice pool): fixed persistent grids, the work list
// lengths live on the device so one captured sequence serves any mix.
template <typename ST>
static void fluid_batch_aa(const FluidArgs* slots, const int2* work, const int* nwork, int parity, int inplace,
                           int blocks, size_t smem, cudaStream_t s) {
  const dim3 block(TILE_X, TILE_Y, 2);
  if (inplace == 1) fluid_batch_kernel<ST, 1><<<blocks, block, smem, s>>>(slots, work, nwork, parity);
  else if (inplace == 2) fluid_batch_kernel<ST, 2><<<blocks, block, smem, s>>>(slots, work, nwork, parity);
  else fluid_batch_kernel<ST, 0><<<blocks, block, smem, s>>>(slots, work, nwork, parity);
}

cudaError_t launch_fluid_batch(const FluidArgs* slots, const int2* work, const int* nwork, int parity, int storage,
                               int inplace, int blocks, cudaStream_t s) {
  const size_t smem = fluid_smem_bytes(true);
  if (storage == STORE_F16) fluid_batch_aa<__half>(slots, work, nwork, parity, inplace, blocks, smem, s);
  else if (storage == STORE_BF16) fluid_batch_aa<__nv_bfloat16>(slots, work, nwork, parity, inplace, blocks, smem, s);
  else fluid_batch_aa<float>(slots, work, nwork, parity, inplace, blocks, smem, s);
  return cudaGetLastError();
}

cudaError_t launch_particle_batch(const ParticleArgs* slots, const int2* work, const int* nwork, int parity,
                                  int threads, int blocks, cudaStream_t s) {
  particle_batch_kernel<<<blocks, threads, sizeof(float4) * 2 * threads, s>>>(slots, work, nwork, parity);
  return cudaGetLastError();
}

cudaError_t launch_contact_batch(const ParticleArgs* slots, const int2* work, const int* nwork, int parity,
                                 int blocks, cudaStream_t s) {
  contact_batch_kernel<<<blocks, 128, 0, s>>>(slots, work, nwork, parity);
  return cudaGetLastError();
}

cudaError_t launch_zone_batch(const ZoneArgs* args, const int* slots, const int* nslots, int parity, int max_slots,
                              cudaStream_t s) {
  zone_batch_kernel<<<max_slots, 1024, 0, s>>>(args, slots, nslots, parity);
  return cudaGetLastError();
}

cudaError_t launch_zones(const ZoneArgs& a, cudaStream_t s) {
  zone_rebuild_kernel<<<1, 1024, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_spread_field(const Geom& g, const TileLists& t, int last_step, float* out, unsigned* err,
                                cudaStream_t s) {
  dim3 grid(g.ntx, g.nty, g.ntz);
  spread_field_kernel<<<grid, FLUID_THREADS, 0, s>>>(g, t, last_step, out, err);
  return cudaGetLastError();
}

__global__ void widen_kernel(const float* __restrict__ in, double* __restrict__ out, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    out[k] = in[k];
}

cudaError_t launch_widen(const float* in, double* out, long long n, cudaStream_t s) {
  widen_kernel<<<1184, 256, 0, s>>>(in, out, n);
  return cudaGetLastError();
}

__global__ void copy_err_kernel(const unsigned* err, double* out) { *out = (double)*err; }

cudaError_t launch_copy_err(const unsigned* err, double* out, cudaStream_t s) {
  copy_err_kernel<<<1, 1, 0, s>>>(err, out);
  return cudaGetLastError();
}

cudaError_t launch_plane_stats(const Geom& g, const float* u, const float* tau, float tauN, int variable,
                               double* out, cudaStream_t s) {
  plane_stats_kernel<<<g.Nz, 256, 0, s>>>(g, u, tau, tauN, variable, out);
  return cudaGetLastError();
}

cudaError_t launch_marker_cells(const float4* mrec, int M, int* cells, cudaStream_t s) {
  marker_cells_kernel<<<(M + 255) / 256, 256, 0, s>>>(mrec, M, cells);
  return cudaGetLastError();
}

}  // namespace d3q19
