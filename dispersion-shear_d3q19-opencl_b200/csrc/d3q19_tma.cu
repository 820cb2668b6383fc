// d3q19_tma.cu -- the collide-stream pass as a TMA-pipelined persistent kernel.
//
// Same step as fluid_step_kernel (d3q19_kernels.cu; reference
// collideMRT_stream_D3Q19 GPU_program.cl:316-624 with boundary_periodic
// 626-735, boundary_velocity 737-865 and the IBM force of 81-289, 356-377),
// organised for the B200 memory system:
//   * persistent CTAs of 512 threads (two per SM where shared memory allows,
//     64 registers each) loop over 32x4x4 tiles (one node per thread);
//   * the populations a tile reads are brought into shared memory by TMA, one
//     box per population (cp.async.bulk.tensor), into a ring of
//     TMA_STAGES stages, so the loads of the next tiles are in flight while
//     the current tile accumulates its IBM force and collides;
//   * the pulled boxes are the tile shifted by -c_q; an x-shifted box starts
//     on the 16-byte boundary below and is wider, and each node reads its
//     value at a compile-time offset.  All boxes of a step come from one
//     tensor map (every pulled box has the widened shape): loads that
//     alternate between tensor maps issued about 25x slower on B200 (measured,
//     1.6 us per load), so the local tau is read with plain loads;
//   * periodic wrap needs no index arithmetic in the pulls: every step that
//     is followed by a pull writes, besides its own cell, a copy into the
//     buffer-layer (ghost) node that the periodic neighbour pulls from.
// Results are those of fluid_step_kernel with the same arguments (the same
// arithmetic in the same order per node).
//
// Selected with d3q19_options.fluid_kernel = 1 for periodic x/y with walls on
// z (the shear cell), the reference's MRT and FP32 or 16-bit storage when the
// lattice's x extent keeps TMA rows 16-byte aligned; other contexts use
// fluid_step_kernel.  Measured on B200 it is the slower of the two for this
// step (128^3 power-law fluid: 0.0995 against 0.0743 ms; with the IBM halo
// the kernel fits one CTA per SM and takes 0.180 against 0.1035 ms): the loads
// are in time (a CTA waits about 1 us per launch for its stages), but the step
// is bound by instruction issue, and staging the loads removes few
// instructions while the tile loop and its barriers add some.
#include "d3q19_device.cuh"

#include <cuda.h>

namespace d3q19 {

constexpr int TMA_THREADS = TILE_X * TILE_Y * TILE_Z;  // one node per thread
#ifndef TMA_STAGES_N
#define TMA_STAGES_N 2
#endif
#ifndef TMA_MIN_BLOCKS
#define TMA_MIN_BLOCKS 2
#endif
constexpr int TMA_STAGES = TMA_STAGES_N;
// Load / store patterns of a step.
constexpr int TM_EVEN = 0;      // in place, even step: own cells in, own cells reversed out
constexpr int TM_ODD = 1;       // in place, odd step: upwind reversed cells in, push downwind
constexpr int TM_TWO_OWN = 2;   // two buffers, first step after an upload: own cells in
constexpr int TM_TWO_PULL = 3;  // two buffers: pull from the upwind nodes

template <int MODE>
struct TmaPull {
  static constexpr bool value = MODE == TM_ODD || MODE == TM_TWO_PULL;
};

// Shared-memory layout of one stage: box q holds width(q) x TILE_Y x TILE_Z
// stored values, x fastest.
template <typename ST, int MODE>
struct TmaLayout {
  static constexpr int ES = (int)sizeof(ST);
  static constexpr int XPAD = 16 / ES;  // elements per 16 bytes
  static constexpr int WIDE = TILE_X + XPAD;
  static constexpr int YZ = TILE_Y * TILE_Z;
  static constexpr bool PULL = TmaPull<MODE>::value;
  __host__ __device__ static constexpr int width(int) { return PULL ? WIDE : TILE_X; }
  __host__ __device__ static constexpr int box_bytes(int q) { return width(q) * YZ * ES; }
  __host__ __device__ static constexpr int offset(int q) { return q == 0 ? 0 : offset(q - 1) + box_bytes(q - 1); }
  static constexpr int F_BYTES = offset(19);
  static constexpr int STAGE_BYTES = (F_BYTES + 127) / 128 * 128;
  // x index of node tx in box q: a pull from x-1 starts XPAD nodes early, a
  // pull from x+1 at the tile origin.
  __host__ __device__ static constexpr int xoff(int q) {
    return !PULL ? 0 : (CXQ(q) == 1 ? XPAD - 1 : (CXQ(q) == -1 ? 1 : 0));
  }
  // The row (population slot) box q is read from.
  __host__ __device__ static constexpr int row(int q) { return MODE == TM_ODD ? OPPQ(q) : q; }
};

// Shared memory of the kernel: the stages, their barriers, and the IBM
// halo when the lattice has spheres.
template <typename ST, int MODE>
__host__ __device__ constexpr size_t tma_smem_bytes(bool ibm) {
  return (size_t)TMA_STAGES * TmaLayout<ST, MODE>::STAGE_BYTES + 16 * TMA_STAGES + (ibm ? sizeof(SpreadSmem) : 0);
}
static_assert(TmaLayout<float, TM_ODD>::box_bytes(1) % 128 == 0 && TmaLayout<float, TM_ODD>::box_bytes(0) % 128 == 0,
              "boxes keep 128-byte alignment");
static_assert(TmaLayout<__half, TM_ODD>::box_bytes(1) % 128 == 0, "boxes keep 128-byte alignment");

// ---------------------------------------------------------------------------
// mbarrier and TMA primitives (PTX ISA: mbarrier, cp.async.bulk.tensor).
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits for phase `parity` of the barrier to complete, for at most limit_ns
// nanoseconds; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned it = 1;; it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63) == 0 && global_ns() - t0 > limit_ns) return false;
  }
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// Value of a population read from shared memory (the stored form).
template <typename ST>
__device__ __forceinline__ float smem_value(const ST* p, float w);
template <>
__device__ __forceinline__ float smem_value<float>(const float* p, float) { return *p; }
template <>
__device__ __forceinline__ float smem_value<__half>(const __half* p, float w) { return __half2float(*p) + w; }
template <>
__device__ __forceinline__ float smem_value<__nv_bfloat16>(const __nv_bfloat16* p, float w) {
  return __bfloat162float(*p) + w;
}

// Issues the TMA loads of tile (X0, Y0, Z0) into a stage (one thread), all
// from the step's one tensor map.
template <typename ST, int MODE>
__device__ __forceinline__ void tma_issue_tile(unsigned char* stage, uint64_t* bar, const CUtensorMap* fmap, int X0,
                                               int Y0, int Z0) {
  using L = TmaLayout<ST, MODE>;
  mbar_expect_tx(bar, (unsigned)L::F_BYTES);
#pragma unroll
  for (int q = 0; q < 19; q++) {
    int x = X0, y = Y0, z = Z0;
    if (L::PULL) {
      x = CXQ(q) == 1 ? X0 - L::XPAD : X0;
      y = Y0 - CYQ(q);
      z = Z0 - CZQ(q);
    }
    tma_load_4d(stage + L::offset(q), fmap, x, y, z, L::row(q), bar);
  }
}

// ---------------------------------------------------------------------------
// IBM force of one tile with TMA_THREADS threads: the tile's listed markers
// spread -w*F on the tile plus a one-node halo in fixed point (as
// accumulate_tile: deterministic), converted to float and smoothed with the
// reference's 27-point stencil at this thread's node.  Work item j of the
// accumulation is (list entry j/8, stencil corner j%8).
template <typename R>
__device__ __forceinline__ void tma_tile_force(SpreadSmem& s, const Geom& g, const TileLists& tl, long long T, int n,
                                               int X0, int Y0, int Z0, int tid, int k, unsigned* err, bool wrap,
                                               R (&sg)[3]) {
  {
    int4* z4 = reinterpret_cast<int4*>(&s.acc[0][0]);
    for (int h = tid; h < 3 * HALO_N / 2; h += TMA_THREADS) z4[h] = make_int4(0, 0, 0, 0);
  }
  __syncthreads();
  const float scale = ldexpf(1.0f, k);
  for (int j = tid; j < 8 * n; j += TMA_THREADS) {
    const int m = tl.list[T * tl.cap + (j >> 3)];
    if (out_of_bounds(m, tl.markers, err)) continue;
    const float4 a = tl.mrec[2 * (long long)m];
    const float4 b = tl.mrec[2 * (long long)m + 1];
    int x0, y0, z0;
    decode_marker(a, b, x0, y0, z0);
    // Corner c of the reference's stencil order (GPU_program.cl:170-178):
    // 0 (0,0,0), 1 x, 2 y, 3 z, 4 xy, 5 xz, 6 yz, 7 xyz.
    const int c = j & 7;
    const bool sx = (0xB2 >> c) & 1, sy = (0xD4 >> c) & 1, sz = (0xE8 >> c) & 1;
    const int xs = (x0 == g.Nx - 2) ? -(g.Nx - 3) : 1;
    const int ys = (y0 == g.Ny - 2) ? -(g.Ny - 3) : 1;
    const int zs = (z0 == g.Nz - 2) ? -(g.Nz - 3) : 1;
    const float w = (sx ? 1.0f - a.x : a.x) * (sy ? 1.0f - a.y : a.y) * (sz ? 1.0f - a.z : a.z);
    const float cf[3] = {w * b.x, w * b.y, w * b.z};
    spread_node(s, g, x0 + (sx ? xs : 0), y0 + (sy ? ys : 0), z0 + (sz ? zs : 0), X0, Y0, Z0, wrap, cf, scale, err);
  }
  __syncthreads();
  // value = (hi * 2^16 + lo) * 2^-k; all sums are read before the field
  // overwrites them.
  constexpr int PER = (3 * HALO_N + TMA_THREADS - 1) / TMA_THREADS;
  const float inv = ldexpf(1.0f, -k), inv_hi = ldexpf(1.0f, 16 - k);
  const double inv64 = ldexp(1.0, -k), inv_hi64 = ldexp(1.0, 16 - k);
  R v[PER];
#pragma unroll
  for (int r = 0; r < PER; r++) {
    const int h = tid + r * TMA_THREADS;
    v[r] = R(0);
    if (h < 3 * HALO_N) {
      const unsigned* slot = reinterpret_cast<const unsigned*>(&(&s.acc[0][0])[h]);
      if (sizeof(R) == 4)
        v[r] = __fmaf_rn((float)(int)slot[1], inv_hi, (float)slot[0] * inv);
      else
        v[r] = (R)((double)(int)slot[1] * inv_hi64 + (double)slot[0] * inv64);
    }
  }
  __syncthreads();
  R* field = halo_field<R>(s);
#pragma unroll
  for (int r = 0; r < PER; r++) {
    const int h = tid + r * TMA_THREADS;
    if (h < 3 * HALO_N) field[h] = v[r];
  }
  __syncthreads();
  // 27-point smoothing (1/4, 1/2, 1/4 per axis) at the thread's node.
  const int tx = tid % TILE_X, ty = (tid / TILE_X) % TILE_Y, tz = tid / (TILE_X * TILE_Y);
#pragma unroll
  for (int d = 0; d < 3; d++) sg[d] = R(0);
#pragma unroll
  for (int pz = 0; pz < 3; pz++) {
    R p3[3] = {R(0), R(0), R(0)};
#pragma unroll
    for (int sy = -1; sy <= 1; sy++)
#pragma unroll
      for (int sx = -1; sx <= 1; sx++) {
        const R ws = R(sx == 0 ? 0.5f : 0.25f) * R(sy == 0 ? 0.5f : 0.25f);
        const int h = (tx + 1 + sx) + HALO_X * ((ty + 1 + sy) + HALO_Y * (tz + pz));
#pragma unroll
        for (int d = 0; d < 3; d++) p3[d] += ws * field[d * HALO_N + h];
      }
    const R wz = R(pz == 1 ? 0.5f : 0.25f);
#pragma unroll
    for (int d = 0; d < 3; d++) sg[d] += wz * p3[d];
  }
}

// Copies of a node's outgoing values into the ghost nodes its periodic
// neighbours pull from (steps followed by a pull: TM_EVEN, TM_TWO_*).  The
// value of direction q leaves through cell `row` of node i; if the node
// i + c_q it is meant for lies across a periodic x or y edge, that node pulls
// it from the ghost i + c_q (unwrapped) - c_q + shift, shift = -+(N-2).
template <typename ST, typename R, bool REV>
__device__ __forceinline__ void ghost_copies(ST* __restrict__ fout, long long NC, int i, int x, int y, const Geom& g,
                                             const R (&f)[19], unsigned* err) {
  const bool xlo = x == 1, xhi = x == g.Nx - 2, ylo = y == 1, yhi = y == g.Ny - 2;
  if (!(xlo || xhi || ylo || yhi)) return;
#pragma unroll
  for (int q = 1; q < 19; q++) {
    const int cx = CXQ(q), cy = CYQ(q);
    const int sx = (cx == 1 && xhi) ? -(g.Nx - 2) : ((cx == -1 && xlo) ? (g.Nx - 2) : 0);
    const int sy = (cy == 1 && yhi) ? -(g.Ny - 2) : ((cy == -1 && ylo) ? (g.Ny - 2) : 0);
    if (sx == 0 && sy == 0) continue;
    const int gi = i + sx + sy * g.Nx;
    if (out_of_bounds(gi, NC, err)) continue;
    Stored<ST>::store_stream(fout + (long long)(REV ? OPPQ(q) : q) * NC + gi, f[q], wq<R>(q));
  }
}

// VISC: the viscosity law fixed at compile time (0 constant tau, 1 stored
// NewtonianTau, 2 power law, 3 Herschel-Bulkley, 4 Casson), the same
// instantiation of the collision as the per-tile kernel's, so both kernels
// round alike.
// Tile coordinates along a CTA's sequence of tiles T0, T0 + stride, ...:
// decomposed once, then advanced with carries (no integer division per
// tile).
struct TileWalk {
  int bx, by, bz, sx, sy, sz, ntx, nty;
  __device__ __forceinline__ TileWalk(int T0, int stride, int ntx_, int nty_) : ntx(ntx_), nty(nty_) {
    bx = T0 % ntx; by = (T0 / ntx) % nty; bz = T0 / (ntx * nty);
    sx = stride % ntx; sy = (stride / ntx) % nty; sz = stride / (ntx * nty);
  }
  __device__ __forceinline__ void next() {
    bx += sx;
    int c = bx >= ntx;
    bx -= c ? ntx : 0;
    by += sy + c;
    c = by >= nty;
    by -= c ? nty : 0;
    bz += sz + c;
  }
};

template <typename ST, int MODE, int VISC>
__global__ void __launch_bounds__(TMA_THREADS, TMA_MIN_BLOCKS)
    fluid_tma_kernel(const __grid_constant__ CUtensorMap fmap, const FluidArgs a, const int first, const int ntiles) {
  using L = TmaLayout<ST, MODE>;
  using R = float;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* stages = smem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TMA_STAGES * L::STAGE_BYTES);
  SpreadSmem& sp = *reinterpret_cast<SpreadSmem*>(smem + TMA_STAGES * L::STAGE_BYTES + 16 * TMA_STAGES);
  const Geom& g = a.g;
  const int tid = threadIdx.x;
  const int tx = tid % TILE_X, ty = (tid / TILE_X) % TILE_Y, tz = tid / (TILE_X * TILE_Y);
  const long long NC = g.NC;
  constexpr bool var = VISC > 0;
  ST* __restrict__ fout = static_cast<ST*>(a.fout);
  constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s: far above any tile's load time

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < TMA_STAGES; s++) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // Everything below reads or writes data of the passes before this one.
  pdl_wait();
  pdl_trigger();

  // The tiles this CTA loads (issue) and computes (walk), in the same order.
  TileWalk issue(blockIdx.x, gridDim.x, g.ntx, g.nty), walk(blockIdx.x, gridDim.x, g.ntx, g.nty);
  if (tid == 0) {
    for (int s = 0; s < TMA_STAGES; s++) {
      if (blockIdx.x + s * gridDim.x >= ntiles) break;
      tma_issue_tile<ST, MODE>(stages + s * L::STAGE_BYTES, &bars[s], &fmap, issue.bx * TILE_X, issue.by * TILE_Y,
                               issue.bz * TILE_Z);
      issue.next();
    }
  }

  int nclamp = 0;
  int k = 0;
  bool aborted = false;
  for (int T = blockIdx.x; T < ntiles; T += gridDim.x, k++, walk.next()) {
    const int s = k % TMA_STAGES;
    const unsigned parity = (unsigned)(k / TMA_STAGES) & 1u;
    const int X0 = walk.bx * TILE_X, Y0 = walk.by * TILE_Y, Z0 = walk.bz * TILE_Z;
    const int x = X0 + tx, y = Y0 + ty, z = Z0 + tz;
    const bool node = x >= 1 && x <= g.Nx - 2 && y >= 1 && y <= g.Ny - 2 && z >= 1 && z <= g.Nz - 2;
    const int i = x + g.Nx * (y + g.Ny * z);
    // The local tau of t-1, requested first so its round trip overlaps the
    // IBM phase and the wait.
    const R tau_old = (var && node) ? R(__ldg(a.tau + i)) : R(a.p.tauN);

    // IBM force of the tile (markers listed by the particle pass of t-1).
    R sg[3] = {R(0), R(0), R(0)};
    if (a.has_ibm) {
      const int cnt = a.tiles.count[T];
      const unsigned fbits = a.tiles.fmax[(a.t + 1) & 1];
      __syncthreads();  // every thread has read the count
      if (tid == 0) {
        a.tiles.count[T] = 0;
        if (T == 0) a.tiles.fmax[a.t & 1] = 0u;
      }
      if (cnt > 0)
        tma_tile_force<R>(sp, g, a.tiles, T, min(cnt, a.tiles.cap), X0, Y0, Z0, tid, fixed_exponent(fbits), a.err,
                          a.p.periodicSmooth != 0, sg);
    }

    // The tile's populations.  One thread waits on the stage's barrier (its
    // acquire makes the TMA writes visible); the others wait in the CTA
    // barrier, which issues nothing while they wait.
    bool ok = true;
    if (tid == 0) ok = mbar_wait(&bars[s], parity, kWaitNs);
    if (!__syncthreads_and(ok)) {
      aborted = true;
      break;
    }
    const unsigned char* st = stages + s * L::STAGE_BYTES;
    R f[19];
    {
      const int nb = tx + TILE_X * (ty + TILE_Y * tz);
      const int nw = tx + L::WIDE * (ty + TILE_Y * tz);
#pragma unroll
      for (int q = 0; q < 19; q++) {
        const ST* box = reinterpret_cast<const ST*>(st + L::offset(q));
        f[q] = smem_value<ST>(box + (L::width(q) == TILE_X ? nb : nw) + L::xoff(q), wq<R>(q));
      }
    }
    __syncthreads();  // stage s is consumed
    if (tid == 0) {
      if (T + TMA_STAGES * gridDim.x < ntiles) {
        tma_issue_tile<ST, MODE>(stages + s * L::STAGE_BYTES, &bars[s], &fmap, issue.bx * TILE_X, issue.by * TILE_Y,
                                 issue.bz * TILE_Z);
        issue.next();
      }
    }

    if (!node || out_of_bounds(i, NC, a.err)) continue;
    // The uploaded state is the reference's buffer after its boundary
    // kernels; every later step rebuilds the wall unknowns.
    if (!first) {
      if (z == 1) velocity_bc<2, 0>(f, a.p.velLower);
      else if (z == g.Nz - 2) velocity_bc<2, 1>(f, a.p.velUpper);
    }
    const R gx = R(a.p.g[0]) + sg[0], gy = R(a.p.g[1]) + sg[1], gz = R(a.p.g[2]) + sg[2];
    R rho = R(0);
#pragma unroll
    for (int q = 0; q < 19; q++) rho += f[q];
    const R jx = f[1] - f[2] + f[7] + f[8] + f[9] + f[10] - f[11] - f[12] - f[13] - f[14];
    const R jy = f[3] - f[4] + f[7] - f[8] + f[11] - f[12] + f[15] + f[16] - f[17] - f[18];
    const R jz = f[5] - f[6] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16] + f[17] - f[18];
    const R ir = RMath<R>::rcp(rho);
    const R ux = (jx + R(0.5f) * gx) * ir, uy = (jy + R(0.5f) * gy) * ir, uz = (jz + R(0.5f) * gz) * ir;
    a.u[i] = ux;
    a.u[i + NC] = uy;
    a.u[i + 2 * NC] = uz;
    if (!(rho > R(0) && rho < R(1e30f))) atomicOr(a.err, ERR_NONFINITE);
    R tau = tau_old;
    bool clamped = false;
    collide<0, VISC, R>(f, rho, ir, ux, uy, uz, gx, gy, gz, tau, a.p, clamped);
    if (var) {
      a.tau[i] = tau;
      nclamp += clamped ? 1 : 0;
    }
    if (MODE == TM_ODD) {
      const int dxm = x == 1 ? g.Nx - 3 : -1, dxp = x == g.Nx - 2 ? -(g.Nx - 3) : 1;
      const int dym = (y == 1 ? g.Ny - 3 : -1) * g.Nx, dyp = (y == g.Ny - 2 ? -(g.Ny - 3) : 1) * g.Nx;
      const int Nxy = g.Nx * g.Ny;
#pragma unroll
      for (int q = 0; q < 19; q++) {
        const int cx = CXQ(q), cy = CYQ(q), cz = CZQ(q);
        const int dst = i + (cx == 1 ? dxp : (cx == -1 ? dxm : 0)) + (cy == 1 ? dyp : (cy == -1 ? dym : 0)) +
                        (cz == 1 ? Nxy : (cz == -1 ? -Nxy : 0));
        if (out_of_bounds(dst, NC, a.err)) continue;
        Stored<ST>::store_stream(fout + q * NC + dst, f[q], wq<R>(q));
      }
    } else if (MODE == TM_EVEN) {
#pragma unroll
      for (int q = 0; q < 19; q++) Stored<ST>::store_stream(fout + OPPQ(q) * NC + i, f[q], wq<R>(q));
      ghost_copies<ST, R, true>(fout, NC, i, x, y, g, f, a.err);
    } else {
#pragma unroll
      for (int q = 0; q < 19; q++) Stored<ST>::store(fout + q * NC + i, f[q], wq<R>(q));
      ghost_copies<ST, R, false>(fout, NC, i, x, y, g, f, a.err);
    }
  }
  if (aborted) {
    // A load did not complete in time: record it, and wait (again with a
    // limit) for the loads this CTA issued after it, so no copy is left in
    // flight into shared memory when the CTA exits.
    if (tid == 0) {
      atomicOr(a.err, ERR_TIMEOUT);
      for (int j = 1; j < TMA_STAGES; j++) {
        const int kk = k + j;
        if (blockIdx.x + kk * gridDim.x >= ntiles) break;
        mbar_wait(&bars[kk % TMA_STAGES], (unsigned)(kk / TMA_STAGES) & 1u, 200000000ull);
      }
    }
    __syncthreads();
    return;
  }
  if (var && nclamp) atomicAdd(a.clamps, (unsigned long long)nclamp);
}

// Buffer-layer copies of a whole buffer: node g on the x or y buffer layer
// (z interior) takes all 19 values of its periodic image.
template <typename T>
__global__ void fill_ghosts_kernel(T* __restrict__ f, const Geom g) {
  const long long NC = g.NC;
  const long long per = 2LL * g.Ny + 2LL * (g.Nx - 2);  // per z-plane: two x-columns, two y-rows
  const long long n = per * (g.Nz - 2);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int z = 1 + (int)(k / per);
    int r = (int)(k % per), x, y;
    if (r < 2 * g.Ny) {
      x = r < g.Ny ? 0 : g.Nx - 1;
      y = r % g.Ny;
    } else {
      r -= 2 * g.Ny;
      y = r < g.Nx - 2 ? 0 : g.Ny - 1;
      x = 1 + r % (g.Nx - 2);
    }
    const int ix = x == 0 ? g.Nx - 2 : (x == g.Nx - 1 ? 1 : x);
    const int iy = y == 0 ? g.Ny - 2 : (y == g.Ny - 1 ? 1 : y);
    const long long src = ix + (long long)g.Nx * (iy + (long long)g.Ny * z);
    const long long dst = x + (long long)g.Nx * (y + (long long)g.Ny * z);
#pragma unroll
    for (int q = 0; q < 19; q++) f[q * NC + dst] = f[q * NC + src];
  }
}

cudaError_t launch_fill_ghosts(const FluidArgs& a, int storage, cudaStream_t s) {
  // In place the buffer is read and written; with two buffers fin is the
  // buffer the next step reads.
  void* f = const_cast<void*>(a.fin);
  if (storage_bytes(storage) == 4) fill_ghosts_kernel<unsigned><<<592, 256, 0, s>>>(static_cast<unsigned*>(f), a.g);
  else fill_ghosts_kernel<unsigned short><<<592, 256, 0, s>>>(static_cast<unsigned short*>(f), a.g);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Host side.

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

bool tma_supported(const Geom& g, int storage) {
  if (storage != STORE_F32 && storage != STORE_F16 && storage != STORE_BF16) return false;
  const int es = storage_bytes(storage);
  if (((long long)g.Nx * es) % 16 != 0 || (g.NC * 4) % 16 != 0) return false;
  if (!(g.periodic[0] && g.periodic[1] && g.wallAxis == 2 && !g.tanBC[0] && !g.tanBC[1] && !g.tanBC[2])) return false;
  if (g.Nx < 4 || g.Ny < 4 || g.Nz < 4) return false;
  return encode_fn() != nullptr;
}

static bool encode_f(CUtensorMap* m, void* base, const Geom& g, int storage, int width) {
  const int es = storage_bytes(storage);
  const CUtensorMapDataType dt = storage == STORE_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                 : storage == STORE_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                        : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  const cuuint64_t dims[4] = {(cuuint64_t)g.Nx, (cuuint64_t)g.Ny, (cuuint64_t)g.Nz, 19};
  const cuuint64_t strides[3] = {(cuuint64_t)g.Nx * es, (cuuint64_t)g.Nx * g.Ny * es, (cuuint64_t)g.NC * es};
  const cuuint32_t box[4] = {(cuuint32_t)width, TILE_Y, TILE_Z, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return encode_fn()(m, dt, 4, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool tma_make_maps(TmaMaps* m, void* const f[2], const Geom& g, int storage) {
  if (!tma_supported(g, storage)) return false;
  const int wide = TILE_X + 16 / storage_bytes(storage);
  static_assert(sizeof(CUtensorMap) <= sizeof(m->f[0][0]), "tensor map storage");
  for (int b = 0; b < 2; b++) {
    if (!encode_f(reinterpret_cast<CUtensorMap*>(m->f[b][0]), f[b], g, storage, TILE_X)) return false;
    if (!encode_f(reinterpret_cast<CUtensorMap*>(m->f[b][1]), f[b], g, storage, wide)) return false;
  }
  m->ready = 1;
  return true;
}

template <typename ST, int MODE, int VISC>
static cudaError_t launch_tma_t(const TmaMaps& m, int buf, const FluidArgs& a, bool first, cudaStream_t s) {
  auto kern = fluid_tma_kernel<ST, MODE, VISC>;
  const size_t smem = tma_smem_bytes<ST, MODE>(a.has_ibm != 0);
  // Per device: the shared-memory opt-in (the largest size) and the resident
  // CTAs per SM for each size.
  static int blocks[64][2] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64) return cudaErrorInvalidDevice;
  int& per_sm = blocks[dev][a.has_ibm ? 1 : 0];
  if (!per_sm) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)tma_smem_bytes<ST, MODE>(true));
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TMA_THREADS, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = a.g.ntx * a.g.nty * a.g.ntz;
  const int grid = ntiles < per_sm * sms ? ntiles : per_sm * sms;
  // The step's one tensor map: widened boxes for pulls, tile-wide boxes for
  // own-cell reads.
  const CUtensorMap* fm = reinterpret_cast<const CUtensorMap*>(m.f[buf][TmaPull<MODE>::value ? 1 : 0]);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(TMA_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, *fm, a, first ? 1 : 0, ntiles);
}

template <typename ST, int VISC>
static cudaError_t launch_tma_v(const TmaMaps& m, int buf, const FluidArgs& a, bool first, cudaStream_t s) {
  if (a.inplace == 1) return launch_tma_t<ST, TM_EVEN, VISC>(m, buf, a, first, s);
  if (a.inplace == 2) return launch_tma_t<ST, TM_ODD, VISC>(m, buf, a, first, s);
  if (first) return launch_tma_t<ST, TM_TWO_OWN, VISC>(m, buf, a, first, s);
  return launch_tma_t<ST, TM_TWO_PULL, VISC>(m, buf, a, first, s);
}

// The viscosity law as the per-tile kernel's launcher picks it
// (d3q19_kernels.cu launch_fluid_v).
template <typename ST>
static cudaError_t launch_tma_st(const TmaMaps& m, int buf, const FluidArgs& a, bool first, cudaStream_t s) {
  if (!a.p.variable) return launch_tma_v<ST, 0>(m, buf, a, first, s);
  switch (a.p.viscModel) {
    case 2: return launch_tma_v<ST, 2>(m, buf, a, first, s);
    case 3: return launch_tma_v<ST, 3>(m, buf, a, first, s);
    case 4: return launch_tma_v<ST, 4>(m, buf, a, first, s);
    default: return launch_tma_v<ST, 1>(m, buf, a, first, s);
  }
}

cudaError_t launch_fluid_tma(const TmaMaps& m, int buf, const FluidArgs& a, bool first, int storage, cudaStream_t s) {
  if (!m.ready) return cudaErrorInvalidValue;
  if (storage == STORE_F16) return launch_tma_st<__half>(m, buf, a, first, s);
  if (storage == STORE_BF16) return launch_tma_st<__nv_bfloat16>(m, buf, a, first, s);
  return launch_tma_st<float>(m, buf, a, first, s);
}

}  // namespace d3q19
