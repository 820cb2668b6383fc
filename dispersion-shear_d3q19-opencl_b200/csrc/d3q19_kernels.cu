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
#include "d3q19_internal.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace d3q19 {

// Bounds-checked build (-DD3Q19_BOUNDS_CHECK=1): the data-dependent indices
// of the kernels (pull sources, marker ids read from the tile lists, the
// interpolation stencil, zone and sphere ids of the contact search) are
// checked; an index outside its array sets ERR_BOUNDS and the access is
// skipped.  In the default build the check compiles to nothing.
#ifndef D3Q19_BOUNDS_CHECK
#define D3Q19_BOUNDS_CHECK 0
#endif
__device__ __forceinline__ bool out_of_bounds(long long idx, long long n, unsigned* err) {
#if D3Q19_BOUNDS_CHECK
  if ((unsigned long long)idx >= (unsigned long long)n) {
    atomicOr(err, ERR_BOUNDS);
    return true;
  }
#endif
  return false;
}

// Programmatic dependent launch of the step's collide-stream and particle
// passes (each launched with programmatic stream serialization): a pass's
// blocks may be scheduled while the pass before it in the stream is still
// running, so its launch and block set-up overlap that pass's last wave.
// pdl_wait() returns once every grid the pass depends on has completed and
// its writes are visible (at once when the launch had no such dependency);
// every read or write of another pass's data comes after it.  pdl_trigger()
// lets the next pass's blocks be scheduled; it is issued only after the wait,
// so a pass never starts before the pass two back has completed.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// D3Q19 velocities in the reference's order (D3Q19-OpenCL.c:9-13), as
// compile-time expressions of q so fully unrolled loops fold them.
#define CXQ(q) (((q) == 1 || (q) == 7 || (q) == 8 || (q) == 9 || (q) == 10) ? 1 : \
                (((q) == 2 || (q) == 11 || (q) == 12 || (q) == 13 || (q) == 14) ? -1 : 0))
#define CYQ(q) (((q) == 3 || (q) == 7 || (q) == 11 || (q) == 15 || (q) == 16) ? 1 : \
                (((q) == 4 || (q) == 8 || (q) == 12 || (q) == 17 || (q) == 18) ? -1 : 0))
#define CZQ(q) (((q) == 5 || (q) == 9 || (q) == 13 || (q) == 15 || (q) == 17) ? 1 : \
                (((q) == 6 || (q) == 10 || (q) == 14 || (q) == 16 || (q) == 18) ? -1 : 0))
#define CAQ(A, q) ((A) == 0 ? CXQ(q) : ((A) == 1 ? CYQ(q) : CZQ(q)))
// Opposite direction.
#define OPPQ(q) ((q) == 0 ? 0 : (q) <= 6 ? (((q) & 1) ? (q) + 1 : (q) - 1) : \
                 (q) == 7 ? 12 : (q) == 12 ? 7 : (q) == 8 ? 11 : (q) == 11 ? 8 : \
                 (q) == 9 ? 14 : (q) == 14 ? 9 : (q) == 10 ? 13 : (q) == 13 ? 10 : \
                 (q) == 15 ? 18 : (q) == 18 ? 15 : (q) == 16 ? 17 : 16)

// ---------------------------------------------------------------------------
// Distribution storage.  ST = float keeps f_q itself; the 16-bit forms keep
// the shifted value f_q - w_q (w_q the rest-state weight 1/3, 1/18, 1/36),
// whose magnitude is a small fraction of w_q, so the 16-bit significand
// spends its bits on the deviation from rest.  Arithmetic stays FP32; the
// stored value is rounded to nearest even once per step.  ST = double is the
// FP64 build (arithmetic in double as well).
#define WQ(q) ((q) == 0 ? (1.0f / 3.0f) : (q) <= 6 ? (1.0f / 18.0f) : (1.0f / 36.0f))
// The same weights in the arithmetic type R.
template <typename R>
__device__ __forceinline__ constexpr R wq(int q) {
  return q == 0 ? R(1) / R(3) : (q <= 6 ? R(1) / R(18) : R(1) / R(36));
}

// Arithmetic type of a storage type: FP32 for float and the 16-bit forms,
// FP64 for double (the FP64 build of the collide-stream kernel).
template <typename ST>
struct RealOf {
  using type = float;
};
template <>
struct RealOf<double> {
  using type = double;
};

// Functions of the collide-stream arithmetic: FP32 uses the hardware
// approximations of the reciprocal, reciprocal square root and power (a few
// ulp); FP64 evaluates them in double.
template <typename R>
struct RMath;
template <>
struct RMath<float> {
  static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }
  static __device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
  static __device__ __forceinline__ float rsqrt(float x) { return rsqrtf(x); }
  static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
  static __device__ __forceinline__ float pow(float x, float e) { return exp2f(__log2f(x) * e); }
};
template <>
struct RMath<double> {
  static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
  static __device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
  static __device__ __forceinline__ double rsqrt(double x) { return ::rsqrt(x); }
  static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
  static __device__ __forceinline__ double pow(double x, double e) { return ::pow(x, e); }
};

template <typename ST>
struct Stored;
// store_stream: the same value with an evict-first (streaming) store.  The
// in-place steps write the cells the next step reads; streaming the writes
// keeps more of them, and the rows neighbouring tiles still read, in L2.
__device__ __forceinline__ void stcs_u16(void* p, unsigned short v) { __stcs(static_cast<unsigned short*>(p), v); }
// load/store take and give f_q (the 16-bit forms through load_dev and
// store_dev, which give and take the stored deviation f_q - w_q).
template <>
struct Stored<float> {
  static __device__ __forceinline__ float load(const float* p, float) { return __ldg(p); }
  static __device__ __forceinline__ void store(float* p, float v, float) { *p = v; }
  static __device__ __forceinline__ void store_stream(float* p, float v, float) { __stcs(p, v); }
};
template <>
struct Stored<double> {
  static __device__ __forceinline__ double load(const double* p, double) { return __ldg(p); }
  static __device__ __forceinline__ void store(double* p, double v, double) { *p = v; }
  static __device__ __forceinline__ void store_stream(double* p, double v, double) { __stcs(p, v); }
};
template <>
struct Stored<__half> {
  static __device__ __forceinline__ float load_dev(const __half* p, float) {
    return __half2float(__ushort_as_half(__ldg(reinterpret_cast<const unsigned short*>(p))));
  }
  static __device__ __forceinline__ void store_dev(__half* p, float d, float) { *p = __float2half_rn(d); }
  static __device__ __forceinline__ float load(const __half* p, float w) { return load_dev(p, w) + w; }
  static __device__ __forceinline__ void store(__half* p, float v, float w) { *p = __float2half_rn(v - w); }
  static __device__ __forceinline__ void store_stream(__half* p, float v, float w) {
    stcs_u16(p, __half_as_ushort(__float2half_rn(v - w)));
  }
};
template <>
struct Stored<__nv_bfloat16> {
  static __device__ __forceinline__ float load_dev(const __nv_bfloat16* p, float) {
    return __bfloat162float(__ushort_as_bfloat16(__ldg(reinterpret_cast<const unsigned short*>(p))));
  }
  static __device__ __forceinline__ void store_dev(__nv_bfloat16* p, float d, float) { *p = __float2bfloat16_rn(d); }
  static __device__ __forceinline__ float load(const __nv_bfloat16* p, float w) { return load_dev(p, w) + w; }
  static __device__ __forceinline__ void store(__nv_bfloat16* p, float v, float w) {
    *p = __float2bfloat16_rn(v - w);
  }
  static __device__ __forceinline__ void store_stream(__nv_bfloat16* p, float v, float w) {
    stcs_u16(p, __bfloat16_as_ushort(__float2bfloat16_rn(v - w)));
  }
};

// ---------------------------------------------------------------------------
// Wet-node velocity boundary (GPU_program.cl:737-865 with calcRho = 0, the
// momentum correction off): on the wall plane of axis A (SIDE 0 = lower,
// inward normal +A; SIDE 1 = upper), rho = 1, the inward normal velocity
// follows from the knowns, and each unknown is its opposite population plus
// rho*(u_n + c_t.u_t)/6, or rho*u_n/3 for the normal direction.
template <int A, int SIDE, typename R>
__device__ __forceinline__ void velocity_bc(R (&f)[19], const float* uw) {
  constexpr int IN = SIDE == 0 ? 1 : -1;
  constexpr int A1 = A == 0 ? 1 : 0;
  constexpr int A2 = A == 2 ? 1 : 2;
  R sum9 = R(0), sum5 = R(0);
#pragma unroll
  for (int q = 0; q < 19; q++) {
    if (CAQ(A, q) == 0) sum9 += f[q];
    else if (CAQ(A, q) == -IN) sum5 += f[q];
  }
  const R rho = R(1);
  const R un = R(1) - (sum9 + R(2) * sum5) / rho;
  const R ua1 = uw[A1], ua2 = uw[A2];
#pragma unroll
  for (int q = 1; q < 19; q++) {
    if (CAQ(A, q) != IN) continue;
    const int t1 = CAQ(A1, q), t2 = CAQ(A2, q);
    R v;
    if (t1 == 0 && t2 == 0) {
      v = f[OPPQ(q)] + rho * un / R(3);
    } else if (t1 != 0) {
      v = f[OPPQ(q)] + rho * (t1 > 0 ? un + ua1 : un - ua1) / R(6);
    } else {
      v = f[OPPQ(q)] + rho * (t2 > 0 ? un + ua2 : un - ua2) / R(6);
    }
    f[q] = v;
  }
}

template <typename R>
__device__ __forceinline__ void apply_wall(R (&f)[19], int axis, int side, const FluidParams& p) {
  const float* uw = side ? p.velUpper : p.velLower;
  if (axis == 0) {
    if (side) velocity_bc<0, 1>(f, uw); else velocity_bc<0, 0>(f, uw);
  } else if (axis == 1) {
    if (side) velocity_bc<1, 1>(f, uw); else velocity_bc<1, 0>(f, uw);
  } else {
    if (side) velocity_bc<2, 1>(f, uw); else velocity_bc<2, 0>(f, uw);
  }
}

// Local relaxation time (GPU_program.cl:1041-1128).  FP32 uses the hardware
// approximations of the reciprocal, reciprocal square root and power (a few
// ulp; the reference-exact arithmetic evaluates them as written), FP64 the
// double functions.  Optional extensions: an upper clamp and a regularised
// Casson yield term.  VISC is the viscosity law fixed at compile time (2
// power law, 3 Herschel-Bulkley, 4 Casson), or -1 to read it from
// p.viscModel.
template <int VISC = -1, typename R = float>
__device__ __forceinline__ R compute_tau(const FluidParams& p, R srt, bool& clamped) {
  using M = RMath<R>;
  R tau = p.tauN;
  const R eps = R(1e-8f);
  const int model = VISC >= 0 ? VISC : p.viscModel;
  if (model == 2) {  // power law
    R k = p.visc[0], n = p.visc[1], nu;
    srt = srt > eps ? srt : eps;
    if (n == R(0.5f)) nu = k * M::rsqrt(srt);
    else if (n == R(1)) nu = k;
    else if (n == R(2)) nu = k * srt;
    else nu = k * M::pow(srt, n - R(1));
    tau = R(3) * nu + R(0.5f);
  } else if (model == 4) {  // Casson
    R tY = p.visc[0], eta = p.visc[1];
    srt = srt > eps ? srt : eps;
    R sr2 = p.cassonReg > 0.0f ? srt * srt + R(p.cassonReg) * R(p.cassonReg) : srt * srt;
    R a = M::sqrt(tY * M::rsqrt(sr2)) + M::sqrt(eta);
    tau = R(3) * (a * a) + R(0.5f);
  } else if (model == 3) {  // Herschel-Bulkley
    R tY = p.visc[0], k = p.visc[1], n = p.visc[2], nu;
    srt = srt > eps ? srt : eps;
    const R yield = M::fdiv(tY, srt);
    if (n == R(0.5f)) nu = yield + k * M::rsqrt(srt);
    else if (n == R(1)) nu = yield + k;
    else if (n == R(2)) nu = yield + k * srt;
    else nu = yield + k * M::pow(srt, n - R(1));
    tau = R(3) * nu + R(0.5f);
  } else {
    return tau;
  }
  clamped = false;
  if (p.tauMin > 0.0f) {
    if (tau < R(p.tauMin)) {
      tau = p.tauMin;
      clamped = true;
    }
  } else if (sizeof(R) == 4 ? tau <= R(0.505f) : tau < R(0.505)) {
    // The reference compares with the double constant MIN_TAU = 0.505
    // (GPU_program.cl:6); (double)tau < 0.505 holds exactly for the floats
    // up to and including 0.505f, which lies below 0.505.
    tau = sizeof(R) == 4 ? R(0.505f) : R(0.505);
    clamped = true;
  }
  if (p.tauMax > 0.0f && tau > R(p.tauMax)) tau = p.tauMax;
  return tau;
}

// Populations pulled from the neighbours' post-collision values:
// population q of node i comes from node i - c_q, wrapped on periodic axes.
// On a wall plane the sources outside the lattice interior are the buffer
// layer; those populations are unknowns and are rebuilt by velocity_bc.
// Addressing: row q of the distributions starts at fin + q*NC (a 64-bit
// offset, the same for every thread); within a row the node index is a
// 32-bit int (N_C < 2^31 is checked when the context is created).
template <typename ST, typename R>
__device__ __forceinline__ void gather(R (&f)[19], const ST* __restrict__ fin, long long NC, int i, int dxm,
                                       int dxp, int dym, int dyp, int dzm, int dzp, unsigned* err) {
#pragma unroll
  for (int q = 0; q < 19; q++) {
    const int cx = CXQ(q), cy = CYQ(q), cz = CZQ(q);
    const int src = i + (cx == 1 ? dxm : (cx == -1 ? dxp : 0)) + (cy == 1 ? dym : (cy == -1 ? dyp : 0)) +
                    (cz == 1 ? dzm : (cz == -1 ? dzp : 0));
    if (out_of_bounds(src, NC, err)) {
      f[q] = wq<R>(q);
      continue;
    }
    f[q] = Stored<ST>::load(fin + q * NC + src, wq<R>(q));
  }
}

// The odd step of the in-place (AA) layout: population q of node i is the
// post-collision value the upwind neighbour i - c_q stored, with the
// direction reversed, in its cell opp(q).
template <typename ST, typename R>
__device__ __forceinline__ void gather_reversed(R (&f)[19], const ST* __restrict__ fin, long long NC, int i, int dxm,
                                                int dxp, int dym, int dyp, int dzm, int dzp, unsigned* err) {
#pragma unroll
  for (int q = 0; q < 19; q++) {
    const int cx = CXQ(q), cy = CYQ(q), cz = CZQ(q);
    const int src = i + (cx == 1 ? dxm : (cx == -1 ? dxp : 0)) + (cy == 1 ? dym : (cy == -1 ? dyp : 0)) +
                    (cz == 1 ? dzm : (cz == -1 ? dzp : 0));
    if (out_of_bounds(src, NC, err)) {
      f[q] = wq<R>(q);
      continue;
    }
    f[q] = Stored<ST>::load(fin + OPPQ(q) * NC + src, wq<R>(q));
  }
}

// Offsets to the neighbours x-1, x+1, y-1, y+1, z-1, z+1 of an interior node
// for a boundary layout (wrapped on periodic axes).
template <int BC>
__device__ __forceinline__ void layout_deltas(const Geom& g, int x, int y, int z, int& dxm, int& dxp, int& dym,
                                              int& dyp, int& dzm, int& dzp);

// Index deltas to the upwind neighbours of node (x,y,z).
__device__ __forceinline__ void neighbour_deltas(const Geom& g, int x, int y, int z, int& dxm, int& dxp, int& dym,
                                                 int& dyp, int& dzm, int& dzp) {
  const int Nxy = g.Nx * g.Ny;
  dxm = (g.periodic[0] && x == 1) ? g.Nx - 3 : -1;
  dxp = (g.periodic[0] && x == g.Nx - 2) ? -(g.Nx - 3) : 1;
  dym = ((g.periodic[1] && y == 1) ? g.Ny - 3 : -1) * g.Nx;
  dyp = ((g.periodic[1] && y == g.Ny - 2) ? -(g.Ny - 3) : 1) * g.Nx;
  dzm = ((g.periodic[2] && z == 1) ? g.Nz - 3 : -1) * Nxy;
  dzp = ((g.periodic[2] && z == g.Nz - 2) ? -(g.Nz - 3) : 1) * Nxy;
}

template <int BC>
__device__ __forceinline__ void layout_deltas(const Geom& g, int x, int y, int z, int& dxm, int& dxp, int& dym,
                                              int& dyp, int& dzm, int& dzp) {
  if (BC == 1) {  // BC_ZWALL: periodic x and y, walls on z
    const int Nxy = g.Nx * g.Ny;
    dxm = x == 1 ? g.Nx - 3 : -1;
    dxp = x == g.Nx - 2 ? -(g.Nx - 3) : 1;
    dym = (y == 1 ? g.Ny - 3 : -1) * g.Nx;
    dyp = (y == g.Ny - 2 ? -(g.Ny - 3) : 1) * g.Nx;
    dzm = -Nxy;
    dzp = Nxy;
  } else {
    neighbour_deltas(g, x, y, z, dxm, dxp, dym, dyp, dzm, dzp);
  }
}

// Boundary rebuild after the gather: the wall plane of the wall axis, then
// the tangential velocity boundaries in axis order (sim_main.c:383-402).
template <typename R>
__device__ __forceinline__ void boundaries(R (&f)[19], const Geom& g, const FluidParams& p, int x, int y, int z) {
  if (g.wallAxis < 0) return;
  const int c[3] = {x, y, z};
  const int N[3] = {g.Nx, g.Ny, g.Nz};
  const int a = g.wallAxis;
  if (c[a] == 1) apply_wall(f, a, 0, p);
  else if (c[a] == N[a] - 2) apply_wall(f, a, 1, p);
#pragma unroll
  for (int t = 0; t < 3; t++) {
    if (!g.tanBC[t]) continue;
    if (c[t] == 1) apply_wall(f, t, 0, p);
    else if (c[t] == N[t] - 2) apply_wall(f, t, 1, p);
  }
}

template <int COLL, int VISC, typename R>
__device__ __forceinline__ void collide(R (&f)[19], R rho, R ir, R ux, R uy, R uz, R gx, R gy, R gz, R& tau,
                                        const FluidParams& p, bool& clamped) {
  // Inverse squared norms of the moment basis rows (rho, e, eps, jx, qx, jy,
  // qy, jz, qz, 3pxx, 3pixx, pww, piww, pxy, pyz, pxz, mx, my, mz).
  const R INV_N1 = R(1) / R(2394), INV_N2 = R(1) / R(252), INV_N3 = R(1) / R(10), INV_N4 = R(1) / R(40);
  const R INV_N9 = R(1) / R(36), INV_N10 = R(1) / R(72), INV_N11 = R(1) / R(12), INV_N12 = R(1) / R(24);
  const R INV_N13 = R(1) / R(4), INV_N16 = R(1) / R(8);
  // Equilibrium minus f, pairwise (GPU_program.cl:978-1007), and the Guo term
  // (GPU_program.cl:1010-1038): for a pair +-c the even parts are shared.
  const R usq15 = R(1.5f) * (ux * ux + uy * uy + uz * uz);
  const R uDg = ux * gx + uy * gy + uz * gz;
  // Correctly rounded rho/3, rho/18, rho/36 as the reference's equilibrium
  // (GPU_program.cl:978-1007): a fluid at rest then has exactly zero
  // non-equilibrium part, which the strain rate of a power-law or yield-
  // stress fluid at rest depends on.
  const R r0 = rho / R(3.0f), r1 = rho / R(18.0f), r2 = rho / R(36.0f);
  R d[19], base[19];
  {
    R feq0 = r0 * (R(1.0f) - usq15);
    R fg0 = -uDg;
    d[0] = (feq0 - f[0]) - R(0.5f) * fg0;
    base[0] = f[0] + fg0;
  }
#define PAIR(qp, qm, cu, cg, rw, gd)                                   \
  {                                                                   \
    const R cu_ = (cu), cg_ = (cg);                               \
    const R ev = (rw) * (R(1.0f) + R(4.5f) * cu_ * cu_ - usq15);        \
    const R od = (rw) * (R(3.0f) * cu_);                             \
    const R gev = (-uDg + R(3.0f) * cu_ * cg_) * (R(1.0f) / (gd));      \
    const R god = cg_ * (R(1.0f) / (gd));                            \
    const R fgp = gev + god, fgm = gev - god;                     \
    d[qp] = ((ev + od) - f[qp]) - R(0.5f) * fgp;                         \
    d[qm] = ((ev - od) - f[qm]) - R(0.5f) * fgm;                         \
    base[qp] = f[qp] + fgp;                                           \
    base[qm] = f[qm] + fgm;                                           \
  }
  PAIR(1, 2, ux, gx, r1, R(6.0f))
  PAIR(3, 4, uy, gy, r1, R(6.0f))
  PAIR(5, 6, uz, gz, r1, R(6.0f))
  PAIR(7, 12, ux + uy, gx + gy, r2, R(12.0f))
  PAIR(8, 11, ux - uy, gx - gy, r2, R(12.0f))
  PAIR(9, 14, ux + uz, gx + gz, r2, R(12.0f))
  PAIR(10, 13, ux - uz, gx - gz, r2, R(12.0f))
  PAIR(15, 18, uy + uz, gy + gz, r2, R(12.0f))
  PAIR(16, 17, uy - uz, gy - gz, r2, R(12.0f))
#undef PAIR

  // Forward transform of d (non-conserved rows only), butterfly form.
  const R Ax = d[1] + d[2], Bx = d[1] - d[2];
  const R Ay = d[3] + d[4], By = d[3] - d[4];
  const R Az = d[5] + d[6], Bz = d[5] - d[6];
  R Sxy, Xxy, Yxy, Pxy, Sxz, Xxz, Zxz, Pxz, Syz, Yyz, Zyz, Pyz;
  {
    R a = d[7] + d[8], b = d[11] + d[12], c = d[7] - d[8], e = d[11] - d[12];
    Sxy = a + b; Xxy = a - b; Yxy = c + e; Pxy = c - e;
  }
  {
    R a = d[9] + d[10], b = d[13] + d[14], c = d[9] - d[10], e = d[13] - d[14];
    Sxz = a + b; Xxz = a - b; Zxz = c + e; Pxz = c - e;
  }
  {
    R a = d[15] + d[16], b = d[17] + d[18], c = d[15] - d[16], e = d[17] - d[18];
    Syz = a + b; Yyz = a - b; Zyz = c + e; Pyz = c - e;
  }
  const R A = Ax + Ay + Az, S = Sxy + Sxz + Syz;
  const R m1 = -R(30.0f) * d[0] - R(11.0f) * A + R(8.0f) * S;
  const R m2 = R(12.0f) * d[0] - R(4.0f) * A + S;
  const R m3 = Bx + Xxy + Xxz;
  const R m5 = By + Yxy + Yyz;
  const R m7 = Bz + Zxz + Zyz;
  const R m4 = -R(4.0f) * Bx + Xxy + Xxz;
  const R m6 = -R(4.0f) * By + Yxy + Yyz;
  const R m8 = -R(4.0f) * Bz + Zxz + Zyz;
  const R T9 = Sxy + Sxz - R(2.0f) * Syz;
  const R m9 = R(2.0f) * Ax - Ay - Az + T9;
  const R m10 = -R(4.0f) * Ax + R(2.0f) * Ay + R(2.0f) * Az + T9;
  const R T11 = Sxy - Sxz;
  const R m11 = Ay - Az + T11;
  const R m12 = -R(2.0f) * Ay + R(2.0f) * Az + T11;
  const R m13 = Pxy, m14 = Pyz, m15 = Pxz;
  const R m16 = Xxy - Xxz, m17 = Yyz - Yxy, m18 = Zxz - Zyz;

  // Rates.
  R s1, s2, s4, s6, s11, s12, s13, s16;
  if (COLL == 0) {
    s1 = R(1.19f); s2 = R(1.40f); s4 = R(1.20f); s6 = R(1.20f); s11 = R(1.20f); s12 = R(1.40f); s13 = R(1.40f); s16 = R(1.98f);
  }

  if (VISC > 0 || (VISC < 0 && p.variable)) {
    // Strain rate from the relaxed non-equilibrium moments with tau(t-1)
    // (GPU_program.cl:459-562): the second moments of M^-1 S_old M d, which
    // only rows e, 3pxx, pww and the off-diagonal p carry.
    const R it = RMath<R>::rcp(tau);
    R a1, a9, a11, a13, a14, a15;
    if (COLL == 0) {
      a1 = s1 * m1 * INV_N1; a9 = it * m9 * INV_N9; a11 = s11 * m11 * INV_N11;
      a13 = s13 * m13 * INV_N13; a14 = it * m14 * INV_N13; a15 = it * m15 * INV_N13;
    } else {
      a1 = it * m1 * INV_N1; a9 = it * m9 * INV_N9; a11 = it * m11 * INV_N11;
      a13 = it * m13 * INV_N13; a14 = it * m14 * INV_N13; a15 = it * m15 * INV_N13;
    }
    const R sxx = R(42.0f) * a1 + R(12.0f) * a9;
    const R syy = R(42.0f) * a1 - R(6.0f) * a9 + R(6.0f) * a11;
    const R szz = R(42.0f) * a1 - R(6.0f) * a9 - R(6.0f) * a11;
    const R sxy = R(4.0f) * a13, syz = R(4.0f) * a14, sxz = R(4.0f) * a15;
    const R ss = sxx * sxx + R(2.0f) * (sxy * sxy + sxz * sxz + syz * syz) + syy * syy + szz * szz;
    const R srt = RMath<R>::sqrt(ss) * R(2.1213203f) * ir;
    tau = compute_tau<VISC, R>(p, srt, clamped);
  }

  const R it = RMath<R>::rcp(tau);
  R a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14, a15, a16, a17, a18;
  if (COLL == 0) {
    a3 = INV_N3 * m3; a5 = INV_N3 * m5; a7 = INV_N3 * m7;
    a1 = s1 * INV_N1 * m1; a2 = s2 * INV_N2 * m2; a4 = s4 * INV_N4 * m4; a6 = s6 * INV_N4 * m6;
    a8 = it * INV_N4 * m8; a9 = it * INV_N9 * m9; a10 = it * INV_N10 * m10; a11 = s11 * INV_N11 * m11;
    a12 = s12 * INV_N12 * m12; a13 = s13 * INV_N13 * m13; a14 = it * INV_N13 * m14; a15 = it * INV_N13 * m15;
    a16 = s16 * INV_N16 * m16; a17 = s16 * INV_N16 * m17; a18 = s16 * INV_N16 * m18;
  } else {
    a3 = it * INV_N3 * m3; a5 = it * INV_N3 * m5; a7 = it * INV_N3 * m7;
    a1 = it * INV_N1 * m1; a2 = it * INV_N2 * m2; a4 = it * INV_N4 * m4; a6 = it * INV_N4 * m6;
    a8 = it * INV_N4 * m8; a9 = it * INV_N9 * m9; a10 = it * INV_N10 * m10; a11 = it * INV_N11 * m11;
    a12 = it * INV_N12 * m12; a13 = it * INV_N13 * m13; a14 = it * INV_N13 * m14; a15 = it * INV_N13 * m15;
    a16 = it * INV_N16 * m16; a17 = it * INV_N16 * m17; a18 = it * INV_N16 * m18;
  }

  // Inverse transform M^T a, butterfly form.
  f[0] = base[0] + (-R(30.0f) * a1 + R(12.0f) * a2);
  const R bax = -R(11.0f) * a1 - R(4.0f) * a2;
  const R Cx = bax + R(2.0f) * a9 - R(4.0f) * a10;
  const R Cy = bax - a9 + R(2.0f) * a10 + a11 - R(2.0f) * a12;
  const R Cz = bax - a9 + R(2.0f) * a10 - a11 + R(2.0f) * a12;
  const R Ox = a3 - R(4.0f) * a4, Oy = a5 - R(4.0f) * a6, Oz = a7 - R(4.0f) * a8;
  f[1] = base[1] + (Cx + Ox);
  f[2] = base[2] + (Cx - Ox);
  f[3] = base[3] + (Cy + Oy);
  f[4] = base[4] + (Cy - Oy);
  f[5] = base[5] + (Cz + Oz);
  f[6] = base[6] + (Cz - Oz);
  const R bd = R(8.0f) * a1 + a2;
  {  // xy: 7 (+,+) 8 (+,-) 11 (-,+) 12 (-,-)
    const R E = bd + a9 + a10 + a11 + a12, X = a3 + a4 + a16, Y = a5 + a6 - a17, P = a13;
    const R u1 = E + P, u2 = E - P, v1 = X + Y, v2 = X - Y;
    f[7] = base[7] + (u1 + v1); f[12] = base[12] + (u1 - v1);
    f[8] = base[8] + (u2 + v2); f[11] = base[11] + (u2 - v2);
  }
  {  // xz: 9 (+,+) 10 (+,-) 13 (-,+) 14 (-,-)
    const R E = bd + a9 + a10 - a11 - a12, X = a3 + a4 - a16, Z = a7 + a8 + a18, P = a15;
    const R u1 = E + P, u2 = E - P, v1 = X + Z, v2 = X - Z;
    f[9] = base[9] + (u1 + v1); f[14] = base[14] + (u1 - v1);
    f[10] = base[10] + (u2 + v2); f[13] = base[13] + (u2 - v2);
  }
  {  // yz: 15 (+,+) 16 (+,-) 17 (-,+) 18 (-,-)
    const R E = bd - R(2.0f) * a9 - R(2.0f) * a10, Y = a5 + a6 + a17, Z = a7 + a8 - a18, P = a14;
    const R u1 = E + P, u2 = E - P, v1 = Y + Z, v2 = Y - Z;
    f[15] = base[15] + (u1 + v1); f[18] = base[18] + (u1 - v1);
    f[16] = base[16] + (u2 + v2); f[17] = base[17] + (u2 - v2);
  }
}

// ---------------------------------------------------------------------------
// Spread force of one tile: accumulate -w*F of every listed marker on the
// tile plus a one-node halo (the reference's gpf slot sum, GPU_program.cl:
// 210-227 and 258-289) in fixed point, then convert to float.  The 64-bit
// accumulators and the float field share the storage: the field replaces the
// sums once they are complete.
struct __align__(16) SpreadSmem {
  union {
    unsigned long long acc[3][HALO_N];  // fixed-point sums: lo parts (low word), hi parts (high word)
    float g[3][HALO_N];                 // the spread force of the halo nodes
    double g64[3][HALO_N];              // the same in the FP64 build
  };
};
template <typename R>
__device__ __forceinline__ R* halo_field(SpreadSmem& s);
template <>
__device__ __forceinline__ float* halo_field<float>(SpreadSmem& s) { return &s.g[0][0]; }
template <>
__device__ __forceinline__ double* halo_field<double>(SpreadSmem& s) { return &s.g64[0][0]; }
static_assert((3 * HALO_N) % 2 == 0, "the sums are cleared sixteen bytes at a time");
constexpr int SPREAD_CONVERT_PER_THREAD = (3 * HALO_N + FLUID_THREADS - 1) / FLUID_THREADS;

__device__ __forceinline__ void marker_weights(float wx, float wy, float wz, float (&w)[8]) {
  // GPU_program.cl:170-178.
  w[0] = wx * wy * wz;
  w[1] = (1.0f - wx) * wy * wz;
  w[2] = wx * (1.0f - wy) * wz;
  w[3] = wx * wy * (1.0f - wz);
  w[4] = (1.0f - wx) * (1.0f - wy) * wz;
  w[5] = (1.0f - wx) * wy * (1.0f - wz);
  w[6] = wx * (1.0f - wy) * (1.0f - wz);
  w[7] = (1.0f - wx) * (1.0f - wy) * (1.0f - wz);
}

__device__ __forceinline__ void decode_marker(const float4& a, const float4& b, int& x0, int& y0, int& z0) {
  const unsigned xy = __float_as_uint(a.w);
  x0 = (int)(xy & 0xffffu);
  y0 = (int)(xy >> 16);
  z0 = (int)__float_as_uint(b.w);
}

// Fixed-point unit of the step whose markers are listed, as a power of two
// 2^k with max|force| * 2^k < 2^FIX_BITS.
__device__ __forceinline__ int fixed_exponent(unsigned fmax_bits) {
  const float fm = __uint_as_float(fmax_bits);
  if (!(fm > 0.0f)) return 0;
  int e;
  frexpf(fm, &e);  // fm < 2^e
  return FIX_BITS - e;
}

// Accumulates the tile's n listed markers into s (X0,Y0,Z0 = tile origin)
// and leaves the halo's spread force in s.g.  Thread t takes list entries
// t, t + FLUID_THREADS, ...; its first entry (first_id, loaded by the caller
// ahead of time) is used when t < n.  Every contribution -w*F (the
// reference's "gpf -= weights[n]*vuForce", GPU_program.cl:222-224) is scaled
// by 2^k (exact), rounded to an integer v = hi*2^16 + lo (0 <= lo < 2^16) and
// the two parts are summed exactly with 32-bit atomics, lo in the low word and
// hi in the high word of the node's 64-bit slot; each sum is converted back
// with one rounding.  Needs all FLUID_THREADS threads.
template <typename R = float>
__device__ void accumulate_tile(SpreadSmem& s, const Geom& g, const TileLists& tl, long long T, int n, int X0,
                                int Y0, int Z0, int tid, int k, int first_id, unsigned* err) {
  float4 ma = make_float4(0.f, 0.f, 0.f, 0.f), mb = ma;
  if (tid < n && !out_of_bounds(first_id, tl.markers, err)) {  // issued before the clear: the round trip overlaps it
    ma = tl.mrec[2 * (long long)first_id];
    mb = tl.mrec[2 * (long long)first_id + 1];
  }
  {
    int4* z4 = reinterpret_cast<int4*>(&s.acc[0][0]);
    for (int h = tid; h < 3 * HALO_N / 2; h += FLUID_THREADS) z4[h] = make_int4(0, 0, 0, 0);
  }
  __syncthreads();
  const float scale = ldexpf(1.0f, k);
  for (int j = tid; j < n; j += FLUID_THREADS) {
    float4 a = ma, b = mb;
    if (j != tid) {
      const int m = tl.list[T * tl.cap + j];
      if (out_of_bounds(m, tl.markers, err)) continue;
      a = tl.mrec[2 * (long long)m];
      b = tl.mrec[2 * (long long)m + 1];
    }
    int x0, y0, z0;
    decode_marker(a, b, x0, y0, z0);
    const int xs = (x0 == g.Nx - 2) ? -(g.Nx - 3) : 1;
    const int ys = (y0 == g.Ny - 2) ? -(g.Ny - 3) : 1;
    const int zs = (z0 == g.Nz - 2) ? -(g.Nz - 3) : 1;
    float w[8];
    marker_weights(a.x, a.y, a.z, w);
    const int sh[8][3] = {{0, 0, 0}, {xs, 0, 0}, {0, ys, 0}, {0, 0, zs}, {xs, ys, 0}, {xs, 0, zs}, {0, ys, zs},
                          {xs, ys, zs}};
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int hx = x0 + sh[q][0] - (X0 - 1), hy = y0 + sh[q][1] - (Y0 - 1), hz = z0 + sh[q][2] - (Z0 - 1);
      if (hx < 0 || hx >= HALO_X || hy < 0 || hy >= HALO_Y || hz < 0 || hz >= HALO_Z) continue;
      const int h = hx + HALO_X * (hy + HALO_Y * hz);
      const float c[3] = {w[q] * b.x, w[q] * b.y, w[q] * b.z};
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const float sv = -c[d] * scale;  // exact: power-of-two scaling
        if (!(fabsf(sv) < 549755813888.0f)) {  // 2^39
          atomicOr(err, ERR_FIXED_RANGE);
          continue;
        }
        const long long v = __float2ll_rn(sv);
        unsigned* slot = reinterpret_cast<unsigned*>(&s.acc[d][h]);
        atomicAdd(slot, (unsigned)(v & 0xffff));
        atomicAdd(reinterpret_cast<int*>(slot + 1), (int)(v >> 16));
      }
    }
  }
  __syncthreads();
  // value = (hi * 2^16 + lo) * 2^-k, both parts scaled exactly by powers of
  // two and joined with one rounding (exactly in FP64).  All sums are read
  // before the field overwrites them.
  const float inv = ldexpf(1.0f, -k), inv_hi = ldexpf(1.0f, 16 - k);
  const double inv64 = ldexp(1.0, -k), inv_hi64 = ldexp(1.0, 16 - k);
  R v[SPREAD_CONVERT_PER_THREAD];
#pragma unroll
  for (int r = 0; r < SPREAD_CONVERT_PER_THREAD; r++) {
    const int h = tid + r * FLUID_THREADS;
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
  for (int r = 0; r < SPREAD_CONVERT_PER_THREAD; r++) {
    const int h = tid + r * FLUID_THREADS;
    if (h < 3 * HALO_N) field[h] = v[r];
  }
  __syncthreads();
}

// Smoothed spread force of the tile's 32x4x4 nodes: the reference's
// 27-point stencil (weights 1/4, 1/2, 1/4 per axis; GPU_program.cl:356-377)
// over the halo field s.g.  Each thread takes two consecutive z-planes, so the
// 9-point x-y sums of the two middle halo planes are shared between its nodes.
template <typename R>
__device__ __forceinline__ void smooth_pair(SpreadSmem& s, int tx, int ty, int tz, R (&sg)[2][3]) {
  const int hx = tx + 1, hy = ty + 1, hz0 = 2 * tz;
  const R* gf = halo_field<R>(s);
#pragma unroll
  for (int pl = 0; pl < 4; pl++) {
    R px = R(0), py = R(0), pz = R(0);
#pragma unroll
    for (int sy = -1; sy <= 1; sy++)
#pragma unroll
      for (int sx = -1; sx <= 1; sx++) {
        const R ws = R(sx == 0 ? 0.5f : 0.25f) * R(sy == 0 ? 0.5f : 0.25f);
        const int h = (hx + sx) + HALO_X * ((hy + sy) + HALO_Y * (hz0 + pl));
        px += ws * gf[h];
        py += ws * gf[HALO_N + h];
        pz += ws * gf[2 * HALO_N + h];
      }
    const R w0 = R(pl == 0 ? 0.25f : (pl == 1 ? 0.5f : (pl == 2 ? 0.25f : 0.0f)));
    const R w1 = R(pl == 0 ? 0.0f : (pl == 1 ? 0.25f : (pl == 2 ? 0.5f : 0.25f)));
    if (pl < 3) {
      sg[0][0] += w0 * px; sg[0][1] += w0 * py; sg[0][2] += w0 * pz;
    }
    if (pl > 0) {
      sg[1][0] += w1 * px; sg[1][1] += w1 * py; sg[1][2] += w1 * pz;
    }
  }
}

// Boundary layouts of the collide-stream kernel, fixed at compile time.
constexpr int BC_GENERIC = 0;  // any combination the context accepts
constexpr int BC_ZWALL = 1;    // periodic x and y, velocity walls on z, no tangential boundaries

// Dynamic shared memory of the collide-stream kernel: the spread halo of the
// tile when there are spheres.
__host__ __device__ constexpr size_t fluid_smem_bytes(bool ibm) { return ibm ? sizeof(SpreadSmem) : 0; }

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
                         a.err);
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

// The collide-stream pass of many independent lattices in one persistent
// launch: CTA b takes work items b, b + gridDim.x, ... of the packed list
// work[k] = {slot, tile} (*nwork items).  slots[2*s + parity] holds lattice
// s's arguments for steps of that buffer parity.  The reference's MRT rates,
// periodic x/y with z walls, and each lattice's own viscosity law.
// AA: the pool's layout for this step (every member of a pool shares it and
// sits at the same phase).
template <typename ST, int AA>
__global__ void __launch_bounds__(FLUID_THREADS, sizeof(ST) == 4 ? (AA ? FLUID_MIN_BLOCKS_AA_F32 : FLUID_MIN_BLOCKS_F32)
                                                                 : FLUID_MIN_BLOCKS)
    fluid_batch_kernel(const FluidArgs* __restrict__ slots, const int2* __restrict__ work,
                       const int* __restrict__ nwork, const int parity) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SpreadSmem& sm = *reinterpret_cast<SpreadSmem*>(smem_raw);
  const int n = *nwork;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const int2 it = work[w];
    const FluidArgs& a = slots[2 * it.x + parity];
    const int ntx = a.g.ntx, nty = a.g.nty;
    const int bx = it.y % ntx, by = (it.y / ntx) % nty, bz = it.y / (ntx * nty);
    fluid_tile<0, -1, BC_ZWALL, ST, AA>(a, 0, bx, by, bz, sm);
    __syncthreads();  // the spread halo is reused by the next item
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

// Distinct tile indices covering two node coordinates (at most 4).
__device__ __forceinline__ int tile_set(int c0, int c1, int T, int nt, int (&out)[4]) {
  int l0, h0, l1, h1, n = 0;
  tile_range(c0, T, nt, l0, h0);
  tile_range(c1, T, nt, l1, h1);
  for (int t = l0; t <= h0 && n < 4; t++) out[n++] = t;
  for (int t = l1; t <= h1 && n < 4; t++) {
    bool dup = false;
    for (int j = 0; j < n; j++) dup |= out[j] == t;
    if (!dup) out[n++] = t;
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
    // The marker template above is constant; the rigid-body update reads the
    // contact forces of the side stream's pass, so it waits too.
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
        nx = tile_set(x0, x0 + xs, TILE_X, g.ntx, tx);
        ny = tile_set(y0, y0 + ys, TILE_Y, g.nty, ty);
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
      nx = tile_set(x0, x0 + xs, TILE_X, g.ntx, tx);
      ny = tile_set(y0, y0 + ys, TILE_Y, g.nty, ty);
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
