// d3q19_device.cuh -- device helpers shared by the collide-stream kernels
// (d3q19_kernels.cu) and the TMA-pipelined collide-stream kernel
// (d3q19_tma.cu): storage forms, the wet-node velocity boundary, the local
// relaxation time, the pull gathers, the MRT collision and the tile spread of
// the IBM force.  Not part of the public interface.
#pragma once
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
  // rho/36 is rho/18 halved: a power-of-two scaling commutes with rounding,
  // so it is the correctly rounded rho/36 without a second division.
  const R r0 = rho / R(3.0f), r1 = rho / R(18.0f), r2 = R(0.5f) * r1;
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
// With periodic smoothing, the image of stencil node c on the periodic
// buffer layer that the smoothing of its neighbours across the seam reads:
// node N-2 also at 0, node 1 also at N-1; -1 for every other node.
__device__ __forceinline__ int seam_image(int c, int N, bool wrap) {
  return !wrap ? -1 : (c == N - 2 ? 0 : (c == 1 ? N - 1 : -1));
}

// Adds the fixed-point contribution c (already scaled by 2^k) of one stencil
// node at halo coordinates (hx, hy, hz), if they lie in the halo.
__device__ __forceinline__ void spread_add(SpreadSmem& s, int hx, int hy, int hz, const float (&c)[3], float scale,
                                           unsigned* err) {
  if (hx < 0 || hx >= HALO_X || hy < 0 || hy >= HALO_Y || hz < 0 || hz >= HALO_Z) return;
  const int h = hx + HALO_X * (hy + HALO_Y * hz);
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

// Adds a stencil node (cx, cy, cz) of a marker to the tile's halo: the node
// itself, and with periodic smoothing (wrap) its images on the periodic x/y
// buffer layers.
__device__ __forceinline__ void spread_node(SpreadSmem& s, const Geom& g, int cx, int cy, int cz, int X0, int Y0,
                                            int Z0, bool wrap, const float (&c)[3], float scale, unsigned* err) {
  const int hx = cx - (X0 - 1), hy = cy - (Y0 - 1), hz = cz - (Z0 - 1);
  spread_add(s, hx, hy, hz, c, scale, err);
  if (!wrap) return;
  const int ix = seam_image(cx, g.Nx, g.periodic[0] != 0), iy = seam_image(cy, g.Ny, g.periodic[1] != 0);
  if (ix >= 0) spread_add(s, ix - (X0 - 1), hy, hz, c, scale, err);
  if (iy >= 0) spread_add(s, hx, iy - (Y0 - 1), hz, c, scale, err);
  if (ix >= 0 && iy >= 0) spread_add(s, ix - (X0 - 1), iy - (Y0 - 1), hz, c, scale, err);
}

template <typename R = float>
__device__ void accumulate_tile(SpreadSmem& s, const Geom& g, const TileLists& tl, long long T, int n, int X0,
                                int Y0, int Z0, int tid, int k, int first_id, unsigned* err, bool wrap = false) {
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
      const float c[3] = {w[q] * b.x, w[q] * b.y, w[q] * b.z};
      spread_node(s, g, x0 + sh[q][0], y0 + sh[q][1], z0 + sh[q][2], X0, Y0, Z0, wrap, c, scale, err);
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

}  // namespace d3q19
