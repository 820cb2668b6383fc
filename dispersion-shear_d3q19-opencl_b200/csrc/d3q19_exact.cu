// d3q19_exact.cu -- the reference-exact collide-stream kernel (arithmetic = 1).
//
// Compiled with --fmad=false: every float operation is evaluated separately
// and in the order of the reference's expressions (GPU_program.cl:316-624,
// 978-1128), so that, from the same state, the kernel reproduces the
// reference's floating-point results bit for bit (sqrt and division are
// correctly rounded on both sides; pow() is not, see compute_tau_ref).
//
// The force field is likewise the reference's: per node, the spread
// contributions of the markers in marker order go round-robin into
// MaxSurfPointsPerNode slots that are then summed in slot order (the serial
// semantics of GPU_program.cl:210-227 and 258-289), and the 27-point
// smoothing adds the stencil terms in the reference's loop order.
#include "d3q19_internal.h"

#include <cuda_runtime.h>
#include <math.h>

namespace d3q19 {

#define CXQ(q) (((q) == 1 || (q) == 7 || (q) == 8 || (q) == 9 || (q) == 10) ? 1 : \
                (((q) == 2 || (q) == 11 || (q) == 12 || (q) == 13 || (q) == 14) ? -1 : 0))
#define CYQ(q) (((q) == 3 || (q) == 7 || (q) == 11 || (q) == 15 || (q) == 16) ? 1 : \
                (((q) == 4 || (q) == 8 || (q) == 12 || (q) == 17 || (q) == 18) ? -1 : 0))
#define CZQ(q) (((q) == 5 || (q) == 9 || (q) == 13 || (q) == 15 || (q) == 17) ? 1 : \
                (((q) == 6 || (q) == 10 || (q) == 14 || (q) == 16 || (q) == 18) ? -1 : 0))
#define CAQ(A, q) ((A) == 0 ? CXQ(q) : ((A) == 1 ? CYQ(q) : CZQ(q)))
#define SQQ(q) (CXQ(q) * CXQ(q) + CYQ(q) * CYQ(q) + CZQ(q) * CZQ(q))

// Moment basis entry M[k][q] in the reference's row order (GPU_program.cl:
// 410-428), as integer expressions of the velocity components.
__host__ __device__ constexpr int Mkq(int k, int q) {
  const int x = CXQ(q), y = CYQ(q), z = CZQ(q), s = SQQ(q);
  const int p = 2 * x * x - y * y - z * z, w = y * y - z * z;
  switch (k) {
    case 0: return 1;
    case 1: return s == 0 ? -30 : (s == 1 ? -11 : 8);
    case 2: return s == 0 ? 12 : (s == 1 ? -4 : 1);
    case 3: return x;
    case 4: return s == 1 ? -4 * x : x;
    case 5: return y;
    case 6: return s == 1 ? -4 * y : y;
    case 7: return z;
    case 8: return s == 1 ? -4 * z : z;
    case 9: return p;
    case 10: return s == 1 ? -2 * p : p;
    case 11: return w;
    case 12: return s == 1 ? -2 * w : w;
    case 13: return x * y;
    case 14: return y * z;
    case 15: return x * z;
    case 16: return x * (y * y - z * z);
    case 17: return y * (z * z - x * x);
    default: return z * (x * x - y * y);
  }
}
__host__ __device__ constexpr int Nk(int k) {
  return k == 0 ? 19 : k == 1 ? 2394 : k == 2 ? 252 : (k == 3 || k == 5 || k == 7) ? 10 :
         (k == 4 || k == 6 || k == 8) ? 40 : k == 9 ? 36 : k == 10 ? 72 : k == 11 ? 12 : k == 12 ? 24 :
         k <= 15 ? 4 : 8;
}
// Inverse transform coefficient M^-1[q][k] = M[k][q] / |row k|^2 rounded to
// float: equal to the reference's decimal literals (GPU_program.cl:473-491).
__host__ __device__ constexpr float Minv(int q, int k) { return (float)((double)Mkq(k, q) / (double)Nk(k)); }

// f_eq (GPU_program.cl:978-1007).
__device__ __forceinline__ void feq_ref(float (&fe)[19], float rho, float ux, float uy, float uz) {
  const float usq = ux * ux + uy * uy + uz * uz;
  fe[0] = (rho / 3.0f) * (1.0f - 1.5f * usq);
#pragma unroll
  for (int q = 1; q < 19; q++) {
    const int cx = CXQ(q), cy = CYQ(q), cz = CZQ(q);
    // c.u as the reference writes it: (+-u_a +- u_b), first component first
    float cu;
    if (cx != 0) {
      cu = cx > 0 ? ux : -ux;
      if (cy != 0) cu = cy > 0 ? cu + uy : cu - uy;
      if (cz != 0) cu = cz > 0 ? cu + uz : cu - uz;
    } else if (cy != 0) {
      cu = cy > 0 ? uy : -uy;
      if (cz != 0) cu = cz > 0 ? cu + uz : cu - uz;
    } else {
      cu = cz > 0 ? uz : -uz;
    }
    const float W = q < 7 ? 18.0f : 36.0f;
    fe[q] = (rho / W) * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * usq);
  }
}

// Guo term (GPU_program.cl:1010-1038).
__device__ __forceinline__ void guo_ref(float (&fg)[19], float ux, float uy, float uz, float gx, float gy, float gz) {
  const float uDg = ux * gx + uy * gy + uz * gz;
  fg[0] = -uDg;
#pragma unroll
  for (int q = 1; q < 19; q++) {
    const int cx = CXQ(q), cy = CYQ(q), cz = CZQ(q);
    float cu, cg;
    if (q < 7) {
      // ( +-g_a - uDg + 3 u_a g_a )/6
      const float ua = cx ? ux : (cy ? uy : uz), ga = cx ? gx : (cy ? gy : gz);
      const int sgn = cx + cy + cz;
      cg = sgn > 0 ? ga : -ga;
      fg[q] = (cg - uDg + 3.0f * ua * ga) / 6.0f;
      continue;
    }
    if (cx != 0) {
      cu = cx > 0 ? ux : -ux;
      cg = cx > 0 ? gx : -gx;
      if (cy != 0) {
        cu = cy > 0 ? cu + uy : cu - uy;
        cg = cy > 0 ? cg + gy : cg - gy;
      } else {
        cu = cz > 0 ? cu + uz : cu - uz;
        cg = cz > 0 ? cg + gz : cg - gz;
      }
    } else {
      cu = cy > 0 ? uy : -uy;
      cg = cy > 0 ? gy : -gy;
      cu = cz > 0 ? cu + uz : cu - uz;
      cg = cz > 0 ? cg + gz : cg - gz;
    }
    fg[q] = (cg - uDg + 3.0f * cu * cg) / 12.0f;
  }
}

// m[k] = sum_q M[k][q] v[q], terms in increasing q, zero coefficients
// skipped (GPU_program.cl:411-449).
template <int K>
__device__ __forceinline__ float moment_k(const float (&v)[19]) {
  float acc = 0.0f;
  bool first = true;
#pragma unroll
  for (int q = 0; q < 19; q++) {
    const int c = Mkq(K, q);
    if (c == 0) continue;
    const float t = (c == 1) ? v[q] : (c == -1 ? -v[q] : (float)c * v[q]);
    if (first) {
      acc = t;
      first = false;
    } else {
      acc = (c == -1) ? acc - v[q] : (c < 0 ? acc - (float)(-c) * v[q] : acc + t);
    }
  }
  return acc;
}

template <int K = 0>
__device__ __forceinline__ void moments(float (&m)[19], const float (&v)[19]) {
  m[K] = moment_k<K>(v);
  if constexpr (K < 18) moments<K + 1>(m, v);
}

// out[q] = sum_k Minv[q][k] sm[k] (GPU_program.cl:473-513): the k = 0 term
// first, then the non-zero terms in increasing k.
template <int Q>
__device__ __forceinline__ float back_q(const float (&sm)[19]) {
  float acc = Minv(Q, 0) * sm[0];
#pragma unroll
  for (int k = 1; k < 19; k++) {
    const float c = Minv(Q, k);
    if (c == 0.0f) continue;
    acc = c < 0.0f ? acc - (-c) * sm[k] : acc + c * sm[k];
  }
  return acc;
}
template <int Q = 0>
__device__ __forceinline__ void back(float (&out)[19], const float (&sm)[19]) {
  out[Q] = back_q<Q>(sm);
  if constexpr (Q < 18) back<Q + 1>(out, sm);
}

// compute_tau (GPU_program.cl:1041-1128).  sqrt and division are correctly
// rounded here and in the reference; pow() is not correctly rounded in
// either library, so power-law and Herschel-Bulkley exponents other than
// 0.5, 1 and 2 can differ in the last bit.
__device__ __forceinline__ float compute_tau_ref(const FluidParams& p, float srt, bool& clamped) {
  float tau = p.tauN;
  if (p.viscModel == 2) {
    float k = p.visc[0], n = p.visc[1], nu;
    srt = srt > 1E-8 ? srt : (float)1E-8;
    if (n == 0.5f) nu = k / sqrtf(srt);
    else if (n == 1.0f) nu = k;
    else if (n == 2.0f) nu = k * srt;
    else nu = k * (float)pow((double)srt, (double)(n - 1.0f));
    tau = 3.0f * nu + 0.5f;
  } else if (p.viscModel == 4) {
    float tY = p.visc[0], eta = p.visc[1];
    srt = srt > 1E-8 ? srt : (float)1E-8;
    const float a = sqrtf(tY / srt) + sqrtf(eta);
    const float b = sqrtf(tY / srt) + sqrtf(eta);
    tau = 3.0f * (a * b) + 0.5f;
  } else if (p.viscModel == 3) {
    float tY = p.visc[0], k = p.visc[1], n = p.visc[2], nu;
    srt = srt > 1E-8 ? srt : (float)1E-8;
    if (n == 0.5f) nu = tY / srt + k / sqrtf(srt);
    else if (n == 1.0f) nu = tY / srt + k;
    else if (n == 2.0f) nu = tY / srt + k * srt;
    else nu = tY / srt + k * (float)pow((double)srt, (double)(n - 1.0f));
    tau = 3.0f * nu + 0.5f;
  } else {
    return tau;
  }
  if ((double)tau < 0.505) {
    tau = 0.505f;
    clamped = true;
  }
  return tau;
}

// The reference's collision for one node (GPU_program.cl:385-623).
template <bool VAR>
__device__ __forceinline__ void collide_ref(float (&f)[19], float rho, float ux, float uy, float uz, float gx, float gy,
                                            float gz, float& tau, const FluidParams& p, bool& clamped) {
  float fe[19], n[19], fg[19], mn[19], mg[19];
  feq_ref(fe, rho, ux, uy, uz);
#pragma unroll
  for (int q = 0; q < 19; q++) n[q] = fe[q] - f[q];
  guo_ref(fg, ux, uy, uz, gx, gy, gz);
  moments(mn, n);
  mn[0] = 0.0f;
  moments(mg, fg);
  float s[19] = {0.0f, 1.19f, 1.40f, 1.0f, 1.20f, 1.0f, 1.20f, 1.0f, 1.0f, 1.0f,
                 1.0f, 1.20f, 1.40f, 1.40f, 1.0f, 1.0f, 1.98f, 1.98f, 1.98f};
  float sm[19], msmn[19], msmg[19];
  if (VAR) {
    const float it = 1.0f / tau;
    s[8] = it; s[9] = it; s[10] = it; s[14] = it; s[15] = it;
#pragma unroll
    for (int k = 0; k < 19; k++) sm[k] = s[k] * mn[k];
    back(msmn, sm);
#pragma unroll
    for (int k = 0; k < 19; k++) sm[k] = s[k] * mg[k];
    back(msmg, sm);
    float ss[19];
#pragma unroll
    for (int q = 0; q < 19; q++) ss[q] = msmn[q] + fg[q] - 0.5f * msmg[q];
    // Strain-rate tensor (GPU_program.cl:521-557).
    float s00 = ss[1] + ss[2] + ss[7] + ss[8] + ss[9] + ss[10] + ss[11] + ss[12] + ss[13] + ss[14];
    float s01 = ss[7] - ss[8] - ss[11] + ss[12];
    float s02 = ss[9] - ss[10] - ss[13] + ss[14];
    float s10 = s01;
    float s11 = ss[3] + ss[4] + ss[7] + ss[8] + ss[11] + ss[12] + ss[15] + ss[16] + ss[17] + ss[18];
    float s12 = ss[15] - ss[16] - ss[17] + ss[18];
    float s20 = s02, s21 = s12;
    float s22 = ss[5] + ss[6] + ss[9] + ss[10] + ss[13] + ss[14] + ss[15] + ss[16] + ss[17] + ss[18];
    s00 -= 2 * ux * gx;
    s01 -= (ux * gy + uy * gx);
    s02 -= (ux * gz + uz * gx);
    s10 -= (uy * gx + ux * gy);
    s11 -= 2 * uy * gy;
    s12 -= (uy * gz + uz * gy);
    s20 -= (uz * gx + ux * gz);
    s21 -= (uz * gy + uy * gz);
    s22 -= 2 * uz * gz;
    float srt = 0.0f;
    srt += s00 * s00; srt += s01 * s01; srt += s02 * s02;
    srt += s10 * s10; srt += s11 * s11; srt += s12 * s12;
    srt += s20 * s20; srt += s21 * s21; srt += s22 * s22;
    srt = (float)((double)sqrtf(srt) * 2.1213203 / (double)rho);
    tau = compute_tau_ref(p, srt, clamped);
  }
  const float it = 1.0f / tau;
  s[8] = it; s[9] = it; s[10] = it; s[14] = it; s[15] = it;
#pragma unroll
  for (int k = 0; k < 19; k++) sm[k] = s[k] * mn[k];
  back(msmn, sm);
#pragma unroll
  for (int k = 0; k < 19; k++) sm[k] = s[k] * mg[k];
  back(msmg, sm);
#pragma unroll
  for (int q = 0; q < 19; q++) f[q] = f[q] + msmn[q] + fg[q] - 0.5f * msmg[q];
}

// Velocity boundary, gather and wall handling, as in the fast kernel (pure
// copies and the reference's own BC arithmetic, which contains no product
// that could contract).
#define OPPQ(q) ((q) == 0 ? 0 : (q) <= 6 ? (((q) & 1) ? (q) + 1 : (q) - 1) : \
                 (q) == 7 ? 12 : (q) == 12 ? 7 : (q) == 8 ? 11 : (q) == 11 ? 8 : \
                 (q) == 9 ? 14 : (q) == 14 ? 9 : (q) == 10 ? 13 : (q) == 13 ? 10 : \
                 (q) == 15 ? 18 : (q) == 18 ? 15 : (q) == 16 ? 17 : 16)

template <int A, int SIDE>
__device__ __forceinline__ void velocity_bc_ref(float (&f)[19], const float* uw) {
  constexpr int IN = SIDE == 0 ? 1 : -1;
  constexpr int A1 = A == 0 ? 1 : 0;
  constexpr int A2 = A == 2 ? 1 : 2;
  float sum9 = 0.0f, sum5 = 0.0f;
#pragma unroll
  for (int q = 0; q < 19; q++) {
    if (CAQ(A, q) == 0) sum9 += f[q];
    else if (CAQ(A, q) == -IN) sum5 += f[q];
  }
  const float rho = 1.0f;
  const float un = 1.0f - (sum9 + 2.0f * sum5) / rho;
  const float ua1 = uw[A1], ua2 = uw[A2];
#pragma unroll
  for (int q = 1; q < 19; q++) {
    if (CAQ(A, q) != IN) continue;
    const int t1 = CAQ(A1, q), t2 = CAQ(A2, q);
    float v;
    if (t1 == 0 && t2 == 0) v = f[OPPQ(q)] + rho * un / 3.0f;
    else if (t1 != 0) v = f[OPPQ(q)] + rho * (t1 > 0 ? un + ua1 : un - ua1) / 6.0f;
    else v = f[OPPQ(q)] + rho * (t2 > 0 ? un + ua2 : un - ua2) / 6.0f;
    f[q] = v;
  }
}

__device__ __forceinline__ void wall_ref(float (&f)[19], int axis, int side, const FluidParams& p) {
  const float* uw = side ? p.velUpper : p.velLower;
  if (axis == 0) {
    if (side) velocity_bc_ref<0, 1>(f, uw); else velocity_bc_ref<0, 0>(f, uw);
  } else if (axis == 1) {
    if (side) velocity_bc_ref<1, 1>(f, uw); else velocity_bc_ref<1, 0>(f, uw);
  } else {
    if (side) velocity_bc_ref<2, 1>(f, uw); else velocity_bc_ref<2, 0>(f, uw);
  }
}

__device__ __forceinline__ void marker_weights_ref(float wx, float wy, float wz, float (&w)[8]) {
  w[0] = wx * wy * wz;
  w[1] = (1.0f - wx) * wy * wz;
  w[2] = wx * (1.0f - wy) * wz;
  w[3] = wx * wy * (1.0f - wz);
  w[4] = (1.0f - wx) * (1.0f - wy) * wz;
  w[5] = (1.0f - wx) * wy * (1.0f - wz);
  w[6] = wx * (1.0f - wy) * (1.0f - wz);
  w[7] = (1.0f - wx) * (1.0f - wy) * (1.0f - wz);
}

constexpr int EXACT_LIST = 2048;  // markers per tile the exact spread sorts in shared memory
constexpr int MAX_SLOTS = 16;     // MaxSurfPointsPerNode supported by the exact spread

struct ExactSmem {
  int ids[EXACT_LIST];
  float g[3][HALO_N];
};

// Spread force of the tile halo with the reference's serial slot semantics.
__device__ void exact_spread_tile(ExactSmem& s, const Geom& g, const TileLists& tl, long long T, int n, int X0, int Y0,
                                  int Z0, int tid, int nthreads, int slots, unsigned* err) {
  if (n > EXACT_LIST) {
    if (tid == 0) atomicOr(err, ERR_TILE_OVERFLOW);
    n = EXACT_LIST;
  }
  int npow = 1;
  while (npow < n) npow <<= 1;
  for (int k = tid; k < npow; k += nthreads) s.ids[k] = k < n ? tl.list[T * tl.cap + k] : 0x7fffffff;
  __syncthreads();
  // Bitonic sort of the marker ids (ascending = the reference's work-item
  // order, in which its atomic slot counter hands out slots).
  for (int size = 2; size <= npow; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int k = tid; k < npow; k += nthreads) {
        const int o = k ^ stride;
        if (o > k) {
          const bool up = (k & size) == 0;
          const int a = s.ids[k], b = s.ids[o];
          if ((a > b) == up) {
            s.ids[k] = b;
            s.ids[o] = a;
          }
        }
      }
      __syncthreads();
    }
  for (int h = tid; h < HALO_N; h += nthreads) {
    const int hx = h % HALO_X, hy = (h / HALO_X) % HALO_Y, hz = h / (HALO_X * HALO_Y);
    const int nx = X0 - 1 + hx, ny = Y0 - 1 + hy, nz = Z0 - 1 + hz;
    float slot[3][MAX_SLOTS];
    for (int j = 0; j < slots; j++) slot[0][j] = slot[1][j] = slot[2][j] = 0.0f;
    int cnt = 0;
    for (int r = 0; r < n; r++) {
      const int m = s.ids[r];
      const float4 a = tl.mrec[2 * (long long)m], b = tl.mrec[2 * (long long)m + 1];
      const unsigned xy = __float_as_uint(a.w);
      const int x0 = (int)(xy & 0xffffu), y0 = (int)(xy >> 16), z0 = (int)__float_as_uint(b.w);
      const int x1 = (x0 == g.Nx - 2) ? 1 : x0 + 1;
      const int y1 = (y0 == g.Ny - 2) ? 1 : y0 + 1;
      const int z1 = (z0 == g.Nz - 2) ? 1 : z0 + 1;
      const int ix = nx == x0 ? 0 : (nx == x1 ? 1 : -1);
      const int iy = ny == y0 ? 0 : (ny == y1 ? 1 : -1);
      const int iz = nz == z0 ? 0 : (nz == z1 ? 1 : -1);
      if (ix < 0 || iy < 0 || iz < 0) continue;
      // stencil index of the node (GPU_program.cl:164 shift table)
      const int code = ix | (iy << 1) | (iz << 2);
      const int qi = code == 0 ? 0 : code == 1 ? 1 : code == 2 ? 2 : code == 4 ? 3 : code == 3 ? 4 :
                     code == 5 ? 5 : code == 6 ? 6 : 7;
      float w[8];
      marker_weights_ref(a.x, a.y, a.z, w);
      const int j = cnt % slots;
      slot[0][j] -= w[qi] * b.x;
      slot[1][j] -= w[qi] * b.y;
      slot[2][j] -= w[qi] * b.z;
      cnt++;
    }
    for (int d = 0; d < 3; d++) {
      float acc = slot[d][0];
      for (int j = 1; j < slots; j++) acc += slot[d][j];
      s.g[d][h] = acc;
    }
  }
  __syncthreads();
}

template <bool FIRST, bool VAR>
__global__ void __launch_bounds__(FLUID_THREADS) fluid_exact_kernel(const FluidArgs a, int slots) {
  __shared__ ExactSmem sm;
  __shared__ int s_cnt;
  const Geom& g = a.g;
  const int tid = threadIdx.x + TILE_X * (threadIdx.y + TILE_Y * threadIdx.z);
  const int X0 = blockIdx.x * TILE_X, Y0 = blockIdx.y * TILE_Y, Z0 = blockIdx.z * TILE_Z;
  const long long T = blockIdx.x + (long long)g.ntx * (blockIdx.y + (long long)g.nty * blockIdx.z);
  int cnt = 0;
  if (a.has_ibm) {
    if (tid == 0) s_cnt = a.tiles.count[T];
    __syncthreads();
    cnt = s_cnt;
    if (T == 0 && tid == 0) a.tiles.fmax[a.t & 1] = 0u;
    if (cnt > 0) {
      __syncthreads();
      if (tid == 0) a.tiles.count[T] = 0;
      exact_spread_tile(sm, g, a.tiles, T, min(cnt, a.tiles.cap), X0, Y0, Z0, tid, FLUID_THREADS, slots, a.err);
    }
  }
  const int x = X0 + threadIdx.x, y = Y0 + threadIdx.y;
  const long long NC = g.NC;
  const float sten[3] = {0.25f, 0.5f, 0.25f};
  int nclamp = 0;
#pragma unroll 1
  for (int zz = 0; zz < TILE_Z / 2; zz++) {
    const int z = Z0 + threadIdx.z + 2 * zz;
    if (x < 1 || x > g.Nx - 2 || y < 1 || y > g.Ny - 2 || z < 1 || z > g.Nz - 2) continue;
    const long long i = x + (long long)g.Nx * (y + (long long)g.Ny * z);
    float f[19];
    if (FIRST) {
#pragma unroll
      for (int q = 0; q < 19; q++) f[q] = ((const float*)a.fin)[q * NC + i];
    } else {
      const int Nxy = g.Nx * g.Ny;
      const int dxm = (g.periodic[0] && x == 1) ? g.Nx - 3 : -1;
      const int dxp = (g.periodic[0] && x == g.Nx - 2) ? -(g.Nx - 3) : 1;
      const int dym = ((g.periodic[1] && y == 1) ? g.Ny - 3 : -1) * g.Nx;
      const int dyp = ((g.periodic[1] && y == g.Ny - 2) ? -(g.Ny - 3) : 1) * g.Nx;
      const int dzm = ((g.periodic[2] && z == 1) ? g.Nz - 3 : -1) * Nxy;
      const int dzp = ((g.periodic[2] && z == g.Nz - 2) ? -(g.Nz - 3) : 1) * Nxy;
#pragma unroll
      for (int q = 0; q < 19; q++) {
        const int cx = CXQ(q), cy = CYQ(q), cz = CZQ(q);
        const long long src = i + (cx == 1 ? dxm : (cx == -1 ? dxp : 0)) + (cy == 1 ? dym : (cy == -1 ? dyp : 0)) +
                              (cz == 1 ? dzm : (cz == -1 ? dzp : 0));
        f[q] = ((const float*)a.fin)[q * NC + src];
      }
      if (g.wallAxis >= 0) {
        const int c[3] = {x, y, z}, N[3] = {g.Nx, g.Ny, g.Nz};
        const int w = g.wallAxis;
        if (c[w] == 1) wall_ref(f, w, 0, a.p);
        else if (c[w] == N[w] - 2) wall_ref(f, w, 1, a.p);
        for (int t = 0; t < 3; t++) {
          if (!g.tanBC[t]) continue;
          if (c[t] == 1) wall_ref(f, t, 0, a.p);
          else if (c[t] == N[t] - 2) wall_ref(f, t, 1, a.p);
        }
      }
    }
    float rho = 0.0f;
#pragma unroll
    for (int q = 0; q < 19; q++) rho += f[q];
    float gx = a.p.g[0], gy = a.p.g[1], gz = a.p.g[2];
    if (a.has_ibm) {
      // 27-point smoothing in the reference's loop order (GPU_program.cl:
      // 364-377); halo nodes without markers hold 0.
      const int hx = x - X0 + 1, hy = y - Y0 + 1, hz = z - Z0 + 1;
      for (int sx = -1; sx <= 1; sx++)
        for (int sy = -1; sy <= 1; sy++)
          for (int sz = -1; sz <= 1; sz++) {
            const float ws = sten[sx + 1] * sten[sy + 1] * sten[sz + 1];
            const int h = (hx + sx) + HALO_X * ((hy + sy) + HALO_Y * (hz + sz));
            const float gv0 = cnt > 0 ? sm.g[0][h] : 0.0f, gv1 = cnt > 0 ? sm.g[1][h] : 0.0f,
                        gv2 = cnt > 0 ? sm.g[2][h] : 0.0f;
            gx += ws * gv0;
            gy += ws * gv1;
            gz += ws * gv2;
          }
    }
    const float jx = f[1] - f[2] + f[7] + f[8] + f[9] + f[10] - f[11] - f[12] - f[13] - f[14];
    const float jy = f[3] - f[4] + f[7] - f[8] + f[11] - f[12] + f[15] + f[16] - f[17] - f[18];
    const float jz = f[5] - f[6] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16] + f[17] - f[18];
    const float ux = (jx + 0.5f * gx) / rho, uy = (jy + 0.5f * gy) / rho, uz = (jz + 0.5f * gz) / rho;
    a.u[i] = ux;
    a.u[i + NC] = uy;
    a.u[i + 2 * NC] = uz;
    if (!(fabsf(ux) + fabsf(uy) + fabsf(uz) < 1e30f) || !(rho > 0.0f)) atomicOr(a.err, ERR_NONFINITE);
    float tau = VAR ? a.tau[i] : a.p.tauN;
    bool clamped = false;
    collide_ref<VAR>(f, rho, ux, uy, uz, gx, gy, gz, tau, a.p, clamped);
    if (VAR) {
      a.tau[i] = tau;
      nclamp += clamped ? 1 : 0;
    }
#pragma unroll
    for (int q = 0; q < 19; q++) ((float*)a.fout)[q * NC + i] = f[q];
  }
  if (VAR && nclamp) atomicAdd(a.clamps, (unsigned long long)nclamp);
}

// Dense spread-force field of the last particle pass with the reference's
// slot semantics (the reference's gpf slot 0 after its sum kernel).
__global__ void __launch_bounds__(FLUID_THREADS) spread_field_exact_kernel(const Geom g, const TileLists tl, int slots,
                                                                           float* __restrict__ out, unsigned* err) {
  __shared__ ExactSmem sm;
  const int tid = threadIdx.x;
  const long long T = blockIdx.x + (long long)g.ntx * (blockIdx.y + (long long)g.nty * blockIdx.z);
  const int X0 = blockIdx.x * TILE_X, Y0 = blockIdx.y * TILE_Y, Z0 = blockIdx.z * TILE_Z;
  const int cnt = tl.count[T];
  if (cnt <= 0) return;
  exact_spread_tile(sm, g, tl, T, min(cnt, tl.cap), X0, Y0, Z0, tid, blockDim.x, slots, err);
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

cudaError_t launch_spread_field_exact(const Geom& g, const TileLists& t, int slots, float* out, unsigned* err,
                                      cudaStream_t s) {
  if (slots < 1 || slots > MAX_SLOTS) return cudaErrorInvalidValue;
  dim3 grid(g.ntx, g.nty, g.ntz);
  spread_field_exact_kernel<<<grid, FLUID_THREADS, 0, s>>>(g, t, slots, out, err);
  return cudaGetLastError();
}

cudaError_t launch_fluid_exact(const FluidArgs& a, bool first, bool variable, int slots, cudaStream_t s) {
  if (slots < 1 || slots > MAX_SLOTS) return cudaErrorInvalidValue;
  dim3 block(TILE_X, TILE_Y, 2);
  dim3 grid(a.g.ntx, a.g.nty, a.g.ntz);
  if (first) {
    if (variable) fluid_exact_kernel<true, true><<<grid, block, 0, s>>>(a, slots);
    else fluid_exact_kernel<true, false><<<grid, block, 0, s>>>(a, slots);
  } else {
    if (variable) fluid_exact_kernel<false, true><<<grid, block, 0, s>>>(a, slots);
    else fluid_exact_kernel<false, false><<<grid, block, 0, s>>>(a, slots);
  }
  return cudaGetLastError();
}

}  // namespace d3q19
