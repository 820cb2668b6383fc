/* d3q19_oracle.c -- CPU restatement of the reference's time step, used only
 * as the checker (see d3q19_oracle.h).  TEST INFRASTRUCTURE: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 *
 * Written to reproduce the reference's floating-point evaluation order term
 * for term (compile with -ffp-contract=off): the moment transforms are loops
 * over q (or k) in increasing order, which matches the order of the
 * reference's unrolled expressions; the inverse transform coefficients are
 * M^T / |row|^2 rounded to float, which equal the reference's decimal
 * literals (GPU_program.cl:473-491) bit for bit.
 */
#include "d3q19_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

_Static_assert(sizeof(orc_int_params) == 332, "int_param_struct layout");
_Static_assert(sizeof(orc_flp_params) == 176, "flp_param_struct layout");

int orc_sizeof_int_params(void) { return (int)sizeof(orc_int_params); }
int orc_sizeof_flp_params(void) { return (int)sizeof(orc_flp_params); }

/* D3Q19 velocity set in the reference's order (D3Q19-OpenCL.c:9-13). */
static const int C[19][3] = {{0, 0, 0},  {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
                             {1, 1, 0},  {1, -1, 0},  {1, 0, 1},  {1, 0, -1}, {-1, 1, 0}, {-1, -1, 0}, {-1, 0, 1},
                             {-1, 0, -1}, {0, 1, 1},  {0, 1, -1}, {0, -1, 1}, {0, -1, -1}};

/* Moment basis in the reference's row order (GPU_program.cl:410-428):
 * rho, e, eps, jx, qx, jy, qy, jz, qz, 3pxx, 3pixx, pww, piww, pxy, pyz,
 * pxz, mx, my, mz.  Built from the velocities, not tabulated. */
static float Mf[19][19];
static float Minv[19][19]; /* Minv[q][k] */
static int basis_ready = 0;

static void build_basis(void) {
  if (basis_ready) return;
  double M[19][19];
  for (int q = 0; q < 19; q++) {
    int x = C[q][0], y = C[q][1], z = C[q][2];
    int s = x * x + y * y + z * z;
    int p = 2 * x * x - y * y - z * z;
    int w = y * y - z * z;
    M[0][q] = 1;
    M[1][q] = s == 0 ? -30 : (s == 1 ? -11 : 8);
    M[2][q] = s == 0 ? 12 : (s == 1 ? -4 : 1);
    M[3][q] = x;
    M[4][q] = s == 1 ? -4 * x : x;
    M[5][q] = y;
    M[6][q] = s == 1 ? -4 * y : y;
    M[7][q] = z;
    M[8][q] = s == 1 ? -4 * z : z;
    M[9][q] = p;
    M[10][q] = s == 1 ? -2 * p : p;
    M[11][q] = w;
    M[12][q] = s == 1 ? -2 * w : w;
    M[13][q] = x * y;
    M[14][q] = y * z;
    M[15][q] = x * z;
    M[16][q] = x * (y * y - z * z);
    M[17][q] = y * (z * z - x * x);
    M[18][q] = z * (x * x - y * y);
  }
  for (int k = 0; k < 19; k++) {
    double n2 = 0;
    for (int q = 0; q < 19; q++) n2 += M[k][q] * M[k][q];
    for (int q = 0; q < 19; q++) {
      Mf[k][q] = (float)M[k][q];
      Minv[q][k] = (float)(M[k][q] / n2);
    }
  }
  basis_ready = 1;
}

/* f_eq for rho, u (GPU_program.cl:978-1007): (rho/W)*(1 + 3cu + 4.5cu^2 - 1.5u^2). */
static void equilibrium(float* feq, float rho, float ux, float uy, float uz) {
  float usq = ux * ux + uy * uy + uz * uz;
  feq[0] = (rho / 3.0f) * (1.0f - 1.5f * usq);
  for (int q = 1; q < 19; q++) {
    float cu = (float)C[q][0] * ux + (float)C[q][1] * uy + (float)C[q][2] * uz;
    float W = q < 7 ? 18.0f : 36.0f;
    feq[q] = (rho / W) * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * usq);
  }
}

/* Guo forcing term before relaxation (GPU_program.cl:1010-1038). */
static void guo_term(float* fg, float ux, float uy, float uz, float gx, float gy, float gz) {
  float uDg = ux * gx + uy * gy + uz * gz;
  fg[0] = -uDg;
  for (int q = 1; q < 19; q++) {
    float cu = (float)C[q][0] * ux + (float)C[q][1] * uy + (float)C[q][2] * uz;
    float cg = (float)C[q][0] * gx + (float)C[q][1] * gy + (float)C[q][2] * gz;
    float D = q < 7 ? 6.0f : 12.0f;
    fg[q] = (cg - uDg + 3.0f * cu * cg) / D;
  }
}

#define VISC_NEWTONIAN 1
#define VISC_POWER_LAW 2
#define VISC_HB 3
#define VISC_CASSON 4
#define MIN_TAU 0.505
#define SRT_EPS 1E-8

/* GPU_program.cl:1041-1128 (device printf on clamp replaced by a counter). */
static long long g_tau_clamps = 0;
static float compute_tau(int model, float srtII, float tauN, const float* prm) {
  float tau = tauN;
  if (model == VISC_POWER_LAW) {
    float k = prm[0], n = prm[1], nu;
    srtII = srtII > SRT_EPS ? srtII : SRT_EPS;
    if (n == 0.5f)
      nu = k / sqrtf(srtII);
    else if (n == 1.0f)
      nu = k;
    else if (n == 2.0f)
      nu = k * srtII;
    else
      nu = k * powf(srtII, n - 1.0f);
    tau = 3.0f * nu + 0.5f;
    if (tau < MIN_TAU) {
      tau = MIN_TAU;
      g_tau_clamps++;
    }
  } else if (model == VISC_CASSON) {
    float tY = prm[0], eta = prm[1];
    srtII = srtII > SRT_EPS ? srtII : SRT_EPS;
    float a = sqrtf(tY / srtII) + sqrtf(eta);
    float nu = a * a;
    tau = 3.0f * nu + 0.5f;
    if (tau < MIN_TAU) {
      tau = MIN_TAU;
      g_tau_clamps++;
    }
  } else if (model == VISC_HB) {
    float tY = prm[0], k = prm[1], n = prm[2], nu;
    srtII = srtII > SRT_EPS ? srtII : SRT_EPS;
    if (n == 0.5f)
      nu = tY / srtII + k / sqrtf(srtII);
    else if (n == 1.0f)
      nu = tY / srtII + k;
    else if (n == 2.0f)
      nu = tY / srtII + k * srtII;
    else
      nu = tY / srtII + k * powf(srtII, n - 1.0f);
    tau = 3.0f * nu + 0.5f;
    if (tau < MIN_TAU) {
      tau = MIN_TAU;
      g_tau_clamps++;
    }
  }
  return tau;
}

long long orc_tau_clamp_count(void) { return g_tau_clamps; }

/* Relaxed moments back to populations: out[q] = sum_k Minv[q][k]*s[k]*m[k]. */
static void relax_back(float* out, const float* s, const float* m) {
  float sm[19];
  for (int k = 0; k < 19; k++) sm[k] = s[k] * m[k];
  for (int q = 0; q < 19; q++) {
    float acc = Minv[q][0] * sm[0];
    for (int k = 1; k < 19; k++) {
      if (Minv[q][k] != 0.0f) acc += Minv[q][k] * sm[k];
    }
    out[q] = acc;
  }
}

void orc_collide_stream(const float* f_c, float* f_s, const float* gpf, float* u, float* tau_lb, int* countPoint,
                        const orc_int_params* ip, const orc_flp_params* fp, int variable_viscosity) {
  build_basis();
  const int Nx = ip->LatticeSize[0], Ny = ip->LatticeSize[1], Nz = ip->LatticeSize[2];
  const long NC = (long)Nx * Ny * Nz;
  const long Nxy = (long)Nx * Ny;
  /* Push destinations i + c_q (stream_locations, GPU_program.cl:951-976). */
  long sh[19];
  for (int q = 0; q < 19; q++) sh[q] = C[q][0] + (long)Nx * C[q][1] + Nxy * C[q][2];
  const float sten[3] = {0.25f, 0.5f, 0.25f};
  /* Rates (GPU_program.cl:453); entries 8,9,10,14,15 become 1/tau. */
  const float s0[19] = {0.0f, 1.19f, 1.40f, 1.0f, 1.20f, 1.0f, 1.20f, 1.0f, 1.0f, 1.0f,
                        1.0f, 1.20f, 1.40f, 1.40f, 1.0f, 1.0f, 1.98f, 1.98f, 1.98f};

#pragma omp parallel for schedule(static)
  for (int z = 1; z < Nz - 1; z++) {
    for (int y = 1; y < Ny - 1; y++) {
      for (int x = 1; x < Nx - 1; x++) {
        long i = x + Nx * (y + (long)Ny * z);
        float f[19], rho = 0.0f;
        for (int q = 0; q < 19; q++) {
          f[q] = f_c[i + q * NC];
          rho += f[q];
        }
        float gx = fp->ConstBodyForce[0], gy = fp->ConstBodyForce[1], gz = fp->ConstBodyForce[2];
        /* 27-point (1/4,1/2,1/4)^3 smoothing of the spread force (356-377). */
        for (int sx = -1; sx <= 1; sx++)
          for (int sy = -1; sy <= 1; sy++)
            for (int sz = -1; sz <= 1; sz++) {
              long iS = (x + sx) + Nx * ((y + sy) + (long)Ny * (z + sz));
              float ws = sten[sx + 1] * sten[sy + 1] * sten[sz + 1];
              gx += ws * gpf[iS];
              gy += ws * gpf[iS + NC];
              gz += ws * gpf[iS + 2 * NC];
            }
        countPoint[i] = 0;
        /* Velocity with half the force (Guo), 387-389. */
        float jx = 0.0f, jy = 0.0f, jz = 0.0f;
        for (int q = 0; q < 19; q++) {
          jx += (float)C[q][0] * f[q];
          jy += (float)C[q][1] * f[q];
          jz += (float)C[q][2] * f[q];
        }
        float ux = (jx + 0.5f * gx) / rho, uy = (jy + 0.5f * gy) / rho, uz = (jz + 0.5f * gz) / rho;
        u[i] = ux;
        u[i + NC] = uy;
        u[i + 2 * NC] = uz;

        float feq[19], n[19], fg[19], mn[19], mg[19];
        equilibrium(feq, rho, ux, uy, uz);
        for (int q = 0; q < 19; q++) n[q] = feq[q] - f[q];
        guo_term(fg, ux, uy, uz, gx, gy, gz);
        mn[0] = 0.0f;
        for (int k = 0; k < 19; k++) {
          float am = Mf[k][0] * n[0], ag = Mf[k][0] * fg[0];
          for (int q = 1; q < 19; q++) {
            am += Mf[k][q] * n[q];
            ag += Mf[k][q] * fg[q];
          }
          if (k > 0) mn[k] = am;
          mg[k] = ag;
        }
        float s[19];
        memcpy(s, s0, sizeof(s));
        float tau;
        float msmn[19], msmg[19];
        if (!variable_viscosity) {
          tau = fp->NewtonianTau;
        } else {
          /* First pass with tau(t-1) gives the strain-rate estimate (459-562). */
          tau = tau_lb[i];
          s[8] = 1.0f / tau;
          s[9] = 1.0f / tau;
          s[10] = 1.0f / tau;
          s[14] = 1.0f / tau;
          s[15] = 1.0f / tau;
          relax_back(msmn, s, mn);
          relax_back(msmg, s, mg);
          float ss[19];
          for (int q = 0; q < 19; q++) ss[q] = msmn[q] + fg[q] - 0.5f * msmg[q];
          float scc[3][3];
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
              float acc = 0.0f;
              int first = 1;
              for (int q = 0; q < 19; q++) {
                int w = C[q][a] * C[q][b];
                if (w == 0) continue;
                if (first) {
                  acc = (float)w * ss[q];
                  first = 0;
                } else {
                  acc += (float)w * ss[q];
                }
              }
              scc[a][b] = acc;
            }
          float uu[3] = {ux, uy, uz}, gg[3] = {gx, gy, gz};
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
              if (a == b)
                scc[a][b] -= 2 * uu[a] * gg[a];
              else
                scc[a][b] -= (uu[a] * gg[b] + uu[b] * gg[a]);
            }
          float srt = 0.0f;
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) srt += scc[a][b] * scc[a][b];
          srt = (float)((double)sqrtf(srt) * 2.1213203 / (double)rho);
          tau = compute_tau(ip->ViscosityModel, srt, fp->NewtonianTau, fp->ViscosityParams);
          tau_lb[i] = tau;
        }
        s[8] = 1.0f / tau;
        s[9] = 1.0f / tau;
        s[10] = 1.0f / tau;
        s[14] = 1.0f / tau;
        s[15] = 1.0f / tau;
        relax_back(msmn, s, mn);
        relax_back(msmg, s, mg);
        /* Push to the neighbours (616-623). */
        for (int q = 0; q < 19; q++) f_s[q * NC + i + sh[q]] = f[q] + msmn[q] + fg[q] - 0.5f * msmg[q];
      }
    }
  }
}

/* Unknown populations per periodic node type (GPU_program.cl:647-677): a
 * population is unknown when it streams in from the buffer layer, i.e. when
 * its velocity has a component along an inward normal of the node. */
static const int inward[26][3] = {{1, 0, 0},  {-1, 0, 0},  {0, 1, 0},   {0, -1, 0},  {0, 0, 1},  {0, 0, -1},  {1, 1, 0},
                                  {1, -1, 0}, {1, 0, 1},   {1, 0, -1},  {-1, 1, 0},  {-1, -1, 0}, {-1, 0, 1}, {-1, 0, -1},
                                  {0, 1, 1},  {0, 1, -1},  {0, -1, 1},  {0, -1, -1}, {1, 1, 1},  {1, 1, -1},  {1, -1, 1},
                                  {1, -1, -1}, {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};

void orc_boundary_periodic(float* f_s, const orc_int_params* ip, const int* strMap, int nBC) {
  const int N[3] = {ip->LatticeSize[0], ip->LatticeSize[1], ip->LatticeSize[2]};
  const long NC = (long)N[0] * N[1] * N[2];
  for (int k = 0; k < nBC; k++) {
    long i = strMap[k];
    int type = strMap[k + nBC];
    for (int q = 1; q < 19; q++) {
      int unknown = 0;
      for (int d = 0; d < 3; d++)
        if (C[q][d] != 0 && C[q][d] == inward[type][d]) unknown = 1;
      if (!unknown) continue;
      /* offset = ((c*m*(c+m))/2)*(N-2) per axis (720-726). */
      long off[3];
      for (int d = 0; d < 3; d++) {
        int c = C[q][d], m = inward[type][d];
        off[d] = (long)((c * m * (c + m)) / 2) * (N[d] - 2);
      }
      long src = i + off[0] + N[0] * (off[1] + (long)N[1] * off[2]);
      f_s[q * NC + i] = f_s[q * NC + src];
    }
  }
}

/* Wet-node velocity boundary (GPU_program.cl:737-865, VEL_BC_MOM_CORR off). */
void orc_boundary_velocity(float* f_s, const orc_int_params* ip, const orc_flp_params* fp, int wallAxis,
                           int calcRho) {
  static const int tabUn[6][5] = {{1, 7, 8, 9, 10},   {2, 11, 12, 13, 14}, {3, 7, 11, 15, 16},
                                  {4, 8, 12, 17, 18}, {5, 9, 13, 15, 17},  {6, 10, 14, 16, 18}};
  static const int tabKn[6][14] = {{0, 3, 4, 5, 6, 15, 16, 17, 18, 2, 11, 12, 13, 14},
                                   {0, 3, 4, 5, 6, 15, 16, 17, 18, 1, 7, 8, 9, 10},
                                   {0, 1, 2, 5, 6, 9, 10, 13, 14, 4, 8, 12, 17, 18},
                                   {0, 1, 2, 5, 6, 9, 10, 13, 14, 3, 7, 11, 15, 16},
                                   {0, 1, 2, 3, 4, 7, 8, 11, 12, 6, 10, 14, 16, 18},
                                   {0, 1, 2, 3, 4, 7, 8, 11, 12, 5, 9, 13, 15, 17}};
  static const int tabAxes[6][3] = {{0, 1, 2}, {0, 1, 2}, {1, 0, 2}, {1, 0, 2}, {2, 0, 1}, {2, 0, 1}};
  const int N[3] = {ip->LatticeSize[0], ip->LatticeSize[1], ip->LatticeSize[2]};
  const long NC = (long)N[0] * N[1] * N[2];
  int R[3];
  for (int d = 0; d < 3; d++) R[d] = d == wallAxis ? 2 : N[d] - 2;
  for (int c2 = 0; c2 < R[2]; c2++)
    for (int c1 = 0; c1 < R[1]; c1++)
      for (int c0 = 0; c0 < R[0]; c0++) {
        int i3[3] = {c0 + 1, c1 + 1, c2 + 1};
        int ilu = i3[wallAxis] - 1;
        int ilu_pm = ilu * 2 - 1;
        int iw = wallAxis * 2 + ilu;
        i3[wallAxis] += (i3[wallAxis] - 1) * (N[wallAxis] - 4);
        long i = i3[0] + N[0] * (i3[1] + (long)N[1] * i3[2]);
        float fk[14];
        for (int k = 0; k < 14; k++) fk[k] = f_s[i + tabKn[iw][k] * NC];
        const float* uw = ilu ? fp->VelUpper : fp->VelLower;
        float un = -ilu_pm * uw[tabAxes[iw][0]];
        float ua1 = uw[tabAxes[iw][1]], ua2 = uw[tabAxes[iw][2]];
        float rho;
        float sum9 = fk[0] + fk[1] + fk[2] + fk[3] + fk[4] + fk[5] + fk[6] + fk[7] + fk[8];
        float sum5 = fk[9] + fk[10] + fk[11] + fk[12] + fk[13];
        if (calcRho) {
          rho = (sum9 + 2 * sum5) / (1.0f - un);
        } else {
          rho = 1.0f;
          un = 1 - (sum9 + 2 * sum5) / rho;
        }
        float Na1 = 0.0f, Na2 = 0.0f;
        f_s[i + tabUn[iw][0] * NC] = fk[9] + rho * un / 3.0f;
        f_s[i + tabUn[iw][1] * NC] = fk[11] + rho * (un + ua1) / 6.0f - Na1;
        f_s[i + tabUn[iw][2] * NC] = fk[10] + rho * (un - ua1) / 6.0f + Na1;
        f_s[i + tabUn[iw][3] * NC] = fk[13] + rho * (un + ua2) / 6.0f - Na2;
        f_s[i + tabUn[iw][4] * NC] = fk[12] + rho * (un - ua2) / 6.0f + Na2;
      }
}

void orc_reset_particle_fluid_forces(const orc_int_params* ip, float* gpf) {
  const int Nx = ip->LatticeSize[0], Ny = ip->LatticeSize[1], Nz = ip->LatticeSize[2];
  const long NC = (long)Nx * Ny * Nz;
  for (int z = 1; z < Nz - 1; z++)
    for (int y = 1; y < Ny - 1; y++)
      for (int x = 1; x < Nx - 1; x++) {
        long i = x + Nx * (y + (long)Ny * z);
        gpf[i] = 0.0f;
        gpf[i + NC] = 0.0f;
        gpf[i + 2 * NC] = 0.0f;
      }
}

void orc_sum_particle_fluid_forces(const orc_int_params* ip, float* gpf) {
  const int Nx = ip->LatticeSize[0], Ny = ip->LatticeSize[1], Nz = ip->LatticeSize[2];
  const long NC = (long)Nx * Ny * Nz;
  for (int z = 1; z < Nz - 1; z++)
    for (int y = 1; y < Ny - 1; y++)
      for (int x = 1; x < Nx - 1; x++) {
        long i = x + Nx * (y + (long)Ny * z);
        for (int j = 1; j < ip->MaxSurfPointsPerNode; j++)
          for (int d = 0; d < 3; d++) {
            gpf[i + NC * d] += gpf[i + NC * (3 * j + d)];
            gpf[i + NC * (3 * j + d)] = 0.0f;
          }
      }
}

static inline orc_float4 f4(float x, float y, float z, float w) {
  orc_float4 r = {x, y, z, w};
  return r;
}
static inline orc_float4 f4add(orc_float4 a, orc_float4 b) { return f4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
static inline orc_float4 f4sub(orc_float4 a, orc_float4 b) { return f4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
static inline orc_float4 f4scale(orc_float4 a, float s) { return f4(a.x * s, a.y * s, a.z * s, a.w * s); }
static inline orc_float4 f4cross(orc_float4 a, orc_float4 b) {
  return f4(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, 0.0f);
}
static inline orc_float4 f4fmod(orc_float4 a, orc_float4 b) {
  return f4(fmodf(a.x, b.x), fmodf(a.y, b.y), fmodf(a.z, b.z), fmodf(a.w, b.w));
}

void orc_particle_fluid_forces(const orc_int_params* ip, const orc_flp_params* fp, float* gpf, const float* u,
                               const orc_float4* parKin, orc_float4* parFluidForce, const orc_float4* spherePoints,
                               int* countPoint, int* marker_cell) {
  const int np = ip->NumParticles;
  const int P = ip->PointsPerParticle;
  const int L = ip->PointsPerWorkGroup;
  const int total = ip->TotalSurfPoints;
  const int ngroups = total / L;
  const int Nx = ip->LatticeSize[0], Ny = ip->LatticeSize[1], Nz = ip->LatticeSize[2];
  const long NC = (long)Nx * Ny * Nz;
  const orc_float4 sys = f4((float)ip->SystemSize[0], (float)ip->SystemSize[1], (float)ip->SystemSize[2], 1.0f);
  orc_float4* F = (orc_float4*)malloc(sizeof(orc_float4) * L);
  orc_float4* T = (orc_float4*)malloc(sizeof(orc_float4) * L);
  (void)np;
  for (int grp = 0; grp < ngroups; grp++) {
    for (int l = 0; l < L; l++) {
      int gid = grp * L + l;
      int par = gid / P, pt = gid % P;
      orc_float4 xp = parKin[par], vp = parKin[par + np], av = parKin[par + 3 * np];
      orc_float4 r0 = spherePoints[pt];
      orc_float4 rpp = f4fmod(f4add(f4add(xp, r0), sys), sys);
      int flX = (int)floorf(rpp.x), flY = (int)floorf(rpp.y), flZ = (int)floorf(rpp.z);
      int x0 = flX + ip->BufferSize[0], y0 = flY + ip->BufferSize[1], z0 = flZ + ip->BufferSize[2];
      if (marker_cell) {
        marker_cell[3 * gid] = x0;
        marker_cell[3 * gid + 1] = y0;
        marker_cell[3 * gid + 2] = z0;
      }
      int xs = (x0 == Nx - 2) ? -(Nx - 3) : 1;
      int ys = (y0 == Ny - 2) ? -(Ny - 3) : 1;
      int zs = (z0 == Nz - 2) ? -(Nz - 3) : 1;
      const int shift[8][3] = {{0, 0, 0},   {xs, 0, 0},  {0, ys, 0},  {0, 0, zs},
                               {xs, ys, 0}, {xs, 0, zs}, {0, ys, zs}, {xs, ys, zs}};
      float wx = 1.0f - (rpp.x - flX), wy = 1.0f - (rpp.y - flY), wz = 1.0f - (rpp.z - flZ);
      float w[8] = {wx * wy * wz,
                    (1.0f - wx) * wy * wz,
                    wx * (1.0f - wy) * wz,
                    wx * wy * (1.0f - wz),
                    (1.0f - wx) * (1.0f - wy) * wz,
                    (1.0f - wx) * wy * (1.0f - wz),
                    wx * (1.0f - wy) * (1.0f - wz),
                    (1.0f - wx) * (1.0f - wy) * (1.0f - wz)};
      orc_float4 upp = f4(0, 0, 0, 0);
      long idx[8];
      for (int n = 0; n < 8; n++) {
        idx[n] = (x0 + shift[n][0]) + Nx * ((y0 + shift[n][1]) + (long)Ny * (z0 + shift[n][2]));
        upp.x += w[n] * u[idx[n]];
        upp.y += w[n] * u[idx[n] + NC];
        upp.z += w[n] * u[idx[n] + 2 * NC];
      }
      orc_float4 vpp = f4add(vp, f4cross(av, r0));
      orc_float4 force = f4scale(f4sub(upp, vpp), fp->PointArea);
      orc_float4 torque = f4cross(r0, force);
      for (int n = 0; n < 8; n++) {
        int wc = countPoint[idx[n]]++;
        int j = wc % ip->MaxSurfPointsPerNode;
        gpf[idx[n] + NC * (3 * j)] -= w[n] * force.x;
        gpf[idx[n] + NC * (3 * j + 1)] -= w[n] * force.y;
        gpf[idx[n] + NC * (3 * j + 2)] -= w[n] * force.z;
      }
      F[l] = force;
      T[l] = torque;
    }
    /* Work-group tree reduction (GPU_program.cl:232-255). */
    for (int is = L / 2; is > 0; is >>= 1)
      for (int l = 0; l < is; l++) {
        F[l] = f4add(F[l], F[l + is]);
        T[l] = f4add(T[l], T[l + is]);
      }
    parFluidForce[grp] = F[0];
    parFluidForce[grp + ngroups] = T[0];
  }
  free(F);
  free(T);
}

void orc_particle_dynamics(const orc_int_params* ip, const orc_flp_params* fp, orc_float4* parKin,
                           orc_float4* parForce, const orc_float4* parFluidForce, const int* threadMembers,
                           const int* numParInThread, int numParThreads) {
  const int np = ip->NumParticles, nfa = ip->WorkGroupsPerParticle;
  const orc_float4 w = f4((float)ip->SystemSize[0], (float)ip->SystemSize[1], (float)ip->SystemSize[2], 1.0f);
  for (int th = 0; th < numParThreads; th++)
    for (int i = 0; i < numParInThread[th]; i++) {
      int p = threadMembers[th * np + i];
      orc_float4 acc = f4(0, 0, 0, 0), aacc = f4(0, 0, 0, 0);
      for (int fa = 0; fa < nfa; fa++) {
        acc = f4add(acc, parFluidForce[p * nfa + fa]);
        aacc = f4add(aacc, parFluidForce[(p + np) * nfa + fa]);
      }
      acc = f4add(acc, parForce[p]);
      aacc = f4add(aacc, parForce[p + np]);
      acc = f4(acc.x / fp->ParticleMass, acc.y / fp->ParticleMass, acc.z / fp->ParticleMass,
               acc.w / fp->ParticleMass);
      aacc = f4(aacc.x / fp->ParticleMomInertia, aacc.y / fp->ParticleMomInertia, aacc.z / fp->ParticleMomInertia,
                aacc.w / fp->ParticleMomInertia);
      acc.x += fp->ConstBodyForce[0];
      acc.y += fp->ConstBodyForce[1];
      acc.z += fp->ConstBodyForce[2];
      orc_float4 rt = f4add(f4add(parKin[p], parKin[p + np]), f4scale(acc, 0.5f));
      parKin[p] = f4fmod(f4add(rt, w), w);
      parKin[p + np] = f4add(parKin[p + np], acc);
      orc_float4 q = parKin[p + 2 * np], av = parKin[p + 3 * np];
      float dqw = -(av.x * q.x + av.y * q.y + av.z * q.z + av.w * q.w);
      orc_float4 dq = f4add(f4scale(av, q.w), f4cross(av, q));
      parKin[p + 2 * np] = f4scale(dq, 0.5f);
      parKin[p + 2 * np].w += 0.5f * dqw;
      parKin[p + 3 * np] = f4add(av, aacc);
      parForce[p] = f4(0, 0, 0, 0);
      parForce[p + np] = f4(0, 0, 0, 0);
    }
}

#define MIN_SEP 0.1
#define SQUEEZE_RANGE 0.1

/* CPU_program.cl:319-343: only the Newtonian branch produces a force. */
static float squeeze_force(int model, float vRel, float minSep, float rp, float tauN) {
  float rStar = rp / 2.0f;
  minSep = minSep < MIN_SEP ? MIN_SEP : minSep;
  float force = 0.0f;
  if (model == VISC_NEWTONIAN) {
    float eta0 = (tauN - 0.5f) / 3.0f;
    force = (float)(6 * M_PI * eta0 * rStar * rStar * vRel / minSep);
  }
  return force;
}

void orc_particle_particle_forces(const orc_int_params* ip, const orc_flp_params* fp, const orc_float4* parKin,
                                  orc_float4* parForce, const int* zoneNeighDat, const int* parsZone,
                                  const int* threadMembers, const int* numParInThread, int numParThreads,
                                  const int* zoneMembers, const int* numParInZone) {
  const int np = ip->NumParticles;
  const float rp = fp->ParticleDiam / 2.0f;
  const float W[3] = {(float)ip->SystemSize[0], (float)ip->SystemSize[1], (float)ip->SystemSize[2]};
  const int nzones = ip->NumZones[0] * ip->NumZones[1] * ip->NumZones[2];
  for (int th = 0; th < numParThreads; th++)
    for (int i = 0; i < numParInThread[th]; i++) {
      int pi = threadMembers[th * np + i];
      int pz = parsZone[pi];
      for (int nz = 1; nz <= zoneNeighDat[pz * 28]; nz++) {
        int zid = zoneNeighDat[pz * 28 + nz];
        /* The y-stride quirk of D3Q19-OpenCL.c:450 can name zones past the
         * end of the zone arrays when NumZones[2] > NumZones[1]; the
         * reference then reads out of bounds.  Such zones count as empty. */
        if (zid < 0 || zid >= nzones) continue;
        for (int j = 0; j < numParInZone[zid]; j++) {
          int pj = zoneMembers[zid * np + j];
          if (!(pi > pj)) continue;
          orc_float4 rij = f4sub(parKin[pj], parKin[pi]);
          float* r = &rij.x;
          for (int d = 0; d < 3; d++) {
            int sg = (r[d] < 0.0f) ? -1 : (r[d] > 0.0f);
            r[d] = (fabsf(r[d]) < W[d] / 2.0f) ? r[d] : (r[d] - (float)sg * W[d]);
          }
          float rSep = sqrtf(rij.x * rij.x + rij.y * rij.y + rij.z * rij.z + rij.w * rij.w);
          orc_float4 vij = f4sub(parKin[pj + np], parKin[pi + np]);
          float minSep = rSep - 2 * rp;
          orc_float4 e = f4(rij.x / rSep, rij.y / rSep, rij.z / rSep, rij.w / rSep);
          float vRel = -(e.x * vij.x + e.y * vij.y + e.z * vij.z);
          float overlap = -minSep;
          if (overlap > 0 && ip->ParForceModel == 1) {
            float fMag = fp->ParForceParams[0] * overlap;
            parForce[pi] = f4sub(parForce[pi], f4scale(e, fMag));
            parForce[pj] = f4add(parForce[pj], f4scale(e, fMag));
          }
          if (minSep > 0 && minSep < SQUEEZE_RANGE * rp) {
            float sq = squeeze_force(ip->ViscosityModel, vRel, minSep, rp, fp->NewtonianTau);
            parForce[pi] = f4sub(parForce[pi], f4scale(e, sq));
            parForce[pj] = f4add(parForce[pj], f4scale(e, sq));
          }
        }
      }
      float lo = fp->ParticleZBuffer - parKin[pi].z;
      if (lo > 0) parForce[pi].z += fp->ParForceParams[0] * lo;
      float up = parKin[pi].z - ((float)ip->SystemSize[2] - fp->ParticleZBuffer);
      if (up > 0) parForce[pi].z -= fp->ParForceParams[0] * up;
    }
}

void orc_update_particle_zones(const orc_int_params* ip, const orc_flp_params* fp, const orc_float4* parKin,
                               const int* threadMembers, const int* numParInThread, int numParThreads,
                               int* parsZone, int* zoneMembers, int* numParInZone) {
  const int np = ip->NumParticles;
  for (int th = 0; th < numParThreads; th++)
    for (int i = 0; i < numParInThread[th]; i++) {
      int p = threadMembers[i + th * np];
      int zx = (int)(parKin[p].x / fp->ZoneWidth[0]);
      int zy = (int)(parKin[p].y / fp->ZoneWidth[1]);
      int zz = (int)(parKin[p].z / fp->ZoneWidth[2]);
      int zid = zx + ip->NumZones[0] * (zy + ip->NumZones[1] * zz);
      parsZone[p] = zid;
      zoneMembers[zid * np + numParInZone[zid]++] = p;
    }
}

int orc_create_periodic_stream_mapping(const orc_int_params* ip, int* strMap) {
  const int N[3] = {ip->LatticeSize[0], ip->LatticeSize[1], ip->LatticeSize[2]};
  const int b = 1;
  const int* bc = ip->BoundaryConds;
  long cap = (long)N[0] * N[1] * N[2];
  int* idx = (int*)malloc(sizeof(int) * cap);
  int* typ = (int*)malloc(sizeof(int) * cap);
  int n = 0;
  /* Faces (D3Q19-OpenCL.c:983-990, 1028-1050): the face's fixed axis sits at
   * layer b or N-b-1; the two other axes run over b+1..N-b-2 (edges and
   * vertices are listed separately). */
  for (int face = 0; face < 6; face++) {
    int ax = face / 2;
    if (bc[ax] != 0) continue;
    int fixed = (face % 2) ? N[ax] - b - 1 : b;
    /* loop order: outer = second listed axis, inner = third (x innermost) */
    int outer = ax == 2 ? 1 : 2, inner = ax == 0 ? 1 : 0;
    for (int i = b + 1; i <= N[outer] - b - 2; i++)
      for (int j = b + 1; j <= N[inner] - b - 2; j++) {
        int r[3];
        r[ax] = fixed;
        r[outer] = i;
        r[inner] = j;
        idx[n] = r[0] + N[0] * (r[1] + r[2] * N[1]);
        typ[n] = face;
        n++;
      }
  }
  /* Edges (993-1006, 1054-1077): two fixed axes, included when either axis
   * is periodic. */
  static const int edge_axes[12][3] = {{0, 1, 2}, {0, 1, 2}, {0, 2, 1}, {0, 2, 1}, {0, 1, 2}, {0, 1, 2},
                                       {0, 2, 1}, {0, 2, 1}, {1, 2, 0}, {1, 2, 0}, {1, 2, 0}, {1, 2, 0}};
  static const int edge_hi[12][2] = {{0, 0}, {0, 1}, {0, 0}, {0, 1}, {1, 0}, {1, 1},
                                     {1, 0}, {1, 1}, {0, 0}, {0, 1}, {1, 0}, {1, 1}};
  for (int e = 0; e < 12; e++) {
    int a0 = edge_axes[e][0], a1 = edge_axes[e][1], run = edge_axes[e][2];
    if (!(bc[a0] == 0 || bc[a1] == 0)) continue;
    for (int i = b + 1; i <= N[run] - b - 2; i++) {
      int r[3];
      r[a0] = edge_hi[e][0] ? N[a0] - b - 1 : b;
      r[a1] = edge_hi[e][1] ? N[a1] - b - 1 : b;
      r[run] = i;
      idx[n] = r[0] + N[0] * (r[1] + r[2] * N[1]);
      typ[n] = 6 + e;
      n++;
    }
  }
  /* Vertices (1009-1018, 1080-1100), included when any axis is periodic. */
  if (bc[0] == 0 || bc[1] == 0 || bc[2] == 0) {
    for (int v = 0; v < 8; v++) {
      int r[3] = {(v & 4) ? N[0] - b - 1 : b, (v & 2) ? N[1] - b - 1 : b, (v & 1) ? N[2] - b - 1 : b};
      idx[n] = r[0] + N[0] * (r[1] + r[2] * N[1]);
      typ[n] = 18 + v;
      n++;
    }
  }
  for (int k = 0; k < n; k++) {
    strMap[k] = idx[k];
    strMap[n + k] = typ[k];
  }
  free(idx);
  free(typ);
  return n;
}

void orc_zone_neighbours(const orc_int_params* ip, int* znd) {
  const int* Z = ip->NumZones;
  const int* bc = ip->BoundaryConds;
  for (int k = 0; k < Z[2]; k++)
    for (int j = 0; j < Z[1]; j++)
      for (int i = 0; i < Z[0]; i++) {
        int zid = i + Z[0] * (j + Z[1] * k);
        znd[28 * zid] = 0;
        int lo[3] = {-1, -1, -1}, hi[3] = {1, 1, 1};
        int pos[3] = {i, j, k};
        for (int d = 0; d < 3; d++) {
          if (bc[d] == 1 && pos[d] == 0) lo[d] = 0;
          if (bc[d] == 1 && pos[d] == Z[d] - 1) hi[d] = 0;
        }
        for (int n = lo[2]; n <= hi[2]; n++)
          for (int m = lo[1]; m <= hi[1]; m++)
            for (int l = lo[0]; l <= hi[0]; l++) {
              int s[3] = {i + l, j + m, k + n}, wr[3];
              for (int d = 0; d < 3; d++) wr[d] = s[d] < 0 ? Z[d] - 1 : s[d] % Z[d];
              /* The reference strides y by NumZones[2] (D3Q19-OpenCL.c:450). */
              int nid = wr[0] + Z[0] * (wr[1] + Z[2] * wr[2]);
              int cnt = ++znd[28 * zid];
              znd[28 * zid + cnt] = nid;
            }
      }
}

void orc_step(orc_state* s, const orc_int_params* ip, const orc_flp_params* fp, int t) {
  const int Nx = ip->LatticeSize[0], Ny = ip->LatticeSize[1], Nz = ip->LatticeSize[2];
  float* fc = (t % 2 == 0) ? s->fA : s->fB;
  float* fs = (t % 2 == 0) ? s->fB : s->fA;
  int usingParticles = ip->NumParticles > 0;
  (void)Nx;
  (void)Ny;
  (void)Nz;
  orc_collide_stream(fc, fs, s->gpf, s->u, s->tau_lb, s->countPoint, ip, fp, s->variable_viscosity);
  if (usingParticles) {
    orc_particle_dynamics(ip, fp, s->parKin, s->parForce, s->parFluidForce, s->threadMembers, s->numParInThread,
                          s->numParThreads);
    orc_reset_particle_fluid_forces(ip, s->gpf);
  }
  orc_boundary_periodic(fs, ip, s->strMap, s->numPeriodicNodes);
  int wallAxis = -1;
  for (int d = 0; d < 3; d++)
    if (ip->BoundaryConds[d] == 1) wallAxis = d;
  if (wallAxis >= 0) {
    orc_boundary_velocity(fs, ip, fp, wallAxis, 0);
    for (int i = 0; i < 3; i++)
      if (s->tangentialVelBC[i] == 1) orc_boundary_velocity(fs, ip, fp, i, 0);
  }
  if (usingParticles) {
    orc_particle_fluid_forces(ip, fp, s->gpf, s->u, s->parKin, s->parFluidForce, s->spherePoints, s->countPoint,
                              NULL);
    orc_sum_particle_fluid_forces(ip, s->gpf);
    orc_particle_particle_forces(ip, fp, s->parKin, s->parForce, s->zoneNeighDat, s->parsZone, s->threadMembers,
                                 s->numParInThread, s->numParThreads, s->zoneMembers, s->numParInZone);
  }
  if (usingParticles && t % s->rebuildFreq == 0) {
    int nz = ip->NumZones[0] * ip->NumZones[1] * ip->NumZones[2];
    memset(s->numParInZone, 0, sizeof(int) * nz);
    orc_update_particle_zones(ip, fp, s->parKin, s->threadMembers, s->numParInThread, s->numParThreads,
                              s->parsZone, s->zoneMembers, s->numParInZone);
  }
}
