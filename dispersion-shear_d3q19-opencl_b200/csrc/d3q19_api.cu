// d3q19_api.cu -- the C ABI (include/d3q19_b200.h): context, device memory,
// the per-step launch sequence, CUDA-graph replay and the read-backs.
#include "../../include/d3q19_b200.h"
#include "d3q19_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

static_assert(sizeof(int_param_struct) == 332, "int_param_struct must match struct_header_device.h");
static_assert(sizeof(flp_param_struct) == 176, "flp_param_struct must match struct_header_device.h");

using namespace d3q19;

struct d3q19_ctx {
  int_param_struct ip;
  flp_param_struct fp;
  d3q19_options opt;
  int dev = 0;
  cudaStream_t stream = nullptr;
  // The particle-particle forces and the zone rebuild of step t feed only
  // the rigid-body update of step t+1: they run on a second stream, forked
  // after the particle pass and joined before the next one, so that the
  // collide of step t+1 overlaps them.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool side_pending = false;
  Geom g;
  FluidParams fpar;
  ParticleParams ppar;
  void* f[2] = {nullptr, nullptr};  // float, or 16-bit shifted storage (opt.storage)
  int cur = 0;         // f[cur] is what the next step reads
  int f_state = 0;     // 0 unset, 1 reference state (pre-collision), 2 post-collision
  float* u = nullptr;
  float* tau = nullptr;
  float4* kin[2] = {nullptr, nullptr};
  float4* pff[2] = {nullptr, nullptr};
  float4* pf[2] = {nullptr, nullptr};
  int pcur = 0;
  float4* sphere = nullptr;
  float4* mrec = nullptr;
  int* tile_count = nullptr;
  unsigned* fmax = nullptr;  // [2]
  int last_t = 0;
  int* tile_list = nullptr;
  int tile_cap = 0;
  long long ntiles = 0;
  int* znd = nullptr;
  int* parsZone = nullptr;
  int* zoneMembers = nullptr;
  int* numParInZone = nullptr;
  int* revStart = nullptr;
  int* revList = nullptr;
  int* zoneOf = nullptr;
  int nzones = 0;
  unsigned* err = nullptr;
  unsigned long long* clamps = nullptr;
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  bool have_particles = false, have_zones = false;
  unsigned sticky = 0;
  std::map<std::tuple<int, int, int, int>, cudaGraphExec_t> graphs;
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_fluid, ev_part;
  char msg[512] = {0};
};

static char g_create_error[512] = {0};

static int ensure_scratch(d3q19_ctx* c, size_t bytes);

static int fail(d3q19_ctx* c, int code, const char* fmt, ...) {
  char* buf = c ? c->msg : g_create_error;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, 512, fmt, ap);
  va_end(ap);
  return code;
}

#define CUDA_TRY(c, call)                                                                      \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return fail((c), D3Q19_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
static int dalloc(d3q19_ctx* c, T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(c, D3Q19_ENOMEM, "cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
  }
  return 0;
}

extern "C" int d3q19_get_device_info(int device, d3q19_device_info* out) {
  if (!out) return D3Q19_EINVAL;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n)
    return fail(nullptr, D3Q19_ENODEV, "no CUDA device %d", device);
  cudaDeviceProp pr;
  if (cudaGetDeviceProperties(&pr, device) != cudaSuccess) return D3Q19_ECUDA;
  memset(out, 0, sizeof(*out));
  snprintf(out->name, sizeof(out->name), "%s", pr.name);
  out->sm_count = pr.multiProcessorCount;
  out->cc_major = pr.major;
  out->cc_minor = pr.minor;
  out->global_mem_bytes = pr.totalGlobalMem;
  out->kernel_work_group_size = 256;
  return 0;
}

static int validate(const int_param_struct* ip, const flp_param_struct* fp, const d3q19_options* o) {
  if ((long long)ip->LatticeSize[0] * ip->LatticeSize[1] * ip->LatticeSize[2] >= (1LL << 31))
    return fail(nullptr, D3Q19_EINVAL, "lattice of 2^31 or more nodes");
  for (int d = 0; d < 3; d++) {
    if (ip->LatticeSize[d] < 4 || ip->LatticeSize[d] > 65535)
      return fail(nullptr, D3Q19_EINVAL, "LatticeSize[%d] = %d outside [4, 65535]", d, ip->LatticeSize[d]);
    if (ip->BufferSize[d] != 1)
      return fail(nullptr, D3Q19_EINVAL, "BufferSize[%d] = %d: the reference kernels assume a 1-node buffer", d,
                  ip->BufferSize[d]);
    if (ip->BoundaryConds[d] != 0 && ip->BoundaryConds[d] != 1)
      return fail(nullptr, D3Q19_EINVAL, "BoundaryConds[%d] = %d (0 periodic, 1 velocity)", d, ip->BoundaryConds[d]);
  }
  if (ip->BoundaryConds[0] + ip->BoundaryConds[1] + ip->BoundaryConds[2] > 1)
    return fail(nullptr, D3Q19_EINVAL, "more than 1 pair of faces with velocity boundaries (D3Q19-OpenCL.c:103)");
  if (o->collision < 0 || o->collision > 1) return fail(nullptr, D3Q19_EINVAL, "collision must be 0 or 1");
  if (o->arithmetic < 0 || o->arithmetic > 1) return fail(nullptr, D3Q19_EINVAL, "arithmetic must be 0 or 1");
  if (o->arithmetic == 1 && o->collision != 0)
    return fail(nullptr, D3Q19_EINVAL, "the reference-exact arithmetic implements the reference's MRT only");
  if (o->arithmetic == 1 && (o->tau_max != 0.0f || o->tau_min != 0.0f || o->casson_reg != 0.0f))
    return fail(nullptr, D3Q19_EINVAL, "the reference-exact arithmetic has the reference's tau limits only");
  if (o->arithmetic == 1 && (ip->MaxSurfPointsPerNode < 1 || ip->MaxSurfPointsPerNode > 16))
    return fail(nullptr, D3Q19_EINVAL, "MaxSurfPointsPerNode must be in [1, 16] for the reference-exact arithmetic");
  if (o->storage < 0 || o->storage > 2)
    return fail(nullptr, D3Q19_EINVAL, "storage %d (0 FP32, 1 FP16 shifted, 2 BF16 shifted)", o->storage);
  if (o->arithmetic == 1 && o->storage != 0)
    return fail(nullptr, D3Q19_EINVAL, "the reference-exact arithmetic stores FP32 distributions only");
  if (o->particle_precision != 0)
    return fail(nullptr, D3Q19_EINVAL, "particle_precision %d not available in this build", o->particle_precision);
  if (fp->NewtonianTau <= 0.5f) return fail(nullptr, D3Q19_EINVAL, "NewtonianTau must exceed 0.5");
  const int np = ip->NumParticles;
  if (np < 0) return fail(nullptr, D3Q19_EINVAL, "NumParticles < 0");
  if (np > 0) {
    const int P = ip->PointsPerParticle, L = ip->PointsPerWorkGroup;
    if (P <= 0 || L <= 0 || L > 1024 || (L & (L - 1)) != 0 || P % L != 0)
      return fail(nullptr, D3Q19_EINVAL, "PointsPerParticle %d / PointsPerWorkGroup %d invalid", P, L);
    if (ip->WorkGroupsPerParticle != P / L)
      return fail(nullptr, D3Q19_EINVAL, "WorkGroupsPerParticle %d != %d", ip->WorkGroupsPerParticle, P / L);
    if ((long long)ip->TotalSurfPoints != (long long)P * np)
      return fail(nullptr, D3Q19_EINVAL, "TotalSurfPoints %d != P*np", ip->TotalSurfPoints);
    for (int d = 0; d < 3; d++)
      if (ip->NumZones[d] <= 0 || ip->SystemSize[d] <= 0)
        return fail(nullptr, D3Q19_EINVAL, "NumZones/SystemSize must be positive");
    if (!(fp->ParticleMass > 0) || !(fp->ParticleMomInertia > 0))
      return fail(nullptr, D3Q19_EINVAL, "particle mass and moment of inertia must be positive");
    if (o->rebuild_freq <= 0) return fail(nullptr, D3Q19_EINVAL, "rebuild_freq must be positive");
  }
  return 0;
}

extern "C" int d3q19_create(const int_param_struct* ip, const flp_param_struct* fp, const d3q19_options* opt,
                            d3q19_ctx** out) {
  if (!ip || !fp || !out) return fail(nullptr, D3Q19_EINVAL, "null argument");
  d3q19_options o;
  memset(&o, 0, sizeof(o));
  if (opt) o = *opt;
  if (o.rebuild_freq <= 0) o.rebuild_freq = 10;  // the reference's default (D3Q19-OpenCL.c:60)
  int rc = validate(ip, fp, &o);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || o.device < 0 || o.device >= ndev)
    return fail(nullptr, D3Q19_ENODEV, "CUDA device %d not available", o.device);
  cudaDeviceProp pr;
  cudaGetDeviceProperties(&pr, o.device);
  if (pr.major != 10) return fail(nullptr, D3Q19_ENODEV, "device %s is sm_%d%d; this build is sm_100a", pr.name, pr.major, pr.minor);

  d3q19_ctx* c = new d3q19_ctx();
  c->ip = *ip;
  c->fp = *fp;
  c->opt = o;
  c->dev = o.device;
  cudaSetDevice(c->dev);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    d3q19_destroy(c);
    return fail(nullptr, D3Q19_ECUDA, "stream or event creation failed");
  }
  Geom& g = c->g;
  g.Nx = ip->LatticeSize[0];
  g.Ny = ip->LatticeSize[1];
  g.Nz = ip->LatticeSize[2];
  g.NC = (long long)g.Nx * g.Ny * g.Nz;
  g.wallAxis = -1;
  for (int d = 0; d < 3; d++) {
    g.periodic[d] = ip->BoundaryConds[d] == 0;
    if (ip->BoundaryConds[d] == 1) g.wallAxis = d;
    g.buffer[d] = ip->BufferSize[d];
    g.tanBC[d] = o.tangential_vel_bc[d] == 1;
  }
  if (g.wallAxis < 0)
    for (int d = 0; d < 3; d++) g.tanBC[d] = 0;  // applied only with a wall axis (sim_main.c:383-405)
  g.ntx = (g.Nx + TILE_X - 1) / TILE_X;
  g.nty = (g.Ny + TILE_Y - 1) / TILE_Y;
  g.ntz = (g.Nz + TILE_Z - 1) / TILE_Z;
  c->ntiles = (long long)g.ntx * g.nty * g.ntz;

  FluidParams& p = c->fpar;
  for (int d = 0; d < 3; d++) {
    p.g[d] = fp->ConstBodyForce[d];
    p.velLower[d] = fp->VelLower[d];
    p.velUpper[d] = fp->VelUpper[d];
  }
  p.tauN = fp->NewtonianTau;
  p.viscModel = ip->ViscosityModel;
  for (int k = 0; k < 4; k++) p.visc[k] = fp->ViscosityParams[k];
  p.tauMax = o.tau_max;
  p.tauMin = o.tau_min;
  p.cassonReg = o.casson_reg;

  ParticleParams& pp = c->ppar;
  memset(&pp, 0, sizeof(pp));
  pp.np = ip->NumParticles;
  pp.P = ip->PointsPerParticle;
  pp.L = ip->PointsPerWorkGroup;
  pp.nfa = ip->WorkGroupsPerParticle;
  for (int d = 0; d < 3; d++) {
    pp.S[d] = (float)ip->SystemSize[d];
    pp.Sint[d] = ip->SystemSize[d];
    pp.buffer[d] = ip->BufferSize[d];
    pp.g[d] = fp->ConstBodyForce[d];
    pp.numZones[d] = ip->NumZones[d];
    pp.zoneWidth[d] = fp->ZoneWidth[d];
  }
  pp.mass = fp->ParticleMass;
  pp.inertia = fp->ParticleMomInertia;
  pp.pointArea = fp->PointArea;
  pp.diam = fp->ParticleDiam;
  pp.zbuf = fp->ParticleZBuffer;
  pp.kcol = fp->ParForceParams[0];
  pp.forceModel = ip->ParForceModel;
  pp.viscModel = ip->ViscosityModel;
  pp.tauN = fp->NewtonianTau;
  pp.fixed = o.fixed_particles ? 1 : 0;
  pp.exact = o.arithmetic == 1 ? 1 : 0;

  const long long NC = g.NC;
  const size_t fbytes = (size_t)storage_bytes(o.storage) * 19 * NC;
  if ((rc = dalloc(c, (char**)&c->f[0], fbytes)) || (rc = dalloc(c, (char**)&c->f[1], fbytes)) ||
      (rc = dalloc(c, &c->u, 3 * NC)) ||
      (rc = dalloc(c, &c->tau, NC)) || (rc = dalloc(c, &c->err, 1)) || (rc = dalloc(c, &c->clamps, 1))) {
    snprintf(g_create_error, sizeof(g_create_error), "%s", c->msg);
    d3q19_destroy(c);
    return rc;
  }
  cudaMemsetAsync(c->err, 0, sizeof(unsigned), c->stream);
  cudaMemsetAsync(c->clamps, 0, sizeof(unsigned long long), c->stream);
  cudaMemsetAsync(c->u, 0, sizeof(float) * 3 * NC, c->stream);
  const int np = pp.np;
  if (np > 0) {
    const long long M = (long long)np * pp.P;
    c->nzones = pp.numZones[0] * pp.numZones[1] * pp.numZones[2];
    c->tile_cap = o.ibm_tile_capacity > 0 ? o.ibm_tile_capacity : (int)std::min<long long>(M, 2048);
    rc = 0;
    for (int b = 0; b < 2 && !rc; b++) {
      rc = dalloc(c, &c->kin[b], 4 * np);
      if (!rc) rc = dalloc(c, &c->pff[b], 2LL * np * pp.nfa);
      if (!rc) rc = dalloc(c, &c->pf[b], 2 * np);
    }
    if (!rc) rc = dalloc(c, &c->sphere, pp.P);
    if (!rc) rc = dalloc(c, &c->mrec, 2 * M);
    if (!rc) rc = dalloc(c, &c->tile_count, c->ntiles);
    if (!rc) rc = dalloc(c, &c->fmax, 2);
    if (!rc) rc = dalloc(c, &c->tile_list, c->ntiles * c->tile_cap);
    if (!rc) rc = dalloc(c, &c->znd, 28LL * c->nzones);
    if (!rc) rc = dalloc(c, &c->parsZone, np);
    if (!rc) rc = dalloc(c, &c->zoneMembers, (long long)c->nzones * np);
    if (!rc) rc = dalloc(c, &c->numParInZone, c->nzones);
    if (!rc) rc = dalloc(c, &c->revStart, c->nzones + 1);
    if (!rc) rc = dalloc(c, &c->revList, 27LL * c->nzones);
    if (!rc) rc = dalloc(c, &c->zoneOf, np);
    if (rc) {
      snprintf(g_create_error, sizeof(g_create_error), "%s", c->msg);
      d3q19_destroy(c);
      return rc;
    }
    cudaMemsetAsync(c->tile_count, 0, sizeof(int) * c->ntiles, c->stream);
    cudaMemsetAsync(c->fmax, 0, sizeof(unsigned) * 2, c->stream);
    cudaMemsetAsync(c->mrec, 0, sizeof(float4) * 2 * M, c->stream);
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    snprintf(g_create_error, sizeof(g_create_error), "initialisation failed");
    d3q19_destroy(c);
    return D3Q19_ECUDA;
  }
  *out = c;
  return 0;
}

extern "C" int d3q19_write_lattice(d3q19_ctx* c, const float* f, const float* u, const float* tau_lb) {
  if (!c || !f || !u) return D3Q19_EINVAL;
  cudaSetDevice(c->dev);
  const long long NC = c->g.NC;
  if (c->opt.storage == STORE_F32) {
    CUDA_TRY(c, cudaMemcpyAsync(c->f[c->cur], f, sizeof(float) * 19 * NC, cudaMemcpyHostToDevice, c->stream));
  } else {
    // Upload in FP32, then round to the shifted 16-bit form on the device.
    int rc = ensure_scratch(c, sizeof(float) * 19 * NC);
    if (rc) return rc;
    CUDA_TRY(c, cudaMemcpyAsync(c->scratch, f, sizeof(float) * 19 * NC, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, launch_store_f((const float*)c->scratch, c->f[c->cur], NC, c->opt.storage, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  CUDA_TRY(c, cudaMemcpyAsync(c->u, u, sizeof(float) * 3 * NC, cudaMemcpyHostToDevice, c->stream));
  if (tau_lb) {
    CUDA_TRY(c, cudaMemcpyAsync(c->tau, tau_lb, sizeof(float) * NC, cudaMemcpyHostToDevice, c->stream));
  } else {
    std::vector<float> t((size_t)NC, c->fp.NewtonianTau);
    CUDA_TRY(c, cudaMemcpyAsync(c->tau, t.data(), sizeof(float) * NC, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  c->f_state = 1;
  return 0;
}

extern "C" int d3q19_write_particles(d3q19_ctx* c, const float* parKin, const float* parForce,
                                     const float* parFluidForce, const float* spherePoints) {
  if (!c) return D3Q19_EINVAL;
  const int np = c->ppar.np;
  if (np == 0) return 0;
  if (!parKin || !parForce || !parFluidForce || !spherePoints) return fail(c, D3Q19_EINVAL, "null particle array");
  cudaSetDevice(c->dev);
  const int b = c->pcur;
  CUDA_TRY(c, cudaMemcpyAsync(c->kin[b], parKin, sizeof(float4) * 4 * np, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->pf[b], parForce, sizeof(float4) * 2 * np, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->pff[b], parFluidForce, sizeof(float4) * 2 * np * c->ppar.nfa,
                              cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->sphere, spherePoints, sizeof(float4) * c->ppar.P, cudaMemcpyHostToDevice,
                              c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->have_particles = true;
  return 0;
}

extern "C" int d3q19_write_zones(d3q19_ctx* c, const int* znd, const int* parsZone, const int* zoneMembers,
                                 const int* numParInZone, const int* threadMembers, const int* numParInThread) {
  (void)threadMembers;
  (void)numParInThread;
  if (!c) return D3Q19_EINVAL;
  const int np = c->ppar.np, nz = c->nzones;
  if (np == 0) return 0;
  if (!znd || !parsZone || !zoneMembers || !numParInZone) return fail(c, D3Q19_EINVAL, "null zone array");
  // Zone lists must be consistent: every sphere listed once, in the zone
  // parsZone names (update_particle_zones and initialize_particle_zones
  // always produce such lists).
  std::vector<int> seen(np, 0);
  for (int z = 0; z < nz; z++) {
    if (numParInZone[z] < 0 || numParInZone[z] > np) return fail(c, D3Q19_EINVAL, "numParInZone[%d] out of range", z);
    for (int j = 0; j < numParInZone[z]; j++) {
      int p = zoneMembers[(long long)z * np + j];
      if (p < 0 || p >= np || parsZone[p] != z || seen[p]++)
        return fail(c, D3Q19_EINVAL, "zone lists inconsistent at zone %d entry %d", z, j);
    }
    const int cnt = znd[28 * z];
    if (cnt < 0 || cnt > 27) return fail(c, D3Q19_EINVAL, "zoneNeighDat count out of range at zone %d", z);
  }
  for (int p = 0; p < np; p++)
    if (!seen[p]) return fail(c, D3Q19_EINVAL, "sphere %d is in no zone list", p);
  // Reverse neighbour table: for zone Z, every zone Y (with multiplicity)
  // whose neighbour list names Z.  Ids past the zone count (the y-stride
  // quirk of D3Q19-OpenCL.c:450) name no zone and are skipped.
  std::vector<int> cnt(nz + 1, 0), start(nz + 1, 0);
  for (int y = 0; y < nz; y++)
    for (int t = 1; t <= znd[28 * y]; t++) {
      int z = znd[28 * y + t];
      if (z >= 0 && z < nz) cnt[z]++;
    }
  for (int z = 0; z < nz; z++) start[z + 1] = start[z] + cnt[z];
  std::vector<int> rev(std::max(1, start[nz])), fillp(start.begin(), start.end() - 1);
  for (int y = 0; y < nz; y++)
    for (int t = 1; t <= znd[28 * y]; t++) {
      int z = znd[28 * y + t];
      if (z >= 0 && z < nz) rev[fillp[z]++] = y;
    }
  cudaSetDevice(c->dev);
  CUDA_TRY(c, cudaMemcpyAsync(c->znd, znd, sizeof(int) * 28 * nz, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->parsZone, parsZone, sizeof(int) * np, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->zoneMembers, zoneMembers, sizeof(int) * (size_t)nz * np, cudaMemcpyHostToDevice,
                              c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->numParInZone, numParInZone, sizeof(int) * nz, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->revStart, start.data(), sizeof(int) * (nz + 1), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->revList, rev.data(), sizeof(int) * start[nz], cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->have_zones = true;
  return 0;
}

// Periodic boundary node list of create_periodic_stream_mapping
// (D3Q19-OpenCL.c:973-1112): faces, then edges, then vertices of the layer-1
// box; a face when its axis is periodic, an edge when either of its axes is,
// a vertex when any axis is.  strMap = [node indices..., node types...].
extern "C" int d3q19_periodic_map(const int_param_struct* ip, int* strMap, int capacity) {
  if (!ip) return D3Q19_EINVAL;
  const int N[3] = {ip->LatticeSize[0], ip->LatticeSize[1], ip->LatticeSize[2]};
  const int* bc = ip->BoundaryConds;
  const int b = 1;
  std::vector<int> idx, typ;
  auto add = [&](int x, int y, int z, int t) {
    idx.push_back(x + N[0] * (y + N[1] * z));
    typ.push_back(t);
  };
  for (int face = 0; face < 6; face++) {
    const int ax = face / 2;
    if (bc[ax] != 0) continue;
    const int fixed = (face & 1) ? N[ax] - b - 1 : b;
    const int outer = ax == 2 ? 1 : 2, inner = ax == 0 ? 1 : 0;
    for (int i = b + 1; i <= N[outer] - b - 2; i++)
      for (int j = b + 1; j <= N[inner] - b - 2; j++) {
        int r[3];
        r[ax] = fixed;
        r[outer] = i;
        r[inner] = j;
        add(r[0], r[1], r[2], face);
      }
  }
  // Edges: the two fixed axes (low/high) and the running axis, in the
  // reference's edge order.
  static const int ax0[12] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1};
  static const int ax1[12] = {1, 1, 2, 2, 1, 1, 2, 2, 2, 2, 2, 2};
  static const int hi0[12] = {0, 0, 0, 0, 1, 1, 1, 1, 0, 0, 1, 1};
  static const int hi1[12] = {0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1};
  for (int e = 0; e < 12; e++) {
    const int a0 = ax0[e], a1 = ax1[e], run = 3 - a0 - a1;
    if (!(bc[a0] == 0 || bc[a1] == 0)) continue;
    for (int i = b + 1; i <= N[run] - b - 2; i++) {
      int r[3];
      r[a0] = hi0[e] ? N[a0] - b - 1 : b;
      r[a1] = hi1[e] ? N[a1] - b - 1 : b;
      r[run] = i;
      add(r[0], r[1], r[2], 6 + e);
    }
  }
  if (bc[0] == 0 || bc[1] == 0 || bc[2] == 0)
    for (int v = 0; v < 8; v++)
      add((v & 4) ? N[0] - b - 1 : b, (v & 2) ? N[1] - b - 1 : b, (v & 1) ? N[2] - b - 1 : b, 18 + v);
  const int n = (int)idx.size();
  if (strMap) {
    if (capacity < 2 * n) return D3Q19_EINVAL;
    for (int k = 0; k < n; k++) {
      strMap[k] = idx[k];
      strMap[n + k] = typ[k];
    }
  }
  return n;
}

extern "C" int d3q19_write_periodic_map(d3q19_ctx* c, const int* strMap, int n) {
  if (!c || (n > 0 && !strMap)) return D3Q19_EINVAL;
  const int expect = d3q19_periodic_map(&c->ip, nullptr, 0);
  if (n != expect) return fail(c, D3Q19_EINVAL, "periodic map has %d nodes, boundary conditions imply %d", n, expect);
  std::vector<int> mine(2 * (size_t)std::max(n, 1));
  d3q19_periodic_map(&c->ip, mine.data(), (int)mine.size());
  for (int k = 0; k < 2 * n; k++)
    if (mine[k] != strMap[k]) return fail(c, D3Q19_EINVAL, "periodic map differs at entry %d", k);
  return 0;
}

static int check_ready(d3q19_ctx* c) {
  if (!c) return D3Q19_EINVAL;
  if (c->f_state == 0) return fail(c, D3Q19_ESTATE, "lattice not written");
  if (c->ppar.np > 0 && (!c->have_particles || !c->have_zones))
    return fail(c, D3Q19_ESTATE, "particles or zones not written");
  return 0;
}

static int enqueue_step(d3q19_ctx* c, int t) {
  FluidArgs fa;
  fa.g = c->g;
  fa.p = c->fpar;
  fa.t = t;
  fa.fin = c->f[c->cur];
  fa.fout = c->f[1 - c->cur];
  fa.u = c->u;
  fa.tau = c->tau;
  fa.tiles.cap = c->tile_cap;
  fa.tiles.count = c->tile_count;
  fa.tiles.list = c->tile_list;
  fa.tiles.mrec = c->mrec;
  fa.tiles.fmax = c->fmax;
  fa.has_ibm = c->ppar.np > 0;
  fa.err = c->err;
  fa.clamps = c->clamps;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->profiling) {
    CUDA_TRY(c, cudaEventCreate(&e0));
    CUDA_TRY(c, cudaEventCreate(&e1));
    CUDA_TRY(c, cudaEventRecord(e0, c->stream));
  }
  if (c->opt.arithmetic == 1)
    CUDA_TRY(c, launch_fluid_exact(fa, c->f_state == 1, c->opt.variable_viscosity != 0, c->ip.MaxSurfPointsPerNode,
                                   c->stream));
  else
    CUDA_TRY(c, launch_fluid(fa, c->f_state == 1, c->opt.variable_viscosity != 0, c->opt.collision, c->opt.storage,
                             c->stream));
  if (c->profiling) {
    CUDA_TRY(c, cudaEventRecord(e1, c->stream));
    c->ev_fluid.emplace_back(e0, e1);
  }
  c->cur = 1 - c->cur;
  c->f_state = 2;
  if (c->ppar.np > 0) {
    ParticleArgs pa;
    pa.g = c->g;
    pa.p = c->ppar;
    pa.kin_old = c->kin[c->pcur];
    pa.kin_new = c->kin[1 - c->pcur];
    pa.pff_old = c->pff[c->pcur];
    pa.pff_new = c->pff[1 - c->pcur];
    pa.pf_old = c->pf[c->pcur];
    pa.pf_new = c->pf[1 - c->pcur];
    pa.sphere = c->sphere;
    pa.u = c->u;
    pa.mrec = c->mrec;
    pa.tiles = fa.tiles;
    pa.znd = c->znd;
    pa.parsZone = c->parsZone;
    pa.zoneMembers = c->zoneMembers;
    pa.numParInZone = c->numParInZone;
    pa.revStart = c->revStart;
    pa.revList = c->revList;
    pa.err = c->err;
    pa.t = t;
    // The rigid-body update reads the contact forces of step t-1.
    if (c->side_pending) CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    if (c->profiling) {
      CUDA_TRY(c, cudaEventCreate(&e0));
      CUDA_TRY(c, cudaEventCreate(&e1));
      CUDA_TRY(c, cudaEventRecord(e0, c->stream));
    }
    CUDA_TRY(c, launch_particles(pa, c->stream));
    if (c->profiling) {
      CUDA_TRY(c, cudaEventRecord(e1, c->stream));
      c->ev_part.emplace_back(e0, e1);
    }
    // Contacts from the positions just written, then (when due) the zone
    // lists the contacts of step t+1 use, on the side stream
    // (sim_main.c:410-447: particle_particle_forces, update_particle_zones).
    CUDA_TRY(c, cudaEventRecord(c->ev_fork, c->stream));
    CUDA_TRY(c, cudaStreamWaitEvent(c->side, c->ev_fork, 0));
    CUDA_TRY(c, launch_contacts(pa, c->side));
    c->pcur = 1 - c->pcur;
    if (t % c->opt.rebuild_freq == 0) {
      ZoneArgs za;
      za.p = c->ppar;
      za.kin = c->kin[c->pcur];
      za.parsZone = c->parsZone;
      za.zoneMembers = c->zoneMembers;
      za.numParInZone = c->numParInZone;
      za.zoneOf = c->zoneOf;
      za.err = c->err;
      CUDA_TRY(c, launch_zones(za, c->side));
    }
    CUDA_TRY(c, cudaEventRecord(c->ev_join, c->side));
    c->side_pending = true;
  }
  c->last_t = t;
  return 0;
}

// Orders the side stream's pending work (contacts, zone rebuild) before
// whatever the main stream runs next.
static int join_side(d3q19_ctx* c) {
  if (!c->side_pending) return 0;
  CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->ev_join, 0));
  c->side_pending = false;
  return 0;
}

extern "C" int d3q19_step(d3q19_ctx* c, int t) {
  int rc = check_ready(c);
  if (rc) return rc;
  cudaSetDevice(c->dev);
  if ((rc = enqueue_step(c, t))) return rc;
  return join_side(c);
}

static int gcd_i(int a, int b) { return b ? gcd_i(b, a % b) : a; }

extern "C" int d3q19_run(d3q19_ctx* c, int t0, int nsteps) {
  int rc = check_ready(c);
  if (rc) return rc;
  cudaSetDevice(c->dev);
  // The launch sequence repeats with period Lp in t (buffer parity and the
  // zone-rebuild schedule), so a captured chunk of CH steps replays at any
  // t0 with the same phase and buffer assignment.
  const int R = c->ppar.np > 0 ? c->opt.rebuild_freq : 2;
  const int Lp = 2 / gcd_i(2, R) * R;
  const int CH = Lp * std::max(1, (64 + Lp - 1) / Lp);
  int t = t0, n = nsteps;
  while (n > 0) {
    if (c->f_state != 2 || n < CH || c->profiling) {
      if ((rc = enqueue_step(c, t))) return rc;
      t++;
      n--;
      continue;
    }
    if ((rc = join_side(c))) return rc;
    auto key = std::make_tuple(((t % Lp) + Lp) % Lp, c->cur, c->pcur, CH);
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) {
      const int cur0 = c->cur, pcur0 = c->pcur;
      cudaGraph_t graph;
      CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      for (int k = 0; k < CH && !rc; k++) rc = enqueue_step(c, t + k);
      if (!rc) rc = join_side(c);
      if (rc) {
        cudaStreamEndCapture(c->stream, &graph);
        c->side_pending = false;
        return rc;
      }
      CUDA_TRY(c, cudaStreamEndCapture(c->stream, &graph));
      cudaGraphExec_t exec;
      CUDA_TRY(c, cudaGraphInstantiate(&exec, graph, 0));
      cudaGraphDestroy(graph);
      it = c->graphs.emplace(key, exec).first;
      c->cur = cur0;  // capture only recorded the launches
      c->pcur = pcur0;
    }
    CUDA_TRY(c, cudaGraphLaunch(it->second, c->stream));
    // CH is even: buffer assignment is unchanged after the chunk.
    t += CH;
    n -= CH;
  }
  return join_side(c);
}

static int device_errors(d3q19_ctx* c) {
  unsigned e = 0;
  CUDA_TRY(c, cudaMemcpy(&e, c->err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  c->sticky |= e;
  if (c->sticky & ERR_TILE_OVERFLOW)
    return fail(c, D3Q19_EOVERFLOW, "a lattice tile received more than %d IBM markers; raise ibm_tile_capacity",
                c->tile_cap);
  if (c->sticky & (ERR_NONFINITE | ERR_FIXED_RANGE))
    return fail(c, D3Q19_ENUMERIC, "non-finite or out-of-range density, velocity or marker position on the device");
  if (c->sticky & ERR_ZONE_RANGE) return fail(c, D3Q19_ENUMERIC, "sphere position outside the zone grid");
  return 0;
}

extern "C" int d3q19_synchronize(d3q19_ctx* c) {
  if (!c) return D3Q19_EINVAL;
  cudaSetDevice(c->dev);
  if (int rc = join_side(c)) return rc;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return device_errors(c);
}

template <typename T>
static int readback(d3q19_ctx* c, T* dst, const T* src, size_t n) {
  if (!c || !dst) return D3Q19_EINVAL;
  cudaSetDevice(c->dev);
  if (int rc = join_side(c)) return rc;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  CUDA_TRY(c, cudaMemcpy(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost));
  return device_errors(c);
}

extern "C" int d3q19_read_u(d3q19_ctx* c, float* u) { return c ? readback(c, u, c->u, 3 * c->g.NC) : D3Q19_EINVAL; }
extern "C" int d3q19_read_tau(d3q19_ctx* c, float* t) { return c ? readback(c, t, c->tau, c->g.NC) : D3Q19_EINVAL; }
extern "C" int d3q19_read_parkin(d3q19_ctx* c, float* k) {
  if (!c) return D3Q19_EINVAL;
  if (c->ppar.np == 0) return 0;
  return readback(c, (float4*)k, c->kin[c->pcur], 4 * (size_t)c->ppar.np);
}
extern "C" int d3q19_read_parforce(d3q19_ctx* c, float* k) {
  if (!c) return D3Q19_EINVAL;
  if (c->ppar.np == 0) return 0;
  return readback(c, (float4*)k, c->pf[c->pcur], 2 * (size_t)c->ppar.np);
}
extern "C" int d3q19_read_parfluidforce(d3q19_ctx* c, float* k) {
  if (!c) return D3Q19_EINVAL;
  if (c->ppar.np == 0) return 0;
  return readback(c, (float4*)k, c->pff[c->pcur], 2 * (size_t)c->ppar.np * c->ppar.nfa);
}

static int ensure_scratch(d3q19_ctx* c, size_t bytes) {
  if (c->scratch_bytes >= bytes) return 0;
  if (c->scratch) cudaFree(c->scratch);
  c->scratch = nullptr;
  c->scratch_bytes = 0;
  CUDA_TRY(c, cudaMalloc(&c->scratch, bytes));
  c->scratch_bytes = bytes;
  return 0;
}

extern "C" int d3q19_read_f(d3q19_ctx* c, float* f) {
  if (!c || !f) return D3Q19_EINVAL;
  if (c->f_state == 0) return fail(c, D3Q19_ESTATE, "lattice not written");
  cudaSetDevice(c->dev);
  const long long NC = c->g.NC;
  if (c->f_state == 1 && c->opt.storage == STORE_F32) return readback(c, f, (const float*)c->f[c->cur], 19 * NC);
  int rc = ensure_scratch(c, sizeof(float) * 19 * NC);
  if (rc) return rc;
  if (c->f_state == 1) {
    CUDA_TRY(c, launch_load_f(c->f[c->cur], (float*)c->scratch, NC, c->opt.storage, c->stream));
    return readback(c, f, (const float*)c->scratch, 19 * NC);
  }
  FluidArgs fa;
  memset(&fa, 0, sizeof(fa));
  fa.g = c->g;
  fa.p = c->fpar;
  fa.fin = c->f[c->cur];
  CUDA_TRY(c, cudaMemsetAsync(c->scratch, 0, sizeof(float) * 19 * NC, c->stream));
  CUDA_TRY(c, launch_materialize_f(fa, c->opt.storage, (float*)c->scratch, c->stream));
  return readback(c, f, (const float*)c->scratch, 19 * NC);
}

extern "C" int d3q19_read_spread_force(d3q19_ctx* c, float* gpf0) {
  if (!c || !gpf0) return D3Q19_EINVAL;
  cudaSetDevice(c->dev);
  const long long NC = c->g.NC;
  int rc = ensure_scratch(c, sizeof(float) * 3 * NC);
  if (rc) return rc;
  CUDA_TRY(c, cudaMemsetAsync(c->scratch, 0, sizeof(float) * 3 * NC, c->stream));
  if (c->ppar.np > 0) {
    TileLists tl;
    tl.cap = c->tile_cap;
    tl.count = c->tile_count;
    tl.list = c->tile_list;
    tl.mrec = c->mrec;
    tl.fmax = c->fmax;
    if (c->opt.arithmetic == 1)
      CUDA_TRY(c, launch_spread_field_exact(c->g, tl, c->ip.MaxSurfPointsPerNode, (float*)c->scratch, c->err,
                                            c->stream));
    else
      CUDA_TRY(c, launch_spread_field(c->g, tl, c->last_t, (float*)c->scratch, c->err, c->stream));
  }
  return readback(c, gpf0, (const float*)c->scratch, 3 * NC);
}

extern "C" int d3q19_read_marker_cells(d3q19_ctx* c, int* cells) {
  if (!c || !cells) return D3Q19_EINVAL;
  const long long M = (long long)c->ppar.np * c->ppar.P;
  if (M == 0) return 0;
  cudaSetDevice(c->dev);
  int rc = ensure_scratch(c, sizeof(int) * 3 * M);
  if (rc) return rc;
  CUDA_TRY(c, launch_marker_cells(c->mrec, (int)M, (int*)c->scratch, c->stream));
  return readback(c, cells, (const int*)c->scratch, 3 * M);
}

extern "C" int d3q19_read_zones(d3q19_ctx* c, int* parsZone, int* zoneMembers, int* numParInZone) {
  if (!c) return D3Q19_EINVAL;
  const int np = c->ppar.np;
  if (np == 0) return 0;
  int rc = 0;
  if (parsZone && (rc = readback(c, parsZone, (const int*)c->parsZone, np))) return rc;
  if (zoneMembers && (rc = readback(c, zoneMembers, (const int*)c->zoneMembers, (size_t)c->nzones * np))) return rc;
  if (numParInZone && (rc = readback(c, numParInZone, (const int*)c->numParInZone, c->nzones))) return rc;
  return 0;
}

extern "C" long long d3q19_tau_clamp_count(d3q19_ctx* c) {
  if (!c) return -1;
  unsigned long long v = 0;
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->stream);
  cudaMemcpy(&v, c->clamps, sizeof(v), cudaMemcpyDeviceToHost);
  return (long long)v;
}

static void drop_events(d3q19_ctx* c) {
  for (auto& e : c->ev_fluid) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  for (auto& e : c->ev_part) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  c->ev_fluid.clear();
  c->ev_part.clear();
}

extern "C" int d3q19_profile(d3q19_ctx* c, int enable) {
  if (!c) return D3Q19_EINVAL;
  cudaSetDevice(c->dev);
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (enable) drop_events(c);
  c->profiling = enable != 0;
  return 0;
}

extern "C" int d3q19_profile_read(d3q19_ctx* c, double* fluid_ms, int* nf, double* part_ms, int* npart) {
  if (!c) return D3Q19_EINVAL;
  cudaSetDevice(c->dev);
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  double a = 0.0, b = 0.0;
  for (auto& e : c->ev_fluid) {
    float ms = 0.0f;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, e.first, e.second));
    a += ms;
  }
  for (auto& e : c->ev_part) {
    float ms = 0.0f;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, e.first, e.second));
    b += ms;
  }
  if (fluid_ms) *fluid_ms = a;
  if (nf) *nf = (int)c->ev_fluid.size();
  if (part_ms) *part_ms = b;
  if (npart) *npart = (int)c->ev_part.size();
  return 0;
}

extern "C" void* d3q19_stream(d3q19_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" const char* d3q19_last_error(d3q19_ctx* c) { return c ? c->msg : g_create_error; }

extern "C" int d3q19_destroy(d3q19_ctx* c) {
  if (!c) return D3Q19_EINVAL;
  cudaSetDevice(c->dev);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->side) cudaStreamSynchronize(c->side);
  for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
  drop_events(c);
  void* ptrs[] = {c->f[0], c->f[1], c->u, c->tau, c->kin[0], c->kin[1], c->pff[0], c->pff[1], c->pf[0], c->pf[1],
                  c->sphere, c->mrec, c->tile_count, c->fmax, c->tile_list, c->znd, c->parsZone, c->zoneMembers,
                  c->numParInZone, c->revStart, c->revList, c->zoneOf, c->err, c->clamps, c->scratch};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  delete c;
  return 0;
}

/* ---------------------------------------------------------------------------
 * Spread force field read-back that allocates nothing.
 *
 * d3q19_read_spread_force builds the 3*N_C-float field in the context's
 * scratch buffer, which it grows with cudaFree + cudaMalloc when a larger
 * read-back comes along.  Two kinds of caller cannot accept that: an output
 * or monitoring thread that samples the field while other contexts on the
 * same device keep stepping (cudaFree waits for the whole device, so the
 * sample would stall every other simulation on it), and a process that has
 * committed the device memory to lattices up to its budget, where a
 * read-back must not fail for want of memory half-way through a run.  This
 * variant builds the field in a fixed array of the library's own device image
 * instead, so it needs no memory beyond what the library was loaded with.
 *
 * Limit: N_C <= D3Q19_STATIC_SPREAD_MAX_CELLS (3 floats a node, 3 MiB).
 * The array exists once per device and process: calls that overlap in time on
 * one device (two host threads, or two contexts on the same device) write the
 * same array and race.  The first call on each device looks the array's
 * address up (and with lazy module loading that makes the runtime load this
 * file's device image); make that first call before any stream capture.
 * ------------------------------------------------------------------------- */
static __device__ __align__(256) float g_spread_static[3 * D3Q19_STATIC_SPREAD_MAX_CELLS];

static constexpr int kStaticMaxDevices = 64;
static std::mutex g_spread_static_mu;
static float* g_spread_static_ptr[kStaticMaxDevices] = {nullptr};

/* Once per device, with that device current: the device address of
 * g_spread_static. */
static int spread_static_address(d3q19_ctx* c, float** out) {
  std::lock_guard<std::mutex> lock(g_spread_static_mu);
  if (c->dev < 0 || c->dev >= kStaticMaxDevices)
    return fail(c, D3Q19_EINVAL, "device %d: the static spread buffer is tracked for devices 0..%d only", c->dev,
                kStaticMaxDevices - 1);
  if (!g_spread_static_ptr[c->dev]) {
    CUDA_TRY(c, cudaSetDevice(c->dev));
    float* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_spread_static);
    if (e != cudaSuccess || !ptr)
      return fail(c, D3Q19_ECUDA, "cudaGetSymbolAddress(g_spread_static) on device %d: %s", c->dev,
                  cudaGetErrorString(e));
    g_spread_static_ptr[c->dev] = ptr;
  }
  *out = g_spread_static_ptr[c->dev];
  return 0;
}

extern "C" int d3q19_read_spread_force_static(d3q19_ctx* c, float* gpf0) {
  if (!c || !gpf0) return D3Q19_EINVAL;
  const long long NC = c->g.NC;
  if (NC > (long long)D3Q19_STATIC_SPREAD_MAX_CELLS)
    return fail(c, D3Q19_EINVAL,
                "lattice of %lld nodes exceeds the %d nodes of the static spread buffer; use d3q19_read_spread_force",
                NC, (int)D3Q19_STATIC_SPREAD_MAX_CELLS);
  float* field = nullptr;
  int rc = spread_static_address(c, &field);
  if (rc) return rc;
  cudaSetDevice(c->dev);
  /* Nodes no marker reaches read 0, and the spread kernels add into the
   * field: the used part starts at zero on every call. */
  CUDA_TRY(c, cudaMemsetAsync(field, 0, sizeof(float) * 3 * NC, c->stream));
  if (c->ppar.np > 0) {
    TileLists tl;
    tl.cap = c->tile_cap;
    tl.count = c->tile_count;
    tl.list = c->tile_list;
    tl.mrec = c->mrec;
    tl.fmax = c->fmax;
    if (c->opt.arithmetic == 1)
      CUDA_TRY(c, launch_spread_field_exact(c->g, tl, c->ip.MaxSurfPointsPerNode, field, c->err, c->stream));
    else
      CUDA_TRY(c, launch_spread_field(c->g, tl, c->last_t, field, c->err, c->stream));
  }
  return readback(c, gpf0, (const float*)field, 3 * NC);
}
