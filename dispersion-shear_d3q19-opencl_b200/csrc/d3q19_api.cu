// d3q19_api.cu -- the C ABI (include/d3q19_b200.h): context, device memory,
// the per-step launch sequence, CUDA-graph replay and the read-backs.
#include "../../include/d3q19_b200.h"
#include "d3q19_internal.h"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

static_assert(sizeof(int_param_struct) == 332, "int_param_struct must match struct_header_device.h");
static_assert(sizeof(flp_param_struct) == 176, "flp_param_struct must match struct_header_device.h");

using namespace d3q19;

// NVTX range over an entry point: named spans on the host timeline of a
// profiler such as Nsight Systems; no cost when no tool is attached.
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};
#define TRACE(name) TraceRange trace_range_(name)

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
  // Pass-by-pass stepping (d3q19_k_*): 0 next is the collide-stream pass,
  // 1 the particle pass, 2 the contacts of step kt.
  int kstage = 0;
  int kt = 0;
  Geom g;
  FluidParams fpar;
  ParticleParams ppar;
  void* f[2] = {nullptr, nullptr};  // float, or 16-bit shifted storage (opt.storage)
  int cur = 0;         // f[cur] is what the next step reads
  int f_state = 0;     // 0 unset, 1 reference state (pre-collision), 2 post-collision
  float* u = nullptr;
  float* tau = nullptr;
  double* tau64 = nullptr;  // arithmetic = 2: the local tau in double
  float4* kin[2] = {nullptr, nullptr};
  // particle_precision = 1: sphere state and force/torque partials in double
  // (the float buffers hold rounded copies for read-back and the contacts).
  double* kin64[2] = {nullptr, nullptr};
  double* pff64[2] = {nullptr, nullptr};
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
  // The TMA-pipelined collide-stream kernel (d3q19_tma.cu) and its tensor
  // maps, when the context allows it (fluid_kernel 0).
  TmaMaps tma;
  bool use_tma = false;
  unsigned* err = nullptr;
  unsigned long long* clamps = nullptr;
  double* pstats = nullptr;  // per-plane FP64 sums [5 * Nz]
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  bool have_particles = false, have_zones = false;
  unsigned sticky = 0;
  // A member of a lattice pool takes its device memory from the pool's
  // stream-ordered memory pool (allocated on its own stream); its release
  // frees it in the order of free_stream, after the pool's work in flight,
  // without waiting for the device.
  cudaMemPool_t mempool = nullptr;
  cudaStream_t free_stream = nullptr;
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

static cudaError_t dev_alloc(d3q19_ctx* c, void** p, size_t bytes) {
  return c->mempool ? cudaMallocFromPoolAsync(p, bytes, c->mempool, c->stream) : cudaMalloc(p, bytes);
}

static void dev_free(d3q19_ctx* c, void* p) {
  if (!p) return;
  if (c->mempool) cudaFreeAsync(p, c->free_stream ? c->free_stream : c->stream);
  else cudaFree(p);
}

template <typename T>
static int dalloc(d3q19_ctx* c, T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = dev_alloc(c, (void**)p, n * sizeof(T));
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
  if (o->arithmetic < 0 || o->arithmetic > 2) return fail(nullptr, D3Q19_EINVAL, "arithmetic must be 0, 1 or 2");
  if (o->inplace != 0 && o->inplace != 1) return fail(nullptr, D3Q19_EINVAL, "inplace must be 0 or 1");
  if (o->inplace && o->arithmetic == 1)
    return fail(nullptr, D3Q19_EINVAL, "in-place streaming is not available with the reference's evaluation order");
  if (o->arithmetic == 2 && (o->collision != 0 || o->storage != 0))
    return fail(nullptr, D3Q19_EINVAL, "the FP64 build runs the reference's MRT on FP64 distributions only");
  if (o->arithmetic == 1 && o->collision != 0)
    return fail(nullptr, D3Q19_EINVAL, "the reference-exact arithmetic implements the reference's MRT only");
  if (o->periodic_smoothing != 0 && o->periodic_smoothing != 1)
    return fail(nullptr, D3Q19_EINVAL, "periodic_smoothing must be 0 or 1");
  if (o->arithmetic == 1 && o->periodic_smoothing)
    return fail(nullptr, D3Q19_EINVAL, "the reference-exact arithmetic smooths the force as the reference does");
  if (o->arithmetic == 1 && (o->tau_max != 0.0f || o->tau_min != 0.0f || o->casson_reg != 0.0f))
    return fail(nullptr, D3Q19_EINVAL, "the reference-exact arithmetic has the reference's tau limits only");
  if (o->arithmetic == 1 && (ip->MaxSurfPointsPerNode < 1 || ip->MaxSurfPointsPerNode > 16))
    return fail(nullptr, D3Q19_EINVAL, "MaxSurfPointsPerNode must be in [1, 16] for the reference-exact arithmetic");
  if (o->storage < 0 || o->storage > 2)
    return fail(nullptr, D3Q19_EINVAL, "storage %d (0 FP32, 1 FP16 shifted, 2 BF16 shifted)", o->storage);
  if (o->arithmetic == 1 && o->storage != 0)
    return fail(nullptr, D3Q19_EINVAL, "the reference-exact arithmetic stores FP32 distributions only");
  if (o->particle_precision < 0 || o->particle_precision > 1)
    return fail(nullptr, D3Q19_EINVAL, "particle_precision %d (0 FP32, 1 FP64)", o->particle_precision);
  if (o->particle_precision == 1 && o->arithmetic == 1)
    return fail(nullptr, D3Q19_EINVAL, "the reference-exact arithmetic keeps the reference's FP32 particle state");
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

static int create_ctx(const int_param_struct* ip, const flp_param_struct* fp, const d3q19_options* opt,
                      cudaMemPool_t mempool, d3q19_ctx** out);

extern "C" int d3q19_create(const int_param_struct* ip, const flp_param_struct* fp, const d3q19_options* opt,
                            d3q19_ctx** out) {
  TRACE("d3q19_create");
  return create_ctx(ip, fp, opt, nullptr, out);
}

static int create_ctx(const int_param_struct* ip, const flp_param_struct* fp, const d3q19_options* opt,
                      cudaMemPool_t mempool, d3q19_ctx** out) {
  if (!ip || !fp || !out) return fail(nullptr, D3Q19_EINVAL, "null argument");
  d3q19_options o;
  memset(&o, 0, sizeof(o));
  if (opt) o = *opt;
  if (o.rebuild_freq <= 0) o.rebuild_freq = 10;  // the reference's default (D3Q19-OpenCL.c:60)
  int rc = validate(ip, fp, &o);
  if (rc) return rc;
  if (o.arithmetic == 2) {  // the FP64 build: FP64 distributions and particles
    o.storage = STORE_F64;
    o.particle_precision = 1;
  }
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
  c->mempool = mempool;
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
  p.variable = o.variable_viscosity ? 1 : 0;
  p.periodicSmooth = o.periodic_smoothing ? 1 : 0;

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
  pp.periodicSmooth = o.periodic_smoothing ? 1 : 0;

  const long long NC = g.NC;
  const size_t fbytes = (size_t)storage_bytes(o.storage) * 19 * NC;
  // In place: one buffer, under both names (fin == fout).
  if ((rc = dalloc(c, (char**)&c->f[0], fbytes)) ||
      (o.inplace ? (c->f[1] = c->f[0], 0) : (rc = dalloc(c, (char**)&c->f[1], fbytes))) ||
      (rc = dalloc(c, &c->u, 3 * NC)) ||
      (rc = dalloc(c, &c->tau, NC)) || (rc = dalloc(c, &c->err, 1)) || (rc = dalloc(c, &c->clamps, 1)) ||
      (rc = dalloc(c, &c->pstats, 5LL * g.Nz)) || (o.arithmetic == 2 && (rc = dalloc(c, &c->tau64, NC)))) {
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
      if (!rc && o.particle_precision == 1) rc = dalloc(c, &c->kin64[b], 16 * (long long)np);
      if (!rc && o.particle_precision == 1) rc = dalloc(c, &c->pff64[b], 8LL * np * pp.nfa);
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
  if (o.fluid_kernel == 1 && o.arithmetic == 0 && o.collision == 0 && tma_supported(g, o.storage))
    c->use_tma = tma_make_maps(&c->tma, c->f, g, o.storage);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    snprintf(g_create_error, sizeof(g_create_error), "initialisation failed");
    d3q19_destroy(c);
    return D3Q19_ECUDA;
  }
  *out = c;
  return 0;
}

extern "C" int d3q19_fluid_kernel(const d3q19_ctx* c) {
  if (!c) return D3Q19_EINVAL;
  return c->opt.arithmetic == 1 ? 2 : (c->use_tma ? 1 : 0);
}

extern "C" int d3q19_write_lattice(d3q19_ctx* c, const float* f, const float* u, const float* tau_lb) {
  if (!c || !f || !u) return D3Q19_EINVAL;
  cudaSetDevice(c->dev);
  if (c->opt.inplace) c->cur = 0;  // the uploaded layout is the one even steps read
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
  if (c->tau64) CUDA_TRY(c, launch_widen(c->tau, c->tau64, NC, c->stream));
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
  if (c->kin64[b]) {
    CUDA_TRY(c, launch_widen((const float*)c->kin[b], c->kin64[b], 16LL * np, c->stream));
    CUDA_TRY(c, launch_widen((const float*)c->pff[b], c->pff64[b], 8LL * np * c->ppar.nfa, c->stream));
  }
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

// Kernel arguments of step t with buffer parities cur (distributions) and
// pcur (particle state).
static FluidArgs fluid_args(const d3q19_ctx* c, int t, int cur) {
  FluidArgs fa;
  memset(&fa, 0, sizeof(fa));
  fa.g = c->g;
  fa.p = c->fpar;
  fa.t = t;
  fa.fin = c->f[cur];
  fa.fout = c->f[1 - cur];
  fa.u = c->u;
  fa.tau = c->tau;
  fa.tau64 = c->tau64;
  fa.tiles.cap = c->tile_cap;
  fa.tiles.count = c->tile_count;
  fa.tiles.list = c->tile_list;
  fa.tiles.mrec = c->mrec;
  fa.tiles.fmax = c->fmax;
  fa.tiles.markers = (long long)c->ppar.np * c->ppar.P;
  fa.has_ibm = c->ppar.np > 0;
  fa.err = c->err;
  fa.clamps = c->clamps;
  fa.inplace = c->opt.inplace ? (cur == 0 ? 1 : 2) : 0;  // even steps read buffer parity 0
  return fa;
}

static ParticleArgs particle_args(const d3q19_ctx* c, int t, int pcur) {
  ParticleArgs pa;
  memset(&pa, 0, sizeof(pa));
  pa.g = c->g;
  pa.p = c->ppar;
  pa.kin_old = c->kin[pcur];
  pa.kin_new = c->kin[1 - pcur];
  pa.pff_old = c->pff[pcur];
  pa.pff_new = c->pff[1 - pcur];
  pa.pf_old = c->pf[pcur];
  pa.pf_new = c->pf[1 - pcur];
  pa.sphere = c->sphere;
  pa.u = c->u;
  pa.mrec = c->mrec;
  pa.tiles.cap = c->tile_cap;
  pa.tiles.count = c->tile_count;
  pa.tiles.list = c->tile_list;
  pa.tiles.mrec = c->mrec;
  pa.tiles.fmax = c->fmax;
  pa.tiles.markers = (long long)c->ppar.np * c->ppar.P;
  pa.znd = c->znd;
  pa.parsZone = c->parsZone;
  pa.zoneMembers = c->zoneMembers;
  pa.numParInZone = c->numParInZone;
  pa.revStart = c->revStart;
  pa.revList = c->revList;
  pa.err = c->err;
  pa.t = t;
  pa.p64 = c->kin64[0] != nullptr;
  pa.kin64_old = c->kin64[pcur];
  pa.kin64_new = c->kin64[1 - pcur];
  pa.pff64_old = c->pff64[pcur];
  pa.pff64_new = c->pff64[1 - pcur];
  return pa;
}

// Zone rebuild from the particle state in kin[pnew].
static ZoneArgs zone_args(const d3q19_ctx* c, int pnew) {
  ZoneArgs za;
  memset(&za, 0, sizeof(za));
  za.p = c->ppar;
  za.kin = c->kin[pnew];
  za.parsZone = c->parsZone;
  za.zoneMembers = c->zoneMembers;
  za.numParInZone = c->numParInZone;
  za.zoneOf = c->zoneOf;
  za.err = c->err;
  return za;
}

// The collide-stream pass of step t on the context's stream.
static cudaError_t fluid_pass(d3q19_ctx* c, const FluidArgs& fa) {
  const bool first = c->f_state == 1;
  if (c->opt.arithmetic == 1)
    return launch_fluid_exact(fa, first, c->opt.variable_viscosity != 0, c->ip.MaxSurfPointsPerNode, c->stream);
  if (c->use_tma) return launch_fluid_tma(c->tma, c->cur, fa, first, c->opt.storage, c->stream);
  return launch_fluid(fa, first, c->opt.variable_viscosity != 0, c->opt.collision, c->opt.storage, c->stream);
}

static int enqueue_step(d3q19_ctx* c, int t) {
  const FluidArgs fa = fluid_args(c, t, c->cur);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->profiling) {
    CUDA_TRY(c, cudaEventCreate(&e0));
    CUDA_TRY(c, cudaEventCreate(&e1));
    CUDA_TRY(c, cudaEventRecord(e0, c->stream));
  }
  CUDA_TRY(c, fluid_pass(c, fa));
  if (c->profiling) {
    CUDA_TRY(c, cudaEventRecord(e1, c->stream));
    c->ev_fluid.emplace_back(e0, e1);
  }
  c->cur = 1 - c->cur;
  c->f_state = 2;
  if (c->ppar.np > 0) {
    const ParticleArgs pa = particle_args(c, t, c->pcur);
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
    if (t % c->opt.rebuild_freq == 0) CUDA_TRY(c, launch_zones(zone_args(c, c->pcur), c->side));
    CUDA_TRY(c, cudaEventRecord(c->ev_join, c->side));
    c->side_pending = true;
  }
  c->last_t = t;
  return 0;
}

// ---------------------------------------------------------------------------
// The step pass by pass, in the reference's kernel order (sim_main.c:324-447),
// all on the context's stream.
extern "C" int d3q19_k_collide_stream(d3q19_ctx* c, int t) {
  int rc = check_ready(c);
  if (rc) return rc;
  if (c->kstage != 0) return fail(c, D3Q19_ESTATE, "the particle pass of step %d comes first", c->kt);
  cudaSetDevice(c->dev);
  if (c->side_pending) CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->ev_join, 0));
  c->side_pending = false;
  const FluidArgs fa = fluid_args(c, t, c->cur);
  CUDA_TRY(c, fluid_pass(c, fa));
  c->cur = 1 - c->cur;
  c->f_state = 2;
  c->last_t = t;
  c->kt = t;
  c->kstage = c->ppar.np > 0 ? 1 : 0;
  return 0;
}

extern "C" int d3q19_k_particles(d3q19_ctx* c, int t) {
  if (!c) return D3Q19_EINVAL;
  if (c->ppar.np == 0) return 0;
  if (c->kstage != 1 || t != c->kt) return fail(c, D3Q19_ESTATE, "the collide-stream pass of step %d comes first", t);
  cudaSetDevice(c->dev);
  CUDA_TRY(c, launch_particles(particle_args(c, t, c->pcur), c->stream));
  c->kstage = 2;
  return 0;
}

extern "C" int d3q19_k_contacts(d3q19_ctx* c, int t) {
  if (!c) return D3Q19_EINVAL;
  if (c->ppar.np == 0) return 0;
  if (c->kstage != 2 || t != c->kt) return fail(c, D3Q19_ESTATE, "the particle pass of step %d comes first", t);
  cudaSetDevice(c->dev);
  CUDA_TRY(c, launch_contacts(particle_args(c, t, c->pcur), c->stream));
  c->pcur = 1 - c->pcur;
  c->kstage = 0;
  return 0;
}

extern "C" int d3q19_k_zones(d3q19_ctx* c) {
  if (!c) return D3Q19_EINVAL;
  if (c->ppar.np == 0) return 0;
  if (c->kstage != 0) return fail(c, D3Q19_ESTATE, "the contacts of step %d come first", c->kt);
  cudaSetDevice(c->dev);
  CUDA_TRY(c, launch_zones(zone_args(c, c->pcur), c->stream));
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
  TRACE("d3q19_step");
  int rc = check_ready(c);
  if (rc) return rc;
  if (c->kstage != 0) return fail(c, D3Q19_ESTATE, "step %d was left between passes", c->kt);
  cudaSetDevice(c->dev);
  if ((rc = enqueue_step(c, t))) return rc;
  return join_side(c);
}

static int gcd_i(int a, int b) { return b ? gcd_i(b, a % b) : a; }

// The CUDA graph of L steps starting at step t with the context's current
// buffer parities (captured on first use; the capture records the launches
// without running them and leaves the context's state as it was).
static int step_graph(d3q19_ctx* c, int t, int L, int Lp, cudaGraphExec_t* out) {
  auto key = std::make_tuple(((t % Lp) + Lp) % Lp, c->cur, c->pcur, L);
  auto it = c->graphs.find(key);
  if (it == c->graphs.end()) {
    int rc = join_side(c);
    if (rc) return rc;
    const int cur0 = c->cur, pcur0 = c->pcur, last0 = c->last_t;
    cudaGraph_t graph;
    CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < L && !rc; k++) rc = enqueue_step(c, t + k);
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
    c->cur = cur0;  // the capture only recorded the launches
    c->pcur = pcur0;
    c->last_t = last0;
  }
  *out = it->second;
  return 0;
}

// The launch sequence repeats with period Lp in t (buffer parity and the
// zone-rebuild schedule), so a captured chunk replays at any t with the same
// phase and buffer assignment.  Chunks are CH steps; a shorter rest of at
// least Lp steps replays a graph of the largest multiple of Lp when one was
// captured before (d3q19_prepare_run), and steps one by one otherwise.
static void run_schedule(const d3q19_ctx* c, int* Lp, int* CH) {
  const int R = c->ppar.np > 0 ? c->opt.rebuild_freq : 2;
  *Lp = 2 / gcd_i(2, R) * R;
  *CH = *Lp * std::max(1, (64 + *Lp - 1) / *Lp);
}

extern "C" int d3q19_run(d3q19_ctx* c, int t0, int nsteps) {
  TRACE("d3q19_run");
  int rc = check_ready(c);
  if (rc) return rc;
  if (c->kstage != 0) return fail(c, D3Q19_ESTATE, "step %d was left between passes", c->kt);
  cudaSetDevice(c->dev);
  int Lp, CH;
  run_schedule(c, &Lp, &CH);
  int t = t0, n = nsteps;
  while (n > 0) {
    int L = 0;
    if (c->f_state == 2 && !c->profiling) {
      if (n >= CH) {
        L = CH;
      } else if (n >= Lp) {
        const int Ls = n / Lp * Lp;
        if (c->graphs.count(std::make_tuple(((t % Lp) + Lp) % Lp, c->cur, c->pcur, Ls))) L = Ls;
      }
    }
    if (L == 0) {
      if ((rc = enqueue_step(c, t))) return rc;
      t++;
      n--;
      continue;
    }
    if ((rc = join_side(c))) return rc;
    cudaGraphExec_t exec;
    if ((rc = step_graph(c, t, L, Lp, &exec))) return rc;
    CUDA_TRY(c, cudaGraphLaunch(exec, c->stream));
    // L is even: the buffer assignment is unchanged after the chunk.
    t += L;
    n -= L;
    c->last_t = t - 1;
  }
  return join_side(c);
}

extern "C" int d3q19_prepare_run(d3q19_ctx* c, int t0, int nsteps) {
  TRACE("d3q19_prepare_run");
  int rc = check_ready(c);
  if (rc) return rc;
  if (c->kstage != 0) return fail(c, D3Q19_ESTATE, "step %d was left between passes", c->kt);
  if (c->f_state != 2) return 0;  // the first step after an upload runs one by one; prepare after it
  cudaSetDevice(c->dev);
  int Lp, CH;
  run_schedule(c, &Lp, &CH);
  int t = t0, n = nsteps;
  while (n >= Lp) {
    const int L = n >= CH ? CH : n / Lp * Lp;
    cudaGraphExec_t exec;
    if ((rc = step_graph(c, t, L, Lp, &exec))) return rc;
    t += L;
    n -= L;
  }
  return 0;
}

static int device_errors(d3q19_ctx* c) {
  unsigned e = 0;
  CUDA_TRY(c, cudaMemcpy(&e, c->err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  c->sticky |= e;
  if (c->sticky & ERR_TILE_OVERFLOW)
    return fail(c, D3Q19_EOVERFLOW, "a lattice tile received more than %d IBM markers; raise ibm_tile_capacity",
                c->tile_cap);
  if (c->sticky & ERR_BOUNDS)
    return fail(c, D3Q19_EBOUNDS, "an index check of the bounds-checked build failed (the access was skipped)");
  if (c->sticky & (ERR_NONFINITE | ERR_FIXED_RANGE))
    return fail(c, D3Q19_ENUMERIC, "non-finite or out-of-range density, velocity or marker position on the device");
  if (c->sticky & ERR_ZONE_RANGE) return fail(c, D3Q19_ENUMERIC, "sphere position outside the zone grid");
  if (c->sticky & ERR_TIMEOUT)
    return fail(c, D3Q19_ETIMEDOUT, "a TMA load of the collide-stream pass did not complete within its limit");
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
extern "C" int d3q19_read_parkin64(d3q19_ctx* c, double* k) {
  if (!c) return D3Q19_EINVAL;
  if (c->ppar.np == 0) return 0;
  if (!c->kin64[0]) return fail(c, D3Q19_ESTATE, "the particle state is FP32 (particle_precision = 0)");
  return readback(c, k, (const double*)c->kin64[c->pcur], 16 * (size_t)c->ppar.np);
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
  dev_free(c, c->scratch);
  c->scratch = nullptr;
  c->scratch_bytes = 0;
  CUDA_TRY(c, dev_alloc(c, &c->scratch, bytes));
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
  fa.inplace = c->opt.inplace ? (c->cur == 0 ? 1 : 2) : 0;
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
    tl.markers = (long long)c->ppar.np * c->ppar.P;
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

// Per-plane FP64 sums (plane_stats_kernel) of the last step, read back.
extern "C" int d3q19_plane_stats(d3q19_ctx* c, double* out) {
  TRACE("d3q19_plane_stats");
  if (!c || !out) return D3Q19_EINVAL;
  if (c->f_state == 0) return fail(c, D3Q19_ESTATE, "lattice not written");
  cudaSetDevice(c->dev);
  if (int rc = join_side(c)) return rc;
  CUDA_TRY(c, launch_plane_stats(c->g, c->u, c->tau, c->fp.NewtonianTau, c->opt.variable_viscosity, c->pstats,
                                 c->stream));
  return readback(c, out, (const double*)c->pstats, 5 * (size_t)c->g.Nz);
}

extern "C" int d3q19_shear_profile(d3q19_ctx* c, double* u_mean, double* wall_rate, double* region_rate) {
  if (!c) return D3Q19_EINVAL;
  const int Nz = c->g.Nz;
  std::vector<double> ps(5 * (size_t)Nz);
  if (int rc = d3q19_plane_stats(c, ps.data())) return rc;
  const double nxy = (double)(c->g.Nx - 2) * (c->g.Ny - 2);
  auto ux = [&](int z) { return ps[5 * (size_t)z] / nxy; };
  if (u_mean) {
    for (int z = 0; z < Nz; z++)
      for (int d = 0; d < 3; d++) u_mean[3 * z + d] = (z >= 1 && z <= Nz - 2) ? ps[5 * (size_t)z + d] / nxy : 0.0;
  }
  if (wall_rate) {
    // compute_shear_stress (D3Q19-OpenCL.c:690-725): forward differences over
    // dz = 4 ending on plane 1 + dz + 1 and on plane Nz - 3, summed and
    // divided by twice the plane's node count.
    const int dz = 4, zA = 1 + dz + 1, zB = Nz - 2 - 1;
    double sum = 0.0;
    if (zA >= 1 && zA <= Nz - 2 && zA - dz >= 0) sum += (ps[5 * (size_t)zA] - ps[5 * (size_t)(zA - dz)]) / dz;
    if (zB != zA && zB >= 1 && zB <= Nz - 2 && zB - dz >= 0) sum += (ps[5 * (size_t)zB] - ps[5 * (size_t)(zB - dz)]) / dz;
    *wall_rate = sum / (2.0 * nxy);
  }
  if (region_rate) {
    // D3Q19-OpenCL.c:739-744: across the planes that spheres can reach.  The
    // reference indexes its profile without a range check; planes outside
    // the lattice give 0 here, planes 0 and Nz-1 have a zero mean.
    const int ib = (int)(c->fp.ParticleZBuffer + 1E-8) + (int)(c->fp.ParticleDiam / 2);
    const int zbL = 1 + ib, zbU = Nz - 2 - ib;
    const bool ok = zbL >= 0 && zbL < Nz && zbU >= 0 && zbU < Nz && zbU != zbL;
    *region_rate = ok ? (ux(zbU) - ux(zbL)) / (zbU - zbL) : 0.0;
  }
  return 0;
}

extern "C" int d3q19_mean_stress(d3q19_ctx* c, double* stress_xz, double* shear_rate, double* eff_viscosity) {
  TRACE("d3q19_mean_stress");
  if (!c) return D3Q19_EINVAL;
  const int Nz = c->g.Nz;
  std::vector<double> ps(5 * (size_t)Nz);
  if (int rc = d3q19_plane_stats(c, ps.data())) return rc;
  double g = 0.0, t = 0.0;
  for (int z = 1; z <= Nz - 2; z++) {
    g += ps[5 * (size_t)z + 3];
    t += ps[5 * (size_t)z + 4];
  }
  const double n = (double)(c->g.Nx - 2) * (c->g.Ny - 2) * (Nz - 2);
  if (stress_xz) *stress_xz = t / n;
  if (shear_rate) *shear_rate = g / n;
  if (eff_viscosity) *eff_viscosity = g != 0.0 ? t / g : 0.0;
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
  if (c->f[1] == c->f[0]) c->f[1] = nullptr;  // in place: one buffer
  void* ptrs[] = {c->f[0], c->f[1], c->u, c->tau, c->kin[0], c->kin[1], c->pff[0], c->pff[1], c->pf[0], c->pf[1],
                  c->sphere, c->mrec, c->tile_count, c->fmax, c->tile_list, c->znd, c->parsZone, c->zoneMembers,
                  c->numParInZone, c->revStart, c->revList, c->zoneOf, c->err, c->clamps, c->pstats, c->scratch,
                  c->tau64, c->kin64[0], c->kin64[1], c->pff64[0], c->pff64[1]};
  for (void* p : ptrs) dev_free(c, p);
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
  CUDA_TRY(c, cudaSetDevice(c->dev));
  /* The spread kernels write the nodes of the tiles that have markers; every
   * other node (tiles without markers, the buffer layer) must read 0, and the
   * array still holds the last call's field: clear the used part first. */
  CUDA_TRY(c, cudaMemsetAsync(field, 0, sizeof(float) * 3 * NC, c->stream));
  if (c->ppar.np > 0) {
    TileLists tl;
    tl.cap = c->tile_cap;
    tl.count = c->tile_count;
    tl.list = c->tile_list;
    tl.mrec = c->mrec;
    tl.fmax = c->fmax;
    tl.markers = (long long)c->ppar.np * c->ppar.P;
    if (c->opt.arithmetic == 1)
      CUDA_TRY(c, launch_spread_field_exact(c->g, tl, c->ip.MaxSurfPointsPerNode, field, c->err, c->stream));
    else
      CUDA_TRY(c, launch_spread_field(c->g, tl, c->last_t, field, c->err, c->stream));
  }
  return readback(c, gpf0, (const float*)field, 3 * NC);
}

/* ---------------------------------------------------------------------------
 * Checkpoints: the whole device state of a context in one host buffer.
 * ------------------------------------------------------------------------- */
namespace {
struct CkptHeader {
  char magic[8];
  int version;
  int storage, p64, arithmetic;
  long long NC, ntiles;
  int np, nfa, P, cap, nzones;
  int f_state, last_t, sticky;
  int inplace, phase;  // in place: the buffer parity the next step reads (the layout of f)
  long long clamps;
};
// The device blocks of a checkpoint in order: {pointer, bytes}.
struct CkptBlock {
  void* ptr;
  size_t bytes;
  const char* name;
};
std::vector<CkptBlock> ckpt_blocks(d3q19_ctx* c) {
  const long long NC = c->g.NC;
  std::vector<CkptBlock> b;
  b.push_back({c->f[c->cur], (size_t)storage_bytes(c->opt.storage) * 19 * NC, "f"});
  b.push_back({c->u, sizeof(float) * 3 * NC, "u"});
  b.push_back({c->tau, sizeof(float) * NC, "tau"});
  if (c->tau64) b.push_back({c->tau64, sizeof(double) * NC, "tau64"});
  const long long np = c->ppar.np;
  if (np > 0) {
    const long long M = np * c->ppar.P, nfa = c->ppar.nfa;
    b.push_back({c->kin[c->pcur], sizeof(float4) * 4 * np, "kin"});
    b.push_back({c->pf[c->pcur], sizeof(float4) * 2 * np, "pf"});
    b.push_back({c->pff[c->pcur], sizeof(float4) * 2 * np * nfa, "pff"});
    if (c->kin64[0]) {
      b.push_back({c->kin64[c->pcur], sizeof(double) * 16 * np, "kin64"});
      b.push_back({c->pff64[c->pcur], sizeof(double) * 8 * np * nfa, "pff64"});
    }
    b.push_back({c->sphere, sizeof(float4) * c->ppar.P, "sphere"});
    b.push_back({c->mrec, sizeof(float4) * 2 * M, "mrec"});
    b.push_back({c->tile_count, sizeof(int) * c->ntiles, "tile_count"});
    b.push_back({c->tile_list, sizeof(int) * c->ntiles * c->tile_cap, "tile_list"});
    b.push_back({c->fmax, sizeof(unsigned) * 2, "fmax"});
    const long long Z = c->nzones;
    b.push_back({c->znd, sizeof(int) * 28 * Z, "znd"});
    b.push_back({c->parsZone, sizeof(int) * np, "parsZone"});
    b.push_back({c->zoneMembers, sizeof(int) * Z * np, "zoneMembers"});
    b.push_back({c->numParInZone, sizeof(int) * Z, "numParInZone"});
    b.push_back({c->revStart, sizeof(int) * (Z + 1), "revStart"});
    b.push_back({c->revList, sizeof(int) * 27 * Z, "revList"});
    b.push_back({c->zoneOf, sizeof(int) * np, "zoneOf"});
  }
  return b;
}

// The integer tables of a checkpoint index device arrays: before they are
// uploaded, every entry the kernels follow must lie inside its array (a
// damaged buffer is refused instead of making a kernel read out of bounds).
const char* ckpt_tables_invalid(d3q19_ctx* c, const char* data) {
  const long long np = c->ppar.np;
  if (np == 0) return nullptr;
  const long long M = np * c->ppar.P, Z = c->nzones, cap = c->tile_cap;
  const int *tile_count = nullptr, *tile_list = nullptr, *znd = nullptr, *members = nullptr, *nin = nullptr,
            *rstart = nullptr, *rlist = nullptr, *pzone = nullptr, *zoneof = nullptr;
  size_t off = 0;
  for (const auto& b : ckpt_blocks(c)) {
    const int* q = reinterpret_cast<const int*>(data + off);
    const std::string n = b.name;
    if (n == "tile_count") tile_count = q;
    else if (n == "tile_list") tile_list = q;
    else if (n == "znd") znd = q;
    else if (n == "zoneMembers") members = q;
    else if (n == "numParInZone") nin = q;
    else if (n == "revStart") rstart = q;
    else if (n == "revList") rlist = q;
    else if (n == "parsZone") pzone = q;
    else if (n == "zoneOf") zoneof = q;
    off += b.bytes;
  }
  for (long long T = 0; T < c->ntiles; T++) {
    if (tile_count[T] < 0) return "tile count";
    const long long n = std::min<long long>(tile_count[T], cap);
    for (long long j = 0; j < n; j++)
      if (tile_list[T * cap + j] < 0 || tile_list[T * cap + j] >= M) return "tile list entry";
  }
  for (long long z = 0; z < Z; z++) {
    if (znd[28 * z] < 0 || znd[28 * z] > 27) return "zone neighbour count";
    for (long long t = 1; t <= znd[28 * z]; t++)
      if (znd[28 * z + t] < 0 || znd[28 * z + t] >= Z) return "zone neighbour";
    if (nin[z] < 0 || nin[z] > np) return "zone member count";
    for (long long j = 0; j < nin[z]; j++)
      if (members[z * np + j] < 0 || members[z * np + j] >= np) return "zone member";
  }
  for (long long p = 0; p < np; p++) {
    if (pzone[p] < 0 || pzone[p] >= Z) return "sphere zone";
    if (zoneof[p] < 0 || zoneof[p] >= Z) return "sphere zone";
  }
  if (rstart[0] != 0 || rstart[Z] > 27 * Z) return "reverse zone table";
  for (long long z = 0; z < Z; z++)
    if (rstart[z + 1] < rstart[z]) return "reverse zone table";
  for (long long r = 0; r < rstart[Z]; r++)
    if (rlist[r] < 0 || rlist[r] >= Z) return "reverse zone entry";
  return nullptr;
}
}  // namespace

extern "C" int d3q19_checkpoint_bytes(d3q19_ctx* c, size_t* bytes) {
  if (!c || !bytes) return D3Q19_EINVAL;
  size_t n = sizeof(CkptHeader);
  for (const auto& b : ckpt_blocks(c)) n += b.bytes;
  *bytes = n;
  return 0;
}

extern "C" int d3q19_checkpoint(d3q19_ctx* c, void* buf, size_t bytes) {
  TRACE("d3q19_checkpoint");
  if (!c || !buf) return D3Q19_EINVAL;
  if (c->f_state == 0) return fail(c, D3Q19_ESTATE, "lattice not written");
  if (c->kstage != 0) return fail(c, D3Q19_ESTATE, "step %d was left between passes", c->kt);
  size_t need = 0;
  d3q19_checkpoint_bytes(c, &need);
  if (bytes < need) return fail(c, D3Q19_EINVAL, "checkpoint needs %zu bytes", need);
  if (int rc = d3q19_synchronize(c)) return rc;  // joins the side stream, reports device errors
  CkptHeader h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, "D3Q19CK", 8);
  h.version = 2;
  h.storage = c->opt.storage;
  h.p64 = c->kin64[0] != nullptr;
  h.arithmetic = c->opt.arithmetic;
  h.NC = c->g.NC;
  h.ntiles = c->ntiles;
  h.np = c->ppar.np;
  h.nfa = c->ppar.nfa;
  h.P = c->ppar.P;
  h.cap = c->tile_cap;
  h.nzones = c->nzones;
  h.f_state = c->f_state;
  h.last_t = c->last_t;
  h.sticky = (int)c->sticky;
  h.inplace = c->opt.inplace;
  h.phase = c->cur;
  unsigned long long cl = 0;
  char* p = static_cast<char*>(buf) + sizeof(h);
  CUDA_TRY(c, cudaMemcpyAsync(&cl, c->clamps, sizeof(cl), cudaMemcpyDeviceToHost, c->stream));
  for (const auto& b : ckpt_blocks(c)) {
    CUDA_TRY(c, cudaMemcpyAsync(p, b.ptr, b.bytes, cudaMemcpyDeviceToHost, c->stream));
    p += b.bytes;
  }
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  h.clamps = (long long)cl;
  memcpy(buf, &h, sizeof(h));
  return 0;
}

extern "C" int d3q19_restore(d3q19_ctx* c, const void* buf, size_t bytes) {
  TRACE("d3q19_restore");
  if (!c || !buf || bytes < sizeof(CkptHeader)) return D3Q19_EINVAL;
  CkptHeader h;
  memcpy(&h, buf, sizeof(h));
  if (memcmp(h.magic, "D3Q19CK", 8) != 0 || h.version != 2) return fail(c, D3Q19_EINVAL, "not a checkpoint");
  if (h.storage != c->opt.storage || h.p64 != (c->kin64[0] != nullptr) || h.arithmetic != c->opt.arithmetic ||
      h.NC != c->g.NC || h.ntiles != c->ntiles || h.np != c->ppar.np || h.nfa != c->ppar.nfa || h.P != c->ppar.P ||
      h.cap != c->tile_cap || h.nzones != c->nzones || h.inplace != c->opt.inplace)
    return fail(c, D3Q19_EINVAL, "checkpoint of a context with other parameters");
  if ((c->opt.inplace && h.phase != 0 && h.phase != 1) || (h.f_state != 1 && h.f_state != 2) || h.last_t < 0 ||
      (h.f_state == 1 && c->opt.inplace && h.phase != 0))
    return fail(c, D3Q19_EINVAL, "checkpoint damaged: header state out of range");
  size_t need = 0;
  d3q19_checkpoint_bytes(c, &need);
  if (bytes < need) return fail(c, D3Q19_EINVAL, "checkpoint truncated (%zu of %zu bytes)", bytes, need);
  if (const char* bad = ckpt_tables_invalid(c, static_cast<const char*>(buf) + sizeof(h)))
    return fail(c, D3Q19_EINVAL, "checkpoint damaged: %s out of range", bad);
  cudaSetDevice(c->dev);
  if (int rc = join_side(c)) return rc;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const char* p = static_cast<const char*>(buf) + sizeof(h);
  for (const auto& b : ckpt_blocks(c)) {
    CUDA_TRY(c, cudaMemcpyAsync(b.ptr, p, b.bytes, cudaMemcpyHostToDevice, c->stream));
    p += b.bytes;
  }
  const unsigned long long cl = (unsigned long long)h.clamps;
  const unsigned e = (unsigned)h.sticky;
  CUDA_TRY(c, cudaMemcpyAsync(c->clamps, &cl, sizeof(cl), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->err, &e, sizeof(e), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));  // the host values above go out of scope
  c->sticky = e;
  if (c->opt.inplace) c->cur = h.phase;  // the buffer's layout
  c->f_state = h.f_state;
  c->last_t = h.last_t;
  c->have_particles = c->have_zones = true;
  // The TMA kernel's pulls read periodic neighbours' values from the
  // buffer-layer copies the step before it wrote; a restored buffer gets them
  // from its periodic images.
  if (c->use_tma && c->f_state == 2 && (!c->opt.inplace || c->cur == 1)) {
    FluidArgs fa = fluid_args(c, c->last_t, c->cur);
    CUDA_TRY(c, launch_fill_ghosts(fa, c->opt.storage, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  return 0;
}

/* ---------------------------------------------------------------------------
 * Device memory of a context, and the lattice pool.
 * ------------------------------------------------------------------------- */
static size_t round_alloc(size_t b) { return (b + 511) / 512 * 512; }

extern "C" int d3q19_context_bytes(const int_param_struct* ip, const d3q19_options* opt, size_t* out) {
  if (!ip || !out) return D3Q19_EINVAL;
  d3q19_options o;
  memset(&o, 0, sizeof(o));
  if (opt) o = *opt;
  if (o.storage < 0 || o.storage > 2 || o.arithmetic < 0 || o.arithmetic > 2) return D3Q19_EINVAL;
  if (o.arithmetic == 2) {
    o.storage = STORE_F64;
    o.particle_precision = 1;
  }
  const long long NC = (long long)ip->LatticeSize[0] * ip->LatticeSize[1] * ip->LatticeSize[2];
  const long long ntiles = (long long)((ip->LatticeSize[0] + TILE_X - 1) / TILE_X) *
                           ((ip->LatticeSize[1] + TILE_Y - 1) / TILE_Y) * ((ip->LatticeSize[2] + TILE_Z - 1) / TILE_Z);
  size_t b = (o.inplace ? 1 : 2) * round_alloc((size_t)storage_bytes(o.storage) * 19 * NC) + round_alloc(12 * (size_t)NC) +
             round_alloc(4 * (size_t)NC) + 3 * 512 + round_alloc(40 * (size_t)ip->LatticeSize[2]) +
             (o.arithmetic == 2 ? round_alloc(8 * (size_t)NC) : 0);
  const long long np = ip->NumParticles;
  if (np > 0) {
    const long long P = ip->PointsPerParticle, nfa = ip->WorkGroupsPerParticle, M = np * P;
    const long long Z = (long long)ip->NumZones[0] * ip->NumZones[1] * ip->NumZones[2];
    const long long cap = o.ibm_tile_capacity > 0 ? o.ibm_tile_capacity : std::min<long long>(M, 2048);
    b += 2 * (round_alloc(64 * np) + round_alloc(32 * np * nfa) + round_alloc(32 * np));
    if (o.particle_precision == 1) b += 2 * (round_alloc(128 * np) + round_alloc(64 * np * nfa));
    b += round_alloc(16 * P) + round_alloc(32 * M) + round_alloc(4 * ntiles) + 512 + round_alloc(4 * ntiles * cap);
    b += round_alloc(4 * 28 * Z) + round_alloc(4 * np) + round_alloc(4 * Z * np) + round_alloc(4 * Z) +
         round_alloc(4 * (Z + 1)) + round_alloc(4 * 27 * Z) + round_alloc(4 * np);
  }
  *out = b;
  return 0;
}

struct d3q19_pool {
  int dev = 0;
  int storage = 0;
  int rebuild = 10;  // zone rebuild period shared by every member
  int period = 10;   // lcm(2, rebuild): admissions and advances keep this phase
  size_t budget = 0, used = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_done = nullptr;
  // Device memory of the members: allocated on a member's stream at
  // admission, freed on the pool's stream at release (after the chunks in
  // flight), kept reserved between members.
  cudaMemPool_t mempool = nullptr;
  std::vector<d3q19_ctx*> slot;  // nullptr: free
  std::vector<size_t> slot_bytes;
  std::vector<long long> slot_steps;
  int max_slots = 0;
  // Device copies of the per-slot kernel arguments (two buffer parities) and
  // the packed work lists.
  FluidArgs* d_fargs = nullptr;
  ParticleArgs* d_pargs = nullptr;
  ZoneArgs* d_zargs = nullptr;
  int2* d_work = nullptr;  // three regions of work_cap items: fluid tiles, particle groups, contact spheres
  int* d_zslots = nullptr;
  int* d_counts = nullptr;  // [fluid, particle, contact, zone] item counts
  size_t work_cap = 0;
  long long nf = 0, ngr = 0, nsph = 0;  // item counts of the current lists
  int part_threads = 128;
  bool dirty = true;
  int fgrid = 1;  // CTAs of the fluid pass: one per tile of the work list, rounded up (pool_upload)
  int pblocks = 0, cblocks = 0;
  int sm_count = 0;
  // Layout of the members (d3q19_options.inplace) while the pool has any; -1
  // when empty.  In place, every member sits at buffer parity 0 between
  // chunks, so step j of a chunk is an even step for all when j is even.
  int inplace = -1;
  double* d_stats = nullptr;  // per-member plane sums and error words (d3q19_pool_mean_stress)
  size_t stats_cap = 0;
  std::map<std::tuple<int, int, int, int, int>, cudaGraphExec_t> graphs;  // (steps, fgrid, pblocks, cblocks, inplace)
  long long steps = 0;
  // Grid autotuner (d3q19_pool_autotune): on or off, and the advance being
  // timed (its table key, candidate and fluid tile steps), if any.
  struct TuneTrial {
    std::string key;  // table entry
    int cand;         // candidate timed
    double units;     // fluid tile steps of the segment
    cudaEvent_t e0, e1;
  };
  bool tune = false;
  std::vector<TuneTrial> tune_trials;                           // timed segments in flight
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> tune_events;  // free event pairs
  char dev_name[256] = {0};
  // Every d3q19_pool_* call holds it: the pool may be driven from several
  // host threads (its members are not stepped outside these calls).
  std::mutex mu;
  char msg[512] = {0};
};

#define POOL_LOCK(p) std::lock_guard<std::mutex> pool_lock_((p)->mu)

static int pfail(d3q19_pool* p, int code, const char* fmt, ...) {
  char* buf = p ? p->msg : g_create_error;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, 512, fmt, ap);
  va_end(ap);
  return code;
}

#define POOL_TRY(p, call)                                                                        \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return pfail((p), D3Q19_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

static void pool_drop_graphs(d3q19_pool* p) {
  for (auto& kv : p->graphs) cudaGraphExecDestroy(kv.second);
  p->graphs.clear();
}

extern "C" int d3q19_pool_create(int device, int storage, int rebuild_freq, int max_slots, size_t hbm_budget,
                                 d3q19_pool** out) {
  if (!out || storage < 0 || storage > 2 || max_slots <= 0 || rebuild_freq <= 0)
    return pfail(nullptr, D3Q19_EINVAL, "pool: invalid arguments");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return pfail(nullptr, D3Q19_ENODEV, "CUDA device %d not available", device);
  cudaDeviceProp pr;
  cudaGetDeviceProperties(&pr, device);
  if (pr.major != 10) return pfail(nullptr, D3Q19_ENODEV, "device %s is sm_%d%d; this build is sm_100a", pr.name,
                                   pr.major, pr.minor);
  cudaSetDevice(device);
  d3q19_pool* p = new d3q19_pool();
  p->dev = device;
  p->storage = storage;
  p->rebuild = rebuild_freq;
  p->period = 2 / gcd_i(2, rebuild_freq) * rebuild_freq;
  p->max_slots = max_slots;
  p->budget = hbm_budget;
  p->slot.assign(max_slots, nullptr);
  p->slot_bytes.assign(max_slots, 0);
  p->slot_steps.assign(max_slots, 0);
  // Persistent grids: blocks per SM the kernels' register and shared memory
  // bounds allow (the autotuner may lower them).
  p->sm_count = pr.multiProcessorCount;
  snprintf(p->dev_name, sizeof(p->dev_name), "%s", pr.name);
  for (char* q = p->dev_name; *q; q++)  // the name is a field of the tuning table's lines
    if (*q == '\t' || *q == '\n' || *q == '|') *q = ' ';
  p->pblocks = pr.multiProcessorCount * 4;
  p->cblocks = pr.multiProcessorCount * 4;
  cudaMemPoolProps mp;
  memset(&mp, 0, sizeof(mp));
  mp.allocType = cudaMemAllocationTypePinned;
  mp.location.type = cudaMemLocationTypeDevice;
  mp.location.id = device;
  const unsigned long long keep = ~0ull;
  if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->ev_done, cudaEventDisableTiming) != cudaSuccess ||
      cudaMemPoolCreate(&p->mempool, &mp) != cudaSuccess ||
      cudaMemPoolSetAttribute(p->mempool, cudaMemPoolAttrReleaseThreshold, (void*)&keep) != cudaSuccess ||
      cudaMalloc(&p->d_fargs, sizeof(FluidArgs) * 2 * max_slots) != cudaSuccess ||
      cudaMalloc(&p->d_pargs, sizeof(ParticleArgs) * 2 * max_slots) != cudaSuccess ||
      cudaMalloc(&p->d_zargs, sizeof(ZoneArgs) * 2 * max_slots) != cudaSuccess ||
      cudaMalloc(&p->d_zslots, sizeof(int) * max_slots) != cudaSuccess ||
      cudaMalloc(&p->d_counts, sizeof(int) * 4) != cudaSuccess) {
    d3q19_pool_destroy(p);
    return pfail(nullptr, D3Q19_ENOMEM, "pool: device set-up failed");
  }
  p->used = sizeof(FluidArgs) * 2 * max_slots + sizeof(ParticleArgs) * 2 * max_slots +
            sizeof(ZoneArgs) * 2 * max_slots;
  *out = p;
  return 0;
}

// Checks a member's parameters against the pool and finds it a slot and
// budget: the options it is created with, the slot and its device bytes.
static int pool_place(d3q19_pool* p, const int_param_struct* ip, const d3q19_options* opt, d3q19_options* out,
                      int* slot, size_t* bytes) {
  d3q19_options& o = *out;
  memset(&o, 0, sizeof(o));
  if (opt) o = *opt;
  o.device = p->dev;
  if (o.storage != p->storage) return pfail(p, D3Q19_EINVAL, "storage %d differs from the pool's %d", o.storage,
                                            p->storage);
  if (o.arithmetic != 0 || o.collision != 0 || o.particle_precision != 0)
    return pfail(p, D3Q19_EINVAL, "the pool runs the fast FP32 arithmetic with the reference's MRT only");
  if (p->inplace >= 0 && o.inplace != p->inplace)
    return pfail(p, D3Q19_EINVAL, "inplace %d differs from the pool members' %d", o.inplace, p->inplace);
  if (ip->BoundaryConds[0] != 0 || ip->BoundaryConds[1] != 0 || ip->BoundaryConds[2] != 1 ||
      o.tangential_vel_bc[0] || o.tangential_vel_bc[1] || o.tangential_vel_bc[2])
    return pfail(p, D3Q19_EINVAL, "the pool runs shear cells: periodic x and y, velocity walls on z");
  if (o.rebuild_freq <= 0) o.rebuild_freq = 10;
  // Members are advanced by the batched per-tile kernels, which fold the
  // periodic wrap into their gathers; their solo warm-up steps use the same
  // kernel family.
  o.fluid_kernel = 0;
  if (ip->NumParticles > 0 && o.rebuild_freq != p->rebuild)
    return pfail(p, D3Q19_EINVAL, "rebuild_freq %d differs from the pool's %d", o.rebuild_freq, p->rebuild);
  if (ip->NumParticles > 0 && ip->PointsPerWorkGroup > 256)
    return pfail(p, D3Q19_EINVAL, "PointsPerWorkGroup above 256");
  *slot = -1;
  for (int k = 0; k < p->max_slots && *slot < 0; k++)
    if (!p->slot[k]) *slot = k;
  if (*slot < 0) return pfail(p, D3Q19_EBUSY, "all %d slots are taken", p->max_slots);
  if (int rc = d3q19_context_bytes(ip, &o, bytes)) return rc;
  if (p->used + *bytes > p->budget)
    return pfail(p, D3Q19_EBUSY, "%zu bytes would exceed the HBM budget (%zu of %zu used)", *bytes, p->used,
                 p->budget);
  return 0;
}

extern "C" int d3q19_pool_admit(d3q19_pool* p, const int_param_struct* ip, const flp_param_struct* fp,
                                const d3q19_options* opt, const float* f, const float* u, const float* tau,
                                const float* parKin, const float* parForce, const float* parFluidForce,
                                const float* spherePoints, const int* zoneNeighDat, const int* parsZone,
                                const int* zoneMembers, const int* numParInZone, int* slot_out) {
  TRACE("d3q19_pool_admit");
  if (!p || !ip || !fp || !f || !u || !slot_out) return D3Q19_EINVAL;
  POOL_LOCK(p);
  d3q19_options o;
  int s = -1;
  size_t bytes = 0;
  if (int rc = pool_place(p, ip, opt, &o, &s, &bytes)) return rc;
  d3q19_ctx* c = nullptr;
  int rc = create_ctx(ip, fp, &o, p->mempool, &c);
  if (rc) return pfail(p, rc, "%s", d3q19_last_error(nullptr));
  rc = d3q19_write_lattice(c, f, u, tau);
  if (!rc && ip->NumParticles > 0) {
    rc = d3q19_write_particles(c, parKin, parForce, parFluidForce, spherePoints);
    if (!rc) rc = d3q19_write_zones(c, zoneNeighDat, parsZone, zoneMembers, numParInZone, nullptr, nullptr);
  }
  // The first steps run alone, so that the member joins in the pool's phase:
  // its next step t satisfies t = 1 (mod period) like every other member's.
  if (!rc) rc = d3q19_run(c, 1, p->period);
  if (!rc) rc = d3q19_synchronize(c);
  if (rc) {
    pfail(p, rc, "admission: %s", d3q19_last_error(c));
    d3q19_destroy(c);
    return rc;
  }
  if (c->opt.inplace && c->cur != 0) {  // cannot happen: the warm-up is an even number of steps
    d3q19_destroy(c);
    return pfail(p, D3Q19_ESTATE, "in-place member out of phase");
  }
  p->inplace = c->opt.inplace;
  p->slot[s] = c;
  p->slot_bytes[s] = bytes;
  p->slot_steps[s] = p->period;
  p->used += bytes;
  p->dirty = true;
  *slot_out = s;
  return 0;
}

// Work lists and arguments of the members, uploaded on the pool's stream.
static int pool_upload(d3q19_pool* p) {
  std::vector<FluidArgs> fa(2 * (size_t)p->max_slots);
  std::vector<ParticleArgs> pa(2 * (size_t)p->max_slots);
  std::vector<ZoneArgs> za(2 * (size_t)p->max_slots);
  std::vector<int2> fw, pw, cw;
  std::vector<int> zs;
  int threads = 128;
  for (int s = 0; s < p->max_slots; s++) {
    d3q19_ctx* c = p->slot[s];
    if (!c) continue;
    // Step j of a chunk (j = 0, 1, ...) runs with distributions parity
    // cur + j and particle parity pcur + j; its step number has parity of
    // j + 1 (only the parity enters the kernels).
    for (int j = 0; j < 2; j++) {
      fa[2 * s + j] = fluid_args(c, j + 1, (c->cur + j) & 1);
      if (c->ppar.np > 0) {
        pa[2 * s + j] = particle_args(c, j + 1, (c->pcur + j) & 1);
        za[2 * s + j] = zone_args(c, (c->pcur + j + 1) & 1);
      }
    }
    for (long long T = 0; T < c->ntiles; T++) fw.push_back(make_int2(s, (int)T));
    if (c->ppar.np > 0) {
      for (int gr = 0; gr < c->ppar.np * c->ppar.nfa; gr++) pw.push_back(make_int2(s, gr));
      for (int q = 0; q < c->ppar.np; q++) cw.push_back(make_int2(s, q));
      zs.push_back(s);
      threads = std::max(threads, c->ppar.L);
    }
  }
  // Each list has a fixed region, so captured launches stay valid while
  // members come and go; only a larger allocation invalidates them.
  const size_t need = std::max(fw.size(), std::max(pw.size(), cw.size()));
  if (need > p->work_cap) {
    POOL_TRY(p, cudaStreamSynchronize(p->stream));
    const size_t cap = std::max<size_t>(need, 2 * p->work_cap) + 4096;
    if (p->d_work) cudaFree(p->d_work);
    p->d_work = nullptr;
    p->work_cap = 0;
    POOL_TRY(p, cudaMalloc(&p->d_work, sizeof(int2) * 3 * cap));
    p->work_cap = cap;
    pool_drop_graphs(p);  // the captured launches name the old list
  }
  p->nf = (long long)fw.size();
  p->ngr = (long long)pw.size();
  // Fluid grid: the tile count rounded up to m * 2^k with m in [8, 15] (at
  // most 1/8 of the CTAs return at once), so that a captured chunk serves
  // every membership of the same rounded size.
  {
    long long g = std::max<long long>(p->nf, 1), unit = 1;
    while (g > 15 * unit) unit *= 2;
    p->fgrid = (int)((g + unit - 1) / unit * unit);
  }
  p->nsph = (long long)cw.size();
  if (threads != p->part_threads) {
    p->part_threads = threads;
    pool_drop_graphs(p);
  }
  const int counts[4] = {(int)fw.size(), (int)pw.size(), (int)cw.size(), (int)zs.size()};
  POOL_TRY(p, cudaMemcpyAsync(p->d_fargs, fa.data(), sizeof(FluidArgs) * fa.size(), cudaMemcpyHostToDevice,
                              p->stream));
  POOL_TRY(p, cudaMemcpyAsync(p->d_pargs, pa.data(), sizeof(ParticleArgs) * pa.size(), cudaMemcpyHostToDevice,
                              p->stream));
  POOL_TRY(p, cudaMemcpyAsync(p->d_zargs, za.data(), sizeof(ZoneArgs) * za.size(), cudaMemcpyHostToDevice,
                              p->stream));
  const std::vector<int2>* lists[3] = {&fw, &pw, &cw};
  for (int k = 0; k < 3; k++)
    if (!lists[k]->empty())
      POOL_TRY(p, cudaMemcpyAsync(p->d_work + k * p->work_cap, lists[k]->data(), sizeof(int2) * lists[k]->size(),
                                  cudaMemcpyHostToDevice, p->stream));
  if (!zs.empty())
    POOL_TRY(p, cudaMemcpyAsync(p->d_zslots, zs.data(), sizeof(int) * zs.size(), cudaMemcpyHostToDevice, p->stream));
  POOL_TRY(p, cudaMemcpyAsync(p->d_counts, counts, sizeof(counts), cudaMemcpyHostToDevice, p->stream));
  // The host vectors go out of scope: wait for the copies.
  POOL_TRY(p, cudaStreamSynchronize(p->stream));
  p->dirty = false;
  return 0;
}

static int pool_enqueue(d3q19_pool* p, int nsteps) {
  const int2* fw = p->d_work;
  const int2* pw = p->d_work + p->work_cap;
  const int2* cw = p->d_work + 2 * p->work_cap;
  for (int j = 0; j < nsteps; j++) {
    const int par = j & 1;
    // In place, the FP32 kernels run 4 blocks/SM: a larger persistent grid
    // would only add a second wave.
    const int aa = p->inplace == 1 ? (par == 0 ? 1 : 2) : 0;
    POOL_TRY(p, launch_fluid_batch(p->d_fargs, fw, p->d_counts + 0, par, p->storage, aa, p->fgrid, p->stream));
    POOL_TRY(p, launch_particle_batch(p->d_pargs, pw, p->d_counts + 1, par, p->part_threads, p->pblocks, p->stream));
    POOL_TRY(p, launch_contact_batch(p->d_pargs, cw, p->d_counts + 2, par, p->cblocks, p->stream));
    if ((j + 1) % p->rebuild == 0)
      POOL_TRY(p, launch_zone_batch(p->d_zargs, p->d_zslots, p->d_counts + 3, par, p->max_slots, p->stream));
  }
  return 0;
}

// ---- Persistent-grid autotuner ---------------------------------------------
// A process-wide table, keyed by the device (name and SM count), the pool's
// storage and layout, and the size class of its work (the bit length of the
// fluid tile count).  An entry holds the candidate grids -- fluid CTAs per SM
// by particle/contact CTAs per SM -- with the time each measured, in ns per
// fluid tile step, and the fastest once every candidate has run.  The batched
// kernels take their items from work lists, so results do not depend on the
// grid: a timed advance is an ordinary advance of the members.
struct TuneEntry {
  std::vector<std::pair<int, int>> cand;  // (fluid, particle/contact) CTAs per SM
  std::vector<double> cost;               // ns per fluid tile step; < 0 until timed
  int best = -1;                          // index of the choice once settled
};
static std::mutex g_tune_mu;
static std::map<std::string, TuneEntry> g_tune;
// Advances shorter than this are not timed (launch overhead would dominate).
constexpr int TUNE_MIN_STEPS = 100;

static int tune_class(long long nf) {
  int c = 0;
  while (nf > 0) {
    c++;
    nf >>= 1;
  }
  return c;
}

static std::string tune_key_of(const char* dev_name, int sms, int storage, int inplace, int cls) {
  char buf[400];
  snprintf(buf, sizeof(buf), "%s\t%d\t%d\t%d\t%d", dev_name, sms, storage, inplace, cls);
  return buf;
}

// The candidates of a pool: particle/contact 1, 2 or 4 CTAs per SM.  The
// fluid pass runs one CTA per tile (fluid entry 0).
static TuneEntry tune_candidates(const d3q19_pool*) {
  TuneEntry e;
  for (int q : {1, 2, 4}) e.cand.push_back({0, q});
  e.cost.assign(e.cand.size(), -1.0);
  return e;
}

// Records the times of the timed segments in flight (waits for them) and
// settles the entries whose candidates have all been timed.
static int tune_collect(d3q19_pool* p) {
  if (p->tune_trials.empty()) return 0;
  std::vector<std::pair<std::string, double>> got;
  std::vector<int> cands;
  cudaError_t err = cudaSuccess;
  for (auto& t : p->tune_trials) {
    float ms = 0.f;
    cudaError_t e = cudaEventSynchronize(t.e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t.e0, t.e1);
    if (e == cudaSuccess) {
      got.emplace_back(t.key, ms * 1e6 / t.units);
      cands.push_back(t.cand);
    } else if (err == cudaSuccess) {
      err = e;
    }
    p->tune_events.emplace_back(t.e0, t.e1);
  }
  p->tune_trials.clear();
  if (err != cudaSuccess) return pfail(p, D3Q19_ECUDA, "tuning events: %s", cudaGetErrorString(err));
  const std::string cur =
      tune_key_of(p->dev_name, p->sm_count, p->storage, p->inplace, tune_class(p->nf));
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (size_t i = 0; i < got.size(); i++) {
    auto it = g_tune.find(got[i].first);
    if (it == g_tune.end() || it->second.best >= 0 || cands[i] >= (int)it->second.cand.size()) continue;
    TuneEntry& e = it->second;
    e.cost[cands[i]] = got[i].second;
    int best = 0;
    bool all = true;
    for (size_t j = 0; j < e.cost.size(); j++) {
      all = all && e.cost[j] >= 0;
      if (e.cost[j] >= 0 && (e.cost[best] < 0 || e.cost[j] < e.cost[best])) best = (int)j;
    }
    if (!all) continue;
    e.best = best;
    if (it->first == cur)  // the choice applies from now on
      p->pblocks = p->cblocks = e.cand[best].second * p->sm_count;
  }
  return 0;
}

// Segment length of an advance of nsteps: while the pool's class has
// candidates left, an advance of at least two segments is run as segments of
// TUNE_MIN_STEPS (rounded up to the period), each timing one candidate.
static int tune_segment(const d3q19_pool* p, int nsteps) {
  if (!p->tune || p->nf <= 0 || p->inplace < 0) return nsteps;
  const int seg = (TUNE_MIN_STEPS + p->period - 1) / p->period * p->period;
  if (nsteps < 2 * seg) return nsteps;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(tune_key_of(p->dev_name, p->sm_count, p->storage, p->inplace, tune_class(p->nf)));
  return it != g_tune.end() && it->second.best >= 0 ? nsteps : seg;
}

// Before a segment of nsteps: sets the grid of the pool's class -- its
// choice, else the next candidate not yet timed nor in flight, else the
// fastest timed so far.  Returns the candidate to time, or -1.
static int tune_choose(d3q19_pool* p, int nsteps, std::string* key_out) {
  if (!p->tune || p->nf <= 0 || p->inplace < 0) return -1;
  const std::string key = tune_key_of(p->dev_name, p->sm_count, p->storage, p->inplace, tune_class(p->nf));
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(key);
  if (it == g_tune.end()) it = g_tune.emplace(key, tune_candidates(p)).first;
  const TuneEntry& e = it->second;
  int c = e.best, timed = -1;
  if (c < 0 && nsteps >= TUNE_MIN_STEPS) {
    for (int i = 0; i < (int)e.cost.size() && timed < 0; i++) {
      if (e.cost[i] >= 0) continue;
      bool busy = false;
      for (const auto& t : p->tune_trials) busy = busy || (t.cand == i && t.key == key);
      if (!busy) timed = i;
    }
    c = timed;
  }
  if (c < 0)
    for (int i = 0; i < (int)e.cost.size(); i++)
      if (e.cost[i] >= 0 && (c < 0 || e.cost[i] < e.cost[c])) c = i;
  if (c < 0) return -1;
  p->pblocks = p->cblocks = e.cand[c].second * p->sm_count;
  if (timed >= 0) *key_out = key;
  return timed;
}

// The graph of a chunk of nsteps at the pool's current grid (captured on
// first use).
static int pool_graph(d3q19_pool* p, int nsteps, cudaGraphExec_t* out) {
  auto key = std::make_tuple(nsteps, p->fgrid, p->pblocks, p->cblocks, p->inplace);
  auto it = p->graphs.find(key);
  if (it == p->graphs.end()) {
    cudaGraph_t graph;
    POOL_TRY(p, cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    int rc = pool_enqueue(p, nsteps);
    cudaError_t e = cudaStreamEndCapture(p->stream, &graph);
    if (rc) return rc;
    if (e != cudaSuccess) return pfail(p, D3Q19_ECUDA, "pool capture: %s", cudaGetErrorString(e));
    cudaGraphExec_t exec;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return pfail(p, D3Q19_ECUDA, "pool graph: %s", cudaGetErrorString(e));
    it = p->graphs.emplace(key, exec).first;
    POOL_TRY(p, cudaGraphUpload(exec, p->stream));  // not inside a timed segment
  }
  *out = it->second;
  return 0;
}

extern "C" int d3q19_pool_advance(d3q19_pool* p, int nsteps) {
  TRACE("d3q19_pool_advance");
  if (!p) return D3Q19_EINVAL;
  POOL_LOCK(p);
  if (nsteps <= 0 || nsteps % p->period != 0)
    return pfail(p, D3Q19_EINVAL, "steps must be a positive multiple of %d", p->period);
  cudaSetDevice(p->dev);
  for (int s = 0; s < p->max_slots; s++)  // members' own streams (admission, read-backs) first
    if (p->slot[s]) {
      if (int rc = join_side(p->slot[s])) return pfail(p, rc, "%s", d3q19_last_error(p->slot[s]));
      POOL_TRY(p, cudaEventRecord(p->slot[s]->ev_fork, p->slot[s]->stream));
      POOL_TRY(p, cudaStreamWaitEvent(p->stream, p->slot[s]->ev_fork, 0));
    }
  if (int rc = tune_collect(p)) return rc;
  if (p->dirty)
    if (int rc = pool_upload(p)) return rc;
  const int seg = tune_segment(p, nsteps);
  for (int done = 0; done < nsteps;) {
    std::string tkey;
    int len = std::min(seg, nsteps - done);
    const int cand = tune_choose(p, len, &tkey);
    if (cand < 0) len = nsteps - done;  // nothing to time: the rest in one graph
    cudaGraphExec_t exec;
    if (int rc = pool_graph(p, len, &exec)) return rc;
    if (cand >= 0) {
      if (p->tune_events.empty()) {
        cudaEvent_t e0, e1;
        POOL_TRY(p, cudaEventCreate(&e0));
        if (cudaEventCreate(&e1) != cudaSuccess) {
          cudaEventDestroy(e0);
          return pfail(p, D3Q19_ECUDA, "tuning events");
        }
        p->tune_events.emplace_back(e0, e1);
      }
      const auto ev = p->tune_events.back();
      p->tune_events.pop_back();
      p->tune_trials.push_back({tkey, cand, (double)len * (double)p->nf, ev.first, ev.second});
      POOL_TRY(p, cudaEventRecord(ev.first, p->stream));
      POOL_TRY(p, cudaGraphLaunch(exec, p->stream));
      POOL_TRY(p, cudaEventRecord(ev.second, p->stream));
    } else {
      POOL_TRY(p, cudaGraphLaunch(exec, p->stream));
    }
    done += len;
  }
  POOL_TRY(p, cudaEventRecord(p->ev_done, p->stream));
  for (int s = 0; s < p->max_slots; s++) {
    d3q19_ctx* c = p->slot[s];
    if (!c) continue;
    // nsteps is even: the buffer parities are where they were.
    c->last_t += nsteps;
    p->slot_steps[s] += nsteps;
    POOL_TRY(p, cudaStreamWaitEvent(c->stream, p->ev_done, 0));  // read-backs after the pool's work
  }
  p->steps += nsteps;
  return 0;
}

extern "C" int d3q19_pool_mean_stress(d3q19_pool* p, double* stress_xz, double* shear_rate, double* eff_viscosity,
                                      int* status) {
  TRACE("d3q19_pool_mean_stress");
  if (!p || !stress_xz || !status) return D3Q19_EINVAL;
  POOL_LOCK(p);
  cudaSetDevice(p->dev);
  // Layout: per member, 5*Nz plane sums then its error word.
  std::vector<size_t> off(p->max_slots, 0);
  size_t need = 0;
  for (int s = 0; s < p->max_slots; s++)
    if (p->slot[s]) {
      off[s] = need;
      need += 5 * (size_t)p->slot[s]->g.Nz + 1;
    }
  if (need > p->stats_cap) {
    POOL_TRY(p, cudaStreamSynchronize(p->stream));
    if (p->d_stats) cudaFree(p->d_stats);
    p->d_stats = nullptr;
    p->stats_cap = 0;
    POOL_TRY(p, cudaMalloc(&p->d_stats, sizeof(double) * (need + 1024)));
    p->stats_cap = need + 1024;
  }
  for (int s = 0; s < p->max_slots; s++) {
    d3q19_ctx* c = p->slot[s];
    if (!c) continue;
    if (int rc = join_side(c)) return pfail(p, rc, "%s", d3q19_last_error(c));
    POOL_TRY(p, cudaEventRecord(c->ev_fork, c->stream));
    POOL_TRY(p, cudaStreamWaitEvent(p->stream, c->ev_fork, 0));
    POOL_TRY(p, launch_plane_stats(c->g, c->u, c->tau, c->fp.NewtonianTau, c->opt.variable_viscosity,
                                   p->d_stats + off[s], p->stream));
    POOL_TRY(p, launch_copy_err(c->err, p->d_stats + off[s] + 5 * (size_t)c->g.Nz, p->stream));
  }
  std::vector<double> h(std::max<size_t>(need, 1));
  POOL_TRY(p, cudaStreamSynchronize(p->stream));
  if (need) POOL_TRY(p, cudaMemcpy(h.data(), p->d_stats, sizeof(double) * need, cudaMemcpyDeviceToHost));
  for (int s = 0; s < p->max_slots; s++) {
    d3q19_ctx* c = p->slot[s];
    const double nan = std::numeric_limits<double>::quiet_NaN();
    if (!c) {
      stress_xz[s] = nan;
      if (shear_rate) shear_rate[s] = nan;
      if (eff_viscosity) eff_viscosity[s] = nan;
      status[s] = D3Q19_EINVAL;
      continue;
    }
    const int Nz = c->g.Nz;
    const unsigned e = (unsigned)h[off[s] + 5 * (size_t)Nz];
    c->sticky |= e;
    status[s] = (c->sticky & ERR_BOUNDS)          ? D3Q19_EBOUNDS
                : (c->sticky & ERR_TILE_OVERFLOW) ? D3Q19_EOVERFLOW
                : (c->sticky & (ERR_NONFINITE | ERR_FIXED_RANGE | ERR_ZONE_RANGE)) ? D3Q19_ENUMERIC
                                                                                     : 0;
    double gs = 0.0, ts = 0.0;
    for (int z = 1; z <= Nz - 2; z++) {
      gs += h[off[s] + 5 * (size_t)z + 3];
      ts += h[off[s] + 5 * (size_t)z + 4];
    }
    const double n = (double)(c->g.Nx - 2) * (c->g.Ny - 2) * (Nz - 2);
    stress_xz[s] = ts / n;
    if (shear_rate) shear_rate[s] = gs / n;
    if (eff_viscosity) eff_viscosity[s] = gs != 0.0 ? ts / gs : 0.0;
  }
  return 0;
}

extern "C" d3q19_ctx* d3q19_pool_context(d3q19_pool* p, int slot) {
  if (!p || slot < 0) return nullptr;
  POOL_LOCK(p);
  return slot < p->max_slots ? p->slot[slot] : nullptr;
}

extern "C" long long d3q19_pool_slot_steps(d3q19_pool* p, int slot) {
  if (!p || slot < 0) return -1;
  POOL_LOCK(p);
  if (slot >= p->max_slots || !p->slot[slot]) return -1;
  return p->slot_steps[slot];
}

// Release with the pool's lock held.
static int release_slot(d3q19_pool* p, int slot) {
  if (slot < 0 || slot >= p->max_slots || !p->slot[slot]) return D3Q19_EINVAL;
  cudaSetDevice(p->dev);
  // No wait for the chunks in flight: the member's memory is freed in the
  // pool stream's order, after them (its own streams are drained by destroy).
  d3q19_ctx* c = p->slot[slot];
  c->free_stream = p->stream;
  d3q19_destroy(c);
  p->slot[slot] = nullptr;
  p->used -= p->slot_bytes[slot];
  p->slot_bytes[slot] = 0;
  p->slot_steps[slot] = 0;
  p->dirty = true;
  bool empty = true;
  for (auto* m : p->slot) empty = empty && !m;
  if (empty) p->inplace = -1;
  return 0;
}

extern "C" int d3q19_pool_release(d3q19_pool* p, int slot) {
  TRACE("d3q19_pool_release");
  if (!p) return D3Q19_EINVAL;
  POOL_LOCK(p);
  return release_slot(p, slot);
}

extern "C" int d3q19_pool_evict(d3q19_pool* p, int slot, void* buf, size_t bytes) {
  TRACE("d3q19_pool_evict");
  if (!p) return D3Q19_EINVAL;
  POOL_LOCK(p);
  if (slot < 0 || slot >= p->max_slots || !p->slot[slot]) return D3Q19_EINVAL;
  cudaSetDevice(p->dev);
  POOL_TRY(p, cudaStreamSynchronize(p->stream));
  d3q19_ctx* c = p->slot[slot];
  if (int rc = d3q19_checkpoint(c, buf, bytes)) return pfail(p, rc, "%s", d3q19_last_error(c));
  return release_slot(p, slot);
}

extern "C" int d3q19_pool_readmit(d3q19_pool* p, const int_param_struct* ip, const flp_param_struct* fp,
                                  const d3q19_options* opt, const void* buf, size_t bytes, int* slot_out) {
  TRACE("d3q19_pool_readmit");
  if (!p || !ip || !fp || !buf || !slot_out) return D3Q19_EINVAL;
  POOL_LOCK(p);
  if (bytes < sizeof(CkptHeader)) return pfail(p, D3Q19_EINVAL, "not a checkpoint");
  CkptHeader h;
  memcpy(&h, buf, sizeof(h));
  // A member leaves and rejoins between chunks, in the pool's phase.
  if (h.f_state != 2 || h.last_t <= 0 || h.last_t % p->period != 0)
    return pfail(p, D3Q19_EINVAL, "checkpoint at step %d is not at a step multiple of the period %d", h.last_t,
                 p->period);
  d3q19_options o;
  int s = -1;
  size_t need = 0;
  if (int rc = pool_place(p, ip, opt, &o, &s, &need)) return rc;
  d3q19_ctx* c = nullptr;
  int rc = create_ctx(ip, fp, &o, p->mempool, &c);
  if (rc) return pfail(p, rc, "%s", d3q19_last_error(nullptr));
  if ((rc = d3q19_restore(c, buf, bytes))) {
    pfail(p, rc, "readmission: %s", d3q19_last_error(c));
    d3q19_destroy(c);
    return rc;
  }
  if (c->opt.inplace && c->cur != 0) {
    d3q19_destroy(c);
    return pfail(p, D3Q19_EINVAL, "in-place checkpoint at an odd phase");
  }
  p->inplace = c->opt.inplace;
  p->slot[s] = c;
  p->slot_bytes[s] = need;
  p->slot_steps[s] = h.last_t;
  p->used += need;
  p->dirty = true;
  *slot_out = s;
  return 0;
}

extern "C" int d3q19_pool_usage(d3q19_pool* p, size_t* used, size_t* budget, int* members) {
  if (!p) return D3Q19_EINVAL;
  POOL_LOCK(p);
  int n = 0;
  for (auto* c : p->slot) n += c != nullptr;
  if (used) *used = p->used;
  if (budget) *budget = p->budget;
  if (members) *members = n;
  return 0;
}

extern "C" int d3q19_pool_set_grid(d3q19_pool* p, int fluid_blocks, int particle_blocks, int contact_blocks) {
  if (!p || fluid_blocks < 0 || particle_blocks <= 0 || contact_blocks <= 0) return D3Q19_EINVAL;
  POOL_LOCK(p);
  p->pblocks = particle_blocks;
  p->cblocks = contact_blocks;
  p->tune = false;
  return 0;
}

extern "C" int d3q19_pool_autotune(d3q19_pool* p, int enable) {
  if (!p || (enable != 0 && enable != 1)) return D3Q19_EINVAL;
  POOL_LOCK(p);
  p->tune = enable != 0;
  return 0;
}

// The table entry of the pool's current work class (under g_tune_mu), or null.
static const TuneEntry* tune_entry_of(const d3q19_pool* p) {
  if (p->nf <= 0 || p->inplace < 0) return nullptr;
  auto it = g_tune.find(tune_key_of(p->dev_name, p->sm_count, p->storage, p->inplace, tune_class(p->nf)));
  return it == g_tune.end() ? nullptr : &it->second;
}

extern "C" int d3q19_pool_tune_state(d3q19_pool* p, int* fluid_per_sm, int* particle_per_sm, int* settled,
                                     int* tried, int* total) {
  if (!p) return D3Q19_EINVAL;
  POOL_LOCK(p);
  cudaSetDevice(p->dev);
  if (int rc = tune_collect(p)) return rc;
  if (fluid_per_sm) *fluid_per_sm = 0;  // one CTA per tile
  if (particle_per_sm) *particle_per_sm = p->pblocks / p->sm_count;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  const TuneEntry* e = tune_entry_of(p);
  int n = 0;
  if (e)
    for (double c : e->cost) n += c >= 0;
  if (settled) *settled = e && e->best >= 0;
  if (tried) *tried = n;
  if (total) *total = e ? (int)e->cand.size() : 0;
  return 0;
}

extern "C" int d3q19_pool_tune_trials(d3q19_pool* p, int* fluid_per_sm, int* particle_per_sm, double* ns_per_tile_step,
                                      int cap, int* n) {
  if (!p || !n || cap < 0) return D3Q19_EINVAL;
  POOL_LOCK(p);
  cudaSetDevice(p->dev);
  if (int rc = tune_collect(p)) return rc;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  const TuneEntry* e = tune_entry_of(p);
  *n = e ? (int)e->cand.size() : 0;
  for (int i = 0; i < *n && i < cap; i++) {
    if (fluid_per_sm) fluid_per_sm[i] = e->cand[i].first;
    if (particle_per_sm) particle_per_sm[i] = e->cand[i].second;
    if (ns_per_tile_step) ns_per_tile_step[i] = e->cost[i];
  }
  return 0;
}

extern "C" int d3q19_tune_export(char* buf, size_t cap, size_t* len) {
  if (!len || (cap && !buf)) return D3Q19_EINVAL;
  std::string out;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    char line[96];
    for (const auto& kv : g_tune) {
      const TuneEntry& e = kv.second;
      if (e.best < 0) continue;
      snprintf(line, sizeof(line), "\t%d\t%d\t%.6g\n", e.cand[e.best].first, e.cand[e.best].second,
               e.cost[e.best]);
      out += kv.first;
      out += line;
    }
  }
  *len = out.size();
  if (cap < out.size() + 1) return cap ? D3Q19_ENOMEM : 0;
  memcpy(buf, out.c_str(), out.size() + 1);
  return 0;
}

extern "C" int d3q19_tune_import(const char* text) {
  if (!text) return D3Q19_EINVAL;
  std::vector<std::pair<std::string, TuneEntry>> add;
  const char* q = text;
  while (*q) {
    const char* eol = strchr(q, '\n');
    const std::string line(q, eol ? (size_t)(eol - q) : strlen(q));
    q = eol ? eol + 1 : q + line.size();
    if (line.empty()) continue;
    // name, SMs, storage, inplace, class: the key; then the choice and its time.
    std::vector<std::string> fld;
    size_t a = 0;
    for (size_t b; (b = line.find('\t', a)) != std::string::npos; a = b + 1) fld.push_back(line.substr(a, b - a));
    fld.push_back(line.substr(a));
    if (fld.size() != 8 || fld[0].empty()) return D3Q19_EINVAL;
    int v[6];
    double ns = 0;
    char* end = nullptr;
    for (int i = 0; i < 6; i++) {
      const long x = strtol(fld[1 + i].c_str(), &end, 10);
      if (*end || fld[1 + i].empty() || x < 0 || x > 1000000) return D3Q19_EINVAL;
      v[i] = (int)x;
    }
    ns = strtod(fld[7].c_str(), &end);
    if (*end || fld[7].empty() || !(ns >= 0)) return D3Q19_EINVAL;
    if (v[1] > 2 || v[2] > 1 || v[5] < 1) return D3Q19_EINVAL;
    TuneEntry e;
    e.cand.push_back({v[4], v[5]});
    e.cost.push_back(ns);
    e.best = 0;
    add.emplace_back(tune_key_of(fld[0].c_str(), v[0], v[1], v[2], v[3]), e);
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (auto& kv : add) g_tune[kv.first] = kv.second;
  return 0;
}

extern "C" int d3q19_tune_clear(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
  return 0;
}

extern "C" int d3q19_pool_get_grid(d3q19_pool* p, int* fluid_blocks, int* particle_blocks, int* contact_blocks) {
  if (!p) return D3Q19_EINVAL;
  POOL_LOCK(p);
  if (fluid_blocks) *fluid_blocks = p->fgrid;
  if (particle_blocks) *particle_blocks = p->pblocks;
  if (contact_blocks) *contact_blocks = p->cblocks;
  return 0;
}

extern "C" int d3q19_pool_poll(d3q19_pool* p) {
  if (!p) return D3Q19_EINVAL;
  POOL_LOCK(p);
  cudaSetDevice(p->dev);
  const cudaError_t e = cudaEventQuery(p->ev_done);
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) return 0;
  return pfail(p, D3Q19_ECUDA, "cudaEventQuery: %s", cudaGetErrorString(e));
}

extern "C" int d3q19_pool_synchronize(d3q19_pool* p) {
  if (!p) return D3Q19_EINVAL;
  POOL_LOCK(p);
  cudaSetDevice(p->dev);
  POOL_TRY(p, cudaStreamSynchronize(p->stream));
  for (int s = 0; s < p->max_slots; s++)
    if (p->slot[s])
      if (int rc = d3q19_synchronize(p->slot[s]))
        return pfail(p, rc, "member %d: %s", s, d3q19_last_error(p->slot[s]));
  return 0;
}

extern "C" void* d3q19_pool_stream(d3q19_pool* p) { return p ? (void*)p->stream : nullptr; }

extern "C" const char* d3q19_pool_last_error(d3q19_pool* p) { return p ? p->msg : g_create_error; }

extern "C" int d3q19_pool_destroy(d3q19_pool* p) {
  if (!p) return D3Q19_EINVAL;
  // Waits for a call in progress on another thread; none may start after it.
  { POOL_LOCK(p); }
  cudaSetDevice(p->dev);
  if (p->stream) cudaStreamSynchronize(p->stream);
  tune_collect(p);  // a timed advance still counts
  pool_drop_graphs(p);
  for (auto*& c : p->slot)
    if (c) {
      c->free_stream = p->stream;
      d3q19_destroy(c);
      c = nullptr;
    }
  void* ptrs[] = {p->d_fargs, p->d_pargs, p->d_zargs, p->d_work, p->d_zslots, p->d_counts, p->d_stats};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (p->stream) cudaStreamSynchronize(p->stream);  // the members' stream-ordered frees
  if (p->mempool) cudaMemPoolDestroy(p->mempool);
  if (p->ev_done) cudaEventDestroy(p->ev_done);
  for (auto& e : p->tune_events) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
  return 0;
}
