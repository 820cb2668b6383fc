// mock_cl.cpp -- a small host-only OpenCL runtime that executes the
// reference's own kernels (compiled as C++ through clshim.hpp) on the host
// cores, so that the reference's unmodified host program runs end to end.
//
// TEST INFRASTRUCTURE ONLY.  It builds the reference into oracle/_ref/, where
// it serves as the parity pin for the oracle restatement and as the timed
// CPU baseline ("kind": "reference").  It is never linked into the product.
//
// Model: one platform exposing one CPU device and one GPU device (the
// reference requires both, D3Q19-OpenCL.c:881-894), both executing on the
// host.  Queues are in-order and every enqueue completes before it returns,
// which is one valid serialisation of the reference's two overlapping queues
// (sim_main.c:358-447: the CPU-queue and GPU-queue kernels of one step touch
// disjoint buffers between the clFinish points).
//
// Execution of one NDRange:
//   * kernels without barrier or cross-item writes run their work-items in
//     parallel over host threads (OpenMP over the outermost dimension);
//   * particle_fluid_forces_linear_stencil (the only kernel with barrier())
//     runs each work-group on one host thread as ucontext fibers, one fiber
//     per work-item, switching at every barrier;  work-groups run in
//     parallel unless MOCKCL_SERIAL=1, which runs them in group order and
//     gives the race-free, deterministic slot semantics;
//   * the CPU-device particle kernels run their work-items serially in
//     work-item order (their cross-item parForce/zone updates race otherwise).
//
// Environment:
//   MOCKCL_KERNEL_WG_SIZE  value reported for CL_KERNEL_WORK_GROUP_SIZE (256)
//   MOCKCL_SERIAL          1 = run every kernel serially, groups in order
//   MOCKCL_SERIAL_FIBERS   1 = run the kernel with barrier() (the IBM spread,
//                          whose slot updates race between concurrent groups)
//                          in group order, the other kernels in parallel
//   MOCKCL_THREADS         host threads (default: all)
//   MOCKCL_DUMP_DIR        dump every buffer to <dir>/buf_<creation#>.bin when
//                          the host releases it (sim_main.c:510-512)
//   MOCKCL_QUIET           1 = drop the kernels' device printf output

#include "CL/cl.h"
#include "clshim.hpp"

#include <omp.h>
#include <ucontext.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

thread_local mockcl_item_state mockcl_item;

typedef void (*mockcl_tramp)(void* const* args);
enum mockcl_mode { MODE_PARALLEL = 0, MODE_FIBERS = 1, MODE_SERIAL = 2 };

struct mockcl_kdef {
  const char* name;
  mockcl_tramp fn;
  int mode;
  int nargs;
};

static std::vector<mockcl_kdef>& registry() {
  static std::vector<mockcl_kdef> r;
  return r;
}

extern "C" void mockcl_register_kernel(const char* name, mockcl_tramp fn, int mode, int nargs) {
  registry().push_back({name, fn, mode, nargs});
}

struct _cl_platform_id { int dummy; };
struct _cl_device_id { cl_device_type type; const char* name; };
struct _cl_context { int dummy; };
struct _cl_command_queue { cl_device_id dev; };
struct _cl_mem { void* data; size_t size; int id; bool live; };
struct _cl_program { std::string src; };
struct _cl_kernel {
  mockcl_kdef def;
  unsigned char bytes[16][16];
  cl_mem mem[16];
  bool is_mem[16];
};

static _cl_platform_id g_platform;
static _cl_device_id g_cpu = {CL_DEVICE_TYPE_CPU, "mockcl host device (CPU role)"};
static _cl_device_id g_gpu = {CL_DEVICE_TYPE_GPU, "mockcl host device (GPU role)"};
static _cl_context g_context;
static std::vector<_cl_mem*> g_mems;

static int env_int(const char* k, int def) {
  const char* v = getenv(k);
  return v && *v ? atoi(v) : def;
}

static bool is_live_mem(const void* p) {
  for (auto* m : g_mems)
    if ((const void*)m == p && m->live) return true;
  return false;
}

extern "C" {

cl_int clGetPlatformIDs(cl_uint n, cl_platform_id* p, cl_uint* num) {
  if (num) *num = 1;
  if (p && n > 0) p[0] = &g_platform;
  return CL_SUCCESS;
}

cl_int clGetPlatformInfo(cl_platform_id, cl_platform_info, size_t sz, void* v, size_t* ret) {
  const char* name = "mockcl host platform";
  size_t need = strlen(name) + 1;
  if (ret) *ret = need;
  if (v && sz >= need) memcpy(v, name, need);
  return CL_SUCCESS;
}

cl_int clGetDeviceIDs(cl_platform_id, cl_device_type t, cl_uint n, cl_device_id* d, cl_uint* num) {
  cl_device_id dev = (t & CL_DEVICE_TYPE_GPU) ? &g_gpu : &g_cpu;
  if (num) *num = 1;
  if (d && n > 0) d[0] = dev;
  return CL_SUCCESS;
}

cl_int clGetDeviceInfo(cl_device_id dev, cl_device_info what, size_t sz, void* v, size_t* ret) {
  if (!v) return CL_SUCCESS;
  switch (what) {
    case CL_DEVICE_NAME: {
      size_t need = strlen(dev->name) + 1;
      if (sz >= need) memcpy(v, dev->name, need);
      if (ret) *ret = need;
      break;
    }
    case CL_DEVICE_MAX_COMPUTE_UNITS: *(cl_uint*)v = (cl_uint)omp_get_max_threads(); break;
    case CL_DEVICE_MAX_CLOCK_FREQUENCY: *(cl_uint*)v = 0; break;
    case CL_DEVICE_GLOBAL_MEM_SIZE:
    case CL_DEVICE_MAX_CONSTANT_BUFFER_SIZE: *(cl_ulong*)v = (cl_ulong)1 << 34; break;
    case CL_DEVICE_MAX_WORK_ITEM_SIZES: {
      size_t* s = (size_t*)v;
      for (size_t i = 0; i < sz / sizeof(size_t) && i < 3; i++) s[i] = 1024;
      break;
    }
    case CL_DEVICE_MAX_WORK_GROUP_SIZE: *(size_t*)v = 1024; break;
    default: break;
  }
  return CL_SUCCESS;
}

cl_context clCreateContext(const cl_context_properties*, cl_uint, const cl_device_id*,
                           void (*)(const char*, const void*, size_t, void*), void*, cl_int* err) {
  if (err) *err = CL_SUCCESS;
  if (env_int("MOCKCL_THREADS", 0) > 0) omp_set_num_threads(env_int("MOCKCL_THREADS", 0));
  return &g_context;
}

cl_command_queue clCreateCommandQueue(cl_context, cl_device_id d, cl_command_queue_properties, cl_int* err) {
  if (err) *err = CL_SUCCESS;
  return new _cl_command_queue{d};
}

cl_command_queue clCreateCommandQueueWithProperties(cl_context c, cl_device_id d, const cl_queue_properties*,
                                                    cl_int* err) {
  return clCreateCommandQueue(c, d, 0, err);
}

cl_program clCreateProgramWithSource(cl_context, cl_uint n, const char** src, const size_t* len, cl_int* err) {
  auto* p = new _cl_program;
  for (cl_uint i = 0; i < n; i++) p->src += len && len[i] ? std::string(src[i], len[i]) : std::string(src[i]);
  if (err) *err = CL_SUCCESS;
  return p;
}

cl_int clBuildProgram(cl_program, cl_uint, const cl_device_id*, const char*, void (*)(cl_program, void*), void*) {
  return CL_SUCCESS;  // kernels are compiled ahead of time from the same sources
}

cl_int clGetProgramBuildInfo(cl_program, cl_device_id, cl_program_build_info, size_t sz, void* v, size_t* ret) {
  if (ret) *ret = 1;
  if (v && sz) ((char*)v)[0] = 0;
  return CL_SUCCESS;
}

cl_kernel clCreateKernel(cl_program prog, const char* name, cl_int* err) {
  // The kernel must both exist in the ahead-of-time registry and appear in
  // the program text the host loaded, as a real OpenCL build would require.
  for (auto& d : registry()) {
    if (strcmp(d.name, name) == 0 && prog->src.find(name) != std::string::npos) {
      auto* k = new _cl_kernel;
      memset(k, 0, sizeof(*k));
      k->def = d;
      if (err) *err = CL_SUCCESS;
      return k;
    }
  }
  if (err) *err = CL_INVALID_KERNEL_NAME;
  return nullptr;
}

cl_int clGetKernelWorkGroupInfo(cl_kernel, cl_device_id, cl_kernel_work_group_info what, size_t sz, void* v,
                                size_t* ret) {
  if (what == CL_KERNEL_WORK_GROUP_SIZE && v && sz >= sizeof(size_t))
    *(size_t*)v = (size_t)env_int("MOCKCL_KERNEL_WG_SIZE", 256);
  if (ret) *ret = sizeof(size_t);
  return CL_SUCCESS;
}

cl_int clSetKernelArg(cl_kernel k, cl_uint idx, size_t sz, const void* val) {
  if (idx >= 16 || sz > 16) return CL_INVALID_ARG_INDEX;
  memset(k->bytes[idx], 0, 16);
  if (val) memcpy(k->bytes[idx], val, sz);
  k->is_mem[idx] = false;
  if (sz == sizeof(cl_mem) && val && is_live_mem(*(void* const*)val)) {
    k->is_mem[idx] = true;
    k->mem[idx] = *(cl_mem const*)val;
  }
  return CL_SUCCESS;
}

cl_mem clCreateBuffer(cl_context, cl_mem_flags flags, size_t size, void* host, cl_int* err) {
  auto* m = new _cl_mem;
  m->size = size;
  m->data = aligned_alloc(64, (size + 63) / 64 * 64);
  memset(m->data, 0, size);
  if ((flags & (CL_MEM_COPY_HOST_PTR | CL_MEM_USE_HOST_PTR)) && host) memcpy(m->data, host, size);
  m->id = (int)g_mems.size();
  m->live = true;
  g_mems.push_back(m);
  if (err) *err = CL_SUCCESS;
  return m;
}

cl_int clEnqueueWriteBuffer(cl_command_queue, cl_mem m, cl_bool, size_t off, size_t n, const void* src, cl_uint,
                            const cl_event*, cl_event*) {
  if (off + n > m->size) return CL_INVALID_VALUE;
  memcpy((char*)m->data + off, src, n);
  return CL_SUCCESS;
}

cl_int clEnqueueReadBuffer(cl_command_queue, cl_mem m, cl_bool, size_t off, size_t n, void* dst, cl_uint,
                           const cl_event*, cl_event*) {
  if (off + n > m->size) return CL_INVALID_VALUE;
  memcpy(dst, (char*)m->data + off, n);
  return CL_SUCCESS;
}

void* clEnqueueMapBuffer(cl_command_queue, cl_mem m, cl_bool, cl_map_flags, size_t off, size_t n, cl_uint,
                         const cl_event*, cl_event*, cl_int* err) {
  if (err) *err = (off + n > m->size) ? CL_INVALID_VALUE : CL_SUCCESS;
  return (char*)m->data + off;
}

cl_int clEnqueueUnmapMemObject(cl_command_queue, cl_mem, void*, cl_uint, const cl_event*, cl_event*) {
  return CL_SUCCESS;
}

cl_int clFinish(cl_command_queue) { return CL_SUCCESS; }

cl_int clReleaseKernel(cl_kernel k) {
  delete k;
  return CL_SUCCESS;
}

cl_int clReleaseMemObject(cl_mem m) {
  const char* dir = getenv("MOCKCL_DUMP_DIR");
  if (dir && *dir) {
    char path[4096];
    snprintf(path, sizeof(path), "%s/buf_%02d.bin", dir, m->id);
    FILE* f = fopen(path, "wb");
    if (f) {
      fwrite(m->data, 1, m->size, f);
      fclose(f);
    }
  }
  m->live = false;
  free(m->data);
  m->data = nullptr;
  return CL_SUCCESS;
}

cl_int clReleaseProgram(cl_program) { return CL_SUCCESS; }
cl_int clReleaseCommandQueue(cl_command_queue) { return CL_SUCCESS; }
cl_int clReleaseContext(cl_context) { return CL_SUCCESS; }
cl_int clReleaseDevice(cl_device_id) { return CL_SUCCESS; }

}  // extern "C"

// --- NDRange execution -------------------------------------------------------

struct launch_t {
  mockcl_tramp fn;
  void* args[16];
  size_t off[3], gsz[3], lsz[3], ngrp[3];
};

static inline void set_item(const launch_t& L, size_t g0, size_t g1, size_t g2, size_t l0, size_t l1, size_t l2) {
  mockcl_item_state& s = mockcl_item;
  size_t g[3] = {g0, g1, g2}, l[3] = {l0, l1, l2};
  for (int d = 0; d < 3; d++) {
    s.grp[d] = g[d];
    s.lid[d] = l[d];
    s.gid[d] = L.off[d] + g[d] * L.lsz[d] + l[d];
    s.gsize[d] = L.gsz[d];
    s.lsize[d] = L.lsz[d];
    s.ngrp[d] = L.ngrp[d];
  }
}

// Fiber machinery for work-groups that call barrier().
static const size_t kFiberStack = 128 * 1024;
struct fiber_group {
  std::vector<ucontext_t> ctx;
  std::vector<char*> stacks;
  std::vector<char> done;
  ucontext_t sched;
  int cur;
  const launch_t* L;
  size_t grp[3];
  size_t lid[1024][3];
};
static thread_local fiber_group* t_fg = nullptr;

void mockcl_barrier(void) {
  fiber_group* fg = t_fg;
  if (!fg) return;  // kernels run without fibers never reach a barrier
  swapcontext(&fg->ctx[fg->cur], &fg->sched);
}

static void fiber_entry() {
  fiber_group* fg = t_fg;
  int i = fg->cur;
  fg->L->fn(fg->L->args);
  fg->done[i] = 1;
}

static void run_group_fibers(fiber_group& fg, const launch_t& L, size_t g0, size_t g1, size_t g2) {
  size_t nloc = L.lsz[0] * L.lsz[1] * L.lsz[2];
  if (nloc > 1024) {
    fprintf(stderr, "mockcl: work-group of %zu items exceeds 1024\n", nloc);
    exit(1);
  }
  if (fg.ctx.size() < nloc) {
    size_t old = fg.ctx.size();
    fg.ctx.resize(nloc);
    fg.stacks.resize(nloc);
    for (size_t i = old; i < nloc; i++) fg.stacks[i] = (char*)malloc(kFiberStack);
  }
  fg.done.assign(nloc, 0);
  fg.L = &L;
  t_fg = &fg;
  size_t i = 0;
  for (size_t c = 0; c < L.lsz[2]; c++)
    for (size_t b = 0; b < L.lsz[1]; b++)
      for (size_t a = 0; a < L.lsz[0]; a++, i++) {
        fg.lid[i][0] = a;
        fg.lid[i][1] = b;
        fg.lid[i][2] = c;
        getcontext(&fg.ctx[i]);
        fg.ctx[i].uc_stack.ss_sp = fg.stacks[i];
        fg.ctx[i].uc_stack.ss_size = kFiberStack;
        fg.ctx[i].uc_link = &fg.sched;
        makecontext(&fg.ctx[i], (void (*)())fiber_entry, 0);
      }
  size_t remaining = nloc;
  while (remaining) {
    for (size_t k = 0; k < nloc; k++) {
      if (fg.done[k]) continue;
      set_item(L, g0, g1, g2, fg.lid[k][0], fg.lid[k][1], fg.lid[k][2]);
      fg.cur = (int)k;
      swapcontext(&fg.sched, &fg.ctx[k]);
      if (fg.done[k]) remaining--;
    }
  }
  t_fg = nullptr;
}

extern "C" cl_int clEnqueueNDRangeKernel(cl_command_queue, cl_kernel k, cl_uint dims, const size_t* off,
                                         const size_t* gsz, const size_t* lsz, cl_uint, const cl_event*,
                                         cl_event*) {
  launch_t L;
  L.fn = k->def.fn;
  for (int i = 0; i < 16; i++) L.args[i] = k->is_mem[i] ? k->mem[i]->data : (void*)k->bytes[i];
  for (int d = 0; d < 3; d++) {
    L.off[d] = (off && d < (int)dims) ? off[d] : 0;
    L.gsz[d] = d < (int)dims ? gsz[d] : 1;
    L.lsz[d] = (lsz && d < (int)dims) ? lsz[d] : 1;
    if (L.gsz[d] % L.lsz[d]) return -54;  // CL_INVALID_WORK_GROUP_SIZE
    L.ngrp[d] = L.gsz[d] / L.lsz[d];
  }
  bool serial = env_int("MOCKCL_SERIAL", 0) != 0;
  int mode = k->def.mode;
  if (mode == MODE_FIBERS) {
    size_t ng = L.ngrp[0] * L.ngrp[1] * L.ngrp[2];
    if (serial || env_int("MOCKCL_SERIAL_FIBERS", 0) != 0) {
      fiber_group fg;
      for (size_t g = 0; g < ng; g++)
        run_group_fibers(fg, L, g % L.ngrp[0], (g / L.ngrp[0]) % L.ngrp[1], g / (L.ngrp[0] * L.ngrp[1]));
      for (auto* s : fg.stacks) free(s);
    } else {
#pragma omp parallel
      {
        fiber_group fg;
#pragma omp for schedule(dynamic, 1)
        for (long long g = 0; g < (long long)ng; g++)
          run_group_fibers(fg, L, g % L.ngrp[0], (g / L.ngrp[0]) % L.ngrp[1], g / (L.ngrp[0] * L.ngrp[1]));
        for (auto* s : fg.stacks) free(s);
      }
    }
    return CL_SUCCESS;
  }
  // Work-items without barriers: one item at a time, groups of size 1 unless
  // the host asked for a local size (group/local ids are still reported).
  long long n2 = (long long)L.gsz[2];
  auto run_slice = [&](long long z) {
    for (size_t y = 0; y < L.gsz[1]; y++)
      for (size_t x = 0; x < L.gsz[0]; x++) {
        set_item(L, x / L.lsz[0], y / L.lsz[1], (size_t)z / L.lsz[2], x % L.lsz[0], y % L.lsz[1],
                 (size_t)z % L.lsz[2]);
        L.fn(L.args);
      }
  };
  if (mode == MODE_SERIAL || serial) {
    for (long long z = 0; z < n2; z++) run_slice(z);
  } else if (dims == 1) {
    long long n0 = (long long)L.gsz[0];
#pragma omp parallel for schedule(static)
    for (long long x = 0; x < n0; x++) {
      set_item(L, (size_t)x / L.lsz[0], 0, 0, (size_t)x % L.lsz[0], 0, 0);
      L.fn(L.args);
    }
  } else {
#pragma omp parallel for schedule(static)
    for (long long z = 0; z < n2; z++) run_slice(z);
  }
  return CL_SUCCESS;
}

// Drop the kernels' device printf when asked (tau-clamp warnings can flood).
extern "C" int mockcl_quiet(void) {
  static int q = -1;
  if (q < 0) q = env_int("MOCKCL_QUIET", 0);
  return q;
}
