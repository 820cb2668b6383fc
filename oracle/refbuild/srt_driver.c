/* srt_driver.c -- runs the reference's BGK kernel collideSRT_newtonian_stream_D3Q19
 * (GPU_program.cl:868-947), which the reference's host program does not call,
 * in the host's per-step order of the fluid passes (sim_main.c:324-405):
 * collide-stream into the other buffer, then boundary_periodic
 * (GPU_program.cl:626-735) over the periodic node list, then
 * boundary_velocity (GPU_program.cl:737-865) on the wall axis, the two
 * buffers swapped by step parity as the host does.  The kernels run through
 * the mock OpenCL runtime, from the reference's own sources compiled by
 * build_ref.sh.  TEST INFRASTRUCTURE ONLY: it produces the BGK golden vectors
 * (tests/golden/make_golden_bgk.py); nothing here ships in the product.
 *
 * The kernel takes its body force from a force field g (the reference's
 * build without USE_CONSTANT_BODY_FORCE); the caller passes ConstBodyForce at
 * every node for a fluid without spheres.
 *
 * Input file (binary, native endianness):
 *   int_param_struct (332 B), flp_param_struct (176 B), int nsteps,
 *   int numPeriodicNodes, float f[19*N_C], float g[3*N_C],
 *   int strMap[2*numPeriodicNodes]
 * Output file: float f[19*N_C] (the buffer the last step wrote, after the
 *   boundary kernels), float u[3*N_C].
 *
 * Usage: srt_driver <input> <output>   (GPU_program.cl in the working directory)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "CL/cl.h"
#include "struct_header_host.h"

static void check(cl_int e, const char* what) {
  if (e != CL_SUCCESS) {
    fprintf(stderr, "srt_driver: %s failed (%d)\n", what, (int)e);
    exit(1);
  }
}

static void* read_exact(FILE* fh, size_t n, const char* what) {
  void* p = malloc(n ? n : 1);
  if (!p || fread(p, 1, n, fh) != n) {
    fprintf(stderr, "srt_driver: short input (%s)\n", what);
    exit(1);
  }
  return p;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: srt_driver <input> <output>\n");
    return 2;
  }
  FILE* in = fopen(argv[1], "rb");
  if (!in) {
    fprintf(stderr, "srt_driver: cannot open %s\n", argv[1]);
    return 1;
  }
  int_param_struct intDat;
  flp_param_struct flpDat;
  int nsteps = 0, nper = 0;
  if (fread(&intDat, sizeof(intDat), 1, in) != 1 || fread(&flpDat, sizeof(flpDat), 1, in) != 1 ||
      fread(&nsteps, sizeof(int), 1, in) != 1 || fread(&nper, sizeof(int), 1, in) != 1) {
    fprintf(stderr, "srt_driver: short header\n");
    return 1;
  }
  const size_t NC = (size_t)intDat.LatticeSize[0] * intDat.LatticeSize[1] * intDat.LatticeSize[2];
  float* f = (float*)read_exact(in, sizeof(float) * 19 * NC, "f");
  float* g = (float*)read_exact(in, sizeof(float) * 3 * NC, "g");
  int* strMap = (int*)read_exact(in, sizeof(int) * 2 * (size_t)nper, "strMap");
  fclose(in);

  cl_int e;
  cl_platform_id plat;
  cl_device_id dev;
  check(clGetPlatformIDs(1, &plat, NULL), "clGetPlatformIDs");
  check(clGetDeviceIDs(plat, CL_DEVICE_TYPE_GPU, 1, &dev, NULL), "clGetDeviceIDs");
  cl_context ctx = clCreateContext(NULL, 1, &dev, NULL, NULL, &e);
  check(e, "clCreateContext");
  cl_command_queue q = clCreateCommandQueue(ctx, dev, 0, &e);
  check(e, "clCreateCommandQueue");
  /* The program text, read from the working directory as the reference's
   * host does (D3Q19-OpenCL.c:465-497). */
  FILE* ph = fopen("GPU_program.cl", "rb");
  if (!ph) {
    fprintf(stderr, "srt_driver: GPU_program.cl not found in the working directory\n");
    return 1;
  }
  fseek(ph, 0, SEEK_END);
  const long plen = ftell(ph);
  fseek(ph, 0, SEEK_SET);
  char* text = (char*)read_exact(ph, (size_t)plen, "GPU_program.cl");
  fclose(ph);
  const char* src = text;
  const size_t srclen = (size_t)plen;
  cl_program prog = clCreateProgramWithSource(ctx, 1, &src, &srclen, &e);
  check(e, "clCreateProgramWithSource");
  check(clBuildProgram(prog, 1, &dev, NULL, NULL, NULL), "clBuildProgram");
  cl_kernel kc = clCreateKernel(prog, "collideSRT_newtonian_stream_D3Q19", &e);
  check(e, "clCreateKernel collideSRT_newtonian_stream_D3Q19");
  cl_kernel kp = clCreateKernel(prog, "boundary_periodic", &e);
  check(e, "clCreateKernel boundary_periodic");
  cl_kernel kv = clCreateKernel(prog, "boundary_velocity", &e);
  check(e, "clCreateKernel boundary_velocity");

  const size_t fb = sizeof(float) * 19 * NC;
  cl_mem fA = clCreateBuffer(ctx, CL_MEM_READ_WRITE | CL_MEM_COPY_HOST_PTR, fb, f, &e);
  check(e, "fA");
  cl_mem fB = clCreateBuffer(ctx, CL_MEM_READ_WRITE | CL_MEM_COPY_HOST_PTR, fb, f, &e);
  check(e, "fB");
  cl_mem gm = clCreateBuffer(ctx, CL_MEM_READ_WRITE | CL_MEM_COPY_HOST_PTR, sizeof(float) * 3 * NC, g, &e);
  check(e, "g");
  cl_mem um = clCreateBuffer(ctx, CL_MEM_READ_WRITE, sizeof(float) * 3 * NC, NULL, &e);
  check(e, "u");
  cl_mem im = clCreateBuffer(ctx, CL_MEM_READ_ONLY | CL_MEM_COPY_HOST_PTR, sizeof(intDat), &intDat, &e);
  check(e, "intDat");
  cl_mem pm = clCreateBuffer(ctx, CL_MEM_READ_ONLY | CL_MEM_COPY_HOST_PTR, sizeof(flpDat), &flpDat, &e);
  check(e, "flpDat");
  cl_mem sm = clCreateBuffer(ctx, CL_MEM_READ_ONLY | CL_MEM_COPY_HOST_PTR, sizeof(int) * 2 * (size_t)(nper ? nper : 1),
                             strMap, &e);
  check(e, "strMap");

  /* Work sizes and the wall axis as the host sets them (sim_main.c:209-236). */
  size_t off[3] = {1, 1, 1}, gsz[3], vsz[3];
  cl_int wallAxis = 0, calcRho = 0;
  int velBoundary = 0;
  for (int d = 0; d < 3; d++) {
    gsz[d] = (size_t)intDat.LatticeSize[d] - 2;
    if (intDat.BoundaryConds[d] == 1) {
      vsz[d] = 2;
      wallAxis = d;
      velBoundary = 1;
    } else {
      vsz[d] = (size_t)intDat.LatticeSize[d] - 2;
    }
  }
  const size_t psz = (size_t)nper;

  check(clSetKernelArg(kc, 2, sizeof(cl_mem), &gm), "arg g");
  check(clSetKernelArg(kc, 3, sizeof(cl_mem), &um), "arg u");
  check(clSetKernelArg(kc, 4, sizeof(cl_mem), &im), "arg intDat");
  check(clSetKernelArg(kc, 5, sizeof(cl_mem), &pm), "arg flpDat");
  check(clSetKernelArg(kp, 1, sizeof(cl_mem), &im), "arg intDat");
  check(clSetKernelArg(kp, 2, sizeof(cl_mem), &sm), "arg strMap");
  check(clSetKernelArg(kv, 1, sizeof(cl_mem), &im), "arg intDat");
  check(clSetKernelArg(kv, 2, sizeof(cl_mem), &pm), "arg flpDat");
  check(clSetKernelArg(kv, 3, sizeof(cl_int), &wallAxis), "arg wallAxis");
  check(clSetKernelArg(kv, 4, sizeof(cl_int), &calcRho), "arg calcRho");

  /* The step loop (sim_main.c:315-405): even t reads fA and writes fB. */
  for (int t = 1; t <= nsteps; t++) {
    cl_mem fc = (t % 2 == 0) ? fA : fB;
    cl_mem fs = (t % 2 == 0) ? fB : fA;
    check(clSetKernelArg(kc, 0, sizeof(cl_mem), &fc), "arg f_c");
    check(clSetKernelArg(kc, 1, sizeof(cl_mem), &fs), "arg f_s");
    check(clSetKernelArg(kp, 0, sizeof(cl_mem), &fs), "arg f (periodic)");
    check(clSetKernelArg(kv, 0, sizeof(cl_mem), &fs), "arg f (velocity)");
    check(clEnqueueNDRangeKernel(q, kc, 3, off, gsz, NULL, 0, NULL, NULL), "collideSRT");
    if (psz) check(clEnqueueNDRangeKernel(q, kp, 1, NULL, &psz, NULL, 0, NULL, NULL), "boundary_periodic");
    if (velBoundary) check(clEnqueueNDRangeKernel(q, kv, 3, off, vsz, NULL, 0, NULL, NULL), "boundary_velocity");
    check(clFinish(q), "clFinish");
  }
  cl_mem last = (nsteps % 2 == 1) ? fA : fB;
  float* u = (float*)malloc(sizeof(float) * 3 * NC);
  check(clEnqueueReadBuffer(q, last, CL_TRUE, 0, fb, f, 0, NULL, NULL), "read f");
  check(clEnqueueReadBuffer(q, um, CL_TRUE, 0, sizeof(float) * 3 * NC, u, 0, NULL, NULL), "read u");
  FILE* out = fopen(argv[2], "wb");
  if (!out || fwrite(f, sizeof(float), 19 * NC, out) != 19 * NC || fwrite(u, sizeof(float), 3 * NC, out) != 3 * NC) {
    fprintf(stderr, "srt_driver: cannot write %s\n", argv[2]);
    return 1;
  }
  fclose(out);
  return 0;
}
