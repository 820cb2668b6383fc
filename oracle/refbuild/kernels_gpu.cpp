// kernels_gpu.cpp -- compiles the reference's GPU_program.cl (the copy made
// by build_ref.sh into oracle/_ref/gen/, unchanged except for the dropped
// "#pragma OPENCL EXTENSION" line, and for the variable-viscosity build the
// dropped "#define USE_CONSTANT_VISCOSITY" line 4) and registers its kernels
// with the mock OpenCL runtime.  TEST INFRASTRUCTURE ONLY.
#include "clshim.hpp"

extern "C" int mockcl_quiet(void);
#define printf(...) (mockcl_quiet() ? 0 : std::printf(__VA_ARGS__))

#include GPU_PROGRAM_SOURCE

#undef printf

typedef void (*mockcl_tramp)(void* const* args);
extern "C" void mockcl_register_kernel(const char* name, mockcl_tramp fn, int mode, int nargs);

#define A(i) (args[i])
#define I(i) (*(const int*)args[i])

// Argument lists follow the kernel signatures in GPU_program.cl:81-90,
// 258-261, 292-295, 316-324, 626-628, 737-742, 868-874.
static void t_pffls(void* const* args) {
  particle_fluid_forces_linear_stencil((int_param_struct*)A(0), (flp_param_struct*)A(1), (float*)A(2),
                                       (float*)A(3), (float4*)A(4), (float4*)A(5), (float4*)A(6), (float4*)A(7),
                                       (int*)A(8));
}
static void t_sum(void* const* args) {
  sum_particle_fluid_forces((int_param_struct*)A(0), (flp_param_struct*)A(1), (float*)A(2));
}
static void t_reset(void* const* args) {
  reset_particle_fluid_forces((int_param_struct*)A(0), (flp_param_struct*)A(1), (float*)A(2));
}
static void t_collide(void* const* args) {
  collideMRT_stream_D3Q19((float*)A(0), (float*)A(1), (float*)A(2), (float*)A(3), (float*)A(4), (int*)A(5),
                          (int_param_struct*)A(6), (flp_param_struct*)A(7));
}
// collideSRT_newtonian_stream_D3Q19 (GPU_program.cl:868-947): the reference's
// BGK collide-stream kernel, which its host does not call; run by
// srt_driver.c for the BGK golden vectors.
static void t_srt(void* const* args) {
  collideSRT_newtonian_stream_D3Q19((float*)A(0), (float*)A(1), (float*)A(2), (float*)A(3), (int_param_struct*)A(4),
                                    (flp_param_struct*)A(5));
}
static void t_periodic(void* const* args) {
  boundary_periodic((float*)A(0), (int_param_struct*)A(1), (int*)A(2));
}
static void t_velocity(void* const* args) {
  boundary_velocity((float*)A(0), (int_param_struct*)A(1), (flp_param_struct*)A(2), I(3), I(4));
}

__attribute__((constructor)) static void register_gpu_kernels() {
  mockcl_register_kernel("particle_fluid_forces_linear_stencil", t_pffls, 1, 9);
  mockcl_register_kernel("sum_particle_fluid_forces", t_sum, 0, 3);
  mockcl_register_kernel("reset_particle_fluid_forces", t_reset, 0, 3);
  mockcl_register_kernel("collideMRT_stream_D3Q19", t_collide, 0, 8);
  mockcl_register_kernel("collideSRT_newtonian_stream_D3Q19", t_srt, 0, 6);
  mockcl_register_kernel("boundary_periodic", t_periodic, 0, 3);
  mockcl_register_kernel("boundary_velocity", t_velocity, 0, 5);
}
