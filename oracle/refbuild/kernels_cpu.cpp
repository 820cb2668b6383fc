// kernels_cpu.cpp -- compiles the reference's CPU_program.cl (the copy made
// by build_ref.sh into oracle/_ref/gen/, where the OpenCL vector literal
// "(float4)(a,b,c,d)" of CPU_program.cl:95 is rewritten as make_float4(...)
// because C++ would read it as a comma expression) and registers its kernels
// with the mock OpenCL runtime.  TEST INFRASTRUCTURE ONLY.
#include "clshim.hpp"

#include CPU_PROGRAM_SOURCE

typedef void (*mockcl_tramp)(void* const* args);
extern "C" void mockcl_register_kernel(const char* name, mockcl_tramp fn, int mode, int nargs);

#define A(i) (args[i])

// Argument lists follow CPU_program.cl:76-86, 187-194, 280-288.
static void t_ppf(void* const* args) {
  particle_particle_forces((int_param_struct*)A(0), (flp_param_struct*)A(1), (float4*)A(2), (float4*)A(3),
                           (int*)A(4), (int*)A(5), (int*)A(6), (int*)A(7), (int*)A(8), (int*)A(9));
}
static void t_dyn(void* const* args) {
  particle_dynamics((int_param_struct*)A(0), (flp_param_struct*)A(1), (float4*)A(2), (float4*)A(3),
                    (float4*)A(4), (int*)A(5), (int*)A(6));
}
static void t_zones(void* const* args) {
  update_particle_zones((int_param_struct*)A(0), (flp_param_struct*)A(1), (float4*)A(2), (int*)A(3), (int*)A(4),
                        (int*)A(5), (int*)A(6), (int*)A(7));
}

__attribute__((constructor)) static void register_cpu_kernels() {
  mockcl_register_kernel("particle_particle_forces", t_ppf, 2, 10);
  mockcl_register_kernel("particle_dynamics", t_dyn, 2, 7);
  mockcl_register_kernel("update_particle_zones", t_zones, 2, 8);
}
