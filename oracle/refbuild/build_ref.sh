#!/usr/bin/env bash
# build_ref.sh -- builds the reference itself (SB8/Dispersion-Shear_D3Q19-OpenCL)
# for the host cores, from its sources where they lie, into oracle/_ref/.
#
# TEST INFRASTRUCTURE ONLY: the result is the parity pin for the oracle
# restatement and the timed CPU baseline.  Nothing here ships in the product.
#
# What it does (no reference build system is run; there is none):
#   1. copies GPU_program.cl / CPU_program.cl into oracle/_ref/gen/ with the
#      minimum edits a C++ compiler needs:
#        - drop "#pragma OPENCL EXTENSION ..." (GPU_program.cl:2);
#        - CPU_program.cl:95 "(float4)(" -> "make_float4(" (OpenCL vector
#          literal that C++ would parse as a comma expression);
#      and a second GPU copy without "#define USE_CONSTANT_VISCOSITY"
#      (GPU_program.cl:4), the reference's own switch for the power-law /
#      Casson / Herschel-Bulkley path;
#   2. compiles the unmodified host program D3Q19-OpenCL.c (which #includes
#      sim_main.c) against the hand-written CL/cl.h here;
#   3. links it with the mock OpenCL runtime (mock_cl.cpp) and the kernels,
#      giving oracle/_ref/ref_const (as shipped) and oracle/_ref/ref_var;
#   4. copies the runtime data the host opens from its working directory
#      (the two .cl files it reads as program text, and the unit-sphere
#      partitions) into oracle/_ref/run_data/ so the binaries can run where
#      the reference tree is absent.
#
# Usage: oracle/refbuild/build_ref.sh <reference_dir>   (or D3Q19_REFERENCE=<reference_dir>)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REPO="$(cd "$HERE/../.." && pwd)"
REF="${1:-${D3Q19_REFERENCE:-}}"
if [ -z "$REF" ]; then
  echo "usage: build_ref.sh <reference_dir> (or set D3Q19_REFERENCE)" >&2
  exit 2
fi
OUT="$REPO/oracle/_ref"

if [ ! -f "$REF/GPU_program.cl" ]; then
  echo "build_ref: reference sources not found at $REF" >&2
  exit 2
fi

mkdir -p "$OUT/gen" "$OUT/obj" "$OUT/run_data/unit_sphere_partitions"

sed -e '/#pragma OPENCL EXTENSION/d' "$REF/GPU_program.cl" > "$OUT/gen/GPU_program_const.cl"
sed -e '/#pragma OPENCL EXTENSION/d' -e '/^#define USE_CONSTANT_VISCOSITY/d' "$REF/GPU_program.cl" \
  > "$OUT/gen/GPU_program_var.cl"
sed -e 's/(float4)(/make_float4(/' "$REF/CPU_program.cl" > "$OUT/gen/CPU_program.cl"

if grep -q 'USE_CONSTANT_VISCOSITY$' "$OUT/gen/GPU_program_var.cl" && \
   grep -q '^#define USE_CONSTANT_VISCOSITY' "$OUT/gen/GPU_program_var.cl"; then
  echo "build_ref: failed to remove USE_CONSTANT_VISCOSITY" >&2
  exit 3
fi

CFLAGS="-O3 -ffp-contract=off -w"
CXXFLAGS="-O3 -ffp-contract=off -std=gnu++17 -fopenmp -Wno-narrowing -w"

gcc $CFLAGS -I"$HERE" -I"$REF" -c "$REF/D3Q19-OpenCL.c" -o "$OUT/obj/host.o"
g++ $CXXFLAGS -I"$HERE" -c "$HERE/mock_cl.cpp" -o "$OUT/obj/mock_cl.o"
g++ $CXXFLAGS -I"$HERE" -I"$OUT" -DCPU_PROGRAM_SOURCE='"gen/CPU_program.cl"' \
  -c "$HERE/kernels_cpu.cpp" -o "$OUT/obj/kernels_cpu.o"
for v in const var; do
  g++ $CXXFLAGS -I"$HERE" -I"$OUT" -DGPU_PROGRAM_SOURCE="\"gen/GPU_program_${v}.cl\"" \
    -c "$HERE/kernels_gpu.cpp" -o "$OUT/obj/kernels_gpu_${v}.o"
  g++ -fopenmp "$OUT/obj/host.o" "$OUT/obj/mock_cl.o" "$OUT/obj/kernels_cpu.o" "$OUT/obj/kernels_gpu_${v}.o" \
    -lm -o "$OUT/ref_${v}"
done

# The BGK driver: the reference's collideSRT_newtonian_stream_D3Q19 with its
# boundary kernels, in the host's per-step order (srt_driver.c).
gcc $CFLAGS -I"$HERE" -I"$REF" -c "$HERE/srt_driver.c" -o "$OUT/obj/srt_driver.o"
g++ -fopenmp "$OUT/obj/srt_driver.o" "$OUT/obj/mock_cl.o" "$OUT/obj/kernels_cpu.o" "$OUT/obj/kernels_gpu_const.o" \
  -lm -o "$OUT/srt_driver"
# The same kernels compiled with fused multiply-add contraction (what an
# OpenCL GPU compiler does by default): the reference's own rounding spread.
if grep -q -m1 ' fma ' /proc/cpuinfo; then
  g++ ${CXXFLAGS/-ffp-contract=off/-ffp-contract=fast} -mfma -I"$HERE" -I"$OUT" \
    -DGPU_PROGRAM_SOURCE='"gen/GPU_program_const.cl"' -c "$HERE/kernels_gpu.cpp" -o "$OUT/obj/kernels_gpu_const_fma.o"
  g++ -fopenmp "$OUT/obj/srt_driver.o" "$OUT/obj/mock_cl.o" "$OUT/obj/kernels_cpu.o" \
    "$OUT/obj/kernels_gpu_const_fma.o" -lm -o "$OUT/srt_driver_fma"
fi

cp "$REF/GPU_program.cl" "$REF/CPU_program.cl" "$OUT/run_data/"
cp "$REF"/unit_sphere_partitions/*.txt "$OUT/run_data/unit_sphere_partitions/"
echo "build_ref: built $OUT/ref_const, $OUT/ref_var and $OUT/srt_driver"
