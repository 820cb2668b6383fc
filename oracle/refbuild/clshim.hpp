// clshim.hpp -- OpenCL C language shim so the reference's unmodified kernel
// sources (GPU_program.cl, CPU_program.cl) compile as C++ on the host.
//
// TEST INFRASTRUCTURE ONLY.  This header is part of the recipe that builds the
// reference itself (into oracle/_ref/) so that it can run on the host cores as
// the parity pin for the oracle and as the timed CPU baseline.  Nothing in the
// product library includes it.
//
// It supplies the OpenCL C built-ins the kernels use (OpenCL C 1.2 spec,
// sections 6.12.1-6.12.8): address-space qualifiers, float4 with the vector
// operators, fmod/floor/sqrt/pow/fabs/length/dot/cross, the work-item
// functions and atomic_inc/barrier.  Work-item state lives in thread-local
// storage set by the mock runtime (mock_cl.cpp) before each work-item runs.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstddef>

#define __kernel
#define __global
#define __local
#define __constant const
#define __private
#define kernel
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2

// --- vector type -----------------------------------------------------------
struct float4 {
  float x, y, z, w;
  float4& operator+=(const float4& b) { x += b.x; y += b.y; z += b.z; w += b.w; return *this; }
  float4& operator-=(const float4& b) { x -= b.x; y -= b.y; z -= b.z; w -= b.w; return *this; }
  float4& operator*=(float s) { x *= s; y *= s; z *= s; w *= s; return *this; }
  float4& operator/=(float s) { x /= s; y /= s; z /= s; w /= s; return *this; }
};
static inline float4 make_float4(float a, float b, float c, float d) { float4 r = {a, b, c, d}; return r; }
static inline float4 operator+(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
static inline float4 operator-(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
static inline float4 operator*(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
static inline float4 operator*(float s, float4 a) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
static inline float4 operator/(float4 a, float s) { return make_float4(a.x / s, a.y / s, a.z / s, a.w / s); }
static inline float4 operator-(float4 a) { return make_float4(-a.x, -a.y, -a.z, -a.w); }

// OpenCL geometric functions on float4 use all four components (6.12.5);
// cross() on float4 returns w = 0.
static inline float dot(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
static inline float length(float4 a) { return std::sqrt(dot(a, a)); }
static inline float4 cross(float4 a, float4 b) {
  return make_float4(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, 0.0f);
}
static inline float4 fmod(float4 a, float4 b) {
  return make_float4(std::fmod(a.x, b.x), std::fmod(a.y, b.y), std::fmod(a.z, b.z), std::fmod(a.w, b.w));
}
using std::fmod;
using std::floor;
using std::sqrt;
using std::pow;
using std::fabs;

// --- work-item functions (set by the mock runtime) -------------------------
struct mockcl_item_state {
  size_t gid[3], lid[3], gsize[3], lsize[3], grp[3], ngrp[3];
};
extern thread_local mockcl_item_state mockcl_item;
static inline size_t get_global_id(int d) { return mockcl_item.gid[d]; }
static inline size_t get_local_id(int d) { return mockcl_item.lid[d]; }
static inline size_t get_global_size(int d) { return mockcl_item.gsize[d]; }
static inline size_t get_local_size(int d) { return mockcl_item.lsize[d]; }
static inline size_t get_group_id(int d) { return mockcl_item.grp[d]; }
static inline size_t get_num_groups(int d) { return mockcl_item.ngrp[d]; }

// atomic_inc returns the old value (6.12.11).  Work-groups of the only kernel
// that uses it may run concurrently on several host threads, so it is a real
// atomic; the non-atomic slot update that follows it races exactly as it does
// on a GPU unless the runtime serialises the kernel (MOCKCL_SERIAL=1).
static inline int atomic_inc(volatile int* p) { return __atomic_fetch_add((int*)p, 1, __ATOMIC_RELAXED); }

// barrier() yields to the work-group's fiber scheduler (mock_cl.cpp).
void mockcl_barrier(void);
static inline void barrier(int) { mockcl_barrier(); }
