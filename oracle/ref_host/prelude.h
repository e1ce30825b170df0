/*
 * Host-C++ prelude that lets the reference's CUDA kernel sources compile as
 * plain CPU code.  TEST INFRASTRUCTURE ONLY: the library built from this
 * directory (oracle/_ref/libblaze_refhost.so) is the checker the parity tests
 * and the CPU baseline use; nothing in the product links or calls it.
 *
 * What it maps (the reference sources themselves are included unmodified):
 *   - __device__/__global__/__constant__/__host__ become empty, so every
 *     `__global__` kernel is an ordinary function and every `__constant__`
 *     object an ordinary global;
 *   - blockIdx/threadIdx/blockDim/gridDim become thread_local globals that the
 *     launch helper in refhost_kernels.cpp sets before each call;
 *   - __syncthreads is a no-op (no kernel on the sphere path depends on it for
 *     correctness; GPU_Memory_Transfer.cuh:149-158 only orders counter writes
 *     that the driver performs itself);
 *   - rsqrtf (absent on the host) is 1/sqrtf;
 *   - float/int atomicAdd use an OpenMP atomic capture (float ones are also
 *     reported to the driver, which sums the energy tallies' values in FP64);
 *   - Thrust is pointed at its sequential C++ backend, so the reference's own
 *     thrust::stable_sort_by_key call (Collision_Detection_BroadPhase.cuh:110-117)
 *     runs on the host unchanged.
 */
#ifndef BLAZE_REFHOST_PRELUDE_H_
#define BLAZE_REFHOST_PRELUDE_H_

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector_types.h>
#include <vector_functions.h>

#undef __device__
#undef __global__
#undef __constant__
#undef __host__
#undef __forceinline__
#define __device__
#define __global__
#define __constant__
#define __host__
#define __forceinline__ inline

extern thread_local uint3 blockIdx;
extern thread_local uint3 threadIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

static inline void __syncthreads() {}
static inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }

/* Every float atomicAdd is also reported to the driver, which keeps an FP64
 * sum of the same values for the energy tallies (refhost_kernels.cpp). */
void refh_float_added(float* a, float v);
static inline float atomicAdd(float* a, float v) {
  float o;
#pragma omp atomic capture
  { o = *a; *a += v; }
  refh_float_added(a, v);
  return o;
}
static inline int atomicAdd(int* a, int v) {
  int o;
#pragma omp atomic capture
  { o = *a; *a += v; }
  return o;
}

#define THRUST_DEVICE_SYSTEM THRUST_DEVICE_SYSTEM_CPP

#endif
