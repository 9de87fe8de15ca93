/*
 * Host-only stand-in for <hip/hip_runtime.h>, written for this project so that
 * SBWT-Search's own index kernels (IndexSearcher.cuh, Presearcher.cuh,
 * Rank.cuh) compile as plain C++ for the CPU.  Each "thread" of a kernel is a
 * call with the thread-local blockIdx/threadIdx set by the driver
 * (oracle/ref_driver.cpp).  TEST INFRASTRUCTURE ONLY.
 */
#ifndef SBWT_ORACLE_HIP_RUNTIME_SHIM_H
#define SBWT_ORACLE_HIP_RUNTIME_SHIM_H
#include <cstdint>

#define __global__
#define __device__
#define __host__
#define __HIP_CPU_SHIM__ 1

struct ulonglong2 {
  unsigned long long x, y;
};
struct shim_dim3 {
  unsigned int x, y, z;
};
extern thread_local shim_dim3 blockIdx;
extern thread_local shim_dim3 blockDim;
extern thread_local shim_dim3 threadIdx;

inline int __popcll(unsigned long long v) { return __builtin_popcountll(v); }
#endif
