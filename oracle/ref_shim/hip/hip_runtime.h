/*
 * Host-only stand-in for <hip/hip_runtime.h>, written for this project so that
 * SBWT-Search's own kernels (IndexSearcher.cuh, Presearcher.cuh, Rank.cuh,
 * ColorSearcher.cuh, ColorPostProcessor.cuh) compile as plain C++ for the
 * CPU.  Each "thread" of a kernel is a call with the thread-local
 * blockIdx/threadIdx set by the driver (oracle/ref_driver.cpp,
 * oracle/ref_colors.cpp).  TEST INFRASTRUCTURE ONLY.
 *
 * Warp collectives (__shfl_xor_sync, __ballot_sync) are served by the warp
 * emulation in oracle/ref_colors.cpp: the 32 lanes of a warp run as fibers
 * on one host thread, each lane posts its operand and yields, and reads the
 * other lanes' operands once all 32 have posted.  ColorSearcher.cuh selects
 * its CUDA spelling of these collectives on __HIP_PLATFORM_NVIDIA__.
 */
#ifndef SBWT_ORACLE_HIP_RUNTIME_SHIM_H
#define SBWT_ORACLE_HIP_RUNTIME_SHIM_H
#include <cstdint>

#define __global__
#define __device__
#define __host__
#define __HIP_CPU_SHIM__ 1
#define __HIP_PLATFORM_NVIDIA__ 1

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
inline int __popc(unsigned int v) { return __builtin_popcount(v); }
inline int __clzll(long long v) {
  return v == 0 ? 64 : __builtin_clzll((unsigned long long)v);
}
inline unsigned long long __brevll(unsigned long long v) {
  unsigned long long r = 0;
  for (int i = 0; i < 64; ++i) r |= ((v >> i) & 1ULL) << (63 - i);
  return r;
}
inline long long llmin(long long a, long long b) { return a < b ? a : b; }
inline long long llmax(long long a, long long b) { return a > b ? a : b; }

/* Warp emulation (oracle/ref_colors.cpp): post this lane's operand, yield
 * until every lane of the warp has posted, return the buffer that holds the
 * 32 operands of this collective. */
const unsigned long long *shim_warp_exchange(unsigned long long v);
unsigned shim_lane_id();

template <class T>
inline T __shfl_xor_sync(unsigned /*mask*/, T v, int lane_mask) {
  const unsigned long long *ops = shim_warp_exchange((unsigned long long)v);
  return (T)ops[(shim_lane_id() ^ (unsigned)lane_mask) & 31u];
}
inline unsigned __ballot_sync(unsigned /*mask*/, int pred) {
  const unsigned long long *ops = shim_warp_exchange(pred != 0 ? 1ULL : 0ULL);
  unsigned r = 0;
  for (unsigned l = 0; l < 32; ++l) r |= (ops[l] ? 1u : 0u) << l;
  return r;
}
#endif
