// Random 32-byte sector gather throughput: the roofline denominator of the
// search kernels, whose every step is one dependent random 32-byte load.
// Each thread runs `chains` independent pointer-chase-like chains over a
// buffer of `bytes` (sector index of the next load = hash of the data just
// loaded), so the loads are random, dependent within a chain and independent
// across chains -- the access pattern of the SBWT walk with the memory-level
// parallelism the hardware can sustain.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.hpp"
#include "rank_blocks.cuh"

namespace sbwt {

template <int CH>
__global__ void __launch_bounds__(256) gather_kernel(const Block *buf, uint64_t n_sectors,
                                                     uint32_t iters, uint64_t *sink) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t idx[CH];
#pragma unroll
  for (int c = 0; c < CH; ++c) idx[c] = ((t * CH + c) * 0x9E3779B97F4A7C15ULL) % n_sectors;
  uint64_t acc = 0;
  for (uint32_t it = 0; it < iters; ++it) {
    Block b[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) b[c] = load_block(buf + idx[c]);
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      const uint64_t h = (b[c].w0 ^ b[c].w3 ^ idx[c]) * 0xBF58476D1CE4E5B9ULL;
      idx[c] = (h ^ (h >> 31)) % n_sectors;
      acc += b[c].w1;
    }
  }
  if (acc == 0x123456789ULL) sink[0] = acc;  // keeps the loads alive
}

__global__ void fill_kernel(Block *buf, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t h = (i + 1) * 0x94D049BB133111EBULL;
    buf[i] = Block{h, h ^ (h >> 29), i, h * 3};
  }
}

}  // namespace sbwt

extern "C" {
// Measures random 32-byte-sector gather throughput on `device` over a buffer
// of `bytes` bytes; writes GB/s (sectors x 32 B / s) and sectors/s.  The
// buffer is allocated and freed inside the call.
int sbwt_measure_random_sectors(int device, uint64_t bytes, int chains,
                                double *gbs, double *sectors_per_s) {
  using namespace sbwt;
  return guarded([&] {
    DeviceGuard g(device);
    const uint64_t n = std::max<uint64_t>(bytes / 32, 1024);
    DeviceBuffer buf(n * 32), sink(8);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    fill_kernel<<<sms * 8, 256>>>(buf.get<Block>(), n);
    const int grid = sms * 8;  // 2048 threads per SM
    const uint32_t iters = 64;
    cudaEvent_t e0, e1;
    SBWT_CUDA(cudaEventCreate(&e0));
    SBWT_CUDA(cudaEventCreate(&e1));
    auto run = [&] {
      switch (chains) {
        case 1: gather_kernel<1><<<grid, 256>>>(buf.get<Block>(), n, iters, sink.get<uint64_t>()); break;
        case 2: gather_kernel<2><<<grid, 256>>>(buf.get<Block>(), n, iters, sink.get<uint64_t>()); break;
        case 4: gather_kernel<4><<<grid, 256>>>(buf.get<Block>(), n, iters, sink.get<uint64_t>()); break;
        default: gather_kernel<8><<<grid, 256>>>(buf.get<Block>(), n, iters, sink.get<uint64_t>()); break;
      }
    };
    run();
    SBWT_CUDA(cudaEventRecord(e0));
    for (int rep = 0; rep < 5; ++rep) run();
    SBWT_CUDA(cudaEventRecord(e1));
    SBWT_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SBWT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int ch = (chains == 1 || chains == 2 || chains == 4) ? chains : 8;
    const double sectors = 5.0 * grid * 256.0 * ch * iters;
    if (sectors_per_s) *sectors_per_s = sectors / (ms / 1e3);
    if (gbs) *gbs = sectors * 32.0 / (ms / 1e3) / 1e9;
  });
}
}
