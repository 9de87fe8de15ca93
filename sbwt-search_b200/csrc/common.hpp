// Shared host-side helpers of the library: status/error plumbing, CUDA error
// checks that turn into status codes (never abort), device buffers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/sbwt_b200.h"

namespace sbwt {

using u64 = uint64_t;
using u32 = uint32_t;
using u8 = uint8_t;

// Thrown inside the library, caught at the C-ABI boundary and mapped to a
// status code + sbwt_last_error() message.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string &msg);

#define SBWT_CUDA(call)                                                      \
  do {                                                                       \
    cudaError_t err__ = (call);                                              \
    if (err__ != cudaSuccess) {                                              \
      int code__ = (err__ == cudaErrorMemoryAllocation) ? SBWT_E_OOM         \
                                                        : SBWT_E_CUDA;       \
      throw ::sbwt::Error(code__, std::string(#call) + ": " +                \
                                      cudaGetErrorString(err__));            \
    }                                                                        \
  } while (0)

// Runs f() and maps exceptions to status codes.
template <class F>
int guarded(F &&f) {
  try {
    f();
    return SBWT_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc &) {
    set_last_error("host allocation failed");
    return SBWT_E_OOM;
  } catch (const std::exception &e) {
    std::string m = e.what();
    set_last_error(m);
    if (m.find("Unable to open") != std::string::npos) return SBWT_E_IO;
    return SBWT_E_FORMAT;
  }
}

// Owning device allocation (cudaMalloc / cudaFree) on the current device.
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t bytes) { resize(bytes); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  DeviceBuffer(DeviceBuffer &&o) noexcept : p_(o.p_), n_(o.n_) {
    o.p_ = nullptr;
    o.n_ = 0;
  }
  void resize(size_t bytes) {
    release();
    if (bytes) SBWT_CUDA(cudaMalloc(&p_, bytes));
    n_ = bytes;
  }
  // grows (never shrinks) keeping nothing
  void ensure(size_t bytes) {
    if (bytes > n_) resize(bytes + bytes / 8);
  }
  void release() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
  }
  template <class T = void>
  T *get() const {
    return static_cast<T *>(p_);
  }
  size_t size() const { return n_; }

 private:
  void *p_ = nullptr;
  size_t n_ = 0;
};

// Restores the caller's current device on scope exit.
class DeviceGuard {
 public:
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev_);
    if (dev != prev_) SBWT_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard() { cudaSetDevice(prev_); }

 private:
  int prev_ = 0;
};

inline bool is_host_pinned(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

}  // namespace sbwt
