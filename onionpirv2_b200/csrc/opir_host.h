// Host-side helpers shared by the server handles: CUDA error translation,
// an owning device buffer and a current-device guard.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <new>
#include <stdexcept>
#include <string>

namespace opir {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { reset(); }
  void reset() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count <= n && p) return;
    reset();
    if (count == 0) return;
    if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      throw std::bad_alloc();
    }
    n = count;
  }
  void swap(DevBuf &o) {
    std::swap(p, o.p);
    std::swap(n, o.n);
  }
};

// Restores the caller's current device on scope exit.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) ck(cudaSetDevice(dev), "cudaSetDevice");
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace opir
