// clast_workspace.h -- error type and the per-context device scratch pool.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>

namespace clast {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CLAST_CK(x)                                                                          \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess)                                                                   \
      throw ::clast::CudaError(e_, std::string(#x) + ": " + cudaGetErrorString(e_) + " (" + \
                                       __FILE__ + ":" + std::to_string(__LINE__) + ")");    \
  } while (0)

// Kernels launched by this thread since the counter was last reset.
extern thread_local int64_t g_kernel_launches;

#define CLAST_LAUNCHED()          \
  do {                            \
    ++::clast::g_kernel_launches; \
    CLAST_CK(cudaGetLastError()); \
  } while (0)

// Named device buffers that grow on demand and are reused across calls, so
// steady-state calls allocate nothing.
struct Workspace {
  struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
  };
  std::map<std::string, Buf> bufs;

  template <class T>
  T* get(const std::string& name, size_t count) {
    size_t bytes = (count ? count : 1) * sizeof(T);
    bytes = (bytes + 255) & ~size_t(255);
    Buf& b = bufs[name];
    if (b.bytes < bytes) {
      if (b.p) CLAST_CK(cudaFree(b.p));
      b.p = nullptr;
      b.bytes = 0;
      const size_t nb = bytes + bytes / 4;
      if (cudaMalloc(&b.p, nb) != cudaSuccess) {
        (void)cudaGetLastError();
        b.p = nullptr;
        throw std::bad_alloc();
      }
      b.bytes = nb;
    }
    return static_cast<T*>(b.p);
  }

  void release_all() {
    for (auto& kv : bufs)
      if (kv.second.p) cudaFree(kv.second.p);
    bufs.clear();
  }
  ~Workspace() { release_all(); }
};

}  // namespace clast
