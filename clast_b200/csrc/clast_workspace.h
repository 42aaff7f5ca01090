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

  // Arena mode, used only by the allocation-free search entry point: every
  // request is carved out of one fixed block [arena, arena + arena_cap) and
  // nothing is ever allocated or freed; a request that does not fit throws
  // std::invalid_argument.  A name asked for again with a size that fits
  // gets its earlier slot back, as in pool mode.
  struct Slot {
    char name[32];
    size_t off, bytes;
  };
  static constexpr int kMaxSlots = 96;
  char* arena = nullptr;
  size_t arena_cap = 0, arena_used = 0;
  Slot slots[kMaxSlots];
  int n_slots = 0;

  void arena_begin(void* base, size_t cap) {
    arena = static_cast<char*>(base);
    arena_cap = cap;
    arena_used = 0;
    n_slots = 0;
  }
  // Drops every slot handed out at or after `mark` (an earlier arena_used).
  void arena_rewind(size_t mark) {
    while (n_slots > 0 && slots[n_slots - 1].off >= mark) --n_slots;
    arena_used = mark;
  }
  void* arena_get(const std::string& name, size_t bytes) {
    for (int i = n_slots - 1; i >= 0; --i)
      if (name == slots[i].name) {
        if (slots[i].bytes >= bytes) return arena + slots[i].off;
        break;
      }
    if (n_slots == kMaxSlots || name.size() >= sizeof(slots[0].name) || bytes > arena_cap - arena_used)
      throw std::invalid_argument("search scratch exhausted: buffer '" + name + "' needs " +
                                  std::to_string(bytes) + " bytes, " + std::to_string(arena_cap - arena_used) +
                                  " of " + std::to_string(arena_cap) + " left");
    Slot& s = slots[n_slots++];
    name.copy(s.name, sizeof(s.name) - 1);
    s.name[name.size()] = '\0';
    s.off = arena_used;
    s.bytes = bytes;
    arena_used += bytes;
    return arena + s.off;
  }

  template <class T>
  T* get(const std::string& name, size_t count) {
    size_t bytes = (count ? count : 1) * sizeof(T);
    bytes = (bytes + 255) & ~size_t(255);
    if (arena) return static_cast<T*>(arena_get(name, bytes));
    Buf& b = bufs[name];
    if (b.bytes < bytes) {
      if (b.p) CLAST_CK(cudaFree(b.p));
      b.p = nullptr;
      b.bytes = 0;
      const size_t nb = bytes + bytes / 4;
      if (cudaMalloc(&b.p, nb) != cudaSuccess) {
        // memory freed by stream-ordered frees stays cached in the device's
        // pool for later stream-ordered allocations; hand it back and retry
        (void)cudaGetLastError();
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
          cudaDeviceSynchronize();
          cudaMemPoolTrimTo(pool, 0);
        }
        (void)cudaGetLastError();
        if (cudaMalloc(&b.p, nb) != cudaSuccess) {
          (void)cudaGetLastError();
          b.p = nullptr;
          throw std::bad_alloc();
        }
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
