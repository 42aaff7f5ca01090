// clast_engine.h -- internal types shared by the host-side translation units of
// libclast_b200.so (engine, TSV formatting, serving loop): the context, the
// resident index of a target window, the resident targets, and the stream-
// ordered device arrays they are built from.  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <map>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/clast_gpu.h"
#include "clast_device.cuh"
#include "clast_kernels.cuh"
#include "clast_workspace.h"

namespace clast {

inline double wall_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Stream used for the stream-ordered allocations of the current API call.
extern thread_local cudaStream_t g_alloc_stream;

// Owning device allocation from the device's stream-ordered memory pool
// (cudaMallocAsync / cudaFreeAsync on the owning context's stream), so
// steady-state calls reuse pool memory instead of calling cudaMalloc.
template <class T>
struct DevArray {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t st = nullptr;
  DevArray() = default;
  DevArray(const DevArray&) = delete;
  DevArray& operator=(const DevArray&) = delete;
  DevArray(DevArray&& o) noexcept : p(o.p), n(o.n), st(o.st) { o.p = nullptr; o.n = 0; }
  DevArray& operator=(DevArray&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      st = o.st;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  void alloc(size_t count) {
    release();
    n = count;
    st = g_alloc_stream;
    if (cudaMallocAsync(reinterpret_cast<void**>(&p), (count ? count : 1) * sizeof(T), st) != cudaSuccess) {
      // blocks freed on other streams become reusable once their frees have
      // run: wait for the device, then try once more
      (void)cudaGetLastError();
      cudaDeviceSynchronize();
      (void)cudaGetLastError();
      if (cudaMallocAsync(reinterpret_cast<void**>(&p), (count ? count : 1) * sizeof(T), st) != cudaSuccess) {
        (void)cudaGetLastError();
        p = nullptr;
        n = 0;
        throw std::bad_alloc();
      }
    }
  }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    n = 0;
  }
  ~DevArray() { release(); }
};

inline void check_params(const clast_params* p) {
  if (!p) throw std::invalid_argument("params is null");
  if (p->lmer < 1 || p->lmer > 31) throw std::invalid_argument("lmer must be in 1..31");
  if (p->stride < 1) throw std::invalid_argument("stride must be >= 1");
  if (p->gap < 2 || p->gap > 16) throw std::invalid_argument("gap must be in 2..16");
}

// Device copy of a base array with kPad 'N' bytes on both sides.
inline void upload_padded(const char* host, int64_t n, DevArray<char>& dev, cudaStream_t st) {
  dev.alloc((size_t)n + 2 * kPad);
  CLAST_CK(cudaMemsetAsync(dev.p, 'N', (size_t)n + 2 * kPad, st));
  if (n > 0) CLAST_CK(cudaMemcpyAsync(dev.p + kPad, host, (size_t)n, cudaMemcpyHostToDevice, st));
}

// CUDA-event timing of device stages on one stream: begin()/end() bracket
// launches, flush() (after a stream synchronisation) adds up the intervals.
struct StageTimer {
  enum Stage { SEED = 0, DP = 1, SORT = 2, FINAL = 3, DPORDER = 4, N_STAGES = 5 };
  std::vector<cudaEvent_t> pool;
  struct Pending { int stage; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  double ms[N_STAGES] = {0, 0, 0, 0, 0};
  int64_t n[N_STAGES] = {0, 0, 0, 0, 0};
  cudaEvent_t cur_a = nullptr;

  cudaEvent_t take() {
    if (pool.empty()) {
      cudaEvent_t e;
      CLAST_CK(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  void begin(cudaStream_t st) {
    cur_a = take();
    CLAST_CK(cudaEventRecord(cur_a, st));
  }
  void end(int stage, cudaStream_t st, int launches = 1) {
    cudaEvent_t b = take();
    CLAST_CK(cudaEventRecord(b, st));
    pending.push_back({stage, cur_a, b});
    n[stage] += launches;
  }
  void flush() {
    for (auto& p : pending) {
      float t = 0;
      CLAST_CK(cudaEventElapsedTime(&t, p.a, p.b));
      ms[p.stage] += t;
      pool.push_back(p.a);
      pool.push_back(p.b);
    }
    pending.clear();
  }
  void reset() {
    flush();
    for (int i = 0; i < N_STAGES; ++i) { ms[i] = 0; n[i] = 0; }
  }
  ~StageTimer() {
    for (auto e : pool) cudaEventDestroy(e);
    for (auto& p : pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
  }
};

// Pinned host buffer that holds one clast_map result; reused once released.
struct PinnedArena {
  void* p = nullptr;
  size_t bytes = 0;
  std::atomic<bool> in_use{false};  // released by the result's owner, possibly on another thread
  // The result's arrays on the device, kept until the arena is reused (so the
  // text of a result can be formatted on the GPU): read strand t_load t_seq
  // t_idx q_idx t_len q_len match score, evalue, and the per-load offsets.
  struct Device {
    DevArray<int32_t> f[10];
    DevArray<double> evalue;
    DevArray<int64_t> load_offsets;
    int64_t n = 0;
    int32_t n_loads = 0;
  } dev;
};

// How the banded DP of one kind of batch runs (measured, see search_seeded):
// order 0 = none, 1 = exact sort by rows, 2 = length buckets; queue = the
// persistent grid with `chunk` hits per lane per take.
struct DpChoice {
  int order = 0;
  bool queue = false;
  int chunk = 1;
};
constexpr int64_t kDpTuneHits = 1 << 16;
constexpr int kBuildStreams = 2;  // target windows indexed at once by clast_targets_create

}  // namespace clast

struct clast_ctx {
  using StageTimer = clast::StageTimer;
  using PinnedArena = clast::PinnedArena;
  using Workspace = clast::Workspace;
  std::vector<std::unique_ptr<PinnedArena>> arenas;      // clast_map results
  std::vector<std::unique_ptr<PinnedArena>> tsv_arenas;  // clast_format_tsv texts
  int device = 0;
  cudaStream_t st = nullptr;
  cudaStream_t st_copy = nullptr;  // query uploads, overlapping index builds still running
  cudaStream_t st_build[clast::kBuildStreams] = {};  // index builds of clast_targets_create
  Workspace ws_build[clast::kBuildStreams];          // their scratch
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
  Workspace ws;
  std::string err;
  double last_ms = 0;
  int64_t last_launches = 0;
  clast_stats stats{};
  StageTimer timer;
  int64_t seed_hint = 0;  // seed buffer capacity that sufficed before
  std::map<int, clast::DpChoice> dp_tuned;  // by (gap, local, uneven)
  cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;  // DP tuning
  // the DP's one-hit-per-warp kernel runs on st_dp beside the one-per-thread
  // kernels on st (forked and joined by these events)
  cudaStream_t st_dp = nullptr;
  cudaEvent_t ev_dp_fork = nullptr, ev_dp_join = nullptr;
  // the DP's warp / thread split when CLAST_DP_WARP does not set it: a
  // server's lanes run every hit one per thread (under load, other lanes'
  // work shares the SMs, and one-per-warp hits lost more than they gained)
  int dp_warp = clast::kDpWarpAuto;
};

struct clast_index {
  int l = 0, stride = 0, cut = 0;
  int32_t t_begin = 0;
  int64_t n = 0;
  int32_t nseqs = 0;
  clast::DevArray<char> bases;  // padded
  clast::DevArray<int32_t> gateway, lengths;
  clast::DevArray<uint32_t> filter;     // blocked Bloom filter, 2^(64 - fshift) words
  clast::DevArray<ulonglong2> table;    // 2 * nbuckets records {key, payload}
  clast::DevArray<int2> entries;
  int64_t n_unique = 0, n_keys = 0, n_entries = 0;
  clast::DevArray<int64_t> kept;  // [0]: distinct keys kept after the repeat cut (written by the build)
  uint32_t nbuckets = 1;
  int64_t n_records = 2;
  int fshift = 63;

  clast::IndexView view() const {
    clast::IndexView v;
    v.l = l;
    v.fshift = fshift;
    v.filter = filter.p;
    v.table = table.p;
    v.nbuckets = nbuckets;
    v.n_records = n_records;
    v.entries = entries.p;
    v.n_keys = n_keys;
    return v;
  }
  clast::TargetView tview() const {
    clast::TargetView t;
    t.bases = bases.p + clast::kPad;
    t.n = n;
    t.gateway = gateway.p;
    t.lengths = lengths.p;
    t.nseqs = nseqs;
    return t;
  }
};

struct clast_targets {
  clast_ctx* ctx = nullptr;
  struct Win {
    int32_t load, first;  // target load, first record within the load
    std::unique_ptr<clast_index> ix;
  };
  std::vector<Win> wins;
  int32_t n_loads = 0;
  std::vector<int64_t> load_first{0};  // first target record of every load, plus the total
  // The index builds run on the context's stream after clast_targets_create
  // returns; the first clast_map waits for them, reads the overflow count and
  // the build time (events) and reports either.
  clast::DevArray<unsigned long long> failed;
  cudaEvent_t ev_start = nullptr, ev_up = nullptr, ev_done = nullptr;  // from the context's event pool
  mutable bool settled = false;
  int64_t launches = 0;
  ~clast_targets() {
    if (ev_done) cudaEventSynchronize(ev_done);
    for (cudaEvent_t e : {ev_start, ev_up, ev_done})
      if (e) ctx->timer.pool.push_back(e);
  }
};

namespace clast {

// Waits for the index builds of clast_targets_create (once), records their
// time in the context's stats and reports a table overflow.
void settle_targets(clast_ctx* ctx, const clast_targets* T);

inline int fail(clast_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

// Runs f() and turns every exception into a status code plus message.
template <class F>
int guarded(clast_ctx* ctx, F&& f) {
  try {
    return f();
  } catch (const CudaError& e) {
    return fail(ctx, CLAST_ERR_CUDA, e.what());
  } catch (const std::bad_alloc&) {
    return fail(ctx, CLAST_ERR_NOMEM, "out of memory");
  } catch (const std::invalid_argument& e) {
    return fail(ctx, CLAST_ERR_ARG, e.what());
  } catch (const std::exception& e) {
    return fail(ctx, CLAST_ERR_INTERNAL, e.what());
  }
}

}  // namespace clast
