// clast_indexfile.cu -- index persistence: every resident target window of a
// clast_targets in one file (clast_targets_save / clast_targets_load /
// clast_targets_verify).  The reference has no counterpart: it rebuilds every
// index for every query RAM load (main.cu:63-89).
//
// File layout (little-endian, version kIndexLayout):
//   "CLASTIX2"  int32 layout  int32 lmer  int32 stride  int32 cut_repeat
//   int32 n_loads  int64 n_windows
//   per window:  int32 load  int32 first  int32 t_begin  int32 nseqs
//                int64 n  uint32 nbuckets  int32 fshift  int64 n_records
//                int64 n_filter  int64 n_entries  int64 n_keys
//                bases[n + 2*kPad]  gateway[nseqs]  lengths[nseqs]
//                entries[n_entries] (int2)  table[n_records] (16 B)  filter[n_filter] (u32)
// A window is read into host memory and checked in full before anything of
// it reaches the device: every offset the kernels will follow (sequence
// starts and lengths, entry ranges of the table payloads, the free record
// that ends every probe) must lie inside its array.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/clast_gpu.h"
#include "clast_engine.h"

using namespace clast;

namespace {

constexpr char kIndexMagic[8] = {'C', 'L', 'A', 'S', 'T', 'I', 'X', '2'};
// Version of the table layout: 16-byte {code, payload} records, home record
// 2 * floor(code * nbuckets / 4^l), linear probing, kMulti payloads, a
// 65,536-record tail, 3-bit blocked filter words.  A file of another layout
// is rejected: its keys would be probed at the wrong records.
constexpr int32_t kIndexLayout = 2;
constexpr int64_t kTailRecords = 1 << 16;

struct FileCloser {
  FILE* f;
  ~FileCloser() {
    if (f) std::fclose(f);
  }
};

template <class T>
void put(FILE* f, const T& v) {
  if (std::fwrite(&v, sizeof(T), 1, f) != 1) throw std::runtime_error("index file write failed");
}
template <class T>
T get(FILE* f) {
  T v;
  if (std::fread(&v, sizeof(T), 1, f) != 1) throw std::invalid_argument("index file truncated");
  return v;
}

// Device array -> file, through a host bounce buffer.
template <class T>
void put_array(FILE* f, const T* dev, int64_t count, std::vector<char>& buf, cudaStream_t st) {
  const int64_t bytes = count * (int64_t)sizeof(T);
  for (int64_t off = 0; off < bytes; off += (int64_t)buf.size()) {
    const size_t len = (size_t)std::min<int64_t>((int64_t)buf.size(), bytes - off);
    CLAST_CK(cudaMemcpyAsync(buf.data(), reinterpret_cast<const char*>(dev) + off, len, cudaMemcpyDeviceToHost, st));
    CLAST_CK(cudaStreamSynchronize(st));
    if (std::fwrite(buf.data(), 1, len, f) != len) throw std::runtime_error("index file write failed");
  }
}

template <class T>
void get_host(FILE* f, std::vector<T>& v, int64_t count) {
  if (count < 0 || count > ((int64_t)1 << 36)) throw std::invalid_argument("index file holds a bad array size");
  v.resize((size_t)count);
  if (count && std::fread(v.data(), sizeof(T), (size_t)count, f) != (size_t)count)
    throw std::invalid_argument("index file truncated");
}

struct FileHeader {
  int32_t l = 0, stride = 0, cut = 0, n_loads = 0;
  int64_t n_wins = 0;
};

// One window as read from the file, checked.
struct HostWindow {
  int32_t load = 0, first = 0, t_begin = 0, nseqs = 0;
  int64_t n = 0, n_records = 0, n_keys = 0;
  uint32_t nbuckets = 0;
  int32_t fshift = 0;
  std::vector<char> bases;
  std::vector<int32_t> gateway, lengths;
  std::vector<int2> entries;
  std::vector<ulonglong2> table;
  std::vector<uint32_t> filter;
};

FileHeader read_header(FILE* f, const char* path, const clast_params* p) {
  char magic[sizeof(kIndexMagic)];
  if (std::fread(magic, 1, sizeof(magic), f) != sizeof(magic) || std::memcmp(magic, kIndexMagic, 7) != 0)
    throw std::invalid_argument(std::string(path) + " is not a clast index file");
  if (magic[7] != kIndexMagic[7]) throw std::invalid_argument(std::string(path) + " has an older index layout");
  const int32_t layout = get<int32_t>(f);
  if (layout != kIndexLayout)
    throw std::invalid_argument(std::string(path) + " has index layout " + std::to_string(layout) + ", not " +
                                std::to_string(kIndexLayout));
  FileHeader h;
  h.l = get<int32_t>(f);
  h.stride = get<int32_t>(f);
  h.cut = get<int32_t>(f);
  h.n_loads = get<int32_t>(f);
  h.n_wins = get<int64_t>(f);
  if (h.n_loads < 0 || h.n_wins < 0 || h.n_wins > (int64_t)1 << 24) throw std::invalid_argument("bad index file header");
  if (h.n_wins > 0 && (h.l != p->lmer || h.stride != p->stride || h.cut != p->cut_repeat))
    throw std::invalid_argument("the index was built with other lMer / stride / repeat settings");
  return h;
}

// Reads and checks one window.  Throws std::invalid_argument naming the first
// inconsistency; nothing of a rejected window is uploaded.
void read_window(FILE* f, const FileHeader& h, HostWindow& w) {
  auto bad = [](const std::string& what) { throw std::invalid_argument("bad index file window: " + what); };
  w.load = get<int32_t>(f);
  w.first = get<int32_t>(f);
  w.t_begin = get<int32_t>(f);
  w.nseqs = get<int32_t>(f);
  w.n = get<int64_t>(f);
  w.nbuckets = get<uint32_t>(f);
  w.fshift = get<int32_t>(f);
  w.n_records = get<int64_t>(f);
  const int64_t n_filter = get<int64_t>(f), n_entries = get<int64_t>(f);
  w.n_keys = get<int64_t>(f);
  if (w.load < 0 || w.load >= h.n_loads) bad("target load out of range");
  if (w.first < 0 || w.nseqs < 0) bad("negative record numbers");
  if (w.n < 0 || w.n >= INT32_MAX) bad("base count out of range");
  const int64_t ns = w.n / h.stride;
  if ((int64_t)w.nbuckets != std::max<int64_t>(1, ns)) bad("bucket count does not match the window size");
  if (w.n_records != 2 * (int64_t)w.nbuckets + kTailRecords) bad("record count does not match the bucket count");
  if (w.fshift < 32 || w.fshift > 63 || n_filter != ((int64_t)1 << (64 - w.fshift))) bad("filter size");
  if (n_entries < 0 || n_entries > ns) bad("entry count");
  if (w.n_keys != ns) bad("key count");
  get_host(f, w.bases, w.n + 2 * kPad);
  get_host(f, w.gateway, w.nseqs);
  get_host(f, w.lengths, w.nseqs);
  get_host(f, w.entries, n_entries);
  get_host(f, w.table, w.n_records);
  get_host(f, w.filter, n_filter);
  // sequences: start + length + joint inside the window, in order
  int64_t prev_end = 0;
  for (int32_t i = 0; i < w.nseqs; ++i) {
    const int64_t g = w.gateway[i], len = w.lengths[i];
    if (g < prev_end || len < 0 || g + len + (h.l - 1) > w.n) bad("sequence " + std::to_string(i) + " outside the window");
    prev_end = g + len;
  }
  // every probe ends at a free record inside the table: the last one is free
  if (w.table.back().y != kNoPayload) bad("last table record in use");
  for (int64_t r = 0; r < w.n_records; ++r) {
    const uint64_t pl = w.table[r].y;
    if (pl == kNoPayload) continue;
    if (pl & kMulti) {
      const int64_t start = (int64_t)((pl >> 32) & 0x7fffffffu), cnt = (int64_t)(uint32_t)pl;
      if (cnt < 1 || start + cnt > n_entries) bad("record " + std::to_string(r) + " points past the entries");
      // the entries a record refers to (the array's tail past the kept ones is unused)
      for (int64_t e = start; e < start + cnt; ++e) {
        const int2 x = w.entries[e];
        if (x.x < 0 || x.x >= w.nseqs || x.y < 0 || x.y >= w.lengths[x.x]) bad("entry " + std::to_string(e));
      }
    } else {
      const int64_t seq = (int64_t)(pl >> 32), idx = (int64_t)(uint32_t)pl;
      if (seq >= w.nseqs || idx >= w.lengths[seq]) bad("record " + std::to_string(r) + " names no target base");
    }
  }
}

}  // namespace

extern "C" int clast_targets_save(clast_ctx* ctx, const clast_targets* T, const char* path) {
  if (!ctx || !T || !path) return CLAST_ERR_ARG;
  return guarded(ctx, [&]() -> int {
    CLAST_CK(cudaSetDevice(ctx->device));
    settle_targets(ctx, T);
    FileCloser fc{std::fopen(path, "wb")};
    if (!fc.f) throw std::invalid_argument(std::string("cannot open ") + path + " for writing");
    FILE* f = fc.f;
    cudaStream_t st = ctx->st;
    std::vector<char> buf((size_t)64 << 20);
    if (std::fwrite(kIndexMagic, 1, sizeof(kIndexMagic), f) != sizeof(kIndexMagic))
      throw std::runtime_error("index file write failed");
    put<int32_t>(f, kIndexLayout);
    const clast_index* first = T->wins.empty() ? nullptr : T->wins[0].ix.get();
    put<int32_t>(f, first ? first->l : 0);
    put<int32_t>(f, first ? first->stride : 0);
    put<int32_t>(f, first ? first->cut : 0);
    put<int32_t>(f, T->n_loads);
    put<int64_t>(f, (int64_t)T->wins.size());
    for (const auto& w : T->wins) {
      const clast_index& ix = *w.ix;
      put<int32_t>(f, w.load);
      put<int32_t>(f, w.first);
      put<int32_t>(f, ix.t_begin);
      put<int32_t>(f, ix.nseqs);
      put<int64_t>(f, ix.n);
      put<uint32_t>(f, ix.nbuckets);
      put<int32_t>(f, ix.fshift);
      put<int64_t>(f, ix.n_records);
      put<int64_t>(f, (int64_t)ix.filter.n);
      put<int64_t>(f, (int64_t)ix.entries.n);
      put<int64_t>(f, ix.n_keys);
      put_array(f, ix.bases.p, ix.n + 2 * kPad, buf, st);
      put_array(f, ix.gateway.p, ix.nseqs, buf, st);
      put_array(f, ix.lengths.p, ix.nseqs, buf, st);
      put_array(f, ix.entries.p, (int64_t)ix.entries.n, buf, st);
      put_array(f, ix.table.p, ix.n_records, buf, st);
      put_array(f, ix.filter.p, (int64_t)ix.filter.n, buf, st);
    }
    if (std::fflush(f) != 0) throw std::runtime_error("index file write failed");
    return CLAST_OK;
  });
}

extern "C" int clast_targets_verify(const clast_params* p, const char* path, char* err, int err_len) {
  std::string msg;
  int rc = CLAST_OK;
  try {
    check_params(p);
    if (!path) throw std::invalid_argument("path is null");
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) throw std::invalid_argument(std::string("cannot open ") + path);
    const FileHeader h = read_header(fc.f, path, p);
    for (int64_t k = 0; k < h.n_wins; ++k) {
      HostWindow w;
      read_window(fc.f, h, w);
    }
    if (std::fgetc(fc.f) != EOF) throw std::invalid_argument("index file has bytes past its last window");
  } catch (const std::invalid_argument& e) {
    rc = CLAST_ERR_ARG;
    msg = e.what();
  } catch (const std::bad_alloc&) {
    rc = CLAST_ERR_NOMEM;
    msg = "out of memory";
  } catch (const std::exception& e) {
    rc = CLAST_ERR_INTERNAL;
    msg = e.what();
  }
  if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", msg.c_str());
  return rc;
}

extern "C" int clast_targets_load(clast_ctx* ctx, const clast_params* p, const char* path, clast_targets** out) {
  if (!ctx || !out || !path) return CLAST_ERR_ARG;
  *out = nullptr;
  return guarded(ctx, [&]() -> int {
    check_params(p);
    CLAST_CK(cudaSetDevice(ctx->device));
    g_alloc_stream = ctx->st;
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) throw std::invalid_argument(std::string("cannot open ") + path);
    FILE* f = fc.f;
    const FileHeader h = read_header(f, path, p);
    cudaStream_t st = ctx->st;
    std::unique_ptr<clast_targets> T(new clast_targets());
    T->ctx = ctx;
    T->n_loads = h.n_loads;
    HostWindow w;
    for (int64_t k = 0; k < h.n_wins; ++k) {
      read_window(f, h, w);  // checked in full before any upload
      clast_targets::Win win;
      win.load = w.load;
      win.first = w.first;
      std::unique_ptr<clast_index> ix(new clast_index());
      ix->l = h.l;
      ix->stride = h.stride;
      ix->cut = h.cut;
      ix->t_begin = w.t_begin;
      ix->nseqs = w.nseqs;
      ix->n = w.n;
      ix->nbuckets = w.nbuckets;
      ix->fshift = w.fshift;
      ix->n_records = w.n_records;
      ix->n_keys = w.n_keys;
      auto up = [&](auto& dev, const auto& host) {
        dev.alloc(host.size());
        if (!host.empty())
          CLAST_CK(cudaMemcpyAsync(dev.p, host.data(), host.size() * sizeof(host[0]), cudaMemcpyHostToDevice, st));
      };
      up(ix->bases, w.bases);
      up(ix->gateway, w.gateway);
      up(ix->lengths, w.lengths);
      up(ix->entries, w.entries);
      up(ix->table, w.table);
      up(ix->filter, w.filter);
      CLAST_CK(cudaStreamSynchronize(st));  // the host window is reused
      win.ix = std::move(ix);
      T->wins.push_back(std::move(win));
    }
    if (std::fgetc(f) != EOF) throw std::invalid_argument("index file has bytes past its last window");
    // records per load: every record of a load lies in one of its windows
    std::vector<int64_t> per_load((size_t)h.n_loads, 0);
    for (const auto& x : T->wins)
      per_load[x.load] = std::max<int64_t>(per_load[x.load], (int64_t)x.first + x.ix->nseqs);
    for (int32_t k = 0; k < h.n_loads; ++k) T->load_first.push_back(T->load_first.back() + per_load[k]);
    // nothing left to wait for: the targets are settled
    T->failed.alloc(1);
    CLAST_CK(cudaMemsetAsync(T->failed.p, 0, sizeof(unsigned long long), st));
    T->ev_start = ctx->timer.take();
    T->ev_up = ctx->timer.take();
    T->ev_done = ctx->timer.take();
    CLAST_CK(cudaEventRecord(T->ev_start, st));
    CLAST_CK(cudaEventRecord(T->ev_up, st));
    CLAST_CK(cudaEventRecord(T->ev_done, st));
    CLAST_CK(cudaStreamSynchronize(st));
    T->settled = true;
    *out = T.release();
    return CLAST_OK;
  });
}
