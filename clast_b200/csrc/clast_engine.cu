// clast_engine.cu -- host orchestration of the device path and the C ABI
// declared in include/clast_gpu.h.
//
// One context owns one CUDA stream and a scratch pool.  An index keeps its
// target window resident in HBM (bases with joints, padded with 'N', plus the
// key directory, unique keys, bucket ranges and resolved entries).  A search
// runs the whole hit pipeline of CDeviceHitList (CDeviceHitList.cu:228-423)
// for a batch of query windows with three host synchronisations (seed total,
// hit total, result total).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/clast_gpu.h"
#include "clast_device.cuh"
#include "clast_kernels.cuh"
#include "clast_workspace.h"
#include "clast_engine.h"

using namespace clast;

namespace clast {
thread_local cudaStream_t g_alloc_stream = nullptr;
}  // namespace clast





namespace {

template <class T>
T read_scalar(const T* dev, cudaStream_t st) {
  T v;
  CLAST_CK(cudaMemcpyAsync(&v, dev, sizeof(T), cudaMemcpyDeviceToHost, st));
  CLAST_CK(cudaStreamSynchronize(st));
  return v;
}

}  // namespace


namespace {

// CDeviceHashTable::CDeviceHashTable (CDeviceHashTable.cu:143-174) for the
// window whose padded bases are already in ix->bases.
// *failed (zeroed by the caller, read once all windows are queued) counts
// table records that fell outside the table.
void build_index_device(Workspace& ws, cudaStream_t st, const clast_params* p, clast_index* ix,
                        unsigned long long* failed) {
  const int l = p->lmer;
  const int64_t n = ix->n;
  const char* bases = ix->bases.p + kPad;
  uint64_t* packed = ws.get<uint64_t>("ix_packed", (size_t)(n / 32 + 4));
  uint64_t* nmask = ws.get<uint64_t>("ix_nmask", (size_t)(n / 64 + 4));
  pack_bases(bases, n, packed, nmask, st);
  const int64_t ns = n / p->stride;  // CDeviceHashTable.cu:34
  // samples sorted by code (equal keys adjacent, in window-position order):
  // one word code << pbits | position when both fit in 64 bits, else
  // (code, position) pairs
  int pbits = 1;
  while ((1ll << pbits) < ns) ++pbits;
  if (2 * l + 1 + pbits > 64) pbits = 0;
  uint64_t* items = ws.get<uint64_t>("ix_items", ns);
  uint64_t* items2 = ws.get<uint64_t>("ix_items2", ns);
  int32_t* pos = pbits ? nullptr : ws.get<int32_t>("ix_pos", ns);
  int32_t* pos2 = pbits ? nullptr : ws.get<int32_t>("ix_pos2", ns);
  sample_keys(packed, nmask, ns, p->stride, l, pbits, items, pos, st);
  const int in_alt = radix_sort_u64(ws, items, pos, items2, pos2, ns, pbits, pbits + 2 * l + 1, st);
  // key heads (first sample of every valid code) come with the split
  const uint64_t bound = 1ull << (2 * l);  // the code of l-mers with a non-ACGT base
  uint64_t* keys;
  int32_t* vals;
  int32_t* head = ws.get<int32_t>("ix_head", ns);
  if (pbits) {
    keys = ws.get<uint64_t>("ix_keys", ns);
    vals = ws.get<int32_t>("ix_vals", ns);
    split_items(in_alt ? items2 : items, ns, pbits, bound, keys, vals, head, st);
  } else {
    keys = in_alt ? items2 : items;
    vals = in_alt ? pos2 : pos;
    index_heads(keys, ns, bound, head, st);
  }
  // From here on no host synchronisation: every array is sized for the ns
  // samples (an upper bound of the valid samples nv, the unique keys nu and
  // the entries); nv = *nv_dev and nu = hpos[ns] stay on the device.
  int64_t* nv_dev = ws.get<int64_t>("ix_nv", 1);
  if (ns > 0) count_below(keys, ns, bound, nv_dev, st);
  else CLAST_CK(cudaMemsetAsync(nv_dev, 0, sizeof(int64_t), st));
  int64_t* hpos = ws.get<int64_t>("ix_hpos", ns + 1);
  scan_i32(ws, head, ns, hpos, st);
  const int64_t* nu_dev = hpos + ns;
  uint64_t* ukeys = ws.get<uint64_t>("ix_ukeys", ns);
  int64_t* ufirst = ws.get<int64_t>("ix_ufirst", ns + 1);
  index_unique(keys, head, hpos, ns, nv_dev, ukeys, ufirst, st);
  int32_t* keep = ws.get<int32_t>("ix_keep", ns);
  int2* resolved = ws.get<int2>("ix_resolved", ns);
  int64_t* kpos = ws.get<int64_t>("ix_kpos", ns + 1);
  index_keep(vals, hpos, ufirst, ns, nv_dev, p->stride, l, p->cut_repeat, ix->gateway.p, ix->lengths.p, ix->nseqs,
             keep, resolved, st);
  scan_i32(ws, keep, ns, kpos, st);
  ix->entries.alloc(ns);
  index_entries(keep, kpos, resolved, ns, ix->entries.p, st);
  int32_t* ustart = ws.get<int32_t>("ix_ustart", ns);
  int32_t* ucnt = ws.get<int32_t>("ix_ucnt", ns);
  index_buckets(ufirst, kpos, ns, nu_dev, ustart, ucnt, st);
  // Hash table: buckets of two records, one bucket per sample, so at most half
  // of the records are used (84 % of the keys then sit in their home bucket),
  // plus a tail for the probe run past the last bucket
  const int64_t nb = std::max<int64_t>(1, ns);
  if (nb >= (int64_t)UINT32_MAX) throw std::invalid_argument("window has too many sampled l-mers");
  ix->nbuckets = (uint32_t)nb;
  int64_t* rank = ws.get<int64_t>("ix_rank", ns + 1);
  scan_positive(ws, ucnt, ns, rank, st);
  ix->kept.alloc(1);
  CLAST_CK(cudaMemcpyAsync(ix->kept.p, rank + ns, sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
  int64_t* run_max = ws.get<int64_t>("ix_runmax", ns);
  table_runmax(ws, ukeys, ucnt, rank, ns, l, ix->nbuckets, run_max, st);
  ix->n_records = 2 * nb + (1 << 16);
  ix->table.alloc((size_t)ix->n_records);
  CLAST_CK(cudaMemsetAsync(ix->table.p, 0xff, (size_t)ix->n_records * sizeof(ulonglong2), st));
  // Bloom filter: about 24 bits per sample, between 2^12 and 2^F bits; F = 27
  // (16 MB: the filters of the two windows a seeding pass reads stay in L2
  // beside the streams that pass through it) unless CLAST_FILTER_BITS says
  // otherwise (16..32)
  int fbits = 27;
  if (const char* e = std::getenv("CLAST_FILTER_BITS")) fbits = std::max(16, std::min(32, std::atoi(e)));
  int bits = 12;
  while (bits < fbits && (1ll << bits) < ns * 24) ++bits;
  ix->fshift = 64 - (bits - 5);
  ix->filter.alloc((size_t)1 << (bits - 5));
  CLAST_CK(cudaMemsetAsync(ix->filter.p, 0, ((size_t)1 << (bits - 5)) * sizeof(uint32_t), st));
  table_place(ukeys, ustart, ucnt, ix->entries.p, rank, run_max, ns, ix->table.p, ix->n_records, ix->filter.p,
              ix->fshift, failed, st);
  ix->n_keys = ns;
}

// Index of a window whose padded base array is already on the device.
clast_index* make_index_resident(Workspace& ws, cudaStream_t st, const clast_params* p, DevArray<char>&& padded,
                                 int64_t n_bases, DevArray<int32_t>&& gateway, DevArray<int32_t>&& lengths,
                                 int32_t n_seqs, int32_t t_begin, unsigned long long* failed) {
  std::unique_ptr<clast_index> ix(new clast_index());
  ix->l = p->lmer;
  ix->stride = p->stride;
  ix->cut = p->cut_repeat;
  ix->t_begin = t_begin;
  ix->n = n_bases;
  ix->nseqs = n_seqs;
  ix->bases = std::move(padded);
  ix->gateway = std::move(gateway);
  ix->lengths = std::move(lengths);
  build_index_device(ws, st, p, ix.get(), failed);
  return ix.release();
}

// Index of a window given as host arrays (the reference's seam).
clast_index* make_index(clast_ctx* c, const clast_params* p, const char* bases, int64_t n_bases,
                        const int32_t* gateway, const int32_t* lengths, int32_t n_seqs, int32_t t_begin) {
  DevArray<char> padded;
  DevArray<int32_t> gw, ln;
  gw.alloc(n_seqs);
  ln.alloc(n_seqs);
  padded.alloc((size_t)n_bases + 2 * kPad);
  CLAST_CK(cudaEventRecord(c->ev0, c->st));
  CLAST_CK(cudaMemsetAsync(padded.p, 'N', (size_t)n_bases + 2 * kPad, c->st));
  if (n_bases > 0) CLAST_CK(cudaMemcpyAsync(padded.p + kPad, bases, (size_t)n_bases, cudaMemcpyHostToDevice, c->st));
  if (n_seqs > 0) {
    CLAST_CK(cudaMemcpyAsync(gw.p, gateway, n_seqs * sizeof(int32_t), cudaMemcpyHostToDevice, c->st));
    CLAST_CK(cudaMemcpyAsync(ln.p, lengths, n_seqs * sizeof(int32_t), cudaMemcpyHostToDevice, c->st));
  }
  CLAST_CK(cudaEventRecord(c->ev1, c->st));
  const int64_t k0 = g_kernel_launches;
  unsigned long long* failed = reinterpret_cast<unsigned long long*>(c->ws.get<int64_t>("ix_failed", 1));
  CLAST_CK(cudaMemsetAsync(failed, 0, sizeof(unsigned long long), c->st));
  std::unique_ptr<clast_index> ix(make_index_resident(c->ws, c->st, p, std::move(padded), n_bases, std::move(gw),
                                                      std::move(ln),
                                                      n_seqs, t_begin, failed));
  CLAST_CK(cudaEventRecord(c->ev2, c->st));
  CLAST_CK(cudaEventSynchronize(c->ev2));
  if (read_scalar(reinterpret_cast<int64_t*>(failed), c->st) != 0) throw std::runtime_error("index table overflow");
  float up = 0, bd = 0;
  CLAST_CK(cudaEventElapsedTime(&up, c->ev0, c->ev1));
  CLAST_CK(cudaEventElapsedTime(&bd, c->ev1, c->ev2));
  c->stats.index_upload_ms += up;
  c->stats.index_ms += bd;
  c->stats.index_launches += g_kernel_launches - k0;
  return ix.release();
}

// Device-resident query strands of one batch, packed once for every index.
struct QueryRef;

struct QueryBatch {
  DevArray<char> bases;  // padded
  int64_t n = 0;
  DevArray<int64_t> start;
  DevArray<int32_t> len;
  DevArray<uint64_t> packed, nmask;
  int32_t nstrands = 0;
  DevArray<int32_t> wstart;  // strand index where each window starts, plus the end
  int32_t nwin = 0;
  int32_t min_len = 0, max_len = 0;  // strand lengths (the DP orders hits by rows when they differ)
  QueryView view() const {
    QueryView q;
    q.bases = bases.p + kPad;
    q.n = n;
    q.packed = packed.p;
    q.nmask = nmask.p;
    q.start = start.p;
    q.len = len.p;
    q.nstrands = nstrands;
    return q;
  }
  void pack(cudaStream_t st) {
    packed.alloc((size_t)(n / 32 + 4));
    nmask.alloc((size_t)(n / 64 + 4));
    pack_bases(bases.p + kPad, n, packed.p, nmask.p, st);
  }
  QueryRef ref() const;
};

// A query batch as the seeding and search stages read it, without ownership
// (a QueryBatch, or clast_search_noalloc's buffers in its fixed scratch).
struct QueryRef {
  QueryView q;
  int64_t n = 0;                     // bases of the strands
  const int32_t* wstart = nullptr;   // strand where each query window starts, plus the end
  int32_t nwin = 0;
  int32_t min_len = 0, max_len = 0;  // strand lengths (the DP orders hits by rows when they differ)
};

QueryRef QueryBatch::ref() const {
  QueryRef r;
  r.q = view();
  r.n = n;
  r.wstart = wstart.p;
  r.nwin = nwin;
  r.min_len = min_len;
  r.max_len = max_len;
  return r;
}

// Host copy of one batch's result (reference order within each query window).
// One batch's hits on the device, reads ascending (reference order within
// every query window), with per-read offsets.
struct DevHits {
  int64_t n = 0;
  DevArray<int32_t> t_id, t_idx, q_id, q_idx, t_len, q_len, match, score;
  DevArray<double> evalue;
  DevArray<int64_t> foff;
};

// Seeds of one target window for a query batch (createRawSeedList +
// deleteSeedsOnSequenceBoundary), in the workspace slots of `slot`.
struct SeedSet {
  const clast_index* ix = nullptr;
  int64_t* off = nullptr;
  int32_t* len32 = nullptr;
  int32_t* nvalid = nullptr;
  unsigned long long* counters = nullptr;  // [1] DP cells, then seed_parts() cursors and l-mer counters
  uint64_t* skey = nullptr;
  uint32_t* sq = nullptr;
  int64_t part_cap = 0;
  int64_t S = 0;
};

// Seeds of up to kMaxSeedWins windows (all of `sets`) in one pass over the
// query: the 2-bit words are read once and every l-mer's lookups in all the
// windows are issued together.  A window whose seed partition overflowed is
// seeded again (alone with the others that overflowed) with partitions sized
// from the exact counts.
void seed_windows(clast_ctx* c, const clast_params* p, const QueryRef& qb, std::vector<SeedSet>& sets) {
  cudaStream_t st = c->st;
  Workspace& ws = c->ws;
  const QueryView q = qb.q;
  const int64_t ns = q.nstrands;
  const int parts = seed_parts();
  StageTimer& tm = c->timer;
  std::vector<int> todo;
  for (size_t k = 0; k < sets.size(); ++k) {
    SeedSet& z = sets[k];
    const std::string tag = "#" + std::to_string(k);
    z.off = ws.get<int64_t>("s_off" + tag, ns + 1);
    z.len32 = ws.get<int32_t>("s_len32" + tag, ns);
    z.nvalid = ws.get<int32_t>("s_nvalid" + tag, ns);
    z.counters = ws.get<unsigned long long>("s_counters" + tag, 2 + 2 * parts);
    z.part_cap = std::max<int64_t>(c->seed_hint, qb.n / 16 + (1 << 20)) / parts + 1;
    todo.push_back((int)k);
  }
  for (int attempt = 0; attempt < 2 && !todo.empty(); ++attempt) {
    SeedWins W{};
    for (size_t j = 0; j < todo.size(); ++j) {
      SeedSet& z = sets[todo[j]];
      const std::string tag = "#" + std::to_string(todo[j]);
      z.skey = ws.get<uint64_t>("s_key" + tag, (size_t)z.part_cap * parts);
      z.sq = ws.get<uint32_t>("s_q" + tag, (size_t)z.part_cap * parts);
      CLAST_CK(cudaMemsetAsync(z.counters, 0, (2 + 2 * parts) * sizeof(unsigned long long), st));
      W.w[j] = SeedWin{z.ix->view(), z.ix->tview(), z.counters + 2, z.counters + 2 + parts, z.off, z.len32,
                       z.nvalid, z.skey, z.sq, z.part_cap};
    }
    tm.begin(st);
    static const bool force_multi = std::getenv("CLAST_SEED_MULTI_ONLY") != nullptr;
    if (todo.size() == 1 && !force_multi) {  // one window: the single-window kernel (round 0 staged while its range is reserved)
      const SeedWin& w = W.w[0];
      seed_fused(q, w.ix, w.t, p->gap, p->local, w.cursor, w.n_kmers, w.off, w.cnt, w.nvalid, w.skey, w.sq,
                 w.part_cap, st);
    } else {
      seed_multi(q, W, (int)todo.size(), p->gap, p->local, st);
    }
    tm.end(StageTimer::SEED, st);
    std::vector<unsigned long long> cur(todo.size() * 2 * parts);
    for (size_t j = 0; j < todo.size(); ++j)
      CLAST_CK(cudaMemcpyAsync(cur.data() + j * 2 * parts, sets[todo[j]].counters + 2,
                               2 * parts * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CLAST_CK(cudaStreamSynchronize(st));
    std::vector<int> again;
    for (size_t j = 0; j < todo.size(); ++j) {
      SeedSet& z = sets[todo[j]];
      const unsigned long long* cj = cur.data() + j * 2 * parts;
      int64_t S = 0, most = 0, kmers = 0;
      for (int i = 0; i < parts; ++i) {
        S += (int64_t)cj[i];
        most = std::max<int64_t>(most, (int64_t)cj[i]);
        kmers += (int64_t)cj[parts + i];
      }
      z.S = S;
      if (most <= z.part_cap) {
        c->stats.query_kmers += kmers;
        c->seed_hint = std::max<int64_t>(c->seed_hint, S + S / 4);
      } else {
        z.part_cap = most;  // strands past a full partition wrote nothing: run again
        again.push_back(todo[j]);
      }
    }
    todo.swap(again);
  }
  if (!todo.empty()) throw std::runtime_error("seed partitions overflowed twice");
}

// Where search_seeded puts a window's final hits: take(F, foff, nr) returns
// the arrays for its F hits (and may keep the nr + 1 per-read offsets), or
// throws when they do not fit.
struct HitSink {
  virtual ~HitSink() = default;
  virtual FinalOut take(int64_t F, const int64_t* foff, int64_t nr, cudaStream_t st) = 0;
};

// Device arrays of their own, with the per-read offsets (clast_search,
// clast_map).
struct DevHitsSink : HitSink {
  DevHits& out;
  explicit DevHitsSink(DevHits& o) : out(o) { out = DevHits(); }
  FinalOut take(int64_t F, const int64_t* foff, int64_t nr, cudaStream_t st) override {
    out.n = F;
    out.t_id.alloc(F); out.t_idx.alloc(F); out.q_id.alloc(F); out.q_idx.alloc(F); out.t_len.alloc(F);
    out.q_len.alloc(F); out.match.alloc(F); out.score.alloc(F); out.evalue.alloc(F);
    out.foff.alloc(nr + 1);
    CLAST_CK(cudaMemcpyAsync(out.foff.p, foff, (nr + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
    return FinalOut{out.t_id.p, out.t_idx.p, out.q_id.p, out.q_idx.p, out.t_len.p, out.q_len.p, out.match.p,
                    out.score.p, out.evalue.p};
  }
};

// CDeviceHitList for every query window of `qb` against the window whose
// seeds are in z: seed filters, DP, result order.
int64_t search_seeded(clast_ctx* c, Workspace& ws, const clast_params* p, const QueryRef& qb, int32_t q_first,
                      SeedSet& z, bool tune, HitSink& sink) {
  cudaStream_t st = c->st;
  const clast_index* ix = z.ix;
  const QueryView q = qb.q;
  const TargetView tv = ix->tview();
  const int64_t ns = q.nstrands, nr = ns / 2;
  StageTimer& tm = c->timer;
  const int64_t S = z.S;
  int64_t* off = z.off;
  int32_t* len32 = z.len32;
  int32_t* nvalid = z.nvalid;
  unsigned long long* counters = z.counters;
  uint64_t* skey = z.skey;
  uint32_t* sq = z.sq;
  const long long* warp_dev = nullptr;  // the DP's split, when it was made on the device
  const int* bad_dev = nullptr;         // the DP's flag of hits outside the window, once it ran
  auto add_counters = [&]() {
    unsigned long long cells = 0;
    long long warp = 0;
    int bad = 0;
    CLAST_CK(cudaMemcpyAsync(&cells, counters + 1, sizeof(cells), cudaMemcpyDeviceToHost, st));
    if (warp_dev) CLAST_CK(cudaMemcpyAsync(&warp, warp_dev, sizeof(warp), cudaMemcpyDeviceToHost, st));
    if (bad_dev) CLAST_CK(cudaMemcpyAsync(&bad, bad_dev, sizeof(bad), cudaMemcpyDeviceToHost, st));
    CLAST_CK(cudaStreamSynchronize(st));
    c->stats.dp_cells += (int64_t)cells;
    c->stats.dp_warp_hits += warp;
    tm.flush();
    if (bad) throw std::runtime_error("internal: a hit named a target sequence or strand outside the window");
  };
  c->stats.seeds += S;
  if (S == 0) {
    add_counters();
    return 0;
  }
  int32_t* wfirst = ws.get<int32_t>("s_wfirst", qb.nwin);
  window_first(nvalid, qb.wstart, qb.nwin, wfirst, st);
  // sortSeeds, deletingIsolateSeeds, deleteDuplicateSeeds
  tm.begin(st);
  int32_t* hcnt = ws.get<int32_t>("s_hcnt", ns);
  seed_sort_filter(ws, skey, sq, off, len32, nvalid, qb.wstart, qb.nwin, wfirst, p->width, p->gap, ns, hcnt, st);
  tm.end(StageTimer::SORT, st, 4);
  int64_t* hoff = ws.get<int64_t>("s_hoff", ns + 1);
  scan_i32(ws, hcnt, ns, hoff, st);
  const int64_t H = read_scalar(hoff + ns, st);
  if (H >= ((int64_t)1 << 32)) throw std::invalid_argument("more than 2^32 hits in one window");  // DP order words
  c->stats.hits += H;
  if (H == 0) {
    add_counters();
    return 0;
  }
  uint64_t* hk = ws.get<uint64_t>("h_key", H);
  int32_t* hq = ws.get<int32_t>("h_q", H);
  int32_t* hs = ws.get<int32_t>("h_s", H);
  gather_hits(skey, sq, off, hcnt, hoff, ns, hk, hq, hs, q.len, p->lmer, 2 * p->gap + 1, counters + 1, st);
  // alignmentHits + calculateEvalue + deleteHits_lowEValue / _tooShort
  DpOut o;
  o.t_idx = ws.get<int32_t>("d_tidx", H);
  o.q_idx = ws.get<int32_t>("d_qidx", H);
  o.t_len = ws.get<int32_t>("d_tlen", H);
  o.q_len = ws.get<int32_t>("d_qlen", H);
  o.match = ws.get<int32_t>("d_match", H);
  o.score = ws.get<int32_t>("d_score", H);
  o.evalue = ws.get<double>("d_e", H);
  o.keep = ws.get<uint8_t>("d_keep", H);
  DpParams dp{p->lmer, p->stride, p->gap, p->local, p->cutoff, p->total_db, p->K, p->lambda};
  // Reads of different lengths: the DP takes the hits longest first, so that a
  // warp's hits have about the same number of rows (the reference sorts them
  // by rows before aligning too, CDeviceHitList_alignmentHits.cu:10-58), by
  // an exact sort or by length buckets; the kernel runs over a grid of all
  // hits or as a persistent grid taking hits from a queue.  Which of these
  // runs fastest is measured once per context and kind of batch (gap, mode,
  // uneven or not) on a batch of at least kDpTuneHits hits; every variant
  // writes the same results.
  // The longest hits of the order may run one per warp (banded_dp decides
  // from the length buckets, or for equal lengths from the row count).
  const bool uneven = qb.max_len != qb.min_len && H > 1;
  const int warp_mode = dp_warp_mode_from_env(c->dp_warp);
  DpBuckets buckets;  // of the order last made
  auto make_order = [&](int kind) -> const uint64_t* {
    buckets = DpBuckets();
    if (kind == 0) return nullptr;
    if (kind == 1) {
      const int rows_max = std::max(1, qb.max_len - p->lmer + 1);
      int bits = 1;
      while ((1ll << bits) <= rows_max) ++bits;
      uint64_t* ok = ws.get<uint64_t>("h_order", H);
      uint64_t* ok2 = ws.get<uint64_t>("h_order2", H);
      dp_order_keys(hs, q.len, H, p->lmer, rows_max, ok, st);
      const uint64_t* sorted = radix_sort_u64(ws, ok, nullptr, ok2, nullptr, H, 32, 32 + bits, st) ? ok2 : ok;
      if (warp_mode == kDpWarpAuto) buckets = dp_bucket_count(ws, hs, q.len, H, p->lmer, st);
      return sorted;
    }
    uint64_t* ob = ws.get<uint64_t>("h_border", H);
    buckets = dp_bucket_order(ws, hs, q.len, H, p->lmer, ob, st);
    return ob;
  };
  unsigned long long* dp_head = ws.get<unsigned long long>("dp_head", 1);
  long long* dp_warp_n = ws.get<long long>("dp_warp_n", 1);
  int* dp_bad = ws.get<int>("dp_bad", 1);
  CLAST_CK(cudaMemsetAsync(dp_bad, 0, sizeof(int), st));
  auto launch_of = [&](const DpChoice& ch) {
    DpLaunch m;
    if (ch.queue) {
      m.head = dp_head;
      m.chunk = ch.chunk;
    }
    m.warp = warp_mode;
    m.buckets = buckets;
    m.warp_n = dp_warp_n;
    m.aux = c->st_dp;
    m.ev_fork = c->ev_dp_fork;
    m.ev_join = c->ev_dp_join;
    m.bad = dp_bad;
    if (!uneven) m.uniform_rows = std::max(0, qb.max_len - p->lmer);
    return m;
  };
  const int tune_key = (p->gap << 2) | (p->local ? 2 : 0) | (uneven ? 1 : 0);
  auto it = c->dp_tuned.find(tune_key);
  if (tune && it == c->dp_tuned.end() && H >= kDpTuneHits && !std::getenv("CLAST_DP_NO_TUNE")) {
    std::vector<DpChoice> cands;
    for (int ord : (uneven ? std::vector<int>{1, 2} : std::vector<int>{0}))
      for (int q_ : {0, 1})
        for (int chunk : (q_ ? std::vector<int>{1, 2} : std::vector<int>{1})) cands.push_back(DpChoice{ord, q_ != 0, chunk});
    float best = 1e30f;
    DpChoice pick = cands[0];
    for (const DpChoice& ch : cands) {
      CLAST_CK(cudaEventRecord(c->ev_t0, st));
      const uint64_t* order = make_order(ch.order);
      banded_dp(tv, q, hk, hq, hs, order, H, dp, o, st, launch_of(ch));
      CLAST_CK(cudaEventRecord(c->ev_t1, st));
      CLAST_CK(cudaEventSynchronize(c->ev_t1));
      float ms = 0;
      CLAST_CK(cudaEventElapsedTime(&ms, c->ev_t0, c->ev_t1));
      if (ms < best) {
        best = ms;
        pick = ch;
      }
    }
    it = c->dp_tuned.emplace(tune_key, pick).first;
  }
  DpChoice ch = it != c->dp_tuned.end() ? it->second : DpChoice{uneven ? 1 : 0, false, 1};
  if (ch.order != 0 && !uneven) ch.order = 0;
  c->stats.dp_order_kind = ch.order;
  c->stats.dp_queue_chunk = ch.queue ? ch.chunk : 0;
  tm.begin(st);
  const uint64_t* order = make_order(ch.order);
  tm.end(StageTimer::DPORDER, st);
  tm.begin(st);
  const DpLaunch dl = launch_of(ch);
  const long long warp_fixed = banded_dp(tv, q, hk, hq, hs, order, H, dp, o, st, dl);
  tm.end(StageTimer::DP, st);
  if (warp_fixed >= 0) c->stats.dp_warp_hits += warp_fixed;
  else warp_dev = dl.warp_n;
  bad_dev = dp_bad;
  // resultSorting + deleteHits_duplicateResult, per read
  uint64_t* k1 = ws.get<uint64_t>("f_k1", H);
  uint64_t* k2 = ws.get<uint64_t>("f_k2", H);
  int32_t* idx = ws.get<int32_t>("f_idx", H);
  final_keys(hk, hq, hs, o, H, k1, k2, idx, st);
  tm.begin(st);
  int64_t* roff = ws.get<int64_t>("f_roff", nr);
  int32_t* rlen = ws.get<int32_t>("f_rlen", nr);
  read_ranges(hoff, nr, roff, rlen, st);
  segmented_sort_u64(ws, k1, k2, idx, roff, rlen, nr, st, 1);
  int32_t* fcnt = ws.get<int32_t>("f_cnt", nr);
  int32_t* fsel = ws.get<int32_t>("f_sel", H);
  final_dedupe(k1, k2, idx, hk, hs, o, roff, rlen, nr, fcnt, fsel, st);
  int64_t* foff = ws.get<int64_t>("f_off", nr + 1);
  scan_i32(ws, fcnt, nr, foff, st);
  tm.end(StageTimer::FINAL, st, 9);
  const int64_t F = read_scalar(foff + nr, st);
  c->stats.results += F;
  add_counters();
  if (F == 0) return 0;
  const FinalOut fo = sink.take(F, foff, nr, st);
  final_compact(fsel, roff, fcnt, foff, nr, hk, hs, o, ix->t_begin, q_first, fo, st);
  return F;
}

// CDeviceHitList for every query window of `qb` against one index.
void search_batch(clast_ctx* c, const clast_index* ix, const clast_params* p, const QueryRef& qb,
                  int32_t q_first, DevHits& out) {
  DevHitsSink sink(out);
  if (qb.q.nstrands == 0 || ix->n_keys == 0) return;
  std::vector<SeedSet> sets(1);
  sets[0].ix = ix;
  seed_windows(c, p, qb, sets);
  search_seeded(c, c->ws, p, qb, q_first, sets[0], true, sink);
}

template <class T>
T* host_copy(const std::vector<T>& v) {
  T* p = static_cast<T*>(std::malloc((v.size() ? v.size() : 1) * sizeof(T)));
  if (!p) throw std::bad_alloc();
  if (!v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}


}  // namespace

// ----------------------------------------------------------------------------
// targets / map: whole job with resident indexes
// ----------------------------------------------------------------------------

namespace clast {

// Waits for the index builds of clast_targets_create (once), records their
// time in the context's stats and reports a table overflow.
void settle_targets(clast_ctx* ctx, const clast_targets* T) {
  if (T->settled) return;
  CLAST_CK(cudaEventSynchronize(T->ev_done));
  T->settled = true;
  float up = 0, bd = 0;
  CLAST_CK(cudaEventElapsedTime(&up, T->ev_start, T->ev_up));
  CLAST_CK(cudaEventElapsedTime(&bd, T->ev_up, T->ev_done));
  ctx->stats.index_upload_ms = up;
  ctx->stats.index_ms = bd;
  ctx->stats.index_launches = T->launches;
  if (read_scalar(reinterpret_cast<const int64_t*>(T->failed.p), ctx->st) != 0)
    throw std::runtime_error("index table overflow");
  ctx->stats.index_bases = ctx->stats.index_keys = 0;
  for (const auto& w : T->wins) {
    ctx->stats.index_bases += w.ix->n;
    if (w.ix->kept.p) ctx->stats.index_keys += read_scalar(w.ix->kept.p, ctx->st);
  }
}

}  // namespace clast

namespace {


// One read window list per query load (moveQueryWindow, CHostSchedular.cu:12-23):
// the window [qb, qe) grows while gateway(2*qe+2) - gateway(2*qb) < q_vram,
// where every read adds two strands of len + l - 1 bases.  With the prefix
// sums cum[], qe = clamp(first j with cum[j] >= cum[qb] + q_vram, minus one,
// to [qb + 1, n]).
void query_windows(const int64_t* offsets, int64_t r0, int64_t r1, int l, int32_t q_vram,
                   std::vector<int64_t>& win_first_read) {
  const int64_t n = r1 - r0;
  std::vector<int64_t> cum(n + 1);
  cum[0] = 0;
  for (int64_t r = 0; r < n; ++r)
    cum[r + 1] = cum[r] + 2 * ((offsets[r0 + r + 1] - offsets[r0 + r]) + (l - 1));
  for (int64_t qb = 0; qb < n;) {
    const int64_t lim = cum[qb] + (int64_t)q_vram;
    const int64_t j = std::lower_bound(cum.begin() + qb, cum.end(), lim) - cum.begin();
    const int64_t qe = std::max(qb + 1, std::min(n, j - 1));
    win_first_read.push_back(r0 + qb);
    qb = qe;
  }
}

}  // namespace

extern "C" {

int clast_ctx_create(int device, clast_ctx** out) {
  if (!out) return CLAST_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<clast_ctx> c(new (std::nothrow) clast_ctx());
  if (!c) return CLAST_ERR_NOMEM;
  c->device = device;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    (void)cudaGetLastError();
    return CLAST_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) return CLAST_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return CLAST_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) return CLAST_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking) != cudaSuccess) return CLAST_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&c->st_dp, cudaStreamNonBlocking) != cudaSuccess) return CLAST_ERR_CUDA;
  if (cudaEventCreateWithFlags(&c->ev_dp_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_dp_join, cudaEventDisableTiming) != cudaSuccess)
    return CLAST_ERR_CUDA;
  for (int b = 0; b < kBuildStreams; ++b)
    if (cudaStreamCreateWithFlags(&c->st_build[b], cudaStreamNonBlocking) != cudaSuccess) return CLAST_ERR_CUDA;
  {  // keep freed pool memory for reuse by later calls of this process
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    (void)cudaGetLastError();
  }
  if (cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaEventCreate(&c->ev2) != cudaSuccess || cudaEventCreate(&c->ev3) != cudaSuccess ||
      cudaEventCreate(&c->ev_t0) != cudaSuccess || cudaEventCreate(&c->ev_t1) != cudaSuccess)
    return CLAST_ERR_CUDA;
  *out = c.release();
  return CLAST_OK;
}

void clast_ctx_destroy(clast_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  for (auto& a : ctx->arenas) {  // device copies of results, freed on the stream before it goes
    for (auto& f : a->dev.f) f.release();
    a->dev.evalue.release();
    a->dev.load_offsets.release();
  }
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  for (int b = 0; b < kBuildStreams; ++b)
    if (ctx->st_build[b]) cudaStreamSynchronize(ctx->st_build[b]);
  ctx->ws.release_all();
  for (auto& w : ctx->ws_build) w.release_all();
  for (auto& a : ctx->arenas)
    if (a->p) cudaFreeHost(a->p);
  for (auto& a : ctx->tsv_arenas)
    if (a->p) cudaFreeHost(a->p);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->ev2) cudaEventDestroy(ctx->ev2);
  if (ctx->ev3) cudaEventDestroy(ctx->ev3);
  if (ctx->ev_t0) cudaEventDestroy(ctx->ev_t0);
  if (ctx->ev_t1) cudaEventDestroy(ctx->ev_t1);
  if (ctx->ev_dp_fork) cudaEventDestroy(ctx->ev_dp_fork);
  if (ctx->ev_dp_join) cudaEventDestroy(ctx->ev_dp_join);
  if (ctx->st_dp) {
    cudaStreamSynchronize(ctx->st_dp);
    cudaStreamDestroy(ctx->st_dp);
  }
  if (ctx->st_copy) {
    cudaStreamSynchronize(ctx->st_copy);
    cudaStreamDestroy(ctx->st_copy);
  }
  for (int b = 0; b < kBuildStreams; ++b)
    if (ctx->st_build[b]) cudaStreamDestroy(ctx->st_build[b]);
  if (ctx->st) cudaStreamDestroy(ctx->st);
  delete ctx;
}

const char* clast_last_error(const clast_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int clast_index_build(clast_ctx* ctx, const clast_params* p, const char* bases, int64_t n_bases,
                      const int32_t* gateway, const int32_t* lengths, int32_t n_seqs, int32_t t_begin,
                      clast_index** out) {
  if (!ctx || !out) return CLAST_ERR_ARG;
  *out = nullptr;
  return guarded(ctx, [&]() -> int {
    check_params(p);
    if (n_bases < 0 || n_seqs < 0 || (n_bases > 0 && !bases) || (n_seqs > 0 && (!gateway || !lengths)))
      throw std::invalid_argument("bad window arrays");
    if (n_bases >= INT32_MAX) throw std::invalid_argument("window larger than 2^31 bases");
    CLAST_CK(cudaSetDevice(ctx->device));
    g_alloc_stream = ctx->st;
    g_kernel_launches = 0;
    ctx->stats.index_ms = ctx->stats.index_upload_ms = 0;
    ctx->stats.index_launches = 0;
    *out = make_index(ctx, p, bases, n_bases, gateway, lengths, n_seqs, t_begin);
    return CLAST_OK;
  });
}

void clast_index_free(clast_index* ix) { delete ix; }

int clast_search(clast_ctx* ctx, const clast_index* ix, const clast_params* p, const char* q_bases,
                 int64_t n_qbases, const int32_t* q_gateway, const int32_t* q_lengths, int32_t n_qseqs,
                 int32_t q_begin, clast_hits* out) {
  if (!ctx || !out) return CLAST_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  return guarded(ctx, [&]() -> int {
    check_params(p);
    if (!ix) throw std::invalid_argument("index is null");
    if (p->lmer != ix->l || p->stride != ix->stride || p->cut_repeat != ix->cut)
      throw std::invalid_argument("params differ from the ones the index was built with");
    if (n_qseqs < 0 || (n_qseqs & 1) || (q_begin & 1))
      throw std::invalid_argument("query windows hold whole reads: n_qseqs and q_begin must be even");
    if (n_qbases < 0 || (n_qbases > 0 && !q_bases) || (n_qseqs > 0 && (!q_gateway || !q_lengths)))
      throw std::invalid_argument("bad query arrays");
    CLAST_CK(cudaSetDevice(ctx->device));
    g_alloc_stream = ctx->st;
    g_kernel_launches = 0;
    cudaStream_t st = ctx->st;
    QueryBatch qb;
    qb.n = n_qbases;
    qb.nstrands = n_qseqs;
    upload_padded(q_bases, n_qbases, qb.bases, st);
    std::vector<int64_t> start(n_qseqs);
    qb.min_len = n_qseqs ? INT32_MAX : 0;
    for (int32_t i = 0; i < n_qseqs; ++i) {
      start[i] = q_gateway[i];
      if (q_gateway[i] < 0 || q_lengths[i] < 0 || (int64_t)q_gateway[i] + q_lengths[i] > n_qbases)
        throw std::invalid_argument("query sequence outside the base array");
      qb.min_len = std::min(qb.min_len, q_lengths[i]);
      qb.max_len = std::max(qb.max_len, q_lengths[i]);
    }
    qb.start.alloc(n_qseqs);
    qb.len.alloc(n_qseqs);
    if (n_qseqs) {
      CLAST_CK(cudaMemcpyAsync(qb.start.p, start.data(), n_qseqs * sizeof(int64_t), cudaMemcpyHostToDevice, st));
      CLAST_CK(cudaMemcpyAsync(qb.len.p, q_lengths, n_qseqs * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    }
    const int32_t ws2[2] = {0, n_qseqs};
    qb.nwin = 1;
    qb.wstart.alloc(2);
    CLAST_CK(cudaMemcpyAsync(qb.wstart.p, ws2, sizeof(ws2), cudaMemcpyHostToDevice, st));
    qb.pack(st);
    DevHits h;
    search_batch(ctx, ix, p, qb.ref(), q_begin, h);
    const int64_t F = h.n;
    out->n = F;
    auto d2h32 = [&](int32_t*& dst, const DevArray<int32_t>& src) {
      dst = static_cast<int32_t*>(std::malloc((F ? F : 1) * sizeof(int32_t)));
      if (!dst) throw std::bad_alloc();
      if (F) CLAST_CK(cudaMemcpyAsync(dst, src.p, F * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    };
    d2h32(out->t_id, h.t_id); d2h32(out->t_idx, h.t_idx); d2h32(out->q_id, h.q_id); d2h32(out->q_idx, h.q_idx);
    d2h32(out->t_len, h.t_len); d2h32(out->q_len, h.q_len); d2h32(out->match, h.match); d2h32(out->score, h.score);
    out->evalue = static_cast<double*>(std::malloc((F ? F : 1) * sizeof(double)));
    if (!out->evalue) throw std::bad_alloc();
    if (F) CLAST_CK(cudaMemcpyAsync(out->evalue, h.evalue.p, F * sizeof(double), cudaMemcpyDeviceToHost, st));
    CLAST_CK(cudaStreamSynchronize(st));
    ctx->last_launches = g_kernel_launches;
    return CLAST_OK;
  });
}

void clast_hits_free(clast_hits* h) {
  if (!h) return;
  std::free(h->t_id); std::free(h->t_idx); std::free(h->q_id); std::free(h->q_idx);
  std::free(h->t_len); std::free(h->q_len); std::free(h->match); std::free(h->score);
  std::free(h->evalue);
  std::memset(h, 0, sizeof(*h));
}

int clast_targets_create(clast_ctx* ctx, const clast_params* p, int32_t t_vram, const clast_seqs* targets,
                         int32_t n_loads, const int64_t* load_sizes, clast_targets** out) {
  if (!ctx || !out) return CLAST_ERR_ARG;
  *out = nullptr;
  return guarded(ctx, [&]() -> int {
    check_params(p);
    if (!targets || n_loads < 0 || (n_loads > 0 && !load_sizes)) throw std::invalid_argument("bad targets");
    int64_t total = 0;
    for (int32_t k = 0; k < n_loads; ++k) total += load_sizes[k];
    if (total != targets->n_seqs) throw std::invalid_argument("load sizes do not add up to n_seqs");
    CLAST_CK(cudaSetDevice(ctx->device));
    g_alloc_stream = ctx->st;
    g_kernel_launches = 0;
    ctx->stats.index_ms = ctx->stats.index_upload_ms = 0;
    ctx->stats.index_launches = 0;
    const double w0 = wall_ms();
    const int l = p->lmer;
    std::unique_ptr<clast_targets> T(new clast_targets());
    T->ctx = ctx;
    T->n_loads = n_loads;
    for (int32_t k = 0; k < n_loads; ++k) T->load_first.push_back(T->load_first.back() + load_sizes[k]);
    cudaStream_t st = ctx->st;
    T->ev_start = ctx->timer.take();
    T->ev_up = ctx->timer.take();
    T->ev_done = ctx->timer.take();
    T->failed.alloc(1);
    // the raw target set on the device, uploaded once unless already resident
    const int64_t nt = targets->n_seqs;
    const int64_t tbytes = nt ? targets->offsets[nt] - targets->offsets[0] : 0;
    // host-resident bases go up on the copy stream window by window, so that a
    // window's index build starts as soon as its bytes have arrived
    const bool host_src = !targets->bases_on_device;
    const char* hsrc = targets->bases + (nt ? targets->offsets[0] : 0);
    DevArray<char> traw;
    cudaStream_t cs = host_src ? ctx->st_copy : st;
    if (host_src) {
      g_alloc_stream = ctx->st_copy;
      traw.alloc((size_t)tbytes + 1);
      g_alloc_stream = st;
      traw.st = st;  // freed in the compute stream's order, after the builds
    }
    const char* src = host_src ? traw.p : hsrc;
    CLAST_CK(cudaEventRecord(T->ev_start, cs));
    if (!host_src) CLAST_CK(cudaEventRecord(T->ev_up, cs));  // nothing to upload
    int64_t copied = 0;  // source bytes already queued for upload
    std::vector<cudaEvent_t> win_ev;
    // the windows are indexed back to back on the stream with no host
    // synchronisation; the table-overflow count is read by the first clast_map
    unsigned long long* failed = T->failed.p;
    CLAST_CK(cudaMemsetAsync(failed, 0, sizeof(unsigned long long), st));
    const int64_t k0 = g_kernel_launches;
    const int64_t base0 = nt ? targets->offsets[0] : 0;
    // the windows of every load (moveTargetWindow, CHostSchedular.cu:25-35) and
    // their sequence tables, planned on the host and uploaded in one go: a copy
    // from pageable memory waits for the stream, so none happens per window
    struct Plan { int32_t load, first, nseqs; int64_t n, meta; };
    std::vector<Plan> plan;
    std::vector<int32_t> gw, ln;
    std::vector<int64_t> so;
    int64_t rec = 0;
    for (int32_t k = 0; k < n_loads; ++k) {
      const int64_t r0 = rec, r1 = rec + load_sizes[k];
      rec = r1;
      // load-relative gateway: prefix sums of len + l - 1 (CHostSeqList_target.cu:8-33)
      std::vector<int64_t> lg(r1 - r0 + 1, 0);
      for (int64_t i = r0; i < r1; ++i)
        lg[i - r0 + 1] = lg[i - r0] + (targets->offsets[i + 1] - targets->offsets[i]) + (l - 1);
      const int64_t tEnd = r1 - r0;
      for (int64_t tb = 0, te = 1; tb < tEnd; tb = te++) {
        while (te < tEnd && lg[te + 1] - lg[tb] < (int64_t)t_vram) ++te;
        const int64_t wn = lg[te] - lg[tb];
        if (wn >= (int64_t)INT32_MAX) throw std::invalid_argument("target window larger than 2^31 bases");
        plan.push_back(Plan{k, (int32_t)tb, (int32_t)(te - tb), wn, (int64_t)gw.size()});
        for (int64_t i = r0 + tb; i < r0 + te; ++i) {
          gw.push_back((int32_t)(lg[i - r0] - lg[tb]));
          ln.push_back((int32_t)(targets->offsets[i + 1] - targets->offsets[i]));
          so.push_back(targets->offsets[i] - base0);
        }
      }
    }
    DevArray<int32_t> all_gw, all_ln;
    DevArray<int64_t> all_so;
    all_gw.alloc(gw.size());
    all_ln.alloc(ln.size());
    all_so.alloc(so.size());
    if (!gw.empty()) {
      CLAST_CK(cudaMemcpyAsync(all_gw.p, gw.data(), gw.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
      CLAST_CK(cudaMemcpyAsync(all_ln.p, ln.data(), ln.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
      CLAST_CK(cudaMemcpyAsync(all_so.p, so.data(), so.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    }
    // Windows are built alternately on the context's build streams, each with
    // its own scratch, so that two builds run at once (a build is a chain of
    // small, latency-bound kernels); every build stream starts after the plan's
    // upload above and the compute stream waits for all of them at the end.
    cudaEvent_t planned = ctx->timer.take();
    win_ev.push_back(planned);
    CLAST_CK(cudaEventRecord(planned, st));
    for (int b = 0; b < kBuildStreams; ++b) CLAST_CK(cudaStreamWaitEvent(ctx->st_build[b], planned, 0));
    for (size_t wi = 0; wi < plan.size(); ++wi) {
      const Plan& w = plan[wi];
      const int b = (int)(wi % kBuildStreams);
      cudaStream_t bs = ctx->st_build[b];
      if (host_src) {  // the window's records: source bytes up to the end of its last record
        const int64_t last = so[w.meta + w.nseqs - 1] + ln[w.meta + w.nseqs - 1];
        if (last > copied) {
          CLAST_CK(cudaMemcpyAsync(traw.p + copied, hsrc + copied, (size_t)(last - copied), cudaMemcpyHostToDevice,
                                   cs));
          copied = last;
        }
        win_ev.push_back(ctx->timer.take());
        CLAST_CK(cudaEventRecord(win_ev.back(), cs));
        CLAST_CK(cudaStreamWaitEvent(bs, win_ev.back(), 0));
      }
      g_alloc_stream = bs;
      DevArray<char> padded;
      DevArray<int32_t> dgw, dln;
      padded.alloc((size_t)w.n + 2 * kPad);
      dgw.alloc(w.nseqs);
      dln.alloc(w.nseqs);
      CLAST_CK(cudaMemcpyAsync(dgw.p, all_gw.p + w.meta, w.nseqs * sizeof(int32_t), cudaMemcpyDeviceToDevice, bs));
      CLAST_CK(cudaMemcpyAsync(dln.p, all_ln.p + w.meta, w.nseqs * sizeof(int32_t), cudaMemcpyDeviceToDevice, bs));
      CLAST_CK(cudaMemsetAsync(padded.p, 'N', (size_t)w.n + 2 * kPad, bs));
      build_window(src, all_so.p + w.meta, dgw.p, dln.p, w.nseqs, w.n, padded.p + kPad, bs);
      clast_targets::Win win;
      win.load = w.load;
      win.first = w.first;
      win.ix.reset(make_index_resident(ctx->ws_build[b], bs, p, std::move(padded), w.n, std::move(dgw),
                                       std::move(dln), w.nseqs, w.first, failed));
      g_alloc_stream = st;
      // the index is used and finally freed in the compute stream's order
      clast_index& ix = *win.ix;
      ix.bases.st = ix.gateway.st = ix.lengths.st = ix.filter.st = ix.table.st = ix.entries.st = ix.kept.st = st;
      T->wins.push_back(std::move(win));
    }
    // the builds end on build stream 0 (which waits for the others): ev_done
    // there; the compute stream is not held up (clast_map prepares the query
    // while the builds run and waits for ev_done before its first search), and
    // the buffers the builds read are freed on build stream 0 after them
    cudaStream_t b0 = ctx->st_build[0];
    for (int b = 1; b < kBuildStreams; ++b) {
      win_ev.push_back(ctx->timer.take());
      CLAST_CK(cudaEventRecord(win_ev.back(), ctx->st_build[b]));
      CLAST_CK(cudaStreamWaitEvent(b0, win_ev.back(), 0));
    }
    if (host_src) {
      if (tbytes > copied)
        CLAST_CK(cudaMemcpyAsync(traw.p + copied, hsrc + copied, (size_t)(tbytes - copied), cudaMemcpyHostToDevice,
                                 cs));
      CLAST_CK(cudaEventRecord(T->ev_up, cs));
      CLAST_CK(cudaStreamWaitEvent(b0, T->ev_up, 0));  // the whole upload is done before traw goes
    }
    CLAST_CK(cudaEventRecord(T->ev_done, b0));
    traw.st = all_gw.st = all_ln.st = all_so.st = b0;
    T->launches = g_kernel_launches - k0;
    // a host source must stay readable until its copy has been made
    if (host_src) CLAST_CK(cudaEventSynchronize(T->ev_up));
    for (cudaEvent_t e : win_ev) ctx->timer.pool.push_back(e);
    ctx->stats.index_wall_ms = wall_ms() - w0;
    *out = T.release();
    return CLAST_OK;
  });
}

void clast_targets_free(clast_targets* t) { delete t; }

static int map_impl(clast_ctx* ctx, const clast_targets* T, const clast_params* p, int32_t q_vram,
                    const clast_seqs* reads, int32_t n_loads, const int64_t* load_sizes, clast_map_result* out);

int clast_map(clast_ctx* ctx, const clast_targets* T, const clast_params* p, int32_t q_vram,
              const clast_seqs* reads, int32_t n_loads, const int64_t* load_sizes, clast_map_result* out) {
  if (!ctx || !out) return CLAST_ERR_ARG;
  const double w0 = wall_ms();
  const int rc = map_impl(ctx, T, p, q_vram, reads, n_loads, load_sizes, out);
  ctx->stats.map_call_ms = wall_ms() - w0;
  return rc;
}

static int map_impl(clast_ctx* ctx, const clast_targets* T, const clast_params* p, int32_t q_vram,
                    const clast_seqs* reads, int32_t n_loads, const int64_t* load_sizes, clast_map_result* out) {
  std::memset(out, 0, sizeof(*out));
  return guarded(ctx, [&]() -> int {
    check_params(p);
    if (!T || !reads || n_loads < 0 || (n_loads > 0 && !load_sizes)) throw std::invalid_argument("bad arguments");
    int64_t total = 0;
    for (int32_t k = 0; k < n_loads; ++k) total += load_sizes[k];
    if (total != reads->n_seqs) throw std::invalid_argument("load sizes do not add up to n_seqs");
    for (const auto& w : T->wins)
      if (p->lmer != w.ix->l || p->stride != w.ix->stride || p->cut_repeat != w.ix->cut)
        throw std::invalid_argument("params differ from the ones the targets were built with");
    CLAST_CK(cudaSetDevice(ctx->device));
    g_alloc_stream = ctx->st;
    g_kernel_launches = 0;
    cudaStream_t st = ctx->st;
    clast_stats& S = ctx->stats;
    const double w0 = wall_ms();
    S.map_ms = S.map_upload_ms = 0;
    S.map_launches = S.query_bases = S.query_kmers = S.seeds = S.hits = S.results = S.dp_cells = 0;
    S.dp_warp_hits = 0;
    ctx->timer.reset();
    const int64_t nreads = reads->n_seqs;
    if (nreads >= ((int64_t)1 << 30)) throw std::invalid_argument("at most 2^30 reads per map (2^31 strands)");
    const int64_t nb = reads->offsets[nreads] - reads->offsets[0];
    // The reads' bases go up first, on the copy stream (allocated there, so
    // nothing waits for the compute stream, which may still be building the
    // target indexes), so that the host preparation below overlaps the
    // transfer; the compute stream waits for the uploads further down and
    // frees the buffers in its order.
    cudaStream_t cs = ctx->st_copy;
    CLAST_CK(cudaEventRecord(ctx->ev0, cs));
    DevArray<char> draw;
    const char* rsrc = reads->bases + reads->offsets[0];
    if (!reads->bases_on_device) {
      g_alloc_stream = cs;
      draw.alloc((size_t)nb + 64);
      g_alloc_stream = st;
      draw.st = st;
      if (nb) CLAST_CK(cudaMemcpyAsync(draw.p, rsrc, nb, cudaMemcpyHostToDevice, cs));
      rsrc = draw.p;
      // the compute stream, which frees draw (also when a check below
      // throws), comes after the copy
      CLAST_CK(cudaEventRecord(ctx->ev3, cs));
      CLAST_CK(cudaStreamWaitEvent(st, ctx->ev3, 0));
    }
    // query windows of every load, in read order
    std::vector<int64_t> wfirst;
    std::vector<int64_t> load_first(n_loads + 1, 0);
    for (int32_t k = 0; k < n_loads; ++k) load_first[k + 1] = load_first[k] + load_sizes[k];
    for (int32_t k = 0; k < n_loads; ++k)
      query_windows(reads->offsets, load_first[k], load_first[k + 1], p->lmer, q_vram, wfirst);
    wfirst.push_back(nreads);
    std::vector<int32_t> wstart(wfirst.size());
    for (size_t i = 0; i < wfirst.size(); ++i) wstart[i] = (int32_t)(2 * wfirst[i]);
    // every read uploaded once; strands are built on the device
    std::vector<int64_t> off0;
    const int64_t* offs_rel = reads->offsets;  // offsets relative to the first read
    if (reads->offsets[0] != 0) {
      off0.resize(nreads + 1);
      for (int64_t i = 0; i <= nreads; ++i) off0[i] = reads->offsets[i] - reads->offsets[0];
      offs_rel = off0.data();
    }
    DevArray<int64_t> doff;
    g_alloc_stream = cs;
    doff.alloc((size_t)nreads + 1);
    QueryBatch qb;
    qb.wstart.alloc(wstart.size());
    g_alloc_stream = st;
    doff.st = qb.wstart.st = st;
    qb.n = 2 * nb;
    qb.nstrands = (int32_t)(2 * nreads);
    qb.min_len = nreads ? INT32_MAX : 0;
    for (int64_t r = 0; r < nreads; ++r) {
      const int64_t len = reads->offsets[r + 1] - reads->offsets[r];
      if (len > INT32_MAX) throw std::invalid_argument("read longer than 2^31 bases");
      qb.min_len = std::min<int32_t>(qb.min_len, (int32_t)len);
      qb.max_len = std::max<int32_t>(qb.max_len, (int32_t)len);
    }
    qb.bases.alloc((size_t)qb.n + 2 * kPad);
    qb.start.alloc(2 * nreads);
    qb.len.alloc(2 * nreads);
    qb.nwin = (int32_t)wfirst.size() - 1;
    S.map_prep_ms = wall_ms() - w0;
    CLAST_CK(cudaMemcpyAsync(doff.p, offs_rel, (nreads + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, cs));
    CLAST_CK(cudaMemcpyAsync(qb.wstart.p, wstart.data(), wstart.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                             cs));
    CLAST_CK(cudaEventRecord(ctx->ev3, cs));
    CLAST_CK(cudaStreamWaitEvent(st, ctx->ev3, 0));
    CLAST_CK(cudaEventRecord(ctx->ev1, st));  // the reads are resident and the compute stream is free
    CLAST_CK(cudaMemsetAsync(qb.bases.p, 'N', (size_t)qb.n + 2 * kPad, st));
    build_strands(rsrc, doff.p, nreads, nb, qb.bases.p + kPad, qb.start.p, qb.len.p, st);
    qb.pack(st);
    S.query_bases = qb.n;
    // the index builds of clast_targets_create end before the first search
    settle_targets(ctx, T);
    CLAST_CK(cudaStreamWaitEvent(st, T->ev_done, 0));
    // every target window, in holder order (target load, window)
    std::vector<DevHits> per_win(T->wins.size());
    const QueryRef qr = qb.ref();
    // windows seeded per pass over the query (CLAST_SEED_WINDOWS, 1..4)
    int group = 2;
    if (const char* e = std::getenv("CLAST_SEED_WINDOWS")) group = std::max(1, std::min(kMaxSeedWins, std::atoi(e)));
    for (size_t g0 = 0; g0 < T->wins.size(); g0 += (size_t)group) {
      std::vector<SeedSet> sets;
      std::vector<size_t> idx;
      for (size_t w = g0; w < std::min(T->wins.size(), g0 + (size_t)group); ++w) {
        const clast_index* ix = T->wins[w].ix.get();
        if (qr.q.nstrands == 0 || ix->n_keys == 0) continue;
        sets.emplace_back();
        sets.back().ix = ix;
        idx.push_back(w);
      }
      if (sets.empty()) continue;
      seed_windows(ctx, p, qr, sets);
      for (size_t j = 0; j < sets.size(); ++j) {
        DevHitsSink sink(per_win[idx[j]]);
        search_seeded(ctx, ctx->ws, p, qr, 0, sets[j], true, sink);
      }
    }
    // fixResult: stable merge by (read, score desc) over the windows, on the device
    std::vector<WinHits> wh;
    int64_t n_items = 0;
    for (size_t w = 0; w < T->wins.size(); ++w) {
      const DevHits& h = per_win[w];
      if (h.n == 0) continue;
      wh.push_back(WinHits{h.t_id.p, h.t_idx.p, h.q_id.p, h.q_idx.p, h.t_len.p, h.q_len.p, h.match.p, h.score.p,
                           h.evalue.p, h.foff.p, n_items, T->wins[w].load});
      n_items += h.n;
    }
    DevArray<WinHits> dwh;
    dwh.alloc(wh.size());
    if (!wh.empty())
      CLAST_CK(cudaMemcpyAsync(dwh.p, wh.data(), wh.size() * sizeof(WinHits), cudaMemcpyHostToDevice, st));
    const int64_t F = n_items;
    DevArray<int32_t> m_read, m_strand, m_load, m_seq, m_tidx, m_qidx, m_tlen, m_qlen, m_match, m_score;
    DevArray<double> m_e;
    for (auto* a : {&m_read, &m_strand, &m_load, &m_seq, &m_tidx, &m_qidx, &m_tlen, &m_qlen, &m_match, &m_score})
      a->alloc(F);
    m_e.alloc(F);
    int32_t* mcnt = ctx->ws.get<int32_t>("m_cnt", nreads + 1);
    int64_t* moff = ctx->ws.get<int64_t>("m_off", nreads + 1);
    MapOut mo{m_read.p, m_strand.p, m_load.p, m_seq.p, m_tidx.p, m_qidx.p, m_tlen.p, m_qlen.p, m_match.p,
              m_score.p, m_e.p};
    merge_windows(dwh.p, (int)wh.size(), n_items, nreads, mcnt, moff, mo, ctx->ws, st);
    // per query load offsets
    std::vector<int64_t> lf(load_first.begin(), load_first.end());
    DevArray<int64_t> dlf, dlo;
    dlf.alloc(lf.size());
    dlo.alloc(lf.size());
    CLAST_CK(cudaMemcpyAsync(dlf.p, lf.data(), lf.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    if (nreads > 0) gather_i64(moff, dlf.p, (int)lf.size(), dlo.p, st);
    else CLAST_CK(cudaMemsetAsync(dlo.p, 0, lf.size() * sizeof(int64_t), st));
    clast_map_result res;
    std::memset(&res, 0, sizeof(res));
    res.n = F;
    // one pinned arena: load offsets, ten int32 arrays, evalue
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t need = al((n_loads + 1) * sizeof(int64_t)) + 10 * al((F ? F : 1) * sizeof(int32_t)) +
                        al((F ? F : 1) * sizeof(double));
    PinnedArena* arena = nullptr;
    for (auto& a : ctx->arenas)
      if (!a->in_use && (arena == nullptr || a->bytes > arena->bytes)) arena = a.get();
    if (!arena) {
      ctx->arenas.emplace_back(new PinnedArena());
      arena = ctx->arenas.back().get();
    }
    if (arena->bytes < need) {
      if (arena->p) CLAST_CK(cudaFreeHost(arena->p));
      arena->p = nullptr;
      arena->bytes = 0;
      const size_t nb = need + need / 4;
      if (cudaMallocHost(&arena->p, nb) != cudaSuccess) {
        (void)cudaGetLastError();
        throw std::bad_alloc();
      }
      arena->bytes = nb;
    }
    arena->in_use = true;
    res.owner = arena;
    char* cur = static_cast<char*>(arena->p);
    auto take = [&](size_t b) { char* q = cur; cur += al(b); return q; };
    res.load_offsets = reinterpret_cast<int64_t*>(take((n_loads + 1) * sizeof(int64_t)));
    std::memset(res.load_offsets, 0, (n_loads + 1) * sizeof(int64_t));
    if (nreads > 0)
      CLAST_CK(cudaMemcpyAsync(res.load_offsets, dlo.p, (n_loads + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                               st));
    auto d2h32 = [&](int32_t*& dst, const DevArray<int32_t>& src) {
      dst = reinterpret_cast<int32_t*>(take((F ? F : 1) * sizeof(int32_t)));
      if (F) CLAST_CK(cudaMemcpyAsync(dst, src.p, F * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    };
    d2h32(res.read, m_read); d2h32(res.strand, m_strand); d2h32(res.t_load, m_load); d2h32(res.t_seq, m_seq);
    d2h32(res.t_idx, m_tidx); d2h32(res.q_idx, m_qidx); d2h32(res.t_len, m_tlen); d2h32(res.q_len, m_qlen);
    d2h32(res.match, m_match); d2h32(res.score, m_score);
    res.evalue = reinterpret_cast<double*>(take((F ? F : 1) * sizeof(double)));
    if (F) CLAST_CK(cudaMemcpyAsync(res.evalue, m_e.p, F * sizeof(double), cudaMemcpyDeviceToHost, st));
    {  // the device copy stays with the arena for clast_format_tsv
      PinnedArena::Device& d = arena->dev;
      DevArray<int32_t>* src[10] = {&m_read, &m_strand, &m_load, &m_seq, &m_tidx, &m_qidx, &m_tlen, &m_qlen,
                                    &m_match, &m_score};
      for (int k = 0; k < 10; ++k) d.f[k] = std::move(*src[k]);
      d.evalue = std::move(m_e);
      d.load_offsets = std::move(dlo);
      d.n = F;
      d.n_loads = n_loads;
    }
    CLAST_CK(cudaEventRecord(ctx->ev2, st));
    CLAST_CK(cudaEventSynchronize(ctx->ev2));
    float up = 0, ms = 0;
    CLAST_CK(cudaEventElapsedTime(&up, ctx->ev0, ctx->ev3));
    CLAST_CK(cudaEventElapsedTime(&ms, ctx->ev1, ctx->ev2));
    ctx->timer.flush();
    S.map_upload_ms = up;
    S.map_ms = ms;
    S.map_launches = g_kernel_launches;
    S.seed_ms = ctx->timer.ms[StageTimer::SEED];
    S.seed_launches = ctx->timer.n[StageTimer::SEED];
    S.dp_ms = ctx->timer.ms[StageTimer::DP];
    S.dp_launches = ctx->timer.n[StageTimer::DP];
    S.sort_ms = ctx->timer.ms[StageTimer::SORT];
    S.final_ms = ctx->timer.ms[StageTimer::FINAL];
    S.dp_order_ms = ctx->timer.ms[StageTimer::DPORDER];
    ctx->last_ms = up + ms;
    ctx->last_launches = g_kernel_launches;
    S.map_wall_ms = wall_ms() - w0;
    *out = res;
    return CLAST_OK;
  });
}

void clast_map_result_free(clast_map_result* r) {
  if (!r) return;
  if (r->owner) static_cast<PinnedArena*>(r->owner)->in_use = false;
  std::memset(r, 0, sizeof(*r));
}

int clast_ctx_trim(clast_ctx* ctx) {
  if (!ctx) return CLAST_ERR_ARG;
  return guarded(ctx, [&]() -> int {
    CLAST_CK(cudaSetDevice(ctx->device));
    CLAST_CK(cudaDeviceSynchronize());
    for (auto& a : ctx->arenas)
      if (!a->in_use) {
        for (auto& f : a->dev.f) f.release();
        a->dev.evalue.release();
        a->dev.load_offsets.release();
      }
    ctx->ws.release_all();
    for (auto& w : ctx->ws_build) w.release_all();
    CLAST_CK(cudaDeviceSynchronize());
    cudaMemPool_t pool;
    CLAST_CK(cudaDeviceGetDefaultMemPool(&pool, ctx->device));
    CLAST_CK(cudaMemPoolTrimTo(pool, 0));
    return CLAST_OK;
  });
}

int clast_int32_peak(clast_ctx* ctx, double* tera_ops) {
  if (!ctx || !tera_ops) return CLAST_ERR_ARG;
  return guarded(ctx, [&]() -> int {
    CLAST_CK(cudaSetDevice(ctx->device));
    int* sink = ctx->ws.get<int>("probe_sink", 1);
    *tera_ops = int32_probe(ctx->st, sink);
    return CLAST_OK;
  });
}

int clast_get_stats(const clast_ctx* ctx, clast_stats* out) {
  if (!ctx || !out) return CLAST_ERR_ARG;
  *out = ctx->stats;
  return CLAST_OK;
}

int clast_last_map_stats(const clast_ctx* ctx, double* device_ms, int64_t* kernel_launches) {
  if (!ctx) return CLAST_ERR_ARG;
  if (device_ms) *device_ms = ctx->last_ms;
  if (kernel_launches) *kernel_launches = ctx->last_launches;
  return CLAST_OK;
}

}  // extern "C"

// ----------------------------------------------------------------------------
// clast_search_noalloc: clast_search on a fixed scratch buffer, allocating
// nothing.  It seeds the one query window itself (partitions sized to fit
// the scratch), then runs search_seeded, the stages clast_search runs, with
// every device buffer a slot of the static scratch (Workspace arena mode);
// the hits go from scratch slots straight into the caller's host arrays.
// ----------------------------------------------------------------------------
namespace {

constexpr size_t kSearchScratchBytes = (size_t)CLAST_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_search_scratch[kSearchScratchBytes];

constexpr int kMaxScratchDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxScratchDevices];           // device address of g_search_scratch, per device
std::atomic<int> g_scratch_busy[kMaxScratchDevices];  // 1 while a call uses that device's scratch

// Address of this device's scratch; the device must be current.  Looked up
// once per device.
char* search_scratch(int device) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void* ptr = nullptr;
    CLAST_CK(cudaGetSymbolAddress((void**)&ptr, g_search_scratch));
    g_scratch_addr[device] = ptr;
  }
  return static_cast<char*>(g_scratch_addr[device]);
}

__global__ void k_widen_i32(const int32_t* __restrict__ in, int64_t n, int64_t* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

// Bytes of the query-sized buffers, as Workspace::get rounds them.
size_t fixed_scratch_bytes(int64_t n, int64_t ns, int parts) {
  auto r = [](size_t b) { return ((b ? b : 1) + 255) & ~size_t(255); };
  const size_t nb = (size_t)n, s = (size_t)ns;
  return r(nb + 2 * kPad) + r(8 * s) + r(4 * s) + r(4 * s) + r(8) + r(8 * (nb / 32 + 4)) + r(8 * (nb / 64 + 4)) +
         r(8 * (s + 1)) + r(4 * s) + r(4 * s) + r(8 * (2 + 2 * (size_t)parts)) + r(4 * s) + r(8 * (s + 1)) +
         r(16 * s) + (64 << 10);
}

// Clears the busy flag of a device's scratch once the call's stream work has
// ended (also when the call failed after launching work).
struct ScratchClaim {
  int device;
  cudaStream_t st;
  ~ScratchClaim() {
    cudaStreamSynchronize(st);
    (void)cudaGetLastError();
    g_scratch_busy[device].store(0);
  }
};

}  // namespace

extern "C" int clast_search_noalloc(clast_ctx* ctx, const clast_index* ix, const clast_params* p,
                                    const char* q_bases, int64_t n_qbases, const int32_t* q_gateway,
                                    const int32_t* q_lengths, int32_t n_qseqs, int32_t q_begin, int64_t capacity,
                                    clast_hits* out) {
  if (!ctx || !out) return CLAST_ERR_ARG;
  out->n = 0;
  return guarded(ctx, [&]() -> int {
    check_params(p);
    if (!ix) throw std::invalid_argument("index is null");
    if (p->lmer != ix->l || p->stride != ix->stride || p->cut_repeat != ix->cut)
      throw std::invalid_argument("params differ from the ones the index was built with");
    if (n_qseqs < 0 || (n_qseqs & 1) || (q_begin & 1))
      throw std::invalid_argument("query windows hold whole reads: n_qseqs and q_begin must be even");
    if (n_qbases < 0 || (n_qbases > 0 && !q_bases) || (n_qseqs > 0 && (!q_gateway || !q_lengths)))
      throw std::invalid_argument("bad query arrays");
    if (capacity < 0 || (capacity > 0 && (!out->t_id || !out->t_idx || !out->q_id || !out->q_idx ||
                                          !out->t_len || !out->q_len || !out->match || !out->score ||
                                          !out->evalue)))
      throw std::invalid_argument("capacity < 0, or a null output array");
    for (int32_t i = 0; i < n_qseqs; ++i)
      if (q_gateway[i] < 0 || q_lengths[i] < 0 || (int64_t)q_gateway[i] + q_lengths[i] > n_qbases)
        throw std::invalid_argument("query sequence outside the base array");
    if (ctx->device < 0 || ctx->device >= kMaxScratchDevices)
      throw std::invalid_argument("device ordinal beyond the scratch table");
    const int parts = seed_parts();
    const size_t fixed = fixed_scratch_bytes(n_qbases, n_qseqs, parts);
    if (fixed > kSearchScratchBytes)
      throw std::invalid_argument("query window of " + std::to_string(n_qbases) + " bases and " +
                                  std::to_string(n_qseqs) + " sequences needs " + std::to_string(fixed) +
                                  " bytes of scratch before seeding; clast_search_noalloc has " +
                                  std::to_string(kSearchScratchBytes) + " (use clast_search)");
    CLAST_CK(cudaSetDevice(ctx->device));
    int idle = 0;
    if (!g_scratch_busy[ctx->device].compare_exchange_strong(idle, 1))
      throw std::invalid_argument("another clast_search_noalloc call is using this device's scratch");
    cudaStream_t st = ctx->st;
    ScratchClaim claim{ctx->device, st};
    char* base = search_scratch(ctx->device);
    g_kernel_launches = 0;
    Workspace ws;
    ws.arena_begin(base, kSearchScratchBytes);
    const int64_t ns = n_qseqs, nr = ns / 2, n = n_qbases;
    // the query window: padded bases, strand starts and lengths, 2-bit words
    char* qbases = ws.get<char>("q_bases", (size_t)n + 2 * kPad);
    CLAST_CK(cudaMemsetAsync(qbases, 'N', (size_t)n + 2 * kPad, st));
    if (n > 0) CLAST_CK(cudaMemcpyAsync(qbases + kPad, q_bases, (size_t)n, cudaMemcpyHostToDevice, st));
    int64_t* qstart = ws.get<int64_t>("q_start", ns);
    int32_t* qlen = ws.get<int32_t>("q_len", ns);
    int32_t* qgw = ws.get<int32_t>("q_gw32", ns);
    int32_t* wstart = ws.get<int32_t>("q_wstart", 2);
    if (ns > 0) {
      CLAST_CK(cudaMemcpyAsync(qgw, q_gateway, ns * sizeof(int32_t), cudaMemcpyHostToDevice, st));
      CLAST_CK(cudaMemcpyAsync(qlen, q_lengths, ns * sizeof(int32_t), cudaMemcpyHostToDevice, st));
      k_widen_i32<<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(qgw, ns, qstart);
      CLAST_LAUNCHED();
    }
    const int32_t ws2[2] = {0, n_qseqs};
    CLAST_CK(cudaMemcpyAsync(wstart, ws2, sizeof(ws2), cudaMemcpyHostToDevice, st));
    uint64_t* packed = ws.get<uint64_t>("q_packed", (size_t)(n / 32 + 4));
    uint64_t* nmask = ws.get<uint64_t>("q_nmask", (size_t)(n / 64 + 4));
    pack_bases(qbases + kPad, n, packed, nmask, st);
    QueryView q;
    q.bases = qbases + kPad;
    q.n = n;
    q.packed = packed;
    q.nmask = nmask;
    q.start = qstart;
    q.len = qlen;
    q.nstrands = n_qseqs;
    const IndexView iv = ix->view();
    const TargetView tv = ix->tview();
    auto finish = [&](int64_t F) {
      CLAST_CK(cudaStreamSynchronize(st));
      ctx->last_launches = g_kernel_launches;
      out->n = F;
      return CLAST_OK;
    };
    if (ns == 0 || ix->n_keys == 0) return finish(0);
    // createRawSeedList + deleteSeedsOnSequenceBoundary, one pass
    int64_t* off = ws.get<int64_t>("s_off", ns + 1);
    int32_t* len32 = ws.get<int32_t>("s_len32", ns);
    int32_t* nvalid = ws.get<int32_t>("s_nvalid", ns);
    unsigned long long* counters = ws.get<unsigned long long>("s_counters", 2 + 2 * parts);
    // the seed partitions take at most half of the scratch still free
    const size_t mark = ws.arena_used;
    const int64_t fit = (int64_t)((ws.arena_cap - mark) / 2 / (12 * (size_t)parts)) - 256;
    int64_t part_cap = std::max<int64_t>(ctx->seed_hint, n / 16 + (1 << 20)) / parts + 1;
    part_cap = std::max<int64_t>(1, std::min(part_cap, fit));
    int64_t S = 0;
    uint64_t* skey = nullptr;
    uint32_t* sq = nullptr;
    for (int attempt = 0; attempt < 2; ++attempt) {
      skey = ws.get<uint64_t>("s_key", (size_t)part_cap * parts);
      sq = ws.get<uint32_t>("s_q", (size_t)part_cap * parts);
      CLAST_CK(cudaMemsetAsync(counters, 0, (2 + 2 * parts) * sizeof(unsigned long long), st));
      seed_fused(q, iv, tv, p->gap, p->local, counters + 2, counters + 2 + parts, off, len32, nvalid, skey, sq,
                 part_cap, st);
      unsigned long long cur[64];
      CLAST_CK(cudaMemcpyAsync(cur, counters + 2, parts * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
      CLAST_CK(cudaStreamSynchronize(st));
      S = 0;
      int64_t most = 0;
      for (int i = 0; i < parts; ++i) {
        S += (int64_t)cur[i];
        most = std::max<int64_t>(most, (int64_t)cur[i]);
      }
      if (most <= part_cap) break;
      if (most > fit)  // the partitions this window needs do not fit the scratch
        throw std::invalid_argument("query window needs seed partitions of " + std::to_string(most) +
                                    " seeds; clast_search_noalloc's scratch holds " + std::to_string(fit) +
                                    " (use clast_search)");
      ws.arena_rewind(mark);  // strands past a full partition wrote nothing: run again, larger
      part_cap = most;
    }
    if (S == 0) return finish(0);
    // the stages after seeding are clast_search's, on the fixed scratch (no
    // autotuner runs: its trial orders would need more of it); the hits go
    // to slots of the scratch, then to the caller's arrays
    int32_t lmin = INT32_MAX, lmax = 0;
    for (int32_t i = 0; i < n_qseqs; ++i) {
      lmin = std::min(lmin, q_lengths[i]);
      lmax = std::max(lmax, q_lengths[i]);
    }
    QueryRef qr;
    qr.q = q;
    qr.n = n;
    qr.wstart = wstart;
    qr.nwin = 1;
    qr.min_len = lmin;
    qr.max_len = lmax;
    SeedSet z;
    z.ix = ix;
    z.off = off;
    z.len32 = len32;
    z.nvalid = nvalid;
    z.counters = counters;
    z.skey = skey;
    z.sq = sq;
    z.part_cap = part_cap;
    z.S = S;
    struct ArenaSink : HitSink {
      Workspace& ws;
      int64_t capacity;
      clast_hits* out;
      FinalOut fo{};
      ArenaSink(Workspace& w, int64_t cap, clast_hits* o) : ws(w), capacity(cap), out(o) {}
      FinalOut take(int64_t F, const int64_t*, int64_t, cudaStream_t) override {
        if (F > capacity) {
          out->n = F;
          throw std::invalid_argument("window has " + std::to_string(F) + " hits, capacity is " +
                                      std::to_string(capacity));
        }
        fo = FinalOut{ws.get<int32_t>("o_tid", F), ws.get<int32_t>("o_tidx", F), ws.get<int32_t>("o_qid", F),
                      ws.get<int32_t>("o_qidx", F), ws.get<int32_t>("o_tlen", F), ws.get<int32_t>("o_qlen", F),
                      ws.get<int32_t>("o_match", F), ws.get<int32_t>("o_score", F), ws.get<double>("o_e", F)};
        return fo;
      }
    } sink(ws, capacity, out);
    const int64_t F = search_seeded(ctx, ws, p, qr, q_begin, z, false, sink);
    if (F == 0) return finish(0);
    const FinalOut& fo = sink.fo;
    int32_t* const dst[8] = {out->t_id, out->t_idx, out->q_id, out->q_idx, out->t_len, out->q_len, out->match,
                             out->score};
    const int32_t* const src[8] = {fo.t_id, fo.t_idx, fo.q_id, fo.q_idx, fo.t_len, fo.q_len, fo.match, fo.score};
    for (int k = 0; k < 8; ++k)
      CLAST_CK(cudaMemcpyAsync(dst[k], src[k], F * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CLAST_CK(cudaMemcpyAsync(out->evalue, fo.evalue, F * sizeof(double), cudaMemcpyDeviceToHost, st));
    return finish(F);
  });
}

