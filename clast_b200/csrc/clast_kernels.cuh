// clast_kernels.cuh -- launch wrappers of the sm_100a kernels (clast_kernels.cu).
// Every wrapper enqueues on `st` and returns immediately; sizes are element counts.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "clast_device.cuh"

namespace clast {

struct Workspace;  // device scratch pool (clast_engine.cu)

// out[0..n] = exclusive prefix sums of in[0..n) (out[n] = total).
void scan_i32(Workspace& ws, const int32_t* in, int64_t n, int64_t* out, cudaStream_t st);
// exclusive scan of (in[i] > 0)
void scan_positive(Workspace& ws, const int32_t* in, int64_t n, int64_t* out, cudaStream_t st);

// 2-bit codes (32 bases per word) and non-ACGT mask (64 per word) of bases[0..n);
// positions >= n count as 'N'.  packed needs ceil(n/32)+2 words, nmask ceil(n/64)+2.
void pack_bases(const char* bases, int64_t n, uint64_t* packed, uint64_t* nmask, cudaStream_t st);

// Query strands of n_reads one-strand reads: strand 2r = read r, strand 2r+1 its
// reverse complement (utilReverseSeq.cpp:3-19), laid out back to back.
void build_strands(const char* reads, const int64_t* offsets, int64_t n_reads, int64_t n_bases,
                   char* strands, int64_t* strand_start, int32_t* strand_len, cudaStream_t st);

// ---- index of one target window (CDeviceHashTable.cu:20-174) ----
// Window base array (sequences with their joints) from a one-strand source set:
// sequence k of the window is src[src_off[k] .. src_off[k]+lengths[k]).
void build_window(const char* src, const int64_t* src_off, const int32_t* gateway, const int32_t* lengths,
                  int nseqs, int64_t n, char* out, cudaStream_t st);
// Samples at window positions j*stride: order_code of the l-mer (4^l when it
// has a non-ACGT base).  pbits > 0: items[j] = code << pbits | j; pbits = 0:
// items[j] = code, vals[j] = j.
void sample_keys(const uint64_t* packed, const uint64_t* nmask, int64_t n_samples, int stride, int l, int pbits,
                 uint64_t* items, int32_t* vals, cudaStream_t st);
// keys[i] = items[i] >> pbits, vals[i] = the low pbits bits, head[i] =
// whether keys[i] < bound and differs from keys[i - 1].
void split_items(const uint64_t* items, int64_t n, int pbits, uint64_t bound, uint64_t* keys, int32_t* vals,
                 int32_t* head, cudaStream_t st);
// Stable LSD radix sort of 64-bit words by bits [lo_bit, hi_bit), carrying
// vals along unless vals is null.  Returns 0 when the result is in (keys,
// vals), 1 when it is in (keys_alt, vals_alt).
int radix_sort_u64(Workspace& ws, uint64_t* keys, int32_t* vals, uint64_t* keys_alt, int32_t* vals_alt, int64_t n,
                   int lo_bit, int hi_bit, cudaStream_t st);
// *out = number of keys < bound in the sorted array keys[0..n)
void count_below(const uint64_t* keys, int64_t n, uint64_t bound, int64_t* out, cudaStream_t st);
// Index build over n samples with the valid count *nv_dev and the unique
// count *nu_dev on the device (no host synchronisation).  head[i] = whether
// keys[i] < bound and differs from keys[i - 1].
void index_heads(const uint64_t* keys, int64_t n, uint64_t bound, int32_t* head, cudaStream_t st);
void index_unique(const uint64_t* keys, const int32_t* head, const int64_t* hpos, int64_t n, const int64_t* nv_dev,
                  uint64_t* ukeys, int64_t* ufirst, cudaStream_t st);
void index_keep(const int32_t* vals, const int64_t* hpos, const int64_t* ufirst, int64_t n, const int64_t* nv_dev,
                int stride, int l, int cut, const int32_t* gateway, const int32_t* lengths, int nseqs, int32_t* keep,
                int2* resolved, cudaStream_t st);
void index_entries(const int32_t* keep, const int64_t* kpos, const int2* resolved, int64_t nv,
                   int2* entries, cudaStream_t st);
void index_buckets(const int64_t* ufirst, const int64_t* kpos, int64_t n, const int64_t* nu_dev, int32_t* ustart,
                   int32_t* ucnt, cudaStream_t st);
// Hash table of the index without atomics (layout: IndexView).  rank =
// exclusive scan of (ucnt > 0), the codes that keep entries; table_runmax:
// run_max[k] = max over kept j <= k of home_j - rank_j; table_place writes
// every kept code's record at rank[k] + run_max[k] and sets its filter bits
// (filter zeroed, table records set to ~0 by the caller); *failed counts
// records that would fall outside the table (none).
void table_runmax(Workspace& ws, const uint64_t* ucode, const int32_t* ucnt, const int64_t* rank, int64_t n_unique,
                  int l, uint32_t nbuckets, int64_t* run_max, cudaStream_t st);
void table_place(const uint64_t* ucode, const int32_t* ustart, const int32_t* ucnt, const int2* entries,
                 const int64_t* rank, const int64_t* run_max, int64_t n_unique, ulonglong2* table, int64_t n_records,
                 uint32_t* filter, int fshift, unsigned long long* failed, cudaStream_t st);

// ---- seeds (CDeviceHitList_createRawSeedList.cu, _deleteSeeds*.cu, _sortSeeds.cu) ----
// One-pass seeding (lookups once): off/cnt/nvalid per strand, seeds in skey/sq,
// which hold seed_parts() partitions of part_cap seeds.  Strand s reserves its
// range in partition s % seed_parts() through cursors[partition]; a partition
// whose cursor ends above part_cap was not fully written and the call must be
// repeated with part_cap >= the largest cursor.  n_kmers holds seed_parts()
// counters (valid l-mers of the strands of each partition; the caller sums
// them), so that no single address takes one atomic per strand.
int seed_parts();
void seed_fused(const QueryView& q, const IndexView& ix, const TargetView& t, int gap, int local,
                unsigned long long* cursors, unsigned long long* n_kmers, int64_t* off, int32_t* cnt, int32_t* nvalid,
                uint64_t* skey, uint32_t* sq, int64_t part_cap, cudaStream_t st);
void window_first(const int32_t* nvalid, const int32_t* win_start, int n_windows, int32_t* win_first,
                  cudaStream_t st);
// The same outputs as seed_fused for up to kMaxSeedWins target windows in one
// pass over the query (each window with its own cursors, counters and seed
// partitions).  Every window must have been built with the same l.
struct SeedWin {
  IndexView ix;
  TargetView t;
  unsigned long long* cursor;   // seed_parts() cursors
  unsigned long long* n_kmers;  // seed_parts() l-mer counters
  int64_t* off;
  int32_t* cnt;
  int32_t* nvalid;
  uint64_t* skey;
  uint32_t* sq;
  int64_t part_cap;
};
constexpr int kMaxSeedWins = 4;
struct SeedWins {
  SeedWin w[kMaxSeedWins];
};
void seed_multi(const QueryView& q, const SeedWins& W, int nw, int gap, int local, cudaStream_t st);

// Sorts every segment [off[i], off[i]+len[i]) of (k1, k2[, payload]) ascending by
// (k1, k2).  Segments of <= 32 are sorted by one warp in registers, <= 2048 by one
// CTA in shared memory, longer ones by one CTA in global memory.
void segmented_sort_u64(Workspace& ws, uint64_t* k1, uint64_t* k2, int32_t* payload, const int64_t* off,
                        const int32_t* len, int64_t n_segments, cudaStream_t st, int tag);

// sortSeeds + deletingIsolateSeeds + deleteDuplicateSeeds per strand: sorts the
// cnt[s] seeds of strand s by (sequence, diagonal, qIdx) and writes the surviving
// hits at off[s] onwards, hcnt[s] of them.
void seed_sort_filter(Workspace& ws, uint64_t* skey, uint32_t* sq, const int64_t* off, const int32_t* cnt,
                      const int32_t* nvalid, const int32_t* win_start, int n_windows, const int32_t* win_first,
                      int width, int gap, int64_t nstrands, int32_t* hcnt, cudaStream_t st);
// also adds band * (qlen - l) DP cells per hit to *cells
void gather_hits(const uint64_t* skey, const uint32_t* sq, const int64_t* off, const int32_t* hcnt,
                 const int64_t* hoff, int64_t nstrands, uint64_t* hk, int32_t* hq, int32_t* hs,
                 const int32_t* qlen, int l, int band, unsigned long long* cells, cudaStream_t st);

// ---- banded DP + E-value (krnlAlignment.cu, krnlCalculateEvalue.cu) ----
struct DpOut {
  int32_t* t_idx; int32_t* q_idx; int32_t* t_len; int32_t* q_len; int32_t* match; int32_t* score;
  double* evalue; uint8_t* keep;
};
struct DpParams {
  int l, stride, gap, local;
  double cutoff, total_db, K, lambda;
};
// How the DP kernel is launched: one thread per hit over a grid of all hits
// (head null), or a persistent grid whose warps take `chunk` x 32 hits at a
// time from a queue (head: a device counter the launch zeroes).  Results are
// the same either way.
//
// Independently of that, the first hits of the order (the longest, when the
// order is longest first) may run one per warp (an anti-diagonal wavefront
// over the band) instead of one per thread: a long hit alone takes about 1/7
// of the time there, at a lower throughput per cell.  `warp` says how many:
// kDpWarpAuto splits where the cost model puts the end of both launches
// earliest -- on the device from the length buckets' counts and row sums
// (buckets + warp_n), or, for hits that all have `uniform_rows` rows, all or
// none on the host; kDpWarpOff runs every hit one per thread, kDpWarpAll one
// per warp.  Results are the same either way.
constexpr int kDpWarpAuto = 0, kDpWarpOff = 1, kDpWarpAll = 2;
struct DpBuckets {
  const unsigned int* count = nullptr;      // hits per length bucket (longest first)
  const unsigned long long* rows = nullptr;  // their rows, summed
};
struct DpLaunch {
  unsigned long long* head = nullptr;
  int chunk = 1;
  int warp = kDpWarpAuto;
  DpBuckets buckets;
  long long* warp_n = nullptr;  // device word for the split (with buckets)
  int uniform_rows = -1;
  // with aux, the one-per-warp kernel runs there, beside the others (forked
  // from and joined back into the launch stream by the two events)
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // device word set to 1 when a hit names a target sequence or strand outside
  // the window (an internal error: the hit is skipped, never read past)
  int* bad = nullptr;
};
// order (may be null): the hits in the order the threads take them, as words
// whose low 32 bits are hit indices; outputs stay at the hit's own index.
// Returns how many hits ran one per warp, or -1 when the split was made on the
// device (the count is then in *m.warp_n).
long long banded_dp(const TargetView& t, const QueryView& q, const uint64_t* hk, const int32_t* hq,
               const int32_t* hs, const uint64_t* order, int64_t n_hits, const DpParams& p, const DpOut& o,
               cudaStream_t st, const DpLaunch& m = DpLaunch());
// Hits per length bucket (16 per power of two of the row count, longest
// first) and their row sums, in the workspace.
DpBuckets dp_bucket_count(Workspace& ws, const int32_t* hs, const int32_t* q_len, int64_t n_hits, int l,
                          cudaStream_t st);
// DP order by length buckets: order[k] = hit index, in one counting pass
// instead of a sort (the counts of dp_bucket_count, which it runs).
DpBuckets dp_bucket_order(Workspace& ws, const int32_t* hs, const int32_t* q_len, int64_t n_hits, int l,
                          uint64_t* order, cudaStream_t st);
// CLAST_DP_WARP=off|all, else `fallback` (the environment overrides a
// context's setting, for tests and measurements).
int dp_warp_mode_from_env(int fallback);
// keys[h] = (rows_max - rows of hit h) << 32 | h, rows = q_len[hs[h]] - l + 1:
// ascending keys take the hits longest first.
void dp_order_keys(const int32_t* hs, const int32_t* q_len, int64_t n_hits, int l, int rows_max, uint64_t* keys,
                   cudaStream_t st);

// ---- per-read result order and duplicate removal (utilResultSorting.cuh, CDeviceHitList.cu:32-128) ----
void final_keys(const uint64_t* hk, const int32_t* hq, const int32_t* hs, const DpOut& o, int64_t n_hits,
                uint64_t* k1, uint64_t* k2, int32_t* idx, cudaStream_t st);
void read_ranges(const int64_t* hoff, int64_t n_reads, int64_t* roff, int32_t* rlen, cudaStream_t st);
void final_dedupe(const uint64_t* k1, const uint64_t* k2, const int32_t* idx, const uint64_t* hk,
                  const int32_t* hs, const DpOut& o, const int64_t* roff, const int32_t* rlen,
                  int64_t n_reads, int32_t* fcnt, int32_t* fsel, cudaStream_t st);
struct FinalOut {
  int32_t* t_id; int32_t* t_idx; int32_t* q_id; int32_t* q_idx; int32_t* t_len; int32_t* q_len;
  int32_t* match; int32_t* score; double* evalue;
};
void final_compact(const int32_t* fsel, const int64_t* roff, const int32_t* fcnt, const int64_t* foff,
                   int64_t n_reads, const uint64_t* hk, const int32_t* hs, const DpOut& o, int32_t t_first,
                   int32_t q_first, const FinalOut& out, cudaStream_t st);

// ---- merge of target windows in holder order (CHostResultHolder::fixResult) ----
struct WinHits {  // one target window's final hits (reads ascending)
  const int32_t* t_id; const int32_t* t_idx; const int32_t* q_id; const int32_t* q_idx;
  const int32_t* t_len; const int32_t* q_len; const int32_t* match; const int32_t* score;
  const double* evalue;
  const int64_t* foff;  // per read offsets, n_reads + 1
  int64_t base;         // position of its first item in the concatenation of all windows
  int32_t load;         // target RAM load of the window
};
struct MapOut {
  int32_t* read; int32_t* strand; int32_t* t_load; int32_t* t_seq; int32_t* t_idx; int32_t* q_idx;
  int32_t* t_len; int32_t* q_len; int32_t* match; int32_t* score; double* evalue;
};
// wins: device array of nw windows; total = items of all windows; moff (nreads+1)
// receives per-read offsets of the merged result.
void merge_windows(const WinHits* wins, int nw, int64_t total, int64_t nreads, int32_t* cnt, int64_t* moff,
                   const MapOut& out, Workspace& ws, cudaStream_t st);
void gather_i64(const int64_t* src, const int64_t* idx, int n, int64_t* out, cudaStream_t st);
// Measured INT32 throughput of this GPU in tera-ops/s (add, max, logic mix).
double int32_probe(cudaStream_t st, int* sink);

}  // namespace clast
