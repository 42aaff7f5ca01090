/*
 * clast_gpu.h -- C ABI of the B200 seed-and-extend engine (libclast_b200.so).
 *
 * The reference (masayano/CLAST) has no plugin API; its in-process seam is
 * the trio of classes its scheduler constructs for every (target window,
 * query window) pair (CHostSchedular.cu:141,169,187,196):
 *
 *   CDeviceHashTable(setting, targetList, t_begin, t_end)      CDeviceHashTable.cuh:17-21
 *   CDeviceSeqList_query(setting, queryList, q_begin, q_end)    CDeviceSeqList_query.cuh:14-18
 *   CDeviceHitList(setting, hashTable, query, t_begin, q_begin) CDeviceHitList.cuh:23-28
 *     + CDeviceHitList::getResult(holder)                        CDeviceHitList.cuh:29
 *
 * clast_index_build() replaces the first, clast_search() the other two.  The
 * whole-job entry points clast_targets_create() / clast_map() replace
 * CHostMapper::getResult + CHostSchedular::search + CHostResultHolder::fixResult
 * (CHostMapper.cu:53-71, CHostSchedular.cu:43-130, CHostResultHolder.cu:75-128)
 * for every RAM load at once, keeping the target indexes resident in HBM.
 *
 * Conventions: every call returns 0 on success or a negative clast_status;
 * nothing aborts or throws across the ABI; the message of the last failure is
 * clast_last_error(ctx).  One context per host thread.  Arrays are plain host
 * pointers; results are allocated by the library and released with
 * clast_hits_free() / clast_map_result_free().
 */
#ifndef CLAST_GPU_H_
#define CLAST_GPU_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum clast_status {
  CLAST_OK = 0,
  CLAST_ERR_ARG = -1,      /* invalid argument (sizes, parameter ranges) */
  CLAST_ERR_CUDA = -2,     /* a CUDA runtime call failed */
  CLAST_ERR_NOMEM = -3,    /* device or host allocation failed */
  CLAST_ERR_INTERNAL = -4, /* internal consistency check failed */
  CLAST_ERR_CANCELLED = -5, /* a served request was cancelled */
  CLAST_PENDING = 1         /* a served request is still queued or running */
} clast_status;

typedef struct clast_ctx clast_ctx;
typedef struct clast_index clast_index;
typedef struct clast_targets clast_targets;

/* The search settings of CHostSetting (CHostSetting.cuh:29-49) that the
 * device path reads.  Defaults (common.hpp:12-43): lmer 15, stride 5,
 * cut_repeat 20, width 100, gap 8, local 0, cutoff 10, K 0.71, lambda 1.37. */
typedef struct clast_params {
  int32_t lmer;        /* 1..31                               */
  int32_t stride;      /* >= 1                                */
  int32_t cut_repeat;  /* -1 = unlimited                      */
  int32_t width;       /* seed-seed distance for the filters  */
  int32_t gap;         /* 2..16: band = 2*gap+1 diagonals     */
  int32_t local;       /* 0 = global alignment, else local    */
  double cutoff;       /* E-value cut-off, -1 = none          */
  double total_db;     /* totalDatabaseSize (CHostSetting.cu:46-58) */
  double K;
  double lambda;
} clast_params;

/* Hit list, structure of arrays (the nine device_vectors of CDeviceHitList,
 * CDeviceHitList.cuh:13-21), in the order the reference produces. */
typedef struct clast_hits {
  int64_t n;
  int32_t* t_id;
  int32_t* t_idx;
  int32_t* q_id;
  int32_t* q_idx;
  int32_t* t_len;
  int32_t* q_len;
  int32_t* match;
  int32_t* score;
  double* evalue;
} clast_hits;

int clast_ctx_create(int device, clast_ctx** out);
void clast_ctx_destroy(clast_ctx* ctx);
const char* clast_last_error(const clast_ctx* ctx);

/* Index of one target window (replaces CDeviceHashTable's constructor).
 * bases: the window's base array exactly as CHostSeqList::getBaseArray(
 * t_begin, t_end) builds it -- every sequence followed by its first l-1
 * bases; gateway: window-relative sequence starts (n_seqs values, first 0);
 * lengths: sequence lengths; t_begin: id of the window's first sequence. */
int clast_index_build(clast_ctx* ctx, const clast_params* p, const char* bases, int64_t n_bases,
                      const int32_t* gateway, const int32_t* lengths, int32_t n_seqs,
                      int32_t t_begin, clast_index** out);
void clast_index_free(clast_index* ix);

/* Hits of one query window against one index (replaces CDeviceSeqList_query
 * + CDeviceHitList + getResult).  q_bases/q_gateway/q_lengths describe the
 * query window as CHostSeqList::getBaseArray(2*qb, 2*qe) does: '+' and '-'
 * strand of every read, each followed by its joint.  q_begin = 2*qb (even). */
int clast_search(clast_ctx* ctx, const clast_index* ix, const clast_params* p,
                 const char* q_bases, int64_t n_qbases, const int32_t* q_gateway,
                 const int32_t* q_lengths, int32_t n_qseqs, int32_t q_begin, clast_hits* out);
void clast_hits_free(clast_hits* h);

/* Allocation-free variant of clast_search.  It has no counterpart in the
 * reference (CDeviceHitList allocates its device_vectors on every call); it
 * serves callers that must not allocate: a process whose device memory is
 * already handed out (a caching allocator that reserved the free HBM, where
 * a cudaMalloc would fail or fragment it), and a serving loop that cannot
 * take the device-wide synchronisation cudaMalloc/cudaFree may cause.
 *
 * Same inputs, same hits in the same order as clast_search.  It calls no
 * cudaMalloc, cudaFree, stream-ordered or pinned allocation and no
 * allocating library routine: all device scratch is carved out of one
 * statically sized buffer of CLAST_NOALLOC_SCRATCH_BYTES inside the library
 * (one per device), and the hits are copied into caller-owned host arrays.
 *   out: t_id .. evalue point at `capacity` elements each (owned by the
 *        caller; never pass them to clast_hits_free); out->n = hit count.
 *   A window whose scratch need exceeds the buffer (its query arrays, or the
 *   seeds / hits it produces) fails with CLAST_ERR_ARG and a message naming
 *   the buffer; more hits than `capacity` fail with CLAST_ERR_ARG and out->n
 *   set to the count needed.  clast_search has neither limit.
 * The scratch is shared by every context of the process on that device, so
 * overlapping calls would race on it: an overlapping call on the same device
 * is rejected with CLAST_ERR_ARG instead.  Each call synchronises its
 * context's stream before returning.  The first call on a device looks up
 * the buffer's address (cudaGetSymbolAddress); make that first call before
 * any stream capture on the device begins. */
#define CLAST_NOALLOC_SCRATCH_BYTES (64ll << 20)
int clast_search_noalloc(clast_ctx* ctx, const clast_index* ix, const clast_params* p,
                         const char* q_bases, int64_t n_qbases, const int32_t* q_gateway,
                         const int32_t* q_lengths, int32_t n_qseqs, int32_t q_begin,
                         int64_t capacity, clast_hits* out);

/* ---- whole job: resident target indexes, every query RAM load at once ---- */

/* One set of sequences, one strand, no joints: record i is
 * bases[offsets[i] .. offsets[i+1]).  offsets is always a host array; bases
 * is a host pointer, or a device pointer on the context's GPU when
 * bases_on_device is 1 (inputs already resident in HBM). */
typedef struct clast_seqs {
  int64_t n_seqs;
  const char* bases;
  const int64_t* offsets; /* n_seqs + 1 values */
  int32_t bases_on_device;
} clast_seqs;

/* Builds and keeps in HBM the index of every target window.  The target
 * records are split into RAM loads (load_sizes[k] records each, in order, as
 * CFASTALoader hands them out) and each load into windows by the rule of
 * moveTargetWindow (CHostSchedular.cu:25-35) with budget t_vram (bases).
 * The index builds are queued on the context's stream and run after the
 * call returns (it waits only for the copy of host-resident bases); the first
 * clast_map on the targets waits for them and reports an index failure, and
 * clast_get_stats shows their times from then on. */
int clast_targets_create(clast_ctx* ctx, const clast_params* p, int32_t t_vram,
                         const clast_seqs* targets, int32_t n_loads, const int64_t* load_sizes,
                         clast_targets** out);
void clast_targets_free(clast_targets* t);

/* Index persistence (no counterpart in the reference, which rebuilds every
 * index for every query RAM load, main.cu:63-89).  clast_targets_save waits for the index builds and
 * writes every window (bases, sequence tables, entries, hash table, filter) to
 * one file; clast_targets_load reads it back onto the context's GPU, ready for
 * clast_map.  Loading fails with CLAST_ERR_ARG when the file was built with
 * other lmer / stride / cut_repeat settings or is not an index file. */
int clast_targets_save(clast_ctx* ctx, const clast_targets* t, const char* path);
int clast_targets_load(clast_ctx* ctx, const clast_params* p, const char* path, clast_targets** out);
/* The checks clast_targets_load makes, on the host only (no device needed):
 * the file's layout version, its settings, and every sequence range, entry
 * range and table payload of every window against its arrays, so that a
 * stale or corrupt file is rejected before any of it is uploaded.  0 when
 * the file would load; otherwise CLAST_ERR_ARG and the reason in err. */
int clast_targets_verify(const clast_params* p, const char* path, char* err, int err_len);

/* Result of clast_map: hits of every query load in the order
 * CHostResultHolder::fixResult leaves them (load by load).  read = record
 * index in the query set; strand 0 '+', 1 '-'; t_load / t_seq locate the
 * target record (t_seq counts within its load).  The arrays live in pinned
 * host memory owned by the context and reused once released: call
 * clast_map_result_free before clast_ctx_destroy. */
typedef struct clast_map_result {
  int64_t n;
  int64_t* load_offsets; /* n_qloads + 1 values: hits of query load k */
  int32_t* read;
  int32_t* strand;
  int32_t* t_load;
  int32_t* t_seq;
  int32_t* t_idx;
  int32_t* q_idx;
  int32_t* t_len;
  int32_t* q_len;
  int32_t* match;
  int32_t* score;
  double* evalue;
  void* owner; /* library-internal: the pinned buffer holding the arrays */
} clast_map_result;

/* Maps every read against every target window.  The reads are split into RAM
 * loads (load_sizes[k] records each) and each load into windows by the rule
 * of moveQueryWindow (CHostSchedular.cu:12-23) with budget q_vram (bases,
 * both strands and joints counted). */
int clast_map(clast_ctx* ctx, const clast_targets* t, const clast_params* p, int32_t q_vram,
              const clast_seqs* reads, int32_t n_loads, const int64_t* load_sizes,
              clast_map_result* out);
void clast_map_result_free(clast_map_result* r);

/* ---- result text: CHostResultHolder::printResult (CHostResultHolder.cu:131-243) ---- */

/* Labels of a set of records: label i = chars[offsets[i] .. offsets[i+1]). */
typedef struct clast_labels {
  int64_t n;
  const char* chars;
  const int64_t* offsets; /* n + 1 values */
} clast_labels;

/* The 10-column tab-separated text of a map result, every query load in
 * order (load k's lines are text[load_offsets[k] .. load_offsets[k+1])).
 * Owned by the library; release with clast_tsv_free. */
typedef struct clast_tsv {
  int64_t n_bytes;
  const char* text;
  int64_t* load_offsets; /* n_loads + 1 values */
  void* owner;           /* library-internal */
} clast_tsv;

/* Formats the hits of a clast_map result as the reference's command line
 * prints them, load by load (printResult is called once per query RAM load):
 *   qLabel qIdx qHitLen strand tLabel tIdx+startIdx tHitLen match(pct%) score E
 * with std::ostream's default number format (%g, 6 significant digits); a
 * hit identical to the last printed line is skipped, and at most num_out
 * lines are printed per run of equal query labels (-1: all).
 *   t:            the targets r was mapped against;
 *   reads:        the labels of every read given to clast_map (same order);
 *   targets:      the labels of every target record given to
 *                 clast_targets_create (all loads, in order);
 *   t_start_idx:  per target record, the '@' start index (null: all 0).
 * r must not have been released yet. */
int clast_format_tsv(clast_ctx* ctx, const clast_targets* t, const clast_map_result* r, int32_t n_loads,
                     const clast_labels* reads, const clast_labels* targets, const int32_t* t_start_idx,
                     int32_t num_out, clast_tsv* out);
void clast_tsv_free(clast_tsv* t);

/* Writes n bytes of buf as a new file at path (created or truncated, as
 * std::ofstream opens printResult's output), with `threads` host threads:
 * the file is sized, mapped, and each thread makes its own range's pages
 * and copies into them (a single write() call holds the file's lock for the
 * whole copy).  Files that cannot be mapped (pipes, devices) get positional
 * writes.  CLAST_ERR_ARG when the file cannot be opened or written. */
int clast_write_file(const char* path, const char* buf, int64_t n, int32_t threads);

/* Hands back the device memory a context keeps for reuse between calls: its
 * scratch buffers, the device copies of released results, and the blocks
 * the device's memory pool holds after stream-ordered frees.  Results and
 * targets still in use are kept.  Waits for the device first. */
int clast_ctx_trim(clast_ctx* ctx);

/* Device-side timing of the last clast_map call in milliseconds (kernels and
 * copies on the context's stream), and how many kernels it launched. */
int clast_last_map_stats(const clast_ctx* ctx, double* device_ms, int64_t* kernel_launches);

/* Measurements of the last clast_targets_create (as of the first clast_map on
 * its targets) and clast_map calls, taken with CUDA events on the context's
 * stream.  Units: milliseconds and counts. */
typedef struct clast_stats {
  double index_ms;           /* index builds, target upload excluded          */
  double index_upload_ms;    /* target host-to-device copies                  */
  double map_ms;             /* clast_map after the reads are resident (result download included) */
  double map_upload_ms;      /* read host-to-device copies                    */
  int64_t index_launches;    /* kernels launched by clast_targets_create      */
  int64_t map_launches;      /* kernels launched by clast_map                 */
  int64_t query_bases;       /* bases of every query strand                   */
  int64_t query_kmers;       /* valid (all-ACGT) query l-mers looked up, summed over target windows */
  int64_t seeds;             /* seeds written (boundary filters applied)      */
  int64_t hits;              /* hits extended by the banded DP               */
  int64_t results;           /* hits returned                                 */
  int64_t dp_cells;          /* sum over hits of (2*gap+1) * (backward + forward rows) */
  double seed_ms;            /* seed_count + seed_write kernels               */
  int64_t seed_launches;
  double dp_ms;              /* banded-DP kernels                             */
  int64_t dp_launches;
  double sort_ms;            /* segmented sorts + seed filter                 */
  double final_ms;           /* result order, duplicate removal, compaction  */
  double index_wall_ms;      /* host wall time of the last clast_targets_create */
  double map_wall_ms;        /* host wall time of the last clast_map          */
  double map_prep_ms;        /* ... of which host preparation before the first copy */
  double map_call_ms;        /* host wall time of the whole clast_map call, buffers released */
  int64_t index_bases;       /* bases of every target window (joints included) of the last targets */
  int64_t index_keys;        /* distinct l-mers kept in those windows' indexes after the repeat cut */
  double dp_order_ms;        /* the DP's hit order (sort or length buckets)  */
  int32_t dp_order_kind;     /* DP order used last: 0 none, 1 sorted by rows, 2 length buckets */
  int32_t dp_queue_chunk;    /* 0: one thread per hit over a full grid; k: persistent grid taking
                                k x 32 hits per warp from a queue              */
  int64_t dp_warp_hits;      /* hits extended one per warp (the longest of their batch) */
} clast_stats;
int clast_get_stats(const clast_ctx* ctx, clast_stats* out);

/* ---- served form: resident targets, requests batched as they arrive ----
 *
 * No counterpart in the reference, whose only mode is the one-shot loop of
 * main.cu:44-89.  A server keeps one clast_targets resident and runs
 * `lanes` batches on the GPU at once, each on its own context (stream,
 * scratch, pinned result buffers) on the targets' device.  A request is a
 * set of reads; it is split into RAM loads of q_ram bases per strand and
 * each load into query windows of q_vram bases, exactly as clast_map does
 * for a query file of those reads, so a request's hits do not depend on the
 * other requests it is batched with.  Admission: a free lane takes the
 * queued requests in arrival order while their bases fit max_batch_bases
 * and the device bytes estimated for every batch in flight fit hbm_budget;
 * requests that arrive while batches run are taken by the next lane that
 * frees up, so their work overlaps the batches already on the GPU. */
typedef struct clast_server clast_server;
typedef struct clast_server_config {
  int32_t lanes;           /* batches in flight at once; 0: 4                         */
  int32_t q_vram;          /* query window budget (bases, moveQueryWindow); 0: 2 MBase */
  int32_t q_ram;           /* RAM load budget per strand (bases); 0: 32 MBase         */
  int32_t reserved0;
  int64_t max_batch_bases; /* read bases of one batch; 0: 8 MBase                     */
  int64_t hbm_budget;      /* device bytes for the batches in flight; 0: free HBM at
                              creation minus hbm_reserve                              */
  int64_t hbm_reserve;     /* device bytes left free when hbm_budget is 0; 0: 2 GiB   */
} clast_server_config;

/* Starts the lanes.  t must have been created on ctx and outlive the server;
 * the server does not use ctx after this call returns. */
int clast_server_create(clast_ctx* ctx, const clast_targets* t, const clast_params* p,
                        const clast_server_config* cfg, clast_server** out);
/* Queues a request (the reads are copied; bases must be host memory) and
 * returns its id at once.  CLAST_ERR_NOMEM when the request alone cannot fit
 * the device budget. */
int clast_server_submit(clast_server* s, const clast_seqs* reads, int64_t* request_id);
/* Waits up to timeout_ms (0: no wait, -1: no limit) for a request.  CLAST_OK
 * and its hits (read = record index within the request, loads = the
 * request's RAM loads) when done; CLAST_PENDING while queued or running;
 * CLAST_ERR_CANCELLED, or the failure's code, otherwise.  The result stays
 * valid until clast_server_release(request_id). */
int clast_server_poll(clast_server* s, int64_t request_id, int32_t timeout_ms, clast_map_result* out);
/* Cancels a request that no lane has taken yet (CLAST_ERR_ARG otherwise). */
int clast_server_cancel(clast_server* s, int64_t request_id);
/* Forgets a finished (done, failed or cancelled) request and frees its result. */
int clast_server_release(clast_server* s, int64_t request_id);
/* Steady-clock nanoseconds (CLOCK_MONOTONIC) at which a request was queued,
 * taken by a lane, and finished (its hits in host memory); 0 = not yet. */
int clast_server_times(clast_server* s, int64_t request_id, int64_t* submit_ns, int64_t* start_ns, int64_t* done_ns);
/* Counters since creation: batches run, requests finished, read bases
 * mapped, and the largest number of requests in one batch. */
typedef struct clast_server_stats {
  int64_t batches, requests, bases, max_batch_requests, queued, running;
  int64_t hbm_budget, hbm_in_flight_max;
} clast_server_stats;
int clast_server_get_stats(clast_server* s, clast_server_stats* out);
const char* clast_server_last_error(const clast_server* s);
/* Cancels every queued request, waits for the batches on the GPU, stops. */
void clast_server_destroy(clast_server* s);

/* Measurement helper, not part of the reference's seam: INT32 throughput of
 * the context's GPU (tera-ops/s) on the banded DP's operation mix (integer
 * add, max and logic; a fused add+max counts as two ops).  The roofline
 * denominator of the DP stage. */
int clast_int32_peak(clast_ctx* ctx, double* tera_ops);

#ifdef __cplusplus
}
#endif

#endif
