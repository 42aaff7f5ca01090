// clast_kernels.cu -- sm_100a kernels of the CLAST seed-and-extend path.
//
// Reference (masayano/CLAST) stages and the kernels that replace them:
//   SRead2bit/SRepelHasOddBase + CDeviceSeqList_query::createHashIndex -> pack_bases, kmer_at
//   CDeviceHashTable (sort_by_key, unique, reduce_by_key, scan, cut)   -> sample_keys,
//       radix_sort_u64, index_*, table_* (hash table + Bloom filter for one-probe lookups)
//   createRawSeedList (binarySearch, writeSeedList)                     -> seed_fused
//   deleteSeedsOnSequenceBoundary                                       -> folded into seed_fused
//   sortSeeds / deletingIsolateSeeds / deleteDuplicateSeeds             -> seed_sort_filter
//   globalAlign* / localAlign* + calculateEvalue + deleteBadHits        -> banded_dp
//   resultSorting + deleteHits_duplicateResult                          -> final_* (per read)
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>

#include "clast_device.cuh"
#include "clast_kernels.cuh"
#include "clast_workspace.h"

namespace clast {

thread_local int64_t g_kernel_launches = 0;

namespace {

constexpr unsigned kFull = 0xffffffffu;

inline int blocks_for(int64_t n, int threads) { return (int)((n + threads - 1) / threads); }
inline int grid_cap(int64_t want) { return (int)(want < 1 ? 1 : (want > 1048576 ? 1048576 : want)); }

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ------------------------------------------------------------------------
// exclusive scan
// ------------------------------------------------------------------------
constexpr int kScanThreads = 256, kScanItems = 8, kScanTile = kScanThreads * kScanItems;

// Element loaders of the scans: an array, or a flag computed from one.
template <class T>
struct ArrayLoad {
  const T* __restrict__ p;
  __device__ __forceinline__ int64_t operator()(int64_t i) const { return (int64_t)p[i]; }
};
struct PositiveLoad {  // 1 where p[i] > 0
  const int32_t* __restrict__ p;
  __device__ __forceinline__ int64_t operator()(int64_t i) const { return p[i] > 0 ? 1 : 0; }
};

// ---- single-pass exclusive scan (decoupled look-back) ----
// Tiles take their index from a counter in launch order, so a tile only waits
// for tiles that have already started.  Each tile publishes its aggregate,
// then its first warp walks back over the predecessors' words, 32 at a time
// (flag in the top two bits: aggregate or inclusive prefix), until it meets an
// inclusive prefix.  The walk waits at most kScanSpinLimit polls per step;
// past that the tile sums the inputs before it directly, so no tile can wait
// for ever.  For non-negative inputs (counts and flags) with sums below 2^62.
constexpr uint64_t kScanAgg = 1ull << 62, kScanInc = 2ull << 62, kScanValue = (1ull << 62) - 1;
constexpr int kScanSpinLimit = 1 << 16;

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

template <class Load>
__global__ void __launch_bounds__(kScanThreads) k_scan_1pass(Load in, int64_t n_in, int64_t n_out,
                                                             int64_t* __restrict__ out,
                                                             unsigned long long* __restrict__ state) {
  __shared__ int64_t warp_tot[kScanThreads / 32];
  __shared__ int64_t s_prefix;
  __shared__ unsigned long long s_tile;
  __shared__ int s_fallback;
  unsigned long long* status = state + 1;  // state[0]: the tile counter
  if (threadIdx.x == 0) s_tile = atomicAdd(state, 1ull);
  __syncthreads();
  const int64_t t = (int64_t)s_tile;
  const int64_t base = t * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t idx = base + i;
    v[i] = (idx < n_in) ? in(idx) : 0;
    sum += v[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  int64_t wpre = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; ++w) {
    const int64_t x = warp_tot[w];
    if (w < warp) wpre += x;
    tot += x;
  }
  if (warp == 0) {
    int64_t run = 0;
    int fallback = 0;
    if (t == 0) {
      if (lane == 0) st_relaxed_u64(status, kScanInc | (unsigned long long)tot);
    } else {
      if (lane == 0) st_relaxed_u64(status + t, kScanAgg | (unsigned long long)tot);
      for (int64_t j = t - 1;; j -= 32) {
        // lane L reads tile j - L; tiles before 0 read as an inclusive 0
        const int64_t jj = j - lane;
        unsigned long long w = jj >= 0 ? ld_relaxed_u64(status + jj) : kScanInc;
        for (int spin = 0; __any_sync(kFull, (w >> 62) == 0) && spin < kScanSpinLimit; ++spin)
          if ((w >> 62) == 0) w = ld_relaxed_u64(status + jj);
        if (__any_sync(kFull, (w >> 62) == 0)) {
          fallback = 1;
          break;
        }
        const unsigned inc = __ballot_sync(kFull, (w & kScanInc) != 0);
        const int last = inc ? __ffs(inc) - 1 : 31;  // nearest inclusive prefix, else the whole step
        int64_t x = lane <= last ? (int64_t)(w & kScanValue) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
        run += x;
        if (inc) break;
      }
    }
    if (lane == 0) {
      s_prefix = run;
      s_fallback = fallback;
    }
  }
  __syncthreads();
  if (s_fallback) {  // a predecessor never published: sum the inputs before this tile
    int64_t part = 0;
    for (int64_t i = threadIdx.x; i < t * kScanTile && i < n_in; i += kScanThreads) part += in(i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
    __syncthreads();
    if (lane == 0) warp_tot[warp] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t run = 0;
      for (int w = 0; w < kScanThreads / 32; ++w) run += warp_tot[w];
      s_prefix = run;
      st_relaxed_u64(status + t, kScanInc | (unsigned long long)(run + tot));
    }
    __syncthreads();
  } else if (threadIdx.x == 0 && t > 0) {
    st_relaxed_u64(status + t, kScanInc | (unsigned long long)(s_prefix + tot));
  }
  int64_t run = s_prefix + wpre + incl - sum;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t idx = base + i;
    if (idx < n_out) out[idx] = run;
    run += v[i];
  }
}

template <class Load>
void scan_1pass(Workspace& ws, Load in, int64_t n, int64_t* out, cudaStream_t st) {
  const int64_t n_out = n + 1;
  const int64_t tiles = (n_out + kScanTile - 1) / kScanTile;
  unsigned long long* state = ws.get<unsigned long long>("scan1_state", tiles + 1);
  CLAST_CK(cudaMemsetAsync(state, 0, (tiles + 1) * sizeof(unsigned long long), st));
  k_scan_1pass<Load><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, n_out, out, state);
  CLAST_LAUNCHED();
}


// ------------------------------------------------------------------------
// packing and query strands
// ------------------------------------------------------------------------
// 2-bit codes and non-ACGT flags of 8 bases (x: 8 bytes, first base in the
// low byte), eight at a time in 64-bit words.  code = ((b >> 1) ^ (b >> 2)) & 3
// maps A C G T to 0 1 2 3; a byte is A/C/G/T iff it equals "ACGT"[code].
// codes16: first base in bits 15..14; bad8: first base in bit 7.
__device__ __forceinline__ void pack8(uint64_t x, uint32_t& codes16, uint32_t& bad8) {
  const uint64_t c = ((x >> 1) ^ (x >> 2)) & 0x0303030303030303ull;
  const uint32_t clo = (uint32_t)c, chi = (uint32_t)(c >> 32);
  // byte-reverse so that the first base ends in the top bits, then gather the
  // eight 2-bit fields
  uint64_t y = ((uint64_t)__byte_perm(clo, 0, 0x0123) << 32) | __byte_perm(chi, 0, 0x0123);
  y = (y | (y >> 6)) & 0x000F000F000F000Full;
  y = (y | (y >> 12)) & 0x000000FF000000FFull;
  codes16 = (uint32_t)((y | (y >> 24)) & 0xFFFF);
  uint32_t bad = 0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t ch = h ? chi : clo;
    const uint32_t sel = (ch & 3u) | ((ch >> 4) & 0x30u) | ((ch >> 8) & 0x300u) | ((ch >> 12) & 0x3000u);
    const uint32_t d = __byte_perm(0x54474341u, 0, sel) ^ (uint32_t)(x >> (32 * h));  // "ACGT"[code] ^ byte
    const uint32_t nz = ((((d & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | d) & 0x80808080u) >> 7;  // 1 per nonzero byte
    bad |= ((nz * 0x08040201u) >> 24 & 0xFu) << (4 * (1 - h));                        // first byte -> bit 3
  }
  bad8 = bad;
}

// One 64-base word per thread: 2-bit codes (first base in the top bits, 32
// per word) and the non-ACGT mask (first base in the top bit).  bases must be
// 16-byte aligned with at least 63 readable bytes past n; bases at or past n
// count as 'N'.
__global__ void k_pack(const char* __restrict__ bases, int64_t n, uint64_t* __restrict__ packed,
                       uint64_t* __restrict__ nmask, int64_t nwords) {
  const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwords) return;
  const int64_t f0 = w * 64;
  uint64_t m = 0, p0 = 0, p1 = 0;
  if (f0 < n) {
    const uint4* src = reinterpret_cast<const uint4*>(bases + f0);
    uint64_t g[8];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const uint4 q = __ldcs(src + v);
      g[2 * v] = ((uint64_t)q.y << 32) | q.x;
      g[2 * v + 1] = ((uint64_t)q.w << 32) | q.z;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int64_t valid = n - (f0 + 8 * k);  // bytes of this group before n
      if (valid < 8) {
        const uint64_t keep = valid <= 0 ? 0ull : ((1ull << (8 * valid)) - 1);
        g[k] = (g[k] & keep) | (0x4E4E4E4E4E4E4E4Eull & ~keep);  // 'N'
      }
      uint32_t c16, b8;
      pack8(g[k], c16, b8);
      m |= (uint64_t)b8 << (56 - 8 * k);
      if (k < 4) p0 |= (uint64_t)c16 << (48 - 16 * k);
      else p1 |= (uint64_t)c16 << (48 - 16 * (k - 4));
    }
  } else {
    m = ~0ull;
  }
  nmask[w] = m;
  packed[2 * w] = p0;
  packed[2 * w + 1] = p1;
}

__device__ __forceinline__ char complement(char c) {
  switch (c) {
    case 'A': return 'T';
    case 'T': return 'A';
    case 'G': return 'C';
    case 'C': return 'G';
    default: return 'N';
  }
}

__global__ void k_strand_meta(const int64_t* __restrict__ off, int64_t n_reads, int64_t* __restrict__ sstart,
                              int32_t* __restrict__ slen) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_reads) return;
  const int64_t a = off[r], len = off[r + 1] - a;
  sstart[2 * r] = 2 * a;
  sstart[2 * r + 1] = 2 * a + len;
  slen[2 * r] = (int32_t)len;
  slen[2 * r + 1] = (int32_t)len;
}

// One warp per read: the '+' strand copy and the reverse complement are both
// coalesced (the reversed writes of a warp still cover one contiguous run).
// The read goes in chunks of 8 x 32 bytes whose loads are all issued before
// the first store, so a short read waits for memory once.
__global__ void k_strands(const char* __restrict__ reads, const int64_t* __restrict__ off, int64_t n_reads,
                          char* __restrict__ out) {
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n_reads) return;
  const int64_t a = off[r], len = off[r + 1] - a;
  char* const fwd = out + 2 * a;
  char* const rev = out + 2 * a + 2 * len - 1;  // base j of the read -> rev[-j]
  for (int64_t j0 = 0; j0 < len; j0 += 8 * 32) {
    char c[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int64_t j = j0 + u * 32 + lane;
      c[u] = j < len ? reads[a + j] : 'N';
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int64_t j = j0 + u * 32 + lane;
      if (j < len) {
        fwd[j] = c[u];
        rev[-j] = complement(c[u]);
      }
    }
  }
}

// Base array of one target window: every sequence followed by its first l-1
// bases (utilAddSequence.cu:15-46); joint bases past a sequence shorter than
// l-1 are 'N'.
__global__ void k_build_window(const char* __restrict__ src, const int64_t* __restrict__ src_off,
                               const int32_t* __restrict__ gw, const int32_t* __restrict__ len, int nseqs,
                               int64_t n, char* __restrict__ out) {
  // 16 output bytes per thread, written as one 16-byte store (out is 16-byte aligned)
  __shared__ int first_seq;
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x * 16;
  if (threadIdx.x == 0) {  // sequence of the block's first base; threads walk forward from it
    int lo = 0, hi = nseqs;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if ((int64_t)gw[mid] <= i0) lo = mid;
      else hi = mid;
    }
    first_seq = lo;
  }
  __syncthreads();
  const int64_t b0 = i0 + (int64_t)threadIdx.x * 16;
  if (b0 >= n) return;
  int lo = first_seq;
  while (lo + 1 < nseqs && (int64_t)gw[lo + 1] <= b0) ++lo;
  unsigned char c[16];
  const int64_t j0 = b0 - gw[lo];
  if (b0 + 16 <= n && j0 + 16 <= (int64_t)len[lo]) {
    // inside one sequence's bases: independent loads
    const char* p = src + src_off[lo] + j0;
#pragma unroll
    for (int k = 0; k < 16; ++k) c[k] = (unsigned char)p[k];
  } else {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int64_t i = b0 + k;
      while (lo + 1 < nseqs && (int64_t)gw[lo + 1] <= i) ++lo;
      const int64_t j = i - gw[lo];
      const int64_t L = len[lo];
      char v = 'N';
      if (i < n) {
        if (j < L) v = src[src_off[lo] + j];
        else if (j - L < L) v = src[src_off[lo] + (j - L)];
      }
      c[k] = (unsigned char)v;
    }
  }
  if (b0 + 16 <= n) {
    uint4 q;
    q.x = c[0] | (c[1] << 8) | (c[2] << 16) | ((uint32_t)c[3] << 24);
    q.y = c[4] | (c[5] << 8) | (c[6] << 16) | ((uint32_t)c[7] << 24);
    q.z = c[8] | (c[9] << 8) | (c[10] << 16) | ((uint32_t)c[11] << 24);
    q.w = c[12] | (c[13] << 8) | (c[14] << 16) | ((uint32_t)c[15] << 24);
    *reinterpret_cast<uint4*>(out + b0) = q;
  } else {
    for (int k = 0; k < 16 && b0 + k < n; ++k) out[b0 + k] = (char)c[k];
  }
}

// ------------------------------------------------------------------------
// index build
// ------------------------------------------------------------------------
// Sample j of the window: its code (4^l for an l-mer with a non-ACGT base).
// pbits > 0: one sortable word code << pbits | j; pbits = 0: the code, with j
// in vals.
__global__ void k_sample_keys(const uint64_t* __restrict__ packed, const uint64_t* __restrict__ nmask,
                              int64_t ns, int stride, int l, int pbits, uint64_t* __restrict__ items,
                              int32_t* __restrict__ vals) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ns) return;
  uint64_t key;
  const uint64_t c = kmer_at(packed, nmask, j * stride, l, key) ? order_code(key, l) : (1ull << (2 * l));
  if (pbits > 0) {
    items[j] = (c << pbits) | (uint64_t)j;
  } else {
    items[j] = c;
    vals[j] = (int32_t)j;
  }
}

// keys / vals of the sorted words, and head[i] = whether key i is valid
// (< bound) and differs from key i - 1.
__global__ void k_split_items(const uint64_t* __restrict__ items, int64_t n, int pbits, uint64_t bound,
                              uint64_t* __restrict__ keys, int32_t* __restrict__ vals, int32_t* __restrict__ head) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t v = items[i];
  const uint64_t k = v >> pbits;
  keys[i] = k;
  vals[i] = (int32_t)(v & ((1ull << pbits) - 1));
  head[i] = (k < bound && (i == 0 || (items[i - 1] >> pbits) != k)) ? 1 : 0;
}

// ---- LSD radix sort of 64-bit words by a bit range, 8 bits per pass ----
// A block takes a tile of kRsTile consecutive words; warp w owns words
// [w * kRsWarpItems, (w + 1) * kRsWarpItems) of it.  Each pass: per-block digit
// counts (k_rs_hist), one scan of the counts laid out digit-major, then
// k_rs_scatter ranks the tile stably in shared memory and writes every
// digit's run out contiguously.  Ranking takes one step per 32 words: the
// lanes holding the same digit are found with eight ballots (one per digit
// bit), the lowest of them adds the group's size to the warp's counter of that
// digit, and each lane's rank is the counter's old value plus the lanes of its
// group below it.
constexpr int kRsThreads = 256, kRsItems = 16, kRsTile = kRsThreads * kRsItems;
constexpr int kRsWarps = kRsThreads / 32, kRsWarpItems = 32 * kRsItems;

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const uint64_t* __restrict__ keys, int64_t n, int shift,
                                                        uint32_t* __restrict__ hist, int nblocks) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRsTile;
#pragma unroll 4
  for (int r = 0; r < kRsItems; ++r) {
    const int64_t idx = base + r * kRsThreads + threadIdx.x;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255], 1u);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Lanes of the warp whose 8-bit digit equals this lane's, among the lanes in `among`.
__device__ __forceinline__ unsigned digit_peers(unsigned d, unsigned among) {
  unsigned peers = among;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const unsigned bit = (d >> b) & 1u;
    const unsigned bb = __ballot_sync(kFull, bit);
    peers &= bit ? bb : ~bb;
  }
  return peers;
}

// PAY: a 32-bit value travels with every word (vin -> vout).  Dynamic shared
// memory: the staged tile, kRsTile words (+ kRsTile values).
template <bool PAY>
__global__ void __launch_bounds__(kRsThreads, 3) k_rs_scatter(const uint64_t* __restrict__ kin,
                                                           const int32_t* __restrict__ vin,
                                                           uint64_t* __restrict__ kout, int32_t* __restrict__ vout,
                                                           int64_t n, int shift, const int64_t* __restrict__ offs,
                                                           int nblocks) {
  __shared__ uint32_t wc[kRsWarps][256];  // per-warp digit counters, then the warps' run starts
  __shared__ uint32_t tile_start[256];
  __shared__ uint32_t wsum[kRsWarps];
  __shared__ int64_t goff[256];
  extern __shared__ uint64_t stage[];
  int32_t* stage_v = reinterpret_cast<int32_t*>(stage + kRsTile);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  goff[tid] = offs[(int64_t)tid * nblocks + blockIdx.x];
#pragma unroll
  for (int w = 0; w < kRsWarps; ++w) wc[w][tid] = 0;
  const int64_t base = (int64_t)blockIdx.x * kRsTile + (int64_t)warp * kRsWarpItems;
  const unsigned lt = lanemask_lt();
  uint64_t k[kRsItems];
  int32_t v[PAY ? kRsItems : 1];
#pragma unroll
  for (int r = 0; r < kRsItems; ++r) {
    const int64_t idx = base + r * 32 + lane;
    k[r] = idx < n ? kin[idx] : 0ull;
    if (PAY) v[r] = idx < n ? vin[idx] : 0;
  }
  __syncthreads();
  // stable ranks within the warp's runs, two 16-bit ranks per register
  uint32_t rk[kRsItems / 2];
#pragma unroll
  for (int r = 0; r < kRsItems; ++r) {
    const bool ok = base + r * 32 + lane < n;
    const unsigned d = (unsigned)(k[r] >> shift) & 255u;
    const unsigned peers = digit_peers(d, __ballot_sync(kFull, ok));
    const int leader = __ffs(peers) - 1;  // -1 only for a lane past n
    uint32_t old = 0;
    if (ok && lane == leader) old = atomicAdd(&wc[warp][d], (uint32_t)__popc(peers));
    old = __shfl_sync(kFull, old, leader & 31);
    const uint32_t rank = old + (uint32_t)__popc(peers & lt);
    if (r & 1) rk[r >> 1] |= rank << 16;
    else rk[r >> 1] = rank;
  }
  __syncthreads();
  // digit d = tid: tile-wide start (exclusive scan over digits), then the
  // start of each warp's run of that digit
  uint32_t tot = 0;
#pragma unroll
  for (int w = 0; w < kRsWarps; ++w) tot += wc[w][tid];
  uint32_t incl = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  uint32_t start = incl - tot;
  for (int w = 0; w < warp; ++w) start += wsum[w];
  tile_start[tid] = start;
#pragma unroll
  for (int w = 0; w < kRsWarps; ++w) {
    const uint32_t c = wc[w][tid];
    wc[w][tid] = start;
    start += c;
  }
  __syncthreads();
  // stage the tile in sorted order
#pragma unroll
  for (int r = 0; r < kRsItems; ++r) {
    if (base + r * 32 + lane < n) {
      const unsigned d = (unsigned)(k[r] >> shift) & 255u;
      const uint32_t at = wc[warp][d] + ((rk[r >> 1] >> (16 * (r & 1))) & 0xffffu);
      stage[at] = k[r];
      if (PAY) stage_v[at] = v[r];
    }
  }
  __syncthreads();
  // digit runs out, contiguous
  const int64_t tile0 = (int64_t)blockIdx.x * kRsTile;
  const int valid = (int)min((int64_t)kRsTile, n - tile0);
  for (int i = tid; i < valid; i += kRsThreads) {
    const uint64_t w = stage[i];
    const unsigned d = (unsigned)((w >> shift) & 255);
    const int64_t at = goff[d] + (i - (int)tile_start[d]);
    kout[at] = w;
    if (PAY) vout[at] = stage_v[i];
  }
}

__global__ void k_count_below(const uint64_t* __restrict__ keys, int64_t n, uint64_t bound,
                              int64_t* __restrict__ out) {
  int64_t lo = 0, hi = n;  // first key >= bound in a sorted array
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] < bound) lo = mid + 1;
    else hi = mid;
  }
  *out = lo;
}

// The index build runs without host synchronisation: kernels cover the n
// samples (an upper bound) and read the counts that matter from the device
// (*nv valid samples; *nu = hpos[n] unique keys, as the scans end with the
// total and every flag past the valid range is 0).
__global__ void k_index_heads(const uint64_t* __restrict__ k, int64_t n, uint64_t bound,
                              int32_t* __restrict__ head) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) head[i] = (k[i] < bound && (i == 0 || k[i] != k[i - 1])) ? 1 : 0;
}

__global__ void k_index_unique(const uint64_t* __restrict__ k, const int32_t* __restrict__ head,
                               const int64_t* __restrict__ hpos, int64_t n, const int64_t* __restrict__ nv_dev,
                               uint64_t* __restrict__ ukeys, int64_t* __restrict__ ufirst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nv = *nv_dev;
  if (i < n && head[i]) {
    ukeys[hpos[i]] = k[i];
    ufirst[hpos[i]] = i;
  }
  if (i == 0) ufirst[hpos[nv]] = nv;
}

__global__ void k_index_keep(const int32_t* __restrict__ vals, const int64_t* __restrict__ hpos,
                             const int64_t* __restrict__ ufirst, int64_t n, const int64_t* __restrict__ nv_dev,
                             int stride, int l, int cut, const int32_t* __restrict__ gw,
                             const int32_t* __restrict__ len, int nseqs, int32_t* __restrict__ keep,
                             int2* __restrict__ resolved) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (i >= *nv_dev) {
    keep[i] = 0;
    return;
  }
  const int64_t u = hpos[i + 1] - 1;
  const int64_t cnt = ufirst[u + 1] - ufirst[u];
  const bool pass = (cut == -1) || (cnt < (int64_t)cut);  // removeRepeatedSequence
  const int64_t pos = (int64_t)vals[i] * stride;
  int lo = 0, hi = nseqs;  // last sequence starting at or before pos
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if ((int64_t)gw[mid] <= pos) lo = mid;
    else hi = mid;
  }
  const int tidx = (int)(pos - gw[lo]);
  const bool joint = (int64_t)tidx + l > (int64_t)len[lo];  // onTargetBoundary
  keep[i] = (pass && !joint) ? 1 : 0;
  resolved[i] = make_int2(lo, tidx);
}

__global__ void k_index_entries(const int32_t* __restrict__ keep, const int64_t* __restrict__ kpos,
                                const int2* __restrict__ resolved, int64_t n, int2* __restrict__ entries) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && keep[i]) entries[kpos[i]] = resolved[i];
}

__global__ void k_index_buckets(const int64_t* __restrict__ ufirst, const int64_t* __restrict__ kpos,
                                int64_t n, const int64_t* __restrict__ nu_dev, int32_t* __restrict__ ustart,
                                int32_t* __restrict__ ucnt) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (k >= *nu_dev) {
    ucnt[k] = 0;
    return;
  }
  const int64_t a = kpos[ufirst[k]], b = kpos[ufirst[k + 1]];
  ustart[k] = (int32_t)a;
  ucnt[k] = (int32_t)(b - a);
}

// ---- hash table of the index, placed without atomics ----
// The unique codes arrive ascending, so their home records do too; with
// r = rank among the kept codes, linear probing puts code r at
// max(home_r, pos_{r-1} + 1) = r + max_{j <= r}(home_j - j).

// The running maximum is taken over the unique codes k (not over the ranks):
// for kept code k it equals max over kept j <= k of home_j - rank_j.  Codes
// without entries (repeat cut, joints only, past the keys: ucnt 0) count as
// INT64_MIN.
struct SlackLoad {
  const uint64_t* __restrict__ ucode;
  const int32_t* __restrict__ ucnt;
  const int64_t* __restrict__ rank;
  int l;
  uint32_t nbuckets;
  __device__ __forceinline__ int64_t operator()(int64_t k) const {
    return ucnt[k] > 0 ? record_home(ucode[k], l, nbuckets) - rank[k] : INT64_MIN;
  }
};

__global__ void k_table_place(const uint64_t* __restrict__ ucode, const int32_t* __restrict__ ustart,
                              const int32_t* __restrict__ ucnt, const int2* __restrict__ entries,
                              const int64_t* __restrict__ rank, const int64_t* __restrict__ run_max, int64_t nu,
                              ulonglong2* __restrict__ table, int64_t n_records, uint32_t* __restrict__ filter,
                              int fshift, unsigned long long* __restrict__ failed) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nu) return;
  const int c = ucnt[k];
  if (c <= 0) return;
  const uint64_t code = ucode[k];
  const uint64_t h = key_hash(code);
  atomicOr(filter + filter_word(h, fshift), filter_mask(h));
  uint64_t payload;
  if (c == 1) {
    const int2 e = entries[ustart[k]];
    payload = ((uint64_t)(uint32_t)e.x << 32) | (uint32_t)e.y;
  } else {
    payload = kMulti | ((uint64_t)(uint32_t)ustart[k] << 32) | (uint32_t)c;
  }
  const int64_t pos = rank[k] + run_max[k];
  if (pos >= 0 && pos < n_records) table[pos] = make_ulonglong2(code, payload);
  else atomicAdd(failed, 1ull);  // unreachable: positions rise to the last one, which the table holds
}

// ---- inclusive running maximum (int64) ----
template <class Load>
__global__ void __launch_bounds__(kScanThreads) k_maxscan_tiles(Load in, int64_t n, int64_t* __restrict__ out,
                                                                int64_t* __restrict__ tile_max) {
  __shared__ int64_t warp_max[kScanThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t m = INT64_MIN;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t idx = base + i;
    v[i] = (idx < n) ? in(idx) : INT64_MIN;
    m = v[i] > m ? v[i] : m;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t incl = m;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o && y > incl) incl = y;
  }
  if (lane == 31) warp_max[warp] = incl;
  __syncthreads();
  int64_t wpre = INT64_MIN, tot = INT64_MIN;
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; ++w) {
    const int64_t t = warp_max[w];
    if (w < warp && t > wpre) wpre = t;
    if (t > tot) tot = t;
  }
  int64_t run = __shfl_up_sync(kFull, incl, 1);
  if (lane == 0) run = INT64_MIN;
  if (wpre > run) run = wpre;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t idx = base + i;
    if (v[i] > run) run = v[i];
    if (idx < n) out[idx] = run;
  }
  if (threadIdx.x == 0) tile_max[blockIdx.x] = tot;
}

__global__ void k_maxscan_apply(int64_t* __restrict__ out, int64_t n, const int64_t* __restrict__ tile_run) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t t = i / kScanTile;
  if (t > 0 && tile_run[t - 1] > out[i]) out[i] = tile_run[t - 1];
}

// ------------------------------------------------------------------------
// seeds
// ------------------------------------------------------------------------
// Seeding in one pass, one warp per strand.  The strand's l-mers go in rounds
// of 32 * kSeedPerLane; in a round lane L takes the kSeedPerLane consecutive
// l-mers from L * kSeedPerLane, so it reads their 2-bit words and N flags once
// and shifts each key out of them.  The lookups of a round are issued
// together, level by level (2-bit words and N flags → filter words → home
// buckets), so a strand waits about one latency per level.  Round 0's results
// are staged for the write pass while the range reservation is in flight (one
// round covers 160 l-mers: a 164 bp strand); later rounds are looked up again
// when written.  The strand's seeds get one
// contiguous range from an atomic cursor; if the range would pass `cap`,
// nothing is written and the host reruns with a larger buffer (the cursor then
// holds the exact total).  Seeds are written in l-mer order, so the seeds of a
// strand on one diagonal arrive already sorted.
constexpr int kSeedPerLane = 5;
constexpr int kSeedRound = 32 * kSeedPerLane;
constexpr int kSeedParts = 32;

// Both records of a home bucket: one 256-bit streaming load (sm_100), the
// address 32-byte aligned (home records are even, the table 256-byte aligned).
__device__ __forceinline__ void ld_bucket(const ulonglong2* a, uint64_t& c0, uint64_t& p0, uint64_t& c1,
                                          uint64_t& p1) {
  asm volatile("ld.global.cs.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(c0), "=l"(p0), "=l"(c1), "=l"(p1) : "l"(a));
}

// (hi << s) | (lo >> (64 - s)) for s in [0, 63]: the 64 bits from bit s of hi:lo
__device__ __forceinline__ uint64_t funnel64(uint64_t hi, uint64_t lo, int s) {
  return (hi << s) | ((lo >> 1) >> (63 - s));
}

// Payloads of the l-mers qi = r0 + lane * P + i (i < P) of a strand; invalid or
// absent ones get kNoPayload (the key search of krnlBinarySearch.cu:3-33 and
// the bucket read of writeSeedList).  Returns the number of valid l-mers.
template <bool SMALL>
__device__ __forceinline__ int round_lookup(const QueryView& q, const IndexView& ix, int64_t st, int nk, int r0,
                                            int lane, uint64_t (&pl)[kSeedPerLane]) {
  constexpr int P = kSeedPerLane;
  const int q0 = r0 + lane * P;
  const int nv = max(0, min(P, nk - q0));  // valid l-mer slots of this lane
  uint64_t code[P];
  uint32_t vmask = 0;
  if (nv > 0) {
    const int64_t f = st + q0;
    // The lane's P l-mers span P - 1 + l <= 35 bases from f: their 2-bit words
    // and non-ACGT flags are read in one batch.  An l-mer with a non-ACGT base
    // is not looked up (SRepelHasOddBase).
    vmask = (1u << nv) - 1;
    if (SMALL) {
      // 16-base units j0 .. j0 + 2 of the codes, 32-base units k0, k0 + 1 of
      // the flags (unit j = 32-bit element j ^ 1)
      const uint32_t* p32 = reinterpret_cast<const uint32_t*>(q.packed);
      const uint32_t* n32 = reinterpret_cast<const uint32_t*>(q.nmask);
      const int64_t j0 = f >> 4, k0 = f >> 5;
      const uint32_t u0 = __ldcs(p32 + (j0 ^ 1)), u1 = __ldcs(p32 + ((j0 + 1) ^ 1)),
                     u2 = __ldcs(p32 + ((j0 + 2) ^ 1));
      const uint32_t m0 = __ldcs(n32 + (k0 ^ 1)), m1 = __ldcs(n32 + ((k0 + 1) ^ 1));
      const uint32_t nflag = __funnelshift_l(m1, m0, (int)(f & 31));  // base f in the top bit
      const int o = 2 * (int)(f & 15);
      const uint32_t mask = (2 * ix.l == 32) ? ~0u : ((1u << (2 * ix.l)) - 1);
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const int bo = o + 2 * i;
        const uint32_t x = bo < 32 ? __funnelshift_l(u1, u0, bo) : __funnelshift_l(u2, u1, bo - 32);
        const uint32_t key = x >> (32 - 2 * ix.l);
        code[i] = (uint32_t)(key * (uint32_t)0x6659FD93u) & mask;  // order_code for l <= 16
        if ((nflag << i) >> (32 - ix.l)) vmask &= ~(1u << i);
      }
    } else {
      // 32-base words w0 .. w0 + 2 of the codes, 64-base words k0, k0 + 1 of the flags
      const int64_t w0 = f >> 5, k0 = f >> 6;
      const uint64_t u0 = ld_stream(q.packed + w0), u1 = ld_stream(q.packed + w0 + 1),
                     u2 = ld_stream(q.packed + w0 + 2);
      const uint64_t nflag = funnel64(ld_stream(q.nmask + k0), ld_stream(q.nmask + k0 + 1), (int)(f & 63));
      const int o = 2 * (int)(f & 31);
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const int bo = o + 2 * i;  // < 2 * (31 + P)
        const uint64_t x = bo < 64 ? funnel64(u0, u1, bo) : funnel64(u1, u2, bo - 64);
        code[i] = order_code(x >> (64 - 2 * ix.l), ix.l);
        if ((nflag << i) >> (64 - ix.l)) vmask &= ~(1u << i);
      }
    }
  }
  uint32_t fw[P], fm[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    const uint64_t h = key_hash(code[i]);
    fm[i] = filter_mask(h);
    fw[i] = ((vmask >> i) & 1u) ? __ldg(ix.filter + filter_word(h, ix.fshift)) : 0u;
  }
  // The home bucket (records home and home + 1, one aligned 32-byte sector)
  // in one load; only keys displaced past it probe further.
  uint64_t c0[P], p0[P], c1[P], p1[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    const bool pass = ((vmask >> i) & 1u) && (fw[i] & fm[i]) == fm[i];
    c0[i] = 0ull;
    p0[i] = kNoPayload;
    c1[i] = 0ull;
    p1[i] = kNoPayload;
    if (pass)
      ld_bucket(ix.table + (SMALL ? record_home16((uint32_t)code[i], ix.l, ix.nbuckets)
                                  : record_home(code[i], ix.l, ix.nbuckets)),
                c0[i], p0[i], c1[i], p1[i]);
  }
#pragma unroll
  for (int i = 0; i < P; ++i) {
    if (c0[i] == code[i] || p0[i] == kNoPayload) pl[i] = p0[i];
    else if (c1[i] == code[i] || p1[i] == kNoPayload) pl[i] = p1[i];
    else pl[i] = table_probe(ix, code[i], record_home(code[i], ix.l, ix.nbuckets) + 2);
  }
  return __popc(vmask);
}

// Writes the seed of entry e (sequence within window, index within sequence)
// for l-mer qi at w; tlen = length of sequence e.x (global mode only).
__device__ __forceinline__ void seed_store(int2 e, int qi, int tlen, int gap, int local, int qlen, int64_t w,
                                           int& valid, uint64_t* __restrict__ skey, uint32_t* __restrict__ sq) {
  const int s0 = e.y - qi;  // tHitStartIdx, is_onCorner
  const bool drop = !local && ((s0 + gap < 0) || (s0 + qlen - gap > tlen));
  // streaming stores: the seeds must not evict the filter from L2
  __stcs(reinterpret_cast<unsigned long long*>(skey + w),
         drop ? kDroppedSeed : (((uint64_t)(uint32_t)e.x << 32) | ((uint32_t)s0 ^ 0x80000000u)));
  __stcs(sq + w, (uint32_t)qi);
  valid += drop ? 0 : 1;
}

// Writes the c = payload_count(pl) seeds of l-mer qi at w onwards.
__device__ __forceinline__ void seed_put(const IndexView& ix, const TargetView& t, int gap, int local, int qlen,
                                         int qi, uint64_t pl, int64_t w, int& valid, uint64_t* __restrict__ skey,
                                         uint32_t* __restrict__ sq) {
  const int c = payload_count(pl);
  const bool multi = (pl & kMulti) != 0;
  const int us = (int)(pl >> 32) & 0x7fffffff;
  for (int i = 0; i < c; ++i) {
    const int2 e = multi ? __ldcs(ix.entries + us + i) : make_int2((int)(pl >> 32), (int)(uint32_t)pl);
    seed_store(e, qi, local ? 0 : t.lengths[e.x], gap, local, qlen, w + i, valid, skey, sq);
  }
}

// Exclusive prefix sum over the warp; *total = the warp's sum.
__device__ __forceinline__ int warp_excl_scan(int v, int lane, int* total) {
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += y;
  }
  *total = __shfl_sync(kFull, incl, 31);
  return incl - v;
}

// Writes a round's seeds (lane L's l-mers r0 + L*P .. in order, lanes in
// order) from w onwards and advances w past them.  When every l-mer of the
// round has at most one entry, the payloads go through the warp's slice of
// shared memory (stage_pl / stage_qi, kSeedRound entries) so that lane j
// writes seed j; otherwise each lane writes its own.
__device__ __forceinline__ void round_emit(const IndexView& ix, const TargetView& t, int gap, int local, int qlen,
                                           int r0, int lane, const uint64_t (&pl)[kSeedPerLane], int64_t& w,
                                           int& valid, uint64_t* __restrict__ skey, uint32_t* __restrict__ sq,
                                           uint64_t* stage_pl, int32_t* stage_qi) {
  int cnt = 0;
  bool multi = false;
#pragma unroll
  for (int i = 0; i < kSeedPerLane; ++i) {
    const int c = payload_count(pl[i]);
    cnt += c;
    multi |= c > 1;
  }
  int round_total;
  const int excl = warp_excl_scan(cnt, lane, &round_total);
  if (!__any_sync(kFull, multi)) {
    int k = excl;
#pragma unroll
    for (int i = 0; i < kSeedPerLane; ++i)
      if (pl[i] != kNoPayload) {
        stage_pl[k] = pl[i];
        stage_qi[k] = r0 + lane * kSeedPerLane + i;
        ++k;
      }
    __syncwarp();
    for (int j = lane; j < round_total; j += 32) seed_put(ix, t, gap, local, qlen, stage_qi[j], stage_pl[j], w + j,
                                                         valid, skey, sq);
    __syncwarp();
  } else {
    int64_t wl = w + excl;
#pragma unroll
    for (int i = 0; i < kSeedPerLane; ++i)
      if (pl[i] != kNoPayload) {
        seed_put(ix, t, gap, local, qlen, r0 + lane * kSeedPerLane + i, pl[i], wl, valid, skey, sq);
        wl += payload_count(pl[i]);
      }
  }
  w += round_total;
}

constexpr int kSeedFusedThreads = 64;  // two strands per block: blocks retire at a finer grain than with four
constexpr int kSeedPrefetchBlocks = 2048;

// The seed buffer is split into kSeedParts partitions of part_cap seeds, each
// with its own cursor; strand s takes its range in partition s % kSeedParts, so
// the range reservations of neighbouring warps hit different counters.
// SMALL: l <= 16, keys read with 32-bit funnel shifts.
template <bool SMALL>
__global__ void __launch_bounds__(kSeedFusedThreads, SMALL ? 16 : 12) k_seed_fused(QueryView q, IndexView ix, TargetView t, int gap,
                                                                   int local, unsigned long long* __restrict__ cursor,
                                                                   unsigned long long* __restrict__ n_kmers,
                                                                   int64_t* __restrict__ off, int32_t* __restrict__ cnt,
                                                                   int32_t* __restrict__ nvalid,
                                                                   uint64_t* __restrict__ skey,
                                                                   uint32_t* __restrict__ sq, int64_t part_cap) {
  constexpr int P = kSeedPerLane;
  __shared__ uint64_t stage_pl[kSeedFusedThreads / 32][kSeedRound];
  __shared__ int32_t stage_qi[kSeedFusedThreads / 32][kSeedRound];
  const int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  if (s >= q.nstrands) return;
  const int64_t st = q.start[s];
  const int qlen = q.len[s];
  const int nk = qlen - ix.l + 1;
  // L2 prefetch for the block kSeedPrefetchBlocks later: its strand table
  // entries and, estimated from this strand's start and the mean strand
  // length, its 2-bit words and N flags, so that its first loads hit L2.
  // Every address stays inside its array.
  if (wib == 0 && lane < 5) {
    const int64_t sp = ((int64_t)blockIdx.x + kSeedPrefetchBlocks) * (kSeedFusedThreads / 32);
    if (sp < q.nstrands && q.n > 0) {
      const int64_t f = min(q.n - 1, st + (sp - s) * (q.n / q.nstrands));
      const void* a = lane == 0 ? (const void*)(q.start + sp)
                    : lane == 1 ? (const void*)(q.len + sp)
                    : lane == 4 ? (const void*)(q.nmask + (f >> 6))
                                : (const void*)(q.packed + min((f >> 5) + 16 * (lane - 2), q.n / 32 + 3));
      asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
    }
  }
  uint64_t pl0[P];
  int valid_kmers = round_lookup<SMALL>(q, ix, st, nk, 0, lane, pl0);
  int lane_cnt = 0;
  bool multi0 = false;
#pragma unroll
  for (int i = 0; i < P; ++i) {
    const int c = payload_count(pl0[i]);
    lane_cnt += c;
    multi0 |= c > 1;
  }
  // Round 0 is staged before its range is known: in the single-entry case
  // lane j takes seed j of the round and reads its sequence length now, so
  // that the load overlaps the range reservation below.
  int rt0;
  const int excl0 = warp_excl_scan(lane_cnt, lane, &rt0);
  const bool simple0 = !__any_sync(kFull, multi0);
  uint64_t* const spl = stage_pl[wib];
  int32_t* const sqi = stage_qi[wib];
  uint64_t pl_j = kNoPayload;
  int qi_j = 0, tl_j = 0;
  if (simple0) {
    int k = excl0;
#pragma unroll
    for (int i = 0; i < P; ++i)
      if (pl0[i] != kNoPayload) {
        spl[k] = pl0[i];
        sqi[k] = lane * P + i;
        ++k;
      }
    __syncwarp();
    if (lane < rt0) {
      pl_j = spl[lane];
      qi_j = sqi[lane];
      if (!local) tl_j = t.lengths[(int)(pl_j >> 32)];
    }
  } else {
    // the payloads wait in the lane's own stage slots
#pragma unroll
    for (int i = 0; i < P; ++i) spl[lane * P + i] = pl0[i];
  }
  for (int r0 = kSeedRound; r0 < nk; r0 += kSeedRound) {
    uint64_t pl[P];
    valid_kmers += round_lookup<SMALL>(q, ix, st, nk, r0, lane, pl);
#pragma unroll
    for (int i = 0; i < P; ++i) lane_cnt += payload_count(pl[i]);
  }
  const int total = (int)__reduce_add_sync(kFull, (unsigned)lane_cnt);
  valid_kmers = (int)__reduce_add_sync(kFull, (unsigned)valid_kmers);
  const int part = (int)(s % kSeedParts);
  unsigned long long rel = 0;
  if (lane == 0) {
    if (valid_kmers) atomicAdd(n_kmers + part, (unsigned long long)valid_kmers);
    rel = total ? atomicAdd(&cursor[part], (unsigned long long)total) : 0ull;
  }
  rel = __shfl_sync(kFull, rel, 0);
  const unsigned long long base = (unsigned long long)part * (unsigned long long)part_cap + rel;
  if (lane == 0) {
    off[s] = (int64_t)base;
    cnt[s] = total;
  }
  const int64_t cap = (int64_t)(part + 1) * part_cap;
  if (total == 0 || (int64_t)(base + total) > cap) {
    if (lane == 0) nvalid[s] = 0;
    return;
  }
  int valid = 0;
  int64_t w = (int64_t)base;
  if (simple0) {
    if (lane < rt0)
      seed_store(make_int2((int)(pl_j >> 32), (int)(uint32_t)pl_j), qi_j, tl_j, gap, local, qlen, w + lane, valid,
                 skey, sq);
    for (int j = lane + 32; j < rt0; j += 32) seed_put(ix, t, gap, local, qlen, sqi[j], spl[j], w + j, valid, skey, sq);
  } else {
    int64_t wl = w + excl0;
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const uint64_t pl = spl[lane * P + i];
      if (pl != kNoPayload) {
        seed_put(ix, t, gap, local, qlen, lane * P + i, pl, wl, valid, skey, sq);
        wl += payload_count(pl);
      }
    }
  }
  __syncwarp();
  w += rt0;
  for (int r0 = kSeedRound; r0 < nk; r0 += kSeedRound) {
    uint64_t pl[P];
    round_lookup<SMALL>(q, ix, st, nk, r0, lane, pl);
    round_emit(ix, t, gap, local, qlen, r0, lane, pl, w, valid, skey, sq, spl, sqi);
  }
  valid = (int)__reduce_add_sync(kFull, (unsigned)valid);
  if (lane == 0) nvalid[s] = valid;
}

// ------------------------------------------------------------------------
// Seeding of several target windows in one pass over the query
// ------------------------------------------------------------------------
// One warp per strand as in k_seed_fused, but every round's l-mers are looked
// up in NW target windows at once: the 2-bit words and N flags are read once
// for all windows, the NW filter words of every l-mer are loaded together, and
// the l-mers that pass a filter are listed in the warp's shared memory (code,
// window, l-mer) so that the 32 lanes share the bucket reads evenly (about one
// per lane and window in a round of 160 l-mers) instead of each lane reading
// the buckets of its own l-mers.  Payloads land in shared memory, one slot per
// (window, l-mer); the emission of each window's seeds is round_emit's.
// A strand reserves its range in every window with one atomic per window,
// issued by lanes 0..NW-1 together.
template <int NW>
struct SeedSmem {
  uint64_t pl[NW][kSeedRound];  // payload of (window, l-mer) of the current round
  union {
    struct {
      uint64_t code[NW * kSeedRound];
      uint16_t tag[NW * kSeedRound];  // window << 8 | l-mer within the round
    } list;                           // the l-mers that passed a window's filter
    struct {
      uint64_t pl[kSeedRound];
      int32_t qi[kSeedRound];
    } stage;  // round_emit's staging
  } u;
};

// Payload of the key of code c in the table of one window (home bucket in one
// 32-byte read, then linear probing).
template <bool SMALL>
__device__ __forceinline__ uint64_t bucket_payload(const IndexView& ix, uint64_t c) {
  const int64_t home = SMALL ? record_home16((uint32_t)c, ix.l, ix.nbuckets) : record_home(c, ix.l, ix.nbuckets);
  uint64_t c0, p0, c1, p1;
  ld_bucket(ix.table + home, c0, p0, c1, p1);
  if (c0 == c || p0 == kNoPayload) return p0;
  if (c1 == c || p1 == kNoPayload) return p1;
  return table_probe(ix, c, home + 2);
}

// Looks up the l-mers r0 + lane * P + i (i < P) of a strand in the NW windows.
// When `keep`, their payloads go to sm.pl (kNoPayload for invalid or absent
// l-mers); cnt[w] adds the entries of the l-mers this lane resolved in window
// w.  Returns the number of valid l-mers of this lane.
template <bool SMALL, int NW>
__device__ __forceinline__ int round_lookup_multi(const QueryView& q, const SeedWins& W, int64_t st, int nk, int r0,
                                                  int lane, SeedSmem<NW>& sm, bool keep, int (&cnt)[NW]) {
  constexpr int P = kSeedPerLane;
  const int l = W.w[0].ix.l;
  const int q0 = r0 + lane * P;
  const int nv = max(0, min(P, nk - q0));
  uint64_t code[P];
  uint32_t vmask = 0;
#pragma unroll
  for (int i = 0; i < P; ++i) code[i] = 0;
  if (nv > 0) {
    const int64_t f = st + q0;
    vmask = (1u << nv) - 1;
    if (SMALL) {
      const uint32_t* p32 = reinterpret_cast<const uint32_t*>(q.packed);
      const uint32_t* n32 = reinterpret_cast<const uint32_t*>(q.nmask);
      const int64_t j0 = f >> 4, k0 = f >> 5;
      const uint32_t u0 = __ldcs(p32 + (j0 ^ 1)), u1 = __ldcs(p32 + ((j0 + 1) ^ 1)),
                     u2 = __ldcs(p32 + ((j0 + 2) ^ 1));
      const uint32_t m0 = __ldcs(n32 + (k0 ^ 1)), m1 = __ldcs(n32 + ((k0 + 1) ^ 1));
      const uint32_t nflag = __funnelshift_l(m1, m0, (int)(f & 31));
      const int o = 2 * (int)(f & 15);
      const uint32_t mask = (2 * l == 32) ? ~0u : ((1u << (2 * l)) - 1);
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const int bo = o + 2 * i;
        const uint32_t x = bo < 32 ? __funnelshift_l(u1, u0, bo) : __funnelshift_l(u2, u1, bo - 32);
        const uint32_t key = x >> (32 - 2 * l);
        code[i] = (uint32_t)(key * (uint32_t)0x6659FD93u) & mask;  // order_code for l <= 16
        if ((nflag << i) >> (32 - l)) vmask &= ~(1u << i);
      }
    } else {
      const int64_t w0 = f >> 5, k0 = f >> 6;
      const uint64_t u0 = ld_stream(q.packed + w0), u1 = ld_stream(q.packed + w0 + 1),
                     u2 = ld_stream(q.packed + w0 + 2);
      const uint64_t nflag = funnel64(ld_stream(q.nmask + k0), ld_stream(q.nmask + k0 + 1), (int)(f & 63));
      const int o = 2 * (int)(f & 31);
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const int bo = o + 2 * i;
        const uint64_t x = bo < 64 ? funnel64(u0, u1, bo) : funnel64(u1, u2, bo - 64);
        code[i] = order_code(x >> (64 - 2 * l), l);
        if ((nflag << i) >> (64 - l)) vmask &= ~(1u << i);
      }
    }
  }
  // the filter words of every window, all in flight together
  uint32_t pass = 0;  // bit w * P + i
  {
    uint32_t fm[P], fw[NW][P];
#pragma unroll
    for (int i = 0; i < P; ++i) {
      const uint64_t h = key_hash(code[i]);
      fm[i] = filter_mask(h);
#pragma unroll
      for (int w = 0; w < NW; ++w)
        fw[w][i] = ((vmask >> i) & 1u) ? __ldg(W.w[w].ix.filter + filter_word(h, W.w[w].ix.fshift)) : 0u;
    }
#pragma unroll
    for (int w = 0; w < NW; ++w)
#pragma unroll
      for (int i = 0; i < P; ++i)
        if (((vmask >> i) & 1u) && (fw[w][i] & fm[i]) == fm[i]) pass |= 1u << (w * P + i);
  }
  if (keep) {
#pragma unroll
    for (int w = 0; w < NW; ++w)
#pragma unroll
      for (int i = 0; i < P; ++i) sm.pl[w][lane * P + i] = kNoPayload;
  }
  int total;
  int k = warp_excl_scan(__popc(pass), lane, &total);
#pragma unroll
  for (int w = 0; w < NW; ++w)
#pragma unroll
    for (int i = 0; i < P; ++i)
      if ((pass >> (w * P + i)) & 1u) {
        sm.u.list.code[k] = code[i];
        sm.u.list.tag[k] = (uint16_t)((w << 8) | (lane * P + i));
        ++k;
      }
  __syncwarp();
  // the bucket reads, shared by the lanes: two in flight per lane
  for (int j = lane; j < total; j += 64) {
    const bool two = j + 32 < total;
    const uint64_t ca = sm.u.list.code[j];
    const int ta = sm.u.list.tag[j];
    const uint64_t cb = two ? sm.u.list.code[j + 32] : 0ull;
    const int tb = two ? sm.u.list.tag[j + 32] : 0;
    const int wa = ta >> 8, wb = tb >> 8;
    const IndexView& ia = W.w[wa].ix;
    const int64_t ha = SMALL ? record_home16((uint32_t)ca, l, ia.nbuckets) : record_home(ca, l, ia.nbuckets);
    uint64_t a0, a1, a2, a3, b0 = 0, b1 = kNoPayload, b2 = 0, b3 = kNoPayload;
    ld_bucket(ia.table + ha, a0, a1, a2, a3);
    int64_t hb = 0;
    if (two) {
      const IndexView& ib = W.w[wb].ix;
      hb = SMALL ? record_home16((uint32_t)cb, l, ib.nbuckets) : record_home(cb, l, ib.nbuckets);
      ld_bucket(ib.table + hb, b0, b1, b2, b3);
    }
    uint64_t pa;
    if (a0 == ca || a1 == kNoPayload) pa = a1;
    else if (a2 == ca || a3 == kNoPayload) pa = a3;
    else pa = table_probe(ia, ca, ha + 2);
    if (keep) sm.pl[wa][ta & 0xff] = pa;
    const int na = payload_count(pa);
#pragma unroll
    for (int w = 0; w < NW; ++w) cnt[w] += (w == wa) ? na : 0;
    if (two) {
      uint64_t pb;
      if (b0 == cb || b1 == kNoPayload) pb = b1;
      else if (b2 == cb || b3 == kNoPayload) pb = b3;
      else pb = table_probe(W.w[wb].ix, cb, hb + 2);
      if (keep) sm.pl[wb][tb & 0xff] = pb;
      const int nb = payload_count(pb);
#pragma unroll
      for (int w = 0; w < NW; ++w) cnt[w] += (w == wb) ? nb : 0;
    }
  }
  __syncwarp();
  return __popc(vmask);
}

template <bool SMALL, int NW>
__global__ void __launch_bounds__(kSeedFusedThreads, NW <= 2 ? 16 : 8) k_seed_multi(QueryView q, SeedWins W, int gap,
                                                                                    int local) {
  constexpr int P = kSeedPerLane;
  __shared__ SeedSmem<NW> smem[kSeedFusedThreads / 32];
  const int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  if (s >= q.nstrands) return;
  SeedSmem<NW>& sm = smem[wib];
  const int64_t st = q.start[s];
  const int qlen = q.len[s];
  const int nk = qlen - W.w[0].ix.l + 1;
  // L2 prefetch for the block kSeedPrefetchBlocks later (as in k_seed_fused);
  // every address stays inside its array
  if (wib == 0 && lane < 5) {
    const int64_t sp = ((int64_t)blockIdx.x + kSeedPrefetchBlocks) * (kSeedFusedThreads / 32);
    if (sp < q.nstrands && q.n > 0) {
      const int64_t f = min(q.n - 1, st + (sp - s) * (q.n / q.nstrands));
      const void* a = lane == 0 ? (const void*)(q.start + sp)
                    : lane == 1 ? (const void*)(q.len + sp)
                    : lane == 4 ? (const void*)(q.nmask + (f >> 6))
                                : (const void*)(q.packed + min((f >> 5) + 16 * (lane - 2), q.n / 32 + 3));
      asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
    }
  }
  // pass 1: counts of every window; round 0's payloads stay in shared memory
  int cnt[NW];
#pragma unroll
  for (int w = 0; w < NW; ++w) cnt[w] = 0;
  int valid_kmers = 0;
  if (nk > 0) {
    for (int r0 = 0; r0 < nk; r0 += kSeedRound)
      valid_kmers += round_lookup_multi<SMALL, NW>(q, W, st, nk, r0, lane, sm, r0 == 0, cnt);
  }
  valid_kmers = (int)__reduce_add_sync(kFull, (unsigned)valid_kmers);
  int tot[NW];
#pragma unroll
  for (int w = 0; w < NW; ++w) tot[w] = (int)__reduce_add_sync(kFull, (unsigned)cnt[w]);
  const int part = (int)(s % kSeedParts);
  // the range reservations: lane w reserves window w's
  unsigned long long rel = 0;
  if (lane < NW) {
    int my = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) my = (w == lane) ? tot[w] : my;
    const SeedWin& sw = W.w[lane];
    if (valid_kmers) atomicAdd(sw.n_kmers + part, (unsigned long long)valid_kmers);
    rel = my ? atomicAdd(&sw.cursor[part], (unsigned long long)my) : 0ull;
  }
  int64_t wpos[NW];
  bool ok[NW];
  bool any = false;
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    const unsigned long long r = __shfl_sync(kFull, rel, w);
    const int64_t base = (int64_t)part * W.w[w].part_cap + (int64_t)r;
    wpos[w] = base;
    ok[w] = tot[w] > 0 && base + tot[w] <= (int64_t)(part + 1) * W.w[w].part_cap;
    any |= ok[w];
    if (lane == 0) {
      W.w[w].off[s] = base;
      W.w[w].cnt[s] = tot[w];
      if (!ok[w]) W.w[w].nvalid[s] = 0;
    }
  }
  if (!any) return;
  // pass 2: the seeds of every window, round by round
  int valid[NW];
  int dummy[NW];
#pragma unroll
  for (int w = 0; w < NW; ++w) valid[w] = dummy[w] = 0;
  for (int r0 = 0; r0 < nk; r0 += kSeedRound) {
    if (r0 > 0) round_lookup_multi<SMALL, NW>(q, W, st, nk, r0, lane, sm, true, dummy);
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      if (!ok[w]) continue;
      uint64_t pl[P];
#pragma unroll
      for (int i = 0; i < P; ++i) pl[i] = sm.pl[w][lane * P + i];
      round_emit(W.w[w].ix, W.w[w].t, gap, local, qlen, r0, lane, pl, wpos[w], valid[w], W.w[w].skey, W.w[w].sq,
                 sm.u.stage.pl, sm.u.stage.qi);
    }
  }
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    const int v = (int)__reduce_add_sync(kFull, (unsigned)valid[w]);
    if (lane == 0 && ok[w]) W.w[w].nvalid[s] = v;
  }
}

__global__ void k_window_first(const int32_t* __restrict__ nvalid, const int32_t* __restrict__ wstart, int nwin,
                               int32_t* __restrict__ wfirst) {
  const int w = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= nwin) return;
  const int a = wstart[w], b = wstart[w + 1];
  int first = -1;
  for (int c = a; c < b && first < 0; c += 32) {
    const int s = c + lane;
    const unsigned m = __ballot_sync(kFull, s < b && nvalid[s] > 0);
    if (m) first = c + __ffs(m) - 1;
  }
  if (lane == 0) wfirst[w] = first;
}

// ---- segmented sort (ascending compare-exchange network, safe with a ragged tail) ----
template <class K2>
__device__ __forceinline__ bool less2(uint64_t a1, K2 a2, uint64_t b1, K2 b2) {
  return a1 < b1 || (a1 == b1 && a2 < b2);
}

// Segments of 2..kThreadSegCap items are sorted one per thread (most reads
// have one or two hits), up to 32 one per warp, up to 2048 per CTA, longer
// in global memory.
constexpr int kThreadSegCap = 8, kSegTiers = 4;

template <class K2, bool PAY>
__global__ void k_classify(const int32_t* __restrict__ len, int64_t nseg, int32_t* __restrict__ lists,
                           int32_t* __restrict__ counts) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = (i < nseg) ? len[i] : 0;
  const int tier = (n <= 1) ? -1 : (n <= kThreadSegCap ? 0 : ((n <= 32) ? 1 : (n <= 2048 ? 2 : 3)));
  const int lane = threadIdx.x & 31;
  // one atomic per warp and tier
#pragma unroll
  for (int t = 0; t < kSegTiers; ++t) {
    const unsigned m = __ballot_sync(kFull, tier == t);
    if (!m) continue;
    int base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd(&counts[t], __popc(m));
    base = __shfl_sync(kFull, base, __ffs(m) - 1);
    if (tier == t) lists[(int64_t)t * nseg + base + __popc(m & lanemask_lt())] = (int32_t)i;
  }
}

// 2..kThreadSegCap items: one thread per segment, an odd-even transposition
// network in registers over the segment's own items only (a compare-exchange
// past its end is skipped, so nothing but its items moves).
template <class K2, bool PAY>
__global__ void k_sort_thread(uint64_t* __restrict__ k1, K2* __restrict__ k2, int32_t* __restrict__ pay,
                              const int64_t* __restrict__ off, const int32_t* __restrict__ len,
                              const int32_t* __restrict__ list, const int32_t* __restrict__ count) {
  const int total = *count;
  for (int64_t li = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; li < total;
       li += (int64_t)gridDim.x * blockDim.x) {
    const int seg = list[li];
    const int64_t o = off[seg];
    const int n = len[seg];
    uint64_t a[kThreadSegCap];
    K2 b[kThreadSegCap];
    int32_t p[kThreadSegCap];
#pragma unroll
    for (int i = 0; i < kThreadSegCap; ++i) {
      a[i] = i < n ? k1[o + i] : 0ull;
      b[i] = i < n ? k2[o + i] : (K2)0;
      p[i] = (PAY && i < n) ? pay[o + i] : 0;
    }
#pragma unroll
    for (int pass = 0; pass < kThreadSegCap; ++pass)
#pragma unroll
      for (int i = pass & 1; i + 1 < kThreadSegCap; i += 2)
        if (i + 1 < n && less2(a[i + 1], b[i + 1], a[i], b[i])) {
          const uint64_t ta = a[i]; a[i] = a[i + 1]; a[i + 1] = ta;
          const K2 tb = b[i]; b[i] = b[i + 1]; b[i + 1] = tb;
          const int32_t tp = p[i]; p[i] = p[i + 1]; p[i + 1] = tp;
        }
#pragma unroll
    for (int i = 0; i < kThreadSegCap; ++i)
      if (i < n) {
        k1[o + i] = a[i];
        k2[o + i] = b[i];
        if (PAY) pay[o + i] = p[i];
      }
  }
}

template <class K2, bool PAY>
__global__ void k_sort_warp(uint64_t* __restrict__ k1, K2* __restrict__ k2, int32_t* __restrict__ pay,
                            const int64_t* __restrict__ off, const int32_t* __restrict__ len,
                            const int32_t* __restrict__ list, const int32_t* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int total = *count;
  for (int64_t li = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; li < total; li += nwarps) {
    const int seg = list[li];
    const int64_t o = off[seg];
    const int n = len[seg];
    uint64_t a1 = ~0ull;
    K2 a2 = (K2)~(K2)0;
    int32_t ap = 0;
    if (lane < n) {
      a1 = k1[o + lane];
      a2 = k2[o + lane];
      if (PAY) ap = pay[o + lane];
    }
    for (int size = 2; size <= 32; size <<= 1) {
      {
        const int partner = lane ^ (size - 1);
        const uint64_t b1 = __shfl_sync(kFull, a1, partner);
        const K2 b2 = __shfl_sync(kFull, a2, partner);
        const int32_t bp = __shfl_sync(kFull, ap, partner);
        const bool lower = lane < partner;
        const bool b_less = less2(b1, b2, a1, a2);
        if (lower ? b_less : !b_less && (b1 != a1 || b2 != a2)) { a1 = b1; a2 = b2; ap = bp; }
      }
      for (int stride = size >> 2; stride > 0; stride >>= 1) {
        const int partner = lane ^ stride;
        const uint64_t b1 = __shfl_sync(kFull, a1, partner);
        const K2 b2 = __shfl_sync(kFull, a2, partner);
        const int32_t bp = __shfl_sync(kFull, ap, partner);
        const bool lower = lane < partner;
        const bool b_less = less2(b1, b2, a1, a2);
        if (lower ? b_less : !b_less && (b1 != a1 || b2 != a2)) { a1 = b1; a2 = b2; ap = bp; }
      }
    }
    if (lane < n) {
      k1[o + lane] = a1;
      k2[o + lane] = a2;
      if (PAY) pay[o + lane] = ap;
    }
  }
}

template <class K2, bool PAY>
__device__ __forceinline__ void cta_network(uint64_t* s1, K2* s2, int32_t* sp, int n) {
  int np = 1;
  while (np < n) np <<= 1;
  for (int size = 2; size <= np; size <<= 1) {
    for (int i = threadIdx.x; i < np / 2; i += blockDim.x) {  // flip stage
      const int blk = i / (size / 2), r = i % (size / 2);
      const int a = blk * size + r, b = blk * size + size - 1 - r;
      if (b < n && less2(s1[b], s2[b], s1[a], s2[a])) {
        const uint64_t t1 = s1[a]; s1[a] = s1[b]; s1[b] = t1;
        const K2 t2 = s2[a]; s2[a] = s2[b]; s2[b] = t2;
        if (PAY) { const int32_t tp = sp[a]; sp[a] = sp[b]; sp[b] = tp; }
      }
    }
    __syncthreads();
    for (int stride = size >> 2; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < np / 2; i += blockDim.x) {
        const int blk = i / stride, r = i % stride;
        const int a = blk * 2 * stride + r, b = a + stride;
        if (b < n && less2(s1[b], s2[b], s1[a], s2[a])) {
          const uint64_t t1 = s1[a]; s1[a] = s1[b]; s1[b] = t1;
          const K2 t2 = s2[a]; s2[a] = s2[b]; s2[b] = t2;
          if (PAY) { const int32_t tp = sp[a]; sp[a] = sp[b]; sp[b] = tp; }
        }
      }
      __syncthreads();
    }
  }
}

constexpr int kCtaSortCap = 2048;

template <class K2, bool PAY>
__global__ void __launch_bounds__(256) k_sort_cta(uint64_t* __restrict__ k1, K2* __restrict__ k2,
                                                  int32_t* __restrict__ pay, const int64_t* __restrict__ off,
                                                  const int32_t* __restrict__ len, const int32_t* __restrict__ list,
                                                  const int32_t* __restrict__ count) {
  __shared__ uint64_t s1[kCtaSortCap];
  __shared__ K2 s2[kCtaSortCap];
  __shared__ int32_t sp[PAY ? kCtaSortCap : 1];
  const int total = *count;
  for (int li = blockIdx.x; li < total; li += gridDim.x) {
    const int seg = list[li];
    const int64_t o = off[seg];
    const int n = len[seg];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      s1[i] = k1[o + i];
      s2[i] = k2[o + i];
      if (PAY) sp[i] = pay[o + i];
    }
    __syncthreads();
    cta_network<K2, PAY>(s1, s2, sp, n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      k1[o + i] = s1[i];
      k2[o + i] = s2[i];
      if (PAY) pay[o + i] = sp[i];
    }
    __syncthreads();
  }
}

template <class K2, bool PAY>
__global__ void __launch_bounds__(1024) k_sort_global(uint64_t* __restrict__ k1, K2* __restrict__ k2,
                                                      int32_t* __restrict__ pay, const int64_t* __restrict__ off,
                                                      const int32_t* __restrict__ len,
                                                      const int32_t* __restrict__ list,
                                                      const int32_t* __restrict__ count) {
  const int total = *count;
  for (int li = blockIdx.x; li < total; li += gridDim.x) {
    const int seg = list[li];
    const int64_t o = off[seg];
    cta_network<K2, PAY>(k1 + o, k2 + o, PAY ? pay + o : pay, len[seg]);
    __syncthreads();
  }
}

template <class K2, bool PAY>
void seg_sort(Workspace& ws, uint64_t* k1, K2* k2, int32_t* pay, const int64_t* off, const int32_t* len,
              int64_t nseg, cudaStream_t st, int tag) {
  if (nseg <= 0) return;
  const std::string t = "segsort" + std::to_string(tag);
  int32_t* lists = ws.get<int32_t>(t + "l", kSegTiers * nseg);
  int32_t* counts = ws.get<int32_t>(t + "c", kSegTiers);
  CLAST_CK(cudaMemsetAsync(counts, 0, kSegTiers * sizeof(int32_t), st));
  k_classify<K2, PAY><<<blocks_for(nseg, 256), 256, 0, st>>>(len, nseg, lists, counts);
  CLAST_LAUNCHED();
  k_sort_thread<K2, PAY><<<grid_cap((nseg + 255) / 256), 256, 0, st>>>(k1, k2, pay, off, len, lists, counts);
  CLAST_LAUNCHED();
  k_sort_warp<K2, PAY><<<grid_cap((nseg * 32 + 255) / 256), 256, 0, st>>>(k1, k2, pay, off, len, lists + nseg,
                                                                          counts + 1);
  CLAST_LAUNCHED();
  k_sort_cta<K2, PAY><<<grid_cap(nseg < 4096 ? nseg : 4096), 256, 0, st>>>(k1, k2, pay, off, len, lists + 2 * nseg,
                                                                           counts + 2);
  CLAST_LAUNCHED();
  k_sort_global<K2, PAY><<<grid_cap(nseg < 1024 ? nseg : 1024), 1024, 0, st>>>(k1, k2, pay, off, len,
                                                                                lists + 3 * nseg, counts + 3);
  CLAST_LAUNCHED();
}


// is "s" near its predecessor "p" (hasNotNearPair / hasNearPair, same strand)
__device__ __forceinline__ bool near_pred(int tid, int tidx, int diag, int ptid, int ptidx, int pdiag,
                                          int width, int gap) {
  return tid == ptid && width >= tidx - ptidx && width >= ptidx - tidx && gap >= pdiag - diag;
}


// ---- seed sort fused with the isolate / duplicate filters ----
struct SeedFilterCtx {
  const int64_t* off;
  const int32_t* cnt;
  const int32_t* nvalid;
  const int32_t* wstart;
  int nwin;
  const int32_t* wfirst;
  int width, gap;
  int32_t* hcnt;
};

__device__ __forceinline__ bool window_first_strand(int64_t s, const SeedFilterCtx& c) {
  int lo = 0, hi = c.nwin;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (c.wstart[mid] <= s) lo = mid;
    else hi = mid;
  }
  return c.wfirst[lo] == (int32_t)s;
}

// State carried from one 32-seed chunk of a strand to the next.
struct FilterState {
  int ptid = 0, ptidx = 0, pdiag = 0;  // last seed of the previous chunk
  bool have_surv = false;
  int stid = 0, stidx = 0, sdiag = 0;  // last isolate-filter survivor so far
  int64_t out = 0;                     // next hit slot
};

// deletingIsolateSeeds then deleteDuplicateSeeds on the chunk of sorted seeds
// j = c0 + lane (valid when j < n); survivors are written at f.out onwards.
__device__ __forceinline__ void filter_chunk(int c0, int n, uint64_t k, uint32_t qi, bool wf, int width, int gap,
                                             FilterState& f, uint64_t* __restrict__ skey,
                                             uint32_t* __restrict__ sq) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  const int j = c0 + lane;
  const bool in = j < n;
  const int tid = (int)(k >> 32);
  const int diag = (int)((uint32_t)k ^ 0x80000000u);
  const int tidx = diag + (int)qi;
  int ptid_l = __shfl_up_sync(kFull, tid, 1);
  int ptidx_l = __shfl_up_sync(kFull, tidx, 1);
  int pdiag_l = __shfl_up_sync(kFull, diag, 1);
  if (lane == 0) { ptid_l = f.ptid; ptidx_l = f.ptidx; pdiag_l = f.pdiag; }
  bool keep8 = false;
  if (in) keep8 = (j == 0) ? wf : near_pred(tid, tidx, diag, ptid_l, ptidx_l, pdiag_l, width, gap);
  const unsigned b8 = __ballot_sync(kFull, keep8);
  const unsigned below = b8 & lt;
  const int src = below ? 31 - __clz(below) : 0;
  const int qtid = __shfl_sync(kFull, tid, src);
  const int qtidx = __shfl_sync(kFull, tidx, src);
  const int qdiag = __shfl_sync(kFull, diag, src);
  bool keep9 = keep8;
  if (keep8) {
    if (below) keep9 = !near_pred(tid, tidx, diag, qtid, qtidx, qdiag, width, gap);
    else if (f.have_surv) keep9 = !near_pred(tid, tidx, diag, f.stid, f.stidx, f.sdiag, width, gap);
  }
  const unsigned b9 = __ballot_sync(kFull, keep9);
  if (keep9) {
    const int64_t w = f.out + __popc(b9 & lt);
    skey[w] = k;
    sq[w] = qi;
  }
  f.out += __popc(b9);
  f.ptid = __shfl_sync(kFull, tid, 31);
  f.ptidx = __shfl_sync(kFull, tidx, 31);
  f.pdiag = __shfl_sync(kFull, diag, 31);
  if (b8) {
    const int last = 31 - __clz(b8);
    f.stid = __shfl_sync(kFull, tid, last);
    f.stidx = __shfl_sync(kFull, tidx, last);
    f.sdiag = __shfl_sync(kFull, diag, last);
    f.have_surv = true;
  }
}

// Seed-sort tiers by a strand's seed count: <= kThreadSortCap (one thread,
// registers; most strands hold a few chance seeds), <= 32 (one warp,
// registers), <= kWarpSmemCap (one warp, shared memory), <= kCtaSortCap (one
// CTA, shared memory), longer (one CTA, global memory).  List entries are the
// strand index with the window-first flag in bit 31.
constexpr int kSortTiers = 5;
constexpr int kThreadSortCap = 8;
constexpr int kWarpSmemCap = 256;
constexpr uint32_t kWinFirstBit = 0x80000000u;

__global__ void k_seed_classify(SeedFilterCtx c, int64_t ns, int32_t* __restrict__ lists,
                                int32_t* __restrict__ counts) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = (i < ns && c.nvalid[i] > 0) ? c.cnt[i] : 0;
  const int tier = (n <= 0)                ? -1
                 : (n <= kThreadSortCap) ? 0
                 : (n <= 32)             ? 1
                 : (n <= kWarpSmemCap)   ? 2
                 : (n <= kCtaSortCap)    ? 3
                                         : 4;
  const int lane = threadIdx.x & 31;
  const uint32_t entry = (uint32_t)i | ((tier >= 0 && window_first_strand(i, c)) ? kWinFirstBit : 0u);
#pragma unroll
  for (int t = 0; t < kSortTiers; ++t) {
    const unsigned m = __ballot_sync(kFull, tier == t);
    if (!m) continue;
    int base = 0;
    if (lane == __ffs(m) - 1) base = atomicAdd(&counts[t], __popc(m));
    base = __shfl_sync(kFull, base, __ffs(m) - 1);
    if (tier == t) lists[(int64_t)t * ns + base + __popc(m & lanemask_lt())] = (int32_t)entry;
  }
}

// Compare-exchange of a warp-wide bitonic network step held one element per
// lane: the lower lane of the pair keeps the smaller element.
__device__ __forceinline__ void warp_cx(uint64_t& a1, uint32_t& a2, int lane, int partner) {
  const uint64_t b1 = __shfl_sync(kFull, a1, partner);
  const uint32_t b2 = __shfl_sync(kFull, a2, partner);
  const bool b_less = less2(b1, b2, a1, a2);
  if (lane < partner ? b_less : !b_less && (b1 != a1 || b2 != a2)) { a1 = b1; a2 = b2; }
}

// 1..kThreadSortCap seeds: one thread per strand.  The seeds (padded with
// keys above every seed) go through an odd-even transposition network in
// registers unless they already ascend; the strand's nvalid valid seeds then
// come first (seeds the boundary filters dropped hold kDroppedSeed, above
// every valid key) and only they are filtered, in seed order, as
// filter_chunk applies the filters to a warp's chunk:
// a seed survives the isolate filter when it is near its predecessor (the
// strand's first seed only when the strand is its window's first), and the
// duplicate filter then drops it when it is near the previous seed that
// survived the isolate filter.
__global__ void k_seed_sort_filter_thread(uint64_t* __restrict__ skey, uint32_t* __restrict__ sq, SeedFilterCtx c,
                                          const int32_t* __restrict__ list, const int32_t* __restrict__ count) {
  const int total = *count;
  for (int64_t li = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; li < total;
       li += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t e = (uint32_t)list[li];
    const int s = (int)(e & ~kWinFirstBit);
    const int64_t o = c.off[s];
    const int n = c.cnt[s];
    const int nv = c.nvalid[s];
    uint64_t k[kThreadSortCap];
    uint32_t q[kThreadSortCap];
    bool sorted = true;
#pragma unroll
    for (int i = 0; i < kThreadSortCap; ++i) {
      k[i] = i < n ? skey[o + i] : ~0ull;
      q[i] = i < n ? sq[o + i] : ~0u;
      if (i > 0 && less2(k[i], q[i], k[i - 1], q[i - 1])) sorted = false;
    }
    if (!sorted) {
#pragma unroll
      for (int pass = 0; pass < kThreadSortCap; ++pass)
#pragma unroll
        for (int i = pass & 1; i + 1 < kThreadSortCap; i += 2)
          if (less2(k[i + 1], q[i + 1], k[i], q[i])) {
            const uint64_t tk = k[i]; k[i] = k[i + 1]; k[i + 1] = tk;
            const uint32_t tq = q[i]; q[i] = q[i + 1]; q[i + 1] = tq;
          }
    }
    const bool wf = (e & kWinFirstBit) != 0;
    int ptid = 0, ptidx = 0, pdiag = 0;  // previous seed
    int stid = 0, stidx = 0, sdiag = 0;  // previous isolate-filter survivor
    bool have = false;
    int64_t out = o;
#pragma unroll
    for (int j = 0; j < kThreadSortCap; ++j) {
      if (j < nv) {
        const int tid = (int)(k[j] >> 32);
        const int diag = (int)((uint32_t)k[j] ^ 0x80000000u);
        const int tidx = diag + (int)q[j];
        const bool k8 = (j == 0) ? wf : near_pred(tid, tidx, diag, ptid, ptidx, pdiag, c.width, c.gap);
        const bool k9 = k8 && !(have && near_pred(tid, tidx, diag, stid, stidx, sdiag, c.width, c.gap));
        if (k9) {
          skey[out] = k[j];
          sq[out] = q[j];
          ++out;
        }
        if (k8) { stid = tid; stidx = tidx; sdiag = diag; have = true; }
        ptid = tid; ptidx = tidx; pdiag = diag;
      }
    }
    c.hcnt[s] = (int32_t)(out - o);
  }
}

// <= 32 seeds: one warp sorts in registers (network sized to the count,
// skipped when the seeds already ascend) and filters from registers.
__global__ void k_seed_sort_filter_warp(uint64_t* __restrict__ skey, uint32_t* __restrict__ sq, SeedFilterCtx c,
                                        const int32_t* __restrict__ list, const int32_t* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int total = *count;
  for (int64_t li = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; li < total; li += nwarps) {
    const uint32_t e = (uint32_t)list[li];
    const int s = (int)(e & ~kWinFirstBit);
    const int64_t o = c.off[s];
    const int n = c.cnt[s];
    uint64_t a1 = ~0ull;
    uint32_t a2 = ~0u;
    if (lane < n) {
      a1 = skey[o + lane];
      a2 = sq[o + lane];
    }
    const uint64_t n1 = __shfl_down_sync(kFull, a1, 1);
    const uint32_t n2 = __shfl_down_sync(kFull, a2, 1);
    if (__any_sync(kFull, lane + 1 < n && less2(n1, n2, a1, a2))) {
      int np = 2;
      while (np < n) np <<= 1;
      for (int size = 2; size <= np; size <<= 1) {
        warp_cx(a1, a2, lane, lane ^ (size - 1));
        for (int stride = size >> 2; stride > 0; stride >>= 1) warp_cx(a1, a2, lane, lane ^ stride);
      }
    }
    FilterState f;
    f.out = o;
    filter_chunk(0, c.nvalid[s], a1, a2, (e & kWinFirstBit) != 0, c.width, c.gap, f, skey, sq);
    if (lane == 0) c.hcnt[s] = (int32_t)(f.out - o);
  }
}

// Bitonic network over n <= np elements in shared memory, run by one warp.
__device__ __forceinline__ void warp_smem_network(uint64_t* s1, uint32_t* s2, int n) {
  const int lane = threadIdx.x & 31;
  int np = 64;
  while (np < n) np <<= 1;
  for (int size = 2; size <= np; size <<= 1) {
    for (int i = lane; i < np / 2; i += 32) {  // flip stage
      const int blk = i / (size / 2), r = i % (size / 2);
      const int a = blk * size + r, b = blk * size + size - 1 - r;
      if (b < n && less2(s1[b], s2[b], s1[a], s2[a])) {
        const uint64_t t1 = s1[a]; s1[a] = s1[b]; s1[b] = t1;
        const uint32_t t2 = s2[a]; s2[a] = s2[b]; s2[b] = t2;
      }
    }
    __syncwarp();
    for (int stride = size >> 2; stride > 0; stride >>= 1) {
      for (int i = lane; i < np / 2; i += 32) {
        const int blk = i / stride, r = i % stride;
        const int a = blk * 2 * stride + r, b = a + stride;
        if (b < n && less2(s1[b], s2[b], s1[a], s2[a])) {
          const uint64_t t1 = s1[a]; s1[a] = s1[b]; s1[b] = t1;
          const uint32_t t2 = s2[a]; s2[a] = s2[b]; s2[b] = t2;
        }
      }
      __syncwarp();
    }
  }
}

constexpr int kWarpSmemThreads = 128;

// 33..kWarpSmemCap seeds: one warp sorts in its own slice of shared memory
// (skipped when the seeds already ascend) and filters from there.
__global__ void __launch_bounds__(kWarpSmemThreads) k_seed_sort_filter_warp_smem(
    uint64_t* __restrict__ skey, uint32_t* __restrict__ sq, SeedFilterCtx c, const int32_t* __restrict__ list,
    const int32_t* __restrict__ count) {
  __shared__ uint64_t sh1[kWarpSmemThreads / 32][kWarpSmemCap];
  __shared__ uint32_t sh2[kWarpSmemThreads / 32][kWarpSmemCap];
  const int lane = threadIdx.x & 31;
  uint64_t* s1 = sh1[threadIdx.x >> 5];
  uint32_t* s2 = sh2[threadIdx.x >> 5];
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int total = *count;
  for (int64_t li = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; li < total; li += nwarps) {
    const uint32_t e = (uint32_t)list[li];
    const int s = (int)(e & ~kWinFirstBit);
    const int64_t o = c.off[s];
    const int n = c.cnt[s];
    for (int i = lane; i < n; i += 32) {
      s1[i] = skey[o + i];
      s2[i] = sq[o + i];
    }
    __syncwarp();
    bool unsorted = false;
    for (int i = lane; i + 1 < n; i += 32) unsorted |= less2(s1[i + 1], s2[i + 1], s1[i], s2[i]);
    if (__any_sync(kFull, unsorted)) warp_smem_network(s1, s2, n);
    const int nv = c.nvalid[s];
    const bool wf = (e & kWinFirstBit) != 0;
    FilterState f;
    f.out = o;
    for (int c0 = 0; c0 < nv; c0 += 32) {
      const int j = c0 + lane;
      filter_chunk(c0, nv, j < nv ? s1[j] : 0ull, j < nv ? s2[j] : 0u, wf, c.width, c.gap, f, skey, sq);
    }
    if (lane == 0) c.hcnt[s] = (int32_t)(f.out - o);
    __syncwarp();
  }
}

// <= kCtaSortCap seeds: one CTA sorts in shared memory, warp 0 filters from there.
__global__ void __launch_bounds__(256) k_seed_sort_filter_cta(uint64_t* __restrict__ skey, uint32_t* __restrict__ sq,
                                                              SeedFilterCtx c, const int32_t* __restrict__ list,
                                                              const int32_t* __restrict__ count) {
  __shared__ uint64_t s1[kCtaSortCap];
  __shared__ uint32_t s2[kCtaSortCap];
  const int total = *count;
  for (int li = blockIdx.x; li < total; li += gridDim.x) {
    const uint32_t e = (uint32_t)list[li];
    const int s = (int)(e & ~kWinFirstBit);
    const int64_t o = c.off[s];
    const int n = c.cnt[s];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      s1[i] = skey[o + i];
      s2[i] = sq[o + i];
    }
    __syncthreads();
    cta_network<uint32_t, false>(s1, s2, nullptr, n);
    if (threadIdx.x < 32) {
      const int nv = c.nvalid[s];
      const bool wf = (e & kWinFirstBit) != 0;
      FilterState f;
      f.out = o;
      for (int c0 = 0; c0 < nv; c0 += 32) {
        const int j = c0 + (int)threadIdx.x;
        filter_chunk(c0, nv, j < nv ? s1[j] : 0ull, j < nv ? s2[j] : 0u, wf, c.width, c.gap, f, skey, sq);
      }
      if (threadIdx.x == 0) c.hcnt[s] = (int32_t)(f.out - o);
    }
    __syncthreads();
  }
}

// Longer: one CTA sorts in global memory, warp 0 filters in place.
__global__ void __launch_bounds__(1024) k_seed_sort_filter_global(uint64_t* __restrict__ skey,
                                                                  uint32_t* __restrict__ sq, SeedFilterCtx c,
                                                                  const int32_t* __restrict__ list,
                                                                  const int32_t* __restrict__ count) {
  const int total = *count;
  for (int li = blockIdx.x; li < total; li += gridDim.x) {
    const uint32_t e = (uint32_t)list[li];
    const int s = (int)(e & ~kWinFirstBit);
    const int64_t o = c.off[s];
    cta_network<uint32_t, false>(skey + o, sq + o, nullptr, c.cnt[s]);
    __syncthreads();
    if (threadIdx.x < 32) {
      const int nv = c.nvalid[s];
      const bool wf = (e & kWinFirstBit) != 0;
      FilterState f;
      f.out = o;
      for (int c0 = 0; c0 < nv; c0 += 32) {
        const int j = c0 + (int)threadIdx.x;
        uint64_t k = 0;
        uint32_t qv = 0;
        if (j < nv) {
          k = skey[o + j];
          qv = sq[o + j];
        }
        filter_chunk(c0, nv, k, qv, wf, c.width, c.gap, f, skey, sq);
      }
      if (threadIdx.x == 0) c.hcnt[s] = (int32_t)(f.out - o);
    }
    __syncthreads();
  }
}

__global__ void k_gather_hits(const uint64_t* __restrict__ skey, const uint32_t* __restrict__ sq,
                              const int64_t* __restrict__ off, const int32_t* __restrict__ hcnt,
                              const int64_t* __restrict__ hoff, int64_t nstrands, uint64_t* __restrict__ hk,
                              int32_t* __restrict__ hq, int32_t* __restrict__ hs, const int32_t* __restrict__ qlen,
                              int l, int band, unsigned long long* __restrict__ cells) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int n = (s < nstrands) ? hcnt[s] : 0;
  // every hit of the strand fills band * (qlen - l) cells: backward rows + forward rows
  unsigned long long c = n ? (unsigned long long)n * (unsigned long long)band * (unsigned long long)(qlen[s] - l) : 0;
#pragma unroll
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(cells, c);
  if (s >= nstrands) return;
  const int64_t a = off[s], b = hoff[s];
  for (int i = 0; i < n; ++i) {
    hk[b + i] = skey[a + i];
    hq[b + i] = (int32_t)sq[a + i];
    hs[b + i] = (int32_t)s;
  }
}

// ------------------------------------------------------------------------
// banded DP
// ------------------------------------------------------------------------
// POINT_MATRIX / MATCH_COUNTER (krnlMatrix.cuh:11-67) depend only on seven
// letter classes: A, C, G, T, any other scored letter (B D H K M N R S U V W Y),
// a '-1' letter (E F I J L O P Q Z) and the bad-area letter X.  Bytes outside
// 'A'..'Z' score as 'N'.
constexpr int kClassX = 6;

__host__ __device__ constexpr int class_of_letter(int i) {  // i = letter - 'A'
  return i == 0 ? 0 : i == 2 ? 1 : i == 6 ? 2 : i == 19 ? 3 : i == 23 ? kClassX
       : (i == 4 || i == 5 || i == 8 || i == 9 || i == 11 || i == 14 || i == 15 || i == 16 || i == 25) ? 5 : 4;
}
// (point, match increment) for target class t, query class q.
__device__ __forceinline__ int2 cell_score(int t, int q) {
  if (t == kClassX || q == kClassX) return make_int2(-1000, -1000);
  if (t == 5 || q == 5) return make_int2(-1, -1);
  if (t == q && t < 4) return make_int2(1, 1);
  return make_int2(-3, 0);
}

// Banded DP of one hit, backward pass then forward pass, in ONE row loop of
// rows_b + rows_f iterations: every hit of a read has qLen - l rows in total,
// so the threads of a warp stay converged although each switches from the
// backward to the forward pass at its own row.
//
// Per band column the registers hold A = S - 7 (score minus gap open +
// extend), B = V - 2 (vertical state minus gap extend) and M (matches); along
// a row the chain carries hA = S - 7 and hB = H - 2 of the previous column.
// Then, exactly as calcutlateCell (krnlAlignment.cu:42-77):
//   V = max(Sv - 7, Vv - 2) = max(A_v, B_v)        H = max(Sh - 7, Hh - 2) = max(hA, hB)
//   pt = S_diag + POINT = A_diag + (POINT + 7)      (the table stores POINT + 7)
//   H wins over V iff H >= V; the diagonal wins iff pt > max(V, H)
// Storing S itself and folding the "- 7" into a fused add-and-max per
// maximum takes one add per cell less, but the row's chain through it is
// slower: a lone thread took 6.8 against 2.7 ms on one 5 kbp hit, with no gain
// on full batches of 150 bp reads.  A long hit's chain sets the latency of
// small batches, so the band keeps S - 7.
template <int GAP>
struct Band {
  static constexpr int W = 2 * GAP + 1;
  int A[W], B[W], M[W], tc[W];

  // initTempNodeArray, krnlAlignment.cu:6-38 (band rows 1..W), and the first W
  // target bases of a pass: index ib0 + step * c, 'X' outside [lo, hi).
  __device__ __forceinline__ void init(const char* __restrict__ tb, int64_t tstart, int64_t ib0, int step,
                                       int64_t lo, int64_t hi) {
#pragma unroll
    for (int c = 0; c < W; ++c) {
      const int r = c + 1;
      int sc, v, m;
      if (r < GAP + 1) { sc = kMarginScore; v = kMarginScore; m = kMarginScore; }
      else if (r == GAP + 1) { sc = 0; v = kGapOpen; m = 0; }
      else { sc = (r - GAP - 1) * kGapExtend + kGapOpen; v = sc + kGapOpen; m = 0; }
      A[c] = sc + kGapOpen + kGapExtend;
      B[c] = v + kGapExtend;
      M[c] = m;
      const int64_t ib = ib0 + (int64_t)step * c;
      tc[c] = ((ib < lo || ib >= hi) ? kBadClass : base_class(tb[tstart + ib])) << 8;  // byte offset of its table row
    }
  }
  // select end node (global mode), krnlAlignment.cu:170-185
  __device__ __forceinline__ void end_node(int& best, int& best_m, int& ep) const {
    best = kMarginScore;
    best_m = kMarginScore;
    ep = -1;
#pragma unroll
    for (int c = 0; c < W; ++c) {
      const int sc = A[c] - (kGapOpen + kGapExtend);
      if (best < sc) { best = sc; best_m = M[c]; ep = c; }
    }
  }
};

template <int GAP, bool LOCAL>
__device__ __forceinline__ void banded_hit(const int2* __restrict__ tab, const char* __restrict__ tb, int64_t tstart,
                                           int tlen, const char* __restrict__ qb, int64_t qstart, int qlen, int tidx,
                                           int qidx, int l, int& t_hl, int& q_hl, int& match, int& score,
                                           int& o_tidx, int& o_qidx) {
  constexpr int W = Band<GAP>::W;
  constexpr int kGapSO = kGapOpen + kGapExtend;  // -7
  constexpr int kBotA = (GAP + 1) * kGapExtend + kGapOpen + kGapSO;  // fixed band row 2*GAP+2
  constexpr int kBotB = (GAP + 1) * kGapExtend + kGapOpen + kGapOpen + kGapExtend;
  constexpr int kMarginA = kMarginScore + kGapSO, kMarginB = kMarginScore + kGapExtend;
  constexpr int kNoLow = INT_MIN / 2, kNoHigh = INT_MAX / 2;
  const int rows_b = qlen - (qidx + l);  // alignmentSize of the backward pass
  const int rows_f = qidx;              // rows of the forward pass
  const int rows = rows_b + rows_f;
  Band<GAP> bd;
  const char* __restrict__ t_seq = tb + tstart;
  // backward pass (globalAlignBackward / localAlignBackward): target bases
  // tIdx + l - gap + q + c ('X' at or past tLen), query bases qIdx + l + q
  const char* q_ptr = qb + qstart + qidx + l;  // query base of the current row
  int q_step = 1;
  int t_ib = tidx + l + GAP + 1;  // next target base to shift in
  int t_step = 1;
  int t_lo = kNoLow, t_hi = tlen;
  int row_end = rows_b;  // last row + 1 of the current pass
  bd.init(tb, tstart, (int64_t)tidx + l - GAP, 1, t_lo, t_hi);
  int bs = 0, bm = 0, calc = -1, ep = GAP, qrow = 0;
  int pass = 0;
  auto finish = [&](int pass_rows) {  // result of the pass that just ended
    int move, best, best_m, e;
    if (LOCAL) { best = bs; best_m = bm; e = ep; move = calc + 1; }
    else { bd.end_node(best, best_m, e); move = pass_rows; }
    e -= GAP;
    if (pass_rows != 0) {
      if (pass == 1) {  // forward: the hit's start moves
        o_tidx -= move + e;
        o_qidx -= move;
      }
      t_hl += move + e;
      q_hl += move;
      match += best_m;
      score += best;
    }
  };
  char q_cur = (rows_b > 0) ? *q_ptr : 'N';
  for (int r = 0; r < rows; ++r) {
    if (r == rows_b) {  // switch to the forward pass (globalAlignForward / localAlignForward)
      finish(rows_b);
      pass = 1;
      q_ptr = qb + qstart + qidx - 1;  // query bases qIdx - q - 1
      q_step = -1;
      t_ib = tidx - GAP - 2;  // target bases tIdx + gap - 1 - q - c ('X' below 0)
      t_step = -1;
      t_lo = 0;
      t_hi = kNoHigh;
      row_end = rows;
      bd.init(tb, tstart, (int64_t)tidx + GAP - 1, -1, t_lo, t_hi);
      bs = 0; bm = 0; calc = -1; ep = GAP; qrow = 0;
      q_cur = *q_ptr;
    }
    // loads for the next row go out first; their latency hides behind this row
    const char t_next = (t_ib < t_lo || t_ib >= t_hi) ? 'X' : t_seq[t_ib];
    t_ib += t_step;
    const char q_next = (r + 1 < row_end) ? q_ptr[q_step] : 'N';
    q_ptr += q_step;
    // the query letter's column in every target row: one add per cell finds
    // the (point + 7, match) pair (byte offsets; no index arithmetic)
    const char* rowp = reinterpret_cast<const char*>(tab) + (base_class(q_cur) << 3);
    int hA = kMarginA, hB = kMarginB, hM = kMarginScore;  // row 0 of the band (left margin)
#pragma unroll
    for (int c = 0; c < W; ++c) {
      const int vA = (c + 1 < W) ? bd.A[(c + 1) % W] : kBotA;
      const int vB = (c + 1 < W) ? bd.B[(c + 1) % W] : kBotB;
      const int vM = (c + 1 < W) ? bd.M[(c + 1) % W] : 0;
      const int nV = max(vA, vB);
      const int nH = max(hA, hB);
      const int2 w = *reinterpret_cast<const int2*>(rowp + bd.tc[c]);  // (POINT + 7, match increment)
      const int pt = bd.A[c] + w.x;
      // (plain compares and maxima: fewer instructions than __vibmax_s32 here)
      const bool h_wins = nH >= nV;
      const int mx = max(nH, nV);
      const bool not_diag = mx >= pt;
      const int nS = max(mx, pt);
      const int side_m = h_wins ? hM : vM;
      const int nM = not_diag ? side_m : (bd.M[c] + w.y);
      const int nA = nS + kGapSO;
      bd.A[c] = nA;
      bd.B[c] = nV + kGapExtend;
      bd.M[c] = nM;
      hA = nA;
      hB = nH + kGapExtend;
      hM = nM;
      if (LOCAL) {
        if (bs < nS) { bs = nS; bm = nM; calc = qrow; ep = c; }
      }
    }
#pragma unroll
    for (int c = 0; c < W - 1; ++c) bd.tc[c] = bd.tc[c + 1];
    bd.tc[W - 1] = base_class(t_next) << 8;  // 'X' above is the bad-area letter itself
    q_cur = q_next;
    ++qrow;
  }
  if (rows_b == rows) {  // the loop never switched: close the backward pass (rows_f == 0)
    finish(rows_b);
  } else {
    finish(rows_f);
  }
}

// The same extension with one warp per hit: the band's anti-diagonal
// wavefront.  Cell (r, c) of the band needs (r, c-1), (r-1, c+1) and (r-1, c),
// so the cells with equal 2r + c are independent.  Lane j owns band columns 2j
// and 2j + 1 and runs row r - j while lane 0 runs row r: column 2j at the even
// step, taking its left neighbour from lane j - 1 (shuffle) and its upper-right
// one from its own odd column; column 2j + 1 at the odd step, with its left
// neighbour its own even column and its upper-right one from lane j + 1
// (shuffle).  A row costs two steps instead of W dependent cells, which is
// what one long hit in a small batch waits for.  Same cell arithmetic as
// banded_hit, same tie rules (the local best is the first maximum in
// row-major order, the global end node the first maximum in column order),
// so every output equals banded_hit's.  Results are returned in every lane.
template <int GAP, bool LOCAL>
__device__ __forceinline__ void banded_hit_warp(const int2* __restrict__ tab, const char* __restrict__ tb,
                                                int64_t tstart, int tlen, const char* __restrict__ qb, int64_t qstart,
                                                int qlen, int tidx, int qidx, int l, int& t_hl, int& q_hl, int& match,
                                                int& score, int& o_tidx, int& o_qidx) {
  constexpr int W = 2 * GAP + 1;
  constexpr int kGapSO = kGapOpen + kGapExtend;  // -7
  constexpr int kBotA = (GAP + 1) * kGapExtend + kGapOpen + kGapSO;
  constexpr int kBotB = (GAP + 1) * kGapExtend + kGapOpen + kGapOpen + kGapExtend;
  constexpr int kMarginA = kMarginScore + kGapSO, kMarginB = kMarginScore + kGapExtend;
  const int lane = threadIdx.x & 31;
  const int ce = 2 * lane, co = 2 * lane + 1;  // this lane's band columns
  const bool has_e = ce < W, has_o = co < W;
  // lane 0's left neighbour is lane 31 (GAP <= 16 leaves it idle), which holds
  // the band's left margin; lane GAP, without an odd column, holds the fixed
  // band row below the last column there instead
  const int left = (lane + 31) & 31, right = (lane + 1) & 31;
  const char* tabb = reinterpret_cast<const char*>(tab);
  const char* __restrict__ t_seq = tb + tstart;
  const char* __restrict__ q_seq = qb + qstart;
  const int rows_b = qlen - (qidx + l);
  const int rows_f = qidx;
  for (int pass = 0; pass < 2; ++pass) {
    const int rows_p = pass == 0 ? rows_b : rows_f;
    if (rows_p <= 0) continue;
    // target base of cell (r, c): ib0 + step * (r + c), the bad-area letter
    // outside [lo, hi); query base of row r: qi0 + step * r (banded_hit's
    // indices, pass by pass)
    const int step = pass == 0 ? 1 : -1;
    const int ib0 = pass == 0 ? tidx + l - GAP : tidx + GAP - 1;
    const int lo = pass == 0 ? INT_MIN : 0, hi = pass == 0 ? tlen : INT_MAX;
    const int qi0 = pass == 0 ? qidx + l : qidx - 1;
    auto t_byte = [&](int ib) -> char { return (ib < lo || ib >= hi) ? 'X' : t_seq[ib]; };
    auto q_byte = [&](int r) -> char { return (unsigned)r < (unsigned)rows_p ? q_seq[qi0 + step * r] : 'N'; };
    // initTempNodeArray for this lane's two columns (the state before row 0)
    auto init_col = [&](int c, int& A, int& B, int& M) {
      const int rr = c + 1;
      int sc, v, m;
      if (rr < GAP + 1) { sc = kMarginScore; v = kMarginScore; m = kMarginScore; }
      else if (rr == GAP + 1) { sc = 0; v = kGapOpen; m = 0; }
      else { sc = (rr - GAP - 1) * kGapExtend + kGapOpen; v = sc + kGapOpen; m = 0; }
      A = sc + kGapSO;
      B = v + kGapExtend;
      M = m;
    };
    int eA, eB, eM, oA = 0, oB = 0, oM = 0, eH = 0, oH = 0;
    init_col(ce, eA, eB, eM);
    if (has_o) {
      init_col(co, oA, oB, oM);
    } else if (lane == 31) {
      oA = kMarginA;
      oH = kMarginB;
      oM = kMarginScore;
    } else {
      oA = kBotA;
      oB = kBotB;
      oM = 0;
    }
    int bs = 0, bm = 0, calc = -1, ep = GAP;
    // Row r of this lane uses the target bases r + 2j (even column; the odd
    // column's base of row r - 1) and r + 2j + 1, and query base r.  Bytes are
    // loaded four rows ahead and turned into table offsets one row ahead, so
    // that no load's latency falls inside a row.
    int r = -lane;
    int te = base_class(t_byte(ib0 + step * (r + ce))) << 8;
    int to = base_class(t_byte(ib0 + step * (r + co))) << 8;
    char t1 = t_byte(ib0 + step * (r + 1 + co)), t2 = t_byte(ib0 + step * (r + 2 + co));
    char t3 = t_byte(ib0 + step * (r + 3 + co));
    int qc = base_class(q_byte(r)) << 3;
    char q1 = q_byte(r + 1), q2 = q_byte(r + 2), q3 = q_byte(r + 3);
    int tk = ib0 + step * (r + 4 + co);
    const int n_iter = rows_p + GAP;  // lane GAP runs the last row at rows_p - 1 + GAP
#pragma unroll 2
    for (int it = 0; it < n_iter; ++it, ++r) {
      const char t4 = t_byte(tk);
      tk += step;
      const char q4 = q_byte(r + 4);
      const bool on = (unsigned)r < (unsigned)rows_p;
      {  // even step: column 2j of row r; left neighbour from lane j - 1, upper right from our odd column
        const int hA = __shfl_sync(kFull, oA, left);
        const int hB = __shfl_sync(kFull, oH, left);
        const int hM = __shfl_sync(kFull, oM, left);
        const int nV = max(oA, oB);
        const int nH = max(hA, hB);
        const int2 w = *reinterpret_cast<const int2*>(tabb + te + qc);
        const int pt = eA + w.x;
        const bool h_wins = nH >= nV;
        const int mx = max(nH, nV);
        const bool not_diag = mx >= pt;
        const int nS = max(mx, pt);
        const int nM = not_diag ? (h_wins ? hM : oM) : (eM + w.y);
        if (on && has_e) {
          eA = nS + kGapSO;
          eB = nV + kGapExtend;
          eH = nH + kGapExtend;
          eM = nM;
          if (LOCAL && bs < nS) { bs = nS; bm = nM; calc = r; ep = ce; }
        }
      }
      {  // odd step: column 2j + 1 of row r; left neighbour our even column, upper right from lane j + 1
        const int vA = __shfl_sync(kFull, eA, right);
        const int vB = __shfl_sync(kFull, eB, right);
        const int vM = __shfl_sync(kFull, eM, right);
        const int nV = max(vA, vB);
        const int nH = max(eA, eH);
        const int2 w = *reinterpret_cast<const int2*>(tabb + to + qc);
        const int pt = oA + w.x;
        const bool h_wins = nH >= nV;
        const int mx = max(nH, nV);
        const bool not_diag = mx >= pt;
        const int nS = max(mx, pt);
        const int nM = not_diag ? (h_wins ? eM : vM) : (oM + w.y);
        if (on && has_o) {
          oA = nS + kGapSO;
          oB = nV + kGapExtend;
          oH = nH + kGapExtend;
          oM = nM;
          if (LOCAL && bs < nS) { bs = nS; bm = nM; calc = r; ep = co; }
        }
      }
      te = to;
      to = base_class(t1) << 8;
      t1 = t2;
      t2 = t3;
      t3 = t4;
      qc = base_class(q1) << 3;
      q1 = q2;
      q2 = q3;
      q3 = q4;
    }
    int best, best_m, e, move;
    if (LOCAL) {  // first maximum in row-major order: (score desc, row asc, column asc)
#pragma unroll
      for (int off = 16; off; off >>= 1) {
        const int xs = __shfl_xor_sync(kFull, bs, off), xm = __shfl_xor_sync(kFull, bm, off);
        const int xc = __shfl_xor_sync(kFull, calc, off), xe = __shfl_xor_sync(kFull, ep, off);
        if (xs > bs || (xs == bs && (xc < calc || (xc == calc && xe < ep)))) { bs = xs; bm = xm; calc = xc; ep = xe; }
      }
      best = bs;
      best_m = bm;
      e = ep;
      move = calc + 1;
    } else {  // end node: the first column of the last row with the highest score above the margin
      int sc = INT_MIN, c = W, m = 0;
      if (has_e) { sc = eA - kGapSO; c = ce; m = eM; }
      if (has_o && oA - kGapSO > sc) { sc = oA - kGapSO; c = co; m = oM; }
#pragma unroll
      for (int off = 16; off; off >>= 1) {
        const int xs = __shfl_xor_sync(kFull, sc, off), xc = __shfl_xor_sync(kFull, c, off);
        const int xm = __shfl_xor_sync(kFull, m, off);
        if (xs > sc || (xs == sc && xc < c)) { sc = xs; c = xc; m = xm; }
      }
      if (sc > kMarginScore) { best = sc; best_m = m; e = c; }
      else { best = kMarginScore; best_m = kMarginScore; e = -1; }
      move = rows_p;
    }
    e -= GAP;
    if (pass == 1) {
      o_tidx -= move + e;
      o_qidx -= move;
    }
    t_hl += move + e;
    q_hl += move;
    match += best_m;
    score += best;
  }
}

struct DpKernelArgs {
  TargetView t;
  QueryView q;
  const uint64_t* hk;
  const int32_t* hq;
  const int32_t* hs;
  const uint64_t* order;
  int64_t n;
  DpParams p;
  DpOut o;
  // the first n_warp hits of the order run one per warp (k_banded_dp_warp),
  // the others one per thread: n_warp = *warp_n when given, else warp_fixed
  const long long* warp_n;
  long long warp_fixed;
  int* bad;  // see DpLaunch::bad
};

// A hit whose target sequence or strand lies outside the window cannot come
// from the seeding stages; it is flagged and given empty outputs instead of
// being read past the window.
__device__ __forceinline__ bool dp_hit_outside(const DpKernelArgs& a, int tid, int s) {
  return (unsigned)tid >= (unsigned)a.t.nseqs || (unsigned)s >= (unsigned)a.q.nstrands;
}

__device__ __forceinline__ int64_t dp_warp_hits(const DpKernelArgs& a) {
  const int64_t w = a.warp_n ? (int64_t)*a.warp_n : (int64_t)a.warp_fixed;
  return w < a.n ? w : a.n;
}

// The letter-pair table (POINT + 7, match increment) of krnlMatrix.cuh in
// shared memory: [target letter][query letter], letters 'A'..'Z'.
__device__ __forceinline__ void dp_table_init(int2* tab) {
  for (int i = threadIdx.x; i < 32 * 32; i += blockDim.x) {
    const int2 w = cell_score(class_of_letter((i >> 5) < 26 ? (i >> 5) : kNClass),
                              class_of_letter((i & 31) < 26 ? (i & 31) : kNClass));
    tab[i] = make_int2(w.x - (kGapOpen + kGapExtend), w.y);
  }
}

// calculateEvalue (krnlCalculateEvalue.cu:21, same operation order) and the
// two hit filters of deleteBadHits, then the hit's outputs at its own index.
__device__ __forceinline__ void dp_store(const DpKernelArgs& a, int64_t h, int qlen, int o_tidx, int o_qidx, int t_hl,
                                         int q_hl, int match, int score) {
  const double e = a.p.K * a.p.total_db * (double)qlen * exp(-a.p.lambda * (double)score);
  const bool keep = !(a.p.cutoff != -1.0 && a.p.cutoff < e) && !(a.p.l + a.p.stride > q_hl);
  a.o.t_idx[h] = o_tidx;
  a.o.q_idx[h] = o_qidx;
  a.o.t_len[h] = t_hl;
  a.o.q_len[h] = q_hl;
  a.o.match[h] = match;
  a.o.score[h] = score;
  a.o.evalue[h] = e;
  a.o.keep[h] = keep ? 1 : 0;
}

__device__ __forceinline__ void dp_skip(const DpKernelArgs& a, int64_t h) {
  a.o.t_idx[h] = a.o.q_idx[h] = a.o.t_len[h] = a.o.q_len[h] = a.o.match[h] = a.o.score[h] = 0;
  a.o.evalue[h] = 0.0;
  a.o.keep[h] = 0;
  if (a.bad) atomicExch(a.bad, 1);
}

// Extension of the hit at position i of the order (alignmentHits +
// calculateEvalue + the two hit filters of deleteBadHits).
template <int GAP, bool LOCAL>
__device__ __forceinline__ void dp_one(const DpKernelArgs& a, const int2* tab, int64_t i) {
  const int64_t h = a.order ? (int64_t)(uint32_t)a.order[i] : i;
  const uint64_t k = a.hk[h];
  const int qidx = a.hq[h];
  const int s = a.hs[h];
  const int tid = (int)(k >> 32);
  if (dp_hit_outside(a, tid, s)) {
    dp_skip(a, h);
    return;
  }
  const int tidx = (int)((uint32_t)k ^ 0x80000000u) + qidx;
  const int64_t tstart = a.t.gateway[tid];
  const int tlen = a.t.lengths[tid];
  const int64_t qstart = a.q.start[s];
  const int qlen = a.q.len[s];
  const int l = a.p.l;
  int t_hl = l, q_hl = l, match = l, score = l;  // CDeviceHitList.cu:283-286
  int o_tidx = tidx, o_qidx = qidx;
  banded_hit<GAP, LOCAL>(tab, a.t.bases, tstart, tlen, a.q.bases, qstart, qlen, tidx, qidx, l, t_hl, q_hl, match,
                         score, o_tidx, o_qidx);
  dp_store(a, h, qlen, o_tidx, o_qidx, t_hl, q_hl, match, score);
}

template <int GAP, bool LOCAL>
__global__ void __launch_bounds__(128, GAP <= 9 ? 4 : (GAP <= 12 ? 3 : 2)) k_banded_dp(DpKernelArgs a) {
  __shared__ int2 tab[32 * 32];
  dp_table_init(tab);
  __syncthreads();
  const int64_t i = dp_warp_hits(a) + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  dp_one<GAP, LOCAL>(a, tab, i);
}

// Persistent form: a grid that fills the GPU once; each warp takes the next
// `chunk` x 32 hits of the order (longest first) from a queue head until the
// queue is empty, so that warps which drew short hits go on to take more
// while the long ones run.  No warp waits on another.
template <int GAP, bool LOCAL>
__global__ void __launch_bounds__(128, GAP <= 9 ? 4 : (GAP <= 12 ? 3 : 2))
    k_banded_dp_queue(DpKernelArgs a, unsigned long long* __restrict__ head, int chunk) {
  __shared__ int2 tab[32 * 32];
  dp_table_init(tab);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const unsigned long long take = 32ull * (unsigned long long)chunk;
  const int64_t first = dp_warp_hits(a);  // the hits before it run one per warp
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(head, take);
    base = __shfl_sync(kFull, base, 0);
    if (first + (int64_t)base >= a.n) break;
    for (int c = 0; c < chunk; ++c) {
      const int64_t i = first + (int64_t)base + 32 * c + lane;
      if (i < a.n) dp_one<GAP, LOCAL>(a, tab, i);
    }
  }
}

// One hit per warp (banded_hit_warp) for the first n_warp hits of the order,
// the longest ones: a grid-stride loop over them, one warp each.
template <int GAP, bool LOCAL>
__global__ void __launch_bounds__(128) k_banded_dp_warp(DpKernelArgs a) {
  __shared__ int2 tab[32 * 32];
  dp_table_init(tab);
  __syncthreads();
  const int64_t nw = dp_warp_hits(a);
  const int lane = threadIdx.x & 31;
  const int64_t wpb = blockDim.x >> 5;
  for (int64_t i = (int64_t)blockIdx.x * wpb + (threadIdx.x >> 5); i < nw; i += (int64_t)gridDim.x * wpb) {
    const int64_t h = a.order ? (int64_t)(uint32_t)a.order[i] : i;
    const uint64_t k = a.hk[h];
    const int qidx = a.hq[h];
    const int s = a.hs[h];
    const int tid = (int)(k >> 32);
    if (dp_hit_outside(a, tid, s)) {  // the same for every lane of the warp
      if (lane == 0) dp_skip(a, h);
      continue;
    }
    const int tidx = (int)((uint32_t)k ^ 0x80000000u) + qidx;
    const int64_t tstart = a.t.gateway[tid];
    const int tlen = a.t.lengths[tid];
    const int64_t qstart = a.q.start[s];
    const int qlen = a.q.len[s];
    const int l = a.p.l;
    int t_hl = l, q_hl = l, match = l, score = l;  // CDeviceHitList.cu:283-286
    int o_tidx = tidx, o_qidx = qidx;
    banded_hit_warp<GAP, LOCAL>(tab, a.t.bases, tstart, tlen, a.q.bases, qstart, qlen, tidx, qidx, l, t_hl, q_hl,
                                match, score, o_tidx, o_qidx);
    if (lane == 0) dp_store(a, h, qlen, o_tidx, o_qidx, t_hl, q_hl, match, score);
  }
}

// Length buckets of the hits for the DP order: 16 buckets per power of two of
// the row count (rows within a bucket differ by at most 1/16), numbered so
// that ascending bucket = longest first.
constexpr int kDpBuckets = 16 * 33;
__device__ __forceinline__ int dp_bucket(int rows) {
  if (rows < 16) return kDpBuckets - 1 - rows;  // exact below 16
  const int e = 31 - __clz(rows);                // rows in [2^e, 2^(e+1))
  const int sub = (rows >> (e - 4)) & 15;
  return kDpBuckets - 1 - (16 * (e - 3) + sub);
}

__global__ void k_dp_bucket_count(const int32_t* __restrict__ hs, const int32_t* __restrict__ q_len, int64_t n, int l,
                                  unsigned int* __restrict__ count, unsigned long long* __restrict__ rows) {
  __shared__ unsigned int c[kDpBuckets];
  __shared__ unsigned long long sr[kDpBuckets];
  for (int i = threadIdx.x; i < kDpBuckets; i += blockDim.x) {
    c[i] = 0;
    sr[i] = 0;
  }
  __syncthreads();
  for (int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; h < n; h += (int64_t)gridDim.x * blockDim.x) {
    const int r = max(0, q_len[hs[h]] - l);
    const int b = dp_bucket(r);
    atomicAdd(&c[b], 1u);
    atomicAdd(&sr[b], (unsigned long long)r);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kDpBuckets; i += blockDim.x)
    if (c[i]) {
      atomicAdd(&count[i], c[i]);
      atomicAdd(&rows[i], sr[i]);
    }
}

// Rows of bucket b (ascending b = longest first): [dp_bucket_lo(b), dp_bucket_hi(b)].
__host__ __device__ __forceinline__ long long dp_bucket_lo(int b) {
  const int x = kDpBuckets - 1 - b;
  if (x < 16) return x;
  const int e = x / 16 + 3, sub = x % 16;
  return (long long)(16 + sub) << (e - 4);
}
__host__ __device__ __forceinline__ long long dp_bucket_hi(int b) {
  const int x = kDpBuckets - 1 - b;
  if (x < 16) return x;
  return dp_bucket_lo(b) + (1ll << (x / 16 - 1)) - 1;
}

// Cost model of the warp / thread split, in SM clock cycles, fitted on the
// B200 at gap 8 (W = 17): a hit in thread mode takes kDpThreadCellCycles per
// cell when its warp has the SM sub-partition to itself (a row is W dependent
// cells), and a full grid runs kDpThreadCellsPerCycle cells per cycle; a hit
// in warp mode takes kDpWarpRowCycles per row alone (two wavefront steps),
// and warps run kDpWarpRowsPerCycle rows per cycle over the GPU.  The two
// kernels run side by side: with L the longer of the two longest hits' times
// and I the issue time of both kernels' work, the batch takes max(L + I/2, I)
// (measured: a lone hit's rows slow down as other warps share its
// sub-partition, and the GPU cannot issue faster than I).  Forking the second
// stream and the launch cost kDpLaunchCycles.  Only the split depends on
// these; results do not.
constexpr double kDpThreadCellCycles = 34.0;
constexpr double kDpThreadCellsPerCycle = 490.0;
constexpr double kDpWarpRowCycles = 289.0;
constexpr double kDpWarpRowsPerCycle = 4.7;
constexpr double kDpLaunchCycles = 10000.0;
constexpr long long kDpWarpMinRows = 16;

// Estimated time of the DP with the `s` longest hits (rows summed: sw, the
// longest r1) one per warp and the rest (rows summed: rest, the longest rn)
// one per thread.
__host__ __device__ __forceinline__ double dp_split_cycles(int W, long long s, double r1, double sw, double rn,
                                                           double rest) {
  double lat = s > 0 ? r1 * kDpWarpRowCycles : 0.0;
  if (rest > 0) lat = fmax(lat, rn * W * kDpThreadCellCycles);
  const double issue = (s > 0 ? sw / kDpWarpRowsPerCycle : 0.0) + rest * W / kDpThreadCellsPerCycle;
  return fmax(lat + 0.5 * issue, issue) + (s > 0 ? kDpLaunchCycles : 0.0);
}

// The split on the device: every bucket boundary (longest first) is a
// candidate; the earliest estimated end wins.  One thread; ~500 buckets.
__global__ void k_dp_warp_split(const unsigned int* __restrict__ count, const unsigned long long* __restrict__ rows,
                                int W, long long cap, long long* __restrict__ warp_n) {
  if (threadIdx.x != 0) return;
  double total = 0;
  for (int b = 0; b < kDpBuckets; ++b) total += (double)rows[b];
  long long s = 0, best_s = 0;
  double sw = 0, r1 = -1, best = 0;
  bool all_taken = true;
  for (int b = 0; b < kDpBuckets; ++b) {
    if (!count[b]) continue;
    const double rn = (double)dp_bucket_hi(b);
    // candidate: the buckets before b one per warp, b and the rest one per thread
    if (r1 < 0) {
      r1 = rn;
      best = dp_split_cycles(W, 0, 0, 0, rn, total);
    } else {
      const double t = dp_split_cycles(W, s, r1, sw, rn, total - sw);
      if (t < best) { best = t; best_s = s; }
    }
    if (dp_bucket_lo(b) < kDpWarpMinRows || s + count[b] > cap) {
      all_taken = false;
      break;
    }
    s += count[b];
    sw += (double)rows[b];
  }
  if (all_taken && s > 0 && dp_split_cycles(W, s, r1, sw, 0, 0) < best) best_s = s;  // every hit one per warp
  *warp_n = best_s;
}

// exclusive scan of the bucket counts in one block (kDpBuckets <= 1024)
__global__ void k_dp_bucket_scan(const unsigned int* __restrict__ count, unsigned long long* __restrict__ cursor) {
  __shared__ unsigned long long v[1024];
  const int i = threadIdx.x;
  v[i] = i < kDpBuckets ? count[i] : 0;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const unsigned long long x = i >= o ? v[i - o] : 0;
    __syncthreads();
    v[i] += x;
    __syncthreads();
  }
  if (i < kDpBuckets) cursor[i] = v[i] - count[i];
}

__global__ void k_dp_bucket_scatter(const int32_t* __restrict__ hs, const int32_t* __restrict__ q_len, int64_t n,
                                    int l, unsigned long long* __restrict__ cursor, uint64_t* __restrict__ order) {
  const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= n) return;
  const unsigned long long at = atomicAdd(&cursor[dp_bucket(max(0, q_len[hs[h]] - l))], 1ull);
  order[at] = (uint64_t)h;
}

template <int GAP, bool LOCAL>
long long launch_dp_mode(DpKernelArgs a, const DpLaunch& m, cudaStream_t st) {
  constexpr int W = 2 * GAP + 1;
  const int threads = 128;
  struct Occupancy {
    int sms = 0, per_sm = 1, warp_per_sm = 1;
  };
  static const Occupancy occ = [] {  // once per kernel pair (thread-safe static initialisation)
    Occupancy o;
    int dev = 0;
    CLAST_CK(cudaGetDevice(&dev));
    CLAST_CK(cudaDeviceGetAttribute(&o.sms, cudaDevAttrMultiProcessorCount, dev));
    CLAST_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.per_sm, k_banded_dp_queue<GAP, LOCAL>, 128, 0));
    CLAST_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.warp_per_sm, k_banded_dp_warp<GAP, LOCAL>, 128, 0));
    o.per_sm = std::max(1, o.per_sm);
    o.warp_per_sm = std::max(1, o.warp_per_sm);
    return o;
  }();
  const int sms = occ.sms, per_sm = occ.per_sm, warp_per_sm = occ.warp_per_sm;
  // hits one per warp: at most one wave of the warp kernel's resident warps
  // (the cost model has no waves)
  const long long cap = (long long)sms * warp_per_sm * (threads / 32);
  a.warp_n = nullptr;
  a.warp_fixed = 0;
  if (m.warp == kDpWarpAll) {
    a.warp_fixed = a.n;
  } else if (m.warp == kDpWarpAuto) {
    if (m.buckets.count && m.warp_n) {
      k_dp_warp_split<<<1, 32, 0, st>>>(m.buckets.count, m.buckets.rows, W, cap, m.warp_n);
      CLAST_LAUNCHED();
      a.warp_n = m.warp_n;
    } else if (m.uniform_rows >= kDpWarpMinRows && a.n <= cap) {
      const double r = (double)m.uniform_rows, rows = r * (double)a.n;
      if (dp_split_cycles(W, a.n, r, rows, 0, 0) < dp_split_cycles(W, 0, 0, 0, r, rows)) a.warp_fixed = a.n;
    }
  }
  const int64_t rest = a.n - (a.warp_n ? 0 : a.warp_fixed);  // hits left for the one-per-thread kernels (at most)
  bool joined = false;
  if (a.warp_n || a.warp_fixed > 0) {
    const long long most = a.warp_n ? std::min<long long>(cap, a.n) : a.warp_fixed;
    const long long blocks = std::min<long long>((most + 3) / 4, (long long)sms * warp_per_sm);
    cudaStream_t sw = st;
    if (m.aux && m.ev_fork && m.ev_join && rest > 0) {  // beside the one-per-thread kernel
      CLAST_CK(cudaEventRecord(m.ev_fork, st));
      CLAST_CK(cudaStreamWaitEvent(m.aux, m.ev_fork, 0));
      sw = m.aux;
    }
    k_banded_dp_warp<GAP, LOCAL><<<(unsigned)std::max<long long>(1, blocks), threads, 0, sw>>>(a);
    CLAST_LAUNCHED();
    if (sw != st) {
      CLAST_CK(cudaEventRecord(m.ev_join, sw));
      joined = true;
    }
  }
  const long long warp_hits = a.warp_n ? -1 : a.warp_fixed;
  if (rest <= 0) return warp_hits;
  // a batch that fits in one wave of the grid runs one hit per thread: the
  // queue's takes of several hits per lane would only lengthen the longest
  if (m.head == nullptr || rest <= (int64_t)sms * per_sm * threads) {
    const unsigned grid = (unsigned)((rest + threads - 1) / threads);
    k_banded_dp<GAP, LOCAL><<<grid, threads, 0, st>>>(a);
  } else {
    const int64_t need = (rest + 32 * m.chunk - 1) / (32 * m.chunk) / (threads / 32) + 1;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)sms * per_sm, need));
    CLAST_CK(cudaMemsetAsync(m.head, 0, sizeof(unsigned long long), st));
    k_banded_dp_queue<GAP, LOCAL><<<grid, threads, 0, st>>>(a, m.head, m.chunk);
  }
  CLAST_LAUNCHED();
  if (joined) CLAST_CK(cudaStreamWaitEvent(st, m.ev_join, 0));
  return warp_hits;
}

template <int GAP>
long long launch_dp_gap(const DpKernelArgs& a, bool local, const DpLaunch& m, cudaStream_t st) {
  return local ? launch_dp_mode<GAP, true>(a, m, st) : launch_dp_mode<GAP, false>(a, m, st);
}

// ------------------------------------------------------------------------
// final per-read order
// ------------------------------------------------------------------------
__global__ void k_final_keys(const uint64_t* __restrict__ hk, const int32_t* __restrict__ hq,
                             const int32_t* __restrict__ hs, DpOut o, int64_t n, uint64_t* __restrict__ k1,
                             uint64_t* __restrict__ k2, int32_t* __restrict__ idx) {
  const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= n) return;
  if (!o.keep[h]) {  // filtered hits sort after every kept one
    k1[h] = ~0ull;
    k2[h] = ~0ull;
    idx[h] = (int32_t)h;
    return;
  }
  const uint64_t k = hk[h];
  const int qidx = hq[h];
  const int tid = (int)(k >> 32);
  const int tidx = (int)((uint32_t)k ^ 0x80000000u) + qidx;
  // (score desc, seed qIdx desc, strand, target sequence, seed tIdx): the order the
  // stable sorts of alignmentHits (by rows desc, then qIdx desc) and
  // resultSorting (qID/2 asc, score desc) leave hits of one read in.
  const uint32_t a1 = (uint32_t)((int64_t)INT_MAX - (int64_t)o.score[h]);
  const uint32_t a2 = (uint32_t)((int64_t)INT_MAX - (int64_t)qidx);
  k1[h] = ((uint64_t)a1 << 32) | a2;
  k2[h] = ((uint64_t)(hs[h] & 1) << 62) | ((uint64_t)(uint32_t)tid << 31) | (uint64_t)(uint32_t)tidx;
  idx[h] = (int32_t)h;
}

__global__ void k_read_ranges(const int64_t* __restrict__ hoff, int64_t n_reads, int64_t* __restrict__ roff,
                              int32_t* __restrict__ rlen) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_reads) return;
  roff[r] = hoff[2 * r];
  rlen[r] = (int32_t)(hoff[2 * r + 2] - hoff[2 * r]);
}

// Duplicate removal within one read (deleteHits_duplicateResult: a hit equal
// in (tID, tIdx, qID, qIdx) to its predecessor in result order is dropped).
__global__ void k_final_dedupe(const uint64_t* __restrict__ k1, const int32_t* __restrict__ idx,
                               const uint64_t* __restrict__ hk, const int32_t* __restrict__ hs, DpOut o,
                               const int64_t* __restrict__ roff, const int32_t* __restrict__ rlen,
                               int64_t n_reads, int32_t* __restrict__ fcnt, int32_t* __restrict__ fsel) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_reads) return;
  const int64_t a = roff[r];
  const int n = rlen[r];
  int cnt = 0;
  int ptid = 0, ptidx = 0, ps = 0, pqidx = 0;
  for (int j = 0; j < n; ++j) {
    if (k1[a + j] == ~0ull) break;  // the filtered hits
    const int h = idx[a + j];
    const int tid = (int)(hk[h] >> 32);
    const int tidx = o.t_idx[h], qidx = o.q_idx[h], s = hs[h];
    const bool dup = j > 0 && tid == ptid && tidx == ptidx && s == ps && qidx == pqidx;
    if (!dup) fsel[a + cnt++] = h;
    ptid = tid; ptidx = tidx; ps = s; pqidx = qidx;
  }
  fcnt[r] = cnt;
}

__global__ void k_final_compact(const int32_t* __restrict__ fsel, const int64_t* __restrict__ roff,
                                const int32_t* __restrict__ fcnt, const int64_t* __restrict__ foff,
                                int64_t n_reads, const uint64_t* __restrict__ hk, const int32_t* __restrict__ hs,
                                DpOut o, int32_t t_first, int32_t q_first, FinalOut out) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_reads) return;
  const int64_t a = roff[r], b = foff[r];
  const int n = fcnt[r];
  for (int j = 0; j < n; ++j) {
    const int h = fsel[a + j];
    const int64_t w = b + j;
    out.t_id[w] = t_first + (int32_t)(hk[h] >> 32);
    out.t_idx[w] = o.t_idx[h];
    out.q_id[w] = q_first + hs[h];
    out.q_idx[w] = o.q_idx[h];
    out.t_len[w] = o.t_len[h];
    out.q_len[w] = o.q_len[h];
    out.match[w] = o.match[h];
    out.score[w] = o.score[h];
    out.evalue[w] = o.evalue[h];
  }
}

// ------------------------------------------------------------------------
// merge of the per-window results in holder order (CHostResultHolder::fixResult)
// ------------------------------------------------------------------------
__global__ void k_merge_count(const WinHits* __restrict__ w, int nw, int64_t nreads, int32_t* __restrict__ cnt) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nreads) return;
  int64_t c = 0;
  for (int i = 0; i < nw; ++i) c += w[i].foff[r + 1] - w[i].foff[r];
  cnt[r] = (int32_t)c;
}

// Item j of window wi goes after every item of the same read from an earlier
// window with score >= its score, and every item of a later window with a
// strictly higher score: the stable sort by (read, score desc) of the
// concatenation in window order.
__global__ void k_merge_place(const WinHits* __restrict__ w, int nw, int64_t total, const int64_t* __restrict__ moff,
                              MapOut out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  int wi = 0;
  while (wi + 1 < nw && w[wi + 1].base <= i) ++wi;
  const WinHits& a = w[wi];
  const int64_t j = i - a.base;
  const int qid = a.q_id[j];
  const int64_t r = qid >> 1;
  const int sc = a.score[j];
  int64_t pos = moff[r] + (j - a.foff[r]);
  for (int k = 0; k < nw; ++k) {
    if (k == wi) continue;
    const WinHits& b = w[k];
    int64_t lo = b.foff[r], hi = b.foff[r + 1];
    const int64_t first = lo;
    // scores are non-increasing within a read: count the prefix that precedes sc
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      const int v = b.score[mid];
      if (k < wi ? v >= sc : v > sc) lo = mid + 1;
      else hi = mid;
    }
    pos += lo - first;
  }
  out.read[pos] = qid >> 1;
  out.strand[pos] = qid & 1;
  out.t_load[pos] = a.load;
  out.t_seq[pos] = a.t_id[j];
  out.t_idx[pos] = a.t_idx[j];
  out.q_idx[pos] = a.q_idx[j];
  out.t_len[pos] = a.t_len[j];
  out.q_len[pos] = a.q_len[j];
  out.match[pos] = a.match[j];
  out.score[pos] = sc;
  out.evalue[pos] = a.evalue[j];
}

// INT32 throughput probe: 8 independent chains per thread of the DP's
// integer operation mix (add, max, logic): 4 ops per chain and iteration.
__global__ void __launch_bounds__(256) k_int32_probe(int iters, int k1, int k2, int* __restrict__ sink) {
  int a[8], b[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    a[c] = threadIdx.x + c * k1;
    b[c] = blockIdx.x - c * k2;
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      a[c] = max(a[c] + k1, b[c]);
      b[c] = (b[c] ^ a[c]) + k2;
    }
  }
  int x = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) x += a[c] ^ b[c];
  if (x == 0x7fffffff) sink[0] = x;  // keeps the chains live
}

__global__ void k_gather_i64(const int64_t* __restrict__ src, const int64_t* __restrict__ idx, int n,
                             int64_t* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = src[idx[i]];
}

}  // namespace

// ------------------------------------------------------------------------
// launch wrappers
// ------------------------------------------------------------------------
void scan_i32(Workspace& ws, const int32_t* in, int64_t n, int64_t* out, cudaStream_t st) {
  scan_1pass(ws, ArrayLoad<int32_t>{in}, n, out, st);
}
void scan_positive(Workspace& ws, const int32_t* in, int64_t n, int64_t* out, cudaStream_t st) {
  scan_1pass(ws, PositiveLoad{in}, n, out, st);
}

void pack_bases(const char* bases, int64_t n, uint64_t* packed, uint64_t* nmask, cudaStream_t st) {
  const int64_t nwords = (n + 63) / 64 + 1;  // one extra word so kmer_at may read w+1
  k_pack<<<blocks_for(nwords, 256), 256, 0, st>>>(bases, n, packed, nmask, nwords);
  CLAST_LAUNCHED();
}

void build_strands(const char* reads, const int64_t* offsets, int64_t n_reads, int64_t n_bases, char* strands,
                   int64_t* strand_start, int32_t* strand_len, cudaStream_t st) {
  if (n_reads <= 0) return;
  k_strand_meta<<<blocks_for(n_reads, 256), 256, 0, st>>>(offsets, n_reads, strand_start, strand_len);
  CLAST_LAUNCHED();
  if (n_bases > 0) {
    k_strands<<<blocks_for(n_reads * 32, 256), 256, 0, st>>>(reads, offsets, n_reads, strands);
    CLAST_LAUNCHED();
  }
}

void build_window(const char* src, const int64_t* src_off, const int32_t* gateway, const int32_t* lengths,
                  int nseqs, int64_t n, char* out, cudaStream_t st) {
  if (n <= 0 || nseqs <= 0) return;
  k_build_window<<<blocks_for((n + 15) / 16, 256), 256, 0, st>>>(src, src_off, gateway, lengths, nseqs, n, out);
  CLAST_LAUNCHED();
}

void sample_keys(const uint64_t* packed, const uint64_t* nmask, int64_t n_samples, int stride, int l, int pbits,
                 uint64_t* items, int32_t* vals, cudaStream_t st) {
  if (n_samples <= 0) return;
  k_sample_keys<<<blocks_for(n_samples, 256), 256, 0, st>>>(packed, nmask, n_samples, stride, l, pbits, items,
                                                             vals);
  CLAST_LAUNCHED();
}

void split_items(const uint64_t* items, int64_t n, int pbits, uint64_t bound, uint64_t* keys, int32_t* vals,
                 int32_t* head, cudaStream_t st) {
  if (n <= 0) return;
  k_split_items<<<blocks_for(n, 256), 256, 0, st>>>(items, n, pbits, bound, keys, vals, head);
  CLAST_LAUNCHED();
}

int radix_sort_u64(Workspace& ws, uint64_t* keys, int32_t* vals, uint64_t* keys_alt, int32_t* vals_alt, int64_t n,
                   int lo_bit, int hi_bit, cudaStream_t st) {
  if (n <= 1) return 0;
  const int nblocks = (int)((n + kRsTile - 1) / kRsTile);
  uint32_t* hist = ws.get<uint32_t>("rs_hist", (size_t)256 * nblocks);
  int64_t* offs = ws.get<int64_t>("rs_offs", (size_t)256 * nblocks + 1);
  const bool pay = vals != nullptr;
  const size_t smem = (size_t)kRsTile * (sizeof(uint64_t) + (pay ? sizeof(int32_t) : 0));
  // more than 48 KB of dynamic shared memory needs the opt-in (per device)
  if (pay) CLAST_CK(cudaFuncSetAttribute(k_rs_scatter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  else CLAST_CK(cudaFuncSetAttribute(k_rs_scatter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  uint64_t* a = keys;
  uint64_t* b = keys_alt;
  int32_t* va = vals;
  int32_t* vb = vals_alt;
  int which = 0;
  for (int shift = lo_bit; shift < hi_bit; shift += 8) {
    k_rs_hist<<<nblocks, kRsThreads, 0, st>>>(a, n, shift, hist, nblocks);
    CLAST_LAUNCHED();
    scan_1pass(ws, ArrayLoad<uint32_t>{hist}, (int64_t)256 * nblocks, offs, st);
    if (pay) k_rs_scatter<true><<<nblocks, kRsThreads, smem, st>>>(a, va, b, vb, n, shift, offs, nblocks);
    else k_rs_scatter<false><<<nblocks, kRsThreads, smem, st>>>(a, nullptr, b, nullptr, n, shift, offs, nblocks);
    CLAST_LAUNCHED();
    std::swap(a, b);
    std::swap(va, vb);
    which ^= 1;
  }
  return which;
}

void count_below(const uint64_t* keys, int64_t n, uint64_t bound, int64_t* out, cudaStream_t st) {
  k_count_below<<<1, 1, 0, st>>>(keys, n, bound, out);
  CLAST_LAUNCHED();
}

void index_heads(const uint64_t* keys, int64_t n, uint64_t bound, int32_t* head, cudaStream_t st) {
  if (n <= 0) return;
  k_index_heads<<<blocks_for(n, 256), 256, 0, st>>>(keys, n, bound, head);
  CLAST_LAUNCHED();
}
void index_unique(const uint64_t* keys, const int32_t* head, const int64_t* hpos, int64_t n, const int64_t* nv_dev,
                  uint64_t* ukeys, int64_t* ufirst, cudaStream_t st) {
  k_index_unique<<<blocks_for(n > 0 ? n : 1, 256), 256, 0, st>>>(keys, head, hpos, n, nv_dev, ukeys, ufirst);
  CLAST_LAUNCHED();
}
void index_keep(const int32_t* vals, const int64_t* hpos, const int64_t* ufirst, int64_t n, const int64_t* nv_dev,
                int stride, int l, int cut, const int32_t* gateway, const int32_t* lengths, int nseqs, int32_t* keep,
                int2* resolved, cudaStream_t st) {
  if (n <= 0) return;
  k_index_keep<<<blocks_for(n, 256), 256, 0, st>>>(vals, hpos, ufirst, n, nv_dev, stride, l, cut, gateway, lengths,
                                                   nseqs, keep, resolved);
  CLAST_LAUNCHED();
}
void index_entries(const int32_t* keep, const int64_t* kpos, const int2* resolved, int64_t nv, int2* entries,
                   cudaStream_t st) {
  if (nv <= 0) return;
  k_index_entries<<<blocks_for(nv, 256), 256, 0, st>>>(keep, kpos, resolved, nv, entries);
  CLAST_LAUNCHED();
}
void index_buckets(const int64_t* ufirst, const int64_t* kpos, int64_t n, const int64_t* nu_dev, int32_t* ustart,
                   int32_t* ucnt, cudaStream_t st) {
  if (n <= 0) return;
  k_index_buckets<<<blocks_for(n, 256), 256, 0, st>>>(ufirst, kpos, n, nu_dev, ustart, ucnt);
  CLAST_LAUNCHED();
}


int seed_parts() { return kSeedParts; }

void seed_fused(const QueryView& q, const IndexView& ix, const TargetView& t, int gap, int local,
                unsigned long long* cursors, unsigned long long* n_kmers, int64_t* off, int32_t* cnt, int32_t* nvalid,
                uint64_t* skey, uint32_t* sq, int64_t part_cap, cudaStream_t st) {
  if (q.nstrands <= 0) return;
  // one warp per strand (one resident wave looping over the strands measured slower)
  const unsigned grid = blocks_for((int64_t)q.nstrands * 32, kSeedFusedThreads);
  if (ix.l <= 16)
    k_seed_fused<true><<<grid, kSeedFusedThreads, 0, st>>>(q, ix, t, gap, local, cursors, n_kmers, off, cnt, nvalid,
                                                          skey, sq, part_cap);
  else
    k_seed_fused<false><<<grid, kSeedFusedThreads, 0, st>>>(q, ix, t, gap, local, cursors, n_kmers, off, cnt, nvalid,
                                                           skey, sq, part_cap);
  CLAST_LAUNCHED();
}

template <int NW>
void launch_seed_multi(const QueryView& q, const SeedWins& W, int gap, int local, cudaStream_t st) {
  const unsigned grid = blocks_for((int64_t)q.nstrands * 32, kSeedFusedThreads);
  if (W.w[0].ix.l <= 16) k_seed_multi<true, NW><<<grid, kSeedFusedThreads, 0, st>>>(q, W, gap, local);
  else k_seed_multi<false, NW><<<grid, kSeedFusedThreads, 0, st>>>(q, W, gap, local);
  CLAST_LAUNCHED();
}

void seed_multi(const QueryView& q, const SeedWins& W, int nw, int gap, int local, cudaStream_t st) {
  if (q.nstrands <= 0 || nw <= 0) return;
  switch (nw) {
    case 1: launch_seed_multi<1>(q, W, gap, local, st); break;
    case 2: launch_seed_multi<2>(q, W, gap, local, st); break;
    case 3: launch_seed_multi<3>(q, W, gap, local, st); break;
    case 4: launch_seed_multi<4>(q, W, gap, local, st); break;
    default: throw std::invalid_argument("seed_multi: 1 to 4 windows per pass");
  }
}

template <class Load>
void maxscan_impl(Workspace& ws, Load in, int64_t n, int64_t* out, cudaStream_t st, int level) {
  if (n <= 0) return;
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  const std::string tag = "maxscan" + std::to_string(level);
  int64_t* tmax = ws.get<int64_t>(tag + "m", tiles);
  k_maxscan_tiles<Load><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, out, tmax);
  CLAST_LAUNCHED();
  if (tiles > 1) {
    int64_t* trun = ws.get<int64_t>(tag + "r", tiles);
    maxscan_impl(ws, ArrayLoad<int64_t>{tmax}, tiles, trun, st, level + 1);
    k_maxscan_apply<<<blocks_for(n, 256), 256, 0, st>>>(out, n, trun);
    CLAST_LAUNCHED();
  }
}

void table_runmax(Workspace& ws, const uint64_t* ucode, const int32_t* ucnt, const int64_t* rank, int64_t n_unique,
                  int l, uint32_t nbuckets, int64_t* run_max, cudaStream_t st) {
  maxscan_impl(ws, SlackLoad{ucode, ucnt, rank, l, nbuckets}, n_unique, run_max, st, 0);
}

void table_place(const uint64_t* ucode, const int32_t* ustart, const int32_t* ucnt, const int2* entries,
                 const int64_t* rank, const int64_t* run_max, int64_t n_unique, ulonglong2* table, int64_t n_records,
                 uint32_t* filter, int fshift, unsigned long long* failed, cudaStream_t st) {
  if (n_unique <= 0) return;
  k_table_place<<<blocks_for(n_unique, 256), 256, 0, st>>>(ucode, ustart, ucnt, entries, rank, run_max, n_unique,
                                                            table, n_records, filter, fshift, failed);
  CLAST_LAUNCHED();
}

void window_first(const int32_t* nvalid, const int32_t* win_start, int n_windows, int32_t* win_first,
                  cudaStream_t st) {
  if (n_windows <= 0) return;
  k_window_first<<<blocks_for((int64_t)n_windows * 32, 256), 256, 0, st>>>(nvalid, win_start, n_windows,
                                                                            win_first);
  CLAST_LAUNCHED();
}
void segmented_sort_u64(Workspace& ws, uint64_t* k1, uint64_t* k2, int32_t* payload, const int64_t* off,
                        const int32_t* len, int64_t n_segments, cudaStream_t st, int tag) {
  seg_sort<uint64_t, true>(ws, k1, k2, payload, off, len, n_segments, st, tag);
}
void seed_sort_filter(Workspace& ws, uint64_t* skey, uint32_t* sq, const int64_t* off, const int32_t* cnt,
                      const int32_t* nvalid, const int32_t* win_start, int n_windows, const int32_t* win_first,
                      int width, int gap, int64_t nstrands, int32_t* hcnt, cudaStream_t st) {
  if (nstrands <= 0) return;
  SeedFilterCtx c{off, cnt, nvalid, win_start, n_windows, win_first, width, gap, hcnt};
  if (nstrands >= (int64_t)kWinFirstBit) throw std::invalid_argument("more than 2^31 strands in one batch");
  int32_t* lists = ws.get<int32_t>("ssf_lists", kSortTiers * nstrands);
  int32_t* counts = ws.get<int32_t>("ssf_counts", kSortTiers);
  CLAST_CK(cudaMemsetAsync(counts, 0, kSortTiers * sizeof(int32_t), st));
  CLAST_CK(cudaMemsetAsync(hcnt, 0, nstrands * sizeof(int32_t), st));
  k_seed_classify<<<blocks_for(nstrands, 256), 256, 0, st>>>(c, nstrands, lists, counts);
  CLAST_LAUNCHED();
  k_seed_sort_filter_thread<<<grid_cap((nstrands + 255) / 256), 256, 0, st>>>(skey, sq, c, lists, counts);
  CLAST_LAUNCHED();
  k_seed_sort_filter_warp<<<grid_cap((nstrands * 32 + 255) / 256), 256, 0, st>>>(skey, sq, c, lists + nstrands,
                                                                                counts + 1);
  CLAST_LAUNCHED();
  k_seed_sort_filter_warp_smem<<<grid_cap(std::min<int64_t>(nstrands, 65536) * 32 / kWarpSmemThreads + 1),
                                 kWarpSmemThreads, 0, st>>>(skey, sq, c, lists + 2 * nstrands, counts + 2);
  CLAST_LAUNCHED();
  k_seed_sort_filter_cta<<<grid_cap(nstrands < 4096 ? nstrands : 4096), 256, 0, st>>>(skey, sq, c,
                                                                                     lists + 3 * nstrands, counts + 3);
  CLAST_LAUNCHED();
  k_seed_sort_filter_global<<<grid_cap(nstrands < 1024 ? nstrands : 1024), 1024, 0, st>>>(
      skey, sq, c, lists + 4 * nstrands, counts + 4);
  CLAST_LAUNCHED();
}

void gather_hits(const uint64_t* skey, const uint32_t* sq, const int64_t* off, const int32_t* hcnt,
                 const int64_t* hoff, int64_t nstrands, uint64_t* hk, int32_t* hq, int32_t* hs,
                 const int32_t* qlen, int l, int band, unsigned long long* cells, cudaStream_t st) {
  if (nstrands <= 0) return;
  k_gather_hits<<<blocks_for(nstrands, 256), 256, 0, st>>>(skey, sq, off, hcnt, hoff, nstrands, hk, hq, hs, qlen, l,
                                                           band, cells);
  CLAST_LAUNCHED();
}

__global__ void k_dp_order_keys(const int32_t* __restrict__ hs, const int32_t* __restrict__ q_len, int64_t n,
                                int l, int rows_max, uint64_t* __restrict__ keys) {
  const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= n) return;
  const int rows = max(0, min(rows_max, q_len[hs[h]] - l + 1));
  keys[h] = ((uint64_t)(rows_max - rows) << 32) | (uint32_t)h;
}

void dp_order_keys(const int32_t* hs, const int32_t* q_len, int64_t n_hits, int l, int rows_max, uint64_t* keys,
                   cudaStream_t st) {
  if (n_hits <= 0) return;
  k_dp_order_keys<<<blocks_for(n_hits, 256), 256, 0, st>>>(hs, q_len, n_hits, l, rows_max, keys);
  CLAST_LAUNCHED();
}

DpBuckets dp_bucket_count(Workspace& ws, const int32_t* hs, const int32_t* q_len, int64_t n_hits, int l,
                          cudaStream_t st) {
  unsigned int* count = ws.get<unsigned int>("dpb_count", kDpBuckets);
  unsigned long long* rows = ws.get<unsigned long long>("dpb_rows", kDpBuckets);
  CLAST_CK(cudaMemsetAsync(count, 0, kDpBuckets * sizeof(unsigned int), st));
  CLAST_CK(cudaMemsetAsync(rows, 0, kDpBuckets * sizeof(unsigned long long), st));
  if (n_hits > 0) {
    k_dp_bucket_count<<<grid_cap(std::min<int64_t>(blocks_for(n_hits, 256), 1184)), 256, 0, st>>>(hs, q_len, n_hits,
                                                                                                    l, count, rows);
    CLAST_LAUNCHED();
  }
  DpBuckets b;
  b.count = count;
  b.rows = rows;
  return b;
}

DpBuckets dp_bucket_order(Workspace& ws, const int32_t* hs, const int32_t* q_len, int64_t n_hits, int l,
                          uint64_t* order, cudaStream_t st) {
  const DpBuckets b = dp_bucket_count(ws, hs, q_len, n_hits, l, st);
  if (n_hits <= 0) return b;
  unsigned long long* cursor = ws.get<unsigned long long>("dpb_cursor", kDpBuckets);
  k_dp_bucket_scan<<<1, 1024, 0, st>>>(b.count, cursor);
  CLAST_LAUNCHED();
  k_dp_bucket_scatter<<<blocks_for(n_hits, 256), 256, 0, st>>>(hs, q_len, n_hits, l, cursor, order);
  CLAST_LAUNCHED();
  return b;
}

int dp_warp_mode_from_env(int fallback) {
  const char* v = std::getenv("CLAST_DP_WARP");
  if (!v) return fallback;
  if (!std::strcmp(v, "off")) return kDpWarpOff;
  if (!std::strcmp(v, "all")) return kDpWarpAll;
  return fallback;
}

long long banded_dp(const TargetView& t, const QueryView& q, const uint64_t* hk, const int32_t* hq,
                    const int32_t* hs, const uint64_t* order, int64_t n_hits, const DpParams& p, const DpOut& o,
                    cudaStream_t st, const DpLaunch& m) {
  if (n_hits <= 0) return 0;
  DpKernelArgs a{t, q, hk, hq, hs, order, n_hits, p, o, nullptr, 0, m.bad};
  const bool local = p.local != 0;
  switch (p.gap) {
    case 2: return launch_dp_gap<2>(a, local, m, st);
    case 3: return launch_dp_gap<3>(a, local, m, st);
    case 4: return launch_dp_gap<4>(a, local, m, st);
    case 5: return launch_dp_gap<5>(a, local, m, st);
    case 6: return launch_dp_gap<6>(a, local, m, st);
    case 7: return launch_dp_gap<7>(a, local, m, st);
    case 8: return launch_dp_gap<8>(a, local, m, st);
    case 9: return launch_dp_gap<9>(a, local, m, st);
    case 10: return launch_dp_gap<10>(a, local, m, st);
    case 11: return launch_dp_gap<11>(a, local, m, st);
    case 12: return launch_dp_gap<12>(a, local, m, st);
    case 13: return launch_dp_gap<13>(a, local, m, st);
    case 14: return launch_dp_gap<14>(a, local, m, st);
    case 15: return launch_dp_gap<15>(a, local, m, st);
    case 16: return launch_dp_gap<16>(a, local, m, st);
    default: throw std::invalid_argument("gap out of range 2..16");
  }
}

void merge_windows(const WinHits* wins, int nw, int64_t total, int64_t nreads, int32_t* cnt, int64_t* moff,
                   const MapOut& out, Workspace& ws, cudaStream_t st) {
  if (nreads <= 0) return;
  k_merge_count<<<blocks_for(nreads, 256), 256, 0, st>>>(wins, nw, nreads, cnt);
  CLAST_LAUNCHED();
  scan_i32(ws, cnt, nreads, moff, st);
  if (total > 0) {
    k_merge_place<<<blocks_for(total, 256), 256, 0, st>>>(wins, nw, total, moff, out);
    CLAST_LAUNCHED();
  }
}

double int32_probe(cudaStream_t st, int* sink) {
  int dev = 0, sms = 0;
  CLAST_CK(cudaGetDevice(&dev));
  CLAST_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 8, threads = 256, iters = 4096;
  cudaEvent_t a, b;
  CLAST_CK(cudaEventCreate(&a));
  CLAST_CK(cudaEventCreate(&b));
  k_int32_probe<<<blocks, threads, 0, st>>>(64, 3, 5, sink);  // warm-up
  CLAST_LAUNCHED();
  CLAST_CK(cudaEventRecord(a, st));
  k_int32_probe<<<blocks, threads, 0, st>>>(iters, 3, 5, sink);
  CLAST_LAUNCHED();
  CLAST_CK(cudaEventRecord(b, st));
  CLAST_CK(cudaEventSynchronize(b));
  float ms = 0;
  CLAST_CK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  const double ops = (double)blocks * threads * iters * 8 * 4;
  return ops / (ms * 1e-3) / 1e12;
}

void gather_i64(const int64_t* src, const int64_t* idx, int n, int64_t* out, cudaStream_t st) {
  if (n <= 0) return;
  k_gather_i64<<<blocks_for(n, 256), 256, 0, st>>>(src, idx, n, out);
  CLAST_LAUNCHED();
}

void final_keys(const uint64_t* hk, const int32_t* hq, const int32_t* hs, const DpOut& o, int64_t n_hits,
                uint64_t* k1, uint64_t* k2, int32_t* idx, cudaStream_t st) {
  if (n_hits <= 0) return;
  k_final_keys<<<blocks_for(n_hits, 256), 256, 0, st>>>(hk, hq, hs, o, n_hits, k1, k2, idx);
  CLAST_LAUNCHED();
}
void read_ranges(const int64_t* hoff, int64_t n_reads, int64_t* roff, int32_t* rlen, cudaStream_t st) {
  if (n_reads <= 0) return;
  k_read_ranges<<<blocks_for(n_reads, 256), 256, 0, st>>>(hoff, n_reads, roff, rlen);
  CLAST_LAUNCHED();
}
void final_dedupe(const uint64_t* k1, const uint64_t* /*k2*/, const int32_t* idx, const uint64_t* hk,
                  const int32_t* hs, const DpOut& o, const int64_t* roff, const int32_t* rlen, int64_t n_reads,
                  int32_t* fcnt, int32_t* fsel, cudaStream_t st) {
  if (n_reads <= 0) return;
  k_final_dedupe<<<blocks_for(n_reads, 128), 128, 0, st>>>(k1, idx, hk, hs, o, roff, rlen, n_reads, fcnt, fsel);
  CLAST_LAUNCHED();
}
void final_compact(const int32_t* fsel, const int64_t* roff, const int32_t* fcnt, const int64_t* foff,
                   int64_t n_reads, const uint64_t* hk, const int32_t* hs, const DpOut& o, int32_t t_first,
                   int32_t q_first, const FinalOut& out, cudaStream_t st) {
  if (n_reads <= 0) return;
  k_final_compact<<<blocks_for(n_reads, 128), 128, 0, st>>>(fsel, roff, fcnt, foff, n_reads, hk, hs, o, t_first,
                                                             q_first, out);
  CLAST_LAUNCHED();
}

}  // namespace clast
