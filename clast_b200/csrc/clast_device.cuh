// clast_device.cuh -- device-side data structures and helpers shared by the
// kernels of libclast_b200 (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace clast {

constexpr int kPad = 64;            // 'N' bytes before and after every device base array
constexpr int kMarginScore = -30000;  // krnlAlignment.cu:20-23
constexpr int kGapOpen = -5;        // common.hpp:40
constexpr int kGapExtend = -2;      // common.hpp:41
constexpr int kBadClass = 23;       // 'X' - 'A': the bad-area letter (common.hpp:36)
constexpr int kNClass = 13;         // 'N' - 'A'
constexpr uint64_t kDroppedSeed = ~0ull;

// Resident index of one target window (the tables of CDeviceHashTable,
// CDeviceHashTable.cuh:13-16, reorganised for direct lookup).
struct IndexView {
  int l;
  int fshift;              // key >> fshift = bit of the presence filter
  const uint32_t* filter;  // one bit per (key >> fshift) of every indexed key
  int shift;               // key >> shift = directory slot
  const uint32_t* dir;     // (1 << dir_bits) + 1 entries: first unique key with slot >= p
  const uint64_t* ukeys;   // unique valid keys, ascending
  const int32_t* ustart;   // first entry of each key
  const int32_t* ucnt;     // entries of each key (0 when the repeat cut removes the key)
  const int2* entries;     // (sequence within window, index within sequence), non-joint only
  int64_t n_unique;
};

// Target window for the DP and the corner filter.
struct TargetView {
  const char* bases;       // window base array incl. joints; bases[-kPad .. n+kPad) readable
  int64_t n;
  const int32_t* gateway;  // window-relative sequence starts
  const int32_t* lengths;
  int32_t nseqs;
};

// A batch of query strands (any number of query windows).
struct QueryView {
  const char* bases;       // strand bases; bases[-kPad .. n+kPad) readable
  int64_t n;
  const uint64_t* packed;  // 2-bit codes, 32 bases per word, first base in the top bits
  const uint64_t* nmask;   // 1 bit per base (non-ACGT), 64 per word, first base in the top bit
  const int64_t* start;    // per strand: offset of its first base
  const int32_t* len;      // per strand length
  int32_t nstrands;
};

__device__ __forceinline__ int base_class(char b) {
  const int c = (int)b - 'A';
  return (c >= 0 && c < 26) ? c : kNClass;
}

// l-mer key at flat position f (SRead2bit.cuh:6-21 with SRepelHasOddBase.cuh:6-14):
// false when any of the l bases is not A/C/G/T.
// Streamed loads (evict-first in L2) so that the words of the query, read once,
// do not push the presence filter out of L2.
__device__ __forceinline__ uint64_t ld_stream(const uint64_t* p) {
  return (uint64_t)__ldcs(reinterpret_cast<const unsigned long long*>(p));
}

__device__ __forceinline__ bool kmer_at(const uint64_t* packed, const uint64_t* nmask, int64_t f,
                                        int l, uint64_t& key) {
  const int64_t w = f >> 6;
  const int o = (int)(f & 63);
  uint64_t m = ld_stream(nmask + w) << o;
  if (o) m |= ld_stream(nmask + w + 1) >> (64 - o);
  if (m >> (64 - l)) return false;
  const int64_t w2 = f >> 5;
  const int o2 = (int)(f & 31) * 2;
  uint64_t b = ld_stream(packed + w2) << o2;
  if (o2) b |= ld_stream(packed + w2 + 1) >> (64 - o2);
  key = b >> (64 - 2 * l);
  return true;
}

// Index of key among the unique keys, or -1 (krnlBinarySearch.cu:3-33).  The
// presence filter (<= 128 MB, mostly L2-resident) answers the common miss
// without touching the directory or the key array.
__device__ __forceinline__ int64_t index_lookup(const IndexView& ix, uint64_t key) {
  const uint64_t fb = key >> ix.fshift;
  if (!((ix.filter[fb >> 5] >> (fb & 31)) & 1u)) return -1;
  const uint32_t p = (uint32_t)(key >> ix.shift);
  int64_t lo = __ldcs(ix.dir + p);
  const int64_t end = __ldcs(ix.dir + p + 1);
  int64_t hi = end;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (ld_stream(ix.ukeys + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return (lo < end && ld_stream(ix.ukeys + lo) == key) ? lo : -1;
}

}  // namespace clast
