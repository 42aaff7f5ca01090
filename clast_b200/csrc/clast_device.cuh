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

// Resident index of one target window: the tables of CDeviceHashTable
// (CDeviceHashTable.cuh:13-16) reorganised for one-probe lookup.  Every key
// that keeps at least one entry after the repeat cut is a 16-byte record
// {code of the key, payload} of a linear-probing table: the code is
// order_code(key), a bijection of the 2l-bit keys; a key's home record is
// 2 * floor(code * nbuckets / 4^l), so home records rise with the code, and the
// records are placed in code order at max(home, previous + 1) (the layout
// linear probing gives in any insertion order).  Payload: the key's only entry
// (sequence within window << 32 | index within sequence) or, for keys with
// several entries, kMulti | start << 32 | count into `entries`.  A blocked
// Bloom filter (3 bits in one 32-bit word per key) answers most absent keys
// from L2.
struct IndexView {
  int l;
  int fshift;                // filter word = key_hash(code) >> fshift (fshift >= 32)
  const uint32_t* filter;
  const ulonglong2* table;   // n_records records; payload ~0 = free
  uint32_t nbuckets;         // home records are 2 * [0, nbuckets)
  int64_t n_records;         // >= 2 * nbuckets; the last record is always free
  const int2* entries;       // (sequence within window, index within sequence), non-joint only
  int64_t n_keys;            // records in use
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

// Whether any of the l bases from flat position f is not A/C/G/T.
__device__ __forceinline__ bool kmer_has_n(const uint64_t* nmask, int64_t f, int l) {
  const int64_t w = f >> 6;
  const int o = (int)(f & 63);
  uint64_t m = ld_stream(nmask + w) << o;
  if (o) m |= ld_stream(nmask + w + 1) >> (64 - o);
  return (m >> (64 - l)) != 0;
}

// 2-bit key of the l bases from flat position f (any non-ACGT base reads as A).
__device__ __forceinline__ uint64_t kmer_key(const uint64_t* packed, int64_t f, int l) {
  const int64_t w2 = f >> 5;
  const int o2 = (int)(f & 31) * 2;
  uint64_t b = ld_stream(packed + w2) << o2;
  if (o2) b |= ld_stream(packed + w2 + 1) >> (64 - o2);
  return b >> (64 - 2 * l);
}

__device__ __forceinline__ bool kmer_at(const uint64_t* packed, const uint64_t* nmask, int64_t f,
                                        int l, uint64_t& key) {
  if (kmer_has_n(nmask, f, l)) return false;
  key = kmer_key(packed, f, l);
  return true;
}

constexpr uint64_t kMulti = 1ull << 63;
constexpr uint64_t kNoPayload = ~0ull;  // also the payload of an empty record

// Code of an l-mer key: the key times an odd constant modulo 4^l, a
// bijection of the 2l-bit keys whose high bits depend on every base.
__host__ __device__ __forceinline__ uint64_t order_code(uint64_t key, int l) {
  return (key * 0xD6E8FEB86659FD93ull) & ((1ull << (2 * l)) - 1);
}
// Home record of a code: 2 * floor(code * nbuckets / 4^l).
__device__ __forceinline__ int64_t record_home(uint64_t code, int l, uint32_t nbuckets) {
  return 2 * (int64_t)__umul64hi(code << (64 - 2 * l), (uint64_t)nbuckets);
}
// The same for l <= 16 in 32-bit arithmetic.
__device__ __forceinline__ int64_t record_home16(uint32_t code, int l, uint32_t nbuckets) {
  return 2 * (int64_t)__umulhi(code << (32 - 2 * l), nbuckets);
}
// Filter hash of a code: an xorshift then a multiply by an odd constant
// (Fibonacci hashing).  The top bits select the 32-bit filter word, bits
// 16..30 the three filter bits.  (Filter words taken from the code's own top
// bits, which would let the sorted codes fill the filter without atomics,
// measured slower at lookup time.)
__host__ __device__ __forceinline__ uint64_t key_hash(uint64_t code) {
  return (code ^ (code >> 31)) * 0x9E3779B97F4A7C15ull;
}
// fshift >= 32: filter word = (h >> 32) >> (fshift - 32)
__host__ __device__ __forceinline__ uint32_t filter_word(uint64_t h, int fshift) {
  return (uint32_t)(h >> 32) >> (fshift - 32);
}
__host__ __device__ __forceinline__ uint32_t filter_mask(uint64_t h) {
  const uint32_t v = (uint32_t)(h >> 16);
  return (1u << (v & 31)) | (1u << ((v >> 5) & 31)) | (1u << ((v >> 10) & 31));
}
// Entries of a payload (0 for none).
__host__ __device__ __forceinline__ int payload_count(uint64_t p) {
  return p == kNoPayload ? 0 : ((p & kMulti) ? (int)(uint32_t)p : 1);
}

// Linear probing from record r for the key of code c.  A free record has
// payload kNoPayload (no real payload has that value), so an absent key ends
// at the first free record; the table's last record is always free.  Loads are
// evict-first so that the filter stays in L2.
__device__ __forceinline__ uint64_t table_probe(const IndexView& ix, uint64_t c, int64_t r) {
  for (; r < ix.n_records; ++r) {
    const ulonglong2 rec = __ldcs(ix.table + r);
    if (rec.x == c || rec.y == kNoPayload) return rec.y;
  }
  return kNoPayload;
}

}  // namespace clast
