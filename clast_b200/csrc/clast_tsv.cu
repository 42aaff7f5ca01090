// clast_tsv.cu -- the result text of a map (CHostResultHolder::printResult,
// CHostResultHolder.cu:131-243) behind clast_format_tsv, formatted on the GPU.
//
// printResult walks the hits of one query RAM load in order, skips a hit
// that repeats the last printed line field for field, and prints at most
// numOut lines per query label (the first line of a label always prints).
// The state it carries from hit to hit only matters inside a run of hits
// whose query labels are equal (the last printed line always belongs to the
// current run: a run's first hit always prints), so one thread walks each run
// (load starts and label changes begin a run), marks the lines to print and
// measures them; a scan places them; a second pass writes them.
//
// Numbers are written as std::ostream writes them: integers in decimal,
// doubles as %g with 6 significant digits (the E-value and the match
// percentage).  The 6-digit rounding is decided exactly: with an exact power
// of ten (10^0..10^22) the sign of value * 10^k - midpoint is taken from one
// fused multiply-add, which rounds once; beyond that range a double-double
// power of ten bounds the error, and a value too close to a rounding midpoint
// to decide, or not finite, is formatted on the host with
// snprintf (its line is left out of the device text and spliced in).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/clast_gpu.h"
#include "clast_engine.h"

using namespace clast;

namespace {

constexpr int kPowBias = 350;  // 10^k for k in [-350, 350]
// Above kBigK the table holds 10^k * 2^-256 (10^k itself would overflow) and
// the value is scaled by 2^256 first, exactly: the products are unchanged.
constexpr int kBigK = 280;
__device__ double2 g_pow10[2 * kPowBias + 1];  // (hi, lo): hi + lo = 10^k to about 64 bits

constexpr int kMaxDevices = 64;
std::mutex g_pow_mu;
bool g_pow_ready[kMaxDevices];

// Powers of ten: each read correctly rounded to the 64-bit mantissa of long
// double (strtold) and split into two doubles.
const std::vector<double2>& pow10_table() {
  static const std::vector<double2> t = [] {
    std::vector<double2> v(2 * kPowBias + 1);
    char buf[32];
    for (int k = -kPowBias; k <= kPowBias; ++k) {
      std::snprintf(buf, sizeof(buf), "1e%d", k);
      long double x = std::strtold(buf, nullptr);
      if (k > kBigK) x = ldexpl(x, -256);
      const double hi = (double)x;
      const double lo = (double)(x - (long double)hi);
      v[k + kPowBias] = make_double2(hi, lo);
    }
    return v;
  }();
  return t;
}

// The table on the current device, once per device.
void ensure_pow10(int device) {
  std::lock_guard<std::mutex> lk(g_pow_mu);
  if (device < 0 || device >= kMaxDevices) throw std::invalid_argument("device ordinal out of range");
  if (g_pow_ready[device]) return;
  const std::vector<double2>& t = pow10_table();
  CLAST_CK(cudaMemcpyToSymbol(g_pow10, t.data(), t.size() * sizeof(double2)));
  g_pow_ready[device] = true;
}

struct TsvArgs {
  int64_t n;  // hits
  const int32_t* read;
  const int32_t* strand;
  const int32_t* t_load;
  const int32_t* t_seq;
  const int32_t* t_idx;
  const int32_t* q_idx;
  const int32_t* t_len;
  const int32_t* q_len;
  const int32_t* match;
  const int32_t* score;
  const double* evalue;
  const char* q_chars;
  const int64_t* q_off;
  int64_t n_reads;
  const char* t_chars;
  const int64_t* t_off;
  int64_t n_trecs;
  const int32_t* t_start;     // may be null
  const int64_t* t_load_first;
  int32_t n_tloads;
  int32_t num_out;
};

// Decimal digits of v.
__host__ __device__ __forceinline__ int len_u(uint64_t v) {
  int k = 1;
  while (v >= 10) {
    v /= 10;
    ++k;
  }
  return k;
}
// Writes the `cnt` low decimal digits of v (zero-padded) at o, straight into
// the output (no local buffer).
__host__ __device__ __forceinline__ void put_digits(char* o, uint64_t v, int cnt) {
  for (int i = cnt - 1; i >= 0; --i) {
    o[i] = (char)('0' + v % 10);
    v /= 10;
  }
}
__host__ __device__ __forceinline__ int put_u(char* o, uint64_t v) {
  const int k = len_u(v);
  put_digits(o, v, k);
  return k;
}
__host__ __device__ __forceinline__ int put_i(char* o, int64_t v) {
  if (v < 0) {
    o[0] = '-';
    return 1 + put_u(o + 1, (uint64_t)(-v));
  }
  return put_u(o, (uint64_t)v);
}
__host__ __device__ __forceinline__ uint64_t ipow10(int k) {
  uint64_t x = 1;
  for (int i = 0; i < k; ++i) x *= 10;
  return x;
}
__host__ __device__ __forceinline__ int len_i(int64_t v) { return v < 0 ? 1 + len_u((uint64_t)(-v)) : len_u((uint64_t)v); }

// Sign of v * 10^k - m (m a half-integer near v * 10^k): -1, 0, 1, or 2 when
// it cannot be decided.
__host__ __device__ int cmp_scaled(const double2* p10, double v, int k, double m) {
  if (k >= 0 && k <= 22) {
    const double P = p10[k + kPowBias].x;  // exact
    const double d = fma(v, P, -m);            // v * P - m, rounded once: exact sign
    return d > 0 ? 1 : (d < 0 ? -1 : 0);
  }
  if (k < 0 && k >= -22) {
    const double D = p10[-k + kPowBias].x;  // exact
    const double d = fma(-m, D, v);              // v - m * D: the sign of v / D - m
    return d > 0 ? 1 : (d < 0 ? -1 : 0);
  }
  if (k < -kPowBias || k > kPowBias) return 2;
  const double2 P = p10[k + kPowBias];
  if (k > kBigK) v = ldexp(v, 256);
  const double s_hi = v * P.x;
  const double e1 = fma(v, P.x, -s_hi);
  const double d = (s_hi - m) + (e1 + v * P.y);
  if (fabs(d) < 1e-12) return 2;  // the table is good to about 2^-64 relative: |error| < 6e-14 here
  return d > 0 ? 1 : -1;
}

// v rounded to 6 significant digits at decimal exponent e: n in
// [100000, 1000000] with v ~ n * 10^(e-5), round half to even.  Returns false
// when undecided.
__host__ __device__ bool round6(const double2* p10, double v, int e, int64_t& n) {
  const int k = 5 - e;
  double s;
  if (k >= 0 && k <= 22) s = v * p10[k + kPowBias].x;
  else if (k < 0 && k >= -22) s = v / p10[-k + kPowBias].x;
  else if (k >= -kPowBias && k <= kPowBias) s = (k > kBigK ? ldexp(v, 256) : v) * p10[k + kPowBias].x;
  else return false;
  if (!(s < 1e7) || !(s > 1e4)) {  // the exponent estimate is off by more than one
    n = s >= 1e7 ? 10000000 : 0;
    return true;
  }
  const int64_t n0 = (int64_t)llrint(s);
  const int lo = cmp_scaled(p10, v, k, (double)n0 - 0.5);
  const int hi = cmp_scaled(p10, v, k, (double)n0 + 0.5);
  if (lo == 2 || hi == 2) return false;
  if (lo < 0) n = n0 - 1;
  else if (lo == 0) n = ((n0 - 1) & 1) ? n0 : n0 - 1;  // tie between n0 - 1 and n0: the even one
  else if (hi > 0) n = n0 + 1;
  else if (hi == 0) n = (n0 & 1) ? n0 + 1 : n0;
  else n = n0;
  return true;
}

// %g with precision 6 (the default of std::ostream).  Returns the length,
// writing the text at o unless o is null (length only), or -1 when the host
// must format v.  Digits go straight into o: no local buffers.
__host__ __device__ int fmt_g6(const double2* p10, double v, char* o) {
  if (!isfinite(v)) return -1;
  int len = 0;
  auto put = [&](char c) {
    if (o) o[len] = c;
    ++len;
  };
  auto digits = [&](uint64_t x, int cnt) {
    if (o) put_digits(o + len, x, cnt);
    len += cnt;
  };
  if (v == 0.0) {
    if (signbit(v)) put('-');
    put('0');
    return len;
  }
  if (v < 0) {
    put('-');
    v = -v;
  }
  int e = (int)floor(log10(v));
  int64_t n = 0;
  bool ok = false;
  for (int it = 0; it < 4; ++it) {
    if (!round6(p10, v, e, n)) return -1;
    if (n > 1000000) { ++e; continue; }
    if (n == 1000000) { n = 100000; ++e; ok = true; break; }
    if (n < 100000) { --e; continue; }
    ok = true;
    break;
  }
  if (!ok) return -1;
  // the 6 significant digits without their trailing zeros: m, nd digits
  uint64_t m = (uint64_t)n;
  int nd = 6;
  while (nd > 1 && m % 10 == 0) {
    m /= 10;
    --nd;
  }
  if (e < -4 || e >= 6) {
    const uint64_t rest = ipow10(nd - 1);
    digits(m / rest, 1);
    if (nd > 1) {
      put('.');
      digits(m % rest, nd - 1);
    }
    put('e');
    put(e < 0 ? '-' : '+');
    const int ae = e < 0 ? -e : e;
    digits((uint64_t)ae, ae < 100 ? 2 : 3);
  } else if (e >= 0) {
    if (nd <= e + 1) {
      digits(m * ipow10(e + 1 - nd), e + 1);
    } else {
      const uint64_t frac = ipow10(nd - e - 1);
      digits(m / frac, e + 1);
      put('.');
      digits(m % frac, nd - e - 1);
    }
  } else {
    put('0');
    put('.');
    for (int i = 0; i < -e - 1; ++i) put('0');
    digits(m, nd);
  }
  return len;
}

__device__ __forceinline__ bool label_eq(const char* c, const int64_t* off, int64_t a, int64_t b) {
  const int64_t la = off[a + 1] - off[a], lb = off[b + 1] - off[b];
  if (la != lb) return false;
  const char* pa = c + off[a];
  const char* pb = c + off[b];
  for (int64_t i = 0; i < la; ++i)
    if (pa[i] != pb[i]) return false;
  return true;
}

// Line of hit i: qLabel qIdx qHitLen strand tLabel tIdx tHitLen match(pct%)
// score E.  Writes it at o when o is not null; returns its length, or -1 when
// a number needs the host.
__device__ int tsv_line(const TsvArgs& a, int64_t i, int64_t trec, char* o) {
  const int64_t r = a.read[i];
  const int64_t ql = a.q_off[r + 1] - a.q_off[r], tl = a.t_off[trec + 1] - a.t_off[trec];
  const int tidx = a.t_idx[i] + (a.t_start ? a.t_start[trec] : 0);
  const double pct = (double)(a.match[i] * 100) / (double)a.q_len[i];
  const int lp = fmt_g6(g_pow10, pct, nullptr);
  const int le = fmt_g6(g_pow10, a.evalue[i], nullptr);
  if (lp < 0 || le < 0) return -1;
  if (!o) {
    return (int)ql + (int)tl + 9 + len_i(a.q_idx[i]) + len_i(a.q_len[i]) + 1 + len_i(tidx) + len_i(a.t_len[i]) +
           len_i(a.match[i]) + 1 + lp + 2 + len_i(a.score[i]) + le + 1;
  }
  int k = 0;
  for (int64_t j = 0; j < ql; ++j) o[k++] = a.q_chars[a.q_off[r] + j];
  o[k++] = '\t';
  k += put_i(o + k, a.q_idx[i]);
  o[k++] = '\t';
  k += put_i(o + k, a.q_len[i]);
  o[k++] = '\t';
  o[k++] = a.strand[i] ? '-' : '+';
  o[k++] = '\t';
  for (int64_t j = 0; j < tl; ++j) o[k++] = a.t_chars[a.t_off[trec] + j];
  o[k++] = '\t';
  k += put_i(o + k, tidx);
  o[k++] = '\t';
  k += put_i(o + k, a.t_len[i]);
  o[k++] = '\t';
  k += put_i(o + k, a.match[i]);
  o[k++] = '(';
  k += fmt_g6(g_pow10, pct, o + k);
  o[k++] = '%';
  o[k++] = ')';
  o[k++] = '\t';
  k += put_i(o + k, a.score[i]);
  o[k++] = '\t';
  k += fmt_g6(g_pow10, a.evalue[i], o + k);
  o[k++] = '\n';
  return k;
}

// head[i] = 1 where a run starts: the first hit of a query load, or a hit
// whose query label differs from the previous hit's.  Also checks that every
// label the text needs exists (*bad).
__global__ void k_tsv_heads(TsvArgs a, const int64_t* __restrict__ load_off, int32_t n_loads,
                            uint8_t* __restrict__ head, int32_t* __restrict__ bad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int64_t r = a.read[i];
  const int tl = a.t_load[i];
  bool ok = r >= 0 && r < a.n_reads && tl >= 0 && tl < a.n_tloads;
  if (ok) {
    const int64_t trec = a.t_load_first[tl] + a.t_seq[i];
    ok = trec >= 0 && trec < a.n_trecs && a.t_seq[i] >= 0;
  }
  if (!ok) {
    atomicExch(bad, 1);
    head[i] = 1;
    return;
  }
  bool h = i == 0;
  if (!h) {
    const int64_t rp = a.read[i - 1];
    h = rp != r && (rp < 0 || rp >= a.n_reads || !label_eq(a.q_chars, a.q_off, rp, r));
  }
  if (!h) {  // a load's first hit
    int lo = 0, hi = n_loads;  // largest k with load_off[k] <= i
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (load_off[mid] <= i) lo = mid;
      else hi = mid;
    }
    h = load_off[lo] == i;
  }
  head[i] = h ? 1 : 0;
}

// One thread per run: printResult's selection over the run, and the length of
// every printed line (0 for skipped ones and for lines the host formats, whose
// indices go to `host`).
__global__ void k_tsv_select(TsvArgs a, const uint8_t* __restrict__ head, const int32_t* __restrict__ bad,
                             int32_t* __restrict__ len, int32_t* __restrict__ n_host, int64_t* __restrict__ host,
                             int32_t host_cap) {
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i0 >= a.n || !head[i0] || *bad) return;
  int count = 0;
  int pre_qidx = 0, pre_tidx = 0, pre_tlen = 0, pre_qlen = 0, pre_match = 0, pre_score = 0, pre_strand = 0;
  int64_t pre_trec = -1;
  double pre_e = 0;
  for (int64_t i = i0; i < a.n && (i == i0 || !head[i]); ++i) {
    const bool new_label = i == i0;
    if (new_label) count = 0;
    int L = 0;
    if (a.num_out == -1 || new_label || count < a.num_out) {
      const int64_t trec = a.t_load_first[a.t_load[i]] + a.t_seq[i];
      const int tidx = a.t_idx[i] + (a.t_start ? a.t_start[trec] : 0);
      const bool same_t = trec == pre_trec || (pre_trec >= 0 && label_eq(a.t_chars, a.t_off, trec, pre_trec));
      if (new_label || pre_qidx != a.q_idx[i] || pre_strand != a.strand[i] || !same_t || pre_tidx != tidx ||
          pre_tlen != a.t_len[i] || pre_qlen != a.q_len[i] || pre_match != a.match[i] ||
          pre_score != a.score[i] || pre_e != a.evalue[i]) {
        ++count;
        pre_qidx = a.q_idx[i];
        pre_strand = a.strand[i];
        pre_trec = trec;
        pre_tidx = tidx;
        pre_tlen = a.t_len[i];
        pre_qlen = a.q_len[i];
        pre_match = a.match[i];
        pre_score = a.score[i];
        pre_e = a.evalue[i];
        L = tsv_line(a, i, trec, nullptr);
        if (L < 0) {
          L = 0;
          const int k = atomicAdd(n_host, 1);
          if (k < host_cap) host[k] = i;
        }
      }
    }
    len[i] = L;
  }
}

__global__ void k_tsv_write(TsvArgs a, const int32_t* __restrict__ len, const int64_t* __restrict__ off,
                            char* __restrict__ text) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n || len[i] == 0) return;
  const int64_t trec = a.t_load_first[a.t_load[i]] + a.t_seq[i];
  tsv_line(a, i, trec, text + off[i]);
}

__global__ void k_tsv_gather(const int64_t* __restrict__ off, const int64_t* __restrict__ idx, int n,
                             int64_t* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = off[idx[k]];
}

struct TsvOwner {
  clast::PinnedArena* arena = nullptr;  // the device text, downloaded
  std::string spliced;                  // used instead when lines came from the host
  std::vector<int64_t> load_offsets;
};

void check_labels(const clast_labels* L, const char* what) {
  if (!L || L->n < 0 || (L->n > 0 && (!L->chars || !L->offsets)))
    throw std::invalid_argument(std::string("bad ") + what + " labels");
}

// printResult's line for hit i, on the host (snprintf).
std::string host_line(const clast_map_result& r, int64_t i, const clast_labels& reads, const clast_labels& targets,
                      const int32_t* t_start_idx, const int64_t* t_load_first) {
  const int64_t trec = t_load_first[r.t_load[i]] + r.t_seq[i];
  const int tidx = r.t_idx[i] + (t_start_idx ? t_start_idx[trec] : 0);
  std::string o(reads.chars + reads.offsets[r.read[i]], (size_t)(reads.offsets[r.read[i] + 1] - reads.offsets[r.read[i]]));
  char line[512];
  int k = std::snprintf(line, sizeof(line), "\t%d\t%d\t%c\t", r.q_idx[i], r.q_len[i], r.strand[i] ? '-' : '+');
  o.append(line, (size_t)k);
  o.append(targets.chars + targets.offsets[trec], (size_t)(targets.offsets[trec + 1] - targets.offsets[trec]));
  // std::ostream's default double format is %g with precision 6
  k = std::snprintf(line, sizeof(line), "\t%d\t%d\t%d(%g%%)\t%d\t%g\n", tidx, r.t_len[i], r.match[i],
                    (double)(r.match[i] * 100) / r.q_len[i], r.score[i], r.evalue[i]);
  o.append(line, (size_t)k);
  return o;
}

template <class T>
T* upload(Workspace& ws, const char* name, const T* host, size_t n, cudaStream_t st) {
  T* d = ws.get<T>(name, n ? n : 1);
  if (n) CLAST_CK(cudaMemcpyAsync(d, host, n * sizeof(T), cudaMemcpyHostToDevice, st));
  return d;
}

}  // namespace

extern "C" int clast_format_tsv(clast_ctx* ctx, const clast_targets* T, const clast_map_result* r, int32_t n_loads,
                                const clast_labels* reads, const clast_labels* targets, const int32_t* t_start_idx,
                                int32_t num_out, clast_tsv* out) {
  if (!ctx || !out) return CLAST_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  return guarded(ctx, [&]() -> int {
    if (!T) throw std::invalid_argument("targets are null");
    if (!r || n_loads < 0 || !r->load_offsets || !r->owner) throw std::invalid_argument("bad map result");
    check_labels(reads, "read");
    check_labels(targets, "target");
    if (targets->n != T->load_first.back()) throw std::invalid_argument("one target label per target record is needed");
    PinnedArena* ra = static_cast<PinnedArena*>(r->owner);
    if (!ra->in_use || ra->dev.n != r->n || ra->dev.n_loads != n_loads || r->load_offsets[n_loads] != r->n)
      throw std::invalid_argument("the map result was released, or n_loads does not match it");
    CLAST_CK(cudaSetDevice(ctx->device));
    g_alloc_stream = ctx->st;
    ensure_pow10(ctx->device);
    cudaStream_t st = ctx->st;
    Workspace& ws = ctx->ws;
    const int64_t F = r->n;
    TsvArgs a{};
    a.n = F;
    a.read = ra->dev.f[0].p;
    a.strand = ra->dev.f[1].p;
    a.t_load = ra->dev.f[2].p;
    a.t_seq = ra->dev.f[3].p;
    a.t_idx = ra->dev.f[4].p;
    a.q_idx = ra->dev.f[5].p;
    a.t_len = ra->dev.f[6].p;
    a.q_len = ra->dev.f[7].p;
    a.match = ra->dev.f[8].p;
    a.score = ra->dev.f[9].p;
    a.evalue = ra->dev.evalue.p;
    const int64_t qc = reads->n ? reads->offsets[reads->n] : 0, tc = targets->n ? targets->offsets[targets->n] : 0;
    a.q_chars = upload(ws, "tsv_qchars", reads->chars, (size_t)qc, st);
    a.q_off = upload(ws, "tsv_qoff", reads->offsets, (size_t)reads->n + 1, st);
    a.n_reads = reads->n;
    a.t_chars = upload(ws, "tsv_tchars", targets->chars, (size_t)tc, st);
    a.t_off = upload(ws, "tsv_toff", targets->offsets, (size_t)targets->n + 1, st);
    a.n_trecs = targets->n;
    a.t_start = t_start_idx ? upload(ws, "tsv_tstart", t_start_idx, (size_t)targets->n, st) : nullptr;
    a.t_load_first = upload(ws, "tsv_tlf", T->load_first.data(), T->load_first.size(), st);
    a.n_tloads = T->n_loads;
    a.num_out = num_out;
    std::unique_ptr<TsvOwner> own(new TsvOwner());
    own->load_offsets.assign((size_t)n_loads + 1, 0);
    // counters: [0] bad label index, [1] lines for the host
    int32_t* cnt = ws.get<int32_t>("tsv_cnt", 2);
    CLAST_CK(cudaMemsetAsync(cnt, 0, 2 * sizeof(int32_t), st));
    constexpr int32_t kHostCap = 1 << 16;
    int64_t* host_idx = ws.get<int64_t>("tsv_host", kHostCap);
    uint8_t* head = ws.get<uint8_t>("tsv_head", (size_t)F);
    int32_t* len = ws.get<int32_t>("tsv_len", (size_t)F);
    int64_t* off = ws.get<int64_t>("tsv_off", (size_t)F + 1);
    const unsigned blocks = (unsigned)((F + 255) / 256);
    if (F > 0) {
      k_tsv_heads<<<blocks, 256, 0, st>>>(a, ra->dev.load_offsets.p, n_loads, head, cnt);
      CLAST_LAUNCHED();
      k_tsv_select<<<blocks, 256, 0, st>>>(a, head, cnt, len, cnt + 1, host_idx, kHostCap);
      CLAST_LAUNCHED();
    }
    scan_i32(ws, len, F, off, st);
    struct { int32_t c[2]; int64_t total; } h{};
    CLAST_CK(cudaMemcpyAsync(h.c, cnt, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    CLAST_CK(cudaMemcpyAsync(&h.total, off + F, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CLAST_CK(cudaStreamSynchronize(st));
    if (h.c[0]) throw std::invalid_argument("a hit's read or target record has no label");
    if (h.c[1] > kHostCap) throw std::runtime_error("too many result lines need host formatting");
    const int64_t total = h.total;
    // the device text, downloaded into a reusable pinned arena
    char* text = ws.get<char>("tsv_text", (size_t)total + 1);
    if (F > 0) {
      k_tsv_write<<<blocks, 256, 0, st>>>(a, len, off, text);
      CLAST_LAUNCHED();
    }
    int64_t* lo_dev = ws.get<int64_t>("tsv_loadoff", (size_t)n_loads + 1);
    int64_t* pos_dev = ws.get<int64_t>("tsv_hostpos", (size_t)std::max(1, h.c[1]));
    gather_i64(off, ra->dev.load_offsets.p, n_loads + 1, lo_dev, st);
    if (h.c[1] > 0) {
      k_tsv_gather<<<(unsigned)((h.c[1] + 255) / 256), 256, 0, st>>>(off, host_idx, h.c[1], pos_dev);
      CLAST_LAUNCHED();
    }
    PinnedArena* ta = nullptr;
    for (auto& x : ctx->tsv_arenas)
      if (!x->in_use && (ta == nullptr || x->bytes > ta->bytes)) ta = x.get();
    if (!ta) {
      ctx->tsv_arenas.emplace_back(new PinnedArena());
      ta = ctx->tsv_arenas.back().get();
    }
    if (ta->bytes < (size_t)total + 1) {
      if (ta->p) CLAST_CK(cudaFreeHost(ta->p));
      ta->p = nullptr;
      ta->bytes = 0;
      const size_t nb = (size_t)total + (size_t)total / 4 + (1 << 20);
      if (cudaMallocHost(&ta->p, nb) != cudaSuccess) {
        (void)cudaGetLastError();
        throw std::bad_alloc();
      }
      ta->bytes = nb;
    }
    if (total) CLAST_CK(cudaMemcpyAsync(ta->p, text, (size_t)total, cudaMemcpyDeviceToHost, st));
    CLAST_CK(cudaMemcpyAsync(own->load_offsets.data(), lo_dev, ((size_t)n_loads + 1) * sizeof(int64_t),
                             cudaMemcpyDeviceToHost, st));
    std::vector<int64_t> hidx((size_t)h.c[1]), hpos((size_t)h.c[1]);
    if (h.c[1] > 0) {
      CLAST_CK(cudaMemcpyAsync(hidx.data(), host_idx, hidx.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
      CLAST_CK(cudaMemcpyAsync(hpos.data(), pos_dev, hpos.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    }
    CLAST_CK(cudaStreamSynchronize(st));
    ta->in_use = true;
    own->arena = ta;
    const char* base = static_cast<const char*>(ta->p);
    if (h.c[1] == 0) {
      out->text = base;
      out->n_bytes = total;
    } else {  // splice the host-formatted lines in at their positions, in hit order
      std::vector<size_t> ord(hidx.size());
      for (size_t k = 0; k < ord.size(); ++k) ord[k] = k;
      std::sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return hidx[x] < hidx[y]; });
      std::vector<std::string> lines(hidx.size());
      for (size_t k = 0; k < hidx.size(); ++k)
        lines[k] = host_line(*r, hidx[k], *reads, *targets, t_start_idx, T->load_first.data());
      std::string& s = own->spliced;
      int64_t at = 0;
      for (size_t k : ord) {  // a host line has length 0 in the device text: it goes at its scan offset
        s.append(base + at, (size_t)(hpos[k] - at));
        s += lines[k];
        at = hpos[k];
      }
      s.append(base + at, (size_t)(total - at));
      // a load's text starts later by the host lines of the hits before it
      size_t j = 0;
      int64_t added = 0;
      for (int32_t li = 0; li <= n_loads; ++li) {
        while (j < ord.size() && hidx[ord[j]] < r->load_offsets[li]) added += (int64_t)lines[ord[j++]].size();
        own->load_offsets[li] += added;
      }
      ta->in_use = false;  // the text now lives in the spliced copy
      own->arena = nullptr;
      out->text = s.data();
      out->n_bytes = (int64_t)s.size();
    }
    out->load_offsets = own->load_offsets.data();
    out->owner = own.release();
    return CLAST_OK;
  });
}

// The %g formatter of the device path run on the host, for checking its
// digits against the C library's printf without a GPU: out receives the n
// strings back to back (32 bytes each, NUL-terminated); lens[i] = length or
// -1 where the device would leave the value to the host.  Not part of the
// public interface.
extern "C" int clast_format_g6_host(const double* v, int64_t n, char* out, int32_t* lens) {
  if (!v || !out || !lens || n < 0) return CLAST_ERR_ARG;
  const double2* p10 = pow10_table().data();
  for (int64_t i = 0; i < n; ++i) {
    char* o = out + 32 * i;
    const int L = fmt_g6(p10, v[i], o);
    lens[i] = L;
    o[L < 0 ? 0 : L] = '\0';
  }
  return CLAST_OK;
}

namespace {
__global__ void k_fmt_g6(const double* __restrict__ v, int64_t n, char* __restrict__ out, int32_t* __restrict__ lens) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  char* o = out + 32 * i;
  const int L = fmt_g6(g_pow10, v[i], o);
  lens[i] = L;
  o[L < 0 ? 0 : L] = '\0';
}
}  // namespace

// The same formatter run as a kernel on the context's GPU (the path
// clast_format_tsv takes), for checking the device's digits against the C
// library's printf: host arrays in and out, as clast_format_g6_host.  Not
// part of the public interface.
extern "C" int clast_format_g6_device(clast_ctx* ctx, const double* v, int64_t n, char* out, int32_t* lens) {
  if (!ctx || !v || !out || !lens || n < 0) return CLAST_ERR_ARG;
  return guarded(ctx, [&]() -> int {
    CLAST_CK(cudaSetDevice(ctx->device));
    ensure_pow10(ctx->device);
    cudaStream_t st = ctx->st;
    double* dv = ctx->ws.get<double>("fmt_v", (size_t)n);
    char* dout = ctx->ws.get<char>("fmt_out", (size_t)n * 32);
    int32_t* dl = ctx->ws.get<int32_t>("fmt_len", (size_t)n);
    if (n) {
      CLAST_CK(cudaMemcpyAsync(dv, v, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
      k_fmt_g6<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dv, n, dout, dl);
      CLAST_LAUNCHED();
      CLAST_CK(cudaMemcpyAsync(out, dout, (size_t)n * 32, cudaMemcpyDeviceToHost, st));
      CLAST_CK(cudaMemcpyAsync(lens, dl, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    }
    CLAST_CK(cudaStreamSynchronize(st));
    return CLAST_OK;
  });
}

extern "C" void clast_tsv_free(clast_tsv* t) {
  if (!t) return;
  TsvOwner* o = static_cast<TsvOwner*>(t->owner);
  if (o && o->arena) o->arena->in_use = false;
  delete o;
  std::memset(t, 0, sizeof(*t));
}
