/*
 * clast_oracle.cpp -- CPU restatement of CLAST's seed-and-extend path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * in clast_b200/: it is loaded by tests/, by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline leg, and never by the product itself.
 *
 * It restates, in plain scalar C++, the algorithm of the reference
 * (masayano/CLAST, a flat directory of sources; citations are file:line
 * there).  Every step keeps the reference's order of operations, including
 * its stable sorts, its remove_if passes with original-predecessor stencils
 * and its chunking into RAM loads and VRAM windows, because the result order
 * and the duplicate filters depend on them.  Parity of this restatement is
 * pinned against the reference itself compiled for the CPU
 * (oracle/build_ref.py, tests/test_oracle_pin.py).
 *
 * Defined behaviour where the reference reads outside its buffers (its
 * results there depend on neighbouring memory): any base outside a window's
 * base array, and any joint base past the end of a sequence shorter than
 * l-1, is 'N'.  Letters outside 'A'..'Z' score as 'N' as well.
 */
#include "clast_oracle.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

std::string g_last_error;

struct OracleError {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const std::string& msg) { throw OracleError{code, msg}; }

/* ------------------------------------------------------------------ */
/* Constants: common.hpp:12-43                                         */
/* ------------------------------------------------------------------ */
constexpr int kMaxLmer = 31;           // common.hpp:28
constexpr int kMaxGap = 16;            // common.hpp:29
constexpr int kBadAreaPoint = -1000;   // common.hpp:37
constexpr int kMatch = 1;              // common.hpp:38
constexpr int kMismatch = -3;          // common.hpp:39
constexpr int kGapOpen = -5;           // common.hpp:40
constexpr int kGapExtend = -2;         // common.hpp:41
constexpr int kMarginScore = -30000;   // krnlAlignment.cu:20-23

/* ------------------------------------------------------------------ */
/* Settings: CHostSetting.cu:62-142, listenCommandLine.cpp:281-325     */
/* ------------------------------------------------------------------ */
struct Settings {
  double tRAM = 64, qRAM = 64, tVRAM = 64, qVRAM = 2;  // common.hpp:12-15
  int lmer = 15, stride = 5, cutRepeat = 20, width = 100, gap = 8;
  int numOut = -1, local = 0, device = 0, sleep = 0;
  double cutOff = 10;
  std::vector<std::string> tfiles, qfiles;
  std::string out;
  double totalDB = 0, K = 0.71, lambda = 1.37;
};

/* boost::lexical_cast semantics: the whole string is one number. */
int parse_int(const std::string& s, const char* flag) {
  errno = 0;
  char* end = nullptr;
  if (s.empty() || s[0] == ' ' || s[0] == '\t') fail(-2, std::string("bad value after ") + flag);
  long v = std::strtol(s.c_str(), &end, 10);
  if (end != s.c_str() + s.size() || errno == ERANGE || v < INT_MIN || v > INT_MAX)
    fail(-2, std::string("bad value after ") + flag);
  return (int)v;
}
double parse_double(const std::string& s, const char* flag) {
  char* end = nullptr;
  if (s.empty() || s[0] == ' ' || s[0] == '\t') fail(-2, std::string("bad value after ") + flag);
  double v = std::strtod(s.c_str(), &end);
  if (end != s.c_str() + s.size()) fail(-2, std::string("bad value after ") + flag);
  return v;
}

/* The reference turns MBase sizes into int budgets by truncation
 * (main.cu:42,63-65; CHostSchedular.cu:127-128,157-161). */
int budget_to_int(double v) {
  if (!(v < 2147483648.0) || v < -2147483648.0) fail(-2, "RAM/VRAM budget does not fit a 32-bit int");
  return (int)v;
}

/* totalDatabaseSize: characters of every target line without '>'
 * (CHostSetting.cu:46-58). */
long total_db_size(const std::vector<std::string>& files) {
  long total = 0;
  for (const auto& f : files) {
    std::ifstream ifs(f.c_str(), std::ios::binary);
    std::string buf;
    while (ifs && std::getline(ifs, buf))
      if (buf.find('>') == std::string::npos) total += (long)buf.size();
  }
  return total;
}

Settings parse_settings(int argc, const char** argv) {
  Settings s;
  enum St { START, T_RAM, Q_RAM, T_VRAM, Q_VRAM, L_MER, STRIDE, REPEAT, WIDTH, GAP, NUM_OUT,
            CUT_OFF, LOCAL, DEVICE, SLEEP, T_FILE, Q_FILE, O_FILE };
  auto flag_state = [](const std::string& a, St& st) -> bool {
    static const struct { const char* f; St s; } tab[] = {
        {"-tRAM", T_RAM}, {"-qRAM", Q_RAM}, {"-tVRAM", T_VRAM}, {"-qVRAM", Q_VRAM},
        {"-lMer", L_MER}, {"-stride", STRIDE}, {"-repeat", REPEAT}, {"-width", WIDTH},
        {"-gap", GAP}, {"-numOut", NUM_OUT}, {"-cutOff", CUT_OFF}, {"-local", LOCAL},
        {"-device", DEVICE}, {"-sleep", SLEEP}};
    for (const auto& e : tab)
      if (a == e.f) { st = e.s; return true; }
    return false;
  };
  St st = START;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    switch (st) {
      case START:  // listenCommandLine.cpp:13-37
        if (flag_state(a, st)) break;
        if (a == "-t") st = T_FILE;
        else if (a == "-q") st = Q_FILE;
        else if (a == "-o") st = O_FILE;
        else fail(-2, "Odd parameter was inputted. Check the command line parameter.");
        break;
      case T_RAM: s.tRAM = parse_double(a, "-tRAM"); st = START; break;
      case Q_RAM: s.qRAM = parse_double(a, "-qRAM"); st = START; break;
      case T_VRAM: s.tVRAM = parse_double(a, "-tVRAM"); st = START; break;
      case Q_VRAM: s.qVRAM = parse_double(a, "-qVRAM"); st = START; break;
      case L_MER: s.lmer = parse_int(a, "-lMer"); st = START; break;
      case STRIDE: s.stride = parse_int(a, "-stride"); st = START; break;
      case REPEAT: s.cutRepeat = parse_int(a, "-repeat"); st = START; break;
      case WIDTH: s.width = parse_int(a, "-width"); st = START; break;
      case GAP: s.gap = parse_int(a, "-gap"); st = START; break;
      case NUM_OUT: s.numOut = parse_int(a, "-numOut"); st = START; break;
      case CUT_OFF: s.cutOff = parse_double(a, "-cutOff"); st = START; break;
      case LOCAL: s.local = parse_int(a, "-local"); st = START; break;
      case DEVICE: s.device = parse_int(a, "-device"); st = START; break;
      case SLEEP: s.sleep = parse_int(a, "-sleep"); st = START; break;
      case T_FILE:  // listenCommandLine.cpp:221-245
        if (flag_state(a, st)) break;
        if (a == "-t") fail(-2, "Odd parameter was inputted. Check the after of \"-t\".");
        else if (a == "-q") st = Q_FILE;
        else if (a == "-o") st = O_FILE;
        else s.tfiles.push_back(a);
        break;
      case Q_FILE:  // listenCommandLine.cpp:247-271
        if (flag_state(a, st)) break;
        if (a == "-t") st = T_FILE;
        else if (a == "-q") fail(-2, "Odd parameter was inputted. Check the after of \"-q\".");
        else if (a == "-o") st = O_FILE;
        else s.qfiles.push_back(a);
        break;
      case O_FILE: s.out = a; st = START; break;
    }
  }
  // validator, CHostSetting.cu:14-44
  if (s.lmer > kMaxLmer) fail(-2, "too large lMerLength was inputted.");
  if (s.gap > kMaxGap) fail(-2, "too large allowableGap was inputted.");
  if (s.gap < 2) fail(-2, "allowableGap must be larger than 1.");
  if (s.tfiles.empty()) fail(-2, "no target file was inputted.");
  if (s.qfiles.empty()) fail(-2, "no query file was inputted.");
  if (s.out.empty()) fail(-2, "no output file was inputted.");
  // The reference divides by stride and sizes arrays by lMer-1 without checks.
  if (s.lmer < 1) fail(-2, "lMerLength must be at least 1.");
  if (s.stride < 1) fail(-2, "strideLength must be at least 1.");
  for (const auto& f : s.tfiles)
    if (!std::ifstream(f.c_str())) fail(-3, "file \"" + f + "\" open failed.");
  for (const auto& f : s.qfiles)
    if (!std::ifstream(f.c_str())) fail(-3, "file \"" + f + "\" open failed.");
  // CHostSetting.cu:133-141
  s.tRAM *= 1000 * 1000;
  s.qRAM *= 1000 * 1000;
  s.tVRAM *= 1000 * 1000;
  s.qVRAM *= 1000 * 1000;
  s.totalDB = (double)total_db_size(s.tfiles);
  return s;
}

/* ------------------------------------------------------------------ */
/* FASTA loading: CFASTALoader.cpp:11-170                              */
/* ------------------------------------------------------------------ */
struct Fasta {
  std::string label, seq;
  int startIdx;
};

/* CFASTALoader.cpp:89-106 */
void normalise_line(std::string& s) {
  std::string o;
  o.reserve(s.size());
  for (char c : s) {
    if (c == ' ') continue;
    if (c > 'Z') c -= 32;
    if (c < 'A' || c > 'Z') c = 'N';
    o.push_back(c);
  }
  s.swap(o);
}

class FileReader {  // CFASTALoader::CFASTAFileLoader
 public:
  /* CFASTALoader.cpp:43-87 */
  bool judge(long pos, int budget, std::string& label, std::string& seq, int& startIdx,
             std::vector<Fasta>& out) {
    if (!label.empty()) {
      const int len = (int)seq.size();
      if (len > budget) {  // record longer than the budget: skipped with a warning
        label.clear();
        seq.clear();
        startIdx = 0;
        readPos_ = pos;
      } else if (sum_ + len < budget) {
        out.push_back(Fasta{label, seq, startIdx});
        sum_ += len;
        label.clear();
        seq.clear();
        startIdx = 0;
        readPos_ = pos;
      } else {
        sum_ = 0;
        return false;
      }
    }
    return true;
  }
  /* CFASTALoader.cpp:112-170 */
  bool read(int budget, const std::string& path, std::vector<Fasta>& out) {
    std::ifstream ifs(path.c_str(), std::ios::binary);
    if (!ifs) fail(-3, "file \"" + path + "\" open failed.");
    std::string buf, label, seq;
    int startIdx = 0;
    ifs.seekg(readPos_);
    long tempPos = readPos_;
    while (ifs && std::getline(ifs, buf)) {
      if (buf.find('>') != std::string::npos) {
        if (!judge(tempPos, budget, label, seq, startIdx, out)) return false;
        label = buf.substr(1);
      } else if (buf.find('@') != std::string::npos) {
        try {
          startIdx = parse_int(buf.substr(1), "@");
        } catch (const OracleError&) {
          fail(-4, "bad file type: something was strange at the line which contains '@'.");
        }
      } else if (buf.empty()) {
        if (!judge(tempPos, budget, label, seq, startIdx, out)) return false;
      } else if (!label.empty()) {
        normalise_line(buf);
        seq += buf;
      }
      tempPos = (long)ifs.tellg();
    }
    if (ifs.eof()) {
      if (!judge(tempPos, budget, label, seq, startIdx, out)) return false;
    }
    readPos_ = 0;
    return true;
  }

 private:
  long readPos_ = 0;
  long sum_ = 0;
};

class Loader {  // CFASTALoader
 public:
  Loader(const std::vector<std::string>& files, int budget) : files_(files), budget_(budget) {}
  void load(std::vector<Fasta>& out) {  // CFASTALoader.cpp:27-36
    const int before = fileIndex_;
    for (; fileIndex_ < (int)files_.size(); ++fileIndex_)
      if (!reader_.read(budget_, files_[fileIndex_], out)) break;
    if (fileIndex_ == (int)files_.size()) fileIndex_ = -1;
    // A record exactly as long as the budget neither fits nor is skipped, so
    // the reference returns the same empty load forever.
    if (out.empty() && fileIndex_ == before && fileIndex_ != -1)
      fail(-5, "a FASTA record is exactly as long as the RAM budget; the reference never terminates");
  }
  int fileIndex() const { return fileIndex_; }

 private:
  std::vector<std::string> files_;
  int budget_;
  FileReader reader_;
  int fileIndex_ = 0;
};

/* ------------------------------------------------------------------ */
/* Host sequence lists: utilAddSequence.cu:6-47, CHostSeqList_*.cu     */
/* ------------------------------------------------------------------ */
struct SeqList {
  std::vector<std::string> labels;
  std::vector<int> startIdx;
  std::vector<char> bases;     // sequence followed by its first l-1 bases
  std::vector<int> lengths;
  std::vector<int> gateway;    // prefix sums of len+l-1, starting at 0
  void add(const std::string& seq, int l) {
    const int len = (int)seq.size();
    bases.insert(bases.end(), seq.begin(), seq.end());
    for (int i = 0; i < l - 1; ++i) bases.push_back(i < len ? seq[i] : 'N');
    lengths.push_back(len);
    if (gateway.empty()) gateway.push_back(0);
    gateway.push_back(gateway.back() + len + l - 1);
  }
};

/* utilReverseSeq.cpp:3-19 */
std::string reverse_complement(const std::string& s) {
  std::string r;
  r.reserve(s.size());
  for (auto it = s.rbegin(); it != s.rend(); ++it) {
    switch (*it) {
      case 'A': r.push_back('T'); break;
      case 'T': r.push_back('A'); break;
      case 'G': r.push_back('C'); break;
      case 'C': r.push_back('G'); break;
      default: r.push_back('N');
    }
  }
  return r;
}

/* ------------------------------------------------------------------ */
/* A window: a contiguous run of sequences of a SeqList               */
/* ------------------------------------------------------------------ */
struct Window {
  const char* bases;
  int64_t n;               // bases in the window (joints included)
  const int32_t* gateway;  // window-relative starts, nseqs entries
  const int32_t* lengths;
  int32_t nseqs;
  int32_t first_id;
  char base(int64_t i) const { return (i < 0 || i >= n) ? 'N' : bases[i]; }
  /* window position -> sequence (CDeviceSeqList IDArray / indexArray) */
  int seq_of(int64_t pos) const {
    return (int)(std::upper_bound(gateway, gateway + nseqs, (int32_t)pos) - gateway) - 1;
  }
};

/* k-mer key: SRead2bit.cuh:6-21 + SRepelHasOddBase.cuh:6-14 */
int64_t kmer_key(const Window& w, int64_t pos, int l) {
  int64_t key = 0;
  for (int i = 0; i < l; ++i) {
    key <<= 2;
    switch (w.base(pos + i)) {
      case 'A': break;
      case 'C': key += 1; break;
      case 'G': key += 2; break;
      case 'T': key += 3; break;
      default: return -1;
    }
  }
  return key;
}

/* ------------------------------------------------------------------ */
/* Index: CDeviceHashTable.cu:20-174                                   */
/* ------------------------------------------------------------------ */
struct Index {
  std::vector<int64_t> ukeys;  // gatewayKey
  std::vector<int> count;      // cellSizeArray (after the repeat cut)
  std::vector<int> offset;     // gatewayIndex
  std::vector<int> pos;        // indexArray: window positions sorted by key
};

Index build_index(const Window& t, int l, int stride, int cutRepeat) {
  Index ix;
  const int64_t ns = t.n / stride;  // CDeviceHashTable.cu:34
  std::vector<int64_t> keys(ns);
  std::vector<int> order(ns);
  for (int64_t j = 0; j < ns; ++j) {
    keys[j] = kmer_key(t, j * stride, l);  // strided k-mers, CDeviceHashTable.cu:37-64
    order[j] = (int)j;
  }
  // sort_by_key (stable), CDeviceHashTable.cu:159
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return keys[a] < keys[b]; });
  ix.pos.resize(ns);
  for (int64_t j = 0; j < ns; ++j) ix.pos[j] = order[j] * stride;  // makeIndexArray :72-84
  // unique + reduce_by_key + exclusive_scan, :87-120
  for (int64_t j = 0; j < ns; ++j) {
    const int64_t k = keys[order[j]];
    if (j == 0 || k != ix.ukeys.back()) {
      ix.ukeys.push_back(k);
      ix.count.push_back(0);
      ix.offset.push_back((int)j);
    }
    ix.count.back()++;
  }
  if (cutRepeat != -1)  // removeRepeatedSequence, :122-137,165-168
    for (auto& c : ix.count) c = (c < cutRepeat) ? c : 0;
  if (!ix.ukeys.empty() && ix.ukeys[0] == -1) ix.count[0] = 0;  // :171-173
  return ix;
}

/* ------------------------------------------------------------------ */
/* Seeds and hits                                                      */
/* ------------------------------------------------------------------ */
struct Hit {
  int tID, tIdx, qID, qIdx, tLen, qLen, match, score;
  double evalue;
};

/* remove_if with a stencil reading element i and the ORIGINAL element i-1;
 * element 0 is never removed (CDeviceHitList_deleteIsolateSeeds.cu:19-77,
 * _deleteDuplicateSeeds.cu:15-71, CDeviceHitList.cu:32-128). */
template <class Pred>
void remove_with_predecessor(std::vector<Hit>& v, Pred remove) {
  if (v.size() <= 1) return;
  std::vector<char> drop(v.size(), 0);
  for (size_t i = 1; i < v.size(); ++i) drop[i] = remove(v[i], v[i - 1]) ? 1 : 0;
  size_t o = 0;
  for (size_t i = 0; i < v.size(); ++i)
    if (!drop[i]) v[o++] = v[i];
  v.resize(o);
}

/* hasNotNearPair / hasNearPair, _deleteIsolateSeeds.cuh:14-39 */
bool near_pair(const Hit& s, const Hit& prev, int width, int gap) {
  if (s.qID == prev.qID && s.tID == prev.tID) {
    if (width >= s.tIdx - prev.tIdx && width >= prev.tIdx - s.tIdx) {
      const int prevDiag = prev.tIdx - prev.qIdx;
      const int diag = s.tIdx - s.qIdx;
      if (gap >= prevDiag - diag) return true;
    }
  }
  return false;
}

/* POINT_MATRIX / MATCH_COUNTER, krnlMatrix.cuh:11-67, as a rule over
 * letter classes: 'X' (bad area) -1000; E F I J L O P Q Z -1; equal
 * A/C/G/T +1 (1 match); any other letter pair -3 (0 matches). */
int letter_class(char c) {  // 0..3 ACGT, 4 other scored letter, 5 "-1" letter, 6 X
  switch (c) {
    case 'A': return 0;
    case 'C': return 1;
    case 'G': return 2;
    case 'T': return 3;
    case 'X': return 6;
    case 'E': case 'F': case 'I': case 'J': case 'L': case 'O': case 'P': case 'Q': case 'Z':
      return 5;
    default: return 4;  // other letters; bytes outside A..Z are treated as 'N'
  }
}
int point_of(char t, char q) {
  const int a = letter_class(t), b = letter_class(q);
  if (a == 6 || b == 6) return kBadAreaPoint;
  if (a == 5 || b == 5) return -1;
  if (a == b && a < 4) return kMatch;
  return kMismatch;
}
int match_of(char t, char q) {
  const int a = letter_class(t), b = letter_class(q);
  if (a == 6 || b == 6) return kBadAreaPoint;
  if (a == 5 || b == 5) return -1;
  return (a == b && a < 4) ? 1 : 0;
}

/* The temporary band of krnlAlignment.cu: rows 0..2gap+2, four values each. */
struct Band {
  std::vector<int> S, V, H, M;
  explicit Band(int gap) {
    const int half = gap + 1, rows = 1 + 2 * half;  // MARGIN = 1
    S.assign(rows, 0); V.assign(rows, 0); H.assign(rows, 0); M.assign(rows, 0);
    for (int r = 0; r < rows; ++r) {  // initTempNodeArray, krnlAlignment.cu:6-38
      if (r < half) {
        S[r] = V[r] = H[r] = M[r] = kMarginScore;
      } else if (r == half) {
        S[r] = 0; V[r] = kGapOpen; H[r] = kGapOpen; M[r] = 0;
      } else {
        const int i = r - half, sc = i * kGapExtend + kGapOpen;
        S[r] = sc; V[r] = sc + kGapOpen; H[r] = sc; M[r] = 0;
      }
    }
  }
  /* calcutlateCell, krnlAlignment.cu:42-77, for slant row p */
  void cell(int p, char tb, char qb) {
    const int vs = S[p + 1], vv = V[p + 1], vm = M[p + 1];  // lower/upper row, old values
    const int hs = S[p - 1], hh = H[p - 1], hm = M[p - 1];  // left/right row, this query row
    V[p] = std::max(vs + kGapOpen + kGapExtend, vv + kGapExtend);
    H[p] = std::max(hs + kGapOpen + kGapExtend, hh + kGapExtend);
    const int pt = S[p] + point_of(tb, qb);
    if (pt > std::max(V[p], H[p])) {
      S[p] = pt;
      M[p] += match_of(tb, qb);
    } else if (V[p] > H[p]) {
      S[p] = V[p];
      M[p] = vm;
    } else {
      S[p] = H[p];
      M[p] = hm;
    }
  }
};

struct SeqInfo {
  int64_t start;
  int len;
};

/* global/localAlignBackward, krnlAlignment.cu:81-195 and :312-423 */
void align_backward(Hit& h, const Window& t, const Window& q, int gap, bool local) {
  const int ti = h.tID - t.first_id, qi = h.qID - q.first_id;
  const int64_t tStart = t.gateway[ti], qStart = q.gateway[qi];
  const int tLen = t.lengths[ti], qLen = q.lengths[qi];
  const int W = 1 + 2 * gap;
  std::vector<char> ring(W);
  for (int c = 0; c < W; ++c) {
    const int64_t ib = (int64_t)h.tIdx + h.qLen - gap + c;
    ring[c] = (ib >= tLen) ? 'X' : t.base(tStart + ib);
  }
  Band b(gap);
  int calcIdx = -1, endPoint = local ? gap : 0, bestS = 0, bestM = 0;
  int ring_at = 0;
  const int from = h.qIdx + h.qLen;
  const int rows = qLen - from;
  for (int qq = 0; qq < rows; ++qq) {
    const char qb = q.base(qStart + from + qq);
    for (int c = 0; c < W; ++c) {
      b.cell(c + 1, ring[ring_at++], qb);
      if (ring_at == W) ring_at = 0;
      if (local && bestS < b.S[c + 1]) {
        bestS = b.S[c + 1]; bestM = b.M[c + 1]; calcIdx = qq; endPoint = c;
      }
    }
    const int64_t ib = (int64_t)h.tIdx + h.qLen + gap + qq + 1;
    ring[ring_at] = (ib >= tLen) ? 'X' : t.base(tStart + ib);
    if (++ring_at == W) ring_at = 0;
  }
  int move = rows;
  if (local) {
    move = calcIdx + 1;
  } else {  // select end node, krnlAlignment.cu:170-185
    endPoint = -1; bestS = b.S[0]; bestM = b.M[0];
    for (int c = 0; c < W; ++c)
      if (bestS < b.S[c + 1]) { bestS = b.S[c + 1]; bestM = b.M[c + 1]; endPoint = c; }
  }
  endPoint -= gap;
  if (rows != 0) {
    h.tLen += move + endPoint;
    h.qLen += move;
    h.match += bestM;
    h.score += bestS;
  }
}

/* global/localAlignForward, krnlAlignment.cu:197-308 and :425-533 */
void align_forward(Hit& h, const Window& t, const Window& q, int gap, bool local) {
  const int ti = h.tID - t.first_id, qi = h.qID - q.first_id;
  const int64_t tStart = t.gateway[ti], qStart = q.gateway[qi];
  const int W = 1 + 2 * gap;
  std::vector<char> ring(W);
  for (int c = 0; c < W; ++c) {
    const int64_t ib = (int64_t)h.tIdx + gap - c - 1;
    ring[c] = (ib < 0) ? 'X' : t.base(tStart + ib);
  }
  Band b(gap);
  int calcIdx = -1, endPoint = local ? gap : 0, bestS = 0, bestM = 0;
  int ring_at = 0;
  const int rows = h.qIdx;
  for (int qq = 0; qq < rows; ++qq) {
    const char qb = q.base(qStart + h.qIdx - qq - 1);
    for (int c = 0; c < W; ++c) {
      b.cell(c + 1, ring[ring_at++], qb);
      if (ring_at == W) ring_at = 0;
      if (local && bestS < b.S[c + 1]) {
        bestS = b.S[c + 1]; bestM = b.M[c + 1]; calcIdx = qq; endPoint = c;
      }
    }
    const int64_t ib = (int64_t)h.tIdx - gap - qq - 2;
    ring[ring_at] = (ib < 0) ? 'X' : t.base(tStart + ib);
    if (++ring_at == W) ring_at = 0;
  }
  int move = rows;
  if (local) {
    move = calcIdx + 1;
  } else {
    endPoint = -1; bestS = b.S[0]; bestM = b.M[0];
    for (int c = 0; c < W; ++c)
      if (bestS < b.S[c + 1]) { bestS = b.S[c + 1]; bestM = b.M[c + 1]; endPoint = c; }
  }
  endPoint -= gap;
  if (rows != 0) {
    h.tIdx -= move + endPoint;
    h.qIdx -= move;
    h.tLen += move + endPoint;
    h.qLen += move;
    h.match += bestM;
    h.score += bestS;
  }
}

struct Params {
  int l, stride, cutRepeat, width, gap, local;
  double cutOff, totalDB, K, lambda;
};

/* CDeviceHitList::CDeviceHitList, CDeviceHitList.cu:228-423 */
std::vector<Hit> window_search(const Params& p, const Index& ix, const Window& t, const Window& q,
                               int stage) {
  std::vector<Hit> v;
  const int l = p.l;
  // createRawSeedList, CDeviceHitList_createRawSeedList.cu:139-232
  const int64_t nkeys = q.n - (l - 1);  // CDeviceSeqList_query.cu:17
  for (int64_t pq = 0; pq < nkeys; ++pq) {
    const int64_t key = kmer_key(q, pq, l);
    auto it = std::lower_bound(ix.ukeys.begin(), ix.ukeys.end(), key);  // binarySearch
    if (it == ix.ukeys.end() || *it != key) continue;
    const size_t u = it - ix.ukeys.begin();
    const int qs = q.seq_of(pq);
    const int qID = q.first_id + qs, qIdx = (int)(pq - q.gateway[qs]);
    for (int i = 0; i < ix.count[u]; ++i) {  // writeSeedList, krnlWriteSeedList.cu:28-35
      const int pos = ix.pos[ix.offset[u] + i];
      const int ts = t.seq_of(pos);
      v.push_back(Hit{t.first_id + ts, (int)(pos - t.gateway[ts]), qID, qIdx, 0, 0, 0, 0, 0.0});
    }
  }
  if (stage == ORACLE_STAGE_RAW_SEEDS) return v;
  auto tlen = [&](const Hit& h) { return t.lengths[h.tID - t.first_id]; };
  auto qlen = [&](const Hit& h) { return q.lengths[h.qID - q.first_id]; };
  // deleteSeedsOnSequenceBoundary, _deleteSeedsOnSequenceBoundary.cu:192-269
  v.erase(std::remove_if(v.begin(), v.end(), [&](const Hit& h) { return l + h.qIdx > qlen(h); }), v.end());
  v.erase(std::remove_if(v.begin(), v.end(), [&](const Hit& h) { return l + h.tIdx > tlen(h); }), v.end());
  if (!p.local)
    v.erase(std::remove_if(v.begin(), v.end(),
                           [&](const Hit& h) {  // is_onCorner, .cuh:21-49
                             const int s = h.tIdx - h.qIdx;
                             return (s + p.gap < 0) || (s + qlen(h) - p.gap > tlen(h));
                           }),
            v.end());
  // sortSeeds / measure_distance, _sortSeeds.cuh:14-55
  std::stable_sort(v.begin(), v.end(), [](const Hit& a, const Hit& b) {
    if (a.qID != b.qID) return a.qID < b.qID;
    if (a.tID != b.tID) return a.tID < b.tID;
    const int da = a.tIdx - a.qIdx, db = b.tIdx - b.qIdx;
    if (da != db) return da < db;
    return a.qIdx < b.qIdx;
  });
  // deletingIsolateSeeds then deleteDuplicateSeeds
  remove_with_predecessor(v, [&](const Hit& s, const Hit& pr) { return !near_pair(s, pr, p.width, p.gap); });
  remove_with_predecessor(v, [&](const Hit& s, const Hit& pr) { return near_pair(s, pr, p.width, p.gap); });
  if (stage == ORACLE_STAGE_FILTERED_SEEDS) return v;
  // hit arrays start at (l, l, l, l*MATCH_POINT), CDeviceHitList.cu:283-286
  for (auto& h : v) { h.tLen = l; h.qLen = l; h.match = l; h.score = l * kMatch; }
  // alignmentHits, CDeviceHitList_alignmentHits.cu:122-348
  std::stable_sort(v.begin(), v.end(), [&](const Hit& a, const Hit& b) {  // alignLengthBackward
    return qlen(a) - (a.qIdx + a.qLen) > qlen(b) - (b.qIdx + b.qLen);
  });
  for (auto& h : v) align_backward(h, t, q, p.gap, p.local != 0);
  std::stable_sort(v.begin(), v.end(), [](const Hit& a, const Hit& b) { return a.qIdx > b.qIdx; });
  for (auto& h : v) align_forward(h, t, q, p.gap, p.local != 0);
  // calculateEvalue, krnlCalculateEvalue.cu:5-23
  for (auto& h : v) h.evalue = p.K * p.totalDB * qlen(h) * std::exp(-p.lambda * h.score);
  if (stage == ORACLE_STAGE_ALIGNED) return v;
  // deleteHits_lowEValue / deleteHits_tooShort, _deleteBadHits.cu:7-221
  if (p.cutOff != -1)
    v.erase(std::remove_if(v.begin(), v.end(), [&](const Hit& h) { return p.cutOff < h.evalue; }), v.end());
  v.erase(std::remove_if(v.begin(), v.end(), [&](const Hit& h) { return l + p.stride > h.qLen; }), v.end());
  // resultSorting, utilResultSorting.cuh:7-26, then deleteHits_duplicateResult
  std::stable_sort(v.begin(), v.end(), [](const Hit& a, const Hit& b) {
    if (a.qID / 2 != b.qID / 2) return a.qID / 2 < b.qID / 2;
    return a.score > b.score;
  });
  remove_with_predecessor(v, [](const Hit& s, const Hit& pr) {
    return s.tID == pr.tID && s.tIdx == pr.tIdx && s.qID == pr.qID && s.qIdx == pr.qIdx;
  });
  return v;
}

/* ------------------------------------------------------------------ */
/* Results: CHostResultHolder.cu                                       */
/* ------------------------------------------------------------------ */
struct Holder {
  std::vector<std::string> qLabels;  // two per read
  std::vector<char> qStrand;
  std::vector<std::string> tLabels;  // one per result row
  std::vector<int> tStart;
  std::vector<Hit> hits;
  explicit Holder(const std::vector<Fasta>& q) {
    for (const auto& f : q) {
      qLabels.push_back(f.label); qLabels.push_back(f.label);
      qStrand.push_back('+'); qStrand.push_back('-');
    }
  }
  /* fixResult: global stable sort by (qID/2, score desc), :75-128 */
  void fix() {
    std::vector<int> idx(hits.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
      if (hits[a].qID / 2 != hits[b].qID / 2) return hits[a].qID / 2 < hits[b].qID / 2;
      return hits[a].score > hits[b].score;
    });
    std::vector<Hit> h2; std::vector<std::string> l2; std::vector<int> s2;
    for (int i : idx) { h2.push_back(hits[i]); l2.push_back(tLabels[i]); s2.push_back(tStart[i]); }
    hits.swap(h2); tLabels.swap(l2); tStart.swap(s2);
  }
  /* printResult, :131-243 */
  void print(int numOut, const std::string& path) const {
    std::ofstream ofs(path.c_str(), std::ios::app);
    std::string preLabel, preTLabel;
    int preQIdx = 0, preTIdx = 0, preTLen = 0, preQLen = 0, preMatch = 0, preScore = 0;
    char preStrand = 0;
    double preE = 0;
    int count = 0;
    for (size_t i = 0; i < hits.size(); ++i) {
      const Hit& h = hits[i];
      const std::string& ql = qLabels[h.qID];
      if (preLabel != ql) count = 0;
      if (numOut == -1 || preLabel != ql || count < numOut) {
        const std::string& tl = tLabels[i];
        const char strand = qStrand[h.qID];
        const int tIdx = h.tIdx + tStart[i];
        if (preLabel != ql || preQIdx != h.qIdx || preStrand != strand || preTLabel != tl ||
            preTIdx != tIdx || preTLen != h.tLen || preQLen != h.qLen || preMatch != h.match ||
            preScore != h.score || preE != h.evalue) {
          ofs << ql << "\t" << h.qIdx << "\t" << h.qLen << "\t" << strand << "\t" << tl << "\t"
              << tIdx << "\t" << h.tLen << "\t" << h.match << "("
              << static_cast<double>(h.match * 100) / h.qLen << "%)" << "\t" << h.score << "\t"
              << h.evalue << std::endl;
          ++count;
          preLabel = ql; preQIdx = h.qIdx; preStrand = strand; preTLabel = tl; preTIdx = tIdx;
          preTLen = h.tLen; preQLen = h.qLen; preMatch = h.match; preScore = h.score; preE = h.evalue;
        }
      }
    }
  }
};

Window window_of(const SeqList& s, int b, int e, std::vector<int32_t>& gw) {
  gw.clear();
  for (int i = b; i < e; ++i) gw.push_back(s.gateway[i] - s.gateway[b]);
  Window w;
  w.bases = s.bases.data() + s.gateway[b];
  w.n = s.gateway[e] - s.gateway[b];
  w.gateway = gw.data();
  w.lengths = s.lengths.data() + b;
  w.nseqs = e - b;
  w.first_id = b;
  return w;
}

/* CHostSchedular::search, CHostSchedular.cu:43-130, with OpenMP over the
 * query windows of one target window (results appended in window order). */
void search(const Params& p, const Settings& st, const SeqList& tl, const SeqList& ql, Holder& holder) {
  const int tVRAM = budget_to_int(st.tVRAM), qVRAM = budget_to_int(st.qVRAM);
  const int tEnd = (int)tl.gateway.size() - 1;
  for (int tb = 0, te = 1; tb < tEnd; tb = te++) {
    const int tBase = tl.gateway[tb];  // moveTargetWindow
    while (te < tEnd && tl.gateway[te + 1] - tBase < tVRAM) ++te;
    std::vector<int32_t> tgw;
    const Window tw = window_of(tl, tb, te, tgw);
    const Index ix = build_index(tw, p.l, p.stride, p.cutRepeat);
    const int qEnd = ((int)ql.gateway.size() - 1) / 2;
    std::vector<std::pair<int, int>> qwins;
    for (int qb = 0, qe = 1; qb < qEnd; qb = qe++) {  // moveQueryWindow
      const int qBase = ql.gateway[qb * 2];
      while (qe < qEnd && ql.gateway[qe * 2 + 2] - qBase < qVRAM) ++qe;
      qwins.emplace_back(qb, qe);
    }
    std::vector<std::vector<Hit>> res(qwins.size());
    bool failed = false;
    std::string err;
#pragma omp parallel for schedule(dynamic, 1)
    for (long k = 0; k < (long)qwins.size(); ++k) {
      try {
        std::vector<int32_t> qgw;
        const Window qw = window_of(ql, qwins[k].first * 2, qwins[k].second * 2, qgw);
        res[k] = window_search(p, ix, tw, qw, ORACLE_STAGE_FINAL);
      } catch (const std::exception& e) {
#pragma omp critical
        { failed = true; err = e.what(); }
      }
    }
    if (failed) fail(-6, err);
    for (auto& r : res) {  // getResult + addLabel + addStartIdx
      for (const Hit& h : r) {
        holder.hits.push_back(h);
        holder.tLabels.push_back(tl.labels[h.tID]);
        holder.tStart.push_back(tl.startIdx[h.tID]);
      }
    }
  }
}

int run_main(int argc, const char** argv) {
  const Settings st = parse_settings(argc, argv);
  { std::ofstream ofs(st.out.c_str()); }  // main.cu:26-27
  Params p{st.lmer, st.stride, st.cutRepeat, st.width, st.gap, st.local,
           st.cutOff, st.totalDB, st.K, st.lambda};
  Loader qload(st.qfiles, budget_to_int(st.qRAM / 2));
  while (qload.fileIndex() != -1) {  // main.cu:44-104
    std::vector<Fasta> qf;
    qload.load(qf);
    Holder holder(qf);
    Loader tload(st.tfiles, budget_to_int(st.tRAM));
    while (tload.fileIndex() != -1) {
      std::vector<Fasta> tf;
      tload.load(tf);
      SeqList tl, ql;
      for (const auto& f : tf) { tl.add(f.seq, st.lmer); tl.labels.push_back(f.label); tl.startIdx.push_back(f.startIdx); }
      for (const auto& f : qf) {
        ql.add(f.seq, st.lmer); ql.labels.push_back(f.label); ql.startIdx.push_back(0);
        ql.add(reverse_complement(f.seq), st.lmer); ql.labels.push_back(f.label); ql.startIdx.push_back(0);
      }
      search(p, st, tl, ql, holder);
    }
    holder.fix();
    holder.print(st.numOut, st.out);
  }
  return 0;
}

oracle_hits to_c(const std::vector<Hit>& v) {
  oracle_hits o;
  o.n = (int64_t)v.size();
  const size_t n = v.size() ? v.size() : 1;
  o.t_id = (int32_t*)std::malloc(n * 4); o.t_idx = (int32_t*)std::malloc(n * 4);
  o.q_id = (int32_t*)std::malloc(n * 4); o.q_idx = (int32_t*)std::malloc(n * 4);
  o.t_len = (int32_t*)std::malloc(n * 4); o.q_len = (int32_t*)std::malloc(n * 4);
  o.match = (int32_t*)std::malloc(n * 4); o.score = (int32_t*)std::malloc(n * 4);
  o.evalue = (double*)std::malloc(n * 8);
  for (size_t i = 0; i < v.size(); ++i) {
    o.t_id[i] = v[i].tID; o.t_idx[i] = v[i].tIdx; o.q_id[i] = v[i].qID; o.q_idx[i] = v[i].qIdx;
    o.t_len[i] = v[i].tLen; o.q_len[i] = v[i].qLen; o.match[i] = v[i].match; o.score[i] = v[i].score;
    o.evalue[i] = v[i].evalue;
  }
  return o;
}

}  // namespace

extern "C" {

int oracle_window_search(const oracle_params* p, const char* t_bases, int64_t t_nbases,
                         const int32_t* t_gateway, const int32_t* t_lengths, int32_t t_nseqs,
                         int32_t t_begin, const char* q_bases, int64_t q_nbases,
                         const int32_t* q_gateway, const int32_t* q_lengths, int32_t q_nseqs,
                         int32_t q_begin, int32_t stage, oracle_hits* out) {
  try {
    if (!p || !out || p->lmer < 1 || p->lmer > kMaxLmer || p->stride < 1 || p->gap < 2 ||
        p->gap > kMaxGap || (q_begin & 1))
      fail(-1, "bad argument");
    Params pp{p->lmer, p->stride, p->cut_repeat, p->width, p->gap, p->local,
              p->cutoff, p->total_db, p->K, p->lambda};
    Window t{t_bases, t_nbases, t_gateway, t_lengths, t_nseqs, t_begin};
    Window q{q_bases, q_nbases, q_gateway, q_lengths, q_nseqs, q_begin};
    const Index ix = build_index(t, pp.l, pp.stride, pp.cutRepeat);
    *out = to_c(window_search(pp, ix, t, q, stage));
    return 0;
  } catch (const OracleError& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return -100;
  }
}

void oracle_hits_free(oracle_hits* h) {
  if (!h) return;
  std::free(h->t_id); std::free(h->t_idx); std::free(h->q_id); std::free(h->q_idx);
  std::free(h->t_len); std::free(h->q_len); std::free(h->match); std::free(h->score);
  std::free(h->evalue);
  std::memset(h, 0, sizeof(*h));
}

int oracle_main(int argc, const char** argv, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  try {
    return run_main(argc, argv);
  } catch (const OracleError& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return -100;
  }
}

const char* oracle_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"

#ifdef CLAST_ORACLE_MAIN
int main(int argc, const char** argv) {
  const int rc = oracle_main(argc, argv, 0);
  if (rc != 0) {
    std::fprintf(stderr, "error: %s\n", oracle_last_error());
    return 1;
  }
  return 0;
}
#endif
