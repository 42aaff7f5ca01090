// clast_host.cpp -- host side of the drop-in `clast` command line.
//
// Keeps the reference's command line (listenCommandLine.cpp:281-325,
// CHostSetting.cu:62-142), its FASTA RAM loads (CFASTALoader.cpp:11-170) and
// its 10-column TSV (CHostResultHolder.cu:131-243), and hands the device
// work to the C ABI in include/clast_gpu.h: every target window is indexed
// once and kept in HBM, and every query RAM load is mapped in one pass.
#include "clast_host.h"

#include <cerrno>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <chrono>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../../include/clast_gpu.h"

namespace {

struct UsageError : std::runtime_error {
  int code;
  UsageError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// ---------------------------------------------------------------------------
// settings
// ---------------------------------------------------------------------------
struct Settings {
  double tRAM = 64, qRAM = 64, tVRAM = 64, qVRAM = 2;  // common.hpp:12-15 (MBase)
  int lmer = 15, stride = 5, cutRepeat = 20, width = 100, gap = 8, numOut = -1, local = 0, device = 0,
      sleep = 0;
  double cutOff = 10;
  std::vector<std::string> tfiles, qfiles;
  std::string out;
  double totalDB = 0;
};

// Whole-string numbers, as boost::lexical_cast requires.
int to_int(const std::string& s, const char* flag) {
  if (s.empty() || s[0] == ' ' || s[0] == '\t') throw UsageError(1, std::string("Odd parameter after ") + flag);
  errno = 0;
  char* end = nullptr;
  const long v = std::strtol(s.c_str(), &end, 10);
  if (end != s.c_str() + s.size() || errno == ERANGE || v < INT_MIN || v > INT_MAX)
    throw UsageError(1, std::string("Odd parameter was inputted. Check the after of \"") + flag + "\".");
  return (int)v;
}
double to_double(const std::string& s, const char* flag) {
  if (s.empty() || s[0] == ' ' || s[0] == '\t') throw UsageError(1, std::string("Odd parameter after ") + flag);
  char* end = nullptr;
  const double v = std::strtod(s.c_str(), &end);
  if (end != s.c_str() + s.size())
    throw UsageError(1, std::string("Odd parameter was inputted. Check the after of \"") + flag + "\".");
  return v;
}

bool read_file(const std::string& path, std::string& data) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  data.clear();
  if (std::fseek(f, 0, SEEK_END) == 0) {
    const long size = std::ftell(f);
    if (size > 0 && std::fseek(f, 0, SEEK_SET) == 0) {
      data.resize((size_t)size);
      const size_t got = std::fread(&data[0], 1, (size_t)size, f);
      data.resize(got);
    }
  }
  char buf[1 << 16];  // whatever remains (streams whose size is unknown)
  size_t k;
  while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) data.append(buf, k);
  std::fclose(f);
  return true;
}

// One FASTA file split into lines, in parallel, and into records the way
// CFASTAFileLoader::read walks it (CFASTALoader.cpp:112-170): a record is
// finalised at the next line holding '>', at an empty line and at the end of
// the file, and only if its label is not empty; a line holding '@' sets the
// start index of the record being read (to_int of the rest of the line);
// sequence lines read while there is no label are ignored.
struct ParsedFasta {
  enum : uint8_t { kSeq = 0, kLabel = 1, kAt = 2, kEmpty = 3 };
  std::string data;
  std::vector<int64_t> start;  // line i: [start[i], end(i)), '\n' excluded
  std::vector<uint8_t> type;
  std::vector<int64_t> kept;   // sequence lines: characters kept (spaces removed)
  struct Rec {
    int64_t label_line, first, last;  // sequence lines in [first, last)
    int64_t len;
    int32_t start_idx;
  };
  std::vector<Rec> recs;
  int64_t end(int64_t i) const {
    if (i + 1 < (int64_t)start.size()) return start[i + 1] - 1;
    const int64_t n = (int64_t)data.size();  // the last line, with or without its '\n'
    return (n > 0 && data[n - 1] == '\n') ? n - 1 : n;
  }

  void parse() {
    const int64_t n = (int64_t)data.size();
    const char* d = data.data();
    // line starts: 0 and every position after a '\n' that is inside the file
    int nt = 1;
#ifdef _OPENMP
    nt = std::max(1, omp_get_max_threads());
#endif
    std::vector<std::vector<int64_t>> part(nt);
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int t = 0; t < nt; ++t) {
      const int64_t a = n * t / nt, b = n * (t + 1) / nt;
      const char* q = d + a;
      while (q < d + b) {
        const char* e = (const char*)std::memchr(q, '\n', (size_t)(d + b - q));
        if (!e) break;
        if (e + 1 < d + n) part[t].push_back((int64_t)(e + 1 - d));
        q = e + 1;
      }
    }
    start.clear();
    if (n > 0) start.push_back(0);
    for (auto& v : part) start.insert(start.end(), v.begin(), v.end());
    const int64_t nl = (int64_t)start.size();
    type.assign(nl, kSeq);
    kept.assign(nl, 0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nl; ++i) {
      const char* ln = d + start[i];
      const size_t len = (size_t)(end(i) - start[i]);
      if (std::memchr(ln, '>', len)) type[i] = kLabel;
      else if (std::memchr(ln, '@', len)) type[i] = kAt;
      else if (len == 0) type[i] = kEmpty;
      else {
        int64_t spaces = 0;
        for (size_t k = 0; k < len; ++k) spaces += ln[k] == ' ';
        kept[i] = (int64_t)len - spaces;
      }
    }
    recs.clear();
    int64_t label = -1, first = -1, last = -1, len = 0;
    int32_t start_idx = 0;
    auto finish = [&](int64_t i) {  // judgeContinueReading on the record read so far
      if (label < 0) return;
      recs.push_back(Rec{label, first < 0 ? i : first, first < 0 ? i : last, len, start_idx});
      label = -1;
      first = last = -1;
      len = 0;
      start_idx = 0;
    };
    for (int64_t i = 0; i < nl; ++i) {
      switch (type[i]) {
        case kLabel:
          finish(i);
          label = (end(i) - start[i] > 1) ? i : -1;  // the label is the line after its first character
          break;
        case kAt:
          try {
            const int64_t a = start[i] + 1, e = std::max(a, end(i));
            start_idx = to_int(std::string(d + a, (size_t)(e - a)), "@");
          } catch (const UsageError&) {
            throw UsageError(4, "bad file type: something was strange at the line which contains '@'.");
          }
          break;
        case kEmpty:
          finish(i);
          break;
        default:
          if (label >= 0) {
            if (first < 0) first = i;
            last = i + 1;
            len += kept[i];
          }
      }
    }
    finish(nl);
  }
};

// totalDatabaseSize: characters of every target line that has no '>'
// (CHostSetting.cu:46-58, std::getline splits on '\n' only).
long total_db_size(const std::vector<std::string>& files) {
  long total = 0;
  for (const auto& f : files) {
    ParsedFasta P;
    if (!read_file(f, P.data)) continue;
    const int64_t n = (int64_t)P.data.size();
    const char* d = P.data.data();
    int64_t sum = 0;
    // every byte that is not a '\n', minus the lines holding a '>'
#pragma omp parallel for reduction(+ : sum) schedule(static)
    for (int64_t i = 0; i < n; ++i) sum += d[i] != '\n';
    int64_t gt = 0;
    {
      int64_t a = 0;
      while (a < n) {
        const char* e = (const char*)std::memchr(d + a, '\n', (size_t)(n - a));
        const int64_t end = e ? (int64_t)(e - d) : n;
        if (std::memchr(d + a, '>', (size_t)(end - a))) gt += end - a;
        if (!e) break;
        a = end + 1;
      }
    }
    total += (long)(sum - gt);
  }
  return total;
}

Settings parse_args(int argc, const char* const* argv) {
  Settings s;
  enum St { START, VALUE, T_FILE, Q_FILE, O_FILE } st = START;
  std::string flag;
  static const char* kValueFlags[] = {"-tRAM", "-qRAM", "-tVRAM", "-qVRAM", "-lMer", "-stride", "-repeat",
                                      "-width", "-gap", "-numOut", "-cutOff", "-local", "-device", "-sleep"};
  auto is_value_flag = [](const std::string& a) {
    for (const char* f : kValueFlags)
      if (a == f) return true;
    return false;
  };
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    switch (st) {
      case START:
      case T_FILE:
      case Q_FILE:
        if (is_value_flag(a)) {
          flag = a;
          st = VALUE;
        } else if (a == "-t") {
          if (st == T_FILE) throw UsageError(1, "Odd parameter was inputted. Check the after of \"-t\".");
          st = T_FILE;
        } else if (a == "-q") {
          if (st == Q_FILE) throw UsageError(1, "Odd parameter was inputted. Check the after of \"-q\".");
          st = Q_FILE;
        } else if (a == "-o") {
          st = O_FILE;
        } else if (st == T_FILE) {
          s.tfiles.push_back(a);
        } else if (st == Q_FILE) {
          s.qfiles.push_back(a);
        } else {
          throw UsageError(1, "Odd parameter was inputted. Check the command line parameter.");
        }
        break;
      case VALUE: {
        const char* f = flag.c_str();
        if (flag == "-tRAM") s.tRAM = to_double(a, f);
        else if (flag == "-qRAM") s.qRAM = to_double(a, f);
        else if (flag == "-tVRAM") s.tVRAM = to_double(a, f);
        else if (flag == "-qVRAM") s.qVRAM = to_double(a, f);
        else if (flag == "-lMer") s.lmer = to_int(a, f);
        else if (flag == "-stride") s.stride = to_int(a, f);
        else if (flag == "-repeat") s.cutRepeat = to_int(a, f);
        else if (flag == "-width") s.width = to_int(a, f);
        else if (flag == "-gap") s.gap = to_int(a, f);
        else if (flag == "-numOut") s.numOut = to_int(a, f);
        else if (flag == "-cutOff") s.cutOff = to_double(a, f);
        else if (flag == "-local") s.local = to_int(a, f);
        else if (flag == "-device") s.device = to_int(a, f);
        else if (flag == "-sleep") s.sleep = to_int(a, f);
        st = START;
        break;
      }
      case O_FILE:
        s.out = a;
        st = START;
        break;
    }
  }
  // CHostSetting.cu:14-44, plus the ranges the reference needs but never checks
  if (s.lmer > 31) throw UsageError(1, "too large lMerLength was inputted.");
  if (s.gap > 16) throw UsageError(1, "too large allowableGap was inputted.");
  if (s.gap < 2) throw UsageError(1, "allowableGap must be larger than 1.");
  if (s.tfiles.empty()) throw UsageError(1, "no target file was inputted.");
  if (s.qfiles.empty()) throw UsageError(1, "no query file was inputted.");
  if (s.out.empty()) throw UsageError(1, "no output file was inputted.");
  if (s.lmer < 1) throw UsageError(1, "lMerLength must be at least 1.");
  if (s.stride < 1) throw UsageError(1, "strideLength must be at least 1.");
  s.tRAM *= 1000 * 1000;
  s.qRAM *= 1000 * 1000;
  s.tVRAM *= 1000 * 1000;
  s.qVRAM *= 1000 * 1000;
  return s;
}

int to_budget(double v) {
  if (!(v < 2147483648.0) || v < -2147483648.0)
    throw UsageError(1, "RAM/VRAM size does not fit a 32-bit base count");
  return (int)v;
}

// ---------------------------------------------------------------------------
// FASTA RAM loads (CFASTALoader.cpp)
// ---------------------------------------------------------------------------
struct Load {  // records of one RAM load
  std::vector<std::string> labels;
  std::vector<int32_t> start_idx;
  std::string bases;
  std::vector<int64_t> offsets{0};
  size_t size() const { return labels.size(); }
};

class Loader {
 public:
  Loader(const std::vector<std::string>& files, int budget) : files_(files), budget_(budget) {}

  // CFASTALoader::loadFASTA (CFASTALoader.cpp:11-41) with judgeContinueReading
  // (:43-87): records join the load while the load's bases plus the record's
  // stay below the budget; a record longer than the budget is skipped; the
  // load ends at the first record that does not fit, which opens the next
  // load.  Files are parsed once, in parallel; the bases of a load are
  // normalised (removeSpace + replaceSmallToBig, :89-106) in parallel.
  bool next(Load& out) {
    if (file_ < 0) return false;
    const int file_before = file_;
    int64_t sum = 0;
    std::vector<const ParsedFasta::Rec*> take;  // records of the current file
    for (; file_ < (int)files_.size(); ++file_, rec_ = 0) {
      const ParsedFasta& P = parsed(file_);
      take.clear();
      for (; rec_ < (int64_t)P.recs.size(); ++rec_) {
        const ParsedFasta::Rec& r = P.recs[rec_];
        if (r.len > budget_) continue;  // longer than the budget: skipped
        if (sum + r.len < budget_) {
          take.push_back(&r);
          sum += r.len;
        } else {
          if (take.empty() && out.size() == 0 && file_ == file_before)
            throw UsageError(2, "a FASTA record is exactly as long as the RAM budget (the reference never terminates)");
          flush(out, take);
          return true;
        }
      }
      flush(out, take);  // the load goes on in the next file
    }
    file_ = -1;
    return true;
  }
  bool done() const { return file_ < 0; }

 private:
  const ParsedFasta& parsed(int f) {
    if (f != cached_) {
      cache_ = ParsedFasta();
      if (!read_file(files_[f], cache_.data)) throw UsageError(3, "file \"" + files_[f] + "\" open failed.");
      cache_.parse();
      cached_ = f;
    }
    return cache_;
  }
  // appends records of the cached file to the load
  void flush(Load& out, const std::vector<const ParsedFasta::Rec*>& take) {
    const size_t k0 = out.labels.size();
    const size_t m = take.size();
    out.labels.resize(k0 + m);
    out.start_idx.resize(k0 + m);
    out.offsets.resize(k0 + m + 1);
    for (size_t i = 0; i < m; ++i) out.offsets[k0 + i + 1] = out.offsets[k0 + i] + take[i]->len;
    const size_t b0 = out.bases.size();
    out.bases.resize((size_t)out.offsets[k0 + m]);
    const ParsedFasta& P = cache_;
    const char* d = P.data.data();
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)m; ++i) {
      const ParsedFasta::Rec& r = *take[i];
      const int64_t la = P.start[r.label_line] + 1;
      out.labels[k0 + i].assign(d + la, (size_t)(P.end(r.label_line) - la));
      out.start_idx[k0 + i] = r.start_idx;
      char* w = &out.bases[0] + b0 + (out.offsets[k0 + i] - out.offsets[k0]);
      for (int64_t ln = r.first; ln < r.last; ++ln) {
        if (P.type[ln] != ParsedFasta::kSeq) continue;
        const int64_t e = P.end(ln);
        for (int64_t k = P.start[ln]; k < e; ++k) {
          char c = d[k];
          if (c == ' ') continue;
          if (c > 'Z') c = (char)(c - 32);
          if (c < 'A' || c > 'Z') c = 'N';
          *w++ = c;
        }
      }
    }
  }

  std::vector<std::string> files_;
  int budget_;
  int file_ = 0;
  int64_t rec_ = 0;
  int cached_ = -1;
  ParsedFasta cache_;
};

// Labels of every record of a list of loads, flat (clast_labels).
struct FlatLabels {
  std::string chars;
  std::vector<int64_t> offsets{0};
  std::vector<int32_t> start_idx;
  void add(const std::vector<Load>& loads) {
    for (const Load& L : loads)
      for (size_t i = 0; i < L.size(); ++i) {
        chars += L.labels[i];
        offsets.push_back((int64_t)chars.size());
        start_idx.push_back(L.start_idx[i]);
      }
  }
  clast_labels view() const { return clast_labels{(int64_t)offsets.size() - 1, chars.data(), offsets.data()}; }
};

// Wall-clock phases of one command-line run, printed to stderr when the
// environment variable CLAST_CLI_TIMING is set.
struct PhaseClock {
  bool on = std::getenv("CLAST_CLI_TIMING") != nullptr;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  void mark(const char* what) {
    const auto now = std::chrono::steady_clock::now();
    if (on) std::fprintf(stderr, "clast: %-22s %9.1f ms\n", what, std::chrono::duration<double, std::milli>(now - t).count());
    t = now;
  }
};

int run(int argc, const char* const* argv, std::string& err) {
  PhaseClock clock;
  Settings s = parse_args(argc, argv);
  // the CUDA context comes up on its own thread while the FASTA files are read
  clast_ctx* ctx = nullptr;
  int ctx_rc = CLAST_OK;
  std::thread ctx_thread([&]() { ctx_rc = clast_ctx_create(s.device, &ctx); });
  bool adopted = false;  // ctx_guard below owns the context
  struct Joiner {
    std::thread& th;
    clast_ctx*& ctx;
    bool& adopted;
    ~Joiner() {  // an early return or error: wait for the context and release it
      if (th.joinable()) th.join();
      if (ctx && !adopted) clast_ctx_destroy(ctx);
    }
  } joiner{ctx_thread, ctx, adopted};
  for (const auto& f : s.tfiles) {
    FILE* t = std::fopen(f.c_str(), "rb");
    if (!t) throw UsageError(3, "file \"" + f + "\" open failed.");
    std::fclose(t);
  }
  s.totalDB = (double)total_db_size(s.tfiles);
  clock.mark("database size");
  {  // main.cu:26-27: the output file is truncated first
    FILE* f = std::fopen(s.out.c_str(), "wb");
    if (!f) throw UsageError(3, "cannot open output file " + s.out);
    std::fclose(f);
  }
  const int t_budget = to_budget(s.tRAM), q_budget = to_budget(s.qRAM / 2);  // main.cu:42,63-65
  const int t_vram = to_budget(s.tVRAM), q_vram = to_budget(s.qVRAM);
  // every target RAM load (identical for every query load, main.cu:63-89)
  std::vector<Load> tloads;
  {
    Loader tl(s.tfiles, t_budget);
    while (!tl.done()) {
      tloads.emplace_back();
      tl.next(tloads.back());
    }
  }
  clock.mark("target FASTA");
  std::vector<Load> qloads;
  {
    Loader ql(s.qfiles, q_budget);
    while (!ql.done()) {
      qloads.emplace_back();
      ql.next(qloads.back());
    }
  }
  clock.mark("query FASTA");
  clast_params p;
  p.lmer = s.lmer;
  p.stride = s.stride;
  p.cut_repeat = s.cutRepeat;
  p.width = s.width;
  p.gap = s.gap;
  p.local = s.local;
  p.cutoff = s.cutOff;
  p.total_db = s.totalDB;
  p.K = 0.71;       // common.hpp:42
  p.lambda = 1.37;  // common.hpp:43
  // concatenated targets and reads (a load's bases are contiguous already)
  std::string tb, qb;
  std::vector<int64_t> toff{0}, qoff{0}, tsizes, qsizes;
  auto concat = [](const std::vector<Load>& loads, std::string& b, std::vector<int64_t>& off,
                   std::vector<int64_t>& sizes) {
    size_t total = 0, recs = 0;
    for (const Load& L : loads) {
      total += L.bases.size();
      recs += L.size();
    }
    b.reserve(total);
    off.reserve(recs + 1);
    for (const Load& L : loads) {
      const int64_t base = (int64_t)b.size();
      b.append(L.bases);
      for (size_t i = 1; i < L.offsets.size(); ++i) off.push_back(base + L.offsets[i]);
      sizes.push_back((int64_t)L.size());
    }
  };
  concat(tloads, tb, toff, tsizes);
  concat(qloads, qb, qoff, qsizes);
  FlatLabels tlabels, qlabels;
  tlabels.add(tloads);
  qlabels.add(qloads);
  clock.mark("concatenate");
  ctx_thread.join();
  clock.mark("CUDA context (wait)");
  int rc = ctx_rc;
  if (rc != CLAST_OK) {
    err = "cannot create a CUDA context on device " + std::to_string(s.device);
    return 5;
  }
  std::unique_ptr<clast_ctx, void (*)(clast_ctx*)> ctx_guard(ctx, clast_ctx_destroy);
  adopted = true;
  clast_seqs ts{(int64_t)(toff.size() - 1), tb.data(), toff.data()};
  clast_targets* targets = nullptr;
  rc = clast_targets_create(ctx, &p, t_vram, &ts, (int32_t)tsizes.size(), tsizes.data(), &targets);
  if (rc != CLAST_OK) {
    err = clast_last_error(ctx);
    return 6;
  }
  std::unique_ptr<clast_targets, void (*)(clast_targets*)> t_guard(targets, clast_targets_free);
  clast_seqs qs{(int64_t)(qoff.size() - 1), qb.data(), qoff.data()};
  clast_map_result res;
  rc = clast_map(ctx, targets, &p, q_vram, &qs, (int32_t)qsizes.size(), qsizes.data(), &res);
  if (rc != CLAST_OK) {
    err = clast_last_error(ctx);
    return 6;
  }
  std::unique_ptr<clast_map_result, void (*)(clast_map_result*)> r_guard(&res, clast_map_result_free);
  clock.mark("GPU search");
  const clast_labels ql = qlabels.view(), tl = tlabels.view();
  clast_tsv text;
  rc = clast_format_tsv(ctx, targets, &res, (int32_t)qsizes.size(), &ql, &tl, tlabels.start_idx.data(), s.numOut,
                        &text);
  if (rc != CLAST_OK) {
    err = clast_last_error(ctx);
    return 6;
  }
  std::unique_ptr<clast_tsv, void (*)(clast_tsv*)> text_guard(&text, clast_tsv_free);
  clock.mark("TSV text");
  // the file was truncated at start; the text goes in with several threads
  if (clast_write_file(s.out.c_str(), text.text, text.n_bytes, 8) != CLAST_OK)
    throw UsageError(3, "cannot write output file " + s.out);
  clock.mark("TSV write");
  return 0;
}

}  // namespace

#ifndef MADV_POPULATE_WRITE
#define MADV_POPULATE_WRITE 23  // Linux 5.14 (uapi/asm-generic/mman-common.h)
#endif

namespace {
// positional writes of buf[a, b) at the same offsets
bool pwrite_range(int fd, const char* buf, int64_t a, int64_t b) {
  while (a < b) {
    const ssize_t w = ::pwrite(fd, buf + a, (size_t)std::min<int64_t>(b - a, (int64_t)1 << 30), (off_t)a);
    if (w < 0 && errno == EINTR) continue;
    if (w <= 0) return false;
    a += w;
  }
  return true;
}
}  // namespace

extern "C" int clast_write_file(const char* path, const char* buf, int64_t n, int32_t threads) {
  if (!path || n < 0 || (n > 0 && !buf)) return CLAST_ERR_ARG;
  const int fd = ::open(path, O_RDWR | O_CREAT | O_TRUNC, 0644);
  if (fd < 0) return CLAST_ERR_ARG;
  bool ok = true;
  if (n > 0) {
    struct stat sb;
    void* map = MAP_FAILED;
    if (::fstat(fd, &sb) == 0 && S_ISREG(sb.st_mode) && ::ftruncate(fd, (off_t)n) == 0)
      map = ::mmap(nullptr, (size_t)n, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
    if (map == MAP_FAILED) {
      ok = pwrite_range(fd, buf, 0, n);  // one write at a time holds the file's lock anyway
    } else {
      // Each thread makes the pages of its own range in one call and copies
      // into them.  Where that call fails (no space, or a kernel without it)
      // the range goes in with positional writes, which report the error
      // instead of faulting on a page that cannot be made.
      char* dst = static_cast<char*>(map);
      const int64_t page = std::max<long>(4096, ::sysconf(_SC_PAGESIZE));
      const int parts = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(1, (int)threads), n >> 22));
      std::vector<int> part_ok(parts, 1);
      std::vector<std::thread> ts;
      for (int k = 0; k < parts; ++k)
        ts.emplace_back([&, k]() {
          const int64_t a = n * k / parts, b = n * (k + 1) / parts;
          const int64_t pa = a / page * page;
          if (::madvise(dst + pa, (size_t)(b - pa), MADV_POPULATE_WRITE) == 0) std::memcpy(dst + a, buf + a, (size_t)(b - a));
          else part_ok[k] = pwrite_range(fd, buf, a, b) ? 1 : 0;
        });
      for (auto& t : ts) t.join();
      for (int v : part_ok) ok = ok && v;
      if (::munmap(map, (size_t)n) != 0) ok = false;
    }
  }
  if (::close(fd) != 0) ok = false;
  return ok ? CLAST_OK : CLAST_ERR_ARG;
}

extern "C" int clast_cli_main(int argc, const char* const* argv, char* err_buf, int err_len) {
  std::string err;
  int rc = 0;
  try {
    rc = run(argc, argv, err);
  } catch (const UsageError& e) {
    err = e.what();
    rc = e.code;
  } catch (const std::exception& e) {
    err = e.what();
    rc = 7;
  }
  if (err_buf && err_len > 0) {
    std::snprintf(err_buf, (size_t)err_len, "%s", err.c_str());
  }
  return rc;
}
