// clast_host.cpp -- host side of the drop-in `clast` command line.
//
// Keeps the reference's command line (listenCommandLine.cpp:281-325,
// CHostSetting.cu:62-142), its FASTA RAM loads (CFASTALoader.cpp:11-170) and
// its 10-column TSV (CHostResultHolder.cu:131-243), and hands the device
// work to the C ABI in include/clast_gpu.h: every target window is indexed
// once and kept in HBM, and every query RAM load is mapped in one pass.
#include "clast_host.h"

#include <cerrno>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
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
  char buf[1 << 16];
  size_t k;
  while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) data.append(buf, k);
  std::fclose(f);
  return true;
}

// totalDatabaseSize: characters of every target line that has no '>'
// (CHostSetting.cu:46-58, std::getline splits on '\n' only).
long total_db_size(const std::vector<std::string>& files) {
  long total = 0;
  std::string d;
  for (const auto& f : files) {
    if (!read_file(f, d)) continue;
    size_t a = 0;
    while (a < d.size()) {
      size_t e = d.find('\n', a);
      const size_t end = (e == std::string::npos) ? d.size() : e;
      if (std::memchr(d.data() + a, '>', end - a) == nullptr) total += (long)(end - a);
      if (e == std::string::npos) break;
      a = e + 1;
    }
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

  // CFASTALoader::loadFASTA: records until one does not fit the budget.
  bool next(Load& out) {
    if (index_ < 0) return false;
    const int before = index_;
    for (; index_ < (int)files_.size(); ++index_)
      if (!read_file_part(files_[index_], out)) break;
    if (index_ == (int)files_.size()) index_ = -1;
    if (out.size() == 0 && index_ == before && index_ != -1)
      throw UsageError(2, "a FASTA record is exactly as long as the RAM budget (the reference never terminates)");
    return true;
  }
  bool done() const { return index_ < 0; }

 private:
  // judgeContinueReading, CFASTALoader.cpp:43-87
  bool judge(long pos, std::string& label, std::string& seq, int& start_idx, Load& out) {
    if (!label.empty()) {
      const long len = (long)seq.size();
      if (len > budget_) {  // longer than the budget: skipped
        label.clear();
        seq.clear();
        start_idx = 0;
        read_pos_ = pos;
      } else if (sum_ + len < budget_) {
        out.labels.push_back(label);
        out.start_idx.push_back(start_idx);
        out.bases += seq;
        out.offsets.push_back((int64_t)out.bases.size());
        sum_ += len;
        label.clear();
        seq.clear();
        start_idx = 0;
        read_pos_ = pos;
      } else {
        sum_ = 0;
        return false;
      }
    }
    return true;
  }

  // CFASTAFileLoader::read, CFASTALoader.cpp:112-170
  bool read_file_part(const std::string& path, Load& out) {
    if (path != cached_path_) {
      if (!read_file(path, data_)) throw UsageError(3, "file \"" + path + "\" open failed.");
      cached_path_ = path;
    }
    std::string label, seq;
    int start_idx = 0;
    size_t a = (size_t)read_pos_;
    long line_start = read_pos_;
    while (a < data_.size()) {
      const size_t e = data_.find('\n', a);
      const size_t end = (e == std::string::npos) ? data_.size() : e;
      const char* ln = data_.data() + a;
      const size_t n = end - a;
      if (std::memchr(ln, '>', n)) {
        if (!judge(line_start, label, seq, start_idx, out)) return false;
        label.assign(n ? ln + 1 : ln, n ? n - 1 : 0);
      } else if (std::memchr(ln, '@', n)) {
        try {
          start_idx = to_int(std::string(ln + 1, n - 1), "@");
        } catch (const UsageError&) {
          throw UsageError(4, "bad file type: something was strange at the line which contains '@'.");
        }
      } else if (n == 0) {
        if (!judge(line_start, label, seq, start_idx, out)) return false;
      } else if (!label.empty()) {  // removeSpace + replaceSmallToBig, :89-106
        for (size_t i = 0; i < n; ++i) {
          char c = ln[i];
          if (c == ' ') continue;
          if (c > 'Z') c = (char)(c - 32);
          if (c < 'A' || c > 'Z') c = 'N';
          seq.push_back(c);
        }
      }
      if (e == std::string::npos) break;
      a = e + 1;
      line_start = (long)a;
    }
    if (!judge((long)data_.size(), label, seq, start_idx, out)) return false;
    read_pos_ = 0;
    return true;
  }

  std::vector<std::string> files_;
  int budget_;
  int index_ = 0;
  long read_pos_ = 0, sum_ = 0;
  std::string cached_path_, data_;
};

// ---------------------------------------------------------------------------
// TSV (CHostResultHolder::printResult)
// ---------------------------------------------------------------------------
struct TargetMeta {
  std::vector<std::vector<std::string>> labels;  // per load
  std::vector<std::vector<int32_t>> start_idx;
};

void write_tsv(FILE* f, const Load& q, int64_t read0, const TargetMeta& tm, const clast_map_result& r, int64_t a,
               int64_t b, int num_out) {
  // which hits print: consecutive identical records are skipped and at most
  // num_out per query label (the first is always printed)
  const int64_t n = b - a;
  std::vector<char> print(n, 0);
  const std::string* pre_label = nullptr;
  const std::string* pre_tlabel = nullptr;
  int pre_qidx = 0, pre_tidx = 0, pre_tlen = 0, pre_qlen = 0, pre_match = 0, pre_score = 0;
  char pre_strand = 0;
  double pre_e = 0;
  int count = 0;
  static const std::string kEmpty;
  for (int64_t j = 0; j < n; ++j) {
    const int64_t i = a + j;
    const std::string& ql = q.labels[r.read[i] - read0];
    const bool new_label = !pre_label || *pre_label != ql;
    if (new_label) count = 0;
    if (num_out == -1 || new_label || count < num_out) {
      const std::string& tl = tm.labels[r.t_load[i]][r.t_seq[i]];
      const int tidx = r.t_idx[i] + tm.start_idx[r.t_load[i]][r.t_seq[i]];
      const char strand = r.strand[i] ? '-' : '+';
      if (new_label || pre_qidx != r.q_idx[i] || pre_strand != strand || *pre_tlabel != tl || pre_tidx != tidx ||
          pre_tlen != r.t_len[i] || pre_qlen != r.q_len[i] || pre_match != r.match[i] ||
          pre_score != r.score[i] || pre_e != r.evalue[i]) {
        print[j] = 1;
        ++count;
        pre_label = &ql;
        pre_qidx = r.q_idx[i];
        pre_strand = strand;
        pre_tlabel = &tl;
        pre_tidx = tidx;
        pre_tlen = r.t_len[i];
        pre_qlen = r.q_len[i];
        pre_match = r.match[i];
        pre_score = r.score[i];
        pre_e = r.evalue[i];
      }
    }
  }
  // format in parallel chunks, write in order
  const int64_t chunk = 1 << 14;
  const int64_t nchunks = (n + chunk - 1) / chunk;
  std::vector<std::string> bufs(nchunks);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t c = 0; c < nchunks; ++c) {
    std::string& o = bufs[c];
    char line[512];
    for (int64_t j = c * chunk; j < std::min(n, (c + 1) * chunk); ++j) {
      if (!print[j]) continue;
      const int64_t i = a + j;
      const std::string& ql = q.labels[r.read[i] - read0];
      const std::string& tl = tm.labels[r.t_load[i]][r.t_seq[i]];
      const int tidx = r.t_idx[i] + tm.start_idx[r.t_load[i]][r.t_seq[i]];
      // std::ostream's default double format is %g with precision 6
      const int k = std::snprintf(line, sizeof(line), "\t%d\t%d\t%c\t", r.q_idx[i], r.q_len[i],
                                  r.strand[i] ? '-' : '+');
      o += ql;
      o.append(line, k);
      o += tl;
      const int k2 = std::snprintf(line, sizeof(line), "\t%d\t%d\t%d(%g%%)\t%d\t%g\n", tidx, r.t_len[i], r.match[i],
                                   (double)(r.match[i] * 100) / r.q_len[i], r.score[i], r.evalue[i]);
      o.append(line, k2);
    }
  }
  for (const auto& o : bufs) std::fwrite(o.data(), 1, o.size(), f);
}

int run(int argc, const char* const* argv, std::string& err) {
  Settings s = parse_args(argc, argv);
  for (const auto& f : s.tfiles) {
    FILE* t = std::fopen(f.c_str(), "rb");
    if (!t) throw UsageError(3, "file \"" + f + "\" open failed.");
    std::fclose(t);
  }
  s.totalDB = (double)total_db_size(s.tfiles);
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
  std::vector<Load> qloads;
  {
    Loader ql(s.qfiles, q_budget);
    while (!ql.done()) {
      qloads.emplace_back();
      ql.next(qloads.back());
    }
  }
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
  // concatenated targets and reads
  std::string tb, qb;
  std::vector<int64_t> toff{0}, qoff{0}, tsizes, qsizes;
  TargetMeta tm;
  for (const Load& L : tloads) {
    for (size_t i = 0; i < L.size(); ++i) {
      tb.append(L.bases, L.offsets[i], L.offsets[i + 1] - L.offsets[i]);
      toff.push_back((int64_t)tb.size());
    }
    tsizes.push_back((int64_t)L.size());
    tm.labels.push_back(L.labels);
    tm.start_idx.push_back(L.start_idx);
  }
  for (const Load& L : qloads) {
    for (size_t i = 0; i < L.size(); ++i) {
      qb.append(L.bases, L.offsets[i], L.offsets[i + 1] - L.offsets[i]);
      qoff.push_back((int64_t)qb.size());
    }
    qsizes.push_back((int64_t)L.size());
  }
  clast_ctx* ctx = nullptr;
  int rc = clast_ctx_create(s.device, &ctx);
  if (rc != CLAST_OK) {
    err = "cannot create a CUDA context on device " + std::to_string(s.device);
    return 5;
  }
  std::unique_ptr<clast_ctx, void (*)(clast_ctx*)> ctx_guard(ctx, clast_ctx_destroy);
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
  FILE* f = std::fopen(s.out.c_str(), "ab");
  if (!f) throw UsageError(3, "cannot open output file " + s.out);
  int64_t read0 = 0;
  for (size_t k = 0; k < qloads.size(); ++k) {
    write_tsv(f, qloads[k], read0, tm, res, res.load_offsets[k], res.load_offsets[k + 1], s.numOut);
    read0 += (int64_t)qloads[k].size();
  }
  std::fclose(f);
  return 0;
}

}  // namespace

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
