// clast_serve.cu -- the served form: resident targets, requests admitted and
// batched as they arrive, several batches on the GPU at once.
//
// No counterpart in the reference, which maps one query file per process run
// and rebuilds every index per query RAM load (main.cu:44-89).  Here the
// target indexes stay resident; `lanes` worker threads each own a context
// (stream, scratch pool, pinned result buffers) and run one batch at a time
// through clast_map.  A batch is the queued requests a free lane takes, in
// arrival order, while their read bases fit max_batch_bases and the device
// bytes estimated for all batches in flight fit the HBM budget.  Every
// request becomes its own RAM loads in the batch (the load rule of
// CFASTALoader.cpp:43-87 over the request's reads), so its query windows,
// and with them its hits, are those of the request mapped alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/clast_gpu.h"
#include "clast_engine.h"

using namespace clast;

namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Device bytes a batch may take while it runs: padded strands, 2-bit words and
// N masks, per-strand tables, seeds and hits, results (a generous bound per
// base and per read, plus a fixed part for the per-window buffers).
int64_t batch_bytes(int64_t bases, int64_t reads) { return 32 * bases + 96 * reads + (16ll << 20); }

struct Request {
  enum State { QUEUED, RUNNING, DONE, FAILED, CANCELLED };
  int64_t id = 0;
  State state = QUEUED;
  std::vector<char> bases;
  std::vector<int64_t> offsets;    // n_reads + 1, from 0
  std::vector<int64_t> load_sizes;  // RAM loads of the request
  int64_t n_reads = 0, n_bases = 0, bytes = 0;
  int64_t t_submit = 0, t_start = 0, t_done = 0;
  int code = CLAST_OK;
  std::string err;
  // result (clast_map_result fields)
  std::vector<int64_t> load_offsets;
  std::vector<int32_t> f[10];  // read strand t_load t_seq t_idx q_idx t_len q_len match score
  std::vector<double> evalue;
};

}  // namespace

struct clast_server {
  const clast_targets* T = nullptr;
  clast_params p{};
  clast_server_config cfg{};
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
  std::vector<std::thread> lanes;
  std::vector<clast_ctx*> ctxs;
  bool stop = false;
  int64_t next_id = 1;
  int64_t in_flight = 0;  // estimated device bytes of the batches running
  clast_server_stats stats{};
  mutable std::mutex err_mu;
  std::string err;

  void set_err(const std::string& e) {
    std::lock_guard<std::mutex> lk(err_mu);
    err = e;
  }
  void lane_main(int k);
  void run_batch(clast_ctx* ctx, std::vector<Request*>& batch, char*& pinned, size_t& pinned_bytes);
};

namespace {

// CFASTALoader's RAM loads over one request's reads: a record joins the load
// while the load's bases plus its own stay below the budget.
std::vector<int64_t> request_loads(const std::vector<int64_t>& offsets, int64_t budget) {
  std::vector<int64_t> loads;
  int64_t cur = 0, sum = 0;
  for (size_t i = 0; i + 1 < offsets.size(); ++i) {
    const int64_t len = offsets[i + 1] - offsets[i];
    if (cur > 0 && sum + len >= budget) {
      loads.push_back(cur);
      cur = 0;
      sum = 0;
    }
    ++cur;
    sum += len;
  }
  if (cur) loads.push_back(cur);
  return loads;
}

}  // namespace

void clast_server::run_batch(clast_ctx* ctx, std::vector<Request*>& batch, char*& pinned, size_t& pinned_bytes) {
  // the batch's reads back to back in pinned memory, every request its own loads
  int64_t nb = 0, nr = 0;
  for (Request* r : batch) {
    nb += r->n_bases;
    nr += r->n_reads;
  }
  if ((size_t)nb + 1 > pinned_bytes) {
    if (pinned) cudaFreeHost(pinned);
    pinned = nullptr;
    pinned_bytes = 0;
    const size_t want = (size_t)nb + (size_t)nb / 2 + (1 << 20);
    if (cudaMallocHost(&pinned, want) != cudaSuccess) {
      (void)cudaGetLastError();
      throw std::bad_alloc();
    }
    pinned_bytes = want;
  }
  std::vector<int64_t> offsets;
  offsets.reserve((size_t)nr + 1);
  offsets.push_back(0);
  std::vector<int64_t> loads;
  std::vector<size_t> first_load;  // per request: index of its first load
  int64_t at = 0;
  for (Request* r : batch) {
    if (r->n_bases) std::memcpy(pinned + at, r->bases.data(), (size_t)r->n_bases);
    for (int64_t i = 1; i <= r->n_reads; ++i) offsets.push_back(at + r->offsets[i]);
    at += r->n_bases;
    first_load.push_back(loads.size());
    loads.insert(loads.end(), r->load_sizes.begin(), r->load_sizes.end());
  }
  clast_seqs seqs{nr, pinned, offsets.data(), 0};
  clast_map_result res;
  const int rc = clast_map(ctx, T, &p, cfg.q_vram, &seqs, (int32_t)loads.size(), loads.data(), &res);
  if (rc != CLAST_OK) {
    const std::string e = clast_last_error(ctx);
    for (Request* r : batch) {
      r->code = rc;
      r->err = e;
    }
    return;
  }
  // split by request: its loads are a contiguous run of the batch's loads
  int64_t read0 = 0;
  for (size_t k = 0; k < batch.size(); ++k) {
    Request* r = batch[k];
    const size_t l0 = first_load[k], nl = r->load_sizes.size();
    const int64_t a = res.load_offsets[l0], b = res.load_offsets[l0 + nl];
    r->load_offsets.resize(nl + 1);
    for (size_t j = 0; j <= nl; ++j) r->load_offsets[j] = res.load_offsets[l0 + j] - a;
    int32_t* src[10] = {res.read, res.strand, res.t_load, res.t_seq, res.t_idx, res.q_idx, res.t_len, res.q_len,
                        res.match, res.score};
    for (int j = 0; j < 10; ++j) r->f[j].assign(src[j] + a, src[j] + b);
    for (int32_t& x : r->f[0]) x -= (int32_t)read0;
    r->evalue.assign(res.evalue + a, res.evalue + b);
    r->code = CLAST_OK;
    read0 += r->n_reads;
  }
  clast_map_result_free(&res);
}

void clast_server::lane_main(int k) {
  clast_ctx* ctx = ctxs[k];
  char* pinned = nullptr;
  size_t pinned_bytes = 0;
  for (;;) {
    std::vector<Request*> batch;
    int64_t bytes = 0, bases = 0;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] {
        return stop || (!queue.empty() && in_flight + queue.front()->bytes <= cfg.hbm_budget);
      });
      if (stop) break;
      while (!queue.empty()) {
        Request* r = queue.front();
        if (!batch.empty() && (bases + r->n_bases > cfg.max_batch_bases || in_flight + bytes + r->bytes > cfg.hbm_budget))
          break;
        queue.pop_front();
        r->state = Request::RUNNING;
        r->t_start = now_ns();
        batch.push_back(r);
        bases += r->n_bases;
        bytes += r->bytes;
      }
      in_flight += bytes;
      stats.hbm_in_flight_max = std::max(stats.hbm_in_flight_max, in_flight);
      stats.running += (int64_t)batch.size();
      stats.queued = (int64_t)queue.size();
    }
    try {
      run_batch(ctx, batch, pinned, pinned_bytes);
    } catch (const std::bad_alloc&) {
      for (Request* r : batch) {
        r->code = CLAST_ERR_NOMEM;
        r->err = "out of host memory for the batch";
      }
    } catch (const std::exception& e) {
      for (Request* r : batch) {
        r->code = CLAST_ERR_INTERNAL;
        r->err = e.what();
      }
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      const int64_t t = now_ns();
      for (Request* r : batch) {
        r->state = r->code == CLAST_OK ? Request::DONE : Request::FAILED;
        r->t_done = t;
        std::vector<char>().swap(r->bases);  // the reads are no longer needed
        std::vector<int64_t>().swap(r->offsets);
      }
      in_flight -= bytes;
      stats.running -= (int64_t)batch.size();
      stats.batches += 1;
      stats.requests += (int64_t)batch.size();
      stats.bases += bases;
      stats.max_batch_requests = std::max<int64_t>(stats.max_batch_requests, (int64_t)batch.size());
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
  if (pinned) cudaFreeHost(pinned);
}

extern "C" {

int clast_server_create(clast_ctx* ctx, const clast_targets* t, const clast_params* p,
                        const clast_server_config* cfg, clast_server** out) {
  if (!ctx || !out) return CLAST_ERR_ARG;
  *out = nullptr;
  return guarded(ctx, [&]() -> int {
    check_params(p);
    if (!t) throw std::invalid_argument("targets are null");
    if (t->ctx != ctx) throw std::invalid_argument("the targets were created on another context");
    for (const auto& w : t->wins)
      if (p->lmer != w.ix->l || p->stride != w.ix->stride || p->cut_repeat != w.ix->cut)
        throw std::invalid_argument("params differ from the ones the targets were built with");
    CLAST_CK(cudaSetDevice(ctx->device));
    settle_targets(ctx, t);  // the lanes read the indexes only once they are built
    std::unique_ptr<clast_server> s(new clast_server());
    s->T = t;
    s->p = *p;
    s->device = ctx->device;
    clast_server_config c = cfg ? *cfg : clast_server_config{};
    if (c.lanes <= 0) c.lanes = 4;
    if (c.lanes > 16) throw std::invalid_argument("at most 16 lanes");
    if (c.q_vram <= 0) c.q_vram = 2000000;
    if (c.q_ram <= 0) c.q_ram = 32000000;
    if (c.max_batch_bases <= 0) c.max_batch_bases = 8000000;
    if (c.hbm_reserve <= 0) c.hbm_reserve = 2ll << 30;
    if (c.hbm_budget <= 0) {
      size_t free_b = 0, total_b = 0;
      CLAST_CK(cudaMemGetInfo(&free_b, &total_b));
      c.hbm_budget = (int64_t)free_b - c.hbm_reserve;
      if (c.hbm_budget <= 0) throw std::bad_alloc();
    }
    s->cfg = c;
    s->stats.hbm_budget = c.hbm_budget;
    for (int k = 0; k < c.lanes; ++k) {
      clast_ctx* lc = nullptr;
      const int rc = clast_ctx_create(ctx->device, &lc);
      if (rc != CLAST_OK) {
        for (clast_ctx* x : s->ctxs) clast_ctx_destroy(x);
        throw std::runtime_error("cannot create a lane context");
      }
      lc->dp_warp = clast::kDpWarpOff;  // see clast_ctx::dp_warp
      s->ctxs.push_back(lc);
    }
    clast_server* raw = s.get();
    for (int k = 0; k < c.lanes; ++k)
      s->lanes.emplace_back([raw, k]() {
        cudaSetDevice(raw->device);
        raw->lane_main(k);
      });
    *out = s.release();
    return CLAST_OK;
  });
}

int clast_server_submit(clast_server* s, const clast_seqs* reads, int64_t* request_id) {
  if (!s || !reads || !request_id) return CLAST_ERR_ARG;
  *request_id = 0;
  try {
    if (reads->bases_on_device) throw std::invalid_argument("served requests take host reads");
    const int64_t n = reads->n_seqs;
    if (n < 0 || (n > 0 && (!reads->offsets || !reads->bases))) throw std::invalid_argument("bad reads");
    std::unique_ptr<Request> r(new Request());
    r->n_reads = n;
    r->offsets.resize((size_t)n + 1);
    const int64_t o0 = n ? reads->offsets[0] : 0;
    for (int64_t i = 0; i <= n; ++i) {
      r->offsets[i] = reads->offsets[i] - o0;
      if (i && r->offsets[i] < r->offsets[i - 1]) throw std::invalid_argument("read offsets decrease");
      if (i && r->offsets[i] - r->offsets[i - 1] >= s->cfg.q_ram)
        throw std::invalid_argument("a read is not shorter than the RAM load budget");
    }
    r->n_bases = r->offsets[n];
    r->bases.assign(reads->bases + o0, reads->bases + o0 + r->n_bases);
    r->load_sizes = request_loads(r->offsets, s->cfg.q_ram);
    r->bytes = batch_bytes(r->n_bases, r->n_reads);
    if (r->bytes > s->cfg.hbm_budget) {
      s->set_err("request needs about " + std::to_string(r->bytes) + " device bytes; the budget is " +
                 std::to_string(s->cfg.hbm_budget));
      return CLAST_ERR_NOMEM;
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->stop) throw std::invalid_argument("server is stopping");
      r->id = s->next_id++;
      r->t_submit = now_ns();
      *request_id = r->id;
      s->queue.push_back(r.get());
      s->stats.queued = (int64_t)s->queue.size();
      s->reqs.emplace(r->id, std::move(r));
    }
    s->cv_work.notify_one();
    return CLAST_OK;
  } catch (const std::bad_alloc&) {
    s->set_err("out of host memory");
    return CLAST_ERR_NOMEM;
  } catch (const std::exception& e) {
    s->set_err(e.what());
    return CLAST_ERR_ARG;
  }
}

int clast_server_poll(clast_server* s, int64_t request_id, int32_t timeout_ms, clast_map_result* out) {
  if (!s || !out) return CLAST_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) {
    s->set_err("unknown request " + std::to_string(request_id));
    return CLAST_ERR_ARG;
  }
  Request* r = it->second.get();
  auto final_state = [r] { return r->state == Request::DONE || r->state == Request::FAILED ||
                                  r->state == Request::CANCELLED; };
  if (timeout_ms < 0) s->cv_done.wait(lk, final_state);
  else if (timeout_ms > 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), final_state);
  if (!final_state()) return CLAST_PENDING;
  if (r->state == Request::CANCELLED) return CLAST_ERR_CANCELLED;
  if (r->state == Request::FAILED) {
    s->set_err(r->err);
    return r->code;
  }
  out->n = (int64_t)r->evalue.size();
  out->load_offsets = r->load_offsets.data();
  int32_t** dst[10] = {&out->read, &out->strand, &out->t_load, &out->t_seq, &out->t_idx, &out->q_idx, &out->t_len,
                       &out->q_len, &out->match, &out->score};
  for (int j = 0; j < 10; ++j) *dst[j] = r->f[j].data();
  out->evalue = r->evalue.data();
  out->owner = nullptr;
  return CLAST_OK;
}

int clast_server_cancel(clast_server* s, int64_t request_id) {
  if (!s) return CLAST_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end() || it->second->state != Request::QUEUED) {
      s->set_err("request " + std::to_string(request_id) + " is not queued");
      return CLAST_ERR_ARG;
    }
    Request* r = it->second.get();
    s->queue.erase(std::find(s->queue.begin(), s->queue.end(), r));
    r->state = Request::CANCELLED;
    r->t_done = now_ns();
    s->stats.queued = (int64_t)s->queue.size();
  }
  s->cv_done.notify_all();
  s->cv_work.notify_all();
  return CLAST_OK;
}

int clast_server_release(clast_server* s, int64_t request_id) {
  if (!s) return CLAST_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) {
    s->set_err("unknown request " + std::to_string(request_id));
    return CLAST_ERR_ARG;
  }
  const Request::State st = it->second->state;
  if (st == Request::QUEUED || st == Request::RUNNING) {
    s->set_err("request " + std::to_string(request_id) + " has not finished");
    return CLAST_ERR_ARG;
  }
  s->reqs.erase(it);
  return CLAST_OK;
}

int clast_server_times(clast_server* s, int64_t request_id, int64_t* submit_ns, int64_t* start_ns, int64_t* done_ns) {
  if (!s) return CLAST_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return CLAST_ERR_ARG;
  if (submit_ns) *submit_ns = it->second->t_submit;
  if (start_ns) *start_ns = it->second->t_start;
  if (done_ns) *done_ns = it->second->t_done;
  return CLAST_OK;
}

int clast_server_get_stats(clast_server* s, clast_server_stats* out) {
  if (!s || !out) return CLAST_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  return CLAST_OK;
}

const char* clast_server_last_error(const clast_server* s) {
  if (!s) return "null server";
  std::lock_guard<std::mutex> lk(s->err_mu);
  return s->err.c_str();
}

void clast_server_destroy(clast_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    const int64_t t = now_ns();
    for (Request* r : s->queue) {
      r->state = Request::CANCELLED;
      r->t_done = t;
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  s->cv_done.notify_all();
  for (auto& th : s->lanes) th.join();
  for (clast_ctx* c : s->ctxs) clast_ctx_destroy(c);
  delete s;
}

}  // extern "C"
