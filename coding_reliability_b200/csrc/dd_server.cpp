// dd_server.cpp — the query server: continuous batching of distance-distribution
// queries on one GPU.
//
// Each admitted query owns a resident slot of 64 uint64 bins in one device
// array sized by the memory budget, plus a host-side cursor into its tile
// space.  A scheduler thread runs rounds: it admits queued queries into free
// slots (clearing their bins on the device), gives every active query a fair
// share of a round budget (round_ms x the measured pairs/ms), launches ONE
// persistent kernel over all those tile sub-ranges (dd::launch_round), then
// advances the cursors, reads back and post-processes the queries that
// finished, frees their slots and records their latency.  Queries that arrive
// while a round runs are admitted at the next round, so large and small
// queries overlap on the device and a small one never waits for a large one
// to finish.
//
// Host memory stays bounded for a long-running server: a finished query's
// record (its result) is kept until the result has been delivered (a wait
// that returned it, a poll that reported it done, or the query was cancelled
// by its client); the last kKeepDelivered delivered records stay answerable,
// older ones are dropped (never while a thread waits on them), and
// dd_server_release drops one at once.  Latency percentiles cover the last
// kLatencyWindow completed queries.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/codrel_b200.h"
#include "dd_host.h"

namespace {

using dd::u128;

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

constexpr uint64_t kSlotBytes = dd::kMaxBins * 8 + sizeof(dd::Job) + 16;  // bins + job entry + cursor
constexpr size_t kKeepDelivered = 4096;   // delivered results that stay answerable
constexpr size_t kLatencyWindow = 65536;  // completed queries behind p50 / p99

struct Query {
  uint64_t ticket = 0;
  dd_request req;
  dd::Shape shape;
  dd::Job job;            // the whole instance (tile_offset 0, tiles = all)
  u128 pairs = 0;
  uint64_t cursor = 0;    // next tile of the instance
  int slot = -1;
  bool cancelled = false;
  bool done = false;
  bool delivered = false; // its result reached the client (or the client cancelled it)
  int waiters = 0;        // threads inside dd_server_wait on this query: it is not dropped meanwhile
  double t_submit = 0;
  dd_result result{};     // zero until the query finishes
};

}  // namespace

struct dd_server {
  int device = 0;
  dd_server_options opt;
  dd_context* ctx = nullptr;  // null in dry-run mode
  unsigned long long* d_slots = nullptr;
  uint32_t nslots = 0;
  std::vector<int> free_slots;
  std::deque<uint64_t> queue;
  std::vector<uint64_t> active;
  std::unordered_map<uint64_t, Query> queries;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread worker;
  std::mutex shutdown_mu;      // serialises dd_server_shutdown (the worker is joined once)
  bool stop = false;
  // calls inside the API functions below; dd_server_destroy frees nothing until
  // every one has left (a waiter woken by the shutdown still has to re-take mu)
  int inside = 0;
  std::condition_variable cv_idle;
  int failed = DD_OK;
  std::string failure;
  uint64_t next_ticket = 1;
  double rate_pairs_per_ms = 4.0e9;  // refined from every round
  // stats
  uint64_t submitted = 0, admitted = 0, completed = 0, rejected = 0, cancelled = 0, rounds = 0;
  double busy_ms = 0;
  u128 pairs_done = 0;
  std::vector<double> latencies;  // ring of the last kLatencyWindow completions
  size_t latency_next = 0;
  std::deque<uint64_t> delivered;  // delivered records, oldest first
};

namespace {

// Marks an API call as inside the server; constructed and destroyed with s->mu held.
struct Inside {
  dd_server* s;
  explicit Inside(dd_server* srv) : s(srv) { ++s->inside; }
  ~Inside() {
    if (--s->inside == 0) s->cv_idle.notify_all();
  }
  Inside(const Inside&) = delete;
  Inside& operator=(const Inside&) = delete;
};

// Records that q's result reached its client; drops the oldest delivered
// records beyond kKeepDelivered (skipping any a thread still waits on).
void note_delivered(dd_server* s, Query& q) {
  if (q.delivered) return;
  q.delivered = true;
  s->delivered.push_back(q.ticket);
  for (size_t tries = s->delivered.size(); s->delivered.size() > kKeepDelivered && tries > 0; --tries) {
    const uint64_t t = s->delivered.front();
    s->delivered.pop_front();
    auto it = s->queries.find(t);
    if (it == s->queries.end()) continue;
    if (it->second.waiters > 0) { s->delivered.push_back(t); continue; }
    s->queries.erase(it);
  }
}

void finish(dd_server* s, Query& q, int status) {
  q.done = true;
  q.result.status = (uint32_t)status;
  q.result.nbins = q.shape.nbins;
  q.result.h = q.shape.h;
  q.result.A = q.shape.A;
  q.result.user_tag = q.req.user_tag;
  q.result.total_ms = now_ms() - q.t_submit;
  if (status == DD_OK) {
    s->completed++;
    if (s->latencies.size() < kLatencyWindow) s->latencies.push_back(q.result.total_ms);
    else s->latencies[s->latency_next] = q.result.total_ms;
    s->latency_next = (s->latency_next + 1) % kLatencyWindow;
    s->pairs_done += q.pairs;
  } else if (status == DD_ERR_CANCELLED) {
    s->cancelled++;
  }
  if (q.slot >= 0) {
    s->free_slots.push_back(q.slot);
    q.slot = -1;
  }
  if (q.cancelled) note_delivered(s, q);  // its client went away (or asked for the status, which stays)
  s->cv_done.notify_all();
}

uint64_t pairs_per_tile(const Query& q) {
  const u128 per = q.job.tiles ? q.pairs / q.job.tiles : 1;
  return per ? (uint64_t)per : 1;
}

void scheduler(dd_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_work.wait(lk, [s] { return s->stop || !s->queue.empty() || !s->active.empty(); });
    if (s->stop) break;
    // admission: queued queries take free slots (their bins are cleared on the stream)
    while (!s->queue.empty() && !s->free_slots.empty()) {
      Query& q = s->queries[s->queue.front()];
      s->queue.pop_front();
      if (q.cancelled) { finish(s, q, DD_ERR_CANCELLED); continue; }
      q.slot = s->free_slots.back();
      s->free_slots.pop_back();
      s->admitted++;
      if (s->ctx) {
        const cudaError_t e = cudaMemsetAsync(s->d_slots + (size_t)q.slot * dd::kMaxBins, 0, dd::kMaxBins * 8,
                                              (cudaStream_t)dd::context_stream(s->ctx));
        if (e != cudaSuccess) { s->failed = DD_ERR_CUDA; s->failure = cudaGetErrorString(e); }
      }
      s->active.push_back(q.ticket);
    }
    if (s->active.empty()) continue;
    // plan one round: a fair share of the round budget for every active query
    const double budget = s->rate_pairs_per_ms * (double)s->opt.round_ms;
    const double share = budget / (double)s->active.size();
    std::vector<dd::Job> jobs;
    std::vector<uint32_t> kernels;
    std::vector<uint64_t> take(s->active.size(), 0);
    u128 round_pairs = 0;
    for (size_t k = 0; k < s->active.size(); ++k) {
      Query& q = s->queries[s->active[k]];
      const uint64_t remaining = q.job.tiles - q.cursor;
      uint64_t t = (uint64_t)(share / (double)pairs_per_tile(q));
      t = std::max<uint64_t>(1, std::min(t, remaining));
      take[k] = t;
      dd::Job j = q.job;
      j.tile_offset = q.cursor;
      j.tiles = t;
      j.bins = s->d_slots ? s->d_slots + (size_t)q.slot * dd::kMaxBins : nullptr;
      jobs.push_back(j);
      kernels.push_back(q.req.kernel);
      round_pairs += (u128)t * pairs_per_tile(q);
    }
    // run it (outside the lock: submit / poll / cancel stay responsive)
    lk.unlock();
    float ms = 0;
    int st = s->failed;
    if (st == DD_OK && s->ctx) {
      st = dd::launch_round(s->ctx, jobs, kernels, &ms);
    } else if (st == DD_OK) {
      // dry run: a round "takes" round_ms, so queues, slots and latencies behave
      // as on a device whose throughput is the initial rate estimate
      std::this_thread::sleep_for(std::chrono::milliseconds(s->opt.round_ms));
      ms = (float)s->opt.round_ms;
    }
    lk.lock();
    s->rounds++;
    s->busy_ms += ms;
    if (ms > 0.05) s->rate_pairs_per_ms = std::max(1e6, (double)round_pairs / ms);
    if (st != DD_OK) {
      s->failed = st;
      s->failure = std::string("round failed: ") + dd_last_error();
    }
    // advance cursors; read back and finish what completed
    std::vector<uint64_t> still;
    for (size_t k = 0; k < s->active.size(); ++k) {
      Query& q = s->queries[s->active[k]];
      q.cursor += take[k];
      if (s->failed != DD_OK) { finish(s, q, s->failed); continue; }
      if (q.cancelled) { finish(s, q, DD_ERR_CANCELLED); continue; }
      if (q.cursor < q.job.tiles) { still.push_back(q.ticket); continue; }
      uint64_t raw[dd::kMaxBins] = {0};
      if (s->ctx) {
        const cudaError_t e = cudaMemcpy(raw, s->d_slots + (size_t)q.slot * dd::kMaxBins, dd::kMaxBins * 8,
                                         cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { s->failed = DD_ERR_CUDA; s->failure = cudaGetErrorString(e); finish(s, q, DD_ERR_CUDA); continue; }
      }
      std::memset(&q.result, 0, sizeof(q.result));
      dd::postprocess(q.req, q.shape, raw, q.result);
      q.result.pairs_lo = (uint64_t)q.pairs;
      q.result.pairs_hi = (uint64_t)(q.pairs >> 64);
      q.result.kernel_used = s->ctx ? (dd::uses_mma(s->ctx, q.job, q.req.kernel) ? DD_KERNEL_MMA : DD_KERNEL_POPC)
                                    : 0xFFFFFFFFu;
      q.result.mma_epilogue = q.result.kernel_used == DD_KERNEL_MMA ? dd::mma_epilogue_used(s->ctx) : 0u;
      q.result.kernel_ms = ms;
      finish(s, q, DD_OK);
    }
    s->active.swap(still);
  }
  // shutting down: everything unfinished is cancelled
  for (uint64_t t : s->active) finish(s, s->queries[t], DD_ERR_CANCELLED);
  for (uint64_t t : s->queue) finish(s, s->queries[t], DD_ERR_CANCELLED);
  s->active.clear();
  s->queue.clear();
}

}  // namespace

extern "C" {

int dd_server_create(int device, const dd_server_options* opts, dd_server** out) {
  if (!out) { dd::set_error("out is NULL"); return DD_ERR_INVALID_ARGUMENT; }
  *out = nullptr;
  dd_server* s = new dd_server();
  s->device = device;
  std::memset(&s->opt, 0, sizeof(s->opt));
  if (opts) s->opt = *opts;
  if (!s->opt.memory_budget_bytes) s->opt.memory_budget_bytes = 64ull << 20;
  if (!s->opt.max_queue) s->opt.max_queue = 1024;
  if (!s->opt.round_ms) s->opt.round_ms = 20;
  const uint64_t slots = s->opt.memory_budget_bytes / kSlotBytes;
  if (slots == 0) { delete s; dd::set_error("memory budget below one query slot"); return DD_ERR_OUT_OF_MEMORY; }
  s->nslots = (uint32_t)std::min<uint64_t>(slots, 1u << 20);
  if (s->opt.inject_alloc_failure) {
    delete s;
    dd::set_error("slot allocation failed (injected)");
    return DD_ERR_OUT_OF_MEMORY;
  }
  if (!s->opt.dry_run) {
    int st = dd_context_create(device, nullptr, &s->ctx);
    if (st != DD_OK) { delete s; return st; }
    // KERNEL_AUTO queries run on the kernel the autotuner measures fastest on this
    // GPU (about a second, once per server)
    st = dd_autotune(s->ctx, nullptr);
    if (st != DD_OK) { dd_context_destroy(s->ctx); delete s; return st; }
    const cudaError_t e = cudaMalloc(&s->d_slots, (size_t)s->nslots * dd::kMaxBins * 8);
    if (e != cudaSuccess) {
      dd_context_destroy(s->ctx);
      delete s;
      dd::set_error(std::string("query slots: ") + cudaGetErrorString(e));
      return DD_ERR_OUT_OF_MEMORY;
    }
  }
  for (int i = (int)s->nslots - 1; i >= 0; --i) s->free_slots.push_back(i);
  s->worker = std::thread(scheduler, s);
  *out = s;
  return DD_OK;
}

int dd_server_submit(dd_server* s, const dd_request* req, uint64_t* ticket) {
  if (!s || !req) { dd::set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  Query q;
  std::string err;
  int st = dd::derive_shape(*req, q.shape, err);
  if (st != DD_OK) { dd::set_error(err); return st; }
  std::vector<dd::Job> jobs;
  dd::plan_jobs(q.shape, *req, jobs);
  q.job = jobs[0];
  q.req = *req;
  q.pairs = dd::planned_pairs(q.shape, *req);
  q.t_submit = now_ms();
  std::lock_guard<std::mutex> lk(s->mu);
  Inside in(s);
  if (s->failed != DD_OK) { dd::set_error("server failed: " + s->failure); return s->failed; }
  if (s->stop) { dd::set_error("server is shutting down"); return DD_ERR_CANCELLED; }
  if (s->queue.size() >= s->opt.max_queue && s->free_slots.empty()) {
    s->rejected++;
    dd::set_error("admission refused: all query slots busy and the queue is full");
    return DD_ERR_BUSY;
  }
  q.ticket = s->next_ticket++;
  s->submitted++;
  s->queue.push_back(q.ticket);
  if (ticket) *ticket = q.ticket;
  s->queries.emplace(q.ticket, q);
  s->cv_work.notify_one();
  return DD_OK;
}

int dd_server_poll(dd_server* s, uint64_t ticket, dd_result* res, int* done) {
  if (!s || !done) { dd::set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  std::lock_guard<std::mutex> lk(s->mu);
  Inside in(s);
  auto it = s->queries.find(ticket);
  if (it == s->queries.end()) { dd::set_error("unknown ticket"); return DD_ERR_NOT_FOUND; }
  *done = it->second.done ? 1 : 0;
  if (it->second.done && res) {
    *res = it->second.result;
    note_delivered(s, it->second);
  }
  return DD_OK;
}

int dd_server_wait(dd_server* s, uint64_t ticket, double timeout_s, dd_result* res) {
  if (!s) { dd::set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  std::unique_lock<std::mutex> lk(s->mu);
  Inside in(s);
  auto it = s->queries.find(ticket);
  if (it == s->queries.end()) { dd::set_error("unknown ticket"); return DD_ERR_NOT_FOUND; }
  // the record stays put while waiters > 0 (references into the map survive rehashing)
  Query* q = &it->second;
  q->waiters++;
  auto ready = [q] { return q->done; };
  bool finished = true;
  if (timeout_s < 0) s->cv_done.wait(lk, ready);
  else finished = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
  q->waiters--;
  if (!finished) {
    dd::set_error("query still running");
    return DD_ERR_TIMEOUT;
  }
  if (res) *res = q->result;
  const int st = (int)q->result.status;
  note_delivered(s, *q);  // may drop older records, never this one's reference before here
  return st;
}

int dd_server_cancel(dd_server* s, uint64_t ticket) {
  if (!s) { dd::set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  std::lock_guard<std::mutex> lk(s->mu);
  Inside in(s);
  auto it = s->queries.find(ticket);
  if (it == s->queries.end()) { dd::set_error("unknown ticket"); return DD_ERR_NOT_FOUND; }
  Query& q = it->second;
  if (q.done) return DD_OK;
  q.cancelled = true;
  auto qi = std::find(s->queue.begin(), s->queue.end(), ticket);
  if (qi != s->queue.end()) {  // not admitted yet: drop it now
    s->queue.erase(qi);
    finish(s, q, DD_ERR_CANCELLED);
  }
  return DD_OK;
}

int dd_server_release(dd_server* s, uint64_t ticket) {
  if (!s) { dd::set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  std::lock_guard<std::mutex> lk(s->mu);
  Inside in(s);
  auto it = s->queries.find(ticket);
  if (it == s->queries.end()) { dd::set_error("unknown ticket"); return DD_ERR_NOT_FOUND; }
  if (!it->second.done) { dd::set_error("query still running (cancel it and wait first)"); return DD_ERR_BUSY; }
  if (it->second.waiters > 0) { dd::set_error("threads are waiting on this query"); return DD_ERR_BUSY; }
  if (it->second.delivered) {
    auto d = std::find(s->delivered.begin(), s->delivered.end(), ticket);
    if (d != s->delivered.end()) s->delivered.erase(d);
  }
  s->queries.erase(it);
  return DD_OK;
}

int dd_server_get_stats(dd_server* s, dd_server_stats* out) {
  if (!s || !out) { dd::set_error("NULL argument"); return DD_ERR_INVALID_ARGUMENT; }
  std::lock_guard<std::mutex> lk(s->mu);
  Inside in(s);
  std::memset(out, 0, sizeof(*out));
  out->submitted = s->submitted;
  out->admitted = s->admitted;
  out->completed = s->completed;
  out->rejected = s->rejected;
  out->cancelled = s->cancelled;
  out->rounds = s->rounds;
  out->active = (uint32_t)s->active.size();
  out->queued = (uint32_t)s->queue.size();
  out->slots = s->nslots;
  out->slots_free = (uint32_t)s->free_slots.size();
  out->busy_ms = s->busy_ms;
  out->pairs_lo = (uint64_t)s->pairs_done;
  out->pairs_hi = (uint64_t)(s->pairs_done >> 64);
  out->pairs_per_s = s->busy_ms > 0 ? (double)s->pairs_done / (s->busy_ms * 1e-3) : 0.0;
  if (!s->latencies.empty()) {
    std::vector<double> v = s->latencies;
    auto pct = [&](double p) {  // nearest rank
      const size_t i = (size_t)std::max(0.0, std::min<double>((double)v.size() - 1, std::ceil(p * v.size()) - 1));
      std::nth_element(v.begin(), v.begin() + (std::ptrdiff_t)i, v.end());
      return v[i];
    };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
  }
  return DD_OK;
}

int dd_server_shutdown(dd_server* s) {
  if (!s) return DD_OK;
  std::lock_guard<std::mutex> once(s->shutdown_mu);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  // the scheduler cancels every unfinished query on its way out, which wakes the waiters
  if (s->worker.joinable()) s->worker.join();
  return DD_OK;
}

int dd_server_destroy(dd_server* s) {
  if (!s) return DD_OK;
  dd_server_shutdown(s);
  {
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_idle.wait(lk, [s] { return s->inside == 0; });
  }
  if (s->d_slots) cudaFree(s->d_slots);
  if (s->ctx) dd_context_destroy(s->ctx);
  delete s;
  return DD_OK;
}

}  // extern "C"
