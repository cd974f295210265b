// gw_serve.cu -- serving PPR queries with continuous batching.
//
// A server owns one context's stream and a device arena of visit tables.  Its
// scheduler thread repeats supersteps:
//   1. admit arrived queries in FIFO order while their visit table fits in the
//      arena (a query that does not fit waits until completed queries free
//      space), clearing each new table;
//   2. launch one walk kernel over a mix of walk chunks: every admitted query
//      with walks left contributes up to `quantum` of them (the plain mode
//      takes one whole query per superstep instead);
//   3. for the queries whose last walks ran, launch the top-k kernel, copy
//      the lists back, free their tables and complete their tickets.
// Queries arriving while a superstep runs join the next one, next to queries
// already in flight.  Walk w of a query draws from Philox counter
// (w, hop, query stream, 0), so a query's result depends only on its source,
// budget and stream, not on what it was mixed with.  A query whose table fills
// up is restarted with a table four times larger (same draws, same result).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "gw_ctx.h"
#include "gw_ppr.h"

namespace {

uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Arrivals closer than this are waited for by spinning (yielding) rather
// than by a timed sleep.
constexpr uint64_t kSpinNs = 300000;

uint64_t pow2_at_least(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// First-fit allocator over [0, size) slots with coalescing frees.
class Arena {
 public:
  explicit Arena(uint64_t size = 0) { reset(size); }
  void reset(uint64_t size) {
    free_.clear();
    if (size) free_[0] = size;
  }
  bool alloc(uint64_t n, uint64_t* off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      *off = it->first;
      const uint64_t rest = it->second - n, start = it->first + n;
      free_.erase(it);
      if (rest) free_[start] = rest;
      return true;
    }
    return false;
  }
  void release(uint64_t off, uint64_t n) {
    auto it = free_.emplace(off, n).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }

 private:
  std::map<uint64_t, uint64_t> free_;
};

struct Query {
  uint32_t source = 0, budget = 0, stream = 0;
  uint64_t arrival_ns = 0, admit_ns = 0, done_ns = 0;
  uint64_t table_off = 0, table_slots = 0;
  uint64_t factor = 0;
  uint32_t issued = 0;  // walks launched so far
  uint32_t restarts = 0;
  bool done = false;
  gw_status status = GW_OK;
  std::vector<uint32_t> ids, counts;
};

}  // namespace

struct gw_server {
  gw_ctx* ctx = nullptr;
  gw_walk_params params{};
  gw::WalkArgs args{};
  gw_serve_config cfg{};
  std::thread thread;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  // earliest arrival the scheduler may be spinning for; a submission of an
  // earlier query lowers it so the spin ends at once
  std::atomic<uint64_t> next_due{~0ull};
  uint64_t next_ticket = 1;
  std::deque<uint64_t> pending;              // submitted, not admitted (FIFO)
  std::vector<uint64_t> active;              // admitted, not complete
  std::unordered_map<uint64_t, Query> queries;
  Arena arena;
  gw_devbuf tables;
  gw_serve_stats stats{};
  gw_status fatal = GW_OK;
  // per-superstep staging: pinned host mirrors and device arrays
  gw_hostbuf h_stage;
  gw_devbuf d_stage;
  uint32_t stage_cap = 0;
  gw_devbuf d_topk_segs, d_topk_cand;  // segmented top-k of large finishing tables
};

namespace {

// Staging layout for up to n queries in one superstep: the launch's chunk
// cursor; the per-query inputs (copied up); then the results, one contiguous
// range copied back: the launch's status word, the table-full flags and the
// top-k lists.  The status word and the flags are also copied up, as zeros.
struct Stage {
  unsigned long long *cursor, *prefix, *id_base, *toff;
  uint32_t *sources, *tmask, *stream, *status, *full, *ids, *counts;
};

size_t stage_bytes(uint32_t n, uint32_t k) {
  return 8 + (size_t)(n + 1) * 8 + 2 * (size_t)n * 8 + 3 * (size_t)n * 4 + 4 + (size_t)n * 4 +
         2 * (size_t)n * k * 4;
}

Stage carve(void* base, uint32_t n, uint32_t k) {
  Stage s;
  char* p = static_cast<char*>(base);
  s.cursor = reinterpret_cast<unsigned long long*>(p);
  p += 8;
  s.prefix = reinterpret_cast<unsigned long long*>(p);
  p += (size_t)(n + 1) * 8;
  s.id_base = reinterpret_cast<unsigned long long*>(p);
  p += (size_t)n * 8;
  s.toff = reinterpret_cast<unsigned long long*>(p);
  p += (size_t)n * 8;
  s.sources = reinterpret_cast<uint32_t*>(p);
  p += (size_t)n * 4;
  s.tmask = reinterpret_cast<uint32_t*>(p);
  p += (size_t)n * 4;
  s.stream = reinterpret_cast<uint32_t*>(p);
  p += (size_t)n * 4;
  s.status = reinterpret_cast<uint32_t*>(p);
  p += 4;
  s.full = reinterpret_cast<uint32_t*>(p);
  p += (size_t)n * 4;
  s.ids = reinterpret_cast<uint32_t*>(p);
  p += (size_t)n * k * 4;
  s.counts = reinterpret_cast<uint32_t*>(p);
  return s;
}

gw::QueryView make_view(const Stage& d, unsigned long long* tables, uint32_t n) {
  gw::QueryView qv{};
  qv.sources = d.sources;
  qv.walk_prefix = d.prefix;
  qv.id_base = d.id_base;
  qv.table_off = d.toff;
  qv.table_mask = d.tmask;
  qv.tables = tables;
  qv.full = d.full;
  qv.stream = d.stream;
  qv.cursor = d.cursor;
  qv.nq = n;
  return qv;
}

// One superstep; returns false on a CUDA error (recorded in srv->fatal).
bool superstep(gw_server* srv) {
  gw_ctx* ctx = srv->ctx;
  cudaStream_t st = ctx->stream;
  const uint32_t k = srv->cfg.k;
  // Queries are reached through pointers taken under the lock: map nodes do
  // not move, and only this thread changes an admitted query's fields.
  std::vector<Query*> admitted, cq;
  std::vector<uint64_t> chosen;
  std::vector<uint32_t> take;
  {
    std::unique_lock<std::mutex> lock(srv->mu);
    const uint64_t t = now_ns();
    while (!srv->pending.empty()) {
      Query& q = srv->queries[srv->pending.front()];
      if (q.arrival_ns > t) break;
      const uint64_t slots = pow2_at_least(std::max<uint64_t>(256, (uint64_t)q.budget * q.factor));
      uint64_t off;
      if (!srv->arena.alloc(slots, &off)) break;  // wait for completed queries to free space
      q.table_off = off;
      q.table_slots = slots;
      q.admit_ns = t;
      srv->active.push_back(srv->pending.front());
      admitted.push_back(&q);
      srv->pending.pop_front();
    }
    // the walk chunks of this superstep; queries that finish in it go first
    uint64_t total = 0;
    std::vector<uint64_t> later;
    std::vector<uint32_t> later_take;
    for (uint64_t tk : srv->active) {
      Query& q = srv->queries[tk];
      const uint32_t left = q.budget - q.issued;
      uint32_t n;
      if (srv->cfg.mode == GW_SERVE_PLAIN) {
        if (!chosen.empty() || !later.empty()) break;
        n = left;
      } else {
        if (total >= srv->cfg.max_walks_per_step) break;
        n = (uint32_t)std::min<uint64_t>({(uint64_t)left, srv->cfg.quantum, srv->cfg.max_walks_per_step - total});
      }
      if (n == left) {
        chosen.push_back(tk);
        take.push_back(n);
      } else {
        later.push_back(tk);
        later_take.push_back(n);
      }
      total += n;
    }
    chosen.insert(chosen.end(), later.begin(), later.end());
    take.insert(take.end(), later_take.begin(), later_take.end());
    for (uint64_t tk : chosen) cq.push_back(&srv->queries[tk]);
  }
  for (Query* q : admitted)
    gw::launch_clear_tables(srv->tables.as<unsigned long long>() + q->table_off, q->table_slots, st);
  if (chosen.empty()) return true;
  const uint32_t n = (uint32_t)chosen.size();
  if (n > srv->stage_cap) {
    const size_t bytes = stage_bytes(n, k);
    if (srv->h_stage.ensure(bytes) != cudaSuccess || srv->d_stage.ensure(bytes) != cudaSuccess) {
      srv->fatal = ctx->fail(GW_E_NOMEM, "serve staging allocation");
      return false;
    }
    srv->stage_cap = n;
  }
  Stage h = carve(srv->h_stage.p, n, k), d = carve(srv->d_stage.p, n, k);
  unsigned long long acc = 0;
  uint32_t nfin = 0;  // leading queries whose last walks run now
  for (uint32_t i = 0; i < n; ++i) {
    const Query& q = *cq[i];
    if (q.issued + take[i] == q.budget && nfin == i) ++nfin;
    h.prefix[i] = acc;
    h.id_base[i] = q.issued;  // walk index inside the query = its stream id
    h.toff[i] = q.table_off;
    h.sources[i] = q.source;
    h.tmask[i] = (uint32_t)(q.table_slots - 1);
    h.full[i] = 0;
    h.stream[i] = q.stream;
    acc += take[i];
  }
  h.prefix[n] = acc;
  h.status[0] = 0;
  const size_t head = stage_bytes(n, k) - 8 - 2 * (size_t)n * k * 4;  // prefix .. full
  cudaError_t e = cudaMemcpyAsync(d.prefix, h.prefix, head, cudaMemcpyHostToDevice, st);
  gw::QueryView qv = make_view(d, srv->tables.as<unsigned long long>(), n);
  qv.chunk = ctx->ppr_chunk;
  if (e == cudaSuccess)
    e = gw::launch_walk_queries((int)srv->params.rule, qv, 0, acc, ctx->view(), srv->args, d.status,
                                ctx->ppr_threads_per_sm, st);
  // queries whose last walks are in this superstep get their top-k now; a
  // large table is ranked by several CTAs (segmented top-k)
  if (e == cudaSuccess && nfin) {
    const uint32_t seg_slots = gw::topk_segment_slots(nfin);
    std::vector<unsigned long long> sf(nfin + 1);
    gw::topk_segment_prefix(h.tmask, nfin, seg_slots, sf.data());
    if (sf[nfin] == nfin) {
      e = gw::launch_topk(qv, 0, nfin, k, d.ids, d.counts, st);
    } else {
      e = srv->d_topk_segs.ensure((nfin + 1) * 8);
      if (e == cudaSuccess) e = srv->d_topk_cand.ensure(sf[nfin] * k * 8);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(srv->d_topk_segs.p, sf.data(), (nfin + 1) * 8, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess)
        e = gw::launch_topk_segmented(qv, 0, nfin, k, d.ids, d.counts, srv->d_topk_segs.as<unsigned long long>(),
                                      sf.data(), seg_slots, srv->d_topk_cand.as<unsigned long long>(), nullptr, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // sf is read by the copy above
    }
  }
  // status, flags and lists come back in one copy, then one synchronisation
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h.status, d.status, 4 + (size_t)n * 4 + (size_t)n * k * 4 * 2, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    srv->fatal = ctx->cuda_fail(e, "serve superstep");
    return false;
  }
  const gw_status status = gw::status_of(ctx, h.status[0]);
  const uint64_t t = now_ns();
  std::lock_guard<std::mutex> lock(srv->mu);
  srv->stats.supersteps++;
  srv->stats.walks += acc;
  for (uint32_t i = 0; i < n; ++i) {
    Query& q = *cq[i];
    q.issued += take[i];
    if (h.full[i]) {  // restart with a larger table: the same draws, from walk 0
      srv->arena.release(q.table_off, q.table_slots);
      q.factor *= 4;
      q.issued = 0;
      q.restarts++;
      srv->stats.restarts++;
      const uint64_t slots = pow2_at_least(std::max<uint64_t>(256, (uint64_t)q.budget * q.factor));
      srv->active.erase(std::find(srv->active.begin(), srv->active.end(), chosen[i]));
      if (q.restarts > 4 || slots > srv->cfg.table_slots) {
        q.status = GW_E_OVERFLOW;
        q.done = true;
        q.done_ns = t;
        continue;
      }
      uint64_t off;
      if (srv->arena.alloc(slots, &off)) {
        q.table_off = off;
        q.table_slots = slots;
        srv->active.push_back(chosen[i]);
        gw::launch_clear_tables(srv->tables.as<unsigned long long>() + off, slots, st);
      } else {
        srv->pending.push_front(chosen[i]);  // waits at the head of the queue for space
      }
      continue;
    }
    if (q.issued == q.budget) {  // i < nfin: its top-k was computed above
      q.ids.assign(h.ids + (size_t)i * k, h.ids + (size_t)(i + 1) * k);
      q.counts.assign(h.counts + (size_t)i * k, h.counts + (size_t)(i + 1) * k);
      q.status = status;
      q.done = true;
      q.done_ns = t;
      srv->arena.release(q.table_off, q.table_slots);
      srv->active.erase(std::find(srv->active.begin(), srv->active.end(), chosen[i]));
      srv->stats.completed++;
    }
  }
  srv->cv_done.notify_all();
  return true;
}

void serve_loop(gw_server* srv) {
  cudaSetDevice(srv->ctx->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lock(srv->mu);
      for (;;) {
        if (srv->stop && srv->active.empty()) return;
        if (!srv->active.empty()) break;
        if (!srv->pending.empty()) {
          const uint64_t due = srv->queries[srv->pending.front()].arrival_ns;
          const uint64_t t = now_ns();
          if (due <= t) break;
          if (due - t > kSpinNs) {  // sleep until shortly before the arrival
            srv->cv_work.wait_for(lock, std::chrono::nanoseconds(due - t - kSpinNs));
            continue;
          }
          // the last stretch is spun: a timed sleep wakes tens of microseconds late
          srv->next_due.store(due);
          lock.unlock();
          while (now_ns() < srv->next_due.load(std::memory_order_relaxed)) std::this_thread::yield();
          lock.lock();
          continue;
        }
        srv->cv_work.wait(lock);
      }
    }
    if (!superstep(srv)) {
      std::lock_guard<std::mutex> lock(srv->mu);
      for (auto& kv : srv->queries)
        if (!kv.second.done) {
          kv.second.done = true;
          kv.second.status = srv->fatal;
        }
      srv->active.clear();
      srv->pending.clear();
      srv->cv_done.notify_all();
      return;
    }
  }
}

}  // namespace

extern "C" {

gw_status gw_serve_open(gw_ctx* ctx, const gw_walk_params* params, const gw_serve_config* cfg, gw_server** out) {
  if (!ctx || !params || !out) return GW_E_INVALID;
  if (ctx->residency != GW_RESIDENT_HBM) return ctx->fail(GW_E_STATE, "serving needs a resident graph");
  gw_server* srv = new gw_server();
  srv->ctx = ctx;
  srv->params = *params;
  gw_status s = gw::make_walk_args(ctx, params, &srv->args);
  if (s != GW_OK) {
    delete srv;
    return s;
  }
  if (cfg) srv->cfg = *cfg;
  if (!srv->cfg.table_slots) srv->cfg.table_slots = 1ull << 28;
  if (!srv->cfg.max_walks_per_step) srv->cfg.max_walks_per_step = 1u << 22;
  if (!srv->cfg.quantum) srv->cfg.quantum = 1u << 16;
  if (!srv->cfg.k) srv->cfg.k = 100;
  if (srv->cfg.k > gw::kTopkMaxK) {
    delete srv;
    return ctx->fail(GW_E_INVALID, "k must be <= %u", gw::kTopkMaxK);
  }
  cudaError_t e = srv->tables.ensure(srv->cfg.table_slots * 8);
  if (e != cudaSuccess) {
    const unsigned long long slots = srv->cfg.table_slots;
    delete srv;
    return ctx->fail(GW_E_NOMEM, "serve table arena of %llu slots: %s", slots, cudaGetErrorString(e));
  }
  srv->arena.reset(srv->cfg.table_slots);
  srv->thread = std::thread(serve_loop, srv);
  *out = srv;
  return GW_OK;
}

gw_status gw_serve_submit(gw_server* srv, uint32_t source, uint32_t budget, uint32_t stream, uint64_t arrival_ns,
                          uint64_t* ticket) {
  if (!srv || !ticket) return GW_E_INVALID;
  if (source >= srv->ctx->nv) return srv->ctx->fail(GW_E_INVALID, "source %u >= nvertices", source);
  if (budget == 0) return srv->ctx->fail(GW_E_INVALID, "empty budget");
  Query q;
  q.source = source;
  q.budget = budget;
  q.stream = stream;
  q.arrival_ns = arrival_ns ? arrival_ns : now_ns();
  q.factor = srv->params.table_factor ? srv->params.table_factor : 8;
  const uint64_t slots = pow2_at_least(std::max<uint64_t>(256, (uint64_t)budget * q.factor));
  if (slots > srv->cfg.table_slots)
    return srv->ctx->fail(GW_E_NOMEM, "a query of %u walks needs %llu table slots; the arena has %llu", budget,
                          (unsigned long long)slots, (unsigned long long)srv->cfg.table_slots);
  std::lock_guard<std::mutex> lock(srv->mu);
  if (srv->stop || srv->fatal != GW_OK) return srv->ctx->fail(GW_E_STATE, "server is closing");
  const uint64_t t = srv->next_ticket++;
  srv->queries.emplace(t, std::move(q));
  // keep the pending queue ordered by arrival time (submissions may be pre-scheduled)
  auto pos = srv->pending.end();
  while (pos != srv->pending.begin() && srv->queries[*std::prev(pos)].arrival_ns > srv->queries[t].arrival_ns) --pos;
  srv->pending.insert(pos, t);
  srv->stats.submitted++;
  uint64_t due = srv->next_due.load();
  while (srv->queries[t].arrival_ns < due && !srv->next_due.compare_exchange_weak(due, srv->queries[t].arrival_ns)) {
  }
  *ticket = t;
  srv->cv_work.notify_one();
  return GW_OK;
}

gw_status gw_serve_wait(gw_server* srv, uint64_t ticket, int64_t timeout_ms, uint32_t* ids, uint32_t* counts,
                        gw_serve_timing* timing) {
  if (!srv) return GW_E_INVALID;
  std::unique_lock<std::mutex> lock(srv->mu);
  auto it = srv->queries.find(ticket);
  if (it == srv->queries.end()) return srv->ctx->fail(GW_E_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
  auto ready = [&] { return it->second.done; };
  if (timeout_ms < 0) srv->cv_done.wait(lock, ready);
  else if (!srv->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready)) return GW_E_TIMEOUT;
  const Query& q = it->second;
  if (ids && !q.ids.empty()) std::copy(q.ids.begin(), q.ids.end(), ids);
  if (counts && !q.counts.empty()) std::copy(q.counts.begin(), q.counts.end(), counts);
  if (timing) {
    timing->arrival_ns = q.arrival_ns;
    timing->admit_ns = q.admit_ns;
    timing->done_ns = q.done_ns;
    timing->restarts = q.restarts;
  }
  const gw_status s = q.status;
  srv->queries.erase(it);
  if (s == GW_E_OVERFLOW)
    return srv->ctx->fail(s, "query %llu: its visit table still filled up after 4 restarts",
                          (unsigned long long)ticket);
  if (s == GW_E_STATE) return srv->ctx->fail(s, "query %llu was cancelled by gw_serve_close", (unsigned long long)ticket);
  return s;
}

gw_status gw_serve_get_stats(gw_server* srv, gw_serve_stats* out) {
  if (!srv || !out) return GW_E_INVALID;
  std::lock_guard<std::mutex> lock(srv->mu);
  *out = srv->stats;
  out->pending = srv->pending.size();
  out->active = srv->active.size();
  return GW_OK;
}

uint64_t gw_serve_clock_ns(void) { return now_ns(); }

gw_status gw_serve_close(gw_server* srv) {
  if (!srv) return GW_OK;
  {
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->stop = true;
    // queries not yet admitted are cancelled
    for (uint64_t t : srv->pending) {
      srv->queries[t].done = true;
      srv->queries[t].status = GW_E_STATE;
    }
    srv->pending.clear();
  }
  srv->cv_work.notify_all();
  if (srv->thread.joinable()) srv->thread.join();
  srv->cv_done.notify_all();
  srv->tables.release();
  srv->h_stage.release();
  srv->d_stage.release();
  srv->d_topk_segs.release();
  srv->d_topk_cand.release();
  const gw_status s = srv->fatal;
  delete srv;
  return s;
}

}  // extern "C"
