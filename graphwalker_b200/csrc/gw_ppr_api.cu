// gw_ppr_api.cu -- C ABI of the multi-source PPR queries (gw_ppr_run,
// gw_ppr_autotune); the kernels are in gw_ppr.cu.
//
// The context's tables are not cleared between batches: each batch writes
// its slots under a new tag (QueryView::tag), which frees the slots of every
// earlier batch at once.  They are cleared when first allocated, when they
// grow, and when the tags run out (2^(32 - vertex id bits) - 1 of them: 63 at
// R-MAT scale 26).  GW_PPR_TAG_BITS caps the tag width (0 = untagged, every
// batch cleared), so that tests reach the wrap-around on small graphs.
//
// Tables are sized for the typical query (table_factor slots per walk of the
// budget).  A query whose table fills up is flagged by the kernel and run
// again, alone with the other flagged queries, with tables four times larger:
// its walks keep their stream ids, so the retried result is exactly the one a
// large enough table would have given.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "gw_ctx.h"
#include "gw_ppr.h"

namespace {

constexpr int kMaxRetries = 3;

uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// A set of queries laid out for one launch.  Its device buffers are the
// context's (kept across calls) for the first round, its own for retries.
struct QuerySet {
  std::vector<uint32_t> sources, qmap;  // qmap: index in the caller's query list
  std::vector<unsigned long long> prefix, id_base, toff;
  std::vector<uint32_t> tmask;
  std::vector<unsigned long long> seg_first;  // top-k segments per query (prefix)
  std::vector<uint32_t> seg_order;            // top-k segments in launch order, largest first
  uint32_t seg_slots = gw::kTopkSegment;
  uint64_t walks = 0, slots = 0;
  bool shared = false;        // the context's buffers (tagged), or this set's own (cleared, untagged)
  bool fresh_tables = false;  // d_tables was (re)allocated by upload_set: its content is undefined
  gw_devbuf own[12];
  gw_devbuf *d_sources, *d_prefix, *d_id_base, *d_toff, *d_tmask, *d_tables, *d_full, *d_ids, *d_cnt, *d_cursor,
      *d_segs, *d_cand;
  gw::QueryView qv{};

  QuerySet(gw_ctx* ctx, bool use_ctx_buffers) {
    gw_devbuf* b[12] = {&ctx->d_q_sources, &ctx->d_q_prefix, &ctx->d_q_idbase, &ctx->d_q_toff,
                        &ctx->d_q_tmask,   &ctx->d_q_tables, &ctx->d_q_full,   &ctx->d_q_ids,
                        &ctx->d_q_counts,  &ctx->d_q_cursor, &ctx->d_q_segs,   &ctx->d_q_cand};
    gw_devbuf** d[12] = {&d_sources, &d_prefix, &d_id_base, &d_toff, &d_tmask, &d_tables,
                         &d_full,    &d_ids,    &d_cnt,     &d_cursor, &d_segs, &d_cand};
    for (int i = 0; i < 12; ++i) *d[i] = use_ctx_buffers ? b[i] : &own[i];
    shared = use_ctx_buffers;
  }
  ~QuerySet() {
    for (auto& b : own) b.release();
  }
};

gw_status plan_set(gw_ctx* ctx, const uint32_t* sources, const uint32_t* budgets, const unsigned long long* ids,
                   const std::vector<uint32_t>& which, uint64_t factor, QuerySet* s) {
  const uint32_t n = (uint32_t)which.size();
  s->qmap = which;
  s->sources.resize(n);
  s->prefix.assign(n + 1, 0);
  s->id_base.resize(n);
  s->toff.resize(n);
  s->tmask.resize(n);
  s->slots = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t q = which[i];
    if (sources[q] >= ctx->nv) return ctx->fail(GW_E_INVALID, "query %u: source %u >= nvertices", q, sources[q]);
    s->sources[i] = sources[q];
    s->prefix[i + 1] = s->prefix[i] + budgets[q];
    s->id_base[i] = ids[q];
    const uint64_t cap = next_pow2(std::max<uint64_t>(256, (uint64_t)budgets[q] * factor));
    if (cap > (1ull << 31)) return ctx->fail(GW_E_OVERFLOW, "query %u: visit table would exceed 2^31 slots", q);
    s->toff[i] = s->slots;
    s->tmask[i] = (uint32_t)(cap - 1);
    s->slots += cap;
  }
  s->walks = s->prefix[n];
  return GW_OK;
}

// batched: the top-k segments grow with the set (64 queries per doubling),
// so one launch ranks the whole set; one query at a time (plain), every table
// splits into kTopkSegment-slot segments, so a large table is ranked by many
// CTAs instead of one.
gw_status upload_set(gw_ctx* ctx, QuerySet* s, uint32_t k, cudaStream_t st, bool batched) {
  const uint32_t n = (uint32_t)s->qmap.size();
  GW_CUDA(ctx, s->d_sources->ensure(n * 4), "query alloc");
  GW_CUDA(ctx, s->d_prefix->ensure((n + 1) * 8), "query alloc");
  GW_CUDA(ctx, s->d_id_base->ensure(n * 8), "query alloc");
  GW_CUDA(ctx, s->d_toff->ensure(n * 8), "query alloc");
  GW_CUDA(ctx, s->d_tmask->ensure(n * 4), "query alloc");
  const void* tables0 = s->d_tables->p;
  const size_t table_bytes0 = s->d_tables->bytes;
  GW_CUDA(ctx, s->d_tables->ensure(s->slots * 8), "query tables alloc");
  s->fresh_tables = s->d_tables->p != tables0 || s->d_tables->bytes != table_bytes0;
  GW_CUDA(ctx, s->d_full->ensure(n * 4), "query alloc");
  GW_CUDA(ctx, s->d_ids->ensure((uint64_t)n * k * 4), "top-k alloc");
  GW_CUDA(ctx, s->d_cnt->ensure((uint64_t)n * k * 4), "top-k alloc");
  GW_CUDA(ctx, s->d_cursor->ensure(sizeof(unsigned long long)), "query alloc");
  s->seg_first.resize(n + 1);
  s->seg_slots = batched ? gw::topk_segment_slots(n) : gw::kTopkSegment;
  gw::topk_segment_prefix(s->tmask.data(), n, s->seg_slots, s->seg_first.data());
  s->seg_order.resize(s->seg_first[n]);
  gw::topk_segment_order(s->tmask.data(), n, s->seg_slots, s->seg_first.data(), s->seg_order.data());
  // d_segs: seg_first (n + 1 u64), then seg_order (u32 per segment)
  GW_CUDA(ctx, s->d_segs->ensure((n + 1) * 8 + s->seg_first[n] * 4), "top-k segments");
  GW_CUDA(ctx, s->d_cand->ensure(s->seg_first[n] * k * 8 + 8), "top-k candidates");
  GW_CUDA(ctx, cudaMemcpyAsync(s->d_segs->p, s->seg_first.data(), (n + 1) * 8, cudaMemcpyHostToDevice, st), "copy");
  GW_CUDA(ctx, cudaMemcpyAsync(s->d_segs->as<unsigned long long>() + n + 1, s->seg_order.data(), s->seg_first[n] * 4,
                               cudaMemcpyHostToDevice, st), "copy");
  GW_CUDA(ctx, cudaMemcpyAsync(s->d_sources->p, s->sources.data(), n * 4, cudaMemcpyHostToDevice, st), "copy");
  GW_CUDA(ctx, cudaMemcpyAsync(s->d_prefix->p, s->prefix.data(), (n + 1) * 8, cudaMemcpyHostToDevice, st), "copy");
  GW_CUDA(ctx, cudaMemcpyAsync(s->d_id_base->p, s->id_base.data(), n * 8, cudaMemcpyHostToDevice, st), "copy");
  GW_CUDA(ctx, cudaMemcpyAsync(s->d_toff->p, s->toff.data(), n * 8, cudaMemcpyHostToDevice, st), "copy");
  GW_CUDA(ctx, cudaMemcpyAsync(s->d_tmask->p, s->tmask.data(), n * 4, cudaMemcpyHostToDevice, st), "copy");
  GW_CUDA(ctx, cudaMemsetAsync(s->d_full->p, 0, n * 4, st), "clear flags");
  s->qv.sources = s->d_sources->as<uint32_t>();
  s->qv.walk_prefix = s->d_prefix->as<unsigned long long>();
  s->qv.id_base = s->d_id_base->as<unsigned long long>();
  s->qv.table_off = s->d_toff->as<unsigned long long>();
  s->qv.table_mask = s->d_tmask->as<uint32_t>();
  s->qv.tables = s->d_tables->as<unsigned long long>();
  s->qv.full = s->d_full->as<uint32_t>();
  s->qv.cursor = s->d_cursor->as<unsigned long long>();
  s->qv.nq = n;
  return GW_OK;
}

// Makes the set's tables free for a new batch: the next tag of the context's
// tables (cleared only when they are fresh or the tags have run out), or a
// clear of the set's own tables.  *cleared: a clear was launched.
cudaError_t assign_tag(gw_ctx* ctx, QuerySet* s, cudaStream_t st, bool* cleared) {
  *cleared = true;
  const uint32_t top = ctx->nv > 1 ? ctx->nv - 1 : 1;
  const uint32_t vbits = 32 - (uint32_t)__builtin_clz(top);  // bits of the largest vertex id
  uint32_t tbits = 32 - vbits;
  if (const char* cap = getenv("GW_PPR_TAG_BITS")) tbits = std::min<uint32_t>(tbits, (uint32_t)atoi(cap));
  const uint32_t ntags = tbits >= 2 ? (1u << tbits) - 1 : 0;  // the all-ones tag is the empty pattern's
  if (!s->shared || ntags == 0) {
    s->qv.tag = s->qv.tag_mask = 0;
    if (s->shared) ctx->q_tags_ok = false;  // untagged slots look like tag 0
    return gw::launch_clear_tables(s->qv.tables, s->slots, st);
  }
  cudaError_t e = cudaSuccess;
  if (s->fresh_tables || !ctx->q_tags_ok || ctx->q_tag_next >= ntags) {
    ctx->q_tags_ok = false;
    e = gw::launch_clear_tables(s->qv.tables, s->d_tables->bytes / 8, st);
    if (e != cudaSuccess) return e;
    ctx->q_tags_ok = true;
    ctx->q_tag_next = 0;
    s->fresh_tables = false;
  } else {
    *cleared = false;
  }
  s->qv.tag_mask = ~0u << vbits;
  s->qv.tag = ctx->q_tag_next++ << vbits;
  return e;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

// Tag (or clear) + walk + top-k of a whole set in two to four launches
// (batched), or clear + walk + top-k query by query (plain).  Timing events:
// ev[0] start, ev[1] tables free, ev[2] walked, ev[3] done.
cudaError_t run_set(gw_ctx* ctx, const gw_walk_params* p, const gw::WalkArgs& a, QuerySet* s, uint32_t k,
                    bool batched, int threads_per_sm, cudaStream_t st, cudaEvent_t* ev, uint32_t* launches) {
  cudaError_t e = cudaSuccess;
  const uint32_t n = s->qv.nq;
  cudaEventRecord(ev[0], st);
  bool cleared = false;
  e = assign_tag(ctx, s, st, &cleared);
  if (batched) {
    cudaEventRecord(ev[1], st);
    if (e == cudaSuccess)
      e = gw::launch_walk_queries((int)p->rule, s->qv, 0, s->walks, ctx->view(), a, ctx->d_status.as<uint32_t>(),
                                  threads_per_sm, st);
    cudaEventRecord(ev[2], st);
    if (e == cudaSuccess)
      e = gw::launch_topk_segmented(s->qv, 0, n, k, s->d_ids->as<uint32_t>(), s->d_cnt->as<uint32_t>(),
                                    s->d_segs->as<unsigned long long>(), s->seg_first.data(), s->seg_slots,
                                    s->d_cand->as<unsigned long long>(),
                                    reinterpret_cast<const uint32_t*>(s->d_segs->as<unsigned long long>() + n + 1), st);
    cudaEventRecord(ev[3], st);
    *launches += (s->seg_first[n] > n ? 3 : 2) + (cleared ? 1 : 0);
  } else {
    cudaEventRecord(ev[1], st);
    *launches += cleared ? 1 : 0;
    for (uint32_t q = 0; q < n && e == cudaSuccess; ++q) {
      e = gw::launch_clear_tables(s->qv.tables + s->toff[q], (uint64_t)s->tmask[q] + 1, st);
      if (e == cudaSuccess)
        e = gw::launch_walk_queries((int)p->rule, s->qv, s->prefix[q], s->prefix[q + 1], ctx->view(), a,
                                    ctx->d_status.as<uint32_t>(), 0, st);
      if (e == cudaSuccess)
        e = gw::launch_topk_segmented(s->qv, q, 1, k, s->d_ids->as<uint32_t>(), s->d_cnt->as<uint32_t>(),
                                      s->d_segs->as<unsigned long long>(), s->seg_first.data(), s->seg_slots,
                                      s->d_cand->as<unsigned long long>(), nullptr, st);
      *launches += s->seg_first[q + 1] - s->seg_first[q] > 1 ? 1 : 0;
    }
    cudaEventRecord(ev[2], st);
    cudaEventRecord(ev[3], st);
    *launches += 3 * n;
  }
  return e;
}

}  // namespace

extern "C" gw_status gw_ppr_run(gw_ctx* ctx, const gw_walk_params* params, const uint32_t* sources,
                                const uint32_t* budgets, uint32_t nq, uint32_t k, uint32_t batched,
                                uint32_t* topk_ids, uint32_t* topk_counts, gw_ppr_stats* stats) {
  if (!ctx) return GW_E_INVALID;
  if (ctx->residency != GW_RESIDENT_HBM) return ctx->fail(GW_E_STATE, "PPR queries need a resident graph");
  if (nq == 0) return GW_OK;
  if (!sources || !budgets || !topk_ids || !topk_counts) return ctx->fail(GW_E_INVALID, "NULL buffer");
  if (k == 0 || k > gw::kTopkMaxK) return ctx->fail(GW_E_INVALID, "k must lie in [1, %u]", gw::kTopkMaxK);
  gw::WalkArgs a;
  gw_status s = gw::make_walk_args(ctx, params, &a);
  if (s != GW_OK) return s;
  // stream id of each query's first walk: budgets laid end to end
  std::vector<unsigned long long> ids(nq);
  unsigned long long total = 0;
  for (uint32_t q = 0; q < nq; ++q) {
    ids[q] = total;
    total += budgets[q];
  }
  std::vector<uint32_t> which(nq);
  for (uint32_t q = 0; q < nq; ++q) which[q] = q;
  uint64_t factor = params->table_factor ? params->table_factor : 8;
  cudaStream_t st = ctx->stream;
  GW_CUDA(ctx, ctx->d_q_visits.ensure(8), "visit counter");
  GW_CUDA(ctx, cudaMemsetAsync(ctx->d_q_visits.p, 0, 8, st), "visit counter");
  cudaEvent_t ev[4];
  for (auto& e : ev) cudaEventCreate(&e);
  gw_ppr_stats local{};
  local.walks = total;
  std::vector<uint32_t> full, hid, hcnt;
  for (int round = 0; round <= kMaxRetries && !which.empty(); ++round) {
    QuerySet set(ctx, round == 0);
    s = plan_set(ctx, sources, budgets, ids.data(), which, factor, &set);
    const bool b = batched || round > 0;
    if (s == GW_OK) s = upload_set(ctx, &set, k, st, b);
    if (s != GW_OK) break;
    set.qv.visits = ctx->d_q_visits.as<unsigned long long>();
    set.qv.chunk = ctx->ppr_chunk;
    cudaError_t e = run_set(ctx, params, a, &set, k, b, b ? ctx->ppr_threads_per_sm : 0, st, ev, &local.launches);
    const uint32_t n = (uint32_t)which.size();
    // The first round holds every query in the caller's order: its lists go
    // straight into the caller's arrays (a rerun query's rows are overwritten
    // later); a rerun's lists go through host staging to their rows.
    const bool direct = round == 0;
    full.resize(n);
    if (!direct) {
      hid.resize((size_t)n * k);
      hcnt.resize((size_t)n * k);
    }
    uint32_t* ids_out = direct ? topk_ids : hid.data();
    uint32_t* cnt_out = direct ? topk_counts : hcnt.data();
    if (e == cudaSuccess) e = cudaMemcpyAsync(full.data(), set.d_full->p, n * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ids_out, set.d_ids->p, (size_t)n * k * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cnt_out, set.d_cnt->p, (size_t)n * k * 4, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) {
      s = ctx->cuda_fail(e, "gw_ppr_run");
      break;
    }
    s = gw::take_status(ctx, st);
    if (s != GW_OK) break;
    if (round == 0 && b) {
      local.ms_clear = elapsed(ev[0], ev[1]);
      local.ms_walk = elapsed(ev[1], ev[2]);
      local.ms_topk = elapsed(ev[2], ev[3]);
    }
    local.ms_total += elapsed(ev[0], ev[3]);
    local.table_slots += set.slots;
    std::vector<uint32_t> again;
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t q = which[i];
      if (full[i]) {
        again.push_back(q);
        continue;
      }
      if (direct) continue;
      std::copy(hid.begin() + (size_t)i * k, hid.begin() + (size_t)(i + 1) * k, topk_ids + (size_t)q * k);
      std::copy(hcnt.begin() + (size_t)i * k, hcnt.begin() + (size_t)(i + 1) * k, topk_counts + (size_t)q * k);
    }
    which.swap(again);
    factor *= 4;
  }
  for (auto& x : ev) cudaEventDestroy(x);
  unsigned long long nvis = 0;
  if (cudaMemcpy(&nvis, ctx->d_q_visits.p, 8, cudaMemcpyDeviceToHost) == cudaSuccess) local.visits = nvis;
  if (s == GW_OK && !which.empty())
    s = ctx->fail(GW_E_OVERFLOW, "%zu queries still filled their visit tables after %d retries",
                  which.size(), kMaxRetries);
  if (s != GW_OK) {
    // The queries without a complete list (still in `which`) get empty rows
    // (ids all-ones, counts 0), so a partial round-0 list is never mistaken
    // for a result.  Copies into those rows may still be queued: wait first.
    cudaStreamSynchronize(st);
    for (const uint32_t q : which) {
      std::fill(topk_ids + (size_t)q * k, topk_ids + (size_t)(q + 1) * k, 0xffffffffu);
      std::fill(topk_counts + (size_t)q * k, topk_counts + (size_t)(q + 1) * k, 0u);
    }
  }
  if (stats) *stats = local;
  return s;
}

extern "C" gw_status gw_ppr_autotune(gw_ctx* ctx, const gw_walk_params* params, const uint32_t* sources,
                                     const uint32_t* budgets, uint32_t nq, uint32_t* threads_per_sm,
                                     uint32_t* walks_per_chunk) {
  if (!ctx) return GW_E_INVALID;
  if (nq == 0 || !sources || !budgets) return ctx->fail(GW_E_INVALID, "empty sample");
  gw::WalkArgs a;
  gw_status s = gw::make_walk_args(ctx, params, &a);
  if (s != GW_OK) return s;
  std::vector<unsigned long long> ids(nq);
  unsigned long long total = 0;
  for (uint32_t q = 0; q < nq; ++q) {
    ids[q] = total;
    total += budgets[q];
  }
  std::vector<uint32_t> which(nq);
  for (uint32_t q = 0; q < nq; ++q) which[q] = q;
  QuerySet set(ctx, true);
  s = plan_set(ctx, sources, budgets, ids.data(), which, params->table_factor ? params->table_factor : 8, &set);
  if (s == GW_OK) s = upload_set(ctx, &set, 1, ctx->stream, true);
  if (s != GW_OK) return s;
  cudaStream_t st = ctx->stream;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // launch shape (threads per SM) x walks per cursor grab
  const int thread_candidates[] = {512, 1024, 1536, 2048};
  const uint32_t chunk_candidates[] = {64, 128, 256, 512};
  int best = 0;
  uint32_t best_chunk = gw::kWarpChunk;
  float best_ms = 1e30f;
  for (int c : thread_candidates) {
    for (uint32_t ch : chunk_candidates) {
      set.qv.chunk = ch;
      float ms_sum = 0.f;
      for (int rep = 0; rep < 3; ++rep) {
        bool cleared = false;
        if (assign_tag(ctx, &set, st, &cleared) != cudaSuccess) break;
        cudaEventRecord(e0, st);
        gw::launch_walk_queries((int)params->rule, set.qv, 0, set.walks, ctx->view(), a,
                                ctx->d_status.as<uint32_t>(), c, st);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        if (rep) ms_sum += elapsed(e0, e1);  // the first run warms up
      }
      if (ms_sum < best_ms) {
        best_ms = ms_sum;
        best = c;
        best_chunk = ch;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s = gw::take_status(ctx, st);
  if (s != GW_OK) return s;
  ctx->ppr_threads_per_sm = best;
  ctx->ppr_chunk = best_chunk;
  if (threads_per_sm) *threads_per_sm = (uint32_t)best;
  if (walks_per_chunk) *walks_per_chunk = best_chunk;
  return GW_OK;
}
