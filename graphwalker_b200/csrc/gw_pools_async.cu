// gw_pools_async.cu -- gw_run_pools as a two-deep pipeline.
//
// gw_run_pools (one engine run over host walk pools, graphwalker.hpp:272-311
// with the pools of walk.hpp:114-137 given by the caller) copies the walk
// words in, walks them and copies the visit counts back before it returns.
// The count read-back (4 bytes per vertex) can start only after the last walk
// of the run, since any walk may visit any vertex, so back-to-back calls leave
// the walk kernels idle while it crosses the host link.
//
// gw_run_pools_submit queues the same work and returns.  Each of two slots
// (ticket & 1) owns its device words, walk records, counters and status word,
// and a run's read-back goes on a stream of its own, so it overlaps the next
// run's copies in and walks.  A slot is reused only after the host has waited
// for its previous run, so no device-side ordering between the two slots is
// needed beyond the streams the runs share.
#include <algorithm>

#include "gw_ctx.h"

namespace gw {

namespace {

cudaError_t pipe_init(gw_ctx* ctx) {
  auto& P = ctx->pipe;
  if (P.readback) return cudaSuccess;  // created last: everything else exists
  cudaError_t e = P.h_status.ensure(2 * sizeof(uint32_t));
  for (int s = 0; s < 2 && e == cudaSuccess; ++s) {
    if (!P.run_done[s]) e = cudaEventCreateWithFlags(&P.run_done[s], cudaEventDisableTiming);
    if (e == cudaSuccess && !P.out_done[s]) e = cudaEventCreateWithFlags(&P.out_done[s], cudaEventDisableTiming);
    if (e == cudaSuccess && !P.start[s]) e = cudaEventCreateWithFlags(&P.start[s], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&P.readback, cudaStreamNonBlocking);
  return e;
}

}  // namespace

std::vector<uint64_t> chunk_bounds(uint64_t n) {
  std::vector<uint64_t> lo{0};
  for (uint64_t m = 1ull << 17; lo.back() < n; m += m * 3 / 4) lo.push_back(std::min(n, lo.back() + m));
  return lo;
}

void pipe_release(gw_ctx* ctx) {
  auto& P = ctx->pipe;
  if (P.readback) cudaStreamSynchronize(P.readback);
  for (int s = 0; s < 2; ++s) {
    for (gw_devbuf* b : {&P.walks[s], &P.words[s], &P.ids[s], &P.offsets[s], &P.counts[s], &P.status[s]})
      b->release();
    for (cudaEvent_t* ev : {&P.run_done[s], &P.out_done[s], &P.start[s]})
      if (*ev) {
        cudaEventDestroy(*ev);
        *ev = nullptr;
      }
    P.ticket[s] = 0;
    P.waited[s] = true;
  }
  P.h_status.release();
  if (P.readback) cudaStreamDestroy(P.readback);
  P.readback = nullptr;
}

}  // namespace gw

extern "C" gw_status gw_run_pools_submit(gw_ctx* ctx, const gw_walk_params* params, const uint64_t* words,
                                         const uint64_t* pool_offsets, const uint32_t* ids, uint32_t* counts,
                                         uint64_t* ticket) {
  if (!ctx) return gw::thread_error(GW_E_INVALID, "NULL context");
  if (!params || !pool_offsets || !counts || !ticket) return ctx->fail(GW_E_INVALID, "NULL argument");
  if (params->sink != GW_SINK_VERTEX_COUNT && params->sink != GW_SINK_NONE)
    return ctx->fail(GW_E_INVALID, "gw_run_pools_submit returns vertex counts only");
  if (ctx->residency != GW_RESIDENT_HBM) return ctx->fail(GW_E_STATE, "gw_run_pools_submit needs a resident graph");
  gw::WalkArgs a;
  gw_status st = gw::make_walk_args(ctx, params, &a);
  if (st != GW_OK) return st;
  const uint64_t n = pool_offsets[ctx->nblocks];
  if (n && !words) return ctx->fail(GW_E_INVALID, "words is NULL");
  auto& P = ctx->pipe;
  GW_CUDA(ctx, gw::pipe_init(ctx), "pipeline init");
  const uint64_t t = P.next_ticket;
  const int s = (int)(t & 1);
  if (!P.waited[s])
    return ctx->fail(GW_E_STATE, "two runs in flight: wait for ticket %llu first", (unsigned long long)P.ticket[s]);
  // The slot's previous run has been waited on: nothing reads its buffers.
  GW_CUDA(ctx, P.walks[s].ensure(n * sizeof(gw_walk_rec)), "walk alloc");
  GW_CUDA(ctx, P.words[s].ensure(n * 8), "word alloc");
  if (ids) GW_CUDA(ctx, P.ids[s].ensure(n * 4), "id alloc");
  GW_CUDA(ctx, P.offsets[s].ensure((ctx->nblocks + 1) * 8), "offsets alloc");
  GW_CUDA(ctx, P.counts[s].ensure((size_t)ctx->nv * 4), "counts alloc");
  GW_CUDA(ctx, P.status[s].ensure(sizeof(uint32_t)), "status alloc");

  const std::vector<uint64_t> lo = gw::chunk_bounds(n);
  const uint64_t nchunks = lo.size() - 1;
  cudaStream_t cs = ctx->stream, as = ctx->aux_stream, xs = ctx->copy_stream, rs = P.readback;
  uint32_t* d_counts = P.counts[s].as<uint32_t>();
  uint32_t* d_status = P.status[s].as<uint32_t>();
  std::vector<cudaEvent_t> ready(nchunks, nullptr);
  cudaEvent_t aux_done = nullptr;
  cudaError_t e = cudaEventCreateWithFlags(&aux_done, cudaEventDisableTiming);
  for (auto& ev : ready)
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  // counters and status word cleared on the compute stream; the second
  // compute stream starts after them
  if (e == cudaSuccess) e = cudaMemsetAsync(d_counts, 0, (size_t)ctx->nv * 4, cs);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_status, 0, sizeof(uint32_t), cs);
  if (e == cudaSuccess) e = cudaEventRecord(P.start[s], cs);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(as, P.start[s], 0);
  // copies in: the pool offsets, then the words (and ids) chunk by chunk
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(P.offsets[s].p, pool_offsets, (ctx->nblocks + 1) * 8, cudaMemcpyHostToDevice, xs);
  for (uint64_t c = 0; c < nchunks && e == cudaSuccess; ++c) {
    const uint64_t l = lo[c], m = lo[c + 1] - l;
    e = cudaMemcpyAsync(P.words[s].as<uint64_t>() + l, words + l, m * 8, cudaMemcpyHostToDevice, xs);
    if (e == cudaSuccess && ids)
      e = cudaMemcpyAsync(P.ids[s].as<uint32_t>() + l, ids + l, m * 4, cudaMemcpyHostToDevice, xs);
    if (e == cudaSuccess) e = cudaEventRecord(ready[c], xs);
  }
  // walks: chunk kernels alternate between the two compute streams
  gw::SinkView sv{};
  sv.counts = d_counts;
  cudaAccessPolicyWindow win;
  const bool use_win = params->sink == GW_SINK_VERTEX_COUNT && ctx->counts_window(d_counts, &win);
  for (uint64_t c = 0; c < nchunks && e == cudaSuccess; ++c) {
    const uint64_t l = lo[c], m = lo[c + 1] - l;
    const cudaStream_t ks = (c & 1) ? as : cs;
    e = cudaStreamWaitEvent(ks, ready[c], 0);
    if (e == cudaSuccess)
      e = gw::launch_unpack_pools(P.words[s].as<uint64_t>() + l, ids ? P.ids[s].as<uint32_t>() + l : nullptr, l, m,
                                  P.offsets[s].as<uint64_t>(), ctx->d_blocks.as<uint32_t>(), ctx->nblocks,
                                  P.walks[s].as<gw_walk_rec>() + l, ks);
    if (e == cudaSuccess)
      e = gw::launch_walk_resident((int)params->rule, (int)params->sink, params->aggregate != 0,
                                   P.walks[s].as<gw_walk_rec>() + l, m, ctx->view(), a, sv, d_status,
                                   gw::resident_grid(ctx, m), ks, use_win ? &win : nullptr);
  }
  // the run is done once both compute streams are; its counts and status go
  // back on the read-back stream
  if (e == cudaSuccess) e = cudaEventRecord(aux_done, as);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, aux_done, 0);
  if (e == cudaSuccess) e = cudaEventRecord(P.run_done[s], cs);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(rs, P.run_done[s], 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(counts, d_counts, (size_t)ctx->nv * 4, cudaMemcpyDeviceToHost, rs);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(P.h_status.as<uint32_t>() + s, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, rs);
  if (e == cudaSuccess) e = cudaEventRecord(P.out_done[s], rs);
  for (auto ev : ready)
    if (ev) cudaEventDestroy(ev);  // released once the work that uses them is done
  if (aux_done) cudaEventDestroy(aux_done);
  if (e != cudaSuccess) {
    // leave no queued work behind that could touch the slot's buffers later
    for (cudaStream_t q : {xs, cs, as, rs}) cudaStreamSynchronize(q);
    return ctx->cuda_fail(e, "gw_run_pools_submit");
  }
  P.ticket[s] = t;
  P.waited[s] = false;
  P.next_ticket = t + 1;
  *ticket = t;
  return GW_OK;
}

extern "C" gw_status gw_run_pools_wait(gw_ctx* ctx, uint64_t ticket) {
  if (!ctx) return gw::thread_error(GW_E_INVALID, "NULL context");
  auto& P = ctx->pipe;
  const int s = (int)(ticket & 1);
  if (ticket == 0 || P.ticket[s] != ticket || P.waited[s])
    return ctx->fail(GW_E_INVALID, "ticket %llu is not a run in flight", (unsigned long long)ticket);
  const cudaError_t e = cudaEventSynchronize(P.out_done[s]);
  P.waited[s] = true;
  if (e != cudaSuccess) return ctx->cuda_fail(e, "gw_run_pools_wait");
  return gw::status_of(ctx, P.h_status.as<uint32_t>()[s]);
}
