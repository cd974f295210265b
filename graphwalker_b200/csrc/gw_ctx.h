// gw_ctx.h -- the engine context behind the C ABI (one per graph).
#pragma once

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "gw_internal.h"

namespace gw {
// Host-side fault injection (gw_inject_fault): true when the calling
// allocation or read of this kind is the one chosen to fail.
bool fault_now(uint32_t kind);
}  // namespace gw

// A device allocation owned by the context.
struct gw_devbuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    if (gw::fault_now(GW_FAULT_DEVICE_ALLOC)) return cudaErrorMemoryAllocation;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, n ? n : 16);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  // ensure() for a buffer whose need creeps up call after call: a growth
  // takes at least half again the current size, so a run of slowly growing
  // needs reallocates (and synchronises the device in cudaFree) a few times,
  // not once per call.
  cudaError_t grow(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    return ensure(n > bytes + bytes / 2 ? n : bytes + bytes / 2);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// A pinned host allocation owned by the context.
struct gw_hostbuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    if (gw::fault_now(GW_FAULT_PINNED_ALLOC)) return cudaErrorMemoryAllocation;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaHostAlloc(&p, n ? n : 16, cudaHostAllocDefault);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

struct gw_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;       // compute stream
  cudaStream_t copy_stream = nullptr;  // block / walk copies
  cudaStream_t aux_stream = nullptr;   // second compute stream (gw_run_pools alternates chunk kernels)
  uint32_t residency = GW_RESIDENT_HBM;
  uint32_t nmblocks = 2;
  uint64_t mapped_max_walks = GW_MAPPED_AUTO;  // streamed blocks read in place at or below this many walks

  // graph
  uint32_t nv = 0;
  uint64_t ne = 0;
  uint32_t nblocks = 0;
  std::vector<uint32_t> blocks;  // nblocks + 1
  gw_devbuf d_rowptr, d_colidx, d_vrec, d_blocks;
  gw_devbuf d_erec;                     // edge records (empty = not built)
  gw_devbuf d_meet, d_sr_rows;          // SimRank meeting counts, per-query path rows
  uint32_t erec_mode = GW_EDGE_RECORDS_AUTO;
  gw_hostbuf h_rowptr, h_colidx;  // pinned copy (streaming residency)

  // device status word (+ pinned mirror)
  gw_devbuf d_status;
  gw_hostbuf h_status;

  // walk pools on the host side (WalkManager::pwalks analogue before upload)
  std::vector<std::vector<uint64_t>> pool_words;
  std::vector<std::vector<uint32_t>> pool_ids;
  bool pools_have_ids = false;

  // run outputs
  gw_devbuf d_walks, d_words, d_ids, d_counts, d_paths, d_plen, d_closure, d_pool_offsets;
  uint64_t last_nwalks = 0;
  uint32_t last_stride = 0;
  uint32_t last_sink = GW_SINK_NONE;
  bool have_run = false;
  gw_run_stats stats{};

  // blocked engine scratch
  gw_devbuf d_dest, d_tile_hist, d_tile_off, d_totals, d_minhop, d_scan_temp, d_out_ptr,
      d_out_base;
  std::vector<gw_devbuf> pools;   // per-block device pools
  // The older part of each block's pool, moved to host memory when the device
  // pools exceed pool_budget bytes (0 = no limit): pool_host_n[b] records in
  // the pinned arena's chunks pool_chunks[b], in order.  A block's pool is
  // this part followed by the first pool_size - pool_host_n records on the
  // device.
  static constexpr uint64_t kPoolChunk = 65536;  // walk records per arena chunk (1 MiB)
  gw_hostbuf pool_arena;
  std::vector<uint32_t> arena_free;               // chunks not in use
  std::vector<std::vector<uint32_t>> pool_chunks;
  std::vector<uint64_t> pool_host_n;
  uint64_t pool_budget = 0;
  std::vector<uint64_t> pool_size;
  std::vector<uint32_t> minstep;  // per-block min hop (WalkManager::minstep)

  // L2 persisting reservation for the visit counters (0 = none)
  uint64_t l2_persist_bytes = 0;

  // gw_run_pools_submit / gw_run_pools_wait: two runs in flight, each with
  // its own device buffers, status word and events (slot = ticket & 1).
  struct PoolsPipe {
    gw_devbuf walks[2], words[2], ids[2], offsets[2], counts[2], status[2];
    gw_hostbuf h_status;                 // 2 words, pinned
    cudaEvent_t run_done[2] = {};        // the run's walks finished
    cudaEvent_t out_done[2] = {};        // its counts and status are on the host
    cudaEvent_t start[2] = {};           // the run's counters are clear
    cudaStream_t readback = nullptr;     // device-to-host copies of finished runs
    uint64_t next_ticket = 1;
    uint64_t ticket[2] = {0, 0};         // ticket held by the slot (0 = free)
    bool waited[2] = {true, true};
  } pipe;

  // multi-source PPR queries
  gw_devbuf d_q_sources, d_q_prefix, d_q_idbase, d_q_toff, d_q_tmask, d_q_tables, d_q_full, d_q_ids,
      d_q_counts, d_q_visits, d_q_cursor, d_q_segs, d_q_cand;
  int ppr_threads_per_sm = 0;  // autotuned launch shape (0 = full occupancy)
  int walk_ctas_per_sm = 0;    // autotuned resident-walk launch shape (0 = full occupancy)
  uint32_t ppr_chunk = 0;      // autotuned walks per cursor grab (0 = default)
  // Batch tags of d_q_tables: the next tag, and whether every slot is empty
  // or carries a tag below it.
  uint32_t q_tag_next = 0;
  bool q_tags_ok = false;

  std::string err;

  size_t max_window_bytes = 0;  // cudaDevAttrMaxAccessPolicyWindowSize

  // Access policy window over `counts` when an L2 reservation is active
  // (the window covers at most the device's maximum window size).
  bool counts_window(const void* counts, cudaAccessPolicyWindow* w) const {
    if (!l2_persist_bytes || !counts || !max_window_bytes) return false;
    size_t bytes = (size_t)nv * sizeof(uint32_t);
    if (bytes > max_window_bytes) bytes = max_window_bytes;
    w->base_ptr = const_cast<void*>(counts);
    w->num_bytes = bytes;
    w->hitRatio = bytes <= l2_persist_bytes ? 1.0f : (float)l2_persist_bytes / (float)bytes;
    w->hitProp = cudaAccessPropertyPersisting;
    w->missProp = cudaAccessPropertyStreaming;
    return true;
  }

  gw_status fail(gw_status code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return code;
  }
  gw_status cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? GW_E_NOMEM : GW_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
  }
  gw::GraphView view() const {
    gw::GraphView g;
    g.vrec = d_vrec.as<const unsigned long long>();
    g.rowptr = d_rowptr.as<const unsigned long long>();
    g.colidx = d_colidx.as<const uint32_t>();
    g.erec = d_erec.p && d_erec.bytes >= ne * sizeof(ulonglong2) ? d_erec.as<const ulonglong2>() : nullptr;
    g.out_bits = d_vrec.p && d_vrec.bytes >= gw::vrec_bytes(nv) ? reinterpret_cast<const uint32_t*>(g.vrec + nv) : nullptr;
    g.nv = nv;
    return g;
  }
};

namespace gw {
// Records an error of an entry point without a context (gw_last_error(NULL)).
gw_status thread_error(gw_status code, const std::string& msg);
// Grid of a resident walk launch over n walks (the context's tuned shape).
int resident_grid(gw_ctx* ctx, uint64_t n);
// Fills launch constants from the API parameters; validates them.
gw_status make_walk_args(gw_ctx* ctx, const gw_walk_params* p, WalkArgs* a);
// Reads and clears the device status word (synchronises ctx->stream).
gw_status take_status(gw_ctx* ctx, cudaStream_t stream);
// The same in two halves: enqueue the read and clear on a stream, then, after
// the caller has synchronised it, interpret the word.
cudaError_t enqueue_status_read(gw_ctx* ctx, cudaStream_t stream);
gw_status read_status(gw_ctx* ctx);
// The error a status word's bits stand for (GW_OK for none).
gw_status status_of(gw_ctx* ctx, uint32_t bits);
// GraphWalker's block loop on the device (gw_engine.cu).
gw_status run_blocked(gw_ctx* ctx, const gw_walk_params* p);
// Frees the buffers, events and stream of gw_run_pools_submit (gw_pools_async.cu).
void pipe_release(gw_ctx* ctx);
// Chunk boundaries (n_chunks + 1 entries) of a host call over n walk words:
// the walk words cross the host link faster than their walks run, so the
// chunks start small (the first kernel waits only for a short copy) and grow
// by 7/4 each time, which keeps each copy shorter than the kernel it hides
// behind (gw_run_pools, gw_run_pools_submit).
std::vector<uint64_t> chunk_bounds(uint64_t n);
}  // namespace gw

#define GW_CUDA(ctx, expr, what)                    \
  do {                                              \
    cudaError_t _e = (expr);                        \
    if (_e != cudaSuccess) return (ctx)->cuda_fail(_e, what); \
  } while (0)
