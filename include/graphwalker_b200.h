/*
 * graphwalker_b200.h -- C ABI of the B200 random-walk engine.
 *
 * This is the thin boundary between GraphWalker-style host programs (the
 * drop-in C++ headers under graphwalker_b200/compat, a cgo/JNI/ctypes
 * binding, the Python tests) and the sm_100a kernels.  Plain pointers and
 * sizes only.
 *
 * Ownership: a gw_ctx owns every device buffer it allocates; the caller owns
 * every host buffer it passes, and no pointer is retained past the call that
 * received it.  *_device entry points take device pointers and a CUDA
 * stream (cudaStream_t passed as void*; NULL = the default stream) and are
 * stream-ordered: they return once the work is enqueued.
 * Errors: every call returns a gw_status (0 = GW_OK).  Device-side
 * violations (an out-of-range vertex id, a full sink) are reported through a
 * device status word and surface as GW_E_BOUNDS / GW_E_OVERFLOW from the
 * next synchronising call; kernels never trap.  gw_last_error() gives text.
 * Threading: one context per host thread; calls on one context are not
 * reentrant.
 *
 * Reference interfaces replaced (GraphWalker, paths in its project root):
 *   graphwalker_engine ctor + run()      src/engine/graphwalker.hpp:74-126, 272-311
 *   WalkManager (pools, codec, counts)   src/walks/walk.hpp:17-267
 *   RandomWalk*::updateByWalk            src/walks/randomwalk*.hpp
 *   convert_if_notexists / compute_block src/preprocess/conversions.hpp:300-404
 */
#ifndef GRAPHWALKER_B200_H
#define GRAPHWALKER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gw_status;
typedef struct gw_ctx gw_ctx;

#define GW_OK 0
#define GW_E_INVALID 1  /* bad argument                                  */
#define GW_E_CUDA 2     /* a CUDA runtime call failed                    */
#define GW_E_NOMEM 3    /* device or pinned allocation failed            */
#define GW_E_IO 4       /* graph file missing / short read               */
#define GW_E_BOUNDS 5   /* a kernel met a vertex id >= nvertices         */
#define GW_E_OVERFLOW 6 /* a sink ran out of room (path stride, table)   */
#define GW_E_STATE 7    /* call not valid in the context's state         */
#define GW_E_TIMEOUT 8  /* a bounded device wait gave up                 */

/* Walk update rules: the else-branch of the per-hop continuation test. */
#define GW_RULE_JUMP 0    /* RandomWalkwithJump: jump to rand % N, cap L          */
#define GW_RULE_STOP 1    /* RandomWalkwithStop: terminate, cap L                 */
#define GW_RULE_PROB 2    /* RandomWalkwithProb: terminate, no cap                */
#define GW_RULE_RESTART 3 /* RandomWalkwithRestartwithJoint: back to source,
                             segment ends when hop % L == L-1                     */
#define GW_RULE_PPR 4     /* terminate; a dangling vertex sends the walk back to
                             its source; cap L (single-source PPR workload)       */

/* Visit sinks: what the engine accumulates per visit (the app's updateInfo). */
#define GW_SINK_NONE 0         /* rawrandomwalks                                  */
#define GW_SINK_VERTEX_COUNT 1 /* rwdomination: counts[v] += 1                    */
#define GW_SINK_PATH_RECORD 2  /* simrank: paths[walk][visit] = v                 */
#define GW_SINK_CLOSURE_COUNT 3/* graphlet: visits at hop >= L-1 with v == source */

#define GW_MODE_RESIDENT 0 /* whole graph in HBM: one launch runs every walk out  */
#define GW_MODE_BLOCKED 1  /* GraphWalker's block loop: supersteps over one block  */

/* Random stream of the walks.  The reference draws with glibc rand_r seeded
   per block visit with walkid + dstId + hop + time(NULL)
   (randomwalkwithjump.hpp:37), a stream no run can reproduce.
   GW_RNG_PHILOX, the deterministic mode: the two draws of hop h are words 0
   and 1 of Philox4x32-10(key = seed, counter = (walk id, h, stream, 0)),
   consumed in the reference's order, so results equal the reference engine's
   when its rand_r is routed to the same stream.  GW_RNG_NATIVE: one Philox
   block serves two hops (words 0-1 for hop 2m, words 2-3 for hop 2m+1 of
   counter (walk id, m, stream, "NATV")); still a function of (seed, walk id,
   hop), checked statistically against the FP64 power series.             */
#define GW_RNG_PHILOX 0
#define GW_RNG_NATIVE 1

#define GW_HINT_EXPLICIT 0x80000000u    /* cache_hints: use exactly these bits     */
#define GW_HINT_COLUMNS_EVICT_FIRST 1u  /* column loads leave L2 first              */
#define GW_HINT_COUNTS_EVICT_LAST 2u    /* visit-counter atomics stay in L2         */
#define GW_HINT_RECORDS_EVICT_LAST 4u   /* vertex-record loads stay in L2           */
#define GW_HINT_STREAMS_EVICT_FIRST 8u  /* walk-record and start-record loads of the
                                           resident kernel leave L2 first          */

#define GW_RESIDENT_HBM 0  /* CSR copied to device memory once                   */
#define GW_STREAM_PINNED 1 /* CSR kept in pinned host memory, blocks streamed    */

/* One walk as the kernels hold it in HBM (16 bytes, one 128-bit load). */
typedef struct gw_walk_rec {
  uint32_t cur; /* current vertex (global id)                 */
  uint32_t id;  /* Philox stream key (walk id)                 */
  uint32_t src; /* source: restart target and sink key         */
  uint32_t hop; /* hop counter                                 */
} gw_walk_rec;

typedef struct gw_walk_params {
  uint32_t rule;        /* GW_RULE_*                                          */
  uint32_t sink;        /* GW_SINK_*                                          */
  uint32_t L;           /* length cap / segment length                        */
  uint32_t njump;       /* N of `rand_r % N` (JUMP); 0 = number of vertices   */
  double jump_prob;     /* else-branch probability; the reference's 0.15      */
  uint64_t seed;        /* Philox key                                         */
  uint32_t mode;        /* GW_MODE_*                                          */
  uint32_t path_stride; /* visits recorded per walk (PATH_RECORD)             */
  uint32_t max_hops;    /* hop guard for GW_RULE_PROB; 0 = 65535              */
  float prob;           /* chooseBlock's min-step probability (blocked mode)  */
  uint32_t aggregate;   /* 1 = warp-aggregate counter atomics                 */
  uint32_t max_supersteps; /* blocked mode: stop after this many block
                              executions, leaving the pools as they are (0 = run
                              until no walk is pending)                        */
  uint32_t cache_hints; /* L2 eviction priorities of the walk kernels: 0 = the
                           engine default; otherwise GW_HINT_EXPLICIT | bits  */
  uint32_t table_factor; /* PPR queries: table slots per walk of the budget,
                            rounded up to a power of two (0 = 8)           */
  uint32_t block_lo;     /* blocked mode: only blocks [block_lo, block_hi)
                            execute; walks that move to other blocks stay in
                            their pools for gw_read_pool (one rank of a
                            vertex-partitioned run).  No counterpart in the
                            reference, whose engine runs every block.       */
  uint32_t block_hi;     /* 0 = every block                                 */
  uint32_t rng;          /* GW_RNG_PHILOX (0) or GW_RNG_NATIVE (1)           */
  uint32_t reserved;
} gw_walk_params;

typedef struct gw_run_stats {
  uint64_t walks;          /* walks run                                      */
  uint64_t supersteps;     /* block executions (blocked mode)                */
  uint64_t block_loads;    /* blocks copied host->device (streaming)         */
  uint64_t bytes_h2d;      /* graph bytes copied host->device (streaming)    */
  double ms_total;         /* device time of the last gw_run                 */
  double ms_walk;          /* of which walk kernels                          */
  double ms_partition;     /* of which pool partitioning                     */
  double ms_copy_wait;     /* of which waiting for block copies              */
  uint64_t mapped_supersteps; /* block executions read in place from pinned
                                 host memory (streaming, gw_set_mapped_block_walks) */
  uint64_t mapped_walks;   /* walks those executions advanced                 */
  uint64_t pools_spilled;  /* block pools moved to host memory (pool budget)  */
  uint64_t pools_refilled; /* spilled pools brought back to run their block   */
} gw_run_stats;

/* ---- version / codec (host only, no device needed) -------------------- */
const char *gw_version(void);
/* WalkManager::encode / getSourceId / getCurrentId / getHop (walk.hpp:69-84) */
uint64_t gw_encode(uint32_t source, uint32_t current, uint32_t hop);
uint32_t gw_get_source(uint64_t walk);
uint32_t gw_get_current(uint64_t walk);
uint32_t gw_get_hop(uint64_t walk);
/* Smallest 31-bit draw r that passes `(float)r/RAND_MAX > p`
   (randomwalkwithjump.hpp:45); the kernels compare draw >= threshold. */
uint32_t gw_continue_threshold(double p);
/* RandomWalk::getblock (randomwalk.hpp:74-82): nblocks when v >= blocks[nblocks] */
uint32_t gw_getblock(const uint32_t *blocks, uint32_t nblocks, uint32_t v);
/* compute_block (conversions.hpp:300-364): block boundaries from the row
   pointer; returns nblocks + 1 entries written, 0 if cap is too small.     */
uint32_t gw_compute_blocks(const uint64_t *rowptr, uint32_t nvertices, uint64_t blocksize_kb,
                           uint32_t *blocks, uint32_t cap);
/* RandomWalk::compBlockSize / compNmblocks (randomwalk.hpp:96-114)          */
uint64_t gw_comp_block_size(uint64_t nwalks);
uint32_t gw_comp_nmblocks(uint64_t blocksize_kb, uint64_t mem_budget_kb);

/* ---- graph -------------------------------------------------------------- */
typedef struct gw_graph_desc {
  const char *base_filename; /* reads <base>_GraphWalker/graphinfo/file_0.{beg_pos,csr} */
  uint64_t blocksize_kb;     /* and <base>_GraphWalker/blocksize_<KB>KB.blockrange     */
  uint32_t nmblocks;         /* device block slots when streaming (0 = 2)            */
  uint32_t residency;        /* GW_RESIDENT_HBM or GW_STREAM_PINNED                  */
  int32_t device;            /* CUDA device ordinal                                   */
} gw_graph_desc;

/* graphwalker_engine(base, blocksize_kb, nblocks, nmblocks, m) (graphwalker.hpp:74) */
gw_status gw_open(const gw_graph_desc *desc, gw_ctx **out);
/* Same, from host CSR arrays (copied); blocks[nblocks+1] as in a .blockrange */
gw_status gw_open_csr(const uint64_t *rowptr, const uint32_t *colidx, uint32_t nvertices,
                      const uint32_t *blocks, uint32_t nblocks, uint32_t residency,
                      int32_t device, gw_ctx **out);
/* Seeded R-MAT graph generated on the device (self-loops dropped, duplicates
   kept, ids permuted, rows sorted by (src, dst)); blocks from compute_block
   with blocksize_kb.  a, b, c: quadrant probabilities (d = 1 - a - b - c).  */
gw_status gw_open_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, double a, double b,
                       double c, uint64_t blocksize_kb, int32_t device, gw_ctx **out);
gw_status gw_close(gw_ctx *ctx);
/* Last error text of ctx (or of the calling thread when ctx is NULL). */
const char *gw_last_error(gw_ctx *ctx);
gw_status gw_graph_info(gw_ctx *ctx, uint32_t *nvertices, uint64_t *nedges, uint32_t *nblocks);
gw_status gw_get_blocks(gw_ctx *ctx, uint32_t *blocks, uint32_t cap);
/* Copies the CSR to host buffers (rowptr: nvertices+1, colidx: nedges).     */
gw_status gw_export_csr(gw_ctx *ctx, uint64_t *rowptr, uint32_t *colidx);
/* Moves the CSR between HBM (GW_RESIDENT_HBM) and pinned host memory
   (GW_STREAM_PINNED, blocks streamed into `nmblocks` device slots, the
   reference's in-memory block budget, graphwalker.hpp:84-86).  Streamed, the
   row pointer (8 bytes per vertex) stays in HBM and a slot holds one block's
   column slice.                                                             */
gw_status gw_set_residency(gw_ctx *ctx, uint32_t residency, uint32_t nmblocks);
/* Streamed residency: a block the scheduler chooses that is in no device slot
   and has at most `max_walks` pending walks is not copied into a slot; its
   walks read the block's beg_pos and csr in place from pinned host memory over
   the host link, a few sectors per hop instead of the whole block.  Which
   block runs when is unchanged, and so are walks and counts.  0 copies every
   block, as findSubGraph does (graphwalker.hpp:210-228); GW_MAPPED_AUTO (the
   default) reads a block in place when it has at most one pending walk per
   128 bytes of its column slice.                                            */
#define GW_MAPPED_AUTO 0xFFFFFFFFFFFFFFFFull
gw_status gw_set_mapped_block_walks(gw_ctx *ctx, uint64_t max_walks);
/* Device bytes the blocked engine's walk pools may hold (0, the default: no
   limit).  Past it, after a superstep, whole pools move to host memory, the
   pools with the fewest pending walks first (never the fullest, the likely
   next choice), until the rest hold half the budget, as
   WalkManager::writeWalks2Disk spills pool buffers
   (walk.hpp:103-112); a block whose pool was moved is brought back, older
   walks first, when it is chosen (readWalksfromDisk, walk.hpp:139-157).  Pool
   order, walks and counts are unchanged; the pool of the block being run may
   exceed the budget.  This lets the walk state outgrow the device.          */
gw_status gw_set_pool_budget(gw_ctx *ctx, uint64_t bytes);

/* ---- walk pools (WalkManager) ------------------------------------------- */
gw_status gw_walks_clear(gw_ctx *ctx);
/* WalkManager::moveWalk(walk, block, t, cur) for n walks: words are the
   reference's 64-bit walks whose current field is relative to blocks[block];
   ids (may be NULL) key each walk's Philox stream, default = source field. */
gw_status gw_walks_add(gw_ctx *ctx, uint32_t block, const uint64_t *words, const uint32_t *ids,
                       size_t n);
/* walknum[] per block and walksum (walk.hpp:25-32)                          */
gw_status gw_walks_count(gw_ctx *ctx, uint64_t *per_block, uint64_t *total);

/* ---- run ---------------------------------------------------------------- */
/* graphwalker_engine::run(program, prob): runs every pooled walk to its end. */
gw_status gw_run(gw_ctx *ctx, const gw_walk_params *params);
gw_status gw_read_counts(gw_ctx *ctx, uint32_t *counts, size_t n);
/* paths[walk * path_stride + k], lens[walk] (walks in pool order).          */
gw_status gw_read_paths(gw_ctx *ctx, uint32_t *paths, uint32_t *lens, size_t nwalks);
gw_status gw_read_closure(gw_ctx *ctx, uint64_t *closure);
gw_status gw_read_stats(gw_ctx *ctx, gw_run_stats *stats);
/* The pending walks of one block's device pool after a blocked-mode run
   (WalkManager::getCurrentWalks, walk.hpp:114-137); *n = pool size, at most
   cap records are copied, in pool order.                                    */
gw_status gw_read_pool(gw_ctx *ctx, uint32_t block, gw_walk_rec *out, size_t cap, uint64_t *n);

/* One call from host buffers: the walks of every pool (pool b = words
   [pool_offsets[b], pool_offsets[b+1])) are copied in chunks that overlap
   with the walk kernels, and the visit counts come back in counts[nvertices]
   (VERTEX_COUNT sink; counts is overwritten).  ids may be NULL.            */
gw_status gw_run_pools(gw_ctx *ctx, const gw_walk_params *params, const uint64_t *words,
                       const uint64_t *pool_offsets, const uint32_t *ids, uint32_t *counts);
/* gw_run_pools in two halves, so that back-to-back runs overlap.  submit
   queues one run (the copy of the words in, the walks, the copy of the counts
   out to `counts`) and returns its ticket; wait blocks until that run's counts
   are in `counts` and returns the run's status.  Two runs can be in flight: a
   third submit fails with GW_E_STATE until the older one is waited on.  Each
   run in flight has its own device words, walks, counters and status word,
   so a run's count read-back overlaps the next run's copies and walks.
   words, pool_offsets, ids and counts must stay valid, and counts unread,
   until the wait returns; pinned host memory keeps the copies asynchronous.
   The counts equal gw_run_pools's for the same arguments.                  */
gw_status gw_run_pools_submit(gw_ctx *ctx, const gw_walk_params *params, const uint64_t *words,
                              const uint64_t *pool_offsets, const uint32_t *ids, uint32_t *counts,
                              uint64_t *ticket);
gw_status gw_run_pools_wait(gw_ctx *ctx, uint64_t ticket);

/* ---- multi-source PPR queries (msppr, apps/msppr.cpp:25-145) ------------ */
typedef struct gw_ppr_stats {
  uint64_t walks;        /* walks run                                          */
  uint64_t table_slots;  /* per-query table slots allocated                    */
  uint32_t launches;     /* kernels + clears issued                            */
  uint32_t reserved;
  double ms_clear;       /* device time clearing tables                        */
  double ms_walk;        /* device time of the walk kernels                    */
  double ms_topk;        /* device time of the top-k kernels                   */
  double ms_total;       /* device time of the whole call (first to last op)   */
  uint64_t visits;       /* walk steps (visits) run, re-runs of full tables too */
} gw_ppr_stats;

/* Runs budgets[q] walks from sources[q] for each of nq queries with the
   walk class of params->rule (msppr: GW_RULE_STOP, L = maxwalklength) and
   returns each query's top k visited vertices: topk_ids[q*k + r] by visit
   count, ties broken by the smaller vertex id (0xffffffff / 0 pad a short
   list); k <= 512.  Walk j of the batch (queries in order, budgets laid end
   to end) uses stream id j, so a query's result does not depend on the
   other queries.  batched = 1: all queries in one persistent walk launch and
   one top-k launch (the replacement of msppr's per-source
   DiscreteDistribution); batched = 0: one query at a time (clear, walk,
   top-k per query) -- the plain per-query path.  stats may be NULL.
   On an error return, the rows of queries whose lists are not complete (for
   GW_E_OVERFLOW, those whose tables still filled after the retries) hold an
   empty list (ids 0xffffffff, counts 0); the other rows hold their results. */
gw_status gw_ppr_run(gw_ctx *ctx, const gw_walk_params *params, const uint32_t *sources,
                     const uint32_t *budgets, uint32_t nq, uint32_t k, uint32_t batched,
                     uint32_t *topk_ids, uint32_t *topk_counts, gw_ppr_stats *stats);
/* Exact expected visits per vertex of ONE walk from `source` under
   params->rule / L / jump_prob, in FP64 (out[nvertices]): the truncated
   power series the Monte Carlo counts estimate (count / walks -> out).      */
gw_status gw_expected_visits(gw_ctx *ctx, const gw_walk_params *params, uint32_t source, double *out);
/* Times candidate launch shapes of the batched query kernel on the given
   queries (a sample of the workload) -- threads per SM in {512, 1024, 1536,
   2048} x walks a warp takes per grab of the batch cursor in {64, 128, 256,
   512} -- and keeps the fastest for this context's later gw_ppr_run and
   server launches.  The choice does not change any result.  Outputs may be
   NULL.  (The reference has no tuner; msppr's launch is its OpenMP loop,
   graphwalker.hpp:257-270.)                                                */
gw_status gw_ppr_autotune(gw_ctx *ctx, const gw_walk_params *params, const uint32_t *sources,
                          const uint32_t *budgets, uint32_t nq, uint32_t *threads_per_sm,
                          uint32_t *walks_per_chunk);

/* ---- serving PPR queries (continuous batching) --------------------------
   No counterpart in the reference, which runs one batch of sources per
   process.  A server owns its context's stream while open (make no other
   calls on that context meanwhile).  Its scheduler thread admits arrived
   queries while their visit tables fit in a device arena, and runs
   supersteps that mix walk chunks of every admitted query; queries that
   arrive while a superstep runs join the next one.  Query walk w uses Philox
   counter (w, hop, stream, 0): a query's top-k depends only on (source,
   budget, stream), alone or in any mix.                                     */
typedef struct gw_server gw_server;
#define GW_SERVE_BATCHED 0 /* continuous batching across queries            */
#define GW_SERVE_PLAIN 1   /* one whole query per superstep (per-query path) */
typedef struct gw_serve_config {
  uint64_t table_slots;        /* table arena size in 8-byte slots (0 = 2^28)  */
  uint32_t max_walks_per_step; /* walks per superstep (0 = 2^22)               */
  uint32_t quantum;            /* walks of one query per superstep (0 = 2^16)  */
  uint32_t k;                  /* top-k length (0 = 100, at most 512)          */
  uint32_t mode;               /* GW_SERVE_BATCHED or GW_SERVE_PLAIN           */
  uint32_t reserved[4];
} gw_serve_config;
typedef struct gw_serve_timing {
  uint64_t arrival_ns, admit_ns, done_ns; /* gw_serve_clock_ns() time base    */
  uint32_t restarts;                      /* table-full restarts               */
  uint32_t reserved;
} gw_serve_timing;
typedef struct gw_serve_stats {
  uint64_t submitted, completed, supersteps, walks, restarts, pending, active;
} gw_serve_stats;
gw_status gw_serve_open(gw_ctx *ctx, const gw_walk_params *params, const gw_serve_config *cfg,
                        gw_server **out);
/* Queues one query; arrival_ns = 0 means now, a later gw_serve_clock_ns()
   time schedules it (open-loop load replay).                               */
gw_status gw_serve_submit(gw_server *srv, uint32_t source, uint32_t budget, uint32_t stream,
                          uint64_t arrival_ns, uint64_t *ticket);
/* Waits (timeout_ms < 0: forever) and returns the top-k lists (k entries
   each) and timing of a ticket, then forgets it; GW_E_TIMEOUT if not done. */
gw_status gw_serve_wait(gw_server *srv, uint64_t ticket, int64_t timeout_ms, uint32_t *ids,
                        uint32_t *counts, gw_serve_timing *timing);
gw_status gw_serve_get_stats(gw_server *srv, gw_serve_stats *stats);
uint64_t gw_serve_clock_ns(void);
/* Finishes admitted queries, cancels queued ones (GW_E_STATE), frees all.   */
gw_status gw_serve_close(gw_server *srv);

/* ---- device-pointer entry points (stream-ordered) ----------------------- */
/* Runs n walks resident in HBM over the whole resident graph.  Sink buffers
   by params->sink: d_counts[nvertices] (accumulated, not cleared),
   d_paths[n * path_stride] + d_plen[n], d_closure[1] (accumulated).        */
gw_status gw_walk_device(gw_ctx *ctx, const gw_walk_params *params, const gw_walk_rec *d_walks,
                         uint64_t n, uint32_t *d_counts, uint32_t *d_paths, uint32_t *d_plen,
                         unsigned long long *d_closure, void *stream);
/* Decodes n 64-bit walks of pool `block` into walk records (cur made global,
   id = d_ids[i] or the source field).                                      */
gw_status gw_unpack_words_device(gw_ctx *ctx, uint32_t block, const uint64_t *d_words,
                                 const uint32_t *d_ids, uint64_t n, gw_walk_rec *d_out,
                                 void *stream);
/* Encodes walk records back to 64-bit words relative to their own block.    */
gw_status gw_pack_words_device(gw_ctx *ctx, const gw_walk_rec *d_walks, uint64_t n,
                               uint64_t *d_words, uint32_t *d_blocks, void *stream);
/* Synchronises the stream and returns the device status of earlier kernels. */
gw_status gw_sync(gw_ctx *ctx, void *stream);
/* Times the resident walk kernel on the caller's device walks (counts into a
   scratch array of the context) at each occupancy from a quarter to full CTAs
   per SM, and keeps the fastest for this context's later resident launches
   (gw_run, gw_run_pools, gw_walk_device).  The choice changes no result.
   *ctas_per_sm (may be NULL) receives it.  (The reference has no tuner;
   its update loop is an OpenMP loop, graphwalker.hpp:257-270.)            */
gw_status gw_walk_autotune(gw_ctx *ctx, const gw_walk_params *params, const gw_walk_rec *d_walks, uint64_t n,
                           uint32_t *ctas_per_sm);
/* SimRank's meeting reduction (replaces the O(R^2 L) host loop of
   SimRank::computeResult, apps/simrank.cpp:71-84).  d_paths_a / d_paths_b:
   R walks of L visits each, row-major (walk i = row i), 0xFFFFFFFF = no
   visit.  meet[L] (host) receives, per position l, the number of pairs
   (i, j) whose first common vertex is at position l; the app's estimate is
   sum_l meet[l] * 0.8^l / R^2.  R <= 4194240.  Synchronises the stream.     */
gw_status gw_simrank_meet(gw_ctx *ctx, const uint32_t *d_paths_a, const uint32_t *d_paths_b, uint32_t R,
                          uint32_t L, uint64_t *meet, void *stream);
/* A batch of SimRank queries (a[q], b[q]) on the resident graph, each as the
   SimRank app runs one (apps/simrank.cpp:30-84): R walks from each vertex
   under params->rule = GW_RULE_RESTART (RandomWalkwithRestartwithJoint),
   replica i starting at hop i*L and keyed on its source vertex, recording
   L - 1 visits; then the meeting reduction.  Walks are run once per distinct
   vertex of the batch and shared by its queries (for a[q] == b[q] both sides
   are the same walks; the app, which files a's walks before b's, would see no
   walks from b).  meet (host, nq * L, may be NULL) receives each query's
   first-meeting counts, scores (host, nq) sum_l meet[l] * decay^l / R^2.    */
gw_status gw_simrank_batch(gw_ctx *ctx, const gw_walk_params *params, const uint32_t *a, const uint32_t *b,
                           uint32_t nq, uint32_t R, double decay, uint64_t *meet, double *scores);

/* One superstep of the blocked engine that allocates no memory.  This entry
   point has no counterpart in the reference (whose engine allocates host
   buffers per block); it exists for callers that cannot call cudaMalloc
   while they drive walks: a host framework whose caching allocator already
   holds the device's free memory, or a serving loop that must not stall on
   the device-wide synchronisation an allocation or free can cause.
   The n walks of `block` (d_walks, device records) are advanced while they
   stay inside the block (in place, as gw_run's blocked mode does); visits go
   to d_counts (VERTEX_COUNT sink, accumulated); the walks that left the block
   are written to d_moved grouped by destination block, each group in input
   order, group d starting at d_offsets[d] (nblocks + 1 entries, the last =
   walks moved); d_minhop[d] = lowest hop moved into block d (0xffffffff if
   none).  All scratch comes from one fixed device array of the library
   (about 12 MiB per GPU that loads it, held until exit): at most 1,048,576
   walks and 256 blocks per call, else GW_E_INVALID.  The first call on a
   device (and the first after that device's context was recreated, e.g. by
   cudaDeviceReset) looks up that array's address, so make it before any
   stream capture.  The caller's current device is restored on return.
   Calls share the array: two calls that overlap on the GPU race.          */
gw_status gw_superstep_static(gw_ctx *ctx, const gw_walk_params *params, uint32_t block,
                              gw_walk_rec *d_walks, uint64_t n, uint32_t *d_counts,
                              gw_walk_rec *d_moved, uint32_t *d_offsets, uint32_t *d_minhop,
                              void *stream);

/* ---- L2 controls (per CUDA context; nothing outlasts the process) ------- */
/* cudaLimitMaxL2FetchGranularity for this process's context: the bytes L2
   fetches from DRAM on a miss (32 suits random 4/8-byte gathers).  0 leaves
   the limit unchanged; *previous (may be NULL) receives the old value.     */
gw_status gw_set_l2_fetch_granularity(gw_ctx *ctx, uint32_t bytes, uint32_t *previous);
/* Reserves up to `bytes` of L2 for persisting accesses and marks the visit
   counters of later VERTEX_COUNT walk launches as persisting (an access
   policy window on the launch).  0 releases the reservation.               */
gw_status gw_set_l2_persisting(gw_ctx *ctx, uint64_t bytes);

/* ---- graph preprocessing -------------------------------------------------- */
/* Text edge list -> the reference's preprocessed files, on the device:
   convert_to_csr + compute_block (convert_if_notexists,
   src/preprocess/conversions.hpp:181-404).  Writes, after removing any old
   <path>_GraphWalker/ directory as the reference does:
   graphinfo/file_0.beg_pos, graphinfo/file_0.csr, filesize_1024GB.filerange,
   N.nvertices and, when blocksize_kb > 0, blocksize_<KB>KB.blockrange.
   Lines follow the reference's parser: '#'/'%' comment lines, the first two
   tokens split on tab, comma or space and read by atoi (the low 32 bits of
   strtol), self-loops dropped, duplicates kept.  The reference needs the
   lines grouped by ascending source; here lines are grouped by source with a
   stable sort, which leaves such a file unchanged.  GW_E_INVALID names the
   first line the reference rejects (fewer than two tokens), or a line longer
   than 1023 bytes (which its fgets would split).  The text streams through
   the device in chunks of whole lines; stats may be NULL.                  */
typedef struct gw_convert_stats {
  uint64_t bytes, lines, edges;  /* text bytes, lines read, edges kept       */
  uint32_t nvertices, nblocks;
  uint32_t sorted;               /* 1 when the lines were already grouped    */
  uint32_t reserved0;
  double ms_read, ms_device, ms_write, ms_total;
  uint64_t reserved[4];
} gw_convert_stats;
gw_status gw_convert_edgelist(const char *path, uint64_t blocksize_kb, int32_t device, gw_convert_stats *stats);

/* ---- graph layout -------------------------------------------------------- */
/* Edge records: a second copy of the column array in which each edge also
   carries its target's packed (first-edge offset, out-degree) record, 16 bytes
   per edge.  A resident walk then moves along an edge with one random gather
   instead of two (the record of the vertex it stands on comes with the edge
   that led there).  Walks, counts and top-k lists are the same either way.
   No counterpart in the reference, whose graph is the plain CSR
   (graphwalker.hpp:168-209 loads beg_pos and csr only).
   OFF frees them; ON builds them (GW_E_NOMEM if the device lacks the room);
   AUTO, the default of a resident graph, builds them when they take at most
   half of the free device memory (environment GW_EDGE_RECORDS=0 makes OFF
   the default).  Streamed residency drops them; a return to HBM residency
   applies the mode again.  *built (may be NULL) = 1 when they are in use.   */
#define GW_EDGE_RECORDS_OFF 0u
#define GW_EDGE_RECORDS_ON 1u
#define GW_EDGE_RECORDS_AUTO 2u
gw_status gw_set_edge_records(gw_ctx *ctx, uint32_t mode, uint32_t *built);

/* ---- failure injection (tests) ------------------------------------------ */
/* Makes the `after`-th next host-side operation of one kind fail, once, in
   this process: a device allocation by the engine (GW_E_NOMEM / GW_E_CUDA
   from the call that needed it), a pinned host allocation, or a graph-file
   read (a short read: GW_E_IO).  GW_FAULT_NONE disarms.  Nothing is done to
   the GPU; a failed call leaves its context usable.  No counterpart in the
   reference, whose failures are asserts (logger.hpp:215-217).              */
#define GW_FAULT_NONE 0u
#define GW_FAULT_DEVICE_ALLOC 1u
#define GW_FAULT_PINNED_ALLOC 2u
#define GW_FAULT_FILE_READ 3u
gw_status gw_inject_fault(uint32_t kind, uint32_t after);

/* ---- measurement -------------------------------------------------------- */
/* Random 32-byte-sector gather microbenchmark over d_buf (n_words uint32):
   `loads` dependent-free random 4-byte loads; result in *sectors_per_s.     */
gw_status gw_probe_gather(gw_ctx *ctx, const uint32_t *d_buf, uint64_t n_words, uint64_t loads,
                          int iters, double *bytes_per_s);
/* Visit-counter update microbenchmark: `ops` red.add of 1 (the instruction
   and L2 policy the walk kernels count visits with) at pseudo-random counters
   of d_counters (n_words uint32, rounded down to a power of two, counters
   modified); result in *ops_per_s.                                          */
gw_status gw_probe_red(gw_ctx *ctx, uint32_t *d_counters, uint64_t n_words, uint64_t ops, int iters,
                       double *ops_per_s);

#ifdef __cplusplus
}
#endif
#endif
