// gw_ppr.h -- multi-source PPR kernels (per-query sparse counts + top-k).
#pragma once

#include "gw_internal.h"

namespace gw {

constexpr int kPprThreads = 256;
constexpr int kTopkThreads = 512;
constexpr uint32_t kTopkBuffer = 1024;  // candidate keys per CTA
constexpr uint32_t kTopkMaxK = kTopkBuffer - kTopkThreads;
constexpr uint32_t kTopkUnroll = 8;     // table slots a top-k thread loads at once
constexpr uint32_t kTopkSegment = 16384;  // fewest table slots one top-k CTA ranks (segmented top-k)

// Walks a warp takes from the batch cursor at a time, by default: small
// enough that the walks in flight stay inside a narrow window of the batch
// (and of its queries), large enough that the cursor's atomic is not
// contended (64 and 1024 were both slower at R-MAT scale 26 with 4096
// queries).  gw_ppr_autotune picks it per context with the launch shape.
constexpr uint32_t kWarpChunk = 256;

struct QueryView {
  const uint32_t* sources;                 // nq source vertices
  const unsigned long long* walk_prefix;   // nq + 1: walks of query q = [prefix[q], prefix[q+1])
  const unsigned long long* id_base;       // nq: stream id of query q's first walk (NULL = prefix)
  const unsigned long long* table_off;     // nq: first slot of query q's table
  const uint32_t* table_mask;              // nq: table size - 1 (power of two)
  unsigned long long* tables;              // all tables, slots ((tag | vertex) << 32 | count), ~0 = empty
  uint32_t* full;                          // nq: set to 1 when query q's table filled up
  const uint32_t* stream;                  // nq: Philox stream word of query q (NULL = 0)
  unsigned long long* visits;              // total visits counter (may be NULL)
  unsigned long long* cursor;              // batch positions handed out (zeroed by the launcher)
  uint32_t chunk;                          // walks per cursor grab (0 = kWarpChunk)
  uint32_t nq;
  // Batch tag: the high bits of a slot's vertex word (tag_mask) hold the tag
  // of the batch that wrote it.  A slot whose tag is not this batch's is free,
  // so a new tag frees every table at once without a clear.  tag_mask = 0:
  // untagged, only ~0 is free.
  uint32_t tag;
  uint32_t tag_mask;
};

// Walks [w_begin, w_end) of the batch; threads_per_sm <= 0 = full occupancy.
cudaError_t launch_walk_queries(int rule, const QueryView& qv, unsigned long long w_begin,
                                unsigned long long w_end, const GraphView& g, const WalkArgs& a,
                                uint32_t* status, int threads_per_sm, cudaStream_t stream);
// Sets slots [0, n) of a table area to empty.
cudaError_t launch_clear_tables(unsigned long long* tables, unsigned long long n, cudaStream_t stream);
// Table slots per top-k segment for a set of nq queries: kTopkSegment for a
// few queries (one large table is split over many CTAs), growing with nq so
// that a large batch, which fills the GPU with whole tables, is not split
// into small segments that each pay for their own sorts.
uint32_t topk_segment_slots(uint32_t nq);
// seg_first[q + 1] = seg_first[q] + segments of query q's table (host).
void topk_segment_prefix(const uint32_t* table_mask, uint32_t nq, uint32_t seg_slots, unsigned long long* seg_first);
// Top-k of queries [q_begin, q_begin + q_count) into out[q * k + r], one CTA
// per kTopkSegment slots of table: seg_first (nq + 1, on the device and the
// host) from topk_segment_prefix, seg_cand k keys of scratch per segment.
// d_order (NULL = segment order): the launch order of the segments, from
// topk_segment_order, as offsets from seg_first[q_begin].
cudaError_t launch_topk_segmented(const QueryView& qv, uint32_t q_begin, uint32_t q_count, uint32_t k,
                                  uint32_t* out_ids, uint32_t* out_counts, const unsigned long long* d_seg_first,
                                  const unsigned long long* h_seg_first, uint32_t seg_slots,
                                  unsigned long long* d_seg_cand, const uint32_t* d_order, cudaStream_t stream);
// The segments of all nq queries (seg_first[nq] of them), largest first (host):
// a CTA ranking a large table starts in the first wave instead of after the
// small ones, where it would run alone at the end of the launch.
void topk_segment_order(const uint32_t* table_mask, uint32_t nq, uint32_t seg_slots,
                        const unsigned long long* seg_first, uint32_t* order);
// Top-k of queries [q_begin, q_begin + q_count) into out[q * k + r], one CTA per query.
cudaError_t launch_topk(const QueryView& qv, uint32_t q_begin, uint32_t q_count, uint32_t k, uint32_t* out_ids,
                        uint32_t* out_counts, cudaStream_t stream);

}  // namespace gw
