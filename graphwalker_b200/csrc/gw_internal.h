// gw_internal.h -- host-side declarations shared by the library's sources.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/graphwalker_b200.h"
#include "gw_device.cuh"

namespace gw {

constexpr int kWalkThreads = 256;

// Device status bits (OR-ed into the context's status word by kernels).
constexpr uint32_t kStBounds = 1u;    // vertex id >= nvertices met
constexpr uint32_t kStOverflow = 2u;  // path stride / table capacity exceeded
constexpr uint32_t kStHops = 4u;      // uncapped walk exceeded max_hops

// L2 hints the walk kernels use when the caller asks for the default: column
// loads are evicted first and the visit counters kept (measured on B200 at
// R-MAT scale 24: 1.10x alone, 1.41x with the counters' persisting window).
constexpr uint32_t kDefaultHints = kHintColumnsEvictFirst | kHintCountsEvictLast;

// ---- walk kernels (gw_walk.cu) ----
// window (may be NULL): an L2 access policy window attached to the launch.
cudaError_t launch_walk_resident(int rule, int sink, bool agg, const gw_walk_rec* walks, uint64_t n,
                                 const GraphView& g, const WalkArgs& a, const SinkView& s,
                                 uint32_t* status, int grid, cudaStream_t stream,
                                 const cudaAccessPolicyWindow* window = nullptr);
// Blocked-mode superstep: advances the n walks of one block while they stay
// inside [a.lo, a.hi); writes them back in place and dest[i] = destination
// block (nblocks when the walk ended).  beg_pos/csr non-null = block slice.
cudaError_t launch_walk_block(int rule, int sink, bool agg, gw_walk_rec* walks, uint64_t n,
                              const GraphView& g, const unsigned long long* beg_pos,
                              const uint32_t* csr, const WalkArgs& a, const SinkView& s,
                              const uint32_t* blocks, uint32_t nblocks, uint32_t* dest,
                              uint32_t* status, cudaStream_t stream);
int walk_resident_grid(int rule, int sink, bool agg, uint64_t n);

// ---- codec kernels (gw_walk.cu) ----
cudaError_t launch_unpack_words(const uint64_t* words, const uint32_t* ids, uint64_t n,
                                uint32_t block_base, gw_walk_rec* out, cudaStream_t stream);
// Words of several pools laid end to end: pool p = [pool_offsets[p], pool_offsets[p+1]).
cudaError_t launch_unpack_pools(const uint64_t* words, const uint32_t* ids, uint64_t first,
                                uint64_t n, const uint64_t* pool_offsets, const uint32_t* blocks,
                                uint32_t nblocks, gw_walk_rec* out, cudaStream_t stream);
cudaError_t launch_pack_words(const gw_walk_rec* walks, uint64_t n, const uint32_t* blocks,
                              uint32_t nblocks, uint64_t* words, uint32_t* wblock,
                              cudaStream_t stream);
// SimRank meeting counts meet[q * L + l] of nq queries: query q compares the
// R x L path rows at element offset rows[2q] of a with rows[2q + 1] of b
// (rows NULL: one query at offset 0 of both) (gw_simrank.cu).
cudaError_t launch_simrank_meet(const uint32_t* a, const uint32_t* b, const unsigned long long* rows, uint32_t nq,
                                uint32_t R, uint32_t L, unsigned long long* meet, cudaStream_t stream);
// Walk records of SimRank's placement: walk k * R + i = replica i of verts[k].
cudaError_t launch_simrank_walks(const uint32_t* verts, uint32_t nverts, uint32_t R, uint32_t L, gw_walk_rec* out,
                                 cudaStream_t stream);
// erec[e] = (packed record of colidx[e], colidx[e]) for e < ne (gw_walk.cu).
cudaError_t launch_build_erec(const uint32_t* colidx, const unsigned long long* vrec, uint64_t ne, uint32_t nv,
                              ulonglong2* erec, cudaStream_t stream);

// ---- graph kernels (gw_graph.cu) ----
// Bytes of the vertex-record buffer: nv packed records, then the out-edge
// bitmap (one bit per vertex, in 32-bit words).
inline size_t vrec_bytes(uint32_t nv) { return (size_t)nv * 8 + (((size_t)nv + 31) / 32) * 4; }
// Fills the packed records and the out-edge bitmap (vrec_bytes(nv) bytes at vrec).
cudaError_t launch_build_vrec(const unsigned long long* rowptr, uint32_t nv,
                              unsigned long long* vrec, cudaStream_t stream);
// rowptr[nv + 1] and colidx[n] of edge keys (source << 32 | target) sorted by
// source (gw_graph.cu).
cudaError_t launch_rowptr_from_sorted(const unsigned long long* keys, uint64_t n, uint32_t nv,
                                      unsigned long long* rowptr, uint32_t* colidx, cudaStream_t stream);
// R-MAT CSR on the device.  On success *rowptr_out / *colidx_out are new
// device allocations (cudaMalloc) and *nedges the kept edge count.
cudaError_t rmat_build_csr(uint32_t scale, uint64_t nedges_raw, uint64_t seed, uint32_t ta,
                           uint32_t tab, uint32_t tabc, unsigned long long** rowptr_out,
                           uint32_t** colidx_out, uint64_t* nedges, cudaStream_t stream);

// ---- partition kernels (gw_partition.cu) ----
struct PartitionPlan {
  uint32_t nbuckets = 0;  // destination blocks + 1 (the "ended" bucket)
  uint32_t ntiles = 0;
  size_t scan_temp_bytes = 0;
};
constexpr int kPartThreads = 256;
constexpr int kPartItems = 8;  // walks per thread per tile
constexpr uint32_t kPartTile = kPartThreads * kPartItems;
PartitionPlan partition_plan(uint64_t n, uint32_t nbuckets);
// Histogram of dest over tiles (tile_hist[bucket * ntiles + tile]) and the
// per-bucket minimum hop (atomicMin into minhop[bucket]).
cudaError_t launch_partition_hist(const gw_walk_rec* walks, const uint32_t* dest, uint64_t n,
                                  const PartitionPlan& plan, uint32_t* tile_hist,
                                  uint32_t* minhop, cudaStream_t stream);
// Exclusive scan of tile_hist (bucket-major) into tile_off, and per-bucket
// totals; with minhop_src, also moves the nbuckets minimum hops to
// minhop_dst and resets minhop_src to 0xffffffff for the next histogram
// (totals and minhop_dst may be mapped pinned host memory, which the host
// reads after a stream synchronisation, with no copy call).
cudaError_t launch_partition_scan(const uint32_t* tile_hist, uint32_t* tile_off, uint32_t* totals,
                                  const PartitionPlan& plan, void* temp, cudaStream_t stream,
                                  uint32_t* minhop_src = nullptr, uint32_t* minhop_dst = nullptr);
// dst_a[i] = src_a[i], dst_b[i] = src_b[i] for i < n, by a kernel: the
// sources may be mapped pinned host memory written by the host before the
// launch.  Unlike an async host-to-device copy this does not queue behind
// large block copies on the copy engine.
cudaError_t launch_fetch_u64_pair(const uint64_t* src_a, uint64_t* dst_a, const uint64_t* src_b,
                                  uint64_t* dst_b, uint32_t n, cudaStream_t stream);
// Stable scatter: walk i with dest d lands at out_ptr[d][out_base[d] + rank],
// rank = position among the walks with dest d in input order.  Bucket
// nbuckets-1 (ended walks) is not written.
cudaError_t launch_partition_scatter(const gw_walk_rec* walks, const uint32_t* dest, uint64_t n,
                                     const PartitionPlan& plan, const uint32_t* tile_off,
                                     gw_walk_rec* const* out_ptr, const uint64_t* out_base,
                                     cudaStream_t stream);

// ---- measurement ----
cudaError_t launch_gather_probe(const uint32_t* buf, uint64_t n_words, uint64_t loads,
                                unsigned long long* sink, cudaStream_t stream);
// `ops` red.add of 1 at pseudo-random counters of counters[0 .. mask].
cudaError_t launch_red_probe(uint32_t* counters, uint32_t mask, uint64_t ops, cudaStream_t stream);

}  // namespace gw
