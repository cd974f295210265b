// gw_ppr.cu -- multi-source personalized PageRank (the msppr app,
// apps/msppr.cpp:25-145): per-query visit counts and top-k lists.
//
// Query q has a source vertex and a budget of walks.  Walk j of the whole
// batch belongs to the query whose prefix range holds j, starts at that
// query's source with hop 0 and uses j as its Philox stream id, so a query's
// walks are the same whether it runs alone or inside any batch.
//
// Visits go to a per-query open-addressing table of 64-bit slots
// (vertex << 32 | count; all-ones = empty) -- the sparse replacement of
// msppr's per-source DiscreteDistribution (discretedistribution.hpp:44-57).
// Lanes of a warp that visit the same (query, vertex) in the same step are
// folded into one table update (every walk of a query visits its source at
// hop 0).
//
// Top-k: one CTA per query scans its table and keeps a candidate buffer of
// keys (count << 32 | ~vertex): whenever the buffer could overflow it is
// sorted and cut to the best k, and the k-th key becomes the admission
// threshold.  The result is the exact top k by count, ties broken by the
// smaller vertex id.
#include "gw_ppr.h"

namespace gw {

namespace {

constexpr unsigned long long kEmptySlot = ~0ull;

__device__ __forceinline__ uint32_t slot_hash(uint32_t v) {  // MurmurHash3 fmix32 (Appleby)
  v ^= v >> 16;
  v *= 0x85ebca6bu;
  v ^= v >> 13;
  v *= 0xc2b2ae35u;
  v ^= v >> 16;
  return v;
}

// Adds n visits of vertex v to a table; false when the table is full.
__device__ __forceinline__ bool table_add(unsigned long long* __restrict__ t, uint32_t mask, uint32_t v,
                                          uint32_t n) {
  uint32_t s = slot_hash(v) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    unsigned long long* e = t + s;
    unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(e);
    if (cur == kEmptySlot) {
      cur = atomicCAS(e, kEmptySlot, ((unsigned long long)v << 32) | n);
      if (cur == kEmptySlot) return true;
    }
    if ((uint32_t)(cur >> 32) == v) {
      atomicAdd(e, (unsigned long long)n);
      return true;
    }
    s = (s + 1) & mask;
  }
  return false;
}

__device__ __forceinline__ uint32_t query_of(const unsigned long long* __restrict__ prefix, uint32_t nq,
                                             unsigned long long j) {
  uint32_t lo = 0, hi = nq - 1;  // last q with prefix[q] <= j
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (__ldg(prefix + mid) <= j) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int RULE>
__global__ void __launch_bounds__(kPprThreads)
    walk_query_kernel(QueryView qv, unsigned long long w_begin, unsigned long long w_end, GraphView g,
                      WalkArgs a, uint32_t* __restrict__ status) {
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long j = w_begin + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= w_end) return;
  const L2Hints hp = make_hints(a.hints);
  uint32_t q = query_of(qv.walk_prefix, qv.nq, j);
  uint32_t src = __ldg(qv.sources + q);
  // stream id = the walk's position in the original batch
  unsigned long long id_shift = qv.id_base ? __ldg(qv.id_base + q) - __ldg(qv.walk_prefix + q) : 0ull;
  uint32_t sid = qv.stream ? __ldg(qv.stream + q) : 0u;
  uint32_t v = src, hop = 0, st = 0, nvisit = 0;
  for (;;) {
    bool end;
    if (rule_capped<RULE>() && hop >= a.L) {
      end = true;
    } else if (RULE == GW_RULE_PROB && hop >= a.max_hops) {
      st |= kStHops;
      end = true;
    } else if (v >= g.nv) {
      st |= kStBounds;
      end = true;
    } else {
      // the record load is issued before the table update so the two overlap
      const unsigned long long rec = ld_nc_u64(g.vrec + v, hp.rec);
      ++nvisit;
      // fold lanes visiting the same (query, vertex) into one update
      const unsigned active = __activemask();
      const unsigned long long key = ((unsigned long long)q << 32) | v;
      const unsigned peers = __match_any_sync(active, key);
      if ((threadIdx.x & 31) == __ffs(peers) - 1) {
        unsigned long long* t = qv.tables + __ldg(qv.table_off + q);
        if (!table_add(t, __ldg(qv.table_mask + q), v, (uint32_t)__popc(peers))) qv.full[q] = 1u;
      }
      end = !hop_advance_rec<RULE>(g, a, hp, (uint32_t)(j + id_shift), src, hop, v, rec, sid);
      if (!end) {
        ++hop;
        if (RULE == GW_RULE_RESTART && hop % a.L == a.L - 1) end = true;
      }
    }
    if (end) {
      j += stride;
      if (j >= w_end) break;
      if (j >= __ldg(qv.walk_prefix + q + 1)) {
        q = query_of(qv.walk_prefix, qv.nq, j);
        src = __ldg(qv.sources + q);
        id_shift = qv.id_base ? __ldg(qv.id_base + q) - __ldg(qv.walk_prefix + q) : 0ull;
        sid = qv.stream ? __ldg(qv.stream + q) : 0u;
      }
      v = src;
      hop = 0;
    }
  }
  if (st) atomicOr(status, st);
  if (qv.visits) {
    const unsigned m = __activemask();
    const unsigned long long w = __reduce_add_sync(m, nvisit);
    if ((threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(qv.visits, w);
  }
}

// Sorts keys[0, n) in shared memory, largest first (bitonic; n a power of two).
__device__ void block_sort_desc(unsigned long long* keys, uint32_t n) {
  for (uint32_t size = 2; size <= n; size <<= 1) {
    for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t partner = i ^ stride;
        if (partner > i) {
          const bool desc = (i & size) == 0;
          const unsigned long long x = keys[i], y = keys[partner];
          if (desc ? x < y : x > y) {
            keys[i] = y;
            keys[partner] = x;
          }
        }
      }
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kTopkThreads)
    topk_kernel(QueryView qv, uint32_t q_begin, uint32_t k, uint32_t* __restrict__ out_ids,
                uint32_t* __restrict__ out_counts) {
  __shared__ unsigned long long cand[kTopkBuffer];
  __shared__ uint32_t ncand;
  __shared__ unsigned long long thresh;
  const uint32_t q = q_begin + blockIdx.x;
  const unsigned long long* t = qv.tables + qv.table_off[q];
  const uint32_t cap = qv.table_mask[q] + 1;
  if (threadIdx.x == 0) {
    ncand = 0;
    thresh = 0;
  }
  __syncthreads();
  for (uint32_t base = 0; base < cap; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    if (i < cap) {
      const unsigned long long e = t[i];
      if (e != kEmptySlot) {
        const unsigned long long key = ((e & 0xffffffffull) << 32) | (uint32_t)~(uint32_t)(e >> 32);
        if (key > thresh) {
          const uint32_t pos = atomicAdd(&ncand, 1u);
          cand[pos] = key;  // room for one full round is kept free below
        }
      }
    }
    __syncthreads();
    if (ncand > kTopkBuffer - blockDim.x) {  // cut to the best k before the next round
      for (uint32_t x = ncand + threadIdx.x; x < kTopkBuffer; x += blockDim.x) cand[x] = 0;
      block_sort_desc(cand, kTopkBuffer);
      if (threadIdx.x == 0) {
        ncand = k;
        thresh = cand[k - 1];
      }
      __syncthreads();
    }
  }
  for (uint32_t x = ncand + threadIdx.x; x < kTopkBuffer; x += blockDim.x) cand[x] = 0;
  block_sort_desc(cand, kTopkBuffer);
  for (uint32_t r = threadIdx.x; r < k; r += blockDim.x) {
    const unsigned long long key = cand[r];
    out_ids[(unsigned long long)q * k + r] = key ? ~(uint32_t)key : 0xffffffffu;
    out_counts[(unsigned long long)q * k + r] = (uint32_t)(key >> 32);
  }
}

template <int RULE>
cudaError_t query_dispatch(const QueryView& qv, unsigned long long w_begin, unsigned long long w_end,
                           const GraphView& g, const WalkArgs& a, uint32_t* status, int threads_per_sm,
                           cudaStream_t stream) {
  auto kern = walk_query_kernel<RULE>;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPprThreads, 0);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (per_sm <= 0) per_sm = 1;
  if (threads_per_sm > 0) per_sm = std::max(1, std::min(per_sm, threads_per_sm / kPprThreads));
  const unsigned long long n = w_end - w_begin;
  const unsigned long long need = (n + kPprThreads - 1) / kPprThreads;
  const unsigned long long full = (unsigned long long)sms * per_sm;
  const int grid = (int)(need < full ? (need ? need : 1) : full);
  kern<<<grid, kPprThreads, 0, stream>>>(qv, w_begin, w_end, g, a, status);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_walk_queries(int rule, const QueryView& qv, unsigned long long w_begin,
                                unsigned long long w_end, const GraphView& g, const WalkArgs& a,
                                uint32_t* status, int threads_per_sm, cudaStream_t stream) {
  if (w_end <= w_begin || qv.nq == 0) return cudaSuccess;
  switch (rule) {
    case GW_RULE_JUMP: return query_dispatch<GW_RULE_JUMP>(qv, w_begin, w_end, g, a, status, threads_per_sm, stream);
    case GW_RULE_STOP: return query_dispatch<GW_RULE_STOP>(qv, w_begin, w_end, g, a, status, threads_per_sm, stream);
    case GW_RULE_PROB: return query_dispatch<GW_RULE_PROB>(qv, w_begin, w_end, g, a, status, threads_per_sm, stream);
    case GW_RULE_RESTART:
      return query_dispatch<GW_RULE_RESTART>(qv, w_begin, w_end, g, a, status, threads_per_sm, stream);
    case GW_RULE_PPR: return query_dispatch<GW_RULE_PPR>(qv, w_begin, w_end, g, a, status, threads_per_sm, stream);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_topk(const QueryView& qv, uint32_t q_begin, uint32_t q_count, uint32_t k, uint32_t* out_ids,
                        uint32_t* out_counts, cudaStream_t stream) {
  if (q_count == 0) return cudaSuccess;
  if (k == 0 || k > kTopkMaxK) return cudaErrorInvalidValue;
  topk_kernel<<<q_count, kTopkThreads, 0, stream>>>(qv, q_begin, k, out_ids, out_counts);
  return cudaGetLastError();
}

}  // namespace gw
