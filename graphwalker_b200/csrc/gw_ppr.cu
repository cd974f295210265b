// gw_ppr.cu -- multi-source personalized PageRank (the msppr app,
// apps/msppr.cpp:25-145): per-query visit counts and top-k lists.
//
// Query q has a source vertex and a budget of walks.  Walk j of the whole
// batch belongs to the query whose prefix range holds j, starts at that
// query's source with hop 0 and uses j as its Philox stream id, so a query's
// walks are the same whether it runs alone or inside any batch.
//
// Visits go to a per-query open-addressing table of 64-bit slots
// ((tag | vertex) << 32 | count; all-ones = empty) -- the sparse replacement
// of msppr's per-source DiscreteDistribution (discretedistribution.hpp:44-57).
// The tag, in the vertex word's bits above the largest vertex id, names the
// batch that wrote the slot: a batch treats the slots of earlier batches as
// free, so its tables need no clearing pass.
// Lanes of a warp that visit the same (query, vertex) in the same step are
// folded into one table update, and the hop-0 visits of a query's walks (all
// at its source) are added in one update.  Warps take walks in small chunks
// of consecutive batch positions from a global cursor, so the walks in flight
// belong to a narrow window of queries whose tables stay in L2.
//
// Top-k: a CTA scans a table (or a segment of one) and keeps a candidate
// buffer of keys (count << 32 | ~vertex): whenever the buffer could overflow
// it is sorted and cut to the best k, and the k-th key becomes the admission
// threshold.  Large tables are split into segments ranked by separate CTAs,
// whose lists a second kernel merges.  The result is the exact top k by
// count, ties broken by the smaller vertex id.
#include "gw_ppr.h"

namespace gw {

namespace {

constexpr unsigned long long kEmptySlot = ~0ull;

// Longest probe sequence an update walks before it reports the table full:
// bounds the cost of a filling table (whose query is then rerun with a larger
// one) instead of letting every further update scan the whole table.
constexpr uint32_t kMaxProbes = 256;

__device__ __forceinline__ uint32_t probe_limit(uint32_t mask) { return mask < kMaxProbes ? mask : kMaxProbes - 1; }

__device__ __forceinline__ uint32_t slot_hash(uint32_t v) {  // MurmurHash3 fmix32 (Appleby)
  v ^= v >> 16;
  v *= 0x85ebca6bu;
  v ^= v >> 13;
  v *= 0xc2b2ae35u;
  v ^= v >> 16;
  return v;
}

// Slot operations.  The add carries an L2 eviction policy (the tables of the
// queries in flight should stay in L2 while the graph streams through it);
// the compare-and-swap form of atom takes none, so a slot's line is first
// touched by a prefetch marked evict_last (prefetch_slot).
__device__ __forceinline__ void prefetch_slot(const unsigned long long* a) {
  asm volatile("prefetch.global.L2::evict_last [%0];" ::"l"(a));
}

__device__ __forceinline__ unsigned long long cas_u64(unsigned long long* a, unsigned long long cmp,
                                                      unsigned long long val) {
  unsigned long long old;
  asm volatile("atom.relaxed.gpu.global.cas.b64 %0, [%1], %2, %3;" : "=l"(old) : "l"(a), "l"(cmp), "l"(val)
               : "memory");
  return old;
}

__device__ __forceinline__ void red_add_u64(unsigned long long* a, unsigned long long v, uint64_t pol) {
  asm volatile("red.relaxed.gpu.global.add.L2::cache_hint.u64 [%0], %1, %2;" ::"l"(a), "l"(v), "l"(pol)
               : "memory");
}

// A slot another batch wrote (or never written): free for this one.
__device__ __forceinline__ bool slot_free(unsigned long long old, uint32_t tag, uint32_t tag_mask) {
  return old == kEmptySlot || ((uint32_t)(old >> 32) & tag_mask) != tag;
}

// Completes a table update of n visits under key = tag | v whose first probe
// (a CAS of the empty pattern at slot s) returned `old`: nothing to do if the
// CAS claimed the slot, an add if the slot holds the key; a slot left by an
// earlier batch is claimed by a second CAS against its content (within a
// batch only current keys are written, so a slot is resolved in at most two
// CAS); otherwise linear probing from s + 1.  False when the table is full
// (no free slot or slot holding the key within kMaxProbes of s).
__device__ __forceinline__ bool table_finish(unsigned long long* __restrict__ t, uint32_t mask, uint32_t s,
                                             unsigned long long old, uint32_t key, uint32_t n, uint64_t pol,
                                             uint32_t tag_mask) {
  const unsigned long long val = ((unsigned long long)key << 32) | n;
  unsigned long long cmp = kEmptySlot;
  const uint32_t last = probe_limit(mask);
  for (uint32_t probe = 0;;) {
    if (old == cmp) return true;
    if ((uint32_t)(old >> 32) == key) {
      red_add_u64(t + s, n, pol);
      return true;
    }
    if (slot_free(old, key & tag_mask, tag_mask)) {
      cmp = old;
      old = cas_u64(t + s, cmp, val);
      continue;
    }
    if (++probe > last) return false;
    s = (s + 1) & mask;
    cmp = kEmptySlot;
    old = cas_u64(t + s, cmp, val);
  }
}

// Adds n visits under key = tag | v to a table; false when the table is full.
__device__ __forceinline__ bool table_add(unsigned long long* __restrict__ t, uint32_t mask, uint32_t key,
                                          uint32_t n, uint64_t pol, uint32_t tag_mask) {
  const uint32_t s = slot_hash(key & ~tag_mask) & mask;
  return table_finish(t, mask, s, cas_u64(t + s, kEmptySlot, ((unsigned long long)key << 32) | n), key, n, pol,
                      tag_mask);
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

template <int RULE, bool ER>
__global__ void __launch_bounds__(kPprThreads)
    walk_query_kernel(QueryView qv, unsigned long long w_begin, unsigned long long w_end, GraphView g,
                      WalkArgs a, uint32_t* __restrict__ status) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t below = (1u << lane) - 1u;  // lanes under this one
  const unsigned long long total = w_end - w_begin;
  const unsigned long long chunk = qv.chunk ? qv.chunk : kWarpChunk;
  const L2Hints hp = make_hints(a.hints);
  // Every walk visits its source at hop 0: the first walk of each query in
  // this launch adds all of them at once and the walks skip that update.
  const bool visits_source =
      !(rule_capped<RULE>() && a.L == 0) && !(RULE == GW_RULE_PROB && a.max_hops == 0);
  unsigned long long c_next = 0, c_end = 0;  // the warp's current chunk of batch positions
  bool drained = false;                      // the cursor has run past the batch (warp-uniform)
  bool busy = false;                         // this lane holds a walk
  unsigned long long j = 0, id_shift = 0, q_lo = 1, q_hi = 0;
  unsigned long long cur_rec = 0, src_rec = 0;  // edge-record mode: records of v and of the source
  uint32_t q = 0, src = 0, sid = 0, v = 0, hop = 0, st = 0, nvisit = 0;
  DrawCache dc;
  dc.reset();
  for (;;) {
    // Idle lanes take the next walks of the warp's chunk, in lane order.
    uint32_t idle = __ballot_sync(~0u, !busy);
    while (idle && !drained) {
      if (c_next >= c_end) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(qv.cursor, chunk);
        base = __shfl_sync(~0u, base, 0);
        if (base >= total) {
          drained = true;
          break;
        }
        c_next = base;
        c_end = base + chunk < total ? base + chunk : total;
      }
      const unsigned long long avail = c_end - c_next;
      if (!busy && __popc(idle & below) < avail) {
        j = w_begin + c_next + __popc(idle & below);
        busy = true;
        if (j < q_lo || j >= q_hi) {
          q = query_of(qv.walk_prefix, qv.nq, j);
          q_lo = __ldg(qv.walk_prefix + q);
          q_hi = __ldg(qv.walk_prefix + q + 1);
          src = __ldg(qv.sources + q);
          // stream id = the walk's position in the original batch
          id_shift = qv.id_base ? __ldg(qv.id_base + q) - q_lo : 0ull;
          sid = qv.stream ? __ldg(qv.stream + q) : 0u;
          if (ER) src_rec = vertex_rec(g, hp, src);
        }
        const unsigned long long lo = q_lo > w_begin ? q_lo : w_begin, hi = q_hi < w_end ? q_hi : w_end;
        if (visits_source && j == lo && src < g.nv &&
            !table_add(qv.tables + __ldg(qv.table_off + q), __ldg(qv.table_mask + q), qv.tag | src,
                       (uint32_t)(hi - lo), hp.cnt, qv.tag_mask))
          qv.full[q] = 1u;
        v = src;
        cur_rec = src_rec;
        hop = 0;
        dc.reset();
      }
      const uint32_t n_idle = __popc(idle);
      c_next += n_idle < avail ? n_idle : avail;
      idle = __ballot_sync(~0u, !busy);
    }
    if (!__any_sync(~0u, busy)) break;
    if (!busy) continue;
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
      // the move after a walk's last visit is never observed: skipped
      const bool last = last_visit<RULE>(a, hop);
      const unsigned long long rec = (ER || last) ? cur_rec : ld_nc_u64(g.vrec + v, hp.rec);
      ++nvisit;
      // Table update for hops >= 1: lanes visiting the same (query, vertex)
      // fold into one; its first probe (a CAS) is issued now and resolved
      // only after this hop's column load is in flight.
      bool leader = false;
      uint32_t n = 0, s0 = 0, mask = 0;
      unsigned long long old = kEmptySlot, *t = nullptr;
      if (hop > 0) {
        const unsigned active = __activemask();
        const unsigned peers = __match_any_sync(active, ((unsigned long long)q << 32) | v);
        leader = lane == (uint32_t)__ffs(peers) - 1;
        if (leader) {
          n = (uint32_t)__popc(peers);
          t = qv.tables + __ldg(qv.table_off + q);
          mask = __ldg(qv.table_mask + q);
          s0 = slot_hash(v) & mask;
          prefetch_slot(t + s0);  // keeps the table's lines in L2 ahead of the graph's (walk phase -34 %)
          old = cas_u64(t + s0, kEmptySlot, ((unsigned long long)(qv.tag | v) << 32) | n);
        }
      }
      // the hop itself: hop_advance_rec's draws and choices, written out so
      // the table update above can complete after the column load is issued
      uint32_t next = v;
      unsigned long long next_rec = 0;
      bool moved = !last;
      if (!last) {
        const Draws dr = hop_draws(a, (uint32_t)(j + id_shift), hop, sid, dc);
        const uint32_t d0 = dr.d0, d1 = dr.d1;
        unsigned long long off = rec >> kDegBits, deg = rec & kDegEscape;
        if (deg == kDegEscape) {
          off = __ldg(g.rowptr + v);
          deg = __ldg(g.rowptr + v + 1) - off;
        }
        if (deg > 0 && d0 >= a.thr) {
          const unsigned long long r =
              deg > 0x7fffffffull ? (unsigned long long)d1 : (unsigned long long)(d1 % (uint32_t)deg);
          if (ER) {
            const ulonglong2 e = ld_nc_u64x2(g.erec + off + r, hp.col);
            next = (uint32_t)e.y;
            next_rec = e.x;
          } else {
            next = ld_nc_u32(g.colidx + off + r, hp.col);
          }
        } else {
          const uint32_t dj = deg > 0 ? d1 : d0;
          if (RULE == GW_RULE_JUMP) {
            next = dj % a.njump;
            if (ER) next_rec = jump_rec(g, hp, next);
          } else if (RULE == GW_RULE_RESTART || (RULE == GW_RULE_PPR && deg == 0)) {
            next = src;
            next_rec = src_rec;
          } else {
            moved = false;
          }
        }
      }
      if (leader && !table_finish(t, mask, s0, old, qv.tag | v, n, hp.cnt, qv.tag_mask)) qv.full[q] = 1u;
      end = !moved;
      if (moved) {
        v = next;
        cur_rec = next_rec;
        ++hop;
        if (RULE == GW_RULE_RESTART && hop % a.L == a.L - 1) end = true;
      }
    }
    if (end) busy = false;
  }
  if (st) atomicOr(status, st);
  if (qv.visits) {
    const unsigned long long w = __reduce_add_sync(~0u, nvisit);
    if (lane == 0 && w) atomicAdd(qv.visits, w);
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

// Cuts cand[0, nc) (distinct nonzero keys, nc > k) to its k largest, in any
// order, at cand[0, *kept), and returns the smallest of them.  The k-th
// largest key is found by an MSB-first radix select on 8-bit digits (a
// histogram of the keys that match the digits chosen so far, one warp picks
// the digit holding rank k), which stops early once the wanted key is the
// smallest of its bucket; one compaction pass then keeps the keys >= it.
// Costs about 3 barriers per digit, where a bitonic sort of the buffer
// takes 55.
__device__ unsigned long long cut_to_k(unsigned long long* cand, uint32_t nc, uint32_t k, uint32_t* kept_out) {
  __shared__ uint32_t hist[256];
  __shared__ uint32_t sel[3];  // chosen digit, rank left inside it, keys in its bucket
  __shared__ unsigned long long kth;
  __shared__ uint32_t kept;
  const uint32_t lane = threadIdx.x & 31;
  unsigned long long prefix = 0, pmask = 0;
  uint32_t need = k;  // rank (1 = largest) of the wanted key among those matching prefix
  bool smallest_of_bucket = false;
  for (int shift = 56; shift >= 0 && !smallest_of_bucket; shift -= 8) {
    for (uint32_t b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < nc; x += blockDim.x) {
      const unsigned long long key = cand[x];
      if ((key & pmask) == prefix) atomicAdd(&hist[(uint32_t)(key >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // lane l holds bins 255 - 8l down to 248 - 8l
      uint32_t sum = 0;
      for (uint32_t i = 0; i < 8; ++i) sum += hist[255 - 8 * lane - i];
      uint32_t incl = sum;  // keys in the bins of lanes 0..l
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(~0u, incl, o);
        if (lane >= (uint32_t)o) incl += y;
      }
      const uint32_t above = incl - sum;
      if (above < need && need <= incl) {
        uint32_t c = above;
        for (uint32_t i = 0; i < 8; ++i) {
          const uint32_t h = hist[255 - 8 * lane - i];
          if (c + h >= need) {
            sel[0] = 255 - 8 * lane - i;
            sel[1] = need - c;
            sel[2] = h;
            break;
          }
          c += h;
        }
      }
    }
    __syncthreads();
    prefix |= (unsigned long long)sel[0] << shift;
    pmask |= 255ull << shift;
    need = sel[1];
    smallest_of_bucket = sel[2] == need;
    __syncthreads();  // sel and hist are rewritten by the next digit
  }
  if (threadIdx.x == 0) {
    kth = smallest_of_bucket ? ~0ull : prefix;
    kept = 0;
  }
  __syncthreads();
  if (smallest_of_bucket) {
    for (uint32_t x = threadIdx.x; x < nc; x += blockDim.x) {
      const unsigned long long key = cand[x];
      if ((key & pmask) == prefix) atomicMin(&kth, key);
    }
    __syncthreads();
  }
  const unsigned long long t = kth;
  unsigned long long mine[kTopkBuffer / kTopkThreads];
#pragma unroll
  for (uint32_t i = 0; i < kTopkBuffer / kTopkThreads; ++i) {
    const uint32_t x = threadIdx.x + i * blockDim.x;
    mine[i] = x < nc ? cand[x] : 0ull;
  }
  __syncthreads();
#pragma unroll
  for (uint32_t i = 0; i < kTopkBuffer / kTopkThreads; ++i)
    if (mine[i] != 0ull && mine[i] >= t) cand[atomicAdd(&kept, 1u)] = mine[i];
  __syncthreads();
  *kept_out = kept;
  return t;
}

// The best k keys of n (key i = src.key(src.fetch(i)); 0 = no key) into
// cand[0, k), largest first.  kTopkUnroll values per thread are fetched
// before any is converted (the loads issue back to back, so a large table is
// read with that many loads in flight per thread), then filtered one step of
// blockDim.x keys at a time into the candidate buffer; whenever the buffer
// could overflow it is cut to the best k (cut_to_k), and the k-th key
// becomes the admission threshold.  Only the final k are sorted.
template <typename Src>
__device__ void block_best(Src src, uint32_t n, uint32_t k, unsigned long long* cand, uint32_t& ncand,
                           unsigned long long& thresh) {
  if (threadIdx.x == 0) {
    ncand = 0;
    thresh = 0;
  }
  __syncthreads();
  // nc: the candidate count, kept in a register by every thread alike.  The
  // shared ncand only hands out positions: a thread that already appends in
  // the next step changes it while slower threads would still be reading it
  // for the cut decision, so that decision must not read it.
  uint32_t nc = 0;
  for (uint32_t base = 0; base < n; base += blockDim.x * kTopkUnroll) {
    unsigned long long raw[kTopkUnroll];
#pragma unroll
    for (uint32_t u = 0; u < kTopkUnroll; ++u) {
      const uint32_t i = base + u * blockDim.x + threadIdx.x;
      raw[u] = i < n ? src.fetch(i) : Src::kNone;
    }
#pragma unroll
    for (uint32_t u = 0; u < kTopkUnroll; ++u) {
      const unsigned long long key = src.key(raw[u]);
      const bool take = key > thresh;
      if (take) cand[atomicAdd(&ncand, 1u)] = key;  // room for one full step is kept free below
      nc += (uint32_t)__syncthreads_count(take);
      if (nc > kTopkBuffer - blockDim.x) {  // cut to the best k before the next step
        uint32_t kept = 0;
        const unsigned long long t = cut_to_k(cand, nc, k, &kept);
        if (threadIdx.x == 0) {
          ncand = kept;
          thresh = t;
        }
        nc = kept;
        __syncthreads();
      }
    }
  }
  if (nc > k) {
    uint32_t kept = 0;
    cut_to_k(cand, nc, k, &kept);
    nc = kept;
  }
  uint32_t m = 1;
  while (m < k) m <<= 1;
  for (uint32_t x = nc + threadIdx.x; x < m; x += blockDim.x) cand[x] = 0;
  block_sort_desc(cand, m);
}

// Key of a table slot: count << 32 | ~vertex (larger = more visits, then the
// smaller vertex id); 0 for a free slot (empty, or another batch's).
struct SlotKey {
  static constexpr unsigned long long kNone = kEmptySlot;
  const unsigned long long* t;
  uint64_t pol;
  uint32_t tag, tag_mask;
  __device__ unsigned long long fetch(uint32_t i) const { return ld_nc_u64(t + i, pol); }
  __device__ unsigned long long key(unsigned long long e) const {
    return slot_free(e, tag, tag_mask) ? 0ull
                                       : ((e & 0xffffffffull) << 32) | (uint32_t)~((uint32_t)(e >> 32) & ~tag_mask);
  }
};

struct CandKey {  // candidate lists hold keys already (0 = none)
  static constexpr unsigned long long kNone = 0ull;
  const unsigned long long* c;
  __device__ unsigned long long fetch(uint32_t i) const { return c[i]; }
  __device__ static unsigned long long key(unsigned long long v) { return v; }
};

__device__ void write_topk(const unsigned long long* cand, uint32_t q, uint32_t k, uint32_t* out_ids,
                           uint32_t* out_counts) {
  for (uint32_t r = threadIdx.x; r < k; r += blockDim.x) {
    const unsigned long long key = cand[r];
    out_ids[(unsigned long long)q * k + r] = key ? ~(uint32_t)key : 0xffffffffu;
    out_counts[(unsigned long long)q * k + r] = (uint32_t)(key >> 32);
  }
}

// One CTA per query over its whole table; CTA i takes query q_begin +
// order[i] (order NULL: i).
__global__ void __launch_bounds__(kTopkThreads, 3)
    topk_kernel(QueryView qv, uint32_t q_begin, uint32_t k, const uint32_t* __restrict__ order,
                uint32_t* __restrict__ out_ids, uint32_t* __restrict__ out_counts) {
  __shared__ unsigned long long cand[kTopkBuffer];
  __shared__ uint32_t ncand;
  __shared__ unsigned long long thresh;
  const uint32_t q = q_begin + (order ? __ldg(order + blockIdx.x) : blockIdx.x);
  block_best(SlotKey{qv.tables + qv.table_off[q], l2_policy(true, false), qv.tag, qv.tag_mask}, qv.table_mask[q] + 1,
             k, cand, ncand, thresh);
  write_topk(cand, q, k, out_ids, out_counts);
}

// One CTA per table segment of seg_slots slots (CTA i takes segment
// seg_first[q_begin] + order[i]; order NULL: i): a query with one segment
// gets its list here; the others leave their segments' best k keys in
// seg_cand for topk_merge_kernel.
__global__ void __launch_bounds__(kTopkThreads, 3)
    topk_segment_kernel(QueryView qv, uint32_t q_begin, uint32_t q_count, uint32_t k, uint32_t seg_slots,
                        const unsigned long long* __restrict__ seg_first, const uint32_t* __restrict__ order,
                        unsigned long long* __restrict__ seg_cand, uint32_t* __restrict__ out_ids,
                        uint32_t* __restrict__ out_counts) {
  __shared__ unsigned long long cand[kTopkBuffer];
  __shared__ uint32_t ncand;
  __shared__ unsigned long long thresh;
  const unsigned long long g = seg_first[q_begin] + (order ? __ldg(order + blockIdx.x) : blockIdx.x);
  uint32_t lo = q_begin, hi = q_begin + q_count - 1;  // the query holding segment g
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (seg_first[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  const uint32_t q = lo;
  const unsigned long long nseg = seg_first[q + 1] - seg_first[q];
  const uint32_t cap = qv.table_mask[q] + 1;
  const uint32_t first = (uint32_t)(g - seg_first[q]) * seg_slots;
  const uint32_t n = cap - first < seg_slots ? cap - first : seg_slots;
  block_best(SlotKey{qv.tables + qv.table_off[q] + first, l2_policy(true, false), qv.tag, qv.tag_mask}, n, k, cand,
             ncand, thresh);
  if (nseg == 1) {
    write_topk(cand, q, k, out_ids, out_counts);
  } else {
    for (uint32_t r = threadIdx.x; r < k; r += blockDim.x) seg_cand[g * k + r] = cand[r];
  }
}

// One CTA per query with several segments: the best k of its segments' lists.
__global__ void __launch_bounds__(kTopkThreads, 3)
    topk_merge_kernel(uint32_t q_begin, uint32_t k, const unsigned long long* __restrict__ seg_first,
                      const unsigned long long* __restrict__ seg_cand, uint32_t* __restrict__ out_ids,
                      uint32_t* __restrict__ out_counts) {
  __shared__ unsigned long long cand[kTopkBuffer];
  __shared__ uint32_t ncand;
  __shared__ unsigned long long thresh;
  const uint32_t q = q_begin + blockIdx.x;
  const unsigned long long s0 = seg_first[q], nseg = seg_first[q + 1] - s0;
  if (nseg < 2) return;
  block_best(CandKey{seg_cand + s0 * k}, (uint32_t)(nseg * k), k, cand, ncand, thresh);
  write_topk(cand, q, k, out_ids, out_counts);
}

__global__ void clear_tables_kernel(ulonglong2* __restrict__ t, unsigned long long n2) {
  const ulonglong2 empty = make_ulonglong2(kEmptySlot, kEmptySlot);
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n2;
       i += (unsigned long long)gridDim.x * blockDim.x)
    t[i] = empty;
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

template <int RULE>
cudaError_t query_dispatch(const QueryView& qv, unsigned long long w_begin, unsigned long long w_end,
                           const GraphView& g, const WalkArgs& a, uint32_t* status, int threads_per_sm,
                           cudaStream_t stream) {
  auto kern = g.erec ? walk_query_kernel<RULE, true> : walk_query_kernel<RULE, false>;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPprThreads, 0);
  const int sms = sm_count();
  if (per_sm <= 0) per_sm = 1;
  if (threads_per_sm > 0) per_sm = std::max(1, std::min(per_sm, threads_per_sm / kPprThreads));
  const unsigned long long n = w_end - w_begin;
  const unsigned long long need = (n + kPprThreads - 1) / kPprThreads;
  const unsigned long long full = (unsigned long long)sms * per_sm;
  const int grid = (int)(need < full ? (need ? need : 1) : full);
  // Walks per cursor grab: no larger than gives every warp of the grid a
  // share, so a launch of few walks (one query, a small serving step) runs
  // them side by side instead of a lane's worth of walks one after another.
  QueryView q = qv;
  const unsigned long long warps = (unsigned long long)grid * (kPprThreads / 32);
  const unsigned long long fair = ((n + warps - 1) / warps + 31) / 32 * 32;
  const unsigned long long chunk = qv.chunk ? qv.chunk : kWarpChunk;
  q.chunk = (uint32_t)(fair < chunk ? fair : chunk);
  kern<<<grid, kPprThreads, 0, stream>>>(q, w_begin, w_end, g, a, status);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_walk_queries(int rule, const QueryView& qv, unsigned long long w_begin,
                                unsigned long long w_end, const GraphView& g, const WalkArgs& a,
                                uint32_t* status, int threads_per_sm, cudaStream_t stream) {
  if (w_end <= w_begin || qv.nq == 0) return cudaSuccess;
  if (!qv.cursor) return cudaErrorInvalidValue;
  const cudaError_t e = cudaMemsetAsync(qv.cursor, 0, sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return e;
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

cudaError_t launch_clear_tables(unsigned long long* tables, unsigned long long n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  if ((reinterpret_cast<uintptr_t>(tables) & 15) || (n & 1))  // not in 16-byte pairs: byte fill
    return cudaMemsetAsync(tables, 0xff, n * sizeof(unsigned long long), stream);
  const unsigned long long n2 = n / 2, need = (n2 + 255) / 256, full = (unsigned long long)sm_count() * 32;
  clear_tables_kernel<<<(unsigned)(need < full ? need : full), 256, 0, stream>>>(
      reinterpret_cast<ulonglong2*>(tables), n2);
  return cudaGetLastError();
}

uint32_t topk_segment_slots(uint32_t nq) {
  uint64_t s = kTopkSegment;
  while (s < (1ull << 30) && s / kTopkSegment * 64 < nq) s <<= 1;  // 64 queries per doubling
  return (uint32_t)s;
}

void topk_segment_prefix(const uint32_t* table_mask, uint32_t nq, uint32_t seg_slots, unsigned long long* seg_first) {
  seg_first[0] = 0;
  for (uint32_t q = 0; q < nq; ++q)
    seg_first[q + 1] = seg_first[q] + ((unsigned long long)table_mask[q] + seg_slots) / seg_slots;
}

void topk_segment_order(const uint32_t* table_mask, uint32_t nq, uint32_t seg_slots,
                        const unsigned long long* seg_first, uint32_t* order) {
  // a table is a power of two, so is a segment: bucket the segments by
  // log2(size), largest bucket first, each bucket in segment order
  std::vector<uint32_t> start(34, 0);
  auto bucket = [&](uint32_t q, unsigned long long i) {
    const unsigned long long cap = (unsigned long long)table_mask[q] + 1, first = i * seg_slots;
    const unsigned long long size = cap - first < seg_slots ? cap - first : seg_slots;
    return 63 - __builtin_clzll(size);  // 0..32
  };
  for (uint32_t q = 0; q < nq; ++q)
    for (unsigned long long i = 0; i < seg_first[q + 1] - seg_first[q]; ++i) ++start[32 - bucket(q, i) + 1];
  for (int b = 1; b < 34; ++b) start[b] += start[b - 1];
  for (uint32_t q = 0; q < nq; ++q)
    for (unsigned long long i = 0; i < seg_first[q + 1] - seg_first[q]; ++i)
      order[start[32 - bucket(q, i)]++] = (uint32_t)(seg_first[q] + i);
}

cudaError_t launch_topk_segmented(const QueryView& qv, uint32_t q_begin, uint32_t q_count, uint32_t k,
                                  uint32_t* out_ids, uint32_t* out_counts, const unsigned long long* d_seg_first,
                                  const unsigned long long* h_seg_first, uint32_t seg_slots,
                                  unsigned long long* d_seg_cand, const uint32_t* d_order, cudaStream_t stream) {
  if (q_count == 0) return cudaSuccess;
  if (k == 0 || k > kTopkMaxK) return cudaErrorInvalidValue;
  const unsigned long long nseg = h_seg_first[q_begin + q_count] - h_seg_first[q_begin];
  if (nseg == 0 || nseg > 0x7fffffffull) return cudaErrorInvalidValue;
  if (nseg == q_count) {  // no table is split: one CTA per query
    topk_kernel<<<q_count, kTopkThreads, 0, stream>>>(qv, q_begin, k, d_order, out_ids, out_counts);
    return cudaGetLastError();
  }
  topk_segment_kernel<<<(unsigned)nseg, kTopkThreads, 0, stream>>>(qv, q_begin, q_count, k, seg_slots, d_seg_first,
                                                                    d_order, d_seg_cand, out_ids, out_counts);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && nseg > q_count) {  // some query has several segments
    topk_merge_kernel<<<q_count, kTopkThreads, 0, stream>>>(q_begin, k, d_seg_first, d_seg_cand, out_ids, out_counts);
    e = cudaGetLastError();
  }
  return e;
}

cudaError_t launch_topk(const QueryView& qv, uint32_t q_begin, uint32_t q_count, uint32_t k, uint32_t* out_ids,
                        uint32_t* out_counts, cudaStream_t stream) {
  if (q_count == 0) return cudaSuccess;
  if (k == 0 || k > kTopkMaxK) return cudaErrorInvalidValue;
  topk_kernel<<<q_count, kTopkThreads, 0, stream>>>(qv, q_begin, k, nullptr, out_ids, out_counts);
  return cudaGetLastError();
}

}  // namespace gw
