// gw_walk.cu -- the walk-advance kernels (the per-block update loop of
// GraphWalker, src/engine/graphwalker.hpp:257-270 + the updateByWalk of each
// walk class, src/walks/randomwalk*.hpp) and the 64-bit walk codec kernels
// (src/walks/walk.hpp:69-91).
//
// Resident mode: one persistent launch runs every walk to its end.  Each
// thread holds one walk and advances it one hop per loop iteration; when its
// walk ends it takes the next one (index += grid stride) inside the same
// iteration, so lanes never wait for the longest walk of their warp.  Per hop:
// one 8-byte packed vertex record load, one 4-byte column load, one Philox
// block computed while the record load is in flight, and one visit atomic.
// With edge records (ER) the record of the current vertex is carried from the
// previous hop, so a hop along an edge is a single 16-byte gather.
#include "gw_internal.h"

namespace gw {

namespace {

__device__ __forceinline__ uint4 load_walk(const gw_walk_rec* __restrict__ walks, uint64_t i) {
  return __ldg(reinterpret_cast<const uint4*>(walks) + i);
}

// The walk record of the resident kernel, read once: with
// kHintStreamsEvictFirst it is marked to leave L2 first.
__device__ __forceinline__ uint4 load_walk_hinted(const gw_walk_rec* __restrict__ walks, uint64_t i,
                                                  const WalkArgs& a, const L2Hints& hp) {
  return (a.hints & kHintStreamsEvictFirst) ? ld_nc_u32x4(reinterpret_cast<const uint4*>(walks) + i, hp.strm)
                                            : load_walk(walks, i);
}

// A walk's start record: like vertex_rec, with the stream policy when asked.
__device__ __forceinline__ unsigned long long start_rec(const GraphView& g, const WalkArgs& a, const L2Hints& hp,
                                                        uint32_t v) {
  if (v >= g.nv) return 0ull;
  return ld_nc_u64(g.vrec + v, (a.hints & kHintStreamsEvictFirst) ? hp.strm : hp.rec);
}

template <int RULE, int SINK, bool AGG, bool ER>
__global__ void __launch_bounds__(kWalkThreads)
    walk_resident_kernel(const gw_walk_rec* __restrict__ walks, uint64_t n, GraphView g,
                         WalkArgs a, SinkView s, uint32_t* __restrict__ status) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const L2Hints hp = make_hints(a.hints);
  uint4 w = load_walk_hinted(walks, i, a, hp);
  uint32_t v = w.x, id = w.y, src = w.z, hop = w.w, k = 0;
  uint32_t st = 0;
  uint32_t clos = 0;
  DrawCache dc;
  dc.reset();
  // edge-record mode: the records of the current vertex and of the source
  unsigned long long rec = 0, src_rec = 0;
  if (ER) {
    rec = start_rec(g, a, hp, v);
    if (rule_returns<RULE>()) src_rec = src == v ? rec : vertex_rec(g, hp, src);
  }
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
      // the app's updateInfo(src, v, tid, hop) precedes the draws
      if (SINK == GW_SINK_VERTEX_COUNT) {
        count_visit<AGG>(s.counts, v, hp.cnt);
      } else if (SINK == GW_SINK_PATH_RECORD) {
        if (k < a.path_stride) s.paths[i * a.path_stride + k] = v;
        else st |= kStOverflow;
      } else if (SINK == GW_SINK_CLOSURE_COUNT) {
        clos += ((int)hop >= (int)a.L - 1 && v == src) ? 1u : 0u;
      }
      ++k;
      if (last_visit<RULE>(a, hop)) {
        end = true;  // the move after the last visit is never observed
      } else {
        end = ER ? !hop_advance_carried<RULE>(g, a, hp, id, src, src_rec, hop, v, rec, dc)
                 : !hop_advance<RULE>(g, a, hp, id, src, hop, v, dc);
        if (!end) {
          ++hop;
          if (RULE == GW_RULE_RESTART && hop % a.L == a.L - 1) end = true;
        }
      }
    }
    if (end) {
      if (SINK == GW_SINK_PATH_RECORD) s.plen[i] = k;
      i += stride;
      if (i >= n) break;
      w = load_walk_hinted(walks, i, a, hp);
      v = w.x;
      id = w.y;
      src = w.z;
      hop = w.w;
      k = 0;
      dc.reset();
      if (ER) {
        rec = start_rec(g, a, hp, v);
        if (rule_returns<RULE>()) src_rec = src == v ? rec : vertex_rec(g, hp, src);
      }
    }
  }
  if (st) atomicOr(status, st);
  if (SINK == GW_SINK_CLOSURE_COUNT && clos) atomicAdd(s.closure, (unsigned long long)clos);
}

// Edge records: erec[e] = (packed record of colidx[e], colidx[e]).
__global__ void build_erec_kernel(const uint32_t* __restrict__ colidx, const unsigned long long* __restrict__ vrec,
                                  uint64_t ne, uint32_t nv, ulonglong2* __restrict__ erec) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ne;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t w = __ldg(colidx + e);
    erec[e] = make_ulonglong2(w < nv ? __ldg(vrec + w) : 0ull, (unsigned long long)w);
  }
}

__device__ __forceinline__ uint32_t find_block(const uint32_t* __restrict__ blocks,
                                               uint32_t nblocks, uint32_t v) {
  // first p with v < blocks[p+1] (RandomWalk::getblock, randomwalk.hpp:74-82)
  uint32_t lo = 0, hi = nblocks;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (v < __ldg(blocks + mid + 1)) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// Blocked-mode superstep over the walks of block [a.lo, a.hi): the in-block
// loop of updateByWalk and, on leaving, getblock + moveWalk
// (randomwalkwithjump.hpp:40-60 and siblings).
template <int RULE, int SINK, bool AGG, bool SLICE>
__global__ void __launch_bounds__(kWalkThreads)
    walk_block_kernel(gw_walk_rec* __restrict__ walks, uint64_t n, GraphView g,
                      const unsigned long long* __restrict__ beg_pos,
                      const uint32_t* __restrict__ csr, WalkArgs a, SinkView s,
                      const uint32_t* __restrict__ blocks, uint32_t nblocks,
                      uint32_t* __restrict__ dest, uint32_t* __restrict__ status) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint32_t st = 0, clos = 0;
  const L2Hints hp = make_hints(a.hints);
  DrawCache dc;
  // the slice's first edge index (csr[0] is edge b0); read once, since the
  // slice may be pinned host memory read over the host link
  const unsigned long long b0 = SLICE && n ? __ldg(beg_pos) : 0ull;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint4 w = *(reinterpret_cast<const uint4*>(walks) + i);
    uint32_t v = w.x, id = w.y, src = w.z, hop = w.w;
    bool ended = false;
    dc.reset();
    while (v >= a.lo && v < a.hi) {
      if (rule_capped<RULE>() && hop >= a.L) break;
      if (RULE == GW_RULE_PROB && hop >= a.max_hops) {
        st |= kStHops;
        ended = true;
        break;
      }
      if (v >= g.nv) {
        st |= kStBounds;
        ended = true;
        break;
      }
      if (SINK == GW_SINK_VERTEX_COUNT) count_visit<AGG>(s.counts, v, hp.cnt);
      else if (SINK == GW_SINK_CLOSURE_COUNT)
        clos += ((int)hop >= (int)a.L - 1 && v == src) ? 1u : 0u;
      if (last_visit<RULE>(a, hop)) {  // its move is never observed: the walk ends here
        ++hop;
        ended = true;
        break;
      }
      bool moved;
      if (SLICE) moved = hop_advance_slice<RULE>(beg_pos, csr, b0, a, id, src, hop, v, dc);
      else moved = hop_advance<RULE>(g, a, hp, id, src, hop, v, dc);
      if (!moved) {
        ended = true;
        break;
      }
      ++hop;
      if (RULE == GW_RULE_RESTART && hop % a.L == a.L - 1) {
        ended = true;
        break;
      }
    }
    uint32_t d = nblocks;
    if (!ended) {
      bool alive;
      if (rule_capped<RULE>()) alive = hop < a.L;
      else if (RULE == GW_RULE_RESTART) alive = hop % a.L != a.L - 1;
      else alive = true;
      if (alive) d = find_block(blocks, nblocks, v);  // nblocks = dropped (v >= N)
    }
    w.x = v;
    w.w = hop;
    *(reinterpret_cast<uint4*>(walks) + i) = w;
    dest[i] = d;
  }
  if (st) atomicOr(status, st);
  if (SINK == GW_SINK_CLOSURE_COUNT && clos) atomicAdd(s.closure, (unsigned long long)clos);
}

__global__ void unpack_words_kernel(const uint64_t* __restrict__ words,
                                    const uint32_t* __restrict__ ids, uint64_t n,
                                    uint32_t block_base, gw_walk_rec* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t wd = words[i];
    const uint32_t src = (uint32_t)(wd >> 40) & 0xffffffu;
    uint4 r;
    r.x = block_base + ((uint32_t)(wd >> 14) & 0x3ffffffu);
    r.y = ids ? ids[i] : src;
    r.z = src;
    r.w = (uint32_t)(wd & 0x3fffu);
    *(reinterpret_cast<uint4*>(out) + i) = r;
  }
}

__global__ void unpack_pools_kernel(const uint64_t* __restrict__ words,
                                    const uint32_t* __restrict__ ids, uint64_t first, uint64_t n,
                                    const uint64_t* __restrict__ pool_offsets,
                                    const uint32_t* __restrict__ blocks, uint32_t nblocks,
                                    gw_walk_rec* __restrict__ out) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = first + j;
    // pool of walk i: last p with pool_offsets[p] <= i
    uint32_t lo = 0, hi = nblocks;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (__ldg(pool_offsets + mid) <= i) lo = mid;
      else hi = mid - 1;
    }
    const uint64_t wd = words[j];
    const uint32_t src = (uint32_t)(wd >> 40) & 0xffffffu;
    uint4 r;
    r.x = __ldg(blocks + lo) + ((uint32_t)(wd >> 14) & 0x3ffffffu);
    r.y = ids ? ids[j] : src;
    r.z = src;
    r.w = (uint32_t)(wd & 0x3fffu);
    *(reinterpret_cast<uint4*>(out) + j) = r;
  }
}

__global__ void pack_words_kernel(const gw_walk_rec* __restrict__ walks, uint64_t n,
                                  const uint32_t* __restrict__ blocks, uint32_t nblocks,
                                  uint64_t* __restrict__ words, uint32_t* __restrict__ wblock) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 w = *(reinterpret_cast<const uint4*>(walks) + i);
    const uint32_t p = find_block(blocks, nblocks, w.x);
    const uint32_t rel = p < nblocks ? w.x - __ldg(blocks + p) : w.x;
    words[i] = (((uint64_t)w.z & 0xffffffu) << 40) | (((uint64_t)rel & 0x3ffffffu) << 14) |
               ((uint64_t)w.w & 0x3fffu);
    if (wblock) wblock[i] = p;
  }
}

// Random-sector gather probe: each thread issues independent 4-byte loads at
// hashed positions of a buffer much larger than L2, so every load is its own
// 32-byte DRAM sector.  The sum is kept live through *sink.
__global__ void __launch_bounds__(256)
    gather_probe_kernel(const uint32_t* __restrict__ buf, uint64_t n_words, uint64_t loads,
                        unsigned long long* __restrict__ sink) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint32_t acc = 0;
  // sectors in the buffer, rounded down to a power of two (mask, no modulo)
  uint64_t nsect = 1;
  while (nsect * 2 <= n_words / 8) nsect *= 2;
  const uint32_t mask = (uint32_t)(nsect - 1);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < loads; i += stride * 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint64_t j = i + u * stride;
      if (j < loads) {
        uint32_t h = (uint32_t)j * 0x9E3779B9u;
        h ^= h >> 15;
        h *= 0x85EBCA6Bu;
        h ^= h >> 13;
        acc += __ldg(buf + (uint64_t)(h & mask) * 8 + (j & 7));
      }
    }
  }
  if (acc == 0x9e3779b9u) atomicAdd(sink, 1ull);
}

// Random visit-counter updates alone: `ops` red.add of 1 at pseudo-random
// counters of c[0 .. mask] (mask + 1 a power of two), with the counters'
// evict_last policy, the same instruction the walk kernels count visits with.
__global__ void __launch_bounds__(256)
    red_probe_kernel(uint32_t* __restrict__ c, uint32_t mask, uint64_t ops) {
  const uint64_t pol = l2_policy(false, true);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ops; i += stride) {
    uint32_t h = (uint32_t)i * 0x9E3779B9u + (uint32_t)(i >> 32);
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    red_add_u32(c + (h & mask), 1u, pol);
  }
}

int g_num_sms = 0;

int num_sms() {
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

template <typename K>
int occupancy_grid(K kernel, uint64_t n) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kWalkThreads, 0);
  if (per_sm <= 0) per_sm = 1;
  const uint64_t full = (uint64_t)num_sms() * per_sm;
  const uint64_t need = (n + kWalkThreads - 1) / kWalkThreads;
  return (int)(need < full ? (need > 0 ? need : 1) : full);
}

template <int RULE, int SINK, bool AGG>
cudaError_t resident_dispatch(const gw_walk_rec* walks, uint64_t n, const GraphView& g,
                              const WalkArgs& a, const SinkView& s, uint32_t* status, int grid,
                              cudaStream_t stream, const cudaAccessPolicyWindow* window) {
  auto k = g.erec ? walk_resident_kernel<RULE, SINK, AGG, true> : walk_resident_kernel<RULE, SINK, AGG, false>;
  if (grid <= 0) grid = occupancy_grid(k, n);
  if (!window) {
    k<<<grid, kWalkThreads, 0, stream>>>(walks, n, g, a, s, status);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kWalkThreads);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
  attr[0].val.accessPolicyWindow = *window;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, walks, n, g, a, s, status);
}

template <int RULE, int SINK, bool AGG>
int resident_grid(uint64_t n) {
  // both variants have the same block shape; the larger register count bounds the grid
  const int a = occupancy_grid(walk_resident_kernel<RULE, SINK, AGG, false>, n);
  const int b = occupancy_grid(walk_resident_kernel<RULE, SINK, AGG, true>, n);
  return a < b ? a : b;
}

template <int RULE, int SINK, bool AGG>
cudaError_t block_dispatch(gw_walk_rec* walks, uint64_t n, const GraphView& g,
                           const unsigned long long* beg_pos, const uint32_t* csr,
                           const WalkArgs& a, const SinkView& s, const uint32_t* blocks,
                           uint32_t nblocks, uint32_t* dest, uint32_t* status,
                           cudaStream_t stream) {
  if (beg_pos) {
    auto k = walk_block_kernel<RULE, SINK, AGG, true>;
    k<<<occupancy_grid(k, n), kWalkThreads, 0, stream>>>(walks, n, g, beg_pos, csr, a, s, blocks,
                                                        nblocks, dest, status);
  } else {
    auto k = walk_block_kernel<RULE, SINK, AGG, false>;
    k<<<occupancy_grid(k, n), kWalkThreads, 0, stream>>>(walks, n, g, beg_pos, csr, a, s, blocks,
                                                        nblocks, dest, status);
  }
  return cudaGetLastError();
}

}  // namespace

// Dispatch a (rule, sink, aggregate) triple to its template instance.
#define GW_SINK_CASES(RULE, FN, ...)                                                   \
  switch (sink) {                                                                      \
    case GW_SINK_NONE: return FN<RULE, GW_SINK_NONE, false>(__VA_ARGS__);              \
    case GW_SINK_VERTEX_COUNT:                                                         \
      return agg ? FN<RULE, GW_SINK_VERTEX_COUNT, true>(__VA_ARGS__)                   \
                 : FN<RULE, GW_SINK_VERTEX_COUNT, false>(__VA_ARGS__);                 \
    case GW_SINK_PATH_RECORD: return FN<RULE, GW_SINK_PATH_RECORD, false>(__VA_ARGS__); \
    case GW_SINK_CLOSURE_COUNT: return FN<RULE, GW_SINK_CLOSURE_COUNT, false>(__VA_ARGS__); \
  }
#define GW_RULE_CASES(FN, ...)                                         \
  switch (rule) {                                                      \
    case GW_RULE_JUMP: GW_SINK_CASES(GW_RULE_JUMP, FN, __VA_ARGS__) break;       \
    case GW_RULE_STOP: GW_SINK_CASES(GW_RULE_STOP, FN, __VA_ARGS__) break;       \
    case GW_RULE_PROB: GW_SINK_CASES(GW_RULE_PROB, FN, __VA_ARGS__) break;       \
    case GW_RULE_RESTART: GW_SINK_CASES(GW_RULE_RESTART, FN, __VA_ARGS__) break; \
    case GW_RULE_PPR: GW_SINK_CASES(GW_RULE_PPR, FN, __VA_ARGS__) break;         \
  }

cudaError_t launch_walk_resident(int rule, int sink, bool agg, const gw_walk_rec* walks, uint64_t n,
                                 const GraphView& g, const WalkArgs& a, const SinkView& s,
                                 uint32_t* status, int grid, cudaStream_t stream,
                                 const cudaAccessPolicyWindow* window) {
  if (n == 0) return cudaSuccess;
  GW_RULE_CASES(resident_dispatch, walks, n, g, a, s, status, grid, stream, window)
  return cudaErrorInvalidValue;
}

int walk_resident_grid(int rule, int sink, bool agg, uint64_t n) {
  GW_RULE_CASES(resident_grid, n)
  return 0;
}

cudaError_t launch_walk_block(int rule, int sink, bool agg, gw_walk_rec* walks, uint64_t n,
                              const GraphView& g, const unsigned long long* beg_pos,
                              const uint32_t* csr, const WalkArgs& a, const SinkView& s,
                              const uint32_t* blocks, uint32_t nblocks, uint32_t* dest,
                              uint32_t* status, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  if (sink == GW_SINK_PATH_RECORD) return cudaErrorInvalidValue;
  GW_RULE_CASES(block_dispatch, walks, n, g, beg_pos, csr, a, s, blocks, nblocks, dest, status,
                stream)
  return cudaErrorInvalidValue;
}

static int elementwise_grid(uint64_t n) {
  const uint64_t need = (n + 255) / 256;
  const uint64_t cap = (uint64_t)num_sms() * 16;
  return (int)(need < cap ? (need ? need : 1) : cap);
}

cudaError_t launch_unpack_words(const uint64_t* words, const uint32_t* ids, uint64_t n,
                                uint32_t block_base, gw_walk_rec* out, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  unpack_words_kernel<<<elementwise_grid(n), 256, 0, stream>>>(words, ids, n, block_base, out);
  return cudaGetLastError();
}

cudaError_t launch_unpack_pools(const uint64_t* words, const uint32_t* ids, uint64_t first,
                                uint64_t n, const uint64_t* pool_offsets, const uint32_t* blocks,
                                uint32_t nblocks, gw_walk_rec* out, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  unpack_pools_kernel<<<elementwise_grid(n), 256, 0, stream>>>(words, ids, first, n, pool_offsets,
                                                               blocks, nblocks, out);
  return cudaGetLastError();
}

cudaError_t launch_pack_words(const gw_walk_rec* walks, uint64_t n, const uint32_t* blocks,
                              uint32_t nblocks, uint64_t* words, uint32_t* wblock,
                              cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  pack_words_kernel<<<elementwise_grid(n), 256, 0, stream>>>(walks, n, blocks, nblocks, words,
                                                             wblock);
  return cudaGetLastError();
}

cudaError_t launch_build_erec(const uint32_t* colidx, const unsigned long long* vrec, uint64_t ne, uint32_t nv,
                              ulonglong2* erec, cudaStream_t stream) {
  if (ne == 0) return cudaSuccess;
  build_erec_kernel<<<elementwise_grid(ne), 256, 0, stream>>>(colidx, vrec, ne, nv, erec);
  return cudaGetLastError();
}

cudaError_t launch_gather_probe(const uint32_t* buf, uint64_t n_words, uint64_t loads,
                                unsigned long long* sink, cudaStream_t stream) {
  const int grid = num_sms() * 8;
  gather_probe_kernel<<<grid, 256, 0, stream>>>(buf, n_words, loads, sink);
  return cudaGetLastError();
}

cudaError_t launch_red_probe(uint32_t* counters, uint32_t mask, uint64_t ops, cudaStream_t stream) {
  red_probe_kernel<<<num_sms() * 8, 256, 0, stream>>>(counters, mask, ops);
  return cudaGetLastError();
}

}  // namespace gw
