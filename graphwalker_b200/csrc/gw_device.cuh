// gw_device.cuh -- device-side building blocks of the walk engine.
//
// Per-hop draws: words 0 and 1 of Philox4x32-10 (Salmon et al., SC'11) with
// key = seed and counter = (walk id, hop, 0, 0), each shifted right by one so
// that they span rand_r's [0, RAND_MAX] (src/api/datatype.hpp:8).  The draw
// consumption order is the reference's (randomwalkwithjump.hpp:45-50): when
// the vertex has out-edges the first word is the continuation test and the
// second picks the neighbour (or the jump target when the test fails); a
// dangling vertex skips the test (short-circuit `outd > 0 && ...`) and its
// jump uses the first word.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/graphwalker_b200.h"

namespace gw {

// Packed vertex record: (first-edge offset << 24) | min(out-degree, 0xFFFFFF).
// One 8-byte load (always inside one 32-byte sector) replaces the two 8-byte
// row-pointer loads; a degree field of 0xFFFFFF means "read the row pointer".
constexpr uint32_t kDegEscape = 0xFFFFFFu;
constexpr int kDegBits = 24;

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

struct Philox4 {
  uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                         uint32_t c3, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)kPhiloxM0 * c0;
    const uint64_t p1 = (uint64_t)kPhiloxM1 * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c0 = n0;
    c1 = (uint32_t)p1;
    c2 = n2;
    c3 = (uint32_t)p0;
    k0 += kPhiloxW0;
    k1 += kPhiloxW1;
  }
  return Philox4{c0, c1, c2, c3};
}

// ---- L2 eviction-priority hints (PTX createpolicy / .L2::cache_hint) ----
// The column array is read once per visit at a random position and gains
// nothing from staying in L2; the visit counters are read-modify-written at
// every visit and the vertex records of hub vertices are re-read often.
// Hints let the kernel keep the latter resident at the expense of the former.
constexpr uint32_t kHintColumnsEvictFirst = 1u;
constexpr uint32_t kHintCountsEvictLast = 2u;
constexpr uint32_t kHintRecordsEvictLast = 4u;
// The resident kernel reads every walk record once and every walk's start
// record once, in order: streams that gain nothing from staying in L2.
constexpr uint32_t kHintStreamsEvictFirst = 8u;

__device__ __forceinline__ uint64_t l2_policy(bool first, bool last) {
  uint64_t p;
  if (first) asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  else if (last) asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  else asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ uint32_t ld_nc_u32(const uint32_t* a, uint64_t pol) {
  uint32_t r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(r) : "l"(a), "l"(pol));
  return r;
}

__device__ __forceinline__ unsigned long long ld_nc_u64(const unsigned long long* a, uint64_t pol) {
  unsigned long long r;
  asm volatile("ld.global.nc.L2::cache_hint.b64 %0, [%1], %2;" : "=l"(r) : "l"(a), "l"(pol));
  return r;
}

__device__ __forceinline__ uint4 ld_nc_u32x4(const uint4* a, uint64_t pol) {
  uint4 r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(a), "l"(pol));
  return r;
}

__device__ __forceinline__ ulonglong2 ld_nc_u64x2(const ulonglong2* a, uint64_t pol) {
  ulonglong2 r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;"
               : "=l"(r.x), "=l"(r.y)
               : "l"(a), "l"(pol));
  return r;
}

__device__ __forceinline__ void red_add_u32(uint32_t* a, uint32_t v, uint64_t pol) {
  asm volatile("red.relaxed.gpu.global.add.L2::cache_hint.u32 [%0], %1, %2;" ::"l"(a), "r"(v), "l"(pol)
               : "memory");
}

// Launch-constant parameters of a walk kernel (passed by value, lands in the
// constant bank).
struct WalkArgs {
  uint32_t hints;      // kHint* bits
  uint32_t L;          // length cap (JUMP/STOP/PPR) or segment length (RESTART)
  uint32_t thr;        // continuation passes iff draw >= thr
  uint32_t njump;      // JUMP target range
  uint32_t max_hops;   // hop guard of the uncapped rule
  uint32_t seed_lo, seed_hi;
  uint32_t path_stride;
  uint32_t lo, hi;     // block range [lo, hi) in blocked mode
  uint32_t native;     // 1 = native-RNG mode (one Philox block per two hops)
};

struct GraphView {
  const unsigned long long* __restrict__ vrec;    // packed vertex records (nv)
  const unsigned long long* __restrict__ rowptr;  // row pointer (nv + 1)
  const uint32_t* __restrict__ colidx;
  // Edge records (one per edge, NULL when not built): x = the packed record
  // of the edge's target, y = the target's id.  Moving along an edge then
  // reads the next vertex and its record in one 16-byte load.
  const ulonglong2* __restrict__ erec;
  // Out-edge bitmap (nv bits, stored right after the packed records; NULL
  // when the records are not built): bit v is set when v has out-edges.
  const uint32_t* __restrict__ out_bits;
  uint32_t nv;
};

struct SinkView {
  uint32_t* __restrict__ counts;             // VERTEX_COUNT
  uint32_t* __restrict__ paths;              // PATH_RECORD, [walk][visit]
  uint32_t* __restrict__ plen;               // PATH_RECORD, visits per walk
  unsigned long long* __restrict__ closure;  // CLOSURE_COUNT
};

template <int RULE>
__device__ __forceinline__ constexpr bool rule_capped() {
  return RULE == GW_RULE_JUMP || RULE == GW_RULE_STOP || RULE == GW_RULE_PPR;
}

// One hop of one walk at vertex v (already visited).  Returns false when the
// walk ends inside this hop (stop rules); otherwise v is the next vertex and
// the caller increments the hop.  Loads go through the read-only path.
struct L2Hints {
  uint64_t rec, col, cnt, bits, strm;
};

__device__ __forceinline__ L2Hints make_hints(uint32_t flags) {
  L2Hints h;
  h.rec = l2_policy(false, flags & kHintRecordsEvictLast);
  h.col = l2_policy(flags & kHintColumnsEvictFirst, false);
  h.cnt = l2_policy(false, flags & kHintCountsEvictLast);
  h.bits = l2_policy(false, true);  // the out-edge bitmap is small and read at every jump
  h.strm = l2_policy(flags & kHintStreamsEvictFirst, false);
  return h;
}

// ---- per-hop draws ----
// Philox mode (GW_RNG_PHILOX, the deterministic mode): the hop's two draws
// are words 0 and 1 of Philox(key = seed, counter = (id, hop, stream, 0)),
// consumed in the reference's order, so trajectories equal the shimmed
// reference's.  Native-RNG mode (GW_RNG_NATIVE): one Philox block serves two
// hops -- words 0, 1 for the even hop 2m and words 2, 3 for hop 2m + 1 of
// Philox(seed, (id, m, stream, kNativeTag)) -- so a walk computes one block
// per two hops.  Its draws are still a pure function of (seed, id, hop,
// stream), independent of the schedule; the mode is checked statistically
// against the FP64 power series, not against the reference's trajectories.
constexpr uint32_t kNativeTag = 0x4E415456u;  // "NATV"
constexpr uint32_t kNoHop = 0xffffffffu;

// The spare words of the last native block a thread computed, valid for
// hop `hop` of the walk the thread holds; reset whenever it takes a walk.
struct DrawCache {
  uint32_t z, w, hop;
  __device__ __forceinline__ void reset() { hop = kNoHop; }
};

struct Draws {
  uint32_t d0, d1;
};

__device__ __forceinline__ Draws hop_draws(const WalkArgs& a, uint32_t id, uint32_t hop, uint32_t stream,
                                           DrawCache& dc) {
  if (!a.native) {
    const Philox4 ph = philox4x32_10(id, hop, stream, 0u, a.seed_lo, a.seed_hi);
    return Draws{ph.x >> 1, ph.y >> 1};
  }
  if (dc.hop == hop) {
    dc.hop = kNoHop;
    return Draws{dc.z >> 1, dc.w >> 1};
  }
  const Philox4 ph = philox4x32_10(id, hop >> 1, stream, kNativeTag, a.seed_lo, a.seed_hi);
  if (hop & 1u) return Draws{ph.z >> 1, ph.w >> 1};
  dc.z = ph.z;
  dc.w = ph.w;
  dc.hop = hop + 1;
  return Draws{ph.x >> 1, ph.y >> 1};
}

template <int RULE>
__device__ __forceinline__ bool hop_advance_rec(const GraphView& g, const WalkArgs& a, const L2Hints& hp,
                                                uint32_t id, uint32_t src, uint32_t hop, uint32_t& v,
                                                unsigned long long rec, DrawCache& dc, uint32_t stream = 0u);

template <int RULE>
__device__ __forceinline__ bool hop_advance(const GraphView& g, const WalkArgs& a, const L2Hints& hp,
                                            uint32_t id, uint32_t src, uint32_t hop, uint32_t& v, DrawCache& dc) {
  return hop_advance_rec<RULE>(g, a, hp, id, src, hop, v, ld_nc_u64(g.vrec + v, hp.rec), dc);
}

// The hop with v's packed record already loaded (callers that have other
// memory work per visit issue the record load first to overlap the two).
// `stream` is the third Philox counter word: 0 for walks keyed by a global
// walk id; a served query's own stream id otherwise.
template <int RULE>
__device__ __forceinline__ bool hop_advance_rec(const GraphView& g, const WalkArgs& a, const L2Hints& hp,
                                                uint32_t id, uint32_t src, uint32_t hop, uint32_t& v,
                                                unsigned long long rec, DrawCache& dc, uint32_t stream) {
  const Draws dr = hop_draws(a, id, hop, stream, dc);
  const uint32_t d0 = dr.d0;
  const uint32_t d1 = dr.d1;
  unsigned long long off = rec >> kDegBits;
  unsigned long long deg = rec & kDegEscape;
  if (deg == kDegEscape) {  // mega-hub: exact degree from the row pointer
    const unsigned long long b = __ldg(g.rowptr + v);
    deg = __ldg(g.rowptr + v + 1) - b;
    off = b;
  }
  if (deg > 0 && d0 >= a.thr) {
    // (eid_t)rand_r % outd with a 31-bit draw: equals the draw when outd > 2^31
    const unsigned long long r =
        deg > 0x7fffffffull ? (unsigned long long)d1 : (unsigned long long)(d1 % (uint32_t)deg);
    v = ld_nc_u32(g.colidx + off + r, hp.col);
    return true;
  }
  const uint32_t dj = deg > 0 ? d1 : d0;
  if (RULE == GW_RULE_JUMP) {
    v = dj % a.njump;
    return true;
  } else if (RULE == GW_RULE_RESTART) {
    v = src;
    return true;
  } else if (RULE == GW_RULE_PPR) {
    if (deg == 0) {
      v = src;
      return true;
    }
    return false;
  }
  return false;  // STOP, PROB
}

// v's packed record, or 0 (no edges) when v is out of range: the caller's
// bounds check ends the walk before that record is used.
__device__ __forceinline__ unsigned long long vertex_rec(const GraphView& g, const L2Hints& hp, uint32_t v) {
  return v < g.nv ? ld_nc_u64(g.vrec + v, hp.rec) : 0ull;
}

// The record of a jump target.  A target without out-edges needs none: its
// next hop reads only the degree, which is 0 (its record's offset field is
// never used), so the 8-byte record load -- a DRAM miss for most uniformly
// drawn targets -- is replaced by a read of the out-edge bitmap, which stays
// in L2.  Targets with out-edges load their record as before.
__device__ __forceinline__ unsigned long long jump_rec(const GraphView& g, const L2Hints& hp, uint32_t v) {
  if (v >= g.nv) return 0ull;
  if (g.out_bits && !((ld_nc_u32(g.out_bits + (v >> 5), hp.bits) >> (v & 31u)) & 1u)) return 0ull;
  return ld_nc_u64(g.vrec + v, hp.rec);
}

// A jump target with out-edges whose record is not loaded yet.  The load
// waits for the target's own hop, and happens only if that hop moves along an
// edge (or never, when the target's visit is the walk's last): its test can
// fail (a jump needs only "degree > 0", which the bitmap gave), and the last
// visit makes no move.  No packed record has this value: its offset field
// would name edge 2^40 - 1.
constexpr unsigned long long kDeferredRec = ~0ull;

__device__ __forceinline__ unsigned long long jump_rec_deferred(const GraphView& g, const L2Hints& hp, uint32_t v) {
  if (v >= g.nv) return 0ull;
  if (g.out_bits) return ((ld_nc_u32(g.out_bits + (v >> 5), hp.bits) >> (v & 31u)) & 1u) ? kDeferredRec : 0ull;
  return ld_nc_u64(g.vrec + v, hp.rec);
}

// The same hop over the edge-record layout: the record of v is carried in
// `rec` from the previous hop.  Moving along an edge reads the next vertex and
// its record together; a jump defers the record of its target (above); a
// return to the source takes the source's record, src_rec, held by the caller.
template <int RULE>
__device__ __forceinline__ bool hop_advance_carried(const GraphView& g, const WalkArgs& a, const L2Hints& hp,
                                                    uint32_t id, uint32_t src, unsigned long long src_rec,
                                                    uint32_t hop, uint32_t& v, unsigned long long& rec,
                                                    DrawCache& dc, uint32_t stream = 0u) {
  const Draws dr = hop_draws(a, id, hop, stream, dc);
  const uint32_t d0 = dr.d0;
  const uint32_t d1 = dr.d1;
  if (rec == kDeferredRec) {
    // v has out-edges: a failed test jumps with the second draw (outd > 0),
    // without v's record; a passed one needs it now
    if (RULE == GW_RULE_JUMP && d0 < a.thr) {
      v = d1 % a.njump;
      rec = jump_rec_deferred(g, hp, v);
      return true;
    }
    rec = ld_nc_u64(g.vrec + v, hp.rec);
  }
  unsigned long long off = rec >> kDegBits;
  unsigned long long deg = rec & kDegEscape;
  if (deg == kDegEscape) {  // mega-hub: exact degree from the row pointer
    const unsigned long long b = __ldg(g.rowptr + v);
    deg = __ldg(g.rowptr + v + 1) - b;
    off = b;
  }
  if (deg > 0 && d0 >= a.thr) {
    const unsigned long long r =
        deg > 0x7fffffffull ? (unsigned long long)d1 : (unsigned long long)(d1 % (uint32_t)deg);
    const ulonglong2 e = ld_nc_u64x2(g.erec + off + r, hp.col);
    v = (uint32_t)e.y;
    rec = e.x;
    return true;
  }
  const uint32_t dj = deg > 0 ? d1 : d0;
  if (RULE == GW_RULE_JUMP) {
    v = dj % a.njump;
    rec = jump_rec_deferred(g, hp, v);
    return true;
  } else if (RULE == GW_RULE_RESTART) {
    v = src;
    rec = src_rec;
    return true;
  } else if (RULE == GW_RULE_PPR) {
    if (deg == 0) {
      v = src;
      rec = src_rec;
      return true;
    }
    return false;
  }
  return false;  // STOP, PROB
}

// Whether the visit at `hop` is the walk's last: the capped rules visit hops
// 0 .. L-1, and a restart segment ends on reaching hop % L == L-1.  The move
// after a last visit is never observed -- the reference's loop tests
// hop < L (or the segment end) before it uses the vertex it moved to
// (randomwalkwithjump.hpp:40,55; randomwalkwithrestartwithjoint.hpp:52) --
// so the kernels skip it, with its draws and its gather.  The uncapped rule
// has no last visit: its walk ends by the draw itself.
template <int RULE>
__device__ __forceinline__ bool last_visit(const WalkArgs& a, uint32_t hop) {
  if (RULE == GW_RULE_JUMP || RULE == GW_RULE_STOP || RULE == GW_RULE_PPR) return hop + 1 >= a.L;
  if (RULE == GW_RULE_RESTART) return hop % a.L == (2 * a.L - 2) % a.L;
  return false;
}

// Whether a rule's hop can return a walk to its source.
template <int RULE>
__device__ __forceinline__ constexpr bool rule_returns() {
  return RULE == GW_RULE_RESTART || RULE == GW_RULE_PPR;
}

// Same hop over a block-local CSR slice (streamed blocks): beg_pos is the
// slice of the row pointer for [lo, hi] (global edge offsets) and csr the
// slice of the column array that starts at beg_pos[0], exactly the buffers
// the reference's loadSubGraph fills (graphwalker.hpp:168-209).
template <int RULE>
__device__ __forceinline__ bool hop_advance_slice(const unsigned long long* __restrict__ beg_pos,
                                                  const uint32_t* __restrict__ csr,
                                                  unsigned long long b0, const WalkArgs& a,
                                                  uint32_t id, uint32_t src, uint32_t hop,
                                                  uint32_t& v, DrawCache& dc) {
  const uint32_t vl = v - a.lo;
  const unsigned long long b = __ldg(beg_pos + vl);
  const unsigned long long deg = __ldg(beg_pos + vl + 1) - b;
  const Draws dr = hop_draws(a, id, hop, 0u, dc);
  const uint32_t d0 = dr.d0;
  const uint32_t d1 = dr.d1;
  if (deg > 0 && d0 >= a.thr) {
    const unsigned long long r =
        deg > 0x7fffffffull ? (unsigned long long)d1 : (unsigned long long)(d1 % (uint32_t)deg);
    v = __ldg(csr + (b - b0) + r);
    return true;
  }
  const uint32_t dj = deg > 0 ? d1 : d0;
  if (RULE == GW_RULE_JUMP) {
    v = dj % a.njump;
    return true;
  } else if (RULE == GW_RULE_RESTART) {
    v = src;
    return true;
  } else if (RULE == GW_RULE_PPR) {
    if (deg == 0) {
      v = src;
      return true;
    }
    return false;
  }
  return false;
}

// Count one visit of v.  AGG folds lanes of the warp that visit the same
// vertex in the same instruction into one atomic (hub vertices, and every
// walk of a single-source query at hop 0).
template <bool AGG>
__device__ __forceinline__ void count_visit(uint32_t* __restrict__ counts, uint32_t v, uint64_t pol) {
  if (AGG) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, v);
    const int lane = threadIdx.x & 31;
    if (lane == __ffs(peers) - 1) red_add_u32(counts + v, (uint32_t)__popc(peers), pol);
  } else {
    red_add_u32(counts + v, 1u, pol);
  }
}

}  // namespace gw
