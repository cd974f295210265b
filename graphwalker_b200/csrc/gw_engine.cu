// gw_engine.cu -- GraphWalker's block loop on the device.
//
//   graphwalker_engine::run            src/engine/graphwalker.hpp:272-311
//   findSubGraph / loadSubGraph        src/engine/graphwalker.hpp:168-234
//   swapOut (evict fewest walks)       src/engine/graphwalker.hpp:236-251
//   WalkManager::chooseBlock & co.     src/walks/walk.hpp:204-252
//   getCurrentWalks / updateWalkNum    src/walks/walk.hpp:114-192
//   writeWalks2Disk / readWalksfromDisk src/walks/walk.hpp:103-157 (pool budget)
//
// Each superstep picks a block with the reference's state-aware policy (with
// probability `prob` the block holding the lowest-hop walk, otherwise the
// block with the most pending walks), makes its CSR available (resident HBM,
// or a slot filled from pinned host memory by async copies on a side stream),
// advances every walk of its pool while it stays inside the block, and stably
// partitions the walks that left into the pools of their new blocks.  The
// per-block pending counts and minimum hops the policy reads come back from
// the partition's histogram each superstep, through mapped pinned memory, so
// no small copy of a superstep queues behind a block copy.
//
// Streaming differs from findSubGraph in three ways that change neither the
// order of blocks nor any walk:
//  * the row pointer stays in HBM, and a slot holds a block's column slice;
//  * a chosen block in no slot whose pool is small (ctx->mapped_max_walks,
//    or per block its column bytes / kMappedBytesPerWalk) is read in place
//    from the pinned host columns through their mapped device address: each
//    hop fetches one sector over the host link instead of the whole block;
//  * while a block runs, up to kCopyAhead blocks with many pending walks are
//    copied into slots before their turn, each taking the room of the slot
//    with the fewest pending walks (swapOut's victim) when it has more.
//
// With a pool budget (ctx->pool_budget), walk pools beyond it wait in a
// pinned host arena, in either residency; a pool is the arena part (older
// walks) followed by its device part, so pool order is kept.
#include <algorithm>
#include <cstring>

#include "gw_ctx.h"

namespace gw {

namespace {

constexpr uint32_t kNoBlock = 0xffffffffu;
// GW_MAPPED_AUTO: a streamed block runs in place when it has at most one
// pending walk per this many bytes of its column slice.  Copying a block
// costs its bytes at the host link's rate; a walk run in place costs a sector
// per hop fetched over the same link and waits on its latency.
constexpr uint64_t kMappedBytesPerWalk = 128;
// Blocks copied ahead of their turn at most (1 to 5 measured within 2 % of
// one another on an out-of-core scale-27 graph, the deeper the faster).
constexpr size_t kCopyAhead = 3;

struct Slots {
  // One device slot holds the column slice of one block,
  //   csr[beg_pos[blocks[b]] .. beg_pos[blocks[b+1]]);
  // the row pointer of every block stays in HBM.
  std::vector<gw_devbuf> csr;
  std::vector<uint32_t> block;      // block held, kNoBlock if empty
  std::vector<cudaEvent_t> ready;   // copy finished
  std::vector<cudaEvent_t> free_ev; // last kernel reading the slot finished
  std::vector<int> slot_of;         // per block: slot index or -1
  ~Slots() {
    for (auto& b : csr) b.release();
    for (auto e : ready) cudaEventDestroy(e);
    for (auto e : free_ev) cudaEventDestroy(e);
  }
};

// chooseBlock (walk.hpp:245-252) over the engine's pending counts.
uint32_t block_with_max_walks(const std::vector<uint64_t>& walknum) {
  uint64_t maxw = 0;
  uint32_t maxp = 0;
  for (uint32_t p = 0; p < walknum.size(); ++p)
    if (maxw < walknum[p]) {
      maxw = walknum[p];
      maxp = p;
    }
  return maxp;
}

uint32_t block_with_min_step(const std::vector<uint64_t>& walknum, const std::vector<uint32_t>& minstep) {
  uint32_t mins = 0xffff, minp = 0;
  for (uint32_t p = 0; p < minstep.size(); ++p)
    if (mins > minstep[p]) {
      mins = minstep[p];
      minp = p;
    }
  if (walknum[minp] > 0) return minp;
  return block_with_max_walks(walknum);
}

uint32_t choose_block(const std::vector<uint64_t>& walknum, const std::vector<uint32_t>& minstep,
                      float prob, uint64_t seed, uint64_t superstep) {
  // the reference's coin is ((float)rand())/RAND_MAX; here its 31-bit draw
  // comes from Philox(seed, (superstep, "CHOS")) so a run is reproducible
  const Philox4 ph = philox4x32_10((uint32_t)superstep, (uint32_t)(superstep >> 32), 0x43484F53u,
                                   0u, (uint32_t)seed, (uint32_t)(seed >> 32));
  const float cc = (float)(int32_t)(ph.x >> 1) / 2147483647;
  if (cc < prob) return block_with_min_step(walknum, minstep);
  return block_with_max_walks(walknum);
}

}  // namespace

gw_status run_blocked(gw_ctx* ctx, const gw_walk_params* p) {
  WalkArgs a;
  gw_status s = make_walk_args(ctx, p, &a);
  if (s != GW_OK) return s;
  if (p->sink == GW_SINK_PATH_RECORD)
    return ctx->fail(GW_E_INVALID, "PATH_RECORD needs GW_MODE_RESIDENT");
  const uint32_t nb = ctx->nblocks;
  if (nb + 1 > 8000) return ctx->fail(GW_E_INVALID, "at most 7999 blocks in blocked mode");
  // Owned blocks (one rank of a vertex-partitioned run): only the blocks in
  // [own_lo, own_hi) execute, and walks that move to other blocks wait in
  // those blocks' pools for gw_read_pool.  block_hi = 0: every block.
  const uint32_t own_lo = p->block_hi ? p->block_lo : 0, own_hi = p->block_hi ? p->block_hi : nb;
  if (own_lo >= own_hi || own_hi > nb)
    return ctx->fail(GW_E_INVALID, "owned blocks [%u, %u) not inside [0, %u)", p->block_lo, p->block_hi, nb);
  const bool restricted = own_lo > 0 || own_hi < nb;
  const bool streaming = ctx->residency == GW_STREAM_PINNED;
  cudaStream_t st = ctx->stream, xs = ctx->copy_stream;

  // ---- initial pools (startWalks; getCurrentWalks reads them back) ----
  ctx->pools.resize(nb);
  ctx->pool_chunks.assign(nb, {});
  ctx->pool_host_n.assign(nb, 0);
  ctx->pool_size.assign(nb, 0);
  ctx->minstep.assign(nb, 0xffff);
  ctx->stats = gw_run_stats{};
  std::vector<uint64_t> cap(nb, 0);
  for (uint32_t b = 0; b < nb; ++b) cap[b] = ctx->pools[b].bytes / sizeof(gw_walk_rec);
  // Grown pools come from the stream-ordered allocator, so replacing one
  // queues its free behind the copy out of it; a pool from gw_walks_add is
  // retired instead and freed with the events.
  std::vector<char> pool_async(nb, 0);
  // records of block d's pool held on the device (after its host part)
  auto dev_n = [&](uint32_t d) { return ctx->pool_size[d] - ctx->pool_host_n[d]; };
  constexpr uint64_t kChunk = gw_ctx::kPoolChunk;
  if (ctx->pool_budget) {
    // pinned chunks for every walk of the run, plus a partly filled one per block
    uint64_t total = 0;
    for (uint32_t b = 0; b < nb; ++b) total += ctx->pool_words[b].size();
    const uint64_t nchunks = (total + kChunk - 1) / kChunk + nb;
    GW_CUDA(ctx, ctx->pool_arena.ensure(nchunks * kChunk * sizeof(gw_walk_rec)), "pool arena");
    ctx->arena_free.resize(nchunks);
    for (uint64_t c = 0; c < nchunks; ++c) ctx->arena_free[c] = (uint32_t)(nchunks - 1 - c);
  }
  gw_walk_rec* const arena = ctx->pool_arena.as<gw_walk_rec>();
  // writeWalks2Disk: once the device pools hold more than the budget, the
  // pools with the fewest pending walks (never the fullest) move to host
  // memory, empty pools first giving back their room, until they hold half
  // of it: the headroom takes many supersteps' arrivals before the next
  // spill, so pools move out in a few large batches, not a few every step.
  auto spill_to_budget = [&]() -> cudaError_t {
    if (!ctx->pool_budget) return cudaSuccess;
    uint64_t held = 0;
    for (uint32_t d = 0; d < nb; ++d) held += cap[d];
    if (held * sizeof(gw_walk_rec) <= ctx->pool_budget) return cudaSuccess;
    const uint64_t low = ctx->pool_budget / 2;
    uint32_t fullest = 0;
    for (uint32_t d = 1; d < nb; ++d)
      if (ctx->pool_size[d] > ctx->pool_size[fullest]) fullest = d;
    std::vector<uint32_t> order;
    for (uint32_t d = 0; d < nb; ++d)
      if (cap[d] && d != fullest) order.push_back(d);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
      const bool ex = dev_n(x) == 0, ey = dev_n(y) == 0;
      return ex != ey ? ex : ctx->pool_size[x] < ctx->pool_size[y];
    });
    // Copies out and frees of stream-ordered pools queue on st behind the
    // scatter that filled them; pools from gw_walks_add are freed after a
    // synchronisation.
    cudaError_t e = cudaSuccess;
    std::vector<void*> sync_free;
    for (size_t i = 0; i < order.size() && e == cudaSuccess && held * sizeof(gw_walk_rec) > low; ++i) {
      const uint32_t d = order[i];
      const uint64_t dn = dev_n(d);
      for (uint64_t off = 0; off < dn && e == cudaSuccess;) {
        uint64_t& hn = ctx->pool_host_n[d];
        const uint64_t used = hn % kChunk;
        if (used == 0) {
          if (ctx->arena_free.empty()) return cudaErrorMemoryAllocation;
          ctx->pool_chunks[d].push_back(ctx->arena_free.back());
          ctx->arena_free.pop_back();
        }
        const uint64_t c = ctx->pool_chunks[d].back(), m = std::min(kChunk - used, dn - off);
        e = cudaMemcpyAsync(arena + c * kChunk + used, ctx->pools[d].as<gw_walk_rec>() + off,
                            m * sizeof(gw_walk_rec), cudaMemcpyDeviceToHost, st);
        hn += m;
        off += m;
      }
      if (e != cudaSuccess) break;
      if (dn) ctx->stats.pools_spilled++;
      if (pool_async[d]) e = cudaFreeAsync(ctx->pools[d].p, st);
      else sync_free.push_back(ctx->pools[d].p);
      ctx->pools[d].p = nullptr;
      ctx->pools[d].bytes = 0;
      held -= cap[d];
      cap[d] = 0;
      pool_async[d] = 0;
    }
    if (!sync_free.empty()) {
      const cudaError_t e2 = cudaStreamSynchronize(st);
      for (void* q : sync_free) cudaFree(q);
      if (e == cudaSuccess) e = e2;
    }
    return e;
  };
  uint64_t walksum = 0, maxpool = 0;
  for (uint32_t b = 0; b < nb; ++b) maxpool = std::max<uint64_t>(maxpool, ctx->pool_words[b].size());
  GW_CUDA(ctx, ctx->d_words.ensure(maxpool * 8), "word alloc");
  if (ctx->pools_have_ids) GW_CUDA(ctx, ctx->d_ids.ensure(maxpool * 4), "id alloc");
  for (uint32_t b = 0; b < nb; ++b) {
    const uint64_t m = ctx->pool_words[b].size();
    if (!m) continue;
    if (cap[b] < m) {
      GW_CUDA(ctx, ctx->pools[b].ensure(m * sizeof(gw_walk_rec)), "pool alloc");
      cap[b] = m;
    }
    GW_CUDA(ctx, cudaMemcpyAsync(ctx->d_words.p, ctx->pool_words[b].data(), m * 8,
                                 cudaMemcpyHostToDevice, st), "walk upload");
    if (ctx->pools_have_ids)
      GW_CUDA(ctx, cudaMemcpyAsync(ctx->d_ids.p, ctx->pool_ids[b].data(), m * 4,
                                   cudaMemcpyHostToDevice, st), "id upload");
    GW_CUDA(ctx, launch_unpack_words(ctx->d_words.as<uint64_t>(),
                                     ctx->pools_have_ids ? ctx->d_ids.as<uint32_t>() : nullptr, m,
                                     ctx->blocks[b], ctx->pools[b].as<gw_walk_rec>(), st), "unpack");
    GW_CUDA(ctx, cudaStreamSynchronize(st), "walk upload");  // host words are reused next block
    ctx->pool_size[b] = m;
    for (uint64_t w : ctx->pool_words[b]) ctx->minstep[b] = std::min<uint32_t>(ctx->minstep[b], gw_get_hop(w));
    walksum += m;
    GW_CUDA(ctx, spill_to_budget(), "pool spill");
  }
  const uint64_t nwalks = walksum;
  walksum = 0;  // from here on: walks pending in the owned blocks
  for (uint32_t b = own_lo; b < own_hi; ++b) walksum += ctx->pool_size[b];
  std::vector<uint64_t> own_num;
  std::vector<uint32_t> own_min;

  // ---- sinks ----
  SinkView sv{};
  GW_CUDA(ctx, ctx->d_counts.ensure((size_t)ctx->nv * 4), "counts alloc");
  GW_CUDA(ctx, cudaMemsetAsync(ctx->d_counts.p, 0, (size_t)ctx->nv * 4, st), "counts clear");
  GW_CUDA(ctx, ctx->d_closure.ensure(8), "closure alloc");
  GW_CUDA(ctx, cudaMemsetAsync(ctx->d_closure.p, 0, 8, st), "closure clear");
  sv.counts = ctx->d_counts.as<uint32_t>();
  sv.closure = ctx->d_closure.as<unsigned long long>();

  // ---- partition scratch ----
  const uint32_t nbk = nb + 1;  // + the "ended" bucket
  GW_CUDA(ctx, ctx->d_totals.ensure(nbk * 4), "minhop alloc");  // per-bucket minimum hop
  // cleared once; each superstep's totals kernel resets it after reading it
  GW_CUDA(ctx, cudaMemsetAsync(ctx->d_totals.p, 0xff, nbk * 4, st), "minhop clear");
  GW_CUDA(ctx, ctx->d_out_ptr.ensure(nbk * sizeof(void*)), "ptr alloc");
  GW_CUDA(ctx, ctx->d_out_base.ensure(nbk * 8), "base alloc");
  gw_hostbuf h_xfer;  // pinned: totals|minhop down, ptr|base up
  GW_CUDA(ctx, h_xfer.ensure(2 * nbk * 4 + nbk * (sizeof(void*) + 8)), "pinned scratch");
  uint32_t* h_totals = h_xfer.as<uint32_t>();
  uint32_t* h_minhop = h_totals + nbk;
  gw_walk_rec** h_ptr = reinterpret_cast<gw_walk_rec**>(h_totals + 2 * nbk);
  uint64_t* h_base = reinterpret_cast<uint64_t*>(h_ptr + nbk);
  // The device reaches h_xfer at its mapped address: the totals kernel writes
  // totals|minhop there and a fetch kernel reads ptr|base, so the small
  // transfers of a superstep never wait behind a block copy on the copy engine.
  void* m_xfer = nullptr;
  GW_CUDA(ctx, cudaHostGetDevicePointer(&m_xfer, h_xfer.p, 0), "mapped scratch");
  uint32_t* m_totals = static_cast<uint32_t*>(m_xfer);
  const uint64_t* m_ptr = reinterpret_cast<const uint64_t*>(m_totals + 2 * nbk);
  const uint64_t* m_base = m_ptr + nbk;

  // ---- streamed block slots ----
  Slots slots;
  const uint32_t nslots = streaming ? std::max<uint32_t>(2, std::min(ctx->nmblocks, nb)) : 0;
  if (streaming) {
    uint64_t max_e = 0;
    const uint64_t* hr = ctx->h_rowptr.as<uint64_t>();
    for (uint32_t b = 0; b < nb; ++b) max_e = std::max<uint64_t>(max_e, hr[ctx->blocks[b + 1]] - hr[ctx->blocks[b]]);
    slots.csr.resize(nslots);
    slots.block.assign(nslots, kNoBlock);
    slots.ready.resize(nslots);
    slots.free_ev.resize(nslots);
    slots.slot_of.assign(nb, -1);
    for (uint32_t i = 0; i < nslots; ++i) {
      GW_CUDA(ctx, slots.csr[i].ensure(std::max<uint64_t>(max_e, 1) * 4), "slot alloc");
      cudaEventCreateWithFlags(&slots.ready[i], cudaEventDisableTiming);
      cudaEventCreateWithFlags(&slots.free_ev[i], cudaEventDisableTiming);
      cudaEventRecord(slots.free_ev[i], st);
    }
  }
  // mapped device address of the pinned host columns (blocks read in place)
  const uint32_t* m_colidx = nullptr;
  if (streaming && ctx->mapped_max_walks) {
    void* mp = nullptr;
    const cudaError_t me = cudaHostGetDevicePointer(&mp, ctx->h_colidx.p, 0);
    if (me == cudaSuccess) {
      m_colidx = static_cast<const uint32_t*>(mp);
    } else if (ctx->mapped_max_walks == GW_MAPPED_AUTO) {
      cudaGetLastError();  // no mapped host memory here: the default copies every block
    } else {
      return ctx->cuda_fail(me, "mapped colidx (gw_set_mapped_block_walks)");
    }
  }
  // the most pending walks at which block q runs in place (0 = never)
  auto mapped_limit = [&](uint32_t q) -> uint64_t {
    if (!m_colidx) return 0;
    if (ctx->mapped_max_walks != GW_MAPPED_AUTO) return ctx->mapped_max_walks;
    const uint64_t* hr = ctx->h_rowptr.as<uint64_t>();
    return (hr[ctx->blocks[q + 1]] - hr[ctx->blocks[q]]) * 4 / kMappedBytesPerWalk;
  };
  ctx->stats.walks = nwalks;

  std::vector<uint32_t> ahead;  // blocks copied ahead of their turn, not yet run
  // findSubGraph: make block b resident in a slot (never the slot `keep`).
  auto load_block = [&](uint32_t b, int keep) -> int {
    if (slots.slot_of[b] >= 0) return slots.slot_of[b];
    int victim = -1;
    for (uint32_t i = 0; i < nslots && victim < 0; ++i)
      if (slots.block[i] == kNoBlock && (int)i != keep) victim = (int)i;
    if (victim < 0) {  // swapOut: resident block with the fewest pending walks
      uint64_t minw = ~0ull;
      for (uint32_t i = 0; i < nslots; ++i) {
        if ((int)i == keep) continue;
        const uint64_t w = ctx->pool_size[slots.block[i]];
        if (w < minw) {
          minw = w;
          victim = (int)i;
        }
      }
      slots.slot_of[slots.block[victim]] = -1;
      ahead.erase(std::remove(ahead.begin(), ahead.end(), slots.block[victim]), ahead.end());
    }
    const uint64_t* hr = ctx->h_rowptr.as<uint64_t>();
    const uint32_t v0 = ctx->blocks[b], v1 = ctx->blocks[b + 1];
    const uint64_t e0 = hr[v0], e1 = hr[v1];
    cudaStreamWaitEvent(xs, slots.free_ev[victim], 0);
    if (e1 > e0)
      cudaMemcpyAsync(slots.csr[victim].p, ctx->h_colidx.as<uint32_t>() + e0, (e1 - e0) * 4,
                      cudaMemcpyHostToDevice, xs);
    cudaEventRecord(slots.ready[victim], xs);
    slots.block[victim] = b;
    slots.slot_of[b] = victim;
    ctx->stats.block_loads++;
    ctx->stats.bytes_h2d += (e1 - e0) * 4;
    return victim;
  };

  double ms_walk = 0, ms_partition = 0, ms_copy_wait = 0;
  // run start/end, and the phases of each superstep in two alternating sets
  // (a superstep's set is read after the next superstep's synchronisation):
  // ph[0] before the copy wait, ph[1] walk start, ph[2] walk end, ph[3]
  // partition end.  Destroyed on every return; so are the pools that grown
  // pools replaced, once no queued copy reads them.
  struct Events {
    cudaEvent_t e[10];
    std::vector<void*> retired;
    Events() {
      for (auto& x : e) cudaEventCreate(&x);
    }
    ~Events() {
      for (auto& x : e) cudaEventDestroy(x);
      for (void* p : retired) cudaFree(p);
    }
  } evs;
  cudaEvent_t t0 = evs.e[0], t1 = evs.e[1];
  auto phase_set = [&](uint64_t step) { return evs.e + 2 + 4 * (step & 1); };
  auto add_phases = [&](uint64_t step) {
    cudaEvent_t* q = phase_set(step);
    float a = 0.f, w = 0.f, m = 0.f;
    cudaEventElapsedTime(&a, q[0], q[1]);
    cudaEventElapsedTime(&w, q[1], q[2]);
    cudaEventElapsedTime(&m, q[2], q[3]);
    ms_copy_wait += a;
    ms_walk += w;
    ms_partition += m;
  };
  cudaEventRecord(t0, st);
  uint64_t superstep = 0;
  cudaError_t e = cudaSuccess;
  // The scatter of superstep k is left queued: the host next waits on the
  // stream for the partition totals of superstep k + 1, which orders it.
  bool pending = false;
  while (walksum > 0 && e == cudaSuccess &&
         (p->max_supersteps == 0 || superstep < p->max_supersteps)) {
    uint32_t b;
    if (restricted) {  // the policy sees the owned blocks only
      own_num.assign(nb, 0);
      own_min.assign(nb, 0xffff);
      for (uint32_t q = own_lo; q < own_hi; ++q) {
        own_num[q] = ctx->pool_size[q];
        own_min[q] = ctx->minstep[q];
      }
      b = choose_block(own_num, own_min, p->prob, p->seed, superstep);
    } else {
      b = choose_block(ctx->pool_size, ctx->minstep, p->prob, p->seed, superstep);
    }
    const uint64_t n = ctx->pool_size[b];
    if (n == 0) return ctx->fail(GW_E_STATE, "scheduler chose an empty block (walksum %llu)",
                                 (unsigned long long)walksum);
    if (ctx->pool_host_n[b]) {
      // readWalksfromDisk: the pool's host part (its older walks) goes first,
      // then the walks that arrived on the device since it moved out.  Its
      // chunks return to the arena at once: whatever reuses them next is a
      // copy queued on st behind these.
      const uint64_t hn = ctx->pool_host_n[b], dn = n - hn;
      const uint64_t ncap = std::max<uint64_t>(n, 1024);
      void* np = nullptr;
      e = cudaMallocAsync(&np, ncap * sizeof(gw_walk_rec), st);
      if (e != cudaSuccess) break;
      for (uint64_t i = 0; i * kChunk < hn && e == cudaSuccess; ++i) {
        const uint64_t c = ctx->pool_chunks[b][i], m = std::min(kChunk, hn - i * kChunk);
        e = cudaMemcpyAsync(static_cast<gw_walk_rec*>(np) + i * kChunk, arena + c * kChunk, m * sizeof(gw_walk_rec),
                            cudaMemcpyHostToDevice, st);
      }
      if (e == cudaSuccess && dn)
        e = cudaMemcpyAsync(static_cast<gw_walk_rec*>(np) + hn, ctx->pools[b].p, dn * sizeof(gw_walk_rec),
                            cudaMemcpyDeviceToDevice, st);
      if (ctx->pools[b].p) {
        if (pool_async[b])
          cudaFreeAsync(ctx->pools[b].p, st);
        else
          evs.retired.push_back(ctx->pools[b].p);
      }
      pool_async[b] = 1;
      ctx->pools[b].p = np;
      ctx->pools[b].bytes = ncap * sizeof(gw_walk_rec);
      cap[b] = ncap;
      for (uint32_t c : ctx->pool_chunks[b]) ctx->arena_free.push_back(c);
      ctx->pool_chunks[b].clear();
      ctx->pool_host_n[b] = 0;
      ctx->stats.pools_refilled++;
      if (e != cudaSuccess) break;
    }
    WalkArgs ab = a;
    ab.lo = ctx->blocks[b];
    ab.hi = ctx->blocks[b + 1];
    const unsigned long long* beg_pos = nullptr;
    const uint32_t* csr = nullptr;
    int slot = -1;
    const PartitionPlan plan = partition_plan(n, nbk);
    const size_t hist_n = (size_t)plan.nbuckets * plan.ntiles;
    if (pending && (n * 4 > ctx->d_dest.bytes || hist_n * 4 > ctx->d_tile_hist.bytes ||
                    hist_n * 4 > ctx->d_tile_off.bytes || plan.scan_temp_bytes > ctx->d_scan_temp.bytes)) {
      // a buffer the queued scatter reads is about to be replaced
      e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) break;
    }
    GW_CUDA(ctx, ctx->d_dest.grow(n * 4), "dest alloc");
    GW_CUDA(ctx, ctx->d_tile_hist.grow(hist_n * 4), "hist alloc");
    GW_CUDA(ctx, ctx->d_tile_off.grow(hist_n * 4), "hist alloc");
    GW_CUDA(ctx, ctx->d_scan_temp.grow(plan.scan_temp_bytes), "scan alloc");
    cudaEvent_t* ph = phase_set(superstep);
    cudaEventRecord(ph[0], st);
    if (streaming) {
      ahead.erase(std::remove(ahead.begin(), ahead.end(), b), ahead.end());
      beg_pos = ctx->d_rowptr.as<unsigned long long>() + ab.lo;
      if (slots.slot_of[b] < 0 && n <= mapped_limit(b)) {
        csr = m_colidx + ctx->h_rowptr.as<uint64_t>()[ab.lo];
        ctx->stats.mapped_supersteps++;
        ctx->stats.mapped_walks += n;
      } else {
        slot = load_block(b, -1);
        cudaStreamWaitEvent(st, slots.ready[slot], 0);
        csr = slots.csr[slot].as<uint32_t>();
      }
    }
    // ---- exec_updates ----
    cudaEventRecord(ph[1], st);
    e = launch_walk_block((int)p->rule, (int)p->sink, p->aggregate != 0, ctx->pools[b].as<gw_walk_rec>(),
                          n, ctx->view(), beg_pos, csr, ab, sv, ctx->d_blocks.as<uint32_t>(), nb,
                          ctx->d_dest.as<uint32_t>(), ctx->d_status.as<uint32_t>(), st);
    if (e != cudaSuccess) break;
    cudaEventRecord(ph[2], st);
    if (streaming) {
      if (slot >= 0) cudaEventRecord(slots.free_ev[slot], st);
      // Copy ahead: keep up to kCopyAhead blocks copied before their turn,
      // so the host link stays busy while blocks in slots run.  The candidate
      // is the block in no slot with the most pending walks (more than it
      // needs to be read in place); it takes the room of the slot with the
      // fewest pending walks, and only when it has more.
      while (ahead.size() < kCopyAhead) {
        uint64_t best = 0;
        uint32_t nxt = kNoBlock;
        for (uint32_t q = 0; q < nb; ++q)
          if (q != b && slots.slot_of[q] < 0 && ctx->pool_size[q] > best && ctx->pool_size[q] > mapped_limit(q)) {
            best = ctx->pool_size[q];
            nxt = q;
          }
        if (nxt == kNoBlock) break;
        bool room = false;
        uint64_t minw = ~0ull;
        for (uint32_t i = 0; i < nslots; ++i) {
          if ((int)i == slot) continue;
          if (slots.block[i] == kNoBlock) room = true;
          else minw = std::min<uint64_t>(minw, ctx->pool_size[slots.block[i]]);
        }
        if (!room && best <= minw) break;
        load_block(nxt, slot);
        ahead.push_back(nxt);
      }
    }
    // ---- moveWalk: stable partition by destination block ----
    uint32_t* d_minhop = ctx->d_totals.as<uint32_t>();
    e = launch_partition_hist(ctx->pools[b].as<gw_walk_rec>(), ctx->d_dest.as<uint32_t>(), n, plan,
                              ctx->d_tile_hist.as<uint32_t>(), d_minhop, st);
    if (e == cudaSuccess)
      e = launch_partition_scan(ctx->d_tile_hist.as<uint32_t>(), ctx->d_tile_off.as<uint32_t>(), m_totals,
                                plan, ctx->d_scan_temp.p, st, d_minhop, m_totals + nbk);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) break;
    if (superstep > 0) add_phases(superstep - 1);
    // updateWalkNum: grow destination pools, then scatter into them
    for (uint32_t d = 0; d < nb; ++d) {
      const uint64_t held = dev_n(d);  // the device part; a host part stays where it is
      const uint64_t need = held + h_totals[d];
      if (d != b && need > cap[d]) {
        uint64_t ncap = std::max<uint64_t>(need, cap[d] * 2);
        ncap = std::max<uint64_t>(ncap, 1024);
        void* np = nullptr;
        e = cudaMallocAsync(&np, ncap * sizeof(gw_walk_rec), st);
        if (e != cudaSuccess) break;
        if (held)
          e = cudaMemcpyAsync(np, ctx->pools[d].p, held * sizeof(gw_walk_rec), cudaMemcpyDeviceToDevice, st);
        if (ctx->pools[d].p) {
          if (pool_async[d])
            cudaFreeAsync(ctx->pools[d].p, st);
          else
            evs.retired.push_back(ctx->pools[d].p);
        }
        pool_async[d] = 1;
        ctx->pools[d].p = np;
        ctx->pools[d].bytes = ncap * sizeof(gw_walk_rec);
        cap[d] = ncap;
        if (e != cudaSuccess) break;
      }
      h_ptr[d] = ctx->pools[d].as<gw_walk_rec>();
      h_base[d] = dev_n(d);
    }
    if (e != cudaSuccess) break;
    h_ptr[nb] = nullptr;
    h_base[nb] = 0;
    e = launch_fetch_u64_pair(m_ptr, ctx->d_out_ptr.as<uint64_t>(), m_base, ctx->d_out_base.as<uint64_t>(),
                              nbk, st);
    if (e == cudaSuccess)
      e = launch_partition_scatter(ctx->pools[b].as<gw_walk_rec>(), ctx->d_dest.as<uint32_t>(), n, plan,
                                   ctx->d_tile_off.as<uint32_t>(),
                                   ctx->d_out_ptr.as<gw_walk_rec* const>(),
                                   ctx->d_out_base.as<uint64_t>(), st);
    if (e != cudaSuccess) break;
    cudaEventRecord(ph[3], st);
    // h_ptr/h_base are rewritten only after the next totals wait, when the
    // fetch kernel has read them
    pending = true;
    uint64_t forwarded = 0;
    for (uint32_t d = 0; d < nb; ++d) {
      if (!h_totals[d]) continue;
      ctx->pool_size[d] += h_totals[d];
      if (d >= own_lo && d < own_hi) forwarded += h_totals[d];
      ctx->minstep[d] = std::min<uint32_t>(ctx->minstep[d], std::min<uint32_t>(h_minhop[d], 0xffff));
    }
    walksum = walksum - n + forwarded;
    ctx->pool_size[b] = 0;
    ctx->minstep[b] = 0xffff;
    ++superstep;
    e = spill_to_budget();
  }
  cudaEventRecord(t1, st);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "blocked engine");
  s = take_status(ctx, st);  // synchronises the stream
  if (superstep > 0) add_phases(superstep - 1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  ctx->stats.supersteps = superstep;
  ctx->stats.ms_total = ms;
  ctx->stats.ms_walk = ms_walk;
  ctx->stats.ms_partition = ms_partition;
  ctx->stats.ms_copy_wait = ms_copy_wait;
  ctx->last_nwalks = nwalks;
  ctx->last_sink = p->sink;
  ctx->last_stride = 0;
  ctx->have_run = true;
  return s;
}

}  // namespace gw
