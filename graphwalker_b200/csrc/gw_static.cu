// gw_static.cu -- one blocked-engine superstep that allocates no memory.
//
// Why it exists: some programs that drive walks cannot call cudaMalloc at the
// point where they run a superstep.  A host framework may have handed all of
// the device's free memory to its own caching allocator, so a fresh
// cudaMalloc fails; a latency-bound serving loop cannot afford the implicit
// device-wide synchronisation that cudaMalloc/cudaFree can introduce, which
// would stall work other streams have in flight.  gw_superstep_static() gives
// those callers the superstep of the blocked engine (advance the walks of one
// block, then partition the walks that left it by destination block) with
// every scratch buffer taken from the fixed array below instead of from the
// allocator.  The caller passes the walks, the counters and the outputs.
//
// Limits and sharing: the array holds scratch for at most kStaticMaxWalks
// walks and kStaticMaxBlocks blocks per call (larger requests are rejected
// with GW_E_INVALID).  Every GPU that loads this library reserves the array
// (about 12 MiB) until the process exits.  All calls share it and it keeps
// the previous call's contents: this file clears what must start from a known
// value on every call, and two calls whose work overlaps on the GPU (for
// instance on two streams without ordering between them) race on the array.
#include <mutex>

#include "gw_ctx.h"

namespace gw {
namespace {

constexpr uint64_t kStaticMaxWalks = 1ull << 20;
constexpr uint32_t kStaticMaxBlocks = 256;
constexpr uint32_t kStaticBuckets = kStaticMaxBlocks + 1;        // + "walk ended"
constexpr uint32_t kStaticWarpTile = kPartTile / (kPartThreads / 32);  // walks per warp tile
constexpr uint64_t kStaticMaxTiles = kStaticMaxWalks / kStaticWarpTile;

constexpr uint64_t align256(uint64_t x) { return (x + 255) & ~255ull; }
constexpr uint64_t kOffDest = 0;
constexpr uint64_t kOffHist = align256(kOffDest + kStaticMaxWalks * 4);
constexpr uint64_t kOffTileOff = align256(kOffHist + kStaticMaxTiles * kStaticBuckets * 4);
constexpr uint64_t kOffMinhop = align256(kOffTileOff + kStaticMaxTiles * kStaticBuckets * 4);
constexpr uint64_t kOffPtr = align256(kOffMinhop + kStaticBuckets * 4);
constexpr uint64_t kOffBase = align256(kOffPtr + kStaticBuckets * 8);
constexpr uint64_t kStaticBytes = align256(kOffBase + kStaticBuckets * 8);

// The scratch of every gw_superstep_static call on this device.  In host code
// this name is only a stand-in for the symbol; the device address comes from
// cudaGetSymbolAddress (static_scratch_address below).
static __device__ __align__(256) unsigned char g_superstep_scratch[kStaticBytes];

// Per-device address of g_superstep_scratch, looked up once per device with
// that device current.
constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
void* g_addr[kMaxDevices] = {};

cudaError_t static_scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_superstep_scratch);
    if (e != cudaSuccess) return e;
    g_addr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_addr[device]);
  return cudaSuccess;
}

// Exclusive scan of the bucket-major tile histogram in one CTA, then the
// bucket starts: offsets[d] (first moved walk of destination d), and the
// per-bucket output pointers the partition scatter writes through.
constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads)
    static_scan_kernel(const uint32_t* __restrict__ hist, uint32_t* __restrict__ off, uint32_t m,
                       uint32_t nbuckets, uint32_t ntiles, gw_walk_rec* moved,
                       gw_walk_rec** __restrict__ out_ptr, uint64_t* __restrict__ out_base,
                       uint32_t* __restrict__ offsets) {
  __shared__ uint32_t warp_sum[kScanThreads / 32];
  const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint32_t chunk = (m + kScanThreads - 1) / kScanThreads;
  const uint32_t lo = min(m, t * chunk), hi = min(m, lo + chunk);
  uint32_t sum = 0;
  for (uint32_t i = lo; i < hi; ++i) sum += hist[i];
  // inclusive scan of the per-thread sums: inside each warp, then across warps
  uint32_t x = sum;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= (uint32_t)d) x += y;
  }
  if (lane == 31) warp_sum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = warp_sum[lane];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
      if (lane >= (uint32_t)d) w += y;
    }
    warp_sum[lane] = w;
  }
  __syncthreads();
  uint32_t run = x - sum + (warp ? warp_sum[warp - 1] : 0u);  // exclusive prefix of this thread
  for (uint32_t i = lo; i < hi; ++i) {
    off[i] = run;
    run += hist[i];
  }
  __syncthreads();
  for (uint32_t d = t; d < nbuckets; d += kScanThreads) {
    const uint32_t start = off[(uint64_t)d * ntiles];
    offsets[d] = start;
    out_ptr[d] = d + 1 < nbuckets ? moved + start : nullptr;
    out_base[d] = 0;
  }
}

}  // namespace
}  // namespace gw

extern "C" gw_status gw_superstep_static(gw_ctx* ctx, const gw_walk_params* params, uint32_t block,
                                         gw_walk_rec* d_walks, uint64_t n, uint32_t* d_counts,
                                         gw_walk_rec* d_moved, uint32_t* d_offsets,
                                         uint32_t* d_minhop, void* stream) {
  using namespace gw;
  if (!ctx) return GW_E_INVALID;
  if (ctx->residency != GW_RESIDENT_HBM)
    return ctx->fail(GW_E_STATE, "gw_superstep_static needs a graph resident in HBM");
  if (block >= ctx->nblocks) return ctx->fail(GW_E_INVALID, "block %u >= nblocks %u", block, ctx->nblocks);
  if (ctx->nblocks > kStaticMaxBlocks)
    return ctx->fail(GW_E_INVALID, "gw_superstep_static handles at most %u blocks (graph has %u)",
                     kStaticMaxBlocks, ctx->nblocks);
  if (n > kStaticMaxWalks)
    return ctx->fail(GW_E_INVALID, "gw_superstep_static handles at most %llu walks per call (got %llu)",
                     (unsigned long long)kStaticMaxWalks, (unsigned long long)n);
  if ((n && (!d_walks || !d_moved)) || !d_offsets || !d_minhop)
    return ctx->fail(GW_E_INVALID, "gw_superstep_static: NULL buffer");
  if (params && params->sink == GW_SINK_VERTEX_COUNT && !d_counts)
    return ctx->fail(GW_E_INVALID, "d_counts is NULL");
  if (params && params->sink != GW_SINK_VERTEX_COUNT && params->sink != GW_SINK_NONE)
    return ctx->fail(GW_E_INVALID, "gw_superstep_static supports the NONE and VERTEX_COUNT sinks");
  WalkArgs a;
  gw_status s = make_walk_args(ctx, params, &a);
  if (s != GW_OK) return s;
  a.lo = ctx->blocks[block];
  a.hi = ctx->blocks[block + 1];
  cudaStream_t st = (cudaStream_t)stream;  // NULL = the default stream

  GW_CUDA(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
  unsigned char* base = nullptr;
  GW_CUDA(ctx, static_scratch_address(ctx->device, &base), "cudaGetSymbolAddress(scratch)");
  uint32_t* dest = reinterpret_cast<uint32_t*>(base + kOffDest);
  uint32_t* tile_hist = reinterpret_cast<uint32_t*>(base + kOffHist);
  uint32_t* tile_off = reinterpret_cast<uint32_t*>(base + kOffTileOff);
  uint32_t* minhop = reinterpret_cast<uint32_t*>(base + kOffMinhop);
  gw_walk_rec** out_ptr = reinterpret_cast<gw_walk_rec**>(base + kOffPtr);
  uint64_t* out_base = reinterpret_cast<uint64_t*>(base + kOffBase);

  const uint32_t nbk = ctx->nblocks + 1;
  PartitionPlan plan;
  plan.nbuckets = nbk;
  plan.ntiles = (uint32_t)((n + kStaticWarpTile - 1) / kStaticWarpTile);
  if (plan.ntiles == 0) plan.ntiles = 1;
  plan.scan_temp_bytes = 0;

  SinkView sv{};
  sv.counts = d_counts;
  // minhop starts at "no walk": the previous call left its own values there
  GW_CUDA(ctx, cudaMemsetAsync(minhop, 0xff, nbk * sizeof(uint32_t), st), "clear minhop");
  if (n) {
    GW_CUDA(ctx, launch_walk_block((int)params->rule, (int)params->sink, params->aggregate != 0, d_walks, n,
                                   ctx->view(), nullptr, nullptr, a, sv, ctx->d_blocks.as<uint32_t>(),
                                   ctx->nblocks, dest, ctx->d_status.as<uint32_t>(), st),
            "advance");
  }
  // every (bucket, tile) histogram entry is written, so no clearing is needed
  GW_CUDA(ctx, launch_partition_hist(d_walks, dest, n, plan, tile_hist, minhop, st), "histogram");
  static_scan_kernel<<<1, kScanThreads, 0, st>>>(tile_hist, tile_off, plan.nbuckets * plan.ntiles,
                                                 plan.nbuckets, plan.ntiles, d_moved, out_ptr, out_base,
                                                 d_offsets);
  GW_CUDA(ctx, cudaGetLastError(), "scan");
  GW_CUDA(ctx, launch_partition_scatter(d_walks, dest, n, plan, tile_off, out_ptr, out_base, st), "scatter");
  GW_CUDA(ctx, cudaMemcpyAsync(d_minhop, minhop, ctx->nblocks * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st),
          "minhop out");
  return GW_OK;
}
