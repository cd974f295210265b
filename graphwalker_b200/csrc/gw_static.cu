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

// Address of g_superstep_scratch in the current device's context.  The
// lookup runs once per (device, context) with that device current, and again
// if the device's context changes (after cudaDeviceReset, the primary context
// is recreated and the array gets a new address).  The driver's context handle
// comes through the runtime's driver entry point, so the library needs no
// link to libcuda.  The first lookup on a device must not happen during a
// stream capture.
constexpr int kMaxDevices = 64;
struct ScratchSlot {
  void* ctx = nullptr;
  void* addr = nullptr;
};
std::mutex g_addr_mutex;
ScratchSlot g_addr[kMaxDevices];

typedef int (*CtxGetCurrentFn)(void**);  // CUresult cuCtxGetCurrent(CUcontext*)

void* current_context() {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  void* c = nullptr;
  if (!fn || fn(&c) != 0) return nullptr;
  return c;
}

cudaError_t static_scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  // the caller has made `device` current (cudaSetDevice initialises its
  // primary context), so the driver's current context is that device's
  void* const cur = current_context();
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  ScratchSlot& slot = g_addr[device];
  if (!slot.addr || !cur || slot.ctx != cur) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_superstep_scratch);
    if (e != cudaSuccess) return e;
    slot.addr = p;
    slot.ctx = cur;
  }
  *out = static_cast<unsigned char*>(slot.addr);
  return cudaSuccess;
}

// Keeps the calling thread's current device across a call that switches to
// the context's device.
struct DeviceGuard {
  int saved = -1;
  DeviceGuard() {
    if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
  }
  ~DeviceGuard() {
    if (saved >= 0) cudaSetDevice(saved);
  }
};

// Exclusive scan of the bucket-major tile histogram in one CTA, then the
// bucket starts: offsets[d] (first moved walk of destination d), and the
// per-bucket output pointers the partition scatter writes through.  Each warp
// owns one contiguous segment of the histogram and reads it in rows of 32
// consecutive entries (coalesced): once to total the segment, and once more,
// after the segment totals are scanned, to write the offsets.
constexpr int kScanThreads = 1024;
constexpr int kScanWarps = kScanThreads / 32;

__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t x, uint32_t lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= (uint32_t)d) x += y;
  }
  return x;
}

__global__ void __launch_bounds__(kScanThreads)
    static_scan_kernel(const uint32_t* __restrict__ hist, uint32_t* __restrict__ off, uint32_t m,
                       uint32_t nbuckets, uint32_t ntiles, gw_walk_rec* moved,
                       gw_walk_rec** __restrict__ out_ptr, uint64_t* __restrict__ out_base,
                       uint32_t* __restrict__ offsets) {
  __shared__ uint32_t seg_base[kScanWarps];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t seg = ((m + kScanWarps - 1) / kScanWarps + 31) & ~31u;  // whole rows per warp
  const uint32_t lo = min(m, warp * seg), hi = min(m, lo + seg);
  uint32_t part = 0;
  for (uint32_t i = lo + lane; i < hi; i += 32) part += hist[i];
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) part += __shfl_xor_sync(0xffffffffu, part, d);
  if (lane == 0) seg_base[warp] = part;
  __syncthreads();
  if (warp == 0) {
    const uint32_t t = seg_base[lane];
    const uint32_t incl = warp_inclusive_scan(t, lane);
    seg_base[lane] = incl - t;
  }
  __syncthreads();
  uint32_t carry = seg_base[warp];
  for (uint32_t row = lo; row < hi; row += 32) {
    const uint32_t i = row + lane;
    const uint32_t h = i < hi ? hist[i] : 0u;
    const uint32_t incl = warp_inclusive_scan(h, lane);
    if (i < hi) off[i] = carry + incl - h;
    carry += __shfl_sync(0xffffffffu, incl, 31);
  }
  __syncthreads();
  for (uint32_t d = threadIdx.x; d < nbuckets; d += kScanThreads) {
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

  DeviceGuard keep_device;  // the caller's current device is restored on return
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
