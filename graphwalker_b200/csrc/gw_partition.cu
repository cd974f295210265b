// gw_partition.cu -- stable on-device partition of walks by destination block.
//
// Replaces WalkManager::moveWalk + WalkBuffer::push_back + the per-block
// pools (src/walks/walk.hpp:93-137, src/walks/walkbuffer.hpp:32-39).  The
// reference appends each exiting walk to a per-(thread, block) buffer, so the
// order inside a pool depends on the thread schedule; here the order is
// defined: a destination pool receives the walks of a superstep in input
// order (a stable counting sort over one digit = the destination block).
//
// Tiling: one warp owns one tile of kPartTile walks, processed in rows of 32
// lanes; stability inside a tile comes from a warp match on the destination
// and the rank among lower lanes, across tiles from an exclusive scan over a
// bucket-major histogram.
#include <algorithm>

#include <cub/device/device_scan.cuh>

#include "gw_internal.h"

namespace gw {

namespace {

constexpr int kWarpsPerCta = kPartThreads / 32;
constexpr uint32_t kWarpTile = kPartTile / kWarpsPerCta;  // walks per warp tile

__global__ void __launch_bounds__(kPartThreads)
    partition_hist_kernel(const gw_walk_rec* __restrict__ walks, const uint32_t* __restrict__ dest,
                          uint64_t n, uint32_t nbuckets, uint32_t ntiles,
                          uint32_t* __restrict__ tile_hist, uint32_t* __restrict__ minhop) {
  extern __shared__ uint32_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* hist = smem + warp * nbuckets;             // per-warp histogram
  uint32_t* mh = smem + kWarpsPerCta * nbuckets;       // per-CTA min hop
  for (uint32_t b = threadIdx.x; b < nbuckets * kWarpsPerCta; b += blockDim.x) smem[b] = 0;
  for (uint32_t b = threadIdx.x; b < nbuckets; b += blockDim.x) mh[b] = 0xffffffffu;
  __syncthreads();
  const uint64_t tile = (uint64_t)blockIdx.x * kWarpsPerCta + warp;
  const uint64_t base = tile * kWarpTile;
  for (uint32_t r = 0; r < kWarpTile; r += 32) {
    const uint64_t i = base + r + lane;
    if (i < n) {
      const uint32_t d = dest[i];
      atomicAdd(hist + d, 1u);
      if (d + 1 < nbuckets) atomicMin(mh + d, walks[i].hop);
    }
  }
  __syncthreads();
  if (tile < ntiles) {
    for (uint32_t b = lane; b < nbuckets; b += 32) tile_hist[(uint64_t)b * ntiles + tile] = hist[b];
  }
  for (uint32_t b = threadIdx.x; b < nbuckets; b += blockDim.x)
    if (mh[b] != 0xffffffffu) atomicMin(minhop + b, mh[b]);
}

__global__ void partition_totals_kernel(const uint32_t* __restrict__ tile_hist,
                                        const uint32_t* __restrict__ tile_off, uint32_t nbuckets,
                                        uint32_t ntiles, uint32_t* __restrict__ totals,
                                        uint32_t* __restrict__ minhop_src,
                                        uint32_t* __restrict__ minhop_dst) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nbuckets;
       b += gridDim.x * blockDim.x) {
    const uint64_t first = (uint64_t)b * ntiles, last = first + ntiles - 1;
    totals[b] = tile_off[last] + tile_hist[last] - tile_off[first];
    if (minhop_src) {  // hand the minimum hops over and reset them for the next histogram
      minhop_dst[b] = minhop_src[b];
      minhop_src[b] = 0xffffffffu;
    }
  }
}

__global__ void fetch_u64_pair_kernel(const uint64_t* src_a, uint64_t* __restrict__ dst_a,
                                      const uint64_t* src_b, uint64_t* __restrict__ dst_b, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    dst_a[i] = src_a[i];
    dst_b[i] = src_b[i];
  }
}

__global__ void __launch_bounds__(kPartThreads)
    partition_scatter_kernel(const gw_walk_rec* __restrict__ walks,
                             const uint32_t* __restrict__ dest, uint64_t n, uint32_t nbuckets,
                             uint32_t ntiles, const uint32_t* __restrict__ tile_off,
                             gw_walk_rec* const* __restrict__ out_ptr,
                             const uint64_t* __restrict__ out_base) {
  extern __shared__ uint64_t run64[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* running = run64 + (uint64_t)warp * nbuckets;
  const uint64_t tile = (uint64_t)blockIdx.x * kWarpsPerCta + warp;
  if (tile >= ntiles) return;
  for (uint32_t b = lane; b < nbuckets; b += 32) {
    const uint64_t row = (uint64_t)b * ntiles;
    running[b] = (uint64_t)(tile_off[row + tile] - tile_off[row]) + out_base[b];
  }
  __syncwarp();
  const uint64_t base = tile * kWarpTile;
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t r = 0; r < kWarpTile; r += 32) {
    const uint64_t i = base + r + lane;
    const bool ok = i < n;
    const uint32_t d = ok ? dest[i] : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    if (ok) {
      const uint64_t pos = running[d] + __popc(peers & lt);
      if (d + 1 < nbuckets) {
        const uint4 w = *(reinterpret_cast<const uint4*>(walks) + i);
        *(reinterpret_cast<uint4*>(out_ptr[d]) + pos) = w;
      }
    }
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) running[d] += __popc(peers);
    __syncwarp();
  }
}

}  // namespace

PartitionPlan partition_plan(uint64_t n, uint32_t nbuckets) {
  PartitionPlan p;
  p.nbuckets = nbuckets;
  p.ntiles = (uint32_t)((n + kWarpTile - 1) / kWarpTile);
  if (p.ntiles == 0) p.ntiles = 1;
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                (int64_t)nbuckets * p.ntiles);
  p.scan_temp_bytes = bytes;
  return p;
}

static uint32_t ctas_for(const PartitionPlan& p) {
  return (p.ntiles + kWarpsPerCta - 1) / kWarpsPerCta;
}

cudaError_t launch_partition_hist(const gw_walk_rec* walks, const uint32_t* dest, uint64_t n,
                                  const PartitionPlan& plan, uint32_t* tile_hist,
                                  uint32_t* minhop, cudaStream_t stream) {
  const size_t smem = (size_t)(kWarpsPerCta + 1) * plan.nbuckets * sizeof(uint32_t);
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(partition_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  partition_hist_kernel<<<ctas_for(plan), kPartThreads, smem, stream>>>(
      walks, dest, n, plan.nbuckets, plan.ntiles, tile_hist, minhop);
  return cudaGetLastError();
}

cudaError_t launch_partition_scan(const uint32_t* tile_hist, uint32_t* tile_off, uint32_t* totals,
                                  const PartitionPlan& plan, void* temp, cudaStream_t stream,
                                  uint32_t* minhop_src, uint32_t* minhop_dst) {
  size_t bytes = plan.scan_temp_bytes;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(temp, bytes, tile_hist, tile_off,
                                                (int64_t)plan.nbuckets * plan.ntiles, stream);
  if (e != cudaSuccess) return e;
  partition_totals_kernel<<<(plan.nbuckets + 255) / 256, 256, 0, stream>>>(
      tile_hist, tile_off, plan.nbuckets, plan.ntiles, totals, minhop_src, minhop_dst);
  return cudaGetLastError();
}

cudaError_t launch_fetch_u64_pair(const uint64_t* src_a, uint64_t* dst_a, const uint64_t* src_b,
                                  uint64_t* dst_b, uint32_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const uint32_t grid = std::min<uint32_t>((n + 255) / 256, 64);
  fetch_u64_pair_kernel<<<grid, 256, 0, stream>>>(src_a, dst_a, src_b, dst_b, n);
  return cudaGetLastError();
}

cudaError_t launch_partition_scatter(const gw_walk_rec* walks, const uint32_t* dest, uint64_t n,
                                     const PartitionPlan& plan, const uint32_t* tile_off,
                                     gw_walk_rec* const* out_ptr, const uint64_t* out_base,
                                     cudaStream_t stream) {
  const size_t smem = (size_t)kWarpsPerCta * plan.nbuckets * sizeof(uint64_t);
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(partition_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  partition_scatter_kernel<<<ctas_for(plan), kPartThreads, smem, stream>>>(
      walks, dest, n, plan.nbuckets, plan.ntiles, tile_off, out_ptr, out_base);
  return cudaGetLastError();
}

}  // namespace gw
