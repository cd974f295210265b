// gw_simrank.cu -- SimRank's meeting reduction on the device: the triple loop
// of SimRank::computeResult (apps/simrank.cpp:71-84).  For every pair (i, j)
// of the R walks from a and the R walks from b, the first position l < L at
// which both walks stand on the same vertex (0xFFFFFFFF = no visit never
// matches); meet[l] counts the pairs.  The app's estimate is
// sum_l meet[l] * 0.8^l / R^2.
//
// The host loop is O(R^2 L).  Here a CTA takes a 64 x 64 tile of pairs: the
// two tiles' visits are staged in shared memory 32 positions at a time, each
// thread owns a 4 x 4 block of pairs and keeps their "met" flags in a 16-bit
// mask, so positions beyond a pair's first meeting are skipped by masking.
// The grid's z dimension runs over queries: query q compares the R walks at
// row offset rows[2q] of `a` with those at rows[2q + 1] of `b`.
#include "gw_internal.h"

namespace gw {

namespace {

constexpr int kSrTile = 64;      // walks per tile side
constexpr int kSrChunk = 32;     // positions staged at a time
constexpr int kSrThreads = 256;  // 16 x 16 threads, 4 x 4 pairs each

__global__ void __launch_bounds__(kSrThreads)
    simrank_meet_kernel(const uint32_t* __restrict__ a0, const uint32_t* __restrict__ b0,
                        const unsigned long long* __restrict__ rows, uint32_t q0, uint32_t R, uint32_t L,
                        unsigned long long* __restrict__ meet0) {
  __shared__ uint32_t sa[kSrChunk][kSrTile + 1];
  __shared__ uint32_t sb[kSrChunk][kSrTile + 1];
  __shared__ uint32_t hist[kSrChunk];
  const uint32_t q = q0 + blockIdx.z;
  const uint32_t* __restrict__ a = a0 + (rows ? rows[2 * (size_t)q] : 0ull);
  const uint32_t* __restrict__ b = b0 + (rows ? rows[2 * (size_t)q + 1] : 0ull);
  unsigned long long* __restrict__ meet = meet0 + (size_t)q * L;
  const uint32_t i0 = blockIdx.y * kSrTile, j0 = blockIdx.x * kSrTile;
  const uint32_t tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  uint32_t met = 0;  // bit u * 4 + w: pair (i0 + ty + 16u, j0 + tx + 16w) has met
  for (uint32_t l0 = 0; l0 < L; l0 += kSrChunk) {
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < kSrTile * kSrChunk; x += kSrThreads) {
      const uint32_t r = x / kSrChunk, c = x % kSrChunk;  // walk r of the tile, position l0 + c
      const bool in_l = l0 + c < L;
      sa[c][r] = in_l && i0 + r < R ? __ldg(a + (size_t)(i0 + r) * L + l0 + c) : 0xffffffffu;
      sb[c][r] = in_l && j0 + r < R ? __ldg(b + (size_t)(j0 + r) * L + l0 + c) : 0xffffffffu;
    }
    if (threadIdx.x < kSrChunk) hist[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t lend = L - l0 < (uint32_t)kSrChunk ? L - l0 : (uint32_t)kSrChunk;
    for (uint32_t c = 0; c < lend && met != 0xffffu; ++c) {
      uint32_t va[4], vb[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        va[u] = sa[c][ty + 16 * u];
        vb[u] = sb[c][tx + 16 * u];
      }
      uint32_t now = 0;
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int w = 0; w < 4; ++w)
          now |= (va[u] == vb[w] && va[u] != 0xffffffffu ? 1u : 0u) << (u * 4 + w);
      now &= ~met;
      if (now) {
        atomicAdd(&hist[c], (uint32_t)__popc(now));
        met |= now;
      }
    }
    __syncthreads();
    if (threadIdx.x < lend && hist[threadIdx.x]) atomicAdd(meet + l0 + threadIdx.x, (unsigned long long)hist[threadIdx.x]);
  }
}

// The app's placement (simrank.cpp:30-57): replica i of vertex v starts at v
// with hop i*L, keyed on v; walk k * R + i is replica i of verts[k].
__global__ void simrank_walks_kernel(const uint32_t* __restrict__ verts, uint64_t n, uint32_t R, uint32_t L,
                                     gw_walk_rec* __restrict__ out) {
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n; w += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = __ldg(verts + w / R), i = (uint32_t)(w % R);
    reinterpret_cast<uint4*>(out)[w] = make_uint4(v, v, v, i * L);
  }
}

}  // namespace

cudaError_t launch_simrank_walks(const uint32_t* verts, uint32_t nverts, uint32_t R, uint32_t L, gw_walk_rec* out,
                                 cudaStream_t stream) {
  const uint64_t n = (uint64_t)nverts * R;
  if (n == 0) return cudaSuccess;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t need = (n + 255) / 256, cap = (uint64_t)sms * 16;
  simrank_walks_kernel<<<(unsigned)(need < cap ? need : cap), 256, 0, stream>>>(verts, n, R, L, out);
  return cudaGetLastError();
}

cudaError_t launch_simrank_meet(const uint32_t* a, const uint32_t* b, const unsigned long long* rows, uint32_t nq,
                                uint32_t R, uint32_t L, unsigned long long* meet, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(meet, 0, (size_t)nq * L * sizeof(unsigned long long), stream);
  if (e != cudaSuccess || R == 0 || L == 0) return e;
  const uint32_t tiles = (R + kSrTile - 1) / kSrTile;
  for (uint32_t q0 = 0; q0 < nq && e == cudaSuccess; q0 += 65535u) {
    const uint32_t nz = nq - q0 < 65535u ? nq - q0 : 65535u;
    simrank_meet_kernel<<<dim3(tiles, tiles, nz), kSrThreads, 0, stream>>>(a, b, rows, q0, R, L, meet);
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace gw
