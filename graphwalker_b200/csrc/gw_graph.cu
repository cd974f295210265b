// gw_graph.cu -- graph layout kernels.
//
// * Packed vertex records for the resident walk kernel.
// * Seeded R-MAT generation and CSR construction on the device (the
//   synthetic stand-in for the reference's datasets; its text preprocessor
//   is convert_to_csr, src/preprocess/conversions.hpp:181-298: self-loops
//   dropped, duplicates kept, one global CSR with u64 row pointer and u32
//   column ids).  Rows are sorted by (src, dst).
#include <cub/device/device_radix_sort.cuh>

#include "gw_internal.h"

namespace gw {

namespace {

__global__ void build_vrec_kernel(const unsigned long long* __restrict__ rowptr, uint32_t nv,
                                  unsigned long long* __restrict__ vrec) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long b = rowptr[v], e = rowptr[v + 1];
    unsigned long long deg = e - b;
    if (deg > kDegEscape || b >= (1ull << (64 - kDegBits))) deg = kDegEscape;
    vrec[v] = (b << kDegBits) | deg;
  }
}

// Out-edge bitmap: word w holds the bits of vertices 32w .. 32w + 31.
__global__ void build_out_bits_kernel(const unsigned long long* __restrict__ rowptr, uint32_t nv,
                                      uint32_t* __restrict__ bits) {
  const uint64_t nw = ((uint64_t)nv + 31) / 32;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw;
       w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t x = 0;
    const uint64_t v0 = w * 32;
    for (uint32_t j = 0; j < 32 && v0 + j < nv; ++j)
      x |= (rowptr[v0 + j + 1] > rowptr[v0 + j] ? 1u : 0u) << j;
    bits[w] = x;
  }
}

struct RmatArgs {
  uint32_t scale, mask, half;
  uint32_t key0, key1;
  uint32_t ta, tab, tabc;
  uint32_t pk[4], pm[4];  // permutation round keys and odd multipliers
};

__device__ __forceinline__ uint32_t rmat_permute(uint32_t x, const RmatArgs& r) {
  x &= r.mask;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    x = (x ^ r.pk[k]) & r.mask;
    x = (x * r.pm[k]) & r.mask;
    if (r.half > 0 && r.half < 32) x ^= x >> r.half;
  }
  return x;
}

__global__ void rmat_keys_kernel(uint64_t m, RmatArgs r, unsigned long long* __restrict__ keys,
                                 unsigned long long* __restrict__ nself) {
  uint32_t self = 0;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s = 0, d = 0;
    for (uint32_t l = 0; l < r.scale; l += 4) {
      const Philox4 p = philox4x32_10((uint32_t)e, (uint32_t)(e >> 32), l >> 2, 0u, r.key0, r.key1);
      const uint32_t u[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
      for (uint32_t j = 0; j < 4; ++j) {
        if (l + j < r.scale) {
          const uint32_t bit = 1u << (r.scale - 1 - (l + j));
          const uint32_t x = u[j];
          if (x < r.ta) {
          } else if (x < r.tab) {
            d |= bit;
          } else if (x < r.tabc) {
            s |= bit;
          } else {
            s |= bit;
            d |= bit;
          }
        }
      }
    }
    s = rmat_permute(s, r);
    d = rmat_permute(d, r);
    if (s == d) {
      ++self;
      keys[e] = (unsigned long long)(r.mask + 1ull) << 32;  // sorts after every kept edge
    } else {
      keys[e] = ((unsigned long long)s << 32) | d;
    }
  }
  if (self) atomicAdd(nself, (unsigned long long)self);
}

// rowptr[v] = first sorted position whose source is >= v.
__global__ void rowptr_from_sorted_kernel(const unsigned long long* __restrict__ keys,
                                          uint64_t kept, uint32_t nv,
                                          unsigned long long* __restrict__ rowptr,
                                          uint32_t* __restrict__ colidx) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j <= kept;
       j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t sj = j < kept ? (keys[j] >> 32) : (uint64_t)nv;
    const uint64_t sp = j > 0 ? (keys[j - 1] >> 32) + 1 : 0;
    for (uint64_t v = sp; v <= sj && v <= nv; ++v) rowptr[v] = j;
    if (j < kept) colidx[j] = (uint32_t)keys[j];
  }
}

uint64_t splitmix64(uint64_t x) {  // Steele, Lea, Flood (OOPSLA'14)
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

int grid_for(uint64_t n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t need = (n + 255) / 256;
  const uint64_t cap = (uint64_t)sms * 16;
  return (int)(need < cap ? (need ? need : 1) : cap);
}

}  // namespace

cudaError_t launch_build_vrec(const unsigned long long* rowptr, uint32_t nv,
                              unsigned long long* vrec, cudaStream_t stream) {
  if (nv == 0) return cudaSuccess;
  build_vrec_kernel<<<grid_for(nv), 256, 0, stream>>>(rowptr, nv, vrec);
  build_out_bits_kernel<<<grid_for((nv + 31) / 32), 256, 0, stream>>>(rowptr, nv,
                                                                      reinterpret_cast<uint32_t*>(vrec + nv));
  return cudaGetLastError();
}

#define GW_TRY(x)                          \
  do {                                     \
    cudaError_t _e = (x);                  \
    if (_e != cudaSuccess) {               \
      err = _e;                            \
      goto done;                           \
    }                                      \
  } while (0)

cudaError_t launch_rowptr_from_sorted(const unsigned long long* keys, uint64_t n, uint32_t nv,
                                      unsigned long long* rowptr, uint32_t* colidx, cudaStream_t stream) {
  rowptr_from_sorted_kernel<<<grid_for(n + 1), 256, 0, stream>>>(keys, n, nv, rowptr, colidx);
  return cudaGetLastError();
}

cudaError_t rmat_build_csr(uint32_t scale, uint64_t nedges_raw, uint64_t seed, uint32_t ta,
                           uint32_t tab, uint32_t tabc, unsigned long long** rowptr_out,
                           uint32_t** colidx_out, uint64_t* nedges, cudaStream_t stream) {
  cudaError_t err = cudaSuccess;
  unsigned long long *keys = nullptr, *sorted = nullptr, *nself = nullptr, *rowptr = nullptr;
  uint32_t* colidx = nullptr;
  void* temp = nullptr;
  size_t temp_bytes = 0;
  unsigned long long h_self = 0;
  uint64_t kept = 0;
  const uint32_t nv = scale >= 32 ? 0xffffffffu : (1u << scale);
  RmatArgs r;
  r.scale = scale;
  r.mask = scale >= 32 ? 0xffffffffu : ((1u << scale) - 1u);
  r.half = (scale + 1) / 2;
  r.key0 = (uint32_t)seed;
  r.key1 = (uint32_t)(seed >> 32) ^ 0x524D4154u;  // "RMAT"
  r.ta = ta;
  r.tab = tab;
  r.tabc = tabc;
  for (uint32_t k = 0; k < 4; ++k) {
    const uint64_t x = splitmix64(seed ^ (0x5045524Dull + k));  // "PERM" + round
    r.pk[k] = (uint32_t)x;
    r.pm[k] = (uint32_t)(x >> 32) | 1u;
  }
  *rowptr_out = nullptr;
  *colidx_out = nullptr;
  if (scale == 0 || scale > 31) return cudaErrorInvalidValue;
  const uint64_t m = nedges_raw;
  GW_TRY(cudaMalloc(&keys, (m ? m : 1) * sizeof(unsigned long long)));
  GW_TRY(cudaMalloc(&sorted, (m ? m : 1) * sizeof(unsigned long long)));
  GW_TRY(cudaMalloc(&nself, sizeof(unsigned long long)));
  GW_TRY(cudaMemsetAsync(nself, 0, sizeof(unsigned long long), stream));
  if (m) {
    rmat_keys_kernel<<<grid_for(m), 256, 0, stream>>>(m, r, keys, nself);
    GW_TRY(cudaGetLastError());
  }
  GW_TRY(cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, keys, sorted, (int64_t)m, 0,
                                        (int)(32 + scale + 1), stream));
  GW_TRY(cudaMalloc(&temp, temp_bytes ? temp_bytes : 1));
  GW_TRY(cub::DeviceRadixSort::SortKeys(temp, temp_bytes, keys, sorted, (int64_t)m, 0,
                                        (int)(32 + scale + 1), stream));
  GW_TRY(cudaMemcpyAsync(&h_self, nself, sizeof(h_self), cudaMemcpyDeviceToHost, stream));
  GW_TRY(cudaStreamSynchronize(stream));
  cudaFree(temp);
  temp = nullptr;
  cudaFree(keys);
  keys = nullptr;
  kept = m - h_self;
  GW_TRY(cudaMalloc(&rowptr, ((uint64_t)nv + 1) * sizeof(unsigned long long)));
  GW_TRY(cudaMalloc(&colidx, (kept ? kept : 1) * sizeof(uint32_t)));
  rowptr_from_sorted_kernel<<<grid_for(kept + 1), 256, 0, stream>>>(sorted, kept, nv, rowptr,
                                                                    colidx);
  GW_TRY(cudaGetLastError());
  GW_TRY(cudaStreamSynchronize(stream));
  *rowptr_out = rowptr;
  *colidx_out = colidx;
  *nedges = kept;
  rowptr = nullptr;
  colidx = nullptr;
done:
  if (keys) cudaFree(keys);
  if (sorted) cudaFree(sorted);
  if (nself) cudaFree(nself);
  if (temp) cudaFree(temp);
  if (rowptr) cudaFree(rowptr);
  if (colidx) cudaFree(colidx);
  return err;
}

}  // namespace gw
